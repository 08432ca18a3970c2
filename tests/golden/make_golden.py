"""Generates the golden fixtures of tests/golden/ by running the reference's own
CPU g2g path (oracle/_ref/libg2g_ref.so, built from the reference sources by
oracle/Makefile) on small seeded workloads through its C ABI.

    python tests/golden/make_golden.py

Each fixture stores E_xc, the packed Kohn-Sham matrices, the XC forces of a
g2g_solve_groups_ type 2 call (natoms x 3) and the partition summary (per group: points, functions, a hash-free digest = sum of weights) so
that the C restatement can be checked even where the reference cannot be built.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lio_b200 import workloads as W  # noqa: E402
from tests import helpers as H  # noqa: E402

CASES = {
    "cfg1_lda_vwn": lambda: W.config(1),
    "pbe_closed_12": lambda: W.small_workload(12, 21, 9, False),
    "pbe_open_10": lambda: W.small_workload(10, 31, 9, True),
    "lda_gl_8": lambda: W.small_workload(8, 41, 2, False),
    "slater_6": lambda: W.small_workload(6, 43, 1, False),
    "p86_9": lambda: W.small_workload(9, 205, 4, False),
    "b88_vwn_8": lambda: W.small_workload(8, 207, 6, False),
    "blyp_10": lambda: W.small_workload(10, 208, 7, False),
}


def main():
    for name, make in CASES.items():
        wl = make()
        L = H.lib(H.REF_LIB, False)
        L.init()
        E, K, Kb = H.run(L, wl)
        _, F = L.solve_forces(2)
        # partition summary straight from the reference's groups
        ng = L.num_groups(ref=True)
        npts, wsum, nfun = [], [], []
        for g in range(ng):
            d = L.partition_group(g, ref=True)
            npts.append(d["meta"][0])
            nfun.append(d["meta"][5])
            wsum.append(float(np.sum(d["xyzw"][:, 3])))
        L.deinit()
        order = np.lexsort((np.array(wsum), np.array(nfun), np.array(npts)))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), E=E, K=K, Kb=Kb if wl.open_shell else np.zeros(0), F=F,
                            npts=np.array(npts)[order], nfun=np.array(nfun)[order], wsum=np.array(wsum)[order])
        print(name, E, len(K), ng)


if __name__ == "__main__":
    main()
