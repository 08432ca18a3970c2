"""The drop-in link recipe: a caller with lioamber's link line (this library
first, then the reference's g2g with its analytic integrals) resolves g2g_* to
this library and aint_* to the reference's, and the reference still receives
the state its analytic integrals read (g2g_parameter_init_ is passed on to it).
Runs without a GPU; needs the reference sources (to build its library) and gcc.
"""
import os
import subprocess

import pytest

from . import helpers as H

REF_TREE = os.path.abspath(os.path.join(H.ROOT, os.pardir, "reference"))
pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF_TREE, "g2g")), reason="reference sources absent")


def test_lioamber_link_line_resolves_both_libraries(tmp_path):
    subprocess.run(["make", "-s", "-C", os.path.join(H.ROOT, "oracle"), "full", "REF=" + REF_TREE], check=True)
    prod, ref = os.path.join(H.ROOT, "lio_b200"), os.path.join(H.ROOT, "oracle", "_ref")
    exe = str(tmp_path / "stub")
    subprocess.run(["gcc", "-o", exe, os.path.join(H.ROOT, "tests", "link", "lioamber_stub.c"),
                    "-I", os.path.join(H.ROOT, "include"), "-Wl,--no-as-needed", "-L" + prod, "-lg2g_b200",
                    "-L" + ref, "-llio_g2g_full", "-Wl,-rpath," + prod + ":" + ref, "-ldl"], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    print(out.stdout, out.stderr)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "atoms recorded by the reference's g2g_parameter_init_: 1" in out.stdout
