"""tcgen05 int8 tensor-core primitive: exact against a host integer product."""
import ctypes as C
import os

import numpy as np
import pytest

from . import helpers as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(16, 32), (64, 64), (48, 96), (128, 256), (256, 128), (208, 224)])
def test_int8_mma_exact(N, K):
    lib = C.CDLL(os.path.join(H.ROOT, "lio_b200", "libg2g_b200.so"))
    rng = np.random.default_rng(N * 1000 + K)
    A = rng.integers(-127, 128, size=(128, K), dtype=np.int8)
    B = rng.integers(-127, 128, size=(N, K), dtype=np.int8)
    D = np.zeros((128, N), dtype=np.int32)
    rc = lib.lio_tc_selftest_(C.c_int(N), C.c_int(K), A.ctypes.data_as(C.c_void_p), B.ctypes.data_as(C.c_void_p),
                              D.ctypes.data_as(C.c_void_p))
    assert rc == 0
    ref = A.astype(np.int64) @ B.astype(np.int64).T
    assert np.array_equal(D.astype(np.int64), ref)
