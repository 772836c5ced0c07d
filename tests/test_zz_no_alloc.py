"""GPU test of p3mx_error_estimate_noalloc, the allocation-free entry point.

Some host programs cannot allocate device memory while they run (engines
that give all GPU memory to their own pool at start-up, or loops that cannot
take the synchronisation cudaMalloc/cudaFree may imply).  The no-alloc entry
point serves them: it computes the same real- and k-space error estimate as
p3mx_error_estimate, keeping its scratch in a fixed device array inside the
library.  This file runs last so a failure here never hides another test's
result; it passes on its own in a fresh process and after the full suite.
"""
import ctypes

import numpy as np
import pytest

from espresso_b200 import _lib

pytestmark = pytest.mark.gpu

_P = ctypes.POINTER


def _noalloc(mesh, cao, n_c, sum_q2, alpha_L, r_cut_iL, box, pref):
    lib = _lib.load()
    m = np.ascontiguousarray(np.broadcast_to(mesh, (3,)), dtype=np.int32)
    b = np.ascontiguousarray(np.broadcast_to(box, (3,)), dtype=np.float64)
    rs, ks = ctypes.c_double(), ctypes.c_double()
    err = ctypes.create_string_buffer(256)
    rc = lib.p3mx_error_estimate_noalloc(m.ctypes.data_as(_P(ctypes.c_int)), cao, n_c, sum_q2,
                                         alpha_L, r_cut_iL, b.ctypes.data_as(_P(ctypes.c_double)),
                                         pref, ctypes.byref(rs), ctypes.byref(ks), None, err,
                                         len(err))
    return rc, rs.value, ks.value, err.value.decode()


def _existing(mesh, cao, n_c, sum_q2, alpha_L, r_cut_iL, box, pref):
    lib = _lib.load()
    m = np.ascontiguousarray(np.broadcast_to(mesh, (3,)), dtype=np.int32)
    b = np.ascontiguousarray(np.broadcast_to(box, (3,)), dtype=np.float64)
    rs, ks = ctypes.c_double(), ctypes.c_double()
    rc = lib.p3mx_error_estimate(m.ctypes.data_as(_P(ctypes.c_int)), cao, n_c, sum_q2, alpha_L,
                                 r_cut_iL, b.ctypes.data_as(_P(ctypes.c_double)), pref,
                                 ctypes.byref(rs), ctypes.byref(ks))
    assert rc == 0
    return rs.value, ks.value


def test_noalloc_matches_existing_entry_point_on_consecutive_calls():
    # a large mesh first, then a smaller one: the second call must ignore the
    # partial sums the first one left in the shared array
    cases = [((128, 128, 128), 7, 1 << 20, float(1 << 20), 110.0, 0.03, (128.0,) * 3, 1.0),
             ((32, 32, 32), 5, 2000, 2000.0, 12.0, 0.15, (20.0,) * 3, 1.0)]
    for case in cases:
        rc, rs, ks, msg = _noalloc(*case)
        assert rc == 0, msg
        rs0, ks0 = _existing(*case)
        # same kernel, different number of partial sums: FP64 rounding only
        np.testing.assert_allclose(ks, ks0, rtol=1e-10, atol=0)
        np.testing.assert_allclose(rs, rs0, rtol=1e-14, atol=0)
        assert ks > 0.0


def test_noalloc_at_its_largest_mesh():
    # 256 x 256 x 1024 = 4096 * 16384 points: every one of the 4096 partial
    # sums is written, and the final sum's strided loop covers all of them
    case = ((256, 256, 1024), 7, 1 << 20, float(1 << 20), 110.0, 0.03, (128.0, 128.0, 512.0), 1.0)
    for _ in range(2):
        rc, rs, ks, msg = _noalloc(*case)
        assert rc == 0, msg
        rs0, ks0 = _existing(*case)
        np.testing.assert_allclose(ks, ks0, rtol=1e-10, atol=0)
        np.testing.assert_allclose(rs, rs0, rtol=1e-14, atol=0)


def test_noalloc_rejects_meshes_beyond_its_scratch():
    rc, _, _, msg = _noalloc((512, 512, 512), 7, 1000, 1000.0, 50.0, 0.1, (100.0,) * 3, 1.0)
    assert rc == 1
    assert "exceeds the allocation-free maximum" in msg
    # one point over the limit (4096 * 16384 + 1 = 5 * 13421773)
    rc, _, _, msg = _noalloc((5, 13421773, 1), 7, 1000, 1000.0, 50.0, 0.1, (100.0,) * 3, 1.0)
    assert rc == 1
    assert "exceeds the allocation-free maximum" in msg
