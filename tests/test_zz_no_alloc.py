"""The no-allocation band entry point (ifea_band_factor_solve_noalloc) against the allocating one.

Callers whose device memory is owned by their own pooling allocator, or that run a solve inside a loop where
cudaMalloc/cudaFree must not happen, hand in device buffers they already own; the entry point's only working
memory is a fixed device array inside the library. This test calls it twice in a row through the C ABI (the
array keeps the previous call's contents, so the second call checks nothing stale leaks in) and compares each
result with ifea_band_factor_solve on the same system.
"""
import ctypes as C

import numpy as np
import pytest

from impressionfea_b200 import _lib
from impressionfea_b200.forging2d import band_factor_solve

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _spd_band(n, b, seed):
    rng = np.random.default_rng(seed)
    w = b + 1
    a = np.zeros(n * w)
    for i in range(n):
        for j in range(max(0, i - b), i):
            a[i * w + (j - i + b)] = rng.random() - 0.5
        a[i * w + b] = 2.0 * b + 1.0 + rng.random()
    return a, rng.standard_normal(n)


def _noalloc(a, rhs, b):
    import torch

    L = _lib.lib()
    f = L.ifea_band_factor_solve_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_void_p]
    da = torch.tensor(a, dtype=torch.float64, device="cuda")
    dr = torch.tensor(rhs, dtype=torch.float64, device="cuda")
    row, piv = C.c_int32(7), C.c_double(7.0)
    stream = torch.cuda.current_stream().cuda_stream
    st = f(len(rhs), b, C.c_void_p(da.data_ptr()), C.c_void_p(dr.data_ptr()), C.byref(row), C.byref(piv), C.c_void_p(stream))
    return st, row.value, da.cpu().numpy(), dr.cpu().numpy()


def test_noalloc_matches_allocating_entry_on_two_calls_in_a_row():
    for call, (n, b, seed) in enumerate([(900, 85, 11), (400, 40, 12)]):
        a, rhs = _spd_band(n, b, seed)
        L_ref, x_ref = band_factor_solve(a, b, rhs)
        st, row, L_gpu, x_gpu = _noalloc(a, rhs, b)
        assert st == 0 and row == -1, f"call {call + 1}: status {st}, row {row}"
        np.testing.assert_allclose(L_gpu, L_ref, rtol=RTOL, atol=0)
        np.testing.assert_allclose(x_gpu, x_ref, rtol=RTOL, atol=1e-300)


def test_noalloc_reports_non_positive_pivot_and_rejects_oversized_band():
    a = np.zeros(3 * 2)
    a[1], a[3], a[5] = 1.0, -1.0, 1.0
    st, row, _, _ = _noalloc(a, np.ones(3), 1)
    assert st == 4 and row == 1
    n, b = 600, 511  # (b + 1)^2 doubles exceed the fixed scratch array
    st, _, _, _ = _noalloc(np.ones(n * (b + 1)), np.ones(n), b)
    assert st == 1
