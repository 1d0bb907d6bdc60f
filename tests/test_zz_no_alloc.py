"""The no-allocation band entry point (ifea_band_factor_solve_noalloc) against the allocating one.

Callers whose device memory is owned by their own pooling allocator, or that run a solve inside a loop where
cudaMalloc/cudaFree must not happen, hand in device buffers they already own; the entry point's working rows sit
in shared memory (or, for a band too wide for that window, in the caller's band) and its status words in a fixed
device array inside the library, shared by every call on a GPU and never cleared between them. These tests call
it through the C ABI several times in a row and compare each result bit for bit with ifea_band_factor_solve on the
same system, or with the reference's band loop (oracle):

- three successful calls in a row: a band factorised in place (too wide for the shared-memory window), a band
  whose circular window is reloaded as the factorisation walks down it, and a band resident as a whole;
- a call that fails on a non-positive pivot followed by a good call, so that the failed call's status words,
  which stay in the array, must not leak into the next result;
- a half-bandwidth of 511 (wider than any shared-memory window), against the reference loop.
"""
import ctypes as C

import numpy as np
import pytest

from impressionfea_b200 import _lib
from impressionfea_b200.forging2d import band_factor_solve
from oracle import OracleBand

pytestmark = pytest.mark.gpu

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
    return st, row.value, piv.value, da.cpu().numpy(), dr.cpu().numpy()


def _check_against_allocating_entry(n, b, seed, label):
    a, rhs = _spd_band(n, b, seed)
    L_ref, x_ref = band_factor_solve(a, b, rhs)
    st, row, _, L_gpu, x_gpu = _noalloc(a, rhs, b)
    assert st == 0 and row == -1, f"{label}: status {st}, row {row}"
    np.testing.assert_array_equal(L_gpu, L_ref, err_msg=label)
    np.testing.assert_array_equal(x_gpu, x_ref, err_msg=label)


def test_noalloc_matches_allocating_entry_on_calls_in_a_row():
    _check_against_allocating_entry(3000, 160, 11, "call 1 (in place: 162-double rows do not fit the window)")
    _check_against_allocating_entry(3000, 60, 14, "call 2 (circular window of 124 rows, reloaded)")
    _check_against_allocating_entry(400, 40, 12, "call 3 (whole band in the window)")


def test_noalloc_good_call_after_a_failed_one_reports_no_stale_status():
    a = np.zeros(3 * 2)
    a[1], a[3], a[5] = 1.0, -1.0, 1.0  # pivot of row 1 is -1 - 0 < 0
    st, row, piv, _, _ = _noalloc(a, np.ones(3), 1)
    assert st == 4 and row == 1 and piv == -1.0
    _check_against_allocating_entry(900, 85, 13, "good call after a NOT_SPD call")


def test_noalloc_wide_band_matches_the_reference_loop():
    n, b = 600, 511
    a, rhs = _spd_band(n, b, 15)
    ob = OracleBand(n, b)
    ob.set_data(a)
    assert ob.factorize()[0] == -1
    x_ref = ob.solve(rhs)
    st, row, _, L_gpu, x_gpu = _noalloc(a, rhs, b)
    assert st == 0 and row == -1
    np.testing.assert_array_equal(L_gpu, ob.data())
    np.testing.assert_array_equal(x_gpu, x_ref)
