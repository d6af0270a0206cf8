"""The allocation-free relax entry point against the allocating one (GPU).

cw_field_relax_noalloc is for callers that cannot let the library allocate
device memory (a framework that owns all of it through a caching pool, a
loop that cannot take the device-wide stall of cudaMalloc/cudaFree): they
hand it device buffers they own, and its scratch is a fixed array inside the
library.  Here the caller is this test, which owns its buffers through
torch.  Two calls in a row, of different sizes, must each give the field the
ordinary entry point (cw_field_relax, FP32 defect correction) gives, to the
tolerance the field tests use: both solves stop at a residual below 1e-9,
and their fields agree to 1e-6 of the field's scale.  This file is collected
last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import _lib

pytestmark = pytest.mark.gpu


def problem(n, seed):
    rng = np.random.default_rng(seed)
    sink = np.where(rng.random(n * n) < 0.6, 0.01, 0.0)
    held = np.zeros(n * n, np.uint8)
    held[:n] = 1
    values = np.where(held == 1, 1.0, 0.0)
    return values, held, sink


def reference(n, values, held, sink):
    f = cw.ScalarField.new(n, n, 1.0, 0.0, 0.0)
    f.set_values(values)
    f.set_linear_sink(sink)
    f.hold_where(1.0, held)
    st = f.relax(1e-9, 1_000_000, omega=1.9, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, stats=True)
    assert st[0]["residual"] < 1e-9
    return f.values()


def noalloc(n, values, held, sink):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    v = torch.tensor(values, dtype=torch.float64, device=dev)
    h = torch.tensor(held, dtype=torch.uint8, device=dev)
    k = torch.tensor(sink, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    sweeps, resid = C.c_int64(), C.c_double()
    _lib.check(_lib.lib().cw_field_relax_noalloc(
        C.c_void_p(v.data_ptr()), C.c_void_p(h.data_ptr()), C.c_void_p(k.data_ptr()), None, None, n, n, 1.0, 0.0,
        0.0, 1.9, 1e-9, 1_000_000, 16, C.byref(sweeps), C.byref(resid)))
    assert resid.value < 1e-9 and sweeps.value > 0
    return v.cpu().numpy()


def test_two_calls_in_a_row_match_the_allocating_entry_point():
    for n, seed in [(300, 1), (181, 2)]:
        values, held, sink = problem(n, seed)
        want = reference(n, values, held, sink)
        got = noalloc(n, values, held, sink)
        assert np.abs(got - want).max() < 1e-6 * np.abs(want).max()


def test_a_field_past_the_fixed_scratch_is_refused():
    torch = pytest.importorskip("torch")
    v = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    h = torch.zeros(1, dtype=torch.uint8, device="cuda:0")
    # the size is checked before any buffer is touched
    with pytest.raises(cw.ConfigError, match="at most"):
        _lib.check(_lib.lib().cw_field_relax_noalloc(
            C.c_void_p(v.data_ptr()), C.c_void_p(h.data_ptr()), None, None, None, 1025, 1024, 1.0, 0.0, 0.0, 1.9,
            1e-6, 10, 16, None, None))


def test_a_call_takes_no_device_memory():
    # what the entry point is for: after a first call (which loads the
    # library's module with its fixed array), a call of another size leaves
    # the device's free memory exactly as it was
    torch = pytest.importorskip("torch")
    noalloc(200, *problem(200, 3))
    n = 150
    values, held, sink = problem(n, 4)
    dev = torch.device("cuda:0")
    v = torch.tensor(values, dtype=torch.float64, device=dev)
    h = torch.tensor(held, dtype=torch.uint8, device=dev)
    k = torch.tensor(sink, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    sweeps, resid = C.c_int64(), C.c_double()
    _lib.check(_lib.lib().cw_field_relax_noalloc(
        C.c_void_p(v.data_ptr()), C.c_void_p(h.data_ptr()), C.c_void_p(k.data_ptr()), None, None, n, n, 1.0, 0.0,
        0.0, 1.9, 1e-6, 1_000_000, 16, C.byref(sweeps), C.byref(resid)))
    _lib.check(_lib.lib().cw_synchronize())
    assert torch.cuda.mem_get_info()[0] == free_before
    assert resid.value < 1e-6


def test_a_relaxation_factor_or_tolerance_out_of_range_is_refused():
    torch = pytest.importorskip("torch")
    v = torch.zeros(64, dtype=torch.float64, device="cuda:0")
    h = torch.zeros(64, dtype=torch.uint8, device="cuda:0")
    for omega, tol in [(2.0, 1e-6), (float("nan"), 1e-6), (1.9, float("nan")), (1.9, -1.0), (1.9, 0.0)]:
        with pytest.raises(cw.ConfigError):
            _lib.check(_lib.lib().cw_field_relax_noalloc(
                C.c_void_p(v.data_ptr()), C.c_void_p(h.data_ptr()), None, None, None, 8, 8, 1.0, 0.0, 0.0, omega,
                tol, 10, 16, None, None))
