"""zqd_fft_execute_noalloc: the FFT for callers that cannot allocate device memory.

Some hosts may not call cudaMalloc at all (a framework that owns every byte of
device memory through its own pool, or an embedded host with one fixed
arena).  For them the library keeps the transform's twiddle table in a static
device array instead of a plan buffer.  This test drives that entry point
through the C-ABI on caller-owned buffers and checks it against the
plan-based zqd_fft_plan_create/zqd_fft_execute path, twice in a row (the
static table keeps the previous call's contents and must be rewritten), with
the tolerance of the other FFT tests.  It sits in its own file so a run that
stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from zinq_b200 import _abi

pytestmark = pytest.mark.gpu


def _plan_fft(x, sign, precision):
    import torch

    L = _abi.load()
    shape = (C.c_int * x.ndim)(*x.shape)
    plan = C.c_void_p()
    _abi.check(L.zqd_fft_plan_create(x.ndim, shape, sign, _abi.PRECISION[precision], C.byref(plan)))
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    t = torch.tensor(x, dtype=dt, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _abi.check(L.zqd_fft_execute(plan, C.c_void_p(t.data_ptr()), C.c_void_p(stream)))
    torch.cuda.synchronize()
    L.zqd_fft_destroy(plan)
    return t.cpu().numpy()


def _noalloc_fft(x, sign, precision):
    import torch

    L = _abi.load()
    shape = (C.c_int * x.ndim)(*x.shape)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    t = torch.tensor(x, dtype=dt, device="cuda")  # the caller owns the data buffer
    stream = torch.cuda.current_stream().cuda_stream
    _abi.check(L.zqd_fft_execute_noalloc(x.ndim, shape, sign, _abi.PRECISION[precision], C.c_void_p(t.data_ptr()),
                                         C.c_void_p(stream)))
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_fft_matches_plan_fft_on_two_calls_in_a_row(precision):
    rng = np.random.default_rng(2024)
    tol = 1e-12 if precision == "fp64" else 2e-6
    for shape, sign in (((8192,), -1), ((64, 64), +1)):  # two calls with different sizes and directions
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        ref = _plan_fft(x, sign, precision)
        got = _noalloc_fft(x, sign, precision)
        scale = np.sqrt(x.size) * np.abs(x).max() if sign < 0 else np.abs(x).max()
        assert np.max(np.abs(got - ref)) <= tol * scale


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_fft_3d_matches_numpy(precision):
    # three strided axis passes and the twiddles made on the device, against numpy directly
    rng = np.random.default_rng(7)
    x = rng.standard_normal((16, 16, 16)) + 1j * rng.standard_normal((16, 16, 16))
    tol = 1e-12 if precision == "fp64" else 2e-6
    fwd = _noalloc_fft(x, -1, precision)
    assert np.max(np.abs(fwd - np.fft.fftn(x))) <= tol * np.sqrt(x.size) * np.abs(x).max()
    inv = _noalloc_fft(x, +1, precision)
    assert np.max(np.abs(inv - np.fft.ifftn(x))) <= tol * np.abs(x).max()


def test_noalloc_fft_rejects_sizes_beyond_its_table():
    import torch

    L = _abi.load()
    t = torch.zeros(16384, dtype=torch.complex128, device="cuda")
    shape = (C.c_int * 1)(16384)
    rc = L.zqd_fft_execute_noalloc(1, shape, -1, 0, C.c_void_p(t.data_ptr()), None)
    assert rc == -7
    assert b"8192" in L.zqd_last_error()
