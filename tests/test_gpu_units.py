"""GPU unit tests of the three seams: FFT (FftPlan, src/fourier_transform.zig),
eigendecomposition (eighBatch / dsyevd, src/linear_algebra.zig:28-70) and the
expression interpreter (ExprTk, src/exprtk.cpp:32-40), each through the C-ABI."""
import ctypes as C

import numpy as np
import pytest

from oracle import qd_ref
from zinq_b200 import _abi

pytestmark = pytest.mark.gpu


def dptr(a):
    return a.ctypes.data_as(_abi.DP)


def device_fft(x, sign, precision="fp64"):
    import torch

    L = _abi.load()
    shape = (C.c_int * x.ndim)(*x.shape)
    plan = C.c_void_p()
    _abi.check(L.zqd_fft_plan_create(x.ndim, shape, sign, _abi.PRECISION[precision], C.byref(plan)))
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    t = torch.tensor(x, dtype=dt, device="cuda")
    _abi.check(L.zqd_fft_execute(plan, C.c_void_p(t.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    L.zqd_fft_destroy(plan)
    return t.cpu().numpy()


@pytest.mark.parametrize("shape", [(2,), (8,), (64,), (1024,), (8192,), (32, 32), (16, 16, 16), (128, 128)])
def test_fft_seam_matches_numpy(shape):
    rng = np.random.default_rng(len(shape) * 1000 + shape[0])
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = device_fft(x, -1)
    np.testing.assert_allclose(f, np.fft.fftn(x), rtol=0, atol=1e-12 * np.sqrt(x.size) * np.abs(x).max())
    b = device_fft(f, +1)  # inverse carries the reference's 1/N
    np.testing.assert_allclose(b, x, rtol=0, atol=1e-13 * np.sqrt(x.size))
    o = qd_ref.fft(x, -1)
    assert np.max(np.abs(f - o)) <= 1e-12 * np.sqrt(x.size)


def test_fft_seam_fp32():
    rng = np.random.default_rng(5)
    x = rng.standard_normal(4096) + 1j * rng.standard_normal(4096)
    f = device_fft(x, -1, "fp32")
    rel = np.linalg.norm(f - np.fft.fft(x)) / np.linalg.norm(np.fft.fft(x))
    assert rel < 5e-7


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_eigh_matches_oracle(n):
    rng = np.random.default_rng(n)
    count = 4096
    A = rng.standard_normal((count, n, n)) * 0.01
    A = A + A.transpose(0, 2, 1)
    A[:64] = 0.0  # zero matrices
    if n == 2:
        A[64:128, 0, 1] = A[64:128, 1, 0] = 1e-300  # negligible coupling
        A[128:192, 0, 0] = 0.0  # Tully-2 style zero diagonal
    L = _abi.load()
    W, U = np.zeros((count, n)), np.zeros((count, n, n))
    _abi.check(L.zqd_eigh_batch(n, count, dptr(np.ascontiguousarray(A)), dptr(W), dptr(U)))
    for i in range(count):
        wo, uo = qd_ref.eigh(A[i])
        np.testing.assert_allclose(W[i], wo, atol=1e-15)
        np.testing.assert_allclose(U[i], uo, atol=1e-12)
        np.testing.assert_allclose(U[i] @ np.diag(W[i]) @ U[i].T, A[i], atol=1e-15)


@pytest.mark.parametrize("n", [3, 4])
def test_eigh_orthonormal_at_every_coupling_scale(n):
    # equal couplings from 1e-1 down to denormals over (partly) degenerate diagonals, as on the far
    # edges of coupled-surface grids: eigenvectors orthonormal and equal to the oracle's
    rng = np.random.default_rng(40 + n)
    count = 3000
    d = rng.standard_normal((count, n)) * 1e-3
    d[::5, 1] = d[::5, 0]
    sc = 10.0 ** rng.uniform(-320, -1, count)
    A = np.einsum("ki,ij->kij", d, np.eye(n)) + sc[:, None, None] * (np.ones((n, n)) - np.eye(n))
    L = _abi.load()
    W, U = np.zeros((count, n)), np.zeros((count, n, n))
    _abi.check(L.zqd_eigh_batch(n, count, dptr(np.ascontiguousarray(A)), dptr(W), dptr(U)))
    for i in range(count):
        assert np.max(np.abs(U[i] @ U[i].T - np.eye(n))) <= 1e-14, A[i]
        wo, uo = qd_ref.eigh(A[i])
        np.testing.assert_allclose(U[i], uo, atol=1e-14)


@pytest.mark.parametrize("n", [2, 3, 4])
def test_eigh_signs_match_lapack(n):
    # numpy.linalg.eigh calls LAPACK ?syevd, the routine the reference uses (src/linear_algebra.zig:67);
    # eigenvectors compared without any sign freedom, random and nearly diagonal matrices
    rng = np.random.default_rng(7 + n)
    A = rng.standard_normal((3000, n, n))
    A = A + A.transpose(0, 2, 1)
    A[1000:2000] = 0.01 * A[1000:2000] + np.einsum("ki,ij->kij", rng.standard_normal((1000, n)), np.eye(n))
    L = _abi.load()
    W, U = np.zeros((3000, n)), np.zeros((3000, n, n))
    _abi.check(L.zqd_eigh_batch(n, 3000, dptr(np.ascontiguousarray(A)), dptr(W), dptr(U)))
    w_np, u_np = np.linalg.eigh(A, UPLO="U")
    np.testing.assert_allclose(W, w_np, atol=1e-13)
    np.testing.assert_allclose(U, u_np, atol=1e-12)


EXPRS = ["0.5*r1^2", "+sgn(r1) * 0.01 * (1.0 - exp(-1.6 * abs(r1)))", "0.005 * exp(-r1^2)",
         "0.01*tanh(1.6*r1)", "-r1^3/3 + 0.1*(r1^2*r2 - r2^3/3) + 0.05*r3^4", "sqrt(abs(r1)) * cos(r2) - sin(t)",
         "min(r1, r2, r3) + max(r1, 1) + if(r1 < r2, 2, 3)", "2r1 + 3(r2-1)", "pow(abs(r1), 2.5) + r1^-2",
         "atan2(r1, r2) + hypot(r1, r3) + log(1 + r3^2) + erf(r1)", "(r1 - t) * 10 % 3"]


@pytest.mark.parametrize("text", EXPRS)
def test_expression_vm_matches_oracle(text):
    rng = np.random.default_rng(11)
    pts = rng.uniform(-3, 3, size=(257, 3))
    L = _abi.load()
    h = C.c_void_p()
    _abi.check(L.zqd_expr_compile(text.encode(), len(text), 3, C.byref(h)))
    out = np.zeros(len(pts))
    _abi.check(L.zqd_expr_eval_points(h, dptr(np.ascontiguousarray(pts)), len(pts), 0.7, dptr(out)))
    L.zqd_expr_destroy(h)
    ref = np.array([qd_ref.expr_eval(text, p, 0.7) for p in pts])
    # CUDA's and glibc's libm agree to a few ulp; the interpreter itself rounds every operation like the oracle
    np.testing.assert_allclose(out, ref, rtol=1e-13, atol=1e-14)


def test_potential_plot_matches_expression_oracle_and_lapack(tmp_path):
    from oracle import qd_ref
    from zinq_b200 import quantum_dynamics as qd

    mat = [["0.02*tanh(1.2*r1)+0.01*r2^2", "0.01*exp(-r1^2-r2^2)+0.001*t"],
           ["0.01*exp(-r1^2-r2^2)+0.001*t", "-0.02*tanh(1.2*r1)+0.01*r2^2"]]
    opt = {"potential": {"custom": {"ndim": 2, "matrix": mat, "time_dependent": True}},
           "grid": {"bounds": [[-6, 6], [-4, 4]], "npoint": 16}, "time": 1.5,
           "write": {"potential": str(tmp_path / "pot.mat")}}
    U = qd.potential_plot(opt, write=True)
    n = 16
    r = np.array([[-6 + i * 12 / n, -4 + j * 8 / n] for i in range(n) for j in range(n)])
    ref = np.array([[[qd_ref.expr_eval(mat[a][b], p, 1.5) for b in range(2)] for a in range(2)] for p in r])
    np.testing.assert_allclose(U, ref, rtol=1e-13, atol=1e-15)
    lines = open(tmp_path / "pot.mat").read().splitlines()
    assert lines[0] == f"{n * n} 6"
    rows = np.array([[float(x) for x in l.split()] for l in lines[1:]])
    np.testing.assert_allclose(rows[:, :2], r, atol=1e-13)
    np.testing.assert_allclose(rows[:, 2:], ref.reshape(-1, 4), atol=6e-15)
    Ua = qd.potential_plot({**opt, "adiabatic": True})
    w = np.linalg.eigvalsh(ref)
    np.testing.assert_allclose(Ua[:, [0, 1], [0, 1]], w, rtol=1e-13, atol=1e-15)
    assert np.all(Ua[:, 0, 1] == 0) and np.all(Ua[:, 1, 0] == 0)
