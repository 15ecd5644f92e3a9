"""The oracle's eigensolver restates LAPACK dsyevd('V', 'U') (the reference's eighBatch,
src/linear_algebra.zig:55-70).  Pinned here against numpy.linalg.eigh(UPLO='U'), which calls LAPACK
?syevd (OpenBLAS): eigenvalues and eigenvectors, signs included, for n = 2..4 on random matrices,
nearly diagonal ones, exactly diagonal ones and potential matrices of the coupled-surface workloads."""
import numpy as np
import pytest

from oracle import qd_ref


@pytest.mark.parametrize("n", [2, 3, 4])
def test_eigh_matches_lapack_with_signs(n):
    rng = np.random.default_rng(100 + n)
    worst = 0.0
    for k in range(1500):
        A = rng.standard_normal((n, n))
        A = A + A.T
        if k % 3 == 1:
            A = np.diag(rng.standard_normal(n)) + 1e-3 * A
        if k % 3 == 2:
            A = np.diag(rng.standard_normal(n))
        w, U = np.linalg.eigh(A, UPLO="U")
        wo, Uo = qd_ref.eigh(A)
        assert np.max(np.abs(w - wo)) <= 1e-13 * max(1.0, np.max(np.abs(w)))
        worst = max(worst, float(np.max(np.abs(U - Uo))))
    assert worst <= 1e-12, worst


def test_eigh_of_the_three_state_workload_potential_matches_lapack():
    # The 2-D three-state coupled harmonic surfaces on a 64^2 grid of [-12, 12)^2.  Where the couplings
    # fall below 1e-13 of the diagonal, dsytd2 reflects two equal, negligible couplings into a 2 x 2 block
    # with (nearly) equal diagonals, and LAPACK's own signs follow the last-bit rounding of its BLAS
    # kernels there; those points are counted, not compared.
    rng = np.random.default_rng(20261203)
    a, b, c = rng.uniform(-1, 1, 3), rng.uniform(-1, 1, 3), rng.uniform(0, 0.2, 3)
    g = -12 + 24 * np.arange(64) / 64
    compared = 0
    for x in g:
        for y in g:
            coupling = 0.05 * np.exp(-(x * x + y * y) / 2)
            V = np.full((3, 3), coupling)
            for i in range(3):
                V[i, i] = 0.5 * (x * x + y * y) + a[i] * x + b[i] * y + c[i]
            if coupling < 1e-13 * np.max(np.abs(np.diag(V))):
                continue
            compared += 1
            w, U = np.linalg.eigh(V, UPLO="U")
            wo, Uo = qd_ref.eigh(V)
            assert np.max(np.abs(U - Uo)) <= 1e-11, (x, y)
    assert compared > 1000


def test_eigenvectors_stay_orthonormal_at_every_coupling_scale():
    # couplings from 1e-1 down to denormals, with exactly degenerate diagonals: the reflector norm is
    # scaled and dlarfg rescales tiny betas (a naive sum of squares underflows and breaks orthogonality)
    rng = np.random.default_rng(3)
    for k in range(6000):
        n = 3 if k % 2 else 4
        d = rng.standard_normal(n) * 1e-3
        if k % 5 == 0:
            d[rng.integers(n)] = d[0]
        sc = 10.0 ** rng.uniform(-320, -1)
        A = np.diag(d) + sc * rng.choice([-1, 1]) * (np.ones((n, n)) - np.eye(n))
        if k % 3 == 0:
            A = np.diag(d) + sc * rng.standard_normal((n, n))
            A = (A + A.T) / 2
        W, U = qd_ref.eigh(A)
        assert np.max(np.abs(U @ U.T - np.eye(n))) <= 1e-14, A
        assert np.max(np.abs(U @ np.diag(W) @ U.T - A)) <= 1e-15 + 1e-14 * np.max(np.abs(A))
