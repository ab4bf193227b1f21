"""GPU parity of the divide-and-conquer tridiagonal solver (tridiag_dc.cuh), called through the C
ABI inside the Householder eigensolver, against LAPACK (numpy eigvalsh), against the bisection
solver of the same library and against the reference's fixtures at the benchmark geometries.

Tolerances are those of the Householder tests (double precision):
  eigenvalues        max|w - w_ref| <= 1e-12 * max|w_ref|
  residual           ||M X - X diag(w)||_F <= 1e-12 * ||M||_F   (2e-15 n from order 700)
  orthogonality      ||X^H X - I||_F <= 1e-11                   (2e-14 n from order 700)
  Chern numbers      rint() identical, |C - C_ref| <= 1e-8
  twist energies     max|E - E_ref| <= 1e-10 * max|E_ref|
"""
import numpy as np
import pytest

from conftest import golden
from test_gpu_parity import _check_eig, _hermitian, _run_heevd

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import rlmb
    c = rlmb.Context(0)
    yield c
    c.close()


def _dc(ctx, n):
    ctx.set_heev_solver(n, ctx.SOLVER_HOUSEHOLDER)
    ctx.set_tridiag_solver(n, ctx.TRIDIAG_DC)
    assert ctx.tridiag_solver(n) == ctx.TRIDIAG_DC


@pytest.mark.parametrize("n", [1, 2, 3, 5, 16, 17, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 200, 256, 300,
                               457, 512, 513])
def test_dc_random(ctx, n):
    _dc(ctx, n)
    rng = np.random.default_rng(2000 + n)
    mats = [_hermitian(rng, n) for _ in range(3)]
    w, X = _run_heevd(ctx, mats)
    for b, M in enumerate(mats):
        _check_eig(M, w[b], X[b], np.linalg.eigvalsh(M))


@pytest.mark.parametrize("n", [700, 1000, 1537, 2048, 2049])
def test_dc_large_orders(ctx, n):
    _dc(ctx, n)
    rng = np.random.default_rng(n)
    mats = [_hermitian(rng, n) for _ in range(2)]
    w, X = _run_heevd(ctx, mats)
    for b, M in enumerate(mats):
        wref = np.linalg.eigvalsh(M)
        assert np.abs(w[b] - wref).max() <= 1e-12 * np.abs(wref).max()
        res = np.linalg.norm(M @ X[b] - X[b] * w[b][None, :]) / np.linalg.norm(M)
        assert res <= 2e-15 * n, res
        orth = np.linalg.norm(X[b].conj().T @ X[b] - np.eye(n))
        assert orth <= 2e-14 * n, orth


@pytest.mark.parametrize("kind", ["identity", "degenerate", "diagonal", "zero", "blocks", "tridiag_split"])
@pytest.mark.parametrize("n", [7, 48, 160, 300])
def test_dc_structured(ctx, kind, n):
    """Exact and near degeneracies: every deflation branch (small z, rotated pole pairs, rho = 0)."""
    _dc(ctx, n)
    rng = np.random.default_rng(7 * n)
    M = _hermitian(rng, n, kind)
    w, X = _run_heevd(ctx, [M])
    wref = np.linalg.eigvalsh(M)
    if kind == "zero":
        assert np.abs(w[0]).max() == 0.0
        assert np.linalg.norm(X[0].conj().T @ X[0] - np.eye(n)) <= 1e-11
    else:
        _check_eig(M, w[0], X[0], wref)


def _tridiagonal(kind, n, rng):
    if kind == "wilkinson":     # W+_n: pairs of eigenvalues close to 1e-(n/2)
        d = np.abs(np.arange(n) - (n - 1) / 2.0)
        e = np.ones(n - 1)
    elif kind == "glued":       # glued Wilkinson blocks: clusters of near-equal eigenvalues
        d = np.tile(np.abs(np.arange(21) - 10.0), n // 21 + 1)[:n]
        e = np.ones(n - 1)
        e[20::21] = 1e-10
    elif kind == "tiny_coupling":
        d = np.ones(n)
        e = np.full(n - 1, 1e-18)
    elif kind == "graded":      # entries over 30 orders of magnitude
        d = 10.0 ** np.linspace(-15, 15, n)
        e = np.sqrt(d[:-1] * d[1:]) * 0.1
    else:
        raise ValueError(kind)
    # a phase on the off-diagonal: the reduction turns it back into the real tridiagonal
    ph = np.exp(1j * rng.uniform(0, 2 * np.pi, n - 1))
    return np.diag(d).astype(np.complex128) + np.diag(e * ph, 1) + np.diag(e * ph.conj(), -1)


@pytest.mark.parametrize("kind", ["wilkinson", "glued", "tiny_coupling", "graded"])
@pytest.mark.parametrize("n", [21, 101, 420])
def test_dc_hard_tridiagonals(ctx, kind, n):
    _dc(ctx, n)
    M = _tridiagonal(kind, n, np.random.default_rng(n))
    w, X = _run_heevd(ctx, [M])
    _check_eig(M, w[0], X[0], np.linalg.eigvalsh(M))


@pytest.mark.parametrize("n", [48, 256, 600])
def test_dc_matches_bisection(n):
    """Both tridiagonal solvers give the same spectrum and eigenvectors (up to a phase)."""
    import rlmb
    rng = np.random.default_rng(300 + n)
    mats = [_hermitian(rng, n) for _ in range(3)]
    out = {}
    for solver in (rlmb.Context.TRIDIAG_DC, rlmb.Context.TRIDIAG_BISECTION):
        c = rlmb.Context(0)
        try:
            c.set_heev_solver(n, c.SOLVER_HOUSEHOLDER)
            c.set_tridiag_solver(n, solver)
            out[solver] = _run_heevd(c, mats)
        finally:
            c.close()
    (wd, Xd), (wb, Xb) = out[rlmb.Context.TRIDIAG_DC], out[rlmb.Context.TRIDIAG_BISECTION]
    assert np.abs(wd - wb).max() <= 1e-12 * np.abs(wb).max()
    for b in range(len(mats)):
        ov = np.abs(np.sum(Xd[b].conj() * Xb[b], axis=0))
        assert np.abs(ov - 1.0).max() <= 1e-9


@pytest.mark.parametrize("n", [300, 1000])
def test_dc_mixed_mode(n):
    """The mixed mode's double-precision tridiagonal stage by divide and conquer, then the
    refinement: the mixed mode's tolerances (test_gpu_mixed)."""
    import rlmb
    c = rlmb.Context(0)
    try:
        c.precision = c.MIXED
        c.set_tridiag_solver(n, c.TRIDIAG_DC)
        assert c.tridiag_solver(n) == c.TRIDIAG_DC
        rng = np.random.default_rng(n + 9)
        mats = [_hermitian(rng, n) for _ in range(2)]
        w, X = _run_heevd(c, mats)
        for b, M in enumerate(mats):
            wref = np.linalg.eigvalsh(M)
            assert np.abs(w[b] - wref).max() <= 1e-10 * np.abs(wref).max()
            assert np.linalg.norm(M @ X[b] - X[b] * w[b][None, :]) <= 1e-10 * np.linalg.norm(M)
            assert np.linalg.norm(X[b].conj().T @ X[b] - np.eye(n)) <= 1e-10
    finally:
        c.close()


def test_dc_solver_api():
    import rlmb
    c = rlmb.Context(0)
    try:
        assert c.tridiag_solver(3000) in (c.TRIDIAG_DC, c.TRIDIAG_BISECTION)
        with pytest.raises(rlmb.RlmbError):
            c.set_tridiag_solver(3601, c.TRIDIAG_DC)      # beyond the top merge's shared memory
        with pytest.raises(rlmb.RlmbError):
            c.set_tridiag_solver(100, 9)
        c.set_tridiag_solver(100, c.TRIDIAG_BISECTION)
        assert c.tridiag_solver(100) == c.TRIDIAG_BISECTION
        c.set_heev_config(100, 1, 1, 0, 0, 0)               # launch choices keep the solver
        assert c.tridiag_solver(100) == c.TRIDIAG_BISECTION
        c.set_tridiag_solver(100, c.TRIDIAG_DC)
        assert c.tridiag_solver(100) == c.TRIDIAG_DC
    finally:
        c.close()


# ---------------------------------------------- benchmark geometries through divide and conquer
def test_dc_hlm_benchmark_geometry_samples_0_to_7():
    """hlm 48x16, q=3, band 0, g=32 (order 256), seed 1, samples 0-7 against the reference."""
    import rlmb
    d = golden("hlm_48x16_q3_b0_g32_s1_samples0-7.npz")
    c = rlmb.Context(0)
    try:
        c.set_tridiag_solver(256, c.TRIDIAG_DC)
        e, ch = c.hlm_mesh_solve(48, 16, 3, 0, 32, d["potentials"])
        assert c.last_failures == 0
    finally:
        c.close()
    for i in range(8):
        eref, cref = d["energies"][i], d["chern"][i]
        assert np.abs(e[i] - eref).max() <= 1e-10 * np.abs(eref).max()
        assert np.array_equal(np.rint(ch[i]), np.rint(cref))
        assert np.abs(ch[i] - cref).max() < 1e-8


@pytest.mark.parametrize("mixed", [False, True])
def test_dc_rlm_512_samples_0_to_3(mixed):
    """rlm n_phi=512 (8192 impurities, g=16, seed 1), samples 0-3, in either precision mode."""
    import rlmb
    d = golden("rlm_n512_g16_c4_s1_full.npz")
    c = rlmb.Context(0)
    try:
        if mixed:
            c.precision = c.MIXED
        c.set_tridiag_solver(512, c.TRIDIAG_DC)
        e, ch = c.rlm_mesh_solve(512, 1.0, 16.0, 16, 1, 0, 4)
        assert c.last_failures == 0
    finally:
        c.close()
    for i in range(4):
        eref, cref = d["energies"][i], d["chern"][i]
        assert np.abs(e[i] - eref).max() <= 1e-10 * np.abs(eref).max()
        assert np.array_equal(np.rint(ch[i]), np.rint(cref))
        assert np.abs(ch[i] - cref).max() < 1e-8


def test_dc_rlm_3000_matches_reference():
    """rlm n_phi=3000 (48,000 impurities, g=4, seed 1, sample 0): 25 solves of order 3000."""
    import os
    import rlmb
    from conftest import GOLDEN
    name = "rlm_n3000_g4_c1_s1_full.npz"
    if not os.path.exists(os.path.join(GOLDEN, name)):
        pytest.skip(f"{name} not generated")
    d = golden(name)
    c = rlmb.Context(0)
    try:
        c.set_tridiag_solver(3000, c.TRIDIAG_DC)
        e, ch = c.rlm_mesh_solve(3000, 1.0, 16.0, 4, 1, 0, 1)
        assert c.last_failures == 0
    finally:
        c.close()
    eref, cref = d["energies"][0], d["chern"][0]
    assert np.abs(e[0] - eref).max() <= 1e-10 * np.abs(eref).max()
    assert np.array_equal(np.rint(ch[0]), np.rint(cref))
    assert np.abs(ch[0] - cref).max() < 1e-8
