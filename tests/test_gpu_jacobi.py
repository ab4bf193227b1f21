"""GPU parity of the batched Jacobi eigensolver (k_jacobi, orders <= 80), called through the C
ABI, against LAPACK (numpy eigvalsh) and against the Householder path of the same library.

Tolerances are those of the Householder tests (double precision):
  eigenvalues        max|w - w_ref| <= 1e-12 * max|w_ref|
  residual           ||M X - X diag(w)||_F <= 1e-12 * ||M||_F
  orthogonality      ||X^H X - I||_F <= 1e-11
"""
import numpy as np
import pytest

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


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 8, 15, 16, 17, 31, 32, 33, 47, 48, 63, 64, 65, 79, 80])
def test_jacobi_random(ctx, n):
    ctx.set_heev_solver(n, ctx.SOLVER_JACOBI)
    assert ctx.heev_solver(n) == ctx.SOLVER_JACOBI
    rng = np.random.default_rng(1000 + n)
    mats = [_hermitian(rng, n) for _ in range(5)]
    w, X = _run_heevd(ctx, mats)
    for b, M in enumerate(mats):
        _check_eig(M, w[b], X[b], np.linalg.eigvalsh(M))


@pytest.mark.parametrize("kind", ["identity", "degenerate", "diagonal", "zero", "blocks", "tridiag_split"])
@pytest.mark.parametrize("n", [7, 32, 48, 80])
def test_jacobi_structured(ctx, kind, n):
    ctx.set_heev_solver(n, ctx.SOLVER_JACOBI)
    rng = np.random.default_rng(7 * n)
    M = _hermitian(rng, n, kind)
    w, X = _run_heevd(ctx, [M])
    wref = np.linalg.eigvalsh(M)
    if kind == "zero":
        assert np.abs(w[0]).max() == 0.0
        assert np.linalg.norm(X[0].conj().T @ X[0] - np.eye(n)) <= 1e-11
    else:
        _check_eig(M, w[0], X[0], wref)


def test_jacobi_reads_upper_triangle_only(ctx):
    """The lower triangle is never read: garbage there changes nothing."""
    n = 40
    ctx.set_heev_solver(n, ctx.SOLVER_JACOBI)
    rng = np.random.default_rng(3)
    M = _hermitian(rng, n)
    G = M.copy()
    il = np.tril_indices(n, -1)
    G[il] = rng.normal(size=len(il[0])) * 1e3 + 7j
    G[np.diag_indices(n)] += 5j   # the imaginary part of the diagonal is ignored too
    w, X = _run_heevd(ctx, [G])
    _check_eig(M, w[0], X[0], np.linalg.eigvalsh(M))


@pytest.mark.parametrize("n", [12, 32, 64])
def test_jacobi_matches_householder(n):
    """Both solvers of the library give the same spectrum and the same eigenspaces."""
    import rlmb
    rng = np.random.default_rng(90 + n)
    mats = [_hermitian(rng, n) for _ in range(4)]
    out = {}
    for solver in (rlmb.Context.SOLVER_JACOBI, rlmb.Context.SOLVER_HOUSEHOLDER):
        c = rlmb.Context(0)
        try:
            c.set_heev_solver(n, solver)
            assert c.heev_solver(n) == solver
            out[solver] = _run_heevd(c, mats)
        finally:
            c.close()
    (wj, Xj), (wh, Xh) = out[rlmb.Context.SOLVER_JACOBI], out[rlmb.Context.SOLVER_HOUSEHOLDER]
    assert np.abs(wj - wh).max() <= 1e-12 * np.abs(wh).max()
    for b in range(len(mats)):
        # |<x_j|x_h>| = 1 per (non-degenerate) eigenvector: the same vectors up to a phase
        ov = np.abs(np.sum(Xj[b].conj() * Xh[b], axis=0))
        assert np.abs(ov - 1.0).max() <= 1e-9


def test_jacobi_large_batch_and_mixed_context():
    """Thousands of small matrices in one call, in a mixed-precision context: Jacobi runs in
    double precision in either mode, so the FP64 tolerances hold."""
    import rlmb
    n, nb = 16, 3000
    rng = np.random.default_rng(11)
    a0 = rng.normal(size=(nb, n, n)) + 1j * rng.normal(size=(nb, n, n))
    a0 = (a0 + np.conj(np.transpose(a0, (0, 2, 1)))) / 2
    c = rlmb.Context(0)
    try:
        c.precision = c.MIXED
        c.set_heev_solver(n, c.SOLVER_JACOBI)
        a = torch.tensor(np.ascontiguousarray(np.transpose(a0, (0, 2, 1))), device="cuda")
        info = torch.full((nb,), 7, dtype=torch.int32, device="cuda")
        w = c.heevd(a, info=info)
        torch.cuda.synchronize()
        assert int(info.abs().sum()) == 0
        w = w.cpu().numpy()
        X = a.cpu().numpy()
        wref = np.linalg.eigvalsh(a0)
        assert np.abs(w - wref).max() <= 1e-12 * np.abs(wref).max()
        for b in (0, 1, nb // 2, nb - 1):
            _check_eig(a0[b], w[b], X[b].T, wref[b])
    finally:
        c.close()


def test_jacobi_solver_api_and_builtin_choice():
    import rlmb
    c = rlmb.Context(0)
    try:
        assert c.heev_solver(20) == c.SOLVER_JACOBI        # built-in up to order 20
        assert c.heev_solver(21) == c.SOLVER_HOUSEHOLDER
        assert c.heev_solver(500) == c.SOLVER_HOUSEHOLDER
        with pytest.raises(rlmb.RlmbError):
            c.set_heev_solver(81, c.SOLVER_JACOBI)             # beyond the shared-memory limit
        with pytest.raises(rlmb.RlmbError):
            c.set_heev_solver(16, 7)
        c.set_heev_solver(20, c.SOLVER_HOUSEHOLDER)
        assert c.heev_solver(20) == c.SOLVER_HOUSEHOLDER
        c.set_heev_config(20, 0, 0, 0, 0, 0)                   # launch choices keep the solver
        assert c.heev_solver(20) == c.SOLVER_HOUSEHOLDER
        c.set_heev_solver(20, c.SOLVER_AUTO)
        assert c.heev_solver(20) == c.SOLVER_JACOBI
        c.set_heev_solver(64, c.SOLVER_JACOBI)
        assert c.heev_solver(64) == c.SOLVER_JACOBI
    finally:
        c.close()


@pytest.mark.parametrize("n", [24, 56])
def test_autotune_between_jacobi_and_householder(n):
    """The autotuner times Jacobi against the Householder configurations at small orders and
    keeps one; the result is correct either way."""
    import rlmb
    c = rlmb.Context(0)
    try:
        c.set_autotune(True)
        rng = np.random.default_rng(n)
        mats = [_hermitian(rng, n) for _ in range(3)]
        w, X = _run_heevd(c, mats)
        for b, M in enumerate(mats):
            _check_eig(M, w[b], X[b], np.linalg.eigvalsh(M))
        tuned, cfg = c.heev_config(n)
        assert tuned and cfg["ms_per_matrix"] > 0
        assert c.heev_solver(n) in (c.SOLVER_JACOBI, c.SOLVER_HOUSEHOLDER)
    finally:
        c.close()
