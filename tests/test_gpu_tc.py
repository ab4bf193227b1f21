"""The batched complex GEMM engines through the C ABI (rlmb_zgemm_batched), against numpy's
complex128 product of the same inputs.

  RLMB_GEMM_FP64           (FP64 tensor path)                   |C - C_ref| <= 1e-13 * (|A| |B|)
  RLMB_GEMM_TF32X3         (tcgen05, split TF32 operands)       |C - C_ref| <= 4e-6 * (|A| |B|)
  RLMB_GEMM_TF32X3_F64ACC  (the same, TMA-fed, FP64 sums over K) |C - C_ref| <= 1e-6 * (|A| |B|)

|A| |B| is the product of the entrywise absolute values, the scale of each entry's rounding
error.  The TF32X3 bound allows for the 2^-21 relative error of the split products and the
FP32 accumulation over k.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = {0: 1e-13, 1: 4e-6, 2: 1e-6}


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import rlmb
    c = rlmb.Context(0)
    yield c
    assert c.tc_fault_count() == 0
    c.close()


def _rand(rng, *shape, scale=1.0):
    return scale * (rng.normal(size=shape) + 1j * rng.normal(size=shape))


def _run(ctx, A, B, engine):
    """A[batch, m, k], B[batch, k, n] numpy -> C[batch, m, n] through the column-major ABI."""
    at = torch.tensor(np.ascontiguousarray(np.transpose(A, (0, 2, 1))), device="cuda")
    bt = torch.tensor(np.ascontiguousarray(np.transpose(B, (0, 2, 1))), device="cuda")
    ct = ctx.zgemm(at, bt, engine)
    torch.cuda.synchronize()
    return np.transpose(ct.cpu().numpy(), (0, 2, 1))


@pytest.mark.parametrize("engine", [0, 1, 2])
@pytest.mark.parametrize("m,n,k,batch", [(64, 128, 16, 1), (1, 1, 1, 1), (100, 70, 33, 3), (257, 300, 129, 2),
                                         (128, 256, 512, 2), (640, 512, 1000, 1), (33, 129, 7, 4)])
def test_zgemm_matches_numpy(ctx, engine, m, n, k, batch):
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    A = _rand(rng, batch, m, k)
    B = _rand(rng, batch, k, n)
    C = _run(ctx, A, B, engine)
    ref = A @ B
    bound = np.abs(A) @ np.abs(B)
    assert np.all(np.abs(C - ref) <= TOL[engine] * bound + 1e-300), np.max(np.abs(C - ref) / bound)


@pytest.mark.parametrize("engine", [0, 1, 2])
def test_zgemm_scaled_operands(ctx, engine):
    """Operands of very different magnitudes (a residual-sized B) keep the relative bound."""
    rng = np.random.default_rng(7)
    A = _rand(rng, 2, 200, 300)
    B = _rand(rng, 2, 300, 150, scale=1e-9)
    C = _run(ctx, A, B, engine)
    bound = np.abs(A) @ np.abs(B)
    assert np.all(np.abs(C - A @ B) <= TOL[engine] * bound)


def test_zgemm_empty_inner_dimension(ctx):
    """k = 0: the product is zero (the output is written, not left untouched)."""
    at = torch.zeros((1, 0, 70), dtype=torch.complex128, device="cuda")
    bt = torch.zeros((1, 50, 0), dtype=torch.complex128, device="cuda")
    for engine in (0, 1, 2):
        ct = ctx.zgemm(at, bt, engine)
        torch.cuda.synchronize()
        assert float(ct.abs().max()) == 0.0


def test_zgemm_arguments(ctx):
    import rlmb
    a = torch.zeros((1, 4, 4), dtype=torch.complex128, device="cuda")
    with pytest.raises(rlmb.RlmbError):
        ctx.zgemm(a, a, engine=7)


def test_double_accumulation_is_more_accurate(ctx):
    """At the refinement's inner dimension (k = 3000) the engine that sums the accumulator in
    double precision after every 32 real terms is at least three times closer to the exact
    product than the one that accumulates all of k in FP32."""
    rng = np.random.default_rng(11)
    A = _rand(rng, 1, 128, 3000)
    B = _rand(rng, 1, 3000, 256)
    ref = A @ B
    bound = np.abs(A) @ np.abs(B)
    e1 = np.max(np.abs(_run(ctx, A, B, 1) - ref) / bound)
    e2 = np.max(np.abs(_run(ctx, A, B, 2) - ref) / bound)
    assert e2 * 3 <= e1, (e1, e2)
