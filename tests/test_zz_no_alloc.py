"""The allocation-free eigensolver entry point, through the C ABI.

rlmb_heevd_batched_noalloc serves callers that cannot allocate device memory (device
memory already reserved in full by another allocator, or no tolerance for cudaMalloc's
implicit synchronisation mid-run): its scratch is a fixed file-scope device array.  Every
call is checked on its own against numpy (eigenvalues, residual, orthogonality, with the
tolerances of test_gpu_parity._check_eig) and against rlmb_heevd_batched on the same
inputs, call after call, since every call reuses the same array.  This file is collected
last so that a failure here leaves the other tests run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

# the eigensolver tolerances of tests/test_gpu_parity.py
EIG_TOL = 1e-12
VEC_TOL = 1e-9


def _hermitian_batch(rng, batch, n):
    a = rng.normal(size=(batch, n, n)) + 1j * rng.normal(size=(batch, n, n))
    return np.ascontiguousarray(a + np.conj(np.transpose(a, (0, 2, 1))))


def _run_batched(ctx, a0):
    a = torch.tensor(a0, device="cuda")
    w = ctx.heevd(a)
    torch.cuda.synchronize()
    return w.cpu().numpy(), a.cpu().numpy()


def _run_noalloc(lib, a0):
    a = torch.tensor(a0, device="cuda")
    batch, n = a0.shape[0], a0.shape[-1]
    w = torch.empty((batch, n), dtype=torch.float64, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.rlmb_heevd_batched_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(w.data_ptr()), n,
                                        batch, ctypes.c_void_p(info.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, lib.rlmb_status_string(rc)
    torch.cuda.synchronize()
    assert int(info.abs().sum()) == 0
    return w.cpu().numpy(), a.cpu().numpy()


def _check_eig(a0, w, X):
    """Eigenpairs of each column-major matrix a0[b] (stored transposed: a0[b] = M^T) against
    numpy: eigenvalues vs eigvalsh, residual ||M X - X diag(w)||_F and ||X^H X - I||_F."""
    for b in range(a0.shape[0]):
        M = a0[b].T
        Xb = X[b].T   # column k = eigenvector k
        wref = np.linalg.eigvalsh(M)
        scale = np.abs(wref).max()
        assert np.abs(w[b] - wref).max() <= 1e-12 * scale
        nrm = np.linalg.norm(M)
        assert np.linalg.norm(M @ Xb - Xb * w[b][None, :]) <= 1e-12 * nrm
        assert np.linalg.norm(Xb.conj().T @ Xb - np.eye(M.shape[0])) <= 1e-11


def _same(wa, Xa, wb, Xb):
    scale = np.abs(wa).max()
    assert np.abs(wa - wb).max() <= EIG_TOL * scale
    # eigenvectors agree up to a phase each (rows are eigenvectors)
    ov = np.abs(np.einsum("bkr,bkr->bk", np.conj(Xa), Xb))
    assert np.abs(ov - 1).max() < VEC_TOL


@pytest.mark.parametrize("n,batch", [(48, 5), (256, 19), (900, 3)])
def test_noalloc_matches_batched_twice(n, batch):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import rlmb
    lib = rlmb.lib()
    ctx = rlmb.Context(0)
    rng = np.random.default_rng(n)
    for call in range(2):
        a0 = _hermitian_batch(rng, batch, n)
        wb, Xb = _run_batched(ctx, a0)
        wn, Xn = _run_noalloc(lib, a0)
        _check_eig(a0, wn, Xn)
        _same(wb, Xb, wn, Xn)
    ctx.close()


def test_noalloc_rejects_orders_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import rlmb
    lib = rlmb.lib()
    n = 928
    a = torch.zeros((1, n, n), dtype=torch.complex128, device="cuda")
    w = torch.zeros((1, n), dtype=torch.float64, device="cuda")
    rc = lib.rlmb_heevd_batched_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(w.data_ptr()), n, 1,
                                        None, None)
    assert rc == -5
    assert b"scratch limit" in lib.rlmb_status_string(rc)
