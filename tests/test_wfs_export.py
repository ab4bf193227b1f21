"""Eigenvector export (diag_wrappers/wfs_file.cpp, rlm/main_rlm_gpu.cu:187,227 with -DwfsIO).

CPU: the reference-named write_wfs/read_wfs of the library write byte-identical files to
the reference's own write_wfs (oracle/_ref/wfs_ref, compiled from its source).
GPU: rlmb_rlm_mesh_export writes one file per k-point whose columns are eigenvectors of the
reference's H(theta_1, theta_2) (oracle assembly) and returns rlmb_rlm_mesh_solve's results."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_ROOT, REPO

LIB = os.path.join(PKG_ROOT, "lib", "librlmb.so")
REF = os.path.join(REPO, "oracle", "_ref", "wfs_ref")   # the reference's write_wfs, own process
WRITE = "_Z9write_wfsiiPSt7complexIdEm"   # write_wfs(int, int, std::complex<double>*, unsigned long)
READ = "_Z8read_wfsiiPSt7complexIdEm"


def _fn(name):
    f = getattr(ctypes.CDLL(LIB), name)
    f.restype = None
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_ulong]
    return f


def test_write_wfs_matches_reference_bytes(tmp_path, monkeypatch):
    for p in (LIB, REF):
        if not os.path.exists(p):
            pytest.skip(f"{p} not built")
    rng = np.random.default_rng(3)
    data = np.ascontiguousarray(rng.normal(size=77) + 1j * rng.normal(size=77))
    (tmp_path / "ours").mkdir()
    (tmp_path / "ref").mkdir()
    data.tofile(tmp_path / "in.bin")
    subprocess.run([REF, "3", "11", str(tmp_path / "in.bin")], cwd=tmp_path / "ref", check=True)
    monkeypatch.chdir(tmp_path / "ours")
    _fn(WRITE)(3, 11, data.ctypes.data, data.size)
    ours = (tmp_path / "ours" / "wfs_3_11.bin").read_bytes()
    assert ours == (tmp_path / "ref" / "wfs_3_11.bin").read_bytes()
    assert len(ours) == 16 * data.size
    # the library reads the reference's file back
    monkeypatch.chdir(tmp_path / "ref")
    back = np.zeros_like(data)
    _fn(READ)(3, 11, back.ctypes.data, back.size)
    assert np.array_equal(back, data)


@pytest.mark.gpu
def test_rlm_mesh_export(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import rlmb
    from oracle import rlm as orlm, vsl
    n, g, sample = 16, 4, 1
    ctx = rlmb.Context(0)
    e, c = ctx.rlm_mesh_export(n, 1.0, 16.0, g, 1, sample, str(tmp_path))
    e2, c2 = ctx.rlm_mesh_solve(n, 1.0, 16.0, g, 1, sample, 1)
    ctx.close()
    assert np.array_equal(e, e2[0]) and np.array_equal(c, c2[0])
    p = orlm.RlmParams(n, 1.0, 16.0, g, 1, 1)
    cmn, cmt, cjm = orlm.prepare_coeff(p)
    x, y, s = vsl.rlm_disorder(p.impurity_num, p.L1, p.L2, p.seed, sample)
    vmn = orlm.potential_coeff(x, y, s, cmn, p.dim, p.off_head)
    files = sorted(os.listdir(tmp_path))
    assert len(files) == (g + 1) ** 2
    for t1 in range(g + 1):
        for t2 in range(g + 1):
            raw = np.fromfile(tmp_path / f"wfs_{t1}_{t2}.bin", np.complex128)
            assert raw.size == n * n
            X = raw.reshape(n, n).T                       # column k = eigenvector k
            M = orlm.assemble(p, vmn, cmt, cjm, t1, t2).reshape(n, n).T
            w = np.linalg.eigvalsh(M)
            assert np.linalg.norm(M @ X - X * w[None, :]) <= 1e-12 * np.linalg.norm(M)
            assert np.linalg.norm(X.conj().T @ X - np.eye(n)) <= 1e-12
