"""The reference-named C++ entry points (include/diag_wrappers_b200.h), called from C++ as
the reference's own call sites call them (tests/wrappers_check.cpp), against the oracle and
the reference's golden fixtures."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_ROOT, REPO, golden

LIBDIR = os.path.join(PKG_ROOT, "lib")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if not os.path.exists(os.path.join(LIBDIR, "librlmb.so")):
        pytest.skip("library not built")
    exe = str(tmp_path_factory.mktemp("wrap") / "wrappers_check")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(REPO, "tests", "wrappers_check.cpp"),
                    "-I" + os.path.join(REPO, "include"), "-I" + os.path.join(cuda, "include"),
                    "-L" + LIBDIR, "-lrlmb", "-L" + os.path.join(cuda, "lib64"), "-lcudart",
                    "-Wl,-rpath," + LIBDIR + ":" + os.path.join(cuda, "lib64"), "-o", exe], check=True)
    return exe


def _call(exe, *args):
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stderr == "", r.stderr     # the wrappers report failures on stderr


def test_host_tables_and_disorder_wrappers(harness, tmp_path):
    d = golden("rlm_n32_g4_c1_s7.npz")
    n_phi, o, g = int(d["n_phi"]), int(d["off_head"]), int(d["n_mesh"])
    L = float(np.sqrt(n_phi * float(d["qc"])))
    out = tmp_path / "t.bin"
    _call(harness, "tables", out, n_phi, o, g, repr(L))
    raw = np.fromfile(out, np.complex128)
    dim = 2 * o + 1
    assert np.array_equal(raw[:dim * dim], d["coeff_mn"])
    assert np.array_equal(raw[dim * dim:dim * dim + (g + 1) * dim], d["coeff_m_theta"])
    assert np.array_equal(raw[dim * dim + (g + 1) * dim:], d["coeff_jm"])
    nimp = int(d["impurity_num"])
    _call(harness, "disorder", out, nimp, repr(L), int(d["seed"]), 0)
    raw = np.fromfile(out, np.float64)
    assert np.array_equal(raw[:nimp], d["x"][0]) and np.array_equal(raw[2 * nimp:], d["s"][0])


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
def test_mkl_heevd_wrapper(harness, tmp_path):
    _gpu()
    rng = np.random.default_rng(5)
    n = 40
    a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    M = (a + a.conj().T) / 2
    inp = tmp_path / "in.bin"
    M.T.astype(np.complex128).tofile(inp)          # column-major
    _call(harness, "heevd", inp, tmp_path / "out.bin", n)
    raw = np.fromfile(tmp_path / "out.bin", np.float64)
    w = raw[:n]
    X = raw[n:].view(np.complex128).reshape(n, n).T   # columns = eigenvectors
    assert np.abs(w - np.linalg.eigvalsh(M)).max() <= 1e-12 * np.abs(w).max()
    assert np.linalg.norm(M @ X - X * w) <= 1e-12 * np.linalg.norm(M)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["cusolver", "magma"])
def test_single_precision_device_wrappers(harness, tmp_path, mode):
    _gpu()
    rng = np.random.default_rng(9)
    n = 33
    a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    M = (a + a.conj().T) / 2
    buf = M.T.astype(np.complex64)            # column-major: buf[c][r] = M[r][c]
    buf[np.tril_indices(n, -1)] = 99 + 99j     # garbage in the upper triangle: uplo = lower
    buf.tofile(tmp_path / "in.bin")
    _call(harness, mode, tmp_path / "in.bin", tmp_path / "out.bin", n)
    raw = np.fromfile(tmp_path / "out.bin", np.float32)
    w = raw[:n].astype(np.float64)
    X = raw[n:].view(np.complex64).reshape(n, n).T.astype(np.complex128)
    wref = np.linalg.eigvalsh(M.astype(np.complex64).astype(np.complex128))
    assert np.abs(w - wref).max() <= 1e-5 * np.abs(wref).max()
    assert np.linalg.norm(M @ X - X * w) <= 1e-5 * np.linalg.norm(M)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["chern", "peer"])
def test_chern_wrappers_match_reference_layout(harness, tmp_path, mode):
    _gpu()
    from oracle import fhs, rlm as orlm
    d = golden("rlm_n16_g8_c2_s1.npz")
    p = orlm.RlmParams(16, 1.0, 16.0, 8, 1, 1)
    X = orlm.run_sample(p, 0, keep=True)["eigvecs"]       # [(g+1), (g+1), N, N]
    g, N = 8, 16
    t1 = 3
    ring = np.empty((2, g + 1, N, N), np.complex128)
    ring[t1 % 2] = X[t1]
    ring[1 - t1 % 2] = X[t1 - 1]
    ring.tofile(tmp_path / "w.bin")
    _call(harness, mode, tmp_path / "w.bin", tmp_path / "c.bin", N, N, g, t1)
    got = np.fromfile(tmp_path / "c.bin", np.float64).reshape(N, g)   # [n][m]
    ref = fhs.line_chern(X[t1 - 1], X[t1]).T
    cols = range(g) if mode == "chern" else range(1, g, 2)
    for m in cols:
        assert np.abs(got[:, m] - ref[:, m]).max() < 1e-10
    if mode == "peer":
        assert np.all(got[:, 0::2] == -7.0)      # untouched plaquettes
    assert d is not None


@pytest.mark.gpu
def test_get_potential_coeff_wrapper(harness, tmp_path):
    _gpu()
    d = golden("rlm_n64_g4_c1_s3.npz")
    nimp, o = int(d["impurity_num"]), int(d["off_head"])
    dim = 2 * o + 1
    np.concatenate([d["x"][0], d["y"][0], d["s"][0], d["coeff_mn"].view(np.float64)]).tofile(tmp_path / "i.bin")
    _call(harness, "vmn", tmp_path / "i.bin", tmp_path / "v.bin", nimp, dim, o)
    v = np.fromfile(tmp_path / "v.bin", np.complex128)
    assert np.abs(v - d["v_mn"][0]).max() <= 1e-12 * np.abs(d["v_mn"][0]).max()


@pytest.mark.gpu
def test_prepare_potential_coeff_wrapper(harness, tmp_path):
    """The GPU driver's V_mn (rlm/potential_coeff.cu:3-26) from float device arrays, against
    the oracle's restatement of that kernel evaluated in double on the same float inputs."""
    _gpu()
    from oracle import rlm as orlm
    d = golden("rlm_n64_g4_c1_s3.npz")
    nimp, o = int(d["impurity_num"]), int(d["off_head"])
    dim = 2 * o + 1
    x, y, s = (d[k][0].astype(np.float32) for k in ("x", "y", "s"))
    cmn = d["coeff_mn"].astype(np.complex64)
    np.concatenate([x, y, s, cmn.view(np.float32)]).astype(np.float32).tofile(tmp_path / "i.bin")
    _call(harness, "vmngpu", tmp_path / "i.bin", tmp_path / "v.bin", nimp, dim, o)
    v = np.fromfile(tmp_path / "v.bin", np.complex64).astype(np.complex128)
    ref = orlm.gpu_potential_coeff(x.astype(np.float64), y.astype(np.float64), s.astype(np.float64),
                                   cmn.astype(np.complex128), dim, o)
    assert np.abs(v - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("n_phi,t1,t2", [(64, 1, 3), (30, 0, 2), (17, 4, 4)])
def test_set_hamil_matrix_wrapper(harness, tmp_path, n_phi, t1, t2):
    """The GPU driver's assembly (rlm/hamiltonian_rlm_gpu.cu:9-50) on float device tables,
    including orders that are not multiples of 8 (the reference's launch needs them)."""
    _gpu()
    import rlmb
    from oracle import rlm as orlm
    prm = rlmb.rlm_params(n_phi)
    o, dim, g = prm["off_head"], prm["dim"], 4
    _, cmt, cjm = rlmb.rlm_coeff_tables(n_phi, o, g, prm["L1"], prm["L2"])
    rng = np.random.default_rng(n_phi)
    v = (rng.normal(size=dim * dim) + 1j * rng.normal(size=dim * dim)).astype(np.complex64)
    ct1 = cmt[t1 * dim:(t1 + 1) * dim].astype(np.complex64)
    ct2 = cmt[t2 * dim:(t2 + 1) * dim].astype(np.complex64)
    cjm = cjm.astype(np.complex64)
    np.concatenate([ct1, ct2, cjm, v]).tofile(tmp_path / "i.bin")
    _call(harness, "sethamil", tmp_path / "i.bin", tmp_path / "h.bin", n_phi, o)
    h = np.fromfile(tmp_path / "h.bin", np.complex64).astype(np.complex128)
    ref = orlm.gpu_assemble(ct1.astype(np.complex128), ct2.astype(np.complex128), cjm.astype(np.complex128),
                            v.astype(np.complex128), n_phi, o)
    assert np.abs(h - ref).max() <= 1e-6 * np.abs(ref).max()
    H = h.reshape(n_phi, n_phi)
    off = ~np.eye(n_phi, dtype=bool)
    assert np.array_equal(H[off], np.conj(H.T)[off])   # every off-diagonal entry written, lower = conj(upper)


@pytest.mark.gpu
@pytest.mark.parametrize("t1", [3, 4])
def test_cal_chern_wfs_io_wrapper(harness, tmp_path, t1):
    """cal_Chern_wfs_IO (diag_wrappers/chern.cpp:77-123) on eigenvector files in the
    write_wfs layout, named by ring slot theta_1 % 2, against the oracle's plaquettes."""
    _gpu()
    from oracle import fhs, rlm as orlm
    p = orlm.RlmParams(16, 1.0, 16.0, 8, 1, 1)
    X = orlm.run_sample(p, 0, keep=True)["eigvecs"]       # [(g+1), (g+1), N, N]
    g, N = 8, 16
    for line in (t1 - 1, t1):
        for t2 in range(g + 1):
            X[line, t2].astype(np.complex128).tofile(tmp_path / f"wfs_{line % 2}_{t2}.bin")
    out = tmp_path / "c.bin"
    _call(harness, "chernio", tmp_path, out, N, N, g, t1)
    got = np.fromfile(out, np.float64).reshape(N, g)
    ref = fhs.line_chern(X[t1 - 1], X[t1]).T
    assert np.abs(got - ref).max() < 1e-10
