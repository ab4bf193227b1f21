"""GPU parity of every pipeline stage, called through the C ABI, against the oracle and the
reference's golden fixtures.

Tolerances (double precision throughout):
  eigenvalues        max|w - w_ref| <= 1e-12 * max|w_ref|   (reference: zheevd)
  residual           ||M X - X diag(w)||_F <= 1e-12 * ||M||_F
  orthogonality      ||X^H X - I||_F <= 1e-11
  H / V_mn entries   max|H - H_ref| <= 1e-12 * max|H_ref|
  Chern numbers      rint() identical, |C - C_ref| <= 1e-8
  twist energies     max|E - E_ref| <= 1e-10 * max|E_ref|
"""
import numpy as np
import pytest

from conftest import golden

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


def _hermitian(rng, n, kind="random"):
    if kind == "random":
        a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        return (a + a.conj().T) / 2
    if kind == "identity":
        return np.eye(n, dtype=np.complex128)
    if kind == "degenerate":
        q = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))[0]
        w = np.repeat(np.arange((n + 2) // 3, dtype=float), 3)[:n]
        return (q * w) @ q.conj().T
    if kind == "diagonal":
        return np.diag(rng.normal(size=n)).astype(np.complex128)
    if kind == "zero":
        return np.zeros((n, n), np.complex128)
    if kind == "blocks":
        h = np.zeros((n, n), np.complex128)
        b = _hermitian(rng, n // 2)
        h[: n // 2, : n // 2] = b
        h[n // 2 : 2 * (n // 2), n // 2 : 2 * (n // 2)] = b
        if n % 2:
            h[-1, -1] = 0.25
        return h
    if kind == "tridiag_split":
        h = np.diag(rng.normal(size=n)).astype(np.complex128)
        for i in range(n - 1):
            if i % 5 != 4:
                h[i, i + 1] = rng.normal() + 1j * rng.normal()
                h[i + 1, i] = np.conj(h[i, i + 1])
        return h
    raise ValueError(kind)


def _check_eig(M, w, X, wref):
    scale = max(np.abs(wref).max(), 1e-300)
    assert np.abs(w - wref).max() <= 1e-12 * scale + 1e-300, np.abs(w - wref).max() / scale
    nrm = max(np.linalg.norm(M), 1e-300)
    res = np.linalg.norm(M @ X - X * w[None, :])
    assert res <= 1e-12 * nrm + 1e-300, res / nrm
    orth = np.linalg.norm(X.conj().T @ X - np.eye(M.shape[0]))
    assert orth <= 1e-11, orth


def _run_heevd(ctx, mats):
    n = mats[0].shape[0]
    a = torch.tensor(np.stack([m.T for m in mats]), dtype=torch.complex128, device="cuda").contiguous()
    info = torch.zeros(len(mats), dtype=torch.int32, device="cuda")
    w = ctx.heevd(a, info=info)
    torch.cuda.synchronize()
    assert int(info.abs().sum()) == 0
    X = a.cpu().numpy()   # row k = eigenvector k
    return w.cpu().numpy(), [X[b].T for b in range(len(mats))]


@pytest.mark.parametrize("n", [1, 2, 3, 5, 16, 31, 32, 33, 64, 100, 128, 129, 200, 256, 300, 384, 457, 512])
def test_heevd_random(ctx, n):
    rng = np.random.default_rng(n)
    mats = [_hermitian(rng, n) for _ in range(3)]
    w, X = _run_heevd(ctx, mats)
    for b, M in enumerate(mats):
        _check_eig(M, w[b], X[b], np.linalg.eigvalsh(M))


@pytest.mark.parametrize("n", [700, 800, 1000, 1537])
def test_heevd_large_orders(ctx, n):
    """Orders past the register-resident back-transform (n > ~720 runs the blocked
    64-reflector path).  Norm-wise tolerances grow with n like LAPACK's own bounds."""
    rng = np.random.default_rng(n)
    mats = [_hermitian(rng, n) for _ in range(2)]
    w, X = _run_heevd(ctx, mats)
    for b, M in enumerate(mats):
        wref = np.linalg.eigvalsh(M)
        scale = np.abs(wref).max()
        assert np.abs(w[b] - wref).max() <= 1e-12 * scale
        res = np.linalg.norm(M @ X[b] - X[b] * w[b][None, :]) / np.linalg.norm(M)
        assert res <= 2e-15 * n, res
        orth = np.linalg.norm(X[b].conj().T @ X[b] - np.eye(n))
        assert orth <= 2e-14 * n, orth


@pytest.mark.parametrize("kind", ["identity", "degenerate", "diagonal", "zero", "blocks", "tridiag_split"])
@pytest.mark.parametrize("n", [7, 48, 160, 300])
def test_heevd_structured(ctx, kind, n):
    rng = np.random.default_rng(7 * n)
    M = _hermitian(rng, n, kind)
    w, X = _run_heevd(ctx, [M])
    wref = np.linalg.eigvalsh(M)
    if kind == "zero":
        assert np.abs(w[0]).max() == 0.0
        assert np.linalg.norm(X[0].conj().T @ X[0] - np.eye(n)) <= 1e-11
        return
    _check_eig(M, w[0], X[0], wref)


def test_heevd_reads_upper_triangle_only(ctx):
    rng = np.random.default_rng(3)
    M = _hermitian(rng, 20)
    buf = M.copy()
    buf[np.tril_indices(20, -1)] = 1e3 + 7j   # garbage below the diagonal, as LAPACK 'U' allows
    buf[np.diag_indices(20)] += 0.5j          # imaginary diagonal parts are ignored
    w, X = _run_heevd(ctx, [buf])
    _check_eig(M, w[0], X[0], np.linalg.eigvalsh(M))


def test_mkl_heevd_host_dropin(ctx):
    rng = np.random.default_rng(11)
    M = _hermitian(rng, 24)
    w, vec = ctx.mkl_heevd(M.T.reshape(-1).copy(), 24)   # column-major buffer
    X = vec.reshape(24, 24).T
    _check_eig(M, w, X, np.linalg.eigvalsh(M))


# -------------------------------------------------------------------------- rlm stages
def _rlm_setup(d):
    import rlmb
    n_phi, g = int(d["n_phi"]), int(d["n_mesh"])
    p = rlmb.rlm_params(n_phi, float(d["qc"]), float(d["ic"]))
    return n_phi, g, p


@pytest.mark.parametrize("name", ["rlm_n16_g8_c2_s1.npz", "rlm_n64_g4_c1_s3.npz", "rlm_n128_g2_c1_s5.npz"])
def test_rlm_potential_matches_reference(ctx, name):
    d = golden(name)
    n_phi, g, p = _rlm_setup(d)
    ns = int(d["n_sample"])
    x = torch.tensor(d["x"], device="cuda")
    y = torch.tensor(d["y"], device="cuda")
    s = torch.tensor(d["s"], device="cuda")
    cmn = torch.tensor(d["coeff_mn"], device="cuda")
    v = ctx.rlm_potential(x, y, s, cmn, p["off_head"]).cpu().numpy()
    for n in range(ns):
        ref = d["v_mn"][n]
        assert np.abs(v[n] - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("name", ["rlm_n16_g8_c2_s1.npz", "rlm_n32_g4_c1_s7.npz", "rlm_n128_g2_c1_s5.npz"])
def test_rlm_assemble_matches_oracle(ctx, name):
    from oracle import rlm as orlm
    d = golden(name)
    n_phi, g, p = _rlm_setup(d)
    op = orlm.RlmParams(n_phi, float(d["qc"]), float(d["ic"]), g, 1, int(d["seed"]))
    vmn = d["v_mn"][0]
    t1 = np.array([0, 1, g, g // 2, 0], np.int32)
    t2 = np.array([0, g, 1, g // 2, g], np.int32)
    H = ctx.rlm_assemble(torch.tensor(vmn, device="cuda"), torch.tensor(d["coeff_m_theta"], device="cuda"),
                         torch.tensor(d["coeff_jm"], device="cuda"), n_phi, p["off_head"], g, t1, t2)
    H = H.cpu().numpy()
    for i in range(len(t1)):
        ref = orlm.assemble(op, vmn, d["coeff_m_theta"], d["coeff_jm"], int(t1[i]), int(t2[i]))
        ref = ref.reshape(n_phi, n_phi)
        assert np.abs(H[i] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_rlm_eigenpairs_match_reference_kpoints(ctx):
    """Assemble + eigensolve at k-points whose reference eigenvectors are recorded."""
    from oracle import rlm as orlm
    for name in ("rlm_n16_g8_c2_s1.npz", "rlm_n32_g4_c1_s7.npz", "rlm_n64_g4_c1_s3.npz"):
        d = golden(name)
        n_phi, g, p = _rlm_setup(d)
        for key in d.files:
            if not key.startswith("eigvec_s"):
                continue
            _, sn, k1, k2 = key.split("_")
            sample, k1, k2 = int(sn[1:]), int(k1), int(k2)
            H = ctx.rlm_assemble(torch.tensor(d["v_mn"][sample], device="cuda"),
                                 torch.tensor(d["coeff_m_theta"], device="cuda"),
                                 torch.tensor(d["coeff_jm"], device="cuda"), n_phi, p["off_head"], g,
                                 [k1], [k2])
            w = ctx.heevd(H)
            torch.cuda.synchronize()
            wref = d["energies_mesh"][sample][k1, k2]
            assert np.abs(w.cpu().numpy()[0] - wref).max() <= 1e-12 * np.abs(wref).max()
            Xr = d[key].reshape(n_phi, n_phi)   # row n = reference eigenvector n
            Xg = H.cpu().numpy()[0]
            ov = np.abs(np.einsum("nr,nr->n", np.conj(Xr), Xg))
            assert np.abs(ov - 1).max() < 1e-9


@pytest.mark.parametrize("name", ["rlm_n16_g8_c2_s1.npz", "rlm_n32_g4_c1_s7.npz"])
def test_fhs_line_matches_oracle(ctx, name):
    from oracle import fhs, rlm as orlm
    d = golden(name)
    n_phi, g, p = _rlm_setup(d)
    op = orlm.RlmParams(n_phi, float(d["qc"]), float(d["ic"]), g, 1, int(d["seed"]))
    r = orlm.run_sample(op, 0, keep=True)
    X = r["eigvecs"]
    for t1 in (1, g):
        ref = fhs.line_chern(X[t1 - 1], X[t1])          # [g, N]
        out = ctx.fhs_line(torch.tensor(X[t1 - 1], device="cuda"), torch.tensor(X[t1], device="cuda"))
        assert np.abs(out.cpu().numpy().T - ref).max() < 1e-10


RLM_MESH = ["rlm_n16_g8_c2_s1.npz", "rlm_n32_g4_c1_s7.npz", "rlm_n64_g4_c1_s3.npz",
            "rlm_n128_g2_c1_s5.npz", "rlm_n16_g64_c2_s1.npz"]


@pytest.mark.parametrize("name", RLM_MESH)
def test_rlm_mesh_solve_matches_reference(ctx, name):
    d = golden(name)
    n_phi, g, p = _rlm_setup(d)
    ns = int(d["n_sample"])
    e, c = ctx.rlm_mesh_solve(n_phi, float(d["qc"]), float(d["ic"]), g, int(d["seed"]), 0, ns)
    for n in range(ns):
        eref, cref = d["energies"][n], d["chern"][n]
        assert np.abs(e[n] - eref).max() <= 1e-10 * np.abs(eref).max()
        assert np.array_equal(np.rint(c[n]), np.rint(cref))
        assert np.abs(c[n] - cref).max() < 1e-8


def test_rlm_mesh_solve_sample_offset(ctx):
    d = golden("rlm_n16_g8_c2_s1.npz")
    e, c = ctx.rlm_mesh_solve(16, 1.0, 16.0, 8, 1, 1, 1)
    assert np.abs(e[0] - d["energies"][1]).max() <= 1e-10 * np.abs(d["energies"][1]).max()
    assert np.array_equal(np.rint(c[0]), np.rint(d["chern"][1]))


# -------------------------------------------------------------------------- hlm stages
@pytest.mark.parametrize("name", ["hlm_6x6_q3_b0_g8_c2_s1.npz", "hlm_9x6_q3_b1_g8_c1_s2.npz",
                                  "hlm_8x8_q2_b0_g4_c1_s4.npz"])
def test_hlm_basis_matches_reference(ctx, name):
    d = golden(name)
    lx, ly, Q, b, g = (int(d[k]) for k in ("lx", "ly", "Q", "band", "n_mesh"))
    for key in d.files:
        if not key.startswith("basis_"):
            continue
        _, t1, t2 = key.split("_")
        W = ctx.hlm_basis(lx, ly, Q, b, g, int(t1), int(t2)).cpu().numpy()
        Wr = d[key].reshape(-1, lx * ly)
        ov = np.abs(np.einsum("cr,cr->c", np.conj(Wr), W))
        assert np.abs(ov - 1).max() < 1e-12


@pytest.mark.parametrize("name", ["hlm_6x6_q3_b0_g8_c2_s1.npz", "hlm_12x8_q3_b2_g8_c1_s2.npz",
                                  "hlm_48x16_q3_b0_g2_c1_s1.npz"])
def test_hlm_project_spectrum_matches_reference(ctx, name):
    d = golden(name)
    lx, ly, Q, b, g = (int(d[k]) for k in ("lx", "ly", "Q", "band", "n_mesh"))
    pot = torch.tensor(d["potentials"][0], device="cuda")
    t1 = np.array([0, 1, g, g], np.int32)
    t2 = np.array([0, g - 1, 0, g // 2], np.int32)
    H = ctx.hlm_project(lx, ly, Q, b, g, pot, t1, t2)
    Hn = H.cpu().numpy()
    for i in range(len(t1)):
        M = Hn[i].T
        assert np.abs(M - M.conj().T).max() < 1e-14 * max(1.0, np.abs(M).max())
        wref = d["energies_mesh"][0][t1[i], t2[i]]
        w = np.linalg.eigvalsh(M)
        assert np.abs(w - wref).max() <= 1e-12 * np.abs(wref).max()
    w = ctx.heevd(H).cpu().numpy()
    for i in range(len(t1)):
        wref = d["energies_mesh"][0][t1[i], t2[i]]
        assert np.abs(w[i] - wref).max() <= 1e-12 * np.abs(wref).max()


HLM_MESH = ["hlm_3x3_q3_g64_c2_s1.npz", "hlm_6x6_q3_b0_g8_c2_s1.npz", "hlm_9x6_q3_b1_g8_c1_s2.npz",
            "hlm_12x8_q3_b2_g8_c1_s2.npz", "hlm_48x16_q3_b0_g2_c1_s1.npz"]


@pytest.mark.parametrize("name", HLM_MESH)
def test_hlm_mesh_solve_matches_reference(ctx, name):
    d = golden(name)
    lx, ly, Q, b, g = (int(d[k]) for k in ("lx", "ly", "Q", "band", "n_mesh"))
    e, c = ctx.hlm_mesh_solve(lx, ly, Q, b, g, d["potentials"])
    for n in range(int(d["n_sample"])):
        eref, cref = d["energies"][n], d["chern"][n]
        assert np.abs(e[n] - eref).max() <= 1e-10 * np.abs(eref).max()
        assert np.array_equal(np.rint(c[n]), np.rint(cref))
        assert np.abs(c[n] - cref).max() < 1e-8


# ----------------------------------------------------- full-size geometries (reference fixtures)
def test_hlm_benchmark_geometry_matches_reference(ctx):
    """hlm 48x16, q=3, band 0, g=32 (the benchmarked configuration): samples 0, 5 and 22 of
    seed 1, whose per-state Chern sums the reference gives as 1, 2 and 0."""
    d = golden("hlm_48x16_q3_b0_g32_s1_full.npz")
    e, c = ctx.hlm_mesh_solve(48, 16, 3, 0, 32, d["potentials"])
    assert ctx.last_failures == 0
    for i in range(len(d["samples"])):
        eref, cref = d["energies"][i], d["chern"][i]
        assert np.abs(e[i] - eref).max() <= 1e-10 * np.abs(eref).max()
        assert np.array_equal(np.rint(c[i]), np.rint(cref))
        assert np.abs(c[i] - cref).max() < 1e-8
    assert [round(float(x)) for x in c.sum(axis=1)] == [round(float(x)) for x in d["chern"].sum(axis=1)]


def test_hlm_benchmark_geometry_samples_0_to_7(ctx):
    """hlm 48x16, q=3, band 0, g=32, seed 1: the first eight samples of a bench step, with the
    potentials drawn by the library's own generator."""
    import rlmb
    d = golden("hlm_48x16_q3_b0_g32_s1_samples0-7.npz")
    pots = rlmb.hlm_potentials(1, 768, 8)
    assert np.array_equal(pots, d["potentials"])
    e, c = ctx.hlm_mesh_solve(48, 16, 3, 0, 32, pots)
    assert ctx.last_failures == 0
    for i in range(8):
        eref, cref = d["energies"][i], d["chern"][i]
        assert np.abs(e[i] - eref).max() <= 1e-10 * np.abs(eref).max()
        assert np.array_equal(np.rint(c[i]), np.rint(cref))
        assert np.abs(c[i] - cref).max() < 1e-8


def test_rlm_512_samples_0_to_3(ctx):
    """rlm n_phi=512 (8192 impurities, g=16, seed 1): samples 0 .. 3 in one call."""
    d = golden("rlm_n512_g16_c4_s1_full.npz")
    e, c = ctx.rlm_mesh_solve(512, 1.0, 16.0, 16, 1, 0, 4)
    assert ctx.last_failures == 0
    for i in range(4):
        eref, cref = d["energies"][i], d["chern"][i]
        assert np.abs(e[i] - eref).max() <= 1e-10 * np.abs(eref).max()
        assert np.array_equal(np.rint(c[i]), np.rint(cref))
        assert np.abs(c[i] - cref).max() < 1e-8


@pytest.mark.parametrize("n_phi", [64, 128, 192, 256, 384, 512])
def test_rlm_finite_size_geometries_match_reference(ctx, n_phi):
    """rlm at the finite-size-scaling sizes (impurity concentration 16, g=16, seed 1, sample 0)."""
    d = golden(f"rlm_n{n_phi}_g16_c1_s1_full.npz")
    e, c = ctx.rlm_mesh_solve(n_phi, 1.0, 16.0, 16, 1, 0, 1)
    assert ctx.last_failures == 0
    eref, cref = d["energies"][0], d["chern"][0]
    assert np.abs(e[0] - eref).max() <= 1e-10 * np.abs(eref).max()
    assert np.array_equal(np.rint(c[0]), np.rint(cref))
    assert np.abs(c[0] - cref).max() < 1e-8


def test_rlm_large_order_matches_reference(ctx):
    """rlm at n_phi=3000 (48,000 impurities, g=4, seed 1, sample 0): 25 solves of order 3000."""
    import os
    from conftest import GOLDEN
    name = "rlm_n3000_g4_c1_s1_full.npz"
    if not os.path.exists(os.path.join(GOLDEN, name)):
        pytest.skip(f"{name} not generated")
    d = golden(name)
    e, c = ctx.rlm_mesh_solve(3000, 1.0, 16.0, 4, 1, 0, 1)
    assert ctx.last_failures == 0
    eref, cref = d["energies"][0], d["chern"][0]
    assert np.abs(e[0] - eref).max() <= 1e-10 * np.abs(eref).max()
    assert np.array_equal(np.rint(c[0]), np.rint(cref))
    assert np.abs(c[0] - cref).max() < 1e-8


# ------------------------------------------------------------- device disorder generation
@pytest.mark.parametrize("nimp,samples", [(256, [0, 1, 5]), (8192, [0, 3, 31]), (48000, [0, 7])])
def test_rlm_disorder_device_matches_host(ctx, nimp, samples):
    """MT19937 on the device, skipped per sample, equals the host stream bit for bit."""
    import rlmb
    L = float(np.sqrt(nimp / 16.0))
    lo, hi = min(samples), max(samples)
    x, y, s = (t.cpu().numpy() for t in ctx.rlm_disorder_device(nimp, L, L, 1, lo, hi - lo + 1))
    for smp in samples:
        hx, hy, hs = rlmb.rlm_disorder(nimp, L, L, 1, smp)
        k = smp - lo
        assert np.array_equal(x[k], hx) and np.array_equal(y[k], hy) and np.array_equal(s[k], hs)


@pytest.mark.parametrize("nimp", [256, 4096, 48000])
def test_rlm_disorder_device_continuation_matches_host(ctx, nimp):
    """Consecutive calls continue the context's saved MT19937 stream (one CTA draws the samples
    in order) instead of skipping ahead per sample: the draws are still the host stream's,
    bit for bit, including calls whose boundary falls inside a 624-output block, a call that
    jumps back (fresh skip), and a call that resumes after it."""
    import rlmb
    L = float(np.sqrt(nimp / 16.0))
    for lo, cnt in ((0, 2), (2, 3), (5, 1), (1, 2), (3, 2)):
        x, y, s = (t.cpu().numpy() for t in ctx.rlm_disorder_device(nimp, L, L, 7, lo, cnt))
        for k in range(cnt):
            hx, hy, hs = rlmb.rlm_disorder(nimp, L, L, 7, lo + k)
            assert np.array_equal(x[k], hx) and np.array_equal(y[k], hy) and np.array_equal(s[k], hs)


def test_hlm_potentials_device_matches_host(ctx):
    import rlmb
    host = rlmb.hlm_potentials(1, 768, 70)
    dev = ctx.hlm_potentials_device(1, 768, 3, 67).cpu().numpy()
    assert np.array_equal(dev, host[3:70])


@pytest.mark.parametrize("precision", [0, 1])
def test_fss_graph_matches_mesh_solve(ctx, precision):
    """Several orders in one captured CUDA graph, replayed for two sample blocks: every order's
    energies and Chern numbers equal the plain mesh solve of the same samples, and order 64
    sample 0 matches the reference fixture."""
    import rlmb
    sizes = (16, 48, 64)
    fg = rlmb.FssGraph(0, sizes, 1.0, 16.0, 4, 3, 2, precision)
    ctx.precision = precision
    try:
        for s0 in (0, 2):
            fg.launch(s0)
            for i, n in enumerate(sizes):
                e, c = fg.results(i)
                er, cr = ctx.rlm_mesh_solve(n, 1.0, 16.0, 4, 3, s0, 2)
                assert np.abs(e - er).max() <= 1e-12 * np.abs(er).max()
                assert np.array_equal(np.rint(c), np.rint(cr)) and np.abs(c - cr).max() < 1e-9
        fg.launch(0)
        d = golden("rlm_n64_g4_c1_s3.npz")
        e, c = fg.results(2)
        assert np.abs(e[0] - d["energies"][0]).max() <= 1e-10 * np.abs(d["energies"][0]).max()
        assert np.array_equal(np.rint(c[0]), np.rint(d["chern"][0]))
    finally:
        ctx.precision = 0
        fg.close()


@pytest.mark.parametrize("n", [100, 300])
def test_heevd_every_launch_configuration(n):
    """Each configuration the autotuner can pick gives a correct eigendecomposition."""
    import rlmb
    c = rlmb.Context(0)
    try:
        rng = np.random.default_rng(50 + n)
        mats = [_hermitian(rng, n) for _ in range(2)]
        for blocked in (0, 1):
            for gemm in (0, 1):
                for nt in (256, 512):
                    for xt in (64, 128):
                        for bs in ((64, 128) if gemm else (0,)):
                            c.set_heev_config(n, blocked, gemm, nt, xt, bs)
                            w, X = _run_heevd(c, mats)
                            for b, M in enumerate(mats):
                                _check_eig(M, w[b], X[b], np.linalg.eigvalsh(M))
    finally:
        c.close()


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("n,bs", [(1000, 128), (1000, 64), (1600, 0), (300, 128), (385, 128)])
def test_heevd_back_transformation_blocks(n, bs, mixed):
    """The GEMM back-transformation in blocks of 128 reflectors (T from two 64-reflector halves)
    against 64, at orders whose last block is partial in either half; 0 = the built-in choice
    (64)."""
    import rlmb
    c = rlmb.Context(0)
    try:
        if mixed:
            c.precision = c.MIXED
        c.set_heev_config(n, 1, 1, 0, 0, bs)
        assert c.heev_config(n)[1]["bt_block"] == (bs or 64)
        rng = np.random.default_rng(n + bs)
        mats = [_hermitian(rng, n) for _ in range(2)]
        w, X = _run_heevd(c, mats)
        tol = 1e-10 if mixed else 1e-12   # the mixed mode's bound (test_gpu_mixed) or FP64's
        for b, M in enumerate(mats):
            wref = np.linalg.eigvalsh(M)
            assert np.abs(w[b] - wref).max() <= tol * np.abs(wref).max()
            assert np.linalg.norm(M @ X[b] - X[b] * w[b][None, :]) <= tol * np.linalg.norm(M)
            assert np.linalg.norm(X[b].conj().T @ X[b] - np.eye(n)) <= (1e-10 if mixed else 1e-11)
    finally:
        c.close()


@pytest.mark.parametrize("qnt", [512, 256])
@pytest.mark.parametrize("mixed", [False, True])
def test_panel_queue_matches_per_matrix_panels(mixed, qnt):
    """A chunk of more matrices than SMs above order 512 runs its panels as resident CTAs (512
    threads one per SM, or 256 threads two per SM) taking (matrix, column) units from a queue;
    it must give the results of the one-CTA-per-matrix kernel (pinned with panel_threads =
    512), and no bounded wait may run out."""
    import rlmb
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    n, nb = 576, sms + 13
    rng = np.random.default_rng(5)
    a0 = rng.normal(size=(nb, n, n)) + 1j * rng.normal(size=(nb, n, n))
    a0 = a0 + np.conj(np.transpose(a0, (0, 2, 1)))
    out = []
    for nt in (0, 512):
        c = rlmb.Context(0)
        try:
            if mixed:
                c.precision = c.MIXED
            c.set_heev_config(n, 1, 1, nt, 0, 0)
            if nt == 0:
                c.set_panel_queue(n, qnt)
            a = torch.tensor(np.ascontiguousarray(np.transpose(a0, (0, 2, 1))), device="cuda")
            info = torch.zeros(nb, dtype=torch.int32, device="cuda")
            w = c.heevd(a, info=info)
            torch.cuda.synchronize()
            assert int(info.abs().sum()) == 0
            assert c.tc_fault_count() == 0
            out.append((w.cpu().numpy(), a.cpu().numpy()))
        finally:
            c.close()
    (wq, xq), (wp, xp) = out
    tol = 1e-10 if mixed else 1e-12
    assert np.abs(wq - wp).max() <= tol * np.abs(wp).max()
    for b in (0, nb // 2, nb - 1):
        M = a0[b]
        X = xq[b].T
        wref = np.linalg.eigvalsh(M)
        assert np.abs(wq[b] - wref).max() <= tol * np.abs(wref).max()
        assert np.linalg.norm(M @ X - X * wq[b][None, :]) <= tol * np.linalg.norm(M)
        assert np.linalg.norm(X.conj().T @ X - np.eye(n)) <= (1e-10 if mixed else 1e-11)


def test_heevd_autotune_picks_and_caches():
    import rlmb
    c = rlmb.Context(0)
    try:
        c.set_autotune(True)
        rng = np.random.default_rng(77)
        for n in (160, 320):
            assert c.heev_config(n)[0] is False
            mats = [_hermitian(rng, n) for _ in range(3)]
            w, X = _run_heevd(c, mats)
            for b, M in enumerate(mats):
                _check_eig(M, w[b], X[b], np.linalg.eigvalsh(M))
            tuned, cfg = c.heev_config(n)
            assert tuned and cfg["ms_per_matrix"] > 0 and cfg["x_tile"] in (64, 128)
            w2, X2 = _run_heevd(c, mats)    # cached choice
            assert np.abs(w2[0] - w[0]).max() <= 1e-12 * np.abs(w[0]).max()
    finally:
        c.close()


@pytest.mark.parametrize("n,width,mixed", [(300, 32, False), (700, 32, False), (1537, 16, False),
                                           (1100, 0, False), (1537, 16, True), (1100, 0, True), (700, 32, True)])
def test_heevd_panel_widths(n, width, mixed):
    """Panels of 16 and 32 columns (rank-32 / rank-64 updates) at orders where they are not the
    built-in width (0 = built-in: 32 from order 1024 in FP64, 16 in the mixed mode); the mixed
    mode's bound or FP64's, except the orthogonality of the mixed mode, 1e-9: at orders around
    1500, two refinement steps leave defects of 1e-10 .. 3e-10 (Frobenius norm over n^2 entries)
    on some random matrices, with either width."""
    import rlmb
    c = rlmb.Context(0)
    try:
        if mixed:
            c.precision = c.MIXED
        c.set_panel_width(n, width)
        rng = np.random.default_rng(n + width)
        mats = [_hermitian(rng, n) for _ in range(2)]
        w, X = _run_heevd(c, mats)
        tol = 1e-10 if mixed else 1e-12
        for b, M in enumerate(mats):
            wref = np.linalg.eigvalsh(M)
            assert np.abs(w[b] - wref).max() <= tol * np.abs(wref).max()
            assert np.linalg.norm(M @ X[b] - X[b] * w[b][None, :]) <= (tol if mixed else 2e-15 * n) * np.linalg.norm(M)
            orth = 1e-9 if mixed else 2e-14 * n
            assert np.linalg.norm(X[b].conj().T @ X[b] - np.eye(n)) <= orth
        with pytest.raises(rlmb.RlmbError):
            c.set_panel_width(n, 24)
    finally:
        c.close()


def _n3000_sample_fixtures():
    import os
    from conftest import GOLDEN
    return {k: os.path.join(GOLDEN, f"rlm_n3000_g4_s1_sample{k}.npz") for k in range(1, 8)
            if os.path.exists(os.path.join(GOLDEN, f"rlm_n3000_g4_s1_sample{k}.npz"))}


def test_rlm_3000_bench_step_samples(ctx):
    """rlm n_phi = 3000, g = 4, seed 1: the other samples of the headline bench step (1 .. 7,
    one reference file each) solved in one call, against the reference."""
    fx = _n3000_sample_fixtures()
    if not fx:
        pytest.skip("no n_phi = 3000 sample fixtures generated")
    lo, hi = min(fx), max(fx)
    e, c = ctx.rlm_mesh_solve(3000, 1.0, 16.0, 4, 1, lo, hi - lo + 1)
    assert ctx.last_failures == 0
    for k, path in fx.items():
        d = np.load(path)
        eref, cref = d["energies"][0], d["chern"][0]
        assert np.abs(e[k - lo] - eref).max() <= 1e-10 * np.abs(eref).max()
        assert np.array_equal(np.rint(c[k - lo]), np.rint(cref))
        assert np.abs(c[k - lo] - cref).max() < 1e-8
