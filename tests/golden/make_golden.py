"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference sources (it is never run by the tests):

    make -C oracle            # builds oracle/_ref from the reference's sources
    python tests/golden/make_golden.py

Every number stored here comes from the reference's own double-precision functions,
compiled unmodified into oracle/_ref/libref_{rlm,hlm}.so and driven in the order of
rlm/main_rlm_cpu.cpp:109-243 and hlm/main_hlm_cpu.cpp:75-197, or from the
reference's command-line programs oracle/_ref/{rlm,hlm}_cpu_dp (text output, 8
significant digits).  Seeds and sizes are recorded in each file.
"""
import ctypes
import math
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(REPO, "oracle", "_ref")

c_dp = ctypes.POINTER(ctypes.c_double)


def ptr(a):
    return a.ctypes.data_as(c_dp)


def rlm_lib():
    lib = ctypes.CDLL(os.path.join(REF, "libref_rlm.so"))
    for name in ("ref_rlm_prepare_coeff", "ref_rlm_disorder", "ref_rlm_potential",
                 "ref_rlm_solve_line", "ref_peer_cal_chern", "ref_mkl_heevd"):
        getattr(lib, name).restype = None
    return lib


def hlm_lib():
    lib = ctypes.CDLL(os.path.join(REF, "libref_hlm.so"))
    for name in ("ref_hlm_wfs_ktheta", "ref_hlm_solve_line", "ref_peer_cal_chern",
                 "ref_hlm_potentials", "ref_mkl_heevd"):
        getattr(lib, name).restype = None
    return lib


def rlm_reference(n_phi, qc, ic, g, n_sample, seed, threads=8, keep_kpoints=(), first=0):
    """Per-sample loop of rlm/main_rlm_cpu.cpp:109-243 over the reference's functions, for
    samples first .. n_sample - 1 (each sample's disorder is its own draw of the seeded stream)."""
    lib = rlm_lib()
    L1 = L2 = math.sqrt(n_phi * qc)
    n_imp = int(ic * n_phi / qc)
    o = int(math.sqrt(n_imp) / 2 + 1)
    d = 2 * o + 1
    cmn = np.zeros(d * d, np.complex128)
    cmt = np.zeros((g + 1) * d, np.complex128)
    cjm = np.zeros(n_phi * d, np.complex128)
    lib.ref_rlm_prepare_coeff(ptr(cmn), ptr(cmt), ptr(cjm), n_phi, o, d, d, g,
                              ctypes.c_double(L1), ctypes.c_double(L2))
    out = dict(n_phi=n_phi, qc=qc, ic=ic, n_mesh=g, n_sample=n_sample, seed=seed,
               impurity_num=n_imp, off_head=o, coeff_mn=cmn, coeff_m_theta=cmt, coeff_jm=cjm)
    E_all, C_all, Craw_all, emesh, x_all, y_all, s_all, v_all, lines_all = [], [], [], [], [], [], [], [], []
    kp = {}
    for n in range(first, n_sample):
        x = np.zeros(n_imp)
        y = np.zeros(n_imp)
        s = np.zeros(n_imp)
        lib.ref_rlm_disorder(ptr(x), ptr(y), ptr(s), n_imp, ctypes.c_double(L1),
                             ctypes.c_double(L2), ctypes.c_ulong(seed), n)
        v = np.zeros(d * d, np.complex128)
        lib.ref_rlm_potential(ptr(x), ptr(y), ptr(s), ptr(v), ptr(cmn), d, d, o, n_imp)
        wf = np.zeros(2 * (g + 1) * n_phi * n_phi, np.complex128)
        et = np.zeros((g + 1) * n_phi)
        ct = np.zeros(g * n_phi)
        energy = np.zeros(n_phi)
        chern = np.zeros(n_phi)
        em = np.zeros((g + 1, g + 1, n_phi))
        lines = np.zeros((g, n_phi))
        for t1 in range(g + 1):
            lib.ref_rlm_solve_line(t1, n_phi, g, d, o, ptr(wf), ptr(et), ptr(v), ptr(cjm), ptr(cmt), threads)
            em[t1] = et.reshape(g + 1, n_phi)
            for i in range(n_phi):
                for j in range(g + 1):
                    energy[i] += et[j * n_phi + i]
            for (ks, k1, k2) in keep_kpoints:
                if ks == n and k1 == t1:
                    sl = ((t1 % 2) * (g + 1) + k2) * n_phi * n_phi
                    kp[f"eigvec_s{n}_{k1}_{k2}"] = wf[sl:sl + n_phi * n_phi].copy()
            if t1 >= 1:
                lib.ref_peer_cal_chern(ptr(wf), ptr(ct), n_phi, n_phi, g, t1, threads)
                c2 = ct.reshape(n_phi, g)
                lines[t1 - 1] = c2.sum(axis=1)
                for k in range(n_phi):
                    for i in range(g):
                        chern[k] += ct[k * g + i]
        craw = chern.copy()
        for k in range(n_phi):
            energy[k] /= (g + 1) * (g + 1)
            chern[k] += 1.0 / n_phi
        E_all.append(energy)
        C_all.append(chern)
        Craw_all.append(craw)
        emesh.append(em)
        x_all.append(x)
        y_all.append(y)
        s_all.append(s)
        v_all.append(v)
        lines_all.append(lines)
    out.update(energies=np.array(E_all), chern=np.array(C_all), chern_raw=np.array(Craw_all),
               energies_mesh=np.array(emesh), x=np.array(x_all), y=np.array(y_all),
               s=np.array(s_all), v_mn=np.array(v_all), line_chern=np.array(lines_all), **kp)
    return out


def hlm_reference(lx, ly, Q, band, g, n_sample, seed, threads=8, keep_basis=(), only=None,
                  keep_mesh=True):
    """Per-sample loop of hlm/main_hlm_cpu.cpp:75-197 over the reference's functions
    (`only`: the subset of sample indices to solve; the potentials stream covers them all)."""
    lib = hlm_lib()
    n_sites = lx * ly
    n_phi = n_sites // Q
    dim_wfs = n_phi * n_sites
    pots = np.zeros(n_sample * n_sites)
    lib.ref_hlm_potentials(ctypes.c_ulong(seed), n_sites, n_sample, ptr(pots))
    pots = pots.reshape(n_sample, n_sites)
    out = dict(lx=lx, ly=ly, Q=Q, band=band, n_mesh=g, n_sample=n_sample, seed=seed, potentials=pots)
    for (t1, t2) in keep_basis:
        w = np.zeros(dim_wfs, np.complex128)
        lib.ref_hlm_wfs_ktheta(lx, ly, Q, band, g, t1, t2, ptr(w))
        out[f"basis_{t1}_{t2}"] = w
    E_all, C_all, emesh = [], [], []
    for n in (range(n_sample) if only is None else only):
        wf = np.zeros(2 * (g + 1) * dim_wfs, np.complex128)
        et = np.zeros((g + 1) * n_phi)
        ct = np.zeros(g * n_phi)
        energy = np.zeros(n_phi)
        chern = np.zeros(n_phi)
        em = np.zeros((g + 1, g, n_phi))
        for t1 in range(g + 1):
            lib.ref_hlm_solve_line(t1, lx, ly, Q, band, g, ptr(wf), ptr(et), ptr(pots[n]), threads)
            em[t1] = et.reshape(g + 1, n_phi)[:g]
            for i in range(n_phi):
                for j in range(g):
                    energy[i] += et[j * n_phi + i]
                energy[i] += et[i]
            if t1 >= 1:
                lib.ref_peer_cal_chern(ptr(wf), ptr(ct), n_phi, n_sites, g, t1, threads)
                for k in range(n_phi):
                    for i in range(g):
                        chern[k] += -ct[k * g + i]
        for k in range(n_phi):
            energy[k] /= (g + 1) * (g + 1)
        E_all.append(energy)
        C_all.append(chern)
        emesh.append(em)
    out.update(energies=np.array(E_all), chern=np.array(C_all))
    if keep_mesh:
        out["energies_mesh"] = np.array(emesh)
    if only is not None:
        out["samples"] = np.array(only)
        out["potentials"] = pots[list(only)]
    return out


def full_size(which):
    """Full-size fixtures at the benchmark geometries (final energies and Chern numbers)."""
    if which == "hlm":
        # the benchmarked hlm configuration (48 x 16, q=3, band 0, g=32, seed 1): samples 0, 5, 22
        # (5 and 22 are samples whose per-state FHS Chern numbers do not sum to 1)
        h = hlm_reference(48, 16, 3, 0, 32, 23, 1, only=[0, 5, 22], keep_mesh=False)
        np.savez_compressed(os.path.join(HERE, "hlm_48x16_q3_b0_g32_s1_full.npz"), **h)
    if which == "rlm":
        # rlm n_phi = 512 (g=16) and the finite-size-scaling sizes, sample 0 of seed 1
        for n_phi in (64, 128, 192, 256, 384, 512):
            r = rlm_reference(n_phi, 1.0, 16.0, 16, 1, 1)
            keep = ("n_phi", "qc", "ic", "n_mesh", "n_sample", "seed", "impurity_num", "off_head",
                    "energies", "chern", "chern_raw")
            np.savez_compressed(os.path.join(HERE, f"rlm_n{n_phi}_g16_c1_s1_full.npz"),
                                **{k: v for k, v in r.items() if k in keep})
    if which == "hlm8":
        # the benchmarked hlm configuration, samples 0 .. 7 (one eighth of a bench step)
        h = hlm_reference(48, 16, 3, 0, 32, 8, 1, only=list(range(8)), keep_mesh=False)
        np.savez_compressed(os.path.join(HERE, "hlm_48x16_q3_b0_g32_s1_samples0-7.npz"), **h)
    if which == "rlm512x4":
        # rlm n_phi = 512, g = 16, samples 0 .. 3 of seed 1
        r = rlm_reference(512, 1.0, 16.0, 16, 4, 1)
        keep = ("n_phi", "qc", "ic", "n_mesh", "n_sample", "seed", "impurity_num", "off_head",
                "energies", "chern", "chern_raw")
        np.savez_compressed(os.path.join(HERE, "rlm_n512_g16_c4_s1_full.npz"),
                            **{k: v for k, v in r.items() if k in keep})
    if which == "n3000":
        # the large rlm geometry (n_phi = 3000, 48,000 impurities, g=4), sample 0 of seed 1:
        # 25 reference zheevd calls of order 3000 (tens of minutes on 8 cores)
        r = rlm_reference(3000, 1.0, 16.0, 4, 1, 1, threads=8)
        keep = ("n_phi", "qc", "ic", "n_mesh", "n_sample", "seed", "impurity_num", "off_head",
                "energies", "chern", "chern_raw", "energies_mesh")
        np.savez_compressed(os.path.join(HERE, "rlm_n3000_g4_c1_s1_full.npz"),
                            **{k: v for k, v in r.items() if k in keep})


def rlm_n3000_samples(first, last, threads=8):
    """rlm n_phi = 3000, g = 4, seed 1: samples first .. last (the rest of the headline bench
    step, whose sample 0 is rlm_n3000_g4_c1_s1_full.npz), one file per sample so that the run can
    be split and resumed."""
    keep = ("n_phi", "qc", "ic", "n_mesh", "n_sample", "seed", "impurity_num", "off_head",
            "energies", "chern", "chern_raw")
    for smp in range(first, last + 1):
        path = os.path.join(HERE, f"rlm_n3000_g4_s1_sample{smp}.npz")
        if os.path.exists(path):
            continue
        r = rlm_reference(3000, 1.0, 16.0, 4, smp + 1, 1, threads=threads, first=smp)
        r["sample"] = np.array(smp)
        np.savez_compressed(path, sample=r["sample"], **{k: v for k, v in r.items() if k in keep})


def run_program(args, workdir):
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    subprocess.run(args, cwd=workdir, env=env, check=True, capture_output=True)
    txt = open(os.path.join(workdir, "energy_Chern_No.txt")).read()
    return txt


def main():
    if not os.path.exists(os.path.join(REF, "libref_rlm.so")):
        sys.exit("build oracle/_ref first: make -C oracle")
    # rlm, the reference's README configuration (rlm_cpu_dp -n 16 -i 16 -g 64 -c 2) with seed 1
    with tempfile.TemporaryDirectory() as td:
        txt = run_program([os.path.join(REF, "rlm_cpu_dp"), "-n", "16", "-i", "16", "-g", "64",
                           "-c", "2", "-s", "1", "-t", "8"], td)
    r = rlm_reference(16, 1.0, 16.0, 64, 2, 1)
    np.savez_compressed(os.path.join(HERE, "rlm_n16_g64_c2_s1.npz"), text=np.array(txt),
                        **{k: v for k, v in r.items() if k in (
                            "n_phi", "qc", "ic", "n_mesh", "n_sample", "seed", "impurity_num",
                            "off_head", "energies", "chern", "chern_raw", "coeff_mn",
                            "coeff_m_theta", "coeff_jm", "x", "y", "s", "v_mn", "line_chern")})
    # rlm with intermediates at small meshes
    for (n_phi, g, ns, seed, kps) in ((16, 8, 2, 1, ((0, 0, 0), (1, 3, 5))),
                                      (32, 4, 1, 7, ((0, 2, 1),)),
                                      (64, 4, 1, 3, ((0, 1, 2),)),
                                      (128, 2, 1, 5, ())):
        r = rlm_reference(n_phi, 1.0, 16.0, g, ns, seed, keep_kpoints=kps)
        np.savez_compressed(os.path.join(HERE, f"rlm_n{n_phi}_g{g}_c{ns}_s{seed}.npz"), **r)
    # hlm, the reference's README configuration (hlm_cpu_dp -x 3 -y 3 -q 3 -g 64 -b 0 -c 2)
    with tempfile.TemporaryDirectory() as td:
        txt = run_program([os.path.join(REF, "hlm_cpu_dp"), "-x", "3", "-y", "3", "-q", "3",
                           "-g", "64", "-b", "0", "-c", "2", "-s", "1", "-t", "8"], td)
    h = hlm_reference(3, 3, 3, 0, 64, 2, 1)
    np.savez_compressed(os.path.join(HERE, "hlm_3x3_q3_g64_c2_s1.npz"), text=np.array(txt), **h)
    # (8x8, Q=2 has touching subbands: some link overlaps vanish, so its Chern values are
    # rounding noise in the reference too; it pins energies and the Q=2 basis only)
    for (lx, ly, Q, b, g, ns, seed, kb) in ((6, 6, 3, 0, 8, 2, 1, ((0, 0), (3, 5))),
                                            (9, 6, 3, 1, 8, 1, 2, ((1, 2),)),
                                            (12, 8, 3, 2, 8, 1, 2, ()),
                                            (8, 8, 2, 0, 4, 1, 4, ((2, 3),)),
                                            (48, 16, 3, 0, 2, 1, 1, ())):
        h = hlm_reference(lx, ly, Q, b, g, ns, seed, keep_basis=kb)
        np.savez_compressed(os.path.join(HERE, f"hlm_{lx}x{ly}_q{Q}_b{b}_g{g}_c{ns}_s{seed}.npz"), **h)
    # hlm config-2 geometry through the reference program at a tiny mesh
    with tempfile.TemporaryDirectory() as td:
        txt = run_program([os.path.join(REF, "hlm_cpu_dp"), "-x", "48", "-y", "16", "-q", "3",
                           "-g", "2", "-b", "0", "-c", "1", "-s", "1", "-t", "8"], td)
    np.savez_compressed(os.path.join(HERE, "hlm_48x16_q3_g2_text.npz"), text=np.array(txt))
    # rlm n_phi=512 geometry through the reference program at a tiny mesh
    with tempfile.TemporaryDirectory() as td:
        txt = run_program([os.path.join(REF, "rlm_cpu_dp"), "-n", "512", "-i", "16", "-g", "1",
                           "-c", "1", "-s", "1", "-t", "8"], td)
    np.savez_compressed(os.path.join(HERE, "rlm_n512_g1_text.npz"), text=np.array(txt))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--n3000-samples":   # --n3000-samples FIRST LAST
        rlm_n3000_samples(int(sys.argv[2]), int(sys.argv[3]))
    elif len(sys.argv) > 1 and sys.argv[1] == "--full":
        for w in sys.argv[2:] or ["hlm", "rlm", "n3000"]:
            full_size(w)
    else:
        main()
