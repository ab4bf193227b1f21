#!/usr/bin/env python
"""Throughput of the twist-mesh pipeline on B200: k-point eigensolves/s and samples/hour.

Headline workload (the configuration the north-star target is stated on): random Landau-level
model, n_phi = 3000 (every k-point a 3000 x 3000 complex Hermitian eigenproblem, 144 MB in
complex128), 48,000 impurities with strengths +-1 at uniform positions (impurity
concentration 16), K-space cut o = 110, twist mesh g = 4 ((g+1)^2 = 25 k-points per sample),
8 disorder samples per step = 200 eigensolves plus the V_mn, assembly and Chern steps.  The
disorder is drawn on the device from the reference's seeded MT19937 stream (seed 1 + rank).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload rlm3000|hlm48x16|rlm512|fss]

value : FP64 mode, rlmb_rlm_mesh_solve_device per step (results stay in device memory).
e2e   : the host-buffer C-ABI call rlmb_rlm_mesh_solve (coefficient tables H2D, energies and
        Chern numbers D2H inside the timed region), FP64 mode.
mixed : the mixed-precision mode (tcgen05 tensor-core products, FP64 refinement) on the same
        samples, with its agreement with the FP64 mode and with the reference fixture, in two
        variants: one refinement step + the Rayleigh-quotient eigenvalue pass, and two steps.
        The headline mixed figure is the faster variant that meets the accuracy target in
        this run (energies within 1e-10 of the FP64 mode and of the fixture, Chern integers
        identical); the other is nested in it.
extra : the hlm 48x16 configuration (n_phi = 256, g = 32, 64 samples per step).
--impl reference : the reference's own CPU implementation (oracle/_ref, compiled from the
        reference sources) on this host's cores, one k-point per step.
Multi-GPU (torchrun): every rank solves its own samples (weak scaling, no data-path
collective); the step time is the max over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "random-landau-model_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "k-point eigensolves/s & samples/hr, mixed-refined vs FP64 GPU; Chern ints exact"
UNIT = "k-point eigensolves/s"
SEED = 1
# headline: rlm n_phi=3000, g=4, 8 samples per step
RLM_N, RLM_G, RLM_NS = 3000, 4, 8
RLM_KPTS = (RLM_G + 1) ** 2
RLM_FIXTURE = os.path.join(REPO, "tests", "golden", "rlm_n3000_g4_c1_s1_full.npz")
# hlm 48x16 (the extra block and --workload hlm48x16)
LX, LY, Q, BAND, G, NS = 48, 16, 3, 0, 32, 64
N_PHI = LX * LY // Q
N_SITES = LX * LY
KPTS = (G + 1) * G
SOLVES_PER_STEP = NS * KPTS


def _config(extra=None):
    c = {"workload": f"hlm {LX}x{LY} sites, flux 1/{Q}, band {BAND}, n_phi={N_PHI}, g={G} "
                     f"({KPTS} k-points/sample), {NS} samples/step, seed {SEED}+rank",
         "n_phi": N_PHI, "n_mesh": G, "samples_per_step": NS, "solves_per_step": SOLVES_PER_STEP,
         "precision": "fp64 (complex128) eigensolve, FP64 phase accumulation",
         "l2": "working set per step >> 126 MB L2 (each sample's 1056 matrices are 1.1 GB)"}
    if extra:
        c.update(extra)
    return c


def _rlm_config(extra=None):
    c = {"workload": f"rlm n_phi={RLM_N}, 48000 impurities (concentration 16, strengths +-1), K-space cut o=110, "
                     f"g={RLM_G} ({RLM_KPTS} k-points/sample), {RLM_NS} samples/step, seed {SEED}+rank",
         "n_phi": RLM_N, "n_mesh": RLM_G, "samples_per_step": RLM_NS, "solves_per_step": RLM_NS * RLM_KPTS,
         "precision": "fp64 (complex128) eigensolve, FP64 phase accumulation",
         "l2": "working set per step >> 126 MB L2 (each matrix is 144 MB; a step's 200 matrices are 29 GB)"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for nm, v in zip(names, r[4:8]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------- reference arm (CPU)
def _ref_hlm_lib():
    path = os.path.join(REPO, "oracle", "_ref", "libref_hlm.so")
    if not os.path.exists(path):
        return None, f"{path} not built (make -C oracle needs the reference sources)"
    lib = ctypes.CDLL(path)
    lib.ref_hlm_solve_line.restype = None
    lib.ref_peer_cal_chern.restype = None
    lib.ref_hlm_potentials.restype = None
    return lib, None


def _ref_line_runner(threads):
    """Closure running one theta_1 line of the reference hlm path (projection + heevd +
    back-transform for 32 k-points, then the FHS plaquettes of that line)."""
    import numpy as np
    lib, err = _ref_hlm_lib()
    if lib is None:
        return None, err
    c_dp = ctypes.POINTER(ctypes.c_double)
    pots = np.zeros(N_SITES)
    lib.ref_hlm_potentials(ctypes.c_ulong(SEED), N_SITES, 1, pots.ctypes.data_as(c_dp))
    dim_wfs = N_PHI * N_SITES
    wf = np.zeros(2 * (G + 1) * dim_wfs, np.complex128)
    et = np.zeros((G + 1) * N_PHI)
    ct = np.zeros(G * N_PHI)
    state = {"t1": 0}

    def run_line():
        t1 = state["t1"] % (G + 1)
        lib.ref_hlm_solve_line(t1, LX, LY, Q, BAND, G, wf.ctypes.data_as(c_dp), et.ctypes.data_as(c_dp),
                               pots.ctypes.data_as(c_dp), threads)
        if t1 >= 1:
            lib.ref_peer_cal_chern(wf.ctypes.data_as(c_dp), ct.ctypes.data_as(c_dp), N_PHI, N_SITES, G, t1,
                                   threads)
        state["t1"] += 1
        return G   # k-point solves in this line
    return run_line, None


def _ref_rlm_runner(threads):
    """Closure running one k-point of the reference rlm path at n_phi=3000 (assembly + zheevd
    by the reference's peer_solve_projected) per call, with the BLAS inside zheevd on
    `threads` threads.  V_mn of sample 0 is computed once at set-up (the reference's
    get_potential_coeff on slices of the impurities in parallel) and its time is reported
    separately."""
    import numpy as np
    os.environ["OPENBLAS_NUM_THREADS"] = str(threads)   # before the reference's BLAS loads
    path = os.path.join(REPO, "oracle", "_ref", "libref_rlm.so")
    if not os.path.exists(path):
        return None, f"{path} not built (make -C oracle needs the reference sources)", None
    lib = ctypes.CDLL(path)
    for fn in ("ref_rlm_prepare_coeff", "ref_rlm_disorder", "ref_rlm_potential", "ref_rlm_solve_list"):
        getattr(lib, fn).restype = None
    c_dp = ctypes.POINTER(ctypes.c_double)
    L = float(np.sqrt(RLM_N * 1.0))
    nimp = int(16.0 * RLM_N / 1.0)
    o = int(np.sqrt(nimp) / 2 + 1)
    d = 2 * o + 1
    cmn = np.zeros(d * d, np.complex128)
    cmt = np.zeros((RLM_G + 1) * d, np.complex128)
    cjm = np.zeros(RLM_N * d, np.complex128)
    lib.ref_rlm_prepare_coeff(cmn.ctypes.data_as(c_dp), cmt.ctypes.data_as(c_dp), cjm.ctypes.data_as(c_dp),
                              RLM_N, o, d, d, RLM_G, ctypes.c_double(L), ctypes.c_double(L))
    x, y, s = (np.zeros(nimp) for _ in range(3))
    lib.ref_rlm_disorder(x.ctypes.data_as(c_dp), y.ctypes.data_as(c_dp), s.ctypes.data_as(c_dp), nimp,
                         ctypes.c_double(L), ctypes.c_double(L), ctypes.c_ulong(SEED), 0)
    # V_mn is linear in the impurities: the reference's get_potential_coeff runs on `threads`
    # slices of them in parallel (ctypes releases the GIL) and the partial tables are summed
    from concurrent.futures import ThreadPoolExecutor
    bounds = [nimp * i // threads for i in range(threads + 1)]
    parts = [np.zeros(d * d, np.complex128) for _ in range(threads)]

    def part(i):
        lo, hi = bounds[i], bounds[i + 1]
        if hi > lo:
            xs, ys, ss = (np.ascontiguousarray(a[lo:hi]) for a in (x, y, s))
            lib.ref_rlm_potential(xs.ctypes.data_as(c_dp), ys.ctypes.data_as(c_dp), ss.ctypes.data_as(c_dp),
                                  parts[i].ctypes.data_as(c_dp), cmn.ctypes.data_as(c_dp), d, d, o, hi - lo)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(part, range(threads)))
    vmn = np.sum(parts, axis=0)
    vmn_s = time.perf_counter() - t0
    wf = np.zeros(2 * (RLM_G + 1) * RLM_N * RLM_N, np.complex128)
    et = np.zeros((RLM_G + 1) * RLM_N)
    state = {"k": 0}

    def run_point():
        k = state["k"] % RLM_KPTS
        t1, t2 = k // (RLM_G + 1), k % (RLM_G + 1)
        lst = (ctypes.c_int * 1)(t2)
        lib.ref_rlm_solve_list(t1, lst, 1, RLM_N, RLM_G, d, o, wf.ctypes.data_as(c_dp), et.ctypes.data_as(c_dp),
                               vmn.ctypes.data_as(c_dp), cjm.ctypes.data_as(c_dp), cmt.ctypes.data_as(c_dp), 1)
        state["k"] += 1
        return 1
    return run_point, None, vmn_s


def cpu_baseline_rlm(min_seconds=10.0, max_points=4):
    """The reference's own CPU rlm path at n_phi=3000 timed on this host (bounded sample: a
    few k-points, each assembly + zheevd with the BLAS on every host thread)."""
    threads = os.cpu_count() or 1
    run_point, err, vmn_s = _ref_rlm_runner(threads)
    if run_point is None:
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": err}
    solves, t0 = 0, time.perf_counter()
    while solves < max_points and (time.perf_counter() - t0 < min_seconds or solves < 1):
        solves += run_point()
    dt = time.perf_counter() - t0
    return {"value": solves / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"sample 0 of the rlm n_phi={RLM_N} g={RLM_G} workload: {solves} k-points (assembly + "
                      f"LAPACKE_zheevd by peer_solve_projected, BLAS on {threads} threads) in {dt:.1f} s; "
                      f"the per-sample V_mn (get_potential_coeff on {threads} threads) took {vmn_s:.1f} s and "
                      f"is not in the rate"}


def cpu_baseline(min_seconds=10.0, max_lines=G + 1):
    """The reference's own CPU path timed on this host (bounded sample of the workload)."""
    threads = os.cpu_count() or 1
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    run_line, err = _ref_line_runner(threads)
    if run_line is None:
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": err}
    run_line()   # line theta_1 = 0 (warm-up, not timed: it has no plaquettes)
    solves, t0 = 0, time.perf_counter()
    lines = 0
    while lines < max_lines - 1 and (time.perf_counter() - t0 < min_seconds or lines < 1):
        solves += run_line()
        lines += 1
    dt = time.perf_counter() - t0
    return {"value": solves / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"sample 0, theta_1 lines 1..{lines} ({solves} k-point solves: projection, "
                      f"zheevd, back-transform, FHS) with {threads} threads, {dt:.1f} s"}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.workload == "hlm48x16":
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        run_step, err = _ref_line_runner(threads)
        cfg = _config({"reference_step": f"one theta_1 line ({G} k-point solves + FHS) of sample 0"})
        sample = f"{args.steps} theta_1 lines of sample 0, {threads} threads"
        vmn_s = None
    else:
        run_step, err, vmn_s = _ref_rlm_runner(threads)
        cfg = _rlm_config({"reference_step": "one k-point (assembly + zheevd) of sample 0, BLAS on all host "
                                             "threads"})
        sample = f"{args.steps} k-points of sample 0, BLAS on {threads} threads"
    if run_step is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    # one untimed step warms the host code and caches (a k-point of order 3000 is seconds of
    # CPU work, so the run stays within minutes)
    for _ in range(min(args.warmup, 1)):
        run_step()
    solves, times = 0, []
    for _ in range(args.steps):
        t = time.perf_counter()
        solves += run_step()
        times.append(time.perf_counter() - t)
    total = sum(times)
    value = solves / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if vmn_s is not None:
        line["cpu_baseline"]["per_sample_vmn_s"] = vmn_s
    print(json.dumps(line))
# ------------------------------------------------------------------------- GPU arm
def _traffic_per_matrix(kernel, n=N_PHI):
    """DRAM bytes per matrix of `kernel` at order n from the committed ncu capture summaries
    (profiles/dram_traffic*.json), if one covers that order."""
    import glob
    for path in sorted(glob.glob(os.path.join(REPO, "profiles", "dram_traffic*.json"))):
        try:
            with open(path) as f:
                d = json.load(f)
            key = "k_hetrd_total" if kernel == "reduction" else kernel
            if d.get("n") == n and key in d.get("bytes_per_matrix", {}):
                return d["bytes_per_matrix"][key]
        except (OSError, ValueError):
            continue
    return None


# profile labels of the eigensolver: the reduction (16-column panels, their rank-32 GEMM
# updates, the unblocked tail), the tridiagonal solve, the back-transformation
REDUCTION_LABELS = ("k_hetrd_panel", "k_hetrd_her2k", "k_hetrd")
EIG_LABELS = REDUCTION_LABELS + ("k_stebz", "k_stein", "k_larft", "k_ormtr")


def _with_reduction(prof):
    """Profile {label: (ms, launches)} with the reduction's labels also summed as 'reduction'."""
    out = dict(prof)
    ms = sum(prof.get(k, (0, 0))[0] for k in REDUCTION_LABELS)
    ln = sum(prof.get(k, (0, 0))[1] for k in REDUCTION_LABELS)
    if ln:
        out["reduction"] = (ms, ln)
    return out


# algorithmic DRAM bytes per matrix of the blocked reduction's panels at order n (FP64): the
# stored triangle of the leading c x c block read once for every column c the panels reduce
# (columns n-1 down to the unblocked tail's order; panels of 16 columns, tail order < 64 + 16)
def _panel_bytes_per_matrix(n, width=16, tail=64, elem=16):
    npanels = (n - tail + width - 1) // width if n >= 256 else 0
    m_tail = n - npanels * width
    return elem * sum(c * (c + 1) / 2 for c in range(m_tail, n))


# algorithmic FP64 flops per matrix of n_phi (LAPACK counts: zhetrd 16/3 n^3, zunmtr 8 n^3)
def _kernel_flops_per_matrix(kernel, n):
    return {"reduction": 16.0 / 3.0 * n ** 3, "k_ormtr": 8.0 * n ** 3}.get(kernel)


def run_gpu(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import rlmb

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    ctx = rlmb.Context(local)
    pots_h = rlmb.hlm_potentials(SEED + rank, N_SITES, NS)
    d_pot = torch.tensor(pots_h, device="cuda")
    d_e = torch.empty((NS, N_PHI), dtype=torch.float64, device="cuda")
    d_c = torch.empty((NS, N_PHI), dtype=torch.float64, device="cuda")
    pinned = torch.from_numpy(pots_h).pin_memory()

    def step_device():
        ctx.hlm_mesh_solve_device(LX, LY, Q, BAND, G, d_pot, d_e, d_c)

    def step_e2e():
        return ctx.hlm_mesh_solve(LX, LY, Q, BAND, G, pinned.numpy())

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        step_device()
    barrier()
    # ---- value: device-resident inputs
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ctx.profile(True)
    launches0 = ctx.launches
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step_device()
    ev1.record()
    barrier()
    ms_dev = max_over_ranks(ev0.elapsed_time(ev1))
    launches = ctx.launches - launches0
    prof = ctx.profile_report()
    ctx.profile(False)
    clk = clocks.stop()
    # results sanity: every Chern number integral (the per-state FHS sum need not be 1: the
    # reference gives 2 or 0 for some samples of this mesh as well, e.g. seed 1 samples 5, 22)
    c = d_c.cpu().numpy()
    chern_ok = bool(np.abs(c - np.rint(c)).max() < 1e-6)
    sum_rule_fraction = float(np.mean(np.abs(c.sum(axis=1) - 1) < 1e-6))
    # ---- e2e: host buffers through the C ABI
    step_e2e()
    barrier()
    ev0.record()
    for _ in range(args.steps):
        step_e2e()
    ev1.record()
    barrier()
    ms_e2e = max_over_ranks(ev0.elapsed_time(ev1))

    # ---- the mixed-precision mode on the same inputs (device-resident, same step)
    mixed = None
    if not args.no_mixed:
        c64 = d_c.cpu().numpy()
        e64 = d_e.cpu().numpy()
        ctx.precision = ctx.MIXED
        step_device()
        barrier()
        ctx.profile(True)
        ev0.record()
        for _ in range(args.steps):
            step_device()
        ev1.record()
        barrier()
        ms_mix = max_over_ranks(ev0.elapsed_time(ev1))
        prof_mix = ctx.profile_report()
        ctx.profile(False)
        ctx.precision = ctx.FP64
        cm_, em_ = d_c.cpu().numpy(), d_e.cpu().numpy()
        v_mix = ws * SOLVES_PER_STEP * args.steps / (ms_mix * 1e-3)
        mixed = {"value": v_mix, "unit": UNIT, "ms_per_step": ms_mix / args.steps,
                 "samples_per_hour": v_mix / KPTS * 3600.0,
                 "refinement_steps": 2,
                 "chern_integers_identical_to_fp64": bool(np.array_equal(np.rint(cm_), np.rint(c64))),
                 "max_chern_deviation_from_fp64": float(np.abs(cm_ - c64).max()),
                 "max_energy_rel_error_vs_fp64": float(np.abs(em_ - e64).max() / np.abs(e64).max()),
                 "kernel_ms_per_step": {k: v[0] / args.steps for k, v in sorted(prof_mix.items())}}

    value = ws * SOLVES_PER_STEP * args.steps / (ms_dev * 1e-3)
    e2e = ws * SOLVES_PER_STEP * args.steps / (ms_e2e * 1e-3)
    line = None
    if rank == 0:
        peak = ctx.fp64_peak_tflops()
        # dominant kernel of the timed region and its roofline
        prof_r = {k: v for k, v in _with_reduction(prof).items() if k not in REDUCTION_LABELS}
        kname, (kms, klaunch) = max(prof_r.items(), key=lambda kv: kv[1][0])
        fpm = _kernel_flops_per_matrix(kname, N_PHI)
        total_ms = sum(v[0] for v in prof.values())
        roof = None
        if fpm is not None:
            matrices_per_launch = SOLVES_PER_STEP * args.steps / klaunch
            achieved = fpm * matrices_per_launch / (kms / klaunch * 1e-3) / 1e12
            tr = _traffic_per_matrix(kname)
            roof = {"bound": "fp64", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak,
                    "traffic": tr * matrices_per_launch if tr is not None else None,
                    "peak_source": "measured in this run: FP64 FMA throughput probe "
                                   "(MEASURED_PEAKS.json holds no FP64 figure)",
                    "share_of_gpu_time": kms / total_ms,
                    "launches": klaunch,
                    "note": "per launch = averaged over the label's launches ('reduction' sums the "
                            "labels k_hetrd_panel, k_hetrd_her2k and the unblocked tail k_hetrd); traffic = ncu "
                            "DRAM bytes per matrix (profiles/dram_traffic.json) x matrices per launch"}
        eig_ms = sum(prof.get(k, (0, 0))[0] for k in EIG_LABELS)
        eig_tflops = 13.33 * N_PHI ** 3 * SOLVES_PER_STEP * args.steps / (eig_ms * 1e-3) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config({"parallelism": f"replicas x{ws} (sample-sharded)",
                               "samples_per_hour": value / KPTS * 3600.0,
                               "chern_integral": chern_ok,
                               "fraction_of_samples_with_sum_1": sum_rule_fraction,
                               "eigensolve_failures": int(ctx.last_failures)}),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(pots_h.nbytes),
                    "d2h_bytes_per_step": int(2 * NS * N_PHI * 8)},
            "roofline": roof,
            "eigensolve_roofline": {"flops_per_solve": "13.33 n^3",
                                    "kernels": "hetrd_panel+hetrd_her2k+hetrd+stebz+stein+larft+ormtr",
                                    "achieved_tflops": eig_tflops, "peak_tflops": peak,
                                    "frac": eig_tflops / peak},
            "mixed": mixed,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in sorted(prof.items())},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
    if ws > 1:
        dist.barrier()
    ctx.close()
    if rank == 0:
        line["cpu_baseline"] = cpu_baseline() if ws == 1 else None
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


RLM_WORKLOADS = {
    # name: (n_phi, g, samples per step) -- rlm with impurity concentration 16, +-1 strengths
    "rlm512": (512, 16, 32),
}


def run_gpu_rlm(args):
    """rlm workloads (n_phi=512, g=16, 32 samples; n_phi=3000, g=4, 8 samples): one
    rlmb_rlm_mesh_solve call per step (host disorder generation, device assembly, eigensolve
    and Chern step, energies and Chern numbers returned to the host), both precisions.
    Each step solves new samples (sample index advances by the samples per step)."""
    import numpy as np
    import torch
    import rlmb
    ws, rank, local = _dist()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    n_phi, g, ns = RLM_WORKLOADS[args.workload]
    kpts = (g + 1) ** 2
    ctx = rlmb.Context(local)
    out = {}
    for mode in ("fp64", "mixed"):
        ctx.precision = ctx.MIXED if mode == "mixed" else ctx.FP64
        sample = 0
        for _ in range(args.warmup):
            ctx.rlm_mesh_solve(n_phi, 1.0, 16.0, g, SEED, sample, ns)
            sample += ns
        ctx.profile(True)
        l0 = ctx.launches
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = []
        for _ in range(args.steps):
            res.append(ctx.rlm_mesh_solve(n_phi, 1.0, 16.0, g, SEED, sample, ns))
            sample += ns
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        prof = ctx.profile_report()
        ctx.profile(False)
        v = ns * kpts * args.steps / dt
        out[mode] = {"value": v, "ms_per_step": 1e3 * dt / args.steps, "samples_per_hour": v / kpts * 3600,
                     "launches": ctx.launches - l0, "results": res,
                     "kernel_ms_per_step": {k: x[0] / args.steps for k, x in sorted(prof.items())}}
    c64 = np.concatenate([r[1] for r in out["fp64"]["results"]])
    cmx = np.concatenate([r[1] for r in out["mixed"]["results"]])
    e64 = np.concatenate([r[0] for r in out["fp64"]["results"]])
    emx = np.concatenate([r[0] for r in out["mixed"]["results"]])
    f, m = out["fp64"], out["mixed"]
    line = {"metric": METRIC, "value": f["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": f["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"rlm n_phi={n_phi}, impurity concentration 16 (+-1 strengths), "
                                   f"g={g} ({kpts} k-points/sample), {ns} samples/step, seed {SEED}",
                       "api": "rlmb_rlm_mesh_solve (host results; disorder drawn on the host)",
                       "samples_per_hour": f["samples_per_hour"],
                       "l2": f"each matrix is {16 * n_phi * n_phi / 1e6:.1f} MB; a step's matrices exceed L2"},
            "kernel_ms_per_step": f["kernel_ms_per_step"], "gpu_launches": f["launches"],
            "mixed": {"value": m["value"], "ms_per_step": m["ms_per_step"],
                      "samples_per_hour": m["samples_per_hour"], "refinement_steps": 2,
                      "chern_integers_identical_to_fp64": bool(np.array_equal(np.rint(cmx), np.rint(c64))),
                      "max_chern_deviation_from_fp64": float(np.abs(cmx - c64).max()),
                      "max_energy_rel_error_vs_fp64": float(np.abs(emx - e64).max() / np.abs(e64).max()),
                      "kernel_ms_per_step": m["kernel_ms_per_step"]}}
    ctx.close()
    print(json.dumps(line), flush=True)


def _measured_peaks():
    """MEASURED_PEAKS.json (written by the pool's driver beside the repository), or {}."""
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _peak(peaks, key, fallback):
    v = peaks.get(key)
    if isinstance(v, (int, float)) and v > 0:
        return float(v), "measured"
    return fallback, "fallback"


def _hlm_extra(ctx, steps=2):
    """The hlm 48x16 configuration (n_phi=256, g=32, 64 samples per step), both modes, device
    resident, a short run nested in the headline line."""
    import numpy as np
    import torch
    import rlmb
    pots = torch.tensor(rlmb.hlm_potentials(SEED, N_SITES, NS), device="cuda")
    d_e = torch.empty((NS, N_PHI), dtype=torch.float64, device="cuda")
    d_c = torch.empty((NS, N_PHI), dtype=torch.float64, device="cuda")
    out = {"workload": _config()["workload"]}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = {}
    for mode in ("fp64", "mixed"):
        ctx.precision = ctx.MIXED if mode == "mixed" else ctx.FP64
        ctx.hlm_mesh_solve_device(LX, LY, Q, BAND, G, pots, d_e, d_c)
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(steps):
            ctx.hlm_mesh_solve_device(LX, LY, Q, BAND, G, pots, d_e, d_c)
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        res[mode] = (d_e.cpu().numpy(), d_c.cpu().numpy())
        out[mode] = {"value": SOLVES_PER_STEP / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                     "samples_per_hour": NS / (ms * 1e-3) * 3600.0, "steps": steps, "warmup": 1}
    ctx.precision = ctx.FP64
    (e64, c64), (em, cm) = res["fp64"], res["mixed"]
    out["chern_integral"] = bool(np.abs(c64 - np.rint(c64)).max() < 1e-6)
    out["mixed"]["chern_integers_identical_to_fp64"] = bool(np.array_equal(np.rint(cm), np.rint(c64)))
    out["mixed"]["max_energy_rel_error_vs_fp64"] = float(np.abs(em - e64).max() / np.abs(e64).max())
    return out


def run_headline(args):
    """The headline: rlm n_phi=3000, g=4, 8 samples per step (see the module docstring)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import rlmb

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    ctx = rlmb.Context(local)
    n, g, ns = RLM_N, RLM_G, RLM_NS
    seed = SEED + rank
    solves = ns * RLM_KPTS
    d_e = torch.empty((ns, n), dtype=torch.float64, device="cuda")
    d_c = torch.empty((ns, n), dtype=torch.float64, device="cuda")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # Sample indices stay small: the device draws sample s's disorder by skipping its MT19937
    # stream ahead 3 * 48000 * s outputs, a cost that grows with s.
    spare = [args.steps]   # next unused block of ns samples (blocks 0 .. steps-1 are the timed ones)

    def fresh():
        spare[0] += 1
        return ns * (spare[0] - 1)

    def timed(mode, steps, warmup, sampler=None):
        """Warm-up steps on samples outside the timed range, then `steps` timed steps whose last
        one solves samples 0 .. ns-1 (left in d_e, d_c).  Returns (max-over-ranks ms, profile,
        launches, clocks)."""
        ctx.precision = ctx.MIXED if mode == "mixed" else ctx.FP64
        for w in range(warmup):
            ctx.rlm_mesh_solve_device(n, 1.0, 16.0, g, seed, fresh(), d_e, d_c)
        barrier()
        if sampler:
            sampler.start()
        ctx.profile(True)
        l0 = ctx.launches
        barrier()
        ev0.record()
        for i in range(steps):
            ctx.rlm_mesh_solve_device(n, 1.0, 16.0, g, seed, ns * (steps - 1 - i), d_e, d_c)
        ev1.record()
        barrier()
        ms = max_over_ranks(ev0.elapsed_time(ev1))
        launches = ctx.launches - l0
        prof = ctx.profile_report()
        ctx.profile(False)
        clk = sampler.stop() if sampler else None
        return ms, prof, launches, clk

    # ---- value: FP64 mode, device-resident results
    ms_dev, prof, launches, clk = timed("fp64", args.steps, args.warmup, ClockSampler(torch.cuda.current_device()))
    e64, c64 = d_e.cpu().numpy(), d_c.cpu().numpy()
    # ---- e2e: the host-buffer C ABI (tables H2D, results D2H inside the timed region), FP64
    e2e_steps = max(1, min(args.steps, 3))
    ctx.precision = ctx.FP64
    ctx.rlm_mesh_solve(n, 1.0, 16.0, g, seed, fresh(), ns)
    e2e_samples = [fresh() for _ in range(e2e_steps)]
    barrier()
    ev0.record()
    for s0 in e2e_samples:
        ctx.rlm_mesh_solve(n, 1.0, 16.0, g, seed, s0, ns)
    ev1.record()
    barrier()
    ms_e2e = max_over_ranks(ev0.elapsed_time(ev1))
    # ---- mixed mode on the same samples: one refinement step + the Rayleigh-quotient
    #      eigenvalue pass (the accuracy the energies and Chern numbers need) ...
    mq_steps = max(1, min(args.steps, 5))
    ctx.set_refinement_steps(1)
    ctx.set_eigenvalue_pass(True)
    ms_rq, prof_rq, _, _ = timed("mixed", mq_steps, 3)
    erq, crq = d_e.cpu().numpy(), d_c.cpu().numpy()
    ctx.set_eigenvalue_pass(False)
    ctx.set_refinement_steps(2)
    # ---- ... and two refinement steps (double-precision eigenvectors as well)
    m_steps = max(1, min(args.steps, 3))
    ms_mix, prof_mix, _, _ = timed("mixed", m_steps, 3)
    em, cm = d_e.cpu().numpy(), d_c.cpu().numpy()
    ctx.precision = ctx.FP64
    faults = ctx.tc_fault_count()
    extra = _hlm_extra(ctx) if (ws == 1 and not args.no_extra) else None

    value = ws * solves * args.steps / (ms_dev * 1e-3)
    e2e = ws * solves * e2e_steps / (ms_e2e * 1e-3)
    v_mix = ws * solves * m_steps / (ms_mix * 1e-3)
    v_rq = ws * solves * mq_steps / (ms_rq * 1e-3)
    line = None
    if rank == 0:
        peaks = _measured_peaks()
        fp64_peak = ctx.fp64_peak_tflops()
        hbm, hbm_src = _peak(peaks, "hbm_gbs", 6650.0)
        bf16, bf16_src = _peak(peaks, "bf16_tflops_sustained", 1400.0)
        # parity of sample 0 against the reference's fixture (seed 1: rank 0)
        # (the last timed step solved samples 0 .. ns-1; sample 0's fixture holds the whole
        # reference output, samples 1 .. 7 have one file each where they were generated)
        par = None
        if seed == 1 and os.path.exists(RLM_FIXTURE):
            refs = {0: RLM_FIXTURE}
            for k in range(1, ns):
                fk = os.path.join(REPO, "tests", "golden", f"rlm_n3000_g4_s1_sample{k}.npz")
                if os.path.exists(fk):
                    refs[k] = fk
            par = {"fixtures": sorted({os.path.relpath(f, REPO) for f in refs.values()}),
                   "samples": sorted(refs)}
            for mode, (e, c) in (("fp64", (e64, c64)), ("mixed_one_step_rq", (erq, crq)),
                                 ("mixed_two_steps", (em, cm))):
                err, same, dev = 0.0, True, 0.0
                for k, f in refs.items():
                    fx = np.load(f)
                    eref, cref = fx["energies"][0], fx["chern"][0]
                    err = max(err, float(np.abs(e[k] - eref).max() / np.abs(eref).max()))
                    same = same and bool(np.array_equal(np.rint(c[k]), np.rint(cref)))
                    dev = max(dev, float(np.abs(c[k] - cref).max()))
                par[mode] = {"max_energy_rel_error": err, "chern_integers_identical": same,
                             "max_chern_deviation": dev}
        total_ms = sum(v[0] for v in prof.values())
        # the dominant kernel of the FP64 step, k_hetrd_panel, is bound by HBM: each column's
        # Hermitian matrix-vector product streams the stored triangle of the leading block
        roof = None
        if "k_hetrd_panel" in prof:
            pms, plaunch = prof["k_hetrd_panel"]
            bpm = _panel_bytes_per_matrix(n)
            achieved = bpm * solves * args.steps / (pms * 1e-3) / 1e9
            tr = _traffic_per_matrix("k_hetrd_panel", n)
            roof = {"bound": "hbm", "kernel": "k_hetrd_panel", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                    "frac": achieved / hbm,
                    "traffic": tr * solves * args.steps / plaunch if tr else None,
                    "peak_source": hbm_src, "share_of_gpu_time": pms / total_ms, "launches": plaunch,
                    "note": "algorithmic bytes = the stored triangle of the leading c x c block read once per "
                            "reduced column c (16 c(c+1)/2 B), summed over the panel columns, x matrices / the "
                            "label's summed CUDA-event time; traffic = ncu DRAM bytes per matrix (profiles/) x "
                            "matrices per launch"}
        # the reduction as a whole against the FP64 peak (algorithmic flops)
        red = _with_reduction(prof).get("reduction")
        red_roof = None
        if red:
            achieved = _kernel_flops_per_matrix("reduction", n) * solves * args.steps / (red[0] * 1e-3) / 1e12
            red_roof = {"bound": "fp64", "kernels": "k_hetrd_panel + k_hetrd_her2k + k_hetrd", "achieved": achieved,
                        "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                        "peak_source": "measured in this run: FP64 FMA throughput probe (MEASURED_PEAKS.json "
                                       "holds no FP64 figure)",
                        "share_of_gpu_time": red[0] / total_ms,
                        "note": "16/3 n^3 flops per matrix (LAPACK zhetrd count)"}
        eig_ms = sum(prof.get(k, (0, 0))[0] for k in EIG_LABELS)
        eig_tf = 13.33 * n ** 3 * solves * args.steps / (eig_ms * 1e-3) / 1e12
        # HBM-bound stages (a) assembly and (c) links / plaquettes: algorithmic bytes per step
        hbm_bytes = {"k_rlm_assemble": 16.0 * n * n * solves,          # H written once
                     "k_rlm_links": 16.0 * n * n * solves,             # each eigenvector matrix read once
                     "k_plaquettes": (2 * 16.0 + 8.0) * n * solves}    # U1, U2 read, W read
        roof_hbm = {}
        for k, b in hbm_bytes.items():
            if k in prof:
                gbs = b * args.steps / (prof[k][0] * 1e-3) / 1e9
                roof_hbm[k] = {"achieved_gbs": gbs, "peak_gbs": hbm, "frac": gbs / hbm, "peak_source": hbm_src}
        # tensor-core products of the mixed mode (tcgen05, split TF32: 3 products per term)
        tc = {}
        tf32_peak = bf16 / 2.0
        for k in ("k_ref_coupling", "k_ref_update"):
            if k in prof_mix:
                flops = 8.0 * n ** 3 * solves * m_steps * 2   # two refinement steps, one N^3 complex GEMM each
                tf = 3.0 * flops / (prof_mix[k][0] * 1e-3) / 1e12
                tc[k] = {"achieved_tf32_tflops": tf, "useful_complex_tflops": tf / 3.0, "peak_tf32_tflops": tf32_peak,
                         "frac": tf / tf32_peak,
                         "peak_source": f"{bf16_src} bf16 dense / 2 (TF32 runs at half the BF16 rate)"}
        def variant(v, ms, steps, e, c, prf, refinement):
            rec = {"value": v, "unit": UNIT, "ms_per_step": ms / steps, "steps": steps, "warmup": 3,
                   "samples_per_hour": v / RLM_KPTS * 3600.0,
                   "samples_per_hour_ratio_to_fp64": v / value,
                   "refinement": refinement,
                   "chern_integers_identical_to_fp64": bool(np.array_equal(np.rint(c), np.rint(c64))),
                   "max_chern_deviation_from_fp64": float(np.abs(c - c64).max()),
                   "max_energy_rel_error_vs_fp64": float(np.abs(e - e64).max() / np.abs(e64).max()),
                   "kernel_ms_per_step": {k: x[0] / steps for k, x in sorted(prf.items())}}
            # the north star's accuracy target, checked on this run's timed samples (against the
            # FP64 mode) and on sample 0 (against the reference's fixture)
            ok = rec["chern_integers_identical_to_fp64"] and rec["max_energy_rel_error_vs_fp64"] <= 1e-10
            return rec, ok
        rq, rq_ok = variant(v_rq, ms_rq, mq_steps, erq, crq, prof_rq,
                            "1 step + Rayleigh-quotient eigenvalues (rlmb_set_eigenvalue_pass)")
        two, two_ok = variant(v_mix, ms_mix, m_steps, em, cm, prof_mix, "2 steps")
        two["tensor_core_roofline"] = tc
        if par:
            rq_ok = rq_ok and par["mixed_one_step_rq"]["max_energy_rel_error"] <= 1e-10 and \
                par["mixed_one_step_rq"]["chern_integers_identical"]
            two_ok = two_ok and par["mixed_two_steps"]["max_energy_rel_error"] <= 1e-10 and \
                par["mixed_two_steps"]["chern_integers_identical"]
        rq["meets_accuracy_target"], two["meets_accuracy_target"] = rq_ok, two_ok
        # headline mixed figure: the faster variant that meets the accuracy target
        if rq_ok and v_rq >= v_mix:
            mixed = dict(rq, two_refinement_steps=two)
        else:
            mixed = dict(two, one_refinement_step_rq=rq)
        mixed["tc_faults"] = faults
        nb = 2 * 221 * 221 + 2 * (g + 1) * 221 + 2 * n * 221   # coefficient tables (complex) ...
        h2d = 8 * nb + 2 * RLM_KPTS * ns * 4                    # ... + the theta lists
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _rlm_config({"parallelism": f"replicas x{ws} (sample-sharded)",
                                   "api": "rlmb_rlm_mesh_solve_device (value), rlmb_rlm_mesh_solve (e2e)",
                                   "samples_per_hour": value / RLM_KPTS * 3600.0,
                                   "chern_integral": bool(np.abs(c64 - np.rint(c64)).max() < 1e-6),
                                   "eigensolve_failures": int(ctx.last_failures)}),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(2 * ns * n * 8),
                    "steps": e2e_steps},
            "mixed": mixed,
            "parity": par,
            "roofline": roof,
            "reduction_roofline": red_roof,
            "eigensolve_roofline": {"flops_per_solve": "13.33 n^3",
                                    "kernels": "hetrd_panel+hetrd_her2k+hetrd+stebz+stein+larft+ormtr",
                                    "achieved_tflops": eig_tf, "peak_tflops": fp64_peak, "frac": eig_tf / fp64_peak},
            "roofline_hbm": roof_hbm,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in sorted(prof.items())},
            "gpu_launches": int(launches),
            "clocks": clk,
            "extra": {"hlm48x16": extra} if extra else None,
        }
    if ws > 1:
        dist.barrier()
    ctx.close()
    if rank == 0:
        line["cpu_baseline"] = cpu_baseline_rlm() if ws == 1 else None
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


FSS_SIZES = (64, 128, 192, 256, 384, 512)


def run_gpu_fss(args):
    """Finite-size-scaling workload: rlm with n_phi in FSS_SIZES, 16 samples each, g=16,
    impurity concentration 16, FP64.  Two forms of the same work: one rlmb_rlm_mesh_solve call
    per size per step (sizes one after another), and one CUDA-graph launch per step that runs
    every size on its own concurrent branch (rlmb_rlm_fss_graph_*).  Reports k-point solves/s
    per size (sequential form) and for the whole step in both forms, and each size's
    eigensolver throughput against the FP64 roofline (13.33 n^3 flops per solve)."""
    import numpy as np
    import torch
    import rlmb
    ws, rank, local = _dist()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    g, ns = 16, 16
    kpts = (g + 1) ** 2
    ctx = rlmb.Context(local)
    peak = ctx.fp64_peak_tflops()
    per = {}
    seq_res = {}
    for n in FSS_SIZES:
        for _ in range(args.warmup):
            ctx.rlm_mesh_solve(n, 1.0, 16.0, g, SEED, ns, ns)
        ctx.profile(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for st in range(args.steps):
            seq_res[n] = ctx.rlm_mesh_solve(n, 1.0, 16.0, g, SEED, 0, ns)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        prof = ctx.profile_report()
        ctx.profile(False)
        eig_ms = sum(prof.get(k, (0, 0))[0] for k in EIG_LABELS)
        solves = ns * kpts * args.steps
        eig_tf = 13.33 * n ** 3 * solves / (eig_ms * 1e-3) / 1e12
        per[str(n)] = {"solves_per_s": solves / dt, "ms_per_step": 1e3 * dt / args.steps,
                       "eigensolve_tflops": eig_tf, "eigensolve_frac_of_fp64_peak": eig_tf / peak}
    ctx.close()
    total_solves = len(FSS_SIZES) * ns * kpts * args.steps
    seq_s = sum(v["ms_per_step"] for v in per.values()) * args.steps / 1e3
    # one graph launch per step, all sizes concurrent
    fg = rlmb.FssGraph(local, FSS_SIZES, 1.0, 16.0, g, SEED, ns, 0)
    st = fg.stream()
    for _ in range(args.warmup):
        fg.launch(0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        fg.launch(0)
    e1.record(st)
    torch.cuda.synchronize()
    graph_ms = e0.elapsed_time(e1) / args.steps
    same = True
    for i, n in enumerate(FSS_SIZES):
        e, c = fg.results(i)
        er, cr = seq_res[n]
        same = same and bool(np.array_equal(np.rint(c), np.rint(cr))) and \
            bool(np.abs(e - er).max() <= 1e-12 * np.abs(er).max())
    fg.close()
    graph_value = len(FSS_SIZES) * ns * kpts / (graph_ms * 1e-3)
    line = {"metric": METRIC, "value": graph_value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": graph_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "rlm finite-size scaling: n_phi in " + ",".join(map(str, FSS_SIZES)) +
                                   f", {ns} samples each per step, g={g}, impurity concentration 16, seed {SEED}",
                       "api": "one rlmb_rlm_fss_graph_launch per step (value); rlmb_rlm_mesh_solve per size "
                              "(sequential)"},
            "graph": {"launches_per_step": 1, "ms_per_step": graph_ms, "solves_per_s": graph_value,
                      "results_identical_to_sequential": same},
            "sequential": {"ms_per_step": 1e3 * seq_s / args.steps, "solves_per_s": total_solves / seq_s},
            "per_size": per, "fp64_peak_tflops": peak}
    print(json.dumps(line), flush=True)


def run_probe(args):
    """Small cases for profiler captures: --probe heevd runs one rlmb_heevd_batched call on
    `batch` random Hermitian matrices of order n (--mixed: in the mixed mode; --solver and
    --tridiag pin the eigensolver and its tridiagonal stage); --probe tcgemm
    runs batched n x n x n complex GEMMs on the two tcgen05 engines (three each) and one on the
    DMMA engine, and prints their CUDA-event times; --probe rlm runs one rlm mesh solve of
    `batch` samples at order n, g=4."""
    import numpy as np
    import torch
    import rlmb
    ctx = rlmb.Context(0)
    rng = np.random.default_rng(0)
    n, b = args.n, args.batch
    if args.probe == "tcgemm":
        at = torch.randn((b, n, n), dtype=torch.complex128, device="cuda")
        bt = torch.randn((b, n, n), dtype=torch.complex128, device="cuda")
        out = {}
        for name, eng, reps in (("tf32x3_f64acc_tma", ctx.GEMM_TF32X3_F64ACC, 3), ("tf32x3", ctx.GEMM_TF32X3, 3),
                                ("fp64_dmma", ctx.GEMM_FP64, 1)):
            ctx.zgemm(at, bt, eng)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                ctx.zgemm(at, bt, eng)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            out[name] = {"ms": ms, "complex_tflops": 8.0 * n ** 3 * b / (ms * 1e-3) / 1e12}
        print(json.dumps({"probe": "tcgemm", "n": n, "batch": b, "faults": ctx.tc_fault_count(), **out}))
        return
    if args.probe == "rlm":
        if args.mixed:
            ctx.precision = ctx.MIXED
        if args.eigenvalue_pass:
            ctx.set_refinement_steps(1)
            ctx.set_eigenvalue_pass(True)
        ctx.rlm_mesh_solve(n, 1.0, 16.0, 4 if n > 1024 else 16, SEED, 0, b)
        torch.cuda.synchronize()
        print(json.dumps({"probe": "rlm", "n": n, "samples": b, "launches": ctx.launches}))
        return
    if args.probe == "hlm":
        pots = rlmb.hlm_potentials(SEED, N_SITES, b)
        ctx.hlm_mesh_solve(LX, LY, Q, BAND, G, pots)
        torch.cuda.synchronize()
        print(json.dumps({"probe": "hlm", "samples": b, "launches": ctx.launches}))
        return
    if args.probe == "fhs":
        # one line pair of the reference layout at the hlm benchmark geometry
        prev = torch.randn((G + 1, N_PHI, N_SITES), dtype=torch.complex128, device="cuda")
        cur = torch.randn((G + 1, N_PHI, N_SITES), dtype=torch.complex128, device="cuda")
        for _ in range(3):
            ctx.fhs_line(prev, cur)
        torch.cuda.synchronize()
        print(json.dumps({"probe": "fhs", "n_phi": N_PHI, "dim_vec": N_SITES, "g": G}))
        return
    if args.mixed:
        ctx.precision = ctx.MIXED
    if args.eigenvalue_pass:
        ctx.set_refinement_steps(1)
        ctx.set_eigenvalue_pass(True)
    if args.solver != "auto":
        ctx.set_heev_solver(n, ctx.SOLVER_JACOBI if args.solver == "jacobi" else ctx.SOLVER_HOUSEHOLDER)
    if args.tridiag != "auto":
        ctx.set_tridiag_solver(n, ctx.TRIDIAG_DC if args.tridiag == "dc" else ctx.TRIDIAG_BISECTION)
    a0 = rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))
    a = torch.tensor(np.ascontiguousarray(a0 + np.conj(np.transpose(a0, (0, 2, 1)))), device="cuda")
    ctx.heevd(a)
    torch.cuda.synchronize()
    print(json.dumps({"probe": "heevd", "n": n, "batch": b, "launches": ctx.launches}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="rlm3000", choices=["rlm3000", "hlm48x16", "rlm512", "fss"],
                    help="rlm3000 (default, the headline), hlm48x16, rlm512 (1 GPU, both precisions), "
                         "or fss (the rlm finite-size-scaling sizes, 1 GPU)")
    ap.add_argument("--no-extra", action="store_true", help="skip the nested hlm48x16 block of the headline")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision measurement on the same inputs")
    ap.add_argument("--mixed", action="store_true", help="probe in the mixed-precision mode")
    ap.add_argument("--eigenvalue-pass", action="store_true",
                    help="probes in the mixed mode: one refinement step + the eigenvalue pass")
    ap.add_argument("--probe", default=None, choices=["heevd", "tcgemm", "rlm", "hlm", "fhs"],
                    help="run one small eigensolver batch only (for profiler captures)")
    ap.add_argument("--solver", default="auto", choices=["auto", "householder", "jacobi"],
                    help="--probe heevd: pin the eigensolver of order n")
    ap.add_argument("--tridiag", default="auto", choices=["auto", "bisection", "dc"],
                    help="--probe heevd: pin the tridiagonal solver of order n")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--batch", type=int, default=296)
    args = ap.parse_args()
    if args.probe:
        run_probe(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "rlm3000":
        run_headline(args)
    elif args.workload in RLM_WORKLOADS:
        run_gpu_rlm(args)
    elif args.workload == "fss":
        run_gpu_fss(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
