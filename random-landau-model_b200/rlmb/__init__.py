"""Python host mirror of the B200 twist-mesh library, over its C ABI (include/rlm_b200.h).

The entry points keep the reference's names and argument meanings (diag_wrappers/mkl_diag.cpp
``mkl_heevd``, diag_wrappers/chern.cpp ``cal_Chern``, the rlm/hlm drivers' options); data
live in torch CUDA tensors (device memory and streams only -- the arithmetic is the
library's CUDA kernels).  There is no CPU fallback: without the built library or a CUDA
device every compute call raises.
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "librlmb.so")

_c_dp = ctypes.POINTER(ctypes.c_double)
_c_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); mirrors include/rlm_b200.h
_SIGNATURES = {
    "rlmb_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int]),
    "rlmb_destroy": (ctypes.c_int, [_vp]),
    "rlmb_set_stream": (ctypes.c_int, [_vp, _vp]),
    "rlmb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "rlmb_launch_count": (ctypes.c_longlong, [_vp]),
    "rlmb_profile_enable": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rlmb_profile_count": (ctypes.c_int, [_vp]),
    "rlmb_profile_entry": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]),
    "rlmb_probe_fp64_peak": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "rlmb_set_precision": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rlmb_get_precision": (ctypes.c_int, [_vp]),
    "rlmb_set_refinement_steps": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rlmb_set_eigenvalue_pass": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rlmb_heevd_batched": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "rlmb_heevd_host": (ctypes.c_int, [_vp, _c_dp, _c_dp, ctypes.c_int, ctypes.c_int]),
    "rlmb_heevd_batched_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "rlmb_set_autotune": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rlmb_heev_config": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_ip, _c_ip, _c_ip, _c_ip, _c_ip, _c_dp]),
    "rlmb_set_heev_config": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "rlmb_set_heev_solver": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "rlmb_heev_solver": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_ip]),
    "rlmb_set_tridiag_solver": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "rlmb_set_panel_queue": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "rlmb_set_panel_width": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "rlmb_tridiag_solver": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_ip]),
    "rlmb_zgemm_batched": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int]),
    "rlmb_tc_fault_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    "rlmb_rlm_coeff_tables": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, _c_dp, _c_dp, _c_dp]),
    "rlmb_rlm_disorder": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_ulong,
                                         ctypes.c_int, _c_dp, _c_dp, _c_dp]),
    "rlmb_rlm_potential": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp,
                                          ctypes.c_int, ctypes.c_int, _vp]),
    "rlmb_rlm_assemble": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, _c_ip, _c_ip, ctypes.c_int, _vp]),
    "rlmb_hlm_potentials": (ctypes.c_int, [ctypes.c_ulong, ctypes.c_int, ctypes.c_int, _c_dp]),
    "rlmb_hlm_basis": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "rlmb_hlm_project": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, _vp, _c_ip, _c_ip, ctypes.c_int, _vp]),
    "rlmb_fhs_line": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "rlmb_rlm_mesh_solve": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int, ctypes.c_ulong, ctypes.c_int, ctypes.c_int,
                                           _c_dp, _c_dp]),
    "rlmb_rlm_mesh_solve_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                  ctypes.c_int, ctypes.c_ulong, ctypes.c_int, ctypes.c_int,
                                                  _vp, _vp]),
    "rlmb_rlm_fss_graph_create": (ctypes.c_int, [ctypes.c_int, _c_ip, ctypes.c_int, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_int, ctypes.c_ulong, ctypes.c_int,
                                                 ctypes.c_int, ctypes.POINTER(_vp)]),
    "rlmb_rlm_fss_graph_launch": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rlmb_rlm_fss_graph_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "rlmb_rlm_fss_graph_results": (ctypes.c_int, [_vp, ctypes.c_int, _c_dp, _c_dp]),
    "rlmb_rlm_fss_graph_destroy": (ctypes.c_int, [_vp]),
    "rlmb_rlm_mesh_export": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_ulong, ctypes.c_int, ctypes.c_char_p, _c_dp, _c_dp]),
    "rlmb_rlm_disorder_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_ulong,
                                                 ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "rlmb_hlm_potentials_device": (ctypes.c_int, [_vp, ctypes.c_ulong, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "rlmb_hlm_mesh_solve": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _c_dp, ctypes.c_int, _c_dp, _c_dp]),
    "rlmb_hlm_mesh_solve_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                  _vp, _vp]),
}

_lib = None


class RlmbError(RuntimeError):
    pass


def lib():
    """The loaded C library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RlmbError(f"{LIB_PATH} is missing: build it with random-landau-model_b200/build.py")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def _check(rc, what):
    if rc > 0:
        # positive status: number of matrices whose inverse iteration did not converge
        import warnings
        warnings.warn(f"{what}: eigenvectors of {rc} matrices did not converge")
        return rc
    if rc != 0:
        msg = lib().rlmb_status_string(rc).decode()
        raise RlmbError(f"{what} failed with status {rc}: {msg}")


def _dp(a):
    return a.ctypes.data_as(_c_dp)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


# ---------------------------------------------------------------- host-side inputs
def rlm_params(n_phi, quanta_concentration=1.0, impurity_concentration=16.0):
    """Derived sizes of rlm/main_rlm_cpu.cpp:29-33 (C truncations kept)."""
    L = math.sqrt(n_phi * quanta_concentration)
    nimp = int(impurity_concentration * n_phi / quanta_concentration)
    off_head = int(math.sqrt(nimp) / 2 + 1)
    return dict(L1=L, L2=L, impurity_num=nimp, off_head=off_head, dim=2 * off_head + 1)


def rlm_coeff_tables(n_phi, off_head, n_mesh, L1, L2):
    """(coeff_mn, coeff_m_theta, coeff_jm) as complex128 arrays, bit-exact with
    rlm/matrix_coefficients.cpp:3-25 (computed on the host by the library)."""
    dim = 2 * off_head + 1
    cmn = np.zeros(dim * dim, np.complex128)
    cmt = np.zeros((n_mesh + 1) * dim, np.complex128)
    cjm = np.zeros(n_phi * dim, np.complex128)
    _check(lib().rlmb_rlm_coeff_tables(n_phi, off_head, dim, n_mesh, L1, L2,
                                       _dp(cmn.view(np.float64)), _dp(cmt.view(np.float64)),
                                       _dp(cjm.view(np.float64))), "rlm_coeff_tables")
    return cmn, cmt, cjm


def rlm_disorder(impurity_num, L1, L2, seed, sample):
    """(x, y, s) of rlm/disorder_potential.cpp:3-21."""
    x, y, s = (np.zeros(impurity_num) for _ in range(3))
    _check(lib().rlmb_rlm_disorder(impurity_num, L1, L2, seed, sample, _dp(x), _dp(y), _dp(s)),
           "rlm_disorder")
    return x, y, s


def hlm_potentials(seed, n_sites, n_sample):
    """[n_sample, n_sites] on-site potentials of hlm/main_hlm_cpu.cpp:66-67,79."""
    out = np.zeros((n_sample, n_sites))
    _check(lib().rlmb_hlm_potentials(seed, n_sites, n_sample, _dp(out)), "hlm_potentials")
    return out


# ---------------------------------------------------------------------- contexts
class Context:
    """One device context of the library, bound to torch's current CUDA stream."""

    def __init__(self, device=0):
        import torch
        if not torch.cuda.is_available():
            raise RlmbError("no CUDA device: the library has no CPU path")
        self.device = device
        self.last_failures = 0
        h = ctypes.c_void_p()
        _check(lib().rlmb_create(ctypes.byref(h), device), "rlmb_create")
        self.h = h
        self.sync_stream()

    def sync_stream(self):
        import torch
        st = torch.cuda.current_stream(self.device).cuda_stream
        _check(lib().rlmb_set_stream(self.h, ctypes.c_void_p(st)), "rlmb_set_stream")

    def close(self):
        if getattr(self, "h", None):
            lib().rlmb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self):
        return lib().rlmb_launch_count(self.h)

    def profile(self, on=True):
        """Start (clearing) or stop per-kernel CUDA-event timing on the context stream."""
        _check(lib().rlmb_profile_enable(self.h, 1 if on else 0), "rlmb_profile_enable")

    def profile_report(self):
        """{kernel name: (total device ms, launches)} accumulated since profile(True)."""
        out = {}
        for i in range(lib().rlmb_profile_count(self.h)):
            name = ctypes.create_string_buffer(128)
            ms = ctypes.c_double()
            cnt = ctypes.c_longlong()
            _check(lib().rlmb_profile_entry(self.h, i, name, 128, ctypes.byref(ms), ctypes.byref(cnt)),
                   "rlmb_profile_entry")
            out[name.value.decode()] = (ms.value, cnt.value)
        return out

    FP64, MIXED = 0, 1

    @property
    def precision(self):
        """RLMB_PRECISION_FP64 (0) or RLMB_PRECISION_MIXED (1) for this context's solves."""
        return lib().rlmb_get_precision(self.h)

    @precision.setter
    def precision(self, mode):
        _check(lib().rlmb_set_precision(self.h, int(mode)), "rlmb_set_precision")

    def set_refinement_steps(self, steps):
        """Mixed mode: 1 or 2 double-precision refinement steps (default 2)."""
        _check(lib().rlmb_set_refinement_steps(self.h, int(steps)), "rlmb_set_refinement_steps")

    def set_eigenvalue_pass(self, on=True):
        """Mixed mode, one refinement step: recompute the eigenvalues as Rayleigh quotients of
        the refined vectors (double-precision eigenvalues for the cost of one residual)."""
        _check(lib().rlmb_set_eigenvalue_pass(self.h, 1 if on else 0), "rlmb_set_eigenvalue_pass")

    def fp64_peak_tflops(self):
        t = ctypes.c_double()
        _check(lib().rlmb_probe_fp64_peak(self.h, ctypes.byref(t)), "rlmb_probe_fp64_peak")
        return t.value

    # (b) eigensolver --------------------------------------------------------
    def heevd(self, a, w=None, info=None):
        """In-place batched eigendecomposition of torch complex128 CUDA tensor a[batch, n, n].

        Each a[b] holds M^T (the column-major matrix, upper triangle read) and receives X^T:
        row k of a[b] is eigenvector k.  Returns w[batch, n] (ascending)."""
        import torch
        assert a.is_cuda and a.dtype == torch.complex128 and a.is_contiguous()
        batch, n = a.shape[0], a.shape[-1]
        if w is None:
            w = torch.empty((batch, n), dtype=torch.float64, device=a.device)
        self.sync_stream()
        rc = lib().rlmb_heevd_batched(self.h, _ptr(a), _ptr(w), n, batch,
                                      _ptr(info) if info is not None else None)
        if rc < 0:
            _check(rc, "rlmb_heevd_batched")
        return w

    def set_autotune(self, on=True):
        """Time the eigensolver's launch configurations on the first solve of each order."""
        _check(lib().rlmb_set_autotune(self.h, 1 if on else 0), "rlmb_set_autotune")

    def heev_config(self, n, precision=None):
        """(tuned, {blocked, gemm_bt, panel_threads, x_tile, bt_block, ms_per_matrix}) used for order n."""
        prec = self.precision if precision is None else precision
        vals = [ctypes.c_int() for _ in range(5)]
        ms = ctypes.c_double()
        rc = lib().rlmb_heev_config(self.h, n, prec, *[ctypes.byref(v) for v in vals], ctypes.byref(ms))
        if rc < 0:
            _check(rc, "rlmb_heev_config")
        keys = ("blocked", "gemm_bt", "panel_threads", "x_tile", "bt_block")
        return rc == 1, dict(zip(keys, [v.value for v in vals]), ms_per_matrix=ms.value)

    def set_heev_config(self, n, blocked=-1, gemm_bt=-1, panel_threads=0, x_tile=0, bt_block=0, precision=None):
        prec = self.precision if precision is None else precision
        _check(lib().rlmb_set_heev_config(self.h, n, prec, blocked, gemm_bt, panel_threads, x_tile, bt_block),
               "rlmb_set_heev_config")

    SOLVER_AUTO, SOLVER_HOUSEHOLDER, SOLVER_JACOBI = 0, 1, 2

    def set_heev_solver(self, n, solver, precision=None):
        """Pin the solver of order-n eigensolves: SOLVER_JACOBI (n <= 80), SOLVER_HOUSEHOLDER or
        SOLVER_AUTO (built-in / autotuned)."""
        prec = self.precision if precision is None else precision
        _check(lib().rlmb_set_heev_solver(self.h, n, prec, solver), "rlmb_set_heev_solver")

    def heev_solver(self, n, precision=None):
        """SOLVER_JACOBI or SOLVER_HOUSEHOLDER: the solver order-n eigensolves run with now."""
        prec = self.precision if precision is None else precision
        v = ctypes.c_int()
        _check(lib().rlmb_heev_solver(self.h, n, prec, ctypes.byref(v)), "rlmb_heev_solver")
        return v.value

    TRIDIAG_AUTO, TRIDIAG_BISECTION, TRIDIAG_DC = 0, 1, 2

    def set_tridiag_solver(self, n, solver, precision=None):
        """Pin the tridiagonal stage of order-n eigensolves: TRIDIAG_DC (divide and conquer,
        n <= 3600), TRIDIAG_BISECTION or TRIDIAG_AUTO (built-in / autotuned)."""
        prec = self.precision if precision is None else precision
        _check(lib().rlmb_set_tridiag_solver(self.h, n, prec, solver), "rlmb_set_tridiag_solver")

    def set_panel_queue(self, n, threads, precision=None):
        """Pin the panel queue's CTAs for order n: 512 threads (one per SM), 256 (two per SM) or
        0 (built-in)."""
        prec = self.precision if precision is None else precision
        _check(lib().rlmb_set_panel_queue(self.h, n, prec, int(threads)), "rlmb_set_panel_queue")

    def set_panel_width(self, n, width, precision=None):
        """Pin the blocked reduction's panel width for order n: 16, 32 or 0 (built-in)."""
        prec = self.precision if precision is None else precision
        _check(lib().rlmb_set_panel_width(self.h, n, prec, int(width)), "rlmb_set_panel_width")

    def tridiag_solver(self, n, precision=None):
        """TRIDIAG_DC or TRIDIAG_BISECTION: the tridiagonal solver order-n eigensolves run with."""
        prec = self.precision if precision is None else precision
        v = ctypes.c_int()
        _check(lib().rlmb_tridiag_solver(self.h, n, prec, ctypes.byref(v)), "rlmb_tridiag_solver")
        return v.value

    GEMM_FP64, GEMM_TF32X3, GEMM_TF32X3_F64ACC = 0, 1, 2

    def zgemm(self, at, bt, engine=GEMM_TF32X3):
        """C = A B for torch complex128 CUDA tensors at[batch, k, m] = A^T and bt[batch, n, k] =
        B^T (the column-major matrices); returns ct[batch, n, m] = C^T."""
        import torch
        assert at.is_cuda and bt.is_cuda and at.dtype == bt.dtype == torch.complex128
        assert at.is_contiguous() and bt.is_contiguous()
        batch, k, m = at.shape
        n = bt.shape[1]
        assert bt.shape == (batch, n, k)
        ct = torch.empty((batch, n, m), dtype=torch.complex128, device=at.device)
        self.sync_stream()
        _check(lib().rlmb_zgemm_batched(self.h, _ptr(at), _ptr(bt), _ptr(ct), m, n, k, batch, int(engine)),
               "rlmb_zgemm_batched")
        return ct

    def tc_fault_count(self):
        c = ctypes.c_int()
        _check(lib().rlmb_tc_fault_count(self.h, ctypes.byref(c)), "rlmb_tc_fault_count")
        return c.value

    def mkl_heevd(self, h, n):
        """Drop-in for diag_wrappers/mkl_diag.cpp:2-9 on a host buffer of n*n complex
        (col-major, 'U'): overwrites h with eigenvectors, returns eigenvalues."""
        h = np.ascontiguousarray(h, dtype=np.complex128)
        w = np.zeros(n)
        rc = lib().rlmb_heevd_host(self.h, _dp(h.view(np.float64)), _dp(w), n, 1)
        if rc < 0:
            _check(rc, "rlmb_heevd_host")
        return w, h

    # (a) rlm ------------------------------------------------------------------
    def rlm_potential(self, x, y, s, coeff_mn, off_head):
        """V_mn for samples x,y,s [n_samples, n_imp] (torch float64 CUDA)."""
        import torch
        dim = 2 * off_head + 1
        ns, nimp = x.shape
        v = torch.empty((ns, dim * dim), dtype=torch.complex128, device=x.device)
        self.sync_stream()
        _check(lib().rlmb_rlm_potential(self.h, _ptr(x), _ptr(y), _ptr(s), nimp, ns, _ptr(coeff_mn),
                                        dim, off_head, _ptr(v)), "rlmb_rlm_potential")
        return v

    def rlm_assemble(self, vmn, cmt, cjm, n_phi, off_head, n_mesh, theta1, theta2):
        """Row-major H(theta1[i], theta2[i]) buffers as the reference fills them."""
        import torch
        theta1 = np.ascontiguousarray(theta1, dtype=np.int32)
        theta2 = np.ascontiguousarray(theta2, dtype=np.int32)
        out = torch.empty((len(theta1), n_phi, n_phi), dtype=torch.complex128, device=vmn.device)
        self.sync_stream()
        _check(lib().rlmb_rlm_assemble(self.h, _ptr(vmn), _ptr(cmt), _ptr(cjm), n_phi, 2 * off_head + 1,
                                       off_head, n_mesh, theta1.ctypes.data_as(_c_ip),
                                       theta2.ctypes.data_as(_c_ip), len(theta1), _ptr(out)),
               "rlmb_rlm_assemble")
        return out

    # (a) hlm ------------------------------------------------------------------
    def hlm_basis(self, lx, ly, Q, band, n_mesh, theta_1, theta_2):
        """W(theta) as [n_phi, n_sites]: row c = clean Bloch state c."""
        import torch
        n_phi = lx * ly // Q
        w = torch.empty((n_phi, lx * ly), dtype=torch.complex128, device="cuda")
        self.sync_stream()
        _check(lib().rlmb_hlm_basis(self.h, lx, ly, Q, band, n_mesh, theta_1, theta_2, _ptr(w)),
               "rlmb_hlm_basis")
        return w

    def hlm_project(self, lx, ly, Q, band, n_mesh, potential, theta1, theta2):
        """Column-major projected H for each k-point: returns [count, n, n] holding H^T."""
        import torch
        theta1 = np.ascontiguousarray(theta1, dtype=np.int32)
        theta2 = np.ascontiguousarray(theta2, dtype=np.int32)
        n_phi = lx * ly // Q
        out = torch.empty((len(theta1), n_phi, n_phi), dtype=torch.complex128, device=potential.device)
        self.sync_stream()
        _check(lib().rlmb_hlm_project(self.h, lx, ly, Q, band, n_mesh, _ptr(potential),
                                      theta1.ctypes.data_as(_c_ip), theta2.ctypes.data_as(_c_ip),
                                      len(theta1), _ptr(out)), "rlmb_hlm_project")
        return out

    # (c) FHS --------------------------------------------------------------------
    def fhs_line(self, prev, cur):
        """cal_Chern (diag_wrappers/chern.cpp:3-75) for one line pair: prev/cur are
        [(g+1), n_phi, dim_vec] complex128; returns chern_theta[m + n*g] as [n_phi, g]."""
        import torch
        g = prev.shape[0] - 1
        n_phi, dim_vec = prev.shape[1], prev.shape[2]
        out = torch.empty((n_phi, g), dtype=torch.float64, device=prev.device)
        self.sync_stream()
        _check(lib().rlmb_fhs_line(self.h, _ptr(prev), _ptr(cur), n_phi, dim_vec, g, _ptr(out)),
               "rlmb_fhs_line")
        return out

    # whole mesh -------------------------------------------------------------------
    def rlm_mesh_solve(self, n_phi, quanta_concentration=1.0, impurity_concentration=16.0,
                       n_mesh=32, seed=1, sample0=0, n_samples=1):
        """(energies, chern) [n_samples, n_phi]: the columns of energy_Chern_No.txt."""
        e = np.zeros((n_samples, n_phi))
        c = np.zeros((n_samples, n_phi))
        self.sync_stream()
        rc = lib().rlmb_rlm_mesh_solve(self.h, n_phi, quanta_concentration, impurity_concentration,
                                       n_mesh, seed, sample0, n_samples, _dp(e), _dp(c))
        self.last_failures = max(rc, 0)
        _check(rc, "rlmb_rlm_mesh_solve")
        return e, c

    def rlm_mesh_solve_device(self, n_phi, quanta_concentration, impurity_concentration, n_mesh, seed, sample0,
                              d_energies, d_chern):
        """rlm_mesh_solve into torch float64 CUDA tensors [n_samples, n_phi] (results stay on
        the device)."""
        self.sync_stream()
        rc = lib().rlmb_rlm_mesh_solve_device(self.h, n_phi, quanta_concentration, impurity_concentration, n_mesh,
                                              seed, sample0, d_energies.shape[0], _ptr(d_energies), _ptr(d_chern))
        self.last_failures = max(rc, 0)
        _check(rc, "rlmb_rlm_mesh_solve_device")

    def rlm_disorder_device(self, impurity_num, L1, L2, seed, sample0, count):
        """(x, y, s) torch float64 CUDA tensors [count, impurity_num] drawn on the device."""
        import torch
        out = [torch.empty((count, impurity_num), dtype=torch.float64, device="cuda") for _ in range(3)]
        self.sync_stream()
        _check(lib().rlmb_rlm_disorder_device(self.h, impurity_num, L1, L2, seed, sample0, count,
                                              *[_ptr(t) for t in out]), "rlmb_rlm_disorder_device")
        return out

    def hlm_potentials_device(self, seed, n_sites, sample0, count):
        """torch float64 CUDA tensor [count, n_sites] of hlm potentials drawn on the device."""
        import torch
        out = torch.empty((count, n_sites), dtype=torch.float64, device="cuda")
        self.sync_stream()
        _check(lib().rlmb_hlm_potentials_device(self.h, seed, n_sites, sample0, count, _ptr(out)),
               "rlmb_hlm_potentials_device")
        return out

    def rlm_mesh_export(self, n_phi, quanta_concentration, impurity_concentration, n_mesh, seed, sample,
                        directory):
        """One sample of rlm_mesh_solve that also writes every k-point's eigenvectors to
        directory/wfs_<theta_1>_<theta_2>.bin; returns (energies, chern) [n_phi]."""
        e = np.zeros(n_phi)
        c = np.zeros(n_phi)
        self.sync_stream()
        rc = lib().rlmb_rlm_mesh_export(self.h, n_phi, quanta_concentration, impurity_concentration, n_mesh,
                                        seed, sample, os.fsencode(directory), _dp(e), _dp(c))
        self.last_failures = max(rc, 0)
        _check(rc, "rlmb_rlm_mesh_export")
        return e, c

    def hlm_mesh_solve(self, lx, ly, Q, band, n_mesh, potentials):
        potentials = np.ascontiguousarray(potentials, dtype=np.float64)
        ns = potentials.shape[0]
        n_phi = lx * ly // Q
        e = np.zeros((ns, n_phi))
        c = np.zeros((ns, n_phi))
        self.sync_stream()
        rc = lib().rlmb_hlm_mesh_solve(self.h, lx, ly, Q, band, n_mesh, _dp(potentials), ns, _dp(e), _dp(c))
        self.last_failures = max(rc, 0)
        _check(rc, "rlmb_hlm_mesh_solve")
        return e, c

    def hlm_mesh_solve_device(self, lx, ly, Q, band, n_mesh, d_potentials, d_energies, d_chern):
        self.sync_stream()
        rc = lib().rlmb_hlm_mesh_solve_device(self.h, lx, ly, Q, band, n_mesh, _ptr(d_potentials),
                                              d_potentials.shape[0], _ptr(d_energies), _ptr(d_chern))
        self.last_failures = max(rc, 0)
        _check(rc, "rlmb_hlm_mesh_solve_device")


class FssGraph:
    """Several rlm orders solved by one CUDA graph launch per step (rlmb_rlm_fss_graph_*):
    every launch solves samples sample0 .. sample0+n_samples-1 of each order in n_phis, the
    orders on concurrent branches of the graph."""

    def __init__(self, device, n_phis, quanta_concentration=1.0, impurity_concentration=16.0, n_mesh=16, seed=1,
                 n_samples=16, precision=0):
        self.n_phis = [int(n) for n in n_phis]
        self.n_samples = int(n_samples)
        arr = (ctypes.c_int * len(self.n_phis))(*self.n_phis)
        h = ctypes.c_void_p()
        _check(lib().rlmb_rlm_fss_graph_create(device, arr, len(self.n_phis), quanta_concentration,
                                               impurity_concentration, n_mesh, seed, self.n_samples, int(precision),
                                               ctypes.byref(h)), "rlmb_rlm_fss_graph_create")
        self.h = h

    def launch(self, sample0):
        _check(lib().rlmb_rlm_fss_graph_launch(self.h, int(sample0)), "rlmb_rlm_fss_graph_launch")

    def stream(self):
        """The graph's stream as a torch ExternalStream (for CUDA-event timing)."""
        import torch
        st = ctypes.c_void_p()
        _check(lib().rlmb_rlm_fss_graph_stream(self.h, ctypes.byref(st)), "rlmb_rlm_fss_graph_stream")
        return torch.cuda.ExternalStream(st.value)

    def results(self, index):
        """(energies, chern) [n_samples, n_phi] of order index from the last launch."""
        n = self.n_phis[index]
        e = np.zeros((self.n_samples, n))
        c = np.zeros((self.n_samples, n))
        _check(lib().rlmb_rlm_fss_graph_results(self.h, index, _dp(e), _dp(c)), "rlmb_rlm_fss_graph_results")
        return e, c

    def close(self):
        if getattr(self, "h", None):
            lib().rlmb_rlm_fss_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
