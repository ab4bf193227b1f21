"""Random Landau-level model (rlm) -- CPU oracle restatement (test infrastructure).

Follows the reference's double-precision CPU path (rlm_cpu_dp); each function cites
the file:line it restates.  Layout conventions are the reference's:

* coeff tables row-major ``complex128``: coeff_mn[m*dim+n], coeff_m_theta[theta*dim+m],
  coeff_jm[j*dim+m];
* a k-point's matrix buffer ``buf`` (n_phi*n_phi complex) is filled row-major by the
  assembly and handed to a column-major, uplo='U' heevd, which therefore diagonalises
  M[r][c] = buf[c*N + r] (r <= c) = conj(H[r][c]); on return buf[n*N + r] holds
  component r of eigenvector n (eigenvalues ascending).
"""
import ctypes
import ctypes.util
import math

import numpy as np
import scipy.linalg

from . import vsl
from .fhs import line_chern

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.expf.restype = ctypes.c_float
_libm.expf.argtypes = [ctypes.c_float]


class RlmParams:
    """Derived sizes of rlm/main_rlm_cpu.cpp:28-34 (C integer truncations kept)."""

    def __init__(self, n_phi, quanta_concentration=1.0, impurity_concentration=16.0,
                 n_mesh=32, n_sample=1, seed=1):
        self.n_phi = int(n_phi)
        self.qc = float(quanta_concentration)
        self.ic = float(impurity_concentration)
        self.n_mesh = int(n_mesh)
        self.n_sample = int(n_sample)
        self.seed = int(seed)
        self.L1 = math.sqrt(self.n_phi * self.qc)
        self.L2 = math.sqrt(self.n_phi * self.qc)
        self.impurity_num = int(self.ic * self.n_phi / self.qc)
        self.off_head = int(math.sqrt(self.impurity_num) / 2 + 1)
        self.dim = 2 * self.off_head + 1


def prepare_coeff(p: RlmParams):
    """rlm/matrix_coefficients.cpp:3-25.  Uses libm cos/sin and single-precision expf
    with a float 1.0f/n_phi, exactly as the -DDP build does (line 11)."""
    N, o, d, g = p.n_phi, p.off_head, p.dim, p.n_mesh
    L1, L2 = p.L1, p.L2
    inv_n = float(np.float32(1.0) / np.float32(N))
    coeff_mn = np.empty(d * d, dtype=np.complex128)
    for m in range(d):
        for n in range(d):
            a = math.pi * (m - o) * (n - o) / N
            e = _libm.expf(-math.pi * ((m - o) * (m - o) * L2 / L1 + (n - o) * (n - o) * L1 / L2)
                           / 2.0 / N)
            coeff_mn[m * d + n] = complex(math.cos(a), -math.sin(a)) * float(e) * inv_n
    coeff_m_theta = np.empty((g + 1) * d, dtype=np.complex128)
    pi2 = math.pi * 2.0
    for t in range(g + 1):
        dtheta = t * pi2 / g
        for m in range(d):
            a = (m - o) * dtheta / N
            coeff_m_theta[t * d + m] = complex(math.cos(a), math.sin(a))
    coeff_jm = np.empty(N * d, dtype=np.complex128)
    for j in range(N):
        for m in range(d):
            a = pi2 * (m - o) * (j + 1) / N
            coeff_jm[j * d + m] = complex(math.cos(a), -math.sin(a))
    return coeff_mn, coeff_m_theta, coeff_jm


def potential_coeff(x, y, s, coeff_mn, dim, off_head):
    """rlm/matrix_coefficients.cpp:27-44: V[m,n] = coeff_mn * sum_i s_i e^{-i(kx x_i + ky y_i)},
    kx = 2pi(m-o), ky = 2pi(n-o) (positions are not divided by L, as in the reference)."""
    pi2 = math.pi * 2.0
    kx = pi2 * (np.arange(dim) - off_head)
    v = np.empty((dim, dim), dtype=np.complex128)
    for m in range(dim):
        phase = kx[m] * x[None, :] + kx[:, None] * y[None, :]
        v[m] = (np.cos(phase) - 1j * np.sin(phase)) @ s
    return v.reshape(-1) * coeff_mn


def assemble(p: RlmParams, v_mn, coeff_m_theta, coeff_jm, theta_1, theta_2):
    """rlm/hamiltonian_rlm_cpu.cpp:14-48: row-major buffer of H(theta_1, theta_2).

    H[j][k] (k >= j) = sum_m conj(c_theta2[m]) c_jm[j,m] * sum_{n in {o+k-j, o+k-j-N}}
    V[m,n] c_theta1[n]; lower triangle = conj(upper); the diagonal is stored conjugated."""
    N, o, d = p.n_phi, p.off_head, p.dim
    V = v_mn.reshape(d, d)
    c1 = coeff_m_theta[theta_1 * d:(theta_1 + 1) * d]
    c2 = coeff_m_theta[theta_2 * d:(theta_2 + 1) * d]
    G = V * c1[None, :]                      # G[m][n] = V[m][n] c_theta1[n]
    T = np.zeros((d, N), dtype=np.complex128)  # T[m][delta], delta = k - j
    for delta in range(N):
        if delta <= o:
            T[:, delta] += G[:, o + delta]
        if N - delta <= o:
            T[:, delta] += G[:, o + delta - N]
    P = np.conj(c2)[None, :] * coeff_jm.reshape(N, d)   # P[j][m]
    R = P @ T                                           # R[j][delta]
    jj, kk = np.triu_indices(N)
    buf = np.zeros((N, N), dtype=np.complex128)
    buf[jj, kk] = R[jj, kk - jj]
    buf[kk, jj] = np.conj(buf[jj, kk])
    return buf.reshape(-1)


def gpu_potential_coeff(x, y, s, coeff_mn, dim, off_head):
    """rlm/potential_coeff.cu:3-19, the single-precision GPU driver's V_mn (evaluated here in
    double): V[m,n] = coeff_mn * sum_i s_i e^{+i(kx x_i + ky y_i)} -- the opposite phase sign
    of the CPU path's get_potential_coeff."""
    return np.conj(potential_coeff(x, y, s, np.ones_like(coeff_mn), dim, off_head)) * coeff_mn


def gpu_assemble(ct1, ct2, coeff_jm, v_mn, N, o):
    """rlm/hamiltonian_rlm_gpu.cu:9-41, the GPU driver's row-major buffer (in double):
    H[j][k] (k >= j) = sum_m c_jm[j,m] ct2[m] * sum_{n in {o+k-j, o+k-j-N}} V[m,n] conj(ct1[n]),
    lower triangle = conj(upper), diagonal stored conjugated.  ct1 / ct2 are the coeff_m_theta
    rows of theta_1 / theta_2 (rlm/main_rlm_gpu.cu:170-173)."""
    d = 2 * o + 1
    V = np.asarray(v_mn).reshape(d, d)
    G = V * np.conj(ct1)[None, :]
    T = np.zeros((d, N), dtype=np.complex128)
    for delta in range(N):
        if delta <= o:
            T[:, delta] += G[:, o + delta]
        if N - delta <= o:
            T[:, delta] += G[:, o + delta - N]
    P = np.asarray(ct2)[None, :] * np.asarray(coeff_jm).reshape(N, d)
    R = P @ T
    jj, kk = np.triu_indices(N)
    buf = np.zeros((N, N), dtype=np.complex128)
    buf[jj, kk] = R[jj, kk - jj]
    buf[kk, jj] = np.conj(buf[jj, kk])
    return buf.reshape(-1)


def heevd(buf, n):
    """diag_wrappers/mkl_diag.cpp:2-9: column-major, uplo='U', jobz='V', in place.
    Returns (eigenvalues ascending, buffer with eigenvector n at buf[n*N:(n+1)*N])."""
    M = buf.reshape(n, n).T   # M[r][c] = buf[c*n + r]
    w, X = scipy.linalg.eigh(M, lower=False, driver="evd")
    return w, np.ascontiguousarray(X.T).reshape(-1)


def solve_kpoint(p, v_mn, cmt, cjm, theta_1, theta_2):
    """rlm/hamiltonian_rlm_cpu.cpp:2-52 for one (theta_1, theta_2): assemble + heevd.
    Returns (energies[N], eigenvectors[N, N] with row n = eigenvector n)."""
    buf = assemble(p, v_mn, cmt, cjm, theta_1, theta_2)
    w, vec = heevd(buf, p.n_phi)
    return w, vec.reshape(p.n_phi, p.n_phi)


def run_sample(p: RlmParams, sample: int, tables=None, keep=False):
    """rlm/main_rlm_cpu.cpp:109-243 for one disorder sample.

    Returns dict with energies [N] (twist-averaged), chern [N] (with the +1/N shift of
    :238), chern_raw [N] (without it), energies_mesh [(g+1),(g+1),N] and, if keep,
    the eigenvectors of the whole mesh [(g+1),(g+1),N,N]."""
    N, g = p.n_phi, p.n_mesh
    coeff_mn, cmt, cjm = tables if tables is not None else prepare_coeff(p)
    x, y, s = vsl.rlm_disorder(p.impurity_num, p.L1, p.L2, p.seed, sample)
    v_mn = potential_coeff(x, y, s, coeff_mn, p.dim, p.off_head)
    E = np.empty((g + 1, g + 1, N))
    X = np.empty((g + 1, g + 1, N, N), dtype=np.complex128)
    for t1 in range(g + 1):
        for t2 in range(g + 1):
            E[t1, t2], X[t1, t2] = solve_kpoint(p, v_mn, cmt, cjm, t1, t2)
    chern_raw = np.zeros(N)
    for t1 in range(1, g + 1):
        ct = line_chern(X[t1 - 1], X[t1])        # [g, N]: -arg(prod)/2pi
        chern_raw += ct.sum(axis=0)
    energies = E.sum(axis=(0, 1)) / ((g + 1) * (g + 1))
    out = dict(energies=energies, chern=chern_raw + 1.0 / N, chern_raw=chern_raw,
               energies_mesh=E, v_mn=v_mn, disorder=(x, y, s))
    if keep:
        out["eigvecs"] = X
    return out


def run(p: RlmParams, keep=False):
    tables = prepare_coeff(p)
    return [run_sample(p, n, tables, keep) for n in range(p.n_sample)]
