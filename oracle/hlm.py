"""Hofstadter lattice model (hlm) -- CPU oracle restatement (test infrastructure).

Follows the reference's double-precision CPU path (hlm_cpu_dp); each function cites
the file:line it restates.  Sites are r = j*lx + x (y = j in [0,ly), x in [0,lx)),
x = m + q with m a multiple of Q; the n_phi = lx*ly/Q clean Bloch states are
indexed c = kx*ly + ky (kx in [0, lx/Q), ky in [0, ly)).
"""
import math

import numpy as np
import scipy.linalg

from . import vsl
from .fhs import line_chern


class HlmParams:
    """hlm/main_hlm_cpu.cpp:28-30."""

    def __init__(self, lx=3, ly=3, Q=3, band=0, n_mesh=32, n_sample=1, seed=1):
        self.lx, self.ly, self.Q, self.band = int(lx), int(ly), int(Q), int(band)
        self.n_mesh, self.n_sample, self.seed = int(n_mesh), int(n_sample), int(seed)
        self.n_sites = self.lx * self.ly
        self.n_phi = self.n_sites // self.Q


def harper_matrix(p: HlmParams, kx_s, ky_s):
    """hlm/hamiltonian_hlm_cpu.cpp:25-32: the Q x Q k-space matrix, as the column-major
    array handed to heevd (element [r][c] at index c*Q + r)."""
    Q = p.Q
    pi2 = 2.0 * math.pi
    inv_Q = 1.0 / Q
    h = np.zeros(Q * Q, dtype=np.complex128)
    for q in range(Q):
        h[q * Q + q] = -2.0 * math.cos(ky_s * (pi2 / p.ly) + pi2 * q * inv_Q)
        if q + 1 < Q:
            h[q * Q + q + 1] = h[(q + 1) * Q + q] = -1.0
    ph = kx_s * Q * (pi2 / p.lx)
    h[Q * (Q - 1)] = -complex(math.cos(ph), math.sin(ph))
    h[Q - 1] = np.conj(h[Q * (Q - 1)])
    return h


def bloch_basis(p: HlmParams, theta_1, theta_2):
    """hlm/hamiltonian_hlm_cpu.cpp:2-56 (get_wfs_ktheta, per-theta overload).
    Returns Wc [n_phi, n_sites]: row c = normalised clean Bloch state c of band `band`."""
    Q, lx, ly = p.Q, p.lx, p.ly
    pi2 = 2.0 * math.pi
    inv_g = 1.0 / p.n_mesh
    j = np.arange(ly)[:, None, None]
    m = (np.arange(lx // Q) * Q)[None, :, None]
    Wc = np.empty((p.n_phi, p.n_sites), dtype=np.complex128)
    for kx in range(lx // Q):
        kx_s = kx + theta_1 * inv_g
        for ky in range(ly):
            ky_s = ky + theta_2 * inv_g
            h = harper_matrix(p, kx_s, ky_s)
            _, U = scipy.linalg.eigh(h.reshape(Q, Q).T, lower=False, driver="evd")
            u = U[:, p.band]
            phase = kx_s * (pi2 / lx) * m + ky_s * (pi2 / ly) * j          # [ly, lx/Q, 1]
            w = (np.cos(phase) - 1j * np.sin(phase)) * u[None, None, :]    # [ly, lx/Q, Q]
            w = w.reshape(-1)
            w = w * (1.0 / math.sqrt(np.sum(w.real ** 2 + w.imag ** 2)))
            Wc[kx * ly + ky] = w
    return Wc


def solve_kpoint(p: HlmParams, potential, theta_1, theta_2, basis=None):
    """hlm/hamiltonian_hlm_cpu.cpp:162-181 for one k-point: H = W^H diag(V) W (:173-176),
    heevd (:178), wfs_full = W U (:180).
    Returns (energies[N], H [N,N], psi [N, n_sites] with row n = state n)."""
    Wc = bloch_basis(p, theta_1, theta_2) if basis is None else basis
    H = (np.conj(Wc) * potential[None, :]) @ Wc.T        # H[a][b]
    w, U = scipy.linalg.eigh(H, lower=False, driver="evd")
    psi = U.T @ Wc
    return w, H, psi


def run_sample(p: HlmParams, potential, keep=False):
    """hlm/main_hlm_cpu.cpp:75-197 for one sample's potential.
    theta_2 runs over [0, g) per line; slot g is the periodic copy of slot 0 (:396-397,
    :428-429); energies add theta_2 = 0 twice (:390-394); Chern = sum of +arg/2pi
    (:463-466).  Returns energies [N], chern [N], energies_mesh [(g+1), g, N]."""
    g, N = p.n_mesh, p.n_phi
    E = np.empty((g + 1, g, N))
    X = np.empty((g + 1, g + 1, N, p.n_sites), dtype=np.complex128)
    for t1 in range(g + 1):
        for t2 in range(g):
            E[t1, t2], _, X[t1, t2] = solve_kpoint(p, potential, t1, t2)
        X[t1, g] = X[t1, 0]
    chern = np.zeros(N)
    for t1 in range(1, g + 1):
        chern += -line_chern(X[t1 - 1], X[t1]).sum(axis=0)
    energies = (E.sum(axis=(0, 1)) + E[:, 0, :].sum(axis=0)) / ((g + 1) * (g + 1))
    out = dict(energies=energies, chern=chern, energies_mesh=E)
    if keep:
        out["eigvecs"] = X
    return out


def run(p: HlmParams, keep=False):
    pots = vsl.hlm_potentials(p.seed, p.n_sites, p.n_sample)
    return [run_sample(p, pots[n], keep) for n in range(p.n_sample)]
