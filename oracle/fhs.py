"""Fukui-Hatsugai-Suzuki plaquette phases -- CPU oracle (test infrastructure).

Restates diag_wrappers/chern.cpp:37-75 (peer_cal_Chern; cal_Chern :3-35 is the same
loop).  For the plaquettes between mesh lines theta_1-1 ("prev") and theta_1 ("cur"),
plaquette m in [0, n_mesh) walks
    (prev,m) -> (cur,m) -> (cur,m+1) -> (prev,m+1) -> (prev,m)     (chern.cpp:15-17,47-50)
multiplying, per state n, the link overlaps <u_n(a)|u_n(b)> = zdotc(u_a, u_b)
(chern.cpp:57-70) and stores -arg(prod)/2pi (chern.cpp:72).
"""
import numpy as np


def links(a, b):
    """<u_n(a)|u_n(b)> for every state n; a, b are [N, dim_vec] (row n = state n)."""
    return np.einsum("nr,nr->n", np.conj(a), b)


def line_chern(prev, cur):
    """prev, cur: [(g+1), N, dim_vec] eigenvectors of two adjacent theta_1 lines.
    Returns [g, N]: -arg(prod)/(2 pi) per plaquette m and state n."""
    g = prev.shape[0] - 1
    out = np.empty((g, prev.shape[1]))
    for m in range(g):
        prod = np.ones(prev.shape[1], dtype=np.complex128)
        prod *= links(prev[m], cur[m])
        prod *= links(cur[m], cur[m + 1])
        prod *= links(cur[m + 1], prev[m + 1])
        prod *= links(prev[m + 1], prev[m])
        out[m] = -np.angle(prod) / (np.pi * 2.0)
    return out
