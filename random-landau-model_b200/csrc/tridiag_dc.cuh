// Symmetric tridiagonal eigensolver by divide and conquer (double precision, batched).
//
// The alternative to k_tridiag (bisection + inverse iteration) for the tridiagonal stage of the
// Householder eigensolver.  Both stand in for the tridiagonal part of LAPACK's zheevd, which the
// reference reaches through LAPACKE_zheevd (diag_wrappers/mkl_diag.cpp:2-9); zheevd itself
// solves that stage by divide and conquer (zstedc / dlaed*), whose published method this file
// restates in its own kernels:
//
//   Cuppen's split: T = diag(T1', T2') + rho u u^T at every split point, with
//   rho = 2|beta|, u = (e_last ; sign(beta) e_first) / sqrt(2) and |beta| taken off the two
//   diagonal entries next to the split.  The recursion runs bottom-up from 1 x 1 leaves, level
//   by level (subproblem size S = 2, 4, 8, ...), every level one launch over the whole chunk.
//
//   Merge of two solved children (k_dc_merge, a group of threads per subproblem):
//     z = Q^T u from the children's boundary rows; the children's sorted eigenvalues merged;
//     deflation (dlaed2): rho |z_k| <= tol drops k, and a Givens rotation drops the first of
//       two poles closer than tol (|t c s| <= tol), tol = 8 eps max(|d|, rho |z|);
//     the K remaining roots of the secular equation 1/rho + sum z_k^2 / (d_k - x) = 0, one
//       thread per root: origin at the nearer pole (x = d_org + tau, so that every d_k - x is
//       formed as (d_k - d_org) - tau), a bracket kept from the sign of f, and steps from a
//       rational model with the two nearest poles (value and slope matched), a bisection where
//       the step leaves the bracket;
//     z recomputed from the roots (Gu & Eisenstat): z_i^2 = prod_j (x_j - d_i) /
//       (rho prod_{j != i} (d_j - d_i)), which makes the eigenvectors
//       u_j = (z_i / (d_i - x_j))_i numerically orthogonal;
//     U = G [u_0 .. u_{K-1}, unit vectors of the deflated poles], G the deflation rotations,
//       columns in ascending eigenvalue order.
//   Q_new = blockdiag(Q1, Q2) U: inside k_dc_merge for S <= DC_SMALL, else k_dc_gemm (double
//   precision on the FP64 tensor path, mma.sync m8n8k4 .f64) over (matrix, subproblem, half).
//
// Q is row-major (Q[j*n + k] = component j of eigenvector k), the layout of k_tridiag's Z that
// the back-transformation reads.  The tridiagonal is scaled by a power of two (exact) so that
// its largest entry is ~1.  No kernel waits on another CTA.
#pragma once
#include <cfloat>

#include "common.cuh"

namespace rlmb {

static constexpr int DC_THREADS = 512;
static constexpr int DC_SMALL = 64;      // merges up to this size form their product in k_dc_merge
static constexpr int DC_MAX_N = 3600;    // the top merge keeps 56 bytes per entry in shared memory
static constexpr int DC_MAX_ITS = 64;    // secular iterations per root before it counts as failed

struct DcRot {
    int a, b;      // child indices of the two rotated basis vectors
    double c, s;   // rows (a, b) of U <- (c a - s b, s a + c b), applied in reverse order
};

// Threads per subproblem group: at least S (rounded to warps, at most DC_THREADS), and no more
// groups than there are subproblems, so that every level keeps all DC_THREADS threads busy.
// A power of two from 32 to DC_THREADS (at most 16 groups).
__host__ __device__ inline int dc_group_threads(int S, int n) {
    int g = ((S + 31) / 32) * 32;
    g = g < DC_THREADS ? g : DC_THREADS;
    const int nsub = (n + S - 1) / S;
    int ng = DC_THREADS / g;
    while (ng > 1 && ng > nsub) ng >>= 1;
    return DC_THREADS / ng;
}
__host__ __device__ inline int dc_smax(int S, int n) { return S < n ? S : n; }
__host__ __device__ inline size_t dc_group_bytes(int smax) {
    const size_t m = (size_t)(smax + 7) / 8 * 8;
    return 56 * m + 64;
}
__host__ __device__ inline size_t dc_smem(int S, int n) {
    return (size_t)(DC_THREADS / dc_group_threads(S, n)) * dc_group_bytes(dc_smax(S, n));
}
// number of merge levels: S = 2, 4, ... while S / 2 < n
__host__ __device__ inline int dc_levels(int n) {
    int l = 0;
    for (int S = 2; S / 2 < n; S *= 2) ++l;
    return l;
}

__device__ __forceinline__ void dc_sync(int grp, int gs) {
    if (gs == 32) __syncwarp();
    else if (gs == DC_THREADS) __syncthreads();
    else asm volatile("bar.sync %0, %1;\n" ::"r"(grp + 1), "r"(gs) : "memory");
}

// Scale (a power of two, per matrix), leaf values and Q_0 = I: one CTA of 256 threads per matrix.
__global__ void __launch_bounds__(256) k_dc_init(const double* __restrict__ D, const double* __restrict__ E,
                                                 double* __restrict__ W, double* __restrict__ Q0,
                                                 double* __restrict__ SC, int* __restrict__ info, int n) {
    __shared__ double red[8];
    const size_t mat = blockIdx.x;
    const double* d = D + mat * n;
    const double* e = E + mat * n;
    double mx = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) {
        mx = fmax(mx, fabs(d[i]));
        if (i < n - 1) mx = fmax(mx, fabs(e[i]));
    }
    for (int m = 16; m >= 1; m >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, m));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    mx = 0.0;
    for (int w = 0; w < 8; ++w) mx = fmax(mx, red[w]);
    double sc = 1.0;
    if (mx > 0.0 && mx < DBL_MAX) {
        int ex;
        frexp(mx, &ex);
        sc = ldexp(1.0, ex);
    }
    const double rs = 1.0 / sc;   // exact: sc is a power of two
    double* w = W + mat * n;
    double* q = Q0 + mat * (size_t)n * n;
    for (int i = threadIdx.x; i < n; i += 256) {
        double v = d[i] * rs;
        if (i > 0) v -= fabs(e[i - 1] * rs);
        if (i < n - 1) v -= fabs(e[i] * rs);
        w[i] = v;
        q[(size_t)i * n + i] = 1.0;
    }
    if (threadIdx.x == 0) {
        SC[mat] = sc;
        if (info) info[mat] = 0;
    }
}

// Eigenvalues back to the matrix's scale.
__global__ void k_dc_finish(double* __restrict__ W, const double* __restrict__ SC, int n, size_t total) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        W[i] *= SC[i / n];
}

// number of entries of the sorted v[0..m) below x (strictly, or not above x)
__device__ __forceinline__ int dc_lower(const double* v, int m, double x) {
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (v[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int dc_upper(const double* v, int m, double x) {
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (v[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Pole sums of the secular function over k in [k0, k1): sw = sum w_k and sw2 = sum w_k / delta_k
// with w_k = z_k^2 / delta_k, delta_k = (d_k - d0) - t.  Four independent accumulator pairs,
// so that four reciprocals are in flight at once.
__device__ __forceinline__ void dc_pole_sums(const double* __restrict__ ds, const double* __restrict__ zs, int k0,
                                             int k1, double d0, double t, double& sw, double& sw2) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0;
    int k = k0;
    for (; k + 3 < k1; k += 4) {
        const double r0 = 1.0 / ((ds[k] - d0) - t), r1 = 1.0 / ((ds[k + 1] - d0) - t);
        const double r2 = 1.0 / ((ds[k + 2] - d0) - t), r3 = 1.0 / ((ds[k + 3] - d0) - t);
        const double w0 = zs[k] * zs[k] * r0, w1 = zs[k + 1] * zs[k + 1] * r1;
        const double w2 = zs[k + 2] * zs[k + 2] * r2, w3 = zs[k + 3] * zs[k + 3] * r3;
        a0 += w0;
        a1 += w1;
        a2 += w2;
        a3 += w3;
        b0 = fma(w0, r0, b0);
        b1 = fma(w1, r1, b1);
        b2 = fma(w2, r2, b2);
        b3 = fma(w3, r3, b3);
    }
    for (; k < k1; ++k) {
        const double r = 1.0 / ((ds[k] - d0) - t);
        const double w = zs[k] * zs[k] * r;
        a0 += w;
        b0 = fma(w, r, b0);
    }
    sw = (a0 + a1) + (a2 + a3);
    sw2 = (b0 + b1) + (b2 + b3);
}

// One level of merges: one CTA of DC_THREADS per matrix, a group of dc_group_threads(S, n)
// threads per subproblem of size S (children S/2 and the rest).  W holds the children's
// sorted eigenvalues on entry and the merged ones on return; Qo the children's eigenvectors,
// Qn the merged ones (for S <= DC_SMALL, else U for k_dc_gemm).
__global__ void __launch_bounds__(DC_THREADS, 1)
k_dc_merge(const double* __restrict__ E, const double* __restrict__ SC, double* __restrict__ W,
           const double* __restrict__ Qo, double* __restrict__ Qn, double* __restrict__ U, DcRot* __restrict__ ROT,
           int* __restrict__ info, int n, int S) {
    extern __shared__ __align__(16) unsigned char dc_sm[];
    const int gs = dc_group_threads(S, n), ng = DC_THREADS / gs;
    const int grp = threadIdx.x / gs, gt = threadIdx.x % gs;
    const int smax = dc_smax(S, n);
    const int sm8 = (smax + 7) / 8 * 8;
    unsigned char* gb = dc_sm + (size_t)grp * dc_group_bytes(smax);
    double* ds = reinterpret_cast<double*>(gb);   // sorted poles, then the K kept ones first
    double* zs = ds + sm8;                        // z in the same order
    double* tau = zs + sm8;                       // root j = ds[org[j]] + tau[j]
    double* zh = tau + sm8;                       // recomputed z
    double* vals = zh + sm8;                      // merged eigenvalue of output column c
    int* perm = reinterpret_cast<int*>(vals + sm8);   // sorted index -> child index
    int* src = perm + sm8;                        // compact index -> sorted index (kept, then deflated)
    int* org = src + sm8;
    int* pos = org + sm8;                         // output column -> sorted position (first a flag array)
    int* scal = pos + sm8;                        // K, number of rotations, failure flag
    const size_t mat = blockIdx.x;
    const double rs = 1.0 / SC[mat];
    const double* e = E + mat * n;
    double* lam = W + mat * n;
    const double* qo = Qo + mat * (size_t)n * n;
    double* qn = Qn + mat * (size_t)n * n;
    const int nsub = (n + S - 1) / S;
    int fail = 0;
    for (int s = grp; s < nsub; s += ng) {
        const int o = s * S;
        const int K0 = min(S, n - o), n1 = min(S / 2, K0), n2 = K0 - n1;
        if (n2 <= 0) {   // a single child: its block carries over
            for (int idx = gt; idx < n1 * n1; idx += gs) {
                const int r = idx / n1, c = idx % n1;
                qn[(size_t)(o + r) * n + o + c] = qo[(size_t)(o + r) * n + o + c];
            }
            continue;
        }
        double* us = U + mat * (size_t)n * n + (size_t)o * smax;   // this subproblem's U, K0 x K0 row-major
        DcRot* rl = ROT + mat * n + o;                              // its rotations (< K0)
        const double beta = e[o + n1 - 1] * rs;
        const double rho = 2.0 * fabs(beta);
        const double sg = beta >= 0.0 ? 1.0 : -1.0;
        // children's eigenvalues merged into one ascending list (ties: first child first)
        for (int i = gt; i < K0; i += gs) {
            const double v = lam[o + i];
            double z;
            int rk;
            if (i < n1) {
                z = qo[(size_t)(o + n1 - 1) * n + o + i];
                rk = i + dc_lower(lam + o + n1, n2, v);
            } else {
                z = sg * qo[(size_t)(o + n1) * n + o + i];
                rk = (i - n1) + dc_upper(lam + o, n1, v);
            }
            perm[rk] = i;
            ds[rk] = v;
            zs[rk] = z * 0.70710678118654752440;
        }
        dc_sync(grp, gs);
        // deflation, one thread (a chain over the sorted poles)
        if (gt == 0) {
            double dmax = 0.0, zmax = 0.0;
            for (int k = 0; k < K0; ++k) {
                dmax = fmax(dmax, fabs(ds[k]));
                zmax = fmax(zmax, fabs(zs[k]));
                pos[k] = 0;
            }
            const double tol = 8.0 * 0x1p-53 * fmax(dmax, rho * zmax);
            int nrot = 0, pj = -1;
            for (int k = 0; k < K0; ++k) {
                if (rho * fabs(zs[k]) <= tol) {
                    pos[k] = 1;
                    continue;
                }
                if (pj >= 0) {
                    const double sv = zs[pj], cv = zs[k];
                    const double h = hypot(cv, sv);
                    const double t = ds[k] - ds[pj];
                    const double c = cv / h, sn = -sv / h;
                    if (fabs(t * c * sn) <= tol) {
                        zs[k] = h;
                        zs[pj] = 0.0;
                        rl[nrot].a = perm[pj];
                        rl[nrot].b = perm[k];
                        rl[nrot].c = c;
                        rl[nrot].s = sn;
                        ++nrot;
                        const double dp = ds[pj] * c * c + ds[k] * sn * sn;
                        ds[k] = ds[pj] * sn * sn + ds[k] * c * c;
                        ds[pj] = dp;
                        pos[pj] = 1;
                    }
                }
                pj = k;
            }
            int K = 0;
            for (int k = 0; k < K0; ++k) K += pos[k] == 0;
            int j = 0, m = 0;
            for (int k = 0; k < K0; ++k) {
                if (pos[k] == 0) {   // kept: compacted in place (j <= k)
                    const double dk = ds[k], zk = zs[k];
                    ds[j] = dk;
                    zs[j] = zk;
                    src[j] = k;
                    ++j;
                } else {
                    vals[K + m] = ds[k];
                    src[K + m] = k;
                    ++m;
                }
            }
            scal[0] = K;
            scal[1] = nrot;
        }
        dc_sync(grp, gs);
        const int K = scal[0], nrot = scal[1];
        const double rrho = 1.0 / fmax(rho, DBL_MIN);
        // secular equation, one thread per root
        for (int j = gt; j < K; j += gs) {
            int og;
            double lo, hi;
            if (j < K - 1) {
                const double dj = ds[j];
                const double mid = 0.5 * (ds[j + 1] - dj);
                double fs, fd;
                dc_pole_sums(ds, zs, 0, K, dj, mid, fs, fd);
                const double f = rrho + fs;
                if (f >= 0.0) {
                    og = j;
                    lo = 0.0;
                    hi = mid;
                } else {
                    og = j + 1;
                    lo = -mid;
                    hi = 0.0;
                }
            } else {
                double zz = 0.0;
                for (int k = 0; k < K; ++k) zz += zs[k] * zs[k];
                og = j;
                lo = 0.0;
                hi = rho * zz;
            }
            const double d0 = ds[og];
            double t = 0.5 * (lo + hi);
            bool conv = false;
            for (int it = 0; it < DC_MAX_ITS; ++it) {
                double psi, dpsi, phi, dphi;
                dc_pole_sums(ds, zs, 0, j + 1, d0, t, psi, dpsi);
                dc_pole_sums(ds, zs, j + 1, K, d0, t, phi, dphi);
                const double f = rrho + psi + phi;
                if (f < 0.0) lo = t;
                else hi = t;
                if (fabs(f) <= 8.0 * 0x1p-53 * K * (rrho + fabs(psi) + fabs(phi)) ||
                    hi - lo <= 4.0 * 0x1p-53 * fmax(fabs(lo), fabs(hi))) {
                    conv = true;
                    break;
                }
                // two-pole rational model, value and slope matched at t
                const double D1 = (ds[j] - d0) - t;
                const double b1 = dpsi * D1 * D1, a1 = psi - b1 / D1;
                double tn;
                bool ok = false;
                if (j < K - 1) {
                    const double D2 = (ds[j + 1] - d0) - t;
                    const double b2 = dphi * D2 * D2, a2 = phi - b2 / D2;
                    const double c = rrho + a1 + a2;
                    const double B = c * (D1 + D2) + b1 + b2, C = c * D1 * D2 + b1 * D2 + b2 * D1;
                    double eta = 0.0;
                    if (c == 0.0) {
                        if (B != 0.0) {
                            eta = C / B;
                            ok = eta > D1 && eta < D2;
                        }
                    } else {
                        const double sq = sqrt(fmax(B * B - 4.0 * c * C, 0.0));
                        const double e1 = B >= 0.0 ? (B + sq) / (2.0 * c) : 2.0 * C / (B - sq);
                        const double e2 = B >= 0.0 ? (B + sq != 0.0 ? 2.0 * C / (B + sq) : D2) : (B - sq) / (2.0 * c);
                        if (e1 > D1 && e1 < D2) {
                            eta = e1;
                            ok = true;
                        }
                        if (e2 > D1 && e2 < D2) {
                            eta = e2;
                            ok = true;
                        }
                    }
                    tn = t + eta;
                } else {
                    const double c = rrho + a1 + phi;
                    ok = c > 0.0;
                    tn = ok ? t + D1 + b1 / c : t;
                }
                if (!ok || !(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
                t = tn;
            }
            if (!conv) fail = 1;
            org[j] = og;
            tau[j] = t;
        }
        dc_sync(grp, gs);
        // z from the roots (Gu & Eisenstat): pairs (x_j - d_i) / (d_j - d_i), and (x_i - d_i) / rho
        for (int i = gt; i < K; i += gs) {
            const double di = ds[i];
            double p0 = 1.0, p1 = 1.0;   // even and odd j: two divisions in flight
            int j = 0;
            for (; j + 1 < K; j += 2) {
                const double x0 = (ds[org[j]] - di) + tau[j], x1 = (ds[org[j + 1]] - di) + tau[j + 1];
                p0 *= x0 / (j == i ? rho : ds[j] - di);
                p1 *= x1 / (j + 1 == i ? rho : ds[j + 1] - di);
            }
            if (j < K) p0 *= ((ds[org[j]] - di) + tau[j]) / (j == i ? rho : ds[j] - di);
            zh[i] = copysign(sqrt(fmax(p0 * p1, 0.0)), zs[i]);
        }
        for (int j = gt; j < K; j += gs) vals[j] = ds[org[j]] + tau[j];
        dc_sync(grp, gs);
        // output order: rank of every merged eigenvalue (ties by column)
        for (int c = gt; c < K0; c += gs) {
            const double v = vals[c];
            int rk = 0;
            for (int c2 = 0; c2 < K0; ++c2) {
                const double v2 = vals[c2];
                rk += (v2 < v || (v2 == v && c2 < c)) ? 1 : 0;
            }
            pos[c] = rk;   // (the deflation flags in pos are no longer needed)
        }
        dc_sync(grp, gs);
        for (int c = gt; c < K0; c += gs) lam[o + pos[c]] = vals[c];
        // U: column pos[c] = eigenvector c in the children's basis (rows = child indices)
        for (int c = gt; c < K0; c += gs) {
            const int col = pos[c];
            if (c < K) {
                const double x0 = ds[org[c]], tc = tau[c];
                double n0 = 0.0, n1 = 0.0, n2 = 0.0, n3 = 0.0;
                int i = 0;
                for (; i + 3 < K; i += 4) {
                    const double u0 = zh[i] / ((ds[i] - x0) - tc), u1 = zh[i + 1] / ((ds[i + 1] - x0) - tc);
                    const double u2 = zh[i + 2] / ((ds[i + 2] - x0) - tc), u3 = zh[i + 3] / ((ds[i + 3] - x0) - tc);
                    n0 = fma(u0, u0, n0);
                    n1 = fma(u1, u1, n1);
                    n2 = fma(u2, u2, n2);
                    n3 = fma(u3, u3, n3);
                }
                for (; i < K; ++i) {
                    const double u = zh[i] / ((ds[i] - x0) - tc);
                    n0 = fma(u, u, n0);
                }
                const double rn = 1.0 / sqrt((n0 + n1) + (n2 + n3));
                for (int i = 0; i < K; ++i) {
                    const double dl = (ds[i] - x0) - tc;
                    us[(size_t)perm[src[i]] * K0 + col] = zh[i] / dl * rn;
                }
                for (int i = K; i < K0; ++i) us[(size_t)perm[src[i]] * K0 + col] = 0.0;
            } else {
                const int row = perm[src[c]];
                for (int i = 0; i < K0; ++i) us[(size_t)i * K0 + col] = i == row ? 1.0 : 0.0;
            }
        }
        dc_sync(grp, gs);
        if (nrot > 0) {   // U <- G U, the deflation rotations last to first
            for (int col = gt; col < K0; col += gs)
                for (int r = nrot - 1; r >= 0; --r) {
                    const DcRot R = rl[r];
                    const double ua = us[(size_t)R.a * K0 + col], ub = us[(size_t)R.b * K0 + col];
                    us[(size_t)R.a * K0 + col] = R.c * ua - R.s * ub;
                    us[(size_t)R.b * K0 + col] = R.s * ua + R.c * ub;
                }
            dc_sync(grp, gs);
        }
        if (S <= DC_SMALL) {   // Q_new = blockdiag(Q1, Q2) U here
            for (int idx = gt; idx < K0 * K0; idx += gs) {
                const int r = idx / K0, c = idx % K0;
                const int k0 = r < n1 ? 0 : n1, k1 = r < n1 ? n1 : K0;
                double acc = 0.0;
                for (int k = k0; k < k1; ++k) acc = fma(qo[(size_t)(o + r) * n + o + k], us[(size_t)k * K0 + c], acc);
                qn[(size_t)(o + r) * n + o + c] = acc;
            }
        }
        dc_sync(grp, gs);   // the group's shared arrays are rewritten by its next subproblem
    }
    if (fail && info) atomicMax(info + mat, 1);
}

// Q_new = blockdiag(Q1, Q2) U of every merge of one level with S > DC_SMALL, double precision
// on the FP64 tensor path: blockIdx.z = (matrix * nsub + subproblem) * 2 + half, half 0 the
// rows of the first child (Q1 times rows 0..n1-1 of U), half 1 the second.  Output tiles of
// 64 x 128 per CTA of 256 threads; 8 warps of 32 x 32 (4 x 4 DMMA blocks of 8 x 8 each, lane
// (g, q) holding C(8i+g, 8j+2q .. 2q+1)); the inner dimension advances 16 at a time through two
// shared-memory stages, the next stage's global loads issued into registers before the current
// one is consumed.  Leading dimension 68 of the shared tiles: the 16-lane phases of the 8-byte
// fragment loads (rows q, columns g) hit distinct banks.
static constexpr int DG_BM = 64, DG_BN = 128, DG_KC = 16, DG_LD = 68, DG_LDB = 132;
struct DgTiles {
    double a[2][DG_KC][DG_LD];
    double b[2][DG_KC][DG_LDB];
};

__device__ __forceinline__ void dmma884r(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256, 2)
k_dc_gemm(const double* __restrict__ Qo, const double* __restrict__ U, double* __restrict__ Qn, int n, int S,
          int nsub) {
    extern __shared__ __align__(16) unsigned char dg_smem[];
    DgTiles& s = *reinterpret_cast<DgTiles*>(dg_smem);
    const int z = blockIdx.z;
    const int h = z & 1;
    const int sub = (z >> 1) % nsub;
    const size_t mat = (size_t)(z >> 1) / nsub;
    const int o = sub * S;
    const int K0 = min(S, n - o), n1 = min(S / 2, K0), n2 = K0 - n1;
    if (n2 <= 0) return;   // single child: copied by k_dc_merge
    const int M = h ? n2 : n1, off = h ? n1 : 0;   // rows and inner dimension of this half
    const int r0 = blockIdx.x * DG_BM, c0 = blockIdx.y * DG_BN;
    if (r0 >= M || c0 >= K0) return;   // whole CTA leaves together
    const int smax = dc_smax(S, n);
    const double* A = Qo + mat * (size_t)n * n + (size_t)(o + off) * n + (o + off);   // A(r, k) = A[r*n + k]
    const double* B = U + mat * (size_t)n * n + (size_t)o * smax + (size_t)off * K0;  // B(k, c) = B[k*K0 + c]
    double* C = Qn + mat * (size_t)n * n + (size_t)(o + off) * n + o;                 // C(r, c) = C[r*n + c]
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wr = warp & 1, wc = warp >> 1, g = lane >> 2, q = lane & 3;
    double fa[4], fb[8];
    auto load = [&](int k0) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {   // A tile 64 x 16, k fastest
            const int idx = t + 256 * e, kk = idx % DG_KC, rr = idx / DG_KC;
            const int r = r0 + rr, k = k0 + kk;
            fa[e] = (r < M && k < M) ? A[(size_t)r * n + k] : 0.0;
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {   // B tile 16 x 128, c fastest
            const int idx = t + 256 * e, cc = idx % DG_BN, kk = idx / DG_BN;
            const int c = c0 + cc, k = k0 + kk;
            fb[e] = (c < K0 && k < M) ? B[(size_t)k * K0 + c] : 0.0;
        }
    };
    auto put = [&](int buf) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int idx = t + 256 * e;
            s.a[buf][idx % DG_KC][idx / DG_KC] = fa[e];
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int idx = t + 256 * e;
            s.b[buf][idx / DG_BN][idx % DG_BN] = fb[e];
        }
    };
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int nk = (M + DG_KC - 1) / DG_KC;
    load(0);
    put(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        const int cur = kt & 1;
        const bool more = kt + 1 < nk;
        if (more) load((kt + 1) * DG_KC);
#pragma unroll
        for (int k4 = 0; k4 < DG_KC; k4 += 4) {
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) av[i] = s.a[cur][k4 + q][32 * wr + 8 * i + g];
#pragma unroll
            for (int j = 0; j < 4; ++j) bv[j] = s.b[cur][k4 + q][32 * wc + 8 * j + g];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma884r(acc[i][j], av[i], bv[j]);
        }
        if (more) put(cur ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = r0 + 32 * wr + 8 * i + g;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int c = c0 + 32 * wc + 8 * j + 2 * q + e;
                if (c < K0) C[(size_t)r * n + c] = acc[i][j][e];
            }
    }
}

// Largest number of matrices one divide-and-conquer launch sequence may take: the grid z extent
// of k_dc_gemm (two halves per subproblem at the first GEMM level).
__host__ inline size_t dc_max_chunk(int n) {
    int S = 2;
    while (S <= DC_SMALL) S *= 2;
    const size_t nsub = ((size_t)n + S - 1) / S;
    return S / 2 < n ? 65535 / (2 * nsub) : 65535;
}

}  // namespace rlmb
