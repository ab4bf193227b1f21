// Batched two-sided cyclic Jacobi eigensolver for small complex Hermitian matrices, double
// precision, one CTA per matrix with the matrix and its rotations resident in shared memory.
//
// It is the small-order alternative to the Householder path of heev.cu (reduction,
// tridiagonal solve, back-transformation), both replacing the reference's per-matrix
// LAPACKE_zheevd (diag_wrappers/mkl_diag.cpp:2-9).  Same contract: the upper triangle of each
// column-major matrix is read, eigenvalues ascend, eigenvector k overwrites column k.
//
// Algorithm (cyclic Jacobi with the round-robin "tournament" ordering, so that the n/2 rotations
// of one round touch disjoint index pairs and run in parallel):
//   for each sweep, until the off-diagonal mass is below 1e-32 of the total mass:
//     for each of the m-1 rounds (m = n rounded up to even; index n is a bye for odd n):
//       1. thread k computes the rotation of pair k from A_pp, A_qq and A_pq = r e (|e| = 1):
//          tau = (A_qq - A_pp) / 2r, t = sgn(tau) / (|tau| + sqrt(1 + tau^2)),
//          c = 1/sqrt(1 + t^2), s = t c, J = [[c, s e], [-s conj(e), c]] on (p, q);
//          then J^H A J has (p, q) entry 0 and diagonal A_pp - t r, A_qq + t r;
//       2. column phase, thread = (row, pair group):    A <- A J,   V <- V J;
//       3. row phase,    thread = (column, pair group): A <- J^H A, with the (p,p), (q,q),
//          (p,q), (q,p) entries set to their exact values.
// Each phase is a __syncthreads apart; there are no other waits.  Within a phase the pairs are
// disjoint, so the threads of a phase never touch the same element.
//
// Shared memory: A with an odd leading dimension (the row phase's stride-ld accesses of 16
// bytes then hit distinct banks), V with leading dimension n, the round's rotations, the
// block reduction partials.  16 (n (n|1) + n^2) bytes: 33 KB at n = 32, 131 KB at n = 64,
// 206 KB at n = 80, the largest order served (JAC_MAX_N).
#pragma once
#include "common.cuh"

namespace rlmb {

static constexpr int JAC_MAX_N = 80;
static constexpr int JAC_MAX_SWEEPS = 30;

struct JacRot {
    double c, ap, aq;   // cosine, new diagonal entries (p,p) and (q,q)
    cplx se;            // s e
    int p, q;           // q < 0: no rotation this round (bye, or A_pq already zero)
};

// Thread layout: thread = (row or column r, pair group g), r = tid % n, g = tid / n; group g
// takes pairs g, g + G, g + 2G, ...  The CTA gets W warps, enough that the matrices resident
// per SM (as many as fit in its 228 KB of shared memory) bring about 20 warps, and G fills
// those warps' lanes: at small orders many one-warp CTAs share an SM, from order ~60 on the
// matrix alone fills the SM's shared memory and its own 8 warps must hide the latency.
__host__ __device__ inline int jacobi_groups(int n);
__host__ __device__ inline size_t jacobi_smem(int n);
__host__ __device__ inline int jacobi_warps(int n) {
    int per_sm = (int)((size_t)233472 / (jacobi_smem(n) + 1024));
    per_sm = per_sm < 1 ? 1 : per_sm > 32 ? 32 : per_sm;
    const int w = (20 + per_sm - 1) / per_sm;
    return w > 8 ? 8 : w;
}
__host__ __device__ inline int jacobi_groups(int n) {
    const int np = (n + (n & 1)) / 2;
    int g = 32 * jacobi_warps(n) / (n > 0 ? n : 1);
    g = g < np ? g : np;
    return g > 0 ? g : 1;
}
__host__ __device__ inline int jacobi_threads(int n) {
    const int np = (n + (n & 1)) / 2;
    int t = n * jacobi_groups(n);
    t = t > np ? t : np;   // step 1 needs a thread per pair
    return ((t + 31) / 32) * 32;
}
__host__ __device__ inline int jacobi_ld(int n) { return n | 1; }
__host__ __device__ inline size_t jacobi_smem(int n) {
    const int m = n + (n & 1);
    return (size_t)sizeof(cplx) * ((size_t)n * jacobi_ld(n) + (size_t)n * n) + sizeof(JacRot) * (size_t)(m / 2) +
           sizeof(double) * (2 * 32 + 2 * (size_t)n) + sizeof(int) * (size_t)n;
}

// (x_p, x_q) <- (c x_p - conj(se) x_q, se x_p + c x_q): columns p, q of A J or V J
__device__ __forceinline__ void jac_rot_cols(cplx& xp, cplx& xq, double c, cplx se) {
    const cplx p0 = xp, q0 = xq;
    xp = cscale(p0, c);
    xq = cscale(q0, c);
    cfmac(xp, se, mk(-q0.x, -q0.y));
    cfma(xq, se, p0);
}
// (y_p, y_q) <- (c y_p - se y_q, conj(se) y_p + c y_q): rows p, q of J^H A
__device__ __forceinline__ void jac_rot_rows(cplx& yp, cplx& yq, double c, cplx se) {
    const cplx p0 = yp, q0 = yq;
    yp = cscale(p0, c);
    yq = cscale(q0, c);
    cfma(yp, se, mk(-q0.x, -q0.y));
    cfmac(yq, se, p0);
}

// One CTA of jacobi_threads(n) threads per matrix; dynamic shared memory jacobi_smem(n).
__global__ void __launch_bounds__(256) k_jacobi(cplx* __restrict__ Ag, double* __restrict__ W, int* __restrict__ info,
                                                int n) {
    extern __shared__ __align__(16) unsigned char jac_smem[];
    const int ld = jacobi_ld(n);
    const int m = n + (n & 1);
    const int np = m / 2;
    const int G = jacobi_groups(n);
    cplx* A = reinterpret_cast<cplx*>(jac_smem);
    cplx* V = A + (size_t)n * ld;
    JacRot* rot = reinterpret_cast<JacRot*>(V + (size_t)n * n);
    double* red = reinterpret_cast<double*>(rot + np);   // [2][32] warp partials
    double* lam = red + 64;                              // eigenvalues
    int* rank = reinterpret_cast<int*>(lam + 2 * n);
    const int tid = threadIdx.x;
    const int nt = blockDim.x;
    const int r = tid % n;             // row (column phase) or column (row phase)
    const int g = tid / n;             // pair group; g >= G: idle in the phases
    const bool act = g < G;
    const size_t mat = blockIdx.x;
    cplx* Am = Ag + mat * (size_t)n * n;

    // load: the upper triangle of column c is rows 0..c; the lower triangle is its conjugate
    for (int c = g; act && c < n; c += G) {
        if (r <= c) {
            cplx v = Am[(size_t)c * n + r];
            if (c == r) v.y = 0.0;
            A[(size_t)c * ld + r] = v;
            A[(size_t)r * ld + c] = cconj(v);
        }
        V[(size_t)c * n + r] = mk(c == r ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();

    int converged = 0;
    for (int sweep = 0; sweep <= JAC_MAX_SWEEPS; ++sweep) {
        // off-diagonal and diagonal mass
        double off = 0.0, dia = 0.0;
        for (int c = g; act && c < n; c += G) {
            const double a2 = cabs2(A[(size_t)c * ld + r]);
            if (c == r) dia += a2;
            else off += a2;
        }
        off = warp_sum(off);
        dia = warp_sum(dia);
        if ((tid & 31) == 0) {
            red[tid >> 5] = off;
            red[32 + (tid >> 5)] = dia;
        }
        __syncthreads();
        off = 0.0;
        dia = 0.0;
        for (int w = 0; w < nt / 32; ++w) {
            off += red[w];
            dia += red[32 + w];
        }
        __syncthreads();   // red is rewritten by the next sweep's check
        if (off <= 1e-32 * (off + dia)) {
            converged = 1;
            break;
        }
        if (sweep == JAC_MAX_SWEEPS) break;
        for (int rd = 0; rd < m - 1; ++rd) {
            // 1. rotations of the round, thread k for pair k
            if (tid < np) {
                int p, q;
                if (tid == 0) {
                    p = m - 1;
                    q = rd;
                } else {
                    p = (rd + tid) % (m - 1);
                    q = (rd - tid + m - 1) % (m - 1);
                }
                if (p > q) {
                    const int s = p;
                    p = q;
                    q = s;
                }
                JacRot R;
                R.p = p;
                R.q = -1;
                R.c = 1.0;
                R.se = mk(0.0, 0.0);
                R.ap = R.aq = 0.0;
                if (q < n) {
                    const cplx b = A[(size_t)q * ld + p];
                    const double rr = sqrt(cabs2(b));
                    if (rr >= 1e-300) {
                        const double a = A[(size_t)p * ld + p].x, d = A[(size_t)q * ld + q].x;
                        const double tau = (d - a) / (2.0 * rr);
                        const double at = fabs(tau);
                        const double tt = at > 1e150 ? 0.5 / at : 1.0 / (at + sqrt(1.0 + tau * tau));
                        const double tn = tau >= 0.0 ? tt : -tt;
                        const double c = 1.0 / sqrt(1.0 + tn * tn);
                        const double s = tn * c;
                        R.q = q;
                        R.c = c;
                        R.se = mk(s * b.x / rr, s * b.y / rr);
                        R.ap = a - tn * rr;
                        R.aq = d + tn * rr;
                    }
                }
                rot[tid] = R;
            }
            __syncthreads();
            // 2. columns: A <- A J, V <- V J (r = row); two pairs in flight per thread
            if (act) {
                for (int k = g; k < np; k += 2 * G) {
                    const JacRot R0 = rot[k];
                    const bool two = k + G < np;
                    const JacRot R1 = two ? rot[k + G] : R0;
                    const bool d0 = R0.q >= 0, d1 = two && R1.q >= 0;
                    cplx a0p, a0q, v0p, v0q, a1p, a1q, v1p, v1q;
                    if (d0) {
                        a0p = A[(size_t)R0.p * ld + r];
                        a0q = A[(size_t)R0.q * ld + r];
                        v0p = V[(size_t)R0.p * n + r];
                        v0q = V[(size_t)R0.q * n + r];
                    }
                    if (d1) {
                        a1p = A[(size_t)R1.p * ld + r];
                        a1q = A[(size_t)R1.q * ld + r];
                        v1p = V[(size_t)R1.p * n + r];
                        v1q = V[(size_t)R1.q * n + r];
                    }
                    if (d0) {
                        jac_rot_cols(a0p, a0q, R0.c, R0.se);
                        jac_rot_cols(v0p, v0q, R0.c, R0.se);
                        A[(size_t)R0.p * ld + r] = a0p;
                        A[(size_t)R0.q * ld + r] = a0q;
                        V[(size_t)R0.p * n + r] = v0p;
                        V[(size_t)R0.q * n + r] = v0q;
                    }
                    if (d1) {
                        jac_rot_cols(a1p, a1q, R1.c, R1.se);
                        jac_rot_cols(v1p, v1q, R1.c, R1.se);
                        A[(size_t)R1.p * ld + r] = a1p;
                        A[(size_t)R1.q * ld + r] = a1q;
                        V[(size_t)R1.p * n + r] = v1p;
                        V[(size_t)R1.q * n + r] = v1q;
                    }
                }
            }
            __syncthreads();
            // 3. rows: A <- J^H A (r = column); the pair's own 2x2 block gets its exact values
            if (act) {
                cplx* col = A + (size_t)r * ld;
                for (int k = g; k < np; k += 2 * G) {
                    const JacRot R0 = rot[k];
                    const bool two = k + G < np;
                    const JacRot R1 = two ? rot[k + G] : R0;
                    const bool d0 = R0.q >= 0, d1 = two && R1.q >= 0;
                    cplx y0p, y0q, y1p, y1q;
                    if (d0) {
                        y0p = col[R0.p];
                        y0q = col[R0.q];
                    }
                    if (d1) {
                        y1p = col[R1.p];
                        y1q = col[R1.q];
                    }
                    if (d0) {
                        if (r == R0.p) {
                            y0p = mk(R0.ap, 0.0);
                            y0q = mk(0.0, 0.0);
                        } else if (r == R0.q) {
                            y0p = mk(0.0, 0.0);
                            y0q = mk(R0.aq, 0.0);
                        } else {
                            jac_rot_rows(y0p, y0q, R0.c, R0.se);
                        }
                        col[R0.p] = y0p;
                        col[R0.q] = y0q;
                    }
                    if (d1) {
                        if (r == R1.p) {
                            y1p = mk(R1.ap, 0.0);
                            y1q = mk(0.0, 0.0);
                        } else if (r == R1.q) {
                            y1p = mk(0.0, 0.0);
                            y1q = mk(R1.aq, 0.0);
                        } else {
                            jac_rot_rows(y1p, y1q, R1.c, R1.se);
                        }
                        col[R1.p] = y1p;
                        col[R1.q] = y1q;
                    }
                }
            }
            __syncthreads();
        }
    }

    // ascending order: the rank of eigenvalue t among all (ties by index)
    if (tid < n) lam[tid] = A[(size_t)tid * ld + tid].x;
    __syncthreads();
    if (tid < n) {
        const double l = lam[tid];
        int rk = 0;
        for (int j = 0; j < n; ++j) {
            const double lj = lam[j];
            rk += (lj < l || (lj == l && j < tid)) ? 1 : 0;
        }
        rank[tid] = rk;
        W[mat * n + rk] = l;
    }
    __syncthreads();
    for (int c = g; act && c < n; c += G) Am[(size_t)rank[c] * n + r] = V[(size_t)c * n + r];
    if (tid == 0 && info) info[mat] = converged ? 0 : 1;
}

}  // namespace rlmb
