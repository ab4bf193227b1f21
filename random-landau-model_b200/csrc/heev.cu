// Batched complex Hermitian eigensolver, double precision (sm_100a).
//
// Replaces the reference's dense solver calls: mkl_heevd (diag_wrappers/mkl_diag.cpp:2-9,
// LAPACKE_zheevd col-major 'U'), cusolver_diag_hamil (diag_wrappers/cusolver_diag.cu:3-22)
// and magma_diag_hamil (diag_wrappers/magma_diag.cu:2-49).  The LAPACK arithmetic those
// calls reach is restated from its published algorithms, in three kernels per batch:
//
//   k_hetrd   Householder reduction A = Q T Q^H (LAPACK zhetd2, uplo='U'): one CTA per
//             matrix, the matrix itself in global memory (L2 resident while its CTA
//             runs); per column a reflector (zlarfg), a Hermitian matrix-vector product
//             over 32x32 tiles that reads every stored element once and uses it for
//             both the row and the transposed contribution, and a rank-2 update.
//   k_tridiag Eigenvalues of T by Sturm-count bisection (one thread per eigenvalue,
//             LAPACK dstebz), eigenvectors by inverse iteration with partial-pivoting
//             LU of T - lambda I and modified Gram-Schmidt inside clusters (dstein).
//   k_ormtr   Back-transformation X = Q Z (zunmtr): one CTA per (matrix, 16-column
//             chunk of Z) holding the chunk in shared memory.
//
// Every wait is a __syncthreads inside one CTA: no inter-CTA dependencies, no spins.
#include "common.cuh"

#include <cfloat>
#include <cmath>

namespace rlmb {

static constexpr int HETRD_THREADS = 256;   // 8 warps
static constexpr int ORMTR_COLS = 16;       // Z columns per back-transform CTA
static constexpr int ORMTR_THREADS = 256;

// --------------------------------------------------------------- block reductions
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) s += red[i];
    return s;
}
template <int NT>
__device__ __forceinline__ cplx block_sum(cplx v, double* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        red[2 * w] = v.x;
        red[2 * w + 1] = v.y;
    }
    __syncthreads();
    cplx s = mk(0, 0);
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) s = cadd(s, mk(red[2 * i], red[2 * i + 1]));
    return s;
}

// Transpose-reduce: lane l holds vals[j] (j < 32, the contribution of row l to column j);
// on return vals[0] on lane l is the sum over all 32 lanes of vals[l].
__device__ __forceinline__ cplx transpose_reduce32(cplx (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool up = (lane & s) != 0;
#pragma unroll
        for (int j = 0; j < s; ++j) {
            cplx send = up ? v[j] : v[j + s];
            cplx keep = up ? v[j + s] : v[j];
            v[j] = cadd(keep, shfl_xor(send, s));
        }
    }
    return v[0];
}

__device__ __forceinline__ void tile_of(int t, int& R, int& C) {
    // t-th tile (row block R <= column block C) in column-major order of the upper triangle
    int c = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((c + 1) * (c + 2) / 2 <= t) ++c;
    while (c * (c + 1) / 2 > t) --c;
    C = c;
    R = t - c * (c + 1) / 2;
}

__device__ __forceinline__ void smem_atomic_add(cplx* p, cplx v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}

// ------------------------------------------------------------------ k_hetrd
// a: n*n col-major, upper triangle.  On exit: column c (c >= 1) rows 0..c-2 hold the
// reflector of step c-1 (v[c-1] = 1 implicit), diag/offdiag in dd/ee, tau in tt.
__global__ void __launch_bounds__(HETRD_THREADS)
k_hetrd(cplx* __restrict__ A, double* __restrict__ D, double* __restrict__ E,
        cplx* __restrict__ TAU, int n) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* v = reinterpret_cast<cplx*>(smem_raw);   // [n] reflector
    cplx* p = v + n;                                // [n] A v, then w
    double* red = reinterpret_cast<double*>(p + n); // [2*warps]
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    constexpr int NW = HETRD_THREADS / 32;
    const size_t mat = blockIdx.x;
    cplx* a = A + mat * (size_t)n * n;
    double* dd = D + mat * n;
    double* ee = E + mat * n;
    cplx* tt = TAU + mat * n;

    for (int i = n - 2; i >= 0; --i) {
        const int c = i + 1;   // column holding the vector to annihilate
        const int m = i + 1;   // leading block rows/cols 0..i
        // ---- (1) reflector from column c, rows 0..i  (zlarfg)
        double part = 0.0;
        for (int r = tid; r <= i; r += HETRD_THREADS) {
            cplx x = a[(size_t)c * n + r];
            v[r] = x;
            if (r < i) part += cabs2(x);
        }
        const double xnorm2 = block_sum<HETRD_THREADS>(part, red);   // syncs
        const cplx alpha = v[i];
        double beta = 0.0;
        cplx tau = mk(0, 0), scal = mk(0, 0);
        if (xnorm2 == 0.0 && alpha.y == 0.0) {
            beta = alpha.x;
        } else {
            const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
            beta = alpha.x >= 0.0 ? -nrm : nrm;
            tau = mk((beta - alpha.x) / beta, -alpha.y / beta);
            const cplx den = mk(alpha.x - beta, alpha.y);
            const double dn = cabs2(den);
            scal = mk(den.x / dn, -den.y / dn);
        }
        const bool active = !(tau.x == 0.0 && tau.y == 0.0);
        __syncthreads();
        for (int r = tid; r < i; r += HETRD_THREADS) {
            cplx x = active ? cmul(scal, v[r]) : v[r];
            v[r] = x;
            a[(size_t)c * n + r] = x;
        }
        if (tid == 0) {
            v[i] = mk(1.0, 0.0);
            a[(size_t)c * n + i] = mk(beta, 0.0);
            ee[i] = beta;
            tt[i] = tau;
        }
        for (int r = tid; r < m; r += HETRD_THREADS) p[r] = mk(0, 0);
        __syncthreads();
        if (active) {
            // ---- (2) p = A(0:i,0:i) v over 32x32 tiles of the upper triangle
            const int nb = (m + 31) / 32;
            const int ntiles = nb * (nb + 1) / 2;
            for (int t = warp; t < ntiles; t += NW) {
                int R, C;
                tile_of(t, R, C);
                const int r = R * 32 + lane;
                const cplx vr = r < m ? v[r] : mk(0, 0);
                cplx rowacc = mk(0, 0);
                cplx col[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int cc = C * 32 + j;
                    cplx e = mk(0, 0);
                    if (r < m && cc < m && r <= cc) e = a[(size_t)cc * n + r];
                    const cplx vc = cc < m ? v[cc] : mk(0, 0);
                    if (r == cc) {
                        rowacc = cadd(rowacc, cscale(vc, e.x));
                        col[j] = mk(0, 0);
                    } else {
                        cfma(rowacc, e, vc);
                        col[j] = cmulc(e, vr);
                    }
                }
                const cplx cs = transpose_reduce32(col);
                if (r < m) smem_atomic_add(&p[r], rowacc);
                const int cl = C * 32 + lane;
                if (cl < m) smem_atomic_add(&p[cl], cs);
            }
            __syncthreads();
            // ---- (3) x = tau p;  alpha2 = -tau/2 (x^H v);  w = x + alpha2 v
            cplx dpart = mk(0, 0);
            for (int r = tid; r < m; r += HETRD_THREADS) {
                const cplx x = cmul(tau, p[r]);
                p[r] = x;
                cfmac(dpart, x, v[r]);
            }
            const cplx xv = block_sum<HETRD_THREADS>(dpart, red);   // syncs
            const cplx al = cscale(cmul(tau, xv), -0.5);
            for (int r = tid; r < m; r += HETRD_THREADS) cfma(p[r], al, v[r]);
            __syncthreads();
            // ---- (4) A(0:i,0:i) -= v w^H + w v^H  (upper triangle, diagonal kept real)
            for (int cc = warp; cc < m; cc += NW) {
                const cplx vc = v[cc], wc = p[cc];
                for (int r = lane; r <= cc; r += 32) {
                    cplx e = a[(size_t)cc * n + r];
                    const cplx vr = v[r], wr = p[r];
                    // e -= v_r conj(w_c) + w_r conj(v_c)
                    cplx u = cmul(vr, cconj(wc));
                    cfma(u, wr, cconj(vc));
                    e = csub(e, u);
                    if (r == cc) e.y = 0.0;
                    a[(size_t)cc * n + r] = e;
                }
            }
            __syncthreads();
        } else {
            if (tid == 0) a[(size_t)i * n + i].y = 0.0;
            __syncthreads();
        }
        if (tid == 0) dd[c] = a[(size_t)c * n + c].x;
    }
    if (tid == 0) {
        dd[0] = a[0].x;
        ee[n - 1] = 0.0;
        tt[n - 1] = mk(0, 0);
    }
}

// ------------------------------------------------------------ k_tridiag
// Eigen-decomposition of the real symmetric tridiagonal (d, e), one CTA per matrix.
// Eigenvalues by bisection; eigenvector k by inverse iteration, stored row-major in
// Z (Z[j*n + k] = component j of eigenvector k) so that the recurrences of the n
// threads touch consecutive addresses.  Per-thread LU factors live in the interleaved
// workspace lu (5*n*n doubles per matrix, same layout).
static constexpr int TRI_THREADS = 256;
static constexpr int INV_MAXITS = 5;

__device__ int sturm_count(const double* __restrict__ d, const double* __restrict__ e2, int n,
                           double x, double pivmin) {
    double q = d[0] - x;
    if (fabs(q) <= pivmin) q = -pivmin;
    int cnt = q < 0.0;
    for (int j = 1; j < n; ++j) {
        q = d[j] - x - e2[j - 1] / q;
        if (fabs(q) <= pivmin) q = -pivmin;
        cnt += q < 0.0;
    }
    return cnt;
}

// deterministic start vector entries in (-1, 1)
__device__ __forceinline__ double start_entry(int k, int j) {
    uint32_t h = (uint32_t)k * 0x9E3779B1u ^ ((uint32_t)j * 0x85EBCA77u + 0x165667B1u);
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    h *= 0x297A2D39u;
    h ^= h >> 15;
    return ((double)h + 0.5) * (2.0 / 4294967296.0) - 1.0;
}

__global__ void __launch_bounds__(TRI_THREADS)
k_tridiag(const double* __restrict__ D, const double* __restrict__ E, double* __restrict__ W,
          double* __restrict__ Z, double* __restrict__ LU, int* __restrict__ info, int n) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* d = reinterpret_cast<double*>(smem_raw);   // [n]
    double* e = d + n;                                  // [n]
    double* e2 = e + n;                                 // [n]
    double* lam = e2 + n;                               // [n]
    int* leader = reinterpret_cast<int*>(lam + n);      // [n] first index of k's cluster
    __shared__ double s_gl, s_gu, s_pivmin, s_onenrm;
    __shared__ int s_fail;
    const int tid = threadIdx.x;
    const size_t mat = blockIdx.x;
    const size_t nn = (size_t)n * n;
    double* z = Z + mat * nn;
    double* la = LU + mat * 5 * nn;    // a (U main), b (U super1), c2 (U super2), mult, piv
    double* lb = la + nn;
    double* lc2 = lb + nn;
    double* lm = lc2 + nn;
    double* lp = lm + nn;

    for (int j = tid; j < n; j += TRI_THREADS) {
        d[j] = D[mat * n + j];
        const double ej = j < n - 1 ? E[mat * n + j] : 0.0;
        e[j] = ej;
        e2[j] = ej * ej;
    }
    if (tid == 0) s_fail = 0;
    __syncthreads();
    if (tid == 0) {
        double gl = d[0], gu = d[0], emax2 = 0.0, onenrm = 0.0;
        for (int j = 0; j < n; ++j) {
            const double off = (j > 0 ? fabs(e[j - 1]) : 0.0) + (j < n - 1 ? fabs(e[j]) : 0.0);
            gl = fmin(gl, d[j] - off);
            gu = fmax(gu, d[j] + off);
            onenrm = fmax(onenrm, fabs(d[j]) + off);
            if (j < n - 1) emax2 = fmax(emax2, e2[j]);
        }
        const double pivmin = DBL_MIN * fmax(1.0, emax2);
        const double tnorm = fmax(fabs(gl), fabs(gu));
        gl -= 2.1 * tnorm * DBL_EPSILON * n + 4.2 * pivmin;
        gu += 2.1 * tnorm * DBL_EPSILON * n + 4.2 * pivmin;
        s_gl = gl;
        s_gu = gu;
        s_pivmin = pivmin;
        s_onenrm = fmax(onenrm, DBL_MIN);
    }
    __syncthreads();
    const double pivmin = s_pivmin, onenrm = s_onenrm;
    // ---- eigenvalues: bisection for index k
    const double atol = 2.0 * DBL_EPSILON * onenrm;
    for (int k = tid; k < n; k += TRI_THREADS) {
        double lo = s_gl, hi = s_gu;
        for (int it = 0; it < 200 && hi - lo > fmax(atol, 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi))); ++it) {
            const double mid = 0.5 * (lo + hi);
            if (mid <= lo || mid >= hi) break;
            if (sturm_count(d, e2, n, mid, pivmin) > k) hi = mid; else lo = mid;
        }
        lam[k] = 0.5 * (lo + hi);
    }
    __syncthreads();
    // ---- clusters (relative gap 1e-5 of the norm) and eigenvalue output
    const double ortol = 1e-5 * onenrm;
    if (tid == 0) {
        int lead = 0;
        for (int k = 0; k < n; ++k) {
            if (k > 0 && lam[k] - lam[k - 1] > ortol) lead = k;
            leader[k] = lead;
        }
    }
    for (int k = tid; k < n; k += TRI_THREADS) W[mat * n + k] = lam[k];
    __syncthreads();
    // ---- eigenvectors by inverse iteration; a cluster is handled by its leader's thread
    const double eps = DBL_EPSILON;
    const double dtpcrt = sqrt(0.1 / n);
    if (!(onenrm > 1e3 * DBL_MIN)) {
        // T = 0 (to underflow): every vector is an eigenvector; return the unit vectors
        for (int k = tid; k < n; k += TRI_THREADS)
            for (int j = 0; j < n; ++j) z[(size_t)j * n + k] = j == k ? 1.0 : 0.0;
        __syncthreads();
        if (tid == 0 && info) info[mat] = 0;
        return;
    }
    for (int k0 = tid; k0 < n; k0 += TRI_THREADS) {
        if (leader[k0] != k0) continue;
        int k1 = k0;
        while (k1 + 1 < n && leader[k1 + 1] == k0) ++k1;
        double xjm = lam[k0];
        for (int k = k0; k <= k1; ++k) {
            double x = lam[k];
            if (k > k0) {
                const double pertol = 10.0 * fabs(x) * eps + 10.0 * eps * onenrm * 1e-3;
                if (x - xjm < pertol) x = xjm + pertol;
            }
            xjm = x;
            // LU with partial pivoting of T - x I (dlagtf).  The active row carries
            // (u0, u1) = its entries in columns j, j+1; the row pivoted into position j is
            // stored as U diag / super1 / super2 (la, lb, lc2), the multiplier in lm and
            // the swap flag in lp, all at [j*n + k].
            double u0 = d[0] - x, u1 = n > 1 ? e[0] : 0.0;
            for (int j = 0; j < n - 1; ++j) {
                const double cj = e[j];
                const double anext = d[j + 1] - x;
                const double bnext = j + 1 < n - 1 ? e[j + 1] : 0.0;
                const size_t o = (size_t)j * n + k;
                if (fabs(u0) >= fabs(cj)) {
                    const double mult = u0 != 0.0 ? cj / u0 : 0.0;
                    la[o] = u0;
                    lb[o] = u1;
                    lc2[o] = 0.0;
                    lm[o] = mult;
                    lp[o] = 0.0;
                    u0 = anext - mult * u1;
                    u1 = bnext;
                } else {
                    const double mult = u0 / cj;
                    la[o] = cj;
                    lb[o] = anext;
                    lc2[o] = bnext;
                    lm[o] = mult;
                    lp[o] = 1.0;
                    u0 = u1 - mult * anext;
                    u1 = -mult * bnext;
                }
            }
            la[(size_t)(n - 1) * n + k] = u0;
            lb[(size_t)(n - 1) * n + k] = 0.0;
            lc2[(size_t)(n - 1) * n + k] = 0.0;
            // tiny pivots are perturbed to +-tolp in the solves (dlagts job = -1)
            double umax = 0.0;
            for (int j = 0; j < n; ++j) umax = fmax(umax, fabs(la[(size_t)j * n + k]));
            const double tolp = fmax(eps * fmax(umax, onenrm), DBL_MIN);
            for (int j = 0; j < n; ++j) z[(size_t)j * n + k] = start_entry(k, j);
            int nrmchk = 0;
            bool conv = false;
            for (int its = 0; its < INV_MAXITS; ++its) {
                // scale the right-hand side to ||b||_1 = n * onenrm * max(eps, |u_nn|)
                double b1 = 0.0;
                for (int j = 0; j < n; ++j) b1 += fabs(z[(size_t)j * n + k]);
                const double unn = fabs(la[(size_t)(n - 1) * n + k]);
                const double sc = n * onenrm * fmax(eps, unn) / fmax(b1, DBL_MIN);
                // forward: y = L^{-1} P b  (the active right-hand side value is carried)
                double rc = z[k] * sc;
                for (int j = 0; j < n - 1; ++j) {
                    const size_t o = (size_t)j * n + k;
                    const double bnext = z[(size_t)(j + 1) * n + k] * sc;
                    const double mult = lm[o];
                    if (lp[o] != 0.0) {
                        z[o] = bnext;
                        rc = rc - mult * bnext;
                    } else {
                        z[o] = rc;
                        rc = bnext - mult * rc;
                    }
                }
                z[(size_t)(n - 1) * n + k] = rc;
                // backward: U x = y
                double x1 = 0.0, x2 = 0.0;   // x_{j+1}, x_{j+2}
                double xmax = 0.0;
                for (int j = n - 1; j >= 0; --j) {
                    const size_t o = (size_t)j * n + k;
                    double u = la[o];
                    if (fabs(u) < tolp) u = u >= 0.0 ? tolp : -tolp;
                    const double xj = (z[o] - lb[o] * x1 - lc2[o] * x2) / u;
                    z[o] = xj;
                    x2 = x1;
                    x1 = xj;
                }
                // modified Gram-Schmidt against the earlier members of the cluster
                for (int q = k0; q < k; ++q) {
                    double dot = 0.0;
                    for (int j = 0; j < n; ++j) dot += z[(size_t)j * n + q] * z[(size_t)j * n + k];
                    for (int j = 0; j < n; ++j) z[(size_t)j * n + k] -= dot * z[(size_t)j * n + q];
                }
                for (int j = 0; j < n; ++j) xmax = fmax(xmax, fabs(z[(size_t)j * n + k]));
                if (xmax < dtpcrt) continue;   // not yet amplified enough
                if (++nrmchk < 3) continue;    // two extra iterations after acceptance
                conv = true;
                break;
            }
            // normalise, largest component positive (dstein)
            double x2s = 0.0, big = 0.0;
            for (int j = 0; j < n; ++j) {
                const double t = z[(size_t)j * n + k];
                x2s += t * t;
                if (fabs(t) > fabs(big)) big = t;
            }
            double rn = 1.0 / sqrt(fmax(x2s, DBL_MIN));
            if (big < 0.0) rn = -rn;
            for (int j = 0; j < n; ++j) z[(size_t)j * n + k] *= rn;
            if (!conv) atomicAdd(&s_fail, 1);
        }
    }
    __syncthreads();
    if (tid == 0 && info) info[mat] = s_fail;
}

// --------------------------------------------------------------- k_ormtr
// X = Q Z, Q = H_{n-2} ... H_0; H_i = I - tau_i v_i v_i^H, v_i on rows 0..i with
// v_i[i] = 1 and v_i[0..i-1] stored in A[0..i-1][i+1].  One CTA per `ch` columns of Z
// (ch <= ORMTR_COLS, chosen so that the n x ch chunk fits in shared memory).
__global__ void __launch_bounds__(ORMTR_THREADS)
k_ormtr(const cplx* __restrict__ A, const cplx* __restrict__ TAU, const double* __restrict__ Z,
        cplx* __restrict__ X, int n, int ch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* xs = reinterpret_cast<cplx*>(smem_raw);        // [n][ch]
    cplx* sv = xs + (size_t)n * ch;                       // [ch] tau v^H x per column
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = ORMTR_THREADS / 32;
    const size_t mat = blockIdx.y;
    const int col0 = blockIdx.x * ch;
    const int ncols = min(ch, n - col0);
    const cplx* a = A + mat * (size_t)n * n;
    const double* z = Z + mat * (size_t)n * n;
    for (int idx = tid; idx < n * ch; idx += ORMTR_THREADS) {
        const int r = idx / ch, j = idx % ch;
        xs[idx] = j < ncols ? mk(z[(size_t)r * n + col0 + j], 0.0) : mk(0, 0);
    }
    __syncthreads();
    for (int i = 0; i <= n - 2; ++i) {
        const cplx tau = TAU[mat * n + i];
        if (tau.x == 0.0 && tau.y == 0.0) continue;
        const cplx* vcol = a + (size_t)(i + 1) * n;
        for (int j = warp; j < ncols; j += NW) {
            cplx s = mk(0, 0);
            for (int r = lane; r <= i; r += 32) {
                const cplx vr = r < i ? vcol[r] : mk(1.0, 0.0);
                cfmac(s, vr, xs[r * ch + j]);
            }
            s = warp_sum(s);
            if (lane == 0) sv[j] = cmul(tau, s);
        }
        __syncthreads();
        for (int idx = tid; idx < (i + 1) * ch; idx += ORMTR_THREADS) {
            const int r = idx / ch, j = idx % ch;
            if (j < ncols) {
                const cplx vr = r < i ? vcol[r] : mk(1.0, 0.0);
                xs[idx] = csub(xs[idx], cmul(vr, sv[j]));
            }
        }
        __syncthreads();
    }
    cplx* x = X + mat * (size_t)n * n;
    for (int idx = tid; idx < n * ch; idx += ORMTR_THREADS) {
        const int j = idx / n, r = idx % n;   // coalesced along r of column col0+j
        if (j < ncols) x[(size_t)(col0 + j) * n + r] = xs[r * ch + j];
    }
}

}  // namespace rlmb

using namespace rlmb;

extern "C" int rlmb_heevd_batched(rlmb_context* ctx, double* d_a, double* d_w, int n, int batch,
                                  int* d_info) {
    if (!ctx || !d_a || !d_w || n <= 0 || batch < 0) return RLMB_ERR_ARG;
    if (batch == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t nn = (size_t)n * n;
    // workspace per matrix: D,E (2n), TAU (2n doubles), Z (nn), LU (5nn), X (2nn)
    const size_t per = (size_t)(4 * n) + nn + 5 * nn + 2 * nn;
    // process in chunks bounded by a workspace budget (~8 GB)
    const size_t budget = (size_t)8 << 30;
    size_t chunk = budget / (per * sizeof(double));
    if (chunk < 1) chunk = 1;
    if (chunk > (size_t)batch) chunk = batch;
    if (int rc = ensure_workspace(ctx, chunk * per * sizeof(double))) return rc;
    double* ws = reinterpret_cast<double*>(ctx->ws);
    double* Dw = ws;
    double* Ew = Dw + chunk * n;
    cplx* TAUw = reinterpret_cast<cplx*>(Ew + chunk * n);
    double* Zw = reinterpret_cast<double*>(TAUw + chunk * n);
    double* LUw = Zw + chunk * nn;
    cplx* Xw = reinterpret_cast<cplx*>(LUw + 5 * chunk * nn);

    const size_t smem_trd = 2 * n * sizeof(cplx) + 2 * (HETRD_THREADS / 32) * sizeof(double);
    const size_t smem_tri = 4 * n * sizeof(double) + n * sizeof(int);
    int ch = ORMTR_COLS;
    while (ch > 1 && (size_t)(n + 1) * ch * sizeof(cplx) > 200 * 1024) ch >>= 1;
    const size_t smem_orm = (size_t)(n + 1) * ch * sizeof(cplx);
    if (smem_trd > 227 * 1024 || smem_tri > 227 * 1024 || smem_orm > 227 * 1024) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaFuncSetAttribute(k_hetrd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_trd));
    RLMB_CUDA_TRY(cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_tri));
    RLMB_CUDA_TRY(cudaFuncSetAttribute(k_ormtr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_orm));

    for (size_t b0 = 0; b0 < (size_t)batch; b0 += chunk) {
        const int nb = (int)std::min(chunk, (size_t)batch - b0);
        cplx* A = reinterpret_cast<cplx*>(d_a) + b0 * nn;
        prof_begin(ctx, "k_hetrd");
        k_hetrd<<<nb, HETRD_THREADS, smem_trd, st>>>(A, Dw, Ew, TAUw, n);
        RLMB_LAUNCHED(ctx);
        prof_begin(ctx, "k_tridiag");
        k_tridiag<<<nb, TRI_THREADS, smem_tri, st>>>(Dw, Ew, d_w + b0 * n, Zw, LUw,
                                                    d_info ? d_info + b0 : nullptr, n);
        RLMB_LAUNCHED(ctx);
        dim3 g((n + ch - 1) / ch, nb);
        prof_begin(ctx, "k_ormtr");
        k_ormtr<<<g, ORMTR_THREADS, smem_orm, st>>>(A, TAUw, Zw, Xw, n, ch);
        RLMB_LAUNCHED(ctx);
        RLMB_CUDA_TRY(cudaMemcpyAsync(A, Xw, nb * nn * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    }
    return RLMB_OK;
}
