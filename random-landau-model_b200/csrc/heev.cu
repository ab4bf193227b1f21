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

// As transpose_reduce32 for a 16-column group: lane l (and l^16) receives the sum over
// all 32 lanes of v[l & 15].
__device__ __forceinline__ cplx transpose_reduce16(cplx (&v)[16]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = cadd(v[j], shfl_xor(v[j], 16));
#pragma unroll
    for (int s = 8; s >= 1; s >>= 1) {
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
// Storage of the active leading block: global column-major (ld = n) while it is large,
// packed upper triangle in shared memory (column c at c(c+1)/2) once it fits.
struct GlobalStore {
    cplx* a;
    int n;
    __device__ __forceinline__ cplx* at(int r, int c) const { return a + (size_t)c * n + r; }
};
struct SharedStore {
    cplx* s;
    __device__ __forceinline__ cplx* at(int r, int c) const { return s + (c * (c + 1) / 2 + r); }
};

// One pass over the upper triangle of the leading m x m block, 32x32 tiles dealt to
// warps: applies the rank-2 update A -= v w^H + w v^H of the previous reflector (if upd)
// and accumulates pn += A' vn for the next one (if acc), reading and writing every
// stored element once.  All 32 loads of a tile are issued before any of its stores.
template <int NT, class S>
__device__ __forceinline__ void fused_pass(S st, int m, const cplx* __restrict__ v,
                                           const cplx* __restrict__ w, bool upd,
                                           const cplx* __restrict__ vn, bool acc, cplx* pn) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    const int nb = (m + 31) / 32;
    const int nitems = nb * (nb + 1);   // two 16-column halves per 32x32 tile
    for (int it = warp; it < nitems; it += NW) {
        int R, C;
        tile_of(it >> 1, R, C);
        const int c0 = C * 32 + 16 * (it & 1);
        if (c0 >= m) continue;
        const int r = R * 32 + lane;
        const bool rin = r < m;
        const cplx vr = rin ? v[r] : mk(0, 0);
        const cplx wr = rin ? w[r] : mk(0, 0);
        const cplx vnr = rin ? vn[r] : mk(0, 0);
        cplx rowacc = mk(0, 0);
        cplx e[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int cc = c0 + j;
            e[j] = (rin && cc < m && r <= cc) ? *st.at(r, cc) : mk(0, 0);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int cc = c0 + j;
            const bool valid = rin && cc < m && r <= cc;
            cplx x = e[j];
            if (upd) {
                const cplx vc = cc < m ? v[cc] : mk(0, 0);
                const cplx wc = cc < m ? w[cc] : mk(0, 0);
                cplx u = cmul(vr, cconj(wc));
                cfma(u, wr, cconj(vc));
                x = csub(x, u);
                if (r == cc) x.y = 0.0;
                if (valid) *st.at(r, cc) = x;
            }
            if (acc) {
                const cplx vnc = cc < m ? vn[cc] : mk(0, 0);
                if (!valid) {
                    e[j] = mk(0, 0);
                } else if (r == cc) {
                    rowacc = cadd(rowacc, cscale(vnc, x.x));
                    e[j] = mk(0, 0);
                } else {
                    cfma(rowacc, x, vnc);
                    e[j] = cmulc(x, vnr);   // column partial: conj(A'[r][cc]) vn[r]
                }
            }
        }
        if (acc) {
            const cplx cs = transpose_reduce16(e);
            const int cl = c0 + (lane & 15);
            if (lane < 16 && cl < m) smem_atomic_add(&pn[cl], cs);
            if (rin) smem_atomic_add(&pn[r], rowacc);
        }
    }
}

// Householder reflector of zlarfg for (alpha, x[0..len-1]) held in col[0..len]
// (alpha = col[len]); returns beta, tau and the scale applied to x.
__device__ __forceinline__ void reflector(const cplx alpha, double xnorm2, double& beta, cplx& tau,
                                          cplx& scal) {
    if (xnorm2 == 0.0 && alpha.y == 0.0) {
        beta = alpha.x;
        tau = mk(0, 0);
        scal = mk(1, 0);
        return;
    }
    const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
    beta = alpha.x >= 0.0 ? -nrm : nrm;
    tau = mk((beta - alpha.x) / beta, -alpha.y / beta);
    const cplx den = mk(alpha.x - beta, alpha.y);
    const double dn = cabs2(den);
    scal = mk(den.x / dn, -den.y / dn);
}

// Unblocked reduction A = Q T Q^H (zhetd2, uplo='U') with look-ahead: step i's rank-2
// update and step i-1's matrix-vector product share one pass over the leading block.
// a: n*n col-major (upper triangle).  On exit column c (c >= 1) rows 0..c-2 hold the
// reflector of step c-1 (its entry c-1 is 1 and not stored), D/E the tridiagonal and TAU
// the reflector scalars.  The leading block moves into shared memory once its packed
// upper triangle fits in `tri_cap` elements.
template <int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 4)
k_hetrd(cplx* __restrict__ A, double* __restrict__ D, double* __restrict__ E,
        cplx* __restrict__ TAU, int n, int tri_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* v = reinterpret_cast<cplx*>(smem_raw);   // [n] current reflector
    cplx* w = v + n;                                // [n] its w vector
    cplx* vn = w + n;                               // [n] next reflector / column buffer
    cplx* pn = vn + n;                              // [n] A' vn accumulator
    double* red = reinterpret_cast<double*>(pn + n);  // [2*warps]
    cplx* tri = reinterpret_cast<cplx*>(red + 2 * (NT / 32));   // packed triangle
    const int tid = threadIdx.x;
    const size_t mat = blockIdx.x;
    GlobalStore gs{A + mat * (size_t)n * n, n};
    SharedStore ss{tri};
    double* dd = D + mat * n;
    double* ee = E + mat * n;
    cplx* tt = TAU + mat * n;
    if (n == 1) {
        if (tid == 0) {
            dd[0] = gs.at(0, 0)->x;
            ee[0] = 0.0;
            tt[0] = mk(0, 0);
        }
        return;
    }
    bool resident = false;
    // -- prologue: reflector of step n-2 from column n-1, then p = A v over [0..n-2]^2
    {
        const int i = n - 2;
        double part = 0.0;
        for (int r = tid; r <= i + 1; r += NT) {
            const cplx x = *gs.at(r, i + 1);
            vn[r] = x;
            if (r < i) part += cabs2(x);
        }
        const double xn2 = block_sum<NT>(part, red);
        double beta;
        cplx tau, scal;
        reflector(vn[i], xn2, beta, tau, scal);
        const bool act = !(tau.x == 0.0 && tau.y == 0.0);
        __syncthreads();
        for (int r = tid; r < i; r += NT) {
            const cplx x = act ? cmul(scal, vn[r]) : vn[r];
            v[r] = x;
            *gs.at(r, i + 1) = x;
        }
        for (int r = tid; r < n; r += NT) {
            w[r] = mk(0, 0);
            pn[r] = mk(0, 0);
        }
        if (tid == 0) {
            v[i] = mk(1.0, 0.0);
            dd[n - 1] = vn[n - 1].x;
            *gs.at(i, i + 1) = mk(beta, 0.0);
            ee[i] = beta;
            tt[i] = tau;
        }
        __syncthreads();
        fused_pass<NT>(gs, i + 1, v, w, false, v, act, pn);
        __syncthreads();
        cplx dpart = mk(0, 0);
        for (int r = tid; r <= i; r += NT) {
            const cplx x = cmul(tau, pn[r]);
            pn[r] = x;
            cfmac(dpart, x, v[r]);
        }
        const cplx xv = block_sum<NT>(dpart, red);
        const cplx al = cscale(cmul(tau, xv), -0.5);
        for (int r = tid; r <= i; r += NT) w[r] = cadd(pn[r], cmul(al, v[r]));
        __syncthreads();
    }
    // -- main loop: v, w belong to step i (column i+1 done); finish column i, build the
    //    reflector of step i-1 from it, then one fused pass over [0..i-1]^2
    for (int i = n - 2; i >= 1; --i) {
        if (!resident && (i + 1) * (i + 2) / 2 <= tri_cap) {
            // move the leading (i+1)x(i+1) upper triangle into shared memory
            for (int c = 0; c <= i; ++c)
                for (int r = tid; r <= c; r += NT) *ss.at(r, c) = *gs.at(r, c);
            resident = true;
            __syncthreads();
        }
        // (1) updated column i, rows 0..i
        double part = 0.0;
        const cplx wi = w[i], vi = v[i];
        for (int r = tid; r <= i; r += NT) {
            cplx x = resident ? *ss.at(r, i) : *gs.at(r, i);
            cplx u = cmul(v[r], cconj(wi));
            cfma(u, w[r], cconj(vi));
            x = csub(x, u);
            vn[r] = x;
            if (r < i - 1) part += cabs2(x);
            pn[r] = mk(0, 0);
        }
        const double xn2 = block_sum<NT>(part, red);
        // (2) reflector of step i-1: alpha = A'[i-1][i], x = A'[0..i-2][i]
        double beta;
        cplx tau, scal;
        reflector(vn[i - 1], xn2, beta, tau, scal);
        const bool act = !(tau.x == 0.0 && tau.y == 0.0);
        __syncthreads();
        if (tid == 0) dd[i] = vn[i].x;
        for (int r = tid; r < i - 1; r += NT) {
            const cplx x = act ? cmul(scal, vn[r]) : vn[r];
            vn[r] = x;
            *gs.at(r, i) = x;   // reflector storage stays in global memory
        }
        if (tid == 0) {
            vn[i - 1] = mk(1.0, 0.0);
            *gs.at(i - 1, i) = mk(beta, 0.0);
            ee[i - 1] = beta;
            tt[i - 1] = tau;
        }
        __syncthreads();
        // (3) fused pass: update [0..i-1]^2 with (v, w), accumulate pn = A' vn
        if (resident) fused_pass<NT>(ss, i, v, w, true, vn, act, pn);
        else fused_pass<NT>(gs, i, v, w, true, vn, act, pn);
        __syncthreads();
        // (4) w' = tau pn - tau/2 (x^H vn) vn; v <- vn
        cplx dpart = mk(0, 0);
        for (int r = tid; r < i; r += NT) {
            const cplx x = cmul(tau, pn[r]);
            pn[r] = x;
            cfmac(dpart, x, vn[r]);
        }
        const cplx xv = block_sum<NT>(dpart, red);
        const cplx al = cscale(cmul(tau, xv), -0.5);
        for (int r = tid; r < i; r += NT) {
            w[r] = act ? cadd(pn[r], cmul(al, vn[r])) : mk(0, 0);
            v[r] = vn[r];
        }
        __syncthreads();
    }
    // -- step 0's update reaches only A[0][0]
    if (tid == 0) {
        cplx x = resident ? *ss.at(0, 0) : *gs.at(0, 0);
        cplx u = cmul(v[0], cconj(w[0]));
        cfma(u, w[0], cconj(v[0]));
        dd[0] = x.x - u.x;
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

// Division-free Sturm count: the leading principal minors p_j of T - x I obey
//   p_j = (d_j - x) p_{j-1} - e_{j-1}^2 p_{j-2},   p_{-1} = 1,
// and the number of sign changes along p_{-1}, p_0, ..., p_{n-1} is the number of
// eigenvalues below x (Sturm).  The pair (p_j, p_{j-1}) is rescaled by exact powers of two
// to stay in range; a minor that is tiny relative to its predecessor is replaced by
// -pivmin * p_{j-1}, the same substitution the pivot form q_j = p_j / p_{j-1} uses
// (dstebz).  The derivatives p_j' ride along for the Newton step ratio = p_{n-1}/p_{n-1}'.
__device__ __forceinline__ int sturm_poly(const double* __restrict__ d, const double* __restrict__ e2, int n,
                                          double x, double pivmin, double& ratio) {
    double pm = 1.0, p = d[0] - x;       // p_{j-1}, p_j
    double dpm = 0.0, dp = -1.0;          // their derivatives in x
    if (fabs(p) <= pivmin) p = -pivmin;
    int cnt = p < 0.0;
    for (int j = 1; j < n; ++j) {
        const double a = d[j] - x;
        double pn = fma(a, p, -e2[j - 1] * pm);
        double dpn = fma(a, dp, -fma(e2[j - 1], dpm, p));
        if (fabs(pn) <= pivmin * fabs(p)) pn = -pivmin * p;
        cnt += (pn < 0.0) != (p < 0.0);
        pm = p;
        dpm = dp;
        p = pn;
        dp = dpn;
        const double big = fmax(fabs(p), fabs(pm));
        if (big > 0x1p+400 || big < 0x1p-400) {
            int ex;
            frexp(big, &ex);
            const double sc = ldexp(1.0, -ex);
            p *= sc;
            pm *= sc;
            dp *= sc;
            dpm *= sc;
        }
    }
    ratio = p / dp;
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

// Eigenvector of an isolated eigenvalue x of (d, e) by the twisted factorisation of
// T - x I (Parlett & Dhillon): forward pivots D+ (the Sturm recurrence) and backward
// pivots D-, twist index r minimising |gamma_r| = |D+_r + D-_r - (d_r - x)|, then
// z_r = 1, z_j = -e_j z_{j+1} / D+_j (j < r), z_j = -e_{j-1} z_{j-1} / D-_j (j > r).
// D+ and D- go to their own scratch columns so the final recurrences can prefetch them.
__device__ void twisted_vector(const double* __restrict__ d, const double* __restrict__ e,
                               const double* __restrict__ e2, int n, double x, double pivmin,
                               double* __restrict__ z, int k, double* __restrict__ dplus,
                               double* __restrict__ dminus, int sc) {
    double q = d[0] - x;
    if (fabs(q) <= pivmin) q = -pivmin;
    dplus[sc] = q;
    for (int j = 1; j < n; ++j) {
        q = d[j] - x - e2[j - 1] / q;
        if (fabs(q) <= pivmin) q = -pivmin;
        dplus[(size_t)j * TRI_THREADS + sc] = q;
    }
    double qb = d[n - 1] - x;
    if (fabs(qb) <= pivmin) qb = -pivmin;
    dminus[(size_t)(n - 1) * TRI_THREADS + sc] = qb;
    int r = n - 1;
    double gbest = fabs(q);   // gamma_{n-1} = D+_{n-1}
    for (int j = n - 2; j >= 0; --j) {
        const double aj = d[j] - x;
        double qn = aj - e2[j] / qb;
        if (fabs(qn) <= pivmin) qn = -pivmin;
        qb = qn;
        dminus[(size_t)j * TRI_THREADS + sc] = qb;
        const double gam = fabs(dplus[(size_t)j * TRI_THREADS + sc] + qb - aj);
        if (gam < gbest) {
            gbest = gam;
            r = j;
        }
    }
    double zz = 1.0, nrm2 = 1.0, big = 1.0;
    for (int j = r - 1; j >= 0; --j) {
        zz = -e[j] * zz / dplus[(size_t)j * TRI_THREADS + sc];
        z[(size_t)j * n + k] = zz;
        nrm2 += zz * zz;
        if (fabs(zz) > fabs(big)) big = zz;
    }
    z[(size_t)r * n + k] = 1.0;
    zz = 1.0;
    for (int j = r + 1; j < n; ++j) {
        zz = -e[j - 1] * zz / dminus[(size_t)j * TRI_THREADS + sc];
        z[(size_t)j * n + k] = zz;
        nrm2 += zz * zz;
        if (fabs(zz) > fabs(big)) big = zz;
    }
    double rn = 1.0 / sqrt(nrm2);
    if (big < 0.0) rn = -rn;
    for (int j = 0; j < n; ++j) z[(size_t)j * n + k] *= rn;
}

// PHASE 1 (k_stebz): eigenvalues into W.  PHASE 2 (k_stein): eigenvectors from W.
template <int PHASE>
__global__ void __launch_bounds__(TRI_THREADS, 2)
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
    // per-thread scratch columns (column = thread, stride TRI_THREADS): U diag / super1 /
    // super2, multipliers and swap flags of the LU of T - x I; the twisted solve uses the
    // first two as D+ and D-
    const size_t lus = (size_t)n * TRI_THREADS;
    double* la = LU + mat * 5 * lus;
    double* lb = la + lus;
    double* lc2 = lb + lus;
    double* lm = lc2 + lus;
    double* lp = lm + lus;

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
    if (!(onenrm > 1e3 * DBL_MIN)) {
        // T = 0 to underflow: eigenvalues are the diagonal (sorted), eigenvectors unit vectors
        if (PHASE == 2) return;
        if (tid == 0) {
            for (int k = 0; k < n; ++k) leader[k] = k;
            for (int k = 1; k < n; ++k)
                for (int q = k; q > 0 && d[leader[q]] < d[leader[q - 1]]; --q) {
                    const int tmp = leader[q];
                    leader[q] = leader[q - 1];
                    leader[q - 1] = tmp;
                }
        }
        __syncthreads();
        for (int k = tid; k < n; k += TRI_THREADS) {
            W[mat * n + k] = d[leader[k]];
            for (int j = 0; j < n; ++j) z[(size_t)j * n + k] = j == leader[k] ? 1.0 : 0.0;
        }
        if (tid == 0 && info) info[mat] = 0;
        return;
    }
    // ---- eigenvalue k: bisection on Sturm counts, accelerated by safeguarded Newton steps
    //      on det(T - x I) once the bracket holds k alone (dstebz bracketing, restated)
    if (PHASE == 1) {
    const double atol = 2.0 * DBL_EPSILON * onenrm;
    for (int k = tid; k < n; k += TRI_THREADS) {
        double lo = s_gl, hi = s_gu;
        int clo = 0, chi = n;
        double x = 0.5 * (lo + hi);
        double res = x;
        bool done = false;
        for (int it = 0; it < 200; ++it) {
            double ratio;
            const int c = sturm_poly(d, e2, n, x, pivmin, ratio);
            if (c > k) { hi = x; chi = c; } else { lo = x; clo = c; }
            const double tol = fmax(atol, 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)));
            if (hi - lo <= tol) { res = 0.5 * (lo + hi); done = true; break; }
            double xn = 0.5 * (lo + hi);
            if (chi - clo == 1 && (it % 4) != 3 && isfinite(ratio)) {
                const double nt = x - ratio;
                if (nt > lo && nt < hi) {
                    if (fabs(nt - x) <= tol) {
                        // converged step: accept only if Sturm counts bracket index k at nt +- 2 tol
                        const double a0 = fmax(lo, nt - 2.0 * tol), b0 = fmin(hi, nt + 2.0 * tol);
                        double rr;
                        const int ca = sturm_poly(d, e2, n, a0, pivmin, rr);
                        const int cb = sturm_poly(d, e2, n, b0, pivmin, rr);
                        if (ca <= k && cb > k) { res = nt; done = true; break; }
                        if (ca > k) { hi = a0; chi = ca; } else { lo = a0; clo = ca; }
                        if (cb > k) { hi = fmin(hi, b0); chi = cb; } else { lo = fmax(lo, b0); clo = cb; }
                        xn = 0.5 * (lo + hi);
                    } else {
                        xn = nt;
                    }
                }
            }
            if (xn <= lo || xn >= hi) { res = 0.5 * (lo + hi); done = true; break; }
            x = xn;
            res = x;
        }
        (void)done;
        W[mat * n + k] = res;
    }
    return;
    }
    for (int k = tid; k < n; k += TRI_THREADS) lam[k] = W[mat * n + k];
    __syncthreads();
    // ---- clusters (relative gap 1e-4 of the norm) and eigenvalue output
    const double ortol = 1e-4 * onenrm;
    if (tid == 0) {
        int lead = 0;
        for (int k = 0; k < n; ++k) {
            if (k > 0 && lam[k] - lam[k - 1] > ortol) lead = k;
            leader[k] = lead;
        }
    }
    __syncthreads();
    // ---- eigenvectors: isolated eigenvalues by one twisted solve; clusters by inverse
    //      iteration with modified Gram-Schmidt, handled by the leader's thread
    const double eps = DBL_EPSILON;
    const double dtpcrt = sqrt(0.1 / n);
    for (int k0 = tid; k0 < n; k0 += TRI_THREADS) {
        if (leader[k0] != k0) continue;
        int k1 = k0;
        while (k1 + 1 < n && leader[k1 + 1] == k0) ++k1;
        if (k1 == k0) {
            twisted_vector(d, e, e2, n, lam[k0], pivmin, z, k0, la, lb, tid);
            continue;
        }
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
            // the swap flag in lp, all at [j*TRI_THREADS + thread] (one column per thread).
            double u0 = d[0] - x, u1 = n > 1 ? e[0] : 0.0;
            for (int j = 0; j < n - 1; ++j) {
                const double cj = e[j];
                const double anext = d[j + 1] - x;
                const double bnext = j + 1 < n - 1 ? e[j + 1] : 0.0;
                const size_t o = (size_t)j * TRI_THREADS + tid;
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
            la[(size_t)(n - 1) * TRI_THREADS + tid] = u0;
            lb[(size_t)(n - 1) * TRI_THREADS + tid] = 0.0;
            lc2[(size_t)(n - 1) * TRI_THREADS + tid] = 0.0;
            // tiny pivots are perturbed to +-tolp in the solves (dlagts job = -1)
            double umax = 0.0;
            for (int j = 0; j < n; ++j) umax = fmax(umax, fabs(la[(size_t)j * TRI_THREADS + tid]));
            const double tolp = fmax(eps * fmax(umax, onenrm), DBL_MIN);
            for (int j = 0; j < n; ++j) z[(size_t)j * n + k] = start_entry(k, j);
            int nrmchk = 0;
            bool conv = false;
            for (int its = 0; its < INV_MAXITS; ++its) {
                // scale the right-hand side to ||b||_1 = n * onenrm * max(eps, |u_nn|)
                double b1 = 0.0;
                for (int j = 0; j < n; ++j) b1 += fabs(z[(size_t)j * n + k]);
                const double unn = fabs(la[(size_t)(n - 1) * TRI_THREADS + tid]);
                const double sc = n * onenrm * fmax(eps, unn) / fmax(b1, DBL_MIN);
                // forward: y = L^{-1} P b  (the active right-hand side value is carried)
                double rc = z[k] * sc;
                for (int j = 0; j < n - 1; ++j) {
                    const size_t o = (size_t)j * n + k;
                    const size_t ol = (size_t)j * TRI_THREADS + tid;
                    const double bnext = z[(size_t)(j + 1) * n + k] * sc;
                    const double mult = lm[ol];
                    if (lp[ol] != 0.0) {
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
                    const size_t ol = (size_t)j * TRI_THREADS + tid;
                    double u = la[ol];
                    if (fabs(u) < tolp) u = u >= 0.0 ? tolp : -tolp;
                    const double xj = (z[o] - lb[ol] * x1 - lc2[ol] * x2) / u;
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

// --------------------------------------------------------------- back-transformation
// X = Q Z with Q = H_{n-2} ... H_0 (H_i = I - tau_i v_i v_i^H, v_i on rows 0..i, v_i[i] = 1,
// v_i[0..i-1] stored in A[0..i-1][i+1]).  Reflectors are grouped in blocks of ORM_NB
// consecutive indices i0..i1; a block's product P = H_{i1} ... H_{i0} = I - V T V^H
// (compact WY form, T lower triangular, built by k_larft) is applied as
//   X <- X - V (T (V^H X)),
// blocks in increasing order (LAPACK zlarft / zlarfb, restated).
static constexpr int ORM_NB = 16;     // reflectors per block
static constexpr int ORM_RPT = 16;    // rows of the Z chunk held per thread
static constexpr int ORM_VS = ORM_NB + 1;   // padded shared-memory row stride of a V block

__device__ __forceinline__ cplx refl_entry(const cplx* __restrict__ a, int n, int i, int r) {
    // component r of reflector i (zero for i > n-2 padding)
    if (i > n - 2 || r > i) return mk(0, 0);
    if (r == i) return mk(1.0, 0.0);
    return a[(size_t)(i + 1) * n + r];
}

// T factors of every block of one matrix (one CTA per matrix):
//   T[k][k] = tau_k,  T[k][q] = -tau_k sum_{l=q}^{k-1} (v_k^H v_l) T[l][q]   (q < k)
__global__ void __launch_bounds__(256)
k_larft(const cplx* __restrict__ A, const cplx* __restrict__ TAU, cplx* __restrict__ Tw, int n) {
    __shared__ cplx G[ORM_NB][ORM_NB];
    __shared__ cplx T[ORM_NB][ORM_NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t mat = blockIdx.x;
    const cplx* a = A + mat * (size_t)n * n;
    const cplx* tau = TAU + mat * n;
    const int nblk = (n - 1 + ORM_NB - 1) / ORM_NB;
    for (int j = 0; j < nblk; ++j) {
        const int i0 = j * ORM_NB;
        // G[k][l] = v_k^H v_l for l < k: rows 0..i0+l overlap
        for (int pr = warp; pr < ORM_NB * ORM_NB; pr += 8) {
            const int k = pr / ORM_NB, l = pr % ORM_NB;
            if (l >= k) continue;
            const int ik = i0 + k, il = i0 + l;
            cplx s = mk(0, 0);
            if (ik <= n - 2) {
                for (int r = lane; r <= il; r += 32) cfmac(s, refl_entry(a, n, ik, r), refl_entry(a, n, il, r));
            }
            s = warp_sum(s);
            if (lane == 0) G[k][l] = s;
        }
        __syncthreads();
        if (warp == 0) {
            for (int k = 0; k < ORM_NB; ++k) {
                const int ik = i0 + k;
                const cplx tk = ik <= n - 2 ? tau[ik] : mk(0, 0);
                if (lane < ORM_NB) {
                    cplx val = mk(0, 0);
                    if (lane == k) {
                        val = tk;
                    } else if (lane < k) {
                        cplx s = mk(0, 0);
                        for (int l = lane; l < k; ++l) cfma(s, G[k][l], T[l][lane]);
                        val = cscale(cmul(tk, s), -1.0);
                    }
                    T[k][lane] = val;
                }
                __syncwarp();
            }
        }
        __syncthreads();
        cplx* out = Tw + (mat * nblk + j) * ORM_NB * ORM_NB;
        out[threadIdx.x] = T[threadIdx.x / ORM_NB][threadIdx.x % ORM_NB];
        __syncthreads();
    }
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Stage block j of V (rows 0..i1, layout [r][k]) and its T factor into shared memory:
// stored reflector entries by cp.async, the implicit 1 and the zeros below by plain stores.
__device__ __forceinline__ void stage_block(const cplx* __restrict__ a, const cplx* __restrict__ tsrc,
                                            cplx* vsb, cplx* tsb, int n, int j) {
    const int t = threadIdx.x;
    const int i0 = j * ORM_NB;
    const int i1 = min(i0 + ORM_NB - 1, n - 2);
    for (int idx = t; idx < (i1 + 1) * ORM_NB; idx += 256) {
        const int r = idx / ORM_NB, k = idx % ORM_NB;
        const int i = i0 + k;
        cplx* dst = &vsb[r * ORM_VS + k];
        if (i <= n - 2 && r < i) cp_async16(dst, &a[(size_t)(i + 1) * n + r]);
        else *dst = (i <= n - 2 && r == i) ? mk(1.0, 0.0) : mk(0, 0);
    }
    cp_async16(&tsb[t], &tsrc[t]);
    cp_async_commit();
}

// Apply all blocks to a chunk of CH columns of Z (row-major Z[r*n + col], real) and write
// the chunk of X (column-major, column = eigenvector).  Thread t owns column t % CH and the
// rows g + RG*q (g = t / CH, RG = 256/CH, q < ORM_RPT) in registers.  With dbuf the next
// block's V and T are copied asynchronously while the current block is applied.
template <int CH>
__global__ void __launch_bounds__(256)
k_ormtr(const cplx* __restrict__ A, const cplx* __restrict__ Tw, const double* __restrict__ Z,
        cplx* __restrict__ X, int n, int dbuf) {
    constexpr int RG = 256 / CH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* vsbuf[2];
    vsbuf[0] = reinterpret_cast<cplx*>(smem_raw);                    // [n][ORM_VS]
    vsbuf[1] = dbuf ? vsbuf[0] + (size_t)n * ORM_VS : vsbuf[0];
    cplx* tsbuf[2];
    tsbuf[0] = vsbuf[0] + (size_t)(dbuf ? 2 : 1) * n * ORM_VS;       // [ORM_NB][ORM_NB]
    tsbuf[1] = dbuf ? tsbuf[0] + ORM_NB * ORM_NB : tsbuf[0];
    cplx* wsum = tsbuf[0] + (size_t)(dbuf ? 2 : 1) * ORM_NB * ORM_NB;   // [8][ORM_NB][CH]
    cplx* w2 = wsum + 8 * ORM_NB * CH;                                // [ORM_NB][CH]
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int c = t % CH, g = t / CH;
    const size_t mat = blockIdx.y;
    const int col = blockIdx.x * CH + c;
    const cplx* a = A + mat * (size_t)n * n;
    const double* z = Z + mat * (size_t)n * n;
    const int nblk = (n - 1 + ORM_NB - 1) / ORM_NB;
    const cplx* tw = Tw + mat * (size_t)nblk * ORM_NB * ORM_NB;
    cplx x[ORM_RPT];
#pragma unroll
    for (int q = 0; q < ORM_RPT; ++q) {
        const int r = g + RG * q;
        x[q] = (r < n && col < n) ? mk(z[(size_t)r * n + col], 0.0) : mk(0, 0);
    }
    if (dbuf && nblk > 0) stage_block(a, tw, vsbuf[0], tsbuf[0], n, 0);
    for (int j = 0; j < nblk; ++j) {
        const int i0 = j * ORM_NB;
        const int i1 = min(i0 + ORM_NB - 1, n - 2);
        if (dbuf) {
            if (j + 1 < nblk) {
                stage_block(a, tw + (size_t)(j + 1) * ORM_NB * ORM_NB, vsbuf[(j + 1) & 1],
                            tsbuf[(j + 1) & 1], n, j + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
        } else {
            stage_block(a, tw + (size_t)j * ORM_NB * ORM_NB, vsbuf[0], tsbuf[0], n, j);
            cp_async_wait<0>();
        }
        __syncthreads();
        const cplx* vs = vsbuf[j & 1];
        const cplx* ts = tsbuf[j & 1];
        // partial W = V^H X over this thread's rows
        cplx wp[ORM_NB];
#pragma unroll
        for (int k = 0; k < ORM_NB; ++k) wp[k] = mk(0, 0);
#pragma unroll
        for (int q = 0; q < ORM_RPT; ++q) {
            const int r = g + RG * q;
            if (r <= i1) {
                const cplx* vr = vs + r * ORM_VS;
#pragma unroll
                for (int k = 0; k < ORM_NB; ++k) cfmac(wp[k], vr[k], x[q]);
            }
        }
        // reduce over the row groups: inside the warp, then across the 8 warps
#pragma unroll
        for (int s2 = CH; s2 < 32; s2 <<= 1)
#pragma unroll
            for (int k = 0; k < ORM_NB; ++k) wp[k] = cadd(wp[k], shfl_xor(wp[k], s2));
        if (lane < CH)
#pragma unroll
            for (int k = 0; k < ORM_NB; ++k) wsum[(warp * ORM_NB + k) * CH + lane] = wp[k];
        __syncthreads();
        cplx wk = mk(0, 0);
        if (t < ORM_NB * CH) {
            for (int w8 = 0; w8 < 8; ++w8) wk = cadd(wk, wsum[w8 * ORM_NB * CH + t]);
            wsum[t] = wk;   // W[k][c] at t = k*CH + c (slot of warp 0, already read)
        }
        __syncthreads();
        if (t < ORM_NB * CH) {
            const int k = t / CH, cc = t % CH;
            cplx s = mk(0, 0);
            for (int q2 = 0; q2 <= k; ++q2) cfma(s, ts[k * ORM_NB + q2], wsum[q2 * CH + cc]);
            w2[t] = s;
        }
        __syncthreads();
        // X -= V W2 on rows <= i1
        cplx wc[ORM_NB];
#pragma unroll
        for (int k = 0; k < ORM_NB; ++k) wc[k] = w2[k * CH + c];
#pragma unroll
        for (int q = 0; q < ORM_RPT; ++q) {
            const int r = g + RG * q;
            if (r <= i1) {
                const cplx* vr = vs + r * ORM_VS;
                cplx s = mk(0, 0);
#pragma unroll
                for (int k = 0; k < ORM_NB; ++k) cfma(s, vr[k], wc[k]);
                x[q] = csub(x[q], s);
            }
        }
        __syncthreads();
    }
    // write the chunk column-major through shared memory (coalesced along rows)
    cplx* xs = vsbuf[0];   // [CH][n]
#pragma unroll
    for (int q = 0; q < ORM_RPT; ++q) {
        const int r = g + RG * q;
        if (r < n) xs[(size_t)c * n + r] = x[q];
    }
    __syncthreads();
    cplx* xo = X + mat * (size_t)n * n;
    const int col0 = blockIdx.x * CH;
    for (int idx = t; idx < CH * n; idx += 256) {
        const int cc = idx / n, r = idx % n;
        if (col0 + cc < n) xo[(size_t)(col0 + cc) * n + r] = xs[idx];
    }
}

// ------------------------------------------------ back-transformation for large orders
// For orders whose 16-reflector blocks do not fit the register/shared-memory scheme of
// k_ormtr, X = Q Z is applied with blocks of BT_NB = 64 reflectors as two tiled complex
// GEMMs per block (LAPACK zlarfb restated): W' = T (V^H X), then X -= V W'.  X lives in
// global memory (column-major, column = eigenvector) and is read twice and written once
// per block.
static constexpr int BT_NB = 64;

// T factor of block j (reflectors 64j .. 64j+63) of one matrix; grid (blocks, matrices).
__global__ void __launch_bounds__(256)
k_larft64(const cplx* __restrict__ A, const cplx* __restrict__ TAU, cplx* __restrict__ Tw, int n) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* G = reinterpret_cast<cplx*>(smem_raw);   // [64][64]
    cplx* T = G + BT_NB * BT_NB;                   // [64][64]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = blockIdx.x;
    const size_t mat = blockIdx.y;
    const cplx* a = A + mat * (size_t)n * n;
    const cplx* tau = TAU + mat * n;
    const int nblk = (n - 1 + BT_NB - 1) / BT_NB;
    const int i0 = j * BT_NB;
    for (int pr = warp; pr < BT_NB * BT_NB; pr += 8) {
        const int k = pr / BT_NB, l = pr % BT_NB;
        if (l >= k) continue;
        const int ik = i0 + k, il = i0 + l;
        cplx s = mk(0, 0);
        if (ik <= n - 2)
            for (int r = lane; r <= il; r += 32) cfmac(s, refl_entry(a, n, ik, r), refl_entry(a, n, il, r));
        s = warp_sum(s);
        if (lane == 0) G[k * BT_NB + l] = s;
    }
    __syncthreads();
    for (int k = 0; k < BT_NB; ++k) {
        const int ik = i0 + k;
        const cplx tk = ik <= n - 2 ? tau[ik] : mk(0, 0);
        if (threadIdx.x < BT_NB) {
            const int q = threadIdx.x;
            cplx val = mk(0, 0);
            if (q == k) {
                val = tk;
            } else if (q < k) {
                cplx s = mk(0, 0);
                for (int l = q; l < k; ++l) cfma(s, G[k * BT_NB + l], T[l * BT_NB + q]);
                val = cscale(cmul(tk, s), -1.0);
            }
            T[k * BT_NB + q] = val;
        }
        __syncthreads();
    }
    cplx* out = Tw + (mat * nblk + j) * BT_NB * BT_NB;
    for (int i = threadIdx.x; i < BT_NB * BT_NB; i += 256) out[i] = T[i];
}

// Z (row-major real) -> X (column-major complex), grid-stride over all batch entries.
__global__ void k_z_to_x(const double* __restrict__ Z, cplx* __restrict__ X, int n, size_t total) {
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const size_t nn = (size_t)n * n;
        const size_t mat = idx / nn, rem = idx % nn;
        const int c = (int)(rem / n), r = (int)(rem % n);
        X[idx] = mk(Z[mat * nn + (size_t)r * n + c], 0.0);
    }
}

// W' = T (V^H X) for block j and 32 columns of X: grid (ceil(n/32), matrices).
// Thread t owns W rows k0, k0+1 (k0 = 2*(t/8)) and columns c0..c0+3 (c0 = 4*(t%8)).
__global__ void __launch_bounds__(256)
k_bt_w(const cplx* __restrict__ A, const cplx* __restrict__ Tw, const cplx* __restrict__ X,
       cplx* __restrict__ Wp, int n, int j) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    typedef cplx VRow[BT_NB + 1];
    typedef cplx CRow[33];
    VRow* Vs = reinterpret_cast<VRow*>(smem_raw);          // [32][65]
    CRow* Xs = reinterpret_cast<CRow*>(Vs + 32);           // [32][33]
    CRow* Ws = Xs + 32;                                    // [64][33]
    const int t = threadIdx.x;
    const int k0 = 2 * (t / 8), c0 = 4 * (t % 8);
    const size_t mat = blockIdx.y;
    const int col0 = blockIdx.x * 32;
    const cplx* a = A + mat * (size_t)n * n;
    const cplx* x = X + mat * (size_t)n * n;
    const int i0 = j * BT_NB, i1 = min(i0 + BT_NB - 1, n - 2);
    cplx acc[2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = mk(0, 0);
    for (int r0 = 0; r0 <= i1; r0 += 32) {
        __syncthreads();
        for (int idx = t; idx < 32 * BT_NB; idx += 256) {
            const int rr = idx / BT_NB, k = idx % BT_NB;
            Vs[rr][k] = r0 + rr <= i1 ? refl_entry(a, n, i0 + k, r0 + rr) : mk(0, 0);
        }
        for (int idx = t; idx < 32 * 32; idx += 256) {
            const int cc = idx / 32, rr = idx % 32;   // coalesced along rows of column col0+cc
            Xs[rr][cc] = (r0 + rr <= i1 && col0 + cc < n) ? x[(size_t)(col0 + cc) * n + r0 + rr] : mk(0, 0);
        }
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < 32; ++rr) {
            const cplx va = Vs[rr][k0], vb = Vs[rr][k0 + 1];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const cplx xv = Xs[rr][c0 + v];
                cfmac(acc[0][v], va, xv);
                cfmac(acc[1][v], vb, xv);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) Ws[k0 + u][c0 + v] = acc[u][v];
    __syncthreads();
    const int nblk = (n - 1 + BT_NB - 1) / BT_NB;
    const cplx* T = Tw + (mat * nblk + j) * BT_NB * BT_NB;
    cplx* wp = Wp + mat * (size_t)BT_NB * n;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int k = k0 + u;
        cplx s[4] = {mk(0, 0), mk(0, 0), mk(0, 0), mk(0, 0)};
        for (int q = 0; q <= k; ++q) {
            const cplx tq = T[k * BT_NB + q];
#pragma unroll
            for (int v = 0; v < 4; ++v) cfma(s[v], tq, Ws[q][c0 + v]);
        }
#pragma unroll
        for (int v = 0; v < 4; ++v)
            if (col0 + c0 + v < n) wp[(size_t)k * n + col0 + c0 + v] = s[v];
    }
}

// X[0..i1][cols] -= V W' for block j: grid (row tiles of 64, column tiles of 32, matrices).
// Thread t owns rows r0+2*(t/8)+{0,1} and columns c0..c0+3.
__global__ void __launch_bounds__(256)
k_bt_upd(const cplx* __restrict__ A, const cplx* __restrict__ Wp, cplx* __restrict__ X, int n, int j) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    typedef cplx VRow[BT_NB + 1];
    typedef cplx CRow[33];
    VRow* Vs = reinterpret_cast<VRow*>(smem_raw);          // [64][65]
    CRow* Ws = reinterpret_cast<CRow*>(Vs + 64);           // [64][33]
    const int t = threadIdx.x;
    const size_t mat = blockIdx.z;
    const int row0 = blockIdx.x * 64, col0 = blockIdx.y * 32;
    const int i0 = j * BT_NB, i1 = min(i0 + BT_NB - 1, n - 2);
    if (row0 > i1) return;
    const cplx* a = A + mat * (size_t)n * n;
    const cplx* wp = Wp + mat * (size_t)BT_NB * n;
    for (int idx = t; idx < 64 * BT_NB; idx += 256) {
        const int rr = idx / BT_NB, k = idx % BT_NB;
        Vs[rr][k] = row0 + rr <= i1 ? refl_entry(a, n, i0 + k, row0 + rr) : mk(0, 0);
    }
    for (int idx = t; idx < BT_NB * 32; idx += 256) {
        const int k = idx / 32, cc = idx % 32;
        Ws[k][cc] = col0 + cc < n ? wp[(size_t)k * n + col0 + cc] : mk(0, 0);
    }
    __syncthreads();
    const int rl = 2 * (t / 8), c0 = 4 * (t % 8);
    cplx s[2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) s[u][v] = mk(0, 0);
#pragma unroll 4
    for (int k = 0; k < BT_NB; ++k) {
        const cplx va = Vs[rl][k], vb = Vs[rl + 1][k];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const cplx w = Ws[k][c0 + v];
            cfma(s[0][v], va, w);
            cfma(s[1][v], vb, w);
        }
    }
    cplx* x = X + mat * (size_t)n * n;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int r = row0 + rl + u;
        if (r > i1) continue;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int c = col0 + c0 + v;
            if (c < n) {
                cplx* p = &x[(size_t)c * n + r];
                *p = csub(*p, s[u][v]);
            }
        }
    }
}

// Launch shape of k_hetrd: small matrices keep their whole triangle in shared memory with
// 128 threads and several CTAs per SM; larger ones run 512 threads, one CTA per SM, with
// as much of the leading triangle resident as ~220 KB allows.
struct HetrdCfg {
    int nt;
    int tri_cap;
    size_t smem;
};
static HetrdCfg hetrd_config(int n) {
    const size_t tri_full = (size_t)n * (n + 1) / 2;
    const size_t vec128 = 4 * (size_t)n * sizeof(cplx) + 2 * (128 / 32) * sizeof(double);
    if (vec128 + tri_full * sizeof(cplx) <= 76 * 1024)
        return {128, (int)tri_full, vec128 + tri_full * sizeof(cplx)};
    const size_t vec512 = 4 * (size_t)n * sizeof(cplx) + 2 * (512 / 32) * sizeof(double);
    const size_t budget = 220 * 1024;
    size_t cap = budget > vec512 ? (budget - vec512) / sizeof(cplx) : 0;
    cap = std::min(cap, tri_full);
    return {512, (int)cap, vec512 + cap * sizeof(cplx)};
}
static cudaError_t launch_hetrd(const HetrdCfg& c, cudaStream_t st, int nb, cplx* A, double* D, double* E,
                                cplx* TAU, int n) {
    if (c.smem > 227 * 1024) return cudaErrorInvalidValue;
    if (c.nt == 128) {
        cudaError_t e = cudaFuncSetAttribute(k_hetrd<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
        if (e != cudaSuccess) return e;
        k_hetrd<128><<<nb, 128, c.smem, st>>>(A, D, E, TAU, n, c.tri_cap);
    } else {
        cudaError_t e = cudaFuncSetAttribute(k_hetrd<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
        if (e != cudaSuccess) return e;
        k_hetrd<512><<<nb, 512, c.smem, st>>>(A, D, E, TAU, n, c.tri_cap);
    }
    return cudaGetLastError();
}

// Shape of one eigensolve chunk: kernel configurations and the scratch layout per matrix.
struct HeevPlan {
    int n;
    HetrdCfg hc;
    size_t smem_tri;
    bool small_bt;       // k_ormtr (register-resident Z chunk) or the large-order GEMM path
    int ch, dbuf;
    size_t smem_orm;
    int nblk16, nblk64;
    // per-matrix scratch, in doubles
    size_t off_d, off_e, off_tau, off_z, off_lu, off_x, off_t, off_w, per;
};

static HeevPlan heev_plan(int n) {
    HeevPlan p{};
    p.n = n;
    p.hc = hetrd_config(n);
    p.smem_tri = 4 * (size_t)n * sizeof(double) + n * sizeof(int);
    p.nblk16 = (n - 1 + ORM_NB - 1) / ORM_NB;
    p.nblk64 = (n - 1 + BT_NB - 1) / BT_NB;
    int ch = 16;
    while (ch > 1 && (n + 256 / ch - 1) / (256 / ch) > ORM_RPT) ch >>= 1;
    p.ch = ch;
    size_t smem = ((size_t)2 * n * ORM_VS + 2 * ORM_NB * ORM_NB + 8 * ORM_NB * ch + ORM_NB * ch) * sizeof(cplx);
    p.dbuf = smem <= 220 * 1024 ? 1 : 0;
    if (!p.dbuf)
        smem = ((size_t)std::max(n * ORM_VS, n * ch) + ORM_NB * ORM_NB + 8 * ORM_NB * ch + ORM_NB * ch) * sizeof(cplx);
    p.smem_orm = smem;
    p.small_bt = (n + 256 / ch - 1) / (256 / ch) <= ORM_RPT && smem <= 220 * 1024;
    // every region is a multiple of 32 doubles per matrix, so that each region of a chunk
    // starts 256-byte aligned whatever the chunk size (complex and cp.async accesses)
    const size_t nn = (size_t)n * n;
    auto r32 = [](size_t v) { return (v + 31) / 32 * 32; };
    size_t off = 0;
    p.off_d = off; off += r32(n);
    p.off_e = off; off += r32(n);
    p.off_tau = off; off += r32(2 * (size_t)n);
    p.off_z = off; off += r32(nn);
    p.off_lu = off; off += r32(5 * (size_t)n * TRI_THREADS);
    p.off_x = off; off += r32(2 * nn);
    p.off_t = off; off += r32(2 * (size_t)(p.small_bt ? p.nblk16 * ORM_NB * ORM_NB : p.nblk64 * BT_NB * BT_NB));
    p.off_w = off; off += p.small_bt ? 0 : r32(2 * (size_t)BT_NB * n);
    p.per = off;
    return p;
}

// Bytes of scratch one matrix of order n needs in heev_chunk_on_scratch.
size_t heev_scratch_bytes_per_matrix(int n) { return heev_plan(n).per * sizeof(double); }

#define RLMB_CHUNK_LAUNCHED()                                     \
    do {                                                          \
        if (ctx) {                                                \
            prof_end(ctx);                                        \
            ctx->launches++;                                      \
        } else {                                                  \
            ++*launches;                                          \
        }                                                         \
        if (cudaGetLastError() != cudaSuccess) return RLMB_ERR_CUDA; \
    } while (0)
#define RLMB_CHUNK_PROF(name) \
    do {                      \
        if (ctx) prof_begin(ctx, name); \
    } while (0)

// The kernel sequence of one eigensolve chunk of nb matrices of order n on scratch laid out
// per matrix as heev_plan describes (nb * heev_scratch_bytes_per_matrix(n) bytes, no
// allocation).  Every scratch region is written by a kernel before any kernel reads it.
// ctx (optional) receives the launch count and profile; otherwise *launches is advanced.
static int heev_chunk(rlmb_context* ctx, cudaStream_t st, cplx* A, double* W, int* info, int n, int nb,
                      void* scratch, long long* launches) {
    const HeevPlan p = heev_plan(n);
    double* base = static_cast<double*>(scratch);
    const size_t B = (size_t)nb;
    double* Dw = base + p.off_d * B;
    double* Ew = base + p.off_e * B;
    cplx* TAUw = reinterpret_cast<cplx*>(base + p.off_tau * B);
    double* Zw = base + p.off_z * B;
    double* LUw = base + p.off_lu * B;
    cplx* Xw = reinterpret_cast<cplx*>(base + p.off_x * B);
    cplx* Tw = reinterpret_cast<cplx*>(base + p.off_t * B);
    cplx* Wp = reinterpret_cast<cplx*>(base + p.off_w * B);
    const size_t nn = (size_t)n * n;
    if (p.hc.smem > 227 * 1024 || p.smem_tri > 227 * 1024) return RLMB_ERR_ARG;
    if (cudaFuncSetAttribute(k_tridiag<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_tri) != cudaSuccess ||
        cudaFuncSetAttribute(k_tridiag<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_tri) != cudaSuccess)
        return RLMB_ERR_CUDA;
    RLMB_CHUNK_PROF("k_hetrd");
    if (launch_hetrd(p.hc, st, nb, A, Dw, Ew, TAUw, n) != cudaSuccess) return RLMB_ERR_CUDA;
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_stebz");
    k_tridiag<1><<<nb, TRI_THREADS, p.smem_tri, st>>>(Dw, Ew, W, Zw, LUw, info, n);
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_stein");
    k_tridiag<2><<<nb, TRI_THREADS, p.smem_tri, st>>>(Dw, Ew, W, Zw, LUw, info, n);
    RLMB_CHUNK_LAUNCHED();
    if (p.small_bt) {
        auto ormtr = p.ch == 16 ? k_ormtr<16> : p.ch == 8 ? k_ormtr<8> : p.ch == 4 ? k_ormtr<4>
                   : p.ch == 2 ? k_ormtr<2> : k_ormtr<1>;
        if (cudaFuncSetAttribute(ormtr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_orm) != cudaSuccess)
            return RLMB_ERR_CUDA;
        if (n > 1) {
            RLMB_CHUNK_PROF("k_larft");
            k_larft<<<nb, 256, 0, st>>>(A, TAUw, Tw, n);
            RLMB_CHUNK_LAUNCHED();
        }
        RLMB_CHUNK_PROF("k_ormtr");
        ormtr<<<dim3((n + p.ch - 1) / p.ch, nb), 256, p.smem_orm, st>>>(A, Tw, Zw, Xw, n, p.dbuf);
        RLMB_CHUNK_LAUNCHED();
    } else {
        const size_t smem_t = 2 * BT_NB * BT_NB * sizeof(cplx);
        const size_t smem_w = (32 * (BT_NB + 1) + 32 * 33 + BT_NB * 33) * sizeof(cplx);
        const size_t smem_u = (64 * (BT_NB + 1) + BT_NB * 33) * sizeof(cplx);
        if (cudaFuncSetAttribute(k_larft64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t) != cudaSuccess ||
            cudaFuncSetAttribute(k_bt_w, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_w) != cudaSuccess ||
            cudaFuncSetAttribute(k_bt_upd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_u) != cudaSuccess)
            return RLMB_ERR_CUDA;
        RLMB_CHUNK_PROF("k_larft");
        k_larft64<<<dim3(p.nblk64, nb), 256, smem_t, st>>>(A, TAUw, Tw, n);
        RLMB_CHUNK_LAUNCHED();
        RLMB_CHUNK_PROF("k_ormtr");
        k_z_to_x<<<2048, 256, 0, st>>>(Zw, Xw, n, B * nn);
        RLMB_CHUNK_LAUNCHED();
        for (int j = 0; j < p.nblk64; ++j) {
            const int i1 = std::min(j * BT_NB + BT_NB - 1, n - 2);
            RLMB_CHUNK_PROF("k_ormtr");
            k_bt_w<<<dim3((n + 31) / 32, nb), 256, smem_w, st>>>(A, Tw, Xw, Wp, n, j);
            RLMB_CHUNK_LAUNCHED();
            RLMB_CHUNK_PROF("k_ormtr");
            k_bt_upd<<<dim3(i1 / 64 + 1, (n + 31) / 32, nb), 256, smem_u, st>>>(A, Wp, Xw, n, j);
            RLMB_CHUNK_LAUNCHED();
        }
    }
    if (cudaMemcpyAsync(A, Xw, B * nn * sizeof(cplx), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return RLMB_ERR_CUDA;
    return RLMB_OK;
}
#undef RLMB_CHUNK_LAUNCHED
#undef RLMB_CHUNK_PROF

int heev_chunk_on_scratch(cudaStream_t st, cplx* A, double* W, int* info, int n, int nb, void* scratch,
                          long long* launches) {
    return heev_chunk(nullptr, st, A, W, info, n, nb, scratch, launches);
}

}  // namespace rlmb

using namespace rlmb;

extern "C" int rlmb_heevd_batched(rlmb_context* ctx, double* d_a, double* d_w, int n, int batch,
                                  int* d_info) {
    if (!ctx || !d_a || !d_w || n <= 0 || batch < 0) return RLMB_ERR_ARG;
    if (batch == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t per = heev_scratch_bytes_per_matrix(n);
    // workspace: 8 GB, or for large orders enough for two resident matrices per SM (one
    // CTA each in k_tridiag), capped at 60 % of the free memory
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = (size_t)8 << 30;
    }
    size_t budget = std::max<size_t>((size_t)8 << 30, 2 * 148 * per);
    budget = std::min<size_t>(budget, free_b / 10 * 6 + ctx->ws_bytes);
    budget = std::max<size_t>(budget, per);
    size_t chunk = std::max<size_t>(1, std::min<size_t>(budget / per, (size_t)batch));
    if (int rc = ensure_workspace(ctx, chunk * per)) return rc;
    const size_t nn = (size_t)n * n;
    long long unused = 0;
    for (size_t b0 = 0; b0 < (size_t)batch; b0 += chunk) {
        const int nb = (int)std::min(chunk, (size_t)batch - b0);
        if (int rc = heev_chunk(ctx, ctx->stream, reinterpret_cast<cplx*>(d_a) + b0 * nn, d_w + b0 * n,
                                d_info ? d_info + b0 : nullptr, n, nb, ctx->ws, &unused))
            return rc;
    }
    return RLMB_OK;
}
