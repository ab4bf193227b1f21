// Batched complex Hermitian eigensolver (sm_100a), double precision or mixed precision.
//
// Replaces the reference's dense solver calls: mkl_heevd (diag_wrappers/mkl_diag.cpp:2-9,
// LAPACKE_zheevd col-major 'U'), cusolver_diag_hamil (diag_wrappers/cusolver_diag.cu:3-22)
// and magma_diag_hamil (diag_wrappers/magma_diag.cu:2-49).  The LAPACK arithmetic those
// calls reach is restated from its published algorithms:
//
//   reduction      A = Q T Q^H (zhetrd, uplo='U').  From order 256: panels of 16 columns
//                  (32 from order 1024 in double precision; k_hetrd_panel, zlatrd restated)
//                  whose rank-32 (rank-64) updates run as batched GEMMs over all SMs
//                  (launch_zgemm); the last leading
//                  block (order <= 64, or all of a smaller matrix) by the unblocked,
//                  look-ahead k_hetrd (zhetd2), its triangle resident in shared memory.
//   tridiagonal    below order 600 k_tridiag: eigenvalues by Sturm counts (dstebz restated,
//                  seeded from a shared grid, Newton-accelerated); eigenvectors by twisted
//                  factorisation, or for clusters inverse iteration / twisted solves with
//                  modified Gram-Schmidt (dstein restated).  From order 600 divide and
//                  conquer (tridiag_dc.cuh: secular equations, Gu-Eisenstat vectors, DMMA
//                  merges).  Either one may be pinned or autotuned per order.
//   back-transform X = Q Z (zunmtr): k_larft + k_ormtr (register-resident Z chunks, blocks
//                  of 16 reflectors) below order 256, else T factors from batched Gram
//                  GEMMs and three GEMM launches per block of 64 reflectors.
//   mixed mode     the reduction and back-transformation in single precision, then double
//                  refinement of every eigenpair (k_ref_*, Ogita-Aishima restated, with
//                  cluster Rayleigh-Ritz).
//   small orders   up to order 20 (autotuned up to 80) the whole eigensolve is batched
//                  two-sided Jacobi instead (jacobi.cuh).
//
// Waits are __syncthreads inside one CTA, except the panel queue's per-column counts
// (k_hetrd_panel_q), whose spins are bounded in time and abort the chunk when they run out.
#include "common.cuh"
#include "jacobi.cuh"
#include "tridiag_dc.cuh"
#include "small_eig.cuh"
#include "zgemm.cuh"
#include "zgemm_tc.cuh"
#include "zgemm_tma.cuh"

#include <cfloat>
#include <map>
#include <vector>
#include <cmath>

namespace rlmb {


// --------------------------------------------------------------- block reductions
template <int NT, class R>
__device__ __forceinline__ R block_sum(R v, R* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    R s = 0;
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) s += red[i];
    return s;
}
template <int NT, class C, class R>
__device__ __forceinline__ C block_sum_c(C v, R* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        red[2 * w] = v.x;
        red[2 * w + 1] = v.y;
    }
    __syncthreads();
    C s = cz<C>();
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) {
        s.x += red[2 * i];
        s.y += red[2 * i + 1];
    }
    return s;
}

// Transpose-reduce for a 16-column group: lane l holds v[j] (the contribution of row l
// to column j); on return lane l (and l^16) holds the sum over all 32 lanes of v[l & 15].
template <class C>
__device__ __forceinline__ C transpose_reduce16(C (&v)[16]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = cadd(v[j], shfl_xor(v[j], 16));
#pragma unroll
    for (int s = 8; s >= 1; s >>= 1) {
        const bool up = (lane & s) != 0;
#pragma unroll
        for (int j = 0; j < s; ++j) {
            C send = up ? v[j] : v[j + s];
            C keep = up ? v[j + s] : v[j];
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

template <class C>
__device__ __forceinline__ void smem_atomic_add(C* p, C v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}

// ------------------------------------------------------------------ k_hetrd
// Storage of the active leading block: global column-major (ld = n) while it is large,
// packed upper triangle in shared memory (column c at c(c+1)/2) once it fits.
template <class C>
struct GlobalStore {
    C* a;
    int n;
    __device__ __forceinline__ C* at(int r, int c) const { return a + (size_t)c * n + r; }
};
template <class C>
struct SharedStore {
    C* s;
    __device__ __forceinline__ C* at(int r, int c) const { return s + (c * (c + 1) / 2 + r); }
};

// One pass over the upper triangle of the leading m x m block, 32x32 tiles dealt to
// warps: applies the rank-2 update A -= v w^H + w v^H of the previous reflector (if upd)
// and accumulates pn += A' vn for the next one (if acc), reading and writing every
// stored element once.  All loads of a 16-column half tile are issued before its stores.
template <int NT, class C, class S>
__device__ __forceinline__ void fused_pass(S st, int m, const C* __restrict__ v,
                                           const C* __restrict__ w, bool upd,
                                           const C* __restrict__ vn, bool acc, C* pn) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    const int nb = (m + 31) / 32;
    const int nitems = nb * (nb + 1);   // two 16-column halves per 32x32 tile
    for (int it = warp; it < nitems; it += NW) {
        int R, Cb;
        tile_of(it >> 1, R, Cb);
        const int c0 = Cb * 32 + 16 * (it & 1);
        if (c0 >= m) continue;
        const int r = R * 32 + lane;
        const bool rin = r < m;
        const C vr = rin ? v[r] : cz<C>();
        const C wr = rin ? w[r] : cz<C>();
        const C vnr = rin ? vn[r] : cz<C>();
        C rowacc = cz<C>();
        C e[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int cc = c0 + j;
            e[j] = (rin && cc < m && r <= cc) ? *st.at(r, cc) : cz<C>();
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int cc = c0 + j;
            const bool valid = rin && cc < m && r <= cc;
            C x = e[j];
            if (upd) {
                const C vc = cc < m ? v[cc] : cz<C>();
                const C wc = cc < m ? w[cc] : cz<C>();
                C u = cmul(vr, cconj(wc));
                cfma(u, wr, cconj(vc));
                x = csub(x, u);
                if (r == cc) x.y = 0;
                if (valid) *st.at(r, cc) = x;
            }
            if (acc) {
                const C vnc = cc < m ? vn[cc] : cz<C>();
                if (!valid) {
                    e[j] = cz<C>();
                } else if (r == cc) {
                    rowacc = cadd(rowacc, cscale(vnc, x.x));
                    e[j] = cz<C>();
                } else {
                    cfma(rowacc, x, vnc);
                    e[j] = cmulc(x, vnr);   // column partial: conj(A'[r][cc]) vn[r]
                }
            }
        }
        if (acc) {
            const C cs = transpose_reduce16(e);
            const int cl = c0 + (lane & 15);
            if (lane < 16 && cl < m) smem_atomic_add(&pn[cl], cs);
            if (rin) smem_atomic_add(&pn[r], rowacc);
        }
    }
}

// Householder reflector of zlarfg for (alpha, x) with ||x||^2 = xnorm2: returns beta, tau
// and the scale applied to x.
template <class C, class R>
__device__ __forceinline__ void reflector(const C alpha, R xnorm2, R& beta, C& tau, C& scal) {
    if (xnorm2 == 0 && alpha.y == 0) {
        beta = alpha.x;
        tau = cz<C>();
        scal = cm<C>(1, 0);
        return;
    }
    const R nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
    beta = alpha.x >= 0 ? -nrm : nrm;
    tau = cm<C>((beta - alpha.x) / beta, -alpha.y / beta);
    const C den = cm<C>(alpha.x - beta, alpha.y);
    const R dn = cabs2(den);
    scal = cm<C>(den.x / dn, -den.y / dn);
}

// Unblocked reduction A = Q T Q^H (zhetd2, uplo='U') with look-ahead: step i's rank-2
// update and step i-1's matrix-vector product share one pass over the leading block.
// a: n*n col-major (upper triangle), real type R (double, or float in the mixed mode); the
// leading m x m block is reduced (m < n after the blocked panels of k_hetrd_panel, which
// own E and TAU from index m - 1 on).
// On exit column c (c >= 1) rows 0..c-2 hold the reflector of step c-1 (its entry c-1 is
// 1 and not stored), D/E the tridiagonal (double) and TAU the reflector scalars.  The
// leading block moves into shared memory once its packed upper triangle fits in
// `tri_cap` elements.
template <int NT, class R>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 4)
k_hetrd(typename Cx<R>::T* __restrict__ A, double* __restrict__ D, double* __restrict__ E,
        typename Cx<R>::T* __restrict__ TAU, int n, int m, int tri_cap) {
    typedef typename Cx<R>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* v = reinterpret_cast<C*>(smem_raw);   // [m] current reflector
    C* w = v + m;                             // [m] its w vector
    C* vn = w + m;                            // [m] next reflector / column buffer
    C* pn = vn + m;                           // [m] A' vn accumulator
    R* red = reinterpret_cast<R*>(pn + m);    // [2*warps]
    C* tri = reinterpret_cast<C*>(red + 2 * (NT / 32));   // packed triangle
    const int tid = threadIdx.x;
    const size_t mat = blockIdx.x;
    GlobalStore<C> gs{A + mat * (size_t)n * n, n};
    SharedStore<C> ss{tri};
    double* dd = D + mat * n;
    double* ee = E + mat * n;
    C* tt = TAU + mat * n;
    if (m == 1) {
        if (tid == 0) {
            dd[0] = gs.at(0, 0)->x;
            if (m == n) {
                ee[0] = 0.0;
                tt[0] = cz<C>();
            }
        }
        return;
    }
    bool resident = false;
    // -- prologue: reflector of step m-2 from column m-1, then p = A v over [0..m-2]^2
    {
        const int i = m - 2;
        R part = 0;
        for (int r = tid; r <= i + 1; r += NT) {
            const C x = *gs.at(r, i + 1);
            vn[r] = x;
            if (r < i) part += cabs2(x);
        }
        const R xn2 = block_sum<NT>(part, red);
        R beta;
        C tau, scal;
        reflector(vn[i], xn2, beta, tau, scal);
        const bool act = !(tau.x == 0 && tau.y == 0);
        __syncthreads();
        for (int r = tid; r < i; r += NT) {
            const C x = act ? cmul(scal, vn[r]) : vn[r];
            v[r] = x;
            *gs.at(r, i + 1) = x;
        }
        for (int r = tid; r < m; r += NT) {
            w[r] = cz<C>();
            pn[r] = cz<C>();
        }
        if (tid == 0) {
            v[i] = cm<C>(1, 0);
            dd[m - 1] = vn[m - 1].x;
            *gs.at(i, i + 1) = cm<C>(beta, 0);
            ee[i] = beta;
            tt[i] = tau;
        }
        __syncthreads();
        fused_pass<NT>(gs, i + 1, v, w, false, v, act, pn);
        __syncthreads();
        C dpart = cz<C>();
        for (int r = tid; r <= i; r += NT) {
            const C x = cmul(tau, pn[r]);
            pn[r] = x;
            cfmac(dpart, x, v[r]);
        }
        const C xv = block_sum_c<NT>(dpart, red);
        const C al = cscale(cmul(tau, xv), (R)-0.5);
        for (int r = tid; r <= i; r += NT) w[r] = cadd(pn[r], cmul(al, v[r]));
        __syncthreads();
    }
    // -- main loop: v, w belong to step i (column i+1 done); finish column i, build the
    //    reflector of step i-1 from it, then one fused pass over [0..i-1]^2
    for (int i = m - 2; i >= 1; --i) {
        if (!resident && (i + 1) * (i + 2) / 2 <= tri_cap) {
            // move the leading (i+1)x(i+1) upper triangle into shared memory
            for (int c = 0; c <= i; ++c)
                for (int r = tid; r <= c; r += NT) *ss.at(r, c) = *gs.at(r, c);
            resident = true;
            __syncthreads();
        }
        // (1) updated column i, rows 0..i
        R part = 0;
        const C wi = w[i], vi = v[i];
        for (int r = tid; r <= i; r += NT) {
            C x = resident ? *ss.at(r, i) : *gs.at(r, i);
            C u = cmul(v[r], cconj(wi));
            cfma(u, w[r], cconj(vi));
            x = csub(x, u);
            vn[r] = x;
            if (r < i - 1) part += cabs2(x);
            pn[r] = cz<C>();
        }
        const R xn2 = block_sum<NT>(part, red);
        // (2) reflector of step i-1: alpha = A'[i-1][i], x = A'[0..i-2][i]
        R beta;
        C tau, scal;
        reflector(vn[i - 1], xn2, beta, tau, scal);
        const bool act = !(tau.x == 0 && tau.y == 0);
        __syncthreads();
        if (tid == 0) dd[i] = vn[i].x;
        for (int r = tid; r < i - 1; r += NT) {
            const C x = act ? cmul(scal, vn[r]) : vn[r];
            vn[r] = x;
            *gs.at(r, i) = x;   // reflector storage stays in global memory
        }
        if (tid == 0) {
            vn[i - 1] = cm<C>(1, 0);
            *gs.at(i - 1, i) = cm<C>(beta, 0);
            ee[i - 1] = beta;
            tt[i - 1] = tau;
        }
        __syncthreads();
        // (3) fused pass: update [0..i-1]^2 with (v, w), accumulate pn = A' vn
        if (resident) fused_pass<NT>(ss, i, v, w, true, vn, act, pn);
        else fused_pass<NT>(gs, i, v, w, true, vn, act, pn);
        __syncthreads();
        // (4) w' = tau pn - tau/2 (x^H vn) vn; v <- vn
        C dpart = cz<C>();
        for (int r = tid; r < i; r += NT) {
            const C x = cmul(tau, pn[r]);
            pn[r] = x;
            cfmac(dpart, x, vn[r]);
        }
        const C xv = block_sum_c<NT>(dpart, red);
        const C al = cscale(cmul(tau, xv), (R)-0.5);
        for (int r = tid; r < i; r += NT) {
            w[r] = act ? cadd(pn[r], cmul(al, vn[r])) : cz<C>();
            v[r] = vn[r];
        }
        __syncthreads();
    }
    // -- step 0's update reaches only A[0][0]
    if (tid == 0) {
        C x = resident ? *ss.at(0, 0) : *gs.at(0, 0);
        C u = cmul(v[0], cconj(w[0]));
        cfma(u, w[0], cconj(v[0]));
        dd[0] = x.x - u.x;
        if (m == n) {
            ee[n - 1] = 0.0;
            tt[n - 1] = cz<C>();
        }
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
            const double sc = ldexp(1.0, min(max(-ex, -1000), 1000));   // a denormal pair: no overflow
            p *= sc;
            pm *= sc;
            dp *= sc;
            dpm *= sc;
        }
    }
    ratio = p / dp;
    return cnt;
}

// The counts of sturm_poly at two shifts, the two recurrences interleaved (no derivatives).
__device__ __forceinline__ void sturm_count2(const double* __restrict__ d, const double* __restrict__ e2, int n,
                                             double xa, double xb, double pivmin, int& ca, int& cb) {
    double pma = 1.0, pa = d[0] - xa, pmb = 1.0, pb = d[0] - xb;
    if (fabs(pa) <= pivmin) pa = -pivmin;
    if (fabs(pb) <= pivmin) pb = -pivmin;
    int na = pa < 0.0, nb = pb < 0.0;
    for (int j = 1; j < n; ++j) {
        const double ee = e2[j - 1], dj = d[j];
        double qa = fma(dj - xa, pa, -ee * pma);
        double qb = fma(dj - xb, pb, -ee * pmb);
        if (fabs(qa) <= pivmin * fabs(pa)) qa = -pivmin * pa;
        if (fabs(qb) <= pivmin * fabs(pb)) qb = -pivmin * pb;
        na += (qa < 0.0) != (pa < 0.0);
        nb += (qb < 0.0) != (pb < 0.0);
        pma = pa;
        pa = qa;
        pmb = pb;
        pb = qb;
        const double biga = fmax(fabs(pa), fabs(pma)), bigb = fmax(fabs(pb), fabs(pmb));
        if (biga > 0x1p+400 || biga < 0x1p-400) {
            int ex;
            frexp(biga, &ex);
            const double sc = ldexp(1.0, min(max(-ex, -1000), 1000));   // a denormal pair: no overflow
            pa *= sc;
            pma *= sc;
        }
        if (bigb > 0x1p+400 || bigb < 0x1p-400) {
            int ex;
            frexp(bigb, &ex);
            const double sc = ldexp(1.0, min(max(-ex, -1000), 1000));   // a denormal pair: no overflow
            pb *= sc;
            pmb *= sc;
        }
    }
    ca = na;
    cb = nb;
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
    // D+ (forward, stationary) and D- (backward, progressive) are independent division
    // chains: one loop advances both, j forward and n-1-j backward
    double q = d[0] - x;
    if (fabs(q) <= pivmin) q = -pivmin;
    dplus[sc] = q;
    double qb = d[n - 1] - x;
    if (fabs(qb) <= pivmin) qb = -pivmin;
    dminus[(size_t)(n - 1) * TRI_THREADS + sc] = qb;
    for (int j = 1; j < n; ++j) {
        q = d[j] - x - e2[j - 1] / q;
        if (fabs(q) <= pivmin) q = -pivmin;
        dplus[(size_t)j * TRI_THREADS + sc] = q;
        const int jb = n - 1 - j;
        double qn = (d[jb] - x) - e2[jb] / qb;
        if (fabs(qn) <= pivmin) qn = -pivmin;
        qb = qn;
        dminus[(size_t)jb * TRI_THREADS + sc] = qb;
    }
    // twist index r = argmin |gamma_j|, gamma_j = D+_j + D-_j - (d_j - x), gamma_{n-1} = D+_{n-1}
    int r = n - 1;
    double gbest = fabs(q);
    for (int j = n - 2; j >= 0; --j) {
        const double gam = fabs(dplus[(size_t)j * TRI_THREADS + sc] + dminus[(size_t)j * TRI_THREADS + sc] - (d[j] - x));
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
    // ---- eigenvalue k: bisection on Sturm counts (dstebz bracketing, restated), accelerated
    //      by safeguarded Newton steps on det(T - x I), taken from the current point or from
    //      either end of the bracket, with the step scaled by the number m of eigenvalues in
    //      the bracket (exact for an m-fold root)
    if (PHASE == 1) {
    const double atol = 2.0 * DBL_EPSILON * onenrm;
    // one collective pass first: Sturm counts at the TRI_THREADS+1 equally spaced points of
    // the Gershgorin interval (count 0 at its left end, n at its right end), so that every
    // eigenvalue starts from the grid cell holding it instead of the whole interval
    __shared__ double s_gx[TRI_THREADS + 1];
    __shared__ int s_gc[TRI_THREADS + 1];
    {
        const double gl = s_gl, gu = s_gu;
        const int t = tid;
        s_gx[t] = t == 0 ? gl : gl + (gu - gl) * ((double)t / TRI_THREADS);
        if (t == 0) {
            s_gc[0] = 0;
            s_gx[TRI_THREADS] = gu;
            s_gc[TRI_THREADS] = n;
        } else {
            double rr;
            s_gc[t] = sturm_poly(d, e2, n, s_gx[t], pivmin, rr);
        }
    }
    __syncthreads();
    for (int k = tid; k < n; k += TRI_THREADS) {
        int cell = 0;   // largest grid point with count <= k
        for (int step = TRI_THREADS / 2; step >= 1; step >>= 1)
            if (cell + step < TRI_THREADS && s_gc[cell + step] <= k) cell += step;
        double lo = s_gx[cell], hi = s_gx[cell + 1];
        int clo = s_gc[cell], chi = s_gc[cell + 1];
        // Newton steps p/p' recorded at the bracket ends (valid flags), bracket widths of the
        // last two steps (bisection is forced when the bracket did not halve over two steps)
        double rlo = 0.0, rhi = 0.0;
        bool vlo = false, vhi = false;
        double w1 = hi - lo, w2 = hi - lo;
        double x = 0.5 * (lo + hi);
        double res = x;
        for (int it = 0; it < 200; ++it) {
            double ratio;
            const int c = sturm_poly(d, e2, n, x, pivmin, ratio);
            const bool rok = isfinite(ratio);
            if (c > k) { hi = x; chi = c; rhi = ratio; vhi = rok; } else { lo = x; clo = c; rlo = ratio; vlo = rok; }
            const double tol = fmax(atol, 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)));
            if (hi - lo <= tol) { res = 0.5 * (lo + hi); break; }
            double xn = 0.5 * (lo + hi);
            // Newton candidates x - m p/p' from x and from the two bracket ends, m = eigenvalues
            // in the bracket (the modified step converges on an m-fold cluster); the smallest
            // step first: a step within tol is verified by paired counts, else the first
            // candidate inside the bracket is taken
            const double m = (double)(chi - clo);
            double cs[3], cn[3];
            int nc = 0;
            if (rok) { cs[nc] = fabs(m * ratio); cn[nc++] = x - m * ratio; }
            if (vlo && x != lo) { cs[nc] = fabs(m * rlo); cn[nc++] = lo - m * rlo; }
            if (vhi && x != hi) { cs[nc] = fabs(m * rhi); cn[nc++] = hi - m * rhi; }
            for (int i = 1; i < nc; ++i)
                for (int j = i; j > 0 && cs[j] < cs[j - 1]; --j) {
                    const double ts = cs[j], tn = cn[j];
                    cs[j] = cs[j - 1]; cn[j] = cn[j - 1];
                    cs[j - 1] = ts; cn[j - 1] = tn;
                }
            bool accepted = false;
            for (int ci = 0; ci < nc; ++ci) {
                const double nt = cn[ci];
                if (cs[ci] <= tol) {
                    // converged step: accept only if Sturm counts bracket index k at nt +- 2 tol
                    const double a0 = fmax(lo, nt - 2.0 * tol), b0 = fmin(hi, nt + 2.0 * tol);
                    int ca, cb;
                    sturm_count2(d, e2, n, a0, b0, pivmin, ca, cb);
                    if (ca <= k && cb > k) { res = fmin(fmax(nt, lo), hi); accepted = true; break; }
                    if (ca > k) { hi = a0; chi = ca; vhi = false; } else { lo = b0; clo = cb; vlo = false; }
                    xn = 0.5 * (lo + hi);
                    break;
                }
                if (nt > lo && nt < hi) { xn = nt; break; }
            }
            if (accepted) break;
            if (hi - lo > 0.5 * w2) xn = 0.5 * (lo + hi);
            w2 = w1;
            w1 = hi - lo;
            if (xn <= lo || xn >= hi) { res = 0.5 * (lo + hi); break; }
            x = xn;
            res = x;
        }
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
    // ---- eigenvectors: isolated eigenvalues by one twisted solve; clusters (handled by the
    //      leader's thread) by twisted solves + modified Gram-Schmidt when their members are
    //      still separated, else by inverse iteration with modified Gram-Schmidt
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
        // a cluster whose members are still 1e-9 * ||T|| apart: each twisted vector is
        // accurate to ~eps ||T|| / gap, so a twisted solve per member followed by modified
        // Gram-Schmidt inside the cluster replaces the iterations
        double mingap = DBL_MAX;
        for (int k = k0 + 1; k <= k1; ++k) mingap = fmin(mingap, lam[k] - lam[k - 1]);
        if (mingap > 1e-9 * onenrm) {
            for (int k = k0; k <= k1; ++k) {
                twisted_vector(d, e, e2, n, lam[k], pivmin, z, k, la, lb, tid);
                for (int q = k0; q < k; ++q) {
                    double dot = 0.0;
                    for (int j = 0; j < n; ++j) dot += z[(size_t)j * n + q] * z[(size_t)j * n + k];
                    for (int j = 0; j < n; ++j) z[(size_t)j * n + k] -= dot * z[(size_t)j * n + q];
                }
                double x2s = 0.0, big = 0.0;
                for (int j = 0; j < n; ++j) {
                    const double t = z[(size_t)j * n + k];
                    x2s += t * t;
                    if (fabs(t) > fabs(big)) big = t;
                }
                double rn = 1.0 / sqrt(fmax(x2s, DBL_MIN));
                if (big < 0.0) rn = -rn;
                for (int j = 0; j < n; ++j) z[(size_t)j * n + k] *= rn;
            }
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

template <class C>
__device__ __forceinline__ C refl_entry(const C* __restrict__ a, int n, int i, int r) {
    // component r of reflector i (zero for i > n-2 padding)
    if (i > n - 2 || r > i) return cz<C>();
    if (r == i) return cm<C>(1, 0);
    return a[(size_t)(i + 1) * n + r];
}

// T factors of every block of one matrix (one CTA per matrix):
//   T[k][k] = tau_k,  T[k][q] = -tau_k sum_{l=q}^{k-1} (v_k^H v_l) T[l][q]   (q < k)
template <class R>
__global__ void __launch_bounds__(256)
k_larft(const typename Cx<R>::T* __restrict__ A, const typename Cx<R>::T* __restrict__ TAU,
        typename Cx<R>::T* __restrict__ Tw, int n) {
    typedef typename Cx<R>::T C;
    __shared__ C G[ORM_NB][ORM_NB];
    __shared__ C T[ORM_NB][ORM_NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t mat = blockIdx.x;
    const C* a = A + mat * (size_t)n * n;
    const C* tau = TAU + mat * n;
    const int nblk = (n - 1 + ORM_NB - 1) / ORM_NB;
    for (int j = 0; j < nblk; ++j) {
        const int i0 = j * ORM_NB;
        // G[k][l] = v_k^H v_l for l < k: rows 0..i0+l overlap
        for (int pr = warp; pr < ORM_NB * ORM_NB; pr += 8) {
            const int k = pr / ORM_NB, l = pr % ORM_NB;
            if (l >= k) continue;
            const int ik = i0 + k, il = i0 + l;
            C s = cz<C>();
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
                const C tk = ik <= n - 2 ? tau[ik] : cz<C>();
                if (lane < ORM_NB) {
                    C val = cz<C>();
                    if (lane == k) {
                        val = tk;
                    } else if (lane < k) {
                        C s = cz<C>();
                        for (int l = lane; l < k; ++l) cfma(s, G[k][l], T[l][lane]);
                        val = cscale(cmul(tk, s), (R)-1);
                    }
                    T[k][lane] = val;
                }
                __syncwarp();
            }
        }
        __syncthreads();
        C* out = Tw + (mat * nblk + j) * ORM_NB * ORM_NB;
        out[threadIdx.x] = T[threadIdx.x / ORM_NB][threadIdx.x % ORM_NB];
        __syncthreads();
    }
}

// asynchronous global -> shared copy of one complex element (16 or 8 bytes)
__device__ __forceinline__ void cp_async_elem(double2* smem_dst, const double2* gmem_src) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_elem(float2* smem_dst, const float2* gmem_src) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Stage block j of V (rows 0..i1, layout [r][k]) and its T factor into shared memory:
// stored reflector entries by cp.async, the implicit 1 and the zeros below by plain stores.
template <class C>
__device__ __forceinline__ void stage_block(const C* __restrict__ a, const C* __restrict__ tsrc,
                                            C* vsb, C* tsb, int n, int j) {
    const int t = threadIdx.x;
    const int i0 = j * ORM_NB;
    const int i1 = min(i0 + ORM_NB - 1, n - 2);
    for (int idx = t; idx < (i1 + 1) * ORM_NB; idx += blockDim.x) {
        const int r = idx / ORM_NB, k = idx % ORM_NB;
        const int i = i0 + k;
        C* dst = &vsb[r * ORM_VS + k];
        if (i <= n - 2 && r < i) cp_async_elem(dst, &a[(size_t)(i + 1) * n + r]);
        else *dst = (i <= n - 2 && r == i) ? cm<C>(1, 0) : cz<C>();
    }
    if (t < ORM_NB * ORM_NB) cp_async_elem(&tsb[t], &tsrc[t]);
    cp_async_commit();
}

// Apply all blocks to a chunk of CH columns of Z (row-major Z[r*n + col], real) and write
// the chunk of X (column-major, column = eigenvector).  NT threads; thread t owns column
// t % CH and the rows g + RG*q (g = t / CH, RG = NT/CH, q < RPT) in registers.  With dbuf
// the next block's V and T are copied asynchronously while the current block is applied.
template <int CH, int NT, int RPT, class R, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB)
k_ormtr(const typename Cx<R>::T* __restrict__ A, const typename Cx<R>::T* __restrict__ Tw,
        const double* __restrict__ Z, typename Cx<R>::T* __restrict__ X, int n, int dbuf) {
    typedef typename Cx<R>::T C;
    constexpr int RG = NT / CH, NW = NT / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* vsbuf[2];
    vsbuf[0] = reinterpret_cast<C*>(smem_raw);                    // [n][ORM_VS]
    vsbuf[1] = dbuf ? vsbuf[0] + (size_t)n * ORM_VS : vsbuf[0];
    C* tsbuf[2];
    tsbuf[0] = vsbuf[0] + (size_t)(dbuf ? 2 : 1) * n * ORM_VS;       // [ORM_NB][ORM_NB]
    tsbuf[1] = dbuf ? tsbuf[0] + ORM_NB * ORM_NB : tsbuf[0];
    C* wsum = tsbuf[0] + (size_t)(dbuf ? 2 : 1) * ORM_NB * ORM_NB;   // [NW][ORM_NB][CH]
    C* w2 = wsum + NW * ORM_NB * CH;                               // [ORM_NB][CH]
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int c = t % CH, g = t / CH;
    const size_t mat = blockIdx.y;
    const int col = blockIdx.x * CH + c;
    const C* a = A + mat * (size_t)n * n;
    const double* z = Z + mat * (size_t)n * n;
    const int nblk = (n - 1 + ORM_NB - 1) / ORM_NB;
    const C* tw = Tw + mat * (size_t)nblk * ORM_NB * ORM_NB;
    C x[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
        const int r = g + RG * q;
        x[q] = (r < n && col < n) ? cm<C>(z[(size_t)r * n + col], 0) : cz<C>();
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
        const C* vs = vsbuf[j & 1];
        const C* ts = tsbuf[j & 1];
        // partial W = V^H X over this thread's rows
        C wp[ORM_NB];
#pragma unroll
        for (int k = 0; k < ORM_NB; ++k) wp[k] = cz<C>();
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            const int r = g + RG * q;
            if (r <= i1) {
                const C* vr = vs + r * ORM_VS;
#pragma unroll
                for (int k = 0; k < ORM_NB; ++k) cfmac(wp[k], vr[k], x[q]);
            }
        }
        // reduce over the row groups: inside the warp, then across the NW warps
#pragma unroll
        for (int s2 = CH; s2 < 32; s2 <<= 1)
#pragma unroll
            for (int k = 0; k < ORM_NB; ++k) wp[k] = cadd(wp[k], shfl_xor(wp[k], s2));
        if (lane < CH)
#pragma unroll
            for (int k = 0; k < ORM_NB; ++k) wsum[(warp * ORM_NB + k) * CH + lane] = wp[k];
        __syncthreads();
        C wk = cz<C>();
        if (t < ORM_NB * CH) {
            for (int w8 = 0; w8 < NW; ++w8) wk = cadd(wk, wsum[w8 * ORM_NB * CH + t]);
            wsum[t] = wk;   // W[k][c] at t = k*CH + c (slot of warp 0, already read)
        }
        __syncthreads();
        if (t < ORM_NB * CH) {
            const int k = t / CH, cc = t % CH;
            C s = cz<C>();
            for (int q2 = 0; q2 <= k; ++q2) cfma(s, ts[k * ORM_NB + q2], wsum[q2 * CH + cc]);
            w2[t] = s;
        }
        __syncthreads();
        // X -= V W2 on rows <= i1
        C wc[ORM_NB];
#pragma unroll
        for (int k = 0; k < ORM_NB; ++k) wc[k] = w2[k * CH + c];
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            const int r = g + RG * q;
            if (r <= i1) {
                const C* vr = vs + r * ORM_VS;
                C s = cz<C>();
#pragma unroll
                for (int k = 0; k < ORM_NB; ++k) cfma(s, vr[k], wc[k]);
                x[q] = csub(x[q], s);
            }
        }
        __syncthreads();
    }
    // write the chunk column-major through shared memory (coalesced along rows)
    C* xs = vsbuf[0];   // [CH][n]
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
        const int r = g + RG * q;
        if (r < n) xs[(size_t)c * n + r] = x[q];
    }
    __syncthreads();
    C* xo = X + mat * (size_t)n * n;
    const int col0 = blockIdx.x * CH;
    for (int idx = t; idx < CH * n; idx += NT) {
        const int cc = idx / n, r = idx % n;
        if (col0 + cc < n) xo[(size_t)(col0 + cc) * n + r] = xs[idx];
    }
}

// ------------------------------------------------ back-transformation for large orders
// For orders whose 16-reflector blocks do not fit the register/shared-memory scheme of
// k_ormtr, X = Q Z is applied with blocks of BT_NB = 64 reflectors (or 128, a tuning choice)
// as tiled complex GEMMs per block (LAPACK zlarfb restated): W' = T (V^H X), then
// X -= V W'.  X lives in global memory (column-major, column = eigenvector) and is read twice
// and written once per block.
static constexpr int BT_NB = 64;
static constexpr int BT_GEMM_MIN = 256;   // order from which the GEMM back-transformation runs
// Blocks of 128 reflectors (T from two 64-reflector halves, k_larft128) halve the passes
// over X, but at order 3000 they were no faster in double precision and 10 % slower in single
// precision (the block GEMMs are bound by the tensor pipes, not by X's traffic): they are a
// tuning choice (HeevTune::bt_nb, rlmb_set_heev_config), not the built-in one.
static constexpr int BT128_MIN = 1 << 30;

// T factor of block j (reflectors 64j .. 64j+63) of one matrix from its Gram matrix
// G = V_j^H V_j (column-major 64 x 64, computed by a batched GEMM into the same slot of Tw):
//   T[k][k] = tau_k,  T[k][q] = -tau_k sum_{l=q}^{k-1} G[k][l] T[l][q]   (q < k),
// written back row-major (T[k][q] at k*64 + q); grid (blocks, matrices), 128 threads.
// The recurrence reads G only above its diagonal (S[l][k], l < k, with S[l][k] = G[k][l])
// and T only on and below it, so T overwrites the lower half of the one shared table S as
// it is formed.  Two threads share row q of T (even and odd l), halving the dependent chain.
template <class R>
__global__ void __launch_bounds__(2 * BT_NB)
k_larft64(const typename Cx<R>::T* __restrict__ TAU, typename Cx<R>::T* __restrict__ Tw, int n) {
    typedef typename Cx<R>::T C;
    typedef C Row[BT_NB + 1];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Row* S = reinterpret_cast<Row*>(smem_raw);   // S[l][k] = G[k][l] (l < k); T[k][q] at S[k][q] (q <= k)
    const int j = blockIdx.x, q = threadIdx.x >> 1, h = threadIdx.x & 1;
    const size_t mat = blockIdx.y;
    const C* tau = TAU + mat * n;
    const int nblk = (n - 1 + BT_NB - 1) / BT_NB;
    const int i0 = j * BT_NB;
    C* blk = Tw + (mat * nblk + j) * BT_NB * BT_NB;
    for (int idx = threadIdx.x; idx < BT_NB * BT_NB; idx += 2 * BT_NB) S[idx / BT_NB][idx % BT_NB] = blk[idx];
    __syncthreads();
    for (int k = 0; k < BT_NB; ++k) {
        const int ik = i0 + k;
        const C tk = ik <= n - 2 ? tau[ik] : cz<C>();
        C sum = cz<C>();
        if (q < k)
            for (int l = q + h; l < k; l += 2) cfma(sum, S[l][k], S[l][q]);
        sum = cadd(sum, shfl_xor(sum, 1));
        if (h == 0 && q <= k) S[k][q] = q == k ? tk : cscale(cmul(tk, sum), (R)-1);
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < BT_NB * BT_NB; idx += 2 * BT_NB) {
        const int k = idx / BT_NB, c = idx % BT_NB;
        blk[idx] = c <= k ? S[k][c] : cz<C>();
    }
}

// T factor of a block of 128 reflectors (128j .. 128j+127) from its 128 x 128 Gram matrix
// G = V^H V (column-major, in the block's slot of Tw), written back row-major:
//   T = [[T1, 0], [T21, T2]],   T21 = -T2 (G21 T1),   G21 = V2^H V1,
// where T1 and T2 are the T factors of the two halves (the k_larft64 recurrence, run on both
// at once by the two halves of the CTA) -- the same matrix the zlarft recurrence gives for
// all 128 reflectors.  Grid (blocks, matrices), 256 threads; shared memory: S1, S2 (the
// halves' recurrence tables as in k_larft64) and Y (G21, then G21 T1).
template <class R>
__global__ void __launch_bounds__(256)
k_larft128(const typename Cx<R>::T* __restrict__ TAU, typename Cx<R>::T* __restrict__ Tw, int n) {
    typedef typename Cx<R>::T C;
    constexpr int H = 64, B = 128;
    typedef C Row[H + 1];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Row* S1 = reinterpret_cast<Row*>(smem_raw);
    Row* S2 = S1 + H;
    Row* Y = S2 + H;
    const int j = blockIdx.x, tid = threadIdx.x;
    const size_t mat = blockIdx.y;
    const C* tau = TAU + mat * n;
    const int nblk = (n - 1 + B - 1) / B;
    const int i0 = j * B;
    C* blk = Tw + (mat * nblk + j) * B * B;
    // S1[l][k] = G(k, l), S2[l][k] = G(64 + k, 64 + l), Y[k][l] = G21(k, l) = G(64 + k, l)
    for (int idx = tid; idx < H * H; idx += 256) {
        const int a = idx / H, b = idx % H;
        S1[a][b] = blk[(size_t)a * B + b];
        S2[a][b] = blk[(size_t)(H + a) * B + H + b];
        Y[b][a] = blk[(size_t)a * B + H + b];
    }
    __syncthreads();
    {
        const int half = tid >> 7, q = (tid & 127) >> 1, h = tid & 1;
        Row* S = half ? S2 : S1;
        const int ib = i0 + H * half;
        for (int k = 0; k < H; ++k) {
            const int ik = ib + k;
            const C tk = ik <= n - 2 ? tau[ik] : cz<C>();
            C sum = cz<C>();
            if (q < k)
                for (int l = q + h; l < k; l += 2) cfma(sum, S[l][k], S[l][q]);
            sum = cadd(sum, shfl_xor(sum, 1));
            if (h == 0 && q <= k) S[k][q] = q == k ? tk : cscale(cmul(tk, sum), (R)-1);
            __syncthreads();
        }
    }
    // thread: row k of the 64 x 64 products, columns q = c4 + 4 i
    const int k = tid >> 2, c4 = tid & 3;
    C acc[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = cz<C>();
    // Y <- G21 T1: (G21 T1)[k][q] = sum_{l >= q} G21[k][l] T1[l][q], T1[l][q] = S1[l][q]
    for (int l = 0; l < H; ++l) {
        const C g = Y[k][l];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int q = c4 + 4 * i;
            if (l >= q) cfma(acc[i], g, S1[l][q]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 16; ++i) Y[k][c4 + 4 * i] = acc[i];
    __syncthreads();
    // T21 = -T2 Y: T21[k][q] = -sum_{l <= k} T2[k][l] Y[l][q], T2[k][l] = S2[k][l]
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = cz<C>();
    for (int l = 0; l <= k; ++l) {
        const C t2 = S2[k][l];
#pragma unroll
        for (int i = 0; i < 16; ++i) cfma(acc[i], t2, Y[l][c4 + 4 * i]);
    }
    // row-major T: rows 0..63 [T1 0], rows 64..127 [T21 T2]
    for (int idx = tid; idx < H * H; idx += 256) {
        const int a = idx / H, b = idx % H;
        blk[(size_t)a * B + b] = b <= a ? S1[a][b] : cz<C>();
        blk[(size_t)a * B + H + b] = cz<C>();
        blk[(size_t)(H + a) * B + H + b] = b <= a ? S2[a][b] : cz<C>();
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) blk[(size_t)(H + k) * B + c4 + 4 * i] = cscale(acc[i], (R)-1);
}

// Z (row-major real) -> X (column-major complex), grid-stride over all batch entries.
template <class C>
__global__ void k_z_to_x(const double* __restrict__ Z, C* __restrict__ X, int n, size_t total) {
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const size_t nn = (size_t)n * n;
        const size_t mat = idx / nn, rem = idx % nn;
        const int c = (int)(rem / n), r = (int)(rem % n);
        X[idx] = cm<C>(Z[mat * nn + (size_t)r * n + c], 0);
    }
}

// ------------------------------------------------------------------ GEMM operands
// Element accessors for the GEMM engines of launch_zgemm (A: elem(mat, r, k), B: elem(mat, k, c)).

// A(r, k) = P(r, k) of a column-major P (entry at p[k*ld + r]): r contiguous.
template <class C, class PT>
struct OpColA {
    static constexpr bool RFAST = true;
    const PT* p;
    int ld;
    size_t stride;
    __device__ __forceinline__ C elem(size_t mat, int r, int k) const {
        return from_c64<C>(to_c64(p[mat * stride + (size_t)k * ld + r]));
    }
};

// A(r, k) = P(k, r), conjugated if CONJ, of a column-major P (entry (k, r) at p[r*ld + k]):
// the (conjugate) transpose, k contiguous.
template <class C, class PT, bool CONJ>
struct OpRowA {
    static constexpr bool RFAST = false;
    const PT* p;
    int ld;
    size_t stride;
    __device__ __forceinline__ C elem(size_t mat, int r, int k) const {
        C v = from_c64<C>(to_c64(p[mat * stride + (size_t)r * ld + k]));
        if (CONJ) v.y = -v.y;
        return v;
    }
};

// B(k, c) = P(k, c) of a column-major P (entry at p[c*ld + k]): k contiguous.
template <class C, class PT>
struct OpColB {
    static constexpr bool KFAST = true;
    const PT* p;
    int ld;
    size_t stride;
    __device__ __forceinline__ C elem(size_t mat, int k, int c) const {
        return from_c64<C>(to_c64(p[mat * stride + (size_t)c * ld + k]));
    }
};

// Reflectors i0 + q of a reduced matrix as columns of V (V(r, q) = v_{i0+q}[r], with the
// implicit 1 and the zeros): OpRefl gives A = V (r contiguous), OpReflH A = V^H.
template <class C>
struct OpRefl {
    static constexpr bool RFAST = true;
    const C* a;
    int n, i0;
    __device__ __forceinline__ C elem(size_t mat, int r, int q) const {
        return refl_entry(a + mat * (size_t)n * n, n, i0 + q, r);
    }
};
template <class C>
struct OpReflH {
    static constexpr bool RFAST = false;
    const C* a;
    int n, i0;
    __device__ __forceinline__ C elem(size_t mat, int q, int r) const {
        C v = refl_entry(a + mat * (size_t)n * n, n, i0 + q, r);
        v.y = -v.y;
        return v;
    }
};

// Gram matrices of all blocks of bs reflectors in one batched GEMM: batch index z = mat * nblk
// + j; A(q, r) = conj(v_{bs j+q}[r]), B(r, l) = v_{bs j+l}[r].
template <class C>
struct OpBlkReflH {
    static constexpr bool RFAST = false;
    const C* a;
    int n, nblk, bs;
    __device__ __forceinline__ C elem(size_t z, int q, int r) const {
        C v = refl_entry(a + (z / nblk) * (size_t)n * n, n, (int)(z % nblk) * bs + q, r);
        v.y = -v.y;
        return v;
    }
};
template <class C>
struct OpBlkRefl {
    static constexpr bool KFAST = true;
    const C* a;
    int n, nblk, bs;
    __device__ __forceinline__ C elem(size_t z, int r, int l) const {
        return refl_entry(a + (z / nblk) * (size_t)n * n, n, (int)(z % nblk) * bs + l, r);
    }
};

// Complete a Hermitian matrix stored in the upper triangle (column-major, 'U') in place:
// lower triangle = conjugate of the upper, imaginary part of the diagonal zeroed.  Tiles of
// 32 x 32 through shared memory, both sides coalesced; grid (n/32, n/32, matrices), only
// tiles on or below the diagonal work.  Reads (strict upper) and writes (strict lower and
// diagonal) never overlap.
__global__ void k_herm_fill(cplx* __restrict__ A, int n) {
    __shared__ cplx tile[32][33];
    const int cb = blockIdx.x, rb = blockIdx.y;   // output tile: rows rb, columns cb
    if (rb < cb) return;
    cplx* a = A + (size_t)blockIdx.z * n * n;
    const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
    // input: upper entries (c, r) at a[r*n + c] for r in block rb, c in block cb
    for (int j = ty; j < 32; j += 8) {
        const int r = rb * 32 + j, c = cb * 32 + tx;
        if (r < n && c < n && c < r) tile[j][tx] = a[(size_t)r * n + c];
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int c = cb * 32 + j, r = rb * 32 + tx;
        if (r < n && c < n) {
            if (r > c) a[(size_t)c * n + r] = cconj(tile[tx][j]);
            else if (r == c) a[(size_t)c * n + r].y = 0.0;
        }
    }
}

// Epilogues
template <class C>
struct EpStore {   // P(r, c) = acc, column-major P with leading dimension ld
    C* p;
    int ld;
    size_t stride;
    __device__ __forceinline__ bool skip(int, int, int) const { return false; }
    __device__ __forceinline__ void store(size_t mat, int r, int c, C acc) const {
        p[mat * stride + (size_t)c * ld + r] = acc;
    }
};
template <class C>
struct EpSub {     // X(r, c) -= acc
    C* x;
    int n;
    __device__ __forceinline__ bool skip(int, int, int) const { return false; }
    __device__ __forceinline__ void store(size_t mat, int r, int c, C acc) const {
        C* q = x + mat * (size_t)n * n + (size_t)c * n + r;
        *q = csub(*q, acc);
    }
    // the GEMM engines prefetch X(r, c) (the DMMA engine into shared memory, the tcgen05
    // engine into registers) and pass it back as `old`
    __device__ __forceinline__ const C* pre_src(size_t mat, int r, int c) const {
        return x + mat * (size_t)n * n + (size_t)c * n + r;
    }
    __device__ __forceinline__ void store_pre(size_t mat, int r, int c, C acc, C old) const {
        x[mat * (size_t)n * n + (size_t)c * n + r] = csub(old, acc);
    }
};

// ------------------------------------------------------------- blocked k_hetrd (large n)
// For large orders the reduction runs in panels of pw (16 or 32) columns (LAPACK zlatrd + zher2k,
// uplo='U', restated): k_hetrd_panel reduces columns m-1 .. m-pw of the leading m x m
// block one CTA per matrix, keeping each column's reflector v and its w = tau A' v - ...
// in the panel buffers V, W instead of updating the leading block: column c is first
// brought up to date with the panel's earlier pairs, its matrix-vector product reads the
// leading c x c block as stored (read only) and is corrected by the same pairs.  The
// rank-2*pw update A -= V W^H + W V^H of the remaining leading block then runs as a GEMM
// over all SMs (launch_zgemm, EpHer2k), and the last block (order <= HT_TAIL) is reduced by
// k_hetrd.  D, E, TAU and the reflector storage are those of the unblocked reduction.
// Panel width: in double precision 32 columns from order HP_W_WIDE_MIN (at n = 3000 the
// rank-64 updates save 17 % of the update time, the panels cost the same), 16 below (measured
// faster than 8, 12, 24 and 32 at orders 256-1000).  Single precision keeps 16: with 32 the
// panel folds up to 31 pairs into each column in FP32, and two refinement steps then left an
// orthogonality defect of 2.6e-10 at n = 1600 (1e-12 with 16), for a 3 % saving.  Shared
// memory and the pair storage are laid out for the plan's width; HP_W_MAX bounds it.
static constexpr int HP_W_MAX = 32;
static constexpr int HP_W_WIDE_MIN = 1024;
static constexpr int HT_TAIL = 64;   // order below which the unblocked kernel finishes
static constexpr int HT_BLOCKED_MIN = 256;   // orders from which the blocked reduction runs
static constexpr int DC_DEFAULT_MIN = 600;   // orders from which divide and conquer is the built-in tridiagonal solver (measured: even with bisection at 512, 1.4x at 1024, 2.3x at 3000)
static constexpr int JAC_DEFAULT_MAX = 20;    // orders up to which k_jacobi is the built-in solver (measured: 2.1x the Householder path at 16, even at 24)
static constexpr int QUEUE_NT_DEFAULT = 512;   // panel queue CTAs: 512 threads, one per SM
static constexpr int TUNE_MIN_N = 16;         // orders the autotuner tunes: TUNE_MIN_N .. TUNE_MAX_N
static constexpr int TUNE_MAX_N = 1024;

// p += A v for the Hermitian leading m x m block stored in the upper triangle of a
// (column-major, leading dimension ld; read only), v and p in shared memory.  Work is dealt
// to warps as strips of HV_W columns (dealt back and forth for balance); a lane holds one
// row of a 32-row block of the strip:
// its row contributions go to p[r] (shared atomics, once per block), its column
// contributions conj(A[r][c]) v[r] stay in registers for the whole strip and are reduced
// across the warp once at the end.  Interior blocks (entirely above the diagonal and inside
// the matrix) run without predicates.
// Strip width: 8 columns in double precision, 16 in single precision, so that a lane has the
// same bytes of loads in flight (128) in both modes: the product streams the leading block
// from memory and is bound by the loads each SM keeps in flight, not by its arithmetic.
template <class C>
__host__ __device__ constexpr int hv_width() { return sizeof(C) == 8 ? 16 : 8; }
template <int NT, class C>
__device__ __forceinline__ void hemv_upper(const C* __restrict__ a, int ld, int m, const C* __restrict__ v,
                                           C* p) {
    constexpr int HV_W = hv_width<C>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    const int nstrips = (m + HV_W - 1) / HV_W;
    // strip s holds s*HV_W/32 + 1 row blocks: deal them back and forth (warp w takes strips
    // w, 2NW-1-w, 2NW+w, ...) so that every warp gets a similar amount of work
    for (int base = 0; base < nstrips; base += NW) {
        const int s = ((base / NW) & 1) ? base + NW - 1 - warp : base + warp;
        if (s >= nstrips) continue;
        const int c0 = s * HV_W;
        C vc[HV_W], e[HV_W];
#pragma unroll
        for (int j = 0; j < HV_W; ++j) {
            vc[j] = c0 + j < m ? v[c0 + j] : cz<C>();
            e[j] = cz<C>();
        }
        const C* colp = a + (size_t)c0 * ld;
        const int rend = min(c0 + HV_W, m);   // rows that meet the strip on or above the diagonal
        const bool full = c0 + HV_W <= m;
#pragma unroll 1
        for (int r0 = 0; r0 < rend; r0 += 32) {
            const int r = r0 + lane;
            const bool interior = full && r0 + 32 <= c0;
            C x[HV_W];
            if (interior) {
#pragma unroll
                for (int j = 0; j < HV_W; ++j) x[j] = colp[(size_t)j * ld + r];
            } else {
#pragma unroll
                for (int j = 0; j < HV_W; ++j) {
                    const int cc = c0 + j;
                    x[j] = (cc < m && r <= cc) ? colp[(size_t)j * ld + r] : cz<C>();
                }
            }
            const C vr = r < m ? v[r] : cz<C>();
            C rowacc = cz<C>();
#pragma unroll
            for (int j = 0; j < HV_W; ++j) {
                if (interior || r < c0 + j) {
                    cfma(rowacc, x[j], vc[j]);
                    cfmac(e[j], x[j], vr);
                } else if (r == c0 + j) {
                    rowacc = cadd(rowacc, cscale(vc[j], x[j].x));
                }
            }
            if (r < rend) smem_atomic_add(&p[r], rowacc);
        }
        // column sums: lane l ends with the sum over the warp of e[l & (HV_W - 1)]
#pragma unroll
        for (int mask = 16; mask >= HV_W; mask >>= 1)
#pragma unroll
            for (int j = 0; j < HV_W; ++j) e[j] = cadd(e[j], shfl_xor(e[j], mask));
#pragma unroll
        for (int sh = HV_W / 2; sh >= 1; sh >>= 1) {
            const bool up = (lane & sh) != 0;
#pragma unroll
            for (int j = 0; j < sh; ++j) {
                const C send = up ? e[j] : e[j + sh];
                const C keep = up ? e[j + sh] : e[j];
                e[j] = cadd(keep, shfl_xor(send, sh));
            }
        }
        if (lane < HV_W && c0 + lane < m) smem_atomic_add(&p[c0 + lane], e[0]);
    }
}

// Loads of the panel pairs V, W: through L1 (ld) when one CTA owns the matrix for the whole
// panel, around it (ld.global.cg) when other CTAs wrote them during the same launch.
template <bool CG, class C>
__device__ __forceinline__ C pv_ld(const C* p) {
    if constexpr (CG) return __ldcg(p);
    else return *p;
}

// Column j of the panel (column c = m - 1 - j of the leading m x m block) of matrix mat, by
// the NT threads of one CTA; vn, pn, coef, red: the CTA's shared work arrays.
template <int NT, class R, bool CG>
__device__ __forceinline__ void panel_column(typename Cx<R>::T* __restrict__ A, double* __restrict__ D,
                                             double* __restrict__ E, typename Cx<R>::T* __restrict__ TAU,
                                             typename Cx<R>::T* __restrict__ PV, typename Cx<R>::T* __restrict__ PW,
                                             int n, int m, size_t mat, int j, int pw, typename Cx<R>::T* vn,
                                             typename Cx<R>::T* pn, typename Cx<R>::T* coef, R* red) {
    typedef typename Cx<R>::T C;
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    GlobalStore<C> gs{A + mat * (size_t)n * n, n};
    double* dd = D + mat * n;
    double* ee = E + mat * n;
    C* tt = TAU + mat * n;
    C* V = PV + mat * (size_t)pw * n;   // pair q at V + q*n, W + q*n
    C* W = PW + mat * (size_t)pw * n;
    if (m == n && j == 0 && tid == 0) {
        ee[n - 1] = 0.0;
        tt[n - 1] = cz<C>();
    }
    const int c = m - 1 - j;
    // (1) column c brought up to date with the panel's pairs q < j
    R part = 0;
    for (int r = tid; r <= c; r += NT) {
        C x = *gs.at(r, c);
        for (int q = 0; q < j; ++q) {
            const C* vq = V + (size_t)q * n;
            const C* wq = W + (size_t)q * n;
            C u = cmul(pv_ld<CG>(vq + r), cconj(pv_ld<CG>(wq + c)));
            cfma(u, pv_ld<CG>(wq + r), cconj(pv_ld<CG>(vq + c)));
            x = csub(x, u);
        }
        if (r == c) x.y = 0;
        vn[r] = x;
        if (r < c - 1) part += cabs2(x);
        if (r < c) pn[r] = cz<C>();
    }
    const R xn2 = block_sum<NT>(part, red);
    // (2) reflector of step c-1: alpha = A'[c-1][c], x = A'[0..c-2][c]
    R beta;
    C tau, scal;
    reflector(vn[c - 1], xn2, beta, tau, scal);
    const bool act = !(tau.x == 0 && tau.y == 0);
    __syncthreads();
    if (tid == 0) dd[c] = vn[c].x;
    for (int r = tid; r < c - 1; r += NT) {
        const C x = act ? cmul(scal, vn[r]) : vn[r];
        vn[r] = x;
        *gs.at(r, c) = x;
    }
    if (tid == 0) {
        vn[c - 1] = cm<C>(1, 0);
        *gs.at(c - 1, c) = cm<C>(beta, 0);
        ee[c - 1] = beta;
        tt[c - 1] = tau;
    }
    __syncthreads();
    // (3) pn = A v over the stored leading c x c block (read only)
    if (act) hemv_upper<NT>(gs.a, n, c, vn, pn);
    // (4) w_q^H v (even slots) and v_q^H v (odd slots) for q < j
    for (int t2 = warp; t2 < 2 * j; t2 += NW) {
        const int q = t2 >> 1;
        const C* y = (t2 & 1) ? V + (size_t)q * n : W + (size_t)q * n;
        C sd = cz<C>();
        for (int r = lane; r < c; r += 32) cfmac(sd, pv_ld<CG>(y + r), vn[r]);
        sd = warp_sum(sd);
        if (lane == 0) coef[t2] = sd;
    }
    __syncthreads();
    // (5) x = tau (pn - sum_q V_q (w_q^H v) + W_q (v_q^H v)); w = x - tau/2 (x^H v) v
    C dpart = cz<C>();
    for (int r = tid; r < c; r += NT) {
        C x = pn[r];
        for (int q = 0; q < j; ++q) {
            C u = cmul(pv_ld<CG>(V + (size_t)q * n + r), coef[2 * q]);
            cfma(u, pv_ld<CG>(W + (size_t)q * n + r), coef[2 * q + 1]);
            x = csub(x, u);
        }
        x = cmul(tau, x);
        pn[r] = x;
        cfmac(dpart, x, vn[r]);
    }
    const C xv = block_sum_c<NT>(dpart, red);
    const C al = cscale(cmul(tau, xv), (R)-0.5);
    C* vj = V + (size_t)j * n;
    C* wj = W + (size_t)j * n;
    for (int r = tid; r < c; r += NT) {
        vj[r] = vn[r];
        wj[r] = act ? cadd(pn[r], cmul(al, vn[r])) : cz<C>();
    }
    __syncthreads();
}

// Shared work arrays of the panel kernels: vn [m] (column / reflector), pn [m] (A' v
// accumulator), coef [2*HP_W_MAX] (w_q^H v, v_q^H v), red [2*warps].
template <int NT, class R>
__host__ __device__ constexpr size_t panel_smem(int m) {
    return (2 * (size_t)m + 2 * HP_W_MAX) * sizeof(typename Cx<R>::T) + 2 * (NT / 32) * sizeof(R);
}

// One CTA per matrix: the panel's pw columns in order.
template <int NT, class R>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2)
k_hetrd_panel(typename Cx<R>::T* __restrict__ A, double* __restrict__ D, double* __restrict__ E,
              typename Cx<R>::T* __restrict__ TAU, typename Cx<R>::T* __restrict__ PV,
              typename Cx<R>::T* __restrict__ PW, int n, int m, int pw) {
    typedef typename Cx<R>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* vn = reinterpret_cast<C*>(smem_raw);
    C* pn = vn + m;
    C* coef = pn + m;
    R* red = reinterpret_cast<R*>(coef + 2 * HP_W_MAX);
    for (int j = 0; j < pw; ++j)
        panel_column<NT, R, false>(A, D, E, TAU, PV, PW, n, m, blockIdx.x, j, pw, vn, pn, coef, red);
}

// The same panel for chunks of more matrices than SMs: one resident CTA of NT threads per SM
// (grid <= SMs) takes units (matrix, column) from a queue, unit u = claim - base = matrix
// u % nb, column u / nb, so that every SM keeps NT threads of loads in flight whatever the
// number of matrices (one CTA per matrix would leave SMs with a single CTA when the chunk has
// between one and two matrices per SM).  Column j of a matrix needs column j - 1 (its panel
// pair): q[2 + mat] counts the columns of each matrix completed in the chunk; a unit waits
// for done = col0 + j, a wait bounded by TC_WAIT_NS that sets the abort flag q[1] (and counts
// in g_tc_fault) when it runs out.  The claims of a launch end with one failed claim per CTA,
// so launch k's units start at base = k * (nb * pw + grid).  Units are claimed in order and
// wait only on earlier claims, which CTAs already running hold: no wait depends on a CTA
// that has not started.
template <int NT, class R>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2)
k_hetrd_panel_q(typename Cx<R>::T* __restrict__ A, double* __restrict__ D, double* __restrict__ E,
                typename Cx<R>::T* __restrict__ TAU, typename Cx<R>::T* __restrict__ PV,
                typename Cx<R>::T* __restrict__ PW, int n, int m, int pw, int nb, int* q, long long base, int col0,
                int* __restrict__ info) {
    typedef typename Cx<R>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* vn = reinterpret_cast<C*>(smem_raw);
    C* pn = vn + m;
    C* coef = pn + m;
    R* red = reinterpret_cast<R*>(coef + 2 * HP_W_MAX);
    __shared__ long long s_unit;
    __shared__ int s_go;
    const int tid = threadIdx.x;
    const long long units = (long long)nb * pw;
    for (;;) {
        if (tid == 0) {
            long long u = (long long)atomicAdd(reinterpret_cast<unsigned long long*>(q + 4), 1ull) - base;
            if (*(volatile int*)(q + 1)) u = units;   // aborted: stop claiming work
            s_unit = u;
            s_go = 1;
            if (u < units && u >= nb) {   // column j > 0: wait for column j - 1 of the matrix
                const int mat = (int)(u % nb), j = (int)(u / nb);
                const int* dp = q + 8 + mat;
                int v;
                asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(dp) : "memory");
                if (v < col0 + j) {
                    const unsigned long long t0 = tc_ns();
                    for (;;) {
                        __nanosleep(64);
                        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(dp) : "memory");
                        if (v >= col0 + j) break;
                        if (*(volatile int*)(q + 1) || tc_ns() - t0 > TC_WAIT_NS) {
                            if (atomicExch(q + 1, 1) == 0) atomicAdd(&g_tc_fault, 1);
                            if (info) info[mat] = -1;
                            s_go = 0;
                            break;
                        }
                    }
                }
            }
        }
        __syncthreads();
        const long long u = s_unit;
        const int go = s_go;
        __syncthreads();
        if (u >= units || !go) break;
        __threadfence();
        const int mat = (int)(u % nb), j = (int)(u / nb);
        panel_column<NT, R, true>(A, D, E, TAU, PV, PW, n, m, mat, j, pw, vn, pn, coef, red);
        // every thread's writes of the column, then the release of the column count
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            const int v = col0 + j + 1;
            int* dp = q + 8 + mat;
            asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(dp), "r"(v) : "memory");
        }
    }
}

// [V | W] (r, k) and [W | V]^H (k, c) of a panel: the operands of A -= V W^H + W V^H.
template <class C, int w>
struct OpPanelA {
    static constexpr bool RFAST = true;
    const C* pv;
    const C* pw;
    int n;
    __device__ __forceinline__ C elem(size_t mat, int r, int k) const {
        const size_t o = mat * (size_t)w * n;
        return k < w ? pv[o + (size_t)k * n + r] : pw[o + (size_t)(k - w) * n + r];
    }
};
template <class C, int w>
struct OpPanelB {
    static constexpr bool KFAST = false;
    const C* pv;
    const C* pw;
    int n;
    __device__ __forceinline__ C elem(size_t mat, int k, int c) const {
        const size_t o = mat * (size_t)w * n;
        return cconj(k < w ? pw[o + (size_t)k * n + c] : pv[o + (size_t)(k - w) * n + c]);
    }
};
// A(r, c) -= acc on and above the diagonal (real diagonal); tiles below it are skipped.
template <class C>
struct EpHer2k {
    C* a;
    int n;
    __device__ __forceinline__ bool skip(int r0, int c0, int) const { return r0 > c0 + ZG_BN - 1; }
    __device__ __forceinline__ bool skip_tile(int r0, int c0, int, int cols) const { return r0 > c0 + cols - 1; }
    __device__ __forceinline__ void store(size_t mat, int r, int c, C acc) const {
        if (r > c) return;
        C* q = a + mat * (size_t)n * n + (size_t)c * n + r;
        C x = csub(*q, acc);
        if (r == c) x.y = 0;
        *q = x;
    }
    // the GEMM engines prefetch A(r, c) (on and above the diagonal) when the tile starts
    __device__ __forceinline__ const C* pre_src(size_t mat, int r, int c) const {
        return r > c ? nullptr : a + mat * (size_t)n * n + (size_t)c * n + r;
    }
    __device__ __forceinline__ void store_pre(size_t mat, int r, int c, C acc, C old) const {
        C x = csub(old, acc);
        if (r == c) x.y = 0;
        a[mat * (size_t)n * n + (size_t)c * n + r] = x;
    }
};

// The GEMMs of the reduction and back-transformation in the working precision C: double on
// the FP64 tensor path (DMMA engine, BM-row tiles), single precision (the mixed mode) on the
// tcgen05 tensor cores with split TF32 operands.
template <class C, int BM, class LA, class LB, class EP>
static cudaError_t launch_work_gemm(cudaStream_t st, const LA& la, const LB& lb, const EP& ep, int M, int N, int K,
                                    int nb) {
    if constexpr (std::is_same<C, cplxf>::value) return launch_zgemm_tc<C>(st, la, lb, ep, M, N, K, nb);
    else return launch_zgemm<C, BM>(st, la, lb, ep, M, N, K, nb);
}

// ------------------------------------------------- mixed mode: FP64 refinement kernels
// The mixed mode reduces and back-transforms in single precision (k_hetrd<.., float>,
// k_larft / k_ormtr or the blocked path on float), solves the tridiagonal in double
// (k_tridiag), then refines the eigenpairs (X, lambda) of H in double, in the manner of
// Ogita & Aishima (2018, "Iterative refinement for symmetric eigenvalue decomposition"),
// one or two steps:
//   R = H X - X diag(lambda)                            k_ref_resid     (double)
//   E = X^H R,  F_ij = E_ij / (lambda_j - lambda_i)     k_ref_coupling  (double, i != j)
//   F_jj = (1 - x_j^H x_j) / 2,
//   lambda_j += Re(x_j^H r_j) / x_j^H x_j               k_ref_diag      (double)
//   X <- X + X F                                        k_ref_update    (single product,
//                                                                        double sum)
// X F is a first-order correction of the size of the current error, so a single-precision
// product carries it; R, E and the diagonal need double.  Each step roughly squares the
// relative error of the vectors.
// Two neighbouring eigenpairs whose gap is within 8 x their residual norms ||r_j|| are not
// separated by the current vectors (first-order theory needs |x_i^H r_j| << gap), and for
// gaps below 2^-14 of the spectral radius the first-order correction cannot restore
// orthogonality to double precision (its error is ~ u ||H|| / gap; LAPACK's inverse
// iteration likewise re-orthogonalises eigenvalues closer than 1e-3 ||T||, dstein): chains
// of such gaps form clusters (k_ref_clusters).  Inside a cluster of at most RF_KMAX members the vectors are re-resolved
// by a Rayleigh-Ritz step on the cluster's subspace in double (k_ref_cluster_solve: S =
// X_C^H H X_C = E_CC + G_CC Lambda, G_CC = X_C^H X_C, S y = mu G y; k_ref_cluster_apply:
// X_C <- X_C Y, lambda_C <- mu).  Larger clusters, and any other pair whose gap is within
// 8 |E_ij|, are orthogonalised only, F_ij = -(x_i^H x_j)/2, and keep Rayleigh quotients.
static constexpr int RF_KMAX = 16;             // largest cluster resolved by Rayleigh-Ritz
static constexpr double RF_RES = 8.0;          // gap / residual ratio below which pairs cluster
static constexpr double RF_CLUSTER = 0x1p-14;  // relative gap below which pairs cluster

// R = H X - X diag(lambda): epilogue of the GEMM H X (H completed by k_herm_fill).
template <class XT>
struct EpResid {
    const XT* x;
    const double* w;
    cplx* res;
    int n;
    __device__ __forceinline__ bool skip(int, int, int) const { return false; }
    __device__ __forceinline__ void store(size_t mat, int r, int c, cplx acc) const {
        const size_t o = mat * (size_t)n * n + (size_t)c * n + r;
        const cplx xr = to_c64(x[o]);
        const double lam = w[mat * n + c];
        res[o] = mk(acc.x - lam * xr.x, acc.y - lam * xr.y);
    }
};

// R = H X - X diag(lambda) for a cyclic band matrix H of half-bandwidth o (H(r, k) = 0 unless
// the cyclic distance of r and k is at most o -- the rlm Hamiltonian's structure,
// rlm/hamiltonian_rlm_cpu.cpp:26-38), in double, with 32 + 2o <= n.  An output tile of 32 rows
// x 64 columns needs only the 32 + 2o rows k = r0 - o .. r0 + 31 + o (cyclic) of X: the tile's
// band rows of H, zero-padded to a dense 32 x (32 + 2o) block, times those rows of X, in
// chunks of 16.  Row r of H is read as the conjugate of column r (contiguous in k) of the
// Hermitian matrix stored in full.  Thread (tr, tc) computes rows 2 tr, 2 tr + 1 and columns
// tc + 16 j (j < 4) of the tile: 8 complex multiply-adds per 6 shared-memory loads.
template <class XT>
__global__ void __launch_bounds__(256)
k_ref_resid_band(const cplx* __restrict__ A, const XT* __restrict__ X, const double* __restrict__ W,
                 cplx* __restrict__ Res, int n, int o) {
    __shared__ cplx hs[16][32 + 1];   // hs[kk][rl] = H(r0 + rl, k(kk))
    __shared__ cplx xs[16][64 + 1];   // xs[kk][cl] = X(k(kk), c0 + cl)
    const int t = threadIdx.x, tr = t >> 4, tc = t & 15;
    const size_t mat = blockIdx.z;
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 64;
    const size_t nn = (size_t)n * n;
    const cplx* Am = A + mat * nn;
    const XT* Xm = X + mat * nn;
    const int span = 32 + 2 * o;   // k(kk) = (r0 - o + kk) mod n, kk < span
    cplx acc[2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = mk(0, 0);
    for (int k0 = 0; k0 < span; k0 += 16) {
        {   // H band: (kk, rl) = (t % 16, t / 16 + 16 h)
            const int kk = t & 15;
            const int kg = k0 + kk;
            int k = r0 - o + kg;
            k = k < 0 ? k + n : (k >= n ? k - n : k);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int rl = (t >> 4) + 16 * h, r = r0 + rl;
                const int dist = kg - rl;   // k - r + o
                cplx v = mk(0, 0);
                if (kg < span && r < n && dist >= 0 && dist <= 2 * o) v = cconj(Am[(size_t)r * n + k]);
                hs[kk][rl] = v;
            }
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int cl = (t >> 4) + 16 * h, c = c0 + cl;
                xs[kk][cl] = (kg < span && c < n) ? to_c64(Xm[(size_t)c * n + k]) : mk(0, 0);
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            const cplx h0 = hs[kk][2 * tr], h1 = hs[kk][2 * tr + 1];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const cplx x = xs[kk][tc + 16 * j];
                cfma(acc[0][j], h0, x);
                cfma(acc[1][j], h1, x);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int c = c0 + tc + 16 * j;
        if (c >= n) continue;
        const double lam = W[mat * n + c];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = r0 + 2 * tr + i;
            if (r >= n) continue;
            const size_t off = mat * nn + (size_t)c * n + r;
            const cplx xr = to_c64(X[off]);
            Res[off] = mk(acc[i][j].x - lam * xr.x, acc[i][j].y - lam * xr.y);
        }
    }
}

// The same band product on the FP64 tensor path: operands of the DMMA engine (64-row output
// tiles) for R = H X - X diag(lambda) with a cyclic band H of half-width o, 64 + 2o <= n.  The
// tile of rows r0 = 64 blockIdx.x .. r0 + 63 needs only the columns k(kk) = (r0 - o + kk) mod n,
// kk < 64 + 2o, of H, which becomes the inner dimension:
//   A(r, kk) = H(r, k(kk)) where 0 <= kk - (r - r0) <= 2o, else 0 (read as the conjugate of
//              column r of the stored Hermitian H, contiguous in kk);
//   B(kk, c) = X(k(kk), c).
// 64 + 2o inner terms per output against 2o + 1 nonzero ones (1.29x at o = 110), on a pipe
// ~4x faster than the FP64 FMA of k_ref_resid_band.
static constexpr int RB_BM = 64;
struct OpBandA {
    static constexpr bool RFAST = false;
    const cplx* p;
    int n, o;
    __device__ __forceinline__ cplx elem(size_t mat, int r, int kk) const {
        const int r0 = r - r % RB_BM;
        const int dist = kk - (r - r0);
        if (dist < 0 || dist > 2 * o) return mk(0.0, 0.0);
        int k = r0 - o + kk;
        k = k < 0 ? k + n : (k >= n ? k - n : k);
        return cconj(p[mat * (size_t)n * n + (size_t)r * n + k]);
    }
};
template <class XT>
struct OpBandB {
    static constexpr bool KFAST = true;
    const XT* p;
    int n, o;
    __device__ __forceinline__ cplx elem(size_t mat, int kk, int c) const {
        int k = (int)blockIdx.x * RB_BM - o + kk;   // the tile's r0 (the engine's row tile is RB_BM)
        k = k < 0 ? k + n : (k >= n ? k - n : k);
        return to_c64(p[mat * (size_t)n * n + (size_t)c * n + k]);
    }
};

// R = H X - X diag(W): cyclic band H on DMMA where the band fits a 64-row tile's span, else the
// FP64-FMA band kernel; dense H as a full DMMA GEMM.
template <class XT>
static cudaError_t launch_resid(cudaStream_t st, const cplx* A, const XT* X, const double* W, cplx* Res, int n,
                                int band, int nb) {
    const size_t nn = (size_t)n * n;
    if (band >= 0 && RB_BM + 2 * band <= n)
        return launch_zgemm<cplx, RB_BM>(st, OpBandA{A, n, band}, OpBandB<XT>{X, n, band},
                                         EpResid<XT>{X, W, Res, n}, n, n, RB_BM + 2 * band, nb);
    if (band >= 0) {
        k_ref_resid_band<XT><<<dim3((n + 31) / 32, (n + 63) / 64, nb), 256, 0, st>>>(A, X, W, Res, n, band);
        return cudaGetLastError();
    }
    return launch_zgemm<cplx, 64>(st, OpColA<cplx, cplx>{A, n, nn}, OpColB<cplx, XT>{X, n, nn},
                                  EpResid<XT>{X, W, Res, n}, n, n, n, nb);
}

// Per eigenvector j (one warp each), in double: G_jj = x_j^H x_j, q_j = Re(x_j^H r_j) and
// ||r_j||, stored as ST[3 (mat n + j) + {0, 1, 2}].
template <class XT>
__global__ void k_ref_colstats(const XT* __restrict__ X, const cplx* __restrict__ Res, double* __restrict__ ST,
                               int n, int nmat) {
    const int lane = threadIdx.x & 31;
    const size_t gw = (size_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (gw >= (size_t)nmat * n) return;
    const size_t mat = gw / n;
    const int j = (int)(gw % n);
    const XT* x = X + mat * (size_t)n * n + (size_t)j * n;
    const cplx* r = Res + mat * (size_t)n * n + (size_t)j * n;
    double g = 0.0, q = 0.0, rr = 0.0;
    for (int k = lane; k < n; k += 32) {
        const cplx xv = to_c64(x[k]), rv = r[k];
        g += xv.x * xv.x + xv.y * xv.y;
        q += xv.x * rv.x + xv.y * rv.y;
        rr += rv.x * rv.x + rv.y * rv.y;
    }
    g = warp_sum(g);
    q = warp_sum(q);
    rr = warp_sum(rr);
    if (lane == 0) {
        ST[3 * gw] = g;
        ST[3 * gw + 1] = q;
        ST[3 * gw + 2] = sqrt(rr);
    }
}

// Clusters of the ascending eigenvalues of each matrix (one thread per matrix): chains of
// consecutive pairs with gap <= RF_RES * max(||r||/||x||) or <= RF_CLUSTER * spectral radius.
// cl[j] = (first index, size).
__global__ void k_ref_clusters(const double* __restrict__ W, const double* __restrict__ ST, int2* __restrict__ cl,
                               int n, int nmat) {
    const int mat = blockIdx.x * blockDim.x + threadIdx.x;
    if (mat >= nmat) return;
    const double* w = W + (size_t)mat * n;
    const double* st = ST + (size_t)mat * n * 3;
    int2* c = cl + (size_t)mat * n;
    const double tie = RF_CLUSTER * fmax(fabs(w[0]), fabs(w[n - 1]));
    int a = 0;
    double rho_prev = st[2] / sqrt(fmax(st[0], DBL_MIN));
    for (int j = 1; j <= n; ++j) {
        bool split = true;
        double rho = 0.0;
        if (j < n) {
            rho = st[3 * j + 2] / sqrt(fmax(st[3 * j], DBL_MIN));
            const double gap = w[j] - w[j - 1];
            split = gap > tie && gap > RF_RES * fmax(rho, rho_prev);
        }
        if (split) {
            for (int m = a; m < j; ++m) c[m] = make_int2(a, j - a);
            a = j;
        }
        rho_prev = rho;
    }
}

// double overlap of two columns (single or double storage)
template <class XT>
__device__ __forceinline__ cplx col_dot(const XT* __restrict__ xi, const XT* __restrict__ xj, int n) {
    cplx g = mk(0, 0);
    for (int k = 0; k < n; ++k) cfmac(g, to_c64(xi[k]), to_c64(xj[k]));
    return g;
}

// F_ij = (X^H R)_ij / (lambda_j - lambda_i) for i != j; zero on the diagonal (set by
// k_ref_diag) and inside Rayleigh-Ritz clusters; -(x_i^H x_j)/2 inside larger clusters and
// for pairs too close for a first-order correction.  Epilogue of the GEMM X^H R taken in
// double: F + F^H must cancel the orthogonality defect (E_ij - conj(E_ji) = (lambda_i -
// lambda_j) x_i^H x_j).
template <class XT>
struct EpCoupling {
    const XT* x;
    const double* w;
    const int2* cl;
    cplxf* f;
    int n;
    __device__ __forceinline__ bool skip(int, int, int) const { return false; }
    __device__ __forceinline__ void store(size_t mat, int i, int j, cplx acc) const {
        cplxf val = make_float2(0.f, 0.f);
        if (i != j) {
            const double* wm = w + mat * n;
            const int2* cm_ = cl + mat * n;
            const double gap = wm[j] - wm[i];
            const int2 cj = cm_[j];
            const bool same = cm_[i].x == cj.x;
            if (same && cj.y <= RF_KMAX) {
                val = make_float2(0.f, 0.f);   // resolved by k_ref_cluster_solve
            } else if (!same && fabs(gap) > 8.0 * sqrt(cabs2(acc))) {
                const double ig = 1.0 / gap;
                val = make_float2((float)(acc.x * ig), (float)(acc.y * ig));
            } else {
                const XT* xm = x + mat * (size_t)n * n;
                const cplx g = col_dot(xm + (size_t)i * n, xm + (size_t)j * n, n);
                val = make_float2((float)(-0.5 * g.x), (float)(-0.5 * g.y));
            }
        }
        f[mat * (size_t)n * n + (size_t)j * n + i] = val;
    }
};

// Rayleigh-Ritz on each cluster of 2..RF_KMAX members (one warp per cluster, found at its
// first index): G = X_C^H X_C and E = X_C^H R_C by warp sums in double, S = E + G Lambda
// (Hermitian part), then in one lane G = L L^H, C = L^-1 S L^-H, Jacobi C = V diag(mu) V^H,
// Y = L^-H V (ascending mu).  Y[j][p] (column j's coefficients) and mu[j] go to YB / MU.
// Lane 0's part of k_ref_cluster_solve for the cluster of k members starting at eigenpair a
// of matrix mat: G (Gram) and S (Rayleigh) of the cluster in, Y and mu out.
__device__ __noinline__ void cluster_rr_serial(cplx* G, cplx* S, cplx* T, int k, size_t mat, int a, int n,
                                               const double* __restrict__ w, cplx* __restrict__ YB,
                                               double* __restrict__ MU) {
    // Hermitian parts
    for (int p = 0; p < k; ++p)
        for (int q = p; q < k; ++q) {
            const cplx gs = cscale(cadd(G[p + q * k], cconj(G[q + p * k])), 0.5);
            const cplx ss = cscale(cadd(S[p + q * k], cconj(S[q + p * k])), 0.5);
            G[p + q * k] = gs;
            G[q + p * k] = cconj(gs);
            S[p + q * k] = ss;
            S[q + p * k] = cconj(ss);
        }
    // Cholesky G = L L^H (L lower, stored in G's lower triangle and diagonal)
    for (int j = 0; j < k; ++j) {
        double d = G[j + j * k].x;
        for (int m = 0; m < j; ++m) d -= cabs2(G[j + m * k]);
        if (!(d > 0.0)) {   // not positive definite: leave the cluster as it is
            for (int q = 0; q < k; ++q) {
                cplx* yo = YB + (mat * n + a + q) * RF_KMAX;
                for (int p = 0; p < k; ++p) yo[p] = mk(p == q ? 1.0 : 0.0, 0.0);
                MU[mat * n + a + q] = w[a + q];
            }
            return;
        }
        const double ljj = sqrt(d);
        G[j + j * k] = mk(ljj, 0.0);
        for (int i = j + 1; i < k; ++i) {
            cplx s = G[i + j * k];
            for (int m = 0; m < j; ++m) s = csub(s, cmul(G[i + m * k], cconj(G[j + m * k])));
            G[i + j * k] = cscale(s, 1.0 / ljj);
        }
    }
    // T = L^-1 S (columns), then C = L^-1 T^H  (= L^-1 S L^-H, Hermitian)
    for (int q = 0; q < k; ++q)
        for (int i = 0; i < k; ++i) {
            cplx s = S[i + q * k];
            for (int m = 0; m < i; ++m) s = csub(s, cmul(G[i + m * k], T[m + q * k]));
            T[i + q * k] = cscale(s, 1.0 / G[i + i * k].x);
        }
    for (int q = 0; q < k; ++q)
        for (int i = 0; i < k; ++i) {
            cplx s = cconj(T[q + i * k]);
            for (int m = 0; m < i; ++m) s = csub(s, cmul(G[i + m * k], S[m + q * k]));
            S[i + q * k] = cscale(s, 1.0 / G[i + i * k].x);   // S now holds C
        }
    for (int p = 0; p < k; ++p)
        for (int q = p + 1; q < k; ++q) {
            const cplx h = cscale(cadd(S[p + q * k], cconj(S[q + p * k])), 0.5);
            S[p + q * k] = h;
            S[q + p * k] = cconj(h);
        }
    for (int p = 0; p < k; ++p) S[p + p * k].y = 0.0;
    for (int i = 0; i < k * k; ++i) T[i] = mk(i % (k + 1) == 0 ? 1.0 : 0.0, 0.0);
    herm_jacobi(S, T, k);   // T <- V
    // ascending order
    int order[RF_KMAX];
    for (int i = 0; i < k; ++i) order[i] = i;
    for (int i = 1; i < k; ++i)
        for (int j = i; j > 0 && S[order[j] * (k + 1)].x < S[order[j - 1] * (k + 1)].x; --j) {
            const int tmp = order[j];
            order[j] = order[j - 1];
            order[j - 1] = tmp;
        }
    // Y = L^-H V by back substitution, column by column
    for (int q = 0; q < k; ++q) {
        const int col = order[q];
        cplx y[RF_KMAX];
        for (int i = k - 1; i >= 0; --i) {
            cplx s = T[i + col * k];
            for (int m = i + 1; m < k; ++m) s = csub(s, cmul(cconj(G[m + i * k]), y[m]));
            y[i] = cscale(s, 1.0 / G[i + i * k].x);
        }
        cplx* yo = YB + (mat * n + a + q) * RF_KMAX;
        for (int p = 0; p < k; ++p) yo[p] = y[p];
        MU[mat * n + a + q] = S[col * (k + 1)].x;
    }
}

template <class XT>
__global__ void k_ref_cluster_solve(const XT* __restrict__ X, const cplx* __restrict__ Res,
                                    const double* __restrict__ W, const int2* __restrict__ CL,
                                    cplx* __restrict__ YB, double* __restrict__ MU, int n, int nmat) {
    const int lane = threadIdx.x & 31;
    // G, S and T of this warp's cluster in shared memory (column-major [p + q*k]); only lane 0
    // writes and reads them
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* G = reinterpret_cast<cplx*>(smem_raw) + (size_t)(threadIdx.x / 32) * 3 * RF_KMAX * RF_KMAX;
    cplx* S = G + RF_KMAX * RF_KMAX;
    cplx* T = S + RF_KMAX * RF_KMAX;
    // grid-stride over the eigenpairs: most are not cluster leaders and are skipped at once
    const size_t nwarps = (size_t)gridDim.x * (blockDim.x / 32);
    for (size_t gw = (size_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; gw < (size_t)nmat * n;
         gw += nwarps) {
        const size_t mat = gw / n;
        const int a = (int)(gw % n);
        const int2 c = CL[mat * n + a];
        const int k = c.y;
        if (c.x != a || k < 2 || k > RF_KMAX) continue;
        const XT* x = X + mat * (size_t)n * n;
        const cplx* res = Res + mat * (size_t)n * n;
        const double* w = W + mat * n;
        for (int p = 0; p < k; ++p)
            for (int q = 0; q < k; ++q) {
                const XT* xp = x + (size_t)(a + p) * n;
                const XT* xq = x + (size_t)(a + q) * n;
                const cplx* rq = res + (size_t)(a + q) * n;
                cplx g = mk(0, 0), e = mk(0, 0);
                for (int r = lane; r < n; r += 32) {
                    const cplx xpr = to_c64(xp[r]);
                    cfmac(g, xpr, to_c64(xq[r]));
                    cfmac(e, xpr, rq[r]);
                }
                g = warp_sum(g);
                e = warp_sum(e);
                if (lane == 0) {
                    G[p + q * k] = g;
                    S[p + q * k] = mk(e.x + w[a + q] * g.x, e.y + w[a + q] * g.y);
                }
            }
        if (lane == 0) cluster_rr_serial(G, S, T, k, mat, a, n, w, YB, MU);
        __syncwarp();
    }
}

// Per eigenvector j (one thread each): lambda_j += q_j / G_jj (Rayleigh quotient) and
// F_jj = (1 - G_jj) / 2 from k_ref_colstats -- except for members of Rayleigh-Ritz clusters
// (F_jj = 0, lambda from k_ref_cluster_apply).
__global__ void k_ref_diag(const double* __restrict__ ST, const int2* __restrict__ CL, double* __restrict__ W,
                           cplxf* __restrict__ F, int n, int nmat) {
    const size_t gj = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gj >= (size_t)nmat * n) return;
    const size_t mat = gj / n;
    const int j = (int)(gj % n);
    const int2 c = CL[gj];
    cplxf* fjj = F + mat * (size_t)n * n + (size_t)j * n + j;
    if (c.y >= 2 && c.y <= RF_KMAX) {
        *fjj = make_float2(0.f, 0.f);
        return;
    }
    const double g = ST[3 * gj], q = ST[3 * gj + 1];
    W[gj] += q / g;
    *fjj = make_float2((float)(0.5 * (1.0 - g)), 0.f);
}

// X_out = X + X F: epilogue of the single-precision GEMM X F, sum in double, into a
// buffer other than X.
template <class XT>
struct EpUpdate {
    const XT* x;
    cplx* out;
    int n;
    __device__ __forceinline__ bool skip(int, int, int) const { return false; }
    __device__ __forceinline__ void store(size_t mat, int r, int c, cplxf acc) const {
        const size_t o = mat * (size_t)n * n + (size_t)c * n + r;
        const cplx xr = to_c64(x[o]);
        out[o] = mk(xr.x + (double)acc.x, xr.y + (double)acc.y);
    }
};

// X_C <- X_C Y and lambda_C <- mu for every Rayleigh-Ritz cluster (one warp per cluster,
// rows dealt to lanes; every row is read before it is written, so in place).
__global__ void k_ref_cluster_apply(cplx* __restrict__ X, const int2* __restrict__ CL, const cplx* __restrict__ YB,
                                    const double* __restrict__ MU, double* __restrict__ W, int n, int nmat) {
    const int lane = threadIdx.x & 31;
    const size_t gw = (size_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (gw >= (size_t)nmat * n) return;
    const size_t mat = gw / n;
    const int a = (int)(gw % n);
    const int2 c = CL[gw];
    const int k = c.y;
    if (c.x != a || k < 2 || k > RF_KMAX) return;
    cplx y[RF_KMAX * RF_KMAX];   // y[p + q*k]
    for (int q = 0; q < k; ++q)
        for (int p = 0; p < k; ++p) y[p + q * k] = YB[(mat * n + a + q) * RF_KMAX + p];
    cplx* x = X + mat * (size_t)n * n + (size_t)a * n;
    for (int r = lane; r < n; r += 32) {
        cplx old[RF_KMAX];
        for (int p = 0; p < k; ++p) old[p] = x[(size_t)p * n + r];
        for (int q = 0; q < k; ++q) {
            cplx s = mk(0, 0);
            for (int p = 0; p < k; ++p) cfma(s, old[p], y[p + q * k]);
            x[(size_t)q * n + r] = s;
        }
    }
    if (lane < k) W[mat * n + a + lane] = MU[mat * n + a + lane];
}

// double -> single copy of the matrices (the single-precision reduction works on the copy;
// the double input stays for the residual)
__global__ void k_to_single(const cplx* __restrict__ A, cplxf* __restrict__ B, size_t total) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        B[i] = from_c64<cplxf>(A[i]);
}

// Launch shape of k_hetrd: small matrices keep their whole triangle in shared memory with
// 128 threads and several CTAs per SM; larger ones run 512 threads, one CTA per SM, with
// as much of the leading triangle resident as ~220 KB allows.
struct HetrdCfg {
    int nt;
    int tri_cap;
    size_t smem;
};
template <class R>
static HetrdCfg hetrd_config(int n) {
    const size_t ce = 2 * sizeof(R);   // complex element
    const size_t tri_full = (size_t)n * (n + 1) / 2;
    const size_t vec128 = 4 * (size_t)n * ce + 2 * (128 / 32) * sizeof(R);
    if (vec128 + tri_full * ce <= 110 * 1024) return {128, (int)tri_full, vec128 + tri_full * ce};
    const size_t vec512 = 4 * (size_t)n * ce + 2 * (512 / 32) * sizeof(R);
    const size_t budget = 220 * 1024;
    size_t cap = budget > vec512 ? (budget - vec512) / ce : 0;
    cap = std::min(cap, tri_full);
    return {512, (int)cap, vec512 + cap * ce};
}
template <class R>
static cudaError_t launch_hetrd(const HetrdCfg& c, cudaStream_t st, int nb, typename Cx<R>::T* A, double* D,
                                double* E, typename Cx<R>::T* TAU, int n, int m) {
    if (c.smem > 227 * 1024) return cudaErrorInvalidValue;
    if (c.nt == 128) {
        cudaError_t e = cudaFuncSetAttribute(k_hetrd<128, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
        if (e != cudaSuccess) return e;
        k_hetrd<128, R><<<nb, 128, c.smem, st>>>(A, D, E, TAU, n, m, c.tri_cap);
    } else {
        cudaError_t e = cudaFuncSetAttribute(k_hetrd<512, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
        if (e != cudaSuccess) return e;
        k_hetrd<512, R><<<nb, 512, c.smem, st>>>(A, D, E, TAU, n, m, c.tri_cap);
    }
    return cudaGetLastError();
}

// Launch choices of one eigensolve configuration that the autotuner may set (0 / -1: the
// built-in choice for the order).
struct HeevTune {
    int blocked = -1;    // 1: blocked reduction (16-column panels + GEMM updates), 0: unblocked only
    int gemm_bt = -1;    // 1: GEMM back-transformation, 0: register-resident k_ormtr (where it fits)
    int panel_nt = 0;    // threads per panel CTA, 256 or 512
    int xtile = 0;       // row tile of the double-precision X -= V W' update, 64 or 128
    int bt_nb = 0;       // reflectors per block of the GEMM back-transformation, 64 or 128
    int jacobi = -1;     // 1: batched Jacobi (k_jacobi, orders <= JAC_MAX_N), 0: the Householder path
    int queue_nt = 0;    // panel queue CTAs: 512 threads (one per SM) or 256 (two per SM); 0: built-in
    int panel_w = 0;     // panel width, 16 or 32; 0: built-in (32 from order HP_W_WIDE_MIN in FP64)
    int dc = -1;         // tridiagonal stage: 1 divide and conquer (orders <= DC_MAX_N), 0 bisection +
                         // inverse iteration (k_tridiag)
};

// Shape of one eigensolve chunk: kernel configurations and the scratch layout per matrix
// (byte offsets, each region a multiple of 256 bytes so that every region of a chunk
// starts aligned whatever the chunk size).
struct HeevPlan {
    int n;
    bool jacobi;         // k_jacobi in double precision (either mode); nothing below applies
    size_t smem_jac;
    bool dc;             // divide-and-conquer tridiagonal stage (tridiag_dc.cuh) instead of k_tridiag
    size_t off_q2, off_u, off_rot, off_sc;   // its second Q, U, rotations and scale
    bool mixed;          // single-precision reduction + double refinement
    int refine_steps;    // mixed mode: 1 or 2
    bool rq;             // mixed mode, one step: then the eigenvalues as Rayleigh quotients (H kept until then)
    int band;            // >= 0: every matrix is a cyclic band of this half-bandwidth (rlm), else -1
    HetrdCfg hc;
    size_t smem_tri;
    bool small_bt;       // k_ormtr (register-resident Z chunk) or the blocked GEMM path
    int ch, dbuf;
    size_t smem_orm;
    int nblk16, bt_nb, nblkbt;   // k_ormtr blocks; GEMM back-transformation block size and count
    int npanels, m_tail;  // blocked reduction: panels of pw columns, then k_hetrd on m_tail
    int pw;               // panel width, 16 or 32
    int panel_nt, xtile;  // tuned launch choices (0: built-in)
    int queue_nt;         // threads of the panel queue's CTAs (512: one per SM, 256: two per SM)
    // per: bytes per matrix of the chunk's regions (offsets off_*, times the chunk size);
    // per2: bytes per matrix of the mixed mode's refinement regions (Res, X1), which the
    // refinement uses for one sub-chunk of matrices at a time
    size_t per2, off2_x1;
    size_t off_d, off_e, off_tau, off_a, off_z, off_lu, off_x, off_t, off_w, off_res, off_x1, off_cl,
        off_y, off_mu, off_st, off_pv, off_q, per;
};

static HeevPlan heev_plan(int n, bool mixed, int refine_steps = 2, int band = -1, HeevTune tune = HeevTune{}) {
    HeevPlan p{};
    p.panel_nt = tune.panel_nt;
    p.xtile = tune.xtile;
    p.queue_nt = tune.queue_nt ? tune.queue_nt : QUEUE_NT_DEFAULT;
    p.n = n;
    p.mixed = mixed;
    p.band = band >= 0 && 32 + 2 * band <= n ? band : -1;   // the band residual needs 32 + 2o <= n
    // refine_steps 3 (heev_steps): one step, then the Rayleigh-quotient eigenvalue pass
    p.rq = mixed && refine_steps == 3;
    p.refine_steps = mixed ? (refine_steps == 3 ? 1 : refine_steps) : 0;
    p.jacobi = n <= JAC_MAX_N && (tune.jacobi < 0 ? n <= JAC_DEFAULT_MAX : tune.jacobi > 0);
    if (p.jacobi) {   // no scratch: the matrix and its rotations live in shared memory
        p.smem_jac = jacobi_smem(n);
        p.per = 256;
        return p;
    }
    const size_t ce = mixed ? sizeof(cplxf) : sizeof(cplx);   // working complex element
    p.pw = tune.panel_w ? tune.panel_w : n >= HP_W_WIDE_MIN && !mixed ? 32 : 16;
    const bool blocked = tune.blocked < 0 ? n >= HT_BLOCKED_MIN : (tune.blocked > 0 && n > HT_TAIL + p.pw);
    p.npanels = blocked ? (n - HT_TAIL + p.pw - 1) / p.pw : 0;
    p.m_tail = n - p.npanels * p.pw;
    p.hc = mixed ? hetrd_config<float>(p.m_tail) : hetrd_config<double>(p.m_tail);
    p.smem_tri = 4 * (size_t)n * sizeof(double) + n * sizeof(int);
    p.nblk16 = (n - 1 + ORM_NB - 1) / ORM_NB;
    p.bt_nb = tune.bt_nb ? tune.bt_nb : n >= BT128_MIN ? 2 * BT_NB : BT_NB;
    p.nblkbt = (n - 1 + p.bt_nb - 1) / p.bt_nb;
    int ch = 16;
    while (ch > 1 && (n + 256 / ch - 1) / (256 / ch) > ORM_RPT) ch >>= 1;
    p.ch = ch;
    const int onw = 8;   // warps of k_ormtr (256 threads; 512 threads of 8 rows, or 8 columns
                         // of 8 rows at two CTAs per SM, measured slower)
    size_t smem = ((size_t)2 * n * ORM_VS + 2 * ORM_NB * ORM_NB + onw * ORM_NB * ch + ORM_NB * ch) * ce;
    p.dbuf = smem <= 220 * 1024 ? 1 : 0;
    if (!p.dbuf)
        smem = ((size_t)std::max(n * ORM_VS, n * ch) + ORM_NB * ORM_NB + onw * ORM_NB * ch + ORM_NB * ch) * ce;
    p.smem_orm = smem;
    // register-resident k_ormtr up to order 255 (it beats the GEMM path there), the GEMM path
    // (double precision on the DMMA engine) from 256 on
    const bool reg_fits = (n + 256 / ch - 1) / (256 / ch) <= ORM_RPT && smem <= 220 * 1024;
    p.small_bt = reg_fits && (tune.gemm_bt < 0 ? n < BT_GEMM_MIN : tune.gemm_bt == 0);
    const size_t nn = (size_t)n * n;
    auto r256 = [](size_t v) { return (v + 255) / 256 * 256; };
    size_t off = 0;
    p.off_d = off; off += r256(n * sizeof(double));
    p.off_e = off; off += r256(n * sizeof(double));
    p.off_tau = off; off += r256(n * ce);
    p.off_a = off; off += mixed ? r256(nn * ce) : 0;        // single-precision copy of H, then F
    p.dc = n <= DC_MAX_N && (tune.dc < 0 ? n >= DC_DEFAULT_MIN : tune.dc > 0);
    p.off_z = off; off += r256(nn * sizeof(double));
    p.off_lu = off; off += p.dc ? 0 : r256(5 * (size_t)n * TRI_THREADS * sizeof(double));
    p.off_q2 = off; off += p.dc ? r256(nn * sizeof(double)) : 0;
    p.off_u = off; off += p.dc ? r256(nn * sizeof(double)) : 0;
    p.off_rot = off; off += p.dc ? r256((size_t)n * sizeof(DcRot)) : 0;
    p.off_sc = off; off += p.dc ? 256 : 0;
    p.off_x = off; off += r256(nn * ce);
    p.off_t = off; off += r256((p.small_bt ? (size_t)p.nblk16 * ORM_NB * ORM_NB : (size_t)p.nblkbt * p.bt_nb * p.bt_nb) * ce);
    p.off_w = off; off += p.small_bt ? 0 : r256(2 * (size_t)p.bt_nb * n * ce);   // G and W' of a block
    p.off_res = 0;   // (the refinement regions: per2 below)
    p.off_x1 = 0;
    p.off_cl = off; off += mixed ? r256(n * sizeof(int2)) : 0;
    p.off_y = off; off += mixed ? r256((size_t)n * RF_KMAX * sizeof(cplx)) : 0;
    p.off_mu = off; off += mixed ? r256(n * sizeof(double)) : 0;
    p.off_st = off; off += mixed ? r256(3 * (size_t)n * sizeof(double)) : 0;
    p.off_pv = off; off += p.npanels > 0 ? r256(2 * (size_t)p.pw * n * ce) : 0;   // panel V, W
    p.off_q = off; off += p.npanels > 0 ? r256(16) : 0;   // panel queue: claims, abort flag, column counts
    p.per = off;
    p.per2 = mixed ? r256(nn * sizeof(cplx)) : 0;                              // residual R
    p.off2_x1 = p.per2;
    p.per2 += p.refine_steps >= 2 || p.rq ? r256(nn * sizeof(cplx)) : 0;         // step-1 vectors
    return p;
}

// The allocation-free path's configuration: the built-in one with the bisection tridiagonal
// solver, whose scratch sets its order limit.
static HeevPlan noalloc_plan(int n) {
    HeevTune t;
    t.dc = 0;
    return heev_plan(n, false, 2, -1, t);
}

// Bytes of scratch one matrix of order n needs in heev_chunk_on_scratch (double precision).
size_t heev_scratch_bytes_per_matrix(int n) { return noalloc_plan(n).per; }

// Largest chunk of matrices one heev_chunk call may take: the grid y / z extent (65535) of
// the per-matrix launches, and of the (matrix, block) batches of the GEMM back-transformation.
size_t heev_max_chunk(int n) {
    const HeevPlan p = noalloc_plan(n);
    size_t c = 65535;
    if (!p.small_bt) c = std::min<size_t>(c, 65535 / std::max(p.nblkbt, 1));
    return c;
}

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

// Householder tridiagonalisation in the working precision R: blocked panels (k_hetrd_panel +
// rank-2*pw GEMM update) down to order m_tail, then k_hetrd on the leading block.  PV holds
// the panel pairs of the chunk (V of every matrix, then W of every matrix).
template <class R>
static int tridiagonalise(rlmb_context* ctx, cudaStream_t st, const HeevPlan& p, int nb, typename Cx<R>::T* A,
                          double* D, double* E, typename Cx<R>::T* TAU, typename Cx<R>::T* PV, int* Q, int* info,
                          long long* launches) {
    typedef typename Cx<R>::T C;
    const int n = p.n;
    int m = n;
    if (p.npanels > 0) {
        const int pw = p.pw;
        C* PWb = PV + (size_t)nb * pw * n;
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return RLMB_ERR_CUDA;
        // built-in choice above order 512 for chunks of more matrices than SMs: one 512-thread
        // CTA per SM taking (matrix, column) units from a queue (k_hetrd_panel_q)
        const int qnt = p.queue_nt == 256 ? 256 : 512;
        const int qper = qnt == 256 ? 2 : 1;   // resident queue CTAs per SM
        const bool queue = p.panel_nt == 0 && n > 512 && nb > sms &&
                           (qnt == 512 ? panel_smem<512, R>(n) <= 227 * 1024 : panel_smem<256, R>(n) <= 113 * 1024);
        // otherwise one CTA per matrix: 256 threads (two CTAs per SM) for orders 385..512,
        // 512 threads otherwise (measured), unless tuned
        bool mid = n > 384 && n <= 512;
        if (p.panel_nt == 256 && panel_smem<256, R>(n) <= 113 * 1024) mid = true;
        if (p.panel_nt == 512) mid = false;
        auto panel = mid ? k_hetrd_panel<256, R> : k_hetrd_panel<512, R>;
        const int pnt = mid ? 256 : 512;
        const size_t smem = queue ? (qnt == 256 ? panel_smem<256, R>(n) : panel_smem<512, R>(n))
                                  : mid ? panel_smem<256, R>(n) : panel_smem<512, R>(n);
        const void* qk = qnt == 256 ? (const void*)k_hetrd_panel_q<256, R> : (const void*)k_hetrd_panel_q<512, R>;
        if (cudaFuncSetAttribute(queue ? qk : (const void*)panel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return RLMB_ERR_CUDA;
        const int grid = std::min(nb, queue ? qper * sms : sms);
        // the queue's counters, and its abort flag, which k_panel_abort_info reads in every case
        if (cudaMemsetAsync(Q, 0, (8 + (size_t)nb) * sizeof(int), st) != cudaSuccess) return RLMB_ERR_CUDA;
        for (int k = 0; k < p.npanels; ++k) {
            RLMB_CHUNK_PROF("k_hetrd_panel");
            if (queue && qnt == 256)
                k_hetrd_panel_q<256, R><<<grid, 256, smem, st>>>(A, D, E, TAU, PV, PWb, n, m, pw, nb, Q,
                                                                 (long long)k * ((long long)nb * pw + grid),
                                                                 k * pw, info);
            else if (queue)
                k_hetrd_panel_q<512, R><<<grid, 512, smem, st>>>(A, D, E, TAU, PV, PWb, n, m, pw, nb, Q,
                                                                 (long long)k * ((long long)nb * pw + grid),
                                                                 k * pw, info);
            else
                panel<<<nb, pnt, smem, st>>>(A, D, E, TAU, PV, PWb, n, m, pw);
            RLMB_CHUNK_LAUNCHED();
            m -= pw;
            RLMB_CHUNK_PROF("k_hetrd_her2k");
            // (the width a compile-time constant of the operands: their loads are the tile's work)
            const cudaError_t eu =
                pw == 32 ? launch_work_gemm<C, 64>(st, OpPanelA<C, 32>{PV, PWb, n}, OpPanelB<C, 32>{PV, PWb, n},
                                                   EpHer2k<C>{A, n}, m, m, 64, nb)
                         : launch_work_gemm<C, 64>(st, OpPanelA<C, 16>{PV, PWb, n}, OpPanelB<C, 16>{PV, PWb, n},
                                                   EpHer2k<C>{A, n}, m, m, 32, nb);
            if (eu != cudaSuccess)
                return RLMB_ERR_CUDA;
            RLMB_CHUNK_LAUNCHED();
        }
    }
    RLMB_CHUNK_PROF("k_hetrd");
    if (launch_hetrd<R>(p.hc, st, nb, A, D, E, TAU, n, m) != cudaSuccess) return RLMB_ERR_CUDA;
    RLMB_CHUNK_LAUNCHED();
    return RLMB_OK;
}

// After the tridiagonal solve (which writes every matrix's info): a panel queue that ran out
// of its bounded wait marks every matrix of the chunk as failed.
__global__ void k_panel_abort_info(const int* __restrict__ Q, int* __restrict__ info, int nb) {
    if (!*(volatile const int*)(Q + 1)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) info[i] = -1;
}

// Back-transformation X = Q Z in the working precision R (X column-major, column =
// eigenvector): k_larft + k_ormtr, or the blocked GEMM path (Gram GEMM + k_larft64, then
// three GEMMs per block of 64 reflectors).
template <class R>
static int back_transform(rlmb_context* ctx, cudaStream_t st, const HeevPlan& p, int nb,
                          const typename Cx<R>::T* Aw, const typename Cx<R>::T* TAUw, const double* Zw,
                          typename Cx<R>::T* Xw, typename Cx<R>::T* Tw, typename Cx<R>::T* Wp,
                          long long* launches) {
    typedef typename Cx<R>::T C;
    const int n = p.n;
    const size_t nn = (size_t)n * n;
    if (p.small_bt) {
        auto ormtr = p.ch == 16 ? k_ormtr<16, 256, ORM_RPT, R> : p.ch == 8 ? k_ormtr<8, 256, ORM_RPT, R>
                   : p.ch == 4 ? k_ormtr<4, 256, ORM_RPT, R> : p.ch == 2 ? k_ormtr<2, 256, ORM_RPT, R>
                   : k_ormtr<1, 256, ORM_RPT, R>;
        if (cudaFuncSetAttribute(ormtr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_orm) != cudaSuccess)
            return RLMB_ERR_CUDA;
        if (n > 1) {
            RLMB_CHUNK_PROF("k_larft");
            k_larft<R><<<nb, 256, 0, st>>>(Aw, TAUw, Tw, n);
            RLMB_CHUNK_LAUNCHED();
        }
        RLMB_CHUNK_PROF("k_ormtr");
        ormtr<<<dim3((n + p.ch - 1) / p.ch, nb), 256, p.smem_orm, st>>>(Aw, Tw, Zw, Xw, n, p.dbuf);
        RLMB_CHUNK_LAUNCHED();
        return RLMB_OK;
    }
    const int bs = p.bt_nb, nblk = p.nblkbt;
    RLMB_CHUNK_PROF("k_larft");
    if (launch_work_gemm<C, 64>(st, OpBlkReflH<C>{Aw, n, nblk, bs}, OpBlkRefl<C>{Aw, n, nblk, bs},
                            EpStore<C>{Tw, bs, (size_t)bs * bs}, bs, bs, n, nb * nblk) != cudaSuccess)
        return RLMB_ERR_CUDA;
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_larft");
    if (bs == BT_NB) {
        const size_t smem_t = BT_NB * (BT_NB + 1) * sizeof(C);
        if (cudaFuncSetAttribute(k_larft64<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t) != cudaSuccess)
            return RLMB_ERR_CUDA;
        k_larft64<R><<<dim3(nblk, nb), 2 * BT_NB, smem_t, st>>>(TAUw, Tw, n);
    } else {
        const size_t smem_t = 3 * BT_NB * (BT_NB + 1) * sizeof(C);
        if (cudaFuncSetAttribute(k_larft128<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t) != cudaSuccess)
            return RLMB_ERR_CUDA;
        k_larft128<R><<<dim3(nblk, nb), 256, smem_t, st>>>(TAUw, Tw, n);
    }
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ormtr");
    k_z_to_x<C><<<2048, 256, 0, st>>>(Zw, Xw, n, (size_t)nb * nn);
    RLMB_CHUNK_LAUNCHED();
    // per block j of bs reflectors (zlarfb): G = V^H X, W' = T G, X -= V W'; G and W' are
    // [n][bs] per matrix (column c of G at c*bs)
    C* G = Wp;
    C* W2 = Wp + (size_t)nb * bs * n;
    const size_t gs = (size_t)bs * n;
    for (int j = 0; j < nblk; ++j) {
        const int i0 = j * bs;
        const int rows = std::min(i0 + bs - 1, n - 2) + 1;   // rows 0..i1 carry the block
        RLMB_CHUNK_PROF("k_ormtr");
        if (launch_work_gemm<C, 64>(st, OpReflH<C>{Aw, n, i0}, OpColB<C, C>{Xw, n, nn}, EpStore<C>{G, bs, gs},
                                bs, n, rows, nb) != cudaSuccess)
            return RLMB_ERR_CUDA;
        RLMB_CHUNK_LAUNCHED();
        RLMB_CHUNK_PROF("k_ormtr");
        if (launch_work_gemm<C, 64>(st, OpRowA<C, C, false>{Tw + (size_t)j * bs * bs, bs, (size_t)nblk * bs * bs},
                                OpColB<C, C>{G, bs, gs}, EpStore<C>{W2, bs, gs}, bs, n, bs, nb) != cudaSuccess)
            return RLMB_ERR_CUDA;
        RLMB_CHUNK_LAUNCHED();
        RLMB_CHUNK_PROF("k_ormtr");
        // X -= V W': 64-row tiles (two CTAs per SM) on the DMMA engine unless tuned to 128
        // (the tcgen05 engine of the single-precision mode has its own tile)
        const cudaError_t ex =
            p.xtile == 128 ? launch_work_gemm<C, 128>(st, OpRefl<C>{Aw, n, i0}, OpColB<C, C>{W2, bs, gs},
                                                      EpSub<C>{Xw, n}, rows, n, bs, nb)
                           : launch_work_gemm<C, 64>(st, OpRefl<C>{Aw, n, i0}, OpColB<C, C>{W2, bs, gs},
                                                     EpSub<C>{Xw, n}, rows, n, bs, nb);
        if (ex != cudaSuccess) return RLMB_ERR_CUDA;
        RLMB_CHUNK_LAUNCHED();
    }
    return RLMB_OK;
}

// cuTensorMapEncodeTiled, looked up once from the driver through the runtime.
TmaEncodeFn tma_encode_fn() {
    static TmaEncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<TmaEncodeFn>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// Planes of the TMA-fed GEMMs of one refinement chunk: up to 4 GB, at least one matrix.
static int refine_planes(rlmb_context* ctx, int n, int nb) {
    const size_t per = tma_plane_bytes(n, n, n);
    const size_t want = std::max(per, std::min((size_t)nb * per, (size_t)4 << 30));
    return ensure_tma_planes(ctx, want);
}

// One refinement step from the vectors X (single or double) to Out (double, not X).
template <class XT>
static int refine_step(rlmb_context* ctx, cudaStream_t st, int n, int band, int nb, const cplx* A, const XT* X,
                       double* W, cplx* Res, cplxf* F, int2* CL, cplx* YB, double* MU, double* ST,
                       cplx* Out, long long* launches) {
    const size_t nn = (size_t)n * n;
    const unsigned gw = (unsigned)(((size_t)nb * n + 7) / 8);   // one warp per column
    RLMB_CHUNK_PROF("k_ref_resid");
    if (launch_resid<XT>(st, A, X, W, Res, n, band, nb) != cudaSuccess) return RLMB_ERR_CUDA;
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_colstats");
    k_ref_colstats<XT><<<gw, 256, 0, st>>>(X, Res, ST, n, nb);
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_clusters");
    k_ref_clusters<<<(nb + 127) / 128, 128, 0, st>>>(W, ST, CL, n, nb);
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_coupling");
    // E = X^H R on the TMA-fed engine with double-precision accumulation: its error, relative
    // to |X| |R|, is the orthogonality defect the step leaves (F + F^H cancels x_i^H x_j only
    // as well as E is known)
    if (!ctx) return RLMB_ERR_ARG;
    if (int rc = refine_planes(ctx, n, nb)) return rc;
    if (launch_zgemm_tma<cplx>(st, OpRowA<cplx, XT, true>{X, n, nn}, OpColB<cplx, cplx>{Res, n, nn},
                               EpCoupling<XT>{X, W, CL, F, n}, n, n, n, nb, ctx->tws, ctx->tws_bytes) != cudaSuccess)
        return RLMB_ERR_CUDA;
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_cluster");
    {
        const size_t smem_cs = 8 * 3 * RF_KMAX * RF_KMAX * sizeof(cplx);   // 8 warps x (G, S, T)
        if (cudaFuncSetAttribute(k_ref_cluster_solve<XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cs) !=
            cudaSuccess)
            return RLMB_ERR_CUDA;
        // a bounded grid (8 warps per CTA, two CTAs per SM by shared memory) strides over gw warps
        const unsigned grid = (unsigned)std::min<size_t>(gw, 4 * 2 * 148);
        k_ref_cluster_solve<XT><<<grid, 256, smem_cs, st>>>(X, Res, W, CL, YB, MU, n, nb);
    }
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_diag");
    k_ref_diag<<<(unsigned)(((size_t)nb * n + 255) / 256), 256, 0, st>>>(ST, CL, W, F, n, nb);
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_update");
    // X F is a correction of the size of the current error: FP32 sums over K (one drain per
    // tile) carry it to well below the step's target
    if (launch_zgemm_tma<cplxf>(st, OpColA<cplx, XT>{X, n, nn}, OpColB<cplxf, cplxf>{F, n, nn},
                                EpUpdate<XT>{X, Out, n}, n, n, n, nb, ctx->tws, ctx->tws_bytes, false) != cudaSuccess)
        return RLMB_ERR_CUDA;
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_cluster");
    k_ref_cluster_apply<<<gw, 256, 0, st>>>(Out, CL, YB, MU, W, n, nb);
    RLMB_CHUNK_LAUNCHED();
    return RLMB_OK;
}

// w_j <- w_j + Re(x_j^H r_j) / x_j^H x_j for every column: the Rayleigh quotient of x_j, r = H x - x w.
__global__ void k_ref_rq(const double* __restrict__ ST, double* __restrict__ W, size_t total) {
    const size_t gj = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gj < total) W[gj] += ST[3 * gj + 1] / ST[3 * gj];
}

// The eigenvalue pass after one refinement step: residual of the refined double-precision
// vectors X against H (banded for the rlm meshes), column statistics, Rayleigh quotients.
static int rayleigh_pass(cudaStream_t st, int n, int band, int nb, const cplx* A, const cplx* X, double* W,
                         cplx* Res, double* ST, rlmb_context* ctx, long long* launches) {
    const unsigned gw = (unsigned)(((size_t)nb * n + 7) / 8);
    RLMB_CHUNK_PROF("k_ref_resid");
    if (launch_resid<cplx>(st, A, X, W, Res, n, band, nb) != cudaSuccess) return RLMB_ERR_CUDA;
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_colstats");
    k_ref_colstats<cplx><<<gw, 256, 0, st>>>(X, Res, ST, n, nb);
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_ref_diag");
    k_ref_rq<<<(unsigned)(((size_t)nb * n + 255) / 256), 256, 0, st>>>(ST, W, (size_t)nb * n);
    RLMB_CHUNK_LAUNCHED();
    return RLMB_OK;
}

// Eigenvalues W and eigenvectors Z (row-major) of the chunk's tridiagonals (D, E): bisection +
// inverse iteration (k_tridiag), or divide and conquer level by level (k_dc_*), ending in Zw.
static int tridiag_solve(rlmb_context* ctx, cudaStream_t st, const HeevPlan& p, int nb, unsigned char* base,
                         const double* Dw, const double* Ew, double* W, double* Zw, double* LUw, int* info,
                         long long* launches) {
    const int n = p.n;
    const size_t B = (size_t)nb;
    if (!p.dc) {
        RLMB_CHUNK_PROF("k_stebz");
        k_tridiag<1><<<nb, TRI_THREADS, p.smem_tri, st>>>(Dw, Ew, W, Zw, LUw, info, n);
        RLMB_CHUNK_LAUNCHED();
        RLMB_CHUNK_PROF("k_stein");
        k_tridiag<2><<<nb, TRI_THREADS, p.smem_tri, st>>>(Dw, Ew, W, Zw, LUw, info, n);
        RLMB_CHUNK_LAUNCHED();
        return RLMB_OK;
    }
    double* Q2 = reinterpret_cast<double*>(base + p.off_q2 * B);
    double* Uw = reinterpret_cast<double*>(base + p.off_u * B);
    DcRot* Rw = reinterpret_cast<DcRot*>(base + p.off_rot * B);
    double* SCw = reinterpret_cast<double*>(base + p.off_sc * B);
    const int levels = dc_levels(n);
    // ping-pong so that the last level writes Zw
    double* qa = levels % 2 ? Q2 : Zw;
    double* qb = levels % 2 ? Zw : Q2;
    size_t smem_max = 0;   // (not monotone in S: small levels run 16 groups per CTA)
    for (int S = 2; S / 2 < n; S *= 2) smem_max = std::max(smem_max, dc_smem(S, n));
    if (smem_max > 227 * 1024) return RLMB_ERR_ARG;
    if (cudaFuncSetAttribute(k_dc_merge, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max) != cudaSuccess ||
        cudaFuncSetAttribute(k_dc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DgTiles)) !=
            cudaSuccess)
        return RLMB_ERR_CUDA;
    RLMB_CHUNK_PROF("k_dc_merge");
    k_dc_init<<<nb, 256, 0, st>>>(Dw, Ew, W, qa, SCw, info, n);
    RLMB_CHUNK_LAUNCHED();
    for (int S = 2; S / 2 < n; S *= 2) {
        RLMB_CHUNK_PROF("k_dc_merge");
        k_dc_merge<<<nb, DC_THREADS, dc_smem(S, n), st>>>(Ew, SCw, W, qa, qb, Uw, Rw, info, n, S);
        RLMB_CHUNK_LAUNCHED();
        if (S > DC_SMALL) {
            const int nsub = (n + S - 1) / S;
            const int mh = std::min(S / 2, n);
            const dim3 grid((mh + DG_BM - 1) / DG_BM, (std::min(S, n) + DG_BN - 1) / DG_BN, nb * nsub * 2);
            if (grid.z > 65535) return RLMB_ERR_ARG;
            RLMB_CHUNK_PROF("k_dc_gemm");
            k_dc_gemm<<<grid, 256, sizeof(DgTiles), st>>>(qa, Uw, qb, n, S, nsub);
            RLMB_CHUNK_LAUNCHED();
        }
        std::swap(qa, qb);
    }
    RLMB_CHUNK_PROF("k_dc_merge");
    k_dc_finish<<<std::min<size_t>(2048, (B * n + 255) / 256), 256, 0, st>>>(W, SCw, n, B * n);
    RLMB_CHUNK_LAUNCHED();
    return RLMB_OK;
}

// The kernel sequence of one eigensolve chunk of nb matrices of order n on scratch laid out
// per matrix as heev_plan describes (nb * plan.per bytes, no allocation).  Every scratch
// region is written by a kernel before any kernel reads it.  ctx (optional) receives the
// launch count and profile; otherwise *launches is advanced.
static int heev_chunk(rlmb_context* ctx, cudaStream_t st, const HeevPlan& p, cplx* A, double* W, int* info,
                      int nb, void* scratch, int nb2, long long* launches) {
    const int n = p.n;
    unsigned char* base = static_cast<unsigned char*>(scratch);
    const size_t B = (size_t)nb;
    double* Dw = reinterpret_cast<double*>(base + p.off_d * B);
    double* Ew = reinterpret_cast<double*>(base + p.off_e * B);
    double* Zw = reinterpret_cast<double*>(base + p.off_z * B);
    double* LUw = reinterpret_cast<double*>(base + p.off_lu * B);
    int* Qw = reinterpret_cast<int*>(base + p.off_q * B);
    const size_t nn = (size_t)n * n;
    if (p.jacobi) {
        if (p.smem_jac > 227 * 1024) return RLMB_ERR_ARG;
        if (cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_jac) != cudaSuccess)
            return RLMB_ERR_CUDA;
        RLMB_CHUNK_PROF("k_jacobi");
        k_jacobi<<<nb, jacobi_threads(n), p.smem_jac, st>>>(A, W, info, n);
        RLMB_CHUNK_LAUNCHED();
        return RLMB_OK;
    }
    if (p.hc.smem > 227 * 1024 || p.smem_tri > 227 * 1024) return RLMB_ERR_ARG;
    if (cudaFuncSetAttribute(k_tridiag<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_tri) != cudaSuccess ||
        cudaFuncSetAttribute(k_tridiag<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_tri) != cudaSuccess)
        return RLMB_ERR_CUDA;
    if (!p.mixed) {
        cplx* TAUw = reinterpret_cast<cplx*>(base + p.off_tau * B);
        cplx* Xw = reinterpret_cast<cplx*>(base + p.off_x * B);
        cplx* Tw = reinterpret_cast<cplx*>(base + p.off_t * B);
        cplx* Wp = reinterpret_cast<cplx*>(base + p.off_w * B);
        if (int rc = tridiagonalise<double>(ctx, st, p, nb, A, Dw, Ew, TAUw,
                                            reinterpret_cast<cplx*>(base + p.off_pv * B), Qw, info, launches))
            return rc;
        if (int rc = tridiag_solve(ctx, st, p, nb, base, Dw, Ew, W, Zw, LUw, info, launches)) return rc;
        if (info && p.npanels > 0) {
            RLMB_CHUNK_PROF("k_stein");
            k_panel_abort_info<<<(nb + 255) / 256, 256, 0, st>>>(Qw, info, nb);
            RLMB_CHUNK_LAUNCHED();
        }
        if (int rc = back_transform<double>(ctx, st, p, nb, A, TAUw, Zw, Xw, Tw, Wp, launches)) return rc;
        if (cudaMemcpyAsync(A, Xw, B * nn * sizeof(cplx), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return RLMB_ERR_CUDA;
        return RLMB_OK;
    }
    cplxf* TAUw = reinterpret_cast<cplxf*>(base + p.off_tau * B);
    cplxf* As = reinterpret_cast<cplxf*>(base + p.off_a * B);
    cplxf* Xw = reinterpret_cast<cplxf*>(base + p.off_x * B);
    cplxf* Tw = reinterpret_cast<cplxf*>(base + p.off_t * B);
    cplxf* Wp = reinterpret_cast<cplxf*>(base + p.off_w * B);
    // refinement regions for nb2 matrices at a time, after the chunk's regions
    unsigned char* base2 = base + p.per * B;
    cplx* Res = reinterpret_cast<cplx*>(base2);
    cplx* X1 = reinterpret_cast<cplx*>(base2 + p.off2_x1 * (size_t)nb2);
    int2* CL = reinterpret_cast<int2*>(base + p.off_cl * B);
    cplx* YB = reinterpret_cast<cplx*>(base + p.off_y * B);
    double* MU = reinterpret_cast<double*>(base + p.off_mu * B);
    double* ST = reinterpret_cast<double*>(base + p.off_st * B);
    RLMB_CHUNK_PROF("k_herm_fill");
    k_herm_fill<<<dim3((n + 31) / 32, (n + 31) / 32, nb), dim3(32, 8), 0, st>>>(A, n);
    RLMB_CHUNK_LAUNCHED();
    RLMB_CHUNK_PROF("k_to_single");
    k_to_single<<<2048, 256, 0, st>>>(A, As, B * nn);
    RLMB_CHUNK_LAUNCHED();
    if (int rc = tridiagonalise<float>(ctx, st, p, nb, As, Dw, Ew, TAUw,
                                       reinterpret_cast<cplxf*>(base + p.off_pv * B), Qw, info, launches))
        return rc;
    if (int rc = tridiag_solve(ctx, st, p, nb, base, Dw, Ew, W, Zw, LUw, info, launches)) return rc;
    if (info && p.npanels > 0) {
        RLMB_CHUNK_PROF("k_stein");
        k_panel_abort_info<<<(nb + 255) / 256, 256, 0, st>>>(Qw, info, nb);
        RLMB_CHUNK_LAUNCHED();
    }
    if (int rc = back_transform<float>(ctx, st, p, nb, As, TAUw, Zw, Xw, Tw, Wp, launches)) return rc;
    // refinement, nb2 matrices at a time: the single-precision copy of H is free now and
    // holds F.  Step 1 starts from the single-precision vectors, step 2 from step 1's double
    // vectors (X1); the last step writes the caller's buffer (every step's residual reads H
    // first).
    if (nb2 < 1) return RLMB_ERR_ARG;
    for (int m0 = 0; m0 < nb; m0 += nb2) {
        const int ns = std::min(nb2, nb - m0);
        const size_t o = (size_t)m0 * nn, on = (size_t)m0 * n;
        cplx* Am = A + o;
        double* Wm = W + on;
        cplxf* Fm = As + o;
        int2* CLm = CL + on;
        cplx* YBm = YB + (size_t)m0 * n * RF_KMAX;
        double* MUm = MU + on;
        double* STm = ST + 3 * on;
        if (int rc = refine_step<cplxf>(ctx, st, n, p.band, ns, Am, Xw + o, Wm, Res, Fm, CLm, YBm, MUm, STm,
                                        p.refine_steps >= 2 || p.rq ? X1 : Am, launches))
            return rc;
        if (p.rq) {   // eigenvalues as Rayleigh quotients of the step-1 vectors, then the vectors out
            if (int rc = rayleigh_pass(st, n, p.band, ns, Am, X1, Wm, Res, STm, ctx, launches)) return rc;
            if (cudaMemcpyAsync(Am, X1, (size_t)ns * nn * sizeof(cplx), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                return RLMB_ERR_CUDA;
        }
        if (p.refine_steps >= 2)
            if (int rc = refine_step<cplx>(ctx, st, n, p.band, ns, Am, X1, Wm, Res, Fm, CLm, YBm, MUm, STm, Am,
                                           launches))
                return rc;
    }
    return RLMB_OK;
}
#undef RLMB_CHUNK_LAUNCHED
#undef RLMB_CHUNK_PROF

int heev_chunk_on_scratch(cudaStream_t st, cplx* A, double* W, int* info, int n, int nb, void* scratch,
                          long long* launches) {
    return heev_chunk(nullptr, st, noalloc_plan(n), A, W, info, nb, scratch, 0, launches);
}

}  // namespace rlmb

using namespace rlmb;

// ----------------------------------------------------------------------- autotuner
// Per context, per (order, precision): the launch choices of HeevTune picked by timing every
// feasible candidate -- unblocked or blocked reduction (from order 128), 256- or 512-thread
// panels, register-resident or GEMM back-transformation, 64- or 128-reflector blocks and 64- or
// 128-row X-update tiles (double precision) of the latter, either tridiagonal solver (bisection +
// inverse iteration, or divide and conquer), and up to order JAC_MAX_N the batched Jacobi solver -- on copies of up to 2 x SMs of the call's own matrices (at most 2 GB of them),
// each candidate run twice and timed the second time with CUDA events.  Orders
// TUNE_MIN_N .. TUNE_MAX_N are tuned; others keep the built-in choices.
struct TuneEntry {
    HeevTune t;
    double ms_per_matrix;
};
typedef std::map<std::pair<int, int>, TuneEntry> TuneCache;
static TuneCache& tune_cache(rlmb_context* ctx) {
    if (!ctx->tune) ctx->tune = new TuneCache();
    return *static_cast<TuneCache*>(ctx->tune);
}
void rlmb::tune_free(rlmb_context* ctx) {
    delete static_cast<TuneCache*>(ctx->tune);
    ctx->tune = nullptr;
}

static std::vector<HeevTune> tune_candidates(int n, bool mixed) {
    std::vector<HeevTune> out;
    if (n <= JAC_MAX_N) {
        HeevTune t;
        t.jacobi = 1;
        out.push_back(t);
    }
    for (int blocked = 0; blocked <= 1; ++blocked) {
        if (blocked && n < 128) continue;
        for (int gemm = 0; gemm <= 1; ++gemm)
            for (int nt : {256, 512}) {
                if (!blocked && nt == 256) continue;   // no panels: one entry
                for (int xt : {64, 128})
                    for (int bs : {64, 128}) {
                        if ((!gemm || mixed) && xt == 128) continue;
                        if (!gemm && bs == 128) continue;
                        HeevTune t;
                        t.jacobi = 0;
                        t.blocked = blocked;
                        t.gemm_bt = gemm;
                        t.panel_nt = blocked ? nt : 0;
                        t.xtile = gemm && !mixed ? xt : 0;
                        t.bt_nb = gemm ? bs : 0;
                        const HeevPlan p = heev_plan(n, mixed, 2, -1, t);
                        if (!gemm && !p.small_bt) continue;   // register back-transformation does not fit
                        for (int dc = 0; dc <= (n <= DC_MAX_N ? 1 : 0); ++dc) {   // tridiagonal solver
                            t.dc = dc;
                            out.push_back(t);
                        }
                    }
            }
    }
    return out;
}

static int autotune(rlmb_context* ctx, int n, bool mixed, int refine_steps, int band, const cplx* A, int batch,
                    HeevTune* best) {
    int dev = 0, sms = 148;
    RLMB_CUDA_TRY(cudaGetDevice(&dev));
    RLMB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t nn = (size_t)n * n;
    const size_t cap = std::min<size_t>((size_t)2 * sms, ((size_t)2 << 30) / (nn * sizeof(cplx)));
    const int tb = (int)std::max<size_t>(1, std::min<size_t>((size_t)batch, cap));
    const std::vector<HeevTune> cands = tune_candidates(n, mixed);
    size_t per = 0;
    for (const HeevTune& t : cands) {
        const HeevPlan pl = heev_plan(n, mixed, refine_steps, band, t);
        per = std::max(per, pl.per + pl.per2);
    }
    void* buf = nullptr;
    const size_t work = (size_t)tb * (2 * nn * sizeof(cplx) + n * sizeof(double) + sizeof(int)) + 1024;
    if (cudaMalloc(&buf, work) != cudaSuccess) {
        cudaGetLastError();
        return RLMB_ERR_ALLOC;
    }
    if (int rc = ensure_workspace(ctx, (size_t)tb * per)) {
        cudaFree(buf);
        return rc;
    }
    cplx* src = static_cast<cplx*>(buf);
    cplx* wk = src + (size_t)tb * nn;
    double* w = reinterpret_cast<double*>(wk + (size_t)tb * nn);
    int* info = reinterpret_cast<int*>(w + (size_t)tb * n);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = RLMB_OK;
    if (cudaMemcpyAsync(src, A, (size_t)tb * nn * sizeof(cplx), cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        rc = RLMB_ERR_CUDA;
    double best_ms = 1e300;
    long long unused = 0;
    void* prof = ctx->prof;
    ctx->prof = nullptr;   // tuning launches stay out of the caller's profile
    for (size_t c = 0; c < cands.size() && rc == RLMB_OK; ++c) {
        const HeevPlan p = heev_plan(n, mixed, refine_steps, band, cands[c]);
        float ms = 0.f;
        for (int rep = 0; rep < 2 && rc == RLMB_OK; ++rep) {
            if (cudaMemcpyAsync(wk, src, (size_t)tb * nn * sizeof(cplx), cudaMemcpyDeviceToDevice, ctx->stream) !=
                    cudaSuccess ||
                cudaEventRecord(e0, ctx->stream) != cudaSuccess) {
                rc = RLMB_ERR_CUDA;
                break;
            }
            rc = heev_chunk(ctx, ctx->stream, p, wk, w, info, tb, ctx->ws, tb, &unused);
            if (rc == RLMB_OK && (cudaEventRecord(e1, ctx->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                                  cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                rc = RLMB_ERR_CUDA;
        }
        if (rc == RLMB_OK && ms / tb < best_ms) {
            best_ms = ms / tb;
            *best = cands[c];
        }
    }
    ctx->prof = prof;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(buf);
    if (rc == RLMB_OK) tune_cache(ctx)[{n, mixed ? 1 : 0}] = TuneEntry{*best, best_ms};
    return rc;
}

// Refinement steps handed to heev_plan: 1 or 2, or 3 for one step followed by the eigenvalue pass.
static int heev_steps(const rlmb_context* ctx) { return ctx->refine_steps == 1 && ctx->rq_pass ? 3 : ctx->refine_steps; }

// The batched eigensolve of rlmb_heevd_batched with a structure hint: band >= 0 declares every
// matrix a cyclic band of that half-bandwidth (the rlm Hamiltonian), which the mixed mode's
// refinement uses for its residual; band < 0 is a dense matrix.
int rlmb::heevd_batched_band(rlmb_context* ctx, double* d_a, double* d_w, int n, int batch, int* d_info, int band) {
    if (!ctx || !d_a || !d_w || n <= 0 || batch < 0) return RLMB_ERR_ARG;
    if (batch == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    const bool mixed = ctx->precision == RLMB_PRECISION_MIXED;
    HeevTune tune;
    {
        TuneCache& tc = tune_cache(ctx);
        auto it = tc.find({n, mixed ? 1 : 0});
        if (it != tc.end()) {
            tune = it->second.t;
        } else if (ctx->autotune && !ctx->frozen && n >= TUNE_MIN_N && n <= TUNE_MAX_N) {
            if (int rc = autotune(ctx, n, mixed, heev_steps(ctx), band, reinterpret_cast<const cplx*>(d_a), batch, &tune))
                return rc;
        }
    }
    const HeevPlan plan = heev_plan(n, mixed, heev_steps(ctx), band, tune);
    const size_t per = plan.per;
    // workspace: 8 GB, or for large orders enough for two resident matrices per SM (one
    // CTA each in k_tridiag), capped at 60 % of the free memory
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = (size_t)8 << 30;
    }
    const size_t per2 = plan.per2;
    size_t budget = std::max<size_t>((size_t)8 << 30, 2 * 148 * (per + per2));
    budget = std::min<size_t>(budget, free_b / 10 * 6 + ctx->ws_bytes);
    budget = std::max<size_t>(budget, per + per2);
    if (ctx->frozen) budget = std::max<size_t>(per + per2, ctx->ws_bytes);   // capture: the workspace as sized before
    // the refinement regions take up to an eighth of the budget (its GEMMs fill the GPU from a
    // few matrices on); the chunk -- all of whose matrices the one-CTA-per-matrix reduction and
    // tridiagonal kernels run at once -- takes the rest
    size_t nb2 = per2 ? std::max<size_t>(1, std::min<size_t>((size_t)batch, budget / 8 / per2)) : 0;
    size_t chunk = std::max<size_t>(1, std::min<size_t>((budget - nb2 * per2) / per, (size_t)batch));
    chunk = std::min<size_t>(chunk, 65535);   // grid y / z extent of the per-matrix launches
    if (!plan.small_bt) chunk = std::min<size_t>(chunk, 65535 / std::max(plan.nblkbt, 1));   // (matrix, block) batches
    if (plan.dc) chunk = std::min<size_t>(chunk, dc_max_chunk(n));   // (matrix, subproblem, half) GEMM batches
    // equal chunks: a short last chunk would leave most SMs idle in the one-CTA-per-matrix kernels
    const size_t nchunks = (batch + chunk - 1) / chunk;
    chunk = (batch + nchunks - 1) / nchunks;
    if (per2) {   // equal refinement sub-chunks too
        nb2 = std::min(nb2, chunk);
        const size_t nsub = (chunk + nb2 - 1) / nb2;
        nb2 = (chunk + nsub - 1) / nsub;
    }
    if (int rc = ensure_workspace(ctx, chunk * per + nb2 * per2)) return rc;
    const size_t nn = (size_t)n * n;
    long long unused = 0;
    for (size_t b0 = 0; b0 < (size_t)batch; b0 += chunk) {
        const int nb = (int)std::min(chunk, (size_t)batch - b0);
        if (int rc = heev_chunk(ctx, ctx->stream, plan, reinterpret_cast<cplx*>(d_a) + b0 * nn, d_w + b0 * n,
                                d_info ? d_info + b0 : nullptr, nb, ctx->ws, (int)nb2, &unused))
            return rc;
    }
    return RLMB_OK;
}

extern "C" int rlmb_heevd_batched(rlmb_context* ctx, double* d_a, double* d_w, int n, int batch, int* d_info) {
    return rlmb::heevd_batched_band(ctx, d_a, d_w, n, batch, d_info, -1);
}

extern "C" int rlmb_set_autotune(rlmb_context* ctx, int on) {
    if (!ctx) return RLMB_ERR_ARG;
    ctx->autotune = on ? 1 : 0;
    return RLMB_OK;
}

extern "C" int rlmb_heev_config(rlmb_context* ctx, int n, int precision, int* blocked, int* gemm_bt,
                                int* panel_threads, int* x_tile, int* bt_block, double* ms_per_matrix) {
    if (!ctx || n <= 0 || (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED)) return RLMB_ERR_ARG;
    auto& tc = tune_cache(ctx);
    auto it = tc.find({n, precision});
    HeevTune t;
    double ms = 0.0;
    if (it != tc.end()) {
        t = it->second.t;
        ms = it->second.ms_per_matrix;
    }
    const HeevPlan p = heev_plan(n, precision == RLMB_PRECISION_MIXED, 2, -1, t);
    if (blocked) *blocked = p.npanels > 0;
    if (gemm_bt) *gemm_bt = !p.small_bt;
    if (panel_threads) *panel_threads = p.panel_nt;
    if (x_tile) *x_tile = p.xtile == 128 ? 128 : 64;
    if (bt_block) *bt_block = p.bt_nb;
    if (ms_per_matrix) *ms_per_matrix = ms;
    return it != tc.end() ? 1 : 0;
}

extern "C" int rlmb_set_heev_config(rlmb_context* ctx, int n, int precision, int blocked, int gemm_bt,
                                    int panel_threads, int x_tile, int bt_block) {
    if (!ctx || n <= 0 || (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED) || blocked < -1 ||
        blocked > 1 || gemm_bt < -1 || gemm_bt > 1 || (panel_threads != 0 && panel_threads != 256 && panel_threads != 512) ||
        (x_tile != 0 && x_tile != 64 && x_tile != 128) || (bt_block != 0 && bt_block != 64 && bt_block != 128))
        return RLMB_ERR_ARG;
    auto& tc = tune_cache(ctx);
    auto it = tc.find({n, precision});
    HeevTune t;
    if (it != tc.end()) {   // the solver and panel-queue choices are set separately
        t.jacobi = it->second.t.jacobi;
        t.dc = it->second.t.dc;
        t.queue_nt = it->second.t.queue_nt;
        t.panel_w = it->second.t.panel_w;
    }
    t.blocked = blocked;
    t.gemm_bt = gemm_bt;
    t.panel_nt = panel_threads;
    t.xtile = x_tile;
    t.bt_nb = bt_block;
    tc[{n, precision}] = TuneEntry{t, 0.0};
    return RLMB_OK;
}

extern "C" int rlmb_set_heev_solver(rlmb_context* ctx, int n, int precision, int solver) {
    if (!ctx || n <= 0 || (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED) ||
        (solver != RLMB_SOLVER_AUTO && solver != RLMB_SOLVER_HOUSEHOLDER && solver != RLMB_SOLVER_JACOBI) ||
        (solver == RLMB_SOLVER_JACOBI && n > JAC_MAX_N))
        return RLMB_ERR_ARG;
    auto& tc = tune_cache(ctx);
    auto it = tc.find({n, precision});
    TuneEntry e{HeevTune{}, 0.0};
    if (it != tc.end()) e = it->second;
    e.t.jacobi = solver == RLMB_SOLVER_AUTO ? -1 : solver == RLMB_SOLVER_JACOBI ? 1 : 0;
    tc[{n, precision}] = e;
    return RLMB_OK;
}

extern "C" int rlmb_set_panel_queue(rlmb_context* ctx, int n, int precision, int threads) {
    if (!ctx || n <= 0 || (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED) ||
        (threads != 0 && threads != 256 && threads != 512))
        return RLMB_ERR_ARG;
    auto& tc = tune_cache(ctx);
    auto it = tc.find({n, precision});
    TuneEntry e{HeevTune{}, 0.0};
    if (it != tc.end()) e = it->second;
    e.t.queue_nt = threads;
    tc[{n, precision}] = e;
    return RLMB_OK;
}

extern "C" int rlmb_set_panel_width(rlmb_context* ctx, int n, int precision, int width) {
    if (!ctx || n <= 0 || (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED) ||
        (width != 0 && width != 16 && width != 32))
        return RLMB_ERR_ARG;
    auto& tc = tune_cache(ctx);
    auto it = tc.find({n, precision});
    TuneEntry e{HeevTune{}, 0.0};
    if (it != tc.end()) e = it->second;
    e.t.panel_w = width;
    tc[{n, precision}] = e;
    return RLMB_OK;
}

extern "C" int rlmb_set_tridiag_solver(rlmb_context* ctx, int n, int precision, int solver) {
    if (!ctx || n <= 0 || (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED) ||
        (solver != RLMB_TRIDIAG_AUTO && solver != RLMB_TRIDIAG_BISECTION && solver != RLMB_TRIDIAG_DC) ||
        (solver == RLMB_TRIDIAG_DC && n > DC_MAX_N))
        return RLMB_ERR_ARG;
    auto& tc = tune_cache(ctx);
    auto it = tc.find({n, precision});
    TuneEntry e{HeevTune{}, 0.0};
    if (it != tc.end()) e = it->second;
    e.t.dc = solver == RLMB_TRIDIAG_AUTO ? -1 : solver == RLMB_TRIDIAG_DC ? 1 : 0;
    tc[{n, precision}] = e;
    return RLMB_OK;
}

extern "C" int rlmb_tridiag_solver(rlmb_context* ctx, int n, int precision, int* solver) {
    if (!ctx || n <= 0 || !solver || (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED))
        return RLMB_ERR_ARG;
    auto& tc = tune_cache(ctx);
    auto it = tc.find({n, precision});
    const HeevTune t = it != tc.end() ? it->second.t : HeevTune{};
    *solver = heev_plan(n, precision == RLMB_PRECISION_MIXED, 2, -1, t).dc ? RLMB_TRIDIAG_DC : RLMB_TRIDIAG_BISECTION;
    return RLMB_OK;
}

extern "C" int rlmb_heev_solver(rlmb_context* ctx, int n, int precision, int* solver) {
    if (!ctx || n <= 0 || !solver || (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED))
        return RLMB_ERR_ARG;
    auto& tc = tune_cache(ctx);
    auto it = tc.find({n, precision});
    const HeevTune t = it != tc.end() ? it->second.t : HeevTune{};
    *solver = heev_plan(n, precision == RLMB_PRECISION_MIXED, 2, -1, t).jacobi ? RLMB_SOLVER_JACOBI
                                                                              : RLMB_SOLVER_HOUSEHOLDER;
    return RLMB_OK;
}

// Batched complex GEMM C = A B (column-major complex128, A m x k, B k x n, C m x n, matrices
// packed back to back) on either engine: the FP64 tensor path (DMMA) or the tcgen05 TF32
// tensor cores with split operands (FP32-class accuracy).
extern "C" int rlmb_zgemm_batched(rlmb_context* ctx, const double* d_a, const double* d_b, double* d_c, int m,
                                  int n, int k, int batch, int engine) {
    if (!ctx || (k > 0 && (!d_a || !d_b)) || !d_c || m <= 0 || n <= 0 || k < 0 || batch < 0 ||
        (engine != RLMB_GEMM_FP64 && engine != RLMB_GEMM_TF32X3 && engine != RLMB_GEMM_TF32X3_F64ACC))
        return RLMB_ERR_ARG;
    if (batch == 0) return RLMB_OK;
    if (batch > 65535) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    const cplx* A = reinterpret_cast<const cplx*>(d_a);
    const cplx* B = reinterpret_cast<const cplx*>(d_b);
    cplx* Cm = reinterpret_cast<cplx*>(d_c);
    const OpColA<cplx, cplx> la{A, m, (size_t)m * k};
    const OpColB<cplx, cplx> lb{B, k, (size_t)k * n};
    const EpStore<cplx> ep{Cm, m, (size_t)m * n};
    if (engine == RLMB_GEMM_TF32X3_F64ACC && k > 0) {
        const size_t per = tma_plane_bytes(m, n, k);
        if (int rc = ensure_tma_planes(ctx, std::max(per, std::min((size_t)batch * per, (size_t)4 << 30)))) return rc;
    }
    prof_begin(ctx, engine == RLMB_GEMM_FP64 ? "k_zgemm_dmma" : engine == RLMB_GEMM_TF32X3 ? "k_zgemm_tc" : "k_zgemm_tma");
    const cudaError_t e =
        engine == RLMB_GEMM_FP64     ? launch_zgemm<cplx, 64>(ctx->stream, la, lb, ep, m, n, k, batch)
        : engine == RLMB_GEMM_TF32X3 ? launch_zgemm_tc<cplx>(ctx->stream, la, lb, ep, m, n, k, batch)
                                     : launch_zgemm_tma<cplx>(ctx->stream, la, lb, ep, m, n, k, batch, ctx->tws, ctx->tws_bytes);
    prof_end(ctx);
    ctx->launches++;
    return e == cudaSuccess ? RLMB_OK : RLMB_ERR_CUDA;
}

// Number of tcgen05 GEMM tiles whose bounded mbarrier waits ran out since the library was
// loaded on the current device (synchronises the device).
extern "C" int rlmb_tc_fault_count(rlmb_context* ctx, int* count) {
    if (!ctx || !count) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    RLMB_CUDA_TRY(cudaDeviceSynchronize());
    RLMB_CUDA_TRY(cudaMemcpyFromSymbol(count, g_tc_fault, sizeof(int)));
    return RLMB_OK;
}
