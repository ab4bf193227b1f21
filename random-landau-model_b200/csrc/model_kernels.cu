// Assembly and Chern-step kernels of the rlm and hlm twist-mesh pipelines (sm_100a, FP64).
#include "model_kernels.cuh"
#include "small_eig.cuh"

#include <cfloat>
#include <cmath>

namespace rlmb {

// ======================================================================= rlm
// V_mn (rlm/matrix_coefficients.cpp:27-44): the phase of impurity i factorises,
// e^{-i 2pi((m-o)x + (n-o)y)} = e^{-i 2pi (m-o) x} e^{-i 2pi (n-o) y}, so V is a
// (dim x N_imp) by (N_imp x dim) complex product.  One CTA computes a 32x32 tile of
// (m, n) over one chunk of impurities; partial tiles are summed in a fixed order by
// k_vmn_reduce (deterministic).
static constexpr int VMN_T = 32;       // output tile edge
static constexpr int VMN_KC = 32;      // impurities staged per step
static constexpr int VMN_KSPLIT = 2048;  // impurities per CTA

__global__ void __launch_bounds__(256)
k_vmn_partial(const double* __restrict__ X, const double* __restrict__ Y,
              const double* __restrict__ S, int nimp, int dim, int off_head, int nsplit,
              cplx* __restrict__ partial) {
    __shared__ cplx ex[VMN_T][VMN_KC + 1];   // s_i e^{-i 2pi (m-o) x_i}
    __shared__ cplx ey[VMN_T][VMN_KC + 1];   // e^{-i 2pi (n-o) y_i}
    const int tid = threadIdx.x;
    const int m0 = blockIdx.x * VMN_T, n0 = blockIdx.y * VMN_T;
    const int sample = blockIdx.z / nsplit, split = blockIdx.z % nsplit;
    const double* x = X + (size_t)sample * nimp;
    const double* y = Y + (size_t)sample * nimp;
    const double* s = S + (size_t)sample * nimp;
    const int i_begin = split * VMN_KSPLIT, i_end = min(nimp, i_begin + VMN_KSPLIT);
    // thread owns outputs (m0 + tm + 8*u, n0 + tn) for u = 0..3
    const int tn = tid & 31, tm = tid >> 5;
    cplx acc[4] = {mk(0, 0), mk(0, 0), mk(0, 0), mk(0, 0)};
    for (int ib = i_begin; ib < i_end; ib += VMN_KC) {
        __syncthreads();
        for (int idx = tid; idx < VMN_T * VMN_KC; idx += 256) {
            const int r = idx / VMN_KC, k = idx % VMN_KC;
            const int i = ib + k;
            cplx vx = mk(0, 0), vy = mk(0, 0);
            if (i < i_end) {
                double sn, cs;
                sincospi(2.0 * (double)(m0 + r - off_head) * x[i], &sn, &cs);
                vx = mk(cs * s[i], -sn * s[i]);
                sincospi(2.0 * (double)(n0 + r - off_head) * y[i], &sn, &cs);
                vy = mk(cs, -sn);
            }
            ex[r][k] = vx;
            ey[r][k] = vy;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < VMN_KC; ++k) {
            const cplx b = ey[tn][k];
#pragma unroll
            for (int u = 0; u < 4; ++u) cfma(acc[u], ex[tm + 8 * u][k], b);
        }
    }
    for (int u = 0; u < 4; ++u) {
        const int m = m0 + tm + 8 * u, n = n0 + tn;
        if (m < dim && n < dim)
            partial[(((size_t)sample * nsplit + split) * dim + m) * dim + n] = acc[u];
    }
}

__global__ void k_vmn_reduce(const cplx* __restrict__ partial, const cplx* __restrict__ coeff_mn,
                             int dim, int nsplit, int nsamples, cplx* __restrict__ vmn) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t per = (size_t)dim * dim;
    if (idx >= per * nsamples) return;
    const size_t sample = idx / per, mn = idx % per;
    cplx sum = mk(0, 0);
    for (int k = 0; k < nsplit; ++k) sum = cadd(sum, partial[(sample * nsplit + k) * per + mn]);
    vmn[idx] = cmul(sum, coeff_mn[mn]);
}

int launch_rlm_potential(rlmb_context* ctx, const double* x, const double* y, const double* s,
                         int nimp, int nsamples, const cplx* coeff_mn, int dim, int off_head,
                         cplx* partial_ws, cplx* vmn) {
    const int nsplit = (nimp + VMN_KSPLIT - 1) / VMN_KSPLIT;
    const int nt = (dim + VMN_T - 1) / VMN_T;
    dim3 g(nt, nt, nsamples * nsplit);
    prof_begin(ctx, "k_vmn_partial");
    k_vmn_partial<<<g, 256, 0, ctx->stream>>>(x, y, s, nimp, dim, off_head, nsplit, partial_ws);
    RLMB_LAUNCHED(ctx);
    const size_t total = (size_t)dim * dim * nsamples;
    prof_begin(ctx, "k_vmn_reduce");
    k_vmn_reduce<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(partial_ws, coeff_mn, dim,
                                                                          nsplit, nsamples, vmn);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}
size_t rlm_potential_ws_elems(int nimp, int nsamples, int dim) {
    const int nsplit = (nimp + VMN_KSPLIT - 1) / VMN_KSPLIT;
    return (size_t)nsamples * nsplit * dim * dim;
}

// H(theta_1, theta_2) (rlm/hamiltonian_rlm_cpu.cpp:14-48).  For k >= j:
//   F[j][k] = sum_m conj(c_t2[m]) c_jm[j][m] * sum_{n in {o+k-j, o+k-j-N}} V[m][n] c_t1[n]
// stored row-major as the reference does: buf[j*N+k] = F[j][k] (k > j), conj(F[j][j]) on
// the diagonal, buf[k*N+j] = conj(F[j][k]); zero outside the cyclic band.
__device__ __forceinline__ cplx rlm_entry(const cplx* __restrict__ V, const cplx* __restrict__ c1,
                                          const cplx* __restrict__ c2, const cplx* __restrict__ cj,
                                          int n_phi, int dim, int o, int j, int delta) {
    const bool ta = delta <= o, tb = n_phi - delta <= o;
    const int na = o + delta, nb = o + delta - n_phi;
    cplx f = mk(0, 0);
    const cplx g1a = ta ? c1[na] : mk(0, 0);
    const cplx g1b = tb ? c1[nb] : mk(0, 0);
    for (int m = 0; m < dim; ++m) {
        cplx t = mk(0, 0);
        if (ta) cfma(t, V[m * dim + na], g1a);
        if (tb) cfma(t, V[m * dim + nb], g1b);
        const cplx p = cmulc(c2[m], cj[j * dim + m]);   // conj(c_t2[m]) * c_jm[j][m]
        cfma(f, t, p);
    }
    return f;
}

__global__ void __launch_bounds__(256)
k_rlm_assemble(const cplx* __restrict__ vmn, const cplx* __restrict__ cmt, const cplx* __restrict__ cjm,
               const int* __restrict__ t1s, const int* __restrict__ t2s, int n_phi, int dim, int o,
               int samples_stride_kpts, cplx* __restrict__ H) {
    const int kp = blockIdx.y;
    const int sample = kp / samples_stride_kpts;
    const cplx* V = vmn + (size_t)sample * dim * dim;
    const cplx* c1 = cmt + (size_t)t1s[kp] * dim;
    const cplx* c2 = cmt + (size_t)t2s[kp] * dim;
    cplx* h = H + (size_t)kp * n_phi * n_phi;
    const size_t nn = (size_t)n_phi * n_phi;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < nn;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / n_phi), k = (int)(idx % n_phi);   // buf[j*N + k]
        const int lo = min(j, k), hi = max(j, k);
        const int delta = hi - lo;
        cplx val = mk(0, 0);
        if (delta <= o || n_phi - delta <= o) {
            const cplx f = rlm_entry(V, c1, c2, cjm, n_phi, dim, o, lo, delta);
            val = (k > j) ? f : cconj(f);
        }
        h[idx] = val;
    }
}

int launch_rlm_assemble(rlmb_context* ctx, const cplx* vmn, const cplx* cmt, const cplx* cjm,
                        const int* d_t1, const int* d_t2, int count, int kpts_per_sample,
                        int n_phi, int dim, int o, cplx* H) {
    const size_t nn = (size_t)n_phi * n_phi;
    const int bx = (int)std::min<size_t>((nn + 255) / 256, 1024);
    dim3 g(bx, count);
    prof_begin(ctx, "k_rlm_assemble");
    k_rlm_assemble<<<g, 256, 0, ctx->stream>>>(vmn, cmt, cjm, d_t1, d_t2, n_phi, dim, o,
                                               kpts_per_sample, H);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// rlm links: U1(t1,t2) = <u_n(t1,t2)|u_n(t1+1,t2)>, U2(t1,t2) = <u_n(t1,t2)|u_n(t1,t2+1)>
// on the full (g+1)^2 mesh of one sample, eigenvector n of k-point t at X[(t*N + n)*N].
__global__ void __launch_bounds__(256)
k_rlm_links(const cplx* __restrict__ X, int n_phi, int g, cplx* __restrict__ U1, cplx* __restrict__ U2) {
    const int kpt = blockIdx.y;                 // sample * (g+1)^2 + t1*(g+1) + t2
    const int per = (g + 1) * (g + 1);
    const int sample = kpt / per, t = kpt % per, t1 = t / (g + 1), t2 = t % (g + 1);
    const int lane = threadIdx.x & 31;
    const int state = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (state >= n_phi) return;
    const size_t nn = (size_t)n_phi * n_phi;
    const cplx* a = X + (size_t)kpt * nn + (size_t)state * n_phi;
    const cplx* b1 = t1 < g ? a + (size_t)(g + 1) * nn : nullptr;
    const cplx* b2 = t2 < g ? a + nn : nullptr;
    cplx s1 = mk(0, 0), s2 = mk(0, 0);
    for (int r = lane; r < n_phi; r += 32) {
        const cplx av = a[r];
        if (b1) cfmac(s1, av, b1[r]);
        if (b2) cfmac(s2, av, b2[r]);
    }
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    if (lane == 0) {
        const size_t o = ((size_t)sample * per + t) * n_phi + state;
        U1[o] = b1 ? s1 : mk(1.0, 0.0);
        U2[o] = b2 ? s2 : mk(1.0, 0.0);
    }
}

int launch_rlm_links(rlmb_context* ctx, const cplx* X, int n_phi, int g, int nsamples, cplx* U1, cplx* U2) {
    dim3 grid((n_phi + 7) / 8, nsamples * (g + 1) * (g + 1));
    prof_begin(ctx, "k_rlm_links");
    k_rlm_links<<<grid, 256, 0, ctx->stream>>>(X, n_phi, g, U1, U2);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// Plaquette phases and sample accumulation (rlm/main_rlm_cpu.cpp:155-158,187-190,230-239;
// hlm/main_hlm_cpu.cpp:111-115,143-147,184-187; diag_wrappers/chern.cpp:47-72).
// Mesh arrays are [sample][t1 (g+1)][t2 (n2)][N]; for hlm n2 = g and slot g of a line is
// the periodic copy of slot 0.  Plaquette (line L = 1..g, m = 0..g-1):
//   prod = U1(L-1,m) * U2(L,m) * conj(U1(L-1,m+1)) * conj(U2(L-1,m))
// contributes -arg(prod)/2pi (rlm, then + 1/N) or +arg(prod)/2pi (hlm).
__global__ void k_plaquettes(const cplx* __restrict__ U1, const cplx* __restrict__ U2,
                             const double* __restrict__ W, int n_phi, int g, int nsamples,
                             int hlm, double* __restrict__ energies, double* __restrict__ chern) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n_phi * nsamples) return;
    const int sample = idx / n_phi, n = idx % n_phi;
    const int n2 = hlm ? g : g + 1;
    const size_t base = (size_t)sample * (g + 1) * n2;
    auto at = [&](int t1, int t2) -> size_t {
        if (hlm && t2 == g) t2 = 0;
        return (base + (size_t)t1 * n2 + t2) * n_phi + n;
    };
    double c = 0.0;
    for (int L = 1; L <= g; ++L) {
        double line = 0.0;
        for (int m = 0; m < g; ++m) {
            cplx prod = mk(1.0, 0.0);
            prod = cmul(prod, U1[at(L - 1, m)]);
            prod = cmul(prod, U2[at(L, m)]);
            prod = cmul(prod, cconj(U1[at(L - 1, m + 1)]));
            prod = cmul(prod, cconj(U2[at(L - 1, m)]));
            line += -atan2(prod.y, prod.x) / (M_PI * 2.0);
        }
        c += hlm ? -line : line;
    }
    double e = 0.0;
    for (int t1 = 0; t1 <= g; ++t1) {
        for (int t2 = 0; t2 < n2; ++t2) e += W[at(t1, t2)];
        if (hlm) e += W[at(t1, 0)];
    }
    energies[idx] = e / ((double)(g + 1) * (g + 1));
    chern[idx] = hlm ? c : c + 1.0 / n_phi;
}

int launch_plaquettes(rlmb_context* ctx, const cplx* U1, const cplx* U2, const double* W, int n_phi,
                      int g, int nsamples, int hlm, double* energies, double* chern) {
    const int total = n_phi * nsamples;
    prof_begin(ctx, "k_plaquettes");
    k_plaquettes<<<(total + 127) / 128, 128, 0, ctx->stream>>>(U1, U2, W, n_phi, g, nsamples, hlm,
                                                              energies, chern);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// Reference-layout FHS for one line pair (diag_wrappers/chern.cpp:3-75): prev/cur hold
// (g+1) k-points of N states of length dim_vec; out[m + n*g] = -arg(prod)/2pi.
__global__ void __launch_bounds__(256)
k_fhs_line(const cplx* __restrict__ prev, const cplx* __restrict__ cur, int n_phi, int dim_vec,
           int g, double* __restrict__ out) {
    const int m = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const int n = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (n >= n_phi) return;
    const size_t kstride = (size_t)n_phi * dim_vec;
    const cplx* pm = prev + (size_t)m * kstride + (size_t)n * dim_vec;
    const cplx* pm1 = pm + kstride;
    const cplx* cm = cur + (size_t)m * kstride + (size_t)n * dim_vec;
    const cplx* cm1 = cm + kstride;
    cplx l0 = mk(0, 0), l1 = mk(0, 0), l2 = mk(0, 0), l3 = mk(0, 0);
    for (int r = lane; r < dim_vec; r += 32) {
        const cplx a = pm[r], b = cm[r], c = cm1[r], d = pm1[r];
        cfmac(l0, a, b);   // <prev,m | cur,m>
        cfmac(l1, b, c);   // <cur,m | cur,m+1>
        cfmac(l2, c, d);   // <cur,m+1 | prev,m+1>
        cfmac(l3, d, a);   // <prev,m+1 | prev,m>
    }
    l0 = warp_sum(l0);
    l1 = warp_sum(l1);
    l2 = warp_sum(l2);
    l3 = warp_sum(l3);
    if (lane == 0) {
        cplx prod = mk(1.0, 0.0);
        prod = cmul(prod, l0);
        prod = cmul(prod, l1);
        prod = cmul(prod, l2);
        prod = cmul(prod, l3);
        out[m + (size_t)n * g] = -atan2(prod.y, prod.x) / (M_PI * 2.0);
    }
}

int launch_fhs_line(rlmb_context* ctx, const cplx* prev, const cplx* cur, int n_phi, int dim_vec,
                    int g, double* out) {
    dim3 grid((n_phi + 7) / 8, g);
    prof_begin(ctx, "k_fhs_line");
    k_fhs_line<<<grid, 256, 0, ctx->stream>>>(prev, cur, n_phi, dim_vec, g, out);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// ======================================================================= hlm
// Clean Bloch vectors (hlm/hamiltonian_hlm_cpu.cpp:18-51).  For each k-point t of the
// mesh (t1 in [0,g], t2 in [0,g)) and Bloch index c = kx*ly + ky: the Q x Q Harper matrix
// exactly as the reference writes its column-major array (:25-32), diagonalised by
// cyclic complex Jacobi rotations, band `band` of the ascending spectrum, scaled by
// 1/sqrt(N |h|^2) -- the norm of the full plane-wave column (:43-51).
__global__ void k_hlm_bloch(int lx, int ly, int Q, int band, int g, int t1_0, int t1_1, int t2_0,
                            int t2_1, cplx* __restrict__ hb) {
    const int Lxp = lx / Q, N = Lxp * ly;
    const int n2 = t2_1 - t2_0;
    const long total = (long)(t1_1 - t1_0) * n2 * N;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % N);
    const int t = (int)(idx / N);
    const int t1 = t1_0 + t / n2, t2 = t2_0 + t % n2;
    const int kx = c / ly, ky = c % ly;
    const double inv_g = 1.0 / g, pi2 = 2.0 * M_PI;
    const double kxs = kx + t1 * inv_g, kys = ky + t2 * inv_g;
    cplx a[RLMB_MAX_Q * RLMB_MAX_Q];   // column-major [r + c*Q]
    cplx v[RLMB_MAX_Q * RLMB_MAX_Q];
    for (int i = 0; i < Q * Q; ++i) a[i] = mk(0, 0);
    const double inv_Q = 1.0 / Q;
    for (int p = 0; p < Q; ++p) {
        a[p * Q + p] = mk(-2.0 * cos(kys * (pi2 / ly) + pi2 * p * inv_Q), 0.0);
        if (p + 1 < Q) a[p * Q + p + 1] = a[(p + 1) * Q + p] = mk(-1.0, 0.0);
    }
    const double ph = kxs * Q * (pi2 / lx);
    a[Q * (Q - 1)] = mk(-cos(ph), -sin(ph));
    a[Q - 1] = cconj(a[Q * (Q - 1)]);
    // heevd reads the upper triangle (col-major): A[r][c] = a[r + c*Q], r <= c
    for (int cc = 0; cc < Q; ++cc)
        for (int r = 0; r < Q; ++r) {
            if (r < cc) a[cc + r * Q] = cconj(a[r + cc * Q]);
            else if (r == cc) a[r + cc * Q].y = 0.0;
        }
    for (int i = 0; i < Q * Q; ++i) v[i] = mk(i % (Q + 1) == 0 ? 1.0 : 0.0, 0.0);
    herm_jacobi(a, v, Q);
    // eigenvector of the band-th smallest eigenvalue
    int order[RLMB_MAX_Q];
    for (int i = 0; i < Q; ++i) order[i] = i;
    for (int i = 1; i < Q; ++i)
        for (int j = i; j > 0 && a[order[j] * (Q + 1)].x < a[order[j - 1] * (Q + 1)].x; --j) {
            const int tmp = order[j];
            order[j] = order[j - 1];
            order[j - 1] = tmp;
        }
    const int col = order[band];
    double h2 = 0.0;
    for (int q = 0; q < Q; ++q) h2 += cabs2(v[q + col * Q]);
    const double sc = 1.0 / sqrt((double)N * h2);
    cplx* out = hb + ((size_t)t * N + c) * Q;
    for (int q = 0; q < Q; ++q) out[q] = cscale(v[q + col * Q], sc);
}

int launch_hlm_bloch(rlmb_context* ctx, int lx, int ly, int Q, int band, int g, int t1_0, int t1_1,
                     int t2_0, int t2_1, cplx* hb) {
    const int N = lx * ly / Q;
    const long total = (long)(t1_1 - t1_0) * (t2_1 - t2_0) * N;
    prof_begin(ctx, "k_hlm_bloch");
    k_hlm_bloch<<<(unsigned)((total + 127) / 128), 128, 0, ctx->stream>>>(lx, ly, Q, band, g, t1_0,
                                                                         t1_1, t2_0, t2_1, hb);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// Full basis column W(r, c) = e^{-i phi_c(r)} hhat_c[q(r)] (hlm/hamiltonian_hlm_cpu.cpp:37-42)
__global__ void k_hlm_basis_expand(const cplx* __restrict__ hb, int lx, int ly, int Q, int g, int t1,
                                   int t2, cplx* __restrict__ W) {
    const int Lxp = lx / Q, N = Lxp * ly, ns = lx * ly;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)N * ns) return;
    const int c = (int)(idx / ns), r = (int)(idx % ns);
    const int kx = c / ly, ky = c % ly;
    const int j = r / lx, xm = r % lx, q = xm % Q, m = xm - q;
    const double inv_g = 1.0 / g, pi2 = 2.0 * M_PI;
    const double kxs = kx + t1 * inv_g, kys = ky + t2 * inv_g;
    const double phase = kxs * (pi2 / lx) * m + kys * (pi2 / ly) * j;
    double sn, cs;
    sincos(phase, &sn, &cs);
    W[idx] = cmul(mk(cs, -sn), hb[(size_t)c * Q + q]);
}

int launch_hlm_basis_expand(rlmb_context* ctx, const cplx* hb, int lx, int ly, int Q, int g, int t1,
                            int t2, cplx* W) {
    const long total = (long)(lx * ly / Q) * lx * ly;
    prof_begin(ctx, "k_hlm_basis_expand");
    k_hlm_basis_expand<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(hb, lx, ly, Q, g, t1, t2, W);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// Sublattice Fourier transform of the on-site potential (one sample per blockIdx.y):
//   Vt[q][dx][dy] = sum_{m'<Lx', j<ly} V[j*lx + Q m' + q] e^{+i 2pi (dx m'/Lx' + dy j/ly)}
// so that W^H diag(V) W [a][b] = sum_q conj(hhat_a[q]) hhat_b[q] Vt[q][kxa-kxb][kya-kyb]:
// the twist phases of the two columns cancel in the difference.
__global__ void k_hlm_vtilde(const double* __restrict__ pot, int lx, int ly, int Q, cplx* __restrict__ vt) {
    const int Lxp = lx / Q, N = Lxp * ly, ns = lx * ly;
    const int sample = blockIdx.y;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ns) return;
    const int q = idx / N, rest = idx % N, dx = rest / ly, dy = rest % ly;
    const double* V = pot + (size_t)sample * ns;
    cplx acc = mk(0, 0);
    for (int mp = 0; mp < Lxp; ++mp) {
        const int fx = (dx * mp) % Lxp;
        for (int j = 0; j < ly; ++j) {
            const int fy = (dy * j) % ly;
            // exact fraction fx/Lxp + fy/ly, taken through sincospi
            const double f = 2.0 * ((double)fx / Lxp + (double)fy / ly);
            double sn, cs;
            sincospi(f, &sn, &cs);
            const double val = V[j * lx + Q * mp + q];
            acc.x = fma(val, cs, acc.x);
            acc.y = fma(val, sn, acc.y);
        }
    }
    vt[(size_t)sample * ns + idx] = acc;
}

int launch_hlm_vtilde(rlmb_context* ctx, const double* pot, int lx, int ly, int Q, int nsamples, cplx* vt) {
    const int ns = lx * ly;
    dim3 grid((ns + 127) / 128, nsamples);
    prof_begin(ctx, "k_hlm_vtilde");
    k_hlm_vtilde<<<grid, 128, 0, ctx->stream>>>(pot, lx, ly, Q, vt);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// Projected H of k-point (sample, t) into column-major buf[b*N + a] = H[a][b].
// blockIdx.y = sample * kpts + k, kpts = number of mesh k-points given in tlist.
// Thread = row a (its Bloch indices and hhat_a held in registers); the CTA's x-slice of the
// columns b is walked in order, so consecutive threads store consecutive entries of a
// column (coalesced) and every per-b quantity is a warp-uniform shared-memory broadcast.
// The sublattice offsets (kxa - kxb) mod Lx', (kya - kyb) mod ly advance by wrap-around
// subtraction instead of integer division.  QT: the flux denominator Q as a compile-time
// constant (hhat_a in registers), or 0 for the generic form (hhat_a re-read from shared
// memory).
template <int QT>
__global__ void __launch_bounds__(256)
k_hlm_project(const cplx* __restrict__ hb, const cplx* __restrict__ vt, const int* __restrict__ tlist,
              int lx, int ly, int Qr, int kpts, cplx* __restrict__ H) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Q = QT > 0 ? QT : Qr;
    const int Lxp = lx / Q, N = Lxp * ly, ns = lx * ly;
    cplx* sh = reinterpret_cast<cplx*>(smem_raw);   // [N*Q] hhat of this k-point
    cplx* sv = sh + (size_t)N * Q;                   // [ns]  Vt of this sample
    const int job = blockIdx.y;
    const int sample = job / kpts, k = job % kpts;
    const int t = tlist[k];
    for (int i = threadIdx.x; i < N * Q; i += blockDim.x) sh[i] = hb[(size_t)t * N * Q + i];
    for (int i = threadIdx.x; i < ns; i += blockDim.x) sv[i] = vt[(size_t)sample * ns + i];
    __syncthreads();
    cplx* h = H + (size_t)job * N * N;
    // columns of this CTA: [b0, b1)
    const int per = (N + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * per, b1 = min(N, b0 + per);
    if (b0 >= b1) return;
    for (int a = threadIdx.x; a < N; a += blockDim.x) {
        const int kxa = a / ly, kya = a % ly;
        constexpr int QR = QT > 0 ? QT : 1;
        cplx ha[QR];
#pragma unroll
        for (int q = 0; q < QR; ++q) ha[q] = cconj(sh[a * Q + q]);
        const int kxb = b0 / ly, kyb0 = b0 % ly;
        int kyb = kyb0;
        int dx = kxa - kxb;
        if (dx < 0) dx += Lxp;
        int dy = kya - kyb;
        if (dy < 0) dy += ly;
        for (int b = b0; b < b1; ++b) {
            cplx acc = mk(0, 0);
            const cplx* hbq = sh + b * Q;
            if constexpr (QT > 0) {
#pragma unroll
                for (int q = 0; q < QT; ++q) cfma(acc, cmul(ha[q], hbq[q]), sv[(q * Lxp + dx) * ly + dy]);
            } else {
                for (int q = 0; q < Q; ++q)
                    cfma(acc, cmul(cconj(sh[a * Q + q]), hbq[q]), sv[(q * Lxp + dx) * ly + dy]);
            }
            h[(size_t)b * N + a] = acc;
            // next column: kyb + 1 (wrapping into kxb + 1)
            if (++kyb == ly) {
                kyb = 0;
                dy = kya;
                if (--dx < 0) dx += Lxp;
            } else if (--dy < 0) {
                dy += ly;
            }
        }
    }
}

int launch_hlm_project(rlmb_context* ctx, const cplx* hb, const cplx* vt, const int* d_tlist, int lx,
                       int ly, int Q, int kpts, int nsamples, cplx* H) {
    const int N = lx * ly / Q;
    const size_t smem = ((size_t)N * Q + (size_t)lx * ly) * sizeof(cplx);
    if (smem > 200 * 1024) return RLMB_ERR_ARG;
    auto kern = Q == 1 ? k_hlm_project<1> : Q == 2 ? k_hlm_project<2> : Q == 3 ? k_hlm_project<3>
              : Q == 4 ? k_hlm_project<4> : k_hlm_project<0>;
    RLMB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int bx = std::max(1, std::min(N / 32, 16));   // column slices of >= 32 columns per k-point
    dim3 grid(bx, kpts * nsamples);
    prof_begin(ctx, "k_hlm_project");
    kern<<<grid, 256, smem, ctx->stream>>>(hb, vt, d_tlist, lx, ly, Q, kpts, H);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// hlm link overlaps from the eigenvectors U of the projected problems, without forming
// the n_sites-long states W U (hlm/hamiltonian_hlm_cpu.cpp:180):
//   <psi_n(a)|psi_n(b)> = U_n(a)^H S U_n(b),  S = W(a)^H W(b).
// S is block diagonal: theta_2 links (same t1) couple equal kx only,
//   S[(kx,ky),(kx,ky')] = Lx' D_ly(ky - ky' + (t2 - t2')/g) <hhat|hhat'>,
// theta_1 links (same t2) couple equal ky only,
//   S[(kx,ky),(kx',ky)] = ly D_Lx'(kx - kx' + (t1 - t1')/g) <hhat|hhat'>,
// with D_L(s) = sum_{j<L} e^{i 2pi s j / L}.  The theta_2 = g neighbour is the periodic
// copy of theta_2 = 0 (hlm/main_hlm_cpu.cpp:149-150).
// blockIdx.x = state chunk, blockIdx.y = sample*kpts + t (t = t1*g + t2), blockIdx.z = dir.
static constexpr int LINK_STATES = 16;

__global__ void __launch_bounds__(256)
k_hlm_links_generic(const cplx* __restrict__ hb, const cplx* __restrict__ X, int lx, int ly, int Q, int g,
            cplx* __restrict__ U1, cplx* __restrict__ U2) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Lxp = lx / Q, N = Lxp * ly;
    const int dir = blockIdx.y;                       // 0: theta_1 link, 1: theta_2 link
    const int kpts = (g + 1) * g;
    const int job = blockIdx.x, sample = job / kpts, t = job % kpts;
    const int t1 = t / g, t2 = t % g;
    if (dir == 0 && t1 == g) return;                  // no theta_1 neighbour of the last line
    const int L = dir == 0 ? Lxp : ly;                // block size
    const int tb1 = dir == 0 ? t1 + 1 : t1;
    const int tb2 = dir == 0 ? t2 : (t2 + 1 == g ? 0 : t2 + 1);
    const int tb = tb1 * g + tb2;
    // theta offset (t - t') / g entering D: theta_1 link: -1/g; theta_2 link: (t2 - t2')/g
    const double shift = dir == 0 ? -1.0 / g : (double)(t2 - tb2) / g;
    cplx* S = reinterpret_cast<cplx*>(smem_raw);      // [N][L]: S[a][l], b = partner l of a
    cplx* ub = S + (size_t)N * L;                     // [LINK_STATES][N]
    __shared__ cplx Dtab[64];
    __shared__ cplx red[8][LINK_STATES];
    for (int dlt = threadIdx.x; dlt < L; dlt += blockDim.x) {
        // D_L(dlt + shift), dlt = (index difference) mod L
        cplx acc = mk(0, 0);
        for (int j = 0; j < L; ++j) {
            double sn, cs;
            sincospi(2.0 * (dlt + shift) * j / L, &sn, &cs);
            acc = cadd(acc, mk(cs, sn));
        }
        Dtab[dlt] = acc;
    }
    __syncthreads();
    // Bloch tables cover the (g+1) x (g+1) mesh: index t1*(g+1) + t2
    const cplx* ha = hb + ((size_t)t1 * (g + 1) + t2) * N * Q;
    const cplx* hbb = hb + ((size_t)tb1 * (g + 1) + tb2) * N * Q;
    const double pref = dir == 0 ? (double)ly : (double)Lxp;
    for (int idx = threadIdx.x; idx < N * L; idx += blockDim.x) {
        const int a = idx / L, l = idx % L;
        const int kxa = a / ly, kya = a % ly;
        int b, dlt;
        if (dir == 0) { b = l * ly + kya; dlt = (kxa - l + Lxp) % Lxp; }
        else { b = kxa * ly + l; dlt = (kya - l + ly) % ly; }
        cplx ov = mk(0, 0);
        for (int q = 0; q < Q; ++q) cfmac(ov, ha[(size_t)a * Q + q], hbb[(size_t)b * Q + q]);
        S[idx] = cscale(cmul(Dtab[dlt], ov), pref);
    }
    const size_t nn = (size_t)N * N;
    const cplx* Xa = X + ((size_t)sample * kpts + t) * nn;
    const cplx* Xb = X + ((size_t)sample * kpts + tb) * nn;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int s0 = 0; s0 < N; s0 += LINK_STATES) {
        const int ns = min(LINK_STATES, N - s0);
        __syncthreads();
        for (int i = threadIdx.x; i < LINK_STATES * N; i += blockDim.x) {
            const int s = i / N, bidx = i % N;
            ub[i] = s < ns ? Xb[(size_t)(s0 + s) * N + bidx] : mk(0, 0);
        }
        __syncthreads();
        cplx part[LINK_STATES];
#pragma unroll
        for (int s = 0; s < LINK_STATES; ++s) part[s] = mk(0, 0);
        for (int a = threadIdx.x; a < N; a += blockDim.x) {
            const int kxa = a / ly, kya = a % ly;
            const cplx* Sa = S + (size_t)a * L;
#pragma unroll
            for (int s = 0; s < LINK_STATES; ++s) {
                if (s < ns) {
                    cplx y = mk(0, 0);
                    for (int l = 0; l < L; ++l) {
                        const int b = dir == 0 ? l * ly + kya : kxa * ly + l;
                        cfma(y, Sa[l], ub[s * N + b]);
                    }
                    cfmac(part[s], Xa[(size_t)(s0 + s) * N + a], y);
                }
            }
        }
#pragma unroll
        for (int s = 0; s < LINK_STATES; ++s) {
            const cplx v = warp_sum(part[s]);
            if (lane == 0) red[w][s] = v;
        }
        __syncthreads();
        if (threadIdx.x < ns) {
            cplx tot = mk(0, 0);
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot = cadd(tot, red[i][threadIdx.x]);
            const size_t o = ((size_t)sample * kpts + t) * N + s0 + threadIdx.x;
            if (dir == 0) U1[o] = tot; else U2[o] = tot;
        }
    }
}

int launch_hlm_links_generic(rlmb_context* ctx, const cplx* hb, const cplx* X, int lx, int ly, int Q, int g,
                     int nsamples, cplx* U1, cplx* U2) {
    const int N = lx * ly / Q;
    const int Lmax = std::max(lx / Q, ly);
    if (Lmax > 64) return RLMB_ERR_ARG;
    const size_t smem = ((size_t)N * Lmax + (size_t)LINK_STATES * N) * sizeof(cplx);
    if (smem > 200 * 1024) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaFuncSetAttribute(k_hlm_links_generic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid(nsamples * (g + 1) * g, 2);
    prof_begin(ctx, "k_hlm_links_generic");
    k_hlm_links_generic<<<grid, 256, smem, ctx->stream>>>(hb, X, lx, ly, Q, g, U1, U2);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// One CTA per (sample, k-point t): both links of t.  S blocks of the two directions are
// built once in shared memory; thread = state n, which loads one Bloch block of U'(n) into
// registers and reuses it for the block's L rows (S entries are warp-uniform broadcasts).
static constexpr int LINK_MAXL = 32;

template <int L>
__device__ __forceinline__ cplx link_dir(const cplx* __restrict__ S, const cplx* __restrict__ ua,
                                         const cplx* __restrict__ ub, int nblk, int ly, int dir) {
    // blocks: dir 1 (theta_2) -> block kx, rows a = kx*ly + i, partners kx*ly + l;
    //         dir 0 (theta_1) -> block ky, rows a = i*ly + ky, partners l*ly + ky.
    cplx acc = mk(0, 0);
    for (int beta = 0; beta < nblk; ++beta) {
        cplx u[L];
#pragma unroll
        for (int l = 0; l < L; ++l) u[l] = ub[dir ? beta * ly + l : l * ly + beta];
#pragma unroll 2
        for (int i = 0; i < L; ++i) {
            const int a = dir ? beta * ly + i : i * ly + beta;
            const cplx* Sa = S + (size_t)a * L;
            cplx y = mk(0, 0);
#pragma unroll
            for (int l = 0; l < L; ++l) cfma(y, Sa[l], u[l]);
            cfmac(acc, ua[a], y);
        }
    }
    return acc;
}

__device__ void build_link_S(cplx* S, cplx* Dtab, const cplx* __restrict__ ha, const cplx* __restrict__ hbb,
                             int N, int L, int ly, int Lxp, int Q, int dir, double shift, bool transposed = false) {
    for (int dlt = threadIdx.x; dlt < L; dlt += blockDim.x) {
        // D_L(dlt + shift) = sum_j e^{i 2pi (dlt + shift) j / L}, dlt = index difference mod L
        cplx acc = mk(0, 0);
        for (int j = 0; j < L; ++j) {
            double sn, cs;
            sincospi(2.0 * (dlt + shift) * j / L, &sn, &cs);
            acc = cadd(acc, mk(cs, sn));
        }
        Dtab[dlt] = acc;
    }
    __syncthreads();
    const double pref = dir == 0 ? (double)ly : (double)Lxp;
    for (int idx = threadIdx.x; idx < N * L; idx += blockDim.x) {
        const int a = idx / L, l = idx % L;
        const int kxa = a / ly, kya = a % ly;
        int b, dlt;
        if (dir == 0) { b = l * ly + kya; dlt = (kxa - l + Lxp) % Lxp; }
        else { b = kxa * ly + l; dlt = (kya - l + ly) % ly; }
        cplx ov = mk(0, 0);
        for (int q = 0; q < Q; ++q) cfmac(ov, ha[(size_t)a * Q + q], hbb[(size_t)b * Q + q]);
        S[transposed ? (size_t)l * N + a : (size_t)idx] = cscale(cmul(Dtab[dlt], ov), pref);
    }
}

template <int L1, int L2>
__global__ void __launch_bounds__(256)
k_hlm_links(const cplx* __restrict__ hb, const cplx* __restrict__ X, int lx, int ly, int Q, int g,
            cplx* __restrict__ U1, cplx* __restrict__ U2) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Lxp = lx / Q, N = Lxp * ly;
    const int kpts = (g + 1) * g;
    const int job = blockIdx.x, sample = job / kpts, t = job % kpts;
    const int t1 = t / g, t2 = t % g;
    cplx* S1 = reinterpret_cast<cplx*>(smem_raw);      // theta_1 link: [N][Lxp]
    cplx* S2 = S1 + (size_t)N * L1;                      // theta_2 link: [N][ly]
    __shared__ cplx Dtab[LINK_MAXL];
    const bool has1 = t1 < g;
    const int t2n = t2 + 1 == g ? 0 : t2 + 1;            // theta_2 = g is the copy of theta_2 = 0
    const cplx* ha = hb + ((size_t)t1 * (g + 1) + t2) * N * Q;
    if (has1) {
        build_link_S(S1, Dtab, ha, hb + ((size_t)(t1 + 1) * (g + 1) + t2) * N * Q, N, L1, ly, Lxp, Q, 0,
                     -1.0 / g);
        __syncthreads();
    }
    build_link_S(S2, Dtab, ha, hb + ((size_t)t1 * (g + 1) + t2n) * N * Q, N, L2, ly, Lxp, Q, 1,
                 (double)(t2 - t2n) / g);
    __syncthreads();
    const size_t nn = (size_t)N * N;
    const cplx* Xa = X + ((size_t)sample * kpts + t) * nn;
    const cplx* Xb1 = X + ((size_t)sample * kpts + (t1 + 1) * g + t2) * nn;
    const cplx* Xb2 = X + ((size_t)sample * kpts + t1 * g + t2n) * nn;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        const cplx* ua = Xa + (size_t)n * N;
        const size_t o = ((size_t)sample * kpts + t) * N + n;
        if (has1) U1[o] = link_dir<L1>(S1, ua, Xb1 + (size_t)n * N, ly, ly, 0);
        U2[o] = link_dir<L2>(S2, ua, Xb2 + (size_t)n * N, Lxp, ly, 1);
    }
}

// The same links with one warp per state n: the warp stages rows n of the two neighbours'
// eigenvector matrices in shared memory, its lanes walk the Bloch index a of row n of its own
// matrix (coalesced 16-byte loads of all three rows), and the S blocks are stored transposed
// (S[l][a]) so that consecutive lanes read consecutive words.  Per-lane partial overlaps are
// reduced across the warp.
template <int L1, int L2>
__global__ void __launch_bounds__(256)
k_hlm_links_w(const cplx* __restrict__ hb, const cplx* __restrict__ X, int lx, int ly, int Q, int g,
              cplx* __restrict__ U1, cplx* __restrict__ U2) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Lxp = lx / Q, N = Lxp * ly;
    const int kpts = (g + 1) * g;
    const int job = blockIdx.x, sample = job / kpts, t = job % kpts;
    const int t1 = t / g, t2 = t % g;
    cplx* T1 = reinterpret_cast<cplx*>(smem_raw);      // theta_1 link, transposed: T1[l][a]
    cplx* T2 = T1 + (size_t)N * L1;                      // theta_2 link, T2[l][a]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    cplx* r1 = T2 + (size_t)N * L2 + (size_t)w * 2 * N;   // this warp's two staged rows
    cplx* r2 = r1 + N;
    __shared__ cplx Dtab[LINK_MAXL];
    const bool has1 = t1 < g;
    const int t2n = t2 + 1 == g ? 0 : t2 + 1;            // theta_2 = g is the copy of theta_2 = 0
    const cplx* ha = hb + ((size_t)t1 * (g + 1) + t2) * N * Q;
    if (has1) {
        build_link_S(T1, Dtab, ha, hb + ((size_t)(t1 + 1) * (g + 1) + t2) * N * Q, N, L1, ly, Lxp, Q, 0,
                     -1.0 / g, true);
        __syncthreads();
    }
    build_link_S(T2, Dtab, ha, hb + ((size_t)t1 * (g + 1) + t2n) * N * Q, N, L2, ly, Lxp, Q, 1,
                 (double)(t2 - t2n) / g, true);
    __syncthreads();
    const size_t nn = (size_t)N * N;
    const cplx* Xa = X + ((size_t)sample * kpts + t) * nn;
    const cplx* Xb1 = X + ((size_t)sample * kpts + (t1 + 1) * g + t2) * nn;
    const cplx* Xb2 = X + ((size_t)sample * kpts + t1 * g + t2n) * nn;
    for (int n = w; n < N; n += blockDim.x >> 5) {
        for (int b = lane; b < N; b += 32) {
            if (has1) r1[b] = Xb1[(size_t)n * N + b];
            r2[b] = Xb2[(size_t)n * N + b];
        }
        __syncwarp();
        cplx acc1 = mk(0, 0), acc2 = mk(0, 0);
        for (int a = lane; a < N; a += 32) {
            const int kxa = a / ly, kya = a % ly;
            const cplx ua = Xa[(size_t)n * N + a];
            if (has1) {   // theta_1 link: partners b = l * ly + kya
                cplx y = mk(0, 0);
#pragma unroll
                for (int l = 0; l < L1; ++l) cfma(y, T1[(size_t)l * N + a], r1[l * ly + kya]);
                cfmac(acc1, ua, y);
            }
            cplx y = mk(0, 0);   // theta_2 link: partners b = kxa * ly + l
#pragma unroll
            for (int l = 0; l < L2; ++l) cfma(y, T2[(size_t)l * N + a], r2[kxa * ly + l]);
            cfmac(acc2, ua, y);
        }
        acc1 = warp_sum(acc1);
        acc2 = warp_sum(acc2);
        if (lane == 0) {
            const size_t o = ((size_t)sample * kpts + t) * N + n;
            if (has1) U1[o] = acc1;
            U2[o] = acc2;
        }
        __syncwarp();   // the staged rows are rewritten for the next state
    }
}

template <int L1, int L2>
static int launch_links_thread(rlmb_context* ctx, const cplx* hb, const cplx* X, int lx, int ly, int Q, int g,
                               int nsamples, cplx* U1, cplx* U2) {
    const int N = lx * ly / Q;
    const size_t smem = (size_t)N * (L1 + L2) * sizeof(cplx);
    if (smem > 220 * 1024) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaFuncSetAttribute(k_hlm_links<L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    prof_begin(ctx, "k_hlm_links");
    k_hlm_links<L1, L2><<<nsamples * (g + 1) * g, 256, smem, ctx->stream>>>(hb, X, lx, ly, Q, g, U1, U2);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

// Warp-per-state links where their shared memory fits (the transposed S blocks and two
// staged rows per warp), else the thread-per-state kernel.
template <int L1, int L2>
static int launch_links_t(rlmb_context* ctx, const cplx* hb, const cplx* X, int lx, int ly, int Q, int g,
                          int nsamples, cplx* U1, cplx* U2) {
    const int N = lx * ly / Q;
    const size_t smem_w = ((size_t)N * (L1 + L2) + (size_t)8 * 2 * N) * sizeof(cplx);
    if (smem_w <= 220 * 1024) {
        RLMB_CUDA_TRY(cudaFuncSetAttribute(k_hlm_links_w<L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_w));
        prof_begin(ctx, "k_hlm_links");
        k_hlm_links_w<L1, L2><<<nsamples * (g + 1) * g, 256, smem_w, ctx->stream>>>(hb, X, lx, ly, Q, g, U1, U2);
        RLMB_LAUNCHED(ctx);
        return RLMB_OK;
    }
    return launch_links_thread<L1, L2>(ctx, hb, X, lx, ly, Q, g, nsamples, U1, U2);
}

int launch_hlm_links(rlmb_context* ctx, const cplx* hb, const cplx* X, int lx, int ly, int Q, int g,
                     int nsamples, cplx* U1, cplx* U2) {
    const int Lxp = lx / Q;
    // block sizes are compile-time so the U' block lives in registers; others are unsupported
#define RLMB_LINKS_CASE(A, B) \
    if (Lxp == A && ly == B) return launch_links_t<A, B>(ctx, hb, X, lx, ly, Q, g, nsamples, U1, U2);
    RLMB_LINKS_CASE(1, 1) RLMB_LINKS_CASE(1, 2) RLMB_LINKS_CASE(1, 3) RLMB_LINKS_CASE(1, 4)
    RLMB_LINKS_CASE(2, 2) RLMB_LINKS_CASE(2, 3) RLMB_LINKS_CASE(2, 4) RLMB_LINKS_CASE(2, 6)
    RLMB_LINKS_CASE(2, 8) RLMB_LINKS_CASE(3, 3) RLMB_LINKS_CASE(3, 6) RLMB_LINKS_CASE(4, 4)
    RLMB_LINKS_CASE(4, 8) RLMB_LINKS_CASE(8, 8) RLMB_LINKS_CASE(8, 16) RLMB_LINKS_CASE(16, 16)
    RLMB_LINKS_CASE(16, 8) RLMB_LINKS_CASE(4, 2) RLMB_LINKS_CASE(3, 2) RLMB_LINKS_CASE(6, 6)
    RLMB_LINKS_CASE(8, 4) RLMB_LINKS_CASE(12, 12) RLMB_LINKS_CASE(16, 32) RLMB_LINKS_CASE(32, 32)
    RLMB_LINKS_CASE(32, 16)
#undef RLMB_LINKS_CASE
    return launch_hlm_links_generic(ctx, hb, X, lx, ly, Q, g, nsamples, U1, U2);
}

}  // namespace rlmb
