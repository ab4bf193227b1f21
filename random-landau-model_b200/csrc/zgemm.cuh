// Batched complex GEMM tile engines (sm_100a): k_zgemm on the FMA pipes (single precision)
// and k_zgemm_dmma on the FP64 tensor path (double precision); launch_zgemm picks by type.
//
// C = A B for every matrix of a batch (blockIdx.z), output tiles of BM x 64 per CTA of
// 256 threads; thread t = 16 tr + tc owns rows RM*tr .. RM*tr+RM-1 (RM = BM/16) and
// columns tc + 16 v (v < 4) of the tile: RM x 4 complex accumulators in registers, so that
// every complex operand read from shared memory feeds 4 (A) or RM (B) multiply-adds.
// The inner dimension advances ZG_KC at a time through two shared-memory stages; the
// global loads of the next stage are issued into registers before the current stage is
// consumed and stored to shared memory after it, so that their latency overlaps the math.
//
// Operands are functors with an element accessor and a coalescing hint:
//   A: la.elem(mat, r, k), LA::RFAST (r contiguous in memory, else k contiguous)
//   B: lb.elem(mat, k, c), LB::KFAST (k contiguous in memory, else c contiguous)
// called only inside the matrix (r < M, k < K, c < N); the epilogue ep.store(mat, r, c,
// acc) is called once per output entry, and ep.skip(r0, c0, BM) may drop whole output tiles
// (a triangular update).
#pragma once
#include "common.cuh"

#include <type_traits>

namespace rlmb {

static constexpr int ZG_BN = 64;
static constexpr int ZG_KC = 8;

template <class C, int BM>
struct ZgTiles {
    C a[2][ZG_KC][BM + 1];
    C b[2][ZG_KC][ZG_BN + 1];
};

template <class C, int BM, class LA, class LB, class EP>
__global__ void __launch_bounds__(256, BM == 64 ? 2 : 1)
k_zgemm(LA la, LB lb, EP ep, int M, int N, int K) {
    constexpr int RM = BM / 16;
    constexpr int EA = BM * ZG_KC / 256;      // A-tile entries per thread
    constexpr int EB = ZG_BN * ZG_KC / 256;   // B-tile entries per thread
    extern __shared__ __align__(16) unsigned char zg_smem[];
    ZgTiles<C, BM>& s = *reinterpret_cast<ZgTiles<C, BM>*>(zg_smem);
    const int t = threadIdx.x, tr = t / 16, tc = t % 16;
    const size_t mat = blockIdx.z;
    const int r0 = blockIdx.x * BM, c0 = blockIdx.y * ZG_BN;
    if (ep.skip(r0, c0, BM)) return;   // output tile not needed (whole CTA leaves together)
    C fa[EA], fb[EB];
    auto a_pos = [&](int e, int& kk, int& rr) {
        const int idx = t + 256 * e;
        if (LA::RFAST) { kk = idx / BM; rr = idx % BM; }
        else { kk = idx % ZG_KC; rr = idx / ZG_KC; }
    };
    auto b_pos = [&](int e, int& kk, int& cc) {
        const int idx = t + 256 * e;
        if (LB::KFAST) { kk = idx % ZG_KC; cc = idx / ZG_KC; }
        else { kk = idx / ZG_BN; cc = idx % ZG_BN; }
    };
    auto load = [&](int k0) {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            int kk, rr;
            a_pos(e, kk, rr);
            const int r = r0 + rr, k = k0 + kk;
            fa[e] = (r < M && k < K) ? la.elem(mat, r, k) : cz<C>();
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            int kk, cc;
            b_pos(e, kk, cc);
            const int c = c0 + cc, k = k0 + kk;
            fb[e] = (c < N && k < K) ? lb.elem(mat, k, c) : cz<C>();
        }
    };
    auto put = [&](int buf) {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            int kk, rr;
            a_pos(e, kk, rr);
            s.a[buf][kk][rr] = fa[e];
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            int kk, cc;
            b_pos(e, kk, cc);
            s.b[buf][kk][cc] = fb[e];
        }
    };
    C acc[RM][4];
#pragma unroll
    for (int u = 0; u < RM; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = cz<C>();
    const int nk = (K + ZG_KC - 1) / ZG_KC;
    if (nk > 0) {
        load(0);
        put(0);
    }
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        const int cur = kt & 1;
        const bool more = kt + 1 < nk;
        if (more) load((kt + 1) * ZG_KC);
#pragma unroll
        for (int kk = 0; kk < ZG_KC; ++kk) {
            C av[RM], bv[4];
#pragma unroll
            for (int u = 0; u < RM; ++u) av[u] = s.a[cur][kk][RM * tr + u];
#pragma unroll
            for (int v = 0; v < 4; ++v) bv[v] = s.b[cur][kk][tc + 16 * v];
#pragma unroll
            for (int u = 0; u < RM; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) cfma(acc[u][v], av[u], bv[v]);
        }
        if (more) put(cur ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const int c = c0 + tc + 16 * v;
        if (c >= N) continue;
#pragma unroll
        for (int u = 0; u < RM; ++u) {
            const int r = r0 + RM * tr + u;
            if (r < M) ep.store(mat, r, c, acc[u][v]);
        }
    }
}

template <class C, int BM>
constexpr size_t zgemm_smem() { return sizeof(ZgTiles<C, BM>); }

// ---- double precision on the FP64 tensor path (mma.sync m8n8k4 .f64, "DMMA")
// Same tiles, operands, staging and epilogue as k_zgemm; the math runs as 8x8x4 real DMMAs.
// The 8 warps split the BM x 64 tile into 32 x WN warp tiles (WN = 16 for BM = 64, 32 for
// BM = 128), i.e. 4 x WN/8 blocks of 8 x 8 with a real and an imaginary accumulator each.
// Per k-step of 4, lane (g = lane / 4, q = lane % 4) reads the complex entries A(8i+g, q) and
// B(q, 8j+g) of its blocks from shared memory (both fragments of the real and imaginary
// parts at once), and every block takes four DMMAs:
//   Cr += Ar Br - Ai Bi,   Ci += Ar Bi + Ai Br.
// The accumulator of block (i, j) holds C(8i+g, 8j+2q) and C(8i+g, 8j+2q+1).  Rows of the
// shared tiles are padded by 2 entries so that the 8-lane phases of these 16-byte loads hit
// distinct banks.
static constexpr int ZT_PAD = 2;
template <int BM>
struct ZtTiles {
    cplx a[2][ZG_KC][BM + ZT_PAD];
    cplx b[2][ZG_KC][ZG_BN + ZT_PAD];
};

// An epilogue that updates C in place may expose pre_src(mat, r, c) (address of C(r, c), or
// null where it writes nothing) and store_pre(mat, r, c, acc, old).  k_zgemm_dmma then copies
// each thread's C entries into shared memory with cp.async when it starts, so that the
// epilogue's reads of C overlap the main loop instead of following it.  Thread t's entry
// idx sits at slot idx * 256 + t (consecutive threads, consecutive 16-byte words).
template <class T, class = void>
struct zg_has_pre : std::false_type {};
template <class T>
struct zg_has_pre<T, std::void_t<decltype(&T::pre_src)>> : std::true_type {};

template <int BM, class EP>
constexpr size_t zgemm_dmma_smem() {
    return sizeof(ZtTiles<BM>) + (zg_has_pre<EP>::value ? (size_t)256 * 4 * (ZG_BN * (BM / 32) / 64) * 2 * sizeof(cplx) : 0);
}

__device__ __forceinline__ void zg_cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

template <int BM, class LA, class LB, class EP>
__global__ void __launch_bounds__(256, BM == 64 ? 2 : 1)
k_zgemm_dmma(LA la, LB lb, EP ep, int M, int N, int K) {
    constexpr int WR = BM / 32;        // warps along the rows of the tile
    constexpr int WN = ZG_BN * WR / 8; // columns of a warp tile
    constexpr int MI = 4, NJ = WN / 8;
    constexpr int EA = BM * ZG_KC / 256;
    constexpr int EB = ZG_BN * ZG_KC / 256;
    extern __shared__ __align__(16) unsigned char zg_smem[];
    ZtTiles<BM>& s = *reinterpret_cast<ZtTiles<BM>*>(zg_smem);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wr = warp % WR, wc = warp / WR, g = lane >> 2, q = lane & 3;
    const size_t mat = blockIdx.z;
    const int r0 = blockIdx.x * BM, c0 = blockIdx.y * ZG_BN;
    if (ep.skip(r0, c0, BM)) return;   // output tile not needed (whole CTA leaves together)
    constexpr bool PRE = zg_has_pre<EP>::value;
    cplx* pre = reinterpret_cast<cplx*>(zg_smem + sizeof(ZtTiles<BM>));
    if constexpr (PRE) {
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
            for (int j = 0; j < NJ; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int r = r0 + 32 * wr + 8 * i + g, c = c0 + WN * wc + 8 * j + 2 * q + e;
                    const cplx* src = (r < M && c < N) ? ep.pre_src(mat, r, c) : nullptr;
                    if (src) zg_cp_async16(pre + ((i * NJ + j) * 2 + e) * 256 + t, src);
                }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    cplx fa[EA], fb[EB];
    auto a_pos = [&](int e, int& kk, int& rr) {
        const int idx = t + 256 * e;
        if (LA::RFAST) { kk = idx / BM; rr = idx % BM; }
        else { kk = idx % ZG_KC; rr = idx / ZG_KC; }
    };
    auto b_pos = [&](int e, int& kk, int& cc) {
        const int idx = t + 256 * e;
        if (LB::KFAST) { kk = idx % ZG_KC; cc = idx / ZG_KC; }
        else { kk = idx / ZG_BN; cc = idx % ZG_BN; }
    };
    auto load = [&](int k0) {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            int kk, rr;
            a_pos(e, kk, rr);
            const int r = r0 + rr, k = k0 + kk;
            fa[e] = (r < M && k < K) ? la.elem(mat, r, k) : cz<cplx>();
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            int kk, cc;
            b_pos(e, kk, cc);
            const int c = c0 + cc, k = k0 + kk;
            fb[e] = (c < N && k < K) ? lb.elem(mat, k, c) : cz<cplx>();
        }
    };
    auto put = [&](int buf) {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            int kk, rr;
            a_pos(e, kk, rr);
            s.a[buf][kk][rr] = fa[e];
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            int kk, cc;
            b_pos(e, kk, cc);
            s.b[buf][kk][cc] = fb[e];
        }
    };
    double cr[MI][NJ][2], ci[MI][NJ][2];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;
    const int nk = (K + ZG_KC - 1) / ZG_KC;
    if (nk > 0) {
        load(0);
        put(0);
    }
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        const int cur = kt & 1;
        const bool more = kt + 1 < nk;
        if (more) load((kt + 1) * ZG_KC);
#pragma unroll
        for (int ks = 0; ks < ZG_KC / 4; ++ks) {
            double ar[MI], ai[MI], an[MI], br[NJ], bi[NJ];
#pragma unroll
            for (int i = 0; i < MI; ++i) {
                const cplx x = s.a[cur][4 * ks + q][32 * wr + 8 * i + g];
                ar[i] = x.x;
                ai[i] = x.y;
                an[i] = -x.y;
            }
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const cplx y = s.b[cur][4 * ks + q][WN * wc + 8 * j + g];
                br[j] = y.x;
                bi[j] = y.y;
            }
#pragma unroll
            for (int i = 0; i < MI; ++i)
#pragma unroll
                for (int j = 0; j < NJ; ++j) {
                    dmma884(cr[i][j], ar[i], br[j]);
                    dmma884(ci[i][j], ar[i], bi[j]);
                    dmma884(cr[i][j], an[i], bi[j]);
                    dmma884(ci[i][j], ai[i], br[j]);
                }
        }
        if (more) put(cur ^ 1);
        __syncthreads();
    }
    if constexpr (PRE) asm volatile("cp.async.wait_group 0;\n" ::: "memory");   // this thread's own copies
#pragma unroll
    for (int i = 0; i < MI; ++i) {
        const int r = r0 + 32 * wr + 8 * i + g;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < NJ; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int c = c0 + WN * wc + 8 * j + 2 * q + e;
                if (c >= N) continue;
                if constexpr (PRE) {
                    if (ep.pre_src(mat, r, c))
                        ep.store_pre(mat, r, c, mk(cr[i][j][e], ci[i][j][e]), pre[((i * NJ + j) * 2 + e) * 256 + t]);
                } else {
                    ep.store(mat, r, c, mk(cr[i][j][e], ci[i][j][e]));
                }
            }
    }
}

// Launch on a batch of nb matrices; returns the launch error.  Double precision runs on the
// DMMA engine, single precision on the FP32 FMA engine.
template <class C, int BM, class LA, class LB, class EP>
cudaError_t launch_zgemm(cudaStream_t st, const LA& la, const LB& lb, const EP& ep, int M, int N, int K, int nb) {
    const dim3 grid((M + BM - 1) / BM, (N + ZG_BN - 1) / ZG_BN, nb);
    if constexpr (std::is_same<C, cplx>::value) {
        auto kern = k_zgemm_dmma<BM, LA, LB, EP>;
        const size_t smem = zgemm_dmma_smem<BM, EP>();
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, 256, smem, st>>>(la, lb, ep, M, N, K);
    } else {
        auto kern = k_zgemm<C, BM, LA, LB, EP>;
        const size_t smem = zgemm_smem<C, BM>();
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, 256, smem, st>>>(la, lb, ep, M, N, K);
    }
    return cudaGetLastError();
}

}  // namespace rlmb
