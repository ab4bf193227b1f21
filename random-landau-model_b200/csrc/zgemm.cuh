// Batched complex GEMM tile engine (sm_100a, SIMT FP64 or FP32 FMA pipes).
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

// Launch on a batch of nb matrices; returns the launch error.
template <class C, int BM, class LA, class LB, class EP>
cudaError_t launch_zgemm(cudaStream_t st, const LA& la, const LB& lb, const EP& ep, int M, int N, int K, int nb) {
    auto kern = k_zgemm<C, BM, LA, LB, EP>;
    const size_t smem = zgemm_smem<C, BM>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((M + BM - 1) / BM, (N + ZG_BN - 1) / ZG_BN, nb);
    kern<<<grid, 256, smem, st>>>(la, lb, ep, M, N, K);
    return cudaGetLastError();
}

}  // namespace rlmb
