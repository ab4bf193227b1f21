// Batched complex GEMM on the tcgen05 tensor cores with TMA-fed operands and double-precision
// accumulation across K (sm_100a).
//
// The products of the mixed-precision refinement, E = X^H R and X F, have K = n (up to 3000
// complex): accumulated in the tensor core's FP32 accumulator over the whole K, their error
// grows to ~1e-6 of |A||B|, which becomes the orthogonality defect a refinement step leaves.
// This engine keeps the split-TF32 products of k_zgemm_tc (x = hi + lo, products hi.hi +
// hi.lo + lo.hi, exact in FP32) but empties the accumulator into double-precision registers
// after every K block (32 real terms x 3 products), so FP32 rounding only ever acts on short
// partial sums.
//
// Operands are first written as TF32 planes in global memory (k_tma_planes_a / _b, through the
// same element accessors as the other engines), in the real forms of zgemm_tc.cuh:
//   A planes  [piece][matrix][2 Mp][2 Kp]: rows 2r, 2r+1 and columns 2k, 2k+1 of A(r, k) hold
//             [Re a, -Im a ; Im a, Re a];
//   B planes  [piece][matrix][Np][2 Kp]: row c, columns 2k, 2k+1 hold [Re b, Im b] of B(k, c);
// piece 0 = hi, 1 = lo, zero outside M x K and K x N (Mp, Np, Kp the padded sizes).  Then, per
// CTA (one output tile of 64 complex rows x 128 columns, 320 threads):
//   * warp 8 (one thread) loads each K block (16 complex k = 32 floats = one 128-byte row) of
//     both pieces of both operands with cp.async.bulk.tensor (3-D tensor maps, 128-byte
//     swizzle, the canonical K-major layout of the MMA descriptors) into a free stage of three,
//     signalling a full mbarrier with the transaction byte count;
//   * warp 9 (one thread) waits for the stage, issues its 12 MMAs (4 K steps x 3 products,
//     M = N = 128) into one of two TMEM accumulators (256 columns), and frees the stage with
//     tcgen05.commit; after every G blocks it commits the accumulator to the drain warps and
//     switches to the other one (after the drain warps have released it).  G = 1 sums every
//     block's FP32 partial in double precision (error independent of K); G = all of K
//     accumulates in FP32 in TMEM and drains once, leaving the tensor pipe unthrottled;
//   * warps 0-7 (one TMEM lane quarter x 64 columns each) wait for each filled accumulator,
//     read it with tcgen05.ld into FP32 registers, add it to 64 double-precision sums per
//     thread, and release it; at the end they pair real and imaginary parts across lanes and
//     call the epilogue with double-precision values.
// No cluster launch and no multicast: every TMA load reads this GPU's own planes.  Every
// mbarrier wait is bounded (TC_WAIT_NS); a wait that runs out records a fault (g_tc_fault),
// stops the CTA's issuing, skips its epilogue, and the CTA still frees its tensor memory.
#pragma once
#include <cuda.h>

#include "zgemm_tc.cuh"

namespace rlmb {

static constexpr int TMA_THREADS = 320;      // warps 0-7 drain, warp 8 loads, warp 9 issues MMAs
static constexpr int TMA_STAGES = 3;
static constexpr int TMA_G = 1;              // K blocks per accumulator drain (double-precision sums)
static constexpr int TMA_G_ALL = 1 << 20;    // one drain at the end (FP32 accumulation)
static constexpr int TMA_STAGE = 2 * TC_PLANE_A + 2 * TC_PLANE_B;   // both pieces of both operands
static constexpr size_t TMA_SMEM = (size_t)TMA_STAGES * TMA_STAGE + 1024;
static constexpr int TMA_KP = 32;            // K padding (complex) of the planes

__device__ __forceinline__ void tma_load3(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(tc_smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc_smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc_smem_u32(bar)) : "memory");
}

// ---------------------------------------------------------------- operand planes
// A planes of matrices mat0 .. mat0 + gridDim.z - 1 (plane matrix index blockIdx.z): a tile of
// 32 rows x 32 k per CTA of 256 threads, read in the accessor's contiguous direction into
// shared memory, written as whole 256-byte row segments of each plane.
template <class LA>
__global__ void __launch_bounds__(256)
k_tma_planes_a(LA la, int M, int K, int Mp, int Kp, size_t mat0, float* __restrict__ planes) {
    typedef decltype(la.elem(0, 0, 0)) CA;
    __shared__ double2 tile[32][33];
    const int t = threadIdx.x;
    const int k0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const size_t m = blockIdx.z, nbl = gridDim.z;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int rl, kl;
        if (LA::RFAST) { rl = t & 31; kl = (t >> 5) + 8 * i; }
        else { kl = t & 31; rl = (t >> 5) + 8 * i; }
        const int r = r0 + rl, k = k0 + kl;
        CA v = (r < M && k < K) ? la.elem(mat0 + m, r, k) : cz<CA>();
        tile[rl][kl] = make_double2((double)v.x, (double)v.y);
    }
    __syncthreads();
    const int rl = t >> 3, kq = (t & 7) * 4;   // 4 consecutive k of one row
    const size_t plane = (size_t)nbl * 2 * Mp * 2 * Kp;
    const size_t row0 = (m * 2 * Mp + 2 * (size_t)(r0 + rl)) * 2 * Kp + 2 * (size_t)(k0 + kq);
    float hi0[8], lo0[8], hi1[8], lo1[8];   // rows 2r (Re, -Im) and 2r+1 (Im, Re), 4 k each
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double2 a = tile[rl][kq + j];
        float rh, rlo, ih, ilo;
        tc_split((float)a.x, rh, rlo);
        tc_split((float)a.y, ih, ilo);
        hi0[2 * j] = rh;  hi0[2 * j + 1] = -ih;  lo0[2 * j] = rlo;  lo0[2 * j + 1] = -ilo;
        hi1[2 * j] = ih;  hi1[2 * j + 1] = rh;   lo1[2 * j] = ilo;  lo1[2 * j + 1] = rlo;
    }
    float* p0 = planes + row0;
    float* p1 = p0 + 2 * (size_t)Kp;   // row 2r + 1
    reinterpret_cast<float4*>(p0)[0] = make_float4(hi0[0], hi0[1], hi0[2], hi0[3]);
    reinterpret_cast<float4*>(p0)[1] = make_float4(hi0[4], hi0[5], hi0[6], hi0[7]);
    reinterpret_cast<float4*>(p1)[0] = make_float4(hi1[0], hi1[1], hi1[2], hi1[3]);
    reinterpret_cast<float4*>(p1)[1] = make_float4(hi1[4], hi1[5], hi1[6], hi1[7]);
    reinterpret_cast<float4*>(p0 + plane)[0] = make_float4(lo0[0], lo0[1], lo0[2], lo0[3]);
    reinterpret_cast<float4*>(p0 + plane)[1] = make_float4(lo0[4], lo0[5], lo0[6], lo0[7]);
    reinterpret_cast<float4*>(p1 + plane)[0] = make_float4(lo1[0], lo1[1], lo1[2], lo1[3]);
    reinterpret_cast<float4*>(p1 + plane)[1] = make_float4(lo1[4], lo1[5], lo1[6], lo1[7]);
}

// B planes: a tile of 32 k x 32 columns per CTA; row c of a plane holds (Re, Im) of B(k, c)
// along k.
template <class LB>
__global__ void __launch_bounds__(256)
k_tma_planes_b(LB lb, int N, int K, int Np, int Kp, size_t mat0, float* __restrict__ planes) {
    typedef decltype(lb.elem(0, 0, 0)) CB;
    __shared__ double2 tile[32][33];   // tile[c][k]
    const int t = threadIdx.x;
    const int k0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const size_t m = blockIdx.z, nbl = gridDim.z;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int cl, kl;
        if (LB::KFAST) { kl = t & 31; cl = (t >> 5) + 8 * i; }
        else { cl = t & 31; kl = (t >> 5) + 8 * i; }
        const int c = c0 + cl, k = k0 + kl;
        CB v = (c < N && k < K) ? lb.elem(mat0 + m, k, c) : cz<CB>();
        tile[cl][kl] = make_double2((double)v.x, (double)v.y);
    }
    __syncthreads();
    const int cl = t >> 3, kq = (t & 7) * 4;
    const size_t plane = (size_t)nbl * Np * 2 * Kp;
    float* p = planes + (m * Np + (size_t)(c0 + cl)) * 2 * Kp + 2 * (size_t)(k0 + kq);
    float hi[8], lo[8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double2 b = tile[cl][kq + j];
        tc_split((float)b.x, hi[2 * j], lo[2 * j]);
        tc_split((float)b.y, hi[2 * j + 1], lo[2 * j + 1]);
    }
    reinterpret_cast<float4*>(p)[0] = make_float4(hi[0], hi[1], hi[2], hi[3]);
    reinterpret_cast<float4*>(p)[1] = make_float4(hi[4], hi[5], hi[6], hi[7]);
    reinterpret_cast<float4*>(p + plane)[0] = make_float4(lo[0], lo[1], lo[2], lo[3]);
    reinterpret_cast<float4*>(p + plane)[1] = make_float4(lo[4], lo[5], lo[6], lo[7]);
}

// ---------------------------------------------------------------- the GEMM
template <class C, class EP, int G = TMA_G>
__global__ void __launch_bounds__(TMA_THREADS, 1)
k_zgemm_tma(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, EP ep, int M, int N,
            int Kp, int nbl, size_t mat0) {
    extern __shared__ unsigned char tma_raw[];
    __shared__ __align__(8) uint64_t bar_full[TMA_STAGES], bar_empty[TMA_STAGES];
    __shared__ __align__(8) uint64_t bar_acc[2], bar_accfree[2], bar_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int fault, skip_cta;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const size_t m = blockIdx.z;
    const int r0 = blockIdx.x * TC_BM, c0 = blockIdx.y * TC_BN;
    if constexpr (tc_has_skip<EP>::value)
        if (ep.skip_tile(r0, c0, TC_BM, TC_BN)) return;
    if (t == 0) skip_cta = *(volatile int*)&g_tc_fault;
    __syncthreads();
    if (skip_cta) return;
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tma_raw) + 1023) & ~(uintptr_t)1023);
    const uint32_t sbase = tc_smem_u32(smem);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(&tmem_slot)),
                     "r"(2 * TC_BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 32) {
        for (int s = 0; s < TMA_STAGES; ++s) {
            tc_mbar_init(&bar_full[s], 1);
            tc_mbar_init(&bar_empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc_mbar_init(&bar_acc[b], 1);
            tc_mbar_init(&bar_accfree[b], 8);   // one arrival per drain warp
        }
        tc_mbar_init(&bar_done, 1);
        fault = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const int nk = Kp / TC_KB;                   // K blocks
    const int ng = (nk + G - 1) / G;             // accumulator groups

    if (warp == 8) {
        if (lane == 0) {   // ---- TMA producer
            int loaded = 0;   // K blocks whose loads were issued
            for (int kb = 0; kb < nk; ++kb) {
                const int s = kb % TMA_STAGES;
                if (kb >= TMA_STAGES && !tc_mbar_wait(&bar_empty[s], (unsigned)((kb / TMA_STAGES - 1) & 1))) {
                    atomicExch(&fault, 1);
                    break;
                }
                if (*(volatile int*)&fault) break;
                const uint32_t st = sbase + (uint32_t)(s * TMA_STAGE);
                tma_expect(&bar_full[s], (uint32_t)TMA_STAGE);
                for (int p = 0; p < 2; ++p) {
                    tma_load3(st + p * TC_PLANE_A, &ta, 32 * kb, 2 * r0, p * (int)nbl + (int)m, &bar_full[s]);
                    tma_load3(st + 2 * TC_PLANE_A + p * TC_PLANE_B, &tb, 32 * kb, c0, p * (int)nbl + (int)m,
                              &bar_full[s]);
                }
                loaded = kb + 1;
            }
            // no load may still be landing when the CTA exits: wait (bounded) for the last
            // use of every stage (already complete unless the MMA thread stopped early)
            for (int kb = loaded - 1; kb >= 0 && kb >= loaded - TMA_STAGES; --kb)
                if (!tc_mbar_wait(&bar_full[kb % TMA_STAGES], (unsigned)((kb / TMA_STAGES) & 1))) atomicExch(&fault, 1);
        }
    } else if (warp == 9) {
        if (lane == 0) {   // ---- MMA issuer
            for (int g = 0; g < ng && !*(volatile int*)&fault; ++g) {
                const int b = g & 1;
                if (g >= 2 && !tc_mbar_wait(&bar_accfree[b], (unsigned)((g / 2 - 1) & 1))) {
                    atomicExch(&fault, 1);
                    break;
                }
                const uint32_t acc = tmem + (uint32_t)(b * TC_BN);
                bool ok = true;
                for (int kb = g * G; kb < min(nk, (g + 1) * G); ++kb) {
                    const int s = kb % TMA_STAGES;
                    if (!tc_mbar_wait(&bar_full[s], (unsigned)((kb / TMA_STAGES) & 1))) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a = sbase + (uint32_t)(s * TMA_STAGE);
                    const uint32_t bb = a + 2 * TC_PLANE_A;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const uint64_t ah = tc_desc(a + 32 * j), al = tc_desc(a + TC_PLANE_A + 32 * j);
                        const uint64_t bh = tc_desc(bb + 32 * j), bl = tc_desc(bb + TC_PLANE_B + 32 * j);
                        tc_mma(acc, ah, bh, (kb != g * G || j != 0) ? 1u : 0u);
                        tc_mma(acc, ah, bl, 1);
                        tc_mma(acc, al, bh, 1);
                    }
                    tc_commit(&bar_empty[s]);
                }
                // the group's MMAs (all issued so far) complete before the drain reads them
                tc_commit(&bar_acc[b]);
                if (!ok) {
                    atomicExch(&fault, 1);
                    break;
                }
            }
            // every MMA this thread issued has completed before the tensor memory is freed
            tc_commit(&bar_done);
            if (!tc_mbar_wait(&bar_done, 0)) atomicExch(&fault, 1);
        }
    } else {   // ---- warps 0-7: drain the accumulators into double-precision sums
        const int q = warp & 3, cbase = (warp >> 2) * 64;
        double sum[64];
#pragma unroll
        for (int i = 0; i < 64; ++i) sum[i] = 0.0;
        for (int g = 0; g < ng; ++g) {
            const int b = g & 1;
            // warp-uniform decisions: tcgen05.ld below is a collective of the whole warp
            const bool ok = __all_sync(0xffffffffu, tc_mbar_wait(&bar_acc[b], (unsigned)((g / 2) & 1)));
            if (!ok) {
                atomicExch(&fault, 1);
                break;
            }
            if (__any_sync(0xffffffffu, *(volatile int*)&fault != 0)) break;
            tc_fence_after();
            const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * TC_BN + cbase);
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) {
                float v[16];
                tc_ld16(base + 16 * ch, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) sum[16 * ch + i] += (double)v[i];
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) tma_arrive(&bar_accfree[b]);
        }
        // all drain warps agree on the fault state before the epilogue (named barrier 1)
        asm volatile("bar.sync 1, 256;" ::: "memory");
        if (!__any_sync(0xffffffffu, *(volatile int*)&fault != 0)) {
            const bool odd = lane & 1;   // odd lanes hold imaginary parts
            const int r = r0 + 16 * q + (lane >> 1);
#pragma unroll
            for (int ch = 0; ch < 4; ++ch)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    // even lanes take columns 16 ch + j, odd lanes 16 ch + 8 + j
                    const double x = __shfl_xor_sync(0xffffffffu, odd ? sum[16 * ch + j] : sum[16 * ch + 8 + j], 1);
                    const int c = c0 + cbase + 16 * ch + j + (odd ? 8 : 0);
                    if (r < M && c < N)
                        ep.store(mat0 + m, r, c,
                                 cm<C>(odd ? x : sum[16 * ch + j], odd ? sum[16 * ch + 8 + j] : x));
                }
        }
    }
    __syncthreads();
    if (t == 0 && fault) atomicAdd(&g_tc_fault, 1);
    // every issued MMA has completed (the MMA thread waited for its last commit) and no TMA
    // load is in flight (the producer waited for its last ones)
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_BN) : "memory");
}

// ---------------------------------------------------------------- host side
typedef CUresult (*TmaEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
TmaEncodeFn tma_encode_fn();   // cuTensorMapEncodeTiled from the driver (nullptr if unavailable)

// 3-D map over float planes [depth][rows][cols], box 32 x 128 x 1, 128-byte swizzle.
inline bool tma_map(CUtensorMap* map, float* base, size_t cols, size_t rows, size_t depth) {
    TmaEncodeFn enc = tma_encode_fn();
    if (!enc) return false;
    const cuuint64_t dims[3] = {cols, rows, depth};
    const cuuint64_t strides[2] = {cols * sizeof(float), cols * rows * sizeof(float)};
    const cuuint32_t box[3] = {32, 128, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Bytes of planes one matrix needs for an M x N x K product.
inline size_t tma_plane_bytes(int M, int N, int K) {
    const size_t Mp = (size_t)(M + TC_BM - 1) / TC_BM * TC_BM, Np = (size_t)(N + TC_BN - 1) / TC_BN * TC_BN;
    const size_t Kp = (size_t)(K + TMA_KP - 1) / TMA_KP * TMA_KP;
    return 2 * (2 * Mp * 2 * Kp + Np * 2 * Kp) * sizeof(float);
}

// C = A B for nb matrices through planes in `ws` (ws_bytes, 256-byte aligned), in
// sub-batches of as many matrices as the planes fit; the sums over K in double precision
// (fp64_sum) or in FP32; returns a CUDA error.
template <class C, class LA, class LB, class EP>
cudaError_t launch_zgemm_tma(cudaStream_t st, const LA& la, const LB& lb, const EP& ep, int M, int N, int K, int nb,
                             void* ws, size_t ws_bytes, bool fp64_sum = true) {
    if (M <= 0 || N <= 0 || nb <= 0) return cudaSuccess;
    if (K <= 0) return launch_zgemm_tc<C>(st, la, lb, ep, M, N, K, nb);   // zero product
    const int Mp = (M + TC_BM - 1) / TC_BM * TC_BM, Np = (N + TC_BN - 1) / TC_BN * TC_BN;
    const int Kp = (K + TMA_KP - 1) / TMA_KP * TMA_KP;
    const size_t per = tma_plane_bytes(M, N, K);
    const int sub = (int)std::min<size_t>((size_t)nb, ws_bytes / per);
    if (sub < 1 || !ws) return cudaErrorMemoryAllocation;
    auto kern = fp64_sum ? k_zgemm_tma<C, EP, TMA_G> : k_zgemm_tma<C, EP, TMA_G_ALL>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TMA_SMEM);
    if (e != cudaSuccess) return e;
    for (int m0 = 0; m0 < nb; m0 += sub) {
        const int nbl = std::min(sub, nb - m0);
        float* pa = static_cast<float*>(ws);
        float* pb = pa + 2 * (size_t)nbl * 2 * Mp * 2 * Kp;
        k_tma_planes_a<LA><<<dim3(Kp / 32, Mp / 32, nbl), 256, 0, st>>>(la, M, K, Mp, Kp, (size_t)m0, pa);
        k_tma_planes_b<LB><<<dim3(Kp / 32, Np / 32, nbl), 256, 0, st>>>(lb, N, K, Np, Kp, (size_t)m0, pb);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        CUtensorMap ta, tb;
        if (!tma_map(&ta, pa, 2 * (size_t)Kp, 2 * (size_t)Mp, 2 * (size_t)nbl) ||
            !tma_map(&tb, pb, 2 * (size_t)Kp, (size_t)Np, 2 * (size_t)nbl))
            return cudaErrorInvalidValue;
        kern<<<dim3(Mp / TC_BM, Np / TC_BN, nbl), TMA_THREADS, TMA_SMEM, st>>>(ta, tb, ep, M, N, Kp, nbl, (size_t)m0);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace rlmb
