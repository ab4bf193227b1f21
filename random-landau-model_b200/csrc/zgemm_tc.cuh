// Batched complex GEMM on the fifth-generation tensor cores (sm_100a tcgen05, kind::tf32),
// FP32-class accuracy from split operands.
//
// C = A B for every matrix of a batch (blockIdx.z), with the operand accessors and epilogues
// of the SIMT/DMMA engines in zgemm.cuh (la.elem(mat, r, k), lb.elem(mat, k, c),
// ep.store(mat, r, c, acc)).  The complex product is one real GEMM of the real forms
//
//   A''(2r + p, 2k + q) = [Re a, -Im a ; Im a, Re a](p, q),   B''(2k + q, c) = [Re b ; Im b](q),
//   C''(2r + p, c)      = [Re c ; Im c](p),
//
// so an output tile of 64 complex rows x 128 columns is one 128 x 128 FP32 accumulator in
// tensor memory (TMEM), whose even lanes hold real parts and odd lanes imaginary parts.
// Every operand value x is split into two TF32 numbers, x = hi + lo + O(2^-22 |x|)
// (hi = x rounded to 11 significant bits, lo = the remainder rounded the same way), and the
// product takes three MMAs per K step: hi.hi + hi.lo + lo.hi, i.e. relative error ~2^-21 per
// product term plus the FP32 accumulation.  TF32 products of 11-bit operands are exact in
// FP32.
//
// Pipeline (one CTA of 256 threads per output tile; three stages and one CTA per SM, or for
// short inner dimensions one stage and two CTAs per SM):
//   * all threads load the next K block (16 complex k) of A and B through the accessors into
//     registers one block ahead, split it and store it to a free stage of shared memory in
//     the canonical K-major 128-byte-swizzled layout (8-row atoms of 128-byte rows, the
//     16-byte chunk index XORed with the row index mod 8);
//   * thread 0 issues the block's 12 MMAs (4 K steps of 8 x 3 products, M = N = 128) with
//     tcgen05.mma and commits them to the stage's mbarrier, which frees the stage when the
//     tensor core has read it;
//   * after the last block a final commit signals the epilogue: each warp reads its 32 TMEM
//     lanes x 64 columns with tcgen05.ld, pairs real and imaginary parts across lanes and
//     calls the epilogue.
// Every mbarrier wait is bounded (1 s of wall-clock time); a wait that runs out records a
// fault in g_tc_fault (read by rlmb_tc_fault_count), stops issuing and skips the epilogue,
// and the CTA still waits (bounded) for its issued MMAs and frees its tensor memory before it
// exits.  Tiles that start after a fault was recorded exit at once.
#pragma once
#include "common.cuh"

#include <type_traits>
#include <utility>

namespace rlmb {

static constexpr int TC_BM = 64;            // complex rows per tile (128 real rows, UMMA M)
static constexpr int TC_BN = 128;           // complex columns per tile (UMMA N)
static constexpr int TC_KB = 16;            // complex k per stage (32 real k = one 128-byte row)
static constexpr int TC_STAGES = 3;
static constexpr int TC_THREADS = 256;
static constexpr int TC_PLANE_A = 128 * 128;      // bytes of one A plane (128 rows x 128 B)
static constexpr int TC_PLANE_B = TC_BN * 128;    // bytes of one B plane
static constexpr int TC_STAGE = 2 * TC_PLANE_A + 2 * TC_PLANE_B;
static constexpr size_t TC_SMEM = (size_t)TC_STAGES * TC_STAGE + 1024;   // + alignment slack
static constexpr unsigned long long TC_WAIT_NS = 1000000000ull;   // 1 s: a longer mbarrier wait is a fault

// Instruction descriptor of tcgen05.mma kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
static constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                                     ((uint32_t)(128 >> 4) << 24);

static __device__ int g_tc_fault;   // number of CTAs whose mbarrier wait ran out (never expected)

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand tile whose 8-row
// atoms are 1024 bytes apart: start address >> 4, leading offset 1 (unused inside a swizzle
// row), stride offset 1024 >> 4, descriptor version 1 (bit 46), layout SWIZZLE_128B (2 << 61).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tc_mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool tc_mbar_try(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(tc_smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long tc_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for the phase of the given parity; false if it did not complete within
// TC_WAIT_NS of wall-clock time (the global nanosecond timer).
__device__ __forceinline__ bool tc_mbar_wait(uint64_t* bar, unsigned parity) {
    if (tc_mbar_try(bar, parity)) return true;
    const unsigned long long t0 = tc_ns();
    while (!tc_mbar_try(bar, parity))
        if (tc_ns() - t0 > TC_WAIT_NS) return false;
    return true;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     tc_smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(acc)
        : "memory");
}
// 32 TMEM lanes (this warp's quarter) x 16 consecutive 32-bit columns into v[0..15].
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// x = hi + lo with hi, lo TF32 numbers (low 13 mantissa bits zero), each rounded to nearest
// (ties away from zero) by integer rounding of the bit pattern; x - hi is exact in FP32.
__device__ __forceinline__ float tc_tf32(float x) { return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u); }
__device__ __forceinline__ void tc_split(float x, float& hi, float& lo) {
    hi = tc_tf32(x);
    lo = tc_tf32(x - hi);
}

// byte offset of float element (row, col) in a K-major 128-byte-swizzled plane (cols < 32)
__device__ __forceinline__ uint32_t tc_off(int row, int col) {
    return (uint32_t)row * 128u + ((uint32_t)(((col >> 2) ^ (row & 7))) << 4) + ((uint32_t)(col & 3) << 2);
}

// Epilogues may drop whole output tiles with skip_tile(r0, c0, rows, cols).
template <class T, class = void>
struct tc_has_skip : std::false_type {};
template <class T>
struct tc_has_skip<T, std::void_t<decltype(&T::skip_tile)>> : std::true_type {};

// An epilogue that updates C in place may expose pre_src(mat, r, c) (address of C(r, c), or
// null where it writes nothing) and store_pre(mat, r, c, acc, old): each thread then loads
// its 32 entries of C into registers when the tile starts, so that these reads overlap the
// operand loads and the MMAs instead of following them.
template <class T, class = void>
struct tc_has_pre : std::false_type {};
template <class T>
struct tc_has_pre<T, std::void_t<decltype(&T::pre_src)>> : std::true_type {};
template <class EP, bool P = tc_has_pre<EP>::value>
struct tc_pre_type {
    typedef float2 T;
};
template <class EP>
struct tc_pre_type<EP, true> {
    typedef std::remove_cv_t<std::remove_pointer_t<decltype(std::declval<EP>().pre_src(0, 0, 0))>> T;
};

// STAGES shared-memory stages of one K block each; MINB CTAs per SM.  Short inner
// dimensions (K <= 4 blocks: the rank-32 panel updates, the 64-reflector block updates)
// take one stage and two CTAs per SM, so that one CTA's epilogue overlaps the other's
// loads; the next block's global loads are in flight while the tensor core reads the stage.
template <class C, class LA, class LB, class EP, int STAGES = TC_STAGES, int MINB = 1>
__global__ void __launch_bounds__(TC_THREADS, MINB)
k_zgemm_tc(LA la, LB lb, EP ep, int M, int N, int K) {
    extern __shared__ unsigned char tc_raw[];
    __shared__ __align__(8) uint64_t bar_free[STAGES];
    __shared__ __align__(8) uint64_t bar_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int fault;
    typedef decltype(la.elem(0, 0, 0)) CA;
    typedef decltype(lb.elem(0, 0, 0)) CB;
    constexpr int EA = TC_BM * TC_KB / TC_THREADS;   // A entries per thread per block (4)
    constexpr int EB = TC_BN * TC_KB / TC_THREADS;   // B entries per thread per block (8)
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const size_t mat = blockIdx.z;
    const int r0 = blockIdx.x * TC_BM, c0 = blockIdx.y * TC_BN;
    if constexpr (tc_has_skip<EP>::value)
        if (ep.skip_tile(r0, c0, TC_BM, TC_BN)) return;   // whole CTA leaves before any set-up
    // after a fault anywhere (a wait that ran out) the remaining tiles are not attempted; the
    // flag is read once so that the whole CTA takes the same branch
    __shared__ int skip_cta;
    if (threadIdx.x == 0) skip_cta = *(volatile int*)&g_tc_fault;
    __syncthreads();
    if (skip_cta) return;
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~(uintptr_t)1023);
    const uint32_t sbase = tc_smem_u32(smem);
    // epilogue coordinates of this thread: TMEM lane quarter q, accumulator columns cbase..+63,
    // row r; entry i = 8 (chunk of 16 columns) + j sits at column c0 + cbase + 16 (i / 8) +
    // (i % 8) + (odd ? 8 : 0)
    const int q = warp & 3;
    const int cbase = (warp >> 2) * 64;
    const bool odd = lane & 1;   // odd lanes hold imaginary parts
    const int r = r0 + 16 * q + (lane >> 1);
    constexpr bool PRE = tc_has_pre<EP>::value;
    typedef typename tc_pre_type<EP>::T CO;
    CO old[PRE ? 32 : 1];
    if constexpr (PRE) {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int c = c0 + cbase + 16 * (i >> 3) + (i & 7) + (odd ? 8 : 0);
            const CO* src = (r < M && c < N) ? ep.pre_src(mat, r, c) : nullptr;
            old[i] = src ? *src : CO{};
        }
    }

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(&tmem_slot)),
                     "r"(TC_BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 32) {
        for (int s = 0; s < STAGES; ++s) tc_mbar_init(&bar_free[s], 1);
        tc_mbar_init(&bar_done, 1);
        fault = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    // ---- operand staging: thread t's entries of the A and B blocks
    auto a_pos = [&](int e, int& rl, int& kl) {
        const int idx = t + TC_THREADS * e;
        if (LA::RFAST) { rl = idx % TC_BM; kl = idx / TC_BM; }
        else { kl = idx % TC_KB; rl = idx / TC_KB; }
    };
    auto b_pos = [&](int e, int& kl, int& cl) {
        const int idx = t + TC_THREADS * e;
        if (LB::KFAST) { kl = idx % TC_KB; cl = idx / TC_KB; }
        else { cl = idx % TC_BN; kl = idx / TC_BN; }
    };
    CA fa[EA];
    CB fb[EB];
    auto load = [&](int k0) {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            int rl, kl;
            a_pos(e, rl, kl);
            const int r = r0 + rl, k = k0 + kl;
            fa[e] = (r < M && k < K) ? la.elem(mat, r, k) : cz<CA>();
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            int kl, cl;
            b_pos(e, kl, cl);
            const int c = c0 + cl, k = k0 + kl;
            fb[e] = (c < N && k < K) ? lb.elem(mat, k, c) : cz<CB>();
        }
    };
    auto put = [&](int s) {
        unsigned char* st = smem + (size_t)s * TC_STAGE;
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            int rl, kl;
            a_pos(e, rl, kl);
            float rh, rlo, ih, ilo;
            tc_split((float)fa[e].x, rh, rlo);
            tc_split((float)fa[e].y, ih, ilo);
            const uint32_t o0 = tc_off(2 * rl, 2 * kl), o1 = tc_off(2 * rl + 1, 2 * kl);
            *reinterpret_cast<float2*>(st + o0) = make_float2(rh, -ih);
            *reinterpret_cast<float2*>(st + o1) = make_float2(ih, rh);
            *reinterpret_cast<float2*>(st + TC_PLANE_A + o0) = make_float2(rlo, -ilo);
            *reinterpret_cast<float2*>(st + TC_PLANE_A + o1) = make_float2(ilo, rlo);
        }
        unsigned char* sb = st + 2 * TC_PLANE_A;
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            int kl, cl;
            b_pos(e, kl, cl);
            float rh, rlo, ih, ilo;
            tc_split((float)fb[e].x, rh, rlo);
            tc_split((float)fb[e].y, ih, ilo);
            const uint32_t o = tc_off(cl, 2 * kl);
            *reinterpret_cast<float2*>(sb + o) = make_float2(rh, ih);
            *reinterpret_cast<float2*>(sb + TC_PLANE_B + o) = make_float2(rlo, ilo);
        }
    };

    const int nk = (K + TC_KB - 1) / TC_KB;
    int issued = 0;   // thread 0: whether any MMA was issued
    if (nk > 0) load(0);
    for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % STAGES;
        if (kb >= STAGES) {
            // the stage is free once the MMAs of block kb - STAGES have read it
            if (!tc_mbar_wait(&bar_free[s], (unsigned)((kb / STAGES - 1) & 1))) atomicExch(&fault, 1);
        }
        __syncthreads();
        if (fault) break;
        put(s);
        if (kb + 1 < nk) load((kb + 1) * TC_KB);   // next block's loads overlap this block's MMAs
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // st.shared -> tensor core
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            const uint32_t a = sbase + (uint32_t)(s * TC_STAGE);
            const uint32_t b = a + 2 * TC_PLANE_A;
#pragma unroll
            for (int j = 0; j < 4; ++j) {   // K steps of 8 TF32 (32 bytes) inside the 128-byte rows
                const uint64_t ah = tc_desc(a + 32 * j), al = tc_desc(a + TC_PLANE_A + 32 * j);
                const uint64_t bh = tc_desc(b + 32 * j), bl = tc_desc(b + TC_PLANE_B + 32 * j);
                tc_mma(tmem, ah, bh, (kb | j) != 0);
                tc_mma(tmem, ah, bl, 1);
                tc_mma(tmem, al, bh, 1);
            }
            tc_commit(&bar_free[s]);
            issued = 1;
        }
    }
    // ---- epilogue: wait for every issued MMA (bar_done is committed after the last one),
    // then read the accumulator
    if (t == 0 && issued) tc_commit(&bar_done);
    const int any_issued = __syncthreads_or(issued);
    if (any_issued && !tc_mbar_wait(&bar_done, 0)) atomicExch(&fault, 1);
    tc_fence_after();
    __syncthreads();
    if (!fault) {
#pragma unroll
        for (int ch = 0; ch < 64; ch += 16) {
            float v[16];
            if (any_issued) {
                tc_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(cbase + ch), v);
            } else {   // K == 0: the product is zero
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = 0.0f;
            }
            // even lanes take columns ch..ch+7 of the chunk, odd lanes ch+8..ch+15
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float x = __shfl_xor_sync(0xffffffffu, odd ? v[j] : v[j + 8], 1);
                const int c = c0 + cbase + ch + j + (odd ? 8 : 0);
                if (r < M && c < N) {
                    const C acc = cm<C>(odd ? x : v[j], odd ? v[j + 8] : x);
                    if constexpr (PRE) {
                        if (ep.pre_src(mat, r, c)) ep.store_pre(mat, r, c, acc, old[(ch >> 4) * 8 + j]);
                    } else {
                        ep.store(mat, r, c, acc);
                    }
                }
            }
        }
    } else if (t == 0) {
        atomicAdd(&g_tc_fault, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN) : "memory");
}

// Launch on a batch of nb matrices (grid: row tiles, column tiles, matrices); returns the
// launch error.  C is the accumulator type the epilogue receives (cplx or cplxf).
template <class C, class LA, class LB, class EP>
cudaError_t launch_zgemm_tc(cudaStream_t st, const LA& la, const LB& lb, const EP& ep, int M, int N, int K, int nb) {
    if (M <= 0 || N <= 0 || nb <= 0) return cudaSuccess;
    const dim3 grid((M + TC_BM - 1) / TC_BM, (N + TC_BN - 1) / TC_BN, nb);
    if (grid.y > 65535 || grid.z > 65535) return cudaErrorInvalidConfiguration;
    const bool short_k = K <= 4 * TC_KB;
    auto kern = short_k ? k_zgemm_tc<C, LA, LB, EP, 1, 2> : k_zgemm_tc<C, LA, LB, EP, TC_STAGES, 1>;
    const size_t smem = short_k ? (size_t)TC_STAGE + 1024 : TC_SMEM;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, TC_THREADS, smem, st>>>(la, lb, ep, M, N, K);
    return cudaGetLastError();
}

}  // namespace rlmb
