// Disorder generation on the device: MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998)
// with init_genrand seeding and the tempered 32-bit output -- the same stream as the host
// generator of host_tables.cpp (the reference's vslNewStream(VSL_BRNG_MT19937, seed) and
// vdRngUniform / viRngUniformBits calls), bit for bit.
//
// One CTA per stream: thread 0 seeds the 624-word state, the state is advanced a block of
// 624 outputs at a time by a parallel twist in four dependency phases (outputs i in [0,227)
// read only old words; [227,454) and [454,623) read words of earlier phases; 623 reads the
// new word 0), each phase loading its inputs before any thread writes.  Skipping ahead by p
// outputs costs p/624 twists.
#include "common.cuh"

namespace rlmb {

static constexpr int MT_N = 624, MT_M = 397;

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

// one twist of the state in shared memory, by the CTA (blockDim.x >= 227)
__device__ __forceinline__ void mt_twist(uint32_t* mt) {
    const int t = threadIdx.x;
    const int lo[4] = {0, 227, 454, 623}, hi[4] = {227, 454, 623, 624};
#pragma unroll
    for (int ph = 0; ph < 4; ++ph) {
        const int i = lo[ph] + t;
        uint32_t v = 0;
        const bool act = i < hi[ph];
        if (act) {
            const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % MT_N] & 0x7fffffffu);
            v = mt[(i + MT_M) % MT_N] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908b0dfu;
        }
        __syncthreads();
        if (act) mt[i] = v;
        __syncthreads();
    }
}

__device__ __forceinline__ void mt_seed(uint32_t* mt, uint32_t seed) {
    if (threadIdx.x == 0) {
        mt[0] = seed;
        for (int i = 1; i < MT_N; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
    }
    __syncthreads();
}

// state words and the index of the output block they hold, for a later continuation
__device__ __forceinline__ void mt_save(const uint32_t* mt, long long blk, uint32_t* out) {
    __syncthreads();
    for (int i = threadIdx.x; i < MT_N; i += blockDim.x) out[i] = mt[i];
    if (threadIdx.x == 0) {
        out[MT_N] = (uint32_t)((uint64_t)blk & 0xffffffffu);
        out[MT_N + 1] = (uint32_t)((uint64_t)blk >> 32);
    }
}

// a + (b - a) * u / 2^32 with the host's roundings (no contraction)
__device__ __forceinline__ double mt_uniform(uint32_t u, double a, double b) {
    return __dadd_rn(a, __dmul_rn(b - a, __dmul_rn((double)u, 1.0 / 4294967296.0)));
}

// rlm disorder of samples sample0 .. sample0+count-1 (rlm/disorder_potential.cpp:3-21): stream
// `seed` skipped by 3*nimp*sample; x_i ~ U[0,L1), y_i ~ U[0,L2), s_i = +1 for an even 32-bit
// output else -1.  Output [sample][i] in x, y, s (row stride ld).
__global__ void __launch_bounds__(256)
k_rlm_disorder(uint32_t seed, int nimp, double L1, double L2, int sample0, double* __restrict__ x,
               double* __restrict__ y, double* __restrict__ s, size_t ld, uint32_t* __restrict__ save,
               const int* __restrict__ dsample0) {
    __shared__ uint32_t mt[MT_N];
    const int smp = blockIdx.x;
    if (dsample0) sample0 += *dsample0;   // first sample read from device memory (graph replays)
    mt_seed(mt, seed);
    long long pos = 3LL * nimp * (sample0 + smp);   // outputs consumed before this sample
    const long long end = pos + 3LL * nimp;
    for (long long b = 0; b < pos / MT_N; ++b) mt_twist(mt);   // skip whole blocks
    long long blk = pos / MT_N;
    mt_twist(mt);                                                // the block holding `pos`
    double* xo = x + ld * smp;
    double* yo = y + ld * smp;
    double* so = s + ld * smp;
    while (pos < end) {
        const long long base = blk * MT_N;
        for (long long k = pos + threadIdx.x; k < min(end, base + MT_N); k += blockDim.x) {
            const uint32_t u = mt_temper(mt[k - base]);
            const long long r = k - 3LL * nimp * (sample0 + smp);
            const int i = (int)(r % nimp), which = (int)(r / nimp);
            if (which == 0) xo[i] = mt_uniform(u, 0.0, L1);
            else if (which == 1) yo[i] = mt_uniform(u, 0.0, L2);
            else so[i] = (u % 2u == 0u) ? 1.0 : -1.0;
        }
        pos = min(end, base + MT_N);
        if (pos < end) {
            __syncthreads();
            mt_twist(mt);
            ++blk;
        }
    }
    if (save && smp == (int)gridDim.x - 1) mt_save(mt, blk, save);   // the stream after the last sample
}

// The same draws for samples sample0 .. sample0+count-1 by one CTA that continues the stream
// from a state saved by an earlier call (the block of outputs holding position
// 3 nimp sample0, and its index), generating the samples one after another: a run that
// draws its samples in order pays each output once instead of a skip-ahead per sample.
__global__ void __launch_bounds__(256)
k_rlm_disorder_cont(int nimp, double L1, double L2, int sample0, int count, double* __restrict__ x,
                    double* __restrict__ y, double* __restrict__ s, size_t ld, uint32_t* __restrict__ state) {
    __shared__ uint32_t mt[MT_N];
    __shared__ long long blk_s;
    for (int i = threadIdx.x; i < MT_N; i += blockDim.x) mt[i] = state[i];
    if (threadIdx.x == 0) blk_s = (long long)(((uint64_t)state[MT_N + 1] << 32) | state[MT_N]);
    __syncthreads();
    long long blk = blk_s;
    const long long first = 3LL * nimp * sample0;
    long long pos = first;
    const long long end = first + 3LL * nimp * count;
    while (blk < pos / MT_N) {   // (an earlier call may have stopped short of this block)
        mt_twist(mt);
        ++blk;
    }
    while (pos < end) {
        const long long base = blk * MT_N;
        for (long long k = pos + threadIdx.x; k < min(end, base + MT_N); k += blockDim.x) {
            const uint32_t u = mt_temper(mt[k - base]);
            const long long r = k - first;
            const int smp = (int)(r / (3LL * nimp));
            const long long q = r - 3LL * nimp * smp;
            const int i = (int)(q % nimp), which = (int)(q / nimp);
            if (which == 0) x[ld * smp + i] = mt_uniform(u, 0.0, L1);
            else if (which == 1) y[ld * smp + i] = mt_uniform(u, 0.0, L2);
            else s[ld * smp + i] = (u % 2u == 0u) ? 1.0 : -1.0;
        }
        pos = min(end, base + MT_N);
        if (pos < end) {
            __syncthreads();
            mt_twist(mt);
            ++blk;
        }
    }
    mt_save(mt, blk, state);
}

// hlm on-site potentials (hlm/main_hlm_cpu.cpp:66-67,79): one stream for the whole run,
// sample k uses outputs [k*n_sites, (k+1)*n_sites), each U[-1,1).  Output [sample][site].
__global__ void __launch_bounds__(256)
k_hlm_potentials(uint32_t seed, int n_sites, int sample0, double* __restrict__ out) {
    __shared__ uint32_t mt[MT_N];
    const int smp = blockIdx.x;
    mt_seed(mt, seed);
    long long pos = (long long)n_sites * (sample0 + smp);
    const long long first = pos, end = pos + n_sites;
    for (long long b = 0; b < pos / MT_N; ++b) mt_twist(mt);
    long long blk = pos / MT_N;
    mt_twist(mt);
    double* o = out + (size_t)n_sites * smp;
    while (pos < end) {
        const long long base = blk * MT_N;
        for (long long k = pos + threadIdx.x; k < min(end, base + MT_N); k += blockDim.x)
            o[k - first] = mt_uniform(mt_temper(mt[k - base]), -1.0, 1.0);
        pos = min(end, base + MT_N);
        if (pos < end) {
            __syncthreads();
            mt_twist(mt);
            ++blk;
        }
    }
}

}  // namespace rlmb

using namespace rlmb;

extern "C" int rlmb_rlm_disorder_device(rlmb_context* ctx, int impurity_num, double L1, double L2,
                                        unsigned long seed, int sample0, int count, double* d_x,
                                        double* d_y, double* d_s) {
    if (!ctx || impurity_num <= 0 || sample0 < 0 || count < 0 || (count > 0 && (!d_x || !d_y || !d_s)))
        return RLMB_ERR_ARG;
    if (count == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (!ctx->mt_state) {
        if (cudaMalloc(reinterpret_cast<void**>(&ctx->mt_state), (MT_N + 2) * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            ctx->mt_state = nullptr;
            return RLMB_ERR_ALLOC;
        }
        ctx->mt_valid = 0;
    }
    // continue the context's saved stream when this call starts where the last one ended
    // (same seed and impurity count); otherwise every sample's CTA skips ahead on its own
    const long long first = 3LL * impurity_num * sample0;
    const bool cont = ctx->mt_valid && ctx->mt_seed == (unsigned long)(uint32_t)seed && ctx->mt_nimp == impurity_num &&
                      ctx->mt_next == first;
    if (cont) {
        prof_begin(ctx, "k_rlm_disorder");
        k_rlm_disorder_cont<<<1, 256, 0, ctx->stream>>>(impurity_num, L1, L2, sample0, count, d_x, d_y, d_s,
                                                         (size_t)impurity_num, ctx->mt_state);
    } else {
        prof_begin(ctx, "k_rlm_disorder");
        k_rlm_disorder<<<count, 256, 0, ctx->stream>>>((uint32_t)seed, impurity_num, L1, L2, sample0, d_x, d_y, d_s,
                                                      (size_t)impurity_num, ctx->mt_state, nullptr);
    }
    RLMB_LAUNCHED(ctx);
    ctx->mt_valid = 1;
    ctx->mt_seed = (unsigned long)(uint32_t)seed;
    ctx->mt_nimp = impurity_num;
    ctx->mt_next = first + 3LL * impurity_num * count;
    return RLMB_OK;
}

namespace rlmb {
// rlm disorder of samples *d_sample0 + offset .. + count - 1, the first sample index read from
// device memory when the kernel runs (for a captured graph replayed with new samples); no
// stream state is saved or continued.
int launch_rlm_disorder_at(rlmb_context* ctx, int nimp, double L1, double L2, unsigned long seed,
                           const int* d_sample0, int offset, int count, double* d_x, double* d_y, double* d_s) {
    prof_begin(ctx, "k_rlm_disorder");
    k_rlm_disorder<<<count, 256, 0, ctx->stream>>>((uint32_t)seed, nimp, L1, L2, offset, d_x, d_y, d_s, (size_t)nimp,
                                                  nullptr, d_sample0);
    RLMB_LAUNCHED(ctx);
    ctx->mt_valid = 0;
    return RLMB_OK;
}
}  // namespace rlmb

extern "C" int rlmb_hlm_potentials_device(rlmb_context* ctx, unsigned long seed, int n_sites, int sample0,
                                          int count, double* d_out) {
    if (!ctx || n_sites <= 0 || sample0 < 0 || count < 0 || (count > 0 && !d_out)) return RLMB_ERR_ARG;
    if (count == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    prof_begin(ctx, "k_hlm_potentials");
    k_hlm_potentials<<<count, 256, 0, ctx->stream>>>((uint32_t)seed, n_sites, sample0, d_out);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}
