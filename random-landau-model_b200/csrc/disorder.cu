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

// a + (b - a) * u / 2^32 with the host's roundings (no contraction)
__device__ __forceinline__ double mt_uniform(uint32_t u, double a, double b) {
    return __dadd_rn(a, __dmul_rn(b - a, __dmul_rn((double)u, 1.0 / 4294967296.0)));
}

// rlm disorder of samples sample0 .. sample0+count-1 (rlm/disorder_potential.cpp:3-21): stream
// `seed` skipped by 3*nimp*sample; x_i ~ U[0,L1), y_i ~ U[0,L2), s_i = +1 for an even 32-bit
// output else -1.  Output [sample][i] in x, y, s (row stride ld).
__global__ void __launch_bounds__(256)
k_rlm_disorder(uint32_t seed, int nimp, double L1, double L2, int sample0, double* __restrict__ x,
               double* __restrict__ y, double* __restrict__ s, size_t ld) {
    __shared__ uint32_t mt[MT_N];
    const int smp = blockIdx.x;
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
    prof_begin(ctx, "k_rlm_disorder");
    k_rlm_disorder<<<count, 256, 0, ctx->stream>>>((uint32_t)seed, impurity_num, L1, L2, sample0, d_x, d_y, d_s,
                                                  (size_t)impurity_num);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}

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
