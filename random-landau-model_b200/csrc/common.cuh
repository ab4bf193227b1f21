// Shared device/host helpers of the rlm/hlm B200 library.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/rlm_b200.h"

namespace rlmb {

// ---------------------------------------------------------------- complex (re, im)
typedef double2 cplx;

__host__ __device__ __forceinline__ cplx mk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ cplx cmulc(cplx a, cplx b) {
    return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cconj(cplx a) { return mk(a.x, -a.y); }
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return mk(a.x * s, a.y * s); }
// acc += a * b
__host__ __device__ __forceinline__ void cfma(cplx& acc, cplx a, cplx b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
// acc += conj(a) * b
__host__ __device__ __forceinline__ void cfmac(cplx& acc, cplx a, cplx b) {
    acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(-a.y, b.x, acc.y));
}
__host__ __device__ __forceinline__ double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

__device__ __forceinline__ cplx shfl_xor(cplx v, int m) {
    return mk(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;
}
__device__ __forceinline__ cplx warp_sum(cplx v) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v = cadd(v, shfl_xor(v, m));
    return v;
}

}  // namespace rlmb

// -------------------------------------------------------------------- context
struct rlmb_context {
    int device;
    cudaStream_t stream;
    long long launches;
    // grow-only device buffers owned by the context: solver internals and pipeline data
    void* ws;
    size_t ws_bytes;
    void* pipe;
    size_t pipe_bytes;
    // pinned host staging
    void* pinned;
    size_t pinned_bytes;
    // cached hlm tables (Bloch vectors and link overlaps of one mesh geometry)
    int hlm_key[6];
    void* hlm_tables;
    size_t hlm_tables_bytes;
    // optional per-kernel CUDA-event timing (rlmb_profile_enable)
    void* prof;
};

#define RLMB_CUDA_TRY(expr)                                                       \
    do {                                                                          \
        cudaError_t _e = (expr);                                                  \
        if (_e != cudaSuccess) {                                                  \
            fprintf(stderr, "rlmb: CUDA error %s at %s:%d: %s\n", #expr, __FILE__, \
                    __LINE__, cudaGetErrorString(_e));                            \
            return RLMB_ERR_CUDA;                                                 \
        }                                                                         \
    } while (0)

namespace rlmb {
// Per-kernel event timing: prof_begin records a start event on the context stream
// before a launch, prof_end the stop event after it (no-ops unless profiling is on).
void prof_begin(rlmb_context* ctx, const char* kernel);
void prof_end(rlmb_context* ctx);
}  // namespace rlmb

#define RLMB_LAUNCHED(ctx)                                                        \
    do {                                                                          \
        rlmb::prof_end(ctx);                                                      \
        (ctx)->launches++;                                                        \
        cudaError_t _e = cudaGetLastError();                                      \
        if (_e != cudaSuccess) {                                                  \
            fprintf(stderr, "rlmb: launch failed at %s:%d: %s\n", __FILE__,        \
                    __LINE__, cudaGetErrorString(_e));                            \
            return RLMB_ERR_CUDA;                                                 \
        }                                                                         \
    } while (0)

namespace rlmb {
// Grow-only workspace of the context (cudaMallocAsync on its stream would also do; a
// plain grow-only buffer keeps repeated calls allocation-free).
int ensure_workspace(rlmb_context* ctx, size_t bytes);
int ensure_pipe(rlmb_context* ctx, size_t bytes);
int ensure_pinned(rlmb_context* ctx, size_t bytes);
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
}  // namespace rlmb
