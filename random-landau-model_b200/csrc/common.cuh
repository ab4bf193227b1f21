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

// -------------------------------------------- single-precision complex (mixed mode)
typedef float2 cplxf;
__host__ __device__ __forceinline__ cplxf cadd(cplxf a, cplxf b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplxf csub(cplxf a, cplxf b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplxf cmul(cplxf a, cplxf b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplxf cmulc(cplxf a, cplxf b) {
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ cplxf cconj(cplxf a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ cplxf cscale(cplxf a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ void cfma(cplxf& acc, cplxf a, cplxf b) {
    acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
    acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
}
__host__ __device__ __forceinline__ void cfmac(cplxf& acc, cplxf a, cplxf b) {
    acc.x = fmaf(a.x, b.x, fmaf(a.y, b.y, acc.x));
    acc.y = fmaf(a.x, b.y, fmaf(-a.y, b.x, acc.y));
}
__host__ __device__ __forceinline__ float cabs2(cplxf a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ cplxf shfl_xor(cplxf v, int m) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;
}
__device__ __forceinline__ cplxf warp_sum(cplxf v) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v = cadd(v, shfl_xor(v, m));
    return v;
}

// Precision-generic access: Cx<R>::T is the complex type of real type R.
template <class R> struct Cx;
template <> struct Cx<double> { typedef double2 T; };
template <> struct Cx<float> { typedef float2 T; };
template <class C> __host__ __device__ __forceinline__ C cm(double r, double i);
template <> __host__ __device__ __forceinline__ double2 cm<double2>(double r, double i) { return make_double2(r, i); }
template <> __host__ __device__ __forceinline__ float2 cm<float2>(double r, double i) {
    return make_float2((float)r, (float)i);
}
template <class C> __host__ __device__ __forceinline__ C cz() { return cm<C>(0.0, 0.0); }
__host__ __device__ __forceinline__ double2 to_c64(double2 a) { return a; }
__host__ __device__ __forceinline__ double2 to_c64(float2 a) { return make_double2(a.x, a.y); }
template <class C> __host__ __device__ __forceinline__ C from_c64(double2 a);
template <> __host__ __device__ __forceinline__ double2 from_c64<double2>(double2 a) { return a; }
template <> __host__ __device__ __forceinline__ float2 from_c64<float2>(double2 a) {
    return make_float2((float)a.x, (float)a.y);
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
    // device staging of the host-buffer pipeline calls, and the device counter of
    // eigensolves that did not converge (accumulated on the device, read once per call)
    void* io;
    size_t io_bytes;
    int* fail;
    // the device rlm disorder stream of the last call (state words + block index), for
    // continuing it when the next call starts at the next sample
    uint32_t* mt_state;
    // set while a stream capture records this context's work: buffers may not grow then
    int frozen;
    // TF32 operand planes of the TMA-fed tensor-core GEMMs (grow-only)
    void* tws;
    size_t tws_bytes;
    // eigensolver autotuning (rlmb_set_autotune) and its per-(order, precision) choices
    int autotune;
    void* tune;
    int mt_valid;
    unsigned long mt_seed;
    int mt_nimp;
    long long mt_next;
    // cached hlm tables (Bloch vectors and link overlaps of one mesh geometry)
    int hlm_key[6];
    void* hlm_tables;
    size_t hlm_tables_bytes;
    // optional per-kernel CUDA-event timing (rlmb_profile_enable)
    void* prof;
    // RLMB_PRECISION_FP64 or RLMB_PRECISION_MIXED, and the mixed mode's refinement
    // steps (rlmb_set_precision, rlmb_set_refinement_steps)
    int precision;
    int refine_steps;
    // mixed mode, one refinement step: recompute every eigenvalue afterwards as the Rayleigh
    // quotient of its refined vector (rlmb_set_eigenvalue_pass)
    int rq_pass;
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
// rlmb_heevd_batched with a structure hint (band >= 0: cyclic band of that half-bandwidth).
int heevd_batched_band(rlmb_context* ctx, double* d_a, double* d_w, int n, int batch, int* d_info, int band);
void tune_free(rlmb_context* ctx);
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
int ensure_tma_planes(rlmb_context* ctx, size_t bytes);
int ensure_pipe(rlmb_context* ctx, size_t bytes);
int ensure_pinned(rlmb_context* ctx, size_t bytes);
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
}  // namespace rlmb
