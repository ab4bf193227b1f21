// Per-kernel CUDA-event timing on the context stream, and an FP64 throughput probe.
#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace rlmb {

struct ProfRec {
    const char* name;
    cudaEvent_t a, b;
};
struct Prof {
    bool on = false;
    const char* cur = nullptr;
    cudaEvent_t cur_a = nullptr;
    std::vector<cudaEvent_t> pool;
    std::vector<ProfRec> pending;
    std::map<std::string, std::pair<double, long long>> acc;
    std::vector<std::pair<std::string, std::pair<double, long long>>> snapshot;
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
};

static Prof* prof_of(rlmb_context* ctx) { return static_cast<Prof*>(ctx->prof); }

void prof_begin(rlmb_context* ctx, const char* kernel) {
    Prof* p = prof_of(ctx);
    if (!p || !p->on) return;
    p->cur = kernel;
    p->cur_a = p->get();
    cudaEventRecord(p->cur_a, ctx->stream);
}

void prof_end(rlmb_context* ctx) {
    Prof* p = prof_of(ctx);
    if (!p || !p->on || !p->cur) return;
    cudaEvent_t b = p->get();
    cudaEventRecord(b, ctx->stream);
    p->pending.push_back({p->cur, p->cur_a, b});
    p->cur = nullptr;
}

static void prof_collect(rlmb_context* ctx, Prof* p) {
    cudaStreamSynchronize(ctx->stream);
    for (auto& r : p->pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        auto& e = p->acc[r.name];
        e.first += ms;
        e.second += 1;
        p->pool.push_back(r.a);
        p->pool.push_back(r.b);
    }
    p->pending.clear();
}

void prof_free(rlmb_context* ctx) {
    Prof* p = prof_of(ctx);
    if (!p) return;
    cudaStreamSynchronize(ctx->stream);
    for (auto& r : p->pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : p->pool) cudaEventDestroy(e);
    delete p;
    ctx->prof = nullptr;
}

// Dependent FMA chains on every SM: 8 independent chains per thread, 2 flops per FMA.
__global__ void k_fp64_fma_probe(double* out, int iters) {
    double a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = 1.0 + 1e-9 * (threadIdx.x + i);
    const double m = 0.999999999, c = 1e-12;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = fma(a[i], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678) out[0] = s;   // keeps the chains alive
}

}  // namespace rlmb

using namespace rlmb;

extern "C" {

int rlmb_profile_enable(rlmb_context* ctx, int on) {
    if (!ctx) return RLMB_ERR_ARG;
    if (!ctx->prof) ctx->prof = new Prof();
    Prof* p = prof_of(ctx);
    prof_collect(ctx, p);
    p->acc.clear();
    p->on = on != 0;
    return RLMB_OK;
}

int rlmb_profile_count(rlmb_context* ctx) {
    if (!ctx || !ctx->prof) return 0;
    Prof* p = prof_of(ctx);
    prof_collect(ctx, p);
    p->snapshot.assign(p->acc.begin(), p->acc.end());
    return (int)p->snapshot.size();
}

int rlmb_profile_entry(rlmb_context* ctx, int index, char* name, int name_cap, double* total_ms,
                       long long* launches) {
    if (!ctx || !ctx->prof || !name || name_cap <= 0 || !total_ms || !launches) return RLMB_ERR_ARG;
    Prof* p = prof_of(ctx);
    if (index < 0 || index >= (int)p->snapshot.size()) return RLMB_ERR_ARG;
    const auto& e = p->snapshot[index];
    std::snprintf(name, name_cap, "%s", e.first.c_str());
    *total_ms = e.second.first;
    *launches = e.second.second;
    return RLMB_OK;
}

int rlmb_probe_fp64_peak(rlmb_context* ctx, double* tflops) {
    if (!ctx || !tflops) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    int sms = 0;
    RLMB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    double* out = nullptr;
    RLMB_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&out), sizeof(double), ctx->stream));
    const int threads = 512, blocks = sms * 4, iters = 1 << 14;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_fp64_fma_probe<<<blocks, threads, 0, ctx->stream>>>(out, iters / 16);   // warm-up
    cudaEventRecord(a, ctx->stream);
    k_fp64_fma_probe<<<blocks, threads, 0, ctx->stream>>>(out, iters);
    cudaEventRecord(b, ctx->stream);
    cudaError_t err = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFreeAsync(out, ctx->stream);
    if (err != cudaSuccess) return RLMB_ERR_CUDA;
    *tflops = 2.0 * 8.0 * (double)iters * threads * blocks / (ms * 1e-3) / 1e12;
    return RLMB_OK;
}

}  // extern "C"
