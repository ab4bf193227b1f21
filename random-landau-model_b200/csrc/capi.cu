// C ABI of the library (include/rlm_b200.h): contexts, standalone stages and the two
// whole-mesh pipelines.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "model_kernels.cuh"

namespace rlmb {

void prof_free(rlmb_context* ctx);

static int grow(rlmb_context* ctx, void** buf, size_t* have, size_t bytes) {
    if (bytes <= *have) return RLMB_OK;
    if (ctx->frozen) return RLMB_ERR_ALLOC;   // a stream capture is recording: no reallocation
    if (*buf) {
        RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        RLMB_CUDA_TRY(cudaFree(*buf));
        *buf = nullptr;
        *have = 0;
    }
    bytes = align_up(bytes, (size_t)1 << 20);
    if (cudaMalloc(buf, bytes) != cudaSuccess) {
        cudaGetLastError();
        *buf = nullptr;
        return RLMB_ERR_ALLOC;
    }
    *have = bytes;
    return RLMB_OK;
}
int ensure_workspace(rlmb_context* ctx, size_t bytes) { return grow(ctx, &ctx->ws, &ctx->ws_bytes, bytes); }
int ensure_pipe(rlmb_context* ctx, size_t bytes) { return grow(ctx, &ctx->pipe, &ctx->pipe_bytes, bytes); }
static int ensure_io(rlmb_context* ctx, size_t bytes) { return grow(ctx, &ctx->io, &ctx->io_bytes, bytes); }
int ensure_tma_planes(rlmb_context* ctx, size_t bytes) { return grow(ctx, &ctx->tws, &ctx->tws_bytes, bytes); }
int ensure_pinned(rlmb_context* ctx, size_t bytes) {
    if (bytes <= ctx->pinned_bytes) return RLMB_OK;
    if (ctx->pinned) {
        RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        RLMB_CUDA_TRY(cudaFreeHost(ctx->pinned));
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
    }
    bytes = align_up(bytes, (size_t)1 << 20);
    if (cudaMallocHost(&ctx->pinned, bytes) != cudaSuccess) {
        cudaGetLastError();
        ctx->pinned = nullptr;
        return RLMB_ERR_ALLOC;
    }
    ctx->pinned_bytes = bytes;
    return RLMB_OK;
}

// Carves consecutive aligned regions out of one buffer.
struct Carver {
    char* base;
    size_t off = 0;
    explicit Carver(void* b) : base(static_cast<char*>(b)) {}
    template <typename T>
    T* take(size_t count) {
        off = align_up(off, 256);
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};
template <typename T>
static size_t need(size_t& acc, size_t count) {
    acc = align_up(acc, 256) + count * sizeof(T);
    return acc;
}

// Bloch tables of an hlm mesh geometry, cached in the context (disorder independent).
static int hlm_tables(rlmb_context* ctx, int lx, int ly, int Q, int band, int g, cplx** out) {
    const int key[6] = {lx, ly, Q, band, g, 1};
    const int N = lx * ly / Q;
    const size_t bytes = (size_t)(g + 1) * (g + 1) * N * Q * sizeof(cplx);
    if (ctx->hlm_tables && std::memcmp(key, ctx->hlm_key, sizeof(key)) == 0) {
        *out = static_cast<cplx*>(ctx->hlm_tables);
        return RLMB_OK;
    }
    if (ctx->hlm_tables) {
        RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        RLMB_CUDA_TRY(cudaFree(ctx->hlm_tables));
        ctx->hlm_tables = nullptr;
    }
    if (cudaMalloc(&ctx->hlm_tables, bytes) != cudaSuccess) {
        cudaGetLastError();
        ctx->hlm_tables = nullptr;
        return RLMB_ERR_ALLOC;
    }
    ctx->hlm_tables_bytes = bytes;
    if (int rc = launch_hlm_bloch(ctx, lx, ly, Q, band, g, 0, g + 1, 0, g + 1,
                                  static_cast<cplx*>(ctx->hlm_tables)))
        return rc;
    std::memcpy(ctx->hlm_key, key, sizeof(key));
    *out = static_cast<cplx*>(ctx->hlm_tables);
    return RLMB_OK;
}

// Eigensolve failures of a pipeline call are tallied on the device (no host round trip per
// batch) and read once, when the call ends.
__global__ void k_count_nonzero(const int* __restrict__ info, int count, int* __restrict__ fail) {
    int c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) c += info[i] != 0;
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(fail, c);
}
static int reset_failures(rlmb_context* ctx) {
    if (!ctx->fail) {
        if (cudaMalloc(reinterpret_cast<void**>(&ctx->fail), sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            ctx->fail = nullptr;
            return RLMB_ERR_ALLOC;
        }
    }
    RLMB_CUDA_TRY(cudaMemsetAsync(ctx->fail, 0, sizeof(int), ctx->stream));
    return RLMB_OK;
}
static int tally_failures(rlmb_context* ctx, const int* d_info, int count) {
    if (count <= 0) return RLMB_OK;
    k_count_nonzero<<<std::min((count + 255) / 256, 1024), 256, 0, ctx->stream>>>(d_info, count, ctx->fail);
    RLMB_LAUNCHED(ctx);
    return RLMB_OK;
}
// Synchronises the context stream and returns the call's status: the failure count, if any.
static int finish_call(rlmb_context* ctx) {
    int h = 0;
    RLMB_CUDA_TRY(cudaMemcpyAsync(&h, ctx->fail, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return h > 0 ? h : RLMB_OK;
}

static bool hlm_args_ok(int lx, int ly, int Q, int band, int g) {
    return lx > 0 && ly > 0 && Q > 0 && Q <= RLMB_MAX_Q && lx % Q == 0 && band >= 0 && band < Q &&
           g > 0 && lx / Q <= 64 && ly <= 64;
}

// Device memory budget for one batch of mesh data: a third of the free memory, counting the
// context's own pipeline buffer (reused by the batch) as free so that repeated calls batch
// alike, at most 40 GB.
static size_t mesh_budget_bytes(const rlmb_context* ctx) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return (size_t)8 << 30;
    }
    const size_t cap = (size_t)40 << 30;
    return std::min(cap, (free_b + ctx->pipe_bytes) / 3);
}

// Samples per batch: at most `fit`, and the batches of one call equal in size (a short last
// batch would leave most SMs idle in the one-CTA-per-matrix kernels).
static int balanced_batch(int n_samples, size_t fit) {
    const size_t cap = std::max<size_t>(1, std::min<size_t>((size_t)n_samples, fit));
    const size_t nbatches = ((size_t)n_samples + cap - 1) / cap;
    return (int)(((size_t)n_samples + nbatches - 1) / nbatches);
}

}  // namespace rlmb

using namespace rlmb;

extern "C" {

int rlmb_create(rlmb_context** out, int device) {
    if (!out) return RLMB_ERR_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return RLMB_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(device));
    rlmb_context* ctx = new rlmb_context();
    std::memset(ctx, 0, sizeof(*ctx));
    ctx->device = device;
    ctx->stream = 0;
    ctx->precision = RLMB_PRECISION_FP64;
    ctx->refine_steps = 2;
    *out = ctx;
    return RLMB_OK;
}

int rlmb_destroy(rlmb_context* ctx) {
    if (!ctx) return RLMB_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    prof_free(ctx);
    tune_free(ctx);
    if (ctx->ws) cudaFree(ctx->ws);
    if (ctx->pipe) cudaFree(ctx->pipe);
    if (ctx->io) cudaFree(ctx->io);
    if (ctx->tws) cudaFree(ctx->tws);
    if (ctx->fail) cudaFree(ctx->fail);
    if (ctx->mt_state) cudaFree(ctx->mt_state);
    if (ctx->hlm_tables) cudaFree(ctx->hlm_tables);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    delete ctx;
    return RLMB_OK;
}

int rlmb_set_stream(rlmb_context* ctx, void* stream) {
    if (!ctx) return RLMB_ERR_ARG;
    ctx->stream = static_cast<cudaStream_t>(stream);
    return RLMB_OK;
}

long long rlmb_launch_count(const rlmb_context* ctx) { return ctx ? ctx->launches : -1; }

int rlmb_set_precision(rlmb_context* ctx, int mode) {
    if (!ctx || (mode != RLMB_PRECISION_FP64 && mode != RLMB_PRECISION_MIXED)) return RLMB_ERR_ARG;
    ctx->precision = mode;
    return RLMB_OK;
}

int rlmb_get_precision(const rlmb_context* ctx) { return ctx ? ctx->precision : RLMB_ERR_ARG; }

int rlmb_set_refinement_steps(rlmb_context* ctx, int steps) {
    if (!ctx || steps < 1 || steps > 2) return RLMB_ERR_ARG;
    ctx->refine_steps = steps;
    return RLMB_OK;
}

int rlmb_set_eigenvalue_pass(rlmb_context* ctx, int on) {
    if (!ctx) return RLMB_ERR_ARG;
    ctx->rq_pass = on ? 1 : 0;
    return RLMB_OK;
}

const char* rlmb_status_string(int status) {
    switch (status) {
        case RLMB_OK: return "ok";
        case RLMB_ERR_ARG: return "invalid argument";
        case RLMB_ERR_CUDA: return "CUDA error";
        case RLMB_ERR_ALLOC: return "device or pinned allocation failed";
        case RLMB_ERR_NO_DEVICE: return "no CUDA device";
        case RLMB_ERR_TOO_LARGE: return "matrix order exceeds the allocation-free scratch limit";
        default: return status > 0 ? "eigenvectors did not converge for some matrices" : "unknown status";
    }
}

int rlmb_heevd_host(rlmb_context* ctx, double* h_a, double* h_w, int n, int batch) {
    if (!ctx || !h_a || !h_w || n <= 0 || batch < 0) return RLMB_ERR_ARG;
    if (batch == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t nn = (size_t)n * n;
    size_t bytes = 0;
    need<cplx>(bytes, nn * batch);
    need<double>(bytes, (size_t)n * batch);
    need<int>(bytes, batch);
    if (int rc = ensure_pipe(ctx, bytes)) return rc;
    Carver cv(ctx->pipe);
    cplx* dA = cv.take<cplx>(nn * batch);
    double* dW = cv.take<double>((size_t)n * batch);
    int* dInfo = cv.take<int>(batch);
    RLMB_CUDA_TRY(cudaMemcpyAsync(dA, h_a, nn * batch * sizeof(cplx), cudaMemcpyHostToDevice, ctx->stream));
    if (int rc = rlmb_heevd_batched(ctx, reinterpret_cast<double*>(dA), dW, n, batch, dInfo)) return rc;
    RLMB_CUDA_TRY(cudaMemcpyAsync(h_a, dA, nn * batch * sizeof(cplx), cudaMemcpyDeviceToHost, ctx->stream));
    RLMB_CUDA_TRY(cudaMemcpyAsync(h_w, dW, (size_t)n * batch * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<int> info(batch);
    RLMB_CUDA_TRY(cudaMemcpyAsync(info.data(), dInfo, batch * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    int bad = 0;
    for (int b = 0; b < batch; ++b) bad += info[b] != 0;
    return bad;
}

int rlmb_rlm_potential(rlmb_context* ctx, const double* d_x, const double* d_y, const double* d_s,
                       int impurity_num, int n_samples, const double* d_coeff_mn, int dim,
                       int off_head, double* d_vmn) {
    if (!ctx || !d_x || !d_y || !d_s || !d_coeff_mn || !d_vmn || impurity_num <= 0 || n_samples <= 0 ||
        dim != 2 * off_head + 1)
        return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (int rc = ensure_workspace(ctx, rlm_potential_ws_elems(impurity_num, n_samples, dim) * sizeof(cplx)))
        return rc;
    return launch_rlm_potential(ctx, d_x, d_y, d_s, impurity_num, n_samples,
                                reinterpret_cast<const cplx*>(d_coeff_mn), dim, off_head,
                                static_cast<cplx*>(ctx->ws), reinterpret_cast<cplx*>(d_vmn));
}

int rlmb_rlm_assemble(rlmb_context* ctx, const double* d_vmn, const double* d_coeff_m_theta,
                      const double* d_coeff_jm, int n_phi, int dim, int off_head, int n_mesh,
                      const int* h_theta1, const int* h_theta2, int count, double* d_h) {
    if (!ctx || !d_vmn || !d_coeff_m_theta || !d_coeff_jm || !h_theta1 || !h_theta2 || !d_h ||
        n_phi <= 0 || dim != 2 * off_head + 1 || count < 0)
        return RLMB_ERR_ARG;
    for (int i = 0; i < count; ++i)
        if (h_theta1[i] < 0 || h_theta1[i] > n_mesh || h_theta2[i] < 0 || h_theta2[i] > n_mesh)
            return RLMB_ERR_ARG;
    if (count == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    if (int rc = ensure_workspace(ctx, 2 * (size_t)count * sizeof(int))) return rc;
    int* d_t = static_cast<int*>(ctx->ws);
    RLMB_CUDA_TRY(cudaMemcpyAsync(d_t, h_theta1, count * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    RLMB_CUDA_TRY(cudaMemcpyAsync(d_t + count, h_theta2, count * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    return launch_rlm_assemble(ctx, reinterpret_cast<const cplx*>(d_vmn),
                               reinterpret_cast<const cplx*>(d_coeff_m_theta),
                               reinterpret_cast<const cplx*>(d_coeff_jm), d_t, d_t + count, count,
                               count, n_phi, dim, off_head, reinterpret_cast<cplx*>(d_h));
}

int rlmb_hlm_basis(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh, int theta_1,
                   int theta_2, double* d_wfs) {
    if (!ctx || !d_wfs || !hlm_args_ok(lx, ly, Q, band, n_mesh) || theta_1 < 0 || theta_2 < 0)
        return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    const int N = lx * ly / Q;
    if (int rc = ensure_workspace(ctx, (size_t)N * Q * sizeof(cplx))) return rc;
    cplx* hb = static_cast<cplx*>(ctx->ws);
    if (int rc = launch_hlm_bloch(ctx, lx, ly, Q, band, n_mesh, theta_1, theta_1 + 1, theta_2,
                                  theta_2 + 1, hb))
        return rc;
    return launch_hlm_basis_expand(ctx, hb, lx, ly, Q, n_mesh, theta_1, theta_2,
                                   reinterpret_cast<cplx*>(d_wfs));
}

int rlmb_hlm_project(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh,
                     const double* d_potential, const int* h_theta1, const int* h_theta2, int count,
                     double* d_h) {
    if (!ctx || !d_potential || !h_theta1 || !h_theta2 || !d_h || count < 0 ||
        !hlm_args_ok(lx, ly, Q, band, n_mesh))
        return RLMB_ERR_ARG;
    for (int i = 0; i < count; ++i)
        if (h_theta1[i] < 0 || h_theta1[i] > n_mesh || h_theta2[i] < 0 || h_theta2[i] > n_mesh)
            return RLMB_ERR_ARG;
    if (count == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    cplx* hb = nullptr;
    if (int rc = hlm_tables(ctx, lx, ly, Q, band, n_mesh, &hb)) return rc;
    const int ns = lx * ly;
    size_t bytes = 0;
    need<cplx>(bytes, ns);
    need<int>(bytes, count);
    if (int rc = ensure_workspace(ctx, bytes)) return rc;
    Carver cv(ctx->ws);
    cplx* vt = cv.take<cplx>(ns);
    int* d_t = cv.take<int>(count);
    std::vector<int> tl(count);
    for (int i = 0; i < count; ++i) tl[i] = h_theta1[i] * (n_mesh + 1) + h_theta2[i];
    RLMB_CUDA_TRY(cudaMemcpyAsync(d_t, tl.data(), count * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));   // tl is a host temporary
    if (int rc = launch_hlm_vtilde(ctx, d_potential, lx, ly, Q, 1, vt)) return rc;
    return launch_hlm_project(ctx, hb, vt, d_t, lx, ly, Q, count, 1, reinterpret_cast<cplx*>(d_h));
}

int rlmb_fhs_line(rlmb_context* ctx, const double* d_prev, const double* d_cur, int n_phi,
                  int dim_vec, int n_mesh, double* d_chern_theta) {
    if (!ctx || !d_prev || !d_cur || !d_chern_theta || n_phi <= 0 || dim_vec <= 0 || n_mesh <= 0)
        return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    return launch_fhs_line(ctx, reinterpret_cast<const cplx*>(d_prev),
                           reinterpret_cast<const cplx*>(d_cur), n_phi, dim_vec, n_mesh, d_chern_theta);
}

// --------------------------------------------------------------------- rlm pipeline
// Eigenvector matrices of one sample's mesh, already solved in place in d_H (kpts matrices
// of n x n complex128), written as wfs_<t1>_<t2>.bin under dir: the raw layout of the
// reference's write_wfs (diag_wrappers/wfs_file.cpp:2-11, dim_wfs complex values, column k
// = eigenvector k).  Device-to-host copies go through two pinned slots on the context
// stream, so that the copy of k-point t overlaps the file write of k-point t-1.
static int export_wfs(rlmb_context* ctx, const cplx* d_H, int n, int g, const char* dir) {
    const size_t nn = (size_t)n * n, bytes = nn * sizeof(cplx);
    const int kpts = (g + 1) * (g + 1);
    if (int rc = ensure_pinned(ctx, 2 * bytes)) return rc;
    unsigned char* slot[2] = {static_cast<unsigned char*>(ctx->pinned),
                              static_cast<unsigned char*>(ctx->pinned) + bytes};
    cudaEvent_t ev[2];
    RLMB_CUDA_TRY(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    if (cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        return RLMB_ERR_CUDA;
    }
    int rc = RLMB_OK;
    auto write = [&](int t) -> int {
        char name[4096];
        snprintf(name, sizeof(name), "%s/wfs_%d_%d.bin", dir, t / (g + 1), t % (g + 1));
        FILE* f = fopen(name, "wb");
        if (!f) {
            fprintf(stderr, "rlmb: cannot write %s\n", name);
            return RLMB_ERR_ARG;
        }
        const size_t w = fwrite(slot[t & 1], 1, bytes, f);
        fclose(f);
        return w == bytes ? RLMB_OK : RLMB_ERR_ARG;
    };
    for (int t = 0; t <= kpts && rc == RLMB_OK; ++t) {
        if (t < kpts) {
            if (cudaMemcpyAsync(slot[t & 1], d_H + (size_t)t * nn, bytes, cudaMemcpyDeviceToHost, ctx->stream) !=
                    cudaSuccess ||
                cudaEventRecord(ev[t & 1], ctx->stream) != cudaSuccess) {
                rc = RLMB_ERR_CUDA;
                break;
            }
        }
        if (t > 0) {
            if (cudaEventSynchronize(ev[(t - 1) & 1]) != cudaSuccess) {
                rc = RLMB_ERR_CUDA;
                break;
            }
            rc = write(t - 1);
        }
    }
    if (rc != RLMB_OK) cudaStreamSynchronize(ctx->stream);   // no copy left in flight into the slots
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return rc;
}

static int rlm_mesh(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh, unsigned long seed,
                    int sample0, int n_samples, double* energies, double* chern, bool dev_out, const char* wfs_dir);

int rlmb_rlm_mesh_solve(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh,
                        unsigned long seed, int sample0, int n_samples, double* h_energies,
                        double* h_chern) {
    return rlm_mesh(ctx, n_phi, qc, ic, n_mesh, seed, sample0, n_samples, h_energies, h_chern, false, nullptr);
}

int rlmb_rlm_mesh_solve_device(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh,
                               unsigned long seed, int sample0, int n_samples, double* d_energies,
                               double* d_chern) {
    return rlm_mesh(ctx, n_phi, qc, ic, n_mesh, seed, sample0, n_samples, d_energies, d_chern, true, nullptr);
}

int rlmb_rlm_mesh_export(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh,
                         unsigned long seed, int sample, const char* dir, double* h_energies,
                         double* h_chern) {
    if (!dir) return RLMB_ERR_ARG;
    return rlm_mesh(ctx, n_phi, qc, ic, n_mesh, seed, sample, 1, h_energies, h_chern, false, dir);
}

// One prepared rlm pipeline geometry: sizes, the batch of samples, and the regions of the
// context's pipeline buffer (coefficient tables and theta lists uploaded once).
struct RlmPlan {
    int n_phi, nimp, o, dim, g, kpts, nb, n_samples;
    double L1, L2;
    unsigned long seed;
    cplx *d_cmn, *d_cmt, *d_cjm, *d_vmn, *d_H, *d_U;
    double *d_imp, *d_W, *d_out;
    int *d_t, *d_info;
};

// Sizes (with the reference's C truncations, rlm/main_rlm_cpu.cpp:29-33), buffers and the
// disorder-independent tables of an rlm mesh call; synchronises the context stream.
static int rlm_prepare(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh, unsigned long seed,
                       int n_samples, RlmPlan* p) {
    const double L1 = std::sqrt(n_phi * qc), L2 = std::sqrt(n_phi * qc);
    const long nimp_l = (long)(ic * n_phi / qc);
    const long o_l = (long)(std::sqrt((double)nimp_l) / 2 + 1);
    if (nimp_l <= 0 || nimp_l > (1L << 28)) return RLMB_ERR_ARG;
    const int nimp = (int)nimp_l, o = (int)o_l, dim = 2 * o + 1;
    const int g = n_mesh, kpts = (g + 1) * (g + 1);
    const size_t nn = (size_t)n_phi * n_phi;
    std::vector<double> cmn(2 * (size_t)dim * dim), cmt(2 * (size_t)(g + 1) * dim), cjm(2 * (size_t)n_phi * dim);
    if (int rc = rlmb_rlm_coeff_tables(n_phi, o, dim, g, L1, L2, cmn.data(), cmt.data(), cjm.data())) return rc;
    // batch of samples that fits the budget
    const size_t per_sample = kpts * (nn * sizeof(cplx) + (size_t)n_phi * (sizeof(double) + 2 * sizeof(cplx))) +
                              (size_t)dim * dim * sizeof(cplx) + 3 * (size_t)nimp * sizeof(double);
    const int nb = balanced_batch(n_samples, mesh_budget_bytes(ctx) / per_sample);
    size_t bytes = 0;
    need<cplx>(bytes, cmn.size() / 2);
    need<cplx>(bytes, cmt.size() / 2);
    need<cplx>(bytes, cjm.size() / 2);
    need<double>(bytes, 3 * (size_t)nimp * nb);
    need<cplx>(bytes, (size_t)dim * dim * nb);
    need<int>(bytes, 2 * (size_t)kpts * nb);
    need<cplx>(bytes, nn * kpts * nb);
    need<double>(bytes, (size_t)n_phi * kpts * nb);
    need<cplx>(bytes, 2 * (size_t)n_phi * kpts * nb);
    need<double>(bytes, 2 * (size_t)n_phi * nb);
    need<int>(bytes, (size_t)kpts * nb);
    if (int rc = ensure_pipe(ctx, bytes)) return rc;
    Carver cv(ctx->pipe);
    *p = RlmPlan{};
    p->n_phi = n_phi;
    p->nimp = nimp;
    p->o = o;
    p->dim = dim;
    p->g = g;
    p->kpts = kpts;
    p->nb = nb;
    p->n_samples = n_samples;
    p->L1 = L1;
    p->L2 = L2;
    p->seed = seed;
    p->d_cmn = cv.take<cplx>(cmn.size() / 2);
    p->d_cmt = cv.take<cplx>(cmt.size() / 2);
    p->d_cjm = cv.take<cplx>(cjm.size() / 2);
    p->d_imp = cv.take<double>(3 * (size_t)nimp * nb);
    p->d_vmn = cv.take<cplx>((size_t)dim * dim * nb);
    p->d_t = cv.take<int>(2 * (size_t)kpts * nb);
    p->d_H = cv.take<cplx>(nn * kpts * nb);
    p->d_W = cv.take<double>((size_t)n_phi * kpts * nb);
    p->d_U = cv.take<cplx>(2 * (size_t)n_phi * kpts * nb);
    p->d_out = cv.take<double>(2 * (size_t)n_phi * nb);
    p->d_info = cv.take<int>((size_t)kpts * nb);
    if (int rc = ensure_pinned(ctx, 2 * (size_t)kpts * nb * sizeof(int))) return rc;
    if (int rc = ensure_workspace(ctx, rlm_potential_ws_elems(nimp, nb, dim) * sizeof(cplx))) return rc;
    RLMB_CUDA_TRY(cudaMemcpyAsync(p->d_cmn, cmn.data(), cmn.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    RLMB_CUDA_TRY(cudaMemcpyAsync(p->d_cmt, cmt.data(), cmt.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    RLMB_CUDA_TRY(cudaMemcpyAsync(p->d_cjm, cjm.data(), cjm.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    int* pt = static_cast<int*>(ctx->pinned);
    for (int s = 0; s < nb; ++s)
        for (int t = 0; t < kpts; ++t) {
            pt[s * kpts + t] = t / (g + 1);
            pt[(size_t)nb * kpts + s * kpts + t] = t % (g + 1);
        }
    RLMB_CUDA_TRY(cudaMemcpyAsync(p->d_t, pt, 2 * (size_t)kpts * nb * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    // the host tables are call-local and the pinned staging is reused by the next call: both
    // copies must have completed before this function returns
    RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return RLMB_OK;
}

// The stream-ordered work of an rlm mesh call on a prepared plan: samples sample0 ..
// sample0 + n_samples - 1 (plus *d_sample0 when given: the first sample index is then read
// from device memory, for a captured graph), energies / chern n_samples * n_phi values each,
// in device memory if dev_out, else in host memory.  No host round trips: eigensolve
// failures are tallied on the device.
static int rlm_enqueue(rlmb_context* ctx, const RlmPlan& p, int sample0, const int* d_sample0, double* energies,
                       double* chern, bool dev_out, const char* wfs_dir) {
    const int n_phi = p.n_phi, nimp = p.nimp, nb = p.nb, kpts = p.kpts, g = p.g, dim = p.dim, o = p.o;
    for (int s0 = 0; s0 < p.n_samples; s0 += nb) {
        const int cnt = std::min(nb, p.n_samples - s0);
        double* dx = p.d_imp;
        double* dy = p.d_imp + (size_t)nb * nimp;
        double* ds = p.d_imp + 2 * (size_t)nb * nimp;
        // disorder drawn on the device, bit-identical to the host stream (csrc/disorder.cu)
        if (d_sample0) {
            if (int rc = launch_rlm_disorder_at(ctx, nimp, p.L1, p.L2, p.seed, d_sample0, sample0 + s0, cnt, dx, dy, ds))
                return rc;
        } else if (int rc = rlmb_rlm_disorder_device(ctx, nimp, p.L1, p.L2, p.seed, sample0 + s0, cnt, dx, dy, ds)) {
            return rc;
        }
        if (int rc = launch_rlm_potential(ctx, dx, dy, ds, nimp, cnt, p.d_cmn, dim, o, static_cast<cplx*>(ctx->ws),
                                          p.d_vmn))
            return rc;
        if (int rc = launch_rlm_assemble(ctx, p.d_vmn, p.d_cmt, p.d_cjm, p.d_t, p.d_t + (size_t)nb * kpts, cnt * kpts,
                                         kpts, n_phi, dim, o, p.d_H))
            return rc;
        if (int rc = heevd_batched_band(ctx, reinterpret_cast<double*>(p.d_H), p.d_W, n_phi, cnt * kpts, p.d_info, o))
            return rc;
        if (int rc = tally_failures(ctx, p.d_info, cnt * kpts)) return rc;
        if (wfs_dir)
            if (int rc = export_wfs(ctx, p.d_H, n_phi, g, wfs_dir)) return rc;   // one sample (cnt == 1)
        cplx* d_U1 = p.d_U;
        cplx* d_U2 = p.d_U + (size_t)n_phi * kpts * nb;
        if (int rc = launch_rlm_links(ctx, p.d_H, n_phi, g, cnt, d_U1, d_U2)) return rc;
        double* out_e = dev_out ? energies + (size_t)s0 * n_phi : p.d_out;
        double* out_c = dev_out ? chern + (size_t)s0 * n_phi : p.d_out + (size_t)n_phi * nb;
        if (int rc = launch_plaquettes(ctx, d_U1, d_U2, p.d_W, n_phi, g, cnt, 0, out_e, out_c)) return rc;
        if (!dev_out) {
            RLMB_CUDA_TRY(cudaMemcpyAsync(energies + (size_t)s0 * n_phi, p.d_out, (size_t)cnt * n_phi * sizeof(double),
                                          cudaMemcpyDeviceToHost, ctx->stream));
            RLMB_CUDA_TRY(cudaMemcpyAsync(chern + (size_t)s0 * n_phi, p.d_out + (size_t)n_phi * nb,
                                          (size_t)cnt * n_phi * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    return RLMB_OK;
}

// The rlm pipeline: energies / chern receive n_samples * n_phi values each, in device memory
// if dev_out, else in host memory.  After its set-up the call's device work is stream-ordered
// without host round trips between batches; it synchronises once, at the end, to return its
// status.
static int rlm_mesh(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh, unsigned long seed,
                    int sample0, int n_samples, double* energies, double* chern, bool dev_out, const char* wfs_dir) {
    if (!ctx || n_phi <= 0 || !(qc > 0) || !(ic > 0) || n_mesh <= 0 || sample0 < 0 || n_samples < 0 ||
        (n_samples > 0 && (!energies || !chern)))
        return RLMB_ERR_ARG;
    if (n_samples == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    RlmPlan p;
    if (int rc = rlm_prepare(ctx, n_phi, qc, ic, n_mesh, seed, n_samples, &p)) return rc;
    if (int rc = reset_failures(ctx)) return rc;
    if (int rc = rlm_enqueue(ctx, p, sample0, nullptr, energies, chern, dev_out, wfs_dir)) return rc;
    return finish_call(ctx);
}

// ----------------------------------------------- rlm orders captured in one CUDA graph
// Several rlm mesh geometries (a finite-size-scaling set of n_phi) solved by ONE graph launch
// per step.  Each order has its own library context (stream, workspace, pipeline buffers and
// failure counter), prepared and run once outside the capture so that every buffer has its
// final size; the capture then forks one branch per order from the graph's origin stream,
// records each order's whole pipeline (disorder, V_mn, assembly, eigensolve, links,
// plaquettes, device-side failure tally) on its context stream, and joins them.  The orders
// run concurrently on the device: the small ones fill the SMs the large ones leave idle.
// The first sample of a launch is written to device memory just before the graph runs, and
// the disorder kernels read it there.  Each order's eigensolver launch configuration is
// autotuned (rlmb_set_autotune) during its set-up run.
struct FssOrder {
    rlmb_context* ctx;
    RlmPlan plan;
    double* d_e;   // n_samples * n_phi energies, then as many Chern numbers
    cudaEvent_t done;
};

struct rlmb_fss_graph {
    int device;
    int n_samples;
    std::vector<FssOrder> orders;
    cudaStream_t origin;
    cudaEvent_t fork;
    int* d_sample0;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

__global__ void k_store_int(int* p, int v) { *p = v; }

static void fss_release(rlmb_fss_graph* f) {
    if (!f) return;
    cudaSetDevice(f->device);
    if (f->origin) cudaStreamSynchronize(f->origin);
    if (f->exec) cudaGraphExecDestroy(f->exec);
    if (f->graph) cudaGraphDestroy(f->graph);
    for (FssOrder& o : f->orders) {
        if (o.ctx) {
            cudaStream_t st = o.ctx->stream;
            rlmb_destroy(o.ctx);
            if (st) cudaStreamDestroy(st);
        }
        if (o.d_e) cudaFree(o.d_e);
        if (o.done) cudaEventDestroy(o.done);
    }
    if (f->d_sample0) cudaFree(f->d_sample0);
    if (f->fork) cudaEventDestroy(f->fork);
    if (f->origin) cudaStreamDestroy(f->origin);
    delete f;
}

int rlmb_rlm_fss_graph_create(int device, const int* n_phi, int count, double qc, double ic, int n_mesh,
                              unsigned long seed, int n_samples, int precision, rlmb_fss_graph** out) {
    if (!out) return RLMB_ERR_ARG;
    *out = nullptr;
    if (!n_phi || count <= 0 || count > 64 || !(qc > 0) || !(ic > 0) || n_mesh <= 0 || n_samples <= 0 ||
        (precision != RLMB_PRECISION_FP64 && precision != RLMB_PRECISION_MIXED))
        return RLMB_ERR_ARG;
    for (int i = 0; i < count; ++i)
        if (n_phi[i] <= 0) return RLMB_ERR_ARG;
    rlmb_fss_graph* f = new rlmb_fss_graph();
    f->device = device;
    f->n_samples = n_samples;
    f->orders.resize(count);
    for (FssOrder& o : f->orders) o = FssOrder{nullptr, RlmPlan{}, nullptr, nullptr};
    f->origin = nullptr;
    f->fork = nullptr;
    f->d_sample0 = nullptr;
    f->graph = nullptr;
    f->exec = nullptr;
    int rc = rlmb_create(&f->orders[0].ctx, device);   // (also validates the device)
    if (rc == RLMB_OK) {
        rlmb_destroy(f->orders[0].ctx);
        f->orders[0].ctx = nullptr;
    }
    auto fail = [&](int code) {
        fss_release(f);
        return code;
    };
    if (rc) return fail(rc);
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&f->origin, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&f->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&f->d_sample0), sizeof(int)) != cudaSuccess ||
        cudaMemset(f->d_sample0, 0, sizeof(int)) != cudaSuccess)
        return fail(RLMB_ERR_CUDA);
    // set-up and one uncaptured run per order: every buffer reaches its final size
    for (int i = 0; i < count; ++i) {
        FssOrder& o = f->orders[i];
        cudaStream_t st = nullptr;
        if ((rc = rlmb_create(&o.ctx, device))) return fail(rc);
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&o.done, cudaEventDisableTiming) != cudaSuccess) {
            if (st) cudaStreamDestroy(st);
            return fail(RLMB_ERR_CUDA);
        }
        o.ctx->stream = st;
        o.ctx->precision = precision;
        o.ctx->autotune = 1;   // the set-up run tunes this order's eigensolver configuration
        if (cudaMalloc(reinterpret_cast<void**>(&o.d_e), 2 * (size_t)n_samples * n_phi[i] * sizeof(double)) != cudaSuccess)
            return fail(RLMB_ERR_ALLOC);
        if ((rc = rlm_prepare(o.ctx, n_phi[i], qc, ic, n_mesh, seed, n_samples, &o.plan))) return fail(rc);
        if ((rc = reset_failures(o.ctx))) return fail(rc);
        if ((rc = rlm_enqueue(o.ctx, o.plan, 0, f->d_sample0, o.d_e, o.d_e + (size_t)n_samples * n_phi[i], true,
                              nullptr)))
            return fail(rc);
        if ((rc = finish_call(o.ctx)) < 0) return fail(rc);
    }
    // capture: fork, one branch per order, join
    if (cudaStreamBeginCapture(f->origin, cudaStreamCaptureModeRelaxed) != cudaSuccess) return fail(RLMB_ERR_CUDA);
    rc = cudaEventRecord(f->fork, f->origin) == cudaSuccess ? RLMB_OK : RLMB_ERR_CUDA;
    for (int i = 0; i < count && rc == RLMB_OK; ++i) {
        FssOrder& o = f->orders[i];
        if (cudaStreamWaitEvent(o.ctx->stream, f->fork, 0) != cudaSuccess) {
            rc = RLMB_ERR_CUDA;
            break;
        }
        o.ctx->frozen = 1;
        if (cudaMemsetAsync(o.ctx->fail, 0, sizeof(int), o.ctx->stream) != cudaSuccess) rc = RLMB_ERR_CUDA;
        if (rc == RLMB_OK)
            rc = rlm_enqueue(o.ctx, o.plan, 0, f->d_sample0, o.d_e, o.d_e + (size_t)n_samples * n_phi[i], true, nullptr);
        o.ctx->frozen = 0;
        if (rc == RLMB_OK && (cudaEventRecord(o.done, o.ctx->stream) != cudaSuccess ||
                              cudaStreamWaitEvent(f->origin, o.done, 0) != cudaSuccess))
            rc = RLMB_ERR_CUDA;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(f->origin, &graph);
    f->graph = graph;
    if (rc == RLMB_OK && ec != cudaSuccess) rc = RLMB_ERR_CUDA;
    if (rc != RLMB_OK) {
        cudaGetLastError();
        return fail(rc);
    }
    if (cudaGraphInstantiate(&f->exec, f->graph, 0) != cudaSuccess) return fail(RLMB_ERR_CUDA);
    *out = f;
    return RLMB_OK;
}

int rlmb_rlm_fss_graph_launch(rlmb_fss_graph* f, int sample0) {
    if (!f || sample0 < 0) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(f->device));
    k_store_int<<<1, 1, 0, f->origin>>>(f->d_sample0, sample0);
    RLMB_CUDA_TRY(cudaGetLastError());
    RLMB_CUDA_TRY(cudaGraphLaunch(f->exec, f->origin));
    return RLMB_OK;
}

int rlmb_rlm_fss_graph_stream(rlmb_fss_graph* f, void** stream) {
    if (!f || !stream) return RLMB_ERR_ARG;
    *stream = f->origin;
    return RLMB_OK;
}

int rlmb_rlm_fss_graph_results(rlmb_fss_graph* f, int index, double* h_energies, double* h_chern) {
    if (!f || index < 0 || index >= (int)f->orders.size() || !h_energies || !h_chern) return RLMB_ERR_ARG;
    RLMB_CUDA_TRY(cudaSetDevice(f->device));
    RLMB_CUDA_TRY(cudaStreamSynchronize(f->origin));
    const FssOrder& o = f->orders[index];
    const size_t cnt = (size_t)f->n_samples * o.plan.n_phi;
    RLMB_CUDA_TRY(cudaMemcpy(h_energies, o.d_e, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    RLMB_CUDA_TRY(cudaMemcpy(h_chern, o.d_e + cnt, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    int fails = 0;
    RLMB_CUDA_TRY(cudaMemcpy(&fails, o.ctx->fail, sizeof(int), cudaMemcpyDeviceToHost));
    return fails > 0 ? fails : RLMB_OK;
}

int rlmb_rlm_fss_graph_destroy(rlmb_fss_graph* f) {
    if (!f) return RLMB_ERR_ARG;
    fss_release(f);
    return RLMB_OK;
}

// --------------------------------------------------------------------- hlm pipeline
int rlmb_hlm_mesh_solve_device(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh,
                               const double* d_potentials, int n_samples, double* d_energies,
                               double* d_chern) {
    if (!ctx || !hlm_args_ok(lx, ly, Q, band, n_mesh) || n_samples < 0 ||
        (n_samples > 0 && (!d_potentials || !d_energies || !d_chern)))
        return RLMB_ERR_ARG;
    if (n_samples == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    const int g = n_mesh, N = lx * ly / Q, ns = lx * ly;
    const int kpts = (g + 1) * g;   // theta_1 in [0,g], theta_2 in [0,g)
    const size_t nn = (size_t)N * N;
    cplx* hb = nullptr;
    if (int rc = hlm_tables(ctx, lx, ly, Q, band, g, &hb)) return rc;
    const size_t per_sample = kpts * (nn * sizeof(cplx) + (size_t)N * (sizeof(double) + 2 * sizeof(cplx))) +
                              (size_t)ns * sizeof(cplx);
    const int nb = balanced_batch(n_samples, mesh_budget_bytes(ctx) / per_sample);
    size_t bytes = 0;
    need<int>(bytes, kpts);
    need<cplx>(bytes, (size_t)ns * nb);
    need<cplx>(bytes, nn * kpts * nb);
    need<double>(bytes, (size_t)N * kpts * nb);
    need<cplx>(bytes, 2 * (size_t)N * kpts * nb);
    need<int>(bytes, (size_t)kpts * nb);
    if (int rc = ensure_pipe(ctx, bytes)) return rc;
    Carver cv(ctx->pipe);
    int* d_t = cv.take<int>(kpts);
    cplx* d_vt = cv.take<cplx>((size_t)ns * nb);
    cplx* d_H = cv.take<cplx>(nn * kpts * nb);
    double* d_W = cv.take<double>((size_t)N * kpts * nb);
    cplx* d_U1 = cv.take<cplx>((size_t)N * kpts * nb);
    cplx* d_U2 = cv.take<cplx>((size_t)N * kpts * nb);
    int* d_info = cv.take<int>((size_t)kpts * nb);
    if (int rc = reset_failures(ctx)) return rc;
    {
        std::vector<int> tl(kpts);
        for (int t1 = 0; t1 <= g; ++t1)
            for (int t2 = 0; t2 < g; ++t2) tl[t1 * g + t2] = t1 * (g + 1) + t2;
        RLMB_CUDA_TRY(cudaMemcpyAsync(d_t, tl.data(), kpts * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    for (int s0 = 0; s0 < n_samples; s0 += nb) {
        const int cnt = std::min(nb, n_samples - s0);
        if (int rc = launch_hlm_vtilde(ctx, d_potentials + (size_t)s0 * ns, lx, ly, Q, cnt, d_vt)) return rc;
        if (int rc = launch_hlm_project(ctx, hb, d_vt, d_t, lx, ly, Q, kpts, cnt, d_H)) return rc;
        if (int rc = rlmb_heevd_batched(ctx, reinterpret_cast<double*>(d_H), d_W, N, cnt * kpts, d_info))
            return rc;
        if (int rc = tally_failures(ctx, d_info, cnt * kpts)) return rc;
        if (int rc = launch_hlm_links(ctx, hb, d_H, lx, ly, Q, g, cnt, d_U1, d_U2)) return rc;
        if (int rc = launch_plaquettes(ctx, d_U1, d_U2, d_W, N, g, cnt, 1, d_energies + (size_t)s0 * N,
                                       d_chern + (size_t)s0 * N))
            return rc;
    }
    return finish_call(ctx);
}

int rlmb_hlm_mesh_solve(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh,
                        const double* h_potentials, int n_samples, double* h_energies, double* h_chern) {
    if (!ctx || !hlm_args_ok(lx, ly, Q, band, n_mesh) || n_samples < 0 ||
        (n_samples > 0 && (!h_potentials || !h_energies || !h_chern)))
        return RLMB_ERR_ARG;
    if (n_samples == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    const int N = lx * ly / Q, ns = lx * ly;
    const size_t io = ((size_t)ns + 2 * (size_t)N) * n_samples;
    if (int rc = ensure_io(ctx, io * sizeof(double))) return rc;   // grow-only staging, kept by the context
    double* d_pot = static_cast<double*>(ctx->io);
    double* d_e = d_pot + (size_t)ns * n_samples;
    double* d_c = d_e + (size_t)N * n_samples;
    RLMB_CUDA_TRY(cudaMemcpyAsync(d_pot, h_potentials, (size_t)ns * n_samples * sizeof(double), cudaMemcpyHostToDevice,
                                  ctx->stream));
    const int rc = rlmb_hlm_mesh_solve_device(ctx, lx, ly, Q, band, n_mesh, d_pot, n_samples, d_e, d_c);
    if (rc < 0) return rc;
    RLMB_CUDA_TRY(cudaMemcpyAsync(h_energies, d_e, (size_t)N * n_samples * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    RLMB_CUDA_TRY(cudaMemcpyAsync(h_chern, d_c, (size_t)N * n_samples * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return rc;
}

}  // extern "C"
