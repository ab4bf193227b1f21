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

// Adds the number of nonzero entries of d_info[0..count) to *failures (synchronous).
static int count_failures(rlmb_context* ctx, const int* d_info, int count, long long* failures) {
    std::vector<int> h(count);
    RLMB_CUDA_TRY(cudaMemcpyAsync(h.data(), d_info, count * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < count; ++i) *failures += h[i] != 0;
    return RLMB_OK;
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
    if (ctx->ws) cudaFree(ctx->ws);
    if (ctx->pipe) cudaFree(ctx->pipe);
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
                    int sample0, int n_samples, double* h_energies, double* h_chern, const char* wfs_dir);

int rlmb_rlm_mesh_solve(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh,
                        unsigned long seed, int sample0, int n_samples, double* h_energies,
                        double* h_chern) {
    return rlm_mesh(ctx, n_phi, qc, ic, n_mesh, seed, sample0, n_samples, h_energies, h_chern, nullptr);
}

int rlmb_rlm_mesh_export(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh,
                         unsigned long seed, int sample, const char* dir, double* h_energies,
                         double* h_chern) {
    if (!dir) return RLMB_ERR_ARG;
    return rlm_mesh(ctx, n_phi, qc, ic, n_mesh, seed, sample, 1, h_energies, h_chern, dir);
}

static int rlm_mesh(rlmb_context* ctx, int n_phi, double qc, double ic, int n_mesh, unsigned long seed,
                    int sample0, int n_samples, double* h_energies, double* h_chern, const char* wfs_dir) {
    if (!ctx || n_phi <= 0 || !(qc > 0) || !(ic > 0) || n_mesh <= 0 || sample0 < 0 || n_samples < 0 ||
        (n_samples > 0 && (!h_energies || !h_chern)))
        return RLMB_ERR_ARG;
    if (n_samples == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    // derived sizes, with the reference's C truncations (rlm/main_rlm_cpu.cpp:29-33)
    const double L1 = std::sqrt(n_phi * qc), L2 = std::sqrt(n_phi * qc);
    const long nimp_l = (long)(ic * n_phi / qc);
    const long o_l = (long)(std::sqrt((double)nimp_l) / 2 + 1);
    if (nimp_l <= 0 || nimp_l > (1L << 28)) return RLMB_ERR_ARG;
    const int nimp = (int)nimp_l, o = (int)o_l, dim = 2 * o + 1;
    const int g = n_mesh, kpts = (g + 1) * (g + 1);
    const size_t nn = (size_t)n_phi * n_phi;
    // host tables
    std::vector<double> cmn(2 * (size_t)dim * dim), cmt(2 * (size_t)(g + 1) * dim), cjm(2 * (size_t)n_phi * dim);
    if (int rc = rlmb_rlm_coeff_tables(n_phi, o, dim, g, L1, L2, cmn.data(), cmt.data(), cjm.data())) return rc;
    // batch of samples that fits the budget
    const size_t per_sample = kpts * (nn * sizeof(cplx) + (size_t)n_phi * (sizeof(double) + 2 * sizeof(cplx))) +
                              (size_t)dim * dim * sizeof(cplx) + 3 * (size_t)nimp * sizeof(double);
    int nb = balanced_batch(n_samples, mesh_budget_bytes(ctx) / per_sample);
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
    cplx* d_cmn = cv.take<cplx>(cmn.size() / 2);
    cplx* d_cmt = cv.take<cplx>(cmt.size() / 2);
    cplx* d_cjm = cv.take<cplx>(cjm.size() / 2);
    double* d_imp = cv.take<double>(3 * (size_t)nimp * nb);
    cplx* d_vmn = cv.take<cplx>((size_t)dim * dim * nb);
    int* d_t = cv.take<int>(2 * (size_t)kpts * nb);
    cplx* d_H = cv.take<cplx>(nn * kpts * nb);
    double* d_W = cv.take<double>((size_t)n_phi * kpts * nb);
    cplx* d_U = cv.take<cplx>(2 * (size_t)n_phi * kpts * nb);
    double* d_out = cv.take<double>(2 * (size_t)n_phi * nb);
    int* d_info = cv.take<int>((size_t)kpts * nb);
    long long failures = 0;
    if (int rc = ensure_pinned(ctx, std::max(3 * (size_t)nimp * nb * sizeof(double), 2 * (size_t)kpts * nb * sizeof(int))))
        return rc;
    RLMB_CUDA_TRY(cudaMemcpyAsync(d_cmn, cmn.data(), cmn.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    RLMB_CUDA_TRY(cudaMemcpyAsync(d_cmt, cmt.data(), cmt.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    RLMB_CUDA_TRY(cudaMemcpyAsync(d_cjm, cjm.data(), cjm.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    {
        int* pt = static_cast<int*>(ctx->pinned);
        for (int s = 0; s < nb; ++s)
            for (int t = 0; t < kpts; ++t) {
                pt[s * kpts + t] = t / (g + 1);
                pt[(size_t)nb * kpts + s * kpts + t] = t % (g + 1);
            }
        RLMB_CUDA_TRY(cudaMemcpyAsync(d_t, pt, 2 * (size_t)kpts * nb * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    for (int s0 = 0; s0 < n_samples; s0 += nb) {
        const int cnt = std::min(nb, n_samples - s0);
        // disorder drawn on the device, bit-identical to the host stream (csrc/disorder.cu)
        if (int rc = rlmb_rlm_disorder_device(ctx, nimp, L1, L2, seed, sample0 + s0, cnt, d_imp,
                                              d_imp + (size_t)nb * nimp, d_imp + 2 * (size_t)nb * nimp))
            return rc;
        if (int rc = ensure_workspace(ctx, rlm_potential_ws_elems(nimp, cnt, dim) * sizeof(cplx))) return rc;
        if (int rc = launch_rlm_potential(ctx, d_imp, d_imp + (size_t)nb * nimp, d_imp + 2 * (size_t)nb * nimp,
                                          nimp, cnt, d_cmn, dim, o, static_cast<cplx*>(ctx->ws), d_vmn))
            return rc;
        if (int rc = launch_rlm_assemble(ctx, d_vmn, d_cmt, d_cjm, d_t, d_t + (size_t)nb * kpts, cnt * kpts, kpts,
                                         n_phi, dim, o, d_H))
            return rc;
        if (int rc = rlmb_heevd_batched(ctx, reinterpret_cast<double*>(d_H), d_W, n_phi, cnt * kpts, d_info))
            return rc;
        if (int rc = count_failures(ctx, d_info, cnt * kpts, &failures)) return rc;
        if (wfs_dir)
            if (int rc = export_wfs(ctx, d_H, n_phi, g, wfs_dir)) return rc;   // one sample (cnt == 1)
        cplx* d_U1 = d_U;
        cplx* d_U2 = d_U + (size_t)n_phi * kpts * nb;
        if (int rc = launch_rlm_links(ctx, d_H, n_phi, g, cnt, d_U1, d_U2)) return rc;
        if (int rc = launch_plaquettes(ctx, d_U1, d_U2, d_W, n_phi, g, cnt, 0, d_out, d_out + (size_t)n_phi * nb))
            return rc;
        RLMB_CUDA_TRY(cudaMemcpyAsync(h_energies + (size_t)s0 * n_phi, d_out, (size_t)cnt * n_phi * sizeof(double),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        RLMB_CUDA_TRY(cudaMemcpyAsync(h_chern + (size_t)s0 * n_phi, d_out + (size_t)n_phi * nb,
                                      (size_t)cnt * n_phi * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        RLMB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    return failures > 0 ? (int)std::min<long long>(failures, 1 << 30) : RLMB_OK;
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
    long long failures = 0;
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
        if (int rc = count_failures(ctx, d_info, cnt * kpts, &failures)) return rc;
        if (int rc = launch_hlm_links(ctx, hb, d_H, lx, ly, Q, g, cnt, d_U1, d_U2)) return rc;
        if (int rc = launch_plaquettes(ctx, d_U1, d_U2, d_W, N, g, cnt, 1, d_energies + (size_t)s0 * N,
                                       d_chern + (size_t)s0 * N))
            return rc;
    }
    return failures > 0 ? (int)std::min<long long>(failures, 1 << 30) : RLMB_OK;
}

int rlmb_hlm_mesh_solve(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh,
                        const double* h_potentials, int n_samples, double* h_energies, double* h_chern) {
    if (!ctx || !hlm_args_ok(lx, ly, Q, band, n_mesh) || n_samples < 0 ||
        (n_samples > 0 && (!h_potentials || !h_energies || !h_chern)))
        return RLMB_ERR_ARG;
    if (n_samples == 0) return RLMB_OK;
    RLMB_CUDA_TRY(cudaSetDevice(ctx->device));
    const int N = lx * ly / Q, ns = lx * ly;
    double* d_io = nullptr;
    const size_t io = ((size_t)ns + 2 * (size_t)N) * n_samples;
    RLMB_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d_io), io * sizeof(double), ctx->stream));
    int rc = RLMB_OK;
    double* d_pot = d_io;
    double* d_e = d_io + (size_t)ns * n_samples;
    double* d_c = d_e + (size_t)N * n_samples;
    if (cudaMemcpyAsync(d_pot, h_potentials, (size_t)ns * n_samples * sizeof(double), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess)
        rc = RLMB_ERR_CUDA;
    if (rc == RLMB_OK) rc = rlmb_hlm_mesh_solve_device(ctx, lx, ly, Q, band, n_mesh, d_pot, n_samples, d_e, d_c);
    if (rc == RLMB_OK) {
        if (cudaMemcpyAsync(h_energies, d_e, (size_t)N * n_samples * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream) != cudaSuccess ||
            cudaMemcpyAsync(h_chern, d_c, (size_t)N * n_samples * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream) != cudaSuccess)
            rc = RLMB_ERR_CUDA;
    }
    cudaFreeAsync(d_io, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = RLMB_ERR_CUDA;
    return rc;
}

}  // extern "C"
