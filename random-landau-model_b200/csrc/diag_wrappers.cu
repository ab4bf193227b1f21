// The reference's C++ entry points (include/diag_wrappers_b200.h) on the B200 library.
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/diag_wrappers_b200.h"
#include "common.cuh"

namespace {

// One library context per host thread (the reference calls mkl_heevd concurrently from
// pthreads, rlm/hamiltonian_rlm_cpu.cpp:49).
rlmb_context* thread_ctx() {
    static thread_local rlmb_context* ctx = nullptr;
    if (!ctx) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            dev = 0;
        }
        if (rlmb_create(&ctx, dev) != RLMB_OK) ctx = nullptr;
    }
    return ctx;
}

void report(const char* fn, int rc) {
    if (rc != RLMB_OK) fprintf(stderr, "%s: %s (status %d)\n", fn, rlmb_status_string(rc), rc);
}

// Single-precision column-major matrix whose LOWER triangle holds the Hermitian matrix
// (cusolver/MAGMA calls of the reference use uplo = lower) -> double-precision buffer whose
// upper triangle (read by the library) holds the same matrix.
__global__ void k_lower_c64_to_upper_c128(const cuFloatComplex* __restrict__ in, rlmb::cplx* __restrict__ out,
                                          int n) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * n) return;
    const int c = (int)(idx / n), r = (int)(idx % n);
    // upper element (r <= c) of column c = conj of lower element (c, r) of column r
    const cuFloatComplex x = r <= c ? in[(size_t)r * n + c] : in[idx];
    out[idx] = r <= c ? rlmb::mk(x.x, -x.y) : rlmb::mk(x.x, x.y);
}
__global__ void k_c128_to_c64(const rlmb::cplx* __restrict__ in, cuFloatComplex* __restrict__ out, size_t count) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < count) out[idx] = make_cuFloatComplex((float)in[idx].x, (float)in[idx].y);
}
__global__ void k_f64_to_f32(const double* __restrict__ in, float* __restrict__ out, int count) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < count) out[idx] = (float)in[idx];
}

// Shared body of the single-precision device wrappers: solves in double precision,
// returns eigenvectors in dev_wfs and eigenvalues in d_w64 (device, double).
int solve_fp32_device(rlmb_context* ctx, cuFloatComplex* dev_wfs, int n, double** d_w64, rlmb::cplx** buf) {
    const size_t nn = (size_t)n * n;
    if (cudaMalloc(reinterpret_cast<void**>(buf), nn * sizeof(rlmb::cplx) + n * sizeof(double)) != cudaSuccess)
        return RLMB_ERR_ALLOC;
    *d_w64 = reinterpret_cast<double*>(*buf + nn);
    const unsigned blocks = (unsigned)((nn + 255) / 256);
    k_lower_c64_to_upper_c128<<<blocks, 256, 0, ctx->stream>>>(dev_wfs, *buf, n);
    int rc = rlmb_heevd_batched(ctx, reinterpret_cast<double*>(*buf), *d_w64, n, 1, nullptr);
    if (rc < 0) return rc;
    k_c128_to_c64<<<blocks, 256, 0, ctx->stream>>>(*buf, dev_wfs, nn);
    return cudaGetLastError() == cudaSuccess ? RLMB_OK : RLMB_ERR_CUDA;
}

int chern_line(const std::complex<double>* wfs_full, double* chern_theta, int n_phi, int dim_vec, int n_mesh,
               int theta_1) {
    rlmb_context* ctx = thread_ctx();
    if (!ctx) return RLMB_ERR_NO_DEVICE;
    const size_t line = (size_t)(n_mesh + 1) * n_phi * dim_vec;
    const int cur = theta_1 % 2, prev = 1 - theta_1 % 2;   // ring slots (chern.cpp:15-18)
    void* d = nullptr;
    if (cudaMalloc(&d, 2 * line * sizeof(rlmb::cplx) + (size_t)n_mesh * n_phi * sizeof(double)) != cudaSuccess)
        return RLMB_ERR_ALLOC;
    rlmb::cplx* dprev = static_cast<rlmb::cplx*>(d);
    rlmb::cplx* dcur = dprev + line;
    double* dout = reinterpret_cast<double*>(dcur + line);
    int rc = RLMB_OK;
    if (cudaMemcpy(dprev, wfs_full + prev * line, line * sizeof(rlmb::cplx), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dcur, wfs_full + cur * line, line * sizeof(rlmb::cplx), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = RLMB_ERR_CUDA;
    if (rc == RLMB_OK)
        rc = rlmb_fhs_line(ctx, reinterpret_cast<double*>(dprev), reinterpret_cast<double*>(dcur), n_phi, dim_vec,
                           n_mesh, dout);
    if (rc == RLMB_OK &&
        cudaMemcpy(chern_theta, dout, (size_t)n_mesh * n_phi * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = RLMB_ERR_CUDA;
    cudaFree(d);
    return rc;
}

}  // namespace

void mkl_heevd(std::complex<double>* hamiltonian, double* energy, int l) {
    rlmb_context* ctx = thread_ctx();
    if (!ctx) return report("mkl_heevd", RLMB_ERR_NO_DEVICE);
    const int rc = rlmb_heevd_host(ctx, reinterpret_cast<double*>(hamiltonian), energy, l, 1);
    report("mkl_heevd", rc);
}

void cusolver_diag_hamil(cuFloatComplex* dev_wfs, float* dev_energy, int n_phi) {
    rlmb_context* ctx = thread_ctx();
    if (!ctx || !dev_wfs || !dev_energy || n_phi <= 0) return report("cusolver_diag_hamil", RLMB_ERR_ARG);
    rlmb_set_stream(ctx, nullptr);   // the reference's default stream
    double* w64 = nullptr;
    rlmb::cplx* buf = nullptr;
    int rc = solve_fp32_device(ctx, dev_wfs, n_phi, &w64, &buf);
    if (rc == RLMB_OK) {
        k_f64_to_f32<<<(n_phi + 255) / 256, 256, 0, ctx->stream>>>(w64, dev_energy, n_phi);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = RLMB_ERR_CUDA;
    }
    if (buf) cudaFree(buf);
    report("cusolver_diag_hamil", rc);
}

void magma_diag_hamil(cuFloatComplex* dev_wfs, float* energy, int n_phi) {
    rlmb_context* ctx = thread_ctx();
    if (!ctx || !dev_wfs || !energy || n_phi <= 0) return report("magma_diag_hamil", RLMB_ERR_ARG);
    rlmb_set_stream(ctx, nullptr);
    double* w64 = nullptr;
    rlmb::cplx* buf = nullptr;
    int rc = solve_fp32_device(ctx, dev_wfs, n_phi, &w64, &buf);
    if (rc == RLMB_OK) {
        std::vector<double> w(n_phi);
        if (cudaMemcpy(w.data(), w64, n_phi * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = RLMB_ERR_CUDA;
        for (int i = 0; i < n_phi; ++i) energy[i] = (float)w[i];
    }
    if (buf) cudaFree(buf);
    report("magma_diag_hamil", rc);
}

void cal_Chern(std::complex<double>* wfs_full, double* chern_numbers_theta, int n_phi, int dim_vec, int n_mesh,
               int theta_1) {
    report("cal_Chern", chern_line(wfs_full, chern_numbers_theta, n_phi, dim_vec, n_mesh, theta_1));
}

void* peer_cal_Chern(void* peer_Chern_params) {
    struct_Chern* p = static_cast<struct_Chern*>(peer_Chern_params);
    std::vector<double> all((size_t)p->n_mesh * p->n_phi);
    const int rc = chern_line(p->wave_function, all.data(), p->n_phi, p->dim_vec, p->n_mesh, p->theta_1);
    report("peer_cal_Chern", rc);
    if (rc == RLMB_OK)
        for (int l = 0; l < p->theta_len; ++l) {
            const int m = p->theta_2[l];
            for (int n = 0; n < p->n_phi; ++n)
                p->chern_numbers_theta[m + (size_t)n * p->n_mesh] = all[m + (size_t)n * p->n_mesh];
        }
    return peer_Chern_params;
}

void prepare_coeff(std::complex<double>* coeff_mn, std::complex<double>* coeff_m_theta,
                   std::complex<double>* coeff_jm, int n_phi, int off_head, int dim_m, int dim_n, int n_mesh,
                   double L1, double L2) {
    if (dim_m != dim_n) return report("prepare_coeff", RLMB_ERR_ARG);
    report("prepare_coeff", rlmb_rlm_coeff_tables(n_phi, off_head, dim_m, n_mesh, L1, L2,
                                                 reinterpret_cast<double*>(coeff_mn),
                                                 reinterpret_cast<double*>(coeff_m_theta),
                                                 reinterpret_cast<double*>(coeff_jm)));
}

void get_potential_coeff(double* impurity_x, double* impurity_y, double* impurity_intensity,
                         std::complex<double>* Vmn, std::complex<double>* coeff_mn, int dim_m, int dim_n,
                         int off_head, int impurity_num) {
    rlmb_context* ctx = thread_ctx();
    if (!ctx || dim_m != dim_n) return report("get_potential_coeff", RLMB_ERR_ARG);
    const size_t dd = (size_t)dim_m * dim_n;
    void* d = nullptr;
    if (cudaMalloc(&d, 3 * (size_t)impurity_num * sizeof(double) + 2 * dd * sizeof(rlmb::cplx)) != cudaSuccess)
        return report("get_potential_coeff", RLMB_ERR_ALLOC);
    double* dx = static_cast<double*>(d);
    double* dy = dx + impurity_num;
    double* ds = dy + impurity_num;
    rlmb::cplx* dc = reinterpret_cast<rlmb::cplx*>(ds + impurity_num);
    rlmb::cplx* dv = dc + dd;
    int rc = RLMB_OK;
    if (cudaMemcpy(dx, impurity_x, impurity_num * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dy, impurity_y, impurity_num * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(ds, impurity_intensity, impurity_num * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dc, coeff_mn, dd * sizeof(rlmb::cplx), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = RLMB_ERR_CUDA;
    if (rc == RLMB_OK)
        rc = rlmb_rlm_potential(ctx, dx, dy, ds, impurity_num, 1, reinterpret_cast<double*>(dc), dim_m, off_head,
                                reinterpret_cast<double*>(dv));
    if (rc == RLMB_OK && cudaMemcpy(Vmn, dv, dd * sizeof(rlmb::cplx), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = RLMB_ERR_CUDA;
    cudaFree(d);
    report("get_potential_coeff", rc);
}

void generate_disorder_potential(double* impurity_x, double* impurity_y, double* impurity_intensity,
                                 int impurity_num, double L1, double L2, unsigned long seed, int sample_offset) {
    report("generate_disorder_potential",
           rlmb_rlm_disorder(impurity_num, L1, L2, seed, sample_offset, impurity_x, impurity_y, impurity_intensity));
}

// diag_wrappers/wfs_file.cpp:2-23: raw dumps named wfs_<theta_1>_<theta_2>.bin in the current
// directory (no header, size complex doubles); a failure is reported on stderr.
static void wfs_name(char* buf, size_t cap, int theta_1, int theta_2) {
    snprintf(buf, cap, "wfs_%d_%d.bin", theta_1, theta_2);
}

void write_wfs(int theta_1, int theta_2, std::complex<double>* wfs, unsigned long size) {
    char name[64];
    wfs_name(name, sizeof(name), theta_1, theta_2);
    FILE* f = fopen(name, "wb");
    if (!f || fwrite(wfs, sizeof(std::complex<double>), size, f) != size) fprintf(stderr, "write_wfs: cannot write %s\n", name);
    if (f) fclose(f);
}

void read_wfs(int theta_1, int theta_2, std::complex<double>* wfs, unsigned long size) {
    char name[64];
    wfs_name(name, sizeof(name), theta_1, theta_2);
    FILE* f = fopen(name, "rb");
    if (!f || fread(wfs, sizeof(std::complex<double>), size, f) != size) fprintf(stderr, "read_wfs: cannot read %s\n", name);
    if (f) fclose(f);
}
