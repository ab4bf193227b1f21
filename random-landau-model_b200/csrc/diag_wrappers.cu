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

// H(theta_1, theta_2) of the reference's single-precision GPU driver
// (rlm/hamiltonian_rlm_gpu.cu:9-41): row-major wfs[j*n + k] for k >= j is
//   sum_m coeff_jm[j*d + m] ct2[m] sum_{n: (n - o) = k - j mod N, |n - o| <= o} Vmn[m*d + n] conj(ct1[n]),
// the lower triangle its conjugate and the diagonal conjugated (the reference's last store
// at wfs[k*n + j] overwrites the diagonal with its conjugate).  Products and sums in double,
// rounded to float once.  One thread per (j, k); k < j threads return, so every entry is
// written exactly once (the reference zeroes the lower triangle from one thread while
// another writes it; this writes the full Hermitian matrix it intends).
__global__ void k_set_hamil_f32(const cuFloatComplex* __restrict__ ct1, const cuFloatComplex* __restrict__ ct2,
                                const cuFloatComplex* __restrict__ cjm, const cuFloatComplex* __restrict__ vmn,
                                cuFloatComplex* __restrict__ wfs, int N, int d, int o) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= N || k >= N || k < j) return;
    // the (at most two) n of the cyclic band: n - o = k - j, or k - j - N
    int nn[2], cnt = 0;
    if (k - j <= o) nn[cnt++] = o + k - j;
    if (N + j - k <= o) nn[cnt++] = o + k - j - N;
    double hr = 0.0, hi = 0.0;
    if (cnt > 0) {
        double tr[2], ti[2];   // conj(ct1[n])
        for (int q = 0; q < cnt; ++q) {
            tr[q] = ct1[nn[q]].x;
            ti[q] = -ct1[nn[q]].y;
        }
        for (int m = 0; m < d; ++m) {
            double sr = 0.0, si = 0.0;
            for (int q = 0; q < cnt; ++q) {
                const cuFloatComplex v = vmn[(size_t)m * d + nn[q]];
                sr += v.x * tr[q] - v.y * ti[q];
                si += v.x * ti[q] + v.y * tr[q];
            }
            const cuFloatComplex a = cjm[(size_t)j * d + m], b = ct2[m];
            const double pr = sr * a.x - si * a.y, pi = sr * a.y + si * a.x;
            hr += pr * b.x - pi * b.y;
            hi += pr * b.y + pi * b.x;
        }
    }
    const cuFloatComplex h = make_cuFloatComplex((float)hr, (float)hi);
    const cuFloatComplex hc = make_cuFloatComplex((float)hr, (float)-hi);
    if (j == k) {
        wfs[(size_t)j * N + j] = hc;
    } else {
        wfs[(size_t)j * N + k] = h;
        wfs[(size_t)k * N + j] = hc;
    }
}

// V_mn of the reference's single-precision GPU path (rlm/potential_coeff.cu:3-19):
//   Vmn[m*dim_n + n] = coeff_mn[m*dim_n + n] * sum_i s_i exp(+i 2 pi ((m - o) x_i + (n - o) y_i))
// (the GPU path's sign; its CPU path uses exp(-i ...)).  One warp per (m, n), lanes over the
// impurities, phases and sums in double, rounded to float once.
__global__ void k_potential_f32(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ s,
                                cuFloatComplex* __restrict__ vmn, const cuFloatComplex* __restrict__ cmn, int dim_m,
                                int dim_n, int o, int nimp) {
    const int lane = threadIdx.x & 31;
    const long w = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= (long)dim_m * dim_n) return;
    const int m = (int)(w / dim_n), n = (int)(w % dim_n);
    const double km = 2.0 * (m - o), kn = 2.0 * (n - o);
    double sr = 0.0, si = 0.0;
    for (int i = lane; i < nimp; i += 32) {
        double sn, cs;
        sincospi(km * (double)x[i] + kn * (double)y[i], &sn, &cs);
        sr += cs * (double)s[i];
        si += sn * (double)s[i];
    }
    for (int off = 16; off > 0; off >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, off);
        si += __shfl_xor_sync(0xffffffffu, si, off);
    }
    if (lane == 0) {
        const cuFloatComplex c = cmn[(size_t)m * dim_n + n];
        vmn[(size_t)m * dim_n + n] = make_cuFloatComplex((float)(sr * c.x - si * c.y), (float)(sr * c.y + si * c.x));
    }
}

}  // namespace

void set_hamil_matrix(const cuFloatComplex* dev_coeff_m_theta_1, const cuFloatComplex* dev_coeff_m_theta_2,
                      const cuFloatComplex* dev_coeff_jm, const cuFloatComplex* dev_Vmn, cuFloatComplex* dev_wfs,
                      int n_phi, int dim_n, int off_head) {
    if (!dev_coeff_m_theta_1 || !dev_coeff_m_theta_2 || !dev_coeff_jm || !dev_Vmn || !dev_wfs || n_phi <= 0 ||
        dim_n != 2 * off_head + 1 || off_head < 0)
        return report("set_hamil_matrix", RLMB_ERR_ARG);
    const dim3 block(32, 8), grid((n_phi + 31) / 32, (n_phi + 7) / 8);
    k_set_hamil_f32<<<grid, block, 0, 0>>>(dev_coeff_m_theta_1, dev_coeff_m_theta_2, dev_coeff_jm, dev_Vmn, dev_wfs,
                                           n_phi, dim_n, off_head);
    int rc = cudaGetLastError() == cudaSuccess ? RLMB_OK : RLMB_ERR_CUDA;
    if (rc == RLMB_OK && cudaStreamSynchronize(0) != cudaSuccess) rc = RLMB_ERR_CUDA;
    report("set_hamil_matrix", rc);
}

void prepare_potential_coeff(float* impurity_x, float* impurity_y, float* impurity_intensity, cuFloatComplex* Vmn,
                             cuFloatComplex* coeff_mn, int dim_m, int dim_n, int off_head, int impurity_num) {
    if (!impurity_x || !impurity_y || !impurity_intensity || !Vmn || !coeff_mn || dim_m <= 0 || dim_n <= 0 ||
        impurity_num < 0)
        return report("prepare_potential_coeff", RLMB_ERR_ARG);
    const long warps = (long)dim_m * dim_n;
    k_potential_f32<<<(unsigned)((warps + 7) / 8), 256, 0, 0>>>(impurity_x, impurity_y, impurity_intensity, Vmn,
                                                                 coeff_mn, dim_m, dim_n, off_head, impurity_num);
    int rc = cudaGetLastError() == cudaSuccess ? RLMB_OK : RLMB_ERR_CUDA;
    if (rc == RLMB_OK && cudaStreamSynchronize(0) != cudaSuccess) rc = RLMB_ERR_CUDA;
    report("prepare_potential_coeff", rc);
}

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

// diag_wrappers/chern.cpp:77-123: the plaquettes of line theta_1 from the eigenvector files
// wfs_<slot>_<theta_2>.bin (slot = theta_1 % 2 ring index, theta_2 = 0..n_mesh, as the GPU
// driver writes them with -DwfsIO).  The reference multiplies <u_{l+1}|u_l> around each
// plaquette and stores +arg/2pi; that is the conjugate product of cal_Chern's, so the values
// are cal_Chern's -arg/2pi of the same ring (atan2 is odd in its first argument, signed
// zeros included).  All 2 (n_mesh + 1) files are read, then the ring goes through cal_Chern.
void cal_Chern_wfs_IO(double* chern_numbers_theta, int n_phi, int dim_vec, int n_mesh, int theta_1) {
    if (!chern_numbers_theta || n_phi <= 0 || dim_vec <= 0 || n_mesh <= 0 || theta_1 < 0)
        return report("cal_Chern_wfs_IO", RLMB_ERR_ARG);
    const size_t dim_wfs = (size_t)n_phi * dim_vec;
    std::vector<std::complex<double>> ring(2 * (size_t)(n_mesh + 1) * dim_wfs);
    for (int slot = 0; slot < 2; ++slot)
        for (int t2 = 0; t2 <= n_mesh; ++t2)
            read_wfs(slot, t2, ring.data() + ((size_t)slot * (n_mesh + 1) + t2) * dim_wfs, dim_wfs);
    report("cal_Chern_wfs_IO", chern_line(ring.data(), chern_numbers_theta, n_phi, dim_vec, n_mesh, theta_1));
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
