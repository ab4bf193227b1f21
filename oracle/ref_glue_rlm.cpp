// oracle/ref_glue_rlm.cpp -- test infrastructure only.
//
// extern "C" entry points over the reference's own double-precision rlm functions,
// compiled together with the unmodified reference sources into
// oracle/_ref/libref_rlm.so by oracle/Makefile.  The tests and the golden-fixture
// script drive these through ctypes to obtain the reference's intermediate results
// (coefficient tables, disorder, V_mn, per-k-point eigenpairs, per-line Chern sums)
// at full double precision; the reference's text output keeps only 8 digits.
#include "rlm/hamiltonian_rlm_cpu.h"
#include "rlm/matrix_coefficients.h"
#include "rlm/disorder_potential.h"
#include "diag_wrappers/chern.h"
#include "diag_wrappers/mkl_diag.h"
#include <pthread.h>
#include <vector>

extern "C" {

// rlm/matrix_coefficients.cpp:3-25
void ref_rlm_prepare_coeff(std::complex<double>* coeff_mn, std::complex<double>* coeff_m_theta,
                           std::complex<double>* coeff_jm, int n_phi, int off_head, int dim_m,
                           int dim_n, int n_mesh, double L1, double L2) {
    prepare_coeff(coeff_mn, coeff_m_theta, coeff_jm, n_phi, off_head, dim_m, dim_n, n_mesh, L1, L2);
}

// rlm/disorder_potential.cpp:3-21
void ref_rlm_disorder(double* x, double* y, double* s, int impurity_num, double L1, double L2,
                      unsigned long seed, int sample) {
    generate_disorder_potential(x, y, s, impurity_num, L1, L2, seed, sample);
}

// rlm/matrix_coefficients.cpp:27-44
void ref_rlm_potential(double* x, double* y, double* s, std::complex<double>* vmn,
                       std::complex<double>* coeff_mn, int dim_m, int dim_n, int off_head,
                       int impurity_num) {
    get_potential_coeff(x, y, s, vmn, coeff_mn, dim_m, dim_n, off_head, impurity_num);
}

// One theta_1 line of assembly + heevd, dealt round-robin over threads exactly as
// rlm/main_rlm_cpu.cpp:84-90,125-143 does (peer_solve_projected ends in pthread_exit,
// so it must run on its own thread).  wave_functions is the 2-line ring,
// 2*(n_mesh+1)*n_phi*n_phi complex values; energy_theta is (n_mesh+1)*n_phi.
void ref_rlm_solve_line(int theta_1, int n_phi, int n_mesh, int dim, int off_head,
                        std::complex<double>* wave_functions, double* energy_theta,
                        std::complex<double>* v_mn, std::complex<double>* coeff_jm,
                        std::complex<double>* coeff_m_theta, int num_threads) {
    std::vector<std::vector<int>> lists(num_threads);
    for (int i = 0; i < n_mesh + 1; ++i) lists[i % num_threads].push_back(i);
    std::vector<struct_solve> params(num_threads);
    std::vector<pthread_t> th(num_threads);
    for (int id = 0; id < num_threads; ++id) {
        params[id].theta_1 = theta_1;
        params[id].n_phi = n_phi;
        params[id].n_mesh = n_mesh;
        params[id].dim_m = dim;
        params[id].dim_n = dim;
        params[id].off_head = off_head;
        params[id].theta_2 = lists[id].data();
        params[id].theta_len = (int)lists[id].size();
        params[id].wave_function = wave_functions;
        params[id].energy = energy_theta;
        params[id].v_mn = v_mn;
        params[id].coeff_jm = coeff_jm;
        params[id].coeff_m_theta = coeff_m_theta;
        pthread_create(&th[id], NULL, peer_solve_projected, (void*)&params[id]);
    }
    for (int id = 0; id < num_threads; ++id) pthread_join(th[id], NULL);
}

// The k-points (theta_1, theta_2[i]), i < count, of one line: assembly + heevd by the
// reference's peer_solve_projected, the list dealt round-robin over num_threads threads (a
// bounded sample of a line for the CPU baseline of large orders).
void ref_rlm_solve_list(int theta_1, const int* theta_2, int count, int n_phi, int n_mesh, int dim, int off_head,
                        std::complex<double>* wave_functions, double* energy_theta, std::complex<double>* v_mn,
                        std::complex<double>* coeff_jm, std::complex<double>* coeff_m_theta, int num_threads) {
    std::vector<std::vector<int>> lists(num_threads);
    for (int i = 0; i < count; ++i) lists[i % num_threads].push_back(theta_2[i]);
    std::vector<struct_solve> params(num_threads);
    std::vector<pthread_t> th(num_threads);
    int started = 0;
    for (int id = 0; id < num_threads; ++id) {
        if (lists[id].empty()) break;
        params[id].theta_1 = theta_1;
        params[id].n_phi = n_phi;
        params[id].n_mesh = n_mesh;
        params[id].dim_m = dim;
        params[id].dim_n = dim;
        params[id].off_head = off_head;
        params[id].theta_2 = lists[id].data();
        params[id].theta_len = (int)lists[id].size();
        params[id].wave_function = wave_functions;
        params[id].energy = energy_theta;
        params[id].v_mn = v_mn;
        params[id].coeff_jm = coeff_jm;
        params[id].coeff_m_theta = coeff_m_theta;
        pthread_create(&th[id], NULL, peer_solve_projected, (void*)&params[id]);
        ++started;
    }
    for (int id = 0; id < started; ++id) pthread_join(th[id], NULL);
}

// FHS Chern contributions of the plaquettes between lines theta_1-1 and theta_1,
// diag_wrappers/chern.cpp:37-75 dealt over threads as rlm/main_rlm_cpu.cpp:195-208.
// chern_theta is n_mesh*n_phi, entry [m + n*n_mesh].
void ref_peer_cal_chern(std::complex<double>* wave_functions, double* chern_theta, int n_phi,
                        int dim_vec, int n_mesh, int theta_1, int num_threads) {
    std::vector<std::vector<int>> lists(num_threads);
    for (int i = 0; i < n_mesh; ++i) lists[i % num_threads].push_back(i);
    std::vector<struct_Chern> params(num_threads);
    std::vector<pthread_t> th(num_threads);
    for (int id = 0; id < num_threads; ++id) {
        params[id].n_phi = n_phi;
        params[id].dim_vec = dim_vec;
        params[id].n_mesh = n_mesh;
        params[id].theta_1 = theta_1;
        params[id].theta_2 = lists[id].data();
        params[id].theta_len = (int)lists[id].size();
        params[id].wave_function = wave_functions;
        params[id].chern_numbers_theta = chern_theta;
        pthread_create(&th[id], NULL, peer_cal_Chern, (void*)&params[id]);
    }
    for (int id = 0; id < num_threads; ++id) pthread_join(th[id], NULL);
}

// diag_wrappers/chern.cpp:3-35 (serial variant used by rlm/main_rlm_gpu.cu:265)
void ref_cal_chern(std::complex<double>* wave_functions, double* chern_theta, int n_phi,
                   int dim_vec, int n_mesh, int theta_1) {
    cal_Chern(wave_functions, chern_theta, n_phi, dim_vec, n_mesh, theta_1);
}

// diag_wrappers/mkl_diag.cpp:2-9
void ref_mkl_heevd(std::complex<double>* h, double* w, int n) { mkl_heevd(h, w, n); }

}  // extern "C"
