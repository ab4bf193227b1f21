// oracle/ref_glue_hlm.cpp -- test infrastructure only.
//
// extern "C" entry points over the reference's own double-precision hlm functions,
// compiled with the unmodified reference sources into oracle/_ref/libref_hlm.so by
// oracle/Makefile (a separate library from the rlm one: both models define a
// struct_solve and a peer_solve_projected of their own).
#include "hlm/hamiltonian_hlm_cpu.h"
#include "diag_wrappers/chern.h"
#include "diag_wrappers/mkl_diag.h"
#include <pthread.h>
#include <vector>

// Defined in hlm/hamiltonian_hlm_cpu.cpp:2 (the header declares a different overload).
void get_wfs_ktheta(int lx, int ly, int Q, int band, int n_mesh, int theta_1, int theta_2,
                    std::complex<double>* wfs);

extern "C" {

// hlm/hamiltonian_hlm_cpu.cpp:2-56: clean Bloch basis W(theta), n_sites x n_phi col-major.
void ref_hlm_wfs_ktheta(int lx, int ly, int Q, int band, int n_mesh, int theta_1, int theta_2,
                        std::complex<double>* wfs) {
    get_wfs_ktheta(lx, ly, Q, band, n_mesh, theta_1, theta_2, wfs);
}

// One theta_1 line (theta_2 = 0..n_mesh-1) of projection + heevd + back-transform,
// dealt over threads as hlm/main_hlm_cpu.cpp:55-57,84-103 does.  wfs_full is the
// 2-line ring, 2*(n_mesh+1)*n_phi*n_sites values; energy_theta is (n_mesh+1)*n_phi.
// Also applies the periodic copy theta_2=n_mesh <- theta_2=0 of hlm/main_hlm_cpu.cpp:117-118,149-150.
void ref_hlm_solve_line(int theta_1, int lx, int ly, int Q, int band, int n_mesh,
                        std::complex<double>* wfs_full, double* energy_theta, double* potential,
                        int num_threads) {
    int n_sites = lx * ly;
    int n_phi = n_sites / Q;
    unsigned long dim_wfs = (unsigned long)n_phi * n_sites;
    std::vector<std::vector<int>> lists(num_threads);
    for (int i = 0; i < n_mesh; ++i) lists[i % num_threads].push_back(i);
    std::vector<std::complex<double>> wfs(num_threads * dim_wfs), wfs_clean(num_threads * dim_wfs),
        truc((size_t)num_threads * n_phi * n_phi);
    std::vector<struct_solve> params(num_threads);
    std::vector<pthread_t> th(num_threads);
    for (int id = 0; id < num_threads; ++id) {
        params[id].lx = lx;
        params[id].ly = ly;
        params[id].Q = Q;
        params[id].band = band;
        params[id].n_mesh = n_mesh;
        params[id].theta_1 = theta_1;
        params[id].theta_2 = lists[id].data();
        params[id].theta_len = (int)lists[id].size();
        params[id].wfs_full = wfs_full;
        params[id].energy_theta = energy_theta;
        params[id].potential = potential;
        params[id].wfs = wfs.data() + id * dim_wfs;
        params[id].wfs_clean = wfs_clean.data() + id * dim_wfs;
        params[id].truc_hamiltonian = truc.data() + (size_t)id * n_phi * n_phi;
        pthread_create(&th[id], NULL, peer_solve_projected, (void*)&params[id]);
    }
    for (int id = 0; id < num_threads; ++id) pthread_join(th[id], NULL);
    for (unsigned long k = 0; k < dim_wfs; ++k)
        wfs_full[((theta_1 % 2) * (n_mesh + 1) + n_mesh) * dim_wfs + k] =
            wfs_full[((theta_1 % 2) * (n_mesh + 1)) * dim_wfs + k];
}

// diag_wrappers/chern.cpp:37-75 over threads (hlm/main_hlm_cpu.cpp:155-168).
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

// hlm/main_hlm_cpu.cpp:66-67,79: the run-long MT19937 stream, one n_sites draw per sample.
void ref_hlm_potentials(unsigned long seed, int n_sites, int n_sample, double* out) {
    VSLStreamStatePtr s;
    vslNewStream(&s, VSL_BRNG_MT19937, seed);
    for (int n = 0; n < n_sample; ++n)
        vdRngUniform(VSL_RNG_METHOD_UNIFORM_STD, s, n_sites, out + (size_t)n * n_sites, -1, 1);
    vslDeleteStream(&s);
}

void ref_mkl_heevd(std::complex<double>* h, double* w, int n) { mkl_heevd(h, w, n); }

}  // extern "C"
