/*
 * diag_wrappers_b200.h -- the reference's C++ entry points, same names and signatures,
 * implemented on the B200 library (rlm_b200.h).  Link against librlmb.so and include this
 * header instead of diag_wrappers/{mkl_diag,cusolver_diag,magma_diag,chern}.h and the rlm
 * model headers of qiongz/Random-Landau-Model (double-precision build, dtype = double).
 *
 * Behaviour kept from the reference: all functions return void; a failure is reported on
 * stderr and the call returns (the reference discards LAPACK's info, mkl_diag.cpp:8).
 * One library context per calling host thread is created on first use (device 0, or the
 * device current on that thread).
 */
#ifndef DIAG_WRAPPERS_B200_H
#define DIAG_WRAPPERS_B200_H

#include <complex>
#include <cuComplex.h>

/* diag_wrappers/mkl_diag.h:13 -- host buffer, column-major, uplo 'U', eigenvectors in place */
void mkl_heevd(std::complex<double>* hamiltonian, double* energy, int l);

/* diag_wrappers/cusolver_diag.h:6 -- device pointers, single precision, in place (the
 * eigensolve itself runs in double precision on the device; results are rounded to float). */
void cusolver_diag_hamil(cuFloatComplex* dev_wfs, float* dev_energy, int n_phi);

/* diag_wrappers/magma_diag.h:9 -- device matrix (packed n x n), HOST eigenvalue array. */
void magma_diag_hamil(cuFloatComplex* dev_wfs, float* energy, int n_phi);

/* rlm/hamiltonian_rlm_gpu.h:8 (rlm/hamiltonian_rlm_gpu.cu:42-50) -- the single-precision GPU
 * driver's assembly: device tables coeff_m_theta rows theta_1 (conjugated, band index n) and
 * theta_2 (index m), coeff_jm, Vmn; dev_wfs receives the row-major n_phi x n_phi H with the
 * reference GPU path's twist convention (rlm/main_rlm_gpu.cu:170-173), lower triangle
 * = conj(upper), diagonal conjugated.  Any n_phi (the reference needs n_phi % 8 == 0);
 * default stream, synchronous. */
void set_hamil_matrix(const cuFloatComplex* dev_coeff_m_theta_1, const cuFloatComplex* dev_coeff_m_theta_2,
                      const cuFloatComplex* dev_coeff_jm, const cuFloatComplex* dev_Vmn, cuFloatComplex* dev_wfs,
                      int n_phi, int dim_n, int off_head);

/* rlm/potential_coeff.h:7 (rlm/potential_coeff.cu:21-26) -- V_mn of the GPU driver from device
 * impurity arrays (float), with its exp(+i k.r) sign; default stream, synchronous. */
void prepare_potential_coeff(float* impurity_x, float* impurity_y, float* impurity_intensity, cuFloatComplex* Vmn,
                             cuFloatComplex* coeff_mn, int dim_m, int dim_n, int off_head, int impurity_num);

/* diag_wrappers/chern.h:17-31 */
struct struct_Chern {
    int n_phi;
    int dim_vec;
    int n_mesh;
    int theta_1;
    int* theta_2;
    int theta_len;
    std::complex<double>* wave_function;
    double* chern_numbers_theta;
};
/* Plaquettes between ring slots of lines theta_1-1 and theta_1 of wfs_full (host,
 * 2*(n_mesh+1)*n_phi*dim_vec values); chern_numbers_theta[m + n*n_mesh] = -arg/2pi. */
void cal_Chern(std::complex<double>* wfs_full, double* chern_numbers_theta, int n_phi, int dim_vec,
               int n_mesh, int theta_1);
/* The same for the plaquettes m = theta_2[0..theta_len) of a struct_Chern. */
void* peer_cal_Chern(void* peer_Chern_params);
/* diag_wrappers/chern.h:30 (chern.cpp:77-123) -- line theta_1 from the files
 * wfs_<theta_1 % 2 ring slot>_<theta_2>.bin of the current directory (write_wfs layout). */
void cal_Chern_wfs_IO(double* chern_numbers_theta, int n_phi, int dim_vec, int n_mesh, int theta_1);

/* rlm/matrix_coefficients.h:10-13 (host, bit-exact tables; V_mn on the device) */
void prepare_coeff(std::complex<double>* coeff_mn, std::complex<double>* coeff_m_theta,
                   std::complex<double>* coeff_jm, int n_phi, int off_head, int dim_m, int dim_n,
                   int n_mesh, double L1, double L2);
void get_potential_coeff(double* impurity_x, double* impurity_y, double* impurity_intensity,
                         std::complex<double>* Vmn, std::complex<double>* coeff_mn, int dim_m,
                         int dim_n, int off_head, int impurity_num);
/* rlm/disorder_potential.h:12 */
void generate_disorder_potential(double* impurity_x, double* impurity_y, double* impurity_intensity,
                                 int impurity_num, double L1, double L2, unsigned long seed,
                                 int sample_offset);

/* diag_wrappers/wfs_file.h:11-12 -- raw eigenvector files wfs_<theta_1>_<theta_2>.bin in the
 * current directory, size complex values (host). */
void write_wfs(int theta_1, int theta_2, std::complex<double>* wfs, unsigned long size);
void read_wfs(int theta_1, int theta_2, std::complex<double>* wfs, unsigned long size);

#endif