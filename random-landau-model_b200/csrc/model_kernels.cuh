// Launch wrappers of the assembly and Chern-step kernels (model_kernels.cu).
#pragma once
#include "common.cuh"

#define RLMB_MAX_Q 16

namespace rlmb {
// rlm
int launch_rlm_potential(rlmb_context* ctx, const double* x, const double* y, const double* s,
                         int nimp, int nsamples, const cplx* coeff_mn, int dim, int off_head,
                         cplx* partial_ws, cplx* vmn);
size_t rlm_potential_ws_elems(int nimp, int nsamples, int dim);
int launch_rlm_assemble(rlmb_context* ctx, const cplx* vmn, const cplx* cmt, const cplx* cjm,
                        const int* d_t1, const int* d_t2, int count, int kpts_per_sample,
                        int n_phi, int dim, int o, cplx* H);
int launch_rlm_links(rlmb_context* ctx, const cplx* X, int n_phi, int g, int nsamples, cplx* U1, cplx* U2);
int launch_plaquettes(rlmb_context* ctx, const cplx* U1, const cplx* U2, const double* W, int n_phi,
                      int g, int nsamples, int hlm, double* energies, double* chern);
int launch_fhs_line(rlmb_context* ctx, const cplx* prev, const cplx* cur, int n_phi, int dim_vec,
                    int g, double* out);
int launch_rlm_disorder_at(rlmb_context* ctx, int nimp, double L1, double L2, unsigned long seed,
                           const int* d_sample0, int offset, int count, double* d_x, double* d_y, double* d_s);
// hlm
int launch_hlm_bloch(rlmb_context* ctx, int lx, int ly, int Q, int band, int g, int t1_0, int t1_1,
                     int t2_0, int t2_1, cplx* hb);
int launch_hlm_basis_expand(rlmb_context* ctx, const cplx* hb, int lx, int ly, int Q, int g, int t1,
                            int t2, cplx* W);
int launch_hlm_vtilde(rlmb_context* ctx, const double* pot, int lx, int ly, int Q, int nsamples, cplx* vt);
int launch_hlm_project(rlmb_context* ctx, const cplx* hb, const cplx* vt, const int* d_tlist, int lx,
                       int ly, int Q, int kpts, int nsamples, cplx* H);
int launch_hlm_links(rlmb_context* ctx, const cplx* hb, const cplx* X, int lx, int ly, int Q, int g,
                     int nsamples, cplx* U1, cplx* U2);
}  // namespace rlmb
