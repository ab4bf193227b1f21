/*
 * rlm_b200.h -- C ABI of the B200 (sm_100a) twist-mesh pipeline for the random
 * Landau-level model (rlm) and the Hofstadter lattice model (hlm).
 *
 * Conventions (those of the reference, qiongz/Random-Landau-Model):
 *   - complex numbers are interleaved double pairs (re, im), i.e. the memory layout of
 *     std::complex<double>; a "complex array of length L" is 2*L doubles;
 *   - matrices are column-major with leading dimension n; Hermitian input is read from
 *     the upper triangle (LAPACK uplo='U'), as diag_wrappers/mkl_diag.cpp:2-9 does;
 *   - eigenvalues ascend; eigenvector k overwrites column k (elements [k*n, k*n+n));
 *   - arguments named d_* are device pointers, h_* host pointers;
 *   - every call returns an int status: 0 success, <0 argument/CUDA/allocation error,
 *     >0 number of matrices whose eigensolve did not converge.
 * All device work is queued on the context's stream; functions returning host results
 * synchronise that stream.  A context is bound to one device and is not thread-safe;
 * use one context per host thread.
 */
#ifndef RLM_B200_H
#define RLM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define RLMB_OK 0
#define RLMB_ERR_ARG -1
#define RLMB_ERR_CUDA -2
#define RLMB_ERR_ALLOC -3
#define RLMB_ERR_NO_DEVICE -4
#define RLMB_ERR_TOO_LARGE -5

typedef struct rlmb_context rlmb_context;

/* ------------------------------------------------------------------ context */
int rlmb_create(rlmb_context** ctx, int device);
int rlmb_destroy(rlmb_context* ctx);
/* stream: a cudaStream_t (0 = the legacy default stream). */
int rlmb_set_stream(rlmb_context* ctx, void* stream);
const char* rlmb_status_string(int status);
/* Number of kernel launches this context has issued since creation. */
long long rlmb_launch_count(const rlmb_context* ctx);
/* Per-kernel timing with CUDA events recorded on the context stream around every launch
 * (no counterpart in the reference, whose drivers time whole phases with cudaEvent /
 * std::chrono, rlm/main_rlm_gpu.cu:115-283).  enable clears the accumulators;
 * count synchronises the stream and returns the number of kernels seen; entry i gives
 * the kernel name, its summed device time and its number of launches. */
int rlmb_profile_enable(rlmb_context* ctx, int on);
int rlmb_profile_count(rlmb_context* ctx);
int rlmb_profile_entry(rlmb_context* ctx, int index, char* name, int name_cap, double* total_ms,
                       long long* launches);
/* Measured double-precision FMA throughput of the device (TFLOP/s), the roofline
 * denominator of the FP64 kernels. */
int rlmb_probe_fp64_peak(rlmb_context* ctx, double* tflops);

/* Precision mode of the context's eigensolves (rlmb_heevd_batched, rlmb_heevd_host and the
 * mesh solves); no counterpart in the reference, whose precision is fixed at build time
 * (-DDP, Makefile).  RLMB_PRECISION_FP64 (default): every stage in double precision.
 * RLMB_PRECISION_MIXED: Householder reduction and back-transformation in single
 * precision, tridiagonal solve in double, then double-precision refinement of every
 * eigenpair from the residual R = H X - X diag(w); results are returned in double with
 * the same layout.  Other values return RLMB_ERR_ARG. */
#define RLMB_PRECISION_FP64 0
#define RLMB_PRECISION_MIXED 1
int rlmb_set_precision(rlmb_context* ctx, int mode);
int rlmb_get_precision(const rlmb_context* ctx);
/* Refinement steps of the mixed mode, 1 or 2 (default 2).  Each step roughly squares the
 * relative eigenvector error: one step from single precision leaves residual and
 * orthogonality defects of ~1e-12..1e-7 (growing with n), two reach double-precision
 * level.  Eigenvalues are within ~1e-11 relative after one step. */
int rlmb_set_refinement_steps(rlmb_context* ctx, int steps);
/* Mixed mode with one refinement step only (no counterpart in the reference): with the pass on,
 * every eigenvalue is recomputed after the step as the Rayleigh quotient of its refined vector,
 * x^H H x / x^H x, from a double-precision residual R = H X - X diag(w) (banded for the rlm
 * meshes).  The quotient's error is of the order of the square of the vector's (~1e-7 after
 * one step), so the eigenvalues reach double-precision level at the cost of one residual
 * instead of a second full step; the eigenvectors keep the one-step accuracy (residual and
 * orthogonality ~1e-7).  Off by default; no effect with two steps or in the FP64 mode. */
int rlmb_set_eigenvalue_pass(rlmb_context* ctx, int on);

/* Eigensolver launch choices (no counterpart in the reference, whose solver is a library
 * call).  With autotuning on, the first eigensolve of each order n in 16..1024 and precision
 * mode on the context times every feasible configuration -- unblocked or blocked reduction,
 * 256- or 512-thread panels, register-resident or GEMM back-transformation, 64- or
 * 128-reflector blocks and 64- or 128-row tiles of the double-precision X update of the
 * latter, and for n <= 80 the batched Jacobi solver -- on copies of up to 2 x SMs of the
 * call's own matrices and keeps the fastest for later calls of that order.  rlmb_heev_config reports the configuration used for
 * (n, precision) (the tuned one, or the built-in one) and returns 1 if it was tuned or set,
 * 0 if built-in; rlmb_set_heev_config pins one (-1 / 0 = built-in choice for that item).
 * panel_threads, x_tile and bt_block 0 mean the built-in choice. */
int rlmb_set_autotune(rlmb_context* ctx, int on);
int rlmb_heev_config(rlmb_context* ctx, int n, int precision, int* blocked, int* gemm_bt, int* panel_threads,
                     int* x_tile, int* bt_block, double* ms_per_matrix);
int rlmb_set_heev_config(rlmb_context* ctx, int n, int precision, int blocked, int gemm_bt, int panel_threads,
                         int x_tile, int bt_block);
/* Solver of the order-n eigensolves (no counterpart in the reference; both solvers stand in
 * for its LAPACKE_zheevd call, diag_wrappers/mkl_diag.cpp:2-9).  RLMB_SOLVER_HOUSEHOLDER: the
 * reduction / tridiagonal solve / back-transformation path above.  RLMB_SOLVER_JACOBI
 * (n <= 80): two-sided cyclic Jacobi, one CTA per matrix with the matrix and its rotations in
 * shared memory, double precision in either precision mode.  RLMB_SOLVER_AUTO: the built-in
 * choice (Jacobi up to n = 20) or the autotuner's.  rlmb_heev_solver reports the solver that
 * (n, precision) runs with now.  Jacobi above n = 80 returns RLMB_ERR_ARG. */
#define RLMB_SOLVER_AUTO 0
#define RLMB_SOLVER_HOUSEHOLDER 1
#define RLMB_SOLVER_JACOBI 2
int rlmb_set_heev_solver(rlmb_context* ctx, int n, int precision, int solver);
int rlmb_heev_solver(rlmb_context* ctx, int n, int precision, int* solver);
/* Tridiagonal stage of the Householder solver (no counterpart in the reference; LAPACK's zheevd
 * behind its LAPACKE_zheevd call solves this stage by divide and conquer).
 * RLMB_TRIDIAG_BISECTION: eigenvalues by Sturm-count bisection, eigenvectors by twisted
 * factorisation / inverse iteration.  RLMB_TRIDIAG_DC (n <= 3600): divide and conquer
 * (Cuppen splits, deflation, secular equation per root, Gu-Eisenstat eigenvectors, merges as
 * FP64 tensor-core GEMMs).  RLMB_TRIDIAG_AUTO: the built-in choice (divide and conquer from
 * n = 600) or the autotuned one.  Both run in
 * double precision in either precision mode. */
/* Panel queue of the blocked reduction (orders above 512, chunks of more matrices than SMs; no
 * counterpart in the reference): CTAs of `threads` = 512 threads, one per SM, or 256 threads,
 * two per SM, take (matrix, column) units; 0 = the built-in choice. */
int rlmb_set_panel_queue(rlmb_context* ctx, int n, int precision, int threads);
/* Columns per panel of the blocked reduction: 16 or 32 (rank-32 or rank-64 updates); 0 = the
 * built-in choice (32 from order 1024 in the FP64 mode, 16 otherwise: in the mixed mode 32
 * leaves the refinement a larger single-precision error). */
int rlmb_set_panel_width(rlmb_context* ctx, int n, int precision, int width);
#define RLMB_TRIDIAG_AUTO 0
#define RLMB_TRIDIAG_BISECTION 1
#define RLMB_TRIDIAG_DC 2
int rlmb_set_tridiag_solver(rlmb_context* ctx, int n, int precision, int solver);
int rlmb_tridiag_solver(rlmb_context* ctx, int n, int precision, int* solver);

/* ------------------------------------------------- (b) Hermitian eigensolver
 * Batched full eigendecomposition, double precision, in place.
 * Replaces: mkl_heevd            diag_wrappers/mkl_diag.cpp:2-9   (host, col-major, 'U')
 *           cusolver_diag_hamil  diag_wrappers/cusolver_diag.cu:3-22
 *           magma_diag_hamil     diag_wrappers/magma_diag.cu:2-49
 * d_a:    batch matrices of n*n complex, col-major, upper triangle read; on return
 *         column k of matrix b holds eigenvector k.
 * d_w:    batch*n eigenvalues, ascending per matrix.
 * d_info: optional (may be NULL) batch ints: 0 ok, >0 eigenvectors not converged. */
int rlmb_heevd_batched(rlmb_context* ctx, double* d_a, double* d_w, int n, int batch, int* d_info);
/* Host-pointer form of the same call (copies in and out): the drop-in for mkl_heevd. */
int rlmb_heevd_host(rlmb_context* ctx, double* h_a, double* h_w, int n, int batch);

/* Allocation-free form of rlmb_heevd_batched; it has no counterpart in the reference.
 * It is for callers that cannot allocate device memory: processes whose device memory is
 * already reserved in full by another allocator (a framework's caching pool, a job's fixed
 * memory budget) and callers that must not take cudaMalloc/cudaFree's implicit device
 * synchronisation mid-run.  Same layout and arguments as rlmb_heevd_batched; it always
 * solves in double precision (the FP64 mode, no mixed-precision refinement), whatever
 * precision mode contexts use elsewhere.  No context: work is queued on `stream` (a
 * cudaStream_t of the current device, 0 = legacy default stream; a stream of another
 * device returns RLMB_ERR_ARG).  A launch error the caller left pending returns
 * RLMB_ERR_CUDA at entry and is left in place.
 * Scratch is a fixed file-scope device array of RLMB_NOALLOC_SCRATCH_BYTES that every GPU
 * loading the library holds until exit; a matrix order whose scratch does not fit
 * (n > 927) returns RLMB_ERR_TOO_LARGE, larger batches are processed in equal chunks.  The
 * first call on each device looks the array's device address up (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  All calls share the array: calls whose
 * GPU work overlaps in time (other streams or host threads) race. */
#define RLMB_NOALLOC_SCRATCH_BYTES (32ull << 20)
int rlmb_heevd_batched_noalloc(double* d_a, double* d_w, int n, int batch, int* d_info, void* stream);

/* Batched complex GEMM C = A B on the device (no counterpart in the reference, whose dense
 * products are MKL cblas_zgemm3m calls, hlm/hamiltonian_hlm_cpu.cpp:176,180): d_a, d_b, d_c
 * hold batch column-major complex matrices back to back (A m x k, B k x n, C m x n).
 * engine RLMB_GEMM_FP64: double precision on the FP64 tensor path (DMMA);
 * engine RLMB_GEMM_TF32X3: the tcgen05 tensor cores, each operand split into two TF32
 * numbers and three products accumulated in FP32 (relative error ~1e-6 of |A||B|), the
 * engine of the reduction's and back-transformation's products in the mixed mode;
 * engine RLMB_GEMM_TF32X3_F64ACC: the same products with the operands loaded by TMA from
 * TF32 planes and the accumulator emptied into double-precision sums after every 32 real
 * terms (relative error ~1e-7 of |A||B|), the engine of the mixed mode's refinement products.
 * batch <= 65535; with k = 0 the product is zero and d_a, d_b may be NULL. */
#define RLMB_GEMM_FP64 0
#define RLMB_GEMM_TF32X3 1
#define RLMB_GEMM_TF32X3_F64ACC 2
int rlmb_zgemm_batched(rlmb_context* ctx, const double* d_a, const double* d_b, double* d_c, int m, int n,
                       int k, int batch, int engine);
/* Tiles of the tcgen05 engine whose bounded mbarrier waits ran out (a fault: the tile's
 * output is not written) since the library was loaded; synchronises the device. */
int rlmb_tc_fault_count(rlmb_context* ctx, int* count);

/* ------------------------------------------------------- (a) rlm assembly
 * Disorder-independent coefficient tables, computed on the host exactly as
 * rlm/matrix_coefficients.cpp:3-25 (prepare_coeff) does, bit for bit:
 * coeff_mn[dim*dim], coeff_m_theta[(n_mesh+1)*dim], coeff_jm[n_phi*dim] (complex). */
int rlmb_rlm_coeff_tables(int n_phi, int off_head, int dim, int n_mesh, double L1, double L2,
                          double* h_coeff_mn, double* h_coeff_m_theta, double* h_coeff_jm);
/* Impurities of one sample, as rlm/disorder_potential.cpp:3-21 draws them (host MT19937). */
int rlmb_rlm_disorder(int impurity_num, double L1, double L2, unsigned long seed, int sample,
                      double* h_x, double* h_y, double* h_s);
/* The same draws on the device, for samples sample0 .. sample0+count-1 at once (one
 * MT19937 stream per sample, skipped on the device): d_x, d_y, d_s are count*impurity_num
 * doubles, sample k at [k*impurity_num], bit-identical to rlmb_rlm_disorder. */
int rlmb_rlm_disorder_device(rlmb_context* ctx, int impurity_num, double L1, double L2,
                             unsigned long seed, int sample0, int count, double* d_x, double* d_y,
                             double* d_s);
/* V_mn of one or more samples (rlm/matrix_coefficients.cpp:27-44, rlm/potential_coeff.cu:3-26):
 * d_x,d_y,d_s: n_samples*impurity_num; d_vmn: n_samples*dim*dim complex, row-major m*dim+n. */
int rlmb_rlm_potential(rlmb_context* ctx, const double* d_x, const double* d_y, const double* d_s,
                       int impurity_num, int n_samples, const double* d_coeff_mn, int dim,
                       int off_head, double* d_vmn);
/* H(theta_1, theta_2) for `count` k-points of one sample (rlm/hamiltonian_rlm_cpu.cpp:14-48,
 * rlm/hamiltonian_rlm_gpu.cu:9-50): d_h receives count matrices of n_phi*n_phi complex,
 * filled as the reference fills its buffer (row-major H, lower = conj(upper)), which is the
 * column-major upper triangle the eigensolver reads.  h_theta1/h_theta2: host int[count]. */
int rlmb_rlm_assemble(rlmb_context* ctx, const double* d_vmn, const double* d_coeff_m_theta,
                      const double* d_coeff_jm, int n_phi, int dim, int off_head, int n_mesh,
                      const int* h_theta1, const int* h_theta2, int count, double* d_h);

/* ------------------------------------------------------- (a) hlm assembly
 * On-site potentials of n_sample samples from one run-long stream
 * (hlm/main_hlm_cpu.cpp:66-67,79): h_out[n_sample*n_sites]. */
int rlmb_hlm_potentials(unsigned long seed, int n_sites, int n_sample, double* h_out);
/* hlm potentials of samples sample0 .. sample0+count-1 drawn on the device (outputs
 * [sample*n_sites, (sample+1)*n_sites) of the run's single stream), bit-identical to
 * rlmb_hlm_potentials; d_out is count*n_sites doubles. */
int rlmb_hlm_potentials_device(rlmb_context* ctx, unsigned long seed, int n_sites, int sample0,
                               int count, double* d_out);
/* Clean Bloch basis W(theta_1,theta_2) of band `band` (hlm/hamiltonian_hlm_cpu.cpp:2-56):
 * d_wfs receives n_sites*n_phi complex, column-major (column kx*ly+ky). */
int rlmb_hlm_basis(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh, int theta_1,
                   int theta_2, double* d_wfs);
/* Projected H = W^H diag(V) W for `count` k-points of one sample
 * (hlm/hamiltonian_hlm_cpu.cpp:173-176): d_h receives count column-major n_phi*n_phi. */
int rlmb_hlm_project(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh,
                     const double* d_potential, const int* h_theta1, const int* h_theta2,
                     int count, double* d_h);

/* --------------------------------------------------------- (c) FHS Chern step
 * Plaquette phases between two adjacent theta_1 lines (diag_wrappers/chern.cpp:3-75):
 * d_prev, d_cur: (n_mesh+1) k-points of n_phi states each, state k of k-point t at
 * [(t*n_phi + k)*dim_vec]; d_chern_theta: n_mesh*n_phi, entry [m + k*n_mesh] =
 * -arg(prod)/2pi exactly as the reference stores it. */
int rlmb_fhs_line(rlmb_context* ctx, const double* d_prev, const double* d_cur, int n_phi,
                  int dim_vec, int n_mesh, double* d_chern_theta);

/* ------------------------------------------------------- whole-mesh pipelines
 * rlm: samples sample0 .. sample0+n_samples-1 of the rlm_cpu_dp run with these options
 * (rlm/main_rlm_cpu.cpp:109-243); h_energies/h_chern: n_samples*n_phi, the two columns
 * the reference writes to energy_Chern_No.txt (twist-averaged energy, Chern number). */
int rlmb_rlm_mesh_solve(rlmb_context* ctx, int n_phi, double quanta_concentration,
                        double impurity_concentration, int n_mesh, unsigned long seed,
                        int sample0, int n_samples, double* h_energies, double* h_chern);
/* Device-resident form: energies and Chern numbers go to device memory (d_energies, d_chern:
 * n_samples*n_phi doubles each); the disorder is drawn on the device as in
 * rlmb_rlm_mesh_solve, so nothing but the call's parameters crosses from the host. */
int rlmb_rlm_mesh_solve_device(rlmb_context* ctx, int n_phi, double quanta_concentration,
                               double impurity_concentration, int n_mesh, unsigned long seed,
                               int sample0, int n_samples, double* d_energies, double* d_chern);
/* rlm, one sample, with its eigenvectors exported: besides the energies and Chern numbers
 * of rlmb_rlm_mesh_solve, every k-point's eigenvector matrix is written to
 * dir/wfs_<theta_1>_<theta_2>.bin (theta_1, theta_2 in 0..n_mesh) in the raw format of the
 * reference's write_wfs (diag_wrappers/wfs_file.cpp:2-11; rlm/main_rlm_gpu.cu:187,227 with
 * -DwfsIO): n_phi*n_phi complex doubles, column k = eigenvector k.  The reference keeps only
 * two theta_1 lines (file names use theta_1 % 2); here every line is kept.  Eigenvector
 * phases are those of this solver (any phase is an eigenvector; FHS is gauge invariant). */
int rlmb_rlm_mesh_export(rlmb_context* ctx, int n_phi, double quanta_concentration,
                         double impurity_concentration, int n_mesh, unsigned long seed, int sample,
                         const char* dir, double* h_energies, double* h_chern);
/* Several rlm orders in ONE CUDA graph launch per step (the finite-size-scaling batch; no
 * counterpart in the reference, whose driver runs one n_phi per process).  create prepares
 * the pipeline of each order n_phi[0..count) (its own stream and buffers, every buffer sized
 * and the eigensolver configuration autotuned by one uncaptured run of samples
 * 0 .. n_samples-1) and captures all of them, one concurrent
 * branch per order, in precision mode `precision` (RLMB_PRECISION_FP64 or _MIXED).  launch
 * queues one step -- samples sample0 .. sample0+n_samples-1 of every order -- on the graph's
 * stream (stream returns it, a cudaStream_t) without synchronising; results synchronises and
 * copies order `index`'s energies and Chern numbers of the last step (n_samples*n_phi each,
 * the columns of energy_Chern_No.txt) and returns its failure count. */
typedef struct rlmb_fss_graph rlmb_fss_graph;
int rlmb_rlm_fss_graph_create(int device, const int* n_phi, int count, double quanta_concentration,
                              double impurity_concentration, int n_mesh, unsigned long seed, int n_samples,
                              int precision, rlmb_fss_graph** graph);
int rlmb_rlm_fss_graph_launch(rlmb_fss_graph* graph, int sample0);
int rlmb_rlm_fss_graph_stream(rlmb_fss_graph* graph, void** stream);
int rlmb_rlm_fss_graph_results(rlmb_fss_graph* graph, int index, double* h_energies, double* h_chern);
int rlmb_rlm_fss_graph_destroy(rlmb_fss_graph* graph);

/* hlm: n_samples samples with the given potentials (hlm/main_hlm_cpu.cpp:75-197). */
int rlmb_hlm_mesh_solve(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh,
                        const double* h_potentials, int n_samples, double* h_energies,
                        double* h_chern);
/* Device-resident form: potentials, energies and Chern numbers stay in device memory. */
int rlmb_hlm_mesh_solve_device(rlmb_context* ctx, int lx, int ly, int Q, int band, int n_mesh,
                               const double* d_potentials, int n_samples, double* d_energies,
                               double* d_chern);

#ifdef __cplusplus
}
#endif
#endif
