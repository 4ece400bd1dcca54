/*
 * qdsim_b200 -- C ABI of the B200 (sm_100a) finite-element quantum-dot hot path.
 *
 * Conventions
 *  - Every entry point returns an int status: QD_OK (0) or a negative QD_ERR_*.
 *  - Pointers named d_* are device pointers (any allocator; the caller owns
 *    them), h_* are host pointers.  The library never allocates device
 *    memory: scratch comes from a caller-provided workspace whose size is
 *    returned by the matching *_workspace_size query.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *  - Units are whatever the caller uses consistently; the Python layer passes
 *    nm and eV (kinetic coefficient c = hbar^2/(2 m*) in eV nm^2).
 *  - Matrices are CSR with int32 row pointers / column indices and FP64 values.
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the QDSim source tree).
 */
#ifndef QDSIM_B200_H
#define QDSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  QD_OK = 0,
  QD_ERR_INVALID = -1,        /* bad argument (sizes, null pointers, order)      */
  QD_ERR_CUDA = -2,           /* a CUDA runtime call failed                       */
  QD_ERR_NOT_CONVERGED = -3,  /* iteration cap reached; residuals are returned   */
  QD_ERR_BREAKDOWN = -4,      /* Gram matrix not positive definite / NaN input   */
  QD_ERR_WORKSPACE = -5,      /* workspace too small or misaligned               */
  QD_ERR_DEGENERATE = -6,     /* zero-area element or non-finite coefficient     */
  QD_ERR_LIMIT = -7,          /* a size exceeds a compiled-in limit              */
  QD_ERR_TIMEOUT = -8         /* a device-side wait exceeded its time bound      */
};

/* assembly modes */
enum {
  QD_ASM_FEM = 0,             /* fem.cpp weak form, nodal V/W interpolated        */
  QD_ASM_REF_CYTHON = 1,      /* schrodinger_solver.pyx:201-251 element formulas  */
  QD_ASM_REF_FIXED = 2,       /* fixed_open_system_solver.pyx:197-271 formulas    */
  QD_ASM_REF_CPP = 3          /* schrodinger.cpp:92-230: P1 stiffness, V and M by
                                 the centroid rule (every entry V A/9, A/9)       */
};

/* eigensolver precision modes */
enum {
  QD_PREC_FP64 = 0,           /* FP64 vectors throughout (the plain form)         */
  QD_PREC_MIXED = 1           /* per dot: FP32 vector phase, then a finishing phase
                                 with X, HX, MX in FP64 and W, P and their
                                 products in FP32                                 */
};

const char *qd_version(void);
const char *qd_status_string(int status);
/* Number of kernels this library launched since load (all entry points). */
uint64_t qd_kernel_launch_count(void);

/* ---------------------------------------------------------------------------
 * Sparsity pattern (host, C++).  Replaces the triplet build + setFromTriplets
 * of FEMSolver::assemble_matrices_serial (backend/src/fem.cpp:116-151) and the
 * triplet lists of CythonSchrodingerSolver._assemble_matrices
 * (qdsim_cython/solvers/schrodinger_solver.pyx:131-190).
 *
 * Rows/cols are reduced DOFs: h_dof_map[node] in [0, n_dofs) or -1 for an
 * eliminated (Dirichlet) node.  Call once with all output pointers NULL to get
 * the sizes, then again with buffers of those sizes.
 *   rowptr  int32[n_dofs+1]      col     int32[nnz]   (sorted per row)
 *   adjptr  int32[n_dofs+1]      adj     int32[n_adj]   (elem << 4 | local)
 *   cptr    int32[n_dofs+1]      contrib uint8[n_contrib] (t*k+b, slot order)
 *   slotcnt uint8[nnz]  (contributions per slot)
 * ------------------------------------------------------------------------- */
int qd_pattern_build(int64_t num_nodes, int64_t num_elems, int k,
                     const int32_t *h_elems, const int32_t *h_dof_map, int32_t n_dofs,
                     int64_t *nnz, int64_t *n_adj, int64_t *n_contrib,
                     int32_t *h_rowptr, int32_t *h_col,
                     int32_t *h_adjptr, int32_t *h_adj,
                     int32_t *h_cptr, uint8_t *h_contrib, uint8_t *h_slotcnt);

/* Node -> incident (element, local index) lists over ALL nodes (used by the
 * adjoint's nodal gather).  Same two-call protocol. */
int qd_node_adjacency(int64_t num_nodes, int64_t num_elems, int k, const int32_t *h_elems,
                      int64_t *n_adj, int32_t *h_adjptr, int32_t *h_adj);

/* ---------------------------------------------------------------------------
 * Element-parallel assembly into the precomputed CSR pattern (GPU).
 * Replaces FEMSolver::assemble_element_matrix (backend/src/fem.cpp:736-990),
 * the GPU element kernels (backend/src/gpu_kernels.cu:46-336, 442-745) and the
 * host triplet scatter of GPUAccelerator::assemble_matrices
 * (backend/src/gpu_accelerator.cpp:439-642).
 *
 * One warp per CSR row; each row's slots are summed in a fixed order over the
 * row's contribution list (deterministic, no atomics).
 *   order        1, 2 or 3 (k = 3, 6, 10 nodes per element)
 *   d_nodes      double[num_nodes*2] (x, y)
 *   d_elems      int32[num_elems*k]
 *   d_c          double[num_elems]   kinetic coefficient per element
 *   d_V          FEM mode: double[num_nodes] nodal V; REF modes: double[num_elems]
 *   d_W          FEM mode: double[num_nodes] nodal CAP amplitude or NULL
 *   outputs      d_H[nnz] (real part K + V), d_M[nnz], d_Himag[nnz] (= -W term,
 *                may be NULL)
 * The call is asynchronous.  `d_status` (int32[1], device, zeroed by the
 * caller) receives bit 1 for a zero-area element or non-finite c and bit 2
 * for a non-finite V; callers read it after synchronising and map a nonzero
 * value to QD_ERR_DEGENERATE.  Limits: at most 16 incident elements and 128
 * slots per row (QD_ERR_LIMIT from qd_pattern_build otherwise).
 * ------------------------------------------------------------------------- */
int qd_assemble(int order, int mode, int64_t num_nodes, int64_t num_elems, int32_t n_dofs,
                const double *d_nodes, const int32_t *d_elems,
                const double *d_c, const double *d_V, const double *d_W,
                const int32_t *d_rowptr, const int32_t *d_adjptr, const int32_t *d_adj,
                const int32_t *d_cptr, const uint8_t *d_contrib, const uint8_t *d_slotcnt,
                double *d_H, double *d_M, double *d_Himag, int32_t *d_status, void *stream);

/* ---------------------------------------------------------------------------
 * Fused dual SpMM over the shared H/M pattern: HX = H X, MX = M X for a block
 * of b vectors stored row-major (X[row*b + j]).  FP64 accumulation; vec_fp32
 * selects float (1) or double (0) vector storage.  Supersedes fusedSpMV
 * (backend/src/fused_gpu_kernels.cu:97-125).  Either output may be NULL.
 * ------------------------------------------------------------------------- */
int qd_spmm_dual(int32_t n_rows, int b, int vec_fp32,
                 const int32_t *d_rowptr, const int32_t *d_col,
                 const double *d_H, const double *d_M,
                 const void *d_X, void *d_HX, void *d_MX, void *stream);

/* Fast-sine-transform preconditioner of one dot (see qd_lobpcg_solve).  The
 * dot's reduced DOFs must be the interior points of an nx x ny lattice in
 * row-major order (structured rectangle, homogeneous Dirichlet boundary).
 * T = (cx Kx + cy Ky + shift I)^-1 with Kx, Ky the 1-D second differences,
 * applied as DST-I transforms on the tensor cores (BF16 operands, FP32
 * accumulation); nx = 0 disables preconditioning for the dot.
 * d_prec_mats holds, for each lattice size N in use, the orthonormal DST-I
 * matrix S[i][j] = sqrt(2/(N+1)) sin(pi (i+1)(j+1)/(N+1)) in the tensor-core
 * operand layout written by qd_dst_matrix_fill (BF16, qd_dst_matrix_size(N)
 * elements), starting at element offset sx_off (N = nx) and sy_off (N = ny);
 * offsets are multiples of 8 elements. */
typedef struct {
  int32_t nx, ny;
  int64_t sx_off, sy_off;
  float cx, cy, shift;
  int32_t pad;
} qd_dst_prec;

/* ---------------------------------------------------------------------------
 * Batched LOBPCG for the k lowest eigenpairs of H x = E M x on a
 * block-diagonal batch of n_dots independent problems (rows of dot d are
 * [h_row_off[d], h_row_off[d+1]) with global column indices).  Replaces the
 * eigsh(H, k, M, which='SM') call of CythonSchrodingerSolver.solve
 * (qdsim_cython/solvers/schrodinger_solver.pyx:447-453) and the dense
 * EigenSolver::solve (backend/src/solver.cpp:59-200).
 *   b            block size (k <= b <= 32; b - k guard vectors)
 *   prec_mode    QD_PREC_FP64 or QD_PREC_MIXED
 *   tol          target relative eigenvalue error: converged when, for all k
 *                pairs, (||r||/||Mx||)^2 / ((t_{b-1} - t) |t|) <= tol with
 *                r = H x - t M x (quadratic residual estimate, gap to the block
 *                edge) and ||r|| <= 1e-2 |t| ||Mx||
 *   d_X_out      double[n_rows_total * k] row-major per row (X[row*k + j]),
 *                M-orthonormal per dot
 *   d_E_out      double[n_dots * k]; d_res_out double[n_dots * k] relative
 *                residuals ||r|| / (|t| ||Mx||); d_iters_out int32[n_dots] (FP32 + FP64 iterations)
 *   h_info       int32[4] (host): host iterations, largest FP32 and FP64
 *                iteration counts of any dot, number of converged dots
 *   h_counts     int32[n_dots*6] (host, may be NULL): per dot, the launches of
 *                SpMM, Gram and update that did work in the FP32 and the FP64
 *                phase (for algorithmic-byte accounting)
 *   h_prec/d_prec_mats  optional per-dot DST preconditioner (host descriptor
 *                array, device BF16 matrices); NULL = unpreconditioned
 * The initial block is drawn from `seed` (deterministic).  Returns
 * QD_ERR_NOT_CONVERGED if any dot hits max_iter (results still written).
 * ------------------------------------------------------------------------- */
/* Solver options (pass NULL for the defaults; the same options to the
 * workspace query and the solve):
 *   tol32        estimate at which a dot leaves the FP32 phase (<= 0: max(100 tol, 1e-7))
 *   stag_window  FP32 iterations without halving the estimate before a dot
 *                switches to FP64 anyway (<= 0: 12)
 *   graphs       nonzero: replay blocks of 8 iterations as one CUDA graph
 *                (default); 0: enqueue every kernel directly
 *   x0           optional device array (rows x k, the layout of d_X_out): warm
 *                start for the first k block vectors (e.g. the previous
 *                self-consistent iteration's eigenvectors); NULL: random
 *   eig_scale    energy below which eigenvalue errors are measured absolutely:
 *                the estimate divides by max(|t|, eig_scale) instead of |t|
 *                (levels near zero energy); <= 0: purely relative
 *   chunk_rows   rows per chunk, the CTA unit of every row-parallel kernel
 *                (SpMM, Gram, orthogonalisation, update) and of the per-chunk
 *                partial sums; a multiple of 64 in [256, 8192], else 1024
 *   setup_cached nonzero: the caller asserts that d_work, d_rowptr and d_col
 *                (and their contents) are those of the previous call with
 *                this workspace and that nothing else used the workspace
 *                since; the call then reads no value back during its set-up
 *                and does not copy host tables identical to that call's
 *                (repeated solves of one batch shape, e.g. a sweep pipeline
 *                whose own large copies would hold small ones back).  The
 *                library checks the batch shape, pointers and tables and
 *                falls back to the full set-up when any differs. */
typedef struct {
  double tol32;
  int32_t stag_window;
  int32_t graphs;
  const double *x0;
  double eig_scale;
  int32_t chunk_rows;
  int32_t setup_cached;
} qd_lobpcg_opts;

int qd_lobpcg_workspace_size(int32_t n_dots, int64_t n_rows_total, int64_t nnz_total, int b,
                             int prec_mode, const qd_dst_prec *h_prec,
                             const qd_lobpcg_opts *opts, size_t *bytes);

int qd_lobpcg_solve(int32_t n_dots, const int32_t *h_row_off, const int32_t *d_row_off,
                    const int32_t *d_rowptr, const int32_t *d_col,
                    const double *d_H, const double *d_M,
                    const qd_dst_prec *h_prec, const void *d_prec_mats,
                    int k, int b, int prec_mode, double tol, int max_iter, uint64_t seed,
                    double *d_X_out, double *d_E_out, double *d_res_out, int32_t *d_iters_out,
                    int32_t *h_info, int32_t *h_counts, void *d_work, size_t work_bytes,
                    const qd_lobpcg_opts *opts, void *stream);

/* Apply the DST preconditioner W = T R to a batch of b-column blocks
 * (b >= 4 and even; row-major, float if vec_fp32 else double, d_in and d_out
 * 16-byte aligned; in-place allowed).  Same descriptors as qd_lobpcg_solve;
 * exposed for testing and reuse. */
int qd_dst_precond_workspace_size(int32_t n_dots, const int32_t *h_row_off, int b,
                                  const qd_dst_prec *h_prec, size_t *bytes);

/* Element count (BF16) of the DST-I matrix of lattice size n in the
 * tensor-core layout, and the host routine that writes it (round to nearest
 * even).  Layout: rows padded to R = 16 ceil(n/16), columns (k) to
 * 64 ceil(n/64); rows split into blocks of 256; within a block of r rows,
 * element (row, k) sits at  (k/64) r 64 + ((k%64)/8) r 8 + (row/8) 64 +
 * (row%8) 8 + k%8  (8 x 8 core matrices, 16 bytes per core-matrix row). */
int qd_dst_matrix_size(int32_t n, int64_t *elems);
int qd_dst_matrix_fill(int32_t n, uint16_t *h_out);
int qd_dst_precond_apply(int32_t n_dots, const int32_t *h_row_off, int b, int vec_fp32,
                         const qd_dst_prec *h_prec, const void *d_prec_mats,
                         const void *d_in, void *d_out, void *d_work, size_t work_bytes,
                         void *stream);

/* ---------------------------------------------------------------------------
 * Self-consistent Poisson-Schrodinger loop batched over nb bias points (the
 * loop of qdsim_cython/solvers/self_consistent_solver.pyx:130-286 with the
 * mixing of backend/src/self_consistent.cpp:1262-1468).  Potentials, densities
 * and the mixing history are [node][bias] (qd_pcg_solve's right-hand-side
 * layout); the Schrodinger potential is [bias][node] (the batched union mesh).
 *
 * qd_sc_potential   V_out[b][i] = V_static[i] - phi[i][b]   (eV, phi in V)
 * qd_sc_density     per bias: E_F = E_0 + kT/2, Fermi-Dirac occupations of the
 *                   k states, n = sum f psi^2 rescaled to mean N_D, classical
 *                   holes p = N_A exp(-phi/V_T) where phi > 0 else N_A,
 *                   rho = q (p - n) [C/m^3]; X is rows x k with bias b's rows
 *                   at b * rows_per_bias + dof[i] (dof[i] < 0: boundary node)
 * qd_sc_mix         damping (anderson = 0) or Anderson mixing with history
 *                   h_hist_* (host arrays of nhist device pointers, oldest
 *                   first; this update and its residual are written to slot
 *                   nhist-1): phi_new, per-bias damping factor (adapted in
 *                   place), previous error and error ||phi_new-phi_old||/||phi_new||
 * ------------------------------------------------------------------------- */
int qd_sc_potential(int32_t nb, int64_t n_nodes, const double *d_V_static, const double *d_phi,
                    double *d_V_out, void *stream);
int qd_sc_density(int32_t nb, int64_t n_nodes, int k, int64_t rows_per_bias,
                  const int32_t *d_dof, const double *d_X, const double *d_E, double kT_eV,
                  double N_A, double N_D, const double *d_phi, double *d_n, double *d_p,
                  double *d_rho, void *stream);
int qd_sc_mix(int32_t nb, int64_t n_nodes, int anderson, int nhist, const double *d_phi_old,
              const double *d_phi_upd, double *const *h_hist_upd, double *const *h_hist_res,
              double *d_phi_new, double *d_damping, double *d_prev_error, double *d_error,
              void *stream);

/* ---------------------------------------------------------------------------
 * Jacobi-preconditioned CG, FP64, for nrhs right-hand sides sharing one SPD
 * matrix (row-major X[row*nrhs + j]).  Rows with d_fixed[row] != 0 are
 * Dirichlet rows: X keeps its input value there and the row/column are
 * eliminated (equivalent to the row replacement of
 * qdsim_cython/solvers/poisson_solver.pyx:276-308, which the reference then
 * hands to spsolve at :240).  Replaces PoissonSolver::solve's SimplicialLDLT
 * (backend/src/poisson.cpp:320-334) and fusedPoissonSolver
 * (backend/src/fused_gpu_kernels.cu:159-206).
 *   tol          relative residual ||b - A x|| / ||b - A x_D|| per column over
 *                the free rows, x_D = the initial X with its free entries
 *                zeroed (the Dirichlet values alone): a warm start X lowers
 *                the work, not the target; h_relres reports the same ratio
 *   h_iters/h_relres  host outputs: iterations launched (the host checks
 *                convergence every 16 iterations, so this is the CG iteration
 *                count rounded up to a multiple of 16, or max_iter), final max
 *                relative residual
 * ------------------------------------------------------------------------- */
int qd_pcg_workspace_size(int32_t n, int nrhs, size_t *bytes);
int qd_pcg_solve(int32_t n, int nrhs, const int32_t *d_rowptr, const int32_t *d_col,
                 const double *d_A, const double *d_B, double *d_X, const int32_t *d_fixed,
                 double tol, int max_iter, int32_t *h_iters, double *h_relres,
                 void *d_work, size_t work_bytes, void *stream);

/* Jacobi-PCG without a caller workspace.  No counterpart in the reference.
 *
 * Same arguments, results and status codes as qd_pcg_solve, minus the
 * workspace: the scratch vectors live in a 16 MiB array that the library
 * reserves on every GPU it is loaded on, for the life of the process.  It is
 * for callers that cannot allocate device memory themselves -- code that runs
 * where no allocator is available or allowed (for example a solver step
 * embedded in another runtime that owns all device memory, or a loop that must
 * not call cudaMalloc between launches).  This call allocates nothing.
 *   - Size limit: the layout qd_pcg_workspace_size(n, nrhs) reports must fit
 *     in qd_pcg_static_scratch_bytes() (16 MiB, roughly n * nrhs <= 400k);
 *     larger problems return QD_ERR_LIMIT without launching anything.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress, with that device current); make that first call
 *     before any stream capture.  Under CUDA's default lazy module loading
 *     that lookup is also what loads this code's module on the device, and
 *     so what reserves the 16 MiB there: a caller inside a runtime that owns
 *     all device memory should make the first call during its own set-up,
 *     while memory is still free.  The address is cached per device for the
 *     life of the process; cudaDeviceReset between calls is not supported.
 *   - All calls share the one array and it keeps the previous call's
 *     contents; each call zeroes its block counter (a memset on the stream)
 *     and rewrites every other scratch word before reading it, so nothing
 *     needs clearing, but calls that overlap on the GPU (other streams, other
 *     host threads) race on it and must be serialised by the caller. */
size_t qd_pcg_static_scratch_bytes(void);
int qd_pcg_solve_static(int32_t n, int nrhs, const int32_t *d_rowptr, const int32_t *d_col,
                        const double *d_A, const double *d_B, double *d_X,
                        const int32_t *d_fixed, double tol, int max_iter, int32_t *h_iters,
                        double *h_relres, void *stream);

/* Y = alpha A X for nrhs row-major columns (generic FP64 CSR product).  Used
 * for the Poisson right-hand side M (-rho), which
 * qdsim_cython/solvers/poisson_solver.pyx:254-274 forms as mass_matrix.dot(rhs). */
int qd_csr_spmv(int32_t n, int nrhs, const int32_t *d_rowptr, const int32_t *d_col,
                const double *d_A, const double *d_X, double *d_Y, double alpha, void *stream);

/* Open-system (CAP) pencil products: AX = (H + i Himag) X and MX = M X for b
 * complex vectors (1 <= b <= 64), row-major with re/im interleaved,
 * X[row * ldx + c] and AX/MX[row * ldy + c] (leading dimensions in complex
 * elements, >= b).  H, Himag and M share one CSR pattern (qd_assemble's
 * outputs); Himag may be NULL (Hermitian pencil).  vec_fp32 selects
 * float/float2 for the matrix values and vectors, else double/double2.
 * Replaces the complex SpMV inside scipy's shift-invert eigs, which the
 * oracle of the complex eigenvalue configuration runs, and the dense complex
 * solve of backend/src/schrodinger.cpp:699-818. */
int qd_cap_spmm(int32_t n, int b, int vec_fp32, const int32_t *d_rowptr, const int32_t *d_col,
                const void *d_H, const void *d_Himag, const void *d_M, const void *d_X, int ldx,
                void *d_AX, void *d_MX, int ldy, void *stream);

/* ---------------------------------------------------------------------------
 * Open-system eigensolve: the k eigenvalues nearest sigma of the complex-
 * symmetric pencil (H + i Himag, M), from block LOBPCG over the nev
 * eigenvalues of smallest real part, entirely on the device.  Replaces the
 * dense complex solve of backend/src/schrodinger.cpp:699-818 (regularised
 * Cholesky of M + Eigen ComplexEigenSolver).
 *   pencil       CSR of n rows (Dirichlet rows removed), FP64 H, Himag
 *                (NULL: Hermitian pencil) and M; FP32 copies for the mixed
 *                form (QD_PREC_MIXED: FP32 vectors and products until the
 *                residuals reach tol32 or stop improving for 8 iterations,
 *                then FP64 vectors warm-started from them; QD_PREC_FP64:
 *                FP64 throughout)
 *   h_prec       DST preconditioner descriptor of the pencil's lattice
 *                (qd_dst_prec, one dot; NULL: none), d_prec_mats its
 *                matrices (qd_dst_matrix_fill layout)
 *   b            block size, even, 2..48 (>= nev; the projected problem is
 *                3b x 3b), nev <= b levels must converge, k <= nev returned
 *   tol          relative residual ||A x - theta M x|| / (||M x|| max(|theta|,
 *                eig_scale)) every one of the nev lowest Ritz pairs reaches
 *   seed         start block (uniform complex entries in [-1, 1)^2), or
 *                d_X0 (complex128 [n][b], FP64 form only)
 * Rayleigh-Ritz: Hermitian M-orthonormal basis of [X P W] (Cholesky of the
 * diagonally scaled Gram matrix, SVQB when its pivots fall below 1e-6), the
 * projected non-Hermitian matrix reduced to Schur form by a Jacobi-like
 * method on an 8-CTA cluster (qd_complex_schur), Ritz vectors by back-
 * substitution, the b of smallest real part kept.
 * Outputs: h_E [2k] (re, im) eigenvalues nearest sigma first (the bilinear
 * Rayleigh quotients x^T A x / x^T M x), d_Xout complex128 [n][k] with
 * x^T M x = 1, h_res [k] relative residuals ||A x - E M x|| / (|E| ||M x||),
 * h_info (complete = 1 when no unconverged Ritz value can lie nearer sigma
 * than the k-th returned eigenvalue).  Returns QD_ERR_NOT_CONVERGED (outputs
 * written) when max_iter ends the FP64 phase first.
 * ------------------------------------------------------------------------- */
typedef struct qd_cap_info {
  int32_t iters_fp32, iters_fp64;   /* iterations of each phase */
  int32_t converged, selected;      /* converged among nev; returned (<= k) */
  int32_t complete;                 /* certified nearest sigma */
  int32_t schur_sweeps_max;         /* largest sweep count of a Schur solve */
  int32_t schur_unconverged;        /* Schur solves stopped by the sweep cap */
  int32_t pad;
  double fp32_residual;             /* largest residual at the FP32 hand-over */
  double kth_distance;              /* |E_k - sigma| of the k-th returned */
  double unconverged_bound;         /* min Re(theta) - sigma over unconverged */
  double max_residual;              /* largest h_res */
} qd_cap_info;
int qd_cap_lobpcg_workspace_size(int32_t n, int b, int precision, const qd_dst_prec *h_prec,
                                 size_t *bytes);
int qd_cap_lobpcg_solve(int32_t n, const int32_t *d_rowptr, const int32_t *d_col,
                        const double *d_H, const double *d_Himag, const double *d_M,
                        const float *d_H32, const float *d_Himag32, const float *d_M32,
                        const qd_dst_prec *h_prec, const void *d_prec_mats, int b, int nev, int k,
                        double sigma, double tol, double tol32, int max_iter, int precision,
                        double eig_scale, uint64_t seed, const void *d_X0, double *h_E,
                        void *d_Xout, double *h_res, qd_cap_info *h_info, void *d_work,
                        size_t work_bytes, void *stream);

/* Schur form C = Z T Z^H of one n x n complex matrix (n <= 144; complex128,
 * row-major, leading dimensions ldc and ldt): T upper triangular, Z unitary,
 * by cyclic 2 x 2 unitary rotations in parallel round-robin order (Stewart's
 * Jacobi-like method for non-Hermitian matrices) on an 8-CTA cluster; a
 * Hermitian C gives its eigendecomposition.  Stops after a sweep in which no
 * element below the diagonal exceeded 1e-14 ||C||_F (QD_ERR_NOT_CONVERGED
 * after max_sweeps sweeps, outputs written).  h_sweeps: sweeps run. */
int qd_complex_schur(int n, const void *d_C, int ldc, void *d_T, void *d_Z, int ldt, int max_sweeps,
                     int *h_sweeps, void *stream);

/* ---------------------------------------------------------------------------
 * Finite-element field evaluation at arbitrary points on the structured
 * order-p mesh of [0, Lx] x [0, Ly] with nx x ny cells (lattice node order,
 * element 2 (cj nx + ci) + t).  Replaces FEInterpolator::interpolate,
 * interpolateWithGradient and findElement
 * (backend/src/fe_interpolator.cpp:54-431) and interpolate_field_kernel
 * (backend/src/gpu_kernels.cu:352-423), which scan every element per point;
 * here the point's cell is computed: a point well inside its own cell's
 * triangle is settled by that one test, any other point by testing the
 * triangles of the 3 x 3 cells around it in element order, so the containing
 * element is the one the scan returns (the first with all barycentric
 * coordinates >= -1e-10).
 *   d_field     nfield fields, field f at d_field + f * field_stride
 *               (field_stride >= number of nodes)
 *   d_x, d_y    npts query points
 *   d_value     [nfield * npts] values, value[f * npts + i]
 *   d_grad_x/y  [nfield * npts] gradients, both NULL for none
 *   d_element   [npts] containing element or -1 (NULL for none)
 *   outside_zero  0: points outside every element take the nearest node's
 *               value and the reference's neighbour-difference gradient
 *               estimate (FEInterpolator); 1: value and gradient 0
 *               (interpolate_field_kernel).
 * Returns QD_ERR_LIMIT when node or element indices would exceed int32. */
int qd_fe_interpolate(int order, int32_t nx, int32_t ny, double Lx, double Ly, int nfield,
                      int64_t field_stride, const double *d_field, int64_t npts,
                      const double *d_x, const double *d_y, double *d_value, double *d_grad_x,
                      double *d_grad_y, int32_t *d_element, int outside_zero, void *stream);

/* Field evaluation on an unstructured (refined) order-p triangular mesh over
 * [0, Lx] x [0, Ly], with the same outputs, outside-point rules and element
 * choice as qd_fe_interpolate (the reference scans every element,
 * backend/src/fe_interpolator.cpp:54-431; its refined meshes come from
 * FEMSolver::adapt_mesh, backend/src/fem.cpp:486-542).  Points are located
 * through a bucket grid of grid_nx x grid_ny cells: d_cell_ptr
 * int32[grid_nx * grid_ny + 1] and d_cell_elems list, per cell and in
 * ascending element order, the elements whose vertex bounding box, padded by
 * more than the -1e-10 acceptance band, meets the cell.  The nearest-node
 * search of outside points covers the cells within max(cell width, cell
 * height) of the point's projection onto the rectangle, which holds the
 * nearest node when every corner of every cell is a node (a mesh refined from
 * the grid_nx x grid_ny structured mesh).  d_nadjptr / d_nadj: node adjacency
 * from qd_node_adjacency (needed only with gradients).  d_nodes double2. */
int qd_fe_interpolate_tri(int order, int64_t num_nodes, int64_t num_elems,
                          const double *d_nodes, const int32_t *d_elems, int32_t grid_nx,
                          int32_t grid_ny, double Lx, double Ly, const int32_t *d_cell_ptr,
                          const int32_t *d_cell_elems, const int32_t *d_nadjptr,
                          const int32_t *d_nadj, int nfield, int64_t field_stride,
                          const double *d_field, int64_t npts, const double *d_x,
                          const double *d_y, double *d_value, double *d_grad_x, double *d_grad_y,
                          int32_t *d_element, int outside_zero, void *stream);

/* ---------------------------------------------------------------------------
 * Adjoint (Hellmann-Feynman) gradients of L = Re sum_s w_s E_s with respect
 * to nodal V and the per-element kinetic coefficient c.  M depends on neither,
 * so with normalised eigenvectors dE_s/dp = x_s^T (dH/dp) x_s:
 *   - Hermitian pencil (is_complex = 0): real x_s with x^T M x = 1;
 *   - complex-symmetric open-system pencil H + i Himag (is_complex = 1):
 *     complex x_s with the bilinear normalisation x^T M x = 1 (no
 *     conjugation; the left eigenvector of a complex-symmetric pencil is x
 *     itself), complex weights w_s = dL/dRe E_s - i dL/dIm E_s.
 * No reference counterpart: the reference has no derivatives (its CAP pencil
 * is solved densely in backend/src/schrodinger.cpp:699-818, with the
 * (V + i eta) weak form of backend/src/fem.cpp:970-976); the checker is central
 * finite differences of the FP64 eigenvalues and the FP64 oracle gradient.
 *   d_psi        is_complex = 0: double[n_dofs * n_states] (psi[dof*n_states + s]);
 *                is_complex = 1: interleaved (re, im) pairs, 16-byte aligned
 *   d_w          double[n_states] (real) or [2 * n_states] (re, im per state)
 *   d_nadjptr/d_nadj  node adjacency from qd_node_adjacency
 *   d_dofmap     int32[num_nodes] (-1 for an eliminated node: psi = 0 there)
 *   outputs      d_dLdV[num_nodes], d_dLdc[num_elems] (caller-allocated)
 *   d_work       scratch, double[num_elems * k] (k = 3, 6, 10 nodes per element)
 * Two launches (element pass, node gather); every output is a fixed-order
 * sum (reproducible, no atomics).
 * ------------------------------------------------------------------------- */
int qd_adjoint(int order, int64_t num_nodes, int64_t num_elems, int n_states, int is_complex,
               const double *d_nodes, const int32_t *d_elems, const int32_t *d_dofmap,
               const double *d_psi, const double *d_w,
               const int32_t *d_nadjptr, const int32_t *d_nadj,
               double *d_dLdV, double *d_dLdc, double *d_work, void *stream);

/* ---------------------------------------------------------------------------
 * Per-kernel-kind timing with CUDA events, recorded on the stream of each
 * launch (off by default).  Kinds: 0 SpMM, 1 Gram, 2 Rayleigh-Ritz, 3 update,
 * 4 assembly, 5 PCG, 6 adjoint, 7 DST preconditioner, 8 orthogonalisation,
 * 9 other.  qd_prof_read synchronises the recorded events and returns
 * cumulative milliseconds and launch counts (arrays of 10); reset != 0 clears
 * the totals.  Benchmark instrumentation with
 * no reference counterpart.
 * ------------------------------------------------------------------------- */
int qd_prof_enable(int on);
int qd_prof_read(double *ms, int64_t *launches, int reset);

/* ---------------------------------------------------------------------------
 * Failure-path diagnostic with no reference counterpart (the reference's GPU
 * code has no device-side waits; its failure handling is the host-side
 * RecoveryManager of backend/include/recovery_manager.h:47, which returns
 * dummy eigenpairs from backend/src/solver.cpp:183-192).  Runs the bounded
 * mbarrier wait that every bulk-copy pipeline of this library uses on a
 * barrier that nothing completes, with a limit of limit_ns (capped at 2 s):
 * the wait expires, the kernel records it in *d_status (bit 0), drains its own
 * 256-byte bulk copy from d_src when with_copy != 0 (16-byte aligned; bit 1 if
 * that drain also expired, bit 2 if the copied bytes differ) and returns.
 * Synchronises `stream`; *h_status receives the status word.  Returns
 * QD_ERR_TIMEOUT when the wait expired (the expected outcome), the status
 * production entry points return after such an expiry.
 * ------------------------------------------------------------------------- */
int qd_bounded_wait_selftest(int64_t limit_ns, const void *d_src, int with_copy,
                             int32_t *d_status, int32_t *h_status, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* QDSIM_B200_H */
