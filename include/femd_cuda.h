/*
 * femd_cuda.h -- the C ABI of libfemd_cuda.so: FEMd's 2D Lagrange P_k triangle assembly into
 * CSR and its Jacobi-preconditioned CG solve, on one NVIDIA B200 (sm_100a).
 *
 * This is the drop-in boundary.  Every entry point replaces one function of FEMd's own
 * nanobind module `_femd` (python/src/femd_bindings*.cpp in the FEMd tree), named beside
 * it, with the same argument meaning and the same error behaviour: where the reference
 * throws std::invalid_argument the call returns FEMD_EINVAL, std::logic_error /
 * std::runtime_error give FEMD_EOUTSIDE / FEMD_EZERODIAG, and the text of the reference's
 * exception is available from femd_cuda_last_error().  CG non-convergence and breakdown are
 * not errors (the reference reports them in its result tuple): they are fields of
 * femd_cg_result and the call returns FEMD_OK.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Arrays named *_dev are device pointers (cudaMalloc'd or
 *     any device-accessible memory of the context's device); arrays named *_host are host
 *     pointers (pageable or pinned).  Index arrays are int32, values float64 unless named f32.
 *   - Every call is asynchronous on the context's stream unless it returns a host value or
 *     fills a host array, in which case it synchronizes that stream before returning.
 *   - Handles (femd_pattern, femd_matrix, femd_solver) own device memory; release them with
 *     femd_cuda_release().  Calls on different contexts may run concurrently from different
 *     host threads; one context must not be used by two threads at once.
 *   - femd_cuda_last_error() is per host thread.
 */
#ifndef FEMD_CUDA_H
#define FEMD_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FEMD_API __attribute__((visibility("default")))
#else
#define FEMD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------------- */
#define FEMD_OK          0
#define FEMD_EINVAL      1   /* bad argument (reference: std::invalid_argument -> ValueError) */
#define FEMD_ENOMEM      2   /* device or host allocation failed */
#define FEMD_ECUDA       3   /* a CUDA runtime error; femd_cuda_last_error() has its text */
#define FEMD_EOUTSIDE    4   /* an element entry outside the pattern (reference: std::logic_error) */
#define FEMD_EZERODIAG   5   /* Jacobi: zero diagonal entry (reference: std::invalid_argument) */
#define FEMD_ETIMEOUT    6   /* a bounded device-side wait ran out (batched / served solves) */
#define FEMD_EABORT      7   /* a host-requested abort stopped a batched solve */
#define FEMD_EPIVOT      8   /* ILU(0): a zero pivot (reference: std::runtime_error -> RuntimeError) */

typedef struct femd_ctx_s *femd_ctx;
typedef struct femd_pattern_s *femd_pattern;
typedef struct femd_matrix_s *femd_matrix;
typedef struct femd_precond_s *femd_precond;

/* Last error text of this host thread ("" when none). */
FEMD_API const char *femd_cuda_last_error(void);
/* Library version string. */
FEMD_API const char *femd_cuda_version(void);
/* Kernel launches this library has issued in this process (a launched CUDA graph counts its
 * kernel nodes).  No reference counterpart: an instrumentation counter. */
FEMD_API long long femd_cuda_kernel_launches(void);

/* A context: one device and one stream (created, non-blocking).  device < 0: the current device. */
FEMD_API int femd_cuda_ctx_create(int device, femd_ctx *out);
FEMD_API int femd_cuda_ctx_destroy(femd_ctx ctx);
/* The context's stream, as a cudaStream_t cast to void*. */
FEMD_API void *femd_cuda_ctx_stream(femd_ctx ctx);
/* Wait for all work queued on the context's stream. */
FEMD_API int femd_cuda_ctx_sync(femd_ctx ctx);
/* Release any handle created by this library (pattern, matrix, solver, batch). NULL is a no-op. */
FEMD_API void femd_cuda_release(void *handle);

/* ======================================================================================
 * Sparsity pattern: K1.
 * Replaces cell_pattern(T, S) (python/src/femd_bindings_2d.cpp:762) ->
 * SparsityPattern::from_cells (include/femd/sparse/csr.hpp:84-125), for a square pattern
 * whose rows and columns are numbered by the same cell->dof map (T == S).
 * cell_dofs_dev: ncells x nloc, -1 for a constrained (eliminated) node.
 * The result is bit-identical to the reference's indptr / indices.  The handle also keeps,
 * for every row, the (cell, local index) pairs holding it in increasing cell order (the
 * reference's cellof lists, csr.hpp:90-98), which the assembly kernels use.
 * ====================================================================================== */
FEMD_API int femd_cuda_pattern_from_cells(femd_ctx ctx, int nrows, int ncells, int nloc, const int *cell_dofs_dev,
                                 femd_pattern *out);
FEMD_API int femd_cuda_pattern_info(femd_pattern p, int *nrows, int *ncols, long long *nnz);
/* Device views of the pattern's arrays (owned by the pattern). */
FEMD_API int femd_cuda_pattern_arrays(femd_pattern p, const int **indptr_dev, const int **indices_dev);
/* Copy indptr (nrows + 1) and indices (nnz) to host arrays; synchronizes. */
FEMD_API int femd_cuda_pattern_to_host(femd_pattern p, int *indptr_host, int *indices_host);
/* A pattern from existing CSR arrays (copied to the device; rows must be sorted and unique,
 * as CSRMatrix.from_arrays requires, python/src/femd_bindings_2d.cpp:101-116). */
FEMD_API int femd_cuda_pattern_from_csr_host(femd_ctx ctx, int nrows, int ncols, const int *indptr_host,
                                    const int *indices_host, femd_pattern *out);

/* ======================================================================================
 * Scatter map: K2.
 * Replaces scatter_map_2d(QT, QS, P, 0, 0) (include/femd/forms/assembly_2d.hpp:136-164):
 * map_dev[(e nloc + i) nloc + j] = position of (dof(e,i), dof(e,j)) in the pattern's
 * indices, -1 where either is constrained.  Returns FEMD_EOUTSIDE (the reference throws
 * std::logic_error "assemble_matrix_2d: entry outside the pattern") if an entry is missing.
 * The map is also kept inside the pattern (femd_cuda_pattern_map) for the assembly kernels.
 * ====================================================================================== */
FEMD_API int femd_cuda_scatter_map(femd_ctx ctx, femd_pattern p, int *map_dev);
FEMD_API int femd_cuda_pattern_map(femd_pattern p, const int **map_dev);

/* ======================================================================================
 * Matrices: values on a pattern.
 * Replaces CSRMatrix(pattern) (python/src/femd_bindings_2d.cpp:101) and the Jacobi
 * preconditioner JacobiPreconditioner(K) (include/femd/sparse/precond.hpp:82-102), whose
 * inverse diagonal the matrix keeps (computed by the assembly epilogue or by
 * femd_cuda_matrix_jacobi).
 * ====================================================================================== */
FEMD_API int femd_cuda_matrix_create(femd_ctx ctx, femd_pattern p, femd_matrix *out);
FEMD_API int femd_cuda_matrix_arrays(femd_matrix K, double **data_dev, double **inv_diag_dev);
FEMD_API int femd_cuda_matrix_set_host(femd_matrix K, const double *data_host);
FEMD_API int femd_cuda_matrix_to_host(femd_matrix K, double *data_host);
/* inv_diag = 1 / a_ii; FEMD_EZERODIAG with "Jacobi: zero diagonal entry in row i"
 * (precond.hpp:68-78) when some a_ii is 0 or missing.
 * A new matrix has no inverse diagonal: every preconditioned solve (femd_cuda_cg_jacobi with
 * use_jacobi, femd_cuda_pcg_mixed, femd_cuda_cg_jacobi_noalloc with use_jacobi, femd_cuda_batch_add)
 * returns FEMD_EINVAL until this call, an assembly with want_inv, or femd_cuda_matrix_set_inv_diag
 * has written it.  Changing the values later does not refresh it (the reference's
 * JacobiPreconditioner also keeps the diagonal of the matrix it was made from). */
FEMD_API int femd_cuda_matrix_jacobi(femd_ctx ctx, femd_matrix K);
/* Give K the inverse diagonal inv_dev (nrows device values, copied on the context's stream): the
 * preconditioner of another matrix of the same size, as cg_solve(A, M, ...) accepts an M built from
 * another matrix (python/src/femd_bindings.cpp:799-833).  No zero check. */
FEMD_API int femd_cuda_matrix_set_inv_diag(femd_ctx ctx, femd_matrix K, const double *inv_dev);
/* Copy of the inverse diagonal to the host (nrows); synchronizes. */
FEMD_API int femd_cuda_matrix_inv_diag_to_host(femd_matrix K, double *inv_host);

/* ======================================================================================
 * Assembly: K3 (matrix) and K4 (vector).
 * Replaces assemble_matrix_2d (python/src/femd_bindings_2d.cpp:810-816 ->
 * include/femd/forms/assembly_2d.hpp:219-305) and assemble_vector_2d (:817-822 ->
 * assembly_2d.hpp:173-211) on affine triangles, with the geometry read from the mesh
 * (vertex coordinates and triangles) instead of per-point arrays: J = [P1-P0, P2-P0],
 * w = rw |det J|, J^{-1} as in lagrange_space_2d.hpp:44-52 and cache_2d.hpp:110-118.
 *
 *   K  = sum_t integral c_t (D^{a_t} phi_i)(D^{b_t} phi_j)        codes 0 value, 1 d/dx, 2 d/dy
 *   f  = sum_t integral c_t (D^{a_t} phi_i)
 *
 * The rule is the reference tabulation of the cell cache (Cache2D::ref: nq points x
 * [phi, dphi/dxi, dphi/deta] x nloc, host array) with the reference points and weights.
 * Coefficients: one femd_coef per term.  Each matrix entry and vector entry is summed in
 * increasing cell order with no atomics (deterministic, the reference's order).
 * mode FEMD_ASM_FAST contracts per-cell geometric factors with precomputed reference
 * tensors; FEMD_ASM_EXACT forms every element entry with the reference's own operation
 * order (element_matrix_2d, assembly_2d.hpp:102-126, no fused multiply-adds) and so gives
 * the reference's bits for the same tabulation and coefficients.
 * ====================================================================================== */
#define FEMD_COEF_CONST   0   /* value */
#define FEMD_COEF_POINTS  1   /* points_dev[e nq + q] (the reference's coefficient arrays) */
#define FEMD_COEF_SINSIN  2   /* p0 + p1 sin(p2 x) sin(p3 y) */
#define FEMD_COEF_SINSIN_HELM 3 /* p0 s + s, s = sin(p2 x) sin(p3 y) (the written sum of two terms) */
#define FEMD_COEF_FIELD   4   /* a P_k field at the points: sum_l phi_l(q) field_dev[dof(e,l)] (Cache2D::eval_multi) */

typedef struct {
    int kind;
    double value;
    const double *points_dev;
    const double *field_dev;
    double p[4];
} femd_coef;

#define FEMD_ASM_FAST  0
#define FEMD_ASM_EXACT 1

typedef struct {
    int nverts, ncells;
    const double *points_dev;   /* nverts x 2 */
    const int *tris_dev;        /* ncells x 3, counter-clockwise */
} femd_mesh2d;

typedef struct {
    int k, nloc, nq;
    const double *ref_host;     /* nq x 3 x nloc */
    const double *xi_host, *eta_host, *w_host;   /* nq reference points and weights */
} femd_rule;

/* K (values overwritten) = the form; also refreshes K's inverse diagonal when want_inv. */
FEMD_API int femd_cuda_assemble_matrix(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, femd_pattern p,
                              int nterms, const int *a, const int *b, const femd_coef *coef, int mode, femd_matrix K,
                              int want_inv);
/* f_dev (nrows entries, overwritten) = the rank-1 form; the pattern supplies the row lists. */
FEMD_API int femd_cuda_assemble_vector(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, femd_pattern p,
                              int nterms, const int *a, const femd_coef *coef, int mode, double *f_dev);

/* ======================================================================================
 * Coefficients of a compiled form: the Integrand register program and fields at the points.
 * Replaces Integrand::evaluate (include/femd/forms/integrand.hpp:85-109, the program run of
 * :300-342, checks of :47-66, reached through FormAssembler2D::coefficients,
 * include/femd/forms/assembler_2d.hpp:393-410) and Cache2D::eval_multi
 * (include/femd/fe/cache_2d.hpp:245-288, FormAssembler2D::evaluate_fields).  A program is the
 * reference's format -- what python/femd/forms.py:1822-1938 (_Program) emits: 4 integers per
 * instruction (op, out register, a, b) with the opcodes of integrand.hpp:33-45 (CONST 0, X 1,
 * Y 2, NX 3, NY 4, INPUT 5, ADD 6, MUL 7, POW 8, SIN 9 ... SIGN 19); the result is the last
 * instruction's register.  Errors carry the reference's messages (FEMD_EINVAL).  Sums and
 * products are exact IEEE operations as in the reference; the transcendental functions are
 * CUDA's (within a few ulp of the host C library's).  Limits of this evaluator: 160 registers,
 * 2048 instructions, 1024 constants, 16 inputs.
 * ====================================================================================== */
typedef struct {
    const int *code_host;   /* ncode = 4 x instructions */
    int ncode, nreg, nconst, ninput;
} femd_integrand;

/* out_dev[q] (npts values) = the program at given points: inputs_dev[i] are ninput device arrays
 * of npts values, consts_host nconst values, xs/ys and nx/ny device arrays (NULL when the program
 * does not read them).  Synchronizes. */
FEMD_API int femd_cuda_integrand_eval(femd_ctx ctx, const femd_integrand *prog, const double *consts_host,
                                      const double *const *inputs_dev, long long npts, const double *xs_dev,
                                      const double *ys_dev, const double *nx_dev, const double *ny_dev, double *out_dev);
/* The same at the points of a cell rule, out_dev[e nq + q] (ncells x nq): x and y formed from the
 * mesh as the reference's cell cache does; a program that reads the normal is refused on cells
 * (FormAssembler2D::add_term).  Synchronizes. */
FEMD_API int femd_cuda_integrand_eval_cells(femd_ctx ctx, const femd_integrand *prog, const double *consts_host,
                                            const double *const *inputs_dev, const femd_mesh2d *mesh, const femd_rule *rule,
                                            double *out_dev);
/* A P_k field at the points of a cell rule (Cache2D::eval_multi): out_dev[i np + e nq + q] for
 * codes[i] in {0 value, 1 d/dx, 2 d/dy} (1 to 3 codes, np = ncells nq); cell_dofs_dev the
 * ncells x nloc dof map of the field's coefficients (-1: the node reads 0).  Synchronizes. */
FEMD_API int femd_cuda_eval_field(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, const int *cell_dofs_dev,
                                  const double *field_dev, int ncodes, const int *codes, double *out_dev);

/* ======================================================================================
 * Facet (ds) terms and the Dirichlet lift.
 * Replaces the exterior-facet cache Cache2D(V, degree, markers, all)
 * (include/femd/fe/cache_2d.hpp:126-184) with assemble_matrix_2d / assemble_vector_2d on it
 * (include/femd/forms/assembly_2d.hpp:173-305), i.e. the ds(marker) terms of a form (Robin and
 * Neumann data), and the pieces of the Dirichlet lift of fd.solve(a, L, dirichlet=g)
 * (python/femd/linalg.py:748-755, V.lift at python/femd/spaces2d.py:373-414).  A facet set is a
 * list of (cell, local edge) -- local edge i joins the cell's vertices (i + 1) % 3 and (i + 2) % 3 --
 * in the reference's facet order (femd_host_exterior_facets), on a cell pattern.  Assembly adds
 * into K / f: every touched value gets its facets' element entries in increasing facet order, the
 * order of the reference (no atomics).
 * ====================================================================================== */
typedef struct femd_facets_s *femd_facets;

typedef struct {
    int k, nloc, nq;
    const double *xi_host, *eta_host;   /* 3 x nq: the points on local edge 0, 1, 2 (reference coordinates) */
    const double *gw_host;              /* nq Gauss-Legendre weights on [-1, 1] */
    const double *ref_host;             /* 3 x nq x 3 x nloc: the tabulation per local edge */
} femd_facet_rule;

/* A facet set on a cell pattern (copies the list; release with femd_cuda_release). */
FEMD_API int femd_cuda_facets_create(femd_ctx ctx, femd_pattern p, int nf, const int *fcell_host, const int *flocal_host,
                                     femd_facets *out);
/* Per facet point [f nq + q]: x, y, the weight 0.5 gw len, the outward unit normal (any output may
 * be NULL).  Synchronizes. */
FEMD_API int femd_cuda_facet_points(femd_ctx ctx, femd_facets F, const femd_mesh2d *mesh, const femd_facet_rule *rule,
                                    double *x_dev, double *y_dev, double *w_dev, double *nx_dev, double *ny_dev);
/* K += sum_t integral over the facets of c_t (D^{a_t} phi_i)(D^{b_t} phi_j) ds; coef[t] a constant or
 * an array at the facet points (FEMD_COEF_POINTS, [f nq + q]).  Synchronizes. */
FEMD_API int femd_cuda_assemble_facet_matrix(femd_ctx ctx, femd_facets F, const femd_mesh2d *mesh,
                                             const femd_facet_rule *rule, int nterms, const int *a, const int *b,
                                             const femd_coef *coef, femd_matrix K);
/* f += sum_t integral over the facets of c_t (D^{a_t} phi_i) ds.  Synchronizes. */
FEMD_API int femd_cuda_assemble_facet_vector(femd_ctx ctx, femd_facets F, const femd_mesh2d *mesh,
                                             const femd_facet_rule *rule, int nterms, const int *a, const femd_coef *coef,
                                             double *f_dev);
/* u_raw[raw_of[i]] = x[i] for i < n: a solution on the space's dofs written into the raw numbering
 * over a lift (the reference's V.prolongate(c) + u_g, python/femd/spaces2d.py:373-385). */
FEMD_API int femd_cuda_prolongate(femd_ctx ctx, int n, const int *raw_of_dev, const double *x_dev, double *u_raw_dev);

/* ======================================================================================
 * Sparse kernels on a matrix.
 * ====================================================================================== */
/* y = K x: CSRMatrix::apply (include/femd/sparse/csr.hpp:203-215). */
FEMD_API int femd_cuda_spmv(femd_ctx ctx, femd_matrix K, const double *x_dev, double *y_dev);
/* Autotuner of the SpMV (no reference counterpart: the reference's loop has no launch shape):
 * times the launch shapes on K -- threads per row 2..32 (low byte) | loads in flight per lane
 * 1, 2, 4 (next byte) -- and returns the fastest (and, with set != 0, keeps it for K's SpMV and
 * CG).  Threads per row changes the summation order of a row, so a tuned matrix may give
 * results that differ from an untuned one in the last bits; loads per lane does not. */
FEMD_API int femd_cuda_spmv_autotune(femd_ctx ctx, femd_matrix K, int set, int *shape_out, double *us_out);
/* Fix K's SpMV shape (0 = the built-in heuristic). */
FEMD_API int femd_cuda_spmv_set_tpr(femd_matrix K, int shape);
/* max |a_ij - a_ji| / max |a_ij|: asymmetry (csr.hpp:632-645); synchronizes. */
FEMD_API int femd_cuda_asymmetry(femd_ctx ctx, femd_matrix K, double *out);
/* C = alpha A + beta B on one shared pattern: combine (csr.hpp:315-326). */
FEMD_API int femd_cuda_combine(femd_ctx ctx, double alpha, femd_matrix A, double beta, femd_matrix B, femd_matrix C);

/* ======================================================================================
 * Jacobi-PCG: K5 (SpMV fused with p^T A p) and K6 (fused update with ||r||^2 and r^T D^-1 r).
 * Replaces cg_solve(A, M, b, x0, max_iter, tol) (python/src/femd_bindings.cpp:799-833) with
 * M a JacobiPreconditioner or None -> krylov::cg_jacobi (include/femd/krylov/cg.hpp:296-350)
 * with the same stopping rule, final true residual, 10 tol acceptance and breakdown tests
 * (cg.hpp:222-237).  The reductions are deterministic (fixed order, the same bits on every
 * run) but not the reference's chunk order, so iteration counts may differ by a few.
 * ====================================================================================== */
typedef struct {
    int converged;
    int iterations;
    double residual;      /* ||b - A x|| / ||b||, recomputed at the end */
    int breakdown;        /* p^T A p <= 0 or r^T z <= 0 */
    int status;           /* FEMD_OK, or FEMD_ETIMEOUT / FEMD_EABORT for bounded solves */
    int outer;            /* refinement steps (mixed precision), 0 otherwise */
    double seconds;       /* device time of the solve (CUDA events) */
} femd_cg_result;

/* x_dev: initial guess in, solution out.  use_jacobi 0: no preconditioner (M = None). */
FEMD_API int femd_cuda_cg_jacobi(femd_ctx ctx, femd_matrix K, int use_jacobi, const double *b_dev, double *x_dev, int max_iter,
                        double tol, femd_cg_result *res);
/* The same with host CSR arrays and vectors (the exact data the reference binding holds):
 * uploads A and b, solves, writes x back; inv_host may be NULL (no preconditioner) or the
 * reference's JacobiPreconditioner.inverse_diagonal(). */
FEMD_API int femd_cuda_cg_solve_host(femd_ctx ctx, int n, const int *indptr_host, const int *indices_host,
                            const double *data_host, const double *inv_host, const double *b_host, const double *x0_host,
                            double *x_host, int max_iter, double tol, femd_cg_result *res);

/* Device time of one launch of a kernel of the FP64 Jacobi-PCG loop on K (CUDA events on the
 * context's stream, averaged over reps back-to-back launches after a warm-up): kernel 0 the SpMV
 * with the fused p.Ap (K5), 1 the fused update x += a p, r -= a Ap, ||r||^2, r.D^-1 r (K6), 2 the
 * direction update p = D^-1 r + b p.  Runs on K's solver workspace with a = b = 0 (the same bytes
 * as a real iteration).  Instrumentation with no reference counterpart.  Synchronizes. */
FEMD_API int femd_cuda_kernel_time(femd_ctx ctx, femd_matrix K, int kernel, int reps, double *us_out);

/* ======================================================================================
 * The stronger preconditioners: ILU(0) and SSOR on the natural ordering, and CG with them.
 * Replace ILU0Preconditioner(A) and SSORPreconditioner(A, omega) (include/femd/sparse/precond.hpp:
 * 105-213; python/src/femd_bindings*.cpp, A.preconditioner("ilu0" / "ssor")) and krylov::cg with a
 * general preconditioner (include/femd/krylov/cg.hpp:245-290), reached by A.solver("cg") whose
 * default M is "ilu0" (python/femd/sparse.py:440-446).  The factors and every application are
 * bit-identical to the reference's (each row's arithmetic is the reference's, rows of one level of
 * the triangular dependency done together); CG's reductions are deterministic in their own order.
 * Errors: FEMD_EINVAL "ILU(0): zero diagonal entry in row i" / "SSOR: ..." and "SSOR: omega must
 * lie in (0, 2)"; FEMD_EPIVOT "ILU(0): zero pivot in row i".  The preconditioner copies K's values
 * (later changes to K do not reach it) and keeps K's pattern.
 * ====================================================================================== */
#define FEMD_PC_ILU0 1
#define FEMD_PC_SSOR 2
FEMD_API int femd_cuda_precond_create(femd_ctx ctx, femd_matrix K, int kind, double omega, femd_precond *out);
/* kind, the forward and backward level counts (the sweeps' sequential steps), ILU(0)'s smallest pivot
 * (min_pivot(): negative means the factorization is indefinite). */
FEMD_API int femd_cuda_precond_info(femd_precond P, int *kind, int *levels_forward, int *levels_backward, double *min_pivot);
/* z = M^{-1} r (r and z device vectors of nrows, distinct), asynchronous on the context's stream. */
FEMD_API int femd_cuda_precond_apply(femd_ctx ctx, femd_precond P, const double *r_dev, double *z_dev);
/* krylov::cg(A, M, x, b, max_iter, tol) with M = P (built on K's pattern): the stopping rule, final true
 * residual, 10 tol acceptance and breakdown tests of cg.hpp:245-290 and 222-237. */
FEMD_API int femd_cuda_cg_precond(femd_ctx ctx, femd_matrix K, femd_precond P, const double *b_dev, double *x_dev,
                                  int max_iter, double tol, femd_cg_result *res);

/* Mixed precision: inner Jacobi-PCG on an FP32 copy of K with FP32 vectors and FP32
 * accumulation; the residual r = b - A x is recomputed on the FP64 matrix and the solution
 * updated in FP64 (reliable updates) until ||b - A x|| <= tol ||b||. */
FEMD_API int femd_cuda_pcg_mixed(femd_ctx ctx, femd_matrix K, const double *b_dev, double *x_dev, int max_iter, double tol,
                        femd_cg_result *res);

/* femd_cuda_cg_jacobi without any allocation.  It has no counterpart in the reference.
 * For callers that cannot call cudaMalloc while they solve: a solver embedded in a program
 * whose allocator already owns the device memory (a serving engine that reserved the HBM up
 * front, a framework whose memory pool must not be bypassed), or a latency-bound loop where an
 * allocation and the device synchronization it may bring are not allowed.  The caller passes
 * b and x as before; the solver's work vectors, reduction partials and state live in one fixed
 * static device array (about 25 MB, held by every GPU that loads the library until the process
 * exits) sized for at most 1,048,576 rows -- larger systems are rejected with FEMD_EINVAL.
 * The first call on a device (and the first after the device's CUDA context was made again, e.g.
 * after cudaDeviceReset) looks up that array's device address.  The solve reads its state back
 * between chunks (it synchronizes the context's stream), so it cannot be captured into a CUDA
 * graph: called while that stream is capturing it returns FEMD_EINVAL.  Every call shares the
 * array: calls that overlap on the GPU (any stream or context of the same device) race and must
 * be serialized.  The solve updates x in place and reads b
 * throughout, so b and x must not overlap (FEMD_EINVAL).  Same kernels and iterates as
 * femd_cuda_cg_jacobi; res->seconds is not measured (0). */
FEMD_API int femd_cuda_cg_jacobi_noalloc(femd_ctx ctx, femd_matrix K, int use_jacobi, const double *b_dev, double *x_dev,
                                         int max_iter, double tol, femd_cg_result *res);

/* ======================================================================================
 * Batched solves: K7.  Many independent Jacobi-PCG solves in ONE persistent cooperative
 * launch.  No single reference counterpart: it runs the reference's cg_jacobi
 * (include/femd/krylov/cg.hpp:296-350, stopping rule and final true residual included) for
 * every member system of the batch at once.  Each member gets a team of thread blocks sized
 * from its nonzeros; the ranks of a team meet at software barriers with bounded waits
 * (FEMD_ETIMEOUT when one runs out; every block then returns).  A member's result does not
 * depend on the rest of the batch: its reductions are ordered by the member and the launch
 * shape alone.  mixed != 0: FP32 matrix copy, vectors and SpMV accumulation, with FP64 reliable
 * updates (r = b - A x on the FP64 matrix, x updated in FP64) until ||b - A x|| <= tol ||b||.
 * Solves are resumable: femd_cuda_batch_step advances every armed member by a number of
 * iterations, so members can join (add + arm) and leave between launches (continuous
 * batching).  The matrices must outlive their membership.
 * ====================================================================================== */
typedef struct femd_batch_s *femd_batch;
/* A batch with members 0..nprob-1 = mats (nprob may be 0); nnz_per_block <= 0: 65536. */
FEMD_API int femd_cuda_batch_create(femd_ctx ctx, int nprob, const femd_matrix *mats, int nnz_per_block, femd_batch *out);
/* Solve every member to completion in one launch.  b_dev[p], x_dev[p]: device vectors of the
 * p-th member in id order (x: initial guess in, solution out).  max_iter <= 0: max(1000, 10 n)
 * per member.  results[p] per member; res.seconds = the launch. */
FEMD_API int femd_cuda_batch_solve(femd_ctx ctx, femd_batch B, const double *const *b_dev, double *const *x_dev,
                                   int max_iter, double tol, int mixed, femd_cg_result *results);
/* The same solve by the lockstep engine: every iteration is a few whole-GPU kernels over all the
 * members still running (an SpMV with the direction and p.Ap, the update; in mixed precision a
 * flush and an FP64 residual for the members due a reliable update), the members' sums taken in a
 * fixed order, so each member's iterates do not depend on the other members.  Same stopping rule,
 * acceptance and mixed-precision fallback as femd_cuda_batch_solve; results[p].seconds = the whole
 * solve.  No reference counterpart (the batched form of cg_jacobi, solver/cg.hpp:118). */
FEMD_API int femd_cuda_batch_solve_lockstep(femd_ctx ctx, femd_batch B, const double *const *b_dev, double *const *x_dev,
                                            int max_iter, double tol, int mixed, femd_cg_result *results);
/* Every armed member solved to completion by the lockstep engine (one wave: the members armed
 * now start together, members armed later wait for the next call), then disarmed and listed like
 * femd_cuda_batch_step's finished members.  No reference counterpart. */
FEMD_API int femd_cuda_batch_step_lockstep(femd_ctx ctx, femd_batch B, int mixed, int *nfinished, int *finished_ids,
                                           femd_cg_result *finished);
/* The lockstep engine, continuous: admits every member armed since the last call (members armed
 * while others are in flight join here, at a chunk boundary), runs up to `chunks` chunks of
 * iterations (the configured chunk length each) over every member in flight, finishes the members
 * that are done (the final FP64 residual, or the flush of a mixed member that broke down) and lists
 * them like femd_cuda_batch_step (disarmed); the others stay on the device for the next call.  A mixed
 * member whose FP32 recurrence stagnates goes on in FP64 from the next call (its result counts both
 * phases).  A member's iterates do not depend on when it joined or on the other members.  No
 * reference counterpart (continuous batching of cg_jacobi, cg.hpp:296-350). */
FEMD_API int femd_cuda_batch_advance_lockstep(femd_ctx ctx, femd_batch B, int mixed, int chunks, int *nfinished,
                                              int *finished_ids, femd_cg_result *finished);
/* Shape of the lockstep engine: nonzeros per row range of a member (one thread block each;
 * default 16384), iterations enqueued between two reads of the members' states (default 8), the
 * SpMV by windows of whole rows read by coalesced loads (windows = 1) or by row groups of a few
 * lanes per row (0, the default), and in mixed precision the compact layout (compact = 1, the
 * default): each member's FP32 matrix and vectors in a reverse Cuthill-McKee order of its
 * pattern with the rows of every 256 sorted by length (built once per pattern on the host, kept
 * with the pattern), the entries in slices of 32 rows stored column-major and padded to the
 * slice's longest row (one warp per slice, one lane per row), column indices as 16-bit offsets
 * from the row (6 bytes per nonzero instead of 8), and the SpMV reading the search direction
 * from a shared-memory window of each row range instead of gathering it from global memory; a
 * pattern whose reordered bandwidth exceeds 32767 or whose windows exceed 12288 columns keeps
 * the plain layout.  0 (-1 for windows and compact) keeps the current value.  No reference
 * counterpart. */
FEMD_API int femd_cuda_batch_lockstep_configure(femd_batch B, int nnz_per_entry, int chunk, int windows, int compact);
/* The last lockstep solve's layout (out: 4 entries): [0] members in the compact layout, [1] members
 * in the plain layout, [2] the widest shared-memory column window (columns), [3] table entries.
 * Instrumentation with no reference counterpart. */
FEMD_API int femd_cuda_batch_lockstep_stats(femd_batch B, long long *out);
/* Build (once per pattern) the lockstep engine's compact layout of a square pattern: the reverse
 * Cuthill-McKee order with the rows of every 256 sorted by length, the 32-row slices, 16-bit
 * column offsets, the column window of every slice.  Mixed-
 * precision members on the pattern use it; without this call it is built by the first lockstep
 * solve that meets the pattern (host work, seconds for millions of rows), so a server calls it
 * while it sets its meshes up.  *bandwidth: the reordered bandwidth, -1 when over 32,767 (the
 * pattern then keeps the plain layout).  No reference counterpart. */
FEMD_API int femd_cuda_pattern_batch_layout(femd_ctx ctx, femd_pattern p, int *bandwidth);
/* Add a member (a square matrix with its Jacobi inverse diagonal); *id_out its id (a free id is
 * reused).  Remove frees its solver vectors; a removed member's solve is dropped. */
FEMD_API int femd_cuda_batch_add(femd_batch B, femd_matrix K, int *id_out);
FEMD_API int femd_cuda_batch_remove(femd_batch B, int id);
/* Start a solve of member id on the next steps: b_dev, x_dev (initial guess in, solution out)
 * stay in use until the member finishes.  max_iter <= 0: max(1000, 10 n). */
FEMD_API int femd_cuda_batch_arm(femd_batch B, int id, const double *b_dev, double *x_dev, int max_iter, double tol);
/* One launch: every armed member advances by at most iters iterations (all in FP32-inner mixed
 * mode or all in FP64).  Members that finish are disarmed; *nfinished of them are listed in
 * finished_ids / finished (room for every armed member; either list may be NULL). */
FEMD_API int femd_cuda_batch_step(femd_ctx ctx, femd_batch B, int iters, int mixed, int *nfinished, int *finished_ids,
                                  femd_cg_result *finished);
/* Ask a running batch launch to stop (safe from another host thread): FEMD_EABORT. */
FEMD_API int femd_cuda_batch_abort(femd_batch B);
/* Members, resident blocks, team slots and each member's team size in id order (team_out:
 * one int per member). */
FEMD_API int femd_cuda_batch_info(femd_batch B, int *nprob, int *grid, int *nslots, int *team_out);
/* The launch shape: threads per block (128, 256 or 512), nonzeros per team rank (>= 256: a
 * member's team is ceil(nnz / nnz_per_block) blocks, at most half the grid and one per 64
 * rows) and nonzeros per thread of an SpMV chunk (2, 4 or 8, with block x nnz_per_thread <= 1024): a chunk of
 * whole rows holds at most block x nnz_per_thread nonzeros, i.e. it sets the rows each warp
 * sums per chunk.  A member's iterates depend on these and on the member alone.  No reference
 * counterpart.  Not while a solve is in progress. */
FEMD_API int femd_cuda_batch_configure(femd_batch B, int block, int nnz_per_block, int nnz_per_thread);
/* The current shape, and graph = 1 when launches run as a captured CUDA graph (-1: direct
 * launches, 0: no launch yet). */
FEMD_API int femd_cuda_batch_params(femd_batch B, int *block, int *nnz_per_block, int *nnz_per_thread, int *graph);
/* Autotuner: coordinate descent over nnz_per_block {8192 .. 131072}, block {128, 256, 512} and
 * nnz_per_thread {2, 4, 8}, each shape timed (CUDA events, best of two) on these systems with
 * x_dev zeroed before every run (x_dev is scratch: it holds the last run's iterate), max_iter
 * iterations (<= 0: to convergence).  Leaves the fastest shape configured; best_out = {block,
 * nnz_per_block, nnz_per_thread}, *seconds_out its time.  No reference counterpart. */
FEMD_API int femd_cuda_batch_tune(femd_ctx ctx, femd_batch B, const double *const *b_dev, double *const *x_dev, int max_iter,
                                  double tol, int mixed, int *best_out, double *seconds_out);
/* Failure-detection hook for tests: the next launches make member ghost_member (-1: none) wait
 * at its barriers for one team rank that never comes, and bound every wait by spin_limit spins
 * (<= 0: the default, a few seconds).  The launch then returns FEMD_ETIMEOUT and the context
 * stays usable.  No reference counterpart. */
FEMD_API int femd_cuda_batch_debug(femd_batch B, int ghost_member, long long spin_limit);
/* Counters of the last launch (cycles_out: 7 entries).  Cycles summed over the blocks (thread 0 of
 * each): [0] in the kernel, [1] waiting at team barriers, [2] waiting at the SpMV chunk barriers
 * -- their ratios show how much of a launch is synchronisation.  When a bounded wait gave up
 * (FEMD_ETIMEOUT): [3] which (1 a team barrier, 2 a staging copy, 3 a staging copy that had still
 * not landed when its block exited -- the launch then returns FEMD_ECUDA), [4] the barrier phase or the
 * chunk, [5] the team size, [6] the barrier count seen (team) or the staging parity bits.  No
 * reference counterpart. */
FEMD_API int femd_cuda_batch_profile(femd_batch B, long long *cycles_out);

/* The same numbering on the device (replaces the host setup of LagrangeSpace2D,
 * include/femd/fe/space_2d.hpp:390-526 -- build_edges / build_dofs / number): tris_dev is the
 * mesh's ncells x 3 vertex indices in device memory, cell_dofs_dev receives ncells x nloc dofs
 * (-1: eliminated), identical to femd_host_lagrange_numbering's.  Rejects meshes with a vertex
 * that is the smaller end of more than 512 edges (FEMD_EINVAL; the host numbering takes them).
 * Synchronises the context's stream. */
FEMD_API int femd_cuda_lagrange_numbering(femd_ctx ctx, int nverts, int ncells, const int *tris_dev, int k, int all_exterior,
                                          int *cell_dofs_dev, int *dim, int *raw_dim);

/* ======================================================================================
 * Host-side setup of the synthetic problems (the reference's own setup code runs on the
 * host too).  No GPU work.
 * ====================================================================================== */
/* rectangle_mesh(x0,y0,x1,y1,nx,ny), diagonal "right" (include/femd/mesh/structured.hpp:338-351). */
FEMD_API int femd_host_rectangle_mesh(double x0, double y0, double x1, double y1, int nx, int ny, double *points, int *tris);
/* Continuous P_k numbering with every exterior edge Dirichlet (LagrangeSpace2D(m, k, {}, true),
 * include/femd/fe/space_2d.hpp:390-526).  cell_dofs: ncells x nloc; returns dim via *dim. */
FEMD_API int femd_host_lagrange_numbering(int nverts, int ncells, const int *tris, int k, int all_exterior, int *cell_dofs,
                                 int *dim, int *raw_dim);
/* The raw numbering of the same space (no node eliminated; include/femd/fe/space_2d.hpp:448-470):
 * cell_raw ncells x nloc, *raw_dim the node count. */
FEMD_API int femd_host_lagrange_raw(int nverts, int ncells, const int *tris, int k, int *cell_raw, int *raw_dim);
/* The reference coordinates of the nloc local nodes of equispaced P_k (vertices, edge nodes, interior);
 * returns nloc. */
FEMD_API int femd_host_lagrange_nodes(int k, double *xi, double *eta);
/* The exterior facets of a rectangle mesh [x0, x1] x [y0, y1] in (cell, local edge) order with the
 * marker of their side (markers[0..3]: bottom, right, top, left; 0 elsewhere)
 * (include/femd/fe/space_2d.hpp:430-446, include/femd/mesh/structured.hpp:26-31).  cell, local,
 * marker: room for 3 ncells.  Returns the facet count. */
FEMD_API int femd_host_exterior_facets(int nverts, int ncells, const int *tris, const double *points, double x0, double y0,
                                       double x1, double y1, const int *markers, int *cell, int *local, int *marker);
/* The facet rule of Cache2D(V, degree, ..., true) (include/femd/fe/cache_2d.hpp:126-149):
 * max(1, (degree + 2) / 2) Gauss-Legendre points; xi, eta: 3 x nq, gw: nq, ref: 3 x nq x 3 x nloc.
 * Returns nq (<= 64). */
FEMD_API int femd_host_facet_rule(int k, int degree, double *xi, double *eta, double *gw, double *ref);
/* TriangleQuadrature(degree) (include/femd/quadrature/triangle.hpp:24-58): returns nq (<= 64). */
FEMD_API int femd_host_triangle_quadrature(int degree, double *xi, double *eta, double *w);
/* A reverse Cuthill-McKee order of a square CSR pattern: order[new] = old (George and Liu's
 * pseudo-peripheral start per connected component, neighbours by increasing degree, reversed) --
 * the order of the batched engine's compact layout.  No reference counterpart. */
FEMD_API int femd_host_rcm_order(int n, const int *indptr, const int *indices, int *order);
/* The lockstep engine's compact layout of a square CSR pattern, computed on the host: what
 * femd_cuda_pattern_batch_layout builds and keeps with a pattern, here for inspection and tests.
 * The reverse Cuthill-McKee order with the rows of every 256 sorted by length (iperm: original
 * row -> reordered row); the entries in slices of 32 reordered rows, column-major, each padded to
 * its longest row: entry j of reordered row k at slot rstart[k] + 32 j (rstart[n] = *nsell, the
 * slots with padding); off[slot] = the entry's reordered column minus k (0 in the padding);
 * dst[q] = the slot of entry q; tile_lo / tile_hi = per slice the smallest and largest column,
 * the slice's own rows included.  With off == NULL only *nsell and *bandwidth are set; else
 * iperm (n), rstart (n + 1), dst (nnz), off (*nsell), tile_lo and tile_hi ((n + 31) / 32) are
 * filled.  *bandwidth: the reordered bandwidth, -1 when the layout does not apply (over 32,767);
 * then nothing is filled.  No reference counterpart. */
FEMD_API int femd_host_compact_layout(int n, const int *indptr, const int *indices, long long *nsell, int *bandwidth,
                                      int *iperm, int *rstart, int *dst, short *off, int *tile_lo, int *tile_hi);
/* The equispaced P_k basis and its reference derivatives at points: out[q][3][nloc]. */
FEMD_API int femd_host_tabulate(int k, int nq, const double *xi, const double *eta, double *out);

#ifdef __cplusplus
}
#endif

#endif /* FEMD_CUDA_H */
