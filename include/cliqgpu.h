/*
 * cliqgpu.h -- C ABI of the B200 multifrontal LDL^T engine.
 *
 * Plain C types only: pointers, sizes and an opaque stream (a cudaStream_t
 * passed as void*).  Every function returns an int status (CLIQ_OK == 0).
 * Matrices are column-major; complex values are interleaved (re, im) pairs,
 * i.e. the memory layout of std::complex / numpy complex arrays.
 *
 * Clique itself has no C ABI or plugin layer: its operator interface is the
 * C++ template API in include/clique/.  Each entry point below names the
 * reference function whose behaviour it replaces (paths are relative to the
 * reference project root).  include/clique_b200/clique.hpp wraps these entry
 * points back into that C++ API (cliq::LDL, cliq::Solve, ...), converting
 * non-zero statuses into the reference's exception types.
 */
#ifndef CLIQGPU_H
#define CLIQGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define CLIQ_OK              0
#define CLIQ_ERR_ARG         1   /* invalid argument (maps to El::LogicError)      */
#define CLIQ_ERR_OOM         2   /* device or host allocation failed               */
#define CLIQ_ERR_ZERO_PIVOT  3   /* an exactly-zero D pivot was met                */
#define CLIQ_ERR_CUDA        4   /* CUDA runtime error                             */
#define CLIQ_ERR_TIMEOUT     5   /* a bounded device-side wait gave up             */
#define CLIQ_ERR_STATE       6   /* call out of order (e.g. solve before factor)   */
#define CLIQ_ERR_NOCONV      7   /* iterative refinement did not reach tolerance   */

/* ---- scalar / precision tags -------------------------------------------- */
#define CLIQ_REAL     0
#define CLIQ_COMPLEX  1
#define CLIQ_FP64     0
#define CLIQ_FP32     1

typedef struct cliq_symbolic_s* cliq_symbolic;   /* host symbolic analysis        */
typedef struct cliqgpu_plan_s*  cliqgpu_plan;    /* device-resident front tree    */

/* Plain-array view of cliq::DistSymmInfo (single process) plus the ordering.
 * Reference: include/clique/symbolic/dist_symm_info.hpp:17-36 (SymmNodeInfo). */
typedef struct {
    int32_t        num_nodes;
    const int32_t* size;            /* [num_nodes] pivots of each front (node.size)      */
    const int32_t* off;             /* [num_nodes] first ND index of each node           */
    const int32_t* parent;          /* [num_nodes] parent node, -1 for the root          */
    const int32_t* children;        /* [2*num_nodes] left, right child or -1, -1          */
    const int64_t* lower_ptr;       /* [num_nodes+1] CSR offsets into lower               */
    const int32_t* lower;           /* analysed lowerStruct (sorted ND indices)           */
    const int64_t* orig_lower_ptr;  /* [num_nodes+1] CSR offsets into orig_lower          */
    const int32_t* orig_lower;      /* origLowerStruct (sorted ND indices)                */
} cliq_symm_info;

/* ======================= host symbolic phase ============================== */

/* Natural nested dissection of an nx*ny*nz grid graph followed by the
 * symbolic analysis.  The graph is the CSR pattern of A (both triangles,
 * natural order x + y*nx + z*nx*ny).
 * Replaces cliq::NaturalNestedDissection,
 * include/clique/symbolic/natural_nested_dissection.hpp:17-26,447-488 (P=1). */
int cliq_natural_nested_dissection(int32_t nx, int32_t ny, int32_t nz, int64_t n,
                                   const int64_t* rowptr, const int32_t* colind,
                                   int32_t cutoff, cliq_symbolic* out);

/* Nested dissection of a general graph (the CSR pattern of A, both
 * triangles; structurally symmetric) followed by the symbolic analysis.
 * The tree and numbering follow the reference's sequential recursion; the
 * vertex separators come from this library's own bisection (breadth-first
 * level structures from pseudo-peripheral vertices, the balanced middle
 * level, shrunk greedily; num_seps start vertices tried) instead of METIS.
 * Disconnected graphs split between components with empty separators.
 * Replaces cliq::NestedDissection(graph, map, sepTree, info, sequential,
 * numDistSeps, numSeqSeps, cutoff), include/clique/symbolic/
 * nested_dissection.hpp:35-44,115-230 at P=1 (num_seps = numSeqSeps). */
int cliq_nested_dissection(int64_t n, const int64_t* rowptr, const int32_t* colind, int32_t cutoff,
                           int32_t num_seps, cliq_symbolic* out);

/* Views into the analysis (pointers stay valid until cliq_symbolic_destroy).
 * Replaces reading cliq::DistSymmInfo::localNodes,
 * include/clique/symbolic/dist_symm_info.hpp:108-113. */
int cliq_symbolic_info(cliq_symbolic symb, cliq_symm_info* out);

/* Per-node scalars: out[0..9] = size, off, myOff, parent, leftChild,
 * rightChild, onLeft, |lowerStruct|, |origLowerStruct|, separator-tree parent.
 * Reference: SymmNodeInfo fields (dist_symm_info.hpp:17-36) and
 * SepOrLeaf::parent (dist_separator_tree.hpp). */
int cliq_symbolic_node(cliq_symbolic symb, int32_t s, int32_t out[10]);

/* Per-node index arrays: which = 0 lowerStruct, 1 origLowerStruct,
 * 2 origLowerRelInds, 3 leftRelInds, 4 rightRelInds, 5 separator/leaf
 * natural indices (SepOrLeaf::inds).  *len receives the length; out may be
 * NULL to query it.  Reference: dist_symm_info.hpp:30-35. */
int cliq_symbolic_node_array(cliq_symbolic symb, int32_t s, int32_t which, int32_t* out, int64_t* len);

/* The reordering (natural -> ND) and its inverse.  Either pointer may be NULL.
 * Replaces cliq::BuildMap / DistMap::FormInverse at P=1,
 * include/clique/symbolic/nested_dissection.hpp:1206-1363. */
int cliq_symbolic_map(cliq_symbolic symb, int32_t* map, int32_t* inverse_map);

void cliq_symbolic_destroy(cliq_symbolic symb);

/* ======================= device numeric phase ============================= */

typedef struct {
    int32_t field;        /* CLIQ_REAL or CLIQ_COMPLEX                                  */
    int32_t precision;    /* factor precision: CLIQ_FP64 (plain) or CLIQ_FP32 (mixed)   */
    int32_t conjugate;    /* 1: Hermitian (LDL^H), 0: symmetric (LDL^T)                 */
    int32_t block_size;   /* dense panel width nb, 0 = default                           */
    int32_t keep_matrix;  /* 1: keep A in FP64 on the device for Multiply / refinement  */
} cliqgpu_options;

/* Build the device front tree: front sizes and relative indices from the
 * analysis, the assembly map from A's pattern, and all HBM buffers (factor
 * arena, update stacks, workspaces).  map is natural -> ND (length n).
 * stream: cudaStream_t to run on (cudaStreamLegacy, i.e. (void*)1, for the
 * legacy default stream), or NULL for a private non-blocking stream.
 * Replaces the structural part of cliq::DistSymmFrontTree<F>::DistSymmFrontTree
 * / Initialize, include/clique/numeric/dist_symm_front_tree/impl.hpp:24-385,
 * plus SymmetricAnalysis's relative indices (LocalSymmetricAnalysis.cpp:84-92). */
int cliqgpu_plan_create(const cliq_symm_info* info, int64_t n, const int32_t* map,
                        const int64_t* rowptr, const int32_t* colind,
                        const cliqgpu_options* options, void* stream, cliqgpu_plan* out);

/* Scatter the values of A (CSR order of the pattern given to plan_create)
 * into the fronts.  values: FP64 (real or interleaved complex, as the plan's
 * field), on the host (values_on_device = 0) or the device (= 1).
 * Replaces the value part of DistSymmFrontTree<F>::Initialize,
 * include/clique/numeric/dist_symm_front_tree/impl.hpp:244-297. */
int cliqgpu_assemble(cliqgpu_plan plan, const void* values, int32_t values_on_device);

/* Multifrontal LDL^T (or LDL^H) of the assembled fronts, in place.
 * *zero_pivot receives -1, or the ND index of the first exactly-zero pivot
 * (the factorization still completes; the status is then CLIQ_ERR_ZERO_PIVOT).
 * Replaces cliq::LDL(info, L, LDL_1D/LDL_2D), include/clique/numeric/ldl.hpp:57-75
 * (LocalLDL ldl/local.hpp:25-122, FrontLDL ldl/local_front.hpp:30-71). */
int cliqgpu_factor(cliqgpu_plan plan, int64_t* zero_pivot);

/* The same factorization with intra-front Bunch-Kaufman pivoting: each
 * front's pivot block is factored as P A11 P^T = L D op(L)^T with P a
 * permutation of the front's own pivot rows and D block diagonal (1 x 1 and
 * 2 x 2 blocks), the columns of A21 permuted with it, and the Schur
 * complement passed up as in cliqgpu_factor.  The solves apply P around each
 * front and solve with the 2 x 2 blocks; their inputs and outputs keep the
 * natural / ND order.  *zero_pivot: -1, or the smallest ND index of a pivot
 * row whose whole remaining column within its front's pivot rows is zero
 * (then CLIQ_ERR_ZERO_PIVOT).
 * Replaces cliq::LDL(info, L, LDL_INTRAPIV_1D/LDL_INTRAPIV_2D): LocalLDL's
 * intraPiv branch, include/clique/numeric/ldl/local.hpp:31-33,106-111,
 * FrontLDLIntraPiv ldl/local_front.hpp:74-94, and its solves
 * lower_solve/local_front.hpp:53-93 and diagonal_solve.hpp:53-59. */
int cliqgpu_factor_intrapiv(cliqgpu_plan plan, int64_t* zero_pivot);

/* Pivots of front s after cliqgpu_factor_intrapiv: sub[k] = D(k+1, k) of the
 * 2 x 2 block starting at pivot k, 0 elsewhere (n entries, FP64, complex
 * interleaved; D(k, k+1) = sub[k], conjugated for LDL^H), and piv[i] = the
 * front's assembled pivot row at pivoted position i (n entries), so that
 * cliqgpu_get_front's L and D factor the pivot block with rows and columns
 * ordered by piv.  Unpivoted factorizations give zeros and the identity.
 * Replaces reading L.localFronts[s].subdiag / .piv
 * (dist_symm_front_tree/decl.hpp:174-184). */
int cliqgpu_get_front_pivots(cliqgpu_plan plan, int32_t s, double* sub, int32_t* piv);

/* After cliqgpu_factor: turn every front into the block-LDL form -- the top
 * n x n block holds inv(A11) (full, symmetric or Hermitian), the rows below
 * it the original A21 -- so that the solves are products only (no
 * triangular or diagonal solves).  cliqgpu_solve, cliqgpu_refined_solve and
 * cliqgpu_get_front then use / return that form until the next
 * cliqgpu_factor.  Runs on the plan's stream and returns when done.
 * After cliqgpu_factor_intrapiv the same form is built from the pivoted
 * factors, in each front's pivoted order: inv(P A11 P^T) and A21 P^T, with
 * P from cliqgpu_get_front_pivots.
 * Replaces the blockLDL branch of LocalLDL, include/clique/numeric/ldl/
 * local.hpp:30-33 with FrontBlockLDL (ldl/local_front_block.hpp:27-71, both
 * branches), i.e. cliq::LDL(info, L, BLOCK_LDL_1D/BLOCK_LDL_2D) and
 * (after cliqgpu_factor_intrapiv) BLOCK_LDL_INTRAPIV_1D/2D, and its solves
 * lower_solve/local_front_block.hpp:29-70, solve.hpp:48-53. */
int cliqgpu_block_ldl(cliqgpu_plan plan);

/* Solve A X = B in place using the stored factors: forward sweep, diagonal
 * solve, backward sweep.  X is n x nrhs column-major with leading dimension
 * ldx, FP64 (real or interleaved complex), on the host or the device.
 * nodal = 0: X is in natural order (Pull, Solve, Push); nodal = 1: X is
 * already in ND order (a DistNodalMultiVec).
 * Replaces cliq::Solve(info, L, X), include/clique/numeric/solve.hpp:41-65, with
 * DistNodalMultiVec::Pull/Push (dist_nodal_multi_vec/impl.hpp:67-219). */
int cliqgpu_solve(cliqgpu_plan plan, void* X, int64_t ldx, int32_t nrhs,
                  int32_t x_on_device, int32_t nodal);

/* Y := alpha A X + beta Y with the FP64 copy of A (requires keep_matrix),
 * natural order, X/Y n x nrhs with leading dimension ld, on the device.
 * alpha, beta point to one FP64 scalar (real) or an interleaved pair (complex).
 * Replaces cliq::Multiply, include/clique/numeric/multiply.hpp:18-21,28-166. */
int cliqgpu_multiply(cliqgpu_plan plan, const double* alpha, const void* X, const double* beta,
                     void* Y, int64_t ld, int32_t nrhs);

/* The same product for a CSR matrix held by no plan: the free function
 * cliq::Multiply(alpha, A, X, beta, Y), include/clique/numeric/multiply.hpp:18-21,28-166.
 * rowptr [n+1], colind, values (FP64, real or interleaved complex as field),
 * X, Y: n x nrhs, leading dimension ld; all on the device (on_device = 1) or
 * all on the host (on_device = 0: staged through stream-ordered device
 * buffers, the call returns when Y is back on the host). */
int cliqgpu_sparse_multiply(int32_t field, int64_t n, const int64_t* rowptr, const int32_t* colind,
                            const double* values, const double* alpha, const void* X, const double* beta,
                            void* Y, int64_t ld, int32_t nrhs, int32_t on_device, void* stream);

/* Natural -> ND (pull: Xn[p, j] = X[inverse_map[p], j]) and ND -> natural
 * (push: X[inverse_map[p], j] = Xn[p, j]) reordering of FP64 device
 * multivectors (n x nrhs, real or interleaved complex as field) through a
 * device copy of the inverse map (ND index -> natural index), on stream.
 * Replace cliq::DistNodalMultiVec<F>::Pull / Push at P=1,
 * include/clique/numeric/dist_nodal_multi_vec/impl.hpp:67-219,221-... */
int cliqgpu_nodal_pull(int32_t field, int64_t n, const int32_t* inverse_map, const void* X, int64_t ldx,
                       void* Xn, int64_t ldn, int32_t nrhs, void* stream);
int cliqgpu_nodal_push(int32_t field, int64_t n, const int32_t* inverse_map, const void* Xn, int64_t ldn,
                       void* X, int64_t ldx, int32_t nrhs, void* stream);

/* Mixed-precision solve: X := A^{-1} B by iterative refinement with the
 * stored factors (any precision), FP64 residuals r = B - A X and FP64
 * updates, until max_j ||r_j|| / ||b_j|| <= tol or max_iter refinement steps.
 * B, X: n x nrhs, natural order, leading dimension ld, host or device.
 * *iters receives the refinement steps taken, *relres the final max relative
 * residual.  Returns CLIQ_ERR_NOCONV if tol was not reached.
 * No reference counterpart (Clique has no refinement); it composes cliq::Solve
 * and cliq::Multiply as the examples' residual check does
 * (examples/HelmholtzPML3D.cpp:354-365). */
int cliqgpu_refine(cliqgpu_plan plan, const void* B, void* X, int64_t ld, int32_t nrhs,
                   int32_t on_device, double tol, int32_t max_iter, int32_t* iters, double* relres);

/* Gradient of X = A^{-1} B with respect to the stored entries of A, given the
 * adjoint solution Xbar = A^{-H} (dL/dX) (A^{-T} for real data): for every
 * entry e = (i, j) of A's pattern (the CSR given to plan_create, which must
 * have been created with keep_matrix = 1),
 *     out[e] = - sum_k Xbar[i, k] * op(X[j, k]),   op = conj if conj_x else identity,
 * i.e. dL/dA = -Xbar X^H restricted to the pattern.  Xbar, X: n x nrhs, natural
 * order, leading dimension ld, FP64 (interleaved complex as the plan's field),
 * on the device; out: nnz entries on the device.  The adjoint solve itself is
 * cliqgpu_solve / cliqgpu_refine with the stored factors (A = A^T for the
 * complex-symmetric and real cases, A = A^H for the Hermitian case).
 * No reference counterpart (Clique has no differentiation); used by the
 * torch.autograd.Function in clique_b200/autograd.py. */
int cliqgpu_grad_A_pattern(cliqgpu_plan plan, const void* Xbar, const void* X, int64_t ld, int32_t nrhs,
                           int32_t conj_x, void* out);

/* ======================= many problems, tuning ============================ */

/* Forest of independent grid problems: natural nested dissection of each
 * diagonal block of a block-diagonal matrix (problem p: an nx*ny*nz grid,
 * dims[3p..3p+2], rows rowoff_p .. rowoff_p + n_p - 1 in order, no entries
 * outside its block) and the symbolic analysis of all of them as one forest,
 * problem by problem in post-order.  The result feeds cliqgpu_plan_create like
 * a single analysis: every factor and solve launch then covers the fronts of
 * all problems at one tree depth.  No reference counterpart (Clique analyses
 * one matrix, natural_nested_dissection.hpp:17-26,447-488 per problem). */
int cliq_batch_nested_dissection(int32_t count, const int32_t* dims, int64_t n, const int64_t* rowptr,
                                 const int32_t* colind, int32_t cutoff, cliq_symbolic* out);

/* One run over a batch plan (created from cliq_batch_nested_dissection, with
 * keep_matrix = 1): assemble A from values (device, FP64), factor, then
 * `steps` classical refinement steps x += A_f^{-1} r, r = b - A x (FP64) for
 * B (device, n x nrhs, ld), writing X (device).  Problem s owns rows
 * seg_rows[s] .. seg_rows[s+1]-1 (host array of nseg + 1 offsets, 0 .. n);
 * relres (host, may be NULL) receives ||r_s,j|| / ||b_s,j|| for every
 * (problem s, column j) at relres[j * nseg + s] (0 for a zero column).
 * The first call launches the sequence directly, the second call with the
 * same arguments records it as one CUDA graph and replays it, later calls
 * replay it (CLIQGPU_BATCH_GRAPH=0, or a plan on the legacy default stream,
 * which cannot be captured: direct launches only).  Problems still
 * above tol get up to max_extra further steps; *steps_taken receives the
 * steps done.  Returns CLIQ_ERR_NOCONV if a problem stays above tol.
 * No reference counterpart. */
int cliqgpu_batch_run(cliqgpu_plan plan, int32_t nseg, const int64_t* seg_rows, const void* values, const void* B,
                      void* X, int64_t ld, int32_t nrhs, int32_t steps, double tol, int32_t max_extra,
                      double* relres, int32_t* steps_taken);

/* Autotuner: times the factorization with every update launch on the tensor
 * cores and with every one on the CUDA cores (best of reps, CUDA events around
 * each launch), keeps the faster kernel per launch, and records the choice in
 * a process-wide table keyed by size bucket (field, precision, update kind,
 * log2 of the largest M, N, K and of the problem count) that later plans
 * apply when they are built.  Needs assembled fronts and keep_matrix = 1; the
 * plan is left factored.  report (may be NULL) receives 5 values: GEMM ms on
 * the tensor cores, on the CUDA cores, with the choices made, launches moved
 * to the CUDA cores, launches that could move.  No reference counterpart. */
int cliqgpu_autotune(cliqgpu_plan plan, int32_t reps, double* report);

/* Copy front s back to the host: L (m x n, column-major, in the plan's
 * storage precision widened to FP64) and D (n entries, FP64).
 * Either pointer may be NULL.  dims[0..1] receives m, n.  After
 * cliqgpu_factor_intrapiv the pivot rows of L are in the front's pivoted
 * order and D is the diagonal of the block-diagonal D; the order and the
 * 2 x 2 blocks' off-diagonals come from cliqgpu_get_front_pivots.
 * Replaces reading L.localFronts[s].frontL / .diag
 * (dist_symm_front_tree/decl.hpp:174-184). */
int cliqgpu_get_front(cliqgpu_plan plan, int32_t s, double* L, double* D, int32_t dims[2]);

/* Scalar properties: key 0 factor flops (Clique's FactorizationWork formula),
 * 1 solve flops per right-hand side (SolveWork), 2 factor entries (sum m*n),
 * 3 device bytes held, 4 kernel launches issued by the last call,
 * 5 number of fronts, 6 tree depth, 7 bytes of the factor arena,
 * 8 kernels launched by this plan since creation (all calls).
 * Reference for 0-2: dist_symm_front_tree/impl.hpp:401-640. */
int cliqgpu_plan_query(cliqgpu_plan plan, int32_t key, double* value);

/* Per-kernel timing of the factorization with CUDA events recorded around
 * every launch of cliqgpu_factor on the plan's stream (enable = 1 / 0).
 * cliqgpu_profile_read waits for the stream and fills out[0..nout-1]:
 * 0 extend-add ms, 1 diagonal-block ms, 2 panel ms, 3 in-panel update ms,
 * 4 Schur update ms, 5 in-panel update flops, 6 Schur update flops (Clique's
 * counting: 2 per real multiply-add, x4 complex), 7 extend-add bytes moved,
 * 8 in-panel update launches, 9 Schur launches, 10 factor ms (first to last
 * launch).  No reference counterpart: the reference times phases with
 * mpi::Time (tests/Solve.cpp:224-251). */
int cliqgpu_set_profiling(cliqgpu_plan plan, int32_t enable);
int cliqgpu_profile_read(cliqgpu_plan plan, double* out, int32_t nout);

/* Wait for all work queued on the plan's stream. */
int cliqgpu_synchronize(cliqgpu_plan plan);

/* Failure-detection check (no counterpart in the reference): one CTA waits,
 * through the same bounded wait as the solve sweeps, on a flag that nothing
 * sets.  The wait gives up after limit_ns (0 < limit_ns <= 2e9) and the call
 * returns CLIQ_ERR_TIMEOUT with the wait site in cliqgpu_last_error(); the
 * plan's status word is cleared afterwards, so the plan and the CUDA context
 * stay usable. */
int cliqgpu_wait_selftest(cliqgpu_plan plan, int64_t limit_ns);

void cliqgpu_plan_destroy(cliqgpu_plan plan);

/* Human-readable text for a status code, and the last error detail. */
const char* cliqgpu_status_string(int32_t status);
const char* cliqgpu_last_error(void);

/* ======================= single dense front =============================== */

/* Dense partial LDL^T of one front, in place on device memory:
 * AL (m x n, ld lda) receives unit-lower L with D on its diagonal ... as
 * FrontLDL leaves it before LocalLDL stores D separately, and ABR
 * ((m-n) x (m-n) lower, ld ldabr) receives ABR - L_B D L_B^T.
 * field / precision as in cliqgpu_options; data in that precision.
 * Workspace is allocated with cudaMalloc and freed before return.
 * Replaces cliq::FrontLDL(AL, ABR, conjugate),
 * include/clique/numeric/ldl/local_front.hpp:17-18,30-71. */
int cliqgpu_front_ldl(int32_t field, int32_t precision, int32_t conjugate, int32_t m, int32_t n,
                      void* AL, int64_t lda, void* ABR, int64_t ldabr, void* stream);

/* The same dense partial LDL^T of one front for callers that must not
 * allocate device memory during the call -- for example an application that
 * manages its own memory pool and bans cudaMalloc/cudaFree inside its solve
 * phase (cudaFree synchronises the whole device), or code running under
 * another library's allocation lock.  All scratch lives in one fixed device
 * array inside the library (about 1.2 MB, held on every GPU that loads the
 * library until exit); nothing is allocated or freed.  Limits: n <= 1024,
 * m <= 16384, lda == m, m - n <= ldabr <= INT_MAX; other sizes return
 * CLIQ_ERR_ARG.  The first call on a device looks up the array's address
 * (make it before any stream capture).  Every call waits for its stream and
 * reads a status word back before it returns; a zero pivot returns
 * CLIQ_ERR_ZERO_PIVOT with its column in cliqgpu_last_error().  Calls share
 * the array, so calls that overlap on the GPU race; serialise them.  Uses
 * the CUDA-core update kernel in every precision.
 * No counterpart in the reference (Clique allocates freely in FrontLDL). */
int cliqgpu_front_ldl_noalloc(int32_t field, int32_t precision, int32_t conjugate, int32_t m, int32_t n,
                              void* AL, int64_t lda, void* ABR, int64_t ldabr, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CLIQGPU_H */
