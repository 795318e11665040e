// Internal declarations of the cliqgpu library (not part of the C ABI).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cliqgpu.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#else
struct CUstream_st;
typedef struct CUstream_st* cudaStream_t;
struct CUgraphExec_st;
typedef struct CUgraphExec_st* cudaGraphExec_t;
#endif

namespace cliqgpu {

// ---------------------------------------------------------------------------
// host symbolic analysis (single process)
// ---------------------------------------------------------------------------
struct Symbolic {
    int num_nodes = 0;
    int64_t n = 0;
    std::vector<int> size, off, my_off, parent, sep_parent, children, on_left;
    std::vector<std::vector<int>> lower, orig_lower, orig_rel, left_rel, right_rel, inds;
    std::vector<int> map, inv_map;
    // flattened CSR views for cliq_symm_info
    std::vector<int64_t> lower_ptr, orig_ptr;
    std::vector<int> lower_flat, orig_flat;
    void finalize_views();
};

int natural_nested_dissection(int nx, int ny, int nz, int64_t n, const int64_t* rowptr, const int32_t* colind,
                              int cutoff, Symbolic& S);

int graph_nested_dissection(int64_t n, const int64_t* rowptr, const int32_t* colind, int cutoff, int num_seps, Symbolic& S);
int batch_nested_dissection(int count, const int32_t* dims, int64_t n, const int64_t* rowptr, const int32_t* colind,
                            int cutoff, Symbolic& S);

void set_last_error(const std::string& msg);

// ---------------------------------------------------------------------------
// device-side descriptors
// ---------------------------------------------------------------------------
constexpr int kTile = 64;        // rows per solve block, GEMM tile edge
constexpr int kTcBM = 128;       // tensor-core update tile: rows
constexpr int kTcBN = 128;       // tensor-core update tile: columns (two CTAs per SM at 128)
constexpr int kEACols = 16;      // columns per extend-add work item
constexpr int kEARows = 2048;    // rows per extend-add work item
// Triangular sweeps: the worker of pivot block s adds the contributions of
// the solved blocks up to s - kSolveLag and applies the block's inverse; the
// chain CTA of the front adds the newest block (s - 1) through the stored
// product of that inverse with the coupling tile.
constexpr int kSolveLag = 2;
constexpr int kSolveRhsChunk = 16;   // right-hand sides per sweep (partial-sum stride)
constexpr int kLowerChunkTiles = 16; // backward: 64-row tiles below the pivots per helper
// sweep work items {front, kind, block, chunk}
enum SweepItem : int { kItemChain = 0, kItemPivotRows = 1, kItemLowerRows = 2, kItemColumns = 1, kItemLowerChunk = 2,
                       kItemWhole = 3 };
// fronts solved by one CTA per sweep (no flags): at most two pivot blocks
// and kWholeLowerRows rows below the pivots
constexpr int kWholeLowerRows = 512;
// fronts of one pivot block and at most kTinyLowerRows rows below it are swept
// by one warp each, several fronts per CTA
constexpr int kTinyLowerRows = 64;

// One front as the kernels see it.  Offsets are in elements (a complex
// element is two scalars).
struct FrontDev {
    int64_t L;          // frontL (m x n, ld m) in the factor arena
    int64_t U;          // update ABR (u x u, ld u) in pool[pool]
    int64_t CU[2];      // children's updates in the other pool (-1: none)
    int64_t cmap;       // child maps: [m] left then [m] right (int32, -1 = absent), -1 for leaves
    int64_t lower;      // offset of lowerStruct in the flattened array
    int64_t W;          // solve workspace offset (multiply by nrhs) in wpool[pool]
    int64_t CW[2];      // children's solve workspace offsets (in the other wpool)
    int32_t m, n, off, u;
    int32_t cu[2];      // children's update sizes
    int32_t pool;       // parity of the depth
    int32_t flag_base;  // first pivot-block slot of this front (worker flag, worker result)
    int64_t dinv;       // inverse diagonal blocks (ceil(n/64) blocks of 64 x 64) in the dinv store
    int64_t chain;      // chain tiles (ceil(n/64) blocks of 64 x 64) in the m1 / n1 stores; -1: the front has
                        // none (solved by one CTA, or the sweeps use the substitution form)
    int32_t hbase;      // backward sweep: first helper slot ((nch - 1) per pivot block)
    int32_t nch;        // backward sweep: 16-tile chunks of the rows below the pivots
    int64_t eblk;       // 2xFP16 split: per (row, 64-column block) largest |component| of L and of D op(L), m x nT
    int64_t erow;       // 2xFP16 split: per row, the same over all blocks so far (m)
};

// One GEMM update problem: C -= A diag(d) op(B)^T restricted to i >= j.
struct GemmProb {
    int64_t A, B, C, d;   // A, B in the arena; C in the arena (cpool < 0) or a pool; d in the D array
    int32_t lda, ldc, M, N, K, cpool;
    int64_t packA, packB; // tensor-core path: float offsets of the packed operands in the pack buffer
    int64_t scaleA, scaleB;   // FP16 split: float offsets of the per-row inverse scales (A rows, S rows)
    int32_t front, row0, kb0, nkb;   // operand rows start at front row row0; K covers 64-blocks kb0 .. kb0+nkb-1 (0: all)
};

// One operand panel to pack for the tensor cores: R rows x K columns of the
// arena at src (leading dimension ld), scaled by d[k] when d >= 0, written
// as (row tile, k step) blocks of tile_rows rows at float offset dst.
struct PackJob {
    int64_t src, dst, d;
    int32_t R, K, ld, tile_rows;
    int64_t dst_scale;    // FP16 split: float offset of the R (padded to tiles) inverse row scales
    int64_t emax;         // FP16 split: row maxima of the job's first row (block kb0), in the eblk / erow arrays
    int32_t enT, nkb;     // row stride of eblk (blocks per row); blocks in K (0: use erow)
    // FP16 split: the same job also writes S = D[dS + k] op(rows) for its
    // first RS rows (the B operand, a prefix of the A rows) at dstS with
    // inverse row scales at dst_scaleS, row maxima at emaxS (RS = 0: A only)
    int64_t dstS, dst_scaleS, emaxS, dS;
    int32_t RS;
};

struct Launch {
    enum Kind { EXTEND_ADD, DIAG, PANEL, GEMM } kind;
    int64_t items;        // offset into the int2 item array (EXTEND_ADD / DIAG / PANEL) or prob array (GEMM)
    int32_t nitems;
    int64_t prefix;       // GEMM: offset into the tile prefix array
    int64_t nblocks;      // grid size
    int32_t k;            // DIAG / PANEL: column offset of the step
    int32_t depth;
    double work;          // GEMM: algorithmic flops; EXTEND_ADD: algorithmic bytes
    int32_t schur;        // GEMM: 1 for the Schur-complement update, 0 for an in-panel update
    int32_t simt = 0;     // GEMM: CUDA-core kernel (64 x 64 tiles) even on the tensor path
    // GEMM: 1 = lookahead part of an outer-block update (columns two outer
    // blocks and more to the right), run on stream2, k = the outer block;
    // 2 = one K chunk of the Schur-complement update, run on stream3
    int32_t bulk = 0;
    // GEMM: operands written by the preceding tensor-core panel (no packing);
    // PANEL: offset of that GEMM's problems in the problem array (-1: none),
    // the panel item's w field is the front's problem index there (-1: none)
    int32_t prepacked = 0;
    int64_t pk_probs = -1;
    // tensor-core path: operand packing for this GEMM
    int64_t pack_items = 0, pack_prefix = 0, pack_blocks = 0;
    // offsets into the block map: the job of every pack block, the problem of
    // every GEMM tile (one load instead of a binary search over the prefix)
    int64_t pack_map = 0, gemm_map = 0;
    int32_t pack_njobs = 0;
    // GEMM: the launch may run either on the tensor cores (tcgen05 on the
    // FP32 path, DMMA on the FP64 path) or on the CUDA cores; simt selects
    // the CUDA-core kernel.  The FP32 tensor-core tiling is 128 x 128, so
    // those launches also carry the 64 x 64 tiling of the CUDA-core kernel
    // (alt_*); FP64 launches use 64 x 64 tiles for both kernels.
    int32_t switchable = 0;
    int64_t alt_prefix = -1, alt_gemm_map = 0, alt_nblocks = 0;
    // largest M, N, K over the launch's problems and their number (the
    // autotuner's size bucket)
    int32_t maxM = 0, maxN = 0, maxK = 0;
};

// per-kernel-kind device time of the last profiled factorization (ms) and
// work; on the tensor path trail / schur time is the GEMM alone and the
// operand packing is PROF_PACK_MS
enum ProfSlot {
    PROF_EA_MS = 0, PROF_DIAG_MS, PROF_PANEL_MS, PROF_TRAIL_MS, PROF_SCHUR_MS,
    PROF_TRAIL_FLOPS, PROF_SCHUR_FLOPS, PROF_EA_BYTES, PROF_TRAIL_LAUNCHES, PROF_SCHUR_LAUNCHES,
    PROF_FACTOR_MS, PROF_PACK_MS, PROF_SLOTS = 16
};

struct SolveLevel {
    int64_t fronts;       // offset into level_fronts (int32 front ids)
    int32_t nfronts;
    int64_t fwd_items;    // offset into chain item array (int2: front, block)
    int32_t nfwd;
    int64_t bwd_items;
    int32_t nbwd;
    int32_t depth;
    int32_t gather_chunks;   // 1024-row chunks of the level's tallest front (gather grid y)
    int64_t tiny;            // offset into tiny_fronts: the level's fronts swept one per warp
    int32_t ntiny;
};

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
struct Plan {
    // options
    int field = CLIQ_REAL, precision = CLIQ_FP64, conjugate = 0, nb = 64, keep_matrix = 0;
    bool cplx() const { return field == CLIQ_COMPLEX; }
    int scalar_bytes() const { return precision == CLIQ_FP64 ? 8 : 4; }
    int elem_bytes() const { return scalar_bytes() * (cplx() ? 2 : 1); }

    int64_t n = 0, nnz = 0;
    int num_fronts = 0, max_depth = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // host copies of structure
    std::vector<FrontDev> hfronts;
    std::vector<int> depth;
    std::vector<std::vector<int>> level_list;   // fronts per depth
    std::vector<Launch> launches;
    std::vector<SolveLevel> solve_levels;       // indexed by depth
    double factor_flops = 0, solve_flops = 0, factor_entries = 0;
    int64_t arena_elems = 0, pool_elems[2] = {0, 0}, wpool_elems[2] = {0, 0}, tinv_slots = 0;
    int64_t flags_total = 0;

    // device buffers
    void* L = nullptr;            // factor arena (storage precision)
    double* D = nullptr;          // pivots, FP64 (complex: interleaved), length n
    void* pool[2] = {nullptr, nullptr};
    void* tinv = nullptr;         // U = op(L11^{-1})^T of each front of one panel step (storage precision)
    void* dinv = nullptr;         // L11^{-1} of every 64-block of every front, kept for the solves
    void* dinvT = nullptr;        // the same blocks row-major (backward sweep)
    // chain tiles (64 x 64, column-major, at the front's dinv offset + 64*64*b):
    //   m1 block b >= 1: L_bb^{-1} L_{b,b-1} (forward chain)
    //   n1 block b <= nT-2: op(L_bb^{-1})^T op(L_{b+1,b})^T (backward chain)
    void* m1 = nullptr;
    void* n1 = nullptr;
    int32_t* chain_items = nullptr;   // int4 {front, block b >= 1, 0, 0} of every chain front
    int32_t nchain_items = 0;
    int64_t chain_elems = 0;          // elements of m1 / n1 (chain fronts only)
    unsigned long long* xprog = nullptr;   // per front: (epoch << 32) | blocks its chain has published
    void* hpart = nullptr;        // backward helpers' partial sums (kSolveRhsChunk x 64 per helper)
    int64_t helpers_total = 0;
    void* partial = nullptr;      // per pivot block: 64 x kSolveRhsChunk partial sums from the sweep workers
    // 2xFP16 split: row maxima (float bits) of L panels and of D op(L) panels,
    // [A | S] halves of eblk_total and erow_total entries
    uint32_t* eblk = nullptr;
    uint32_t* erow = nullptr;
    int64_t eblk_total = 0, erow_total = 0;
    bool f16_scales() const { return tensor_path() && split_f16; }
    int64_t dinv_elems = 0;
    FrontDev* fronts = nullptr;
    int32_t* cmaps = nullptr;
    int32_t* lower = nullptr;     // flattened lowerStruct (ND indices)
    int32_t* items = nullptr;     // int2 items for extend-add / diag / panel / chain solves
    GemmProb* probs = nullptr;
    PackJob* packjobs = nullptr;
    void* pack = nullptr;         // packed tensor-core operands of one GEMM launch
    void* pack2 = nullptr;        // the same for the lookahead launches (second stream)
    int64_t pack_floats = 0;
    // lookahead (CLIQGPU_LOOKAHEAD=0: off): the outer-block updates of the
    // columns two outer blocks and more to the right run on stream2 while
    // the next outer block is factored on stream
    int lookahead = 1;
    cudaStream_t stream1 = nullptr;   // internal, highest priority: the factorization's critical path
    cudaStream_t stream2 = nullptr;   // internal, lowest priority: lookahead updates
    cudaStream_t stream3 = nullptr;   // internal, lowest priority: Schur-complement chunks
    void* pack3 = nullptr;            // packed operands of the Schur chunks
    // CLIQGPU_SCHUR_CHUNK=c > 0: the Schur complement is applied in chunks of
    // c pivot columns on stream3 as soon as their panels are final (per-chunk
    // row scales); needs the lookahead streams.  0 (default): one update with
    // K = n at the end of the level (at 100^3 the chunks overlap the next
    // panels but cost as much in extra update traffic: 128.9 vs 128.7 ms)
    int schur_chunk = 0;
    std::vector<cudaEvent_t> sync_events;   // fork / lookahead-done events, one pair per lookahead launch
    // CLIQGPU_GRAPH=1: the factorization's launches replayed as one CUDA
    // graph from the second unprofiled factorization on (off by default: at
    // 100^3 the replay ran 3 ms slower than the direct launches on the two
    // prioritized streams)
    int use_graph = 0;
    int64_t factor_runs = 0;
    cudaGraphExec_t factor_exec = nullptr;
    int64_t graph_launches = 0;
    int64_t* prefix = nullptr;
    int32_t* bmap = nullptr;      // block -> job / problem index of every pack and GEMM launch
    int64_t* dest = nullptr;      // assembly destination per CSR entry (-1: upper, skipped)
    // assembly inside the factorization: the kept entries grouped by the tree
    // depth of their front (CSR entry, destination), level d at
    // [asm_level[d], asm_level[d + 1]); added to the fronts right after the
    // level's extend-add, which writes every lower entry of those fronts
    int64_t* asm_src = nullptr;
    int64_t* asm_dst = nullptr;
    std::vector<int64_t> asm_level;
    int32_t* perm = nullptr;      // inverse map: ND -> natural
    int32_t* level_fronts = nullptr;
    int32_t* tiny_fronts = nullptr;   // per level, fronts swept one per warp (SolveLevel::tiny)
    int32_t* flags = nullptr;     // worker flags (flags_total, one per pivot block), then helper flags
    int32_t* tickets = nullptr;
    int32_t* status = nullptr;    // [0] first zero pivot + 1 (min), [1] timeout flag
    int64_t* rowptr = nullptr;    // FP64 matrix (keep_matrix)
    int32_t* colind = nullptr;
    double* aval = nullptr;
    // solve workspaces (grown on demand)
    void* wpool[2] = {nullptr, nullptr};
    void* xnodal = nullptr;       // n x nrhs in storage precision
    double* xwork = nullptr;      // FP64 workspaces for refinement (3 * n * nrhs)
    double* norms = nullptr;      // 2 * nrhs norms + partial sums
    double* krylov = nullptr;     // Krylov refinement: basis V, preconditioned Z, dots scratch
    int64_t krylov_doubles = 0;
    int refine_gmres = 1;         // FGMRES refinement (default) or classical (CLIQGPU_REFINE=ir)
    int32_t ws_nrhs = 0;
    int64_t device_bytes = 0;

    int32_t epoch = 0;
    bool assembled = false, factored = false;
    bool block = false;           // fronts hold the block-LDL form (inv(A11), A21)
    void* block_state = nullptr;  // block sweeps: schedules per right-hand-side count and scratch
    // intra-front pivoting (cliqgpu_factor_intrapiv; LDL_INTRAPIV_*): Bunch-
    // Kaufman pivots within each front's pivot rows
    bool pivoted = false;         // the current factorization is the pivoted one
    double* E = nullptr;          // like D: D(k + 1, k) of each 2 x 2 pivot block starting at k, 0 elsewhere
    int32_t* pivg = nullptr;      // ND index of the assembled row at pivoted position q
    int32_t* qpos = nullptr;      // inverse of pivg
    int32_t* perm_piv = nullptr;  // natural index of pivoted position q: perm[pivg[q]]
    int32_t* cmaps_orig = nullptr;   // child maps and lowerStruct in assembled order (the extend-add's);
    int32_t* lower_orig = nullptr;   // cmaps / lower hold the solves' pivoted order after a pivoted factorization
    int64_t cmaps_len = 0, lower_len = 0;
    bool maps_pivoted = false;
    int32_t* pstate = nullptr;    // per front: first and one-past-last column of its latest panel
    void* pvec = nullptr;         // 2 n entries: a panel step's candidate columns
    int32_t* pivot_items = nullptr;   // int4 {front, 64-block, 0, 0} of every front's pivot blocks
    int32_t pivot_dinv_items = 0;
    int64_t last_launches = 0;
    int64_t total_launches = 0;   // every kernel this plan has launched
    // FP32 updates on the tensor cores (tcgen05 3xTF32); CLIQGPU_TENSOR_CORES=0 selects the CUDA-core kernel
    int use_tc = 1;
    // triangular sweeps: substitution form of the chain steps (default for
    // FP64 storage) or the product form through the stored chain tiles M, N
    // (default for FP32 storage); CLIQGPU_SOLVE_FORM=exact|tiles overrides
    int solve_exact = 0;
    // FP64 storage: updates on the FP64 tensor cores (DMMA, default) or on the
    // CUDA cores (CLIQGPU_FP64_DMMA=0)
    int fp64_dmma = 1;
    // FP32 storage: diagonal-block LDL in FP64 arithmetic (CLIQGPU_DIAG_FP64=1) instead of FP32
    int diag_fp64 = 0;
    bool tensor_path() const { return use_tc && precision == CLIQ_FP32; }
    // operand split on the tensor path: 2 x FP16 with per-row power-of-two
    // scales (default) or 3 x TF32 (CLIQGPU_SPLIT=tf32)
    int split_f16 = 1;
    // in-panel updates (K = 64) on the tensor cores (default) or on the CUDA
    // cores without operand packing (CLIQGPU_INPANEL_TC=0)
    int inpanel_tc = 1;
    // width of the outer column block whose trailing update is deferred (multiple of nb)
    int outer_nb = 256;
    // optional per-launch CUDA-event timing of the factorization
    int profile = 0;
    bool prof_pending = false;
    std::vector<cudaEvent_t> events;
    double prof[PROF_SLOTS] = {0};

    // host-side staging for host-resident inputs/outputs
    std::vector<int32_t> hitems;

    // batch runs (cliqgpu_batch_run): row segments of the independent
    // problems, their residual norms, and the captured run
    int64_t* seg = nullptr;           // device, nseg + 1 natural-row offsets
    std::vector<int64_t> hseg;
    double* segnorm = nullptr;        // device: nseg * nrhs squared norms of r, then of b
    double* hsegnorm = nullptr;       // pinned host copy
    int64_t segnorm_cap = 0;          // doubles
    cudaGraphExec_t batch_exec = nullptr;
    std::vector<int64_t> batch_key;   // arguments the captured run was recorded with
    int64_t batch_runs = 0, batch_graph_launches = 0;
    int batch_graph = 1;              // CLIQGPU_BATCH_GRAPH=0: direct launches only
    int nseg_run() const { return (int)hseg.size() - 1; }
};

// launchers (factor_kernels.cu)
template <class T, bool C>
int run_factor(Plan& P);
// launchers (solve_kernels.cu)
template <class T, bool C>
int run_solve_nodal(Plan& P, void* xn, int nrhs);   // xn: n x nrhs in storage precision, ND order
// misc (misc_kernels.cu)
// A's values (FP64, device, CSR order) into the plan's copy P.aval; the
// fronts receive them during the factorization (level by level)
int launch_assemble(Plan& P, const double* dvals);
// the fronts as Initialize leaves them (arena cleared, every kept entry
// scattered), for reading an assembled but unfactored tree
int launch_materialize_assembly(Plan& P);
// adds the kept entries of tree depth d to the fronts (after the level's extend-add)
int launch_assemble_level(Plan& P, int d, cudaStream_t st);
int launch_pull(Plan& P, const int32_t* perm, const double* X, int64_t ldx, int nrhs, void* xn, double scale);
int launch_push(Plan& P, const int32_t* perm, const void* xn, double* X, int64_t ldx, int nrhs, double scale, int accumulate);
int launch_spmv(Plan& P, double alpha_r, double alpha_i, const double* X, double beta_r, double beta_i,
                double* Y, int64_t ld, int nrhs);
int launch_col_norms(Plan& P, const double* X, int64_t ld, int nrhs, double* out);
// squared 2-norms per (segment of rows seg[s] .. seg[s+1]-1, column): out[j * nseg + s]
int launch_seg_norms(Plan& P, const double* X, int64_t ld, int nrhs, int nseg, const int64_t* seg, double* out);
int launch_reset_status(Plan& P);
// out[e] = -sum_j Xbar[row(e), j] op(X[col(e), j]) over the kept matrix's pattern
int launch_grad_pattern(Plan& P, const double* Xbar, const double* X, int64_t ld, int nrhs, int conj_x, double* out);
// Krylov refinement: out[i][j] = <V_i[:, j], w[:, j]> (pairs), w += sign * sum_i h[i][j] V_i, v = s_j w
int launch_multi_dot(Plan& P, const double* V, int64_t vstride, int nv, const double* w, int nrhs, double* part, double* out);
int launch_multi_axpy(Plan& P, const double* V, int64_t vstride, int nv, const double* h, double* w, int nrhs, double sign);
int launch_col_scale(Plan& P, const double* w, double* v, int nrhs, const double* s);

int check_cuda(const char* where);
// bounded-wait check: one CTA waits on a flag nothing sets (solve_kernels.cu)
int launch_wait_selftest(Plan& P, uint64_t limit_ns);
// packs the launch's operands into `pack`, records `between` (if given),
// runs the GEMM, all on stream st
int launch_tc2(Plan& P, const Launch& ln, cudaEvent_t between, cudaStream_t st, void* pack);
size_t tc2_smem(bool cplx);
// intra-front pivoting (pivot_ldl.cu)
int pivot_begin(Plan& P, cudaStream_t st);
int pivot_level(Plan& P, int depth, cudaStream_t st, bool schur);
int launch_dmma_front_update(Plan& P, const int32_t* fl, int64_t nfronts, int64_t tpf, cudaStream_t st);
int pivot_rowmax(Plan& P, int depth, cudaStream_t st);
int pivot_finish(Plan& P, cudaStream_t st);
int pivot_restore_maps(Plan& P, cudaStream_t st);
int launch_quasi_diag(Plan& P, void* X, int64_t ldx, int nrhs);
const int32_t* solve_perm(const Plan& P, bool nodal);
// FP64 update C -= A D op(B)^T on the FP64 tensor cores (dmma_update.cu); same tiles as gemm_update_kernel
int launch_dmma_update(Plan& P, const Launch& ln, cudaStream_t st);
int launch_panel_tc(Plan& P, const Launch& ln, cudaStream_t st, void* pack);
int build_plan(Plan& P, const cliq_symm_info* info, int64_t n, const int32_t* map, const int64_t* rowptr,
               const int32_t* colind);
int ensure_workspace(Plan& P, int nrhs);
int solve_nodal_dispatch(Plan& P, void* xn, int nrhs);
int run_factor_dispatch(Plan& P);
// autotuner (batch.cu): sets Launch::simt of switchable GEMM launches from
// the process-wide table of measured choices
void apply_tuned_choices(Plan& P);
void free_plan(Plan& P);
// block-LDL front type (block_ldl.cu)
int convert_to_block(Plan& P);
int run_block_solve(Plan& P, void* xn, int nrhs);
void free_block_state(Plan& P);
template <class T, bool C>
void launch_fwd_gather(Plan& P, const SolveLevel& lv, T* X, T* w0, T* w1, int nrhs);
int read_status(Plan& P, int64_t* zero_pivot);

}  // namespace cliqgpu

// the opaque handle of the C ABI
struct cliqgpu_plan_s {
    cliqgpu::Plan p;
};
