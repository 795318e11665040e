// Many independent problems in one plan, and the kernel-choice autotuner.
//
// A batch is a forest: cliq_batch_nested_dissection builds the union of the
// problems' natural nested dissections (symbolic.cpp), cliqgpu_plan_create
// turns it into one plan, and because every factor and sweep launch already
// processes all fronts of one tree depth, the fronts of all problems at the
// same depth share each launch.  cliqgpu_batch_run then runs
//     assemble -> factor -> `steps` refinement steps -> per-problem residuals
// without a host synchronisation in between: the first call launches the
// sequence directly, the second call with the same arguments captures it as
// one CUDA graph, and later calls replay that graph (one launch).  The
// refinement is classical (x += A_f^{-1} r, r = b - A x in FP64): with a
// block-diagonal A every problem's iterate evolves on its own, so the
// per-problem relative residuals ||r_p|| / ||b_p|| measured at the end are
// exactly those of separate solves.  Problems still above the tolerance get
// further (uncaptured) steps.
//
// Autotuner: every GEMM launch of a plan can run on the tensor cores
// (tcgen05 for FP32 storage, DMMA for FP64) or on the CUDA cores.
// cliqgpu_autotune times the factorization with every launch on each kind
// (CUDA events around each launch, best of `reps`), keeps the faster kind
// per launch, and records the choice in a process-wide table keyed by the
// launch's size bucket (field, precision, update kind, log2 of the largest
// M, N, K and of the number of problems), from which later plans take
// their choices when they are built.
//
// No reference counterpart: Clique factors one matrix at a time and has no
// tuning layer.
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "cliqgpu_internal.h"

namespace cliqgpu {

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
using TuneKey = std::array<int, 8>;
static std::mutex g_tune_mu;
static std::map<TuneKey, int> g_tune;   // size bucket -> 1: CUDA cores, 0: tensor cores

static int lg2(int64_t v) {
    int b = 0;
    while (v > 1) { v >>= 1; ++b; }
    return b;
}

static TuneKey tune_key(const Plan& P, const Launch& ln) {
    return {P.field, P.precision, ln.schur, ln.bulk, lg2(ln.maxM), lg2(ln.maxN), lg2(ln.maxK), lg2(ln.nitems)};
}

void apply_tuned_choices(Plan& P) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune.empty()) return;
    for (Launch& ln : P.launches) {
        if (ln.kind != Launch::GEMM || !ln.switchable) continue;
        auto it = g_tune.find(tune_key(P, ln));
        if (it != g_tune.end()) ln.simt = it->second;
    }
}

static int timed_factor(Plan& P, std::vector<double>& best) {
    const int st = launch_assemble(P, P.aval);
    if (st != CLIQ_OK) return st;
    P.profile = 1;
    const int rc = run_factor_dispatch(P);
    if (rc != CLIQ_OK) return rc;
    if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("autotune sync");
    for (size_t li = 0; li < P.launches.size(); ++li) {
        const Launch& ln = P.launches[li];
        if (ln.kind != Launch::GEMM || ln.nblocks <= 0) continue;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, P.events[3 * li], P.events[3 * li + 1]) == cudaSuccess)
            best[li] = std::min(best[li], (double)ms);
    }
    cudaGetLastError();
    return CLIQ_OK;
}

}  // namespace cliqgpu

using namespace cliqgpu;

extern "C" {

int cliqgpu_autotune(cliqgpu_plan h, int32_t reps, double* report) {
    if (!h) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (!P.assembled || !P.keep_matrix) {
        set_last_error("autotune: needs assembled fronts and the plan's copy of A (keep_matrix = 1)");
        return CLIQ_ERR_STATE;
    }
    reps = std::max(1, std::min(reps, 16));
    const int prof0 = P.profile;
    const size_t nl = P.launches.size();
    std::vector<double> t[2] = {std::vector<double>(nl, INFINITY), std::vector<double>(nl, INFINITY)};
    for (int kind = 0; kind < 2; ++kind) {
        for (Launch& ln : P.launches)
            if (ln.kind == Launch::GEMM && ln.switchable) ln.simt = kind;
        for (int r = 0; r < reps; ++r) {
            const int st = timed_factor(P, t[kind]);
            if (st != CLIQ_OK) { P.profile = prof0; return st; }
        }
    }
    double sum0 = 0, sum1 = 0, sumc = 0;
    int nsw = 0, nsimt = 0;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (size_t li = 0; li < nl; ++li) {
            Launch& ln = P.launches[li];
            if (ln.kind != Launch::GEMM || !ln.switchable || ln.nblocks <= 0) continue;
            ++nsw;
            const bool simt = t[1][li] < t[0][li];
            ln.simt = simt ? 1 : 0;
            nsimt += simt;
            sum0 += t[0][li];
            sum1 += t[1][li];
            sumc += std::min(t[0][li], t[1][li]);
            g_tune[tune_key(P, ln)] = ln.simt;
        }
    }
    P.profile = prof0;
    P.prof_pending = false;
    P.factored = true;   // the last trial factored the assembled values
    if (report) {
        report[0] = sum0;
        report[1] = sum1;
        report[2] = sumc;
        report[3] = nsimt;
        report[4] = nsw;
    }
    return CLIQ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batch run
// ---------------------------------------------------------------------------
namespace cliqgpu {

// assemble, factor, `steps` refinement steps, per-segment norms of r and b
// and their copy to pinned host memory: stream-ordered launches only, so the
// whole sequence can be captured
static int batch_issue(Plan& P, const double* values, const double* B, double* X, int64_t ld, int nrhs, int steps) {
    const int w = P.cplx() ? 2 : 1;
    const int64_t n = P.n;
    const size_t colbytes = sizeof(double) * w * (size_t)n;
    double* b = P.xwork;
    double* x = b + (size_t)w * n * nrhs;
    double* r = x + (size_t)w * n * nrhs;
    int st = launch_reset_status(P);
    if (st != CLIQ_OK) return st;
    const size_t vbytes = sizeof(double) * w * (size_t)P.nnz;
    if (cudaMemcpyAsync(P.aval, values, vbytes, cudaMemcpyDeviceToDevice, P.stream) != cudaSuccess) return check_cuda("batch: A");
    if ((st = launch_assemble(P, P.aval)) != CLIQ_OK) return st;
    if ((st = run_factor_dispatch(P)) != CLIQ_OK) return st;
    // sweep flags: the epochs of a replayed graph repeat, so clear what an
    // earlier replay published
    cudaMemsetAsync(P.flags, 0, sizeof(int32_t) * (size_t)(P.flags_total + P.helpers_total), P.stream);
    cudaMemsetAsync(P.xprog, 0, sizeof(unsigned long long) * (size_t)std::max(P.num_fronts, 1), P.stream);
    if (cudaMemcpy2DAsync(b, colbytes, B, sizeof(double) * w * (size_t)ld, colbytes, nrhs, cudaMemcpyDeviceToDevice,
                          P.stream) != cudaSuccess)
        return check_cuda("batch: B");
    cudaMemsetAsync(x, 0, colbytes * nrhs, P.stream);
    cudaMemcpyAsync(r, b, colbytes * nrhs, cudaMemcpyDeviceToDevice, P.stream);
    for (int s = 0; s < steps; ++s) {
        if ((st = launch_pull(P, P.perm, r, n, nrhs, P.xnodal, 1.0)) != CLIQ_OK) return st;
        if ((st = solve_nodal_dispatch(P, P.xnodal, nrhs)) != CLIQ_OK) return st;
        if ((st = launch_push(P, P.perm, P.xnodal, x, n, nrhs, 1.0, 1)) != CLIQ_OK) return st;
        cudaMemcpyAsync(r, b, colbytes * nrhs, cudaMemcpyDeviceToDevice, P.stream);
        if ((st = launch_spmv(P, -1.0, 0.0, x, 1.0, 0.0, r, n, nrhs)) != CLIQ_OK) return st;
    }
    if ((st = launch_seg_norms(P, r, n, nrhs, P.nseg_run(), P.seg, P.segnorm)) != CLIQ_OK) return st;
    if ((st = launch_seg_norms(P, b, n, nrhs, P.nseg_run(), P.seg, P.segnorm + (size_t)P.nseg_run() * nrhs)) != CLIQ_OK)
        return st;
    if (cudaMemcpy2DAsync(X, sizeof(double) * w * (size_t)ld, x, colbytes, colbytes, nrhs, cudaMemcpyDeviceToDevice,
                          P.stream) != cudaSuccess)
        return check_cuda("batch: X");
    if (cudaMemcpyAsync(P.hsegnorm, P.segnorm, sizeof(double) * 2 * (size_t)P.nseg_run() * nrhs, cudaMemcpyDeviceToHost,
                        P.stream) != cudaSuccess)
        return check_cuda("batch: norms");
    return check_cuda("batch launch");
}

// one more refinement step on the device state of the last run, then the
// residual norms to the host
static int batch_extra_step(Plan& P, double* X, int64_t ld, int nrhs) {
    const int w = P.cplx() ? 2 : 1;
    const int64_t n = P.n;
    const size_t colbytes = sizeof(double) * w * (size_t)n;
    double* b = P.xwork;
    double* x = b + (size_t)w * n * nrhs;
    double* r = x + (size_t)w * n * nrhs;
    int st;
    if ((st = launch_pull(P, P.perm, r, n, nrhs, P.xnodal, 1.0)) != CLIQ_OK) return st;
    if ((st = solve_nodal_dispatch(P, P.xnodal, nrhs)) != CLIQ_OK) return st;
    if ((st = launch_push(P, P.perm, P.xnodal, x, n, nrhs, 1.0, 1)) != CLIQ_OK) return st;
    cudaMemcpyAsync(r, b, colbytes * nrhs, cudaMemcpyDeviceToDevice, P.stream);
    if ((st = launch_spmv(P, -1.0, 0.0, x, 1.0, 0.0, r, n, nrhs)) != CLIQ_OK) return st;
    if ((st = launch_seg_norms(P, r, n, nrhs, P.nseg_run(), P.seg, P.segnorm)) != CLIQ_OK) return st;
    cudaMemcpy2DAsync(X, sizeof(double) * w * (size_t)ld, x, colbytes, colbytes, nrhs, cudaMemcpyDeviceToDevice, P.stream);
    cudaMemcpyAsync(P.hsegnorm, P.segnorm, sizeof(double) * (size_t)P.nseg_run() * nrhs, cudaMemcpyDeviceToHost, P.stream);
    return check_cuda("batch extra step");
}

}  // namespace cliqgpu

extern "C" {

int cliqgpu_batch_run(cliqgpu_plan h, int32_t nseg, const int64_t* seg_rows, const void* values, const void* B, void* X,
                      int64_t ld, int32_t nrhs, int32_t steps, double tol, int32_t max_extra, double* relres,
                      int32_t* steps_taken) {
    if (!h || nseg <= 0 || !seg_rows || !values || !B || !X || nrhs <= 0 || steps < 0 || max_extra < 0) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (ld < P.n || !P.keep_matrix) {
        set_last_error("batch_run: needs ld >= n and a plan with keep_matrix = 1");
        return CLIQ_ERR_ARG;
    }
    if (seg_rows[0] != 0 || seg_rows[nseg] != P.n) {
        set_last_error("batch_run: segments must cover rows 0 .. n");
        return CLIQ_ERR_ARG;
    }
    P.block = false;   // every run refactors in the LDL form
    for (int s = 0; s < nseg; ++s)
        if (seg_rows[s + 1] < seg_rows[s]) { set_last_error("batch_run: segments must be ordered"); return CLIQ_ERR_ARG; }
    int st = ensure_workspace(P, nrhs);
    if (st != CLIQ_OK) return st;
    const bool same_seg = (int)P.hseg.size() == nseg + 1 && std::equal(P.hseg.begin(), P.hseg.end(), seg_rows);
    if (!same_seg) {
        if (P.seg) cudaFree(P.seg);
        P.seg = nullptr;
        if (cudaMalloc(&P.seg, sizeof(int64_t) * (nseg + 1)) != cudaSuccess) return check_cuda("batch: segments");
        if (cudaMemcpy(P.seg, seg_rows, sizeof(int64_t) * (nseg + 1), cudaMemcpyHostToDevice) != cudaSuccess)
            return check_cuda("batch: segments");
        P.hseg.assign(seg_rows, seg_rows + nseg + 1);
    }
    const int64_t need = 2 * (int64_t)nseg * nrhs;
    if (need > P.segnorm_cap) {
        if (P.segnorm) cudaFree(P.segnorm);
        if (P.hsegnorm) cudaFreeHost(P.hsegnorm);
        P.segnorm = nullptr;
        P.hsegnorm = nullptr;
        P.segnorm_cap = 0;
        if (cudaMalloc(&P.segnorm, sizeof(double) * need) != cudaSuccess ||
            cudaMallocHost(&P.hsegnorm, sizeof(double) * need) != cudaSuccess)
            return check_cuda("batch: norms");
        P.segnorm_cap = need;
    }
    const std::vector<int64_t> key = {(int64_t)(uintptr_t)values, (int64_t)(uintptr_t)B, (int64_t)(uintptr_t)X, ld, nrhs,
                                      steps, nseg, (int64_t)(uintptr_t)P.seg, (int64_t)(uintptr_t)P.segnorm,
                                      (int64_t)(uintptr_t)P.xwork};
    if (P.batch_exec && key != P.batch_key) {   // arguments changed: record again
        cudaGraphExecDestroy(P.batch_exec);
        P.batch_exec = nullptr;
        P.batch_runs = 0;
    }
    P.batch_key = key;
    P.last_launches = 0;
    if (P.batch_exec) {
        if (cudaGraphLaunch(P.batch_exec, P.stream) != cudaSuccess) return check_cuda("batch graph launch");
        P.total_launches += P.batch_graph_launches;
        P.last_launches = P.batch_graph_launches;
    } else if (P.batch_graph && P.batch_runs > 0 && P.stream != cudaStreamLegacy && P.stream != nullptr) {
        // (the legacy default stream cannot be captured: such plans keep direct launches)
        const int64_t before = P.total_launches;
        if (cudaStreamBeginCapture(P.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return check_cuda("batch capture");
        st = batch_issue(P, (const double*)values, (const double*)B, (double*)X, ld, nrhs, steps);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(P.stream, &g);
        if (st != CLIQ_OK || e != cudaSuccess || !g || cudaGraphInstantiate(&P.batch_exec, g, 0) != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            P.batch_exec = nullptr;
            cudaGetLastError();
            set_last_error("batch_run: the run could not be captured as a graph");
            return st != CLIQ_OK ? st : CLIQ_ERR_CUDA;
        }
        cudaGraphDestroy(g);
        P.batch_graph_launches = P.total_launches - before;
        P.total_launches = before;
        if (cudaGraphLaunch(P.batch_exec, P.stream) != cudaSuccess) return check_cuda("batch graph launch");
        P.total_launches += P.batch_graph_launches;
        P.last_launches = P.batch_graph_launches;
    } else {
        const int64_t before = P.total_launches;
        st = batch_issue(P, (const double*)values, (const double*)B, (double*)X, ld, nrhs, steps);
        if (st != CLIQ_OK) return st;
        P.last_launches = P.total_launches - before;
    }
    ++P.batch_runs;
    P.assembled = P.factored = true;
    if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("batch sync");
    // per (problem, column) relative residuals; zero right-hand sides count as solved
    std::vector<double> bn(P.hsegnorm + (size_t)nseg * nrhs, P.hsegnorm + 2 * (size_t)nseg * nrhs);
    auto worst = [&](std::vector<double>* out) {
        double wv = 0;
        for (int64_t i = 0; i < (int64_t)nseg * nrhs; ++i) {
            const double rr = bn[i] > 0 ? std::sqrt(P.hsegnorm[i] / bn[i]) : 0.0;
            if (out) (*out)[i] = rr;
            wv = (rr == rr) ? std::max(wv, rr) : INFINITY;
        }
        return wv;
    };
    double wv = worst(nullptr);
    int taken = steps, extra = 0;
    while (wv > tol && extra < max_extra) {
        const int64_t before = P.total_launches;
        if ((st = batch_extra_step(P, (double*)X, ld, nrhs)) != CLIQ_OK) return st;
        P.last_launches += P.total_launches - before;
        if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("batch sync");
        wv = worst(nullptr);
        ++extra;
        ++taken;
    }
    if (relres) {
        std::vector<double> out((size_t)nseg * nrhs);
        worst(&out);
        std::copy(out.begin(), out.end(), relres);
    }
    if (steps_taken) *steps_taken = taken;
    int32_t dst[2];
    if (cudaMemcpy(dst, P.status, sizeof(dst), cudaMemcpyDeviceToHost) != cudaSuccess) return check_cuda("batch status");
    if (dst[1]) { set_last_error("a device-side wait timed out"); return CLIQ_ERR_TIMEOUT; }
    if (dst[0] != INT_MAX) {
        set_last_error("zero pivot at ND index " + std::to_string((int64_t)dst[0] - 1));
        return CLIQ_ERR_ZERO_PIVOT;
    }
    return wv <= tol ? CLIQ_OK : CLIQ_ERR_NOCONV;
}

}  // extern "C"
