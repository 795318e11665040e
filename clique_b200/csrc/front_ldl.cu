// cliqgpu_front_ldl: the dense partial LDL^T of a single front
// (cliq::FrontLDL, include/clique/numeric/ldl/local_front.hpp:30-71) on
// caller-owned device memory, run through the same kernels as the tree
// factorization by describing the front as a one-node tree.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <vector>

#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {

// FrontLDL leaves D on the diagonal of AL; the tree kernels store 1 there
// and D separately, so put D back.
template <class T, bool C>
__global__ void put_diag_kernel(T* __restrict__ A, int64_t lda, int n, const double* __restrict__ D) {
    using W = DV<C>;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        stv<T, C>(A, j + (int64_t)j * lda, conv<V<T, C>>(reinterpret_cast<const W*>(D)[j]));
}

}  // namespace cliqgpu

using namespace cliqgpu;

extern "C" int cliqgpu_front_ldl(int32_t field, int32_t precision, int32_t conjugate, int32_t m, int32_t n, void* AL,
                                 int64_t lda, void* ABR, int64_t ldabr, void* stream) {
    if (m < 0 || n < 0 || n > m || !AL || lda < std::max(m, 1) || (m > n && (!ABR || ldabr < m - n))) return CLIQ_ERR_ARG;
    if (n == 0) return CLIQ_OK;
    Plan P;
    P.field = field == CLIQ_COMPLEX ? CLIQ_COMPLEX : CLIQ_REAL;
    P.precision = precision == CLIQ_FP32 ? CLIQ_FP32 : CLIQ_FP64;
    P.conjugate = conjugate ? 1 : 0;
    P.nb = kTile;
    if (const char* e = getenv("CLIQGPU_TENSOR_CORES")) P.use_tc = atoi(e) != 0;
    if (const char* e = getenv("CLIQGPU_FP64_DMMA")) P.fp64_dmma = atoi(e) != 0;
    P.stream = (cudaStream_t)stream;
    // one node: pivots 0..n-1, update rows n..m-1
    std::vector<int32_t> size{n}, off{0}, parent{-1}, children{-1, -1}, lower(m - n), map(n);
    std::vector<int64_t> lower_ptr{0, (int64_t)(m - n)}, rowptr(n + 1, 0);
    for (int i = 0; i < m - n; ++i) lower[i] = n + i;
    for (int i = 0; i < n; ++i) map[i] = i;
    cliq_symm_info info{1, size.data(), off.data(), parent.data(), children.data(), lower_ptr.data(), lower.data(),
                        nullptr, nullptr};
    int32_t dummy_col = 0;
    int st = build_plan(P, &info, n, map.data(), rowptr.data(), &dummy_col);
    if (st != CLIQ_OK) { free_plan(P); return st; }
    // no extend-add: the caller's ABR is the initial update
    P.launches.erase(std::remove_if(P.launches.begin(), P.launches.end(),
                                    [](const Launch& l) { return l.kind == Launch::EXTEND_ADD; }),
                     P.launches.end());
    const int eb = P.elem_bytes();
    const FrontDev& f = P.hfronts[0];
    cudaMemcpy2DAsync((char*)P.L + (size_t)f.L * eb, (size_t)m * eb, AL, (size_t)lda * eb, (size_t)m * eb, n,
                      cudaMemcpyDeviceToDevice, P.stream);
    if (m > n)
        cudaMemcpy2DAsync((char*)P.pool[f.pool] + (size_t)f.U * eb, (size_t)(m - n) * eb, ABR, (size_t)ldabr * eb,
                          (size_t)(m - n) * eb, m - n, cudaMemcpyDeviceToDevice, P.stream);
    int32_t st0[4] = {INT_MAX, 0, 0, 0};
    cudaMemcpyAsync(P.status, st0, sizeof(st0), cudaMemcpyHostToDevice, P.stream);
    if (P.precision == CLIQ_FP64) st = P.cplx() ? run_factor<double, true>(P) : run_factor<double, false>(P);
    else st = P.cplx() ? run_factor<float, true>(P) : run_factor<float, false>(P);
    if (st == CLIQ_OK) {
        cudaMemcpy2DAsync(AL, (size_t)lda * eb, (char*)P.L + (size_t)f.L * eb, (size_t)m * eb, (size_t)m * eb, n,
                          cudaMemcpyDeviceToDevice, P.stream);
        if (P.precision == CLIQ_FP64) {
            if (P.cplx()) put_diag_kernel<double, true><<<(n + 255) / 256, 256, 0, P.stream>>>((double*)AL, lda, n, P.D);
            else put_diag_kernel<double, false><<<(n + 255) / 256, 256, 0, P.stream>>>((double*)AL, lda, n, P.D);
        } else {
            if (P.cplx()) put_diag_kernel<float, true><<<(n + 255) / 256, 256, 0, P.stream>>>((float*)AL, lda, n, P.D);
            else put_diag_kernel<float, false><<<(n + 255) / 256, 256, 0, P.stream>>>((float*)AL, lda, n, P.D);
        }
        if (m > n)
            cudaMemcpy2DAsync(ABR, (size_t)ldabr * eb, (char*)P.pool[f.pool] + (size_t)f.U * eb, (size_t)(m - n) * eb,
                              (size_t)(m - n) * eb, m - n, cudaMemcpyDeviceToDevice, P.stream);
        st = check_cuda("front_ldl");
        if (st == CLIQ_OK) {
            int64_t zp;
            st = read_status(P, &zp);
        }
    }
    cudaStreamSynchronize(P.stream);
    free_plan(P);
    return st;
}
