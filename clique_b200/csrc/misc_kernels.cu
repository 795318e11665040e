// Bandwidth-bound helpers: front assembly, nodal pull/push with precision
// conversion, FP64 CSR multiply and column norms for refinement.
#include <algorithm>
#include <climits>

#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {

static inline unsigned grid_for(int64_t work, int threads) {
    int64_t b = (work + threads - 1) / threads;
    const int64_t cap = 148 * 16;
    if (b > cap) b = cap;
    return (unsigned)(b < 1 ? 1 : b);
}

// DistSymmFrontTree::Initialize value scatter (dist_symm_front_tree/impl.hpp:275-294):
// frontL[dest[e]] = conj?(A[e]); entries above the front's diagonal have dest = -1.
template <class T, bool C, bool CJ>
__global__ void assemble_kernel(const int64_t* __restrict__ dest, const double* __restrict__ vals, int64_t nnz, T* __restrict__ L) {
    using Xv = V<T, C>;
    using W = DV<C>;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = dest[e];
        if (d < 0) continue;
        W v = reinterpret_cast<const W*>(vals)[e];
        v = opc<CJ>(v);
        stv<T, C>(L, d, conv<Xv>(v));
    }
}

template <class T, bool C>
static int materialize_t(Plan& P) {
    cudaMemsetAsync(P.L, 0, (size_t)P.arena_elems * P.elem_bytes(), P.stream);
    if (P.conjugate && C)
        assemble_kernel<T, C, true><<<grid_for(P.nnz, 256), 256, 0, P.stream>>>(P.dest, P.aval, P.nnz, reinterpret_cast<T*>(P.L));
    else
        assemble_kernel<T, C, false><<<grid_for(P.nnz, 256), 256, 0, P.stream>>>(P.dest, P.aval, P.nnz, reinterpret_cast<T*>(P.L));
    P.total_launches += 1;
    return check_cuda("assemble");
}

int launch_materialize_assembly(Plan& P) {
    if (P.precision == CLIQ_FP64) return P.cplx() ? materialize_t<double, true>(P) : materialize_t<double, false>(P);
    return P.cplx() ? materialize_t<float, true>(P) : materialize_t<float, false>(P);
}

int launch_assemble(Plan& P, const double* dvals) {
    if (dvals != P.aval &&
        cudaMemcpyAsync(P.aval, dvals, sizeof(double) * (P.cplx() ? 2 : 1) * (size_t)P.nnz, cudaMemcpyDeviceToDevice,
                        P.stream) != cudaSuccess)
        return check_cuda("assemble");
    return CLIQ_OK;
}

// DistSymmFrontTree::Initialize's scatter for the fronts of one tree depth,
// as an addition: the level's extend-add has just written every lower entry
// of these fronts (children's contributions, or zero), and each kept entry of
// A has its own destination (dist_symm_front_tree/impl.hpp:275-294)
template <class T, bool C, bool CJ>
__global__ void assemble_add_kernel(const int64_t* __restrict__ src, const int64_t* __restrict__ dst, int64_t cnt,
                                    const double* __restrict__ vals, T* __restrict__ L) {
    using Xv = V<T, C>;
    using W = DV<C>;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = dst[i];
        const W v = opc<CJ>(reinterpret_cast<const W*>(vals)[src[i]]);
        stv<T, C>(L, d, ldv<T, C>(L, d) + conv<Xv>(v));
    }
}

template <class T, bool C>
static int assemble_level_t(Plan& P, int d, cudaStream_t st) {
    const int64_t b = P.asm_level[d], cnt = P.asm_level[d + 1] - b;
    if (cnt <= 0) return CLIQ_OK;
    if (P.conjugate && C)
        assemble_add_kernel<T, C, true><<<grid_for(cnt, 256), 256, 0, st>>>(P.asm_src + b, P.asm_dst + b, cnt, P.aval,
                                                                               reinterpret_cast<T*>(P.L));
    else
        assemble_add_kernel<T, C, false><<<grid_for(cnt, 256), 256, 0, st>>>(P.asm_src + b, P.asm_dst + b, cnt, P.aval,
                                                                                reinterpret_cast<T*>(P.L));
    P.total_launches += 1;
    return CLIQ_OK;
}

int launch_assemble_level(Plan& P, int d, cudaStream_t st) {
    if (d < 0 || d + 1 >= (int)P.asm_level.size()) return CLIQ_OK;
    if (P.precision == CLIQ_FP64) return P.cplx() ? assemble_level_t<double, true>(P, d, st) : assemble_level_t<double, false>(P, d, st);
    return P.cplx() ? assemble_level_t<float, true>(P, d, st) : assemble_level_t<float, false>(P, d, st);
}

// Pull (dist_nodal_multi_vec/impl.hpp:67-219 at P=1): xn[p, j] = scale * X[inv[p], j]
template <class T, bool C>
__global__ void pull_kernel(const double* __restrict__ X, int64_t ldx, int64_t n, int nrhs, const int32_t* __restrict__ perm,
                            T* __restrict__ xn, double scale) {
    using Xv = V<T, C>;
    using W = DV<C>;
    const int64_t total = n * nrhs;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = idx % n, j = idx / n;
        W v = reinterpret_cast<const W*>(X)[(perm ? perm[p] : p) + j * ldx];
        if constexpr (C) { v.r *= scale; v.i *= scale; } else { v *= scale; }
        stv<T, C>(xn, p + j * n, conv<Xv>(v));
    }
}

// Push: X[inv[p], j] (=|+=) scale * xn[p, j]
template <class T, bool C>
__global__ void push_kernel(const T* __restrict__ xn, double* __restrict__ X, int64_t ldx, int64_t n, int nrhs,
                            const int32_t* __restrict__ perm, double scale, int accumulate) {
    using W = DV<C>;
    const int64_t total = n * nrhs;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = idx % n, j = idx / n;
        W v = conv<W>(ldv<T, C>(xn, p + j * n));
        if constexpr (C) { v.r *= scale; v.i *= scale; } else { v *= scale; }
        W* dst = reinterpret_cast<W*>(X) + (perm ? perm[p] : p) + j * ldx;
        if (accumulate) *dst += v; else *dst = v;
    }
}

int launch_pull(Plan& P, const int32_t* perm, const double* X, int64_t ldx, int nrhs, void* xn, double scale) {
    const unsigned g = grid_for(P.n * nrhs, 256);
    if (P.precision == CLIQ_FP64) {
        if (P.cplx()) pull_kernel<double, true><<<g, 256, 0, P.stream>>>(X, ldx, P.n, nrhs, perm, (double*)xn, scale);
        else pull_kernel<double, false><<<g, 256, 0, P.stream>>>(X, ldx, P.n, nrhs, perm, (double*)xn, scale);
    } else {
        if (P.cplx()) pull_kernel<float, true><<<g, 256, 0, P.stream>>>(X, ldx, P.n, nrhs, perm, (float*)xn, scale);
        else pull_kernel<float, false><<<g, 256, 0, P.stream>>>(X, ldx, P.n, nrhs, perm, (float*)xn, scale);
    }
    P.total_launches += 1;
    return check_cuda("pull");
}

int launch_push(Plan& P, const int32_t* perm, const void* xn, double* X, int64_t ldx, int nrhs, double scale, int accumulate) {
    const unsigned g = grid_for(P.n * nrhs, 256);
    if (P.precision == CLIQ_FP64) {
        if (P.cplx()) push_kernel<double, true><<<g, 256, 0, P.stream>>>((const double*)xn, X, ldx, P.n, nrhs, perm, scale, accumulate);
        else push_kernel<double, false><<<g, 256, 0, P.stream>>>((const double*)xn, X, ldx, P.n, nrhs, perm, scale, accumulate);
    } else {
        if (P.cplx()) push_kernel<float, true><<<g, 256, 0, P.stream>>>((const float*)xn, X, ldx, P.n, nrhs, perm, scale, accumulate);
        else push_kernel<float, false><<<g, 256, 0, P.stream>>>((const float*)xn, X, ldx, P.n, nrhs, perm, scale, accumulate);
    }
    P.total_launches += 1;
    return check_cuda("push");
}

// Multiply (multiply.hpp:150-165 at P=1): Y := beta Y + alpha A X, one thread per row
template <bool C>
__global__ void spmv_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ colind, const double* __restrict__ vals,
                            int64_t n, DV<C> alpha, const double* __restrict__ X, DV<C> beta, double* __restrict__ Y, int64_t ld,
                            int nrhs) {
    using W = DV<C>;
    const W* A = reinterpret_cast<const W*>(vals);
    const W* x = reinterpret_cast<const W*>(X);
    W* y = reinterpret_cast<W*>(Y);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e0 = rowptr[i], e1 = rowptr[i + 1];
        for (int j = 0; j < nrhs; ++j) {
            W s{};
            for (int64_t e = e0; e < e1; ++e) mac(s, A[e], x[colind[e] + j * ld]);
            const int64_t o = i + j * ld;
            y[o] = is_zero(beta) ? alpha * s : beta * y[o] + alpha * s;   // beta = 0: Y is not read (BLAS semantics)
        }
    }
}

int launch_spmv(Plan& P, double ar, double ai, const double* X, double br, double bi, double* Y, int64_t ld, int nrhs) {
    const unsigned g = grid_for(P.n, 256);
    if (P.cplx())
        spmv_kernel<true><<<g, 256, 0, P.stream>>>(P.rowptr, P.colind, P.aval, P.n, cx<double>{ar, ai}, X, cx<double>{br, bi}, Y, ld, nrhs);
    else
        spmv_kernel<false><<<g, 256, 0, P.stream>>>(P.rowptr, P.colind, P.aval, P.n, ar, X, br, Y, ld, nrhs);
    P.total_launches += 1;
    return check_cuda("multiply");
}

// Squared 2-norms of the nrhs columns of X (FP64; complex: |re|^2 + |im|^2).
// Stage 1: kNormChunks CTAs per column write partial sums; stage 2 adds
// them in a fixed order, so the result does not depend on scheduling.
constexpr int kNormChunks = 128;

template <bool C>
__global__ void col_norms_partial_kernel(const double* __restrict__ X, int64_t ld, int64_t n, double* __restrict__ part) {
    const int j = blockIdx.y;
    const int w = C ? 2 : 1;
    const double* x = X + (int64_t)w * j * ld;
    const int64_t len = n * w;
    const int64_t per = (len + kNormChunks - 1) / kNormChunks;
    const int64_t b = per * blockIdx.x, e = min(len, b + per);
    double s = 0;
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) s = fma(x[i], x[i], s);
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) part[(int64_t)j * kNormChunks + blockIdx.x] = s;
    }
}

__global__ void col_norms_final_kernel(const double* __restrict__ part, double* __restrict__ out) {
    const int j = blockIdx.x;
    double s = part[(int64_t)j * kNormChunks + threadIdx.x];
    __shared__ double red[kNormChunks / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int q = 0; q < kNormChunks / 32; ++q) t += red[q];
        out[j] = t;
    }
}

int launch_col_norms(Plan& P, const double* X, int64_t ld, int nrhs, double* out) {
    double* part = P.norms + 2 * P.ws_nrhs;   // kNormChunks * nrhs scratch after the two norm vectors
    const dim3 grid(kNormChunks, nrhs);
    if (P.cplx()) col_norms_partial_kernel<true><<<grid, 256, 0, P.stream>>>(X, ld, P.n, part);
    else col_norms_partial_kernel<false><<<grid, 256, 0, P.stream>>>(X, ld, P.n, part);
    col_norms_final_kernel<<<nrhs, kNormChunks, 0, P.stream>>>(part, out);
    P.total_launches += 2;
    return check_cuda("norms");
}

// ---------------------------------------------------------------------------
// FP64 block-vector operations for the Krylov refinement.  A block vector
// holds nrhs columns of length n (complex: interleaved), column j at
// j * n * w doubles; a basis is nv block vectors vstride doubles apart.
// ---------------------------------------------------------------------------
constexpr int kDotChunks = 128;

// part[(i * nrhs + j) * kDotChunks + chunk] = partial of <V_i[:, j], w[:, j]>
// (conjugate-linear in V); fixed-order second stage below
template <bool C>
__global__ void multi_dot_partial_kernel(const double* __restrict__ V, int64_t vstride, const double* __restrict__ w, int64_t n,
                                         int nrhs, double* __restrict__ part) {
    const int i = blockIdx.z, j = blockIdx.y;
    constexpr int ww = C ? 2 : 1;
    const double* v = V + (int64_t)i * vstride + (int64_t)j * n * ww;
    const double* x = w + (int64_t)j * n * ww;
    const int64_t per = (n + kDotChunks - 1) / kDotChunks;
    const int64_t b = per * blockIdx.x, e = min(n, b + per);
    double sr = 0, si = 0;
    for (int64_t p = b + threadIdx.x; p < e; p += blockDim.x) {
        if constexpr (C) {
            const double vr = v[2 * p], vi = v[2 * p + 1], xr = x[2 * p], xi = x[2 * p + 1];
            sr = fma(vr, xr, fma(vi, xi, sr));
            si = fma(vr, xi, fma(-vi, xr, si));
        } else {
            sr = fma(v[p], x[p], sr);
        }
    }
    __shared__ double rr[32], ri[32];
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_down_sync(0xffffffffu, sr, o);
        si += __shfl_down_sync(0xffffffffu, si, o);
    }
    if ((threadIdx.x & 31) == 0) { rr[threadIdx.x >> 5] = sr; ri[threadIdx.x >> 5] = si; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0, ti = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { tr += rr[q]; ti += ri[q]; }
        const int64_t o = ((int64_t)i * nrhs + j) * kDotChunks + blockIdx.x;
        part[2 * o] = tr;
        part[2 * o + 1] = ti;
    }
}

__global__ void multi_dot_final_kernel(const double* __restrict__ part, double* __restrict__ out) {
    const int o = blockIdx.x;
    if (threadIdx.x == 0) {
        double tr = 0, ti = 0;
        for (int c = 0; c < kDotChunks; ++c) { tr += part[2 * ((int64_t)o * kDotChunks + c)]; ti += part[2 * ((int64_t)o * kDotChunks + c) + 1]; }
        out[2 * o] = tr;
        out[2 * o + 1] = ti;
    }
}

// w[:, j] += sign * sum_i h[i][j] V_i[:, j]   (h complex pairs, or reals in the first slot)
template <bool C>
__global__ void multi_axpy_kernel(const double* __restrict__ V, int64_t vstride, int nv, const double* __restrict__ h,
                                  double* __restrict__ w, int64_t n, int nrhs, double sign) {
    constexpr int ww = C ? 2 : 1;
    const int64_t total = n * nrhs;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = idx % n, j = idx / n;
        const int64_t e = (j * n + p) * ww;
        if constexpr (C) {
            double ar = 0, ai = 0;
            for (int i = 0; i < nv; ++i) {
                const double hr = h[2 * (i * nrhs + j)], hi = h[2 * (i * nrhs + j) + 1];
                const double vr = V[(int64_t)i * vstride + e], vi = V[(int64_t)i * vstride + e + 1];
                ar = fma(hr, vr, fma(-hi, vi, ar));
                ai = fma(hr, vi, fma(hi, vr, ai));
            }
            w[e] += sign * ar;
            w[e + 1] += sign * ai;
        } else {
            double a = 0;
            for (int i = 0; i < nv; ++i) a = fma(h[2 * (i * nrhs + j)], V[(int64_t)i * vstride + e], a);
            w[e] += sign * a;
        }
    }
}

// v[:, j] = s_j * w[:, j], s real
__global__ void col_scale_kernel(const double* __restrict__ w, double* __restrict__ v, int64_t len_per_col, int nrhs,
                                 const double* __restrict__ s) {
    const int64_t total = len_per_col * nrhs;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x)
        v[idx] = w[idx] * s[idx / len_per_col];
}

int launch_multi_dot(Plan& P, const double* V, int64_t vstride, int nv, const double* w, int nrhs, double* part, double* out) {
    const dim3 grid(kDotChunks, nrhs, nv);
    if (P.cplx()) multi_dot_partial_kernel<true><<<grid, 256, 0, P.stream>>>(V, vstride, w, P.n, nrhs, part);
    else multi_dot_partial_kernel<false><<<grid, 256, 0, P.stream>>>(V, vstride, w, P.n, nrhs, part);
    multi_dot_final_kernel<<<nv * nrhs, 32, 0, P.stream>>>(part, out);
    P.total_launches += 2;
    return check_cuda("multi_dot");
}

int launch_multi_axpy(Plan& P, const double* V, int64_t vstride, int nv, const double* h, double* w, int nrhs, double sign) {
    if (P.cplx()) multi_axpy_kernel<true><<<1184, 256, 0, P.stream>>>(V, vstride, nv, h, w, P.n, nrhs, sign);
    else multi_axpy_kernel<false><<<1184, 256, 0, P.stream>>>(V, vstride, nv, h, w, P.n, nrhs, sign);
    P.total_launches += 1;
    return check_cuda("multi_axpy");
}

int launch_col_scale(Plan& P, const double* w, double* v, int nrhs, const double* s) {
    col_scale_kernel<<<1184, 256, 0, P.stream>>>(w, v, P.n * (P.cplx() ? 2 : 1), nrhs, s);
    P.total_launches += 1;
    return check_cuda("col_scale");
}

// Nodal pull / push of FP64 multivectors between natural and ND order
// (DistNodalMultiVec::Pull / Push, dist_nodal_multi_vec/impl.hpp:67-219 at P=1):
// dir 0: Y[p, j] = X[perm[p], j]; dir 1: Y[perm[p], j] = X[p, j]
template <bool C>
__global__ void permute_rows_kernel(const double* __restrict__ X, int64_t ldx, double* __restrict__ Y, int64_t ldy, int64_t n,
                                    int nrhs, const int32_t* __restrict__ perm, int dir) {
    using W = DV<C>;
    const int64_t total = n * nrhs;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = idx % n, j = idx / n;
        const int64_t q = perm[p];
        if (dir == 0) reinterpret_cast<W*>(Y)[p + j * ldy] = reinterpret_cast<const W*>(X)[q + j * ldx];
        else reinterpret_cast<W*>(Y)[q + j * ldy] = reinterpret_cast<const W*>(X)[p + j * ldx];
    }
}

// Squared 2-norms per (segment, column): out[j * nseg + s] = sum over rows
// seg[s] .. seg[s+1]-1 of |X[row, j]|^2 (complex: |re|^2 + |im|^2), one CTA
// per (segment, column), fixed reduction order.
template <bool C>
__global__ void seg_norms_kernel(const double* __restrict__ X, int64_t ld, const int64_t* __restrict__ seg, int nseg,
                                 double* __restrict__ out) {
    const int sgi = blockIdx.x, j = blockIdx.y;
    const int w = C ? 2 : 1;
    const int64_t b = seg[sgi] * w, e = seg[sgi + 1] * w;
    const double* x = X + (int64_t)w * j * ld;
    double acc = 0;
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) acc = fma(x[i], x[i], acc);
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
        out[(int64_t)j * nseg + sgi] = t;
    }
}

int launch_seg_norms(Plan& P, const double* X, int64_t ld, int nrhs, int nseg, const int64_t* seg, double* out) {
    const dim3 grid(nseg, nrhs);
    if (P.cplx()) seg_norms_kernel<true><<<grid, 256, 0, P.stream>>>(X, ld, seg, nseg, out);
    else seg_norms_kernel<false><<<grid, 256, 0, P.stream>>>(X, ld, seg, nseg, out);
    P.total_launches += 1;
    return check_cuda("segment norms");
}

// status word := {no zero pivot, no timeout, no site, 0}, written on the
// device so that the reset can be part of a captured graph
__global__ void reset_status_kernel(int32_t* status) {
    if (threadIdx.x == 0) { status[0] = INT_MAX; status[1] = 0; status[2] = 0; status[3] = 0; }
}

int launch_reset_status(Plan& P) {
    reset_status_kernel<<<1, 32, 0, P.stream>>>(P.status);
    P.total_launches += 1;
    return check_cuda("status reset");
}

// Pattern-restricted gradient of a linear solve X = A^{-1} B with respect to
// the stored entries of A: out[e] = -sum_j Xbar[row(e), j] op(X[col(e), j])
// (op = conjugation for the conjugate-linear convention of complex autograd),
// one warp per row, the row's entries split over the lanes.
template <bool C, bool CJ>
__global__ void grad_pattern_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ colind, int64_t n,
                                    const double* __restrict__ Xbar, const double* __restrict__ X, int64_t ld, int nrhs,
                                    double* __restrict__ out) {
    using W = DV<C>;
    const W* gb = reinterpret_cast<const W*>(Xbar);
    const W* x = reinterpret_cast<const W*>(X);
    W* o = reinterpret_cast<W*>(out);
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        const int64_t e0 = rowptr[i], e1 = rowptr[i + 1];
        for (int64_t e = e0 + lane; e < e1; e += 32) {
            const int64_t c = colind[e];
            W s{};
            for (int j = 0; j < nrhs; ++j) mac(s, gb[i + j * ld], opc<CJ>(x[c + j * ld]));
            o[e] = W{} - s;
        }
    }
}

int launch_grad_pattern(Plan& P, const double* Xbar, const double* X, int64_t ld, int nrhs, int conj_x, double* out) {
    const unsigned g = grid_for(P.n * 32, 256);
    if (P.cplx()) {
        if (conj_x) grad_pattern_kernel<true, true><<<g, 256, 0, P.stream>>>(P.rowptr, P.colind, P.n, Xbar, X, ld, nrhs, out);
        else grad_pattern_kernel<true, false><<<g, 256, 0, P.stream>>>(P.rowptr, P.colind, P.n, Xbar, X, ld, nrhs, out);
    } else {
        grad_pattern_kernel<false, false><<<g, 256, 0, P.stream>>>(P.rowptr, P.colind, P.n, Xbar, X, ld, nrhs, out);
    }
    P.total_launches += 1;
    return check_cuda("grad_A_pattern");
}

}  // namespace cliqgpu

using namespace cliqgpu;

// ===========================================================================
// cliqgpu_nodal_pull / cliqgpu_nodal_push: FP64 device multivectors between
// natural and nested-dissection order through a device copy of the inverse
// map (ND index -> natural index).
// ===========================================================================
static int permute_rows(int32_t field, int64_t n, const int32_t* inverse_map, const void* X, int64_t ldx, void* Y, int64_t ldy,
                        int32_t nrhs, int dir, void* stream) {
    if (n < 0 || nrhs < 0 || ldx < n || ldy < n || (n > 0 && nrhs > 0 && (!inverse_map || !X || !Y))) {
        set_last_error("nodal pull/push: invalid sizes or pointers");
        return CLIQ_ERR_ARG;
    }
    if (n == 0 || nrhs == 0) return CLIQ_OK;
    const unsigned g = grid_for(n * nrhs, 256);
    cudaStream_t st = (cudaStream_t)stream;
    if (field == CLIQ_COMPLEX)
        permute_rows_kernel<true><<<g, 256, 0, st>>>((const double*)X, ldx, (double*)Y, ldy, n, nrhs, inverse_map, dir);
    else
        permute_rows_kernel<false><<<g, 256, 0, st>>>((const double*)X, ldx, (double*)Y, ldy, n, nrhs, inverse_map, dir);
    return check_cuda(dir == 0 ? "nodal pull" : "nodal push");
}

extern "C" int cliqgpu_nodal_pull(int32_t field, int64_t n, const int32_t* inverse_map, const void* X, int64_t ldx, void* Xn,
                                  int64_t ldn, int32_t nrhs, void* stream) {
    return permute_rows(field, n, inverse_map, X, ldx, Xn, ldn, nrhs, 0, stream);
}

extern "C" int cliqgpu_nodal_push(int32_t field, int64_t n, const int32_t* inverse_map, const void* Xn, int64_t ldn, void* X,
                                  int64_t ldx, int32_t nrhs, void* stream) {
    return permute_rows(field, n, inverse_map, Xn, ldn, X, ldx, nrhs, 1, stream);
}

// ===========================================================================
// cliqgpu_sparse_multiply: Y := alpha A X + beta Y for a CSR matrix that is not
// held by a plan (the free function cliq::Multiply, multiply.hpp:18-21,28-166).
// Host buffers are staged through stream-ordered device allocations.
// ===========================================================================
extern "C" int cliqgpu_sparse_multiply(int32_t field, int64_t n, const int64_t* rowptr, const int32_t* colind,
                                       const double* values, const double* alpha, const void* X, const double* beta,
                                       void* Y, int64_t ld, int32_t nrhs, int32_t on_device, void* stream) {
    if (n < 0 || nrhs < 0 || !alpha || !beta || (n > 0 && nrhs > 0 && (!rowptr || !colind || !values || !X || !Y)) ||
        ld < n) {
        set_last_error("sparse_multiply: invalid sizes or pointers");
        return CLIQ_ERR_ARG;
    }
    if (n == 0 || nrhs == 0) return CLIQ_OK;
    const bool c = field == CLIQ_COMPLEX;
    const int w = c ? 2 : 1;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t *rp = rowptr;
    const int32_t* ci = colind;
    const double *va = values, *xd = (const double*)X;
    double* yd = (double*)Y;
    void* tmp[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int64_t nnz = 0;
    const size_t vec = sizeof(double) * w * (size_t)ld * nrhs;
    if (!on_device) {
        nnz = rowptr[n];
        const size_t sz[5] = {sizeof(int64_t) * (size_t)(n + 1), sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1),
                              sizeof(double) * w * (size_t)std::max<int64_t>(nnz, 1), vec, vec};
        const void* src[5] = {rowptr, colind, values, X, Y};
        for (int i = 0; i < 5; ++i) {
            if (cudaMallocAsync(&tmp[i], sz[i], st) != cudaSuccess) {
                for (int k = 0; k < i; ++k) cudaFreeAsync(tmp[k], st);
                return check_cuda("sparse_multiply: staging");
            }
            const size_t b = (i == 1 || i == 2) && nnz == 0 ? 0 : sz[i];
            if (b && cudaMemcpyAsync(tmp[i], src[i], b, cudaMemcpyHostToDevice, st) != cudaSuccess) {
                for (int k = 0; k <= i; ++k) cudaFreeAsync(tmp[k], st);
                return check_cuda("sparse_multiply: copy in");
            }
        }
        rp = (const int64_t*)tmp[0];
        ci = (const int32_t*)tmp[1];
        va = (const double*)tmp[2];
        xd = (const double*)tmp[3];
        yd = (double*)tmp[4];
    }
    const unsigned g = grid_for(n, 256);
    if (c)
        spmv_kernel<true><<<g, 256, 0, st>>>(rp, ci, va, n, cx<double>{alpha[0], alpha[1]}, xd, cx<double>{beta[0], beta[1]}, yd, ld, nrhs);
    else
        spmv_kernel<false><<<g, 256, 0, st>>>(rp, ci, va, n, alpha[0], xd, beta[0], yd, ld, nrhs);
    int rc = check_cuda("sparse_multiply");
    if (!on_device) {
        if (rc == CLIQ_OK && cudaMemcpyAsync(Y, yd, vec, cudaMemcpyDeviceToHost, st) != cudaSuccess) rc = check_cuda("copy Y");
        for (void* p : tmp) cudaFreeAsync(p, st);
        if (cudaStreamSynchronize(st) != cudaSuccess && rc == CLIQ_OK) rc = check_cuda("sparse_multiply sync");
    }
    return rc;
}
