// clique.hpp -- single-process drop-in for Clique's numeric API on one B200.
//
// Header-only C++ layer over the C ABI in cliqgpu.h.  The class and function
// names, argument order and error behaviour follow the reference:
//   DistSparseMatrix        include/clique/core/dist_sparse_matrix/decl.hpp:32-100
//   DistMultiVec            include/clique/core/dist_multi_vec/decl.hpp:20-64
//   DistMap                 include/clique/core/dist_map/decl.hpp:21-82
//   NaturalNestedDissection include/clique/symbolic/natural_nested_dissection.hpp:17-26
//   DistSymmFrontTree       include/clique/numeric/dist_symm_front_tree/decl.hpp:206-249
//   LDL                     include/clique/numeric/ldl.hpp:23-26
//   DistNodalMultiVec       include/clique/numeric/dist_nodal_multi_vec/decl.hpp:20-51
//   Solve                   include/clique/numeric/solve.hpp:17-20
//   Multiply                include/clique/numeric/multiply.hpp:18-21
// A program written against those headers for a single process compiles
// against this one after replacing `#include "clique.hpp"`.  Errors from the
// device are raised as LogicError / RuntimeError (std::logic_error /
// std::runtime_error), as El::LogicError / El::RuntimeError do.
//
// Scalar types: double and Complex<double> factor in FP64; float and
// Complex<float> factor in FP32 (values pass through the ABI as FP64).
// Multiply, LDL and Solve run on the device only.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../cliqgpu.h"

namespace cliq {

template <class T>
using Complex = std::complex<T>;

struct LogicError : std::logic_error {
    explicit LogicError(const std::string& s) : std::logic_error(s) {}
};
struct RuntimeError : std::runtime_error {
    explicit RuntimeError(const std::string& s) : std::runtime_error(s) {}
};

inline void Check(int status, const char* where) {
    if (status == CLIQ_OK) return;
    std::string msg = std::string(where) + ": " + cliqgpu_status_string(status);
    const char* d = cliqgpu_last_error();
    if (d && *d) msg += std::string(" (") + d + ")";
    if (status == CLIQ_ERR_ARG || status == CLIQ_ERR_STATE) throw LogicError(msg);
    throw RuntimeError(msg);
}

// ---- environment (one process, no MPI) -------------------------------------
namespace mpi {
struct Comm {};
static const Comm COMM_WORLD{};
inline int Rank(Comm = COMM_WORLD) { return 0; }
inline int Size(Comm = COMM_WORLD) { return 1; }
inline void Barrier(Comm = COMM_WORLD) {}
inline double Time() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}
}  // namespace mpi
inline void Initialize(int&, char**&) {}
inline void Finalize() {}
// El::SetBlocksize: accepted for source compatibility; the device kernels use 64.
inline void SetBlocksize(int) {}

template <class F> struct Traits { static constexpr bool complex = false; static constexpr bool single = false; };
template <> struct Traits<float> { static constexpr bool complex = false; static constexpr bool single = true; };
template <> struct Traits<Complex<double>> { static constexpr bool complex = true; static constexpr bool single = false; };
template <> struct Traits<Complex<float>> { static constexpr bool complex = true; static constexpr bool single = true; };

// ---- sparse matrix ---------------------------------------------------------
class DistGraph;
class DistGraph {
public:
    int NumSources() const { return n_; }
    const std::vector<int64_t>& RowPtr() const { return rowptr_; }
    const std::vector<int32_t>& ColInd() const { return colind_; }
    int n_ = 0;
    std::vector<int64_t> rowptr_;
    std::vector<int32_t> colind_;
};

template <class F>
class DistSparseMatrix {
public:
    DistSparseMatrix(int height, mpi::Comm = mpi::COMM_WORLD) { graph_.n_ = height; }
    int Height() const { return graph_.n_; }
    int FirstLocalRow() const { return 0; }
    int LocalHeight() const { return graph_.n_; }
    void StartAssembly() { tri_.clear(); assembling_ = true; }
    void Reserve(int cap) { tri_.reserve(cap); }
    void Update(int i, int j, F v) {
        if (!assembling_) throw LogicError("Update outside of assembly");
        tri_.push_back({i, j, v});
    }
    // sort and sum duplicates (core/dist_sparse_matrix/impl.hpp:209-257)
    void StopAssembly() {
        if (!assembling_) throw LogicError("Cannot stop assembly without starting");
        assembling_ = false;
        std::stable_sort(tri_.begin(), tri_.end(), [](const Trip& a, const Trip& b) {
            return a.i < b.i || (a.i == b.i && a.j < b.j);
        });
        const int n = graph_.n_;
        graph_.rowptr_.assign(n + 1, 0);
        graph_.colind_.clear();
        vals_.clear();
        for (size_t e = 0; e < tri_.size(); ++e) {
            if (!vals_.empty() && e > 0 && tri_[e].i == tri_[e - 1].i && tri_[e].j == tri_[e - 1].j) {
                vals_.back() += tri_[e].v;
                continue;
            }
            graph_.colind_.push_back(tri_[e].j);
            vals_.push_back(tri_[e].v);
            graph_.rowptr_[tri_[e].i + 1]++;
        }
        for (int i = 0; i < n; ++i) graph_.rowptr_[i + 1] += graph_.rowptr_[i];
        tri_.clear();
    }
    const ::cliq::DistGraph& LockedDistGraph() const { return graph_; }
    const ::cliq::DistGraph& DistGraph() const { return graph_; }
    const std::vector<F>& Values() const { return vals_; }

private:
    struct Trip { int i, j; F v; };
    ::cliq::DistGraph graph_;
    std::vector<Trip> tri_;
    std::vector<F> vals_;
    bool assembling_ = false;
};

// ---- dense multivector ------------------------------------------------------
template <class F>
class DistMultiVec {
public:
    DistMultiVec(int height = 0, int width = 1, mpi::Comm = mpi::COMM_WORLD) { Resize(height, width); }
    void Resize(int h, int w) { h_ = h; w_ = w; d_.assign((size_t)h * w, F(0)); }
    int Height() const { return h_; }
    int Width() const { return w_; }
    int LocalHeight() const { return h_; }
    int FirstLocalRow() const { return 0; }
    F GetLocal(int i, int j) const { return d_[i + (size_t)j * h_]; }
    void SetLocal(int i, int j, F v) { d_[i + (size_t)j * h_] = v; }
    void UpdateLocal(int i, int j, F v) { d_[i + (size_t)j * h_] += v; }
    F* Buffer() { return d_.data(); }
    const F* LockedBuffer() const { return d_.data(); }

private:
    int h_ = 0, w_ = 1;
    std::vector<F> d_;
};

template <class F>
void Zero(DistMultiVec<F>& X) {
    for (int j = 0; j < X.Width(); ++j)
        for (int i = 0; i < X.Height(); ++i) X.SetLocal(i, j, F(0));
}

// MakeUniform: entries drawn uniformly from the unit ball (El::SampleBall)
template <class F>
void MakeUniform(DistMultiVec<F>& X, unsigned seed = 0) {
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (int j = 0; j < X.Width(); ++j)
        for (int i = 0; i < X.Height(); ++i) {
            if constexpr (Traits<F>::complex) {
                const double r = std::sqrt(u(g)), t = 2 * M_PI * u(g);
                X.SetLocal(i, j, F(r * std::cos(t), r * std::sin(t)));
            } else {
                X.SetLocal(i, j, F(2 * u(g) - 1));
            }
        }
}

template <class F>
void Norms(const DistMultiVec<F>& X, std::vector<double>& norms) {
    norms.assign(X.Width(), 0.0);
    for (int j = 0; j < X.Width(); ++j) {
        double s = 0;
        for (int i = 0; i < X.Height(); ++i) s += std::norm(X.GetLocal(i, j));
        norms[j] = std::sqrt(s);
    }
}

// the one-column norm and Y := alpha X + Y (dist_multi_vec/decl.hpp:75-84)
template <class F>
double Norm(const DistMultiVec<F>& x) {
    std::vector<double> n;
    Norms(x, n);
    return n.empty() ? 0.0 : n[0];
}

template <class F>
void Axpy(F alpha, const DistMultiVec<F>& X, DistMultiVec<F>& Y) {
    if (X.Height() != Y.Height() || X.Width() != Y.Width()) throw LogicError("X and Y must be the same size");
    for (int j = 0; j < X.Width(); ++j)
        for (int i = 0; i < X.Height(); ++i) Y.SetLocal(i, j, Y.GetLocal(i, j) + alpha * X.GetLocal(i, j));
}

// Y := alpha A X + beta Y (multiply.hpp:28-166 at P=1), computed on the
// device by cliqgpu_sparse_multiply (host buffers staged through device
// memory; FP64 arithmetic for every scalar type)
template <class F>
void Multiply(F alpha, const DistSparseMatrix<F>& A, const DistMultiVec<F>& X, F beta, DistMultiVec<F>& Y) {
    using D = typename std::conditional<Traits<F>::complex, Complex<double>, double>::type;
    const auto& g = A.LockedDistGraph();
    const int n = g.n_, k = Y.Width();
    if (X.Height() != n || Y.Height() != n || X.Width() != k) throw LogicError("Multiply: nonconformal");
    std::vector<D> v(A.Values().begin(), A.Values().end());
    std::vector<D> x(X.LockedBuffer(), X.LockedBuffer() + (size_t)n * k), y(Y.LockedBuffer(), Y.LockedBuffer() + (size_t)n * k);
    const D a = D(alpha), b = D(beta);
    Check(cliqgpu_sparse_multiply(Traits<F>::complex ? CLIQ_COMPLEX : CLIQ_REAL, n, g.rowptr_.data(), g.colind_.data(),
                                  reinterpret_cast<const double*>(v.data()), reinterpret_cast<const double*>(&a),
                                  x.data(), reinterpret_cast<const double*>(&b), y.data(), n, k, 0, nullptr),
          "Multiply");
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < n; ++i) Y.SetLocal(i, j, F(y[i + (size_t)j * n]));
}

// ---- symbolic --------------------------------------------------------------
class DistMap {
public:
    std::vector<int32_t> map;
    int Translate(int i) const { return map[i]; }
    void FormInverse(DistMap& inv) const {
        inv.map.assign(map.size(), 0);
        for (size_t i = 0; i < map.size(); ++i) inv.map[map[i]] = (int32_t)i;
    }
};

struct SymmNodeInfo {
    int size, off, myOff, parent;
    std::vector<int> children;
    bool onLeft;
    std::vector<int> lowerStruct, origLowerStruct, origLowerRelInds, leftRelInds, rightRelInds;
};

class DistSymmInfo {
public:
    std::vector<SymmNodeInfo> localNodes;
    std::shared_ptr<std::remove_pointer<cliq_symbolic>::type> handle;
    cliq_symm_info view{};
};

class DistSeparatorTree {
public:
    std::vector<std::vector<int>> inds;   // natural indices of each separator / leaf (post-order)
};

// the symbolic handle's tree, analysis and map into the reference's containers
inline void FillSymbolic(cliq_symbolic h, int64_t n, DistMap& map, DistSeparatorTree& sepTree, DistSymmInfo& info) {
    info.handle.reset(h, cliq_symbolic_destroy);
    Check(cliq_symbolic_info(h, &info.view), "NaturalNestedDissection");
    const int nn = info.view.num_nodes;
    info.localNodes.assign(nn, SymmNodeInfo{});
    sepTree.inds.assign(nn, {});
    auto arr = [&](int s, int which, std::vector<int>& out) {
        int64_t len = 0;
        Check(cliq_symbolic_node_array(h, s, which, nullptr, &len), "NaturalNestedDissection");
        std::vector<int32_t> tmp(len);
        Check(cliq_symbolic_node_array(h, s, which, tmp.data(), &len), "NaturalNestedDissection");
        out.assign(tmp.begin(), tmp.end());
    };
    for (int s = 0; s < nn; ++s) {
        int32_t v[10];
        Check(cliq_symbolic_node(h, s, v), "NaturalNestedDissection");
        SymmNodeInfo& nd = info.localNodes[s];
        nd.size = v[0]; nd.off = v[1]; nd.myOff = v[2]; nd.parent = v[3];
        if (v[4] >= 0) nd.children = {v[4], v[5]};
        nd.onLeft = v[6] != 0;
        arr(s, 0, nd.lowerStruct); arr(s, 1, nd.origLowerStruct); arr(s, 2, nd.origLowerRelInds);
        arr(s, 3, nd.leftRelInds); arr(s, 4, nd.rightRelInds); arr(s, 5, sepTree.inds[s]);
    }
    map.map.assign(n, 0);
    Check(cliq_symbolic_map(h, map.map.data(), nullptr), "NaturalNestedDissection");
}

inline void NaturalNestedDissection(int nx, int ny, int nz, const DistGraph& graph, DistMap& map, DistSeparatorTree& sepTree,
                                    DistSymmInfo& info, int cutoff = 128, bool /*storeFactRecvInds*/ = false) {
    cliq_symbolic h = nullptr;
    Check(cliq_natural_nested_dissection(nx, ny, nz, graph.n_, graph.rowptr_.data(), graph.colind_.data(), cutoff, &h),
          "NaturalNestedDissection");
    FillSymbolic(h, graph.n_, map, sepTree, info);
}

// nested_dissection.hpp:35-44 at one process: general graphs, this library's
// own bisection in place of METIS (numSeqSeps start vertices tried)
inline void NestedDissection(const DistGraph& graph, DistMap& map, DistSeparatorTree& sepTree, DistSymmInfo& info,
                             bool /*sequential*/ = true, int /*numDistSeps*/ = 1, int numSeqSeps = 1, int cutoff = 128,
                             bool /*storeFactRecvInds*/ = false) {
    cliq_symbolic h = nullptr;
    Check(cliq_nested_dissection(graph.n_, graph.rowptr_.data(), graph.colind_.data(), cutoff, numSeqSeps, &h),
          "NestedDissection");
    FillSymbolic(h, graph.n_, map, sepTree, info);
}

// ---- numeric ---------------------------------------------------------------
// the reference's enum (dist_symm_front_tree/decl.hpp:17-26), same order
enum SymmFrontType {
    SYMM_1D, SYMM_2D, LDL_1D, LDL_2D, LDL_SELINV_1D, LDL_SELINV_2D, LDL_INTRAPIV_1D, LDL_INTRAPIV_2D,
    LDL_INTRAPIV_SELINV_1D, LDL_INTRAPIV_SELINV_2D, BLOCK_LDL_1D, BLOCK_LDL_2D, BLOCK_LDL_INTRAPIV_1D, BLOCK_LDL_INTRAPIV_2D
};
inline bool Unfactored(SymmFrontType t) { return t == SYMM_1D || t == SYMM_2D; }
// front types this library factors: every factored type.  The
// selective-inversion forms invert no local front at one process
// (change_front_type.hpp:86-98 inverts distributed nodes 1 .. only), so they
// factor and solve as their LDL / pivoted LDL base types.
inline bool PivotedFactorization(SymmFrontType t) {
    return t == LDL_INTRAPIV_1D || t == LDL_INTRAPIV_2D || t == LDL_INTRAPIV_SELINV_1D || t == LDL_INTRAPIV_SELINV_2D ||
           t == BLOCK_LDL_INTRAPIV_1D || t == BLOCK_LDL_INTRAPIV_2D;
}
inline bool BlockFactorization(SymmFrontType t) {
    return t == BLOCK_LDL_1D || t == BLOCK_LDL_2D || t == BLOCK_LDL_INTRAPIV_1D || t == BLOCK_LDL_INTRAPIV_2D;
}
inline bool FrontsAre1d(SymmFrontType t) { return ((int)t & 1) == 0; }
inline bool SelInvFactorization(SymmFrontType t) {
    return t == LDL_SELINV_1D || t == LDL_SELINV_2D || t == LDL_INTRAPIV_SELINV_1D || t == LDL_INTRAPIV_SELINV_2D;
}
// the 1D / 2D members of a family are adjacent in the enum (1D even, 2D odd)
inline SymmFrontType ConvertTo2d(SymmFrontType t) { return (SymmFrontType)((int)t | 1); }
inline SymmFrontType ConvertTo1d(SymmFrontType t) { return (SymmFrontType)((int)t & ~1); }
inline SymmFrontType AppendSelInv(SymmFrontType t) {
    switch (t) {
        case LDL_1D: return LDL_SELINV_1D;
        case LDL_2D: return LDL_SELINV_2D;
        case LDL_INTRAPIV_1D: return LDL_INTRAPIV_SELINV_1D;
        case LDL_INTRAPIV_2D: return LDL_INTRAPIV_SELINV_2D;
        default: throw LogicError("Sel-inv does not make sense for this type");
    }
}
inline SymmFrontType RemoveSelInv(SymmFrontType t) {
    switch (t) {
        case LDL_SELINV_1D: return LDL_1D;
        case LDL_SELINV_2D: return LDL_2D;
        case LDL_INTRAPIV_SELINV_1D: return LDL_INTRAPIV_1D;
        case LDL_INTRAPIV_SELINV_2D: return LDL_INTRAPIV_2D;
        default: throw LogicError("This type did not involve selective inversion");
    }
}
inline bool Provided(SymmFrontType t) {
    return t == LDL_1D || t == LDL_2D || t == LDL_SELINV_1D || t == LDL_SELINV_2D || t == BLOCK_LDL_1D || t == BLOCK_LDL_2D ||
           PivotedFactorization(t);
}

template <class F>
class DistSymmFrontTree {
public:
    bool isHermitian = false;
    SymmFrontType frontType = SYMM_2D;

    DistSymmFrontTree(const DistSparseMatrix<F>& A, const DistMap& map, const DistSeparatorTree&, const DistSymmInfo& info,
                      bool conjugate = false)
        : isHermitian(conjugate), n_(A.Height()) {
        cliqgpu_options opt{Traits<F>::complex ? CLIQ_COMPLEX : CLIQ_REAL, Traits<F>::single ? CLIQ_FP32 : CLIQ_FP64,
                            conjugate ? 1 : 0, 0, 1};
        const auto& g = A.LockedDistGraph();
        cliqgpu_plan p = nullptr;
        Check(cliqgpu_plan_create(&info.view, n_, map.map.data(), g.rowptr_.data(), g.colind_.data(), &opt, nullptr, &p),
              "DistSymmFrontTree");
        plan_.reset(p, cliqgpu_plan_destroy);
        Initialize(A);
    }
    void Initialize(const DistSparseMatrix<F>& A) {
        const auto& v = A.Values();
        if constexpr (Traits<F>::complex) {
            std::vector<std::complex<double>> w(v.begin(), v.end());
            Check(cliqgpu_assemble(plan_.get(), w.data(), 0), "DistSymmFrontTree::Initialize");
        } else {
            std::vector<double> w(v.begin(), v.end());
            Check(cliqgpu_assemble(plan_.get(), w.data(), 0), "DistSymmFrontTree::Initialize");
        }
        frontType = SYMM_2D;
    }
    // FactorizationWork / SolveWork (dist_symm_front_tree/impl.hpp:542-640), P = 1
    void FactorizationWork(double& local, double& mn, double& mx, double& global, bool = false) const {
        cliqgpu_plan_query(plan_.get(), 0, &local);
        mn = mx = global = local;
    }
    void SolveWork(double& local, double& mn, double& mx, double& global, int numRhs = 1) const {
        cliqgpu_plan_query(plan_.get(), 1, &local);
        local *= numRhs;
        mn = mx = global = local;
    }
    cliqgpu_plan Plan() const { return plan_.get(); }
    int Height() const { return n_; }

private:
    std::shared_ptr<std::remove_pointer<cliqgpu_plan>::type> plan_;
    int n_;
};

template <class F>
void LDL(DistSymmInfo&, DistSymmFrontTree<F>& L, SymmFrontType newFrontType = LDL_2D) {
    if (!Unfactored(L.frontType)) throw LogicError("Matrix is already factored");
    if (!Provided(newFrontType))
        throw LogicError("The symmetric (unfactored) front types are no factorization");
    int64_t zp = -1;
    if (PivotedFactorization(newFrontType)) Check(cliqgpu_factor_intrapiv(L.Plan(), &zp), "LDL");
    else Check(cliqgpu_factor(L.Plan(), &zp), "LDL");
    L.frontType = newFrontType;
    if (BlockFactorization(newFrontType)) Check(cliqgpu_block_ldl(L.Plan()), "LDL (block form)");
}

template <class F>
class DistNodalMultiVec {
public:
    std::vector<F> data;   // ND-ordered, n x width column-major
    DistNodalMultiVec() = default;
    DistNodalMultiVec(const DistMap& inverseMap, const DistSymmInfo& info, const DistMultiVec<F>& X) { Pull(inverseMap, info, X); }
    // Pull / Push at P=1 (dist_nodal_multi_vec/impl.hpp:67-219)
    void Pull(const DistMap& inverseMap, const DistSymmInfo&, const DistMultiVec<F>& X) {
        h_ = X.Height(); w_ = X.Width();
        data.assign((size_t)h_ * w_, F(0));
        for (int j = 0; j < w_; ++j)
            for (int p = 0; p < h_; ++p) data[p + (size_t)j * h_] = X.GetLocal(inverseMap.map[p], j);
    }
    void Push(const DistMap& inverseMap, const DistSymmInfo&, DistMultiVec<F>& X) const {
        for (int j = 0; j < w_; ++j)
            for (int p = 0; p < h_; ++p) X.SetLocal(inverseMap.map[p], j, data[p + (size_t)j * h_]);
    }
    int Height() const { return h_; }
    int Width() const { return w_; }

private:
    int h_ = 0, w_ = 0;
};

template <class F>
void Solve(const DistSymmInfo&, const DistSymmFrontTree<F>& L, DistNodalMultiVec<F>& X) {
    if (!Provided(L.frontType)) throw LogicError("Invalid front type for solve");
    const int n = X.Height(), w = X.Width();
    if constexpr (std::is_same<F, double>::value || std::is_same<F, Complex<double>>::value) {
        Check(cliqgpu_solve(L.Plan(), X.data.data(), n, w, 0, 1), "Solve");
    } else {
        using D = typename std::conditional<Traits<F>::complex, std::complex<double>, double>::type;
        std::vector<D> tmp(X.data.begin(), X.data.end());
        Check(cliqgpu_solve(L.Plan(), tmp.data(), n, w, 0, 1), "Solve");
        for (size_t i = 0; i < tmp.size(); ++i) X.data[i] = F(tmp[i]);
    }
}

// ChangeFrontType (change_front_type.hpp:27-107) at one process: 1D <-> 2D
// and appending selective inversion (applied by the reference to distributed
// fronts 1 .. only) leave the device fronts as they are and relabel the tree
template <class F>
void ChangeFrontType(DistSymmFrontTree<F>& L, SymmFrontType frontType) {
    if (frontType == L.frontType) return;
    const SymmFrontType old = L.frontType;
    if (frontType == ConvertTo2d(old) || frontType == ConvertTo1d(old)) {
        L.frontType = frontType;
        return;
    }
    if (SelInvFactorization(frontType) &&
        (old == LDL_1D || old == LDL_2D || old == LDL_INTRAPIV_1D || old == LDL_INTRAPIV_2D) &&
        ConvertTo2d(frontType) == ConvertTo2d(AppendSelInv(old))) {
        L.frontType = frontType;
        return;
    }
    throw LogicError("Unavailable front type change");
}

// DistNodalMatrix (dist_nodal_matrix/decl.hpp:19-50): the [MC,MR] nodal
// matrix of the reference; at one process its nodes hold the same blocks as
// a DistNodalMultiVec, so it is one, with the reference's constructors
template <class F>
class DistNodalMatrix : public DistNodalMultiVec<F> {
public:
    DistNodalMatrix() = default;
    DistNodalMatrix(const DistMap& inverseMap, const DistSymmInfo& info, const DistMultiVec<F>& X)
        : DistNodalMultiVec<F>(inverseMap, info, X) {}
    explicit DistNodalMatrix(const DistNodalMultiVec<F>& X) : DistNodalMultiVec<F>(X) {}
    const DistNodalMatrix<F>& operator=(const DistNodalMultiVec<F>& X) {
        DistNodalMultiVec<F>::operator=(X);
        return *this;
    }
};

// the DistNodalMatrix overload of Solve (solve.hpp:21-24)
template <class F>
void Solve(const DistSymmInfo& info, const DistSymmFrontTree<F>& L, DistNodalMatrix<F>& X) {
    Solve(info, L, static_cast<DistNodalMultiVec<F>&>(X));
}

// Black-box solves (solve.hpp:95-140 at one process): nested dissection of
// A's graph, the front tree, LDL with intra-front pivoting (LDL_INTRAPIV_1D),
// Pull / Solve / Push; X is overwritten with the solution
template <class F>
void SymmetricSolve(const DistSparseMatrix<F>& A, DistMultiVec<F>& X, bool conjugate = false, bool sequential = true,
                    int numDistSeps = 1, int numSeqSeps = 1, int cutoff = 128) {
    DistSymmInfo info;
    DistSeparatorTree sepTree;
    DistMap map, inverseMap;
    NestedDissection(A.LockedDistGraph(), map, sepTree, info, sequential, numDistSeps, numSeqSeps, cutoff);
    map.FormInverse(inverseMap);
    DistSymmFrontTree<F> frontTree(A, map, sepTree, info, conjugate);
    LDL(info, frontTree, LDL_INTRAPIV_1D);
    DistNodalMultiVec<F> XNodal;
    XNodal.Pull(inverseMap, info, X);
    Solve(info, frontTree, XNodal);
    XNodal.Push(inverseMap, info, X);
}

template <class F>
void HermitianSolve(const DistSparseMatrix<F>& A, DistMultiVec<F>& X, bool sequential = true, int numDistSeps = 1,
                    int numSeqSeps = 1, int cutoff = 128) {
    SymmetricSolve(A, X, true, sequential, numDistSeps, numSeqSeps, cutoff);
}

}  // namespace cliq
