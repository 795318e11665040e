// The flow of the reference's tests/Solve.cpp written against the drop-in
// header: 3D 7-point Laplacian (diagonal 6 + shift), manufactured solution
// X, Y := A X, natural nested dissection, front tree, LDL, Pull / Solve /
// Push, and the error || X - X_hat || / || X || per right-hand side.  The
// last case shifts the diagonal to 0.5 (indefinite) and factors with
// intra-front pivoting (LDL_INTRAPIV_1D, the front type of the reference's
// SymmetricSolve).  Exit status 0 when every error is below the tolerance.
#include <cstdio>
#include <cstdlib>

#include "clique_b200/clique.hpp"

using namespace cliq;

template <class F>
int run(int n1, int n2, int n3, int numRhs, int cutoff, double shift, double tol, SymmFrontType ft = LDL_2D) {
    const int N = n1 * n2 * n3;
    DistSparseMatrix<F> A(N, mpi::COMM_WORLD);
    A.StartAssembly();
    A.Reserve(7 * N);
    for (int i = 0; i < N; ++i) {
        const int x = i % n1, y = (i / n1) % n2, z = i / (n1 * n2);
        A.Update(i, i, F(6. + shift));
        if (x != 0) A.Update(i, i - 1, F(-1));
        if (x != n1 - 1) A.Update(i, i + 1, F(-1));
        if (y != 0) A.Update(i, i - n1, F(-1));
        if (y != n2 - 1) A.Update(i, i + n1, F(-1));
        if (z != 0) A.Update(i, i - n1 * n2, F(-1));
        if (z != n3 - 1) A.Update(i, i + n1 * n2, F(-1));
    }
    A.StopAssembly();
    DistMultiVec<F> X(N, numRhs), Y(N, numRhs);
    MakeUniform(X, 7);
    Zero(Y);
    Multiply(F(1), A, X, F(0), Y);

    DistSymmInfo info;
    DistSeparatorTree sepTree;
    DistMap map, inverseMap;
    NaturalNestedDissection(n1, n2, n3, A.DistGraph(), map, sepTree, info, cutoff);
    map.FormInverse(inverseMap);
    DistSymmFrontTree<F> frontTree(A, map, sepTree, info, false);
    const double t0 = mpi::Time();
    LDL(info, frontTree, ft);
    const double t1 = mpi::Time();
    DistNodalMultiVec<F> YNodal;
    YNodal.Pull(inverseMap, info, Y);
    if (numRhs > 3) {   // the DistNodalMatrix overload (solve.hpp:21-24)
        DistNodalMatrix<F> YMat(YNodal);
        Solve(info, frontTree, YMat);
        YMat.Push(inverseMap, info, Y);
    } else {
        Solve(info, frontTree, YNodal);
        YNodal.Push(inverseMap, info, Y);
    }
    const double t2 = mpi::Time();
    double local, mn, mx, flops;
    frontTree.FactorizationWork(local, mn, mx, flops);
    std::printf("N=%d fronts=%zu factor %.3f s (%.1f GFlop/s) solve %.3f s\n", N, info.localNodes.size(), t1 - t0,
                flops / (t1 - t0) / 1e9, t2 - t1);
    int bad = 0;
    for (int j = 0; j < numRhs; ++j) {
        double e = 0, x = 0;
        for (int i = 0; i < N; ++i) {
            e += std::norm(Y.GetLocal(i, j) - X.GetLocal(i, j));
            x += std::norm(X.GetLocal(i, j));
        }
        const double rel = std::sqrt(e / x);
        std::printf("||X - X_hat|| / ||X|| (rhs %d) = %.3e\n", j, rel);
        if (!(rel <= tol)) bad = 1;
    }
    // a second LDL on the factored tree is a logic error, as in the reference
    try {
        LDL(info, frontTree, LDL_2D);
        std::printf("missing LogicError\n");
        bad = 1;
    } catch (const LogicError&) {
    }
    return bad;
}

// the black-box solve (solve.hpp:95-116): nested dissection of A's graph and
// pivoted fronts; HermitianSolve on a Hermitian indefinite operator
template <class F>
int run_blackbox(int n1, int n2, int n3, double shift, double tol, bool hermitian) {
    const int N = n1 * n2 * n3;
    DistSparseMatrix<F> A(N, mpi::COMM_WORLD);
    A.StartAssembly();
    A.Reserve(7 * N);
    F up = F(-1), down = F(-1);   // x couplings: conjugate pair for the Hermitian operator
    if constexpr (Traits<F>::complex) {
        if (hermitian) { up = F(-0.8, -0.6); down = F(-0.8, 0.6); }
    }
    for (int i = 0; i < N; ++i) {
        const int x = i % n1, y = (i / n1) % n2, z = i / (n1 * n2);
        A.Update(i, i, F(6. + shift));
        if (x != 0) A.Update(i, i - 1, down);
        if (x != n1 - 1) A.Update(i, i + 1, up);
        if (y != 0) A.Update(i, i - n1, F(-1));
        if (y != n2 - 1) A.Update(i, i + n1, F(-1));
        if (z != 0) A.Update(i, i - n1 * n2, F(-1));
        if (z != n3 - 1) A.Update(i, i + n1 * n2, F(-1));
    }
    A.StopAssembly();
    DistMultiVec<F> X(N, 2), Y(N, 2);
    MakeUniform(X, 11);
    Zero(Y);
    Multiply(F(1), A, X, F(0), Y);
    if (hermitian) HermitianSolve(A, Y);
    else SymmetricSolve(A, Y);
    // the reference's tests/SimpleSolve.cpp check: || X - Y || / || X || per column
    std::vector<double> xn, en;
    Norms(X, xn);
    Axpy(F(-1), X, Y);
    Norms(Y, en);
    int bad = 0;
    for (int j = 0; j < 2; ++j) {
        const double rel = en[j] / xn[j];
        std::printf("%s ||X - X_hat|| / ||X|| (rhs %d) = %.3e\n", hermitian ? "HermitianSolve" : "SymmetricSolve", j, rel);
        if (!(rel <= tol)) bad = 1;
    }
    return bad;
}

int main(int argc, char* argv[]) {
    Initialize(argc, argv);
    const int n = argc > 1 ? std::atoi(argv[1]) : 30;
    int rc = 0;
    try {
        rc |= run<double>(n, n, n, 5, 128, 0.1, 1e-10);
        rc |= run<Complex<double>>(n / 2 + 3, n / 2, n / 2 + 1, 3, 64, 0.1, 1e-10);
        rc |= run<float>(n / 2, n / 2, n / 2, 2, 64, 0.1, 1e-4);
        rc |= run<double>(n / 2 + 2, n / 2 + 1, n / 2, 3, 64, -5.5, 1e-9, LDL_INTRAPIV_1D);
        rc |= run_blackbox<double>(n / 2, n / 2 + 1, n / 2 + 2, -5.5, 1e-9, false);
        rc |= run_blackbox<Complex<double>>(n / 2, n / 2, n / 2 + 1, -5.5, 1e-9, true);
    } catch (const std::exception& e) {
        std::printf("exception: %s\n", e.what());
        rc = 1;
    }
    Finalize();
    return rc;
}
