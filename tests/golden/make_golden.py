"""Generate the numeric golden fixtures under tests/golden/.

Each fixture holds a small matrix (CSR), a nested-dissection map, and the
dense unpivoted LDL^T factors of the permuted matrix computed here with plain
numpy loops -- an answer independent of any multifrontal code.  The
multifrontal factor must reproduce these entries (front rows x front columns)
and D exactly up to rounding.  Maps: the 3x3x1 case uses the hand-derived map
of nd_known_answers.json; the 6x5x4 case uses the CPU oracle's ordering
(which tests/test_oracle.py pins against the hand-derived cases).

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from clique_b200 import operators as ops  # noqa: E402


def dense_ldl(A, conjugate=False):
    A = np.array(A, dtype=A.dtype, copy=True)
    n = A.shape[0]
    for j in range(n):
        d = A[j, j]
        col = A[j + 1:, j].copy()
        A[j + 1:, j] = col / d
        s = np.conj(col) if conjugate else col
        A[j + 1:, j + 1:] -= np.outer(A[j + 1:, j], s)
    D = np.diag(A).copy()
    L = np.tril(A, -1) + np.eye(n, dtype=A.dtype)
    return L, D


def save(name, csr, nd_map, conjugate=False, seed=0):
    Ad = csr.to_scipy().toarray()
    inv = np.empty_like(nd_map)
    inv[nd_map] = np.arange(len(nd_map))
    Ap = Ad[np.ix_(inv, inv)]
    L, D = dense_ldl(Ap, conjugate)
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(csr.n)
    if np.iscomplexobj(Ad):
        b = b + 1j * rng.standard_normal(csr.n)
    x = np.linalg.solve(Ad, b)
    np.savez(os.path.join(HERE, name), rowptr=csr.rowptr, colind=csr.colind, values=csr.values, map=nd_map,
             L=L, D=D, b=b, x=x, conjugate=conjugate)


def main():
    ka = json.load(open(os.path.join(HERE, "nd_known_answers.json")))
    case = [c for c in ka["cases"] if c["grid"] == [3, 3, 1]][0]
    m331 = np.array(case["map"], np.int32)
    save("ldl_lap_3x3x1.npz", ops.laplacian_3d(3, 3, 1, 6.1), m331)
    save("ldl_helm_3x3x1.npz", ops.helmholtz_pml_3d(3, 3, 1, omega=9.0, b=2), m331)
    from oracle import oracle as O
    A = ops.laplacian_3d(6, 5, 4, 6.1)
    S = O.Symbolic(6, 5, 4, A.rowptr, A.colind, cutoff=8)
    save("ldl_lap_6x5x4_c8.npz", A, S.map.copy())
    H = ops.helmholtz_pml_3d(6, 5, 4, omega=12.0, velocity=ops.smooth_velocity((6, 5, 4), 3), b=2)
    save("ldl_helm_6x5x4_c8.npz", H, S.map.copy())


if __name__ == "__main__":
    main()
