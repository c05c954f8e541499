"""Generates tests/golden/ref_lapack.npz: outputs of the reference's own
LAPACK path -- ATL_getrf (getrfC / getrfR + getf2 + laswp), ATL_getrs,
ATL_potrf (potrfL / potrfU), ATL_potrs and ATL_geqrf (geqrr + geqr2 + larfg +
larft + larfb), compiled from the reference's sources by oracle/build_ref.sh
into oracle/_ref/libatlref_lapack.so over its C reference BLAS.

    sh oracle/build_ref.sh && python tests/golden/make_golden_lapack.py

Inputs are not stored: each case names a deterministic generator of the
oracle (ATL_gegen's LCG, pinned by tests/test_oracle.py, or the seeded
normal / SPD / LU-benchmark matrices) and its parameters, and the tests
regenerate them.  Cases: the testers' sanity sizes (makes/Make.bin: n = 167,
nrhs = 83; QR m <= 83, n <= 167), the benchmark matrix classes at small
sizes, wide and tall shapes, exact ties in the pivot search, a zero column
(getrf info), an indefinite leading minor (potrf info), row-major getrf, and
1 x n / m x 1 edges.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_lapack.npz")

# generator codes stored in the case headers
GEGEN, LU, SPD, NORMAL, TIES, ZEROCOL, NOTSPD = range(7)


def make_input(kind, m, n, seed, extra=0):
    """The case's input matrix (column-major), regenerated the same way by the tests."""
    if kind == GEGEN:
        return np.asfortranarray(O.gegen(m, n, max(m, 1), seed)[:m, :n])
    if kind == LU:
        return O.lu_matrix(n, seed)
    if kind == SPD:
        return O.spd_matrix(n, seed)
    if kind == NORMAL:
        return O.normal((m, n), seed)
    if kind == TIES:  # entries in {-2, ..., 2}: many exactly equal |values| in each column
        return np.asfortranarray(np.round(4.0 * O.gegen(m, n, m, seed)[:m, :n]))
    if kind == ZEROCOL:
        a = np.asfortranarray(O.gegen(m, n, m, seed)[:m, :n])
        a[:, extra] = 0.0
        return a
    if kind == NOTSPD:  # SPD except that the leading minor of order extra+1 is not positive
        a = O.spd_matrix(n, seed)
        a[extra, extra] = -1.0
        return a
    raise ValueError(kind)


GETRF = [  # (kind, m, n, seed, extra, order)
    (GEGEN, 167, 167, 1167, 0, 102), (GEGEN, 83, 167, 83, 0, 102), (GEGEN, 167, 83, 84, 0, 102),
    (GEGEN, 300, 40, 7, 0, 102), (LU, 160, 160, 42, 0, 102), (TIES, 64, 64, 5, 0, 102),
    (TIES, 100, 70, 6, 0, 102), (ZEROCOL, 60, 60, 9, 7, 102), (ZEROCOL, 40, 40, 10, 0, 102),
    (GEGEN, 1, 1, 3, 0, 102), (GEGEN, 5, 1, 4, 0, 102), (GEGEN, 1, 5, 5, 0, 102),
    (GEGEN, 2, 2, 6, 0, 102), (GEGEN, 67, 45, 77, 0, 101), (GEGEN, 45, 67, 78, 0, 101),
]
GETRS = [  # (getrf case index, trans, nrhs, seed)
    (0, 111, 83, 2001), (0, 112, 83, 2002), (4, 111, 16, 2003),
]
POTRF = [  # (kind, n, seed, extra, uplo)
    (SPD, 167, 31, 0, 121), (SPD, 167, 32, 0, 122), (SPD, 200, 33, 0, 122), (SPD, 1, 34, 0, 122),
    (NOTSPD, 50, 35, 12, 122), (NOTSPD, 50, 36, 0, 121),
]
POTRS = [  # (potrf case index, nrhs, seed)
    (0, 83, 3001), (1, 83, 3002),
]
GEQRF = [  # (kind, m, n, seed)
    (GEGEN, 83, 40, 401), (GEGEN, 167, 83, 402), (GEGEN, 40, 83, 403), (NORMAL, 200, 100, 404),
    (GEGEN, 1, 1, 405), (GEGEN, 8, 1, 406), (GEGEN, 1, 8, 407), (GEGEN, 150, 150, 408),
]


def main():
    if not O.ref_lapack_available():
        sys.exit("oracle/_ref/libatlref_lapack.so missing: run `sh oracle/build_ref.sh` first")
    cases = {}
    lus = []
    for i, (kind, m, n, seed, extra, order) in enumerate(GETRF):
        a = make_input(kind, m, n, seed, extra)
        lu, ipiv, info = O.ref_dgetrf(a, order)
        lus.append((lu, ipiv))
        cases[f"getrf{i}"] = np.array([kind, m, n, seed, extra, order, info])
        cases[f"getrf{i}_LU"], cases[f"getrf{i}_ipiv"] = lu, ipiv
    for i, (fi, trans, nrhs, seed) in enumerate(GETRS):
        lu, ipiv = lus[fi]
        b = O.uniform((lu.shape[0], nrhs), seed)
        cases[f"getrs{i}"] = np.array([fi, trans, nrhs, seed])
        cases[f"getrs{i}_X"] = O.ref_dgetrs(trans, lu, ipiv, b)
    fs = []
    for i, (kind, n, seed, extra, uplo) in enumerate(POTRF):
        a = make_input(kind, n, n, seed, extra)
        f, info = O.ref_dpotrf(uplo, a)
        fs.append((f, uplo))
        cases[f"potrf{i}"] = np.array([kind, n, seed, extra, uplo, info])
        cases[f"potrf{i}_F"] = np.triu(f) if uplo == 121 else np.tril(f)
    for i, (fi, nrhs, seed) in enumerate(POTRS):
        f, uplo = fs[fi]
        b = O.uniform((f.shape[0], nrhs), seed)
        cases[f"potrs{i}"] = np.array([fi, nrhs, seed])
        cases[f"potrs{i}_X"] = O.ref_dpotrs(uplo, f, b)
    for i, (kind, m, n, seed) in enumerate(GEQRF):
        a = make_input(kind, m, n, seed)
        qr, tau, info = O.ref_dgeqrf(a)
        cases[f"geqrf{i}"] = np.array([kind, m, n, seed, info])
        cases[f"geqrf{i}_QR"], cases[f"geqrf{i}_tau"] = qr, tau
    cases["counts"] = np.array([len(GETRF), len(GETRS), len(POTRF), len(POTRS), len(GEQRF)])
    np.savez_compressed(OUT, **cases)
    print(f"wrote {OUT}: {len(GETRF)} getrf, {len(GETRS)} getrs, {len(POTRF)} potrf, "
          f"{len(POTRS)} potrs, {len(GEQRF)} geqrf cases")


if __name__ == "__main__":
    main()
