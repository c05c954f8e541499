"""Generates tests/golden/ref_blas.npz: outputs of the reference's own C
reference BLAS (ATL_dref*/ATL_sref*, compiled unmodified into oracle/_ref/
by oracle/build_ref.sh) on the inputs its tester bin/l3blastst.c builds
(ATL_gegen with the tester's seeds, trddom triangles, poisoned lda gaps).

    python tests/golden/make_golden.py

Needs oracle/_ref/libatlref.so (so the reference sources) at generation time
only; the committed .npz is what the tests read.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_blas.npz")


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/libatlref.so missing: run `make -C oracle ref` first")
    R = O.ref()
    P = O.P
    cases = {}
    # GEMM: (M, N, K), all transposes, alpha/beta as in the tester's defaults
    gi = 0
    for (m, n, k) in [(1, 1, 1), (7, 5, 3), (33, 17, 29), (45, 38, 52)]:
        for ta in (O.NoTrans, O.Trans):
            for tb in (O.NoTrans, O.Trans):
                for alpha, beta in ((1.0, 0.0), (-0.7, 1.3)):
                    ma, na = (m, k) if ta == O.NoTrans else (k, m)
                    mb, nb = (k, n) if tb == O.NoTrans else (n, k)
                    sa, sb, sc = O.tester_seeds(ma, na, mb, nb, m, n)
                    a = O.gegen(ma, na, ma + 3, sa)
                    b = O.gegen(mb, nb, mb + 2, sb)
                    c = O.gegen(m, n, m + 1, sc)
                    c0 = c.copy(order="F")
                    R.ATL_drefgemm(ta, tb, m, n, k, alpha, P(a), a.shape[0], P(b), b.shape[0],
                                   beta, P(c), c.shape[0])
                    cases[f"gemm{gi}"] = np.array([m, n, k, ta, tb, alpha, beta])
                    cases[f"gemm{gi}_A"], cases[f"gemm{gi}_B"] = a, b
                    cases[f"gemm{gi}_C0"], cases[f"gemm{gi}_C"] = c0, c
                    gi += 1
    # TRSM / TRMM: every side/uplo/trans/diag
    ti = 0
    for (m, n) in [(5, 3), (37, 21), (70, 9)]:
        for side in (O.Left, O.Right):
            for uplo in (O.Upper, O.Lower):
                for ta in (O.NoTrans, O.Trans):
                    for diag in (O.NonUnit, O.Unit):
                        na = m if side == O.Left else n
                        sa, sb, _ = O.tester_seeds(na, na, m, n, m, n)
                        a = O.gegen(na, na, na + 2, sa)
                        O.trddom(uplo, a, na)
                        b = O.gegen(m, n, m + 3, sb)
                        b0 = b.copy(order="F")
                        alpha = 0.9
                        R.ATL_dreftrsm(side, uplo, ta, diag, m, n, alpha, P(a), a.shape[0], P(b), b.shape[0])
                        bm = b0.copy(order="F")
                        R.ATL_dreftrmm(side, uplo, ta, diag, m, n, alpha, P(a), a.shape[0], P(bm), bm.shape[0])
                        cases[f"trsm{ti}"] = np.array([m, n, side, uplo, ta, diag, alpha])
                        cases[f"trsm{ti}_A"], cases[f"trsm{ti}_B0"] = a, b0
                        cases[f"trsm{ti}_X"], cases[f"trsm{ti}_TB"] = b, bm
                        ti += 1
    # SYRK
    si = 0
    for (n, k) in [(6, 3), (33, 47), (65, 20)]:
        for uplo in (O.Upper, O.Lower):
            for tr in (O.NoTrans, O.Trans):
                ma, na = (n, k) if tr == O.NoTrans else (k, n)
                sa, _, sc = O.tester_seeds(ma, na, 0, 0, n, n)
                a = O.gegen(ma, na, ma + 1, sa)
                c = O.gegen(n, n, n + 2, sc)
                c0 = c.copy(order="F")
                alpha, beta = 1.1, -0.5
                R.ATL_drefsyrk(uplo, tr, n, k, alpha, P(a), a.shape[0], beta, P(c), c.shape[0])
                cases[f"syrk{si}"] = np.array([n, k, uplo, tr, alpha, beta])
                cases[f"syrk{si}_A"], cases[f"syrk{si}_C0"], cases[f"syrk{si}_C"] = a, c0, c
                si += 1
    cases["counts"] = np.array([gi, ti, si])
    np.savez_compressed(OUT, **cases)
    print(f"wrote {OUT}: {gi} gemm, {ti} trsm/trmm, {si} syrk cases")


if __name__ == "__main__":
    main()
