"""Access to tests/golden/ref_lapack.npz (outputs of the reference's own
LAPACK, see tests/golden/make_golden_lapack.py) for the oracle's CPU tests
and the GPU parity tests: the stored outputs plus the regenerated inputs."""
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "ref_lapack.npz")

_spec = importlib.util.spec_from_file_location("make_golden_lapack",
                                               os.path.join(HERE, "golden", "make_golden_lapack.py"))
gen = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(gen)

_gold = None


def gold():
    global _gold
    if _gold is None:
        _gold = np.load(GOLD)
    return _gold


def getrf_cases():
    """(index, input A (column-major logical matrix), order, LU (logical), ipiv, info)."""
    g = gold()
    out = []
    for i in range(int(g["counts"][0])):
        kind, m, n, seed, extra, order, info = (int(v) for v in g[f"getrf{i}"])
        a = gen.make_input(kind, m, n, seed, extra)
        out.append((i, a, order, g[f"getrf{i}_LU"], g[f"getrf{i}_ipiv"], info))
    return out


def getrs_cases():
    """(index, getrf case index, trans, B, X)."""
    g = gold()
    out = []
    for i in range(int(g["counts"][1])):
        fi, trans, nrhs, seed = (int(v) for v in g[f"getrs{i}"])
        n = int(g[f"getrf{fi}"][1])
        b = gen.O.uniform((n, nrhs), seed)
        out.append((i, fi, trans, b, g[f"getrs{i}_X"]))
    return out


def potrf_cases():
    """(index, input A, uplo, factor triangle, info)."""
    g = gold()
    out = []
    for i in range(int(g["counts"][2])):
        kind, n, seed, extra, uplo, info = (int(v) for v in g[f"potrf{i}"])
        a = gen.make_input(kind, n, n, seed, extra)
        out.append((i, a, uplo, g[f"potrf{i}_F"], info))
    return out


def potrs_cases():
    """(index, potrf case index, B, X)."""
    g = gold()
    out = []
    for i in range(int(g["counts"][3])):
        fi, nrhs, seed = (int(v) for v in g[f"potrs{i}"])
        n = int(g[f"potrf{fi}"][1])
        b = gen.O.uniform((n, nrhs), seed)
        out.append((i, fi, b, g[f"potrs{i}_X"]))
    return out


def geqrf_cases():
    """(index, input A, QR, tau, info)."""
    g = gold()
    out = []
    for i in range(int(g["counts"][4])):
        kind, m, n, seed, info = (int(v) for v in g[f"geqrf{i}"])
        a = gen.make_input(kind, m, n, seed)
        out.append((i, a, g[f"geqrf{i}_QR"], g[f"geqrf{i}_tau"], info))
    return out


def tri(f, uplo):
    return np.triu(f) if uplo == 121 else np.tril(f)


def close(x, y, rel=1e-11):
    """max |x - y| <= rel * max(1, max |y|) (factors of the same pivots in a
    different summation order)."""
    x = np.asarray(x)
    y = np.asarray(y)
    if x.size == 0:
        return True
    return float(np.max(np.abs(x - y))) <= rel * max(1.0, float(np.max(np.abs(y))))
