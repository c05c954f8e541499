"""atlas_b200 -- B200 (sm_100a) implementation of ATLAS's dense level-3 BLAS /
LAPACK hot path, behind the reference's C API.

The product is the shared library ``libatlas_b200.so`` (built in-tree by
``python -m atlas_b200.build``) whose C ABI is declared in
``include/atlas_b200.h``.  This module loads it with ctypes and mirrors the
reference's C calls one to one (same names, argument order and meaning,
same return codes) so that Python callers -- and the tests -- use exactly the
entry points a C program links against.  Array arguments may be numpy arrays
(host memory), torch tensors (host or CUDA), or raw integer addresses.

There is no CPU fallback: if the library is missing, importing the calls
raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libatlas_b200.so")

# CBLAS enums (include/cblas.h:5-10 of the reference)
CblasRowMajor, CblasColMajor = 101, 102
CblasNoTrans, CblasTrans, CblasConjTrans = 111, 112, 113
CblasUpper, CblasLower = 121, 122
CblasNonUnit, CblasUnit = 131, 132
CblasLeft, CblasRight = 141, 142

# factor precisions of the mixed-precision solvers
PREC_FP32, PREC_TF32, PREC_BF16, PREC_TF32X3 = 0, 1, 2, 3

_lib = None

_I, _D, _F, _P = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p
_S = ctypes.c_char_p

# name -> (restype, argtypes)
_SIGS = {
    "cblas_dgemm": (None, [_I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I]),
    "cblas_sgemm": (None, [_I, _I, _I, _I, _I, _I, _F, _P, _I, _P, _I, _F, _P, _I]),
    "cblas_dtrsm": (None, [_I, _I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I]),
    "cblas_dtrmm": (None, [_I, _I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I]),
    "cblas_dsyrk": (None, [_I, _I, _I, _I, _I, _D, _P, _I, _D, _P, _I]),
    "clapack_dgetrf": (_I, [_I, _I, _I, _P, _I, _P]),
    "clapack_dgetrs": (_I, [_I, _I, _I, _I, _P, _I, _P, _P, _I]),
    "clapack_dgesv": (_I, [_I, _I, _I, _P, _I, _P, _P, _I]),
    "clapack_dpotrf": (_I, [_I, _I, _I, _P, _I]),
    "clapack_dpotrs": (_I, [_I, _I, _I, _I, _P, _I, _P, _I]),
    "clapack_dposv": (_I, [_I, _I, _I, _I, _P, _I, _P, _I]),
    "clapack_dgeqrf": (_I, [_I, _I, _I, _P, _I, _P]),
    "ATL_dgeqrf": (_I, [_I, _I, _P, _I, _P, _P, _I]),
    "atlb_init": (_I, [_I]),
    "atlb_set_error_mode": (None, [_I]),
    "atlb_get_error_mode": (_I, []),
    "atlb_last_error": (_I, []),
    "atlb_last_cuda_error": (_I, []),
    "atlb_get_stream": (_P, []),
    "atlb_set_stream": (None, [_P]),
    "atlb_sync": (_I, []),
    "atlb_dgemm_dev": (_I, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I]),
    "atlb_sgemm_dev": (_I, [_I, _I, _I, _I, _I, _F, _P, _I, _P, _I, _F, _P, _I]),
    "atlb_sgemm_tc_dev": (_I, [_I, _I, _I, _I, _I, _I, _F, _P, _I, _P, _I, _F, _P, _I]),
    "atlb_dtrsm_dev": (_I, [_I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I]),
    "atlb_dtrsm_dev_noalloc": (_I, [_I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I]),
    "atlb_tune_get": (_I, [_S]),
    "atlb_tune_set": (_I, [_S, _I]),
    "atlb_tune_load": (_I, [_S]),
    "atlb_tune_count": (_I, []),
    "atlb_tune_name": (_S, [_I]),
    "atlb_dsyrk_dev": (_I, [_I, _I, _I, _I, _D, _P, _I, _D, _P, _I]),
    "atlb_dgetrf_dev": (_I, [_I, _I, _P, _I, _P, _P]),
    "atlb_sgetrf_dev": (_I, [_I, _I, _P, _I, _P, _P, _I]),
    "atlb_dgetrs_dev": (_I, [_I, _I, _I, _P, _I, _P, _P, _I]),
    "atlb_dpotrf_dev": (_I, [_I, _I, _P, _I, _P]),
    "atlb_dpotrs_dev": (_I, [_I, _I, _I, _P, _I, _P, _I]),
    "atlb_dgeqrf_dev": (_I, [_I, _I, _P, _I, _P]),
    "atlb_dormqr_dev": (_I, [_I, _I, _I, _I, _I, _P, _I, _P, _P, _I]),
    "cblas_dsymm": (None, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I]),
    "cblas_dsyr2k": (None, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I]),
    "cblas_zgemm": (None, [_I, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I]),
    "clapack_dgetri": (_I, [_I, _I, _P, _I, _P]),
    "clapack_dpotri": (_I, [_I, _I, _I, _P, _I]),
    "clapack_dlauum": (_I, [_I, _I, _I, _P, _I]),
    "clapack_dtrtri": (_I, [_I, _I, _I, _I, _P, _I]),
    "clapack_dgels": (_I, [_I, _I, _I, _I, _I, _P, _I, _P, _I]),
    "clapack_dgelqf": (_I, [_I, _I, _I, _P, _I, _P]),
    "ATL_dormqr": (_I, [_I, _I, _I, _I, _I, _P, _I, _P, _P, _I, _P, _I]),
    "atlb_dgemm_ozaki_dev": (_I, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _I]),
    "atlb_dgemm_ozaki": (_I, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _I]),
    "atlb_dsgesv": (_I, [_I, _I, _P, _I, _P, _P, _I, _P, _I, _I, _P]),
    "atlb_dsgesv_ex": (_I, [_I, _I, _P, _I, _P, _P, _I, _P, _I, _I, _I, _P]),
    "atlb_dgemm_batched_dev": (_I, [_I, _I, _I, _P, _P, _P, _D, _P, _P, _P, _P, _D, _P, _P]),
    "atlb_dposv_batched": (_I, [_I, _P, _P, _P, _P, _P, _P, _P]),
    "atlb_dgesv_batched": (_I, [_I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "atlb_dgetrf_batched": (_I, [_I, _P, _P, _P, _P, _P]),
    "atlb_dpotrf_adjoint_dev": (_I, [_I, _P, _I, _P, _I, _P, _I]),
    "atlb_dpotrs_adjoint_dev": (_I, [_I, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I]),
    "atlb_dgetrs_adjoint_dev": (_I, [_I, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I]),
    "atlb_dgetrf_adjoint_dev": (_I, [_I, _P, _I, _P, _P, _I, _P, _I, _P, _I]),
    "atlb_dsposv": (_I, [_I, _I, _I, _P, _I, _P, _I, _P, _I, _I, _P]),
    "atlb_mixed_krylov_steps": (_I, []),
    "atlb_dpotrf_adjoint_batched_dev": (_I, [_I, _P, _P, _P, _P, _P, _P, _P]),
    "atlb_dpotrs_adjoint_batched_dev": (_I, [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
}
# Fortran 77 entry points: every argument by address
for _f, _n in (("dgemm_", 13), ("sgemm_", 13), ("zgemm_", 13), ("dtrsm_", 11), ("dtrmm_", 11),
               ("dsyrk_", 10), ("dsymm_", 12), ("dsyr2k_", 12), ("dgetrf_", 6), ("dgetrs_", 9),
               ("dgesv_", 8), ("dgetri_", 7), ("dpotrf_", 5), ("dpotrs_", 8), ("dposv_", 8),
               ("dpotri_", 5), ("dtrtri_", 6), ("dlauum_", 5), ("dgeqrf_", 8), ("dgelqf_", 8),
               ("dgels_", 11)):
    _SIGS[_f] = (None, [_P] * _n)


def lib():
    """The loaded libatlas_b200.so with its signatures (raises if unbuilt)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m atlas_b200.build`")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(l, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def ptr(x):
    """Address of a numpy array / torch tensor / int (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, ctypes.Array):
        return ctypes.addressof(x)
    if hasattr(x, "data_ptr"):  # torch tensor
        return x.data_ptr()
    if hasattr(x, "ctypes"):  # numpy array
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")


def _wrap(name):
    def call(*args):
        f = getattr(lib(), name)
        conv = []
        for a, t in zip(args, f.argtypes):
            if t is _P:
                a = ptr(a)
            elif t is _S and isinstance(a, str):
                a = a.encode()
            conv.append(a)
        return f(*conv)
    call.__name__ = name
    call.__doc__ = f"ctypes call of {name} (see include/atlas_b200.h)"
    return call


for _name in _SIGS:
    globals()[_name] = _wrap(_name)


def declared_symbols(header=None):
    """Function names declared in include/atlas_b200.h."""
    import re
    header = header or os.path.join(os.path.dirname(_HERE), "include", "atlas_b200.h")
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)) - {"if", "defined"})
