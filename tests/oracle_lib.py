"""ctypes access to the CPU oracle (test infrastructure).

``orc()``  -> oracle/liborc.so, the plain-C restatement of the reference's
              algorithms (oracle/oracle.c).
``ref()``  -> oracle/_ref/libiclref.so, the reference's own CPU templates and
              serial OpenCL kernels compiled from their sources (present when
              the reference tree was available at build time), else None.
Wrappers take numpy arrays and return results; in/out arrays are modified in
place like the C calls.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORC_PATH = os.path.join(ROOT, "oracle", "liborc.so")
REF_PATH = os.path.join(ROOT, "oracle", "_ref", "libiclref.so")

_orc = None
_ref = None


class C32(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_PATH):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "liborc.so")],
                           check=True, stdout=subprocess.DEVNULL)
        L = C.CDLL(ORC_PATH)
        f, i, p, d = C.c_float, C.c_int, C.c_void_p, C.c_double
        sig = {
            "orc_saxpy": ([i, f, p, i, p, i], None),
            "orc_sscal": ([i, f, p, i], None),
            "orc_sdot": ([i, p, i, p, i], f),
            "orc_snrm2": ([i, p, i], f),
            "orc_sasum": ([i, p, i], f),
            "orc_isamax": ([i, p, i], i),
            "orc_caxpy": ([i, C32, p, i, p, i], None),
            "orc_cscal": ([i, C32, p, i], None),
            "orc_cdot": ([i, p, i, p, i, i], C32),
            "orc_scnrm2": ([i, p, i], f),
            "orc_scasum": ([i, p, i], f),
            "orc_icamax": ([i, p, i], i),
            "orc_sgemv": ([i, i, i, f, p, i, p, i, f, p, i], None),
            "orc_cgemv": ([i, i, i, C32, p, i, p, i, C32, p, i], None),
            "orc_strsv": ([i, i, i, i, p, i, p, i], None),
            "orc_ctrsv": ([i, i, i, i, p, i, p, i], None),
            "orc_sgemm": ([i, i, i, i, i, f, p, i, p, i, f, p, i], None),
            "orc_cgemm": ([i, i, i, i, i, C32, p, i, p, i, C32, p, i], None),
            "orc_strsm": ([i, i, i, i, i, i, f, p, i, p, i], None),
            "orc_ctrsm": ([i, i, i, i, i, i, C32, p, i, p, i], None),
            "orc_dgemm": ([i, i, i, i, i, d, p, i, p, i, d, p, i], None),
            "orc_dtrsm": ([i, i, i, i, i, i, d, p, i, p, i], None),
            "orc_isamin": ([i, p, i], i),
            "orc_icamin": ([i, p, i], i),
            "orc_copy": ([i, p, i, p, i, i], None),
            "orc_swap": ([i, p, i, p, i, i], None),
            "orc_srot": ([i, p, i, p, i, f, f], None),
            "orc_csrot": ([i, p, i, p, i, f, f], None),
            "orc_crot": ([i, p, i, p, i, f, C32], None),
            "orc_srotm": ([i, p, i, p, i, p], None),
            "orc_srotg": ([p, p, p, p], None),
            "orc_crotg": ([p, p, p, p], None),
            "orc_srotmg": ([p, p, p, f, p], None),
            "orc_sger": ([i, i, f, p, i, p, i, p, i], None),
            "orc_cger": ([i, i, i, C32, p, i, p, i, p, i], None),
            "orc_ssymv": ([i, i, f, p, i, p, i, f, p, i], None),
            "orc_chemv": ([i, i, C32, p, i, p, i, C32, p, i], None),
            "orc_ssyrk": ([i, i, i, i, f, p, i, f, p, i], None),
            "orc_ssyr2k": ([i, i, i, i, f, p, i, p, i, f, p, i], None),
            "orc_ssymm": ([i, i, i, i, f, p, i, p, i, f, p, i], None),
            "orc_strmm": ([i, i, i, i, i, i, f, p, i, p, i, p, i], None),
            "orc_hgemm": ([i, i, i, i, i, f, p, i, p, i, f, p, i], None),
        }
        for name, (a, r) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = a
            fn.restype = r
        _orc = L
    return _orc


def ref() -> C.CDLL | None:
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            return None
        L = C.CDLL(REF_PATH)
        f, i, p = C.c_float, C.c_int, C.c_void_p
        sig = {
            "ref_cpu_sgemm": ([i, i, i, i, i, f, p, i, p, i, f, p, i], None),
            "ref_cpu_cgemm": ([i, i, i, i, i, p, p, i, p, i, p, p, i], None),
            "ref_cpu_dgemm": ([i, i, i, i, i, C.c_double, p, i, p, i, C.c_double, p, i], None),
            "ref_cpu_sdot": ([i, p, i, p, i], f),
            "ref_cpu_cdot": ([i, p, i, p, i, i, p], None),
            "ref_cpu_snrm2": ([i, p, i], f),
            "ref_cpu_scnrm2": ([i, p, i], f),
            "ref_cpu_sasum": ([i, p, i], f),
            "ref_cpu_scasum": ([i, p, i], f),
            "ref_cpu_saxpy": ([i, f, p, i, p, i], None),
            "ref_caxpy_reference": ([i, p, p, i, p, i], None),
            "ref_cpu_sscal": ([i, f, p, i], None),
            "ref_cpu_cscal": ([i, p, p, i], None),
            "ref_cpu_isamax": ([i, p, i], i),
            "ref_cpu_icamax": ([i, p, i], i),
            "ref_naive_sgemv": ([i, i, i, f, p, i, p, i, f, p, i], None),
            "ref_naive_cgemv": ([i, i, i, p, p, i, p, i, p, p, i], None),
            "ref_naive_strsv": ([i, i, i, i, p, i, p, i], None),
            "ref_naive_ctrsv": ([i, i, i, i, p, i, p, i], None),
            "ref_naive_strsm": ([i, i, i, i, i, i, f, p, i, p, i], None),
            "ref_naive_ctrsm": ([i, i, i, i, i, i, p, p, i, p, i], None),
            "ref_naive_sgemm": ([i, i, i, i, i, f, p, i, p, i, f, p, i], None),
            "ref_naive_cgemm": ([i, i, i, i, i, p, p, i, p, i, p, p, i], None),
            "ref_naive_isamin": ([i, p, i], i),
            "ref_naive_icamin": ([i, p, i], i),
            "ref_naive_srot": ([i, p, i, p, i, f, f], None),
            "ref_naive_csrot": ([i, p, i, p, i, f, f], None),
            "ref_naive_crot": ([i, p, i, p, i, f, p], None),
            "ref_naive_srotm": ([i, p, i, p, i, p], None),
            "ref_naive_srotg": ([p, p, p, p], None),
            "ref_naive_crotg": ([p, p, p, p], None),
            "ref_naive_srotmg": ([p, p, p, f, p], None),
            "ref_naive_sger": ([i, i, f, p, i, p, i, p, i], None),
            "ref_naive_cger": ([i, i, i, p, p, i, p, i, p, i], None),
            "ref_naive_ssymv": ([i, i, f, p, i, p, i, f, p, i], None),
            "ref_naive_chemv": ([i, i, p, p, i, p, i, p, p, i], None),
            "ref_naive_ssyr2k": ([i, i, i, i, f, p, i, p, i, f, p, i], None),
            "ref_naive_ssymm": ([i, i, i, i, f, p, i, p, i, f, p, i], None),
            "ref_naive_strmm": ([i, i, i, i, i, i, f, p, i, p, i, p, i], None),
            "ref_cpu_ssymv": ([i, i, f, p, i, p, i, f, p, i], None),
            "ref_cpu_chemv": ([i, i, p, p, i, p, i, p, p, i], None),
        }
        for name, (a, r) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = a
            fn.restype = r
        _ref = L
    return _ref


def c32(v) -> C32:
    v = complex(v)
    return C32(v.real, v.imag)


def cbox(v) -> np.ndarray:
    """A complex scalar as a 2-float array (for ref_* functions taking float*)."""
    v = complex(v)
    return np.array([v.real, v.imag], dtype=np.float32)


# ------------------------------------------------------------ oracle wrappers
def saxpy(n, alpha, x, incx, y, incy):
    orc().orc_saxpy(n, alpha, _p(x), incx, _p(y), incy)


def sscal(n, alpha, x, incx):
    orc().orc_sscal(n, alpha, _p(x), incx)


def sdot(n, x, incx, y, incy) -> float:
    return orc().orc_sdot(n, _p(x), incx, _p(y), incy)


def snrm2(n, x, incx) -> float:
    return orc().orc_snrm2(n, _p(x), incx)


def sasum(n, x, incx) -> float:
    return orc().orc_sasum(n, _p(x), incx)


def isamax(n, x, incx) -> int:
    return orc().orc_isamax(n, _p(x), incx)


def caxpy(n, alpha, x, incx, y, incy):
    orc().orc_caxpy(n, c32(alpha), _p(x), incx, _p(y), incy)


def cscal(n, alpha, x, incx):
    orc().orc_cscal(n, c32(alpha), _p(x), incx)


def cdot(n, x, incx, y, incy, conj) -> complex:
    r = orc().orc_cdot(n, _p(x), incx, _p(y), incy, 1 if conj else 0)
    return complex(np.float32(r.re), np.float32(r.im))


def scnrm2(n, x, incx) -> float:
    return orc().orc_scnrm2(n, _p(x), incx)


def scasum(n, x, incx) -> float:
    return orc().orc_scasum(n, _p(x), incx)


def icamax(n, x, incx) -> int:
    return orc().orc_icamax(n, _p(x), incx)


def sgemv(trans, m, n, alpha, A, lda, x, incx, beta, y, incy):
    orc().orc_sgemv(trans, m, n, alpha, _p(A), lda, _p(x), incx, beta, _p(y), incy)


def cgemv(trans, m, n, alpha, A, lda, x, incx, beta, y, incy):
    orc().orc_cgemv(trans, m, n, c32(alpha), _p(A), lda, _p(x), incx, c32(beta), _p(y), incy)


def strsv(uplo, trans, diag, n, A, lda, x, incx):
    orc().orc_strsv(uplo, trans, diag, n, _p(A), lda, _p(x), incx)


def ctrsv(uplo, trans, diag, n, A, lda, x, incx):
    orc().orc_ctrsv(uplo, trans, diag, n, _p(A), lda, _p(x), incx)


def sgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    orc().orc_sgemm(ta, tb, m, n, k, alpha, _p(A), lda, _p(B), ldb, beta, _p(Cm), ldc)


def cgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    orc().orc_cgemm(ta, tb, m, n, k, c32(alpha), _p(A), lda, _p(B), ldb, c32(beta), _p(Cm), ldc)


def strsm(side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb):
    orc().orc_strsm(side, uplo, trans, diag, m, n, alpha, _p(A), lda, _p(B), ldb)


def ctrsm(side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb):
    orc().orc_ctrsm(side, uplo, trans, diag, m, n, c32(alpha), _p(A), lda, _p(B), ldb)


def dgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    orc().orc_dgemm(ta, tb, m, n, k, alpha, _p(A), lda, _p(B), ldb, beta, _p(Cm), ldc)


def dtrsm(side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb):
    orc().orc_dtrsm(side, uplo, trans, diag, m, n, alpha, _p(A), lda, _p(B), ldb)


def isamin(n, x, incx) -> int:
    return orc().orc_isamin(n, _p(x), incx)


def icamin(n, x, incx) -> int:
    return orc().orc_icamin(n, _p(x), incx)


def copy(n, x, incx, y, incy):
    orc().orc_copy(n, _p(x), incx, _p(y), incy, x.itemsize)


def swap(n, x, incx, y, incy):
    orc().orc_swap(n, _p(x), incx, _p(y), incy, x.itemsize)


def srot(n, x, incx, y, incy, c, s):
    orc().orc_srot(n, _p(x), incx, _p(y), incy, c, s)


def csrot(n, x, incx, y, incy, c, s):
    orc().orc_csrot(n, _p(x), incx, _p(y), incy, c, s)


def crot(n, x, incx, y, incy, c, s):
    orc().orc_crot(n, _p(x), incx, _p(y), incy, c, c32(s))


def srotm(n, x, incx, y, incy, param):
    orc().orc_srotm(n, _p(x), incx, _p(y), incy, _p(param))


def srotg(a, b):
    """Returns (r, z, c, s) as float32 for inputs a, b."""
    v = np.array([a, b, 0, 0], dtype=np.float32)
    orc().orc_srotg(_p(v[0:]), _p(v[1:]), _p(v[2:]), _p(v[3:]))
    return tuple(v)


def crotg(a, b):
    """Returns (a', c, s) for complex inputs a, b."""
    v = np.array([a, b, 0], dtype=np.complex64)
    c = np.zeros(1, dtype=np.float32)
    orc().orc_crotg(_p(v[0:]), _p(v[1:]), _p(c), _p(v[2:]))
    return v[0], c[0], v[2]


def srotmg(d1, d2, x1, y1, param):
    """Returns (d1', d2', x1'); param (5 floats) is updated in place."""
    v = np.array([d1, d2, x1], dtype=np.float32)
    orc().orc_srotmg(_p(v[0:]), _p(v[1:]), _p(v[2:]), float(np.float32(y1)), _p(param))
    return tuple(v)


def sger(m, n, alpha, x, incx, y, incy, A, lda):
    orc().orc_sger(m, n, alpha, _p(x), incx, _p(y), incy, _p(A), lda)


def cger(conj, m, n, alpha, x, incx, y, incy, A, lda):
    orc().orc_cger(1 if conj else 0, m, n, c32(alpha), _p(x), incx, _p(y), incy, _p(A), lda)


def ssymv(uplo, n, alpha, A, lda, x, incx, beta, y, incy):
    orc().orc_ssymv(uplo, n, alpha, _p(A), lda, _p(x), incx, beta, _p(y), incy)


def chemv(uplo, n, alpha, A, lda, x, incx, beta, y, incy):
    orc().orc_chemv(uplo, n, c32(alpha), _p(A), lda, _p(x), incx, c32(beta), _p(y), incy)


def ssyrk(uplo, trans, n, k, alpha, A, lda, beta, Cm, ldc):
    orc().orc_ssyrk(uplo, trans, n, k, alpha, _p(A), lda, beta, _p(Cm), ldc)


def ssyr2k(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    orc().orc_ssyr2k(uplo, trans, n, k, alpha, _p(A), lda, _p(B), ldb, beta, _p(Cm), ldc)


def ssymm(side, uplo, m, n, alpha, A, lda, B, ldb, beta, Cm, ldc):
    orc().orc_ssymm(side, uplo, m, n, alpha, _p(A), lda, _p(B), ldb, beta, _p(Cm), ldc)


def strmm(side, uplo, transa, diag, m, n, alpha, A, lda, B, ldb, Cm, ldc):
    orc().orc_strmm(side, uplo, transa, diag, m, n, alpha, _p(A), lda, _p(B), ldb, _p(Cm), ldc)


def hgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    """A, B, Cm: float16 arrays (bit patterns passed through)."""
    orc().orc_hgemm(ta, tb, m, n, k, alpha, _p(A), lda, _p(B), ldb, beta, _p(Cm), ldc)


# ------------------------------------------------------------ data helpers
def colmajor(rows, cols, ld, rng, dtype=np.float32, low=-1.0, high=1.0):
    """A column-major matrix as a flat array of ld*cols elements (padding too)."""
    if np.dtype(dtype) == np.complex64:
        a = rng.uniform(low, high, size=(ld * cols, 2)).astype(np.float32)
        return a.view(np.complex64).reshape(-1)
    return rng.uniform(low, high, size=ld * cols).astype(dtype)


def quarter_ints(size, rng, dtype=np.float32):
    """0.25 * UniformInt[-4, 4]: the reference's blas_funcs test values
    (tests/blas_funcs/test_helpers.hpp:120-127), exact in FP32 products/sums."""
    if np.dtype(dtype) == np.complex64:
        v = 0.25 * rng.integers(-4, 5, size=(size, 2)).astype(np.float32)
        return v.view(np.complex64).reshape(-1)
    return (0.25 * rng.integers(-4, 5, size=size)).astype(dtype)


def ulp_diff(a, b) -> np.ndarray:
    """|a - b| in units of float32 ulps (elementwise, by integer ordering)."""
    a = np.ascontiguousarray(a, dtype=np.float32).view(np.int32).astype(np.int64)
    b = np.ascontiguousarray(b, dtype=np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


def rel_fro(x, ref) -> float:
    x = np.asarray(x, dtype=np.complex128 if np.iscomplexobj(x) else np.float64)
    ref = np.asarray(ref, dtype=np.complex128 if np.iscomplexobj(ref) else np.float64)
    den = np.linalg.norm(ref)
    return float(np.linalg.norm(x - ref) / (den if den > 0 else 1.0))
