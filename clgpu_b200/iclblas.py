"""ctypes binding of libiclblas_b200.so: the iclBLAS C API from Python.

Names, argument order and meaning follow the C header (include/iclBLAS.h),
which mirrors the reference's include/iclBLAS/iclBLAS.h.  Array arguments
accept numpy arrays (host memory: the call copies in, runs, copies out and
blocks, as the reference does) or anything exposing ``data_ptr()`` such as a
CUDA torch tensor (device memory: the call is enqueued on the handle's stream).
Scalars are passed by value here and handed to the library by pointer.

There is no fallback: if the shared library is missing this module raises on
import, and every routine runs the library's sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libiclblas_b200.so")

# status codes (include/iclBLAS.h)
SUCCESS = 0
NOT_INITIALIZED = 1
ALLOC_FAILED = 3
INVALID_VALUE = 7
ARCH_MISMATCH = 8
MAPPING_ERROR = 11
EXECUTION_FAILED = 13
INTERNAL_ERROR = 14
NOT_SUPPORTED = 15
LICENSE_ERROR = 16
ERROR = 17

OP_N, OP_T, OP_C = 0, 1, 2
FILL_UPPER, FILL_LOWER = 0, 1
DIAG_NON_UNIT, DIAG_UNIT = 0, 1
SIDE_LEFT, SIDE_RIGHT = 0, 1
MATH_PLAIN_FP32, MATH_TF32, MATH_BF16X3, MATH_BF16X6 = 0, 1, 2, 3

STATUS_NAMES = {
    0: "SUCCESS", 1: "NOT_INITIALIZED", 3: "ALLOC_FAILED", 7: "INVALID_VALUE", 8: "ARCH_MISMATCH",
    11: "MAPPING_ERROR", 13: "EXECUTION_FAILED", 14: "INTERNAL_ERROR", 15: "NOT_SUPPORTED",
    16: "LICENSE_ERROR", 17: "ERROR",
}


class IclblasError(RuntimeError):
    def __init__(self, fn: str, status: int):
        super().__init__(f"{fn} returned {STATUS_NAMES.get(status, status)}")
        self.status = status


class Complex(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


_P = C.c_void_p
_I = C.c_int
_H = C.c_void_p

# (name, argtypes) for every exported routine; pointer-to-scalar arguments
# are marked with the ctypes type of the pointee so the wrappers can box them.
_SIGS = {
    "iclblasCreate": [C.POINTER(_H)],
    "iclblasDestroy": [_H],
    "iclblasSetStream": [_H, _P],
    "iclblasGetStream": [_H, C.POINTER(_P)],
    "iclblasSetMathMode": [_H, _I],
    "iclblasGetMathMode": [_H, C.POINTER(_I)],
    "iclblasSynchronize": [_H],
    "iclblasSetTrsmRefinement": [_H, _I],
    "iclblasGetTrsmRefinement": [_H, C.POINTER(_I)],
    "iclblasSscal": [_H, _I, _P, _P, _I],
    "iclblasSaxpy": [_H, _I, _P, _P, _I, _P, _I],
    "iclblasSnrm2": [_H, _I, _P, _I, _P],
    "iclblasIsamax": [_H, _I, _P, _I, _P],
    "iclblasSasum": [_H, _I, _P, _I, _P],
    "iclblasSdot": [_H, _I, _P, _I, _P, _I, _P],
    "iclblasSdotNoAlloc": [_H, _I, _P, _I, _P, _I, _P],
    "iclblasCscal": [_H, _I, _P, _P, _I],
    "iclblasCsscal": [_H, _I, _P, _P, _I],
    "iclblasCdotu": [_H, _I, _P, _I, _P, _I, _P],
    "iclblasCdotc": [_H, _I, _P, _I, _P, _I, _P],
    "iclblasScnrm2": [_H, _I, _P, _I, _P],
    "iclblasIcamax": [_H, _I, _P, _I, _P],
    "iclblasCaxpy": [_H, _I, _P, _P, _I, _P, _I],
    "iclblasScasum": [_H, _I, _P, _I, _P],
    "iclblasIsamin": [_H, _I, _P, _I, _P],
    "iclblasScopy": [_H, _I, _P, _I, _P, _I],
    "iclblasSswap": [_H, _I, _P, _I, _P, _I],
    "iclblasSrot": [_H, _I, _P, _I, _P, _I, C.c_float, C.c_float],
    "iclblasSrotm": [_H, _I, _P, _I, _P, _I, _P],
    "iclblasSrotg": [_H, _P, _P, _P, _P],
    "iclblasSrotmg": [_H, _P, _P, _P, _P, _P],
    "iclblasIcamin": [_H, _I, _P, _I, _P],
    "iclblasCcopy": [_H, _I, _P, _I, _P, _I],
    "iclblasCswap": [_H, _I, _P, _I, _P, _I],
    "iclblasCrot": [_H, _I, _P, _I, _P, _I, _P, _P],
    "iclblasCsrot": [_H, _I, _P, _I, _P, _I, _P, _P],
    "iclblasCrotg": [_H, _P, _P, _P, _P],
    "iclblasSger": [_H, _I, _I, _P, _P, _I, _P, _I, _P, _I],
    "iclblasCgeru": [_H, _I, _I, _P, _P, _I, _P, _I, _P, _I],
    "iclblasCgerc": [_H, _I, _I, _P, _P, _I, _P, _I, _P, _I],
    "iclblasSsymv": [_H, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasChemv": [_H, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasSsyrk": [_H, _I, _I, _I, _I, _P, _P, _I, _P, _P, _I],
    "iclblasSsyr2k": [_H, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasSsymm": [_H, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasStrmm": [_H, _I, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _I],
    "iclblasHgemm": [_H, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasStrsv": [_H, _I, _I, _I, _I, _P, _I, _P, _I],
    "iclblasCtrsv": [_H, _I, _I, _I, _I, _P, _I, _P, _I],
    "iclblasSgemv": [_H, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasCgemv": [_H, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasSgemm": [_H, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasCgemm": [_H, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I],
    "iclblasStrsm": [_H, _I, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I],
    "iclblasCtrsm": [_H, _I, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I],
    "iclblasStrsm_backward": [_H, _I, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I],
    "iclblasSgemm_backward": [_H, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I],
    "iclblasStrsmBatchedPlanCreate": [_H, _I, _I, _I, _I, _I, _P, _P, _P, _P, C.POINTER(_P)],
    "iclblasSgemmBatchedPlanCreate": [_H, _I, _I, _I, _P, _P, _P, _P, _P, _P, C.POINTER(_P)],
    "iclblasBatchPlanDestroy": [_P],
    "iclblasBatchPlanGetInfo": [_P, C.POINTER(C.c_double), C.POINTER(_I), C.POINTER(_I)],
    "iclblasBatchPlanSetInverseReuse": [_P, _I],
    "iclblasStrsmBatchedUneven": [_H, _P, _P, _P, _P],
    "iclblasSgemmBatchedUneven": [_H, _P, _P, _P, _P, _P, _P],
    "iclblasStrsmBatchedUnevenBackward": [_H, _P, _P, _P, _P, _P, _P],
}

_lib = None


def lib() -> C.CDLL:
    """Load libiclblas_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m clgpu_b200.build` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, argt in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = argt
            f.restype = C.c_int
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


# ---------------------------------------------------------------- pointers
def ptr(a) -> int | None:
    """Address of an array argument: numpy array, torch tensor, int or None."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"unsupported array argument {type(a)}")


def _fscalar(v) -> C.c_float:
    return C.c_float(float(v))


def _cscalar(v) -> Complex:
    v = complex(v)
    return Complex(v.real, v.imag)


def _call(name: str, *args) -> int:
    return getattr(lib(), name)(*args)


# ---------------------------------------------------------------- handle
class Handle:
    """An iclblasHandle_t.  ``with Handle() as h:`` creates and destroys it."""

    def __init__(self):
        self.value = _H()
        st = _call("iclblasCreate", C.byref(self.value))
        if st != SUCCESS:
            raise IclblasError("iclblasCreate", st)

    @property
    def _as_parameter_(self):
        return self.value

    def set_stream(self, stream) -> None:
        """Use a CUDA stream (an int handle, a torch.cuda.Stream, or None)."""
        s = getattr(stream, "cuda_stream", stream)
        st = _call("iclblasSetStream", self.value, _P(s) if s else None)
        if st != SUCCESS:
            raise IclblasError("iclblasSetStream", st)

    def set_math_mode(self, mode: int) -> None:
        st = _call("iclblasSetMathMode", self.value, mode)
        if st != SUCCESS:
            raise IclblasError("iclblasSetMathMode", st)

    def set_trsm_refinement(self, steps: int) -> None:
        st = _call("iclblasSetTrsmRefinement", self.value, steps)
        if st != SUCCESS:
            raise IclblasError("iclblasSetTrsmRefinement", st)

    def synchronize(self) -> int:
        return _call("iclblasSynchronize", self.value)

    def destroy(self) -> None:
        if self.value:
            st = _call("iclblasDestroy", self.value)
            self.value = _H()
            if st != SUCCESS:
                raise IclblasError("iclblasDestroy", st)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()


def _h(h):
    if isinstance(h, Handle):
        return h.value
    return h


# ---------------------------------------------------------------- routines
# Each wrapper returns the iclblasStatus_t of the call; results of reductions
# are written into the `result` array argument, as in the C API.

def iclblasSscal(h, n, alpha, x, incx):
    return _call("iclblasSscal", _h(h), n, C.byref(_fscalar(alpha)), ptr(x), incx)


def iclblasSaxpy(h, n, alpha, x, incx, y, incy):
    return _call("iclblasSaxpy", _h(h), n, C.byref(_fscalar(alpha)), ptr(x), incx, ptr(y), incy)


def iclblasSnrm2(h, n, x, incx, result):
    return _call("iclblasSnrm2", _h(h), n, ptr(x), incx, ptr(result))


def iclblasIsamax(h, n, x, incx, result):
    return _call("iclblasIsamax", _h(h), n, ptr(x), incx, ptr(result))


def iclblasSasum(h, n, x, incx, result):
    return _call("iclblasSasum", _h(h), n, ptr(x), incx, ptr(result))


def iclblasSdot(h, n, x, incx, y, incy, result):
    return _call("iclblasSdot", _h(h), n, ptr(x), incx, ptr(y), incy, ptr(result))


def iclblasSdotNoAlloc(h, n, x, incx, y, incy, result):
    """SDOT with no device allocation; device operands only (see include/iclBLAS.h)."""
    return _call("iclblasSdotNoAlloc", _h(h), n, ptr(x), incx, ptr(y), incy, ptr(result))


def iclblasCscal(h, n, alpha, x, incx):
    return _call("iclblasCscal", _h(h), n, C.byref(_cscalar(alpha)), ptr(x), incx)


def iclblasCsscal(h, n, alpha, x, incx):
    return _call("iclblasCsscal", _h(h), n, C.byref(_fscalar(alpha)), ptr(x), incx)


def iclblasCdotu(h, n, x, incx, y, incy, result):
    return _call("iclblasCdotu", _h(h), n, ptr(x), incx, ptr(y), incy, ptr(result))


def iclblasCdotc(h, n, x, incx, y, incy, result):
    return _call("iclblasCdotc", _h(h), n, ptr(x), incx, ptr(y), incy, ptr(result))


def iclblasScnrm2(h, n, x, incx, result):
    return _call("iclblasScnrm2", _h(h), n, ptr(x), incx, ptr(result))


def iclblasIcamax(h, n, x, incx, result):
    return _call("iclblasIcamax", _h(h), n, ptr(x), incx, ptr(result))


def iclblasCaxpy(h, n, alpha, x, incx, y, incy):
    return _call("iclblasCaxpy", _h(h), n, C.byref(_cscalar(alpha)), ptr(x), incx, ptr(y), incy)


def iclblasScasum(h, n, x, incx, result):
    return _call("iclblasScasum", _h(h), n, ptr(x), incx, ptr(result))


def iclblasIsamin(h, n, x, incx, result):
    return _call("iclblasIsamin", _h(h), n, ptr(x), incx, ptr(result))


def iclblasScopy(h, n, x, incx, y, incy):
    return _call("iclblasScopy", _h(h), n, ptr(x), incx, ptr(y), incy)


def iclblasSswap(h, n, x, incx, y, incy):
    return _call("iclblasSswap", _h(h), n, ptr(x), incx, ptr(y), incy)


def iclblasSrot(h, n, x, incx, y, incy, c, s):
    return _call("iclblasSrot", _h(h), n, ptr(x), incx, ptr(y), incy, float(c), float(s))


def iclblasSrotm(h, n, x, incx, y, incy, param):
    """param: 5 floats {flag, p1, p2, p3, p4}, host array or device tensor."""
    return _call("iclblasSrotm", _h(h), n, ptr(x), incx, ptr(y), incy, ptr(param))


def iclblasSrotg(h, a, b, c, s):
    """a, b, c, s: one-element float arrays (host or device), updated in place."""
    return _call("iclblasSrotg", _h(h), ptr(a), ptr(b), ptr(c), ptr(s))


def iclblasSrotmg(h, d1, d2, x1, y1, param):
    return _call("iclblasSrotmg", _h(h), ptr(d1), ptr(d2), ptr(x1), ptr(y1), ptr(param))


def iclblasIcamin(h, n, x, incx, result):
    return _call("iclblasIcamin", _h(h), n, ptr(x), incx, ptr(result))


def iclblasCcopy(h, n, x, incx, y, incy):
    return _call("iclblasCcopy", _h(h), n, ptr(x), incx, ptr(y), incy)


def iclblasCswap(h, n, x, incx, y, incy):
    return _call("iclblasCswap", _h(h), n, ptr(x), incx, ptr(y), incy)


def iclblasCrot(h, n, x, incx, y, incy, c, s):
    """c: real scalar, s: complex scalar (both passed by host pointer)."""
    return _call("iclblasCrot", _h(h), n, ptr(x), incx, ptr(y), incy, C.byref(_fscalar(c)), C.byref(_cscalar(s)))


def iclblasCsrot(h, n, x, incx, y, incy, c, s):
    return _call("iclblasCsrot", _h(h), n, ptr(x), incx, ptr(y), incy, C.byref(_fscalar(c)), C.byref(_fscalar(s)))


def iclblasCrotg(h, a, b, c, s):
    """a, b, s: one-element complex64 arrays; c: one-element float array."""
    return _call("iclblasCrotg", _h(h), ptr(a), ptr(b), ptr(c), ptr(s))


def iclblasSger(h, m, n, alpha, x, incx, y, incy, A, lda):
    return _call("iclblasSger", _h(h), m, n, C.byref(_fscalar(alpha)), ptr(x), incx, ptr(y), incy, ptr(A), lda)


def iclblasCgeru(h, m, n, alpha, x, incx, y, incy, A, lda):
    return _call("iclblasCgeru", _h(h), m, n, C.byref(_cscalar(alpha)), ptr(x), incx, ptr(y), incy, ptr(A), lda)


def iclblasCgerc(h, m, n, alpha, x, incx, y, incy, A, lda):
    return _call("iclblasCgerc", _h(h), m, n, C.byref(_cscalar(alpha)), ptr(x), incx, ptr(y), incy, ptr(A), lda)


def iclblasSsymv(h, uplo, n, alpha, A, lda, x, incx, beta, y, incy):
    return _call("iclblasSsymv", _h(h), uplo, n, C.byref(_fscalar(alpha)), ptr(A), lda, ptr(x), incx,
                 C.byref(_fscalar(beta)), ptr(y), incy)


def iclblasChemv(h, uplo, n, alpha, A, lda, x, incx, beta, y, incy):
    return _call("iclblasChemv", _h(h), uplo, n, C.byref(_cscalar(alpha)), ptr(A), lda, ptr(x), incx,
                 C.byref(_cscalar(beta)), ptr(y), incy)


def iclblasSsyrk(h, uplo, trans, n, k, alpha, A, lda, beta, Cm, ldc):
    return _call("iclblasSsyrk", _h(h), uplo, trans, n, k, C.byref(_fscalar(alpha)), ptr(A), lda,
                 C.byref(_fscalar(beta)), ptr(Cm), ldc)


def iclblasSsyr2k(h, uplo, trans, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    return _call("iclblasSsyr2k", _h(h), uplo, trans, n, k, C.byref(_fscalar(alpha)), ptr(A), lda, ptr(B), ldb,
                 C.byref(_fscalar(beta)), ptr(Cm), ldc)


def iclblasSsymm(h, side, uplo, m, n, alpha, A, lda, B, ldb, beta, Cm, ldc):
    return _call("iclblasSsymm", _h(h), side, uplo, m, n, C.byref(_fscalar(alpha)), ptr(A), lda, ptr(B), ldb,
                 C.byref(_fscalar(beta)), ptr(Cm), ldc)


def iclblasStrmm(h, side, uplo, transa, diag, m, n, alpha, A, lda, B, ldb, Cm, ldc):
    return _call("iclblasStrmm", _h(h), side, uplo, transa, diag, m, n, C.byref(_fscalar(alpha)), ptr(A), lda,
                 ptr(B), ldb, ptr(Cm), ldc)


def iclblasHgemm(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    """A, B, Cm: float16 arrays (numpy float16 / torch.half); alpha, beta: floats."""
    return _call("iclblasHgemm", _h(h), transa, transb, m, n, k, C.byref(_fscalar(alpha)), ptr(A), lda, ptr(B), ldb,
                 C.byref(_fscalar(beta)), ptr(Cm), ldc)


def iclblasStrsv(h, uplo, trans, diag, n, A, lda, x, incx):
    return _call("iclblasStrsv", _h(h), uplo, trans, diag, n, ptr(A), lda, ptr(x), incx)


def iclblasCtrsv(h, uplo, trans, diag, n, A, lda, x, incx):
    return _call("iclblasCtrsv", _h(h), uplo, trans, diag, n, ptr(A), lda, ptr(x), incx)


def iclblasSgemv(h, trans, m, n, alpha, A, lda, x, incx, beta, y, incy):
    return _call("iclblasSgemv", _h(h), trans, m, n, C.byref(_fscalar(alpha)), ptr(A), lda, ptr(x), incx,
                 C.byref(_fscalar(beta)), ptr(y), incy)


def iclblasCgemv(h, trans, m, n, alpha, A, lda, x, incx, beta, y, incy):
    return _call("iclblasCgemv", _h(h), trans, m, n, C.byref(_cscalar(alpha)), ptr(A), lda, ptr(x), incx,
                 C.byref(_cscalar(beta)), ptr(y), incy)


def iclblasSgemm(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    return _call("iclblasSgemm", _h(h), transa, transb, m, n, k, C.byref(_fscalar(alpha)), ptr(A), lda, ptr(B), ldb,
                 C.byref(_fscalar(beta)), ptr(Cm), ldc)


def iclblasCgemm(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    return _call("iclblasCgemm", _h(h), transa, transb, m, n, k, C.byref(_cscalar(alpha)), ptr(A), lda, ptr(B), ldb,
                 C.byref(_cscalar(beta)), ptr(Cm), ldc)


def iclblasStrsm(h, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb):
    return _call("iclblasStrsm", _h(h), side, uplo, trans, diag, m, n, C.byref(_fscalar(alpha)), ptr(A), lda, ptr(B),
                 ldb)


def iclblasCtrsm(h, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb):
    return _call("iclblasCtrsm", _h(h), side, uplo, trans, diag, m, n, C.byref(_cscalar(alpha)), ptr(A), lda, ptr(B),
                 ldb)


def iclblasStrsm_backward(h, side, uplo, trans, diag, m, n, alpha, A, lda, X, ldx, G, ldg, dA, ldda):
    return _call("iclblasStrsm_backward", _h(h), side, uplo, trans, diag, m, n, C.byref(_fscalar(alpha)), ptr(A), lda,
                 ptr(X), ldx, ptr(G), ldg, ptr(dA), ldda)


def iclblasSgemm_backward(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, G, ldg, dA, ldda, dB, lddb, dC,
                          lddc):
    return _call("iclblasSgemm_backward", _h(h), transa, transb, m, n, k, C.byref(_fscalar(alpha)), ptr(A), lda,
                 ptr(B), ldb, C.byref(_fscalar(beta)), ptr(G), ldg, ptr(dA), ldda, ptr(dB), lddb, ptr(dC), lddc)


def check(status: int, fn: str = "iclblas call") -> None:
    if status != SUCCESS:
        raise IclblasError(fn, status)


class BatchPlan:
    """An iclblasBatchPlan_t built from per-instance sizes (int sequences).

    ``BatchPlan(h, "trsm", side=, uplo=, trans=, diag=, m=, n=, lda=, ldb=)`` or
    ``BatchPlan(h, "gemm", transa=, transb=, m=, n=, k=, lda=, ldb=, ldc=)``."""

    def __init__(self, h, kind, **kw):
        self.value = _P()
        arr = lambda v: np.ascontiguousarray(np.asarray(v, dtype=np.int32))  # noqa: E731
        d = {k: arr(v) for k, v in kw.items() if isinstance(v, (list, tuple, np.ndarray))}
        if kind == "trsm":
            st = _call("iclblasStrsmBatchedPlanCreate", _h(h), kw["side"], kw["uplo"], kw["trans"], kw["diag"],
                       len(d["m"]), ptr(d["m"]), ptr(d["n"]), ptr(d["lda"]), ptr(d["ldb"]), C.byref(self.value))
        elif kind == "gemm":
            st = _call("iclblasSgemmBatchedPlanCreate", _h(h), kw["transa"], kw["transb"], len(d["m"]), ptr(d["m"]),
                       ptr(d["n"]), ptr(d["k"]), ptr(d["lda"]), ptr(d["ldb"]), ptr(d["ldc"]), C.byref(self.value))
        else:
            raise ValueError(kind)
        if st != SUCCESS:
            raise IclblasError("iclblas*BatchedPlanCreate", st)

    def info(self):
        """(algorithmic flops per call, tile width, CTAs per SM)."""
        f, w, c = C.c_double(), C.c_int(), C.c_int()
        check(_call("iclblasBatchPlanGetInfo", self.value, C.byref(f), C.byref(w), C.byref(c)))
        return f.value, w.value, c.value

    def set_inverse_reuse(self, reuse: bool) -> int:
        """TRSM plans: the backward call reuses the forward call's inverses."""
        return _call("iclblasBatchPlanSetInverseReuse", self.value, 1 if reuse else 0)

    def destroy(self):
        if self.value:
            _call("iclblasBatchPlanDestroy", self.value)
            self.value = _P()


def iclblasStrsmBatchedUneven(h, plan, alpha, A, B):
    """A, B: device arrays of per-instance device pointers (e.g. int64 CUDA tensors)."""
    return _call("iclblasStrsmBatchedUneven", _h(h), plan.value, C.byref(_fscalar(alpha)), ptr(A), ptr(B))


def iclblasSgemmBatchedUneven(h, plan, alpha, A, B, beta, Cm):
    return _call("iclblasSgemmBatchedUneven", _h(h), plan.value, C.byref(_fscalar(alpha)), ptr(A), ptr(B),
                 C.byref(_fscalar(beta)), ptr(Cm))


def iclblasStrsmBatchedUnevenBackward(h, plan, alpha, A, X, G, dA):
    return _call("iclblasStrsmBatchedUnevenBackward", _h(h), plan.value, C.byref(_fscalar(alpha)), ptr(A), ptr(X),
                 ptr(G), ptr(dA))
