"""The C-ABI library loads and exports every symbol include/iclBLAS.h declares;
host-side argument checks follow the reference's rules (no GPU needed: every
case below returns before any device work)."""
import ctypes as C
import os
import re

import numpy as np

from clgpu_b200 import iclblas as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "iclBLAS.h")).read()
    return sorted(set(re.findall(r"ICLBLAS_API\s+iclblasStatus_t\s+(\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(libpath):
    L = C.CDLL(libpath)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert len(declared_symbols()) >= 29


def test_binding_covers_header():
    assert sorted(B.exported_symbols()) == declared_symbols()


def test_enum_values_match_reference():
    # include/iclBLAS/iclBLAS.h:104-158 of the reference
    assert (B.SUCCESS, B.NOT_INITIALIZED, B.ALLOC_FAILED, B.INVALID_VALUE, B.ARCH_MISMATCH, B.MAPPING_ERROR,
            B.EXECUTION_FAILED, B.INTERNAL_ERROR, B.NOT_SUPPORTED, B.LICENSE_ERROR, B.ERROR) == (
        0, 1, 3, 7, 8, 11, 13, 14, 15, 16, 17)
    assert (B.OP_N, B.OP_T, B.OP_C) == (0, 1, 2)
    assert (B.FILL_UPPER, B.FILL_LOWER) == (0, 1)
    assert (B.DIAG_NON_UNIT, B.DIAG_UNIT) == (0, 1)
    assert (B.SIDE_LEFT, B.SIDE_RIGHT) == (0, 1)


def test_create_destroy_null(libpath):
    L = B.lib()
    assert L.iclblasCreate(None) == B.INVALID_VALUE          # iclBLAS.cpp:45-48
    assert L.iclblasDestroy(None) == B.INVALID_VALUE         # a status, not a throw


def test_validation_order_without_device(libpath):
    x = np.ones(8, np.float32)
    y = np.ones(8, np.float32)
    A = np.ones(64, np.float32)
    # n == 0 ends the call successfully before the handle is looked at
    assert B.iclblasSscal(None, 0, 2.0, x, 1) == B.SUCCESS
    assert B.iclblasSscal(None, -1, 2.0, x, 1) == B.INVALID_VALUE
    assert B.iclblasSscal(None, 4, 2.0, None, 1) == B.INVALID_VALUE   # null x
    assert B.iclblasSscal(None, 4, 2.0, x, 0) == B.INVALID_VALUE      # incx == 0
    assert B.iclblasSscal(None, 4, 2.0, x, -1) == B.NOT_SUPPORTED     # negative stride
    assert B.iclblasSscal(None, 4, 2.0, x, 1) == B.INVALID_VALUE      # bad handle last
    # Saxpy: alpha == 0 or n <= 0 returns first (iclBLAS_S.cpp:77-78)
    assert B.iclblasSaxpy(None, 4, 0.0, x, 1, y, 1) == B.SUCCESS
    assert B.iclblasSaxpy(None, -3, 1.0, x, 1, y, 1) == B.SUCCESS
    assert B.iclblasSaxpy(None, 4, 1.0, x, 1, y, -2) == B.NOT_SUPPORTED
    # Sgemm: negative sizes first (iclBLAS_S.cpp:491-492), then validate_params
    assert B.iclblasSgemm(None, 0, 0, -1, 4, 4, 1.0, A, 8, A, 8, 0.0, A, 8) == B.INVALID_VALUE
    assert B.iclblasSgemm(None, 0, 0, 4, 0, 4, 1.0, A, 8, A, 8, 0.0, A, 8) == B.SUCCESS
    assert B.iclblasSgemm(None, 0, 0, 4, 4, 4, 1.0, A, 0, A, 8, 0.0, A, 8) == B.INVALID_VALUE
    assert B.iclblasSgemm(None, 0, 0, 4, 4, 4, 1.0, A, 8, A, 8, 0.0, None, 8) == B.INVALID_VALUE
    # Sgemv: early success on alpha == 0 and beta == 1 (iclBLAS_S.cpp:477)
    assert B.iclblasSgemv(None, 0, 4, 4, 0.0, A, 4, x, 1, 1.0, y, 1) == B.SUCCESS
    assert B.iclblasSgemv(None, 0, 4, 4, 1.0, A, 4, x, 0, 1.0, y, 1) == B.INVALID_VALUE
    # Strsv: n == 0 success, n < 0 / incx == 0 invalid (iclBLAS_S.cpp:242-244)
    assert B.iclblasStrsv(None, 1, 0, 0, 0, A, 4, x, 1) == B.SUCCESS
    assert B.iclblasStrsv(None, 1, 0, 0, -2, A, 4, x, 1) == B.INVALID_VALUE
    assert B.iclblasStrsv(None, 1, 0, 0, 4, A, 4, x, 0) == B.INVALID_VALUE
    # Strsm: m == 0 success before anything (iclBLAS_S.cpp:503-504)
    assert B.iclblasStrsm(None, 0, 1, 0, 0, 0, 4, 1.0, A, 4, A, 4) == B.SUCCESS
    assert B.iclblasStrsm(None, 0, 1, 0, 0, 4, 4, 1.0, A, -1, A, 4) == B.INVALID_VALUE


def test_reduction_early_results_without_device(libpath):
    x = np.ones(8, np.float32)
    r = np.array([123.0], np.float32)
    assert B.iclblasSnrm2(None, 0, x, 1, r) == B.SUCCESS and r[0] == 0.0   # iclBLAS_S.cpp:89-92
    r[0] = 5
    assert B.iclblasSasum(None, 4, x, -1, r) == B.SUCCESS and r[0] == 0.0
    ri = np.array([9], np.int32)
    assert B.iclblasIsamax(None, 0, x, 1, ri) == B.SUCCESS and ri[0] == 0
    r[0] = 7
    assert B.iclblasSdot(None, 0, x, 1, x, 1, r) == B.SUCCESS and r[0] == 7.0  # untouched (:204-205)
    rc = np.array([3 + 4j], np.complex64)
    assert B.iclblasCdotu(None, 0, x, 1, x, 1, rc) == B.SUCCESS and rc[0] == 0
