"""Golden vectors produced by the reference's own CPU code (tests/golden/
reference_cpu_vectors.npz, made by tests/golden/make_golden.py from the
reference's CPU templates and serial kernels compiled from its sources).

CPU tests pin the oracle to them; GPU tests check the library through its C
ABI against them directly, so GPU parity does not depend on the oracle.
Bars: index results and the quarter-integer SGEMM exact; level-1 float
results within 1 ulp (different summation order of the same FP64 sums);
GEMV/TRSV/TRSM/CGEMM relative Frobenius error <= 1e-5 (the reference's serial
kernels round in FP32).
"""
import os

import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_cpu_vectors.npz"))
CASES = sorted({k.split("/")[0] for k in G.files})
TOL = 1e-5


def g(case, name):
    return G[f"{case}/{name}"]


def cases(prefix):
    return [c for c in CASES if c.startswith(prefix)]


def ulps(a, b):
    return int(O.ulp_diff(np.float32(a), np.float32(b)).max())


def cnear(got, want, scale, k=2):
    tol = k * 2.0 ** -23 * max(abs(want.real), abs(want.imag)) + 1e-12 * scale
    return abs(got.real - want.real) <= tol and abs(got.imag - want.imag) <= tol


# ------------------------------------------------------------------ oracle
@pytest.mark.parametrize("case", cases("l1s_"))
def test_oracle_level1_real(case):
    x, y, n, inc = g(case, "x"), g(case, "y"), int(g(case, "n")), int(g(case, "inc"))
    assert O.sdot(n, x, inc, y, inc) == g(case, "sdot")
    assert O.snrm2(n, x, inc) == g(case, "snrm2")
    assert O.sasum(n, x, inc) == g(case, "sasum")
    assert O.isamax(n, x, inc) == g(case, "isamax")
    y2 = y.copy()
    O.saxpy(n, float(g(case, "saxpy_alpha")), x, inc, y2, inc)
    assert np.array_equal(y2, g(case, "saxpy"))
    x2 = x.copy()
    O.sscal(n, float(g(case, "sscal_alpha")), x2, inc)
    assert np.array_equal(x2, g(case, "sscal"))


@pytest.mark.parametrize("case", cases("iamax_edge_"))
def test_oracle_iamax_edges(case):
    x = g(case, "x")
    assert O.isamax(len(x), x, 1) == g(case, "isamax")


@pytest.mark.parametrize("case", cases("l1c_"))
def test_oracle_level1_complex(case):
    x, y, n, inc = g(case, "x"), g(case, "y"), int(g(case, "n")), int(g(case, "inc"))
    assert O.cdot(n, x, inc, y, inc, False) == complex(g(case, "cdotu"))
    assert O.cdot(n, x, inc, y, inc, True) == complex(g(case, "cdotc"))
    assert O.scnrm2(n, x, inc) == g(case, "scnrm2")
    assert O.scasum(n, x, inc) == g(case, "scasum")
    assert O.icamax(n, x, inc) == g(case, "icamax")
    x2 = x.copy()
    O.cscal(n, complex(g(case, "cscal_alpha")), x2, inc)
    assert np.array_equal(x2, g(case, "cscal"))
    y2 = y.copy()
    O.caxpy(n, complex(g(case, "caxpy_alpha")), x, inc, y2, inc)
    assert np.max(np.abs(y2 - g(case, "caxpy"))) <= 4e-7 * (1 + np.max(np.abs(y2)))


@pytest.mark.parametrize("case", cases("sgemm_q_"))
def test_oracle_sgemm_quarter(case):
    ta, tb, m, n, k, lda, ldb, ldc = (int(v) for v in g(case, "dims"))
    al, be = (float(v) for v in g(case, "ab"))
    Cm = g(case, "C").copy()
    O.sgemm(ta, tb, m, n, k, al, g(case, "A"), lda, g(case, "B"), ldb, be, Cm, ldc)
    assert np.array_equal(Cm, g(case, "out"))


@pytest.mark.parametrize("case", cases("cgemm_"))
def test_oracle_cgemm(case):
    ta, tb, m, n, k, lda, ldb, ldc = (int(v) for v in g(case, "dims"))
    al, be = (complex(v) for v in g(case, "ab"))
    Cm = g(case, "C").copy()
    O.cgemm(ta, tb, m, n, k, al, g(case, "A"), lda, g(case, "B"), ldb, be, Cm, ldc)
    assert O.rel_fro(Cm, g(case, "out")) <= 1e-7


@pytest.mark.parametrize("case", cases("sgemv_") + cases("cgemv_"))
def test_oracle_gemv(case):
    trans, m, n, lda, incx, incy = (int(v) for v in g(case, "dims"))
    ab = g(case, "ab")
    y = g(case, "y").copy()
    if case.startswith("s"):
        O.sgemv(trans, m, n, float(ab[0]), g(case, "A"), lda, g(case, "x"), incx, float(ab[1]), y, incy)
    else:
        O.cgemv(trans, m, n, complex(ab[0]), g(case, "A"), lda, g(case, "x"), incx, complex(ab[1]), y, incy)
    assert O.rel_fro(y, g(case, "out")) <= 1e-6


@pytest.mark.parametrize("case", cases("strsv_") + cases("ctrsv_"))
def test_oracle_trsv(case):
    uplo, trans, diag, n, lda, inc = (int(v) for v in g(case, "dims"))
    x = g(case, "x").copy()
    (O.strsv if case.startswith("s") else O.ctrsv)(uplo, trans, diag, n, g(case, "A"), lda, x, inc)
    assert O.rel_fro(x, g(case, "out")) <= TOL


@pytest.mark.parametrize("case", cases("strsm_") + cases("ctrsm_"))
def test_oracle_trsm(case):
    side, uplo, trans, diag, m, n, lda, ldb = (int(v) for v in g(case, "dims"))
    Bm = g(case, "B").copy()
    al = g(case, "alpha")
    if case.startswith("s"):
        O.strsm(side, uplo, trans, diag, m, n, float(al), g(case, "A"), lda, Bm, ldb)
    else:
        O.ctrsm(side, uplo, trans, diag, m, n, complex(al), g(case, "A"), lda, Bm, ldb)
    assert O.rel_fro(Bm, g(case, "out")) <= TOL


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def same(a, b):
    """Bit-identical, except that any two NaNs match (the GPU writes a
    canonical NaN where the CPU propagates its operand's payload)."""
    fa = np.ascontiguousarray(a).view(np.float32)
    fb = np.ascontiguousarray(b).view(np.float32)
    return fa.shape == fb.shape and bool(np.all((bits(fa) == bits(fb)) | (np.isnan(fa) & np.isnan(fb))))


@pytest.mark.parametrize("case", cases("rot_"))
def test_oracle_rotations(case):
    n, incx, incy = (int(v) for v in g(case, "dims"))
    x, y, xc, yc = g(case, "x"), g(case, "y"), g(case, "xc"), g(case, "yc")
    c, s = (float(v) for v in g(case, "cs"))
    assert O.isamin(n, x, incx) == g(case, "isamin")
    assert O.icamin(n, xc, incx) == g(case, "icamin")
    for name, fn, a, b, arg in (("srot", O.srot, x, y, s), ("csrot", O.csrot, xc, yc, s),
                                ("crot", O.crot, xc, yc, complex(g(case, "sc")))):
        a1, b1 = a.copy(), b.copy()
        fn(n, a1, incx, b1, incy, c, arg)
        assert np.array_equal(bits(a1), bits(g(case, name + "_x"))), name
        assert np.array_equal(bits(b1), bits(g(case, name + "_y"))), name
    for flag in (-1, 0, 1):
        a1, b1 = x.copy(), y.copy()
        O.srotm(n, a1, incx, b1, incy, g(case, f"srotm{flag}_param"))
        assert np.array_equal(bits(a1), bits(g(case, f"srotm{flag}_x")))
        assert np.array_equal(bits(b1), bits(g(case, f"srotm{flag}_y")))


def test_oracle_rotation_generators():
    for (a, b), want in zip(g("srotg", "ab"), g("srotg", "out")):
        assert np.array_equal(bits(np.array(O.srotg(a, b), np.float32)), bits(want))
    for (a, b), want in zip(g("crotg", "ab"), g("crotg", "out")):
        ar, c, s = O.crotg(complex(a), complex(b))
        assert np.array_equal(bits(np.array([ar, c, s], np.complex64)), bits(want))
    for row, want in zip(g("srotmg", "in"), g("srotmg", "out")):
        param = np.full(5, 7, np.float32)
        v = O.srotmg(*row, param)
        assert np.array_equal(bits(np.array(v, np.float32)), bits(want[:3]))
        assert np.array_equal(bits(param), bits(want[3:]))


def _l23_cases():
    return cases("sger") + cases("cger") + cases("ssymv") + cases("chemv") + cases("ssyrk") + cases("ssyr2k") + \
        cases("ssymm")


def _l23_run(case, api):
    """Runs one level-2/3 golden case through `api` (the oracle wrappers or
    the GPU library); returns (result, expected, exact)."""
    if case == "sger":
        m, n, incx, incy, lda = (int(v) for v in g(case, "dims"))
        A = g(case, "A").copy()
        api["sger"](m, n, 0.75, g(case, "x"), incx, g(case, "y"), incy, A, lda)
        return A, g(case, "out"), True
    if case.startswith("cger"):
        m, n, incx, incy, lda = (int(v) for v in g(case, "dims"))
        A = g(case, "A").copy()
        api["cger"](case.endswith("1"), m, n, complex(g(case, "alpha")), g(case, "x"), incx, g(case, "y"), incy, A, lda)
        return A, g(case, "out"), True
    if case.startswith("ssymv"):
        uplo, n, lda, incx, incy = (int(v) for v in g(case, "dims"))
        y = g(case, "y").copy()
        api["ssymv"](uplo, n, 1.25, g(case, "A"), lda, g(case, "x"), incx, -0.5, y, incy)
        return y, g(case, "out"), False
    if case.startswith("chemv"):
        uplo, n, lda, incx, incy = (int(v) for v in g(case, "dims"))
        ab = g(case, "ab")
        y = g(case, "y").copy()
        api["chemv"](uplo, n, complex(ab[0]), g(case, "A"), lda, g(case, "x"), incx, complex(ab[1]), y, incy)
        return y, g(case, "out"), False
    if case.startswith("ssyr2k") or case.startswith("ssyrk"):
        uplo, trans, n, k, lda, ldc = (int(v) for v in g(case, "dims"))
        Cm = g(case, "C").copy()
        if case.startswith("ssyr2k"):
            api["ssyr2k"](uplo, trans, n, k, 0.75, g(case, "A"), lda, g(case, "B"), lda, -0.5, Cm, ldc)
        else:
            api["ssyrk"](uplo, trans, n, k, 0.75, g(case, "A"), lda, -0.5, Cm, ldc)
        return Cm, g(case, "out"), False
    side, uplo, m, n, lda, ldb, ldc = (int(v) for v in g(case, "dims"))
    Cm = g(case, "C").copy()
    api["ssymm"](side, uplo, m, n, 1.5, g(case, "A"), lda, g(case, "B"), ldb, 0.25, Cm, ldc)
    return Cm, g(case, "out"), False


ORACLE_API = {"sger": O.sger, "cger": O.cger, "ssymv": O.ssymv, "chemv": O.chemv, "ssyrk": O.ssyrk,
              "ssyr2k": O.ssyr2k, "ssymm": O.ssymm}


@pytest.mark.parametrize("case", _l23_cases())
def test_oracle_level23(case):
    got, want, exact = _l23_run(case, ORACLE_API)
    if exact:
        assert np.array_equal(bits(got), bits(want))
    else:
        assert O.rel_fro(got, want) <= TOL
        assert np.array_equal(np.isnan(got), np.isnan(want))


# ------------------------------------------------------------------ GPU library
@pytest.mark.gpu
def test_gpu_rotations_against_golden(handle):
    for case in cases("rot_"):
        n, incx, incy = (int(v) for v in g(case, "dims"))
        x, y, xc, yc = g(case, "x"), g(case, "y"), g(case, "xc"), g(case, "yc")
        c, s = (float(v) for v in g(case, "cs"))
        ri = np.zeros(1, np.int32)
        assert B.iclblasIsamin(handle, n, x, incx, ri) == B.SUCCESS and ri[0] == g(case, "isamin")
        assert B.iclblasIcamin(handle, n, xc, incx, ri) == B.SUCCESS and ri[0] == g(case, "icamin")
        for name, fn, a, b, arg in (("srot", B.iclblasSrot, x, y, s), ("csrot", B.iclblasCsrot, xc, yc, s),
                                    ("crot", B.iclblasCrot, xc, yc, complex(g(case, "sc")))):
            a1, b1 = a.copy(), b.copy()
            assert fn(handle, n, a1, incx, b1, incy, c, arg) == B.SUCCESS
            assert same(a1, g(case, name + "_x")), (case, name)
            assert same(b1, g(case, name + "_y")), (case, name)
        for flag in (-1, 0, 1):
            a1, b1 = x.copy(), y.copy()
            assert B.iclblasSrotm(handle, n, a1, incx, b1, incy, g(case, f"srotm{flag}_param").copy()) == B.SUCCESS
            assert same(a1, g(case, f"srotm{flag}_x")), (case, flag)
            assert same(b1, g(case, f"srotm{flag}_y")), (case, flag)


@pytest.mark.gpu
def test_gpu_rotation_generators_against_golden(handle):
    for (a, b), want in zip(g("srotg", "ab"), g("srotg", "out")):
        v = np.array([a, b, 0, 0], np.float32)
        assert B.iclblasSrotg(handle, v[0:], v[1:], v[2:], v[3:]) == B.SUCCESS
        assert same(v, want), (a, b)
    for (a, b), want in zip(g("crotg", "ab"), g("crotg", "out")):
        v = np.array([a, b, 0], np.complex64)
        cc = np.zeros(1, np.float32)
        assert B.iclblasCrotg(handle, v[0:], v[1:], cc, v[2:]) == B.SUCCESS
        assert same(np.array([v[0], cc[0], v[2]], np.complex64), want)
    for row, want in zip(g("srotmg", "in"), g("srotmg", "out")):
        v = row[:3].copy()
        y1 = row[3:4].copy()
        param = np.full(5, 7, np.float32)
        assert B.iclblasSrotmg(handle, v[0:], v[1:], v[2:], y1, param) == B.SUCCESS
        assert same(v, want[:3]) and same(param, want[3:]), row



@pytest.mark.gpu
def test_gpu_level1_against_golden(handle):
    for case in cases("l1s_"):
        x, y, n, inc = g(case, "x"), g(case, "y"), int(g(case, "n")), int(g(case, "inc"))
        r = np.zeros(1, np.float32)
        ri = np.zeros(1, np.int32)
        assert B.iclblasSdot(handle, n, x, inc, y, inc, r) == B.SUCCESS and ulps(r[0], g(case, "sdot")) <= 1
        assert B.iclblasSnrm2(handle, n, x, inc, r) == B.SUCCESS and ulps(r[0], g(case, "snrm2")) <= 1
        assert B.iclblasSasum(handle, n, x, inc, r) == B.SUCCESS and ulps(r[0], g(case, "sasum")) <= 1
        assert B.iclblasIsamax(handle, n, x, inc, ri) == B.SUCCESS and ri[0] == g(case, "isamax")
        y2 = y.copy()
        assert B.iclblasSaxpy(handle, n, float(g(case, "saxpy_alpha")), x, inc, y2, inc) == B.SUCCESS
        assert O.ulp_diff(y2, g(case, "saxpy")).max() <= 1
        x2 = x.copy()
        assert B.iclblasSscal(handle, n, float(g(case, "sscal_alpha")), x2, inc) == B.SUCCESS
        assert np.array_equal(x2, g(case, "sscal"))
    for case in cases("iamax_edge_"):
        x = g(case, "x")
        ri = np.zeros(1, np.int32)
        assert B.iclblasIsamax(handle, len(x), x, 1, ri) == B.SUCCESS and ri[0] == g(case, "isamax")
    for case in cases("l1c_"):
        x, y, n, inc = g(case, "x"), g(case, "y"), int(g(case, "n")), int(g(case, "inc"))
        scale = float(np.sum(np.abs(x) * np.abs(y)))
        r = np.zeros(1, np.complex64)
        assert B.iclblasCdotu(handle, n, x, inc, y, inc, r) == B.SUCCESS
        assert cnear(complex(r[0]), complex(g(case, "cdotu")), scale)
        assert B.iclblasCdotc(handle, n, x, inc, y, inc, r) == B.SUCCESS
        assert cnear(complex(r[0]), complex(g(case, "cdotc")), scale)
        rf = np.zeros(1, np.float32)
        assert B.iclblasScnrm2(handle, n, x, inc, rf) == B.SUCCESS and ulps(rf[0], g(case, "scnrm2")) <= 1
        assert B.iclblasScasum(handle, n, x, inc, rf) == B.SUCCESS and ulps(rf[0], g(case, "scasum")) <= 1
        ri = np.zeros(1, np.int32)
        assert B.iclblasIcamax(handle, n, x, inc, ri) == B.SUCCESS and ri[0] == g(case, "icamax")
        x2 = x.copy()
        assert B.iclblasCscal(handle, n, complex(g(case, "cscal_alpha")), x2, inc) == B.SUCCESS
        assert np.array_equal(x2, g(case, "cscal"))
        y2 = y.copy()
        assert B.iclblasCaxpy(handle, n, complex(g(case, "caxpy_alpha")), x, inc, y2, inc) == B.SUCCESS
        assert np.max(np.abs(y2 - g(case, "caxpy"))) <= 4e-7 * (1 + np.max(np.abs(y2)))


@pytest.mark.gpu
def test_gpu_level3_level2_against_golden(handle):
    for case in cases("sgemm_q_"):
        ta, tb, m, n, k, lda, ldb, ldc = (int(v) for v in g(case, "dims"))
        al, be = (float(v) for v in g(case, "ab"))
        Cm = g(case, "C").copy()
        assert B.iclblasSgemm(handle, ta, tb, m, n, k, al, g(case, "A"), lda, g(case, "B"), ldb, be, Cm,
                              ldc) == B.SUCCESS
        assert np.array_equal(Cm, g(case, "out")), case
    for case in cases("cgemm_"):
        ta, tb, m, n, k, lda, ldb, ldc = (int(v) for v in g(case, "dims"))
        al, be = (complex(v) for v in g(case, "ab"))
        Cm = g(case, "C").copy()
        assert B.iclblasCgemm(handle, ta, tb, m, n, k, al, g(case, "A"), lda, g(case, "B"), ldb, be, Cm,
                              ldc) == B.SUCCESS
        assert O.rel_fro(Cm, g(case, "out")) <= TOL, case
    for case in cases("sgemv_") + cases("cgemv_"):
        trans, m, n, lda, incx, incy = (int(v) for v in g(case, "dims"))
        ab = g(case, "ab")
        y = g(case, "y").copy()
        f = B.iclblasSgemv if case.startswith("s") else B.iclblasCgemv
        cv = float if case.startswith("s") else complex
        assert f(handle, trans, m, n, cv(ab[0]), g(case, "A"), lda, g(case, "x"), incx, cv(ab[1]), y,
                 incy) == B.SUCCESS
        assert O.rel_fro(y, g(case, "out")) <= TOL, case
    for case in cases("strsv_") + cases("ctrsv_"):
        uplo, trans, diag, n, lda, inc = (int(v) for v in g(case, "dims"))
        x = g(case, "x").copy()
        f = B.iclblasStrsv if case.startswith("s") else B.iclblasCtrsv
        assert f(handle, uplo, trans, diag, n, g(case, "A"), lda, x, inc) == B.SUCCESS
        assert O.rel_fro(x, g(case, "out")) <= TOL, case
    for case in cases("strsm_") + cases("ctrsm_"):
        side, uplo, trans, diag, m, n, lda, ldb = (int(v) for v in g(case, "dims"))
        Bm = g(case, "B").copy()
        al = g(case, "alpha")
        if case.startswith("s"):
            st = B.iclblasStrsm(handle, side, uplo, trans, diag, m, n, float(al), g(case, "A"), lda, Bm, ldb)
        else:
            st = B.iclblasCtrsm(handle, side, uplo, trans, diag, m, n, complex(al), g(case, "A"), lda, Bm, ldb)
        assert st == B.SUCCESS
        assert O.rel_fro(Bm, g(case, "out")) <= TOL, case


@pytest.mark.gpu
def test_gpu_level23_against_golden(handle):
    def st(fn):
        def call(*a):
            assert fn(handle, *a) == B.SUCCESS
        return call
    api = {"sger": st(B.iclblasSger),
           "cger": lambda conj, *a: st(B.iclblasCgerc if conj else B.iclblasCgeru)(*a),
           "ssymv": st(B.iclblasSsymv), "chemv": st(B.iclblasChemv), "ssyrk": st(B.iclblasSsyrk),
           "ssyr2k": st(B.iclblasSsyr2k), "ssymm": st(B.iclblasSsymm)}
    for case in _l23_cases():
        got, want, exact = _l23_run(case, api)
        if exact:
            assert same(got, want), case
        else:
            assert O.rel_fro(got, want) <= TOL, case
