"""Generates tests/golden/reference_cpu_vectors.npz from the reference's own CPU code.

Inputs are seeded here; outputs come from oracle/_ref/libiclref.so, i.e. the
reference's CPU templates (tests/blas_funcs/*.hpp: cpu_gemm, cpu_dot,
cpu_nrm2, cpu_asum, cpu_axpy, cpu_scal, cpu_amax; tests/blas_reference/
blas_reference.cpp: Isamax_reference, Caxpy_reference) and its serial OpenCL
kernels compiled as C++ (Sgemv/Cgemv/Strsv/Ctrsv/Strsm/Ctrsm/Sgemm/Cgemm
_naive.cl, the level-1 Isamin/Icamin/Srot/Csrot/Crot/Srotm/Srotg/Crotg/
Srotmg _naive.cl, and Sger/Cgeru/Cgerc/Ssyrk/Ssyr2k/Ssymm _naive.cl with the
cpu_symv template for Ssymv/Chemv), all built from the reference's sources by
oracle/Makefile.

Each case is stored under a key prefix "<case>/" with its inputs, scalar
parameters and the reference output.  The fixture is committed; run this
script (with the reference tree built into oracle/_ref) to regenerate it.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as O  # noqa: E402

OUT = os.path.join(HERE, "reference_cpu_vectors.npz")


def P(a):
    return a.ctypes.data


def tri(n, lda, lower, rng, dtype=np.float32):
    A = O.colmajor(n, n, lda, rng, dtype)
    M = A.reshape(n, lda).T[:n]
    d = rng.uniform(1, 2, n)
    if np.dtype(dtype) == np.complex64:
        d = d * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    off = (rng.standard_normal((n, n)) / np.sqrt(n)).astype(np.float32)
    mask = np.tril(np.ones((n, n), bool), -1) if lower else np.triu(np.ones((n, n), bool), 1)
    M[mask] = off[mask]
    M[np.arange(n), np.arange(n)] = d
    return A


def rotmg_passes_host_checks(d1, d2, x1, y1):
    """The reference's host-side Srotmg checks (libs/blas/shlib/iclBLAS_S.cpp:
    101-128) all pass, so its kernel runs."""
    f = np.float32
    return not (f(d1) < 0 or f(d2) == 0 or f(y1) == 0 or f(f(-f(d2) * f(y1)) * f(y1)) >= f(f(f(d1) * f(x1)) * f(x1)))


def rotation_cases(R, d):
    """iamin, rot, csrot, crot, rotm, rotg, crotg and rotmg through the
    reference's serial kernels (Isamin/Icamin/Srot/Csrot/Crot/Srotm/Srotg/
    Crotg/Srotmg _naive.cl); own seed, so the other cases stay unchanged."""
    rng = np.random.default_rng(20261204)
    for n, incx, incy in ((1000, 1, 1), (257, 2, 3)):
        k = f"rot_{n}_{incx}_{incy}/"
        x = rng.uniform(-4, 4, n * incx).astype(np.float32)
        y = rng.uniform(-4, 4, n * incy).astype(np.float32)
        xc = rng.uniform(-4, 4, (n * incx, 2)).astype(np.float32).view(np.complex64).reshape(-1)
        yc = rng.uniform(-4, 4, (n * incy, 2)).astype(np.float32).view(np.complex64).reshape(-1)
        d[k + "x"], d[k + "y"], d[k + "xc"], d[k + "yc"] = x, y, xc, yc
        d[k + "dims"] = np.array([n, incx, incy], np.int32)
        d[k + "isamin"] = np.int32(R.ref_naive_isamin(n, P(x), incx))
        d[k + "icamin"] = np.int32(R.ref_naive_icamin(n, P(xc), incx))
        c, s, sc = np.float32(0.6), np.float32(-0.8), np.complex64(0.25 - 0.5j)
        d[k + "cs"] = np.array([c, s], np.float32)
        d[k + "sc"] = sc
        x1, y1 = x.copy(), y.copy()
        R.ref_naive_srot(n, P(x1), incx, P(y1), incy, float(c), float(s))
        d[k + "srot_x"], d[k + "srot_y"] = x1, y1
        x1, y1 = xc.copy(), yc.copy()
        R.ref_naive_csrot(n, P(x1), incx, P(y1), incy, float(c), float(s))
        d[k + "csrot_x"], d[k + "csrot_y"] = x1, y1
        x1, y1 = xc.copy(), yc.copy()
        scb = O.cbox(sc)   # kept alive across the call
        R.ref_naive_crot(n, P(x1), incx, P(y1), incy, float(c), P(scb))
        d[k + "crot_x"], d[k + "crot_y"] = x1, y1
        for flag in (-1, 0, 1):
            param = np.array([flag, 0.75, -1.5, 2.25, 0.125], np.float32)
            x1, y1 = x.copy(), y.copy()
            R.ref_naive_srotm(n, P(x1), incx, P(y1), incy, P(param))
            d[k + f"srotm{flag}_param"] = param
            d[k + f"srotm{flag}_x"], d[k + f"srotm{flag}_y"] = x1, y1
    ab = np.concatenate([rng.uniform(-10, 10, (64, 2)),
                         [[0, 3], [3, 0], [0, 0], [-2, 2], [1, 1.5], [1e-20, 3e-20], [1e20, -7e19]]]).astype(np.float32)
    out = np.zeros((len(ab), 4), np.float32)
    for i, (a, b) in enumerate(ab):
        v = np.array([a, b, 0, 0], np.float32)
        R.ref_naive_srotg(P(v[0:]), P(v[1:]), P(v[2:]), P(v[3:]))
        out[i] = v
    d["srotg/ab"], d["srotg/out"] = ab, out
    abc = rng.uniform(-10, 10, (64, 4)).astype(np.float32).view(np.complex64)
    outc = np.zeros((64, 3), np.complex64)
    for i, (a, b) in enumerate(abc):
        v = np.array([a, b, 0], np.complex64)
        cc = np.zeros(1, np.float32)
        R.ref_naive_crotg(P(v[0:]), P(v[1:]), P(cc), P(v[2:]))
        outc[i] = [v[0], cc[0], v[2]]
    d["crotg/ab"], d["crotg/out"] = abc, outc
    rows = [r for r in rng.uniform(-2, 10, (200, 4)) if rotmg_passes_host_checks(*r)][:48]
    rows += [(1.1, -1.0, 3.3, 3.2), (0.0, 1.2, 3.3, 3.2), (1 / 4096 / 4096, 1 / 4096 / 4096, 3.3, 3.2),
             (1e-12, 2e-12, 1.0, 0.5), (1e9, 3e9, 2.0, 1.0), (5e8, 1e-10, 1.0, 4.0)]
    rows = np.array(rows, np.float32)
    outm = np.zeros((len(rows), 8), np.float32)
    for i, (d1, d2, x1, y1) in enumerate(rows):
        param = np.full(5, 7, np.float32)
        v = np.array([d1, d2, x1], np.float32)
        R.ref_naive_srotmg(P(v[0:]), P(v[1:]), P(v[2:]), float(y1), P(param))
        outm[i, :3], outm[i, 3:] = v, param
    d["srotmg/in"], d["srotmg/out"] = rows, outm


def level23_cases(R, d):
    """Sger / Cgeru / Cgerc through their serial kernels (bit-exact FP32
    expressions), Ssymv / Chemv through the cpu_symv template
    (tests/blas_funcs/test_symv.hpp, double), Ssyrk / Ssyr2k / Ssymm through
    their serial kernels (FP32 sums); own seed."""
    rng = np.random.default_rng(20261205)
    m, n, lda = 45, 31, 48
    x = rng.uniform(-2, 2, m * 2).astype(np.float32)
    y = rng.uniform(-2, 2, n).astype(np.float32)
    A = rng.uniform(-2, 2, lda * n).astype(np.float32)
    d["sger/x"], d["sger/y"], d["sger/A"] = x, y, A.copy()
    d["sger/dims"] = np.array([m, n, 2, 1, lda], np.int32)
    R.ref_naive_sger(m, n, 0.75, P(x), 2, P(y), 1, P(A), lda)
    d["sger/out"] = A
    xc = rng.uniform(-1, 1, (m, 2)).astype(np.float32).view(np.complex64).reshape(-1)
    yc = rng.uniform(-1, 1, (n * 3, 2)).astype(np.float32).view(np.complex64).reshape(-1)
    Ac = rng.uniform(-1, 1, (lda * n, 2)).astype(np.float32).view(np.complex64).reshape(-1)
    al = np.complex64(0.5 - 0.25j)
    alb = O.cbox(al)
    for conj in (0, 1):
        k = f"cger{conj}/"
        A1 = Ac.copy()
        d[k + "x"], d[k + "y"], d[k + "A"] = xc, yc, Ac.copy()
        d[k + "dims"] = np.array([m, n, 1, 3, lda], np.int32)
        d[k + "alpha"] = al
        R.ref_naive_cger(conj, m, n, P(alb), P(xc), 1, P(yc), 3, P(A1), lda)
        d[k + "out"] = A1
    for uplo in (0, 1):
        nn, ld = 77, 80
        k = f"ssymv{uplo}/"
        A = rng.uniform(-1, 1, ld * nn).astype(np.float32)
        x = rng.uniform(-1, 1, nn).astype(np.float32)
        y = rng.uniform(-1, 1, nn * 2).astype(np.float32)
        d[k + "A"], d[k + "x"], d[k + "y"] = A, x, y.copy()
        d[k + "dims"] = np.array([uplo, nn, ld, 1, 2], np.int32)
        R.ref_cpu_ssymv(uplo, nn, 1.25, P(A), ld, P(x), 1, -0.5, P(y), 2)
        d[k + "out"] = y
        k = f"chemv{uplo}/"
        A = rng.uniform(-1, 1, (ld * nn, 2)).astype(np.float32).view(np.complex64).reshape(-1)
        x = rng.uniform(-1, 1, (nn * 2, 2)).astype(np.float32).view(np.complex64).reshape(-1)
        y = rng.uniform(-1, 1, (nn, 2)).astype(np.float32).view(np.complex64).reshape(-1)
        ab = np.array([0.5 - 1j, 0.25 + 0.5j], np.complex64)
        ab0, ab1 = O.cbox(ab[0]), O.cbox(ab[1])
        d[k + "A"], d[k + "x"], d[k + "y"], d[k + "ab"] = A, x, y.copy(), ab
        d[k + "dims"] = np.array([uplo, nn, ld, 2, 1], np.int32)
        R.ref_cpu_chemv(uplo, nn, P(ab0), P(A), ld, P(x), 2, P(ab1), P(y), 1)
        d[k + "out"] = y
        for trans in (0, 1):
            nn, kk = 53, 21
            ld = (nn if trans == 0 else kk) + 3
            cols = kk if trans == 0 else nn
            A = rng.uniform(-1, 1, ld * cols).astype(np.float32)
            B = rng.uniform(-1, 1, ld * cols).astype(np.float32)
            C = rng.uniform(-1, 1, (nn + 1) * nn).astype(np.float32)
            for name, Bp in (("ssyrk", None), ("ssyr2k", B)):
                k = f"{name}{uplo}{trans}/"
                C1 = C.copy()
                d[k + "A"], d[k + "B"], d[k + "C"] = A, B, C
                d[k + "dims"] = np.array([uplo, trans, nn, kk, ld, nn + 1], np.int32)
                R.ref_naive_ssyr2k(uplo, trans, nn, kk, 0.75, P(A), ld, None if Bp is None else P(Bp), ld, -0.5,
                                   P(C1), nn + 1)
                d[k + "out"] = C1
        for side in (0, 1):
            mm, nn = 41, 27
            na = mm if side == 0 else nn
            k = f"ssymm{side}{uplo}/"
            A = rng.uniform(-1, 1, (na + 2) * na).astype(np.float32)
            B = rng.uniform(-1, 1, (mm + 1) * nn).astype(np.float32)
            C = rng.uniform(-1, 1, (mm + 3) * nn).astype(np.float32)
            C1 = C.copy()
            d[k + "A"], d[k + "B"], d[k + "C"] = A, B, C
            d[k + "dims"] = np.array([side, uplo, mm, nn, na + 2, mm + 1, mm + 3], np.int32)
            R.ref_naive_ssymm(side, uplo, mm, nn, 1.5, P(A), na + 2, P(B), mm + 1, 0.25, P(C1), mm + 3)
            d[k + "out"] = C1


def main():
    R = O.ref()
    if R is None:
        raise SystemExit("oracle/_ref/libiclref.so is missing: build the oracle with the reference tree present")
    rng = np.random.default_rng(20261203)
    d = {}

    # ---- level 1, real
    for n, inc in ((1000, 1), (513, 3)):
        k = f"l1s_{n}_{inc}/"
        x = rng.uniform(-1, 1, n * inc).astype(np.float32)
        y = rng.uniform(-1, 1, n * inc).astype(np.float32)
        d[k + "x"], d[k + "y"] = x, y
        d[k + "n"], d[k + "inc"] = np.int32(n), np.int32(inc)
        d[k + "sdot"] = np.float32(R.ref_cpu_sdot(n, P(x), inc, P(y), inc))
        d[k + "snrm2"] = np.float32(R.ref_cpu_snrm2(n, P(x), inc))
        d[k + "sasum"] = np.float32(R.ref_cpu_sasum(n, P(x), inc))
        d[k + "isamax"] = np.int32(R.ref_cpu_isamax(n, P(x), inc))
        y2 = y.copy()
        R.ref_cpu_saxpy(n, 0.75, P(x), inc, P(y2), inc)
        d[k + "saxpy_alpha"], d[k + "saxpy"] = np.float32(0.75), y2
        x2 = x.copy()
        R.ref_cpu_sscal(n, -1.5, P(x2), inc)
        d[k + "sscal_alpha"], d[k + "sscal"] = np.float32(-1.5), x2
    # ties and NaN for iamax
    for i, x in enumerate((np.array([1, -5, 3, 5, -5, 2], np.float32),
                           np.array([np.nan, 1, 7, 2, 9], np.float32),
                           np.array([1, np.nan, 7, 2, 7], np.float32))):
        k = f"iamax_edge_{i}/"
        d[k + "x"] = x
        d[k + "isamax"] = np.int32(R.ref_cpu_isamax(len(x), P(x), 1))

    # ---- level 1, complex
    for n, inc in ((777, 1), (301, 2)):
        k = f"l1c_{n}_{inc}/"
        x = O.colmajor(n * inc, 1, n * inc, rng, np.complex64)
        y = O.colmajor(n * inc, 1, n * inc, rng, np.complex64)
        d[k + "x"], d[k + "y"] = x, y
        d[k + "n"], d[k + "inc"] = np.int32(n), np.int32(inc)
        for conj, nm in ((0, "cdotu"), (1, "cdotc")):
            out = np.zeros(2, np.float32)
            R.ref_cpu_cdot(n, P(x), inc, P(y), inc, conj, P(out))
            d[k + nm] = np.complex64(complex(out[0], out[1]))
        d[k + "scnrm2"] = np.float32(R.ref_cpu_scnrm2(n, P(x), inc))
        d[k + "scasum"] = np.float32(R.ref_cpu_scasum(n, P(x), inc))
        d[k + "icamax"] = np.int32(R.ref_cpu_icamax(n, P(x), inc))
        a = np.complex64(0.5 - 0.25j)
        ab = O.cbox(a)
        x2 = x.copy()
        R.ref_cpu_cscal(n, P(ab), P(x2), inc)
        d[k + "cscal_alpha"], d[k + "cscal"] = a, x2
        y2 = y.copy()
        xc = x.copy()
        R.ref_caxpy_reference(n, P(ab), P(xc), inc, P(y2), inc)
        d[k + "caxpy_alpha"], d[k + "caxpy"] = a, y2

    # ---- SGEMM: quarter-integer values (exact) through cpu_gemm, all op pairs
    m, n, kk = 24, 20, 28
    for ta in (0, 1, 2):
        for tb in (0, 1, 2):
            for beta in (0.0, 0.5):
                k = f"sgemm_q_{ta}{tb}_{int(beta * 10)}/"
                ar, ac = (m, kk) if ta == 0 else (kk, m)
                br, bc = (kk, n) if tb == 0 else (n, kk)
                lda, ldb, ldc = ar + 1, br + 3, m + 2
                A = O.quarter_ints(lda * ac, rng)
                Bm = O.quarter_ints(ldb * bc, rng)
                Cm = O.quarter_ints(ldc * n, rng)
                d[k + "A"], d[k + "B"], d[k + "C"] = A, Bm, Cm.copy()
                d[k + "dims"] = np.array([ta, tb, m, n, kk, lda, ldb, ldc], np.int32)
                d[k + "ab"] = np.array([1.5, beta], np.float32)
                R.ref_cpu_sgemm(ta, tb, m, n, kk, 1.5, P(A), lda, P(Bm), ldb, beta, P(Cm), ldc)
                d[k + "out"] = Cm
    # ---- CGEMM: random values through cpu_gemm<complex> (double accumulator)
    m, n, kk = 14, 12, 16
    for ta in (0, 1, 2):
        for tb in (0, 1, 2):
            k = f"cgemm_{ta}{tb}/"
            ar, ac = (m, kk) if ta == 0 else (kk, m)
            br, bc = (kk, n) if tb == 0 else (n, kk)
            A = O.colmajor(ar, ac, ar, rng, np.complex64)
            Bm = O.colmajor(br, bc, br, rng, np.complex64)
            Cm = O.colmajor(m, n, m, rng, np.complex64)
            al, be = np.complex64(1.5 - 0.5j), np.complex64(0.25 + 1j)
            alb, beb = O.cbox(al), O.cbox(be)
            d[k + "A"], d[k + "B"], d[k + "C"] = A, Bm, Cm.copy()
            d[k + "dims"] = np.array([ta, tb, m, n, kk, ar, br, m], np.int32)
            d[k + "ab"] = np.array([al, be], np.complex64)
            R.ref_cpu_cgemm(ta, tb, m, n, kk, P(alb), P(A), ar, P(Bm), br, P(beb), P(Cm), m)
            d[k + "out"] = Cm

    # ---- GEMV through the serial kernels
    m, n, lda = 40, 27, 43
    for trans in (0, 1, 2):
        k = f"sgemv_{trans}/"
        A = O.colmajor(m, n, lda, rng)
        xl, yl = (n, m) if trans == 0 else (m, n)
        x = rng.uniform(-1, 1, xl * 2).astype(np.float32)
        y = rng.uniform(-1, 1, yl * 3).astype(np.float32)
        d[k + "A"], d[k + "x"], d[k + "y"] = A, x, y.copy()
        d[k + "dims"] = np.array([trans, m, n, lda, 2, 3], np.int32)
        d[k + "ab"] = np.array([0.75, -0.5], np.float32)
        R.ref_naive_sgemv(trans, m, n, 0.75, P(A), lda, P(x), 2, -0.5, P(y), 3)
        d[k + "out"] = y
        k = f"cgemv_{trans}/"
        A = O.colmajor(m, n, lda, rng, np.complex64)
        x = O.colmajor(xl, 1, xl, rng, np.complex64)
        y = O.colmajor(yl, 1, yl, rng, np.complex64)
        al, be = np.complex64(0.5 + 1j), np.complex64(1 - 0.5j)
        alb, beb = O.cbox(al), O.cbox(be)
        d[k + "A"], d[k + "x"], d[k + "y"] = A, x, y.copy()
        d[k + "dims"] = np.array([trans, m, n, lda, 1, 1], np.int32)
        d[k + "ab"] = np.array([al, be], np.complex64)
        R.ref_naive_cgemv(trans, m, n, P(alb), P(A), lda, P(x), 1, P(beb), P(y), 1)
        d[k + "out"] = y

    # ---- TRSV / TRSM through the serial kernels
    n, lda = 37, 39
    for uplo in (0, 1):
        for trans in (0, 1, 2):
            for diag in (0, 1):
                k = f"strsv_{uplo}{trans}{diag}/"
                A = tri(n, lda, uplo == 1, rng)
                x = rng.uniform(-1, 1, n * 2).astype(np.float32)
                d[k + "A"], d[k + "x"] = A, x.copy()
                d[k + "dims"] = np.array([uplo, trans, diag, n, lda, 2], np.int32)
                R.ref_naive_strsv(uplo, trans, diag, n, P(A), lda, P(x), 2)
                d[k + "out"] = x
                k = f"ctrsv_{uplo}{trans}{diag}/"
                A = tri(n, lda, uplo == 1, rng, np.complex64)
                x = O.colmajor(n, 1, n, rng, np.complex64)
                d[k + "A"], d[k + "x"] = A, x.copy()
                d[k + "dims"] = np.array([uplo, trans, diag, n, lda, 1], np.int32)
                R.ref_naive_ctrsv(uplo, trans, diag, n, P(A), lda, P(x), 1)
                d[k + "out"] = x
    m, n = 20, 13
    for side in (0, 1):
        for uplo in (0, 1):
            for trans in (0, 1, 2):
                for diag in (0, 1):
                    na = m if side == 0 else n
                    lda, ldb = na + 2, m + 3
                    k = f"strsm_{side}{uplo}{trans}{diag}/"
                    A = tri(na, lda, uplo == 1, rng)
                    Bm = O.colmajor(m, n, ldb, rng)
                    d[k + "A"], d[k + "B"] = A, Bm.copy()
                    d[k + "dims"] = np.array([side, uplo, trans, diag, m, n, lda, ldb], np.int32)
                    d[k + "alpha"] = np.float32(-0.75)
                    R.ref_naive_strsm(side, uplo, trans, diag, m, n, -0.75, P(A), lda, P(Bm), ldb)
                    d[k + "out"] = Bm
                    k = f"ctrsm_{side}{uplo}{trans}{diag}/"
                    A = tri(na, lda, uplo == 1, rng, np.complex64)
                    Bm = O.colmajor(m, n, ldb, rng, np.complex64)
                    al = np.complex64(0.5 - 1j)
                    alb = O.cbox(al)
                    d[k + "A"], d[k + "B"] = A, Bm.copy()
                    d[k + "dims"] = np.array([side, uplo, trans, diag, m, n, lda, ldb], np.int32)
                    d[k + "alpha"] = al
                    R.ref_naive_ctrsm(side, uplo, trans, diag, m, n, P(alb), P(A), lda, P(Bm), ldb)
                    d[k + "out"] = Bm

    rotation_cases(R, d)
    level23_cases(R, d)

    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT}: {len(d)} arrays, {os.path.getsize(OUT) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
