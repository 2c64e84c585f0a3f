/*
 * CPU oracle for the iclBLAS hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference's CPU algorithms.  Only the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark use it,
 * as the checker; the GPU library never calls it.  Every function cites the
 * reference file:line it restates (paths relative to the clGPU tree).
 *
 * Pinning: tests/golden/ holds the reference's own C-API known-answer suite
 * compiled against oracle_capi.c (this oracle behind the iclBLAS C API), and
 * the reference's CPU templates compiled from their own sources into
 * oracle/_ref/ (oracle/Makefile) are compared with these functions on seeded
 * random inputs by tests/test_oracle.py.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cd;

static inline cd cd_make(double re, double im) { cd r = { re, im }; return r; }
static inline cd cd_of(orc_c32 a) { return cd_make(a.re, a.im); }
static inline cd cd_add(cd a, cd b) { return cd_make(a.re + b.re, a.im + b.im); }
static inline cd cd_sub(cd a, cd b) { return cd_make(a.re - b.re, a.im - b.im); }
static inline cd cd_mul(cd a, cd b) { return cd_make(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cd cd_conj(cd a) { return cd_make(a.re, -a.im); }
static inline cd cd_div(cd a, cd b)
{
    double d = b.re * b.re + b.im * b.im;
    return cd_make((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}
static inline orc_c32 c32_of(cd a) { orc_c32 r = { (float)a.re, (float)a.im }; return r; }

/* ------------------------------------------------------------------------ */
/* Level 1                                                                  */
/* ------------------------------------------------------------------------ */

/* y += alpha*x in double, rounded once.
 * Restates cpu_axpy (tests/blas_funcs/test_axpy.hpp:22-46). */
void orc_saxpy(int n, float alpha, const float* x, int incx, float* y, int incy)
{
    double a = alpha;
    for (int i = 0; i < n; ++i) {
        double r = (double)y[(long)i * incy] + a * (double)x[(long)i * incx];
        y[(long)i * incy] = (float)r;
    }
}

/* x *= alpha.  Restates cpu_scal (tests/blas_funcs/test_scal.hpp:27-39). */
void orc_sscal(int n, float alpha, float* x, int incx)
{
    double a = alpha;
    for (int i = 0; i < n; ++i)
        x[(long)i * incx] = (float)((double)x[(long)i * incx] * a);
}

/* sum x*y in double.  Restates cpu_dot (tests/blas_funcs/test_dot.hpp:22-51). */
float orc_sdot(int n, const float* x, int incx, const float* y, int incy)
{
    double acc = 0.0;
    for (int i = 0; i < n; ++i)
        acc += (double)x[(long)i * incx] * (double)y[(long)i * incy];
    return (float)acc;
}

/* Scaled two-norm (LAPACK-style scale/ssq update) in double.
 * Restates cpu_nrm2 (tests/blas_funcs/test_nrm2.hpp:23-57). */
float orc_snrm2(int n, const float* x, int incx)
{
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < n; ++i) {
        double ax = fabs((double)x[(long)i * incx]);
        if (ax != 0.0) {
            if (scale < ax) {
                double r = scale / ax;
                ssq = 1.0 + r * r * ssq;
                scale = ax;
            } else {
                double r = ax / scale;
                ssq += r * r;
            }
        }
    }
    return (float)(scale * sqrt(ssq));
}

/* sum |x| in double.  Restates cpu_asum (tests/blas_funcs/test_asum.hpp:23-33). */
float orc_sasum(int n, const float* x, int incx)
{
    double acc = 0.0;
    for (int i = 0; i < n; ++i)
        acc += fabs((double)x[(long)i * incx]);
    return (float)acc;
}

/* 0-based index of the first maximal |x|, strict '>' scan starting from x[0].
 * Restates amax_reference_impl (tests/blas_reference/blas_reference.cpp:46-64)
 * with the -1 of cpu_amax<float> (tests/blas_funcs/test_amax.hpp:45-53).
 * A NaN in x[0] pins the answer to 0; later NaNs are never selected. */
int orc_isamax(int n, const float* x, int incx)
{
    if (n < 1 || incx < 1) return 0;
    float best = fabsf(x[0]);
    int idx = 0;
    for (int i = 1; i < n; ++i) {
        float v = fabsf(x[(long)i * incx]);
        if (v > best) { best = v; idx = i; }
    }
    return idx;
}

/* y += alpha*x, complex, in double.  Restates cpu_axpy for complex<float>
 * (tests/blas_funcs/test_axpy.hpp:22-46, acc = complex<double>). */
void orc_caxpy(int n, orc_c32 alpha, const orc_c32* x, int incx, orc_c32* y, int incy)
{
    cd a = cd_of(alpha);
    for (int i = 0; i < n; ++i) {
        cd r = cd_add(cd_of(y[(long)i * incy]), cd_mul(a, cd_of(x[(long)i * incx])));
        y[(long)i * incy] = c32_of(r);
    }
}

/* x *= alpha, complex.  Restates cpu_scal (tests/blas_funcs/test_scal.hpp:27-39);
 * Csscal is this with alpha = (a, 0) (libs/blas/shlib/iclBLAS_C.cpp:78-84). */
void orc_cscal(int n, orc_c32 alpha, orc_c32* x, int incx)
{
    cd a = cd_of(alpha);
    for (int i = 0; i < n; ++i)
        x[(long)i * incx] = c32_of(cd_mul(cd_of(x[(long)i * incx]), a));
}

/* sum conj?(x)*y in complex<double>.  Restates cpu_dot<complex, conj>
 * (tests/blas_funcs/test_dot.hpp:22-51); conj_x selects cdotc. */
orc_c32 orc_cdot(int n, const orc_c32* x, int incx, const orc_c32* y, int incy, int conj_x)
{
    cd acc = cd_make(0.0, 0.0);
    for (int i = 0; i < n; ++i) {
        cd xv = cd_of(x[(long)i * incx]);
        if (conj_x) xv = cd_conj(xv);
        acc = cd_add(acc, cd_mul(xv, cd_of(y[(long)i * incy])));
    }
    return c32_of(acc);
}

/* Scaled two-norm over real and imaginary parts (every component is one
 * term of the scale/ssq update), in double.  cpu_nrm2 takes abs() of a
 * complex<double> (tests/blas_funcs/test_nrm2.hpp:23-57), i.e. the modulus
 * per element; sqrt(sum |x_i|^2) is the same quantity. */
float orc_scnrm2(int n, const orc_c32* x, int incx)
{
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < n; ++i) {
        cd v = cd_of(x[(long)i * incx]);
        double ax = hypot(v.re, v.im);
        if (ax != 0.0) {
            if (scale < ax) {
                double r = scale / ax;
                ssq = 1.0 + r * r * ssq;
                scale = ax;
            } else {
                double r = ax / scale;
                ssq += r * r;
            }
        }
    }
    return (float)(scale * sqrt(ssq));
}

/* sum |re|+|im| in double.  Restates cpu_asum with blas_abs of a complex
 * (tests/blas_funcs/test_asum.hpp:23-33, test_helpers.hpp:241-246). */
float orc_scasum(int n, const orc_c32* x, int incx)
{
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
        cd v = cd_of(x[(long)i * incx]);
        acc += fabs(v.re) + fabs(v.im);
    }
    return (float)acc;
}

/* 0-based first index of max |re|+|im| in float.  Restates cpu_amax<complex>
 * (tests/blas_funcs/test_amax.hpp:24-42) with scabs1 (core/src/ocl/complex.h.cl:54). */
int orc_icamax(int n, const orc_c32* x, int incx)
{
    if (n < 1 || incx < 1) return 0;
    float best = fabsf(x[0].re) + fabsf(x[0].im);
    int idx = 0;
    for (int i = 1; i < n; ++i) {
        const orc_c32 v = x[(long)i * incx];
        float a = fabsf(v.re) + fabsf(v.im);
        if (a > best) { best = a; idx = i; }
    }
    return idx;
}

/* ------------------------------------------------------------------------ */
/* Level 1: iamin, copy, swap, plane rotations and their generators         */
/* ------------------------------------------------------------------------ */
/* These restate the reference's OpenCL kernels expression by expression in
 * FP32 (this file is compiled with -ffp-contract=off: a product is rounded
 * before it is added unless the kernel writes fma/mad, restated as fmaf). */

/* First index of the smallest |x_i|: Isamin_naive.cl:16-33 (strict '<'
 * scan from x[0]). */
int orc_isamin(int n, const float* x, int incx)
{
    if (n < 1 || incx < 1) return 0;
    float best = fabsf(x[0]);
    int idx = 0;
    for (int i = 1; i < n; ++i) {
        float v = fabsf(x[(long)i * incx]);
        if (v < best) { best = v; idx = i; }
    }
    return idx;
}

/* Icamin_naive.cl:22-44, key scabs1 = |re| + |im|. */
int orc_icamin(int n, const orc_c32* x, int incx)
{
    if (n < 1 || incx < 1) return 0;
    float best = fabsf(x[0].re) + fabsf(x[0].im);
    int idx = 0;
    for (int i = 1; i < n; ++i) {
        const orc_c32 v = x[(long)i * incx];
        float a = fabsf(v.re) + fabsf(v.im);
        if (a < best) { best = a; idx = i; }
    }
    return idx;
}

/* y_i = x_i for elements of esize bytes: copy_interleave_naive.cl:16-23. */
void orc_copy(int n, const void* x, int incx, void* y, int incy, int esize)
{
    for (long i = 0; i < n; ++i)
        memcpy((char*)y + i * incy * esize, (const char*)x + i * incx * esize, (size_t)esize);
}

/* x_i <-> y_i: swap_interleave_naive.cl:16-26. */
void orc_swap(int n, void* x, int incx, void* y, int incy, int esize)
{
    char t[16];
    for (long i = 0; i < n; ++i) {
        char* a = (char*)x + i * incx * esize;
        char* b = (char*)y + i * incy * esize;
        memcpy(t, a, (size_t)esize);
        memcpy(a, b, (size_t)esize);
        memcpy(b, t, (size_t)esize);
    }
}

/* Srot_naive.cl:16-35: sy = s*y, cy = c*y, x' = fma(c, x, sy),
 * y' = fma(-s, x, cy). */
static void rot1(float* x, float* y, float c, float s)
{
    const float sy = s * *y, cy = c * *y;
    const float nx = fmaf(c, *x, sy);
    *y = fmaf(-s, *x, cy);
    *x = nx;
}

void orc_srot(int n, float* x, int incx, float* y, int incy, float c, float s)
{
    for (long i = 0; i < n; ++i) rot1(x + i * incx, y + i * incy, c, s);
}

/* Csrot_naive.cl:16-25: the same map per real component
 * (cfmaf(x, c, y*s) = fma(x, c, y*s) componentwise). */
void orc_csrot(int n, orc_c32* x, int incx, orc_c32* y, int incy, float c, float s)
{
    for (long i = 0; i < n; ++i) {
        orc_c32* a = x + i * incx;
        orc_c32* b = y + i * incy;
        rot1(&a->re, &b->re, c, s);
        rot1(&a->im, &b->im, c, s);
    }
}

/* cmul with the reference's fma placement (core/src/ocl/complex.h.cl:32-34) */
static orc_c32 cmul_fma(orc_c32 a, orc_c32 b)
{
    orc_c32 r;
    r.re = fmaf(a.re, b.re, -(a.im * b.im));
    r.im = fmaf(a.re, b.im, a.im * b.re);
    return r;
}

/* Crot_naive.cl:16-25: x' = x c + s y, y' = y c - conj(s) x. */
void orc_crot(int n, orc_c32* x, int incx, orc_c32* y, int incy, float c, orc_c32 s)
{
    const orc_c32 mcs = { -s.re, s.im };
    for (long i = 0; i < n; ++i) {
        orc_c32* a = x + i * incx;
        orc_c32* b = y + i * incy;
        const orc_c32 sy = cmul_fma(s, *b);
        const orc_c32 mx = cmul_fma(mcs, *a);
        orc_c32 nx, ny;
        nx.re = fmaf(a->re, c, sy.re);
        nx.im = fmaf(a->im, c, sy.im);
        ny.re = fmaf(b->re, c, mx.re);
        ny.im = fmaf(b->im, c, mx.im);
        *a = nx;
        *b = ny;
    }
}

/* Modified rotation, the reference's parameter layout
 * (Srotm_naive.cl:18-48 with Srotm_helpers.h.cl:27-41; mad as fmaf):
 *   flag -1: x' = p1 x + p2 y, y' = p3 x + p4 y
 *   flag  0: x' = x + p2 y,    y' = p3 x + y
 *   flag  1: x' = p1 x + y,    y' = p4 y - x
 * any other flag leaves x and y unchanged. */
void orc_srotm(int n, float* x, int incx, float* y, int incy, const float* p)
{
    const float f = p[0];
    if (!(f == -1.f || f == 0.f || f == 1.f)) return;
    for (long i = 0; i < n; ++i) {
        float* a = x + i * incx;
        float* b = y + i * incy;
        const float xv = *a, yv = *b;
        float nx, ny;
        if (f == -1.f) { nx = fmaf(p[1], xv, p[2] * yv); ny = fmaf(p[3], xv, p[4] * yv); }
        else if (f == 0.f) { nx = fmaf(p[2], yv, xv); ny = fmaf(p[3], xv, yv); }
        else { nx = fmaf(p[1], xv, yv); ny = fmaf(p[4], yv, -xv); }
        *a = nx;
        *b = ny;
    }
}

/* OpenCL sign(): 1, -1, or 0 for zero and NaN. */
static float ocl_sign(float v) { return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f); }

/* Srotg_naive.cl:16-56, including scale = |a| * |b| (zero when either input
 * is zero, giving c = 1, s = 0, r = z = 0). */
void orc_srotg(float* a, float* b, float* c, float* s)
{
    const float av = *a, bv = *b;
    const float fa = fabsf(av), fb = fabsf(bv);
    const float roe = fa > fb ? av : bv;
    const float scale = fa * fb;
    float r, z;
    if (scale == 0.f) {
        *c = 1.f; *s = 0.f; r = 0.f; z = 0.f;
    } else {
        const float a2 = av / scale, b2 = bv / scale;
        const float sg = ocl_sign(roe) * scale;
        r = sg * sqrtf(a2 * a2 + b2 * b2);
        *c = av / r;
        *s = bv / r;
        z = 1.f;
        if (fa > fb) z = *s;
        if (fb >= fa && *c != 0.f) z = 1.f / *c;
    }
    *a = r;
    *b = z;
}

/* |v| as cabs (complex.h.cl:28-30): sqrt(fma(re, re, im*im)). */
static float cabs_fma(orc_c32 v) { return sqrtf(fmaf(v.re, v.re, v.im * v.im)); }

/* Crotg_naive.cl:16-44. */
void orc_crotg(orc_c32* a, orc_c32* b, float* c, orc_c32* s)
{
    const orc_c32 av = *a, bv = *b;
    const float fa = cabs_fma(av), fb = cabs_fma(bv);
    if (fa == 0.f) {
        *c = 0.f;
        s->re = 1.f; s->im = 0.f;
        *a = bv;
        return;
    }
    const float scale = fa + fb;
    orc_c32 as = { av.re / scale, av.im / scale }, bs = { bv.re / scale, bv.im / scale };
    const float da = cabs_fma(as), db = cabs_fma(bs);
    const float norm = scale * sqrtf(da * da + db * db);
    const orc_c32 alpha = { av.re / fa, av.im / fa };
    *c = fa / norm;
    const orc_c32 cb = { bv.re, -bv.im };
    const orc_c32 t = cmul_fma(cb, alpha);
    s->re = t.re / norm;
    s->im = t.im / norm;
    a->re = alpha.re * norm;
    a->im = alpha.im * norm;
}

/* Modified Givens generator: the reference's host-side checks
 * (libs/blas/shlib/iclBLAS_S.cpp:101-128) then its kernel
 * (Srotmg_naive.cl:16-143).  The rescaling loops are capped at 16 steps
 * (finite values need at most 12; the reference's loop never ends for an
 * infinite d1 or d2). */
void orc_srotmg(float* d1, float* d2, float* x1, float y1, float* param)
{
    float dd1 = *d1, dd2 = *d2, bb1 = *x1;
    const float bb2 = y1;
    if (dd1 < 0.f) { param[0] = -1.f; param[1] = param[2] = param[3] = param[4] = 0.f; return; }
    if (dd2 == 0.f || bb2 == 0.f) { param[0] = -2.f; return; }
    if (-dd2 * bb2 * bb2 >= dd1 * bb1 * bb1) {
        param[0] = -1.f; param[1] = param[2] = param[3] = param[4] = 0.f; return;
    }
    const float p1 = dd1 * bb1, p2 = dd2 * bb2;
    const float q1 = p1 * bb1, q2 = p2 * bb2;
    float h11 = 0.f, h12 = 0.f, h21 = 0.f, h22 = 0.f, flag;
    if (q1 > fabsf(q2)) {
        h12 = p2 / p1;
        h21 = -bb2 / bb1;
        const float u = 1.f - h12 * h21;
        flag = 0.f;
        if (u > 0.f) { dd1 /= u; dd2 /= u; bb1 *= u; }
    } else {
        h11 = p1 / p2;
        h22 = bb1 / bb2;
        const float u = 1.f + h11 * h22;
        const float v = dd1 / u;
        flag = 1.f;
        dd1 = dd2 / u;
        dd2 = v;
        bb1 = bb2 * u;
    }
    const float g = 4096.f, gsq = g * g, gmsq = 1.f / gsq;
    if (dd1 != 0.f && (fabsf(dd1) < gmsq || fabsf(dd1) > gsq)) {
        if (flag == 0.f) { h11 = 1.f; h22 = 1.f; }
        else { h12 = 1.f; h21 = -1.f; }
        flag = -1.f;
        for (int it = 0; it < 16 && (fabsf(dd1) < gmsq || fabsf(dd1) > gsq); ++it) {
            if (fabsf(dd1) < gmsq) { dd1 *= gsq; bb1 /= g; h11 /= g; h12 /= g; }
            else { dd1 /= gsq; bb1 *= g; h11 *= g; h12 *= g; }
        }
    }
    if (dd2 != 0.f && (fabsf(dd2) < gmsq || fabsf(dd2) > gsq)) {
        if (flag == 0.f) { h11 = 1.f; h22 = 1.f; flag = -1.f; }
        else if (flag == 1.f) { h12 = 1.f; h21 = -1.f; flag = -1.f; }
        for (int it = 0; it < 16 && (fabsf(dd2) < gmsq || fabsf(dd2) > gsq); ++it) {
            if (fabsf(dd2) < gmsq) { dd2 *= gsq; h21 /= g; h22 /= g; }
            else { dd2 /= gsq; h21 *= g; h22 *= g; }
        }
    }
    param[0] = flag;
    if (flag == -1.f) { param[1] = h11; param[2] = h21; param[3] = h12; param[4] = h22; }
    else if (flag == 0.f) { param[2] = h21; param[3] = h12; }
    else { param[1] = h11; param[4] = h22; }
    *d1 = dd1;
    *d2 = dd2;
    *x1 = bb1;
}

/* ------------------------------------------------------------------------ */
/* Level 2                                                                  */
/* ------------------------------------------------------------------------ */

/* y = alpha*op(A)*x + beta*y, double accumulation; beta == 0 means y is
 * written without being read.  Restates Sgemv_naive
 * (libs/blas/funcs/Sgemv/Sgemv_naive.cl:22-59; the beta != 0 test at :34,54). */
void orc_sgemv(int trans, int m, int n, float alpha, const float* A, int lda,
               const float* x, int incx, float beta, float* y, int incy)
{
    int rows = (trans == 0) ? m : n;
    int cols = (trans == 0) ? n : m;
    for (int r = 0; r < rows; ++r) {
        double acc = 0.0;
        for (int c = 0; c < cols; ++c) {
            double a = (trans == 0) ? A[(long)c * lda + r] : A[(long)r * lda + c];
            acc += a * (double)x[(long)c * incx];
        }
        double out = (double)alpha * acc;
        if (beta != 0.0f) out += (double)beta * (double)y[(long)r * incy];
        y[(long)r * incy] = (float)out;
    }
}

/* Complex GEMV, op in {N, T, C}.  Restates Cgemv_naive
 * (libs/blas/funcs/Cgemv/Cgemv_naive.cl:16-50), accumulated in double.  The
 * reference kernel always reads y (:27,37,47); here, as for SGEMV, beta == 0
 * means y is not read (identical for finite y). */
void orc_cgemv(int trans, int m, int n, orc_c32 alpha, const orc_c32* A, int lda,
               const orc_c32* x, int incx, orc_c32 beta, orc_c32* y, int incy)
{
    int rows = (trans == 0) ? m : n;
    int cols = (trans == 0) ? n : m;
    cd a = cd_of(alpha), b = cd_of(beta);
    int beta_zero = (beta.re == 0.0f && beta.im == 0.0f);
    for (int r = 0; r < rows; ++r) {
        cd acc = cd_make(0, 0);
        for (int c = 0; c < cols; ++c) {
            cd e = (trans == 0) ? cd_of(A[(long)c * lda + r]) : cd_of(A[(long)r * lda + c]);
            if (trans == 2) e = cd_conj(e);
            acc = cd_add(acc, cd_mul(e, cd_of(x[(long)c * incx])));
        }
        cd out = cd_mul(a, acc);
        if (!beta_zero) out = cd_add(out, cd_mul(b, cd_of(y[(long)r * incy])));
        y[(long)r * incy] = c32_of(out);
    }
}

/* Element (i,j) of op(A) for a triangular solve.  op: 0 = N, 1 = T, 2 = C
 * (conjugate transpose), 3 = conjugate without transpose (used by the
 * right-side complex solve). */
static inline cd tri_elem_c(const orc_c32* A, int lda, int i, int j, int op)
{
    switch (op) {
    case 0: return cd_of(A[(long)j * lda + i]);
    case 1: return cd_of(A[(long)i * lda + j]);
    case 2: return cd_conj(cd_of(A[(long)i * lda + j]));
    default: return cd_conj(cd_of(A[(long)j * lda + i]));
    }
}

/* Is op(A) lower triangular? */
static inline int op_lower(int uplo, int op)
{
    int lower = (uplo == 1);
    return (op == 0 || op == 3) ? lower : !lower;
}

/* In-place solve op(A) z = z (complex double). */
static void tri_solve_cd(int uplo, int op, int diag, int n, const orc_c32* A, int lda, cd* z)
{
    if (op_lower(uplo, op)) {
        for (int i = 0; i < n; ++i) {
            cd s = z[i];
            for (int j = 0; j < i; ++j) s = cd_sub(s, cd_mul(tri_elem_c(A, lda, i, j, op), z[j]));
            z[i] = diag == 0 ? cd_div(s, tri_elem_c(A, lda, i, i, op)) : s;
        }
    } else {
        for (int i = n - 1; i >= 0; --i) {
            cd s = z[i];
            for (int j = i + 1; j < n; ++j) s = cd_sub(s, cd_mul(tri_elem_c(A, lda, i, j, op), z[j]));
            z[i] = diag == 0 ? cd_div(s, tri_elem_c(A, lda, i, i, op)) : s;
        }
    }
}

static inline double tri_elem_d(const double* A, int lda, int i, int j, int op)
{
    return (op == 0 || op == 3) ? A[(long)j * lda + i] : A[(long)i * lda + j];
}

/* In-place solve op(A) z = z (real double). */
static void tri_solve_d(int uplo, int op, int diag, int n, const double* A, int lda, double* z)
{
    if (op_lower(uplo, op)) {
        for (int i = 0; i < n; ++i) {
            double s = z[i];
            for (int j = 0; j < i; ++j) s -= tri_elem_d(A, lda, i, j, op) * z[j];
            z[i] = diag == 0 ? s / tri_elem_d(A, lda, i, i, op) : s;
        }
    } else {
        for (int i = n - 1; i >= 0; --i) {
            double s = z[i];
            for (int j = i + 1; j < n; ++j) s -= tri_elem_d(A, lda, i, j, op) * z[j];
            z[i] = diag == 0 ? s / tri_elem_d(A, lda, i, i, op) : s;
        }
    }
}

/* Column-oriented left solve of op(A) Z = Z for `nrhs` columns of a
 * column-major double matrix; forward/back substitution by columns of op(A)
 * so that the op == N inner loop runs down contiguous columns of A. */
static void tri_solve_cols_d(int uplo, int op, int diag, int n, const double* A, int lda,
                             double* Z, long ldz, int nrhs)
{
    int lower = op_lower(uplo, op);
    for (int c = 0; c < nrhs; ++c) {
        double* z = Z + (long)c * ldz;
        if (op == 0 || op == 3) {
            if (lower) {
                for (int i = 0; i < n; ++i) {
                    if (diag == 0) z[i] /= A[(long)i * lda + i];
                    double xi = z[i];
                    const double* col = A + (long)i * lda;
                    for (int k = i + 1; k < n; ++k) z[k] -= col[k] * xi;
                }
            } else {
                for (int i = n - 1; i >= 0; --i) {
                    if (diag == 0) z[i] /= A[(long)i * lda + i];
                    double xi = z[i];
                    const double* col = A + (long)i * lda;
                    for (int k = 0; k < i; ++k) z[k] -= col[k] * xi;
                }
            }
        } else {
            tri_solve_d(uplo, op, diag, n, A, lda, z);
        }
    }
}

/* In-place solve op(A) z = z with float A and a double right-hand side,
 * op 0 = N, 1 = T.  Every case walks a contiguous column of A: the two
 * no-transpose cases as column updates (axpy form), the two transposed cases
 * as dot products with a column. */
static void tri_solve_fa(int uplo, int op, int diag, int n, const float* A, int lda, double* z)
{
    int lower = (uplo == 1);
    if (op == 0 && lower) {
        for (int i = 0; i < n; ++i) {
            const float* col = A + (long)i * lda;
            if (diag == 0) z[i] /= col[i];
            double xi = z[i];
            for (int k = i + 1; k < n; ++k) z[k] -= (double)col[k] * xi;
        }
    } else if (op == 0) {
        for (int i = n - 1; i >= 0; --i) {
            const float* col = A + (long)i * lda;
            if (diag == 0) z[i] /= col[i];
            double xi = z[i];
            for (int k = 0; k < i; ++k) z[k] -= (double)col[k] * xi;
        }
    } else if (lower) {
        for (int i = n - 1; i >= 0; --i) {
            const float* col = A + (long)i * lda;
            double s = z[i];
            for (int j = i + 1; j < n; ++j) s -= (double)col[j] * z[j];
            z[i] = diag == 0 ? s / col[i] : s;
        }
    } else {
        for (int i = 0; i < n; ++i) {
            const float* col = A + (long)i * lda;
            double s = z[i];
            for (int j = 0; j < i; ++j) s -= (double)col[j] * z[j];
            z[i] = diag == 0 ? s / col[i] : s;
        }
    }
}

/* Strsv: solve op(A) x = b in place, double accumulation.  Restates
 * Strsv_naive (libs/blas/funcs/Strsv/Strsv_naive.cl:20-73); op C is op T for
 * real data. */
void orc_strsv(int uplo, int trans, int diag, int n, const float* A, int lda, float* x, int incx)
{
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) z[i] = x[(long)i * incx];
    tri_solve_fa(uplo, trans == 0 ? 0 : 1, diag, n, A, lda, z);
    for (int i = 0; i < n; ++i) x[(long)i * incx] = (float)z[i];
    free(z);
}

/* Ctrsv with op in {N, T, C}.  Restates Ctrsv_naive
 * (libs/blas/funcs/Ctrsv/Ctrsv_naive.cl:20-96). */
void orc_ctrsv(int uplo, int trans, int diag, int n, const orc_c32* A, int lda, orc_c32* x, int incx)
{
    cd* z = (cd*)malloc(sizeof(cd) * (size_t)n);
    for (int i = 0; i < n; ++i) z[i] = cd_of(x[(long)i * incx]);
    tri_solve_cd(uplo, trans, diag, n, A, lda, z);
    for (int i = 0; i < n; ++i) x[(long)i * incx] = c32_of(z[i]);
    free(z);
}

/* ------------------------------------------------------------------------ */
/* Level 3                                                                  */
/* ------------------------------------------------------------------------ */

/* C = alpha*op(A)*op(B) + beta*C.  The accumulator is FP32 and each output
 * sums its k terms in increasing k with fused multiply-adds; the update is
 * fma(alpha, acc, beta*C), or alpha*acc without reading C when beta == 0.
 * Restates the reference's selected SGEMM kernels: the per-element FMA loop
 * of Sgemm_ntransAB (libs/blas/funcs/Sgemm/Sgemm_ntransAB.cl:16-40) and the
 * subgroup kernel's epilogue (libs/blas/funcs/gemm_n3_template.h.cl:493-511).
 * The reference's own 64^3 known-answer test compares against an FP32 loop
 * in this order (tests/iclBLAS/test_Sgemm.cpp:256-270) and fails a double
 * accumulator at 4 ulp, which is why this oracle is FP32; the double
 * accumulating cpu_gemm (tests/blas_funcs/test_gemm.hpp:124-201) agrees with
 * it exactly on the quarter-integer inputs its own tests use. */
void orc_sgemm(int transa, int transb, int m, int n, int k, float alpha,
               const float* A, int lda, const float* B, int ldb, float beta, float* C, int ldc)
{
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) {
            float acc = 0.0f;
            for (int p = 0; p < k; ++p) {
                float a = transa == 0 ? A[(long)p * lda + i] : A[(long)i * lda + p];
                float b = transb == 0 ? B[(long)j * ldb + p] : B[(long)p * ldb + j];
                acc = fmaf(a, b, acc);
            }
            float* c = &C[(long)j * ldc + i];
            if (beta == 0.0f) *c = alpha * acc;
            else *c = fmaf(alpha, acc, beta * *c);
        }
    }
}

/* Complex GEMM, op in {N, T, C} per operand.  Restates cpu_gemm for
 * complex<float> (tests/blas_funcs/test_gemm.hpp:60-201, conj helper :38-57). */
void orc_cgemm(int transa, int transb, int m, int n, int k, orc_c32 alpha,
               const orc_c32* A, int lda, const orc_c32* B, int ldb, orc_c32 beta, orc_c32* C, int ldc)
{
    cd al = cd_of(alpha), be = cd_of(beta);
    int beta_zero = (beta.re == 0.0f && beta.im == 0.0f);
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) {
            cd acc = cd_make(0, 0);
            for (int p = 0; p < k; ++p) {
                cd a = transa == 0 ? cd_of(A[(long)p * lda + i]) : cd_of(A[(long)i * lda + p]);
                cd b = transb == 0 ? cd_of(B[(long)j * ldb + p]) : cd_of(B[(long)p * ldb + j]);
                if (transa == 2) a = cd_conj(a);
                if (transb == 2) b = cd_conj(b);
                acc = cd_add(acc, cd_mul(a, b));
            }
            orc_c32* c = &C[(long)j * ldc + i];
            cd out = cd_mul(acc, al);
            if (!beta_zero) out = cd_add(out, cd_mul(cd_of(*c), be));
            *c = c32_of(out);
        }
    }
}

/* Strsm: op(A) X = alpha B (left) or X op(A) = alpha B (right); X overwrites
 * B.  Restates Strsm_naive (libs/blas/funcs/Strsm/Strsm_naive.cl:18-126): the
 * solve runs on the unscaled B and alpha multiplies each solved entry on the
 * store (:35).  Arithmetic in double. */
void orc_strsm(int side, int uplo, int trans, int diag, int m, int n, float alpha,
               const float* A, int lda, float* B, int ldb)
{
    int op = (trans == 0) ? 0 : 1;
    if (side == 0) {
        double* z = (double*)malloc(sizeof(double) * (size_t)m);
        for (int j = 0; j < n; ++j) {
            for (int i = 0; i < m; ++i) z[i] = B[(long)j * ldb + i];
            tri_solve_fa(uplo, op, diag, m, A, lda, z);
            for (int i = 0; i < m; ++i) B[(long)j * ldb + i] = (float)(z[i] * (double)alpha);
        }
        free(z);
    } else {
        /* X op(A) = B  <=>  op(A)^T X^T = B^T: each row of B is solved with
         * the transposed operator. */
        double* z = (double*)malloc(sizeof(double) * (size_t)n);
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < n; ++j) z[j] = B[(long)j * ldb + i];
            tri_solve_fa(uplo, 1 - op, diag, n, A, lda, z);
            for (int j = 0; j < n; ++j) B[(long)j * ldb + i] = (float)(z[j] * (double)alpha);
        }
        free(z);
    }
}

/* Ctrsm with op in {N, T, C}.  Restates Ctrsm_naive
 * (libs/blas/funcs/Ctrsm/Ctrsm_naive.cl:18-183): division by conj(diag) for
 * op C (:33), alpha applied on the store (:43).  Arithmetic in complex double. */
void orc_ctrsm(int side, int uplo, int trans, int diag, int m, int n, orc_c32 alpha,
               const orc_c32* A, int lda, orc_c32* B, int ldb)
{
    cd al = cd_of(alpha);
    if (side == 0) {
        cd* z = (cd*)malloc(sizeof(cd) * (size_t)m);
        for (int j = 0; j < n; ++j) {
            for (int i = 0; i < m; ++i) z[i] = cd_of(B[(long)j * ldb + i]);
            tri_solve_cd(uplo, trans, diag, m, A, lda, z);
            for (int i = 0; i < m; ++i) B[(long)j * ldb + i] = c32_of(cd_mul(z[i], al));
        }
        free(z);
    } else {
        /* X op(A) = B  <=>  op(A)^T X^T = B^T: solve each row of B with the
         * transposed operator (N -> T, T -> N, C -> conj without transpose). */
        int op = (trans == 0) ? 1 : (trans == 1) ? 0 : 3;
        cd* z = (cd*)malloc(sizeof(cd) * (size_t)n);
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < n; ++j) z[j] = cd_of(B[(long)j * ldb + i]);
            tri_solve_cd(uplo, op, diag, n, A, lda, z);
            for (int j = 0; j < n; ++j) B[(long)j * ldb + i] = c32_of(cd_mul(z[j], al));
        }
        free(z);
    }
}

/* FP64 GEMM, same semantics as orc_sgemm; loops ordered j, p, i so the
 * inner loop walks a column of C and (for op(A) = N) a column of A. */
void orc_dgemm(int transa, int transb, int m, int n, int k, double alpha,
               const double* A, int lda, const double* B, int ldb, double beta, double* C, int ldc)
{
    double* acc = (double*)malloc(sizeof(double) * (size_t)m);
    for (int j = 0; j < n; ++j) {
        memset(acc, 0, sizeof(double) * (size_t)m);
        for (int p = 0; p < k; ++p) {
            double b = transb == 0 ? B[(long)j * ldb + p] : B[(long)p * ldb + j];
            if (transa == 0) {
                const double* col = A + (long)p * lda;
                for (int i = 0; i < m; ++i) acc[i] += col[i] * b;
            } else {
                for (int i = 0; i < m; ++i) acc[i] += A[(long)i * lda + p] * b;
            }
        }
        double* c = C + (long)j * ldc;
        for (int i = 0; i < m; ++i) c[i] = (beta == 0.0) ? acc[i] * alpha : acc[i] * alpha + c[i] * beta;
    }
    free(acc);
}

/* FP64 TRSM, same semantics as orc_strsm (alpha applied after the solve). */
void orc_dtrsm(int side, int uplo, int trans, int diag, int m, int n, double alpha,
               const double* A, int lda, double* B, int ldb)
{
    int op = (trans == 0) ? 0 : 1;
    if (side == 0) {
        tri_solve_cols_d(uplo, op, diag, m, A, lda, B, ldb, n);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < m; ++i) B[(long)j * ldb + i] *= alpha;
    } else {
        int rop = (op == 0) ? 1 : 0;
        double* z = (double*)malloc(sizeof(double) * (size_t)n);
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < n; ++j) z[j] = B[(long)j * ldb + i];
            tri_solve_d(uplo, rop, diag, n, A, lda, z);
            for (int j = 0; j < n; ++j) B[(long)j * ldb + i] = z[j] * alpha;
        }
        free(z);
    }
}

/* ------------------------------------------------------------------------ */
/* Rank-1 updates, symmetric / Hermitian products, GEMM-shaped level 3      */
/* ------------------------------------------------------------------------ */

/* A(i,j) = fma(alpha, x_i*y_j, A(i,j)) in FP32: Sger_naive.cl:16-26 (the
 * product rounded, then mad, restated as fmaf). */
void orc_sger(int m, int n, float alpha, const float* x, int incx, const float* y, int incy, float* A, int lda)
{
    for (long j = 0; j < n; ++j)
        for (long i = 0; i < m; ++i) {
            const float p = x[i * incx] * y[j * incy];
            A[j * lda + i] = fmaf(alpha, p, A[j * lda + i]);
        }
}

/* A(i,j) += cmul(alpha, cmul(x_i, y_j or conj(y_j))) in FP32 with the
 * reference's fma placement: Cgeru_naive.cl:18-33, Cgerc_naive.cl:18-32. */
void orc_cger(int conj, int m, int n, orc_c32 alpha, const orc_c32* x, int incx, const orc_c32* y, int incy,
              orc_c32* A, int lda)
{
    for (long j = 0; j < n; ++j) {
        orc_c32 yv = y[j * incy];
        if (conj) yv.im = -yv.im;
        for (long i = 0; i < m; ++i) {
            const orc_c32 t = cmul_fma(alpha, cmul_fma(x[i * incx], yv));
            orc_c32* a = A + j * lda + i;
            a->re = a->re + t.re;
            a->im = a->im + t.im;
        }
    }
}

/* element (r, c) of the symmetric / Hermitian matrix whose uplo triangle is
 * stored in A (tests/blas_funcs/test_symv.hpp:54-76: the other triangle read
 * transposed, conjugated for Hermitian; a Hermitian diagonal's imaginary part
 * is taken as 0) */
static cd sym_elem(int uplo, int herm, const orc_c32* A, int lda, int r, int c)
{
    const int upper = (uplo == 0);
    cd v;
    if ((upper && c < r) || (!upper && c > r)) {
        v = cd_of(A[(long)r * lda + c]);
        if (herm) v = cd_conj(v);
    } else {
        v = cd_of(A[(long)c * lda + r]);
    }
    if (herm && r == c) v.im = 0.0;
    return v;
}

/* y = alpha A x + beta y, A symmetric (uplo triangle stored).  The sum
 * (A x)_r is cpu_symv's (tests/blas_funcs/test_symv.hpp:21-87: the element
 * choice, accumulated in double), rounded to float once; the final step is
 * the reference kernel's FP32 expression (Ssymv_naive_lower.cl:34-37:
 * beta != 0 ? fma(alpha, s, beta*y) : alpha*s), so beta == 0 does not read
 * y. */
void orc_ssymv(int uplo, int n, float alpha, const float* A, int lda, const float* x, int incx, float beta, float* y,
               int incy)
{
    const int upper = (uplo == 0);
    for (int r = 0; r < n; ++r) {
        double acc = 0.0;
        for (int c = 0; c < n; ++c) {
            const double a = ((upper && c < r) || (!upper && c > r)) ? A[(long)r * lda + c] : A[(long)c * lda + r];
            acc += a * (double)x[(long)c * incx];
        }
        const float s = (float)acc;
        float* yp = y + (long)r * incy;
        *yp = (beta != 0.0f) ? fmaf(alpha, s, beta * *yp) : alpha * s;
    }
}

/* Complex Hermitian y = alpha A x + beta y: the sum as cpu_symv<complex,
 * true> (test_symv.hpp) in double, rounded once; then the reference kernel's
 * FP32 step (Chemv_naive.cl:45-46: y = cmul(beta, y) + cmul(s, alpha), fma
 * placement of complex.h.cl:32-34).  That kernel reads y even for beta == 0;
 * here beta == 0 means y = cmul(s, alpha) without reading y.  (The FP32 final
 * step matters: the reference's own test_Chemv.cpp naive_low_3x3 expects the
 * FP32 cancellation of its 33.7 - 28.4 imaginary part, 5.2999954, which a
 * double evaluation, 5.2999987, misses by 7 ulps.) */
void orc_chemv(int uplo, int n, orc_c32 alpha, const orc_c32* A, int lda, const orc_c32* x, int incx, orc_c32 beta,
               orc_c32* y, int incy)
{
    const int beta_zero = (beta.re == 0.0f && beta.im == 0.0f);
    for (int r = 0; r < n; ++r) {
        cd acc = cd_make(0, 0);
        for (int c = 0; c < n; ++c) acc = cd_add(acc, cd_mul(sym_elem(uplo, 1, A, lda, r, c), cd_of(x[(long)c * incx])));
        const orc_c32 s = c32_of(acc);
        const orc_c32 t = cmul_fma(s, alpha);
        orc_c32* yp = y + (long)r * incy;
        if (beta_zero) {
            *yp = t;
        } else {
            const orc_c32 b = cmul_fma(beta, *yp);
            yp->re = b.re + t.re;
            yp->im = b.im + t.im;
        }
    }
}

/* C = alpha op(A) op(B)^T (+ alpha op(B) op(A)^T when B != NULL) + beta C on
 * the uplo triangle of C (upper 0, lower 1); op(X) = X (n x k) for trans == 0,
 * X^T (X k x n) otherwise.  Restates Ssyrk_naive.cl:18-48 and
 * Ssyr2k_naive.cl:18-49 in double; beta == 0 means C is not read (the
 * kernels read it). */
void orc_ssyr2k(int uplo, int trans, int n, int k, float alpha, const float* A, int lda, const float* B, int ldb,
                float beta, float* C, int ldc)
{
    const int lower = (uplo == 1);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            if (lower ? (i < j) : (i > j)) continue;
            double acc = 0.0;
            for (int l = 0; l < k; ++l) {
                const double ai = trans ? A[(long)i * lda + l] : A[(long)l * lda + i];
                const double aj = trans ? A[(long)j * lda + l] : A[(long)l * lda + j];
                if (!B) {
                    acc += ai * aj;
                } else {
                    const double bi = trans ? B[(long)i * ldb + l] : B[(long)l * ldb + i];
                    const double bj = trans ? B[(long)j * ldb + l] : B[(long)l * ldb + j];
                    acc += ai * bj + bi * aj;
                }
            }
            double out = (double)alpha * acc;
            if (beta != 0.0f) out += (double)beta * (double)C[(long)j * ldc + i];
            C[(long)j * ldc + i] = (float)out;
        }
}

void orc_ssyrk(int uplo, int trans, int n, int k, float alpha, const float* A, int lda, float beta, float* C, int ldc)
{
    orc_ssyr2k(uplo, trans, n, k, alpha, A, lda, NULL, 0, beta, C, ldc);
}

/* C = alpha A B + beta C (side 0) or alpha B A + beta C (side 1), A
 * symmetric with its uplo triangle stored: Ssymm_naive.cl:18-75 in double;
 * beta == 0: C not read. */
void orc_ssymm(int side, int uplo, int m, int n, float alpha, const float* A, int lda, const float* B, int ldb,
               float beta, float* C, int ldc)
{
    const int upper = (uplo == 0);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double acc = 0.0;
            const int kk = side == 0 ? m : n;
            for (int l = 0; l < kk; ++l) {
                int r = side == 0 ? i : l, c = side == 0 ? l : j;   /* A_sym(r, c) */
                const double a = ((upper && c < r) || (!upper && c > r)) ? A[(long)r * lda + c] : A[(long)c * lda + r];
                const double b = side == 0 ? B[(long)j * ldb + l] : B[(long)l * ldb + i];
                acc += a * b;
            }
            double out = (double)alpha * acc;
            if (beta != 0.0f) out += (double)beta * (double)C[(long)j * ldc + i];
            C[(long)j * ldc + i] = (float)out;
        }
}

/* C = alpha op(A) B (side 0) or alpha B op(A) (side 1), A triangular
 * (uplo 0 upper / 1 lower, diag 1 unit), op by transa (1 and 2 both
 * transpose: real data).  The operation documented by the reference's header
 * (include/iclBLAS/iclBLAS.h:1720-1753), in double; C may be B. */
void orc_strmm(int side, int uplo, int transa, int diag, int m, int n, float alpha, const float* A, int lda,
               const float* B, int ldb, float* C, int ldc)
{
    const int lower = (uplo == 1), unit = (diag == 1), tr = (transa != 0);
    const int na = side == 0 ? m : n;
    double* out = (double*)malloc(sizeof(double) * (size_t)m * (size_t)n);
    if (!out) return;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double acc = 0.0;
            for (int l = 0; l < na; ++l) {
                /* op(A)(r, c) */
                const int r = side == 0 ? i : l, c = side == 0 ? l : j;
                const int ar = tr ? c : r, ac = tr ? r : c;   /* element of A */
                double a;
                if (ar == ac) a = unit ? 1.0 : A[(long)ac * lda + ar];
                else if (lower ? (ar > ac) : (ar < ac)) a = A[(long)ac * lda + ar];
                else a = 0.0;
                const double b = side == 0 ? B[(long)j * ldb + l] : B[(long)l * ldb + i];
                acc += a * b;
            }
            out[(size_t)j * m + i] = (double)alpha * acc;
        }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) C[(long)j * ldc + i] = (float)out[(size_t)j * m + i];
    free(out);
}

/* ------------------------------------------------------------------------ */
/* Half-precision GEMM (the library's HGEMM extension)                      */
/* ------------------------------------------------------------------------ */

/* IEEE 754 binary16 bit pattern -> value */
static double half_value(uint16_t h)
{
    const int s = h >> 15, e = (h >> 10) & 31, f = h & 1023;
    double v;
    if (e == 0) v = ldexp((double)f, -24);
    else if (e == 31) v = f ? NAN : INFINITY;
    else v = ldexp((double)(f + 1024), e - 25);
    return s ? -v : v;
}

/* value -> binary16, round to nearest even (one rounding from double) */
static uint16_t half_bits(double x)
{
    if (isnan(x)) return 0x7e00;
    const uint16_t sign = signbit(x) ? 0x8000 : 0;
    double a = fabs(x);
    if (a == 0.0) return sign;
    int e2;
    frexp(a, &e2);              /* a = m 2^e2, m in [0.5, 1) */
    int E = e2 - 1;             /* 2^E <= a < 2^(E+1) */
    if (E < -14) E = -14;       /* subnormal quantum 2^-24 */
    const double q = ldexp(1.0, E - 10);
    a = nearbyint(a / q) * q;   /* default rounding mode: nearest even */
    if (a == 0.0) return sign;
    if (a > 65504.0) return (uint16_t)(sign | 0x7c00);
    frexp(a, &e2);
    E = e2 - 1;
    if (E < -14) return (uint16_t)(sign | (uint16_t)(a / ldexp(1.0, -24)));  /* subnormal */
    const int f = (int)(a / ldexp(1.0, E - 10)) - 1024;
    return (uint16_t)(sign | (uint16_t)((E + 15) << 10) | (uint16_t)f);
}

/* C = alpha op(A) op(B) + beta C on binary16 storage: products and sums in
 * double, one rounding to half; beta == 0 means C is not read. */
void orc_hgemm(int transa, int transb, int m, int n, int k, float alpha, const uint16_t* A, int lda,
               const uint16_t* B, int ldb, float beta, uint16_t* C, int ldc)
{
    /* op(A) rows and op(B) columns converted once, K-contiguous (the sums
       run over l in the same order as a direct loop) */
    double* Ad = (double*)malloc(sizeof(double) * ((size_t)m * (size_t)k + 1));
    double* Bd = (double*)malloc(sizeof(double) * ((size_t)n * (size_t)k + 1));
    if (!Ad || !Bd) {
        free(Ad);
        free(Bd);
        return;
    }
    for (int i = 0; i < m; ++i)
        for (int l = 0; l < k; ++l)
            Ad[(size_t)i * k + l] = half_value(transa ? A[(long)i * lda + l] : A[(long)l * lda + i]);
    for (int j = 0; j < n; ++j)
        for (int l = 0; l < k; ++l)
            Bd[(size_t)j * k + l] = half_value(transb ? B[(long)l * ldb + j] : B[(long)j * ldb + l]);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            const double* a = Ad + (size_t)i * k;
            const double* b = Bd + (size_t)j * k;
            double acc = 0.0;
            for (int l = 0; l < k; ++l) acc += a[l] * b[l];
            double out = (double)alpha * acc;
            if (beta != 0.0f) out += (double)beta * half_value(C[(long)j * ldc + i]);
            C[(long)j * ldc + i] = half_bits(out);
        }
    free(Ad);
    free(Bd);
}
