// OpenCL-C-to-C++ shim -- TEST INFRASTRUCTURE ONLY.
//
// Lets the reference's serial ("naive") OpenCL kernels be compiled as plain
// C++ functions straight from their .cl sources, so that they can serve as a
// CPU check of the oracle.  It supplies the OpenCL address-space keywords,
// work-item queries (driven by run_ndrange below), the float2 vector type with
// OpenCL's scalar broadcast, and the complex helpers that the reference
// prepends to every program (core/src/ocl/complex.h.cl:28-72).  The helpers
// are restated here because the OpenCL vector literal "(complex_t)(a, b)" in
// that file has a different meaning in C++ (a comma expression: it yields
// (b, b)); kernels that write such a literal themselves are only compared on
// inputs that do not reach it.
#pragma once
#include <cmath>
#include <cstdint>

#define __kernel
#define kernel
#define __global
#define global
typedef unsigned int uint;

namespace clshim {
inline thread_local size_t g_gid[3] = {0, 0, 0};
}
inline size_t get_global_id(int d) { return clshim::g_gid[d]; }

inline float mad(float a, float b, float c) { return std::fma(a, b, c); }
using std::fma;
using std::sqrt;
using std::fabs;

struct float2 {
    float x, y;
    float2() : x(0.f), y(0.f) {}
    float2(float s) : x(s), y(s) {}  // OpenCL scalar-to-vector broadcast
    float2(float a, float b) : x(a), y(b) {}
    float2& operator+=(const float2& o) { x += o.x; y += o.y; return *this; }
    float2& operator-=(const float2& o) { x -= o.x; y -= o.y; return *this; }
};
inline float2 operator+(float2 a, float2 b) { return float2(a.x + b.x, a.y + b.y); }
inline float2 operator-(float2 a, float2 b) { return float2(a.x - b.x, a.y - b.y); }
inline float2 operator*(float2 a, float2 b) { return float2(a.x * b.x, a.y * b.y); }
inline float2 operator/(float2 a, float2 b) { return float2(a.x / b.x, a.y / b.y); }
inline float2 operator-(float2 a) { return float2(-a.x, -a.y); }

typedef float2 complex_t;

// complex.h.cl:32 -- product with two fused multiply-adds
inline complex_t cmul(complex_t a, complex_t b)
{
    return complex_t(std::fma(a.x, b.x, -a.y * b.y), std::fma(a.x, b.y, a.y * b.x));
}
// complex.h.cl:36 -- quotient through |b|^2 without scaling
inline complex_t cdiv(complex_t a, complex_t b)
{
    float d = std::fma(b.x, b.x, b.y * b.y);
    return complex_t(std::fma(a.x, b.x, a.y * b.y) / d, std::fma(a.y, b.x, -a.x * b.y) / d);
}
// complex.h.cl:58
inline complex_t conjg(complex_t a) { return complex_t(a.x, -a.y); }
// complex.h.cl:54
inline float scabs1(complex_t a) { return std::fabs(a.x) + std::fabs(a.y); }
// complex.h.cl:28 -- modulus with one fused multiply-add
inline float cabs(complex_t a) { return std::sqrt(std::fma(a.x, a.x, a.y * a.y)); }
// complex.h.cl:41-47, 62-68 -- scalar broadcasts and negation
inline complex_t cmulf(complex_t a, float b) { return a * float2(b); }
inline complex_t cdivf(complex_t a, float b) { return a / float2(b); }
inline complex_t cneg(complex_t a) { return -a; }
// OpenCL's componentwise fma on float2; cfmaf broadcasts b (complex.h.cl:66)
inline float2 fma(float2 a, float2 b, float2 c) { return float2(std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y)); }
inline complex_t cfmaf(complex_t a, float b, complex_t c) { return fma(a, float2(b), c); }
// OpenCL sign(): 1, -1, or 0 for zero and NaN
inline float sign(float v) { return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f); }

namespace clshim {
// Runs a 2-D NDRange of gws0 x gws1 work-items sequentially.
template <class F>
inline void run_ndrange2(size_t gws0, size_t gws1, F&& f)
{
    for (size_t j = 0; j < gws1; ++j)
        for (size_t i = 0; i < gws0; ++i) {
            g_gid[0] = i;
            g_gid[1] = j;
            f();
        }
    g_gid[0] = g_gid[1] = 0;
}
// Runs a 1-D NDRange of `gws` work-items sequentially.
template <class F>
inline void run_ndrange(size_t gws, F&& f)
{
    for (size_t i = 0; i < gws; ++i) {
        g_gid[0] = i;
        f();
    }
    g_gid[0] = 0;
}
}
