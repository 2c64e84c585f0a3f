// C-ABI layer of the B200 iclBLAS library.
//
// Replaces the reference's C API implementation (libs/blas/shlib/iclBLAS.cpp,
// iclBLAS_S.cpp, iclBLAS_C.cpp, iclBLASImpl.hpp) and the OpenCL engine under
// it (core/src/ocl/*): a handle owns a CUDA stream and a device workspace,
// each routine validates its arguments with the reference's rules, moves
// host-resident operands to the device (the reference wraps host arrays in
// OpenCL buffers per call, core/src/ocl/ocl_buffer.cpp:27-58, and reads the
// outputs back before returning, ocl_kernel.cpp:86-92), and launches the
// routine's sm_100a kernels directly (no scored implementation selection, no
// JIT).  Exceptions never cross the ABI, in every build type.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>

#include "internal.h"
#include "memkind.h"

using iclb::cfloat;

namespace {

iclblasStatus_t map_cuda(cudaError_t e)
{
    if (e == cudaSuccess) return ICLBLAS_STATUS_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return ICLBLAS_STATUS_ALLOC_FAILED;
    if (e == cudaErrorInvalidDevicePointer) return ICLBLAS_STATUS_INVALID_VALUE;   // another GPU's memory
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return ICLBLAS_STATUS_NOT_INITIALIZED;
    if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDeviceFunction) return ICLBLAS_STATUS_ARCH_MISMATCH;
    return ICLBLAS_STATUS_EXECUTION_FAILED;
}

bool handle_ok(iclblasHandle_t h) { return h != nullptr && h->tag == iclb::kHandleTag; }

// Argument checks in the reference's order (libs/blas/shlib/iclBLASImpl.hpp:
// validate_params :218-233, then the handle :236-245).  Only the fields
// flagged in `present` exist for a routine.
enum : unsigned {
    P_N = 1u << 0, P_M = 1u << 1, P_K = 1u << 2, P_X = 1u << 3, P_INCX = 1u << 4, P_Y = 1u << 5,
    P_INCY = 1u << 6, P_A = 1u << 7, P_LDA = 1u << 8, P_B = 1u << 9, P_LDB = 1u << 10, P_C = 1u << 11,
    P_LDC = 1u << 12
};
struct Params {
    unsigned present = 0;
    int n = 0, m = 0, k = 0, incx = 0, incy = 0, lda = 0, ldb = 0, ldc = 0;
    const void *x = nullptr, *y = nullptr, *A = nullptr, *B = nullptr, *C = nullptr;
};
// Returns -1 to end the call successfully without work, 0 to run, or a status.
int validate(const Params& p, iclblasHandle_t h)
{
    const unsigned f = p.present;
    if (f & P_N) { if (p.n < 0) return ICLBLAS_STATUS_INVALID_VALUE; if (p.n == 0) return -1; }
    if (f & P_M) { if (p.m < 0) return ICLBLAS_STATUS_INVALID_VALUE; if (p.m == 0) return -1; }
    if ((f & P_K) && p.k < 0) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_X) && !p.x) return ICLBLAS_STATUS_INVALID_VALUE;
    if (f & P_INCX) { if (p.incx == 0) return ICLBLAS_STATUS_INVALID_VALUE; if (p.incx < 0) return ICLBLAS_STATUS_NOT_SUPPORTED; }
    if ((f & P_Y) && !p.y) return ICLBLAS_STATUS_INVALID_VALUE;
    if (f & P_INCY) { if (p.incy == 0) return ICLBLAS_STATUS_INVALID_VALUE; if (p.incy < 0) return ICLBLAS_STATUS_NOT_SUPPORTED; }
    if ((f & P_A) && !p.A) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_LDA) && p.lda <= 0) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_B) && !p.B) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_LDB) && p.ldb <= 0) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_C) && !p.C) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_LDC) && p.ldc <= 0) return ICLBLAS_STATUS_INVALID_VALUE;
    if (!handle_ok(h)) return ICLBLAS_STATUS_INVALID_VALUE;
    return 0;
}

#define VALIDATE(p, h)                                                          \
    do {                                                                        \
        int v_ = validate((p), (h));                                            \
        if (v_ < 0) return ICLBLAS_STATUS_SUCCESS;                              \
        if (v_ > 0) return (iclblasStatus_t)v_;                                 \
    } while (0)

// Where `p` lives, seen from `device` (memkind.h).
iclb::MemKind mem_kind(const void* p, int device)
{
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return iclb::MemKind::Host;
    }
    return iclb::classify_memory((int)a.type, a.device, device);
}

// Can the handle's GPU dereference `p` directly?  Device memory of another
// GPU is not: without peer access a kernel reading it faults.
bool is_device_ptr(iclblasHandle_t h, const void* p) { return mem_kind(p, h->device) == iclb::MemKind::Device; }

size_t vec_extent(int n, int inc) { return n > 0 ? (size_t)(n - 1) * (size_t)inc + 1 : 0; }
size_t mat_extent(int rows, int cols, int ld)
{
    return (rows > 0 && cols > 0) ? (size_t)(cols - 1) * (size_t)ld + (size_t)rows : 0;
}

// Moves host-resident operands through a device staging area.  Device
// operands pass through untouched.  When anything was staged, finish()
// copies outputs back and waits, which gives host callers the reference's
// blocking semantics; all-device calls stay asynchronous.
class Stager {
public:
    explicit Stager(iclblasHandle_t h) : h_(h) {}

    // `in` = false: an output whose every covered byte the call overwrites
    // (no host-to-device copy needed).
    int add(const void* p, size_t bytes, bool out, bool in = true)
    {
        Op& o = ops_[n_];
        o.user = const_cast<void*>(p);
        o.bytes = bytes;
        o.out = out;
        o.in = in;
        const iclb::MemKind k = mem_kind(p, h_->device);
        foreign_ |= k == iclb::MemKind::OtherDevice;
        o.pageable = k == iclb::MemKind::Pageable;
        o.staged = k == iclb::MemKind::Host || o.pageable;
        o.dev = o.staged ? nullptr : o.user;
        return n_++;
    }

    // An operand in another GPU's memory ends the call with INVALID_VALUE
    // before any copy or launch (map_cuda maps this error to it).
    cudaError_t rejected() const { return foreign_ ? cudaErrorInvalidDevicePointer : cudaSuccess; }

    // Device addresses for the staged operands (grows the staging buffer).
    cudaError_t reserve()
    {
        size_t total = 0;
        for (int i = 0; i < n_; ++i)
            if (ops_[i].staged) total += (ops_[i].bytes + 255) & ~(size_t)255;
        if (total == 0) return cudaSuccess;
        if (total > h_->stage_bytes) {
            if (h_->stage) cudaFree(h_->stage);
            h_->stage = nullptr;
            h_->stage_bytes = 0;
            cudaError_t e = cudaMalloc(&h_->stage, total);
            if (e != cudaSuccess) return e;
            h_->stage_bytes = total;
        }
        char* base = (char*)h_->stage;
        size_t off = 0;
        for (int i = 0; i < n_; ++i) {
            Op& o = ops_[i];
            if (!o.staged) continue;
            o.dev = base + off;
            off += (o.bytes + 255) & ~(size_t)255;
        }
        return cudaSuccess;
    }

    cudaError_t stage_in()
    {
        if (foreign_) return rejected();
        cudaError_t e = reserve();
        if (e != cudaSuccess) return e;
        for (int i = 0; i < n_; ++i) {
            Op& o = ops_[i];
            if (!o.staged) continue;
            any_staged_ = true;
            if (!o.in) continue;
            if (o.pageable && o.bytes >= kBounceMin)
                e = iclb::copy_pageable_h2d(h_, o.dev, o.user, o.bytes);
            else
                e = cudaMemcpyAsync(o.dev, o.user, o.bytes, cudaMemcpyHostToDevice, h_->stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    template <class T>
    T* dev(int i) const { return (T*)ops_[i].dev; }

    // Elementwise calls (every operand i covers elements [0, n) with stride
    // incs[i], element size esize): when some operand lives in host memory and
    // the call is large, run it in chunks so that each chunk's outputs are
    // copied back on the handle's second stream while the next chunk's inputs
    // are copied in (H2D and D2H use separate copy engines).  `launch(c0, c1)`
    // runs the kernel on elements [c0, c1) through dev().  Results are those
    // of the unchunked call (elementwise arithmetic).  Returns false in `used`
    // when the call is small or all-device (then run it the usual way).
    template <class F>
    cudaError_t run_chunked(long n, const int* incs, size_t esize, F&& launch, bool& used)
    {
        used = false;
        if (foreign_) return rejected();
        bool any = false;
        size_t total = 0;
        for (int i = 0; i < n_; ++i) {
            any |= ops_[i].staged;
            total += ops_[i].bytes;
            // pageable operands go through the bounce buffers of stage_in / finish
            if (ops_[i].pageable) return cudaSuccess;
        }
        constexpr long kChunk = 1L << 24;  // elements per chunk
        if (!any || total < ((size_t)64 << 20) || n < 2 * kChunk) return cudaSuccess;
        const long nchunks = std::min<long>((n + kChunk - 1) / kChunk, iclblasContext::kMaxChunks);
        const long per = ((n + nchunks - 1) / nchunks + 3) & ~3L;  // multiple of 4: keeps 16-byte alignment
        cudaError_t e = reserve();
        if (e != cudaSuccess) return e;
        if (!h_->aux_stream) {
            if ((e = cudaStreamCreateWithFlags(&h_->aux_stream, cudaStreamNonBlocking)) != cudaSuccess) return e;
        }
        for (int c = 0; c < iclblasContext::kMaxChunks; ++c)
            if (!h_->chunk_ev[c] &&
                (e = cudaEventCreateWithFlags(&h_->chunk_ev[c], cudaEventDisableTiming)) != cudaSuccess)
                return e;
        used = true;
        int c = 0;
        for (long c0 = 0; c0 < n; c0 += per, ++c) {
            const long c1 = std::min(n, c0 + per);
            for (int i = 0; i < n_; ++i) {
                Op& o = ops_[i];
                if (!o.staged || !o.in) continue;
                const size_t b0 = (size_t)c0 * incs[i] * esize, b1 = ((size_t)(c1 - 1) * incs[i] + 1) * esize;
                e = cudaMemcpyAsync((char*)o.dev + b0, (const char*)o.user + b0, b1 - b0, cudaMemcpyHostToDevice,
                                    h_->stream);
                if (e != cudaSuccess) return e;
            }
            if ((e = launch(c0, c1)) != cudaSuccess) return e;
            if ((e = cudaEventRecord(h_->chunk_ev[c], h_->stream)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(h_->aux_stream, h_->chunk_ev[c], 0)) != cudaSuccess) return e;
            for (int i = 0; i < n_; ++i) {
                Op& o = ops_[i];
                if (!o.staged || !o.out) continue;
                const size_t b0 = (size_t)c0 * incs[i] * esize, b1 = ((size_t)(c1 - 1) * incs[i] + 1) * esize;
                e = cudaMemcpyAsync((char*)o.user + b0, (const char*)o.dev + b0, b1 - b0, cudaMemcpyDeviceToHost,
                                    h_->aux_stream);
                if (e != cudaSuccess) return e;
            }
        }
        if ((e = cudaStreamSynchronize(h_->aux_stream)) != cudaSuccess) return e;
        return cudaStreamSynchronize(h_->stream);
    }

    // True when the call blocks (some operand lives in host memory).
    bool blocking() const { return any_staged_; }

    cudaError_t finish()
    {
        if (!any_staged_) return cudaGetLastError();
        for (int i = 0; i < n_; ++i) {
            const Op& o = ops_[i];
            if (o.staged && o.out) {
                cudaError_t e = (o.pageable && o.bytes >= kBounceMin)
                                    ? iclb::copy_pageable_d2h(h_, o.user, o.dev, o.bytes)
                                    : cudaMemcpyAsync(o.user, o.dev, o.bytes, cudaMemcpyDeviceToHost, h_->stream);
                if (e != cudaSuccess) return e;
            }
        }
        return cudaStreamSynchronize(h_->stream);
    }

private:
    // pageable operands at least this large move through the bounce buffers
    // (smaller ones: a plain copy, which the driver stages itself)
    static constexpr size_t kBounceMin = (size_t)4 << 20;
    struct Op {
        void* user;
        void* dev;
        size_t bytes;
        bool out, in, staged, pageable;
    };
    iclblasHandle_t h_;
    Op ops_[6];
    int n_ = 0;
    bool any_staged_ = false;
    bool foreign_ = false;
};

// Reads a device status word after a blocking call (kernels with bounded
// waits record a timeout there instead of trapping).
iclblasStatus_t check_device_status(iclblasHandle_t h)
{
    int st = 0;
    cudaError_t e = cudaMemcpyAsync(&st, h->ws.dev_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return map_cuda(e);
    if (st != iclb::kDevOk) {
        cudaMemsetAsync(h->ws.dev_status, 0, sizeof(int), h->stream);
        return ICLBLAS_STATUS_EXECUTION_FAILED;
    }
    return ICLBLAS_STATUS_SUCCESS;
}

// Writes a zero result for the early-return rules that run before handle
// validation (iclBLAS_S.cpp Snrm2/Sasum/Isamax, iclBLAS_C.cpp Cdotu/Cdotc/
// Scnrm2/Icamax); a device result is cleared in stream order.
void zero_result(iclblasHandle_t h, void* result, size_t bytes)
{
    if (!result) return;
    int dev = 0;
    if (handle_ok(h)) dev = h->device;
    else cudaGetDevice(&dev);
    const iclb::MemKind k = mem_kind(result, dev);
    if (k == iclb::MemKind::Device) {
        if (handle_ok(h)) cudaMemsetAsync(result, 0, bytes, h->stream);
        else cudaMemset(result, 0, bytes);
    } else if (k == iclb::MemKind::OtherDevice) {
        // a copy (not a kernel) reaches another GPU's memory through unified addressing
        const long long zero[2] = {0, 0};
        cudaMemcpy(result, zero, bytes, cudaMemcpyDefault);
        cudaGetLastError();
    } else {
        std::memset(result, 0, bytes);
    }
}

template <class F>
iclblasStatus_t guarded(F&& f)
{
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return ICLBLAS_STATUS_ALLOC_FAILED;
    } catch (const std::invalid_argument&) {
        return ICLBLAS_STATUS_INVALID_VALUE;
    } catch (...) {
        return ICLBLAS_STATUS_ERROR;
    }
}

cfloat cf(const oclComplex_t* p)
{
    const float* f = reinterpret_cast<const float*>(p);
    return cfloat{f[0], f[1]};
}

}  // namespace

// ------------------------------------------------------------------------
// workspace
// ------------------------------------------------------------------------
void* iclb::scratch(iclblasHandle_t h, size_t bytes)
{
    bytes = (bytes + 255) & ~(size_t)255;
    if (bytes <= h->ws.scratch_bytes) return h->ws.scratch;
    // The stream may still be using the old buffer: cudaFree synchronises.
    if (h->ws.scratch) cudaFree(h->ws.scratch);
    h->ws.scratch = nullptr;
    h->ws.scratch_bytes = 0;
    size_t want = bytes < ((size_t)1 << 20) ? ((size_t)1 << 20) : bytes;
    if (cudaMalloc(&h->ws.scratch, want) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    h->ws.scratch_bytes = want;
    return h->ws.scratch;
}

cudaError_t iclb::fork_side(iclblasHandle_t h, cudaStream_t* side)
{
    cudaError_t e;
    if (!h->aux_stream && (e = cudaStreamCreateWithFlags(&h->aux_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return e;
    if (!h->fork_ev && (e = cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming)) != cudaSuccess) return e;
    if (!h->join_ev && (e = cudaEventCreateWithFlags(&h->join_ev, cudaEventDisableTiming)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(h->fork_ev, h->stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(h->aux_stream, h->fork_ev, 0)) != cudaSuccess) return e;
    *side = h->aux_stream;
    return cudaSuccess;
}

cudaError_t iclb::join_side(iclblasHandle_t h)
{
    cudaError_t e = cudaEventRecord(h->join_ev, h->aux_stream);
    if (e != cudaSuccess) return e;
    return cudaStreamWaitEvent(h->stream, h->join_ev, 0);
}

iclb::StreamScope::StreamScope(iclblasHandle_t h, cudaStream_t s) : h_(h), saved_(h->stream) { h->stream = s; }
iclb::StreamScope::~StreamScope() { h_->stream = saved_; }

void* iclb::solver_scratch(iclblasHandle_t h, size_t bytes)
{
    bytes = (bytes + 255) & ~(size_t)255;
    if (bytes <= h->ws.solver_bytes) return h->ws.solver;
    if (h->ws.solver) cudaFree(h->ws.solver);
    h->ws.solver = nullptr;
    h->ws.solver_bytes = 0;
    if (cudaMalloc(&h->ws.solver, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    h->ws.solver_bytes = bytes;
    return h->ws.solver;
}

// ------------------------------------------------------------------------
// utilities (iclBLAS.cpp:42-59)
// ------------------------------------------------------------------------
extern "C" iclblasStatus_t iclblasCreate(iclblasHandle_t* handle)
{
    if (!handle) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        iclblasContext* c = new iclblasContext();
        cudaError_t e = cudaGetDevice(&c->device);
        int sms = 0;
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMalloc(&c->ws.counters, sizeof(unsigned) * iclb::kCounterWords);
        if (e == cudaSuccess) e = cudaMalloc(&c->ws.dev_status, sizeof(int));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->ws.counters, 0, sizeof(unsigned) * iclb::kCounterWords, c->own_stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->ws.dev_status, 0, sizeof(int), c->own_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->own_stream);
        if (e != cudaSuccess) {
            if (c->ws.counters) cudaFree(c->ws.counters);
            if (c->ws.dev_status) cudaFree(c->ws.dev_status);
            if (c->own_stream) cudaStreamDestroy(c->own_stream);
            delete c;
            cudaGetLastError();
            return map_cuda(e);
        }
        c->sm_count = sms > 0 ? sms : 148;
        c->stream = c->own_stream;
        c->tag = iclb::kHandleTag;
        *handle = c;
        return ICLBLAS_STATUS_SUCCESS;
    });
}

extern "C" iclblasStatus_t iclblasDestroy(iclblasHandle_t handle)
{
    // The reference throws out of this extern "C" function on a bad handle
    // (iclBLAS.cpp:54-59 with iclBLAS.cpp:35-39); here it is a status.
    if (!handle_ok(handle)) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        cudaStreamSynchronize(handle->stream);
        if (handle->stage) cudaFree(handle->stage);
        if (handle->ws.scratch) cudaFree(handle->ws.scratch);
        if (handle->ws.solver) cudaFree(handle->ws.solver);
        if (handle->ws.pub) cudaFree(handle->ws.pub);
        if (handle->aux_stream) {
            cudaStreamSynchronize(handle->aux_stream);
            cudaStreamDestroy(handle->aux_stream);
        }
        for (int c = 0; c < iclblasContext::kMaxChunks; ++c)
            if (handle->chunk_ev[c]) cudaEventDestroy(handle->chunk_ev[c]);
        if (handle->fork_ev) cudaEventDestroy(handle->fork_ev);
        if (handle->join_ev) cudaEventDestroy(handle->join_ev);
        iclb::free_bounce(handle);
        cudaFree(handle->ws.counters);
        cudaFree(handle->ws.dev_status);
        cudaStreamDestroy(handle->own_stream);
        handle->tag = 0;
        delete handle;
        return ICLBLAS_STATUS_SUCCESS;
    });
}

extern "C" iclblasStatus_t iclblasSetStream(iclblasHandle_t h, void* stream)
{
    if (!handle_ok(h)) return ICLBLAS_STATUS_INVALID_VALUE;
    h->stream = (cudaStream_t)stream;  // NULL: the legacy default stream
    return ICLBLAS_STATUS_SUCCESS;
}

extern "C" iclblasStatus_t iclblasGetStream(iclblasHandle_t h, void** stream)
{
    if (!handle_ok(h) || !stream) return ICLBLAS_STATUS_INVALID_VALUE;
    *stream = (void*)h->stream;
    return ICLBLAS_STATUS_SUCCESS;
}

extern "C" iclblasStatus_t iclblasSetMathMode(iclblasHandle_t h, iclblasMathMode_t mode)
{
    if (!handle_ok(h)) return ICLBLAS_STATUS_INVALID_VALUE;
    if (mode < ICLBLAS_MATH_PLAIN_FP32 || mode > ICLBLAS_MATH_BF16X6) return ICLBLAS_STATUS_INVALID_VALUE;
    h->math = mode;
    return ICLBLAS_STATUS_SUCCESS;
}

extern "C" iclblasStatus_t iclblasGetMathMode(iclblasHandle_t h, iclblasMathMode_t* mode)
{
    if (!handle_ok(h) || !mode) return ICLBLAS_STATUS_INVALID_VALUE;
    *mode = h->math;
    return ICLBLAS_STATUS_SUCCESS;
}

extern "C" iclblasStatus_t iclblasSetTrsmRefinement(iclblasHandle_t h, int steps)
{
    if (!handle_ok(h) || steps < 0 || steps > 2) return ICLBLAS_STATUS_INVALID_VALUE;
    h->trsm_refine = steps;
    return ICLBLAS_STATUS_SUCCESS;
}

extern "C" iclblasStatus_t iclblasGetTrsmRefinement(iclblasHandle_t h, int* steps)
{
    if (!handle_ok(h) || !steps) return ICLBLAS_STATUS_INVALID_VALUE;
    *steps = h->trsm_refine;
    return ICLBLAS_STATUS_SUCCESS;
}

extern "C" iclblasStatus_t iclblasSynchronize(iclblasHandle_t h)
{
    if (!handle_ok(h)) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return map_cuda(e);
        return check_device_status(h);
    });
}

// ------------------------------------------------------------------------
// level 1, single (iclBLAS_S.cpp:66-228)
// ------------------------------------------------------------------------
namespace {
// Elementwise two-vector calls (copy, swap, rot, rotm): the reference's
// n <= 0 no-op, then the usual x/incx/y/incy checks, host operands staged
// (pipelined in chunks when large).  `kernel(n, x, y)` runs on device
// pointers.  x_out: x is written; y_in: y is read (or only partly written).
template <class T, class F>
iclblasStatus_t pair_call(iclblasHandle_t h, int n, T* x, int incx, bool x_out, T* y, int incy, bool y_in,
                          F&& kernel)
{
    if (n <= 0) return ICLBLAS_STATUS_SUCCESS;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(T), x_out);
        int iy = st.add(y, vec_extent(n, incy) * sizeof(T), true, y_in);
        const int incs[2] = {incx, incy};
        bool chunked = false;
        cudaError_t e = st.run_chunked(n, incs, sizeof(T), [&](long c0, long c1) {
            return kernel((int)(c1 - c0), st.dev<T>(ix) + c0 * incx, st.dev<T>(iy) + c0 * incy);
        }, chunked);
        if (chunked || e != cudaSuccess) return map_cuda(e);
        e = st.stage_in();
        if (e == cudaSuccess) e = kernel(n, st.dev<T>(ix), st.dev<T>(iy));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

cudaError_t iamin_dispatch(iclblasHandle_t h, int n, const float* x, int incx, int* r) { return iclb::isamin(h, n, x, incx, r); }
cudaError_t iamin_dispatch(iclblasHandle_t h, int n, const cfloat* x, int incx, int* r) { return iclb::icamin(h, n, x, incx, r); }

template <class T, class U>
iclblasStatus_t iamin_call(iclblasHandle_t h, int n, U* x, int incx, int* result)
{
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX; p.n = n; p.x = x; p.incx = incx;
        VALIDATE(p, h);
        if (!result) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(T), false);
        int ir = st.add(result, sizeof(int), true, false);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess) e = iamin_dispatch(h, n, st.dev<T>(ix), incx, st.dev<int>(ir));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}
}  // namespace

extern "C" iclblasStatus_t iclblasSscal(iclblasHandle_t h, int n, const float* alpha, float* x, int incx)
{
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX; p.n = n; p.x = x; p.incx = incx;
        VALIDATE(p, h);
        if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(float), true);
        const int incs[1] = {incx};
        bool chunked = false;
        cudaError_t e = st.run_chunked(n, incs, sizeof(float), [&](long c0, long c1) {
            return iclb::sscal(h, (int)(c1 - c0), *alpha, st.dev<float>(ix) + c0 * incx, incx);
        }, chunked);
        if (chunked || e != cudaSuccess) return map_cuda(e);
        e = st.stage_in();
        if (e == cudaSuccess) e = iclb::sscal(h, n, *alpha, st.dev<float>(ix), incx);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasSaxpy(iclblasHandle_t h, int n, const float* alpha, float* x, int incx, float* y, int incy)
{
    if (n <= 0 || (alpha && *alpha == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(float), false);
        int iy = st.add(y, vec_extent(n, incy) * sizeof(float), true);
        const int incs[2] = {incx, incy};
        bool chunked = false;
        cudaError_t e = st.run_chunked(n, incs, sizeof(float), [&](long c0, long c1) {
            return iclb::saxpy(h, (int)(c1 - c0), *alpha, st.dev<float>(ix) + c0 * incx, incx,
                               st.dev<float>(iy) + c0 * incy, incy);
        }, chunked);
        if (chunked || e != cudaSuccess) return map_cuda(e);
        e = st.stage_in();
        if (e == cudaSuccess) e = iclb::saxpy(h, n, *alpha, st.dev<float>(ix), incx, st.dev<float>(iy), incy);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

namespace {
iclblasStatus_t sreduce_call(iclblasHandle_t h, iclb::Red op, int n, float* x, int incx, float* y, int incy,
                             float* result)
{
    return guarded([&]() -> iclblasStatus_t {
        Params p;
        p.present = P_N | P_X | P_INCX;
        p.n = n; p.x = x; p.incx = incx;
        if (op == iclb::Red::Dot) { p.present |= P_Y | P_INCY; p.y = y; p.incy = incy; }
        VALIDATE(p, h);
        if (!result) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(float), false);
        int iy = (op == iclb::Red::Dot) ? st.add(y, vec_extent(n, incy) * sizeof(float), false) : -1;
        int ir = st.add(result, sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::sreduce(h, op, n, st.dev<float>(ix), incx, iy >= 0 ? st.dev<float>(iy) : nullptr, incy,
                              st.dev<float>(ir));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}
}  // namespace

extern "C" iclblasStatus_t iclblasSnrm2(iclblasHandle_t h, int n, float* x, int incx, float* result)
{
    if (n <= 0 || incx <= 0) { zero_result(h, result, sizeof(float)); return ICLBLAS_STATUS_SUCCESS; }
    return sreduce_call(h, iclb::Red::Nrm2, n, x, incx, nullptr, 0, result);
}

extern "C" iclblasStatus_t iclblasSasum(iclblasHandle_t h, int n, float* x, int incx, float* result)
{
    if (n <= 0 || incx <= 0) { zero_result(h, result, sizeof(float)); return ICLBLAS_STATUS_SUCCESS; }
    return sreduce_call(h, iclb::Red::Asum, n, x, incx, nullptr, 0, result);
}

extern "C" iclblasStatus_t iclblasSdot(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, float* result)
{
    if (n <= 0) return ICLBLAS_STATUS_SUCCESS;  // result untouched (iclBLAS_S.cpp:221-222)
    return sreduce_call(h, iclb::Red::Dot, n, x, incx, y, incy, result);
}

// SDOT for callers that cannot allocate device memory (see include/iclBLAS.h).
// Same validation as iclblasSdot; then every array must be device memory,
// because staging host data would allocate.  No cudaMalloc/cudaFree, no
// workspace growth: the kernel's scratch is a fixed array in the library.
extern "C" iclblasStatus_t iclblasSdotNoAlloc(iclblasHandle_t h, int n, const float* x, int incx, const float* y,
                                              int incy, float* result)
{
    if (n <= 0) return ICLBLAS_STATUS_SUCCESS;  // result untouched, as iclblasSdot
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        if (!result) return ICLBLAS_STATUS_INVALID_VALUE;
        if (!is_device_ptr(h, x) || !is_device_ptr(h, y) || !is_device_ptr(h, result)) return ICLBLAS_STATUS_INVALID_VALUE;
        cudaError_t e = iclb::sdot_noalloc(h, n, x, incx, y, incy, result);
        if (e == cudaErrorNotSupported) return ICLBLAS_STATUS_NOT_SUPPORTED;
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasIsamax(iclblasHandle_t h, int n, float* x, int incx, int* result)
{
    if (n <= 0 || incx <= 0) { zero_result(h, result, sizeof(int)); return ICLBLAS_STATUS_SUCCESS; }
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX; p.n = n; p.x = x; p.incx = incx;
        VALIDATE(p, h);
        if (!result) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(float), false);
        int ir = st.add(result, sizeof(int), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess) e = iclb::isamax(h, n, st.dev<float>(ix), incx, st.dev<int>(ir));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasIsamin(iclblasHandle_t h, int n, float* x, int incx, int* result)
{
    // iclBLAS_S.cpp:152-164
    if (n <= 0 || incx <= 0) { zero_result(h, result, sizeof(int)); return ICLBLAS_STATUS_SUCCESS; }
    return iamin_call<float>(h, n, x, incx, result);
}

extern "C" iclblasStatus_t iclblasScopy(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy)
{
    // y is written without being read where it is contiguous
    return pair_call<float>(h, n, x, incx, false, y, incy, incy != 1, [&](int nn, float* dx, float* dy) {
        return iclb::scopy(h, nn, dx, incx, dy, incy);
    });
}

extern "C" iclblasStatus_t iclblasSswap(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy)
{
    return pair_call<float>(h, n, x, incx, true, y, incy, true, [&](int nn, float* dx, float* dy) {
        return iclb::sswap(h, nn, dx, incx, dy, incy);
    });
}

extern "C" iclblasStatus_t iclblasSrot(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, float c,
                                       float s)
{
    if (n <= 0 || (c == 1.f && s == 0.f)) return ICLBLAS_STATUS_SUCCESS;  // iclBLAS_S.cpp:182-183
    return pair_call<float>(h, n, x, incx, true, y, incy, true, [&](int nn, float* dx, float* dy) {
        return iclb::srot(h, nn, dx, incx, dy, incy, c, s);
    });
}

extern "C" iclblasStatus_t iclblasSrotm(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy,
                                        float* param)
{
    if (n <= 0) return ICLBLAS_STATUS_SUCCESS;
    if (!param) return ICLBLAS_STATUS_INVALID_VALUE;
    // Host parameters are read here (the reference's early return for the
    // identity flag -2, iclBLAS_S.cpp:194-195); device parameters are read
    // by the kernel, which skips every flag outside {-1, 0, 1}.
    int dev = 0;
    if (handle_ok(h)) dev = h->device;
    else cudaGetDevice(&dev);
    const iclb::MemKind pk = mem_kind(param, dev);
    if (pk == iclb::MemKind::OtherDevice) return ICLBLAS_STATUS_INVALID_VALUE;
    const bool dev_param = pk == iclb::MemKind::Device;
    if (!dev_param && param[0] == -2.f) return ICLBLAS_STATUS_SUCCESS;
    return pair_call<float>(h, n, x, incx, true, y, incy, true, [&](int nn, float* dx, float* dy) {
        return iclb::srotm(h, nn, dx, incx, dy, incy, dev_param ? nullptr : param, dev_param ? param : nullptr);
    });
}

extern "C" iclblasStatus_t iclblasSrotg(iclblasHandle_t h, float* a, float* b, float* c, float* s)
{
    return guarded([&]() -> iclblasStatus_t {
        if (!handle_ok(h) || !a || !b || !c || !s) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ia = st.add(a, sizeof(float), true), ib = st.add(b, sizeof(float), true);
        int ic = st.add(c, sizeof(float), true, false), is = st.add(s, sizeof(float), true, false);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess) e = iclb::srotg(h, st.dev<float>(ia), st.dev<float>(ib), st.dev<float>(ic), st.dev<float>(is));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasSrotmg(iclblasHandle_t h, float* d1, float* d2, float* x1, const float* y1,
                                         float* param)
{
    // The reference's host-side checks (iclBLAS_S.cpp:101-128) run inside
    // the kernel so that device-resident operands work too.  param is
    // staged in as well: flags 0, 1 and -2 leave some of its entries as
    // they were.
    return guarded([&]() -> iclblasStatus_t {
        if (!handle_ok(h) || !d1 || !d2 || !x1 || !y1 || !param) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int i1 = st.add(d1, sizeof(float), true), i2 = st.add(d2, sizeof(float), true);
        int ix = st.add(x1, sizeof(float), true), iy = st.add(y1, sizeof(float), false);
        int ip = st.add(param, 5 * sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::srotmg(h, st.dev<float>(i1), st.dev<float>(i2), st.dev<float>(ix), st.dev<float>(iy),
                             st.dev<float>(ip));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

// ------------------------------------------------------------------------
// level 1, complex (iclBLAS_C.cpp:69-307)
// ------------------------------------------------------------------------
namespace {
iclblasStatus_t cscal_call(iclblasHandle_t h, int n, cfloat alpha, oclComplex_t* x, int incx)
{
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX; p.n = n; p.x = x; p.incx = incx;
        VALIDATE(p, h);
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(cfloat), true);
        const int incs[1] = {incx};
        bool chunked = false;
        cudaError_t e = st.run_chunked(n, incs, sizeof(cfloat), [&](long c0, long c1) {
            return iclb::cscal(h, (int)(c1 - c0), alpha, st.dev<cfloat>(ix) + c0 * incx, incx);
        }, chunked);
        if (chunked || e != cudaSuccess) return map_cuda(e);
        e = st.stage_in();
        if (e == cudaSuccess) e = iclb::cscal(h, n, alpha, st.dev<cfloat>(ix), incx);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}
}  // namespace

extern "C" iclblasStatus_t iclblasCscal(iclblasHandle_t h, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx)
{
    if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
    return cscal_call(h, n, cf(alpha), x, incx);
}

extern "C" iclblasStatus_t iclblasCsscal(iclblasHandle_t h, int n, const float* alpha, oclComplex_t* x, int incx)
{
    // Cscal with alpha = (a, 0) (iclBLAS_C.cpp:78-84)
    if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
    return cscal_call(h, n, cfloat{*alpha, 0.f}, x, incx);
}

extern "C" iclblasStatus_t iclblasCaxpy(iclblasHandle_t h, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx,
                                        oclComplex_t* y, int incy)
{
    if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
    cfloat a = cf(alpha);
    if (n <= 0 || (a.re == 0.f && a.im == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(cfloat), false);
        int iy = st.add(y, vec_extent(n, incy) * sizeof(cfloat), true);
        const int incs[2] = {incx, incy};
        bool chunked = false;
        cudaError_t e = st.run_chunked(n, incs, sizeof(cfloat), [&](long c0, long c1) {
            return iclb::caxpy(h, (int)(c1 - c0), a, st.dev<cfloat>(ix) + c0 * incx, incx,
                               st.dev<cfloat>(iy) + c0 * incy, incy);
        }, chunked);
        if (chunked || e != cudaSuccess) return map_cuda(e);
        e = st.stage_in();
        if (e == cudaSuccess) e = iclb::caxpy(h, n, a, st.dev<cfloat>(ix), incx, st.dev<cfloat>(iy), incy);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

namespace {
iclblasStatus_t cdot_call(iclblasHandle_t h, bool conj, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy,
                          oclComplex_t* result)
{
    if (n <= 0) { zero_result(h, result, sizeof(cfloat)); return ICLBLAS_STATUS_SUCCESS; }
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        if (!result) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(cfloat), false);
        int iy = st.add(y, vec_extent(n, incy) * sizeof(cfloat), false);
        int ir = st.add(result, sizeof(cfloat), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::cdot(h, conj, n, st.dev<cfloat>(ix), incx, st.dev<cfloat>(iy), incy, st.dev<cfloat>(ir));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

iclblasStatus_t creduce_call(iclblasHandle_t h, iclb::Red op, int n, oclComplex_t* x, int incx, float* result)
{
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX; p.n = n; p.x = x; p.incx = incx;
        VALIDATE(p, h);
        if (!result) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(cfloat), false);
        int ir = st.add(result, sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess) e = iclb::creduce_real(h, op, n, st.dev<cfloat>(ix), incx, st.dev<float>(ir));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}
}  // namespace

extern "C" iclblasStatus_t iclblasCdotu(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy,
                                        oclComplex_t* result)
{
    return cdot_call(h, false, n, x, incx, y, incy, result);
}

extern "C" iclblasStatus_t iclblasCdotc(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy,
                                        oclComplex_t* result)
{
    return cdot_call(h, true, n, x, incx, y, incy, result);
}

extern "C" iclblasStatus_t iclblasScnrm2(iclblasHandle_t h, int n, oclComplex_t* x, int incx, float* result)
{
    if (n <= 0 || incx <= 0) { zero_result(h, result, sizeof(float)); return ICLBLAS_STATUS_SUCCESS; }
    return creduce_call(h, iclb::Red::Nrm2, n, x, incx, result);
}

extern "C" iclblasStatus_t iclblasScasum(iclblasHandle_t h, int n, oclComplex_t* x, int incx, float* result)
{
    // No early return in the reference (iclBLAS_C.cpp:112-118): n == 0
    // succeeds without writing result.
    return creduce_call(h, iclb::Red::Asum, n, x, incx, result);
}

extern "C" iclblasStatus_t iclblasIcamax(iclblasHandle_t h, int n, oclComplex_t* x, int incx, int* result)
{
    if (n <= 0 || incx <= 0) { zero_result(h, result, sizeof(int)); return ICLBLAS_STATUS_SUCCESS; }
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_X | P_INCX; p.n = n; p.x = x; p.incx = incx;
        VALIDATE(p, h);
        if (!result) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(cfloat), false);
        int ir = st.add(result, sizeof(int), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess) e = iclb::icamax(h, n, st.dev<cfloat>(ix), incx, st.dev<int>(ir));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasIcamin(iclblasHandle_t h, int n, oclComplex_t* x, int incx, int* result)
{
    // iclBLAS_C.cpp:153-165
    if (n <= 0 || incx <= 0) { zero_result(h, result, sizeof(int)); return ICLBLAS_STATUS_SUCCESS; }
    return iamin_call<cfloat>(h, n, x, incx, result);
}

extern "C" iclblasStatus_t iclblasCcopy(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y,
                                        int incy)
{
    return pair_call<cfloat>(h, n, (cfloat*)x, incx, false, (cfloat*)y, incy, incy != 1,
                             [&](int nn, cfloat* dx, cfloat* dy) { return iclb::ccopy(h, nn, dx, incx, dy, incy); });
}

extern "C" iclblasStatus_t iclblasCswap(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y,
                                        int incy)
{
    return pair_call<cfloat>(h, n, (cfloat*)x, incx, true, (cfloat*)y, incy, true,
                             [&](int nn, cfloat* dx, cfloat* dy) { return iclb::cswap(h, nn, dx, incx, dy, incy); });
}

extern "C" iclblasStatus_t iclblasCrot(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy,
                                       const float* c, const oclComplex_t* s)
{
    if (n <= 0) return ICLBLAS_STATUS_SUCCESS;
    if (!c || !s) return ICLBLAS_STATUS_INVALID_VALUE;
    const float cv = *c;
    const cfloat sv = cf(s);
    if (cv == 1.f && sv.re == 0.f && sv.im == 0.f) return ICLBLAS_STATUS_SUCCESS;  // iclBLAS_C.cpp:313-314
    return pair_call<cfloat>(h, n, (cfloat*)x, incx, true, (cfloat*)y, incy, true,
                             [&](int nn, cfloat* dx, cfloat* dy) { return iclb::crot(h, nn, dx, incx, dy, incy, cv, sv); });
}

extern "C" iclblasStatus_t iclblasCsrot(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y,
                                        int incy, const float* c, const float* s)
{
    if (n <= 0) return ICLBLAS_STATUS_SUCCESS;
    if (!c || !s) return ICLBLAS_STATUS_INVALID_VALUE;
    const float cv = *c, sv = *s;
    if (cv == 1.f && sv == 0.f) return ICLBLAS_STATUS_SUCCESS;  // iclBLAS_C.cpp:326-327
    return pair_call<cfloat>(h, n, (cfloat*)x, incx, true, (cfloat*)y, incy, true,
                             [&](int nn, cfloat* dx, cfloat* dy) { return iclb::csrot(h, nn, dx, incx, dy, incy, cv, sv); });
}

extern "C" iclblasStatus_t iclblasCrotg(iclblasHandle_t h, oclComplex_t* a, oclComplex_t* b, float* c,
                                        oclComplex_t* s)
{
    return guarded([&]() -> iclblasStatus_t {
        if (!handle_ok(h) || !a || !b || !c || !s) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ia = st.add(a, sizeof(cfloat), true), ib = st.add(b, sizeof(cfloat), false);
        int ic = st.add(c, sizeof(float), true, false), is = st.add(s, sizeof(cfloat), true, false);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::crotg(h, st.dev<cfloat>(ia), st.dev<cfloat>(ib), st.dev<float>(ic), st.dev<cfloat>(is));
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

// ------------------------------------------------------------------------
// level 2
// ------------------------------------------------------------------------
extern "C" iclblasStatus_t iclblasSgemv(iclblasHandle_t h, iclblasOperation_t trans, int m, int n, const float* alpha,
                                        float* A, int lda, float* x, int incx, const float* beta, float* y, int incy)
{
    if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
    // iclBLAS_S.cpp:477-480
    if (m == 0 || n == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    if (m < 0 || n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_A | P_LDA | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.m = m; p.A = A; p.lda = lda; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        const int xl = trans == ICLBLAS_OP_N ? n : m, yl = trans == ICLBLAS_OP_N ? m : n;
        Stager st(h);
        int ia = st.add(A, mat_extent(m, n, lda) * sizeof(float), false);
        int ix = st.add(x, vec_extent(xl, incx) * sizeof(float), false);
        // beta == 0: y is written without being read (contiguous y: nothing to copy in)
        int iy = st.add(y, vec_extent(yl, incy) * sizeof(float), true, *beta != 0.f || incy != 1);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::sgemv(h, trans, m, n, *alpha, st.dev<float>(ia), lda, st.dev<float>(ix), incx, *beta,
                            st.dev<float>(iy), incy);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasCgemv(iclblasHandle_t h, iclblasOperation_t trans, int m, int n,
                                        const oclComplex_t* alpha, oclComplex_t* A, int lda, oclComplex_t* x, int incx,
                                        const oclComplex_t* beta, oclComplex_t* y, int incy)
{
    if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
    const cfloat a = cf(alpha), b = cf(beta);
    // iclBLAS_C.cpp:236-243
    if (m == 0 || n == 0 || (a.re == 0.f && a.im == 0.f && b.re == 1.f && b.im == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    if (m < 0 || n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_A | P_LDA | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.m = m; p.A = A; p.lda = lda; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        const int xl = trans == ICLBLAS_OP_N ? n : m, yl = trans == ICLBLAS_OP_N ? m : n;
        Stager st(h);
        int ia = st.add(A, mat_extent(m, n, lda) * sizeof(cfloat), false);
        int ix = st.add(x, vec_extent(xl, incx) * sizeof(cfloat), false);
        // beta == 0: y is written without being read (contiguous y: nothing to copy in)
        int iy = st.add(y, vec_extent(yl, incy) * sizeof(cfloat), true, b.re != 0.f || b.im != 0.f || incy != 1);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::cgemv(h, trans, m, n, a, st.dev<cfloat>(ia), lda, st.dev<cfloat>(ix), incx, b,
                            st.dev<cfloat>(iy), incy);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasStrsv(iclblasHandle_t h, iclblasFillMode_t uplo, iclblasOperation_t trans,
                                        iclblasDiagType_t diag, int n, float* A, int lda, float* x, int incx)
{
    // iclBLAS_S.cpp:242-244
    if (n == 0) return ICLBLAS_STATUS_SUCCESS;
    if (n < 0 || incx == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_A | P_LDA | P_X | P_INCX;
        p.n = n; p.A = A; p.lda = lda; p.x = x; p.incx = incx;
        VALIDATE(p, h);
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ia = st.add(A, mat_extent(n, n, lda) * sizeof(float), false);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess) e = iclb::strsv(h, uplo, trans, diag, n, st.dev<float>(ia), lda, st.dev<float>(ix), incx);
        if (e == cudaSuccess) e = st.finish();
        if (e != cudaSuccess) return map_cuda(e);
        // device-pointer calls stay asynchronous: iclblasSynchronize reports
        return st.blocking() ? check_device_status(h) : ICLBLAS_STATUS_SUCCESS;
    });
}

extern "C" iclblasStatus_t iclblasCtrsv(iclblasHandle_t h, iclblasFillMode_t uplo, iclblasOperation_t trans,
                                        iclblasDiagType_t diag, int n, oclComplex_t* A, int lda, oclComplex_t* x,
                                        int incx)
{
    if (n == 0) return ICLBLAS_STATUS_SUCCESS;
    if (n < 0 || incx == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_A | P_LDA | P_X | P_INCX;
        p.n = n; p.A = A; p.lda = lda; p.x = x; p.incx = incx;
        VALIDATE(p, h);
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ia = st.add(A, mat_extent(n, n, lda) * sizeof(cfloat), false);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(cfloat), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::ctrsv(h, uplo, trans, diag, n, st.dev<cfloat>(ia), lda, st.dev<cfloat>(ix), incx);
        if (e == cudaSuccess) e = st.finish();
        if (e != cudaSuccess) return map_cuda(e);
        return st.blocking() ? check_device_status(h) : ICLBLAS_STATUS_SUCCESS;
    });
}

// ------------------------------------------------------------------------
// level 2: rank-1 updates and symmetric / Hermitian products
// ------------------------------------------------------------------------
extern "C" iclblasStatus_t iclblasSger(iclblasHandle_t h, int m, int n, const float* alpha, float* x, int incx,
                                       float* y, int incy, float* A, int lda)
{
    if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
    // iclBLAS_S.cpp (Sger): m == 0, n == 0 or alpha == 0 return first
    if (m == 0 || n == 0 || *alpha == 0.f) return ICLBLAS_STATUS_SUCCESS;
    if (m < 0 || n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_X | P_INCX | P_Y | P_INCY | P_A | P_LDA;
        p.n = n; p.m = m; p.x = x; p.incx = incx; p.y = y; p.incy = incy; p.A = A; p.lda = lda;
        VALIDATE(p, h);
        Stager st(h);
        int ix = st.add(x, vec_extent(m, incx) * sizeof(float), false);
        int iy = st.add(y, vec_extent(n, incy) * sizeof(float), false);
        int ia = st.add(A, mat_extent(m, n, lda) * sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::sger(h, m, n, *alpha, st.dev<float>(ix), incx, st.dev<float>(iy), incy, st.dev<float>(ia), lda);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

namespace {
iclblasStatus_t cger_call(iclblasHandle_t h, bool conj, int m, int n, const oclComplex_t* alpha, oclComplex_t* x,
                          int incx, oclComplex_t* y, int incy, oclComplex_t* A, int lda)
{
    if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
    const cfloat a = cf(alpha);
    // iclBLAS_C.cpp (Cgeru / Cgerc): m == 0, n == 0 or alpha == 0 return first
    if (m == 0 || n == 0 || (a.re == 0.f && a.im == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    if (m < 0 || n < 0 || incx == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_X | P_INCX | P_Y | P_INCY | P_A | P_LDA;
        p.n = n; p.m = m; p.x = x; p.incx = incx; p.y = y; p.incy = incy; p.A = A; p.lda = lda;
        VALIDATE(p, h);
        Stager st(h);
        int ix = st.add(x, vec_extent(m, incx) * sizeof(cfloat), false);
        int iy = st.add(y, vec_extent(n, incy) * sizeof(cfloat), false);
        int ia = st.add(A, mat_extent(m, n, lda) * sizeof(cfloat), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::cger(h, conj, m, n, a, st.dev<cfloat>(ix), incx, st.dev<cfloat>(iy), incy, st.dev<cfloat>(ia),
                           lda);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}
}  // namespace

extern "C" iclblasStatus_t iclblasCgeru(iclblasHandle_t h, int m, int n, const oclComplex_t* alpha, oclComplex_t* x,
                                        int incx, oclComplex_t* y, int incy, oclComplex_t* A, int lda)
{
    return cger_call(h, false, m, n, alpha, x, incx, y, incy, A, lda);
}

extern "C" iclblasStatus_t iclblasCgerc(iclblasHandle_t h, int m, int n, const oclComplex_t* alpha, oclComplex_t* x,
                                        int incx, oclComplex_t* y, int incy, oclComplex_t* A, int lda)
{
    return cger_call(h, true, m, n, alpha, x, incx, y, incy, A, lda);
}

extern "C" iclblasStatus_t iclblasSsymv(iclblasHandle_t h, iclblasFillMode_t uplo, int n, const float* alpha,
                                        float* A, int lda, float* x, int incx, const float* beta, float* y, int incy)
{
    if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
    // iclBLAS_S.cpp (Ssymv)
    if (n == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    if (n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_A | P_LDA | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.A = A; p.lda = lda; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        if (uplo != ICLBLAS_FILL_MODE_UPPER && uplo != ICLBLAS_FILL_MODE_LOWER) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ia = st.add(A, mat_extent(n, n, lda) * sizeof(float), false);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(float), false);
        int iy = st.add(y, vec_extent(n, incy) * sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::ssymv(h, uplo, n, *alpha, st.dev<float>(ia), lda, st.dev<float>(ix), incx, *beta,
                            st.dev<float>(iy), incy);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasChemv(iclblasHandle_t h, iclblasFillMode_t uplo, int n, const oclComplex_t* alpha,
                                        oclComplex_t* A, int lda, oclComplex_t* x, int incx, const oclComplex_t* beta,
                                        oclComplex_t* y, int incy)
{
    if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
    const cfloat a = cf(alpha), b = cf(beta);
    // iclBLAS_C.cpp (Chemv)
    if (n == 0 || (a.re == 0.f && a.im == 0.f && b.re == 1.f && b.im == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    if (n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_A | P_LDA | P_X | P_INCX | P_Y | P_INCY;
        p.n = n; p.A = A; p.lda = lda; p.x = x; p.incx = incx; p.y = y; p.incy = incy;
        VALIDATE(p, h);
        if (uplo != ICLBLAS_FILL_MODE_UPPER && uplo != ICLBLAS_FILL_MODE_LOWER) return ICLBLAS_STATUS_INVALID_VALUE;
        Stager st(h);
        int ia = st.add(A, mat_extent(n, n, lda) * sizeof(cfloat), false);
        int ix = st.add(x, vec_extent(n, incx) * sizeof(cfloat), false);
        int iy = st.add(y, vec_extent(n, incy) * sizeof(cfloat), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::chemv(h, uplo, n, a, st.dev<cfloat>(ia), lda, st.dev<cfloat>(ix), incx, b, st.dev<cfloat>(iy),
                            incy);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

// ------------------------------------------------------------------------
// level 3
// ------------------------------------------------------------------------
extern "C" iclblasStatus_t iclblasSgemm(iclblasHandle_t h, iclblasOperation_t transa, iclblasOperation_t transb, int m,
                                        int n, int k, const float* alpha, float* A, int lda, float* B, int ldb,
                                        const float* beta, float* C, int ldc)
{
    if (m < 0 || n < 0 || k < 0) return ICLBLAS_STATUS_INVALID_VALUE;  // iclBLAS_S.cpp:491-492
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_K | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC;
        p.n = n; p.m = m; p.k = k; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
        VALIDATE(p, h);
        if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
        if (transa < ICLBLAS_OP_N || transa > ICLBLAS_OP_C || transb < ICLBLAS_OP_N || transb > ICLBLAS_OP_C)
            return ICLBLAS_STATUS_INVALID_VALUE;
        const int ar = transa == ICLBLAS_OP_N ? m : k, ac = transa == ICLBLAS_OP_N ? k : m;
        const int br = transb == ICLBLAS_OP_N ? k : n, bc = transb == ICLBLAS_OP_N ? n : k;
        Stager st(h);
        int ia = st.add(A, mat_extent(ar, ac, lda) * sizeof(float), false);
        int ib = st.add(B, mat_extent(br, bc, ldb) * sizeof(float), false);
        // beta == 0: C is written without being read (ldc == m: nothing to copy in)
        int ic = st.add(C, mat_extent(m, n, ldc) * sizeof(float), true, *beta != 0.f || ldc != m);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::sgemm(h, transa, transb, m, n, k, *alpha, st.dev<float>(ia), lda, st.dev<float>(ib), ldb, *beta,
                            st.dev<float>(ic), ldc);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasCgemm(iclblasHandle_t h, iclblasOperation_t transa, iclblasOperation_t transb, int m,
                                        int n, int k, const oclComplex_t* alpha, oclComplex_t* A, int lda,
                                        oclComplex_t* B, int ldb, const oclComplex_t* beta, oclComplex_t* C, int ldc)
{
    if (m < 0 || n < 0 || k < 0) return ICLBLAS_STATUS_INVALID_VALUE;  // iclBLAS_C.cpp:462-463
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_K | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC;
        p.n = n; p.m = m; p.k = k; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
        VALIDATE(p, h);
        if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
        if (transa < ICLBLAS_OP_N || transa > ICLBLAS_OP_C || transb < ICLBLAS_OP_N || transb > ICLBLAS_OP_C)
            return ICLBLAS_STATUS_INVALID_VALUE;
        const int ar = transa == ICLBLAS_OP_N ? m : k, ac = transa == ICLBLAS_OP_N ? k : m;
        const int br = transb == ICLBLAS_OP_N ? k : n, bc = transb == ICLBLAS_OP_N ? n : k;
        Stager st(h);
        int ia = st.add(A, mat_extent(ar, ac, lda) * sizeof(cfloat), false);
        int ib = st.add(B, mat_extent(br, bc, ldb) * sizeof(cfloat), false);
        // beta == 0: C is written without being read (ldc == m: nothing to copy in)
        const cfloat bv = cf(beta);
        int ic = st.add(C, mat_extent(m, n, ldc) * sizeof(cfloat), true, bv.re != 0.f || bv.im != 0.f || ldc != m);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::cgemm(h, transa, transb, m, n, k, cf(alpha), st.dev<cfloat>(ia), lda, st.dev<cfloat>(ib), ldb,
                            cf(beta), st.dev<cfloat>(ic), ldc);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasStrsm(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo,
                                        iclblasOperation_t trans, iclblasDiagType_t diag, int m, int n,
                                        const float* alpha, float* A, int lda, float* B, int ldb)
{
    if (m == 0 || n == 0) return ICLBLAS_STATUS_SUCCESS;  // iclBLAS_S.cpp:503-504
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_A | P_LDA | P_B | P_LDB;
        p.n = n; p.m = m; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb;
        VALIDATE(p, h);
        if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        const int na = side == ICLBLAS_SIDE_LEFT ? m : n;
        Stager st(h);
        int ia = st.add(A, mat_extent(na, na, lda) * sizeof(float), false);
        int ib = st.add(B, mat_extent(m, n, ldb) * sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::strsm(h, side, uplo, trans, diag, m, n, *alpha, st.dev<float>(ia), lda, st.dev<float>(ib), ldb);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasCtrsm(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo,
                                        iclblasOperation_t trans, iclblasDiagType_t diag, int m, int n,
                                        const oclComplex_t* alpha, oclComplex_t* A, int lda, oclComplex_t* B, int ldb)
{
    if (m == 0 || n == 0) return ICLBLAS_STATUS_SUCCESS;  // iclBLAS_C.cpp:527-528
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_A | P_LDA | P_B | P_LDB;
        p.n = n; p.m = m; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb;
        VALIDATE(p, h);
        if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        const int na = side == ICLBLAS_SIDE_LEFT ? m : n;
        Stager st(h);
        int ia = st.add(A, mat_extent(na, na, lda) * sizeof(cfloat), false);
        int ib = st.add(B, mat_extent(m, n, ldb) * sizeof(cfloat), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::ctrsm(h, side, uplo, trans, diag, m, n, cf(alpha), st.dev<cfloat>(ia), lda, st.dev<cfloat>(ib),
                            ldb);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

// ------------------------------------------------------------------------
// level 3 on the GEMM engine: syrk, syr2k, symm, trmm
// ------------------------------------------------------------------------
extern "C" iclblasStatus_t iclblasSsyrk(iclblasHandle_t h, iclblasFillMode_t uplo, iclblasOperation_t trans, int n,
                                        int k, const float* alpha, float* A, int lda, const float* beta, float* C,
                                        int ldc)
{
    if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
    // iclBLAS_S.cpp (Ssyrk): n == 0, k == 0 or (alpha == 0 and beta == 1) return first
    if (n == 0 || k == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_K | P_A | P_LDA | P_C | P_LDC;
        p.n = n; p.k = k; p.A = A; p.lda = lda; p.C = C; p.ldc = ldc;
        VALIDATE(p, h);
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        if (uplo != ICLBLAS_FILL_MODE_UPPER && uplo != ICLBLAS_FILL_MODE_LOWER) return ICLBLAS_STATUS_INVALID_VALUE;
        const bool nt = trans == ICLBLAS_OP_N;
        Stager st(h);
        int ia = st.add(A, mat_extent(nt ? n : k, nt ? k : n, lda) * sizeof(float), false);
        int ic = st.add(C, mat_extent(n, n, ldc) * sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::ssyrk(h, uplo, trans, n, k, *alpha, st.dev<float>(ia), lda, *beta, st.dev<float>(ic), ldc);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasSsyr2k(iclblasHandle_t h, iclblasFillMode_t uplo, iclblasOperation_t trans, int n,
                                         int k, const float* alpha, float* A, int lda, float* B, int ldb,
                                         const float* beta, float* C, int ldc)
{
    if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
    // iclBLAS_S.cpp (Ssyr2k)
    if (n == 0 || k == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_K | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC;
        p.n = n; p.k = k; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
        VALIDATE(p, h);
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        if (uplo != ICLBLAS_FILL_MODE_UPPER && uplo != ICLBLAS_FILL_MODE_LOWER) return ICLBLAS_STATUS_INVALID_VALUE;
        const bool nt = trans == ICLBLAS_OP_N;
        Stager st(h);
        int ia = st.add(A, mat_extent(nt ? n : k, nt ? k : n, lda) * sizeof(float), false);
        int ib = st.add(B, mat_extent(nt ? n : k, nt ? k : n, ldb) * sizeof(float), false);
        int ic = st.add(C, mat_extent(n, n, ldc) * sizeof(float), true);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::ssyr2k(h, uplo, trans, n, k, *alpha, st.dev<float>(ia), lda, st.dev<float>(ib), ldb, *beta,
                             st.dev<float>(ic), ldc);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasSsymm(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo, int m,
                                        int n, const float* alpha, float* A, int lda, float* B, int ldb,
                                        const float* beta, float* C, int ldc)
{
    if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
    // iclBLAS_S.cpp (Ssymm)
    if (n == 0 || m == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC;
        p.n = n; p.m = m; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
        VALIDATE(p, h);
        if (side != ICLBLAS_SIDE_LEFT && side != ICLBLAS_SIDE_RIGHT) return ICLBLAS_STATUS_INVALID_VALUE;
        if (uplo != ICLBLAS_FILL_MODE_UPPER && uplo != ICLBLAS_FILL_MODE_LOWER) return ICLBLAS_STATUS_INVALID_VALUE;
        const int na = side == ICLBLAS_SIDE_LEFT ? m : n;
        Stager st(h);
        int ia = st.add(A, mat_extent(na, na, lda) * sizeof(float), false);
        int ib = st.add(B, mat_extent(m, n, ldb) * sizeof(float), false);
        // beta == 0: C is written without being read (ldc == m: nothing to copy in)
        int ic = st.add(C, mat_extent(m, n, ldc) * sizeof(float), true, *beta != 0.f || ldc != m);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::ssymm(h, side, uplo, m, n, *alpha, st.dev<float>(ia), lda, st.dev<float>(ib), ldb, *beta,
                            st.dev<float>(ic), ldc);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasStrmm(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo,
                                        iclblasOperation_t transa, iclblasDiagType_t diag, int m, int n,
                                        const float* alpha, float* A, int lda, float* B, int ldb, float* C, int ldc)
{
    // iclBLAS_S.cpp (Strmm): no early return; the parameter checks end an
    // m == 0 or n == 0 call successfully
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC;
        p.n = n; p.m = m; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
        VALIDATE(p, h);
        if (!alpha) return ICLBLAS_STATUS_INVALID_VALUE;
        if (side != ICLBLAS_SIDE_LEFT && side != ICLBLAS_SIDE_RIGHT) return ICLBLAS_STATUS_INVALID_VALUE;
        if (uplo != ICLBLAS_FILL_MODE_UPPER && uplo != ICLBLAS_FILL_MODE_LOWER) return ICLBLAS_STATUS_INVALID_VALUE;
        if (transa < ICLBLAS_OP_N || transa > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        const int na = side == ICLBLAS_SIDE_LEFT ? m : n;
        Stager st(h);
        int ia = st.add(A, mat_extent(na, na, lda) * sizeof(float), false);
        int ib = st.add(B, mat_extent(m, n, ldb) * sizeof(float), false);
        // C is written in full; its gaps between columns (ldc > m) are kept
        int ic = st.add(C, mat_extent(m, n, ldc) * sizeof(float), true, ldc > m);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::strmm(h, side, uplo, transa, diag, m, n, *alpha, st.dev<float>(ia), lda, st.dev<float>(ib), ldb,
                            st.dev<float>(ic), ldc);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

// ------------------------------------------------------------------------
// half-precision GEMM (extension; the reference ships FP16 GEMM only as the
// stand-alone experimental/kernels/hgemm_buf_*.cl, outside its API)
// ------------------------------------------------------------------------
extern "C" iclblasStatus_t iclblasHgemm(iclblasHandle_t h, iclblasOperation_t transa, iclblasOperation_t transb, int m,
                                        int n, int k, const float* alpha, const unsigned short* A, int lda,
                                        const unsigned short* B, int ldb, const float* beta, unsigned short* C, int ldc)
{
    if (m < 0 || n < 0 || k < 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_K | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC;
        p.n = n; p.m = m; p.k = k; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
        VALIDATE(p, h);
        if (!alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
        if (transa < ICLBLAS_OP_N || transa > ICLBLAS_OP_C || transb < ICLBLAS_OP_N || transb > ICLBLAS_OP_C)
            return ICLBLAS_STATUS_INVALID_VALUE;
        const int ar = transa == ICLBLAS_OP_N ? m : k, ac = transa == ICLBLAS_OP_N ? k : m;
        const int br = transb == ICLBLAS_OP_N ? k : n, bc = transb == ICLBLAS_OP_N ? n : k;
        Stager st(h);
        int ia = st.add(A, mat_extent(ar, ac, lda) * 2, false);
        int ib = st.add(B, mat_extent(br, bc, ldb) * 2, false);
        int ic = st.add(C, mat_extent(m, n, ldc) * 2, true, *beta != 0.f || ldc > m);
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::hgemm(h, transa, transb, m, n, k, *alpha, st.dev<unsigned short>(ia), lda,
                            st.dev<unsigned short>(ib), ldb, *beta, st.dev<unsigned short>(ic), ldc);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

// ------------------------------------------------------------------------
// adjoints (extension)
// ------------------------------------------------------------------------
extern "C" iclblasStatus_t iclblasStrsm_backward(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo,
                                                 iclblasOperation_t trans, iclblasDiagType_t diag, int m, int n,
                                                 const float* alpha, const float* A, int lda, const float* X, int ldx,
                                                 float* G, int ldg, float* dA, int ldda)
{
    if (m == 0 || n == 0) return ICLBLAS_STATUS_SUCCESS;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_A | P_LDA | P_B | P_LDB;
        p.n = n; p.m = m; p.A = A; p.lda = lda; p.B = G; p.ldb = ldg;
        VALIDATE(p, h);
        if (!alpha || !X || ldx <= 0 || (dA && ldda <= 0)) return ICLBLAS_STATUS_INVALID_VALUE;
        if (trans < ICLBLAS_OP_N || trans > ICLBLAS_OP_C) return ICLBLAS_STATUS_INVALID_VALUE;
        const int na = side == ICLBLAS_SIDE_LEFT ? m : n;
        Stager st(h);
        int ia = st.add(A, mat_extent(na, na, lda) * sizeof(float), false);
        int ix = st.add(X, mat_extent(m, n, ldx) * sizeof(float), false);
        int ig = st.add(G, mat_extent(m, n, ldg) * sizeof(float), true);
        int id = dA ? st.add(dA, mat_extent(na, na, ldda) * sizeof(float), true) : -1;
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess)
            e = iclb::strsm_backward(h, side, uplo, trans, diag, m, n, *alpha, st.dev<float>(ia), lda,
                                     st.dev<float>(ix), ldx, st.dev<float>(ig), ldg,
                                     id >= 0 ? st.dev<float>(id) : nullptr, ldda);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

extern "C" iclblasStatus_t iclblasSgemm_backward(iclblasHandle_t h, iclblasOperation_t transa,
                                                 iclblasOperation_t transb, int m, int n, int k, const float* alpha,
                                                 const float* A, int lda, const float* B, int ldb, const float* beta,
                                                 const float* G, int ldg, float* dA, int ldda, float* dB, int lddb,
                                                 float* dC, int lddc)
{
    if (m < 0 || n < 0 || k < 0) return ICLBLAS_STATUS_INVALID_VALUE;
    return guarded([&]() -> iclblasStatus_t {
        Params p; p.present = P_N | P_M | P_K | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC;
        p.n = n; p.m = m; p.k = k; p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = G; p.ldc = ldg;
        VALIDATE(p, h);
        if (!alpha || !beta || (dA && ldda <= 0) || (dB && lddb <= 0) || (dC && lddc <= 0))
            return ICLBLAS_STATUS_INVALID_VALUE;
        if (transa < ICLBLAS_OP_N || transa > ICLBLAS_OP_C || transb < ICLBLAS_OP_N || transb > ICLBLAS_OP_C)
            return ICLBLAS_STATUS_INVALID_VALUE;
        const int ar = transa == ICLBLAS_OP_N ? m : k, ac = transa == ICLBLAS_OP_N ? k : m;
        const int br = transb == ICLBLAS_OP_N ? k : n, bc = transb == ICLBLAS_OP_N ? n : k;
        Stager st(h);
        int ia = st.add(A, mat_extent(ar, ac, lda) * sizeof(float), false);
        int ib = st.add(B, mat_extent(br, bc, ldb) * sizeof(float), false);
        int ig = st.add(G, mat_extent(m, n, ldg) * sizeof(float), false);
        int ida = dA ? st.add(dA, mat_extent(ar, ac, ldda) * sizeof(float), true) : -1;
        int idb = dB ? st.add(dB, mat_extent(br, bc, lddb) * sizeof(float), true) : -1;
        int idc = dC ? st.add(dC, mat_extent(m, n, lddc) * sizeof(float), true) : -1;
        cudaError_t e = st.stage_in();
        if (e == cudaSuccess && k > 0)
            e = iclb::sgemm_backward(h, transa, transb, m, n, k, *alpha, st.dev<float>(ia), lda, st.dev<float>(ib),
                                     ldb, *beta, st.dev<float>(ig), ldg, ida >= 0 ? st.dev<float>(ida) : nullptr,
                                     ldda, idb >= 0 ? st.dev<float>(idb) : nullptr, lddb,
                                     idc >= 0 ? st.dev<float>(idc) : nullptr, lddc);
        else if (e == cudaSuccess && idc >= 0)
            e = iclb::sgemm_backward(h, transa, transb, m, n, 0, *alpha, st.dev<float>(ia), lda, st.dev<float>(ib),
                                     ldb, *beta, st.dev<float>(ig), ldg, nullptr, ldda, nullptr, lddb,
                                     st.dev<float>(idc), lddc);
        if (e == cudaSuccess) e = st.finish();
        return map_cuda(e);
    });
}

// ------------------------------------------------------------------------
// uneven batched TRSM / GEMM (extension)
// ------------------------------------------------------------------------
namespace {

bool plan_ok(iclblasBatchPlan_t p, int kind) { return p != nullptr && p->tag == kBatchPlanTag && p->kind == kind; }

bool op_ok(int t) { return t >= ICLBLAS_OP_N && t <= ICLBLAS_OP_C; }

// Arrays of per-instance pointers must be device memory (the kernels read them).
bool ptr_array_ok(iclblasHandle_t h, const void* p) { return p != nullptr && is_device_ptr(h, p); }

}  // namespace

extern "C" iclblasStatus_t iclblasStrsmBatchedPlanCreate(iclblasHandle_t h, iclblasSideMode_t side,
                                                         iclblasFillMode_t uplo, iclblasOperation_t trans,
                                                         iclblasDiagType_t diag, int batch, const int* m, const int* n,
                                                         const int* lda, const int* ldb, iclblasBatchPlan_t* plan)
{
    return guarded([&]() -> iclblasStatus_t {
        if (!plan) return ICLBLAS_STATUS_INVALID_VALUE;
        *plan = nullptr;
        if (!handle_ok(h) || batch < 0) return ICLBLAS_STATUS_INVALID_VALUE;
        if (batch > 0 && (!m || !n || !lda || !ldb)) return ICLBLAS_STATUS_INVALID_VALUE;
        if ((side != ICLBLAS_SIDE_LEFT && side != ICLBLAS_SIDE_RIGHT) ||
            (uplo != ICLBLAS_FILL_MODE_UPPER && uplo != ICLBLAS_FILL_MODE_LOWER) || !op_ok(trans) ||
            (diag != ICLBLAS_DIAG_NON_UNIT && diag != ICLBLAS_DIAG_UNIT))
            return ICLBLAS_STATUS_INVALID_VALUE;
        const bool right = side == ICLBLAS_SIDE_RIGHT;
        for (int i = 0; i < batch; ++i) {
            if (m[i] < 0 || n[i] < 0) return ICLBLAS_STATUS_INVALID_VALUE;
            const int na = right ? n[i] : m[i];   // order of A
            if (lda[i] < (na > 1 ? na : 1) || ldb[i] < (m[i] > 1 ? m[i] : 1)) return ICLBLAS_STATUS_INVALID_VALUE;
        }
        return map_cuda(iclb::batch_plan_create_trsm(h, side, uplo, trans, diag, batch, m, n, lda, ldb, plan));
    });
}

extern "C" iclblasStatus_t iclblasSgemmBatchedPlanCreate(iclblasHandle_t h, iclblasOperation_t transa,
                                                         iclblasOperation_t transb, int batch, const int* m,
                                                         const int* n, const int* k, const int* lda, const int* ldb,
                                                         const int* ldc, iclblasBatchPlan_t* plan)
{
    return guarded([&]() -> iclblasStatus_t {
        if (!plan) return ICLBLAS_STATUS_INVALID_VALUE;
        *plan = nullptr;
        if (!handle_ok(h) || batch < 0 || !op_ok(transa) || !op_ok(transb)) return ICLBLAS_STATUS_INVALID_VALUE;
        if (batch > 0 && (!m || !n || !k || !lda || !ldb || !ldc)) return ICLBLAS_STATUS_INVALID_VALUE;
        for (int i = 0; i < batch; ++i) {
            if (m[i] < 0 || n[i] < 0 || k[i] < 0) return ICLBLAS_STATUS_INVALID_VALUE;
            const int ar = transa == ICLBLAS_OP_N ? m[i] : k[i];
            const int br = transb == ICLBLAS_OP_N ? k[i] : n[i];
            if (lda[i] < (ar > 1 ? ar : 1) || ldb[i] < (br > 1 ? br : 1) || ldc[i] < (m[i] > 1 ? m[i] : 1))
                return ICLBLAS_STATUS_INVALID_VALUE;
        }
        return map_cuda(iclb::batch_plan_create_gemm(h, transa, transb, batch, m, n, k, lda, ldb, ldc, plan));
    });
}

extern "C" iclblasStatus_t iclblasBatchPlanDestroy(iclblasBatchPlan_t plan)
{
    return guarded([&]() -> iclblasStatus_t {
        if (!plan || plan->tag != kBatchPlanTag) return ICLBLAS_STATUS_INVALID_VALUE;
        iclb::batch_plan_free(plan);
        return ICLBLAS_STATUS_SUCCESS;
    });
}

extern "C" iclblasStatus_t iclblasBatchPlanGetInfo(iclblasBatchPlan_t plan, double* flops, int* tile_width,
                                                   int* ctas_per_sm)
{
    if (!plan || plan->tag != kBatchPlanTag) return ICLBLAS_STATUS_INVALID_VALUE;
    if (flops) *flops = plan->flops;
    if (tile_width) *tile_width = plan->main.rc;
    if (ctas_per_sm) *ctas_per_sm = plan->main.ctas_per_sm;
    return ICLBLAS_STATUS_SUCCESS;
}

extern "C" iclblasStatus_t iclblasBatchPlanSetInverseReuse(iclblasBatchPlan_t plan, int reuse)
{
    if (!plan_ok(plan, 0) || (reuse != 0 && reuse != 1)) return ICLBLAS_STATUS_INVALID_VALUE;
    plan->reuse_inv = reuse == 1;
    return ICLBLAS_STATUS_SUCCESS;
}

extern "C" iclblasStatus_t iclblasStrsmBatchedUneven(iclblasHandle_t h, iclblasBatchPlan_t plan, const float* alpha,
                                                     const float* const* A, float* const* B)
{
    return guarded([&]() -> iclblasStatus_t {
        if (!handle_ok(h) || !plan_ok(plan, 0) || !alpha) return ICLBLAS_STATUS_INVALID_VALUE;
        if (plan->batch == 0) return ICLBLAS_STATUS_SUCCESS;
        if (plan->device != h->device || !ptr_array_ok(h, A) || !ptr_array_ok(h, B)) return ICLBLAS_STATUS_INVALID_VALUE;
        return map_cuda(iclb::batch_trsm(h, plan, *alpha, A, B));
    });
}

extern "C" iclblasStatus_t iclblasSgemmBatchedUneven(iclblasHandle_t h, iclblasBatchPlan_t plan, const float* alpha,
                                                     const float* const* A, const float* const* B, const float* beta,
                                                     float* const* C)
{
    return guarded([&]() -> iclblasStatus_t {
        if (!handle_ok(h) || !plan_ok(plan, 1) || !alpha || !beta) return ICLBLAS_STATUS_INVALID_VALUE;
        if (plan->batch == 0) return ICLBLAS_STATUS_SUCCESS;
        if (plan->device != h->device || !ptr_array_ok(h, A) || !ptr_array_ok(h, B) || !ptr_array_ok(h, C))
            return ICLBLAS_STATUS_INVALID_VALUE;
        return map_cuda(iclb::batch_gemm(h, plan, *alpha, A, B, *beta, C));
    });
}

extern "C" iclblasStatus_t iclblasStrsmBatchedUnevenBackward(iclblasHandle_t h, iclblasBatchPlan_t plan,
                                                             const float* alpha, const float* const* A,
                                                             const float* const* X, float* const* G, float* const* dA)
{
    return guarded([&]() -> iclblasStatus_t {
        if (!handle_ok(h) || !plan_ok(plan, 0) || !alpha) return ICLBLAS_STATUS_INVALID_VALUE;
        if (plan->batch == 0) return ICLBLAS_STATUS_SUCCESS;
        if (plan->device != h->device || !ptr_array_ok(h, A) || !ptr_array_ok(h, X) || !ptr_array_ok(h, G) ||
            (dA && !ptr_array_ok(h, dA)))
            return ICLBLAS_STATUS_INVALID_VALUE;
        return map_cuda(iclb::batch_trsm_backward(h, plan, *alpha, A, X, G, dA));
    });
}
