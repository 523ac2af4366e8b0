// Allocation-free dot product: ltg_dot_noalloc (include/ltg.h).
//
// Variant of the dot kernel of elementwise.cu (per-unit partial sums followed
// by one fixed-order reduction) whose partial sums and result live in a
// file-scope device array instead of memory obtained from cudaMalloc.  After
// the first call on a device, a call allocates nothing, on the device or
// through any library, so it can be used by callers that must not allocate:
//   - error paths after an out-of-memory failure (for example computing a
//     residual norm to decide whether an iteration may continue), where a new
//     allocation would fail again;
//   - programs whose device memory is owned by another allocator that keeps
//     (almost) all of it reserved;
//   - loops sharing the GPU with other streams, where cudaMalloc/cudaFree can
//     synchronise the device and stall them.
//
// Limits and sharing:
//   - the input is cut into units of kUnitElems consecutive elements, one
//     partial sum per unit; at most kMaxUnits units fit the array, so n is
//     limited to kMaxUnits * kUnitElems = 2^30 elements (8 GiB per operand);
//     larger n is rejected with LTG_ERR_BAD_ARG before anything is launched;
//   - every call on a device uses the same array.  Calls that overlap in time
//     on one device (from several host threads, or on several streams without
//     ordering between them) race on it and may return wrong results; callers
//     must serialise them;
//   - nothing in the array has to start at zero: every partial a call reads
//     was written earlier in the same call, and the result slot is written by
//     the reduction (or set to zero by cudaMemsetAsync when n == 0);
//   - the first call on a device is not allocation-free: with CUDA's lazy
//     module loading it loads this file's module (the array and the two
//     kernels' code take device memory then), and it looks the array's
//     address up with cudaGetSymbolAddress, with that device current.  Make
//     one call with n > 0 early on each device, while memory is still free
//     and before any stream capture on the device;
//   - the address is kept per device ordinal for the life of the process;
//     after cudaDeviceReset the module may be loaded at another address, so
//     the entry point must not be used after a device reset.
//
// The summation order depends only on n (units in index order, a fixed tree
// inside each CTA), so repeated calls give bit-identical results.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/ltg.h"

namespace ltg {
void set_last_error(const std::string &msg);
}

constexpr int kNoAllocThreads = 256;
constexpr int64_t kUnitElems = 65536;          // elements per unit (per CTA pass)
constexpr int64_t kMaxUnits = 16384;           // partial sums held by the array
constexpr int64_t kMaxElems = kMaxUnits * kUnitElems;
constexpr int kMaxDevices = 64;

// kMaxUnits partial sums followed by the result slot (128 KiB + 8 bytes).
static __device__ __align__(256) double g_dot_scratch[kMaxUnits + 1];

namespace {

constexpr int kThreads = kNoAllocThreads;

std::mutex g_setup_mtx;
double *g_scratch_ptr[kMaxDevices] = {};

__global__ void __launch_bounds__(kThreads)
dot_units_kernel(const double *__restrict__ x, const double *__restrict__ y, int64_t n,
                 int64_t nunits) {
    __shared__ double red[kThreads];
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int64_t begin = u * kUnitElems;
        const int64_t end = begin + kUnitElems < n ? begin + kUnitElems : n;
        double s = 0.0;
        for (int64_t i = begin + threadIdx.x; i < end; i += kThreads) s += x[i] * y[i];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = kThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) g_dot_scratch[u] = red[0];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads)
dot_reduce_kernel(int64_t nunits) {
    __shared__ double red[kThreads];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < nunits; i += kThreads) s += g_dot_scratch[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) g_dot_scratch[kMaxUnits] = red[0];
}

int fail(int code, const std::string &msg) {
    ltg::set_last_error(msg);
    return code;
}

int cuda_fail(const char *what, cudaError_t e) {
    return fail(e == cudaErrorMemoryAllocation ? LTG_ERR_OOM : LTG_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" int ltg_dot_noalloc(const double *x, const double *y, int64_t n, void *stream,
                               double *out) {
    if (!out) return fail(LTG_ERR_BAD_ARG, "ltg_dot_noalloc: null output pointer");
    if (n < 0) return fail(LTG_ERR_BAD_ARG, "ltg_dot_noalloc: negative element count");
    if (n > kMaxElems)
        return fail(LTG_ERR_BAD_ARG,
                    "ltg_dot_noalloc: " + std::to_string(n) + " elements exceed the maximum of " +
                        std::to_string(kMaxElems) + " (" + std::to_string(kMaxUnits) +
                        " partial sums of " + std::to_string(kUnitElems) + " elements)");
    if (n > 0 && (!x || !y)) return fail(LTG_ERR_BAD_ARG, "ltg_dot_noalloc: null input pointer");
    if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % sizeof(double))
        return fail(LTG_ERR_BAD_ARG, "ltg_dot_noalloc: inputs must be 8-byte aligned");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices)
        return fail(LTG_ERR_UNSUPPORTED, "ltg_dot_noalloc: device ordinal out of range");

    // Per-device set-up, with the device current: the array's address.
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mtx);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_dot_scratch);
            if (e != cudaSuccess) return cuda_fail("cudaGetSymbolAddress", e);
            g_scratch_ptr[dev] = static_cast<double *>(p);
        }
        scratch = g_scratch_ptr[dev];
    }

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double *result = scratch + kMaxUnits;
    const int64_t nunits = (n + kUnitElems - 1) / kUnitElems;
    if (nunits == 0) {
        e = cudaMemsetAsync(result, 0, sizeof(double), s);
        if (e != cudaSuccess) return cuda_fail("cudaMemsetAsync", e);
    } else {
        int nsm = 0;
        e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_fail("cudaDeviceGetAttribute", e);
        if (nsm < 1) nsm = 1;
        const int64_t grid = nunits < 8LL * nsm ? nunits : 8LL * nsm;
        dot_units_kernel<<<(unsigned)grid, kThreads, 0, s>>>(x, y, n, nunits);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail("dot_units_kernel launch", e);
        dot_reduce_kernel<<<1, kThreads, 0, s>>>(nunits);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail("dot_reduce_kernel launch", e);
    }
    e = cudaMemcpyAsync(out, result, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail("cudaMemcpyAsync", e);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail("cudaStreamSynchronize", e);
    return LTG_OK;
}
