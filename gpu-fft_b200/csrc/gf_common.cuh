// gpufft-b200: shared device/host helpers for the sm_100a kernels.
//
// Complex values use the reference's COMPLEX<T> layout (complex.cuh:28-34):
// a float2 / double2 with the real part first. The arithmetic below computes
// the reference's expressions (complex.cuh:65-69 add, 99-104 sub, 133-139 mul)
// with the multiply-add rounding fixed explicitly (see cmul).
#pragma once

#include <atomic>
#include <cstdio>
#include <utility>

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gpufft_b200.h"

namespace gfb
{

template <typename T> struct vec2_of;
template <> struct vec2_of<float> { using type = float2; };
template <> struct vec2_of<double> { using type = double2; };
template <typename T> using cx = typename vec2_of<T>::type;

template <typename T> __host__ __device__ __forceinline__ cx<T> mk(T r, T i)
{
    cx<T> c;
    c.x = r;
    c.y = i;
    return c;
}
template <typename T> __device__ __forceinline__ cx<T> cadd(cx<T> a, cx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cx<T> csub(cx<T> a, cx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
// float: one packed instruction for both components (sm_100's paired FP32
// add / fma; per component they round exactly like the scalar forms, and
// fma(b, -1, a) rounds a - b once, exactly like the subtraction).
template <> __device__ __forceinline__ float2 cadd<float>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub<float>(float2 a, float2 b)
{
    return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
// Products with the rounding spelled out (one plain multiply, one fused
// multiply-add per component) rather than left to the compiler's contraction,
// which may fuse either product of a*b - c*d and may choose differently in
// different kernels: every kernel that runs the same butterfly gets the same
// bits (the batched, per-size, tiled and per-column forms agree exactly).
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T> __device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b)
{
    return mk<T>(rfma(a.x, b.x, -rmul(a.y, b.y)), rfma(a.x, b.y, rmul(a.y, b.x)));
}
// a * conj(b)
template <typename T> __device__ __forceinline__ cx<T> cmulc(cx<T> a, cx<T> b)
{
    return mk<T>(rfma(a.x, b.x, rmul(a.y, b.y)), rfma(a.y, b.x, -rmul(a.x, b.y)));
}

// Radix-2 butterflies, the two units of fft.cuh:69-89.
template <typename T> __device__ __forceinline__ void ct_bfly(cx<T>& U, cx<T>& V, cx<T> w)
{
    cx<T> u = U;
    cx<T> v = cmul<T>(V, w);
    U = cadd<T>(u, v);
    V = csub<T>(u, v);
}
template <typename T> __device__ __forceinline__ void gs_bfly(cx<T>& U, cx<T>& V, cx<T> w)
{
    cx<T> u = U;
    cx<T> v = V;
    U = cadd<T>(u, v);
    V = cmul<T>(csub<T>(u, v), w);
}

// Read-only loads through the non-coherent path; streaming loads and stores
// for data touched once (evict-first in L2 so that twiddle tables and
// inter-pass spectra stay resident).
template <typename T> __device__ __forceinline__ cx<T> ldg(const cx<T>* p) { return __ldg(p); }
template <typename T> __device__ __forceinline__ T ldg_s(const T* p) { return __ldg(p); }
template <typename V> __device__ __forceinline__ V ld_stream(const V* p) { return __ldcs(p); }
template <typename V> __device__ __forceinline__ void st_stream(V* p, V v) { __stcs(p, v); }

// Programmatic dependent launch. The chain kernels are launched with the
// programmatic-serialization attribute (launch_k below), so a kernel's CTAs
// may be scheduled while the previous kernel in the stream is still running.
// Each such kernel calls pdl_begin() before its first global-memory access:
// griddepcontrol.wait returns once every prerequisite grid has completed and
// its writes are visible (at once when the kernel was launched without the
// attribute); launch_dependents then lets the next kernel's CTAs be scheduled
// early in turn. Waiting first keeps at most one grid waiting behind a
// running one.
__device__ __forceinline__ void pdl_begin()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

} // namespace gfb

// Host-side status plumbing shared by every entry point.
namespace gfb
{
int set_cuda_error(cudaError_t e);
int check_launch();

// Launches of the chain kernels (each starts with pdl_begin): with the
// programmatic-serialization attribute while g_pdl is set
// (gpufft_set_programmatic_launch), plain stream order otherwise.
extern std::atomic<int> g_pdl;
template <typename... P, typename... A>
inline int launch_k(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g_pdl.load(std::memory_order_relaxed) ? 1 : 0;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
    if (e != cudaSuccess) return set_cuda_error(e);
    return check_launch();
}

// Per-kernel device-time tracing (gpufft_trace_enable / gpufft_trace_collect).
// While tracing is on, every kernel launch of the product paths is bracketed
// by two CUDA events on its stream and tagged with its name and the
// algorithmic bytes it must move (inputs read once plus outputs written once);
// collecting sums elapsed time and bytes per kernel name. Off, a scope costs
// one relaxed atomic load.
bool trace_on();
void* trace_begin(const char* name, double alg_bytes, cudaStream_t s);
void trace_end(void* rec, cudaStream_t s);
struct TraceScope
{
    void* rec = nullptr;
    cudaStream_t s;
    TraceScope(const char* name, double alg_bytes, cudaStream_t st) : s(st)
    {
        if (trace_on()) rec = trace_begin(name, alg_bytes, st);
    }
    ~TraceScope()
    {
        if (rec) trace_end(rec, s);
    }
    TraceScope(const TraceScope&) = delete;
    TraceScope& operator=(const TraceScope&) = delete;
};
// Declares `var`, a TraceScope named by the printf-style arguments (formatted
// only while tracing is on).
#define GF_TRACE(var, bytes, stream, ...)                                                                              \
    char var##_name[112] = {0};                                                                                        \
    if (::gfb::trace_on()) snprintf(var##_name, sizeof(var##_name), __VA_ARGS__);                                      \
    ::gfb::TraceScope var(var##_name, (double)(bytes), stream)

// Number of SMs of the current device (cached per device ordinal).
inline int sm_count()
{
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev])
    {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

// Round a wave of `w` products down so that w * tiles_per_product CTAs fill
// whole waves of the SMs, when that keeps at least one full step.
inline long long round_wave(long long w, long long tiles_per_product)
{
    long long a = sm_count(), b = tiles_per_product;
    while (b)
    {
        const long long t = a % b;
        a = b;
        b = t;
    }
    const long long step = sm_count() / a;
    if (w >= step) w -= w % step;
    return w;
}

// Opt a kernel into more than 48 KB of dynamic shared memory, once per device.
// `done` must be a per-kernel array of 64 ints (one slot per device ordinal).
template <typename K> int ensure_smem(K* kernel, size_t bytes, int* done)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (dev < 0 || dev >= 64) return set_cuda_error(cudaErrorInvalidDevice);
    if (done[dev] >= (int)bytes) return 0;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return set_cuda_error(e);
    done[dev] = (int)bytes;
    return 0;
}
} // namespace gfb

#define GFB_TRY_CUDA(expr)                                                                       \
    do                                                                                           \
    {                                                                                            \
        cudaError_t _e = (expr);                                                                 \
        if (_e != cudaSuccess) return gfb::set_cuda_error(_e);                                   \
    } while (0)
