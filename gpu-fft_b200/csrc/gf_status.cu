// gpufft-b200: status codes and CUDA error capture for the C ABI.
//
// The reference reports launch failures by throwing CudaException from
// GPUFFT_CUDA_CHECK(cudaGetLastError()) after every launch
// (common_fft.cuh:41-49, e.g. fft.cu:555). Across a C ABI there are no
// exceptions, so the failing cudaError_t is kept per host thread and the
// entry point returns GPUFFT_ERROR_CUDA; the C++ drop-in rethrows it.
#include "gf_common.cuh"

#include <atomic>

namespace
{
thread_local int g_last_cuda_error = 0;
}

namespace gfb
{

// Contiguous 12-stage passes over at most this many 4096-point tiles run as
// thread-block clusters (gf_cluster.cuh); 0 disables them.
std::atomic<int> g_cluster_max_tiles{64};
// Chain kernels launched with programmatic stream serialization (gf_common.cuh).
std::atomic<int> g_pdl{1};
int set_cuda_error(cudaError_t e)
{
    g_last_cuda_error = (int)e;
    return GPUFFT_ERROR_CUDA;
}

int check_launch()
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error(e);
    return GPUFFT_SUCCESS;
}
} // namespace gfb

// ---------------------------------------------------------------------------
// Tracing: per-kernel device time from CUDA events around each launch.
// ---------------------------------------------------------------------------
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace
{
struct TraceRec
{
    std::string name;
    double bytes;
    int device;
    cudaEvent_t a, b;
};
std::atomic<int> g_trace_on{0};
std::mutex g_trace_mu;
std::vector<TraceRec*> g_trace_recs;
// Events are reused (creating two per launch would make the host, not the
// GPU, the bottleneck of a traced run, and a starved stream would count launch
// gaps as kernel time). One pool per device: an event belongs to the device
// that was current when it was created.
std::map<int, std::vector<cudaEvent_t>> g_event_pool;

cudaEvent_t pool_get(int dev)
{
    {
        std::lock_guard<std::mutex> lock(g_trace_mu);
        auto& v = g_event_pool[dev];
        if (!v.empty())
        {
            cudaEvent_t e = v.back();
            v.pop_back();
            return e;
        }
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

void pool_put(int dev, cudaEvent_t e)
{
    if (!e) return;
    std::lock_guard<std::mutex> lock(g_trace_mu);
    g_event_pool[dev].push_back(e);
}
} // namespace

namespace gfb
{
bool trace_on() { return g_trace_on.load(std::memory_order_relaxed) != 0; }

void* trace_begin(const char* name, double alg_bytes, cudaStream_t s)
{
    // launches being captured into a graph are not timed
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    auto* r = new TraceRec{name, alg_bytes, dev, pool_get(dev), pool_get(dev)};
    if (!r->a || !r->b || cudaEventRecord(r->a, s) != cudaSuccess)
    {
        pool_put(dev, r->a);
        pool_put(dev, r->b);
        delete r;
        return nullptr;
    }
    return r;
}

void trace_end(void* rec, cudaStream_t s)
{
    auto* r = static_cast<TraceRec*>(rec);
    if (cudaEventRecord(r->b, s) != cudaSuccess)
    {
        pool_put(r->device, r->a);
        pool_put(r->device, r->b);
        delete r;
        return;
    }
    std::lock_guard<std::mutex> lock(g_trace_mu);
    g_trace_recs.push_back(r);
}
} // namespace gfb

extern "C" int gpufft_trace_enable(int on)
{
    g_trace_on.store(on ? 1 : 0, std::memory_order_relaxed);
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_trace_collect(int max_rows, char* names, int name_len, double* total_ms, double* alg_bytes,
                                    long long* launches, int* rows)
{
    if (!rows || (max_rows > 0 && (!names || name_len < 2 || !total_ms || !alg_bytes || !launches)))
        return GPUFFT_ERROR_INVALID_VALUE;
    std::vector<TraceRec*> recs;
    {
        std::lock_guard<std::mutex> lock(g_trace_mu);
        recs.swap(g_trace_recs);
    }
    struct Agg
    {
        double ms = 0, bytes = 0;
        long long n = 0;
    };
    std::map<std::string, Agg> agg;
    int status = GPUFFT_SUCCESS;
    for (TraceRec* r : recs)
    {
        float ms = 0.f;
        cudaError_t e = cudaEventSynchronize(r->b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, r->a, r->b);
        if (e != cudaSuccess && status == GPUFFT_SUCCESS) status = gfb::set_cuda_error(e);
        Agg& g = agg[r->name];
        g.ms += ms;
        g.bytes += r->bytes;
        g.n += 1;
        pool_put(r->device, r->a);
        pool_put(r->device, r->b);
        delete r;
    }
    int k = 0;
    for (const auto& kv : agg)
    {
        if (k >= max_rows) break;
        snprintf(names + (size_t)k * name_len, (size_t)name_len, "%s", kv.first.c_str());
        total_ms[k] = kv.second.ms;
        alg_bytes[k] = kv.second.bytes;
        launches[k] = kv.second.n;
        k++;
    }
    *rows = k;
    return status;
}

extern "C" int gpufft_last_cuda_error(void) { return g_last_cuda_error; }

extern "C" const char* gpufft_status_string(int status)
{
    switch (status)
    {
    case GPUFFT_SUCCESS: return "success";
    case GPUFFT_ERROR_INVALID_N_POWER: return "Invalid n_power range!";
    case GPUFFT_ERROR_INVALID_VALUE: return "invalid argument";
    case GPUFFT_ERROR_CUDA: return "CUDA error (see gpufft_last_cuda_error)";
    case GPUFFT_ERROR_WORKSPACE: return "workspace too small";
    case GPUFFT_ERROR_MISALIGNED: return "misaligned device pointer";
    default: return "unknown status";
    }
}

extern "C" int gpufft_version(void) { return 100; }

extern "C" int gpufft_set_programmatic_launch(int on)
{
    if (on < 0) return gfb::g_pdl.load(std::memory_order_relaxed);
    return gfb::g_pdl.exchange(on ? 1 : 0, std::memory_order_relaxed);
}

extern "C" int gpufft_set_cluster_tiles(int max_tiles)
{
    if (max_tiles < 0) return gfb::g_cluster_max_tiles.load(std::memory_order_relaxed);
    return gfb::g_cluster_max_tiles.exchange(max_tiles, std::memory_order_relaxed);
}
