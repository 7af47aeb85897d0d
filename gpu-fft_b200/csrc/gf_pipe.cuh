// gpufft-b200: products on host buffers with the PCIe transfers overlapped.
//
// The batch is cut into chunks of whole products. Chunk i is copied host ->
// device on an upload stream, computed on the caller's stream and copied
// device -> host on a download stream, through one of PIPE_SLOTS device
// staging slots, so the upload of chunk i+1 and the download of chunk i-1 run
// while chunk i is computed (PCIe is full duplex: both directions move at
// once). Events order each slot's reuse. The work is ordered after what is
// already queued on the caller's stream, and the caller's stream waits for the
// last download, so the call is asynchronous exactly like the device entry
// points: synchronise the stream before reading the host result.
//
// Host buffers should be page-locked (cudaHostAlloc / pinned tensors); the
// copies are plain cudaMemcpyAsync calls, one per operand and chunk.
#pragma once

#include "gf_common.cuh"

namespace gfb
{

constexpr int PIPE_SLOTS = 3;

inline size_t pipe_align(size_t x) { return (x + 255) & ~(size_t)255; }

// Device bytes of the staging slots for chunks of `chunk` rows.
inline size_t pipe_bytes(long long chunk, size_t in_row, size_t out_row)
{
    return (size_t)PIPE_SLOTS * (2 * pipe_align((size_t)chunk * in_row) + pipe_align((size_t)chunk * out_row));
}

// Streams and events of one call; released when the call returns (the driver
// frees them once the queued work that uses them has finished).
struct PipeRes
{
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t ev[3 * PIPE_SLOTS + 1] = {};
    ~PipeRes()
    {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        if (up) cudaStreamDestroy(up);
        if (down) cudaStreamDestroy(down);
    }
};

// compute(dev_a, dev_b, dev_c, rows, stream) -> status runs one chunk.
template <typename F>
int run_pipeline(const void* a, const void* b, void* c, long long batch, long long chunk, size_t in_row,
                 size_t out_row, void* slots, size_t slots_bytes, cudaStream_t s, F&& compute)
{
    if (!a || !b || !c || batch <= 0 || chunk <= 0) return GPUFFT_ERROR_INVALID_VALUE;
    if (!slots || slots_bytes < pipe_bytes(chunk, in_row, out_row)) return GPUFFT_ERROR_WORKSPACE;
    if ((uintptr_t)slots % 256) return GPUFFT_ERROR_MISALIGNED;
    PipeRes R;
    cudaError_t e = cudaStreamCreateWithFlags(&R.up, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&R.down, cudaStreamNonBlocking);
    for (cudaEvent_t& ev : R.ev)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return set_cuda_error(e);
    cudaEvent_t* loaded = R.ev;
    cudaEvent_t* computed = R.ev + PIPE_SLOTS;
    cudaEvent_t* unloaded = R.ev + 2 * PIPE_SLOTS;
    cudaEvent_t fence = R.ev[3 * PIPE_SLOTS];

#define GF_PIPE_TRY(call)                                                                                              \
    do                                                                                                                 \
    {                                                                                                                  \
        const cudaError_t e_ = (call);                                                                                 \
        if (e_ != cudaSuccess) return set_cuda_error(e_);                                                              \
    } while (0)

    GF_PIPE_TRY(cudaEventRecord(fence, s));
    GF_PIPE_TRY(cudaStreamWaitEvent(R.up, fence, 0));
    GF_PIPE_TRY(cudaStreamWaitEvent(R.down, fence, 0));
    const size_t sa = pipe_align((size_t)chunk * in_row), sc = pipe_align((size_t)chunk * out_row);
    const char* ha = static_cast<const char*>(a);
    const char* hb = static_cast<const char*>(b);
    char* hc = static_cast<char*>(c);
    long long i = 0;
    for (long long p0 = 0; p0 < batch; p0 += chunk, i++)
    {
        const int k = (int)(i % PIPE_SLOTS);
        const long long rows = (batch - p0) < chunk ? (batch - p0) : chunk;
        char* da = static_cast<char*>(slots) + (size_t)k * (2 * sa + sc);
        char* db = da + sa;
        char* dc = db + sa;
        // the slot's inputs are free once the chunk that used it was computed
        if (i >= PIPE_SLOTS) GF_PIPE_TRY(cudaStreamWaitEvent(R.up, computed[k], 0));
        GF_PIPE_TRY(cudaMemcpyAsync(da, ha + (size_t)p0 * in_row, (size_t)rows * in_row, cudaMemcpyHostToDevice, R.up));
        GF_PIPE_TRY(cudaMemcpyAsync(db, hb + (size_t)p0 * in_row, (size_t)rows * in_row, cudaMemcpyHostToDevice, R.up));
        GF_PIPE_TRY(cudaEventRecord(loaded[k], R.up));
        GF_PIPE_TRY(cudaStreamWaitEvent(s, loaded[k], 0));
        // its output is free once that chunk's result was copied out
        if (i >= PIPE_SLOTS) GF_PIPE_TRY(cudaStreamWaitEvent(s, unloaded[k], 0));
        const int st = compute(da, db, dc, rows, s);
        if (st) return st;
        GF_PIPE_TRY(cudaEventRecord(computed[k], s));
        GF_PIPE_TRY(cudaStreamWaitEvent(R.down, computed[k], 0));
        GF_PIPE_TRY(cudaMemcpyAsync(hc + (size_t)p0 * out_row, dc, (size_t)rows * out_row, cudaMemcpyDeviceToHost,
                                    R.down));
        GF_PIPE_TRY(cudaEventRecord(unloaded[k], R.down));
    }
    // the caller's stream resumes after the last download
    GF_PIPE_TRY(cudaEventRecord(fence, R.down));
    GF_PIPE_TRY(cudaStreamWaitEvent(s, fence, 0));
#undef GF_PIPE_TRY
    return GPUFFT_SUCCESS;
}

// Default chunk: one wave of the product, but at least eight chunks per call so
// that uploads, compute and downloads overlap for most of the call (measured at
// N = 2^16, batch 256: eight chunks beat four by 3 % on both the FP64 and the
// split product; sixteen gain nothing more).
inline long long pipe_chunk(long long wave, long long batch)
{
    const long long eighth = (batch + 7) / 8;
    long long c = wave < eighth ? wave : eighth;
    return c < 1 ? 1 : c;
}

} // namespace gfb
