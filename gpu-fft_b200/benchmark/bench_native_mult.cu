// The native products of this library on the drop-in benchmarks' axes (Ring
// Size LogN 12..23, Batch Count 1): the fused FP64 negacyclic product
// (gpufft_negacyclic_mul_f64) and the exact FP32 split product of 24-bit
// coefficients (gpufft_negacyclic_mul_split_f32), each one call per product
// batch on device tables from gpufft_ffnt_make_tables_*. No reference
// counterpart: these entry points exist only here (include/gpufft_b200.h).
#include "gpufft_b200.h"

#include "bench_util.cuh"

namespace
{
__global__ void fill_bits(int32_t* p, size_t n, unsigned seed, int bits)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = (int32_t)(gfbench::unit_hash(seed, i) * (double)(1 << bits));
}

void check(int st, nvbench::state& state, const char* what)
{
    if (st != 0) state.skip(std::string(what) + ": " + gpufft_status_string(st));
}

// inside a timed call: a failed status ends the state (the harness skips it)
void must(int st)
{
    if (st != 0) throw std::runtime_error(gpufft_status_string(st));
}

class raw_buffer
{
  public:
    explicit raw_buffer(size_t bytes)
    {
        if (cudaMalloc(&p_, bytes ? bytes : 16) != cudaSuccess)
        {
            cudaGetLastError();
            throw std::runtime_error("cudaMalloc failed");
        }
    }
    ~raw_buffer() { cudaFree(p_); }
    void* get() const { return p_; }

  private:
    void* p_ = nullptr;
};
} // namespace

void NATIVE_FFNT_Mult_Benchmark(nvbench::state& state)
{
    const int log_n = (int)state.get_int64("Ring Size LogN");
    const int batch = (int)state.get_int64("Batch Count");
    const size_t n = size_t(1) << log_n;
    gfbench::device_array<double> a(n * batch, 1), b(n * batch, 2), c(n * batch, 3);
    raw_buffer tables(gpufft_ffnt_tables_count(log_n) * 16);
    const size_t ws_bytes = gpufft_negacyclic_mul_workspace_bytes(log_n, batch, 64);
    raw_buffer ws(ws_bytes);
    gfbench::owned_stream stream;
    state.set_cuda_stream(nvbench::make_cuda_stream_view(stream.get()));
    check(gpufft_ffnt_make_tables_f64(log_n, tables.get(), stream.get()), state, "tables");
    state.add_global_memory_reads<double>(2 * n * batch, "a, b");
    state.add_global_memory_writes<double>(n * batch, "c");
    state.exec(
        [&](nvbench::launch&)
        {
            must(gpufft_negacyclic_mul_f64(a.data(), b.data(), c.data(), log_n, batch, tables.get(), ws.get(),
                                           ws_bytes, stream.get()));
        });
}

void NATIVE_Split_Mult_Benchmark(nvbench::state& state)
{
    const int log_n = (int)state.get_int64("Ring Size LogN");
    const int batch = (int)state.get_int64("Batch Count");
    const size_t n = size_t(1) << log_n;
    int limb_bits = 0, limbs = 0;
    check(gpufft_split_plan(log_n, 24, 1, &limb_bits, &limbs), state, "limb plan for 24-bit inputs");
    if (state.is_skipped()) return;
    raw_buffer a(n * batch * 4), b(n * batch * 4), c(n * batch * 8), err(4);
    fill_bits<<<1184, 256>>>(static_cast<int32_t*>(a.get()), n * batch, 1, 24);
    fill_bits<<<1184, 256>>>(static_cast<int32_t*>(b.get()), n * batch, 2, 24);
    raw_buffer tables(gpufft_ffnt_tables_count(log_n) * 8);
    const size_t ws_bytes = gpufft_negacyclic_mul_split_workspace_bytes(log_n, batch, limbs);
    raw_buffer ws(ws_bytes);
    gfbench::owned_stream stream;
    state.set_cuda_stream(nvbench::make_cuda_stream_view(stream.get()));
    check(gpufft_ffnt_make_tables_f32(log_n, tables.get(), stream.get()), state, "tables");
    cudaDeviceSynchronize();
    state.add_global_memory_reads<int32_t>(2 * n * batch, "a, b");
    state.add_global_memory_writes<int64_t>(n * batch, "c");
    state.exec(
        [&](nvbench::launch&)
        {
            must(gpufft_negacyclic_mul_split_f32(
                static_cast<const int32_t*>(a.get()), static_cast<const int32_t*>(b.get()),
                static_cast<int64_t*>(c.get()), log_n, batch, 24, 1, limb_bits, limbs, tables.get(), ws.get(),
                ws_bytes, static_cast<float*>(err.get()), stream.get()));
        });
}

NVBENCH_BENCH(NATIVE_FFNT_Mult_Benchmark)
    .add_int64_axis("Ring Size LogN", {12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23})
    .add_int64_axis("Batch Count", {1})
    .set_timeout(1);

NVBENCH_BENCH(NATIVE_Split_Mult_Benchmark)
    .add_int64_axis("Ring Size LogN", {12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23})
    .add_int64_axis("Batch Count", {1})
    .set_timeout(1);
