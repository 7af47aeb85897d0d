// GPU_FFT (COMPLEX<T> in place) forward and inverse, one transform of
// 2^(LogN+1) points per batch row: the benchmark GPU_FFT_Forward_Benchmark /
// GPU_FFT_Inverse_Benchmark of the reference (benchmark/bench_gpu_fft.cu), same
// axes (Ring Size LogN 12..23, Batch Count 1) and the same calls.
// Declared memory traffic: one read and one write of every row.
#include "gpufft/fft.cuh"

#include "bench_util.cuh"

using namespace gpufft;

#ifdef GPUFFT_BENCH_FLOAT32
typedef Float32 BenchmarkDataType;
#else
typedef Float64 BenchmarkDataType;
#endif
using T = BenchmarkDataType;

static void fft_c2c(nvbench::state& state, type dir)
{
    const int log_n = (int)state.get_int64("Ring Size LogN");
    const int batch = (int)state.get_int64("Batch Count");
    const size_t m = size_t(1) << (log_n + 1); // transform length
    gfbench::device_array<COMPLEX<T>, T> inout(2 * m * batch);
    gfbench::device_array<COMPLEX<T>, T> roots(m / 2);
    state.add_global_memory_reads<COMPLEX<T>>(m * batch, "Read Memory Size");
    state.add_global_memory_writes<COMPLEX<T>>(m * batch, "Write Memory Size");
    state.collect_l1_hit_rates();
    state.collect_l2_hit_rates();
    gfbench::owned_stream stream;
    state.set_cuda_stream(nvbench::make_cuda_stream_view(stream.get()));

    fft_configuration<T> cfg{};
    cfg.n_power = log_n + 1;
    cfg.fft_type = dir;
    cfg.reduction_poly = ReductionPolynomial::X_N_minus;
    cfg.zero_padding = false;
    cfg.mod_inverse = COMPLEX<T>(1.0, 1.0);
    cfg.stream = stream.get();
    state.exec([&](nvbench::launch&) { GPU_FFT(inout.data(), roots.data(), cfg, batch, false); });
}

void GPU_FFT_Forward_Benchmark(nvbench::state& state) { fft_c2c(state, FORWARD); }
void GPU_FFT_Inverse_Benchmark(nvbench::state& state) { fft_c2c(state, INVERSE); }

NVBENCH_BENCH(GPU_FFT_Forward_Benchmark)
    .add_int64_axis("Ring Size LogN", {12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23})
    .add_int64_axis("Batch Count", {1})
    .set_timeout(1);

NVBENCH_BENCH(GPU_FFT_Inverse_Benchmark)
    .add_int64_axis("Ring Size LogN", {12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23})
    .add_int64_axis("Batch Count", {1})
    .set_timeout(1);
