// C_C polynomial product through GPU_FFT: forward of 2 x batch rows of
// 2^(LogN+1) complex, then the inverse with multiplication on batch rows.
// The reference's GPU_FFT_Poly_Mult_Benchmark (benchmark/bench_gpu_fft_C_C_mult.cu):
// same axes (Ring Size LogN 12..23, Batch Count 1) and the same two calls.
#include "gpufft/fft.cuh"

#include "bench_util.cuh"

using namespace gpufft;

#ifdef GPUFFT_BENCH_FLOAT32
typedef Float32 BenchmarkDataType;
#else
typedef Float64 BenchmarkDataType;
#endif
using T = BenchmarkDataType;

void GPU_FFT_Poly_Mult_Benchmark(nvbench::state& state)
{
    const int log_n = (int)state.get_int64("Ring Size LogN");
    const int batch = (int)state.get_int64("Batch Count");
    const size_t m = size_t(1) << (log_n + 1);
    gfbench::device_array<COMPLEX<T>, T> inout(m * 2 * batch);
    gfbench::device_array<COMPLEX<T>, T> roots(m / 2);
    state.collect_l1_hit_rates();
    state.collect_l2_hit_rates();
    gfbench::owned_stream stream;
    state.set_cuda_stream(nvbench::make_cuda_stream_view(stream.get()));

    fft_configuration<T> fwd{};
    fwd.n_power = log_n + 1;
    fwd.fft_type = FORWARD;
    fwd.reduction_poly = ReductionPolynomial::X_N_minus;
    fwd.zero_padding = false;
    fwd.stream = stream.get();
    fft_configuration<T> inv = fwd;
    inv.fft_type = INVERSE;
    inv.mod_inverse = COMPLEX<T>(1.0, 1.0);
    state.exec(
        [&](nvbench::launch&)
        {
            GPU_FFT(inout.data(), roots.data(), fwd, 2 * batch, false);
            GPU_FFT(inout.data(), roots.data(), inv, batch, true);
        });
}

NVBENCH_BENCH(GPU_FFT_Poly_Mult_Benchmark)
    .add_int64_axis("Ring Size LogN", {12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23})
    .add_int64_axis("Batch Count", {1})
    .set_timeout(1);
