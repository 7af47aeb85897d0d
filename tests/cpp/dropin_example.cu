// A downstream program written against the reference's C++ API (the flow of
// the reference's example/test_ffnt_gpu_R_R.cu and example/test_fft_gpu_R_R.cu),
// compiled unchanged against the drop-in headers in include/gpufft/ and linked
// with -lgpufft_b200. Seeded inputs; results are checked exactly against a
// 128-bit schoolbook product instead of the reference's mod-7 check.
// Usage: dropin_example <logn> <batch>; exit code 0 on success.
#include "gpufft/fft.cuh"

#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

using namespace gpufft;

typedef Float64 TestDataType;

static std::vector<__int128> negacyclic(const std::vector<long long>& a, const std::vector<long long>& b)
{
    const int n = (int)a.size();
    std::vector<__int128> r(n, 0);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
        {
            const __int128 p = (__int128)a[i] * b[j];
            if (i + j < n)
                r[i + j] += p;
            else
                r[i + j - n] -= p;
        }
    return r;
}

int main(int argc, char* argv[])
{
    const int logn = argc > 1 ? atoi(argv[1]) : 12;
    const int batch = argc > 2 ? atoi(argv[2]) : 2;
    const int n = 1 << logn;
    std::mt19937_64 gen(20261203);
    std::uniform_int_distribution<long long> dis(0, (1 << 12) - 1);

    // ---- FFNT negacyclic product (GPU_FFNT forward on 2*batch, inverse with product)
    std::vector<std::vector<long long>> A(batch, std::vector<long long>(n)), B = A;
    std::vector<TestDataType> host(2 * batch * n);
    for (int k = 0; k < batch; k++)
        for (int i = 0; i < n; i++)
        {
            A[k][i] = dis(gen);
            B[k][i] = dis(gen);
            host[k * n + i] = (TestDataType)A[k][i];
            host[(batch + k) * n + i] = (TestDataType)B[k][i];
        }
    FFNT<TestDataType> gen_tables(n);
    std::vector<COMPLEX<TestDataType>> roots = gen_tables.ReverseRootTable_ffnt();
    std::vector<COMPLEX<TestDataType>> inv_roots = gen_tables.InverseReverseRootTable_ffnt();
    std::vector<COMPLEX<TestDataType>> twist = gen_tables.twist_table_ffnt();
    std::vector<COMPLEX<TestDataType>> untwist = gen_tables.untwist_table_ffnt();

    TestDataType* inout;
    COMPLEX<TestDataType> *temp, *d_roots, *d_inv, *d_tw, *d_utw;
    const size_t tb = (n >> 1) * sizeof(COMPLEX<TestDataType>);
    GPUFFT_CUDA_CHECK(cudaMalloc(&inout, host.size() * sizeof(TestDataType)));
    GPUFFT_CUDA_CHECK(cudaMalloc(&temp, 2 * batch * tb));
    GPUFFT_CUDA_CHECK(cudaMalloc(&d_roots, tb));
    GPUFFT_CUDA_CHECK(cudaMalloc(&d_inv, tb));
    GPUFFT_CUDA_CHECK(cudaMalloc(&d_tw, tb));
    GPUFFT_CUDA_CHECK(cudaMalloc(&d_utw, tb));
    GPUFFT_CUDA_CHECK(cudaMemcpy(inout, host.data(), host.size() * sizeof(TestDataType), cudaMemcpyHostToDevice));
    GPUFFT_CUDA_CHECK(cudaMemcpy(d_roots, roots.data(), tb, cudaMemcpyHostToDevice));
    GPUFFT_CUDA_CHECK(cudaMemcpy(d_inv, inv_roots.data(), tb, cudaMemcpyHostToDevice));
    GPUFFT_CUDA_CHECK(cudaMemcpy(d_tw, twist.data(), tb, cudaMemcpyHostToDevice));
    GPUFFT_CUDA_CHECK(cudaMemcpy(d_utw, untwist.data(), tb, cudaMemcpyHostToDevice));

    fft_configuration<TestDataType> cfg_fft{};
    cfg_fft.n_power = logn;
    cfg_fft.fft_type = FORWARD;
    cfg_fft.zero_padding = false;
    cfg_fft.stream = 0;
    GPU_FFNT(inout, temp, d_tw, d_roots, cfg_fft, batch * 2, false);

    fft_configuration<TestDataType> cfg_ifft{};
    cfg_ifft.n_power = logn;
    cfg_ifft.fft_type = INVERSE;
    cfg_ifft.zero_padding = false;
    cfg_ifft.mod_inverse = COMPLEX<TestDataType>(1.0 / (n >> 1), 0.0);
    cfg_ifft.stream = 0;
    GPU_FFNT(inout, temp, d_utw, d_inv, cfg_ifft, batch, true);

    GPUFFT_CUDA_CHECK(cudaMemcpy(host.data(), inout, batch * n * sizeof(TestDataType), cudaMemcpyDeviceToHost));
    int bad = 0;
    for (int k = 0; k < batch; k++)
    {
        std::vector<__int128> want = negacyclic(A[k], B[k]);
        for (int i = 0; i < n; i++)
            if ((__int128)std::llround(host[k * n + i]) != want[i]) bad++;
    }

    // ---- the reference's range check and exception types
    bool threw = false;
    try
    {
        fft_configuration<TestDataType> bad_cfg = cfg_fft;
        bad_cfg.n_power = 11;
        GPU_FFNT(inout, temp, d_tw, d_roots, bad_cfg, 1, false);
    }
    catch (const std::invalid_argument& e)
    {
        threw = std::string(e.what()) == "Invalid n_power range!";
    }

    cudaFree(inout);
    cudaFree(temp);
    cudaFree(d_roots);
    cudaFree(d_inv);
    cudaFree(d_tw);
    cudaFree(d_utw);
    std::printf("dropin_example logn=%d batch=%d mismatches=%d range_check=%s\n", logn, batch, bad,
                threw ? "ok" : "FAILED");
    return (bad == 0 && threw) ? 0 : 1;
}
