// gpufft-b200 benchmarks: device buffers filled with seeded uniform values.
//
// The benchmark programs in this directory time the drop-in API exactly as
// GPU-FFT's own benchmarks do (reference benchmark/*.cu: the same benchmark
// names, axes and calls), so the same source builds against this library
// (include/) or against the reference's library (its src/include), and the
// two can be compared call for call. Like the reference's, they time on
// uniform [0, 1) data and twiddle tables: the values do not change the work.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include <nvbench/nvbench.cuh>

namespace gfbench
{
// uniform [0, 1) from the 53 high bits of a splitmix64 hash of (seed, i)
__host__ __device__ inline double unit_hash(unsigned long long seed, unsigned long long i)
{
    unsigned long long z = seed * 0x9E3779B97F4A7C15ull + i + 1;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

template <typename T> __global__ void fill_unit(T* p, size_t n, unsigned seed)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = (T)unit_hash(seed, i);
}

// `count` elements of T on the device, filled with uniform [0, 1) values of
// the scalar type S (for T = COMPLEX<S>, both parts).
template <typename T, typename S = T> class device_array
{
    static_assert(sizeof(T) % sizeof(S) == 0, "T must be made of S");

  public:
    explicit device_array(size_t count, unsigned seed = 1234) : n_(count)
    {
        if (cudaMalloc(&p_, count * sizeof(T)) != cudaSuccess)
        {
            cudaGetLastError();
            throw std::runtime_error("cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
        }
        fill_unit<S><<<1184, 256>>>(reinterpret_cast<S*>(p_), count * (sizeof(T) / sizeof(S)), seed);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device fill failed");
    }
    ~device_array() { cudaFree(p_); }
    device_array(const device_array&) = delete;
    device_array& operator=(const device_array&) = delete;
    T* data() const { return p_; }
    size_t size() const { return n_; }

  private:
    T* p_ = nullptr;
    size_t n_;
};

// A stream owned by one benchmark state.
class owned_stream
{
  public:
    owned_stream() { cudaStreamCreate(&s_); }
    ~owned_stream()
    {
        cudaStreamSynchronize(s_);
        cudaStreamDestroy(s_);
    }
    cudaStream_t get() const { return s_; }

  private:
    cudaStream_t s_ = nullptr;
};
} // namespace gfbench
