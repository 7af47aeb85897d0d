// gpufft-b200 drop-in header: the GPU transform API.
//
// Same names and signatures as the reference's src/include/gpufft/fft.cuh
// (namespace gpufft: location_t, type {FORWARD, INVERSE},
// fft_configuration<T>, GPU_FFT for C_C and R_R, GPU_FFNT), implemented as
// thin inline templates over the C ABI of libgpufft_b200 (gpufft_b200.h).
// A program written against the reference recompiles unchanged and links
// -lgpufft_b200 instead of GPUFFT::fft.
//
// Behaviour kept from the reference (fft.cu:517-725, 1386-1515):
//  * std::invalid_argument("Invalid n_power range!") unless 12 <= n_power <= 24;
//  * gpufft::CudaException when a launch fails;
//  * asynchronous on cfg.stream, no synchronisation, no allocation;
//  * for the FFNT inverse the third argument is the untwist table.
// One difference: zero_padding = true is honoured (the upper half of every
// forward input is taken as zero and not read) where the reference ignores it.
#ifndef GPUFFT_B200_FFT_CUH
#define GPUFFT_B200_FFT_CUH

#include <stdexcept>
#include <string>

#include "../gpufft_b200.h"
#include "common_fft.cuh"
#include "complex.cuh"
#include "fft_cpu.cuh"

namespace gpufft
{
typedef unsigned location_t;

enum type
{
    FORWARD,
    INVERSE
};

template <typename T> struct fft_configuration
{
    int n_power;
    type fft_type;
    ReductionPolynomial reduction_poly;
    bool zero_padding;
    COMPLEX<T> mod_inverse;
    cudaStream_t stream;
};

// Launch-shape record of the reference's per-size tables; kept so that code
// naming it still compiles. The library plans its own passes.
struct KernelConfig
{
    int griddim_x;
    int griddim_y;
    int blockdim_x;
    int blockdim_y;
    size_t shared_memory;
    int shared_index;
    int logm;
    int k;
    int outer_iteration_count;
    bool not_last_kernel;
};

#if defined(__CUDACC__)
// The two radix-2 butterflies (reference fft.cuh:69-89).
template <typename T> __device__ __forceinline__ void CooleyTukeyUnit(COMPLEX<T>& U, COMPLEX<T>& V, COMPLEX<T>& root)
{
    const COMPLEX<T> u = U;
    const COMPLEX<T> v = V * root;
    U = u + v;
    V = u - v;
}
template <typename T>
__device__ __forceinline__ void GentlemanSandeUnit(COMPLEX<T>& U, COMPLEX<T>& V, COMPLEX<T>& root)
{
    const COMPLEX<T> u = U;
    const COMPLEX<T> v = V;
    U = u + v;
    V = (u - v) * root;
}
#endif

namespace detail
{
inline void raise_status(int status, const char* file, int line)
{
    if (status == GPUFFT_SUCCESS) return;
    if (status == GPUFFT_ERROR_INVALID_N_POWER) throw std::invalid_argument("Invalid n_power range!");
    if (status == GPUFFT_ERROR_CUDA) throw CudaException(file, line, static_cast<cudaError_t>(gpufft_last_cuda_error()));
    throw std::runtime_error(std::string("gpufft: ") + gpufft_status_string(status));
}

inline void check_range(int n_power)
{
    if (n_power <= 11 || n_power >= 25) throw std::invalid_argument("Invalid n_power range!");
}

inline int c2c(COMPLEX<float>* io, COMPLEX<float>* r, const fft_configuration<float>& c, int b, bool m)
{
    return gpufft_fft_c2c_f32(io, r, c.n_power, c.fft_type, c.reduction_poly, c.zero_padding, c.mod_inverse.real(),
                              c.mod_inverse.imag(), b, m, reinterpret_cast<gpufft_stream_t>(c.stream));
}
inline int c2c(COMPLEX<double>* io, COMPLEX<double>* r, const fft_configuration<double>& c, int b, bool m)
{
    return gpufft_fft_c2c_f64(io, r, c.n_power, c.fft_type, c.reduction_poly, c.zero_padding, c.mod_inverse.real(),
                              c.mod_inverse.imag(), b, m, reinterpret_cast<gpufft_stream_t>(c.stream));
}
inline int r2r(float* io, COMPLEX<float>* t, COMPLEX<float>* r, const fft_configuration<float>& c, int b, bool m)
{
    return gpufft_fft_r2r_f32(io, t, r, c.n_power, c.fft_type, c.reduction_poly, c.zero_padding,
                              c.mod_inverse.real(), c.mod_inverse.imag(), b, m,
                              reinterpret_cast<gpufft_stream_t>(c.stream));
}
inline int r2r(double* io, COMPLEX<double>* t, COMPLEX<double>* r, const fft_configuration<double>& c, int b, bool m)
{
    return gpufft_fft_r2r_f64(io, t, r, c.n_power, c.fft_type, c.reduction_poly, c.zero_padding,
                              c.mod_inverse.real(), c.mod_inverse.imag(), b, m,
                              reinterpret_cast<gpufft_stream_t>(c.stream));
}
inline int ffnt(float* io, COMPLEX<float>* t, COMPLEX<float>* tw, COMPLEX<float>* r,
                const fft_configuration<float>& c, int b, bool m)
{
    return gpufft_ffnt_f32(io, t, tw, r, c.n_power, c.fft_type, c.mod_inverse.real(), c.mod_inverse.imag(), b, m,
                           reinterpret_cast<gpufft_stream_t>(c.stream));
}
inline int ffnt(double* io, COMPLEX<double>* t, COMPLEX<double>* tw, COMPLEX<double>* r,
                const fft_configuration<double>& c, int b, bool m)
{
    return gpufft_ffnt_f64(io, t, tw, r, c.n_power, c.fft_type, c.mod_inverse.real(), c.mod_inverse.imag(), b, m,
                           reinterpret_cast<gpufft_stream_t>(c.stream));
}
inline int special(COMPLEX<float>* io, COMPLEX<float>* r, const fft_configuration<float>& c, int b)
{
    return gpufft_special_fft_f32(io, r, c.n_power, c.fft_type, c.mod_inverse.real(), c.mod_inverse.imag(), b,
                                  reinterpret_cast<gpufft_stream_t>(c.stream));
}
inline int special(COMPLEX<double>* io, COMPLEX<double>* r, const fft_configuration<double>& c, int b)
{
    return gpufft_special_fft_f64(io, r, c.n_power, c.fft_type, c.mod_inverse.real(), c.mod_inverse.imag(), b,
                                  reinterpret_cast<gpufft_stream_t>(c.stream));
}
} // namespace detail

// COMPLEX<T> to COMPLEX<T> (reference fft.cuh:120-124)
template <typename T>
inline void GPU_FFT(COMPLEX<T>* device_inout, COMPLEX<T>* root_of_unity_table, fft_configuration<T> cfg,
                    int batch_size, bool multiplication)
{
    detail::check_range(cfg.n_power);
    detail::raise_status(detail::c2c(device_inout, root_of_unity_table, cfg, batch_size, multiplication), __FILE__,
                         __LINE__);
}

// FFT: real to COMPLEX<T>, IFFT: COMPLEX<T> to real (reference fft.cuh:126-132)
template <typename T>
inline void GPU_FFT(T* device_fix_inout, COMPLEX<T>* device_Complex64_inout, COMPLEX<T>* root_of_unity_table,
                    fft_configuration<T> cfg, int batch_size, bool multiplication)
{
    detail::check_range(cfg.n_power);
    detail::raise_status(detail::r2r(device_fix_inout, device_Complex64_inout, root_of_unity_table, cfg, batch_size,
                                     multiplication),
                         __FILE__, __LINE__);
}

// Negacyclic real transform (reference fft.cuh:269-273)
template <typename T>
inline void GPU_FFNT(T* device_inout, COMPLEX<T>* device_temp, COMPLEX<T>* twist_table,
                     COMPLEX<T>* root_of_unity_table, fft_configuration<T> cfg, int batch_size, bool multiplication)
{
    detail::check_range(cfg.n_power);
    detail::raise_status(
        detail::ffnt(device_inout, device_temp, twist_table, root_of_unity_table, cfg, batch_size, multiplication),
        __FILE__, __LINE__);
}

// Special FFT for HE encoding (reference fft.cuh:194-197; range check as
// fft.cu:933-936: n_power in [11, 24])
template <typename T>
inline void GPU_Special_FFT(COMPLEX<T>* device_inout, COMPLEX<T>* root_of_unity_table, fft_configuration<T> cfg,
                            int batch_size)
{
    if (cfg.n_power <= 10 || cfg.n_power >= 25) throw std::invalid_argument("Invalid n_power range!");
    detail::raise_status(detail::special(device_inout, root_of_unity_table, cfg, batch_size), __FILE__, __LINE__);
}

} // namespace gpufft

#endif // GPUFFT_B200_FFT_CUH
