// gpufft-b200 drop-in header: error handling.
//
// Same names and behaviour as the reference's src/include/gpufft/common_fft.cuh:
// gpufft::CudaException(file, line, cudaError_t) with what() =
// "CUDA Error in <file> at line <line>: <cudaGetErrorString>", the
// GPUFFT_CUDA_CHECK(err) macro that throws it, and customAssert.
#ifndef GPUFFT_B200_COMMON_FFT_CUH
#define GPUFFT_B200_COMMON_FFT_CUH

#include <cuda_runtime.h>

#include <cassert>
#include <exception>
#include <iostream>
#include <string>

namespace gpufft
{
class CudaException : public std::exception
{
  public:
    CudaException(const std::string& file, int line, cudaError_t error)
        : file_(file), line_(line), error_(error),
          message_("CUDA Error in " + file + " at line " + std::to_string(line) + ": " +
                   cudaGetErrorString(error))
    {
    }
    const char* what() const noexcept override { return message_.c_str(); }
    cudaError_t error() const noexcept { return error_; }

  private:
    std::string file_;
    int line_;
    cudaError_t error_;
    std::string message_;
};

#define GPUFFT_CUDA_CHECK(err)                                                                   \
    do                                                                                           \
    {                                                                                            \
        cudaError_t gpufft_check_error_ = (err);                                                 \
        if (gpufft_check_error_ != cudaSuccess)                                                  \
            throw ::gpufft::CudaException(__FILE__, __LINE__, gpufft_check_error_);              \
    } while (0)

inline void customAssert(bool condition, const std::string& errorMessage)
{
    if (!condition)
    {
        std::cerr << "Custom assertion failed: " << errorMessage << std::endl;
        assert(condition);
    }
}
} // namespace gpufft

#endif // GPUFFT_B200_COMMON_FFT_CUH
