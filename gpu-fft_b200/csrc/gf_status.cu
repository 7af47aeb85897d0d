// gpufft-b200: status codes and CUDA error capture for the C ABI.
//
// The reference reports launch failures by throwing CudaException from
// GPUFFT_CUDA_CHECK(cudaGetLastError()) after every launch
// (common_fft.cuh:41-49, e.g. fft.cu:555). Across a C ABI there are no
// exceptions, so the failing cudaError_t is kept per host thread and the
// entry point returns GPUFFT_ERROR_CUDA; the C++ drop-in rethrows it.
#include "gf_common.cuh"

namespace
{
thread_local int g_last_cuda_error = 0;
}

namespace gfb
{
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
