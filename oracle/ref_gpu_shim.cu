// ORACLE — test infrastructure only.
//
// A C-ABI shim over the REFERENCE's own GPU entry points (gpufft::GPU_FFT,
// gpufft::GPU_FFNT from src/lib/fft.cu), compiled with the unmodified
// reference sources for sm_100a by oracle/Makefile into
// oracle/_ref/libgpufft_ref_gpu.so. Tests use it to compare the library's
// drop-in outputs with the reference's own GPU outputs on the same inputs and
// tables, and a timing script uses it to time the reference's GPU path on the
// same GPU. Errors the reference throws are returned as status codes.
#include "gpufft/fft.cuh"

#include <stdexcept>

using namespace gpufft;

namespace
{
template <typename F> int guarded(F&& f)
{
    try
    {
        f();
        return 0;
    }
    catch (const std::invalid_argument&)
    {
        return 1;
    }
    catch (const CudaException&)
    {
        return 3;
    }
    catch (...)
    {
        return 2;
    }
}
} // namespace

extern "C"
{
int ref_gpu_ffnt_f64(double* inout, void* temp, void* twist, void* roots, int n_power, int fft_type, double mi_re,
                     double mi_im, int batch, int mult, void* stream)
{
    fft_configuration<double> cfg{};
    cfg.n_power = n_power;
    cfg.fft_type = fft_type ? INVERSE : FORWARD;
    cfg.zero_padding = false;
    cfg.mod_inverse = COMPLEX<double>(mi_re, mi_im);
    cfg.stream = (cudaStream_t)stream;
    return guarded([&] {
        GPU_FFNT(inout, (COMPLEX<double>*)temp, (COMPLEX<double>*)twist, (COMPLEX<double>*)roots, cfg, batch,
                 mult != 0);
    });
}

int ref_gpu_ffnt_f32(float* inout, void* temp, void* twist, void* roots, int n_power, int fft_type, float mi_re,
                     float mi_im, int batch, int mult, void* stream)
{
    fft_configuration<float> cfg{};
    cfg.n_power = n_power;
    cfg.fft_type = fft_type ? INVERSE : FORWARD;
    cfg.zero_padding = false;
    cfg.mod_inverse = COMPLEX<float>(mi_re, mi_im);
    cfg.stream = (cudaStream_t)stream;
    return guarded([&] {
        GPU_FFNT(inout, (COMPLEX<float>*)temp, (COMPLEX<float>*)twist, (COMPLEX<float>*)roots, cfg, batch,
                 mult != 0);
    });
}

int ref_gpu_fft_c2c_f64(void* inout, void* roots, int n_power, int fft_type, int red, double mi_re, double mi_im,
                        int batch, int mult, void* stream)
{
    fft_configuration<double> cfg{};
    cfg.n_power = n_power;
    cfg.fft_type = fft_type ? INVERSE : FORWARD;
    cfg.reduction_poly = red ? X_N_minus : X_N_plus;
    cfg.zero_padding = false;
    cfg.mod_inverse = COMPLEX<double>(mi_re, mi_im);
    cfg.stream = (cudaStream_t)stream;
    return guarded([&] {
        GPU_FFT((COMPLEX<double>*)inout, (COMPLEX<double>*)roots, cfg, batch, mult != 0);
    });
}

int ref_gpu_special_fft_f64(void* inout, void* table, int n_power, int fft_type, double mi_re, double mi_im,
                            int batch, void* stream)
{
    fft_configuration<double> cfg{};
    cfg.n_power = n_power;
    cfg.fft_type = fft_type ? INVERSE : FORWARD;
    cfg.mod_inverse = COMPLEX<double>(mi_re, mi_im);
    cfg.stream = (cudaStream_t)stream;
    return guarded([&] { GPU_Special_FFT((COMPLEX<double>*)inout, (COMPLEX<double>*)table, cfg, batch); });
}

int ref_gpu_special_fft_f32(void* inout, void* table, int n_power, int fft_type, float mi_re, float mi_im, int batch,
                            void* stream)
{
    fft_configuration<float> cfg{};
    cfg.n_power = n_power;
    cfg.fft_type = fft_type ? INVERSE : FORWARD;
    cfg.mod_inverse = COMPLEX<float>(mi_re, mi_im);
    cfg.stream = (cudaStream_t)stream;
    return guarded([&] { GPU_Special_FFT((COMPLEX<float>*)inout, (COMPLEX<float>*)table, cfg, batch); });
}

int ref_gpu_fft_r2r_f64(double* real_inout, void* temp, void* roots, int n_power, int fft_type, int red,
                        double mi_re, double mi_im, int batch, int mult, void* stream)
{
    fft_configuration<double> cfg{};
    cfg.n_power = n_power;
    cfg.fft_type = fft_type ? INVERSE : FORWARD;
    cfg.reduction_poly = red ? X_N_minus : X_N_plus;
    cfg.zero_padding = false;
    cfg.mod_inverse = COMPLEX<double>(mi_re, mi_im);
    cfg.stream = (cudaStream_t)stream;
    return guarded([&] {
        GPU_FFT(real_inout, (COMPLEX<double>*)temp, (COMPLEX<double>*)roots, cfg, batch, mult != 0);
    });
}
}
