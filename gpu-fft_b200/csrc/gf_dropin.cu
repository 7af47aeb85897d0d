// gpufft-b200: drop-in GPU_FFT (C_C and R_R) and GPU_FFNT.
//
// Each call runs the reference's transform (same stages, same caller-supplied
// twiddle table, same fused product / scale / fold / twist semantics) as one to
// three engine passes instead of the reference's two to four launches of
// 512-element tiles:
//     m <= 12        one pass
//     12 < m <= 21   passes of (m-12, 12) stages
//     21 < m <= 24   passes of (m-21, 9, 12) stages
// where m = log2 of the transform length (n_power for GPU_FFT, n_power-1 for
// GPU_FFNT). Reference: src/lib/fft.cu:517-725 (GPU_FFT), 1386-1515 (GPU_FFNT).
#include "gf_pass.cuh"

#include <cstdio>

namespace gfb
{

template <typename T>
static int run_forward(int m, int neg, long long batch, const void* in, int in_kind, void* out,
                       const cx<T>* table, const cx<T>* twist, int zero_pad, cudaStream_t s)
{
    const Plan p = make_plan(m);
    for (int k = 0; k < p.np; k++)
    {
        long long ctas = 0;
        PassArgs<T> a{};
        a.geo = pass_geo(p, k, m, neg, batch, &ctas);
        a.table = table;
        a.twist = twist;
        a.batch = batch;
        a.in = (k == 0) ? in : out;
        a.out = out;
        a.zero_pad = (k == 0) ? zero_pad : 0;
        a.in_kind = (k == 0) ? in_kind : IN_CPX;
        a.out_kind = OUT_CPX;
        const int st = launch_pass<T, true>(a, p, k, ctas, s);
        if (st) return st;
    }
    return GPUFFT_SUCCESS;
}

// Inverse: passes run from the last (contiguous) to the first. `work` holds the
// spectra (and the product's second operand at prod_off); the final pass writes
// `out` with out_kind.
template <typename T>
static int run_inverse(int m, int neg, long long batch, void* work, int mult, long long prod_off,
                       void* out, int out_kind, const cx<T>* table, const cx<T>* untwist, cx<T> scale,
                       cudaStream_t s)
{
    const Plan p = make_plan(m);
    for (int k = p.np - 1; k >= 0; k--)
    {
        long long ctas = 0;
        PassArgs<T> a{};
        a.geo = pass_geo(p, k, m, neg, batch, &ctas);
        a.table = table;
        a.twist = untwist;
        a.batch = batch;
        a.scale = scale;
        a.prod_off = prod_off;
        a.in = work;
        const bool first = (k == p.np - 1), last = (k == 0);
        a.out = last ? out : work;
        a.do_scale = last ? 1 : 0;
        a.in_kind = (first && mult) ? IN_PROD : IN_CPX;
        a.out_kind = last ? out_kind : OUT_CPX;
        const int st = launch_pass<T, false>(a, p, k, ctas, s);
        if (st) return st;
    }
    return GPUFFT_SUCCESS;
}

template <typename T> static bool aligned(const void* p, size_t a)
{
    return (reinterpret_cast<uintptr_t>(p) % a) == 0;
}

template <typename T>
static int fft_c2c(void* inout, const void* table, int n_power, int fft_type, int red, int zero_pad,
                   T mi_re, T mi_im, int batch, int mult, cudaStream_t s)
{
    if (n_power < 1 || n_power > 24) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!inout || !table || batch <= 0 || (fft_type != GPUFFT_FORWARD && fft_type != GPUFFT_INVERSE) ||
        (red != GPUFFT_X_N_PLUS && red != GPUFFT_X_N_MINUS))
        return GPUFFT_ERROR_INVALID_VALUE;
    if (!aligned<T>(inout, sizeof(cx<T>)) || !aligned<T>(table, sizeof(cx<T>))) return GPUFFT_ERROR_MISALIGNED;
    const int neg = (red == GPUFFT_X_N_PLUS);
    const auto* tb = reinterpret_cast<const cx<T>*>(table);
    if (fft_type == GPUFFT_FORWARD)
        return run_forward<T>(n_power, neg, batch, inout, IN_CPX, inout, tb, nullptr, zero_pad, s);
    return run_inverse<T>(n_power, neg, batch, inout, mult, (long long)batch << n_power, inout, OUT_CPX, tb,
                          nullptr, mk<T>(mi_re, mi_im), s);
}

template <typename T>
static int fft_r2r(T* real_inout, void* temp, const void* table, int n_power, int fft_type, int red,
                   int zero_pad, T mi_re, T mi_im, int batch, int mult, cudaStream_t s)
{
    if (n_power < 1 || n_power > 24) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!real_inout || !temp || !table || batch <= 0 ||
        (fft_type != GPUFFT_FORWARD && fft_type != GPUFFT_INVERSE) ||
        (red != GPUFFT_X_N_PLUS && red != GPUFFT_X_N_MINUS))
        return GPUFFT_ERROR_INVALID_VALUE;
    if (!aligned<T>(real_inout, sizeof(T)) || !aligned<T>(temp, sizeof(cx<T>)) ||
        !aligned<T>(table, sizeof(cx<T>)))
        return GPUFFT_ERROR_MISALIGNED;
    const int neg = (red == GPUFFT_X_N_PLUS);
    const auto* tb = reinterpret_cast<const cx<T>*>(table);
    if (fft_type == GPUFFT_FORWARD)
        return run_forward<T>(n_power, neg, batch, real_inout, IN_REAL, temp, tb, nullptr, zero_pad, s);
    return run_inverse<T>(n_power, neg, batch, temp, mult, (long long)batch << n_power, real_inout, OUT_REAL,
                          tb, nullptr, mk<T>(mi_re, mi_im), s);
}

template <typename T>
static int ffnt(T* inout, void* temp, const void* twist, const void* table, int n_power, int fft_type,
                T mi_re, T mi_im, int batch, int mult, cudaStream_t s)
{
    if (n_power < 2 || n_power > 25) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!inout || !temp || !twist || !table || batch <= 0 ||
        (fft_type != GPUFFT_FORWARD && fft_type != GPUFFT_INVERSE))
        return GPUFFT_ERROR_INVALID_VALUE;
    if (!aligned<T>(inout, sizeof(T)) || !aligned<T>(temp, sizeof(cx<T>)) || !aligned<T>(twist, sizeof(cx<T>)) ||
        !aligned<T>(table, sizeof(cx<T>)))
        return GPUFFT_ERROR_MISALIGNED;
    const int m = n_power - 1;
    const auto* tb = reinterpret_cast<const cx<T>*>(table);
    const auto* tw = reinterpret_cast<const cx<T>*>(twist);
    if (fft_type == GPUFFT_FORWARD)
        return run_forward<T>(m, 0, batch, inout, IN_FOLD, temp, tb, tw, 0, s);
    return run_inverse<T>(m, 0, batch, temp, mult, (long long)batch << m, inout, OUT_UNFOLD, tb, tw,
                          mk<T>(mi_re, mi_im), s);
}

} // namespace gfb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int gpufft_fft_c2c_f32(void* inout, const void* root_table, int n_power, int fft_type,
                                  int reduction_poly, int zero_padding, float mre, float mim, int batch,
                                  int multiplication, gpufft_stream_t stream)
{
    return gfb::fft_c2c<float>(inout, root_table, n_power, fft_type, reduction_poly, zero_padding, mre, mim,
                               batch, multiplication, (cudaStream_t)stream);
}
extern "C" int gpufft_fft_c2c_f64(void* inout, const void* root_table, int n_power, int fft_type,
                                  int reduction_poly, int zero_padding, double mre, double mim, int batch,
                                  int multiplication, gpufft_stream_t stream)
{
    return gfb::fft_c2c<double>(inout, root_table, n_power, fft_type, reduction_poly, zero_padding, mre, mim,
                                batch, multiplication, (cudaStream_t)stream);
}
extern "C" int gpufft_fft_r2r_f32(float* real_inout, void* temp, const void* root_table, int n_power,
                                  int fft_type, int reduction_poly, int zero_padding, float mre, float mim,
                                  int batch, int multiplication, gpufft_stream_t stream)
{
    return gfb::fft_r2r<float>(real_inout, temp, root_table, n_power, fft_type, reduction_poly, zero_padding,
                               mre, mim, batch, multiplication, (cudaStream_t)stream);
}
extern "C" int gpufft_fft_r2r_f64(double* real_inout, void* temp, const void* root_table, int n_power,
                                  int fft_type, int reduction_poly, int zero_padding, double mre, double mim,
                                  int batch, int multiplication, gpufft_stream_t stream)
{
    return gfb::fft_r2r<double>(real_inout, temp, root_table, n_power, fft_type, reduction_poly, zero_padding,
                                mre, mim, batch, multiplication, (cudaStream_t)stream);
}
extern "C" int gpufft_ffnt_f32(float* inout, void* temp, const void* twist_table, const void* root_table,
                               int n_power, int fft_type, float mre, float mim, int batch, int multiplication,
                               gpufft_stream_t stream)
{
    return gfb::ffnt<float>(inout, temp, twist_table, root_table, n_power, fft_type, mre, mim, batch,
                            multiplication, (cudaStream_t)stream);
}
extern "C" int gpufft_ffnt_f64(double* inout, void* temp, const void* twist_table, const void* root_table,
                               int n_power, int fft_type, double mre, double mim, int batch, int multiplication,
                               gpufft_stream_t stream)
{
    return gfb::ffnt<double>(inout, temp, twist_table, root_table, n_power, fft_type, mre, mim, batch,
                             multiplication, (cudaStream_t)stream);
}
