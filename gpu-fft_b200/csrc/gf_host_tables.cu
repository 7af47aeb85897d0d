// gpufft-b200: the host table generators of the drop-in API (gpufft::FFT<T>,
// gpufft::FFNT<T> from include/gpufft/fft_cpu.cuh) exported through the C ABI,
// for callers that are not C++ (the Python mirror builds its drop-in tables
// with these).
#include "../../include/gpufft/fft_cpu.cuh"
#include "gf_common.cuh"

namespace
{
template <typename T> void put(const std::vector<COMPLEX<T>>& v, void* out)
{
    T* p = static_cast<T*>(out);
    for (size_t i = 0; i < v.size(); i++)
    {
        p[2 * i] = v[i].real();
        p[2 * i + 1] = v[i].imag();
    }
}

template <typename T> int fft_tables(int n, void* roots, void* inv_roots, void* n_inverse)
{
    if (n < 1 || (n & (n - 1)) || n > (1 << 24)) return GPUFFT_ERROR_INVALID_VALUE;
    if (!roots || !inv_roots || !n_inverse) return GPUFFT_ERROR_INVALID_VALUE;
    gpufft::FFT<T> g(n);
    put<T>(g.ReverseRootTable(), roots);
    put<T>(g.InverseReverseRootTable(), inv_roots);
    *static_cast<T*>(n_inverse) = g.n_inverse;
    return GPUFFT_SUCCESS;
}

template <typename T> int ffnt_tables(int n, void* roots, void* inv_roots, void* twist, void* untwist)
{
    if (n < 4 || (n & (n - 1)) || n > (1 << 25)) return GPUFFT_ERROR_INVALID_VALUE;
    if (!roots || !inv_roots || !twist || !untwist) return GPUFFT_ERROR_INVALID_VALUE;
    gpufft::FFNT<T> g(n);
    put<T>(g.ReverseRootTable_ffnt(), roots);
    put<T>(g.InverseReverseRootTable_ffnt(), inv_roots);
    put<T>(g.twist_table_ffnt(), twist);
    put<T>(g.untwist_table_ffnt(), untwist);
    return GPUFFT_SUCCESS;
}
} // namespace

extern "C" int gpufft_host_fft_tables_f32(int n, void* r, void* ri, void* ninv) { return fft_tables<float>(n, r, ri, ninv); }
extern "C" int gpufft_host_fft_tables_f64(int n, void* r, void* ri, void* ninv) { return fft_tables<double>(n, r, ri, ninv); }
extern "C" int gpufft_host_ffnt_tables_f32(int n, void* r, void* ri, void* t, void* u) { return ffnt_tables<float>(n, r, ri, t, u); }
extern "C" int gpufft_host_ffnt_tables_f64(int n, void* r, void* ri, void* t, void* u) { return ffnt_tables<double>(n, r, ri, t, u); }
