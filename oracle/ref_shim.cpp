// ORACLE — test infrastructure only.
//
// A C-ABI shim over the REFERENCE's own CPU classes (gpufft::FFT<T>,
// gpufft::FFNT<T>, gpufft::schoolbook_* from fft_cpu.cu), compiled together
// with the unmodified reference sources by oracle/Makefile into
// oracle/_ref/libgpufft_ref_cpu.so. It exists so that the tests can pin the
// C restatement in oracle/oracle.c against the reference itself, so that
// tests/golden/make_golden.py can record golden vectors, and so that bench.py
// can time the reference's CPU product as the baseline.  Nothing in the
// product library links it.
#include "gpufft/fft_cpu.cuh"

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

using namespace gpufft;

namespace
{
template <typename T> void copy_out(const std::vector<COMPLEX<T>>& v, T* out)
{
    for (size_t i = 0; i < v.size(); i++)
    {
        out[2 * i] = v[i].real();
        out[2 * i + 1] = v[i].imag();
    }
}

template <typename T> void fft_tables(int n, T* rev, T* rev_inv, T* n_inverse)
{
    FFT<T> g(n);
    copy_out(g.ReverseRootTable(), rev);
    copy_out(g.InverseReverseRootTable(), rev_inv);
    *n_inverse = g.n_inverse;
}

template <typename T> void ffnt_tables(int n, T* rev, T* rev_inv, T* tw, T* utw)
{
    FFNT<T> g(n);
    copy_out(g.ReverseRootTable_ffnt(), rev);
    copy_out(g.InverseReverseRootTable_ffnt(), rev_inv);
    copy_out(g.twist_table_ffnt(), tw);
    copy_out(g.untwist_table_ffnt(), utw);
}

template <typename T> void cpu_fft(int n, T* data, int inverse)
{
    FFT<T> g(n);
    std::vector<COMPLEX<T>> v(2 * n);
    for (int i = 0; i < 2 * n; i++) v[i] = COMPLEX<T>(data[2 * i], data[2 * i + 1]);
    if (inverse)
        g.ifft(v);
    else
        g.fft(v);
    copy_out(v, data);
}

template <typename T>
void ffnt_mult(int n, const uint64_t* a, const uint64_t* b, uint64_t* out)
{
    FFNT<T> g(n);
    std::vector<unsigned long long> va(a, a + n), vb(b, b + n);
    std::vector<unsigned long long> r = g.MULT(va, vb);
    for (int i = 0; i < n; i++) out[i] = r[i];
}
} // namespace

extern "C"
{
int ref_bitreverse(int index, int n_power) { return bitreverse(index, n_power); }

void ref_fft_tables_f64(int n, double* r, double* ri, double* ninv) { fft_tables<double>(n, r, ri, ninv); }
void ref_fft_tables_f32(int n, float* r, float* ri, float* ninv) { fft_tables<float>(n, r, ri, ninv); }
void ref_ffnt_tables_f64(int n, double* r, double* ri, double* t, double* u) { ffnt_tables<double>(n, r, ri, t, u); }
void ref_ffnt_tables_f32(int n, float* r, float* ri, float* t, float* u) { ffnt_tables<float>(n, r, ri, t, u); }
void ref_cpu_fft_f64(int n, double* d, int inverse) { cpu_fft<double>(n, d, inverse); }
void ref_cpu_fft_f32(int n, float* d, int inverse) { cpu_fft<float>(n, d, inverse); }
void ref_ffnt_mult_f64(int n, const uint64_t* a, const uint64_t* b, uint64_t* o) { ffnt_mult<double>(n, a, b, o); }
void ref_ffnt_mult_f32(int n, const uint64_t* a, const uint64_t* b, uint64_t* o) { ffnt_mult<float>(n, a, b, o); }

// schoolbook_poly_multiplication<unsigned long long> (fft_cpu.cu:23-50):
// negacyclic (lo - hi) % q with unsigned wrap-around, as the reference computes it.
void ref_schoolbook_negacyclic_u64(const uint64_t* a, const uint64_t* b, uint64_t q, int n, uint64_t* out)
{
    std::vector<unsigned long long> va(a, a + n), vb(b, b + n);
    auto r = schoolbook_poly_multiplication<unsigned long long>(va, vb, q, n);
    for (int i = 0; i < n; i++) out[i] = r[i];
}

// schoolbook_poly_multiplication_without_reduction<int> (fft_cpu.cu:52-73): 2n outputs mod q.
void ref_schoolbook_linear_i32(const int32_t* a, const int32_t* b, int32_t q, int n, int32_t* out)
{
    std::vector<int> va(a, a + n), vb(b, b + n);
    auto r = schoolbook_poly_multiplication_without_reduction<int>(va, vb, q, n);
    for (int i = 0; i < 2 * n; i++) out[i] = r[i];
}

// Linear product of two length-n integer polynomials with the reference's
// FFT<double>(n) exactly as its CPU example drives it (example/test_fft_cpu.cu):
// zero-padded to 2n, fft(A), fft(B), pointwise product, ifft, round(real).
void ref_linear_product_f64(int n, const int64_t* a, const int64_t* b, int64_t* out)
{
    FFT<double> g(n);
    std::vector<COMPLEX<double>> A(2 * n), B(2 * n);
    for (int i = 0; i < n; i++)
    {
        A[i] = COMPLEX<double>((double)a[i]);
        B[i] = COMPLEX<double>((double)b[i]);
    }
    g.fft(A);
    g.fft(B);
    for (int i = 0; i < 2 * n; i++) A[i] = A[i] * B[i];
    g.ifft(A);
    for (int i = 0; i < 2 * n; i++) out[i] = (int64_t)std::llround(A[i].real());
}

// CPU baseline: FFNT<double>::MULT (fft_cpu.cu:301-432), one independent product
// per host thread, each thread owning its FFNT object; the timed region covers
// the MULT calls only (table construction excluded). Products are taken
// round-robin from the `distinct` input pairs in `a`/`b` (n coefficients each;
// `out` holds `distinct` results). Returns seconds.
double ref_bench_ffnt_mult_f64(int n, int count, int distinct, int threads, const uint64_t* a,
                               const uint64_t* b, uint64_t* out)
{
    if (threads < 1) threads = 1;
    std::vector<FFNT<double>*> gens(threads);
    for (int t = 0; t < threads; t++) gens[t] = new FFNT<double>(n);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
    {
        pool.emplace_back(
            [&, t]()
            {
                for (int p = t; p < count; p += threads)
                {
                    const size_t q = (size_t)(p % distinct);
                    std::vector<unsigned long long> va(a + q * n, a + (q + 1) * n);
                    std::vector<unsigned long long> vb(b + q * n, b + (q + 1) * n);
                    auto r = gens[t]->MULT(va, vb);
                    std::memcpy(out + q * n, r.data(), sizeof(uint64_t) * n);
                }
            });
    }
    for (auto& th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    for (int t = 0; t < threads; t++) delete gens[t];
    return std::chrono::duration<double>(t1 - t0).count();
}
}
