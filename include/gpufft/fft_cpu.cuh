// gpufft-b200 drop-in header: host-side table generators and CPU transforms.
//
// Same public surface as the reference's src/include/gpufft/fft_cpu.cuh:
// bitreverse, ReductionPolynomial, schoolbook_poly_multiplication[_without_
// reduction], FFT<T> and FFNT<T> with the same members and methods. Callers use
// these classes to build the twiddle tables they pass to GPU_FFT / GPU_FFNT, so
// the tables must hold the reference's values bit for bit: every entry is
// computed with the same T-precision steps as reference fft_cpu.cu:93-128 and
// 234-300 (angle products and complex division in T, std::cos/std::sin of T).
// The library's tests compare these tables with the reference's own build.
#ifndef GPUFFT_B200_FFT_CPU_CUH
#define GPUFFT_B200_FFT_CPU_CUH

#include <cmath>
#include <vector>

#include "complex.cuh"

namespace gpufft
{
// X_N_minus: X^n - 1 (cyclic), X_N_plus: X^n + 1 (negacyclic)
enum ReductionPolynomial
{
    X_N_plus,
    X_N_minus
};

inline int bitreverse(int index, int n_power)
{
    int r = 0;
    for (int i = 0; i < n_power; i++, index >>= 1) r = (r << 1) | (index & 1);
    return r;
}

// Negacyclic schoolbook product: entries [0, size) hold (lo - hi) % modulus,
// entries [size, 2*size) the unreduced upper half, as the reference returns.
template <typename T>
std::vector<T> schoolbook_poly_multiplication(std::vector<T> a, std::vector<T> b, T modulus, int size)
{
    std::vector<T> r(2 * size, T(0));
    for (int i = 0; i < size; i++)
        for (int j = 0; j < size; j++) r[i + j] += a[i] * b[j];
    for (int i = 0; i < size; i++) r[i] = (r[i] - r[i + size]) % modulus;
    return r;
}

// Linear schoolbook product of length 2*size, every entry reduced % modulus.
template <typename T>
std::vector<T> schoolbook_poly_multiplication_without_reduction(std::vector<T> a, std::vector<T> b, T modulus,
                                                                int size)
{
    std::vector<T> r(2 * size, T(0));
    for (int i = 0; i < size; i++)
        for (int j = 0; j < size; j++) r[i + j] += a[i] * b[j];
    for (auto& v : r) v = v % modulus;
    return r;
}

namespace detail
{
// e^{i * k * theta} as the reference forms it: (0,1) * (k,0) * (theta,0) in
// COMPLEX<T> arithmetic, then complex_arithmetic::exp.
template <typename T> COMPLEX<T> unit_root(int k, const COMPLEX<T>& theta)
{
    const COMPLEX<T> j(T(0), T(1));
    return complex_arithmetic::exp(j * COMPLEX<T>(k) * theta);
}
} // namespace detail

// Radix-2 transform of length 2*size over +sign roots of unity; the forward
// output is in bit-reversed order, ifft takes bit-reversed input.
template <typename T> class FFT
{
  public:
    int n;
    int logn;
    COMPLEX<T> x;
    int max_size;

    COMPLEX<T> root;
    std::vector<COMPLEX<T>> root_tables;
    std::vector<COMPLEX<T>> inverse_root_tables;

    Float<T> n_inverse;

    explicit FFT(int size) : n(size), logn(int(std::log2(size))), x(1.0, 0.0), max_size(2 * size)
    {
        root = COMPLEX<T>(2.0) * COMPLEX<T>(M_PI) / COMPLEX<T>(max_size);
        n_inverse = 1.0 / max_size;
        root_tables.reserve(n);
        inverse_root_tables.reserve(n);
        for (int i = 0; i < n; i++) root_tables.push_back(detail::unit_root<T>(i, root));
        const COMPLEX<T> one(1.0);
        for (int i = 0; i < n; i++) inverse_root_tables.push_back(one / root_tables[i]);
    }

    void fft(std::vector<COMPLEX<T>>& v)
    {
        for (int m = 1, t = max_size >> 1; m < max_size; m <<= 1, t >>= 1)
            for (int g = 0; g < m; g++)
            {
                const COMPLEX<T> w = root_tables[bitreverse(g, logn)];
                for (int j = 2 * g * t; j < 2 * g * t + t; j++)
                {
                    const COMPLEX<T> u = v[j];
                    const COMPLEX<T> vw = v[j + t] * w;
                    v[j] = u + vw;
                    v[j + t] = u - vw;
                }
            }
    }

    void ifft(std::vector<COMPLEX<T>>& v)
    {
        for (int m = max_size, t = 1; m > 1; m >>= 1, t <<= 1)
            for (int g = 0; g < (m >> 1); g++)
            {
                const COMPLEX<T> w = inverse_root_tables[bitreverse(g, logn)];
                for (int j = 2 * g * t; j < 2 * g * t + t; j++)
                {
                    const COMPLEX<T> u = v[j];
                    const COMPLEX<T> d = v[j + t];
                    v[j] = u + d;
                    v[j + t] = (u - d) * w;
                }
            }
        for (auto& e : v) e = e * n_inverse; // scalar product: (re*s, re*s), as the reference
    }

    std::vector<COMPLEX<T>> ReverseRootTable()
    {
        std::vector<COMPLEX<T>> r;
        const int lg = int(std::log2(n));
        for (int i = 0; i < n; i++) r.push_back(root_tables[bitreverse(i, lg)]);
        return r;
    }

    std::vector<COMPLEX<T>> InverseReverseRootTable()
    {
        std::vector<COMPLEX<T>> r;
        const int lg = int(std::log2(n));
        for (int i = 0; i < n; i++) r.push_back(inverse_root_tables[bitreverse(i, lg)]);
        return r;
    }
};

// Negacyclic product of real polynomials of length n through a length-n/2
// complex transform (fold, twist, transform, product, inverse, untwist).
template <typename T> class FFNT
{
  public:
    int n;
    int logn;
    COMPLEX<T> x;
    int max_size;

    COMPLEX<T> root;
    std::vector<COMPLEX<T>> root_tables_new;
    std::vector<COMPLEX<T>> inverse_root_tables_new;

    std::vector<COMPLEX<T>> root_tables_twist;
    std::vector<COMPLEX<T>> inverse_root_tables_twist;

    T n_inverse;

    explicit FFNT(int size) : n(size), logn(int(std::log2(size))), x(1.0, 0.0), max_size(2 * size)
    {
        root = 2.0 * M_PI / static_cast<T>(max_size);
        n_inverse = 1.0 / max_size;
        const int h = n >> 1;
        const T step = 2.0 * M_PI / static_cast<T>(h);
        const T step_tw = 2.0 * M_PI / static_cast<T>(2 * n);
        const COMPLEX<T> one(1.0);
        for (int i = 0; i < h; i++) root_tables_new.push_back(detail::unit_root<T>(i, COMPLEX<T>(step)));
        for (int i = 0; i < h; i++) inverse_root_tables_new.push_back(one / root_tables_new[i]);
        for (int i = 0; i < h; i++) root_tables_twist.push_back(detail::unit_root<T>(i, COMPLEX<T>(step_tw)));
        for (int i = 0; i < h; i++) inverse_root_tables_twist.push_back(one / root_tables_twist[i]);
    }

    std::vector<unsigned long long> MULT(std::vector<unsigned long long>& input1,
                                         std::vector<unsigned long long>& input2)
    {
        const int h = n >> 1;
        const int lg = int(std::log2(h)) - 1;
        std::vector<COMPLEX<T>> A(h), B(h);
        for (int i = 0; i < h; i++)
        {
            A[i] = COMPLEX<T>(input1[i], input1[i + h]) * root_tables_twist[i];
            B[i] = COMPLEX<T>(input2[i], input2[i + h]) * root_tables_twist[i];
        }
        for (std::vector<COMPLEX<T>>* v : {&A, &B})
            for (int m = 1, t = h >> 1; m < h; m <<= 1, t >>= 1)
                for (int g = 0; g < m; g++)
                {
                    const COMPLEX<T> w = root_tables_new[bitreverse(g, lg)];
                    for (int j = 2 * g * t; j < 2 * g * t + t; j++)
                    {
                        const COMPLEX<T> u = (*v)[j];
                        const COMPLEX<T> vw = (*v)[j + t] * w;
                        (*v)[j] = u + vw;
                        (*v)[j + t] = u - vw;
                    }
                }
        for (int i = 0; i < h; i++) A[i] = A[i] * B[i];
        for (int m = h, t = 1; m > 1; m >>= 1, t <<= 1)
            for (int g = 0; g < (m >> 1); g++)
            {
                const COMPLEX<T> w = inverse_root_tables_new[bitreverse(g, lg)];
                for (int j = 2 * g * t; j < 2 * g * t + t; j++)
                {
                    const COMPLEX<T> u = A[j];
                    const COMPLEX<T> d = A[j + t];
                    A[j] = u + d;
                    A[j + t] = (u - d) * w;
                }
            }
        const T scale = 1.0 / h;
        std::vector<unsigned long long> out(n);
        for (int i = 0; i < h; i++)
        {
            const COMPLEX<T> v = (A[i] * inverse_root_tables_twist[i]) * COMPLEX<T>(scale);
            out[i] = static_cast<unsigned long long>(static_cast<long long>(std::llround(v.real())));
            out[i + h] = static_cast<unsigned long long>(static_cast<long long>(std::llround(v.imag())));
        }
        return out;
    }

    std::vector<COMPLEX<T>> ReverseRootTable_ffnt()
    {
        std::vector<COMPLEX<T>> r;
        const int lg = int(std::log2(n >> 1)) - 1;
        for (int i = 0; i < (n >> 1); i++) r.push_back(root_tables_new[bitreverse(i, lg)]);
        return r;
    }
    std::vector<COMPLEX<T>> InverseReverseRootTable_ffnt()
    {
        std::vector<COMPLEX<T>> r;
        const int lg = int(std::log2(n >> 1)) - 1;
        for (int i = 0; i < (n >> 1); i++) r.push_back(inverse_root_tables_new[bitreverse(i, lg)]);
        return r;
    }
    std::vector<COMPLEX<T>> twist_table_ffnt() { return root_tables_twist; }
    std::vector<COMPLEX<T>> untwist_table_ffnt() { return inverse_root_tables_twist; }
};

} // namespace gpufft

#endif // GPUFFT_B200_FFT_CPU_CUH
