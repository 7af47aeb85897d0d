// gpufft-b200 drop-in header: the COMPLEX<T> value type.
//
// Same names, layout and operator set as the reference's
// src/include/gpufft/complex.cuh (COMPLEX<T> = complex_arithmetic::
// ComplexOperations<T> holding one float2/double2, Complex32/64, Float32/64,
// fp2<T>, Float<T>), so that code written against the reference compiles
// unchanged. The layout (real then imaginary, 8 or 16 bytes) is part of the
// device ABI: buffers of COMPLEX<T> are passed straight to the kernels.
//
// Two reference behaviours are kept because callers can observe them:
//  * COMPLEX<T> * scalar returns (re*s, re*s) (reference complex.cuh:153-159);
//    FFT<T>::ifft's final scaling goes through it.
//  * complex division computes ((ac+bd)/(c^2+d^2), (bc-ad)/(c^2+d^2)), which
//    the table generators use for inverse roots.
#ifndef GPUFFT_B200_COMPLEX_CUH
#define GPUFFT_B200_COMPLEX_CUH

#include <cmath>
#include <complex>
#include <iostream>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#if defined(__CUDACC__)
#define GPUFFT_HD __host__ __device__ __forceinline__
#else
#define GPUFFT_HD inline
#endif

template <typename T>
using fp2 = typename std::conditional<std::is_same<T, float>::value, float2, double2>::type;

typedef float Float32;
typedef double Float64;

template <typename T>
using Float = typename std::conditional<std::is_same<T, float>::value, Float32, Float64>::type;

namespace complex_arithmetic
{
template <typename T1> struct ComplexOperations
{
    fp2<T1> data;

    GPUFFT_HD T1& real() { return data.x; }
    GPUFFT_HD T1& imag() { return data.y; }
    GPUFFT_HD const T1& real() const { return data.x; }
    GPUFFT_HD const T1& imag() const { return data.y; }

    GPUFFT_HD ComplexOperations() { data.x = T1(0); data.y = T1(0); }
    template <typename T2> GPUFFT_HD ComplexOperations(T2 r, T2 i)
    {
        data.x = static_cast<T1>(r);
        data.y = static_cast<T1>(i);
    }
    template <typename T2> GPUFFT_HD ComplexOperations(T2 r)
    {
        data.x = static_cast<T1>(r);
        data.y = T1(0);
    }

    GPUFFT_HD ComplexOperations operator+(const ComplexOperations& o) const
    {
        return ComplexOperations(data.x + o.data.x, data.y + o.data.y);
    }
    GPUFFT_HD ComplexOperations operator-(const ComplexOperations& o) const
    {
        return ComplexOperations(data.x - o.data.x, data.y - o.data.y);
    }
    GPUFFT_HD ComplexOperations operator*(const ComplexOperations& o) const
    {
        return ComplexOperations(data.x * o.data.x - data.y * o.data.y, data.x * o.data.y + data.y * o.data.x);
    }
    GPUFFT_HD ComplexOperations operator/(const ComplexOperations& o) const
    {
        const T1 den = o.data.x * o.data.x + o.data.y * o.data.y;
        return ComplexOperations((data.x * o.data.x + data.y * o.data.y) / den,
                                 (data.y * o.data.x - data.x * o.data.y) / den);
    }
    template <typename T2> GPUFFT_HD ComplexOperations operator+(const T2& s) const
    {
        return ComplexOperations(data.x + static_cast<T1>(s), data.y);
    }
    template <typename T2> GPUFFT_HD ComplexOperations operator-(const T2& s) const
    {
        return ComplexOperations(data.x - static_cast<T1>(s), data.y);
    }
    // Kept as the reference defines it: both components are re * s.
    template <typename T2> GPUFFT_HD ComplexOperations operator*(const T2& s) const
    {
        return ComplexOperations(data.x * static_cast<T1>(s), data.x * static_cast<T1>(s));
    }
    template <typename T2> GPUFFT_HD ComplexOperations operator/(const T2& s) const
    {
        return ComplexOperations(data.x / static_cast<T1>(s), data.y / static_cast<T1>(s));
    }

    GPUFFT_HD ComplexOperations& operator+=(const ComplexOperations& o)
    {
        data.x += o.data.x;
        data.y += o.data.y;
        return *this;
    }
    GPUFFT_HD ComplexOperations& operator-=(const ComplexOperations& o)
    {
        data.x -= o.data.x;
        data.y -= o.data.y;
        return *this;
    }
    GPUFFT_HD ComplexOperations& operator*=(const ComplexOperations& o)
    {
        *this = *this * o;
        return *this;
    }
    GPUFFT_HD ComplexOperations& operator/=(const ComplexOperations& o)
    {
        *this = *this / o;
        return *this;
    }

    GPUFFT_HD ComplexOperations conjugate() const { return ComplexOperations(data.x, -data.y); }
    GPUFFT_HD ComplexOperations negate() const { return ComplexOperations(-data.x, -data.y); }
    GPUFFT_HD T1 square() const { return data.x * data.x + data.y * data.y; }
    GPUFFT_HD ComplexOperations inverse() const
    {
        const T1 s = square();
        return ComplexOperations(data.x / s, -data.y / s);
    }
    // Integer power by binary exponentiation.
    template <typename I> GPUFFT_HD ComplexOperations exp(I& exponent) const
    {
        ComplexOperations result(T1(1), T1(0));
        ComplexOperations base = *this;
        unsigned long long e = static_cast<unsigned long long>(exponent);
        // most-significant bit first, as a square-and-multiply chain
        int top = -1;
        for (int i = 63; i >= 0; i--)
            if ((e >> i) & 1ull)
            {
                top = i;
                break;
            }
        for (int i = top; i >= 0; i--)
        {
            result = result * result;
            if ((e >> i) & 1ull) result = result * base;
        }
        return result;
    }

    friend std::ostream& operator<<(std::ostream& out, const ComplexOperations& c)
    {
        out << c.data.x;
        if (c.data.y >= 0)
            out << " + " << c.data.y << "i";
        else
            out << " - " << -c.data.y << "i";
        return out;
    }
};

// e^{z} for a complex z (host), evaluated as exp(re) * (cos(im), sin(im)) in T.
template <typename T> ComplexOperations<T> exp(const ComplexOperations<T>& z)
{
    const T e = std::exp(z.real());
    return ComplexOperations<T>(e * std::cos(z.imag()), e * std::sin(z.imag()));
}
} // namespace complex_arithmetic

template <typename T> using COMPLEX = complex_arithmetic::ComplexOperations<T>;
typedef COMPLEX<Float32> Complex32;
typedef COMPLEX<Float64> Complex64;

static_assert(sizeof(Complex32) == 8 && sizeof(Complex64) == 16, "COMPLEX<T> must match float2/double2");

#endif // GPUFFT_B200_COMPLEX_CUH
