/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C restatement of GPU-FFT's polynomial-multiplication path, used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * Nothing in the product library links or calls this file.
 *
 * Parity pins: tests/test_oracle.py checks every function here against
 *   (1) the reference's own CPU classes compiled from source into oracle/_ref
 *       (bit-for-bit on float outputs: the op order below follows the reference),
 *   (2) the committed golden vectors in tests/golden/ (made by that build),
 *   (3) the exact __int128 schoolbook products below.
 *
 * Complex values are interleaved (re, im) pairs of T, the layout of the
 * reference's COMPLEX<T> (complex.cuh:28-34, a float2/double2 wrapper).
 * Every arithmetic helper uses the reference's formulas in the same order
 * (complex.cuh:65-69 add, 99-104 sub, 133-139 mul, 142-150 div) so that the
 * results round the same way on a compiler that does not contract to FMA
 * (this file is built with -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------- */
/* bit reversal: fft_cpu.cu:11-21                                             */
/* ------------------------------------------------------------------------- */
int orc_bitreverse(int index, int n_power)
{
    int r = 0;
    for (int i = 0; i < n_power; i++) {
        r = (r << 1) | (index & 1);
        index >>= 1;
    }
    return r;
}

/* ------------------------------------------------------------------------- */
/* Type-generic body, instantiated for double (f64) and float (f32).          */
/* ------------------------------------------------------------------------- */
#define ORC_DEFINE(T, SFX, COS, SIN, EXP)                                                     \
    typedef struct { T re, im; } cx_##SFX;                                                    \
    static inline cx_##SFX cmk_##SFX(T r, T i) { cx_##SFX c; c.re = r; c.im = i; return c; }  \
    static inline cx_##SFX cadd_##SFX(cx_##SFX a, cx_##SFX b)                                 \
    { return cmk_##SFX(a.re + b.re, a.im + b.im); }                                           \
    static inline cx_##SFX csub_##SFX(cx_##SFX a, cx_##SFX b)                                 \
    { return cmk_##SFX(a.re - b.re, a.im - b.im); }                                           \
    static inline cx_##SFX cmul_##SFX(cx_##SFX a, cx_##SFX b)                                 \
    { return cmk_##SFX(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }               \
    static inline cx_##SFX cdiv_##SFX(cx_##SFX a, cx_##SFX b)                                 \
    {                                                                                         \
        T den = b.re * b.re + b.im * b.im;                                                    \
        return cmk_##SFX((a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den);\
    }                                                                                         \
    /* complex exp of (0 + i*theta) as the reference computes it (complex.cuh:307-312) */    \
    static inline cx_##SFX cexpi_##SFX(cx_##SFX z)                                            \
    {                                                                                         \
        T e = EXP(z.re);                                                                      \
        return cmk_##SFX(e * COS(z.im), e * SIN(z.im));                                       \
    }                                                                                         \
    static inline cx_##SFX ld_##SFX(const T* p, long i) { return cmk_##SFX(p[2 * i], p[2 * i + 1]); } \
    static inline void st_##SFX(T* p, long i, cx_##SFX v) { p[2 * i] = v.re; p[2 * i + 1] = v.im; }   \
                                                                                              \
    /* FFT<T>(n) tables: fft_cpu.cu:93-128 (roots), 200-226 (bit-reversed copies).   */       \
    /* n = polynomial size; the transform length is 2n; each table has n entries.   */       \
    void orc_fft_tables_##SFX(int n, T* rev_roots, T* rev_inv_roots, T* n_inverse)           \
    {                                                                                         \
        int max_size = 2 * n;                                                                 \
        int lg = (int)log2((double)n);                                                        \
        /* root = COMPLEX(2.0) * COMPLEX(pi) / COMPLEX(max_size), complex ops (fft_cpu.cu:100-101) */ \
        cx_##SFX root = cdiv_##SFX(cmul_##SFX(cmk_##SFX((T)2.0, (T)0), cmk_##SFX((T)M_PI, (T)0)), \
                                   cmk_##SFX((T)max_size, (T)0));                             \
        cx_##SFX j = cmk_##SFX((T)0.0, (T)1.0);                                               \
        cx_##SFX* roots = (cx_##SFX*)malloc(sizeof(cx_##SFX) * n);                            \
        cx_##SFX* inv = (cx_##SFX*)malloc(sizeof(cx_##SFX) * n);                              \
        for (int i = 0; i < n; i++) {                                                         \
            roots[i] = cexpi_##SFX(cmul_##SFX(cmul_##SFX(j, cmk_##SFX((T)i, (T)0)), root));   \
            inv[i] = cdiv_##SFX(cmk_##SFX((T)1.0, (T)0), roots[i]);                           \
        }                                                                                     \
        for (int i = 0; i < n; i++) {                                                         \
            int r = orc_bitreverse(i, lg);                                                    \
            st_##SFX(rev_roots, i, roots[r]);                                                 \
            st_##SFX(rev_inv_roots, i, inv[r]);                                               \
        }                                                                                     \
        *n_inverse = (T)(1.0 / max_size);                                                     \
        free(roots);                                                                          \
        free(inv);                                                                            \
    }                                                                                         \
                                                                                              \
    /* FFNT<T>(n) tables: fft_cpu.cu:234-300 and 435-473.                            */      \
    /* rev_roots / rev_inv_roots: n/2 entries, twist / untwist: n/2 entries.         */      \
    void orc_ffnt_tables_##SFX(int n, T* rev_roots, T* rev_inv_roots, T* twist, T* untwist)  \
    {                                                                                         \
        int h = n >> 1;                                                                       \
        int logn_new = (int)log2((double)h);                                                  \
        cx_##SFX j = cmk_##SFX((T)0.0, (T)1.0);                                               \
        T root_new = (T)(2.0 * M_PI / (T)h);                                                  \
        T root_tw = (T)(2.0 * M_PI / (T)(2 * n));                                             \
        cx_##SFX* r = (cx_##SFX*)malloc(sizeof(cx_##SFX) * h);                                \
        cx_##SFX* ri = (cx_##SFX*)malloc(sizeof(cx_##SFX) * h);                               \
        for (int i = 0; i < h; i++) {                                                         \
            r[i] = cexpi_##SFX(cmul_##SFX(cmul_##SFX(j, cmk_##SFX((T)i, (T)0)), cmk_##SFX(root_new, (T)0))); \
            ri[i] = cdiv_##SFX(cmk_##SFX((T)1.0, (T)0), r[i]);                                \
            cx_##SFX tw = cexpi_##SFX(cmul_##SFX(cmul_##SFX(j, cmk_##SFX((T)i, (T)0)), cmk_##SFX(root_tw, (T)0))); \
            st_##SFX(twist, i, tw);                                                           \
            st_##SFX(untwist, i, cdiv_##SFX(cmk_##SFX((T)1.0, (T)0), tw));                    \
        }                                                                                     \
        for (int i = 0; i < h; i++) {                                                         \
            int b = orc_bitreverse(i, logn_new - 1);                                          \
            st_##SFX(rev_roots, i, r[b]);                                                     \
            st_##SFX(rev_inv_roots, i, ri[b]);                                                \
        }                                                                                     \
        free(r);                                                                              \
        free(ri);                                                                             \
    }                                                                                         \
                                                                                              \
    /* Forward transform of one length-2^m vector, natural order in, bit-reversed out. */    \
    /* Radix-2 Cooley-Tukey stages with a bit-reversed twiddle table, as ForwardCore    */   \
    /* (fft.cu:11-152) and FFT<T>::fft (fft_cpu.cu:131-161) compute them. negacyclic=1  */   \
    /* selects the X^N+1 twiddle index m + g (fft.cu:67-74).                             */   \
    static void fwd_stages_##SFX(cx_##SFX* x, int m, const T* table, int negacyclic)          \
    {                                                                                         \
        long M = 1L << m;                                                                     \
        for (int s = 0; s < m; s++) {                                                         \
            long t = M >> (s + 1);                                                            \
            long groups = 1L << s;                                                            \
            for (long g = 0; g < groups; g++) {                                               \
                cx_##SFX w = ld_##SFX(table, negacyclic ? groups + g : g);                    \
                for (long k = 0; k < t; k++) {                                                \
                    long i0 = 2 * g * t + k;                                                  \
                    cx_##SFX u = x[i0];                                                       \
                    cx_##SFX v = cmul_##SFX(x[i0 + t], w);                                    \
                    x[i0] = cadd_##SFX(u, v);                                                 \
                    x[i0 + t] = csub_##SFX(u, v);                                             \
                }                                                                             \
            }                                                                                 \
        }                                                                                     \
    }                                                                                         \
    /* Inverse transform stages, bit-reversed in, natural out, no scaling:             */    \
    /* Gentleman-Sande butterflies as InverseCore (fft.cu:154-260), FFT<T>::ifft        */   \
    /* (fft_cpu.cu:163-198).                                                            */   \
    static void inv_stages_##SFX(cx_##SFX* x, int m, const T* table, int negacyclic)          \
    {                                                                                         \
        long M = 1L << m;                                                                     \
        for (int s = m - 1; s >= 0; s--) {                                                    \
            long t = M >> (s + 1);                                                            \
            long groups = 1L << s;                                                            \
            for (long g = 0; g < groups; g++) {                                               \
                cx_##SFX w = ld_##SFX(table, negacyclic ? groups + g : g);                    \
                for (long k = 0; k < t; k++) {                                                \
                    long i0 = 2 * g * t + k;                                                  \
                    cx_##SFX u = x[i0];                                                       \
                    cx_##SFX v = x[i0 + t];                                                   \
                    x[i0] = cadd_##SFX(u, v);                                                 \
                    x[i0 + t] = cmul_##SFX(csub_##SFX(u, v), w);                              \
                }                                                                             \
            }                                                                                 \
        }                                                                                     \
    }                                                                                         \
                                                                                              \
    /* GPU_FFT, COMPLEX<T>* overload (fft.cu:517-598). inout holds batch vectors of   */     \
    /* 2^n_power complex; for the inverse with multiplication the second operand sits */     \
    /* batch*2^n_power entries later (fft.cu:194-205, 568). fft_type 0 = FORWARD.      */     \
    /* reduction_poly: 0 = X_N_plus, 1 = X_N_minus (fft_cpu.cuh:69-73).                */     \
    void orc_gpu_fft_c2c_##SFX(T* inout, const T* table, int n_power, int fft_type,           \
                               int reduction_poly, const T* mod_inverse, int batch, int mult) \
    {                                                                                         \
        long M = 1L << n_power;                                                               \
        int neg = (reduction_poly == 0);                                                      \
        cx_##SFX* x = (cx_##SFX*)malloc(sizeof(cx_##SFX) * M);                                \
        cx_##SFX sc = cmk_##SFX(mod_inverse[0], mod_inverse[1]);                              \
        for (int b = 0; b < batch; b++) {                                                     \
            T* p = inout + 2 * (long)b * M;                                                   \
            if (fft_type == 0) {                                                              \
                for (long i = 0; i < M; i++) x[i] = ld_##SFX(p, i);                           \
                fwd_stages_##SFX(x, n_power, table, neg);                                     \
            } else {                                                                          \
                const T* q = p + 2 * (long)batch * M;                                         \
                for (long i = 0; i < M; i++)                                                  \
                    x[i] = mult ? cmul_##SFX(ld_##SFX(p, i), ld_##SFX(q, i)) : ld_##SFX(p, i);\
                inv_stages_##SFX(x, n_power, table, neg);                                     \
                for (long i = 0; i < M; i++) x[i] = cmul_##SFX(x[i], sc);                     \
            }                                                                                 \
            for (long i = 0; i < M; i++) st_##SFX(p, i, x[i]);                                \
        }                                                                                     \
        free(x);                                                                              \
    }                                                                                         \
                                                                                              \
    /* GPU_FFT, real overload (fft.cu:600-725): the forward promotes each real to a   */     \
    /* complex with zero imaginary part (fft.cu:303-305) and writes temp; the inverse */     \
    /* reads temp (product fused) and writes .real() of the scaled result            */      \
    /* (fft.cu:499-514) into real_inout.                                              */     \
    void orc_gpu_fft_r2r_##SFX(T* real_inout, T* temp, const T* table, int n_power,           \
                               int fft_type, int reduction_poly, const T* mod_inverse,        \
                               int batch, int mult)                                           \
    {                                                                                         \
        long M = 1L << n_power;                                                               \
        int neg = (reduction_poly == 0);                                                      \
        cx_##SFX* x = (cx_##SFX*)malloc(sizeof(cx_##SFX) * M);                                \
        cx_##SFX sc = cmk_##SFX(mod_inverse[0], mod_inverse[1]);                              \
        for (int b = 0; b < batch; b++) {                                                     \
            T* tp = temp + 2 * (long)b * M;                                                   \
            T* rp = real_inout + (long)b * M;                                                 \
            if (fft_type == 0) {                                                              \
                for (long i = 0; i < M; i++) x[i] = cmk_##SFX(rp[i], (T)0);                   \
                fwd_stages_##SFX(x, n_power, table, neg);                                     \
                for (long i = 0; i < M; i++) st_##SFX(tp, i, x[i]);                           \
            } else {                                                                          \
                const T* q = tp + 2 * (long)batch * M;                                        \
                for (long i = 0; i < M; i++)                                                  \
                    x[i] = mult ? cmul_##SFX(ld_##SFX(tp, i), ld_##SFX(q, i)) : ld_##SFX(tp, i); \
                inv_stages_##SFX(x, n_power, table, neg);                                     \
                for (long i = 0; i < M; i++) rp[i] = cmul_##SFX(x[i], sc).re;                 \
            }                                                                                 \
        }                                                                                     \
        free(x);                                                                              \
    }                                                                                         \
                                                                                              \
    /* GPU_FFNT (fft.cu:1386-1515). n_power = log2 N of the real ring; the transform   */    \
    /* runs on N/2 complex values. Forward: fold f_j + i f_{j+N/2}, multiply by the    */    \
    /* twist table (fft.cu:1057-1069), CT stages, write temp. Inverse: product of the  */    \
    /* two temp spectra (fft.cu:1252-1263), GS stages, multiply by mod_inverse and     */    \
    /* then by the untwist table, unfold re -> [j], im -> [j+N/2] (fft.cu:1366-1383).   */   \
    void orc_gpu_ffnt_##SFX(T* inout, T* temp, const T* twist, const T* table, int n_power,   \
                            int fft_type, const T* mod_inverse, int batch, int mult)          \
    {                                                                                         \
        long M = 1L << (n_power - 1);                                                         \
        cx_##SFX* x = (cx_##SFX*)malloc(sizeof(cx_##SFX) * M);                                \
        cx_##SFX sc = cmk_##SFX(mod_inverse[0], mod_inverse[1]);                              \
        for (int b = 0; b < batch; b++) {                                                     \
            T* tp = temp + 2 * (long)b * M;                                                   \
            T* rp = inout + (long)b * 2 * M;                                                  \
            if (fft_type == 0) {                                                              \
                for (long i = 0; i < M; i++)                                                  \
                    x[i] = cmul_##SFX(cmk_##SFX(rp[i], rp[i + M]), ld_##SFX(twist, i));       \
                fwd_stages_##SFX(x, n_power - 1, table, 0);                                   \
                for (long i = 0; i < M; i++) st_##SFX(tp, i, x[i]);                           \
            } else {                                                                          \
                const T* q = tp + 2 * (long)batch * M;                                        \
                for (long i = 0; i < M; i++)                                                  \
                    x[i] = mult ? cmul_##SFX(ld_##SFX(tp, i), ld_##SFX(q, i)) : ld_##SFX(tp, i); \
                inv_stages_##SFX(x, n_power - 1, table, 0);                                   \
                for (long i = 0; i < M; i++) {                                                \
                    cx_##SFX v = cmul_##SFX(cmul_##SFX(x[i], sc), ld_##SFX(twist, i));        \
                    rp[i] = v.re;                                                             \
                    rp[i + M] = v.im;                                                         \
                }                                                                             \
            }                                                                                 \
        }                                                                                     \
        free(x);                                                                              \
    }                                                                                         \
                                                                                              \
    /* FFT<T>::fft / FFT<T>::ifft on one vector of 2n complex (fft_cpu.cu:131-198).    */    \
    void orc_cpu_fft_##SFX(int n, T* data, const T* rev_roots)                                \
    {                                                                                         \
        int m = (int)log2((double)(2 * n));                                                   \
        cx_##SFX* x = (cx_##SFX*)malloc(sizeof(cx_##SFX) * 2 * n);                            \
        for (long i = 0; i < 2 * n; i++) x[i] = ld_##SFX(data, i);                            \
        fwd_stages_##SFX(x, m, rev_roots, 0);                                                 \
        for (long i = 0; i < 2 * n; i++) st_##SFX(data, i, x[i]);                             \
        free(x);                                                                              \
    }                                                                                         \
    void orc_cpu_ifft_##SFX(int n, T* data, const T* rev_inv_roots, T n_inverse)              \
    {                                                                                         \
        int m = (int)log2((double)(2 * n));                                                   \
        cx_##SFX* x = (cx_##SFX*)malloc(sizeof(cx_##SFX) * 2 * n);                            \
        for (long i = 0; i < 2 * n; i++) x[i] = ld_##SFX(data, i);                            \
        inv_stages_##SFX(x, m, rev_inv_roots, 0);                                             \
        /* input[i] * n_inverse: COMPLEX * Float -> scalar operator* of complex.cuh:153-159, */ \
        /* whose imaginary part is re*s (a reference quirk kept here on purpose).           */ \
        for (long i = 0; i < 2 * n; i++) x[i] = cmk_##SFX(x[i].re * n_inverse, x[i].re * n_inverse); \
        for (long i = 0; i < 2 * n; i++) st_##SFX(data, i, x[i]);                             \
        free(x);                                                                              \
    }                                                                                         \
                                                                                              \
    /* FFNT<T>::MULT (fft_cpu.cu:301-432): fold, twist, two forward transforms,        */    \
    /* product, inverse, untwist then scale, round to unsigned long long.               */   \
    void orc_cpu_ffnt_mult_##SFX(int n, const uint64_t* a, const uint64_t* b, uint64_t* out, \
                                 const T* rev_roots, const T* rev_inv_roots, const T* twist,  \
                                 const T* untwist)                                            \
    {                                                                                         \
        long h = n >> 1;                                                                      \
        int m = (int)log2((double)h);                                                         \
        cx_##SFX* x = (cx_##SFX*)malloc(sizeof(cx_##SFX) * h);                                \
        cx_##SFX* y = (cx_##SFX*)malloc(sizeof(cx_##SFX) * h);                                \
        for (long i = 0; i < h; i++) {                                                        \
            x[i] = cmul_##SFX(cmk_##SFX((T)a[i], (T)a[i + h]), ld_##SFX(twist, i));           \
            y[i] = cmul_##SFX(cmk_##SFX((T)b[i], (T)b[i + h]), ld_##SFX(twist, i));           \
        }                                                                                     \
        fwd_stages_##SFX(x, m, rev_roots, 0);                                                 \
        fwd_stages_##SFX(y, m, rev_roots, 0);                                                 \
        for (long i = 0; i < h; i++) x[i] = cmul_##SFX(x[i], y[i]);                           \
        inv_stages_##SFX(x, m, rev_inv_roots, 0);                                             \
        T ninv = (T)(1.0 / (double)h);                                                        \
        for (long i = 0; i < h; i++) {                                                        \
            cx_##SFX v = cmul_##SFX(x[i], ld_##SFX(untwist, i));                              \
            v = cmul_##SFX(v, cmk_##SFX(ninv, (T)0));                                         \
            out[i] = (uint64_t)(long long)llround((double)v.re);                              \
            out[i + h] = (uint64_t)(long long)llround((double)v.im);                          \
        }                                                                                     \
        free(x);                                                                              \
        free(y);                                                                              \
    }

ORC_DEFINE(double, f64, cos, sin, exp)
ORC_DEFINE(float, f32, cosf, sinf, expf)

/* ------------------------------------------------------------------------- */
/* GPU_Special_FFT (fft.cu:727-1007, launch tables fft.cuh:388-500): radix-2  */
/* stages on vectors of 2^n_power complex, in place. The span t = 2^p pairs   */
/* i and i + t (i the lower element of its group of 2t) and uses             */
/* table[t + (i mod t)] (the kernels' root[m + (omega & (m - 1))]).           */
/*   forward: spans 1, 2, ..., 2^(n-1), CooleyTukeyUnit (fft.cuh:69-78);      */
/*   inverse: spans 2^(n-1), ..., 1, GentlemanSandeUnit (fft.cuh:80-89), then */
/*            every value times mod_inverse (the last inverse kernel).        */
/* ------------------------------------------------------------------------- */
#define ORC_SPECIAL(T, SFX)                                                                   \
    void orc_gpu_special_fft_##SFX(T* inout, const T* table, int n_power, int fft_type,       \
                                   const T* mod_inverse, int batch)                          \
    {                                                                                         \
        long M = 1L << n_power;                                                               \
        cx_##SFX sc = cmk_##SFX(mod_inverse[0], mod_inverse[1]);                              \
        for (int b = 0; b < batch; b++) {                                                     \
            T* p = inout + 2 * (long)b * M;                                                   \
            for (int s = 0; s < n_power; s++) {                                               \
                int e = fft_type == 0 ? s : n_power - 1 - s;                                  \
                long t = 1L << e;                                                             \
                for (long base = 0; base < M; base += 2 * t)                                  \
                    for (long j = 0; j < t; j++) {                                            \
                        cx_##SFX w = ld_##SFX(table, t + j);                                  \
                        cx_##SFX u = ld_##SFX(p, base + j), v = ld_##SFX(p, base + j + t);    \
                        if (fft_type == 0) {                                                  \
                            cx_##SFX vw = cmul_##SFX(v, w);                                   \
                            st_##SFX(p, base + j, cadd_##SFX(u, vw));                         \
                            st_##SFX(p, base + j + t, csub_##SFX(u, vw));                     \
                        } else {                                                              \
                            st_##SFX(p, base + j, cadd_##SFX(u, v));                          \
                            st_##SFX(p, base + j + t, cmul_##SFX(csub_##SFX(u, v), w));       \
                        }                                                                     \
                    }                                                                         \
            }                                                                                 \
            if (fft_type != 0)                                                                \
                for (long i = 0; i < M; i++) st_##SFX(p, i, cmul_##SFX(ld_##SFX(p, i), sc));  \
        }                                                                                     \
    }
ORC_SPECIAL(double, f64)
ORC_SPECIAL(float, f32)

/* ------------------------------------------------------------------------- */
/* Exact integer products (the builder's schoolbook; 128-bit accumulation).   */
/* Outputs are split into low/high signed 64-bit halves of the __int128.      */
/* The reference's own schoolbook (fft_cpu.cu:23-73) reduces mod q; these keep */
/* the full value, and tests reduce where the reference does.                 */
/* ------------------------------------------------------------------------- */
static inline void put128(__int128 v, int64_t* lo, int64_t* hi, long i)
{
    lo[i] = (int64_t)(uint64_t)(unsigned __int128)v;
    hi[i] = (int64_t)(v >> 64);
}

/* kind: 0 = linear (2n outputs), 1 = cyclic mod X^n-1, 2 = negacyclic mod X^n+1 */
void orc_schoolbook_i64(const int64_t* a, const int64_t* b, int n, int kind, int64_t* lo,
                        int64_t* hi)
{
    long outn = (kind == 0) ? 2L * n : n;
    __int128* acc = (__int128*)calloc((size_t)(2L * n), sizeof(__int128));
    for (long i = 0; i < n; i++) {
        __int128 ai = a[i];
        if (ai == 0) continue;
        for (long j = 0; j < n; j++) acc[i + j] += ai * (__int128)b[j];
    }
    for (long k = 0; k < outn; k++) {
        __int128 v = acc[k];
        if (kind == 1) v += acc[k + n];
        if (kind == 2) v -= acc[k + n];
        put128(v, lo, hi, k);
    }
    free(acc);
}

/* Selected coefficients of the negacyclic product (exact), O(n) each. */
void orc_negacyclic_coeffs_i64(const int64_t* a, const int64_t* b, int n, const int* idx, int cnt,
                               int64_t* lo, int64_t* hi)
{
    for (int t = 0; t < cnt; t++) {
        long k = idx[t];
        __int128 v = 0;
        for (long i = 0; i < n; i++) {
            long j = k - i;
            if (j >= 0)
                v += (__int128)a[i] * b[j];
            else
                v -= (__int128)a[i] * b[j + n];
        }
        put128(v, lo, hi, t);
    }
}

/* Selected coefficients of the linear product (exact), indices in [0, 2n). */
void orc_linear_coeffs_i64(const int64_t* a, const int64_t* b, int n, const int* idx, int cnt,
                           int64_t* lo, int64_t* hi)
{
    for (int t = 0; t < cnt; t++) {
        long k = idx[t];
        __int128 v = 0;
        long i0 = k - (n - 1) > 0 ? k - (n - 1) : 0;
        long i1 = k < n - 1 ? k : n - 1;
        for (long i = i0; i <= i1; i++) v += (__int128)a[i] * b[k - i];
        put128(v, lo, hi, t);
    }
}

/* Balanced signed-digit decomposition used by the split-precision product:   */
/* x = sum_l d_l 2^(w l), d_l in [-2^(w-1), 2^(w-1)), last digit absorbs rest. */
void orc_balanced_digits_i64(const int64_t* x, long count, int w, int limbs, int32_t* digits)
{
    int64_t base = (int64_t)1 << w, half = base >> 1;
    for (long i = 0; i < count; i++) {
        int64_t v = x[i];
        for (int l = 0; l < limbs; l++) {
            int64_t d;
            if (l == limbs - 1) {
                d = v;
            } else {
                int64_t r = v & (base - 1);
                d = (r >= half) ? r - base : r;
            }
            digits[(long)l * count + i] = (int32_t)d;
            v = (v - d) >> w;
        }
    }
}
