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
#include "gf_engine.cuh"

#include <cstdio>

namespace gfb
{

enum InKind
{
    IN_CPX = 0,  // complex vector (transform position j)
    IN_REAL = 1, // real promoted to complex (fft.cu:303-305)
    IN_FOLD = 2, // FFNT fold f_j + i f_{j+M} then twist (fft.cu:1057-1069)
    IN_PROD = 3  // product of the two complex operands (fft.cu:194-205, 1252-1263)
};
enum OutKind
{
    OUT_CPX = 0,   // complex vector, optionally scaled by mod_inverse (fft.cu:246-253)
    OUT_REAL = 1,  // real part of the scaled value (fft.cu:499-514)
    OUT_UNFOLD = 2 // scale, untwist, unfold re -> j, im -> j+M (fft.cu:1366-1383)
};

template <typename T> struct PassArgs
{
    const void* in;
    void* out;
    const cx<T>* table;
    const cx<T>* twist;
    cx<T> scale;
    long long prod_off; // element offset of the second operand (IN_PROD)
    long long batch;
    PassGeo geo;
    int zero_pad; // forward first pass: the upper half of each input is zero
    int do_scale; // last inverse pass: multiply by scale
};

// Locate CTA-local element e: transform index j and batch entry b.
struct Where
{
    long long b;
    long long j;
};

__device__ __forceinline__ Where locate(const PassGeo& G, long long cta, int e)
{
    Where w;
    const long long M = 1LL << G.m;
    if (G.contig)
    {
        const long long gi = cta * ECTA + e;
        w.b = gi >> G.m;
        w.j = gi & (M - 1);
    }
    else
    {
        const long long S = 1LL << (G.m - G.s0 - G.L);
        const int cols = 1 << G.cols_log;
        const long long cpb = S >> G.cols_log;         // column blocks per group
        const long long per_b = (1LL << G.s0) * cpb;   // CTAs per transform
        w.b = cta / per_b;
        const long long rem = cta - w.b * per_b;
        const long long g = rem / cpb;
        const long long cblk = rem - g * cpb;
        const int c = e & (cols - 1);
        const int q = e >> G.cols_log;
        w.j = g * (M >> G.s0) + (long long)q * S + cblk * cols + c;
    }
    return w;
}

__device__ __forceinline__ long long cta_group(const PassGeo& G, long long cta)
{
    if (G.contig)
    {
        // sub-networks of 2^L elements; either s0 == 0 (g = 0) or one per CTA
        const long long gi = cta * ECTA;
        return (gi >> G.L) & ((1LL << G.s0) - 1);
    }
    const long long S = 1LL << (G.m - G.s0 - G.L);
    const long long cpb = S >> G.cols_log;
    const long long per_b = (1LL << G.s0) * cpb;
    const long long rem = cta % per_b;
    return rem / cpb;
}

template <typename T, int IN>
__device__ __forceinline__ cx<T> load_elem(const PassArgs<T>& a, long long b, long long j)
{
    const long long M = 1LL << a.geo.m;
    if (IN == IN_CPX)
    {
        if (a.zero_pad && j >= (M >> 1)) return mk<T>(T(0), T(0));
        return reinterpret_cast<const cx<T>*>(a.in)[b * M + j];
    }
    else if (IN == IN_REAL)
    {
        if (a.zero_pad && j >= (M >> 1)) return mk<T>(T(0), T(0));
        return mk<T>(reinterpret_cast<const T*>(a.in)[b * M + j], T(0));
    }
    else if (IN == IN_FOLD)
    {
        const T* p = reinterpret_cast<const T*>(a.in) + b * 2 * M + j;
        const cx<T> f = mk<T>(p[0], p[M]);
        return cmul<T>(f, ldg<T>(a.twist + j));
    }
    else
    {
        const cx<T>* p = reinterpret_cast<const cx<T>*>(a.in) + b * M + j;
        return cmul<T>(p[0], p[a.prod_off]);
    }
}

template <typename T, int OUT>
__device__ __forceinline__ void store_elem(const PassArgs<T>& a, long long b, long long j, cx<T> v)
{
    const long long M = 1LL << a.geo.m;
    if (OUT == OUT_CPX)
    {
        if (a.do_scale) v = cmul<T>(v, a.scale);
        reinterpret_cast<cx<T>*>(a.out)[b * M + j] = v;
    }
    else if (OUT == OUT_REAL)
    {
        if (a.do_scale) v = cmul<T>(v, a.scale);
        reinterpret_cast<T*>(a.out)[b * M + j] = v.x;
    }
    else
    {
        v = cmul<T>(cmul<T>(v, a.scale), ldg<T>(a.twist + j));
        T* p = reinterpret_cast<T*>(a.out) + b * 2 * M + j;
        p[0] = v.x;
        p[M] = v.y;
    }
}

template <typename T, bool FWD, int IN, int OUT>
__global__ void __launch_bounds__(NTHR) pass_kernel(const PassArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const PassGeo& G = a.geo;

    TwCtx c;
    c.qoff = G.qoff;
    c.L = G.L;
    c.qmask = (1 << G.L) - 1;
    c.s0 = G.s0;
    c.neg = G.neg;
    c.g = cta_group(G, cta);

    const Rounds R = make_rounds(G.qoff, G.L, FWD);
    const int w0 = R.lo[0] & ~3;

    cx<T> x[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        const Where w = locate(G, cta, e_of(t, w0, r));
        x[r] = (w.b < a.batch) ? load_elem<T, IN>(a, w.b, w.j) : mk<T>(T(0), T(0));
    }

    const int wl = run_pass_rounds<T, FWD>(x, sm, a.table, c, R, t);

#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        const Where w = locate(G, cta, e_of(t, wl, r));
        if (w.b < a.batch) store_elem<T, OUT>(a, w.b, w.j, x[r]);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Plan
{
    int np;
    int L[3];
};

static Plan make_plan(int m)
{
    Plan p;
    if (m <= EBITS)
    {
        p.np = 1;
        p.L[0] = m;
    }
    else if (m <= EBITS + 9)
    {
        p.np = 2;
        p.L[0] = m - EBITS;
        p.L[1] = EBITS;
    }
    else
    {
        p.np = 3;
        p.L[0] = m - EBITS - 9;
        p.L[1] = 9;
        p.L[2] = EBITS;
    }
    return p;
}

// Geometry and grid size of pass k of plan p for a 2^m transform.
static PassGeo pass_geo(const Plan& p, int k, int m, int neg, long long batch, long long* ctas)
{
    PassGeo G{};
    G.m = m;
    G.L = p.L[k];
    G.s0 = 0;
    for (int i = 0; i < k; i++) G.s0 += p.L[i];
    G.neg = neg;
    const long long M = 1LL << m;
    if (k == p.np - 1)
    {
        G.contig = 1;
        G.qoff = 0;
        G.cols_log = 0;
        *ctas = (batch * M + ECTA - 1) / ECTA;
    }
    else
    {
        G.contig = 0;
        G.cols_log = EBITS - G.L;
        G.qoff = G.cols_log;
        const long long S = 1LL << (m - G.s0 - G.L);
        *ctas = batch * (1LL << G.s0) * (S >> G.cols_log);
    }
    return G;
}

template <typename T, bool FWD, int IN, int OUT>
static int launch_pass(PassArgs<T> a, long long ctas, cudaStream_t s)
{
    if (ctas <= 0) return GPUFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return GPUFFT_ERROR_INVALID_VALUE;
    const size_t smem = sizeof(cx<T>) * SMEM_ELEMS;
    int st = ensure_smem(pass_kernel<T, FWD, IN, OUT>, smem);
    if (st) return st;
    pass_kernel<T, FWD, IN, OUT><<<dim3((unsigned)ctas), dim3(NTHR), smem, s>>>(a);
    return check_launch();
}

// Dispatch helpers so that every (IN, OUT) pair used below is instantiated once.
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
        int st;
        const int ik = (k == 0) ? in_kind : IN_CPX;
        if (ik == IN_CPX)
            st = launch_pass<T, true, IN_CPX, OUT_CPX>(a, ctas, s);
        else if (ik == IN_REAL)
            st = launch_pass<T, true, IN_REAL, OUT_CPX>(a, ctas, s);
        else
            st = launch_pass<T, true, IN_FOLD, OUT_CPX>(a, ctas, s);
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
        const int ik = (first && mult) ? IN_PROD : IN_CPX;
        const int ok = last ? out_kind : OUT_CPX;
        int st;
        if (ik == IN_PROD)
        {
            if (ok == OUT_CPX)
                st = launch_pass<T, false, IN_PROD, OUT_CPX>(a, ctas, s);
            else if (ok == OUT_REAL)
                st = launch_pass<T, false, IN_PROD, OUT_REAL>(a, ctas, s);
            else
                st = launch_pass<T, false, IN_PROD, OUT_UNFOLD>(a, ctas, s);
        }
        else
        {
            if (ok == OUT_CPX)
                st = launch_pass<T, false, IN_CPX, OUT_CPX>(a, ctas, s);
            else if (ok == OUT_REAL)
                st = launch_pass<T, false, IN_CPX, OUT_REAL>(a, ctas, s);
            else
                st = launch_pass<T, false, IN_CPX, OUT_UNFOLD>(a, ctas, s);
        }
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
