// gpufft-b200: FP32 split-precision negacyclic product with exact int64 output.
//
// c = a * b mod (X^N + 1) for integer coefficients, computed exactly with
// single-precision transforms:
//   1. every coefficient is cut into k balanced signed digits of w bits,
//      x = sum_l d_l 2^(w l), d_l in [-2^(w-1), 2^(w-1)) (the top digit takes
//      what is left), giving k small-integer "limb" polynomials per operand;
//   2. each limb polynomial goes through the FFNT forward transform (fold,
//      twist, half-length FFT; reference fft.cu:1013-1212) in FP32;
//   3. for every shift s = 0 .. 2k-2 the limb spectra are combined pointwise,
//      C^_s = sum_{i+j=s} A^_i B^_j, and C_s is brought back by the inverse
//      transform (reference fft.cu:1214-1384);
//   4. each C_s is rounded to an integer and c = sum_s C_s 2^(w s) is formed in
//      exact int64 arithmetic (wrapping modulo 2^64).
// The limb width is chosen so that every C_s stays well inside FP32's exact
// range (an error model calibrated on this transform); the largest distance
// of any C_s value to its nearest integer ("pre-rounding error") is measured
// on the device and returned, so exactness (error < 0.5) is checked per call.
//
// Kernels (N > 8192, per wave of products; workspace in L2):
//   split_fwd0   strided first forward pass for the 2k limb polynomials of a
//                product column block: the int32 inputs are loaded once, each
//                limb is extracted, folded, twisted and transformed in turn;
//   split_mid    contiguous last forward pass of all 2k limb spectra, the
//                2k-1 pointwise group sums and the first inverse pass of each;
//   split_inv0   strided last inverse pass of every group with scale, untwist,
//                unfold, rounding and the int64 recombination in registers.
// N <= 8192 runs all of it in one kernel (split_mid<true>).
#include "gf_pass.cuh"

#include <algorithm>
#include <cmath>

namespace gfb
{

constexpr int SPLIT_MAX_LIMBS = 8;

// Balanced signed digit l (width w, k digits) of v.
__device__ __forceinline__ int limb_digit(long long v, int l, int w, int k)
{
    const long long base = 1LL << w, half = base >> 1;
    long long d = 0;
    for (int i = 0; i <= l; i++)
    {
        if (i == k - 1)
        {
            d = v;
        }
        else
        {
            const long long r = v & (base - 1);
            d = (r >= half) ? r - base : r;
        }
        v = (v - d) >> w;
    }
    return (int)d;
}

struct SplitArgs
{
    const int32_t* a;
    const int32_t* b;
    int64_t* c;
    cx<float>* spec;  // [2k][W][M] limb spectra (operand-major: a limbs then b limbs)
    cx<float>* group; // [2k-1][W][M] group spectra
    const cx<float>* roots;
    const cx<float>* inv_roots;
    const cx<float>* twist;
    const cx<float>* untwist;
    unsigned* max_err; // float bits of the largest pre-rounding error (may be null)
    float scale;
    int w, k;
    long long W; // products per wave (stride of the workspace)
    long long batch;
    PassGeo geo;
};

// Distance of a group value to its nearest integer. Above 2^22 every float is
// (nearly) an integer and the distance no longer certifies exactness, so such
// values report 1.0.
__device__ __forceinline__ float group_error(cx<float> v, float rr, float ri)
{
    const float lim = 4194304.0f; // 2^22
    if (fabsf(v.x) >= lim || fabsf(v.y) >= lim) return 1.0f;
    return fmaxf(fabsf(v.x - rr), fabsf(v.y - ri));
}

__device__ __forceinline__ void report_err(unsigned* dst, float e)
{
    if (!dst) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
    if ((threadIdx.x & 31) == 0) atomicMax(dst, __float_as_uint(e));
}

// --------------------------------------------------------------------------
// strided first forward pass of every limb polynomial
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(NTHR) split_fwd0(const SplitArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* sm = reinterpret_cast<cx<float>*>(smraw);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const PassGeo& G = a.geo; // strided, batch index = operand * W + product
    const long long M = 1LL << G.m;

    TwCtx c;
    c.qoff = G.qoff;
    c.L = G.L;
    c.qmask = (1 << G.L) - 1;
    c.s0 = 0;
    c.neg = 0;
    c.g = cta_group(G, cta);
    const Rounds R = make_rounds(G.qoff, G.L, true);
    const int w0 = R.lo[0] & ~3;

    // the raw coefficients (fold pair j, j+M) of this CTA's elements
    int vlo[RPT], vhi[RPT];
    long long jj[RPT];
    long long bb = 0;
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        const Where wh = locate(G, cta, e_of(t, w0, r));
        bb = wh.b;
        jj[r] = wh.j;
        const long long op = wh.b / a.W, p = wh.b - op * a.W;
        const int32_t* src = (op == 0 ? a.a : a.b) + p * 2 * M + wh.j;
        vlo[r] = (p < a.batch) ? __ldcs(src) : 0;
        vhi[r] = (p < a.batch) ? __ldcs(src + M) : 0;
    }
    const long long op = bb / a.W, p = bb - op * a.W;
    for (int l = 0; l < a.k; l++)
    {
        cx<float> x[RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const cx<float> f = mk<float>((float)limb_digit(vlo[r], l, a.w, a.k), (float)limb_digit(vhi[r], l, a.w, a.k));
            x[r] = cmul<float>(f, ldg<float>(a.twist + jj[r]));
        }
        if (l > 0) __syncthreads();
        const int wl = run_pass_rounds<float, true>(x, sm, a.roots, c, R, t);
        cx<float>* dst = a.spec + ((op * a.k + l) * a.W + p) * M;
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const Where wh = locate(G, cta, e_of(t, wl, r));
            if (p < a.batch) dst[wh.j] = x[r];
        }
    }
}

// --------------------------------------------------------------------------
// contiguous middle: last forward pass of the 2k limb spectra, group sums,
// first inverse pass of every group (SINGLE: whole transforms, int32 in,
// int64 out, everything in this kernel)
// --------------------------------------------------------------------------
template <bool SINGLE> __global__ void __launch_bounds__(NTHR) split_mid(const SplitArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* sm = reinterpret_cast<cx<float>*>(smraw);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const PassGeo& G = a.geo; // contiguous, batch index = product
    const long long M = 1LL << G.m;

    TwCtx c;
    c.qoff = 0;
    c.L = G.L;
    c.qmask = (1 << G.L) - 1;
    c.s0 = G.s0;
    c.neg = 0;
    c.g = cta_group(G, cta);
    const Rounds Rf = make_rounds(0, G.L, true);
    const Rounds Ri = make_rounds(0, G.L, false);
    const int w0 = Rf.lo[0] & ~3;
    const int wl = Ri.lo[0] & ~3; // last forward window == first inverse window

    long long jl[RPT], bl[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        const Where wh = locate(G, cta, e_of(t, wl, r));
        jl[r] = wh.j;
        bl[r] = wh.b;
    }

    // forward last pass of every limb spectrum; results parked in a.spec
    for (int tau = 0; tau < 2 * a.k; tau++)
    {
        const int op = tau / a.k, l = tau - op * a.k;
        cx<float> x[RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const Where wh = locate(G, cta, e_of(t, w0, r));
            if (wh.b >= a.batch)
            {
                x[r] = mk<float>(0.f, 0.f);
                continue;
            }
            if (SINGLE)
            {
                const int32_t* src = (op == 0 ? a.a : a.b) + wh.b * 2 * M + wh.j;
                const cx<float> f =
                    mk<float>((float)limb_digit(__ldg(src), l, a.w, a.k), (float)limb_digit(__ldg(src + M), l, a.w, a.k));
                x[r] = cmul<float>(f, ldg<float>(a.twist + wh.j));
            }
            else
            {
                x[r] = a.spec[((long long)tau * a.W + wh.b) * M + wh.j];
            }
        }
        if (tau > 0) __syncthreads();
        run_pass_rounds<float, true>(x, sm, a.roots, c, Rf, t);
#pragma unroll
        for (int r = 0; r < RPT; r++)
            if (bl[r] < a.batch) a.spec[((long long)tau * a.W + bl[r]) * M + jl[r]] = x[r];
    }

    // group sums and the first inverse pass (the whole inverse when SINGLE)
    long long acc_lo[RPT], acc_hi[RPT];
    float err = 0.f;
    if (SINGLE)
    {
#pragma unroll
        for (int r = 0; r < RPT; r++) acc_lo[r] = acc_hi[r] = 0;
    }
    int wend = wl;
    for (int s = 0; s <= 2 * (a.k - 1); s++)
    {
        const int i0 = s - (a.k - 1) > 0 ? s - (a.k - 1) : 0;
        const int i1 = s < a.k - 1 ? s : a.k - 1;
        cx<float> x[RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            cx<float> acc = mk<float>(0.f, 0.f);
            if (bl[r] < a.batch)
                for (int i = i0; i <= i1; i++)
                {
                    const cx<float> u = a.spec[((long long)i * a.W + bl[r]) * M + jl[r]];
                    const cx<float> v = a.spec[((long long)(a.k + s - i) * a.W + bl[r]) * M + jl[r]];
                    acc = cadd<float>(acc, cmul<float>(u, v));
                }
            x[r] = acc;
        }
        __syncthreads();
        wend = run_pass_rounds<float, false>(x, sm, a.inv_roots, c, Ri, t);
        if (SINGLE)
        {
            const int sh = a.w * s;
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                const Where wh = locate(G, cta, e_of(t, wend, r));
                if (wh.b >= a.batch) continue;
                const cx<float> v = cmul<float>(cmul<float>(x[r], mk<float>(a.scale, 0.f)), ldg<float>(a.untwist + wh.j));
                const float rr = rintf(v.x), ri = rintf(v.y);
                err = fmaxf(err, group_error(v, rr, ri));
                acc_lo[r] += (long long)((unsigned long long)(long long)rr << sh);
                acc_hi[r] += (long long)((unsigned long long)(long long)ri << sh);
            }
        }
        else
        {
            cx<float>* dst = a.group + (long long)s * a.W * M;
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                const Where wh = locate(G, cta, e_of(t, wend, r));
                if (wh.b < a.batch) dst[wh.b * M + wh.j] = x[r];
            }
        }
    }
    if (SINGLE)
    {
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const Where wh = locate(G, cta, e_of(t, wend, r));
            if (wh.b >= a.batch) continue;
            int64_t* dst = a.c + wh.b * 2 * M + wh.j;
            __stcs(reinterpret_cast<long long*>(dst), acc_lo[r]);
            __stcs(reinterpret_cast<long long*>(dst + M), acc_hi[r]);
        }
        report_err(a.max_err, err);
    }
}

// --------------------------------------------------------------------------
// strided last inverse pass of every group, rounding and int64 recombination
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(NTHR) split_inv0(const SplitArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* sm = reinterpret_cast<cx<float>*>(smraw);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const PassGeo& G = a.geo; // strided, batch index = product
    const long long M = 1LL << G.m;

    TwCtx c;
    c.qoff = G.qoff;
    c.L = G.L;
    c.qmask = (1 << G.L) - 1;
    c.s0 = 0;
    c.neg = 0;
    c.g = cta_group(G, cta);
    const Rounds R = make_rounds(G.qoff, G.L, false);
    const int w0 = R.lo[0] & ~3;

    long long acc_lo[RPT], acc_hi[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++) acc_lo[r] = acc_hi[r] = 0;
    float err = 0.f;
    int wend = w0;
    for (int s = 0; s <= 2 * (a.k - 1); s++)
    {
        const cx<float>* src = a.group + (long long)s * a.W * M;
        cx<float> x[RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const Where wh = locate(G, cta, e_of(t, w0, r));
            x[r] = (wh.b < a.batch) ? src[wh.b * M + wh.j] : mk<float>(0.f, 0.f);
        }
        if (s > 0) __syncthreads();
        wend = run_pass_rounds<float, false>(x, sm, a.inv_roots, c, R, t);
        const int sh = a.w * s;
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const Where wh = locate(G, cta, e_of(t, wend, r));
            if (wh.b >= a.batch) continue;
            const cx<float> v = cmul<float>(cmul<float>(x[r], mk<float>(a.scale, 0.f)), ldg<float>(a.untwist + wh.j));
            const float rr = rintf(v.x), ri = rintf(v.y);
            err = fmaxf(err, group_error(v, rr, ri));
            acc_lo[r] += (long long)((unsigned long long)(long long)rr << sh);
            acc_hi[r] += (long long)((unsigned long long)(long long)ri << sh);
        }
    }
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        const Where wh = locate(G, cta, e_of(t, wend, r));
        if (wh.b >= a.batch) continue;
        int64_t* dst = a.c + wh.b * 2 * M + wh.j;
        __stcs(reinterpret_cast<long long*>(dst), acc_lo[r]);
        __stcs(reinterpret_cast<long long*>(dst + M), acc_hi[r]);
    }
    report_err(a.max_err, err);
}

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
// Largest pre-rounding error expected for k limbs of width w at ring size N.
// For one limb pair the measured maximum over a batch follows
//     err ~ C * rms(d_a) * rms(d_b) * sqrt(N) * sqrt(log2(N/2)) * 2^-24,  C = 7.1
// (calibrated on FP32 negacyclic limb products: balanced 6-bit limbs at
// N = 2^16 give 0.144). A group sum of several pairs adds their errors in
// quadrature. Balanced digits have rms 2^(w-1)/sqrt(3); the top digit holds the
// tb = input_bits - w(k-1) leftover bits: rms 0.577 * 2^tb when the inputs are
// non-negative (digit in [0, 2^tb]), 2^tb / sqrt(3) when signed.
static double predicted_error(int n_power, int input_bits, int w, int k, bool non_negative)
{
    double r[SPLIT_MAX_LIMBS];
    for (int l = 0; l < k; l++) r[l] = std::ldexp(1.0, w - 1) / std::sqrt(3.0);
    const int tb = input_bits - w * (k - 1);
    r[k - 1] = non_negative ? 0.577 * std::ldexp(1.0, tb) : std::ldexp(1.0, tb) / std::sqrt(3.0);
    double worst = 0.0;
    for (int s = 0; s <= 2 * (k - 1); s++)
    {
        double e2 = 0.0;
        for (int i = 0; i < k; i++)
        {
            const int j = s - i;
            if (j >= 0 && j < k) e2 += (r[i] * r[j]) * (r[i] * r[j]);
        }
        worst = std::max(worst, std::sqrt(e2));
    }
    return 7.1 * worst * std::sqrt(std::ldexp(1.0, n_power)) * std::sqrt((double)(n_power - 1)) * std::ldexp(1.0, -24);
}

static bool choose_limbs(int n_power, int input_bits, bool non_negative, int* w_out, int* k_out)
{
    // the plan with the fewest limbs whose predicted error is at most 0.2
    for (int k = 1; k <= SPLIT_MAX_LIMBS; k++)
    {
        const int w = (input_bits + k - 1) / k;
        if (w < 1 || w > 20) continue;
        if (predicted_error(n_power, input_bits, w, k, non_negative) <= 0.2)
        {
            *w_out = w;
            *k_out = k;
            return true;
        }
    }
    return false;
}

static long long split_wave(int m, int k, long long batch)
{
    const size_t per = (size_t)(4 * k - 1) * ((size_t)1 << m) * sizeof(cx<float>);
    long long w = (long long)((64ull << 20) / per);
    if (w < 1) w = 1;
    return w < batch ? w : batch;
}

static size_t split_ws_bytes(int m, int k, long long W)
{
    return (size_t)(4 * k - 1) * (size_t)W * ((size_t)1 << m) * sizeof(cx<float>);
}

template <typename K> static int launch_split(K* kern, int* done, const SplitArgs& a, long long ctas, cudaStream_t s)
{
    if (ctas <= 0) return GPUFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return GPUFFT_ERROR_INVALID_VALUE;
    const size_t smem = sizeof(cx<float>) * SMEM_ELEMS;
    int st = ensure_smem(kern, smem, done);
    if (st) return st;
    kern<<<dim3((unsigned)ctas), dim3(NTHR), smem, s>>>(a);
    return check_launch();
}

static int split_mul(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch, int input_bits,
                     int non_negative, int limb_bits, int num_limbs, const void* tables, void* ws, size_t ws_bytes,
                     unsigned* max_err, cudaStream_t s)
{
    if (n_power < 2 || n_power > 22) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!a || !b || !c || !tables || batch <= 0 || input_bits < 1 || input_bits > 31) return GPUFFT_ERROR_INVALID_VALUE;
    if ((uintptr_t)a % 4 || (uintptr_t)b % 4 || (uintptr_t)c % 8 || (uintptr_t)tables % 8 || (uintptr_t)ws % 8)
        return GPUFFT_ERROR_MISALIGNED;
    int w = limb_bits, k = num_limbs;
    if (w <= 0 || k <= 0)
    {
        if (!choose_limbs(n_power, input_bits, non_negative != 0, &w, &k)) return GPUFFT_ERROR_INVALID_VALUE;
    }
    if (k > SPLIT_MAX_LIMBS || w < 1 || w > 20 || (long long)w * k < input_bits) return GPUFFT_ERROR_INVALID_VALUE;

    const int m = n_power - 1;
    const long long M = 1LL << m;
    const auto* tab = reinterpret_cast<const cx<float>*>(tables);
    SplitArgs A{};
    A.a = a;
    A.b = b;
    A.roots = tab;
    A.inv_roots = tab + M / 2;
    A.twist = tab + M;
    A.untwist = tab + 2 * M;
    A.max_err = max_err;
    A.scale = (float)(1.0 / (double)M);
    A.w = w;
    A.k = k;

    long long W = split_wave(m, k, batch);
    const size_t need1 = split_ws_bytes(m, k, 1);
    if (!ws || ws_bytes < need1) return GPUFFT_ERROR_WORKSPACE;
    if (split_ws_bytes(m, k, W) > ws_bytes) W = (long long)(ws_bytes / need1);
    if (max_err)
    {
        cudaError_t e = cudaMemsetAsync(max_err, 0, sizeof(unsigned), s);
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    static int done_mid1[64] = {0}, done_mid0[64] = {0}, done_f0[64] = {0}, done_i0[64] = {0};
    const Plan p = make_plan(m);
    for (long long p0 = 0; p0 < batch; p0 += W)
    {
        const long long wv = (batch - p0) < W ? (batch - p0) : W;
        A.a = a + p0 * 2 * M;
        A.b = b + p0 * 2 * M;
        A.c = c + p0 * 2 * M;
        A.W = wv;
        A.batch = wv;
        A.spec = reinterpret_cast<cx<float>*>(ws);
        A.group = A.spec + (size_t)(2 * k) * wv * M;
        if (m <= EBITS)
        {
            A.geo = PassGeo{};
            A.geo.m = m;
            A.geo.L = m;
            A.geo.contig = 1;
            const long long ctas = (wv * M + ECTA - 1) / ECTA;
            int st = launch_split(split_mid<true>, done_mid1, A, ctas, s);
            if (st) return st;
            continue;
        }
        long long ctas = 0;
        A.geo = pass_geo(p, 0, m, 0, 2 * wv, &ctas);
        int st = launch_split(split_fwd0, done_f0, A, ctas, s);
        if (st) return st;
        A.geo = pass_geo(p, 1, m, 0, wv, &ctas);
        st = launch_split(split_mid<false>, done_mid0, A, ctas, s);
        if (st) return st;
        A.geo = pass_geo(p, 0, m, 0, wv, &ctas);
        st = launch_split(split_inv0, done_i0, A, ctas, s);
        if (st) return st;
    }
    return GPUFFT_SUCCESS;
}

} // namespace gfb

extern "C" int gpufft_split_plan(int n_power, int input_bits, int non_negative, int* limb_bits, int* num_limbs)
{
    if (!limb_bits || !num_limbs || input_bits < 1 || input_bits > 31) return GPUFFT_ERROR_INVALID_VALUE;
    if (n_power < 2 || n_power > 22) return GPUFFT_ERROR_INVALID_N_POWER;
    return gfb::choose_limbs(n_power, input_bits, non_negative != 0, limb_bits, num_limbs) ? GPUFFT_SUCCESS
                                                                                          : GPUFFT_ERROR_INVALID_VALUE;
}

extern "C" size_t gpufft_negacyclic_mul_split_workspace_bytes(int n_power, int batch, int num_limbs)
{
    if (n_power < 2 || n_power > 22 || batch <= 0 || num_limbs < 1 || num_limbs > gfb::SPLIT_MAX_LIMBS) return 0;
    const int m = n_power - 1;
    const long long W = gfb::split_wave(m, num_limbs, batch);
    return gfb::split_ws_bytes(m, num_limbs, W);
}

extern "C" int gpufft_negacyclic_mul_split_f32(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch,
                                               int input_bits, int non_negative, int limb_bits, int num_limbs,
                                               const void* tables, void* workspace, size_t workspace_bytes,
                                               float* max_error, gpufft_stream_t stream)
{
    return gfb::split_mul(a, b, c, n_power, batch, input_bits, non_negative, limb_bits, num_limbs, tables, workspace,
                          workspace_bytes, reinterpret_cast<unsigned*>(max_error), (cudaStream_t)stream);
}
