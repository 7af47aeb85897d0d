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
    long long* offs;   // [W][N] exact offset corrections (centred inputs), or null
    long long K;       // centring offset subtracted from every coefficient (0: none)
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

// Non-negative inputs are centred before they are cut into limbs,
// a = a' + K u with u = 1 + X + ... + X^(N-1), so that every limb is balanced
// (a non-centred top limb would make its group values grow like N * mean^2).
// The product is then
//     a b = a'b' + K (a'u + b'u) + K^2 uu        (mod X^N + 1)
// with (x u)_k = 2 P_x(k) - T_x (P = prefix sum, T = total) and (u u)_k =
// 2k + 2 - N, all exact integers. split_offsets computes
//     D(k) = 2 (P_a'(k) + P_b'(k)) - T_a' - T_b'
// for every product of a wave; the recombination adds K D(k) + K^2 (2k+2-N).
__device__ __forceinline__ long long offset_term(const SplitArgs& a, long long b, long long k, long long N)
{
    if (!a.offs) return 0;
    const long long d = a.offs[b * N + k];
    return (long long)((unsigned long long)a.K * (unsigned long long)d +
                       (unsigned long long)a.K * (unsigned long long)a.K * (unsigned long long)(2 * k + 2 - N));
}

constexpr int OFF_THREADS = 1024;

// One CTA per product: D(k) for k in [0, N) (a block-wide scan of the centred
// coefficient sums a'_i + b'_i).
__global__ void __launch_bounds__(OFF_THREADS) split_offsets(const SplitArgs a, int n_power)
{
    __shared__ long long part[OFF_THREADS];
    const long long N = 1LL << n_power;
    const long long p = blockIdx.x;
    const int t = threadIdx.x;
    const long long per = (N + OFF_THREADS - 1) / OFF_THREADS;
    const long long k0 = t * per;
    const int32_t* pa = a.a + p * N;
    const int32_t* pb = a.b + p * N;
    long long sum = 0;
    for (long long k = k0; k < k0 + per && k < N; k++) sum += (long long)pa[k] + (long long)pb[k] - 2 * a.K;
    part[t] = sum;
    __syncthreads();
    // inclusive scan of the per-thread sums (Hillis-Steele)
    for (int off = 1; off < OFF_THREADS; off <<= 1)
    {
        const long long v = (t >= off) ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    const long long total = part[OFF_THREADS - 1];
    long long run = (t > 0) ? part[t - 1] : 0;
    long long* out = a.offs + p * N;
    for (long long k = k0; k < k0 + per && k < N; k++)
    {
        run += (long long)pa[k] + (long long)pb[k] - 2 * a.K;
        out[k] = 2 * run - total;
    }
}

// --------------------------------------------------------------------------
// strided first forward pass of every limb polynomial
// --------------------------------------------------------------------------
template <int L> __global__ void __launch_bounds__(NTHR, 2) split_fwd0(const SplitArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* sm = reinterpret_cast<cx<float>*>(smraw);
    constexpr int QOFF = EBITS - L;
    using S = Sched<QOFF, L>;
    constexpr int W0 = S::win(0, true), WL = S::win(S::n - 1, true);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const long long M = 1LL << a.geo.m;

    // the raw coefficients (fold pair j, j+M) of this CTA's elements, loaded once
    const Tile<L, true, W0> tl(a.geo, cta, t); // batch index = operand * W + product
    const long long op = tl.b[0] / a.W, p = tl.b[0] - op * a.W;
    const int32_t* src = (op == 0 ? a.a : a.b) + p * 2 * M;
    int vlo[RPT], vhi[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        vlo[r] = (int)((long long)__ldcs(src + tl.j[r]) - a.K);
        vhi[r] = (int)((long long)__ldcs(src + tl.j[r] + M) - a.K);
    }
    TwCtx c;
    c.g = tl.g;
    c.s0 = 0;
    c.neg = 0;
    const Tile<L, true, WL> to(a.geo, cta, t);
    for (int l = 0; l < a.k; l++)
    {
        cx<float> x[1][RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const cx<float> f = mk<float>((float)limb_digit(vlo[r], l, a.w, a.k), (float)limb_digit(vhi[r], l, a.w, a.k));
            x[0][r] = cmul<float>(f, ldg<float>(a.twist + tl.j[r]));
        }
        if (l > 0) __syncthreads();
        run_rounds<float, true, QOFF, L, 1>(x, sm, a.roots, c, t);
        cx<float>* dst = a.spec + ((op * a.k + l) * a.W + p) * M;
#pragma unroll
        for (int r = 0; r < RPT; r++) dst[to.j[r]] = x[0][r];
    }
}

// --------------------------------------------------------------------------
// contiguous middle: last forward pass of the 2k limb spectra, group sums,
// first inverse pass of every group (SINGLE: whole transforms, int32 in,
// int64 out, everything in this kernel)
// --------------------------------------------------------------------------
template <int L, bool SINGLE> __global__ void __launch_bounds__(NTHR, 2) split_mid(const SplitArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* sm = reinterpret_cast<cx<float>*>(smraw);
    using S = Sched<0, L>;
    constexpr int W0 = S::win(0, true), WM = S::win(S::n - 1, true), WE = S::win(S::n - 1, false);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const long long M = 1LL << a.geo.m;

    const Tile<L, false, W0> ti(a.geo, cta, t);
    const Tile<L, false, WM> tm(a.geo, cta, t);
    TwCtx c;
    c.g = ti.g;
    c.s0 = a.geo.s0;
    c.neg = 0;

    // forward last pass of every limb spectrum; results parked in a.spec
    for (int tau = 0; tau < 2 * a.k; tau++)
    {
        const int op = tau / a.k, l = tau - op * a.k;
        cx<float> x[1][RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            if (ti.b[r] >= a.batch)
            {
                x[0][r] = mk<float>(0.f, 0.f);
                continue;
            }
            if (SINGLE)
            {
                const int32_t* src = (op == 0 ? a.a : a.b) + ti.b[r] * 2 * M + ti.j[r];
                const long long v0 = (long long)__ldg(src) - a.K, v1 = (long long)__ldg(src + M) - a.K;
                const cx<float> f = mk<float>((float)limb_digit(v0, l, a.w, a.k), (float)limb_digit(v1, l, a.w, a.k));
                x[0][r] = cmul<float>(f, ldg<float>(a.twist + ti.j[r]));
            }
            else
            {
                x[0][r] = a.spec[((long long)tau * a.W + ti.b[r]) * M + ti.j[r]];
            }
        }
        if (tau > 0) __syncthreads();
        run_rounds<float, true, 0, L, 1>(x, sm, a.roots, c, t);
#pragma unroll
        for (int r = 0; r < RPT; r++)
            if (tm.b[r] < a.batch) a.spec[((long long)tau * a.W + tm.b[r]) * M + tm.j[r]] = x[0][r];
    }

    // group sums and the first inverse pass (the whole inverse when SINGLE)
    static_assert(WM == S::win(0, false), "the inverse starts where the forward ends");
    long long acc_lo[RPT], acc_hi[RPT];
    float err = 0.f;
#pragma unroll
    for (int r = 0; r < RPT; r++) acc_lo[r] = acc_hi[r] = 0;
    const Tile<L, false, WE> te(a.geo, cta, t);
    for (int s = 0; s <= 2 * (a.k - 1); s++)
    {
        const int i0 = s - (a.k - 1) > 0 ? s - (a.k - 1) : 0;
        const int i1 = s < a.k - 1 ? s : a.k - 1;
        cx<float> x[1][RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            cx<float> acc = mk<float>(0.f, 0.f);
            if (tm.b[r] < a.batch)
                for (int i = i0; i <= i1; i++)
                {
                    const cx<float> u = a.spec[((long long)i * a.W + tm.b[r]) * M + tm.j[r]];
                    const cx<float> v = a.spec[((long long)(a.k + s - i) * a.W + tm.b[r]) * M + tm.j[r]];
                    acc = cadd<float>(acc, cmul<float>(u, v));
                }
            x[0][r] = acc;
        }
        __syncthreads();
        run_rounds<float, false, 0, L, 1>(x, sm, a.inv_roots, c, t);
        if (SINGLE)
        {
            const int sh = a.w * s;
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                if (te.b[r] >= a.batch) continue;
                const cx<float> v =
                    cmul<float>(cmul<float>(x[0][r], mk<float>(a.scale, 0.f)), ldg<float>(a.untwist + te.j[r]));
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
                if (te.b[r] < a.batch) dst[te.b[r] * M + te.j[r]] = x[0][r];
        }
    }
    if (SINGLE)
    {
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            if (te.b[r] >= a.batch) continue;
            int64_t* dst = a.c + te.b[r] * 2 * M + te.j[r];
            __stcs(reinterpret_cast<long long*>(dst), acc_lo[r] + offset_term(a, te.b[r], te.j[r], 2 * M));
            __stcs(reinterpret_cast<long long*>(dst + M), acc_hi[r] + offset_term(a, te.b[r], te.j[r] + M, 2 * M));
        }
        report_err(a.max_err, err);
    }
}

// --------------------------------------------------------------------------
// strided last inverse pass of every group, rounding and int64 recombination
// --------------------------------------------------------------------------
template <int L> __global__ void __launch_bounds__(NTHR) split_inv0(const SplitArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* sm = reinterpret_cast<cx<float>*>(smraw);
    constexpr int QOFF = EBITS - L;
    using S = Sched<QOFF, L>;
    constexpr int W0 = S::win(0, false), WE = S::win(S::n - 1, false);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const long long M = 1LL << a.geo.m;

    const Tile<L, true, W0> ti(a.geo, cta, t); // batch index = product
    const Tile<L, true, WE> te(a.geo, cta, t);
    TwCtx c;
    c.g = ti.g;
    c.s0 = 0;
    c.neg = 0;
    const long long p = ti.b[0];

    long long acc_lo[RPT], acc_hi[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++) acc_lo[r] = acc_hi[r] = 0;
    float err = 0.f;
    for (int s = 0; s <= 2 * (a.k - 1); s++)
    {
        const cx<float>* src = a.group + ((long long)s * a.W + p) * M;
        cx<float> x[1][RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++) x[0][r] = src[ti.j[r]];
        if (s > 0) __syncthreads();
        run_rounds<float, false, QOFF, L, 1>(x, sm, a.inv_roots, c, t);
        const int sh = a.w * s;
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const cx<float> v =
                cmul<float>(cmul<float>(x[0][r], mk<float>(a.scale, 0.f)), ldg<float>(a.untwist + te.j[r]));
            const float rr = rintf(v.x), ri = rintf(v.y);
            err = fmaxf(err, group_error(v, rr, ri));
            acc_lo[r] += (long long)((unsigned long long)(long long)rr << sh);
            acc_hi[r] += (long long)((unsigned long long)(long long)ri << sh);
        }
    }
    int64_t* dst = a.c + p * 2 * M;
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        __stcs(reinterpret_cast<long long*>(dst + te.j[r]), acc_lo[r] + offset_term(a, p, te.j[r], 2 * M));
        __stcs(reinterpret_cast<long long*>(dst + te.j[r] + M), acc_hi[r] + offset_term(a, p, te.j[r] + M, 2 * M));
    }
    report_err(a.max_err, err);
}

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
// Largest pre-rounding error expected for k balanced limbs of width w.
// For one limb pair the measured maximum over a batch follows
//     err ~ C * rms(d_a) * rms(d_b) * sqrt(N) * sqrt(log2(N/2)) * 2^-24,  C = 7.1
// (calibrated on FP32 negacyclic limb products: balanced 6-bit limbs at
// N = 2^16 give 0.144). A group sum of several pairs adds their errors in
// quadrature. The coefficients are signed values of magnitude below 2^B
// (B = input_bits, or input_bits - 1 after centring non-negative inputs);
// digits have rms 2^(w-1)/sqrt(3), the top digit 2^tb/sqrt(3) with
// tb = B - w(k-1) leftover bits. Also returns the typical largest group value
// (4 sigma) through *mag.
static double predicted_error(int n_power, int B, int w, int k, double* mag)
{
    double r[SPLIT_MAX_LIMBS];
    for (int l = 0; l < k; l++) r[l] = std::ldexp(1.0, w - 1) / std::sqrt(3.0);
    const int tb = B - w * (k - 1);
    r[k - 1] = std::ldexp(1.0, tb) / std::sqrt(3.0);
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
    const double sqn = std::sqrt(std::ldexp(1.0, n_power));
    if (mag) *mag = 4.0 * worst * sqn;
    return 7.1 * worst * sqn * std::sqrt((double)(n_power - 1)) * std::ldexp(1.0, -24);
}

static bool choose_limbs(int n_power, int input_bits, bool non_negative, int* w_out, int* k_out)
{
    // the plan with the fewest limbs whose predicted error is at most 0.2 and
    // whose group values stay far inside FP32's certifiable range (< 2^21)
    const int B = non_negative ? input_bits - 1 : input_bits;
    for (int k = 1; k <= SPLIT_MAX_LIMBS; k++)
    {
        const int w = (B + 1 + k - 1) / k; // k balanced digits of w bits cover 2^B in magnitude
        if (w < 1 || w > 20 || B - w * (k - 1) > w - 1) continue;
        double mag = 0;
        if (predicted_error(n_power, B, w, k, &mag) <= 0.2 && mag < std::ldexp(1.0, 21))
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
    const size_t per = (size_t)(4 * k - 1) * ((size_t)1 << m) * sizeof(cx<float>) + ((size_t)2 << m) * 8;
    long long w = (long long)((64ull << 20) / per);
    if (w < 1) w = 1;
    return w < batch ? w : batch;
}

// [2k limb spectra | 2k-1 group spectra] of W products (complex float, M each)
// followed by W x N int64 offset corrections
static size_t split_ws_bytes(int m, int k, long long W)
{
    return (size_t)(4 * k - 1) * (size_t)W * ((size_t)1 << m) * sizeof(cx<float>) +
           (size_t)W * ((size_t)2 << m) * sizeof(long long);
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

template <int L, bool SINGLE> static int launch_mid(const SplitArgs& a, long long ctas, cudaStream_t s)
{
    static int done[64] = {0};
    return launch_split(split_mid<L, SINGLE>, done, a, ctas, s);
}
template <int L> static int launch_fwd0(const SplitArgs& a, long long ctas, cudaStream_t s)
{
    static int done[64] = {0};
    return launch_split(split_fwd0<L>, done, a, ctas, s);
}
template <int L> static int launch_inv0(const SplitArgs& a, long long ctas, cudaStream_t s)
{
    static int done[64] = {0};
    return launch_split(split_inv0<L>, done, a, ctas, s);
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
    if (non_negative && input_bits > 30) return GPUFFT_ERROR_INVALID_VALUE;

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
    A.K = non_negative ? (1LL << (input_bits - 1)) : 0;

    long long W = split_wave(m, k, batch);
    const size_t need1 = split_ws_bytes(m, k, 1);
    if (!ws || ws_bytes < need1) return GPUFFT_ERROR_WORKSPACE;
    if (split_ws_bytes(m, k, W) > ws_bytes) W = (long long)(ws_bytes / need1);
    if (max_err)
    {
        cudaError_t e = cudaMemsetAsync(max_err, 0, sizeof(unsigned), s);
        if (e != cudaSuccess) return set_cuda_error(e);
    }
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
        A.offs = nullptr;
        if (A.K)
        {
            A.offs = reinterpret_cast<long long*>(A.group + (size_t)(2 * k - 1) * wv * M);
            split_offsets<<<(unsigned)wv, OFF_THREADS, 0, s>>>(A, n_power);
            const int st = check_launch();
            if (st) return st;
        }
        if (m <= EBITS)
        {
            A.geo = PassGeo{};
            A.geo.m = m;
            const long long ctas = (wv * M + ECTA - 1) / ECTA;
            int st = dispatch_int<1, EBITS>(m, [&]<int LL>() { return launch_mid<LL, true>(A, ctas, s); });
            if (st) return st;
            continue;
        }
        long long ctas = 0;
        const int L0 = p.L[0];
        A.geo = pass_geo(p, 0, m, 0, 2 * wv, &ctas);
        int st = dispatch_int<1, 9>(L0, [&]<int LL>() { return launch_fwd0<LL>(A, ctas, s); });
        if (st) return st;
        A.geo = pass_geo(p, 1, m, 0, wv, &ctas);
        st = launch_mid<EBITS, false>(A, ctas, s);
        if (st) return st;
        A.geo = pass_geo(p, 0, m, 0, wv, &ctas);
        st = dispatch_int<1, 9>(L0, [&]<int LL>() { return launch_inv0<LL>(A, ctas, s); });
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
