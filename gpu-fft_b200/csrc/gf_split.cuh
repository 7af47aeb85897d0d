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
// Kernels (N > 8192, per wave of products; the workspace size sets the wave):
//   split_fwd0_col / split_fwd0   first forward pass (strided) of the 2k limb
//                polynomials: limb digit extraction, fold and twist in the load
//                (one thread per column when the pass has <= 4 stages, 4096-
//                element tiles otherwise);
//   pass_kernel  contiguous last forward pass of all 2k limb spectra;
//   split_groups the 2k-1 pointwise limb-group sums (plus the centring term);
//   pass_kernel  contiguous first inverse pass of every group;
//   split_inv0_col / split_inv0   last inverse pass (strided) of every group
//                with scale, untwist, unfold, rounding and the int64
//                recombination in registers.
// N <= 8192 runs all of it in one kernel (split_mid<true>).
#pragma once

#include <type_traits>

#include "gf_pass.cuh"

#include <algorithm>
#include <cmath>

namespace gfb
{

constexpr int SPLIT_MAX_LIMBS = 8;

// Balanced signed digits: v = sum_l d_l 2^(w l) with d_l in [-2^(w-1), 2^(w-1))
// for l < k-1 and the top digit d_(k-1) taking what is left. Digit l is read
// directly from V = v + voff, where voff = 2^(w-1) (1 + 2^w + ... + 2^(w(k-2))):
// adding half of every lower digit's range turns the balanced digits into the
// plain base-2^w digits e_l = d_l + 2^(w-1) of V, so
// d_l = ((V >> wl) mod 2^w) - 2^(w-1) for l < k-1, and the top digit is
// V >> w(k-1) (arithmetic shift).
__device__ __forceinline__ int split_digit(long long V, int l, int w, int k)
{
    if (l == k - 1) return (int)(V >> (w * l));
    return (int)((V >> (w * l)) & ((1LL << w) - 1)) - (1 << (w - 1));
}

template <typename T> struct SplitArgsT
{
    const int32_t* a;
    const int32_t* b;
    int64_t* c;
    cx<T>* spec;  // [2k][W][M] limb spectra (operand-major: a limbs then b limbs)
    cx<T>* group; // [2k-1][W][M] group spectra
    const cx<T>* roots;
    const cx<T>* inv_roots;
    const cx<T>* twist;
    const cx<T>* untwist;
    unsigned* max_err; // float bits of the largest pre-rounding error (may be null)
    const cx<T>* uspec; // transform of the all-ones polynomial (table block)
    long long K;       // centring offset subtracted from every coefficient (0: none)
    long long voff;    // split_digit offset minus K: V = x + voff for a raw coefficient x
    long long uucoef;  // K^2 - K S (mod 2^64): exact int64 u*u correction (uu_term)
    int uq, ur;        // K = 2^(w uq + ur): centring term joins groups s = l + uq, scaled 2^ur
    T scale;
    int w, k;
    int dig32; // every V = x + voff fits an int32 and w (k - 1) <= 30: 32-bit digits
    long long W; // products per wave (stride of the workspace)
    long long batch;
    PassGeo geo;
};
using SplitArgs = SplitArgsT<float>;

// Distance of a group value to its nearest integer. Above 2^22 (float) or
// 2^51 (double) every value is (nearly) an integer and the distance no longer
// certifies exactness, so such values report 1.0.
template <typename T> __device__ __forceinline__ float group_error(cx<T> v, T rr, T ri)
{
    const T lim = sizeof(T) == 4 ? (T)4194304.0 : (T)2251799813685248.0; // 2^22, 2^51
    if (fabs(v.x) >= lim || fabs(v.y) >= lim) return 1.0f;
    return (float)fmax(fabs(v.x - rr), fabs(v.y - ri));
}

__device__ __forceinline__ void report_err(unsigned* dst, float e)
{
    if (!dst) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
    if ((threadIdx.x & 31) == 0) atomicMax(dst, __float_as_uint(e));
}

// Non-negative inputs are centred before they are cut into limbs,
// a = a' + K u with u = 1 + X + ... + X^(N-1) and K = 2^(B) (B = input_bits-1),
// so that every limb is balanced (a non-centred top limb would make its group
// values grow like N * mean^2). The product is then
//     a b = a'b' + K (a' u + b' u) + K^2 u u        (mod X^N + 1).
// With K = 2^(w q + r) (0 <= r < w) the middle term is
//     sum_l 2^(w (l + q)) * 2^r (e^a_l + e^b_l) u,
// i.e. 2^r (E^a_l + E^b_l) U joins limb group s = l + q in the frequency domain
// (U = transform of u, part of the native table block), and K^2 u u, whose
// coefficients are K^2 (2k + 2 - N), is added exactly in int64 at the end.
//
// Balanced digits below the top one have mean -1/2 on uniformly spread
// values (the top digit, which takes what is left, has mean ~0), so for
// l < k-1, e^a_l + e^b_l drifts by -u and (e^a_l + e^b_l) u grows like N/2 --
// eight times the group values the limb plan is sized for at N = 2^16. For
// those limbs the frequency domain carries 2^r (E^a_l + E^b_l + U) U instead,
// the transform of a zero-mean integer polynomial times u, and the extra
// sum_{l<k-1} 2^(w (l + q) + r) u u = K S u u (S = sum_{l<k-1} 2^(w l)) is
// subtracted exactly in int64 with the K^2 term: uucoef = K^2 - K S.
template <typename T> __device__ __forceinline__ long long uu_term(const SplitArgsT<T>& a, long long k, long long N)
{
    return (long long)((unsigned long long)a.uucoef * (unsigned long long)(2 * k + 2 - N));
}

// --------------------------------------------------------------------------
// strided first forward pass of every limb polynomial
// --------------------------------------------------------------------------
template <int L> __global__ void __launch_bounds__(NTHR, 2) split_fwd0(const SplitArgs a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
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
    const long long op = tl.b(0) / a.W, p = tl.b(0) - op * a.W;
    const int32_t* src = (op == 0 ? a.a : a.b) + p * 2 * M;
    int vlo[RPT], vhi[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        vlo[r] = __ldcs(src + tl.j(r));
        vhi[r] = __ldcs(src + tl.j(r) + M);
    }
    TwCtx c;
    c.g = tl.g;
    c.s0 = 0;
    c.neg = 0;
    c.vec = tw_vec_ok<float>(a.roots) && tw_vec_ok<float>(a.inv_roots);
    const Tile<L, true, WL> to(a.geo, cta, t);
    for (int l = 0; l < a.k; l++)
    {
        cx<float> x[1][RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const cx<float> f = mk<float>((float)split_digit((long long)vlo[r] + a.voff, l, a.w, a.k),
                                          (float)split_digit((long long)vhi[r] + a.voff, l, a.w, a.k));
            x[0][r] = cmul<float>(f, ldg<float>(a.twist + tl.j(r)));
        }
        if (l > 0) __syncthreads();
        run_rounds<float, true, QOFF, L, 1>(x, sm, a.roots, c, t);
        cx<float>* dst = a.spec + ((op * a.k + l) * a.W + p) * M;
#pragma unroll
        for (int r = 0; r < RPT; r++) dst[to.j(r)] = x[0][r];
    }
}

// --------------------------------------------------------------------------
// contiguous middle: last forward pass of the 2k limb spectra, group sums,
// first inverse pass of every group (SINGLE: whole transforms, int32 in,
// int64 out, everything in this kernel)
// --------------------------------------------------------------------------
template <int L, bool SINGLE, int K> __global__ void __launch_bounds__(NTHR, 2) split_mid(const SplitArgs a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* sm = reinterpret_cast<cx<float>*>(smraw);
    using S = Sched<0, L>;
    constexpr int W0 = S::win(0, true), WM = S::win(S::n - 1, true), WE = S::win(S::n - 1, false);
    constexpr int NG = 2 * K - 1;
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const long long M = 1LL << a.geo.m;

    const Tile<L, false, W0> ti(a.geo, cta, t);
    const Tile<L, false, WM> tm(a.geo, cta, t);
    TwCtx c;
    c.g = ti.g;
    c.s0 = a.geo.s0;
    c.neg = 0;
    c.vec = tw_vec_ok<float>(a.roots) && tw_vec_ok<float>(a.inv_roots);

    // 1. last forward pass (SINGLE: every forward stage, limb extraction in the
    //    load) of every limb spectrum; results parked in a.spec
    for (int tau = 0; tau < 2 * K; tau++)
    {
        const int op = tau / K, l = tau - op * K;
        cx<float> x[1][RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            if (ti.b(r) >= a.batch)
            {
                x[0][r] = mk<float>(0.f, 0.f);
                continue;
            }
            if (SINGLE)
            {
                const int32_t* src = (op == 0 ? a.a : a.b) + ti.b(r) * 2 * M + ti.j(r);
                const long long v0 = (long long)__ldg(src) + a.voff, v1 = (long long)__ldg(src + M) + a.voff;
                const cx<float> f = mk<float>((float)split_digit(v0, l, a.w, K), (float)split_digit(v1, l, a.w, K));
                x[0][r] = cmul<float>(f, ldg<float>(a.twist + ti.j(r)));
            }
            else
            {
                x[0][r] = a.spec[((long long)tau * a.W + ti.b(r)) * M + ti.j(r)];
            }
        }
        if (tau > 0) __syncthreads();
        run_rounds<float, true, 0, L, 1>(x, sm, a.roots, c, t);
#pragma unroll
        for (int r = 0; r < RPT; r++)
            if (tm.b(r) < a.batch) a.spec[((long long)tau * a.W + tm.b(r)) * M + tm.j(r)] = x[0][r];
    }

    // 2. group sums C^_s = sum_{i+j=s} A^_i B^_j (+ the centring term), four
    //    elements at a time so that all 2K limb loads of a chunk are in flight
    //    together; the thread reads only what it wrote in step 1
    const float uscale = (float)(1 << a.ur);
#pragma unroll
    for (int ch = 0; ch < RPT / 4; ch++)
    {
        cx<float> v[2 * K][4], u[4];
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            const int r = 4 * ch + q;
            const bool ok = tm.b(r) < a.batch;
#pragma unroll
            for (int tau = 0; tau < 2 * K; tau++)
                v[tau][q] = ok ? a.spec[((long long)tau * a.W + tm.b(r)) * M + tm.j(r)] : mk<float>(0.f, 0.f);
            u[q] = (a.K && ok) ? ldg<float>(a.uspec + tm.j(r)) : mk<float>(0.f, 0.f);
        }
#pragma unroll
        for (int sg = 0; sg < NG; sg++)
        {
#pragma unroll
            for (int q = 0; q < 4; q++)
            {
                const int r = 4 * ch + q;
                cx<float> acc = mk<float>(0.f, 0.f);
#pragma unroll
                for (int i = 0; i < K; i++)
                    if (sg - i >= 0 && sg - i < K) acc = cadd<float>(acc, cmul<float>(v[i][q], v[K + sg - i][q]));
                const int l = sg - a.uq;
                if (a.K && l >= 0 && l < K)
                {
#pragma unroll
                    for (int ll = 0; ll < K; ll++)
                        if (ll == l)
                        {
                            cx<float> e = cadd<float>(v[ll][q], v[K + ll][q]);
                            if (ll < K - 1) e = cadd<float>(e, u[q]);
                            acc = cadd<float>(acc, cmul<float>(mk<float>(e.x * uscale, e.y * uscale), u[q]));
                        }
                }
                if (tm.b(r) < a.batch) a.group[((long long)sg * a.W + tm.b(r)) * M + tm.j(r)] = acc;
            }
        }
    }

    // 3. first inverse pass of every group (the whole inverse when SINGLE)
    static_assert(WM == S::win(0, false), "the inverse starts where the forward ends");
    long long acc_lo[RPT], acc_hi[RPT];
    float err = 0.f;
#pragma unroll
    for (int r = 0; r < RPT; r++) acc_lo[r] = acc_hi[r] = 0;
    const Tile<L, false, WE> te(a.geo, cta, t);
    for (int sg = 0; sg < NG; sg++)
    {
        cx<float> x[1][RPT];
        cx<float>* grp = a.group + (long long)sg * a.W * M;
#pragma unroll
        for (int r = 0; r < RPT; r++) x[0][r] = (tm.b(r) < a.batch) ? grp[tm.b(r) * M + tm.j(r)] : mk<float>(0.f, 0.f);
        __syncthreads();
        run_rounds<float, false, 0, L, 1>(x, sm, a.inv_roots, c, t);
        if (SINGLE)
        {
            const int sh = a.w * sg;
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                if (te.b(r) >= a.batch) continue;
                const cx<float> v =
                    cmul<float>(cmul<float>(x[0][r], mk<float>(a.scale, 0.f)), ldg<float>(a.untwist + te.j(r)));
                const float rr = rintf(v.x), ri = rintf(v.y);
                err = fmaxf(err, group_error(v, rr, ri));
                acc_lo[r] += (long long)((unsigned long long)(long long)rr << sh);
                acc_hi[r] += (long long)((unsigned long long)(long long)ri << sh);
            }
        }
        else
        {
            // every thread has loaded its group-sg elements before any store:
            // the rounds of an L = 12 pass contain block-wide barriers
            __syncthreads();
#pragma unroll
            for (int r = 0; r < RPT; r++)
                if (te.b(r) < a.batch) grp[te.b(r) * M + te.j(r)] = x[0][r];
        }
    }
    if (SINGLE)
    {
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            if (te.b(r) >= a.batch) continue;
            int64_t* dst = a.c + te.b(r) * 2 * M + te.j(r);
            __stcs(reinterpret_cast<long long*>(dst), acc_lo[r] + uu_term(a, te.j(r), 2 * M));
            __stcs(reinterpret_cast<long long*>(dst + M), acc_hi[r] + uu_term(a, te.j(r) + M, 2 * M));
        }
        report_err(a.max_err, err);
    }
}

// --------------------------------------------------------------------------
// strided last inverse pass of every group, rounding and int64 recombination
// --------------------------------------------------------------------------
template <int L> __global__ void __launch_bounds__(NTHR) split_inv0(const SplitArgs a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
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
    c.vec = tw_vec_ok<float>(a.roots) && tw_vec_ok<float>(a.inv_roots);
    const long long p = ti.b(0);

    long long acc_lo[RPT], acc_hi[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++) acc_lo[r] = acc_hi[r] = 0;
    float err = 0.f;
    for (int s = 0; s <= 2 * (a.k - 1); s++)
    {
        const cx<float>* src = a.group + ((long long)s * a.W + p) * M;
        cx<float> x[1][RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++) x[0][r] = src[ti.j(r)];
        if (s > 0) __syncthreads();
        run_rounds<float, false, QOFF, L, 1>(x, sm, a.inv_roots, c, t);
        const int sh = a.w * s;
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const cx<float> v =
                cmul<float>(cmul<float>(x[0][r], mk<float>(a.scale, 0.f)), ldg<float>(a.untwist + te.j(r)));
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
        __stcs(reinterpret_cast<long long*>(dst + te.j(r)), acc_lo[r] + uu_term(a, te.j(r), 2 * M));
        __stcs(reinterpret_cast<long long*>(dst + te.j(r) + M), acc_hi[r] + uu_term(a, te.j(r) + M, 2 * M));
    }
    report_err(a.max_err, err);
}

// --------------------------------------------------------------------------
// Column kernels for short first/last passes (L0 <= 4 stages, rings up to
// N = 2^17): the stages [0, L0) of a 2^m transform are closed 2^L0-point
// networks on the columns c of the M / 2^L0 x 2^L0 view, j = c + i C
// (C = 2^(m-L0)). One thread owns one column (of one limb, or of one product
// for the inverse) in registers: no shared memory, no barriers, coalesced
// across the warp, and many more threads in flight than 4096-element tiles.
// Stage s pairs i with i + 2^(L0-1-s) and uses table[i >> (L0-s)] -- the same
// butterflies, twiddles and order as the engine's pass, so the values are
// identical.
// --------------------------------------------------------------------------
constexpr int SPLIT_COL_MAX = 4;
// log2 of the tile kernel's tile (gf_split_tile.cuh); its column passes run the
// first / last m - SPLIT_TILE_LT stages
constexpr int SPLIT_TILE_LT = 11;
constexpr int SPLIT_COL_THREADS = 128;

// One thread per column of one operand of one product: the column's 2 x 2^L0
// coefficients and twist factors are loaded once, and the K limbs are peeled
// off in turn (d_l = (V mod 2^w) - 2^(w-1), then V >>= w, the same digits as
// split_digit), each through the column network and stored.
template <typename T, int L0, int K>
__global__ void __launch_bounds__(SPLIT_COL_THREADS) split_fwd0_col(const SplitArgsT<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    constexpr int R = 1 << L0;
    const int m = a.geo.m;
    const long long M = 1LL << m, C = M >> L0;
    const long long idx = (long long)blockIdx.x * SPLIT_COL_THREADS + threadIdx.x;
    // thread order: column fastest, then (operand, product)
    const long long c = idx & (C - 1);
    const long long bb = idx >> (m - L0);
    if (bb >= 2 * a.W) return;
    const long long op = bb >= a.W ? 1 : 0, p = bb - op * a.W;
    const int32_t* src = (op == 0 ? a.a : a.b) + p * 2 * M + c;
    long long v0[R], v1[R];
    cx<T> tw[R];
#pragma unroll
    for (int i = 0; i < R; i++)
    {
        v0[i] = (long long)__ldg(src + i * C) + a.voff;
        v1[i] = (long long)__ldg(src + i * C + M) + a.voff;
        tw[i] = ldg<T>(a.twist + c + i * C);
    }
    const int w = a.w;
    const long long mask = (1LL << w) - 1;
    const int half = 1 << (w - 1);
    cx<T>* dst = a.spec + (op * K * a.W + p) * M + c;
#pragma unroll
    for (int l = 0; l < K; l++)
    {
        cx<T> x[R];
#pragma unroll
        for (int i = 0; i < R; i++)
        {
            int d0, d1;
            if (l < K - 1)
            {
                d0 = (int)(v0[i] & mask) - half;
                d1 = (int)(v1[i] & mask) - half;
                v0[i] >>= w;
                v1[i] >>= w;
            }
            else
            {
                d0 = (int)v0[i];
                d1 = (int)v1[i];
            }
            x[i] = cmul<T>(mk<T>((T)d0, (T)d1), tw[i]);
        }
#pragma unroll
        for (int s = 0; s < L0; s++)
        {
            const int h = 1 << (L0 - 1 - s);
#pragma unroll
            for (int i = 0; i < R; i++)
                if (!(i & h)) ct_bfly<T>(x[i], x[i + h], ldg<T>(a.roots + (i >> (L0 - s))));
        }
        cx<T>* d = dst + (long long)l * a.W * M;
#pragma unroll
        for (int i = 0; i < R; i++) d[i * C] = x[i];
    }
}

// Paired-lane column kernels for 2^L0-point columns (L0 >= 2): lanes l and
// l ^ 16 of a warp share 16 columns, lane half hb = (l >> 4) & 1 holding rows
// i = 2 m + hb (m < 2^(L0-1)). Every stage with span h >= 2 pairs rows of one
// parity and runs in the thread (twiddle table[i >> (L0 - s)] = table[m >>
// (L0 - s - 1)]); the span-1 stage pairs rows 2m and 2m+1 across the two
// lanes through one register exchange (__shfl_xor_sync). Same butterflies,
// twiddles and order as split_fwd0_col / split_inv0_col, so the same values, at
// half the registers per thread.
constexpr int SPLIT_COL2_THREADS = 128; // five CTAs per SM (forward), four (inverse)

__device__ __forceinline__ void prefetch_l2(const void* p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ cx<float> shfl16(cx<float> v)
{
    return mk<float>(__shfl_xor_sync(0xffffffffu, v.x, 16), __shfl_xor_sync(0xffffffffu, v.y, 16));
}

// The float value of a w-bit digit u (< 2^23) minus 2^(w-1): u placed in the
// mantissa of 2^23, then one exact subtraction.
__device__ __forceinline__ float digit_f(unsigned u, float bias) { return __int_as_float((int)(u | 0x4B000000u)) - bias; }

// D32: every V = x + voff fits an int32 (a.dig32), digits in 32-bit arithmetic
template <int L0, int K, bool D32>
__global__ void __launch_bounds__(SPLIT_COL2_THREADS, 4) split_fwd0_col2(const SplitArgs a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    constexpr int R = 1 << L0, H = R / 2;
    // the tile path's column passes only: m = L0 + SPLIT_TILE_LT, all
    // column offsets compile-time
    constexpr int m = L0 + SPLIT_TILE_LT;
    constexpr long long M = 1LL << m, C = M >> L0;
    const long long idx = (long long)blockIdx.x * SPLIT_COL2_THREADS + threadIdx.x;
    const int hb = (int)((idx >> 4) & 1);
    const long long col = ((idx >> 5) << 4) + (idx & 15); // column over all (operand, product)
    const long long c = col & (C - 1);
    const long long bb = col >> (m - L0);
    const bool ok = bb < 2 * a.W; // the grid covers whole warps; every lane joins the exchange
    const long long op = bb >= a.W ? 1 : 0, p = ok ? bb - op * a.W : 0;
    const int32_t* src = (op == 0 ? a.a : a.b) + p * 2 * M + c;
    using V = typename std::conditional<D32, int, long long>::type;
    V v0[H], v1[H];
    cx<float> tw[H];
#pragma unroll
    for (int q = 0; q < H; q++)
    {
        const long long i = 2 * q + hb;
        // out-of-range lanes read product 0 (p = 0 keeps src inside the inputs):
        // their results are never stored, and their exchange partner (lane ^ 16,
        // the same column) is out of range too
        v0[q] = (V)((long long)__ldg(src + i * C) + a.voff);
        v1[q] = (V)((long long)__ldg(src + i * C + M) + a.voff);
        tw[q] = ldg<float>(a.twist + c + i * C);
    }
    // the column's twiddles, the same for every limb: table[0 .. H/2) for the
    // spans >= 2 and, for the span-1 stage, table[q] on half 1 (half 0 sends
    // U unchanged, through a multiplication by 1)
    cx<float> tws[H / 2], t1[H];
    const float sg = hb ? -1.f : 1.f;
#pragma unroll
    for (int q = 0; q < H; q++)
    {
        const cx<float> t = ldg<float>(a.roots + q);
        if (q < H / 2) tws[q] = t;
        t1[q] = hb ? t : mk<float>(1.f, 0.f);
    }
    const int w = a.w;
    const long long mask = (1LL << w) - 1;
    const int half = 1 << (w - 1);
    const float bias = 8388608.f + (float)half; // 2^23 + 2^(w-1)
    cx<float>* dst = a.spec + (op * K * a.W + p) * M + c;
#pragma unroll
    for (int l = 0; l < K; l++)
    {
        cx<float> x[H];
#pragma unroll
        for (int q = 0; q < H; q++)
        {
            float f0, f1;
            if constexpr (D32)
            {
                // 32-bit digits: extract, then convert through the mantissa
                if (l < K - 1)
                {
                    f0 = digit_f(((unsigned)v0[q] >> (w * l)) & (unsigned)mask, bias);
                    f1 = digit_f(((unsigned)v1[q] >> (w * l)) & (unsigned)mask, bias);
                }
                else
                {
                    f0 = (float)(v0[q] >> (w * l));
                    f1 = (float)(v1[q] >> (w * l));
                }
            }
            else
            {
                int d0, d1;
                if (l < K - 1)
                {
                    d0 = (int)(v0[q] & mask) - half;
                    d1 = (int)(v1[q] & mask) - half;
                    v0[q] >>= w;
                    v1[q] >>= w;
                }
                else
                {
                    d0 = (int)v0[q];
                    d1 = (int)v1[q];
                }
                f0 = (float)d0;
                f1 = (float)d1;
            }
            x[q] = cmul<float>(mk<float>(f0, f1), tw[q]);
        }
        // stages s = 0 .. L0-2 (span h = 2^(L0-1-s) >= 2): rows q and q + h/2 of this lane
#pragma unroll
        for (int s = 0; s < L0 - 1; s++)
        {
            const int hh = 1 << (L0 - 2 - s);
#pragma unroll
            for (int q = 0; q < H; q++)
                if (!(q & hh)) ct_bfly<float>(x[q], x[q + hh], tws[q >> (L0 - 1 - s)]);
        }
        // stage L0-1 (span 1): U = row 2q (half 0), V = row 2q+1 (half 1),
        // table[q]: half 1 sends V table[q], half 0 sends U; half 0 keeps the
        // sum, half 1 the difference
#pragma unroll
        for (int q = 0; q < H; q++)
        {
            const cx<float> mine = cmul<float>(x[q], t1[q]);
            const cx<float> other = shfl16(mine);
            x[q] = __ffma2_rn(mine, make_float2(sg, sg), other);
        }
        if (ok)
        {
            cx<float>* d = dst + (long long)l * a.W * M;
#pragma unroll
            for (int q = 0; q < H; q++) d[(2 * q + hb) * C] = x[q];
        }
    }
}

// Round-to-nearest-even of |v| < 2^22 by one addition: v + 1.5 2^23 lands in
// [2^23, 2^24), where the float spacing is 1, and the integer is the low bits
// of the sum's encoding. Larger values are not certified (group_error), so
// their integer does not matter.
constexpr float RND_MAGIC = 12582912.0f; // 1.5 * 2^23
constexpr int RND_MAGIC_BITS = 0x4B400000;

// acc + i 2^sh (mod 2^64) in the form MODE names (the caller picks it once
// per group, sh being uniform): 0 one wide multiply-add (sh <= 30), 1 one add
// to the high word (sh >= 32), 2 a 64-bit shift (sh = 31)
template <int MODE> __device__ __forceinline__ long long add_shifted(long long acc, int i, int sh)
{
    if constexpr (MODE == 0) return acc + (long long)i * (long long)(1 << sh);
    if constexpr (MODE == 1)
        return (long long)((unsigned long long)acc + ((unsigned long long)((unsigned)i << (sh - 32)) << 32));
    return (long long)((unsigned long long)acc + ((unsigned long long)(long long)i << sh));
}

template <int L0, int K> __global__ void __launch_bounds__(SPLIT_COL2_THREADS, 4) split_inv0_col2(const SplitArgs a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    constexpr int R = 1 << L0, H = R / 2;
    // the tile path's column passes only: m = L0 + SPLIT_TILE_LT, all
    // column offsets compile-time
    constexpr int m = L0 + SPLIT_TILE_LT;
    constexpr long long M = 1LL << m, C = M >> L0;
    const long long idx = (long long)blockIdx.x * SPLIT_COL2_THREADS + threadIdx.x;
    const int hb = (int)((idx >> 4) & 1);
    const long long col = ((idx >> 5) << 4) + (idx & 15);
    const long long c = col & (C - 1);
    const long long p0 = col >> (m - L0);
    const bool ok = p0 < a.W;
    const long long p = ok ? p0 : 0;
    cx<float> un[H];
#pragma unroll
    for (int q = 0; q < H; q++)
    {
        const cx<float> u = ldg<float>(a.untwist + c + (2 * q + hb) * C);
        un[q] = mk<float>(u.x * a.scale, u.y * a.scale); // scale folded in: exact, scale is 2^-m
    }
    // the column's twiddles, the same for every group: table[0 .. H) for the
    // span-1 stage (half 1 multiplies its difference; half 0 passes its sum on
    // through a multiplication by 1) and table[0 .. H/2) for the others
    cx<float> t1[H], tw[H / 2];
    const float sg = hb ? -1.f : 1.f;
#pragma unroll
    for (int q = 0; q < H; q++)
    {
        const cx<float> t = ldg<float>(a.inv_roots + q);
        if (q < H / 2) tw[q] = t;
        t1[q] = hb ? t : mk<float>(1.f, 0.f);
    }
    long long acc_lo[H], acc_hi[H];
#pragma unroll
    for (int q = 0; q < H; q++) acc_lo[q] = acc_hi[q] = 0;
    float err = 0.f, big = 0.f;
    const cx<float>* src = a.group + p * M + c + hb * C;
    const long long gstride = a.W * M;
    cx<float> nx[H];
#pragma unroll
    for (int q = 0; q < H; q++) nx[q] = __ldcs(src + 2 * q * C);
    // group s + 1 is loaded into registers while group s is transformed, and
    // group s + 2 is prefetched into L2 (more bytes in flight than the
    // registers could hold)
    if (2 * K - 1 > 1)
    {
#pragma unroll
        for (int q = 0; q < H; q++) prefetch_l2(src + gstride + 2 * q * C);
    }
#pragma unroll 1
    for (int s = 0; s < 2 * K - 1; s++)
    {
        cx<float> x[H];
#pragma unroll
        for (int q = 0; q < H; q++) x[q] = nx[q];
        if (s + 2 < 2 * K - 1)
        {
#pragma unroll
            for (int q = 0; q < H; q++) prefetch_l2(src + (s + 2) * gstride + 2 * q * C);
        }
        if (s + 1 < 2 * K - 1)
        {
#pragma unroll
            for (int q = 0; q < H; q++) nx[q] = __ldcs(src + (s + 1) * gstride + 2 * q * C);
        }
        // stage L0-1 (span 1) first: U = row 2q (half 0), V = row 2q+1 (half 1),
        // table[q]: half 0 keeps U + V, half 1 takes (U - V) table[q]
#pragma unroll
        for (int q = 0; q < H; q++)
        {
            const cx<float> other = shfl16(x[q]);
            x[q] = cmul<float>(__ffma2_rn(x[q], make_float2(sg, sg), other), t1[q]);
        }
        // stages L0-2 .. 0 (span 2^(L0-1-st) >= 2), rows q and q + h/2 of this lane
#pragma unroll
        for (int st = L0 - 2; st >= 0; st--)
        {
            const int hh = 1 << (L0 - 2 - st);
#pragma unroll
            for (int q = 0; q < H; q++)
                if (!(q & hh)) gs_bfly<float>(x[q], x[q + hh], tw[q >> (L0 - 1 - st)]);
        }
        const int sh = a.w * s;
        auto finish = [&](auto mode) {
            constexpr int MODE = decltype(mode)::value;
#pragma unroll
            for (int q = 0; q < H; q++)
            {
                const cx<float> v = cmul<float>(x[q], un[q]);
                const float tr = __fadd_rn(v.x, RND_MAGIC), ti = __fadd_rn(v.y, RND_MAGIC);
                err = fmaxf(err, fmaxf(fabsf(__fsub_rn(v.x, __fsub_rn(tr, RND_MAGIC))),
                                       fabsf(__fsub_rn(v.y, __fsub_rn(ti, RND_MAGIC)))));
                big = fmaxf(big, fmaxf(fabsf(v.x), fabsf(v.y)));
                acc_lo[q] = add_shifted<MODE>(acc_lo[q], __float_as_int(tr) - RND_MAGIC_BITS, sh);
                acc_hi[q] = add_shifted<MODE>(acc_hi[q], __float_as_int(ti) - RND_MAGIC_BITS, sh);
            }
        };
        // one uniform branch per group
        if (sh <= 30)
            finish(std::integral_constant<int, 0>{});
        else if (sh >= 32)
            finish(std::integral_constant<int, 1>{});
        else
            finish(std::integral_constant<int, 2>{});
    }
    if (ok)
    {
        int64_t* dst = a.c + p * 2 * M + c;
#pragma unroll
        for (int q = 0; q < H; q++)
        {
            const long long i = 2 * q + hb;
            const long long j = c + i * C;
            __stcs(reinterpret_cast<long long*>(dst + i * C), acc_lo[q] + uu_term(a, j, 2 * M));
            __stcs(reinterpret_cast<long long*>(dst + i * C + M), acc_hi[q] + uu_term(a, j + M, 2 * M));
        }
    }
    // values of 2^22 or more are not certified (group_error)
    report_err(a.max_err, ok ? (big >= 4194304.0f ? 1.0f : err) : 0.f);
}

// FP32 columns of 8 points fit 128 registers: four CTAs (16 warps) per
// SM keep more group loads in flight.
template <typename T, int L0> constexpr int inv0_col_min_blocks() { return (sizeof(T) == 4 && L0 == 3) ? 4 : 1; }

template <typename T, int L0, int K>
__global__ void __launch_bounds__(SPLIT_COL_THREADS, inv0_col_min_blocks<T, L0>()) split_inv0_col(const SplitArgsT<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    constexpr int R = 1 << L0;
    const int m = a.geo.m;
    const long long M = 1LL << m, C = M >> L0;
    const long long idx = (long long)blockIdx.x * SPLIT_COL_THREADS + threadIdx.x;
    const long long c = idx & (C - 1);
    const long long p0 = idx >> (m - L0);
    // the grid covers W C threads exactly (C is a multiple of the block size);
    // out-of-range threads still reach report_err's warp shuffle
    const bool ok = p0 < a.W;
    const long long p = ok ? p0 : 0;
    cx<T> un[R];
#pragma unroll
    for (int i = 0; i < R; i++)
    {
        const cx<T> u = ldg<T>(a.untwist + c + i * C);
        un[i] = mk<T>(u.x * a.scale, u.y * a.scale); // scale folded in: exact, scale is 2^-m
    }
    long long acc_lo[R], acc_hi[R];
#pragma unroll
    for (int i = 0; i < R; i++) acc_lo[i] = acc_hi[i] = 0;
    float err = 0.f;
    // short columns: group s + 1 is loaded while group s is transformed and
    // rounded (longer ones would spill the second copy)
    constexpr bool PF = R * sizeof(cx<T>) <= 64;
    const cx<T>* src = a.group + p * M + c;
    const long long gstride = a.W * M;
    cx<T> nx[R];
    if constexpr (PF)
    {
#pragma unroll
        for (int i = 0; i < R; i++) nx[i] = __ldcs(src + i * C);
    }
#pragma unroll
    for (int s = 0; s < 2 * K - 1; s++)
    {
        cx<T> x[R];
        if constexpr (PF)
        {
#pragma unroll
            for (int i = 0; i < R; i++) x[i] = nx[i];
            if (s + 1 < 2 * K - 1)
            {
#pragma unroll
                for (int i = 0; i < R; i++) nx[i] = __ldcs(src + (s + 1) * gstride + i * C);
            }
        }
        else
        {
            const cx<T>* g = a.group + ((long long)s * a.W + p) * M + c;
#pragma unroll
            for (int i = 0; i < R; i++) x[i] = __ldcs(g + i * C);
        }
#pragma unroll
        for (int st = L0 - 1; st >= 0; st--)
        {
            const int h = 1 << (L0 - 1 - st);
#pragma unroll
            for (int i = 0; i < R; i++)
                if (!(i & h)) gs_bfly<T>(x[i], x[i + h], ldg<T>(a.inv_roots + (i >> (L0 - st))));
        }
        const int sh = a.w * s;
#pragma unroll
        for (int i = 0; i < R; i++)
        {
            const cx<T> v = cmul<T>(x[i], un[i]);
            const T rr = rint(v.x), ri = rint(v.y);
            err = fmaxf(err, group_error(v, rr, ri));
            acc_lo[i] += (long long)((unsigned long long)(long long)rr << sh);
            acc_hi[i] += (long long)((unsigned long long)(long long)ri << sh);
        }
    }
    int64_t* dst = a.c + p * 2 * M + c;
    if (ok)
    {
#pragma unroll
        for (int i = 0; i < R; i++)
        {
            const long long j = c + i * C;
            __stcs(reinterpret_cast<long long*>(dst + i * C), acc_lo[i] + uu_term(a, j, 2 * M));
            __stcs(reinterpret_cast<long long*>(dst + i * C + M), acc_hi[i] + uu_term(a, j + M, 2 * M));
        }
    }
    report_err(a.max_err, ok ? err : 0.f);
}

constexpr int SPLIT_SINGLE_MAX_LIMBS = 6; // limb counts compiled for rings N <= 8192

// Limb-group sums of a wave (rings N > 8192), one spectral point per thread:
//     G_s[p][j] = sum_{i+l=s} A_i[p][j] B_l[p][j]  (+ 2^ur (A_l + B_l) U[j] for s = l + uq)
// from the limb spectra [2K][W][M] into the group spectra [2K-1][W][M]. All 2K
// loads of a point are independent and coalesced across the warp.
template <typename T, int K> __global__ void __launch_bounds__(256) split_groups(const SplitArgsT<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    const long long M = 1LL << a.geo.m;
    const long long n = a.W * M;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const long long j = idx & (M - 1);
    cx<T> v[2 * K];
#pragma unroll
    for (int t = 0; t < 2 * K; t++) v[t] = __ldcs(a.spec + t * n + idx);
    cx<T> u = mk<T>(T(0), T(0));
    if (a.K) u = ldg<T>(a.uspec + j);
    const T uscale = (T)(1 << a.ur);
#pragma unroll
    for (int s = 0; s < 2 * K - 1; s++)
    {
        cx<T> acc = mk<T>(T(0), T(0));
#pragma unroll
        for (int i = 0; i < K; i++)
            if (s - i >= 0 && s - i < K) acc = cadd<T>(acc, cmul<T>(v[i], v[K + s - i]));
        if (a.K)
        {
#pragma unroll
            for (int l = 0; l < K; l++)
                if (l + a.uq == s)
                {
                    cx<T> e = cadd<T>(v[l], v[K + l]);
                    if (l < K - 1) e = cadd<T>(e, u);
                    acc = cadd<T>(acc, cmul<T>(mk<T>(e.x * uscale, e.y * uscale), u));
                }
        }
        a.group[s * n + idx] = acc;
    }
}

template <typename K> static int launch_split(K* kern, int* done, const SplitArgs& a, long long ctas, cudaStream_t s)
{
    if (ctas <= 0) return GPUFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return GPUFFT_ERROR_INVALID_VALUE;
    const size_t smem = sizeof(cx<float>) * SMEM_ELEMS;
    int st = ensure_smem(kern, smem, done);
    if (st) return st;
    // tiled split kernels: int32 inputs of W products in, int64 outputs, and
    // the spectra of the chain's other side (upper estimate)
    const double M = (double)(1LL << a.geo.m);
    GF_TRACE(tr, (double)a.W * M * (2 * 2 * 4 + 2 * 8 + (4 * a.k - 1) * 8), s, "split_tiled<k%d>", a.k);
    return launch_k(kern, dim3((unsigned)ctas), dim3(NTHR), smem, s, a);
}

template <int L, bool SINGLE, int K> static int launch_mid_k(const SplitArgs& a, long long ctas, cudaStream_t s)
{
    static int done[64] = {0};
    return launch_split(split_mid<L, SINGLE, K>, done, a, ctas, s);
}

// The split product's contiguous stages of every limb and limb group on
// 2^SPLIT_TILE_LT-point tiles held in shared memory (gf_split_tile.cuh), for
// up to SPLIT_TILE_MAXK limbs; compiled in gf_split_tile.cu.
// (SPLIT_TILE_LT is defined with the column kernels above.)
constexpr int SPLIT_TILE_MAXK = 5;
int launch_split_tile(int k, const SplitArgs& a, long long tiles, cudaStream_t s);

// one-kernel products for rings N <= 8192 (transform length 2^L, L = 1..12),
// compiled in separate translation units by L range
int launch_split_single_lo(int L, const SplitArgs& a, long long ctas, cudaStream_t s);  // L 1..6
int launch_split_single_mid(int L, const SplitArgs& a, long long ctas, cudaStream_t s); // L 7..9
int launch_split_single_hi(int L, const SplitArgs& a, long long ctas, cudaStream_t s);  // L 10..12

} // namespace gfb
