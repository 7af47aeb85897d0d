// gpufft-b200: the CTA-level transform engine.
//
// Mathematics. GPU-FFT's transforms are radix-2 decimation-in-time stages over
// a twiddle table stored in bit-reversed order (reference fft.cu:11-152 for
// Cooley-Tukey, 154-260 for Gentleman-Sande). For a length M = 2^m transform,
// stage s pairs element i with i + M/2^(s+1) and multiplies by
//     table[g]                  (cyclic,     X^N - 1)
//     table[2^s + g]            (negacyclic, X^N + 1)      (fft.cu:67-74)
// where g = i / (M / 2^s) is the stage-s group of i. The engine computes exactly
// these butterflies with the caller's table values, so results agree with the
// reference up to FMA contraction, but it reorganises them for Blackwell:
//
//  * A CTA owns E = 4096 elements and runs L consecutive stages on them ("a
//    pass"); a transform of 2^m points needs one pass per 12 stages (one HBM
//    read + one HBM write each) instead of the reference's 2-4 launches of 512
//    elements.
//  * Inside a pass each thread holds 16 elements in registers and runs up to 4
//    stages ("a round") as a radix-16 register network; between rounds the CTA
//    re-distributes elements through a padded shared-memory transpose.
//  * Element placement inside the CTA uses a 12-bit local index e. The pass's
//    L "q bits" (which element of a closed butterfly sub-network) occupy e-bits
//    [QOFF, QOFF+L); the other bits number sub-networks that share the pass
//    (columns of a strided pass, or whole short transforms of a batch). A
//    round's 16 registers are the 4 e-bits of an aligned window W; the thread
//    index supplies the other 8 bits in order, which keeps global accesses
//    coalesced and the shared-memory transposes bank-conflict free.
//  * Everything about a pass's shape (QOFF, L, round windows, register -> e
//    offsets) is a compile-time constant: the rounds are straight-line code and
//    all per-element address arithmetic folds to constant offsets.
#pragma once

#include "gf_common.cuh"

namespace gfb
{

constexpr int EBITS = 12;
constexpr int ECTA = 1 << EBITS; // elements per CTA
constexpr int RPT = 16;          // elements per thread
constexpr int NTHR = ECTA / RPT; // threads per CTA
constexpr int SMEM_ELEMS = ECTA + ECTA / 16;

__host__ __device__ constexpr int spad(int e) { return e + (e >> 4); }

// e of register 0 for thread t when the register window starts at e-bit W.
template <int W> __device__ __forceinline__ int e_base(int t)
{
    return (t & ((1 << W) - 1)) | ((t >> W) << (W + 4));
}
// spad(e_base + (r << W)) - spad(e_base), for every r in [0, 16)
template <int W> constexpr int sstride() { return W == 0 ? 1 : (1 << W) + (1 << (W - 4)); }

// Round schedule of q bits [QOFF, QOFF+L), cut at multiples of 4. Round i of a
// forward pass handles the i-th most significant piece, of an inverse pass the
// i-th least significant one.
template <int QOFF, int L> struct Sched
{
    static constexpr int first = QOFF;
    static constexpr int end = QOFF + L;
    static constexpr int n = ((end - 1) >> 2) - (first >> 2) + 1;
    static constexpr int alo(int i) { return 4 * ((first >> 2) + i) > first ? 4 * ((first >> 2) + i) : first; }
    static constexpr int ahi(int i) { return 4 * ((first >> 2) + i + 1) < end ? 4 * ((first >> 2) + i + 1) : end; }
    static constexpr int lo(int i, bool fwd) { return fwd ? alo(n - 1 - i) : alo(i); }
    static constexpr int hi(int i, bool fwd) { return fwd ? ahi(n - 1 - i) : ahi(i); }
    static constexpr int win(int i, bool fwd) { return lo(i, fwd) & ~3; }
};

// Runtime part of the twiddle index: stage-s0 group of the CTA and the table mode.
struct TwCtx
{
    long long g; // group of this CTA's sub-networks at the first stage of the pass
    int s0;      // first stage of the pass
    int neg;     // negacyclic (X^N+1) twiddle indexing
    int vec = 0; // float tables on a 16-byte boundary: load twiddle pairs as float4
};

// Twiddle-table base suitable for paired (16-byte) loads.
template <typename T> __device__ __forceinline__ int tw_vec_ok(const cx<T>* tw)
{
    return sizeof(T) == 4 && (reinterpret_cast<uintptr_t>(tw) & 15) == 0;
}

// One round: radix-2^RB network on window bits [A, A+RB) of the registers, for
// NA arrays that share placement and twiddles. All twiddles of the round are
// loaded first so their latencies overlap.
template <typename T, bool FWD, int QOFF, int L, int LO, int HI, int NA>
__device__ __forceinline__ void round_net(cx<T> (&x)[NA][RPT], const cx<T>* __restrict__ tw, const TwCtx& c,
                                          int t)
{
    constexpr int W = LO & ~3, A = LO - W, RB = HI - LO;
    const int eb = e_base<W>(t);
    constexpr int qmask = (1 << L) - 1;
    cx<T> w[15];
#pragma unroll
    for (int k = 0; k < RB; k++)
    {
        const int pb = FWD ? (A + RB - 1 - k) : (A + k);
        const int nhi = A + RB - 1 - pb;
        const int u = QOFF + L - 1 - (W + pb);
        const long long gbase = (c.g << u) + (c.neg ? (1LL << (c.s0 + u)) : 0LL);
        // The 2^nhi twiddles of this step are consecutive table entries
        // idx0 + h, and idx0 is a multiple of 2^nhi: the register bits above
        // pb are the lowest bits of the group index, and e_base leaves the
        // window's bits clear.
        const cx<T>* p0 = tw + gbase + (((eb >> QOFF) & qmask) >> (L - u));
        cx<T>* wk = w + (1 << nhi) - 1;
        if (sizeof(T) == 4 && nhi >= 1 && c.vec)
        {
#pragma unroll
            for (int h = 0; h < (1 << nhi); h += 2)
            {
                const float4 v = __ldg(reinterpret_cast<const float4*>(p0 + h));
                wk[h] = mk<T>((T)v.x, (T)v.y);
                wk[h + 1] = mk<T>((T)v.z, (T)v.w);
            }
        }
        else
        {
#pragma unroll
            for (int h = 0; h < (1 << nhi); h++) wk[h] = ldg<T>(p0 + h);
        }
    }
#pragma unroll
    for (int k = 0; k < RB; k++)
    {
        const int pb = FWD ? (A + RB - 1 - k) : (A + k);
        const int nhi = A + RB - 1 - pb;
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            if (r & (1 << pb)) continue;
            const int h = (r >> (pb + 1)) & ((1 << nhi) - 1);
            const cx<T> wt = w[(1 << nhi) - 1 + h];
#pragma unroll
            for (int a = 0; a < NA; a++)
            {
                if (FWD)
                    ct_bfly<T>(x[a][r], x[a][r | (1 << pb)], wt);
                else
                    gs_bfly<T>(x[a][r], x[a][r | (1 << pb)], wt);
            }
        }
    }
}

// Move NA register arrays from window WA to window WB through shared memory
// (sm holds NA buffers of SMEM_ELEMS, or is reused array by array when SHARED).
template <typename T, int WA, int WB, int NA>
__device__ __forceinline__ void transpose(cx<T> (&x)[NA][RPT], cx<T>* sm, int t)
{
    const int sa = spad(e_base<WA>(t));
    const int sb = spad(e_base<WB>(t));
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
        for (int r = 0; r < RPT; r++) sm[a * SMEM_ELEMS + sa + r * sstride<WA>()] = x[a][r];
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
        for (int r = 0; r < RPT; r++) x[a][r] = sm[a * SMEM_ELEMS + sb + r * sstride<WB>()];
}

// All rounds of a pass on registers loaded in window Sched::win(0, FWD); the
// data ends in window Sched::win(n-1, FWD).
template <typename T, bool FWD, int QOFF, int L, int NA, int I = 0>
__device__ __forceinline__ void run_rounds(cx<T> (&x)[NA][RPT], cx<T>* sm, const cx<T>* __restrict__ tw,
                                           const TwCtx& c, int t)
{
    using S = Sched<QOFF, L>;
    if constexpr (I < S::n)
    {
        if constexpr (I > 0) transpose<T, S::win(I - 1, FWD), S::win(I, FWD), NA>(x, sm, t);
        round_net<T, FWD, QOFF, L, S::lo(I, FWD), S::hi(I, FWD), NA>(x, tw, c, t);
        run_rounds<T, FWD, QOFF, L, NA, I + 1>(x, sm, tw, c, t);
    }
}

// Compile-time dispatch of a runtime value v in [LO, HI] to F::template run<v>().
template <int LO, int HI, typename F> __host__ int dispatch_int(int v, F&& f)
{
    if constexpr (LO <= HI)
    {
        if (v == LO) return f.template operator()<LO>();
        return dispatch_int<LO + 1, HI>(v, static_cast<F&&>(f));
    }
    else
    {
        return GPUFFT_ERROR_INVALID_VALUE;
    }
}

} // namespace gfb
