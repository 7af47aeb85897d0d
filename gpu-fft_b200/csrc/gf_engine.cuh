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
//    pass"); a transform of 2^m points needs ceil-ish(m / 12) passes (one HBM
//    read + one HBM write each) instead of the reference's 2-4 launches of 512
//    elements.
//  * Inside a pass each thread holds 16 elements in registers and runs up to
//    4 stages ("a round") as a radix-16 register network; between rounds the
//    CTA re-distributes elements through a padded shared-memory transpose.
//  * Element placement inside the CTA uses a 12-bit local index e. The pass's
//    L "q bits" (which element of a closed butterfly sub-network) occupy
//    e-bits [qoff, qoff+L); the remaining bits number sub-networks that share
//    the pass (columns of a strided pass, or whole short transforms of a batch).
//    A round's 16 registers are the 4 e-bits of an aligned window; the thread
//    index supplies the other 8 bits in order, which keeps global accesses
//    coalesced and the shared-memory transposes bank-conflict free.
#pragma once

#include "gf_common.cuh"

namespace gfb
{

constexpr int EBITS = 12;
constexpr int ECTA = 1 << EBITS; // elements per CTA
constexpr int RPT = 16;          // elements per thread
constexpr int NTHR = ECTA / RPT; // threads per CTA
constexpr int SMEM_ELEMS = ECTA + ECTA / 16;

__device__ __forceinline__ int spad(int e) { return e + (e >> 4); }

// e-index of register r for thread t when the register window starts at e-bit wlo.
__device__ __forceinline__ int e_of(int t, int wlo, int r)
{
    return (t & ((1 << wlo) - 1)) | (r << wlo) | ((t >> wlo) << (wlo + 4));
}

// Geometry of one pass (stages [s0, s0+L) of a 2^m transform).
struct PassGeo
{
    int m;        // log2 transform length
    int s0;       // first stage
    int L;        // number of stages (q bits)
    int qoff;     // e-bit of q bit 0
    int contig;   // 1: CTA covers ECTA consecutive transform elements
    int cols_log; // strided: log2 of columns per CTA
    int neg;      // negacyclic (X^N+1) twiddle indexing
    int pad_;
};

// Round schedule: q bits [qoff, qoff+L) cut at multiples of 4.
struct Rounds
{
    int n;
    int lo[4], hi[4];
};

__device__ __forceinline__ Rounds make_rounds(int qoff, int L, bool fwd)
{
    Rounds R;
    int tmp_lo[4], tmp_hi[4], k = 0;
    int b = qoff, end = qoff + L;
    while (b < end)
    {
        int nb = ((b >> 2) + 1) << 2;
        if (nb > end) nb = end;
        tmp_lo[k] = b;
        tmp_hi[k] = nb;
        k++;
        b = nb;
    }
    R.n = k;
    for (int i = 0; i < k; i++)
    {
        int src = fwd ? (k - 1 - i) : i; // forward: most significant bits first
        R.lo[i] = tmp_lo[src];
        R.hi[i] = tmp_hi[src];
    }
    return R;
}

// Twiddle-index context for one CTA.
struct TwCtx
{
    int qoff, L, qmask, s0, neg;
    long long g; // stage-s0 group of this CTA's sub-networks
};

// One round: radix-2^RB network on window bits [A, A+RB) of the 16 registers.
template <typename T, bool FWD, int A, int RB>
__device__ __forceinline__ void round_net(cx<T> (&x)[RPT], const cx<T>* __restrict__ tw,
                                          const TwCtx& c, int ebase, int wlo)
{
#pragma unroll
    for (int k = 0; k < RB; k++)
    {
        const int pb = FWD ? (A + RB - 1 - k) : (A + k); // window bit paired this stage
        const int nhi = A + RB - 1 - pb;                 // round bits above it
        const int p = wlo + pb;                          // e-bit
        const int u = c.qoff + c.L - 1 - p;              // stage inside the pass
        const long long gbase = (c.g << u) + (c.neg ? (1LL << (c.s0 + u)) : 0LL);
#pragma unroll
        for (int h = 0; h < (1 << nhi); h++)
        {
            const int rrep = h << (pb + 1);
            const int e = ebase | (rrep << wlo);
            const int q = (e >> c.qoff) & c.qmask;
            const cx<T> w = ldg<T>(tw + gbase + (q >> (c.L - u)));
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                if (r & (1 << pb)) continue;
                if (((r >> (pb + 1)) & ((1 << nhi) - 1)) != h) continue;
                if (FWD)
                    ct_bfly<T>(x[r], x[r | (1 << pb)], w);
                else
                    gs_bfly<T>(x[r], x[r | (1 << pb)], w);
            }
        }
    }
}

template <typename T, bool FWD>
__device__ __forceinline__ void run_round(cx<T> (&x)[RPT], const cx<T>* __restrict__ tw,
                                          const TwCtx& c, int ebase, int wlo, int a, int rb)
{
    switch ((a << 3) | rb)
    {
    case (0 << 3) | 1: round_net<T, FWD, 0, 1>(x, tw, c, ebase, wlo); break;
    case (0 << 3) | 2: round_net<T, FWD, 0, 2>(x, tw, c, ebase, wlo); break;
    case (0 << 3) | 3: round_net<T, FWD, 0, 3>(x, tw, c, ebase, wlo); break;
    case (0 << 3) | 4: round_net<T, FWD, 0, 4>(x, tw, c, ebase, wlo); break;
    case (1 << 3) | 1: round_net<T, FWD, 1, 1>(x, tw, c, ebase, wlo); break;
    case (1 << 3) | 2: round_net<T, FWD, 1, 2>(x, tw, c, ebase, wlo); break;
    case (1 << 3) | 3: round_net<T, FWD, 1, 3>(x, tw, c, ebase, wlo); break;
    case (2 << 3) | 1: round_net<T, FWD, 2, 1>(x, tw, c, ebase, wlo); break;
    case (2 << 3) | 2: round_net<T, FWD, 2, 2>(x, tw, c, ebase, wlo); break;
    case (3 << 3) | 1: round_net<T, FWD, 3, 1>(x, tw, c, ebase, wlo); break;
    default: break;
    }
}

// Move the thread's 16 registers from window wa to window wb through shared memory.
template <typename T>
__device__ __forceinline__ void transpose(cx<T> (&x)[RPT], cx<T>* sm, int t, int wa, int wb)
{
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPT; r++) sm[spad(e_of(t, wa, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPT; r++) x[r] = sm[spad(e_of(t, wb, r))];
}

// Run every round of a pass on registers already loaded in the first round's
// window; returns the window of the last round (where the data now sits).
template <typename T, bool FWD>
__device__ __forceinline__ int run_pass_rounds(cx<T> (&x)[RPT], cx<T>* sm, const cx<T>* __restrict__ tw,
                                               const TwCtx& c, const Rounds& R, int t)
{
    int wcur = R.lo[0] & ~3;
    for (int i = 0; i < R.n; i++)
    {
        const int wlo = R.lo[i] & ~3;
        if (wlo != wcur)
        {
            transpose<T>(x, sm, t, wcur, wlo);
            wcur = wlo;
        }
        run_round<T, FWD>(x, tw, c, e_of(t, wlo, 0), wlo, R.lo[i] - wlo, R.hi[i] - R.lo[i]);
    }
    return wcur;
}

// ---------------------------------------------------------------------------
// Two arrays through the same rounds (the two operands of a product share the
// element placement, the twiddles and the index arithmetic).
// ---------------------------------------------------------------------------
template <typename T, bool FWD, int A, int RB>
__device__ __forceinline__ void round_net2(cx<T> (&x)[RPT], cx<T> (&y)[RPT], const cx<T>* __restrict__ tw,
                                           const TwCtx& c, int ebase, int wlo)
{
#pragma unroll
    for (int k = 0; k < RB; k++)
    {
        const int pb = FWD ? (A + RB - 1 - k) : (A + k);
        const int nhi = A + RB - 1 - pb;
        const int p = wlo + pb;
        const int u = c.qoff + c.L - 1 - p;
        const long long gbase = (c.g << u) + (c.neg ? (1LL << (c.s0 + u)) : 0LL);
#pragma unroll
        for (int h = 0; h < (1 << nhi); h++)
        {
            const int rrep = h << (pb + 1);
            const int e = ebase | (rrep << wlo);
            const int q = (e >> c.qoff) & c.qmask;
            const cx<T> w = ldg<T>(tw + gbase + (q >> (c.L - u)));
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                if (r & (1 << pb)) continue;
                if (((r >> (pb + 1)) & ((1 << nhi) - 1)) != h) continue;
                if (FWD)
                {
                    ct_bfly<T>(x[r], x[r | (1 << pb)], w);
                    ct_bfly<T>(y[r], y[r | (1 << pb)], w);
                }
                else
                {
                    gs_bfly<T>(x[r], x[r | (1 << pb)], w);
                    gs_bfly<T>(y[r], y[r | (1 << pb)], w);
                }
            }
        }
    }
}

template <typename T, bool FWD>
__device__ __forceinline__ void run_round2(cx<T> (&x)[RPT], cx<T> (&y)[RPT], const cx<T>* __restrict__ tw,
                                           const TwCtx& c, int ebase, int wlo, int a, int rb)
{
    switch ((a << 3) | rb)
    {
    case (0 << 3) | 1: round_net2<T, FWD, 0, 1>(x, y, tw, c, ebase, wlo); break;
    case (0 << 3) | 2: round_net2<T, FWD, 0, 2>(x, y, tw, c, ebase, wlo); break;
    case (0 << 3) | 3: round_net2<T, FWD, 0, 3>(x, y, tw, c, ebase, wlo); break;
    case (0 << 3) | 4: round_net2<T, FWD, 0, 4>(x, y, tw, c, ebase, wlo); break;
    case (1 << 3) | 1: round_net2<T, FWD, 1, 1>(x, y, tw, c, ebase, wlo); break;
    case (1 << 3) | 2: round_net2<T, FWD, 1, 2>(x, y, tw, c, ebase, wlo); break;
    case (1 << 3) | 3: round_net2<T, FWD, 1, 3>(x, y, tw, c, ebase, wlo); break;
    case (2 << 3) | 1: round_net2<T, FWD, 2, 1>(x, y, tw, c, ebase, wlo); break;
    case (2 << 3) | 2: round_net2<T, FWD, 2, 2>(x, y, tw, c, ebase, wlo); break;
    case (3 << 3) | 1: round_net2<T, FWD, 3, 1>(x, y, tw, c, ebase, wlo); break;
    default: break;
    }
}

template <typename T>
__device__ __forceinline__ void transpose2(cx<T> (&x)[RPT], cx<T> (&y)[RPT], cx<T>* sx, cx<T>* sy, int t, int wa,
                                           int wb)
{
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        const int s = spad(e_of(t, wa, r));
        sx[s] = x[r];
        sy[s] = y[r];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        const int s = spad(e_of(t, wb, r));
        x[r] = sx[s];
        y[r] = sy[s];
    }
}

template <typename T, bool FWD>
__device__ __forceinline__ int run_pass_rounds2(cx<T> (&x)[RPT], cx<T> (&y)[RPT], cx<T>* sx, cx<T>* sy,
                                                const cx<T>* __restrict__ tw, const TwCtx& c, const Rounds& R,
                                                int t)
{
    int wcur = R.lo[0] & ~3;
    for (int i = 0; i < R.n; i++)
    {
        const int wlo = R.lo[i] & ~3;
        if (wlo != wcur)
        {
            transpose2<T>(x, y, sx, sy, t, wcur, wlo);
            wcur = wlo;
        }
        run_round2<T, FWD>(x, y, tw, c, e_of(t, wlo, 0), wlo, R.lo[i] - wlo, R.hi[i] - R.lo[i]);
    }
    return wcur;
}

} // namespace gfb
