// gpufft-b200: the FP64 fused product's middle pass (the last 12 forward stages
// of both operands, their pointwise product and the first 12 inverse stages of
// a 4096-point tile) on 512 threads of 8 points per operand.
//
// The engine's form of this pass (fused_body with 256 threads x 16 points per
// operand) needs 255 registers in double precision, so one CTA of 8 warps runs
// per SM and the FP64 pipe waits on loads. Here a thread holds 8 points of each
// operand: the 12 stages run as four radix-8 register rounds (e-bits [9,12),
// [6,9), [3,6), [0,3) forward; the reverse order inverse) with three padded
// shared-memory transposes between them, at about 110 registers, so the CTA
// has 16 warps. Register window W holds e-bits [W, W+3) (e = ebase(t) + (r <<
// W), the thread's nine bits filling the others in order); point e sits at the
// padded position e + (e >> 3), which every window addresses without bank
// conflicts (a quarter-warp's 16-byte accesses land in eight distinct 16-byte
// bank groups) and with one per-thread base plus compile-time offsets.
//
// Butterflies and twiddle indices are the engine's: stage u of the pass (e-bit
// 11 - u) pairs e with e + 2^(11-u) and uses table[(g << u) + (e >> (12 - u))]
// for the tile's group g, A and B sharing every twiddle load. It runs on the
// native tables only (gpufft_ffnt_make_tables_*), whose odd entries are exact
// quarter turns of their even neighbours, so half the twiddles are loaded and
// the other half rotated -- the same values, half the loads.
#pragma once

#include "gf_fused.cuh"

namespace gfb
{
namespace r8
{
constexpr int THREADS = 512;
constexpr int RP = 8;                     // points per thread and operand
constexpr int BUF = ECTA + ECTA / 8;      // padded transpose buffer (4608 points)

template <int W> __device__ __forceinline__ int ebase(int t)
{
    return (t & ((1 << W) - 1)) | ((t >> W) << (W + 3));
}
__device__ __forceinline__ constexpr int ppos(int e) { return e + (e >> 3); }
// ppos(ebase + (r << W)) - ppos(ebase): the window bits of ebase are clear
template <int W> __device__ __forceinline__ constexpr int poff(int r) { return (r << W) + ((r << W) >> 3); }

// One radix-8 round on the e-bits [W, W+3) of NA arrays. Stage u = 11 - q of
// e-bit q = W + pb: table[(g << u) + (eb >> (q + 1)) + (r >> (pb + 1))].
template <typename T, bool FWD, int W, int NA>
__device__ __forceinline__ void round8(cx<T> (&x)[NA][RP], const cx<T>* __restrict__ tw, long long g, int eb)
{
    cx<T> w[7];
#pragma unroll
    for (int k = 0; k < 3; k++)
    {
        const int pb = FWD ? 2 - k : k;
        const int q = W + pb;
        const int u = EBITS - 1 - q;
        const int nt = 1 << (2 - pb);
        const cx<T>* p0 = tw + (g << u) + (eb >> (q + 1));
        // the native tables store entry 2j+1 as exactly i (forward) or -i
        // (inverse) times entry 2j: load the even entries, rotate for the odd
#pragma unroll
        for (int h = 0; h < nt; h += 2)
        {
            const cx<T> e = ldg<T>(p0 + h);
            w[nt - 1 + h] = e;
            if (nt > 1) w[nt + h] = FWD ? mk<T>(-e.y, e.x) : mk<T>(e.y, -e.x);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
    {
        const int pb = FWD ? 2 - k : k;
        const int nt = 1 << (2 - pb);
#pragma unroll
        for (int r = 0; r < RP; r++)
        {
            if (r & (1 << pb)) continue;
            const cx<T> wt = w[nt - 1 + (r >> (pb + 1))];
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

// Registers from window WA to window WB through the padded buffers (one per array).
template <typename T, int WA, int WB, int NA>
__device__ __forceinline__ void transpose8(cx<T> (&x)[NA][RP], cx<T>* sm, int t)
{
    const int ba = ppos(ebase<WA>(t)), bb = ppos(ebase<WB>(t));
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
        for (int r = 0; r < RP; r++) sm[a * BUF + ba + poff<WA>(r)] = x[a][r];
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
        for (int r = 0; r < RP; r++) x[a][r] = sm[a * BUF + bb + poff<WB>(r)];
}

constexpr size_t smem_bytes(size_t cxb) { return 2 * (size_t)BUF * cxb; }
} // namespace r8

// The middle pass of a two-pass product (M > 4096): tile `blockIdx.x` of the
// workspace (A rows, then B rows, W products each); the product's first 12
// inverse stages overwrite A's tile.
template <typename T> __global__ void __launch_bounds__(r8::THREADS, 1) fused_r8_kernel(const FusedArgs<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    using namespace r8;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
    const int t = threadIdx.x;
    const long long tile = blockIdx.x;
    const long long M = 1LL << a.geo.m;
    const long long g = tile & ((1LL << a.geo.s0) - 1); // the tile's group at the pass's first stage
    const cx<T>* pa = a.ws + (tile << EBITS);
    const cx<T>* pb = pa + a.batch * M;
    const bool ok = (tile << EBITS) < a.batch * M; // the grid covers whole tiles of the batch

    cx<T> x[2][RP];
    // window 9: e = t + 512 r (coalesced)
#pragma unroll
    for (int r = 0; r < RP; r++)
    {
        x[0][r] = ok ? pa[t + (r << 9)] : mk<T>(T(0), T(0));
        x[1][r] = ok ? pb[t + (r << 9)] : mk<T>(T(0), T(0));
    }
    round8<T, true, 9, 2>(x, a.roots, g, ebase<9>(t));
    transpose8<T, 9, 6, 2>(x, sm, t);
    round8<T, true, 6, 2>(x, a.roots, g, ebase<6>(t));
    transpose8<T, 6, 3, 2>(x, sm, t);
    round8<T, true, 3, 2>(x, a.roots, g, ebase<3>(t));
    transpose8<T, 3, 0, 2>(x, sm, t);
    round8<T, true, 0, 2>(x, a.roots, g, ebase<0>(t));
    cx<T> z[1][RP];
#pragma unroll
    for (int r = 0; r < RP; r++) z[0][r] = cmul<T>(x[0][r], x[1][r]);
    round8<T, false, 0, 1>(z, a.inv_roots, g, ebase<0>(t));
    transpose8<T, 0, 3, 1>(z, sm, t);
    round8<T, false, 3, 1>(z, a.inv_roots, g, ebase<3>(t));
    transpose8<T, 3, 6, 1>(z, sm, t);
    round8<T, false, 6, 1>(z, a.inv_roots, g, ebase<6>(t));
    transpose8<T, 6, 9, 1>(z, sm, t);
    round8<T, false, 9, 1>(z, a.inv_roots, g, ebase<9>(t));
    if (ok)
    {
        cx<T>* pz = a.ws + (tile << EBITS);
#pragma unroll
        for (int r = 0; r < RP; r++) pz[t + (r << 9)] = z[0][r];
    }
}

} // namespace gfb
