// gpufft-b200: the contiguous 12-stage pass of a 4096-point tile spread over a
// thread-block cluster, for launches with few tiles.
//
// A 4096-point tile on one CTA (the engine's pass) keeps one SM busy per tile:
// a product of one N = 2^16 polynomial has 8 tiles, so 140 of the 148 SMs
// idle while 8 run the 12 stages back to back. Here a cluster of CL_CTAS = 8
// CTAs (64 threads, 512 points each) shares the tile through distributed
// shared memory:
//
//   X layout   CTA c, thread t holds tile points e = 64 c + t + 512 k (k < 8):
//              the three stages on e-bits 11..9 (the bits that cross CTAs)
//              are one radix-8 network in registers;
//   exchange   register k goes to CTA k's shared memory (DSMEM stores), one
//              cluster barrier;
//   Y layouts  CTA c holds the 512 consecutive points e = 512 c + l; the nine
//              stages on l-bits 8..0 are three radix-8 rounds with padded
//              shared-memory transposes between them (Y1: l = t + 64 r,
//              Y2: l = (t & 7) + 64 (t >> 3) + 8 r, Y3: l = 8 t + r).
//
// The inverse runs the same layouts backwards (Y3, Y2, Y1, exchange, X). Every
// butterfly is the engine's: stage u of the pass on e-bit q = 11 - u pairs e
// with e + 2^q and uses table[(g << u) + (e >> (q + 1))], g the tile's group at
// the pass's first stage, so the values are bit-identical to the one-CTA
// pass. Global loads and stores are coalesced in every mode (X layout: 32
// consecutive points per warp and register; Y1 likewise inside the CTA's 512).
//
// Modes: CLM_FWD   one forward pass (complex in, complex out, optional scale);
//        CLM_INV   one inverse pass (complex or pointwise-product in);
//        CLM_FUSED forward of two operands, product, inverse (the fused
//                  product's middle pass, operands and result in the workspace).
//
// Smaller tiles: a whole transform of 2^LT points, LT = 10 or 11, runs on a
// cluster of 2^(LT-9) CTAs of 512 points. The X layout then holds the cross-
// CTA e-bits 9..LT-1 on the upper register bits and two (LT = 11) or four
// (LT = 10) low positions on the lower ones: register k = (h, lo) of thread t
// in CTA c holds e = 64 c + t + 64 2^(LT-9) lo + 512 h. The Y layouts are
// unchanged. Transforms of at most 4096 points are a single pass, so their
// loads and stores may also be the FFNT fold (rows of 2M reals, f_j + i
// f_{j+M}, times the twist), the linear-product load (rows of M reals) and the
// unfold (scale, untwist, real and imaginary parts to f_j and f_{j+M}).
#pragma once

#include "gf_engine.cuh"

#include <atomic>

#include <cooperative_groups.h>

namespace gfb
{

namespace cgx = cooperative_groups;

constexpr int CL_CTAS = 8;                  // CTAs per tile (one cluster)
constexpr int CL_THREADS = 64;              // threads per CTA
constexpr int CL_PTS = ECTA / CL_CTAS;      // 512 points per CTA
constexpr int CL_SMEM = CL_PTS + CL_PTS / 8; // padded: one slot per 8

enum ClusterMode
{
    CLM_FWD = 0,
    CLM_INV = 1,
    CLM_FUSED = 2
};

enum ClusterLoad
{
    CL_IN_CPX = 0,  // complex rows of M
    CL_IN_FOLD = 1, // single pass: rows of 2M reals, (f_j + i f_{j+M}) twist_j
    CL_IN_LIN = 2   // single pass: rows of M reals, f_j twist_j
};
enum ClusterStore
{
    CL_OUT_CPX = 0,   // complex rows of M (times scale when do_scale)
    CL_OUT_UNFOLD = 1 // single pass: v = x scale untwist_j, rows of 2M reals: v.x at j, v.y at j + M
};

template <typename T> struct ClusterArgs
{
    const cx<T>* in;   // operand rows of M (CLM_FUSED: the first operand)
    const cx<T>* in2;  // CLM_FUSED: rows of the second operand
    cx<T>* out;        // result rows of M (may alias in)
    const cx<T>* table;     // forward twiddles (CLM_FWD, CLM_FUSED)
    const cx<T>* inv_table; // inverse twiddles (CLM_INV, CLM_FUSED)
    cx<T> scale;
    long long prod_off; // CLM_INV with prod: element offset of the second factor
    int m;              // log2 transform length (> 12, or the tile's LT for a single pass)
    int neg;            // negacyclic (X^N+1) twiddle indexing: table[2^s + ...]
    int prod;           // CLM_INV: load in[i] * in[i + prod_off]
    int do_scale;       // multiply the stored values by scale
    // single pass (m = LT) over real rows
    int in_kind;           // ClusterLoad (CLM_FWD, CLM_FUSED)
    int out_kind;          // ClusterStore (CLM_INV, CLM_FUSED)
    const T* rin;          // CL_IN_FOLD / CL_IN_LIN: rows of the (first) operand
    const T* rin2;         // CLM_FUSED: rows of the second operand
    T* rout;               // CL_OUT_UNFOLD: rows of 2M reals
    const cx<T>* twist;    // CL_IN_FOLD / CL_IN_LIN
    const cx<T>* untwist;  // CL_OUT_UNFOLD
};

__device__ __forceinline__ int cpad(int l) { return l + (l >> 3); }

// The first cluster barrier only has to show that every CTA of the cluster is
// running (its shared memory exists) before DSMEM stores reach it: a relaxed
// arrive right after the global loads are issued, and the wait just before the
// first remote store, so the barrier overlaps the load latency. Every thread
// arrives and waits once.
__device__ __forceinline__ void cl_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cl_wait() { asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory"); }

// Local point of register r of thread t in layout Y1 / Y2 / Y3.
template <int Y> __device__ __forceinline__ int ypos(int t, int r)
{
    if constexpr (Y == 1) return t + 64 * r;
    else if constexpr (Y == 2) return (t & 7) + ((t >> 3) << 6) + 8 * r;
    else return 8 * t + r;
}

// Radix-8 round on the e-bits [P, P+3) held by register bits [0, 3); ebase is
// the thread's e with those bits clear; g is the tile's group plus, for
// negacyclic indexing, 2^s0 (table[2^(s0+u) + (g << u) + ...]).
template <typename T, bool FWD, int P, int NA, int LT = 12>
__device__ __forceinline__ void cl_round(cx<T> (&x)[NA][8], int ebase, const cx<T>* __restrict__ tab, long long g)
{
#pragma unroll
    for (int k = 0; k < 3; k++)
    {
        const int i = FWD ? 2 - k : k; // register bit of this stage
        const int q = P + i;           // its e-bit
        const int u = LT - 1 - q;      // its stage within the pass
        // e >> (q+1) of the lower point of a pair = (ebase >> (q+1)) + (r >> (i+1))
        const cx<T>* tw = tab + (g << u) + (ebase >> (q + 1));
        cx<T> w[4];
#pragma unroll
        for (int h = 0; h < (4 >> i); h++) w[h] = ldg<T>(tw + h);
#pragma unroll
        for (int r = 0; r < 8; r++)
        {
            if (r & (1 << i)) continue;
            const cx<T> wt = w[r >> (i + 1)];
#pragma unroll
            for (int a = 0; a < NA; a++)
            {
                if (FWD)
                    ct_bfly<T>(x[a][r], x[a][r | (1 << i)], wt);
                else
                    gs_bfly<T>(x[a][r], x[a][r | (1 << i)], wt);
            }
        }
    }
}

// The cross-CTA stages in the X layout: e-bits 9..LT-1 on register bits
// LOB..2 (LOB = 12 - LT); e >> (q + 1) of a pair's lower point is h >> (i + 1)
// for the stage on bit i of h, since the other parts of e are below 512.
template <typename T, bool FWD, int LT, int NA>
__device__ __forceinline__ void cl_xround(cx<T> (&x)[NA][8], const cx<T>* __restrict__ tab, long long g)
{
    constexpr int LC = LT - 9, LOB = 3 - LC;
#pragma unroll
    for (int k = 0; k < LC; k++)
    {
        const int i = FWD ? LC - 1 - k : k; // bit of h
        const int u = LT - 1 - (9 + i);     // stage of e-bit 9 + i within the pass
        const cx<T>* tw = tab + (g << u);
        cx<T> w[4];
#pragma unroll
        for (int h = 0; h < ((1 << LC) >> (i + 1)); h++) w[h] = ldg<T>(tw + h);
#pragma unroll
        for (int r = 0; r < 8; r++)
        {
            if (r & (1 << (LOB + i))) continue;
            const cx<T> wt = w[(r >> LOB) >> (i + 1)];
#pragma unroll
            for (int a = 0; a < NA; a++)
            {
                if (FWD)
                    ct_bfly<T>(x[a][r], x[a][r | (1 << (LOB + i))], wt);
                else
                    gs_bfly<T>(x[a][r], x[a][r | (1 << (LOB + i))], wt);
            }
        }
    }
}

// Registers from layout YA to layout YB through this CTA's buffers (one per array).
template <typename T, int YA, int YB, int NA>
__device__ __forceinline__ void cl_transpose(cx<T> (&x)[NA][8], cx<T> (*buf)[CL_SMEM], int t)
{
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
        for (int r = 0; r < 8; r++) buf[a][cpad(ypos<YA>(t, r))] = x[a][r];
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
        for (int r = 0; r < 8; r++) x[a][r] = buf[a][cpad(ypos<YB>(t, r))];
}

template <typename T, int MODE, int LT>
__global__ void __cluster_dims__(1 << (LT - 9), 1, 1) __launch_bounds__(CL_THREADS) cluster_pass_kernel(const ClusterArgs<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    constexpr int NA = MODE == CLM_FUSED ? 2 : 1;
    constexpr int LC = LT - 9, CT = 1 << LC, LOB = 3 - LC;
    __shared__ __align__(16) cx<T> ybuf[NA][CL_SMEM];
    __shared__ __align__(16) cx<T> xbuf[1][CL_SMEM];
    cgx::cluster_group cluster = cgx::this_cluster();
    const int c = (int)cluster.block_rank();
    const int t = threadIdx.x;
    const long long tile = blockIdx.x / CT;
    const int m = a.m;
    // group at the pass's first stage s0 = m - LT (plus 2^s0 for negacyclic indexing)
    const long long g = (tile & ((1LL << (m - LT)) - 1)) + (a.neg ? (1LL << (m - LT)) : 0LL);
    const long long row = tile << LT; // = batch entry * M + g * 2^LT
    const int ey = 512 * c;           // Y layouts: e = ey + l
    // X layout: register k holds e = xl(k) + 512 (k >> LOB), xl(k) its local point in CTA k >> LOB
    auto xl = [&](int k) { return 64 * c + t + 64 * CT * (k & ((1 << LOB) - 1)); };

    cx<T> x[NA][8];
    if constexpr (MODE == CLM_INV)
    {
        // inverse: the first stages are on the lowest bits; load in Y1 (coalesced)
#pragma unroll
        for (int r = 0; r < 8; r++)
        {
            const long long i = row + ey + ypos<1>(t, r);
            x[0][r] = a.prod ? cmul<T>(a.in[i], a.in[i + a.prod_off]) : a.in[i];
        }
        cl_arrive_relaxed();
        cl_transpose<T, 1, 3, 1>(x, ybuf, t);
    }
    else
    {
        if (a.in_kind == CL_IN_CPX)
        {
#pragma unroll
            for (int k = 0; k < 8; k++)
            {
                const int e = xl(k) + 512 * (k >> LOB);
                x[0][k] = a.in[row + e];
                if constexpr (NA == 2) x[NA - 1][k] = a.in2[row + e];
            }
        }
        else
        {
            // a single pass over real rows: the tile is batch entry `tile`, j = e
            const long long M = 1LL << m;
            const bool fold = a.in_kind == CL_IN_FOLD;
            const long long stride = fold ? 2 * M : M;
            T re[NA][8], im[NA][8];
            cx<T> tw[8];
#pragma unroll
            for (int k = 0; k < 8; k++)
            {
                const int e = xl(k) + 512 * (k >> LOB);
                tw[k] = ldg<T>(a.twist + e);
#pragma unroll
                for (int q = 0; q < NA; q++)
                {
                    const T* p = (q == 0 ? a.rin : a.rin2) + tile * stride + e;
                    re[q][k] = ld_stream(p);
                    im[q][k] = fold ? ld_stream(p + M) : T(0);
                }
            }
#pragma unroll
            for (int k = 0; k < 8; k++)
#pragma unroll
                for (int q = 0; q < NA; q++) x[q][k] = cmul<T>(mk<T>(re[q][k], im[q][k]), tw[k]);
        }
        cl_arrive_relaxed();
        cl_xround<T, true, LT, NA>(x, a.table, g);
        cl_wait(); // every CTA of the cluster runs: its shared memory can be written
        // X -> Y1: register k to CTA k >> LOB at its local point
#pragma unroll
        for (int k = 0; k < 8; k++)
        {
#pragma unroll
            for (int q = 0; q < NA; q++)
            {
                cx<T>* dst = cluster.map_shared_rank(&ybuf[q][0], k >> LOB);
                dst[cpad(xl(k))] = x[q][k];
            }
        }
        cluster.sync();
#pragma unroll
        for (int q = 0; q < NA; q++)
#pragma unroll
            for (int r = 0; r < 8; r++) x[q][r] = ybuf[q][cpad(ypos<1>(t, r))];
        cl_round<T, true, 6, NA, LT>(x, ey + ypos<1>(t, 0), a.table, g);
        cl_transpose<T, 1, 2, NA>(x, ybuf, t);
        cl_round<T, true, 3, NA, LT>(x, ey + ypos<2>(t, 0), a.table, g);
        cl_transpose<T, 2, 3, NA>(x, ybuf, t);
        cl_round<T, true, 0, NA, LT>(x, ey + ypos<3>(t, 0), a.table, g);
        if constexpr (MODE == CLM_FWD)
        {
            cl_transpose<T, 3, 1, 1>(x, ybuf, t);
#pragma unroll
            for (int r = 0; r < 8; r++)
            {
                const cx<T> v = a.do_scale ? cmul<T>(x[0][r], a.scale) : x[0][r];
                a.out[row + ey + ypos<1>(t, r)] = v;
            }
            return;
        }
        else
        {
#pragma unroll
            for (int r = 0; r < 8; r++) x[0][r] = cmul<T>(x[0][r], x[NA - 1][r]);
        }
    }
    if constexpr (MODE != CLM_FWD)
    {
        cx<T> z[1][8];
#pragma unroll
        for (int r = 0; r < 8; r++) z[0][r] = x[0][r];
        cl_round<T, false, 0, 1, LT>(z, ey + ypos<3>(t, 0), a.inv_table, g);
        cl_transpose<T, 3, 2, 1>(z, ybuf, t);
        cl_round<T, false, 3, 1, LT>(z, ey + ypos<2>(t, 0), a.inv_table, g);
        cl_transpose<T, 2, 1, 1>(z, ybuf, t);
        cl_round<T, false, 6, 1, LT>(z, ey + ypos<1>(t, 0), a.inv_table, g);
        if constexpr (MODE == CLM_INV) cl_wait(); // the first remote store of this mode
        // Y1 -> X: point e = 512 c + t + 64 r belongs to CTA r & (CT - 1), thread t,
        // register (c << LOB) | (r >> LC)
#pragma unroll
        for (int r = 0; r < 8; r++)
        {
            cx<T>* dst = cluster.map_shared_rank(&xbuf[0][0], r & (CT - 1));
            dst[cpad(64 * ((c << LOB) | (r >> LC)) + t)] = z[0][r];
        }
        cluster.sync();
#pragma unroll
        for (int k = 0; k < 8; k++) z[0][k] = xbuf[0][cpad(64 * k + t)];
        cl_xround<T, false, LT, 1>(z, a.inv_table, g);
        if (a.out_kind == CL_OUT_UNFOLD)
        {
            // a single pass: the tile is batch entry `tile`, j = e
            const long long M = 1LL << m;
            T* pc = a.rout + tile * 2 * M;
            cx<T> u[8];
#pragma unroll
            for (int k = 0; k < 8; k++) u[k] = ldg<T>(a.untwist + xl(k) + 512 * (k >> LOB));
#pragma unroll
            for (int k = 0; k < 8; k++)
            {
                const int e = xl(k) + 512 * (k >> LOB);
                const cx<T> v = cmul<T>(cmul<T>(z[0][k], a.scale), u[k]);
                st_stream(pc + e, v.x);
                st_stream(pc + M + e, v.y);
            }
        }
        else
        {
#pragma unroll
            for (int k = 0; k < 8; k++)
            {
                const cx<T> v = a.do_scale ? cmul<T>(z[0][k], a.scale) : z[0][k];
                a.out[row + xl(k) + 512 * (k >> LOB)] = v;
            }
        }
    }
}

// Tiles at or below which the contiguous 12-stage passes run as clusters
// (0: never). Set by gpufft_set_cluster_tiles.
extern std::atomic<int> g_cluster_max_tiles;

inline bool cluster_ok(long long tiles)
{
    // the grid (8 CTAs per tile) must stay within the 2^31 - 1 limit of gridDim.x
    return tiles > 0 && tiles <= g_cluster_max_tiles.load(std::memory_order_relaxed) &&
           tiles <= 0x7fffffffLL / CL_CTAS;
}

// A pass over `tiles` tiles of 2^lt points (lt = 12 for the contiguous pass
// of a longer transform; 10..12 for a single pass of a transform of 2^lt).
template <typename T, int MODE>
static inline int launch_cluster_pass(const ClusterArgs<T>& a, long long tiles, long long rows, cudaStream_t s,
                                      int lt = EBITS)
{
    if (lt < 10 || lt > EBITS || a.m < lt) return GPUFFT_ERROR_INVALID_VALUE;
    if ((a.in_kind != CL_IN_CPX || a.out_kind != CL_OUT_CPX) && a.m != lt) return GPUFFT_ERROR_INVALID_VALUE;
    const long long ctas = tiles << (lt - 9);
    if (tiles <= 0 || ctas > 0x7fffffffLL) return GPUFFT_ERROR_INVALID_VALUE;
    // bytes: every point read once per operand and written once, in its format
    const double pts = (double)rows * (double)(1LL << a.m);
    const double cb = sizeof(cx<T>);
    const double in_b = a.in_kind == CL_IN_CPX ? cb : (a.in_kind == CL_IN_FOLD ? cb : cb / 2);
    const double nin = MODE == CLM_FUSED ? 2.0 : ((MODE == CLM_INV && a.prod) ? 2.0 : 1.0);
    GF_TRACE(tr, pts * (nin * (MODE == CLM_INV ? cb : in_b) + cb), s, "cluster_pass<%s,%s,L%d>",
             sizeof(T) == 4 ? "f32" : "f64", MODE == CLM_FWD ? "fwd" : (MODE == CLM_INV ? "inv" : "fused"), lt);
    if (lt == 12) return launch_k(cluster_pass_kernel<T, MODE, 12>, dim3((unsigned)ctas), dim3(CL_THREADS), 0, s, a);
    if (lt == 11) return launch_k(cluster_pass_kernel<T, MODE, 11>, dim3((unsigned)ctas), dim3(CL_THREADS), 0, s, a);
    return launch_k(cluster_pass_kernel<T, MODE, 10>, dim3((unsigned)ctas), dim3(CL_THREADS), 0, s, a);
}

} // namespace gfb
