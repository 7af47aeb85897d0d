// gpufft-b200: the split product's middle on 2048-point tiles held in shared
// memory (rings N = 2^14 .. 2^16, up to six limbs).
//
// The split product (gf_split.cuh) transforms 2k limb polynomials, forms 2k-1
// limb-group sums per spectral point and inverse-transforms every group. Each
// transform of M = N/2 points has m = log2 M stages; the first L0 = m - 11 run
// in the column kernels (split_fwd0_col / split_inv0_col), the other eleven on
// contiguous tiles of 2048 points. This kernel runs, for one tile of one
// product, every one of those contiguous stages of all 2k limbs, the group
// sums and the contiguous stages of all 2k-1 groups without leaving the SM:
//
//   slots       2k shared-memory slots of one tile (16 KB each, 160 KB for
//               k = 5, 192 KB for k = 6); limb tile tau is bulk-copied (cp.async.bulk, the TMA
//               unit) from the column kernel's output into slot tau, completed
//               on mbarrier tau;
//   teams       the CTA's 512 threads are four teams of 128 (16 points per
//               thread); a team transforms one limb or group at a time, in
//               place in its slot: eleven stages as three radix-16 register
//               rounds (e-bits [7,11), [3,7), [0,3)) with the slot itself as
//               the transpose buffer, point e at the padded position
//               e + (e >> 4), where every register window is free of bank
//               conflicts and every register's address is a per-thread base
//               plus a compile-time offset (the bulk copy lands unpadded in
//               the slot's first 16 KB, read once by the first round);
//   groups      all 512 threads form G_s = sum_{i+j=s} A_i B_j (+ the centring
//               term) at every point and write G_s over slot s;
//   queue       the CTA is persistent; the inverse items of tile i (the eleven
//               stages of each group in the reverse order, then the group tile
//               to the workspace for split_inv0_col) and the forward items of
//               tile i+1 share one work queue that the teams draw from, so
//               the teams stay busy across the tile boundary; each inverse item
//               starts the bulk copy of the next tile's limb into its slot as
//               soon as its team has read the slot, so loads overlap compute.
//
// HBM traffic per product drops from the five-kernel chain's four passes over
// the limb and group spectra to two (the column kernels' write and read stay).
// Butterflies and twiddle indices are the engine's (table[(T << u) + (e >>
// (11 - u))] at stage L0 + u for tile T), so the spectra equal the engine
// path's up to the order of floating-point operations inside a round.
//
// Waits on the mbarriers are bounded (gf_async.cuh). A team whose wait runs out
// reports it at the next CTA-wide barrier; the CTA then marks the call's error
// report as infinite (not exact), counts the timeout in g_split_wait_timeouts,
// drains its outstanding copies with a bounded wait and returns.
#pragma once

#include <type_traits>

#include "gf_async.cuh"
#include "gf_split.cuh"

namespace gfb
{
namespace stile
{
constexpr int LT = SPLIT_TILE_LT; // log2 points per tile (11)
constexpr int P = 1 << LT; // 2048 points per tile
constexpr int HT = 128;    // threads per team
constexpr int R = P / HT;  // 16 points per thread
constexpr int MAXK = SPLIT_TILE_MAXK; // limb counts whose 2k slots fit in shared memory (5: 10 slots, 170 KB)
constexpr int SLOT = P + P / 16;      // padded slot (2176 points, 17 KB)

// e of register 0 of thread t (0..127) when the registers are the four e-bits
// [W, W+4): the thread supplies the other seven bits in order
template <int W> __device__ __forceinline__ int ebase(int t)
{
    return (t & ((1 << W) - 1)) | ((t >> W) << (W + 4));
}
__device__ __forceinline__ constexpr int ppos(int e) { return e + (e >> 4); }

// Padded slot addresses of a thread's 16 registers in window W:
// ppos(ebase(t) + (r << W)) = ppos(ebase(t)) + off(r), because the window bits
// of ebase are clear and no addition carries across bit 4:
//   W = 7: off = 136 r;  W = 3: off = 8 r + (r >> 1);  W = 0: off = r.
template <int W> struct SlotAddr
{
    int b;
    __device__ __forceinline__ explicit SlotAddr(int t) : b(ppos(ebase<W>(t))) {}
    __device__ __forceinline__ int operator()(int r) const { return b + (r << W) + ((r << W) >> 4); }
};

// Window-0 twiddles of a tile (stages u = 8, 9, 10 on e-bits 2, 1, 0): thread
// t's are table[(T << u) + (16 t >> (11 - u)) + h] for h < 2^(u - 7), i.e.
// pairs (T << (u - 1)) + 2^(u - 8) t + i for i < 2^(u - 8): one pair at u = 8,
// two at u = 9, four at u = 10 -- seven 16-byte pairs, 1792 entries per tile.
// Read straight from the table, a warp's paired loads would stride 64 bytes
// (half of every sector wasted, sixteen cache lines per instruction); staged
// thread-major in shared memory (pair j of thread t at j * 128 + t) each round
// reads them conflict-free. w0_pair(pb) is the first pair index j of the
// stage on e-bit pb.
__device__ __forceinline__ constexpr int w0_pair(int pb) { return pb == 2 ? 0 : (pb == 1 ? 1 : 3); }
constexpr int W0_PAIRS = 7 * HT; // float4 per staged table

// All 512 threads copy the window-0 twiddles of tile T (table `tw`, 16-byte
// aligned when `vec`) into `dst` (W0_PAIRS float4).
__device__ __forceinline__ void stage_w0(float4* dst, const cx<float>* __restrict__ tw, long long T, int tid,
                                         int nthreads, bool vec)
{
    // linear pair p over the three stages: [0, 128) u = 8, [128, 384) u = 9, [384, 896) u = 10
    for (int p = tid; p < W0_PAIRS; p += nthreads)
    {
        int u, q, t, j;
        if (p < 128)
        {
            u = 8, q = p, t = q, j = 0;
        }
        else if (p < 384)
        {
            u = 9, q = p - 128, t = q >> 1, j = 1 + (q & 1);
        }
        else
        {
            u = 10, q = p - 384, t = q >> 2, j = 3 + (q & 3);
        }
        const cx<float>* src = tw + (T << u) + 2 * q;
        float4 v;
        if (vec)
        {
            v = __ldg(reinterpret_cast<const float4*>(src));
        }
        else
        {
            const cx<float> a = ldg<float>(src), b = ldg<float>(src + 1);
            v = make_float4(a.x, a.y, b.x, b.y);
        }
        dst[j * HT + t] = v;
    }
}

// Twiddles of the outer rounds (windows 7 and 3: stages u = 0 .. 7 of the
// tile) use table[(T << u) + i] for i < 2^u only (window 7: all threads the
// same 2^u entries; window 3: thread t the 2^(u-4) entries from i = (t >> 3)
// 2^(u-4)). Staged as entry 2^u + i of a 256-entry buffer, every pair stays
// 16-byte aligned.
constexpr int W37_ENTRIES = 256;

__device__ __forceinline__ void stage_w37(cx<float>* dst, const cx<float>* __restrict__ tw, long long T, int tid,
                                          int nthreads)
{
    for (int idx = tid + 1; idx < W37_ENTRIES; idx += nthreads)
    {
        const int u = 31 - __clz(idx);
        dst[idx] = ldg<float>(tw + (T << u) + (idx - (1 << u)));
    }
}

// One round: the butterflies of e-bits [LO, HI) inside window W. Stage u of the
// tile's eleven (e-bit q = 10 - u) pairs e with e + 2^q and uses
// table[(T << u) + (e >> (q + 1))]; for register r (bit pb of r = q - W clear)
// that is table[base + (r >> (pb + 1))] with base = (T << u) + (eb >> (q + 1)):
// 2^(3 - pb) consecutive entries, loaded first so their latencies overlap.
template <bool FWD, int W, int LO, int HI>
__device__ __forceinline__ void round(cx<float> (&x)[R], const cx<float>* __restrict__ tw, long long T, int eb,
                                      bool vec, const float4* staged = nullptr, int t = 0,
                                      const cx<float>* outer = nullptr)
{
    constexpr int A = LO - W, RB = HI - LO;
    static_assert(A >= 0 && RB >= 1 && A + RB <= 4, "the round's bits lie in its window");
    cx<float> w[15];
#pragma unroll
    for (int k = 0; k < RB; k++)
    {
        const int pb = FWD ? (A + RB - 1 - k) : (A + k);
        const int q = W + pb;
        const int u = LT - 1 - q;
        const int nt = 1 << (3 - pb);
        const cx<float>* p0 = tw + (T << u) + (eb >> (q + 1));
        cx<float>* wk = w + nt - 1;
        if constexpr (W == 7 || W == 3)
        {
            if (outer)
            {
                // entries 2^u + i, i = (eb >> (q + 1)) = 0 (window 7) or (t >> 3) 2^(u-4) (window 3)
                const cx<float>* q0 = outer + (1 << u) + (eb >> (q + 1));
                if (nt >= 2)
                {
#pragma unroll
                    for (int h = 0; h < nt; h += 2)
                    {
                        const float4 v = *reinterpret_cast<const float4*>(q0 + h);
                        wk[h] = mk<float>(v.x, v.y);
                        wk[h + 1] = mk<float>(v.z, v.w);
                    }
                }
                else
                {
                    wk[0] = q0[0];
                }
                continue;
            }
        }
        if constexpr (W == 0 && LO == 0 && HI == 3)
        {
            if (staged)
            {
                // the tile's window-0 twiddles, staged thread-major (see stage_w0)
#pragma unroll
                for (int h = 0; h < nt; h += 2)
                {
                    const float4 v = staged[(w0_pair(pb) + (h >> 1)) * HT + t];
                    wk[h] = mk<float>(v.x, v.y);
                    wk[h + 1] = mk<float>(v.z, v.w);
                }
                continue;
            }
        }
        if (nt >= 2 && vec)
        {
#pragma unroll
            for (int h = 0; h < nt; h += 2)
            {
                const float4 v = __ldg(reinterpret_cast<const float4*>(p0 + h));
                wk[h] = mk<float>(v.x, v.y);
                wk[h + 1] = mk<float>(v.z, v.w);
            }
        }
        else
        {
#pragma unroll
            for (int h = 0; h < nt; h++) wk[h] = ldg<float>(p0 + h);
        }
    }
#pragma unroll
    for (int k = 0; k < RB; k++)
    {
        const int pb = FWD ? (A + RB - 1 - k) : (A + k);
        const int nt = 1 << (3 - pb);
#pragma unroll
        for (int r = 0; r < R; r++)
        {
            if (r & (1 << pb)) continue;
            const cx<float> wt = w[nt - 1 + (r >> (pb + 1))];
            if (FWD)
                ct_bfly<float>(x[r], x[r | (1 << pb)], wt);
            else
                gs_bfly<float>(x[r], x[r | (1 << pb)], wt);
        }
    }
}

template <int W> __device__ __forceinline__ void slot_load(cx<float> (&x)[R], const cx<float>* sl, const SlotAddr<W>& ad)
{
#pragma unroll
    for (int r = 0; r < R; r++) x[r] = sl[ad(r)];
}
template <int W> __device__ __forceinline__ void slot_store(const cx<float> (&x)[R], cx<float>* sl, const SlotAddr<W>& ad)
{
#pragma unroll
    for (int r = 0; r < R; r++) sl[ad(r)] = x[r];
}

constexpr int NTEAM = 6;        // teams of HT threads (768 threads, 80 registers each)
constexpr int NTT = NTEAM * HT; // threads per CTA

// slots, the staged twiddles (window 0, then windows 7 and 3) of the forward
// and of the inverse tile, one mbarrier per slot, the queue counter and the
// teams' items
constexpr size_t smem_bytes(int k)
{
    return (size_t)(2 * k) * SLOT * sizeof(float2) + 2 * (size_t)W0_PAIRS * sizeof(float4) +
           2 * (size_t)W37_ENTRIES * sizeof(float2) + (size_t)(2 * k) * 8 + 64;
}

} // namespace stile

// Timeouts of the tile kernel's bounded waits (read and cleared by
// gpufft_split_wait_timeouts in gf_split_tile.cu, the one file that includes
// this header).
static __device__ unsigned g_split_wait_timeouts;

template <int K>
__global__ void __launch_bounds__(stile::NTT, 1) split_tile_kernel(const SplitArgs a, long long tiles)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    using namespace stile;
    constexpr int NS = 2 * K;     // slots: limbs of A then B
    constexpr int NG = 2 * K - 1; // limb groups
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* slot = reinterpret_cast<cx<float>*>(smraw);
    float4* twf = reinterpret_cast<float4*>(slot + NS * SLOT); // window-0 twiddles of the forward tile
    float4* twi = twf + W0_PAIRS;                             // ... and of the inverse tile
    cx<float>* tof = reinterpret_cast<cx<float>*>(twi + W0_PAIRS); // windows 7 and 3, forward tile
    cx<float>* toi = tof + W37_ENTRIES;                             // ... inverse tile
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(toi + W37_ENTRIES);
    int* ctl = reinterpret_cast<int*>(bar + NS); // [0] queue counter, [4 + team] the team's current item

    const int tid = threadIdx.x;
    const int team = tid >> 7;
    const int t = tid & (HT - 1);
    const int tbar = 1 + team; // the team's named barrier
    const long long M = 1LL << a.geo.m;
    const int lg_tiles = a.geo.m - LT; // log2 tiles per transform
    const long long G = gridDim.x;
    const bool vec = (reinterpret_cast<uintptr_t>(a.roots) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(a.inv_roots) & 15) == 0;
    const SlotAddr<7> a7(t);
    const SlotAddr<3> a3(t);
    const SlotAddr<0> a0(t);

    if (tid == 0)
    {
#pragma unroll
        for (int i = 0; i < NS; i++) mbar_init(&bar[i], 1);
        fence_mbar_init();
        ctl[0] = 0;
    }
    if (blockIdx.x < tiles)
    {
        const long long T0 = (long long)blockIdx.x & ((1LL << lg_tiles) - 1);
        stage_w0(twf, a.roots, T0, tid, NTT, vec);
        stage_w37(tof, a.roots, T0, tid, NTT);
    }
    __syncthreads();

    auto issue = [&](long long tile, int tau) {
        const long long p = tile >> lg_tiles, T = tile & ((1LL << lg_tiles) - 1);
        const cx<float>* src = a.spec + ((long long)tau * a.W + p) * M + (T << LT);
        mbar_arrive_expect_tx(&bar[tau], P * sizeof(float2));
        bulk_g2s(slot + (long long)tau * SLOT, src, P * sizeof(float2), &bar[tau]);
    };

    // The last forward stage of limb tau of `tile`: wait for its copy (bounded),
    // then the eleven stages in place. Returns false (uniformly over the team)
    // when the wait ran out.
    auto forward_item = [&](long long tile, int tau, unsigned parity) -> bool {
        const bool ok = mbar_wait_bounded(&bar[tau], parity);
        if (bar_any(tbar, HT, !ok)) return false;
        const long long T = tile & ((1LL << lg_tiles) - 1);
        cx<float>* sl = slot + tau * SLOT;
        cx<float> x[R];
#pragma unroll
        for (int r = 0; r < R; r++) x[r] = sl[t + (r << 7)]; // unpadded natural order, as copied
        round<true, 7, 7, 11>(x, a.roots, T, ebase<7>(t), vec, nullptr, t, tof);
        bar_named(tbar, HT); // the team has read the natural order
        slot_store<7>(x, sl, a7);
        bar_named(tbar, HT);
        slot_load<3>(x, sl, a3);
        round<true, 3, 3, 7>(x, a.roots, T, ebase<3>(t), vec, nullptr, t, tof);
        slot_store<3>(x, sl, a3); // the positions this thread read
        bar_named(tbar, HT);
        slot_load<0>(x, sl, a0);
        round<true, 0, 0, 3>(x, a.roots, T, ebase<0>(t), vec, twf, t);
        slot_store<0>(x, sl, a0);
        return true;
    };

    // The first inverse stages of group s of `tile`, in place, then the group
    // tile to the workspace; the slot's copy for `next` starts once the team
    // has read it.
    auto inverse_item = [&](long long tile, int s, long long next) {
        const long long p = tile >> lg_tiles, T = tile & ((1LL << lg_tiles) - 1);
        cx<float>* sl = slot + s * SLOT;
        cx<float> x[R];
        slot_load<0>(x, sl, a0);
        round<false, 0, 0, 3>(x, a.inv_roots, T, ebase<0>(t), vec, twi, t);
        slot_store<0>(x, sl, a0);
        bar_named(tbar, HT);
        slot_load<3>(x, sl, a3);
        round<false, 3, 3, 7>(x, a.inv_roots, T, ebase<3>(t), vec, nullptr, t, toi);
        slot_store<3>(x, sl, a3);
        bar_named(tbar, HT);
        slot_load<7>(x, sl, a7);
        bar_named(tbar, HT); // the team has read slot s
        if (next >= 0 && t == 0)
        {
            fence_proxy_async();
            issue(next, s);
        }
        round<false, 7, 7, 11>(x, a.inv_roots, T, ebase<7>(t), vec, nullptr, t, toi);
        cx<float>* dst = a.group + ((long long)s * a.W + p) * M + (T << LT) + t;
#pragma unroll
        for (int r = 0; r < R; r++) dst[r << 7] = x[r];
    };

    // Draw items from the queue until it is empty: items [0, n_inv) are the
    // inverse items of `tile`, the next n_fwd the forward items of `ftile`.
    // Returns false if a forward wait of this team ran out.
    auto run_queue = [&](long long tile, int n_inv, long long ftile, int n_fwd, unsigned fpar,
                         long long next) -> bool {
        bool ok = true;
        for (;;)
        {
            if (t == 0) ctl[4 + team] = atomicAdd(&ctl[0], 1);
            bar_named(tbar, HT);
            const int item = ctl[4 + team];
            bar_named(tbar, HT); // every thread has the item before the leader draws again
            if (item >= n_inv + n_fwd) break;
            if (item < n_inv)
                inverse_item(tile, item, next);
            else if (ok)
                ok = forward_item(ftile, item - n_inv, fpar);
        }
        return ok;
    };

    long long tile = blockIdx.x;
    if (tid == 0)
        for (int tau = 0; tau < NS; tau++) issue(tile, tau);
    bool ok = run_queue(-1, 0, tile, NS, 0u, -1);
    for (unsigned it = 0;; it++)
    {
        // every limb spectrum of `tile` is in its slot (or some team's wait ran out)
        if (__syncthreads_or(ok ? 0 : 1))
        {
            if (tid == 0)
            {
                // all copies of this iteration were issued: drain them (bounded)
                for (int tau = 0; tau < NS; tau++) (void)mbar_wait_bounded(&bar[tau], it & 1);
                atomicAdd(&g_split_wait_timeouts, 1u);
                if (a.max_err) atomicMax(a.max_err, 0x7f800000u); // +inf: the call's result is not certified
            }
            return;
        }
        const long long T = tile & ((1LL << lg_tiles) - 1);
        // ---- group sums at every point, over slots 0 .. NG-1 ----
        {
            const float uscale = (float)(1 << a.ur);
#pragma unroll 1
            for (int e = tid; e < P; e += NTT)
            {
                const int ad = ppos(e);
                cx<float> v[NS];
#pragma unroll
                for (int tau = 0; tau < NS; tau++) v[tau] = slot[tau * SLOT + ad];
                // A_i B_j accumulated with paired fused multiply-adds:
                // (a.x, a.x) (b.x, b.y) + (a.y, a.y) (-b.y, b.x), the pairs formed
                // once per limb
                float2 ax[K], ay[K], bs[K];
#pragma unroll
                for (int l = 0; l < K; l++)
                {
                    ax[l] = make_float2(v[l].x, v[l].x);
                    ay[l] = make_float2(v[l].y, v[l].y);
                    bs[l] = make_float2(-v[K + l].y, v[K + l].x);
                }
                cx<float> acc[NG];
#pragma unroll
                for (int sg = 0; sg < NG; sg++)
                {
                    acc[sg] = mk<float>(0.f, 0.f);
#pragma unroll
                    for (int i2 = 0; i2 < K; i2++)
                        if (sg - i2 >= 0 && sg - i2 < K)
                        {
                            acc[sg] = __ffma2_rn(ax[i2], v[K + sg - i2], acc[sg]);
                            acc[sg] = __ffma2_rn(ay[i2], bs[sg - i2], acc[sg]);
                        }
                }
                if (a.K)
                {
                    // U is stored in the 4096-point-tile permuted order of the table block
                    const long long j = (T << LT) + e;
                    const long long ju = (M > 4096) ? ((j & ~4095LL) | ((j & 4095) >> 4) | ((j & 15) << 8)) : j;
                    const cx<float> u = ldg<float>(a.uspec + ju);
                    cx<float> cen[K];
#pragma unroll
                    for (int l = 0; l < K; l++)
                    {
                        cx<float> ee = cadd<float>(v[l], v[K + l]);
                        if (l < K - 1) ee = cadd<float>(ee, u);
                        cen[l] = cmul<float>(mk<float>(ee.x * uscale, ee.y * uscale), u);
                    }
                    // limb l's term joins group l + uq: one uniform branch, compile-time indices
                    auto add_from = [&](auto q) {
                        constexpr int Q = decltype(q)::value;
#pragma unroll
                        for (int l = 0; l < K; l++)
                            if (l + Q < NG) acc[l + Q] = cadd<float>(acc[l + Q], cen[l]);
                    };
                    static_assert(K <= 6, "the switch below covers uq <= 6");
                    switch (a.uq)
                    {
                    case 0: add_from(std::integral_constant<int, 0>{}); break;
                    case 1: add_from(std::integral_constant<int, 1>{}); break;
                    case 2: add_from(std::integral_constant<int, 2>{}); break;
                    case 3: add_from(std::integral_constant<int, 3>{}); break;
                    case 4: add_from(std::integral_constant<int, 4>{}); break;
                    case 5: add_from(std::integral_constant<int, 5>{}); break;
                    case 6: add_from(std::integral_constant<int, 6>{}); break;
                    default: break;
                    }
                }
#pragma unroll
                for (int sg = 0; sg < NG; sg++) slot[sg * SLOT + ad] = acc[sg];
            }
        }
        const long long next = tile + G;
        const bool has_next = next < tiles;
        // window-0 twiddles: the inverse items of this tile and the forward items
        // of the next (the previous tile's inverse and this tile's forward items
        // are done)
        stage_w0(twi, a.inv_roots, T, tid, NTT, vec);
        stage_w37(toi, a.inv_roots, T, tid, NTT);
        if (has_next)
        {
            stage_w0(twf, a.roots, next & ((1LL << lg_tiles) - 1), tid, NTT, vec);
            stage_w37(tof, a.roots, next & ((1LL << lg_tiles) - 1), tid, NTT);
        }
        if (tid == 0) ctl[0] = 0; // the queue restarts
        __syncthreads();
        // slot NS-1 held a limb only: the next tile's copy can start now
        if (has_next && tid == 0)
        {
            fence_proxy_async();
            issue(next, NS - 1);
        }
        ok = run_queue(tile, NG, next, has_next ? NS : 0, (it + 1) & 1, has_next ? next : -1);
        if (!has_next) break;
        tile = next;
    }
}

} // namespace gfb
