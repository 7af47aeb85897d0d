// gpufft-b200: GPU_Special_FFT (the reference's "special FFT" for the CKKS
// canonical embedding, fft.cu:727-1007, launch tables fft.cuh:388-500).
//
// The reference's network on vectors of 2^m complex, in place: the span
// t = 2^p pairs i and i + t (i the lower element of its group of 2t) with the
// twiddle table[t + (i mod t)] -- indexed by the position inside the group,
// where the FFT/FFNT stages index by the group. The forward runs the spans
// 1, 2, ..., 2^(m-1) with Cooley-Tukey butterflies; the inverse runs them
// back down with Gentleman-Sande butterflies and multiplies every value by
// cfg.mod_inverse at the end.
//
// B200 form: the spans are cut into passes of at most four; a pass is one
// thread per column (the 2^L points base + k 2^p0 of one lower offset below
// the pass's first span p0), in registers, with no barrier. Neighbouring
// threads take neighbouring lower offsets, so passes with p0 >= 5 are
// coalesced as they stand; the pass of spans 1..8 (p0 = 0), whose columns are
// 16 consecutive points, stages 2048-point runs through padded shared memory
// so that its global loads and stores stay coalesced too.
//
// Launches with few 4096-point tiles (small batches, vectors of >= 4096
// points) instead run the twelve smallest spans of every aligned tile as one
// pass on an 8-CTA thread-block cluster (the layouts and DSMEM exchange of
// gf_cluster.cuh): span 2^q of the tile is e-bit q, and its twiddle depends on
// the bits below q, table[2^q + (e mod 2^q)].
#include "gf_cluster.cuh"

namespace gfb
{

template <typename T> struct SpecialArgs
{
    cx<T>* data;
    const cx<T>* table;
    cx<T> scale;
    long long batch;
    int m, p0, do_scale;
};

constexpr int SPECIAL_THREADS = 128;

// The 2^L - 1 twiddles of a column at lower offset lo: span 2^(p0+s) uses
// table[2^(p0+s) + lo + (k mod 2^s) 2^p0], stored at w[2^s - 1 + (k mod 2^s)].
// Loaded before the data so that their latency overlaps the data loads.
template <typename T, int L>
__device__ __forceinline__ void special_twiddles(cx<T> (&w)[(1 << L) - 1], const SpecialArgs<T>& a, long long lo)
{
#pragma unroll
    for (int s = 0; s < L; s++)
    {
        const cx<T>* tw = a.table + (1LL << (a.p0 + s)) + lo;
#pragma unroll
        for (int k = 0; k < (1 << s); k++) w[(1 << s) - 1 + k] = ldg<T>(tw + ((long long)k << a.p0));
    }
}

template <typename T, int L, bool FWD>
__device__ __forceinline__ void special_network(cx<T> (&x)[1 << L], const cx<T> (&w)[(1 << L) - 1],
                                                const SpecialArgs<T>& a)
{
#pragma unroll
    for (int q = 0; q < L; q++)
    {
        const int s = FWD ? q : L - 1 - q; // span 2^(p0 + s)
        const int h = 1 << s;
#pragma unroll
        for (int k = 0; k < (1 << L); k++)
        {
            if (k & h) continue;
            const cx<T> wt = w[h - 1 + (k & (h - 1))];
            if (FWD)
                ct_bfly<T>(x[k], x[k + h], wt);
            else
                gs_bfly<T>(x[k], x[k + h], wt);
        }
    }
    if (a.do_scale)
    {
#pragma unroll
        for (int k = 0; k < (1 << L); k++) x[k] = cmul<T>(x[k], a.scale);
    }
}

// A pass of spans 2^p0 .. 2^(p0+L-1) (p0 > 0), one column per thread.
template <typename T, int L, bool FWD>
__global__ void __launch_bounds__(SPECIAL_THREADS) special_col_kernel(const SpecialArgs<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    constexpr int R = 1 << L;
    const long long idx = (long long)blockIdx.x * SPECIAL_THREADS + threadIdx.x;
    const int m = a.m, p0 = a.p0;
    const long long lo = idx & ((1LL << p0) - 1);
    const long long rest = idx >> p0;
    const long long hi = rest & ((1LL << (m - p0 - L)) - 1);
    const long long b = rest >> (m - p0 - L);
    if (b >= a.batch) return;
    cx<T>* p = a.data + (b << m) + (hi << (p0 + L)) + lo;
    cx<T> w[R - 1];
    special_twiddles<T, L>(w, a, lo);
    cx<T> x[R];
#pragma unroll
    for (int k = 0; k < R; k++) x[k] = p[(long long)k << p0];
    special_network<T, L, FWD>(x, w, a);
#pragma unroll
    for (int k = 0; k < R; k++) p[(long long)k << p0] = x[k];
}

// The pass of the smallest spans (p0 = 0): every column is 2^L consecutive
// points. A CTA moves a run of SPECIAL_THREADS * 2^L points through shared
// memory (padded one slot per 16 so that the column reads are conflict-free).
template <typename T, int L, bool FWD>
__global__ void __launch_bounds__(SPECIAL_THREADS) special_first_kernel(const SpecialArgs<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    constexpr int R = 1 << L;
    constexpr int RUN = SPECIAL_THREADS * R;
    __shared__ cx<T> sm[RUN + RUN / 16];
    const int t = threadIdx.x;
    const long long run0 = (long long)blockIdx.x * RUN; // first point of the run (flat over the batch)
    // the run lies in one vector or covers whole vectors (both are powers of
    // two, and a vector holds whole columns); the last run may be partial
    const long long rem = (a.batch << a.m) - run0;
    if (rem <= 0) return;
    cx<T> w[R - 1];
    special_twiddles<T, L>(w, a, 0);
    cx<T>* g = a.data + run0;
#pragma unroll
    for (int k = 0; k < R; k++)
    {
        const int e = k * SPECIAL_THREADS + t;
        sm[e + (e >> 4)] = e < rem ? g[e] : mk<T>(T(0), T(0));
    }
    __syncthreads();
    cx<T> x[R];
#pragma unroll
    for (int k = 0; k < R; k++)
    {
        const int e = t * R + k;
        x[k] = sm[e + (e >> 4)];
    }
    special_network<T, L, FWD>(x, w, a);
#pragma unroll
    for (int k = 0; k < R; k++)
    {
        const int e = t * R + k;
        sm[e + (e >> 4)] = x[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < R; k++)
    {
        const int e = k * SPECIAL_THREADS + t;
        if (e < rem) g[e] = sm[e + (e >> 4)];
    }
}

// Radix-8 round of the special network on the e-bits [P, P+3) held by register
// bits [0, 3): the forward runs them upwards with Cooley-Tukey butterflies, the
// inverse downwards with Gentleman-Sande. ebase is the thread's e with those
// bits clear; the lower point of a pair at e-bit q = P + i uses
// table[2^q + (ebase mod 2^P) + ((r mod 2^i) << P)].
template <typename T, bool FWD, int P>
__device__ __forceinline__ void special_cl_round(cx<T> (&x)[1][8], int ebase, const cx<T>* __restrict__ tab)
{
#pragma unroll
    for (int k = 0; k < 3; k++)
    {
        const int i = FWD ? k : 2 - k;
        const cx<T>* tw = tab + (1 << (P + i)) + (ebase & ((1 << P) - 1));
        cx<T> w[4];
#pragma unroll
        for (int h = 0; h < (1 << i); h++) w[h] = ldg<T>(tw + (h << P));
#pragma unroll
        for (int r = 0; r < 8; r++)
        {
            if (r & (1 << i)) continue;
            const cx<T> wt = w[r & ((1 << i) - 1)];
            if (FWD)
                ct_bfly<T>(x[0][r], x[0][r | (1 << i)], wt);
            else
                gs_bfly<T>(x[0][r], x[0][r | (1 << i)], wt);
        }
    }
}

// Spans 2^0 .. 2^11 of every 4096-point tile (vectors of 2^m >= 4096 points),
// one tile per cluster. Forward: Y3, Y2, Y1 rounds, exchange, X round;
// inverse: the reverse, scaled by mod_inverse when it ends the transform.
template <typename T, bool FWD>
__global__ void __cluster_dims__(CL_CTAS, 1, 1) __launch_bounds__(CL_THREADS) special_cluster_kernel(const SpecialArgs<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    __shared__ __align__(16) cx<T> ybuf[1][CL_SMEM];
    __shared__ __align__(16) cx<T> xbuf[1][CL_SMEM];
    cgx::cluster_group cluster = cgx::this_cluster();
    const int c = (int)cluster.block_rank();
    const int t = threadIdx.x;
    const long long row = (long long)(blockIdx.x / CL_CTAS) << EBITS; // tiles are aligned inside vectors
    const int ex = 64 * c + t; // X layout: e = ex + 512 k
    const int ey = 512 * c;    // Y layouts: e = ey + l
    cx<T> x[1][8];
    if constexpr (FWD)
    {
#pragma unroll
        for (int r = 0; r < 8; r++) x[0][r] = a.data[row + ey + ypos<1>(t, r)];
        cl_arrive_relaxed();
        cl_transpose<T, 1, 3, 1>(x, ybuf, t);
        special_cl_round<T, true, 0>(x, ey + ypos<3>(t, 0), a.table);
        cl_transpose<T, 3, 2, 1>(x, ybuf, t);
        special_cl_round<T, true, 3>(x, ey + ypos<2>(t, 0), a.table);
        cl_transpose<T, 2, 1, 1>(x, ybuf, t);
        special_cl_round<T, true, 6>(x, ey + ypos<1>(t, 0), a.table);
        cl_wait(); // every CTA of the cluster runs: its shared memory can be written
        // Y1 -> X: point e = 512 c + t + 64 r belongs to CTA r, thread t, register c
#pragma unroll
        for (int r = 0; r < 8; r++)
        {
            cx<T>* dst = cluster.map_shared_rank(&xbuf[0][0], r);
            dst[cpad(64 * c + t)] = x[0][r];
        }
        cluster.sync();
#pragma unroll
        for (int k = 0; k < 8; k++) x[0][k] = xbuf[0][cpad(64 * k + t)];
        special_cl_round<T, true, 9>(x, ex, a.table);
#pragma unroll
        for (int k = 0; k < 8; k++) a.data[row + ex + 512 * k] = x[0][k];
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 8; k++) x[0][k] = a.data[row + ex + 512 * k];
        cl_arrive_relaxed();
        special_cl_round<T, false, 9>(x, ex, a.table);
        cl_wait(); // every CTA of the cluster runs: its shared memory can be written
        // X -> Y1: register k to CTA k at local point ex
#pragma unroll
        for (int k = 0; k < 8; k++)
        {
            cx<T>* dst = cluster.map_shared_rank(&ybuf[0][0], k);
            dst[cpad(ex)] = x[0][k];
        }
        cluster.sync();
#pragma unroll
        for (int r = 0; r < 8; r++) x[0][r] = ybuf[0][cpad(ypos<1>(t, r))];
        special_cl_round<T, false, 6>(x, ey + ypos<1>(t, 0), a.table);
        cl_transpose<T, 1, 2, 1>(x, ybuf, t);
        special_cl_round<T, false, 3>(x, ey + ypos<2>(t, 0), a.table);
        cl_transpose<T, 2, 3, 1>(x, ybuf, t);
        special_cl_round<T, false, 0>(x, ey + ypos<3>(t, 0), a.table);
        cl_transpose<T, 3, 1, 1>(x, ybuf, t);
#pragma unroll
        for (int r = 0; r < 8; r++)
        {
            const cx<T> v = a.do_scale ? cmul<T>(x[0][r], a.scale) : x[0][r];
            a.data[row + ey + ypos<1>(t, r)] = v;
        }
    }
}

template <typename T, bool FWD> static int launch_special_cluster(const SpecialArgs<T>& a, cudaStream_t s)
{
    const long long tiles = (a.batch << a.m) >> EBITS;
    GF_TRACE(tr, (double)(a.batch << a.m) * 2 * sizeof(cx<T>), s, "special_cluster<%s,%s>",
             sizeof(T) == 4 ? "f32" : "f64", FWD ? "fwd" : "inv");
    return launch_k(special_cluster_kernel<T, FWD>, (unsigned)(tiles * CL_CTAS), CL_THREADS, 0, s, a);
}

template <typename T, bool FWD> static int launch_special_pass(const SpecialArgs<T>& a, int L, cudaStream_t s)
{
    const long long points = a.batch << a.m;
    return dispatch_int<1, 4>(L, [&]<int LL>() {
        GF_TRACE(tr, (double)points * 2 * sizeof(cx<T>), s, "special_%s<%s,%s,L%d,p0=%d>",
                 a.p0 == 0 ? "first" : "col", sizeof(T) == 4 ? "f32" : "f64", FWD ? "fwd" : "inv", LL, a.p0);
        if (a.p0 == 0)
        {
            constexpr long long RUN = (long long)SPECIAL_THREADS << LL;
            return launch_k(special_first_kernel<T, LL, FWD>, dim3((unsigned)((points + RUN - 1) / RUN)),
                            dim3(SPECIAL_THREADS), 0, s, a);
        }
        const long long threads = points >> LL;
        return launch_k(special_col_kernel<T, LL, FWD>,
                        dim3((unsigned)((threads + SPECIAL_THREADS - 1) / SPECIAL_THREADS)), dim3(SPECIAL_THREADS), 0,
                        s, a);
    });
}

template <typename T>
static int special_fft(cx<T>* inout, const cx<T>* table, int n_power, int fft_type, cx<T> mod_inverse, int batch,
                       cudaStream_t s)
{
    if (n_power < 1 || n_power > 24) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!inout || !table || batch <= 0 || (fft_type != GPUFFT_FORWARD && fft_type != GPUFFT_INVERSE))
        return GPUFFT_ERROR_INVALID_VALUE;
    if ((uintptr_t)inout % sizeof(cx<T>) || (uintptr_t)table % sizeof(cx<T>)) return GPUFFT_ERROR_MISALIGNED;
    // few tiles: the twelve smallest spans as one cluster pass (L = 12 below)
    const long long tiles = ((long long)batch << n_power) >> EBITS;
    const bool cl = n_power >= EBITS && cluster_ok(tiles);
    int p0s[8], Ls[8], np = 0;
    for (int p0 = 0; p0 < n_power; p0 += (cl && p0 == 0) ? EBITS : 4)
    {
        p0s[np] = p0;
        Ls[np] = (cl && p0 == 0) ? EBITS : ((n_power - p0) < 4 ? (n_power - p0) : 4);
        np++;
    }
    SpecialArgs<T> a{};
    a.data = inout;
    a.table = table;
    a.batch = batch;
    a.m = n_power;
    a.scale = mod_inverse;
    for (int i = 0; i < np; i++)
    {
        const int k = fft_type == GPUFFT_FORWARD ? i : np - 1 - i;
        a.p0 = p0s[k];
        a.do_scale = fft_type == GPUFFT_INVERSE && i == np - 1;
        int st;
        if (Ls[k] == EBITS)
            st = fft_type == GPUFFT_FORWARD ? launch_special_cluster<T, true>(a, s)
                                            : launch_special_cluster<T, false>(a, s);
        else
            st = fft_type == GPUFFT_FORWARD ? launch_special_pass<T, true>(a, Ls[k], s)
                                            : launch_special_pass<T, false>(a, Ls[k], s);
        if (st) return st;
    }
    return GPUFFT_SUCCESS;
}

} // namespace gfb

extern "C" int gpufft_special_fft_f32(void* inout, const void* table, int n_power, int fft_type, float mod_inverse_re,
                                      float mod_inverse_im, int batch, gpufft_stream_t stream)
{
    using C = gfb::cx<float>;
    return gfb::special_fft<float>(static_cast<C*>(inout), static_cast<const C*>(table), n_power, fft_type,
                                   gfb::mk<float>(mod_inverse_re, mod_inverse_im), batch, (cudaStream_t)stream);
}

extern "C" int gpufft_special_fft_f64(void* inout, const void* table, int n_power, int fft_type,
                                      double mod_inverse_re, double mod_inverse_im, int batch,
                                      gpufft_stream_t stream)
{
    using C = gfb::cx<double>;
    return gfb::special_fft<double>(static_cast<C*>(inout), static_cast<const C*>(table), n_power, fft_type,
                                    gfb::mk<double>(mod_inverse_re, mod_inverse_im), batch, (cudaStream_t)stream);
}
