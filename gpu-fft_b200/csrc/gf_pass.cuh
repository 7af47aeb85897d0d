// gpufft-b200: one engine pass as a kernel (load variant -> rounds -> store
// variant) and the host-side pass plans. Shared by the drop-in transforms and
// the native products.
#pragma once

#include "gf_engine.cuh"

namespace gfb
{

enum InKind
{
    IN_CPX = 0,  // complex vector (transform position j)
    IN_REAL = 1, // real promoted to complex (fft.cu:303-305)
    IN_FOLD = 2, // FFNT fold f_j + i f_{j+M} then twist (fft.cu:1057-1069)
    IN_PROD = 3,  // product of the two complex operands (fft.cu:194-205, 1252-1263)
    IN_FOLD2 = 4  // IN_FOLD with batch entries [0, split) from `in`, the rest from `in2`
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
    const void* in2; // IN_FOLD2: second operand array
    void* out;
    const cx<T>* table;
    const cx<T>* twist;
    cx<T> scale;
    long long prod_off; // element offset of the second operand (IN_PROD)
    long long batch;
    PassGeo geo;
    long long split; // IN_FOLD2: batch entries taken from `in`
    int zero_pad;    // forward first pass: the upper half of each input is zero
    int do_scale;    // last inverse pass: multiply by scale
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
    else if (IN == IN_FOLD || IN == IN_FOLD2)
    {
        const T* base = reinterpret_cast<const T*>(a.in);
        if (IN == IN_FOLD2 && b >= a.split)
        {
            base = reinterpret_cast<const T*>(a.in2);
            b -= a.split;
        }
        const T* p = base + b * 2 * M + j;
        const cx<T> f = mk<T>(ld_stream(p), ld_stream(p + M));
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

static inline Plan make_plan(int m)
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
static inline PassGeo pass_geo(const Plan& p, int k, int m, int neg, long long batch, long long* ctas)
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
static inline int launch_pass(PassArgs<T> a, long long ctas, cudaStream_t s)
{
    if (ctas <= 0) return GPUFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return GPUFFT_ERROR_INVALID_VALUE;
    const size_t smem = sizeof(cx<T>) * SMEM_ELEMS;
    static int smem_done[64] = {0}; // one set per kernel instantiation
    int st = ensure_smem(pass_kernel<T, FWD, IN, OUT>, smem, smem_done);
    if (st) return st;
    pass_kernel<T, FWD, IN, OUT><<<dim3((unsigned)ctas), dim3(NTHR), smem, s>>>(a);
    return check_launch();
}

} // namespace gfb
