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
    IN_PROD = 3, // product of the two complex operands (fft.cu:194-205, 1252-1263)
    IN_FOLD2 = 4 // IN_FOLD with batch entries [0, split) from `in`, the rest from `in2`
};
enum OutKind
{
    OUT_CPX = 0,   // complex vector, optionally scaled by mod_inverse (fft.cu:246-253)
    OUT_REAL = 1,  // real part of the scaled value (fft.cu:499-514)
    OUT_UNFOLD = 2 // scale, untwist, unfold re -> j, im -> j+M (fft.cu:1366-1383)
};

// Geometry of one pass (stages [s0, s0+L) of a 2^m transform); L and the
// strided/contiguous choice are template parameters of the kernels.
struct PassGeo
{
    int m;    // log2 transform length
    int s0;   // first stage of the pass
    int neg;  // negacyclic (X^N+1) twiddle indexing
    int pad_;
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
    long long split; // IN_FOLD2: batch entries taken from `in`
    PassGeo geo;
    int in_kind, out_kind;
    int zero_pad; // forward first pass: the upper half of each input is zero
    int do_scale; // last inverse pass: multiply by scale
};

// Where the 16 registers of thread t (window W) live: batch entry b[r] and
// transform index j[r] of every register, for a CTA `cta` of a pass with L
// stages, strided (columns of the pass share a CTA) or contiguous.
template <int L, bool STRIDED, int W> struct Tile
{
    long long b[RPT];
    long long j[RPT];
    long long g; // stage-s0 group (uniform over the CTA)

    __device__ __forceinline__ Tile(const PassGeo& G, long long cta, int t)
    {
        const int eb = e_base<W>(t);
        const long long M = 1LL << G.m;
        if constexpr (STRIDED)
        {
            constexpr int CL = EBITS - L; // log2 columns per CTA
            const int lgcpb = G.m - G.s0 - EBITS; // log2 column blocks per group
            const long long bb = cta >> (G.m - EBITS);
            const long long rem = cta & ((1LL << (G.m - EBITS)) - 1);
            g = rem >> lgcpb;
            const long long cblk = rem & ((1LL << lgcpb) - 1);
            const int sl = G.m - G.s0 - L; // log2 stride S
            const long long j0 = (g << (G.m - G.s0)) + (cblk << CL) + (eb & ((1 << CL) - 1)) +
                                 ((long long)(eb >> CL) << sl);
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                // register bits r<<W split into column (below CL) and q (above) parts
                const int e_r = r << W;
                const int cpart = e_r & ((1 << CL) - 1);
                const int qpart = e_r >> CL;
                b[r] = bb;
                j[r] = j0 + cpart + ((long long)qpart << sl);
            }
        }
        else
        {
            const long long gi0 = cta * ECTA + eb;
            g = ((cta * ECTA) >> L) & ((1LL << G.s0) - 1);
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                const long long gi = gi0 + (r << W);
                b[r] = gi >> G.m;
                j[r] = gi & (M - 1);
            }
        }
    }
};

template <typename T>
__device__ __forceinline__ cx<T> load_elem(const PassArgs<T>& a, int kind, long long b, long long j)
{
    const long long M = 1LL << a.geo.m;
    if (kind == IN_CPX)
    {
        if (a.zero_pad && j >= (M >> 1)) return mk<T>(T(0), T(0));
        return reinterpret_cast<const cx<T>*>(a.in)[b * M + j];
    }
    else if (kind == IN_REAL)
    {
        if (a.zero_pad && j >= (M >> 1)) return mk<T>(T(0), T(0));
        return mk<T>(reinterpret_cast<const T*>(a.in)[b * M + j], T(0));
    }
    else if (kind == IN_FOLD || kind == IN_FOLD2)
    {
        const T* base = reinterpret_cast<const T*>(a.in);
        if (kind == IN_FOLD2 && b >= a.split)
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

template <typename T>
__device__ __forceinline__ void store_elem(const PassArgs<T>& a, int kind, long long b, long long j, cx<T> v)
{
    const long long M = 1LL << a.geo.m;
    if (kind == OUT_CPX)
    {
        if (a.do_scale) v = cmul<T>(v, a.scale);
        reinterpret_cast<cx<T>*>(a.out)[b * M + j] = v;
    }
    else if (kind == OUT_REAL)
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

template <typename T, bool FWD, int L, bool STRIDED>
__global__ void __launch_bounds__(NTHR, 2) pass_kernel(const PassArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
    constexpr int QOFF = STRIDED ? EBITS - L : 0;
    using S = Sched<QOFF, L>;
    constexpr int W0 = S::win(0, FWD), WL = S::win(S::n - 1, FWD);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;

    cx<T> x[1][RPT];
    {
        const Tile<L, STRIDED, W0> tl(a.geo, cta, t);
        const int kind = a.in_kind;
#pragma unroll
        for (int r = 0; r < RPT; r++)
            x[0][r] = (tl.b[r] < a.batch) ? load_elem<T>(a, kind, tl.b[r], tl.j[r]) : mk<T>(T(0), T(0));
    }
    TwCtx c;
    c.g = Tile<L, STRIDED, W0>(a.geo, cta, t).g;
    c.s0 = a.geo.s0;
    c.neg = a.geo.neg;
    run_rounds<T, FWD, QOFF, L, 1>(x, sm, a.table, c, t);
    {
        const Tile<L, STRIDED, WL> tl(a.geo, cta, t);
        const int kind = a.out_kind;
#pragma unroll
        for (int r = 0; r < RPT; r++)
            if (tl.b[r] < a.batch) store_elem<T>(a, kind, tl.b[r], tl.j[r], x[0][r]);
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

// m <= 12: one pass; 12 < m <= 21: (m-12, 12); 21 < m <= 24: (m-21, 9, 12)
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

// Geometry and grid size of pass k of plan p for `batch` transforms of 2^m.
static inline PassGeo pass_geo(const Plan& p, int k, int m, int neg, long long batch, long long* ctas)
{
    PassGeo G{};
    G.m = m;
    G.s0 = 0;
    for (int i = 0; i < k; i++) G.s0 += p.L[i];
    G.neg = neg;
    if (k == p.np - 1)
        *ctas = ((batch << m) + ECTA - 1) / ECTA;
    else
        *ctas = batch << (m - EBITS);
    return G;
}

template <typename T, bool FWD, int L, bool STRIDED>
static inline int launch_pass_shape(const PassArgs<T>& a, long long ctas, cudaStream_t s)
{
    const size_t smem = sizeof(cx<T>) * SMEM_ELEMS;
    static int smem_done[64] = {0};
    int st = ensure_smem(pass_kernel<T, FWD, L, STRIDED>, smem, smem_done);
    if (st) return st;
    pass_kernel<T, FWD, L, STRIDED><<<dim3((unsigned)ctas), dim3(NTHR), smem, s>>>(a);
    return check_launch();
}

// Launch pass k of plan p (the pass's L selects the compiled shape).
template <typename T, bool FWD>
static inline int launch_pass(const PassArgs<T>& a, const Plan& p, int k, long long ctas, cudaStream_t s)
{
    if (ctas <= 0) return GPUFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return GPUFFT_ERROR_INVALID_VALUE;
    const int L = p.L[k];
    if (k == p.np - 1)
        return dispatch_int<1, EBITS>(L, [&]<int LL>() { return launch_pass_shape<T, FWD, LL, false>(a, ctas, s); });
    return dispatch_int<1, 9>(L, [&]<int LL>() { return launch_pass_shape<T, FWD, LL, true>(a, ctas, s); });
}

} // namespace gfb
