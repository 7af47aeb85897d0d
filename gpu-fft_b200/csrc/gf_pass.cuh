// gpufft-b200: one engine pass as a kernel (load variant -> rounds -> store
// variant) and the host-side pass plans. Shared by the drop-in transforms and
// the native products.
#pragma once

#include "gf_cluster.cuh"

namespace gfb
{

enum InKind
{
    IN_CPX = 0,  // complex vector (transform position j)
    IN_REAL = 1, // real promoted to complex (fft.cu:303-305)
    IN_FOLD = 2, // FFNT fold f_j + i f_{j+M} then twist (fft.cu:1057-1069)
    IN_PROD = 3, // product of the two complex operands (fft.cu:194-205, 1252-1263)
    IN_FOLD2 = 4, // IN_FOLD with batch entries [0, split) from `in`, the rest from `in2`
    IN_LIN2 = 5,  // zero-padded linear operand: x_j = f_j (real, rows of M), then twist;
                  // batch entries [0, split) from `in`, the rest from `in2`
    IN_VJP3 = 6,  // batch entries [0, split): IN_FOLD from `in` (rows of 2M);
                  // [split, 2 split): IN_LIN from `in2`; [2 split, 3 split): IN_LIN from `in3`
    IN_CPX2 = 7   // complex rows of M: batch entries [0, split) from `in`, the rest from `in2`
};
enum OutKind
{
    OUT_CPX = 0,   // complex vector, optionally scaled by mod_inverse (fft.cu:246-253)
    OUT_REAL = 1,  // real part of the scaled value (fft.cu:499-514)
    OUT_UNFOLD = 2, // scale, untwist, unfold re -> j, im -> j+M (fft.cu:1366-1383)
    OUT_RE2 = 3     // scale, untwist, keep the real part (coefficient j < M) only;
                    // batch entries [0, split) to `out`, the rest to `out2`
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
    const void* in2; // IN_FOLD2 / IN_LIN2 / IN_VJP3: second operand array
    const void* in3; // IN_VJP3: third operand array
    void* out;
    void* out2;      // OUT_RE2: second output array
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
    int perm;     // contiguous 12-stage pass: forward stores, inverse loads, each
                  // 4096-point tile in the order e -> (e >> 4) + 256 (e & 15)
};

// Where the 16 registers of thread t (window W) live, for a CTA `cta` of a
// pass with L stages, strided (columns of the pass share a CTA) or contiguous:
// register r holds the point with flat index f0 + df(r) = b M + j (batch entry
// b, transform index j). df(r) is a compile-time constant after unrolling
// (contiguous: r << W; strided: one shift by the pass's stride), so loads and
// stores of a tile address a base pointer plus constant offsets; b(r) and
// j(r) are derived on demand for the variants that need them.
template <int L, bool STRIDED, int W> struct Tile
{
    long long g;  // stage-s0 group (uniform over the CTA)
    long long f0; // flat index of register 0
    int m;        // log2 transform length
    int sl;       // strided: log2 stride of the pass's q bits

    __device__ __forceinline__ Tile(const PassGeo& G, long long cta, int t)
    {
        const int eb = e_base<W>(t);
        m = G.m;
        if constexpr (STRIDED)
        {
            constexpr int CL = EBITS - L; // log2 columns per CTA
            const int lgcpb = G.m - G.s0 - EBITS; // log2 column blocks per group
            const long long bb = cta >> (G.m - EBITS);
            const long long rem = cta & ((1LL << (G.m - EBITS)) - 1);
            g = rem >> lgcpb;
            const long long cblk = rem & ((1LL << lgcpb) - 1);
            sl = G.m - G.s0 - L; // log2 stride S
            f0 = (bb << G.m) + (g << (G.m - G.s0)) + (cblk << CL) + (eb & ((1 << CL) - 1)) +
                 ((long long)(eb >> CL) << sl);
        }
        else
        {
            sl = 0;
            f0 = cta * ECTA + eb;
            g = ((cta * ECTA) >> L) & ((1LL << G.s0) - 1);
        }
    }
    // register bits r << W split into column (below CL) and q (above) parts
    __device__ __forceinline__ long long df(int r) const
    {
        const int e_r = r << W;
        if constexpr (STRIDED)
        {
            constexpr int CL = EBITS - L;
            return (long long)(e_r & ((1 << CL) - 1)) + ((long long)(e_r >> CL) << sl);
        }
        else
        {
            return (long long)e_r;
        }
    }
    __device__ __forceinline__ long long flat(int r) const { return f0 + df(r); }
    __device__ __forceinline__ long long b(int r) const { return flat(r) >> m; }
    __device__ __forceinline__ long long j(int r) const { return flat(r) & ((1LL << m) - 1); }
};

template <typename T>
__device__ __forceinline__ cx<T> load_elem(const PassArgs<T>& a, int kind, long long b, long long j)
{
    const long long M = 1LL << a.geo.m;
    if (kind == IN_CPX2)
    {
        const cx<T>* base = reinterpret_cast<const cx<T>*>(b < a.split ? a.in : a.in2);
        return ld_stream(base + (b < a.split ? b : b - a.split) * M + j);
    }
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
    else if (kind == IN_LIN2)
    {
        const T* base = reinterpret_cast<const T*>(a.in);
        if (b >= a.split)
        {
            base = reinterpret_cast<const T*>(a.in2);
            b -= a.split;
        }
        return cmul<T>(mk<T>(ld_stream(base + b * M + j), T(0)), ldg<T>(a.twist + j));
    }
    else if (kind == IN_VJP3)
    {
        if (b < a.split)
        {
            const T* p = reinterpret_cast<const T*>(a.in) + b * 2 * M + j;
            return cmul<T>(mk<T>(ld_stream(p), ld_stream(p + M)), ldg<T>(a.twist + j));
        }
        const T* base = reinterpret_cast<const T*>(b < 2 * a.split ? a.in2 : a.in3);
        b -= (b < 2 * a.split) ? a.split : 2 * a.split;
        return cmul<T>(mk<T>(ld_stream(base + b * M + j), T(0)), ldg<T>(a.twist + j));
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
    else if (kind == OUT_UNFOLD)
    {
        v = cmul<T>(cmul<T>(v, a.scale), ldg<T>(a.twist + j));
        T* p = reinterpret_cast<T*>(a.out) + b * 2 * M + j;
        p[0] = v.x;
        p[M] = v.y;
    }
    else
    {
        v = cmul<T>(cmul<T>(v, a.scale), ldg<T>(a.twist + j));
        T* base = reinterpret_cast<T*>(b < a.split ? a.out : a.out2);
        b -= (b < a.split) ? 0 : a.split;
        st_stream(base + b * M + j, v.x);
    }
}

// Every register of a tile through one load (store) variant. The variant is
// uniform over the launch; dispatching it once outside the register loop keeps
// each variant straight-line, so the 16 loads of a thread are issued together
// (a switch per element serialises them into 16 memory round trips, which a
// launch of a few CTAs cannot hide).
template <typename T, int K, typename TL>
__device__ __forceinline__ void load_regs(const PassArgs<T>& a, const TL& tl, cx<T> (&x)[RPT])
{
#pragma unroll
    for (int r = 0; r < RPT; r++)
        x[r] = (tl.b(r) < a.batch) ? load_elem<T>(a, K, tl.b(r), tl.j(r)) : mk<T>(T(0), T(0));
}
template <typename T, typename TL>
__device__ __forceinline__ void load_tile(const PassArgs<T>& a, int kind, const TL& tl, cx<T> (&x)[RPT])
{
    switch (kind)
    {
    case IN_CPX: load_regs<T, IN_CPX>(a, tl, x); break;
    case IN_REAL: load_regs<T, IN_REAL>(a, tl, x); break;
    case IN_FOLD: load_regs<T, IN_FOLD>(a, tl, x); break;
    case IN_PROD: load_regs<T, IN_PROD>(a, tl, x); break;
    case IN_FOLD2: load_regs<T, IN_FOLD2>(a, tl, x); break;
    case IN_LIN2: load_regs<T, IN_LIN2>(a, tl, x); break;
    case IN_VJP3: load_regs<T, IN_VJP3>(a, tl, x); break;
    case IN_CPX2: load_regs<T, IN_CPX2>(a, tl, x); break;
    default: break;
    }
}
template <typename T, int K, typename TL>
__device__ __forceinline__ void store_regs(const PassArgs<T>& a, const TL& tl, const cx<T> (&x)[RPT])
{
#pragma unroll
    for (int r = 0; r < RPT; r++)
        if (tl.b(r) < a.batch) store_elem<T>(a, K, tl.b(r), tl.j(r), x[r]);
}
template <typename T, typename TL>
__device__ __forceinline__ void store_tile(const PassArgs<T>& a, int kind, const TL& tl, const cx<T> (&x)[RPT])
{
    switch (kind)
    {
    case OUT_CPX: store_regs<T, OUT_CPX>(a, tl, x); break;
    case OUT_REAL: store_regs<T, OUT_REAL>(a, tl, x); break;
    case OUT_UNFOLD: store_regs<T, OUT_UNFOLD>(a, tl, x); break;
    case OUT_RE2: store_regs<T, OUT_RE2>(a, tl, x); break;
    default: break;
    }
}

// Row pointers of one batch entry for the load kinds whose rows are real
// coefficients (fold pairs f_j, f_{j+M}, or linear rows with zero imaginary
// part): selected once per CTA when the whole tile lies in one batch entry.
template <typename T> struct RealRows
{
    const T* re;
    long long im_off; // offset of f_{j+M} from f_j; < 0: imaginary part is zero
};

template <typename T>
__device__ __forceinline__ RealRows<T> real_rows(const PassArgs<T>& a, int kind, long long b)
{
    const long long M = 1LL << a.geo.m;
    RealRows<T> r;
    if (kind == IN_FOLD || kind == IN_FOLD2)
    {
        const T* base = reinterpret_cast<const T*>((kind == IN_FOLD2 && b >= a.split) ? a.in2 : a.in);
        if (kind == IN_FOLD2 && b >= a.split) b -= a.split;
        r.re = base + b * 2 * M;
        r.im_off = M;
    }
    else if (kind == IN_LIN2)
    {
        const T* base = reinterpret_cast<const T*>(b >= a.split ? a.in2 : a.in);
        if (b >= a.split) b -= a.split;
        r.re = base + b * M;
        r.im_off = -1;
    }
    else // IN_VJP3
    {
        if (b < a.split)
        {
            r.re = reinterpret_cast<const T*>(a.in) + b * 2 * M;
            r.im_off = M;
        }
        else
        {
            const T* base = reinterpret_cast<const T*>(b < 2 * a.split ? a.in2 : a.in3);
            b -= (b < 2 * a.split) ? a.split : 2 * a.split;
            r.re = base + b * M;
            r.im_off = -1;
        }
    }
    return r;
}

// One pass of CTA-tile `cta` (sm: SMEM_ELEMS complex elements of shared memory).
// PERM (contiguous 12-stage passes whose spectra are only consumed pointwise
// and by the matching inverse pass): a forward pass stores the registers of its
// last round (window 0: thread t holds tile points 16 t + r) at the window-8
// addresses t + 256 r, and an inverse pass loads that order straight into
// window 0 -- one shared-memory transpose fewer each.
template <typename T, bool FWD, int L, bool STRIDED, bool PERM = false>
__device__ __forceinline__ void pass_body(const PassArgs<T>& a, long long cta, cx<T>* sm)
{
    static_assert(!PERM || (L == EBITS && !STRIDED), "PERM: contiguous 12-stage passes only");
    constexpr int QOFF = STRIDED ? EBITS - L : 0;
    using S = Sched<QOFF, L>;
    constexpr int W0 = S::win(0, FWD), WL = S::win(S::n - 1, FWD);
    // A round in window 0 keeps 16 consecutive elements in each thread, so a
    // warp's access would touch 32 separate sectors. Such passes load (store)
    // in window 8, where the thread index runs along the lowest element bits,
    // and move to (from) window 0 with one more shared-memory transpose.
    constexpr int WIN = W0 == 0 ? 8 : W0;
    constexpr int WOUT = WL == 0 ? 8 : WL;
    const int t = threadIdx.x;
    // the tile lies in one batch entry: strided passes, and contiguous passes of
    // transforms with at least ECTA elements
    const bool one_entry = STRIDED || a.geo.m >= EBITS;

    cx<T> x[1][RPT];
    TwCtx c;
    {
        const Tile<L, STRIDED, WIN> tl(a.geo, cta, t);
        c.g = tl.g;
        const int kind = a.in_kind;
        const bool real_rows_kind = kind == IN_FOLD || kind == IN_FOLD2 || kind == IN_LIN2 || kind == IN_VJP3;
        if (one_entry && real_rows_kind && tl.b(0) < a.batch)
        {
            // straight-line loads: every address is row + j
            const RealRows<T> rr = real_rows<T>(a, kind, tl.b(0));
            const long long j0 = tl.j(0);
            const T* pre = rr.re + j0;
            const cx<T>* ptw = a.twist + j0;
            T re[RPT], im[RPT];
            cx<T> tw[RPT];
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                re[r] = ld_stream(pre + tl.df(r));
                im[r] = (rr.im_off >= 0) ? ld_stream(pre + rr.im_off + tl.df(r)) : T(0);
                tw[r] = ldg<T>(ptw + tl.df(r));
            }
#pragma unroll
            for (int r = 0; r < RPT; r++) x[0][r] = cmul<T>(mk<T>(re[r], im[r]), tw[r]);
        }
        else if (one_entry && kind == IN_CPX && tl.b(0) < a.batch)
        {
            const long long M = 1LL << a.geo.m;
            const cx<T>* p = reinterpret_cast<const cx<T>*>(a.in) + tl.f0;
            const bool zp = a.zero_pad != 0;
            const long long jz = (M >> 1) - tl.j(0); // j(r) >= M/2 <=> df(r) >= jz
#pragma unroll
            for (int r = 0; r < RPT; r++)
                x[0][r] = (zp && tl.df(r) >= jz) ? mk<T>(T(0), T(0)) : p[tl.df(r)];
        }
        else
        {
            load_tile<T>(a, kind, tl, x[0]);
        }
    }
    c.s0 = a.geo.s0;
    c.neg = a.geo.neg;
    c.vec = tw_vec_ok<T>(a.table);
    if constexpr (WIN != W0 && !PERM) transpose<T, WIN, W0, 1>(x, sm, t);
    run_rounds<T, FWD, QOFF, L, 1>(x, sm, a.table, c, t);
    if constexpr (WOUT != WL && !PERM) transpose<T, WL, WOUT, 1>(x, sm, t);
    {
        const Tile<L, STRIDED, WOUT> tl(a.geo, cta, t);
        const int kind = a.out_kind;
        if (one_entry && tl.b(0) < a.batch && (kind == OUT_UNFOLD || kind == OUT_CPX))
        {
            const long long M = 1LL << a.geo.m;
            if (kind == OUT_UNFOLD)
            {
                const long long j0 = tl.j(0);
                T* row = reinterpret_cast<T*>(a.out) + tl.b(0) * 2 * M + j0;
                const cx<T>* ptw = a.twist + j0;
                cx<T> u[RPT];
#pragma unroll
                for (int r = 0; r < RPT; r++) u[r] = ldg<T>(ptw + tl.df(r));
#pragma unroll
                for (int r = 0; r < RPT; r++)
                {
                    const cx<T> v = cmul<T>(cmul<T>(x[0][r], a.scale), u[r]);
                    st_stream(row + tl.df(r), v.x);
                    st_stream(row + M + tl.df(r), v.y);
                }
            }
            else
            {
                cx<T>* p = reinterpret_cast<cx<T>*>(a.out) + tl.f0;
#pragma unroll
                for (int r = 0; r < RPT; r++) p[tl.df(r)] = a.do_scale ? cmul<T>(x[0][r], a.scale) : x[0][r];
            }
        }
        else
        {
            store_tile<T>(a, kind, tl, x[0]);
        }
    }
}

// Resident CTAs per SM the pass kernels are compiled for: float passes hold 32
// data registers per thread and fit three CTAs; double passes fit two.
template <typename T> constexpr int pass_min_blocks() { return sizeof(T) == 4 ? 3 : 2; }

template <typename T, bool FWD, int L, bool STRIDED, bool PERM = false>
__global__ void __launch_bounds__(NTHR, pass_min_blocks<T>()) pass_kernel(const PassArgs<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    extern __shared__ __align__(16) unsigned char smraw[];
    pass_body<T, FWD, L, STRIDED, PERM>(a, blockIdx.x, reinterpret_cast<cx<T>*>(smraw));
}

// Algorithmic bytes of one pass launch: every element of the pass read once in
// its load variant's format and written once in its store variant's format.
template <typename T> inline double pass_alg_bytes(const PassArgs<T>& a)
{
    const double E = (double)a.batch * (double)(1LL << a.geo.m), t = sizeof(T), c = 2 * sizeof(T);
    double in = c, out = c;
    switch (a.in_kind)
    {
    case IN_REAL: in = a.zero_pad ? t / 2 : t; break;
    case IN_LIN2: in = t; break;
    case IN_VJP3: in = 4 * t / 3; break;
    case IN_PROD: in = 2 * c; break;
    case IN_CPX: in = a.zero_pad ? c / 2 : c; break;
    default: break;
    }
    if (a.out_kind == OUT_REAL || a.out_kind == OUT_RE2) out = t;
    return E * (in + out);
}
inline const char* kind_name(int fwd) { return fwd ? "fwd" : "inv"; }

// ---------------------------------------------------------------------------
// Column form of a strided pass of L <= 4 stages. The pass's closed
// sub-networks are the columns of each stage-s0 group: elements
// j = g M / 2^s0 + c + i C (i < 2^L, C = M / 2^(s0+L)). One thread owns one
// column in registers and runs the pass's radix-2 steps with the same
// twiddles (table[(neg ? 2^s : 0) + (g << u) + (i >> (L-u))] at stage s = s0+u)
// and in the same order as the tiled kernel, so the values are identical;
// there is no shared memory and no barrier, neighbouring threads take
// neighbouring columns (coalesced), and with 2^L elements per thread many
// more threads are in flight than with 4096-element tiles. Load and store
// variants are compile-time, so their selection costs nothing per element.
// ---------------------------------------------------------------------------
constexpr int COL_MAX_L = 4;
constexpr int COL_THREADS = 128;

// Column `idx` (over all batch entries) of the pass; no shared memory, no
// barrier, so it can run inside a persistent kernel too.
template <typename T, bool FWD, int L, int IK, int OK>
__device__ __forceinline__ void col_pass_body(const PassArgs<T>& a, long long idx)
{
    constexpr int R = 1 << L;
    const int m = a.geo.m, s0 = a.geo.s0;
    const int lc = m - s0 - L; // log2 columns per group
    const long long b = idx >> (m - L);
    if (b >= a.batch) return;
    const long long r = idx & ((1LL << (m - L)) - 1);
    const long long g = r >> lc;
    const long long C = 1LL << lc;
    const long long j0 = (g << (m - s0)) + (r & (C - 1));
    // every twiddle of the column's stages (2^u at stage s0 + u), and the
    // untwist factors of an unfolding store, are loaded before the data: one
    // memory latency instead of one per stage
    cx<T> w[R - 1];
#pragma unroll
    for (int u = 0; u < L; u++)
    {
        const cx<T>* tw = a.table + (a.geo.neg ? (1LL << (s0 + u)) : 0LL) + (g << u);
#pragma unroll
        for (int h = 0; h < (1 << u); h++) w[(1 << u) - 1 + h] = ldg<T>(tw + h);
    }
    constexpr bool UNTW = OK == OUT_UNFOLD || OK == OUT_RE2;
    cx<T> un[UNTW ? R : 1];
    if constexpr (UNTW)
    {
#pragma unroll
        for (int i = 0; i < R; i++) un[i] = ldg<T>(a.twist + j0 + i * C);
    }
    cx<T> x[R];
#pragma unroll
    for (int i = 0; i < R; i++) x[i] = load_elem<T>(a, IK, b, j0 + i * C);
#pragma unroll
    for (int k = 0; k < L; k++)
    {
        const int u = FWD ? k : L - 1 - k; // stage s0 + u
        const int h = 1 << (L - 1 - u);
#pragma unroll
        for (int i = 0; i < R; i++)
        {
            if (i & h) continue;
            const cx<T> wt = w[(1 << u) - 1 + (i >> (L - u))];
            if (FWD)
                ct_bfly<T>(x[i], x[i + h], wt);
            else
                gs_bfly<T>(x[i], x[i + h], wt);
        }
    }
    if constexpr (OK == OUT_UNFOLD)
    {
        const long long M = 1LL << m;
        T* p = reinterpret_cast<T*>(a.out) + b * 2 * M + j0;
#pragma unroll
        for (int i = 0; i < R; i++)
        {
            const cx<T> v = cmul<T>(cmul<T>(x[i], a.scale), un[i]);
            p[i * C] = v.x;
            p[i * C + M] = v.y;
        }
    }
    else if constexpr (OK == OUT_RE2)
    {
        const long long M = 1LL << m;
        T* base = reinterpret_cast<T*>(b < a.split ? a.out : a.out2);
        const long long bb = (b < a.split) ? b : b - a.split;
#pragma unroll
        for (int i = 0; i < R; i++)
        {
            const cx<T> v = cmul<T>(cmul<T>(x[i], a.scale), un[i]);
            st_stream(base + bb * M + j0 + i * C, v.x);
        }
    }
    else
    {
#pragma unroll
        for (int i = 0; i < R; i++) store_elem<T>(a, OK, b, j0 + i * C, x[i]);
    }
}

// The column passes wait on global loads (one column's points and twiddles
// per thread): eight-point double columns are compiled for eight CTAs per SM
// (64 registers) so that more loads are in flight.
template <typename T, int L> constexpr int col_min_blocks() { return (sizeof(T) == 8 && L <= 3) ? 8 : 1; }

template <typename T, bool FWD, int L, int IK, int OK>
__global__ void __launch_bounds__(COL_THREADS, col_min_blocks<T, L>()) col_pass_kernel(const PassArgs<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    col_pass_body<T, FWD, L, IK, OK>(a, (long long)blockIdx.x * COL_THREADS + threadIdx.x);
}

// Launch the column form when a kernel for (in_kind, out_kind) is compiled:
// forward first passes (any load, complex store) and inverse last passes
// (complex load, any store). Returns -1 when the pair has no column kernel.
template <typename T, bool FWD, int L>
static inline int launch_col_pass(const PassArgs<T>& a, cudaStream_t s)
{
    const long long threads = a.batch << (a.geo.m - L);
    const unsigned blocks = (unsigned)((threads + COL_THREADS - 1) / COL_THREADS);
    auto go = [&](auto kern) {
        GF_TRACE(tr, pass_alg_bytes(a), s, "col_pass<%s,%s,L%d,in%d,out%d>", sizeof(T) == 4 ? "f32" : "f64",
                 kind_name(FWD), L, a.in_kind, a.out_kind);
        return launch_k(kern, blocks, COL_THREADS, 0, s, a);
    };
    if constexpr (FWD)
    {
        if (a.out_kind != OUT_CPX) return -1;
        switch (a.in_kind)
        {
        case IN_CPX: return go(col_pass_kernel<T, true, L, IN_CPX, OUT_CPX>);
        case IN_REAL: return go(col_pass_kernel<T, true, L, IN_REAL, OUT_CPX>);
        case IN_FOLD: return go(col_pass_kernel<T, true, L, IN_FOLD, OUT_CPX>);
        case IN_FOLD2: return go(col_pass_kernel<T, true, L, IN_FOLD2, OUT_CPX>);
        case IN_LIN2: return go(col_pass_kernel<T, true, L, IN_LIN2, OUT_CPX>);
        case IN_VJP3: return go(col_pass_kernel<T, true, L, IN_VJP3, OUT_CPX>);
        case IN_CPX2: return go(col_pass_kernel<T, true, L, IN_CPX2, OUT_CPX>);
        default: return -1;
        }
    }
    else
    {
        if (a.in_kind != IN_CPX) return -1;
        switch (a.out_kind)
        {
        case OUT_CPX: return go(col_pass_kernel<T, false, L, IN_CPX, OUT_CPX>);
        case OUT_REAL: return go(col_pass_kernel<T, false, L, IN_CPX, OUT_REAL>);
        case OUT_UNFOLD: return go(col_pass_kernel<T, false, L, IN_CPX, OUT_UNFOLD>);
        case OUT_RE2: return go(col_pass_kernel<T, false, L, IN_CPX, OUT_RE2>);
        default: return -1;
        }
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

template <typename T, bool FWD, int L, bool STRIDED, bool PERM = false>
static inline int launch_pass_shape(const PassArgs<T>& a, long long ctas, cudaStream_t s)
{
    if constexpr (L == EBITS && !STRIDED && !PERM)
    {
        if (a.perm) return launch_pass_shape<T, FWD, L, false, true>(a, ctas, s);
    }
    const size_t smem = sizeof(cx<T>) * SMEM_ELEMS;
    static int smem_done[64] = {0};
    int st = ensure_smem(pass_kernel<T, FWD, L, STRIDED, PERM>, smem, smem_done);
    if (st) return st;
    GF_TRACE(tr, pass_alg_bytes(a), s, "pass_kernel<%s,%s,L%d,%s>", sizeof(T) == 4 ? "f32" : "f64",
             kind_name(FWD), L, STRIDED ? "strided" : "contiguous");
    return launch_k(pass_kernel<T, FWD, L, STRIDED, PERM>, dim3((unsigned)ctas), dim3(NTHR), smem, s, a);
}

// Launch pass k of plan p (the pass's L selects the compiled shape).
template <typename T, bool FWD>
static inline int launch_pass(const PassArgs<T>& a, const Plan& p, int k, long long ctas, cudaStream_t s)
{
    if (ctas <= 0) return GPUFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return GPUFFT_ERROR_INVALID_VALUE;
    const int L = p.L[k];
    if (k == p.np - 1)
    {
        // a contiguous 12-stage pass over few tiles: spread each tile over a cluster
        const bool ck = FWD ? a.in_kind == IN_CPX : (a.in_kind == IN_CPX || a.in_kind == IN_PROD);
        if (L == EBITS && a.geo.m > EBITS && ck && a.out_kind == OUT_CPX && !a.zero_pad && !a.perm &&
            cluster_ok(ctas))
        {
            ClusterArgs<T> c{};
            c.in = static_cast<const cx<T>*>(a.in);
            c.out = static_cast<cx<T>*>(a.out);
            c.table = a.table;
            c.inv_table = a.table;
            c.scale = a.scale;
            c.prod_off = a.prod_off;
            c.m = a.geo.m;
            c.neg = a.geo.neg;
            c.prod = a.in_kind == IN_PROD;
            c.do_scale = a.do_scale;
            return launch_cluster_pass<T, FWD ? CLM_FWD : CLM_INV>(c, ctas, a.batch, s);
        }
        // a whole transform of 2^10 .. 2^12 points in one pass, few rows: one
        // cluster of 2^(L-9) CTAs per row instead of one CTA for the whole
        // transform (or for several rows)
        const bool in_ok = FWD ? (a.in_kind == IN_CPX || a.in_kind == IN_FOLD)
                               : (a.in_kind == IN_CPX || a.in_kind == IN_PROD);
        const bool out_ok = FWD ? a.out_kind == OUT_CPX : (a.out_kind == OUT_CPX || a.out_kind == OUT_UNFOLD);
        if (p.np == 1 && L >= 10 && L == a.geo.m && in_ok && out_ok && !a.zero_pad && !a.perm &&
            cluster_ok(a.batch))
        {
            ClusterArgs<T> c{};
            c.in = static_cast<const cx<T>*>(a.in);
            c.out = static_cast<cx<T>*>(a.out);
            c.table = a.table;
            c.inv_table = a.table;
            c.scale = a.scale;
            c.prod_off = a.prod_off;
            c.m = a.geo.m;
            c.neg = a.geo.neg;
            c.prod = a.in_kind == IN_PROD;
            c.do_scale = a.do_scale;
            c.in_kind = a.in_kind == IN_FOLD ? CL_IN_FOLD : CL_IN_CPX;
            c.out_kind = a.out_kind == OUT_UNFOLD ? CL_OUT_UNFOLD : CL_OUT_CPX;
            c.rin = static_cast<const T*>(a.in);
            c.rout = static_cast<T*>(a.out);
            c.twist = a.twist;
            c.untwist = a.twist;
            return launch_cluster_pass<T, FWD ? CLM_FWD : CLM_INV>(c, a.batch, a.batch, s, L);
        }
        return dispatch_int<1, EBITS>(L, [&]<int LL>() { return launch_pass_shape<T, FWD, LL, false>(a, ctas, s); });
    }
    if (L <= COL_MAX_L)
    {
        const int st = dispatch_int<1, COL_MAX_L>(L, [&]<int LL>() { return launch_col_pass<T, FWD, LL>(a, s); });
        if (st >= 0) return st;
    }
    return dispatch_int<1, 9>(L, [&]<int LL>() { return launch_pass_shape<T, FWD, LL, true>(a, ctas, s); });
}

} // namespace gfb
