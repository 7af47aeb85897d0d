// gpufft-b200: the fused product pass (forward of both operands, pointwise
// product, inverse) as a device function, shared by the product kernels and
// the batched multi-size kernel.
#pragma once

#include "gf_pass.cuh"

namespace gfb
{

template <typename T> struct FusedArgs
{
    const T* a;
    const T* b;
    T* c;
    cx<T>* ws;
    const cx<T>* roots;
    const cx<T>* inv_roots;
    const cx<T>* twist;
    const cx<T>* untwist;
    T scale;
    long long batch; // products handled by this launch
    PassGeo geo;
    int lin;  // linear (zero-padded) operands: rows of M reals, x_j = f_j
    int cplx; // cyclic product of complex rows of M (no twist): a, b, c point to
              // COMPLEX<T> rows, c is scaled, SINGLE only
};

// Root i (0 <= i < M/2) of the native tables of a 2^m-point transform:
// exp(2 pi i br(i) / M), br the m-1 bit reversal, in double precision. Odd
// entries are exactly i times their even neighbour (bit reversal makes index
// 2j+1 the angle of 2j plus a quarter turn), and the tables store that relation
// exactly: kernels of the native products load the even entry only and rotate
// it. Every generator of native tables goes through this function.
__device__ __forceinline__ void native_root(long long i, int m, double& c, double& s)
{
    const long long M = 1LL << m;
    const long long ie = i & ~1LL;
    const unsigned br = (m > 1) ? (__brev((unsigned)ie) >> (33 - m)) : 0u;
    sincospi(2.0 * (double)br / (double)M, &s, &c);
    if (i & 1)
    {
        const double t = c;
        c = -s;
        s = t;
    }
}

// Contiguous pass over both operands: all forward stages of the pass on A and
// B, the pointwise product, and all inverse stages on the product. SINGLE: the
// pass is the whole transform (fold + twist in the load, scale + untwist +
// unfold in the store); otherwise A/B come from and the product returns to the
// workspace.
template <typename T, int L, bool SINGLE>
__device__ __forceinline__ void fused_body(const FusedArgs<T>& a, long long cta, cx<T>* sm)
{
    using S = Sched<0, L>;
    constexpr int W0 = S::win(0, true), WM = S::win(S::n - 1, true), WE = S::win(S::n - 1, false);
    const int t = threadIdx.x;
    const long long M = 1LL << a.geo.m;

    cx<T> x[2][RPT];
    TwCtx c;
    {
        const Tile<L, false, W0> tl(a.geo, cta, t);
        c.g = tl.g;
        c.vec = tw_vec_ok<T>(a.roots) && tw_vec_ok<T>(a.inv_roots);
        // the variant is uniform: one straight-line loop per variant, so a
        // thread's loads are issued together
        const cx<T> zero = mk<T>(T(0), T(0));
        if (SINGLE && a.cplx)
        {
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                const bool ok = tl.b(r) < a.batch;
                x[0][r] = ok ? ld_stream(reinterpret_cast<const cx<T>*>(a.a) + tl.b(r) * M + tl.j(r)) : zero;
                x[1][r] = ok ? ld_stream(reinterpret_cast<const cx<T>*>(a.b) + tl.b(r) * M + tl.j(r)) : zero;
            }
        }
        else if (SINGLE && a.lin)
        {
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                if (tl.b(r) >= a.batch)
                {
                    x[0][r] = x[1][r] = zero;
                    continue;
                }
                const cx<T> tw = ldg<T>(a.twist + tl.j(r));
                x[0][r] = cmul<T>(mk<T>(ld_stream(a.a + tl.b(r) * M + tl.j(r)), T(0)), tw);
                x[1][r] = cmul<T>(mk<T>(ld_stream(a.b + tl.b(r) * M + tl.j(r)), T(0)), tw);
            }
        }
        else if (SINGLE)
        {
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                if (tl.b(r) >= a.batch)
                {
                    x[0][r] = x[1][r] = zero;
                    continue;
                }
                const cx<T> tw = ldg<T>(a.twist + tl.j(r));
                const T* pa = a.a + tl.b(r) * 2 * M + tl.j(r);
                const T* pb = a.b + tl.b(r) * 2 * M + tl.j(r);
                x[0][r] = cmul<T>(mk<T>(ld_stream(pa), ld_stream(pa + M)), tw);
                x[1][r] = cmul<T>(mk<T>(ld_stream(pb), ld_stream(pb + M)), tw);
            }
        }
        else
        {
            // the middle pass (M >= 4096): the tile lies in one product
            const bool ok = tl.b(0) < a.batch;
            const cx<T>* pa = a.ws + tl.f0;
            const cx<T>* pb = pa + a.batch * M;
#pragma unroll
            for (int r = 0; r < RPT; r++)
            {
                x[0][r] = ok ? pa[tl.df(r)] : zero;
                x[1][r] = ok ? pb[tl.df(r)] : zero;
            }
        }
    }
    c.s0 = a.geo.s0;
    c.neg = 0;

    run_rounds<T, true, 0, L, 2>(x, sm, a.roots, c, t);
    static_assert(WM == S::win(0, false), "the inverse starts where the forward ends");
    cx<T> z[1][RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++) z[0][r] = cmul<T>(x[0][r], x[1][r]);
    run_rounds<T, false, 0, L, 1>(z, sm, a.inv_roots, c, t);

    const Tile<L, false, WE> tl(a.geo, cta, t);
    const cx<T> sc = mk<T>(a.scale, T(0));
    if (SINGLE && a.cplx)
    {
#pragma unroll
        for (int r = 0; r < RPT; r++)
            if (tl.b(r) < a.batch)
                st_stream(reinterpret_cast<cx<T>*>(a.c) + tl.b(r) * M + tl.j(r), cmul<T>(z[0][r], sc));
    }
    else if (SINGLE)
    {
        cx<T> u[RPT]; // untwist factors, loaded together
#pragma unroll
        for (int r = 0; r < RPT; r++) u[r] = ldg<T>(a.untwist + tl.j(r));
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            if (tl.b(r) >= a.batch) continue;
            const cx<T> v = cmul<T>(cmul<T>(z[0][r], sc), u[r]);
            T* pc = a.c + tl.b(r) * 2 * M + tl.j(r);
            st_stream(pc, v.x);
            st_stream(pc + M, v.y);
        }
    }
    else if (tl.b(0) < a.batch)
    {
        cx<T>* pz = a.ws + tl.f0;
#pragma unroll
        for (int r = 0; r < RPT; r++) pz[tl.df(r)] = z[0][r];
    }
}

} // namespace gfb
