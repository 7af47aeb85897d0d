// gpufft-b200: vector-Jacobian product (adjoint) of the real linear product.
//
// Forward: c = a * b, a and b of length N, c of length 2N (the linear product,
// computed as a negacyclic product mod X^(2N) + 1 of the zero-padded rows,
// gpufft_linear_mul_*). Backward, for an upstream gradient g of length 2N:
//     grad_a[i] = sum_k g[k] b[k - i],   grad_b[j] = sum_k g[k] a[k - j]   (i, j < N),
// i.e. the first N coefficients of g b* and g a*, where x*(X) = x(X^-1) is the
// adjoint of multiplication by x in the ring. The FFNT spectrum holds the
// evaluations of a polynomial at roots z of X^(2N) + 1 on the unit circle, so
// for a real x the spectrum of x* is the complex conjugate of the spectrum of x.
// The VJP is therefore the forward product pipeline with conjugated spectra:
// three forward transforms (g folded, a and b zero-padded), the pointwise
// products G conj(B) and G conj(A), two inverse transforms, and only the real
// parts (the coefficients below N) are written.
//
//   2N <= 8192:  one kernel per product group (vjp_kernel<L, true>);
//   otherwise:   strided first forward pass of g, a, b (pass_kernel, IN_VJP3),
//                contiguous middle pass (vjp_kernel<12, false>), strided last
//                inverse pass keeping the real parts (pass_kernel, OUT_RE2).
#include "gf_pass.cuh"

namespace gfb
{

struct VjpArgs
{
    const float* g;
    const float* a;
    const float* b;
    float* ga;
    float* gb;
    cx<float>* ws; // [3][W][M]: G, A, B spectra; the two products overwrite G and A
    const cx<float>* roots;
    const cx<float>* inv_roots;
    const cx<float>* twist;
    const cx<float>* untwist;
    float scale;
    long long batch;
    PassGeo geo;
};

template <int L, bool SINGLE> __global__ void __launch_bounds__(NTHR, 1) vjp_kernel(const VjpArgs a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<float>* sm = reinterpret_cast<cx<float>*>(smraw);
    using S = Sched<0, L>;
    constexpr int W0 = S::win(0, true), WE = S::win(S::n - 1, false);
    const int t = threadIdx.x;
    const long long cta = blockIdx.x;
    const long long M = 1LL << a.geo.m;

    cx<float> x[3][RPT];
    TwCtx c;
    {
        const Tile<L, false, W0> tl(a.geo, cta, t);
        c.g = tl.g;
        c.vec = tw_vec_ok<float>(a.roots) && tw_vec_ok<float>(a.inv_roots);
#pragma unroll
        for (int r = 0; r < RPT; r++)
        {
            const long long bb = tl.b(r), j = tl.j(r);
            if (bb >= a.batch)
            {
                x[0][r] = x[1][r] = x[2][r] = mk<float>(0.f, 0.f);
                continue;
            }
            if (SINGLE)
            {
                const cx<float> tw = ldg<float>(a.twist + j);
                const float* pg = a.g + bb * 2 * M + j;
                x[0][r] = cmul<float>(mk<float>(__ldcs(pg), __ldcs(pg + M)), tw);
                x[1][r] = cmul<float>(mk<float>(__ldcs(a.a + bb * M + j), 0.f), tw);
                x[2][r] = cmul<float>(mk<float>(__ldcs(a.b + bb * M + j), 0.f), tw);
            }
            else
            {
                x[0][r] = a.ws[bb * M + j];
                x[1][r] = a.ws[(a.batch + bb) * M + j];
                x[2][r] = a.ws[(2 * a.batch + bb) * M + j];
            }
        }
    }
    c.s0 = a.geo.s0;
    c.neg = 0;
    run_rounds<float, true, 0, L, 3>(x, sm, a.roots, c, t);
    cx<float> p[2][RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        p[0][r] = cmulc<float>(x[0][r], x[2][r]); // G conj(B) -> grad_a
        p[1][r] = cmulc<float>(x[0][r], x[1][r]); // G conj(A) -> grad_b
    }
    run_rounds<float, false, 0, L, 2>(p, sm, a.inv_roots, c, t);

    const Tile<L, false, WE> te(a.geo, cta, t);
#pragma unroll
    for (int r = 0; r < RPT; r++)
    {
        const long long bb = te.b(r), j = te.j(r);
        if (bb >= a.batch) continue;
        if (SINGLE)
        {
            const cx<float> u = ldg<float>(a.untwist + j);
            const cx<float> s = mk<float>(a.scale, 0.f);
            __stcs(a.ga + bb * M + j, cmul<float>(cmul<float>(p[0][r], s), u).x);
            __stcs(a.gb + bb * M + j, cmul<float>(cmul<float>(p[1][r], s), u).x);
        }
        else
        {
            a.ws[bb * M + j] = p[0][r];
            a.ws[(a.batch + bb) * M + j] = p[1][r];
        }
    }
}

template <int L, bool SINGLE> static int launch_vjp_shape(const VjpArgs& a, long long ctas, cudaStream_t s)
{
    const size_t smem = 3 * sizeof(cx<float>) * SMEM_ELEMS;
    static int done[64] = {0};
    int st = ensure_smem(vjp_kernel<L, SINGLE>, smem, done);
    if (st) return st;
    // three spectra (G, A, B) in, two gradients out, per point of the half-length transform
    GF_TRACE(tr, (double)a.batch * (double)(1LL << a.geo.m) * 5 * sizeof(cx<float>), s, "vjp_kernel<L%d,%s>", L,
             SINGLE ? "single" : "middle");
    return launch_k(vjp_kernel<L, SINGLE>, dim3((unsigned)ctas), dim3(NTHR), smem, s, a);
}

static long long vjp_wave(int m, long long batch)
{
    if (m <= EBITS) return batch;
    const size_t per = 3 * ((size_t)1 << m) * sizeof(cx<float>);
    long long w = (long long)((48ull << 20) / per);
    if (w < 1) w = 1;
    return w < batch ? w : batch;
}

// n_power: log2 of the operand length N (the product and g have 2N entries).
static int linear_vjp(const float* g, const float* a, const float* b, float* ga, float* gb, int n_power, int batch,
                      const void* tables, void* ws, size_t ws_bytes, cudaStream_t s)
{
    if (n_power < 1 || n_power > 20) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!g || !a || !b || !ga || !gb || !tables || batch <= 0) return GPUFFT_ERROR_INVALID_VALUE;
    if ((uintptr_t)g % 4 || (uintptr_t)a % 4 || (uintptr_t)b % 4 || (uintptr_t)ga % 4 || (uintptr_t)gb % 4 ||
        (uintptr_t)tables % 8 || (uintptr_t)ws % 8)
        return GPUFFT_ERROR_MISALIGNED;
    const int m = n_power; // transform length M = N (ring 2N)
    const long long M = 1LL << m;
    const auto* tab = reinterpret_cast<const cx<float>*>(tables);
    VjpArgs A{};
    A.roots = tab;
    A.inv_roots = tab + M / 2;
    A.twist = tab + M;
    A.untwist = tab + 2 * M;
    A.scale = (float)(1.0 / (double)M);
    if (m <= EBITS)
    {
        A.g = g;
        A.a = a;
        A.b = b;
        A.ga = ga;
        A.gb = gb;
        A.batch = batch;
        A.geo = PassGeo{};
        A.geo.m = m;
        const long long ctas = ((long long)batch * M + ECTA - 1) / ECTA;
        return dispatch_int<1, EBITS>(m, [&]<int LL>() { return launch_vjp_shape<LL, true>(A, ctas, s); });
    }
    long long W = vjp_wave(m, batch);
    const size_t per = 3 * (size_t)M * sizeof(cx<float>);
    if (!ws || ws_bytes < per) return GPUFFT_ERROR_WORKSPACE;
    if ((size_t)W * per > ws_bytes) W = (long long)(ws_bytes / per);
    auto* wsp = reinterpret_cast<cx<float>*>(ws);
    const Plan p = make_plan(m);
    for (long long p0 = 0; p0 < batch; p0 += W)
    {
        const long long w = (batch - p0) < W ? (batch - p0) : W;
        long long ctas = 0;
        PassArgs<float> k{};
        k.geo = pass_geo(p, 0, m, 0, 3 * w, &ctas);
        k.in = g + p0 * 2 * M;
        k.in2 = a + p0 * M;
        k.in3 = b + p0 * M;
        k.split = w;
        k.out = wsp;
        k.table = A.roots;
        k.twist = A.twist;
        k.batch = 3 * w;
        k.in_kind = IN_VJP3;
        k.out_kind = OUT_CPX;
        int st = launch_pass<float, true>(k, p, 0, ctas, s);
        if (st) return st;

        A.geo = pass_geo(p, 1, m, 0, w, &ctas);
        A.ws = wsp;
        A.batch = w;
        st = launch_vjp_shape<EBITS, false>(A, ctas, s);
        if (st) return st;

        PassArgs<float> q{};
        q.geo = pass_geo(p, 0, m, 0, 2 * w, &ctas);
        q.in = wsp;
        q.out = ga + p0 * M;
        q.out2 = gb + p0 * M;
        q.split = w;
        q.table = A.inv_roots;
        q.twist = A.untwist;
        q.scale = mk<float>(A.scale, 0.f);
        q.do_scale = 1;
        q.batch = 2 * w;
        q.in_kind = IN_CPX;
        q.out_kind = OUT_RE2;
        st = launch_pass<float, false>(q, p, 0, ctas, s);
        if (st) return st;
    }
    return GPUFFT_SUCCESS;
}

} // namespace gfb

extern "C" size_t gpufft_linear_mul_vjp_workspace_bytes(int n_power, int batch)
{
    if (n_power < 1 || n_power > 20 || batch <= 0) return 0;
    if (n_power <= gfb::EBITS) return 0;
    return (size_t)gfb::vjp_wave(n_power, batch) * 3 * ((size_t)1 << n_power) * sizeof(float2);
}

extern "C" int gpufft_linear_mul_vjp_f32(const float* g, const float* a, const float* b, float* grad_a,
                                         float* grad_b, int n_power, int batch, const void* tables, void* workspace,
                                         size_t workspace_bytes, gpufft_stream_t stream)
{
    return gfb::linear_vjp(g, a, b, grad_a, grad_b, n_power, batch, tables, workspace, workspace_bytes,
                           (cudaStream_t)stream);
}

extern "C" int gpufft_conv_vjp_f32(const float* g, const float* a, const float* b, float* grad_a, float* grad_b,
                                   int n_power, int batch, const void* tables, void* workspace, size_t workspace_bytes,
                                   gpufft_stream_t stream)
{
    return gpufft_linear_mul_vjp_f32(g, a, b, grad_a, grad_b, n_power, batch, tables, workspace, workspace_bytes,
                                     stream);
}
