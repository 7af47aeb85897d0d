// gpufft-b200: native fused negacyclic product c = a * b mod (X^N + 1).
//
// The product is the reference's FFNT chain (fold f_j + i f_{j+N/2}, twist by
// e^{i pi j / N}, half-length FFT, pointwise product, inverse, scale, untwist,
// unfold: reference fft.cu:1013-1384, fft_cpu.cu:301-432) fused so that the
// two spectra are never written out as a caller-visible intermediate:
//
//   N <= 8192:  one kernel. A CTA loads both operands of 4096/(N/2) products,
//               runs every forward stage on both in registers (shared twiddles
//               and index arithmetic), multiplies, runs every inverse stage,
//               untwists and writes the real product: one HBM read of a and b
//               and one HBM write of c.
//   N > 8192:   three kernels per wave of products -- the first forward pass
//               (strided, fold+twist fused into the load), the fused last pass
//               (forward both, multiply, inverse, in registers) and the last
//               inverse pass (strided, scale+untwist+unfold fused into the
//               store). The two spectra of a wave live in a caller-provided
//               workspace; its size sets the wave (products per launch).
//
// Twiddles come from gpufft_ffnt_make_tables_*, generated on the device with
// sincospi in double precision (then rounded to float for the f32 path).
#include "gf_fused.cuh"
#include "gf_fused_r8.cuh"

#include <atomic>

namespace gfb
{

// ---------------------------------------------------------------------------
// device twiddle tables:  [roots M/2 | inverse roots M/2 | twist M | untwist M | U M]
// roots[i] = e^{+2 pi i bitrev_{m-1}(i) / M}, twist[j] = e^{+i pi j / N}, M = N/2;
// roots[2j+1] = i roots[2j] exactly (the inverse roots are exact conjugates)
// (the values of the reference's ReverseRootTable_ffnt / twist_table_ffnt,
// fft_cpu.cu:251-297, 435-473, computed here in double precision).
// U[r] is the FFNT spectrum of the all-ones polynomial u = 1 + X + ... + X^(N-1)
// in the transform's output order: at frequency k = bitrev_m(r),
//     U = sum_j (1+i) psi^j w^(jk) = 2 / (1 - e^{i theta}) = 1 + i cot(theta/2),
// theta = pi (4k+1) / (2M). The split-precision product uses it to centre its
// inputs without an integer prefix scan; for M > 4096 it is stored in that
// product's spectrum order (each 4096-point tile permuted e -> (e >> 4) +
// 256 (e & 15)).
// ---------------------------------------------------------------------------
template <typename T> __global__ void ffnt_tables_kernel(cx<T>* tab, int m)
{
    const long long M = 1LL << m;
    const long long H = M >> 1;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < H)
    {
        double s, c;
        native_root(i, m, c, s);
        tab[i] = mk<T>((T)c, (T)s);
        tab[H + i] = mk<T>((T)c, (T)-s);
    }
    if (i < M)
    {
        double s, c;
        sincospi((double)i / (double)(2 * M), &s, &c);
        tab[2 * H + i] = mk<T>((T)c, (T)s);
        tab[2 * H + M + i] = mk<T>((T)c, (T)-s);
        const unsigned k = (m > 0) ? (__brev((unsigned)i) >> (32 - m)) : 0u;
        double sh, ch;
        sincospi((4.0 * (double)k + 1.0) / (4.0 * (double)M), &sh, &ch);
        // M > 4096: in the split product's spectrum order, each 4096-point tile
        // permuted e -> (e >> 4) + 256 (e & 15)
        const long long pu = (m > EBITS) ? ((i & ~4095LL) | ((i & 4095) >> 4) | ((i & 15) << 8)) : i;
        tab[2 * H + 2 * M + pu] = mk<T>((T)1, (T)(ch / sh));
    }
}

// Both operands live in registers: double needs 255 per thread (one CTA per
// SM), float fits 128 (two CTAs per SM, 16 warps).
template <typename T, int L, bool SINGLE>
__global__ void __launch_bounds__(NTHR, sizeof(T) == 4 ? 2 : 1) fused_kernel(const FusedArgs<T> a)
{
    pdl_begin(); // before any global-memory access (programmatic launch)
    extern __shared__ __align__(16) unsigned char smraw[];
    fused_body<T, L, SINGLE>(a, blockIdx.x, reinterpret_cast<cx<T>*>(smraw));
}

template <typename T, int L, bool SINGLE>
static int launch_fused_shape(const FusedArgs<T>& a, long long ctas, cudaStream_t s)
{
    const size_t smem = 2 * sizeof(cx<T>) * SMEM_ELEMS;
    static int smem_done[64] = {0};
    int st = ensure_smem(fused_kernel<T, L, SINGLE>, smem, smem_done);
    if (st) return st;
    // per product: SINGLE reads a, b (2 x N reals) and writes c (N reals); the
    // middle pass reads two spectra and writes one (3 x N/2 complex): 6 M T bytes
    const double M = (double)(1LL << a.geo.m);
    GF_TRACE(tr, (double)a.batch * M * 6.0 * sizeof(T), s, "fused_kernel<%s,L%d,%s>", sizeof(T) == 4 ? "f32" : "f64",
             L, SINGLE ? "single" : "middle");
    return launch_k(fused_kernel<T, L, SINGLE>, dim3((unsigned)ctas), dim3(NTHR), smem, s, a);
}

// The FP64 middle pass runs on 512 threads x 8 points per operand
// (fused_r8_kernel, 1: the default) or in the engine's 256 x 16 form (0); the
// values are identical. Set by gpufft_set_f64_middle.
static std::atomic<int> g_f64_middle_r8{1};

static int launch_fused_r8(const FusedArgs<double>& a, long long ctas, cudaStream_t s)
{
    static int done[64] = {0};
    const size_t smem = r8::smem_bytes(sizeof(cx<double>));
    int st = ensure_smem(fused_r8_kernel<double>, smem, done);
    if (st) return st;
    const double M = (double)(1LL << a.geo.m);
    GF_TRACE(tr, (double)a.batch * M * 6.0 * sizeof(double), s, "fused_r8_kernel<f64,L12,middle>");
    return launch_k(fused_r8_kernel<double>, dim3((unsigned)ctas), dim3(r8::THREADS), smem, s, a);
}

template <typename T, bool SINGLE> static int launch_fused(const FusedArgs<T>& a, long long ctas, cudaStream_t s)
{
    if (ctas <= 0) return GPUFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return GPUFFT_ERROR_INVALID_VALUE;
    if (!SINGLE && cluster_ok(ctas))
    {
        // few tiles: each tile's middle pass on a cluster of CTAs
        const long long M = 1LL << a.geo.m;
        ClusterArgs<T> c{};
        c.in = a.ws;
        c.in2 = a.ws + a.batch * M;
        c.out = a.ws;
        c.table = a.roots;
        c.inv_table = a.inv_roots;
        c.m = a.geo.m;
        return launch_cluster_pass<T, CLM_FUSED>(c, ctas, a.batch, s);
    }
    if constexpr (!SINGLE && sizeof(T) == 8)
    {
        if (g_f64_middle_r8.load(std::memory_order_relaxed)) return launch_fused_r8(a, ctas, s);
    }
    if (!SINGLE) return launch_fused_shape<T, EBITS, false>(a, ctas, s);
    if (a.geo.m >= 10 && cluster_ok(a.batch))
    {
        // few products of 2^10 .. 2^12 points: each product on one cluster of
        // 2^(m-9) CTAs (fold or linear load, product, unfold, or the cyclic
        // product's complex rows) instead of one CTA for whole products
        ClusterArgs<T> c{};
        c.table = a.roots;
        c.inv_table = a.inv_roots;
        c.m = a.geo.m;
        c.scale = mk<T>(a.scale, T(0));
        if (a.cplx)
        {
            c.in = reinterpret_cast<const cx<T>*>(a.a);
            c.in2 = reinterpret_cast<const cx<T>*>(a.b);
            c.out = reinterpret_cast<cx<T>*>(a.c);
            c.do_scale = 1;
            c.in_kind = CL_IN_CPX;
            c.out_kind = CL_OUT_CPX;
        }
        else
        {
            c.rin = a.a;
            c.rin2 = a.b;
            c.rout = a.c;
            c.twist = a.twist;
            c.untwist = a.untwist;
            c.in_kind = a.lin ? CL_IN_LIN : CL_IN_FOLD;
            c.out_kind = CL_OUT_UNFOLD;
        }
        return launch_cluster_pass<T, CLM_FUSED>(c, a.batch, a.batch, s, a.geo.m);
    }
    return dispatch_int<1, EBITS>(a.geo.m, [&]<int LL>() { return launch_fused_shape<T, LL, true>(a, ctas, s); });
}

constexpr int NATIVE_MIN_NPOWER = 2;
constexpr int NATIVE_MAX_NPOWER = 22; // two-pass plans: M = N/2 <= 2^21
// Recommended wave: 80 MiB of spectra (then rounded to whole waves of the SMs).
// Measured at N = 2^16 (1 MiB of spectra per product), batch 256: waves of
// 37 / 74 / 256 products run 718k / 770k / 750k products/s.
constexpr size_t WAVE_TARGET_BYTES = 80ull << 20;

static long long wave_products(int n_power, long long batch, size_t cx_bytes)
{
    const int m = n_power - 1;
    if (m <= EBITS) return batch;
    const size_t per = 2 * ((size_t)1 << m) * cx_bytes;
    long long w = (long long)(WAVE_TARGET_BYTES / per);
    if (w < 1) w = 1;
    w = round_wave(w, ((long long)1 << m) / ECTA);
    return w < batch ? w : batch;
}

// lin = 0: c = a b mod (X^N + 1), N = 2^n_power, a/b/c rows of N.
// lin = 1: the linear product of rows of N/2 (a, b zero-padded to N; the
//          product has degree < N - 1 so no wrap-around), c rows of N.
template <typename T>
static int negacyclic_mul(const T* a, const T* b, T* c, int n_power, int batch, const void* tables, void* ws,
                          size_t ws_bytes, cudaStream_t s, int lin = 0)
{
    if (n_power < NATIVE_MIN_NPOWER || n_power > NATIVE_MAX_NPOWER) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!a || !b || !c || !tables || batch <= 0) return GPUFFT_ERROR_INVALID_VALUE;
    if ((uintptr_t)a % sizeof(T) || (uintptr_t)b % sizeof(T) || (uintptr_t)c % sizeof(T) ||
        (uintptr_t)tables % sizeof(cx<T>) || (uintptr_t)ws % sizeof(cx<T>))
        return GPUFFT_ERROR_MISALIGNED;
    const int m = n_power - 1;
    const long long M = 1LL << m;
    const auto* tab = reinterpret_cast<const cx<T>*>(tables);
    FusedArgs<T> f{};
    f.roots = tab;
    f.inv_roots = tab + M / 2;
    f.twist = tab + M;
    f.untwist = tab + 2 * M;
    f.scale = (T)(1.0 / (double)M);
    f.lin = lin;
    const long long in_row = lin ? M : 2 * M; // reals per input row

    if (m <= EBITS)
    {
        f.a = a;
        f.b = b;
        f.c = c;
        f.batch = batch;
        f.geo = PassGeo{};
        f.geo.m = m;
        const long long ctas = ((long long)batch * M + ECTA - 1) / ECTA;
        return launch_fused<T, true>(f, ctas, s);
    }

    // the workspace sets the wave: as many products as it holds (more products
    // per wave means more CTAs per launch), rounded to whole waves of the SMs
    const size_t per = 2 * (size_t)M * sizeof(cx<T>);
    if (!ws || ws_bytes < per) return GPUFFT_ERROR_WORKSPACE;
    long long W = (long long)(ws_bytes / per);
    if (W >= batch)
        W = batch;
    else
        W = round_wave(W, M / ECTA);
    cx<T>* wsp = reinterpret_cast<cx<T>*>(ws);
    const Plan p = make_plan(m);
    for (long long p0 = 0; p0 < batch; p0 += W)
    {
        const long long w = (batch - p0) < W ? (batch - p0) : W;
        // 1. first forward pass of both operands: fold + twist in the load
        {
            long long ctas = 0;
            PassArgs<T> k{};
            k.geo = pass_geo(p, 0, m, 0, 2 * w, &ctas);
            k.in = a + p0 * in_row;
            k.in2 = b + p0 * in_row;
            k.split = w;
            k.out = wsp;
            k.table = f.roots;
            k.twist = f.twist;
            k.batch = 2 * w;
            k.in_kind = lin ? IN_LIN2 : IN_FOLD2;
            k.out_kind = OUT_CPX;
            int st = launch_pass<T, true>(k, p, 0, ctas, s);
            if (st) return st;
        }
        // 2. last forward pass of both, product, first inverse pass
        {
            long long ctas = 0;
            f.geo = pass_geo(p, 1, m, 0, w, &ctas);
            f.ws = wsp;
            f.batch = w;
            int st = launch_fused<T, false>(f, ctas, s);
            if (st) return st;
        }
        // 3. last inverse pass: scale, untwist, unfold into c
        {
            long long ctas = 0;
            PassArgs<T> k{};
            k.geo = pass_geo(p, 0, m, 0, w, &ctas);
            k.in = wsp;
            k.out = c + p0 * 2 * M;
            k.table = f.inv_roots;
            k.twist = f.untwist;
            k.scale = mk<T>(f.scale, T(0));
            k.do_scale = 1;
            k.batch = w;
            k.in_kind = IN_CPX;
            k.out_kind = OUT_UNFOLD;
            int st = launch_pass<T, false>(k, p, 0, ctas, s);
            if (st) return st;
        }
    }
    return GPUFFT_SUCCESS;
}

// Cyclic product of complex vectors, c = a * b mod (X^M - 1), M = 2^n_power:
// the C_C product the reference forms with GPU_FFT (forward of both operands,
// inverse with the product, fft.cu:517-598), fused like the negacyclic
// product. The transforms are cyclic, so no twist: the roots are the first
// M/2 entries of the native block of the ring 2M, the same values as
// FFT<T>(M/2)'s bit-reversed table.
template <typename T>
static int cyclic_mul(const cx<T>* a, const cx<T>* b, cx<T>* c, int n_power, int batch, const void* tables, void* ws,
                      size_t ws_bytes, cudaStream_t s)
{
    if (n_power < 1 || n_power > NATIVE_MAX_NPOWER - 1) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!a || !b || !c || !tables || batch <= 0) return GPUFFT_ERROR_INVALID_VALUE;
    if ((uintptr_t)a % sizeof(cx<T>) || (uintptr_t)b % sizeof(cx<T>) || (uintptr_t)c % sizeof(cx<T>) ||
        (uintptr_t)tables % sizeof(cx<T>) || (uintptr_t)ws % sizeof(cx<T>))
        return GPUFFT_ERROR_MISALIGNED;
    const int m = n_power;
    const long long M = 1LL << m;
    const auto* tab = reinterpret_cast<const cx<T>*>(tables);
    FusedArgs<T> f{};
    f.roots = tab;
    f.inv_roots = tab + M / 2;
    f.scale = (T)(1.0 / (double)M);
    f.cplx = 1;
    if (m <= EBITS)
    {
        f.a = reinterpret_cast<const T*>(a);
        f.b = reinterpret_cast<const T*>(b);
        f.c = reinterpret_cast<T*>(c);
        f.batch = batch;
        f.geo = PassGeo{};
        f.geo.m = m;
        const long long ctas = ((long long)batch * M + ECTA - 1) / ECTA;
        return launch_fused<T, true>(f, ctas, s);
    }
    const size_t per = 2 * (size_t)M * sizeof(cx<T>);
    if (!ws || ws_bytes < per) return GPUFFT_ERROR_WORKSPACE;
    long long W = (long long)(ws_bytes / per);
    if (W >= batch)
        W = batch;
    else
        W = round_wave(W, M / ECTA);
    cx<T>* wsp = reinterpret_cast<cx<T>*>(ws);
    const Plan p = make_plan(m);
    if (p.np != 2) return GPUFFT_ERROR_INVALID_N_POWER;
    for (long long p0 = 0; p0 < batch; p0 += W)
    {
        const long long w = (batch - p0) < W ? (batch - p0) : W;
        {
            long long ctas = 0;
            PassArgs<T> k{};
            k.geo = pass_geo(p, 0, m, 0, 2 * w, &ctas);
            k.in = a + p0 * M;
            k.in2 = b + p0 * M;
            k.split = w;
            k.out = wsp;
            k.table = f.roots;
            k.batch = 2 * w;
            k.in_kind = IN_CPX2;
            k.out_kind = OUT_CPX;
            int st = launch_pass<T, true>(k, p, 0, ctas, s);
            if (st) return st;
        }
        {
            long long ctas = 0;
            f.geo = pass_geo(p, 1, m, 0, w, &ctas);
            f.ws = wsp;
            f.batch = w;
            int st = launch_fused<T, false>(f, ctas, s);
            if (st) return st;
        }
        {
            long long ctas = 0;
            PassArgs<T> k{};
            k.geo = pass_geo(p, 0, m, 0, w, &ctas);
            k.in = wsp;
            k.out = c + p0 * M;
            k.table = f.inv_roots;
            k.scale = mk<T>(f.scale, T(0));
            k.do_scale = 1;
            k.batch = w;
            k.in_kind = IN_CPX;
            k.out_kind = OUT_CPX;
            int st = launch_pass<T, false>(k, p, 0, ctas, s);
            if (st) return st;
        }
    }
    return GPUFFT_SUCCESS;
}

template <typename T> static int make_tables(int n_power, void* tables, cudaStream_t s)
{
    if (n_power < NATIVE_MIN_NPOWER || n_power > 25) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!tables) return GPUFFT_ERROR_INVALID_VALUE;
    if ((uintptr_t)tables % sizeof(cx<T>)) return GPUFFT_ERROR_MISALIGNED;
    const int m = n_power - 1;
    const long long M = 1LL << m;
    const int thr = 256;
    const long long blocks = (M + thr - 1) / thr;
    ffnt_tables_kernel<T><<<(unsigned)blocks, thr, 0, s>>>(reinterpret_cast<cx<T>*>(tables), m);
    return check_launch();
}

} // namespace gfb

extern "C" int gpufft_set_f64_middle(int r8)
{
    if (r8 < 0) return gfb::g_f64_middle_r8.load();
    return gfb::g_f64_middle_r8.exchange(r8 ? 1 : 0);
}

extern "C" size_t gpufft_ffnt_tables_count(int n_power)
{
    if (n_power < gfb::NATIVE_MIN_NPOWER || n_power > 25) return 0;
    // [roots M/2 | inverse roots M/2 | twist M | untwist M | U M], M = N/2
    return (size_t)4 << (n_power - 1);
}

extern "C" int gpufft_ffnt_make_tables_f32(int n_power, void* tables, gpufft_stream_t stream)
{
    return gfb::make_tables<float>(n_power, tables, (cudaStream_t)stream);
}
extern "C" int gpufft_ffnt_make_tables_f64(int n_power, void* tables, gpufft_stream_t stream)
{
    return gfb::make_tables<double>(n_power, tables, (cudaStream_t)stream);
}

extern "C" size_t gpufft_negacyclic_mul_workspace_bytes(int n_power, int batch, int precision_bits)
{
    if (n_power < gfb::NATIVE_MIN_NPOWER || n_power > gfb::NATIVE_MAX_NPOWER || batch <= 0) return 0;
    if (precision_bits != 32 && precision_bits != 64) return 0;
    const size_t cxb = precision_bits == 64 ? 16 : 8;
    const int m = n_power - 1;
    if (m <= gfb::EBITS) return 0;
    const long long w = gfb::wave_products(n_power, batch, cxb);
    return (size_t)w * 2 * ((size_t)1 << m) * cxb;
}

extern "C" size_t gpufft_cyclic_mul_workspace_bytes(int n_power, int batch, int precision_bits)
{
    if (n_power < 1 || n_power > gfb::NATIVE_MAX_NPOWER - 1 || batch <= 0) return 0;
    if (precision_bits != 32 && precision_bits != 64) return 0;
    const size_t cxb = precision_bits == 64 ? 16 : 8;
    if (n_power <= gfb::EBITS) return 0;
    const long long w = gfb::wave_products(n_power + 1, batch, cxb);
    return (size_t)w * 2 * ((size_t)1 << n_power) * cxb;
}

extern "C" int gpufft_cyclic_mul_f32(const void* a, const void* b, void* c, int n_power, int batch,
                                     const void* tables, void* workspace, size_t workspace_bytes,
                                     gpufft_stream_t stream)
{
    using C = gfb::cx<float>;
    return gfb::cyclic_mul<float>(static_cast<const C*>(a), static_cast<const C*>(b), static_cast<C*>(c), n_power,
                                  batch, tables, workspace, workspace_bytes, (cudaStream_t)stream);
}
extern "C" int gpufft_cyclic_mul_f64(const void* a, const void* b, void* c, int n_power, int batch,
                                     const void* tables, void* workspace, size_t workspace_bytes,
                                     gpufft_stream_t stream)
{
    using C = gfb::cx<double>;
    return gfb::cyclic_mul<double>(static_cast<const C*>(a), static_cast<const C*>(b), static_cast<C*>(c), n_power,
                                   batch, tables, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int gpufft_negacyclic_mul_f32(const float* a, const float* b, float* c, int n_power, int batch,
                                         const void* tables, void* workspace, size_t workspace_bytes,
                                         gpufft_stream_t stream)
{
    return gfb::negacyclic_mul<float>(a, b, c, n_power, batch, tables, workspace, workspace_bytes,
                                      (cudaStream_t)stream);
}
extern "C" int gpufft_negacyclic_mul_f64(const double* a, const double* b, double* c, int n_power, int batch,
                                         const void* tables, void* workspace, size_t workspace_bytes,
                                         gpufft_stream_t stream)
{
    return gfb::negacyclic_mul<double>(a, b, c, n_power, batch, tables, workspace, workspace_bytes,
                                       (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Host-buffer variants: a, b, c in (page-locked) host memory, chunks of the
// batch staged through the workspace with the transfers overlapped
// (gf_pipe.cuh). Workspace = staging slots, then the product workspace of
// one chunk.
// ---------------------------------------------------------------------------
#include "gf_pipe.cuh"

namespace gfb
{
static long long host_chunk(int n_power, long long batch, long long chunk, size_t cxb)
{
    if (chunk > 0) return chunk < batch ? chunk : batch;
    return pipe_chunk(wave_products(n_power, batch, cxb), batch);
}

template <typename T>
static int negacyclic_mul_host(const T* a, const T* b, T* c, int n_power, int batch, int chunk, const void* tables,
                               void* ws, size_t ws_bytes, cudaStream_t s)
{
    if (n_power < NATIVE_MIN_NPOWER || n_power > NATIVE_MAX_NPOWER) return GPUFFT_ERROR_INVALID_N_POWER;
    if (batch <= 0) return GPUFFT_ERROR_INVALID_VALUE;
    const long long ch = host_chunk(n_power, batch, chunk, sizeof(cx<T>));
    const size_t row = sizeof(T) << n_power;
    const size_t slots = pipe_bytes(ch, row, row);
    if (!ws || ws_bytes < slots) return GPUFFT_ERROR_WORKSPACE;
    void* pws = static_cast<char*>(ws) + slots;
    const size_t pws_bytes = ws_bytes - slots;
    return run_pipeline(a, b, c, batch, ch, row, row, ws, slots, s,
                        [&](void* da, void* db, void* dc, long long rows, cudaStream_t st) {
                            return negacyclic_mul<T>(static_cast<const T*>(da), static_cast<const T*>(db),
                                                     static_cast<T*>(dc), n_power, (int)rows, tables, pws, pws_bytes,
                                                     st);
                        });
}
} // namespace gfb

extern "C" size_t gpufft_negacyclic_mul_host_workspace_bytes(int n_power, int batch, int chunk, int precision_bits)
{
    if (n_power < gfb::NATIVE_MIN_NPOWER || n_power > gfb::NATIVE_MAX_NPOWER || batch <= 0) return 0;
    if (precision_bits != 32 && precision_bits != 64) return 0;
    const size_t cxb = precision_bits == 64 ? 16 : 8;
    const long long ch = gfb::host_chunk(n_power, batch, chunk, cxb);
    const size_t row = (cxb / 2) << n_power;
    return gfb::pipe_bytes(ch, row, row) + gpufft_negacyclic_mul_workspace_bytes(n_power, (int)ch, precision_bits);
}

extern "C" int gpufft_negacyclic_mul_f32_host(const float* a, const float* b, float* c, int n_power, int batch,
                                              int chunk, const void* tables, void* workspace, size_t workspace_bytes,
                                              gpufft_stream_t stream)
{
    return gfb::negacyclic_mul_host<float>(a, b, c, n_power, batch, chunk, tables, workspace, workspace_bytes,
                                           (cudaStream_t)stream);
}
extern "C" int gpufft_negacyclic_mul_f64_host(const double* a, const double* b, double* c, int n_power, int batch,
                                              int chunk, const void* tables, void* workspace, size_t workspace_bytes,
                                              gpufft_stream_t stream)
{
    return gfb::negacyclic_mul_host<double>(a, b, c, n_power, batch, chunk, tables, workspace, workspace_bytes,
                                            (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of gpufft_negacyclic_mul_f64.
//
// Some callers cannot call cudaMalloc at all: code running where the CUDA
// allocator is off limits (inside a foreign runtime's memory pool, a plugin
// host that owns every device allocation, or a process that must not grow its
// device footprint after start-up), and callers that only hold the buffers
// they were handed. For them this entry point takes its scratch from a
// library-owned, file-scope device array instead of a caller workspace.
//
// * The array is NOALLOC_SCRATCH_BYTES (16 MiB). It is part of this module's
//   device image, so every GPU on which the library's kernels are loaded holds
//   it until the process exits.
// * Host code may not use the array's name as a device address (on the host it
//   names a host-side shadow). Every call looks the device address up with
//   cudaGetSymbolAddress for the current device (so the address stays right
//   after a cudaDeviceReset); the first call on a device also loads the
//   module's device image there, so make that first call before any stream
//   capture.
// * Rings whose one-product workspace exceeds the array (N > 2^20) are
//   rejected with GPUFFT_ERROR_WORKSPACE. Larger batches run in more waves.
// * All calls share the array and nothing in it needs to start at zero (every
//   byte a wave reads was written earlier in the same wave). Calls whose work
//   overlaps on the GPU (different streams, or different host threads without
//   ordering) race on the array: serialise them.
// ---------------------------------------------------------------------------
namespace gfb
{
constexpr size_t NOALLOC_SCRATCH_BYTES = 16ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static int noalloc_scratch(void** out)
{
    // looked up on every call (a cheap runtime query, no allocation): the
    // address stays right across cudaDeviceReset, which reloads this module's
    // device image and may move the array
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return set_cuda_error(e);
    *out = p;
    return GPUFFT_SUCCESS;
}
} // namespace gfb

extern "C" int gpufft_negacyclic_mul_f64_noalloc(const double* a, const double* b, double* c, int n_power,
                                                 int batch, const void* tables, gpufft_stream_t stream)
{
    if (n_power < gfb::NATIVE_MIN_NPOWER || n_power > gfb::NATIVE_MAX_NPOWER) return GPUFFT_ERROR_INVALID_N_POWER;
    const int m = n_power - 1;
    if (m > gfb::EBITS && 2 * ((size_t)1 << m) * sizeof(double2) > gfb::NOALLOC_SCRATCH_BYTES)
        return GPUFFT_ERROR_WORKSPACE;
    void* scratch = nullptr;
    int st = gfb::noalloc_scratch(&scratch);
    if (st) return st;
    return gfb::negacyclic_mul<double>(a, b, c, n_power, batch, tables, scratch, gfb::NOALLOC_SCRATCH_BYTES,
                                       (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Linear product of real polynomials (the R_R product of the reference,
// reference fft.cu:600-725 with example/test_fft_gpu_R_R.cu's zero padding):
// computed as the negacyclic product of length 2N whose upper input halves are
// zero, so each operand folds into N real complex values -- a half-length
// transform, where the reference transforms 2N complex values.
// ---------------------------------------------------------------------------
extern "C" size_t gpufft_linear_mul_workspace_bytes(int n_power, int batch, int precision_bits)
{
    return gpufft_negacyclic_mul_workspace_bytes(n_power + 1, batch, precision_bits);
}

extern "C" int gpufft_linear_mul_f32(const float* a, const float* b, float* c, int n_power, int batch,
                                     const void* tables, void* workspace, size_t workspace_bytes,
                                     gpufft_stream_t stream)
{
    if (n_power < 1 || n_power > gfb::NATIVE_MAX_NPOWER - 1) return GPUFFT_ERROR_INVALID_N_POWER;
    return gfb::negacyclic_mul<float>(a, b, c, n_power + 1, batch, tables, workspace, workspace_bytes,
                                      (cudaStream_t)stream, 1);
}
extern "C" int gpufft_linear_mul_f64(const double* a, const double* b, double* c, int n_power, int batch,
                                     const void* tables, void* workspace, size_t workspace_bytes,
                                     gpufft_stream_t stream)
{
    if (n_power < 1 || n_power > gfb::NATIVE_MAX_NPOWER - 1) return GPUFFT_ERROR_INVALID_N_POWER;
    return gfb::negacyclic_mul<double>(a, b, c, n_power + 1, batch, tables, workspace, workspace_bytes,
                                       (cudaStream_t)stream, 1);
}
