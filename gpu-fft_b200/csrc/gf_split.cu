// gpufft-b200: split-precision negacyclic products (FP32 and FP64 transforms,
// exact int64 results) -- host side (plans, workspace, launches) and the C
// ABI. The kernels are in gf_split.cuh.
#include "gf_split.cuh"
#include "gf_pipe.cuh"

#include <atomic>
#include <map>
#include <vector>

namespace gfb
{
// FP32 split products of rings N = 2^14 .. 2^16 with at most six limbs run
// their contiguous stages in split_tile_kernel (1, the default) or in the
// five-kernel chain of pass kernels and split_groups (0). Both give the same
// integers; set by gpufft_set_split_tile. The tile kernel's bulk copies need a
// 16-byte aligned workspace, and it needs a tile per SM; others take the chain.
static std::atomic<int> g_split_tile{1};

// The tile kernel runs one persistent CTA per SM; a launch with fewer tiles
// than SMs (a few products) leaves most of the GPU idle and takes the chain.
static bool split_tile_ok(int m, int k, long long products)
{
    return g_split_tile.load(std::memory_order_relaxed) != 0 && m > EBITS && m - SPLIT_TILE_LT <= SPLIT_COL_MAX &&
           k <= SPLIT_TILE_MAXK && (products << (m - SPLIT_TILE_LT)) >= (long long)sm_count();
}

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
// Largest pre-rounding error expected for k balanced limbs of width w.
// For one limb pair the measured maximum over a batch follows
//     err ~ C * rms(d_a) * rms(d_b) * sqrt(N) * sqrt(log2(N/2)) * 2^-p,  C = 7.1
// with p = 24 (FP32) or 53 (FP64) mantissa bits (calibrated on FP32 negacyclic
// limb products: balanced 6-bit limbs at N = 2^16 give 0.144). A group sum of
// several pairs adds their errors in
// quadrature. The coefficients are signed values of magnitude below 2^B
// (B = input_bits, or input_bits - 1 after centring non-negative inputs);
// digits have rms 2^(w-1)/sqrt(3), the top digit 2^tb/sqrt(3) with
// tb = B - w(k-1) leftover bits. Also returns the typical largest group value
// (4 sigma) through *mag.
static double predicted_error(int n_power, int B, int w, int k, bool centred, double* mag, int prec = 24)
{
    double r[SPLIT_MAX_LIMBS];
    for (int l = 0; l < k; l++) r[l] = std::ldexp(1.0, w - 1) / std::sqrt(3.0);
    const int tb = B - w * (k - 1);
    r[k - 1] = std::ldexp(1.0, tb) / std::sqrt(3.0);
    // centring term 2^ur (e^a_l + e^b_l) u joins group l + uq (u has rms 1)
    const int uq = B / w, ur = B - w * uq;
    double worst = 0.0;
    for (int s = 0; s <= 2 * (k - 1); s++)
    {
        double e2 = 0.0;
        for (int i = 0; i < k; i++)
        {
            const int j = s - i;
            if (j >= 0 && j < k) e2 += (r[i] * r[j]) * (r[i] * r[j]);
        }
        const int l = s - uq;
        if (centred && l >= 0 && l < k) e2 += 2.0 * std::ldexp(r[l], ur) * std::ldexp(r[l], ur);
        worst = std::max(worst, std::sqrt(e2));
    }
    const double sqn = std::sqrt(std::ldexp(1.0, n_power));
    if (mag) *mag = 4.0 * worst * sqn;
    return 7.1 * worst * sqn * std::sqrt((double)(n_power - 1)) * std::ldexp(1.0, -prec);
}

static bool choose_limbs(int n_power, int input_bits, bool non_negative, int* w_out, int* k_out, int prec = 24)
{
    // the plan with the fewest limbs whose predicted error is at most 0.2 and
    // whose group values stay far inside the certifiable range (< 2^(p-3))
    const int B = non_negative ? input_bits - 1 : input_bits;
    for (int k = 1; k <= SPLIT_MAX_LIMBS; k++)
    {
        const int w = (B + 1 + k - 1) / k; // k balanced digits of w bits cover 2^B in magnitude
        if (w < 1 || w > 20 || B - w * (k - 1) > w - 1) continue;
        double mag = 0;
        if (predicted_error(n_power, B, w, k, non_negative, &mag, prec) <= 0.2 && mag < std::ldexp(1.0, prec - 3))
        {
            *w_out = w;
            *k_out = k;
            return true;
        }
    }
    return false;
}

static long long split_wave(int m, int k, long long batch, size_t cxb = sizeof(cx<float>))
{
    const size_t per = (size_t)(4 * k - 1) * ((size_t)1 << m) * cxb;
    // Recommended wave: up to 1.25 GiB of limb and group spectra, rounded so
    // that the contiguous passes fill whole waves of the SMs. Measured at
    // N = 2^16 (k = 5, 4.75 MiB per product), batch 256: waves of 23 / 74 / 256
    // products run 161k / 183k / 198k products/s -- CTAs per launch matter more
    // than keeping a wave inside the 126 MB L2.
    long long w = (long long)((1280ull << 20) / per);
    if (m > EBITS) w = round_wave(w, ((long long)1 << m) / ECTA);
    if (w < 1) w = 1;
    return w < batch ? w : batch;
}

// [2k limb spectra | 2k-1 group spectra] of W products (complex, M each)
static size_t split_ws_bytes(int m, int k, long long W, size_t cxb = sizeof(cx<float>))
{
    return (size_t)(4 * k - 1) * (size_t)W * ((size_t)1 << m) * cxb;
}


template <int L> static int launch_fwd0(const SplitArgs& a, long long ctas, cudaStream_t s)
{
    static int done[64] = {0};
    return launch_split(split_fwd0<L>, done, a, ctas, s);
}
template <int L> static int launch_inv0(const SplitArgs& a, long long ctas, cudaStream_t s)
{
    static int done[64] = {0};
    return launch_split(split_inv0<L>, done, a, ctas, s);
}

// T = float: N = 4 .. 2^22; T = double: N = 4 .. 2^17 (the column-form passes).
template <typename T>
static int split_mul(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch, int input_bits,
                     int non_negative, int limb_bits, int num_limbs, const void* tables, void* ws, size_t ws_bytes,
                     unsigned* max_err, cudaStream_t s, bool reset_err = true)
{
    constexpr bool F32 = sizeof(T) == 4;
    constexpr int PREC = F32 ? 24 : 53;
    if (n_power < 2 || n_power > (F32 ? 22 : 17)) return GPUFFT_ERROR_INVALID_N_POWER;
    if (!a || !b || !c || !tables || batch <= 0 || input_bits < 1 || input_bits > 31) return GPUFFT_ERROR_INVALID_VALUE;
    if ((uintptr_t)a % 4 || (uintptr_t)b % 4 || (uintptr_t)c % 8 || (uintptr_t)tables % 8 || (uintptr_t)ws % 8)
        return GPUFFT_ERROR_MISALIGNED;
    int w = limb_bits, k = num_limbs;
    if (w <= 0 || k <= 0)
    {
        if (!choose_limbs(n_power, input_bits, non_negative != 0, &w, &k, PREC)) return GPUFFT_ERROR_INVALID_VALUE;
    }
    // digits are read from a 64-bit offset value: limbs far above the input
    // range (w (k-1) >= 48) are rejected
    if (k > SPLIT_MAX_LIMBS || w < 1 || w > 20 || (long long)w * k < input_bits || w * (k - 1) >= 48)
        return GPUFFT_ERROR_INVALID_VALUE;
    if (non_negative && input_bits > 30) return GPUFFT_ERROR_INVALID_VALUE;

    const int m = n_power - 1;
    const long long M = 1LL << m;
    if ((uintptr_t)tables % sizeof(cx<T>) || (uintptr_t)ws % sizeof(cx<T>)) return GPUFFT_ERROR_MISALIGNED;
    const auto* tab = reinterpret_cast<const cx<T>*>(tables);
    SplitArgsT<T> A{};
    A.a = a;
    A.b = b;
    A.roots = tab;
    A.inv_roots = tab + M / 2;
    A.twist = tab + M;
    A.untwist = tab + 2 * M;
    A.max_err = max_err;
    A.scale = (T)(1.0 / (double)M);
    A.w = w;
    A.k = k;
    A.K = non_negative ? (1LL << (input_bits - 1)) : 0;
    A.uspec = tab + 3 * M;
    A.uq = (input_bits - 1) / w;
    A.ur = (input_bits - 1) - w * A.uq;
    {
        long long hoff = 0; // 2^(w-1) (1 + 2^w + ... + 2^(w(k-2)))
        for (int i = 0; i + 1 < k; i++) hoff += 1LL << (w * i + w - 1);
        A.voff = hoff - A.K;
        // V = x + voff over the input range (|x| < 2^input_bits, or 0 <= x <
        // 2^input_bits for non-negative inputs)
        const long long xlo = non_negative ? 0 : -(1LL << input_bits) + 1, xhi = (1LL << input_bits) - 1;
        A.dig32 = (xlo + A.voff >= (long long)INT32_MIN && xhi + A.voff <= (long long)INT32_MAX && w * (k - 1) <= 30)
                      ? 1
                      : 0;
        unsigned long long S = 0; // sum_{l<k-1} 2^(w l)
        for (int i = 0; i + 1 < k; i++) S += 1ULL << (w * i);
        const unsigned long long K = (unsigned long long)A.K;
        A.uucoef = (long long)(K * K - K * S);
    }

    // the workspace sets the wave (as many products as it holds, rounded to
    // whole waves of the SMs for the tiled passes)
    const size_t need1 = split_ws_bytes(m, k, 1, sizeof(cx<T>));
    if (!ws || ws_bytes < need1) return GPUFFT_ERROR_WORKSPACE;
    long long W = (long long)(ws_bytes / need1);
    if (W >= batch)
        W = batch;
    else if (m > EBITS)
        W = round_wave(W, M / ECTA);
    if (max_err && reset_err)
    {
        cudaError_t e = cudaMemsetAsync(max_err, 0, sizeof(unsigned), s);
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    const Plan p = make_plan(m);
    for (long long p0 = 0; p0 < batch; p0 += W)
    {
        const long long wv = (batch - p0) < W ? (batch - p0) : W;
        A.a = a + p0 * 2 * M;
        A.b = b + p0 * 2 * M;
        A.c = c + p0 * 2 * M;
        A.W = wv;
        A.batch = wv;
        A.spec = reinterpret_cast<cx<T>*>(ws);
        A.group = A.spec + (size_t)(2 * k) * wv * M;
        if constexpr (F32)
        {
            const long long ctas = (wv * M + ECTA - 1) / ECTA;
            // one kernel (a CTA runs every limb and group transform of its
            // products in turn) once it fills the SMs; fewer products take the
            // chain below, whose passes spread those transforms over CTAs and
            // clusters
            if (m <= EBITS && (m < 10 || ctas >= sm_count()))
            {
                A.geo = PassGeo{};
                A.geo.m = m;
                if (k > SPLIT_SINGLE_MAX_LIMBS) return GPUFFT_ERROR_INVALID_VALUE;
                int st = (m <= 6)   ? launch_split_single_lo(m, A, ctas, s)
                         : (m <= 9) ? launch_split_single_mid(m, A, ctas, s)
                                    : launch_split_single_hi(m, A, ctas, s);
                if (st) return st;
                continue;
            }
        }
        long long ctas = 0;
        if constexpr (F32)
        {
            if (split_tile_ok(m, k, wv) && (reinterpret_cast<uintptr_t>(ws) & 15) == 0)
            {
                // column kernels for the first / last m - 11 stages around the
                // tile kernel's eleven contiguous stages of every limb and group
                const int L0 = m - SPLIT_TILE_LT;
                A.geo = PassGeo{};
                A.geo.m = m;
                int st;
                if (L0 == SPLIT_COL_MAX)
                {
                    // 16-point columns: each column on two lanes (half the registers)
                    const long long threads = 2 * (2 * wv * (M >> L0));
                    const unsigned blocks = (unsigned)((threads + SPLIT_COL2_THREADS - 1) / SPLIT_COL2_THREADS);
                    GF_TRACE(tr, (double)wv * M * (2 * 2 * 4 + 2 * k * sizeof(cx<T>)), s,
                             "split_fwd0_col2<f32,L%d,k%d>", L0, k);
                    st = dispatch_int<1, SPLIT_TILE_MAXK>(k, [&]<int KK>() {
                        return A.dig32 ? launch_k(split_fwd0_col2<SPLIT_COL_MAX, KK, true>, blocks,
                                                  SPLIT_COL2_THREADS, 0, s, A)
                                       : launch_k(split_fwd0_col2<SPLIT_COL_MAX, KK, false>, blocks,
                                                  SPLIT_COL2_THREADS, 0, s, A);
                    });
                }
                else
                {
                    const long long threads = 2 * wv * (M >> L0);
                    const unsigned blocks = (unsigned)((threads + SPLIT_COL_THREADS - 1) / SPLIT_COL_THREADS);
                    GF_TRACE(tr, (double)wv * M * (2 * 2 * 4 + 2 * k * sizeof(cx<T>)), s,
                             "split_fwd0_col<f32,L%d,k%d>", L0, k);
                    st = dispatch_int<1, SPLIT_COL_MAX - 1>(L0, [&]<int LL>() {
                        return dispatch_int<1, SPLIT_TILE_MAXK>(k, [&]<int KK>() {
                            return launch_k(split_fwd0_col<T, LL, KK>, blocks, SPLIT_COL_THREADS, 0, s, A);
                        });
                    });
                }
                if (st) return st;
                st = launch_split_tile(k, A, wv * (M >> SPLIT_TILE_LT), s);
                if (st) return st;
                if (L0 == SPLIT_COL_MAX)
                {
                    const long long threads = 2 * (wv * (M >> L0));
                    const unsigned blocks = (unsigned)((threads + SPLIT_COL2_THREADS - 1) / SPLIT_COL2_THREADS);
                    GF_TRACE(tr, (double)wv * M * ((2 * k - 1) * sizeof(cx<T>) + 2 * 8), s,
                             "split_inv0_col2<f32,L%d,k%d>", L0, k);
                    st = dispatch_int<1, SPLIT_TILE_MAXK>(k, [&]<int KK>() {
                        return launch_k(split_inv0_col2<SPLIT_COL_MAX, KK>, blocks, SPLIT_COL2_THREADS, 0, s, A);
                    });
                }
                else
                {
                    const long long threads = wv * (M >> L0);
                    const unsigned blocks = (unsigned)((threads + SPLIT_COL_THREADS - 1) / SPLIT_COL_THREADS);
                    GF_TRACE(tr, (double)wv * M * ((2 * k - 1) * sizeof(cx<T>) + 2 * 8), s,
                             "split_inv0_col<f32,L%d,k%d>", L0, k);
                    st = dispatch_int<1, SPLIT_COL_MAX - 1>(L0, [&]<int LL>() {
                        return dispatch_int<1, SPLIT_TILE_MAXK>(k, [&]<int KK>() {
                            return launch_k(split_inv0_col<T, LL, KK>, blocks, SPLIT_COL_THREADS, 0, s, A);
                        });
                    });
                }
                if (st) return st;
                continue;
            }
        }
        // rings with one pass (FP64, and FP32 batches too small to fill the
        // SMs) run a zero-stage column form (digits, fold, twist) around that
        // single contiguous pass
        const int L0 = p.np == 1 ? 0 : p.L[0];
        const int kc = p.np == 1 ? 0 : 1; // the contiguous pass
        // 1. limb extraction + first forward pass (strided), all 2k limbs of a column block
        A.geo = pass_geo(p, 0, m, 0, 2 * wv, &ctas);
        A.geo.m = m;
        int st;
        if (L0 <= SPLIT_COL_MAX)
        {
            const long long threads = 2 * wv * (M >> L0);
            const unsigned blocks = (unsigned)((threads + SPLIT_COL_THREADS - 1) / SPLIT_COL_THREADS);
            // int32 rows of both operands in, 2k limb spectra out
            GF_TRACE(tr, (double)wv * M * (2 * 2 * 4 + 2 * k * sizeof(cx<T>)), s, "split_fwd0_col<%s,L%d,k%d>",
                     F32 ? "f32" : "f64", L0, k);
            st = dispatch_int<0, SPLIT_COL_MAX>(L0, [&]<int LL>() {
                return dispatch_int<1, SPLIT_MAX_LIMBS>(k, [&]<int KK>() {
                    return launch_k(split_fwd0_col<T, LL, KK>, blocks, SPLIT_COL_THREADS, 0, s, A);
                });
            });
        }
        else if constexpr (F32)
        {
            st = dispatch_int<1, 9>(L0, [&]<int LL>() { return launch_fwd0<LL>(A, ctas, s); });
        }
        else
        {
            return GPUFFT_ERROR_INVALID_N_POWER;
        }
        if (st) return st;
        // 2. last forward pass of the 2k W limb spectra, in place
        {
            PassArgs<T> q{};
            q.geo = pass_geo(p, kc, m, 0, 2 * k * wv, &ctas);
            q.in = A.spec;
            q.out = A.spec;
            q.table = A.roots;
            q.batch = 2 * k * wv;
            q.in_kind = IN_CPX;
            q.out_kind = OUT_CPX;
            q.perm = m > EBITS; // the spectra are only read pointwise and by the inverse pass
            st = launch_pass<T, true>(q, p, kc, ctas, s);
            if (st) return st;
        }
        // 3. group sums (a streaming kernel), then the first inverse pass of the
        //    (2k-1) W groups in place
        {
            const long long pts = wv * M;
            {
                // 2k limb spectra in, 2k-1 group spectra out
                GF_TRACE(tr, (double)pts * sizeof(cx<T>) * (4 * k - 1), s, "split_groups<%s,k%d>",
                         F32 ? "f32" : "f64", k);
                st = dispatch_int<1, SPLIT_MAX_LIMBS>(k, [&]<int KK>() {
                    return launch_k(split_groups<T, KK>, (unsigned)((pts + 255) / 256), 256, 0, s, A);
                });
            }
            if (st) return st;
            PassArgs<T> q{};
            q.geo = pass_geo(p, kc, m, 0, (2 * k - 1) * wv, &ctas);
            q.in = A.group;
            q.out = A.group;
            q.table = A.inv_roots;
            q.batch = (2 * k - 1) * wv;
            q.in_kind = IN_CPX;
            q.out_kind = OUT_CPX;
            q.perm = m > EBITS;
            st = launch_pass<T, false>(q, p, kc, ctas, s);
            if (st) return st;
        }
        // 4. last inverse pass of every group (strided), rounding, int64 recombination
        A.geo = pass_geo(p, 0, m, 0, wv, &ctas);
        A.geo.m = m;
        if (L0 <= SPLIT_COL_MAX)
        {
            const long long threads = wv * (M >> L0);
            const unsigned blocks = (unsigned)((threads + SPLIT_COL_THREADS - 1) / SPLIT_COL_THREADS);
            // 2k-1 group spectra in, int64 rows out
            GF_TRACE(tr, (double)wv * M * ((2 * k - 1) * sizeof(cx<T>) + 2 * 8), s, "split_inv0_col<%s,L%d,k%d>",
                     F32 ? "f32" : "f64", L0, k);
            st = dispatch_int<0, SPLIT_COL_MAX>(L0, [&]<int LL>() {
                return dispatch_int<1, SPLIT_MAX_LIMBS>(k, [&]<int KK>() {
                    return launch_k(split_inv0_col<T, LL, KK>, blocks, SPLIT_COL_THREADS, 0, s, A);
                });
            });
        }
        else if constexpr (F32)
        {
            st = dispatch_int<1, 9>(L0, [&]<int LL>() { return launch_inv0<LL>(A, ctas, s); });
        }
        else
        {
            return GPUFFT_ERROR_INVALID_N_POWER;
        }
        if (st) return st;
    }
    return GPUFFT_SUCCESS;
}

// Host-buffer variant: chunks staged through the workspace with the transfers
// overlapped (gf_pipe.cuh); the error report is the maximum over all chunks.
static long long split_host_chunk(int n_power, int k, long long batch, long long chunk)
{
    if (chunk > 0) return chunk < batch ? chunk : batch;
    return pipe_chunk(split_wave(n_power - 1, k, batch), batch);
}

static int split_mul_host(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch, int chunk,
                          int input_bits, int non_negative, int limb_bits, int num_limbs, const void* tables, void* ws,
                          size_t ws_bytes, unsigned* max_err, cudaStream_t s)
{
    if (n_power < 2 || n_power > 22) return GPUFFT_ERROR_INVALID_N_POWER;
    if (batch <= 0 || input_bits < 1 || input_bits > 31) return GPUFFT_ERROR_INVALID_VALUE;
    int w = limb_bits, k = num_limbs;
    if (w <= 0 || k <= 0)
    {
        if (!choose_limbs(n_power, input_bits, non_negative != 0, &w, &k)) return GPUFFT_ERROR_INVALID_VALUE;
    }
    if (k > SPLIT_MAX_LIMBS) return GPUFFT_ERROR_INVALID_VALUE;
    const long long ch = split_host_chunk(n_power, k, batch, chunk);
    const size_t in_row = sizeof(int32_t) << n_power, out_row = sizeof(int64_t) << n_power;
    const size_t slots = pipe_bytes(ch, in_row, out_row);
    if (!ws || ws_bytes < slots) return GPUFFT_ERROR_WORKSPACE;
    if (max_err)
    {
        cudaError_t e = cudaMemsetAsync(max_err, 0, sizeof(unsigned), s);
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    void* sws = static_cast<char*>(ws) + slots;
    const size_t sws_bytes = ws_bytes - slots;
    return run_pipeline(a, b, c, batch, ch, in_row, out_row, ws, slots, s,
                        [&](void* da, void* db, void* dc, long long rows, cudaStream_t st) {
                            return split_mul<float>(static_cast<const int32_t*>(da), static_cast<const int32_t*>(db),
                                             static_cast<int64_t*>(dc), n_power, (int)rows, input_bits, non_negative,
                                             w, k, tables, sws, sws_bytes, max_err, st, false);
                        });
}

} // namespace gfb

extern "C" int gpufft_set_split_tile(int on)
{
    if (on < 0) return gfb::g_split_tile.load();
    return gfb::g_split_tile.exchange(on ? 1 : 0);
}

extern "C" int gpufft_split_plan(int n_power, int input_bits, int non_negative, int* limb_bits, int* num_limbs)
{
    if (!limb_bits || !num_limbs || input_bits < 1 || input_bits > 31) return GPUFFT_ERROR_INVALID_VALUE;
    if (n_power < 2 || n_power > 22) return GPUFFT_ERROR_INVALID_N_POWER;
    return gfb::choose_limbs(n_power, input_bits, non_negative != 0, limb_bits, num_limbs) ? GPUFFT_SUCCESS
                                                                                          : GPUFFT_ERROR_INVALID_VALUE;
}

extern "C" size_t gpufft_negacyclic_mul_split_workspace_bytes(int n_power, int batch, int num_limbs)
{
    if (n_power < 2 || n_power > 22 || batch <= 0 || num_limbs < 1 || num_limbs > gfb::SPLIT_MAX_LIMBS) return 0;
    const int m = n_power - 1;
    const long long W = gfb::split_wave(m, num_limbs, batch);
    return gfb::split_ws_bytes(m, num_limbs, W);
}

extern "C" int gpufft_negacyclic_mul_split_f32(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch,
                                               int input_bits, int non_negative, int limb_bits, int num_limbs,
                                               const void* tables, void* workspace, size_t workspace_bytes,
                                               float* max_error, gpufft_stream_t stream)
{
    return gfb::split_mul<float>(a, b, c, n_power, batch, input_bits, non_negative, limb_bits, num_limbs, tables, workspace,
                          workspace_bytes, reinterpret_cast<unsigned*>(max_error), (cudaStream_t)stream);
}

// FP64 split product: the same chain with double transforms; its error model
// (2^-53) takes far fewer limbs (two 12-bit limbs for 24-bit coefficients at
// N = 2^16: 7 transforms per product instead of 19).
extern "C" int gpufft_split_plan_f64(int n_power, int input_bits, int non_negative, int* limb_bits, int* num_limbs)
{
    if (!limb_bits || !num_limbs || input_bits < 1 || input_bits > 31) return GPUFFT_ERROR_INVALID_VALUE;
    if (n_power < 2 || n_power > 17) return GPUFFT_ERROR_INVALID_N_POWER;
    return gfb::choose_limbs(n_power, input_bits, non_negative != 0, limb_bits, num_limbs, 53)
               ? GPUFFT_SUCCESS
               : GPUFFT_ERROR_INVALID_VALUE;
}

extern "C" size_t gpufft_negacyclic_mul_split_f64_workspace_bytes(int n_power, int batch, int num_limbs)
{
    if (n_power < 2 || n_power > 17 || batch <= 0 || num_limbs < 1 || num_limbs > gfb::SPLIT_MAX_LIMBS) return 0;
    const int m = n_power - 1;
    const long long W = gfb::split_wave(m, num_limbs, batch, sizeof(gfb::cx<double>));
    return gfb::split_ws_bytes(m, num_limbs, W, sizeof(gfb::cx<double>));
}

extern "C" int gpufft_negacyclic_mul_split_f64(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch,
                                               int input_bits, int non_negative, int limb_bits, int num_limbs,
                                               const void* tables, void* workspace, size_t workspace_bytes,
                                               float* max_error, gpufft_stream_t stream)
{
    return gfb::split_mul<double>(a, b, c, n_power, batch, input_bits, non_negative, limb_bits, num_limbs, tables,
                                  workspace, workspace_bytes, reinterpret_cast<unsigned*>(max_error),
                                  (cudaStream_t)stream);
}

extern "C" size_t gpufft_negacyclic_mul_split_f32_host_workspace_bytes(int n_power, int batch, int chunk,
                                                                       int num_limbs)
{
    if (n_power < 2 || n_power > 22 || batch <= 0 || num_limbs < 1 || num_limbs > gfb::SPLIT_MAX_LIMBS) return 0;
    const long long ch = gfb::split_host_chunk(n_power, num_limbs, batch, chunk);
    return gfb::pipe_bytes(ch, sizeof(int32_t) << n_power, sizeof(int64_t) << n_power) +
           gpufft_negacyclic_mul_split_workspace_bytes(n_power, (int)ch, num_limbs);
}

extern "C" int gpufft_negacyclic_mul_split_f32_host(const int32_t* a, const int32_t* b, int64_t* c, int n_power,
                                                    int batch, int chunk, int input_bits, int non_negative,
                                                    int limb_bits, int num_limbs, const void* tables,
                                                    void* workspace, size_t workspace_bytes, float* max_error,
                                                    gpufft_stream_t stream)
{
    return gfb::split_mul_host(a, b, c, n_power, batch, chunk, input_bits, non_negative, limb_bits, num_limbs, tables,
                               workspace, workspace_bytes, reinterpret_cast<unsigned*>(max_error),
                               (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Mixed ring sizes, exact: the split product over a packed batch of requests
// of different ring sizes. Requests are grouped by size (class-major, original
// order inside a class, the same layout as gpufft_batch_plan); each class runs
// the split chain with its own limb plan and twiddles, all on one stream, and
// capture/replay puts the whole batch in one CUDA graph.
// ---------------------------------------------------------------------------
namespace gfb
{
struct SplitClass
{
    int n_power, w, k;
    long long count, off; // requests, coefficient offset of the class
    size_t tab_off;       // complex-float offset of its twiddle block
};

struct SplitBatchPlan
{
    int input_bits = 0, non_negative = 0, count = 0, device = 0;
    std::vector<int> n_powers;
    std::vector<long long> offsets;
    std::vector<SplitClass> classes;
    long long total = 0;
    void* d_tabs = nullptr;
    void* d_ws = nullptr;
    size_t ws_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static void free_split_plan(SplitBatchPlan* P)
{
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    cudaFree(P->d_tabs);
    cudaFree(P->d_ws);
    delete P;
}

static int split_batch_create(SplitBatchPlan** out, const int* n_powers, int count, int input_bits, int non_negative,
                              cudaStream_t s)
{
    if (!out || !n_powers || count <= 0 || input_bits < 1 || input_bits > 31) return GPUFFT_ERROR_INVALID_VALUE;
    for (int i = 0; i < count; i++)
        if (n_powers[i] < 2 || n_powers[i] > 22) return GPUFFT_ERROR_INVALID_N_POWER;
    auto* P = new SplitBatchPlan();
    P->input_bits = input_bits;
    P->non_negative = non_negative != 0;
    P->count = count;
    P->n_powers.assign(n_powers, n_powers + count);
    P->offsets.assign(count, 0);
    cudaGetDevice(&P->device);
    std::map<int, std::vector<int>> by;
    for (int i = 0; i < count; i++) by[n_powers[i]].push_back(i);
    long long coef = 0;
    size_t tab = 0, ws = 0;
    for (auto& kv : by)
    {
        SplitClass C{};
        C.n_power = kv.first;
        if (!choose_limbs(C.n_power, input_bits, P->non_negative, &C.w, &C.k))
        {
            delete P;
            return GPUFFT_ERROR_INVALID_VALUE;
        }
        C.count = (long long)kv.second.size();
        C.off = coef;
        C.tab_off = tab;
        for (int r : kv.second)
        {
            P->offsets[r] = coef;
            coef += 1LL << C.n_power;
        }
        tab += gpufft_ffnt_tables_count(C.n_power);
        const int m = C.n_power - 1;
        ws = std::max(ws, split_ws_bytes(m, C.k, split_wave(m, C.k, C.count)));
        P->classes.push_back(C);
    }
    P->total = coef;
    P->ws_bytes = ws;
    cudaError_t e = cudaMalloc(&P->d_tabs, tab * sizeof(cx<float>));
    if (e == cudaSuccess) e = cudaMalloc(&P->d_ws, std::max<size_t>(ws, 256));
    if (e != cudaSuccess)
    {
        free_split_plan(P);
        return set_cuda_error(e);
    }
    for (const SplitClass& C : P->classes)
    {
        const int st = gpufft_ffnt_make_tables_f32(C.n_power, static_cast<cx<float>*>(P->d_tabs) + C.tab_off, s);
        if (st)
        {
            free_split_plan(P);
            return st;
        }
    }
    *out = P;
    return GPUFFT_SUCCESS;
}

static int split_batch_execute(SplitBatchPlan* P, const int32_t* a, const int32_t* b, int64_t* c, unsigned* max_err,
                               cudaStream_t s)
{
    if (!a || !b || !c) return GPUFFT_ERROR_INVALID_VALUE;
    bool first = true;
    for (const SplitClass& C : P->classes)
    {
        const int st = split_mul<float>(a + C.off, b + C.off, c + C.off, C.n_power, (int)C.count, P->input_bits,
                                 P->non_negative, C.w, C.k, static_cast<cx<float>*>(P->d_tabs) + C.tab_off, P->d_ws,
                                 P->ws_bytes, max_err, s, first);
        if (st) return st;
        first = false;
    }
    return GPUFFT_SUCCESS;
}
} // namespace gfb

struct gpufft_split_batch_plan_s
{
    gfb::SplitBatchPlan* p;
};

extern "C" int gpufft_split_batch_plan_create(gpufft_split_batch_plan* plan, const int* n_powers, int count,
                                              int input_bits, int non_negative, gpufft_stream_t stream)
{
    if (!plan) return GPUFFT_ERROR_INVALID_VALUE;
    gfb::SplitBatchPlan* P = nullptr;
    const int st = gfb::split_batch_create(&P, n_powers, count, input_bits, non_negative, (cudaStream_t)stream);
    if (st) return st;
    *plan = new gpufft_split_batch_plan_s{P};
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_split_batch_plan_layout(gpufft_split_batch_plan plan, long long* offsets, long long* total,
                                              int* limb_bits, int* num_limbs)
{
    if (!plan || !offsets || !total) return GPUFFT_ERROR_INVALID_VALUE;
    const gfb::SplitBatchPlan* P = plan->p;
    for (int i = 0; i < P->count; i++)
    {
        offsets[i] = P->offsets[i];
        if (limb_bits || num_limbs)
            for (const auto& C : P->classes)
                if (C.n_power == P->n_powers[i])
                {
                    if (limb_bits) limb_bits[i] = C.w;
                    if (num_limbs) num_limbs[i] = C.k;
                }
    }
    *total = P->total;
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_split_batch_plan_execute(gpufft_split_batch_plan plan, const int32_t* a, const int32_t* b,
                                               int64_t* c, float* max_error, gpufft_stream_t stream)
{
    if (!plan) return GPUFFT_ERROR_INVALID_VALUE;
    return gfb::split_batch_execute(plan->p, a, b, c, reinterpret_cast<unsigned*>(max_error), (cudaStream_t)stream);
}

extern "C" int gpufft_split_batch_plan_capture(gpufft_split_batch_plan plan, const int32_t* a, const int32_t* b,
                                               int64_t* c, float* max_error, gpufft_stream_t stream)
{
    if (!plan || !stream) return GPUFFT_ERROR_INVALID_VALUE;
    gfb::SplitBatchPlan* P = plan->p;
    cudaStream_t s = (cudaStream_t)stream;
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    P->exec = nullptr;
    P->graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return gfb::set_cuda_error(e);
    const int st = gfb::split_batch_execute(P, a, b, c, reinterpret_cast<unsigned*>(max_error), s);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    if (st)
    {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return gfb::set_cuda_error(e);
    P->graph = g;
    e = cudaGraphInstantiate(&P->exec, g, 0);
    if (e != cudaSuccess) return gfb::set_cuda_error(e);
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_split_batch_plan_replay(gpufft_split_batch_plan plan, gpufft_stream_t stream)
{
    if (!plan || !plan->p->exec) return GPUFFT_ERROR_INVALID_VALUE;
    const cudaError_t e = cudaGraphLaunch(plan->p->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? GPUFFT_SUCCESS : gfb::set_cuda_error(e);
}

extern "C" int gpufft_split_batch_plan_destroy(gpufft_split_batch_plan plan)
{
    if (!plan) return GPUFFT_ERROR_INVALID_VALUE;
    gfb::free_split_plan(plan->p);
    delete plan;
    return GPUFFT_SUCCESS;
}
