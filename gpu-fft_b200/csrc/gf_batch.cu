// gpufft-b200: batched negacyclic products of mixed ring sizes in one
// persistent launch (captured in a CUDA graph), with an autotuned launch shape.
//
// A plan groups its requests by ring size ("classes", N = 2^2 .. 2^17). The
// caller packs the operands class by class (gpufft_batch_plan_order gives the
// order and the coefficient offsets). One cooperative launch then runs three
// phases separated by a grid barrier:
//   phase 1: every product of rings N <= 8192 (fused_body SINGLE: one tile of
//            4096/(N/2) products, whole transforms, fold/twist and
//            untwist/unfold fused) and the first forward pass of the larger
//            rings (pass_body, strided, fold + twist in the load);
//   phase 2: the fused middle pass of the larger rings (forward of both
//            operands, product, inverse);
//   phase 3: the last inverse pass of the larger rings (strided, scale +
//            untwist + unfold in the store).
// Work items (one CTA tile each) are taken from a per-phase device counter, so
// the uneven sizes balance dynamically. Every item runs exactly the device code
// of the single-size entry points, so the outputs are identical to per-size
// gpufft_negacyclic_mul_* calls on the same data.
//
// The grid barrier is a monotonic arrival counter with a bounded wait: a CTA
// that waits longer than the plan's poll limit (BARRIER_MAX_POLLS unless
// gpufft_batch_plan_set_barrier changed it) sets the plan's timeout flag and
// continues (the launch is cooperative, so all CTAs are co-resident and the
// barrier normally completes in microseconds); gpufft_batch_plan_status
// reports the flag.
//
// Autotuning: the launch shape (CTAs per SM, and how many work items a CTA
// takes per counter update) and, as one more candidate, per-class fused chains
// instead of the persistent kernel, are timed on the caller's data and the
// fastest is kept, cached in a JSON file keyed by GPU name, driver version,
// precision and the size histogram.
#include "gf_fused.cuh"

#include <cmath>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace gfb
{

constexpr int BATCH_MIN_NPOWER = 2;
constexpr int BATCH_MAX_NPOWER = 17; // two-pass rings with a first pass of <= 4 stages
constexpr unsigned BARRIER_MAX_POLLS = 1u << 26;

struct BatchClass
{
    int m;              // log2 transform length (N = 2^(m+1))
    int L1;             // stages of the first pass (0: one-pass ring)
    long long count;    // products of this size
    long long coef_off; // offset of the class's first row in a/b/c (coefficients)
    long long ws_off;   // offset of the class's spectra in the workspace (complex)
    long long tab_off;  // offset of the class's twiddle block in the table arena (complex)
};

struct WorkItem
{
    unsigned short kind; // 0 one-pass product tile, 1 first forward pass, 2 fused middle, 3 last inverse pass
    unsigned short cls;
    unsigned tile;
};

template <typename T> struct BatchArgs
{
    const T* a;
    const T* b;
    T* c;
    cx<T>* ws;
    const cx<T>* tabs;
    const BatchClass* classes;
    const WorkItem* items[3];
    unsigned nitems[3];
    unsigned* counters; // [3] work counters, [3] barrier arrivals, [1] timeout flag
    int grab;
    unsigned max_polls;     // polls before a grid barrier gives up
    unsigned barrier_extra; // arrivals a barrier waits for beyond the grid (0; raised only to test the timeout)
};

__device__ __forceinline__ void grid_barrier(unsigned* arrivals, unsigned target, unsigned* flag, unsigned max_polls)
{
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        atomicAdd(arrivals, 1u);
        unsigned polls = 0;
        while (*((volatile unsigned*)arrivals) < target)
        {
            if (++polls > max_polls)
            {
                atomicExch(flag, 1u);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
}

template <typename T>
__device__ __forceinline__ void run_item(const BatchArgs<T>& A, const WorkItem it, cx<T>* sm)
{
    const BatchClass C = A.classes[it.cls];
    const long long M = 1LL << C.m;
    const cx<T>* tab = A.tabs + C.tab_off;
    if (it.kind == 0 || it.kind == 2)
    {
        FusedArgs<T> f{};
        f.roots = tab;
        f.inv_roots = tab + M / 2;
        f.twist = tab + M;
        f.untwist = tab + 2 * M;
        f.scale = (T)(1.0 / (double)M);
        f.geo.m = C.m;
        if (it.kind == 0)
        {
            f.a = A.a + C.coef_off;
            f.b = A.b + C.coef_off;
            f.c = A.c + C.coef_off;
            f.batch = C.count;
            switch (C.m)
            {
#define GFB_SINGLE_CASE(LL)                                                                                            \
    case LL: fused_body<T, LL, true>(f, it.tile, sm); break;
                GFB_SINGLE_CASE(1)
                GFB_SINGLE_CASE(2)
                GFB_SINGLE_CASE(3)
                GFB_SINGLE_CASE(4)
                GFB_SINGLE_CASE(5)
                GFB_SINGLE_CASE(6)
                GFB_SINGLE_CASE(7)
                GFB_SINGLE_CASE(8)
                GFB_SINGLE_CASE(9)
                GFB_SINGLE_CASE(10)
                GFB_SINGLE_CASE(11)
                GFB_SINGLE_CASE(12)
#undef GFB_SINGLE_CASE
            default: break;
            }
        }
        else
        {
            f.ws = A.ws + C.ws_off;
            f.batch = C.count;
            f.geo.s0 = C.L1;
            fused_body<T, EBITS, false>(f, it.tile, sm);
        }
        return;
    }
    PassArgs<T> p{};
    p.geo.m = C.m;
    p.geo.s0 = 0;
    p.table = (it.kind == 1) ? tab : tab + M / 2;
    if (it.kind == 1)
    {
        p.in = A.a + C.coef_off;
        p.in2 = A.b + C.coef_off;
        p.split = C.count;
        p.out = A.ws + C.ws_off;
        p.twist = tab + M;
        p.batch = 2 * C.count;
        p.in_kind = IN_FOLD2;
        p.out_kind = OUT_CPX;
        switch (C.L1)
        {
        case 1: pass_body<T, true, 1, true>(p, it.tile, sm); break;
        case 2: pass_body<T, true, 2, true>(p, it.tile, sm); break;
        case 3: pass_body<T, true, 3, true>(p, it.tile, sm); break;
        case 4: pass_body<T, true, 4, true>(p, it.tile, sm); break;
        default: break;
        }
    }
    else
    {
        p.in = A.ws + C.ws_off;
        p.out = A.c + C.coef_off;
        p.twist = tab + 2 * M;
        p.scale = mk<T>((T)(1.0 / (double)M), T(0));
        p.do_scale = 1;
        p.batch = C.count;
        p.in_kind = IN_CPX;
        p.out_kind = OUT_UNFOLD;
        switch (C.L1)
        {
        case 1: pass_body<T, false, 1, true>(p, it.tile, sm); break;
        case 2: pass_body<T, false, 2, true>(p, it.tile, sm); break;
        case 3: pass_body<T, false, 3, true>(p, it.tile, sm); break;
        case 4: pass_body<T, false, 4, true>(p, it.tile, sm); break;
        default: break;
        }
    }
}

template <typename T, int MINB> __global__ void __launch_bounds__(NTHR, MINB) batch_kernel(const BatchArgs<T> A)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
    __shared__ unsigned s_base;
    for (int ph = 0; ph < 3; ph++)
    {
        for (;;)
        {
            if (threadIdx.x == 0) s_base = atomicAdd(&A.counters[ph], (unsigned)A.grab);
            __syncthreads();
            const unsigned base = s_base;
            __syncthreads();
            if (base >= A.nitems[ph]) break;
            for (int g = 0; g < A.grab; g++)
            {
                const unsigned i = base + g;
                if (i >= A.nitems[ph]) break;
                run_item<T>(A, A.items[ph][i], sm);
                __syncthreads(); // the next item reuses shared memory
            }
        }
        if (ph < 2) grid_barrier(&A.counters[3 + ph], gridDim.x + A.barrier_extra, &A.counters[6], A.max_polls);
    }
}

// ---------------------------------------------------------------------------
// host side: the plan
// ---------------------------------------------------------------------------
struct BatchPlan
{
    int precision; // 32 or 64
    int count;
    std::vector<int> n_powers;
    std::vector<int> order;          // class-major request order
    std::vector<long long> offsets;  // coefficient offset of each request (in request index order)
    std::vector<BatchClass> classes; // host copy
    unsigned nitems[3] = {0, 0, 0};
    void* d_tabs = nullptr;
    void* d_ws = nullptr;
    void* d_classes = nullptr;
    void* d_items = nullptr;
    unsigned* d_counters = nullptr;
    size_t ws_bytes = 0, tab_bytes = 0;
    int minb = 1, grab = 1, grid = 0;
    unsigned max_polls = BARRIER_MAX_POLLS, barrier_extra = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
};

template <typename T, int MINB> static int batch_smem_setup(size_t* smem)
{
    *smem = 2 * sizeof(cx<T>) * SMEM_ELEMS; // the fused bodies use two transpose buffers
    static int done[64] = {0};
    return ensure_smem(batch_kernel<T, MINB>, *smem, done);
}

template <typename T, int MINB> static int batch_launch(BatchPlan* P, const void* a, const void* b, void* c,
                                                        cudaStream_t s)
{
    size_t smem = 0;
    int st = batch_smem_setup<T, MINB>(&smem);
    if (st) return st;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<T, MINB>, NTHR, smem);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (per_sm < 1) return set_cuda_error(cudaErrorLaunchOutOfResources);
    const int grid = sm_count() * std::min(per_sm, MINB);
    P->grid = grid;
    BatchArgs<T> A{};
    A.a = static_cast<const T*>(a);
    A.b = static_cast<const T*>(b);
    A.c = static_cast<T*>(c);
    A.ws = static_cast<cx<T>*>(P->d_ws);
    A.tabs = static_cast<const cx<T>*>(P->d_tabs);
    A.classes = static_cast<const BatchClass*>(P->d_classes);
    const WorkItem* items = static_cast<const WorkItem*>(P->d_items);
    A.items[0] = items;
    A.items[1] = items + P->nitems[0];
    A.items[2] = items + P->nitems[0] + P->nitems[1];
    for (int i = 0; i < 3; i++) A.nitems[i] = P->nitems[i];
    A.counters = P->d_counters;
    A.grab = P->grab;
    A.max_polls = P->max_polls;
    A.barrier_extra = P->barrier_extra;
    // work counters and barrier arrivals start at zero every execution (the
    // timeout flag, slot 6, is cleared only by gpufft_batch_plan_status)
    e = cudaMemsetAsync(P->d_counters, 0, 6 * sizeof(unsigned), s);
    if (e != cudaSuccess) return set_cuda_error(e);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(NTHR);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    double coeffs = 0;
    for (int np : P->n_powers) coeffs += std::ldexp(1.0, np);
    // a and b read, c written once each
    GF_TRACE(tr, 3.0 * coeffs * sizeof(T), s, "batch_kernel<%s,%d CTA/SM>", sizeof(T) == 4 ? "f32" : "f64", MINB);
    e = cudaLaunchKernelEx(&cfg, batch_kernel<T, MINB>, A);
    if (e != cudaSuccess) return set_cuda_error(e);
    return check_launch();
}

// The other execution mode: one fused product chain per size class (the
// single-size entry point on the class's rows, twiddles and workspace),
// launched back to back on the stream. The persistent kernel keeps one CTA of
// 8 warps per SM for every phase (its fused middle needs the registers), while
// the per-class chains run their first and last passes as high-occupancy
// column kernels; the autotuner times both.
static int class_chains(BatchPlan* P, const void* a, const void* b, void* c, cudaStream_t s)
{
    const size_t cxb = P->precision == 64 ? 16 : 8, eb = cxb / 2;
    for (const BatchClass& C : P->classes)
    {
        const long long M = 1LL << C.m;
        const char* pa = static_cast<const char*>(a) + C.coef_off * eb;
        const char* pb = static_cast<const char*>(b) + C.coef_off * eb;
        char* pc = static_cast<char*>(c) + C.coef_off * eb;
        const void* tab = static_cast<const char*>(P->d_tabs) + C.tab_off * cxb;
        void* ws = C.m > EBITS ? static_cast<char*>(P->d_ws) + C.ws_off * cxb : nullptr;
        const size_t wsb = C.m > EBITS ? (size_t)(2 * C.count * M) * cxb : 0;
        const int st = P->precision == 64
                           ? gpufft_negacyclic_mul_f64(reinterpret_cast<const double*>(pa),
                                                       reinterpret_cast<const double*>(pb),
                                                       reinterpret_cast<double*>(pc), C.m + 1, (int)C.count, tab, ws,
                                                       wsb, s)
                           : gpufft_negacyclic_mul_f32(reinterpret_cast<const float*>(pa),
                                                       reinterpret_cast<const float*>(pb),
                                                       reinterpret_cast<float*>(pc), C.m + 1, (int)C.count, tab, ws,
                                                       wsb, s);
        if (st) return st;
    }
    return GPUFFT_SUCCESS;
}

// minb 0 selects the per-class chains; 1 or 2 the persistent kernel with that
// many CTAs per SM.
static int batch_execute(BatchPlan* P, const void* a, const void* b, void* c, cudaStream_t s)
{
    if (P->minb == 0) return class_chains(P, a, b, c, s);
    if (P->precision == 64) return P->minb == 2 ? batch_launch<double, 2>(P, a, b, c, s) : batch_launch<double, 1>(P, a, b, c, s);
    return P->minb == 2 ? batch_launch<float, 2>(P, a, b, c, s) : batch_launch<float, 1>(P, a, b, c, s);
}

template <typename T> __global__ void batch_tables_kernel(cx<T>* tab, int m)
{
    const long long M = 1LL << m;
    const long long H = M >> 1;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < H)
    {
        double sn, cs;
        native_root(i, m, cs, sn);
        tab[i] = mk<T>((T)cs, (T)sn);
        tab[H + i] = mk<T>((T)cs, (T)-sn);
    }
    if (i < M)
    {
        double sn, cs;
        sincospi((double)i / (double)(2 * M), &sn, &cs);
        tab[2 * H + i] = mk<T>((T)cs, (T)sn);
        tab[2 * H + M + i] = mk<T>((T)cs, (T)-sn);
    }
}

static void free_plan(BatchPlan* P)
{
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    cudaFree(P->d_tabs);
    cudaFree(P->d_ws);
    cudaFree(P->d_classes);
    cudaFree(P->d_items);
    cudaFree(P->d_counters);
    delete P;
}

static int create_plan(BatchPlan** out, const int* n_powers, int count, int precision, cudaStream_t s)
{
    if (!out || !n_powers || count <= 0 || (precision != 32 && precision != 64)) return GPUFFT_ERROR_INVALID_VALUE;
    for (int i = 0; i < count; i++)
        if (n_powers[i] < BATCH_MIN_NPOWER || n_powers[i] > BATCH_MAX_NPOWER) return GPUFFT_ERROR_INVALID_N_POWER;
    auto* P = new BatchPlan();
    P->precision = precision;
    P->count = count;
    P->n_powers.assign(n_powers, n_powers + count);
    cudaGetDevice(&P->device);
    const size_t cxb = precision == 64 ? 16 : 8;

    // classes in ascending size; requests class-major in their original order
    std::map<int, std::vector<int>> by;
    for (int i = 0; i < count; i++) by[n_powers[i]].push_back(i);
    P->offsets.assign(count, 0);
    long long coef = 0, ws = 0, tab = 0;
    std::vector<WorkItem> ph[3];
    for (auto& kv : by)
    {
        BatchClass C{};
        const int np = kv.first;
        C.m = np - 1;
        C.L1 = C.m > EBITS ? C.m - EBITS : 0;
        C.count = (long long)kv.second.size();
        C.coef_off = coef;
        C.ws_off = ws;
        C.tab_off = tab;
        const long long M = 1LL << C.m;
        for (int r : kv.second)
        {
            P->order.push_back(r);
            P->offsets[r] = coef;
            coef += 2 * M;
        }
        const unsigned short cls = (unsigned short)P->classes.size();
        if (C.m <= EBITS)
        {
            const long long tiles = (C.count * M + ECTA - 1) / ECTA;
            for (long long t = 0; t < tiles; t++) ph[0].push_back({0, cls, (unsigned)t});
        }
        else
        {
            const long long per = M / ECTA; // tiles per transform
            for (long long t = 0; t < 2 * C.count * per; t++) ph[0].push_back({1, cls, (unsigned)t});
            for (long long t = 0; t < C.count * per; t++) ph[1].push_back({2, cls, (unsigned)t});
            for (long long t = 0; t < C.count * per; t++) ph[2].push_back({3, cls, (unsigned)t});
            ws += 2 * C.count * M;
        }
        tab += 4 * M;
        P->classes.push_back(C);
    }
    // larger tiles first in phase 1 so the many small tiles fill the tail
    std::stable_sort(ph[0].begin(), ph[0].end(), [&](const WorkItem& x, const WorkItem& y) {
        return P->classes[x.cls].m > P->classes[y.cls].m;
    });
    for (int i = 0; i < 3; i++) P->nitems[i] = (unsigned)ph[i].size();
    std::vector<WorkItem> all;
    for (int i = 0; i < 3; i++) all.insert(all.end(), ph[i].begin(), ph[i].end());

    P->ws_bytes = (size_t)ws * cxb;
    P->tab_bytes = (size_t)tab * cxb;
    cudaError_t e = cudaMalloc(&P->d_tabs, P->tab_bytes);
    if (e == cudaSuccess && P->ws_bytes) e = cudaMalloc(&P->d_ws, P->ws_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&P->d_classes, sizeof(BatchClass) * P->classes.size());
    if (e == cudaSuccess) e = cudaMalloc(&P->d_items, sizeof(WorkItem) * std::max<size_t>(1, all.size()));
    if (e == cudaSuccess) e = cudaMalloc(&P->d_counters, 8 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(P->d_counters, 0, 8 * sizeof(unsigned), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->d_classes, P->classes.data(), sizeof(BatchClass) * P->classes.size(),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !all.empty())
        e = cudaMemcpyAsync(P->d_items, all.data(), sizeof(WorkItem) * all.size(), cudaMemcpyHostToDevice, s);
    for (auto& C : P->classes)
    {
        if (e != cudaSuccess) break;
        const long long M = 1LL << C.m;
        const unsigned blocks = (unsigned)((M + 255) / 256);
        if (precision == 64)
            batch_tables_kernel<double><<<blocks, 256, 0, s>>>(static_cast<cx<double>*>(P->d_tabs) + C.tab_off, C.m);
        else
            batch_tables_kernel<float><<<blocks, 256, 0, s>>>(static_cast<cx<float>*>(P->d_tabs) + C.tab_off, C.m);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s); // host vectors above are released on return
    if (e != cudaSuccess)
    {
        free_plan(P);
        return set_cuda_error(e);
    }
    *out = P;
    return GPUFFT_SUCCESS;
}

static std::string tune_key(const BatchPlan* P)
{
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, P->device);
    int drv = 0;
    cudaDriverGetVersion(&drv);
    std::ostringstream k;
    k << prop.name << "|driver " << drv << "|fp" << P->precision << "|sizes";
    std::map<int, int> h;
    for (int np : P->n_powers) h[np]++;
    for (auto& kv : h) k << " " << kv.first << ":" << kv.second;
    return k.str();
}

// Tiny JSON cache: one object per line {"key": "...", "minb": x, "grab": y, "ms": z}.
static bool cache_lookup(const char* path, const std::string& key, int* minb, int* grab)
{
    if (!path) return false;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line))
    {
        const std::string pat = "\"key\": \"" + key + "\"";
        if (line.find(pat) == std::string::npos) continue;
        int mb = 0, gb = 0;
        const size_t a = line.find("\"minb\": "), b = line.find("\"grab\": ");
        if (a == std::string::npos || b == std::string::npos) continue;
        mb = std::atoi(line.c_str() + a + 8);
        gb = std::atoi(line.c_str() + b + 8);
        if ((mb == 0 || mb == 1 || mb == 2) && gb >= 1 && gb <= 8)
        {
            *minb = mb;
            *grab = gb;
            return true;
        }
    }
    return false;
}

static void cache_store(const char* path, const std::string& key, int minb, int grab, float ms)
{
    if (!path) return;
    std::ofstream f(path, std::ios::app);
    f << "{\"key\": \"" << key << "\", \"minb\": " << minb << ", \"grab\": " << grab << ", \"ms\": " << ms << "}\n";
}

static long long total_coeffs(const BatchPlan* P)
{
    long long t = 0;
    for (int np : P->n_powers) t += 1LL << np;
    return t;
}

static int autotune(BatchPlan* P, const void* a, const void* b, void* c, const char* cache, cudaStream_t s)
{
    const std::string key = tune_key(P);
    int mb = 0, gb = 0;
    if (cache_lookup(cache, key, &mb, &gb))
    {
        P->minb = mb;
        P->grab = gb;
        return GPUFFT_SUCCESS;
    }
    // the product is run about 28 times on the caller's buffers: c must not
    // overlap a or b (the inputs would be overwritten between runs)
    {
        const size_t bytes = (size_t)(P->precision / 8) * (size_t)total_coeffs(P);
        auto overlap = [bytes](const void* x, const void* y) {
            const char* px = static_cast<const char*>(x);
            const char* py = static_cast<const char*>(y);
            return px < py + bytes && py < px + bytes;
        };
        if (overlap(c, a) || overlap(c, b)) return GPUFFT_ERROR_INVALID_VALUE;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    {
        const cudaError_t err = cudaGetLastError();
        if (e0) cudaEventDestroy(e0);
        return set_cuda_error(err);
    }
    float best = 1e30f;
    int bmb = 1, bgb = 1;
    const int minbs[3] = {1, 2, 0};
    const int grabs[3] = {1, 2, 4};
    for (int mbv : minbs)
        for (int gbv : grabs)
        {
            if (mbv == 0 && gbv != 1) continue; // per-class chains take no grab size
            P->minb = mbv;
            P->grab = gbv;
            int st = batch_execute(P, a, b, c, s); // warm-up (also checks the shape launches)
            if (st) continue;
            cudaEventRecord(e0, s);
            for (int r = 0; r < 3; r++) st |= batch_execute(P, a, b, c, s);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess)
            {
                const cudaError_t err = cudaGetLastError();
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return set_cuda_error(err);
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (!st && ms < best)
            {
                best = ms;
                bmb = mbv;
                bgb = gbv;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P->minb = bmb;
    P->grab = bgb;
    cache_store(cache, key, bmb, bgb, best / 3);
    return GPUFFT_SUCCESS;
}

} // namespace gfb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int gpufft_batch_plan_create(gpufft_batch_plan* plan, const int* n_powers, int count, int precision_bits,
                                        gpufft_stream_t stream)
{
    gfb::BatchPlan* P = nullptr;
    const int st = gfb::create_plan(&P, n_powers, count, precision_bits, (cudaStream_t)stream);
    if (st) return st;
    *plan = reinterpret_cast<gpufft_batch_plan>(P);
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_plan_layout(gpufft_batch_plan plan, int* order, long long* offsets, long long* total)
{
    if (!plan) return GPUFFT_ERROR_INVALID_VALUE;
    auto* P = reinterpret_cast<gfb::BatchPlan*>(plan);
    if (order) std::memcpy(order, P->order.data(), sizeof(int) * P->count);
    if (offsets) std::memcpy(offsets, P->offsets.data(), sizeof(long long) * P->count);
    if (total)
    {
        long long t = 0;
        for (int np : P->n_powers) t += 1LL << np;
        *total = t;
    }
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_plan_execute(gpufft_batch_plan plan, const void* a, const void* b, void* c,
                                         gpufft_stream_t stream)
{
    if (!plan || !a || !b || !c) return GPUFFT_ERROR_INVALID_VALUE;
    return gfb::batch_execute(reinterpret_cast<gfb::BatchPlan*>(plan), a, b, c, (cudaStream_t)stream);
}

extern "C" int gpufft_batch_plan_run(gpufft_batch_plan plan, const void* a, const void* b, void* c,
                                     gpufft_stream_t stream)
{
    return gpufft_batch_plan_execute(plan, a, b, c, stream);
}

extern "C" int gpufft_batch_plan_autotune(gpufft_batch_plan plan, const void* a, const void* b, void* c,
                                          const char* cache_path, gpufft_stream_t stream)
{
    if (!plan || !a || !b || !c) return GPUFFT_ERROR_INVALID_VALUE;
    return gfb::autotune(reinterpret_cast<gfb::BatchPlan*>(plan), a, b, c, cache_path, (cudaStream_t)stream);
}

extern "C" int gpufft_batch_plan_capture(gpufft_batch_plan plan, const void* a, const void* b, void* c,
                                         gpufft_stream_t stream)
{
    if (!plan || !a || !b || !c || !stream) return GPUFFT_ERROR_INVALID_VALUE;
    auto* P = reinterpret_cast<gfb::BatchPlan*>(plan);
    cudaStream_t s = (cudaStream_t)stream;
    if (P->exec)
    {
        cudaGraphExecDestroy(P->exec);
        P->exec = nullptr;
    }
    if (P->graph)
    {
        cudaGraphDestroy(P->graph);
        P->graph = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return gfb::set_cuda_error(e);
    const int st = gfb::batch_execute(P, a, b, c, s);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    if (st) return st;
    if (e != cudaSuccess) return gfb::set_cuda_error(e);
    P->graph = g;
    e = cudaGraphInstantiate(&P->exec, g, 0);
    if (e != cudaSuccess) return gfb::set_cuda_error(e);
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_plan_replay(gpufft_batch_plan plan, gpufft_stream_t stream)
{
    if (!plan) return GPUFFT_ERROR_INVALID_VALUE;
    auto* P = reinterpret_cast<gfb::BatchPlan*>(plan);
    if (!P->exec) return GPUFFT_ERROR_INVALID_VALUE;
    const cudaError_t e = cudaGraphLaunch(P->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? GPUFFT_SUCCESS : gfb::set_cuda_error(e);
}

extern "C" int gpufft_batch_plan_set_shape(gpufft_batch_plan plan, int ctas_per_sm, int items_per_grab)
{
    if (!plan || ctas_per_sm < 0 || ctas_per_sm > 2 || items_per_grab < 1 || items_per_grab > 8)
        return GPUFFT_ERROR_INVALID_VALUE;
    auto* P = reinterpret_cast<gfb::BatchPlan*>(plan);
    P->minb = ctas_per_sm;
    P->grab = ctas_per_sm == 0 ? 1 : items_per_grab;
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_plan_info(gpufft_batch_plan plan, int* ctas_per_sm, int* items_per_grab, int* grid,
                                      long long* workspace_bytes)
{
    if (!plan) return GPUFFT_ERROR_INVALID_VALUE;
    auto* P = reinterpret_cast<gfb::BatchPlan*>(plan);
    if (ctas_per_sm) *ctas_per_sm = P->minb;
    if (items_per_grab) *items_per_grab = P->grab;
    if (grid) *grid = P->grid;
    if (workspace_bytes) *workspace_bytes = (long long)P->ws_bytes;
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_plan_set_barrier(gpufft_batch_plan plan, unsigned max_polls, unsigned extra_arrivals)
{
    if (!plan || max_polls < 1 || extra_arrivals > 1024) return GPUFFT_ERROR_INVALID_VALUE;
    auto* P = reinterpret_cast<gfb::BatchPlan*>(plan);
    P->max_polls = max_polls;
    P->barrier_extra = extra_arrivals;
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_plan_status(gpufft_batch_plan plan, int* barrier_timeouts)
{
    if (!plan || !barrier_timeouts) return GPUFFT_ERROR_INVALID_VALUE;
    auto* P = reinterpret_cast<gfb::BatchPlan*>(plan);
    unsigned flag = 0;
    cudaError_t e = cudaMemcpy(&flag, P->d_counters + 6, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(P->d_counters + 6, 0, sizeof(unsigned));
    if (e != cudaSuccess) return gfb::set_cuda_error(e);
    *barrier_timeouts = (int)flag;
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_plan_destroy(gpufft_batch_plan plan)
{
    if (!plan) return GPUFFT_ERROR_INVALID_VALUE;
    gfb::free_plan(reinterpret_cast<gfb::BatchPlan*>(plan));
    return GPUFFT_SUCCESS;
}
