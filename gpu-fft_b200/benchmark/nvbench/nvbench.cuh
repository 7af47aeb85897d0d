// gpufft-b200 benchmark harness: the part of NVIDIA nvbench's benchmark API
// that GPU-FFT's benchmark programs use (reference benchmark/*.cu), written
// here so that those programs build without fetching nvbench.
//
//   NVBENCH_BENCH(fn).add_int64_axis("Name", {...}).set_timeout(s);
//   nvbench::state: get_int64, set_cuda_stream, add_global_memory_reads/writes,
//                   add_element_count, collect_* (recorded, not collected),
//                   skip, exec(lambda(nvbench::launch&))
//   nvbench::make_cuda_stream_view, nvbench::launch::get_stream
//
// Measurement follows nvbench's "cold" mode: before every sample the L2 is
// flushed (a memset of twice its size on the state's stream), then one call
// of the lambda is timed with CUDA events on that stream (GPU time) and with
// a host clock around record..synchronize (CPU time). Sampling stops once at
// least min_samples samples and min_time seconds of GPU time are in and the
// relative standard deviation of the GPU times is at most max_noise, or when
// the state's timeout (wall clock) has passed. One untimed call comes first.
//
// Output: a markdown table per benchmark in nvbench's column layout (axes,
// Samples, CPU Time, Noise, GPU Time, Noise, and GlobalMem BW / BWUtil when
// the state declared its memory traffic), and with --json FILE the same
// numbers as JSON. Options: -l/--list, -b/--benchmark NAME|INDEX,
// -a/--axis "Name=[v1,v2]" | "Name=[lo:hi]" | "Name=v", --timeout S,
// --min-samples N, --min-time S, --max-noise PERCENT, --no-l2-flush,
// --json FILE, --md FILE.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace nvbench
{
using int64_t = std::int64_t;

class cuda_stream
{
  public:
    explicit cuda_stream(cudaStream_t s = nullptr) : s_(s) {}
    cudaStream_t get_stream() const { return s_; }
    operator cudaStream_t() const { return s_; }

  private:
    cudaStream_t s_;
};

inline cuda_stream make_cuda_stream_view(cudaStream_t s) { return cuda_stream(s); }

class launch
{
  public:
    explicit launch(cudaStream_t s) : s_(s) {}
    cudaStream_t get_stream() const { return s_; }

  private:
    cudaStream_t s_;
};

struct criteria
{
    int min_samples = 10;
    double min_time = 0.5;   // seconds of GPU time
    double max_noise = 0.005; // relative standard deviation
    double timeout = 15.0;   // seconds of wall clock per state
    bool flush_l2 = true;
};

// What one state measured.
struct result
{
    std::vector<std::pair<std::string, int64_t>> axes;
    long samples = 0;
    double gpu_mean = 0, gpu_noise = 0, gpu_min = 0; // seconds, relative
    double cpu_mean = 0, cpu_noise = 0;
    double bytes = 0; // declared global-memory reads + writes per call
    double elements = 0;
    std::string skipped;
    std::vector<std::string> collect; // requested counter collections (not collected)
};

namespace detail
{
inline double mean(const std::vector<double>& v)
{
    double s = 0;
    for (double x : v) s += x;
    return v.empty() ? 0.0 : s / (double)v.size();
}
inline double rel_stdev(const std::vector<double>& v)
{
    if (v.size() < 2) return INFINITY;
    const double m = mean(v);
    double q = 0;
    for (double x : v) q += (x - m) * (x - m);
    return m > 0 ? std::sqrt(q / (double)(v.size() - 1)) / m : INFINITY;
}

// A device buffer of twice the L2 size, written once per sample.
class l2_flusher
{
  public:
    l2_flusher()
    {
        int dev = 0, l2 = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
        bytes_ = 2 * (size_t)(l2 > 0 ? l2 : (64 << 20));
        if (cudaMalloc(&buf_, bytes_) != cudaSuccess)
        {
            buf_ = nullptr;
            cudaGetLastError();
        }
    }
    ~l2_flusher()
    {
        if (buf_) cudaFree(buf_);
    }
    void flush(cudaStream_t s)
    {
        if (buf_) cudaMemsetAsync(buf_, ++tag_ & 0xff, bytes_, s);
    }

  private:
    void* buf_ = nullptr;
    size_t bytes_ = 0;
    int tag_ = 0;
};
} // namespace detail

class state
{
  public:
    state(std::vector<std::pair<std::string, int64_t>> axes, criteria c) : crit_(c) { res_.axes = std::move(axes); }

    int64_t get_int64(const std::string& name) const
    {
        for (const auto& a : res_.axes)
            if (a.first == name) return a.second;
        throw std::invalid_argument("nvbench: no int64 axis named '" + name + "'");
    }
    void set_cuda_stream(const cuda_stream& s) { stream_ = s.get_stream(); }
    cuda_stream get_cuda_stream() const { return cuda_stream(stream_); }

    template <typename T> void add_global_memory_reads(size_t count, const std::string& = std::string())
    {
        res_.bytes += (double)count * sizeof(T);
    }
    template <typename T> void add_global_memory_writes(size_t count, const std::string& = std::string())
    {
        res_.bytes += (double)count * sizeof(T);
    }
    void add_element_count(size_t count, const std::string& = std::string()) { res_.elements += (double)count; }

    void collect_l1_hit_rates() { res_.collect.push_back("l1_hit_rate"); }
    void collect_l2_hit_rates() { res_.collect.push_back("l2_hit_rate"); }
    void collect_loads_efficiency() { res_.collect.push_back("loads_efficiency"); }
    void collect_stores_efficiency() { res_.collect.push_back("stores_efficiency"); }
    void collect_dram_throughput() { res_.collect.push_back("dram_throughput"); }
    void collect_cupti_metrics() {}

    void skip(const std::string& reason) { res_.skipped = reason; }
    bool is_skipped() const { return !res_.skipped.empty(); }

    template <typename F> void exec(F&& fn)
    {
        if (is_skipped()) return;
        launch l(stream_);
        try
        {
            fn(l);
        }
        catch (const std::exception& e)
        {
            skip(std::string("first call threw: ") + e.what());
            return;
        }
        cudaError_t e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess)
        {
            skip(std::string("first call failed: ") + cudaGetErrorString(e));
            return;
        }
        detail::l2_flusher fl;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        std::vector<double> gpu, cpu;
        double gpu_total = 0;
        const auto t_start = std::chrono::steady_clock::now();
        for (;;)
        {
            if (crit_.flush_l2) fl.flush(stream_);
            cudaStreamSynchronize(stream_); // the CPU time starts with an idle stream
            const auto c0 = std::chrono::steady_clock::now();
            cudaEventRecord(e0, stream_);
            try
            {
                fn(l);
            }
            catch (const std::exception& ex)
            {
                skip(std::string("a timed call threw: ") + ex.what());
                cudaStreamSynchronize(stream_);
                break;
            }
            cudaEventRecord(e1, stream_);
            e = cudaEventSynchronize(e1);
            const auto c1 = std::chrono::steady_clock::now();
            if (e != cudaSuccess)
            {
                skip(std::string("a timed call failed: ") + cudaGetErrorString(e));
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            gpu.push_back(ms * 1e-3);
            cpu.push_back(std::chrono::duration<double>(c1 - c0).count());
            gpu_total += ms * 1e-3;
            const double wall = std::chrono::duration<double>(c1 - t_start).count();
            const bool done = (long)gpu.size() >= crit_.min_samples && gpu_total >= crit_.min_time &&
                              detail::rel_stdev(gpu) <= crit_.max_noise;
            if (done || wall >= crit_.timeout) break;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        res_.samples = (long)gpu.size();
        res_.gpu_mean = detail::mean(gpu);
        res_.gpu_noise = detail::rel_stdev(gpu);
        res_.gpu_min = gpu.empty() ? 0.0 : *std::min_element(gpu.begin(), gpu.end());
        res_.cpu_mean = detail::mean(cpu);
        res_.cpu_noise = detail::rel_stdev(cpu);
    }

    const result& get_result() const { return res_; }

  private:
    criteria crit_;
    cudaStream_t stream_ = nullptr;
    result res_;
};

class benchmark
{
  public:
    benchmark(std::string name, std::function<void(state&)> fn) : name_(std::move(name)), fn_(std::move(fn)) {}

    benchmark& set_name(std::string n)
    {
        name_ = std::move(n);
        return *this;
    }
    benchmark& add_int64_axis(std::string name, std::vector<int64_t> values)
    {
        axes_.emplace_back(std::move(name), std::move(values));
        return *this;
    }
    benchmark& add_int64_power_of_two_axis(std::string name, std::vector<int64_t> exponents)
    {
        for (auto& v : exponents) v = int64_t(1) << v;
        return add_int64_axis(std::move(name), std::move(exponents));
    }
    benchmark& set_timeout(double s)
    {
        crit_.timeout = s;
        return *this;
    }
    benchmark& set_min_samples(int n)
    {
        crit_.min_samples = n;
        return *this;
    }
    benchmark& set_min_time(double s)
    {
        crit_.min_time = s;
        return *this;
    }
    benchmark& set_max_noise(double percent)
    {
        crit_.max_noise = percent / 100.0;
        return *this;
    }

    const std::string& name() const { return name_; }
    std::vector<std::pair<std::string, std::vector<int64_t>>>& axes() { return axes_; }
    criteria& crit() { return crit_; }

    // Every combination of the axis values, the first axis varying slowest.
    std::vector<result> run(const criteria& c) const
    {
        std::vector<result> out;
        std::vector<size_t> at(axes_.size(), 0);
        for (const auto& a : axes_)
            if (a.second.empty()) return out;
        for (;;)
        {
            std::vector<std::pair<std::string, int64_t>> v;
            for (size_t i = 0; i < axes_.size(); i++) v.emplace_back(axes_[i].first, axes_[i].second[at[i]]);
            state st(v, c);
            try
            {
                fn_(st);
            }
            catch (const std::exception& e)
            {
                st.skip(std::string("threw: ") + e.what());
            }
            out.push_back(st.get_result());
            size_t k = axes_.size();
            while (k > 0)
            {
                if (++at[k - 1] < axes_[k - 1].second.size()) break;
                at[k - 1] = 0;
                k--;
            }
            if (k == 0) break;
        }
        return out;
    }

  private:
    std::string name_;
    std::function<void(state&)> fn_;
    std::vector<std::pair<std::string, std::vector<int64_t>>> axes_;
    criteria crit_;
};

inline std::vector<std::unique_ptr<benchmark>>& registry()
{
    static std::vector<std::unique_ptr<benchmark>> r;
    return r;
}

inline benchmark& add_benchmark(const char* name, void (*fn)(state&))
{
    registry().push_back(std::make_unique<benchmark>(name, fn));
    return *registry().back();
}

namespace detail
{
inline std::string fmt_time(double s)
{
    char b[64];
    if (s >= 1.0)
        std::snprintf(b, sizeof b, "%.3f s", s);
    else if (s >= 1e-3)
        std::snprintf(b, sizeof b, "%.3f ms", s * 1e3);
    else
        std::snprintf(b, sizeof b, "%.3f us", s * 1e6);
    return b;
}
inline std::string fmt_pct(double r)
{
    char b[32];
    if (!std::isfinite(r)) return "inf";
    std::snprintf(b, sizeof b, "%.2f%%", r * 100.0);
    return b;
}

// "Name=[a,b,c]", "Name=[lo:hi]" (inclusive) or "Name=v"
inline std::pair<std::string, std::vector<int64_t>> parse_axis(const std::string& s)
{
    const size_t eq = s.find('=');
    if (eq == std::string::npos) throw std::invalid_argument("axis option needs Name=values: " + s);
    std::string name = s.substr(0, eq), v = s.substr(eq + 1);
    while (!name.empty() && name.back() == ' ') name.pop_back();
    std::vector<int64_t> vals;
    if (!v.empty() && v.front() == '[' && v.back() == ']') v = v.substr(1, v.size() - 2);
    const size_t colon = v.find(':');
    if (colon != std::string::npos)
    {
        const int64_t lo = std::stoll(v.substr(0, colon)), hi = std::stoll(v.substr(colon + 1));
        for (int64_t x = lo; x <= hi; x++) vals.push_back(x);
    }
    else
    {
        size_t p = 0;
        while (p < v.size())
        {
            size_t q = v.find(',', p);
            if (q == std::string::npos) q = v.size();
            vals.push_back(std::stoll(v.substr(p, q - p)));
            p = q + 1;
        }
    }
    return {name, vals};
}

inline void json_str(std::FILE* f, const std::string& s)
{
    std::fputc('"', f);
    for (char c : s)
    {
        if (c == '"' || c == '\\') std::fputc('\\', f);
        std::fputc(c, f);
    }
    std::fputc('"', f);
}
} // namespace detail

// The program's entry point: run the selected benchmarks, print the tables.
inline int main(int argc, char** argv)
{
    criteria over;
    bool have_timeout = false, have_samples = false, have_time = false, have_noise = false, list = false;
    std::vector<std::string> pick;
    std::vector<std::pair<std::string, std::vector<int64_t>>> axis_over;
    std::string json_path, md_path;
    try
    {
        for (int i = 1; i < argc; i++)
        {
            const std::string a = argv[i];
            auto next = [&]() -> std::string {
                if (i + 1 >= argc) throw std::invalid_argument("missing value after " + a);
                return argv[++i];
            };
            if (a == "-l" || a == "--list")
                list = true;
            else if (a == "-b" || a == "--benchmark")
                pick.push_back(next());
            else if (a == "-a" || a == "--axis")
                axis_over.push_back(detail::parse_axis(next()));
            else if (a == "--timeout")
                over.timeout = std::stod(next()), have_timeout = true;
            else if (a == "--min-samples")
                over.min_samples = std::stoi(next()), have_samples = true;
            else if (a == "--min-time")
                over.min_time = std::stod(next()), have_time = true;
            else if (a == "--max-noise")
                over.max_noise = std::stod(next()) / 100.0, have_noise = true;
            else if (a == "--no-l2-flush")
                over.flush_l2 = false;
            else if (a == "--json")
                json_path = next();
            else if (a == "--md")
                md_path = next();
            else
                throw std::invalid_argument("unknown option " + a);
        }
    }
    catch (const std::exception& e)
    {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }

    auto& reg = registry();
    for (auto& o : axis_over)
        for (auto& b : reg)
            for (auto& ax : b->axes())
                if (ax.first == o.first) ax.second = o.second;
    if (list)
    {
        for (size_t i = 0; i < reg.size(); i++)
        {
            std::printf("%zu: %s\n", i, reg[i]->name().c_str());
            for (auto& ax : reg[i]->axes())
            {
                std::printf("    %s:", ax.first.c_str());
                for (auto v : ax.second) std::printf(" %lld", (long long)v);
                std::printf("\n");
            }
        }
        return 0;
    }

    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
    {
        std::fprintf(stderr, "nvbench: no CUDA device\n");
        return 1;
    }
    int mem_khz = 0, bus_bits = 0;
    cudaDeviceGetAttribute(&mem_khz, cudaDevAttrMemoryClockRate, dev);
    cudaDeviceGetAttribute(&bus_bits, cudaDevAttrGlobalMemoryBusWidth, dev);
    const double peak_bw = 2.0 * mem_khz * 1e3 * (bus_bits / 8.0); // bytes/s, DDR

    std::FILE* md = md_path.empty() ? stdout : std::fopen(md_path.c_str(), "w");
    if (!md)
    {
        std::fprintf(stderr, "nvbench: cannot write %s\n", md_path.c_str());
        return 1;
    }
    std::fprintf(md, "# Devices\n\n## [%d] `%s`\n* SM Version: %d\n* Number of SMs: %d\n* Global Memory: %zu MiB\n",
                 dev, prop.name, prop.major * 100 + prop.minor * 10, prop.multiProcessorCount,
                 (size_t)(prop.totalGlobalMem >> 20));
    std::fprintf(md, "* Global Memory Bus Peak: %.0f GB/sec (%d-bit DDR @%dMHz)\n\n# Benchmark Results\n",
                 peak_bw / 1e9, bus_bits, mem_khz / 1000);

    struct done_bench
    {
        std::string name;
        std::vector<result> rows;
    };
    std::vector<done_bench> all;
    for (size_t i = 0; i < reg.size(); i++)
    {
        benchmark& b = *reg[i];
        if (!pick.empty() && std::find(pick.begin(), pick.end(), b.name()) == pick.end() &&
            std::find(pick.begin(), pick.end(), std::to_string(i)) == pick.end())
            continue;
        criteria c = b.crit();
        if (have_timeout) c.timeout = over.timeout;
        if (have_samples) c.min_samples = over.min_samples;
        if (have_time) c.min_time = over.min_time;
        if (have_noise) c.max_noise = over.max_noise;
        c.flush_l2 = over.flush_l2;
        done_bench d{b.name(), b.run(c)};

        std::fprintf(md, "\n## %s\n\n### [%d] %s\n\n", d.name.c_str(), dev, prop.name);
        const bool bw = std::any_of(d.rows.begin(), d.rows.end(), [](const result& r) { return r.bytes > 0; });
        for (auto& ax : b.axes()) std::fprintf(md, "| %s ", ax.first.c_str());
        std::fprintf(md, "| Samples | CPU Time | Noise | GPU Time | Noise |%s\n", bw ? " GlobalMem BW | BWUtil |" : "");
        for (size_t k = 0; k < b.axes().size(); k++) std::fprintf(md, "|---");
        std::fprintf(md, "|---|---|---|---|---|%s\n", bw ? "---|---|" : "");
        for (const auto& r : d.rows)
        {
            for (const auto& a : r.axes) std::fprintf(md, "| %lld ", (long long)a.second);
            if (!r.skipped.empty())
            {
                std::fprintf(md, "| skipped: %s |\n", r.skipped.c_str());
                continue;
            }
            std::fprintf(md, "| %ldx | %s | %s | %s | %s |", r.samples, detail::fmt_time(r.cpu_mean).c_str(),
                         detail::fmt_pct(r.cpu_noise).c_str(), detail::fmt_time(r.gpu_mean).c_str(),
                         detail::fmt_pct(r.gpu_noise).c_str());
            if (bw)
            {
                const double gbs = r.gpu_mean > 0 ? r.bytes / r.gpu_mean : 0.0;
                std::fprintf(md, " %.3f GB/s | %.2f%% |", gbs / 1e9, peak_bw > 0 ? 100.0 * gbs / peak_bw : 0.0);
            }
            std::fprintf(md, "\n");
        }
        if (!d.rows.empty() && !d.rows[0].collect.empty())
            std::fprintf(md, "\nRequested counter collections (%zu) need CUPTI and are not collected here.\n",
                         d.rows[0].collect.size());
        std::fflush(md);
        all.push_back(std::move(d));
    }
    if (md != stdout) std::fclose(md);

    if (!json_path.empty())
    {
        std::FILE* f = std::fopen(json_path.c_str(), "w");
        if (!f)
        {
            std::fprintf(stderr, "nvbench: cannot write %s\n", json_path.c_str());
            return 1;
        }
        std::fprintf(f, "{\"device\": ");
        detail::json_str(f, prop.name);
        std::fprintf(f, ", \"global_memory_peak_gbs\": %.1f, \"l2_flush\": %s, \"benchmarks\": [", peak_bw / 1e9,
                     over.flush_l2 ? "true" : "false");
        for (size_t i = 0; i < all.size(); i++)
        {
            std::fprintf(f, "%s{\"name\": ", i ? ", " : "");
            detail::json_str(f, all[i].name);
            std::fprintf(f, ", \"states\": [");
            for (size_t j = 0; j < all[i].rows.size(); j++)
            {
                const result& r = all[i].rows[j];
                std::fprintf(f, "%s{\"axes\": {", j ? ", " : "");
                for (size_t k = 0; k < r.axes.size(); k++)
                {
                    std::fprintf(f, "%s", k ? ", " : "");
                    detail::json_str(f, r.axes[k].first);
                    std::fprintf(f, ": %lld", (long long)r.axes[k].second);
                }
                std::fprintf(f, "}");
                if (!r.skipped.empty())
                {
                    std::fprintf(f, ", \"skipped\": ");
                    detail::json_str(f, r.skipped);
                }
                else
                {
                    auto num = [](double x) { return std::isfinite(x) ? x : -1.0; };
                    std::fprintf(f,
                                 ", \"samples\": %ld, \"gpu_time_mean_s\": %.9g, \"gpu_time_min_s\": %.9g, "
                                 "\"gpu_noise\": %.6g, \"cpu_time_mean_s\": %.9g, \"cpu_noise\": %.6g, "
                                 "\"global_memory_bytes\": %.0f",
                                 r.samples, r.gpu_mean, r.gpu_min, num(r.gpu_noise), r.cpu_mean, num(r.cpu_noise),
                                 r.bytes);
                }
                std::fprintf(f, "}");
            }
            std::fprintf(f, "]}");
        }
        std::fprintf(f, "]}\n");
        std::fclose(f);
    }
    return 0;
}
} // namespace nvbench

#define NVBENCH_CONCAT_INNER(a, b) a##b
#define NVBENCH_CONCAT(a, b) NVBENCH_CONCAT_INNER(a, b)
#define NVBENCH_BENCH(fn)                                                                                             \
    static ::nvbench::benchmark& NVBENCH_CONCAT(nvbench_registered_, __LINE__) = ::nvbench::add_benchmark(#fn, fn)

// nvbench::main is linked as a library; here the entry point comes from one
// translation unit that defines NVBENCH_MAIN_HERE (nvbench_main.cu).
#if defined(NVBENCH_MAIN_HERE)
int main(int argc, char** argv) { return ::nvbench::main(argc, argv); }
#endif
