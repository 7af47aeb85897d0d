"""Benchmark: batched negacyclic polynomial products (FFNT) on B200.

Workload (default): N = 2^16 ring, batch 256 products per GPU, coefficients
uniform integers in [0, 2^24), seeded synthetic data (no dataset exists for this
path). A "step" is one batched product c = a * b mod (X^N + 1) over the whole
batch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--path f64|f32|dropin_f64] [--n-power 16] [--batch 256]

`value` is whole-job products/s with inputs resident in HBM; `e2e` is the same
metric through the public API with host buffers (pinned host -> device copy of
a and b, the product, device -> host copy of c, every step). Timing uses CUDA
events on the launching stream, warm-up first; the inputs (2 x 256 x 2^16
doubles = 256 MiB) exceed the 126 MB L2, so no flush is needed between steps.
Multi-GPU runs (torchrun) shard the batch per rank with no collective on the
data path (weak scaling) and report the max time over ranks.

At N = 1 the line also carries: `cpu_baseline` (the --impl reference arm run in
a fresh process, which also checks sampled outputs of every path against the
exact product and times the reference's GPU build), `ref_gpu` (the reference's
two GPU_FFNT calls against this library's drop-in and native products, at the
workload's batch and at batch 1) and `nvbench` (the benchmark program
gpu_ffnt_R_R_mult_benchmark built against this library and against the
reference's, on the reference benchmark's axes).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20261203 + 3  # seed of the N = 2^16, batch 256 product workload


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--path", choices=["split", "split64", "f64", "f32", "dropin_f64", "batch", "vjp", "cc"],
                   default="split",
                   help="split (exact, FP32 transforms) / split64 (exact, FP64 transforms) / f64 / f32 / dropin_f64: "
                        "N = 2^16 negacyclic products, batch 256, 24-bit coefficients; "
                        "batch: 4096 mixed ring sizes 2^10..2^17 (one persistent launch in a CUDA "
                        "graph); vjp: FP32 linear convolution N = 2^14, batch 512, forward + VJP; cc: C_C cyclic "
                        "products through GPU_FFT, FP32 and FP64, N = 2^10..2^16, ~1 GiB batches")
    p.add_argument("--no-compare", dest="compare", action="store_false",
                   help="time only --path (by default FP64 is timed beside it)")
    p.add_argument("--n-power", type=int, default=16)
    p.add_argument("--batch", type=int, default=256)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-ref-gpu", dest="ref_gpu", action="store_false",
                   help="skip timing the reference's own GPU build beside ours (N = 1 only)")
    p.add_argument("--check", default=None,
                   help="(--impl reference) .npz of sampled GPU outputs to check against the exact product; "
                        "written by the GPU arm for its cpu_baseline leg")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t_lo=None, t_hi=None):
        """Median SM clock and active throttle reasons of the samples taken in
        [t_lo, t_hi] (widened by 0.25 s each side when none falls inside)."""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines
        if t_lo is not None:
            inside = [x for x in lines if t_lo <= x[0] <= t_hi]
            if not inside:
                inside = [x for x in lines if t_lo - 0.25 <= x[0] <= t_hi + 0.25]
            lines = inside
        for _, ln in lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def reduce_max(value, dist, device):
    """Max of a per-rank float over all ranks (the whole-job step time)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_inputs(batch, n, rank):
    import torch
    g = torch.Generator().manual_seed(SEED + rank)
    a = torch.randint(0, 1 << 24, (batch, n), generator=g, dtype=torch.int64)
    b = torch.randint(0, 1 << 24, (batch, n), generator=g, dtype=torch.int64)
    return a, b


def cpu_baseline_reference(n, count, threads, distinct=32):
    """The reference's FFNT<double>::MULT on the host cores (oracle/_ref build, or
    the oracle's restatement when that build is absent): `count` products, one
    per host thread at a time, cycling over `distinct` seeded input pairs."""
    import numpy as np
    import oracle as O
    rng = np.random.default_rng(SEED)
    a = rng.integers(0, 1 << 24, (distinct, n)).astype(np.uint64)
    b = rng.integers(0, 1 << 24, (distinct, n)).astype(np.uint64)
    out = np.zeros((distinct, n), np.uint64)
    R = O.ref()
    if R is not None:
        secs = R.ref_bench_ffnt_mult_f64(n, count, distinct, threads, a.ravel(), b.ravel(), out.ravel())
        return count / secs, "reference", threads
    count = min(count, 64)  # the restatement runs on one thread
    t0 = time.perf_counter()
    for k in range(count):
        O.cpu_ffnt_mult(n, a[k % distinct], b[k % distinct], "f64")
    return count / (time.perf_counter() - t0), "port", 1


def cpu_sample_count(n, threads):
    # about 10 s of single-core work for the reference's FFNT<double>::MULT
    # (about 4.4 ms per product at N = 2^16), spread over the host threads
    per = 4.4e-3 * (n / 65536.0) * max(1.0, (n.bit_length() - 1) / 16.0)
    return max(threads, int(10.0 / per))


def cpu_reference_error(n, samples=256):
    """Largest |error| of the reference's FFNT<double>::MULT on the first product
    of the workload (24-bit coefficients), at `samples` sampled coefficients,
    against the exact product (int64 wrap-around semantics). The reference
    casts its rounded doubles to unsigned long long, so the difference is taken
    modulo 2^64 and read as signed."""
    import numpy as np
    import oracle as O
    R = O.ref()
    if R is None:
        return None
    a64, b64 = make_inputs(1, n, 0)
    a = a64[0].numpy().astype(np.uint64)
    b = b64[0].numpy().astype(np.uint64)
    out = np.zeros(n, np.uint64)
    R.ref_ffnt_mult_f64(n, a, b, out)
    rng = np.random.default_rng(2)
    idx = np.sort(rng.choice(n, samples, replace=False)).astype(np.int32)
    want = O.wrap64(O.negacyclic_coeffs(a64[0].numpy(), b64[0].numpy(), idx))
    diff = (out[idx].astype(np.int64) - want)  # wraps modulo 2^64
    return float(np.max(np.abs(diff.astype(np.float64))))


def cpu_baseline_subprocess(args, check_path=None):
    """The cpu_baseline leg: the --impl reference arm itself (same code, same
    sample, a fresh process without the GPU arm's threads), 3 timed steps after
    one warm-up; its value is the median step. The same process checks the GPU
    arm's sampled outputs (`check_path`) against the exact product and times the
    reference's GPU build. Returns (cpu_baseline, the reference arm's line)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--n-power", str(args.n_power),
           "--batch", str(args.batch), "--steps", "3", "--warmup", "1"]
    if check_path:
        cmd += ["--check", check_path]
    if not args.ref_gpu:
        cmd += ["--no-ref-gpu"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=env).stdout.strip().splitlines()
        ref = json.loads(out[-1])
    except (subprocess.SubprocessError, ValueError, IndexError) as exc:
        return {"unavailable": f"reference CPU arm failed: {exc}"}, {}
    cb = dict(ref["cpu_baseline"])
    cb["exact"] = ref.get("exact")
    cb["max_abs_error_on_sample"] = ref.get("max_abs_error_on_sample")
    cb["note"] = ("the reference's FP64 product is not exact at this size (results reach about 2^62, where an FP64 "
                  "ulp is 2^10); the GPU line's split product is")
    cb["how"] = "bench.py --impl reference --steps 3 --warmup 1 in a fresh process (median step)"
    return cb, ref


def check_samples(path):
    """Exactness of the GPU arm's sampled outputs: the first product of each
    path at 64 seeded coefficient indices against the exact negacyclic product
    (int64 wrap-around)."""
    import numpy as np
    import oracle as O
    d = np.load(path)
    idx = d["idx"].astype(np.int32)
    want = O.wrap64(O.negacyclic_coeffs(d["a0"], d["b0"], idx))
    res = {}
    for k in d.files:
        if not k.startswith("out_"):
            continue
        got = d[k]
        if got.dtype != np.int64:
            err = float(np.max(np.abs(got.astype(np.float64) - want.astype(np.float64))))
            exact = bool(np.array_equal(np.rint(got).astype(np.int64), want))
        else:
            err = float(np.max(np.abs((got - want).astype(np.float64))))
            exact = bool(np.array_equal(got, want))
        res[k[4:]] = {"exact": exact, "max_abs_error": err}
    return res


def run_reference(args, rank, world):
    if rank != 0:
        return
    n = 1 << args.n_power
    threads = os.cpu_count() or 1
    # each step: the same bounded sample as the cpu_baseline leg of the GPU arm
    cnt = cpu_sample_count(n, threads)
    vals = []
    kind, cores = "reference", threads
    for i in range(args.warmup + args.steps):
        v, kind, cores = cpu_baseline_reference(n, cnt, threads)
        if i >= args.warmup:
            vals.append(v)
    val = statistics.median(vals)
    err = cpu_reference_error(n)
    line = {"impl": "reference", "metric": f"negacyclic poly-mults/s at N=2^{args.n_power}", "value": val,
            "unit": "products/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cnt / val * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded uniform [0, 2^24))",
            "config": {"workload": f"FFNT negacyclic product N=2^{args.n_power}, batch {args.batch}, "
                                   "coefficients in [0, 2^24)", "ring_log2": args.n_power, "batch": args.batch,
                       "l2": "inputs > L2"},
            "exact": False if err is None or err > 0 else True, "max_abs_error_on_sample": err,
            "cpu_baseline": {"value": val, "unit": "products/s", "cores": cores, "kind": kind,
                             "sample": f"{cnt} products of N=2^{args.n_power} per step, FFNT<double>::MULT, "
                                       "one product per host thread at a time"},
            "e2e": {"value": val, "unit": "products/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.check:
        line["check"] = check_samples(args.check)
    if args.ref_gpu:
        line["ref_gpu"] = reference_gpu_cases(args)
        if "unavailable" not in line["ref_gpu"]:
            line["nvbench"] = run_nvbench(os.path.join(ROOT, "oracle", "_ref", "bench", NVBENCH_PROGRAM))
    print(json.dumps(line), flush=True)


def events_ms(fn, args, torch, stream):
    """Mean ms of fn() over K calls, CUDA events on `stream`, after W (>= 3) warm-ups."""
    for _ in range(max(3, args.warmup)):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / args.steps


def ffnt_product_calls(fn, bufs, tables, n_power, bt, status):
    """The reference API's FFNT product as its benchmark bench_gpu_ffnt_R_R_mult.cu
    forms it: GPU_FFNT forward of 2*bt rows, then GPU_FFNT inverse with the
    product (mod_inverse 2/N) of bt rows. `fn` is a GPU_FFNT C entry point
    (inout, temp, twist, roots, n_power, fft_type, mod_inverse re/im, batch, mult,
    stream); the call statuses are appended to `status`."""
    inout, temp = bufs
    roots, inv_roots, twist, untwist = tables
    h = (1 << n_power) // 2

    def run():
        st = fn(inout.data_ptr(), temp.data_ptr(), twist.data_ptr(), roots.data_ptr(), n_power, 0, 1.0, 0.0,
                2 * bt, 0, None)
        st |= fn(inout.data_ptr(), temp.data_ptr(), untwist.data_ptr(), inv_roots.data_ptr(), n_power, 1, 1.0 / h,
                 0.0, bt, 1, None)
        status.append(st)
    return run


REF_GPU_BATCHES = (None, 1)  # the workload's batch, and batch 1


def ours_gpu_cases(gf, a64, b64, n_power, batch, args, dev, torch):
    """This library's side of the comparison with the reference's GPU build on
    the workload's inputs: the drop-in GPU_FFNT (the reference benchmark's two
    calls on FFNT<double> tables from this library's host generator, bitwise
    equal to the reference's), and the native FP64 and exact split products, at
    the workload's batch and at batch 1. The --impl reference arm times the
    reference's build the same way; the GPU arm divides the two."""
    import numpy as np
    n = 1 << n_power
    h = n // 2
    tables = [torch.from_numpy(np.ascontiguousarray(t)).to(dev) for t in gf.host_ffnt_tables(n, "f64")]
    L = gf.lib()
    stream = torch.cuda.current_stream()
    cases = []
    for bt in (batch if b is None else b for b in REF_GPU_BATCHES):
        inout = torch.cat([a64[:bt].reshape(-1), b64[:bt].reshape(-1)]).double().to(dev)
        temp = torch.empty(2 * bt * h, dtype=torch.complex128, device=dev)  # spectra of 2 bt rows
        status = []
        ms_drop = events_ms(ffnt_product_calls(L.gpufft_ffnt_f64, (inout, temp), tables, n_power, bt, status),
                            args, torch, stream)
        ad, bd = a64[:bt].double().to(dev), b64[:bt].double().to(dev)
        cd = torch.empty_like(ad)
        tf = gf.ffnt_tables(n_power, "f64", dev)
        ws = torch.empty(max(1, gf.negacyclic_mul_workspace_bytes(n_power, bt, 64)), dtype=torch.uint8, device=dev)
        ms_f64 = events_ms(lambda: gf.negacyclic_mul(ad, bd, out=cd, tables=tf, workspace=ws), args, torch, stream)
        ai, bi = a64[:bt].to(torch.int32).to(dev), b64[:bt].to(torch.int32).to(dev)
        ci = torch.empty((bt, n), dtype=torch.int64, device=dev)
        w, k = gf.split_plan(n_power, 24, True)
        t32 = gf.ffnt_tables(n_power, "f32", dev)
        wss = torch.empty(max(1, int(L.gpufft_negacyclic_mul_split_workspace_bytes(n_power, bt, k))),
                          dtype=torch.uint8, device=dev)
        ms_split = events_ms(lambda: gf.negacyclic_mul_split(ai, bi, out=ci, input_bits=24, non_negative=True,
                                                             limbs=(w, k), tables=t32, workspace=wss),
                             args, torch, stream)
        if any(status):
            return {"unavailable": f"a GPU_FFNT call failed (status {max(status)})"}
        cases.append({"batch": bt, "ring_log2": n_power, "ours_dropin_ms": ms_drop, "ours_f64_ms": ms_f64,
                      "ours_split_ms": ms_split})
        del inout, temp, ad, bd, cd, ws, ai, bi, ci, wss
        torch.cuda.empty_cache()
    return {"cases": cases}


def reference_gpu_cases(args):
    """The reference's own GPU path on the workload's inputs: its src/lib/fft.cu
    built unmodified for sm_100a (oracle/_ref), called through its C++ API
    GPU_FFNT as its benchmark bench_gpu_ffnt_R_R_mult.cu does (forward of
    2*batch, inverse with the product), on the reference's FFNT<double>
    tables, at the workload's batch and at batch 1. CUDA events around K steps
    after W warm-ups."""
    try:
        import torch
    except ImportError:
        return {"unavailable": "torch is not importable"}
    if not torch.cuda.is_available():
        return {"unavailable": "no GPU"}
    import numpy as np
    import oracle as O
    R = O.ref_gpu()
    if R is None:
        return {"unavailable": "the reference's GPU build (oracle/_ref/libgpufft_ref_gpu.so) is absent"}
    dev = torch.device("cuda", 0)
    n_power, batch = args.n_power, args.batch
    n = 1 << n_power
    h = n // 2
    a64, b64 = make_inputs(batch, n, 0)
    tables = [torch.from_numpy(np.ascontiguousarray(t)).to(dev) for t in O.ffnt_tables(n, "f64")]
    stream = torch.cuda.current_stream()
    cases = []
    for bt in (batch if b is None else b for b in REF_GPU_BATCHES):
        inout = torch.cat([a64[:bt].reshape(-1), b64[:bt].reshape(-1)]).double().to(dev)
        temp = torch.empty(2 * bt * h, dtype=torch.complex128, device=dev)  # spectra of 2 bt rows
        status = []
        ms = events_ms(ffnt_product_calls(R.ref_gpu_ffnt_f64, (inout, temp), tables, n_power, bt, status),
                       args, torch, stream)
        if any(status):
            return {"unavailable": f"a reference GPU_FFNT call failed (status {max(status)})"}
        cases.append({"batch": bt, "ring_log2": n_power, "ref_gpu_ms": ms, "ref_gpu_value": bt / (ms * 1e-3)})
        del inout, temp
    return {"cases": cases, "unit": "products/s",
            "timed": "CUDA events around K steps (each step: the reference benchmark's two GPU_FFNT calls)"}


def merge_gpu_cases(ours, ref):
    """Per batch: both sides' ms and the reference's time over ours."""
    if "cases" not in ours:
        return ours
    if not ref or "cases" not in ref:
        return {"ours": ours, "reference": ref or {"unavailable": "the cpu_baseline leg did not run"}}
    out = {"timed": "CUDA events around K steps on each side (the reference in the --impl reference arm's process)",
           "tables": "FFNT<double> tables in the reference's format on the device", "unit": "products/s",
           "cases": []}
    for o, r in zip(ours["cases"], ref["cases"]):
        bt = o["batch"]
        c = {"batch": bt, "ring_log2": o["ring_log2"], "ref_gpu_ms": r["ref_gpu_ms"],
             "ref_gpu_value": bt / (r["ref_gpu_ms"] * 1e-3)}
        for k in ("dropin", "f64", "split"):
            c[f"ours_{k}_ms"] = o[f"ours_{k}_ms"]
            c[f"ours_{k}_value"] = bt / (o[f"ours_{k}_ms"] * 1e-3)
            c[f"{k}_vs_ref"] = r["ref_gpu_ms"] / o[f"ours_{k}_ms"]
        out["cases"].append(c)
    out["ref_gpu_value"] = out["cases"][0]["ref_gpu_value"]
    return out


NVBENCH_PROGRAM = "gpu_ffnt_R_R_mult_benchmark"  # GPU_FFNT product, Ring Size LogN 12..23, Batch Count 1


def run_nvbench(exe, timeout_s=180):
    """One benchmark program on the nvbench-compatible harness (its own axes and
    stopping rule: cold L2, CUDA events per sample, 1 s per state); returns the
    harness's JSON."""
    import tempfile
    if not os.path.exists(exe):
        return {"unavailable": f"{os.path.relpath(exe, ROOT)} is not built"}
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "states.json")
        try:
            subprocess.run([exe, "--json", out, "--md", os.devnull], check=True, timeout=timeout_s,
                           capture_output=True)
            with open(out) as f:
                return json.load(f)
        except (subprocess.SubprocessError, OSError, ValueError) as exc:
            return {"unavailable": f"{os.path.basename(exe)} failed: {exc}"}


def merge_nvbench(ours, ref):
    """Per state of the program: both libraries' mean GPU time and the
    reference's over ours."""
    if "benchmarks" not in ours:
        return {"ours": ours, "reference": ref}
    if not ref or "benchmarks" not in ref:
        return {"ours": ours, "reference": ref or {"unavailable": "the cpu_baseline leg did not run"}}
    out = {"program": f"gpu-fft_b200/benchmark/bin/{NVBENCH_PROGRAM} (ours) and oracle/_ref/bench/{NVBENCH_PROGRAM} "
                      "(the same source built on the reference's library)",
           "timed": "cold L2 per sample, CUDA events, mean GPU time per state", "cases": []}
    for bo, br in zip(ours["benchmarks"], ref["benchmarks"]):
        for so, sr in zip(bo["states"], br["states"]):
            c = {"benchmark": bo["name"], **{k.lower().replace(" ", "_"): v for k, v in so["axes"].items()}}
            if "gpu_time_mean_s" in so and "gpu_time_mean_s" in sr:
                c.update(ours_us=so["gpu_time_mean_s"] * 1e6, ref_us=sr["gpu_time_mean_s"] * 1e6,
                         ref_over_ours=sr["gpu_time_mean_s"] / so["gpu_time_mean_s"])
            else:
                c.update(skipped=so.get("skipped") or sr.get("skipped"))
            out["cases"].append(c)
    return out


def make_path(gf, name, n_power, batch, dev, torch):
    """(step(a, b, c), algorithmic bytes per product, input/output element types,
    kernel launches per step) for one product path."""
    n = 1 << n_power
    m = n_power - 1
    if name in ("f64", "f32"):
        f64 = name == "f64"
        tables = gf.ffnt_tables(n_power, "f64" if f64 else "f32", dev)
        ws_bytes = gf.negacyclic_mul_workspace_bytes(n_power, batch, 64 if f64 else 32)
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
        esz = 8 if f64 else 4
        per = 2 * (1 << m) * (16 if f64 else 8)
        waves = 1 if m <= 12 else -(-batch // max(1, ws_bytes // per))

        def step(x, y, out):
            gf.negacyclic_mul(x, y, out=out, tables=tables, workspace=ws)
        hws = torch.empty(gf.lib().gpufft_negacyclic_mul_host_workspace_bytes(n_power, batch, 0, 64 if f64 else 32),
                          dtype=torch.uint8, device=dev)

        def host_step(x, y, out):
            gf.negacyclic_mul_host(x, y, out=out, tables=tables, workspace=hws)
        dt = torch.float64 if f64 else torch.float32
        return step, host_step, 3 * n * esz, dt, dt, (1 if m <= 12 else 3 * waves)
    if name == "split64":
        # the exact product with FP64 transforms (two 12-bit limbs at N = 2^16)
        w, k = gf.split_plan(n_power, 24, True, "f64")
        tables = gf.ffnt_tables(n_power, "f64", dev)
        need = int(gf.lib().gpufft_negacyclic_mul_split_f64_workspace_bytes(n_power, batch, k))
        ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)

        def step(x, y, out):
            gf.negacyclic_mul_split(x, y, out=out, input_bits=24, non_negative=True, limbs=(w, k), tables=tables,
                                    workspace=ws, precision="f64")

        def host_step(x, y, out):
            # no host-buffer variant of the FP64 split: copy in, product, copy out
            xd, yd = x.to(dev, non_blocking=True), y.to(dev, non_blocking=True)
            od = torch.empty(out.shape, dtype=out.dtype, device=dev)
            step(xd, yd, od)
            out.copy_(od, non_blocking=True)
        return step, host_step, 16 * n, torch.int32, torch.int64, 5
    if name == "split":
        w, k = gf.split_plan(n_power, 24, True)
        tables = gf.ffnt_tables(n_power, "f32", dev)
        need = int(gf.lib().gpufft_negacyclic_mul_split_workspace_bytes(n_power, batch, k))
        ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)
        per = (4 * k - 1) * (1 << m) * 8
        waves = -(-batch // max(1, need // per))

        def step(x, y, out):
            gf.negacyclic_mul_split(x, y, out=out, input_bits=24, non_negative=True, limbs=(w, k), tables=tables,
                                    workspace=ws)
        hws = torch.empty(gf.lib().gpufft_negacyclic_mul_split_f32_host_workspace_bytes(n_power, batch, 0, k),
                          dtype=torch.uint8, device=dev)

        def host_step(x, y, out):
            gf.negacyclic_mul_split_host(x, y, out=out, input_bits=24, non_negative=True, limbs=(w, k), tables=tables,
                                         workspace=hws)
        return step, host_step, 16 * n, torch.int32, torch.int64, (5 if m > 12 else 1) * waves
    # drop-in: the reference API's two GPU_FFNT calls (forward of 2*batch, inverse with product)
    import numpy as np
    roots, inv_roots, twist, untwist = [torch.from_numpy(np.ascontiguousarray(t)).to(dev)
                                        for t in gf.host_ffnt_tables(n, "f64")]
    inout = torch.empty(2 * batch * n, dtype=torch.float64, device=dev)
    temp = torch.empty(batch * n, dtype=torch.complex128, device=dev)
    cf = gf.fft_configuration(n_power=n_power, fft_type=gf.FORWARD)
    ci = gf.fft_configuration(n_power=n_power, fft_type=gf.INVERSE, mod_inverse=1.0 / (n // 2))

    def step(x, y, out):
        inout[: batch * n].copy_(x.view(-1))
        inout[batch * n:].copy_(y.view(-1))
        gf.GPU_FFNT(inout, temp, twist, roots, cf, 2 * batch, False)
        gf.GPU_FFNT(inout, temp, untwist, inv_roots, ci, batch, True)
        out.view(-1).copy_(inout[: batch * n])

    def host_step(x, y, out):
        # what a caller of the reference API does with host data: copy in, two
        # GPU_FFNT calls, copy out
        inout[: batch * n].copy_(x.view(-1), non_blocking=True)
        inout[batch * n:].copy_(y.view(-1), non_blocking=True)
        gf.GPU_FFNT(inout, temp, twist, roots, cf, 2 * batch, False)
        gf.GPU_FFNT(inout, temp, untwist, inv_roots, ci, batch, True)
        out.view(-1).copy_(inout[: batch * n], non_blocking=True)
    return step, host_step, 3 * n * 8, torch.float64, torch.float64, (4 if m > 12 else 2)


def time_path(step, host_step, a, b, c, hosts, args, stream, torch, barrier, max_over_ranks):
    """Device-resident and end-to-end timing of one path: returns (ms, ms_e2e, t0, t1).
    The end-to-end step is the public host-buffer call: pinned host inputs in,
    pinned host result out, every transfer inside the timed region."""
    a_host, b_host, c_host = hosts
    for _ in range(args.warmup):
        step(a, b, c)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    e0.record(stream)
    for _ in range(args.steps):
        step(a, b, c)
    e1.record(stream)
    barrier()
    t1 = time.time()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    for _ in range(max(1, args.warmup // 2)):
        host_step(a_host, b_host, c_host)
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        host_step(a_host, b_host, c_host)
    e3.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3) / args.steps)
    return ms, ms_e2e, t0, t1


# DRAM traffic of the dominant kernels as a fraction of the bytes the library's
# tracing tags them with (their own inputs read once and outputs written once),
# from one ncu capture each of a smaller wave of the same kernel
# (dram__bytes_read.sum + dram__bytes_write.sum; ncu flushes caches before each
# replay, so this is the cold-cache figure). Both scale with the products per
# launch, so traffic per launch = ratio x the kernel's tagged bytes per launch.
NCU_TRAFFIC = {
    # 64 products (1024 tiles): 168.8 MB read + 99.8 MB written of 318.8 MB tagged
    "split_tile<k5>": (268.5 / 318.8, "ncu capture of a 64-product launch"),
    # wave of 74 products (592 tiles): 78.1 MB read + 2.7 MB written of 116.4 MB tagged
    "fused_r8_kernel<f64,L12,middle>": (80.9 / 116.4, "ncu capture of a 74-product wave"),
    # wave of 46 products (3680 CTAs): 120.8 MB read + 63.5 MB written of 241.2 MB tagged
    "pass_kernel<f32,fwd,L12,contiguous>": (184.3 / 241.2, "ncu capture of a 46-product wave"),
}


def traced_kernels(gf, step, a, b, c, args, stream, torch, barrier, max_over_ranks):
    """Re-run the K timed steps with the library's per-kernel event tracing on:
    (per-kernel rows longest first, ms per step of the traced run)."""
    barrier()
    gf.trace_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step(a, b, c)
    e1.record(stream)
    barrier()
    gf.trace_enable(False)
    rows = gf.trace_collect()
    return rows, max_over_ranks(e0.elapsed_time(e1) / args.steps)


def kernel_roofline(rows, peak, peak_kind, ms_traced, steps, alg_per_product=None, products_per_step=None):
    """Roofline of the dominant kernel (largest summed device time).

    `achieved` / `frac` count the path's algorithmic bytes per product (the API
    inputs read once and outputs written once: 16N for the split product, 24N
    for the FP64 product) times the products one launch of that kernel covers,
    over its mean CUDA-event launch duration. `kernel_bytes_gbs` /
    `kernel_bytes_frac` count instead the bytes the kernel itself must move
    (its own inputs and outputs, intermediate spectra included)."""
    dom = rows[0]
    per_launch_ms = dom["ms"] / dom["launches"]
    per_launch_bytes = dom["alg_bytes"] / dom["launches"]
    own = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9
    launches_per_step = dom["launches"] / steps
    total = sum(r["ms"] for r in rows)
    traffic = NCU_TRAFFIC.get(dom["kernel"])
    out = {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
           "traffic": traffic[0] * per_launch_bytes if traffic else None,
           "traffic_source": (traffic[1] + ", scaled by products per launch") if traffic else None,
           "kernel": dom["kernel"], "launches_per_step": launches_per_step,
           "mean_launch_us": per_launch_ms * 1e3, "kernel_bytes_per_launch": per_launch_bytes,
           "kernel_bytes_gbs": own, "kernel_bytes_frac": own / peak,
           "share_of_step": dom["ms"] / total if total else None,
           "timed": "CUDA events around each launch (library tracing) over a repeat of the timed steps",
           "traced_ms_per_step": ms_traced,
           "kernels": [{"kernel": r["kernel"], "launches_per_step": r["launches"] / steps,
                        "ms_per_step": r["ms"] / steps,
                        "gbs": (r["alg_bytes"] / (r["ms"] * 1e-3) / 1e9) if r["ms"] else None} for r in rows]}
    if alg_per_product is not None and products_per_step:
        per_launch_products = products_per_step / launches_per_step
        alg = alg_per_product * per_launch_products
        achieved = alg / (per_launch_ms * 1e-3) / 1e9
        out.update({"achieved": achieved, "frac": achieved / peak, "alg_bytes_per_launch": alg,
                    "alg_bytes_per_product": alg_per_product, "products_per_launch": per_launch_products})
    else:
        out.update({"achieved": own, "frac": own / peak, "alg_bytes_per_launch": per_launch_bytes})
    return out


def run_batch(args, gf, dev, torch, world, rank, barrier, max_over_ranks, clk_cls, peak, peak_kind):
    """Mixed sizes: 4096 negacyclic products, ring sizes log-uniform over 2^10..2^17,
    coefficients in [-2^15, 2^15), FP64, one persistent launch replayed from a
    CUDA graph; per-size sequential launches timed beside it."""
    import numpy as np
    rng = np.random.default_rng(SEED + 1 + rank)
    n_powers = [int(x) for x in rng.integers(10, 18, 4096)]
    plan = gf.BatchPlan(n_powers, torch.float64)
    g = torch.Generator().manual_seed(SEED + 1 + rank)
    a_host = torch.randint(-(1 << 15), 1 << 15, (plan.total,), generator=g).double().pin_memory()
    b_host = torch.randint(-(1 << 15), 1 << 15, (plan.total,), generator=g).double().pin_memory()
    c_host = torch.empty_like(a_host).pin_memory()
    a, b = a_host.to(dev), b_host.to(dev)
    c = torch.empty_like(a)
    plan.autotune(a, b, c, os.path.join(ROOT, "gpu-fft_b200", "lib", "batch_autotune.jsonl"))
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    plan.capture(a, b, c, s)
    # per-size sequential reference path (same data, one call per ring size)
    sizes = sorted(set(n_powers))
    offs = plan.offsets
    groups = []
    for np_ in sizes:
        idx = [i for i, n in enumerate(n_powers) if n == np_]
        o0 = int(min(offs[i] for i in idx))
        groups.append((np_, len(idx), o0))
    tabs = {np_: gf.ffnt_tables(np_, "f64", dev) for np_ in sizes}
    wss = {np_: torch.empty(max(1, gf.negacyclic_mul_workspace_bytes(np_, cnt, 64)), dtype=torch.uint8, device=dev)
           for np_, cnt, _ in groups}

    def seq_step(out):
        for np_, cnt, o0 in groups:
            n = 1 << np_
            gf.negacyclic_mul(a[o0:o0 + cnt * n].view(cnt, n), b[o0:o0 + cnt * n].view(cnt, n),
                              out=out[o0:o0 + cnt * n].view(cnt, n), tables=tabs[np_], workspace=wss[np_],
                              stream=s)
    with torch.cuda.stream(s):
        with clk_cls(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
            time.sleep(0.5)
            for _ in range(args.warmup):
                plan.replay(s)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.time()
            e0.record(s)
            for _ in range(args.steps):
                plan.replay(s)
            e1.record(s)
            barrier()
            t1 = time.time()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        c_seq = torch.empty_like(a)
        for _ in range(args.warmup):
            seq_step(c_seq)
        barrier()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(s)
        for _ in range(args.steps):
            seq_step(c_seq)
        e3.record(s)
        barrier()
        ms_seq = max_over_ranks(e2.elapsed_time(e3) / args.steps)
        identical = bool(torch.equal(c, c_seq))
        # end to end: host operands in, host products out, every step
        for _ in range(max(1, args.warmup // 2)):
            a.copy_(a_host, non_blocking=True)
            b.copy_(b_host, non_blocking=True)
            plan.replay(s)
            c_host.copy_(c, non_blocking=True)
        barrier()
        e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e4.record(s)
        for _ in range(args.steps):
            a.copy_(a_host, non_blocking=True)
            b.copy_(b_host, non_blocking=True)
            plan.replay(s)
            c_host.copy_(c, non_blocking=True)
        e5.record(s)
        barrier()
        ms_e2e = max_over_ranks(e4.elapsed_time(e5) / args.steps)
        # the persistent kernel timed per launch (direct launches: graph replays are not traced)
        rows, ms_traced = traced_kernels(gf, lambda x, y, z: plan.execute(x, y, z, stream=s), a, b, c, args, s,
                                         torch, barrier, max_over_ranks)
        split_line = run_batch_split(args, gf, dev, torch, n_powers, a, b, s, barrier, max_over_ranks, world)
    alg = 3 * plan.total * 8
    achieved = alg / (ms * 1e-3) / 1e9
    info = plan.info()
    line = {
        "metric": "negacyclic poly-mults/s, 4096 mixed ring sizes 2^10..2^17", "value": world * 4096 / (ms * 1e-3),
        "unit": "products/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, log-uniform ring sizes, coefficients uniform in [-2^15, 2^15))",
        "config": {"workload": "4096 negacyclic products, ring sizes log-uniform 2^10..2^17, FP64, one persistent "
                               "cooperative launch replayed from a CUDA graph", "requests": 4096,
                   "coefficients": plan.total, "launch_shape": info, "l2": "inputs larger than L2 (no flush)"},
        "roofline": kernel_roofline(rows, peak, peak_kind, ms_traced, args.steps, alg / 4096, 4096),
        "chain": {"achieved_gbs": achieved, "frac": achieved / peak, "algorithmic_bytes_per_step": alg,
                  "timed": "graph replay of the persistent launch, CUDA events"},
        "e2e": {"value": world * 4096 / (ms_e2e * 1e-3), "unit": "products/s", "h2d_bytes_per_step": 2 * alg // 3,
                "d2h_bytes_per_step": alg // 3},
        "per_size_sequential": {"value": world * 4096 / (ms_seq * 1e-3), "unit": "products/s", "ms_per_step": ms_seq,
                                "identical_outputs": identical},
        "split": split_line,
        "gpu_launches": sum(r["launches"] for r in rows), "clocks": clk.summary(t0, t1),
    }
    plan.close()
    return line


def run_batch_split(args, gf, dev, torch, n_powers, a64, b64, s, barrier, max_over_ranks, world):
    """The same 4096 mixed-size requests, exact: FP32 split products per size
    class replayed from one CUDA graph, and per-size split calls beside it."""
    plan = gf.SplitBatchPlan(n_powers, input_bits=16, non_negative=False)
    a, b = a64.to(torch.int32), b64.to(torch.int32)
    c = torch.empty(plan.total, dtype=torch.int64, device=dev)
    err = torch.zeros(1, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    plan.capture(a, b, c, err, s)
    groups = []
    for np_ in sorted(set(n_powers)):
        idx = [i for i, n in enumerate(n_powers) if n == np_]
        groups.append((np_, len(idx), int(min(plan.offsets[i] for i in idx))))
    tabs = {np_: gf.ffnt_tables(np_, "f32", dev) for np_, _, _ in groups}
    wss = {}
    for np_, cnt, _ in groups:
        w, k = gf.split_plan(np_, 16, False)
        wss[np_] = (torch.empty(max(1, int(gf.lib().gpufft_negacyclic_mul_split_workspace_bytes(np_, cnt, k))),
                                dtype=torch.uint8, device=dev), (w, k))
    c_seq = torch.empty_like(c)

    def seq_step():
        for np_, cnt, o0 in groups:
            n = 1 << np_
            ws, limbs = wss[np_]
            gf.negacyclic_mul_split(a[o0:o0 + cnt * n].view(cnt, n), b[o0:o0 + cnt * n].view(cnt, n),
                                    out=c_seq[o0:o0 + cnt * n].view(cnt, n), input_bits=16, non_negative=False,
                                    limbs=limbs, tables=tabs[np_], workspace=ws, stream=s)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(args.steps):
            fn()
        e1.record(s)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / args.steps)
    ms = timed(lambda: plan.replay(s))
    ms_seq = timed(seq_step)
    line = {"value": world * 4096 / (ms * 1e-3), "unit": "products/s", "ms_per_step": ms, "dtype": "f32 split, exact",
            "timed": "graph replay of the per-class split chains",
            "max_pre_rounding_error": float(err.item()), "limbs": sorted(set(plan.limbs)),
            "per_size_sequential": {"value": world * 4096 / (ms_seq * 1e-3), "ms_per_step": ms_seq,
                                    "identical_outputs": bool(torch.equal(c, c_seq))}}
    plan.close()
    return line


def run_vjp(args, gf, dev, torch, world, rank, barrier, max_over_ranks, clk_cls, peak, peak_kind):
    """Convolution training step: FP32 linear convolution N = 2^14 (zero-padded to 2^15), batch
    512; a step is the forward product plus the VJP for both operands."""
    n, batch = 1 << 14, 512
    g = torch.Generator().manual_seed(SEED + 2 + rank)
    a_host = torch.randn((batch, n), generator=g).pin_memory()
    b_host = torch.randn((batch, n), generator=g).pin_memory()
    g_host = torch.randn((batch, 2 * n), generator=g).pin_memory()
    outs_host = [torch.empty((batch, n)).pin_memory(), torch.empty((batch, n)).pin_memory(),
                 torch.empty((batch, 2 * n)).pin_memory()]
    a, b, gr = a_host.to(dev), b_host.to(dev), g_host.to(dev)
    tables = gf.ffnt_tables(15, "f32", dev)
    ws_f = torch.empty(max(1, int(gf.lib().gpufft_linear_mul_workspace_bytes(14, batch, 32))), dtype=torch.uint8,
                       device=dev)
    ws_b = torch.empty(max(1, int(gf.lib().gpufft_linear_mul_vjp_workspace_bytes(14, batch))), dtype=torch.uint8,
                       device=dev)
    c = torch.empty((batch, 2 * n), device=dev)
    ga, gb = torch.empty_like(a), torch.empty_like(b)
    stream = torch.cuda.current_stream()

    def step():
        gf.linear_mul(a, b, out=c, tables=tables, workspace=ws_f)
        gf.linear_mul_vjp(gr, a, b, grad_a=ga, grad_b=gb, tables=tables, workspace=ws_b)
    with clk_cls(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        time.sleep(0.5)
        for _ in range(args.warmup):
            step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.time()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        barrier()
        t1 = time.time()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    for _ in range(max(1, args.warmup // 2)):
        step()
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        a.copy_(a_host, non_blocking=True)
        b.copy_(b_host, non_blocking=True)
        gr.copy_(g_host, non_blocking=True)
        step()
        outs_host[0].copy_(ga, non_blocking=True)
        outs_host[1].copy_(gb, non_blocking=True)
        outs_host[2].copy_(c, non_blocking=True)
    e3.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3) / args.steps)
    rows, ms_traced = traced_kernels(gf, lambda x, y, z: step(), a, b, c, args, stream, torch, barrier,
                                     max_over_ranks)
    # forward: a, b in (2N*4 bytes), c out (2N*4); backward: g (2N*4), a, b in, grads out (2N*4)
    alg = batch * (4 * n * 4 + 6 * n * 4)
    achieved = alg / (ms * 1e-3) / 1e9
    return {
        "metric": "forward+backward linear-convolution products/s (N=2^14, FP32)",
        "value": world * batch / (ms * 1e-3), "unit": "products/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded i.i.d. N(0,1))",
        "config": {"workload": "real FP32 linear convolution N=2^14 zero-padded to 2^15, batch 512, forward + VJP",
                   "batch_per_gpu": batch, "l2": "inputs larger than L2 (no flush)"},
        "roofline": kernel_roofline(rows, peak, peak_kind, ms_traced, args.steps, alg / batch, batch),
        "chain": {"achieved_gbs": achieved, "frac": achieved / peak, "algorithmic_bytes_per_step": alg,
                  "timed": "forward product + VJP per step, CUDA events"},
        "e2e": {"value": world * batch / (ms_e2e * 1e-3), "unit": "products/s",
                "h2d_bytes_per_step": batch * 4 * n * 4, "d2h_bytes_per_step": batch * 4 * n * 4},
        "gpu_launches": sum(r["launches"] for r in rows), "clocks": clk.summary(t0, t1),
    }


def run_cc(args, gf, dev, torch, world, rank, barrier, max_over_ranks, clk_cls, peak, peak_kind):
    """C_C cyclic products through the reference API: re/im i.i.d. N(0,1), N =
    2^10, 2^12, 2^14, 2^16, batch sized to ~1 GiB of input, FP32 and FP64; a step is
    GPU_FFT forward of both operands and GPU_FFT inverse with the product. Each
    case reports products/s, HBM GB/s of its algorithmic bytes (3 N complex per
    product) and the relative L2 error of sampled products against an FP64
    cyclic convolution."""
    import numpy as np
    cases = []
    stream = torch.cuda.current_stream()
    with clk_cls(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        time.sleep(0.3)
        t_first = None
        for tdt, rdt, tag in ((torch.complex128, np.float64, "f64"), (torch.complex64, np.float32, "f32")):
            for n_power in (10, 12, 14, 16):
                M = 1 << n_power
                csz = 16 if tag == "f64" else 8
                batch = (1 << 30) // (2 * M * csz)
                g = torch.Generator(device="cpu").manual_seed(SEED + n_power + rank)
                x = torch.randn(2 * batch * M, dtype=tdt, generator=g)
                buf = x.to(dev)
                roots, inv_roots, _ = gf.host_fft_tables(M // 2, tag)
                d_roots = torch.from_numpy(np.ascontiguousarray(roots)).to(dev)
                d_inv = torch.from_numpy(np.ascontiguousarray(inv_roots)).to(dev)
                L = gf.lib()
                fn = L.gpufft_fft_c2c_f64 if tag == "f64" else L.gpufft_fft_c2c_f32

                def step():
                    # the ABI call GPU_FFT makes (the Python mirror enforces the
                    # reference's n_power >= 12; 2^10 goes straight to the ABI)
                    gf.check(fn(buf.data_ptr(), d_roots.data_ptr(), n_power, 0, 1, 0, 1.0, 0.0, 2 * batch, 0,
                                None), "GPU_FFT forward")
                    gf.check(fn(buf.data_ptr(), d_inv.data_ptr(), n_power, 1, 1, 0, 1.0 / M, 0.0, batch, 1,
                                None), "GPU_FFT inverse")
                step()
                torch.cuda.synchronize()
                errs = []
                for k in (0, batch - 1):
                    a = x[k * M:(k + 1) * M].numpy().astype(np.complex128)
                    b = x[(batch + k) * M:(batch + k + 1) * M].numpy().astype(np.complex128)
                    want = np.fft.ifft(np.fft.fft(a) * np.fft.fft(b))
                    got = buf[k * M:(k + 1) * M].cpu().numpy().astype(np.complex128)
                    errs.append(float(np.linalg.norm(got - want) / np.linalg.norm(want)))
                buf.copy_(x.to(dev))
                for _ in range(args.warmup):
                    step()
                barrier()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0 = time.time()
                t_first = t_first or t0
                e0.record(stream)
                for _ in range(args.steps):
                    step()
                e1.record(stream)
                barrier()
                t1 = time.time()
                ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
                rows, ms_traced = traced_kernels(gf, lambda p, q, r: step(), None, None, None, args, stream, torch,
                                                 barrier, max_over_ranks)
                alg = 3 * M * csz * batch
                dropin = {"ms_per_step": ms, "products_s": world * batch / (ms * 1e-3),
                          "achieved_gbs": alg / (ms * 1e-3) / 1e9, "frac": alg / (ms * 1e-3) / 1e9 / peak,
                          "rel_l2_vs_fp64_cpu": max(errs),
                          "roofline": kernel_roofline(rows, peak, peak_kind, ms_traced, args.steps, alg / batch,
                                                      batch)}
                # the native fused cyclic product on the same operands
                xa = x.to(dev)
                av, bv = xa[: batch * M].view(batch, M), xa[batch * M:].view(batch, M)
                out = torch.empty_like(av)
                tab = gf.ffnt_tables(n_power + 1, tag, dev)
                need = int(gf.lib().gpufft_cyclic_mul_workspace_bytes(n_power, batch, 64 if tag == "f64" else 32))
                ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)

                def nstep():
                    gf.cyclic_mul(av, bv, out=out, tables=tab, workspace=ws)
                nstep()
                torch.cuda.synchronize()
                nerr = []
                for k in (0, batch - 1):
                    a = x[k * M:(k + 1) * M].numpy().astype(np.complex128)
                    b = x[(batch + k) * M:(batch + k + 1) * M].numpy().astype(np.complex128)
                    want = np.fft.ifft(np.fft.fft(a) * np.fft.fft(b))
                    got = out[k].cpu().numpy().astype(np.complex128)
                    nerr.append(float(np.linalg.norm(got - want) / np.linalg.norm(want)))
                for _ in range(args.warmup):
                    nstep()
                barrier()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(args.steps):
                    nstep()
                e1.record(stream)
                barrier()
                nms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
                nrows, nms_traced = traced_kernels(gf, lambda p, q, r: nstep(), None, None, None, args, stream,
                                                   torch, barrier, max_over_ranks)
                cases.append({"dtype": tag, "ring_log2": n_power, "batch": batch, "ms_per_step": nms,
                              "products_s": world * batch / (nms * 1e-3), "achieved_gbs": alg / (nms * 1e-3) / 1e9,
                              "frac": alg / (nms * 1e-3) / 1e9 / peak, "rel_l2_vs_fp64_cpu": max(nerr),
                              "roofline": kernel_roofline(nrows, peak, peak_kind, nms_traced, args.steps,
                                                          alg / batch, batch),
                              "dropin_gpu_fft": dropin})
                del x, buf, xa, av, bv, out, ws
                torch.cuda.empty_cache()
        t_last = time.time()
    head = [c for c in cases if c["dtype"] == "f64" and c["ring_log2"] == 16][0]
    return {
        "metric": "C_C cyclic products/s at N=2^16 (FP64, native fused product), with HBM GB/s per size",
        "value": head["products_s"], "unit": "products/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded i.i.d. N(0,1) re and im)",
        "config": {"workload": "C_C cyclic products, native fused (gpufft_cyclic_mul) with the reference API's "
                               "two GPU_FFT calls beside it, N = 2^10..2^16, batch ~1 GiB of input per size, "
                               "FP32 and FP64",
                   "l2": "inputs larger than L2 (no flush)"},
        "roofline": head["roofline"], "cases": cases,
        "gpu_launches": int(round(sum(k["launches_per_step"] for c in cases for r in (c["roofline"],
                                                                                       c["dropin_gpu_fft"]["roofline"])
                                      for k in r["kernels"]) * args.steps)),
        "clocks": clk.summary(t_first, t_last),
    }


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import __graft_entry__
    gf = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", device_id=dev, timeout=timedelta(seconds=120))

    n_power, batch = args.n_power, args.batch
    n = 1 << n_power
    a64, b64 = make_inputs(batch, n, rank)
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(ms):
        return reduce_max(ms, dist, dev)

    peak, peak_kind = peaks()
    if args.path in ("batch", "vjp", "cc"):
        fn = {"batch": run_batch, "vjp": run_vjp, "cc": run_cc}[args.path]
        line = fn(args, gf, dev, torch, world, rank, barrier, max_over_ranks, ClockSampler, peak, peak_kind)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    results = {}
    paths = [args.path] + ([p for p in ("split64", "f64") if p != args.path] if args.compare else [])
    with ClockSampler(local) as clk:
        time.sleep(0.5)  # let the sampler start before the timed regions
        for name in paths:
            step, host_step, alg, din, dout, launches = make_path(gf, name, n_power, batch, dev, torch)
            a_host = a64.to(din).pin_memory()
            b_host = b64.to(din).pin_memory()
            c_host = torch.empty((batch, n), dtype=dout).pin_memory()
            a, b = a_host.to(dev), b_host.to(dev)
            c = torch.empty((batch, n), dtype=dout, device=dev)
            ms, ms_e2e, t0, t1 = time_path(step, host_step, a, b, c, (a_host, b_host, c_host), args, stream, torch,
                                           barrier, max_over_ranks)
            rows, ms_traced = traced_kernels(gf, step, a, b, c, args, stream, torch, barrier, max_over_ranks)
            achieved = alg * batch / (ms * 1e-3) / 1e9
            results[name] = dict(ms=ms, ms_e2e=ms_e2e, t0=t0, t1=t1, alg=alg, launches=launches,
                                 kroof=kernel_roofline(rows, peak, peak_kind, ms_traced, args.steps, alg, batch),
                                 traced_launches=sum(r["launches"] for r in rows),
                                 value=world * batch / (ms * 1e-3), achieved=achieved,
                                 h2d=2 * batch * n * a_host.element_size(), d2h=batch * n * c_host.element_size(),
                                 dtype="f64" if name in ("f64", "dropin_f64", "split64") else "f32",
                                 c=c[:2].cpu() if rank == 0 else None)
            del a, b, c, a_host, b_host, c_host
        time.sleep(0.3)

    main_r = results[args.path]
    t_lo, t_hi = main_r["t0"], main_r["t1"]
    line = {
        "metric": f"negacyclic poly-mults/s at N=2^{n_power}", "value": main_r["value"], "unit": "products/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": main_r["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": main_r["dtype"],
        "data": "synthetic (seeded uniform integers in [0, 2^24))",
        "config": {"workload": f"FFNT negacyclic product N=2^{n_power}, batch {batch} per GPU, "
                               f"coefficients in [0, 2^24), path {args.path}",
                   "ring_log2": n_power, "batch_per_gpu": batch, "path": args.path,
                   "l2": "inputs larger than L2 (no flush)"},
        "roofline": main_r["kroof"],
        "chain": {"achieved_gbs": main_r["achieved"], "frac": main_r["achieved"] / peak,
                  "algorithmic_bytes_per_product": main_r["alg"],
                  "timed": "whole product chain (all launches of one step), CUDA events"},
        "e2e": {"value": world * batch / (main_r["ms_e2e"] * 1e-3), "unit": "products/s",
                "h2d_bytes_per_step": main_r["h2d"], "d2h_bytes_per_step": main_r["d2h"]},
        "gpu_launches": main_r["traced_launches"],
        "clocks": clk.summary(t_lo, t_hi),
    }
    for name, r in results.items():
        if name == args.path:
            continue
        line[name] = {"value": r["value"], "unit": "products/s", "ms_per_step": r["ms"],
                      "roofline_frac": r["achieved"] / peak, "achieved_gbs": r["achieved"],
                      "dominant_kernel": {k: r["kroof"][k] for k in ("kernel", "achieved", "frac", "mean_launch_us",
                                                                     "share_of_step", "traffic")},
                      "e2e_value": world * batch / (r["ms_e2e"] * 1e-3)}
    ours_gpu = ours_nv = None
    if rank == 0 and world == 1 and args.ref_gpu:
        ours_gpu = ours_gpu_cases(gf, a64, b64, n_power, batch, args, dev, torch)
        torch.cuda.synchronize()
        ours_nv = run_nvbench(os.path.join(ROOT, "gpu-fft_b200", "benchmark", "bin", NVBENCH_PROGRAM))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the cpu_baseline leg also checks the first product of each path at 64
        # seeded coefficients against the exact product, and times the
        # reference's GPU build
        import tempfile
        import numpy as np
        rng = np.random.default_rng(1)
        idx = np.sort(rng.choice(n, 64, replace=False)).astype(np.int32)
        with tempfile.TemporaryDirectory() as tmp:
            chk = os.path.join(tmp, "samples.npz")
            np.savez(chk, idx=idx, a0=a64[0].numpy(), b0=b64[0].numpy(),
                     **{f"out_{name}": r["c"][0].numpy()[idx] for name, r in results.items()})
            line["cpu_baseline"], ref_line = cpu_baseline_subprocess(args, chk)
        for name, r in ref_line.get("check", {}).items():
            tgt = line if name == args.path else line.get(name)
            if tgt is not None:
                tgt["exact_on_sample"] = r["exact"]
                tgt["max_abs_error_on_sample"] = r["max_abs_error"]
        if ours_gpu is not None:
            line["ref_gpu"] = merge_gpu_cases(ours_gpu, ref_line.get("ref_gpu"))
            line["nvbench"] = merge_nvbench(ours_nv, ref_line.get("nvbench"))
    elif ours_gpu is not None:
        line["ref_gpu"] = merge_gpu_cases(ours_gpu, None)
        line["nvbench"] = merge_nvbench(ours_nv, None)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
