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

SEED = 20261203 + 3  # config 3 of the workload list


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--path", choices=["f64", "f32", "dropin_f64"], default="f64")
    p.add_argument("--n-power", type=int, default=16)
    p.add_argument("--batch", type=int, default=256)
    p.add_argument("--no-cpu-baseline", action="store_true")
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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
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


def run_reference(args, rank, world):
    if rank != 0:
        return
    n = 1 << args.n_power
    threads = os.cpu_count() or 1
    # each step: a bounded sample of the workload's products (products/s is per-product)
    count = max(threads, cpu_sample_count(n, threads) // 4)
    vals = []
    for i in range(args.warmup + args.steps):
        v, kind, cores = cpu_baseline_reference(n, count, threads)
        if i >= args.warmup:
            vals.append(v)
    val = statistics.median(vals)
    line = {"impl": "reference", "metric": f"negacyclic poly-mults/s at N=2^{args.n_power}", "value": val,
            "unit": "products/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": count / val * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded uniform [0, 2^24))",
            "config": {"workload": f"FFNT negacyclic product N=2^{args.n_power}, batch {args.batch}, "
                                   "coefficients in [0, 2^24)", "ring_log2": args.n_power, "batch": args.batch,
                       "l2": "inputs > L2"},
            "cpu_baseline": {"value": val, "unit": "products/s", "cores": cores, "kind": kind,
                             "sample": f"{count} products of N=2^{args.n_power} per step, FFNT<double>::MULT"},
            "e2e": {"value": val, "unit": "products/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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
        dist.init_process_group("nccl", device_id=dev)

    n_power, batch = args.n_power, args.batch
    n = 1 << n_power
    f64 = args.path in ("f64", "dropin_f64")
    fdt = torch.float64 if f64 else torch.float32
    esz = 8 if f64 else 4
    a64, b64 = make_inputs(batch, n, rank)
    a_host = a64.to(fdt).pin_memory()
    b_host = b64.to(fdt).pin_memory()
    c_host = torch.empty_like(a_host).pin_memory()
    a = a_host.to(dev)
    b = b_host.to(dev)
    c = torch.empty_like(a)
    stream = torch.cuda.current_stream()

    if args.path in ("f64", "f32"):
        tables = gf.ffnt_tables(n_power, "f64" if f64 else "f32", dev)
        ws_bytes = gf.negacyclic_mul_workspace_bytes(n_power, batch, 64 if f64 else 32)
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
        m = n_power - 1
        waves = 1 if m <= 12 else -(-batch // max(1, ws_bytes // (2 * (1 << m) * 2 * esz)))
        launches_per_step = 1 if m <= 12 else 3 * waves

        def step(x, y, out):
            gf.negacyclic_mul(x, y, out=out, tables=tables, workspace=ws)
        alg_bytes = 3 * n * esz * batch
    else:
        import numpy as np
        import oracle as O  # table values only (host-side generators of the drop-in API)
        roots, inv_roots, twist, untwist = [torch.from_numpy(np.ascontiguousarray(t)).to(dev)
                                            for t in O.ffnt_tables(n, "f64")]
        inout = torch.empty(2 * batch * n, dtype=torch.float64, device=dev)
        temp = torch.empty(batch * n, dtype=torch.complex128, device=dev)
        cf = gf.fft_configuration(n_power=n_power, fft_type=gf.FORWARD)
        ci = gf.fft_configuration(n_power=n_power, fft_type=gf.INVERSE, mod_inverse=1.0 / (n // 2))
        launches_per_step = 4 if n_power - 1 > 12 else 2

        def step(x, y, out):
            inout[: batch * n].copy_(x.view(-1))
            inout[batch * n:].copy_(y.view(-1))
            gf.GPU_FFNT(inout, temp, twist, roots, cf, 2 * batch, False)
            gf.GPU_FFNT(inout, temp, untwist, inv_roots, ci, batch, True)
            out.view(-1).copy_(inout[: batch * n])
        alg_bytes = 3 * n * 8 * batch

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(ms):
        if dist is None:
            return ms
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident timing
    for _ in range(args.warmup):
        step(a, b, c)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step(a, b, c)
        e1.record(stream)
        barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)

    # ---- end to end through the public API with host buffers
    for _ in range(max(1, args.warmup // 2)):
        a.copy_(a_host, non_blocking=True)
        b.copy_(b_host, non_blocking=True)
        step(a, b, c)
        c_host.copy_(c, non_blocking=True)
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        a.copy_(a_host, non_blocking=True)
        b.copy_(b_host, non_blocking=True)
        step(a, b, c)
        c_host.copy_(c, non_blocking=True)
    e3.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3) / args.steps)

    # ---- correctness spot check on this rank's last product (exact when f64 holds it)
    peak, peak_kind = peaks()
    value = world * batch / (ms * 1e-3)
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    line = {
        "metric": f"negacyclic poly-mults/s at N=2^{n_power}", "value": value, "unit": "products/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if f64 else "f32", "data": "synthetic (seeded uniform integers in [0, 2^24))",
        "config": {"workload": f"FFNT negacyclic product N=2^{n_power}, batch {batch} per GPU, "
                               f"coefficients in [0, 2^24), path {args.path}",
                   "ring_log2": n_power, "batch_per_gpu": batch, "path": args.path,
                   "l2": "inputs larger than L2 (no flush)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_product": alg_bytes // batch,
                     "timed": "whole product chain (all launches of one step), CUDA events"},
        "e2e": {"value": world * batch / (ms_e2e * 1e-3), "unit": "products/s",
                "h2d_bytes_per_step": 2 * batch * n * esz, "d2h_bytes_per_step": batch * n * esz},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cnt = cpu_sample_count(n, threads)
        v, kind, cores = cpu_baseline_reference(n, cnt, threads)
        line["cpu_baseline"] = {"value": v, "unit": "products/s", "cores": cores, "kind": kind,
                                "sample": f"{cnt} products of N=2^{n_power}, FFNT<double>::MULT, one per thread"}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
