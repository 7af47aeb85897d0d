"""Time the reference's own GPU path (oracle/_ref/libgpufft_ref_gpu.so, its
src/lib/fft.cu built for sm_100a) against this library on the same B200, same
data and same tables, and print one JSON line per case.

  python tests/compare_reference_gpu.py

Cases: the reference's benchmark shape (bench_gpu_ffnt_R_R_mult.cu: FFNT
product, LogN 12..23, batch 1) and the batched workload (N = 2^16, batch 256,
FP64); the C_C product through GPU_FFT (batched); GPU_Special_FFT forward +
inverse. "ours_dropin" is the same drop-in API; "ours_fused" is the native
fused product through its C ABI entry point (as the other two are called).
CUDA events, 3 warm-ups, median of 20 timed calls.
"""
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import __graft_entry__  # noqa: E402
import oracle as O  # noqa: E402


def timed(fn, reps=20):
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def main():
    gf = __graft_entry__.load_package()
    R = O.ref_gpu()
    if R is None:
        print(json.dumps({"unavailable": "reference GPU build absent (make -C oracle refgpu)"}))
        return
    dev = torch.device("cuda:0")
    cases = [(16, 256), (15, 256)] + [(lg, 1) for lg in range(12, 24)]
    for n_power, batch in cases:
        n = 1 << n_power
        h = n // 2
        tabs = [torch.from_numpy(np.ascontiguousarray(t)).to(dev) for t in O.ffnt_tables(n, "f64")]
        roots, inv_roots, twist, untwist = tabs
        inout = torch.randint(0, 1 << 10, (2 * batch * n,), device=dev).double()
        temp = torch.empty(2 * batch * h, dtype=torch.complex128, device=dev)

        def two_calls(f):
            def run():
                f(inout.data_ptr(), temp.data_ptr(), twist.data_ptr(), roots.data_ptr(), n_power, 0, 1.0, 0.0,
                  2 * batch, 0, None)
                f(inout.data_ptr(), temp.data_ptr(), untwist.data_ptr(), inv_roots.data_ptr(), n_power, 1, 1.0 / h,
                  0.0, batch, 1, None)
            return run
        t_ref = timed(two_calls(R.ref_gpu_ffnt_f64))
        t_ours = timed(two_calls(gf.lib().gpufft_ffnt_f64))
        t_fused = None
        if n_power <= 22:  # the native fused product covers rings up to 2^22
            a = inout[: batch * n].view(batch, n).clone()
            b = inout[batch * n:].view(batch, n).clone()
            ntab = gf.ffnt_tables(n_power, "f64", dev)
            c = torch.empty_like(a)
            ws = torch.empty(max(1, gf.negacyclic_mul_workspace_bytes(n_power, batch, 64)), dtype=torch.uint8,
                             device=dev)
            L = gf.lib()
            args = (a.data_ptr(), b.data_ptr(), c.data_ptr(), n_power, batch, ntab.data_ptr(), ws.data_ptr(),
                    ws.numel(), None)
            # through the C ABI, like the reference and the drop-in calls
            t_fused = timed(lambda: gf.check(L.gpufft_negacyclic_mul_f64(*args), "negacyclic_mul"))
        print(json.dumps({"case": f"FFNT product f64 N=2^{n_power} batch {batch}", "ref_gpu_ms": t_ref,
                          "ours_dropin_ms": t_ours, "ours_fused_ms": t_fused, "speedup_dropin": t_ref / t_ours,
                          "speedup_fused": (t_ref / t_fused) if t_fused else None}), flush=True)
    more_cases(gf, R, dev)


def more_cases(gf, R, dev):
    """C_C product through GPU_FFT and GPU_Special_FFT (forward + inverse)."""
    L = gf.lib()
    for n_power, batch in ((12, 1024), (16, 64), (16, 1), (20, 4)):
        M = 1 << n_power
        roots, inv_roots, _ = O.fft_tables(M // 2, "f64")
        d_r = torch.from_numpy(np.ascontiguousarray(roots)).to(dev)
        d_i = torch.from_numpy(np.ascontiguousarray(inv_roots)).to(dev)
        buf = torch.randn(2 * batch * M, dtype=torch.complex128, device=dev)

        def ref_c2c():
            R.ref_gpu_fft_c2c_f64(buf.data_ptr(), d_r.data_ptr(), n_power, 0, 1, 1.0, 0.0, 2 * batch, 0, None)
            R.ref_gpu_fft_c2c_f64(buf.data_ptr(), d_i.data_ptr(), n_power, 1, 1, 1.0 / M, 0.0, batch, 1, None)

        def our_c2c():
            L.gpufft_fft_c2c_f64(buf.data_ptr(), d_r.data_ptr(), n_power, 0, 1, 0, 1.0, 0.0, 2 * batch, 0, None)
            L.gpufft_fft_c2c_f64(buf.data_ptr(), d_i.data_ptr(), n_power, 1, 1, 0, 1.0 / M, 0.0, batch, 1, None)
        t_ref = timed(ref_c2c)
        t_ours = timed(our_c2c)
        a = buf[: batch * M].view(batch, M).clone()
        b = buf[batch * M:].view(batch, M).clone()
        tab = gf.ffnt_tables(n_power + 1, "f64", dev)
        out = torch.empty_like(a)
        ws = torch.empty(max(1, int(L.gpufft_cyclic_mul_workspace_bytes(n_power, batch, 64))), dtype=torch.uint8,
                         device=dev)
        cargs = (a.data_ptr(), b.data_ptr(), out.data_ptr(), n_power, batch, tab.data_ptr(), ws.data_ptr(),
                 ws.numel(), None)
        t_nat = timed(lambda: gf.check(L.gpufft_cyclic_mul_f64(*cargs), "cyclic_mul"))
        print(json.dumps({"case": f"C_C product f64 N=2^{n_power} batch {batch}", "ref_gpu_ms": t_ref,
                          "ours_dropin_ms": t_ours, "ours_fused_ms": t_nat, "speedup_dropin": t_ref / t_ours,
                          "speedup_fused": t_ref / t_nat}), flush=True)
    for n_power, batch in ((12, 1), (16, 1), (20, 1), (16, 64), (12, 1024)):
        M = 1 << n_power
        x = torch.randn(batch * M, dtype=torch.complex128, device=dev)
        tab = torch.exp(2j * np.pi * torch.rand(M, dtype=torch.float64, device=dev))

        def special(f):
            def run():
                f(x.data_ptr(), tab.data_ptr(), n_power, 0, 1.0, 0.0, batch, None)
                f(x.data_ptr(), tab.data_ptr(), n_power, 1, 1.0 / M, 0.0, batch, None)
            return run
        t_ref = timed(special(R.ref_gpu_special_fft_f64))
        t_ours = timed(special(L.gpufft_special_fft_f64))
        print(json.dumps({"case": f"GPU_Special_FFT f64 fwd+inv N=2^{n_power} batch {batch}", "ref_gpu_ms": t_ref,
                          "ours_dropin_ms": t_ours, "ours_fused_ms": None, "speedup_dropin": t_ref / t_ours,
                          "speedup_fused": None}), flush=True)


if __name__ == "__main__":
    main()
