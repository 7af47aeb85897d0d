"""The benchmark programs (gpu-fft_b200/benchmark) on the nvbench-compatible
harness: the reference's four benchmark programs (benchmark/*.cu: the same
benchmark names, axes Ring Size LogN 12..23 and Batch Count 1, and the same
GPU_FFT / GPU_FFNT calls) plus the native products. The same sources built
against the reference's library (oracle/_ref/bench) must list the same
benchmarks. CPU tests check the harness's command line; GPU tests run a few
states of each program."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "gpu-fft_b200", "benchmark", "bin")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "bench")
AXES = {"Ring Size LogN": list(range(12, 24)), "Batch Count": [1]}
PROGRAMS = {
    "gpu_fft_benchmark": ["GPU_FFT_Forward_Benchmark", "GPU_FFT_Inverse_Benchmark"],
    "gpu_fft_C_C_mult_benchmark": ["GPU_FFT_Poly_Mult_Benchmark"],
    "gpu_fft_R_R_mult_benchmark": ["GPU_FFT_Poly_Mult_Benchmark"],
    "gpu_ffnt_R_R_mult_benchmark": ["GPU_FFT_Poly_Mult_Benchmark"],
    "native_mult_benchmark": ["NATIVE_FFNT_Mult_Benchmark", "NATIVE_Split_Mult_Benchmark"],
}


def exe(name, where=BIN):
    p = os.path.join(where, name)
    if not os.path.exists(p):
        pytest.skip(f"{p} is not built (make -C gpu-fft_b200 benchmarks)")
    return p


def listing(path, *extra):
    out = subprocess.run([path, "--list", *extra], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    benches, cur = {}, None
    for line in out.stdout.splitlines():
        if not line.startswith(" "):
            cur = line.split(": ", 1)[1]
            benches[cur] = {}
        else:
            name, vals = line.strip().split(":", 1)
            benches[cur][name] = [int(v) for v in vals.split()]
    return benches


@pytest.mark.parametrize("prog", sorted(PROGRAMS))
def test_program_lists_reference_benchmarks_and_axes(prog):
    got = listing(exe(prog))
    assert list(got) == PROGRAMS[prog]
    for axes in got.values():
        assert axes == AXES


@pytest.mark.parametrize("prog", sorted(p for p in PROGRAMS if p != "native_mult_benchmark"))
def test_reference_build_lists_the_same(prog):
    assert listing(exe(prog, REF_BIN)) == listing(exe(prog))


def test_axis_overrides_and_bad_options():
    p = exe("gpu_ffnt_R_R_mult_benchmark")
    got = listing(p, "-a", "Ring Size LogN=[12:14]", "--axis", "Batch Count=[1,4]")
    assert got["GPU_FFT_Poly_Mult_Benchmark"] == {"Ring Size LogN": [12, 13, 14], "Batch Count": [1, 4]}
    got = listing(p, "-a", "Ring Size LogN=16")
    assert got["GPU_FFT_Poly_Mult_Benchmark"]["Ring Size LogN"] == [16]
    bad = subprocess.run([p, "--no-such-option"], capture_output=True, text=True, timeout=60)
    assert bad.returncode == 2 and "unknown option" in bad.stderr


def run_states(path, axis, tmp_path, *extra):
    out = tmp_path / (os.path.basename(path) + ".json")
    r = subprocess.run([path, "-a", axis, "--timeout", "0.2", "--json", str(out), "--md", os.devnull, *extra],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return json.loads(out.read_text())


@pytest.mark.gpu
@pytest.mark.parametrize("prog", sorted(PROGRAMS))
def test_program_runs_states(prog, tmp_path):
    res = run_states(exe(prog), "Ring Size LogN=[12,16]", tmp_path)
    assert [b["name"] for b in res["benchmarks"]] == PROGRAMS[prog]
    for b in res["benchmarks"]:
        assert [s["axes"]["Ring Size LogN"] for s in b["states"]] == [12, 16]
        for s in b["states"]:
            assert "skipped" not in s, s
            assert s["samples"] >= 1 and s["gpu_time_mean_s"] > 0 and s["cpu_time_mean_s"] > 0


@pytest.mark.gpu
def test_native_program_skips_unsupported_rings(tmp_path):
    # the native products take N up to 2^22: LogN 23 is reported as skipped, not timed
    res = run_states(exe("native_mult_benchmark"), "Ring Size LogN=23", tmp_path, "-b", "NATIVE_FFNT_Mult_Benchmark")
    (state,) = res["benchmarks"][0]["states"]
    assert "skipped" in state


@pytest.mark.gpu
def test_reference_build_runs(tmp_path):
    res = run_states(exe("gpu_ffnt_R_R_mult_benchmark", REF_BIN), "Ring Size LogN=[12,16]", tmp_path)
    for s in res["benchmarks"][0]["states"]:
        assert "skipped" not in s and s["gpu_time_mean_s"] > 0
