"""The C++ drop-in boundary: a program written against the reference's API
(include/gpufft/fft.cuh, complex.cuh, fft_cpu.cuh, common_fft.cuh) compiles
unchanged and links against libgpufft_b200.so (CPU test); on a GPU it runs
and its products are exact (gpu test)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_example.cu")
LIBDIR = os.path.join(ROOT, "gpu-fft_b200", "lib")


def build(tmp_path):
    exe = str(tmp_path / "dropin_example")
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), SRC, "-o", exe, "-L", LIBDIR, "-lgpufft_b200",
           "-Xlinker", "-rpath," + LIBDIR]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_dropin_program_compiles_and_links(gf, tmp_path):
    gf.lib()  # library built
    exe = build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
@pytest.mark.parametrize("logn,batch", [(12, 2), (14, 1)])
def test_dropin_program_runs_exact(gf, dev, tmp_path, logn, batch):
    exe = build(tmp_path)
    r = subprocess.run([exe, str(logn), str(batch)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches=0 range_check=ok" in r.stdout
