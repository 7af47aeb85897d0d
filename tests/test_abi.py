"""CPU tests of the C ABI: the library loads, exports every function that
include/gpufft_b200.h declares, and rejects bad arguments with the documented
status codes before any device work (no GPU needed for these calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    hdr = open(os.path.join(ROOT, "include", "gpufft_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(gpufft_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol(gf):
    L = gf.lib()
    names = declared_functions()
    assert len(names) >= 9
    for name in names:
        assert hasattr(L, name), name


def test_status_strings(gf):
    L = gf.lib()
    assert L.gpufft_status_string(0) == b"success"
    assert L.gpufft_status_string(1) == b"Invalid n_power range!"
    assert L.gpufft_version() >= 100


def test_range_and_argument_errors(gf):
    L = gf.lib()
    dummy = ctypes.c_void_p(256)
    # n_power outside the ABI range -> GPUFFT_ERROR_INVALID_N_POWER
    assert L.gpufft_fft_c2c_f64(dummy, dummy, 25, 0, 1, 0, 1.0, 0.0, 1, 0, None) == gf.ERROR_INVALID_N_POWER
    assert L.gpufft_fft_c2c_f32(dummy, dummy, 0, 0, 1, 0, 1.0, 0.0, 1, 0, None) == gf.ERROR_INVALID_N_POWER
    assert L.gpufft_ffnt_f64(dummy, dummy, dummy, dummy, 1, 0, 1.0, 0.0, 1, 0, None) == gf.ERROR_INVALID_N_POWER
    # null pointer / bad batch / bad enum -> GPUFFT_ERROR_INVALID_VALUE
    assert L.gpufft_fft_c2c_f64(None, dummy, 12, 0, 1, 0, 1.0, 0.0, 1, 0, None) == gf.ERROR_INVALID_VALUE
    assert L.gpufft_fft_r2r_f64(dummy, dummy, dummy, 12, 0, 1, 0, 1.0, 0.0, 0, 0, None) == gf.ERROR_INVALID_VALUE
    assert L.gpufft_fft_c2c_f64(dummy, dummy, 12, 7, 1, 0, 1.0, 0.0, 1, 0, None) == gf.ERROR_INVALID_VALUE
    assert L.gpufft_fft_c2c_f64(dummy, dummy, 12, 0, 9, 0, 1.0, 0.0, 1, 0, None) == gf.ERROR_INVALID_VALUE
    # misaligned complex pointers -> GPUFFT_ERROR_MISALIGNED
    odd = ctypes.c_void_p(264)  # 8 mod 16
    assert L.gpufft_fft_c2c_f64(odd, dummy, 12, 0, 1, 0, 1.0, 0.0, 1, 0, None) == gf.ERROR_MISALIGNED


def test_python_mirror_range_check_matches_reference(gf):
    # The reference throws std::invalid_argument("Invalid n_power range!") for
    # n_power <= 11 or >= 25 (fft.cu:522-525); the mirror raises ValueError
    # before touching any device buffer.
    cfg = gf.fft_configuration(n_power=11)
    with pytest.raises(ValueError, match="Invalid n_power range!"):
        gf.GPU_FFT(None, None, cfg, 1, False)
    cfg.n_power = 25
    with pytest.raises(ValueError, match="Invalid n_power range!"):
        gf.GPU_FFNT(None, None, None, None, cfg, 1, False)


@pytest.mark.parametrize("sfx", ["f64", "f32"])
def test_host_table_generators_match_reference_bitwise(gf, O, sfx):
    # the drop-in API's FFT<T>/FFNT<T> table generators (host code in the
    # library) give the reference's tables bit for bit (golden fixtures made by
    # the reference's own build, and the oracle for other sizes)
    import numpy as np
    gold = os.path.join(ROOT, "tests", "golden")
    g = np.load(os.path.join(gold, f"fft_tables_{sfx}.npz"))
    r, ri, ninv = gf.host_fft_tables(int(g["n"]), sfx)
    T = np.float64 if sfx == "f64" else np.float32
    assert np.array_equal(r.view(T), g["rev_roots"]) and np.array_equal(ri.view(T), g["rev_inv_roots"])
    assert ninv == g["n_inverse"][0]
    g = np.load(os.path.join(gold, f"ffnt_tables_{sfx}.npz"))
    for got, key in zip(gf.host_ffnt_tables(int(g["n"]), sfx), ["rev_roots", "rev_inv_roots", "twist", "untwist"]):
        assert np.array_equal(got.view(T), g[key]), key
    for n in (4, 64, 1 << 15):
        for got, want in zip(gf.host_ffnt_tables(n, sfx), O.ffnt_tables(n, sfx)):
            assert np.array_equal(got, want)
        r, ri, ninv = gf.host_fft_tables(n, sfx)
        wr, wri, wn = O.fft_tables(n, sfx)
        assert np.array_equal(r, wr) and np.array_equal(ri, wri) and ninv == wn


def test_split_plan_host_logic(gf):
    # limb plans picked by the error model (host-only, no GPU)
    assert gf.split_plan(16, 24, True) == (5, 5)
    w, k = gf.split_plan(12, 24, True)
    assert w * k >= 24 and k <= 4
    assert gf.split_plan(16, 16, False)[0] * gf.split_plan(16, 16, False)[1] >= 16


def test_trace_collect_without_records(gf):
    # tracing is off by default; collecting with nothing recorded needs no GPU
    gf.trace_enable(False)
    assert gf.trace_collect() == []


def test_cluster_tile_limit_roundtrip(gf):
    # host-only setting: no device work; a negative value queries
    prev = gf.set_cluster_tiles(-1)
    assert prev >= 0
    try:
        assert gf.set_cluster_tiles(0) == prev
        assert gf.set_cluster_tiles(-1) == 0
        assert gf.set_cluster_tiles(1 << 30) == 0
        assert gf.set_cluster_tiles(-5) == 1 << 30
    finally:
        gf.set_cluster_tiles(prev)
    assert gf.set_cluster_tiles(-1) == prev
