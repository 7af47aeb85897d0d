"""ORACLE — test infrastructure only.

ctypes front end for the CPU checker:

* ``liboracle.so``  — ``oracle.c``, a C restatement of GPU-FFT's product path
  (reference ``src/lib/fft_cpu.cu`` and the device math of ``src/lib/fft.cu``)
  plus exact ``__int128`` schoolbook products;
* ``_ref/libgpufft_ref_cpu.so`` — the reference's own CPU classes compiled from
  source by ``oracle/Makefile`` (present where the reference sources were).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module, and only to check or to time the reference's CPU path.
The product library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_c_int = ctypes.c_int


def build(ref: bool = True) -> None:
    """Compile liboracle.so (and the reference CPU build when its sources exist)."""
    ref_dir = os.environ.get("REF_DIR", os.path.normpath(os.path.join(HERE, "..", "..", "reference")))
    target = ["all", f"REF_DIR={ref_dir}"] if ref and os.path.isdir(ref_dir) else [
        os.path.join(HERE, "liboracle.so")]
    subprocess.run(["make", "-s", "-C", HERE] + target, check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = ctypes.CDLL(path)
        for sfx, p, T in (("f64", _dp, ctypes.c_double), ("f32", _fp, ctypes.c_float)):
            getattr(L, f"orc_fft_tables_{sfx}").argtypes = [_c_int, p, p, p]
            getattr(L, f"orc_ffnt_tables_{sfx}").argtypes = [_c_int, p, p, p, p]
            getattr(L, f"orc_gpu_fft_c2c_{sfx}").argtypes = [p, p, _c_int, _c_int, _c_int, p, _c_int, _c_int]
            getattr(L, f"orc_gpu_fft_r2r_{sfx}").argtypes = [p, p, p, _c_int, _c_int, _c_int, p, _c_int, _c_int]
            getattr(L, f"orc_gpu_ffnt_{sfx}").argtypes = [p, p, p, p, _c_int, _c_int, p, _c_int, _c_int]
            getattr(L, f"orc_gpu_special_fft_{sfx}").argtypes = [p, p, _c_int, _c_int, p, _c_int]
            getattr(L, f"orc_cpu_fft_{sfx}").argtypes = [_c_int, p, p]
            getattr(L, f"orc_cpu_ifft_{sfx}").argtypes = [_c_int, p, p, T]
            getattr(L, f"orc_cpu_ffnt_mult_{sfx}").argtypes = [_c_int, _u64p, _u64p, _u64p, p, p, p, p]
        L.orc_bitreverse.argtypes = [_c_int, _c_int]
        L.orc_schoolbook_i64.argtypes = [_i64p, _i64p, _c_int, _c_int, _i64p, _i64p]
        L.orc_negacyclic_coeffs_i64.argtypes = [_i64p, _i64p, _c_int, _i32p, _c_int, _i64p, _i64p]
        L.orc_linear_coeffs_i64.argtypes = [_i64p, _i64p, _c_int, _i32p, _c_int, _i64p, _i64p]
        L.orc_balanced_digits_i64.argtypes = [_i64p, ctypes.c_long, _c_int, _c_int, _i32p]
        _LIB = L
    return _LIB


def ref():
    """The reference's own CPU build, or None where it was never compiled."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libgpufft_ref_cpu.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        for sfx, p in (("f64", _dp), ("f32", _fp)):
            getattr(R, f"ref_fft_tables_{sfx}").argtypes = [_c_int, p, p, p]
            getattr(R, f"ref_ffnt_tables_{sfx}").argtypes = [_c_int, p, p, p, p]
            getattr(R, f"ref_cpu_fft_{sfx}").argtypes = [_c_int, p, _c_int]
            getattr(R, f"ref_ffnt_mult_{sfx}").argtypes = [_c_int, _u64p, _u64p, _u64p]
        R.ref_bitreverse.argtypes = [_c_int, _c_int]
        R.ref_schoolbook_negacyclic_u64.argtypes = [_u64p, _u64p, ctypes.c_uint64, _c_int, _u64p]
        R.ref_schoolbook_linear_i32.argtypes = [_i32p, _i32p, ctypes.c_int32, _c_int, _i32p]
        R.ref_bench_ffnt_mult_f64.argtypes = [_c_int, _c_int, _c_int, _c_int, _u64p, _u64p, _u64p]
        R.ref_bench_ffnt_mult_f64.restype = ctypes.c_double
        R.ref_linear_product_f64.argtypes = [_c_int, _i64p, _i64p, _i64p]
        _REF = R
    return _REF


_REFGPU = None


def ref_gpu():
    """The reference's own GPU library (src/lib/fft.cu compiled for sm_100a by
    oracle/Makefile), or None where it was never compiled."""
    global _REFGPU
    if _REFGPU is None:
        path = os.path.join(HERE, "_ref", "libgpufft_ref_gpu.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        vp, i, d, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_float
        R.ref_gpu_ffnt_f64.argtypes = [vp, vp, vp, vp, i, i, d, d, i, i, vp]
        R.ref_gpu_ffnt_f32.argtypes = [vp, vp, vp, vp, i, i, f, f, i, i, vp]
        R.ref_gpu_fft_c2c_f64.argtypes = [vp, vp, i, i, i, d, d, i, i, vp]
        R.ref_gpu_fft_r2r_f64.argtypes = [vp, vp, vp, i, i, i, d, d, i, i, vp]
        R.ref_gpu_special_fft_f64.argtypes = [vp, vp, i, i, d, d, i, vp]
        R.ref_gpu_special_fft_f32.argtypes = [vp, vp, i, i, f, f, i, vp]
        _REFGPU = R
    return _REFGPU


def _np(dtype):
    return np.float64 if dtype in ("f64", np.float64) else np.float32


def _sfx(dtype):
    return "f64" if dtype in ("f64", np.float64) else "f32"


# --------------------------------------------------------------------------- tables
def fft_tables(n: int, dtype="f64"):
    """FFT<T>(n) tables: (reverse roots, inverse reverse roots, n_inverse); n complex each."""
    T = _np(dtype)
    r = np.zeros(2 * n, T)
    ri = np.zeros(2 * n, T)
    ninv = np.zeros(1, T)
    getattr(lib(), f"orc_fft_tables_{_sfx(dtype)}")(n, r, ri, ninv)
    return r.view(np.complex128 if T == np.float64 else np.complex64), \
        ri.view(np.complex128 if T == np.float64 else np.complex64), T(ninv[0])


def ffnt_tables(n: int, dtype="f64"):
    """FFNT<T>(n) tables: (reverse roots, inverse reverse roots, twist, untwist); n/2 complex each."""
    T = _np(dtype)
    C = np.complex128 if T == np.float64 else np.complex64
    h = n // 2
    out = [np.zeros(2 * h, T) for _ in range(4)]
    getattr(lib(), f"orc_ffnt_tables_{_sfx(dtype)}")(n, *out)
    return tuple(o.view(C) for o in out)


# --------------------------------------------------------------------------- GPU-API semantics
def _as_float_view(x, T):
    return np.ascontiguousarray(x).view(T)


def gpu_fft_c2c(inout, table, n_power, fft_type, reduction_poly, mod_inverse, batch, mult):
    """GPU_FFT (complex overload) semantics on the CPU; returns the updated buffer."""
    C = inout.dtype
    T = np.float64 if C == np.complex128 else np.float32
    buf = np.array(inout, dtype=C, copy=True)
    fv = buf.view(T)
    mi = np.array([np.real(mod_inverse), np.imag(mod_inverse)], T)
    getattr(lib(), f"orc_gpu_fft_c2c_{_sfx(T)}")(fv, _as_float_view(table.astype(C), T), n_power, fft_type,
                                                  reduction_poly, mi, batch, int(mult))
    return buf


def gpu_special_fft(inout, table, n_power, fft_type, mod_inverse, batch):
    """GPU_Special_FFT semantics on the CPU (reference fft.cu:727-1007); returns the
    updated buffer of batch vectors of 2^n_power complex."""
    C = inout.dtype
    T = np.float64 if C == np.complex128 else np.float32
    buf = np.array(inout, dtype=C, copy=True)
    mi = np.array([np.real(mod_inverse), np.imag(mod_inverse)], T)
    getattr(lib(), f"orc_gpu_special_fft_{_sfx(T)}")(buf.view(T), _as_float_view(table.astype(C), T), n_power,
                                                      fft_type, mi, batch)
    return buf


def gpu_fft_r2r(real_inout, temp, table, n_power, fft_type, reduction_poly, mod_inverse, batch, mult):
    """GPU_FFT (real overload) semantics; returns (real_inout, temp) after the call."""
    T = real_inout.dtype.type
    C = np.complex128 if T == np.float64 else np.complex64
    r = np.array(real_inout, dtype=T, copy=True)
    t = np.array(temp, dtype=C, copy=True)
    mi = np.array([np.real(mod_inverse), np.imag(mod_inverse)], T)
    getattr(lib(), f"orc_gpu_fft_r2r_{_sfx(T)}")(r, t.view(T), _as_float_view(table.astype(C), T), n_power,
                                                  fft_type, reduction_poly, mi, batch, int(mult))
    return r, t


def gpu_ffnt(inout, temp, twist, table, n_power, fft_type, mod_inverse, batch, mult):
    """GPU_FFNT semantics; returns (inout, temp) after the call."""
    T = inout.dtype.type
    C = np.complex128 if T == np.float64 else np.complex64
    r = np.array(inout, dtype=T, copy=True)
    t = np.array(temp, dtype=C, copy=True)
    mi = np.array([np.real(mod_inverse), np.imag(mod_inverse)], T)
    getattr(lib(), f"orc_gpu_ffnt_{_sfx(T)}")(r, t.view(T), _as_float_view(twist.astype(C), T),
                                               _as_float_view(table.astype(C), T), n_power, fft_type, mi, batch,
                                               int(mult))
    return r, t


def cpu_fft(n, data, dtype="f64", inverse=False):
    T = _np(dtype)
    C = np.complex128 if T == np.float64 else np.complex64
    d = np.array(data, dtype=C, copy=True)
    r, ri, ninv = fft_tables(n, dtype)
    if inverse:
        getattr(lib(), f"orc_cpu_ifft_{_sfx(dtype)}")(n, d.view(T), ri.view(T), ninv)
    else:
        getattr(lib(), f"orc_cpu_fft_{_sfx(dtype)}")(n, d.view(T), r.view(T))
    return d


def cpu_ffnt_mult(n, a, b, dtype="f64"):
    T = _np(dtype)
    r, ri, tw, utw = ffnt_tables(n, dtype)
    out = np.zeros(n, np.uint64)
    getattr(lib(), f"orc_cpu_ffnt_mult_{_sfx(dtype)}")(n, np.ascontiguousarray(a, np.uint64),
                                                       np.ascontiguousarray(b, np.uint64), out, r.view(T),
                                                       ri.view(T), tw.view(T), utw.view(T))
    return out


# --------------------------------------------------------------------------- exact products
LINEAR, CYCLIC, NEGACYCLIC = 0, 1, 2


def schoolbook(a, b, kind=NEGACYCLIC):
    """Exact product as Python ints packed in an object array (128-bit range)."""
    a = np.ascontiguousarray(a, np.int64)
    b = np.ascontiguousarray(b, np.int64)
    n = a.shape[0]
    outn = 2 * n if kind == LINEAR else n
    lo = np.zeros(outn, np.int64)
    hi = np.zeros(outn, np.int64)
    lib().orc_schoolbook_i64(a, b, n, kind, lo, hi)
    return _join128(lo, hi)


def negacyclic_coeffs(a, b, idx):
    a = np.ascontiguousarray(a, np.int64)
    b = np.ascontiguousarray(b, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    lo = np.zeros(idx.shape[0], np.int64)
    hi = np.zeros(idx.shape[0], np.int64)
    lib().orc_negacyclic_coeffs_i64(a, b, a.shape[0], idx, idx.shape[0], lo, hi)
    return _join128(lo, hi)


def linear_coeffs(a, b, idx):
    a = np.ascontiguousarray(a, np.int64)
    b = np.ascontiguousarray(b, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    lo = np.zeros(idx.shape[0], np.int64)
    hi = np.zeros(idx.shape[0], np.int64)
    lib().orc_linear_coeffs_i64(a, b, a.shape[0], idx, idx.shape[0], lo, hi)
    return _join128(lo, hi)


def _join128(lo, hi):
    out = np.empty(lo.shape[0], dtype=object)
    for i in range(lo.shape[0]):
        out[i] = (int(hi[i]) << 64) + (int(lo[i]) & ((1 << 64) - 1))
    return out


def wrap64(vals):
    """Exact values reduced to signed 64-bit two's complement (int64 output semantics)."""
    out = np.empty(len(vals), np.int64)
    for i, v in enumerate(vals):
        v &= (1 << 64) - 1
        out[i] = v - (1 << 64) if v >= (1 << 63) else v
    return out


def balanced_digits(x, w, limbs):
    x = np.ascontiguousarray(x, np.int64).ravel()
    d = np.zeros(limbs * x.shape[0], np.int32)
    lib().orc_balanced_digits_i64(x, x.shape[0], w, limbs, d)
    return d.reshape(limbs, x.shape[0])
