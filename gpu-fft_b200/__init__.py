"""gpufft_b200 — Python mirror of GPU-FFT's polynomial-multiplication API.

The names, argument order and error behaviour follow the reference's C++ API
(src/include/gpufft/fft.cuh:37-51, 120-132, 269-273; src/lib/fft.cu:517-725,
1386-1515):

* ``fft_configuration`` (n_power, fft_type, reduction_poly, zero_padding,
  mod_inverse, stream), ``FORWARD``/``INVERSE``, ``X_N_plus``/``X_N_minus``;
* ``GPU_FFT(inout, roots, cfg, batch, multiplication)`` (C_C) and
  ``GPU_FFT(real_inout, temp, roots, cfg, batch, multiplication)`` (R_R);
* ``GPU_FFNT(inout, temp, twist_or_untwist, roots, cfg, batch, multiplication)``;
* ``ValueError("Invalid n_power range!")`` where the reference throws
  ``std::invalid_argument`` and ``CudaException`` where it throws one.

Every call goes through the C ABI of ``lib/libgpufft_b200.so`` (declared in
``include/gpufft_b200.h``) on hand-written sm_100a kernels. Device buffers are
torch CUDA tensors, used only for memory and streams. There is no CPU
fallback: importing this package without the built library raises.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgpufft_b200.so")

FORWARD, INVERSE = 0, 1
X_N_plus, X_N_minus = 0, 1

SUCCESS = 0
ERROR_INVALID_N_POWER = 1
ERROR_INVALID_VALUE = 2
ERROR_CUDA = 3
ERROR_WORKSPACE = 4
ERROR_MISALIGNED = 5


class CudaException(RuntimeError):
    """A CUDA error raised under a library call (reference common_fft.cuh:19-49)."""

    def __init__(self, where: str, code: int):
        self.code = code
        super().__init__(f"CUDA Error in {where}: cudaError {code}")


class GpufftError(RuntimeError):
    def __init__(self, status: int, msg: str):
        self.status = status
        super().__init__(msg)


_lib = None


def lib() -> ctypes.CDLL:
    """Load the native library; raise if it was not built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"gpufft_b200 native library missing: {LIB_PATH} (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        L.gpufft_fft_c2c_f32.argtypes = [vp, vp, i, i, i, i, f, f, i, i, vp]
        L.gpufft_fft_c2c_f64.argtypes = [vp, vp, i, i, i, i, d, d, i, i, vp]
        L.gpufft_fft_r2r_f32.argtypes = [vp, vp, vp, i, i, i, i, f, f, i, i, vp]
        L.gpufft_fft_r2r_f64.argtypes = [vp, vp, vp, i, i, i, i, d, d, i, i, vp]
        L.gpufft_ffnt_f32.argtypes = [vp, vp, vp, vp, i, i, f, f, i, i, vp]
        L.gpufft_ffnt_f64.argtypes = [vp, vp, vp, vp, i, i, d, d, i, i, vp]
        L.gpufft_special_fft_f32.argtypes = [vp, vp, i, i, f, f, i, vp]
        L.gpufft_special_fft_f64.argtypes = [vp, vp, i, i, d, d, i, vp]
        sz = ctypes.c_size_t
        L.gpufft_ffnt_tables_count.argtypes = [i]
        L.gpufft_ffnt_tables_count.restype = sz
        L.gpufft_ffnt_make_tables_f32.argtypes = [i, vp, vp]
        L.gpufft_ffnt_make_tables_f64.argtypes = [i, vp, vp]
        L.gpufft_negacyclic_mul_workspace_bytes.argtypes = [i, i, i]
        L.gpufft_negacyclic_mul_workspace_bytes.restype = sz
        L.gpufft_negacyclic_mul_f32.argtypes = [vp, vp, vp, i, i, vp, vp, sz, vp]
        L.gpufft_negacyclic_mul_f64.argtypes = [vp, vp, vp, i, i, vp, vp, sz, vp]
        L.gpufft_negacyclic_mul_f64_noalloc.argtypes = [vp, vp, vp, i, i, vp, vp]
        L.gpufft_cyclic_mul_workspace_bytes.argtypes = [i, i, i]
        L.gpufft_cyclic_mul_workspace_bytes.restype = sz
        L.gpufft_cyclic_mul_f32.argtypes = [vp, vp, vp, i, i, vp, vp, sz, vp]
        L.gpufft_cyclic_mul_f64.argtypes = [vp, vp, vp, i, i, vp, vp, sz, vp]
        L.gpufft_host_fft_tables_f32.argtypes = [i, vp, vp, vp]
        L.gpufft_host_fft_tables_f64.argtypes = [i, vp, vp, vp]
        L.gpufft_host_ffnt_tables_f32.argtypes = [i, vp, vp, vp, vp]
        L.gpufft_host_ffnt_tables_f64.argtypes = [i, vp, vp, vp, vp]
        L.gpufft_linear_mul_workspace_bytes.argtypes = [i, i, i]
        L.gpufft_linear_mul_workspace_bytes.restype = sz
        L.gpufft_linear_mul_f32.argtypes = [vp, vp, vp, i, i, vp, vp, sz, vp]
        L.gpufft_linear_mul_f64.argtypes = [vp, vp, vp, i, i, vp, vp, sz, vp]
        L.gpufft_linear_mul_vjp_workspace_bytes.argtypes = [i, i]
        L.gpufft_linear_mul_vjp_workspace_bytes.restype = sz
        L.gpufft_linear_mul_vjp_f32.argtypes = [vp, vp, vp, vp, vp, i, i, vp, vp, sz, vp]
        L.gpufft_conv_vjp_f32.argtypes = [vp, vp, vp, vp, vp, i, i, vp, vp, sz, vp]
        ll = ctypes.c_longlong
        vpp = ctypes.POINTER(ctypes.c_void_p)
        L.gpufft_batch_plan_create.argtypes = [vpp, ctypes.POINTER(ctypes.c_int), i, i, vp]
        L.gpufft_batch_plan_layout.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ll),
                                               ctypes.POINTER(ll)]
        L.gpufft_batch_plan_execute.argtypes = [vp, vp, vp, vp, vp]
        L.gpufft_batch_plan_run.argtypes = [vp, vp, vp, vp, vp]
        L.gpufft_batch_plan_autotune.argtypes = [vp, vp, vp, vp, ctypes.c_char_p, vp]
        L.gpufft_batch_plan_capture.argtypes = [vp, vp, vp, vp, vp]
        L.gpufft_batch_plan_replay.argtypes = [vp, vp]
        L.gpufft_batch_plan_set_shape.argtypes = [vp, i, i]
        L.gpufft_batch_plan_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ll)]
        L.gpufft_batch_plan_status.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.gpufft_batch_plan_destroy.argtypes = [vp]
        ip = ctypes.POINTER(ctypes.c_int)
        L.gpufft_split_plan.argtypes = [i, i, i, ip, ip]
        L.gpufft_negacyclic_mul_split_workspace_bytes.argtypes = [i, i, i]
        L.gpufft_negacyclic_mul_split_workspace_bytes.restype = sz
        L.gpufft_negacyclic_mul_split_f32.argtypes = [vp, vp, vp, i, i, i, i, i, i, vp, vp, sz, vp, vp]
        L.gpufft_negacyclic_mul_split_f64.argtypes = [vp, vp, vp, i, i, i, i, i, i, vp, vp, sz, vp, vp]
        L.gpufft_split_plan_f64.argtypes = [i, i, i, ip, ip]
        L.gpufft_negacyclic_mul_split_f64_workspace_bytes.argtypes = [i, i, i]
        L.gpufft_negacyclic_mul_split_f64_workspace_bytes.restype = sz
        L.gpufft_split_batch_plan_create.argtypes = [vpp, ctypes.POINTER(ctypes.c_int), i, i, i, vp]
        L.gpufft_split_batch_plan_layout.argtypes = [vp, ctypes.POINTER(ll), ctypes.POINTER(ll),
                                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.gpufft_split_batch_plan_execute.argtypes = [vp, vp, vp, vp, vp, vp]
        L.gpufft_split_batch_plan_capture.argtypes = [vp, vp, vp, vp, vp, vp]
        L.gpufft_split_batch_plan_replay.argtypes = [vp, vp]
        L.gpufft_split_batch_plan_destroy.argtypes = [vp]
        L.gpufft_trace_enable.argtypes = [i]
        L.gpufft_trace_collect.argtypes = [i, ctypes.c_char_p, i, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ll), ctypes.POINTER(i)]
        L.gpufft_negacyclic_mul_host_workspace_bytes.argtypes = [i, i, i, i]
        L.gpufft_negacyclic_mul_host_workspace_bytes.restype = sz
        L.gpufft_negacyclic_mul_f32_host.argtypes = [vp, vp, vp, i, i, i, vp, vp, sz, vp]
        L.gpufft_negacyclic_mul_f64_host.argtypes = [vp, vp, vp, i, i, i, vp, vp, sz, vp]
        L.gpufft_negacyclic_mul_split_f32_host_workspace_bytes.argtypes = [i, i, i, i]
        L.gpufft_negacyclic_mul_split_f32_host_workspace_bytes.restype = sz
        L.gpufft_negacyclic_mul_split_f32_host.argtypes = [vp, vp, vp, i, i, i, i, i, i, i, vp, vp, sz, vp, vp]
        L.gpufft_last_cuda_error.restype = i
        L.gpufft_status_string.restype = ctypes.c_char_p
        L.gpufft_status_string.argtypes = [i]
        L.gpufft_version.restype = i
        L.gpufft_set_cluster_tiles.argtypes = [i]
        L.gpufft_set_cluster_tiles.restype = i
        L.gpufft_set_programmatic_launch.argtypes = [i]
        L.gpufft_set_programmatic_launch.restype = i
        L.gpufft_batch_plan_set_barrier.argtypes = [vp, ctypes.c_uint, ctypes.c_uint]
        L.gpufft_set_f64_middle.argtypes = [i]
        L.gpufft_set_f64_middle.restype = i
        L.gpufft_set_split_tile.argtypes = [i]
        L.gpufft_set_split_tile.restype = i
        L.gpufft_split_wait_timeouts.argtypes = [vp, i]
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    """Map a C-ABI status to the reference's exceptions."""
    if status == SUCCESS:
        return
    if status == ERROR_INVALID_N_POWER:
        raise ValueError("Invalid n_power range!")
    if status == ERROR_CUDA:
        raise CudaException(where, lib().gpufft_last_cuda_error())
    raise GpufftError(status, f"{where}: {lib().gpufft_status_string(status).decode()}")


@dataclasses.dataclass
class fft_configuration:
    """gpufft::fft_configuration<T> (reference fft.cuh:43-51)."""
    n_power: int = 0
    fft_type: int = FORWARD
    reduction_poly: int = X_N_minus
    zero_padding: bool = False
    mod_inverse: complex = 1.0 + 0.0j
    stream: Optional[object] = None  # torch.cuda.Stream, a raw cudaStream_t int, or None


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream or None
    if isinstance(stream, int):
        return stream or None
    return stream.cuda_stream or None


def _ptr(t) -> int:
    if not t.is_cuda:
        raise GpufftError(ERROR_INVALID_VALUE, "device buffers must be CUDA tensors")
    return t.data_ptr()


def _is_f64(t) -> bool:
    import torch
    return t.dtype in (torch.float64, torch.complex128)


def _range_check(n_power: int) -> None:
    # reference fft.cu:522-525, 606-609, 1392-1395
    if n_power <= 11 or n_power >= 25:
        raise ValueError("Invalid n_power range!")


def GPU_FFT(*args):
    """GPU_FFT(inout, roots, cfg, batch, multiplication)            -- C_C
    GPU_FFT(real_inout, temp, roots, cfg, batch, multiplication)     -- R_R
    (reference fft.cuh:120-132)."""
    L = lib()
    if len(args) == 5:
        inout, roots, cfg, batch, mult = args
        _range_check(cfg.n_power)
        f = L.gpufft_fft_c2c_f64 if _is_f64(inout) else L.gpufft_fft_c2c_f32
        st = f(_ptr(inout), _ptr(roots), cfg.n_power, int(cfg.fft_type), int(cfg.reduction_poly),
               int(bool(cfg.zero_padding)), complex(cfg.mod_inverse).real, complex(cfg.mod_inverse).imag,
               int(batch), int(bool(mult)), _stream_handle(cfg.stream))
        check(st, "GPU_FFT")
        return
    if len(args) == 6:
        real_inout, temp, roots, cfg, batch, mult = args
        _range_check(cfg.n_power)
        f = L.gpufft_fft_r2r_f64 if _is_f64(real_inout) else L.gpufft_fft_r2r_f32
        st = f(_ptr(real_inout), _ptr(temp), _ptr(roots), cfg.n_power, int(cfg.fft_type),
               int(cfg.reduction_poly), int(bool(cfg.zero_padding)), complex(cfg.mod_inverse).real,
               complex(cfg.mod_inverse).imag, int(batch), int(bool(mult)), _stream_handle(cfg.stream))
        check(st, "GPU_FFT")
        return
    raise TypeError("GPU_FFT takes 5 (C_C) or 6 (R_R) arguments")


def GPU_Special_FFT(inout, root_table, cfg, batch):
    """GPU_Special_FFT (reference fft.cuh:194-197, fft.cu:929-1007): the special FFT
    of CKKS encoding, in place on batch vectors of 2^n_power complex."""
    if cfg.n_power <= 10 or cfg.n_power >= 25:  # fft.cu:933-936
        raise ValueError("Invalid n_power range!")
    L = lib()
    f = L.gpufft_special_fft_f64 if _is_f64(inout) else L.gpufft_special_fft_f32
    mi = complex(cfg.mod_inverse)
    check(f(_ptr(inout), _ptr(root_table), cfg.n_power, int(cfg.fft_type), mi.real, mi.imag, int(batch),
            _stream_handle(cfg.stream)), "GPU_Special_FFT")


def GPU_FFNT(inout, temp, twist_table, root_table, cfg, batch, multiplication):
    """GPU_FFNT (reference fft.cuh:269-273, fft.cu:1386-1515). For the inverse,
    pass the untwist table as twist_table, as the reference's callers do."""
    _range_check(cfg.n_power)
    L = lib()
    f = L.gpufft_ffnt_f64 if _is_f64(inout) else L.gpufft_ffnt_f32
    st = f(_ptr(inout), _ptr(temp), _ptr(twist_table), _ptr(root_table), cfg.n_power, int(cfg.fft_type),
           complex(cfg.mod_inverse).real, complex(cfg.mod_inverse).imag, int(batch), int(bool(multiplication)),
           _stream_handle(cfg.stream))
    check(st, "GPU_FFNT")


def host_fft_tables(n: int, dtype="f64"):
    """FFT<T>(n) tables on the host: (ReverseRootTable, InverseReverseRootTable, n_inverse)
    as numpy arrays (reference fft_cpu.cu:93-128, 200-226)."""
    import numpy as np
    f64 = dtype in ("f64", np.float64)
    C = np.complex128 if f64 else np.complex64
    r, ri = np.zeros(n, C), np.zeros(n, C)
    ninv = np.zeros(1, np.float64 if f64 else np.float32)
    f = lib().gpufft_host_fft_tables_f64 if f64 else lib().gpufft_host_fft_tables_f32
    check(f(n, r.ctypes.data, ri.ctypes.data, ninv.ctypes.data), "host_fft_tables")
    return r, ri, ninv[0]


def host_ffnt_tables(n: int, dtype="f64"):
    """FFNT<T>(n) tables on the host: (ReverseRootTable_ffnt, InverseReverseRootTable_ffnt,
    twist_table_ffnt, untwist_table_ffnt), n/2 entries each (reference fft_cpu.cu:234-300, 435-473)."""
    import numpy as np
    f64 = dtype in ("f64", np.float64)
    C = np.complex128 if f64 else np.complex64
    out = [np.zeros(n // 2, C) for _ in range(4)]
    f = lib().gpufft_host_ffnt_tables_f64 if f64 else lib().gpufft_host_ffnt_tables_f32
    check(f(n, *[o.ctypes.data for o in out]), "host_ffnt_tables")
    return tuple(out)


# ---------------------------------------------------------------------------
# Native fused products (one call per batch of products; no reference
# counterpart as a single call, see include/gpufft_b200.h)
# ---------------------------------------------------------------------------
def ffnt_tables(n_power: int, dtype="f64", device=None, stream=None):
    """Device twiddle block [roots | inverse roots | twist | untwist] for N = 2^n_power,
    generated on the GPU with sincospi."""
    import torch
    L = lib()
    cnt = L.gpufft_ffnt_tables_count(n_power)
    if cnt == 0:
        raise ValueError("Invalid n_power range!")
    f64 = dtype in ("f64", torch.float64, torch.complex128)
    t = torch.empty(cnt, dtype=torch.complex128 if f64 else torch.complex64, device=device or "cuda")
    f = L.gpufft_ffnt_make_tables_f64 if f64 else L.gpufft_ffnt_make_tables_f32
    check(f(n_power, t.data_ptr(), _stream_handle(stream)), "ffnt_tables")
    return t


def negacyclic_mul_workspace_bytes(n_power: int, batch: int, precision_bits: int) -> int:
    return int(lib().gpufft_negacyclic_mul_workspace_bytes(n_power, batch, precision_bits))


def negacyclic_mul(a, b, out=None, tables=None, workspace=None, stream=None):
    """c = a * b mod (X^N + 1) for every row of the (batch, N) float tensors a, b.
    Not rounded, as GPU_FFNT."""
    import torch
    batch, n = a.shape
    n_power = n.bit_length() - 1
    if (1 << n_power) != n or b.shape != a.shape or a.dtype != b.dtype:
        raise GpufftError(ERROR_INVALID_VALUE, "a and b must be (batch, 2^k) tensors of one dtype")
    f64 = a.dtype == torch.float64
    bits = 64 if f64 else 32
    if tables is None:
        tables = ffnt_tables(n_power, "f64" if f64 else "f32", a.device, stream)
    if out is None:
        out = torch.empty_like(a)
    need = negacyclic_mul_workspace_bytes(n_power, batch, bits)
    if workspace is None and need:
        workspace = torch.empty(need, dtype=torch.uint8, device=a.device)
    ws_ptr = workspace.data_ptr() if workspace is not None else None
    ws_len = workspace.numel() * workspace.element_size() if workspace is not None else 0
    L = lib()
    f = L.gpufft_negacyclic_mul_f64 if f64 else L.gpufft_negacyclic_mul_f32
    check(f(_ptr(a), _ptr(b), _ptr(out), n_power, batch, _ptr(tables), ws_ptr, ws_len, _stream_handle(stream)),
          "negacyclic_mul")
    return out


def cyclic_mul(a, b, out=None, tables=None, workspace=None, stream=None):
    """c = a * b mod (X^M - 1) for every row of the (batch, M) complex tensors a, b:
    the C_C product of GPU_FFT forward + inverse-with-multiplication, fused."""
    import torch
    batch, n = a.shape
    n_power = n.bit_length() - 1
    if (1 << n_power) != n or b.shape != a.shape or a.dtype != b.dtype or a.dtype not in (torch.complex64,
                                                                                          torch.complex128):
        raise GpufftError(ERROR_INVALID_VALUE, "a and b must be (batch, 2^k) complex tensors of one dtype")
    f64 = a.dtype == torch.complex128
    if tables is None:
        tables = ffnt_tables(n_power + 1, "f64" if f64 else "f32", a.device, stream)
    if out is None:
        out = torch.empty_like(a)
    L = lib()
    need = int(L.gpufft_cyclic_mul_workspace_bytes(n_power, batch, 64 if f64 else 32))
    if workspace is None and need:
        workspace = torch.empty(need, dtype=torch.uint8, device=a.device)
    ws_ptr = workspace.data_ptr() if workspace is not None else None
    ws_len = workspace.numel() * workspace.element_size() if workspace is not None else 0
    f = L.gpufft_cyclic_mul_f64 if f64 else L.gpufft_cyclic_mul_f32
    check(f(_ptr(a), _ptr(b), _ptr(out), n_power, batch, _ptr(tables), ws_ptr, ws_len, _stream_handle(stream)),
          "cyclic_mul")
    return out


def split_plan(n_power: int, input_bits: int, non_negative: bool = False, precision: str = "f32"):
    """(limb_bits, num_limbs) the library uses for exact split products with
    FP32 ("f32") or FP64 ("f64") transforms."""
    w, k = ctypes.c_int(), ctypes.c_int()
    f = lib().gpufft_split_plan_f64 if precision == "f64" else lib().gpufft_split_plan
    check(f(n_power, input_bits, int(non_negative), ctypes.byref(w), ctypes.byref(k)), "split_plan")
    return w.value, k.value


def negacyclic_mul_split(a, b, out=None, input_bits=None, non_negative=None, limbs=None, tables=None,
                         workspace=None, stream=None, return_error=False, precision="f32"):
    """Exact c = a * b mod (X^N + 1) for (batch, N) int32 tensors, computed with FP32
    (precision="f32", N <= 2^22) or FP64 (precision="f64", N <= 2^17) transforms on
    limbs; returns an int64 tensor (and the max pre-rounding error)."""
    import torch
    batch, n = a.shape
    n_power = n.bit_length() - 1
    if (1 << n_power) != n or b.shape != a.shape or a.dtype != torch.int32 or b.dtype != torch.int32:
        raise GpufftError(ERROR_INVALID_VALUE, "a and b must be (batch, 2^k) int32 tensors")
    if input_bits is None or non_negative is None:
        mx = int(torch.maximum(a.abs().max(), b.abs().max()).item())
        mn = int(torch.minimum(a.min(), b.min()).item())
        input_bits = max(1, mx.bit_length()) if input_bits is None else input_bits
        non_negative = (mn >= 0) if non_negative is None else non_negative
    f64 = precision == "f64"
    w, k = limbs if limbs is not None else split_plan(n_power, input_bits, non_negative, precision)
    if tables is None:
        tables = ffnt_tables(n_power, "f64" if f64 else "f32", a.device, stream)
    if out is None:
        out = torch.empty((batch, n), dtype=torch.int64, device=a.device)
    L = lib()
    wsf = L.gpufft_negacyclic_mul_split_f64_workspace_bytes if f64 else L.gpufft_negacyclic_mul_split_workspace_bytes
    need = int(wsf(n_power, batch, k))
    if workspace is None:
        workspace = torch.empty(max(need, 1), dtype=torch.uint8, device=a.device)
    err = torch.empty(1, dtype=torch.float32, device=a.device)  # zeroed by the call
    fn = L.gpufft_negacyclic_mul_split_f64 if f64 else L.gpufft_negacyclic_mul_split_f32
    st = fn(
        _ptr(a), _ptr(b), _ptr(out), n_power, batch, int(input_bits), int(bool(non_negative)), w, k,
        _ptr(tables), workspace.data_ptr(), workspace.numel() * workspace.element_size(), err.data_ptr(),
        _stream_handle(stream))
    check(st, "negacyclic_mul_split")
    return (out, err) if return_error else out


# ---------------------------------------------------------------------------
# Per-kernel device-time tracing
# ---------------------------------------------------------------------------
def set_f64_middle(r8: int) -> int:
    """FP64 products' middle pass on 512 threads x 8 points (1, the default) or
    256 x 16 (0); identical values. A negative value queries."""
    return int(lib().gpufft_set_f64_middle(int(r8)))


def set_split_tile(on: int) -> int:
    """FP32 split products of rings 2^14..2^16 (up to five limbs) run their
    contiguous stages in the shared-memory tile kernel (1, the default) or in
    the chain of pass and group-sum kernels (0); a negative value queries.
    The integers are the same either way. Returns the previous setting."""
    return int(lib().gpufft_set_split_tile(int(on)))


def split_wait_timeouts(clear: bool = True) -> int:
    """Bounded waits of the split tile kernel that ran out since the last clear
    (each makes its call report an infinite error). Synchronous."""
    n = ctypes.c_uint()
    check(lib().gpufft_split_wait_timeouts(ctypes.byref(n), int(bool(clear))), "split_wait_timeouts")
    return n.value


def set_cluster_tiles(max_tiles: int) -> int:
    """Contiguous 12-stage passes over at most `max_tiles` 4096-point tiles run
    as 8-CTA clusters (small batches); 0 disables, a negative value queries.
    Results are bit-identical either way. Returns the previous limit."""
    return int(lib().gpufft_set_cluster_tiles(int(max_tiles)))


def set_programmatic_launch(on: int) -> int:
    """Chain kernels launched with programmatic stream serialization (1, the
    default) or in plain stream order (0); identical results. A negative value
    queries. Returns the previous setting."""
    return int(lib().gpufft_set_programmatic_launch(int(on)))


def trace_enable(on: bool = True) -> None:
    """Bracket every library kernel launch with CUDA events (off by default)."""
    check(lib().gpufft_trace_enable(int(bool(on))), "trace_enable")


def trace_collect(max_rows: int = 64):
    """Per-kernel totals recorded since the last collect, longest first:
    [{"kernel", "ms", "launches", "alg_bytes"}]. Waits for the recorded events."""
    name_len = 112
    names = ctypes.create_string_buffer(max_rows * name_len)
    ms = (ctypes.c_double * max_rows)()
    by = (ctypes.c_double * max_rows)()
    n = (ctypes.c_longlong * max_rows)()
    rows = ctypes.c_int()
    check(lib().gpufft_trace_collect(max_rows, names, name_len, ms, by, n, ctypes.byref(rows)), "trace_collect")
    out = []
    for k in range(rows.value):
        nm = names.raw[k * name_len:(k + 1) * name_len].split(b"\0", 1)[0].decode()
        out.append({"kernel": nm, "ms": ms[k], "launches": int(n[k]), "alg_bytes": by[k]})
    return sorted(out, key=lambda r: -r["ms"])


def _host_operands(a, b, dtypes, what):
    import torch
    if a.device.type != "cpu" or b.device.type != "cpu":
        raise GpufftError(ERROR_INVALID_VALUE, f"{what}: a and b must be host tensors")
    if a.dim() != 2 or b.shape != a.shape or a.dtype not in dtypes or b.dtype != a.dtype:
        raise GpufftError(ERROR_INVALID_VALUE, f"{what}: a and b must be (batch, 2^k) tensors of one supported dtype")
    if not (a.is_contiguous() and b.is_contiguous()):
        raise GpufftError(ERROR_INVALID_VALUE, f"{what}: a and b must be contiguous")
    batch, n = a.shape
    n_power = n.bit_length() - 1
    if (1 << n_power) != n:
        raise GpufftError(ERROR_INVALID_VALUE, f"{what}: rows must have 2^k entries")
    return batch, n, n_power


def negacyclic_mul_host(a, b, out=None, tables=None, workspace=None, chunk=0, device=None, stream=None):
    """negacyclic_mul on HOST tensors (pin them for overlap): chunks are copied in,
    multiplied and copied out with the transfers overlapping the computation.
    Asynchronous on `stream` like the device call; synchronise before reading out."""
    import torch
    batch, n, n_power = _host_operands(a, b, (torch.float32, torch.float64), "negacyclic_mul_host")
    f64 = a.dtype == torch.float64
    dev = torch.device(device) if device is not None else (tables.device if tables is not None else
                                                            torch.device("cuda", torch.cuda.current_device()))
    if tables is None:
        tables = ffnt_tables(n_power, "f64" if f64 else "f32", dev, stream)
    if out is None:
        out = torch.empty((batch, n), dtype=a.dtype, pin_memory=True)
    L = lib()
    need = int(L.gpufft_negacyclic_mul_host_workspace_bytes(n_power, batch, int(chunk), 64 if f64 else 32))
    if need == 0:
        raise ValueError("Invalid n_power range!")
    if workspace is None:
        workspace = torch.empty(need, dtype=torch.uint8, device=dev)
    f = L.gpufft_negacyclic_mul_f64_host if f64 else L.gpufft_negacyclic_mul_f32_host
    check(f(a.data_ptr(), b.data_ptr(), out.data_ptr(), n_power, batch, int(chunk), _ptr(tables),
            workspace.data_ptr(), workspace.numel() * workspace.element_size(), _stream_handle(stream)),
          "negacyclic_mul_host")
    return out


def negacyclic_mul_split_host(a, b, out=None, input_bits=24, non_negative=False, limbs=None, tables=None,
                              workspace=None, chunk=0, device=None, stream=None, return_error=False):
    """negacyclic_mul_split on HOST int32 tensors (pin them for overlap), chunked with
    the transfers overlapping the computation; int64 host result. Asynchronous on
    `stream`; synchronise before reading out (or the error)."""
    import torch
    batch, n, n_power = _host_operands(a, b, (torch.int32,), "negacyclic_mul_split_host")
    dev = torch.device(device) if device is not None else (tables.device if tables is not None else
                                                            torch.device("cuda", torch.cuda.current_device()))
    w, k = limbs if limbs is not None else split_plan(n_power, input_bits, non_negative)
    if tables is None:
        tables = ffnt_tables(n_power, "f32", dev, stream)
    if out is None:
        out = torch.empty((batch, n), dtype=torch.int64, pin_memory=True)
    L = lib()
    need = int(L.gpufft_negacyclic_mul_split_f32_host_workspace_bytes(n_power, batch, int(chunk), k))
    if need == 0:
        raise ValueError("Invalid n_power range!")
    if workspace is None:
        workspace = torch.empty(need, dtype=torch.uint8, device=dev)
    err = torch.empty(1, dtype=torch.float32, device=dev)  # zeroed by the call
    check(L.gpufft_negacyclic_mul_split_f32_host(
        a.data_ptr(), b.data_ptr(), out.data_ptr(), n_power, batch, int(chunk), int(input_bits),
        int(bool(non_negative)), w, k, _ptr(tables), workspace.data_ptr(),
        workspace.numel() * workspace.element_size(), err.data_ptr(), _stream_handle(stream)),
        "negacyclic_mul_split_host")
    return (out, err) if return_error else out


def linear_mul(a, b, out=None, tables=None, workspace=None, stream=None):
    """Linear product of the rows of (batch, N) float tensors: (batch, 2N) result
    (the R_R product, computed with half-length transforms). Not rounded."""
    import torch
    batch, n = a.shape
    n_power = n.bit_length() - 1
    if (1 << n_power) != n or b.shape != a.shape or a.dtype != b.dtype:
        raise GpufftError(ERROR_INVALID_VALUE, "a and b must be (batch, 2^k) tensors of one dtype")
    f64 = a.dtype == torch.float64
    if tables is None:
        tables = ffnt_tables(n_power + 1, "f64" if f64 else "f32", a.device, stream)
    if out is None:
        out = torch.empty((batch, 2 * n), dtype=a.dtype, device=a.device)
    need = int(lib().gpufft_linear_mul_workspace_bytes(n_power, batch, 64 if f64 else 32))
    if workspace is None and need:
        workspace = torch.empty(need, dtype=torch.uint8, device=a.device)
    ws_ptr = workspace.data_ptr() if workspace is not None else None
    ws_len = workspace.numel() * workspace.element_size() if workspace is not None else 0
    f = lib().gpufft_linear_mul_f64 if f64 else lib().gpufft_linear_mul_f32
    check(f(_ptr(a), _ptr(b), _ptr(out), n_power, batch, _ptr(tables), ws_ptr, ws_len, _stream_handle(stream)),
          "linear_mul")
    return out


def linear_mul_vjp(g, a, b, grad_a=None, grad_b=None, tables=None, workspace=None, stream=None):
    """Adjoint of linear_mul (float32): for the upstream gradient g (batch, 2N),
    returns (grad_a, grad_b), each (batch, N)."""
    import torch
    batch, n = a.shape
    n_power = n.bit_length() - 1
    if tables is None:
        tables = ffnt_tables(n_power + 1, "f32", a.device, stream)
    if grad_a is None:
        grad_a = torch.empty_like(a)
    if grad_b is None:
        grad_b = torch.empty_like(b)
    need = int(lib().gpufft_linear_mul_vjp_workspace_bytes(n_power, batch))
    if workspace is None and need:
        workspace = torch.empty(need, dtype=torch.uint8, device=a.device)
    ws_ptr = workspace.data_ptr() if workspace is not None else None
    ws_len = workspace.numel() * workspace.element_size() if workspace is not None else 0
    check(lib().gpufft_linear_mul_vjp_f32(_ptr(g), _ptr(a), _ptr(b), _ptr(grad_a), _ptr(grad_b), n_power, batch,
                                          _ptr(tables), ws_ptr, ws_len, _stream_handle(stream)), "linear_mul_vjp")
    return grad_a, grad_b


class BatchPlan:
    """Negacyclic products of mixed ring sizes in one persistent launch.

    plan = BatchPlan(n_powers, torch.float64)
    a_packed = plan.pack([a_0, a_1, ...])          # requests grouped by size
    c_packed = plan.execute(a_packed, b_packed)   # or capture() once, replay() after
    c_list = plan.unpack(c_packed)
    """

    def __init__(self, n_powers, dtype, stream=None):
        import numpy as np
        import torch
        self.n_powers = [int(x) for x in n_powers]
        self.dtype = dtype
        self.bits = 64 if dtype == torch.float64 else 32
        arr = (ctypes.c_int * len(self.n_powers))(*self.n_powers)
        h = ctypes.c_void_p()
        check(lib().gpufft_batch_plan_create(ctypes.byref(h), arr, len(self.n_powers), self.bits,
                                             _stream_handle(stream)), "batch_plan_create")
        self.h = h
        n = len(self.n_powers)
        order = (ctypes.c_int * n)()
        offs = (ctypes.c_longlong * n)()
        total = ctypes.c_longlong()
        check(lib().gpufft_batch_plan_layout(self.h, order, offs, ctypes.byref(total)), "batch_plan_layout")
        self.order = np.array(order[:], dtype=np.int64)
        self.offsets = np.array(offs[:], dtype=np.int64)
        self.total = int(total.value)

    def pack(self, polys):
        """Concatenate per-request rows (length 2^n_powers[i]) in the plan's layout."""
        import torch
        out = torch.empty(self.total, dtype=self.dtype, device=polys[0].device)
        for i, p in enumerate(polys):
            o = int(self.offsets[i])
            out[o: o + p.numel()].copy_(p.reshape(-1))
        return out

    def unpack(self, packed):
        return [packed[int(o): int(o) + (1 << n)] for o, n in zip(self.offsets, self.n_powers)]

    def execute(self, a, b, out=None, stream=None):
        import torch
        if out is None:
            out = torch.empty_like(a)
        check(lib().gpufft_batch_plan_execute(self.h, _ptr(a), _ptr(b), _ptr(out), _stream_handle(stream)),
              "batch_plan_execute")
        return out

    def set_barrier(self, max_polls=1 << 26, extra_arrivals=0):
        """Poll limit of the persistent launch's grid barriers; extra_arrivals > 0
        makes every barrier run out (tests of the timeout path only)."""
        check(lib().gpufft_batch_plan_set_barrier(self.h, int(max_polls), int(extra_arrivals)),
              "batch_plan_set_barrier")

    def autotune(self, a, b, out, cache_path=None, stream=None):
        cp = cache_path.encode() if cache_path else None
        check(lib().gpufft_batch_plan_autotune(self.h, _ptr(a), _ptr(b), _ptr(out), cp, _stream_handle(stream)),
              "batch_plan_autotune")
        return self.info()

    def capture(self, a, b, out, stream):
        check(lib().gpufft_batch_plan_capture(self.h, _ptr(a), _ptr(b), _ptr(out), _stream_handle(stream)),
              "batch_plan_capture")

    def replay(self, stream):
        check(lib().gpufft_batch_plan_replay(self.h, _stream_handle(stream)), "batch_plan_replay")

    def set_shape(self, ctas_per_sm, items_per_grab=1):
        """Persistent launch (ctas_per_sm 1 or 2) or per-class chains (0)."""
        check(lib().gpufft_batch_plan_set_shape(self.h, int(ctas_per_sm), int(items_per_grab)), "batch_plan_set_shape")

    def info(self):
        m, g, gr, ws = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        check(lib().gpufft_batch_plan_info(self.h, ctypes.byref(m), ctypes.byref(g), ctypes.byref(gr),
                                           ctypes.byref(ws)), "batch_plan_info")
        return {"mode": "persistent" if m.value else "per-class chains", "ctas_per_sm": m.value,
                "items_per_grab": g.value, "grid": gr.value, "workspace_bytes": ws.value}

    def status(self):
        f = ctypes.c_int()
        check(lib().gpufft_batch_plan_status(self.h, ctypes.byref(f)), "batch_plan_status")
        return f.value

    def close(self):
        if getattr(self, "h", None):
            lib().gpufft_batch_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SplitBatchPlan:
    """Exact (FP32 split) negacyclic products of mixed ring sizes.

    plan = SplitBatchPlan(n_powers, input_bits=16)
    a_packed = plan.pack([a_0, a_1, ...])            # int32 rows, grouped by size
    c_packed, err = plan.execute(a_packed, b_packed)   # int64; or capture() once, replay() after
    c_list = plan.unpack(c_packed)
    """

    def __init__(self, n_powers, input_bits, non_negative=False, stream=None):
        import numpy as np
        self.n_powers = [int(x) for x in n_powers]
        n = len(self.n_powers)
        arr = (ctypes.c_int * n)(*self.n_powers)
        h = ctypes.c_void_p()
        check(lib().gpufft_split_batch_plan_create(ctypes.byref(h), arr, n, int(input_bits), int(bool(non_negative)),
                                                   _stream_handle(stream)), "split_batch_plan_create")
        self.h = h
        offs = (ctypes.c_longlong * n)()
        total = ctypes.c_longlong()
        wb, kb = (ctypes.c_int * n)(), (ctypes.c_int * n)()
        check(lib().gpufft_split_batch_plan_layout(self.h, offs, ctypes.byref(total), wb, kb),
              "split_batch_plan_layout")
        self.offsets = np.array(offs[:], dtype=np.int64)
        self.total = int(total.value)
        self.limbs = list(zip(wb[:], kb[:]))

    def pack(self, polys):
        import torch
        out = torch.empty(self.total, dtype=torch.int32, device=polys[0].device)
        for i, p in enumerate(polys):
            o = int(self.offsets[i])
            out[o: o + p.numel()].copy_(p.reshape(-1))
        return out

    def unpack(self, packed):
        return [packed[int(o): int(o) + (1 << n)] for o, n in zip(self.offsets, self.n_powers)]

    def execute(self, a, b, out=None, err=None, stream=None):
        import torch
        if out is None:
            out = torch.empty(self.total, dtype=torch.int64, device=a.device)
        if err is None:
            err = torch.empty(1, dtype=torch.float32, device=a.device)  # zeroed by the call
        check(lib().gpufft_split_batch_plan_execute(self.h, _ptr(a), _ptr(b), _ptr(out), _ptr(err),
                                                    _stream_handle(stream)), "split_batch_plan_execute")
        return out, err

    def capture(self, a, b, out, err, stream):
        check(lib().gpufft_split_batch_plan_capture(self.h, _ptr(a), _ptr(b), _ptr(out), _ptr(err),
                                                    _stream_handle(stream)), "split_batch_plan_capture")

    def replay(self, stream):
        check(lib().gpufft_split_batch_plan_replay(self.h, _stream_handle(stream)), "split_batch_plan_replay")

    def close(self):
        if getattr(self, "h", None):
            lib().gpufft_split_batch_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

