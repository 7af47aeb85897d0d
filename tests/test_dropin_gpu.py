"""GPU parity tests for the drop-in GPU_FFT (C_C, R_R) and GPU_FFNT entry
points: every case runs through the C ABI on cuda:0 and is compared with the
oracle's restatement of the reference's device math on the same inputs and
tables.

Tolerances: float outputs are compared by relative L2 error against the oracle
(double: 1e-12, float: 2e-5; the kernels use the reference's butterflies with
FMA contraction, the oracle does not contract); integer products are compared
bit-exactly with the exact schoolbook product after rounding.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = {np.float64: 1e-12, np.float32: 2e-5}


def cdt(T):
    return np.complex128 if T == np.float64 else np.complex64


def rel_l2(got, want):
    got = np.asarray(got, np.complex128).ravel()
    want = np.asarray(want, np.complex128).ravel()
    return np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300)


def td(x, dev):
    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


def fft_table(O, n_power, T, neg=False, inverse=False):
    # cyclic: FFT<T>(M/2) tables (M/2 entries); negacyclic: FFT<T>(M) (M entries)
    sfx = "f64" if T == np.float64 else "f32"
    n = (1 << n_power) if neg else (1 << (n_power - 1))
    r, ri, ninv = O.fft_tables(n, sfx)
    return (ri if inverse else r), ninv


C2C_SIZES = [1, 2, 3, 5, 8, 10, 11, 12, 13, 14, 15, 16, 17, 20, 22]


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("n_power", C2C_SIZES)
def test_c2c_forward_and_inverse_mult(gf, O, dev, T, n_power):
    rng = np.random.default_rng(n_power)
    M = 1 << n_power
    batch = 3 if n_power <= 17 else 1
    C = cdt(T)
    x = (rng.standard_normal((2 * batch, M)) + 1j * rng.standard_normal((2 * batch, M))).astype(C)
    roots, _ = fft_table(O, n_power, T)
    inv_roots, _ = fft_table(O, n_power, T, inverse=True)
    d_roots, d_inv = td(roots, dev), td(inv_roots, dev)
    buf = td(x.ravel(), dev)
    L = gf.lib()
    f = L.gpufft_fft_c2c_f64 if T == np.float64 else L.gpufft_fft_c2c_f32
    gf.check(f(buf.data_ptr(), d_roots.data_ptr(), n_power, 0, 1, 0, 1.0, 0.0, 2 * batch, 0, None), "fwd")
    want = O.gpu_fft_c2c(x.ravel(), roots, n_power, 0, 1, 1.0, 2 * batch, False)
    got = buf.cpu().numpy()
    assert rel_l2(got, want) < TOL[T]
    mi = 1.0 / M
    gf.check(f(buf.data_ptr(), d_inv.data_ptr(), n_power, 1, 1, 0, mi, 0.0, batch, 1, None), "inv")
    want2 = O.gpu_fft_c2c(want, inv_roots, n_power, 1, 1, mi, batch, True)
    got2 = buf.cpu().numpy()
    assert rel_l2(got2[: batch * M], want2[: batch * M]) < TOL[T]
    # the second operand is untouched, as in the reference
    assert np.array_equal(got2[batch * M:], got[batch * M:])


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("n_power", [4, 12, 14, 19])
def test_c2c_negacyclic_table_mode(gf, O, dev, T, n_power):
    # reduction_poly = X_N_plus: twiddle index 2^s + g into an M-entry table (fft.cu:67-74)
    rng = np.random.default_rng(100 + n_power)
    M = 1 << n_power
    C = cdt(T)
    x = (rng.standard_normal((2, M)) + 1j * rng.standard_normal((2, M))).astype(C)
    roots, _ = fft_table(O, n_power, T, neg=True)
    buf = td(x.ravel(), dev)
    L = gf.lib()
    f = L.gpufft_fft_c2c_f64 if T == np.float64 else L.gpufft_fft_c2c_f32
    d_roots = td(roots, dev)
    gf.check(f(buf.data_ptr(), d_roots.data_ptr(), n_power, 0, 0, 0, 1.0, 0.0, 2, 0, None), "fwd")
    want = O.gpu_fft_c2c(x.ravel(), roots, n_power, 0, 0, 1.0, 2, False)
    assert rel_l2(buf.cpu().numpy(), want) < TOL[T]
    inv_roots, _ = fft_table(O, n_power, T, neg=True, inverse=True)
    d_inv = td(inv_roots, dev)
    gf.check(f(buf.data_ptr(), d_inv.data_ptr(), n_power, 1, 0, 0, 0.5, 0.25, 1, 1, None), "inv")
    want2 = O.gpu_fft_c2c(want, inv_roots, n_power, 1, 0, 0.5 + 0.25j, 1, True)
    assert rel_l2(buf.cpu().numpy()[:M], want2[:M]) < TOL[T]


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("n_power", [6, 12, 13, 16, 18])
@pytest.mark.parametrize("zero_padding", [False, True])
def test_r2r_linear_product(gf, O, dev, T, n_power, zero_padding):
    rng = np.random.default_rng(200 + n_power)
    M = 1 << n_power
    n = M // 2
    batch = 2
    real = np.zeros((2 * batch, M), T)
    real[:, :n] = rng.integers(-64, 64, (2 * batch, n))
    roots, _ = fft_table(O, n_power, T)
    inv_roots, ninv = fft_table(O, n_power, T, inverse=True)
    rbuf = td(real.ravel(), dev)
    temp = torch.zeros(2 * batch * M, dtype=torch.complex128 if T == np.float64 else torch.complex64, device=dev)
    L = gf.lib()
    f = L.gpufft_fft_r2r_f64 if T == np.float64 else L.gpufft_fft_r2r_f32
    d_roots, d_inv = td(roots, dev), td(inv_roots, dev)
    gf.check(f(rbuf.data_ptr(), temp.data_ptr(), d_roots.data_ptr(), n_power, 0, 1, int(zero_padding),
               1.0, 0.0, 2 * batch, 0, None), "fwd")
    r1, t1 = O.gpu_fft_r2r(real.ravel(), np.zeros(2 * batch * M, cdt(T)), roots, n_power, 0, 1, 1.0, 2 * batch,
                           False)
    assert rel_l2(temp.cpu().numpy(), t1) < TOL[T]
    gf.check(f(rbuf.data_ptr(), temp.data_ptr(), d_inv.data_ptr(), n_power, 1, 1, 0, float(ninv),
               0.0, batch, 1, None), "inv")
    r2, _ = O.gpu_fft_r2r(r1, t1, inv_roots, n_power, 1, 1, float(ninv), batch, True)
    got = rbuf.cpu().numpy()
    assert rel_l2(got[: batch * M], r2[: batch * M]) < TOL[T]
    if T == np.float32 and n_power > 13:
        return  # |c| reaches 2^29: beyond float's exact integers
    for k in range(batch):
        exact = O.wrap64(O.schoolbook(real[k, :n].astype(np.int64), real[batch + k, :n].astype(np.int64),
                                      O.LINEAR))
        assert np.array_equal(np.rint(got[k * M:(k + 1) * M]).astype(np.int64), exact)


def test_cpu_example_linear_product_bit_exact_vs_reference(gf, O, dev):
    # the CPU-example product: R_R, N = 2^12, batch 1, FP64, coefficients in [-2^15, 2^15)
    g = np.load(os.path.join(GOLD, "linear_f64.npz"))
    n = int(g["n"])
    M = 2 * n
    real = np.zeros((2, M))
    real[0, :n] = g["a"]
    real[1, :n] = g["b"]
    roots, inv_roots, ninv = O.fft_tables(n, "f64")
    rbuf = td(real.ravel(), dev)
    temp = torch.zeros(2 * M, dtype=torch.complex128, device=dev)
    cfg = gf.fft_configuration(n_power=13, fft_type=gf.FORWARD, reduction_poly=gf.X_N_minus)
    gf.GPU_FFT(rbuf, temp, td(roots, dev), cfg, 2, False)
    cfg_i = gf.fft_configuration(n_power=13, fft_type=gf.INVERSE, reduction_poly=gf.X_N_minus,
                                 mod_inverse=complex(ninv))
    gf.GPU_FFT(rbuf, temp, td(inv_roots, dev), cfg_i, 1, True)
    got = np.rint(rbuf.cpu().numpy()[:M]).astype(np.int64)
    assert np.array_equal(got, g["out"])  # the reference's own CPU output
    assert np.array_equal(got, O.wrap64(O.schoolbook(g["a"], g["b"], O.LINEAR)))


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("n_power", [2, 3, 6, 12, 13, 14, 16, 17, 22])
def test_ffnt_product(gf, O, dev, T, n_power):
    rng = np.random.default_rng(300 + n_power)
    n = 1 << n_power
    h = n // 2
    batch = 3 if n_power <= 17 else 1
    bits = 10 if T == np.float64 else 4
    ab = rng.integers(0, 1 << bits, (2 * batch, n)).astype(T)
    sfx = "f64" if T == np.float64 else "f32"
    roots, inv_roots, twist, untwist = O.ffnt_tables(n, sfx)
    buf = td(ab.ravel(), dev)
    temp = torch.zeros(2 * batch * h, dtype=torch.complex128 if T == np.float64 else torch.complex64, device=dev)
    # keep every device table alive for the duration of the calls
    d_roots, d_inv, d_tw, d_utw = (td(x, dev) for x in (roots, inv_roots, twist, untwist))
    L = gf.lib()
    f = L.gpufft_ffnt_f64 if T == np.float64 else L.gpufft_ffnt_f32
    gf.check(f(buf.data_ptr(), temp.data_ptr(), d_tw.data_ptr(), d_roots.data_ptr(), n_power, 0,
               1.0, 0.0, 2 * batch, 0, None), "fwd")
    r1, t1 = O.gpu_ffnt(ab.ravel(), np.zeros(2 * batch * h, cdt(T)), twist, roots, n_power, 0, 1.0, 2 * batch,
                        False)
    assert rel_l2(temp.cpu().numpy(), t1) < TOL[T]
    mi = 1.0 / h
    gf.check(f(buf.data_ptr(), temp.data_ptr(), d_utw.data_ptr(), d_inv.data_ptr(),
               n_power, 1, mi, 0.0, batch, 1, None), "inv")
    r2, _ = O.gpu_ffnt(r1, t1, untwist, inv_roots, n_power, 1, mi, batch, True)
    got = buf.cpu().numpy()
    assert rel_l2(got[: batch * n], r2[: batch * n]) < TOL[T]
    if n_power <= (16 if T == np.float64 else 10):
        for k in range(batch):
            exact = O.wrap64(O.schoolbook(ab[k].astype(np.int64), ab[batch + k].astype(np.int64)))
            assert np.array_equal(np.rint(got[k * n:(k + 1) * n]).astype(np.int64), exact)


def test_ffnt_reference_example_semantics(gf, O, dev):
    # example/test_ffnt_gpu_R_R.cu: coefficients in [0, 6], q = 7, logn = 12, batch 1,
    # results reduced mod 7 after rounding to unsigned long long.
    rng = np.random.default_rng(11)
    n = 1 << 12
    a = rng.integers(0, 7, n).astype(np.uint64)
    b = rng.integers(0, 7, n).astype(np.uint64)
    roots, inv_roots, twist, untwist = O.ffnt_tables(n, "f64")
    buf = td(np.concatenate([a, b]).astype(np.float64), dev)
    temp = torch.zeros(n, dtype=torch.complex128, device=dev)
    gf.GPU_FFNT(buf, temp, td(twist, dev), td(roots, dev), gf.fft_configuration(n_power=12, fft_type=gf.FORWARD),
                2, False)
    cfg_i = gf.fft_configuration(n_power=12, fft_type=gf.INVERSE, mod_inverse=complex(1.0 / (n >> 1)))
    gf.GPU_FFNT(buf, temp, td(untwist, dev), td(inv_roots, dev), cfg_i, 1, True)
    got = np.rint(buf.cpu().numpy()[:n]).astype(np.int64).view(np.uint64) % np.uint64(7)
    R = O.ref()
    want = np.zeros(n, np.uint64)
    if R is not None:
        R.ref_schoolbook_negacyclic_u64(a, b, 7, n, want)
    else:
        want = np.array([(int(v) & ((1 << 64) - 1)) % 7 for v in O.schoolbook(a.astype(np.int64),
                                                                              b.astype(np.int64))], np.uint64)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n_power", [12, 24])
def test_reference_range_ends(gf, O, dev, n_power):
    # the reference accepts exactly 12 <= n_power <= 24 (fft.cu:522-525)
    M = 1 << n_power
    x = (np.random.default_rng(n_power).standard_normal(M) + 0j).astype(np.complex64)
    roots, _ = fft_table(O, n_power, np.float32)
    buf = td(x, dev)
    gf.GPU_FFT(buf, td(roots, dev), gf.fft_configuration(n_power=n_power), 1, False)
    want = O.gpu_fft_c2c(x, roots, n_power, 0, 1, 1.0, 1, False)
    assert rel_l2(buf.cpu().numpy(), want) < 1e-4
    with pytest.raises(ValueError, match="Invalid n_power range!"):
        gf.GPU_FFT(buf, td(roots, dev), gf.fft_configuration(n_power=n_power + (1 if n_power == 24 else -1)), 1,
                   False)


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("n_power", [10, 12, 14, 16])
def test_c2c_cyclic_product_gib_batch(gf, O, dev, T, n_power):
    # the C_C product workload: re/im i.i.d. N(0,1), batch sized to ~1 GiB of
    # input; forward of 2 batch, inverse with the product; sampled products
    # against an FP64 cyclic convolution (numpy FFT)
    M = 1 << n_power
    C = cdt(T)
    csz = np.dtype(C).itemsize
    batch = (1 << 30) // (2 * M * csz)
    g = torch.Generator(device="cpu").manual_seed(2000 + n_power)
    tdt = torch.complex128 if T == np.float64 else torch.complex64
    x = torch.randn(2 * batch * M, dtype=tdt, generator=g)
    buf = x.to(dev)
    roots, _ = fft_table(O, n_power, T)
    inv_roots, _ = fft_table(O, n_power, T, inverse=True)
    d_roots, d_inv = td(roots, dev), td(inv_roots, dev)
    L = gf.lib()
    f = L.gpufft_fft_c2c_f64 if T == np.float64 else L.gpufft_fft_c2c_f32
    gf.check(f(buf.data_ptr(), d_roots.data_ptr(), n_power, 0, 1, 0, 1.0, 0.0, 2 * batch, 0, None), "fwd")
    gf.check(f(buf.data_ptr(), d_inv.data_ptr(), n_power, 1, 1, 0, 1.0 / M, 0.0, batch, 1, None), "inv")
    for k in (0, batch // 2, batch - 1):
        a = x[k * M:(k + 1) * M].numpy().astype(np.complex128)
        b = x[(batch + k) * M:(batch + k + 1) * M].numpy().astype(np.complex128)
        want = np.fft.ifft(np.fft.fft(a) * np.fft.fft(b))
        got = buf[k * M:(k + 1) * M].cpu().numpy()
        assert rel_l2(got, want) < (1e-13 if T == np.float64 else 2e-6) * n_power

