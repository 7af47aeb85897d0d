"""GPU parity tests for the native fused negacyclic product (C ABI
gpufft_negacyclic_mul_*): integer products are bit-exact against the exact
schoolbook product after rounding; float products agree with the oracle's
restatement of the reference FFNT chain within relative L2 1e-12 (double) and
2e-5 (float)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def exact_rows(O, a, b):
    return np.stack([O.wrap64(O.schoolbook(a[k].astype(np.int64), b[k].astype(np.int64))) for k in range(a.shape[0])])


@pytest.mark.parametrize("T", ["f64", "f32"])
@pytest.mark.parametrize("n_power", [2, 4, 12, 13, 14, 17, 22])
def test_device_tables_match_reference_values(gf, O, dev, T, n_power):
    t = gf.ffnt_tables(n_power, T, dev).cpu().numpy()
    n = 1 << n_power
    M = n // 2
    r, ri, tw, utw = O.ffnt_tables(n, "f64")  # reference table values (computed in double)
    tol = 1e-15 if T == "f64" else 1e-7
    np.testing.assert_allclose(t[: M // 2], r[: M // 2], rtol=0, atol=tol)
    np.testing.assert_allclose(t[M // 2: M], ri[: M // 2], rtol=0, atol=tol)
    np.testing.assert_allclose(t[M: 2 * M], tw, rtol=0, atol=tol)
    np.testing.assert_allclose(t[2 * M: 3 * M], utw, rtol=0, atol=tol)
    # U: transform of the all-ones polynomial in output (bit-reversed) order
    br = np.array([O.lib().orc_bitreverse(i, n_power - 1) for i in range(M)]) if M > 1 else np.zeros(1, int)
    x = (1 + 1j) * np.exp(1j * np.pi * np.arange(M) / n)
    want_u = (M * np.fft.ifft(x))[br]
    if M > 4096:
        # stored in the split product's spectrum order: each 4096-block permuted e -> (e >> 4) + 256 (e & 15)
        i = np.arange(M)
        pos = (i & ~4095) | ((i & 4095) >> 4) | ((i & 15) << 8)
        perm_u = np.empty_like(want_u)
        perm_u[pos] = want_u
        want_u = perm_u
    # (numpy's own FFT of length M carries ~1e-16 * M absolute error)
    scale = np.max(np.abs(want_u))
    np.testing.assert_allclose(t[3 * M:], want_u, rtol=1e-6 if T == "f32" else 1e-11,
                               atol=(1e-6 if T == "f32" else 1e-13) * scale)


@pytest.mark.parametrize("n_power,batch", [(2, 5), (3, 3), (10, 9), (12, 3), (13, 5), (14, 2), (15, 3), (16, 3),
                                           (17, 2)])
def test_f64_product_bit_exact(gf, O, dev, n_power, batch):
    rng = np.random.default_rng(1000 + n_power)
    n = 1 << n_power
    a = rng.integers(-(1 << 15), 1 << 15, (batch, n))
    b = rng.integers(-(1 << 15), 1 << 15, (batch, n))
    c = gf.negacyclic_mul(torch.from_numpy(a.astype(np.float64)).to(dev), torch.from_numpy(b.astype(np.float64)).to(dev))
    got = np.rint(c.cpu().numpy()).astype(np.int64)
    assert np.array_equal(got, exact_rows(O, a, b))


def test_f64_output_aliases_input_and_small_workspace(gf, O, dev):
    rng = np.random.default_rng(5)
    n_power, batch = 15, 7
    n = 1 << n_power
    a = rng.integers(0, 1 << 12, (batch, n))
    b = rng.integers(0, 1 << 12, (batch, n))
    ta = torch.from_numpy(a.astype(np.float64)).to(dev)
    tb = torch.from_numpy(b.astype(np.float64)).to(dev)
    per = 2 * (n // 2) * 16
    ws = torch.empty(2 * per + 100, dtype=torch.uint8, device=dev)  # room for 2 products per wave
    gf.negacyclic_mul(ta, tb, out=ta, workspace=ws)
    assert np.array_equal(np.rint(ta.cpu().numpy()).astype(np.int64), exact_rows(O, a, b))
    with pytest.raises(gf.GpufftError):
        gf.negacyclic_mul(tb, tb, workspace=torch.empty(per - 16, dtype=torch.uint8, device=dev))


@pytest.mark.parametrize("n_power", [6, 12, 14, 16])
def test_f32_product_vs_oracle(gf, O, dev, n_power):
    rng = np.random.default_rng(2000 + n_power)
    n = 1 << n_power
    batch = 3
    a = rng.integers(0, 16, (batch, n)).astype(np.float32)
    b = rng.integers(0, 16, (batch, n)).astype(np.float32)
    c = gf.negacyclic_mul(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)).cpu().numpy()
    ex = exact_rows(O, a, b).astype(np.float64)
    rel = np.linalg.norm(c - ex) / np.linalg.norm(ex)
    assert rel < 2e-5
    if n_power <= 12:
        assert np.array_equal(np.rint(c).astype(np.int64), ex.astype(np.int64))


def test_f64_linearity_full_size(gf, dev):
    # size-independent property at the benchmark size (N = 2^16, batch 256):
    # (a1 + a2) * b == a1 * b + a2 * b within floating-point tolerance
    g = torch.Generator(device=dev).manual_seed(3)
    n, batch = 1 << 16, 256
    a1 = torch.randint(0, 1 << 10, (batch, n), device=dev, generator=g).double()
    a2 = torch.randint(0, 1 << 10, (batch, n), device=dev, generator=g).double()
    b = torch.randint(0, 1 << 10, (batch, n), device=dev, generator=g).double()
    lhs = gf.negacyclic_mul(a1 + a2, b)
    rhs = gf.negacyclic_mul(a1, b) + gf.negacyclic_mul(a2, b)
    assert torch.equal(torch.round(lhs), torch.round(rhs))


@pytest.mark.parametrize("n_power,batch,dtype", [
    (1, 5, torch.complex128), (4, 9, torch.complex64), (10, 7, torch.complex128), (12, 3, torch.complex64),
    (13, 3, torch.complex128), (16, 5, torch.complex64), (16, 4, torch.complex128), (18, 2, torch.complex128)])
def test_cyclic_product_vs_fp64_convolution(gf, dev, n_power, batch, dtype):
    # the native C_C product against an FP64 cyclic convolution (numpy FFT)
    g = torch.Generator(device="cpu").manual_seed(300 + n_power)
    M = 1 << n_power
    a = torch.randn(batch, M, dtype=dtype, generator=g)
    b = torch.randn(batch, M, dtype=dtype, generator=g)
    got = gf.cyclic_mul(a.to(dev), b.to(dev)).cpu().numpy().astype(np.complex128)
    A, B = a.numpy().astype(np.complex128), b.numpy().astype(np.complex128)
    want = np.fft.ifft(np.fft.fft(A, axis=1) * np.fft.fft(B, axis=1), axis=1)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < (1e-14 if dtype == torch.complex128 else 2e-6) * max(n_power, 1), err


def test_cyclic_product_matches_dropin(gf, O, dev):
    # identical arithmetic to the reference API's two GPU_FFT calls on the
    # same tables (FFT<T>(M/2) values): equal within rounding
    n_power, batch = 14, 6
    M = 1 << n_power
    g = torch.Generator(device="cpu").manual_seed(5)
    a = torch.randn(batch, M, dtype=torch.complex128, generator=g)
    b = torch.randn(batch, M, dtype=torch.complex128, generator=g)
    got = gf.cyclic_mul(a.to(dev), b.to(dev)).cpu()
    roots, inv_roots, _ = gf.host_fft_tables(M // 2, "f64")
    buf = torch.cat([a.reshape(-1), b.reshape(-1)]).to(dev)
    L = gf.lib()
    d_r = torch.from_numpy(np.ascontiguousarray(roots)).to(dev)
    d_i = torch.from_numpy(np.ascontiguousarray(inv_roots)).to(dev)
    gf.check(L.gpufft_fft_c2c_f64(buf.data_ptr(), d_r.data_ptr(), n_power, 0, 1, 0, 1.0, 0.0, 2 * batch, 0, None), "f")
    gf.check(L.gpufft_fft_c2c_f64(buf.data_ptr(), d_i.data_ptr(), n_power, 1, 1, 0, 1.0 / M, 0.0, batch, 1, None), "i")
    ref = buf[: batch * M].cpu().view(batch, M)
    assert (torch.linalg.norm(got - ref) / torch.linalg.norm(ref)).item() < 1e-14


@pytest.mark.parametrize("n_power,batch", [(14, 40), (16, 33), (17, 20), (20, 3)])
def test_f64_middle_forms_identical(gf, O, dev, n_power, batch):
    # the FP64 middle pass on 512 x 8 points (radix-8 rounds) and on 256 x 16
    # (the engine's radix-16 rounds) runs the same butterflies: identical bits,
    # for the negacyclic and the cyclic products; exact on sampled coefficients
    rng = np.random.default_rng(880 + n_power)
    n = 1 << n_power
    a = torch.from_numpy(rng.integers(-(1 << 15), 1 << 15, (batch, n)).astype(np.float64)).to(dev)
    b = torch.from_numpy(rng.integers(-(1 << 15), 1 << 15, (batch, n)).astype(np.float64)).to(dev)
    prev = gf.set_f64_middle(1)
    try:
        gf.set_cluster_tiles(0)  # the tiled middle pass, not its cluster form
        c1 = gf.negacyclic_mul(a, b)
        x = torch.complex(a, b)
        y = torch.complex(b, a)
        k1 = gf.cyclic_mul(x, y)
        gf.set_f64_middle(0)
        c0 = gf.negacyclic_mul(a, b)
        k0 = gf.cyclic_mul(x, y)
    finally:
        gf.set_f64_middle(prev)
        gf.set_cluster_tiles(64)
    assert torch.equal(c1, c0)
    assert torch.equal(k1, k0)
    idx = np.sort(rng.choice(n, 64, replace=False)).astype(np.int32)
    got = np.rint(c1[batch - 1].cpu().numpy()[idx]).astype(np.int64)
    want = O.wrap64(O.negacyclic_coeffs(a[batch - 1].cpu().numpy().astype(np.int64),
                                        b[batch - 1].cpu().numpy().astype(np.int64), idx))
    assert np.array_equal(got, want)
