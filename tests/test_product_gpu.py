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
