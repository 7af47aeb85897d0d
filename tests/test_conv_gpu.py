"""GPU tests of the native linear product (the R_R product with half-length
transforms) and of its hand-written VJP (adjoint).

Tolerances: integer products bit-exact vs the exact schoolbook after rounding;
float32 results within relative L2 2e-5 of an FP64 reference; the VJP's
directional derivatives within relative 1e-4 of FP64 central finite
differences (eps = 1e-3, 64 random directions)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def np_linear(a, b):
    n = a.shape[-1]
    L = 2 * n
    return np.fft.irfft(np.fft.rfft(a, L) * np.fft.rfft(b, L), L)


def np_vjp(g, a, b):
    # grad_a[i] = sum_k g[k] b[k-i], grad_b[j] = sum_k g[k] a[k-j] (FP64 direct correlation via FFT)
    n = a.shape[-1]
    L = 2 * n
    G = np.fft.rfft(g, L)
    ga = np.fft.irfft(G * np.conj(np.fft.rfft(b, L)), L)[..., :n]
    gb = np.fft.irfft(G * np.conj(np.fft.rfft(a, L)), L)[..., :n]
    return ga, gb


def rel(x, y):
    return float(np.linalg.norm(np.asarray(x, np.float64) - y) / np.linalg.norm(y))


@pytest.mark.parametrize("n_power,batch", [(1, 3), (4, 5), (11, 3), (12, 2), (13, 2), (15, 2)])
def test_linear_f64_exact(gf, O, dev, n_power, batch):
    rng = np.random.default_rng(50 + n_power)
    n = 1 << n_power
    a = rng.integers(-(1 << 15), 1 << 15, (batch, n))
    b = rng.integers(-(1 << 15), 1 << 15, (batch, n))
    c = gf.linear_mul(torch.from_numpy(a.astype(np.float64)).to(dev), torch.from_numpy(b.astype(np.float64)).to(dev))
    got = np.rint(c.cpu().numpy()).astype(np.int64)
    for k in range(batch):
        assert np.array_equal(got[k], O.wrap64(O.schoolbook(a[k], b[k], O.LINEAR)))


@pytest.mark.parametrize("n_power", [5, 12, 14])
def test_linear_f32_vs_fp64(gf, dev, n_power):
    rng = np.random.default_rng(60 + n_power)
    n = 1 << n_power
    a = rng.standard_normal((4, n)).astype(np.float32)
    b = rng.standard_normal((4, n)).astype(np.float32)
    c = gf.linear_mul(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)).cpu().numpy()
    assert rel(c, np_linear(a.astype(np.float64), b.astype(np.float64))) < 2e-5


@pytest.mark.parametrize("n_power,batch", [(3, 3), (10, 4), (12, 3), (14, 4)])
def test_vjp_vs_direct_correlation(gf, dev, n_power, batch):
    rng = np.random.default_rng(70 + n_power)
    n = 1 << n_power
    a = rng.standard_normal((batch, n)).astype(np.float32)
    b = rng.standard_normal((batch, n)).astype(np.float32)
    g = rng.standard_normal((batch, 2 * n)).astype(np.float32)
    gd, ad, bd = (torch.from_numpy(x).to(dev) for x in (g, a, b))
    ga, gb = gf.linear_mul_vjp(gd, ad, bd)
    wa, wb = np_vjp(g.astype(np.float64), a.astype(np.float64), b.astype(np.float64))
    assert rel(ga.cpu().numpy(), wa) < 2e-5
    assert rel(gb.cpu().numpy(), wb) < 2e-5
    # gpufft_conv_vjp_f32 is the same entry point
    L = gf.lib()
    tables = gf.ffnt_tables(n_power + 1, "f32", dev)
    ws = torch.empty(max(1, int(L.gpufft_linear_mul_vjp_workspace_bytes(n_power, batch))), dtype=torch.uint8,
                     device=dev)
    ga2, gb2 = torch.empty_like(ad), torch.empty_like(bd)
    gf.check(L.gpufft_conv_vjp_f32(gd.data_ptr(), ad.data_ptr(), bd.data_ptr(), ga2.data_ptr(), gb2.data_ptr(),
                                   n_power, batch, tables.data_ptr(), ws.data_ptr(), ws.numel(), None), "conv_vjp")
    torch.cuda.synchronize()
    assert torch.equal(ga2, ga) and torch.equal(gb2, gb)


def test_vjp_n16384_batch512_finite_differences(gf, dev):
    # the convolution workload: N = 2^14 (padded to 2^15), batch 512, a, b, g i.i.d. N(0,1); the VJP
    # of L = <g, a*b> against FP64 central differences along 64 random directions
    rng = np.random.default_rng(5)
    n, batch = 1 << 14, 512
    a = rng.standard_normal((batch, n)).astype(np.float32)
    b = rng.standard_normal((batch, n)).astype(np.float32)
    g = rng.standard_normal((batch, 2 * n)).astype(np.float32)
    ga, gb = gf.linear_mul_vjp(*(torch.from_numpy(x).to(dev) for x in (g, a, b)))
    ga, gb = ga.cpu().numpy().astype(np.float64), gb.cpu().numpy().astype(np.float64)
    eps = 1e-3
    rows = rng.choice(batch, 8, replace=False)
    A, B, G = a[rows].astype(np.float64), b[rows].astype(np.float64), g[rows].astype(np.float64)

    def loss(x, y):
        return float(np.sum(G * np_linear(x, y)))
    for _ in range(64):
        da = rng.standard_normal(A.shape)
        db = rng.standard_normal(B.shape)
        fd = (loss(A + eps * da, B + eps * db) - loss(A - eps * da, B - eps * db)) / (2 * eps)
        an = float(np.sum(ga[rows] * da) + np.sum(gb[rows] * db))
        assert abs(an - fd) <= 1e-4 * max(1.0, abs(fd)), (an, fd)
    # and the whole batch against the direct correlation
    wa, wb = np_vjp(g.astype(np.float64), a.astype(np.float64), b.astype(np.float64))
    assert rel(ga, wa) < 2e-5 and rel(gb, wb) < 2e-5
