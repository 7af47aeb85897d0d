"""GPU tests of the cluster form of the contiguous 12-stage pass (few tiles:
each 4096-point tile spread over 8 CTAs through distributed shared memory),
and of its single-pass form for whole transforms of 2^10..2^12 points (2, 4
or 8 CTAs per row, with the FFNT fold / unfold and the linear-product load).
It runs the engine's butterflies with the same twiddles in the same stage
order, so every result must be bit-identical to the one-CTA-per-tile form:
each case runs twice, with the cluster form forced on and off. Parity with
the oracle at these sizes is covered by the product and drop-in tests, which
reach the cluster form under the default limit."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture
def both(gf):
    prev = gf.set_cluster_tiles(-1)

    def run(fn):
        gf.set_cluster_tiles(1 << 20)
        on = fn()
        torch.cuda.synchronize()
        gf.set_cluster_tiles(0)
        off = fn()
        torch.cuda.synchronize()
        return on, off

    yield run
    gf.set_cluster_tiles(prev)


def test_limit_roundtrip(gf):
    prev = gf.set_cluster_tiles(-1)
    assert prev >= 0
    assert gf.set_cluster_tiles(7) == prev
    assert gf.set_cluster_tiles(-1) == 7
    gf.set_cluster_tiles(prev)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n_power,batch", [(11, 1), (12, 2), (13, 1), (13, 64), (14, 1), (16, 1), (16, 3), (17, 2),
                                           (18, 1), (20, 1), (22, 1)])
def test_negacyclic_mul_cluster_identical(gf, dev, both, dtype, n_power, batch):
    g = torch.Generator().manual_seed(n_power * 11 + batch)
    n = 1 << n_power
    a = torch.randint(-(1 << 15), 1 << 15, (batch, n), generator=g).to(dtype).to(dev)
    b = torch.randint(-(1 << 15), 1 << 15, (batch, n), generator=g).to(dtype).to(dev)
    tables = gf.ffnt_tables(n_power, "f64" if dtype == torch.float64 else "f32", dev)
    on, off = both(lambda: gf.negacyclic_mul(a, b, tables=tables).clone())
    assert torch.equal(on, off)
    if dtype == torch.float64 and n_power <= 16:
        # |c| < 2^30 * N: the FP64 product rounds to the exact integers
        got = on.cpu().numpy()
        k = 0
        aa, bb = a[k].cpu().numpy().astype(np.int64), b[k].cpu().numpy().astype(np.int64)
        for j in (0, 1, n // 2, n - 1):
            idx = np.arange(n)
            want = int(np.sum(np.where(idx <= j, aa[idx] * bb[(j - idx) % n], -aa[idx] * bb[(j - idx) % n])))
            assert round(float(got[k, j])) == want


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("n_power,batch", [(10, 1), (11, 3), (12, 2), (13, 1), (15, 2), (17, 1)])
def test_cyclic_mul_cluster_identical(gf, dev, both, dtype, n_power, batch):
    g = torch.Generator().manual_seed(n_power + 5 * batch)
    M = 1 << n_power
    a = torch.randn((batch, M), dtype=dtype, generator=g).to(dev)
    b = torch.randn((batch, M), dtype=dtype, generator=g).to(dev)
    on, off = both(lambda: gf.cyclic_mul(a, b).clone())
    assert torch.equal(on, off)


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("n_power,neg", [(10, 0), (11, 0), (12, 0), (10, 1), (12, 1), (13, 0), (15, 0), (14, 1),
                                         (17, 1)])
def test_c2c_cluster_identical(gf, O, dev, both, T, n_power, neg):
    rng = np.random.default_rng(300 + n_power)
    M = 1 << n_power
    C = np.complex128 if T == np.float64 else np.complex64
    sfx = "f64" if T == np.float64 else "f32"
    x = (rng.standard_normal((2, M)) + 1j * rng.standard_normal((2, M))).astype(C)
    r, ri, _ = O.fft_tables((1 << n_power) if neg else (1 << (n_power - 1)), sfx)
    d_r = torch.from_numpy(np.ascontiguousarray(r)).to(dev)
    d_ri = torch.from_numpy(np.ascontiguousarray(ri)).to(dev)
    L = gf.lib()
    f = L.gpufft_fft_c2c_f64 if T == np.float64 else L.gpufft_fft_c2c_f32
    red = 0 if neg else 1

    def run():
        buf = torch.from_numpy(x.ravel().copy()).to(dev)
        gf.check(f(buf.data_ptr(), d_r.data_ptr(), n_power, 0, red, 0, 1.0, 0.0, 2, 0, None), "fwd")
        spec = buf.clone()
        gf.check(f(buf.data_ptr(), d_ri.data_ptr(), n_power, 1, red, 0, 1.0 / M, 0.0, 1, 1, None), "inv")
        return torch.cat([spec, buf])

    on, off = both(run)
    assert torch.equal(on, off)


@pytest.mark.parametrize("n_power", [11, 12, 13, 14, 16, 17])
def test_ffnt_dropin_cluster_identical(gf, O, dev, both, n_power):
    n = 1 << n_power
    h = n // 2
    roots, inv_roots, twist, untwist = [torch.from_numpy(np.ascontiguousarray(t)).to(dev)
                                        for t in O.ffnt_tables(n, "f64")]
    rng = np.random.default_rng(n_power)
    src = torch.from_numpy(rng.integers(-1000, 1000, 2 * n).astype(np.float64)).to(dev)
    L = gf.lib()

    def run():
        inout = src.clone()
        temp = torch.empty(2 * h, dtype=torch.complex128, device=dev)
        gf.check(L.gpufft_ffnt_f64(inout.data_ptr(), temp.data_ptr(), twist.data_ptr(), roots.data_ptr(), n_power,
                                   0, 1.0, 0.0, 2, 0, None), "fwd")
        gf.check(L.gpufft_ffnt_f64(inout.data_ptr(), temp.data_ptr(), untwist.data_ptr(), inv_roots.data_ptr(),
                                   n_power, 1, 1.0 / h, 0.0, 1, 1, None), "inv")
        return torch.cat([inout, torch.view_as_real(temp).ravel()])

    on, off = both(run)
    assert torch.equal(on, off)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n_power,batch", [(10, 1), (11, 2), (12, 1), (13, 1)])
def test_linear_mul_cluster_identical(gf, dev, both, dtype, n_power, batch):
    # rows of N = 2^n_power reals, product rows of 2N: one pass of 2^n_power points
    g = torch.Generator().manual_seed(n_power * 3 + batch)
    n = 1 << n_power
    a = torch.randn((batch, n), generator=g).to(dtype).to(dev)
    b = torch.randn((batch, n), generator=g).to(dtype).to(dev)
    on, off = both(lambda: gf.linear_mul(a, b).clone())
    assert torch.equal(on, off)


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("n_power,batch", [(12, 1), (13, 3), (16, 1), (18, 2)])
def test_special_fft_cluster_identical(gf, dev, both, T, n_power, batch):
    # GPU_Special_FFT forward then inverse on random vectors and a random table of
    # 2^n_power entries: the twelve smallest spans run on clusters or as column passes
    rng = np.random.default_rng(400 + n_power)
    M = 1 << n_power
    C = np.complex128 if T == np.float64 else np.complex64
    x = (rng.standard_normal((batch, M)) + 1j * rng.standard_normal((batch, M))).astype(C)
    tab = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(C)
    d_tab = torch.from_numpy(tab).to(dev)
    L = gf.lib()
    f = L.gpufft_special_fft_f64 if T == np.float64 else L.gpufft_special_fft_f32

    def run():
        buf = torch.from_numpy(x.ravel().copy()).to(dev)
        gf.check(f(buf.data_ptr(), d_tab.data_ptr(), n_power, 0, 1.0, 0.0, batch, None), "fwd")
        spec = buf.clone()
        gf.check(f(buf.data_ptr(), d_tab.data_ptr(), n_power, 1, 1.0 / M, 0.25, batch, None), "inv")
        return torch.cat([spec, buf])

    on, off = both(run)
    assert torch.equal(on, off)
