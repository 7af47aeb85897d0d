"""GPU tests of GPU_Special_FFT (the CKKS special FFT, reference fft.cu:727-1007):
the C ABI against the oracle's restatement of the reference kernels and
against the reference's own GPU build on the same inputs and tables (relative
L2: 1e-12 double, 2e-5 float), on tables of random unit values (every index
matters) and on the natural table, where the forward of a bit-reversed vector
is the +sign DFT."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = {np.complex128: 1e-12, np.complex64: 2e-5}


def rel_l2(got, want):
    got = np.asarray(got, np.complex128).ravel()
    want = np.asarray(want, np.complex128).ravel()
    return np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300)


def random_table(rng, M, C):
    return np.exp(2j * np.pi * rng.random(M)).astype(C)


def run_ours(gf, dev, x, table, n_power, fft_type, mi, batch):
    C = x.dtype
    buf = torch.from_numpy(x.copy()).to(dev)
    tab = torch.from_numpy(table.astype(C)).to(dev)
    L = gf.lib()
    f = L.gpufft_special_fft_f64 if C == np.complex128 else L.gpufft_special_fft_f32
    gf.check(f(buf.data_ptr(), tab.data_ptr(), n_power, fft_type, mi.real, mi.imag, batch, None), "special")
    return buf.cpu().numpy()


@pytest.mark.parametrize("C", [np.complex128, np.complex64])
@pytest.mark.parametrize("n_power,batch", [(1, 3), (3, 5), (4, 7), (7, 3), (11, 4), (12, 2), (13, 3), (16, 2),
                                           (17, 1), (20, 1)])
def test_special_fft_vs_oracle(gf, O, dev, C, n_power, batch):
    rng = np.random.default_rng(50 + n_power)
    M = 1 << n_power
    x = (rng.standard_normal(batch * M) + 1j * rng.standard_normal(batch * M)).astype(C)
    table = random_table(rng, M, C)
    for fft_type, mi in ((0, 1.0 + 0j), (1, complex(1.0 / M, 0.25 / M))):
        got = run_ours(gf, dev, x, table, n_power, fft_type, mi, batch)
        want = O.gpu_special_fft(x, table, n_power, fft_type, mi, batch)
        assert rel_l2(got, want) < TOL[C], (fft_type, rel_l2(got, want))


def test_special_fft_known_answer(gf, dev):
    # natural table t + j -> e^{i pi j / t}: forward of the bit-reversed vector
    # is the +sign DFT; the conjugate table with 1/M inverts it
    n = 14
    M = 1 << n
    rng = np.random.default_rng(3)
    tab = np.zeros(M, np.complex128)
    for e in range(n):
        t = 1 << e
        tab[t:2 * t] = np.exp(1j * np.pi * np.arange(t) / t)
    x = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    br = np.array([int(format(i, f"0{n}b")[::-1], 2) for i in range(M)])
    y = run_ours(gf, dev, x[br].astype(np.complex128), tab, n, 0, 1.0 + 0j, 1)
    assert rel_l2(y, M * np.fft.ifft(x)) < 1e-13
    z = run_ours(gf, dev, y, np.conj(tab), n, 1, complex(1.0 / M, 0.0), 1)
    assert rel_l2(z, x[br]) < 1e-13


@pytest.mark.parametrize("C", [np.complex128, np.complex64])
@pytest.mark.parametrize("n_power", [11, 12, 15, 17, 20, 24])
def test_special_fft_vs_reference_gpu_build(gf, O, dev, C, n_power):
    R = O.ref_gpu()
    if R is None:
        pytest.skip("the reference's GPU library was not compiled here")
    rng = np.random.default_rng(90 + n_power)
    M = 1 << n_power
    batch = 2 if n_power <= 20 else 1
    x = (rng.standard_normal(batch * M) + 1j * rng.standard_normal(batch * M)).astype(C)
    table = random_table(rng, M, C)
    f = R.ref_gpu_special_fft_f64 if C == np.complex128 else R.ref_gpu_special_fft_f32
    for fft_type, mi in ((0, 1.0 + 0j), (1, complex(1.0 / M, 0.0))):
        ref = torch.from_numpy(x.copy()).to(dev)
        tab = torch.from_numpy(table).to(dev)
        assert f(ref.data_ptr(), tab.data_ptr(), n_power, fft_type, mi.real, mi.imag, batch, None) == 0
        torch.cuda.synchronize()
        got = run_ours(gf, dev, x, table, n_power, fft_type, mi, batch)
        assert rel_l2(got, ref.cpu().numpy()) < TOL[C], (fft_type, rel_l2(got, ref.cpu().numpy()))


def test_special_fft_python_mirror_range(gf, dev):
    cfg = gf.fft_configuration(n_power=10)
    buf = torch.zeros(1 << 10, dtype=torch.complex128, device=dev)
    with pytest.raises(ValueError, match="Invalid n_power range!"):
        gf.GPU_Special_FFT(buf, buf, cfg, 1)
    cfg = gf.fft_configuration(n_power=11, fft_type=gf.FORWARD)
    x = torch.randn(1 << 11, dtype=torch.complex128, device=dev)
    tab = torch.exp(2j * np.pi * torch.rand(1 << 11, dtype=torch.float64, device=dev))
    y = x.clone()
    gf.GPU_Special_FFT(y, tab, cfg, 1)
    want = run_ours(gf, dev, x.cpu().numpy(), tab.cpu().numpy(), 11, 0, 1.0 + 0j, 1)
    assert np.allclose(y.cpu().numpy(), want, rtol=0, atol=0)
