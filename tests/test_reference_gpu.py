"""GPU parity against the reference's OWN GPU library (its src/lib/fft.cu
compiled for sm_100a into oracle/_ref by oracle/Makefile), on the same inputs
and the same tables: integer products are identical after rounding, and the
float spectra agree within relative L2 1e-13 (f64). Skipped where that build
is absent."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R(O):
    r = O.ref_gpu()
    if r is None:
        pytest.skip("reference GPU build (oracle/_ref/libgpufft_ref_gpu.so) not present")
    return r


def td(x, dev):
    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


@pytest.mark.parametrize("n_power", [12, 14, 16, 18])
def test_ffnt_matches_reference_gpu(gf, O, R, dev, n_power):
    rng = np.random.default_rng(900 + n_power)
    n = 1 << n_power
    h = n // 2
    batch = 3
    ab = rng.integers(0, 1 << 10, (2 * batch, n)).astype(np.float64)
    tabs = [td(t, dev) for t in O.ffnt_tables(n, "f64")]
    roots, inv_roots, twist, untwist = tabs
    outs = []
    for impl in ("ours", "ref"):
        buf = td(ab.ravel(), dev)
        temp = torch.zeros(2 * batch * h, dtype=torch.complex128, device=dev)
        if impl == "ours":
            f = gf.lib().gpufft_ffnt_f64
        else:
            f = R.ref_gpu_ffnt_f64
        assert f(buf.data_ptr(), temp.data_ptr(), twist.data_ptr(), roots.data_ptr(), n_power, 0, 1.0, 0.0,
                 2 * batch, 0, None) == 0
        spec = temp.clone()
        assert f(buf.data_ptr(), temp.data_ptr(), untwist.data_ptr(), inv_roots.data_ptr(), n_power, 1, 1.0 / h,
                 0.0, batch, 1, None) == 0
        torch.cuda.synchronize()
        outs.append((spec.cpu().numpy(), buf.cpu().numpy()[: batch * n]))
    (s0, p0), (s1, p1) = outs
    assert np.linalg.norm(s0 - s1) / np.linalg.norm(s1) < 1e-13
    assert np.array_equal(np.rint(p0), np.rint(p1))


@pytest.mark.parametrize("n_power", [13, 17])
def test_c2c_and_r2r_match_reference_gpu(gf, O, R, dev, n_power):
    rng = np.random.default_rng(950 + n_power)
    M = 1 << n_power
    n = M // 2
    batch = 2
    roots, inv_roots, ninv = O.fft_tables(n, "f64")
    d_roots, d_inv = td(roots, dev), td(inv_roots, dev)
    x = (rng.standard_normal((2 * batch, M)) + 1j * rng.standard_normal((2 * batch, M))).astype(np.complex128)
    res = []
    for f in (gf.lib().gpufft_fft_c2c_f64, None):
        buf = td(x.ravel(), dev)
        if f is None:
            st = R.ref_gpu_fft_c2c_f64(buf.data_ptr(), d_roots.data_ptr(), n_power, 0, 1, 1.0, 0.0, 2 * batch, 0, None)
            st |= R.ref_gpu_fft_c2c_f64(buf.data_ptr(), d_inv.data_ptr(), n_power, 1, 1, float(ninv), 0.0, batch, 1,
                                        None)
        else:
            st = f(buf.data_ptr(), d_roots.data_ptr(), n_power, 0, 1, 0, 1.0, 0.0, 2 * batch, 0, None)
            st |= f(buf.data_ptr(), d_inv.data_ptr(), n_power, 1, 1, 0, float(ninv), 0.0, batch, 1, None)
        assert st == 0
        torch.cuda.synchronize()
        res.append(buf.cpu().numpy()[: batch * M])
    assert np.linalg.norm(res[0] - res[1]) / np.linalg.norm(res[1]) < 1e-13
    # R_R linear product of integers: identical after rounding
    real = np.zeros((2 * batch, M))
    real[:, :n] = rng.integers(-(1 << 12), 1 << 12, (2 * batch, n))
    out = []
    for impl in ("ours", "ref"):
        rb = td(real.ravel(), dev)
        temp = torch.zeros(2 * batch * M, dtype=torch.complex128, device=dev)
        if impl == "ours":
            f = gf.lib().gpufft_fft_r2r_f64
            st = f(rb.data_ptr(), temp.data_ptr(), d_roots.data_ptr(), n_power, 0, 1, 0, 1.0, 0.0, 2 * batch, 0,
                   None)
            st |= f(rb.data_ptr(), temp.data_ptr(), d_inv.data_ptr(), n_power, 1, 1, 0, float(ninv), 0.0, batch, 1,
                    None)
        else:
            st = R.ref_gpu_fft_r2r_f64(rb.data_ptr(), temp.data_ptr(), d_roots.data_ptr(), n_power, 0, 1, 1.0, 0.0,
                                       2 * batch, 0, None)
            st |= R.ref_gpu_fft_r2r_f64(rb.data_ptr(), temp.data_ptr(), d_inv.data_ptr(), n_power, 1, 1,
                                        float(ninv), 0.0, batch, 1, None)
        assert st == 0
        torch.cuda.synchronize()
        out.append(np.rint(rb.cpu().numpy()[: batch * M]))
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("n_power", [12, 13, 16, 18])
def test_c2c_negacyclic_mode_matches_reference_gpu(gf, O, R, dev, n_power):
    # GPU_FFT with reduction_poly = X_N_plus (twiddle index 2^s + g into an
    # M-entry psi table, reference fft.cu:67-74): forward of 2 * batch vectors,
    # then the inverse with the product, ours and the reference's on the same
    # data and the same FFT<double>(M) tables. A product of integer vectors
    # through the negacyclic transforms is the product mod X^M + 1: identical
    # after rounding.
    rng = np.random.default_rng(970 + n_power)
    M = 1 << n_power
    batch = 2
    roots, inv_roots, ninv = O.fft_tables(M, "f64")
    d_roots, d_inv = td(roots, dev), td(inv_roots, dev)
    x = (rng.standard_normal((2 * batch, M)) + 1j * rng.standard_normal((2 * batch, M))).astype(np.complex128)
    ints = rng.integers(-(1 << 10), 1 << 10, (2 * batch, M)).astype(np.complex128)
    for data, exact in ((x, False), (ints, True)):
        res, specs = [], []
        for impl in ("ours", "ref"):
            buf = td(data.ravel(), dev)
            if impl == "ours":
                f = gf.lib().gpufft_fft_c2c_f64
                st = f(buf.data_ptr(), d_roots.data_ptr(), n_power, 0, 0, 0, 1.0, 0.0, 2 * batch, 0, None)
                spec = buf.clone()
                st |= f(buf.data_ptr(), d_inv.data_ptr(), n_power, 1, 0, 0, 1.0 / M, 0.0, batch, 1, None)
            else:
                st = R.ref_gpu_fft_c2c_f64(buf.data_ptr(), d_roots.data_ptr(), n_power, 0, 0, 1.0, 0.0, 2 * batch,
                                           0, None)
                spec = buf.clone()
                st |= R.ref_gpu_fft_c2c_f64(buf.data_ptr(), d_inv.data_ptr(), n_power, 1, 0, 1.0 / M, 0.0, batch,
                                            1, None)
            assert st == 0
            torch.cuda.synchronize()
            specs.append(spec.cpu().numpy())
            res.append(buf.cpu().numpy()[: batch * M])
        assert np.linalg.norm(specs[0] - specs[1]) / np.linalg.norm(specs[1]) < 1e-13
        assert np.linalg.norm(res[0] - res[1]) / np.linalg.norm(res[1]) < 1e-13
        if exact:
            assert np.array_equal(np.rint(res[0].real), np.rint(res[1].real))
            assert np.array_equal(np.rint(res[0].imag), np.rint(res[1].imag))
            # and it is the negacyclic product
            a0 = ints[0].real.astype(np.int64)
            b0 = ints[batch].real.astype(np.int64)
            want = O.wrap64(O.schoolbook(a0, b0)) if M <= 4096 else None
            if want is not None:
                assert np.array_equal(np.rint(res[0][:M].real).astype(np.int64), want)
