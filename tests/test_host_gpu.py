"""GPU tests of the host-buffer products (chunked, transfers overlapped with
the computation): the results equal the device-buffer calls on the same data,
for ragged last chunks, pinned and pageable host memory, and the split
product's error report covers every chunk."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_power,batch,chunk,dtype,pinned", [
    (13, 10, 3, torch.float64, True), (16, 9, 0, torch.float64, True), (11, 7, 2, torch.float32, False),
    (16, 5, 2, torch.float32, True)])
def test_host_product_matches_device(gf, dev, n_power, batch, chunk, dtype, pinned):
    g = torch.Generator().manual_seed(n_power * 7 + batch)
    n = 1 << n_power
    a = torch.randint(-(1 << 15), 1 << 15, (batch, n), generator=g).to(dtype)
    b = torch.randint(-(1 << 15), 1 << 15, (batch, n), generator=g).to(dtype)
    if pinned:
        a, b = a.pin_memory(), b.pin_memory()
    tables = gf.ffnt_tables(n_power, "f64" if dtype == torch.float64 else "f32", dev)
    got = gf.negacyclic_mul_host(a, b, tables=tables, chunk=chunk)
    torch.cuda.synchronize()
    want = gf.negacyclic_mul(a.to(dev), b.to(dev), tables=tables).cpu()
    assert torch.equal(got, want)


@pytest.mark.parametrize("n_power,batch,chunk", [(12, 11, 4), (16, 7, 0), (16, 9, 2)])
def test_host_split_exact(gf, O, dev, n_power, batch, chunk):
    rng = np.random.default_rng(500 + n_power)
    n = 1 << n_power
    a = rng.integers(0, 1 << 24, (batch, n)).astype(np.int32)
    b = rng.integers(0, 1 << 24, (batch, n)).astype(np.int32)
    ah, bh = torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()
    got, err = gf.negacyclic_mul_split_host(ah, bh, input_bits=24, non_negative=True, chunk=chunk,
                                            return_error=True, device=dev)
    torch.cuda.synchronize()
    want, err_dev = gf.negacyclic_mul_split(ah.to(dev), bh.to(dev), input_bits=24, non_negative=True,
                                            return_error=True)
    assert torch.equal(got, want.cpu())
    # the host call's report is the maximum over its chunks: the whole-batch value
    assert float(err.item()) == float(err_dev.item())
    assert float(err.item()) < 0.5
    idx = np.sort(rng.choice(n, 64, replace=False)).astype(np.int32)
    for k in (0, batch - 1):
        assert np.array_equal(got.numpy()[k, idx], O.wrap64(O.negacyclic_coeffs(a[k], b[k], idx)))


def test_host_product_argument_errors(gf, dev):
    a = torch.zeros((2, 1 << 12), dtype=torch.float64)
    with pytest.raises(gf.GpufftError):
        gf.negacyclic_mul_host(a.to(dev), a.to(dev))
    tables = gf.ffnt_tables(12, "f64", dev)
    small = torch.empty(16, dtype=torch.uint8, device=dev)
    with pytest.raises(gf.GpufftError):
        gf.negacyclic_mul_host(a, a, tables=tables, workspace=small)
