"""GPU test of gpufft_negacyclic_mul_f64_noalloc, the entry point for callers
that cannot allocate device memory (it takes its scratch from a library-owned
16 MiB device array instead of a caller workspace).

Through the C ABI it must give the same products as gpufft_negacyclic_mul_f64
(relative L2 within 1e-12, the double-precision tolerance of the other product
tests, and identical after rounding), on two calls in a row -- the second call
reuses the scratch left by the first -- and it must reject rings whose scratch
would not fit. This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel_l2(x, y):
    return float(torch.linalg.norm(x - y) / torch.linalg.norm(y))


@pytest.mark.parametrize("n_power,batch", [(16, 40), (10, 7)])
def test_noalloc_matches_workspace_entry_point_twice(gf, dev, n_power, batch):
    L = gf.lib()
    n = 1 << n_power
    gen = torch.Generator(device=dev).manual_seed(77 + n_power)
    tables = gf.ffnt_tables(n_power, "f64", dev)
    ws_bytes = gf.negacyclic_mul_workspace_bytes(n_power, batch, 64)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream().cuda_stream or None
    for call in range(2):
        a = torch.randint(0, 1 << 12, (batch, n), device=dev, generator=gen).double()
        b = torch.randint(-(1 << 12), 1 << 12, (batch, n), device=dev, generator=gen).double()
        want = torch.empty_like(a)
        got = torch.full_like(a, float("nan"))
        gf.check(L.gpufft_negacyclic_mul_f64(a.data_ptr(), b.data_ptr(), want.data_ptr(), n_power, batch,
                                             tables.data_ptr(), ws.data_ptr(), ws_bytes, stream), "with workspace")
        gf.check(L.gpufft_negacyclic_mul_f64_noalloc(a.data_ptr(), b.data_ptr(), got.data_ptr(), n_power, batch,
                                                     tables.data_ptr(), stream), "noalloc")
        torch.cuda.synchronize()
        assert rel_l2(got, want) < 1e-12, call
        assert torch.equal(torch.round(got), torch.round(want)), call


def test_noalloc_rejects_rings_beyond_scratch(gf, dev):
    L = gf.lib()
    n_power = 21  # one product's scratch is 32 MiB, above the 16 MiB array
    tables = gf.ffnt_tables(n_power, "f64", dev)
    x = torch.zeros(1 << n_power, dtype=torch.float64, device=dev)
    st = L.gpufft_negacyclic_mul_f64_noalloc(x.data_ptr(), x.data_ptr(), x.data_ptr(), n_power, 1,
                                             tables.data_ptr(), None)
    assert st == gf.ERROR_WORKSPACE
