"""GPU tests of the programmatic launch of the chain kernels: with CUDA's
programmatic stream serialization a kernel's CTAs may be scheduled while the
previous kernel in the stream runs, and each waits for it before touching
memory. The results must be bit-identical to plain stream order, for chains
whose kernels read what the previous one wrote (drop-in GPU_FFNT and C_C
passes, the native and split products, the special FFT), including work that
another stream's kernel or a host copy fills just before, and inside a
captured CUDA graph."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture
def both(gf):
    prev = gf.set_programmatic_launch(-1)

    def run(fn):
        gf.set_programmatic_launch(1)
        on = fn()
        torch.cuda.synchronize()
        gf.set_programmatic_launch(0)
        off = fn()
        torch.cuda.synchronize()
        return on, off

    yield run
    gf.set_programmatic_launch(prev)


def test_switch_roundtrip(gf):
    prev = gf.set_programmatic_launch(-1)
    assert prev in (0, 1)
    assert gf.set_programmatic_launch(0) == prev
    assert gf.set_programmatic_launch(-1) == 0
    gf.set_programmatic_launch(prev)


@pytest.mark.parametrize("n_power,batch", [(11, 1), (13, 1), (14, 1), (16, 1), (16, 70), (19, 1), (23, 1)])
def test_ffnt_dropin_chain_identical(gf, O, dev, both, n_power, batch):
    n = 1 << n_power
    h = n // 2
    roots, inv_roots, twist, untwist = [torch.from_numpy(np.ascontiguousarray(t)).to(dev)
                                        for t in O.ffnt_tables(n, "f64")]
    rng = np.random.default_rng(n_power + batch)
    src = torch.from_numpy(rng.integers(-1000, 1000, 2 * batch * n).astype(np.float64)).to(dev)
    L = gf.lib()

    def run():
        inout = src.clone()
        temp = torch.empty(2 * batch * h, dtype=torch.complex128, device=dev)
        for _ in range(3):  # back-to-back calls: each reads the previous call's output
            gf.check(L.gpufft_ffnt_f64(inout.data_ptr(), temp.data_ptr(), twist.data_ptr(), roots.data_ptr(),
                                       n_power, 0, 1.0, 0.0, 2 * batch, 0, None), "fwd")
            gf.check(L.gpufft_ffnt_f64(inout.data_ptr(), temp.data_ptr(), untwist.data_ptr(), inv_roots.data_ptr(),
                                       n_power, 1, 1.0 / h, 0.0, batch, 1, None), "inv")
        return torch.cat([inout, torch.view_as_real(temp).ravel()])

    on, off = both(run)
    assert torch.equal(on, off)


@pytest.mark.parametrize("n_power", [12, 15, 21])
def test_c2c_chain_identical(gf, O, dev, both, n_power):
    rng = np.random.default_rng(500 + n_power)
    M = 1 << n_power
    x = (rng.standard_normal((2, M)) + 1j * rng.standard_normal((2, M))).astype(np.complex128)
    r, ri, _ = O.fft_tables(1 << (n_power - 1), "f64")
    d_r, d_ri = [torch.from_numpy(np.ascontiguousarray(t)).to(dev) for t in (r, ri)]
    L = gf.lib()

    def run():
        buf = torch.from_numpy(x.ravel().copy()).to(dev)
        gf.check(L.gpufft_fft_c2c_f64(buf.data_ptr(), d_r.data_ptr(), n_power, 0, 1, 0, 1.0, 0.0, 2, 0, None), "f")
        gf.check(L.gpufft_fft_c2c_f64(buf.data_ptr(), d_ri.data_ptr(), n_power, 1, 1, 0, 1.0 / M, 0.0, 1, 1, None),
                 "i")
        return buf

    on, off = both(run)
    assert torch.equal(on, off)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n_power,batch", [(12, 3), (16, 1), (16, 100), (18, 2)])
def test_native_product_identical(gf, dev, both, dtype, n_power, batch):
    g = torch.Generator().manual_seed(n_power * 7 + batch)
    n = 1 << n_power
    a = torch.randint(-(1 << 15), 1 << 15, (batch, n), generator=g).to(dtype).to(dev)
    b = torch.randint(-(1 << 15), 1 << 15, (batch, n), generator=g).to(dtype).to(dev)
    tables = gf.ffnt_tables(n_power, "f64" if dtype == torch.float64 else "f32", dev)
    on, off = both(lambda: gf.negacyclic_mul(a, b, tables=tables).clone())
    assert torch.equal(on, off)


@pytest.mark.parametrize("n_power,batch", [(13, 2), (16, 1), (16, 160)])
def test_split_product_identical_and_exact(gf, O, dev, both, n_power, batch):
    g = torch.Generator().manual_seed(n_power + batch)
    n = 1 << n_power
    a = torch.randint(0, 1 << 24, (batch, n), generator=g, dtype=torch.int32).to(dev)
    b = torch.randint(0, 1 << 24, (batch, n), generator=g, dtype=torch.int32).to(dev)
    on, off = both(lambda: gf.negacyclic_mul_split(a, b, input_bits=24, non_negative=True).clone())
    assert torch.equal(on, off)
    idx = np.array([0, 1, n // 2, n - 1], np.int32)
    want = O.wrap64(O.negacyclic_coeffs(a[0].cpu().numpy().astype(np.int64), b[0].cpu().numpy().astype(np.int64),
                                        idx))
    assert np.array_equal(on[0].cpu().numpy()[idx], want)


def test_chain_after_other_stream_and_host_copy(gf, dev):
    # the operands are produced by a kernel on another stream (event-ordered)
    # and by a host copy on the product's stream; the product's first kernel
    # must see them
    n_power, batch = 16, 4
    n = 1 << n_power
    tables = gf.ffnt_tables(n_power, "f64", dev)
    host = torch.randint(-1000, 1000, (batch, n), dtype=torch.float64).pin_memory()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    want = gf.negacyclic_mul(host.to(dev), host.to(dev) * 2.0, tables=tables)
    torch.cuda.synchronize()
    for _ in range(5):
        a = torch.empty((batch, n), dtype=torch.float64, device=dev)
        b = torch.empty_like(a)
        with torch.cuda.stream(s1):
            b.copy_(host, non_blocking=True)
            b.mul_(2.0)
            ev = torch.cuda.Event()
            ev.record(s1)
        s2.wait_event(ev)
        with torch.cuda.stream(s2):
            a.copy_(host, non_blocking=True)
            got = gf.negacyclic_mul(a, b, tables=tables, stream=s2)
        s2.synchronize()
        assert torch.equal(got, want)


def test_graph_capture_of_a_programmatic_chain(gf, dev):
    n_power, batch = 16, 2
    n = 1 << n_power
    prev = gf.set_programmatic_launch(1)
    try:
        g = torch.Generator().manual_seed(3)
        a = torch.randint(-1000, 1000, (batch, n), generator=g).double().to(dev)
        b = torch.randint(-1000, 1000, (batch, n), generator=g).double().to(dev)
        tables = gf.ffnt_tables(n_power, "f64", dev)
        ws = torch.empty(gf.negacyclic_mul_workspace_bytes(n_power, batch, 64), dtype=torch.uint8, device=dev)
        want = gf.negacyclic_mul(a, b, tables=tables, workspace=ws).clone()
        out = torch.empty_like(a)
        s = torch.cuda.Stream()
        graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with torch.cuda.graph(graph, stream=s):
            gf.negacyclic_mul(a, b, out=out, tables=tables, workspace=ws, stream=s)
        for _ in range(3):
            out.zero_()
            graph.replay()
            torch.cuda.synchronize()
            assert torch.equal(out, want)
    finally:
        gf.set_programmatic_launch(prev)
