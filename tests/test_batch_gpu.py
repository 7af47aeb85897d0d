"""GPU tests of the mixed-size batch plan (4096 requests, ring sizes 2^10..2^17):
requests with ring sizes 2^10 .. 2^17 run in one persistent cooperative launch
(captured in a CUDA graph) and must give outputs identical to per-size
sequential launches of gpufft_negacyclic_mul_*; FP64 results of 16-bit
coefficients are exact."""
import os
import tempfile

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def make_requests(rng, count, lo=10, hi=17):
    return [int(x) for x in rng.integers(lo, hi + 1, count)]


def per_size_reference(gf, plan, a_list, b_list, dtype):
    # one negacyclic_mul call per ring size on the same data
    out = [None] * len(a_list)
    sizes = sorted(set(plan.n_powers))
    for np_ in sizes:
        idx = [i for i, n in enumerate(plan.n_powers) if n == np_]
        A = torch.stack([a_list[i] for i in idx])
        B = torch.stack([b_list[i] for i in idx])
        C = gf.negacyclic_mul(A, B)
        for k, i in enumerate(idx):
            out[i] = C[k]
    return out


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_batch_matches_per_size_launches(gf, O, dev, dtype):
    rng = np.random.default_rng(44)
    n_powers = make_requests(rng, 96, 2, 17)
    plan = gf.BatchPlan(n_powers, dtype)
    a_list = [torch.from_numpy(rng.integers(-(1 << 15), 1 << 15, 1 << n).astype(np.float64)).to(dev, dtype)
              for n in n_powers]
    b_list = [torch.from_numpy(rng.integers(-(1 << 15), 1 << 15, 1 << n).astype(np.float64)).to(dev, dtype)
              for n in n_powers]
    a, b = plan.pack(a_list), plan.pack(b_list)
    ref = per_size_reference(gf, plan, a_list, b_list, dtype)
    for shape in ((1, 1), (2, 4), (0, 1)):  # persistent launches and per-class chains
        plan.set_shape(*shape)
        c = plan.execute(a, b)
        got = plan.unpack(c)
        for i in range(len(n_powers)):
            assert torch.equal(got[i], ref[i]), (shape, i, n_powers[i])
    assert plan.status() == 0
    # gpufft_batch_plan_run is the same entry point
    c_run = torch.empty_like(a)
    gf.check(gf.lib().gpufft_batch_plan_run(plan.h, a.data_ptr(), b.data_ptr(), c_run.data_ptr(), None), "run")
    torch.cuda.synchronize()
    assert torch.equal(c_run, c)
    if dtype == torch.float64:  # |c| < 2^47: exact
        for i in rng.choice(len(n_powers), 6, replace=False):
            n = 1 << n_powers[i]
            ai = a_list[i].cpu().numpy().astype(np.int64)
            bi = b_list[i].cpu().numpy().astype(np.int64)
            idx = np.sort(rng.choice(n, min(n, 64), replace=False)).astype(np.int32)
            want = O.wrap64(O.negacyclic_coeffs(ai, bi, idx))
            assert np.array_equal(np.rint(got[i].cpu().numpy()[idx]).astype(np.int64), want)
    plan.close()


def test_batch_4096_mixed_sizes_graph_and_autotune(gf, O, dev):
    # the full mixed workload: 4096 requests, ring sizes log-uniform over 2^10..2^17, FP64,
    # one persistent launch captured in a CUDA graph, autotuned launch shape
    rng = np.random.default_rng(4)
    n_powers = make_requests(rng, 4096)
    plan = gf.BatchPlan(n_powers, torch.float64)
    g = torch.Generator(device=dev).manual_seed(4)
    a = torch.randint(-(1 << 15), 1 << 15, (plan.total,), device=dev, generator=g).double()
    b = torch.randint(-(1 << 15), 1 << 15, (plan.total,), device=dev, generator=g).double()
    plan.set_shape(1, 1)  # the persistent launch
    c0 = plan.execute(a, b)
    # identical to one gpufft_negacyclic_mul_f64 call per ring size on the same data
    got = plan.unpack(c0)
    for np_ in sorted(set(n_powers)):
        idx = [i for i, n in enumerate(n_powers) if n == np_]
        o0 = int(min(plan.offsets[i] for i in idx))
        n = 1 << np_
        ref = gf.negacyclic_mul(a[o0:o0 + len(idx) * n].view(len(idx), n), b[o0:o0 + len(idx) * n].view(len(idx), n))
        assert torch.equal(c0[o0:o0 + len(idx) * n].view(len(idx), n), ref), np_
    # the per-class chains: about 512 requests per class, so the classes above
    # 2^12 run the non-cluster middle pass on the plan's own tables
    plan.set_shape(0, 1)
    assert torch.equal(plan.execute(a, b), c0)
    plan.set_shape(1, 1)
    # |c| < 2^47: exact against the __int128 product on sampled coefficients
    for i in rng.choice(len(n_powers), 12, replace=False):
        n = 1 << n_powers[i]
        o = int(plan.offsets[i])
        ai = a[o:o + n].cpu().numpy().astype(np.int64)
        bi = b[o:o + n].cpu().numpy().astype(np.int64)
        idx = np.sort(rng.choice(n, 64, replace=False)).astype(np.int32)
        assert np.array_equal(np.rint(got[i].cpu().numpy()[idx]).astype(np.int64),
                              O.wrap64(O.negacyclic_coeffs(ai, bi, idx)))
    with tempfile.TemporaryDirectory() as d:
        cache = os.path.join(d, "tune.jsonl")
        info = plan.autotune(a, b, torch.empty_like(a), cache)
        assert info["ctas_per_sm"] in (0, 1, 2) and info["items_per_grab"] in (1, 2, 4)
        assert os.path.exists(cache)
        plan.autotune(a, b, torch.empty_like(a), cache)  # cache hit
    s = torch.cuda.Stream()
    c1 = torch.full_like(a, float("nan"))
    torch.cuda.synchronize()
    plan.capture(a, b, c1, s)
    plan.replay(s)
    plan.replay(s)
    s.synchronize()
    assert torch.equal(c0, c1)
    assert plan.status() == 0
    plan.close()


def test_split_batch_exact_and_graph(gf, O, dev):
    # exact mixed-size products (FP32 split): every request equals the per-size
    # split call bit for bit and the exact negacyclic product on sampled
    # coefficients; a captured graph replays to the same output
    rng = np.random.default_rng(45)
    n_powers = make_requests(rng, 60, 2, 17)
    plan = gf.SplitBatchPlan(n_powers, input_bits=16, non_negative=False)
    a_list = [torch.from_numpy(rng.integers(-(1 << 15), 1 << 15, 1 << n).astype(np.int32)).to(dev)
              for n in n_powers]
    b_list = [torch.from_numpy(rng.integers(-(1 << 15), 1 << 15, 1 << n).astype(np.int32)).to(dev)
              for n in n_powers]
    a, b = plan.pack(a_list), plan.pack(b_list)
    c, err = plan.execute(a, b)
    assert float(err.item()) < 0.5
    got = plan.unpack(c)
    for np_ in sorted(set(n_powers)):
        idx = [i for i, n in enumerate(n_powers) if n == np_]
        C = gf.negacyclic_mul_split(torch.stack([a_list[i] for i in idx]), torch.stack([b_list[i] for i in idx]),
                                    input_bits=16, non_negative=False)
        for k, i in enumerate(idx):
            assert torch.equal(got[i], C[k]), (i, np_)
    for i in rng.choice(len(n_powers), 8, replace=False):
        n = 1 << n_powers[i]
        ai, bi = a_list[i].cpu().numpy(), b_list[i].cpu().numpy()
        idx = np.sort(rng.choice(n, min(n, 64), replace=False)).astype(np.int32)
        assert np.array_equal(got[i].cpu().numpy()[idx], O.wrap64(O.negacyclic_coeffs(ai, bi, idx)))
    s = torch.cuda.Stream()
    c2 = torch.empty_like(c)
    err2 = torch.zeros(1, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    plan.capture(a, b, c2, err2, s)
    plan.replay(s)
    plan.replay(s)
    s.synchronize()
    assert torch.equal(c2, c)
    assert float(err2.item()) == float(err.item())
    plan.close()


def test_batch_barrier_timeout_is_reported(gf, dev):
    # the persistent launch's grid barriers are bounded waits: with a target
    # that no barrier can reach (extra arrivals) and a short poll limit, every
    # barrier gives up, the kernel returns, the plan reports the timeout, and
    # the context stays usable -- the same plan then runs normally again
    rng = np.random.default_rng(46)
    n_powers = [14, 15, 16, 12, 13, 16, 14, 15]
    plan = gf.BatchPlan(n_powers, torch.float64)
    a = torch.from_numpy(rng.integers(-(1 << 15), 1 << 15, plan.total).astype(np.float64)).to(dev)
    b = torch.from_numpy(rng.integers(-(1 << 15), 1 << 15, plan.total).astype(np.float64)).to(dev)
    plan.set_shape(1, 1)
    ref = plan.execute(a, b)
    torch.cuda.synchronize()
    assert plan.status() == 0
    plan.set_barrier(max_polls=4096, extra_arrivals=1)
    plan.execute(a, b)
    torch.cuda.synchronize()
    assert plan.status() == 1
    assert plan.status() == 0  # reading clears the flag
    plan.set_barrier()  # defaults
    again = plan.execute(a, b)
    torch.cuda.synchronize()
    assert plan.status() == 0
    assert torch.equal(again, ref)
    plan.close()


def test_batch_autotune_rejects_aliased_output(gf, dev):
    plan = gf.BatchPlan([12, 13], torch.float64)
    a = torch.zeros(plan.total, dtype=torch.float64, device=dev)
    b = torch.zeros_like(a)
    with pytest.raises(gf.GpufftError):
        plan.autotune(a, b, a)
    plan.close()
