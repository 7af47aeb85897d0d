"""GPU tests of the per-kernel tracing: every launch of a product chain is
recorded under its kernel name with its algorithmic bytes, and nothing is
recorded while tracing is off."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_trace_records_the_fused_chain(gf, dev):
    n_power, batch = 16, 40
    n, m = 1 << n_power, 1 << (n_power - 1)
    a = torch.randn(batch, n, dtype=torch.float64, device=dev)
    b = torch.randn(batch, n, dtype=torch.float64, device=dev)
    tables = gf.ffnt_tables(n_power, "f64", dev)
    gf.negacyclic_mul(a, b, tables=tables)  # untraced
    torch.cuda.synchronize()
    assert gf.trace_collect() == []
    gf.trace_enable(True)
    try:
        gf.negacyclic_mul(a, b, tables=tables)
        torch.cuda.synchronize()
    finally:
        gf.trace_enable(False)
    rows = {r["kernel"]: r for r in gf.trace_collect()}
    # the FP64 middle pass: 512 threads x 8 points (the default) or 256 x 16
    middle = "fused_r8_kernel<f64,L12,middle>" if gf.set_f64_middle(-1) else "fused_kernel<f64,L12,middle>"
    fused = rows[middle]
    first = [r for k, r in rows.items() if k.startswith("col_pass<f64,fwd,L3")]
    last = [r for k, r in rows.items() if k.startswith("col_pass<f64,inv,L3")]
    assert len(first) == 1 and len(last) == 1
    waves = fused["launches"]
    assert waves >= 1 and first[0]["launches"] == waves and last[0]["launches"] == waves
    # algorithmic bytes: fold pairs in + spectra out; 2 spectra in + 1 out; spectrum in + reals out
    assert first[0]["alg_bytes"] == pytest.approx(2 * batch * m * (16 + 16))
    assert fused["alg_bytes"] == pytest.approx(batch * m * 6 * 8)
    assert last[0]["alg_bytes"] == pytest.approx(batch * m * (16 + 16))
    assert all(r["ms"] > 0 for r in rows.values())
    assert gf.trace_collect() == []
