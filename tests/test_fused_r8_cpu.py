"""CPU checks of the index schedule of fused_r8_kernel
(gpu-fft_b200/csrc/gf_fused_r8.cuh), restated from its layout rules: a
4096-point tile on 512 threads x 8 points per operand; register window W
holds e-bits [W, W+3) with e = ebase_W(t) + (r << W); radix-8 rounds on e-bits
[9,12), [6,9), [3,6), [0,3) forward (the reverse inverse) with padded
transposes (point e at e + (e >> 3)). Stage u (e-bit 11 - u) uses
table[(g << u) + (e >> (12 - u))]: the rounds must reproduce the plain
12-stage loop exactly (on native tables, whose odd entries are +-i times the
even ones: only even entries are loaded), every shared-memory index must stay
in its buffer, each transpose must write every slot once, and a quarter-warp's
16-byte accesses must land in distinct 16-byte bank groups."""
import numpy as np
import pytest

E, T, RP = 4096, 512, 8
BUF = E + E // 8


def ebase(w, t):
    return (t & ((1 << w) - 1)) | ((t >> w) << (w + 3))


def ppos(e):
    return e + (e >> 3)


def poff(w, r):
    return (r << w) + ((r << w) >> 3)


def ct(x, y, w):
    return x + w * y, x - w * y


def gs(x, y, w):
    return x + y, (x - y) * w


def plain(x, tab, g, fwd):
    x = list(x)
    for u in (range(12) if fwd else range(11, -1, -1)):
        q = 11 - u
        for e in range(E):
            if e >> q & 1:
                continue
            w = tab[(g << u) + (e >> (q + 1))]
            x[e], x[e + (1 << q)] = (ct if fwd else gs)(x[e], x[e + (1 << q)], w)
    return x


def round8(st, fwd, w, tab, g):
    for t in range(T):
        eb = ebase(w, t)
        ws = {}
        for k in range(3):
            pb = 2 - k if fwd else k
            q = w + pb
            u = 11 - q
            nt = 1 << (2 - pb)
            base = (g << u) + (eb >> (q + 1))
            # the even entries are loaded, the odd ones rotated by +-i
            for h in range(0, nt, 2):
                assert 0 <= base + h < len(tab) and (nt == 1 or (base + h) % 2 == 0)
                ws[pb, h] = tab[base + h]
                if nt > 1:
                    ws[pb, h + 1] = (1j if fwd else -1j) * tab[base + h]
        for k in range(3):
            pb = 2 - k if fwd else k
            for r in range(RP):
                if r >> pb & 1:
                    continue
                st[t][r], st[t][r | 1 << pb] = (ct if fwd else gs)(st[t][r], st[t][r | 1 << pb], ws[pb, r >> (pb + 1)])


def groups_ok(addrs):
    """16-byte accesses of a quarter-warp (8 threads) hit 8 distinct 16-byte bank groups."""
    for q0 in range(0, len(addrs), 8):
        assert len({a % 8 for a in addrs[q0:q0 + 8]}) == 8


def transpose8(st, wa, wb):
    buf = [None] * BUF
    for t in range(T):
        for r in range(RP):
            a = ppos(ebase(wa, t)) + poff(wa, r)
            assert a == ppos(ebase(wa, t) + (r << wa)) and 0 <= a < BUF and buf[a] is None
            buf[a] = st[t][r]
    for r in range(RP):
        groups_ok([ppos(ebase(wa, t)) + poff(wa, r) for t in range(T)])
        groups_ok([ppos(ebase(wb, t)) + poff(wb, r) for t in range(T)])
    for t in range(T):
        st[t] = [buf[ppos(ebase(wb, t)) + poff(wb, r)] for r in range(RP)]


@pytest.mark.parametrize("m,g", [(15, 0), (15, 5), (16, 11), (13, 1)])
def test_fused_r8_matches_stage_loop(m, g):
    rng = np.random.default_rng(m * 31 + g)
    M = 1 << m
    # native tables: entry 2j+1 is exactly i (inverse: -i) times entry 2j
    tab = rng.standard_normal(M // 2) + 1j * rng.standard_normal(M // 2)
    tab[1::2] = 1j * tab[0::2]
    itab = np.conj(tab)
    a = list(rng.standard_normal(E) + 1j * rng.standard_normal(E))
    b = list(rng.standard_normal(E) + 1j * rng.standard_normal(E))
    sts = []
    for src in (a, b):
        st = [[src[t + (r << 9)] for r in range(RP)] for t in range(T)]  # window 9, coalesced
        for w_from, w_to in ((9, 6), (6, 3), (3, 0)):
            round8(st, True, w_from, tab, g)
            transpose8(st, w_from, w_to)
        round8(st, True, 0, tab, g)
        sts.append(st)
    fa, fb = plain(a, tab, g, True), plain(b, tab, g, True)
    for t in range(T):
        for r in range(RP):
            e = ebase(0, t) + r
            assert sts[0][t][r] == fa[e] and sts[1][t][r] == fb[e]
    z = [[sts[0][t][r] * sts[1][t][r] for r in range(RP)] for t in range(T)]
    for w_from, w_to in ((0, 3), (3, 6), (6, 9)):
        round8(z, False, w_from, itab, g)
        transpose8(z, w_from, w_to)
    round8(z, False, 9, itab, g)
    want = plain([fa[e] * fb[e] for e in range(E)], itab, g, False)
    got = [None] * E
    for t in range(T):
        for r in range(RP):
            got[t + (r << 9)] = z[t][r]
    np.testing.assert_array_equal(np.array(got), np.array(want))


def test_shared_memory_budget():
    # two padded double-complex buffers
    assert 2 * BUF * 16 <= 232448
