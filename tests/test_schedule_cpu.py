"""CPU checks of the index schedules of the cluster kernels and of the split
product's permuted spectrum order, restated in Python from the kernels'
layout rules (gpu-fft_b200/csrc/gf_cluster.cuh, gf_special.cu, gf_engine.cuh):

* the cluster form of a contiguous 12-stage pass (8 CTAs x 64 threads x 8
  points per 4096-point tile; X layout e = 64 c + t + 512 k, Y layouts inside
  each CTA's 512 points; DSMEM exchanges into padded buffers) must perform
  exactly the butterflies of the plain stage loop -- stage u on e-bit 11 - u
  with table[(g << u) + (e >> (12 - u))] -- for the fused, forward and inverse
  modes, cyclic and negacyclic indexing; and so must its single-pass form for
  2^LT-point transforms, LT = 10, 11 (2^(LT-9) CTAs; X register k = (h, lo)
  holds e = 64 c + t + 64 2^(LT-9) lo + 512 h);
* the special-FFT cluster pass must perform the special network's spans
  2^0..2^11 with table[2^q + (e mod 2^q)];
* every shared-memory slot stays inside its buffer, every exchange slot is
  written exactly once, and every twiddle index stays inside its table.

Both sides use the same Python butterflies, so results must be identical.
"""
import numpy as np
import pytest

CL, TH = 8, 64
SMEM = 512 + 512 // 8


def cpad(l):
    return l + (l >> 3)


def ypos(y, t, r):
    if y == 1:
        return t + 64 * r
    if y == 2:
        return (t & 7) + ((t >> 3) << 6) + 8 * r
    return 8 * t + r


def ct(x, y, w):
    return x + w * y, x - w * y


def gs(x, y, w):
    return x + y, (x - y) * w


# ---------------------------------------------------------------- the FFT pass
def plain_pass(x, tab, g, fwd, lt=12):
    x = list(x)
    for u in (range(lt) if fwd else range(lt - 1, -1, -1)):
        q = lt - 1 - u
        for e in range(1 << lt):
            if e >> q & 1:
                continue
            w = tab[(g << u) + (e >> (q + 1))]
            x[e], x[e + (1 << q)] = (ct if fwd else gs)(x[e], x[e + (1 << q)], w)
    return x


def cl_round(regs, p, ebase, tab, g, fwd, lt=12):
    for k in range(3):
        i = 2 - k if fwd else k
        q = p + i
        u = lt - 1 - q
        base = (g << u) + (ebase >> (q + 1))
        w = []
        for h in range(4 >> i):
            assert 0 <= base + h < len(tab)
            w.append(tab[base + h])
        for r in range(8):
            if r >> i & 1:
                continue
            for arr in regs:
                arr[r], arr[r | (1 << i)] = (ct if fwd else gs)(arr[r], arr[r | (1 << i)], w[r >> (i + 1)])


def cl_xround(regs, tab, g, fwd, lt):
    """The cross-CTA stages: e-bits 9..lt-1 on register bits lob..2."""
    lc = lt - 9
    lob = 3 - lc
    for k in range(lc):
        i = lc - 1 - k if fwd else k
        u = lt - 1 - (9 + i)
        w = []
        for h in range((1 << lc) >> (i + 1)):
            assert 0 <= (g << u) + h < len(tab)
            w.append(tab[(g << u) + h])
        for r in range(8):
            if r >> (lob + i) & 1:
                continue
            for arr in regs:
                b = r | (1 << (lob + i))
                arr[r], arr[b] = (ct if fwd else gs)(arr[r], arr[b], w[(r >> lob) >> (i + 1)])


def transpose(state, bufs, ya, yb, na, cl=CL):
    for c in range(cl):
        for t in range(TH):
            for a in range(na):
                for r in range(8):
                    slot = cpad(ypos(ya, t, r))
                    assert slot < SMEM
                    bufs[c][a][slot] = state[c, t][a][r]
    for c in range(cl):
        for t in range(TH):
            state[c, t] = [[bufs[c][a][cpad(ypos(yb, t, r))] for r in range(8)] for a in range(na)]


def cluster_pass(mode, ops, tab, itab, g, lt=12):
    na = 2 if mode == "fused" else 1
    lc = lt - 9
    cl, lob = 1 << lc, 3 - lc

    def xl(c, t, k):  # local point of X register k (in CTA k >> lob)
        return 64 * c + t + 64 * cl * (k & ((1 << lob) - 1))

    def xe(c, t, k):
        return xl(c, t, k) + 512 * (k >> lob)

    ybuf = [[[None] * SMEM for _ in range(na)] for _ in range(cl)]
    xbuf = [[[None] * SMEM] for _ in range(cl)]
    st = {}
    out = [None] * (1 << lt)
    if mode == "inv":
        for c in range(cl):
            for t in range(TH):
                st[c, t] = [[ops[0][512 * c + ypos(1, t, r)] for r in range(8)]]
        transpose(st, ybuf, 1, 3, 1, cl)
    else:
        seen = set()
        for c in range(cl):
            for t in range(TH):
                for k in range(8):
                    assert xe(c, t, k) not in seen
                    seen.add(xe(c, t, k))
                st[c, t] = [[ops[a][xe(c, t, k)] for k in range(8)] for a in range(na)]
                cl_xround(st[c, t], tab, g, True, lt)
        assert seen == set(range(1 << lt))
        for c in range(cl):  # X -> Y1: register k to CTA k >> lob at its local point
            for t in range(TH):
                for k in range(8):
                    for a in range(na):
                        slot = cpad(xl(c, t, k))
                        assert slot < SMEM and ybuf[k >> lob][a][slot] is None
                        ybuf[k >> lob][a][slot] = st[c, t][a][k]
        for c in range(cl):
            for t in range(TH):
                st[c, t] = [[ybuf[c][a][cpad(ypos(1, t, r))] for r in range(8)] for a in range(na)]
                cl_round(st[c, t], 6, 512 * c + ypos(1, t, 0), tab, g, True, lt)
        for ya, yb, p in ((1, 2, 3), (2, 3, 0)):
            transpose(st, ybuf, ya, yb, na, cl)
            for c in range(cl):
                for t in range(TH):
                    cl_round(st[c, t], p, 512 * c + ypos(yb, t, 0), tab, g, True, lt)
        if mode == "fwd":
            transpose(st, ybuf, 3, 1, 1, cl)
            for c in range(cl):
                for t in range(TH):
                    for r in range(8):
                        e = 512 * c + ypos(1, t, r)
                        assert out[e] is None
                        out[e] = st[c, t][0][r]
            return out
        for c in range(cl):
            for t in range(TH):
                st[c, t] = [[st[c, t][0][r] * st[c, t][1][r] for r in range(8)]]
    for c in range(cl):
        for t in range(TH):
            cl_round(st[c, t], 0, 512 * c + ypos(3, t, 0), itab, g, False, lt)
    for ya, yb, p in ((3, 2, 3), (2, 1, 6)):
        transpose(st, ybuf, ya, yb, 1, cl)
        for c in range(cl):
            for t in range(TH):
                cl_round(st[c, t], p, 512 * c + ypos(yb, t, 0), itab, g, False, lt)
    for c in range(cl):  # Y1 -> X: point 512 c + t + 64 r to CTA r & (cl-1), register (c << lob) | (r >> lc)
        for t in range(TH):
            for r in range(8):
                k = (c << lob) | (r >> lc)
                dst = r & (cl - 1)
                assert xe(dst, t, k) == 512 * c + t + 64 * r
                slot = cpad(64 * k + t)
                assert slot < SMEM and xbuf[dst][0][slot] is None
                xbuf[dst][0][slot] = st[c, t][0][r]
    for c in range(cl):
        for t in range(TH):
            z = [[xbuf[c][0][cpad(64 * k + t)] for k in range(8)]]
            cl_xround(z, itab, g, False, lt)
            for k in range(8):
                assert out[xe(c, t, k)] is None
                out[xe(c, t, k)] = z[0][k]
    return out


def cvec(rng, n):
    return [complex(v) for v in rng.standard_normal(n) + 1j * rng.standard_normal(n)]


@pytest.mark.parametrize("m,tile,neg", [(13, 1, 0), (15, 5, 0), (14, 2, 1)])
def test_cluster_pass_schedule(m, tile, neg):
    rng = np.random.default_rng(m + tile)
    s0 = m - 12
    size = (1 << m) if neg else (1 << (m - 1))  # negacyclic tables carry 2^s offsets
    tab, itab = cvec(rng, size), cvec(rng, size)
    g = tile + ((1 << s0) if neg else 0)
    a, b = cvec(rng, 4096), cvec(rng, 4096)
    fa, fb = plain_pass(a, tab, g, True), plain_pass(b, tab, g, True)
    assert cluster_pass("fwd", [a], tab, itab, g) == fa
    assert cluster_pass("inv", [a], itab, itab, g) == plain_pass(a, itab, g, False)
    prod = [x * y for x, y in zip(fa, fb)]
    assert cluster_pass("fused", [a, b], tab, itab, g) == plain_pass(prod, itab, g, False)


@pytest.mark.parametrize("lt,neg", [(10, 0), (11, 0), (12, 0), (11, 1), (10, 1)])
def test_single_pass_cluster_schedule(lt, neg):
    # a whole transform of 2^lt points (one tile, group 0 at stage 0)
    rng = np.random.default_rng(90 + lt + neg)
    size = (1 << (lt + 1)) if neg else (1 << (lt - 1))
    tab, itab = cvec(rng, size), cvec(rng, size)
    g = 1 if neg else 0
    n = 1 << lt
    a, b = cvec(rng, n), cvec(rng, n)
    fa, fb = plain_pass(a, tab, g, True, lt), plain_pass(b, tab, g, True, lt)
    assert cluster_pass("fwd", [a], tab, itab, g, lt) == fa
    assert cluster_pass("inv", [a], itab, itab, g, lt) == plain_pass(a, itab, g, False, lt)
    prod = [x * y for x, y in zip(fa, fb)]
    assert cluster_pass("fused", [a, b], tab, itab, g, lt) == plain_pass(prod, itab, g, False, lt)


# ------------------------------------------------------------ the special FFT
def plain_special(x, tab, fwd):
    x = list(x)
    for q in (range(12) if fwd else range(11, -1, -1)):
        t = 1 << q
        for e in range(4096):
            if e >> q & 1:
                continue
            x[e], x[e + t] = (ct if fwd else gs)(x[e], x[e + t], tab[t + (e & (t - 1))])
    return x


def special_round(regs, p, ebase, tab, fwd):
    for k in range(3):
        i = k if fwd else 2 - k
        base = (1 << (p + i)) + (ebase & ((1 << p) - 1))
        w = []
        for h in range(1 << i):
            assert base + (h << p) < len(tab)
            w.append(tab[base + (h << p)])
        for r in range(8):
            if r >> i & 1:
                continue
            regs[0][r], regs[0][r | (1 << i)] = (ct if fwd else gs)(regs[0][r], regs[0][r | (1 << i)],
                                                                     w[r & ((1 << i) - 1)])


def special_cluster(x, tab, fwd):
    ybuf = [[[None] * SMEM] for _ in range(CL)]
    xbuf = [[None] * SMEM for _ in range(CL)]
    st = {}
    out = [None] * 4096
    if fwd:
        for c in range(CL):
            for t in range(TH):
                st[c, t] = [[x[512 * c + ypos(1, t, r)] for r in range(8)]]
        transpose(st, ybuf, 1, 3, 1)
        for ya, yb, p in ((None, 3, 0), (3, 2, 3), (2, 1, 6)):
            if ya is not None:
                transpose(st, ybuf, ya, yb, 1)
            for c in range(CL):
                for t in range(TH):
                    special_round(st[c, t], p, 512 * c + ypos(yb, t, 0), tab, True)
        for c in range(CL):
            for t in range(TH):
                for r in range(8):
                    assert xbuf[r][cpad(64 * c + t)] is None
                    xbuf[r][cpad(64 * c + t)] = st[c, t][0][r]
        for c in range(CL):
            for t in range(TH):
                ex = 64 * c + t
                z = [[xbuf[c][cpad(64 * k + t)] for k in range(8)]]
                special_round(z, 9, ex, tab, True)
                for k in range(8):
                    out[ex + 512 * k] = z[0][k]
    else:
        for c in range(CL):
            for t in range(TH):
                ex = 64 * c + t
                z = [[x[ex + 512 * k] for k in range(8)]]
                special_round(z, 9, ex, tab, False)
                for k in range(8):
                    assert ybuf[k][0][cpad(ex)] is None
                    ybuf[k][0][cpad(ex)] = z[0][k]
        for c in range(CL):
            for t in range(TH):
                st[c, t] = [[ybuf[c][0][cpad(ypos(1, t, r))] for r in range(8)]]
                special_round(st[c, t], 6, 512 * c + ypos(1, t, 0), tab, False)
        for ya, yb, p in ((1, 2, 3), (2, 3, 0)):
            transpose(st, ybuf, ya, yb, 1)
            for c in range(CL):
                for t in range(TH):
                    special_round(st[c, t], p, 512 * c + ypos(yb, t, 0), tab, False)
        transpose(st, ybuf, 3, 1, 1)
        for c in range(CL):
            for t in range(TH):
                for r in range(8):
                    out[512 * c + ypos(1, t, r)] = st[c, t][0][r]
    assert all(v is not None for v in out)
    return out


@pytest.mark.parametrize("m", [12, 14])
def test_special_cluster_schedule(m):
    rng = np.random.default_rng(50 + m)
    tab, x = cvec(rng, 1 << m), cvec(rng, 4096)
    for fwd in (True, False):
        assert special_cluster(x, tab, fwd) == plain_special(x, tab, fwd)


# ------------------------------------------- the split product's spectrum order
def test_split_permuted_order_is_window8_addressing():
    # the forward pass's last round holds tile point 16 t + r in thread t,
    # register r (window 0); it is stored at the window-8 address t + 256 r,
    # which the all-ones spectrum U reproduces as (e >> 4) + 256 (e & 15)
    def e_base(w, t):
        return (t & ((1 << w) - 1)) | ((t >> w) << (w + 4))

    seen = set()
    for t in range(256):
        for r in range(16):
            e = e_base(0, t) + r
            stored = e_base(8, t) + (r << 8)
            assert stored == (e >> 4) + 256 * (e & 15)
            seen.add(stored)
    assert seen == set(range(4096))
