"""CPU checks of the index schedule of split_tile_kernel
(gpu-fft_b200/csrc/gf_split_tile.cuh), restated in Python from the kernel's
layout rules:

* a 2048-point tile, teams of 128 threads x 16 registers; register window W
  holds e-bits [W, W+4) with e = ebase_W(t) + (r << W), ebase_W(t) = (t mod
  2^W) | ((t >> W) << (W + 4));
* forward rounds on e-bits [7,11), [3,7), [0,3) (windows 7, 3, 0), each team
  transposing in place through its own slot with point e at the padded
  position spad(e) = e + (e >> 4) (the bulk copy lands unpadded, in natural
  order, read by the first forward round only); the inverse runs the reverse
  order; stage u of the tile (e-bit 10 - u) uses table[(T << u) + (e >> (11 -
  u))] -- the engine's butterflies, so the rounds must reproduce the plain
  stage loop exactly;
* the kernel's per-thread address arithmetic (SlotAddr: a base plus a
  compile-time offset per register) equals spad of the window's points; after
  the forward stages point e sits at spad(e), which the group phase and the
  inverse's first read assume;
* every shared-memory and global index stays inside its buffer, every store
  after a load goes to the positions the thread just read (so only the
  barriers the kernel has are needed), and 8-byte accesses of each half-warp
  fall in distinct bank pairs (no bank conflicts);
* the centring spectrum U is read at the index the table kernel stored it at.
"""
import numpy as np
import pytest

LT, P, HT, R = 11, 2048, 128, 16


def ebase(w, t):
    return (t & ((1 << w) - 1)) | ((t >> w) << (w + 4))


SLOT = P + P // 16


def spad(e):
    return e + (e >> 4)


def slot_addr(w, t, r):
    """SlotAddr<W>: spad(ebase) plus the compile-time offset of register r."""
    return spad(ebase(w, t)) + (r << w) + ((r << w) >> 4)


def ct(x, y, w):
    return x + w * y, x - w * y


def gs(x, y, w):
    return x + y, (x - y) * w


def plain(x, tab, T, fwd):
    """The engine's stage loop over one tile: stage u on e-bit 10 - u."""
    x = list(x)
    for u in (range(LT) if fwd else range(LT - 1, -1, -1)):
        q = LT - 1 - u
        for e in range(P):
            if e >> q & 1:
                continue
            w = tab[(T << u) + (e >> (q + 1))]
            x[e], x[e + (1 << q)] = (ct if fwd else gs)(x[e], x[e + (1 << q)], w)
    return x


def kround(regs, fwd, w, lo, hi, tab, T, eb):
    """split_tile's round<FWD, W, LO, HI> on one thread's 16 registers."""
    a, rb = lo - w, hi - lo
    ws = {}
    for k in range(rb):
        pb = (a + rb - 1 - k) if fwd else (a + k)
        q = w + pb
        u = LT - 1 - q
        nt = 1 << (3 - pb)
        base = (T << u) + (eb >> (q + 1))
        assert base % nt == 0  # paired (16-byte) twiddle loads stay aligned
        for h in range(nt):
            assert 0 <= base + h < len(tab)
            ws[pb, h] = tab[base + h]
    for k in range(rb):
        pb = (a + rb - 1 - k) if fwd else (a + k)
        for r in range(R):
            if r >> pb & 1:
                continue
            regs[r], regs[r | 1 << pb] = (ct if fwd else gs)(regs[r], regs[r | 1 << pb], ws[pb, r >> (pb + 1)])


def banks_ok(addrs):
    """8-byte accesses of one half-warp (16 consecutive threads) hit distinct bank pairs."""
    for h0 in range(0, len(addrs), 16):
        banks = set()
        for a in addrs[h0:h0 + 16]:
            b = (2 * a) % 32
            assert b not in banks and b + 1 not in banks, "bank conflict"
            banks.update((b, b + 1))
    return True


class Team:
    """One team's 128 threads on one slot; loads record the positions each
    thread read so that a store without a barrier is checked to hit only them."""

    def __init__(self, slot):
        self.slot = slot
        self.read = {}

    def load(self, w, natural=False):
        st = []
        for t in range(HT):
            pos = [(t + (r << 7)) if natural else slot_addr(w, t, r) for r in range(R)]
            for r, q in enumerate(pos):
                assert 0 <= q < (P if natural else SLOT)
                if not natural:
                    assert q == spad(ebase(w, t) + (r << w))
            self.read[t] = set(pos)
            st.append([self.slot[q] for q in pos])
        for r in range(R):
            banks_ok([(t + (r << 7)) if natural else slot_addr(w, t, r) for t in range(HT)])
        return st

    def store(self, st, w, barrier_before):
        written = set()
        for t in range(HT):
            pos = [slot_addr(w, t, r) for r in range(R)]
            if not barrier_before:
                assert set(pos) == self.read[t], "store outside the thread's own positions needs a barrier"
            for r, q in enumerate(pos):
                assert q not in written
                written.add(q)
                self.slot[q] = st[t][r]
        for r in range(R):
            banks_ok([slot_addr(w, t, r) for t in range(HT)])
        assert len(written) == P and max(written) < SLOT


def kernel_forward(tile_in, tab, T):
    """slot (unpadded natural order, as bulk-copied) -> slot (padded order), in place."""
    tm = Team(list(tile_in) + [None] * (SLOT - P))
    st = tm.load(7, natural=True)
    for t in range(HT):
        kround(st[t], True, 7, 7, 11, tab, T, ebase(7, t))
    tm.store(st, 7, barrier_before=True)  # the kernel's barrier after the natural-order read
    st = tm.load(3)
    for t in range(HT):
        kround(st[t], True, 3, 3, 7, tab, T, ebase(3, t))
    tm.store(st, 3, barrier_before=False)
    st = tm.load(0)
    for t in range(HT):
        kround(st[t], True, 0, 0, 3, tab, T, ebase(0, t))
    tm.store(st, 0, barrier_before=False)
    return tm.slot


def kernel_inverse(slot, tab, T):
    """slot (padded order) -> the group tile in natural order (global store)."""
    tm = Team(list(slot))
    st = tm.load(0)
    for t in range(HT):
        kround(st[t], False, 0, 0, 3, tab, T, ebase(0, t))
    tm.store(st, 0, barrier_before=False)
    st = tm.load(3)
    for t in range(HT):
        kround(st[t], False, 3, 3, 7, tab, T, ebase(3, t))
    tm.store(st, 3, barrier_before=False)
    st = tm.load(7)
    for t in range(HT):
        kround(st[t], False, 7, 7, 11, tab, T, ebase(7, t))
    out = [None] * P
    for t in range(HT):
        for r in range(R):
            e = t + (r << 7)  # window 7: e = ebase_7(t) + (r << 7)
            assert e == ebase(7, t) + (r << 7) and out[e] is None
            out[e] = st[t][r]
    return out




@pytest.mark.parametrize("m,T", [(15, 0), (15, 13), (14, 7), (13, 3)])
def test_rounds_match_the_stage_loop(m, T):
    rng = np.random.default_rng(7 + m + T)
    M = 1 << m
    tab = rng.standard_normal(M // 2) + 1j * rng.standard_normal(M // 2)
    itab = rng.standard_normal(M // 2) + 1j * rng.standard_normal(M // 2)
    x = list(rng.standard_normal(P) + 1j * rng.standard_normal(P))
    slot = kernel_forward(x, tab, T)
    want = plain(x, tab, T, True)
    # the slot holds point e at position spad(e)
    got = [slot[spad(e)] for e in range(P)]
    np.testing.assert_array_equal(np.array(got), np.array(want))
    y = kernel_inverse(slot, itab, T)
    np.testing.assert_array_equal(np.array(y), np.array(plain(want, itab, T, False)))


def test_group_phase_points_cover_the_slot():
    seen = np.zeros(P, int)
    for tid in range(512):
        for i in range(P // 512):
            seen[tid + 512 * i] += 1
    assert (seen == 1).all()
    # each warp's accesses (32 consecutive points at their padded positions) are conflict-free
    for i in range(P // 512):
        banks_ok([spad(tid + 512 * i) for tid in range(512)])


@pytest.mark.parametrize("m", [13, 14, 15])
def test_centring_spectrum_index(m):
    """The kernel reads U for point e of tile T at the index ffnt_tables_kernel
    stored it at (4096-point tiles permuted e -> (e >> 4) + 256 (e & 15))."""
    M = 1 << m
    stored = {}
    for i in range(M):
        pu = ((i & ~4095) | ((i & 4095) >> 4) | ((i & 15) << 8)) if m > 12 else i
        stored[pu] = i
    assert sorted(stored) == list(range(M))
    for T in range(M >> LT):
        for e in range(0, P, 37):
            j = (T << LT) + e
            ju = (j & ~4095) | ((j & 4095) >> 4) | ((j & 15) << 8)
            assert stored[ju] == j


@pytest.mark.parametrize("m,k,W", [(15, 5, 256), (14, 5, 3), (13, 4, 1)])
def test_global_ranges(m, k, W):
    """Bulk-copy sources and group stores stay inside the workspace arrays:
    spec [2k][W][M] and group [2k-1][W][M] complex floats, tiles = W M / 2048."""
    M = 1 << m
    lg = m - LT
    tiles = W * (M >> LT)
    spec_len, group_len = 2 * k * W * M, (2 * k - 1) * W * M
    for tile in {0, tiles - 1, tiles // 2}:
        p, T = tile >> lg, tile & ((1 << lg) - 1)
        for tau in range(2 * k):
            src = (tau * W + p) * M + (T << LT)
            assert 0 <= src and src + P <= spec_len
            assert (src * 8) % 16 == 0  # 16-byte aligned bulk copy
        for s in range(2 * k - 1):
            dst = (s * W + p) * M + (T << LT)
            assert 0 <= dst and dst + P <= group_len


def test_shared_memory_budget():
    for k in range(1, 6):
        total = 2 * k * SLOT * 8 + 2 * 7 * HT * 16 + 2 * k * 8 + 64
        assert total <= 232448  # sharedMemPerBlockOptin of B200
        # slots, the staged twiddles and the mbarriers start on 16-byte boundaries
        assert (SLOT * 8) % 16 == 0 and (2 * k * SLOT * 8) % 16 == 0


def test_queue_issue_order():
    """Inverse items come first in the queue; a forward item of the next tile
    waits on the copy its slot's inverse item issues after reading the slot (the
    last limb slot is copied after the group phase). Because items are drawn in
    queue order, every awaited copy is issued by an item drawn earlier: no
    forward wait can depend on an item that no team has drawn."""
    for k in range(1, 6):
        ns, ng = 2 * k, 2 * k - 1
        for teams in (1, 2, 4):
            # simulate draws: team i draws items in turn; a forward item of slot
            # tau needs inverse item tau drawn before it (or tau == ns - 1)
            drawn = []
            for item in range(ng + ns):
                drawn.append(item)
                if item >= ng:
                    tau = item - ng
                    assert tau == ns - 1 or tau in drawn[:item]


def w0_pair(pb):
    return 0 if pb == 2 else (1 if pb == 1 else 3)


def stage_w0(tab, T):
    """stage_w0: the seven window-0 twiddle pairs of every thread, thread-major."""
    dst = [None] * (7 * HT)
    for p in range(7 * HT):
        if p < 128:
            u, q, t, j = 8, p, p, 0
        elif p < 384:
            u, q = 9, p - 128
            t, j = q >> 1, 1 + (q & 1)
        else:
            u, q = 10, p - 384
            t, j = q >> 2, 3 + (q & 3)
        src = (T << u) + 2 * q
        assert 0 <= src and src + 2 <= len(tab) and src % 2 == 0  # 16-byte aligned pair
        assert dst[j * HT + t] is None
        dst[j * HT + t] = (tab[src], tab[src + 1])
    return dst


@pytest.mark.parametrize("m,T", [(15, 0), (15, 15), (14, 5), (13, 3)])
def test_staged_window0_twiddles(m, T):
    """Every pair the window-0 round reads from the staged buffer is the pair it
    would have read from the table (stages u = 8, 9, 10 of the tile)."""
    M = 1 << m
    tab = np.arange(M // 2) + 0j  # entry index as its value
    st = stage_w0(tab, T)
    for t in range(HT):
        eb = ebase(0, t)
        for pb in (2, 1, 0):
            q = pb
            u = LT - 1 - q
            nt = 1 << (3 - pb)
            base = (T << u) + (eb >> (q + 1))
            for h in range(0, nt, 2):
                pair = st[(w0_pair(pb) + (h >> 1)) * HT + t]
                assert pair == (tab[base + h], tab[base + h + 1])
    # shared-memory reads of a warp (32 consecutive t, one 16-byte pair each) are contiguous
    for j in range(7):
        addrs = [j * HT + t for t in range(32)]
        assert addrs == list(range(addrs[0], addrs[0] + 32))


def stage_w37(tab, T):
    """stage_w37: entry 2^u + i = table[(T << u) + i], u = 0 .. 7, i < 2^u."""
    dst = [None] * 256
    for idx in range(1, 256):
        u = idx.bit_length() - 1
        src = (T << u) + (idx - (1 << u))
        assert 0 <= src < len(tab)
        dst[idx] = tab[src]
    return dst


@pytest.mark.parametrize("m,T", [(15, 0), (15, 15), (14, 7), (13, 2)])
def test_staged_outer_twiddles(m, T):
    """The window-7 and window-3 rounds read from the staged buffer exactly the
    entries they read from the table, and their paired (16-byte) reads are
    aligned."""
    M = 1 << m
    tab = np.arange(M // 2) + 0j
    st = stage_w37(tab, T)
    for w in (7, 3):
        for t in range(HT):
            eb = ebase(w, t)
            for pb in range(4):
                q = w + pb
                u = LT - 1 - q
                nt = 1 << (3 - pb)
                base_tab = (T << u) + (eb >> (q + 1))
                base_st = (1 << u) + (eb >> (q + 1))
                assert base_st + nt <= 256
                if nt >= 2:
                    assert base_st % 2 == 0
                for h in range(nt):
                    assert st[base_st + h] == tab[base_tab + h]
