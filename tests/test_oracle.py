"""CPU tests: pin the oracle (oracle/oracle.c) against the reference's own CPU
code — through the committed golden vectors in tests/golden/ and, where it was
built, the reference build in oracle/_ref — and against exact schoolbook
products and known-answer identities."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name), allow_pickle=False)


@pytest.mark.parametrize("sfx,T", [("f64", np.float64), ("f32", np.float32)])
def test_fft_tables_match_golden(O, sfx, T):
    g = load(f"fft_tables_{sfx}.npz")
    r, ri, ninv = O.fft_tables(int(g["n"]), sfx)
    assert np.array_equal(r.view(T), g["rev_roots"])
    assert np.array_equal(ri.view(T), g["rev_inv_roots"])
    assert ninv == g["n_inverse"][0]


@pytest.mark.parametrize("sfx,T", [("f64", np.float64), ("f32", np.float32)])
def test_ffnt_tables_match_golden(O, sfx, T):
    g = load(f"ffnt_tables_{sfx}.npz")
    tabs = O.ffnt_tables(int(g["n"]), sfx)
    for got, key in zip(tabs, ["rev_roots", "rev_inv_roots", "twist", "untwist"]):
        assert np.array_equal(got.view(T), g[key]), key


def test_cpu_fft_matches_golden_bitwise(O):
    g = load("cpu_fft_f64.npz")
    n = int(g["n"])
    y = O.cpu_fft(n, g["x"], "f64")
    assert np.array_equal(y, g["fft"])
    z = O.cpu_fft(n, y, "f64", inverse=True)
    assert np.array_equal(z, g["ifft_of_fft"])


def test_ffnt_mult_matches_golden_and_schoolbook(O):
    g = load("ffnt_mult_f64.npz")
    n = int(g["n"])
    out = O.cpu_ffnt_mult(n, g["a"], g["b"], "f64")
    assert np.array_equal(out, g["out"])
    exact = O.wrap64(O.schoolbook(g["a"].astype(np.int64), g["b"].astype(np.int64), O.NEGACYCLIC))
    assert np.array_equal(out.view(np.int64), exact)


def test_linear_cpu_example_golden_is_exact(O):
    # the CPU-example product: N = 2^12, coefficients in [-2^15, 2^15): the reference's FFT<double>
    # product rounds to the exact schoolbook product.
    g = load("linear_f64.npz")
    exact = O.wrap64(O.schoolbook(g["a"], g["b"], O.LINEAR))
    assert np.array_equal(g["out"], exact)


def test_gpu_semantics_linear_product_matches_golden(O):
    # The GPU_FFT(R_R) pipeline restated in the oracle gives the same rounded
    # product as the reference's CPU example on the same inputs.
    g = load("linear_f64.npz")
    n = int(g["n"])
    M = 2 * n
    roots, inv_roots, ninv = O.fft_tables(n, "f64")
    real = np.zeros((2, M))
    real[0, :n] = g["a"]
    real[1, :n] = g["b"]
    temp = np.zeros(2 * M, np.complex128)
    real, temp = O.gpu_fft_r2r(real.ravel(), temp, roots, 13, 0, 1, 1.0, 2, False)
    real, temp = O.gpu_fft_r2r(real, temp, inv_roots, 13, 1, 1, complex(ninv), 1, True)
    assert np.array_equal(np.rint(real[:M]).astype(np.int64), g["out"])


def test_schoolbook_mod7_matches_reference(O):
    g = load("schoolbook_q7.npz")
    a = g["a"].astype(np.int64)
    b = g["b"].astype(np.int64)
    lin = O.schoolbook(a, b, O.LINEAR)
    assert [int(v) % 7 for v in lin] == list(g["linear"])
    neg = O.schoolbook(a, b, O.NEGACYCLIC)
    # the reference computes (lo - hi) % q in unsigned 64-bit arithmetic
    want = [((int(v)) & ((1 << 64) - 1)) % 7 for v in neg]
    assert want == [int(v) for v in g["negacyclic"]]


def test_reference_build_agrees_with_oracle(O):
    R = O.ref()
    if R is None:
        pytest.skip("reference CPU build not present (oracle/_ref)")
    rng = np.random.default_rng(7)
    for sfx, T in (("f64", np.float64), ("f32", np.float32)):
        for n in (64, 1 << 13):
            h = n // 2
            tabs = [np.zeros(2 * h, T) for _ in range(4)]
            getattr(R, f"ref_ffnt_tables_{sfx}")(n, *tabs)
            for got, want in zip(O.ffnt_tables(n, sfx), tabs):
                assert np.array_equal(got.view(T), want)
        n = 1 << 12
        a = rng.integers(0, 1 << 10, n).astype(np.uint64)
        b = rng.integers(0, 1 << 10, n).astype(np.uint64)
        ro = np.zeros(n, np.uint64)
        getattr(R, f"ref_ffnt_mult_{sfx}")(n, a, b, ro)
        assert np.array_equal(O.cpu_ffnt_mult(n, a, b, sfx), ro)


def test_forward_convention_is_plus_sign_bitreversed(O):
    # forward output[r] = sum_j x_j e^{+2 pi i j k / M} at k = bitrev(r)
    n = 512
    M = 2 * n
    x = np.random.default_rng(3).standard_normal(M) + 1j * np.random.default_rng(4).standard_normal(M)
    y = O.cpu_fft(n, x, "f64")
    br = np.array([O.lib().orc_bitreverse(i, 10) for i in range(M)])
    np.testing.assert_allclose(y, (M * np.fft.ifft(x))[br], rtol=0, atol=1e-9)


def test_delta_impulse_gives_all_ones(O):
    n = 256
    x = np.zeros(2 * n, np.complex128)
    x[0] = 1
    y = O.cpu_fft(n, x, "f64")
    assert np.array_equal(y, np.ones(2 * n, np.complex128))


@pytest.mark.parametrize("n", [16, 256, 4096])
def test_monomial_products_negacyclic(O, n):
    # X^a * X^b = +-X^{(a+b) mod n} in Z[X]/(X^n+1), through the FFNT oracle
    rng = np.random.default_rng(n)
    for _ in range(4):
        i, j = rng.integers(0, n, 2)
        a = np.zeros(n, np.uint64)
        b = np.zeros(n, np.uint64)
        a[i] = 1
        b[j] = 1
        out = O.cpu_ffnt_mult(n, a, b, "f64").view(np.int64)
        want = np.zeros(n, np.int64)
        k = (i + j) % n
        want[k] = 1 if i + j < n else -1
        assert np.array_equal(out, want)


def test_parseval(O):
    n = 1024
    M = 2 * n
    x = np.random.default_rng(5).standard_normal(M) + 0j
    y = O.cpu_fft(n, x, "f64")
    assert abs(np.sum(np.abs(y) ** 2) - M * np.sum(np.abs(x) ** 2)) < 1e-8 * M * np.sum(np.abs(x) ** 2)


def test_balanced_digits_roundtrip(O):
    x = np.random.default_rng(6).integers(0, 1 << 24, 1000)
    for w, k in ((6, 4), (8, 3), (12, 2)):
        d = O.balanced_digits(x, w, k)
        assert np.all(d[:-1] >= -(1 << (w - 1))) and np.all(d[:-1] < (1 << (w - 1)))
        rec = sum(d[l].astype(np.int64) << (w * l) for l in range(k))
        assert np.array_equal(rec, x)


def test_special_fft_restatement_known_answer(O):
    # GPU_Special_FFT's network (fft.cu:727-1007) with the natural table
    # t + j -> e^{i pi j / t}: the forward of a bit-reversed vector is the
    # +sign DFT, and the conjugate table with 1/M inverts it
    n = 6
    M = 1 << n
    tab = np.zeros(M, np.complex128)
    for e in range(n):
        t = 1 << e
        tab[t:2 * t] = np.exp(1j * np.pi * np.arange(t) / t)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    br = np.array([int(format(i, f"0{n}b")[::-1], 2) for i in range(M)])
    y = O.gpu_special_fft(x[br].copy(), tab, n, 0, 1.0, 1)
    assert np.abs(y - M * np.fft.ifft(x)).max() < 1e-12
    z = O.gpu_special_fft(y, np.conj(tab), n, 1, 1.0 / M, 1)
    assert np.abs(z - x[br]).max() < 1e-13
