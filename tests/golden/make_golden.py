"""Generate the golden fixtures in this directory from the REFERENCE's own CPU
code (oracle/_ref/libgpufft_ref_cpu.so, compiled from the reference sources by
oracle/Makefile). Run from the repository root:

    make -C oracle all && python tests/golden/make_golden.py

Each .npz holds seeded inputs and the reference's outputs for them:

* fft_tables_{f64,f32}.npz   FFT<T>(2048) ReverseRootTable / InverseReverseRootTable / n_inverse
* ffnt_tables_{f64,f32}.npz  FFNT<T>(4096) root / inverse-root / twist / untwist tables
* cpu_fft_f64.npz            FFT<double>(1024).fft and .ifft of a seeded complex vector
* ffnt_mult_f64.npz          FFNT<double>(4096).MULT of seeded inputs in [0, 2^12)
* linear_f64.npz             CPU-example product: N = 2^12, coefficients in [-2^15, 2^15),
                             FFT<double>(4096) fft/fft/product/ifft/round as in the
                             reference's CPU example (example/test_fft_cpu.cu)
* schoolbook_q7.npz          schoolbook_poly_multiplication (negacyclic, mod 7) and
                             schoolbook_poly_multiplication_without_reduction (mod 7), n = 64
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle as O  # noqa: E402

SEED = 20261203


def main():
    R = O.ref()
    if R is None:
        raise SystemExit("oracle/_ref not built: run `make -C oracle all` where the reference sources exist")
    rng = np.random.default_rng(SEED)
    for sfx, T in (("f64", np.float64), ("f32", np.float32)):
        n = 2048
        r, ri, ni = np.zeros(2 * n, T), np.zeros(2 * n, T), np.zeros(1, T)
        getattr(R, f"ref_fft_tables_{sfx}")(n, r, ri, ni)
        np.savez_compressed(os.path.join(HERE, f"fft_tables_{sfx}.npz"), n=n, rev_roots=r, rev_inv_roots=ri,
                            n_inverse=ni)
        n = 4096
        h = n // 2
        tabs = [np.zeros(2 * h, T) for _ in range(4)]
        getattr(R, f"ref_ffnt_tables_{sfx}")(n, *tabs)
        np.savez_compressed(os.path.join(HERE, f"ffnt_tables_{sfx}.npz"), n=n, rev_roots=tabs[0],
                            rev_inv_roots=tabs[1], twist=tabs[2], untwist=tabs[3])

    n = 1024
    x = (rng.standard_normal(2 * n) + 1j * rng.standard_normal(2 * n)).astype(np.complex128)
    fx = x.copy().view(np.float64).copy()
    R.ref_cpu_fft_f64(n, fx, 0)
    ix = fx.copy()
    R.ref_cpu_fft_f64(n, ix, 1)
    np.savez_compressed(os.path.join(HERE, "cpu_fft_f64.npz"), n=n, x=x, fft=fx.view(np.complex128),
                        ifft_of_fft=ix.view(np.complex128))

    n = 4096
    a = rng.integers(0, 1 << 12, n).astype(np.uint64)
    b = rng.integers(0, 1 << 12, n).astype(np.uint64)
    out = np.zeros(n, np.uint64)
    R.ref_ffnt_mult_f64(n, a, b, out)
    np.savez_compressed(os.path.join(HERE, "ffnt_mult_f64.npz"), n=n, a=a, b=b, out=out)

    n = 4096
    a = rng.integers(-(1 << 15), 1 << 15, n).astype(np.int64)
    b = rng.integers(-(1 << 15), 1 << 15, n).astype(np.int64)
    out = np.zeros(2 * n, np.int64)
    R.ref_linear_product_f64(n, a, b, out)
    np.savez_compressed(os.path.join(HERE, "linear_f64.npz"), n=n, a=a, b=b, out=out)

    n = 64
    a = rng.integers(0, 7, n).astype(np.uint64)
    b = rng.integers(0, 7, n).astype(np.uint64)
    neg = np.zeros(n, np.uint64)
    R.ref_schoolbook_negacyclic_u64(a, b, 7, n, neg)
    lin = np.zeros(2 * n, np.int32)
    R.ref_schoolbook_linear_i32(a.astype(np.int32), b.astype(np.int32), 7, n, lin)
    np.savez_compressed(os.path.join(HERE, "schoolbook_q7.npz"), n=n, a=a, b=b, negacyclic=neg, linear=lin)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
