"""Known-answer tests of the oracle's canonical 2-D DFT (no reference test pins
the FFTW boundary, so the transform is pinned to the DFT definition)."""
import numpy as np
import pytest

import pyoracle as po


def naive_dft2(a, sign):
    a = np.asarray(a, dtype=np.clongdouble)
    nx, ny = a.shape
    kx = np.arange(nx)
    ky = np.arange(ny)
    Fx = np.exp(sign * 2j * np.pi * np.outer(kx, kx).astype(np.longdouble) / nx)
    Fy = np.exp(sign * 2j * np.pi * np.outer(ky, ky).astype(np.longdouble) / ny)
    return Fx @ a @ Fy


@pytest.mark.parametrize("shape", [(8, 8), (6, 10), (16, 12), (30, 14), (2, 126), (40, 56)])
@pytest.mark.parametrize("forward", [True, False])
def test_against_naive_long_double(shape, forward):
    g = np.random.default_rng(1)
    a = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    got = po.canon_fft2d(a, forward)
    ref = naive_dft2(a, -1 if forward else +1)
    err = np.abs(got - ref.astype(np.complex128)).max() / np.abs(ref).max()
    assert err < 5e-14


@pytest.mark.parametrize("n", [256, 512, 768, 1080, 64 * 7])
def test_against_numpy_pocketfft(n):
    g = np.random.default_rng(n)
    a = g.standard_normal((n, 64)) + 1j * g.standard_normal((n, 64))
    f = po.canon_fft2d(a, True)
    assert np.abs(f - np.fft.fft2(a)).max() / np.abs(f).max() < 1e-14
    b = po.canon_fft2d(a, False)
    assert np.abs(b - np.fft.ifft2(a) * a.size).max() / np.abs(b).max() < 1e-14


def test_delta_and_constant():
    n = 64
    d = np.zeros((n, n), complex)
    d[0, 0] = 1
    assert np.array_equal(po.canon_fft2d(d), np.ones((n, n)))
    c = np.ones((n, n), complex)
    f = po.canon_fft2d(c)
    assert f[0, 0] == n * n and np.abs(f).sum() == n * n


def test_parseval_and_round_trip():
    g = np.random.default_rng(3)
    a = g.standard_normal((96, 80)) + 1j * g.standard_normal((96, 80))
    f = po.canon_fft2d(a, True)
    assert abs((np.abs(f) ** 2).sum() / a.size - (np.abs(a) ** 2).sum()) < 1e-10 * (np.abs(a) ** 2).sum()
    back = po.canon_fft2d(f, False) / a.size
    assert np.abs(back - a).max() < 1e-13


@pytest.mark.parametrize("n", [134, 262, 3 * 127])
def test_large_prime_factors(n):
    """Prime factors above 64 (67, 131, 127): the prime butterfly's direct sum."""
    g = np.random.default_rng(n)
    a = g.standard_normal((n, 8)) + 1j * g.standard_normal((n, 8))
    f = po.canon_fft2d(a, True)
    assert np.abs(f - np.fft.fft2(a)).max() / np.abs(f).max() < 1e-12


def test_unsupported_prime():
    with pytest.raises(ValueError):
        po.canon_fft2d(np.zeros((1031, 4), complex))   # 1031: a prime above 1021
