"""The oracle's transforms follow the reference FFT wrappers (rft_buff.f:24-86,
cft_buff.f:1-65): checked against numpy.fft and a direct O(n^2) DFT."""
import numpy as np
import pytest

from oracle import oracle as O

LENGTHS = [6, 12, 18, 24, 48, 64, 96, 192, 384, 768]


def naive_dft(x, sign):
    n = x.shape[-1]
    k = np.arange(n)
    return x @ np.exp(sign * 2j * np.pi * np.outer(k, k) / n)


@pytest.mark.parametrize("n", LENGTHS)
def test_cft_forward_scaled_inverse_unscaled(n):
    rng = np.random.default_rng(n)
    m = 3
    x = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    c = np.empty(2 * n * m)
    c[0::2], c[1::2] = x.ravel().real, x.ravel().imag
    f = O.cft(c.copy(), n, 2, 2 * n, m, -1)
    X = (f[0::2] + 1j * f[1::2]).reshape(m, n)
    np.testing.assert_allclose(X, np.fft.fft(x, axis=1) / n, atol=1e-14, rtol=0)
    b = O.cft(f, n, 2, 2 * n, m, +1)
    np.testing.assert_allclose((b[0::2] + 1j * b[1::2]).reshape(m, n), x, atol=1e-13, rtol=0)


@pytest.mark.parametrize("n", [6, 12, 18, 24, 48])
def test_cft_against_naive_dft(n):
    rng = np.random.default_rng(1)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    c = np.empty(2 * n)
    c[0::2], c[1::2] = x.real, x.imag
    b = O.cft(c, n, 2, 2 * n, 1, +1)
    np.testing.assert_allclose(b[0::2] + 1j * b[1::2], naive_dft(x, +1), atol=1e-12)


@pytest.mark.parametrize("n", LENGTHS)
def test_rft_fftpack_storage(n):
    rng = np.random.default_rng(n + 7)
    m = 4
    isa = n + 2
    x = rng.standard_normal((m, n))
    c = np.zeros((m, isa))
    c[:, :n] = x
    f = O.rft(c.ravel(), n, isa, m, -1).reshape(m, isa)
    ref = np.fft.rfft(x, axis=1) / n
    np.testing.assert_allclose(f[:, 0::2] + 1j * f[:, 1::2], ref, atol=1e-15)
    assert np.all(f[:, 1] == 0.0) and np.all(f[:, n + 1] == 0.0)   # Im cc(0), Im cc(n/2)
    b = O.rft(f.ravel(), n, isa, m, +1).reshape(m, isa)
    np.testing.assert_allclose(b[:, :n], x, atol=1e-13)


def test_rft_inverse_ignores_imag_of_mean_and_nyquist():
    n = 24
    rng = np.random.default_rng(3)
    c = rng.standard_normal(n + 2)
    a = O.rft(c.copy(), n, n + 2, 1, +1)[:n]
    c2 = c.copy()
    c2[1] = 0.0
    c2[n + 1] = 0.0
    b = O.rft(c2, n, n + 2, 1, +1)[:n]
    np.testing.assert_array_equal(a, b)


def test_bad_length_rejected():
    with pytest.raises(AssertionError):
        O.cft(np.zeros(2 * 10), 10, 2, 20, 1, -1)
