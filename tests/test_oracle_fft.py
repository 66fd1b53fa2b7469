"""The oracle's FFT (replacing cuFFT, density.h:67-74) against numpy.fft."""
import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 12, 30, 48, 64, 96, 100, 128, 150, 200])
def test_fft1d_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    scale = np.abs(x).sum()
    assert np.abs(O.fft1d(x, -1) - np.fft.fft(x)).max() <= 1e-14 * scale
    assert np.abs(O.fft1d(x, +1) - np.fft.ifft(x) * n).max() <= 1e-14 * scale


def test_fft1d_rejects_large_prime():
    with pytest.raises(ValueError):
        O.fft1d(np.ones(11), -1)


@pytest.mark.parametrize("m", [(8, 8, 8), (12, 10, 6), (6, 5, 9), (16, 12, 15), (4, 4, 1), (3, 7, 2)])
def test_r2c_c2r_match_numpy(m):
    rng = np.random.default_rng(sum(m))
    g = O.Grid(m, (4.0, 4.0, 4.0))
    a = rng.normal(size=m)
    h = g.r2c(a)
    ref = np.fft.rfftn(a)
    assert np.abs(h - ref).max() <= 1e-13 * np.abs(a).sum()
    back = g.c2r(h) / g.M
    assert np.abs(back - a).max() <= 1e-13
    # c2r semantics: imaginary parts of self-conjugate bins are ignored
    h2 = ref.copy()
    h2[..., 0] += 1j * 3.0
    assert np.abs(g.c2r(h2) - g.c2r(ref)).max() <= 1e-10


def test_ksq_table_matches_definition():
    m, D = (6, 5, 8), (2.0, 3.0, 4.0)
    g = O.Grid(m, D)
    ksq = g.ksq()
    k0 = np.fft.fftfreq(m[0], 1 / m[0])
    k1 = np.fft.fftfreq(m[1], 1 / m[1])
    k2 = np.arange(m[2] // 2 + 1)
    K0, K1, K2 = np.meshgrid(k0, k1, k2, indexing="ij")
    ref = 4 * np.pi ** 2 * (K0 ** 2 / D[0] ** 2 + K1 ** 2 / D[1] ** 2 + K2 ** 2 / D[2] ** 2)
    assert np.allclose(ksq, ref, rtol=1e-15, atol=1e-12)
