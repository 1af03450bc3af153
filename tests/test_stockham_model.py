"""The FFT schedule of the pass kernel (modelled in tests/stockham_model.py) against numpy."""
import numpy as np
import pytest

from stockham_model import pruned_pass, radices, stockham


@pytest.mark.parametrize("L", [2, 3, 4, 5, 7, 8, 12, 14, 16, 20, 28, 30, 40, 56, 64, 96, 100, 128, 160, 250, 256, 320, 384, 448, 640])
@pytest.mark.parametrize("inverse", [False, True])
def test_stockham_matches_numpy(L, inverse):
    rng = np.random.default_rng(L)
    x = rng.standard_normal((L, 3)) + 1j * rng.standard_normal((L, 3))
    got = stockham(x, inverse)
    ref = np.fft.ifft(x, axis=0) * L if inverse else np.fft.fft(x, axis=0)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())


def test_radix_plan():
    assert radices(320) == [8, 8, 5]
    assert radices(640) == [8, 8, 2, 5]
    assert radices(28) == [4, 7]
    with pytest.raises(ValueError):
        radices(22)


@pytest.mark.parametrize("N,L", [(4, 8), (5, 10), (7, 14), (7, 16), (9, 20), (14, 28), (16, 32)])
def test_pruned_maps(N, L):
    """pad / crop (Toeplitz) and centred-mode (NUFFT) position maps of the pass kernel."""
    rng = np.random.default_rng(N)
    x = rng.standard_normal((N, 2)) + 1j * rng.standard_normal((N, 2))
    # Toeplitz: pad N -> 2N at [0,N), keep [N-1, 2N-1) after a round trip
    if L == 2 * N:
        y = pruned_pass(x, L, N, 0, L, 0, False)
        assert np.allclose(y, np.fft.fft(x, n=L, axis=0), atol=1e-5)
        back = pruned_pass(y, L, L, 0, N, N - 1, True) / L
        ref = np.fft.ifft(np.fft.fft(x, n=L, axis=0), axis=0)[N - 1:2 * N - 1]
        assert np.allclose(back, ref, atol=1e-6)
    # NUFFT: modes i <-> k = i - N//2 placed at k mod L
    y = pruned_pass(x, L, N, -(N // 2), L, 0, True)
    g = np.zeros((L, 2), complex)
    g[(np.arange(N) - N // 2) % L] = x
    assert np.allclose(y, np.fft.ifft(g, axis=0) * L, atol=1e-5)
    z = pruned_pass(g, L, L, 0, N, -(N // 2), False)
    assert np.allclose(z, np.fft.fft(g, axis=0)[(np.arange(N) - N // 2) % L], atol=1e-5)
