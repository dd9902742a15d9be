"""The device FFT (mmp_dft: Forward_DFT / Inverse_DFT on the GPU) against numpy.fft,
every supported size, both precisions, single-CTA and cluster rows."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("fp64", [True, False])
def test_forward_inverse(mmp, n, fp64):
    rng = np.random.default_rng(n + fp64)
    rows = 3
    x = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
    y = mmp.dft(x, inverse=False, fp64=fp64)
    ref = np.fft.fft(x, axis=-1)
    err = np.abs(y - ref).max() / np.abs(ref).max()
    tol = 1e-13 if fp64 else 2e-6
    assert err < tol, f"forward n={n} fp64={fp64}: {err:.3e}"
    z = mmp.dft(y, inverse=True, fp64=fp64)
    err2 = np.abs(z - x).max() / np.abs(x).max()
    assert err2 < tol, f"inverse n={n} fp64={fp64}: {err2:.3e}"


def test_impulses(mmp):
    # exact known answers: DFT of a unit impulse at t0 is exp(-2 pi i k t0 / n)
    n = 4096
    for t0 in (0, 1, 7, n // 2, n - 1):
        x = np.zeros(n, complex)
        x[t0] = 1.0
        y = mmp.dft(x, fp64=True)
        k = np.arange(n)
        assert np.allclose(y, np.exp(-2j * np.pi * k * t0 / n), atol=1e-13)
