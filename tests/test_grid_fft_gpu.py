"""The Toeplitz path's own grid FFT (imp_grid_fft, the replacement of the
reference's cuFFT C2C calls) against numpy's FP64 FFT, through the C-ABI:
forward and inverse (unnormalised), 1-D / 2-D / 3-D, batched, power-of-two
and mixed-radix lengths (3, 5, 7 and generic primes 11, 13, 67, 113), the
gridding-grid shapes of the benchmark configurations, host and device
pointers.  Tolerance 1e-6 relative L2 (FP32 arithmetic, exact twiddles)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-6


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


def run(pkg, ctx, x, shape, batch, inverse, device=False):
    n0, n1, n2 = shape
    xr = np.ascontiguousarray(x.real, np.float32).ravel()
    xi = np.ascontiguousarray(x.imag, np.float32).ravel()
    if device:
        from gpu_util import dev, host
        dr, di = dev(xr), dev(xi)
        pkg.grid_fft(ctx, dr, di, n0, n1, n2, batch, inverse)
        return (host(dr) + 1j * host(di)).reshape(x.shape)
    pkg.grid_fft(ctx, xr, xi, n0, n1, n2, batch, inverse)
    return (xr + 1j * xi.astype(np.float64)).reshape(x.shape)


def want(x, inverse):
    axes = (1, 2, 3)
    if inverse:
        return np.fft.ifftn(x, axes=axes) * np.prod([x.shape[a] for a in axes])
    return np.fft.fftn(x, axes=axes)


SHAPES = [(1, 1, 64), (1, 1, 4096), (1, 1, 7), (1, 1, 134), (1, 1, 226), (1, 16, 48),
          (1, 384, 384), (1, 72, 144), (1, 2048, 16), (4, 6, 10), (24, 24, 12), (8, 22, 26),
          (48, 48, 48), (30, 40, 2), (2, 572, 4)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("inverse", [False, True])
def test_grid_fft_matches_numpy(pkg, ctx, shape, inverse):
    rng = np.random.default_rng(sum(shape) + inverse)
    batch = 3 if np.prod(shape) < 20000 else 1
    x = rng.standard_normal((batch, *shape)) + 1j * rng.standard_normal((batch, *shape))
    got = run(pkg, ctx, x, shape, batch, inverse)
    ref = want(x, inverse)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print(f"{shape} x{batch} {'inverse' if inverse else 'forward'}: {err:.2e}")
    assert err < TOL


@pytest.mark.parametrize("shape", [(384, 384, 48), (128, 256, 256)])
def test_grid_fft_benchmark_grids(pkg, ctx, shape):
    """The 3-D F^H d gridding grid of the Toeplitz configuration (384 x 384 x
    48: radix 16, 8 and 3) and a 2N-grid shape, on device pointers."""
    rng = np.random.default_rng(7)
    x = (rng.standard_normal((1, *shape)) + 1j * rng.standard_normal((1, *shape))).astype(
        np.complex64)
    got = run(pkg, ctx, x, shape, 1, True, device=True)
    ref = want(x.astype(np.complex128), True)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print(f"{shape} inverse: {err:.2e}")
    assert err < TOL


def test_grid_fft_round_trip(pkg, ctx):
    rng = np.random.default_rng(3)
    shape = (16, 20, 30)
    x = rng.standard_normal((2, *shape)) + 1j * rng.standard_normal((2, *shape))
    y = run(pkg, ctx, x, shape, 2, False)
    z = run(pkg, ctx, y, shape, 2, True) / np.prod(shape)
    assert np.linalg.norm(z - x) / np.linalg.norm(x) < TOL


def test_grid_fft_rejects_unsupported(pkg, ctx):
    x = np.zeros(2 * 257, np.float32)
    with pytest.raises(pkg.ImpError, match="UNSUPPORTED"):
        pkg.grid_fft(ctx, x, x.copy(), 1, 1, 2 * 257)
    y = np.zeros(8192, np.float32)
    with pytest.raises(pkg.ImpError, match="UNSUPPORTED"):
        pkg.grid_fft(ctx, y, y.copy(), 1, 1, 8192)
