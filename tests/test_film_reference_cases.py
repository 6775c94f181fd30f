"""The film's sample splat against the reference's HdrRgbFilm and its sample filters.

* The reference's known answer, HdrRgbFilmTest.DevelopesToFrame (symmetric case,
  Engine/EngineTest/Source/Core/Filmic/HdrRgbFilm_test.cpp:60-104): a 1 x 2 film with the
  gaussian filter receives 0.7 at the sample window's corner + 0.2 px and 0.3 at + 0.4 px; pixel
  (0, 0) develops to (w1 0.7 + w2 0.3) / (w1 + w2), with w the filter at the pixel centre minus
  the sample position, equal in r, g and b and non-zero.
* Every 4 x 4 filter, seeded samples over a 7 x 5 film's whole sample window: the (R, G, B, W)
  sums equal an FP64 restatement of HdrRgbFilm::addRgbSample (HdrRgbFilm.cpp:82-123) with the
  reference's filter functions (SampleFilter.cpp:12-59, TGaussian2D, TMitchellNetravaliCubic2D,
  TBlackmanHarris2D), within 2e-5 absolute + 1e-5 relative: the GPU evaluates the weights in
  FP32 (the reference in FP64), and about 80 samples reach each pixel.
* The filters' support ends two pixels from the sample: at the corner of the support every filter
  is zero up to rounding (at most 1e-6), and pixels beyond it receive nothing.

The GPU side goes through pgpu_film_splat, which runs the renderer's own deposit function.
"""

import numpy as np
import pytest

HALF = 2.0   # half size of the 4 x 4 filters, in pixels


def _gaussian(x, y):
    """TGaussian2D(sigma 0.5, amplitude 1) sunk by its value at (2, 2) (SampleFilter.cpp:19-36)."""
    edge = np.exp(-(HALF * HALF + HALF * HALF) / (2 * 0.25))
    return np.maximum(np.exp(-(x * x + y * y) / (2 * 0.25)) - edge, 0.0)


def _mn1(x, b=1.0 / 3.0, c=1.0 / 3.0):
    a = np.abs(x)
    inner = ((12 - 9 * b - 6 * c) * a ** 3 + (-18 + 12 * b + 6 * c) * a ** 2 + (6 - 2 * b)) / 6
    outer = ((-b - 6 * c) * a ** 3 + (6 * b + 30 * c) * a ** 2 + (-12 * b - 48 * c) * a + (8 * b + 24 * c)) / 6
    return np.where(a < 1, inner, np.where(a < 2, outer, 0.0))


def _bh1(n):
    return (0.35875 - 0.48829 * np.cos(2 * np.pi * n) + 0.14128 * np.cos(4 * np.pi * n)
            - 0.01174 * np.cos(6 * np.pi * n))


FILTERS = {
    "gaussian": _gaussian,
    "mitchell-netravali": lambda x, y: _mn1(x) * _mn1(y),
    "blackman-harris": lambda x, y: _bh1((x / HALF + 1) * 0.5) * _bh1((y / HALF + 1) * 0.5),
}


def film_add_samples(sample_filter, width, height, samples):
    """FP64 restatement of HdrRgbFilm::addRgbSample over an effective window [0, W) x [0, H)."""
    f = FILTERS[sample_filter]
    sums = np.zeros((height, width, 4), np.float64)
    for xs, ys, r, g, b in samples.astype(np.float64):
        lo_x, hi_x = max(xs - HALF, 0.0), min(xs + HALF, float(width))
        lo_y, hi_y = max(ys - HALF, 0.0), min(ys + HALF, float(height))
        for y in range(int(np.ceil(lo_y - 0.5)), int(np.floor(hi_y - 0.5)) + 1):
            for x in range(int(np.ceil(lo_x - 0.5)), int(np.floor(hi_x - 0.5)) + 1):
                w = float(f(x - (xs - 0.5), y - (ys - 0.5)))
                sums[y, x] += (r * w, g * w, b * w, w)
    return sums


def _seeded_samples(width, height, n, seed):
    rng = np.random.default_rng(seed)
    xy = rng.uniform([0.5 - HALF, 0.5 - HALF], [width - 0.5 + HALF, height - 0.5 + HALF], size=(n, 2))
    rgb = rng.uniform(0.0, 1.0, size=(n, 3))
    return np.concatenate([xy, rgb], 1).astype(np.float32)


def test_restatement_reproduces_the_reference_known_answer():
    """The FP64 restatement itself gives the reference test's answer (checked without a GPU)."""
    x0 = 0.5 - HALF   # sample window minimum of a 1 x 2 film with a 4 x 4 filter
    smp = np.array([[x0 + 0.2, x0 + 0.2, 0.7, 0.7, 0.7], [x0 + 0.4, x0 + 0.4, 0.3, 0.3, 0.3]])
    sums = film_add_samples("gaussian", 1, 2, smp)
    w1, w2 = _gaussian(0.5 - smp[0, 0], 0.5 - smp[0, 1]), _gaussian(0.5 - smp[1, 0], 0.5 - smp[1, 1])
    assert w1 > 0 and w2 > 0 and w1 != w2
    assert sums[0, 0, 0] / sums[0, 0, 3] == pytest.approx((w1 * 0.7 + w2 * 0.3) / (w1 + w2), rel=1e-12)


@pytest.mark.gpu
def test_gpu_film_reference_known_answer(gpu_lib):
    import photon_gpu

    x0 = 0.5 - HALF
    smp = np.array([[x0 + 0.2, x0 + 0.2, 0.7, 0.7, 0.7], [x0 + 0.4, x0 + 0.4, 0.3, 0.3, 0.3]], np.float32)
    sums = photon_gpu.film_splat("gaussian", 1, 2, smp)
    pixel = sums[0, 0, :3] / sums[0, 0, 3]
    assert pixel[0] == pixel[1] == pixel[2]
    assert np.all(pixel != 0)
    s64 = smp.astype(np.float64)
    w1, w2 = _gaussian(0.5 - s64[0, 0], 0.5 - s64[0, 1]), _gaussian(0.5 - s64[1, 0], 0.5 - s64[1, 1])
    assert pixel[0] == pytest.approx((w1 * 0.7 + w2 * 0.3) / (w1 + w2), rel=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("sample_filter", list(FILTERS))
def test_gpu_film_splat_matches_restatement(gpu_lib, sample_filter):
    import photon_gpu

    width, height = 7, 5
    smp = _seeded_samples(width, height, 400, seed=11)
    got = photon_gpu.film_splat(sample_filter, width, height, smp)
    want = film_add_samples(sample_filter, width, height, smp)
    assert np.allclose(got, want, rtol=1e-5, atol=2e-5), float(np.abs(got - want).max())
    # every pixel is reached: the sample window covers the whole filter support of each one
    assert np.all(want[..., 3] != 0)


@pytest.mark.gpu
@pytest.mark.parametrize("sample_filter", list(FILTERS))
def test_gpu_film_filter_support_ends_at_two_pixels(gpu_lib, sample_filter):
    import photon_gpu

    # a sample at (2.5, 2.5): pixel (0, 0) (centre (0.5, 0.5)) lies on the corner of its support,
    # where every filter falls to zero up to rounding; pixels 3 px away lie outside it
    smp = np.array([[2.5, 2.5, 1.0, 1.0, 1.0]], np.float32)
    sums = photon_gpu.film_splat(sample_filter, 6, 6, smp)
    assert abs(sums[0, 0, 3]) <= 1e-6
    assert np.all(sums[5, :, :] == 0.0) and np.all(sums[:, 5, :] == 0.0)
    assert sums[2, 2, 3] == pytest.approx(FILTERS[sample_filter](0.0, 0.0), rel=1e-5)


@pytest.mark.gpu
def test_gpu_film_splat_rejects_bad_arguments(gpu_lib):
    import ctypes

    import photon_gpu

    smp = np.zeros((1, 5), np.float32)
    sums = np.zeros((1, 1, 4), np.float64)
    lib = photon_gpu.load()
    p_smp = smp.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    p_sums = sums.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert lib.pgpu_film_splat(0, 1, 1, p_smp, 1, p_sums) != 0   # box: not splatted
    assert lib.pgpu_film_splat(1, 0, 1, p_smp, 1, p_sums) != 0   # empty film
    assert lib.pgpu_film_splat(1, 1, 1, None, 1, p_sums) != 0    # samples missing
    assert lib.pgpu_film_splat(1, 1, 1, p_smp, 0, p_sums) == 0   # no samples: zero sums
    assert np.all(sums == 0.0)
