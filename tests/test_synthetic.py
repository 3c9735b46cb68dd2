import numpy as np

from msgpu import synthetic as syn


def test_series_is_seeded_and_shaped():
    a = syn.make_series(65, 3, syn.HEX_513, seed=11)
    b = syn.make_series(65, 3, syn.HEX_513, seed=11)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    frames, clean, disp = a
    assert frames.shape == (3, 65, 65) and disp.shape == (3, 2, 65, 65)
    assert np.all(frames >= 0) and np.all(frames == np.round(frames))  # Poisson counts
    smooth = np.sqrt(disp[:, 0] ** 2 + disp[:, 1] ** 2)
    assert smooth.max() < syn.HEX_513.max_disp + 6 * syn.HEX_513.jitter
    assert clean.max() <= syn.HEX_513.peak * 1.2


def test_square_lattice_peak_spacing():
    n = 129
    y, x = np.mgrid[0:n, 0:n].astype(float)
    img = syn.clean_image(n, syn.SQUARE_257, x, y, amp_seed=1)
    row = img[int(4.1 + 12 * 3)]
    peaks = [i for i in range(1, n - 1) if row[i] > row[i - 1] and row[i] >= row[i + 1] and row[i] > 0.3]
    assert np.allclose(np.diff(peaks), 12, atol=1)


def test_psnr():
    a = np.zeros((8, 8))
    b = np.ones((8, 8))
    b[0, 0] = 0
    assert syn.psnr(b, b) == float("inf")
    assert 0 < syn.psnr(a, b) < 10
