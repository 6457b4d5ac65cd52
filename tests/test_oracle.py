"""The oracle (oracle/, a CPU restatement of the reference path) pinned against
the reference's own known-answer tests and against scipy fixtures.  CPU only."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def sample_f64(n):
    """crates/lucem-ops/src/test_support.rs:10-12."""
    i = np.arange(n, dtype=np.int64)
    return ((i * 7919 + 104729) % 1013).astype(np.float64) * 0.1 - 50.0


def host_pad_index(p, n, mode):
    """crates/lucem-ops/src/test_support.rs:21-46 (the reference's own f64 model)."""
    if 0 <= p < n:
        return p
    if mode == "constant":
        return None
    if mode == "nearest":
        return min(max(p, 0), n - 1)
    if mode == "wrap":
        return p % n
    if mode == "reflect":
        period = 2 * n
        r = p % period
        return r if r < n else period - 1 - r
    if n <= 1:
        return 0
    period = 2 * n - 2
    r = p % period
    return r if r < n else period - r


def host_correlate_1d(x, dims, w, axis, mode, cval, origin):
    """crates/lucem-ops/src/filter/convolve.rs:185-209."""
    outer = int(np.prod(dims[:axis], dtype=np.int64))
    length = dims[axis]
    inner = int(np.prod(dims[axis + 1:], dtype=np.int64))
    left = len(w) // 2 + origin
    out = np.zeros(len(x))
    for idx in range(len(x)):
        i = (idx // inner) % length
        base = idx - i * inner
        start = i - left
        s = 0.0
        for t, wt in enumerate(w):
            q = host_pad_index(start + t, length, mode)
            s += wt * (cval if q is None else x[base + q * inner])
        out[idx] = s
    return out


MODES = ["reflect", "constant", "nearest", "mirror", "wrap"]


def test_gaussian_kernel_sums(oracle):
    """crates/lucem-ops/src/filter/gaussian.rs:442-446."""
    k0 = oracle.gaussian_kernel_1d(2.0, 0, 8)
    assert abs(k0.sum() - 1.0) < 1e-12
    k1 = oracle.gaussian_kernel_1d(2.0, 1, 8)
    assert abs(k1.sum()) < 1e-12
    assert oracle.resolved_radius(4.0, 2.0) == 8
    assert len(oracle.gaussian_kernel_1d(2.0, 0, 8)) == 17


def test_constant_image_stays_constant(oracle):
    """crates/lucem-ops/src/filter/gaussian.rs:448-457."""
    x = sample_f64(17 * 21).reshape(17, 21).astype(np.float32)
    assert oracle.gaussian_blur(x, [1.5]).shape == (17, 21)
    ones = np.full((17, 21), 7.25, np.float32)
    oracle.assert_close(oracle.gaussian_blur(ones, [2.0]), np.full(ones.shape, 7.25), 1e-5, "constant")


@pytest.mark.parametrize("dims", [[1], [7], [32, 33], [5, 1, 9]])
def test_correlate_1d_matches_reference_host_model(oracle, dims):
    """crates/lucem-ops/src/filter/convolve.rs:211-228 restated."""
    x = sample_f64(int(np.prod(dims)))
    xf = x.astype(np.float32).reshape(dims)
    for axis in range(len(dims)):
        for w, origin in (([1.0, -2.0, 3.0], 0), ([0.5] * 4, -1)):
            for mode in MODES:
                got = oracle.correlate_1d(xf, w, axis=axis, mode=mode, cval=1.5, origin=origin)
                want = host_correlate_1d(x, dims, w, axis, mode, 1.5, origin)
                oracle.assert_close(got, want, 1e-5, f"{dims} axis {axis} {mode}")


def test_pad_index_matches_reference_model(oracle):
    for n in (1, 2, 5, 8):
        for p in range(-23, 30):
            for m in MODES:
                q = host_pad_index(p, n, m)
                assert oracle.pad_index(p, n, m) == (-1 if q is None else q), (p, n, m)


def test_scipy_fixtures_pin_the_restatement(oracle):
    g = np.load(os.path.join(HERE, "golden", "scipy_filters.npz"))
    x2, x3 = g["x2"], g["x3"]
    for key in g["cases"]:
        key = str(key)
        if key.startswith("g2_"):
            _, mode, sigma, order = key.split("_")
            got = oracle.gaussian_blur(x2, [float(sigma)], orders=[int(order[0]), int(order[1])], mode=mode, cval=1.5)
        else:
            got = oracle.gaussian_blur(x3, [1.0, 2.0, 1.5], mode=key.split("_")[1], cval=1.5)
        assert np.abs(got - g[key]).max() <= 1e-10 * max(1.0, np.abs(g[key]).max()), key
    # The f32 restatement stays within the reference's 1e-5 of FP64.
    got32 = oracle.gaussian_blur(x2.astype(np.float32), [2.0], orders=[0, 2], mode="reflect", cval=1.5)
    oracle.assert_close(got32, g["g2_reflect_2.0_02"], 1e-5, "f32")


def test_composites_against_scipy(oracle):
    g = np.load(os.path.join(HERE, "golden", "scipy_filters.npz"))
    x2 = g["x2"].astype(np.float32)
    oracle.assert_close(oracle.gaussian_laplace(x2, [2.0]), g["laplace_reflect_2.0"], 1e-5, "LoG")
    oracle.assert_close(oracle.gaussian_grad_mag(x2, [1.5]), g["gradmag_reflect_1.5"], 1e-5, "|grad|")
    dog = oracle.difference_of_gaussians(x2, [1.0], [3.0])
    want = oracle.gaussian_blur(g["x2"], [1.0]) - oracle.gaussian_blur(g["x2"], [3.0])
    oracle.assert_close(dog, want, 1e-5, "DoG")
    um = oracle.unsharp_mask(x2, [2.0], 0.7)
    oracle.assert_close(um, 1.7 * g["x2"] - 0.7 * oracle.gaussian_blur(g["x2"], [2.0]), 1e-5, "unsharp")


def test_rl_delta_psf_recovers_image(oracle):
    """crates/lucem-ops/src/restore/deconvolve.rs:517-539."""
    img = (np.arange(64, dtype=np.float32) / 64.0 * 0.8 + 0.1).reshape(8, 8)
    psf = np.zeros((3, 3), np.float32)
    psf[1, 1] = 1.0
    out = oracle.richardson_lucy(img, psf, num_iter=15, clip=False)
    oracle.assert_close(out, img.astype(np.float64), 1e-4, "delta psf")


def test_rl_box_psf_sharpens(oracle):
    """crates/lucem-ops/src/restore/deconvolve.rs:551-566."""
    spot = np.full((8, 8), 0.1, np.float32)
    spot[4, 4] = 0.9
    box = np.full((3, 3), 1.0 / 9.0, np.float32)
    blurred = oracle.correlate_nd(spot, box, mode="reflect")
    restored = oracle.richardson_lucy(blurred, box, num_iter=25, clip=True)
    assert restored[4, 4] > blurred[4, 4] + 0.15


def test_rl_direct_equals_fft_formulation(oracle):
    """Zero-padded RL computed directly (as the reference) equals the FFT form,
    odd and even PSF sizes, 2-D and 3-D (FP64)."""
    rng = np.random.default_rng(5)
    for shape, kshape in (((21, 17), (5, 4)), ((20, 19), (7, 7)), ((6, 9, 11), (3, 4, 5))):
        obs = rng.uniform(0.1, 1.0, shape)
        psf = rng.uniform(0.0, 1.0, kshape)
        a = oracle.richardson_lucy(obs, psf, num_iter=6, clip=False, filter_epsilon=1e-6, mode="constant")
        b = oracle.richardson_lucy_fft64(obs, psf, num_iter=6, filter_epsilon=1e-6)
        assert np.abs(a - b).max() < 1e-12 * np.abs(a).max(), shape


def test_tiled_equals_whole(oracle):
    """engine/lucem-pipeline/src/custom.rs:478-495: blocks of 128 with a halo of
    16, each blurred on its read part and cropped, equal the whole image."""
    x = sample_f64(300 * 310).reshape(300, 310).astype(np.float32)
    whole = oracle.gaussian_blur(x, [2.0, 2.0])
    got = np.zeros_like(whole)
    for y in range(0, 300, 128):
        for xx in range(0, 310, 128):
            sy, sx = min(128, 300 - y), min(128, 310 - xx)
            ry0, rx0 = max(0, y - 16), max(0, xx - 16)
            ry1, rx1 = min(300, y + sy + 16), min(310, xx + sx + 16)
            part = oracle.gaussian_blur(np.ascontiguousarray(x[ry0:ry1, rx0:rx1]), [2.0, 2.0])
            got[y:y + sy, xx:xx + sx] = part[y - ry0:y - ry0 + sy, xx - rx0:xx - rx0 + sx]
    assert np.abs(got - whole).max() < 1e-3


def test_halo_of_sigma_two_is_eight(oracle):
    """bindings/python/tests/test_runtime_io.py:28."""
    assert oracle.resolved_radius(4.0, 2.0) == 8
    assert int(np.ceil(4 * 2.0)) == 8


@pytest.mark.parametrize("shape,kshape", [((12, 10), (3, 5)), ((11, 9), (4, 4)), ((6, 7, 8), (2, 3, 4))])
def test_rl_backward_oracle_against_central_differences(oracle, shape, kshape):
    """The FP64 reverse-mode oracle against FP64 central differences of the
    FP64 RL (h 1e-5): PSF and observation gradients."""
    rng = np.random.default_rng(sum(shape))
    obs = rng.uniform(0.5, 2.0, shape)
    psf = rng.uniform(0.2, 1.0, kshape)
    w = rng.standard_normal(shape)
    gp, gy = oracle.richardson_lucy_backward_fft64(obs, psf, w, num_iter=5, filter_epsilon=1e-6)

    def loss(o, p):
        return float(np.sum(w * oracle.richardson_lucy_fft64(o, p, num_iter=5, filter_epsilon=1e-6)))

    h = 1e-5
    fd = np.zeros(psf.size)
    for i in range(psf.size):
        pp = psf.copy().reshape(-1)
        pp[i] += h
        lp = loss(obs, pp.reshape(kshape))
        pp[i] -= 2 * h
        fd[i] = (lp - loss(obs, pp.reshape(kshape))) / (2 * h)
    assert np.abs(gp.reshape(-1) - fd).max() <= 1e-7 * np.abs(fd).max()
    for i in range(0, obs.size, max(1, obs.size // 6)):
        oo = obs.copy().reshape(-1)
        oo[i] += h
        lp = loss(oo.reshape(shape), psf)
        oo[i] -= 2 * h
        d = (lp - loss(oo.reshape(shape), psf)) / (2 * h)
        assert abs(gy.reshape(-1)[i] - d) <= 1e-7 * max(1.0, abs(d))


def test_direct_dft_matches_numpy_fft(oracle):
    """The restated direct DFT (core/kernels/fft.rs:9-47) against numpy's FP64
    FFT, forward and inverse, axis by axis and N-D."""
    rng = np.random.default_rng(3)
    for shape in [(7,), (13, 4), (5, 6, 7), (16, 9)]:
        re, im = rng.standard_normal(shape), rng.standard_normal(shape)
        x = re + 1j * im
        for inverse in (False, True):
            r, i = oracle.dft_nd(re, im, inverse)
            want = np.fft.ifftn(x) if inverse else np.fft.fftn(x)
            np.testing.assert_allclose(r + 1j * i, want, rtol=1e-11, atol=1e-11)


def test_fft_round_trip_like_the_reference(oracle):
    """crates/lucem-ops/src/core/fft.rs:146-161: a 7 x 9 sample through the
    forward and inverse transforms comes back within 1e-4."""
    x = sample_f64(63).reshape(7, 9)
    r, i = oracle.dft_nd(x, np.zeros_like(x))
    back, _ = oracle.dft_nd(r, i, inverse=True)
    oracle.assert_close(back, x, 1e-4, "round trip")


def test_wiener_oracle_recovers_a_delta_psf_image(oracle):
    """crates/lucem-ops/src/restore/deconvolve.rs:541-550: with a delta PSF and
    balance 1e-7 Wiener returns the image within 1e-3."""
    img = (np.arange(64) / 64.0 * 0.8 + 0.1).reshape(8, 8)
    psf = np.zeros((3, 3))
    psf[1, 1] = 1.0
    out = oracle.wiener_deconvolve(img, psf, balance=1e-7, clip=False)
    oracle.assert_close(out, img, 1e-3, "delta psf")
    fast = oracle.wiener_deconvolve(img, psf, balance=1e-7, clip=False, fft=oracle.numpy_fft)
    np.testing.assert_allclose(fast, out, rtol=1e-12, atol=1e-12)


def _fourier_shifted(img, shift):
    f = np.fft.fftn(img)
    for d, s in enumerate(shift):
        n = img.shape[d]
        k = np.arange(n)
        sh = [1] * img.ndim
        sh[d] = -1
        f = f * np.exp(-2j * np.pi * s * (np.where(k <= n // 2, k, k - n) / n)).reshape(sh)
    return np.fft.ifftn(f).real


def test_phase_correlation_oracle_reference_cases(oracle):
    """crates/lucem-ops/src/register/phase.rs:262-296: a 16x16 sample image
    shifted by (2.25, -1.5), upsample 20, recovered as (-2.25, 1.5) within
    0.1; an integer roll is recovered exactly with zero error."""
    i = np.arange(256, dtype=np.int64)
    base = (((i * 6151 + 49_999) % 1013).astype(np.float64) * 0.1 + 0.1).reshape(16, 16)
    shift, err, _ = oracle.phase_correlation(base, _fourier_shifted(base, (2.25, -1.5)), 20, True)
    assert abs(shift[0] + 2.25) < 0.1 and abs(shift[1] - 1.5) < 0.1
    shift, err, pd = oracle.phase_correlation(base, np.roll(base, (3, -4), (0, 1)), 1, True)
    assert shift == [-3.0, 4.0] and err < 1e-6 and abs(pd) < 1e-9


def test_fourier_filter_oracle_reference_cases(oracle):
    """filter/spectral.rs:272-281 (a zero shift leaves the spectrum unchanged);
    a Gaussian of sigma 0 and a box of size 0 are the identity; the
    Butterworth low and high passes sum to one, the low pass keeps DC."""
    re, im = np.ones((4, 4), np.float32), np.zeros((4, 4), np.float32)
    for kind in ("shift", "gaussian", "box"):
        r, i = oracle.fourier_filter(re, im, [0.0], kind)
        assert np.array_equal(r, re) and np.array_equal(i, im)
    lp = oracle.butterworth_weights((9, 12), 0.2, False, 2.0).astype(np.float64)
    hp = oracle.butterworth_weights((9, 12), 0.2, True, 2.0).astype(np.float64)
    np.testing.assert_allclose(lp + hp, 1.0, atol=1e-7)
    assert lp[0, 0] == 1.0


def test_unsupervised_wiener_oracle_reference_case(oracle):
    """crates/lucem-ops/src/restore/deconvolve.rs:551-575: the 8x8 spot blurred
    by a 3x3 box, 12 iterations, burn-in 4, seed 7: a chain of 12 balances in
    [1e-6, 1e3] and an 8x8 image; the chain depends on the seed."""
    spot = np.full((8, 8), 0.1)
    spot[4, 4] = 0.9
    box = np.full((3, 3), 1.0 / 9.0)
    blurred = oracle.correlate_nd(spot.astype(np.float32), box.astype(np.float32), mode="reflect")
    out, chain = oracle.unsupervised_wiener(blurred, box, 12, 4, True, 7)
    assert len(chain) == 12 and out.shape == (8, 8)
    assert all(1e-6 <= b <= 1e3 for b in chain)
    _, other = oracle.unsupervised_wiener(blurred, box, 12, 4, True, 8)
    assert other != chain


def test_shape_index_oracle_distinguishes_dome_and_cup(oracle):
    """crates/lucem-ops/src/feature/structure.rs:193-214: on 17x17 paraboloids,
    sigma 1.5, nearest padding, the centre's shape index is +1 for a dome and
    -1 for a cup within 2e-2."""
    y, x = np.mgrid[0:17, 0:17]
    r2 = ((y - 8.0) ** 2 + (x - 8.0) ** 2).astype(np.float32)
    assert abs(oracle.shape_index(-r2, 1.5, "nearest")[8, 8] - 1.0) < 2e-2
    assert abs(oracle.shape_index(r2, 1.5, "nearest")[8, 8] + 1.0) < 2e-2


def test_structure_and_ridge_oracle_properties(oracle):
    """The structure tensor of a linear ramp is constant away from the borders
    (gradient outer products of a constant gradient); the ridge filters of a
    constant image are zero (a zero Hessian)."""
    y, x = np.mgrid[0:24, 0:24].astype(np.float32)
    arr, arc, acc = oracle.structure_tensor(2.0 * y + 3.0 * x, 1.0, "nearest")
    # Sobel of 2y + 3x: g_r = 2 * 2 * 4 = 16, g_c = 3 * 2 * 4 = 24 inside.
    np.testing.assert_allclose(arr[8:16, 8:16], 256.0, rtol=1e-6)
    np.testing.assert_allclose(arc[8:16, 8:16], 384.0, rtol=1e-6)
    np.testing.assert_allclose(acc[8:16, 8:16], 576.0, rtol=1e-6)
    const = np.full((16, 16), 3.0, np.float32)
    for kind in ("frangi", "sato", "meijering"):
        assert np.abs(oracle.ridge_filter(const, kind, [1.0, 2.0])).max() < 1e-6


def test_blob_oracle_reference_case(oracle):
    """crates/lucem-ops/src/feature/blobs.rs:350-392: a 25x25 Gaussian blob
    (sigma 2.5) at (12, 12); LoG, DoG and DoH each report it first."""
    y, x = np.mgrid[0:25, 0:25]
    img = np.exp(-((y - 12.0) ** 2 + (x - 12.0) ** 2) / (2 * 2.5 ** 2)).astype(np.float32)
    sig = oracle.blob_sigmas(1.5, 4.0, 6, False)
    for kind, thr, sigmas in (("log", 0.05, sig), ("dog", 0.05, oracle.dog_sigmas(1.5, 4.0, 1.3)),
                              ("doh", 0.01, sig)):
        blobs = oracle.extract_blobs(oracle.blob_stack(img, kind, sigmas, 1.3), sigmas, thr, 0.5, 2)
        assert blobs and blobs[0][:2] == (12, 12), (kind, blobs[:2])


def test_pyramid_oracle_reference_case(oracle):
    """crates/lucem-ops/src/transform/pyramid.rs:271-292: a 4x4 ramp; the
    Gaussian pyramid of 2 layers has shapes 4x4, 2x2, 1x1 and the Laplacian
    one three levels starting at 4x4; bilinear resize of a constant is the
    constant, and resizing by 1 is the identity."""
    img = np.arange(1, 17, dtype=np.float32).reshape(4, 4)
    g = oracle.gaussian_pyramid(img, 2)
    assert [a.shape for a in g] == [(4, 4), (2, 2), (1, 1)]
    lap = oracle.laplacian_pyramid(img, 2)
    assert len(lap) == 3 and lap[0].shape == (4, 4)
    c = np.full((7, 9), 3.0, np.float32)
    np.testing.assert_allclose(oracle.resize(c, 4, 5), 3.0, rtol=1e-6)
    np.testing.assert_array_equal(oracle.resize(img, 4, 4, order=1), img)


def test_canny_oracle_reference_case(oracle):
    """crates/lucem-ops/src/feature/canny.rs:172-189: a 10x10 square of ones
    in a 20x20 image, sigma 1: 28..60 edge pixels, none inside or at the
    corner.  Then the hysteresis rules on a hand-made suppression map: weak
    pixels join only through 8-connected chains to a strong one, and a low
    threshold of 0 grows nothing."""
    data = np.zeros((20, 20), np.float32)
    data[5:15, 5:15] = 1.0
    e = oracle.canny(data, 1.0)
    assert e.dtype == np.uint32 and 28 <= int(e.sum()) <= 60
    assert e[10, 10] == 0 and e[0, 0] == 0
    nms = np.zeros((6, 7), np.float32)
    nms[1, 1], nms[2, 2], nms[3, 3] = 5.0, 2.0, 2.0   # strong, then a diagonal chain of weak pixels
    nms[1, 5], nms[2, 5] = 2.0, 2.0                     # weak, not connected
    np.testing.assert_array_equal(np.argwhere(oracle.canny_hysteresis(nms, 1.0, 4.0)), [[1, 1], [2, 2], [3, 3]])
    np.testing.assert_array_equal(np.argwhere(oracle.canny_hysteresis(nms, 0.0, 4.0)), [[1, 1]])
    assert oracle.canny_hysteresis(nms, 1.0, 0.0).sum() == 0
    with pytest.raises(ValueError):
        oracle.canny_thresholds(10.0, 0.5, 0.4)


def test_canny_oracle_sectors_and_suppression(oracle):
    """feature/kernels/canny.rs:13-86: the sector of a gradient along x is 0,
    along y 2, along the main diagonal 1 and the anti-diagonal 3 (Sobel of
    integer ramps is exact); suppression keeps a pixel only when it is >= both
    neighbours along its sector, and clears the one-pixel border."""
    y, x = np.mgrid[0:9, 0:9].astype(np.float32)
    for img, sec in ((x, 0), (y, 2), (x + y, 1), (x - y, 3)):
        mag, sector = oracle.canny_gradients(img, 0.0, mode="nearest")
        assert (sector[2:-2, 2:-2] == sec).all(), sec
        assert np.allclose(mag[2:-2, 2:-2], mag[4, 4])
    # A ridge of magnitudes along x with a peak row: sector 2 compares rows.
    mag = np.tile(np.array([1, 2, 5, 2, 1], np.float32)[:, None], (1, 6))
    nms = oracle.canny_nms(mag, np.full(mag.shape, 2))
    assert (nms[2, 1:-1] == 5).all() and nms[[1, 3]].max() == 0
    assert nms[0].max() == 0 and nms[:, 0].max() == 0 and nms[:, -1].max() == 0


def test_blob_oracle_scales_and_overlap(oracle):
    """feature/blobs.rs:96-136, 256-263: linear and log-spaced scales, the DoG
    ladder sigma * ratio^k up to max_sigma, and the circle-overlap fraction
    (radius sqrt(2) sigma): 1 for a blob inside another, 0 when apart, the
    lens area over the smaller disc in between (two equal discs at distance
    r: 2 acos(1/2) - sqrt(3)/2 over pi = 0.391)."""
    np.testing.assert_allclose(oracle.blob_sigmas(1.0, 3.0, 5, False), [1.0, 1.5, 2.0, 2.5, 3.0])
    np.testing.assert_allclose(oracle.blob_sigmas(1.0, 4.0, 3, True), [1.0, 2.0, 4.0])
    np.testing.assert_allclose(oracle.dog_sigmas(1.0, 10.0, 1.6), [1.0, 1.6, 2.56, 4.096, 6.5536])
    assert oracle.blob_overlap((5, 5, 2.0), (5, 5, 1.0)) == 1.0
    assert oracle.blob_overlap((0, 0, 1.0), (0, 10, 1.0)) == 0.0
    r = np.sqrt(2.0) * 2.0
    got = oracle.blob_overlap((0, 0, 2.0), (0, r, 2.0))
    assert abs(got - (2 * np.arccos(0.5) - np.sqrt(3) / 2) / np.pi) < 1e-12
