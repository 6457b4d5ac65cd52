"""Frequency-domain operators on the FFT, through the C ABI, against the
oracle's restatements:
  - fourier_gaussian / fourier_box / fourier_shift
    (crates/lucem-ops/src/filter/spectral.rs:21-164): the same f32 products in
    the same axis order, so equal to 1e-6 (table values cast once from FP64);
  - butterworth (filter/spectral.rs:168-213) against FP64 at 1e-5;
  - phase_correlation (crates/lucem-ops/src/register/phase.rs:51-255): the
    snapped shift equal to the FP64 restatement's, error and phase difference
    to 1e-5, and the reference's own subpixel test (16x16, shift (2.25, -1.5),
    upsample 20, recovered within 0.1);
  - unsupervised_wiener (restore/deconvolve.rs:357-509): balance chain to
    rel 1e-5 and the image at the reference's assert_close 1e-4, and the
    reference's own test case (8x8 blurred spot, 12 iterations, burn-in 4,
    seed 7).
Tolerances follow crates/lucem-core/src/test_support.rs:42-50."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.float64)


def sample_positive(n):
    """crates/lucem-ops/src/test_support.rs:15-17."""
    i = np.arange(n, dtype=np.int64)
    return ((i * 6151 + 49_999) % 1013).astype(np.float64) * 0.1 + 0.1


@pytest.mark.parametrize("kind", ["gaussian", "box", "shift"])
@pytest.mark.parametrize("shape,values", [((17,), [1.5]), ((8, 12), [2.0]), ((9, 10), [0.7, 3.1]),
                                          ((4, 5, 6), [1.0, -2.25, 0.5]), ((1, 31), [4.0])])
def test_fourier_filters_equal_the_restatement(oracle, kind, shape, values):
    rng = np.random.default_rng(len(shape) * 7 + len(kind))
    re = rng.standard_normal(shape).astype(np.float32)
    im = rng.standard_normal(shape).astype(np.float32)
    fn = {"gaussian": lb.fourier_gaussian, "box": lb.fourier_box, "shift": lb.fourier_shift}[kind]
    gr, gi = fn(dev(re), dev(im), values)
    wr, wi = oracle.fourier_filter(re, im, values, kind)
    oracle.assert_close(host(gr), wr.astype(np.float64), 1e-6, f"{kind} re {shape}")
    oracle.assert_close(host(gi), wi.astype(np.float64), 1e-6, f"{kind} im {shape}")


def test_fourier_shift_zero_leaves_the_spectrum_unchanged():
    """filter/spectral.rs:272-281."""
    re, im = torch.ones((4, 4), device="cuda"), torch.zeros((4, 4), device="cuda")
    gr, gi = lb.fourier_shift(re, im, [0.0, 0.0])
    assert torch.equal(gr, torch.ones_like(gr)) and torch.equal(gi, torch.zeros_like(gi))


def test_fourier_filter_errors():
    re, im = torch.ones((4, 4), device="cuda"), torch.zeros((4, 4), device="cuda")
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.fourier_gaussian(re, im, [1.0, 2.0, 3.0])
    with pytest.raises(lb.LucemError, match="SHAPE_MISMATCH"):
        lb.fourier_box(re, torch.zeros((4, 5), device="cuda"), [1.0])


@pytest.mark.parametrize("shape", [(64,), (31, 40), (128, 97), (12, 18, 20), (2048, 2048)])
@pytest.mark.parametrize("high_pass,order", [(False, 2.0), (True, 2.0), (False, 4.5)])
def test_butterworth_against_fp64(oracle, shape, high_pass, order):
    rng = np.random.default_rng(sum(shape) + int(order))
    x = rng.random(shape).astype(np.float32)
    got = lb.butterworth(dev(x), 0.15, high_pass, order)
    oracle.assert_close(host(got), oracle.butterworth(x, 0.15, high_pass, order), 1e-5, f"{shape}")


def test_butterworth_errors():
    x = torch.ones((8, 8), device="cuda")
    for c in (0.0, 0.51, -0.1):
        with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
            lb.butterworth(x, c)


@pytest.mark.parametrize("shape,roll", [((32, 32), (3, -5)), ((48, 40), (-7, 11)), ((17, 23), (4, 2)),
                                        ((8, 16, 12), (1, -3, 5)), ((100,), (13,))])
@pytest.mark.parametrize("normalize", [True, False])
def test_phase_correlation_integer_shifts(oracle, shape, roll, normalize):
    rng = np.random.default_rng(len(shape) + int(normalize))
    ref = rng.random(shape).astype(np.float32)
    mov = np.roll(ref, roll, axis=tuple(range(len(shape)))).astype(np.float32)
    r = lb.phase_correlation(dev(ref), dev(mov), normalize_phase=normalize)
    ws, we, wp = oracle.phase_correlation(ref, mov, 1, normalize)
    assert r.shift == ws == [-float(v) for v in roll]
    close_error(r, we, wp)


def close_error(r, want_error, want_phasediff):
    """error = sqrt(1 - ratio) is ill-conditioned where the ratio is 1 (an
    exact shift, where f32 rounding alone moves it by ~1e-7): compared
    squared, 1 - ratio to 1e-5."""
    assert abs(r.error ** 2 - want_error ** 2) < 1e-5, (r.error, want_error)
    assert abs(r.phasediff - want_phasediff) < 1e-5, (r.phasediff, want_phasediff)


def _fourier_shifted(img, shift):
    f = np.fft.fftn(img)
    for d, s in enumerate(shift):
        n = img.shape[d]
        k = np.arange(n)
        fr = np.where(k <= n // 2, k, k - n) / n
        sh = [1] * img.ndim
        sh[d] = -1
        f = f * np.exp(-2j * np.pi * s * fr).reshape(sh)
    return np.fft.ifftn(f).real


def test_phase_correlation_reference_subpixel_case(oracle):
    """register/phase.rs:262-296: a 16x16 sample image shifted by (2.25, -1.5)
    in the Fourier domain; upsample 20 recovers (-2.25, 1.5) within 0.1, and
    the snapped shift equals the FP64 restatement's.  The phase difference is
    not compared here: the half-pixel shift leaves cross-power bins of
    magnitude ~1e-9 (the moving image's Nyquist column), which the
    normalisation raises to unit weight with a phase set by rounding alone,
    so any two f32 implementations differ there (the smooth cases below
    compare it)."""
    base = sample_positive(256).reshape(16, 16)
    mov = _fourier_shifted(base, (2.25, -1.5))
    r = lb.phase_correlation(dev(base), dev(mov), upsample_factor=20)
    assert abs(r.shift[0] + 2.25) < 0.1 and abs(r.shift[1] - 1.5) < 0.1
    ws, we, _ = oracle.phase_correlation(base.astype(np.float32), mov.astype(np.float32), 20, True)
    assert r.shift == ws
    assert abs(r.error ** 2 - we ** 2) < 1e-5


# Well-conditioned inputs: white noise (no spectral zeros), shifts that are
# not half-integers, and odd sides in 3-D.  A Fourier shift of a real image
# by s multiplies a Nyquist bin by cos(pi s) after taking the real part, and
# in several dimensions such factors can cancel exactly; the normalised
# cross-power phase of a zeroed bin is rounding noise (see the reference
# case above).
@pytest.mark.parametrize("shape,shift,u", [((64, 64), (3.4, -7.7), 10), ((41, 56), (-5.25, 2.75), 4),
                                           ((23, 21, 19), (1.25, -2.75, 3.0), 4), ((256, 256), (10.3, 20.6), 20)])
def test_phase_correlation_subpixel_against_fp64(oracle, shape, shift, u):
    rng = np.random.default_rng(int(np.prod(shape)))
    base = rng.random(shape)
    mov = _fourier_shifted(base, shift)
    ref32, mov32 = base.astype(np.float32), mov.astype(np.float32)
    r = lb.phase_correlation(dev(ref32), dev(mov32), upsample_factor=u)
    ws, we, wp = oracle.phase_correlation(ref32, mov32, u, True)
    assert r.shift == ws
    for g, t in zip(r.shift, shift):
        assert abs(g + t) <= 1.0 / u + 1e-9
    close_error(r, we, wp)


def test_phase_correlation_errors():
    a = torch.ones((8, 8), device="cuda")
    with pytest.raises(lb.LucemError, match="SHAPE_MISMATCH"):
        lb.phase_correlation(a, torch.ones((8, 9), device="cuda"))
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.phase_correlation(a, a, upsample_factor=0)
    with pytest.raises(lb.LucemError, match="EMPTY_INPUT"):
        e = torch.empty((0, 4), device="cuda")
        lb.phase_correlation(e, e)


def test_unsupervised_wiener_reference_case(oracle):
    """restore/deconvolve.rs:551-575: the 8x8 spot blurred by the 3x3 box,
    12 iterations, burn-in 4, clip, seed 7: a chain of 12 and an 8x8 image."""
    spot = np.full((8, 8), 0.1, np.float32)
    spot[4, 4] = 0.9
    box = np.full((3, 3), 1.0 / 9.0, np.float32)
    blurred = oracle.correlate_nd(spot, box, mode="reflect").astype(np.float32)
    out, chain = lb.unsupervised_wiener(dev(blurred), dev(box), num_iter=12, burnin=4, clip=True, seed=7)
    assert len(chain) == 12 and tuple(out.shape) == (8, 8)
    wo, wc = oracle.unsupervised_wiener(blurred, box, 12, 4, True, 7)
    np.testing.assert_allclose(chain, wc, rtol=1e-5)
    oracle.assert_close(host(out), wo, 1e-4, "reference case")


@pytest.mark.parametrize("shape,psf_sigma,clip,seed", [((64, 48), 1.5, False, 0), ((100, 100), 2.0, True, 3),
                                                       ((37, 53), 1.0, False, 11), ((512, 512), 2.5, False, 5)])
def test_unsupervised_wiener_against_the_restatement(oracle, shape, psf_sigma, clip, seed):
    rng = np.random.default_rng(seed + shape[0])
    img = rng.random(shape).astype(np.float32) * 0.8
    r = int(3 * psf_sigma)
    yy, xx = np.mgrid[-r:r + 1, -r:r + 1]
    psf = np.exp(-(yy ** 2 + xx ** 2) / (2 * psf_sigma ** 2)).astype(np.float32)
    psf /= psf.sum()
    out, chain = lb.unsupervised_wiener(dev(img), dev(psf), num_iter=20, burnin=5, clip=clip, seed=seed)
    wo, wc = oracle.unsupervised_wiener(img, psf, 20, 5, clip, seed)
    np.testing.assert_allclose(chain, wc, rtol=1e-5)
    oracle.assert_close(host(out), wo, 1e-4, f"{shape}")


def test_unsupervised_wiener_errors():
    x = torch.ones((8, 8), device="cuda")
    k = torch.ones((3, 3), device="cuda")
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.unsupervised_wiener(x, k, num_iter=5, burnin=5)
    with pytest.raises(lb.LucemError, match="INVALID_DIMENSION"):
        lb.unsupervised_wiener(torch.ones((2, 8, 8), device="cuda"), k)
    with pytest.raises(lb.LucemError, match="INVALID_WEIGHTS"):
        lb.unsupervised_wiener(x, torch.ones((0, 3), device="cuda"))
    out, chain = lb.unsupervised_wiener(torch.ones((0, 8), device="cuda"), k)
    assert out.numel() == 0 and chain == []
