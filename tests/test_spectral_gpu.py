"""The general complex FFT (lucem_fft_nd / lucem_fft_1d, the replacement of
the reference's direct DFT, crates/lucem-ops/src/core/fft.rs:14-100 and
core/kernels/fft.rs:9-47), complex_mul and Wiener deconvolution
(restore/deconvolve.rs:210-295), through the C ABI, against the oracle's FP64
restatements.  Lengths cover every path: smooth lengths in shared memory,
four-step above 8192, Bluestein for other lengths up to 4096, the direct DFT
beyond.  Tolerance: the reference's assert_close semantics
(crates/lucem-core/src/test_support.rs:42-50) at 1e-5 for transforms and
1e-4 for Wiener (a division by the regularised spectrum)."""
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


def want_fft(oracle, re, im, inverse, direct):
    if direct:
        return oracle.dft_nd(re, im, inverse)
    x = oracle.numpy_fft(re.astype(np.float64) + 1j * im.astype(np.float64), inverse)
    return x.real, x.imag


@pytest.mark.parametrize("shape", [(1,), (2,), (13,), (97,), (1000,), (4096,), (8192,), (3001,), (12000,),
                                   (16384,), (4099,), (7, 9), (64, 100), (33, 257), (5, 6, 7), (16, 32, 24),
                                   (3, 1, 5), (2, 2, 2, 3)])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft_nd_against_the_direct_dft(oracle, shape, inverse):
    rng = np.random.default_rng(int(np.prod(shape)) + inverse)
    re = rng.standard_normal(shape).astype(np.float32)
    im = rng.standard_normal(shape).astype(np.float32)
    gr, gi = lb.fft_nd(dev(re), dev(im), inverse=inverse)
    direct = int(np.prod(shape)) <= 4096
    wr, wi = want_fft(oracle, re, im, inverse, direct)
    oracle.assert_close(host(gr), wr, 1e-5, f"re {shape}")
    oracle.assert_close(host(gi), wi, 1e-5, f"im {shape}")


@pytest.mark.parametrize("shape,axis", [((6, 10, 7), 0), ((6, 10, 7), 1), ((6, 10, 7), -1), ((3, 5000), 1),
                                        ((9000, 2), 0)])
def test_fft_1d_along_one_axis(oracle, shape, axis):
    rng = np.random.default_rng(sum(shape) + axis)
    re = rng.standard_normal(shape).astype(np.float32)
    im = rng.standard_normal(shape).astype(np.float32)
    for inverse in (False, True):
        gr, gi = lb.fft_1d(dev(re), dev(im), axis=axis, inverse=inverse)
        x = re.astype(np.float64) + 1j * im.astype(np.float64)
        w = np.fft.ifft(x, axis=axis) if inverse else np.fft.fft(x, axis=axis)
        oracle.assert_close(host(gr), w.real, 1e-5, f"{shape} axis {axis}")
        oracle.assert_close(host(gi), w.imag, 1e-5, f"{shape} axis {axis}")


def test_round_trip_like_the_reference(oracle):
    """crates/lucem-ops/src/core/fft.rs:146-161 on the device."""
    n = 63
    x = (np.arange(n, dtype=np.float64) * 0.37 + 0.11) % 1.0 - 0.5
    x = x.reshape(7, 9).astype(np.float32)
    fr, fi = lb.fft_nd(dev(x))
    br, _ = lb.fft_nd(fr, fi, inverse=True)
    oracle.assert_close(host(br), x.astype(np.float64), 1e-4, "round trip")


def test_complex_mul(oracle):
    rng = np.random.default_rng(2)
    a, b, c, d = (rng.standard_normal((17, 23)).astype(np.float32) for _ in range(4))
    for conj in (False, True):
        r, i = lb.complex_mul(dev(a), dev(b), dev(c), dev(d), conj_b=conj)
        w = (a + 1j * b) * (np.conj(c + 1j * d) if conj else (c + 1j * d))
        np.testing.assert_allclose(host(r), w.real, rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(host(i), w.imag, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("shape,kshape,balance,clip", [((8, 8), (3, 3), 0.1, True), ((64, 80), (7, 7), 0.01, False),
                                                       ((100, 131), (9, 5), 0.5, False), ((2, 40), (1, 3), 0.2, False),
                                                       ((256, 256), (15, 15), 0.05, True)])
def test_wiener_against_the_oracle(oracle, shape, kshape, balance, clip):
    rng = np.random.default_rng(shape[0] * shape[1])
    img = rng.uniform(0.0, 1.0, shape).astype(np.float32)
    psf = rng.uniform(0.0, 1.0, kshape).astype(np.float32)
    psf /= psf.sum()
    got = host(lb.wiener_deconvolve(dev(img), dev(psf), balance=balance, clip=clip))
    fft = None if shape[0] * shape[1] <= 4096 else oracle.numpy_fft
    want = oracle.wiener_deconvolve(img, psf, balance=balance, clip=clip, fft=fft)
    oracle.assert_close(got, want, 1e-4, f"{shape} {kshape}")


def test_wiener_delta_psf_recovers_the_image(oracle):
    """crates/lucem-ops/src/restore/deconvolve.rs:541-550."""
    img = (np.arange(64) / 64.0 * 0.8 + 0.1).reshape(8, 8).astype(np.float32)
    psf = np.zeros((3, 3), np.float32)
    psf[1, 1] = 1.0
    out = host(lb.wiener_deconvolve(dev(img), dev(psf), balance=1e-7, clip=False))
    oracle.assert_close(out, img.astype(np.float64), 1e-3, "delta psf")


def test_wiener_errors_mirror_the_reference():
    x = torch.ones((8, 8), device="cuda")
    with pytest.raises(lb.LucemError) as e:
        lb.wiener_deconvolve(x, torch.ones((3, 3), device="cuda"), balance=-1.0)
    assert e.value.name == "INVALID_PARAMETER"
    with pytest.raises(lb.LucemError) as e:
        lb.wiener_deconvolve(x, torch.ones((9, 3), device="cuda"))
    assert e.value.name == "INVALID_WEIGHTS"
    with pytest.raises(lb.LucemError) as e:
        lb.wiener_deconvolve(torch.ones((2, 8, 8), device="cuda"), torch.ones((3, 3), device="cuda"))
    assert e.value.name == "INVALID_DIMENSION"
    with pytest.raises(lb.LucemError) as e:
        lb.wiener_deconvolve(x, torch.ones((0, 3), device="cuda"))
    assert e.value.name == "INVALID_WEIGHTS"
    assert lb.wiener_deconvolve(torch.ones((0, 4), device="cuda"), torch.ones((1, 1), device="cuda")).shape == (0, 4)


class _Producer:
    """A device-memory DLPack producer that is not a torch tensor (as CuPy or
    JAX arrays are): only __dlpack__ and __dlpack_device__."""

    def __init__(self, t):
        self._t = t

    def __dlpack__(self, *a, **k):
        return self._t.__dlpack__(*a, **k)

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


def test_dlpack_producers_in_and_out(oracle):
    rng = np.random.default_rng(8)
    x = rng.uniform(0.0, 1.0, (40, 50)).astype(np.float32)
    src = _Producer(dev(x))
    got = lb.gaussian_blur(src, 2.0)
    assert hasattr(got, "__dlpack__")
    want = oracle.gaussian_blur(x, [2.0])
    oracle.assert_close(host(got), want.astype(np.float64), 1e-5, "blur via dlpack")
    # zero copy: the view shares the producer's memory
    t = dev(x)
    assert lb.from_dlpack(_Producer(t)).data_ptr() == t.data_ptr()
    psf = np.full((3, 3), 1 / 9.0, np.float32)
    w = host(lb.wiener_deconvolve(_Producer(dev(x)), _Producer(dev(psf)), balance=0.1, clip=False))
    oracle.assert_close(w, oracle.wiener_deconvolve(x, psf, balance=0.1, clip=False, fft=oracle.numpy_fft), 1e-4,
                        "wiener via dlpack")


@pytest.mark.parametrize("shape", [(2048, 2048), (64, 128, 96), (3000, 7), (16384,)])
def test_fft_nd_against_cufft(shape):
    """Cross-check of the library's own transforms against cuFFT (torch.fft in
    float64 on the device), at sizes the host DFT oracle is too slow for;
    cuFFT is only this cross-check, never on the library's path."""
    g = torch.Generator(device="cuda")
    g.manual_seed(int(np.prod(shape)))
    re = torch.rand(shape, generator=g, device="cuda") - 0.5
    im = torch.rand(shape, generator=g, device="cuda") - 0.5
    z = torch.complex(re.double(), im.double())
    for inverse in (False, True):
        gr, gi = lb.fft_nd(re, im, inverse=inverse)
        w = torch.fft.ifftn(z) if inverse else torch.fft.fftn(z)
        scale = float(w.abs().max())
        err = max(float((gr.double() - w.real).abs().max()), float((gi.double() - w.imag).abs().max()))
        assert err <= 1e-5 * scale, (shape, inverse, err / scale)
