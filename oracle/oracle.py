"""Python face of the oracle: ctypes over oracle/_build/liblucem_oracle.so plus
an FP64 FFT Richardson-Lucy in numpy.

TEST INFRASTRUCTURE ONLY.  The parity tests, the smoke check and the
benchmark's CPU-baseline leg use it to check results; the product never imports
it.  Parity status: pinned to the reference's own known-answer tests and to
scipy.ndimage fixtures, not to bit-level CubeCL output (the reference cannot be
built here); see lucem_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np
import scipy.fft as sfft

_HERE = os.path.dirname(os.path.abspath(__file__))
if _HERE not in sys.path:
    sys.path.insert(0, _HERE)
import build as _build  # noqa: E402

_lib = None

PAD_MODES = {"reflect": 0, "constant": 1, "nearest": 2, "mirror": 3, "wrap": 4}


def parse_mode(mode) -> int:
    """crates/lucem-ops/src/core/pad.rs:47-56 (aliases included)."""
    if isinstance(mode, int):
        return mode
    m = mode.strip().lower()
    aliases = {"symmetric": "reflect", "grid-mirror": "reflect", "grid-constant": "constant",
               "zeros": "constant", "edge": "nearest", "replicate": "nearest",
               "grid-wrap": "wrap", "periodic": "wrap"}
    m = aliases.get(m, m)
    if m not in PAD_MODES:
        raise ValueError(f"boundary pad mode '{mode}' is not supported")
    return PAD_MODES[m]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        P = C.c_void_p
        i64p = C.POINTER(C.c_int64)
        L.orc_gaussian_kernel_1d.argtypes = [C.c_double, C.c_uint32, C.c_int64, P]
        L.orc_resolved_radius.argtypes = [C.c_double, C.c_double]
        L.orc_resolved_radius.restype = C.c_int64
        L.orc_pad_index.argtypes = [C.c_int64, C.c_int64, C.c_int]
        L.orc_pad_index.restype = C.c_int64
        for s, real in (("f32", C.c_float), ("f64", C.c_double)):
            getattr(L, f"orc_correlate_1d_{s}").argtypes = [P, P, i64p, C.c_int, C.c_int, P, C.c_int64,
                                                             C.c_int32, C.c_int, real]
            getattr(L, f"orc_gaussian_blur_{s}").argtypes = [P, P, i64p, C.c_int, P, C.c_int, P, P, P,
                                                              C.c_int, C.c_double, C.c_double]
            getattr(L, f"orc_correlate_nd_{s}").argtypes = [P, P, i64p, C.c_int, P, i64p, C.c_int, real]
            getattr(L, f"orc_richardson_lucy_{s}").argtypes = [P, P, P, i64p, i64p, C.c_int, C.c_int,
                                                                C.c_int, C.c_double, C.c_int]
        L.orc_linear_comb_f32.argtypes = [P, P, P, C.c_int64, C.c_float, C.c_float, C.c_float]
        L.orc_gaussian_laplace_f32.argtypes = [P, P, i64p, C.c_int, P, C.c_int, C.c_double, C.c_double]
        L.orc_gaussian_grad_mag_f32.argtypes = [P, P, i64p, C.c_int, P, C.c_int, C.c_double, C.c_double]
        L.orc_difference_of_gaussians_f32.argtypes = [P, P, i64p, C.c_int, P, P, C.c_int, C.c_double,
                                                      C.c_double]
        L.orc_unsharp_mask_f32.argtypes = [P, P, i64p, C.c_int, P, C.c_double, C.c_int, C.c_double,
                                           C.c_double]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _dims(shape):
    return (C.c_int64 * max(1, len(shape)))(*shape)


def _sfx(dtype):
    if dtype == np.float32:
        return "f32"
    if dtype == np.float64:
        return "f64"
    raise TypeError(f"oracle supports float32/float64, got {dtype}")


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return lib().orc_get_threads()


def gaussian_kernel_1d(sigma: float, order: int, radius: int) -> np.ndarray:
    out = np.empty(2 * radius + 1, np.float64)
    lib().orc_gaussian_kernel_1d(float(sigma), int(order), int(radius), _ptr(out))
    return out


def resolved_radius(truncate: float, sigma: float) -> int:
    return int(lib().orc_resolved_radius(float(truncate), float(sigma)))


def pad_index(p: int, n: int, mode) -> int:
    return int(lib().orc_pad_index(int(p), int(n), parse_mode(mode)))


def _norm_axis(axis: int, ndim: int) -> int:
    a = axis + ndim if axis < 0 else axis
    if not 0 <= a < ndim:
        raise ValueError(f"axis {axis} is out of bounds for array of dimension {ndim}")
    return a


def correlate_1d(x: np.ndarray, w, axis=-1, mode="reflect", cval=0.0, origin=0) -> np.ndarray:
    """crates/lucem-ops/src/filter/convolve.rs:40-92 (weights cast to x's type)."""
    x = np.ascontiguousarray(x)
    s = _sfx(x.dtype)
    w = np.ascontiguousarray(np.asarray(w, dtype=np.float64).astype(x.dtype))
    out = np.empty_like(x)
    if x.size == 0:
        return out
    ax = _norm_axis(axis, x.ndim)
    getattr(lib(), f"orc_correlate_1d_{s}")(_ptr(x), _ptr(out), _dims(x.shape), x.ndim, ax, _ptr(w),
                                             len(w), int(origin), parse_mode(mode), float(cval))
    return out


def broadcast_per_axis(name, values, n):
    """crates/lucem-ops/src/core/check.rs:95-109."""
    values = list(values)
    if n == 0:
        return []
    if len(values) == 1:
        return values * n
    if len(values) == n:
        return values
    raise ValueError(f"invalid parameter `{name}`: expected 1 or {n} values, got {len(values)}")


def blur_axes(ndim, axes=None, channel_axis=None):
    """crates/lucem-ops/src/filter/gaussian.rs:184-188 (numpy axis rules)."""
    if axes is None:
        out = list(range(ndim))
    else:
        out = []
        for a in axes:
            n = _norm_axis(a, ndim)
            if n in out:
                raise ValueError(f"repeated axis {a}")
            out.append(n)
    if channel_axis is not None:
        ch = _norm_axis(channel_axis, ndim)
        out = [a for a in out if a != ch]
    return out


def gaussian_blur(x, sigmas, orders=(0,), mode="reflect", cval=0.0, truncate=4.0, radii=None,
                  axes=None, channel_axis=None) -> np.ndarray:
    """crates/lucem-ops/src/filter/gaussian.rs:176-250."""
    x = np.ascontiguousarray(x)
    s = _sfx(x.dtype)
    if np.isscalar(sigmas):
        sigmas = [sigmas]
    ax = blur_axes(x.ndim, axes, channel_axis)
    sig = broadcast_per_axis("sigmas", sigmas, len(ax))
    for v in sig:
        if not np.isfinite(v) or v < 0:
            raise ValueError(f"sigma must be non-negative and finite, got {v}")
    ords = broadcast_per_axis("orders", orders, len(ax))
    rad = broadcast_per_axis("radii", radii, len(ax)) if radii is not None else [-1] * len(ax)
    out = np.empty_like(x)
    if x.size == 0:
        return out
    n = max(1, len(ax))
    axes_c = (C.c_int * n)(*ax)
    sig_c = (C.c_double * n)(*sig)
    ord_c = (C.c_uint32 * n)(*ords)
    rad_c = (C.c_int64 * n)(*rad)
    getattr(lib(), f"orc_gaussian_blur_{s}")(_ptr(x), _ptr(out), _dims(x.shape), x.ndim, axes_c, len(ax),
                                              sig_c, ord_c, rad_c, parse_mode(mode), float(cval),
                                              float(truncate))
    return out


def _sig_all(sigmas, ndim):
    if np.isscalar(sigmas):
        sigmas = [sigmas]
    return (C.c_double * max(1, ndim))(*broadcast_per_axis("sigmas", sigmas, ndim))


def gaussian_laplace(x, sigmas, mode="reflect", cval=0.0, truncate=4.0):
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_gaussian_laplace_f32(_ptr(x), _ptr(out), _dims(x.shape), x.ndim, _sig_all(sigmas, x.ndim),
                                   parse_mode(mode), float(cval), float(truncate))
    return out


def gaussian_grad_mag(x, sigmas, mode="reflect", cval=0.0, truncate=4.0):
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_gaussian_grad_mag_f32(_ptr(x), _ptr(out), _dims(x.shape), x.ndim, _sig_all(sigmas, x.ndim),
                                    parse_mode(mode), float(cval), float(truncate))
    return out


def difference_of_gaussians(x, low, high, mode="reflect", cval=0.0, truncate=4.0):
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_difference_of_gaussians_f32(_ptr(x), _ptr(out), _dims(x.shape), x.ndim,
                                          _sig_all(low, x.ndim), _sig_all(high, x.ndim),
                                          parse_mode(mode), float(cval), float(truncate))
    return out


def unsharp_mask(x, sigmas, amount, mode="reflect", cval=0.0, truncate=4.0):
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_unsharp_mask_f32(_ptr(x), _ptr(out), _dims(x.shape), x.ndim, _sig_all(sigmas, x.ndim),
                               float(amount), parse_mode(mode), float(cval), float(truncate))
    return out


def correlate_nd(x, w, mode="reflect", cval=0.0):
    x = np.ascontiguousarray(x)
    s = _sfx(x.dtype)
    w = np.ascontiguousarray(np.asarray(w).astype(x.dtype))
    assert w.ndim == x.ndim and 1 <= x.ndim <= 3
    out = np.empty_like(x)
    getattr(lib(), f"orc_correlate_nd_{s}")(_ptr(x), _ptr(out), _dims(x.shape), x.ndim, _ptr(w),
                                             _dims(w.shape), parse_mode(mode), float(cval))
    return out


def rl_epsilon(filter_epsilon=None) -> float:
    """crates/lucem-ops/src/restore/deconvolve.rs:104."""
    return max(1e-12 if filter_epsilon is None else float(filter_epsilon), 1e-15)


def richardson_lucy(obs, psf, num_iter=30, clip=True, filter_epsilon=None, mode="reflect"):
    """crates/lucem-ops/src/restore/deconvolve.rs:45-162 in the obs dtype, any
    ndim 1..3 (direct spatial correlation, as the reference computes it)."""
    obs = np.ascontiguousarray(obs)
    s = _sfx(obs.dtype)
    psf = np.ascontiguousarray(np.asarray(psf).astype(obs.dtype))
    assert psf.ndim == obs.ndim
    if psf.size == 0:
        raise ValueError("psf: PSF cannot be empty")
    if num_iter < 1:
        raise ValueError("invalid parameter `num_iter`: num_iter must be >= 1")
    out = np.empty_like(obs)
    if obs.size == 0:
        return out
    rc = getattr(lib(), f"orc_richardson_lucy_{s}")(_ptr(obs), _ptr(psf), _ptr(out), _dims(obs.shape),
                                                     _dims(psf.shape), obs.ndim, int(num_iter), int(bool(clip)),
                                                     rl_epsilon(filter_epsilon), parse_mode(mode))
    assert rc == 0
    return out


def centred_otf(psf_norm: np.ndarray, grid, centre) -> np.ndarray:
    """Zero-padded PSF with tap `centre` wrapped to the origin (the convention of
    crates/lucem-ops/src/restore/kernels/deconvolve.rs:79-99), real FFT over `grid`."""
    buf = np.zeros(grid, np.float64)
    idx = np.indices(psf_norm.shape).reshape(psf_norm.ndim, -1)
    dst = tuple((idx[d] - centre[d]) % grid[d] for d in range(psf_norm.ndim))
    np.add.at(buf, dst, psf_norm.reshape(-1).astype(np.float64))
    return sfft.rfftn(buf, axes=tuple(range(psf_norm.ndim)), workers=-1)


def richardson_lucy_fft64(obs, psf, num_iter=30, clip=False, filter_epsilon=None, grid=None):
    """FP64 Richardson-Lucy with zero padding (PadMode::Constant, cval 0) computed
    through FFTs on `grid` (>= dims + k - 1 per axis).  Mathematically equal to
    the reference's direct Constant-mode iteration (deconvolve.rs:109-147)."""
    return richardson_lucy_fft(obs, psf, num_iter, clip, filter_epsilon, grid, np.float64)


def richardson_lucy_fft(obs, psf, num_iter=30, clip=False, filter_epsilon=None, grid=None, dtype=np.float64,
                        workers=-1):
    """richardson_lucy_fft64 in `dtype` (float64, or float32 with complex64
    spectra: the host FFT restatement the benchmark times), on `workers`
    threads (-1: all host cores).  The transfer functions are built in FP64
    and rounded once to `dtype`."""
    obs = np.asarray(obs, dtype)
    psf = np.asarray(psf, np.float64)
    nd = obs.ndim
    if grid is None:
        grid = tuple(obs.shape[d] + psf.shape[d] - 1 for d in range(nd))
    ssum = psf.sum()
    norm = 1.0 / ssum if abs(ssum) > 1e-12 else 1.0
    p = psf * norm
    k = psf.shape
    # correlate(src, flipped psf) == convolution with p centred at k-1-k//2;
    # correlate(src, p) == correlation with p centred at k//2 (convolve.rs:144-145).
    cdt = np.complex128 if dtype == np.float64 else np.complex64
    h_conv = centred_otf(p, grid, [k[d] - 1 - k[d] // 2 for d in range(nd)]).astype(cdt, copy=False)
    h_corr = np.conj(centred_otf(p, grid, [k[d] // 2 for d in range(nd)])).astype(cdt, copy=False)
    eps = dtype(rl_epsilon(filter_epsilon))
    sl = tuple(slice(0, n) for n in obs.shape)
    est = np.full(obs.shape, 0.5, dtype)
    for it in range(num_iter):
        ax = tuple(range(nd))
        conv = sfft.irfftn(sfft.rfftn(est, grid, axes=ax, workers=workers) * h_conv, grid, axes=ax,
                           workers=workers)[sl]
        safe = np.where(np.abs(conv) < eps, eps, conv)
        ratio = obs / safe
        corr = sfft.irfftn(sfft.rfftn(ratio, grid, axes=ax, workers=workers) * h_corr, grid, axes=ax,
                           workers=workers)[sl]
        est = est * corr
        if clip and it + 1 == num_iter:
            est = np.clip(est, -1.0, 1.0)
    return est


def assert_close(got, want, rtol, context=""):
    """crates/lucem-core/src/test_support.rs:42-50: |g - w| <= rtol*|w| + rtol*max|w|."""
    got = np.asarray(got, np.float64).reshape(-1)
    want = np.asarray(want, np.float64).reshape(-1)
    assert got.shape == want.shape, f"{context}: {got.size} values, expected {want.size}"
    scale = np.max(np.abs(want)) if want.size else 0.0
    bad = np.abs(got - want) > rtol * np.abs(want) + rtol * scale
    if bad.any():
        i = int(np.argmax(bad))
        raise AssertionError(f"{context}: index {i}: got {got[i]}, expected {want[i]} (rtol {rtol}); "
                             f"{int(bad.sum())} of {bad.size} outside")


def max_rel_err(got, want) -> float:
    """The smallest rtol for which assert_close passes."""
    got = np.asarray(got, np.float64).reshape(-1)
    want = np.asarray(want, np.float64).reshape(-1)
    if want.size == 0:
        return 0.0
    scale = np.max(np.abs(want))
    den = np.abs(want) + scale
    den = np.where(den == 0, 1.0, den)
    return float(np.max(np.abs(got - want) / den))


def richardson_lucy_backward_fft64(obs, psf, grad_out, num_iter=30, filter_epsilon=None, grid=None):
    """Reverse mode of richardson_lucy_fft64 (zero padding, clip off) in FP64:
    (d loss / d psf, d loss / d obs) given d loss / d estimate.  The adjoint
    of each step of the iteration (c = A e, r = y / guard(c), a = B r,
    e' = e * a) with A the convolution and B the correlation by the
    normalised PSF, then through the normalisation p_n = p / sum(p).  The
    reference has no reverse mode; this is the test oracle for the device
    gradients besides central differences."""
    obs = np.asarray(obs, np.float64)
    psf = np.asarray(psf, np.float64)
    w = np.asarray(grad_out, np.float64)
    nd = obs.ndim
    k = psf.shape
    if grid is None:
        grid = tuple(obs.shape[d] + k[d] - 1 for d in range(nd))
    ssum = psf.sum()
    norm = 1.0 / ssum if abs(ssum) > 1e-12 else 1.0
    p = psf * norm
    cc = [k[d] - 1 - k[d] // 2 for d in range(nd)]
    cr = [k[d] // 2 for d in range(nd)]
    hc = centred_otf(p, grid, cc)
    hr = centred_otf(p, grid, cr)
    ax = tuple(range(nd))
    sl = tuple(slice(0, n) for n in obs.shape)
    eps = rl_epsilon(filter_epsilon)

    def apply(h, conj, x):
        X = sfft.rfftn(x, grid, axes=ax, workers=-1)
        return sfft.irfftn(X * (np.conj(h) if conj else h), grid, axes=ax, workers=-1)[sl], X

    est = [np.full(obs.shape, 0.5)]
    for _ in range(num_iter):
        c, _ = apply(hc, 0, est[-1])
        r = obs / np.where(np.abs(c) < eps, eps, c)
        a, _ = apply(hr, 1, r)
        est.append(est[-1] * a)
    ebar = w.copy()
    ybar = np.zeros_like(obs)
    pb_conv = 0.0
    pb_corr = 0.0
    for t in range(num_iter - 1, -1, -1):
        e = est[t]
        c, se = apply(hc, 0, e)
        guarded = np.abs(c) < eps
        d = np.where(guarded, eps, c)
        r = obs / d
        a, sr = apply(hr, 1, r)
        abar = ebar * e
        rbar, sab = apply(hr, 0, abar)
        cbar = np.where(guarded, 0.0, -rbar * obs / (d * d))
        ybar += rbar / d
        tbar, scb = apply(hc, 1, cbar)
        ebar = ebar * a + tbar
        pb_conv = pb_conv + scb * np.conj(se)
        pb_corr = pb_corr + sr * np.conj(sab)

    def lags(pb, centre):
        full = sfft.irfftn(pb, grid, axes=ax, workers=-1)
        idx = np.indices(k).reshape(nd, -1)
        src = tuple((idx[dd] - centre[dd]) % grid[dd] for dd in range(nd))
        return full[src].reshape(k)

    gn = lags(pb_conv, cc) + lags(pb_corr, cr)
    gp = norm * (gn - np.sum(gn * p)) if abs(ssum) > 1e-12 else gn
    return gp, ybar


# ---------------------------------------------------------------------------
# Spectral operators (test infrastructure, FP64).


def dft_axis(re, im, axis, inverse=False):
    """The reference's direct DFT along `axis` (dft_axis_kernel,
    crates/lucem-ops/src/core/kernels/fft.rs:9-47) in FP64: X[f] = sum_n
    x[n] e^{-+2 pi i f n / len}, the inverse scaled by 1/len.  Phases reduced
    exactly ((f n) mod len)."""
    x = np.asarray(re, np.float64) + 1j * np.asarray(im, np.float64)
    x = np.moveaxis(x, axis, -1)
    n = x.shape[-1]
    k = np.arange(n)
    ph = (np.outer(k, k) % n).astype(np.float64)
    sign = 1.0 if inverse else -1.0
    w = np.exp(sign * 2j * np.pi * ph / n)
    y = x @ w.T
    if inverse:
        y = y / n
    y = np.moveaxis(y, -1, axis)
    return y.real, y.imag


def dft_nd(re, im, inverse=False):
    """fft_nd_into (crates/lucem-ops/src/core/fft.rs:55-100): dft_axis over
    axes 0, 1, ... in order."""
    r, i = np.asarray(re, np.float64), np.asarray(im, np.float64)
    for ax in range(r.ndim):
        r, i = dft_axis(r, i, ax, inverse)
    return r, i


def centred_kernel_2d(k, shape):
    """fft_shift_2d_kernel (restore/kernels/deconvolve.rs:79-99): tap (ky, kx)
    at ((ky - kh/2) mod H, (kx - kw/2) mod W) of a zero [H, W] array."""
    out = np.zeros(shape, np.float64)
    kh, kw = k.shape
    for ky in range(kh):
        for kx in range(kw):
            out[(ky - kh // 2) % shape[0], (kx - kw // 2) % shape[1]] += float(k[ky, kx])
    return out


def wiener_deconvolve(img, psf, balance=0.1, clip=True, fft=None):
    """wiener_deconvolve_into (crates/lucem-ops/src/restore/deconvolve.rs:
    210-295) in FP64: Y = DFT(img), H = DFT(centred psf), L = DFT(centred
    Laplacian [0 -1 0; -1 4 -1; 0 -1 0], a 1x1 one below 3x3 images),
    X = conj(H) Y / max(|H|^2 + balance |L|^2, 1e-12), out = Re(IDFT(X)),
    clipped to [-1, 1] when `clip`.  `fft`: the N-D transform to use (default
    dft_nd; numpy.fft for sizes where the direct DFT is too slow)."""
    img = np.asarray(img, np.float64)
    shape = img.shape
    if fft is None:
        def fft(x, inverse=False):
            r, i = dft_nd(x.real, x.imag, inverse)
            return r + 1j * i
    y = fft(img + 0j)
    h = fft(centred_kernel_2d(np.asarray(psf, np.float64), shape) + 0j)
    if shape[0] >= 3 and shape[1] >= 3:
        lap = np.array([[0, -1, 0], [-1, 4, -1], [0, -1, 0]], np.float64)
    else:
        lap = np.ones((1, 1))
    l = fft(centred_kernel_2d(lap, shape) + 0j)
    l2 = (l * np.conj(l)).real
    den = np.maximum(np.abs(h) ** 2 + balance * l2, 1e-12)
    x = np.conj(h) * y / den
    out = fft(x, inverse=True).real
    return np.clip(out, -1.0, 1.0) if clip else out


def numpy_fft(x, inverse=False):
    """numpy's FP64 FFT with fft_nd_into's scaling (pinned to dft_nd in the
    oracle tests)."""
    return np.fft.ifftn(x) if inverse else np.fft.fftn(x)


def bin_freq(n):
    """Signed normalised frequency of every bin of an n-point axis
    (crates/lucem-ops/src/filter/spectral.rs:38-41)."""
    k = np.arange(n)
    return np.where(k <= n // 2, k, k - n).astype(np.float64) / n


def _axis_view(v, d, ndim):
    shape = [1] * ndim
    shape[d] = -1
    return v.reshape(shape)


def fourier_filter(re, im, values, kind):
    """fourier_gaussian_into / fourier_box_into / fourier_shift_into
    (crates/lucem-ops/src/filter/spectral.rs:21-164): per axis in order, the
    f32 spectrum times the axis's f32 table (FP64 values cast once, as
    cast_all), with the reference kernels' f32 products
    (filter/kernels/spectral.rs:10-51)."""
    re = np.array(re, np.float32)
    im = np.array(im, np.float32)
    per = broadcast_per_axis("values", values, re.ndim)
    for d, v in enumerate(per):
        f = bin_freq(re.shape[d])
        if kind == "gaussian":
            w = np.exp(-2.0 * np.pi * np.pi * v * v * f * f).astype(np.float32)
            re, im = re * _axis_view(w, d, re.ndim), im * _axis_view(w, d, re.ndim)
        elif kind == "box":
            x = np.pi * v * f
            with np.errstate(invalid="ignore", divide="ignore"):
                w = np.where(np.abs(x) < 1e-12, 1.0, np.sin(x) / np.where(x == 0, 1.0, x)).astype(np.float32)
            re, im = re * _axis_view(w, d, re.ndim), im * _axis_view(w, d, re.ndim)
        else:
            c = _axis_view(np.cos(-2.0 * np.pi * v * f).astype(np.float32), d, re.ndim)
            s = _axis_view(np.sin(-2.0 * np.pi * v * f).astype(np.float32), d, re.ndim)
            re, im = (re * c - im * s).astype(np.float32), (re * s + im * c).astype(np.float32)
    return re, im


def butterworth_weights(shape, cutoff_ratio, high_pass=False, order=2.0):
    """The Butterworth transfer function of filter/spectral.rs:185-199 (FP64,
    cast to f32 as the reference's host array)."""
    r2 = np.zeros(shape, np.float64)
    for d, n in enumerate(shape):
        r2 = r2 + _axis_view((bin_freq(n) / cutoff_ratio) ** 2, d, len(shape))
    lp = 1.0 / (1.0 + np.sqrt(r2) ** (2.0 * order))
    return (1.0 - lp if high_pass else lp).astype(np.float32)


def butterworth(x, cutoff_ratio, high_pass=False, order=2.0):
    """butterworth (filter/spectral.rs:168-213) in FP64 on numpy's FFT:
    Re(IFFT(FFT(x) w))."""
    x = np.asarray(x, np.float64)
    w = butterworth_weights(x.shape, cutoff_ratio, high_pass, order).astype(np.float64)
    return np.fft.ifftn(np.fft.fftn(x) * w).real


def phase_correlation(ref, mov, upsample_factor=1, normalize_phase=True):
    """phase_correlation (crates/lucem-ops/src/register/phase.rs:51-255) in
    FP64: cross-power spectrum, |cc|^2 argmax (first index), the two-pass
    coordinate-wise candidate search (every candidate's sum over the whole
    spectrum), the snap to 1/upsample_factor, phasediff and the RMS error.
    Returns (shift, error, phasediff)."""
    ref = np.asarray(ref, np.float64)
    mov = np.asarray(mov, np.float64)
    shape, nd, n = ref.shape, ref.ndim, ref.size
    A, B = np.fft.fftn(ref), np.fft.fftn(mov)
    R = A * np.conj(B)
    if normalize_phase:
        mag = np.abs(R)
        R = np.where(mag > 1e-12, R / np.where(mag > 1e-12, mag, 1.0), 0.0)
    cc = np.fft.ifftn(R)
    mi = int(np.argmax(np.abs(cc) ** 2))
    idx = np.unravel_index(mi, shape)
    shift = [float(k if k <= shape[d] // 2 else k - shape[d]) for d, k in enumerate(idx)]
    peak = complex(cc.flat[mi])
    if upsample_factor > 1:
        u = float(upsample_factor)
        half = int(np.ceil(1.5 * u))
        freqs = [bin_freq(s) for s in shape]
        for ps in range(2):
            radius, step = (half, 1.0 / u) if ps == 0 else (2, 0.25 / u)
            for ax in range(nd):
                other = np.zeros(shape)
                for d in range(nd):
                    if d != ax:
                        other = other + 2.0 * np.pi * _axis_view(freqs[d], d, nd) * shift[d]
                oth = np.exp(1j * other)
                center, best, bs, bp = shift[ax], -1.0, shift[ax], peak
                for m in range(-radius, radius + 1):
                    cs = center + m * step
                    tot = (R * oth * _axis_view(np.exp(1j * 2.0 * np.pi * freqs[ax] * cs), ax, nd)).sum() / n
                    mag2 = abs(tot) ** 2
                    if mag2 > best:
                        best, bs, bp = mag2, cs, tot
                shift[ax], peak = bs, bp
        # f64::round: half away from zero (not Python's round-half-even).
        shift = [float(np.copysign(np.floor(abs(s * u) + 0.5), s * u)) / u for s in shift]
    phasediff = float(np.arctan2(peak.imag, peak.real))
    denom = float((ref ** 2).sum() * (mov ** 2).sum())
    if denom <= np.finfo(np.float64).eps:
        error = 0.0
    else:
        if normalize_phase:
            peak_u = np.fft.ifftn(A * np.conj(B)).flat[mi]
        else:
            peak_u = peak
        amp2 = abs(peak_u) ** 2 * n * n
        error = float(np.sqrt(1.0 - min(max(amp2 / denom, 0.0), 1.0)))
    return shift, error, phasediff


def unsupervised_wiener(img, psf, num_iter=30, burnin=10, clip=True, seed=0):
    """unsupervised_wiener (crates/lucem-ops/src/restore/deconvolve.rs:357-509):
    the spectra as f32 arrays (FP64 FFTs rounded once; the reference's device
    arrays are f32), their products in f32 as complex_mul_into, the chain in
    FP64 with the reference's update and PCG jitter.  Returns (out, chain)."""
    img = np.asarray(img, np.float64)
    shape, n = img.shape, float(img.size)
    c64 = lambda z: (z.real.astype(np.float32), z.imag.astype(np.float32))  # noqa: E731
    yr, yi = c64(np.fft.fftn(img))
    hr, hi = c64(np.fft.fftn(centred_kernel_2d(np.asarray(psf, np.float64), shape)))
    if shape[0] >= 3 and shape[1] >= 3:
        lap = np.array([[0, -1, 0], [-1, 4, -1], [0, -1, 0]], np.float64)
    else:
        lap = np.ones((1, 1))
    lr, li = c64(np.fft.fftn(centred_kernel_2d(lap, shape)))
    f = lambda a: a.astype(np.float64)  # noqa: E731
    hm2 = f(hr * hr - hi * (np.float32(0) - hi))
    lm2 = f(lr * lr - li * (np.float32(0) - li))
    hyr = f(yr * hr - yi * (np.float32(0) - hi))
    hyi = f(yr * (np.float32(0) - hi) + yi * hr)
    img_var = float(np.asarray(img, np.float32).astype(np.float64).var())
    balance, chain = 0.05, []
    mean = np.zeros(shape, np.complex128)
    rng = (int(seed) + 0x9E3779B97F4A7C15) % (1 << 64)
    for it in range(num_iter):
        den = np.maximum(hm2 + balance * lm2, 1e-12)
        xr, xi = hyr / den, hyi / den
        hxr, hxi = f(hr) * xr - f(hi) * xi, f(hr) * xi + f(hi) * xr
        dr, di = f(yr) - hxr, f(yi) - hxi
        rss = float(((dr * dr + di * di) / n).sum())
        reg = float((lm2 * ((xr * xr + xi * xi) / n)).sum())
        tr = float((hm2 / den).sum())
        if it >= burnin:
            mean += xr + 1j * xi
        eff = max(n - tr, 1.0)
        sn2 = max(rss / eff, 1e-8 * max(img_var, 1e-6))
        sx2 = max(reg / max(tr, 1.0), 1e-8)
        rng = (rng * 6364136223846793005 + 1) % (1 << 64)
        u = (rng >> 33) / float(1 << 31) - 0.5
        balance = min(max(sn2 / sx2 * np.exp(u * (2.0 / np.sqrt(n))), 1e-6), 1e3)
        chain.append(balance)
    mean /= max(num_iter - burnin, 1)
    m32 = mean.real.astype(np.float32).astype(np.float64) + 1j * mean.imag.astype(np.float32).astype(np.float64)
    out = np.fft.ifftn(m32).real
    return (np.clip(out, -1.0, 1.0) if clip else out), chain


# ---------------------------------------------------------------------------
# Gaussian-consumer operators (feature/structure.rs, filter/ridge.rs): the
# f32 restatement of the filters above, then the per-pixel kernels in f32
# with every operation rounded as the reference's CubeCL kernels.

_F = np.float32


def hessian_matrix(x, sigma, mode="reflect", cval=0.0):
    """feature/structure.rs:16-54: Gaussian derivatives of orders (2,0),
    (1,1), (0,2)."""
    x = np.asarray(x, _F)
    return tuple(gaussian_blur(x, [sigma, sigma], orders=o, mode=mode, cval=cval).astype(_F)
                 for o in ((2, 0), (1, 1), (0, 2)))


def eigvals_2x2(a, b, c):
    """core/kernels/eigen.rs:13-33."""
    a, b, c = (np.asarray(v, _F) for v in (a, b, c))
    mean = (a + c) * _F(0.5)
    diff = (a - c) * _F(0.5)
    r = np.sqrt(diff * diff + b * b).astype(_F)
    return mean + r, mean - r


def hessian_det(x, sigma, mode="reflect", cval=0.0):
    """feature/structure.rs:57-83 with hessian_det_2d_kernel."""
    a, b, c = hessian_matrix(x, sigma, mode, cval)
    return a * c - b * b


def shape_index_of(l1, l2):
    """shape_index_2d_kernel (feature/kernels/structure.rs:40-80), f32."""
    l1, l2 = np.asarray(l1, _F), np.asarray(l2, _F)
    diff, s = l1 - l2, l1 + l2
    scale = np.abs(l1) + np.abs(l2)
    flat = (np.abs(diff) <= _F(1e-6) * scale) | (scale <= _F(1e-20))
    lim = np.where((s < 0) & (scale > _F(1e-20)), _F(1), np.where((s > 0) & (scale > _F(1e-20)), _F(-1), _F(0)))
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = (-s) / np.where(flat, _F(1), diff)
        ax = np.abs(ratio)
        inv = ax > 1
        z = np.where(inv, _F(1) / np.where(ax == 0, _F(1), ax), ax).astype(_F)
    z2 = z * z
    poly = _F(-0.085133) + z2 * _F(0.0208351)
    poly = _F(0.180141) + z2 * poly
    poly = _F(-0.3302995) + z2 * poly
    poly = _F(0.999866) + z2 * poly
    at = z * poly
    ang = np.where(inv, _F(1.5707964) - at, at)
    out = np.where(ratio < 0, -ang, ang) * _F(0.63661975)
    return np.where(flat, lim, out).astype(_F)


def shape_index(x, sigma, mode="reflect", cval=0.0):
    """feature/structure.rs:164-191."""
    return shape_index_of(*eigvals_2x2(*hessian_matrix(x, sigma, mode, cval)))


def structure_tensor(x, sigma, mode="reflect", cval=0.0):
    """feature/structure.rs:102-147: Sobel gradients by two correlate_1d
    passes each (filter/gradient.rs:71-107), outer products, Gaussian window."""
    x = np.asarray(x, _F)
    d, sm = [-1.0, 0.0, 1.0], [1.0, 2.0, 1.0]
    gy = correlate_1d(correlate_1d(x, d, 0, mode, cval), sm, 1, mode, cval).astype(_F)
    gx = correlate_1d(correlate_1d(x, sm, 0, mode, cval), d, 1, mode, cval).astype(_F)
    return tuple(gaussian_blur(p, [sigma, sigma], mode=mode, cval=cval).astype(_F)
                 for p in (gy * gy, gy * gx, gx * gx))


def ridge_filter(x, kind, sigmas=(1.0, 3.0, 5.0, 7.0, 9.0), black_ridges=True, mode="reflect", cval=0.0,
                 beta=0.5, gamma=15.0):
    """frangi_into / sato_into / meijering_into (filter/ridge.rs:87-245) with
    the scale kernels of filter/kernels/ridge.rs:11-98, f32."""
    out = np.zeros(np.shape(x), _F)
    ib = _F(1.0 / (2.0 * max(beta * beta, 1e-12)))
    ic = _F(1.0 / (2.0 * max(gamma * gamma, 1e-12)))
    for sg in sigmas:
        e1, e2 = eigvals_2x2(*hessian_matrix(x, sg, mode, cval))
        if kind == "frangi":
            le = np.abs(e1) <= np.abs(e2)
            l1, l2 = np.where(le, e1, e2), np.where(le, e2, e1)
            valid = l2 > 0 if black_ridges else l2 < 0
            al2 = np.maximum(np.abs(l2), _F(1e-10))
            rb = l1 / al2
            s2 = l1 * l1 + l2 * l2
            resp = (np.exp(_F(0) - rb * rb * ib) * (_F(1) - np.exp(_F(0) - s2 * ic))).astype(_F)
            out = np.where(valid, np.maximum(out, resp), out)
        elif kind == "sato":
            ss = _F(sg * sg)
            s1, s2 = e1 * ss, e2 * ss
            l2 = np.where(np.abs(s1) <= np.abs(s2), s2, s1)
            out = np.maximum(out, np.maximum(l2, _F(0)) if black_ridges else np.maximum(_F(0) - l2, _F(0)))
        else:
            third = _F(-1.0 / 3.0)
            m1, m2 = e1 + third * e2, e2 + third * e1
            dom = np.where(np.abs(m1) >= np.abs(m2), m1, m2)
            out = np.maximum(out, np.maximum(dom, _F(0)) if black_ridges else np.maximum(_F(0) - dom, _F(0)))
    return out.astype(_F)


# ---------------------------------------------------------------------------
# Blob detectors (feature/blobs.rs): the f32 scale stack from the restated
# filters, then the reference's maxima, sort and overlap pruning.


def blob_sigmas(min_sigma, max_sigma, num_sigma, log_scale):
    """BlobDetector::sigmas (blobs.rs:96-111)."""
    if num_sigma == 1 or abs(max_sigma - min_sigma) <= np.finfo(np.float64).eps:
        return [min_sigma]
    out = []
    for i in range(num_sigma):
        t = i / (num_sigma - 1)
        out.append(min_sigma * (max_sigma / min_sigma) ** t if log_scale else min_sigma + t * (max_sigma - min_sigma))
    return out


def dog_sigmas(min_sigma, max_sigma, ratio):
    """blobs.rs:256-263."""
    out, s = [], min_sigma
    while s <= max_sigma * (1.0 + 1e-9):
        out.append(s)
        s *= ratio
    return out or [min_sigma]


def blob_stack(x, kind, sigmas, ratio=1.6):
    """The scale responses of blobs_log / blobs_dog / blobs_doh (blobs.rs:
    219-232, 265-283, 313-339), f32, reflect padding."""
    x = np.asarray(x, _F)
    out = []
    for sg in sigmas:
        if kind == "log":
            a = gaussian_blur(x, [sg, sg], orders=(2, 0)).astype(_F)
            b = gaussian_blur(x, [sg, sg], orders=(0, 2)).astype(_F)
            out.append(((a + b) * _F(-(sg * sg))).astype(_F))
        elif kind == "dog":
            a = gaussian_blur(x, [sg, sg]).astype(_F)
            b = gaussian_blur(x, [sg * ratio, sg * ratio]).astype(_F)
            out.append(((a - b) * _F(1.0 / (ratio - 1.0))).astype(_F))
        else:
            a, b, c = hessian_matrix(x, sg)
            out.append((_F(sg ** 4) * (a * c - b * b)).astype(_F))
    return np.stack(out)


def blob_overlap(a, b):
    """circle_overlap_fraction (blobs.rs:114-136); a, b: (y, x, sigma)."""
    r1, r2 = np.sqrt(2.0) * a[2], np.sqrt(2.0) * b[2]
    d = np.sqrt((a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2)
    if d >= r1 + r2:
        return 0.0
    if d <= abs(r1 - r2):
        return 1.0
    rmin = min(r1, r2)
    if rmin <= 0.0:
        return 0.0
    c1 = min(max((d * d + r1 * r1 - r2 * r2) / (2.0 * d * r1), -1.0), 1.0)
    c2 = min(max((d * d + r2 * r2 - r1 * r1) / (2.0 * d * r2), -1.0), 1.0)
    s = (-d + r1 + r2) * (d + r1 - r2) * (d - r1 + r2) * (d + r1 + r2)
    area = r1 * r1 * np.arccos(c1) + r2 * r2 * np.arccos(c2) - 0.5 * np.sqrt(max(s, 0.0))
    return area / (np.pi * rmin * rmin)


def extract_blobs(cube, sigmas, threshold, overlap, exclude_border=1):
    """extract_scale_space_blobs (blobs.rs:139-201): strict 3x3x3 maxima with
    the reference's tie rule (an equal neighbour earlier in (scale, y, x) order
    wins), threshold and border; sorted by response (descending), y, x; greedy
    overlap pruning.  Returns [(y, x, sigma, response)]."""
    cube = np.asarray(cube, _F)
    ns, H, W = cube.shape
    b = max(exclude_border, 1)
    if H <= 2 * b or W <= 2 * b:
        return []
    raw = []
    for s in range(ns):
        val = cube[s, b:H - b, b:W - b]
        is_max = val.astype(np.float64) > threshold
        for ds in (-1, 0, 1):
            t = s + ds
            if t < 0 or t >= ns:
                continue
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    if ds == 0 and dy == 0 and dx == 0:
                        continue
                    nv = cube[t, b + dy:H - b + dy, b + dx:W - b + dx]
                    before = ds < 0 or (ds == 0 and (dy < 0 or (dy == 0 and dx < 0)))
                    is_max &= ~((nv > val) | ((nv == val) & before))
        for y, x in zip(*np.nonzero(is_max)):
            raw.append((int(y) + b, int(x) + b, sigmas[s], float(val[y, x]), s))
    raw.sort(key=lambda r: (-r[3], r[0], r[1], r[4]))
    kept = []
    for r in raw:
        if all(blob_overlap(r, k) <= overlap for k in kept):
            kept.append(r)
    return [k[:4] for k in kept]


# ---------------------------------------------------------------------------
# Pyramids (transform/pyramid.rs) with resize's order 0 / 1 resampling
# (transform/warp.rs:207-251, core/kernels/spline.rs:90-139), f32.


def pad_map(p, n, mode):
    """core/kernels/pad.rs:11-34 on an integer array; -1: the constant."""
    m = parse_mode(mode) if isinstance(mode, str) else mode
    p = np.asarray(p, np.int64)
    inside = (p >= 0) & (p < n)
    if m == 1:  # constant
        out = np.full(p.shape, -1, np.int64)
    elif m == 2:  # nearest
        out = np.clip(p, 0, n - 1)
    elif m == 4:  # wrap
        out = np.mod(p, n)
    elif m == 0:  # reflect
        r = np.mod(p, 2 * n)
        out = np.where(r < n, r, 2 * n - 1 - r)
    else:  # mirror
        per = max(2 * n - 2, 1)
        r = np.mod(p, per)
        out = np.where(r < n, r, per - r)
    return np.where(inside, p, out)


def resize(x, oh, ow, order=1, mode="reflect", cval=0.0):
    """resize without anti-aliasing: output (oy, ox) samples the input at
    (sy oy + (sy - 1)/2, sx ox + (sx - 1)/2), f32, nearest or bilinear."""
    x = np.asarray(x, _F)
    H, W = x.shape
    sy, sx = H / oh, W / ow
    oy = np.arange(oh, dtype=_F)[:, None]
    ox = np.arange(ow, dtype=_F)[None, :]
    y = (_F(sy) * oy + _F(0.5 * (sy - 1.0))).astype(_F)
    xx = (_F(sx) * ox + _F(0.5 * (sx - 1.0))).astype(_F)
    y, xx = np.broadcast_to(y, (oh, ow)), np.broadcast_to(xx, (oh, ow))

    def sample(py, px):
        ok = (py >= 0) & (px >= 0)
        return np.where(ok, x[np.maximum(py, 0), np.maximum(px, 0)], _F(cval)).astype(_F)

    if order == 0:
        return sample(pad_map(np.floor(y + _F(0.5)), H, mode), pad_map(np.floor(xx + _F(0.5)), W, mode))
    y0, x0 = np.floor(y), np.floor(xx)
    fy, fx = (y - y0).astype(_F), (xx - x0).astype(_F)
    acc = np.zeros((oh, ow), _F)
    for dy in (0, 1):
        wy = (_F(1) - fy) if dy == 0 else fy
        py = pad_map(y0.astype(np.int64) + dy, H, mode)
        for dx in (0, 1):
            wx = (_F(1) - fx) if dx == 0 else fx
            px = pad_map(x0.astype(np.int64) + dx, W, mode)
            acc = (acc + (wy * wx).astype(_F) * sample(py, px)).astype(_F)
    return acc


def _pyr_sigma(downscale, sigma):
    return 2.0 * downscale / 6.0 if sigma is None else sigma


def pyramid_reduce(x, downscale=2.0, sigma=None, order=1, mode="reflect", cval=0.0):
    """pyramid.rs:135-168."""
    x = np.asarray(x, _F)
    sg = _pyr_sigma(downscale, sigma)
    sm = gaussian_blur(x, [sg, sg], mode=mode, cval=cval).astype(_F) if sg > 0 else x
    oh = max(1, int(np.ceil(x.shape[0] / downscale)))
    ow = max(1, int(np.ceil(x.shape[1] / downscale)))
    return resize(sm, oh, ow, order, mode, cval)


def pyramid_expand(x, shape=None, downscale=2.0, sigma=None, order=1, mode="reflect", cval=0.0):
    """pyramid.rs:171-208."""
    x = np.asarray(x, _F)
    if shape is None:
        shape = (max(1, int(np.ceil(x.shape[0] * downscale))), max(1, int(np.ceil(x.shape[1] * downscale))))
    up = resize(x, shape[0], shape[1], order, mode, cval)
    sg = _pyr_sigma(downscale, sigma)
    return gaussian_blur(up, [sg, sg], mode=mode, cval=cval).astype(_F) if sg > 0 else up


def gaussian_pyramid(x, max_layer, **kw):
    """pyramid.rs:211-236."""
    levels = [np.asarray(x, _F).copy()]
    for _ in range(max_layer):
        cur = levels[-1]
        if cur.shape[0] <= 1 and cur.shape[1] <= 1:
            break
        nxt = pyramid_reduce(cur, **kw)
        levels.append(nxt)
        if nxt.shape == cur.shape:
            break
    return levels


def laplacian_pyramid(x, max_layer, **kw):
    """pyramid.rs:239-266."""
    g = gaussian_pyramid(x, max_layer, **kw)
    if len(g) <= 1:
        return g
    return [(f - pyramid_expand(c, f.shape, **kw)).astype(_F) for f, c in zip(g[:-1], g[1:])] + [g[-1]]


def canny_gradients(x, sigma=1.0, mode="reflect", cval=0.0):
    """canny.rs:64-106 with canny_grad_dir_kernel (feature/kernels/canny.rs:
    13-41): the Gaussian pre-smoothing, the Sobel stencils as two correlate
    passes each (filter/gradient.rs:71-107), then in f32 the magnitude and the
    direction sector (0 along rows, 2 along columns, 1 / 3 the diagonals)."""
    x = np.asarray(x, _F)
    sm = gaussian_blur(x, [sigma, sigma], mode=mode, cval=cval).astype(_F)
    d, s = [-1.0, 0.0, 1.0], [1.0, 2.0, 1.0]
    gy = correlate_1d(correlate_1d(sm, d, 0, mode, cval), s, 1, mode, cval).astype(_F)
    gx = correlate_1d(correlate_1d(sm, s, 0, mode, cval), d, 1, mode, cval).astype(_F)
    mag = np.sqrt(gy * gy + gx * gx).astype(_F)
    ay, ax, t = np.abs(gy), np.abs(gx), _F(0.41421357)
    sector = np.where(ay <= ax * t, 0, np.where(ax <= ay * t, 2, np.where(gy * gx >= 0, 1, 3)))
    return mag, sector.astype(np.int32)


def canny_nms(mag, sector):
    """canny_nms_kernel (feature/kernels/canny.rs:44-86): border pixels 0; an
    interior pixel keeps its magnitude when it is >= both neighbours along its
    sector's direction."""
    mag = np.asarray(mag, _F)
    H, W = mag.shape
    nms = np.zeros_like(mag)
    if H < 3 or W < 3:
        return nms
    c, s = mag[1:-1, 1:-1], sector[1:-1, 1:-1]

    def at(dy, dx):
        return mag[1 + dy:H - 1 + dy, 1 + dx:W - 1 + dx]

    conds = [s == 0, s == 2, s == 1]
    n1 = np.select(conds, [at(0, -1), at(-1, 0), at(-1, -1)], at(-1, 1))
    n2 = np.select(conds, [at(0, 1), at(1, 0), at(1, 1)], at(1, -1))
    nms[1:-1, 1:-1] = np.where((c >= n1) & (c >= n2), c, _F(0))
    return nms


def canny_thresholds(max_mag, low=None, high=None, use_quantiles=False):
    """canny.rs:108-121."""
    lo = 0.1 * max_mag if low is None else float(low)
    hi = 0.2 * max_mag if high is None else float(high)
    if use_quantiles:
        lo, hi = lo * max_mag, hi * max_mag
    if hi < lo:
        raise ValueError(f"high_threshold ({hi}) must be >= low_threshold ({lo})")
    return lo, hi


def canny_hysteresis(nms, low, high):
    """canny.rs:123-162: breadth-first from every pixel with nms >= high
    (when high > 0) through the 8-neighbours with nms >= low (when low > 0)."""
    from collections import deque
    v = np.asarray(nms, np.float64)
    H, W = v.shape
    edges = ((v >= high) & (high > 0)).ravel()
    weak = ((v >= low) & (low > 0)).ravel()
    q = deque(np.flatnonzero(edges).tolist())
    while q:
        i = q.popleft()
        y, x = divmod(i, W)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ny, nx = y + dy, x + dx
                if (dy or dx) and 0 <= ny < H and 0 <= nx < W:
                    j = ny * W + nx
                    if not edges[j] and weak[j]:
                        edges[j] = True
                        q.append(j)
    return edges.reshape(H, W).astype(np.uint32)


def canny(x, sigma=1.0, low_threshold=None, high_threshold=None, use_quantiles=False, mode="reflect", cval=0.0):
    """canny (feature/canny.rs:47-165): u32 edge map."""
    x = np.asarray(x, _F)
    if x.ndim != 2:
        raise ValueError("canny expects a 2-D array")
    if not np.isfinite(sigma) or sigma < 0:
        raise ValueError(f"sigma must be non-negative and finite, got {sigma}")
    if x.size == 0:
        return np.zeros(x.shape, np.uint32)
    mag, sector = canny_gradients(x, sigma, mode, cval)
    nms = canny_nms(mag, sector)
    max_mag = max(float(np.max(mag)), 0.0)
    lo, hi = canny_thresholds(max_mag, low_threshold, high_threshold, use_quantiles)
    return canny_hysteresis(nms, lo, hi)
