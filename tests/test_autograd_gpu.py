"""Reverse mode on the GPU: the Gaussian adjoint passes, the FFT convolution's
backward and the reverse pass through unrolled Richardson-Lucy, through the
C ABI and the torch.autograd Functions.

Checks, all against the oracle:
* linear filters: the adjoint equals A^T y with A assembled column by column
  from the oracle's forward filter (f64) on unit vectors (tolerance 1e-5,
  assert_close semantics);
* Richardson-Lucy: PSF and observation gradients against FP64 central finite
  differences (h = 1e-4) of the oracle's FP64 FFT iteration, relative 1e-3.
"""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu

RTOL = 1e-5
FD_RTOL = 1e-3
MODES = ["reflect", "constant", "nearest", "mirror", "wrap"]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def assert_linear_close(got, A, y, rtol, context, tap_mass=0.0):
    """|got - A^T y| <= rtol * max(max(|A|^T |y|), tap_mass * max|y|).  The
    second term is the size of the unfolded f32 sums: on a wrapped line
    shorter than the filter, derivative taps fold onto a few samples and
    cancel to ~1e-6 of their own size, below what f32 sums resolve."""
    yv = np.asarray(y, np.float64).reshape(-1)
    want = A.T @ yv
    bound = rtol * max(float(np.max(np.abs(A).T @ np.abs(yv))), tap_mass * float(np.max(np.abs(yv))))
    err = np.abs(np.asarray(got, np.float64).reshape(-1) - want)
    assert err.max() <= bound, f"{context}: max error {err.max():.3g} > {bound:.3g}"


def matrix(f, shape):
    """Columns f(e_j) of a linear map on arrays of `shape` (f64)."""
    n = int(np.prod(shape))
    cols = []
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        cols.append(np.asarray(f(e.reshape(shape)), np.float64).reshape(-1))
    return np.stack(cols, axis=1)


# ---------------------------------------------------------------------------
# Gaussian adjoint

BLUR_CASES = [
    # shape, sigmas, orders, extra
    ((9, 11), (1.5, 2.0), (0, 0), {}),
    ((9, 11), 1.2, (1, 2), {}),
    ((5, 4), 3.0, (0, 1), {}),                       # lines shorter than the radius
    ((4, 5, 6), 1.0, (0, 0, 2), {}),
    ((4, 5, 6), (0.8, 1.3), (1, 0), {"axes": (0, 2)}),
    ((13,), 2.0, (1,), {}),
    ((7, 8), 1.0, (0, 0), {"radii": (2, 5)}),
]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", range(len(BLUR_CASES)))
def test_gaussian_adjoint_is_the_transpose(oracle, mode, case):
    shape, sigmas, orders, extra = BLUR_CASES[case]
    A = matrix(lambda e: oracle.gaussian_blur(e, sigmas if not np.isscalar(sigmas) else [sigmas], orders=orders,
                                              mode=mode, cval=0.0, **extra), shape)
    rng = np.random.default_rng(case)
    y = rng.standard_normal(shape).astype(np.float32)
    got = host(lb.gaussian_blur_adjoint(dev(y), sigmas, orders=orders, mode=mode, **extra))
    axes = extra.get("axes", range(len(shape)))
    sig = oracle.broadcast_per_axis("sigmas", [sigmas] if np.isscalar(sigmas) else sigmas, len(axes))
    ords = oracle.broadcast_per_axis("orders", orders, len(axes))
    rads = extra.get("radii", [oracle.resolved_radius(4.0, s) for s in sig])
    mass = float(np.prod([np.abs(oracle.gaussian_kernel_1d(s, o, r)).sum() for s, o, r in zip(sig, ords, rads)]))
    assert_linear_close(got, A, y, RTOL, f"{mode} case {case}", mass)


def test_gaussian_adjoint_input_scale_and_cval(oracle):
    shape = (10, 12)
    A = matrix(lambda e: oracle.gaussian_blur(e, [1.7], mode="constant", cval=0.0), shape)
    y = np.random.default_rng(1).standard_normal(shape).astype(np.float32)
    want = 0.25 * (A.T @ y.reshape(-1)).reshape(shape)
    got = host(lb.gaussian_blur_adjoint(dev(y), 1.7, mode="constant", input_scale=0.25))
    oracle.assert_close(got, want, RTOL, "input_scale")
    # The forward is affine in the constant mode with cval != 0; its gradient
    # does not depend on cval.
    x = dev(np.random.default_rng(2).standard_normal(shape)).requires_grad_(True)
    lb.autograd.gaussian_blur(x, 1.7, mode="constant", cval=3.0, input_scale=0.25).mul(dev(y)).sum().backward()
    oracle.assert_close(host(x.grad), want, RTOL, "autograd cval")


def test_gaussian_adjoint_large_image_dot_product(oracle):
    """<A x, y> = <x, A^T y> at 1024 x 768, sigma 4 (radius 16), reflect."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal((1024, 768)).astype(np.float32)
    y = rng.standard_normal((1024, 768)).astype(np.float32)
    ax = host(lb.gaussian_blur(dev(x), 4.0, mode="reflect"))
    aty = host(lb.gaussian_blur_adjoint(dev(y), 4.0, mode="reflect"))
    lhs = float(np.dot(ax.reshape(-1), y.reshape(-1).astype(np.float64)))
    rhs = float(np.dot(x.reshape(-1).astype(np.float64), aty.reshape(-1)))
    scale = float(np.abs(ax).reshape(-1) @ np.abs(y).reshape(-1))
    assert abs(lhs - rhs) <= 1e-5 * scale


@pytest.mark.parametrize("mode", ["reflect", "wrap", "constant"])
def test_composite_filter_gradients(oracle, mode):
    shape = (9, 10)
    rng = np.random.default_rng(4)
    xn = rng.standard_normal(shape).astype(np.float32)
    w = rng.standard_normal(shape).astype(np.float32)
    wv = w.reshape(-1).astype(np.float64)
    cases = {
        "dog": (lambda t: lb.autograd.difference_of_gaussians(t, 1.0, 2.0, mode=mode),
                lambda e: oracle.difference_of_gaussians(e.astype(np.float32), 1.0, 2.0, mode=mode)),
        "laplace": (lambda t: lb.autograd.gaussian_laplace(t, 1.5, mode=mode),
                    lambda e: oracle.gaussian_laplace(e.astype(np.float32), 1.5, mode=mode)),
        "unsharp": (lambda t: lb.autograd.unsharp_mask(t, 1.2, 0.7, mode=mode),
                    lambda e: oracle.unsharp_mask(e.astype(np.float32), 1.2, 0.7, mode=mode)),
    }
    for name, (f, ref) in cases.items():
        x = dev(xn).requires_grad_(True)
        f(x).mul(dev(w)).sum().backward()
        want = (matrix(ref, shape).T @ wv).reshape(shape)
        oracle.assert_close(host(x.grad), want, RTOL, f"{name} {mode}")
    # Gradient magnitude: sum_a D_a^T (w d_a / |grad|).
    x = dev(xn).requires_grad_(True)
    lb.autograd.gaussian_grad_mag(x, 1.3, mode=mode).mul(dev(w)).sum().backward()
    mats = [matrix(lambda e, o=o: oracle.gaussian_blur(e, [1.3], orders=o, mode=mode), shape)
            for o in ((1, 0), (0, 1))]
    d = [m @ xn.reshape(-1).astype(np.float64) for m in mats]
    mag = np.sqrt(sum(di * di for di in d))
    want = sum(m.T @ (wv * di / mag) for m, di in zip(mats, d)).reshape(shape)
    oracle.assert_close(host(x.grad), want, RTOL, f"grad_mag {mode}")


# ---------------------------------------------------------------------------
# FFT convolution (the deconvolution's forward model)


@pytest.mark.parametrize("shape,kshape", [((12, 10), (3, 5)), ((11, 9), (4, 2)), ((5, 6, 7), (3, 2, 3))])
def test_fft_convolve_and_its_gradients(oracle, shape, kshape):
    rng = np.random.default_rng(len(shape) * 10 + kshape[0])
    x = rng.uniform(0.2, 1.5, shape).astype(np.float32)
    psf = rng.uniform(0.0, 1.0, kshape).astype(np.float32)
    g = rng.standard_normal(shape).astype(np.float32)
    flip = tuple(slice(None, None, -1) for _ in kshape)
    conv = lambda xx, pp: oracle.correlate_nd(np.asarray(xx, np.float64), np.asarray(pp, np.float64)[flip],
                                              mode="constant")
    got = host(lb.fft_convolve(dev(x), dev(psf)))
    oracle.assert_close(got, conv(x, psf), RTOL, "forward")
    gp, gx = lb.fft_convolve_backward(dev(x), dev(psf), dev(g))
    A = matrix(lambda e: conv(e, psf), shape)
    oracle.assert_close(host(gx), (A.T @ g.reshape(-1).astype(np.float64)).reshape(shape), RTOL, "grad x")
    B = matrix(lambda e: conv(x, e), kshape)
    oracle.assert_close(host(gp), (B.T @ g.reshape(-1).astype(np.float64)).reshape(kshape), RTOL, "grad psf")
    # Through autograd.
    xt, pt = dev(x).requires_grad_(True), dev(psf).requires_grad_(True)
    lb.autograd.fft_convolve(xt, pt).mul(dev(g)).sum().backward()
    oracle.assert_close(host(xt.grad), host(gx), RTOL, "autograd x")
    oracle.assert_close(host(pt.grad), host(gp), RTOL, "autograd psf")


# ---------------------------------------------------------------------------
# Richardson-Lucy reverse pass vs FP64 finite differences


def _rl_loss64(oracle, obs, psf, w, T, eps):
    est = oracle.richardson_lucy_fft64(obs, psf, num_iter=T, clip=False, filter_epsilon=eps)
    return float(np.sum(w * est))


def _fd(fun, base, idx, h=1e-4):
    out = []
    for i in idx:
        p = base.copy().reshape(-1)
        p[i] += h
        lp = fun(p.reshape(base.shape))
        p[i] -= 2 * h
        lm = fun(p.reshape(base.shape))
        out.append((lp - lm) / (2 * h))
    return np.array(out)


RL_CASES = [
    # obs shape, psf shape, iterations, checkpoint_every
    ((24, 20), (5, 5), 6, 2),
    ((19, 22), (4, 4), 5, 5),        # even sides: two centres
    ((8, 12, 10), (3, 5, 5), 4, 3),
    ((6, 10, 9), (2, 4, 3), 3, 1),
]


@pytest.mark.parametrize("case", range(len(RL_CASES)))
def test_rl_gradients_against_fp64_finite_differences(oracle, case):
    shape, kshape, T, K = RL_CASES[case]
    rng = np.random.default_rng(100 + case)
    obs = rng.uniform(0.5, 2.0, shape)
    psf = rng.uniform(0.2, 1.0, kshape)
    w = rng.standard_normal(shape)
    eps = 1e-6
    gp, gx = lb.richardson_lucy_backward(dev(obs), dev(psf), dev(w), num_iter=T, filter_epsilon=eps,
                                         checkpoint_every=K)
    gp, gx = host(gp), host(gx)
    obs32, psf32 = obs.astype(np.float32).astype(np.float64), psf.astype(np.float32).astype(np.float64)
    kidx = rng.choice(psf.size, size=min(64, psf.size), replace=False)
    fd_p = _fd(lambda p: _rl_loss64(oracle, obs32, p, w, T, eps), psf32, kidx)
    oracle.assert_close(gp.reshape(-1)[kidx], fd_p, FD_RTOL, "psf gradient")
    xidx = rng.choice(obs.size, size=24, replace=False)
    fd_x = _fd(lambda o: _rl_loss64(oracle, o, psf32, w, T, eps), obs32, xidx)
    oracle.assert_close(gx.reshape(-1)[xidx], fd_x, FD_RTOL, "observation gradient")


def test_rl_gradient_does_not_depend_on_checkpoint_spacing(oracle):
    rng = np.random.default_rng(7)
    obs = dev(rng.uniform(0.5, 2.0, (6, 18, 16)))
    psf = dev(rng.uniform(0.2, 1.0, (3, 5, 5)))
    w = dev(rng.standard_normal((6, 18, 16)))
    ref = None
    for K in (1, 3, 7, 50):
        gp, gx = lb.richardson_lucy_backward(obs, psf, w, num_iter=7, filter_epsilon=1e-6, checkpoint_every=K)
        cur = (host(gp), host(gx))
        if ref is None:
            ref = cur
        else:
            oracle.assert_close(cur[0], ref[0], 1e-6, f"psf K={K}")
            oracle.assert_close(cur[1], ref[1], 1e-6, f"obs K={K}")


def test_rl_backward_rejects_what_it_cannot_differentiate():
    x = dev(np.ones((8, 8)))
    p = dev(np.ones((3, 3)))
    g = dev(np.ones((8, 8)))
    with pytest.raises(lb.LucemError):
        lb.richardson_lucy_backward(x, p, g, checkpoint_every=0)
    with pytest.raises(lb.LucemError):
        lb.richardson_lucy_backward(x, p, dev(np.ones((8, 9))))


def test_blind_psf_fit_gradient(oracle):
    """A learnable PSF (softplus, then normalised) through unrolled RL on a
    batch of volumes, gradient w.r.t. the raw parameters against FP64 central
    differences of the same pipeline on the oracle."""
    rng = np.random.default_rng(11)
    B, shape, kshape, T, K = 2, (6, 16, 14), (3, 5, 5), 6, 2
    truth = rng.uniform(0.2, 1.0, (B,) + shape).astype(np.float32).astype(np.float64)
    theta = rng.standard_normal(kshape) * 0.3
    blur = np.full(kshape, 1.0 / np.prod(kshape))
    obs = np.stack([oracle.correlate_nd(t, blur, mode="constant") for t in truth])
    obs = (obs + rng.uniform(0.0, 0.1, obs.shape)).astype(np.float32).astype(np.float64)
    eps = 1e-6

    def psf_of(th):
        sp = np.log1p(np.exp(th))
        return sp / sp.sum()

    def loss64(th):
        p = psf_of(th)
        tot = 0.0
        for b in range(B):
            est = oracle.richardson_lucy_fft64(obs[b], p, num_iter=T, clip=False, filter_epsilon=eps)
            tot += float(np.mean((est - truth[b]) ** 2))
        return tot

    th = dev(theta).requires_grad_(True)
    sp = torch.nn.functional.softplus(th)
    psf = sp / sp.sum()
    est = lb.autograd.richardson_lucy(dev(obs), psf, num_iter=T, filter_epsilon=eps, checkpoint_every=K)
    loss = ((est - dev(truth)) ** 2).mean(dim=tuple(range(1, est.dim()))).sum()
    loss.backward()
    got = host(th.grad).reshape(-1)
    th32 = theta.astype(np.float32).astype(np.float64)
    idx = rng.choice(theta.size, size=32, replace=False)
    fd = _fd(loss64, th32, idx)
    oracle.assert_close(got[idx], fd, FD_RTOL, "blind PSF fit")


def test_psf_fit_configuration_gradient_on_64_taps(oracle):
    """The blind-PSF-fit configuration's operator (PSF 15 x 9 x 9 through
    softplus and normalisation, 20 unrolled iterations, checkpoints every 5)
    on one 16 x 64 x 64 bead volume: d loss / d theta on 64 taps against FP64
    central differences, h = 1e-4, relative 1e-3."""
    shape, kshape, T, K = (16, 64, 64), (15, 9, 9), 20, 5
    obs, _ = lb.synth.bead_volume(shape=shape, n_beads=40, psf_shape=kshape, psf_sigmas=(2.0, 1.2, 1.2), seed=77)
    obs = obs.astype(np.float64) / float(obs.max())
    rng = np.random.default_rng(78)
    truth = rng.uniform(0.0, 1.0, shape).astype(np.float32).astype(np.float64)
    theta = (rng.standard_normal(kshape) * 0.2).astype(np.float32).astype(np.float64)
    eps = 1e-6

    def loss64(th):
        sp = np.log1p(np.exp(th))
        est = oracle.richardson_lucy_fft64(obs, sp / sp.sum(), num_iter=T, clip=False, filter_epsilon=eps)
        return float(np.mean((est - truth) ** 2))

    th = dev(theta).requires_grad_(True)
    sp = torch.nn.functional.softplus(th)
    est = lb.autograd.richardson_lucy(dev(obs), sp / sp.sum(), num_iter=T, filter_epsilon=eps, checkpoint_every=K)
    ((est - dev(truth)) ** 2).mean().backward()
    got = host(th.grad).reshape(-1)
    idx = rng.choice(theta.size, size=64, replace=False)
    oracle.assert_close(got[idx], _fd(loss64, theta, idx), FD_RTOL, "15x9x9 PSF, 20 iterations")


@pytest.mark.parametrize("shape,kshape,T,gauss", [((40, 36), (7, 6), 8, False), ((12, 30, 28), (5, 7, 7), 6, False),
                                                  ((40, 36), (6, 9), 8, True), ((12, 30, 28), (5, 7, 7), 6, True)])
def test_rl_gradients_against_the_fp64_reverse_oracle(oracle, shape, kshape, T, gauss):
    """Every PSF tap and every observation pixel against the FP64 reverse
    pass (itself checked against central differences on the host); a
    Gaussian PSF takes the factored (separable) transfer-function path."""
    rng = np.random.default_rng(sum(shape))
    obs = rng.uniform(0.5, 2.0, shape).astype(np.float32).astype(np.float64)
    if gauss:
        psf = lb.synth.gaussian_psf(kshape, [1.3 + 0.2 * i for i in range(len(kshape))])
    else:
        psf = rng.uniform(0.2, 1.0, kshape)
    psf = psf.astype(np.float32).astype(np.float64)
    w = rng.standard_normal(shape).astype(np.float32).astype(np.float64)
    gp, gx = lb.richardson_lucy_backward(dev(obs), dev(psf), dev(w), num_iter=T, filter_epsilon=1e-6,
                                         checkpoint_every=3)
    wp, wx = oracle.richardson_lucy_backward_fft64(obs, psf, w, num_iter=T, filter_epsilon=1e-6)
    oracle.assert_close(host(gp), wp, FD_RTOL, "psf gradient")
    oracle.assert_close(host(gx), wx, FD_RTOL, "observation gradient")


@pytest.mark.parametrize("gauss", [False, True])
def test_batched_rl_backward_sums_the_psf_gradient(gauss):
    """One call over a batch of volumes (one PSF): the observation gradients
    equal the single-volume calls' bit for bit, the PSF gradient is their sum
    (1e-5: the batch is summed inside the cross-spectrum accumulation)."""
    rng = np.random.default_rng(41 + gauss)
    obs = rng.uniform(0.5, 2.0, (3, 8, 20, 18)).astype(np.float32)
    kshape = (3, 5, 5)
    psf = (lb.synth.gaussian_psf(kshape, (1.0, 1.3, 1.1)) if gauss else rng.uniform(0.2, 1.0, kshape)).astype(np.float32)
    w = rng.standard_normal(obs.shape).astype(np.float32)
    kw = dict(num_iter=6, filter_epsilon=1e-6, checkpoint_every=2)
    gp, gx = lb.richardson_lucy_backward(dev(obs), dev(psf), dev(w), **kw)
    gp_sum = np.zeros(kshape)
    for b in range(obs.shape[0]):
        gpb, gxb = lb.richardson_lucy_backward(dev(obs[b]), dev(psf), dev(w[b]), **kw)
        np.testing.assert_array_equal(host(gx)[b], host(gxb))
        gp_sum += host(gpb)
    np.testing.assert_allclose(host(gp), gp_sum, rtol=1e-5, atol=1e-5 * np.abs(gp_sum).max())
