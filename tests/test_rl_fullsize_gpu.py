"""Richardson-Lucy at the benchmarked sizes, as benchmarked, against FP64.

- the 64 x 512 x 512 bead volume with the 31 x 15 x 15 Gaussian PSF, 50
  iterations on the 128 x 1024 x 1024 grid (the headline workload);
- the same volume with a non-separable PSF (the Gaussian plus a seeded
  asymmetric perturbation of 1e-3 of its peak), which takes the dense
  transfer-function path;
- the 256 uneven 2-D bead images (sides 256..2048, PSF sigma 1..3), 30
  iterations, as one planned batch.

The FP64 result comes from cuFFT in float64 (tests/fp64_cufft.py), pinned here
to the host FP64 oracle (oracle.richardson_lucy_fft64) on the full grid.
Tolerance 1e-4 with the reference's assert_close semantics
(crates/lucem-core/src/test_support.rs:42-50), the RL tolerance the reference
uses (crates/lucem-ops/src/restore/deconvolve.rs:517-539)."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

import fp64_cufft as F

pytestmark = pytest.mark.gpu

RTOL = 1e-4
GRID = (128, 1024, 1024)


def perturbed_psf(psf, seed=0x6C7563656D + 11, amount=1e-3):
    """The Gaussian PSF plus a seeded non-negative asymmetric term: no longer
    a product of per-axis factors."""
    rng = np.random.default_rng(seed)
    p = psf.astype(np.float64)
    p = p + amount * p.max() * rng.uniform(0.0, 1.0, p.shape) * (np.arange(p.shape[2]) / p.shape[2])[None, None, :]
    return (p / p.sum()).astype(np.float32)


def test_fp64_crosscheck_matches_the_host_oracle_on_the_full_grid(oracle):
    """cuFFT FP64 against scipy FP64 (the host oracle), headline volume and grid,
    two iterations, separable and non-separable PSFs."""
    obs, psf = lb.synth.bead_volume()
    for p in (psf, perturbed_psf(psf)):
        want = oracle.richardson_lucy_fft64(obs, p, num_iter=2, filter_epsilon=1e-6, grid=GRID)
        got = F.richardson_lucy(obs, p, 2, 1e-6, GRID).cpu().numpy()
        assert oracle.max_rel_err(got, want) < 1e-10


def run_timed(y, p, num_iter):
    """richardson_lucy on the headline grid; also returns the pass kinds that ran."""
    ws = lb.Workspace()
    ws.set_timing(True)
    got = lb.richardson_lucy(y, torch.from_numpy(p).cuda(), num_iter=num_iter, clip=False, filter_epsilon=1e-6,
                             mode="constant", grid=GRID, workspace=ws)
    kinds = ws.timings()
    ws.set_timing(False)
    return got, kinds


def test_headline_volume_50_iterations_against_fp64():
    obs, psf = lb.synth.bead_volume()
    y = torch.from_numpy(obs).cuda()
    got, kinds = run_timed(y, psf, 50)
    # The Gaussian PSF is separable: per-axis convolutions on the row spectra,
    # no y-forward / y-inverse passes through the full y spectrum.
    assert "rl_col_forward" not in kinds and "rl_col_inverse" not in kinds
    want = F.richardson_lucy(y, psf, 50, 1e-6, GRID)
    err = F.max_rel_err(got, want)
    print(f"headline 50 iterations: max rel err vs FP64 {err:.3e}")
    assert err <= RTOL


def test_dense_psf_volume_50_iterations_against_fp64():
    obs, psf = lb.synth.bead_volume()
    p = perturbed_psf(psf)
    y = torch.from_numpy(obs).cuda()
    got, kinds = run_timed(y, p, 50)
    # Not separable: the dense transfer function through the full spectrum.
    assert "rl_col_forward" in kinds and "rl_col_inverse" in kinds
    want = F.richardson_lucy(y, p, 50, 1e-6, GRID)
    err = F.max_rel_err(got, want)
    print(f"dense psf 50 iterations: max rel err vs FP64 {err:.3e}")
    assert err <= RTOL


@pytest.mark.parametrize("mode", ["reflect", "wrap", "nearest", "mirror", "constant"])
def test_separable_volume_every_mode_against_direct(oracle, mode):
    """The separable factorisation (y convolution then z convolution on the
    row spectra) in every pad mode, against the reference's direct iteration."""
    rng = np.random.default_rng(17)
    obs = rng.uniform(0.5, 2.0, (14, 33, 28)).astype(np.float32)
    psf = lb.synth.gaussian_psf((7, 5, 5), (1.5, 1.0, 0.8)).astype(np.float32)
    got = lb.richardson_lucy(torch.from_numpy(obs).cuda(), torch.from_numpy(psf).cuda(), num_iter=6, clip=False,
                             filter_epsilon=1e-6, mode=mode)
    torch.cuda.synchronize()
    want = oracle.richardson_lucy(obs, psf, num_iter=6, clip=False, filter_epsilon=1e-6, mode=mode)
    oracle.assert_close(got.cpu().numpy(), want.astype(np.float64), RTOL, mode)


def test_even_separable_psf_against_fp64(oracle):
    """Even PSF sides: the convolution and correlation centres differ, so each
    has its own pair of axis factors."""
    rng = np.random.default_rng(19)
    obs = rng.uniform(0.5, 2.0, (20, 40, 36)).astype(np.float32)
    psf = lb.synth.gaussian_psf((6, 8, 4), (1.2, 1.8, 0.9)).astype(np.float32)
    got = lb.richardson_lucy(torch.from_numpy(obs).cuda(), torch.from_numpy(psf).cuda(), num_iter=12, clip=False,
                             filter_epsilon=1e-6, mode="constant")
    torch.cuda.synchronize()
    want = oracle.richardson_lucy_fft64(obs, psf, num_iter=12, filter_epsilon=1e-6)
    oracle.assert_close(got.cpu().numpy(), want, RTOL, "even psf")


def test_uneven_batch_at_config_sizes_against_fp64():
    """256 images, sides U[256, 2048], 30 iterations, one planned batch; every
    image against FP64 on the grid the plan chose for it."""
    specs = lb.synth.uneven_bead_batch(256)
    images, psfs = lb.synth.bead_batch(specs, device="cuda")
    plan = lb.RlBatch(images, psfs, num_iter=30, clip=False, filter_epsilon=1e-6, mode="constant")
    outs = plan.run()
    grids, _, _ = plan.info()
    torch.cuda.synchronize()
    worst = 0.0
    for i, (x, k, g) in enumerate(zip(images, psfs, grids)):
        want = F.richardson_lucy(x, k, 30, 1e-6, g)
        err = F.max_rel_err(outs[i], want)
        worst = max(worst, err)
        assert err <= RTOL, f"image {i} {tuple(x.shape)} grid {g}: {err:.3e}"
    print(f"batch of 256, 30 iterations: worst max rel err vs FP64 {worst:.3e}")
    plan.close()
