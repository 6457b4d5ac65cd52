"""Richardson-Lucy on the GPU (FFT kernels through the C ABI) against the
oracle: the reference's direct-correlation iteration restated in f32 (small
sizes) and its FP64 FFT form (larger sizes).  Tolerance 1e-4 (assert_close
semantics), the reference's own RL tolerance."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu

RTOL = 1e-4
MODES = ["reflect", "constant", "nearest", "mirror", "wrap"]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_delta_psf_recovers_the_image(oracle):
    """crates/lucem-ops/src/restore/deconvolve.rs:517-539."""
    img = (np.arange(64, dtype=np.float32) / 64.0 * 0.8 + 0.1).reshape(8, 8)
    psf = np.zeros((3, 3), np.float32)
    psf[1, 1] = 1.0
    out = host(lb.richardson_lucy(dev(img), dev(psf), num_iter=15, clip=False))
    oracle.assert_close(out, img.astype(np.float64), 1e-4, "delta psf")


def test_box_psf_sharpens_like_the_reference(oracle):
    """crates/lucem-ops/src/restore/deconvolve.rs:551-566."""
    spot = np.full((8, 8), 0.1, np.float32)
    spot[4, 4] = 0.9
    box = np.full((3, 3), 1.0 / 9.0, np.float32)
    blurred = oracle.correlate_nd(spot, box, mode="reflect")
    restored = host(lb.richardson_lucy(dev(blurred), dev(box), num_iter=25, clip=True))
    assert restored[4, 4] > blurred[4, 4] + 0.15
    want = oracle.richardson_lucy(blurred, box, num_iter=25, clip=True)
    oracle.assert_close(restored, want.astype(np.float64), RTOL, "box psf")


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape,kshape", [((40, 53), (7, 5)), ((33, 30), (6, 4)), ((17, 64), (1, 9)),
                                          ((5, 7), (9, 9))])
def test_2d_against_direct_restatement(oracle, mode, shape, kshape):
    rng = np.random.default_rng(hash((shape, kshape)) % 2**32)
    obs = rng.uniform(0.5, 2.0, shape).astype(np.float32)
    psf = rng.uniform(0.0, 1.0, kshape).astype(np.float32)
    got = host(lb.richardson_lucy(dev(obs), dev(psf), num_iter=9, clip=False, filter_epsilon=1e-6, mode=mode))
    want = oracle.richardson_lucy(obs, psf, num_iter=9, clip=False, filter_epsilon=1e-6, mode=mode)
    oracle.assert_close(got, want.astype(np.float64), RTOL, f"{mode} {shape} {kshape}")


@pytest.mark.parametrize("mode", ["constant", "reflect", "wrap"])
def test_3d_against_direct_restatement(oracle, mode):
    rng = np.random.default_rng(7)
    obs = rng.uniform(0.5, 2.0, (12, 30, 26)).astype(np.float32)
    psf = rng.uniform(0.0, 1.0, (5, 7, 3)).astype(np.float32)
    got = host(lb.richardson_lucy(dev(obs), dev(psf), num_iter=8, clip=False, filter_epsilon=1e-6, mode=mode))
    want = oracle.richardson_lucy(obs, psf, num_iter=8, clip=False, filter_epsilon=1e-6, mode=mode)
    oracle.assert_close(got, want.astype(np.float64), RTOL, mode)


def test_clip_and_default_epsilon(oracle):
    rng = np.random.default_rng(9)
    obs = rng.uniform(0.0, 1.5, (31, 29)).astype(np.float32)
    obs[3:6, 4:9] = 0.0  # zero observations: the ratio guard is exercised
    psf = rng.uniform(0.0, 1.0, (5, 5)).astype(np.float32)
    got = host(lb.richardson_lucy(dev(obs), dev(psf), num_iter=6))
    want = oracle.richardson_lucy(obs, psf, num_iter=6)
    oracle.assert_close(got, want.astype(np.float64), RTOL, "defaults")
    assert got.max() <= 1.0 and got.min() >= -1.0


def test_bead_volume_with_the_config_psf_against_fp64(oracle):
    """A bead volume with the anisotropic 31 x 15 x 15 PSF, 50 iterations,
    eps 1e-6, zero padding: against the FP64 FFT oracle, automatic grid and
    a power-of-two grid."""
    obs, psf = lb.synth.bead_volume(shape=(24, 96, 80), n_beads=60, seed=123)
    want = oracle.richardson_lucy_fft64(obs, psf, num_iter=50, filter_epsilon=1e-6)
    for grid in (None, (64, 128, 128)):
        got = host(lb.richardson_lucy(dev(obs), dev(psf), num_iter=50, clip=False, filter_epsilon=1e-6,
                                      mode="constant", grid=grid))
        oracle.assert_close(got, want, RTOL, f"grid {grid}")


def test_uneven_2d_beads_against_fp64(oracle):
    for (h, w, s, seed) in [(257, 300, 1.3, 1), (311, 256, 2.9, 2)]:
        obs, psf = lb.synth.bead_image(h, w, s, seed=seed)
        got = host(lb.richardson_lucy(dev(obs), dev(psf), num_iter=30, clip=False, filter_epsilon=1e-6,
                                      mode="constant"))
        want = oracle.richardson_lucy_fft64(obs, psf, num_iter=30, filter_epsilon=1e-6)
        oracle.assert_close(got, want, RTOL, f"{h}x{w}")


def test_full_size_volume_first_iterations_against_fp64(oracle):
    """The 64 x 512 x 512 bead volume on the 128 x 1024 x 1024 grid: the first
    two iterations against the FP64 FFT oracle on the same grid."""
    obs, psf = lb.synth.bead_volume()
    got = host(lb.richardson_lucy(dev(obs), dev(psf), num_iter=2, clip=False, filter_epsilon=1e-6,
                                  mode="constant", grid=(128, 1024, 1024)))
    want = oracle.richardson_lucy_fft64(obs, psf, num_iter=2, filter_epsilon=1e-6, grid=(128, 1024, 1024))
    oracle.assert_close(got, want, RTOL, "full size")


def test_transfer_function_cache_follows_the_psf(oracle):
    rng = np.random.default_rng(4)
    obs = rng.uniform(0.5, 2.0, (20, 24)).astype(np.float32)
    p1 = rng.uniform(0.0, 1.0, (3, 3)).astype(np.float32)
    p2 = rng.uniform(0.0, 1.0, (3, 3)).astype(np.float32)
    ws = lb.Workspace()
    a = host(lb.richardson_lucy(dev(obs), dev(p1), num_iter=4, clip=False, mode="constant", workspace=ws))
    b = host(lb.richardson_lucy(dev(obs), dev(p2), num_iter=4, clip=False, mode="constant", workspace=ws))
    c = host(lb.richardson_lucy(dev(obs), dev(p1), num_iter=4, clip=False, mode="constant", workspace=ws))
    np.testing.assert_array_equal(a, c)
    oracle.assert_close(b, oracle.richardson_lucy(obs, p2, num_iter=4, clip=False, mode="constant").astype(np.float64),
                        RTOL, "second psf")


def test_errors_mirror_the_reference():
    x = torch.ones((8, 8), device="cuda")
    with pytest.raises(lb.LucemError) as e:
        lb.richardson_lucy(torch.ones(8, device="cuda"), torch.ones(3, device="cuda"))
    assert e.value.name == "INVALID_DIMENSION"
    with pytest.raises(lb.LucemError) as e:
        lb.richardson_lucy(x, torch.ones((3, 3, 3), device="cuda"))
    assert e.value.name == "INVALID_DIMENSION"
    with pytest.raises(lb.LucemError) as e:
        lb.richardson_lucy(x, torch.ones((0, 3), device="cuda"))
    assert e.value.name == "INVALID_WEIGHTS"
    with pytest.raises(lb.LucemError) as e:
        lb.richardson_lucy(x, torch.ones((3, 3), device="cuda"), num_iter=0)
    assert e.value.name == "INVALID_PARAMETER"
    with pytest.raises(lb.LucemError) as e:
        lb.richardson_lucy(x, torch.ones((3, 3), device="cuda"), out=x)
    assert e.value.name == "ALIASED_BUFFERS"
    with pytest.raises(lb.LucemError) as e:
        lb.richardson_lucy(x, torch.ones((3, 3), device="cuda"), mode="constant", grid=(8, 10))
    assert e.value.name == "INVALID_PARAMETER"
    assert lb.richardson_lucy(torch.ones((0, 5), device="cuda"), torch.ones((3, 3), device="cuda")).shape == (0, 5)


@pytest.mark.parametrize("py,px", [(64, 128), (128, 256), (256, 512), (512, 1024), (1024, 2048), (128, 2048),
                                   (1024, 128)])
@pytest.mark.parametrize("mode", ["constant", "reflect"])
def test_2d_register_fft_lengths(oracle, py, px, mode):
    """Every power-of-two length of the register-resident transforms (rows:
    packed lengths 64..1024, columns 64..1024) against the reference's direct
    iteration."""
    h, w = py // 2 - 3, px // 2 - 5
    rng = np.random.default_rng(py * 7 + px)
    obs = rng.uniform(0.5, 2.0, (h, w)).astype(np.float32)
    psf = rng.uniform(0.0, 1.0, (5, 7)).astype(np.float32)
    got = host(lb.richardson_lucy(dev(obs), dev(psf), num_iter=3, clip=False, filter_epsilon=1e-6, mode=mode,
                                  grid=(py, px)))
    want = oracle.richardson_lucy(obs, psf, num_iter=3, clip=False, filter_epsilon=1e-6, mode=mode)
    oracle.assert_close(got, want.astype(np.float64), RTOL, f"{py}x{px} {mode}")


@pytest.mark.parametrize("grid", [(64, 64, 128), (128, 256, 64), (256, 128, 256), (64, 512, 128), (64, 1024, 256)])
def test_3d_register_fft_lengths(oracle, grid):
    rng = np.random.default_rng(sum(grid))
    shape = (min(20, grid[0] // 2), min(40, grid[1] // 2 - 2), min(50, grid[2] // 2 - 3))
    obs = rng.uniform(0.5, 2.0, shape).astype(np.float32)
    psf = rng.uniform(0.0, 1.0, (3, 5, 3)).astype(np.float32)
    got = host(lb.richardson_lucy(dev(obs), dev(psf), num_iter=3, clip=False, filter_epsilon=1e-6, mode="reflect",
                                  grid=grid))
    want = oracle.richardson_lucy(obs, psf, num_iter=3, clip=False, filter_epsilon=1e-6, mode="reflect")
    oracle.assert_close(got, want.astype(np.float64), RTOL, str(grid))


@pytest.mark.parametrize("shape,kshape,gauss,mode", [((3, 12, 30, 26), (5, 7, 3), False, "constant"),
                                                     ((3, 12, 30, 26), (5, 7, 5), True, "constant"),
                                                     ((2, 10, 24, 20), (3, 5, 5), True, "reflect"),
                                                     ((4, 40, 53), (7, 5), False, "constant"),
                                                     ((3, 33, 30), (5, 5), True, "wrap")])
def test_leading_batch_axis_equals_one_call_per_volume(oracle, shape, kshape, gauss, mode):
    """A leading batch axis (one PSF for the batch) runs every volume in the
    same launches; each result equals the single-volume call bit for bit, and
    the oracle's iteration at 1e-4."""
    rng = np.random.default_rng(len(shape) * 100 + kshape[0])
    obs = rng.uniform(0.5, 2.0, shape).astype(np.float32)
    if gauss:
        psf = lb.synth.gaussian_psf(kshape, [1.0 + 0.3 * i for i in range(len(kshape))]).astype(np.float32)
    else:
        psf = rng.uniform(0.0, 1.0, kshape).astype(np.float32)
    kw = dict(num_iter=5, clip=False, filter_epsilon=1e-6, mode=mode)
    got = host(lb.richardson_lucy(dev(obs), dev(psf), **kw))
    for b in range(shape[0]):
        one = host(lb.richardson_lucy(dev(obs[b]), dev(psf), **kw))
        np.testing.assert_array_equal(got[b], one)
    want = oracle.richardson_lucy(obs[0], psf, **kw)
    oracle.assert_close(got[0], want.astype(np.float64), RTOL, f"{shape} {mode}")


def test_batched_fft_convolve_equals_one_call_per_volume():
    rng = np.random.default_rng(5)
    x = rng.uniform(0.0, 1.0, (3, 9, 20, 17)).astype(np.float32)
    p = rng.uniform(0.0, 1.0, (3, 5, 4)).astype(np.float32)
    got = host(lb.fft_convolve(dev(x), dev(p)))
    for b in range(3):
        np.testing.assert_array_equal(got[b], host(lb.fft_convolve(dev(x[b]), dev(p))))
