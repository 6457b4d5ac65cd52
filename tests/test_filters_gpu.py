"""Gaussian family on the GPU (sm_100a kernels through the C ABI) against the
oracle's f32 restatement of the reference, assert_close semantics of
crates/lucem-core/src/test_support.rs:42-50 at rtol 1e-5."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu

RTOL = 1e-5
MODES = ["reflect", "constant", "nearest", "mirror", "wrap"]


def sample_f64(n):
    i = np.arange(n, dtype=np.int64)
    return ((i * 7919 + 104729) % 1013).astype(np.float64) * 0.1 - 50.0


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("dims", [[1], [7], [32, 33], [5, 1, 9], [3, 40, 1500], [1100, 6]])
def test_correlate_1d_reference_cases(oracle, dims):
    """crates/lucem-ops/src/filter/convolve.rs:211-228 on the device."""
    x = sample_f64(int(np.prod(dims))).astype(np.float32).reshape(dims)
    xd = dev(x)
    for axis in range(len(dims)):
        for w, origin in (([1.0, -2.0, 3.0], 0), ([0.5] * 4, -1)):
            for mode in MODES:
                got = host(lb.correlate_1d(xd, w, axis=axis, mode=mode, cval=1.5, origin=origin))
                want = oracle.correlate_1d(x, w, axis=axis, mode=mode, cval=1.5, origin=origin)
                oracle.assert_close(got, want.astype(np.float64), RTOL, f"{dims} ax{axis} {mode}")


def test_convolve_1d_is_mirrored_correlation(oracle):
    x = sample_f64(257).astype(np.float32)
    w = [0.1, 0.2, 0.3, 0.4]
    got = host(lb.convolve_1d(dev(x), w, origin=0))
    want = oracle.correlate_1d(x, w[::-1], origin=-1)
    oracle.assert_close(got, want.astype(np.float64), RTOL, "convolve")


@pytest.mark.parametrize("shape", [(1, 1), (7, 5), (64, 64), (65, 129), (300, 310), (3, 37, 41)])
@pytest.mark.parametrize("mode", MODES)
def test_gaussian_blur_f32(oracle, shape, mode):
    x = sample_f64(int(np.prod(shape))).astype(np.float32).reshape(shape)
    for sigma in (0.7, 2.0, 3.3):
        got = host(lb.gaussian_blur(dev(x), sigma, mode=mode, cval=1.5))
        want = oracle.gaussian_blur(x, [sigma], mode=mode, cval=1.5)
        oracle.assert_close(got, want.astype(np.float64), RTOL, f"{shape} {mode} s={sigma}")


def test_gaussian_blur_orders_axes_radii_channel(oracle):
    x = sample_f64(4 * 33 * 47).astype(np.float32).reshape(4, 33, 47)
    xd = dev(x)
    cases = [
        dict(sigmas=[1.5, 2.5], orders=[1, 2], channel_axis=0),
        dict(sigmas=[2.0], orders=[3], axes=[2]),
        dict(sigmas=[1.0, 0.0, 2.0]),
        dict(sigmas=[1.2, 1.9, 2.7], orders=[0, 1, 0], mode="nearest"),
        dict(sigmas=[2.0], radii=[3]),
        dict(sigmas=[2.0], axes=[2, 1]),
        dict(sigmas=[0.0]),
        dict(sigmas=[40.0], axes=[1]),  # radius 160 > the fused kernel's: per-axis passes
    ]
    for c in cases:
        kw = dict(c)
        sig = kw.pop("sigmas")
        mode = kw.pop("mode", "reflect")
        got = host(lb.gaussian_blur(xd, sig, mode=mode, cval=0.5, **kw))
        want = oracle.gaussian_blur(x, sig, mode=mode, cval=0.5, **{k: v for k, v in kw.items()})
        oracle.assert_close(got, want.astype(np.float64), RTOL, str(c))


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_integer_input_cast_is_fused(oracle, dtype):
    rng = np.random.default_rng(3)
    hi = 255 if dtype == np.uint8 else 65535
    x = rng.integers(0, hi + 1, (130, 257)).astype(dtype)
    xt = torch.from_numpy(x.astype(np.int32)).cuda().to(torch.uint8 if dtype == np.uint8 else torch.uint16)
    got = host(lb.gaussian_blur(xt, 2.0))
    want = oracle.gaussian_blur(x.astype(np.float32), [2.0])
    oracle.assert_close(got, want.astype(np.float64), RTOL, str(dtype))
    got = host(lb.gaussian_blur(xt, 2.0, input_scale=1.0 / hi))
    oracle.assert_close(got, want.astype(np.float64) / hi, RTOL, "scaled")
    # 3-D volume: a per-axis pass reading the integers, then the fused 2-D pass
    x3 = rng.integers(0, hi + 1, (6, 40, 50)).astype(dtype)
    x3t = torch.from_numpy(x3.astype(np.int32)).cuda().to(xt.dtype)
    got = host(lb.gaussian_blur(x3t, [1.0, 2.0, 1.5]))
    want = oracle.gaussian_blur(x3.astype(np.float32), [1.0, 2.0, 1.5])
    oracle.assert_close(got, want.astype(np.float64), RTOL, "3-D")


def test_gaussian_1d(oracle):
    x = sample_f64(9 * 70).astype(np.float32).reshape(9, 70)
    for axis in (0, 1, -1):
        for order in (0, 1, 2):
            got = host(lb.gaussian_1d(dev(x), 1.7, axis=axis, order=order, mode="mirror"))
            want = oracle.gaussian_blur(x, [1.7], orders=[order], axes=[axis], mode="mirror")
            oracle.assert_close(got, want.astype(np.float64), RTOL, f"ax{axis} o{order}")


@pytest.mark.parametrize("shape", [(37, 41), (2, 70, 90), (5, 20, 30)])
def test_composites(oracle, shape):
    x = sample_f64(int(np.prod(shape))).astype(np.float32).reshape(shape)
    xd = dev(x)
    oracle.assert_close(host(lb.difference_of_gaussians(xd, 1.0, 3.0)),
                        oracle.difference_of_gaussians(x, [1.0], [3.0]).astype(np.float64), RTOL, "dog")
    oracle.assert_close(host(lb.gaussian_laplace(xd, 2.0)),
                        oracle.gaussian_laplace(x, [2.0]).astype(np.float64), RTOL, "log")
    oracle.assert_close(host(lb.gaussian_grad_mag(xd, 1.5)),
                        oracle.gaussian_grad_mag(x, [1.5]).astype(np.float64), RTOL, "gradmag")
    oracle.assert_close(host(lb.unsharp_mask(xd, 2.0, 0.7)),
                        oracle.unsharp_mask(x, [2.0], 0.7).astype(np.float64), RTOL, "unsharp")
    # anisotropic sigmas take the per-axis composition
    s = [1.0] * (x.ndim - 1) + [2.0]
    oracle.assert_close(host(lb.difference_of_gaussians(xd, s, 3.0)),
                        oracle.difference_of_gaussians(x, s, [3.0]).astype(np.float64), RTOL, "dog aniso")


def test_family_equals_the_separate_ops(oracle):
    """The multi-response pass of the tiled workload: G(1), G(2), G(4), DoG(1,3)."""
    rng = np.random.default_rng(11)
    x = rng.integers(0, 4000, (2, 200, 333)).astype(np.uint16)
    xt = torch.from_numpy(x.astype(np.int32)).cuda().to(torch.uint16)
    outs = lb.gaussian_family(xt, [("gaussian", 1.0), ("gaussian", 2.0), ("gaussian", 4.0), ("dog", 1.0, 3.0)])
    xf = x.astype(np.float32)
    wants = [oracle.gaussian_blur(xf, [1.0], axes=[1, 2]), oracle.gaussian_blur(xf, [2.0], axes=[1, 2]),
             oracle.gaussian_blur(xf, [4.0], axes=[1, 2]),
             oracle.gaussian_blur(xf, [1.0], axes=[1, 2]) - oracle.gaussian_blur(xf, [3.0], axes=[1, 2])]
    for o, w, n in zip(outs, wants, ["g1", "g2", "g4", "dog"]):
        oracle.assert_close(host(o), w.astype(np.float64), RTOL, n)
    outs = lb.gaussian_family(xt, [("laplace", 1.5), ("grad_mag", 2.0), ("unsharp", 1.0, 0.5)], mode="wrap")
    planes = [oracle.gaussian_laplace(xf[i], [1.5], mode="wrap") for i in range(2)]
    oracle.assert_close(host(outs[0]), np.stack(planes).astype(np.float64), RTOL, "log")
    planes = [oracle.gaussian_grad_mag(xf[i], [2.0], mode="wrap") for i in range(2)]
    oracle.assert_close(host(outs[1]), np.stack(planes).astype(np.float64), RTOL, "gradmag")
    planes = [oracle.unsharp_mask(xf[i], [1.0], 0.5, mode="wrap") for i in range(2)]
    oracle.assert_close(host(outs[2]), np.stack(planes).astype(np.float64), RTOL, "unsharp")


def test_blob_image_config_full_size(oracle):
    """The 2048^2 u16 blob image, sigma 2, reflect, f32 out."""
    x = lb.synth.blob_image()
    xt = torch.from_numpy(x.astype(np.int32)).cuda().to(torch.uint16)
    got = host(lb.gaussian_blur(xt, 2.0))
    want = oracle.gaussian_blur(x.astype(np.float32), [2.0])
    oracle.assert_close(got, want.astype(np.float64), RTOL, "blob image")
    want64 = oracle.gaussian_blur(x.astype(np.float64), [2.0])
    assert oracle.max_rel_err(got, want64) < 1e-6


@pytest.mark.parametrize("persistent", [True, False])
def test_tiled_walk_matches_per_block_filtering(oracle, persistent):
    """engine/lucem-pipeline/src/custom.rs:199-251: each block's read part is
    filtered with reflect at the read part's borders, the owned part kept.
    Uneven edge blocks included; with halo >= radius it equals the whole image
    (custom.rs:478-495)."""
    rng = np.random.default_rng(2)
    C, H, W = 2, 300, 455
    x = rng.integers(0, 5000, (C, H, W)).astype(np.uint16)
    xt = torch.from_numpy(x.astype(np.int32)).cuda().to(torch.uint16)
    resp = [("gaussian", 1.0), ("gaussian", 2.0), ("gaussian", 4.0), ("dog", 1.0, 3.0)]
    for halo in (32, 3):
        blocks = lb.schedule((1, H, W), (1, 128, 128), (0, halo, halo))
        outs = lb.gaussian_family_tiles(xt, blocks, resp, persistent=persistent)
        got = [host(o) for o in outs]
        xf = x.astype(np.float32)
        for c in range(C):
            for b in blocks:
                ry, rx, rh, rw = b.read_origin[1], b.read_origin[2], b.read_size[1], b.read_size[2]
                oy, ox = b.origin[1] - ry, b.origin[2] - rx
                part = np.ascontiguousarray(xf[c, ry:ry + rh, rx:rx + rw])
                g1 = oracle.gaussian_blur(part, [1.0])
                wants = [g1, oracle.gaussian_blur(part, [2.0]), oracle.gaussian_blur(part, [4.0]),
                         g1 - oracle.gaussian_blur(part, [3.0])]
                sl = (c, slice(b.origin[1], b.origin[1] + b.size[1]), slice(b.origin[2], b.origin[2] + b.size[2]))
                for k in range(4):
                    w = wants[k][oy:oy + b.size[1], ox:ox + b.size[2]]
                    oracle.assert_close(got[k][sl], w.astype(np.float64), RTOL, f"halo {halo} block {b.index} r{k}")
        if halo == 32:
            whole = oracle.gaussian_blur(x.astype(np.float32), [2.0], axes=[1, 2])
            assert np.abs(got[1] - whole).max() < 1e-3


@pytest.mark.parametrize("dtype,W", [(np.uint16, 1536), (np.uint16, 1030), (np.uint8, 1024), (np.float32, 1000)])
def test_persistent_walk_with_prefetch_equals_per_block(oracle, dtype, W):
    """The persistent walk copies each CTA's next tile window ahead
    (16-byte chunks when rows allow, else 4-byte); with ~4 tiles per CTA most
    tiles take that path.  Its responses must equal the per-block launches
    (no copies ahead) bit for bit, and the oracle on a block."""
    rng = np.random.default_rng(W)
    C, H = 3, 1000
    x = rng.integers(0, 250 if dtype == np.uint8 else 5000, (C, H, W)).astype(dtype)
    xt = torch.from_numpy(x.astype(np.int32)).cuda().to(getattr(torch, np.dtype(dtype).name))
    resp = [("gaussian", 1.0), ("gaussian", 2.0), ("gaussian", 4.0), ("dog", 1.0, 3.0)]
    for halo in (32, 3):
        blocks = lb.schedule((1, H, W), (1, 256, 256), (0, halo, halo))
        a = [host(o) for o in lb.gaussian_family_tiles(xt, blocks, resp, persistent=True)]
        b = [host(o) for o in lb.gaussian_family_tiles(xt, blocks, resp, persistent=False)]
        for k in range(4):
            assert np.array_equal(a[k], b[k]), (halo, k)
        blk = blocks[len(blocks) // 2]
        ry, rx, rh, rw = blk.read_origin[1], blk.read_origin[2], blk.read_size[1], blk.read_size[2]
        part = np.ascontiguousarray(x[1, ry:ry + rh, rx:rx + rw].astype(np.float32))
        w = oracle.gaussian_blur(part, [4.0])[blk.origin[1] - ry:blk.origin[1] - ry + blk.size[1],
                                              blk.origin[2] - rx:blk.origin[2] - rx + blk.size[2]]
        got = a[2][1, blk.origin[1]:blk.origin[1] + blk.size[1], blk.origin[2]:blk.origin[2] + blk.size[2]]
        oracle.assert_close(got, w.astype(np.float64), RTOL, f"halo {halo} prefetch block")


def test_errors_mirror_the_reference():
    x = torch.zeros((4, 5), device="cuda")
    with pytest.raises(lb.LucemError) as e:
        lb.gaussian_blur(x, [1.0, 2.0, 3.0])
    assert e.value.name == "INVALID_PARAMETER"
    with pytest.raises(lb.LucemError) as e:
        lb.gaussian_blur(x, -1.0)
    assert e.value.name == "INVALID_PARAMETER"
    with pytest.raises(lb.LucemError) as e:
        lb.gaussian_blur(x, 1.0, out=torch.zeros((5, 4), device="cuda"))
    assert e.value.name == "SHAPE_MISMATCH"
    with pytest.raises(lb.LucemError) as e:
        lb.gaussian_blur(x, 1.0, out=x)
    assert e.value.name == "ALIASED_BUFFERS"
    with pytest.raises(lb.LucemError) as e:
        lb.gaussian_blur(x, 1.0, axes=[2])
    assert e.value.name == "AXIS_OUT_OF_BOUNDS"
    with pytest.raises(lb.LucemError) as e:
        lb.gaussian_blur(x, 1.0, axes=[1, -1])
    assert e.value.name == "REPEATED_AXIS"
    with pytest.raises(lb.LucemError) as e:
        lb.correlate_1d(x, [1.0, 2.0, 3.0], origin=2)
    assert e.value.name == "INVALID_ORIGIN"
    with pytest.raises(lb.LucemError) as e:
        lb.correlate_1d(x, [])
    assert e.value.name == "INVALID_WEIGHTS"
    with pytest.raises(lb.LucemError) as e:
        lb.correlate_1d(x, [1.0, float("nan")])
    assert e.value.name == "INVALID_WEIGHTS"
    with pytest.raises(lb.LucemError) as e:
        lb.gaussian_blur(x, 1.0, mode="bogus")
    assert e.value.name == "UNKNOWN_PAD_MODE"
    # empty input: OK, no work
    e0 = torch.zeros((0, 7), device="cuda")
    assert lb.gaussian_blur(e0, 2.0).shape == (0, 7)
