"""The pipeline stage on the device: run_op / run_chain equal the direct
operator calls (device input: zero-copy, results on the device; NumPy u16
input: raw upload, the cast and scale fused into the first kernel), and the
reference's tiled-equals-whole property (engine/lucem-pipeline/src/custom.rs:
478-495: halo from Op.halo(), blocks of lucem_schedule, within 1e-3) for the
Gaussian operators and the Richardson-Lucy node."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb
from lucem_b200 import pipeline as P

pytestmark = pytest.mark.gpu


def image(shape, seed=0):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:shape[0], 0:shape[1]].astype(np.float64)
    img = np.full(shape, 20.0)
    for _ in range(10):
        cy, cx, s = rng.uniform(0, shape[0]), rng.uniform(0, shape[1]), rng.uniform(1.5, 4)
        img += rng.uniform(100, 900) * np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2 * s * s))
    return img.astype(np.float32)


SPECS = ['{"op": "gaussian_blur", "sigma": 2.0}',
         '{"op": "unsharp_mask", "sigma": 1.5, "amount": 0.7}',
         '{"op": "difference_of_gaussians", "low_sigma": 1.0, "high_sigma": 3.0}',
         '{"op": "frangi", "sigma_min": 1.0, "sigma_max": 3.0, "black_ridges": false}',
         '{"op": "sato", "sigma_min": 1.0, "sigma_max": 3.0, "black_ridges": true}',
         '{"op": "richardson_lucy", "num_iter": 8, "psf_sigma": 1.5, "clip": false, "filter_epsilon": 1e-6}']


def direct(spec, x):
    op = P.parse_op(spec)
    p = op.params
    if op.op == "gaussian_blur":
        return lb.gaussian_blur(x, [p["sigma"]] * 2)
    if op.op == "unsharp_mask":
        return lb.unsharp_mask(x, [p["sigma"]] * 2, p["amount"])
    if op.op == "difference_of_gaussians":
        return lb.difference_of_gaussians(x, [p["low_sigma"]] * 2, [p["high_sigma"]] * 2)
    if op.op in ("frangi", "sato"):
        fn = lb.frangi if op.op == "frangi" else lb.sato
        return fn(x, P.ridge_sigmas(p["sigma_min"], p["sigma_max"]), black_ridges=p["black_ridges"])
    psf = torch.from_numpy(op.psf()).cuda()
    return lb.richardson_lucy(x, psf, num_iter=p["num_iter"], clip=p["clip"], filter_epsilon=p["filter_epsilon"],
                              mode="constant")


@pytest.mark.parametrize("spec", SPECS)
def test_run_op_equals_the_direct_call(spec):
    x = torch.from_numpy(image((96, 120))).cuda()
    got = P.run_op(spec, [x])
    assert isinstance(got, torch.Tensor) and got.is_cuda
    assert torch.equal(got, direct(spec, x))
    # NumPy in, NumPy out (one upload, one download).
    host = P.run_op(spec, [x.cpu().numpy()])
    assert isinstance(host, np.ndarray) and np.array_equal(host, got.cpu().numpy())


@pytest.mark.parametrize("spec", SPECS)
def test_u16_upload_with_the_fused_cast(spec, oracle):
    """The raw u16 tile goes to the device at 2 bytes per pixel; the cast and
    the input scale happen in the first kernel.  Same result as the host
    decode to f32 (x * scale) within 1e-6."""
    img = (image((80, 100), seed=3) * 40).astype(np.uint16)
    scale = 1.0 / 65535.0
    got = P.run_op(spec, [img], input_scale=scale)
    want = P.run_op(spec, [(img.astype(np.float32) * np.float32(scale))])
    oracle.assert_close(got.astype(np.float64), want.astype(np.float64), 1e-6, spec)


def test_run_chain_stays_on_the_device():
    x = torch.from_numpy(image((64, 64))).cuda()
    specs = [SPECS[0], SPECS[5], SPECS[2]]
    got = P.run_chain(specs, x)
    want = x
    for s in specs:
        want = direct(s, want)
    assert torch.equal(got, want)
    with pytest.raises(ValueError, match="at least one"):
        P.run_chain([], x)


@pytest.mark.parametrize("spec,block", [(SPECS[0], 48), (SPECS[2], 40), (SPECS[5], 64)])
def test_tiled_equals_whole(spec, block, oracle):
    """custom.rs:478-495: blocks of lucem_schedule with the operator's halo,
    each run on its read box and cropped to its owned box, equal the whole
    image's result within 1e-3 (the Richardson-Lucy node with zero padding:
    its halo 2 num_iter ceil(3 sigma) keeps the tile borders' padding away
    from the owned pixels)."""
    img = image((150, 170), seed=5)
    x = torch.from_numpy(img).cuda()
    op = P.parse_op(spec)
    h = op.halo()
    whole = P.run_op(spec, [x]).cpu().numpy().astype(np.float64)
    tiled = np.zeros_like(whole)
    for b in lb.schedule((1,) + img.shape, (1, block, block), (0, h, h)):
        ry, rx = b.read_origin[1], b.read_origin[2]
        rh, rw = b.read_size[1], b.read_size[2]
        oy, ox = b.origin[1], b.origin[2]
        sh, sw = b.size[1], b.size[2]
        part = P.run_op(spec, [x[ry:ry + rh, rx:rx + rw].contiguous()]).cpu().numpy()
        tiled[oy:oy + sh, ox:ox + sw] = part[oy - ry:oy - ry + sh, ox - rx:ox - rx + sw]
    oracle.assert_close(tiled, whole, 1e-3, spec)
