"""lucem_gaussian_batch: separate 2-D images of any sizes, one sigma set per
image, one persistent launch per set.  Every output equals gaussian_blur of
that image (the same tile kernel: bit for bit), which itself matches the
oracle at 1e-5; the oracle is checked here too on a few images."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu

RTOL = 1e-5
MODES = ["reflect", "constant", "nearest", "mirror", "wrap"]
SHAPES = [(1, 1), (3, 200), (65, 64), (64, 65), (130, 7), (257, 129), (40, 300), (2, 2), (199, 201)]


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dtype", [np.uint16, np.float32])
def test_batch_equals_per_image_blur(oracle, mode, dtype):
    rng = np.random.default_rng(len(mode))
    imgs = [(rng.integers(0, 4000, s) if dtype == np.uint16 else rng.standard_normal(s)).astype(dtype)
            for s in SHAPES]
    sigmas = [(0.7, 1.5, 3.0, 0.0)[i % 4] for i in range(len(imgs))]
    xs = [torch.from_numpy(x).cuda() for x in imgs]
    outs = lb.gaussian_batch(xs, sigmas, mode=mode, cval=0.5)
    for i, (x, s, o) in enumerate(zip(xs, sigmas, outs)):
        want = lb.gaussian_blur(x, s, mode=mode, cval=0.5)
        assert np.array_equal(host(o), host(want)), f"image {i} {tuple(x.shape)} sigma {s}"
    for i in (2, 5, 8):
        ref = oracle.gaussian_blur(imgs[i].astype(np.float32), [sigmas[i]], mode=mode, cval=0.5)
        oracle.assert_close(host(outs[i]), ref.astype(np.float64), RTOL, f"{mode} image {i} vs oracle")


def test_repeated_calls_and_graph_replay():
    rng = np.random.default_rng(5)
    xs = [torch.from_numpy(rng.integers(0, 4000, s).astype(np.uint16)).cuda() for s in SHAPES]
    sig = [1.0, 2.0] * 5
    outs = [torch.empty(x.shape, dtype=torch.float32, device="cuda") for x in xs]
    first = [host(o).copy() for o in lb.gaussian_batch(xs, sig[:len(xs)], outs=outs)]
    second = [host(o).copy() for o in lb.gaussian_batch(xs, sig[:len(xs)], outs=outs)]
    for a, b in zip(first, second):
        assert np.array_equal(a, b)
    for o in outs:
        o.zero_()
    g = lb.Graph()
    with g:
        lb.gaussian_batch(xs, sig[:len(xs)], outs=outs)
    g.launch()
    for a, o in zip(first, outs):
        assert np.array_equal(a, host(o))
    g.close()


def test_batch_argument_errors():
    x = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
    with pytest.raises(lb.LucemError):
        lb.gaussian_batch([torch.zeros((2, 8, 8), device="cuda")], 1.0)
    with pytest.raises(lb.LucemError):
        lb.gaussian_batch([x, torch.zeros((8, 8), dtype=torch.uint16, device="cuda")], 1.0)
    with pytest.raises(lb.LucemError):
        lb.gaussian_batch([x], 9.0)  # radius 36 > 32
    with pytest.raises(lb.LucemError):
        lb.gaussian_batch([x], -1.0)
    with pytest.raises(lb.LucemError):
        lb.gaussian_batch([x], [1.0, 2.0])
