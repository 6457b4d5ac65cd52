"""Canny (crates/lucem-ops/src/feature/canny.rs) through the C ABI against
the oracle's restatement (f32 smoothing, two-pass Sobel stencils, the
reference's magnitude, sector and suppression, and its breadth-first
hysteresis).

With sigma 0 and integer images every step is exact in f32 on both sides
(the stencils sum small integers, the square root is correctly rounded), so
those edge maps must be identical: every pad mode, every threshold form,
ragged and tiny shapes, u8 / u16 inputs, and label-merging stress patterns
(a long spiral, a comb, a noise field).  With sigma > 0 the device
composes the stencils with the Gaussian (reflect, mirror, wrap) or smooths
first (constant, nearest, wide kernels); rounding differs from the
reference's passes at the 1e-7 level and can break near-ties of the
suppression, so there the edge maps may differ in a handful of pixels
(bounded below).  Plus the reference's own square test and its errors."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu


def dev(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def integer_image(shape, seed, levels=4, block=8):
    rng = np.random.default_rng(seed)
    H, W = shape
    coarse = rng.integers(0, levels, (H // block + 1, W // block + 1))
    img = coarse.repeat(block, 0).repeat(block, 1)[:H, :W] * 40 + rng.integers(0, 12, shape)
    return img.astype(np.float32)


def smooth_image(shape, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:shape[0], 0:shape[1]].astype(np.float64)
    img = rng.random(shape) * 0.2
    for _ in range(12):
        cy, cx = rng.uniform(0, shape[0]), rng.uniform(0, shape[1])
        s = rng.uniform(2, 12)
        img += rng.uniform(0.5, 2.0) * (((y - cy) ** 2 + (x - cx) ** 2) < s * s)
    return img.astype(np.float32)


def test_reference_square():
    """feature/canny.rs:172-189."""
    data = np.zeros((20, 20), np.float32)
    data[5:15, 5:15] = 1.0
    edges = host(lb.canny(dev(data), sigma=1.0))
    assert edges.dtype == np.uint32
    assert 28 <= int(edges.sum()) <= 60
    assert edges[10, 10] == 0 and edges[0, 0] == 0


@pytest.mark.parametrize("shape", [(64, 64), (77, 131), (300, 257), (5, 3), (3, 200), (1, 50), (2, 2)])
@pytest.mark.parametrize("mode", ["reflect", "constant", "nearest", "mirror", "wrap"])
def test_integer_images_equal_the_restatement(oracle, shape, mode):
    img = integer_image(shape, shape[0] * 7 + shape[1])
    got = host(lb.canny(dev(img), sigma=0.0, mode=mode, cval=13.0))
    want = oracle.canny(img, 0.0, mode=mode, cval=13.0)
    assert np.array_equal(got, want), (int(got.sum()), int(want.sum()))


@pytest.mark.parametrize("kw", [dict(low_threshold=40.0, high_threshold=120.0), dict(low_threshold=0.05),
                                dict(high_threshold=300.0), dict(low_threshold=0.1, high_threshold=0.4,
                                                                 use_quantiles=True),
                                dict(low_threshold=0.0, high_threshold=150.0), dict(use_quantiles=True),
                                dict(low_threshold=60.0, high_threshold=60.0)])
def test_threshold_forms(oracle, kw):
    img = integer_image((150, 190), 5)
    got = host(lb.canny(dev(img), sigma=0.0, **kw))
    want = oracle.canny(img, 0.0, **kw)
    assert np.array_equal(got, want), (kw, int(got.sum()), int(want.sum()))


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_integer_inputs(oracle, dtype):
    img = integer_image((120, 97), 11)
    got = host(lb.canny(dev(img, dtype), sigma=0.0))
    assert np.array_equal(got, oracle.canny(img, 0.0))


def spiral(n):
    img = np.zeros((n, n), np.float32)
    y, x, dy, dx = n // 2, n // 2, 0, 1
    steps = 1
    while 0 <= y < n and 0 <= x < n:
        for _ in range(2):
            for _ in range(steps):
                if 0 <= y < n and 0 <= x < n:
                    img[y, x] = 10.0
                y += dy * 3
                x += dx * 3
                if 0 <= y - dy < n and 0 <= x - dx < n:
                    img[y - dy, x - dx] = 10.0
                    img[y - 2 * dy, x - 2 * dx] = 10.0
            dy, dx = dx, -dy
        steps += 1
    img[n // 2, n // 2] = 200.0
    return img


def comb(H, W):
    img = np.zeros((H, W), np.float32)
    img[:, ::4] = 10.0
    img[H - 3, :] = 10.0
    img[H - 3, W // 2] = 200.0
    return img


@pytest.mark.parametrize("name", ["spiral", "comb", "noise"])
def test_label_merging_patterns(oracle, name):
    if name == "spiral":
        img = spiral(255)
    elif name == "comb":
        img = comb(257, 300)
    else:
        img = np.random.default_rng(3).integers(0, 50, (400, 333)).astype(np.float32)
    # spiral and comb: one long component over the whole mask; noise: many
    # components, about a third of the mask kept.
    kw = dict(low_threshold=60.0, high_threshold=150.0) if name == "noise" else dict(low_threshold=1.0,
                                                                                      high_threshold=300.0)
    got = host(lb.canny(dev(img), sigma=0.0, **kw))
    want = oracle.canny(img, 0.0, **kw)
    assert want.sum() > 10000
    assert np.array_equal(got, want), (int(got.sum()), int(want.sum()))


@pytest.mark.parametrize("sigma,mode", [(1.0, "reflect"), (2.5, "mirror"), (1.5, "wrap"), (7.0, "reflect"),
                                        (2.0, "constant"), (1.0, "nearest"), (8.5, "reflect")])
def test_smoothed_images_close_to_the_restatement(oracle, sigma, mode):
    img = smooth_image((210, 230), int(sigma * 10))
    got = host(lb.canny(dev(img), sigma=sigma, mode=mode))
    want = oracle.canny(img, sigma, mode=mode)
    diff = int((got != want).sum())
    assert want.sum() > 50
    assert diff <= max(4, int(0.01 * want.sum())), (diff, int(want.sum()))


def test_large_integer_image(oracle):
    img = integer_image((2048, 1536), 21, levels=6, block=32)
    got = host(lb.canny(dev(img), sigma=0.0))
    assert np.array_equal(got, oracle.canny(img, 0.0))


def test_output_buffer_and_dlpack():
    img = dev(integer_image((64, 80), 2))
    out = torch.empty((64, 80), dtype=torch.uint32, device="cuda")
    r = lb.canny(img, sigma=0.0, out=out)
    assert r is out and set(np.unique(host(out)).tolist()) <= {0, 1}


def test_canny_errors_and_empty():
    x = torch.ones((16, 16), device="cuda")
    with pytest.raises(lb.LucemError, match="INVALID_DIMENSION"):
        lb.canny(torch.ones((2, 8, 8), device="cuda"))
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.canny(x, sigma=-1.0)
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.canny(x, low_threshold=2.0, high_threshold=1.0)
    with pytest.raises(lb.LucemError, match="UNSUPPORTED_DTYPE"):
        lb.canny(x, out=torch.empty((16, 16), device="cuda"))
    with pytest.raises(lb.LucemError, match="SHAPE_MISMATCH"):
        lb.canny(x, out=torch.empty((16, 15), dtype=torch.uint32, device="cuda"))
    with pytest.raises(lb.LucemError, match="UNSUPPORTED_DTYPE"):
        lb.gaussian_blur(torch.ones((8, 8), dtype=torch.uint32, device="cuda"), 1.0)
    e = lb.canny(torch.empty((0, 8), device="cuda"))
    assert e.shape == (0, 8) and e.dtype == torch.uint32
    assert int(host(lb.canny(torch.zeros((32, 32), device="cuda"))).sum()) == 0


def test_default_thresholds_run_in_a_cuda_graph(oracle):
    """With both thresholds left to their defaults they are computed on the
    device: the call captures into a CUDA graph, and a replay on new data in
    the same buffers equals the restatement."""
    a = integer_image((160, 200), 31)
    b = integer_image((160, 200), 32)
    x = dev(a)
    out = torch.empty((160, 200), dtype=torch.uint32, device="cuda")
    lb.canny(x, sigma=0.0, out=out)  # sizes the workspace before capture
    g = lb.Graph()
    with g:
        lb.canny(x, sigma=0.0, out=out)
    x.copy_(dev(b))
    g.launch()
    assert np.array_equal(host(out), oracle.canny(b, 0.0))
    for q in (True, False):
        assert np.array_equal(host(lb.canny(dev(a), sigma=0.0, use_quantiles=q)),
                              oracle.canny(a, 0.0, use_quantiles=q))
