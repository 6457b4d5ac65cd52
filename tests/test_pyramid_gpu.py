"""Pyramids (crates/lucem-ops/src/transform/pyramid.rs) through the C ABI
against the oracle's f32 restatement (the restated Gaussian, then resize's
order 0 / 1 resampling with the reference's f32 coordinates): reduce and
expand for downscale 2, 3 and 1.5, every pad mode, odd sizes, nearest and
bilinear; the Gaussian and Laplacian pyramids level by level; the
reference's own shape test.  Tolerance 1e-5 (the reference's assert_close)."""
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


def image(shape, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:shape[0], 0:shape[1]].astype(np.float64)
    return (np.sin(y / 3.0) * np.cos(x / 5.0) * 50 + rng.random(shape) * 10 + 100).astype(np.float32)


@pytest.mark.parametrize("shape,ds,order,mode", [((64, 64), 2.0, 1, "reflect"), ((77, 51), 2.0, 1, "constant"),
                                                 ((90, 65), 3.0, 1, "nearest"), ((40, 41), 1.5, 0, "mirror"),
                                                 ((33, 70), 2.0, 0, "wrap"), ((5, 3), 2.0, 1, "reflect")])
def test_reduce_and_expand_against_the_restatement(oracle, shape, ds, order, mode):
    img = image(shape, int(ds * 10) + order)
    got = lb.pyramid_reduce(dev(img), downscale=ds, order=order, mode=mode)
    want = oracle.pyramid_reduce(img, ds, None, order, mode)
    assert tuple(got.shape) == want.shape
    oracle.assert_close(host(got), want.astype(np.float64), 1e-5, f"reduce {shape} {ds} {order} {mode}")
    small = want.astype(np.float32)
    got = lb.pyramid_expand(dev(small), shape, downscale=ds, order=order, mode=mode)
    want = oracle.pyramid_expand(small, shape, ds, None, order, mode)
    oracle.assert_close(host(got), want.astype(np.float64), 1e-5, f"expand {shape} {ds} {order} {mode}")


def test_pyramids_level_by_level(oracle):
    img = image((100, 130), 3)
    g = lb.gaussian_pyramid(dev(img), 4)
    w = oracle.gaussian_pyramid(img, 4)
    assert [tuple(a.shape) for a in g] == [a.shape for a in w]
    for a, b in zip(g, w):
        oracle.assert_close(host(a), b.astype(np.float64), 1e-5, "gaussian level")
    lap = lb.laplacian_pyramid(dev(img), 3, sigma=1.2)
    wl = oracle.laplacian_pyramid(img, 3, sigma=1.2)
    assert len(lap) == len(wl)
    for a, b in zip(lap, wl):
        # Bands are differences of nearby values: compared against the level's scale.
        assert np.abs(host(a) - b).max() <= 1e-5 * np.abs(img).max()


def test_reference_shapes():
    """transform/pyramid.rs:271-292."""
    img = dev(np.arange(1, 17, dtype=np.float32).reshape(4, 4))
    assert [tuple(a.shape) for a in lb.gaussian_pyramid(img, 2)] == [(4, 4), (2, 2), (1, 1)]
    lap = lb.laplacian_pyramid(img, 2)
    assert len(lap) == 3 and tuple(lap[0].shape) == (4, 4)


def test_pyramid_errors():
    x = torch.ones((8, 8), device="cuda")
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.pyramid_reduce(x, downscale=1.0)
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.pyramid_reduce(x, order=3)
    with pytest.raises(lb.LucemError, match="INVALID_DIMENSION"):
        lb.pyramid_expand(torch.ones((2, 4, 4), device="cuda"))
