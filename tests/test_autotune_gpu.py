"""Launch-settings autotuning of the Gaussian family kernels (the reference
tunes CubeCL launch candidates once per device and size class,
crates/lucem-core/src/compute/tune.rs:1-27): with tuning on, the first call
of each key times its candidates and caches the fastest; results are equal
bit for bit to the untuned launches (every candidate computes the same
thing); later calls reuse the plan; plans survive save / load."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_tuned_launches_equal_the_untuned_and_are_cached(tmp_path):
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.integers(0, 4000, (3, 900, 1536)).astype(np.int32)).cuda().to(torch.uint16)
    img = torch.from_numpy(rng.random((1536, 2048)).astype(np.float32)).cuda()
    resp = [("gaussian", 1.0), ("gaussian", 2.0), ("gaussian", 4.0), ("dog", 1.0, 3.0)]
    blocks = lb.schedule((1, 900, 1536), (1, 256, 256), (0, 32, 32))
    # Untuned first (no plans cached for these keys yet).
    lb.autotune_enable(False)
    before = set(lb.autotune_plans())
    walk0 = [host(o) for o in lb.gaussian_family_tiles(x, blocks, resp)]
    fam0 = [host(o) for o in lb.gaussian_family(img, resp)]
    blur0 = host(lb.gaussian_blur(img, 2.0))
    assert set(lb.autotune_plans()) == before
    lb.autotune_enable(True)
    try:
        walk1 = [host(o) for o in lb.gaussian_family_tiles(x, blocks, resp)]
        fam1 = [host(o) for o in lb.gaussian_family(img, resp)]
        blur1 = host(lb.gaussian_blur(img, 2.0))
        plans = lb.autotune_plans()
        new = {k: v for k, v in plans.items() if k not in before}
        kinds = {k.split("-")[0] for k in new}
        assert {"walk", "blur"} <= kinds, new
        assert all(1 <= v <= 4 for v in new.values())
        for a, b in zip(walk0 + fam0 + [blur0], walk1 + fam1 + [blur1]):
            assert np.array_equal(a, b)
        # A second call of the same keys reuses the plans (no new keys).
        walk2 = [host(o) for o in lb.gaussian_family_tiles(x, blocks, resp)]
        assert lb.autotune_plans() == plans
        for a, b in zip(walk0, walk2):
            assert np.array_equal(a, b)
    finally:
        lb.autotune_enable(False)
    path = tmp_path / "tune.txt"
    lb.autotune_save(str(path))
    text = path.read_text()
    assert all(f"plan {k} {v}" in text for k, v in new.items())
    lb.autotune_load(str(path))
    assert lb.autotune_plans() == plans
    bad = tmp_path / "bad.txt"
    bad.write_text("plan walk-x 9\n")
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.autotune_load(str(bad))


def test_tuned_image_batch_equals_the_untuned():
    """The batch's candidates include the window copies ahead (off by
    default): every candidate runs once while tuning, and the result equals
    the untuned launch bit for bit."""
    rng = np.random.default_rng(17)
    imgs = [torch.from_numpy(rng.integers(0, 4000, (int(h), int(w))).astype(np.int32)).cuda().to(torch.uint16)
            for h, w in rng.integers(64, 700, (40, 2))]
    sig = list(rng.choice([1.0, 2.0, 4.0], len(imgs)))
    want = [host(o) for o in lb.gaussian_batch(imgs, sig)]
    lb.autotune_enable(True)
    try:
        got = [host(o) for o in lb.gaussian_batch(imgs, sig)]
    finally:
        lb.autotune_enable(False)
    assert any(k.startswith("batch") for k in lb.autotune_plans())
    for a, b in zip(want, got):
        assert np.array_equal(a, b)


def test_tuning_is_skipped_during_capture():
    img = torch.from_numpy(np.random.default_rng(9).random((333, 517)).astype(np.float32)).cuda()
    want = host(lb.gaussian_blur(img, 3.0))
    lb.autotune_enable(True)
    try:
        out = torch.empty_like(img)
        g = lb.Graph()
        with g:
            lb.gaussian_blur(img, 3.0, out=out)
        g.launch()
        assert np.array_equal(host(out), want)
    finally:
        lb.autotune_enable(False)
