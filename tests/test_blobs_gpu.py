"""Blob detectors (crates/lucem-ops/src/feature/blobs.rs) through the C ABI:
the reference's own test (a 25x25 Gaussian blob at (12, 12) found first by
LoG, DoG and DoH), and whole blob lists against the oracle's restatement
(f32 scale stack from the restated filters, the reference's maxima, sort
and pruning) on fields of separated blobs — scales on the fused path (radius
<= 32) and beyond it (per-axis passes).  Positions, scales and order must be
equal; responses agree to the filters' 1e-5 relative error (1e-4 here)."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu


def gaussian_field(shape, blobs, background=0.0):
    y, x = np.mgrid[0:shape[0], 0:shape[1]].astype(np.float64)
    img = np.full(shape, background)
    for cy, cx, s, a in blobs:
        img += a * np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2 * s * s))
    return img.astype(np.float32)


def test_reference_case():
    """feature/blobs.rs:350-392."""
    img = torch.from_numpy(gaussian_field((25, 25), [(12.0, 12.0, 2.5, 1.0)])).cuda()
    kw = dict(min_sigma=1.5, max_sigma=4.0, overlap=0.5, exclude_border=2)
    log = lb.blobs_log(img, num_sigma=6, threshold=0.05, **kw)
    dog = lb.blobs_dog(img, sigma_ratio=1.3, threshold=0.05, **kw)
    doh = lb.blobs_doh(img, num_sigma=6, threshold=0.01, **kw)
    for name, b in (("log", log), ("dog", dog), ("doh", doh)):
        assert b and (b[0].y, b[0].x) == (12, 12), (name, b[:2])


def _field(seed, shape, n, smin, smax):
    rng = np.random.default_rng(seed)
    blobs = []
    while len(blobs) < n:
        s = rng.uniform(smin, smax)
        cy, cx = rng.uniform(3 * s, shape[0] - 3 * s), rng.uniform(3 * s, shape[1] - 3 * s)
        if all((cy - b[0]) ** 2 + (cx - b[1]) ** 2 > (3 * (s + b[2])) ** 2 for b in blobs):
            blobs.append((cy, cx, s, rng.uniform(0.5, 1.5)))
    return gaussian_field(shape, blobs, background=0.05)


@pytest.mark.parametrize("kind,smin,smax,log_scale", [("log", 1.5, 6.0, False), ("dog", 1.5, 6.0, False),
                                                      ("doh", 1.5, 6.0, True), ("log", 2.0, 10.0, True),
                                                      ("dog", 2.0, 9.0, False)])
def test_blob_lists_equal_the_restatement(oracle, kind, smin, smax, log_scale):
    img = _field(len(kind) * 10 + int(smax), (150, 170), 10, smin, smax * 0.8)
    x = torch.from_numpy(img).cuda()
    thr = 0.002 if kind == "doh" else 0.02
    if kind == "dog":
        got = lb.blobs_dog(x, min_sigma=smin, max_sigma=smax, sigma_ratio=1.4, threshold=thr, overlap=0.5)
        sig = oracle.dog_sigmas(smin, smax, 1.4)
    else:
        fn = lb.blobs_log if kind == "log" else lb.blobs_doh
        got = fn(x, min_sigma=smin, max_sigma=smax, num_sigma=7, threshold=thr, overlap=0.5, log_scale=log_scale)
        sig = oracle.blob_sigmas(smin, smax, 7, log_scale)
    want = oracle.extract_blobs(oracle.blob_stack(img, kind, sig, 1.4), sig, thr, 0.5, 1)
    assert len(got) == len(want) > 0, (len(got), len(want))
    for g, w in zip(got, want):
        assert (g.y, g.x) == w[:2] and g.sigma == pytest.approx(w[2], rel=1e-12)
        assert g.response == pytest.approx(w[3], rel=1e-4, abs=1e-6)


def test_blob_errors_and_empty():
    x = torch.ones((16, 16), device="cuda")
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.blobs_log(x, min_sigma=0.0)
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.blobs_log(x, min_sigma=3.0, max_sigma=2.0)
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.blobs_dog(x, sigma_ratio=1.0)
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.blobs_doh(x, overlap=1.5)
    with pytest.raises(lb.LucemError, match="INVALID_DIMENSION"):
        lb.blobs_log(torch.ones((2, 8, 8), device="cuda"))
    assert lb.blobs_log(torch.empty((0, 8), device="cuda")) == []
    assert lb.blobs_log(torch.ones((2, 2), device="cuda")) == []  # inside the border


@pytest.mark.parametrize("kind", ["log", "doh"])
def test_crowded_field_pruning_equals_the_restatement(oracle, kind):
    """Blobs close enough to overlap, so the greedy pruning (done on the
    host over a grid of cells as wide as the overlap reach) drops many
    candidates: the kept list must equal the oracle's all-pairs pass."""
    rng = np.random.default_rng(41 if kind == "log" else 43)
    blobs = [(rng.uniform(8, 152), rng.uniform(8, 172), rng.uniform(1.5, 4.0), rng.uniform(0.5, 1.5))
             for _ in range(70)]
    img = gaussian_field((160, 180), blobs, background=0.02)
    x = torch.from_numpy(img).cuda()
    thr = 0.002 if kind == "doh" else 0.02
    fn = lb.blobs_log if kind == "log" else lb.blobs_doh
    got = fn(x, min_sigma=1.5, max_sigma=5.0, num_sigma=6, threshold=thr, overlap=0.3)
    sig = oracle.blob_sigmas(1.5, 5.0, 6, False)
    want = oracle.extract_blobs(oracle.blob_stack(img, kind, sig, 1.6), sig, thr, 0.3, 1)
    assert len(got) == len(want) > 20, (len(got), len(want))
    for g, w in zip(got, want):
        assert (g.y, g.x) == w[:2] and g.sigma == pytest.approx(w[2], rel=1e-12)
