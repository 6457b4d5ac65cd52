"""Gaussian-consumer operators (crates/lucem-ops/src/feature/structure.rs,
filter/ridge.rs) through the C ABI against the oracle's f32 restatement:
Hessian components, determinant, eigenvalues, shape index, structure tensor
and its eigenvalues, Frangi / Sato / Meijering.  Covers the fused path
(kernel radius <= 32) and the per-axis path (sigma 9 and 10), every pad mode,
u16 input, sigma 0, empty input and the argument errors.  Tolerance: the
reference's assert_close (crates/lucem-core/src/test_support.rs:42-50) at
1e-5 for the filters and 1e-4 for the nonlinear per-pixel functions of them
(eigenvalue square roots, ratios, exponentials); the shape index, an
angle, to 1e-3 in its own units."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu

MODES = ["reflect", "constant", "nearest", "mirror", "wrap"]


def dev(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.float64)


def blob_image(shape, seed, n=12):
    """Bright Gaussian blobs and lines on a dim background (smooth: the
    nonlinear functions are well conditioned away from isolated pixels)."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:shape[0], 0:shape[1]].astype(np.float64)
    img = np.full(shape, 10.0)
    for _ in range(n):
        cy, cx = rng.uniform(0, shape[0]), rng.uniform(0, shape[1])
        s = rng.uniform(1.5, 5.0)
        img += rng.uniform(50, 200) * np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2 * s * s))
    for _ in range(3):  # ridges
        a, b = rng.uniform(-1, 1), rng.uniform(0, shape[1])
        d = np.abs(x - (a * y + b)) / np.sqrt(1 + a * a)
        img += 80.0 * np.exp(-d ** 2 / (2 * 1.5 ** 2))
    return img.astype(np.float32)


@pytest.mark.parametrize("shape,sigma,mode", [((64, 64), 1.0, "reflect"), ((77, 130), 2.5, "constant"),
                                              ((40, 33), 2.0, "nearest"), ((130, 70), 4.0, "mirror"),
                                              ((50, 50), 1.5, "wrap"), ((96, 80), 9.0, "reflect"),
                                              ((20, 30), 0.0, "reflect")])
def test_hessian_family_against_the_restatement(oracle, shape, sigma, mode):
    img = blob_image(shape, seed=int(sigma * 10) + len(mode))
    x = dev(img)
    want = oracle.hessian_matrix(img, sigma, mode)
    for g, w in zip(lb.hessian_matrix(x, sigma, mode), want):
        oracle.assert_close(host(g), w.astype(np.float64), 1e-5, f"hessian {shape} {sigma} {mode}")
    oracle.assert_close(host(lb.hessian_det(x, sigma, mode)), (want[0] * want[2] - want[1] * want[1]).astype(np.float64),
                        1e-4, "det")
    we1, we2 = oracle.eigvals_2x2(*want)
    g1, g2 = lb.hessian_eigvals(x, sigma, mode)
    oracle.assert_close(host(g1), we1.astype(np.float64), 1e-4, "eig1")
    oracle.assert_close(host(g2), we2.astype(np.float64), 1e-4, "eig2")
    si = host(lb.shape_index(x, sigma, mode))
    wsi = oracle.shape_index_of(we1, we2).astype(np.float64)
    # The shape index is an angle of a ratio of eigenvalue sums and
    # differences: where l1 ~ l2 the ratio amplifies the eigenvalues' 1e-6
    # relative rounding (and can switch branch), so it is compared in its own
    # units ([-1, 1]) to 1e-3, all but a handful of pixels.
    bad = np.abs(si - wsi) > 1e-3
    assert bad.mean() < 2e-3, (bad.sum(), np.abs(si - wsi).max())


def test_hessian_u16_input(oracle):
    img = (blob_image((70, 90), seed=3) * 100).astype(np.uint16)
    got = lb.hessian_matrix(dev(img, np.uint16), 2.0)
    for g, w in zip(got, oracle.hessian_matrix(img.astype(np.float32), 2.0)):
        oracle.assert_close(host(g), w.astype(np.float64), 1e-5, "u16")


def test_shape_index_distinguishes_dome_and_cup():
    """feature/structure.rs:193-214."""
    y, x = np.mgrid[0:17, 0:17]
    r2 = ((y - 8.0) ** 2 + (x - 8.0) ** 2).astype(np.float32)
    assert abs(host(lb.shape_index(dev(-r2), 1.5, "nearest"))[8, 8] - 1.0) < 2e-2
    assert abs(host(lb.shape_index(dev(r2), 1.5, "nearest"))[8, 8] + 1.0) < 2e-2


@pytest.mark.parametrize("shape,sigma,mode", [((64, 64), 1.0, "reflect"), ((75, 121), 2.0, "constant"),
                                              ((33, 47), 3.0, "wrap"), ((90, 60), 10.0, "nearest"),
                                              ((20, 25), 0.0, "mirror")])
def test_structure_tensor_against_the_restatement(oracle, shape, sigma, mode):
    img = blob_image(shape, seed=7 + len(mode))
    got = lb.structure_tensor(dev(img), sigma, mode)
    want = oracle.structure_tensor(img, sigma, mode)
    for g, w in zip(got, want):
        oracle.assert_close(host(g), w.astype(np.float64), 1e-5, f"structure {shape} {sigma} {mode}")
    e1, e2 = lb.structure_tensor_eigvals(*got)
    w1, w2 = oracle.eigvals_2x2(*[host(g).astype(np.float32) for g in got])
    oracle.assert_close(host(e1), w1.astype(np.float64), 1e-5, "eig1")
    oracle.assert_close(host(e2), w2.astype(np.float64), 1e-5, "eig2")


@pytest.mark.parametrize("kind", ["frangi", "sato", "meijering"])
@pytest.mark.parametrize("black", [True, False])
def test_ridge_filters_against_the_restatement(oracle, kind, black):
    img = blob_image((96, 112), seed=11)
    fn = {"frangi": lb.frangi, "sato": lb.sato, "meijering": lb.meijering}[kind]
    # Default sigmas (1, 3, 5, 7, 9): the last scale takes the per-axis path.
    got = host(fn(dev(img), black_ridges=black))
    want = oracle.ridge_filter(img, kind, black_ridges=black).astype(np.float64)
    oracle.assert_close(got, want, 1e-4, f"{kind} black={black}")
    got = host(fn(dev(img), [0.5, 2.0], black_ridges=black, mode="constant"))
    want = oracle.ridge_filter(img, kind, [0.5, 2.0], black_ridges=black, mode="constant").astype(np.float64)
    oracle.assert_close(got, want, 1e-4, f"{kind} two scales")


def test_structure_family_errors():
    x = torch.ones((8, 8), device="cuda")
    with pytest.raises(lb.LucemError, match="INVALID_DIMENSION"):
        lb.hessian_matrix(torch.ones((2, 8, 8), device="cuda"), 1.0)
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.hessian_det(x, -1.0)
    with pytest.raises(lb.LucemError, match="UNKNOWN_PAD_MODE"):
        lb.structure_tensor(x, 1.0, mode="bogus")
    with pytest.raises(lb.LucemError, match="INVALID_PARAMETER"):
        lb.frangi(x, [])
    assert torch.count_nonzero(lb.sato(x, [])) == 0
    e = torch.empty((0, 5), device="cuda")
    assert lb.shape_index(e, 1.0).numel() == 0
    assert lb.frangi(e).numel() == 0
