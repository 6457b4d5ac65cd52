"""Writes tests/golden/scipy_filters.npz: scipy.ndimage outputs (FP64) for the
Gaussian family on deterministic inputs.  scipy implements the same published
filters as the reference (radius floor(truncate*sigma+0.5), half-sample
'reflect', derivative orders), so its outputs pin the oracle's restatement.

    python tests/golden/make_golden.py
"""
import os

import numpy as np
import scipy
import scipy.ndimage as ndi

HERE = os.path.dirname(os.path.abspath(__file__))


def sample_f64(n):
    # crates/lucem-ops/src/test_support.rs:10-12
    i = np.arange(n, dtype=np.int64)
    return ((i * 7919 + 104729) % 1013).astype(np.float64) * 0.1 - 50.0


def main():
    out = {"scipy_version": np.array(scipy.__version__)}
    x2 = sample_f64(37 * 41).reshape(37, 41)
    x3 = sample_f64(9 * 23 * 19).reshape(9, 23, 19)
    out["x2"], out["x3"] = x2, x3
    cases = []
    for mode in ("reflect", "constant", "nearest", "mirror", "wrap"):
        for sigma in (0.8, 2.0, 3.5):
            for order in ((0, 0), (1, 0), (0, 2), (3, 1)):
                key = f"g2_{mode}_{sigma}_{order[0]}{order[1]}"
                out[key] = ndi.gaussian_filter(x2, sigma, order=order, mode=mode, cval=1.5, truncate=4.0)
                cases.append(key)
    for mode in ("reflect", "constant"):
        key = f"g3_{mode}"
        out[key] = ndi.gaussian_filter(x3, (1.0, 2.0, 1.5), mode=mode, cval=1.5, truncate=4.0)
        cases.append(key)
    out["laplace_reflect_2.0"] = ndi.gaussian_laplace(x2, 2.0, mode="reflect", truncate=4.0)
    out["gradmag_reflect_1.5"] = ndi.gaussian_gradient_magnitude(x2, 1.5, mode="reflect", truncate=4.0)
    out["cases"] = np.array(cases)
    np.savez_compressed(os.path.join(HERE, "scipy_filters.npz"), **out)
    print("wrote", len(cases) + 2, "fixtures")


if __name__ == "__main__":
    main()
