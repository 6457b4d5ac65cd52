"""FP64 Richardson-Lucy through cuFFT (torch.fft in float64 on the device):
the cross-check for results too large for the host FP64 oracle to run in
test time (the 64 x 512 x 512 volume over 50 iterations, the 256-image batch).

TEST INFRASTRUCTURE.  It is the same arithmetic as the host oracle's
richardson_lucy_fft64 (oracle/oracle.py), which follows the reference's
Constant-mode iteration (crates/lucem-ops/src/restore/deconvolve.rs:109-147,
guard at restore/kernels/deconvolve.rs:18-20), and
tests/test_rl_fullsize_gpu.py pins the two against each other (to 1e-10) on
the full 128 x 1024 x 1024 grid before trusting it.  cuFFT is used here only
as that cross-check; the library's transforms are its own.
"""
from __future__ import annotations

import numpy as np
import torch


def centred_otf(p: torch.Tensor, grid, centre) -> torch.Tensor:
    """Real FFT over `grid` of the PSF with tap `centre` moved to the origin
    (restore/kernels/deconvolve.rs:79-99)."""
    nd = p.dim()
    buf = torch.zeros(tuple(grid), dtype=torch.float64, device=p.device)
    buf[tuple(slice(0, n) for n in p.shape)] = p
    buf = torch.roll(buf, shifts=tuple(-int(c) for c in centre), dims=tuple(range(nd)))
    return torch.fft.rfftn(buf, dim=tuple(range(nd)))


def richardson_lucy(obs, psf, num_iter, filter_epsilon=1e-6, grid=None, device="cuda"):
    """Zero padding, clip off; obs / psf are numpy or torch arrays.  Returns a
    float64 tensor on `device`."""
    y = torch.as_tensor(np.asarray(obs) if not torch.is_tensor(obs) else obs).to(device, torch.float64)
    k = torch.as_tensor(np.asarray(psf) if not torch.is_tensor(psf) else psf).to(device, torch.float64)
    nd = y.dim()
    if grid is None:
        grid = tuple(y.shape[d] + k.shape[d] - 1 for d in range(nd))
    s = float(k.sum())
    p = k * (1.0 / s if abs(s) > 1e-12 else 1.0)
    ks = k.shape
    h_conv = centred_otf(p, grid, [ks[d] - 1 - ks[d] // 2 for d in range(nd)])
    h_corr = torch.conj(centred_otf(p, grid, [ks[d] // 2 for d in range(nd)]))
    eps = max(float(filter_epsilon), 1e-15)
    ax = tuple(range(nd))
    sl = tuple(slice(0, n) for n in y.shape)
    est = torch.full(y.shape, 0.5, dtype=torch.float64, device=device)
    for _ in range(num_iter):
        conv = torch.fft.irfftn(torch.fft.rfftn(est, s=grid, dim=ax) * h_conv, s=grid, dim=ax)[sl]
        conv = torch.where(conv.abs() < eps, torch.full_like(conv, eps), conv)
        ratio = y / conv
        del conv
        corr = torch.fft.irfftn(torch.fft.rfftn(ratio, s=grid, dim=ax) * h_corr, s=grid, dim=ax)[sl]
        est = est * corr
        del corr, ratio
    return est


def max_rel_err(got, want) -> float:
    """The smallest rtol for which the reference's assert_close passes
    (crates/lucem-core/src/test_support.rs:42-50): max |g - w| / (|w| + max|w|)."""
    g = torch.as_tensor(got).to(want.device, torch.float64).reshape(-1)
    w = want.reshape(-1)
    if w.numel() == 0:
        return 0.0
    den = w.abs() + w.abs().max()
    den = torch.where(den == 0, torch.ones_like(den), den)
    return float(((g - w).abs() / den).max())
