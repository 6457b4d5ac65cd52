"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark workloads (there is no dataset: every input is generated).

PRNG: numpy's PCG64 (`np.random.default_rng(seed)`), and for the large slide a
torch CUDA generator seeded the same way.  Seeds are `SEED_BASE + workload`.

- blob_image: background + isotropic Gaussian blobs (centres uniform, radius
  r ~ U[3, 8] used as the blob sigma, amplitude ~ U[500, 4000]) + Poisson
  noise, clipped to u16.
- bead_volume / bead_image: point beads (intensity ~ U[1e3, 1e4]) at uniform
  integer positions, blurred by a normalised Gaussian PSF (zero-padded linear
  convolution), + background 10, + Poisson noise, f32.
- blob_slide: a [C, H, W] u16 slide of blob fields with per-channel densities,
  generated on the GPU.
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 0x6C7563656D  # "lucem"


def gaussian_psf(shape, sigmas) -> np.ndarray:
    """Normalised (sum 1) Gaussian PSF of odd `shape`, centred, per-axis sigma."""
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) - (n // 2) for n in shape], indexing="ij")
    q = sum((g / s) ** 2 for g, s in zip(grids, sigmas))
    p = np.exp(-0.5 * q)
    return (p / p.sum()).astype(np.float64)


def blob_image(height=2048, width=2048, n_blobs=4000, background=200.0, seed=SEED_BASE + 0) -> np.ndarray:
    """u16 [height, width] blob field with Poisson noise."""
    rng = np.random.default_rng(seed)
    img = np.full((height, width), background, np.float64)
    cy = rng.uniform(0, height, n_blobs)
    cx = rng.uniform(0, width, n_blobs)
    r = rng.uniform(3.0, 8.0, n_blobs)
    a = rng.uniform(500.0, 4000.0, n_blobs)
    for i in range(n_blobs):
        h = int(np.ceil(4 * r[i]))
        y0, y1 = max(0, int(cy[i]) - h), min(height, int(cy[i]) + h + 1)
        x0, x1 = max(0, int(cx[i]) - h), min(width, int(cx[i]) + h + 1)
        if y0 >= y1 or x0 >= x1:
            continue
        yy = np.arange(y0, y1)[:, None] - cy[i]
        xx = np.arange(x0, x1)[None, :] - cx[i]
        img[y0:y1, x0:x1] += a[i] * np.exp(-(yy * yy + xx * xx) / (2 * r[i] * r[i]))
    noisy = rng.poisson(img)
    return np.clip(noisy, 0, 65535).astype(np.uint16)


def _stamp(vol: np.ndarray, psf: np.ndarray, pos, amp):
    """vol += amp * psf centred at pos (zero outside the volume)."""
    c = [n // 2 for n in psf.shape]
    src, dst = [], []
    for d in range(vol.ndim):
        lo = pos[d] - c[d]
        a0, a1 = max(0, lo), min(vol.shape[d], lo + psf.shape[d])
        if a0 >= a1:
            return
        dst.append(slice(a0, a1))
        src.append(slice(a0 - lo, a1 - lo))
    vol[tuple(dst)] += amp * psf[tuple(src)]


def bead_volume(shape=(64, 512, 512), n_beads=3000, psf_shape=(31, 15, 15), psf_sigmas=(3.0, 1.5, 1.5),
                background=10.0, seed=SEED_BASE + 1):
    """(observation f32, psf f32): beads blurred by the PSF + background + Poisson."""
    rng = np.random.default_rng(seed)
    psf = gaussian_psf(psf_shape, psf_sigmas)
    vol = np.zeros(shape, np.float64)
    pos = np.stack([rng.integers(0, n, n_beads) for n in shape], axis=1)
    amp = rng.uniform(1e3, 1e4, n_beads)
    for p, a in zip(pos, amp):
        _stamp(vol, psf, p, a)
    vol += background
    obs = rng.poisson(vol).astype(np.float32)
    return obs, psf.astype(np.float32)


def bead_image(height, width, sigma, density=3000 / (64 * 512 * 512), background=10.0, seed=0):
    """(observation f32 [h, w], psf f32 [k, k]) with k = 2*ceil(3 sigma) + 1."""
    rng = np.random.default_rng(seed)
    k = 2 * int(np.ceil(3 * sigma)) + 1
    psf = gaussian_psf((k, k), (sigma, sigma))
    img = np.zeros((height, width), np.float64)
    n = max(1, int(round(density * height * width)))
    pos = np.stack([rng.integers(0, height, n), rng.integers(0, width, n)], axis=1)
    amp = rng.uniform(1e3, 1e4, n)
    for p, a in zip(pos, amp):
        _stamp(img, psf, p, a)
    img += background
    return rng.poisson(img).astype(np.float32), psf.astype(np.float32)


def uneven_bead_batch(n_images=256, lo=256, hi=2048, seed=SEED_BASE + 3):
    """Sizes and PSF sigmas of the uneven 2-D batch: sides ~ U[lo, hi] (integers,
    independent), sigma ~ U[1, 3]."""
    rng = np.random.default_rng(seed)
    hs = rng.integers(lo, hi + 1, n_images)
    ws = rng.integers(lo, hi + 1, n_images)
    sig = rng.uniform(1.0, 3.0, n_images)
    return [(int(h), int(w), float(s), int(seed * 1000 + i)) for i, (h, w, s) in enumerate(zip(hs, ws, sig))]


def blob_slide(channels=5, height=34560, width=24960, densities=(1e-4, 2.5e-4, 5e-4, 7.5e-4, 1e-3),
               background=200.0, seed=SEED_BASE + 2, device="cuda", chunk=40000):
    """u16 [channels, height, width] blob fields generated on the GPU (torch):
    blob stamps are scatter-added in chunks, then Poisson noise is drawn."""
    import torch

    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    out = torch.empty((channels, height, width), dtype=torch.uint16, device=device)
    win = torch.arange(-32, 33, device=device, dtype=torch.float32)  # 4 * r_max = 32
    for c in range(channels):
        img = torch.full((height * width,), background, dtype=torch.float32, device=device)
        n = int(round(densities[c % len(densities)] * height * width))
        for s in range(0, n, chunk):
            m = min(chunk, n - s)
            cy = torch.rand(m, generator=gen, device=device) * height
            cx = torch.rand(m, generator=gen, device=device) * width
            r = 3.0 + 5.0 * torch.rand(m, generator=gen, device=device)
            a = 500.0 + 3500.0 * torch.rand(m, generator=gen, device=device)
            yy = torch.floor(cy)[:, None] + win[None, :]          # [m, 65]
            xx = torch.floor(cx)[:, None] + win[None, :]
            dy = (yy - cy[:, None]) ** 2
            dx = (xx - cx[:, None]) ** 2
            inv = 1.0 / (2.0 * r * r)
            vy = torch.exp(-dy * inv[:, None])
            vx = torch.exp(-dx * inv[:, None])
            val = a[:, None, None] * vy[:, :, None] * vx[:, None, :]  # [m, 65, 65]
            ok = ((yy >= 0) & (yy < height))[:, :, None] & ((xx >= 0) & (xx < width))[:, None, :]
            idx = (yy.clamp(0, height - 1).long()[:, :, None] * width + xx.clamp(0, width - 1).long()[:, None, :])
            img.index_add_(0, idx[ok], val[ok])
            del val, ok, idx
        noisy = torch.poisson(img, generator=gen).clamp_(0, 65535)
        out[c] = noisy.to(torch.int32).view(height, width).to(torch.uint16)
        del img, noisy
    return out


def bead_batch(specs, device="cuda", density=3000 / (64 * 512 * 512), background=10.0):
    """The uneven 2-D batch on the GPU: for each (h, w, sigma, seed) of
    uneven_bead_batch, beads (intensity ~ U[1e3, 1e4], density per pixel as
    the bead volume) at uniform integer positions, blurred by the normalised
    Gaussian PSF of support 2*ceil(3 sigma) + 1 (zero padding; the library's
    own separable blur, whose taps are that PSF's separable factors),
    + background, + Poisson noise.  Returns (images f32, psfs f32) lists."""
    import torch

    from . import ops

    images, psfs = [], []
    for h, w, sigma, seed in specs:
        gen = torch.Generator(device=device)
        gen.manual_seed(int(seed))
        n = max(1, int(round(density * h * w)))
        img = torch.zeros(h * w, dtype=torch.float32, device=device)
        pos = torch.randint(0, h * w, (n,), generator=gen, device=device)
        amp = 1e3 + 9e3 * torch.rand(n, generator=gen, device=device)
        img.index_add_(0, pos, amp)
        r = int(np.ceil(3 * sigma))
        blurred = ops.gaussian_blur(img.view(h, w), sigma, mode="constant", radii=r)
        obs = torch.poisson(blurred + background, generator=gen).to(torch.float32)
        k = 2 * r + 1
        images.append(obs.contiguous())
        psfs.append(torch.from_numpy(gaussian_psf((k, k), (sigma, sigma)).astype(np.float32)).to(device))
    return images, psfs
