"""Seeded synthetic single-molecule stacks with the shapes and statistics of the benchmark workloads.

Camera model for every workload: ADU = offset 100 + gain 2 x Poisson(background + emitters), clipped to uint16.
Emitters are Gaussian PSFs integrated over each pixel (erf differences), or the astigmatic model
sigma_x(z) = 1.3 sqrt(1 + u^2 + 0.05 u^3), u = (z - 150)/400, sigma_y(z) = 1.3 sqrt(1 + v^2 - 0.05 v^3), v = (z + 150)/400.

Workloads (frames x height x width):
  "c1"  200 x 256 x 256,   40 emitters/frame, photons log-U[500, 5000], bg 20, sigma 1.3 px
  "c2"  2000 x 1024 x 1024, Poisson(2684) emitters/frame (0.1/um^2 at 160 nm), photons log-U[300, 8000],
        bg 10..80 cosine field, sigma U[1.0, 1.6]
  "c3"  1000 x 512 x 512,   800 emitters/frame, astigmatic z ~ U[-600, 600] nm, photons log-U[1000, 10000], bg 30
  "c4"  1500 x 512 x 512,   U{0..1500} emitters/frame, astigmatic, photons log-U[1000, 10000], bg 30
Frame counts can be reduced with ``frames=`` (parity tests use short stacks of the same shapes).
No public dataset is used; these are stand-ins with the same shapes, sizes and value distributions.
"""
import math

import numpy as np

OFFSET, GAIN = 100.0, 2.0
PIXEL_NM = 160.0

SHAPES = {"c1": (200, 256, 256), "c2": (2000, 1024, 1024), "c3": (1000, 512, 512), "c4": (1500, 512, 512)}


def astig_sigmas(z_nm):
    u = (z_nm - 150.0) / 400.0
    v = (z_nm + 150.0) / 400.0
    sx = 1.3 * np.sqrt(np.maximum(1 + u ** 2 + 0.05 * u ** 3, 1e-6))
    sy = 1.3 * np.sqrt(np.maximum(1 + v ** 2 - 0.05 * v ** 3, 1e-6))
    return sx, sy


def _erf(x):
    from scipy.special import erf
    return erf(x)


def emitters(workload, frames, height, width, seed):
    """Per-emitter table: columns frame, x, y, photons, sigma_x, sigma_y, z_nm (all float64)."""
    rng = np.random.default_rng(seed)
    if workload == "c1":
        counts = np.full(frames, 40)
    elif workload == "c2":
        lam = 0.1 * (width * PIXEL_NM / 1000.0) * (height * PIXEL_NM / 1000.0)
        counts = rng.poisson(lam, frames)
    elif workload == "c3":
        counts = np.full(frames, 800)
    elif workload == "c4":
        counts = rng.integers(0, 1501, frames)
    else:
        raise ValueError(workload)
    n = int(counts.sum())
    f = np.repeat(np.arange(frames), counts).astype(np.float64)
    x = rng.uniform(5.0, width - 5.0, n)
    y = rng.uniform(5.0, height - 5.0, n)
    if workload == "c1":
        ph = np.exp(rng.uniform(math.log(500), math.log(5000), n))
        sx = sy = np.full(n, 1.3)
        z = np.zeros(n)
    elif workload == "c2":
        ph = np.exp(rng.uniform(math.log(300), math.log(8000), n))
        sx = rng.uniform(1.0, 1.6, n)
        sy = sx.copy()
        z = np.zeros(n)
    else:
        ph = np.exp(rng.uniform(math.log(1000), math.log(10000), n))
        z = rng.uniform(-600.0, 600.0, n)
        sx, sy = astig_sigmas(z)
    return np.stack([f, x, y, ph, sx, sy, z], axis=1)


def background(workload, height, width):
    if workload == "c2":
        yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
        field = 0.5 * (np.cos(2 * np.pi * xx / width) * np.cos(2 * np.pi * yy / height) + 1.0)
        return 10.0 + 70.0 * field
    if workload == "c1":
        return np.full((height, width), 20.0)
    return np.full((height, width), 30.0)


def render_frame(em, height, width, bg, rng, patch=8):
    """Expected photons per pixel for one frame's emitters (erf-integrated Gaussian), plus Poisson + camera."""
    mu = bg.copy()
    for _, x, y, ph, sx, sy, _z in em:
        x0, y0 = int(x) - patch, int(y) - patch
        xs = np.arange(x0, x0 + 2 * patch + 1)
        ys = np.arange(y0, y0 + 2 * patch + 1)
        gx = 0.5 * (_erf((xs + 0.5 - x) / (math.sqrt(2) * sx)) - _erf((xs - 0.5 - x) / (math.sqrt(2) * sx)))
        gy = 0.5 * (_erf((ys + 0.5 - y) / (math.sqrt(2) * sy)) - _erf((ys - 0.5 - y) / (math.sqrt(2) * sy)))
        mx = (xs >= 0) & (xs < width)
        my = (ys >= 0) & (ys < height)
        mu[np.ix_(ys[my], xs[mx])] += ph * np.outer(gy[my], gx[mx])
    counts = rng.poisson(mu)
    return np.clip(OFFSET + GAIN * counts, 0, 65535).astype(np.uint16)


def stack(workload, frames=None, seed=1234, size=None):
    """(stack uint16 [Z, H, W], emitter table). ``size`` overrides (H, W) for reduced-size variants."""
    z, h, w = SHAPES[workload]
    if frames is not None:
        z = frames
    if size is not None:
        h, w = size
    em = emitters(workload, z, h, w, seed)
    bg = background(workload, h, w)
    rng = np.random.default_rng(seed + 1)
    out = np.empty((z, h, w), dtype=np.uint16)
    fidx = em[:, 0].astype(np.int64)
    for k in range(z):
        out[k] = render_frame(em[fidx == k], h, w, bg, rng)
    return out, em


def mad_threshold(w1_plane):
    """Detection threshold k = 3 x 1.4826 x MAD of wavelet plane 1 (the reference's PLANE_ID plane)."""
    med = np.median(w1_plane)
    return float(3.0 * 1.4826 * np.median(np.abs(w1_plane - med)))


def stack_cuda(workload, frames=None, seed=1234, size=None, device="cuda", chunk=64):
    """Same statistics as ``stack`` rendered with torch on the GPU (for the multi-GB benchmark stacks).

    Emitter tables come from the same numpy generator; pixel noise uses torch's CUDA Poisson sampler, so the pixels
    differ from ``stack`` for the same seed. Returns (int16 tensor [Z, H, W] holding the uint16 bit patterns, emitters).
    """
    import torch
    z, h, w = SHAPES[workload]
    if frames is not None:
        z = frames
    if size is not None:
        h, w = size
    em = emitters(workload, z, h, w, seed)
    bg = torch.as_tensor(background(workload, h, w), dtype=torch.float32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed + 1)
    out = torch.empty((z, h, w), dtype=torch.int16, device=device)
    patch = 8
    offs = torch.arange(-patch, patch + 1, device=device, dtype=torch.float64)
    fidx = em[:, 0].astype(np.int64)
    bounds = np.searchsorted(fidx, np.arange(0, z + chunk, chunk))
    s2 = math.sqrt(2.0)
    for c0 in range(0, z, chunk):
        c1 = min(z, c0 + chunk)
        e = torch.as_tensor(em[bounds[c0 // chunk]:bounds[c0 // chunk + 1]], device=device)
        mu = bg.unsqueeze(0).repeat(c1 - c0, 1, 1).reshape(-1)
        if e.shape[0]:
            f = e[:, 0].long() - c0
            x, y, ph, sx, sy = e[:, 1], e[:, 2], e[:, 3], e[:, 4], e[:, 5]
            xs = x.floor().unsqueeze(1) + offs  # pixel columns
            ys = y.floor().unsqueeze(1) + offs
            gx = 0.5 * (torch.erf((xs + 0.5 - x[:, None]) / (s2 * sx[:, None])) - torch.erf((xs - 0.5 - x[:, None]) / (s2 * sx[:, None])))
            gy = 0.5 * (torch.erf((ys + 0.5 - y[:, None]) / (s2 * sy[:, None])) - torch.erf((ys - 0.5 - y[:, None]) / (s2 * sy[:, None])))
            val = (ph[:, None, None] * gy[:, :, None] * gx[:, None, :]).float()
            xi = xs.long()[:, None, :].expand(-1, 2 * patch + 1, -1)
            yi = ys.long()[:, :, None].expand(-1, -1, 2 * patch + 1)
            ok = (xi >= 0) & (xi < w) & (yi >= 0) & (yi < h)
            flat = (f[:, None, None] * (h * w) + yi * w + xi)[ok]
            mu.index_add_(0, flat, val[ok])
        counts = torch.poisson(mu.reshape(c1 - c0, h, w), generator=gen)
        adu = torch.clamp(OFFSET + GAIN * counts, 0, 65535).to(torch.int32)
        out[c0:c1] = adu.to(torch.int16)
    return out, em
