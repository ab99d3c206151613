"""Seeded synthetic volumes for tests and benchmarks.

The reference ships no public dataset for this path, so the benchmark workloads
are rendered here.  The nearest reference analogues are
``utils/simulation.py:10-66`` (random smooth motion) and
``utils/preprocess.py:198-261`` (artificial motion on a template).

Volumes are (z, y, x) like the caller-facing API.  Displacements are returned
as (z, y, x, 3) with component 0 = dx, 1 = dy, 2 = dz, the layout
``wbi_registration_3d`` returns (``utils/registration.py:346``).

Template: constant background + isotropic Gaussian blobs (sigma ~ U[1.5, 3],
peak ~ lognormal(mu, s), centres uniform) + Poisson noise.
Field: per component, a sum of random 3-D sinusoids (wavelength ~ U[40, 120]
voxels, random direction and phase) rescaled to a given max |d|.
Moving volume: mov(p) = tmpl(p - d(p)) (trilinear, edge-replicated), so the
pull-warp registration of mov onto tmpl recovers m ~= d, then re-noised.
"""

from __future__ import annotations

import math

import numpy as np
import torch

__all__ = ["render_blobs", "sinusoid_field", "warp_pull", "make_pair", "ellipsoid_inclusion"]


def render_blobs(shape, n_blobs, rng, *, background=100.0, sigma=(1.5, 3.0), amp_mu=6.0,
                 amp_s=0.5, device="cpu", dtype=torch.float32):
    """Background plus ``n_blobs`` Gaussian blobs, (z, y, x), noise-free."""
    zdim, ydim, xdim = shape
    vol = torch.full((zdim * ydim * xdim,), float(background), dtype=dtype, device=device)
    centres = rng.uniform(0, 1, size=(n_blobs, 3)) * np.array([zdim, ydim, xdim])
    sig = rng.uniform(sigma[0], sigma[1], size=n_blobs)
    amp = rng.lognormal(amp_mu, amp_s, size=n_blobs)
    half = int(math.ceil(3 * sigma[1]))
    off = torch.arange(-half, half + 1, device=device)
    oz, oy, ox = torch.meshgrid(off, off, off, indexing="ij")
    oz, oy, ox = oz.reshape(-1), oy.reshape(-1), ox.reshape(-1)
    chunk = max(1, 2_000_000 // oz.numel())
    for s in range(0, n_blobs, chunk):
        c = torch.as_tensor(centres[s:s + chunk], dtype=torch.float64, device=device)
        sg = torch.as_tensor(sig[s:s + chunk], dtype=torch.float64, device=device)
        am = torch.as_tensor(amp[s:s + chunk], dtype=torch.float64, device=device)
        base = torch.floor(c).long()
        iz = base[:, 0:1] + oz
        iy = base[:, 1:2] + oy
        ix = base[:, 2:3] + ox
        d2 = ((iz - c[:, 0:1]) ** 2 + (iy - c[:, 1:2]) ** 2 + (ix - c[:, 2:3]) ** 2)
        val = am[:, None] * torch.exp(-d2 / (2 * sg[:, None] ** 2))
        ok = (iz >= 0) & (iz < zdim) & (iy >= 0) & (iy < ydim) & (ix >= 0) & (ix < xdim)
        lin = (iz * ydim + iy) * xdim + ix
        vol.index_add_(0, lin[ok], val[ok].to(dtype))
    return vol.reshape(zdim, ydim, xdim)


def sinusoid_field(shape, rng, max_disp=(4.0, 4.0, 1.5), n_waves=8, wavelength=(40.0, 120.0),
                   device="cpu"):
    """Smooth displacement (z, y, x, 3) = (dx, dy, dz), max |d_c| = max_disp[c]."""
    zdim, ydim, xdim = shape
    z = torch.arange(zdim, dtype=torch.float64, device=device)[:, None, None]
    y = torch.arange(ydim, dtype=torch.float64, device=device)[None, :, None]
    x = torch.arange(xdim, dtype=torch.float64, device=device)[None, None, :]
    comps = []
    for c in range(3):
        acc = torch.zeros(shape, dtype=torch.float64, device=device)
        for _ in range(n_waves):
            direction = rng.normal(size=3)
            direction /= np.linalg.norm(direction)
            k = 2 * math.pi / rng.uniform(*wavelength)
            phase = rng.uniform(0, 2 * math.pi)
            acc += torch.sin(k * (direction[0] * z + direction[1] * y + direction[2] * x) + phase)
        peak = acc.abs().max()
        comps.append((acc * (max_disp[c] / peak)).to(torch.float32))
    return torch.stack(comps, dim=-1)


def warp_pull(vol, field):
    """out(p) = vol(p + field(p)), trilinear with edge replication, float32.

    ``vol`` (z, y, x); ``field`` (z, y, x, 3) = (dx, dy, dz).
    """
    zdim, ydim, xdim = vol.shape
    dev = vol.device
    v = vol.to(torch.float32).reshape(-1)
    z = torch.arange(zdim, device=dev, dtype=torch.float32)[:, None, None] + field[..., 2]
    y = torch.arange(ydim, device=dev, dtype=torch.float32)[None, :, None] + field[..., 1]
    x = torch.arange(xdim, device=dev, dtype=torch.float32)[None, None, :] + field[..., 0]
    out = torch.zeros_like(z)
    fz, fy, fx = torch.floor(z), torch.floor(y), torch.floor(x)
    tz, ty, tx = z - fz, y - fy, x - fx
    fz, fy, fx = fz.long(), fy.long(), fx.long()
    for a in (0, 1):
        iz = (fz + a).clamp(0, zdim - 1)
        wz = tz if a else 1 - tz
        for b in (0, 1):
            iy = (fy + b).clamp(0, ydim - 1)
            wy = ty if b else 1 - ty
            for c in (0, 1):
                ix = (fx + c).clamp(0, xdim - 1)
                wx = tx if c else 1 - tx
                out += wz * wy * wx * v[(iz * ydim + iy) * xdim + ix]
    return out


def ellipsoid_inclusion(shape, coverage, rng=None, device="cpu"):
    """Boolean (z, y, x) ellipsoid centred in the volume covering ``coverage``
    of the voxels (semi-axes proportional to the volume's half-extents)."""
    zdim, ydim, xdim = shape
    z = (torch.arange(zdim, device=device, dtype=torch.float64) + 0.5 - zdim / 2) / (zdim / 2)
    y = (torch.arange(ydim, device=device, dtype=torch.float64) + 0.5 - ydim / 2) / (ydim / 2)
    x = (torch.arange(xdim, device=device, dtype=torch.float64) + 0.5 - xdim / 2) / (xdim / 2)
    r2 = z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2
    # an ellipsoid touching the box covers pi/6 of it; larger coverage is
    # reached by growing the normalised radius (clipped by the box).
    lo, hi = 0.0, math.sqrt(3.0)
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        frac = float((r2 <= mid * mid).double().mean())
        if frac < coverage:
            lo = mid
        else:
            hi = mid
    return r2 <= hi * hi


def make_pair(shape, seed, *, n_blobs=2000, max_disp=(4.0, 4.0, 1.5), drift=0.0, device="cpu",
              template=None, noise=True):
    """(template, moving, field): uint16 volumes (z, y, x) and the float32 field.

    The moving volume is ``template`` pulled through ``field``, scaled by
    ``1 + drift`` and Poisson re-noised.  A given ``template`` (float) is reused
    (time series); otherwise one is rendered from ``seed``.
    """
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed) * 7919 + 17)
    if template is None:
        clean = render_blobs(shape, n_blobs, rng, device=device)
        tmpl = torch.poisson(clean, generator=gen) if noise else clean
    else:
        tmpl = template.to(device=device, dtype=torch.float32)
    field = sinusoid_field(shape, rng, max_disp=max_disp, device=device)
    mov = warp_pull(tmpl, -field) * (1.0 + drift)
    if noise:
        mov = torch.poisson(mov.clamp_min(0), generator=gen)
    return _to_u16(tmpl), _to_u16(mov), field


def _to_u16(t):
    return t.clamp(0, 65535).round().to(torch.int32).to(torch.uint16)
