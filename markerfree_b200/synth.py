"""Seeded synthetic tilt series with known ground truth.

The reference's own evaluation uses simulated phantoms that are not shipped with
it, so benchmarks and tests run on series generated here: a volume of Gaussian
blobs (optionally over a smooth low-frequency background) projected as line
integrals about a tilt axis, then shifted per tilt and corrupted with noise.

Geometry follows the reference's conventions (Markerfree/src/method/CorrStack.cu:142-179
and CalcReproj.cu:17-64): in the aligned frame a volume point (x, y, z) (centred
pixel coordinates) projects at tilt angle t to detector coordinate
(x cos t + z sin t, y); the raw image is that projection rotated by the tilt-axis
angle `axis` (degrees, measured as in the reference's ``rotate`` parameter) and
translated by the per-tilt shift, so that the reference's resampler
``corrected(p) = raw(R(axis) p + shift + centre)`` undoes it exactly when given
the true parameters.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Series:
    stack: np.ndarray          # (nz, ny, nx) float32, angle-sorted
    angles: np.ndarray         # (nz,) float32 degrees, ascending
    shifts: np.ndarray         # (nz, 2) float32 true shifts (raw px)
    axis: float                # true tilt-axis angle (deg)
    thickness: int             # AlignZ to run with
    nproj: int                 # -p
    name: str


def _render(nx, ny, centres, sigmas, amps, out):
    """Add isotropic 2-D Gaussians (integrated line integrals) into out (ny, nx)."""
    for (cx, cy), s, a in zip(centres, sigmas, amps):
        r = int(math.ceil(4.0 * s))
        x0, x1 = max(0, int(cx) - r), min(nx, int(cx) + r + 2)
        y0, y1 = max(0, int(cy) - r), min(ny, int(cy) + r + 2)
        if x0 >= x1 or y0 >= y1:
            continue
        xs = np.arange(x0, x1, dtype=np.float64) - cx
        ys = np.arange(y0, y1, dtype=np.float64) - cy
        gx = np.exp(-xs * xs / (2 * s * s))
        gy = np.exp(-ys * ys / (2 * s * s))
        out[y0:y1, x0:x1] += (a * s * math.sqrt(2 * math.pi)) * np.outer(gy, gx)


def make_series(nx=512, ny=512, vol_z=128, n_blobs=200, sigma=(2.0, 6.0), amp=(0.5, 1.5),
                tilt_min=-60.0, tilt_max=60.0, tilt_step=3.0, axis=86.3, shift_sd=4.0,
                drift=0.0, snr=0.1, poisson=False, background=False, seed=1001,
                thickness=100, nproj=10, name="synthetic", n_tilts=None):
    """Generate one series.  Defaults are the small plain-method configuration."""
    rng = np.random.default_rng(seed)
    if n_tilts is None:
        n_tilts = int(round((tilt_max - tilt_min) / tilt_step)) + 1
    angles = np.linspace(tilt_min, tilt_max, n_tilts).astype(np.float32)
    cx = rng.uniform(-nx / 2, nx / 2, n_blobs)
    cy = rng.uniform(-ny / 2, ny / 2, n_blobs)
    cz = rng.uniform(-vol_z / 2, vol_z / 2, n_blobs)
    sg = rng.uniform(sigma[0], sigma[1], n_blobs)
    am = rng.uniform(amp[0], amp[1], n_blobs)
    if background:
        nb = 12
        bx = rng.uniform(-nx / 2, nx / 2, nb)
        by = rng.uniform(-ny / 2, ny / 2, nb)
        bz = rng.uniform(-vol_z / 4, vol_z / 4, nb)
        bs = rng.uniform(nx / 6, nx / 3, nb)
        ba = rng.uniform(0.002, 0.006, nb)
        cx, cy, cz = np.r_[cx, bx], np.r_[cy, by], np.r_[cz, bz]
        sg, am = np.r_[sg, bs], np.r_[am, ba]
    zt = int(np.argmin(np.abs(angles)))
    shifts = rng.normal(0.0, shift_sd, (n_tilts, 2))
    shifts[:, 0] += drift * (np.arange(n_tilts) - zt)
    shifts[zt] = 0.0
    ca, sa = math.cos(math.radians(axis)), math.sin(math.radians(axis))
    stack = np.zeros((n_tilts, ny, nx), np.float64)
    for k, t in enumerate(angles.astype(np.float64)):
        tr = math.radians(t)
        u = cx * math.cos(tr) + cz * math.sin(tr)
        v = cy
        # raw position = R(axis) (u, v) + centre + shift
        rx = ca * u - sa * v + nx / 2 + shifts[k, 0]
        ry = sa * u + ca * v + ny / 2 + shifts[k, 1]
        _render(nx, ny, np.stack([rx, ry], 1), sg, am, stack[k])
    sig_sd = float(stack.std())
    if snr and snr > 0:
        noise_sd = sig_sd / math.sqrt(snr)
        if poisson:
            # scale to a dose where shot noise carries half the noise power
            lam = stack / max(stack.mean(), 1e-12) * 20.0
            shot = rng.poisson(lam).astype(np.float64) / 20.0 * stack.mean()
            stack = shot + rng.normal(0.0, noise_sd * math.sqrt(0.5), stack.shape)
        else:
            stack = stack + rng.normal(0.0, noise_sd, stack.shape)
    return Series(stack=stack.astype(np.float32), angles=angles,
                  shifts=shifts.astype(np.float32), axis=float(axis),
                  thickness=int(thickness), nproj=int(nproj), name=name)


def config(cfg: int, scale: float = 1.0, seed: int | None = None) -> Series:
    """The benchmark configurations, optionally shrunk by `scale` for tests.

    1: plain method, small (512^2, 41 tilts, -60..60 step 3, axis 86.3, T=100)
    2: realistic single series (2048^2, 61 tilts, step 2, axis 84.7, T=300,
       drift 0.3 px/tilt, Poisson+Gaussian noise at SNR 0.05)
    3: large detector (4096^2, 61 tilts, T=300, -p 20)
    """
    s = seed if seed is not None else 1000 + cfg
    if cfg == 1:
        n = int(512 * scale) // 2 * 2
        return make_series(nx=n, ny=n, vol_z=max(8, int(128 * scale)),
                           n_blobs=max(20, int(200 * scale * scale)), seed=s,
                           thickness=max(8, int(100 * scale)) // 2 * 2, name="cfg1")
    if cfg == 2:
        n = int(2048 * scale) // 2 * 2
        return make_series(nx=n, ny=n, vol_z=max(8, int(300 * scale)),
                           n_blobs=max(30, int(3000 * scale * scale)), sigma=(1.5, 5.0),
                           tilt_step=2.0, axis=84.7, shift_sd=8.0, drift=0.3, snr=0.05,
                           poisson=True, background=True, seed=s,
                           thickness=max(8, int(300 * scale)) // 2 * 2, name="cfg2")
    if cfg == 3:
        n = int(4096 * scale) // 2 * 2
        return make_series(nx=n, ny=n, vol_z=max(8, int(400 * scale)),
                           n_blobs=max(40, int(12000 * scale * scale)), sigma=(1.5, 5.0),
                           tilt_step=2.0, axis=84.7, shift_sd=12.0, snr=0.05, seed=s,
                           thickness=max(8, int(300 * scale)) // 2 * 2, nproj=20, name="cfg3")
    raise ValueError(f"unknown configuration {cfg}")


def make_series_fast(nx=512, ny=512, vol_z=128, n_blobs=200, sigma=(2.0, 6.0), amp=(0.5, 1.5),
                     tilt_min=-60.0, tilt_max=60.0, tilt_step=3.0, axis=86.3, shift_sd=4.0,
                     drift=0.0, snr=0.1, poisson=False, background=False, seed=1001,
                     thickness=100, nproj=10, name="synthetic", n_tilts=None, device="cpu"):
    """make_series' distribution, generated with torch on `device` in seconds.

    The phantom, the tilt geometry and the shifts are drawn exactly as make_series
    draws them (same numpy generator and order).  Each tilt image is the sum of
    the blobs' separable Gaussians, evaluated over the whole image as one matrix
    product (make_series truncates each blob at 4 sigma and adds blob by blob),
    in float32; the noise comes from a torch generator seeded with `seed` on
    `device`, so images are reproducible per device kind but not equal to
    make_series' bit for bit.  Returns a Series whose `stack` is a float32 torch
    tensor on `device`."""
    import torch
    rng = np.random.default_rng(seed)
    if n_tilts is None:
        n_tilts = int(round((tilt_max - tilt_min) / tilt_step)) + 1
    angles = np.linspace(tilt_min, tilt_max, n_tilts).astype(np.float32)
    cx = rng.uniform(-nx / 2, nx / 2, n_blobs)
    cy = rng.uniform(-ny / 2, ny / 2, n_blobs)
    cz = rng.uniform(-vol_z / 2, vol_z / 2, n_blobs)
    sg = rng.uniform(sigma[0], sigma[1], n_blobs)
    am = rng.uniform(amp[0], amp[1], n_blobs)
    if background:
        nb = 12
        bx = rng.uniform(-nx / 2, nx / 2, nb)
        by = rng.uniform(-ny / 2, ny / 2, nb)
        bz = rng.uniform(-vol_z / 4, vol_z / 4, nb)
        bs = rng.uniform(nx / 6, nx / 3, nb)
        ba = rng.uniform(0.002, 0.006, nb)
        cx, cy, cz = np.r_[cx, bx], np.r_[cy, by], np.r_[cz, bz]
        sg, am = np.r_[sg, bs], np.r_[am, ba]
    zt = int(np.argmin(np.abs(angles)))
    shifts = rng.normal(0.0, shift_sd, (n_tilts, 2))
    shifts[:, 0] += drift * (np.arange(n_tilts) - zt)
    shifts[zt] = 0.0
    ca, sa = math.cos(math.radians(axis)), math.sin(math.radians(axis))
    dev = torch.device(device)
    f32 = dict(dtype=torch.float32, device=dev)
    px = torch.arange(nx, **f32)
    py = torch.arange(ny, **f32)
    inv2s2 = torch.tensor(1.0 / (2.0 * sg * sg), **f32)
    coef = torch.tensor(am * sg * math.sqrt(2 * math.pi), **f32)
    stack = torch.empty((n_tilts, ny, nx), **f32)
    for k, t in enumerate(angles.astype(np.float64)):
        tr = math.radians(t)
        u = cx * math.cos(tr) + cz * math.sin(tr)
        v = cy
        rx = torch.tensor(ca * u - sa * v + nx / 2 + shifts[k, 0], **f32)
        ry = torch.tensor(sa * u + ca * v + ny / 2 + shifts[k, 1], **f32)
        gx = torch.exp(-(px[None, :] - rx[:, None]) ** 2 * inv2s2[:, None])   # (nb, nx)
        gy = torch.exp(-(py[None, :] - ry[:, None]) ** 2 * inv2s2[:, None])   # (nb, ny)
        torch.matmul(gy.t() * coef[None, :], gx, out=stack[k])
    if snr and snr > 0:
        gen = torch.Generator(device=dev).manual_seed(int(seed))
        sig_sd = float(stack.double().std())
        noise_sd = sig_sd / math.sqrt(snr)
        if poisson:
            mean = float(stack.double().mean())
            lam = (stack / max(mean, 1e-12) * 20.0).clamp_(min=0.0)
            shot = torch.poisson(lam, generator=gen)
            del lam
            shot.mul_(mean / 20.0)
            shot.add_(torch.randn(shot.shape, generator=gen, **f32), alpha=noise_sd * math.sqrt(0.5))
            stack = shot
        else:
            stack.add_(torch.randn(stack.shape, generator=gen, **f32), alpha=noise_sd)
    return Series(stack=stack, angles=angles, shifts=shifts.astype(np.float32), axis=float(axis),
                  thickness=int(thickness), nproj=int(nproj), name=name)


def config_fast(cfg: int, seed: int | None = None, device="cpu", scale: float = 1.0) -> Series:
    """config()'s series drawn with make_series_fast (same parameters)."""
    s = seed if seed is not None else 1000 + cfg
    if cfg == 2:
        n = int(2048 * scale) // 2 * 2
        return make_series_fast(nx=n, ny=n, vol_z=max(8, int(300 * scale)),
                                n_blobs=max(30, int(3000 * scale * scale)), sigma=(1.5, 5.0),
                                tilt_step=2.0, axis=84.7, shift_sd=8.0, drift=0.3, snr=0.05,
                                poisson=True, background=True, seed=s,
                                thickness=max(8, int(300 * scale)) // 2 * 2, name="cfg2",
                                device=device)
    raise ValueError(f"no fast form of configuration {cfg}")


def uneven_params(j: int, size=None, seed0: int = 4000) -> dict:
    """Parameters of series j of the uneven batch: image size U{1024, 2048, 3072,
    4096}^2 (or `size`), tilt count U{31, 41, 61} over a range of +-45..+-60
    degrees, slab thickness U{150, 200, 300}, tilt axis U(80, 95) degrees, shifts
    N(0, 6 px), SNR U(0.03, 0.2); drawn from a generator seeded with seed0 + j."""
    rng = np.random.default_rng(seed0 + j)
    n = int(rng.choice([1024, 2048, 3072, 4096]))
    if size is not None:
        n = int(size)
    tilts = int(rng.choice([31, 41, 61]))
    rng_deg = float(rng.uniform(45.0, 60.0))
    return dict(nx=n, ny=n, vol_z=max(32, n * 300 // 2048), n_blobs=max(100, 3000 * n * n // 2048 ** 2),
                sigma=(1.5, 5.0), tilt_min=-rng_deg, tilt_max=rng_deg, n_tilts=tilts,
                axis=float(rng.uniform(80.0, 95.0)), shift_sd=6.0, snr=float(rng.uniform(0.03, 0.2)),
                poisson=True, background=True, seed=seed0 + j,
                thickness=int(rng.choice([150, 200, 300])), name=f"uneven{j}")


def uneven_series(j: int, device="cpu", size=None, seed0: int = 4000) -> Series:
    """Series j of the uneven batch (uneven_params), generated with make_series_fast."""
    return make_series_fast(device=device, **uneven_params(j, size=size, seed0=seed0))
