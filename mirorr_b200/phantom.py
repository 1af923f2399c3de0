"""Seeded synthetic image pairs for the block-matching registration path.

The reference's sample CT/MR pair is not available, so workloads are
synthetic phantoms with the shapes and value distributions of the named
configurations:

* fixed image: sum of K anisotropic 3D Gaussians (centres uniform in the
  volume, sigma per axis U[4, 16] voxels, random orientation, amplitude
  U[0, 1]), normalised to [0, 1] by min/max, plus N(0, 0.01) noise
  (variance 0.01, sigma 0.1);
* moving image: the normalised fixed image through the non-monotone map
  0.6 sin(3v) + 0.4 v^2 (a second "modality"), resampled through the known
  transform T_true (moving -> fixed physical points, centred on the volume
  centre, trilinear, outside = 0), plus fresh noise;
* optional multiplicative quadratic bias field of +-20 %.

Rigid T_true: axis uniform on the sphere, angle U[0, max_angle], translation
U[-max_shift, max_shift] voxels per axis.  Affine T_true adds per-axis scale
U[0.9, 1.1] and shear U[-0.05, 0.05].

Generation is host-side numpy (scipy for the moving-image interpolation);
it is input preparation, not part of the measured path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Phantom:
    fixed: np.ndarray          # (nz, ny, nx) float32
    moving: np.ndarray         # (nz, ny, nx) float32
    spacing: np.ndarray        # (3,) mm, x y z
    origin: np.ndarray         # (3,)
    true_matrix: np.ndarray    # (3, 3): moving -> fixed, about `center`
    true_offset: np.ndarray    # (3,): y = M x + offset
    center: np.ndarray         # (3,) physical centre of the volume
    kind: str
    seed: int


def random_rotation(rng, max_angle_deg):
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    angle = math.radians(rng.uniform(0.0, max_angle_deg))
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + math.sin(angle) * k + (1 - math.cos(angle)) * (k @ k)


def _uniform_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    x, y, z, w = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def gaussian_field(shape_zyx, n_gauss, rng):
    nz, ny, nx = shape_zyx
    vol = np.zeros(shape_zyx, np.float64)
    for _ in range(n_gauss):
        c = rng.uniform([0, 0, 0], [nx - 1, ny - 1, nz - 1])
        sig = rng.uniform(4.0, 16.0, size=3)
        r = _uniform_rotation(rng)
        cov_inv = r @ np.diag(1.0 / sig ** 2) @ r.T
        a = rng.uniform(0.0, 1.0)
        ext = 4.0 * sig.max()
        lo = np.maximum(np.floor(c - ext), 0).astype(int)
        hi = np.minimum(np.ceil(c + ext) + 1, [nx, ny, nz]).astype(int)
        xs = np.arange(lo[0], hi[0]) - c[0]
        ys = np.arange(lo[1], hi[1]) - c[1]
        zs = np.arange(lo[2], hi[2]) - c[2]
        dz, dy, dx = np.meshgrid(zs, ys, xs, indexing="ij")
        q = (cov_inv[0, 0] * dx * dx + cov_inv[1, 1] * dy * dy + cov_inv[2, 2] * dz * dz
             + 2 * cov_inv[0, 1] * dx * dy + 2 * cov_inv[0, 2] * dx * dz
             + 2 * cov_inv[1, 2] * dy * dz)
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += a * np.exp(-0.5 * q)
    return vol


def intensity_map(v):
    return 0.6 * np.sin(3.0 * v) + 0.4 * v * v


def make_phantom(shape_xyz, n_gauss=40, kind="rigid", seed=0, spacing=(1.0, 1.0, 1.0),
                 max_angle_deg=5.0, max_shift_vox=8.0, noise_var=0.01, bias=0.0) -> Phantom:
    """Fixed/moving pair with a known transform (see module docstring)."""
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    nx, ny, nz = shape_xyz
    spacing = np.asarray(spacing, np.float64)
    origin = np.zeros(3)
    clean = gaussian_field((nz, ny, nx), n_gauss, rng)
    lo, hi = clean.min(), clean.max()
    clean = (clean - lo) / (hi - lo if hi > lo else 1.0)
    if bias > 0.0:
        zz, yy, xx = np.meshgrid(np.linspace(-1, 1, nz), np.linspace(-1, 1, ny),
                                 np.linspace(-1, 1, nx), indexing="ij")
        coef = rng.uniform(-1, 1, size=6)
        b = coef[0] * xx * xx + coef[1] * yy * yy + coef[2] * zz * zz + coef[3] * xx * yy \
            + coef[4] * yy * zz + coef[5] * xx * zz
        b = b / max(np.abs(b).max(), 1e-12)
        clean = clean * (1.0 + bias * b)
    sigma = math.sqrt(noise_var)
    fixed = (clean + rng.normal(0.0, sigma, size=clean.shape)).astype(np.float32)

    rot = random_rotation(rng, max_angle_deg)
    if kind == "affine":
        scale = np.diag(rng.uniform(0.9, 1.1, size=3))
        shear = np.eye(3)
        shear[0, 1], shear[0, 2], shear[1, 2] = rng.uniform(-0.05, 0.05, size=3)
        m = rot @ scale @ shear
    else:
        m = rot
    shift = rng.uniform(-max_shift_vox, max_shift_vox, size=3) * spacing
    center = origin + spacing * (np.array([nx, ny, nz], np.float64) - 1.0) / 2.0
    offset = center + shift - m @ center  # T(x) = M (x - c) + c + shift

    mapped = intensity_map(clean)
    # moving(x) = mapped(T(x)) for x on the moving grid (same geometry)
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    pts = np.stack([xx, yy, zz], axis=-1).reshape(-1, 3) * spacing + origin
    tp = pts @ m.T + offset
    ci = (tp - origin) / spacing
    coords = np.stack([ci[:, 2], ci[:, 1], ci[:, 0]])
    mov = ndimage.map_coordinates(mapped, coords, order=1, mode="constant", cval=0.0)
    mov = mov.reshape(nz, ny, nx)
    moving = (mov + rng.normal(0.0, sigma, size=mov.shape)).astype(np.float32)
    return Phantom(fixed, moving, spacing, origin, m, offset, center, kind, seed)


def make_phantom_gpu(shape_xyz, n_gauss=200, kind="affine", seed=0, max_angle_deg=8.0,
                     max_shift_vox=12.0, noise_var=0.01, bias=0.0, device="cuda:0") -> Phantom:
    """The same construction as make_phantom for large volumes, evaluated on a
    GPU with torch (1 mm spacing, origin 0): Gaussians over their +-4 sigma
    boxes, min/max normalisation, the quadratic bias field, N(0, noise_var)
    noise, the intensity map and trilinear resampling through T_true (zero
    outside).  The draws come from the same seeded numpy generator; the
    arithmetic is float32, so values differ from make_phantom's float64 ones
    by rounding.  Input preparation only."""
    import torch

    rng = np.random.default_rng(seed)
    nx, ny, nz = shape_xyz
    dev = torch.device(device)
    vol = torch.zeros((nz, ny, nx), dtype=torch.float32, device=dev)
    for _ in range(n_gauss):
        c = rng.uniform([0, 0, 0], [nx - 1, ny - 1, nz - 1])
        sig = rng.uniform(4.0, 16.0, size=3)
        r = _uniform_rotation(rng)
        ci = r @ np.diag(1.0 / sig ** 2) @ r.T
        a = rng.uniform(0.0, 1.0)
        ext = 4.0 * sig.max()
        lo = np.maximum(np.floor(c - ext), 0).astype(int)
        hi = np.minimum(np.ceil(c + ext) + 1, [nx, ny, nz]).astype(int)
        xs = torch.arange(lo[0], hi[0], device=dev, dtype=torch.float32) - float(c[0])
        ys = torch.arange(lo[1], hi[1], device=dev, dtype=torch.float32) - float(c[1])
        zs = torch.arange(lo[2], hi[2], device=dev, dtype=torch.float32) - float(c[2])
        dz, dy, dx = torch.meshgrid(zs, ys, xs, indexing="ij")
        q = (ci[0, 0] * dx * dx + ci[1, 1] * dy * dy + ci[2, 2] * dz * dz + 2 * ci[0, 1] * dx * dy
             + 2 * ci[0, 2] * dx * dz + 2 * ci[1, 2] * dy * dz)
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += float(a) * torch.exp(-0.5 * q)
    lo_v, hi_v = vol.min(), vol.max()
    clean = (vol - lo_v) / torch.clamp(hi_v - lo_v, min=1e-12)
    if bias > 0.0:
        zz = torch.linspace(-1, 1, nz, device=dev).view(nz, 1, 1)
        yy = torch.linspace(-1, 1, ny, device=dev).view(1, ny, 1)
        xx = torch.linspace(-1, 1, nx, device=dev).view(1, 1, nx)
        coef = rng.uniform(-1, 1, size=6)
        b = (coef[0] * xx * xx + coef[1] * yy * yy + coef[2] * zz * zz + coef[3] * xx * yy
             + coef[4] * yy * zz + coef[5] * xx * zz)
        b = b / torch.clamp(b.abs().max(), min=1e-12)
        clean = clean * (1.0 + bias * b)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(rng.integers(2 ** 62)))
    sigma = math.sqrt(noise_var)
    fixed = clean + sigma * torch.randn(clean.shape, generator=gen, device=dev)

    rot = random_rotation(rng, max_angle_deg)
    if kind == "affine":
        scale = np.diag(rng.uniform(0.9, 1.1, size=3))
        shear = np.eye(3)
        shear[0, 1], shear[0, 2], shear[1, 2] = rng.uniform(-0.05, 0.05, size=3)
        m = rot @ scale @ shear
    else:
        m = rot
    shift = rng.uniform(-max_shift_vox, max_shift_vox, size=3)
    center = (np.array([nx, ny, nz], np.float64) - 1.0) / 2.0
    offset = center + shift - m @ center
    mapped = 0.6 * torch.sin(3.0 * clean) + 0.4 * clean * clean
    # moving(x) = mapped(T(x)), plane by plane (normalised grid_sample coordinates)
    mov = torch.empty_like(mapped)
    mt = torch.tensor(m, dtype=torch.float32, device=dev)
    ot = torch.tensor(offset, dtype=torch.float32, device=dev)
    yy, xx = torch.meshgrid(torch.arange(ny, device=dev, dtype=torch.float32),
                            torch.arange(nx, device=dev, dtype=torch.float32), indexing="ij")
    norm = torch.tensor([2.0 / max(nx - 1, 1), 2.0 / max(ny - 1, 1), 2.0 / max(nz - 1, 1)],
                        device=dev)
    src = mapped.view(1, 1, nz, ny, nx)
    for z in range(nz):
        pts = torch.stack([xx, yy, torch.full_like(xx, float(z))], dim=-1)
        tp = pts @ mt.T + ot
        g = (tp * norm - 1.0).view(1, 1, ny, nx, 3)
        mov[z] = torch.nn.functional.grid_sample(src, g, mode="bilinear", padding_mode="zeros",
                                                 align_corners=True).view(ny, nx)
    moving = mov + sigma * torch.randn(mov.shape, generator=gen, device=dev)
    out = Phantom(fixed.cpu().numpy().astype(np.float32), moving.cpu().numpy().astype(np.float32),
                  np.ones(3), np.zeros(3), m, offset, center, kind, seed)
    del vol, clean, fixed, mapped, mov, moving, src
    torch.cuda.empty_cache()
    return out


def tre(matrix, offset, true_matrix, true_offset, shape_xyz, spacing, origin=None, step=8):
    """Mean target registration error (mm) over a voxel lattice of the volume."""
    nx, ny, nz = shape_xyz
    origin = np.zeros(3) if origin is None else origin
    g = np.stack(np.meshgrid(np.arange(0, nx, step), np.arange(0, ny, step),
                             np.arange(0, nz, step), indexing="ij"), -1).reshape(-1, 3)
    p = g * np.asarray(spacing) + origin
    a = p @ np.asarray(matrix).T + np.asarray(offset)
    b = p @ np.asarray(true_matrix).T + np.asarray(true_offset)
    return float(np.mean(np.linalg.norm(a - b, axis=1)))
