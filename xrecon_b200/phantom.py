"""Analytic ellipse / ellipsoid phantoms.

``phantom`` keeps the call signature of XRecon's ``xrecon.utils.phantom``
(xrecon/utils/phantom.py:10-29): rows span y from +1 to -1, columns x from -1
to 1, each ellipse row is (value, a, b, x0, y0, phi_deg) in 2D and
(value, a, b, c, x0, y0, z0, phi_deg) in 3D (rotation about z).  The
Shepp-Logan tables are the published ones (Shepp & Logan 1974; the
"modified" contrast variant of Toft 1996; the 3D extension of Kak & Slaney).

The ``random_*`` helpers generate the seeded synthetic phantoms used by the
benchmark and the tests (uniform random centres, semi-axes, rotations and
densities).
"""
from __future__ import annotations

import numpy as np

_SL2 = np.array([
    [2.00, 0.6900, 0.9200, 0.00, 0.0000, 0],
    [-0.98, 0.6624, 0.8740, 0.00, -0.0184, 0],
    [-0.02, 0.1100, 0.3100, 0.22, 0.0000, -18],
    [-0.02, 0.1600, 0.4100, -0.22, 0.0000, 18],
    [0.01, 0.2100, 0.2500, 0.00, 0.3500, 0],
    [0.01, 0.0460, 0.0460, 0.00, 0.1000, 0],
    [0.02, 0.0460, 0.0460, 0.00, -0.1000, 0],
    [0.01, 0.0460, 0.0230, -0.08, -0.6050, 0],
    [0.01, 0.0230, 0.0230, 0.00, -0.6060, 0],
    [0.01, 0.0230, 0.0460, 0.06, -0.6050, 0],
])
_MSL2 = _SL2.copy()
_MSL2[:, 0] = [1.0, -0.8, -0.2, -0.2, 0.1, 0.1, 0.1, 0.1, 0.1, 0.1]

_SL3 = np.array([
    [2.00, 0.6900, 0.9200, 0.900, 0.00, 0.000, 0.000, 0],
    [-0.80, 0.6624, 0.8740, 0.880, 0.00, 0.000, 0.000, 0],
    [-0.20, 0.4100, 0.1600, 0.210, -0.22, 0.000, -0.250, 108],
    [-0.20, 0.3100, 0.1100, 0.220, 0.22, 0.000, -0.250, 72],
    [0.20, 0.2100, 0.2500, 0.500, 0.00, 0.350, -0.250, 0],
    [0.20, 0.0460, 0.0460, 0.046, 0.00, 0.100, -0.250, 0],
    [0.10, 0.0460, 0.0230, 0.020, -0.08, -0.650, -0.250, 0],
    [0.10, 0.0460, 0.0230, 0.020, 0.06, -0.650, -0.250, 90],
    [0.20, 0.0560, 0.0400, 0.100, 0.06, -0.105, 0.625, 90],
    [-0.20, 0.0560, 0.0560, 0.100, 0.00, 0.100, 0.625, 0],
])
_MSL3 = _SL3.copy()
_MSL3[:, 0] = [1.0, -0.8, -0.2, -0.2, 0.1, 0.1, 0.1, 0.1, 0.1, -0.1]


def _tables(p_type: str, dim: int) -> np.ndarray:
    key = p_type.lower().strip()
    table = {("shepp-logan", 2): _SL2, ("modified shepp-logan", 2): _MSL2,
             ("shepp-logan", 3): _SL3, ("modified shepp-logan", 3): _MSL3}.get((key, dim))
    if table is None:
        raise ValueError(f"Unknown phantom type '{p_type}' for dim={dim}")
    return table


def create_phantom2d(shape, ellipses) -> np.ndarray:
    if len(shape) != 2:
        raise ValueError("2D phantom shape should have 2 dimensions")
    e = np.asarray(ellipses, dtype=np.float32)
    if e.ndim != 2 or e.shape[1] != 6:
        raise ValueError("2D phantom ellipses should have shape [N, 6]")
    rows, cols = shape
    y = np.linspace(1.0, -1.0, rows, dtype=np.float64)[:, None]
    x = np.linspace(-1.0, 1.0, cols, dtype=np.float64)[None, :]
    img = np.zeros(shape, dtype=np.float32)
    for val, a, b, x0, y0, phi in e:
        c, s = np.cos(np.deg2rad(phi)), np.sin(np.deg2rad(phi))
        u = (x - x0) * c + (y - y0) * s
        v = (y - y0) * c - (x - x0) * s
        img[(u * u) / (a * a) + (v * v) / (b * b) <= 1.0] += val
    return img


def create_phantom3d(shape, ellipses, zlims=(-1.0, 1.0)) -> np.ndarray:
    if len(shape) != 3:
        raise ValueError("3D phantom shape should have 3 dimensions")
    e = np.asarray(ellipses, dtype=np.float32)
    if e.ndim != 2 or e.shape[1] != 8:
        raise ValueError("3D phantom ellipses should have shape [N, 8]")
    if len(zlims) != 2 or zlims[0] > zlims[1]:
        raise ValueError("zlims should be (lower, upper)")
    rows, cols, slices = shape
    y = np.linspace(1.0, -1.0, rows)[:, None, None]
    x = np.linspace(-1.0, 1.0, cols)[None, :, None]
    z = np.linspace(zlims[0], zlims[1], slices)[None, None, :]
    vol = np.zeros(shape, dtype=np.float32)
    for val, a, b, cc, x0, y0, z0, phi in e:
        c, s = np.cos(np.deg2rad(phi)), np.sin(np.deg2rad(phi))
        u = (x - x0) * c + (y - y0) * s
        v = (y - y0) * c - (x - x0) * s
        w = z - z0
        vol[(u * u) / (a * a) + (v * v) / (b * b) + (w * w) / (cc * cc) <= 1.0] += val
    return vol


def phantom(n=256, p_type: str = "Modified Shepp-Logan", ellipses=None, dim: int = 2,
            zlims=(-1.0, 1.0)) -> np.ndarray:
    shape = tuple([int(n)] * dim) if np.isscalar(n) else tuple(int(v) for v in n)
    if ellipses is None:
        ellipses = _tables(p_type, dim)
    if dim == 2:
        return create_phantom2d(shape, ellipses)
    if dim == 3:
        return create_phantom3d(shape, ellipses, zlims)
    raise ValueError(f"Unexpected dim: {dim}")


def random_ellipses2d(count: int, seed: int, axes_px=(5.0, 60.0), n: int = 256,
                      density=(-0.2, 0.5), inner: float = 0.8) -> np.ndarray:
    """Seeded random ellipses in phantom units: centres uniform in the inner
    `inner` fraction, semi-axes uniform in `axes_px` pixels of an n-pixel
    image, rotation uniform, density uniform in `density`."""
    rng = np.random.default_rng(seed)
    e = np.empty((count, 6), dtype=np.float64)
    e[:, 0] = rng.uniform(density[0], density[1], count)
    e[:, 1:3] = rng.uniform(axes_px[0], axes_px[1], (count, 2)) * (2.0 / n)
    e[:, 3:5] = rng.uniform(-inner, inner, (count, 2))
    e[:, 5] = rng.uniform(0.0, 180.0, count)
    return e


def random_ellipsoids3d(count: int, seed: int, axes=(0.05, 0.4), density=(-0.2, 0.5),
                        inner: float = 0.7) -> np.ndarray:
    rng = np.random.default_rng(seed)
    e = np.empty((count, 8), dtype=np.float64)
    e[:, 0] = rng.uniform(density[0], density[1], count)
    e[:, 1:4] = rng.uniform(axes[0], axes[1], (count, 3))
    e[:, 4:7] = rng.uniform(-inner, inner, (count, 3))
    e[:, 7] = rng.uniform(0.0, 180.0, count)
    return e


def shepp_logan_plus_ellipses2d(n: int, count: int, seed: int) -> np.ndarray:
    """Modified Shepp-Logan plus `count` seeded random ellipses (semi-axes 5-60
    px, densities in [-0.2, 0.5])."""
    return create_phantom2d((n, n), np.concatenate([_MSL2, random_ellipses2d(count, seed, n=n)]))


def shepp_logan_plus_ellipsoids3d(shape, count: int, seed: int) -> np.ndarray:
    """3D Shepp-Logan plus `count` seeded random ellipsoids; shape (rows,
    cols, slices) as ``create_phantom3d``."""
    return create_phantom3d(shape, np.concatenate([_SL3, random_ellipsoids3d(count, seed)]))


def ellipsoid_volume_torch(shape_dhw, ellipsoids, device, dtype=None):
    """Rasterise ellipsoids (rows as ``create_phantom3d``) directly on a torch
    device into a [D, H, W] volume; x spans [-1, 1] over W, y [1, -1] over H,
    z [-1, 1] over D."""
    import torch
    D, H, W = shape_dhw
    dtype = dtype or torch.float32
    z = torch.linspace(-1.0, 1.0, D, device=device, dtype=torch.float32)[:, None, None]
    y = torch.linspace(1.0, -1.0, H, device=device, dtype=torch.float32)[None, :, None]
    x = torch.linspace(-1.0, 1.0, W, device=device, dtype=torch.float32)[None, None, :]
    vol = torch.zeros((D, H, W), device=device, dtype=torch.float32)
    for val, a, b, cc, x0, y0, z0, phi in np.asarray(ellipsoids, dtype=np.float64):
        c, s = float(np.cos(np.deg2rad(phi))), float(np.sin(np.deg2rad(phi)))
        u = (x - x0) * c + (y - y0) * s
        v = (y - y0) * c - (x - x0) * s
        w = z - z0
        inside = (u * u) / (a * a) + (v * v) / (b * b) + (w * w) / (cc * cc) <= 1.0
        vol += inside.to(torch.float32) * float(val)
    return vol.to(dtype)


def random_ellipsoid_volume(shape_dhw, count: int, seed: int, density=(0.0, 1.0)) -> np.ndarray:
    """Random-ellipsoid volume in [D, H, W] layout (the projector's image
    layout), densities uniform in `density`."""
    D, H, W = shape_dhw
    vol = create_phantom3d((H, W, D), random_ellipsoids3d(count, seed, density=density))
    return np.ascontiguousarray(np.transpose(vol, (2, 0, 1)))
