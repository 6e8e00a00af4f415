"""Seeded synthetic near-field mmWave scenes.

The reference processes robot-collected 77 GHz data whose sample set is an external
download; these generators stand in for it with point-scatterer scenes of the same
shapes (planar synthetic aperture, FMCW frequency sweep, voxel grid).

Forward model (per antenna position ``a`` and frequency ``f``)::

    s(a, f) = sum_p rho_p * exp(sign * j * 4*pi*f*|p - a| / c) / |p - a|**2  + noise

``sign=-1`` is the convention the benchmark and parity runs use.  ``sign=+1`` is the
reference's own channel-simulator convention
(src/data_processing/isosurface_optimization.py:208, ``exp(+j*2*pi*d/lambda)``), under
which the reference's correlation ``exp(-j*2*pi*d*f/c)`` focuses.  Noise is complex
Gaussian at the requested SNR relative to the mean ``|s|^2`` over the whole array.

The frequency sweep is ``f_j = f_lo + j*(f_hi - f_lo)/(F - 1)``; in the reference
kernel's parametrisation that is ``wavelength = c/f_lo`` and ``slope = (f_hi-f_lo)/(F-1)``
(src/data_processing/cuda/imaging_gpu.cu:112).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

C = 2.99792458e8


@dataclasses.dataclass
class Scene:
    name: str
    x_locs: np.ndarray          # float32 [NX]
    y_locs: np.ndarray          # float32 [NY]
    z_locs: np.ndarray          # float32 [NZ]
    antenna_locs: np.ndarray    # float32 [A, 3]
    meas: np.ndarray            # complex64 [A, F]
    f_lo: float
    f_hi: float
    points: np.ndarray          # float64 [P, 3]
    rho: np.ndarray             # float64 [P]
    sign: int
    snr_db: float
    seed: int
    sphere: tuple | None = None  # (centre xyz, radius) when the scene is a sphere

    @property
    def num_freqs(self) -> int:
        return int(self.meas.shape[1])

    @property
    def wavelength(self) -> float:
        return C / self.f_lo

    @property
    def slope(self) -> float:
        return (self.f_hi - self.f_lo) / (self.num_freqs - 1)

    @property
    def grid_shape(self) -> tuple:
        return (len(self.x_locs), len(self.y_locs), len(self.z_locs))

    @property
    def num_voxels(self) -> int:
        nx, ny, nz = self.grid_shape
        return nx * ny * nz

    @property
    def updates(self) -> int:
        """voxel * antenna * frequency updates of one full backprojection."""
        return self.num_voxels * self.antenna_locs.shape[0] * self.num_freqs

    def voxel_centres(self, idx: np.ndarray | None = None) -> np.ndarray:
        """float32 [n, 3] centres of the voxels with flat index idx (x-major, z fastest)."""
        nx, ny, nz = self.grid_shape
        if idx is None:
            idx = np.arange(nx * ny * nz)
        idx = np.asarray(idx, dtype=np.int64)
        ix, rem = np.divmod(idx, ny * nz)
        iy, iz = np.divmod(rem, nz)
        return np.stack([self.x_locs[ix], self.y_locs[iy], self.z_locs[iz]], axis=1)


def planar_aperture(n: int, pitch: float, nx: int | None = None) -> np.ndarray:
    """n x n (or nx x n) antenna positions at ``pitch`` in z=0, centred at x=y=0.

    Index order is raster: antenna (iy, ix) -> iy*nx + ix."""
    nx = n if nx is None else nx
    xs = (np.arange(nx) - (nx - 1) / 2.0) * pitch
    ys = (np.arange(n) - (n - 1) / 2.0) * pitch
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    ant = np.stack([xx.ravel(), yy.ravel(), np.zeros(xx.size)], axis=1)
    return ant.astype(np.float32)


def voxel_axes(n: int, spacing: float, centre) -> tuple:
    k = (np.arange(n) - (n - 1) / 2.0) * spacing
    return tuple((c + k).astype(np.float32) for c in centre)


def sphere_surface(rng, n, radius, centre):
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return np.asarray(centre, dtype=np.float64) + radius * v


def box_surface(rng, n, size, centre):
    """Uniform on the surface of an axis-aligned box with edge lengths ``size``."""
    sx, sy, sz = size
    areas = np.array([sy * sz, sy * sz, sx * sz, sx * sz, sx * sy, sx * sy])
    face = rng.choice(6, size=n, p=areas / areas.sum())
    u = rng.random((n, 3)) - 0.5
    p = u * np.array(size)
    axis = face // 2
    sgn = np.where(face % 2 == 0, -0.5, 0.5)
    p[np.arange(n), axis] = sgn * np.array(size)[axis]
    return p + np.asarray(centre, dtype=np.float64)


def cylinder_surface(rng, n, radius, height, centre):
    """Uniform on the closed surface of a z-axis cylinder (side + caps)."""
    side = 2 * math.pi * radius * height
    cap = math.pi * radius * radius
    which = rng.choice(3, size=n, p=np.array([side, cap, cap]) / (side + 2 * cap))
    th = rng.random(n) * 2 * math.pi
    r = np.where(which == 0, radius, radius * np.sqrt(rng.random(n)))
    z = np.where(which == 0, (rng.random(n) - 0.5) * height,
                 np.where(which == 1, -height / 2, height / 2))
    p = np.stack([r * np.cos(th), r * np.sin(th), z], axis=1)
    return p + np.asarray(centre, dtype=np.float64)


def box_cylinder_union_surface(rng, n, box_size, cyl_radius, cyl_height, centre):
    """Uniform on the boundary of (box U cylinder), both centred at ``centre``."""
    c = np.asarray(centre, dtype=np.float64)
    hb = np.array(box_size) / 2
    out = []
    got = 0
    while got < n:
        m = 2 * (n - got) + 64
        sb = 2 * (box_size[0] * box_size[1] + box_size[0] * box_size[2]
                  + box_size[1] * box_size[2])
        sc = 2 * math.pi * cyl_radius * cyl_height + 2 * math.pi * cyl_radius ** 2
        nb = rng.binomial(m, sb / (sb + sc))
        pb = box_surface(rng, nb, box_size, c)
        pc = cylinder_surface(rng, m - nb, cyl_radius, cyl_height, c)
        # drop points strictly inside the other solid
        q = pb - c
        in_cyl = (q[:, 0] ** 2 + q[:, 1] ** 2 < cyl_radius ** 2 * (1 - 1e-9)) & \
                 (np.abs(q[:, 2]) < cyl_height / 2 * (1 - 1e-9))
        q = pc - c
        in_box = np.all(np.abs(q) < hb * (1 - 1e-9), axis=1)
        pts = np.concatenate([pb[~in_cyl], pc[~in_box]])
        pts = pts[rng.permutation(len(pts))]
        out.append(pts[: n - got])
        got += len(out[-1])
    return np.concatenate(out)


def synthesize(ant, points, rho, freqs, sign=-1, device=None, chunk_elems=None):
    """Noise-free s(a, f) as complex128 [A, F] (float64 arithmetic throughout).

    Uses torch on ``device`` when given (e.g. 'cuda' for the large scenes), else numpy.
    """
    ant = np.asarray(ant, dtype=np.float64)
    pts = np.asarray(points, dtype=np.float64)
    rho = np.asarray(rho, dtype=np.float64)
    freqs = np.asarray(freqs, dtype=np.float64)
    A, F, P = ant.shape[0], freqs.shape[0], pts.shape[0]
    if device is None:
        chunk = chunk_elems or (1 << 23)
        pc = max(1, chunk // max(1, A * F))
        s = np.zeros((A, F), dtype=np.complex128)
        k = sign * 4 * math.pi * freqs / C
        for p0 in range(0, P, pc):
            p = pts[p0:p0 + pc]
            r = np.linalg.norm(ant[:, None, :] - p[None, :, :], axis=2)     # [A, pc]
            w = rho[p0:p0 + pc][None, :] / (r * r)
            ph = r[:, :, None] * k[None, None, :]                           # [A, pc, F]
            s += np.einsum("ap,apf->af", w, np.exp(1j * ph))
        return s
    import torch

    dev = torch.device(device)
    chunk = chunk_elems or (1 << 26)
    ta = torch.as_tensor(ant, device=dev)
    tp = torch.as_tensor(pts, device=dev)
    tr = torch.as_tensor(rho, device=dev)
    k = torch.as_tensor(sign * 4 * math.pi * freqs / C, device=dev)
    s_re = torch.zeros((A, F), dtype=torch.float64, device=dev)
    s_im = torch.zeros((A, F), dtype=torch.float64, device=dev)
    fb = F
    pc = max(1, chunk // max(1, A * fb))
    for p0 in range(0, P, pc):
        r = torch.cdist(ta, tp[p0:p0 + pc])                               # [A, pc]
        w = tr[p0:p0 + pc][None, :] / (r * r)
        ph = r[:, :, None] * k[None, None, :]
        s_re += torch.einsum("ap,apf->af", w, torch.cos(ph))
        s_im += torch.einsum("ap,apf->af", w, torch.sin(ph))
    return (s_re.cpu().numpy() + 1j * s_im.cpu().numpy())


def add_noise(rng, s, snr_db):
    p_sig = float(np.mean(np.abs(s) ** 2))
    p_n = p_sig / (10.0 ** (snr_db / 10.0))
    n = rng.standard_normal(s.shape + (2,))
    return s + math.sqrt(p_n / 2.0) * (n[..., 0] + 1j * n[..., 1])


def _finish(name, x, y, z, ant, pts, rho, f_lo, f_hi, nf, sign, snr, seed, rng,
            device, sphere=None):
    freqs = f_lo + np.arange(nf) * (f_hi - f_lo) / (nf - 1)
    s = synthesize(ant, pts, rho, freqs, sign=sign, device=device)
    s = add_noise(rng, s, snr)
    return Scene(name, x, y, z, ant, s.astype(np.complex64), f_lo, f_hi, pts, rho,
                 sign, snr, seed, sphere)


def sphere_scene(seed=0, n_ap=32, pitch=3e-3, nf=64, n_vox=48, spacing=4e-3,
                 n_pts=200, radius=0.05, centre=(0.0, 0.0, 0.4), snr_db=20.0,
                 sign=-1, device=None, name="sphere"):
    """Config-0 family: points uniform on a sphere, rho ~ U(0.5, 1)."""
    rng = np.random.default_rng(seed)
    pts = sphere_surface(rng, n_pts, radius, centre)
    rho = rng.uniform(0.5, 1.0, n_pts)
    ant = planar_aperture(n_ap, pitch)
    x, y, z = voxel_axes(n_vox, spacing, centre)
    return _finish(name, x, y, z, ant, pts, rho, 77e9, 81e9, nf, sign, snr_db, seed,
                   rng, device, sphere=(tuple(centre), radius))


def config0(sign=-1, device=None):
    """32x32 aperture @3 mm, F=64 over 77-81 GHz, 200-point sphere r=5 cm at z=0.4,
    48^3 voxels @4 mm, 20 dB, seed 0."""
    return sphere_scene(seed=0, sign=sign, device=device, name="sphere48_ap32_f64")


def config1(sign=-1, device=None):
    """128x128 aperture @2 mm, F=256, 128^3 voxels @2 mm centred at z=0.45, 20k points on
    the union of a 12x8x4 cm box and a r=4 cm, h=8 cm cylinder, rho ~ U(0.3,1), 15 dB."""
    rng = np.random.default_rng(1)
    centre = (0.0, 0.0, 0.45)
    pts = box_cylinder_union_surface(rng, 20000, (0.12, 0.08, 0.04), 0.04, 0.08, centre)
    rho = rng.uniform(0.3, 1.0, len(pts))
    ant = planar_aperture(128, 2e-3)
    x, y, z = voxel_axes(128, 2e-3, centre)
    return _finish("boxcyl128_ap128_f256", x, y, z, ant, pts, rho, 77e9, 81e9, 256, sign,
                   15.0, 1, rng, device)


def config3(sign=-1, device=None):
    """64x64 aperture @3 mm, F=128, 64^3 voxels @3 mm, config-0 sphere scene."""
    return sphere_scene(seed=0, n_ap=64, pitch=3e-3, nf=128, n_vox=64, spacing=3e-3,
                        sign=sign, device=device, name="sphere64_ap64_f128")


def config4_objects(sign=-1, device=None, count=24):
    """Uneven batch: per object seed s in 0..count-1, grid n^3 with n in {32,48,64,96},
    aperture m^2 with m in {32,64,96} at 2-4 mm pitch, F in [64,256], 500-5000 points on
    a random box/sphere/cylinder, 10-25 dB."""
    objs = []
    for s in range(count):
        rng = np.random.default_rng(1000 + s)
        n = int(rng.choice([32, 48, 64, 96]))
        m = int(rng.choice([32, 64, 96]))
        pitch = float(rng.choice([2e-3, 3e-3, 4e-3]))
        nf = int(rng.integers(64, 257))
        npts = int(rng.integers(500, 5001))
        snr = float(rng.uniform(10, 25))
        spacing = float(rng.choice([2e-3, 3e-3, 4e-3]))
        centre = (float(rng.uniform(-0.02, 0.02)), float(rng.uniform(-0.02, 0.02)),
                  float(rng.uniform(0.3, 0.5)))
        kind = int(rng.integers(0, 3))
        ext = n * spacing
        if kind == 0:
            pts = sphere_surface(rng, npts, 0.35 * ext, centre)
        elif kind == 1:
            pts = box_surface(rng, npts, (0.6 * ext, 0.5 * ext, 0.4 * ext), centre)
        else:
            pts = cylinder_surface(rng, npts, 0.3 * ext, 0.6 * ext, centre)
        rho = rng.uniform(0.3, 1.0, npts)
        ant = planar_aperture(m, pitch)
        x, y, z = voxel_axes(n, spacing, centre)
        objs.append(_finish("obj%02d" % s, x, y, z, ant, pts, rho, 77e9, 81e9, nf, sign,
                            snr, s, rng, device))
    return objs


CONFIGS = {0: config0, 1: config1, 3: config3}
