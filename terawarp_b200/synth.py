"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark workloads (no public dataset or sample volume exists for this path;
the reference ships none).

Volumes are built with torch on any device (input preparation only, never
timed); all random parameters come from numpy's seeded generator, so a given
seed gives the same landmarks and blob/fibre parameters everywhere.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def _hash_noise(torch, n: int, seed: int, hi: int, device, start: int = 0) -> "torch.Tensor":
    """Uniform integers in [0, hi] from a 32-bit integer hash of the index."""
    idx = torch.arange(start, start + n, dtype=torch.int64, device=device)
    h = (idx * 2654435761 + seed * 97531) & 0xFFFFFFFF
    h = (h ^ (h >> 15)) * 2246822519 & 0xFFFFFFFF
    h = (h ^ (h >> 13)) * 3266489917 & 0xFFFFFFFF
    h = h ^ (h >> 16)
    return (h % (hi + 1)).to(torch.float32)


def blob_volume(shape_zyx, dtype: str, seed: int, n_blobs: int | None = None, sigma=(2.0, 8.0), peak=None,
                noise: int = 10, n_fibres: int = 0, fibre_len: int = 400, fibre_value=None, device="cpu",
                z_range=None):
    """Sum of seeded 3-D Gaussian blobs, clamped to the type's range, plus
    uniform integer noise and optional 1-voxel-wide random-walk fibres.
    Returns a torch tensor (z, y, x) of dtype uint8 or uint16.

    The result is the same bytes on every device: the Gaussian factors are
    computed on the host in numpy and only multiplied and summed (exactly
    rounded float32 operations, in the same order) on the device.  With
    z_range = (z0, z1) only planes z0..z1-1 of the volume of shape_zyx are
    made (identical to those planes of the whole volume)."""
    import torch
    Z, Y, X = (int(v) for v in shape_zyx)
    zr0, zr1 = (0, Z) if z_range is None else (int(z_range[0]), int(z_range[1]))
    if not 0 <= zr0 < zr1 <= Z:
        raise ValueError(f"z_range {z_range} outside the volume's {Z} planes")
    rng = np.random.default_rng(seed)
    vmax = 255 if dtype == "u8" else 4095
    if peak is None:
        peak = (40.0, 255.0) if dtype == "u8" else (400.0, 4095.0)
    if n_blobs is None:
        n_blobs = max(1, int(200 * (X * Y * Z) / (256 * 256 * 128)))
    NZ = zr1 - zr0
    vol = torch.empty((NZ, Y, X), dtype=torch.float32, device=device)
    step = max(1, (1 << 26) // (X * Y))  # noise in chunks of ~64 M voxels
    for z0 in range(zr0, zr1, step):
        z1 = min(zr1, z0 + step)
        n0 = z0 * X * Y
        vol[z0 - zr0:z1 - zr0] = _hash_noise(torch, (z1 - z0) * X * Y, seed, noise, device, n0).reshape(
            z1 - z0, Y, X)
    cen = rng.uniform([0, 0, 0], [X, Y, Z], size=(n_blobs, 3))
    sig = rng.uniform(sigma[0], sigma[1], size=n_blobs)
    pk = rng.uniform(peak[0], peak[1], size=n_blobs)

    def gauss(lo, hi, c, inv):
        t = np.arange(lo, hi, dtype=np.float32) - np.float32(c)
        return torch.as_tensor(np.exp((t * t).astype(np.float64) * inv).astype(np.float32), device=device)

    for (cx, cy, cz), s, p in zip(cen, sig, pk):
        r = int(math.ceil(3 * s))
        x0, x1 = max(0, int(cx) - r), min(X, int(cx) + r + 1)
        y0, y1 = max(0, int(cy) - r), min(Y, int(cy) + r + 1)
        z0, z1 = max(zr0, int(cz) - r), min(zr1, int(cz) + r + 1)
        if x0 >= x1 or y0 >= y1 or z0 >= z1:
            continue
        inv = -0.5 / (s * s)
        g = (gauss(z0, z1, cz, inv)[:, None, None] * gauss(y0, y1, cy, inv)[None, :, None]
             * gauss(x0, x1, cx, inv)[None, None, :])
        vol[z0 - zr0:z1 - zr0, y0:y1, x0:x1] += float(p) * g
    if n_fibres > 0:
        fv = fibre_value or ((200, 255) if dtype == "u8" else (2500, 4095))
        start = rng.uniform([0, 0, 0], [X, Y, Z], size=(n_fibres, 1, 3))
        d0 = rng.normal(size=(n_fibres, 1, 3))
        d0 /= np.linalg.norm(d0, axis=-1, keepdims=True)
        steps = d0 + 0.35 * rng.normal(size=(n_fibres, fibre_len, 3))
        steps /= np.linalg.norm(steps, axis=-1, keepdims=True)
        pts = np.rint(start + np.cumsum(steps, axis=1)).astype(np.int64).reshape(-1, 3)
        ok = (pts[:, 0] >= 0) & (pts[:, 0] < X) & (pts[:, 1] >= 0) & (pts[:, 1] < Y) & (pts[:, 2] >= 0) & (pts[:, 2] < Z)
        pts = pts[ok]
        vals = rng.uniform(fv[0], fv[1], size=len(pts)).astype(np.float32)
        inz = (pts[:, 2] >= zr0) & (pts[:, 2] < zr1)
        pts, vals = pts[inz], vals[inz]
        lin = torch.as_tensor((pts[:, 2] - zr0) * Y * X + pts[:, 1] * X + pts[:, 0], device=device)
        flat = vol.view(-1)
        flat.index_put_((lin,), torch.as_tensor(vals, device=device))
    out = torch.empty((NZ, Y, X), dtype=torch.uint8 if dtype == "u8" else torch.uint16, device=device)
    for z0 in range(0, NZ, step):
        z1 = min(NZ, z0 + step)
        out[z0:z1] = vol[z0:z1].clamp_(0, vmax).round_().to(torch.int32).to(out.dtype)
    return out


def jitter_landmarks(sz_xyz, n: int, seed: int, margin: float = 16.0, sigma: float = 3.0):
    """Subject points uniform in the interior; target = subject + N(0, sigma)
    per axis.  Returns (subject, target) as (n, 3) float32 x, y, z."""
    rng = np.random.default_rng(seed)
    margin = min(margin, min(sz_xyz) / 4.0)
    lo = np.array([margin] * 3)
    hi = np.array(sz_xyz, dtype=np.float64) - 1 - margin
    sub = rng.uniform(lo, hi, size=(n, 3))
    tar = sub + rng.normal(0.0, sigma, size=(n, 3))
    return sub.astype(np.float32), tar.astype(np.float32)


def smooth_displacement(sz_xyz, seed: int, amplitude: float = 12.0, waves: int = 8):
    """A smooth random displacement field: sum of `waves` random-phase
    sinusoids with total amplitude <= `amplitude` voxels per axis."""
    rng = np.random.default_rng(seed)
    L = np.array(sz_xyz, dtype=np.float64)
    # wave vector k[w, a] (1-2 periods across the volume) for output axis a
    k = rng.uniform(0.5, 2.0, size=(waves, 3, 3)) * rng.choice([-1, 1], size=(waves, 3, 3)) * (2 * np.pi / L)
    ph = rng.uniform(0, 2 * np.pi, size=(waves, 3))
    amp = rng.dirichlet(np.ones(waves), size=3).T * amplitude  # (waves, 3), sums to amplitude per axis

    def f(p):
        p = np.asarray(p, np.float64)
        out = np.zeros_like(p)
        for w in range(waves):
            arg = p @ k[w].T + ph[w][None, :]   # (n, 3): one phase per output axis
            out += amp[w][None, :] * np.sin(arg)
        return out
    return f


def lattice_landmarks(sz_xyz, n: int, seed: int, amplitude: float = 12.0, noise: float = 1.0, margin: float = 8.0):
    """Subjects on a jittered lattice, targets = subjects + smooth random
    displacement + N(0, noise).  Returns (subject, target) float32 (n, 3)."""
    rng = np.random.default_rng(seed)
    L = np.array(sz_xyz, dtype=np.float64)
    per = max(2, int(round((n * L[0] * L[0] / (L[1] * L[2])) ** (1 / 3))))
    counts = np.maximum(2, np.round(per * L / L[0]).astype(int))
    while np.prod(counts) < n:
        counts += 1
    axes = [np.linspace(margin, L[a] - 1 - margin, counts[a]) for a in range(3)]
    grid = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
    pick = rng.choice(len(grid), size=n, replace=False)
    spacing = (L - 2 * margin) / counts
    sub = grid[pick] + rng.uniform(-0.3, 0.3, size=(n, 3)) * spacing
    sub = np.clip(sub, margin, L - 1 - margin)
    disp = smooth_displacement(sz_xyz, seed + 1, amplitude)
    tar = sub + disp(sub) + rng.normal(0, noise, size=(n, 3))
    return sub.astype(np.float32), tar.astype(np.float32)


def random_affine(seed: int, sz_xyz, rot_deg=15.0, scale=(0.9, 1.1), trans=20.0):
    """4x4 map (target -> subject) with rotation U(-rot, rot) per axis, scale
    U(scale) per axis and translation U(-trans, trans), about the centre."""
    rng = np.random.default_rng(seed)
    a = np.deg2rad(rng.uniform(-rot_deg, rot_deg, size=3))
    s = rng.uniform(scale[0], scale[1], size=3)
    t = rng.uniform(-trans, trans, size=3)
    cx, cy, cz = np.cos(a)
    sx, sy, sz = np.sin(a)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    A = Rz @ Ry @ Rx @ np.diag(s)
    c = (np.array(sz_xyz, np.float64) - 1) / 2
    M = np.eye(4)
    M[:3, :3] = A
    M[:3, 3] = c - A @ c + t
    return M


def affine_landmarks(M, sz_xyz, n: int, seed: int, noise: float = 0.5, margin: float = 16.0):
    """Target points uniform in the interior; subject = M target + N(0, noise)."""
    rng = np.random.default_rng(seed)
    L = np.array(sz_xyz, np.float64)
    tar = rng.uniform(margin, L - 1 - margin, size=(n, 3))
    sub = tar @ M[:3, :3].T + M[:3, 3] + rng.normal(0, noise, size=(n, 3))
    return sub.astype(np.float32), tar.astype(np.float32)


@dataclass
class JobSpec:
    kind: str            # "affine", "rigid" (rotation + translation) or "tps"
    dtype: str           # "u8" or "u16"
    shape_zyx: tuple
    M: np.ndarray | None = None
    centres: np.ndarray | None = None   # TPS centres (target-image landmarks)
    values: np.ndarray | None = None    # TPS values (subject-image landmarks)
    g: int = 16
    arrival_s: float = 0.0


def serving_jobs(n: int, seed: int = 1239, rate_hz: float = 20.0, dims_lo=(128, 128, 128),
                 dims_hi=(1024, 1024, 256), n_lo: int = 16, n_hi: int = 4096, g: int = 16):
    """The serving mix: Poisson arrivals at `rate_hz`, dims log-uniform per
    axis between dims_lo and dims_hi (x, y, z), uint8/uint16 50/50, 30%
    affine / 10% rotation+translation / 60% TPS with log-uniform landmark
    counts and the smooth sinusoidal displacement model."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for i in range(n):
        t += rng.exponential(1.0 / rate_hz)
        X, Y, Z = (int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))))) for lo, hi in zip(dims_lo, dims_hi))
        dtype = "u8" if rng.random() < 0.5 else "u16"
        u = rng.random()
        if u < 0.3:
            M = random_affine(int(rng.integers(1 << 30)), (X, Y, Z))
            jobs.append(JobSpec("affine", dtype, (Z, Y, X), M=M, arrival_s=t))
        elif u < 0.4:
            # rotation (up to 30 degrees per axis) about the centre + translation
            M = random_affine(int(rng.integers(1 << 30)), (X, Y, Z), rot_deg=30.0, scale=(1.0, 1.0), trans=20.0)
            jobs.append(JobSpec("rigid", dtype, (Z, Y, X), M=M, arrival_s=t))
        else:
            nl = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
            sub, tar = lattice_landmarks((X, Y, Z), nl, int(rng.integers(1 << 30)), margin=min(8.0, min(X, Y, Z) / 8))
            jobs.append(JobSpec("tps", dtype, (Z, Y, X), centres=tar, values=sub, g=g, arrival_s=t))
    return jobs


@dataclass
class Case:
    name: str
    vol: object          # torch tensor (z, y, x)
    marker_sub: np.ndarray
    marker_tar: np.ndarray
    g: int = 16
    M: np.ndarray | None = None


def plain_tps_case(seed: int = 1235, device="cpu", shape_zyx=(128, 256, 256), n: int = 64, g: int = 16) -> Case:
    """Plain TPS warp: 256x256x128 uint8, 200 blobs (sigma 2-8, peak 40-255)
    plus noise 0-10, 64 landmark pairs with N(0, 3) jitter, spacing 16."""
    Z, Y, X = shape_zyx
    vol = blob_volume(shape_zyx, "u8", seed, n_blobs=200 if shape_zyx == (128, 256, 256) else None, device=device)
    sub, tar = jitter_landmarks((X, Y, Z), n, seed + 7)
    return Case("plain_tps_256x256x128_u8", vol, sub, tar, g)


def large_tps_case(seed: int = 1237, device="cpu", shape_zyx=(1024, 2048, 2048), n: int = 2000, g: int = 16,
                   n_blobs: int | None = None, n_fibres: int | None = None, z_range=None) -> Case:
    """Large TPS: uint16 blob+fibre volume (values 0-4095), landmarks on a
    jittered lattice, targets displaced by 8 random-phase sinusoids
    (amplitude <= 12) + N(0, 1).  z_range = (z0, z1) makes only those planes
    of the volume (the landmarks are those of the whole volume)."""
    Z, Y, X = shape_zyx
    vox = X * Y * Z
    if n_blobs is None:
        n_blobs = max(50, min(20000, int(200 * vox / (256 * 256 * 128))))
    if n_fibres is None:
        n_fibres = max(10, min(5000, vox // (1 << 20)))
    vol = blob_volume(shape_zyx, "u16", seed, n_blobs=n_blobs, n_fibres=n_fibres, device=device, z_range=z_range)
    sub, tar = lattice_landmarks((X, Y, Z), n, seed + 7)
    return Case(f"large_tps_{X}x{Y}x{Z}_u16_n{n}_g{g}", vol, sub, tar, g)


def affine_case(seed: int = 1236, device="cpu", shape_zyx=(512, 1024, 1024), n: int = 32) -> Case:
    """Affine warp: uint16 blob+fibre volume, 12-parameter affine fitted
    from 32 landmark pairs with N(0, 0.5) jitter."""
    Z, Y, X = shape_zyx
    vox = X * Y * Z
    vol = blob_volume(shape_zyx, "u16", seed, n_blobs=max(50, min(20000, int(200 * vox / (256 * 256 * 128)))),
                      n_fibres=max(10, min(3000, vox // (1 << 20))), device=device)
    M = random_affine(seed + 3, (X, Y, Z))
    sub, tar = affine_landmarks(M, (X, Y, Z), n, seed + 7)
    return Case(f"affine_{X}x{Y}x{Z}_u16", vol, sub, tar, 0, M)
