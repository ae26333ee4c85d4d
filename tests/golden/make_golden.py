"""Generates the golden fixtures in this folder with an implementation that is
independent of oracle/tw_oracle.c: numpy/scipy, the bordered (N+4)^2 TPS
system instead of the projected one, separable B-spline weights instead of
the n^3 x 64 Kronecker basis, and a vectorised trilinear sampler.  Both
restate the reference's arithmetic (q_imgwarp_tps_quicksmallmemory.cpp:85-203,
:377-699; q_warp_affine_tps.cpp:649-731, :1373-1437); agreement between them
pins the oracle's transcription.  The reference itself ships no fixtures and
cannot be built here, so these are not outputs of the reference.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def tps_bordered(ctr, val, lam=0.2):
    ctr = ctr.astype(np.float64)
    n = len(ctr)
    K = -np.sqrt(((ctr[:, None, :] - ctr[None, :, :]) ** 2).sum(-1))
    X = np.hstack([np.ones((n, 1)), ctr])
    Y = np.hstack([np.ones((n, 1)), val.astype(np.float64)])
    A = np.zeros((n + 4, n + 4))
    A[:n, :n] = K + lam * np.eye(n)
    A[:n, n:] = X
    A[n:, :n] = X.T
    sol = np.linalg.solve(A, np.vstack([Y, np.zeros((4, 4))]))
    return sol[:n], sol[n:]


def grid_size(sz, g):
    return int(np.ceil(sz / g)) + 3


def tps_grid(ctr, c, d, gsz, g):
    gx, gy, gz = gsz
    k, j, i = np.meshgrid(np.arange(gz), np.arange(gy), np.arange(gx), indexing="ij")
    p = np.stack([(i - 1) * g, (j - 1) * g, (k - 1) * g], -1).astype(np.float64).reshape(-1, 3)
    r = -np.sqrt(((p[:, None, :] - ctr.astype(np.float64)[None, :, :]) ** 2).sum(-1))
    f = np.hstack([np.ones((len(p), 1)), p]) @ d + r @ c
    return (f[:, 1:] - p).astype(np.float32).reshape(gz, gy, gx, 3)


def bspline_w(t):
    return np.stack([(1 - t) ** 3, 3 * t ** 3 - 6 * t ** 2 + 4, -3 * t ** 3 + 3 * t ** 2 + 3 * t + 1, t ** 3], -1) / 6.0


def voxel_df(df, g, shape_zyx):
    Z, Y, X = shape_zyx
    out = np.zeros((Z, Y, X, 3), np.float64)
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    cz, cy, cx = z // g, y // g, x // g
    wz, wy, wx = bspline_w((z % g) / g), bspline_w((y % g) / g), bspline_w((x % g) / g)
    for a in range(4):
        for b in range(4):
            for e in range(4):
                w = (wz[..., a] * wx[..., e] * wy[..., b])[..., None]
                out += w * df[cz + a, cy + b, cx + e].astype(np.float64)
    return out.astype(np.float32)


def trilinear(src, q):
    Z, Y, X = src.shape
    s = src.astype(np.float64)
    ok = (q[..., 0] >= 0) & (q[..., 0] <= X - 1) & (q[..., 1] >= 0) & (q[..., 1] <= Y - 1) & (q[..., 2] >= 0) & (q[..., 2] <= Z - 1)
    qq = np.where(ok[..., None], q, 0.0)
    f = np.floor(qq).astype(np.int64)
    c = np.ceil(qq).astype(np.int64)
    fr = qq - f
    v = np.zeros(q.shape[:-1])
    for dz in (0, 1):
        iz = c[..., 2] if dz else f[..., 2]
        wz = fr[..., 2] if dz else 1 - fr[..., 2]
        for dy in (0, 1):
            iy = c[..., 1] if dy else f[..., 1]
            wy = fr[..., 1] if dy else 1 - fr[..., 1]
            for dx in (0, 1):
                ix = c[..., 0] if dx else f[..., 0]
                wx = fr[..., 0] if dx else 1 - fr[..., 0]
                v += wz * wy * wx * s[iz, iy, ix]
    return v, ok


def tps_warp(src, df, g):
    Z, Y, X = src.shape
    dfv = voxel_df(df, g, src.shape).astype(np.float64)
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    q = np.stack([x, y, z], -1) + dfv
    v, ok = trilinear(src, q)
    return np.where(ok, np.floor(v + 0.5), 0).astype(src.dtype)


def affine_fit(tar, sub):
    def norm(p):
        c = p.mean(0)
        q = p - c
        s = 1.0 / np.sqrt((q ** 2).sum(1)).mean()
        N = np.eye(4)
        N[:3, :3] *= s
        N[:3, 3] = -s * c
        return q * s, N
    a, NA = norm(tar.astype(np.float64))
    b, NB = norm(sub.astype(np.float64))
    rows = []
    for i in range(len(a)):
        for r in range(3):
            row = np.zeros(13)
            row[4 * r:4 * r + 3] = a[i]
            row[4 * r + 3] = 1
            row[12] = -b[i, r]
            rows.append(row)
    _, _, vt = np.linalg.svd(np.array(rows))
    h = vt[-1] / vt[-1][12]
    H = np.vstack([h[:12].reshape(3, 4), [0, 0, 0, 1]])
    return np.linalg.inv(NB) @ H @ NA


def affine_warp(src, M, out_zyx):
    oz, oy, ox = out_zyx
    z, y, x = np.meshgrid(np.arange(oz), np.arange(oy), np.arange(ox), indexing="ij")
    p = np.stack([x, y, z, np.ones_like(x)], -1).astype(np.float64)
    q = p @ M.T
    v, ok = trilinear(src, q[..., :3])
    return np.where(ok, np.floor(v), 0).astype(src.dtype)


def main():
    rng = np.random.default_rng(20240601)
    out = {}
    # TPS, uint8, 36 x 30 x 22 voxels, 12 landmarks, spacings 4 and 8
    Z, Y, X = 22, 30, 36
    src8 = rng.integers(0, 256, size=(Z, Y, X), dtype=np.uint8)
    sub = rng.uniform([3, 3, 3], [X - 4, Y - 4, Z - 4], size=(12, 3)).astype(np.float32)
    tar = (sub + rng.normal(0, 1.5, size=sub.shape)).astype(np.float32)
    c, d = tps_bordered(sub, tar)
    out.update(tps_src=src8, tps_ctr=sub, tps_val=tar, tps_c=c, tps_d=d)
    for g in (4, 8):
        gsz = (grid_size(X, g), grid_size(Y, g), grid_size(Z, g))
        df = tps_grid(sub, c, d, gsz, g)
        out[f"tps_df_g{g}"] = df
        out[f"tps_out_g{g}"] = tps_warp(src8, df, g)
    # affine, uint16, 30 x 26 x 18, 10 noisy pairs, output 28 x 24 x 20
    Z2, Y2, X2 = 18, 26, 30
    src16 = rng.integers(0, 4096, size=(Z2, Y2, X2), dtype=np.uint16)
    tarA = rng.uniform(2, [X2 - 3, Y2 - 3, Z2 - 3], size=(10, 3))
    Mtrue = np.eye(4)
    Mtrue[:3, :3] += rng.normal(0, 0.05, size=(3, 3))
    Mtrue[:3, 3] = rng.uniform(-2, 2, 3)
    subA = tarA @ Mtrue[:3, :3].T + Mtrue[:3, 3] + rng.normal(0, 0.3, size=tarA.shape)
    # landmarks cross the ABI as float (Coord3D_JBA / ImageMarker): fit from the rounded values
    tarA = tarA.astype(np.float32).astype(np.float64)
    subA = subA.astype(np.float32).astype(np.float64)
    M = affine_fit(tarA, subA)
    out.update(aff_src=src16, aff_tar=tarA.astype(np.float32), aff_sub=subA.astype(np.float32), aff_M=M,
               aff_out=affine_warp(src16, M, (20, 24, 28)))
    np.savez_compressed(HERE / "golden_small.npz", **out)
    print("wrote", HERE / "golden_small.npz", sorted(out))


if __name__ == "__main__":
    main()
