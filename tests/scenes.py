"""Seeded scene builders shared by the tests (inputs only; no pass logic)."""
from __future__ import annotations

import numpy as np


def lattice_cloud(n_axis: int, seed: int, jitter: float = 0.002, lo: float = -1.0,
                  hi: float = 1.0):
    """An n^3 lattice over [lo, hi]^3 with uniform jitter and packed RGBA8 colours
    (alpha 255), the shape of the 1M-point lattice workload at small n."""
    rng = np.random.default_rng(seed)
    g = np.linspace(lo, hi, n_axis, dtype=np.float64)
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    pos = pos + rng.uniform(-jitter, jitter, pos.shape)
    rgb = rng.integers(0, 256, (len(pos), 3), dtype=np.uint32)
    rgba = rgb[:, 0] | (rgb[:, 1] << 8) | (rgb[:, 2] << 16) | (np.uint32(255) << 24)
    return pos.astype(np.float32), rgba.astype(np.uint32)


def blob_cloud(count: int, seed: int, scale: float = 1.0):
    """Clustered points (gaussian blobs in a unit box, like a scanned node)."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-0.5, 0.5, (16, 3))
    idx = rng.integers(0, len(centers), count)
    pos = centers[idx] + rng.normal(0, 0.06, (count, 3))
    rgb = rng.integers(0, 256, (count, 3), dtype=np.uint32)
    rgba = rgb[:, 0] | (rgb[:, 1] << 8) | (rgb[:, 2] << 16) | (np.uint32(255) << 24)
    return (pos * scale).astype(np.float32), rgba.astype(np.uint32)


def to_product_packed(cr, packed):
    """Oracle PackedPointCloud -> the product's PackedPointCloud (same arrays)."""
    return cr.PackedPointCloud(batches=packed.batches, files=packed.files, xyzLow=packed.xyzLow,
                               xyzMed=packed.xyzMed, xyzHigh=packed.xyzHigh,
                               colors=packed.colors, levels=packed.levels,
                               boundsMin=packed.boundsMin, boundsMax=packed.boundsMax,
                               orderedPositions=packed.orderedPositions,
                               sourceIndices=packed.sourceIndices)


def oracle_config(orc, cfg):
    """The product configuration as the oracle's pass-relevant config."""
    return orc.Config(mode=cfg.mode, depthTolerance=cfg.depthTolerance,
                      backgroundColor=tuple(cfg.backgroundColor),
                      enableFrustumCulling=cfg.enableFrustumCulling, lodBias=cfg.lodBias,
                      enableCLOD=cfg.enableCLOD, enableLODDither=cfg.enableLODDither,
                      holeFillIterations=cfg.holeFillIterations,
                      colorizeChunks=cfg.colorizeChunks, colorizeOverdraw=cfg.colorizeOverdraw,
                      pointSizeMode=cfg.pointSizeMode, minimumPointSize=cfg.minimumPointSize,
                      maximumPointSize=cfg.maximumPointSize, pointSizeScale=cfg.pointSizeScale)


def oracle_cloud_from_device(orc, cloud):
    """The oracle's view of a device slot pool, read back from the device."""
    pts = cloud.points()
    return orc.Cloud(batches=cloud.batches(), files=cloud.files(), xyzLow=pts["xyzLow"],
                     xyzMed=pts["xyzMed"], xyzHigh=pts["xyzHigh"], colors=pts["colors"],
                     levels=pts["levels"])


def look_at_reverse_z(pos, target=(0.0, 0.0, 0.0), aspect=1.0, near=0.01, far=100.0, fov=60.0):
    """Right-handed view looking from `pos` at `target` (up +Y) and a reverse-Z
    perspective projection, both column-major float32[16]."""
    p, t = np.asarray(pos, np.float64), np.asarray(target, np.float64)
    f = (t - p) / np.linalg.norm(t - p)
    s = np.cross(f, [0.0, 1.0, 0.0])
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    v = np.eye(4)
    v[0, :3], v[1, :3], v[2, :3] = s, u, -f
    v[0, 3], v[1, 3], v[2, 3] = -s @ p, -u @ p, f @ p
    k = 1.0 / np.tan(np.radians(fov) / 2)
    pr = np.zeros((4, 4))
    pr[0, 0], pr[1, 1] = k / aspect, k
    pr[2, 2], pr[2, 3], pr[3, 2] = near / (far - near), far * near / (far - near), -1.0
    return v.T.astype(np.float32).reshape(16), pr.T.astype(np.float32).reshape(16)
