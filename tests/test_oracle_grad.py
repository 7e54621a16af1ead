"""The FP64 oracle of the differentiable HQS colours pinned against itself:
its central differences (step 1e-3) agree with its analytic adjoint.

The loss is quadratic in the colours (the visible sets do not depend on
them), so central differences are exact up to FP64 rounding.
"""
import numpy as np

from scenes import blob_cloud


def _camera(pos, target=(0.0, 0.0, 0.0), aspect=1.0, near=0.01, far=100.0, fov=60.0):
    """Right-handed view and reverse-Z projection (column-major float32[16])."""
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


def test_oracle_central_differences_match_adjoint(orc):
    pos, rgba = blob_cloud(4000, 21)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=512)
    cloud = packed.cloud()
    cfg = orc.Config()
    rng = np.random.default_rng(3)
    n = len(cloud.colors)
    colors = rng.uniform(0.0, 1.0, (n, 3))
    grad = np.zeros((n, 3))
    fd = None
    w = h = 48
    for k, eye in enumerate([(0.0, 0.0, 2.5), (1.5, 0.8, 1.8)]):
        view, proj = _camera(eye)
        cloud.files = orc.update_files(packed.files, orc.mat4_mul(proj, view),
                                       np.eye(4, dtype=np.float32))
        target = rng.uniform(0.0, 1.0, (h, w, 3))
        pts = np.arange(0, n, 7, dtype=np.uint32)
        out = orc.hqs_grad_f64(cloud, cfg, view, proj, w, h, colors, target, 1.0 / (w * h * 3),
                               grad=grad, fd_points=pts, fd_h=1e-3, fd=fd)
        fd = out["fd"]
    sel = grad[pts]
    assert np.abs(sel).max() > 0
    assert np.allclose(fd, sel, rtol=1e-9, atol=1e-12 * np.abs(sel).max())
