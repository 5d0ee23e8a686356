"""The large-map workload's generator (CPU): the corridor/office floor, the
spline path's clearance, and per-frame culling leaving every depth below
maxcam unchanged."""
import numpy as np

from fastfusion_b200 import scene


def test_corridor_layout_and_path():
    seq = scene.corridor_sequence(0, n_frames=10000, width=320, height=240)
    sc = seq.scene
    assert len(sc.box_lo) + len(sc.sph_c) - 58 == 400  # 58 walls, 400 primitives
    assert np.allclose(seq.K, [262.5, 262.5, 159.5, 119.5])
    pos = np.array([p[1] for p in seq.poses])
    assert len(pos) == 10000
    assert pos[:, 2].min() >= 0.95 and pos[:, 2].max() <= 1.65
    assert pos[:, 0].min() >= 1.9 and pos[:, 0].max() <= 48.1
    # the camera never comes within 0.3 m of a surface
    assert scene.Scene.sdf(sc, pos[::25]).min() > 0.3
    steps = np.linalg.norm(np.diff(pos, axis=0), axis=1)
    assert steps.max() < 0.01
    for R, _ in seq.poses[::997]:
        assert np.allclose(R.T @ R, np.eye(3), atol=1e-12)


def test_culling_keeps_depths_below_maxcam():
    import torch
    seq = scene.corridor_sequence(1, n_frames=10000, width=96, height=72)
    for k in (0, 2500, 7300):
        R, t = seq.poses[k]
        d0, c0 = scene.render_torch(seq.scene, R, t, 96, 72, seq.K, 1, k, device="cpu")
        d1, c1 = scene.render_torch(seq.scene, R, t, 96, 72, seq.K, 1, k, device="cpu", cull_m=5.0)
        z0 = (d0.numpy().astype(np.int32) & 0xFFFF) / 5000.0
        z1 = (d1.numpy().astype(np.int32) & 0xFFFF) / 5000.0
        near = (z0 > 0) & (z0 < 4.0)
        assert near.mean() > 0.3
        assert np.array_equal(z0[near], z1[near])
        assert np.array_equal(c0.numpy()[near], c1.numpy()[near])
