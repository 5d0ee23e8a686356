"""The incremental cell list equals the full generation, update for update.

updateMeshes keeps the previous update's mesh cells wherever the octree did
not change (no new leaf at or above a cell's sides, no new branch in their
subtrees) and traverses only the changed parts.  Two maps fuse the same
frames, one generating every cell at every update (FF_CELLS_FULL), one
incrementally (the default): after every update the cell lists (type, size,
origin, leaves, in order), the per-cell mesh ranges and the meshes are equal,
and the incremental map generated fewer cells than it lists once the map has
settled.  Frames arrive out of order so that the volume grows between
updates (a growth moves every cell: that update is generated in full), and
coarse leaves appear above finer existing ones.
"""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

pytestmark = pytest.mark.gpu


def _pair(**kw):
    from fastfusion_b200.fusion import CELLS_FULL, FusionMipMapCPU
    a = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact", **kw)
    b = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact", **kw)
    b.set_cell_generation(CELLS_FULL)
    return a, b


def _same_update(a, b, where):
    ca, ra = a.mesh_cells()
    cb, rb = b.mesh_cells()
    assert ca.shape == cb.shape, where
    assert np.array_equal(ca, cb), where
    assert np.array_equal(ra, rb), where
    ma, mb = a.getMeshInterleavedMarchingCubes(), b.getMeshInterleavedMarchingCubes()
    assert np.array_equal(ma.vertices.view(np.uint32), mb.vertices.view(np.uint32)), where
    assert np.array_equal(ma.colors, mb.colors), where
    assert np.array_equal(ma.faces, mb.faces), where
    sa, sb = a.stats(), b.stats()
    assert sb["mesh_cells_generated"] == sb["mesh_cells"], where
    return sa["mesh_cells_generated"], sa["mesh_cells"]


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_incremental_cells_equal_full_generation(lib_built, storage):
    from fastfusion_b200.fusion import CameraInfo
    K, frames = circle_frames(0, 76, 320, 240)
    order = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 50, 51, 52, 10, 11, 12, 60, 75, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22,
             25, 30, 35, 40, 45, 55, 65, 70]
    a, b = _pair(storage=storage)
    partial = 0
    for pos, i in enumerate(order):
        depth, bgr, R, t = frames[i]
        cam = CameraInfo(K, R, t)
        assert a.addMap(depth, cam, bgr, SCALING, MAXCAM) == b.addMap(depth, cam, bgr, SCALING, MAXCAM)
        if pos % 3 == 2:
            a.updateMeshes()
            b.updateMeshes()
            gen, total = _same_update(a, b, (pos, i))
            if gen < total:
                partial += 1
    assert a.stats()["grows"] >= 1
    assert partial >= 5, partial
    a.close()
    b.close()


def test_incremental_cells_on_the_walk(lib_built):
    """The first 120 frames of the 640x480 walk, meshing every 10th frame:
    equal lists and meshes, and once the map has settled the traversal
    produces a small part of the list."""
    import torch
    from fastfusion_b200 import scene
    from fastfusion_b200.fusion import CameraInfo
    seq = scene.room_walk_sequence(0, 1000, 640, 480)
    a, b = _pair()
    ratios, kept_top = [], []
    for k in range(120):
        R, t = seq.poses[k]
        d, c = scene.render_torch(seq.scene, R, t, 640, 480, seq.K, seq.seed, k, device="cuda")
        d16 = torch.empty((480, 640), dtype=torch.int16, device="cuda")
        d16.copy_(d)
        c = c.contiguous()
        torch.cuda.synchronize()  # the maps read the images on their own streams
        cam = CameraInfo(seq.K, R, t)
        qa = a.addMapDevice(d16.data_ptr(), c.data_ptr(), 640, 480, cam, SCALING, MAXCAM)
        qb = b.addMapDevice(d16.data_ptr(), c.data_ptr(), 640, 480, cam, SCALING, MAXCAM)
        assert qa == qb
        if k % 10 == 9:
            a.updateMeshes()
            b.updateMeshes()
            gen, total = _same_update(a, b, k)
            ratios.append(gen / max(total, 1))
            kept_top.append(a.stats()["mesh_top_kept"])
    assert min(ratios[3:]) < 0.5, ratios
    # later updates start from the kept top levels of the traversal
    assert sum(kept_top) >= 1, kept_top
    a.close()
    b.close()


def test_state_restore_regenerates_every_cell(lib_built, tmp_path):
    """After ff_set_state the next update generates every cell (the restored
    octree has no history), and the following ones are incremental again."""
    from fastfusion_b200.fusion import CameraInfo
    K, frames = circle_frames(2, 12, 320, 240)
    a, b = _pair()
    for i in range(6):
        depth, bgr, R, t = frames[i]
        cam = CameraInfo(K, R, t)
        a.addMap(depth, cam, bgr, SCALING, MAXCAM)
        b.addMap(depth, cam, bgr, SCALING, MAXCAM)
    a.updateMeshes()
    b.updateMeshes()
    _same_update(a, b, "before")
    snap = str(tmp_path / "map.npz")
    a.save_snapshot(snap)
    a.load_snapshot(snap)
    a.updateMeshes()
    b.updateMeshes()
    gen, total = _same_update(a, b, "restored")
    assert gen == total
    for i in range(6, 12):
        depth, bgr, R, t = frames[i]
        cam = CameraInfo(K, R, t)
        a.addMap(depth, cam, bgr, SCALING, MAXCAM)
        b.addMap(depth, cam, bgr, SCALING, MAXCAM)
        a.updateMeshes()
        b.updateMeshes()
        _same_update(a, b, i)
    a.close()
    b.close()


def test_kept_top_levels_when_nothing_is_created_near_the_root(lib_built):
    """Frames that add no branch or leaf near the root (the same views again):
    the update starts from the kept top-level items and still equals the
    full generation; a frame of a new area brings the top levels back."""
    from fastfusion_b200.fusion import CameraInfo
    K, frames = circle_frames(4, 40, 320, 240)
    a, b = _pair()
    seen = []
    for block in ([0, 1, 2], [0, 1, 2], [1, 2, 0], [30, 35], [0, 1]):
        for i in block:
            depth, bgr, R, t = frames[i]
            cam = CameraInfo(K, R, t)
            a.addMap(depth, cam, bgr, SCALING, MAXCAM)
            b.addMap(depth, cam, bgr, SCALING, MAXCAM)
        a.updateMeshes()
        b.updateMeshes()
        _same_update(a, b, block)
        seen.append(a.stats()["mesh_top_kept"])
    assert seen[0] == 0          # the first update generates everything
    assert seen[1] == 1 and seen[2] == 1, seen
    a.close()
    b.close()
