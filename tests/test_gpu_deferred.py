"""The deferred voxel update at every batch size gives the reference's voxels.

`ff_set_update_batch(h, k)` lets up to k frames queue their bricks before one
pass applies them (each brick loaded once, the frames that queued it applied
in order, stored once).  The same frames -- out of order, so that the volume
grows in the middle of a batch, with mesh updates and accessors flushing a
batch part-way -- are fused at batch 1, 2, 16 and 32 and compared, bit for
bit, with the oracle after every flush point; the number of brick loads the
pass made falls as the batch grows while the frame-bricks stay the same.
"""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames, queue_set

pytestmark = pytest.mark.gpu

ORDER = [50, 60, 75, 0, 1, 2, 3, 10, 25, 40, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21]
MESH_AFTER = {3, 9, 20}   # positions in ORDER after which updateMeshes runs


def _same_map(g, p):
    sg, sp = g.stats(), p.state()
    assert (sg["n"], sg["leaves_used"]) == (sp["n"], sp["leaves_used"])
    for a, b in zip(g.leaves(), p.leaves()):
        assert np.array_equal(a, b)
    assert queue_set(g.queue()) == queue_set(p.queue())
    (dg, wg, cg), (dp, wp, cp) = g.bricks(), p.bricks()
    assert np.array_equal(dg.view(np.uint32), dp.view(np.uint32)), "SDF bits differ"
    assert np.array_equal(wg.view(np.uint32), wp.view(np.uint32)), "weight bits differ"
    assert np.array_equal(cg, cp), "colour differs"


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_batch_sizes_give_the_same_voxels(lib_built, port_lib, storage):
    from fastfusion_b200.fusion import CameraInfo, FusionMipMapCPU
    K, frames = circle_frames(0, 76, 320, 240)
    fused = {}
    for batch in (1, 2, 16, 32):
        g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact",
                            storage=storage)
        g.set_update_batch(batch)
        p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488, update_mode=1,
                                fp16=(storage == "fp16"))
        for pos, i in enumerate(ORDER):
            depth, bgr, R, t = frames[i]
            q = g.addMap(depth, CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
            assert q == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM), (batch, i)
            if pos in MESH_AFTER:
                g.updateMeshes()
                p.update_meshes()
                _same_map(g, p)
                mesh = g.getMeshInterleavedMarchingCubes()
                _, _, xyz, rgb, faces = p.mesh()
                assert np.array_equal(mesh.vertices.view(np.uint32), xyz.view(np.uint32)), (batch, pos)
                assert np.array_equal(mesh.faces, faces), (batch, pos)
        _same_map(g, p)
        st = g.stats()
        assert st["grows"] >= 1
        assert st["update_batch"] == batch
        fused[batch] = (st["fused_frame_bricks"], st["fused_bricks"])
        g.close()
        p.close()
    # the same frame-bricks at every batch size; fewer brick loads with larger
    # batches (a brick queued by several frames of a batch is loaded once)
    assert len({v[0] for v in fused.values()}) == 1
    assert fused[1][1] == fused[1][0]
    assert fused[32][1] <= fused[16][1] <= fused[2][1] < fused[1][1]
