"""Failure detection on the GPU without a GPU fault.

Every device-side wait of the fusion path is bounded.  These tests make a
wait run out on purpose -- a spin limit of zero, so a grid barrier of the
de-duplication or of the mesh-cell traversal gives up at its first poll --
or inject, from the host, the
error word the confidence network sets when one of its waits gives up.  No
kernel faults, traps or hangs: a wait that runs out sets a flag and returns.
Each test checks that the call reports FF_ERR_TIMEOUT with a message, that
the map is left in the state the error path documents, and that the same
handle then fuses the following frames bit-exactly against the oracle.
"""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames, queue_set, tree_shape

pytestmark = pytest.mark.gpu


def _pair(port_lib):
    from fastfusion_b200.fusion import FusionMipMapCPU
    g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488, update_mode=1)
    return g, p


def _cam(K, R, t):
    from fastfusion_b200.fusion import CameraInfo
    return CameraInfo(K, R, t)


def _same_map(g, p):
    sg, sp = g.stats(), p.state()
    assert (sg["n"], sg["leaves_used"]) == (sp["n"], sp["leaves_used"])
    for a, b in zip(g.leaves(), p.leaves()):
        assert np.array_equal(a, b)
    assert tree_shape(g.tree()) == tree_shape(p.tree())
    dg, wg, cg = g.bricks()
    dp, wp, cp = p.bricks()
    assert np.array_equal(dg.view(np.uint32), dp.view(np.uint32))
    assert np.array_equal(wg.view(np.uint32), wp.view(np.uint32))
    assert np.array_equal(cg, cp)


def test_mesh_traversal_wait_runs_out_and_next_update_recovers(lib_built):
    """Spin limit 0 during updateMeshes: a grid barrier of the mesh-cell
    traversal gives up, the call returns FF_ERR_TIMEOUT and nothing of that
    update is used; at the default limit the same handle's next updates give
    the cells and mesh of a map that never failed."""
    from fastfusion_b200.fusion import FFError, FusionMipMapCPU, SPIN_LIMIT_DEFAULT
    K, frames = circle_frames(1, 12, 320, 240)
    a = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    b = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")

    def fuse(ks):
        for k in ks:
            depth, bgr, R, t = frames[k]
            assert a.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == b.addMap(depth, _cam(K, R, t), bgr,
                                                                                     SCALING, MAXCAM)

    def same():
        ca, ra = a.mesh_cells()
        cb, rb = b.mesh_cells()
        assert np.array_equal(ca, cb) and np.array_equal(ra, rb)
        ma, mb = a.getMeshInterleavedMarchingCubes(), b.getMeshInterleavedMarchingCubes()
        assert len(ma.faces) > 0
        assert np.array_equal(ma.vertices.view(np.uint32), mb.vertices.view(np.uint32))
        assert np.array_equal(ma.colors, mb.colors) and np.array_equal(ma.faces, mb.faces)

    fuse(range(0, 4))
    assert a.updateMeshes() and b.updateMeshes()
    same()
    fuse(range(4, 8))
    a.set_spin_limit(0)
    with pytest.raises(FFError) as e:
        a.updateMeshes()
    assert e.value.status == 5 and "gave up" in str(e.value)
    a.set_spin_limit(SPIN_LIMIT_DEFAULT)
    assert a.updateMeshes() and b.updateMeshes()
    same()
    fuse(range(8, 12))
    assert a.updateMeshes() and b.updateMeshes()
    same()
    a.close()
    b.close()


def test_dedupe_wait_runs_out_and_map_recovers(lib_built, port_lib):
    """Spin limit 0: a de-duplication grid barrier gives up, the call returns
    FF_ERR_TIMEOUT and the frame is left out (map unchanged); at the default
    limit the next frames fuse exactly as the oracle fuses the sequence
    without the dropped frame."""
    from fastfusion_b200.fusion import FF_OK, FFError, SPIN_LIMIT_DEFAULT
    K, frames = circle_frames(0, 6, 160, 120)
    g, p = _pair(port_lib)
    for k in (0, 1):
        depth, bgr, R, t = frames[k]
        assert g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    before = g.stats()
    tree_before = g.tree()
    g.set_spin_limit(0)
    depth, bgr, R, t = frames[2]
    with pytest.raises(FFError) as e:
        g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM)
    assert e.value.status == 5 and "gave up" in str(e.value)
    after = g.stats()
    assert (after["frames"], after["leaves_used"], after["branches_used"]) == \
        (before["frames"], before["leaves_used"], before["branches_used"])
    assert np.array_equal(g.tree(), tree_before)
    g.set_spin_limit(SPIN_LIMIT_DEFAULT)
    for k in (3, 4, 5):
        depth, bgr, R, t = frames[k]
        assert g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        assert queue_set(g.queue()) == queue_set(p.queue())
    _same_map(g, p)
    # meshing works on the recovered map
    assert g.updateMeshes()
    assert len(g.getMeshInterleavedMarchingCubes().faces) > 0
    assert g._L.ff_sync(g._h) == FF_OK
    g.close()


@pytest.mark.parametrize("learned", [False, True])
def test_confidence_timeout_is_reported_and_bookkept(lib_built, port_lib, learned):
    """An injected confidence-network timeout: the frame's bricks are
    allocated (leaf table, octree and counts advance as the oracle's) but its
    voxel update is skipped; the call returns FF_ERR_TIMEOUT; the next frames
    fuse bit-exactly (no leaf index is handed out twice)."""
    from fastfusion_b200.fusion import FFError
    K, frames = circle_frames(1, 6, 160, 120)
    g, p = _pair(port_lib)
    if learned:
        # a network whose confidence is 1 everywhere (output bias far below
        # zero): the fused values equal the plain weight's, so the oracle
        # needs no confidence map
        from fastfusion_b200.fusion import load_library  # noqa: F401
        params = np.zeros(8833, np.float32)
        params[-1] = -100.0
        g.set_confidence(params, tau_m=0.02)
    for k in (0, 1):
        depth, bgr, R, t = frames[k]
        assert g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    _same_map(g, p)
    n0 = p.state()["leaves_used"]
    d0, w0, c0 = p.bricks()
    g.inject_error()
    depth, bgr, R, t = frames[2]
    with pytest.raises(FFError) as e:
        g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM)
    assert e.value.status == 5 and "confidence network" in str(e.value)
    p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    # the oracle's state with that frame's voxel update undone: old bricks as
    # before it, its new bricks at their initial zero
    n1 = p.state()["leaves_used"]
    assert n1 > n0
    pad = n1 - n0
    p.set_bricks(np.concatenate([d0, np.zeros((pad, 512), np.float32)]),
                 np.concatenate([w0, np.zeros((pad, 512), np.float32)]),
                 np.concatenate([c0, np.zeros((pad, 512, 3), np.uint16)]))
    assert g.stats()["frames"] == p.state()["frames"]
    _same_map(g, p)
    for k in (3, 4, 5):
        depth, bgr, R, t = frames[k]
        assert g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    _same_map(g, p)
    g.close()
