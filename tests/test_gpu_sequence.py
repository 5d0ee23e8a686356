"""Several frames of one map per call (ff_add_map_sequence_u16_device): all
frames de-duplicated in one launch set, inserted and finalised frame after
frame on the device, one counter read-back, one deferred voxel-update pass.
It must give exactly what frame-by-frame fusion gives -- queued counts, leaf
table, queue, every voxel bit, and the mesh -- including a sequence in which
one frame must grow the volume (the frames after it are halted on the device
and run again in the grown volume), a sequence longer than one update batch,
and the learned weight."""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames, queue_set

pytestmark = pytest.mark.gpu


def _dev(frames):
    import torch
    out = []
    for depth, bgr, R, t in frames:
        out.append((torch.from_numpy(depth.view(np.int16).copy()).cuda(), torch.from_numpy(bgr.copy()).cuda(), R, t))
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("case", ["grow", "long", "learned"])
def test_sequence_equals_frame_by_frame(lib_built, port_lib, case):
    from fastfusion_b200.fusion import CameraInfo, FusionMipMapCPU
    K, frames = circle_frames(0, 100, 160, 120)
    if case == "grow":
        order = [[50, 60, 75, 0, 10, 25], [30, 31, 32]]   # frame 75 grows the volume
    elif case == "long":
        order = [list(range(0, 40, 2)), list(range(1, 24, 2))]  # 20 frames: more than one batch of 16
    else:
        order = [[3, 4, 5, 6, 7], [8, 9]]
    g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488, update_mode=1)
    if case == "learned":
        # a network whose confidence is 1 everywhere: the plain weight's values
        params = np.zeros(8833, np.float32)
        params[-1] = -100.0
        g.set_confidence(params, tau_m=0.02)
    for chunk in order:
        dev = _dev([frames[i] for i in chunk])
        qg = g.addMapSequenceDevice([d.data_ptr() for d, _, _, _ in dev], [c.data_ptr() for _, c, _, _ in dev], 160,
                                    120, [CameraInfo(K, R, t) for _, _, R, t in dev], SCALING, MAXCAM)
        qp = [p.add_map(frames[i][0], frames[i][1], K, frames[i][2], frames[i][3], SCALING, MAXCAM) for i in chunk]
        assert qg == qp, (chunk, qg, qp)
        assert queue_set(g.queue()) == queue_set(p.queue())
        for a, b in zip(g.leaves(), p.leaves()):
            assert np.array_equal(a, b)
        (dg, wg, cg), (dp, wp, cp) = g.bricks(), p.bricks()
        assert np.array_equal(dg.view(np.uint32), dp.view(np.uint32))
        assert np.array_equal(wg.view(np.uint32), wp.view(np.uint32))
        assert np.array_equal(cg, cp)
    if case == "grow":
        assert g.stats()["grows"] == p.state()["grows"] == 1
    assert g.stats()["frames"] == p.state()["frames"]
    g.updateMeshes()
    p.update_meshes()
    mesh = g.getMeshInterleavedMarchingCubes()
    _, _, xyz, rgb, faces = p.mesh()
    assert np.array_equal(mesh.vertices.view(np.uint32), xyz.view(np.uint32))
    assert np.array_equal(mesh.colors, rgb)
    assert np.array_equal(mesh.faces, faces)
    # single frames after a sequence continue the same map
    depth, bgr, R, t = frames[90]
    assert g.addMap(depth, CameraInfo(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING,
                                                                                    MAXCAM)
    (dg, wg, _), (dp, wp, _) = g.bricks(), p.bricks()
    assert np.array_equal(dg.view(np.uint32), dp.view(np.uint32))
    g.close()
    p.close()


def test_host_image_sequence_equals_frame_by_frame(lib_built, port_lib):
    """ff_add_map_sequence_u16 (host images, the reference's several-frames
    addMap): the same queued counts, leaf table, queue and voxels as the
    restatement fed frame by frame -- over a call of more frames than one
    group of 32 and a call that grows the volume."""
    from fastfusion_b200.fusion import CameraInfo, FusionMipMapCPU
    K, frames = circle_frames(0, 100, 160, 120)
    g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488, update_mode=1)
    # frame 75 grows the volume set by frames 50 and 60; the first call takes
    # 36 frames (two groups)
    for chunk in ([50, 60, 75, 0, 10, 25] + list(range(30, 90, 2)), [3, 5, 7]):
        qg = g.addMapSequence([frames[i][0] for i in chunk], [CameraInfo(K, frames[i][2], frames[i][3]) for i in chunk],
                              [frames[i][1] for i in chunk], SCALING, MAXCAM)
        qp = [p.add_map(frames[i][0], frames[i][1], K, frames[i][2], frames[i][3], SCALING, MAXCAM) for i in chunk]
        assert qg == qp, chunk
        assert queue_set(g.queue()) == queue_set(p.queue())
    assert g.stats()["grows"] >= 1
    for a, b in zip(g.leaves(), p.leaves()):
        assert np.array_equal(a, b)
    (dg, wg, cg), (dp, wp, cp) = g.bricks(), p.bricks()
    assert np.array_equal(dg.view(np.uint32), dp.view(np.uint32))
    assert np.array_equal(wg.view(np.uint32), wp.view(np.uint32))
    assert np.array_equal(cg, cp)
    g.close()
    p.close()
