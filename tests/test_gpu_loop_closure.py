"""Loop closure's removal of fused frames (ff_loop_*) against the compiled
reference's own deleteOldLoopPoses step (its camera set-up and
updateWrapper_deleteloop / update8AddLoopSSESingleDeleteloop, called through
oracle/ref_harness.cpp), bit for bit with the host CPU's RCPPS.

Both maps fuse the same frames (the leaf tables are identical, as the fusion
tests pin); then each frame is removed under a corrected pose (shifted by a
few millimetres and turned slightly), with the frame's float depth (NaN where
the sensor gave none) and its colour planes, over the leaves the frame
queued -- the reference's queue order, which decides the slot order.  The
loop arrays, every brick's slot and the slots in use must be equal, also
when the slots run out in the middle of a frame."""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

pytestmark = pytest.mark.gpu

BRANCHINIT = 0xFFFFFFFE


def _corrected(R, t, k):
    a = 0.002 * (k + 1)
    c, s = np.cos(a), np.sin(a)
    Rz = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    return Rz @ R, t + np.array([0.003, -0.002, 0.001]) * (k + 1)


@pytest.mark.parametrize("capacity", [100000, 700])
def test_loop_removal_matches_reference(lib_built, capacity):
    import torch
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/libffref.so not built")
    from fastfusion_b200.fusion import CameraInfo, FusionMipMapCPU
    K, frames = circle_frames(2, 6, 160, 120)
    r = ref.RefFusion()
    st = r.state()
    g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=st["leaves_total"],
                        branches_max=st["branches_total"], rcp="host")
    queues = []
    for depth, bgr, R, t in frames:
        assert g.addMap(depth, CameraInfo(K, R, t), bgr, SCALING, MAXCAM) == r.add_map(depth, bgr, K, R, t, SCALING,
                                                                                        MAXCAM)
        queues.append(r.queue().copy())
    for a, b in zip(g.leaves(), r.leaves()):
        assert np.array_equal(a, b)
    nleaves = r.state()["leaves_used"]
    # the reference side: its loop arrays in caller memory
    leaf_map = np.full(nleaves, BRANCHINIT, np.uint32)
    dist = np.zeros((capacity, 512), np.float32)
    wgt = np.zeros((capacity, 512), np.float32)
    col = np.zeros((capacity, 512, 3), np.uint16)
    n_mapped = 0
    g.loop_begin(capacity)
    done_ref, done_gpu = [], []
    for k, (depth, bgr, R, t) in enumerate(frames):
        Rc, tc = _corrected(R, t, k)
        dm = depth.astype(np.float32) * np.float32(SCALING)
        dm[depth == 0] = np.nan
        red, green, blue = (np.ascontiguousarray(bgr[:, :, c]) for c in (2, 1, 0))
        ok, n_mapped = r.loop_delete(dm, red, green, blue, K, Rc, tc, queues[k], leaf_map, n_mapped, capacity,
                                     dist, wgt, col)
        done_ref.append(ok)
        dev = [torch.from_numpy(a).cuda() for a in (dm, red, green, blue, queues[k].astype(np.uint32))]
        torch.cuda.synchronize()
        done_gpu.append(g.loop_delete_frame(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(),
                                            dev[3].data_ptr(), 160, 120, CameraInfo(K, Rc, tc), dev[4].data_ptr(),
                                            len(queues[k])))
    assert done_gpu == done_ref
    if capacity < 1000:
        assert not all(done_ref), "the small capacity must run out"
    m, d, w, c = g.loop_arrays()
    assert len(d) == n_mapped > 0
    assert np.array_equal(m, leaf_map)
    assert np.array_equal(d.view(np.uint32), dist[:n_mapped].view(np.uint32)), "loop SDF bits differ"
    assert np.array_equal(w.view(np.uint32), wgt[:n_mapped].view(np.uint32)), "loop weight bits differ"
    assert np.array_equal(c, col[:n_mapped]), "loop colour differs"
    # the fall-off's sign is turned: some weights went below zero
    assert (w < 0).any()
    g.close()
    r.close()
