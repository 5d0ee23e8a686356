"""Batched fusion of several independent maps (ff_add_maps_u16_device): one
set of launches for the frames of all maps must give every map exactly what
fusing its frames alone gives -- leaf tables, queued bricks, voxel bits and
meshes -- including a map whose volume grows (frames taken out of order so
that later frames fall outside the first frame's volume) and maps of
different image sizes."""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames, queue_set

pytestmark = pytest.mark.gpu


def _maps(n, **kw):
    from fastfusion_b200.fusion import FusionMipMapCPU
    return [FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact",
                            **kw) for _ in range(n)]


# launch shapes (ff_tuning) must not change any result: default; the other
# tile height, two bricks per block, a small grid, wide insert blocks and a
# replayed CUDA graph
TUNINGS = {"default": {}, "tuned": dict(dedupe_rows=32, fuse_shape=2, fuse_blocks_per_sm=2, insert_block=512,
                                        graph=True),
           "graph": dict(fuse_shape=1, graph=True),
           "low": dict(dedupe_rows=8, fuse_shape=3)}


@pytest.mark.parametrize("storage,tuning", [("fp32", "default"), ("fp16", "default"), ("fp32", "tuned"),
                                            ("fp16", "graph"), ("fp32", "low")])
def test_batch_equals_one_by_one(lib_built, storage, tuning):
    import torch
    from fastfusion_b200.fusion import CameraInfo, add_maps_device
    seqs = []
    K0, f0 = circle_frames(0, 76, 160, 120)
    seqs.append((K0, [f0[i] for i in (50, 60, 75, 0, 10, 25)], 160, 120))
    K1, f1 = circle_frames(1, 6, 320, 240)
    seqs.append((K1, f1, 320, 240))
    K2, f2 = circle_frames(2, 6, 160, 120)
    seqs.append((K2, f2, 160, 120))
    batched = _maps(len(seqs), storage=storage)
    alone = _maps(len(seqs), storage=storage)
    batched[0].set_tuning(**TUNINGS[tuning])
    for k in range(6):
        dd, db, cams, keep = [], [], [], []
        for K, frames, w, h in seqs:
            depth, bgr, R, t = frames[k]
            td = torch.from_numpy(depth.view(np.int16).copy()).cuda()
            tb = torch.from_numpy(bgr.copy()).cuda()
            keep += [td, tb]
            dd.append(td.data_ptr())
            db.append(tb.data_ptr())
            cams.append(CameraInfo(K, R, t))
        torch.cuda.synchronize()
        qb = add_maps_device(batched, dd, db, [s[2] for s in seqs], [s[3] for s in seqs], cams, SCALING, MAXCAM)
        for i, m in enumerate(alone):
            qa = m.addMapDevice(dd[i], db[i], seqs[i][2], seqs[i][3], cams[i], SCALING, MAXCAM)
            assert qa == qb[i], (k, i)
            assert queue_set(m.queue()) == queue_set(batched[i].queue())
    assert batched[0].stats()["grows"] >= 1
    if TUNINGS[tuning].get("graph"):
        # the batch's launches (cooperative de-duplication included) were recorded and replayed
        assert batched[0].stats()["graph_replays"] == 6
    for a, b in zip(alone, batched):
        sa, sb = a.stats(), b.stats()
        assert sa["n"] == sb["n"] and np.array_equal(sa["offset"], sb["offset"])
        for x, y in zip(a.leaves(), b.leaves()):
            assert np.array_equal(x, y)
        for x, y in zip(a.bricks(), b.bricks()):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
        a.updateMeshes()
        b.updateMeshes()
        ma, mb = a.getMeshInterleavedMarchingCubes(), b.getMeshInterleavedMarchingCubes()
        assert len(ma.faces) > 0
        assert np.array_equal(ma.vertices.view(np.uint32), mb.vertices.view(np.uint32))
        assert np.array_equal(ma.faces, mb.faces)


def test_batch_rejects_bad_input(lib_built):
    from fastfusion_b200.fusion import CameraInfo, FFError, add_maps_device
    a, b = _maps(2)
    cam = CameraInfo((525.0, 525.0, 80.0, 60.0), np.eye(3), np.zeros(3))
    with pytest.raises(FFError):
        add_maps_device([a, a], [1, 1], [1, 1], [160, 160], [120, 120], [cam, cam], SCALING, MAXCAM)
    c = _maps(1, storage="fp16")[0]
    with pytest.raises(FFError):
        add_maps_device([a, c], [1, 1], [1, 1], [160, 160], [120, 120], [cam, cam], SCALING, MAXCAM)


def test_batch_with_learned_weight(lib_built):
    """The learned confidence weight in a batched call equals the same weight
    map by map (every map runs its own network on its frame)."""
    import torch
    from fastfusion_b200.confidence import load_weights
    from fastfusion_b200.fusion import CameraInfo, add_maps_device
    params, tau = load_weights()
    K0, f0 = circle_frames(0, 6, 160, 120)
    K1, f1 = circle_frames(1, 6, 320, 240)
    seqs = [(K0, f0, 160, 120), (K1, f1, 320, 240)]
    batched, alone = _maps(2), _maps(2)
    for m in batched + alone:
        m.set_confidence(params, tau)
    for k in range(6):
        dd, db, cams, keep = [], [], [], []
        for K, frames, w, h in seqs:
            depth, bgr, R, t = frames[k]
            td = torch.from_numpy(depth.view(np.int16).copy()).cuda()
            tb = torch.from_numpy(bgr.copy()).cuda()
            keep += [td, tb]
            dd.append(td.data_ptr())
            db.append(tb.data_ptr())
            cams.append(CameraInfo(K, R, t))
        torch.cuda.synchronize()
        qb = add_maps_device(batched, dd, db, [s[2] for s in seqs], [s[3] for s in seqs], cams, SCALING, MAXCAM)
        for i, m in enumerate(alone):
            assert m.addMapDevice(dd[i], db[i], seqs[i][2], seqs[i][3], cams[i], SCALING, MAXCAM) == qb[i]
            m.sync()
    for a, b in zip(alone, batched):
        for x, y in zip(a.bricks(), b.bricks()):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
        assert np.array_equal(a.confidence_map(), b.confidence_map())
