"""Brick-ownership sharding of one map (ff_set_shard): three parts fed the
same frames hold disjoint bricks that together are exactly the whole map's,
voxel for voxel, with the whole map's queued counts -- including frames out
of order that make the volume grow (the ownership key does not move with
growth).  The parts run as separate maps on one GPU."""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

pytestmark = pytest.mark.gpu

SHARDS = 3


def _map(**kw):
    from fastfusion_b200.fusion import FusionMipMapCPU
    return FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact",
                           **kw)


def _bricks(m):
    """{(x, y, z, scale): (sdf bits, weight bits, colour)} of a map."""
    pos, scale, _ = m.leaves()
    d, w, c = m.bricks()
    return {(int(p[0]), int(p[1]), int(p[2]), int(s)): (d[i].view(np.uint32).tobytes(), w[i].view(np.uint32).tobytes(),
                                                       c[i].tobytes())
            for i, (p, s) in enumerate(zip(pos, scale))}


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_shards_together_are_the_whole_map(lib_built, storage):
    from fastfusion_b200.fusion import CameraInfo
    K, frames = circle_frames(0, 76, 320, 240)
    order = [50, 60, 75, 0, 10, 25, 40]  # later frames outside the first frame's volume: growth
    whole = _map(storage=storage)
    parts = [_map(storage=storage) for _ in range(SHARDS)]
    for k, p in enumerate(parts):
        p.set_shard(k, SHARDS)
    for i in order:
        depth, bgr, R, t = frames[i]
        cam = CameraInfo(K, R, t)
        q = whole.addMap(depth, cam, bgr, SCALING, MAXCAM)
        qs = [p.addMap(depth, cam, bgr, SCALING, MAXCAM) for p in parts]
        assert sum(qs) == q, (i, q, qs)
    assert whole.stats()["grows"] >= 1
    for p in parts:
        assert p.stats()["grows"] == whole.stats()["grows"]
        assert np.array_equal(p.stats()["offset"], whole.stats()["offset"])
    full = _bricks(whole)
    got = {}
    for p in parts:
        b = _bricks(p)
        assert not (set(b) & set(got)), "a brick in two parts"
        assert 0.15 * len(full) < len(b) < 0.55 * len(full)
        got.update(b)
    assert set(got) == set(full)
    for key, val in full.items():
        assert got[key] == val, key
    with pytest.raises(Exception):
        parts[0].set_shard(1, SHARDS)  # only before the first frame
