"""One map split over parts (ff_set_shard), the parts run as separate maps on
one GPU and the halo records moved between them through device buffers (on
several GPUs an NCCL all-gather moves them; fastfusion_b200/shard.py).

Every part holds the whole map's octree and leaf table and returns the whole
map's queued counts; the parts' own bricks partition the map (each brick is
exported by exactly one part); after the halo exchange every part's voxels
equal the whole map's, bit for bit; and the parts' meshes together are the
whole map's mesh: every cell in every part's cell list, each cell meshed by
exactly one part with the whole map's vertices, colours and faces -- across
frames out of order that make the volume grow (the ownership keys do not move
with growth) and over two incremental mesh updates."""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

pytestmark = pytest.mark.gpu

SHARDS = 3


def _map(**kw):
    from fastfusion_b200.fusion import FusionMipMapCPU
    return FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact",
                           **kw)


def _exchange(parts):
    """Each part's changed bricks into every other part; returns the record counts."""
    import torch
    counts = []
    bufs = []
    for p in parts:
        n, rb = p.halo_count()
        buf = torch.empty(max(n, 1) * rb, dtype=torch.uint8, device="cuda")
        assert p.halo_export(buf.data_ptr(), n) == n
        counts.append(n)
        bufs.append(buf)
    for i, p in enumerate(parts):
        for j, buf in enumerate(bufs):
            if j != i and counts[j]:
                p.halo_import(buf.data_ptr(), counts[j])
    # a second count right after an export is empty: nothing changed since
    assert all(p.halo_count()[0] == 0 for p in parts)
    return counts


def _same_voxels(a, b):
    (da, wa, ca), (db, wb, cb) = a.bricks(), b.bricks()
    assert np.array_equal(da.view(np.uint32), db.view(np.uint32))
    assert np.array_equal(wa.view(np.uint32), wb.view(np.uint32))
    assert np.array_equal(ca, cb)


def _union_mesh_is_whole(whole, parts):
    wmesh = whole.getMeshInterleavedMarchingCubes()
    wcells, wranges = whole.mesh_cells()
    meshed = np.zeros(len(wcells), np.int32)
    for p in parts:
        mesh = p.getMeshInterleavedMarchingCubes()
        cells, ranges = p.mesh_cells()
        assert np.array_equal(cells, wcells), "every part has every cell"
        for i in np.nonzero(ranges[:, 1])[0]:
            meshed[i] += 1
            v0, nv, f0, nf = (int(x) for x in ranges[i])
            w0, wnv, g0, wnf = (int(x) for x in wranges[i])
            assert (nv, nf) == (wnv, wnf), i
            assert np.array_equal(mesh.vertices[v0:v0 + nv].view(np.uint32), wmesh.vertices[w0:w0 + nv].view(np.uint32))
            assert np.array_equal(mesh.colors[v0:v0 + nv], wmesh.colors[w0:w0 + nv])
            assert np.array_equal(mesh.faces[f0:f0 + nf] - v0, wmesh.faces[g0:g0 + nf] - w0)
    # cells with vertices in the whole map: each meshed by exactly one part
    has = wranges[:, 1] > 0
    assert has.sum() > 100
    assert np.all(meshed[has] == 1) and np.all(meshed[~has] == 0)


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_parts_with_halo_exchange_are_the_whole_map(lib_built, storage):
    from fastfusion_b200.fusion import CameraInfo
    K, frames = circle_frames(0, 76, 320, 240)
    # later frames outside the first frame's volume: growth
    orders = [[50, 60, 75, 0], [10, 25, 40, 5]]
    whole = _map(storage=storage)
    parts = [_map(storage=storage) for _ in range(SHARDS)]
    for k, p in enumerate(parts):
        p.set_shard(k, SHARDS)
    first = True
    for order in orders:
        for i in order:
            depth, bgr, R, t = frames[i]
            cam = CameraInfo(K, R, t)
            q = whole.addMap(depth, cam, bgr, SCALING, MAXCAM)
            for p in parts:
                assert p.addMap(depth, cam, bgr, SCALING, MAXCAM) == q, i
        for p in parts:
            for a, b in zip(p.leaves(), whole.leaves()):
                assert np.array_equal(a, b)
        counts = _exchange(parts)
        if first:
            # every brick was new: the parts' exports partition the map
            n = whole.stats()["leaves_used"]
            assert sum(counts) == n
            assert all(0.15 * n < c < 0.55 * n for c in counts), counts
            first = False
        for p in parts:
            _same_voxels(p, whole)
        whole.updateMeshes()
        for p in parts:
            p.updateMeshes()
        _union_mesh_is_whole(whole, parts)
    assert whole.stats()["grows"] >= 1
    for p in parts:
        assert p.stats()["grows"] == whole.stats()["grows"]
    with pytest.raises(Exception):
        parts[0].set_shard(1, SHARDS)  # only before the first frame
