"""GPU marching cubes against the oracle.

The oracle's meshing (oracle/ff_port_mesh.c) is pinned cell by cell against
the compiled reference (tests/test_oracle.py).  Both sort cells by (type,
quirk, size, origin), so the GPU mesh must equal the oracle's array for array:
vertex bits, colours and face indices.
"""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

pytestmark = pytest.mark.gpu


def _cam(K, R, t):
    from fastfusion_b200.fusion import CameraInfo
    return CameraInfo(K, R, t)


def _gpu(**kw):
    from fastfusion_b200.fusion import FusionMipMapCPU
    return FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=kw.get("leaves_max", 271420),
                           branches_max=kw.get("branches_max", 4793488), storage=kw.get("storage", "fp32"),
                           rcp=kw.get("rcp", "exact"))


def _assert_same_mesh(gmesh, pmesh):
    cells, ranges, xyz, rgb, faces = pmesh
    assert gmesh.vertices.shape == xyz.shape, (gmesh.vertices.shape, xyz.shape)
    assert gmesh.faces.shape == faces.shape
    assert np.array_equal(gmesh.vertices.view(np.uint32), xyz.view(np.uint32)), "vertex bits differ"
    assert np.array_equal(gmesh.colors, rgb), "colours differ"
    assert np.array_equal(gmesh.faces, faces), "faces differ"


@pytest.mark.parametrize("wh,nframes", [((160, 120), 8), ((640, 480), 4)])
def test_mesh_after_fusion_matches_oracle(lib_built, port_lib, wh, nframes):
    K, frames = circle_frames(0, nframes, *wh)
    g = _gpu()
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488)
    for depth, bgr, R, t in frames:
        g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM)
        p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    g.updateMeshes()
    ncells = p.update_meshes()
    assert g.stats()["mesh_cells"] == ncells
    _assert_same_mesh(g.getMeshInterleavedMarchingCubes(), p.mesh())


def test_incremental_equals_full_remesh(lib_built, port_lib):
    """Meshing every third frame (dirty cells only) ends with the same mesh as
    one full meshing at the end, and as the oracle."""
    K, frames = circle_frames(2, 12, 160, 120)
    a, b = _gpu(), _gpu()
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488)
    dirty = []
    for k, (depth, bgr, R, t) in enumerate(frames):
        for m in (a, b):
            m.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM)
        p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        if k % 3 == 2:
            a.updateMeshes()
            dirty.append((a.stats()["mesh_cells_dirty"], a.stats()["mesh_cells"]))
    a.updateMeshes()
    b.updateMeshes()
    p.update_meshes()
    ma, mb = a.getMeshInterleavedMarchingCubes(), b.getMeshInterleavedMarchingCubes()
    assert np.array_equal(ma.vertices.view(np.uint32), mb.vertices.view(np.uint32))
    assert np.array_equal(ma.faces, mb.faces)
    assert np.array_equal(ma.colors, mb.colors)
    _assert_same_mesh(ma, p.mesh())
    # later updates re-mesh only part of the map
    assert any(d < n for d, n in dirty[1:]), dirty


def test_mesh_of_reference_state(lib_built, port_lib):
    """Mesh the compiled reference's own voxel state (imported as a snapshot):
    GPU == oracle on identical input."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/libffref.so not built")
    K, frames = circle_frames(1, 5, 160, 120)
    r = ref.RefFusion()
    for depth, bgr, R, t in frames:
        r.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    st = r.state()
    pos, scl, par = r.leaves()
    d, w, c = r.bricks()
    tree = r.tree()
    g = _gpu()
    g.set_state(st["n"], st["offset"], tree, pos, scl, par, d, w, c)
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488)
    p.set_state(st["n"], st["offset"], tree, pos, scl, par, d, w, c)
    g.updateMeshes()
    p.update_meshes()
    _assert_same_mesh(g.getMeshInterleavedMarchingCubes(), p.mesh())


def test_mesh_matches_reference_binary_cells(lib_built):
    """rcp="host" end to end against the compiled reference: fuse the same
    frames, then the GPU has the reference's cells, each with the same mesh
    (vertex bits, colours, local faces)."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/libffref.so not built")
    need = {0: 1, 1: 2, 2: 2, 3: 2, 4: 4, 5: 4, 6: 4, 7: 8}
    K, frames = circle_frames(0, 4, 320, 240)
    r = ref.RefFusion()
    g = _gpu(rcp="host")
    for depth, bgr, R, t in frames:
        r.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM)
    r.queue_all_cells()
    r.update_meshes()
    g.updateMeshes()
    mesh = g.getMeshInterleavedMarchingCubes()
    cells, ranges = g.mesh_cells()
    refmap = {}
    for i, row in enumerate(r.cells()):
        t = int(row[0])
        L = tuple(int(x) & 0xFFFFFFFF for x in row[6:6 + need[t]])
        if all(x < ref.BRANCHINIT for x in L):
            refmap[(t, int(row[1]), int(row[2]), int(row[3]), int(row[4]), L)] = i
    common = same = 0
    for i, row in enumerate(cells):
        t = int(row[0])
        key = (t, int(row[2]), int(row[3]), int(row[4]), int(row[5]), tuple(int(x) & 0xFFFFFFFF for x in row[6:6 + need[t]]))
        if key not in refmap:
            continue
        common += 1
        rx, rc, rf = r.cell_mesh(refmap[key])
        v0, nv, f0, nf = (int(x) for x in ranges[i])
        same += (rx.shape[0] == nv and rf.shape[0] == nf
                 and np.array_equal(rx.view(np.uint32), mesh.vertices[v0:v0 + nv].view(np.uint32))
                 and np.array_equal(rc, mesh.colors[v0:v0 + nv]) and np.array_equal(rf, mesh.faces[f0:f0 + nf] - v0))
    assert common == len(refmap) == len(cells)
    assert same == common


def test_async_mesh_export_overlaps_and_matches(lib_built):
    """getMeshInterleavedMarchingCubes(wait=False) (ff_get_mesh_async): the
    copy runs behind the map's work while the next frames -- and the next
    updateMeshes, which rewrites the device mesh -- are issued; after
    mesh_wait() the buffer holds exactly the mesh the blocking export gave."""
    from fastfusion_b200 import fusion as ff
    K, frames = circle_frames(3, 12, 320, 240)
    m = ff.FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    buf = ff.MeshBuffer()
    for k0 in (0, 4):
        for depth, bgr, R, t in frames[k0:k0 + 4]:
            m.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
        m.updateMeshes()
        want = m.getMeshInterleavedMarchingCubes()
        got = m.getMeshInterleavedMarchingCubes(out=buf, wait=False)
        # more work behind the copy: frames and a mesh update that rewrites
        # the device buffers the copy reads
        for depth, bgr, R, t in frames[k0 + 4:k0 + 6]:
            m.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
        m.updateMeshes()
        m.mesh_wait()
        assert len(want.faces) > 0
        assert np.array_equal(got.vertices.view(np.uint32), want.vertices.view(np.uint32))
        assert np.array_equal(got.colors, want.colors)
        assert np.array_equal(got.faces, want.faces)
    m.close()
    buf.close()


def test_async_mesh_exports_two_in_flight(lib_built):
    """Two asynchronous exports in flight with two updates between them and
    the wait: each buffer holds the mesh of its own update (the second update
    rewrites the device buffers the first copy reads, so it waits for that
    copy on the device).  The expected meshes come from a second map fed the
    same frames and read with the blocking export."""
    from fastfusion_b200 import fusion as ff
    K, frames = circle_frames(5, 12, 320, 240)
    m = ff.FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    r = ff.FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    bufs = [ff.MeshBuffer(), ff.MeshBuffer()]
    want, got = [], []
    for u in range(4):
        for depth, bgr, R, t in frames[3 * u:3 * u + 3]:
            m.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
            r.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
        m.updateMeshes()
        r.updateMeshes()
        got.append(m.getMeshInterleavedMarchingCubes(out=bufs[u % 2], wait=False))
        w = r.getMeshInterleavedMarchingCubes()
        want.append((w.vertices, w.colors, w.faces))
        if u % 2 == 1:
            m.mesh_wait()
            for k in (u - 1, u):
                assert len(want[k][2]) > 0
                assert np.array_equal(got[k].vertices.view(np.uint32), want[k][0].view(np.uint32)), k
                assert np.array_equal(got[k].colors, want[k][1]), k
                assert np.array_equal(got[k].faces, want[k][2]), k
    m.close()
    r.close()
    for b in bufs:
        b.close()
