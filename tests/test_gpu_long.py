"""GPU parity over whole sequences, at the benchmark's image size.

The short tests fuse a few frames; these run the configurations the
benchmark is quoted on, so that many volume growths, many incremental mesh
updates and the double-buffered frame pipeline (the voxel update of a frame
still running while the next frame is allocated) are all exercised:

* all 100 frames of the plain-method circle (640x480, 5 mm, meshing every
  10th frame) through the host-image entry point, against the restatement
  with exact round-toward-zero reciprocals;
* the first 60 frames of the 1000-frame random walk through the device-image
  entry point, against the compiled reference itself (the host CPU's RCPPS).

Between checks nothing synchronises the map (the per-frame queued count is
the only read), so the frames run pipelined as in the benchmark.  Frames are
rendered once on the GPU from the seeded scene and given to both sides.
"""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, queue_set

pytestmark = pytest.mark.gpu


def _render(seq, ks):
    import torch
    from fastfusion_b200.scene import render_torch
    out = []
    for k in ks:
        R, t = seq.poses[k]
        d, c = render_torch(seq.scene, R, t, seq.width, seq.height, seq.K, seq.seed, k, device="cuda")
        # uint16 depth bits kept in an int16 tensor (as the benchmark does)
        d16 = torch.empty((seq.height, seq.width), dtype=torch.int16, device="cuda")
        d16.copy_(d)
        out.append((d16, c.contiguous(), R, t))
    torch.cuda.synchronize()
    return out


def _host(d, c):
    return d.cpu().numpy().view(np.uint16), c.cpu().numpy()


def _same_state(g, o):
    sg, so = g.stats(), o.state()
    assert (sg["n"], sg["leaves_used"]) == (so["n"], so["leaves_used"])
    if "grows" in so:
        assert sg["grows"] == so["grows"]
    assert np.array_equal(sg["offset"], so["offset"])
    for a, b, name in zip(g.leaves(), o.leaves(), ("pos", "scale", "parent")):
        assert np.array_equal(a, b), f"leaf {name} differs"
    assert queue_set(g.queue()) == queue_set(o.queue())
    (dg, wg, cg), (do, wo, co) = g.bricks(), o.bricks()
    assert np.array_equal(dg.view(np.uint32), do.view(np.uint32)), "SDF bits differ"
    assert np.array_equal(wg.view(np.uint32), wo.view(np.uint32)), "weight bits differ"
    assert np.array_equal(cg, co), "colour differs"


def _triangles(xyz, rgb, faces):
    """The mesh as a sorted array of triangles (vertex bits and colours of the
    three corners): equal for two meshes made of the same per-cell meshes in
    any cell order."""
    faces = np.asarray(faces, np.int64).reshape(-1, 3)
    v = np.ascontiguousarray(xyz, np.float32).view(np.uint32)[faces].reshape(len(faces), 9)
    c = np.asarray(rgb, np.uint32)[faces].reshape(len(faces), 9)
    t = np.concatenate([v, c], axis=1)
    return t[np.lexsort(t.T[::-1])]


def test_config0_whole_sequence_bit_exact(lib_built, port_lib):
    """100 frames of the 640x480 circle, updateMeshes every 10th frame: leaf
    table, queue, every voxel bit and the mesh array for array equal the
    restatement's after every update."""
    from fastfusion_b200 import scene
    from fastfusion_b200.fusion import CameraInfo, FusionMipMapCPU
    seq = scene.room_circle_sequence(0, 100, 640, 480)
    frames = _render(seq, range(100))
    g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488, update_mode=1)
    updates = 0
    for k, (d, c, R, t) in enumerate(frames):
        hd, hc = _host(d, c)
        assert g.addMap(hd, CameraInfo(seq.K, R, t), hc, SCALING, MAXCAM) == \
            p.add_map(hd, hc, seq.K, R, t, SCALING, MAXCAM), k
        if k % 10 == 9:
            g.updateMeshes()
            ncells = p.update_meshes()
            _same_state(g, p)
            assert g.stats()["mesh_cells"] == ncells
            mesh = g.getMeshInterleavedMarchingCubes()
            _, _, xyz, rgb, faces = p.mesh()
            assert np.array_equal(mesh.vertices.view(np.uint32), xyz.view(np.uint32)), k
            assert np.array_equal(mesh.colors, rgb), k
            assert np.array_equal(mesh.faces, faces), k
            updates += 1
    assert updates == 10
    assert g.stats()["grows"] >= 1
    g.close()
    p.close()


def test_walk_prefix_bit_exact_with_reference_binary(lib_built):
    """The first 60 frames of the 640x480 random walk through the device-image
    entry point, against the compiled reference on this host (rcp="host"):
    queued counts every frame; leaf table, queue and every voxel bit at every
    update; and the mesh equals the reference's mesh of all its cells (its
    updateMeshes after queueing every cell), triangle for triangle."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/libffref.so not built")
    from fastfusion_b200 import scene
    from fastfusion_b200.fusion import CameraInfo, FusionMipMapCPU
    seq = scene.room_walk_sequence(0, 1000, 640, 480)
    frames = _render(seq, range(60))
    r = ref.RefFusion()
    st = r.state()
    g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=st["leaves_total"],
                        branches_max=st["branches_total"], rcp="host")
    for k, (d, c, R, t) in enumerate(frames):
        hd, hc = _host(d, c)
        qg = g.addMapDevice(d.data_ptr(), c.data_ptr(), seq.width, seq.height, CameraInfo(seq.K, R, t), SCALING,
                            MAXCAM)
        assert qg == r.add_map(hd, hc, seq.K, R, t, SCALING, MAXCAM), k
        if k % 10 == 9:
            g.updateMeshes()
            r.queue_all_cells()
            r.update_meshes()
            _same_state(g, r)
            mesh = g.getMeshInterleavedMarchingCubes()
            xr, cr, fr = r.mesh()
            a = _triangles(mesh.vertices, mesh.colors, mesh.faces)
            b = _triangles(xr, cr, fr)
            assert a.shape == b.shape, (k, a.shape, b.shape)
            assert np.array_equal(a, b), k
    g.close()
    r.close()
