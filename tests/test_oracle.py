"""The oracle's C restatement against the compiled reference, run live.

With the host CPU's own approximate reciprocal (update mode 2) the
restatement must reproduce the reference bit for bit: leaf table, queue (in
order), octree, and every SDF, weight and colour value.  Mode 1 (exact
reciprocal, the GPU's target) differs from the reference only where the
reference's ~12-bit reciprocal moves a value.
"""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

ref = pytest.importorskip("oracle.ref")
pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref/libffref.so not built")
NEED = {0: 1, 1: 2, 2: 2, 3: 2, 4: 4, 5: 4, 6: 4, 7: 8}


def test_restatement_bit_exact_with_reference(port_lib):
    K, frames = circle_frames(0, 4, 160, 120)
    r = ref.RefFusion()
    st = r.state()
    p = port_lib.PortFusion(leaves_total=st["leaves_total"], branches_total=st["branches_total"], update_mode=2)
    for depth, bgr, R, t in frames:
        assert r.add_map(depth, bgr, K, R, t, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        for a, b in zip(r.leaves(), p.leaves()):
            assert np.array_equal(a, b)
        assert np.array_equal(r.queue(), p.queue())
        assert np.array_equal(r.tree(), p.tree())
    for a, b in zip(r.bricks(), p.bricks()):
        assert np.array_equal(a, b)


def test_exact_reciprocal_mode_close_to_reference(port_lib):
    K, frames = circle_frames(0, 3, 160, 120)
    r = ref.RefFusion()
    st = r.state()
    p = port_lib.PortFusion(leaves_total=st["leaves_total"], branches_total=st["branches_total"], update_mode=1)
    for depth, bgr, R, t in frames:
        r.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    for a, b in zip(r.leaves(), p.leaves()):
        assert np.array_equal(a, b)  # the traversal has no reciprocal
    (dr, wr, cr), (dp, wp, cp) = r.bricks(), p.bricks()
    seen = (wr > 0) | (wp > 0)
    dd = np.abs(dr - dp)[seen]
    # RCPPS carries ~12 bits: most voxels agree to a few ulp, a few per mille
    # move by up to the truncation band when a projection lands on the next pixel
    assert np.median(dd) < 1e-4 and np.percentile(dd, 99) < 2e-3
    assert np.median(np.abs(wr - wp)[seen] / np.maximum(wr[seen], 1e-6)) < 1e-3
    assert (np.abs(cr.astype(np.int32) - cp.astype(np.int32)).max(axis=-1)[seen] <= 256).mean() > 0.99


def test_meshing_cells_match_reference_live(port_lib):
    K, frames = circle_frames(0, 3, 160, 120)
    r = ref.RefFusion()
    for depth, bgr, R, t in frames:
        r.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    st = r.state()
    pos, scl, par = r.leaves()
    d, w, c = r.bricks()
    p = port_lib.PortFusion(leaves_total=st["leaves_total"], branches_total=st["branches_total"])
    p.set_state(st["n"], st["offset"], r.tree(), pos, scl, par, d, w, c)
    p.update_meshes()
    cells, ranges, xyz, rgb, faces = p.mesh()
    r.queue_all_cells()
    r.update_meshes()
    refmap = {}
    for i, row in enumerate(r.cells()):
        t = int(row[0])
        L = tuple(int(x) & 0xFFFFFFFF for x in row[6:6 + NEED[t]])
        if all(x < ref.BRANCHINIT for x in L):
            refmap[(t, int(row[1]), int(row[2]), int(row[3]), int(row[4]), L)] = i
    n_common = n_same = 0
    for i, row in enumerate(cells):
        t = int(row[0])
        key = (t, int(row[2]), int(row[3]), int(row[4]), int(row[5]), tuple(int(x) & 0xFFFFFFFF for x in row[6:6 + NEED[t]]))
        if key not in refmap:
            continue
        n_common += 1
        rx, rc, rf = r.cell_mesh(refmap[key])
        v0, nv, f0, nf = ranges[i]
        n_same += (rx.shape[0] == nv and rf.shape[0] == nf and np.array_equal(rx.view(np.uint32), xyz[v0:v0 + nv].view(np.uint32))
                   and np.array_equal(rc, rgb[v0:v0 + nv]) and np.array_equal(rf, faces[f0:f0 + nf] - v0))
    assert n_common == len(refmap) == len(cells)
    assert n_same == n_common
