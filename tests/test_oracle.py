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


def test_reference_float_overload_behaviour():
    """What the reference's float-depth addMap (geometryfusion_mipmap_cpu.cpp:1308-1600)
    does, run live with incremental meshing off (with it on, the default, its
    legacy mesh-cell bookkeeping in transformLoopSimPrecalculatedNeg_vis
    crashes the process, so that case is not run): the same octree as the
    16-bit overload for the same depths, but every brick updated twice per
    frame (update8NaiveFloat, then update8AddLoopSSESingleFloat,
    update_functions.cpp:1600-1623), so weights grow twice as fast, and no
    mesh from updateMeshes.  The library therefore offers no float-depth
    overload."""
    K, frames = circle_frames(0, 3, 160, 120)
    a, b = ref.RefFusion(), ref.RefFusion()
    b.L.ref_set_incremental_meshing(b.h, 0)
    for depth, bgr, R, t in frames:
        z = depth.astype(np.float32) * np.float32(SCALING)
        zf = np.where((z > 0) & (z < MAXCAM), z, np.nan).astype(np.float32)
        assert a.add_map(depth, bgr, K, R, t, SCALING, MAXCAM) == b.add_map_f32(zf, bgr, K, R, t)
    assert np.array_equal(a.tree(), b.tree())
    (_, wa, _), (_, wb, _) = a.bricks(), b.bricks()
    assert wa.max() <= 3.01 and wb.max() == 6.0
    assert 1.9 < wb.sum() / wa.sum() < 2.0
    b.update_meshes()
    assert len(b.mesh()[2]) == 0
    a.close()
    b.close()


def test_fp16_storage_rounding_matches_ieee_half(port_lib):
    """The restatement's FP16 storage keeps the nearest binary16 value (ties
    to even, overflow to infinity, subnormals): checked against numpy's
    float16 conversion on edge cases and a million random floats."""
    L = port_lib.lib()
    rng = np.random.default_rng(7)
    bits = rng.integers(0, 2**32, size=1_000_000, dtype=np.uint64).astype(np.uint32)
    vals = bits.view(np.float32)
    vals = vals[np.isfinite(vals)]
    edge = np.array([0.0, -0.0, 1.0, 65504.0, 65519.99, 65520.0, 70000.0, -65520.0, 2.0**-24, 2.0**-25,
                     1.5 * 2.0**-25, 2.0**-14, 2.0**-14 * (1 - 2.0**-11), 1e-9, 0.1, 0.3333333, 1 + 2.0**-11,
                     1 + 3 * 2.0**-11], np.float32)
    xs = np.concatenate([edge, -edge, vals[:200_000], (vals[:200_000] * 1e-30).astype(np.float32),
                         rng.normal(0, 0.02, 200_000).astype(np.float32)])
    want = xs.astype(np.float16).astype(np.float32)
    got = np.array([L.ffp_half_round(float(x)) for x in xs], np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
