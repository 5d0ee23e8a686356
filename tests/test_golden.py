"""The oracle against the golden fixture produced by the reference itself
(tests/golden/make_golden.py runs the reference's own fusion sources).

* traversal: per frame, the volume, offset, number of leaves and the set of
  updated bricks, and the final leaf table -- exactly;
* meshing: the set of mesh cells, and every cell's mesh (vertex bits,
  colours, faces) -- exactly, from the same voxel state;
* the marching-cubes triangle table of the product equals the reference's.
"""
import hashlib
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIX = os.path.join(HERE, "golden", "ref_seq0_64x48.npz")
SCALING, MAXCAM = 1.0 / 5000.0, 4.0
NEED = {0: 1, 1: 2, 2: 2, 3: 2, 4: 4, 5: 4, 6: 4, 7: 8}


@pytest.fixture(scope="module")
def fix():
    return dict(np.load(FIX))


@pytest.fixture(scope="module")
def port_run(fix, port_lib):
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488, update_mode=1)
    per = []
    for k in range(fix["depth"].shape[0]):
        p.add_map(fix["depth"][k], fix["bgr"][k], fix["K"], fix["R"][k], fix["t"][k], SCALING, MAXCAM)
        st = p.state()
        per.append((st["n"], st["offset"].copy(), st["leaves_used"], np.sort(p.queue())))
    return p, per


def test_traversal_matches_reference(fix, port_run):
    p, per = port_run
    q_concat = []
    for k, (n, off, used, q) in enumerate(per):
        assert n == fix["frame_n"][k]
        assert np.array_equal(off, fix["frame_offset"][k].astype(np.float32))
        assert used == fix["frame_leaves_used"][k]
        assert len(q) == fix["frame_queued"][k]
        q_concat.append(q)
    assert np.array_equal(np.concatenate(q_concat), fix["queue_concat"])
    pos, scl, par = p.leaves()
    assert np.array_equal(pos, fix["leaf_pos"])
    assert np.array_equal(scl, fix["leaf_scale"])
    assert np.array_equal(par, fix["leaf_parent"])


def _digest(xyz, rgb, faces):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(xyz, np.float32).tobytes())
    h.update(np.ascontiguousarray(rgb, np.uint8).tobytes())
    h.update(np.ascontiguousarray(faces, np.uint32).tobytes())
    return np.frombuffer(h.digest()[:8], np.uint64)[0]


def test_mesh_cells_match_reference(fix, port_run):
    p, _ = port_run
    p.update_meshes()
    cells, ranges, xyz, rgb, faces = p.mesh()
    mine = {}
    for i, row in enumerate(cells):
        t = int(row[0])
        L = tuple(int(x) & 0xFFFFFFFF for x in row[6:6 + NEED[t]])
        v0, nv, f0, nf = ranges[i]
        mine[(t, int(row[2]), int(row[3]), int(row[4]), int(row[5]), L)] = _digest(
            xyz[v0:v0 + nv], rgb[v0:v0 + nv], faces[f0:f0 + nf] - v0)
    refc = {}
    for row, dg in zip(fix["cells"], fix["cell_digest"]):
        t = int(row[0])
        refc[(t, int(row[1]), int(row[2]), int(row[3]), int(row[4]), tuple(int(x) for x in row[5:5 + NEED[t]]))] = dg
    # the same cells (type, origin, size, side leaves) ...
    assert set(mine) == set(refc)
    # ... each with the same mesh
    bad = [k for k in refc if mine[k] != refc[k]]
    assert not bad, "%d of %d cells mesh differently, e.g. %s" % (len(bad), len(refc), bad[:3])


def _product_table():
    src = open(os.path.join(ROOT, "fastfusion_b200", "csrc", "ff_mc_table.inc")).read()
    vals = [int(x, 16) for x in __import__("re").findall(r"0x([0-9a-f]{16})ull", src)]
    assert len(vals) == 256
    tri = np.full((256, 16), -1, np.int8)
    for c, v in enumerate(vals):
        n = v >> 60
        for k in range(3 * n):
            tri[c, k] = (v >> (4 * k)) & 15
    return tri


def test_marching_cubes_table_matches_reference(fix):
    assert np.array_equal(_product_table(), fix["mc_tri"])
    E = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]
    for c in range(256):
        mask = sum(1 << e for e, (a, b) in enumerate(E) if ((c >> a) & 1) != ((c >> b) & 1))
        assert mask == fix["mc_edge_mask"][c]
