"""Generate the golden fixtures of the parity tests by running the reference
itself: its own fusion sources compiled into oracle/_ref/libffref.so (see
oracle/Makefile).  Run here, where the reference sources are available:

    make -C oracle all && python tests/golden/make_golden.py

Fixture (tests/golden/ref_seq0_64x48.npz):
  * the inputs: 5 seeded synthetic frames at 64x48 (uint16 depth, BGR, poses);
  * per frame, from the reference: volume side n, offset, leaves used and the
    set of bricks it updated, and the final leaf table (pos, scale, parent);
  * the reference's marching-cubes tables (edge mask, triangle edge lists);
  * the reference's mesh cells and, for each, a digest of the mesh the
    reference's own cell-meshing code produces when its bricks hold the
    oracle's round-toward-zero/exact-reciprocal voxel state (that state does
    not depend on the CPU's approximate reciprocal, so the digests hold on any
    machine).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fastfusion_b200 import scene  # noqa: E402
from oracle import port, ref  # noqa: E402

OUT = os.path.join(HERE, "ref_seq0_64x48.npz")
SCALING, MAXCAM = 1.0 / 5000.0, 4.0
NEED = {0: 1, 1: 2, 2: 2, 3: 2, 4: 4, 5: 4, 6: 4, 7: 8}


def cell_digest(xyz, rgb, faces):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(xyz, np.float32).tobytes())
    h.update(np.ascontiguousarray(rgb, np.uint8).tobytes())
    h.update(np.ascontiguousarray(faces, np.uint32).tobytes())
    return np.frombuffer(h.digest()[:8], np.uint64)[0]


def main():
    seq = scene.room_circle_sequence(0, 100, 64, 48)
    frames = [seq.frame(k) for k in (0, 3, 6, 9, 12)]
    r = ref.RefFusion()
    st0 = r.state()
    p = port.PortFusion(leaves_total=st0["leaves_total"], branches_total=st0["branches_total"], update_mode=1)
    out = {"K": seq.K, "depth": np.stack([f[0] for f in frames]), "bgr": np.stack([f[1] for f in frames]),
           "R": np.stack([f[2] for f in frames]), "t": np.stack([f[3] for f in frames])}
    per = {"n": [], "offset": [], "leaves_used": [], "queued": []}
    queues = []
    for depth, bgr, R, t in frames:
        r.add_map(depth, bgr, seq.K, R, t, SCALING, MAXCAM)
        p.add_map(depth, bgr, seq.K, R, t, SCALING, MAXCAM)
        st = r.state()
        per["n"].append(st["n"])
        per["offset"].append(st["offset"])
        per["leaves_used"].append(st["leaves_used"])
        per["queued"].append(st["queued"])
        queues.append(np.sort(r.queue()))
    for k, v in per.items():
        out["frame_" + k] = np.array(v)
    out["queue_concat"] = np.concatenate(queues).astype(np.uint32)
    pos, scl, par = r.leaves()
    out["leaf_pos"], out["leaf_scale"], out["leaf_parent"] = pos, scl, par
    em, tri = ref.mc_tables()
    out["mc_edge_mask"], out["mc_tri"] = em, tri.astype(np.int8)
    # mesh the oracle's exact voxel state with the reference's meshing code
    d, w, c = p.bricks()
    r.set_bricks(d, w, c)
    r.queue_all_cells()
    r.update_meshes()
    rows, digests = [], []
    for i, row in enumerate(r.cells()):
        t_ = int(row[0])
        L = [int(x) & 0xFFFFFFFF for x in row[6:6 + NEED[t_]]]
        if any(x >= ref.BRANCHINIT for x in L):
            continue
        xyz, rgb, faces = r.cell_mesh(i)
        rows.append([t_, int(row[1]), int(row[2]), int(row[3]), int(row[4])] + L + [0xFFFFFFFE] * (8 - len(L)))
        digests.append(cell_digest(xyz, rgb, faces))
    out["cells"] = np.array(rows, np.int64)
    out["cell_digest"] = np.array(digests, np.uint64)
    xyz, rgb, faces = r.mesh()
    out["mesh_counts"] = np.array([xyz.shape[0], faces.shape[0]])
    np.savez_compressed(OUT, **out)
    print(OUT, {k: getattr(v, "shape", None) for k, v in out.items()})


if __name__ == "__main__":
    main()
