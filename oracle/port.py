"""ctypes view of oracle/_ref/libffport.so, the C restatement of the hot path
(oracle/ff_port.c).

ORACLE INFRASTRUCTURE ONLY.  Imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by fastfusion_b200/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libffport.so")
_lib = None


def build() -> str:
    """Compile the restatement (needs only gcc); returns the library path."""
    subprocess.run(["make", "-C", _HERE, "port"], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, u32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_int64
        L.ffp_create.restype = vp
        L.ffp_create.argtypes = [ctypes.c_float, ctypes.c_float, i32, u32, u32]
        L.ffp_destroy.argtypes = [vp]
        L.ffp_set_update_mode.argtypes = [vp, i32]
        L.ffp_set_confidence.argtypes = [vp, vp]
        L.ffp_set_storage_fp16.argtypes = [vp, i32]
        L.ffp_half_round.restype = ctypes.c_float
        L.ffp_half_round.argtypes = [ctypes.c_float]
        L.ffp_add_map.restype = i32
        L.ffp_add_map.argtypes = [vp, vp, vp, i32, i32, vp, vp, vp, ctypes.c_float, ctypes.c_float]
        L.ffp_state.argtypes = [vp, vp, vp]
        L.ffp_leaves.argtypes = [vp, vp, vp, vp]
        L.ffp_queue.argtypes = [vp, vp]
        L.ffp_tree.argtypes = [vp, vp]
        L.ffp_bricks.argtypes = [vp, i64, vp, vp, vp]
        L.ffp_bricks64.argtypes = [vp, i64, vp, vp]
        L.ffp_set_bricks.argtypes = [vp, i64, vp, vp, vp]
        L.ffp_update_meshes.restype = i64
        L.ffp_update_meshes.argtypes = [vp]
        L.ffp_mesh_counts.argtypes = [vp, vp, vp, vp]
        L.ffp_mesh_copy.argtypes = [vp, vp, vp, vp, vp, vp]
        L.ffp_set_state.restype = i32
        L.ffp_set_state.argtypes = [vp, u32, vp, vp, u32, vp, vp, vp, u32, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class PortFusion:
    """The restated addMap path: bit-exact target of the GPU plain FP32 path."""

    def __init__(self, scale=0.005, threshold=0.01, color=True, leaves_total=271420, branches_total=None,
                 update_mode=1, fp16=False):
        if branches_total is None:
            branches_total = max(16 * 4096, leaves_total * 4)
        self.h = lib().ffp_create(scale, threshold, 1 if color else 0, leaves_total, branches_total)
        lib().ffp_set_update_mode(self.h, int(update_mode))
        if fp16:
            lib().ffp_set_storage_fp16(self.h, 1)

    def close(self):
        if self.h:
            lib().ffp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_confidence(self, conf):
        """Per-pixel confidence (H x W float32) for the next add_map calls, or None."""
        if conf is None:
            self._conf = None
            lib().ffp_set_confidence(self.h, None)
            return
        self._conf = np.ascontiguousarray(conf, dtype=np.float32)
        lib().ffp_set_confidence(self.h, _p(self._conf))

    def add_map(self, depth, bgr, K, R, t, scaling=1.0 / 5000.0, maxcam=4.0) -> int:
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        bgr = np.ascontiguousarray(bgr, dtype=np.uint8)
        K = np.ascontiguousarray(K, dtype=np.float64)
        R = np.ascontiguousarray(R, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        h, w = depth.shape
        return lib().ffp_add_map(self.h, _p(depth), _p(bgr), w, h, _p(K), _p(R), _p(t),
                                 ctypes.c_float(scaling), ctypes.c_float(maxcam))

    def state(self) -> dict:
        ints = np.zeros(16, np.int64)
        off = np.zeros(3, np.float32)
        lib().ffp_state(self.h, _p(ints), _p(off))
        keys = ["n", "leaves_used", "branches_used", "queued", "leaves_total", "branches_total", "frames",
                "bandwidth", "meshing_ok", "grows"]
        d = {k: int(v) for k, v in zip(keys, ints)}
        d["offset"] = off
        return d

    def leaves(self):
        st = self.state()
        n = min(st["leaves_used"], st["leaves_total"])
        pos = np.zeros((n, 3), np.uint16)
        scl = np.zeros(n, np.uint16)
        par = np.zeros(n, np.uint32)
        lib().ffp_leaves(self.h, _p(pos), _p(scl), _p(par))
        return pos, scl, par

    def queue(self):
        q = np.zeros(self.state()["queued"], np.uint32)
        lib().ffp_queue(self.h, _p(q))
        return q

    def tree(self):
        tr = np.zeros(self.state()["branches_used"], np.uint32)
        lib().ffp_tree(self.h, _p(tr))
        return tr

    def bricks(self, n=None):
        st = self.state()
        if n is None:
            n = min(st["leaves_used"], st["leaves_total"])
        d = np.zeros((n, 512), np.float32)
        w = np.zeros((n, 512), np.float32)
        c = np.zeros((n, 512, 3), np.uint16)
        lib().ffp_bricks(self.h, n, _p(d), _p(w), _p(c))
        return d, w, c

    def bricks64(self, n=None):
        """SDF and weights of the FP64 oracle (update_mode=3)."""
        st = self.state()
        if n is None:
            n = min(st["leaves_used"], st["leaves_total"])
        d = np.zeros((n, 512), np.float64)
        w = np.zeros((n, 512), np.float64)
        lib().ffp_bricks64(self.h, n, _p(d), _p(w))
        return d, w

    def set_bricks(self, d, w, c):
        d = np.ascontiguousarray(d, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        c = np.ascontiguousarray(c, np.uint16)
        lib().ffp_set_bricks(self.h, d.shape[0], _p(d), _p(w), _p(c))

    # -- meshing ---------------------------------------------------------
    def update_meshes(self) -> int:
        """Re-mesh every cell; returns the number of cells."""
        return lib().ffp_update_meshes(self.h)

    def mesh(self):
        """(cells int32[n,14], ranges int64[n,4], xyz, rgb, faces) of the last update."""
        c = np.zeros(3, np.int64)
        lib().ffp_mesh_counts(self.h, _p(c[0:1]), _p(c[1:2]), _p(c[2:3]))
        nc, nv, nf = (int(x) for x in c)
        cells = np.zeros((nc, 14), np.int32)
        ranges = np.zeros((nc, 4), np.int64)
        xyz = np.zeros((nv, 3), np.float32)
        rgb = np.zeros((nv, 3), np.uint8)
        faces = np.zeros((nf, 3), np.uint32)
        lib().ffp_mesh_copy(self.h, _p(cells), _p(ranges), _p(xyz), _p(rgb), _p(faces))
        return cells, ranges, xyz, rgb, faces

    def set_state(self, n, offset, tree, pos, scale, parent, dist, wgt, col):
        offset = np.ascontiguousarray(offset, np.float32)
        tree = np.ascontiguousarray(tree, np.uint32)
        pos = np.ascontiguousarray(pos, np.uint16)
        scale = np.ascontiguousarray(scale, np.uint16)
        parent = np.ascontiguousarray(parent, np.uint32)
        dist = np.ascontiguousarray(dist, np.float32)
        wgt = np.ascontiguousarray(wgt, np.float32)
        col = np.ascontiguousarray(col, np.uint16)
        r = lib().ffp_set_state(self.h, int(n), _p(offset), _p(tree), tree.shape[0], _p(pos), _p(scale), _p(parent),
                                pos.shape[0], _p(dist), _p(wgt), _p(col))
        if r != 0:
            raise ValueError("state larger than this map's capacity")
