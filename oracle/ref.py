"""ctypes view of oracle/_ref/libffref.so: the reference's own FusionMipMapCPU
compiled from its sources (see oracle/Makefile).

ORACLE INFRASTRUCTURE ONLY.  Imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by fastfusion_b200/.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libffref.so")
_libs = {}

BRANCHINIT = 0xFFFFFFFE


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    key = 0
    if key not in _libs:
        # The reference is C++ and formats numbers through libstdc++'s locale
        # machinery.  When numpy has already pulled libstdc++ in as a private
        # dependency of its bundled BLAS, a library loaded afterwards crashes
        # in that machinery; making libstdc++ global first avoids it.
        ctypes.CDLL("libstdc++.so.6", mode=ctypes.RTLD_GLOBAL)
        L = ctypes.CDLL(LIB_PATH)
        vp, ll, i32 = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int
        L.ref_create.restype = vp
        L.ref_create.argtypes = [ctypes.c_float, ctypes.c_float, i32, ll]
        L.ref_destroy.argtypes = [vp]
        L.ref_quiet.argtypes = [i32]
        L.ref_set_incremental_meshing.argtypes = [vp, i32]
        L.ref_add_map.restype = i32
        L.ref_add_map.argtypes = [vp, vp, vp, i32, i32, vp, vp, vp, ctypes.c_float, ctypes.c_float]
        L.ref_add_map_f32.restype = i32
        L.ref_add_map_f32.argtypes = [vp, vp, vp, vp, vp, i32, i32, vp, vp, vp]
        L.ref_update_meshes.restype = i32
        L.ref_update_meshes.argtypes = [vp]
        L.ref_mesh_counts.argtypes = [vp, ctypes.POINTER(ll), ctypes.POINTER(ll)]
        L.ref_mesh_copy.argtypes = [vp, vp, vp, vp]
        L.ref_write_ply.restype = i32
        L.ref_write_ply.argtypes = [vp, ctypes.c_char_p, i32]
        L.ref_write_obj.restype = i32
        L.ref_write_obj.argtypes = [vp, ctypes.c_char_p]
        L.ref_state.argtypes = [vp, vp, vp]
        L.ref_leaves.argtypes = [vp, ll, vp, vp, vp]
        L.ref_queue.argtypes = [vp, vp]
        L.ref_tree.argtypes = [vp, vp]
        L.ref_bricks.argtypes = [vp, ll, vp, vp, vp]
        L.ref_set_bricks.argtypes = [vp, ll, vp, vp, vp]
        L.ref_cells.restype = ll
        L.ref_cells.argtypes = [vp, vp]
        L.ref_queue_all_cells.argtypes = [vp]
        L.ref_set_thread_meshing.argtypes = [vp, ctypes.c_int]
        L.ref_loop_delete.restype = ctypes.c_int
        L.ref_loop_delete.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, ll, vp, vp,
                                      ctypes.c_uint32, vp, vp, vp]
        L.ref_cell_mesh.restype = ll
        L.ref_cell_mesh.argtypes = [vp, ll, vp, vp, vp, ctypes.POINTER(ll)]
        L.ref_mc_offset_table.argtypes = [vp]
        L.ref_mc_tables.argtypes = [vp, vp]
        _libs[key] = L
    return _libs[key]


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefFusion:
    """The reference FusionMipMapCPU (single-threaded meshing)."""

    def __init__(self, scale=0.005, threshold=0.01, color=True, pool_bytes=0, quiet=True):
        self.L = L = lib()
        if quiet:
            L.ref_quiet(1)
        self.h = L.ref_create(scale, threshold, 1 if color else 0, int(pool_bytes))

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_map(self, depth, bgr, K, R, t, scaling=1.0 / 5000.0, maxcam=4.0) -> int:
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        bgr = np.ascontiguousarray(bgr, dtype=np.uint8)
        K = np.ascontiguousarray(K, dtype=np.float64)
        R = np.ascontiguousarray(R, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        h, w = depth.shape
        return self.L.ref_add_map(self.h, _p(depth), _p(bgr), w, h, _p(K), _p(R), _p(t),
                                 ctypes.c_float(scaling), ctypes.c_float(maxcam))

    def update_meshes(self) -> bool:
        return bool(self.L.ref_update_meshes(self.h))

    def loop_delete(self, depth_m, red, green, blue, K, R, t, queue, leaf_map, n_mapped, capacity, dist, wgt,
                    col) -> tuple[bool, int]:
        """The reference's removal of one fused frame into caller loop arrays
        (deleteOldLoopPoses' camera set-up, then updateWrapper_deleteloop):
        leaf_map (uint32, one per leaf) and the arrays are updated in place;
        returns (completed, slots in use)."""
        depth_m = np.ascontiguousarray(depth_m, np.float32)
        h, w = depth_m.shape
        planes = [np.ascontiguousarray(a, np.uint8) for a in (red, green, blue)]
        K = np.ascontiguousarray(K, np.float64)
        R = np.ascontiguousarray(R, np.float64)
        t = np.ascontiguousarray(t, np.float64)
        q = np.ascontiguousarray(queue, np.uint32)
        nm = np.array([n_mapped], np.uint32)
        ok = self.L.ref_loop_delete(self.h, _p(depth_m), _p(planes[0]), _p(planes[1]), _p(planes[2]), w, h, _p(K),
                                    _p(R), _p(t), _p(q), len(q), _p(leaf_map), _p(nm), int(capacity), _p(dist),
                                    _p(wgt), _p(col))
        return bool(ok), int(nm[0])

    def set_thread_meshing(self, on: bool):
        """The reference's setThreadMeshing: meshing on a second thread,
        updateMeshes returning False while it is busy."""
        self.L.ref_set_thread_meshing(self.h, 1 if on else 0)

    def mesh(self):
        nv, nf = ctypes.c_longlong(), ctypes.c_longlong()
        self.L.ref_mesh_counts(self.h, ctypes.byref(nv), ctypes.byref(nf))
        xyz = np.zeros((nv.value, 3), np.float32)
        rgb = np.zeros((nv.value, 3), np.uint8)
        faces = np.zeros((nf.value, 3), np.uint32)
        self.L.ref_mesh_copy(self.h, _p(xyz), _p(rgb), _p(faces))
        return xyz, rgb, faces

    def write_ply(self, stem: str, binary: bool = True) -> bool:
        """The reference's MeshInterleaved::writePLY of its current mesh (writes stem + ".ply")."""
        return bool(self.L.ref_write_ply(self.h, stem.encode(), 1 if binary else 0))

    def write_obj(self, stem: str) -> bool:
        """The reference's MeshInterleaved::writeOBJ of its current mesh (writes stem + ".obj")."""
        return bool(self.L.ref_write_obj(self.h, stem.encode()))

    def add_map_f32(self, depth, bgr, K, R, t) -> int:
        """The reference's float-depth addMap: depth in metres (non-finite: hole),
        colour passed as its three planes (split here from a BGR image)."""
        depth = np.ascontiguousarray(depth, dtype=np.float32)
        bgr = np.ascontiguousarray(bgr, dtype=np.uint8)
        planes = [np.ascontiguousarray(bgr[..., c]) for c in range(3)]
        K = np.ascontiguousarray(K, dtype=np.float64)
        R = np.ascontiguousarray(R, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        h, w = depth.shape
        return self.L.ref_add_map_f32(self.h, _p(depth), _p(planes[0]), _p(planes[1]), _p(planes[2]), w, h,
                                      _p(K), _p(R), _p(t))

    def state(self) -> dict:
        ints = np.zeros(16, np.int64)
        off = np.zeros(3, np.float32)
        self.L.ref_state(self.h, _p(ints), _p(off))
        keys = ["n", "leaves_used", "branches_used", "queued", "leaves_total", "branches_total",
                "cells", "frames", "bandwidth", "incremental"]
        d = {k: int(v) for k, v in zip(keys, ints)}
        d["offset"] = off
        return d

    def leaves(self, n=None):
        if n is None:
            n = self.state()["leaves_used"]
        pos = np.zeros((n, 3), np.uint16)
        scl = np.zeros(n, np.uint16)
        par = np.zeros(n, np.uint32)
        self.L.ref_leaves(self.h, n, _p(pos), _p(scl), _p(par))
        return pos, scl, par

    def queue(self):
        n = self.state()["queued"]
        q = np.zeros(n, np.uint32)
        self.L.ref_queue(self.h, _p(q))
        return q

    def tree(self):
        n = self.state()["branches_used"]
        tr = np.zeros(n, np.uint32)
        self.L.ref_tree(self.h, _p(tr))
        return tr

    def bricks(self, n=None):
        if n is None:
            n = min(self.state()["leaves_used"], self.state()["leaves_total"])
        d = np.zeros((n, 512), np.float32)
        w = np.zeros((n, 512), np.float32)
        c = np.zeros((n, 512, 3), np.uint16)
        self.L.ref_bricks(self.h, n, _p(d), _p(w), _p(c))
        return d, w, c

    def set_bricks(self, d, w, c):
        d = np.ascontiguousarray(d, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        c = np.ascontiguousarray(c, np.uint16)
        self.L.ref_set_bricks(self.h, d.shape[0], _p(d), _p(w), _p(c))

    def cells(self):
        n = self.L.ref_cells(self.h, None)
        out = np.zeros((n, 14), np.int32)
        self.L.ref_cells(self.h, _p(out))
        return out

    def queue_all_cells(self):
        self.L.ref_queue_all_cells(self.h)

    def cell_mesh(self, i):
        nf = ctypes.c_longlong()
        nv = self.L.ref_cell_mesh(self.h, i, None, None, None, ctypes.byref(nf))
        xyz = np.zeros((nv, 3), np.float32)
        rgb = np.zeros((nv, 3), np.uint8)
        faces = np.zeros((nf.value, 3), np.uint32)
        self.L.ref_cell_mesh(self.h, i, _p(xyz), _p(rgb), _p(faces), ctypes.byref(nf))
        return xyz, rgb, faces


def mc_offset_table() -> np.ndarray:
    out = np.zeros((256, 16), np.int32)
    lib().ref_mc_offset_table(_p(out))
    return out


def mc_tables():
    """(edge mask per case, triangle edge list per case) of the reference."""
    em = np.zeros(256, np.int32)
    tri = np.zeros((256, 16), np.int32)
    lib().ref_mc_tables(_p(em), _p(tri))
    return em, tri
