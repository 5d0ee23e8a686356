"""Python host API of the B200 fusion path, mirroring the reference's C++
interface (tum-vision/fastfusion src/fusion/geometryfusion_mipmap_cpu.hpp):

    fusion = FusionMipMapCPU(0, 0, 0, scale, distanceThreshold, 0, True)
    n = fusion.addMap(depth_u16, CameraInfo(K, R, t), bgr_u8, 1/5000., maxcam)
    fusion.updateMeshes()
    mesh = fusion.getMeshInterleavedMarchingCubes()

Every call goes through the C ABI of libfastfusion_b200.so
(include/fastfusion_b200.h); there is no CPU fallback.  Loading fails loudly
when the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libfastfusion_b200.so")

FF_OK = 0
_STATUS = {0: "FF_OK", 1: "FF_ERR_BAD_ARG", 2: "FF_ERR_CUDA", 3: "FF_ERR_OOM_POOL", 4: "FF_ERR_OOM_MESH",
           5: "FF_ERR_TIMEOUT", 6: "FF_ERR_STATE", 7: "FF_ERR_NO_DEVICE"}
NOALLOC_MAX_CELLS = 65536  # FF_NOALLOC_MAX_CELLS
SPIN_LIMIT_DEFAULT = 1 << 22  # FF_SPIN_LIMIT_DEFAULT
CELLS_INCREMENTAL, CELLS_FULL = 0, 1  # FF_CELLS_INCREMENTAL, FF_CELLS_FULL
INJECT_CONFIDENCE_TIMEOUT = 1  # FF_INJECT_CONFIDENCE_TIMEOUT

STORAGE = {"fp32": 0, "fp16": 1}
RCP = {"host": 0, "exact": 1}
BRANCHINIT = 0xFFFFFFFE


class FFError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


class ff_config(ctypes.Structure):
    _fields_ = [("scale", ctypes.c_float), ("threshold", ctypes.c_float), ("color", ctypes.c_int),
                ("leaves_max", ctypes.c_uint32), ("branches_max", ctypes.c_uint32),
                ("pool_bytes", ctypes.c_uint64), ("device", ctypes.c_int), ("storage", ctypes.c_int),
                ("rcp_mode", ctypes.c_int)]


class ff_stats(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("offset", ctypes.c_float * 3), ("leaves_used", ctypes.c_uint32),
                ("leaves_max", ctypes.c_uint32), ("branches_used", ctypes.c_uint32),
                ("branches_max", ctypes.c_uint32), ("queued", ctypes.c_uint32), ("frames", ctypes.c_uint32),
                ("meshing_ok", ctypes.c_uint32), ("grows", ctypes.c_uint32), ("mesh_vertices", ctypes.c_uint64),
                ("mesh_faces", ctypes.c_uint64), ("mesh_cells", ctypes.c_uint64),
                ("mesh_cells_dirty", ctypes.c_uint64), ("processed_pixels", ctypes.c_uint32),
                ("new_leaves", ctypes.c_uint32), ("dedupe_rounds", ctypes.c_uint32),
                ("graph_replays", ctypes.c_uint32), ("update_batch", ctypes.c_uint32),
                ("fused_bricks", ctypes.c_uint64), ("fused_frame_bricks", ctypes.c_uint64),
                ("mesh_cells_generated", ctypes.c_uint64), ("mesh_top_kept", ctypes.c_uint32)]


class ff_tuning(ctypes.Structure):
    _fields_ = [("dedupe_rows", ctypes.c_int), ("fuse_shape", ctypes.c_int), ("fuse_blocks_per_sm", ctypes.c_int),
                ("insert_block", ctypes.c_int), ("graph", ctypes.c_int)]


# Every entry point of include/fastfusion_b200.h with its ctypes signature.
_vp, _i32, _u32, _u64, _f32, _sz = (ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64,
                                    ctypes.c_float, ctypes.c_size_t)
SIGNATURES = {
    "ff_create": (_i32, [ctypes.POINTER(ff_config), ctypes.POINTER(_vp)]),
    "ff_destroy": (_i32, [_vp]),
    "ff_set_stream": (_i32, [_vp, _vp]),
    "ff_sync": (_i32, [_vp]),
    "ff_set_tuning": (_i32, [_vp, ctypes.POINTER(ff_tuning)]),
    "ff_set_shard": (_i32, [_vp, _i32, _i32]),
    "ff_set_spin_limit": (_i32, [_vp, _u32]),
    "ff_set_cell_generation": (_i32, [_vp, _i32]),
    "ff_get_mesh_async": (_i32, [_vp, _vp, _vp, _vp]),
    "ff_mesh_wait": (_i32, [_vp]),
    "ff_set_update_batch": (_i32, [_vp, _i32]),
    "ff_halo_export": (_i32, [_vp, _vp, _u64, ctypes.POINTER(_u64), ctypes.POINTER(_u64)]),
    "ff_halo_import": (_i32, [_vp, _vp, _u64]),
    "ff_loop_begin": (_i32, [_vp, _u32]),
    "ff_loop_delete_frame": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32, _i32, _vp, _vp, _vp, _vp, _u32,
                                    ctypes.POINTER(_i32)]),
    "ff_loop_get": (_i32, [_vp, ctypes.POINTER(_u32), _vp, _vp, _vp, _vp]),
    "ff_inject_error": (_i32, [_vp, _i32]),
    "ff_add_map_u16": (_i32, [_vp, _vp, _i32, _i32, _sz, _vp, _sz, _vp, _vp, _vp, _f32, _f32, _vp]),
    "ff_add_map_u16_device": (_i32, [_vp, _vp, _vp, _i32, _i32, _vp, _vp, _vp, _f32, _f32, _vp]),
    "ff_add_maps_u16_device": (_i32, [_vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ff_add_map_sequence_u16_device": (_i32, [_vp, _i32, _vp, _vp, _i32, _i32, _vp, _vp, _vp, _f32, _f32, _vp]),
    "ff_add_map_sequence_u16": (_i32, [_vp, _i32, _vp, _vp, _i32, _i32, _sz, _sz, _vp, _vp, _vp, _f32, _f32, _vp]),
    "ff_update_meshes": (_i32, [_vp, _vp]),
    "ff_get_mesh_counts": (_i32, [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64)]),
    "ff_get_mesh": (_i32, [_vp, _vp, _vp, _vp]),
    "ff_get_mesh_device": (_i32, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "ff_get_mesh_cells": (_i32, [_vp, _vp, _vp]),
    "ff_get_mesh_cells_noalloc": (_i32, [_vp, _vp, _vp]),
    "ff_alloc_host": (_i32, [_sz, ctypes.POINTER(_vp)]),
    "ff_free_host": (_i32, [_vp]),
    "ff_get_stats": (_i32, [_vp, ctypes.POINTER(ff_stats)]),
    "ff_get_leaves": (_i32, [_vp, _vp, _vp, _vp]),
    "ff_get_queue": (_i32, [_vp, _vp]),
    "ff_get_bricks": (_i32, [_vp, _u32, _u32, _vp, _vp, _vp]),
    "ff_set_bricks": (_i32, [_vp, _u32, _u32, _vp, _vp, _vp]),
    "ff_get_tree": (_i32, [_vp, _vp]),
    "ff_set_state": (_i32, [_vp, _u32, _vp, _vp, _u32, _vp, _vp, _vp, _u32, _vp, _vp, _vp]),
    "ff_profile": (_i32, [_vp, _i32]),
    "ff_kernel_launches": (_i32, [ctypes.POINTER(_u64), ctypes.POINTER(_u64)]),
    "ff_profile_read": (_i32, [_vp, _vp, _vp, _vp]),
    "ff_set_confidence": (_i32, [_vp, _vp, _i32, _f32]),
    "ff_get_confidence_map": (_i32, [_vp, _vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
    "ff_raycast_depth": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32, _i32, _f32, _f32, _f32, _vp]),
    "ff_cnn_features": (_i32, [_vp, _i32, _i32, _i32, _f32, _vp, _vp, _vp]),
    "ff_cnn_forward": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp, _f32, _vp]),
    "ff_cnn_backward": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp]),
    "ff_cnn_mse": (_i32, [_vp, _vp, ctypes.c_int64, _f32, _vp, _vp, _vp]),
    "ff_cnn_adam": (_i32, [_vp, _vp, _vp, _vp, _vp, _f32, _f32, _f32, _f32, _i32, _vp]),
    "ff_last_error": (ctypes.c_char_p, [_vp]),
    "ff_version": (ctypes.c_char_p, []),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libfastfusion_b200.so (raises if it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise FFError(7, f"{path} is missing; build it with `python -m fastfusion_b200.build`")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class CameraInfo:
    """Pinhole intrinsics plus camera-to-world pose, the reference's CameraInfo
    (src/camerautils/camerautils.hpp:22-56) reduced to what addMap reads."""

    def __init__(self, K, R, t):
        K = np.asarray(K, dtype=np.float64)
        if K.shape == (3, 3):
            K = np.array([K[0, 0], K[1, 1], K[0, 2], K[1, 2]])
        self.K = np.ascontiguousarray(K, dtype=np.float64).reshape(4)
        self.R = np.ascontiguousarray(R, dtype=np.float64).reshape(3, 3)
        self.t = np.ascontiguousarray(t, dtype=np.float64).reshape(3)
        # addresses for the C calls (the arrays live as long as this object)
        self._ptrs = (self.K.ctypes.data, self.R.ctypes.data, self.t.ctypes.data)

    def getIntrinsic(self):
        fx, fy, cx, cy = self.K
        return np.array([[fx, 0, cx], [0, fy, cy], [0, 0, 1.0]])

    def getRotation(self):
        return self.R.copy()

    def getTranslation(self):
        return self.t.reshape(3, 1).copy()


@dataclasses.dataclass
class MeshInterleaved:
    """The reference's MeshInterleaved (mesh_interleaved.hpp:35-69): vertices
    in world metres, one colour per vertex, triangles as vertex indices."""
    vertices: np.ndarray  # (nv, 3) float32
    colors: np.ndarray    # (nv, 3) uint8 (r, g, b)
    faces: np.ndarray     # (nf, 3) uint32

    def writePLY(self, filename: str, binary: bool = True) -> bool:
        """Write `filename` + ".ply" byte for byte as the reference's
        MeshInterleaved::writePLY (mesh_interleaved.cpp:137-198): a header
        with float32 x/y/z, uchar red/green/blue (when there are colours) and
        a uint8/int32 face list, then the vertices (position and colour
        interleaved) and the faces; ascii numbers as C++ streams print them
        (%g with 6 significant digits)."""
        v = np.ascontiguousarray(self.vertices, np.float32).reshape(-1, 3)
        c = np.ascontiguousarray(self.colors, np.uint8).reshape(-1, 3)
        f = np.ascontiguousarray(self.faces, np.uint32).reshape(-1, 3)
        head = ["ply", "format binary_little_endian 1.0" if binary else "format ascii 1.0",
                f"element vertex {len(v)}", "property float32 x\nproperty float32 y\nproperty float32 z"]
        if len(c):
            head.append("property uchar red\nproperty uchar green\nproperty uchar blue")
        if len(f):
            head.append(f"element face {len(f)}")
            head.append("property list uint8 int32 vertex_indices")
        head.append("end_header")
        try:
            out = open(filename + ".ply", "wb")
        except OSError:
            return False
        with out:
            out.write("\n".join(head).encode())
            if binary:
                out.write(b"\n")
                if len(c):
                    rec = np.zeros(len(v), dtype=[("p", "<f4", 3), ("c", "u1", 3)])
                    rec["c"] = c
                else:
                    rec = np.zeros(len(v), dtype=[("p", "<f4", 3)])
                rec["p"] = v
                out.write(rec.tobytes())
                frec = np.zeros(len(f), dtype=[("n", "u1"), ("i", "<u4", 3)])
                frec["n"] = 3
                frec["i"] = f
                out.write(frec.tobytes())
            else:
                lines = []
                for k in range(len(v)):
                    s = "\n%g %g %g" % (float(v[k, 0]), float(v[k, 1]), float(v[k, 2]))
                    if len(c):
                        s += " %d %d %d" % (c[k, 0], c[k, 1], c[k, 2])
                    lines.append(s)
                for k in range(len(f)):
                    lines.append("\n3 %d %d %d" % (f[k, 0], f[k, 1], f[k, 2]))
                out.write("".join(lines).encode())
        return True

    def writeOBJ(self, filename: str) -> bool:
        """Write `filename` + ".obj" byte for byte as the reference's
        MeshInterleaved::writeOBJ (mesh_interleaved.cpp:19-134) writes a mesh
        without normals or textures (the marching-cubes mesh has neither): a
        comment line, one `v x y z r g b` line per vertex with the colour as
        float32 channel / 255, then one `f` line per triangle with 1-based
        vertex indices; numbers as C++ streams print them (%g, 6 significant
        digits).  No material file is written without textures."""
        v = np.ascontiguousarray(self.vertices, np.float32).reshape(-1, 3)
        c = np.ascontiguousarray(self.colors, np.uint8).reshape(-1, 3)
        f = np.ascontiguousarray(self.faces, np.uint32).reshape(-1, 3)
        try:
            out = open(filename + ".obj", "wb")
        except OSError:
            return False
        lines = ["\n#Written from Volume"]
        cf = (c.astype(np.float32) / np.float32(255.0)) if len(c) else None
        for k in range(len(v)):
            s = "\nv %g %g %g" % (float(v[k, 0]), float(v[k, 1]), float(v[k, 2]))
            if cf is not None:
                s += " %g %g %g" % (float(cf[k, 0]), float(cf[k, 1]), float(cf[k, 2]))
            lines.append(s)
        f1 = f.astype(np.int64) + 1
        lines.extend("\nf %d %d %d" % (a, b, d) for a, b, d in f1.tolist())
        with out:
            out.write("".join(lines).encode())
        return True


class MeshBuffer:
    """Reusable page-locked host storage for getMeshInterleavedMarchingCubes(out=...).

    The mesh is copied from the device straight into this memory; the arrays
    of the returned MeshInterleaved are views of it, valid until the buffer is
    filled again (copy them to keep a mesh)."""

    def __init__(self, n_vertices: int = 0, n_faces: int = 0):
        self._L = load_library()
        self._ptr = {}
        self._cap = {"xyz": 0, "rgb": 0, "faces": 0}
        self.reserve(n_vertices, n_faces)

    def _grow(self, key: str, nbytes: int):
        if nbytes <= self._cap[key]:
            return
        # page-locking is slow, so grow in large steps
        nbytes = max(nbytes, 2 * self._cap[key], 1 << 16)
        p = ctypes.c_void_p()
        st = self._L.ff_alloc_host(nbytes, ctypes.byref(p))
        if st != FF_OK:
            raise FFError(st, f"ff_alloc_host({nbytes}) failed")
        old = self._ptr.get(key)
        if old:
            self._L.ff_free_host(old)
        self._ptr[key] = p.value
        self._cap[key] = nbytes

    def needs(self, n_vertices: int, n_faces: int) -> bool:
        """Whether a mesh of this size makes the buffer grow (and replace its memory)."""
        return 12 * n_vertices > self._cap["xyz"] or 3 * n_vertices > self._cap["rgb"] or \
            12 * n_faces > self._cap["faces"]

    def reserve(self, n_vertices: int, n_faces: int):
        self._grow("xyz", 12 * n_vertices)
        self._grow("rgb", 3 * n_vertices)
        self._grow("faces", 12 * n_faces)

    def view(self, key: str, dtype, shape):
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        if n == 0:
            return np.zeros(shape, dtype)
        buf = (ctypes.c_char * n).from_address(self._ptr[key])
        return np.frombuffer(buf, dtype=dtype).reshape(shape)

    def pointers(self):
        return [ctypes.c_void_p(self._ptr.get(k)) for k in ("xyz", "rgb", "faces")]

    def close(self):
        for p in self._ptr.values():
            if p:
                self._L.ff_free_host(p)
        self._ptr = {}
        self._cap = {"xyz": 0, "rgb": 0, "faces": 0}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FusionMipMapCPU:
    """Drop-in for the reference's FusionMipMapCPU on one B200."""

    def __init__(self, offsetX: float = 0.0, offsetY: float = 0.0, offsetZ: float = 0.0, scale: float = 0.005,
                 distanceThreshold: float = 0.01, n: int = 0, color: bool = True, *, leaves_max: int = 0,
                 branches_max: int = 0, pool_bytes: int = 0, device: int = 0, storage: str = "fp32",
                 rcp: str = "host"):
        # The reference ignores the offset and n arguments (its constructor
        # passes 0,0,0 and n=0 to the base class, geometryfusion_mipmap_cpu.cpp:420-424).
        self._L = load_library()
        cfg = ff_config(scale=scale, threshold=distanceThreshold, color=1 if color else 0,
                        leaves_max=leaves_max, branches_max=branches_max, pool_bytes=pool_bytes,
                        device=device, storage=STORAGE[storage], rcp_mode=RCP[rcp])
        h = ctypes.c_void_p()
        st = self._L.ff_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != FF_OK:
            raise FFError(st, self._L.ff_last_error(None).decode())
        self._h = h
        self.storage = storage
        self._q = ctypes.c_int32()
        self._qref = ctypes.byref(self._q)
        self._u = ctypes.c_int()
        self._uref = ctypes.byref(self._u)

    # -- lifetime --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.ff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != FF_OK:
            raise FFError(st, self._L.ff_last_error(self._h).decode())

    # -- the reference's API ----------------------------------------------
    def addMap(self, depth: np.ndarray, caminfo: CameraInfo, rgb: np.ndarray, scaling: float = 1.0 / 5000.0,
               maxcamdistance: float = 10.0) -> int:
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
        if depth.ndim != 2 or rgb.shape != depth.shape + (3,):
            raise FFError(1, "addMap: depth must be HxW uint16 and rgb HxWx3 uint8")
        h, w = depth.shape
        pK, pR, pt = caminfo._ptrs
        st = self._L.ff_add_map_u16(self._h, depth.ctypes.data, w, h, 0, rgb.ctypes.data, 0, pK, pR, pt, scaling,
                                    maxcamdistance, self._qref)
        if st != FF_OK:
            self._check(st)
        return self._q.value

    def addMapDevice(self, d_depth: int, d_bgr: int, width: int, height: int, caminfo: CameraInfo,
                     scaling: float = 1.0 / 5000.0, maxcamdistance: float = 10.0) -> int:
        """addMap with depth/bgr already in device memory (raw device pointers).
        Returns once the frame's bricks are counted; the images must stay
        unchanged until the next call on this map returns or sync()."""
        pK, pR, pt = caminfo._ptrs
        st = self._L.ff_add_map_u16_device(self._h, d_depth, d_bgr, width, height, pK, pR, pt, scaling,
                                           maxcamdistance, self._qref)
        if st != FF_OK:
            self._check(st)
        return self._q.value

    def addMapSequence(self, depths, cams, rgbs, scaling: float = 1.0 / 5000.0,
                       maxcamdistance: float = 10.0) -> list:
        """Several host frames in one call (ff_add_map_sequence_u16): the
        reference's addMap(std::vector<cv::Mat> depthImages,
        std::vector<CameraInfo>, std::vector<cv::Mat> rgbImages), which adds
        them one after another.  depths: HxW uint16 arrays, rgbs: HxWx3 uint8
        BGR arrays, cams: CameraInfo objects; returns each frame's queued
        count.  The same results as addMap frame by frame."""
        n = len(cams)
        if n == 0 or len(depths) != n or len(rgbs) != n:
            raise FFError(1, "addMapSequence: as many depth and colour images as cameras")
        depths = [np.ascontiguousarray(d, dtype=np.uint16) for d in depths]
        rgbs = [np.ascontiguousarray(c, dtype=np.uint8) for c in rgbs]
        h, w = depths[0].shape
        if any(d.shape != (h, w) for d in depths) or any(c.shape != (h, w, 3) for c in rgbs):
            raise FFError(1, "addMapSequence: every depth HxW uint16 and every rgb HxWx3 uint8, one size")
        dp = (ctypes.c_void_p * n)(*[d.ctypes.data for d in depths])
        bp = (ctypes.c_void_p * n)(*[c.ctypes.data for c in rgbs])
        K = np.ascontiguousarray(np.stack([c.K for c in cams]), np.float64)
        R = np.ascontiguousarray(np.stack([c.R.reshape(9) for c in cams]), np.float64)
        t = np.ascontiguousarray(np.stack([c.t for c in cams]), np.float64)
        q = np.zeros(n, np.int32)
        st = self._L.ff_add_map_sequence_u16(self._h, n, dp, bp, w, h, 0, 0, _p(K), _p(R), _p(t), scaling,
                                             maxcamdistance, _p(q))
        self._check(st)
        return [int(x) for x in q]

    def addMapSequenceDevice(self, d_depth, d_bgr, width: int, height: int, cams, scaling: float = 1.0 / 5000.0,
                             maxcamdistance: float = 10.0) -> list:
        """Several frames of this map in one call (ff_add_map_sequence_u16_device):
        d_depth/d_bgr are sequences of device pointers, cams CameraInfo
        objects; returns each frame's queued count.  Same results as
        addMapDevice frame by frame; the images are free when it returns."""
        n = len(cams)
        dd = (ctypes.c_void_p * n)(*[int(p) for p in d_depth])
        db = (ctypes.c_void_p * n)(*[int(p) for p in d_bgr])
        K = np.ascontiguousarray(np.stack([c.K for c in cams]), np.float64)
        R = np.ascontiguousarray(np.stack([c.R.reshape(9) for c in cams]), np.float64)
        t = np.ascontiguousarray(np.stack([c.t for c in cams]), np.float64)
        q = np.zeros(n, np.int32)
        st = self._L.ff_add_map_sequence_u16_device(self._h, n, dd, db, width, height, _p(K), _p(R), _p(t),
                                                    scaling, maxcamdistance, _p(q))
        if st != FF_OK:
            self._check(st)
        return [int(x) for x in q]

    def updateMeshes(self) -> bool:
        st = self._L.ff_update_meshes(self._h, self._uref)
        if st != FF_OK:
            self._check(st)
        return bool(self._u.value)

    def getMeshInterleavedMarchingCubes(self, out: MeshBuffer | None = None, wait: bool = True) -> MeshInterleaved:
        """The mesh of the last updateMeshes as a host copy (the reference
        returns its mesh by value).  With `out`, the copy lands in that
        reusable page-locked buffer and the returned arrays are views of it;
        with wait=False as well, the copy runs behind the map's device work
        and the call returns at once: the arrays hold the mesh after
        mesh_wait() (ff_get_mesh_async), and meanwhile the next frames can be
        issued."""
        nv, nf = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self._L.ff_get_mesh_counts(self._h, ctypes.byref(nv), ctypes.byref(nf)))
        if out is not None:
            if out.needs(nv.value, nf.value):
                self.mesh_wait()  # (a copy into the buffer about to be replaced)
            out.reserve(nv.value, nf.value)
            if wait:
                self.mesh_wait()
                self._check(self._L.ff_get_mesh(self._h, *out.pointers()))
            else:
                self._check(self._L.ff_get_mesh_async(self._h, *out.pointers()))
            return MeshInterleaved(out.view("xyz", np.float32, (nv.value, 3)), out.view("rgb", np.uint8, (nv.value, 3)),
                                   out.view("faces", np.uint32, (nf.value, 3)))
        xyz = np.zeros((nv.value, 3), np.float32)
        rgb = np.zeros((nv.value, 3), np.uint8)
        faces = np.zeros((nf.value, 3), np.uint32)
        self._check(self._L.ff_get_mesh(self._h, _p(xyz), _p(rgb), _p(faces)))
        return MeshInterleaved(xyz, rgb, faces)

    def mesh_wait(self):
        """Wait for the copy of the last getMeshInterleavedMarchingCubes(wait=False)."""
        self._check(self._L.ff_mesh_wait(self._h))

    def mesh_cells(self):
        """(cells int32[n,14], ranges int64[n,4]) of the last updateMeshes."""
        n = self.stats()["mesh_cells"]
        cells = np.zeros((n, 14), np.int32)
        ranges = np.zeros((n, 4), np.int64)
        self._check(self._L.ff_get_mesh_cells(self._h, _p(cells), _p(ranges)))
        return cells, ranges

    def mesh_cells_noalloc(self):
        """mesh_cells() without device allocation: staged in the library's
        fixed device buffer (at most NOALLOC_MAX_CELLS cells; calls on one
        device must not overlap on the GPU)."""
        n = self.stats()["mesh_cells"]
        cells = np.zeros((n, 14), np.int32)
        ranges = np.zeros((n, 4), np.int64)
        self._check(self._L.ff_get_mesh_cells_noalloc(self._h, _p(cells), _p(ranges)))
        return cells, ranges

    def setThreadMeshing(self, threadMeshing: bool):
        """Meshing runs on the GPU stream; there is no mesher thread."""

    def setIncrementalMeshing(self, incrementalMeshing: bool):
        """Meshing is always incremental (dirty cells only)."""

    def setDepthChecks(self, depthchecks: int):
        """A no-op in the reference too (its code is commented out)."""

    def set_tuning(self, dedupe_rows: int = 0, fuse_shape: int = 0, fuse_blocks_per_sm: int = 0,
                   insert_block: int = 0, graph: bool = False):
        """Launch shapes of the calls this map leads (ff_tuning; 0 = default)."""
        t = ff_tuning(dedupe_rows, fuse_shape, fuse_blocks_per_sm, insert_block, 1 if graph else 0)
        self._check(self._L.ff_set_tuning(self._h, ctypes.byref(t)))

    def set_shard(self, shard: int, shards: int):
        """Make this map part `shard` of `shards` of a larger map (brick
        ownership by a hash of each brick's key); before the first frame."""
        self._check(self._L.ff_set_shard(self._h, int(shard), int(shards)))

    def set_update_batch(self, frames: int = 16):
        """Frames whose voxel update waits for one pass over their bricks
        (1 = every frame updated by itself); results are the same either way."""
        self._check(self._L.ff_set_update_batch(self._h, int(frames)))

    def set_spin_limit(self, iterations: int = SPIN_LIMIT_DEFAULT):
        """Bound of the device-side waits of this map's frames and mesh
        updates (polling iterations; 0: a wait gives up at once and the call
        reports FF_ERR_TIMEOUT)."""
        self._check(self._L.ff_set_spin_limit(self._h, int(iterations)))

    def set_cell_generation(self, mode: int = CELLS_INCREMENTAL):
        """How updateMeshes finds the mesh cells: CELLS_INCREMENTAL (only the
        octree parts that changed since the previous update are traversed;
        the other cells are kept) or CELLS_FULL (the whole octree every
        update).  The cell list is the same either way."""
        self._check(self._L.ff_set_cell_generation(self._h, int(mode)))

    def inject_error(self, what: int = INJECT_CONFIDENCE_TIMEOUT):
        """Make the next frame report a failure as the device would (tests of
        the error paths; 0 cancels)."""
        self._check(self._L.ff_inject_error(self._h, int(what)))

    # -- loop closure: removing fused frames (deleteOldLoopPoses) ------------
    def loop_begin(self, capacity: int = 100000):
        """Zeroed loop arrays for `capacity` bricks, no brick mapped."""
        self._check(self._L.ff_loop_begin(self._h, int(capacity)))

    def loop_delete_frame(self, d_depth: int, d_red: int, d_green: int, d_blue: int, width: int, height: int,
                          caminfo: CameraInfo, d_queue: int, n_queue: int) -> bool:
        """One fused frame's removal into the loop arrays (device pointers:
        depth float metres with NaN holes, colour planes, the frame's queued
        leaves); False when the slots ran out."""
        pK, pR, pt = caminfo._ptrs
        done = ctypes.c_int()
        self._check(self._L.ff_loop_delete_frame(self._h, int(d_depth), int(d_red), int(d_green), int(d_blue),
                                                 int(width), int(height), pK, pR, pt, int(d_queue), int(n_queue),
                                                 ctypes.byref(done)))
        return bool(done.value)

    def loop_arrays(self):
        """(leaf -> slot uint32[leaves], sdf float[n,512], weight float[n,512],
        colour uint16[n,512,3]) of the slots in use."""
        n = ctypes.c_uint32()
        self._check(self._L.ff_loop_get(self._h, ctypes.byref(n), None, None, None, None))
        nl = min(self.stats()["leaves_used"], self.stats()["leaves_max"])
        m = np.zeros(nl, np.uint32)
        d = np.zeros((n.value, 512), np.float32)
        w = np.zeros((n.value, 512), np.float32)
        c = np.zeros((n.value, 512, 3), np.uint16)
        self._check(self._L.ff_loop_get(self._h, ctypes.byref(n), _p(m), _p(d), _p(w), _p(c)))
        return m, d, w, c

    def halo_count(self) -> tuple[int, int]:
        """(records, bytes per record) the next halo export would write."""
        n, rb = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self._L.ff_halo_export(self._h, None, 0, ctypes.byref(n), ctypes.byref(rb)))
        return n.value, rb.value

    def halo_export(self, d_records: int, capacity: int) -> int:
        """Write this part's changed bricks as records to device memory
        d_records (room for `capacity`); returns the number written."""
        n, rb = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self._L.ff_halo_export(self._h, ctypes.c_void_p(int(d_records)), int(capacity),
                                           ctypes.byref(n), ctypes.byref(rb)))
        return n.value

    def halo_import(self, d_records: int, n_records: int):
        """Write another part's records (device memory) into this part's pool."""
        self._check(self._L.ff_halo_import(self._h, ctypes.c_void_p(int(d_records)), int(n_records)))

    def sync(self):
        """Wait for the map's outstanding device work (the last voxel update)."""
        self._check(self._L.ff_sync(self._h))

    def set_stream(self, stream_ptr: int | None):
        self._check(self._L.ff_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)))

    # -- profiling ----------------------------------------------------------
    PROFILE_STAGES = ("grow", "dedupe", "insert", "finalize", "fuse", "mesh_cells", "mesh_count", "mesh_emit",
                      "confidence")

    def set_confidence(self, params, tau_m: float = 0.03):
        """Learned per-pixel weight: the network's FF_CNN_PARAMS parameters
        (rounded to BF16 by the library) and the residual tau (m) at which a
        pixel's weight reaches zero; None turns it off (the reference's
        weight)."""
        if params is None:
            self._check(self._L.ff_set_confidence(self._h, None, 0, 0.0))
            return
        p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
        self._check(self._L.ff_set_confidence(self._h, _p(p), int(p.size), float(tau_m)))

    def confidence_map(self) -> np.ndarray:
        """The last frame's per-pixel confidence (H x W float32)."""
        w, h = _i32(0), _i32(0)
        self._check(self._L.ff_get_confidence_map(self._h, None, ctypes.byref(w), ctypes.byref(h)))
        out = np.empty((h.value, w.value), np.float32)
        self._check(self._L.ff_get_confidence_map(self._h, _p(out), None, None))
        return out

    def raycast_depth(self, d_depth: int, width: int, height: int, caminfo: CameraInfo, d_out: int,
                      scaling: float = 1.0 / 5000.0, window_m: float = 0.15, step_m: float = 0.0025):
        """Depth of the fused surface along each pixel's ray near its measured
        depth (device pointers: uint16 depth in, float metres out; 0 = no
        depth, -1 = no surface within the window)."""
        pK, pR, pt = caminfo._ptrs
        self._check(self._L.ff_raycast_depth(self._h, pK, pR, pt, int(d_depth), int(width), int(height),
                                             float(scaling), float(window_m), float(step_m), int(d_out)))

    def profile(self, enable: bool = True):
        """Reset the per-stage CUDA-event profile and switch it on or off."""
        self._check(self._L.ff_profile(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        """{stage: (milliseconds, algorithmic bytes, launches)} summed since profile()."""
        k = len(self.PROFILE_STAGES)
        ms = np.zeros(k, np.float64)
        by = np.zeros(k, np.float64)
        n = np.zeros(k, np.uint64)
        self._check(self._L.ff_profile_read(self._h, _p(ms), _p(by), _p(n)))
        return {name: (float(ms[i]), float(by[i]), int(n[i])) for i, name in enumerate(self.PROFILE_STAGES)}

    # -- inspection ---------------------------------------------------------
    def stats(self) -> dict:
        s = ff_stats()
        self._check(self._L.ff_get_stats(self._h, ctypes.byref(s)))
        d = {f: getattr(s, f) for f, _ in ff_stats._fields_}
        d["offset"] = np.array(list(s.offset), np.float32)
        return d

    def leaves(self):
        st = self.stats()
        n = min(st["leaves_used"], st["leaves_max"])
        pos = np.zeros((n, 3), np.uint16)
        scl = np.zeros(n, np.uint16)
        par = np.zeros(n, np.uint32)
        self._check(self._L.ff_get_leaves(self._h, _p(pos), _p(scl), _p(par)))
        return pos, scl, par

    def queue(self) -> np.ndarray:
        q = np.zeros(self.stats()["queued"], np.uint32)
        self._check(self._L.ff_get_queue(self._h, _p(q)))
        return q

    def tree(self) -> np.ndarray:
        t = np.zeros(self.stats()["branches_used"], np.uint32)
        self._check(self._L.ff_get_tree(self._h, _p(t)))
        return t

    def bricks(self, first: int = 0, count: int | None = None):
        st = self.stats()
        if count is None:
            count = min(st["leaves_used"], st["leaves_max"]) - first
        d = np.zeros((count, 512), np.float32)
        w = np.zeros((count, 512), np.float32)
        c = np.zeros((count, 512, 3), np.uint16)
        self._check(self._L.ff_get_bricks(self._h, first, count, _p(d), _p(w), _p(c)))
        return d, w, c

    def set_bricks(self, first: int, d, w, c):
        d = np.ascontiguousarray(d, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        c = np.ascontiguousarray(c, np.uint16)
        self._check(self._L.ff_set_bricks(self._h, first, d.shape[0], _p(d), _p(w), _p(c)))

    def set_state(self, n: int, offset, tree, pos, scale, parent, sdf=None, weight=None, rgb=None):
        """Snapshot restore of the whole map."""
        offset = np.ascontiguousarray(offset, np.float32)
        tree = np.ascontiguousarray(tree, np.uint32)
        pos = np.ascontiguousarray(pos, np.uint16)
        scale = np.ascontiguousarray(scale, np.uint16)
        parent = np.ascontiguousarray(parent, np.uint32)
        args = [None, None, None]
        if sdf is not None:
            args = [np.ascontiguousarray(sdf, np.float32), np.ascontiguousarray(weight, np.float32),
                    np.ascontiguousarray(rgb, np.uint16)]
        ptrs = [_p(a) if a is not None else None for a in args]
        self._check(self._L.ff_set_state(self._h, n, _p(offset), _p(tree), tree.shape[0], _p(pos), _p(scale),
                                         _p(parent), pos.shape[0], *ptrs))


    # -- snapshot / resume (the reference's copyCPU2HDD / copyHDD2CPU,
    # geometryfusion_mipmap_cpu.cpp:1135-1184, as one .npz file) ----------------
    def save_snapshot(self, path: str):
        """Write the whole map state (volume, octree, leaf table, bricks) to
        `path` (.npz).  load_snapshot on any map of enough capacity resumes it:
        further frames fuse exactly as they would have in this map."""
        st = self.stats()
        pos, scl, par = self.leaves()
        d, w, c = self.bricks()
        np.savez(path, n=np.uint32(st["n"]), offset=st["offset"], tree=self.tree(), pos=pos, scale=scl,
                 parent=par, sdf=d, weight=w, rgb=c, meshing_ok=np.uint32(st["meshing_ok"]))

    def load_snapshot(self, path: str):
        """Replace this map's state by a snapshot written by save_snapshot."""
        z = np.load(path)
        self.set_state(int(z["n"]), z["offset"], z["tree"], z["pos"], z["scale"], z["parent"], z["sdf"],
                       z["weight"], z["rgb"])


def add_maps_device(maps, d_depth, d_bgr, widths, heights, cams, scaling, maxcam) -> list:
    """One frame for each of several maps in one set of launches
    (ff_add_maps_u16_device): d_depth/d_bgr are device pointers (ints), cams
    CameraInfo objects, scaling/maxcam scalars or per-map sequences.  Returns
    each map's queued count; same results as addMapDevice on each map."""
    L = load_library()
    n = len(maps)
    sc = np.broadcast_to(np.asarray(scaling, np.float32), (n,)).copy()
    mc = np.broadcast_to(np.asarray(maxcam, np.float32), (n,)).copy()
    hs = (ctypes.c_void_p * n)(*[m._h for m in maps])
    dd = (ctypes.c_void_p * n)(*[int(p) for p in d_depth])
    db = (ctypes.c_void_p * n)(*[int(p) for p in d_bgr])
    w = np.asarray(widths, np.int32)
    h = np.asarray(heights, np.int32)
    K = np.ascontiguousarray(np.stack([c.K for c in cams]), np.float64)
    R = np.ascontiguousarray(np.stack([c.R.reshape(9) for c in cams]), np.float64)
    t = np.ascontiguousarray(np.stack([c.t for c in cams]), np.float64)
    q = np.zeros(n, np.int32)
    st = L.ff_add_maps_u16_device(hs, n, dd, db, _p(w), _p(h), _p(K), _p(R), _p(t), _p(sc), _p(mc), _p(q))
    if st != FF_OK:
        raise FFError(st, L.ff_last_error(maps[0]._h).decode())
    return [int(x) for x in q]


def version() -> str:
    return load_library().ff_version().decode()


def kernel_launches() -> tuple[int, int]:
    """(own kernel launches, CUB calls) of this process since the library loaded."""
    L = load_library()
    own, lib = ctypes.c_uint64(), ctypes.c_uint64()
    r = L.ff_kernel_launches(ctypes.byref(own), ctypes.byref(lib))
    if r:
        raise FFError(r, "ff_kernel_launches failed")
    return own.value, lib.value
