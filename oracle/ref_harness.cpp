/*
 * C entry points over the reference's own FusionMipMapCPU, compiled from the
 * unmodified reference sources (src/fusion/*.cpp) into oracle/_ref/libffref.so.
 *
 * ORACLE INFRASTRUCTURE ONLY.  Only tests/, the smoke check and bench.py's CPU
 * baseline leg load this library, as the checker and as the timed reference
 * CPU path.  Nothing in fastfusion_b200/ links or calls it.
 *
 * The harness reads the fusion object's internal arrays (leaf table, queue,
 * brick pool, mesh cells) so the GPU path can be compared with it field by
 * field; it therefore compiles the reference header with protected members
 * opened up.  The object layout is unchanged by that.
 */
/* Standard headers first, so opening access below touches only the
 * reference's own classes. */
#include <opencv2/opencv.hpp>
#include <boost/thread.hpp>
#include <fstream>
#include <sstream>
#include <iostream>
#include <thread>
#include <tuple>
#include <xmmintrin.h>
#define protected public
#include <fusion/geometryfusion_mipmap_cpu.hpp>
#undef protected
#include <fusion/loopclosure.hpp>

#include <auxiliary/memory.hpp>
#include <fcntl.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>

/* The reference sizes its brick pool from half the physical memory, capped at
 * 2e9 bytes (geometryfusion_mipmap_cpu.cpp:497-507).  The oracle build links
 * these definitions in place of src/auxiliary/memory.cpp so a test can ask for
 * a small pool (and so force pool overflow) without touching the reference. */
static long long g_total_system_memory = 4000000000LL;
long long getTotalSystemMemory() { return g_total_system_memory; }
long long getAvailableSystemMemory() { return g_total_system_memory; }
ProcessMemoryStats getProcessMemory() {
  ProcessMemoryStats s = {0, 0, 0, 0, 0, 0, 0, 4096};
  return s;
}

extern "C" {

/* Redirect the reference's (very chatty) stderr to /dev/null, or back. */
static int g_saved_stderr = -1;
void ref_quiet(int quiet) {
  fflush(stderr);
  if (quiet && g_saved_stderr < 0) {
    g_saved_stderr = dup(2);
    int fd = open("/dev/null", O_WRONLY);
    dup2(fd, 2);
    close(fd);
  } else if (!quiet && g_saved_stderr >= 0) {
    dup2(g_saved_stderr, 2);
    close(g_saved_stderr);
    g_saved_stderr = -1;
  }
}

/* pool_bytes: the memory budget handed to the reference's sizing rule
 * (0 keeps the default: the 2e9-byte cap). */
void *ref_create(float scale, float threshold, int color, long long pool_bytes) {
  g_total_system_memory = pool_bytes > 0 ? 2 * pool_bytes : 4000000000LL;
  FusionMipMapCPU *f = new FusionMipMapCPU(0, 0, 0, scale, threshold, 0, color != 0);
  f->setThreadMeshing(false);
  return f;
}

void ref_destroy(void *h) { delete (FusionMipMapCPU *)h; }

void ref_set_incremental_meshing(void *h, int on) { ((FusionMipMapCPU *)h)->setIncrementalMeshing(on != 0); }

/* The reference's threaded meshing (setThreadMeshing(true)): updateMeshes
 * starts a mesher thread and returns false while one is still running. */
void ref_set_thread_meshing(void *h, int on) { ((FusionMipMapCPU *)h)->setThreadMeshing(on != 0); }

int ref_add_map(void *h, const uint16_t *depth, const uint8_t *bgr, int w, int hgt, const double *K4,
                const double *R9, const double *t3, float scaling, float maxcam) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  cv::Mat d(hgt, w, CV_16UC1, (void *)depth);
  cv::Mat c(hgt, w, CV_8UC3, (void *)bgr);
  CameraInfo cam;
  cv::Mat K = cv::Mat::eye(3, 3, CV_64FC1);
  K.at<double>(0, 0) = K4[0];
  K.at<double>(1, 1) = K4[1];
  K.at<double>(0, 2) = K4[2];
  K.at<double>(1, 2) = K4[3];
  cam.setIntrinsic(K);
  cv::Mat E = cv::Mat::eye(4, 4, CV_64FC1);
  for (int r = 0; r < 3; r++) {
    for (int k = 0; k < 3; k++) E.at<double>(r, k) = R9[r * 3 + k];
    E.at<double>(r, 3) = t3[r];
  }
  cam.setExtrinsic(E);
  return f->addMap(d, cam, c, scaling, maxcam);
}

/* The reference's float-depth overload, addMap(cv::Mat &, CameraInfo,
 * std::vector<cv::Mat>) (geometryfusion_mipmap_cpu.cpp:1308-1600): depth in
 * metres (any non-finite value is a hole), colour as three planes in the
 * order blue, green, red (cv::split of a BGR image). */
int ref_add_map_f32(void *h, const float *depth, const uint8_t *blue, const uint8_t *green, const uint8_t *red,
                    int w, int hgt, const double *K4, const double *R9, const double *t3) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  cv::Mat d(hgt, w, CV_32FC1, (void *)depth);
  std::vector<cv::Mat> planes;
  planes.push_back(cv::Mat(hgt, w, CV_8UC1, (void *)blue));
  planes.push_back(cv::Mat(hgt, w, CV_8UC1, (void *)green));
  planes.push_back(cv::Mat(hgt, w, CV_8UC1, (void *)red));
  CameraInfo cam;
  cv::Mat K = cv::Mat::eye(3, 3, CV_64FC1);
  K.at<double>(0, 0) = K4[0];
  K.at<double>(1, 1) = K4[1];
  K.at<double>(0, 2) = K4[2];
  K.at<double>(1, 2) = K4[3];
  cam.setIntrinsic(K);
  cv::Mat E = cv::Mat::eye(4, 4, CV_64FC1);
  for (int r = 0; r < 3; r++) {
    for (int k = 0; k < 3; k++) E.at<double>(r, k) = R9[r * 3 + k];
    E.at<double>(r, 3) = t3[r];
  }
  cam.setExtrinsic(E);
  return f->addMap(d, cam, planes);
}

int ref_update_meshes(void *h) { return ((FusionMipMapCPU *)h)->updateMeshes() ? 1 : 0; }

/* Loop closure's removal of one fused frame (deleteOldLoopPoses,
 * geometryfusion_mipmap_cpu.cpp:3933-4025): the frame's camera parameters
 * built as that function builds them (extrinsic inverse of the pose, the
 * map's offset folded in, rounded once to float), then the reference's
 * updateWrapper_deleteloop (loopclosure.cpp:232-309) over the frame's leaf
 * queue, with this object's leaf table and the caller's loop arrays: depth in
 * metres (NaN = no depth), colour planes, leaf_map (leaves -> loop slot,
 * 0xFFFFFFFE = none yet), *n_mapped slots in use of `capacity`; dist/wgt
 * float[capacity * 512], col uint16[capacity * 512][3].  Returns the
 * wrapper's result (0: the slots ran out). */
int ref_loop_delete(void *h, const float *depth, const uint8_t *red, const uint8_t *green, const uint8_t *blue, int w,
                    int hgt, const double *K4, const double *R9, const double *t3, uint32_t *queue, long long nq,
                    uint32_t *leaf_map, uint32_t *n_mapped, uint32_t capacity, float *dist, float *wgt,
                    uint16_t *col) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  CameraInfo cam;
  cv::Mat K = cv::Mat::eye(3, 3, CV_64FC1);
  K.at<double>(0, 0) = K4[0];
  K.at<double>(1, 1) = K4[1];
  K.at<double>(0, 2) = K4[2];
  K.at<double>(1, 2) = K4[3];
  cam.setIntrinsic(K);
  cv::Mat E = cv::Mat::eye(4, 4, CV_64FC1);
  for (int r = 0; r < 3; r++) {
    for (int k = 0; k < 3; k++) E.at<double>(r, k) = R9[r * 3 + k];
    E.at<double>(r, 3) = t3[r];
  }
  cam.setExtrinsic(E);
  cam.setExtrinsic(cam.getExtrinsicInverse());
  cv::Mat rot = cam.getRotation(), tr = cam.getTranslation(), in = cam.getIntrinsic();
  const double ox = f->_offset.x, oy = f->_offset.y, oz = f->_offset.z;
  camPamsFloat p(rot.at<double>(0, 0), rot.at<double>(0, 1), rot.at<double>(0, 2), rot.at<double>(1, 0),
                 rot.at<double>(1, 1), rot.at<double>(1, 2), rot.at<double>(2, 0), rot.at<double>(2, 1),
                 rot.at<double>(2, 2),
                 rot.at<double>(0, 0) * ox + rot.at<double>(0, 1) * oy + rot.at<double>(0, 2) * oz + tr.at<double>(0, 0),
                 rot.at<double>(1, 0) * ox + rot.at<double>(1, 1) * oy + rot.at<double>(1, 2) * oz + tr.at<double>(1, 0),
                 rot.at<double>(2, 0) * ox + rot.at<double>(2, 1) * oy + rot.at<double>(2, 2) * oz + tr.at<double>(2, 0),
                 in.at<double>(0, 0), in.at<double>(1, 1), in.at<double>(0, 2), in.at<double>(1, 2));
  volumetype mapped = *n_mapped;
  // updateWrapper_deleteloop returns false when the slots run out
  // (loopclosure.cpp:287) without restoring the rounding mode it switched to
  // round-toward-zero (:276; restored only at :309): the caller's mode is
  // put back here, so that the next frame's camera set-up rounds as usual
  const unsigned int caller_mode = _MM_GET_ROUNDING_MODE();
  const bool ok = updateWrapper_deleteloop(
      threadparameterLoop(depth, red, green, blue, w, hgt, p.r11, p.r12, p.r13, p.t1, p.r21, p.r22, p.r23, p.t2,
                          p.r31, p.r32, p.r33, p.t3, p.fx, p.fy, p.cx, p.cy, f->_scale, f->_distanceThreshold,
                          (volumetype *)queue, f->_leafPos, f->_leafScale, dist, wgt, (colortype3 *)col,
                          f->_brickLength),
      (size_t)nq, (volumetype *)leaf_map, (volumetype)capacity, &mapped);
  _MM_SET_ROUNDING_MODE(caller_mode);
  *n_mapped = mapped;
  return ok ? 1 : 0;
}

/* Mesh of the last finished update: counts, then copies. */
void ref_mesh_counts(void *h, long long *nv, long long *nf) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  *nv = (long long)f->_meshCurrent->vertices.size();
  *nf = (long long)f->_meshCurrent->faces.size() / 3;
}

/* The reference's own PLY writer (MeshInterleaved::writePLY) on its current
 * mesh; `stem` gets ".ply" appended by the writer. */
int ref_write_ply(void *h, const char *stem, int binary) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  return f->_meshCurrent->writePLY(std::string(stem), binary != 0) ? 1 : 0;
}

/* The reference's own OBJ writer (MeshInterleaved::writeOBJ); `stem` gets
 * ".obj" appended by the writer. */
int ref_write_obj(void *h, const char *stem) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  return f->_meshCurrent->writeOBJ(std::string(stem)) ? 1 : 0;
}

void ref_mesh_copy(void *h, float *xyz, uint8_t *rgb, uint32_t *faces) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  const MeshInterleaved &m = *f->_meshCurrent;
  for (size_t i = 0; i < m.vertices.size(); i++) {
    xyz[3 * i + 0] = m.vertices[i].x;
    xyz[3 * i + 1] = m.vertices[i].y;
    xyz[3 * i + 2] = m.vertices[i].z;
  }
  for (size_t i = 0; i < m.colors.size(); i++) {
    rgb[3 * i + 0] = m.colors[i].r;
    rgb[3 * i + 1] = m.colors[i].g;
    rgb[3 * i + 2] = m.colors[i].b;
  }
  for (size_t i = 0; i < m.faces.size(); i++) faces[i] = m.faces[i];
}

/* Scalar state: n, offset, counters. */
void ref_state(void *h, long long *ints, float *offset) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  ints[0] = f->_n;
  ints[1] = f->_nLeavesUsed;
  ints[2] = f->_nBranchesUsed;
  ints[3] = f->_nLeavesQueuedSurface;
  ints[4] = f->_nLeavesTotal;
  ints[5] = f->_nBranchesTotal;
  ints[6] = (long long)f->_meshCells.size();
  ints[7] = f->_framesAdded;
  ints[8] = f->_bandwidth;
  ints[9] = f->_performIncrementalMeshing ? 1 : 0;
  offset[0] = f->_offset.x;
  offset[1] = f->_offset.y;
  offset[2] = f->_offset.z;
}

/* Leaf table for leaves [0, n): position (3 x uint16), scale, parent leaf. */
void ref_leaves(void *h, long long n, uint16_t *pos, uint16_t *scl, uint32_t *parent) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  for (long long i = 0; i < n; i++) {
    pos[3 * i + 0] = f->_leafPos[i].x;
    pos[3 * i + 1] = f->_leafPos[i].y;
    pos[3 * i + 2] = f->_leafPos[i].z;
    scl[i] = f->_leafScale[i];
    parent[i] = (size_t)i < f->_leafParent.size() ? f->_leafParent[i] : 0xFFFFFFFFu;
  }
}

/* The queue of leaves touched by the last addMap, in the reference's order. */
void ref_queue(void *h, uint32_t *q) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  for (volumetype i = 0; i < f->_nLeavesQueuedSurface; i++) q[i] = f->_leafNumberSurface[i];
}

/* The raw octree array (first nBranchesUsed entries). */
void ref_tree(void *h, uint32_t *tree) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  for (volumetype i = 0; i < f->_nBranchesUsed; i++) tree[i] = f->_tree[i];
}

/* Brick contents of leaves [0, n): 512 SDF, 512 weights, 512x3 colour each. */
void ref_bricks(void *h, long long n, float *dist, float *wgt, uint16_t *col) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  for (long long i = 0; i < n * 512; i++) {
    dist[i] = f->_distance[i];
    wgt[i] = f->_weights[i];
    if (f->_color) {
      col[3 * i + 0] = f->_color[i].x;
      col[3 * i + 1] = f->_color[i].y;
      col[3 * i + 2] = f->_color[i].z;
    }
  }
}

/* Overwrite the brick contents of leaves [0, n) (same layout as ref_bricks),
 * e.g. with a machine-independent voxel state, before re-meshing. */
void ref_set_bricks(void *h, long long n, const float *dist, const float *wgt, const uint16_t *col) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  for (long long i = 0; i < n * 512; i++) {
    f->_distance[i] = dist[i];
    f->_weights[i] = wgt[i];
    if (f->_color) {
      f->_color[i].x = col[3 * i + 0];
      f->_color[i].y = col[3 * i + 1];
      f->_color[i].z = col[3 * i + 2];
    }
  }
}

/* Mesh cells: 14 int32 each: type, ox, oy, oz, size, has_mesh, lastLeaf[8]. */
long long ref_cells(void *h, int32_t *out) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  long long n = (long long)f->_meshCells.size();
  if (!out) return n;
  for (long long i = 0; i < n; i++) {
    const MeshCell &c = f->_meshCells[i];
    int32_t *o = out + 14 * i;
    o[0] = c.type;
    o[1] = c.ox;
    o[2] = c.oy;
    o[3] = c.oz;
    o[4] = c.size;
    o[5] = c.meshinterleaved ? (int32_t)c.meshinterleaved->vertices.size() : -1;
    for (int k = 0; k < 8; k++) o[6 + k] = (int32_t)c.lastLeaf[k];
  }
  return n;
}

/* Queue every mesh cell whose leaves are all allocated, so that the next
 * updateMeshes() re-meshes the whole map from the current voxel data. */
void ref_queue_all_cells(void *h) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  f->_meshCellIsQueuedNext->resize(f->_meshCells.size(), false);
  for (size_t j = 0; j < f->_meshCells.size(); j++) {
    if ((*f->_meshCellIsQueuedNext)[j]) continue;
    const MeshCell &c = f->_meshCells[j];
    int need = c.type == 0 ? 1 : c.type <= 3 ? 2 : c.type <= 6 ? 4 : 8;
    if (c.type > 7) continue;
    bool ok = true;
    for (int k = 0; k < need; k++) ok = ok && c.lastLeaf[k] < BRANCHINIT;
    if (!ok) continue;
    f->_meshCellQueueNext.push_back(j);
    (*f->_meshCellIsQueuedNext)[j] = true;
  }
}

/* Mesh of one cell as last meshed: counts, then copies (vertex order as the
 * reference's per-cell mesh). */
long long ref_cell_mesh(void *h, long long cell, float *xyz, uint8_t *rgb, uint32_t *faces, long long *nf) {
  FusionMipMapCPU *f = (FusionMipMapCPU *)h;
  const MeshCell &c = f->_meshCells[cell];
  if (!c.meshinterleaved) {
    if (nf) *nf = 0;
    return 0;
  }
  const MeshInterleaved &m = *c.meshinterleaved;
  if (nf) *nf = (long long)m.faces.size() / 3;
  if (xyz) {
    for (size_t i = 0; i < m.vertices.size(); i++) {
      xyz[3 * i + 0] = m.vertices[i].x;
      xyz[3 * i + 1] = m.vertices[i].y;
      xyz[3 * i + 2] = m.vertices[i].z;
      rgb[3 * i + 0] = m.colors[i].r;
      rgb[3 * i + 1] = m.colors[i].g;
      rgb[3 * i + 2] = m.colors[i].b;
    }
    for (size_t i = 0; i < m.faces.size(); i++) faces[i] = m.faces[i];
  }
  return (long long)m.vertices.size();
}

/* The marching-cubes triangle table as the reference holds it: per case, up to
 * 5 triangles of (edge-slot offsets), -1 terminated.  Used only to generate a
 * golden fixture that pins the product's own table. */
void ref_mc_offset_table(int32_t *out /* 256 x 16 */) {
  MarchingCubesIndexed mc(8, 8);
  for (int i = 0; i < 256; i++)
    for (int j = 0; j < 16; j++) out[16 * i + j] = mc.offsetTable[i][j];
}

/* The non-indexed tables: edge mask and triangle list (edge numbers) per case. */
void ref_mc_tables(int32_t *edge_mask /* 256 */, int32_t *tri /* 256 x 16 */) {
  MarchingCubesIndexed mc(8, 8);
  for (int i = 0; i < 256; i++) {
    edge_mask[i] = mc.edgeTable[i];
    for (int j = 0; j < 16; j++) tri[16 * i + j] = mc.triTable[i][j];
  }
}

}  // extern "C"
