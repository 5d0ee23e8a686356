/*
 * FusionMipMapCPU over the fastfusion_b200 C ABI: the members of the
 * reference class that its viewer and tools call (tum-vision/fastfusion
 * src/fusion/geometryfusion_mipmap_cpu.hpp:111-534), with the same
 * signatures, so that code written against the reference compiles against
 * this header instead.
 *
 * Include it where the reference's geometryfusion_mipmap_cpu.hpp was
 * included, after the reference's camerautils.hpp (CameraInfo) and
 * mesh_interleaved.hpp (MeshInterleaved), which this header uses as they are.
 * Link with -lfastfusion_b200 -lcudart.
 *
 * Behaviour the caller sees, as in the reference: errors are printed to
 * stderr and the call returns (addMap returns 0, updateMeshes false); meshing
 * is always incremental and runs on the GPU, so updateMeshes always finishes
 * the mesh before returning.
 */
#ifndef FASTFUSION_B200_FUSIONMIPMAPCPU_HPP
#define FASTFUSION_B200_FUSIONMIPMAPCPU_HPP

#include <stdint.h>
#include <stdio.h>

#include "fastfusion_b200.h"

class FusionMipMapCPU {
 public:
  /* FusionMipMapCPU(offsetX, offsetY, offsetZ, scale, distanceThreshold, n, color)
   * (geometryfusion_mipmap_cpu.cpp:420-640; the reference ignores the
   * offsets and n as well). */
  FusionMipMapCPU(float offsetX, float offsetY, float offsetZ, float scale, float distanceThreshold,
                  sidetype n = 0, bool color = true)
      : h_(0) {
    (void)offsetX;
    (void)offsetY;
    (void)offsetZ;
    (void)n;
    ff_config c;
    c.scale = scale;
    c.threshold = distanceThreshold;
    c.color = color ? 1 : 0;
    c.leaves_max = 0;
    c.branches_max = 0;
    c.pool_bytes = 0;
    c.device = 0;
    c.storage = FF_STORAGE_FP32;
    c.rcp_mode = FF_RCP_HOST;
    if (ff_create(&c, &h_) != FF_OK) {
      fprintf(stderr, "\nERROR: fastfusion_b200: %s", ff_last_error(0));
      h_ = 0;
    }
  }
  ~FusionMipMapCPU() {
    if (h_) ff_destroy(h_);
  }

  /* addMap(depth CV_16UC1, CameraInfo, rgb CV_8UC3 BGR, scaling, maxcamdistance)
   * (geometryfusion_mipmap_cpu.cpp:1603-2034): the number of bricks updated. */
  int addMap(const cv::Mat &depth, CameraInfo caminfo, const cv::Mat &rgb, float scaling, float maxcamdistance) {
    if (!h_) return 0;
    const cv::Mat K = caminfo.getIntrinsic(), R = caminfo.getRotation(), T = caminfo.getTranslation();
    const double k[4] = {K.at<double>(0, 0), K.at<double>(1, 1), K.at<double>(0, 2), K.at<double>(1, 2)};
    double r[9], t[3];
    for (int i = 0; i < 9; i++) r[i] = R.at<double>(i / 3, i % 3);
    for (int i = 0; i < 3; i++) t[i] = T.at<double>(i, 0);
    int32_t queued = 0;
    if (ff_add_map_u16(h_, (const uint16_t *)depth.data, depth.cols, depth.rows, depth.step,
                       (const uint8_t *)rgb.data, rgb.step, k, r, t, scaling, maxcamdistance, &queued) != FF_OK) {
      fprintf(stderr, "\nERROR: fastfusion_b200: %s", ff_last_error(h_));
      return 0;
    }
    return queued;
  }

  /* updateMeshes() (geometryfusion_mipmap_cpu.cpp:2884-2954). */
  bool updateMeshes() {
    int updated = 0;
    if (!h_ || ff_update_meshes(h_, &updated) != FF_OK) {
      if (h_) fprintf(stderr, "\nERROR: fastfusion_b200: %s", ff_last_error(h_));
      return false;
    }
    return updated != 0;
  }

  /* getMeshInterleavedMarchingCubes() (geometryfusion_mipmap_cpu.cpp:3359-3374):
   * a copy of the mesh of the last update. */
  MeshInterleaved getMeshInterleavedMarchingCubes(MeshInterleaved mesh = MeshInterleaved(3)) {
    mesh.vertices.clear();
    mesh.colors.clear();
    mesh.faces.clear();
    uint64_t nv = 0, nf = 0;
    if (!h_ || ff_get_mesh_counts(h_, &nv, &nf) != FF_OK) return mesh;
    mesh.vertices.resize((size_t)nv);
    mesh.colors.resize((size_t)nv, Color3b(0, 0, 0));  // Color3b has no default constructor
    mesh.faces.resize((size_t)(3 * nf));
    if (nv || nf) {
      /* Vertex3f and Color3b are packed float[3] / uchar[3] */
      if (ff_get_mesh(h_, nv ? &mesh.vertices[0].x : 0, nv ? &mesh.colors[0].r : 0, nf ? &mesh.faces[0] : 0) !=
          FF_OK)
        fprintf(stderr, "\nERROR: fastfusion_b200: %s", ff_last_error(h_));
    }
    return mesh;
  }

  /* Accepted for compatibility: meshing always runs incrementally on the GPU
   * stream, and the reference's depth checks are a no-op there too. */
  void setThreadMeshing(bool) {}
  void setIncrementalMeshing(bool) {}
  void setDepthChecks(int) {}

  /* The underlying handle, for the C ABI's other calls. */
  ff_handle *handle() { return h_; }

 private:
  FusionMipMapCPU(const FusionMipMapCPU &);
  FusionMipMapCPU &operator=(const FusionMipMapCPU &);
  ff_handle *h_;
};

#endif
