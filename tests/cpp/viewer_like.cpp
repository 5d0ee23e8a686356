// Viewer-style use of the C++ drop-in, as a running program.
//
// Code written the way the reference's viewer drives FusionMipMapCPU (its
// fusion loop, onlinefusionviewer.cpp:910-952: addMap per frame with a
// CameraInfo pose, updateMeshes, getMeshInterleavedMarchingCubes), compiled
// against fastfusion_b200/FusionMipMapCPU.hpp in place of the reference's
// geometryfusion_mipmap_cpu.hpp, with the reference's own CameraInfo
// (camerautils.hpp) and MeshInterleaved (mesh_interleaved.hpp, whose
// writePLY writes the result).  Test program of tests/test_gpu_cpp_facade.py.
//
//   viewer_like FRAMES.bin OUT_STEM
//
// FRAMES.bin: int32 n, width, height, mesh_every; double fx, fy, cx, cy; then
// per frame double R[9] (row-major, camera to world), double t[3], uint16
// depth[height][width], uint8 bgr[height][width][3].  Prints each frame's
// addMap return value, writes OUT_STEM.ply (binary) after the last frame.
#include <camerautils.hpp>
#include <mesh_interleaved.hpp>

#include "FusionMipMapCPU.hpp"

#include <cstdio>
#include <vector>

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s FRAMES.bin OUT_STEM\n", argv[0]);
    return 2;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 3;
  int hdr[4];
  double K[4];
  if (fread(hdr, sizeof(int), 4, f) != 4 || fread(K, sizeof(double), 4, f) != 4) return 4;
  const int n = hdr[0], w = hdr[1], h = hdr[2], every = hdr[3];
  std::vector<unsigned short> depth((size_t)w * h);
  std::vector<unsigned char> bgr((size_t)w * h * 3);

  FusionMipMapCPU *fusion = new FusionMipMapCPU(0, 0, 0, 0.005f, 0.01f, 0, true);
  fusion->setThreadMeshing(false);
  fusion->setIncrementalMeshing(true);
  fusion->setDepthChecks(0);
  cv::Mat intrinsic = cv::Mat::eye(3, 3, CV_64FC1);
  intrinsic.at<double>(0, 0) = K[0];
  intrinsic.at<double>(1, 1) = K[1];
  intrinsic.at<double>(0, 2) = K[2];
  intrinsic.at<double>(1, 2) = K[3];
  for (int k = 0; k < n; k++) {
    double R[9], t[3];
    if (fread(R, sizeof(double), 9, f) != 9 || fread(t, sizeof(double), 3, f) != 3 ||
        fread(depth.data(), 2, depth.size(), f) != depth.size() || fread(bgr.data(), 1, bgr.size(), f) != bgr.size())
      return 5;
    cv::Mat rotation(3, 3, CV_64FC1), translation(3, 1, CV_64FC1);
    for (int i = 0; i < 9; i++) rotation.at<double>(i / 3, i % 3) = R[i];
    for (int i = 0; i < 3; i++) translation.at<double>(i, 0) = t[i];
    CameraInfo cam;
    cam.setIntrinsic(intrinsic);
    cam.setRotation(rotation);
    cam.setTranslation(translation);
    cv::Mat depthImage(h, w, CV_16UC1, depth.data());
    cv::Mat rgbImage(h, w, CV_8UC3, bgr.data());
    const int queued = fusion->addMap(depthImage, cam, rgbImage, 1.0f / 5000.0f, 4.0f);
    printf("%d\n", queued);
    if (k % every == every - 1 && !fusion->updateMeshes()) return 6;
  }
  fclose(f);
  MeshInterleaved mesh = fusion->getMeshInterleavedMarchingCubes();
  if (!mesh.writePLY(argv[2], true)) return 7;
  delete fusion;
  return 0;
}
