"""The C++ facade (fastfusion_b200/FusionMipMapCPU.hpp) compiles against the
reference's own CameraInfo and MeshInterleaved headers and code written the
way the reference's viewer calls FusionMipMapCPU (onlinefusionviewer.cpp:
910-952): the drop-in boundary at the C++ level.  Needs the reference's
headers (present where the oracle is built); the OpenCV header is the
oracle's stand-in."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_src():
    """The reference's src/ directory, as the oracle's build recipe finds it
    (FF_REFERENCE_DIR or its default checkout); '' where it is absent."""
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "refdir"], capture_output=True, text=True)
    d = r.stdout.strip()
    return os.path.join(d, "src") if d else ""


REF_SRC = _reference_src()

VIEWER_LIKE = r'''
#include <camerautils.hpp>
#include <mesh_interleaved.hpp>
#include "FusionMipMapCPU.hpp"

// the reference viewer's per-frame use of the fusion object
int fuse_sequence(FusionMipMapCPU *fusion, const cv::Mat &depth, const cv::Mat &rgb, CameraInfo cam,
                  MeshInterleaved *out) {
  fusion->setThreadMeshing(true);
  fusion->setIncrementalMeshing(true);
  fusion->setDepthChecks(0);
  int queued = fusion->addMap(depth, cam, rgb, 1.0f / 5000.0f, 4.0f);
  if (fusion->updateMeshes()) *out = fusion->getMeshInterleavedMarchingCubes();
  return queued + (int)out->faces.size();
}

FusionMipMapCPU *make_fusion() { return new FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, true); }
'''


@pytest.mark.skipif(not REF_SRC or not os.path.isdir(os.path.join(REF_SRC, "fusion")),
                    reason="reference headers not present")
def test_facade_compiles_against_reference_types(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    src = tmp_path / "viewer_like.cpp"
    src.write_text(VIEWER_LIKE)
    cmd = [gxx, "-std=c++11", "-fsyntax-only", "-w",
           "-I", os.path.join(ROOT, "oracle", "shim"),
           "-I", os.path.join(REF_SRC, "camerautils"), "-I", os.path.join(REF_SRC, "fusion"), "-I", REF_SRC,
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "fastfusion_b200"), str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
