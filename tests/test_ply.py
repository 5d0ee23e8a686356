"""PLY and OBJ export: MeshInterleaved.writePLY must write the same bytes as the
reference's MeshInterleaved::writePLY (mesh_interleaved.cpp:137-198), binary
and ascii, for the same mesh (the compiled reference's own mesh here)."""

import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames


def _ref_mesh(ref_lib, n_frames):
    K, frames = circle_frames(0, n_frames, 160, 120)
    r = ref_lib.RefFusion()
    for depth, bgr, R, t in frames:
        r.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    r.update_meshes()
    return r


@pytest.fixture(scope="module")
def ref_lib():
    from oracle import ref
    if not ref.available():
        pytest.skip("the compiled reference (oracle/_ref/libffref.so) is not built")
    return ref


@pytest.mark.parametrize("binary", [True, False])
def test_ply_bytes_equal_reference(tmp_path, ref_lib, binary):
    from fastfusion_b200.fusion import MeshInterleaved
    r = _ref_mesh(ref_lib, 4)
    xyz, rgb, faces = r.mesh()
    assert len(faces) > 0
    ref_stem = str(tmp_path / "ref")
    ours_stem = str(tmp_path / "ours")
    assert r.write_ply(ref_stem, binary)
    assert MeshInterleaved(xyz, rgb, faces).writePLY(ours_stem, binary)
    a = open(ref_stem + ".ply", "rb").read()
    b = open(ours_stem + ".ply", "rb").read()
    assert a == b
    r.close()


def test_ply_empty_mesh(tmp_path):
    """No vertices and no faces: the header alone (no colour or face
    properties, as the reference writes it for empty arrays)."""
    from fastfusion_b200.fusion import MeshInterleaved
    m = MeshInterleaved(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint8), np.zeros((0, 3), np.uint32))
    assert m.writePLY(str(tmp_path / "empty"), True)
    want = (b"ply\nformat binary_little_endian 1.0\nelement vertex 0\n"
            b"property float32 x\nproperty float32 y\nproperty float32 z\nend_header\n")
    assert open(tmp_path / "empty.ply", "rb").read() == want


def test_obj_bytes_equal_reference(tmp_path, ref_lib):
    """OBJ export: MeshInterleaved.writeOBJ writes the same bytes as the
    reference's MeshInterleaved::writeOBJ (mesh_interleaved.cpp:19-134)."""
    from fastfusion_b200.fusion import MeshInterleaved
    r = _ref_mesh(ref_lib, 4)
    xyz, rgb, faces = r.mesh()
    assert len(faces) > 0
    assert r.write_obj(str(tmp_path / "ref"))
    assert MeshInterleaved(xyz, rgb, faces).writeOBJ(str(tmp_path / "ours"))
    a = open(tmp_path / "ref.obj", "rb").read()
    b = open(tmp_path / "ours.obj", "rb").read()
    assert a == b
    assert not (tmp_path / "ours.mtl").exists()
    r.close()


def test_obj_empty_mesh(tmp_path):
    from fastfusion_b200.fusion import MeshInterleaved
    m = MeshInterleaved(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint8), np.zeros((0, 3), np.uint32))
    assert m.writeOBJ(str(tmp_path / "empty"))
    assert open(tmp_path / "empty.obj", "rb").read() == b"\n#Written from Volume"
