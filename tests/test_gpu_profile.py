"""Per-stage profile and launch accounting of the C ABI (ff_profile,
ff_profile_read, ff_kernel_launches) on a short fusion + meshing run."""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("batch", [16, 1])
def test_profile_counts_match_the_work(lib_built, batch):
    """batch 16: the frames' voxel updates wait for one pass at updateMeshes;
    batch 1: every frame is updated by itself."""
    from fastfusion_b200 import fusion as ff
    K, frames = circle_frames(0, 6, 160, 120)
    m = ff.FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    m.set_update_batch(batch)
    m.profile(True)
    own0, lib0 = ff.kernel_launches()
    queued = 0
    for depth, bgr, R, t in frames:
        queued += m.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
    m.updateMeshes()
    own1, lib1 = ff.kernel_launches()
    prof = m.profile_read()
    assert set(prof) == set(ff.FusionMipMapCPU.PROFILE_STAGES)
    # one launch of each per-frame stage per frame, one update pass per batch;
    # the fuse bytes are the 14,336 B of every queued FP32 brick of every frame
    for stage in ("dedupe", "insert", "finalize"):
        assert prof[stage][2] == len(frames), (stage, prof[stage])
        assert prof[stage][0] > 0.0
    assert prof["fuse"][2] == (1 if batch > 1 else len(frames))
    assert prof["fuse"][0] > 0.0
    assert prof["fuse"][1] == pytest.approx(14336.0 * queued)
    st = m.stats()
    assert st["fused_frame_bricks"] == queued
    if batch > 1:
        # the pass reads and writes each brick once: fewer than the frame-bricks
        assert 0 < st["fused_bricks"] < queued
    for stage in ("mesh_cells", "mesh_count", "mesh_emit"):
        assert prof[stage][2] == 1
    assert prof["mesh_count"][1] > 0
    st = m.stats()
    assert prof["mesh_emit"][1] >= st["mesh_vertices"] * 15 + st["mesh_faces"] * 12
    # own kernels: at least dedupe, insert, fuse per frame plus the mesher's
    assert own1 - own0 >= 3 * len(frames) + 4
    # no library kernel: the cell sort and the scans are this library's own
    assert lib1 - lib0 == 0
    # switching off: nothing more is recorded
    m.profile(False)
    depth, bgr, R, t = frames[0]
    m.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
    assert all(v[2] == 0 for v in m.profile_read().values())
    m.close()


def test_mesh_into_pinned_buffer(lib_built):
    """getMeshInterleavedMarchingCubes(out=MeshBuffer) returns the same mesh as
    the plain copy, and the buffer grows as the mesh grows."""
    from fastfusion_b200 import fusion as ff
    K, frames = circle_frames(1, 8, 160, 120)
    m = ff.FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    buf = ff.MeshBuffer(16, 16)
    sizes = []
    for k, (depth, bgr, R, t) in enumerate(frames):
        m.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
        if k % 3 == 2 or k == len(frames) - 1:
            m.updateMeshes()
            a = m.getMeshInterleavedMarchingCubes()
            b = m.getMeshInterleavedMarchingCubes(out=buf)
            assert np.array_equal(a.vertices.view(np.uint32), b.vertices.view(np.uint32))
            assert np.array_equal(a.colors, b.colors)
            assert np.array_equal(a.faces, b.faces)
            sizes.append(len(a.faces))
    assert sizes[-1] > 0
    buf.close()
    m.close()
