"""GPU parity of brick allocation and voxel fusion against the oracle.

The oracle (oracle/ff_port.c) restates the reference's addMap with
round-toward-zero arithmetic; with the host CPU's RCPPS (update mode 2) it
is pinned bit-exact against the compiled reference (tests/test_oracle.py),
with exact reciprocals (mode 1) it is the host-independent target.  The CUDA
path must reproduce either exactly (rcp="host" / rcp="exact"): leaf table
(positions, scales, parents, in index order), the set of updated bricks, and
every SDF, weight and colour bit.
"""
import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames, queue_set

pytestmark = pytest.mark.gpu


def _pair(port_lib, leaves_max=271420, branches_max=4793488, storage="fp32", rcp="exact"):
    from fastfusion_b200.fusion import FusionMipMapCPU
    g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=leaves_max, branches_max=branches_max,
                        storage=storage, rcp=rcp)
    p = port_lib.PortFusion(leaves_total=leaves_max, branches_total=branches_max,
                            update_mode=1 if rcp == "exact" else 2)
    return g, p


def _cam(K, R, t):
    from fastfusion_b200.fusion import CameraInfo
    return CameraInfo(K, R, t)


def _compare_frame(g, p, check_bricks=True):
    sg, sp = g.stats(), p.state()
    assert sg["n"] == sp["n"]
    assert np.array_equal(sg["offset"], sp["offset"])
    assert sg["leaves_used"] == sp["leaves_used"]
    lg, lp = g.leaves(), p.leaves()
    for a, b, name in zip(lg, lp, ("pos", "scale", "parent")):
        assert np.array_equal(a, b), f"leaf {name} differs"
    assert sg["queued"] == sp["queued"]
    assert queue_set(g.queue()) == queue_set(p.queue())
    if check_bricks:
        dg, wg, cg = g.bricks()
        dp, wp, cp = p.bricks()
        assert np.array_equal(dg.view(np.uint32), dp.view(np.uint32)), "SDF bits differ"
        assert np.array_equal(wg.view(np.uint32), wp.view(np.uint32)), "weight bits differ"
        assert np.array_equal(cg, cp), "colour differs"


@pytest.mark.parametrize("rcp", ["exact", "host"])
@pytest.mark.parametrize("wh", [(160, 120), (640, 480)])
def test_alloc_fuse_bit_exact(lib_built, port_lib, wh, rcp):
    K, frames = circle_frames(0, 6 if wh[0] == 640 else 12, wh[0], wh[1])
    g, p = _pair(port_lib, rcp=rcp)
    for depth, bgr, R, t in frames:
        qg = g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM)
        qp = p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        assert qg == qp
        _compare_frame(g, p)


def test_grow_towards_negative_coordinates(lib_built, port_lib):
    """Frame 75 leaves the first frame's volume on the -x side: grow() adds a
    level, shifts the offset and every leaf, and that frame's update uses the
    pre-grow camera parameters, exactly like the reference."""
    K, frames = circle_frames(0, 100, 160, 120)
    g, p = _pair(port_lib)
    for k in (50, 60, 75, 0, 10, 25):
        depth, bgr, R, t = frames[k]
        assert g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        _compare_frame(g, p)
    assert g.stats()["grows"] == p.state()["grows"] == 1
    assert g.stats()["offset"][0] < -5.0


def test_pool_overflow(lib_built, port_lib):
    """A 600-brick pool overflows in the first frame; later leaves are dead
    (not stored, not queued) and meshing is switched off, like the reference."""
    K, frames = circle_frames(3, 40, 160, 120)
    g, p = _pair(port_lib, leaves_max=600, branches_max=1 << 16)
    for k in range(0, 40, 4):
        depth, bgr, R, t = frames[k]
        assert g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        _compare_frame(g, p)
    assert g.stats()["leaves_used"] > 600
    assert g.stats()["meshing_ok"] == 0


def test_edge_depths_and_size_change(lib_built, port_lib):
    """Holes, 65535 and out-of-range depth, then a change of image size."""
    K, frames = circle_frames(1, 3, 160, 120)
    g, p = _pair(port_lib)
    depth, bgr, R, t = frames[0]
    d = depth.copy()
    d[::7, ::5] = 0
    d[3, :] = 65535
    d[:, 11] = 30000
    for dd in (d, frames[1][0]):
        assert g.addMap(dd, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(dd, bgr, K, R, t, SCALING, MAXCAM)
        _compare_frame(g, p)
    K2, frames2 = circle_frames(1, 2, 96, 64)
    depth, bgr, R, t = frames2[1]
    assert g.addMap(depth, _cam(K2, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K2, R, t, SCALING, MAXCAM)
    _compare_frame(g, p)


def test_empty_frame(lib_built, port_lib):
    K, frames = circle_frames(0, 2, 160, 120)
    g, p = _pair(port_lib)
    depth, bgr, R, t = frames[0]
    z = np.zeros_like(depth)
    assert g.addMap(z, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(z, bgr, K, R, t, SCALING, MAXCAM) == 0
    assert g.stats()["n"] == p.state()["n"] == 0
    assert g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
    _compare_frame(g, p)


def test_bit_exact_with_reference_binary(lib_built):
    """rcp="host": the GPU reproduces the compiled reference itself, run on
    this host's CPU -- leaf table, updated bricks, every voxel bit."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/libffref.so not built")
    from fastfusion_b200.fusion import FusionMipMapCPU
    K, frames = circle_frames(0, 5, 640, 480)
    r = ref.RefFusion()
    st = r.state()
    g = FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=st["leaves_total"],
                        branches_max=st["branches_total"], rcp="host")
    for depth, bgr, R, t in frames:
        assert g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM) == r.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        for a, b in zip(g.leaves(), r.leaves()):
            assert np.array_equal(a, b)
        assert queue_set(g.queue()) == queue_set(r.queue())
    (dg, wg, cg), (dr, wr, cr) = g.bricks(), r.bricks()
    assert np.array_equal(dg.view(np.uint32), dr.view(np.uint32))
    assert np.array_equal(wg.view(np.uint32), wr.view(np.uint32))
    assert np.array_equal(cg, cr)


@pytest.mark.parametrize("wh", [(1280, 960), (1600, 1200)])
def test_many_new_leaves_per_frame(lib_built, port_lib, wh):
    """2 mm voxels on large frames create several thousand bricks per frame.
    1280x960 still takes the one-block leaf finalisation (pixel bitmap in
    shared memory); 1600x1200 is past its limit and takes the sort-based
    kernels.  Results stay bit-exact either way."""
    from fastfusion_b200.fusion import FusionMipMapCPU
    K, frames = circle_frames(0, 2, *wh)
    g = FusionMipMapCPU(0, 0, 0, 0.002, 0.004, 0, True, leaves_max=400000, branches_max=8000000, rcp="exact")
    p = port_lib.PortFusion(0.002, 0.004, True, leaves_total=400000, branches_total=8000000, update_mode=1)
    news = []
    for depth, bgr, R, t in frames:
        qg = g.addMap(depth, _cam(K, R, t), bgr, SCALING, MAXCAM)
        qp = p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM)
        assert qg == qp
        news.append(g.stats()["new_leaves"])
        _compare_frame(g, p)
    assert max(news) > 4096, news
