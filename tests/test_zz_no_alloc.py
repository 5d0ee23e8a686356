"""ff_get_mesh_cells_noalloc: the cell export for callers that cannot
allocate device memory during the call (a fixed memory budget, an allocator
they do not own, code where cudaMalloc is not allowed).  It stages the export
in the library's fixed device buffer instead of temporary allocations, so its
output must equal ff_get_mesh_cells' exactly; the buffer keeps the previous
call's contents, so two calls in a row (after different updates) are checked.

This file is collected last on purpose: a run that stops at the first failure
has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

pytestmark = pytest.mark.gpu


def _noalloc(m):
    """Call the entry point through the C ABI directly."""
    n = m.stats()["mesh_cells"]
    cells = np.full((n, 14), -7, np.int32)
    ranges = np.full((n, 4), -7, np.int64)
    st = m._L.ff_get_mesh_cells_noalloc(m._h, cells.ctypes.data_as(ctypes.c_void_p),
                                        ranges.ctypes.data_as(ctypes.c_void_p))
    return st, cells, ranges


def test_noalloc_cells_equal_allocating_export(lib_built):
    from fastfusion_b200 import fusion as ff
    K, frames = circle_frames(3, 10, 160, 120)
    m = ff.FusionMipMapCPU(0, 0, 0, 0.005, 0.01, 0, True, leaves_max=271420, branches_max=4793488, rcp="exact")
    seen = []
    for k, (depth, bgr, R, t) in enumerate(frames):
        m.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
        if k in (4, 9):
            m.updateMeshes()
            want_cells, want_ranges = m.mesh_cells()
            assert 0 < len(want_cells) <= ff.NOALLOC_MAX_CELLS
            st, cells, ranges = _noalloc(m)
            assert st == ff.FF_OK, m._L.ff_last_error(m._h)
            assert np.array_equal(cells, want_cells)
            assert np.array_equal(ranges, want_ranges)
            seen.append(len(cells))
    # the second call exported a different (larger) mesh through the same buffer
    assert seen[1] > seen[0]
    m.close()


def test_noalloc_rejects_more_cells_than_its_buffer(lib_built):
    """A mesh of more than FF_NOALLOC_MAX_CELLS cells is refused with
    FF_ERR_BAD_ARG and a message, and nothing is written to the caller's
    buffers; the allocating export still returns it."""
    from fastfusion_b200 import fusion as ff
    # a quarter turn of 1280x960 frames at 2 mm voxels: well over 65,536
    # cells (four nearly overlapping frames made 53,432)
    K, frames = circle_frames(0, 10, 1280, 960, total=40)
    m = ff.FusionMipMapCPU(0, 0, 0, 0.002, 0.004, 0, True, leaves_max=400000, branches_max=8000000, rcp="exact")
    for depth, bgr, R, t in frames:
        m.addMap(depth, ff.CameraInfo(K, R, t), bgr, SCALING, MAXCAM)
    m.updateMeshes()
    n = m.stats()["mesh_cells"]
    assert n > ff.NOALLOC_MAX_CELLS, n
    st, cells, ranges = _noalloc(m)
    assert st == 1  # FF_ERR_BAD_ARG
    assert b"cells" in m._L.ff_last_error(m._h)
    assert (cells == -7).all() and (ranges == -7).all()
    want_cells, _ = m.mesh_cells()
    assert len(want_cells) == n
    m.close()
