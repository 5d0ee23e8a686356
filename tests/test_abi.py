"""The C ABI library loads and exports every entry point the public header
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from fastfusion_b200 import fusion

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(ff_[a-z_0-9]+)\s*\(", src, re.M))
    return names


def test_library_exports_every_declared_symbol(lib_built):
    L = ctypes.CDLL(lib_built)
    declared = _declared()
    assert {"ff_create", "ff_add_map_u16", "ff_update_meshes", "ff_get_mesh", "ff_destroy"} <= declared
    for name in declared:
        assert hasattr(L, name), name
    # the Python binding binds exactly the declared set
    assert set(fusion.SIGNATURES) == declared


def test_version_and_errors_without_device(lib_built):
    L = fusion.load_library(lib_built)
    assert b"sm_100a" in L.ff_version()
    cfg = fusion.ff_config(scale=0.005, threshold=0.01, color=1)
    h = ctypes.c_void_p()
    assert L.ff_create(None, ctypes.byref(h)) == 1  # FF_ERR_BAD_ARG
    bad = fusion.ff_config(scale=-1.0, threshold=0.01, color=1)
    assert L.ff_create(ctypes.byref(bad), ctypes.byref(h)) == 1
    assert L.ff_destroy(None) == 1
    st = L.ff_create(ctypes.byref(cfg), ctypes.byref(h))
    if st == 0:
        L.ff_destroy(h)
    else:
        assert st == 7  # FF_ERR_NO_DEVICE on a machine without a GPU
        assert b"no CUDA device" in L.ff_last_error(None)
