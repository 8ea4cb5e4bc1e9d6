"""The C ABI library loads and exports every function include/svp3d.h declares (CPU: no compute calls)."""
import ctypes
import os
import re

from conftest import ROOT


def declared():
    text = open(os.path.join(ROOT, "include", "svp3d.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(svp_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "svp_certify_map" in names and "svp_edge_hull_margins" in names
    assert len(names) >= 9


def test_library_exports_every_declared_symbol():
    from seq_vp_3d_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    # every declared function has a ctypes signature in the binding
    assert not [n for n in declared() if n not in _lib.SIGNATURES]


def test_version_and_error_without_gpu():
    from seq_vp_3d_b200 import _lib
    lib = _lib.load()
    assert lib.svp_version() >= 100
    buf = ctypes.create_string_buffer(64)
    assert lib.svp_last_error(buf, 64) >= 0
