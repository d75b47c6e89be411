"""The C-ABI library loads, exports every symbol include/sph_b200.h declares, and the
host mirror of its structs has the library's layout (no GPU needed)."""
import ctypes as C
import os
import re

from sigmasph_b200 import abi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    with open(os.path.join(ROOT, "include", "sph_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sph_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_exports_every_declared_symbol():
    build.build()
    lib = C.CDLL(abi.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_layout_matches_host_mirror():
    build.build()
    L = abi.lib()
    assert L.sph_params_size() == C.sizeof(abi.SphParams)
    assert L.sph_scalars_size() == C.sizeof(abi.SphScalars)
    assert abi.params_layout_from_lib() == abi.params_layout_from_ctypes()


def test_strerror_names_every_status():
    L = abi.lib()
    for code in abi.STATUS_NAMES:
        assert L.sph_strerror(code)
