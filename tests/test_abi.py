"""The C ABI library loads on a CPU-only machine and exports every entry
point include/nxd.h declares; struct layouts agree with the ctypes mirror."""
import ctypes as C
import os
import re

import pytest

from nexdynipc_b200 import abi, runtime

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "nxd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(nxd_[a-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = runtime.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_default_settings():
    lib = runtime.lib()
    assert b"sm_100a" in lib.nxd_version()
    s = abi.NxdSettings()
    lib.nxd_default_settings(C.byref(s))
    d = abi.default_settings()
    for k, _ in abi.NxdSettings._fields_:
        assert getattr(s, k) == getattr(d, k), k


def test_struct_sizes():
    assert C.sizeof(abi.NxdContact) == 80
    assert C.sizeof(abi.NxdCandidates) == 96
    assert C.sizeof(abi.NxdSettings) == 144


def test_create_without_device_reports_no_device():
    # on a machine without a GPU the library must refuse, not fall back
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a GPU is present")
    from nexdynipc_b200 import scenes
    sc = scenes.cube_stack()
    with pytest.raises(runtime.NxdError) as e:
        runtime.Context(sc)
    assert e.value.status == 9
