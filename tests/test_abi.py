"""CPU tests of the C ABI: the library loads, exports what the header declares,
and fails with a status (not a crash) when no device is present."""
import ctypes
import os
import re

import pytest

from conftest import HAS_GPU, ROOT


def header_symbols():
    text = open(os.path.join(ROOT, "include", "gowalker.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(gw_\w+)\s*\(", text, re.M)))


def test_header_matches_binding(gw):
    from gowalker_b200 import _abi
    assert header_symbols() == sorted(_abi.EXPORTS)


def test_library_exports_every_declared_symbol(gw):
    L = gw.load()
    for name in header_symbols():
        assert hasattr(L, name), name


def test_version_and_defaults(gw):
    L = gw.load()
    assert L.gw_version() == 1
    c = gw.GwConfig()
    assert L.gw_config_default(ctypes.byref(c)) == 0
    # apps/Node2vec.cu:35-59 defaults
    assert abs(c.p - 0.5) < 1e-7 and abs(c.q - 2.0) < 1e-7 and abs(c.alpha - 0.2) < 1e-7
    assert c.maxhops == 30 and c.walkpersource == 1
    assert c.blocksize == 1024 << 20 and c.cache_size == 4 << 30
    assert L.gw_status_string(-4) == b"call out of order"


def test_bad_config_rejected_without_device(gw):
    L = gw.load()
    c = gw.default_config(algorithm=7)
    h = ctypes.c_void_p()
    assert L.gw_create(ctypes.byref(c), ctypes.byref(h)) == -1
    c = gw.default_config(p=0.0)
    assert L.gw_create(ctypes.byref(c), ctypes.byref(h)) == -1


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_create_without_device_returns_status(gw):
    L = gw.load()
    c = gw.default_config()
    h = ctypes.c_void_p()
    st = L.gw_create(ctypes.byref(c), ctypes.byref(h))
    assert st in (-2, -1)
    assert not h.value


def test_null_handle_rejected(gw):
    L = gw.load()
    assert L.gw_run(None, 0, None) == -1
    assert L.gw_destroy(None) == -1


def test_fastmod_is_exact(tmp_path):
    """The direct-computation remainder used by cooperative steps equals %."""
    import subprocess
    exe = tmp_path / "fastmod"
    subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "gowalker_b200", "csrc"),
                    "-o", str(exe), os.path.join(ROOT, "tests", "cuda", "fastmod_check.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout
