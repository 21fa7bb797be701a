"""The C-ABI library loads and exports every entry point include/aurora_b200.h declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aurora_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^AUR_API\s+[\w\s\*]+?\b(aur_\w+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def built():
    from aurora_b200 import build
    return build.build()


def test_header_declares_entry_points():
    names = declared()
    for n in ("aur_bvh_build", "aur_trace_closest", "aur_trace_occluded", "aur_render", "aur_render_adjoint",
              "aur_last_error", "aur_scene_create", "aur_scene_load_json"):
        assert n in names


def test_library_exports_every_declared_symbol(built):
    out = subprocess.run(["nm", "-D", "--defined-only", built], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (aur_\w+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing


def test_ctypes_binds_every_declared_symbol(built):
    from aurora_b200 import _abi
    assert set(declared()) == set(_abi.SIGNATURES), set(declared()) ^ set(_abi.SIGNATURES)
    L = _abi.lib()
    for n in declared():
        assert getattr(L, n) is not None
    assert L.aur_version().decode().startswith("aurora-b200")


def test_errors_without_a_device(built):
    """Without a GPU every entry point returns an error status instead of aborting."""
    import ctypes as C
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from aurora_b200 import _abi
    L = _abi.lib()
    h = C.c_void_p()
    st = L.aur_ctx_create(0, C.byref(h))
    assert st != 0
    assert L.aur_last_error()
    assert L.aur_bvh_build(None, None, 0, None, None, 0, None, C.byref(h)) == 1


def test_record_layouts():
    import ctypes as C
    from aurora_b200 import _abi
    assert C.sizeof(_abi.Ray) == 32
    assert C.sizeof(_abi.Hit) == 20
    assert C.sizeof(_abi.RenderOpts) == 48
    assert C.sizeof(_abi.RenderStats) == 136


def test_accelerator_adapter_driver_links(built):
    """The compiled AccelerationStructure adapter (aurora_b200/adapters) and its C++ driver are
    built beside the library and link against it: without arguments the driver prints its usage
    and exits 2 before touching a GPU."""
    exe = os.path.join(os.path.dirname(built), "test_gpu_accelerator")
    assert os.path.exists(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
