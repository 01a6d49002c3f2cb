"""CPU tests of the drop-in boundary: the C-ABI library loads and exports
every function include/statfem_cuda.h declares; nothing here computes."""
import ctypes
import os
import re

from statfem_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "statfem_cuda.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sfc_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_exports_every_declared_symbol():
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    names = header_functions()
    assert len(names) > 40
    for n in names:
        assert hasattr(lib, n), n


def test_python_binding_covers_the_header():
    assert sorted(api.SIGNATURES) == header_functions()


def test_context_creation_fails_cleanly_without_a_device():
    L = api.load()
    h = ctypes.c_void_p()
    rc = L.sfc_ctx_create(0, ctypes.byref(h))
    if rc == 0:  # a GPU is present: clean up
        L.sfc_ctx_destroy(h)
    else:
        assert rc < 0 and not h.value


def test_null_handles_are_rejected():
    L = api.load()
    assert L.sfc_system_create(None, 10, ctypes.byref(ctypes.c_void_p())) == -2
    assert L.sfc_solve(None, 0) == -2
    assert L.sfc_mesh_num_dofs(None) == -1
