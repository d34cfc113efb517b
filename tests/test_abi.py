"""The C ABI library loads and exports every symbol include/*.h declares
(no device calls: runs without a GPU)."""
import ctypes as C
import os
import re

from paraphysicell_b200 import build, device
from paraphysicell_b200.abi import Agents, Mesh, Params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("ppc.h",):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?[\w\*\s]+?\b(ppc_\w+)\s*\(", src, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    build.ensure_built()
    L = C.CDLL(device.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 35
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert set(device.EXPORTS) <= names


def test_abi_version_and_struct_layout():
    build.ensure_built()
    L = device.lib()
    assert L.ppc_abi_version() == 1
    # field counts mirror include/ppc.h
    assert len(Agents._fields_) == 29
    assert C.sizeof(Mesh) == 40
    assert C.sizeof(Params) == 24


def test_mesh_helpers_match_reference_indexing():
    """get_mesh_index is x-fastest (reference: test/test.cpp:329-330); the
    helpers are host functions and need no device."""
    build.ensure_built()
    L = device.lib()
    m = Mesh.make(3, (0, 0, 0), (200, 200, 200))
    pos = (C.c_double * 3)(45.0, 100.0, 199.9)
    c = (C.c_int32 * 3)()
    assert L.ppc_get_mesh_position(C.byref(m), pos, c) == 0
    assert list(c) == [1, 3, 6]
    idx = C.c_int32()
    assert L.ppc_get_mesh_index(C.byref(m), c, C.byref(idx)) == 0
    assert idx.value == 1 + 7 * (3 + 7 * 6)


def test_create_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        return
    L = device.lib()
    h = C.c_void_p()
    m = Mesh.make(3, (0, 0, 0), (200, 200, 200))
    p = Params.make()
    rc = L.ppc_create(C.byref(m), C.byref(p), 10, C.byref(h))
    assert rc == 8  # PPC_ERR_NO_DEVICE: the product path never falls back to the CPU
