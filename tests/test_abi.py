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
    assert L.ppc_abi_version() == 2
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


def test_noalloc_rejects_meshes_whose_voxel_count_would_wrap():
    """ppc_bin_agents_noalloc sizes the grid in 64-bit arithmetic and checks
    each axis and the running product against its fixed scratch before any
    device call: a mesh of 2^31 um per axis (about 2^31 / 30 voxels each, a
    product far beyond 64 bits of 32-bit wrap-around) is refused, as are
    extents that overflow 32-bit arithmetic."""
    from paraphysicell_b200.abi import PPC_ERR_CAPACITY
    L = device.lib()
    L.ppc_bin_agents_noalloc.argtypes = [C.POINTER(Mesh), C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
    dummy = (C.c_int32 * 4)()
    pos = (C.c_double * 12)()
    for mins, maxs, shape in (((-2 ** 31, -2 ** 31, -2 ** 31), (2 ** 31 - 1,) * 3, (1, 1, 1)),
                              ((0, 0, 0), (2 ** 31 - 1,) * 3, (30, 30, 30)),
                              ((0, 0, 0), (2 ** 21, 2 ** 21, 2 ** 22), (1, 1, 1))):
        m = Mesh.make(3, mins, maxs, shape)
        rc = L.ppc_bin_agents_noalloc(C.byref(m), C.cast(pos, C.c_void_p), 4, C.cast(dummy, C.c_void_p),
                                      C.cast(dummy, C.c_void_p), None)
        assert rc == PPC_ERR_CAPACITY, (mins, maxs, shape, rc)


def test_mesh_index_of_an_extreme_mesh_does_not_wrap():
    """The state path's grid is sized in 64-bit arithmetic and saturated, so
    an extreme mesh cannot produce a small wrapped voxel count."""
    L = device.lib()
    m = Mesh.make(3, (-2 ** 31, 0, 0), (2 ** 31 - 1, 30, 30), (1, 30, 30))
    c = (C.c_int32 * 3)(5, 0, 0)
    idx = C.c_int32()
    assert L.ppc_get_mesh_index(C.byref(m), c, C.byref(idx)) == 0
    assert idx.value == 5
