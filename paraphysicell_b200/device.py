"""Python binding of libppc.so, the CUDA mechanics timestep (include/ppc.h).

`Simulation` owns one device state (one simulation, or a batch of replicate
simulations) and exposes the reference's solver entry points by name
(reference: src/solver/host/position_solver.h:7-21,
src/solver/host/containers_solver.h:13-27). Every call raises PPCError on a
non-zero status. There is no CPU fallback: without the built library or a
CUDA device the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import Agents, GradientField, Interactions, Mesh, Motility, Params, PPCError

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libppc.so")

_lib = None

ENTRY_POINTS = (
    "update_mechanics_mesh", "update_cell_neighbors", "update_cell_forces", "update_motility",
    "update_basement_membrane_interactions", "update_spring_attachments", "update_positions",
    "update_cell_container_for_mechanics", "update_cell_container_for_phenotype",
)

EXPORTS = (
    "ppc_create", "ppc_create_batch", "ppc_destroy", "ppc_set_stream", "ppc_set_precision",
    "ppc_set_random_seed", "ppc_set_neighbor_capacity", "ppc_upload", "ppc_upload_fields",
    "ppc_download", "ppc_get_count", "ppc_synchronize", "ppc_host_alloc", "ppc_host_free",
    "ppc_get_event_counts", "ppc_flag_by_draws", "ppc_step", "ppc_step_with_phenotype",
    "ppc_get_neighbors", "ppc_get_mesh_bins", "ppc_get_voxel_count", "ppc_get_mesh_position",
    "ppc_get_mesh_index", "ppc_get_launch_count", "ppc_last_error", "ppc_abi_version",
    "ppc_set_profiling", "ppc_get_profile", "ppc_set_launch_shape", "ppc_autotune",
    "ppc_update_cell_cell_interactions", "ppc_update_motility_fields", "ppc_set_host_transfer",
    "ppc_upload_interactions", "ppc_download_interactions", "ppc_upload_motility", "ppc_download_motility",
    "ppc_count_flags", "ppc_set_step_form", "ppc_set_wait_limit", "ppc_upload_gradients",
    "ppc_bin_agents_noalloc",
) + tuple("ppc_" + e for e in ENTRY_POINTS)


def lib():
    """Loads libppc.so from the package directory; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run `python -m paraphysicell_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.ppc_create.argtypes = [C.POINTER(Mesh), C.POINTER(Params), C.c_int32, C.POINTER(vp)]
        L.ppc_create_batch.argtypes = [C.POINTER(Mesh), C.POINTER(C.c_int32), C.c_int32, C.POINTER(Params),
                                       C.POINTER(vp)]
        L.ppc_destroy.argtypes = [vp]
        L.ppc_set_stream.argtypes = [vp, vp]
        L.ppc_set_precision.argtypes = [vp, C.c_int32]
        L.ppc_set_random_seed.argtypes = [vp, C.c_uint64]
        L.ppc_set_neighbor_capacity.argtypes = [vp, C.c_int32]
        for f in ("ppc_upload", "ppc_upload_fields", "ppc_download"):
            getattr(L, f).argtypes = [vp, C.c_int32, C.POINTER(Agents)]
        L.ppc_get_count.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32)]
        L.ppc_synchronize.argtypes = [vp]
        L.ppc_host_alloc.argtypes = [C.c_size_t]
        L.ppc_host_alloc.restype = vp
        L.ppc_host_free.argtypes = [vp]
        L.ppc_host_free.restype = None
        L.ppc_get_event_counts.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.ppc_flag_by_draws.argtypes = [vp, C.c_double, C.c_double]
        L.ppc_count_flags.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]
        L.ppc_step.argtypes = [vp, C.c_int32]
        L.ppc_step_with_phenotype.argtypes = [vp, C.c_int32, C.c_double, C.c_double]
        L.ppc_get_neighbors.argtypes = [vp, C.c_int32, vp, vp, C.c_int32]
        L.ppc_get_mesh_bins.argtypes = [vp, C.c_int32, vp, vp]
        L.ppc_get_voxel_count.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64)]
        L.ppc_get_mesh_position.argtypes = [C.POINTER(Mesh), vp, vp]
        L.ppc_get_mesh_index.argtypes = [C.POINTER(Mesh), vp, vp]
        L.ppc_get_launch_count.argtypes = [vp, C.POINTER(C.c_int64)]
        L.ppc_set_profiling.argtypes = [vp, C.c_int32]
        L.ppc_set_launch_shape.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32]
        L.ppc_set_host_transfer.argtypes = [vp, C.c_int32]
        L.ppc_set_step_form.argtypes = [vp, C.c_int32]
        L.ppc_upload_gradients.argtypes = [vp, C.c_int32, C.POINTER(GradientField)]
        L.ppc_set_wait_limit.argtypes = [vp, C.c_int64]
        L.ppc_autotune.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.ppc_get_profile.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.ppc_last_error.restype = C.c_char_p
        for e in ENTRY_POINTS:
            getattr(L, "ppc_" + e).argtypes = [vp]
        L.ppc_update_cell_cell_interactions.argtypes = [vp, C.c_int32, C.POINTER(Interactions)]
        L.ppc_update_motility_fields.argtypes = [vp, C.c_int32, C.POINTER(Motility)]
        L.ppc_upload_interactions.argtypes = [vp, C.c_int32, C.POINTER(Interactions), C.c_int32]
        L.ppc_download_interactions.argtypes = [vp, C.c_int32, C.POINTER(Interactions)]
        L.ppc_upload_motility.argtypes = [vp, C.c_int32, C.POINTER(Motility)]
        L.ppc_download_motility.argtypes = [vp, C.c_int32, C.POINTER(Motility)]
        _lib = L
    return _lib


def _check(rc, where):
    if rc != 0:
        msg = lib().ppc_last_error().decode(errors="replace")
        raise PPCError(rc, where, msg)


class PinnedPool:
    """Page-locked host buffers from ppc_host_alloc, returned as numpy arrays."""

    def __init__(self):
        self.ptrs = []

    def __call__(self, n, dtype):
        dt = np.dtype(dtype)
        nbytes = max(int(n) * dt.itemsize, 1)
        p = lib().ppc_host_alloc(nbytes)
        if not p:
            raise MemoryError("ppc_host_alloc failed")
        self.ptrs.append(p)
        buf = (C.c_char * nbytes).from_address(p)
        return np.frombuffer(buf, dtype=dt, count=int(n))

    def free(self):
        for p in self.ptrs:
            lib().ppc_host_free(p)
        self.ptrs = []


class Simulation:
    """Device state of one simulation (`meshes` a Mesh) or of a batch of
    replicates (`meshes` a list of Mesh, `capacity` a list)."""

    def __init__(self, meshes, params: Params, capacity, seed: int = 0, neighbor_capacity: int | None = None):
        L = lib()
        h = C.c_void_p()
        if isinstance(meshes, Mesh):
            self.meshes = [meshes]
            _check(L.ppc_create(C.byref(meshes), C.byref(params), int(capacity), C.byref(h)), "ppc_create")
        else:
            self.meshes = list(meshes)
            arr = (Mesh * len(self.meshes))(*self.meshes)
            caps = (C.c_int32 * len(self.meshes))(*[int(c) for c in capacity])
            _check(L.ppc_create_batch(arr, caps, len(self.meshes), C.byref(params), C.byref(h)),
                   "ppc_create_batch")
        self.h = h
        self.params = params
        self.dims = self.meshes[0].dims
        self.ndefs = params.cell_definitions_count
        _check(L.ppc_set_random_seed(self.h, seed), "ppc_set_random_seed")
        if neighbor_capacity:
            _check(L.ppc_set_neighbor_capacity(self.h, neighbor_capacity), "ppc_set_neighbor_capacity")
        self.neighbor_capacity = neighbor_capacity or 64

    def close(self):
        if getattr(self, "h", None):
            lib().ppc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # ---- transfer ----
    def upload(self, agents, replicate=0):
        s = agents.struct()
        _check(lib().ppc_upload(self.h, replicate, C.byref(s)), "ppc_upload")

    def upload_fields(self, agents, fields, replicate=0):
        s = agents.struct(fields)
        _check(lib().ppc_upload_fields(self.h, replicate, C.byref(s)), "ppc_upload_fields")

    def download(self, agents, replicate=0, fields=None):
        s = agents.struct(fields)
        rc = lib().ppc_download(self.h, replicate, C.byref(s))
        agents.count = s.count
        _check(rc, "ppc_download")
        return agents

    def count(self, replicate=0):
        n = C.c_int32()
        _check(lib().ppc_get_count(self.h, replicate, C.byref(n)), "ppc_get_count")
        return n.value

    def count_flags(self, flag, replicate=0):
        n = C.c_int32()
        _check(lib().ppc_count_flags(self.h, replicate, flag, C.byref(n)), "ppc_count_flags")
        return n.value

    def event_counts(self, replicate=0):
        d, k = C.c_int64(), C.c_int64()
        _check(lib().ppc_get_event_counts(self.h, replicate, C.byref(d), C.byref(k)), "ppc_get_event_counts")
        return d.value, k.value

    def synchronize(self):
        _check(lib().ppc_synchronize(self.h), "ppc_synchronize")

    def set_stream(self, stream_handle):
        _check(lib().ppc_set_stream(self.h, C.c_void_p(stream_handle)), "ppc_set_stream")

    def set_precision(self, precision):
        _check(lib().ppc_set_precision(self.h, precision), "ppc_set_precision")

    def launches(self):
        n = C.c_int64()
        _check(lib().ppc_get_launch_count(self.h, C.byref(n)), "ppc_get_launch_count")
        return n.value

    def set_host_transfer(self, mode):
        """abi.PPC_TRANSFER_COPY_ENGINE (the default) or PPC_TRANSFER_ZERO_COPY."""
        _check(lib().ppc_set_host_transfer(self.h, mode), "ppc_set_host_transfer")

    def set_step_form(self, form):
        """abi.PPC_STEP_KERNELS (the default) or PPC_STEP_PERSISTENT."""
        _check(lib().ppc_set_step_form(self.h, form), "ppc_set_step_form")

    def set_wait_limit(self, polls):
        _check(lib().ppc_set_wait_limit(self.h, polls), "ppc_set_wait_limit")

    def set_launch_shape(self, tile_edge, threads, smem_bytes=32 * 1024):
        _check(lib().ppc_set_launch_shape(self.h, tile_edge, threads, smem_bytes), "ppc_set_launch_shape")

    def autotune(self, steps=10):
        """Times each candidate launch shape over `steps` steps (after as many
        warm-up steps) and keeps the fastest; returns (tile_edge, threads).
        The simulation advances by 12 x steps steps (six candidate shapes)."""
        e, t = C.c_int32(), C.c_int32()
        _check(lib().ppc_autotune(self.h, steps, C.byref(e), C.byref(t)), "ppc_autotune")
        return e.value, t.value

    def set_profiling(self, on):
        _check(lib().ppc_set_profiling(self.h, int(bool(on))), "ppc_set_profiling")

    def profile(self):
        ms, n = C.c_double(), C.c_int64()
        _check(lib().ppc_get_profile(self.h, C.byref(ms), C.byref(n)), "ppc_get_profile")
        return ms.value, n.value

    # ---- fused step ----
    def step(self, steps=1):
        _check(lib().ppc_step(self.h, steps), "ppc_step")

    def step_with_phenotype(self, steps, p_divide, p_death):
        _check(lib().ppc_step_with_phenotype(self.h, steps, p_divide, p_death), "ppc_step_with_phenotype")

    def flag_by_draws(self, p_divide, p_death):
        _check(lib().ppc_flag_by_draws(self.h, p_divide, p_death), "ppc_flag_by_draws")

    def update_motility_fields(self, fields=None, replicate=0):
        """position_solver::update_motility with motile agents; `fields`
        (abi.MotilityArrays) is read and its motility vectors written back, or
        None to use the resident fields (upload_motility)."""
        if fields is None:
            _check(lib().ppc_update_motility_fields(self.h, replicate, None), "ppc_update_motility_fields")
            return
        st = fields.struct()
        _check(lib().ppc_update_motility_fields(self.h, replicate, C.byref(st)), "ppc_update_motility_fields")

    def update_cell_cell_interactions(self, fields=None, replicate=0):
        """interactions_solver::update_cell_cell_interactions on one replicate;
        `fields` (abi.InteractionArrays) is read and written back in place, or
        None to use the resident fields (upload_interactions)."""
        if fields is None:
            _check(lib().ppc_update_cell_cell_interactions(self.h, replicate, None),
                   "ppc_update_cell_cell_interactions")
            return
        st = fields.struct()
        _check(lib().ppc_update_cell_cell_interactions(self.h, replicate, C.byref(st)),
               "ppc_update_cell_cell_interactions")

    def upload_interactions(self, fields, replicate=0, compute_internalized_substrates=False):
        st = fields.struct()
        _check(lib().ppc_upload_interactions(self.h, replicate, C.byref(st), int(compute_internalized_substrates)),
               "ppc_upload_interactions")

    def download_interactions(self, fields, replicate=0):
        """Fills `fields` (abi.InteractionArrays, capacity rows) and sets its count."""
        st = fields.struct()
        _check(lib().ppc_download_interactions(self.h, replicate, C.byref(st)), "ppc_download_interactions")
        fields.count = st.count
        return fields

    def upload_gradients(self, field, replicate=0):
        """`field`: abi.GradientField (the chemotaxis rules' input)."""
        _check(lib().ppc_upload_gradients(self.h, replicate, C.byref(field)), "ppc_upload_gradients")

    def upload_motility(self, fields, replicate=0):
        st = fields.struct()
        _check(lib().ppc_upload_motility(self.h, replicate, C.byref(st)), "ppc_upload_motility")

    def download_motility(self, fields, replicate=0):
        st = fields.struct()
        _check(lib().ppc_download_motility(self.h, replicate, C.byref(st)), "ppc_download_motility")
        fields.count = st.count
        return fields

    # ---- readback ----
    def neighbors(self, replicate=0, capacity=None):
        n = self.count(replicate)
        cap = capacity or self.neighbor_capacity
        counts = np.zeros(max(n, 1), np.int32)
        lists = np.zeros(max(n, 1) * cap, np.int32)
        _check(lib().ppc_get_neighbors(self.h, replicate, counts.ctypes.data, lists.ctypes.data, cap),
               "ppc_get_neighbors")
        lists = lists.reshape(max(n, 1), cap)
        return [list(lists[i, : counts[i]]) for i in range(n)]

    def mesh_bins(self, replicate=0):
        V = C.c_int64()
        _check(lib().ppc_get_voxel_count(self.h, replicate, C.byref(V)), "ppc_get_voxel_count")
        n = self.count(replicate)
        counts = np.zeros(V.value, np.int32)
        agents = np.zeros(max(n, 1), np.int32)
        _check(lib().ppc_get_mesh_bins(self.h, replicate, counts.ctypes.data, agents.ctypes.data),
               "ppc_get_mesh_bins")
        return counts, agents[:n]

    def __getattr__(self, name):
        if name in ENTRY_POINTS:
            fn = getattr(lib(), "ppc_" + name)

            def call():
                _check(fn(self.h), "ppc_" + name)
            return call
        raise AttributeError(name)
