"""Python binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/_build/libppc_oracle.so (building it with `make` when it is
missing). Only tests, the smoke check and the benchmark's CPU-baseline leg
import this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from paraphysicell_b200.abi import Agents, GradientField, Interactions, Mesh, Motility, Params, PPCError

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libppc_oracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(Mesh), C.POINTER(Params), C.POINTER(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_upload.argtypes = [vp, C.POINTER(Agents)]
        L.orc_download.argtypes = [vp, C.POINTER(Agents)]
        L.orc_count.argtypes = [vp]
        L.orc_count.restype = C.c_int32
        L.orc_event_counts.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_set_random_seed.argtypes = [vp, C.c_uint64]
        L.orc_voxel_count.argtypes = [vp]
        L.orc_voxel_count.restype = C.c_int64
        for name in ("orc_update_mechanics_mesh", "orc_update_cell_neighbors", "orc_update_cell_forces",
                     "orc_update_basement_membrane_interactions", "orc_update_spring_attachments",
                     "orc_update_positions", "orc_update_cell_container_for_mechanics",
                     "orc_update_cell_container_for_phenotype"):
            getattr(L, name).argtypes = [vp]
        L.orc_flag_by_draws.argtypes = [vp, C.c_double, C.c_double]
        L.orc_step.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, C.c_double]
        L.orc_time_steps.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double]
        L.orc_time_steps.restype = C.c_double
        L.orc_update_cell_cell_interactions.argtypes = [vp, C.POINTER(Interactions)]
        L.orc_update_motility_fields.argtypes = [vp, C.POINTER(Motility)]
        L.orc_sincos.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        L.orc_random_walk.argtypes = [C.c_int32, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                      C.c_void_p]
        L.orc_uniform.argtypes = [C.c_uint64] * 5
        L.orc_uniform.restype = C.c_double
        L.orc_upload_interactions.argtypes = [vp, C.POINTER(Interactions), C.c_int32]
        L.orc_download_interactions.argtypes = [vp, C.POINTER(Interactions)]
        L.orc_upload_motility.argtypes = [vp, C.POINTER(Motility)]
        L.orc_upload_gradients.argtypes = [vp, C.POINTER(GradientField)]
        L.orc_download_motility.argtypes = [vp, C.POINTER(Motility)]
        L.orc_get_neighbors.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_int32]
        L.orc_get_mesh_bins.argtypes = [vp, C.c_void_p, C.c_void_p]
        L.orc_get_mesh_position.argtypes = [vp, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


class Oracle:
    """One serial, deterministic restatement of the reference solver state."""

    def __init__(self, mesh: Mesh, params: Params, seed: int = 0):
        self.L = lib()
        self.mesh = mesh
        self.params = params
        h = C.c_void_p()
        rc = self.L.orc_create(C.byref(mesh), C.byref(params), C.byref(h))
        if rc:
            raise PPCError(rc, "orc_create")
        self.h = h
        self.L.orc_set_random_seed(self.h, seed)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def upload(self, agents):
        s = agents.struct()
        rc = self.L.orc_upload(self.h, C.byref(s))
        if rc:
            raise PPCError(rc, "orc_upload")

    def download(self, agents):
        s = agents.struct()
        rc = self.L.orc_download(self.h, C.byref(s))
        agents.count = s.count
        if rc:
            raise PPCError(rc, "orc_download")
        return agents

    @property
    def count(self):
        return self.L.orc_count(self.h)

    def event_counts(self):
        d, k = C.c_int64(), C.c_int64()
        self.L.orc_event_counts(self.h, C.byref(d), C.byref(k))
        return d.value, k.value

    def voxel_count(self):
        return self.L.orc_voxel_count(self.h)

    def __getattr__(self, name):
        # reference entry points: update_mechanics_mesh(), update_cell_forces(), ...
        fn = getattr(lib(), "orc_" + name, None)
        if fn is None:
            raise AttributeError(name)
        return lambda *a: fn(self.h, *a)

    def update_motility_fields(self, fields=None):
        """`fields` (abi.MotilityArrays): motility vectors are written back;
        None uses the resident fields."""
        st = fields.struct() if fields is not None else None
        rc = self.L.orc_update_motility_fields(self.h, C.byref(st) if st is not None else None)
        if rc != 0:
            raise PPCError(rc, "orc_update_motility_fields")

    def update_cell_cell_interactions(self, fields=None):
        """`fields` (abi.InteractionArrays) is read and written back in place;
        None uses the resident fields."""
        st = fields.struct() if fields is not None else None
        rc = self.L.orc_update_cell_cell_interactions(self.h, C.byref(st) if st is not None else None)
        if rc != 0:
            raise PPCError(rc, "orc_update_cell_cell_interactions")

    def upload_interactions(self, fields, compute_internalized_substrates=False):
        rc = self.L.orc_upload_interactions(self.h, C.byref(fields.struct()), int(compute_internalized_substrates))
        if rc != 0:
            raise PPCError(rc, "orc_upload_interactions")

    def download_interactions(self, fields):
        st = fields.struct()
        rc = self.L.orc_download_interactions(self.h, C.byref(st))
        fields.count = st.count
        if rc != 0:
            raise PPCError(rc, "orc_download_interactions")
        return fields

    def upload_gradients(self, field):
        rc = self.L.orc_upload_gradients(self.h, C.byref(field))
        if rc != 0:
            raise PPCError(rc, "orc_upload_gradients")

    def upload_motility(self, fields):
        rc = self.L.orc_upload_motility(self.h, C.byref(fields.struct()))
        if rc != 0:
            raise PPCError(rc, "orc_upload_motility")

    def download_motility(self, fields):
        st = fields.struct()
        rc = self.L.orc_download_motility(self.h, C.byref(st))
        fields.count = st.count
        if rc != 0:
            raise PPCError(rc, "orc_download_motility")
        return fields

    def time_steps(self, steps, threads, with_phenotype=False, p_divide=0.0, p_death=0.0):
        return self.L.orc_time_steps(self.h, steps, threads, int(with_phenotype), p_divide, p_death)

    def neighbors(self, capacity=None):
        import numpy as np
        n = self.count
        cap = capacity or 64
        while True:
            counts = np.zeros(max(n, 1), np.int32)
            lists = np.zeros(max(n, 1) * cap, np.int32)
            rc = self.L.orc_get_neighbors(self.h, counts.ctypes.data, lists.ctypes.data, cap)
            if rc == 0:
                break
            cap = int(counts.max()) + 1
        lists = lists.reshape(max(n, 1), cap)
        return [list(lists[i, : counts[i]]) for i in range(n)]

    def mesh_bins(self):
        import numpy as np
        V = self.voxel_count()
        counts = np.zeros(V, np.int32)
        agents = np.zeros(max(self.count, 1), np.int32)
        self.L.orc_get_mesh_bins(self.h, counts.ctypes.data, agents.ctypes.data)
        return counts, agents[: self.count]


def sincos(theta):
    """ppc_sincos of include/ppc_draws.h over an array of angles."""
    import numpy as np
    th = np.ascontiguousarray(theta, dtype=np.float64)
    sn, cs = np.empty_like(th), np.empty_like(th)
    lib().orc_sincos(th.ctypes.data, th.size, sn.ctypes.data, cs.ctypes.data)
    return sn, cs


def random_walk(dims, seed, epoch, replicate, slot, k0):
    """ppc_random_walk of include/ppc_draws.h: the reference's random walk
    from the counter-based draws."""
    import numpy as np
    w = np.zeros(3)
    lib().orc_random_walk(dims, seed, epoch, replicate, slot, k0, w.ctypes.data)
    return w[:dims]


def uniform(seed, epoch, replicate, slot, k):
    return lib().orc_uniform(seed, epoch, replicate, slot, k)
