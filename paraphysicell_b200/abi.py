"""ctypes mirror of the C ABI declared in include/ppc.h.

The structs here must match include/ppc.h field for field. `AgentArrays`
owns numpy arrays for every field of `ppc_agents` (the structure-of-arrays
view of the reference's `physicell::cell_data` fields that the mechanics step
touches, reference src/cell_data.h:59-79,137-196) and hands out a `ppc_agents`
whose pointers alias those arrays.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PPC_OK = 0
PPC_ERR_ARG = 1
PPC_ERR_CUDA = 2
PPC_ERR_CAPACITY = 3
PPC_ERR_NONFINITE = 4
PPC_ERR_TIMEOUT = 5
PPC_ERR_UNSUPPORTED = 6
PPC_ERR_OUT_OF_MESH = 7
PPC_ERR_NO_DEVICE = 8

STATUS_NAMES = {
    0: "PPC_OK", 1: "PPC_ERR_ARG", 2: "PPC_ERR_CUDA", 3: "PPC_ERR_CAPACITY",
    4: "PPC_ERR_NONFINITE", 5: "PPC_ERR_TIMEOUT", 6: "PPC_ERR_UNSUPPORTED",
    7: "PPC_ERR_OUT_OF_MESH", 8: "PPC_ERR_NO_DEVICE",
}

FLAG_NONE, FLAG_TO_REMOVE, FLAG_TO_DIVIDE = 0, 1, 2
PPC_FP64, PPC_FP32_FORCE = 0, 1
PPC_TRANSFER_COPY_ENGINE, PPC_TRANSFER_ZERO_COPY = 0, 1
PPC_STEP_KERNELS, PPC_STEP_PERSISTENT = 0, 1

# reference defaults (src/data_storage_phenotype.cpp:62-125,194-214, src/cell.cpp:47-61)
DEFAULT_RADIUS = 8.412710547954228
DEFAULT_NUCLEAR_RADIUS = 5.051670902881889
DEFAULT_SURFACE_AREA = 889.3685284131693
DEFAULT_TOTAL_VOLUME = 2494.0
DEFAULT_NUCLEAR_VOLUME = 540.0


class Mesh(C.Structure):
    _fields_ = [
        ("dims", C.c_int32),
        ("bounding_box_mins", C.c_int32 * 3),
        ("bounding_box_maxs", C.c_int32 * 3),
        ("voxel_shape", C.c_int32 * 3),
    ]

    @classmethod
    def make(cls, dims, mins, maxs, voxel=(30, 30, 30)):
        m = cls()
        m.dims = dims
        for d in range(3):
            m.bounding_box_mins[d] = int(mins[d])
            m.bounding_box_maxs[d] = int(maxs[d])
            m.voxel_shape[d] = int(voxel[d])
        return m

    def grid_shape(self):
        g = []
        for d in range(3):
            if d < self.dims:
                ext = self.bounding_box_maxs[d] - self.bounding_box_mins[d]
                g.append(max(1, (ext + self.voxel_shape[d] - 1) // self.voxel_shape[d]))
            else:
                g.append(1)
        return tuple(g)

    def voxel_count(self):
        g = self.grid_shape()
        return g[0] * g[1] * g[2]


class Params(C.Structure):
    _fields_ = [
        ("mechanics_time_step", C.c_double),
        ("cell_definitions_count", C.c_int32),
        ("virtual_wall_at_domain_edges", C.c_int32),
        ("automated_spring_adhesion", C.c_int32),
        ("reserved", C.c_int32),
    ]

    @classmethod
    def make(cls, dt=0.1, ndefs=1, walls=False, springs=True):
        p = cls()
        p.mechanics_time_step = dt
        p.cell_definitions_count = ndefs
        p.virtual_wall_at_domain_edges = int(bool(walls))
        p.automated_spring_adhesion = int(bool(springs))
        return p


_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)
_U8 = C.POINTER(C.c_uint8)


class Agents(C.Structure):
    _fields_ = [
        ("count", C.c_int32),
        ("capacity", C.c_int32),
        ("positions", _D),
        ("velocities", _D),
        ("previous_velocities", _D),
        ("simple_pressure", _D),
        ("radius", _D),
        ("cell_cell_repulsion_strength", _D),
        ("cell_cell_adhesion_strength", _D),
        ("relative_maximum_adhesion_distance", _D),
        ("cell_BM_repulsion_strength", _D),
        ("attachment_elastic_constant", _D),
        ("attachment_rate", _D),
        ("detachment_rate", _D),
        ("maximum_number_of_attachments", _I32),
        ("cell_adhesion_affinities", _D),
        ("cell_definition_indices", _I32),
        ("is_movable", _U8),
        ("flags", _U8),
        ("agent_ids", _I64),
        ("total_volume", _D),
        ("nuclear_volume", _D),
        ("nuclear_radius", _D),
        ("surface_area", _D),
        ("polarity", _D),
        ("orientation", _D),
        ("spring_capacity", C.c_int32),
        ("spring_counts", _I32),
        ("springs", _I32),
    ]


# (field, dtype, per-agent multiplicity: "dims", "defs", "springs" or 1, default)
FIELDS = [
    ("positions", np.float64, "dims", 0.0),
    ("velocities", np.float64, "dims", 0.0),
    ("previous_velocities", np.float64, "dims", 0.0),
    ("simple_pressure", np.float64, 1, 0.0),
    ("radius", np.float64, 1, DEFAULT_RADIUS),
    ("cell_cell_repulsion_strength", np.float64, 1, 10.0),
    ("cell_cell_adhesion_strength", np.float64, 1, 0.4),
    ("relative_maximum_adhesion_distance", np.float64, 1, 1.25),
    ("cell_BM_repulsion_strength", np.float64, 1, 100.0),
    ("attachment_elastic_constant", np.float64, 1, 0.01),
    ("attachment_rate", np.float64, 1, 0.0),
    ("detachment_rate", np.float64, 1, 0.0),
    ("maximum_number_of_attachments", np.int32, 1, 12),
    ("cell_adhesion_affinities", np.float64, "defs", 1.0),
    ("cell_definition_indices", np.int32, 1, 0),
    ("is_movable", np.uint8, 1, 1),
    ("flags", np.uint8, 1, 0),
    ("agent_ids", np.int64, 1, 0),
    ("total_volume", np.float64, 1, DEFAULT_TOTAL_VOLUME),
    ("nuclear_volume", np.float64, 1, DEFAULT_NUCLEAR_VOLUME),
    ("nuclear_radius", np.float64, 1, DEFAULT_NUCLEAR_RADIUS),
    ("surface_area", np.float64, 1, DEFAULT_SURFACE_AREA),
    ("polarity", np.float64, 1, 0.0),
    ("orientation", np.float64, "dims", 0.0),
    ("spring_counts", np.int32, 1, 0),
    ("springs", np.int32, "springs", -1),
]

_PTR = {np.float64: _D, np.int32: _I32, np.int64: _I64, np.uint8: _U8}


class AgentArrays:
    """Host arrays of one simulation's agents, with reference defaults.

    Arrays are sized for `capacity` agents; `count` agents are live. The
    per-agent row width of `springs` is `spring_capacity`.
    """

    def __init__(self, count, dims, ndefs, capacity=None, spring_capacity=12, pinned=None):
        self.dims = dims
        self.ndefs = ndefs
        self.count = int(count)
        self.capacity = int(capacity if capacity is not None else max(count, 1))
        self.spring_capacity = int(spring_capacity)
        self.arrays = {}
        for name, dt, mult, dflt in FIELDS:
            width = {"dims": dims, "defs": ndefs, "springs": self.spring_capacity}.get(mult, 1)
            n = self.capacity * width
            if pinned is not None:
                arr = pinned(n, dt)
            else:
                arr = np.empty(n, dtype=dt)
            arr[:] = dflt
            self.arrays[name] = arr
        self.arrays["agent_ids"][: self.capacity] = np.arange(self.capacity, dtype=np.int64)

    def __getitem__(self, name):
        """Live part of a field, shaped (count,) or (count, width)."""
        arr = self.arrays[name]
        width = arr.size // self.capacity
        a = arr[: self.count * width]
        return a.reshape(self.count, width) if width > 1 or name in ("positions", "velocities",
                                                                     "previous_velocities", "orientation",
                                                                     "cell_adhesion_affinities", "springs") else a

    def struct(self, fields=None):
        """ppc_agents aliasing these arrays. With `fields`, only those
        pointers are set (the rest are NULL). The struct of a field set is
        built once and reused while the arrays stay the same objects (a
        per-step transfer loop then costs no pointer setup)."""
        key = None if fields is None else tuple(fields)
        cache = self.__dict__.setdefault("_structs", {})
        hit = cache.get(key)
        if hit is not None and all(self.arrays[n] is arr for n, arr in hit[1]):
            s = hit[0]
        else:
            s = Agents()
            used = []
            for name, dt, _, _ in FIELDS:
                if fields is not None and name not in fields:
                    continue
                setattr(s, name, self.arrays[name].ctypes.data_as(_PTR[dt]))
                used.append((name, self.arrays[name]))
            cache[key] = (s, used)
        s.count = self.count
        s.capacity = self.capacity
        s.spring_capacity = self.spring_capacity
        return s

    def copy(self):
        out = AgentArrays(self.count, self.dims, self.ndefs, self.capacity, self.spring_capacity)
        for k, v in self.arrays.items():
            out.arrays[k][:] = v
        return out

    def set_springs(self, lists):
        """Sets spring rows from a list of per-agent index lists."""
        cnt = self.arrays["spring_counts"]
        rows = self.arrays["springs"].reshape(self.capacity, self.spring_capacity)
        cnt[:] = 0
        rows[:] = -1
        for i, lst in enumerate(lists):
            cnt[i] = len(lst)
            rows[i, : len(lst)] = lst

    def spring_lists(self):
        cnt = self.arrays["spring_counts"]
        rows = self.arrays["springs"].reshape(self.capacity, self.spring_capacity)
        return [list(rows[i, : cnt[i]]) for i in range(self.count)]


class Interactions(C.Structure):
    """ppc_interactions (include/ppc.h)."""
    _fields_ = [
        ("count", C.c_int32),
        ("substrates", C.c_int32),
        ("dead", _U8),
        ("dead_phagocytosis_rate", _D),
        ("damage_rate", _D),
        ("live_phagocytosis_rates", _D),
        ("attack_rates", _D),
        ("fusion_rates", _D),
        ("immunogenicities", _D),
        ("fraction_transferred_when_ingested", _D),
        ("damage", _D),
        ("total_attack_time", _D),
        ("number_of_nuclei", _I32),
        ("fluid", _D),
        ("solid", _D),
        ("cytoplasmic", _D),
        ("cytoplasmic_fluid", _D),
        ("cytoplasmic_solid", _D),
        ("nuclear_fluid", _D),
        ("nuclear_solid", _D),
        ("fluid_fraction", _D),
        ("cytoplasmic_to_nuclear_ratio", _D),
        ("target_solid_cytoplasmic", _D),
        ("target_solid_nuclear", _D),
        ("internalized_substrates", _D),
    ]


def _volume_defaults():
    """volume_t::set_defaults (reference: src/data_storage_phenotype.cpp:62-95)."""
    ff = 0.75
    total = 2494.0
    fluid = ff * total
    nuclear = 540.0
    nf = ff * nuclear
    cyto = total - nuclear
    cf = ff * cyto
    return {"fluid": fluid, "solid": total - fluid, "cytoplasmic": cyto, "cytoplasmic_fluid": cf,
            "cytoplasmic_solid": cyto - cf, "nuclear_fluid": nf, "nuclear_solid": nuclear - nf,
            "fluid_fraction": ff, "cytoplasmic_to_nuclear_ratio": cyto / (1e-16 + nuclear),
            "target_solid_cytoplasmic": cyto - cf, "target_solid_nuclear": nuclear - nf}


# (field, dtype, per-agent multiplicity: "defs", "subs" or 1, default); the
# interaction defaults are interactions_t::set_defaults and cell_state_t's
# (reference: src/data_storage_phenotype.cpp:320-328, src/cell.cpp:40-45)
INTERACTION_FIELDS = [
    ("dead", np.uint8, 1, 0),
    ("dead_phagocytosis_rate", np.float64, 1, 0.0),
    ("damage_rate", np.float64, 1, 1.0),
    ("live_phagocytosis_rates", np.float64, "defs", 0.0),
    ("attack_rates", np.float64, "defs", 0.0),
    ("fusion_rates", np.float64, "defs", 0.0),
    ("immunogenicities", np.float64, "defs", 1.0),
    ("fraction_transferred_when_ingested", np.float64, "subs", 0.0),
    ("damage", np.float64, 1, 0.0),
    ("total_attack_time", np.float64, 1, 0.0),
    ("number_of_nuclei", np.int32, 1, 1),
] + [(k, np.float64, 1, v) for k, v in _volume_defaults().items()] + [
    ("internalized_substrates", np.float64, "subs", 0.0),
]


class InteractionArrays:
    """Host arrays of the phenotype fields cell-cell interactions use, one row
    per agent, with the reference's defaults."""

    def __init__(self, count, ndefs, substrates=0, pinned=None):
        self.count = int(count)
        self.ndefs = int(ndefs)
        self.substrates = int(substrates)
        self.arrays = {}
        for name, dt, mult, dflt in INTERACTION_FIELDS:
            width = {"defs": self.ndefs, "subs": self.substrates}.get(mult, 1)
            n = max(self.count * width, 1)
            arr = pinned(n, dt) if pinned is not None else np.empty(n, dtype=dt)
            arr[:] = dflt
            self.arrays[name] = arr

    def __getitem__(self, name):
        arr = self.arrays[name]
        mult = next(m for f, _, m, _ in INTERACTION_FIELDS if f == name)
        if mult == 1:
            return arr[: self.count]
        width = self.ndefs if mult == "defs" else self.substrates
        return arr[: self.count * width].reshape(self.count, width)

    def struct(self):
        s = Interactions()
        s.count = self.count
        s.substrates = self.substrates
        for name, dt, _, _ in INTERACTION_FIELDS:
            setattr(s, name, self.arrays[name].ctypes.data_as(_PTR[dt]))
        return s

    def copy(self, pinned=None):
        out = InteractionArrays(self.count, self.ndefs, self.substrates, pinned)
        for k, v in self.arrays.items():
            out.arrays[k][:] = v
        return out


class Motility(C.Structure):
    """ppc_motility (include/ppc.h)."""
    _fields_ = [
        ("count", C.c_int32),
        ("restrict_per_agent", C.c_int32),
        ("is_motile", _U8),
        ("restrict_to_2d", _U8),
        ("persistence_time", _D),
        ("migration_speed", _D),
        ("migration_bias", _D),
        ("migration_bias_direction", _D),
        ("motility_vector", _D),
        ("direction_rule", _U8),
        ("chemotaxis_index", _I32),
        ("chemotaxis_direction", _D),
        ("chemotactic_sensitivities", _D),
        ("substrates", C.c_int32),
        ("reserved", C.c_int32),
    ]


PPC_DIRECTION_NONE, PPC_DIRECTION_CHEMOTAXIS = 0, 1
PPC_DIRECTION_ADVANCED_CHEMOTAXIS, PPC_DIRECTION_ADVANCED_CHEMOTAXIS_NORMALIZED = 2, 3


class GradientField(C.Structure):
    """ppc_gradient_field (include/ppc.h)."""
    _fields_ = [
        ("substrates", C.c_int32),
        ("voxel_shape", C.c_int32 * 3),
        ("gradients", _D),
    ]

    @classmethod
    def make(cls, gradients, voxel_shape):
        """`gradients`: float64 array [voxels, substrates, 3] (kept alive by the
        returned struct)."""
        g = cls()
        arr = np.ascontiguousarray(gradients, dtype=np.float64)
        g.substrates = arr.shape[1]
        for d in range(3):
            g.voxel_shape[d] = int(voxel_shape[d])
        g.gradients = arr.ctypes.data_as(_D)
        g._keep = arr
        return g


# motility_t::set_defaults (reference: src/data_storage_phenotype.cpp:245-256)
MOTILITY_FIELDS = [
    ("is_motile", np.uint8, 1, 0),
    ("restrict_to_2d", np.uint8, 1, 0),
    ("persistence_time", np.float64, 1, 1.0),
    ("migration_speed", np.float64, 1, 1.0),
    ("migration_bias", np.float64, 1, 0.0),
    ("migration_bias_direction", np.float64, "dims", 0.0),
    ("motility_vector", np.float64, "dims", 0.0),
    ("direction_rule", np.uint8, 1, 0),
    ("chemotaxis_index", np.int32, 1, 0),
    ("chemotaxis_direction", np.float64, 1, 1.0),
    ("chemotactic_sensitivities", np.float64, "subs", 0.0),
]


class MotilityArrays:
    """Host arrays of the motility fields, one row per agent, with the
    reference's defaults."""

    def __init__(self, count, dims, pinned=None, restrict_per_agent=False, substrates=0):
        self.count = int(count)
        self.dims = int(dims)
        self.substrates = int(substrates)
        # False: every 3-D walk in the xy-plane, as the reference; True: each
        # agent's restrict_to_2d flag decides
        self.restrict_per_agent = bool(restrict_per_agent)
        self.arrays = {}
        for name, dt, mult, dflt in MOTILITY_FIELDS:
            width = {"dims": self.dims, "subs": self.substrates}.get(mult, 1)
            n = max(self.count * width, 1)
            arr = pinned(n, dt) if pinned is not None else np.empty(n, dtype=dt)
            arr[:] = dflt
            self.arrays[name] = arr

    def __getitem__(self, name):
        arr = self.arrays[name]
        mult = next(m for f, _, m, _ in MOTILITY_FIELDS if f == name)
        if mult == 1:
            return arr[: self.count]
        width = self.dims if mult == "dims" else self.substrates
        return arr[: self.count * width].reshape(self.count, width)

    def struct(self):
        s = Motility()
        s.count = self.count
        s.substrates = self.substrates
        s.restrict_per_agent = int(self.restrict_per_agent)
        for name, dt, _, _ in MOTILITY_FIELDS:
            setattr(s, name, self.arrays[name].ctypes.data_as(_PTR[dt]))
        return s

    def copy(self, pinned=None):
        out = MotilityArrays(self.count, self.dims, pinned, self.restrict_per_agent, self.substrates)
        for k, v in self.arrays.items():
            out.arrays[k][:] = v
        return out


def status_name(rc):
    return STATUS_NAMES.get(rc, f"status {rc}")


class PPCError(RuntimeError):
    def __init__(self, rc, where, msg=""):
        super().__init__(f"{where} failed: {status_name(rc)} {msg}".strip())
        self.rc = rc


def repo_root():
    return os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
