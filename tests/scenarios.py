"""The reference's unit-test geometries (test/test.cpp), as host agent sets.

Each builder returns (mesh, params, agents) for one case; the same inputs
feed the oracle and the CUDA path.
"""
import json
import os

import numpy as np

from paraphysicell_b200.abi import AgentArrays, Mesh, Params  # noqa: F401

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def known_answers():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


PHENOTYPE_FIELDS = ("radius", "cell_cell_repulsion_strength", "cell_cell_adhesion_strength",
                    "relative_maximum_adhesion_distance", "cell_BM_repulsion_strength",
                    "attachment_elastic_constant", "attachment_rate", "detachment_rate",
                    "maximum_number_of_attachments", "cell_adhesion_affinities", "total_volume",
                    "nuclear_volume", "nuclear_radius", "surface_area", "polarity")


def created_agents(count, dims, ndefs, capacity=None):
    """Agents as `cell_container::create()` makes them: the cell constructor
    sets zero velocities, is_movable = true and the state defaults
    (reference: src/cell.cpp:47-61), while the phenotype storage is only
    value-initialised (phenotype_t's constructor sets no defaults,
    src/phenotype.cpp:6-16), so every phenotype field starts at zero."""
    a = AgentArrays(count, dims, ndefs, capacity)
    for f in PHENOTYPE_FIELDS:
        a.arrays[f][:] = 0
    return a


def _update_cell_for_velocity(a, i, offset, dims, def_index):
    """update_cell_for_velocity (reference: test/test.cpp:117-134)."""
    a.arrays["cell_definition_indices"][i] = def_index
    a.arrays["is_movable"][i] = 1
    pos = a.arrays["positions"].reshape(a.capacity, dims)
    for d in range(dims):
        pos[i, d] = 1 + offset + d
    a.arrays["radius"][i] = 4 + offset
    a.arrays["cell_cell_adhesion_strength"][i] = 5 + offset
    a.arrays["cell_cell_repulsion_strength"][i] = 6 + offset
    a.arrays["relative_maximum_adhesion_distance"][i] = 7 + offset
    aff = a.arrays["cell_adhesion_affinities"].reshape(a.capacity, a.ndefs)
    aff[i, 0] = 8 + offset
    aff[i, 1] = 9 + offset
    aff[i, 2] = 10 + offset


def velocity_simple(dims):
    """host_velocity_solver.simple (reference: test/test.cpp:141-191)."""
    mesh = Mesh.make(dims, (0, 0, 0), (80, 80, 80))
    params = Params.make(dt=0.1, ndefs=3)
    a = created_agents(3, dims, 3)
    _update_cell_for_velocity(a, 0, 0, dims, 0)
    _update_cell_for_velocity(a, 1, 10, dims, 1)
    pos = a.arrays["positions"].reshape(a.capacity, dims)
    pos[2, :] = 70
    return mesh, params, a


def velocity_complex(dims):
    """host_velocity_solver.complex (reference: test/test.cpp:265-320)."""
    mesh = Mesh.make(dims, (0, 0, 0), (80, 80, 80))
    params = Params.make(dt=0.1, ndefs=3)
    a = created_agents(3, dims, 3)
    r = 2.0 if dims == 1 else 4.0
    _update_cell_for_velocity(a, 0, 0, dims, 0)
    _update_cell_for_velocity(a, 1, 10, dims, 1)
    pos = a.arrays["positions"].reshape(a.capacity, dims)
    for i, x in enumerate((1.0, 4.0, 7.0)):
        a.arrays["radius"][i] = r
        a.arrays["relative_maximum_adhesion_distance"][i] = 1.0
        pos[i, :] = x
    return mesh, params, a


def expected_velocities_bruteforce(a):
    """compute_expected_velocities (reference: test/test.cpp:193-263): all
    ordered pairs, no clamping."""
    n, dims, D = a.count, a.dims, a.ndefs
    pos = a["positions"]
    r = a["radius"]
    rep = a["cell_cell_repulsion_strength"]
    adh = a["cell_cell_adhesion_strength"]
    rmad = a["relative_maximum_adhesion_distance"]
    aff = a["cell_adhesion_affinities"]
    dfn = a["cell_definition_indices"]
    out = np.zeros((n, dims))
    for i in range(n):
        for j in range(n):
            if i == j:
                continue
            diff = pos[i] - pos[j]
            dist = np.sqrt(np.sum(diff * diff))
            repulsion = (1 - dist / (r[i] + r[j])) ** 2 * np.sqrt(rep[i] * rep[j])
            adhesion = (1 - dist / (rmad[i] * r[i] + rmad[j] * r[j])) ** 2
            adhesion *= np.sqrt(adh[i] * adh[j] * aff[i, dfn[j]] * aff[j, dfn[i]])
            out[i] += (repulsion - adhesion) / dist * diff
    return out


def neighbors_grid(dims, cells_in_one_voxel, adhesion):
    """host_neighbors_solver.grid (reference: test/test.cpp:333-400): agents
    at every mechanics voxel centre, radius 9."""
    ka = known_answers()["host_neighbors_solver_grid"]
    mx = ka["mesh_max"]
    mesh = Mesh.make(dims, (0, 0, 0), mx)
    params = Params.make(dt=0.1, ndefs=3)
    g = mesh.grid_shape()
    V = g[0] * g[1] * g[2]
    n = V * cells_in_one_voxel
    a = created_agents(n, dims, 3)
    pos = a.arrays["positions"].reshape(a.capacity, dims)
    k = 0
    for v in range(V):
        c = (v % g[0], (v // g[0]) % g[1], v // (g[0] * g[1]))
        centre = [mesh.bounding_box_mins[d] + (c[d] + 0.5) * mesh.voxel_shape[d] for d in range(3)]
        for _ in range(cells_in_one_voxel):
            pos[k, :] = centre[:dims]
            k += 1
    a.arrays["radius"][:n] = ka["radius"]
    a.arrays["relative_maximum_adhesion_distance"][:n] = adhesion
    return mesh, params, a


def grid_expected_neighbors(mesh, cells_in_one_voxel, adhesion, coords):
    """Expected neighbour count of an agent in voxel `coords`
    (reference: test/test.cpp:382-398)."""
    g = mesh.grid_shape()
    expected = cells_in_one_voxel - 1
    if adhesion == 3:
        for z in (-1, 0, 1):
            for y in (-1, 0, 1):
                for x in (-1, 0, 1):
                    c = (coords[0] + x, coords[1] + y, coords[2] + z)
                    if all(0 <= c[d] < g[d] for d in range(3)) and (x, y, z) != (0, 0, 0):
                        expected += cells_in_one_voxel
    return expected


def container_four(dims=1):
    """cell_container.add_and_remove (reference: test/test.cpp:52-115): four
    agents with volumes 1..4 and x-velocities 10..40."""
    mesh = Mesh.make(dims, (0, 0, 0), (80, 0, 0), (20, 20, 20))
    params = Params.make(dt=0.1, ndefs=3)
    a = created_agents(4, dims, 3, capacity=8)
    vel = a.arrays["velocities"].reshape(a.capacity, dims)
    for i in range(4):
        a.arrays["total_volume"][i] = i + 1
        vel[i, 0] = 10 * (i + 1)
    return mesh, params, a


def interaction_case(name):
    """host_interactions_solver.<name> (reference: test/test.cpp:402-560):
    cells created from a cell definition (reference phenotype defaults) at
    one point, with the rates the test sets. Returns (mesh, params, agents,
    fields, case) where `case` holds the asserts and the number of calls."""
    from paraphysicell_b200.abi import InteractionArrays
    ka = known_answers()["host_interactions_solver"]
    case = ka["cases"][name]
    ndefs = ka["cell_definitions"]
    dims = case["dims"]
    mesh = Mesh.make(dims, case["mesh_min"], case["mesh_max"])
    params = Params.make(dt=0.1, ndefs=ndefs)
    n = len(case["cells"])
    a = AgentArrays(n, dims, ndefs)
    f = InteractionArrays(n, ndefs)
    pos = a.arrays["positions"].reshape(a.capacity, dims)
    for i, c in enumerate(case["cells"]):
        pos[i] = c["position"][:dims]
        a.arrays["cell_definition_indices"][i] = c["definition"]
        for k, v in c["rates"].items():
            f[k][i] = v
        for k, row in c["rate_rows"].items():
            for d, v in row.items():
                f[k][i, int(d)] = v
        f["dead"][i] = c.get("dead", 0)
    return mesh, params, a, f, case


def random_interaction_fields(a, ndefs, seed, substrates=2, scale=1.0):
    """Interaction fields for a dense agent set with rates high enough that
    agents ingest, attack and fuse neighbours that have already acted or
    been removed in the same call (the order-dependent paths)."""
    from paraphysicell_b200 import workloads as wl
    return wl.interaction_fields(a, ndefs, seed, substrates=substrates, scale=scale)
