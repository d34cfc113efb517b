"""Pins the CPU oracle against the reference's own known answers
(test/test.cpp, transcribed into tests/golden/known_answers.json by
tests/golden/make_golden.py). CPU only."""
import itertools

import numpy as np
import pytest

from oracle.oracle import Oracle
from paraphysicell_b200.abi import FLAG_TO_REMOVE
from tests import scenarios as sc


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_velocity_simple_known_answer(dims):
    """host_velocity_solver.simple: bit-exact FP64 known answers."""
    mesh, params, a = sc.velocity_simple(dims)
    o = Oracle(mesh, params)
    o.upload(a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    o.update_cell_forces()
    o.download(a)
    expected = float(sc.known_answers()["host_velocity_solver_simple"]["expected_velocity_cell1"][str(dims)])
    v = a["velocities"]
    for d in range(dims):
        assert v[0, d] == expected
        assert v[1, d] == -expected
        assert v[2, d] == 0.0


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_velocity_complex_against_bruteforce(dims):
    """host_velocity_solver.complex: neighbour counts {1,2,1} and the
    brute-force O(N^2) velocities (EXPECT_FLOAT_EQ in the reference, so the
    tolerance here is 4 float ulps)."""
    mesh, params, a = sc.velocity_complex(dims)
    o = Oracle(mesh, params)
    o.upload(a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    o.update_cell_forces()
    counts = [len(x) for x in o.neighbors()]
    assert counts == sc.known_answers()["host_velocity_solver_complex"]["neighbor_counts"]
    expected = sc.expected_velocities_bruteforce(a)
    o.download(a)
    np.testing.assert_allclose(a["velocities"], expected, rtol=4 * 2**-23, atol=0)


GRID = sc.known_answers()["host_neighbors_solver_grid"]


@pytest.mark.parametrize("dims,cells,adhesion",
                         list(itertools.product(GRID["dims"], GRID["cells_in_one_voxel"], GRID["adhesion"])))
def test_neighbors_grid(dims, cells, adhesion):
    """host_neighbors_solver.grid: voxel occupancy and neighbour counts."""
    mesh, params, a = sc.neighbors_grid(dims, cells, adhesion)
    o = Oracle(mesh, params)
    o.upload(a)
    o.update_mechanics_mesh()
    counts, _ = o.mesh_bins()
    assert (counts == cells).all()
    o.update_cell_neighbors()
    nb = o.neighbors(capacity=27 * cells + 1)
    pos = a["positions"]
    g = mesh.grid_shape()
    for i in range(a.count):
        c = [int((pos[i, d] - mesh.bounding_box_mins[d]) // 30) if d < dims else 0 for d in range(3)]
        assert len(nb[i]) == sc.grid_expected_neighbors(mesh, cells, adhesion, c)
    assert g[0] == 7


def test_container_swap_with_last_removal():
    """cell_container.add_and_remove: removal moves the last agent into the
    hole (expressed through the to_remove flag and the mechanics container
    update, which removes by the same swap-with-last)."""
    ka = sc.known_answers()["cell_container_add_and_remove"]["after_removals"]
    mesh, params, a = sc.container_four()
    o = Oracle(mesh, params)
    o.upload(a)
    for step, victim in zip(ka, (2, 0)):
        o.download(a)
        a.arrays["flags"][: a.count] = 0
        a.arrays["flags"][victim] = FLAG_TO_REMOVE
        o.upload(a)
        o.update_cell_container_for_mechanics()
        o.download(a)
        assert list(a["total_volume"]) == step["volumes"]
        assert list(a["velocities"][:, 0]) == step["velocities"]
    # add one: appended at the end (reference: test/test.cpp:101-114)
    assert o.event_counts()[1] == 2


def test_bins_descending_index_order():
    """A serial run of the reference's counting sort places agents of one
    voxel in descending index order (containers_solver.cpp:44-55 with
    fetch_sub)."""
    mesh, params, a = sc.neighbors_grid(3, 5, 1)
    o = Oracle(mesh, params)
    o.upload(a)
    o.update_mechanics_mesh()
    counts, agents = o.mesh_bins()
    off = 0
    for c in counts:
        seg = list(agents[off: off + c])
        assert seg == sorted(seg, reverse=True)
        off += c


def _check_interaction_asserts(case, flags, damage):
    names = {"none": 0, "to_remove": FLAG_TO_REMOVE}
    for a in case["asserts"]:
        got = flags[a["cell"]] if a["field"] == "flag" else damage[a["cell"]]
        want = names[a["value"]] if a["field"] == "flag" else a["value"]
        assert (got == want) == (a["op"] == "EQ"), a


@pytest.mark.parametrize("name", ["attack", "dead_phagocytosis", "phagocytosis", "fusion"])
def test_interactions_known_answers(name):
    """host_interactions_solver.{attack,dead_phagocytosis,phagocytosis,fusion}
    (reference: test/test.cpp:402-560): who is damaged or flagged for
    removal after the test's interaction calls."""
    mesh, params, a, f, case = sc.interaction_case(name)
    o = Oracle(mesh, params)
    o.upload(a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    for _ in range(case["calls"]):
        o.update_cell_cell_interactions(f)
    o.download(a)
    _check_interaction_asserts(case, a["flags"], f["damage"])


def test_interactions_ingest_and_fuse_volumes():
    """The ingesting agent gains the prey's fluid and solid volume, the fused
    agent the partner's compartments and nuclei, and both take the
    volume-weighted position and new radius (interactions_solver.cpp:6-131)."""
    mesh, params, a, f, case = sc.interaction_case("fusion")
    o = Oracle(mesh, params)
    before = f.copy()
    vol0 = a["total_volume"].copy()
    o.upload(a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    o.update_cell_cell_interactions(f)
    o.download(a)
    assert f["number_of_nuclei"][0] == 2
    assert a["total_volume"][0] == a["nuclear_volume"][0] + f["cytoplasmic"][0]
    assert a["total_volume"][0] == vol0[0] + vol0[1]
    assert f["nuclear_solid"][0] == before["nuclear_solid"][0] + before["nuclear_solid"][1]
    r = (a["total_volume"][0] / (np.pi * 4.0 / 3.0)) ** (1.0 / 3.0)
    assert abs(a["radius"][0] - r) <= 1e-12 * r
    assert a["flags"][1] == FLAG_TO_REMOVE


def test_interactions_rejects_wrong_count():
    mesh, params, a, f, case = sc.interaction_case("attack")
    o = Oracle(mesh, params)
    o.upload(a)
    from paraphysicell_b200.abi import InteractionArrays, PPCError
    with pytest.raises(PPCError):
        o.update_cell_cell_interactions(InteractionArrays(a.count + 1, 3))
