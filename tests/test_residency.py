"""Resident phenotype fields: interaction and motility columns kept beside
the mechanics state, moved by the container's swap-with-last removal
(src/cell_data.cpp:285-313) and set by division as cell::divide does
(src/cell.cpp:108-163: damage and attack time cleared, volumes and, when
computed, internalized substrates halved; the daughter copies the phenotype
with a fresh state). The oracle's restatement is checked on the CPU; the
device is checked against it on the GPU, bit for bit."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from paraphysicell_b200 import workloads as wl
from paraphysicell_b200.abi import FLAG_TO_DIVIDE, FLAG_TO_REMOVE, InteractionArrays, MotilityArrays

VOLUMES = ("fluid", "solid", "cytoplasmic", "cytoplasmic_fluid", "cytoplasmic_solid", "nuclear_fluid",
           "nuclear_solid", "target_solid_cytoplasmic", "target_solid_nuclear")


def _setup(n=1500, seed=3):
    mesh, params, a = wl.scaled(wl.config3, n, seed=seed, capacity=2 * n)
    a.arrays["positions"][: 3 * n] *= 0.45  # packed: neighbours for the interactions
    f = wl.interaction_fields(a, params.cell_definitions_count, seed=seed + 1, scale=1.0)
    return mesh, params, a, f


def _fetch_ix(x, cap, ndefs, subs):
    out = InteractionArrays(cap, ndefs, subs)
    return x.download_interactions(out)


def _fetch_agents(x, a):
    from paraphysicell_b200.abi import AgentArrays
    out = AgentArrays(0, a.dims, a.ndefs, a.capacity)
    out.count = out.capacity
    x.download(out)
    return out


def test_oracle_resident_interactions_equal_per_call_fields():
    """Interactions on the resident columns (fields=None) give the same
    agents and fields as the same call with the fields passed in."""
    mesh, params, a, f = _setup()
    o1, o2 = Oracle(mesh, params), Oracle(mesh, params)
    for o in (o1, o2):
        o.upload(a)
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
    f1 = f.copy()
    o1.update_cell_cell_interactions(f1)
    o2.upload_interactions(f)
    o2.update_cell_cell_interactions(None)
    f2 = _fetch_ix(o2, a.capacity, params.cell_definitions_count, f.substrates)
    assert f2.count == f1.count
    for k in f1.arrays:
        assert np.array_equal(f2[k], f1[k]), k
    g1, g2 = _fetch_agents(o1, a), _fetch_agents(o2, a)
    for k in ("positions", "total_volume", "radius", "flags"):
        assert np.array_equal(g1[k], g2[k]), k


@pytest.mark.parametrize("halve", [False, True])
def test_oracle_division_and_removal_carry_the_columns(halve):
    """Division: the parent's damage and attack time are cleared and its
    volume compartments (and substrates when computed) halved; the daughter
    copies the parent's columns with no damage or attack time and one
    nucleus. Removal: the last agent's columns move into the hole."""
    mesh, params, a, f = _setup(n=400, seed=9)
    n = a.count
    o = Oracle(mesh, params, seed=4)
    o.upload(a)
    o.upload_interactions(f, compute_internalized_substrates=halve)
    m = MotilityArrays(n, 3)
    m["is_motile"][:] = 1
    m["migration_speed"][:] = np.arange(n) + 0.5
    o.upload_motility(m)
    before = _fetch_ix(o, a.capacity, params.cell_definitions_count, f.substrates)
    ids0 = _fetch_agents(o, a)["agent_ids"].copy()
    flags = np.zeros(n, np.uint8)
    flags[[5, 17]] = FLAG_TO_DIVIDE
    flags[[2]] = FLAG_TO_REMOVE
    g = _fetch_agents(o, a)
    g.arrays["flags"][:n] = flags
    o.upload(g)  # a full upload keeps the resident columns' rows
    o.update_cell_container_for_phenotype()
    after = _fetch_ix(o, a.capacity, params.cell_definitions_count, f.substrates)
    ga = _fetch_agents(o, a)
    assert ga.count == n + 2 - 1
    row = {int(i): r for r, i in enumerate(ga["agent_ids"])}
    for p in (5, 17):
        r = row[int(ids0[p])]
        assert after["damage"][r] == 0 and after["total_attack_time"][r] == 0
        for k in VOLUMES:
            assert after[k][r] == before[k][p] * 0.5, k
        want = before["internalized_substrates"][p] * (0.5 if halve else 1.0)
        assert np.array_equal(after["internalized_substrates"][r], want)
    # daughters are appended in ascending parent order: ids n and n + 1
    parent_of = {n: int(ids0[5]), n + 1: int(ids0[17])}
    daughters = {int(i): r for r, i in enumerate(ga["agent_ids"]) if int(i) >= n}
    assert sorted(daughters) == [n, n + 1]
    for did, dr in daughters.items():
        pr = row[parent_of[did]]
        assert after["damage"][dr] == 0 and after["total_attack_time"][dr] == 0
        assert after["number_of_nuclei"][dr] == 1
        for k in VOLUMES + ("live_phagocytosis_rates", "attack_rates", "dead", "internalized_substrates"):
            assert np.array_equal(after[k][dr], after[k][pr]), k
    # removal: agent 2 is gone, the agent that took its slot kept its columns
    assert int(ids0[2]) not in row
    mo = o.download_motility(MotilityArrays(a.capacity, 3))
    for r, i in enumerate(ga["agent_ids"]):
        src = parent_of.get(int(i), int(i))
        assert mo["migration_speed"][r] == src + 0.5


@pytest.mark.gpu
def test_device_resident_interactions_match_oracle_across_steps():
    """Resident interaction fields on the device and in the oracle, chained:
    interactions, the phenotype container update (divisions and removals of
    agents that carry the columns), more interactions; the fields, agents and
    event counts stay bit-identical."""
    from tests import gpu_util as gu
    mesh, params, a, f = _setup(n=3000, seed=21)
    o, d = gu.make_pair(mesh, params, a, seed=3)
    for x in (o, d):
        x.upload_interactions(f, compute_internalized_substrates=True)
    D, S = params.cell_definitions_count, f.substrates
    for call in range(3):
        for x in (o, d):
            x.update_mechanics_mesh()
            x.update_cell_neighbors()
            x.update_cell_cell_interactions(None)
        o.flag_by_draws(0.01, 0.0)
        d.flag_by_draws(0.01, 0.0)
        o.update_cell_container_for_phenotype()
        d.update_cell_container_for_phenotype()
        fo, fd = _fetch_ix(o, a.capacity, D, S), _fetch_ix(d, a.capacity, D, S)
        assert fo.count == fd.count
        for k in fo.arrays:
            assert np.array_equal(fo[k], fd[k]), (call, k)
        go, gd = _fetch_agents(o, a), _fetch_agents(d, a)
        for k in ("agent_ids", "positions", "total_volume", "radius", "flags"):
            assert np.array_equal(go[k], gd[k]), (call, k)
        assert o.event_counts() == d.event_counts()
    assert o.event_counts()[0] > 0


@pytest.mark.gpu
def test_device_resident_motility_matches_oracle():
    from tests import gpu_util as gu
    mesh, params, a, _ = _setup(n=2000, seed=31)
    n = a.count
    rng = np.random.default_rng(2)
    m = MotilityArrays(n, 3)
    m["is_motile"][:] = (rng.random(n) < 0.7).astype(np.uint8)
    m["persistence_time"][:] = rng.uniform(0.05, 5.0, n)
    m["migration_speed"][:] = rng.uniform(0.1, 2.0, n)
    o, d = gu.make_pair(mesh, params, a, seed=6)
    for x in (o, d):
        x.upload_motility(m)
    for _ in range(3):
        o.update_motility_fields(None)
        d.update_motility_fields(None)
        mo, md = o.download_motility(MotilityArrays(a.capacity, 3)), d.download_motility(MotilityArrays(a.capacity, 3))
        for k in mo.arrays:
            assert np.array_equal(mo[k], md[k]), k
        assert np.array_equal(_fetch_agents(o, a)["velocities"], _fetch_agents(d, a)["velocities"])


@pytest.mark.gpu
def test_interactions_refuse_cut_neighbour_lists():
    """A neighbour list longer than the capacity: the call changes nothing
    and reports PPC_ERR_CAPACITY, even after the neighbour update's own error
    was already returned and cleared."""
    from paraphysicell_b200.abi import PPC_ERR_CAPACITY, PPCError
    from tests import gpu_util as gu
    mesh, params, a, f = _setup(n=2000, seed=41)
    _, d = gu.make_pair(mesh, params, a, neighbor_capacity=2)
    d.upload_interactions(f)
    d.update_mechanics_mesh()
    with pytest.raises(PPCError):
        d.update_cell_neighbors()
    before = _fetch_agents(d, a)
    fb = _fetch_ix(d, a.capacity, params.cell_definitions_count, f.substrates)
    with pytest.raises(PPCError) as e:
        d.update_cell_cell_interactions(None)
    assert e.value.rc == PPC_ERR_CAPACITY
    after = _fetch_agents(d, a)
    fa = _fetch_ix(d, a.capacity, params.cell_definitions_count, f.substrates)
    for k in ("positions", "flags", "total_volume"):
        assert np.array_equal(before[k], after[k])
    for k in fb.arrays:
        assert np.array_equal(fb[k], fa[k]), k
