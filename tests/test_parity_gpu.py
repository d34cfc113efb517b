"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with
the reference's known answers. Needs a CUDA device."""
import itertools

import numpy as np
import pytest

from paraphysicell_b200 import workloads as wl
from paraphysicell_b200.abi import FLAG_TO_REMOVE
from tests import gpu_util as gu
from tests import scenarios as sc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_velocity_simple_known_answer(dims):
    """host_velocity_solver.simple on the device: bit-exact known answers
    (reference: test/test.cpp:141-191)."""
    mesh, params, a = sc.velocity_simple(dims)
    o, d = gu.make_pair(mesh, params, a)
    d.update_mechanics_mesh()
    d.update_cell_neighbors()
    d.update_cell_forces()
    got = gu.fetch(d, a)
    expected = float(sc.known_answers()["host_velocity_solver_simple"]["expected_velocity_cell1"][str(dims)])
    v = got["velocities"]
    for k in range(dims):
        assert v[0, k] == expected
        assert v[1, k] == -expected
        assert v[2, k] == 0.0


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_velocity_complex_matches_oracle(dims):
    """host_velocity_solver.complex: neighbour counts {1,2,1}, velocities
    bit-exact with the oracle (reference: test/test.cpp:265-320)."""
    mesh, params, a = sc.velocity_complex(dims)
    o, d = gu.make_pair(mesh, params, a)
    for x in (o, d):
        x.update_mechanics_mesh()
        x.update_cell_neighbors()
        x.update_cell_forces()
    assert [len(n) for n in d.neighbors()] == [1, 2, 1]
    gu.assert_same_neighbors(d, o)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))


GRID = sc.known_answers()["host_neighbors_solver_grid"]


@pytest.mark.parametrize("dims,cells,adhesion",
                         list(itertools.product(GRID["dims"], GRID["cells_in_one_voxel"], GRID["adhesion"])))
def test_neighbors_grid(dims, cells, adhesion):
    """host_neighbors_solver.grid: occupancy, neighbour counts and the exact
    neighbour lists (reference: test/test.cpp:333-400)."""
    mesh, params, a = sc.neighbors_grid(dims, cells, adhesion)
    cap = 27 * cells + 1
    o, d = gu.make_pair(mesh, params, a, neighbor_capacity=cap)
    for x in (o, d):
        x.update_mechanics_mesh()
        x.update_cell_neighbors()
    counts, _ = d.mesh_bins()
    assert (counts == cells).all()
    gu.assert_same_bins(d, o)
    gu.assert_same_neighbors(d, o, capacity=cap)
    nb = d.neighbors(capacity=cap)
    pos = a["positions"]
    for i in range(a.count):
        c = [int(pos[i, k] // 30) if k < dims else 0 for k in range(3)]
        assert len(nb[i]) == sc.grid_expected_neighbors(mesh, cells, adhesion, c)


def test_container_swap_with_last_removal():
    """cell_container.add_and_remove on the device (reference:
    test/test.cpp:52-115)."""
    ka = sc.known_answers()["cell_container_add_and_remove"]["after_removals"]
    mesh, params, a = sc.container_four()
    o, d = gu.make_pair(mesh, params, a)
    for step, victim in zip(ka, (2, 0)):
        cur = gu.fetch(d, a)
        cur.arrays["flags"][: cur.count] = 0
        cur.arrays["flags"][victim] = FLAG_TO_REMOVE
        d.upload(cur)
        d.update_cell_container_for_mechanics()
        got = gu.fetch(d, a)
        assert list(got["total_volume"]) == step["volumes"]
        assert list(got["velocities"][:, 0]) == step["velocities"]


def _cases():
    return {
        "config1_2d": lambda: wl.config1(seed=11, n=900),
        "config2_3d_walls": lambda: wl.scaled(wl.config2, 3000, seed=12),
        "config3_springs": lambda: wl.scaled(wl.config3, 4000, seed=13),
        "config5_dense": lambda: wl.scaled(wl.config5, 5000, seed=14),
    }


@pytest.mark.parametrize("case", list(_cases()))
def test_fused_steps_match_oracle(case):
    """Several fused steps (forces, membrane, springs, AB2, compaction,
    mesh) against the serial oracle: positions, velocities and previous
    velocities bit-exact, bins and neighbour lists identical, pressure
    within 1e-12 relative (its summation order is not the reference's)."""
    mesh, params, a = _cases()[case]()
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    for _ in range(3):
        o.step(4, 0, 0.0, 0.0)
        d.step(4)
        gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
        gu.assert_same_bins(d, o)
    gu.assert_same_neighbors(d, o)


# launch shapes of the fused pass: (tile edge, threads, shared-memory bytes).
# -1 is one thread per agent with its own pair code; -2 spreads the pair
# code over the warp; 0 does that with each block's candidate ranges staged
# in shared memory, and a budget of 4 KiB leaves no room for them, so blocks
# read the global arrays instead; -3 fetches each thread's candidates in
# batches; -4 (the default) shares the warp's candidates out over its lanes.
SHAPES = [(-1, 128, 0), (-1, 256, 0), (-2, 128, 0), (-2, 64, 0), (0, 128, 32 * 1024), (0, 128, 40 * 1024),
          (0, 64, 4 * 1024), (0, 96, 24 * 1024), (-3, 128, 0), (-4, 128, 0)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "edge%d_t%d_smem%d" % s)
@pytest.mark.parametrize("case", ["config2_3d_walls", "config3_springs", "config1_2d"])
def test_launch_shapes_match_oracle(case, shape):
    """Every launch shape gives the oracle's state bit for bit."""
    mesh, params, a = _cases()[case]()
    o, d = gu.make_pair(mesh, params, a)
    d.set_launch_shape(*shape)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    for _ in range(2):
        o.step(5, 0, 0.0, 0.0)
        d.step(5)
        gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))


def test_autotune_keeps_the_trajectory():
    """The autotuner runs 12 x steps real steps over its candidate shapes and
    keeps one of them; the state then equals the oracle's after as many
    steps, and stepping on with the chosen shape stays equal."""
    mesh, params, a = _cases()["config3_springs"]()
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    edge, threads = d.autotune(steps=3)
    assert (edge, threads) in {(-3, 128), (-4, 128), (-1, 128), (-2, 128), (0, 128), (0, 64)}
    o.step(36, 0, 0.0, 0.0)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
    o.step(7, 0, 0.0, 0.0)
    d.step(7)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))


def test_binning_on_a_large_grid():
    """An 8000 um cube (267^3 voxels, 4,650 scan tiles, more than the GPU
    holds at once) binned and stepped: bins and state equal the oracle's, so
    the two-pass scan is exact when tiles run in several waves."""
    mesh, params, a = wl.config5(seed=31, n=6000, radius=2900.0, cube=8000)
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    gu.assert_same_bins(d, o)
    o.step(3, 0, 0.0, 0.0)
    d.step(3)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
    gu.assert_same_bins(d, o)


def test_kinematic_uploads_keep_or_rebuild_the_mesh():
    """Uploading positions and previous velocities only: unchanged positions
    keep the mesh, moved ones (an agent pushed across voxels) rebuild it; the
    state then follows the oracle given the same host data."""
    mesh, params, a = wl.scaled(wl.config2, 2000, seed=91)
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    o.step(3, 0, 0.0, 0.0)
    d.step(3)
    for shift in (0.0, 45.0):
        host = gu.fetch(d, a)
        host.arrays["positions"][0] += shift  # agent 0, x
        d.upload_fields(host, ("positions", "previous_velocities"))
        full = gu.fetch(o, a)
        full.arrays["positions"][0] += shift
        o.upload(full)
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
        o.step(2, 0, 0.0, 0.0)
        d.step(2)
        gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
        gu.assert_same_bins(d, o)


def test_graph_replay_matches_oracle():
    """A block of steps long enough to be captured and replayed as a CUDA
    graph gives the same state as the oracle."""
    mesh, params, a = wl.scaled(wl.config2, 2000, seed=21)
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    o.step(25, 0, 0.0, 0.0)
    d.step(25)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
    o.step(20, 0, 0.0, 0.0)
    d.step(20)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))


def test_unfused_entry_points_match_fused():
    """The reference's separate entry points, called in simulator order,
    give bit-identical results to the fused step."""
    mesh, params, a = wl.scaled(wl.config3, 3000, seed=31)
    params.virtual_wall_at_domain_edges = 1
    _, d1 = gu.make_pair(mesh, params, a)
    _, d2 = gu.make_pair(mesh, params, a)
    d1.update_mechanics_mesh()
    d1.update_cell_neighbors()
    d2.update_mechanics_mesh()
    for _ in range(3):
        d1.update_cell_forces()
        d1.update_motility()
        d1.update_basement_membrane_interactions()
        d1.update_spring_attachments()
        d1.update_positions()
        d1.update_cell_container_for_mechanics()
        d1.update_mechanics_mesh()
        d1.update_cell_neighbors()
        d2.step(1)
    g1, g2 = gu.fetch(d1, a), gu.fetch(d2, a)
    gu.assert_same_state(g1, g2)
    gu.assert_same_neighbors(d1, d2)


def test_division_and_death_match_oracle():
    """Phenotype container update with counter-based draws: divisions append
    daughters in parent order, deaths swap-with-last; ids, positions and
    radii bit-exact with the oracle."""
    mesh, params, a = wl.scaled(wl.config5, 4000, seed=41, capacity=8000)
    o, d = gu.make_pair(mesh, params, a, seed=7)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    for _ in range(4):
        o.step(3, 1, 2e-3, 1e-3)
        d.step_with_phenotype(3, 2e-3, 1e-3)
        gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a),
                             fields=gu.VEC[:3] + ("radius", "total_volume", "nuclear_volume", "nuclear_radius",
                                                  "surface_area", "orientation", "flags", "is_movable"))
        assert d.event_counts() == o.event_counts()
    assert d.event_counts()[0] > 0 and d.event_counts()[1] > 0


def test_springs_survive_removals_like_oracle():
    """Removals of agents that carry springs rewrite the partners' spring
    rows in the reference's serial order (remove_attached/rename_attached)."""
    mesh, params, a = wl.scaled(wl.config3, 2000, seed=51)
    rng = np.random.default_rng(5)
    flags = a.arrays["flags"]
    with_springs = np.nonzero(a.arrays["spring_counts"][: a.count] > 0)[0]
    flags[rng.choice(with_springs, size=min(40, len(with_springs)), replace=False)] = FLAG_TO_REMOVE
    o, d = gu.make_pair(mesh, params, a)
    o.update_cell_container_for_mechanics()
    d.update_cell_container_for_mechanics()
    go, gd = gu.fetch(o, a), gu.fetch(d, a)
    assert gd.count == go.count < a.count
    assert gd.spring_lists() == go.spring_lists()
    gu.assert_same_state(gd, go)


@pytest.mark.parametrize("phenotype", [False, True])
def test_stochastic_springs_match_oracle(phenotype):
    """Non-zero attachment and detachment rates (update_spring_attachments,
    reference: position_solver.cpp:372-449): springs form and break with the
    oracle's counter-based draws, in its serial order and capacity checks;
    rows, positions and velocities stay equal step after step."""
    mesh, params, a = wl.scaled(wl.config3, 3000, seed=57, capacity=3300)
    a.arrays["attachment_rate"][: a.count] = 0.8
    a.arrays["detachment_rate"][: a.count] = 0.3
    a.arrays["maximum_number_of_attachments"][: a.count] = 3
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    before = a.spring_lists()
    for _ in range(3):
        if phenotype:
            o.step(3, 1, 2e-3, 1e-3)
            d.step_with_phenotype(3, 2e-3, 1e-3)
        else:
            o.step(3, 0, 0.0, 0.0)
            d.step(3)
        go, gd = gu.fetch(o, a), gu.fetch(d, a)
        assert gd.spring_lists() == go.spring_lists()
        gu.assert_same_state(gd, go)
    assert gd.spring_lists() != before  # springs did form and break


def test_dense_spring_attachment_matches_oracle():
    """Dense tissue with a high attachment rate and up to 12 springs: most
    agents appear in many candidates, so the attachments settle over many
    waves (and past the wave limit, in order); rows equal the oracle's."""
    mesh, params, a = wl.scaled(wl.config5, 1000, seed=71)
    n = a.count
    # a 10^3 lattice with 12 um spacing: about 19 neighbours per agent
    g = np.stack(np.meshgrid(np.arange(10), np.arange(10), np.arange(10), indexing="ij"), -1).reshape(-1, 3)[:n]
    pos = (g - 4.5) * 12.0 + np.random.default_rng(3).uniform(-0.5, 0.5, (n, 3))
    a.arrays["positions"][: 3 * n] = pos.ravel()
    a.arrays["attachment_rate"][:n] = 1.5
    a.arrays["detachment_rate"][:n] = 0.0
    a.arrays["maximum_number_of_attachments"][:n] = 12
    a.set_springs([[] for _ in range(n)])
    # the device lists a replicate's attachment candidates in a buffer of its
    # capacity: about 2,900 candidates in the first step
    o, d = gu.make_pair(mesh, params, a, capacity=4096)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    for _ in range(3):
        o.step(2, 0, 0.0, 0.0)
        d.step(2)
        go, gd = gu.fetch(o, a), gu.fetch(d, a)
        assert gd.spring_lists() == go.spring_lists()
        gu.assert_same_state(gd, go)
    assert max(len(x) for x in gd.spring_lists()) == 12


@pytest.mark.parametrize("shape", [(-1, 128, 0), (-2, 128, 0), (0, 128, 32 * 1024), (0, 64, 16 * 1024),
                                   (-3, 128, 0), (-4, 128, 0)],
                         ids=lambda s: "edge%d_t%d" % s[:2])
def test_batch_replicates_match_independent_oracles(shape):
    """Ensemble form: each replicate of one batched state evolves exactly
    like its own single simulation in the oracle, in every launch shape
    (blocks of the key-ordered array span replicate boundaries)."""
    meshes, params, sets = wl.config4(seed=61, replicates=6, n_min=200, n_max=3000)
    from oracle.oracle import Oracle
    from paraphysicell_b200.device import Simulation
    gu.build.ensure_built()
    d = Simulation(meshes, params, [s.capacity for s in sets])
    d.set_launch_shape(*shape)
    oracles = []
    for r, (m, s) in enumerate(zip(meshes, sets)):
        d.upload(s, replicate=r)
        o = Oracle(m, params)
        o.upload(s)
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
        oracles.append(o)
    d.update_mechanics_mesh()
    d.step(12)
    for r, (o, s) in enumerate(zip(oracles, sets)):
        o.step(12, 0, 0.0, 0.0)
        out = gu.AgentArrays(0, s.dims, s.ndefs, s.capacity)
        out.count = out.capacity
        d.download(out, replicate=r)
        gu.assert_same_state(out, gu.fetch(o, s))


@pytest.mark.parametrize("shape", [(-1, 128, 0), (-2, 128, 0), (0, 128, 32 * 1024), (-3, 128, 0), (-4, 128, 0)],
                         ids=lambda s: "edge%d" % s[0])
def test_empty_and_tiny_simulations(shape):
    """No agents, one agent, and every agent removed: the step, the mesh and
    the downloads behave like the oracle's."""
    from paraphysicell_b200.abi import AgentArrays
    mesh, params, a = wl.scaled(wl.config2, 300, seed=95)
    for n in (0, 1):
        b = AgentArrays(n, a.dims, a.ndefs, capacity=4)
        for k in b.arrays:
            width = b.arrays[k].size // b.capacity
            b.arrays[k][: n * width] = a.arrays[k][: n * width]
        o, d = gu.make_pair(mesh, params, b)
        d.set_launch_shape(*shape)
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
        d.update_mechanics_mesh()
        o.step(3, 0, 0.0, 0.0)
        d.step(3)
        gu.assert_same_state(gu.fetch(d, b), gu.fetch(o, b))
    gone = a.copy()
    gone.arrays["flags"][: gone.count] = FLAG_TO_REMOVE  # every agent removed
    o, d = gu.make_pair(mesh, params, gone)
    d.set_launch_shape(*shape)
    o.update_cell_container_for_mechanics()
    d.update_cell_container_for_mechanics()
    assert d.count() == gu.fetch(o, gone).count == 0
    o.update_mechanics_mesh()
    d.update_mechanics_mesh()
    o.step(2, 0, 0.0, 0.0)
    d.step(2)
    assert d.count() == gu.fetch(o, gone).count == 0


@pytest.mark.parametrize("shape", [(-1, 128, 0), (-2, 128, 0), (0, 128, 32 * 1024), (-3, 128, 0), (-4, 128, 0)],
                         ids=lambda s: "edge%d" % s[0])
def test_batch_with_an_empty_replicate(shape):
    """A batched state whose middle replicate has no agents steps the others
    exactly like their own oracles."""
    meshes, params, sets = wl.config4(seed=63, replicates=3, n_min=300, n_max=1200)
    from oracle.oracle import Oracle
    from paraphysicell_b200.abi import AgentArrays
    from paraphysicell_b200.device import Simulation
    gu.build.ensure_built()
    sets[1] = AgentArrays(0, sets[1].dims, sets[1].ndefs, capacity=sets[1].capacity)
    d = Simulation(meshes, params, [s.capacity for s in sets])
    d.set_launch_shape(*shape)
    oracles = []
    for r, (m, s_) in enumerate(zip(meshes, sets)):
        d.upload(s_, replicate=r)
        o = Oracle(m, params)
        o.upload(s_)
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
        oracles.append(o)
    d.update_mechanics_mesh()
    d.step(12)
    for r, (o, s_) in enumerate(zip(oracles, sets)):
        o.step(12, 0, 0.0, 0.0)
        out = gu.AgentArrays(0, s_.dims, s_.ndefs, s_.capacity)
        out.count = out.capacity
        d.download(out, replicate=r)
        gu.assert_same_state(out, gu.fetch(o, s_))


def test_errors_are_reported():
    """Device-detected failures come back as status codes, not faults."""
    from paraphysicell_b200.abi import PPCError, PPC_ERR_CAPACITY, PPC_ERR_NONFINITE
    mesh, params, a = wl.scaled(wl.config2, 500, seed=71)
    bad = a.copy()
    bad.arrays["positions"][3] = np.nan
    _, d = gu.make_pair(mesh, params, bad)
    with pytest.raises(PPCError) as e:
        d.update_mechanics_mesh()
    assert e.value.rc == PPC_ERR_NONFINITE

    mesh, params, g = sc.neighbors_grid(3, 5, 3)
    _, d = gu.make_pair(mesh, params, g, neighbor_capacity=8)
    d.update_mechanics_mesh()
    with pytest.raises(PPCError) as e:
        d.update_cell_neighbors()
    assert e.value.rc == PPC_ERR_CAPACITY

    mesh, params, a = wl.scaled(wl.config5, 500, seed=72, capacity=500)
    _, d = gu.make_pair(mesh, params, a)
    d.update_mechanics_mesh()
    d.flag_by_draws(0.5, 0.0)
    with pytest.raises(PPCError) as e:
        d.update_cell_container_for_phenotype()
    assert e.value.rc == PPC_ERR_CAPACITY

    from paraphysicell_b200.abi import PPC_ERR_ARG
    mesh, params, a = wl.scaled(wl.config2, 300, seed=74)
    _, d = gu.make_pair(mesh, params, a)
    for shape in ((3, 128, 0), (-5, 128, 0), (-8, 128, 0), (0, 100, 0), (0, 512, 0), (0, 128, 200 * 1024)):
        with pytest.raises(PPCError) as e:
            d.set_launch_shape(*shape)
        assert e.value.rc == PPC_ERR_ARG
    with pytest.raises(PPCError) as e:
        d.autotune(steps=0)
    assert e.value.rc == PPC_ERR_ARG


def test_full_size_config3_properties_and_oracle():
    """At the full 88,700-agent size: one step bit-exact with the oracle, and
    size-independent properties of the bins (each agent binned once, in the
    voxel of its position, descending inside a voxel) and the neighbour
    lists (symmetric between movable agents)."""
    mesh, params, a = wl.config3(seed=3)
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    o.step(2, 0, 0.0, 0.0)
    d.step(2)
    got = gu.fetch(d, a)
    gu.assert_same_state(got, gu.fetch(o, a))
    counts, agents = d.mesh_bins()
    assert counts.sum() == got.count
    assert np.array_equal(np.sort(agents), np.arange(got.count))
    g = mesh.grid_shape()
    pos = got["positions"]
    c = np.floor((pos - np.array(mesh.bounding_box_mins)) / 30.0).astype(int)
    key = c[:, 0] + g[0] * (c[:, 1] + g[1] * c[:, 2])
    owner = np.repeat(np.arange(len(counts)), counts)
    assert np.array_equal(key[agents], owner)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    for s, cnt in zip(starts[counts > 1], counts[counts > 1]):
        seg = agents[s: s + cnt]
        assert np.all(np.diff(seg) < 0)
    nb = d.neighbors()
    pairs = {(i, j) for i, lst in enumerate(nb) for j in lst}
    assert all((j, i) in pairs for (i, j) in pairs)


@pytest.mark.parametrize("shape", [(-4, 128, 0), (-3, 128, 0), (-2, 128, 0)], ids=lambda s: "edge%d" % s[0])
def test_removals_inside_fused_steps(shape):
    """Agents flagged for removal when steps start, and agents pushed out of
    the box during them: the compaction inside the fused step removes them,
    and the rebuild recounts every entry (the entries the fused pass made
    no longer hold), giving the oracle's state, bins and neighbours."""
    mesh, params, a = wl.scaled(wl.config2, 3000, seed=57)
    a.arrays["flags"][[3, 40, 41, 777, 1500]] = FLAG_TO_REMOVE
    # a few agents at the wall moving outwards: they leave during the steps
    pos = a.arrays["positions"][: 3 * a.count].reshape(a.count, 3)
    vp = a.arrays["previous_velocities"][: 3 * a.count].reshape(a.count, 3)
    for i in (10, 20, 30):
        pos[i] = (float(mesh.bounding_box_maxs[0]) - 1.0, pos[i][1], pos[i][2])
        vp[i] = (-300.0, 0.0, 0.0)
    params.virtual_wall_at_domain_edges = 0
    o, d = gu.make_pair(mesh, params, a)
    d.set_launch_shape(*shape)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    for k in (1, 10, 1):
        o.step(k, 0, 0.0, 0.0)
        d.step(k)
        gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
    assert gu.fetch(d, a).count < a.count - 5
    gu.assert_same_bins(d, o)
    gu.assert_same_neighbors(d, o)


@pytest.mark.parametrize("shape", [(-4, 128, 0), (-3, 128, 0), (-2, 128, 0)], ids=lambda s: "edge%d" % s[0])
def test_removed_tail_agent_releases_its_partners_springs(shape):
    """An agent with springs removed from the last slot, so that no agent
    moves into its hole: only its partners' spring rows and counts change,
    and the next fused passes must read the new counts (the reference's
    remove_attached, containers_solver.cpp:58-68)."""
    mesh, params, a = wl.scaled(wl.config3, 2000, seed=61)
    n = a.count
    tail = n - 1
    lists = [[j for j in lst if j != tail] for lst in a.spring_lists()]
    partners = [i for i in range(n - 1) if len(lists[i]) < a.spring_capacity - 1][:3]
    lists[tail] = partners
    for p in partners:
        lists[p].append(tail)
    a.set_springs(lists)
    a.arrays["flags"][tail] = FLAG_TO_REMOVE
    o, d = gu.make_pair(mesh, params, a)
    d.set_launch_shape(*shape)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    for k in (1, 1, 5):
        o.step(k, 0, 0.0, 0.0)
        d.step(k)
        go, gd = gu.fetch(o, a), gu.fetch(d, a)
        assert gd.count == go.count == n - 1
        assert gd.spring_lists() == go.spring_lists()
        gu.assert_same_state(gd, go)
