"""Parity at the full sizes of the benchmark workloads: the CUDA path through
the C ABI against the oracle's serial restatement of the reference
(position_solver.cpp:24-113, containers_solver.cpp:15-188) on identical
seeded inputs. Positions, velocities and bins must be bit-exact and the
neighbour lists identical; the FP32-force form must stay within 1e-5
relative per-step velocity error of the FP64 form. Needs a CUDA device."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from paraphysicell_b200 import workloads as wl
from paraphysicell_b200.abi import PPC_FP32_FORCE, AgentArrays
from paraphysicell_b200.device import Simulation
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu

VEL_RTOL = 1e-5  # FP32-force form: per-step velocity, normwise relative to the largest |v|


def _neighbor_arrays(x, n, cap=64):
    lists = x.neighbors(capacity=cap)
    assert len(lists) == n
    return lists


def test_config2_full_size_20_steps():
    """3-D, 14,300 agents, two types, basement-membrane walls on: 20 fused
    steps (two graph replays) bit-exact with the oracle."""
    mesh, params, a = wl.config2(seed=2)
    assert a.count == 14300 and params.virtual_wall_at_domain_edges == 1
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    o.step(20, 0, 0.0, 0.0)
    d.step(20)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
    gu.assert_same_bins(d, o)
    assert _neighbor_arrays(d, a.count) == _neighbor_arrays(o, a.count)


@pytest.mark.parametrize("precision", [0, PPC_FP32_FORCE], ids=["fp64", "fp32_force"])
def test_config4_all_replicates(precision):
    """The whole 256-replicate ensemble (3.26 M agents, N_r log-uniform in
    500..50,000) in one batched state, 5 steps: in FP64 every replicate equals
    its own serial oracle bit for bit; in the FP32-force form the per-step
    velocity of every replicate is within 1e-5 of the FP64 form's and the
    neighbour sets and bins are the FP64 form's."""
    meshes, params, sets = wl.config4(seed=4)
    assert len(sets) == 256
    d = Simulation(meshes, params, [s.capacity for s in sets])
    if precision:
        d.set_precision(precision)
    for r, s in enumerate(sets):
        d.upload(s, replicate=r)
    d.update_mechanics_mesh()
    if precision:
        ref = Simulation(meshes, params, [s.capacity for s in sets])
        for r, s in enumerate(sets):
            ref.upload(s, replicate=r)
        ref.update_mechanics_mesh()
        d.step(1)
        ref.step(1)
        for r, s in enumerate(sets):
            out, want = _fetch_rep(d, s, r), _fetch_rep(ref, s, r)
            assert np.array_equal(out["agent_ids"], want["agent_ids"])
            v32, v64 = out["previous_velocities"], want["previous_velocities"]
            err = np.max(np.linalg.norm(v32 - v64, axis=1)) / np.max(np.linalg.norm(v64, axis=1))
            assert err <= VEL_RTOL, (r, err)
            assert np.array_equal(d.mesh_bins(r)[0], ref.mesh_bins(r)[0])
        for r in range(0, 256, 51):
            assert d.neighbors(replicate=r) == ref.neighbors(replicate=r)
        ref.close()
        d.close()
        return
    d.step(5)
    for r, (m, s) in enumerate(zip(meshes, sets)):
        o = Oracle(m, params)
        o.upload(s)
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
        o.step(5, 0, 0.0, 0.0)
        gu.assert_same_state(_fetch_rep(d, s, r), gu.fetch(o, s))
        dc, da = d.mesh_bins(r)
        oc, oa = o.mesh_bins()
        assert np.array_equal(dc, oc) and np.array_equal(da, oa), r
        if r % 32 == 0:
            assert d.neighbors(replicate=r) == o.neighbors(), r
    d.close()


def _fetch_rep(d, s, r):
    out = AgentArrays(0, s.dims, s.ndefs, s.capacity)
    out.count = out.capacity
    d.download(out, replicate=r)
    return out


def test_config5_full_size_division_and_death():
    """1,000,000 agents with division (1e-4 per step) and death (5e-5) from
    the shared counter-based draws, compaction and rebuild every step: 3
    steps bit-exact with the oracle, ids in the same slots, the same event
    counts, bins and neighbour lists."""
    mesh, params, a = wl.config5(seed=5)
    o, d = gu.make_pair(mesh, params, a, seed=7)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    o.step(3, 1, wl.P_DIVIDE, wl.P_DEATH)
    d.step_with_phenotype(3, wl.P_DIVIDE, wl.P_DEATH)
    got, want = gu.fetch(d, a), gu.fetch(o, a)
    gu.assert_same_state(got, want, fields=gu.VEC[:3] + ("radius", "total_volume", "nuclear_volume",
                                                         "nuclear_radius", "surface_area", "orientation",
                                                         "flags", "is_movable"))
    assert d.event_counts() == o.event_counts()
    divisions, deaths = d.event_counts()
    assert divisions > 100 and deaths > 50
    gu.assert_same_bins(d, o)
    assert _neighbor_arrays(d, got.count) == _neighbor_arrays(o, want.count)
