"""The persistent step (ppc_set_step_form(PPC_STEP_PERSISTENT)): one
cooperative launch per mechanics step over all replicates, its phases (fused
pass, compaction plan, mesh rebuild) separated by bounded grid barriers.
It must give the oracle's state bit for bit, and a barrier that runs out of
polls must come back as PPC_ERR_TIMEOUT with the context still usable. The
wait is made to run out by a one-poll limit: no fault, trap or hang is
involved. Needs a CUDA device."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from paraphysicell_b200 import workloads as wl
from paraphysicell_b200.abi import (FLAG_TO_REMOVE, PPC_ERR_ARG, PPC_ERR_TIMEOUT, PPC_FP32_FORCE,
                                    PPC_STEP_PERSISTENT, AgentArrays, PPCError)
from paraphysicell_b200.device import Simulation
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu

SHAPES = [(-3, 128, 0), (-4, 128, 0), (-2, 128, 0), (0, 128, 32 * 1024)]


def _fetch(d, s, r):
    out = AgentArrays(0, s.dims, s.ndefs, s.capacity)
    out.count = out.capacity
    d.download(out, replicate=r)
    return out


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "edge%d" % s[0])
def test_persistent_batch_matches_independent_oracles(shape):
    """Six replicates of 200..3000 agents, a few agents flagged for removal
    (the compaction plan runs), 12 persistent steps (a replayed graph of 10
    and two single steps): every replicate equals its own serial oracle."""
    meshes, params, sets = wl.config4(seed=62, replicates=6, n_min=200, n_max=3000)
    rng = np.random.default_rng(3)
    for s in sets:
        s.arrays["flags"][rng.choice(s.count, size=3, replace=False)] = FLAG_TO_REMOVE
    gu.build.ensure_built()
    d = Simulation(meshes, params, [s.capacity for s in sets])
    d.set_launch_shape(*shape)
    d.set_step_form(PPC_STEP_PERSISTENT)
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
        got = _fetch(d, s, r)
        assert got.count <= s.count - 3  # the flagged three, and agents pushed out of the cube
        gu.assert_same_state(got, gu.fetch(o, s))
        dc, da = d.mesh_bins(r)
        oc, oa = o.mesh_bins()
        assert np.array_equal(dc, oc) and np.array_equal(da, oa)
    d.close()


@pytest.mark.parametrize("case", ["config3_springs", "config2_walls"])
def test_persistent_single_simulation_matches_oracle(case):
    """Springs (removals rewrite spring rows in the plan) and basement-membrane
    walls through the persistent step."""
    mesh, params, a = {"config3_springs": lambda: wl.scaled(wl.config3, 4000, seed=13),
                       "config2_walls": lambda: wl.scaled(wl.config2, 3000, seed=12)}[case]()
    a.arrays["flags"][[5, 77, 300]] = FLAG_TO_REMOVE
    o, d = gu.make_pair(mesh, params, a)
    d.set_step_form(PPC_STEP_PERSISTENT)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    for _ in range(2):
        o.step(11, 0, 0.0, 0.0)
        d.step(11)
        gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
    gu.assert_same_neighbors(d, o)


def test_persistent_fp32_force_equals_the_kernels():
    """The FP32-force form gives the same bits in both step forms."""
    meshes, params, sets = wl.config4(seed=64, replicates=4, n_min=500, n_max=4000)
    sims = []
    for form in (0, PPC_STEP_PERSISTENT):
        d = Simulation(meshes, params, [s.capacity for s in sets])
        d.set_precision(PPC_FP32_FORCE)
        if form:
            d.set_step_form(form)
        for r, s in enumerate(sets):
            d.upload(s, replicate=r)
        d.update_mechanics_mesh()
        d.step(7)
        sims.append(d)
    for r, s in enumerate(sets):
        a, b = _fetch(sims[0], s, r), _fetch(sims[1], s, r)
        for f in ("positions", "previous_velocities", "agent_ids", "simple_pressure"):
            assert np.array_equal(a[f], b[f]), (r, f)


def test_persistent_barrier_timeout_is_reported_and_recoverable():
    """A one-poll wait limit makes the grid barriers give up: the step comes
    back as PPC_ERR_TIMEOUT at the next synchronising call, later steps are
    refused until the state is uploaded again, and after the upload the
    persistent step runs normally and matches the oracle."""
    mesh, params, a = wl.scaled(wl.config2, 3000, seed=44)
    o, d = gu.make_pair(mesh, params, a)
    d.set_step_form(PPC_STEP_PERSISTENT)
    d.update_mechanics_mesh()
    d.set_wait_limit(1)
    d.step(3)
    with pytest.raises(PPCError) as e:
        d.synchronize()
    assert e.value.rc == PPC_ERR_TIMEOUT
    with pytest.raises(PPCError) as e:
        d.step(1)
    assert e.value.rc == PPC_ERR_ARG
    d.set_wait_limit(1 << 25)
    d.upload(a)
    d.update_mechanics_mesh()
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.step(5)
    o.step(5, 0, 0.0, 0.0)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))


def test_step_form_arguments():
    mesh, params, a = wl.scaled(wl.config2, 300, seed=45)
    _, d = gu.make_pair(mesh, params, a)
    for bad in (2, -1):
        with pytest.raises(PPCError):
            d.set_step_form(bad)
    with pytest.raises(PPCError):
        d.set_wait_limit(0)
