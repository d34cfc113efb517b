"""Host transfers beside the device work: a download right after a step runs
on the state's transfer stream once the step's agent fields are final,
beside the rest of the step's mesh rebuild, and an upload of page-locked
positions copies them there while the stream finishes earlier work. Each
case must read exactly what a fully synchronised call reads, and the
oracle's state. Needs a CUDA device."""
import numpy as np
import pytest

from paraphysicell_b200 import workloads as wl
from paraphysicell_b200.abi import AgentArrays
from paraphysicell_b200.device import PinnedPool, Simulation
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu

DOWN = ("positions", "previous_velocities", "simple_pressure", "agent_ids", "flags")


def _download(sim, like, sync_first):
    if sync_first:
        sim.synchronize()
    out = AgentArrays(0, like.dims, like.ndefs, like.capacity, like.spring_capacity)
    out.count = out.capacity
    sim.download(out)
    return out


@pytest.mark.parametrize("phenotype", [False, True], ids=["mechanics", "division_and_death"])
def test_download_right_after_steps_equals_a_synchronised_one(phenotype):
    """Steps (1 and 10 per call, graph-replayed), each followed at once by a
    download: the same agents and fields as the same run with a full
    synchronisation before every download, and as the oracle."""
    mesh, params, a = wl.scaled(wl.config5, 6000, seed=81, capacity=8000)
    o, d = gu.make_pair(mesh, params, a, seed=5)
    ref = Simulation(mesh, params, a.capacity, seed=5)
    ref.upload(a)
    for x in (o,):
        x.update_mechanics_mesh()
        x.update_cell_neighbors()
    d.update_mechanics_mesh()
    ref.update_mechanics_mesh()
    for k in (1, 10, 1):
        if phenotype:
            d.step_with_phenotype(k, 0.01, 0.005)
            ref.step_with_phenotype(k, 0.01, 0.005)
            o.step(k, 1, 0.01, 0.005)
        else:
            d.step(k)
            ref.step(k)
            o.step(k, 0, 0.0, 0.0)
        got = _download(d, a, sync_first=False)
        want = _download(ref, a, sync_first=True)
        assert got.count == want.count
        for f in DOWN:
            assert np.array_equal(got[f], want[f]), (k, f)
        gu.assert_same_state(got, gu.fetch(o, a))
    d.close()
    ref.close()


def test_upload_after_a_step_is_what_a_download_reads():
    """A step, then an upload of page-locked positions (copied on the
    transfer stream while the step's rebuild may still run), then a
    download: the download returns the uploaded positions, and a further
    step starts from them like the oracle does."""
    mesh, params, a = wl.scaled(wl.config3, 3000, seed=83)
    o, d = gu.make_pair(mesh, params, a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    pool = PinnedPool()
    host = AgentArrays(a.count, a.dims, a.ndefs, a.capacity, a.spring_capacity, pinned=pool)
    for k, v in a.arrays.items():
        host.arrays[k][:] = v
    for step in range(4):
        d.step(1)
        o.step(1, 0, 0.0, 0.0)
        d.download(host, fields=("positions", "previous_velocities"))
        # move every agent a little, as a host model between steps would
        host.arrays["positions"][: 3 * host.count] += 0.25 * (step + 1)
        d.upload_fields(host, ("positions",))
        moved = gu.fetch(o, a)
        moved.arrays["positions"][: 3 * moved.count] += 0.25 * (step + 1)
        o.upload(moved)
        back = _download(d, a, sync_first=False)
        assert np.array_equal(back["positions"], host.arrays["positions"][: 3 * host.count].reshape(-1, 3))
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
    d.step(2)
    o.step(2, 0, 0.0, 0.0)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))
    d.close()
    del host
    pool.free()


def test_download_after_other_work_waits_for_it():
    """A step followed by other device work (flagging agents by draws): the
    download sees that work, like the oracle."""
    mesh, params, a = wl.scaled(wl.config5, 4000, seed=85)
    o, d = gu.make_pair(mesh, params, a, seed=9)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d.update_mechanics_mesh()
    d.step(1)
    o.step(1, 0, 0.0, 0.0)
    d.flag_by_draws(0.05, 0.05)
    o.flag_by_draws(0.05, 0.05)
    got = _download(d, a, sync_first=False)
    gu.assert_same_state(got, gu.fetch(o, a))
    assert np.count_nonzero(got["flags"][: got.count]) > 0
    d.close()
