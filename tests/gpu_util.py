"""Helpers shared by the GPU parity tests: build both libraries, run the
same inputs through the oracle and the device, compare by agent id."""
import numpy as np

from oracle.oracle import Oracle
from paraphysicell_b200 import build
from paraphysicell_b200.abi import AgentArrays
from paraphysicell_b200.device import Simulation

VEC = ("positions", "velocities", "previous_velocities", "orientation")


def make_pair(mesh, params, agents, capacity=None, seed=0, neighbor_capacity=None):
    build.ensure_built()
    o = Oracle(mesh, params, seed=seed)
    o.upload(agents)
    d = Simulation(mesh, params, capacity or agents.capacity, seed=seed, neighbor_capacity=neighbor_capacity)
    d.upload(agents)
    return o, d


def fetch(sim_or_oracle, like, capacity=None):
    out = AgentArrays(0, like.dims, like.ndefs, capacity or like.capacity, like.spring_capacity)
    out.count = out.capacity
    sim_or_oracle.download(out)
    return out


def by_id(a):
    ids = a["agent_ids"]
    order = np.argsort(ids, kind="stable")
    return ids[order], order


def assert_same_state(got, want, exact=True, pressure_rtol=1e-12, fields=None):
    """Compares two downloaded agent sets: same count, same ids in the same
    slots, and the listed fields bit-exact (or pressure within rtol)."""
    assert got.count == want.count
    assert np.array_equal(got["agent_ids"], want["agent_ids"])
    fields = fields or ("positions", "previous_velocities", "velocities", "radius", "cell_definition_indices",
                        "is_movable", "flags", "total_volume", "orientation")
    for f in fields:
        g, w = got[f], want[f]
        if exact:
            assert np.array_equal(g, w), (f, np.max(np.abs(np.asarray(g, float) - np.asarray(w, float))))
        else:
            np.testing.assert_allclose(g, w, rtol=1e-12, atol=0, err_msg=f)
    np.testing.assert_allclose(got["simple_pressure"], want["simple_pressure"], rtol=pressure_rtol, atol=1e-300)


def assert_same_bins(d, o):
    dc, da = d.mesh_bins()
    oc, oa = o.mesh_bins()
    assert np.array_equal(dc, oc)
    assert np.array_equal(da, oa)


def assert_same_neighbors(d, o, capacity=None):
    dn = d.neighbors(capacity=capacity)
    on = o.neighbors(capacity=capacity)
    assert len(dn) == len(on)
    for i, (x, y) in enumerate(zip(dn, on)):
        assert x == y, (i, x, y)
