"""z-slab decomposition (paraphysicell_b200/zslab.py): a simulation split
into slabs of mechanics-voxel z-layers, ghost layers and migrants exchanged
every step, must equal the undivided simulation bit for bit while no agent
leaves the domain. On the CPU the parts' steppers are the oracle's
restatement (in one process, and as two gloo ranks over torch.distributed);
on the GPU they are the CUDA states of the product."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from paraphysicell_b200 import workloads as wl
from paraphysicell_b200 import zslab

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class OracleStepper:
    """The oracle behind the stepper interface (its force pass reads the
    neighbour lists, so they are rebuilt with the mesh)."""

    def __init__(self, mesh, params):
        from oracle.oracle import Oracle
        self.o = Oracle(mesh, params)

    def upload(self, a):
        self.o.upload(a)

    def update_mechanics_mesh(self):
        self.o.update_mechanics_mesh()
        self.o.update_cell_neighbors()

    def step(self, k):
        self.o.step(k, 0, 0.0, 0.0)

    def download(self, a):
        return self.o.download(a)


def _workload():
    # 3-D, two types, walls; a ball well inside the box: no agent leaves
    return wl.scaled(wl.config2, 3000, seed=17)


def _single(mesh, params, a, steps):
    st = OracleStepper(mesh, params)
    st.upload(a)
    st.update_mechanics_mesh()
    st.step(steps)
    from paraphysicell_b200.abi import AgentArrays
    out = AgentArrays(0, a.dims, a.ndefs, a.capacity)
    out.count = out.capacity
    st.download(out)
    return zslab.sort_by_id(out)


def _assert_same(got, want):
    assert got.count == want.count
    for f in ("agent_ids", "positions", "previous_velocities", "simple_pressure", "velocities"):
        assert np.array_equal(got[f], want[f]), f


def test_split_layers_balances_and_covers():
    mesh, params, a = _workload()
    slabs = zslab.split_layers(mesh, a, 4)
    assert slabs[0][0] == 0 and slabs[-1][1] == mesh.grid_shape()[2]
    assert all(s1 == t0 for (_, s1), (t0, _) in zip(slabs, slabs[1:]))
    z = zslab.z_layer(mesh, a["positions"], 3)
    counts = [np.count_nonzero((z >= z0) & (z < z1)) for z0, z1 in slabs]
    assert sum(counts) == a.count and max(counts) < 0.4 * a.count


def test_pack_roundtrip():
    mesh, params, a = _workload()
    b = zslab.unpack(zslab.pack(zslab.subset(a, np.arange(0, a.count, 7))), a.dims, a.ndefs)
    c = zslab.subset(a, np.arange(0, a.count, 7))
    for name in ("positions", "agent_ids", "cell_adhesion_affinities", "is_movable"):
        assert np.array_equal(b[name], c[name]), name


def _fast(a):
    """Agents whose previous velocities carry them across z-layers: the
    first Adams-Bashforth step moves them by -0.05 min x vprev."""
    b = a.copy()
    rng = np.random.default_rng(5)
    vp = b.arrays["previous_velocities"][: 3 * b.count].reshape(b.count, 3)
    vp[:, 2] = rng.choice([-400.0, 400.0, 0.0], b.count)
    return b


@pytest.mark.parametrize("parts", [2, 3])
def test_slabs_in_one_process_equal_the_single_simulation(parts):
    mesh, params, a = _workload()
    a = _fast(a)
    stats = {}
    got = zslab.run_local(mesh, params, a, parts, lambda: OracleStepper(mesh, params), steps=8, stats=stats)
    _assert_same(got, _single(mesh, params, a, 8))
    assert stats["ghosts"] > 0 and stats["migrants"] > 0


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from paraphysicell_b200 import workloads as wl_
    from paraphysicell_b200 import zslab as zs
    from tests.test_zslab import OracleStepper, _fast

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh, params, a = wl_.scaled(wl_.config2, 3000, seed=17)
        a = _fast(a)
        own = zs.run_distributed(mesh, params, a, lambda: OracleStepper(mesh, params), 6, zs.TorchTransport("cpu"))
        out[rank] = zs.pack(own).tobytes()
    finally:
        dist.destroy_process_group()


def test_slabs_as_gloo_ranks_equal_the_single_simulation():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(2, 29541, out), nprocs=2, join=True, start_method="spawn")
    mesh, params, a = _workload()
    a = _fast(a)
    parts = [zslab.unpack(np.frombuffer(out[r], dtype=np.uint8), a.dims, a.ndefs) for r in range(2)]
    assert all(p.count > 0 for p in parts)
    got = zslab.sort_by_id(zslab.concat(parts, a.dims, a.ndefs))
    _assert_same(got, _single(mesh, params, a, 6))


@pytest.mark.gpu
def test_slabs_on_the_device_equal_the_device_simulation():
    """Two slabs, each a CUDA state over the global mesh, exchanging in
    process: bit-identical to one CUDA state of the whole simulation."""
    from paraphysicell_b200.abi import AgentArrays
    from paraphysicell_b200.device import Simulation
    mesh, params, a = _workload()
    a = _fast(a)
    stats = {}
    got = zslab.run_local(mesh, params, a, 2, lambda: Simulation(mesh, params, a.capacity), steps=8, stats=stats)
    assert stats["migrants"] > 0
    d = Simulation(mesh, params, a.capacity)
    d.upload(a)
    d.update_mechanics_mesh()
    d.step(8)
    out = AgentArrays(0, a.dims, a.ndefs, a.capacity)
    out.count = out.capacity
    d.download(out)
    _assert_same(got, zslab.sort_by_id(out))
