"""ppc_bin_agents_noalloc: mesh binning for callers that cannot allocate
device memory (an allocator that forbids hidden cudaMalloc calls, a real-time
loop that must not block in the driver's allocator). It must give exactly the
bins of the state-based path (ppc_update_mechanics_mesh + ppc_get_mesh_bins),
call after call, although every call reuses the same fixed scratch array.

Collected last on purpose: a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from paraphysicell_b200 import build, workloads as wl
from paraphysicell_b200.abi import PPC_ERR_CAPACITY, Mesh

pytestmark = pytest.mark.gpu


def _reference_bins(mesh, params, a):
    from paraphysicell_b200.device import Simulation
    sim = Simulation(mesh, params, a.capacity)
    sim.upload(a)
    sim.update_mechanics_mesh()
    counts, agents = sim.mesh_bins()
    sim.close()
    return counts, agents


def _noalloc(L, mesh, pos_dev, n, counts_dev, agents_dev, stream):
    L.ppc_bin_agents_noalloc.argtypes = [C.POINTER(Mesh), C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
    return L.ppc_bin_agents_noalloc(C.byref(mesh), C.c_void_p(pos_dev), n, C.c_void_p(counts_dev),
                                    C.c_void_p(agents_dev), C.c_void_p(stream))


def _line(n, seed):
    """A 1-D mesh: agents on a 3000 um line (100 voxels)."""
    from paraphysicell_b200.abi import AgentArrays, Params
    rng = np.random.default_rng(seed)
    mesh = Mesh.make(1, (0, 0, 0), (3000, 0, 0))
    a = AgentArrays(n, 1, 1, n)
    a.arrays["positions"][:n] = rng.uniform(0, 3000, n)
    return mesh, Params.make(dt=0.1, ndefs=1), a


def _odd_tiles(seed):
    """4097 voxels (241 x 17 in 2-D, one past a 4096-voxel scan tile), so the
    scan's last tile is partial and writes the final start entry."""
    from paraphysicell_b200.abi import AgentArrays, Params
    rng = np.random.default_rng(seed)
    mesh = Mesh.make(2, (0, 0, 0), (241 * 30, 17 * 30, 0))
    assert mesh.voxel_count() == 4097
    n = 3000
    a = AgentArrays(n, 2, 1, n)
    a.arrays["positions"][: 2 * n] = (rng.random((n, 2)) * [241 * 30, 17 * 30]).ravel()
    return mesh, Params.make(dt=0.1, ndefs=1), a


def _empty(case):
    """No agents: every voxel count must be zeroed, nothing else written."""
    from paraphysicell_b200.abi import AgentArrays
    mesh, params, a = case
    return mesh, params, AgentArrays(0, a.dims, a.ndefs, 4)


def test_noalloc_binning_matches_state_bins_on_consecutive_calls():
    import torch

    from paraphysicell_b200 import device

    build.ensure_built()
    L = device.lib()
    cases = [wl.config2(seed=31), wl.config1(seed=32), wl.scaled(wl.config5, 20000, seed=33), _line(1500, seed=34),
             _odd_tiles(seed=35), _empty(wl.config2(seed=36))]
    stream = torch.cuda.current_stream().cuda_stream
    for mesh, params, a in cases:
        want_counts, want_agents = _reference_bins(mesh, params, a)
        n = a.count
        pos = torch.from_numpy(np.ascontiguousarray(a["positions"]).reshape(-1)).cuda()
        counts = torch.empty(mesh.voxel_count(), dtype=torch.int32, device="cuda")
        agents = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
        for _ in range(2):
            counts.fill_(-7)
            agents.fill_(-7)
            rc = _noalloc(L, mesh, pos.data_ptr(), n, counts.data_ptr(), agents.data_ptr(), stream)
            assert rc == 0, L.ppc_last_error()
            torch.cuda.synchronize()
            assert np.array_equal(counts.cpu().numpy(), want_counts)
            assert np.array_equal(agents.cpu().numpy()[:n], want_agents)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from paraphysicell_b200 import device

    build.ensure_built()
    L = device.lib()
    mesh = Mesh.make(3, (0, 0, 0), (4000, 4000, 4000))  # 134^3 voxels > the fixed maximum
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ibuf = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = _noalloc(L, mesh, buf.data_ptr(), 2, ibuf.data_ptr(), ibuf.data_ptr(), 0)
    assert rc == PPC_ERR_CAPACITY
    L.ppc_last_error.restype = C.c_char_p
    assert b"voxels" in L.ppc_last_error()
