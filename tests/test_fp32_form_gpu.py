"""FP32-force form (ppc_set_precision(PPC_FP32_FORCE)) against the FP64 form:
identical voxel bins and neighbour lists (the neighbour predicate stays exact),
per-step velocities within 1e-5 relative (normwise over agents), positions
after several steps close to FP64. Needs a CUDA device."""
import numpy as np
import pytest

from paraphysicell_b200 import workloads as wl
from paraphysicell_b200.abi import PPC_FP32_FORCE
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu

VEL_RTOL = 1e-5  # per-step velocity, normwise relative to the largest |v|


def _pair(mesh, params, a):
    _, d64 = gu.make_pair(mesh, params, a)
    _, d32 = gu.make_pair(mesh, params, a)
    d32.set_precision(PPC_FP32_FORCE)
    for d in (d64, d32):
        d.update_mechanics_mesh()
    return d64, d32


def _vel_error(g64, g32):
    v64, v32 = g64["previous_velocities"], g32["previous_velocities"]
    scale = np.max(np.linalg.norm(v64, axis=1))
    return np.max(np.linalg.norm(v32 - v64, axis=1)) / scale


@pytest.mark.parametrize("case", ["config2", "config3", "config5", "config1"])
def test_fp32_force_one_step(case):
    mesh, params, a = {
        "config2": lambda: wl.scaled(wl.config2, 4000, seed=81),
        "config3": lambda: wl.scaled(wl.config3, 6000, seed=82),
        "config5": lambda: wl.scaled(wl.config5, 6000, seed=83),
        "config1": lambda: wl.config1(seed=84),
    }[case]()
    d64, d32 = _pair(mesh, params, a)
    gu.assert_same_bins(d64, d32)
    d64.step(1)
    d32.step(1)
    g64, g32 = gu.fetch(d64, a), gu.fetch(d32, a)
    assert g64.count == g32.count
    assert np.array_equal(g64["agent_ids"], g32["agent_ids"])
    err = _vel_error(g64, g32)
    assert err <= VEL_RTOL, err
    np.testing.assert_allclose(g32["simple_pressure"], g64["simple_pressure"], rtol=1e-5, atol=1e-5)
    gu.assert_same_neighbors(d64, d32)


def test_fp32_force_full_size_config3():
    """The 88,700-agent workload: one step within the error bound, ten steps
    with positions within 1e-6 um per unit of displacement."""
    mesh, params, a = wl.config3(seed=3)
    d64, d32 = _pair(mesh, params, a)
    d64.step(1)
    d32.step(1)
    err = _vel_error(gu.fetch(d64, a), gu.fetch(d32, a))
    assert err <= VEL_RTOL, err
    gu.assert_same_neighbors(d64, d32)
    d64.step(9)
    d32.step(9)
    g64, g32 = gu.fetch(d64, a), gu.fetch(d32, a)
    drift = np.max(np.abs(g64["positions"] - g32["positions"]))
    moved = np.max(np.abs(g64["positions"] - a["positions"]))
    assert drift <= 1e-5 * max(moved, 1.0), (drift, moved)
