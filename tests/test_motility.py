"""Motility (position_solver::update_motility, reference:
src/solver/host/position_solver.cpp:115-145,288-314, solver_helper.h:82-101,
160-182,250-287): properties of the oracle's restatement on the CPU, and the
device path bit-exact against it on the GPU. The reference's unit tests have
no motility case, so these properties stand in for known answers."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from paraphysicell_b200 import workloads as wl
from paraphysicell_b200.abi import AgentArrays, Mesh, MotilityArrays, Params


def _agents(dims, n, seed):
    if dims == 3:
        mesh, params, a = wl.scaled(wl.config3, n, seed=seed, capacity=n + 16)
    elif dims == 2:
        mesh, params, a = wl.config1(seed=seed, n=n, capacity=n + 16)
    else:
        # one agent per ~6 um of line on average
        rng = np.random.default_rng(seed)
        mesh = Mesh.make(1, (-1000, 0, 0), (1000, 0, 0))
        params = Params.make(dt=0.1, ndefs=1)
        a = AgentArrays(n, 1, 1, n + 16)
        a.arrays["positions"][:n] = rng.uniform(-6.0 * n / 2, 6.0 * n / 2, n)
    return mesh, params, a


def _fields(n, dims, seed, persistence=(0.05, 5.0)):
    rng = np.random.default_rng(seed)
    m = MotilityArrays(n, dims)
    m["is_motile"][:] = (rng.random(n) < 0.7).astype(np.uint8)
    m["restrict_to_2d"][:] = (rng.random(n) < 0.3).astype(np.uint8)
    m["persistence_time"][:] = rng.uniform(*persistence, n)
    m["migration_speed"][:] = rng.uniform(0.1, 2.0, n)
    m["migration_bias"][:] = rng.random(n) * (rng.random(n) < 0.6)
    d = rng.normal(size=(n, dims))
    m["migration_bias_direction"][:] = d / np.linalg.norm(d, axis=1, keepdims=True)
    m["motility_vector"][:] = rng.normal(size=(n, dims)) * 0.1
    return m


def _velocities(x, a):
    out = AgentArrays(0, a.dims, a.ndefs, a.capacity)
    out.count = out.capacity
    x.download(out)
    return out["velocities"].copy()


@pytest.mark.parametrize("dims,per_agent", [(1, False), (2, False), (3, False), (3, True)])
def test_motility_oracle_properties(dims, per_agent):
    """Non-motile agents keep their velocity; a redraw gives a motility vector
    of length migration_speed (the bias direction when fully biased). In 3-D
    the reference's walk lies in the xy-plane for every agent (its bool
    parameter receives the restrict_to_2d array pointer,
    position_solver.cpp:131); with restrict_per_agent the flagged agents stay
    in the plane and the others get directions uniform on the sphere. Without
    a redraw the stored vector is added unchanged."""
    n = 300 if dims == 1 else 4000
    mesh, params, a = _agents(dims, n, seed=11)
    o = Oracle(mesh, params)
    o.upload(a)
    m = _fields(n, dims, seed=12, persistence=(0.001, 0.001))  # dt / p = 100: always redraw
    m.restrict_per_agent = per_agent
    m["migration_bias"][: n // 2] = 0.0
    m["migration_bias"][n // 2:] = 1.0
    before = m.copy()
    v0 = _velocities(o, a)
    o.update_motility_fields(m)
    v1 = _velocities(o, a)
    motile = m["is_motile"] == 1
    assert np.array_equal(v1[~motile], v0[~motile])
    assert np.array_equal(m["motility_vector"][~motile], before["motility_vector"][~motile])
    lengths = np.linalg.norm(m["motility_vector"], axis=1)
    np.testing.assert_allclose(lengths[motile], m["migration_speed"][motile], rtol=1e-14)
    np.testing.assert_array_equal(v1[motile], v0[motile] + m["motility_vector"][motile])
    biased = motile & (np.arange(n) >= n // 2)
    want = m["migration_bias_direction"] * m["migration_speed"][:, None]
    np.testing.assert_allclose(m["motility_vector"][biased], want[biased], rtol=1e-13, atol=1e-15)
    if dims == 3 and not per_agent:
        unbiased = motile & (np.arange(n) < n // 2)
        assert np.all(m["motility_vector"][unbiased][:, 2] == 0.0)
    if dims == 3 and per_agent:
        flat = motile & (m["restrict_to_2d"] == 1) & (np.arange(n) < n // 2)
        assert np.all(m["motility_vector"][flat][:, 2] == 0.0)
        free = motile & (m["restrict_to_2d"] == 0) & (np.arange(n) < n // 2)
        unit = m["motility_vector"][free] / m["migration_speed"][free][:, None]
        assert np.all(np.abs(unit.mean(axis=0)) < 0.08)
        assert np.count_nonzero(unit[:, 2]) == len(unit)
    if dims == 1:
        unbiased = motile & (np.arange(n) < n // 2)
        assert set(np.unique(np.sign(m["motility_vector"][unbiased, 0]))) == {-1.0, 1.0}

    # no redraw: persistence far above dt keeps the stored vector
    m2 = _fields(n, dims, seed=13, persistence=(1e30, 1e30))
    keep = m2.copy()
    o.update_motility_fields(m2)
    v2 = _velocities(o, a)
    assert np.array_equal(m2["motility_vector"], keep["motility_vector"])
    mot2 = m2["is_motile"] == 1
    np.testing.assert_array_equal(v2[mot2], v1[mot2] + keep["motility_vector"][mot2])


def test_motility_walk_is_the_references():
    """A redrawn, unbiased motility vector is migration_speed times the
    reference's random walk built from the agent's draws: theta = 2 pi u1 and,
    in 3-D with restrict_per_agent, z = 2 u2 - 1 (solver_helper.h:160-165,
    250-267); compared with libm's cos and sin to within 2 ulp."""
    from oracle import oracle as orc
    for dims, per_agent in ((2, False), (3, False), (3, True)):
        n = 2000
        mesh, params, a = _agents(dims, n, seed=41)
        o = Oracle(mesh, params, seed=17)
        o.upload(a)
        m = _fields(n, dims, seed=42, persistence=(0.001, 0.001))
        m.restrict_per_agent = per_agent
        m["migration_bias"][:] = 0.0
        m["migration_speed"][:] = 1.0
        o.update_motility_fields(m)
        for i in np.nonzero(m["is_motile"] == 1)[0][:400]:
            u1 = orc.uniform(17, 0, 0, int(i), 2097152 + 1)
            theta = u1 * (2 * np.pi)
            want = np.zeros(dims)
            if dims == 3 and per_agent and m["restrict_to_2d"][i] == 0:
                z = orc.uniform(17, 0, 0, int(i), 2097152 + 2) * 2.0 - 1.0
                r = np.sqrt(1 - z * z)
                want[:] = (np.cos(theta) * r, np.sin(theta) * r, z)
            else:
                want[:2] = (np.cos(theta), np.sin(theta))
            got = m["motility_vector"][i]
            # unit vector scaled by 1 / length: a few ulp from the walk itself
            np.testing.assert_allclose(got, want, rtol=0, atol=4e-16)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,per_agent", [(1, False), (2, False), (3, False), (3, True)])
def test_motility_matches_oracle(dims, per_agent):
    """The device's motility pass equals the oracle's bit for bit over three
    calls, and a fused step after it starts from the moved velocities."""
    from tests import gpu_util as gu
    n = 300 if dims == 1 else 3000
    mesh, params, a = _agents(dims, n, seed=21 + dims)
    o, d = gu.make_pair(mesh, params, a, seed=5)
    mo, md = _fields(n, dims, seed=31), _fields(n, dims, seed=31)
    mo.restrict_per_agent = md.restrict_per_agent = per_agent
    for _ in range(3):
        o.update_motility_fields(mo)
        d.update_motility_fields(md)
        assert np.array_equal(md["motility_vector"], mo["motility_vector"])
        assert np.array_equal(_velocities(d, a), _velocities(o, a))
    o.update_mechanics_mesh()
    o.update_cell_neighbors()  # the oracle's force pass reads the stored lists
    d.update_mechanics_mesh()
    o.step(1, 0, 0.0, 0.0)
    d.step(1)
    gu.assert_same_state(gu.fetch(d, a), gu.fetch(o, a))


@pytest.mark.gpu
def test_motility_argument_errors():
    from paraphysicell_b200.abi import PPCError
    from tests import gpu_util as gu
    mesh, params, a = _agents(2, 100, seed=3)
    o, d = gu.make_pair(mesh, params, a)
    with pytest.raises(PPCError):
        d.update_motility_fields(MotilityArrays(99, 2))
    with pytest.raises(PPCError):
        d.update_motility_fields(MotilityArrays(100, 2), replicate=3)
    d.update_motility_fields(MotilityArrays(100, 2))  # defaults: nobody is motile
    assert np.all(_velocities(d, a)[:100] == 0.0)


def _gradient_field(mesh, substrates, seed, voxel=20):
    """A gradient field over the diffusion mesh (20 um voxels) whose value
    differs from voxel to voxel, so a wrong voxel lookup shows."""
    from paraphysicell_b200.abi import GradientField
    rng = np.random.default_rng(seed)
    grid = [max(1, -(-(mesh.bounding_box_maxs[d] - mesh.bounding_box_mins[d]) // voxel)) if d < mesh.dims else 1
            for d in range(3)]
    g = rng.normal(size=(grid[0] * grid[1] * grid[2], substrates, 3))
    return GradientField.make(g, (voxel, voxel, voxel)), g, grid


def _voxel_of(mesh, pos, grid, voxel=20):
    c = np.zeros((len(pos), 3), dtype=np.int64)
    for d in range(mesh.dims):
        f = (pos[:, d] - mesh.bounding_box_mins[d]) / voxel
        c[:, d] = np.minimum(np.maximum(f, 0).astype(np.int64), grid[d] - 1)
    return c[:, 0] + grid[0] * (c[:, 1] + grid[1] * c[:, 2])


def _chemotaxis_fields(n, dims, substrates, seed):
    from paraphysicell_b200.abi import (PPC_DIRECTION_ADVANCED_CHEMOTAXIS,
                                        PPC_DIRECTION_ADVANCED_CHEMOTAXIS_NORMALIZED, PPC_DIRECTION_CHEMOTAXIS)
    rng = np.random.default_rng(seed)
    m = MotilityArrays(n, dims, substrates=substrates)
    m["is_motile"][:] = 1
    m["persistence_time"][:] = 0.001  # dt / persistence = 100: every agent redraws
    m["migration_speed"][:] = 1.0
    m["migration_bias"][:] = 1.0  # the direction alone
    m["direction_rule"][:] = rng.choice([0, PPC_DIRECTION_CHEMOTAXIS, PPC_DIRECTION_ADVANCED_CHEMOTAXIS,
                                         PPC_DIRECTION_ADVANCED_CHEMOTAXIS_NORMALIZED], size=n)
    m["chemotaxis_index"][:] = rng.integers(0, substrates, n)
    m["chemotaxis_direction"][:] = rng.choice([-1.0, 1.0], n)
    m["chemotactic_sensitivities"][:] = rng.uniform(-1, 2, (n, substrates))
    d = rng.normal(size=(n, dims))
    m["migration_bias_direction"][:] = d / np.linalg.norm(d, axis=1, keepdims=True)
    return m


@pytest.mark.parametrize("dims", [2, 3])
def test_chemotaxis_rules_in_the_oracle(dims):
    """The standard direction rules (standard_models.cpp:542-583) from the
    gradient of the agent's diffusion voxel: chemotaxis follows one
    substrate's gradient times the direction sign, advanced chemotaxis the
    sensitivity-weighted sum (of normalised gradients in its second form),
    each normalised; agents without a rule keep the caller's direction."""
    n, S = 3000, 3
    mesh, params, a = _agents(dims, n, seed=51)
    o = Oracle(mesh, params)
    o.upload(a)
    field, g, grid = _gradient_field(mesh, S, seed=52)
    o.upload_gradients(field)
    m = _chemotaxis_fields(n, dims, S, seed=53)
    before = m.copy()
    o.update_motility_fields(m)
    vox = _voxel_of(mesh, a["positions"].reshape(n, dims), grid)
    rule = m["direction_rule"]

    def unit(x):
        length = np.sqrt(np.sum(x * x, axis=-1, keepdims=True))
        return np.where(length > 1e-16, x / np.where(length > 0, length, 1), 0)

    want = before["migration_bias_direction"].copy()
    gi = g[vox][:, :, :dims]  # [n, S, dims]
    chem = rule == 1
    want[chem] = unit(gi[chem, m["chemotaxis_index"][chem]] * m["chemotaxis_direction"][chem, None])
    for r, norm in ((2, False), (3, True)):
        sel = rule == r
        gg = unit(gi[sel]) if norm else gi[sel]
        want[sel] = unit(np.sum(gg * m["chemotactic_sensitivities"][sel][:, :, None], axis=1))
    np.testing.assert_allclose(m["migration_bias_direction"], want, rtol=0, atol=1e-14)
    # fully biased, unit speed: the motility vector is the direction (normalised again)
    np.testing.assert_allclose(m["motility_vector"], unit(want), rtol=0, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,resident", [(2, False), (3, False), (3, True)])
def test_chemotaxis_rules_match_oracle(dims, resident):
    from tests import gpu_util as gu
    n, S = 3000, 3
    mesh, params, a = _agents(dims, n, seed=61)
    o, d = gu.make_pair(mesh, params, a, seed=9)
    field, _, _ = _gradient_field(mesh, S, seed=62)
    o.upload_gradients(field)
    d.upload_gradients(field)
    mo, md = _chemotaxis_fields(n, dims, S, seed=63), _chemotaxis_fields(n, dims, S, seed=63)
    mo["persistence_time"][:] = md["persistence_time"][:] = np.linspace(0.05, 2.0, n)
    if resident:
        o.upload_motility(mo)
        d.upload_motility(md)
    for _ in range(3):
        if resident:
            o.update_motility_fields(None)
            d.update_motility_fields(None)
        else:
            o.update_motility_fields(mo)
            d.update_motility_fields(md)
        assert np.array_equal(_velocities(d, a), _velocities(o, a))
    if resident:
        mo = o.download_motility(MotilityArrays(a.capacity, dims, substrates=S))
        md = d.download_motility(MotilityArrays(a.capacity, dims, substrates=S))
    for k in ("motility_vector", "migration_bias_direction"):
        assert np.array_equal(md[k], mo[k]), k
