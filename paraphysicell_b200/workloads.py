"""Seeded synthetic workloads for the mechanics timestep.

The reference has no public dataset for its mechanics path; its README sizes
(900 / 14,300 / 88,700 agents, README.md:16-23) come from a modified
`heterogeneity` sample whose XML drives a builder this build does not carry.
These generators stand in for that setup with seeded numpy draws of the same
shapes, sizes and value distributions:

  config 1  2-D, 900 agents, one type, uniform in [-1000,1000]^2, r = 8.4127
  config 2  3-D, 14,300 agents, types A/B 50/50 in a ball of radius 450,
            r ~ U[7,10], A rep 10 / adh 0.4, B rep 12 / adh 0.8, cross-type
            affinity 0.5, basement-membrane walls on
  config 3  3-D, 88,700 agents in a ball of radius 1300 in a 4000 um cube,
            three types (rep 8/10/12, adh 0.2/0.4/0.8), 20% of agents draw
            1-3 springs to random neighbours within 1.25 (ri + rj), k = 0.05
  config 4  ensemble of replicates, N_r log-uniform in [500, 50000], cube
            side (8000 N_r)^(1/3) um rounded to whole um (one agent per
            8000 um^3), one type, r ~ U[7,10]
  config 5  3-D, 1,000,000 agents in a ball of radius 2900 in an 8000 um
            cube, two types, with division/death draws

Mechanics voxels are 30 um (reference: src/environment.h:10). Each
generator returns (Mesh, Params, AgentArrays) or, for the ensemble, lists.
"""
from __future__ import annotations

import numpy as np

from .abi import AgentArrays, Mesh, Params

FOUR_THIRDS_PI = np.pi * 4.0 / 3.0


def _ball(rng, n, radius, center):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    r = radius * rng.random(n) ** (1.0 / 3.0)
    return center + d * r[:, None]


def _unit(rng, n, dims):
    d = rng.normal(size=(n, dims))
    return d / np.linalg.norm(d, axis=1)[:, None]


def _set_geometry(a, radius):
    a.arrays["radius"][: a.count] = radius
    vol = FOUR_THIRDS_PI * radius ** 3
    a.arrays["total_volume"][: a.count] = vol
    a.arrays["nuclear_volume"][: a.count] = vol * (540.0 / 2494.0)
    a.arrays["nuclear_radius"][: a.count] = np.cbrt(vol * (540.0 / 2494.0) / FOUR_THIRDS_PI)
    a.arrays["surface_area"][: a.count] = 4.0 * np.pi * radius * radius


def _set_types(a, types, rep, adh, cross_affinity):
    n = a.count
    a.arrays["cell_definition_indices"][:n] = types
    a.arrays["cell_cell_repulsion_strength"][:n] = np.asarray(rep)[types]
    a.arrays["cell_cell_adhesion_strength"][:n] = np.asarray(adh)[types]
    aff = a.arrays["cell_adhesion_affinities"][: n * a.ndefs].reshape(n, a.ndefs)
    aff[:] = cross_affinity
    aff[np.arange(n), types] = 1.0


def config1(seed=1, n=900, capacity=None):
    """2-D mechanics-only case."""
    rng = np.random.default_rng(seed)
    mesh = Mesh.make(2, (-1000, -1000, -10), (1000, 1000, 10))
    params = Params.make(dt=0.1, ndefs=1, walls=False)
    a = AgentArrays(n, 2, 1, capacity or n)
    a.arrays["positions"][: 2 * n] = rng.uniform(-1000, 1000, size=(n, 2)).ravel()
    a.arrays["orientation"][: 2 * n] = _unit(rng, n, 2).ravel()
    return mesh, params, a


def config2(seed=2, n=14300, capacity=None):
    """3-D FP64 drop-in case."""
    rng = np.random.default_rng(seed)
    mesh = Mesh.make(3, (-1000, -1000, -1000), (1000, 1000, 1000))
    params = Params.make(dt=0.1, ndefs=2, walls=True)
    a = AgentArrays(n, 3, 2, capacity or n)
    a.arrays["positions"][: 3 * n] = _ball(rng, n, 450.0, np.zeros(3)).ravel()
    _set_geometry(a, rng.uniform(7.0, 10.0, n))
    types = (rng.random(n) < 0.5).astype(np.int32)
    _set_types(a, types, [10.0, 12.0], [0.4, 0.8], 0.5)
    a.arrays["orientation"][: 3 * n] = _unit(rng, n, 3).ravel()
    return mesh, params, a


def _add_springs(rng, a, fraction, k_max, spring_k):
    """Selected agents draw 1..k_max partners among agents within
    1.25 (ri + rj); springs are symmetric and capped at the maximum number of
    attachments (12)."""
    from scipy.spatial import cKDTree

    n, dims = a.count, a.dims
    pos = a.arrays["positions"][: n * dims].reshape(n, dims)
    rad = a.arrays["radius"][:n]
    tree = cKDTree(pos)
    lists = [[] for _ in range(n)]
    cap = a.arrays["maximum_number_of_attachments"][:n]
    chosen = np.nonzero(rng.random(n) < fraction)[0]
    cand = tree.query_ball_point(pos[chosen], r=1.25 * (rad[chosen] + rad.max()))
    for i, cs in zip(chosen, cand):
        cs = [j for j in cs if j != i and np.linalg.norm(pos[j] - pos[i]) <= 1.25 * (rad[i] + rad[j])]
        want = int(rng.integers(1, k_max + 1))
        rng.shuffle(cs)
        for j in cs[:want]:
            if j in lists[i] or len(lists[i]) >= cap[i] or len(lists[j]) >= cap[j]:
                continue
            lists[i].append(int(j))
            lists[j].append(int(i))
    a.set_springs(lists)
    a.arrays["attachment_elastic_constant"][:n] = spring_k
    return lists


def config3(seed=3, n=88700, capacity=None, springs=True):
    """3-D large precision-form case with springs."""
    rng = np.random.default_rng(seed)
    mesh = Mesh.make(3, (-2000, -2000, -2000), (2000, 2000, 2000))
    params = Params.make(dt=0.1, ndefs=3, walls=False)
    a = AgentArrays(n, 3, 3, capacity or n)
    a.arrays["positions"][: 3 * n] = _ball(rng, n, 1300.0, np.zeros(3)).ravel()
    _set_geometry(a, rng.uniform(7.0, 10.0, n))
    types = rng.integers(0, 3, n).astype(np.int32)
    _set_types(a, types, [8.0, 10.0, 12.0], [0.2, 0.4, 0.8], 1.0)
    a.arrays["orientation"][: 3 * n] = _unit(rng, n, 3).ravel()
    if springs:
        _add_springs(rng, a, 0.2, 3, 0.05)
    return mesh, params, a


def config4(seed=4, replicates=256, n_min=500, n_max=50000, spare=1.0):
    """Ensemble of independent replicates. Returns
    (meshes, params, agent_sets)."""
    rng = np.random.default_rng(seed)
    counts = np.rint(np.exp(rng.uniform(np.log(n_min), np.log(n_max), replicates))).astype(int)
    params = Params.make(dt=0.1, ndefs=1, walls=False)
    meshes, sets = [], []
    for n in counts:
        # a cube of (8000 N)^(1/3) um (one agent per 8000 um^3), rounded to
        # whole um: the mesh's bounding box is integer
        side = max(1, int(np.rint((8000.0 * n) ** (1.0 / 3.0))))
        mesh = Mesh.make(3, (0, 0, 0), (side, side, side))
        a = AgentArrays(int(n), 3, 1, int(np.ceil(n * spare)))
        a.arrays["positions"][: 3 * n] = rng.uniform(0, side, size=(n, 3)).ravel()
        _set_geometry(a, rng.uniform(7.0, 10.0, n))
        a.arrays["orientation"][: 3 * n] = _unit(rng, n, 3).ravel()
        meshes.append(mesh)
        sets.append(a)
    return meshes, params, sets


def config5(seed=5, n=1_000_000, capacity=None, radius=2900.0, cube=8000):
    """3-D 1M-agent case with division and death.
    Division/death probabilities per step: 1e-4 / 5e-5."""
    rng = np.random.default_rng(seed)
    h = cube // 2
    mesh = Mesh.make(3, (-h, -h, -h), (h, h, h))
    params = Params.make(dt=0.1, ndefs=2, walls=False)
    a = AgentArrays(n, 3, 2, capacity or int(n * 1.05) + 64)
    a.arrays["positions"][: 3 * n] = _ball(rng, n, radius, np.zeros(3)).ravel()
    _set_geometry(a, rng.uniform(7.0, 10.0, n))
    types = (rng.random(n) < 0.5).astype(np.int32)
    _set_types(a, types, [10.0, 12.0], [0.4, 0.8], 0.5)
    a.arrays["orientation"][: 3 * n] = _unit(rng, n, 3).ravel()
    return mesh, params, a


P_DIVIDE = 1e-4
P_DEATH = 5e-5


def scaled(config_fn, n, seed, **kw):
    """A config's distributions at a smaller agent count, with the ball (or
    domain) scaled so the density matches the full-size case."""
    full = {config1: 900, config2: 14300, config3: 88700, config5: 1_000_000}[config_fn]
    if config_fn is config1:
        return config1(seed=seed, n=n, **kw)
    f = (n / full) ** (1.0 / 3.0)
    if config_fn is config2:
        mesh, params, a = config2(seed=seed, n=n, **kw)
        return _rescale_ball(mesh, params, a, 450.0 * f, seed)
    if config_fn is config3:
        rng = np.random.default_rng(seed)
        mesh, params, a = config3(seed=seed, n=n, springs=False, **kw)
        mesh, params, a = _rescale_ball(mesh, params, a, 1300.0 * f, seed)
        _add_springs(rng, a, 0.2, 3, 0.05)
        return mesh, params, a
    if config_fn is config5:
        r = 2900.0 * f
        cube = 2 * int(np.ceil(r / 30.0 + 2)) * 30
        return config5(seed=seed, n=n, radius=r, cube=cube, **kw)
    raise ValueError(config_fn)


def _rescale_ball(mesh, params, a, radius, seed):
    rng = np.random.default_rng(seed + 1000)
    n = a.count
    a.arrays["positions"][: 3 * n] = _ball(rng, n, radius, np.zeros(3)).ravel()
    return mesh, params, a


def interaction_fields(a, ndefs, seed, substrates=2, scale=1.0, pinned=None):
    """Phenotype fields for cell-cell interactions over the agents of `a`:
    15 % dead agents; per-neighbour action probabilities up to 0.2 (dead
    ingestion), 0.06 (live ingestion), 0.2 x immunogenicity (attack) and 0.05
    (fusion) at scale 1 and dt 0.1; volume compartments around the reference
    defaults; `substrates` internalized substrates. Also sets the agents'
    total and nuclear volume to the compartments' sums."""
    from .abi import InteractionArrays
    rng = np.random.default_rng(seed)
    n = a.count
    f = InteractionArrays(n, ndefs, substrates, pinned)
    f["dead"][:] = (rng.random(n) < 0.15).astype(np.uint8)
    f["dead_phagocytosis_rate"][:] = rng.random(n) * 2.0 * scale
    f["damage_rate"][:] = 0.5 + rng.random(n)
    f["live_phagocytosis_rates"][:] = rng.random((n, ndefs)) * 0.6 * scale
    f["attack_rates"][:] = rng.random((n, ndefs)) * 2.0 * scale
    f["immunogenicities"][:] = rng.random((n, ndefs))
    f["fusion_rates"][:] = rng.random((n, ndefs)) * 0.5 * scale
    f["damage"][:] = rng.random(n)
    f["number_of_nuclei"][:] = 1 + (rng.random(n) < 0.1)
    for k in ("fluid", "solid", "cytoplasmic", "cytoplasmic_fluid", "cytoplasmic_solid", "nuclear_fluid",
              "nuclear_solid", "target_solid_cytoplasmic", "target_solid_nuclear"):
        f[k][:] *= 0.5 + rng.random(n)
    if substrates:
        f["internalized_substrates"][:] = rng.random((n, substrates)) * 10.0
        f["fraction_transferred_when_ingested"][:] = rng.random((n, substrates))
    vol = a.arrays["total_volume"]
    vol[:n] = f["fluid"] + f["solid"]
    a.arrays["nuclear_volume"][:n] = f["nuclear_fluid"] + f["nuclear_solid"]
    return f
