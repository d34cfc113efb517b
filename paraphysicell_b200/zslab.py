"""z-slab decomposition of one simulation over several GPUs (or processes).

The domain's mechanics-voxel z-layers are split into contiguous slabs, one
per part (a rank, or an in-process part). Every step each part

  1. sends the agents of its first and last z-layer to the neighbouring
     parts, which hold them as ghosts for this step;
  2. advances its own agents and the ghosts by one fused mechanics step on
     its own stepper (the CUDA state of paraphysicell_b200.device), and keeps
     the new state of its own agents only;
  3. sends the agents whose new position lies in another part's slab to
     that part (migration).

Exactness. A part's stepper covers the global mesh, so every voxel key is
the one a single simulation computes, and it holds its own agents and the
ghosts in ascending agent-id slots. A voxel belongs to exactly one slab, so
no voxel mixes own agents and ghosts: inside every voxel the agents sit in
descending id, which is the order of a single simulation whose slots follow
the ids. The neighbours of an own agent lie in its own or the adjacent
layers, all present, so its pair sums take the same terms in the same order
as in the single simulation, and the decomposed run is bit-identical to it
as long as no agent leaves the domain (a removal reorders the single
simulation's slots by swap-with-last). Springs, division and removal are not
supported across parts.

Transport. `TorchTransport` exchanges byte buffers with torch.distributed
point-to-point operations (NCCL over NVLink between GPUs, gloo between CPU
processes); `LocalTransport` connects parts that live in one process. The
reference has no domain decomposition: this is the capacity path for
simulations beyond one GPU, outside the single-GPU benchmark.
"""
from __future__ import annotations

import numpy as np

from .abi import FIELDS, AgentArrays

# the fields a part sends for a ghost or a migrant (springs are not supported)
_SENT = [f for f in FIELDS if f[0] not in ("spring_counts", "springs")]


def _width(mult, dims, ndefs):
    return {"dims": dims, "defs": ndefs}.get(mult, 1)


def subset(a: AgentArrays, rows) -> AgentArrays:
    """The agents of `a` at the given row indices, in that order."""
    rows = np.asarray(rows, dtype=np.int64)
    out = AgentArrays(len(rows), a.dims, a.ndefs, max(len(rows), 1), a.spring_capacity)
    for name, _, mult, _ in _SENT:
        w = _width(mult, a.dims, a.ndefs)
        src = a.arrays[name][: a.count * w].reshape(a.count, w)
        out.arrays[name][: len(rows) * w] = src[rows].reshape(-1)
    return out


def concat(parts, dims, ndefs, capacity=None) -> AgentArrays:
    n = sum(p.count for p in parts)
    out = AgentArrays(n, dims, ndefs, max(capacity or n, 1))
    for name, _, mult, _ in _SENT:
        w = _width(mult, dims, ndefs)
        o = 0
        for p in parts:
            out.arrays[name][o * w:(o + p.count) * w] = p.arrays[name][: p.count * w]
            o += p.count
    return out


def sort_by_id(a: AgentArrays) -> AgentArrays:
    return subset(a, np.argsort(a["agent_ids"], kind="stable"))


def pack(a: AgentArrays) -> np.ndarray:
    """One byte buffer: the count, then every sent field's rows."""
    chunks = [np.array([a.count], dtype=np.int64).view(np.uint8)]
    for name, _, mult, _ in _SENT:
        w = _width(mult, a.dims, a.ndefs)
        chunks.append(np.ascontiguousarray(a.arrays[name][: a.count * w]).view(np.uint8))
    return np.concatenate(chunks)


def unpack(buf: np.ndarray, dims, ndefs) -> AgentArrays:
    buf = np.ascontiguousarray(buf, dtype=np.uint8)
    n = int(buf[:8].view(np.int64)[0])
    out = AgentArrays(n, dims, ndefs, max(n, 1))
    o = 8
    for name, dt, mult, _ in _SENT:
        w = _width(mult, dims, ndefs)
        nb = n * w * np.dtype(dt).itemsize
        out.arrays[name][: n * w] = buf[o:o + nb].view(dt)
        o += nb
    return out


class LocalTransport:
    """Parts of one process: a mailbox per (source, destination)."""

    def __init__(self):
        self.box = {}

    def post(self, src, dst, buf):
        self.box[(src, dst)] = buf

    def collect(self, src, dst):
        return self.box.pop((src, dst))


class TorchTransport:
    """torch.distributed point-to-point exchange of byte buffers between a
    part and its neighbours: the sizes first, then the bytes, posted as one
    batch of isend/irecv so the two directions cannot deadlock. `device`
    "cuda" with the NCCL backend, "cpu" with gloo."""

    def __init__(self, device="cpu", group=None):
        self.device = device
        self.group = group

    def exchange(self, rank, sends: dict) -> dict:
        """sends: {peer: uint8 array}; returns {peer: uint8 array} from the
        same peers."""
        import torch
        import torch.distributed as dist

        peers = sorted(sends)
        sizes_out = {p: torch.tensor([len(sends[p])], dtype=torch.int64, device=self.device) for p in peers}
        sizes_in = {p: torch.zeros(1, dtype=torch.int64, device=self.device) for p in peers}
        ops = []
        for p in peers:
            ops.append(dist.P2POp(dist.isend, sizes_out[p], p, self.group))
            ops.append(dist.P2POp(dist.irecv, sizes_in[p], p, self.group))
        for w in dist.batch_isend_irecv(ops) if ops else []:
            w.wait()
        data_out = {p: torch.from_numpy(np.ascontiguousarray(sends[p])).to(self.device) for p in peers}
        data_in = {p: torch.empty(int(sizes_in[p].item()), dtype=torch.uint8, device=self.device) for p in peers}
        ops = []
        for p in peers:
            ops.append(dist.P2POp(dist.isend, data_out[p], p, self.group))
            ops.append(dist.P2POp(dist.irecv, data_in[p], p, self.group))
        for w in dist.batch_isend_irecv(ops) if ops else []:
            w.wait()
        return {p: data_in[p].cpu().numpy() for p in peers}


def z_layer(mesh, positions, dims):
    """Mechanics-voxel z-layer of each position (the truncation the
    binning uses, clamped into the grid)."""
    g = mesh.grid_shape()
    if dims < 3:
        return np.zeros(len(positions), dtype=np.int64)
    f = (positions[:, 2] - mesh.bounding_box_mins[2]) / mesh.voxel_shape[2]
    return np.minimum(np.maximum(f, 0).astype(np.int64), g[2] - 1)


def split_layers(mesh, agents: AgentArrays, parts: int):
    """Contiguous z-layer ranges [z0, z1), one per part, balanced by agent
    count; every part gets at least one layer."""
    g2 = mesh.grid_shape()[2]
    if parts > g2:
        raise ValueError("more parts than z-layers")
    hist = np.bincount(z_layer(mesh, agents["positions"].reshape(agents.count, agents.dims), agents.dims),
                       minlength=g2)
    cum = np.cumsum(hist)
    bounds = [0]
    for p in range(1, parts):
        target = cum[-1] * p / parts
        z = int(np.searchsorted(cum, target, side="left")) + 1
        z = max(z, bounds[-1] + 1)
        z = min(z, g2 - (parts - p))
        bounds.append(z)
    bounds.append(g2)
    return [(bounds[p], bounds[p + 1]) for p in range(parts)]


class ZSlabPart:
    """One part of a z-slab run: its slab of layers, its own agents (kept in
    ascending id order) and its stepper. `stepper` needs upload(agents),
    update_mechanics_mesh(), step(1) and download(agents) over the global
    mesh; device.Simulation is the product stepper."""

    def __init__(self, mesh, params, agents: AgentArrays, slabs, part, stepper):
        self.mesh, self.params = mesh, params
        self.slabs, self.part = slabs, part
        self.dims, self.ndefs = agents.dims, agents.ndefs
        if np.any(agents["spring_counts"] > 0):
            raise ValueError("springs are not supported across z-slabs")
        z = z_layer(mesh, agents["positions"].reshape(agents.count, agents.dims), agents.dims)
        z0, z1 = slabs[part]
        self.own = sort_by_id(subset(agents, np.nonzero((z >= z0) & (z < z1))[0]))
        self.stepper = stepper

    def owner(self, layers):
        starts = np.array([s[0] for s in self.slabs])
        return np.searchsorted(starts, layers, side="right") - 1

    def _layers(self, a):
        return z_layer(self.mesh, a["positions"].reshape(a.count, self.dims), self.dims)

    def ghost_sends(self):
        """The own agents of the slab's first and last layer, for the parts
        below and above."""
        z0, z1 = self.slabs[self.part]
        z = self._layers(self.own)
        out = {}
        if self.part > 0:
            out[self.part - 1] = pack(subset(self.own, np.nonzero(z == z0)[0]))
        if self.part < len(self.slabs) - 1:
            out[self.part + 1] = pack(subset(self.own, np.nonzero(z == z1 - 1)[0]))
        return out

    def advance(self, ghosts):
        """One step of the own agents with the received ghosts; returns the
        migrants to send ({part: bytes})."""
        local = sort_by_id(concat([self.own] + ghosts, self.dims, self.ndefs))
        st = self.stepper
        st.upload(local)
        st.update_mechanics_mesh()
        st.step(1)
        out = AgentArrays(0, self.dims, self.ndefs, max(local.count, 1))
        out.count = out.capacity
        st.download(out)
        mine = np.isin(out["agent_ids"], self.own["agent_ids"])
        moved = sort_by_id(subset(out, np.nonzero(mine)[0]))
        owners = self.owner(self._layers(moved))
        self.own = subset(moved, np.nonzero(owners == self.part)[0])
        return {p: pack(subset(moved, np.nonzero(owners == p)[0]))
                for p in sorted(set(owners.tolist()) - {self.part})}

    def settle(self, immigrants):
        if immigrants:
            self.own = sort_by_id(concat([self.own] + immigrants, self.dims, self.ndefs))


def run_local(mesh, params, agents, parts, make_stepper, steps, stats=None):
    """Every part in this process (LocalTransport): `steps` steps; returns
    all agents, sorted by id. `stats`, a dict, receives the number of ghosts
    and migrants moved."""
    slabs = split_layers(mesh, agents, parts)
    ps = [ZSlabPart(mesh, params, agents, slabs, p, make_stepper()) for p in range(parts)]
    ghosts_moved = migrants_moved = 0
    for _ in range(steps):
        sends = [p.ghost_sends() for p in ps]
        migrants = []
        for k, p in enumerate(ps):
            ghosts = [unpack(sends[q][k], p.dims, p.ndefs) for q in (k - 1, k + 1) if 0 <= q < parts]
            ghosts_moved += sum(g.count for g in ghosts)
            migrants.append(p.advance(ghosts))
        for k, p in enumerate(ps):
            arriving = [unpack(m[k], p.dims, p.ndefs) for m in migrants if k in m]
            migrants_moved += sum(x.count for x in arriving)
            p.settle(arriving)
    if stats is not None:
        stats.update(ghosts=ghosts_moved, migrants=migrants_moved)
    return sort_by_id(concat([p.own for p in ps], agents.dims, agents.ndefs))


def run_distributed(mesh, params, agents, make_stepper, steps, transport: TorchTransport):
    """This rank's part of a run over torch.distributed (rank = part);
    returns the rank's own agents after `steps` steps."""
    import torch.distributed as dist

    rank, world = dist.get_rank(), dist.get_world_size()
    slabs = split_layers(mesh, agents, world)
    part = ZSlabPart(mesh, params, agents, slabs, rank, make_stepper())
    for _ in range(steps):
        got = transport.exchange(rank, part.ghost_sends())
        ghosts = [unpack(got[q], part.dims, part.ndefs) for q in sorted(got)]
        out = part.advance(ghosts)
        # every rank sends to every other rank (empty buffers too), so both
        # sides of each pair post the same operations
        sends = {q: out.get(q, pack(AgentArrays(0, part.dims, part.ndefs, 1))) for q in range(world) if q != rank}
        got = transport.exchange(rank, sends)
        part.settle([unpack(got[q], part.dims, part.ndefs) for q in sorted(got)])
    return part.own
