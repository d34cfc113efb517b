"""Benchmark of the B200 mechanics timestep (agent-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload config3|config2|config5|config1]

One step is one mechanics timestep of the whole simulation (forces,
membrane, springs, Adams-Bashforth update, container compaction, mesh
rebuild) in simulator::simulate_mechanics order. The default workload is
the 3-D 88,700-agent case with springs (ball of radius 1300 um in a 4000 um
cube, three cell types, 20% of agents with 1-3 springs), FP64. Inputs are
seeded synthetic agents (the reference's sample XML setups are not used).

`value`: device time of K steps with the state resident in HBM, each step
bracketed by CUDA events on the library's stream with L2 flushed (a 256 MiB
write) before every timed step. `e2e`: the same steps through the C ABI with
host buffers: every step uploads positions and previous velocities from
pinned host memory and downloads positions, previous velocities and pressure
(the step leaves velocities at zero). `roofline`: algorithmic bytes of the
fused force kernel per launch over its event-timed duration.
`cpu_baseline`: the CPU restatement of the reference's OpenMP path on this
host's cores, on a bounded number of steps of the same workload.

With torchrun (N > 1) every rank advances its own replica of the workload
(the single-simulation path does not shard; replicas only) and the max over
ranks of the device time is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mechanics agent-steps/s at 1 B200 (FP64 vs FP32-force vs batched) vs OpenMP host"
UNIT = "agent-steps/s"

WORKLOADS = {
    "config3": "3-D 88,700 agents in a ball r=1300 um (4000 um cube, 134^3 mechanics voxels), "
               "3 cell types, 20% with 1-3 springs k=0.05, dt 0.1 min, FP64",
    "config2": "3-D 14,300 agents in a ball r=450 um (2000 um cube), 2 types, BM walls on, FP64",
    "config5": "3-D 1,000,000 agents in a ball r=2900 um (8000 um cube), 2 types, division 1e-4 / death 5e-5 "
               "per step, FP64",
    "config1": "2-D 900 agents in 2000x2000 um, one type, FP64",
}


ENSEMBLE = ("256 independent 3-D replicates, N_r log-uniform in [500, 50000], cube side (8000 N_r)^(1/3) um "
            "(one agent per 8000 um^3), one type, FP64, one batched state")


def make_workload(name):
    from paraphysicell_b200 import workloads as wl
    return {"config1": wl.config1, "config2": wl.config2, "config3": wl.config3, "config5": wl.config5}[name]()


def phenotype_args(name):
    from paraphysicell_b200 import workloads as wl
    return (wl.P_DIVIDE, wl.P_DEATH) if name == "config5" else None


def algorithmic_bytes_per_agent(dims, ndefs, walls, springs_per_agent, spring_agents_fraction, produces=False):
    """Bytes the fused force pass must move per agent: reads of position,
    previous velocity, the four pair parameters (radius, repulsion,
    adhesion, rmad), the BM strength when walls are on, the affinity row,
    definition index and movable flag; writes of position, previous velocity
    and pressure; spring rows (count, elastic constant, partner indices).
    `produces`: the pass also does the mesh rebuild's per-agent work (launch
    shapes -3 and -4 in a step without the phenotype update) and writes the
    agent's voxel key (4 B), its entry of the order (8 B) and its next
    key-ordered position in double and single precision (32 + 16 B)."""
    s = 8
    reads = 8 * dims + 8 * dims + 4 * s + (s if walls else 0) + s * ndefs + 4 + 1
    writes = 8 * dims + 8 * dims + s + (4 + 8 + 32 + 16 if produces else 0)
    springs = 4 + spring_agents_fraction * s + 4 * springs_per_agent
    return reads + writes + springs


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        rows = []
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[2 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def error_vs_oracle(name, steps=3):
    """The device's FP64 step against the oracle's serial restatement of the
    reference on the same workload, outside the timed region: `steps` steps
    from the same state, then the largest relative difference of the step's
    velocity (previous_velocities after update_positions) over agents, the
    largest position difference, the number of agents whose neighbour list
    (as the reference orders it) differs, and whether the voxel bins agree."""
    from oracle.oracle import Oracle
    from paraphysicell_b200.abi import AgentArrays
    from paraphysicell_b200.device import Simulation

    mesh, params, a = make_workload(name)
    ph = phenotype_args(name)
    o = Oracle(mesh, params, seed=1)
    o.upload(a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    d = Simulation(mesh, params, a.capacity, seed=1)
    d.upload(a)
    d.update_mechanics_mesh()
    if ph:
        o.step(steps, 1, ph[0], ph[1])
        d.step_with_phenotype(steps, ph[0], ph[1])
    else:
        o.step(steps, 0, 0.0, 0.0)
        d.step(steps)

    def fetch(x):
        out = AgentArrays(0, a.dims, a.ndefs, a.capacity, a.spring_capacity)
        out.count = out.capacity
        x.download(out)
        return out

    go, gd = fetch(o), fetch(d)
    res = {"steps": steps, "agents": int(go.count), "same_count": go.count == gd.count,
           "same_ids": bool(go.count == gd.count and np.array_equal(go["agent_ids"], gd["agent_ids"]))}
    if res["same_ids"]:
        vo, vd = go["previous_velocities"], gd["previous_velocities"]
        scale = max(float(np.max(np.linalg.norm(vo, axis=1))), 1e-300)
        res["max_rel_velocity_err_vs_oracle"] = float(np.max(np.linalg.norm(vd - vo, axis=1)) / scale)
        res["max_abs_position_diff_um"] = float(np.max(np.abs(gd["positions"] - go["positions"])))
        res["velocity_bit_exact"] = bool(np.array_equal(vo, vd))
        no, nd = o.neighbors(), d.neighbors()
        res["neighbor_mismatches"] = int(sum(1 for x, y in zip(no, nd) if x != y))
        co, ao = o.mesh_bins()
        cd, ad = d.mesh_bins()
        res["bins_equal"] = bool(np.array_equal(co, cd) and np.array_equal(ao, ad))
    d.close()
    return res


def cpu_baseline(name, budget_s=8.0, max_steps=400, with_error=True):
    """Times the oracle's OpenMP restatement of the reference on all host
    threads for a bounded number of steps of the workload, then (with_error)
    checks the device's FP64 step against the oracle's serial form of the
    same workload (error_vs_oracle)."""
    from oracle.oracle import Oracle

    threads = len(os.sched_getaffinity(0))
    mesh, params, a = make_workload(name)
    o = Oracle(mesh, params, seed=1)
    o.upload(a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    ph = phenotype_args(name)
    kw = dict(with_phenotype=ph is not None, p_divide=ph[0] if ph else 0.0, p_death=ph[1] if ph else 0.0)
    t = o.time_steps(2, threads, **kw)  # warm-up and step-time estimate
    steps = int(max(3, min(max_steps, budget_s / max(t / 2, 1e-6))))
    t = o.time_steps(steps, threads, **kw)
    out = {"value": a.count * steps / t, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"{steps} steps of the full {a.count}-agent workload, OpenMP over {threads} threads, "
                     f"std::chrono around the step loop ({t:.2f} s)"}
    if with_error:
        out["error_vs_oracle"] = error_vs_oracle(name)
    return out


def ensemble_cpu_baseline(steps=2):
    """The ensemble on the host: every replicate in turn through the oracle's
    OpenMP restatement on all host threads, `steps` steps each (only the
    step loops are timed)."""
    from oracle.oracle import Oracle
    from paraphysicell_b200 import workloads as wl

    threads = len(os.sched_getaffinity(0))
    meshes, params, sets = wl.config4()
    total_t, agent_steps = 0.0, 0
    for m, a in zip(meshes, sets):
        o = Oracle(m, params, seed=1)
        o.upload(a)
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
        total_t += o.time_steps(steps, threads)
        agent_steps += a.count * steps
    return {"value": agent_steps / total_t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"all {len(sets)} replicates one after another, {steps} steps each, OpenMP over {threads} "
                      f"threads, std::chrono around each replicate's step loop ({total_t:.2f} s in total)"}


def max_over_ranks(x, device):
    """Largest value of x over all ranks of the default process group (the
    job's time is its slowest rank's); `device` "cuda" under NCCL, "cpu"
    under gloo."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank, world):
    """`--impl reference`: the reference's CPU path (its OpenMP structure as
    restated by the oracle; the reference itself cannot be built here) on
    all host threads, K timed steps after W warm-up steps."""
    if rank != 0:
        return
    from oracle.oracle import Oracle

    threads = len(os.sched_getaffinity(0))
    mesh, params, a = make_workload(args.workload)
    o = Oracle(mesh, params, seed=1)
    o.upload(a)
    o.update_mechanics_mesh()
    o.update_cell_neighbors()
    ph = phenotype_args(args.workload)
    kw = dict(with_phenotype=ph is not None, p_divide=ph[0] if ph else 0.0, p_death=ph[1] if ph else 0.0)
    o.time_steps(args.warmup, threads, **kw)
    t = o.time_steps(args.steps, threads, **kw)
    value = a.count * args.steps / t  # one host runs one simulation, whatever the rank count
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload], "agents": a.count},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} timed steps of the full workload after {args.warmup} warm-up "
                                   f"steps, OpenMP over {threads} threads (reference not buildable here: "
                                   f"paraBioFVM/pugixml/googletest absent)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fp32_form(args, mesh, params, a, ph, flush):
    """The FP32-force form on the same workload and timing protocol, and its
    error against the FP64 form after one step from the same state."""
    import torch

    from paraphysicell_b200.abi import PPC_FP32_FORCE, AgentArrays
    from paraphysicell_b200.device import Simulation

    def make(precision):
        sim = Simulation(mesh, params, a.capacity, seed=1)
        st = torch.cuda.Stream()
        sim.set_stream(st.cuda_stream)
        if precision:
            sim.set_precision(precision)
        sim.upload(a)
        sim.update_mechanics_mesh()
        return sim, st

    def step(sim, k):
        if ph:
            sim.step_with_phenotype(k, ph[0], ph[1])
        else:
            sim.step(k)

    def fetch(sim):
        out = AgentArrays(0, a.dims, a.ndefs, a.capacity, a.spring_capacity)
        out.count = out.capacity
        sim.download(out, fields=("positions", "previous_velocities", "agent_ids"))
        return out

    s64, _ = make(0)
    s32, st = make(PPC_FP32_FORCE)
    step(s64, 1)
    step(s32, 1)
    g64, g32 = fetch(s64), fetch(s32)
    v64, v32 = g64["previous_velocities"], g32["previous_velocities"]
    norm = np.linalg.norm(v64, axis=1)
    err = float(np.max(np.linalg.norm(v32 - v64, axis=1)) / max(np.max(norm), 1e-300))
    s64.close()
    K = args.steps
    with torch.cuda.stream(st):
        shape = s32.autotune(steps=3)
        step(s32, max(args.warmup, 3))
    s32.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    torch.cuda.synchronize()
    with torch.cuda.stream(st):
        for k in range(K):
            flush.zero_()
            starts[k].record(st)
            step(s32, 1)
            ends[k].record(st)
    torch.cuda.synchronize()
    total_ms = sum(x.elapsed_time(y) for x, y in zip(starts, ends))
    fused_ms, fused_n = fused_pass_time(s32, st, lambda k: step(s32, k), flush, min(K, 50))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        step(s32, 10)  # captures the step graph outside the timed region
        e0.record(st)
        step(s32, max(K, 10))
        e1.record(st)
    torch.cuda.synchronize()
    steady = a.count * max(K, 10) / (e0.elapsed_time(e1) / 1e3)
    s32.close()
    return {"value": a.count * K / (total_ms / 1e3), "unit": UNIT, "ms_per_step": total_ms / K,
            "steady_state": steady, "fused_avg_us": fused_ms / max(fused_n, 1) * 1e3,
            "launch_shape": {"tile_edge": shape[0], "threads": shape[1], "chosen_by": "ppc_autotune"},
            "velocity_rel_err_vs_fp64": err,
            "note": "pair forces in FP32 (Neumaier-compensated sums), exact FP64 neighbour predicate, FP64 "
                    "positions/binning/integration; same L2-flushed protocol as value"}


def e2e_form(sim, host, step, K, world, mode):
    """End to end through the C ABI: every step uploads positions and previous
    velocities from pinned host rows, steps, and downloads positions, previous
    velocities and pressure (the step's result: update_positions leaves the
    step's velocity in previous_velocities and zeroes velocities,
    src/solver/host/position_solver.cpp:481-504). Host clock and CUDA events
    around the loop; the larger is reported."""
    import torch

    sim.set_host_transfer(mode)
    sim.upload(host)
    sim.update_mechanics_mesh()
    up_fields = ("positions", "previous_velocities")
    down_fields = ("positions", "previous_velocities", "simple_pressure")
    d = host.dims
    sim.download(host, fields=down_fields)
    torch.cuda.synchronize()
    counts = []
    E = max(3, min(K, 50))
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    for k in range(E):
        sim.upload_fields(host, up_fields)
        step(1)
        sim.download(host, fields=down_fields)
        counts.append(host.count)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    del stream
    ms = wall * 1e3
    n = float(sum(counts))
    sim.set_host_transfer(0)
    return {"value": n / (ms / 1e3) * world, "unit": UNIT,
            "h2d_bytes_per_step": int(np.mean(counts) * 2 * 8 * d),
            "d2h_bytes_per_step": int(np.mean(counts) * (2 * 8 * d + 8)),
            "steps": E, "ms_per_step": ms / E,
            "transfer": "copy engine + (un)pack kernels" if mode == 0 else "zero-copy (un)pack kernels"}


def host_link_peak(h2d_bytes, d2h_bytes, reps=5):
    """Plain pinned cudaMemcpyAsync of the e2e step's byte counts, one copy
    per direction, best of `reps` (CUDA events): the host link's ceiling for
    the e2e leg."""
    import torch

    out = {}
    for name, nbytes, h2d in (("h2d_gbs", h2d_bytes, True), ("d2h_gbs", d2h_bytes, False)):
        hbuf = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        dbuf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        best = None
        for _ in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if h2d:
                dbuf.copy_(hbuf, non_blocking=True)
            else:
                hbuf.copy_(dbuf, non_blocking=True)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name] = nbytes / (best * 1e-3) / 1e9
    out["note"] = "pinned cudaMemcpyAsync of the e2e step's bytes, one copy per direction, best of 5"
    return out


def fused_pass_time(sim, stream, step, flush, n):
    """Total device time of the fused pass over n L2-flushed steps, from the
    library's events around it, and the number of launches timed."""
    import torch

    torch.cuda.synchronize()
    sim.set_profiling(True)
    with torch.cuda.stream(stream):
        for _ in range(n):
            flush.zero_()
            step(1)
    torch.cuda.synchronize()
    ms, launches = sim.profile()
    sim.set_profiling(False)
    return ms, launches


def _timed_steps(sim, stream, step, count, K, warmup, flush):
    """Device-timed K steps with L2 flushed before each, the fused pass's
    average duration, and back-to-back (graph-replayed) steady state."""
    import torch

    with torch.cuda.stream(stream):
        step(max(warmup, 3))
    sim.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    agent_steps = 0.0
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(K):
            n = count()
            flush.zero_()
            starts[k].record(stream)
            step(1)
            ends[k].record(stream)
            agent_steps += 0.5 * (n + count())
    torch.cuda.synchronize()
    total_ms = sum(x.elapsed_time(y) for x, y in zip(starts, ends))
    fused_ms, fused_n = fused_pass_time(sim, stream, step, flush, min(K, 50))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        step(10)  # captures the step graph outside the timed region
    n0 = count()
    with torch.cuda.stream(stream):
        e0.record(stream)
        step(max(K, 10))
        e1.record(stream)
    torch.cuda.synchronize()
    steady = 0.5 * (n0 + count()) * max(K, 10) / (e0.elapsed_time(e1) / 1e3)
    return {"value": agent_steps / (total_ms / 1e3), "unit": UNIT, "ms_per_step": total_ms / K,
            "steady_state": steady, "fused_avg_us": fused_ms / max(fused_n, 1) * 1e3}


def persistent_form(args, mesh, params, a, flush):
    """The same single simulation with each step as one cooperative launch
    (ppc_set_step_form(PPC_STEP_PERSISTENT)), after the autotuner chose the
    fused pass's shape in the kernels form; same L2-flushed protocol."""
    import torch

    from paraphysicell_b200.abi import PPC_STEP_PERSISTENT
    from paraphysicell_b200.device import Simulation

    sim = Simulation(mesh, params, a.capacity, seed=1)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.upload(a)
    sim.update_mechanics_mesh()
    with torch.cuda.stream(stream):
        shape = sim.autotune(steps=3)
    sim.set_step_form(PPC_STEP_PERSISTENT)
    res = _timed_steps(sim, stream, sim.step, lambda: a.count, args.steps, args.warmup, flush)
    sim.close()
    res.pop("fused_avg_us", None)
    res["launch_shape"] = {"tile_edge": shape[0], "threads": shape[1], "chosen_by": "ppc_autotune"}
    return res


def ensemble_form(args, flush):
    """Config 4: 256 independent replicates of 500..50,000 agents in one
    batched state (one launch per kernel per step for all replicates, CUDA
    graphs over blocks of steps)."""
    import torch

    from paraphysicell_b200 import workloads as wl
    from paraphysicell_b200.device import Simulation

    from paraphysicell_b200.abi import PPC_FP32_FORCE, PPC_STEP_PERSISTENT

    meshes, params, sets = wl.config4()
    total = sum(a.count for a in sets)

    def run(precision):
        sim = Simulation(meshes, params, [a.capacity for a in sets], seed=1)
        stream = torch.cuda.Stream()
        sim.set_stream(stream.cuda_stream)
        if precision:
            sim.set_precision(precision)
        for r, a in enumerate(sets):
            sim.upload(a, replicate=r)
        sim.update_mechanics_mesh()
        with torch.cuda.stream(stream):
            shape = sim.autotune(steps=5)
        res = _timed_steps(sim, stream, sim.step, lambda: total, args.steps, args.warmup, flush)
        res["launch_shape"] = {"tile_edge": shape[0], "threads": shape[1], "chosen_by": "ppc_autotune"}
        # the same steps as one cooperative launch each (ppc_set_step_form)
        sim.set_step_form(PPC_STEP_PERSISTENT)
        per = _timed_steps(sim, stream, sim.step, lambda: total, args.steps, args.warmup, flush)
        res["persistent"] = {"value": per["value"], "ms_per_step": per["ms_per_step"],
                             "steady_state": per["steady_state"]}
        sim.close()
        return res

    out = run(0)
    out["fp32_force"] = run(PPC_FP32_FORCE)
    out.update({"workload": "config4", "replicates": len(sets), "agents": total,
                "description": ENSEMBLE})
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = ensemble_cpu_baseline()
    return out


def stochastic_springs_form(args, flush):
    """Config 3 with non-zero spring attachment (0.8 /min) and detachment
    (0.3 /min) rates and at most 3 springs per agent: the step runs the
    separate kernels with the stochastic spring update."""
    import torch

    from paraphysicell_b200 import workloads as wl
    from paraphysicell_b200.device import Simulation

    mesh, params, a = wl.config3()
    a.arrays["attachment_rate"][: a.count] = 0.8
    a.arrays["detachment_rate"][: a.count] = 0.3
    a.arrays["maximum_number_of_attachments"][: a.count] = 3
    sim = Simulation(mesh, params, a.capacity, seed=1)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.upload(a)
    sim.update_mechanics_mesh()
    out = _timed_steps(sim, stream, sim.step, lambda: a.count, args.steps, args.warmup, flush)
    sim.close()
    out.update({"workload": "config3 + spring rates", "agents": a.count,
                "note": "attachment 0.8/min, detachment 0.3/min, max 3 springs; separate kernels per step"})
    return out


def interactions_form(args):
    """Config 3 (88,700 agents) through ppc_update_cell_cell_interactions at
    two rate settings (per-neighbour action probabilities of a few per mille,
    and up to 0.2). `resident`: the phenotype fields are uploaded once
    (ppc_upload_interactions) and each call works on the device columns;
    `per_call_fields`: each call copies page-locked fields in and out. Calls
    are synchronous, so each is timed on the host clock. `cpu` is the
    oracle's serial restatement of the reference's loop
    (src/solver/host/interactions_solver.cpp:143-251) on the same first call."""
    import time

    from oracle.oracle import Oracle
    from paraphysicell_b200 import workloads as wl
    from paraphysicell_b200.abi import FLAG_TO_REMOVE, AgentArrays
    from paraphysicell_b200.device import PinnedPool, Simulation

    out = {"workload": "config3 cell-cell interactions", "calls": args.steps,
           "note": "host clock around each synchronous call; median over calls"}
    for label, scale in (("low_rates", 0.02), ("high_rates", 1.0)):
        mesh, params, a = wl.config3()
        pool = PinnedPool()
        f = wl.interaction_fields(a, params.cell_definitions_count, seed=9, scale=scale, pinned=pool)
        res = {"rate_scale": scale, "agents": a.count}
        for form in ("resident", "per_call_fields"):
            sim = Simulation(mesh, params, a.capacity, seed=1)
            sim.upload(a)
            sim.update_mechanics_mesh()
            sim.update_cell_neighbors()
            g = f.copy(pinned=pool)
            if form == "resident":
                sim.upload_interactions(g)
                call = lambda: sim.update_cell_cell_interactions(None)  # noqa: E731
            else:
                call = lambda: sim.update_cell_cell_interactions(g)  # noqa: E731
            call()
            sim.synchronize()
            times = []
            for _ in range(max(3, min(args.steps, 50))):
                t0 = time.perf_counter()
                call()
                times.append(time.perf_counter() - t0)
            res[form + "_ms_per_call"] = 1e3 * float(np.median(times))
            if form == "resident":
                b = AgentArrays(a.count, a.dims, a.ndefs, a.capacity)
                sim.download(b)
                res["flagged_for_removal_after_calls"] = int(np.count_nonzero(b["flags"][: b.count] == FLAG_TO_REMOVE))
            sim.close()
        o = Oracle(mesh, params, seed=1)
        o.upload(a)
        o.update_mechanics_mesh()
        o.update_cell_neighbors()
        o.upload_interactions(f.copy())
        t0 = time.perf_counter()
        o.update_cell_cell_interactions(None)
        res["cpu_ms_per_call"] = 1e3 * (time.perf_counter() - t0)
        res["cpu_kind"] = "oracle, serial restatement, first call"
        out[label] = res
        pool.free()
    return out


def config5_form(args, flush):
    """Config 5: 1,000,000 agents with division and death every step."""
    import torch

    from paraphysicell_b200 import workloads as wl
    from paraphysicell_b200.device import Simulation

    mesh, params, a = wl.config5()
    sim = Simulation(mesh, params, a.capacity, seed=1)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.upload(a)
    sim.update_mechanics_mesh()
    with torch.cuda.stream(stream):
        shape = sim.autotune(steps=5)
    out = _timed_steps(sim, stream, lambda k: sim.step_with_phenotype(k, wl.P_DIVIDE, wl.P_DEATH), sim.count,
                       args.steps, args.warmup, flush)
    out["launch_shape"] = {"tile_edge": shape[0], "threads": shape[1], "chosen_by": "ppc_autotune"}
    divisions, deaths = sim.event_counts()
    sim.close()
    out.update({"workload": "config5", "agents": a.count, "divisions": divisions, "deaths": deaths,
                "description": WORKLOADS["config5"]})
    out["fp32_force"] = fp32_form(args, mesh, params, a, (wl.P_DIVIDE, wl.P_DEATH), flush)
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline("config5", budget_s=10.0, with_error=False)
    return out


def run_ours(args, rank, world, local_rank):
    import torch

    from paraphysicell_b200 import build
    from paraphysicell_b200.abi import PPC_TRANSFER_COPY_ENGINE, PPC_TRANSFER_ZERO_COPY, AgentArrays
    from paraphysicell_b200.device import PinnedPool, Simulation

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local_rank)
    build.ensure_built()

    mesh, params, a = make_workload(args.workload)
    ph = phenotype_args(args.workload)
    n0 = a.count
    stream = torch.cuda.Stream()
    sim = Simulation(mesh, params, a.capacity, seed=1)
    sim.set_stream(stream.cuda_stream)
    sim.upload(a)
    sim.update_mechanics_mesh()

    def step(k):
        if ph:
            sim.step_with_phenotype(k, ph[0], ph[1])
        else:
            sim.step(k)

    # the fused pass's launch shape, timed over real steps (ppc_autotune)
    # unless given; the trajectory does not depend on it
    if args.launch_shape is None:
        with torch.cuda.stream(stream):
            shape = sim.autotune(steps=3)
        chosen_by = "ppc_autotune"
    else:
        shape = (args.launch_shape, 128)
        sim.set_launch_shape(args.launch_shape, 128, 32 * 1024 if args.launch_shape == 0 else 0)
        chosen_by = "--launch-shape"

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    with torch.cuda.stream(stream):
        step(max(args.warmup, 3))
    sim.synchronize()

    # ---- value: K steps, L2 flushed before each, device-timed ----
    K = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    counts = []
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = sim.launches()
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.__enter__()
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.zero_()
            starts[k].record(stream)
            step(1)
            ends[k].record(stream)
            if ph:
                counts.append(sim.count())
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__(None, None, None)
    launches = sim.launches() - l0
    sim.synchronize()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    agent_steps = float(sum(counts)) if ph else float(n0 * K)
    if world > 1:
        total_ms = max_over_ranks(total_ms, "cuda")
        agent_steps *= world
        torch.distributed.barrier()
    value = agent_steps / (total_ms / 1e3)

    # ---- the fused pass alone: events around it (which stop the next
    # kernel from overlapping its launch, so they stay out of `value`) ----
    fused_ms, fused_launches = fused_pass_time(sim, stream, step, flush, min(K, 50))

    # ---- steady state: graph-replayed back-to-back steps (L2 warm) ----
    with torch.cuda.stream(stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        step(10)  # captures the step graph outside the timed region
        e0.record(stream)
        step(max(K, 10))
        e1.record(stream)
    torch.cuda.synchronize()
    steady = (n0 * max(K, 10)) / (e0.elapsed_time(e1) / 1e3)

    # ---- e2e through the C ABI with pinned host buffers ----
    pool = PinnedPool()
    host = AgentArrays(n0, a.dims, a.ndefs, a.capacity, a.spring_capacity, pinned=pool)
    for k_, v_ in a.arrays.items():
        host.arrays[k_][:] = v_
    e2e = e2e_form(sim, host, step, K, world, PPC_TRANSFER_COPY_ENGINE)
    e2e["zero_copy"] = e2e_form(sim, host, step, K, world, PPC_TRANSFER_ZERO_COPY)["value"]
    link = host_link_peak(e2e["h2d_bytes_per_step"], e2e["d2h_bytes_per_step"])
    e2e["host_link"] = link
    device_us = total_ms / K * 1e3
    bound_us = (e2e["h2d_bytes_per_step"] / (link["h2d_gbs"] * 1e3) + e2e["d2h_bytes_per_step"] / (link["d2h_gbs"] * 1e3)
                + device_us)
    e2e["bound_us_per_step"] = bound_us
    e2e["us_per_step"] = e2e["ms_per_step"] * 1e3
    e2e["vs_bound"] = e2e["us_per_step"] / bound_us
    pool_free = pool.free

    if rank != 0:
        sim.close()
        del host
        pool_free()
        return

    import json as _json
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = _json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak = 6650.0
        peak_src = "fallback"
    spring_counts = a.arrays["spring_counts"][:n0]
    per_agent = algorithmic_bytes_per_agent(a.dims, a.ndefs, bool(params.virtual_wall_at_domain_edges),
                                            float(spring_counts.mean()), float((spring_counts > 0).mean()),
                                            produces=shape[0] in (-3, -4) and ph is None)
    fused_avg_ms = fused_ms / max(fused_launches, 1)
    achieved = (per_agent * n0) / (fused_avg_ms / 1e3) / 1e9
    traffic = None
    kernel_name = {-3: "k_fused_flat", -4: "k_fused_queue"}.get(shape[0], "k_fused_staged")
    prof = os.path.join(ROOT, "profiles", f"{kernel_name}_{args.workload}.md")
    if os.path.exists(prof):
        for line in open(prof):
            if line.startswith("| dram_bytes_per_launch |"):
                traffic = float(line.split("|")[2])

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload], "agents": n0,
                   "l2": "flushed (256 MiB write) before every timed step", "form": "FP64 drop-in",
                   "launch_shape": {"tile_edge": shape[0], "threads": shape[1], "chosen_by": chosen_by},
                   "parallelism": f"replicas x{world}" if world > 1 else "single simulation"},
        "steady_state": {"value": steady, "unit": UNIT, "note": "back-to-back graph-replayed steps, L2 warm"},
        "roofline": {"bound": "hbm", "kernel": f"{kernel_name} (fused pass: neighbour search + forces + membrane + "
                                                 "springs + AB2)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic, "bytes_per_agent": per_agent,
                     "avg_launch_us": fused_avg_ms * 1e3, "launches": fused_launches},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": sampler.summary() if sampler else None,
    }
    if not args.no_forms:
        line["forms"] = {"fp32_force": fp32_form(args, mesh, params, a, ph, flush)}
        if ph is None:
            line["forms"]["persistent_step"] = persistent_form(args, mesh, params, a, flush)
        if args.workload == "config3":
            line["forms"]["batched_ensemble"] = ensemble_form(args, flush)
            line["forms"]["config5_division_death"] = config5_form(args, flush)
            line["forms"]["stochastic_springs"] = stochastic_springs_form(args, flush)
            line["forms"]["cell_cell_interactions"] = interactions_form(args)
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args.workload)
        line["error_vs_oracle"] = line["cpu_baseline"].pop("error_vs_oracle")
    print(json.dumps(line), flush=True)
    sim.close()
    del host
    pool_free()


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="config3", choices=sorted(WORKLOADS))
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-forms", action="store_true", help="skip the FP32-force form's measurement")
    p.add_argument("--launch-shape", type=int, default=None, choices=[-4, -3, -2, -1, 0],
                   help="fused-pass launch shape of the main line (default: ppc_autotune picks)")
    args = p.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if args.impl == "ours":
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
