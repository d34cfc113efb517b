// Cell-cell interactions on the device: phagocytosis of dead and live
// neighbours, attack and fusion (reference:
// src/solver/host/interactions_solver.cpp:1-265).
//
// The reference walks every live agent's neighbour list under a mutex; each
// neighbour costs one uniform draw, and an action re-checks the removal flags
// of both agents before it changes anything. The outcome therefore depends on
// the order in which agents act. This implementation fixes the order of a
// one-thread run (agents in index order, neighbours in list order) and
// reaches it in three passes:
//  1. k_ix_candidates, one thread per agent: draws every neighbour's number and
//     keeps the neighbours for which some action's threshold passes (the draw
//     and the rates do not depend on any other agent's actions); it also
//     checks that no neighbour list was cut at the list capacity;
//  2. k_ix_independent: an agent's walk reads and writes only itself and its
//     candidate neighbours, so a walk whose agents appear in no earlier walk
//     sees the state a one-thread run would show it, whatever runs beside
//     it. Each such agent (found with a per-slot atomicMin of the first walk
//     that touches the slot) walks at once, in parallel with the others; the
//     rest are marked;
//  3. k_ix_ordered, one block, after every independent walk has finished:
//     the marked agents in waves, each wave the walks that no earlier
//     pending walk shares an agent with, all at once.
// With the rates of a real model nearly every walk is independent.

#include <cuda_runtime.h>

#include "../../include/ppc_draws.h"
#include "ppc_internal.cuh"

namespace ppc {
namespace {

constexpr int kIxThreads = 256;
constexpr int kIxResolveThreads = 1024;
constexpr double kZeroThreshold = 1e-16; // reference: solver_helper.h:12
constexpr double kPi = 3.141592653589793;

__global__ void __launch_bounds__(kIxThreads) k_ix_candidates(view v, ix_fields x)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= x.n)
		return;
	int m = 0;
	const int s = x.base + i;
	if (v.ncnt[s] > v.ncap)
		atomicOr(x.status, 1); // a cut list: the walks below would miss neighbours
	if (x.dead[i] != 1)
	{
		const int nn = min(v.ncnt[s], v.ncap);
		const int D = v.ndefs;
		const double dt = x.dt;
		const int di = v.def[s];
		for (int k = 0; k < nn; k++)
		{
			const int j = v.nidx[(int64_t)s * v.ncap + k] - x.base;
			if ((unsigned)j >= (unsigned)x.n)
				continue; // a list older than the last removal: skip, never read past the rows
			const double r
				= ppc_uniform(v.seed, x.epoch, (uint64_t)x.replicate, (uint64_t)i, PPC_DRAW_INTERACTION + (uint64_t)k);
			bool any;
			if (x.dead[j] == 1)
				any = r < x.dead_phago[i] * dt;
			else
			{
				const int dj = v.def[x.base + j];
				any = r < x.live_phago[(int64_t)i * D + dj] * dt
					  || r < x.attack[(int64_t)i * D + dj] * x.immuno[(int64_t)j * D + di] * dt
					  || r < x.fusion[(int64_t)i * D + dj] * dt;
			}
			if (any)
				x.cand[(int64_t)i * v.ncap + m++] = k;
		}
	}
	x.ncand[i] = m;
	// the first walk that touches each slot (first_end is INT32_MAX between uses)
	if (m > 0)
	{
		atomicMin(v.first_end + s, i);
		for (int c = 0; c < m; c++)
			atomicMin(v.first_end + v.nidx[(int64_t)s * v.ncap + x.cand[(int64_t)i * v.ncap + c]], i);
	}
}

__device__ void ix_geometry(const view& v, int s)
{
	// interactions_solver.cpp:89-96 (update_geometry)
	const double four_thirds_pi = kPi * 4.0 / 3.0;
	double4 prm = v.prm[s];
	prm.x = ppc_cbrt(v.vol[s] / four_thirds_pi);
	v.prm[s] = prm;
	v.nrad[s] = ppc_cbrt(v.nvol[s] / four_thirds_pi);
	v.sarea[s] = 4.0 * kPi * prm.x * prm.x;
}

// ingest_volume + ingest_internalized + update_geometry (interactions_solver.cpp:6-26,64-74,98-112)
__device__ void ix_ingest(const view& v, const ix_fields& x, int l, int r)
{
	const int sl = x.base + l, sr = x.base + r;
	x.cyto_fluid[l] += x.fluid[r];
	x.cyto_solid[l] += x.solid[r];
	x.fluid[l] += x.fluid[r];
	x.solid[l] += x.solid[r];
	x.cyto[l] += x.fluid[r] + x.solid[r];
	v.vol[sl] += x.fluid[r] + x.solid[r];
	x.fluid_fraction[l] = x.fluid[l] / (v.vol[sl] + kZeroThreshold);
	x.c2n[l] = x.cyto_solid[l] / (x.nuc_solid[l] + kZeroThreshold);
	const int S = x.substrates;
	for (int q = 0; q < S; q++)
		x.isub[(int64_t)l * S + q] += x.isub[(int64_t)r * S + q] * x.frac[(int64_t)r * S + q];
	ix_geometry(v, sl);
	v.flags[sr] = PPC_FLAG_TO_REMOVE;
}

// fuse_position + fuse_volume + fuse_internalized + update_geometry
// (interactions_solver.cpp:28-53,76-87,114-131)
template <int DIMS>
__device__ void ix_fuse(const view& v, const ix_fields& x, int cur, int l, int r)
{
	const int sl = x.base + l, sr = x.base + r;
	const double vl = v.vol[sl], vr = v.vol[sr];
	const double both = vl + vr;
	double4 pl = v.pos[cur][sl];
	const double4 pr = v.pos[cur][sr];
	pl.x = (pl.x * vl + pr.x * vr) / both;
	if (DIMS >= 2)
		pl.y = (pl.y * vl + pr.y * vr) / both;
	if (DIMS >= 3)
		pl.z = (pl.z * vl + pr.z * vr) / both;
	v.pos[cur][sl] = pl;

	x.cyto_fluid[l] += x.cyto_fluid[r];
	x.nuc_fluid[l] += x.nuc_fluid[r];
	x.cyto_solid[l] += x.cyto_solid[r];
	x.nuc_solid[l] += x.nuc_solid[r];
	x.target_cyto[l] += x.target_cyto[r];
	x.target_nuc[l] += x.target_nuc[r];
	x.fluid[l] = x.nuc_fluid[l] + x.cyto_fluid[l];
	x.solid[l] = x.nuc_solid[l] + x.cyto_solid[l];
	v.nvol[sl] = x.nuc_fluid[l] + x.nuc_solid[l];
	x.cyto[l] = x.cyto_fluid[l] + x.cyto_solid[l];
	v.vol[sl] = v.nvol[sl] + x.cyto[l];
	x.fluid_fraction[l] = x.fluid[l] / (v.vol[sl] + kZeroThreshold);
	x.c2n[l] = x.cyto_solid[l] / (x.nuc_solid[l] + kZeroThreshold);

	const int S = x.substrates;
	for (int q = 0; q < S; q++)
		x.isub[(int64_t)l * S + q] += x.isub[(int64_t)r * S + q];
	ix_geometry(v, sl);
	x.nuclei[l] += x.nuclei[r];
	v.flags[sr] = PPC_FLAG_TO_REMOVE;
}

// update_cell_cell_interactions_internal (interactions_solver.cpp:143-251)
// for one agent, over its candidate neighbours in list order
template <int DIMS>
__device__ void ix_agent(const view& v, const ix_fields& x, int cur, int i)
{
	bool attacked_once = false, phagocytosed_once = false, fused_once = false;
	const int s = x.base + i;
	const int D = v.ndefs;
	const double dt = x.dt;
	const int di = v.def[s];
	const int m = x.ncand[i];
	for (int c = 0; c < m; c++)
	{
		const int k = x.cand[(int64_t)i * v.ncap + c];
		const int j = v.nidx[(int64_t)s * v.ncap + k] - x.base;
		const int sj = x.base + j;
		const double r
			= ppc_uniform(v.seed, x.epoch, (uint64_t)x.replicate, (uint64_t)i, PPC_DRAW_INTERACTION + (uint64_t)k);
		if (x.dead[j] == 1)
		{
			if (r < x.dead_phago[i] * dt)
			{
				if (v.flags[s] == PPC_FLAG_TO_REMOVE)
					break;
				if (v.flags[sj] == PPC_FLAG_TO_REMOVE)
					continue;
				ix_ingest(v, x, i, j);
			}
			continue;
		}
		const int dj = v.def[sj];
		if (!phagocytosed_once && r < x.live_phago[(int64_t)i * D + dj] * dt)
		{
			if (v.flags[s] == PPC_FLAG_TO_REMOVE)
				break;
			if (v.flags[sj] == PPC_FLAG_TO_REMOVE)
				continue;
			ix_ingest(v, x, i, j);
			phagocytosed_once = true;
			continue;
		}
		const double attack_r = x.attack[(int64_t)i * D + dj];
		const double immuno_r = x.immuno[(int64_t)j * D + di];
		if (!attacked_once && r < attack_r * immuno_r * dt)
		{
			if (v.flags[s] == PPC_FLAG_TO_REMOVE)
				break;
			if (v.flags[sj] == PPC_FLAG_TO_REMOVE)
				continue;
			// attack (interactions_solver.cpp:133-141)
			x.damage[j] += x.damage_rate[i] * dt;
			x.attack_time[j] += dt;
			attacked_once = true;
			continue;
		}
		if (!fused_once && r < x.fusion[(int64_t)i * D + dj] * dt)
		{
			if (v.flags[s] == PPC_FLAG_TO_REMOVE)
				break;
			if (v.flags[sj] == PPC_FLAG_TO_REMOVE)
				continue;
			ix_fuse<DIMS>(v, x, cur, i, j);
			fused_once = true;
			continue;
		}
	}
}

// true when no earlier agent's walk touches this agent or its candidates
__device__ __forceinline__ bool ix_independent(const view& v, const ix_fields& x, int i)
{
	const int s = x.base + i;
	if (__ldcg(v.first_end + s) != i)
		return false;
	const int m = x.ncand[i];
	for (int c = 0; c < m; c++)
		if (__ldcg(v.first_end + v.nidx[(int64_t)s * v.ncap + x.cand[(int64_t)i * v.ncap + c]]) != i)
			return false;
	return true;
}

template <int DIMS>
__global__ void __launch_bounds__(kIxThreads) k_ix_independent(view v, ix_fields x, int cur)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= x.n)
		return;
	int dep = 0;
	if (x.ncand[i] > 0 && __ldcg(x.status) == 0)
	{
		if (ix_independent(v, x, i))
			ix_agent<DIMS>(v, x, cur, i);
		else
			dep = 1;
	}
	x.dep[i] = dep;
}

// claims (atomicMin) or releases the slots a walk touches: its agent and
// its candidate neighbours
__device__ __forceinline__ void ix_slots(const view& v, const ix_fields& x, int i, bool claim)
{
	const int s = x.base + i;
	const int m = x.ncand[i];
	if (claim)
		atomicMin(v.first_end + s, i);
	else
		v.first_end[s] = INT32_MAX;
	for (int c = 0; c < m; c++)
	{
		const int q = v.nidx[(int64_t)s * v.ncap + x.cand[(int64_t)i * v.ncap + c]];
		if (claim)
			atomicMin(v.first_end + q, i);
		else
			v.first_end[q] = INT32_MAX;
	}
}

// The marked walks, after every independent one, in waves: each round every
// pending walk claims its slots (the lowest walk index wins a slot), and the
// walks that won all their slots run at once. Such walks share no slot with
// each other or with any earlier pending walk, so each sees what a run on
// one thread in index order would show it; the lowest pending walk always
// runs, so every round makes progress. The rest stay pending, in order. One
// block; first_end is INT32_MAX again when the kernel ends.
template <int DIMS>
__global__ void __launch_bounds__(kIxResolveThreads) k_ix_ordered(view v, ix_fields x, int cur)
{
	const int tid = threadIdx.x, bd = blockDim.x;
	const bool ok = __ldcg(x.status) == 0;
	for (int i = tid; i < x.n; i += bd)
		if (x.ncand[i] > 0)
			ix_slots(v, x, i, false);
	if (!ok)
		return;
	// the marked walks in index order
	int pending = 0;
	for (int i0 = 0; i0 < x.n; i0 += bd)
	{
		const int i = i0 + tid;
		const int has = i < x.n && x.dep[i] != 0;
		int total;
		const int off = block_exclusive_scan(has, total); // synchronises the block
		if (has)
			x.order[pending + off] = i;
		pending += total;
	}
	__syncthreads();
	for (int round = 0; pending > 0 && round <= x.n; round++)
	{
		for (int e = tid; e < pending; e += bd)
			ix_slots(v, x, x.order[e], true);
		__syncthreads();
		for (int e = tid; e < pending; e += bd)
		{
			const int w = x.order[e];
			const int s = x.base + w;
			bool won = __ldcg(v.first_end + s) == w;
			const int m = x.ncand[w];
			for (int c = 0; c < m && won; c++)
				won = __ldcg(v.first_end + v.nidx[(int64_t)s * v.ncap + x.cand[(int64_t)w * v.ncap + c]]) == w;
			if (won)
			{
				ix_agent<DIMS>(v, x, cur, w);
				x.dep[w] = 0;
			}
		}
		__syncthreads();
		for (int e = tid; e < pending; e += bd)
			ix_slots(v, x, x.order[e], false);
		__syncthreads();
		// keep the walks still pending, in order (a chunk's entries are all
		// read before any of them is overwritten, and the writes land below
		// the next chunk)
		int kept = 0;
		for (int e0 = 0; e0 < pending; e0 += bd)
		{
			const int e = e0 + tid;
			const int w = e < pending ? x.order[e] : -1;
			const int keep = w >= 0 && x.dep[w] != 0;
			int total;
			const int off = block_exclusive_scan(keep, total);
			if (keep)
				x.order[kept + off] = w;
			kept += total;
		}
		pending = kept;
		__syncthreads();
	}
}

} // namespace

int launch_interactions(ppc_state* s, const ix_fields& x)
{
	if (x.n == 0)
		return PPC_OK;
	if (int rc = mark_fields_changed(s)) // ingestion and fusion change volumes and radii
		return rc;
	const int b = blocks_for(x.n, kIxThreads);
	k_ix_candidates<<<b, kIxThreads, 0, PPC_LAUNCH(s)>>>(s->v, x);
	if (s->dims == 1)
	{
		k_ix_independent<1><<<b, kIxThreads, 0, PPC_LAUNCH(s)>>>(s->v, x, s->cur);
		k_ix_ordered<1><<<1, kIxResolveThreads, 0, PPC_LAUNCH(s)>>>(s->v, x, s->cur);
	}
	else if (s->dims == 2)
	{
		k_ix_independent<2><<<b, kIxThreads, 0, PPC_LAUNCH(s)>>>(s->v, x, s->cur);
		k_ix_ordered<2><<<1, kIxResolveThreads, 0, PPC_LAUNCH(s)>>>(s->v, x, s->cur);
	}
	else
	{
		k_ix_independent<3><<<b, kIxThreads, 0, PPC_LAUNCH(s)>>>(s->v, x, s->cur);
		k_ix_ordered<3><<<1, kIxResolveThreads, 0, PPC_LAUNCH(s)>>>(s->v, x, s->cur);
	}
	PPC_CUDA(cudaGetLastError());
	return PPC_OK;
}

} // namespace ppc
