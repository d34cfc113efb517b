// ppc_kernels.cu — CUDA kernels of the mechanics timestep (sm_100a).
//
// Built with -fmad=false: every FP64 expression rounds after each operation,
// exactly like the reference compiled for baseline x86-64 (no FMA), so the
// FP64 path reproduces the reference's values bit for bit when operations are
// written in the reference's order. Each kernel cites the reference lines it
// replaces.
#include <cuda_runtime.h>
#include <utility>

#include "../../include/ppc_draws.h"
#include "ppc_internal.cuh"

namespace ppc {
namespace {

constexpr int kThreads = 256;
constexpr int kSortCap = 4096; // list length sorted in shared memory

// Programmatic dependent launch: every kernel of the library is launched
// with programmatic stream serialisation, so its launch and block
// scheduling overlap the tail of the kernel before it, and waits here, before
// its first memory access, until that kernel has finished and its writes are
// visible. Launched without the attribute, the wait returns at once.
__device__ __forceinline__ void grid_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// a fused step's spring update with all rates zero changes no spring but
// still advances the draw epoch, as the reference's loop does
__device__ __forceinline__ void bump_spring_epochs(const view& v)
{
	if (blockIdx.x == 0 && v.auto_springs)
		for (int r = threadIdx.x; r < v.nreps; r += blockDim.x)
			v.ctr[r].spring_epoch++;
}

__device__ __forceinline__ int rep_of(const view& v, int s) { return v.nreps == 1 ? 0 : v.rid[s]; }

__device__ __forceinline__ double comp(const double4& p, int d) { return d == 0 ? p.x : (d == 1 ? p.y : p.z); }

__device__ __forceinline__ void set_comp(double4& p, int d, double x)
{
	if (d == 0)
		p.x = x;
	else if (d == 1)
		p.y = x;
	else
		p.z = x;
}

// a / b and a % b for 0 <= a < 2^31 through the double reciprocal `inv` of
// b: the product is within an ulp-sized error of a / b, so the truncated
// quotient is off by at most one, which the remainder test corrects
__device__ __forceinline__ void divmod_inv(int32_t a, int32_t b, double inv, int32_t& q, int32_t& r)
{
	q = (int32_t)((double)a * inv);
	r = a - q * b;
	if (r >= b)
	{
		q++;
		r -= b;
	}
	else if (r < 0)
	{
		q--;
		r += b;
	}
}

// voxel coordinates of the local key lk (x fastest)
__device__ __forceinline__ void voxel_coords(const rep_info& R, int32_t lk, int& cx, int& cy, int& cz)
{
	int32_t q;
	divmod_inv(lk, R.grid[0], R.inv_grid[0], q, cx);
	divmod_inv(q, R.grid[1], R.inv_grid[1], cz, cy);
}

// slot s is live when its index inside its replicate is below the count
__device__ __forceinline__ bool live(const view& v, int s, int& r, int& local)
{
	r = rep_of(v, s);
	local = s - v.reps[r].base;
	return local < v.ctr[r].count;
}

// ---------------------------------------------------------------------------
// mesh binning: containers_solver::update_mechanics_mesh
// (reference: src/solver/host/containers_solver.cpp:15-56,
//  common_solver.cpp:10-38)
// ---------------------------------------------------------------------------

// voxel coordinate along one axis: truncation of (x - min) / shape, clamped
// into [0, grid); flags positions outside the box and non-finite values
__device__ __forceinline__ int axis_coord(double x, const rep_info& R, int d, int32_t* err)
{
	double q = (x - R.mins[d]) / R.shape[d];
	if (!(q == q))
	{
		atomicOr(err, ERR_NONFINITE);
		return 0;
	}
	int g = R.grid[d];
	if (q <= 0.0)
	{
		if (q <= -1.0)
			atomicOr(err, ERR_OUT_OF_MESH);
		return 0;
	}
	if (q >= (double)g)
	{
		if (x != R.maxs[d])
			atomicOr(err, ERR_OUT_OF_MESH);
		return g - 1;
	}
	return (int)q;
}

// slot d of every resident phenotype column takes slot s's values
__device__ __forceinline__ void copy_columns(const view& v, int dims, int d, int s)
{
	const ix_columns& x = v.ix;
	if (x.dead)
	{
		const int D = v.ndefs, S = x.S;
		x.dead[d] = x.dead[s];
		double* one[] = { x.dead_phago, x.damage_rate, x.damage, x.attack_time, x.fluid, x.solid, x.cyto,
						  x.cyto_fluid, x.cyto_solid, x.nuc_fluid, x.nuc_solid, x.fluid_fraction, x.c2n,
						  x.target_cyto, x.target_nuc };
#pragma unroll
		for (int k = 0; k < 15; k++)
			one[k][d] = one[k][s];
		double* rows_d[] = { x.live_phago, x.attack, x.fusion, x.immuno };
#pragma unroll
		for (int k = 0; k < 4; k++)
			for (int q = 0; q < D; q++)
				rows_d[k][(int64_t)d * D + q] = rows_d[k][(int64_t)s * D + q];
		for (int q = 0; q < S; q++)
		{
			x.frac[(int64_t)d * S + q] = x.frac[(int64_t)s * S + q];
			x.isub[(int64_t)d * S + q] = x.isub[(int64_t)s * S + q];
		}
		x.nuclei[d] = x.nuclei[s];
	}
	const mot_columns& m = v.mot;
	if (m.motile)
	{
		m.motile[d] = m.motile[s];
		m.restrict2d[d] = m.restrict2d[s];
		m.rule[d] = m.rule[s];
		m.persistence[d] = m.persistence[s];
		m.speed[d] = m.speed[s];
		m.bias[d] = m.bias[s];
		m.chemo_index[d] = m.chemo_index[s];
		m.chemo_dir[d] = m.chemo_dir[s];
		for (int q = 0; q < dims; q++)
		{
			m.direction[(int64_t)d * dims + q] = m.direction[(int64_t)s * dims + q];
			m.vector[(int64_t)d * dims + q] = m.vector[(int64_t)s * dims + q];
		}
		for (int q = 0; q < m.S; q++)
			m.sens[(int64_t)d * m.S + q] = m.sens[(int64_t)s * m.S + q];
	}
}

// copies every per-agent field of slot s into slot d (cell_data::remove,
// reference: src/cell_data.cpp:285-313); spring rows were moved by the plan
__device__ __forceinline__ void move_agent(const view& v, int cur, int d, int s)
{
	copy_columns(v, v.dims, d, s);
	v.pos[cur][d] = v.pos[cur][s];
	v.vel[d] = v.vel[s];
	v.vprev[d] = v.vprev[s];
	v.prm[d] = v.prm[s];
	v.rmad[d] = v.rmad[s];
	v.ec[d] = v.ec[s];
	v.arate[d] = v.arate[s];
	v.drate[d] = v.drate[s];
	v.pressure[d] = v.pressure[s];
	v.vol[d] = v.vol[s];
	v.nvol[d] = v.nvol[s];
	v.nrad[d] = v.nrad[s];
	v.sarea[d] = v.sarea[s];
	v.polarity[d] = v.polarity[s];
	v.orient[d] = v.orient[s];
	for (int q = 0; q < v.ndefs; q++)
		v.aff[(int64_t)d * v.ndefs + q] = v.aff[(int64_t)s * v.ndefs + q];
	v.def[d] = v.def[s];
	v.maxatt[d] = v.maxatt[s];
	v.movable[d] = v.movable[s];
	v.flags[d] = v.flags[s];
	v.ids[d] = v.ids[s];
	const int nn = min(v.ncnt[s], v.ncap);
	for (int q = 0; q < nn; q++)
		v.nidx[(int64_t)d * v.ncap + q] = v.nidx[(int64_t)s * v.ncap + q];
	v.ncnt[d] = v.ncnt[s];
}

// The rebuild starts from the previous one. The previous key order lists,
// tile by tile, the slots that were live then (a tile is a run of 2^tshift
// consecutive voxel keys); tprev holds where each tile's agents start in
// that order and how many there were. k_bin_count recomputes every live
// agent's key: an agent whose key stays in its tile keeps its entry of the
// previous order (porder), every other one, and every slot appended since
// (all slots when there is no previous order), is pushed onto one of the 32
// mover chains of its new tile, and the tile counts change by the difference
// (tdelta, and per 1024 tiles sdelta). k_bin_order then orders each tile by
// itself: its start is its previous start plus the changes of the tiles
// before it; its agents are its kept entries and its chains; their per-voxel
// counts, the voxel starts and the order inside a voxel (descending slot,
// the order a serial run of the reference's fetch_sub scatter gives) are
// formed in shared memory. k_bin_copy, a thread per position of the new
// order, writes the key-ordered copies of the agents' fields. Agents rarely
// leave their tile between steps, so the chains are short.

constexpr int kChains = 32;		 // mover chains per tile
constexpr int kSuperShift = 10;	 // tiles per entry of sdelta: 1024
constexpr int kPlaceThreads = 256;
constexpr int kPlaceList = 1024; // agents of a tile listed in shared memory; the rest in global scratch
constexpr int kMaxTileShift = 12;
constexpr int kOrderBatch = 4;  // previous-order entries a thread of k_bin_order loads at once

// the voxel key of slot s of replicate r at positions pos[cur]
__device__ __forceinline__ int32_t voxel_key(const view& v, int cur, int s, int r)
{
	const rep_info& R = v.reps[r];
	const double4 p = v.pos[cur][s];
	const int c0 = axis_coord(p.x, R, 0, v.err);
	const int c1 = v.dims >= 2 ? axis_coord(p.y, R, 1, v.err) : 0;
	const int c2 = v.dims >= 3 ? axis_coord(p.z, R, 2, v.err) : 0;
	return (int32_t)(R.vox_base + c0 + (int64_t)R.grid[0] * (c1 + (int64_t)R.grid[1] * c2));
}

// a hole the compaction plan filled takes its tail agent first
__device__ __forceinline__ void apply_move(const view& v, int cur, int s)
{
	const int src = v.move_src[s];
	if (src >= 0)
	{
		move_agent(v, cur, s, src);
		v.move_src[s] = -1;
		*v.params_changed = 1; // the slot's agent changed: its key-ordered copies are rewritten
	}
}

// pushes slot q onto a mover chain of the tile of `key`
__device__ __forceinline__ void chain_push(const view& v, int q, int32_t key)
{
	const int64_t c = (int64_t)(key >> v.tshift) * kChains + (q & (kChains - 1));
	v.cnext[q] = atomicExch(v.chead + c, q);
}

// adds `amount` to the change of `tile` (negative: none) and of its group of
// 1024 tiles, one atomic per distinct tile of the warp; every lane calls it
__device__ __forceinline__ void tile_change(const view& v, int tile, int amount)
{
	const int lane = threadIdx.x & 31;
	if (!__any_sync(0xffffffffu, tile >= 0))
		return;
	const int key = tile >= 0 ? tile : -1 - lane;
	const unsigned same = __match_any_sync(0xffffffffu, key);
	if (tile >= 0 && lane == __ffs(same) - 1)
		atomicAdd(v.tdelta + tile, amount * __popc(same));
	const int sup = tile >= 0 ? tile >> kSuperShift : -1 - lane;
	const unsigned same_sup = __match_any_sync(0xffffffffu, sup);
	if (tile >= 0 && lane == __ffs(same_sup) - 1)
		atomicAdd(v.sdelta + sup, amount * __popc(same_sup));
}

// The entry at position t of the previous order, and slot t when it was
// appended since the previous rebuild (or there is no previous order).
// Every lane of the warp calls it.
__device__ __forceinline__ void bin_count_body(const view& v, int cur, int t)
{
	const bool ordered = *v.order_valid != 0;
	const bool moves = *v.moves_pending != 0;
	const bool appended = *v.appended != 0;
	const int sh = v.tshift;
	int leave = -1, enter_a = -1, enter_b = -1;
	if (ordered && t < *v.cursor)
	{
		const int q = v.sorted[t];
		const int32_t okey = v.skey[t];
		int2 e = make_int2(-1, -1);
		int r, local;
		if ((unsigned)q < (unsigned)v.total_cap && live(v, q, r, local))
		{
			if (moves)
				apply_move(v, cur, q);
			const int32_t key = voxel_key(v, cur, q, r);
			v.key[q] = key;
			if ((key >> sh) == (okey >> sh))
				e = make_int2(q, key);
			else
			{
				chain_push(v, q, key);
				leave = okey >> sh;
				enter_a = key >> sh;
			}
		}
		else
			leave = okey >> sh;
		v.porder[t] = e;
	}
	int r, local;
	if ((!ordered || appended) && t < v.total_cap && live(v, t, r, local) && local >= (ordered ? v.binned[r] : 0))
	{
		if (moves)
			apply_move(v, cur, t);
		const int32_t key = voxel_key(v, cur, t, r);
		v.key[t] = key;
		chain_push(v, t, key);
		enter_b = key >> sh;
	}
	tile_change(v, leave, -1);
	tile_change(v, enter_a, 1);
	tile_change(v, enter_b, 1);
}

// A conditional rebuild (after an upload of positions) runs only if the
// upload changed some position; its decision goes to bin_active for
// k_bin_order and k_bin_copy.
// `produced`: the fused pass before this rebuild made every entry (see
// produce_entry); the count then has nothing to do unless the compaction
// removed agents since.
__global__ void __launch_bounds__(kThreads) k_bin_count(view v, int cur, int conditional, int produced)
{
	grid_wait();
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const bool active = !conditional || *v.pos_changed != 0 || *v.moves_pending != 0 || *v.appended != 0;
	if (t == 0)
		*v.bin_active = active ? 1 : 0;
	if (!active || (produced && *v.recount == 0))
		return;
	bin_count_body(v, cur, t);
}

// writes the key-ordered copies of slot s at position t (its entries of
// sorted and skey are the order's). Affinity rows of up to four definitions
// are carried in registers.
__device__ __forceinline__ void place_agent(const view& v, int cur, int s, int t, double4* spos4, float4* sposf)
{
	if ((unsigned)s >= (unsigned)v.total_cap || (unsigned)t >= (unsigned)v.total_cap)
	{
		atomicOr(v.err, ERR_LIST_CAPACITY);
		return;
	}
	const int r = rep_of(v, s);
	const double4 prm = v.prm[s];
	double4 p = v.pos[cur][s];
	const double rmad = v.rmad[s];
	const long long bits = (long long)(uint32_t)v.def[s] | ((long long)(v.movable[s] != 0) << 32)
						   | ((long long)min(v.scnt[s], 255) << 40) | ((long long)(r & 0xffff) << 48);
	const int D = v.ndefs;
	double aff[4];
#pragma unroll
	for (int q = 0; q < 4; q++)
		aff[q] = q < D ? v.aff[(int64_t)s * D + q] : 0.0;
	const rep_info& R = v.reps[r];
	const double m0 = R.mins[0], m1 = R.mins[1], m2 = R.mins[2];
	p.w = rmad * prm.x; // relative_maximum_adhesion_distance * radius
	spos4[t] = p;
	v.sprm4[t] = make_double4(prm.x, prm.y, prm.z, __longlong_as_double(bits));
#pragma unroll
	for (int q = 0; q < 4; q++)
		if (q < D)
			v.saff[(int64_t)t * D + q] = aff[q];
	for (int q = 4; q < D; q++)
		v.saff[(int64_t)t * D + q] = v.aff[(int64_t)s * D + q];
	// single-precision positions relative to the box minimum: the candidate
	// filter of the fused pass
	sposf[t] = make_float4((float)(p.x - m0), (float)(p.y - m1), (float)(p.z - m2), (float)p.w);
	if (v.f32)
	{
		const int fbits = (int)((uint32_t)(bits & 0xffff) | (uint32_t)((bits >> 32) & 1) << 16
								| (uint32_t)((bits >> 40) & 0xff) << 24);
		v.sprmf[t] = make_float4((float)prm.x, (float)prm.y, (float)prm.z, __int_as_float(fbits));
#pragma unroll
		for (int q = 0; q < 4; q++)
			if (q < D)
				v.safff[(int64_t)t * D + q] = (float)aff[q];
		for (int q = 4; q < D; q++)
			v.safff[(int64_t)t * D + q] = (float)v.aff[(int64_t)s * D + q];
	}
}

struct __align__(16) place_smem
{
	int32_t cnt[1 << kMaxTileShift]; // per-voxel counts, then starts, then ends
	int2 list[kPlaceList];			 // the tile's agents: (slot, voxel inside the tile | previous index << 12)
	int32_t group[kPlaceList];		 // slots grouped by voxel
	int32_t wtot[32];				 // per-warp totals of the voxel scan
	int32_t n;
};

constexpr int kVoxelBits = 12;				   // bits of a list item's voxel inside the tile
constexpr int kPrevLimit = 1 << (31 - kVoxelBits); // previous indices that fit above them

// lists slot s (its list word y: voxel inside the tile | previous index + 1
// above kVoxelBits) at index i; items past the shared list go to the global
// scratch at the tile's start
__device__ __forceinline__ void place_store(const view& v, place_smem& sm, int base, int i, int s, int y)
{
	atomicAdd(&sm.cnt[y & ((1 << kVoxelBits) - 1)], 1);
	if (i < kPlaceList)
		sm.list[i] = make_int2(s, y);
	else if ((int64_t)base + i < v.total_cap)
		v.vsc[base + i] = make_int2(s, y);
}

__device__ __forceinline__ int2 place_item(const view& v, const place_smem& sm, int base, int i)
{
	return i < kPlaceList ? sm.list[i] : v.vsc[base + i];
}

// exclusive scan of cnt[0, 4 ceil(nv / 4)) in place: each warp scans a
// contiguous chunk of 16-byte groups in rows of 32 groups (no bank
// conflicts), then the warps' totals are added
template <int THREADS>
__device__ __forceinline__ void place_scan(place_smem& sm, int nv)
{
	constexpr int NW = THREADS / 32;
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	int4* c4 = reinterpret_cast<int4*>(sm.cnt);
	const int nq = (nv + 3) >> 2;
	const int chunk = ((nq + NW - 1) / NW + 31) & ~31;
	const int q0 = min(w * chunk, nq), q1 = min(q0 + chunk, nq);
	int carry = 0;
	for (int q = q0; q < q1; q += 32)
	{
		const int qq = q + lane;
		const int4 c = qq < q1 ? c4[qq] : make_int4(0, 0, 0, 0);
		const int sum = c.x + c.y + c.z + c.w;
		int incl = sum;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1)
		{
			const int y = __shfl_up_sync(0xffffffffu, incl, o);
			if (lane >= o)
				incl += y;
		}
		if (qq < q1)
		{
			int run = carry + incl - sum;
			int4 out;
			out.x = run;
			run += c.x;
			out.y = run;
			run += c.y;
			out.z = run;
			run += c.z;
			out.w = run;
			c4[qq] = out;
		}
		carry += __shfl_sync(0xffffffffu, incl, 31);
	}
	if (lane == 0)
		sm.wtot[w] = carry;
	__syncthreads();
	int off = 0;
#pragma unroll
	for (int k = 0; k < NW; k++)
		off += k < w ? sm.wtot[k] : 0;
	if (off)
		for (int qq = q0 + lane; qq < q1; qq += 32)
		{
			int4 c = c4[qq];
			c.x += off;
			c.y += off;
			c.z += off;
			c.w += off;
			c4[qq] = c;
		}
	__syncthreads();
}

// Orders tile b of the new order (see above): the voxel starts in vstart,
// sorted, skey and tfresh (1 where a position's agent is new to it) over the
// tile's range, its entry of tprev. The key-ordered copies of the agents'
// fields follow in k_bin_copy, which also readies the counters for the next
// rebuild (bin_finish).
// `on`: the rebuild runs (bin_active; the same for the whole block).
template <int THREADS>
__device__ __forceinline__ void bin_order_tile(const view& v, int b, place_smem& sm, int on)
{
	const int tid = threadIdx.x, lane = tid & 31;
	const int sh = v.tshift;
	const int k0 = b << sh;
	const int nv = min(1 << sh, v.nvox - k0);
	// the loads the tile's start, size and chains need, issued together:
	// the start is the previous start plus the changes of the tiles before,
	// four of them loaded at once per thread
	const bool ordered = *v.order_valid != 0;
	const int2 tp0 = v.tprev[b];
	const int db = v.tdelta[b];
	const int chain = tid < kChains ? v.chead[(int64_t)b * kChains + tid] : -1;
	int part = 0;
	const int sb = b >> kSuperShift;
	for (int j = tid; j < sb; j += THREADS)
		part += v.sdelta[j];
	for (int k = (sb << kSuperShift) + tid; k < b; k += 4 * THREADS)
	{
		const int x0 = v.tdelta[k];
		const int x1 = k + THREADS < b ? v.tdelta[k + THREADS] : 0;
		const int x2 = k + 2 * THREADS < b ? v.tdelta[k + 2 * THREADS] : 0;
		const int x3 = k + 3 * THREADS < b ? v.tdelta[k + 3 * THREADS] : 0;
		part += x0 + x1 + x2 + x3;
	}
	if (!on)
		return;
	const int2 tp = ordered ? tp0 : make_int2(0, 0);
	const int L = tp.y + db;
	if (L > 0)
	{
		int4* c4 = reinterpret_cast<int4*>(sm.cnt);
		for (int q = tid; q < (nv + 3) >> 2; q += THREADS)
			c4[q] = make_int4(0, 0, 0, 0);
	}
	if (tid == 0)
		sm.n = 0;
	int moved;
	block_exclusive_scan(part, moved); // synchronises the block
	const int base = tp.x + moved;
	const bool fits = base >= 0 && L >= 0 && (int64_t)base + L <= v.total_cap;

	// the kept entries of the previous order, kOrderBatch per thread loaded
	// together (one list slot reservation per warp and entry), then the chains
	if (fits && L > 0)
		for (int c0 = tid - lane; c0 < tp.y; c0 += kOrderBatch * THREADS)
		{
			int2 e[kOrderBatch];
#pragma unroll
			for (int k = 0; k < kOrderBatch; k++)
			{
				const int i = c0 + k * THREADS + lane;
				e[k] = i < tp.y ? v.porder[tp.x + i] : make_int2(-1, 0);
			}
#pragma unroll
			for (int k = 0; k < kOrderBatch; k++)
			{
				const int i = c0 + k * THREADS + lane;
				const int lv = e[k].y - k0;
				bool keep = e[k].x >= 0;
				if (keep && (unsigned)lv >= (unsigned)nv)
				{
					atomicOr(v.err, ERR_LIST_CAPACITY); // a key outside the tile: the order is broken
					keep = false;
				}
				const unsigned m = __ballot_sync(0xffffffffu, keep);
				int at = 0;
				if (lane == 0 && m)
					at = atomicAdd(&sm.n, __popc(m));
				at = __shfl_sync(0xffffffffu, at, 0);
				if (keep)
					place_store(v, sm, base, at + __popc(m & ((1u << lane) - 1)), e[k].x,
								lv | (i + 1 < kPrevLimit ? (i + 1) << kVoxelBits : 0));
			}
		}
	if (tid < kChains && chain >= 0)
	{
		v.chead[(int64_t)b * kChains + tid] = -1;
		int q = chain;
		for (int hops = 0; q >= 0; hops++)
		{
			if (!fits || L <= 0 || hops >= v.total_cap || q >= v.total_cap)
			{
				atomicOr(v.err, ERR_LIST_CAPACITY); // movers into a tile that expects none, or a broken chain
				break;
			}
			const int lv = v.key[q] - k0;
			if ((unsigned)lv < (unsigned)nv)
				place_store(v, sm, base, atomicAdd(&sm.n, 1), q, lv);
			else
				atomicOr(v.err, ERR_LIST_CAPACITY);
			q = v.cnext[q];
		}
	}
	__syncthreads();
	const int n = sm.n;
	const bool ok = fits && n == L;
	if (!ok && tid == 0)
		atomicOr(v.err, ERR_LIST_CAPACITY);

	if (ok)
	{
		// per-voxel starts; an empty tile's are all its start, and a tile that
		// was and stays empty at the same start keeps them
		if (n > 0)
		{
			place_scan<THREADS>(sm, nv);
			int4* vs4 = reinterpret_cast<int4*>(v.vstart + k0); // k0 is a multiple of 64
			const int4* c4 = reinterpret_cast<const int4*>(sm.cnt);
			for (int q = tid; q < nv >> 2; q += THREADS)
			{
				int4 c = c4[q];
				c.x += base;
				c.y += base;
				c.z += base;
				c.w += base;
				vs4[q] = c;
			}
			for (int j = (nv & ~3) + tid; j < nv; j += THREADS)
				v.vstart[k0 + j] = base + sm.cnt[j];
		}
		else if (!(ordered && tp.y == 0 && base == tp.x))
		{
			int4* vs4 = reinterpret_cast<int4*>(v.vstart + k0);
			for (int q = tid; q < nv >> 2; q += THREADS)
				vs4[q] = make_int4(base, base, base, base);
			for (int j = (nv & ~3) + tid; j < nv; j += THREADS)
				v.vstart[k0 + j] = base;
		}
		if (k0 + nv == v.nvox && tid == 0)
		{
			v.vstart[v.nvox] = base + n;
			*v.cursor = base + n;
		}
		if (n > 0)
		{
			__syncthreads(); // the starts are read above before the grouping moves them
			// slots grouped by voxel; afterwards cnt[j] is the end of voxel j
			for (int i = tid; i < n; i += THREADS)
			{
				const int2 it = place_item(v, sm, base, i);
				const int p = atomicAdd(&sm.cnt[it.y & ((1 << kVoxelBits) - 1)], 1);
				if (p < kPlaceList)
					sm.group[p] = it.x;
				else
					v.tmp[base + p] = it.x;
			}
			__syncthreads();
			// the final place: descending slot inside the voxel
			for (int i = tid; i < n; i += THREADS)
			{
				const int2 it = place_item(v, sm, base, i);
				const int lv = it.y & ((1 << kVoxelBits) - 1);
				const int pidx = it.y >> kVoxelBits;
				const int lo = lv ? sm.cnt[lv - 1] : 0, hi = sm.cnt[lv];
				int rank = 0;
				for (int u = lo; u < hi; u++)
					rank += (u < kPlaceList ? sm.group[u] : v.tmp[base + u]) > it.x;
				const int t = base + lo + rank;
				v.sorted[t] = it.x;
				v.skey[t] = k0 + lv;
				v.tfresh[t] = (pidx == 0 || tp.x + pidx - 1 != t) ? 1 : 0;
			}
		}
		if (tid == 0)
			v.tprev[b] = make_int2(base, n);
	}

	// k_bin_copy writes every field where agents' fields or slots changed
	// since the last rebuild, elsewhere only the positions; the flags read
	// here are reset after the order is complete (bin_finish)
	if (b == 0 && tid == 0)
		*v.copy_full = (*v.params_changed != 0 || !ordered) ? 1 : 0;
	__syncthreads(); // shared memory is reused by the next tile of a persistent block
}

__global__ void __launch_bounds__(kPlaceThreads) k_bin_order(view v)
{
	__shared__ place_smem sm;
	grid_wait();
	bin_order_tile<kPlaceThreads>(v, blockIdx.x, sm, *v.bin_active);
}

// The key-ordered copies of the agent at position t of the new order, into
// the position buffers `spos4` and `sposf` that go with positions pos[cur].
// Where the agent is new to its position, or fields changed since the last
// rebuild (copy_full), every field is copied; elsewhere the fields other
// than the position are those the position already holds, and only the
// position is, unless the fused pass before the rebuild wrote it there
// already (`produced`).
// The counters and flags of the next rebuild, once this one's order is
// complete (nothing in the copy reads them): tile changes, the slots the
// order lists per replicate, and the flags the count and the order read.
// Thread `i` of `n` in the grid.
__device__ __forceinline__ void bin_finish(const view& v, int i, int n)
{
	const int nsup = (v.ntiles + (1 << kSuperShift) - 1) >> kSuperShift;
	for (int k = i; k < v.ntiles; k += n)
		v.tdelta[k] = 0;
	for (int k = i; k < nsup; k += n)
		v.sdelta[k] = 0;
	for (int k = i; k < v.nreps; k += n)
		v.binned[k] = v.ctr[k].count; // the slots this rebuild's order lists
	if (i == 0)
	{
		*v.params_changed = 0;
		*v.recount = 0;
		*v.order_valid = 1;
		*v.moves_pending = 0; // applied by this rebuild's count
		*v.appended = 0;	  // counted by it too
		*v.pos_changed = 0;
	}
}

// `on`: the rebuild runs (bin_active).
__device__ __forceinline__ void bin_copy_agent(const view& v, int cur, int t, int produced, double4* spos4,
											   float4* sposf, int on)
{
	if (t >= v.total_cap)
		return;
	// the loads the decision needs, issued together before any branch
	const int n = *v.cursor;
	const int full = *v.copy_full;
	const int fresh_t = v.tfresh[t];
	const int s = v.sorted[t];
	if (!on || t >= n)
		return;
	const bool fresh = full || fresh_t;
	if (!fresh && produced)
		return;
	if (fresh)
	{
		place_agent(v, cur, s, t, spos4, sposf);
		return;
	}
	if ((unsigned)s >= (unsigned)v.total_cap)
	{
		atomicOr(v.err, ERR_LIST_CAPACITY);
		return;
	}
	const double4 p = v.pos[cur][s];
	const rep_info& R = v.reps[rep_of(v, s)];
	double* q = reinterpret_cast<double*>(spos4 + t);
	q[0] = p.x;
	q[1] = p.y;
	q[2] = p.z;
	float* f = reinterpret_cast<float*>(sposf + t);
	f[0] = (float)(p.x - R.mins[0]);
	f[1] = (float)(p.y - R.mins[1]);
	f[2] = (float)(p.z - R.mins[2]);
}

// `produced`: the fused pass before this rebuild wrote the next step's
// positions into the other buffer pair (spos4_next, sposf_next); the copy
// completes that pair, which becomes the current one after it.
__global__ void __launch_bounds__(kThreads) k_bin_copy(view v, int cur, int produced)
{
	grid_wait();
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int on = *v.bin_active;
	bin_copy_agent(v, cur, t, produced, produced ? v.spos4_next : v.spos4, produced ? v.sposf_next : v.sposf, on);
	if (on)
		bin_finish(v, t, gridDim.x * blockDim.x);
}

// ---------------------------------------------------------------------------
// neighbour scan: common_solver::for_each_in_mech_neighborhood +
// update_cell_neighbors_single (reference: common_solver.h:77-105,
// position_solver.cpp:79-97). Visits voxels z, y, x from -1 to 1 and, in each,
// agents in bin order; calls f for every agent j != i with
// distance <= rmad_i r_i + rmad_j r_j.
// ---------------------------------------------------------------------------

// run-time options of the fused passes: basement-membrane walls, springs,
// a velocity to start the sums from
enum : int
{
	FUSED_WALLS = 1,
	FUSED_SPRINGS = 2,
	FUSED_VEL = 4,
	FUSED_PRODUCE = 8 // the pass does the rebuild count's work for its agents (shapes -3 and -4)
};

// the voxel coordinate of axis_coord without its error reports: the keys the
// fused pass computes for the rebuild are recomputed (with the reports) by
// the count whenever the compaction removes agents, and an agent outside the
// box or with a non-finite position is always removed or reported
__device__ __forceinline__ int axis_coord_quiet(double x, const rep_info& R, int d)
{
	const double q = (x - R.mins[d]) / R.shape[d];
	const int g = R.grid[d];
	if (!(q > 0.0))
		return 0;
	if (q >= (double)g)
		return g - 1;
	return (int)q;
}

// The rebuild count's work for the agent at key-ordered position t (slot s,
// key okey in the current order) that the fused pass moved to p: its new
// key, and either its kept entry of the order or a push onto its new tile's
// mover chain with the tiles' changes. Valid while no agent is removed
// before the rebuild; the compaction plan discards it otherwise.
__device__ __forceinline__ void produce_entry(const view& v, const rep_info& R, int t, int s, int32_t okey,
											  const double4& p, double pw)
{
	const int c0 = axis_coord_quiet(p.x, R, 0);
	const int c1 = v.dims >= 2 ? axis_coord_quiet(p.y, R, 1) : 0;
	const int c2 = v.dims >= 3 ? axis_coord_quiet(p.z, R, 2) : 0;
	const int32_t key = (int32_t)(R.vox_base + c0 + (int64_t)R.grid[0] * (c1 + (int64_t)R.grid[1] * c2));
	v.key[s] = key;
	// the agent's key-ordered position for the next step, at its place in
	// the current order: the rebuild's copy keeps it wherever the agent keeps
	// its place (the fused pass reads the other buffer)
	v.spos4_next[t] = make_double4(p.x, p.y, p.z, pw);
	v.sposf_next[t] = make_float4((float)(p.x - R.mins[0]), (float)(p.y - R.mins[1]), (float)(p.z - R.mins[2]),
								  (float)pw);
	const int sh = v.tshift;
	if ((key >> sh) == (okey >> sh))
		v.porder[t] = make_int2(s, key);
	else
	{
		v.porder[t] = make_int2(-1, -1);
		chain_push(v, s, key);
		atomicAdd(v.tdelta + (okey >> sh), -1);
		atomicAdd(v.sdelta + ((okey >> sh) >> kSuperShift), -1);
		atomicAdd(v.tdelta + (key >> sh), 1);
		atomicAdd(v.sdelta + ((key >> sh) >> kSuperShift), 1);
	}
}

constexpr int kList = 8; // neighbours recorded per thread before the pair pass runs
constexpr int kFusedThreads = 128; // block size limit of the fused pass (five blocks per SM resident)

// Visits, in the reference's order, the neighbours of the agent at position t
// of the key-ordered array: stencil rows z outer then y; in each row the
// voxels x-1..x+1, which are consecutive keys and so one contiguous range
// [vstart[k-1], vstart[k+2]) of the array; inside a voxel descending slot.
// Works in two phases: a candidate scan records the array positions of
// neighbours (distance <= rmad_i r_i + rmad_j r_j) in `list` (kList per
// thread, strided by the block size), then f(u) runs for each recorded
// position. The scan loop stays short, so a warp runs the costly pair code
// max-over-lanes(neighbour count) times rather than once per candidate
// iteration in which any lane found a neighbour.
template <int DIMS, typename F>
__device__ __forceinline__ void for_each_neighbor(const view& v, const rep_info& R, int t, int32_t key,
												  const double4& pi, int32_t* list, F&& f)
{
	const int32_t lk = (int32_t)(key - R.vox_base);
	const int g0 = R.grid[0], g1 = R.grid[1], g2 = R.grid[2];
	int cx, cy, cz;
	voxel_coords(R, lk, cx, cy, cz);
	const int xlo = cx > 0 ? cx - 1 : 0;
	const int xhi = cx + 1 < g0 ? cx + 1 : g0 - 1;
	constexpr int NR = DIMS == 3 ? 9 : (DIMS == 2 ? 3 : 1);
	int lo[NR], hi[NR];
	const int32_t vb = (int32_t)R.vox_base; // voxel keys fit 31 bits (checked at creation)
#pragma unroll
	for (int k = 0; k < NR; k++)
	{
		const int dz = DIMS == 3 ? k / 3 - 1 : 0;
		const int dy = DIMS >= 2 ? k % 3 - 1 : 0;
		const int z = cz + dz, y = cy + dy;
		const bool ok = z >= 0 && z < g2 && y >= 0 && y < g1;
		const int32_t row = ok ? vb + g0 * (y + g1 * z) : 0;
		lo[k] = ok ? v.vstart[row + xlo] : 0;
		hi[k] = ok ? v.vstart[row + xhi + 1] : 0;
	}
	const int stride = blockDim.x;
	int n = 0;
#pragma unroll
	for (int k = 0; k < NR; k++)
	{
		for (int u = lo[k]; u < hi[k]; u++)
		{
			if (u == t)
				continue;
			const double4 q = v.spos4[u];
			const double ddx = pi.x - q.x;
			const double ddy = DIMS >= 2 ? pi.y - q.y : 0.0;
			const double ddz = DIMS >= 3 ? pi.z - q.z : 0.0;
			double d2 = ddx * ddx;
			if (DIMS >= 2)
				d2 = d2 + ddy * ddy;
			if (DIMS >= 3)
				d2 = d2 + ddz * ddz;
			const double ad = pi.w + q.w;
			// exact early reject: d2 > ad^2 (1 + 1e-12) implies sqrt(d2) > ad
			if (d2 > ad * ad * (1.0 + 1e-12))
				continue;
			const double dist = DIMS == 1 ? fabs(ddx) : sqrt(d2);
			if (!(dist <= ad))
				continue;
			list[n * stride] = u;
			if (++n == kList)
			{
				for (int m = 0; m < n; m++)
					f(list[m * stride]);
				n = 0;
			}
		}
	}
	for (int m = 0; m < n; m++)
		f(list[m * stride]);
}

// geometry of the pair (i at pi, neighbour at array position u), recomputed
// with the same operations as the scan
template <int DIMS>
struct pair_geometry
{
	double ddx, ddy, ddz, dist, ad;

	__device__ __forceinline__ pair_geometry(const view& v, const double4& pi, int u)
	{
		const double4 q = v.spos4[u];
		ddx = pi.x - q.x;
		ddy = DIMS >= 2 ? pi.y - q.y : 0.0;
		ddz = DIMS >= 3 ? pi.z - q.z : 0.0;
		double d2 = ddx * ddx;
		if (DIMS >= 2)
			d2 = d2 + ddy * ddy;
		if (DIMS >= 3)
			d2 = d2 + ddz * ddz;
		ad = pi.w + q.w;
		dist = DIMS == 1 ? fabs(ddx) : sqrt(d2);
	}
};

// solve_pair for the lhs side (reference: position_solver.cpp:24-77) with the
// pressure contributions of the pair to lhs. Adds (repulsion - adhesion) /
// distance * difference to v when lhs is movable. `add_pair` takes the
// neighbour's data as values so callers can read it from global or shared
// memory; the operations and their order are the reference's.
struct pair_fp64
{
	double4 prm_i;
	const double* aff_i;
	int def_i;
	bool mov_i;
	double vx = 0, vy = 0, vz = 0, p = 0;
	double last_term = 0; // pressure contribution of the last pair

	__device__ __forceinline__ void add_pair(double r_j, double rep_j, double adh_j, int def_j, bool mov_j,
											 double aff_ji, double ddx, double ddy, double ddz, double dist,
											 double adhesion_distance)
	{
		const double d = dist < 0.00001 ? 0.00001 : dist; // std::max(distance, 0.00001)
		double rep = 1.0 - d / (prm_i.x + r_j);
		rep = rep < 0 ? 0 : rep;
		rep = rep * rep;
		const double term = rep * simple_pressure_coefficient;
		last_term = term;
		if (mov_i)
			p = p + term;
		if (mov_j)
			p = p + term;
		if (!mov_i)
			return;
		rep = rep * sqrt(prm_i.y * rep_j);
		double adh = 1.0 - d / adhesion_distance;
		adh = adh * adh;
		adh = adh * sqrt(prm_i.z * adh_j * aff_i[def_j] * aff_ji);
		const double force = (rep - adh) / d;
		vx = vx + force * ddx;
		vy = vy + force * ddy;
		vz = vz + force * ddz;
	}

	__device__ __forceinline__ void add(const view& v, int j, double ddx, double ddy, double ddz, double dist,
										double adhesion_distance)
	{
		const double4 prm_j = v.prm[j];
		add_pair(prm_j.x, prm_j.y, prm_j.z, v.def[j], v.movable[j] != 0, v.aff[(int64_t)j * v.ndefs + def_i], ddx,
				 ddy, ddz, dist, adhesion_distance);
	}
};

// bits of sprm4.w: definition index (0..31), movable (32), spring count (40..47),
// replicate (48..63, its low 16 bits)
__device__ __forceinline__ void unpack_bits(double w, int& def, bool& mov)
{
	const long long b = __double_as_longlong(w);
	def = (int)(uint32_t)(b & 0xffffffffll);
	mov = ((b >> 32) & 1) != 0;
}

__device__ __forceinline__ int unpack_springs(double w) { return (int)((__double_as_longlong(w) >> 40) & 0xff); }

// bits of sprmf.w: definition index (0..15), movable (16), spring count (24..31)
__device__ __forceinline__ void unpack_fbits(float w, int& def, bool& mov, int& springs)
{
	const uint32_t b = (uint32_t)__float_as_int(w);
	def = (int)(b & 0xffffu);
	mov = ((b >> 16) & 1u) != 0;
	springs = (int)(b >> 24);
}

// update_membrane_velocity (reference: solver_helper.h:14-28)
__device__ __forceinline__ double membrane(double x, double bb, double sign, double radius, double strength, double vel)
{
	double dist = fabs(bb - x);
	dist = dist < 0.00001 ? 0.00001 : dist;
	double rep = 1.0 - dist / radius;
	rep = rep < 0 ? 0 : rep;
	rep = rep * (rep * strength * sign);
	return vel + rep * dist;
}

template <int DIMS>
__device__ __forceinline__ void walls(const view& v, const rep_info& R, const double4& p, double radius,
									  double strength, double4& vel)
{
	// update_membrane_velocities (reference: solver_helper.h:103-110,184-193,288-299);
	// the 1-D version uses the y maximum for the upper wall, kept as in the reference
	for (int d = 0; d < DIMS; d++)
	{
		double x = comp(p, d), u = comp(vel, d);
		u = membrane(x, R.mins[d], 1.0, radius, strength, u);
		u = membrane(x, DIMS == 1 ? R.maxs[1] : R.maxs[d], -1.0, radius, strength, u);
		set_comp(vel, d, u);
	}
}

// spring_contract_function for one agent (reference: position_solver.cpp:337-370).
// Springs are taken two at a time, the loads of both issued before the
// arithmetic; the terms are added in attachment order.
template <int DIMS>
__device__ __forceinline__ void spring_contract(const view& v, int cur, int s, int n, const double4& pi, int def_i,
												double4& vel)
{
	const double ec_i = v.ec[s];
	const double* aff_i = v.aff + (int64_t)s * v.ndefs;
	for (int k0 = 0; k0 < n; k0 += 2)
	{
		const bool two = k0 + 1 < n;
		const int j0 = v.springs[(int64_t)s * v.scap + k0];
		const int j1 = two ? v.springs[(int64_t)s * v.scap + k0 + 1] : j0;
		const int d0 = v.def[j0], d1 = v.def[j1];
		const double e0 = v.ec[j0], e1 = v.ec[j1];
		const double f0 = v.aff[(int64_t)j0 * v.ndefs + def_i], f1 = v.aff[(int64_t)j1 * v.ndefs + def_i];
		const double4 p0 = v.pos[cur][j0], p1 = v.pos[cur][j1];
		const double g0 = aff_i[d0], g1 = aff_i[d1];
		const double a0 = sqrt(ec_i * e0 * g0 * f0);
		for (int d = 0; d < DIMS; d++)
			set_comp(vel, d, comp(vel, d) + a0 * (comp(p0, d) - comp(pi, d)));
		if (two)
		{
			const double a1 = sqrt(ec_i * e1 * g1 * f1);
			for (int d = 0; d < DIMS; d++)
				set_comp(vel, d, comp(vel, d) + a1 * (comp(p1, d) - comp(pi, d)));
		}
	}
}

// Adams-Bashforth update (reference: position_solver.cpp:481-504)
template <int DIMS>
__device__ __forceinline__ void ab2(double dt, double4& p, const double4& vel, double4& vprev)
{
	const double factor = dt * 1.5;
	const double previous_factor = dt * -0.5;
	for (int d = 0; d < DIMS; d++)
	{
		set_comp(p, d, comp(p, d) + (comp(vel, d) * factor + comp(vprev, d) * previous_factor));
		set_comp(vprev, d, comp(vel, d));
	}
}

// removal test of remove_single (reference: containers_solver.cpp:85-98)
template <int DIMS>
__device__ __forceinline__ bool to_remove(const rep_info& R, const double4& p, uint8_t flag)
{
	bool out = false;
	for (int d = 0; d < DIMS; d++)
	{
		double x = comp(p, d);
		if (x < R.mins[d] || x > R.maxs[d])
			out = true;
	}
	return out || flag == PPC_FLAG_TO_REMOVE;
}

__device__ __forceinline__ void append_bad(const view& v, int r, int local)
{
	int k = atomicAdd(&v.ctr[r].nbad, 1);
	if (k < v.reps[r].cap)
		v.bad[v.reps[r].base + k] = local;
	else
		atomicOr(v.err, ERR_LIST_CAPACITY);
}

// Per-agent data the epilogue needs, gathered before the agent's first
// global store: on this GPU a gather that follows scattered stores of the
// same thread stalls far longer than the same gather issued first.
struct agent_tail
{
	double4 vprev;
	double4 vel0;
	double bm;
	uint8_t flag;
};

template <bool WALLS, bool VEL>
__device__ __forceinline__ agent_tail load_tail(const view& v, int s, bool mov)
{
	agent_tail a;
	a.vprev = mov ? v.vprev[s] : make_double4(0, 0, 0, 0);
	a.vel0 = (VEL && mov) ? v.vel[s] : make_double4(0, 0, 0, 0);
	a.bm = (WALLS && mov) ? v.prm[s].w : 0.0;
	a.flag = v.flags[s];
	return a;
}

// membrane + springs + Adams-Bashforth for one agent, then every store of the
// fused pass for it (pressure, previous velocity, velocity, new position) and
// the container-update marking
template <int DIMS, bool WALLS, bool SPRINGS, bool VEL>
__device__ __forceinline__ void finish_agent(const view& v, const rep_info& R, int r, int cur, int s, const double4& pi,
											 double radius, int def_i, bool mov_i, int nspr, const agent_tail& tail,
											 double vx, double vy, double vz, double pressure)
{
	double4 p = make_double4(pi.x, pi.y, pi.z, 0.0);
	double4 vp = tail.vprev;
	if (mov_i)
	{
		double4 vel = make_double4(vx, vy, vz, 0.0);
		if (WALLS)
			walls<DIMS>(v, R, p, radius, tail.bm, vel);
		if (SPRINGS && nspr > 0)
			spring_contract<DIMS>(v, cur, s, nspr, p, def_i, vel);
		ab2<DIMS>(v.dt, p, vel, vp);
	}
	v.pressure[s] = pressure;
	if (mov_i)
	{
		v.vprev[s] = vp;
		if (VEL)
			v.vel[s] = make_double4(0, 0, 0, 0);
	}
	v.pos[cur ^ 1][s] = p;
	if (!(p.x == p.x && p.y == p.y && p.z == p.z))
		atomicOr(v.err, ERR_NONFINITE);
	if (to_remove<DIMS>(R, p, tail.flag))
		append_bad(v, r, s - R.base);
}

// ---------------------------------------------------------------------------
// fused step: neighbour search + forces + membrane + springs + AB2, one
// thread per binned agent, reading positions from pos[cur] and writing the
// new positions to pos[nxt] (the reference finishes all force passes before
// the position update, so every read must see the old positions). Also marks
// agents for the container update that follows.
// ---------------------------------------------------------------------------
template <int DIMS, bool WALLS, bool SPRINGS, bool VEL>
__global__ void __launch_bounds__(kFusedThreads, 5) k_fused(view v, int cur)
{
	grid_wait();
	bump_spring_epochs(v);
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= *v.cursor)
		return;
	const int s = v.sorted[t];
	const int r = rep_of(v, s);
	const rep_info& R = v.reps[r];
	const double4 pi = v.spos4[t];

	pair_fp64 acc;
	acc.prm_i = v.sprm4[t];
	unpack_bits(acc.prm_i.w, acc.def_i, acc.mov_i);
	acc.aff_i = v.saff + (int64_t)t * v.ndefs;
	const agent_tail tail = load_tail<WALLS, VEL>(v, s, acc.mov_i);
	acc.vx = tail.vel0.x;
	acc.vy = tail.vel0.y;
	acc.vz = tail.vel0.z;
	__shared__ int32_t list[kList * kFusedThreads];
	const int D = v.ndefs;
	for_each_neighbor<DIMS>(v, R, t, v.skey[t], pi, list + threadIdx.x, [&](int u) {
		// neighbour data from the key-ordered copies (index u, no indirection)
		const pair_geometry<DIMS> g(v, pi, u);
		const double4 qj = v.sprm4[u];
		int def_j;
		bool mov_j;
		unpack_bits(qj.w, def_j, mov_j);
		acc.add_pair(qj.x, qj.y, qj.z, def_j, mov_j, v.saff[(int64_t)u * D + acc.def_i], g.ddx, g.ddy, g.ddz, g.dist,
					 g.ad);
	});
	finish_agent<DIMS, WALLS, SPRINGS, VEL>(v, R, r, cur, s, pi, acc.prm_i.x, acc.def_i, acc.mov_i,
											unpack_springs(acc.prm_i.w), tail, acc.vx, acc.vy, acc.vz, acc.p);
}

// ---------------------------------------------------------------------------
// FP32-force form of the fused pass. Neighbour sets stay exact: a single
// precision filter on positions relative to the box minimum rejects far
// candidates with a margin of 16 float ulps of the domain extent, and the
// candidates it keeps go through the FP64 predicate. The pair arithmetic
// (distance, sqrt, potentials, force) runs in FP32 on the FP64 difference
// rounded to FP32, and the per-agent sums of velocity and pressure are
// Neumaier-compensated (A. Neumaier, ZAMM 54, 1974). Membrane, springs and
// the Adams-Bashforth update stay FP64.
// ---------------------------------------------------------------------------

struct nsum
{
	float s = 0.f, c = 0.f;
	__device__ __forceinline__ void add(float x)
	{
		const float t = s + x;
		if (fabsf(s) >= fabsf(x))
			c += (s - t) + x;
		else
			c += (x - t) + s;
		s = t;
	}
	__device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

struct pair_fp32
{
	float r_i, rep_i, adh_i;
	const float* aff_i;
	int def_i;
	bool mov_i;
	nsum vx, vy, vz, p;

	__device__ __forceinline__ void add(float r_j, float rep_j, float adh_j, int def_j, bool mov_j, float aff_ji,
										float dx, float dy, float dz, float dist, float ad)
	{
		const float d = dist < 0.00001f ? 0.00001f : dist;
		float rep = 1.f - d / (r_i + r_j);
		rep = rep < 0.f ? 0.f : rep;
		rep = rep * rep;
		const float term = rep * 36.64504274775163f;
		if (mov_i)
			p.add(term);
		if (mov_j)
			p.add(term);
		if (!mov_i)
			return;
		rep = rep * sqrtf(rep_i * rep_j);
		float adh = 1.f - d / ad;
		adh = adh * adh;
		adh = adh * sqrtf(adh_i * adh_j * aff_i[def_j] * aff_ji);
		const float force = (rep - adh) / d;
		vx.add(force * dx);
		vy.add(force * dy);
		vz.add(force * dz);
	}
};

template <int DIMS, bool WALLS, bool SPRINGS, bool VEL>
__global__ void __launch_bounds__(kFusedThreads, 5) k_fused_f32(view v, int cur)
{
	grid_wait();
	bump_spring_epochs(v);
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= *v.cursor)
		return;
	const int s = v.sorted[t];
	const int r = rep_of(v, s);
	const rep_info& R = v.reps[r];
	const double4 pi = v.spos4[t];
	const float4 pf = v.sposf[t];
	const float4 qf = v.sprmf[t];
	const int D = v.ndefs;
	pair_fp32 acc;
	int nspr;
	unpack_fbits(qf.w, acc.def_i, acc.mov_i, nspr);
	acc.r_i = qf.x;
	acc.rep_i = qf.y;
	acc.adh_i = qf.z;
	acc.aff_i = v.safff + (int64_t)t * D;
	const agent_tail tail = load_tail<WALLS, VEL>(v, s, acc.mov_i);
	const float m = R.fmargin;

	const int32_t lk = v.skey[t] - (int32_t)R.vox_base;
	const int g0 = R.grid[0], g1 = R.grid[1], g2 = R.grid[2];
	int cx, cy, cz;
	voxel_coords(R, lk, cx, cy, cz);
	const int xlo = cx > 0 ? cx - 1 : 0;
	const int xhi = cx + 1 < g0 ? cx + 1 : g0 - 1;
	constexpr int NR = DIMS == 3 ? 9 : (DIMS == 2 ? 3 : 1);
	int lo[NR], hi[NR];
#pragma unroll
	for (int k = 0; k < NR; k++)
	{
		const int dz = DIMS == 3 ? k / 3 - 1 : 0;
		const int dy = DIMS >= 2 ? k % 3 - 1 : 0;
		const int z = cz + dz, y = cy + dy;
		const bool ok = z >= 0 && z < g2 && y >= 0 && y < g1;
		const int32_t row = ok ? (int32_t)R.vox_base + g0 * (y + g1 * z) : 0;
		lo[k] = ok ? v.vstart[row + xlo] : 0;
		hi[k] = ok ? v.vstart[row + xhi + 1] : 0;
	}
	__shared__ int32_t list[kList * kFusedThreads];
	int32_t* lst = list + threadIdx.x;
	const int stride = blockDim.x;
	int n = 0;
	auto flush = [&]() {
		for (int q = 0; q < n; q++)
		{
			const int u = lst[q * stride];
			const pair_geometry<DIMS> g(v, pi, u);
			const float dx = (float)g.ddx, dy = (float)g.ddy, dz = (float)g.ddz;
			float d2 = dx * dx;
			if (DIMS >= 2)
				d2 = d2 + dy * dy;
			if (DIMS >= 3)
				d2 = d2 + dz * dz;
			const float dist = DIMS == 1 ? fabsf(dx) : sqrtf(d2);
			const float4 qj = v.sprmf[u];
			const float4 pj = v.sposf[u];
			int def_j, spr_j;
			bool mov_j;
			unpack_fbits(qj.w, def_j, mov_j, spr_j);
			acc.add(qj.x, qj.y, qj.z, def_j, mov_j, v.safff[(int64_t)u * D + acc.def_i], dx, dy, dz, dist, pf.w + pj.w);
		}
		n = 0;
	};
#pragma unroll
	for (int k = 0; k < NR; k++)
	{
		for (int u = lo[k]; u < hi[k]; u++)
		{
			if (u == t)
				continue;
			const float4 c = v.sposf[u];
			const float dxf = pf.x - c.x;
			const float dyf = DIMS >= 2 ? pf.y - c.y : 0.f;
			const float dzf = DIMS >= 3 ? pf.z - c.z : 0.f;
			float d2f = dxf * dxf;
			if (DIMS >= 2)
				d2f = d2f + dyf * dyf;
			if (DIMS >= 3)
				d2f = d2f + dzf * dzf;
			const float adf = pf.w + c.w + m;
			if (d2f > adf * adf * 1.00001f)
				continue;
			// exact FP64 predicate for the candidates the filter keeps
			const double4 q = v.spos4[u];
			const double ddx = pi.x - q.x;
			const double ddy = DIMS >= 2 ? pi.y - q.y : 0.0;
			const double ddz = DIMS >= 3 ? pi.z - q.z : 0.0;
			double d2 = ddx * ddx;
			if (DIMS >= 2)
				d2 = d2 + ddy * ddy;
			if (DIMS >= 3)
				d2 = d2 + ddz * ddz;
			const double ad = pi.w + q.w;
			const double dist = DIMS == 1 ? fabs(ddx) : sqrt(d2);
			if (!(dist <= ad))
				continue;
			lst[n * stride] = u;
			if (++n == kList)
				flush();
		}
	}
	flush();
	finish_agent<DIMS, WALLS, SPRINGS, VEL>(v, R, r, cur, s, pi, (double)acc.r_i, acc.def_i, acc.mov_i, nspr, tail,
											tail.vel0.x + acc.vx.value(), tail.vel0.y + acc.vy.value(),
											tail.vel0.z + acc.vz.value(), acc.p.value());
}

// ---------------------------------------------------------------------------
// fused step with the block's candidates staged in shared memory.
//
// A block takes blockDim consecutive agents of the key-ordered array, keys
// kf..kl. Every candidate of every one of them for stencil row (dy, dz) has a
// key in [kf + off - 1, kl + off + 1], off = dy g0 + dz g0 g1, so it lies in
// one contiguous range of the key-ordered array; the block copies the nine
// ranges (three in 2-D, one in 1-D) of the single-precision positions
// (sposf) into shared memory with all its threads, one memory round trip, and
// each thread then scans its stencil out of shared memory. A block whose
// ranges exceed the budget, or that spans two replicates, reads the same
// arrays from global memory instead.
//
// The scan tests candidates in single precision with the margin of the FP32
// form (16 float ulps of the domain extent, and a relative 1e-5 on the
// squared distance that covers the rounding of the radii and of the float
// arithmetic), which never rejects a pair the FP64 test accepts; each kept
// candidate then goes through the FP64 test (distance <= rmad_i r_i +
// rmad_j r_j) before its pair code runs, so the neighbour sets and their
// order are the reference's. With F32 false the pair arithmetic is the FP64
// drop-in (bit-identical to the reference); with F32 true it is the
// FP32-force form.
// ---------------------------------------------------------------------------

constexpr int kStageThreads = 128;
constexpr int kStageScan = 4; // candidates a lane tests per scan iteration, loads issued together
static_assert(kStageScan >= 1 && kStageScan <= kList, "a scan iteration must fit in the neighbour list");
constexpr size_t kStageStatic = 16 * 1024; // bound on the staged kernel's static shared memory

// array bounds [lo[k], hi[k]) of the stencil rows of the agent in voxel
// `key`: rows z outer then y, each the voxels x-1..x+1, which are consecutive
// keys and so one contiguous range [vstart[k-1], vstart[k+2]) of the
// key-ordered array; rows outside the grid are empty
template <int DIMS>
__device__ __forceinline__ void stencil_bounds(const view& v, const rep_info& R, int32_t key, int* lo, int* hi)
{
	const int32_t lk = (int32_t)(key - R.vox_base);
	const int g0 = R.grid[0], g1 = R.grid[1], g2 = R.grid[2];
	int cx, cy, cz;
	voxel_coords(R, lk, cx, cy, cz);
	const int xlo = cx > 0 ? cx - 1 : 0;
	const int xhi = cx + 1 < g0 ? cx + 1 : g0 - 1;
	constexpr int NR = DIMS == 3 ? 9 : (DIMS == 2 ? 3 : 1);
	const int32_t vb = (int32_t)R.vox_base;
#pragma unroll
	for (int k = 0; k < NR; k++)
	{
		const int dz = DIMS == 3 ? k / 3 - 1 : 0;
		const int dy = DIMS >= 2 ? k % 3 - 1 : 0;
		const int z = cz + dz, y = cy + dy;
		const bool ok = z >= 0 && z < g2 && y >= 0 && y < g1;
		const int32_t row = ok ? vb + g0 * (y + g1 * z) : 0;
		lo[k] = ok ? v.vstart[row + xlo] : 0;
		hi[k] = ok ? v.vstart[row + xhi + 1] : 0;
	}
}

// true when the single-precision filter keeps candidate c for the agent at pf
template <int DIMS>
__device__ __forceinline__ bool filter_keep(const float4& pf, const float4& c, float margin)
{
	const float dxf = pf.x - c.x;
	const float dyf = DIMS >= 2 ? pf.y - c.y : 0.f;
	const float dzf = DIMS >= 3 ? pf.z - c.z : 0.f;
	float d2f = dxf * dxf;
	if (DIMS >= 2)
		d2f = d2f + dyf * dyf;
	if (DIMS >= 3)
		d2f = d2f + dzf * dzf;
	const float adf = pf.w + c.w + margin;
	return !(d2f > adf * adf * 1.00001f);
}

// the block of agents at key-ordered positions [vb * blockDim, (vb + 1) *
// blockDim); `stage` holds `cap` staged positions, then the neighbour lists;
// opts: FUSED_WALLS | FUSED_SPRINGS | FUSED_VEL
template <int DIMS, bool F32>
__device__ void fused_staged_block(const view& v, int cur, int cap, int opts, int vb, float4* stage)
{
	const bool WALLS = (opts & FUSED_WALLS) != 0, SPRINGS = (opts & FUSED_SPRINGS) != 0, VEL = (opts & FUSED_VEL) != 0;
	constexpr int NR = DIMS == 3 ? 9 : (DIMS == 2 ? 3 : 1);
	__shared__ int s_a[NR], s_o[NR + 1];
	__shared__ int2 s_rows[NR][kStageThreads]; // each thread's stencil-row bounds
	int32_t* list = reinterpret_cast<int32_t*>(stage + cap) + threadIdx.x;
	const int stride = blockDim.x;
	const int nsorted = *v.cursor;
	const int t0 = vb * blockDim.x;
	if (t0 >= nsorted)
		return;
	const int tl = min(t0 + (int)blockDim.x, nsorted) - 1;
	const int t = t0 + threadIdx.x;
	const bool act = t <= tl;

	// block set-up (warp 0): the row ranges and their offsets in shared memory
	if (cap == 0)
	{
		if (threadIdx.x == 0)
			s_o[NR] = -1; // no staging: every candidate is read from global memory
	}
	else if (threadIdx.x < 32)
	{
		// the whole of warp 0 takes this branch (cap is uniform)
		const int lane = threadIdx.x;
		const int r0 = rep_of(v, v.sorted[t0]), r1 = rep_of(v, v.sorted[tl]);
		const int64_t kf = v.skey[t0], kl = v.skey[tl];
		int a = 0, n = 0;
		if (lane < NR && r0 == r1)
		{
			const rep_info& R = v.reps[r0];
			const int dz = DIMS == 3 ? lane / 3 - 1 : 0;
			const int dy = DIMS >= 2 ? lane % 3 - 1 : 0;
			const int64_t off = (int64_t)dy * R.grid[0] + (int64_t)dz * R.grid[0] * R.grid[1];
			const int64_t lo = max(R.vox_base, kf + off - 1);
			const int64_t hi = min(R.vox_base + R.voxels, kl + off + 2);
			if (lo < hi)
			{
				a = v.vstart[lo];
				n = v.vstart[hi] - a;
			}
		}
		int incl = n;
		for (int o = 1; o < 32; o <<= 1)
		{
			const int y = __shfl_up_sync(0xffffffffu, incl, o);
			if (lane >= o)
				incl += y;
		}
		const int total = __shfl_sync(0xffffffffu, incl, NR - 1);
		if (lane < NR)
		{
			s_a[lane] = a;
			s_o[lane] = incl - n;
		}
		if (lane == 0)
			s_o[NR] = (r0 == r1 && total <= cap) ? total : -1;
	}

	// per-agent loads, issued before the block waits for its ranges
	const int tt = act ? t : tl;
	const int s = v.sorted[tt];
	const int r = rep_of(v, s);
	const rep_info& R = v.reps[r];
	const double4 pi = v.spos4[tt];
	const float4 pf = v.sposf[tt];
	const double4 qi = v.sprm4[tt];
	int def_i;
	bool mov_i;
	unpack_bits(qi.w, def_i, mov_i);
	const int nspr = unpack_springs(qi.w);
	// the previous velocity is read after the scan; ask L2 for it now
	if (mov_i)
		asm volatile("prefetch.global.L2 [%0];" ::"l"(v.vprev + s));
	const uint8_t flag = v.flags[s];
	const double bm = (WALLS && mov_i) ? v.prm[s].w : 0.0;
	{
		int lo[NR], hi[NR];
		stencil_bounds<DIMS>(v, R, v.skey[tt], lo, hi);
#pragma unroll
		for (int k = 0; k < NR; k++)
			s_rows[k][threadIdx.x] = act ? make_int2(lo[k], hi[k]) : make_int2(0, 0);
	}

	__syncthreads();
	const int S = s_o[NR];
	for (int i = threadIdx.x; i < S; i += blockDim.x)
	{
		int k = 0;
#pragma unroll
		for (int kk = 1; kk < NR; kk++)
			k = i >= s_o[kk] ? kk : k;
		stage[i] = v.sposf[s_a[k] + (i - s_o[k])];
	}
	__syncthreads();

	// candidates at array positions u of row k are read at P[u + soff(k)]:
	// shared memory when staged, else the global sposf
	const bool staged = S >= 0;
	const float4* P = staged ? stage : v.sposf;
	const int D = v.ndefs;
	const float margin = R.fmargin;
	const double4 vel0 = (VEL && mov_i) ? v.vel[s] : make_double4(0, 0, 0, 0);
	// FP64 sums (drop-in) or Neumaier-compensated FP32 sums (FP32-force form)
	double vx = vel0.x, vy = vel0.y, vz = vel0.z, pressure = 0.0;
	nsum fx, fy, fz, fp;

	// Warp-cooperative pair phase. Each lane collects its kept candidates
	// in `list`; when a lane's list is full, or the scan ends, the warp
	// spreads all lanes' entries over its 32 lanes (lane q of a round takes
	// the q-th entry in lane order), each lane runs the exact predicate and
	// the pair arithmetic for its entry and leaves the terms in shared memory,
	// and every owner then adds its own terms in list order, which is the
	// reference's neighbour order. The additions, their operands and their
	// order are those of the sequential pair code.
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	__shared__ uint8_t s_owner[kStageThreads / 32][32 * kList];
	__shared__ double4 s_term[kStageThreads / 32][32]; // {v_x, v_y, v_z, pressure} terms of one pair
	__shared__ int s_flag[kStageThreads / 32][32];	   // 1 accepted, 2 neighbour movable
	const int32_t* lists = reinterpret_cast<const int32_t*>(stage + cap) + warp * 32;
	int n = 0;
	auto flush = [&]() {
		int off = n;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1)
		{
			const int y = __shfl_up_sync(0xffffffffu, off, o);
			if (lane >= o)
				off += y;
		}
		const int total = __shfl_sync(0xffffffffu, off, 31);
		off -= n;
		for (int m = 0; m < n; m++)
			s_owner[warp][off + m] = (uint8_t)lane;
		__syncwarp();
		for (int base = 0; base < total; base += 32)
		{
			const int q = base + lane;
			const int o = q < total ? s_owner[warp][q] : lane;
			const int off_o = __shfl_sync(0xffffffffu, off, o);
			const int t_o = __shfl_sync(0xffffffffu, t, o);
			const int def_o = __shfl_sync(0xffffffffu, def_i, o);
			const bool mov_o = __shfl_sync(0xffffffffu, (int)mov_i, o) != 0;
			const double px = __shfl_sync(0xffffffffu, pi.x, o);
			const double py = __shfl_sync(0xffffffffu, pi.y, o);
			const double pz = __shfl_sync(0xffffffffu, pi.z, o);
			const double pw = __shfl_sync(0xffffffffu, pi.w, o);
			const double ri = __shfl_sync(0xffffffffu, qi.x, o);
			const double repi = __shfl_sync(0xffffffffu, qi.y, o);
			const double adhi = __shfl_sync(0xffffffffu, qi.z, o);
			const float pfw = __shfl_sync(0xffffffffu, pf.w, o);
			if (q < total)
			{
				const int u = lists[(q - off_o) * stride + o];
				const double4 qp = v.spos4[u];
				const double ddx = px - qp.x;
				const double ddy = DIMS >= 2 ? py - qp.y : 0.0;
				const double ddz = DIMS >= 3 ? pz - qp.z : 0.0;
				double d2 = ddx * ddx;
				if (DIMS >= 2)
					d2 = d2 + ddy * ddy;
				if (DIMS >= 3)
					d2 = d2 + ddz * ddz;
				const double ad = pw + qp.w;
				const double dist = DIMS == 1 ? fabs(ddx) : sqrt(d2);
				int fl = 0;
				double4 tm = make_double4(0, 0, 0, 0);
				if (dist <= ad)
				{
					fl = 1;
					if (F32)
					{
						// pair_fp32::add with the owner's values
						const float dx = (float)ddx, dy = (float)ddy, dz = (float)ddz;
						float d2f = dx * dx;
						if (DIMS >= 2)
							d2f = d2f + dy * dy;
						if (DIMS >= 3)
							d2f = d2f + dz * dz;
						const float distf = DIMS == 1 ? fabsf(dx) : sqrtf(d2f);
						const float4 qj = v.sprmf[u];
						const float4 pj = v.sposf[u];
						int def_j, spr_j;
						bool mov_j;
						unpack_fbits(qj.w, def_j, mov_j, spr_j);
						fl |= mov_j ? 2 : 0;
						const float d = distf < 0.00001f ? 0.00001f : distf;
						float rep = 1.f - d / ((float)ri + qj.x);
						rep = rep < 0.f ? 0.f : rep;
						rep = rep * rep;
						const float term = rep * 36.64504274775163f;
						tm.w = (double)term;
						if (mov_o)
						{
							rep = rep * sqrtf((float)repi * qj.y);
							float adh = 1.f - d / (pfw + pj.w);
							adh = adh * adh;
							adh = adh * sqrtf((float)adhi * qj.z * v.safff[(int64_t)t_o * D + def_j]
											  * v.safff[(int64_t)u * D + def_o]);
							const float force = (rep - adh) / d;
							tm.x = (double)(force * dx);
							tm.y = (double)(force * dy);
							tm.z = (double)(force * dz);
						}
					}
					else
					{
						// pair_fp64::add_pair with the owner's values
						const double4 qj = v.sprm4[u];
						int def_j;
						bool mov_j;
						unpack_bits(qj.w, def_j, mov_j);
						fl |= mov_j ? 2 : 0;
						const double d = dist < 0.00001 ? 0.00001 : dist;
						double rep = 1.0 - d / (ri + qj.x);
						rep = rep < 0 ? 0 : rep;
						rep = rep * rep;
						tm.w = rep * simple_pressure_coefficient;
						if (mov_o)
						{
							rep = rep * sqrt(repi * qj.y);
							double adh = 1.0 - d / ad;
							adh = adh * adh;
							adh = adh * sqrt(adhi * qj.z * v.saff[(int64_t)t_o * D + def_j] * v.saff[(int64_t)u * D + def_o]);
							const double force = (rep - adh) / d;
							tm.x = force * ddx;
							tm.y = force * ddy;
							tm.z = force * ddz;
						}
					}
				}
				s_term[warp][lane] = tm;
				s_flag[warp][lane] = fl;
			}
			__syncwarp();
			const int lo = max(off, base), hi = min(off + n, base + 32);
			for (int qq = lo; qq < hi; qq++)
			{
				const int fl = s_flag[warp][qq - base];
				if (!(fl & 1))
					continue;
				const double4 tm = s_term[warp][qq - base];
				if (F32)
				{
					if (mov_i)
						fp.add((float)tm.w);
					if (fl & 2)
						fp.add((float)tm.w);
					if (mov_i)
					{
						fx.add((float)tm.x);
						fy.add((float)tm.y);
						fz.add((float)tm.z);
					}
				}
				else
				{
					if (mov_i)
						pressure = pressure + tm.w;
					if (fl & 2)
						pressure = pressure + tm.w;
					if (mov_i)
					{
						vx = vx + tm.x;
						vy = vy + tm.y;
						vz = vz + tm.z;
					}
				}
			}
			__syncwarp();
		}
		n = 0;
	};

	// warp-uniform scan: one candidate per lane per iteration, rows in order
	int k = 0;
	int2 b = s_rows[0][threadIdx.x];
	int soff = staged ? s_o[0] - s_a[0] : 0;
	int u = b.x;
	while (true)
	{
		while (u >= b.y && k + 1 < NR)
		{
			k++;
			b = s_rows[k][threadIdx.x];
			soff = staged ? s_o[k] - s_a[k] : 0;
			u = b.x;
		}
		const bool has = u < b.y;
		if (!__any_sync(0xffffffffu, has))
			break;
		if (has)
		{
			// up to kStageScan candidates of the current row, loads first
			const int m = min(kStageScan, b.y - u);
			float4 q[kStageScan];
#pragma unroll
			for (int j = 0; j < kStageScan; j++)
				if (j < m)
					q[j] = P[u + j + soff];
#pragma unroll
			for (int j = 0; j < kStageScan; j++)
				if (j < m && u + j != t && filter_keep<DIMS>(pf, q[j], margin))
				{
					list[n * stride] = u + j;
					n++;
				}
			u += m;
		}
		if (__any_sync(0xffffffffu, n > kList - kStageScan))
			flush();
	}
	flush();
	if (!act)
		return;
	double4 p = make_double4(pi.x, pi.y, pi.z, 0.0);
	double4 vp = mov_i ? v.vprev[s] : make_double4(0, 0, 0, 0);
	if (F32)
	{
		vx = vel0.x + fx.value();
		vy = vel0.y + fy.value();
		vz = vel0.z + fz.value();
		pressure = fp.value();
	}
	if (mov_i)
	{
		double4 vel = make_double4(vx, vy, vz, 0.0);
		if (WALLS)
			walls<DIMS>(v, R, p, qi.x, bm, vel);
		if (SPRINGS && nspr > 0)
			spring_contract<DIMS>(v, cur, s, nspr, p, def_i, vel);
		ab2<DIMS>(v.dt, p, vel, vp);
	}
	v.pressure[s] = pressure;
	if (mov_i)
	{
		v.vprev[s] = vp;
		if (VEL)
			v.vel[s] = make_double4(0, 0, 0, 0);
	}
	v.pos[cur ^ 1][s] = p;
	if (!(p.x == p.x && p.y == p.y && p.z == p.z))
		atomicOr(v.err, ERR_NONFINITE);
	if (to_remove<DIMS>(R, p, flag))
		append_bad(v, r, s - R.base);
}

template <int DIMS, bool F32>
__global__ void __launch_bounds__(kStageThreads, 4) k_fused_staged(view v, int cur, int cap, int opts)
{
	grid_wait();
	bump_spring_epochs(v);
	extern __shared__ float4 stage_raw[];
	fused_staged_block<DIMS, F32>(v, cur, cap, opts, blockIdx.x, stage_raw);
}

// ---------------------------------------------------------------------------
// fused step, one thread per agent, candidates fetched in batches.
//
// The per-thread pass above walks each stencil row's candidates one load at a
// time, and a warp runs as many iterations per row as its longest row among
// 32 agents, so a sparse tissue costs a warp some thirty dependent loads. Here
// a thread numbers its candidates in the reference's order (rows z, y; in a
// row the key-ordered range of its three voxels) and fetches them
// kFlatBatch at a time into shared memory with asynchronous copies, which
// keep no registers while they are in flight; the single-precision positions
// go through the filter of the cooperative passes (it never rejects a pair the
// FP64 test accepts), and the candidates it keeps fetch their FP64 position,
// parameters and affinity entry kFlatHits at a time, again as one round trip,
// before the exact test and the pair code run in candidate order. The
// epilogue's per-agent rows and the first two spring partners are prefetched
// into L2 while the scan runs.
// ---------------------------------------------------------------------------

constexpr int kFlatThreads = 128;
constexpr int kFlatBatch = 10; // candidates a thread fetches per round
constexpr int kFlatHits = 2;   // kept candidates whose FP64 data a round fetches (5 slots each)
static_assert(5 * kFlatHits <= kFlatBatch, "a kept candidate's data takes five slots of its thread's column");

// Each thread owns one column [.][tid] of the slot arrays. A round first
// holds up to kFlatBatch single-precision candidate positions; once the
// filter has read them, the same slots take the kept candidates' data: FP64
// position (slots 5h, 5h+1), parameters (5h+2, 5h+3; the FP32 form's float4 in
// 5h+2) and affinity entry (5h+4).
struct flat_smem
{
	float4 slot[kFlatBatch][kFlatThreads];
	int32_t cu[kFlatBatch][kFlatThreads]; // array positions of the round's candidates
	int2 rows[9][kFlatThreads];			  // per stencil row: first candidate number, array position - number
};

__device__ __forceinline__ double4 slots_double4(const float4& a, const float4& b)
{
	const double2 x = *reinterpret_cast<const double2*>(&a);
	const double2 y = *reinterpret_cast<const double2*>(&b);
	return make_double4(x.x, x.y, y.x, y.y);
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

template <int BYTES>
__device__ __forceinline__ void cp_async_small(void* dst, const void* src)
{
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(BYTES) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
	asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }


// membrane, springs, Adams-Bashforth, then the agent's stores: the end of
// the fused pass for the agent in slot s with the pair sums (vx, vy, vz,
// pressure); pi is its key-ordered position, radius its radius
template <int DIMS>
__device__ __forceinline__ void agent_finish(const view& v, int cur, int opts, int t, int32_t key, int s, int r,
											 const rep_info& R, const double4& pi, double radius, int def_i, bool mov_i,
											 int nspr, double vx, double vy, double vz, double pressure)
{
	const bool walls_on = (opts & FUSED_WALLS) != 0;
	const bool vel_on = (opts & FUSED_VEL) != 0;
	double4 p = make_double4(pi.x, pi.y, pi.z, 0.0);
	double4 vp = make_double4(0, 0, 0, 0);
	const uint8_t flag = v.flags[s];
	if (mov_i)
	{
		vp = v.vprev[s];
		double4 vel = make_double4(vx, vy, vz, 0.0);
		if (walls_on)
			walls<DIMS>(v, R, p, radius, v.prm[s].w, vel);
		if (nspr > 0)
			spring_contract<DIMS>(v, cur, s, nspr, p, def_i, vel);
		ab2<DIMS>(v.dt, p, vel, vp);
	}
	v.pressure[s] = pressure;
	if (mov_i)
	{
		v.vprev[s] = vp;
		if (vel_on)
			v.vel[s] = make_double4(0, 0, 0, 0);
	}
	v.pos[cur ^ 1][s] = p;
	if (!(p.x == p.x && p.y == p.y && p.z == p.z))
		atomicOr(v.err, ERR_NONFINITE);
	if (to_remove<DIMS>(R, p, flag))
		append_bad(v, r, s - R.base);
	if (opts & FUSED_PRODUCE)
		produce_entry(v, R, t, s, key, p, pi.w);
}

// the agent at key-ordered position t, with its block's shared slots `sm`
template <int DIMS, bool F32>
__device__ __forceinline__ void fused_flat_agent(const view& v, int cur, int opts, int t, flat_smem& sm)
{
	constexpr int NR = DIMS == 3 ? 9 : (DIMS == 2 ? 3 : 1);
	const bool walls_on = (opts & FUSED_WALLS) != 0;
	const bool springs_on = (opts & FUSED_SPRINGS) != 0;
	const bool vel_on = (opts & FUSED_VEL) != 0;
	const int tid = threadIdx.x;
	if (t >= v.total_cap)
		return;
	// the agent's key-ordered rows, issued before the count is known (t is
	// below the capacity, so the loads stay in bounds)
	const int s = v.sorted[t];
	const int32_t key = v.skey[t];
	const double4 pi = v.spos4[t];
	const float4 pf = v.sposf[t];
	const double4 qi = v.sprm4[t];
	if (t >= *v.cursor)
		return;
	int def_i;
	bool mov_i;
	unpack_bits(qi.w, def_i, mov_i);
	const long long bits_i = __double_as_longlong(qi.w);
	const int r = v.nreps == 1 ? 0 : (v.nreps <= 65536 ? (int)((bits_i >> 48) & 0xffff) : v.rid[s]);
	const rep_info& R = v.reps[r];
	const int D = v.ndefs;
	// this agent's affinity row: read per neighbour by definition index
	if (F32)
		prefetch_l1(v.safff + (int64_t)t * D);
	else
		prefetch_l1(v.saff + (int64_t)t * D);

	// stencil rows and the candidate numbering
	const int32_t lk = key - (int32_t)R.vox_base;
	const int g0 = R.grid[0], g1 = R.grid[1], g2 = R.grid[2];
	int cx, cy, cz;
	voxel_coords(R, lk, cx, cy, cz);
	const int xlo = cx > 0 ? cx - 1 : 0;
	const int xhi = cx + 1 < g0 ? cx + 1 : g0 - 1;
	int lo[NR], hi[NR];
#pragma unroll
	for (int k = 0; k < NR; k++)
	{
		const int dz = DIMS == 3 ? k / 3 - 1 : 0;
		const int dy = DIMS >= 2 ? k % 3 - 1 : 0;
		const int z = cz + dz, y = cy + dy;
		const bool ok = z >= 0 && z < g2 && y >= 0 && y < g1;
		const int32_t row = ok ? (int32_t)R.vox_base + g0 * (y + g1 * z) : 0;
		lo[k] = ok ? v.vstart[row + xlo] : 0;
		hi[k] = ok ? v.vstart[row + xhi + 1] : 0;
	}
	// the epilogue's per-agent rows are read after the scan: ask L2 for them
	// now, with the indices of the first two spring partners
	const int nspr = (springs_on && mov_i) ? unpack_springs(qi.w) : 0;
	prefetch_l2(v.flags + s);
	int j0 = -1, j1 = -1;
	if (mov_i)
	{
		prefetch_l2(v.vprev + s);
		if (walls_on)
			prefetch_l2(&v.prm[s].w);
		if (nspr > 0)
		{
			prefetch_l2(v.ec + s);
			j0 = v.springs[(int64_t)s * v.scap];
			if (nspr > 1)
				j1 = v.springs[(int64_t)s * v.scap + 1];
		}
	}
	// the scan adds its terms to the velocity the agent enters the step with
	double vx = 0.0, vy = 0.0, vz = 0.0, pressure = 0.0;
	if (vel_on && mov_i)
	{
		const double4 v0 = v.vel[s];
		vx = v0.x;
		vy = v0.y;
		vz = v0.z;
	}
	int C = 0;
#pragma unroll
	for (int k = 0; k < NR; k++)
	{
		sm.rows[k][tid] = make_int2(C, lo[k] - C);
		C += hi[k] - lo[k];
	}

	nsum fx, fy, fz, fp;
	const float margin = R.fmargin;
	int k = 0;								 // row of the next candidate
	int knext = NR > 1 ? sm.rows[1][tid].x : C; // first candidate number of row k + 1
	bool partners = false;
	for (int c0 = 0; c0 < C; c0 += kFlatBatch)
	{
		const int nb = min(kFlatBatch, C - c0);
#pragma unroll
		for (int j = 0; j < kFlatBatch; j++)
			if (j < nb)
			{
				const int c = c0 + j;
				while (c >= knext)
				{
					k++;
					knext = k + 1 < NR ? sm.rows[k + 1][tid].x : C;
				}
				const int u = sm.rows[k][tid].y + c;
				sm.cu[j][tid] = u;
				cp_async16(&sm.slot[j][tid], v.sposf + u);
			}
		if (!partners)
		{
			// the partner indices have arrived by now: their rows to L2
			partners = true;
			if (j0 >= 0)
			{
				prefetch_l2(v.pos[cur] + j0);
				prefetch_l2(v.def + j0);
				prefetch_l2(v.ec + j0);
				prefetch_l2(v.aff + (int64_t)j0 * D + def_i);
			}
			if (j1 >= 0)
			{
				prefetch_l2(v.pos[cur] + j1);
				prefetch_l2(v.def + j1);
				prefetch_l2(v.ec + j1);
				prefetch_l2(v.aff + (int64_t)j1 * D + def_i);
			}
		}
		cp_async_wait_all();
		unsigned hm = 0;
#pragma unroll
		for (int j = 0; j < kFlatBatch; j++)
			if (j < nb && sm.cu[j][tid] != t && filter_keep<DIMS>(pf, sm.slot[j][tid], margin))
				hm |= 1u << j;
		while (hm)
		{
			// FP64 position, parameters and affinity of up to kFlatHits kept
			// candidates in one round trip
			int hu[kFlatHits];
#pragma unroll
			for (int h = 0; h < kFlatHits; h++)
			{
				hu[h] = -1;
				if (hm)
				{
					const int j = __ffs(hm) - 1;
					hm &= hm - 1;
					const int u = sm.cu[j][tid];
					hu[h] = u;
					const char* gp = reinterpret_cast<const char*>(v.spos4 + u);
					cp_async16(&sm.slot[5 * h][tid], gp);
					cp_async16(&sm.slot[5 * h + 1][tid], gp + 16);
					if (F32)
					{
						cp_async16(&sm.slot[5 * h + 2][tid], v.sprmf + u);
						cp_async_small<4>(&sm.slot[5 * h + 4][tid], v.safff + (int64_t)u * D + def_i);
					}
					else
					{
						const char* gq = reinterpret_cast<const char*>(v.sprm4 + u);
						cp_async16(&sm.slot[5 * h + 2][tid], gq);
						cp_async16(&sm.slot[5 * h + 3][tid], gq + 16);
						cp_async_small<8>(&sm.slot[5 * h + 4][tid], v.saff + (int64_t)u * D + def_i);
					}
				}
			}
			cp_async_wait_all();
#pragma unroll
			for (int h = 0; h < kFlatHits; h++)
			{
				if (hu[h] < 0)
					continue;
				// exact FP64 neighbour test: distance <= rmad_i r_i + rmad_j r_j
				const double4 q = slots_double4(sm.slot[5 * h][tid], sm.slot[5 * h + 1][tid]);
				const double ddx = pi.x - q.x;
				const double ddy = DIMS >= 2 ? pi.y - q.y : 0.0;
				const double ddz = DIMS >= 3 ? pi.z - q.z : 0.0;
				double d2 = ddx * ddx;
				if (DIMS >= 2)
					d2 = d2 + ddy * ddy;
				if (DIMS >= 3)
					d2 = d2 + ddz * ddz;
				const double ad = pi.w + q.w;
				const double dist = DIMS == 1 ? fabs(ddx) : sqrt(d2);
				if (!(dist <= ad))
					continue;
				if (F32)
				{
					// pair_fp32::add with this agent's values
					const float4 qj = sm.slot[5 * h + 2][tid];
					const float afj = sm.slot[5 * h + 4][tid].x;
					int def_j, spr_j;
					bool mov_j;
					unpack_fbits(qj.w, def_j, mov_j, spr_j);
					const float dx = (float)ddx, dy = (float)ddy, dz = (float)ddz;
					float d2f = dx * dx;
					if (DIMS >= 2)
						d2f = d2f + dy * dy;
					if (DIMS >= 3)
						d2f = d2f + dz * dz;
					const float distf = DIMS == 1 ? fabsf(dx) : sqrtf(d2f);
					const float d = distf < 0.00001f ? 0.00001f : distf;
					float rep = 1.f - d / ((float)qi.x + qj.x);
					rep = rep < 0.f ? 0.f : rep;
					rep = rep * rep;
					const float term = rep * 36.64504274775163f;
					if (mov_i)
						fp.add(term);
					if (mov_j)
						fp.add(term);
					if (mov_i)
					{
						rep = rep * sqrtf((float)qi.y * qj.y);
						float adh = 1.f - d / (pf.w + (float)q.w);
						adh = adh * adh;
						adh = adh * sqrtf((float)qi.z * qj.z * v.safff[(int64_t)t * D + def_j] * afj);
						const float force = (rep - adh) / d;
						fx.add(force * dx);
						fy.add(force * dy);
						fz.add(force * dz);
					}
				}
				else
				{
					// pair_fp64::add_pair with this agent's values
					const double4 pr = slots_double4(sm.slot[5 * h + 2][tid], sm.slot[5 * h + 3][tid]);
					int def_j;
					bool mov_j;
					unpack_bits(pr.w, def_j, mov_j);
					const double d = dist < 0.00001 ? 0.00001 : dist;
					double rep = 1.0 - d / (qi.x + pr.x);
					rep = rep < 0 ? 0 : rep;
					rep = rep * rep;
					const double term = rep * simple_pressure_coefficient;
					if (mov_i)
						pressure = pressure + term;
					if (mov_j)
						pressure = pressure + term;
					if (mov_i)
					{
						rep = rep * sqrt(qi.y * pr.y);
						double adh = 1.0 - d / ad;
						adh = adh * adh;
						const double afj = *reinterpret_cast<const double*>(&sm.slot[5 * h + 4][tid]);
						adh = adh * sqrt(qi.z * pr.z * v.saff[(int64_t)t * D + def_j] * afj);
						const double force = (rep - adh) / d;
						vx = vx + force * ddx;
						vy = vy + force * ddy;
						vz = vz + force * ddz;
					}
				}
			}
		}
	}
	if (F32)
	{
		vx = vx + fx.value();
		vy = vy + fy.value();
		vz = vz + fz.value();
		pressure = fp.value();
	}

	agent_finish<DIMS>(v, cur, opts, t, key, s, r, R, pi, qi.x, def_i, mov_i, nspr, vx, vy, vz, pressure);
}

template <int DIMS, bool F32>
__global__ void __launch_bounds__(kFlatThreads, 5) k_fused_flat(view v, int cur, int opts)
{
	grid_wait();
	bump_spring_epochs(v);
	extern __shared__ __align__(16) unsigned char flat_raw[];
	fused_flat_agent<DIMS, F32>(v, cur, opts, blockIdx.x * kFlatThreads + threadIdx.x,
								*reinterpret_cast<flat_smem*>(flat_raw));
}

// ---------------------------------------------------------------------------
// fused step, one thread per agent, candidates shared out over the warp.
//
// In a sparse tissue the agents of a warp hold very different numbers of
// candidates, and the passes above run a warp for as many rounds as its
// busiest lane needs. Here a warp lays its 32 agents' candidates end to end,
// agent by agent and each agent's in the reference's order (rows z, y; in a
// row the key-ordered range of its three voxels), and lane l takes the
// candidates l, l + 32, ... of that list: the filter runs on full warps. The
// candidates it keeps are listed in the same order; full warps then fetch
// their FP64 data and evaluate the pair terms, and each agent's lane adds its
// own terms in its candidate order, so every sum rounds as in the
// reference's loop.
// ---------------------------------------------------------------------------

constexpr int kQueueThreads = 128;
constexpr int kQueueRounds = 4;	 // candidate rounds whose loads are in flight together
constexpr int kQueueHits = 256; // kept candidates a warp lists before evaluating them

struct queue_warp
{
	int2 rows[9][32];		   // per agent and stencil row: first candidate number, array position - number
	int32_t first[33];		   // each agent's first candidate in the warp's list; first[32]: the total
	int32_t t[32];			   // the agents' key-ordered positions (-1: no agent)
	int32_t key[32], slot[32]; // the agents' voxel keys and slots
	float margin[32];		   // the agents' filter margins
	float4 pf[32];			   // single-precision positions
	double4 pi[32], qi[32];	   // FP64 positions and parameter rows
	int2 hit[kQueueHits];	   // kept candidates: (agent lane, array position)
	double term[32], fx[32], fy[32], fz[32]; // the pair terms of a round of kept candidates
	int32_t hflags[32];		   // bit 0: within range, bit 1: the neighbour is movable
	uint32_t seg[32];		   // per agent: the lanes of the round holding its candidates
};

struct queue_smem
{
	queue_warp w[kQueueThreads / 32];
};

// Evaluates the warp's kept candidates [0, nh) in rounds of 32 and adds each
// agent's terms to its sums in list order.
template <int DIMS, bool F32>
__device__ __forceinline__ void queue_hits(const view& v, queue_warp& w, int nh, bool act, bool mov_i, double& vx,
										   double& vy, double& vz, double& pressure, nsum& fx, nsum& fy, nsum& fz,
										   nsum& fp)
{
	const int lane = threadIdx.x & 31;
	const int D = v.ndefs;
	for (int h0 = 0; h0 < nh; h0 += 32)
	{
		const int h = h0 + lane;
		int own = -1, flags = 0;
		double term = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
		if (h < nh)
		{
			const int2 e = w.hit[h];
			own = e.x;
			const int u = e.y;
			const double4 pa = w.pi[own];
			const double4 qa = w.qi[own];
			const int ta = w.t[own];
			int def_a;
			bool mov_a;
			unpack_bits(qa.w, def_a, mov_a);
			const double4 q = v.spos4[u];
			// exact FP64 neighbour test: distance <= rmad_i r_i + rmad_j r_j
			const double ddx = pa.x - q.x;
			const double ddy = DIMS >= 2 ? pa.y - q.y : 0.0;
			const double ddz = DIMS >= 3 ? pa.z - q.z : 0.0;
			double d2 = ddx * ddx;
			if (DIMS >= 2)
				d2 = d2 + ddy * ddy;
			if (DIMS >= 3)
				d2 = d2 + ddz * ddz;
			const double ad = pa.w + q.w;
			const double dist = DIMS == 1 ? fabs(ddx) : sqrt(d2);
			if (F32)
			{
				// pair_fp32::add with the agent's values
				const float4 qj = v.sprmf[u];
				const float afj = v.safff[(int64_t)u * D + def_a];
				int def_j, spr_j;
				bool mov_j;
				unpack_fbits(qj.w, def_j, mov_j, spr_j);
				if (dist <= ad)
				{
					flags = 1 | (mov_j ? 2 : 0);
					const float dx = (float)ddx, dy = (float)ddy, dz = (float)ddz;
					float d2f = dx * dx;
					if (DIMS >= 2)
						d2f = d2f + dy * dy;
					if (DIMS >= 3)
						d2f = d2f + dz * dz;
					const float distf = DIMS == 1 ? fabsf(dx) : sqrtf(d2f);
					const float d = distf < 0.00001f ? 0.00001f : distf;
					float rep = 1.f - d / ((float)qa.x + qj.x);
					rep = rep < 0.f ? 0.f : rep;
					rep = rep * rep;
					term = rep * 36.64504274775163f;
					if (mov_a)
					{
						rep = rep * sqrtf((float)qa.y * qj.y);
						float adh = 1.f - d / (w.pf[own].w + (float)q.w);
						adh = adh * adh;
						adh = adh * sqrtf((float)qa.z * qj.z * v.safff[(int64_t)ta * D + def_j] * afj);
						const float force = (rep - adh) / d;
						tx = force * dx;
						ty = force * dy;
						tz = force * dz;
					}
				}
			}
			else
			{
				// pair_fp64::add_pair with the agent's values
				const double4 pr = v.sprm4[u];
				const double afj = v.saff[(int64_t)u * D + def_a];
				int def_j;
				bool mov_j;
				unpack_bits(pr.w, def_j, mov_j);
				if (dist <= ad)
				{
					flags = 1 | (mov_j ? 2 : 0);
					const double d = dist < 0.00001 ? 0.00001 : dist;
					double rep = 1.0 - d / (qa.x + pr.x);
					rep = rep < 0 ? 0 : rep;
					rep = rep * rep;
					term = rep * simple_pressure_coefficient;
					if (mov_a)
					{
						rep = rep * sqrt(qa.y * pr.y);
						double adh = 1.0 - d / ad;
						adh = adh * adh;
						adh = adh * sqrt(qa.z * pr.z * v.saff[(int64_t)ta * D + def_j] * afj);
						const double force = (rep - adh) / d;
						tx = force * ddx;
						ty = force * ddy;
						tz = force * ddz;
					}
				}
			}
		}
		w.term[lane] = term;
		w.fx[lane] = tx;
		w.fy[lane] = ty;
		w.fz[lane] = tz;
		w.hflags[lane] = flags;
		const unsigned grp = __match_any_sync(0xffffffffu, own);
		if (own >= 0 && lane == __ffs(grp) - 1)
			w.seg[own] = grp;
		__syncwarp();
		if (act)
		{
			unsigned m = w.seg[lane];
			w.seg[lane] = 0;
			while (m)
			{
				const int l = __ffs(m) - 1;
				m &= m - 1;
				const int f = w.hflags[l];
				if (!(f & 1))
					continue;
				const double tm = w.term[l];
				if (F32)
				{
					if (mov_i)
						fp.add((float)tm);
					if (f & 2)
						fp.add((float)tm);
					if (mov_i)
					{
						fx.add((float)w.fx[l]);
						fy.add((float)w.fy[l]);
						fz.add((float)w.fz[l]);
					}
				}
				else
				{
					if (mov_i)
						pressure = pressure + tm;
					if (f & 2)
						pressure = pressure + tm;
					if (mov_i)
					{
						vx = vx + w.fx[l];
						vy = vy + w.fy[l];
						vz = vz + w.fz[l];
					}
				}
			}
		}
		__syncwarp();
	}
}

// the agent at key-ordered position t; every lane of the warp calls it
template <int DIMS, bool F32>
__device__ __forceinline__ void fused_queue_agent(const view& v, int cur, int opts, int t, queue_warp& w)
{
	constexpr int NR = DIMS == 3 ? 9 : (DIMS == 2 ? 3 : 1);
	const bool springs_on = (opts & FUSED_SPRINGS) != 0;
	const bool walls_on = (opts & FUSED_WALLS) != 0;
	const bool vel_on = (opts & FUSED_VEL) != 0;
	const int lane = threadIdx.x & 31;
	int s = 0;
	int32_t key = 0;
	double4 pi = make_double4(0, 0, 0, 0), qi = make_double4(0, 0, 0, 0);
	float4 pf = make_float4(0, 0, 0, 0);
	bool act = false;
	if (t < v.total_cap)
	{
		// issued before the count is known (t is below the capacity)
		s = v.sorted[t];
		key = v.skey[t];
		pi = v.spos4[t];
		pf = v.sposf[t];
		qi = v.sprm4[t];
		act = t < *v.cursor;
	}
	int def_i = 0, r = 0;
	bool mov_i = false;
	if (act)
	{
		unpack_bits(qi.w, def_i, mov_i);
		const long long bits_i = __double_as_longlong(qi.w);
		r = v.nreps == 1 ? 0 : (v.nreps <= 65536 ? (int)((bits_i >> 48) & 0xffff) : v.rid[s]);
	}
	const rep_info& R = v.reps[r];
	const int D = v.ndefs;
	int lo[NR], hi[NR];
	if (act)
	{
		// this agent's affinity row: read per neighbour by definition index
		if (F32)
			prefetch_l1(v.safff + (int64_t)t * D);
		else
			prefetch_l1(v.saff + (int64_t)t * D);
		const int32_t lk = key - (int32_t)R.vox_base;
		const int g0 = R.grid[0], g1 = R.grid[1], g2 = R.grid[2];
		int cx, cy, cz;
		voxel_coords(R, lk, cx, cy, cz);
		const int xlo = cx > 0 ? cx - 1 : 0;
		const int xhi = cx + 1 < g0 ? cx + 1 : g0 - 1;
#pragma unroll
		for (int k = 0; k < NR; k++)
		{
			const int dz = DIMS == 3 ? k / 3 - 1 : 0;
			const int dy = DIMS >= 2 ? k % 3 - 1 : 0;
			const int z = cz + dz, y = cy + dy;
			const bool ok = z >= 0 && z < g2 && y >= 0 && y < g1;
			const int32_t row = ok ? (int32_t)R.vox_base + g0 * (y + g1 * z) : 0;
			lo[k] = ok ? v.vstart[row + xlo] : 0;
			hi[k] = ok ? v.vstart[row + xhi + 1] : 0;
		}
	}
	else
	{
#pragma unroll
		for (int k = 0; k < NR; k++)
			lo[k] = hi[k] = 0;
	}
	// the epilogue's per-agent rows are read after the scan: ask L2 for them
	// now, with the first two spring partners' rows once their indices arrive
	const int nspr = (act && springs_on && mov_i) ? unpack_springs(qi.w) : 0;
	int j0 = -1, j1 = -1;
	if (act)
	{
		prefetch_l2(v.flags + s);
		if (mov_i)
		{
			prefetch_l2(v.vprev + s);
			if (walls_on)
				prefetch_l2(&v.prm[s].w);
			if (nspr > 0)
			{
				prefetch_l2(v.ec + s);
				j0 = v.springs[(int64_t)s * v.scap];
				if (nspr > 1)
					j1 = v.springs[(int64_t)s * v.scap + 1];
			}
		}
	}
	double vx = 0.0, vy = 0.0, vz = 0.0, pressure = 0.0;
	if (vel_on && mov_i)
	{
		const double4 v0 = v.vel[s];
		vx = v0.x;
		vy = v0.y;
		vz = v0.z;
	}
	// the warp's list of candidates
	int C = 0;
#pragma unroll
	for (int k = 0; k < NR; k++)
	{
		w.rows[k][lane] = make_int2(C, lo[k] - C);
		C += hi[k] - lo[k];
	}
	int incl = C;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1)
	{
		const int y = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o)
			incl += y;
	}
	const int total = __shfl_sync(0xffffffffu, incl, 31);
	w.first[lane] = incl - C;
	if (lane == 31)
		w.first[32] = total;
	w.t[lane] = act ? t : -1;
	w.key[lane] = key;
	w.slot[lane] = s;
	w.margin[lane] = R.fmargin;
	w.pf[lane] = pf;
	w.pi[lane] = pi;
	w.qi[lane] = qi;
	w.seg[lane] = 0;
	__syncwarp();
	if (j0 >= 0)
	{
		prefetch_l2(v.pos[cur] + j0);
		prefetch_l2(v.def + j0);
		prefetch_l2(v.ec + j0);
		prefetch_l2(v.aff + (int64_t)j0 * D + def_i);
	}
	if (j1 >= 0)
	{
		prefetch_l2(v.pos[cur] + j1);
		prefetch_l2(v.def + j1);
		prefetch_l2(v.ec + j1);
		prefetch_l2(v.aff + (int64_t)j1 * D + def_i);
	}

	nsum fx, fy, fz, fp;
	int nh = 0; // kept candidates listed (the same in every lane)
	for (int base = 0; base < total; base += 32 * kQueueRounds)
	{
		float4 cand[kQueueRounds];
		int cu[kQueueRounds], own[kQueueRounds];
#pragma unroll
		for (int q = 0; q < kQueueRounds; q++)
		{
			const int x = base + q * 32 + lane;
			own[q] = -1;
			cu[q] = 0;
			if (x < total)
			{
				// the agent: the last one whose first candidate is at most x
				// (an agent without candidates shares its successor's first)
				int i = 0;
#pragma unroll
				for (int step = 16; step >= 1; step >>= 1)
					if (w.first[i + step] <= x)
						i += step;
				const int c = x - w.first[i];
				// the row: the last one whose first candidate is at most c
				int k = 0;
#pragma unroll
				for (int kk = 1; kk < NR; kk++)
					k += w.rows[kk][i].x <= c;
				own[q] = i;
				cu[q] = w.rows[k][i].y + c;
				cand[q] = v.sposf[cu[q]];
			}
		}
#pragma unroll
		for (int q = 0; q < kQueueRounds; q++)
		{
			bool keep = false;
			if (own[q] >= 0)
				keep = cu[q] != w.t[own[q]] && filter_keep<DIMS>(w.pf[own[q]], cand[q], w.margin[own[q]]);
			const unsigned m = __ballot_sync(0xffffffffu, keep);
			if (keep)
				w.hit[nh + __popc(m & ((1u << lane) - 1))] = make_int2(own[q], cu[q]);
			nh += __popc(m);
		}
		__syncwarp();
		if (nh > kQueueHits - 32 * kQueueRounds)
		{
			queue_hits<DIMS, F32>(v, w, nh, act, mov_i, vx, vy, vz, pressure, fx, fy, fz, fp);
			nh = 0;
		}
	}
	if (nh > 0)
		queue_hits<DIMS, F32>(v, w, nh, act, mov_i, vx, vy, vz, pressure, fx, fy, fz, fp);
	if (!act)
		return;
	if (F32)
	{
		vx = vx + fx.value();
		vy = vy + fy.value();
		vz = vz + fz.value();
		pressure = fp.value();
	}
	// the agent's FP64 rows from the warp's shared copies, so that none of
	// them occupies registers through the scan
	const double4 pi_own = w.pi[lane];
	const double radius = w.qi[lane].x;
	agent_finish<DIMS>(v, cur, opts, t, w.key[lane], w.slot[lane], r, R, pi_own, radius, def_i, mov_i, nspr, vx, vy,
					   vz, pressure);
}

template <int DIMS, bool F32>
__global__ void __launch_bounds__(kQueueThreads, 5) k_fused_queue(view v, int cur, int opts)
{
	grid_wait();
	bump_spring_epochs(v);
	extern __shared__ __align__(16) unsigned char queue_raw[];
	queue_smem& sm = *reinterpret_cast<queue_smem*>(queue_raw);
	fused_queue_agent<DIMS, F32>(v, cur, opts, blockIdx.x * kQueueThreads + threadIdx.x, sm.w[threadIdx.x >> 5]);
}

// ---------------------------------------------------------------------------
// separate reference entry points
// ---------------------------------------------------------------------------

// position_solver::update_cell_neighbors (reference: position_solver.cpp:262-286)
template <int DIMS>
__global__ void __launch_bounds__(kThreads) k_neighbors(view v)
{
	grid_wait();
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= *v.cursor)
		return;
	const int s = v.sorted[t];
	if (v.movable[s] == 0)
	{
		v.ncnt[s] = 0;
		return;
	}
	const rep_info& R = v.reps[rep_of(v, s)];
	int n = 0;
	int32_t* out = v.nidx + (int64_t)s * v.ncap;
	const int cap = v.ncap;
	__shared__ int32_t list[kList * kThreads];
	for_each_neighbor<DIMS>(v, R, t, v.skey[t], v.spos4[t], list + threadIdx.x, [&](int u) {
		if (n < cap)
			out[n] = v.sorted[u];
		n++;
	});
	if (n > cap)
		atomicOr(v.err, ERR_NEIGHBOR_CAPACITY);
	v.ncnt[s] = n;
}

__global__ void k_clear_pressure(view v)
{
	grid_wait();
	int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, local;
	if (live(v, s, r, local))
		v.pressure[s] = 0;
}

// position_solver::update_cell_forces over the stored neighbour lists
// (reference: position_solver.cpp:15-22,99-113,158-178,233-260). Pressure
// of a movable agent is gathered from its own list (lists are symmetric
// between movable agents); pressure of a non-movable agent is added
// atomically by its movable neighbours.
template <int DIMS>
__global__ void __launch_bounds__(kThreads) k_forces(view v, int cur)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, local;
	if (!live(v, s, r, local) || v.movable[s] == 0)
		return;
	pair_fp64 acc;
	acc.prm_i = v.prm[s];
	acc.def_i = v.def[s];
	acc.mov_i = true;
	acc.aff_i = v.aff + (int64_t)s * v.ndefs;
	const double4 v0 = v.vel[s];
	acc.vx = v0.x;
	acc.vy = v0.y;
	acc.vz = v0.z;
	const double4 pi = v.pos[cur][s];
	const double ar_i = v.rmad[s] * acc.prm_i.x;
	const int n = min(v.ncnt[s], v.ncap);
	for (int k = 0; k < n; k++)
	{
		const int j = v.nidx[(int64_t)s * v.ncap + k];
		const double4 pj = v.pos[cur][j];
		const double ddx = pi.x - pj.x;
		const double ddy = DIMS >= 2 ? pi.y - pj.y : 0.0;
		const double ddz = DIMS >= 3 ? pi.z - pj.z : 0.0;
		double d2 = ddx * ddx;
		if (DIMS >= 2)
			d2 = d2 + ddy * ddy;
		if (DIMS >= 3)
			d2 = d2 + ddz * ddz;
		const double dist = DIMS == 1 ? fabs(ddx) : sqrt(d2);
		const double ad = ar_i + v.rmad[j] * v.prm[j].x;
		acc.add(v, j, ddx, ddy, ddz, dist, ad);
		if (v.movable[j] == 0)
			atomicAdd(&v.pressure[j], acc.last_term);
	}
	v.pressure[s] = acc.p;
	v.vel[s] = make_double4(acc.vx, acc.vy, acc.vz, 0.0);
}

template <int DIMS>
__global__ void k_membrane(view v, int cur)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, local;
	if (!live(v, s, r, local) || v.movable[s] == 0)
		return;
	double4 vel = v.vel[s];
	const double4 prm = v.prm[s];
	walls<DIMS>(v, v.reps[r], v.pos[cur][s], prm.x, prm.w, vel);
	v.vel[s] = vel;
}

template <int DIMS>
__global__ void k_springs(view v, int cur)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, local;
	if (!live(v, s, r, local) || v.movable[s] == 0 || v.scnt[s] == 0)
		return;
	double4 vel = v.vel[s];
	spring_contract<DIMS>(v, cur, s, v.scnt[s], v.pos[cur][s], v.def[s], vel);
	v.vel[s] = vel;
}

template <int DIMS>
__global__ void k_positions(view v, int cur)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, local;
	if (!live(v, s, r, local) || v.movable[s] == 0)
		return;
	double4 p = v.pos[cur][s];
	double4 vel = v.vel[s];
	double4 vp = v.vprev[s];
	ab2<DIMS>(v.dt, p, vel, vp);
	v.pos[cur][s] = p;
	v.vprev[s] = vp;
	v.vel[s] = make_double4(0, 0, 0, 0);
}

// ---------------------------------------------------------------------------
// container update: remove_single / update_cell_container_internal
// (reference: containers_solver.cpp:58-147) and division
// (containers_solver.cpp:149-188, src/cell.cpp:108-163)
// ---------------------------------------------------------------------------

template <int DIMS>
__global__ void k_mark_remove(view v, int cur)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, local;
	if (!live(v, s, r, local))
		return;
	if (to_remove<DIMS>(v.reps[r], v.pos[cur][s], v.flags[s]))
		append_bad(v, r, local);
}

// ascending sort of a short list by one block (bitonic network in shared
// memory); longer lists fall back to a single-thread heap sort
__device__ void block_sort(int32_t* a, int n, int32_t* sh)
{
	if (n <= 1)
		return;
	if (n <= kSortCap)
	{
		int m = 1;
		while (m < n)
			m <<= 1;
		for (int i = threadIdx.x; i < m; i += blockDim.x)
			sh[i] = i < n ? a[i] : INT32_MAX;
		__syncthreads();
		for (int k = 2; k <= m; k <<= 1)
		{
			for (int j = k >> 1; j > 0; j >>= 1)
			{
				for (int i = threadIdx.x; i < m; i += blockDim.x)
				{
					int l = i ^ j;
					if (l > i)
					{
						bool up = (i & k) == 0;
						int x = sh[i], y = sh[l];
						if ((x > y) == up)
						{
							sh[i] = y;
							sh[l] = x;
						}
					}
				}
				__syncthreads();
			}
		}
		for (int i = threadIdx.x; i < n; i += blockDim.x)
			a[i] = sh[i];
		__syncthreads();
		return;
	}
	if (threadIdx.x == 0)
	{
		// heap sort
		auto sift = [&](int start, int end) {
			int root = start;
			while (2 * root + 1 <= end)
			{
				int child = 2 * root + 1, sw = root;
				if (a[sw] < a[child])
					sw = child;
				if (child + 1 <= end && a[sw] < a[child + 1])
					sw = child + 1;
				if (sw == root)
					return;
				int t = a[root];
				a[root] = a[sw];
				a[sw] = t;
				root = sw;
			}
		};
		for (int start = (n - 2) / 2; start >= 0; start--)
			sift(start, n - 1);
		for (int end = n - 1; end > 0; end--)
		{
			int t = a[end];
			a[end] = a[0];
			a[0] = t;
			sift(0, end - 1);
		}
	}
	__syncthreads();
}

// position of `x` in spring row of slot s, or -1
__device__ __forceinline__ int find_in_row(const view& v, int s, int x)
{
	const int n = v.scnt[s];
	const int32_t* row = v.springs + (int64_t)s * v.scap;
	for (int k = 0; k < n; k++)
		if (row[k] == x)
			return k;
	return -1;
}

// remove_attached (reference: containers_solver.cpp:58-68): every partner of
// `a` drops `a` by moving its last entry into the hole
__device__ void springs_remove_attached(const view& v, int a)
{
	const int n = v.scnt[a];
	for (int k = 0; k < n; k++)
	{
		const int s = v.springs[(int64_t)a * v.scap + k];
		const int at = find_in_row(v, s, a);
		if (at < 0)
		{
			atomicOr(v.err, ERR_SPRING_CAPACITY);
			continue;
		}
		int32_t* row = v.springs + (int64_t)s * v.scap;
		row[at] = row[v.scnt[s] - 1];
		v.scnt[s]--;
	}
}

// rename_attached (reference: containers_solver.cpp:70-79)
__device__ void springs_rename_attached(const view& v, int old_slot, int new_slot)
{
	const int n = v.scnt[old_slot];
	for (int k = 0; k < n; k++)
	{
		const int s = v.springs[(int64_t)old_slot * v.scap + k];
		const int at = find_in_row(v, s, old_slot);
		if (at >= 0)
			v.springs[(int64_t)s * v.scap + at] = new_slot;
	}
}

// Plans the removals of one replicate (one block per replicate): the serial
// loop of update_cell_container_internal over slots 0..nvisit-1, where each
// removal moves the current last agent into the hole and re-tests the hole.
// Produces (hole, source) moves for the agents that end up in holes, the new
// count and the death count; with springs it also replays every removal on
// the spring rows in the reference's order.
__device__ void compact_plan_rep(const view& v, int r, int phenotype_pass, int springs, int fold, int produced,
								 int32_t* sh)
{
	rep_counters& C = v.ctr[r];
	const int nb = min(C.nbad, v.reps[r].cap);
	if (nb == 0)
	{
		if (threadIdx.x == 0)
			v.nmoves[r] = 0;
		return;
	}
	// removals after a fused pass that made the rebuild's entries: they no
	// longer hold; the first replicate to find removals clears them and the
	// count recomputes every entry
	__shared__ int s_first;
	if (threadIdx.x == 0)
		s_first = produced && atomicExch(v.recount, 1) == 0;
	__syncthreads();
	if (s_first)
	{
		const int64_t heads = (int64_t)v.ntiles * kChains;
		for (int64_t k = threadIdx.x; k < heads; k += blockDim.x)
			v.chead[k] = -1;
		for (int k = threadIdx.x; k < v.ntiles; k += blockDim.x)
			v.tdelta[k] = 0;
		for (int k = threadIdx.x; k < ((v.ntiles + (1 << kSuperShift) - 1) >> kSuperShift); k += blockDim.x)
			v.sdelta[k] = 0;
	}
	const int base = v.reps[r].base;
	int32_t* B = v.bad + base;
	block_sort(B, nb, sh);
	if (threadIdx.x != 0)
		return;

	const int nvisit = phenotype_pass ? C.nvisit : C.count;
	const int cnt0 = C.count;
	int cnt = cnt0;
	int ti = nb - 1, nm = 0;
	int64_t deaths = 0;
	bool counts_changed = false; // some partner's spring count changed
	int32_t* moves = v.moves + 2 * (int64_t)base;
	for (int bi = 0; bi < nb; bi++)
	{
		const int h = B[bi];
		if (h >= nvisit || h >= cnt)
			break;
		int occ = h; // original index of the agent now in slot h
		while (true)
		{
			deaths += v.flags[base + occ] == PPC_FLAG_TO_REMOVE;
			const int last = cnt - 1;
			if (springs)
			{
				counts_changed = counts_changed || v.scnt[base + h] > 0;
				springs_remove_attached(v, base + h);
				if (last != h)
				{
					springs_rename_attached(v, base + last, base + h);
					const int n = v.scnt[base + last];
					for (int k = 0; k < n; k++)
						v.springs[(int64_t)(base + h) * v.scap + k] = v.springs[(int64_t)(base + last) * v.scap + k];
					v.scnt[base + h] = n;
					v.scnt[base + last] = 0;
				}
			}
			cnt--;
			if (h == cnt)
			{
				occ = -1;
				break;
			}
			occ = last;
			while (ti >= 0 && B[ti] > last)
				ti--;
			if (!(ti >= 0 && B[ti] == last))
				break;
		}
		if (occ >= 0)
		{
			moves[2 * nm] = h;
			moves[2 * nm + 1] = occ;
			nm++;
			if (fold)
			{
				v.move_src[base + h] = base + occ; // applied by the next k_bin_count
				*v.moves_pending = 1;
			}
		}
	}
	C.count = cnt;
	C.deaths += deaths;
	// the partners' key-ordered rows carry their spring counts
	if (counts_changed)
		*v.params_changed = 1;
	C.nbad = 0;
	v.nmoves[r] = nm;
}

__global__ void k_compact_plan(view v, int phenotype_pass, int springs, int fold, int produced)
{
	grid_wait();
	__shared__ int32_t sh[kSortCap];
	compact_plan_rep(v, blockIdx.x, phenotype_pass, springs, fold, produced, sh);
}

// the planned moves, one thread per move
__global__ void k_compact_apply(view v, int cur)
{
	grid_wait();
	const int r = blockIdx.y;
	const int nm = v.nmoves[r];
	const int base = v.reps[r].base;
	const int32_t* moves = v.moves + 2 * (int64_t)base;
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nm; k += gridDim.x * blockDim.x)
	{
		move_agent(v, cur, base + moves[2 * k], base + moves[2 * k + 1]);
		*v.params_changed = 1; // the hole's agent changed
	}
}

// ---------------------------------------------------------------------------
// stochastic spring attachment and detachment
// (update_spring_attachments_internal, reference: position_solver.cpp:372-449)
// with counter-based draws: agent i's k-th draw of a spring update is
// uniform(seed, spring epoch, replicate, i, k); detachment uses k = 1024 +
// position in i's row, attachment k = 4096 + 2 (neighbour position) and the
// next one.
// ---------------------------------------------------------------------------

// The reference walks agents in order; when the draw for position k of the
// walking agent's row passes and that entry is not yet erased, it erases it
// and the first not-yet-erased entry naming the walker in the partner's row.
// Entries of one pair of agents are touched only while one of the two walks,
// so each agent replays that for each of its partners — the lower index
// first, then the higher — from both rows and the draws of both ends, and
// marks its own erased entries. Each agent writes only its own row.
constexpr int kMaxSpringCopies = 16; // copies of one pair an agent can hold

__global__ void k_spring_detach(view v)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, li;
	if (!live(v, s, r, li))
		return;
	const int n = v.scnt[s];
	const int base = v.reps[r].base;
	const uint64_t ep = (uint64_t)v.ctr[r].spring_epoch;
	const int32_t* row = v.springs + (int64_t)s * v.scap;
	for (int k = 0; k < n; k++)
		v.sdel[(int64_t)s * v.scap + k] = 0;
	for (int k = 0; k < n; k++)
	{
		const int j = row[k];
		bool seen = false; // pair handled at its first entry
		for (int q = 0; q < k && !seen; q++)
			seen = row[q] == j;
		if (seen)
			continue;
		const int32_t* rowj = v.springs + (int64_t)j * v.scap;
		const int nj = v.scnt[j];
		int P[kMaxSpringCopies], Q[kMaxSpringCopies];
		int np = 0, nq = 0;
		for (int q = k; q < n && np < kMaxSpringCopies; q++)
			if (row[q] == j)
				P[np++] = q;
		for (int q = 0; q < nj && nq < kMaxSpringCopies; q++)
			if (rowj[q] == s)
				Q[nq++] = q;
		// a walks first: its entries A name b, b's entries B name a
		const bool s_first = li < j - base;
		const int la = s_first ? li : j - base, lb = s_first ? j - base : li;
		const double ra = (s_first ? v.drate[s] : v.drate[j]) * v.dt;
		const double rb = (s_first ? v.drate[j] : v.drate[s]) * v.dt;
		const int* A = s_first ? P : Q;
		const int* B = s_first ? Q : P;
		const int na = s_first ? np : nq, nb = s_first ? nq : np;
		bool ea[kMaxSpringCopies], eb[kMaxSpringCopies];
		for (int q = 0; q < kMaxSpringCopies; q++)
			ea[q] = eb[q] = false;
		for (int q = 0; q < na; q++)
			if (ppc_uniform(v.seed, ep, (uint64_t)r, (uint64_t)la, 1024u + (uint64_t)A[q]) <= ra)
			{
				ea[q] = true;
				int f = 0;
				while (f < nb && eb[f])
					f++;
				if (f < nb)
					eb[f] = true;
			}
		for (int q = 0; q < nb; q++)
			if (!eb[q] && ppc_uniform(v.seed, ep, (uint64_t)r, (uint64_t)lb, 1024u + (uint64_t)B[q]) <= rb)
			{
				eb[q] = true;
				int f = 0;
				while (f < na && ea[f])
					f++;
				if (f < na)
					ea[f] = true;
			}
		const bool* mine = s_first ? ea : eb;
		for (int q = 0; q < np; q++)
			v.sdel[(int64_t)s * v.scap + P[q]] = mine[q] ? 1 : 0;
	}
}

// removes the marked springs from each row, keeping the order of the rest
__global__ void k_spring_compact_rows(view v)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, li;
	if (!live(v, s, r, li))
		return;
	const int n = v.scnt[s];
	int m = 0;
	for (int k = 0; k < n; k++)
		if (!v.sdel[(int64_t)s * v.scap + k])
			v.springs[(int64_t)s * v.scap + m++] = v.springs[(int64_t)s * v.scap + k];
	v.scnt[s] = m;
}

// attachment draws for every neighbour j > i of i (neighbour lists from
// k_neighbors, in the reference's order); the passing (i, position) pairs
// go to the replicate's candidate list, encoded as i * ncap + position
__global__ void k_spring_attach_draws(view v)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, li;
	if (!live(v, s, r, li))
		return;
	const int base = v.reps[r].base;
	const uint64_t ep = (uint64_t)v.ctr[r].spring_epoch;
	const int D = v.ndefs;
	const int nn = min(v.ncnt[s], v.ncap);
	for (int k = 0; k < nn; k++)
	{
		const int j = v.nidx[(int64_t)s * v.ncap + k];
		if (j - base < li)
			continue;
		const double prob_l = v.arate[s] * v.dt * v.aff[(int64_t)s * D + v.def[j]];
		const double prob_r = v.arate[j] * v.dt * v.aff[(int64_t)j * D + v.def[s]];
		if (ppc_uniform(v.seed, ep, (uint64_t)r, (uint64_t)li, 4096u + 2u * (uint64_t)k) <= prob_l
			|| ppc_uniform(v.seed, ep, (uint64_t)r, (uint64_t)li, 4096u + 2u * (uint64_t)k + 1u) <= prob_r)
		{
			const int q = atomicAdd(&v.ctr[r].nattach, 1);
			if (q < v.reps[r].cap)
				v.divl[base + q] = li * v.ncap + k;
			else
				atomicOr(v.err, ERR_LIST_CAPACITY);
		}
	}
}

// One block per replicate: the candidates in the reference's order (agent,
// then neighbour position), attached while both rows are below their
// maximum_number_of_attachments; then the replicate's spring epoch advances.
// Up to kAttachCap candidates the block stages them in shared memory: each
// endpoint's agent, maximum and row length, and the first endpoint of the
// list that names the same agent (found with a per-slot atomicMin), whose
// count slot all its endpoints share; the candidates then settle in waves
// that touch only shared memory apart from the row writes. Longer lists take
// the serial pass over global memory.
constexpr int kAttachCap = 4096;
constexpr int kAttachThreads = 1024;
constexpr int kAttachWaves = 32;	 // parallel waves at most before the remaining candidates go in order
constexpr int kAttachWaveMin = 32;	 // candidates a wave must settle for the next one to run
constexpr int kAttachBatch = 4;		 // candidates a thread stages with their loads issued together
constexpr size_t kAttachSmem =
	(size_t)kAttachCap * (2 * 4 + 2 * 4 + 2 * 4 + 2 * 2 + 2 * 2) + (size_t)kAttachCap * 4 + (size_t)kAttachCap;

// bitonic sort of n <= kAttachCap 64-bit keys in shared memory, ascending;
// every thread of the block calls it
__device__ void block_sort64(long long* a, int n)
{
	if (n <= 1)
		return;
	int m = 1;
	while (m < n)
		m <<= 1;
	for (int i = n + threadIdx.x; i < m; i += blockDim.x)
		a[i] = 0x7fffffffffffffffLL;
	__syncthreads();
	for (int k = 2; k <= m; k <<= 1)
		for (int j = k >> 1; j > 0; j >>= 1)
		{
			for (int i = threadIdx.x; i < m; i += blockDim.x)
			{
				const int l = i ^ j;
				if (l > i)
				{
					const bool up = (i & k) == 0;
					const long long x = a[i], y = a[l];
					if ((x > y) == up)
					{
						a[i] = y;
						a[l] = x;
					}
				}
			}
			__syncthreads();
		}
}

// candidate q (endpoints 2q, 2q+1) against the row lengths kept at each
// agent's first endpoint: attached while both rows are below their maximum
__device__ __forceinline__ void attach_settle(const view& v, const int32_t* agent, int32_t* cnt, const int16_t* mx,
											  const int16_t* rep, int q)
{
	const int ri = rep[2 * q], rj = rep[2 * q + 1];
	const int ni = cnt[ri], nj = cnt[rj];
	if (!(ni < mx[2 * q] && nj < mx[2 * q + 1]))
		return;
	if (ni >= v.scap || nj >= v.scap)
	{
		atomicOr(v.err, ERR_SPRING_CAPACITY);
		return;
	}
	const int i = agent[2 * q], j = agent[2 * q + 1];
	v.springs[(int64_t)i * v.scap + ni] = j;
	v.springs[(int64_t)j * v.scap + nj] = i;
	cnt[ri] = ni + 1;
	cnt[rj] = nj + 1;
}

__global__ void __launch_bounds__(kAttachThreads) k_spring_attach_apply(view v)
{
	grid_wait();
	extern __shared__ int32_t dyn[];
	int32_t* key = dyn;						   // [kAttachCap] candidate codes (agent * ncap + neighbour position)
	int32_t* agent = key + kAttachCap;		   // [2 cap] endpoint agents (slots): 2q = i, 2q+1 = j
	int32_t* cnt = agent + 2 * kAttachCap;	   // [2 cap] row length, kept at each agent's first endpoint
	int32_t* low = cnt + 2 * kAttachCap;	   // [2 cap] per first endpoint: the agent's lowest unsettled code
	int16_t* mx = reinterpret_cast<int16_t*>(low + 2 * kAttachCap); // [2 cap] maximum_number_of_attachments
	int16_t* rep = mx + 2 * kAttachCap;		   // [2 cap] first endpoint naming the same agent
	uint8_t* done = reinterpret_cast<uint8_t*>(rep + 2 * kAttachCap); // [cap] settled
	const int r = blockIdx.x;
	rep_counters& C = v.ctr[r];
	const int base = v.reps[r].base;
	const int nc = min(C.nattach, v.reps[r].cap);
	int32_t* codes = v.divl + base;
	if (nc <= kAttachCap)
	{
		// The candidates stay in the order the draws listed them: the
		// reference's order is that of their codes, and the waves below
		// compare codes. Each thread stages kAttachBatch candidates with their
		// loads issued together (code, then partner, then rows and maxima).
		const int ne = 2 * nc;
		for (int q0 = threadIdx.x; q0 < nc; q0 += kAttachBatch * blockDim.x)
		{
			int code[kAttachBatch], ii[kAttachBatch], jj[kAttachBatch];
#pragma unroll
			for (int k = 0; k < kAttachBatch; k++)
			{
				const int q = q0 + k * blockDim.x;
				code[k] = q < nc ? codes[q] : -1;
			}
#pragma unroll
			for (int k = 0; k < kAttachBatch; k++)
			{
				ii[k] = code[k] >= 0 ? base + code[k] / v.ncap : -1;
				jj[k] = code[k] >= 0 ? v.nidx[(int64_t)ii[k] * v.ncap + code[k] % v.ncap] : -1;
			}
			int ci[kAttachBatch], cj[kAttachBatch], mi[kAttachBatch], mj[kAttachBatch];
#pragma unroll
			for (int k = 0; k < kAttachBatch; k++)
			{
				const bool ok = code[k] >= 0;
				ci[k] = ok ? v.scnt[ii[k]] : 0;
				cj[k] = ok ? v.scnt[jj[k]] : 0;
				mi[k] = ok ? v.maxatt[ii[k]] : 0;
				mj[k] = ok ? v.maxatt[jj[k]] : 0;
			}
#pragma unroll
			for (int k = 0; k < kAttachBatch; k++)
			{
				const int q = q0 + k * blockDim.x;
				if (code[k] < 0)
					continue;
				key[q] = code[k];
				done[q] = 0;
				agent[2 * q] = ii[k];
				agent[2 * q + 1] = jj[k];
				cnt[2 * q] = ci[k];
				cnt[2 * q + 1] = cj[k];
				mx[2 * q] = (int16_t)min(mi[k], 32767);
				mx[2 * q + 1] = (int16_t)min(mj[k], 32767);
			}
		}
		__syncthreads();
		// first endpoint of each agent: atomicMin on a per-slot word (large
		// between uses), read back (a thread's reads issued together), then
		// restored
		for (int e = threadIdx.x; e < ne; e += blockDim.x)
			atomicMin(v.first_end + agent[e], e);
		__syncthreads();
		for (int e0 = threadIdx.x; e0 < ne; e0 += 2 * kAttachBatch * blockDim.x)
		{
			int f[2 * kAttachBatch];
#pragma unroll
			for (int k = 0; k < 2 * kAttachBatch; k++)
			{
				const int e = e0 + k * blockDim.x;
				f[k] = e < ne ? __ldcg(v.first_end + agent[e]) : 0;
			}
#pragma unroll
			for (int k = 0; k < 2 * kAttachBatch; k++)
			{
				const int e = e0 + k * blockDim.x;
				if (e < ne)
					rep[e] = (int16_t)f[k];
			}
		}
		__syncthreads();
		for (int e = threadIdx.x; e < ne; e += blockDim.x)
			v.first_end[agent[e]] = INT32_MAX;
		__syncthreads();
		// Waves: a candidate is ready once every candidate before it in the
		// reference's order (a lower code) that names one of its agents is
		// settled; it then sees the row lengths the serial loop would, and the
		// ready candidates of a wave name distinct agents (each agent's lowest
		// unsettled code), so they settle in parallel. Once a wave settles
		// fewer than kAttachWaveMin candidates (a wave costs about as much as
		// that many serial ones), or after kAttachWaves waves, thread 0 takes
		// the rest in the reference's order.
		__shared__ int s_settled;
		for (int wave = 0; wave < kAttachWaves; wave++)
		{
			for (int e = threadIdx.x; e < ne; e += blockDim.x)
				low[e] = INT32_MAX;
			__syncthreads();
			if (threadIdx.x == 0)
				s_settled = 0;
			int open = 0;
			for (int q = threadIdx.x; q < nc; q += blockDim.x)
				if (!done[q])
				{
					atomicMin(&low[rep[2 * q]], key[q]);
					atomicMin(&low[rep[2 * q + 1]], key[q]);
					open = 1;
				}
			if (!__syncthreads_or(open))
				break;
			int settled = 0;
			for (int q = threadIdx.x; q < nc; q += blockDim.x)
				if (!done[q] && low[rep[2 * q]] == key[q] && low[rep[2 * q + 1]] == key[q])
				{
					attach_settle(v, agent, cnt, mx, rep, q);
					done[q] = 1;
					settled++;
				}
			if (settled)
				atomicAdd(&s_settled, settled);
			__syncthreads();
			if (s_settled < kAttachWaveMin)
				break;
		}
		// the unsettled candidates as (code, index) pairs, sorted by code in
		// the space of low (free now), then settled one after another
		__syncthreads();
		long long* rest = reinterpret_cast<long long*>(low);
		int nrest = 0;
		for (int q0 = 0; q0 < nc; q0 += blockDim.x)
		{
			const int q = q0 + threadIdx.x;
			const int open = q < nc && !done[q];
			int total;
			const int off = block_exclusive_scan(open, total);
			if (open)
				rest[nrest + off] = ((long long)key[q] << 32) | (unsigned)q;
			nrest += total;
		}
		__syncthreads();
		block_sort64(rest, nrest);
		if (threadIdx.x == 0)
			for (int w = 0; w < nrest; w++)
				attach_settle(v, agent, cnt, mx, rep, (int)(rest[w] & 0xffffffff));
		__syncthreads();
		for (int e = threadIdx.x; e < ne; e += blockDim.x)
			if (rep[e] == e)
				v.scnt[agent[e]] = cnt[e];
	}
	else
	{
		block_sort(codes, nc, key); // through global memory: nc > kSortCap
		if (threadIdx.x == 0)
			for (int q = 0; q < nc; q++)
			{
				const int code = codes[q];
				const int i = base + code / v.ncap;
				const int j = v.nidx[(int64_t)i * v.ncap + code % v.ncap];
				const int ni = v.scnt[i], nj = v.scnt[j];
				if (ni < v.maxatt[i] && nj < v.maxatt[j])
				{
					if (ni >= v.scap || nj >= v.scap)
					{
						atomicOr(v.err, ERR_SPRING_CAPACITY);
						continue;
					}
					v.springs[(int64_t)i * v.scap + ni] = j;
					v.springs[(int64_t)j * v.scap + nj] = i;
					v.scnt[i] = ni + 1;
					v.scnt[j] = nj + 1;
				}
			}
	}
	if (threadIdx.x == 0)
	{
		C.nattach = 0;
		C.spring_epoch++;
	}
}

// stand-in for the phenotype models: death with p_death, else division with
// p_divide, from the counter-based draws of (seed, epoch, replicate, index)
__global__ void k_flag_by_draws(view v, double p_divide, double p_death)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, local;
	if (!live(v, s, r, local))
		return;
	const uint64_t ep = v.draw_epoch[r];
	if (ppc_uniform(v.seed, ep, (uint64_t)r, (uint64_t)local, PPC_DRAW_DEATH) < p_death)
		v.flags[s] = PPC_FLAG_TO_REMOVE;
	else if (ppc_uniform(v.seed, ep, (uint64_t)r, (uint64_t)local, PPC_DRAW_DIVIDE) < p_divide)
		v.flags[s] = PPC_FLAG_TO_DIVIDE;
}

// agents of replicate r whose flag equals `flag`, added into *count
__global__ void k_count_flags(view v, int r, int flag, int32_t* count)
{
	grid_wait();
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	const int n = v.ctr[r].count;
	const int hit = i < n && v.flags[v.reps[r].base + i] == flag;
	const int warp_total = __reduce_add_sync(0xffffffffu, hit);
	if ((threadIdx.x & 31) == 0 && warp_total)
		atomicAdd(count, warp_total);
}

__global__ void k_bump_draw_epoch(view v)
{
	grid_wait();
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r < v.nreps)
		v.draw_epoch[r]++;
}

__global__ void k_mark_divide(view v)
{
	grid_wait();
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= v.total_cap)
		return;
	int r, local;
	if (!live(v, s, r, local))
		return;
	if (v.flags[s] == PPC_FLAG_TO_DIVIDE)
	{
		int k = atomicAdd(&v.ctr[r].ndiv, 1);
		if (k < v.reps[r].cap)
			v.divl[v.reps[r].base + k] = local;
		else
			atomicOr(v.err, ERR_LIST_CAPACITY);
	}
}

// Orders the dividing agents (one block per replicate); daughters are
// appended in ascending parent order like the serial reference loop. With
// springs, thread 0 removes each parent from its partners' rows in that order
// (cell::divide, reference: src/cell.cpp:110-114).
__global__ void k_divide_plan(view v, int springs)
{
	grid_wait();
	__shared__ int32_t sh[kSortCap];
	const int r = blockIdx.x;
	rep_counters& C = v.ctr[r];
	const int nd = min(C.ndiv, v.reps[r].cap);
	const int base = v.reps[r].base;
	if (threadIdx.x == 0)
		C.nvisit = C.count;
	if (nd == 0)
		return;
	block_sort(v.divl + base, nd, sh);
	if (threadIdx.x != 0)
		return;
	if (C.count + nd > v.reps[r].cap)
	{
		atomicOr(v.err, ERR_AGENT_CAPACITY);
		C.ndiv = 0;
		return;
	}
	*v.appended = 1; // daughters go past the count: the next k_bin_count takes new slots too
	if (springs)
		for (int k = 0; k < nd; k++)
		{
			const int p = base + v.divl[base + k];
			springs_remove_attached(v, p);
			v.scnt[p] = 0;
		}
}

template <int DIMS>
__global__ void k_divide_apply(view v, int cur)
{
	grid_wait();
	const int r = blockIdx.y;
	rep_counters& C = v.ctr[r];
	const int nd = C.ndiv;
	const int base = v.reps[r].base;
	const int n_pre = C.nvisit;
	const uint64_t ep = v.draw_epoch[r];
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nd; k += gridDim.x * blockDim.x)
	{
		const int lp = v.divl[base + k];
		const int p = base + lp;
		const int c = base + n_pre + k;
		v.flags[p] = PPC_FLAG_NONE;
		*v.params_changed = 1; // the parent's radius and volumes change

		// random direction, projected against the orientation by polarity and
		// scaled by the parent's radius (reference: src/cell.cpp:129-150)
		double w[3] = { 0, 0, 0 };
		ppc_random_walk(DIMS, v.seed, ep, (uint64_t)r, (uint64_t)lp, PPC_DRAW_WALK, w);
		double4 prm = v.prm[p];
		const double4 o = v.orient[p];
		const double pol = v.polarity[p];
		double tmp = 0;
		for (int d = 0; d < DIMS; d++)
			tmp = tmp + w[d] * comp(o, d);
		for (int d = 0; d < DIMS; d++)
			w[d] = (w[d] - tmp * comp(o, d) * pol) * prm.x;

		// volume.divide() and geometry.update() (reference:
		// data_storage_phenotype.cpp:530-550, interactions_solver.cpp:89-96)
		const double vol = v.vol[p] * 0.5;
		const double nvol = v.nvol[p] * 0.5;
		const double four_thirds_pi = 3.141592653589793 * 4.0 / 3.0;
		prm.x = ppc_cbrt(vol / four_thirds_pi);
		const double nrad = ppc_cbrt(nvol / four_thirds_pi);
		const double sarea = 4.0 * 3.141592653589793 * prm.x * prm.x;
		v.vol[p] = vol;
		v.nvol[p] = nvol;
		v.prm[p] = prm;
		v.nrad[p] = nrad;
		v.sarea[p] = sarea;
		// resident phenotype columns (src/cell.cpp:119-125,153,
		// data_storage_phenotype.cpp:530-560): internalized substrates halved
		// when they are computed, damage and attack time cleared, every
		// volume compartment halved
		const ix_columns& x = v.ix;
		if (x.dead)
		{
			if (x.halve_sub)
				for (int q = 0; q < x.S; q++)
					x.isub[(int64_t)p * x.S + q] *= 0.5;
			x.damage[p] = 0;
			x.attack_time[p] = 0;
			double* halved[] = { x.fluid, x.solid, x.cyto, x.cyto_fluid, x.cyto_solid, x.nuc_fluid, x.nuc_solid,
								 x.target_cyto, x.target_nuc };
#pragma unroll
			for (int k = 0; k < 9; k++)
				halved[k][p] *= 0.5;
		}

		// new cell: defaults of a created cell, then copy_from(parent)
		v.prm[c] = prm;
		v.rmad[c] = v.rmad[p];
		v.ec[c] = v.ec[p];
		v.arate[c] = v.arate[p];
		v.drate[c] = v.drate[p];
		v.vol[c] = vol;
		v.nvol[c] = nvol;
		v.nrad[c] = nrad;
		v.sarea[c] = sarea;
		v.polarity[c] = pol;
		for (int q = 0; q < v.ndefs; q++)
			v.aff[(int64_t)c * v.ndefs + q] = v.aff[(int64_t)p * v.ndefs + q];
		v.def[c] = v.def[p];
		v.maxatt[c] = v.maxatt[p];
		v.movable[c] = 1;
		v.flags[c] = PPC_FLAG_NONE;
		v.ids[c] = C.next_id + k;
		v.vel[c] = make_double4(0, 0, 0, 0);
		v.vprev[c] = make_double4(0, 0, 0, 0);
		v.pressure[c] = 0;
		v.scnt[c] = 0;
		v.ncnt[c] = 0;
		// resident columns: the daughter copies the parent's phenotype and
		// keeps the constructor's state (no damage or attack time, one nucleus)
		copy_columns(v, DIMS, c, p);
		if (x.dead)
		{
			x.damage[c] = 0;
			x.attack_time[c] = 0;
			x.nuclei[c] = 1;
		}
		double ow[3] = { 0, 0, 0 };
		ppc_random_walk(DIMS, v.seed, ep, (uint64_t)r, (uint64_t)lp, PPC_DRAW_ORIENTATION, ow);
		v.orient[c] = make_double4(ow[0], ow[1], ow[2], 0.0);

		double4 pp = v.pos[cur][p];
		double4 pc = pp;
		for (int d = 0; d < DIMS; d++)
		{
			set_comp(pc, d, comp(pp, d) + w[d]);
			set_comp(pp, d, comp(pp, d) - w[d] * 0.5);
		}
		v.pos[cur][p] = pp;
		v.pos[cur][c] = pc;
	}
}

__global__ void k_divide_finish(view v)
{
	grid_wait();
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= v.nreps)
		return;
	rep_counters& C = v.ctr[r];
	C.count += C.ndiv;
	C.divisions += C.ndiv;
	C.next_id += C.ndiv;
	C.ndiv = 0;
	v.draw_epoch[r]++;
}

// ---------------------------------------------------------------------------
// host layout <-> device layout
// ---------------------------------------------------------------------------

// host layout (dims doubles per agent) <-> double4 rows, one thread per
// double so that reads of the flat array (device staging or, for pinned host
// buffers, host memory read over the bus) are contiguous across a warp
// `changed`, when given, is set when any value differs from the one it replaces
__global__ void k_unpack_vec(view v, double4* dst, const double* src, int base, int n, int32_t* changed)
{
	grid_wait();
	const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= (int64_t)n * 4)
		return;
	const int i = (int)(e >> 2), d = (int)(e & 3);
	double* row = reinterpret_cast<double*>(dst + base + i);
	const double x = d < v.dims ? src[(int64_t)i * v.dims + d] : 0.0;
	if (changed && __double_as_longlong(row[d]) != __double_as_longlong(x))
		*changed = 1;
	row[d] = x;
}

__global__ void k_pack_vec(view v, double* dst, const double4* src, int base, int n)
{
	grid_wait();
	const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= (int64_t)n * v.dims)
		return;
	const int i = (int)(e / v.dims), d = (int)(e % v.dims);
	dst[e] = reinterpret_cast<const double*>(src + base + i)[d];
}

__global__ void k_unpack_prm(view v, int field, const double* src, int base, int n)
{
	grid_wait();
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	double* p = reinterpret_cast<double*>(v.prm + base + i);
	p[field] = src[i];
}

__global__ void k_pack_prm(view v, int field, double* dst, int base, int n)
{
	grid_wait();
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	dst[i] = reinterpret_cast<const double*>(v.prm + base + i)[field];
}

__global__ void k_neighbors_local(view v, int base, int n, int32_t* counts, int32_t* lists, int cap)
{
	grid_wait();
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const int s = base + i;
	const int c = v.ncnt[s];
	counts[i] = c;
	const int m = min(min(c, v.ncap), cap);
	for (int k = 0; k < m; k++)
		lists[(int64_t)i * cap + k] = v.nidx[(int64_t)s * v.ncap + k] - base;
}

// rows: [n * cap] local indices in host layout; to_device converts to slots
__global__ void k_springs_local(view v, int base, int n, int32_t* rows, int cap, int to_device)
{
	grid_wait();
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const int s = base + i;
	if (to_device)
	{
		const int c = v.scnt[s];
		for (int k = 0; k < c; k++)
			v.springs[(int64_t)s * v.scap + k] = rows[(int64_t)i * cap + k] + base;
	}
	else
	{
		const int c = min(v.scnt[s], cap);
		for (int k = 0; k < c; k++)
			rows[(int64_t)i * cap + k] = v.springs[(int64_t)s * v.scap + k] - base;
	}
}

// ---------------------------------------------------------------------------
// persistent step: one cooperative launch per mechanics step
//
// The grid stays resident for the whole step and walks its phases — the
// fused pass, the compaction plan (folded into the count), the count, the
// scan, the scatter and the fixup of the mesh rebuild — separated by grid
// barriers, instead of six launches. Every phase is the same device code the
// separate kernels run, over a grid-stride loop. A barrier waits at most
// `limit` polls; a block that gives up sets ERR_TIMEOUT and leaves, every
// block checks the flag after each barrier, and a later persistent launch on
// the same state does nothing until the host has read the error.
// ---------------------------------------------------------------------------

constexpr int kPersistThreads = 128;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
	unsigned x;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
	return x;
}

__device__ __forceinline__ int ld_relaxed_i32(const int32_t* p)
{
	int x;
	asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
	return x;
}

// bar[0] arrivals, bar[1] generation (bar[0] is zeroed before every launch)
__device__ bool grid_barrier(const view& v, unsigned* bar, long long limit)
{
	__shared__ int s_ok;
	__syncthreads();
	if (threadIdx.x == 0)
	{
		int ok = 1;
		const unsigned gen = ld_acquire_u32(bar + 1);
		__threadfence();
		if (atomicAdd(bar, 1u) == gridDim.x - 1)
		{
			atomicExch(bar, 0u);
			__threadfence();
			atomicAdd(bar + 1, 1u);
		}
		else
		{
			long long polls = 0;
			while (ld_acquire_u32(bar + 1) == gen)
			{
				if (++polls > limit)
				{
					atomicOr(v.err, ERR_TIMEOUT);
					ok = 0;
					break;
				}
				__nanosleep(64);
			}
		}
		__threadfence();
		if (ok && (ld_relaxed_i32(v.err) & ERR_TIMEOUT))
			ok = 0; // another block gave up: the phases after it are incomplete
		s_ok = ok;
	}
	__syncthreads();
	return s_ok != 0;
}

struct persist_args
{
	unsigned* bar;
	long long limit;
	int32_t opts;	// FUSED_* of the fused pass
	int32_t cap;	// staged pass: staged positions per block (0: global memory)
	int32_t springs; // the compaction replays removals on the spring rows
};

// fused-pass forms of the persistent step
enum : int
{
	PERSIST_FLAT = 0,
	PERSIST_STAGED = 1,
	PERSIST_QUEUE = 2
};

template <int DIMS, bool F32, int FORM>
__global__ void __launch_bounds__(kPersistThreads) k_step_persistent(view v, int cur, persist_args pa)
{
	extern __shared__ __align__(16) unsigned char smem[];
	__shared__ int s_skip;
	if (threadIdx.x == 0)
		s_skip = (ld_relaxed_i32(v.err) & ERR_TIMEOUT) != 0; // an earlier step gave up: wait for the host
	__syncthreads();
	if (s_skip)
		return;
	bump_spring_epochs(v);
	const int nb = gridDim.x;
	const int nxt = cur ^ 1;

	// fused pass: positions from pos[cur] to pos[nxt]
	if (FORM == PERSIST_STAGED)
	{
		const int nvb = (v.total_cap + kPersistThreads - 1) / kPersistThreads;
		for (int vb = blockIdx.x; vb < nvb; vb += nb)
		{
			fused_staged_block<DIMS, F32>(v, cur, pa.cap, pa.opts, vb, reinterpret_cast<float4*>(smem));
			__syncthreads(); // the block's shared rows are rewritten by the next tile
		}
	}
	else if (FORM == PERSIST_QUEUE)
		for (int t0 = blockIdx.x * kPersistThreads; t0 < v.total_cap; t0 += nb * kPersistThreads)
			fused_queue_agent<DIMS, F32>(v, cur, pa.opts, t0 + threadIdx.x,
										 reinterpret_cast<queue_smem*>(smem)->w[threadIdx.x >> 5]);
	else
		for (int t0 = blockIdx.x * kPersistThreads; t0 < v.total_cap; t0 += nb * kPersistThreads)
			fused_flat_agent<DIMS, F32>(v, cur, pa.opts, t0 + threadIdx.x, *reinterpret_cast<flat_smem*>(smem));
	if (!grid_barrier(v, pa.bar, pa.limit))
		return;

	// compaction plan, one replicate per block; its moves are applied by the count
	for (int r = blockIdx.x; r < v.nreps; r += nb)
	{
		compact_plan_rep(v, r, 0, pa.springs, 1, 0, reinterpret_cast<int32_t*>(smem));
		__syncthreads(); // thread 0 finishes the serial plan before the next sort
	}
	if (!grid_barrier(v, pa.bar, pa.limit))
		return;

	// mesh rebuild: count, then the tiles
	if (blockIdx.x == 0 && threadIdx.x == 0)
		*v.bin_active = 1;
	for (int t0 = blockIdx.x * kPersistThreads; t0 < v.total_cap; t0 += nb * kPersistThreads)
		bin_count_body(v, nxt, t0 + threadIdx.x);
	if (!grid_barrier(v, pa.bar, pa.limit))
		return;
	for (int b = blockIdx.x; b < v.ntiles; b += nb)
		bin_order_tile<kPersistThreads>(v, b, *reinterpret_cast<place_smem*>(smem), 1);
	if (!grid_barrier(v, pa.bar, pa.limit))
		return;
	for (int t0 = blockIdx.x * kPersistThreads; t0 < v.total_cap; t0 += nb * kPersistThreads)
		bin_copy_agent(v, nxt, t0 + threadIdx.x, 0, v.spos4, v.sposf, 1);
	bin_finish(v, blockIdx.x * kPersistThreads + threadIdx.x, nb * kPersistThreads);
}

} // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------


template <typename... KArgs, typename... Args>
static void pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args)
{
	cudaLaunchConfig_t cfg {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = smem;
	cfg.stream = st;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	at[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	cudaLaunchKernelEx(&cfg, k, args...);
}

#define PPC_CHECK_LAUNCH()                                                                                             \
	do                                                                                                                 \
	{                                                                                                                  \
		cudaError_t e_ = cudaGetLastError();                                                                           \
		if (e_ != cudaSuccess)                                                                                         \
			return cuda_fail(e_, __func__);                                                                            \
	} while (0)

void flip_sorted_positions(ppc_state* s)
{
	std::swap(s->v.spos4, s->v.spos4_next);
	std::swap(s->v.sposf, s->v.sposf_next);
	s->sbuf ^= 1;
}

// `ready`: record ev_ready after the count, the last kernel of the step
// that changes agent fields (it applies the compaction's moves), so that a
// download can run beside the rest of the rebuild
int launch_bin(ppc_state* s, bool conditional, bool ready, bool produced)
{
	const int b = blocks_for(s->total_cap, kThreads);
	pdl(k_bin_count, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur, conditional ? 1 : 0, produced ? 1 : 0);
	if (ready)
	{
		// Inside a graph capture the record is an external event node on a
		// branch of the transfer stream that forks after the count (the fork
		// adds no node, so the order kernel keeps its programmatic edge from
		// the count); the capture joins the branch back at its end.
		cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
		PPC_CUDA(cudaStreamIsCapturing(s->stream, &cs));
		if (cs == cudaStreamCaptureStatusActive)
		{
			PPC_CUDA(cudaEventRecord(s->ev_fork, s->stream));
			PPC_CUDA(cudaStreamWaitEvent(s->xfer, s->ev_fork, 0));
			PPC_CUDA(cudaEventRecordWithFlags(s->ev_ready, s->xfer, cudaEventRecordExternal));
			s->join_pending = true;
		}
		else
			PPC_CUDA(cudaEventRecord(s->ev_ready, s->stream));
	}
	s->ready_recorded = ready;
	pdl(k_bin_order, s->v.ntiles, kPlaceThreads, 0, PPC_LAUNCH(s), s->v);
	pdl(k_bin_copy, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur, produced ? 1 : 0);
	PPC_CHECK_LAUNCH();
	if (produced)
		flip_sorted_positions(s);
	return PPC_OK;
}

int launch_neighbors(ppc_state* s)
{
	const int b = blocks_for(s->total_cap, kThreads);
	if (s->dims == 1)
		pdl(k_neighbors<1>, b, kThreads, 0, PPC_LAUNCH(s), s->v);
	else if (s->dims == 2)
		pdl(k_neighbors<2>, b, kThreads, 0, PPC_LAUNCH(s), s->v);
	else
		pdl(k_neighbors<3>, b, kThreads, 0, PPC_LAUNCH(s), s->v);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_forces(ppc_state* s)
{
	const int b = blocks_for(s->total_cap, kThreads);
	pdl(k_clear_pressure, b, kThreads, 0, PPC_LAUNCH(s), s->v);
	if (s->dims == 1)
		pdl(k_forces<1>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else if (s->dims == 2)
		pdl(k_forces<2>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else
		pdl(k_forces<3>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_membrane(ppc_state* s)
{
	const int b = blocks_for(s->total_cap, kThreads);
	if (s->dims == 1)
		pdl(k_membrane<1>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else if (s->dims == 2)
		pdl(k_membrane<2>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else
		pdl(k_membrane<3>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_springs(ppc_state* s)
{
	const int b = blocks_for(s->total_cap, kThreads);
	if (s->dims == 1)
		pdl(k_springs<1>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else if (s->dims == 2)
		pdl(k_springs<2>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else
		pdl(k_springs<3>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

// fields other than positions, or slots' agents, change on the device: the
// next rebuild's k_bin_copy rewrites every key-ordered field
int mark_fields_changed(ppc_state* s)
{
	PPC_CUDA(cudaMemsetAsync(s->v.params_changed, 1, sizeof(int32_t), s->stream));
	return PPC_OK;
}

int launch_spring_updates(ppc_state* s)
{
	if (int rc = mark_fields_changed(s)) // spring counts change
		return rc;
	const int b = blocks_for(s->total_cap, kThreads);
	pdl(k_spring_detach, b, kThreads, 0, PPC_LAUNCH(s), s->v);
	pdl(k_spring_compact_rows, b, kThreads, 0, PPC_LAUNCH(s), s->v);
	pdl(k_spring_attach_draws, b, kThreads, 0, PPC_LAUNCH(s), s->v);
	PPC_CUDA(cudaFuncSetAttribute(k_spring_attach_apply, cudaFuncAttributeMaxDynamicSharedMemorySize,
								  (int)kAttachSmem));
	pdl(k_spring_attach_apply, s->nreps, kAttachThreads, kAttachSmem, PPC_LAUNCH(s), s->v);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_positions(ppc_state* s)
{
	const int b = blocks_for(s->total_cap, kThreads);
	if (s->dims == 1)
		pdl(k_positions<1>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else if (s->dims == 2)
		pdl(k_positions<2>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else
		pdl(k_positions<3>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

template <int DIMS>
static void fused_dispatch(ppc_state* s, int b)
{
	const bool walls = s->params.virtual_wall_at_domain_edges != 0;
	const bool springs = s->has_springs && s->params.automated_spring_adhesion != 0;
	const bool vel = s->vel_dirty;
	cudaStream_t st = PPC_LAUNCH(s);
	const int nt = std::min(s->tile_threads, kFusedThreads);
	b = blocks_for(s->total_cap, nt);
	const bool f32 = s->precision == PPC_FP32_FORCE;
#define PPC_FUSED(W, S, V)                                                                                             \
	if (walls == W && springs == S && vel == V)                                                                        \
	{                                                                                                                  \
		if (f32)                                                                                                       \
			pdl(k_fused_f32<DIMS, W, S, V>, b, nt, 0, st, s->v, s->cur);                                                \
		else                                                                                                           \
			pdl(k_fused<DIMS, W, S, V>, b, nt, 0, st, s->v, s->cur);                                                    \
	}
	PPC_FUSED(false, false, false)
	PPC_FUSED(false, false, true)
	PPC_FUSED(false, true, false)
	PPC_FUSED(false, true, true)
	PPC_FUSED(true, false, false)
	PPC_FUSED(true, false, true)
	PPC_FUSED(true, true, false)
	PPC_FUSED(true, true, true)
#undef PPC_FUSED
}

// FUSED_WALLS | FUSED_SPRINGS | FUSED_VEL of the state's next fused pass
static int fused_opts(ppc_state* s)
{
	return (s->params.virtual_wall_at_domain_edges ? FUSED_WALLS : 0)
		   | ((s->has_springs && s->params.automated_spring_adhesion) ? FUSED_SPRINGS : 0)
		   | (s->vel_dirty ? FUSED_VEL : 0) | (s->produce ? FUSED_PRODUCE : 0);
}

// the staged pass's staging capacity (float4 positions) and dynamic shared bytes
static void staged_shape(ppc_state* s, int& cap, size_t& dyn)
{
	const int nt = std::min(s->tile_threads, kStageThreads);
	const int list_bytes = kList * nt * (int)sizeof(int32_t);
	cap = s->staged ? std::max(0, (s->tile_smem - list_bytes) / (int)sizeof(float4)) : 0;
	dyn = (size_t)cap * sizeof(float4) + list_bytes;
}

template <int DIMS>
static int staged_dispatch(ppc_state* s)
{
	const int opts = fused_opts(s);
	const bool f32 = s->precision == PPC_FP32_FORCE;
	cudaStream_t st = PPC_LAUNCH(s);
	const int nt = std::min(s->tile_threads, kStageThreads);
	int cap;
	size_t dyn;
	staged_shape(s, cap, dyn);
	const int b = blocks_for(s->total_cap, nt);
	auto k = f32 ? k_fused_staged<DIMS, true> : k_fused_staged<DIMS, false>;
	if (dyn + kStageStatic > 48 * 1024)
		PPC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
	pdl(k, b, nt, dyn, st, s->v, s->cur, cap, opts);
	return PPC_OK;
}

template <int DIMS>
static int flat_dispatch(ppc_state* s)
{
	const int opts = fused_opts(s);
	const int b = blocks_for(s->total_cap, kFlatThreads);
	cudaStream_t st = PPC_LAUNCH(s);
	const int dyn = (int)sizeof(flat_smem);
	if (s->precision == PPC_FP32_FORCE)
	{
		PPC_CUDA(cudaFuncSetAttribute(k_fused_flat<DIMS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
		pdl(k_fused_flat<DIMS, true>, b, kFlatThreads, dyn, st, s->v, s->cur, opts);
	}
	else
	{
		PPC_CUDA(cudaFuncSetAttribute(k_fused_flat<DIMS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
		pdl(k_fused_flat<DIMS, false>, b, kFlatThreads, dyn, st, s->v, s->cur, opts);
	}
	return PPC_OK;
}

template <int DIMS>
static int queue_dispatch(ppc_state* s)
{
	const int opts = fused_opts(s);
	const int b = blocks_for(s->total_cap, kQueueThreads);
	cudaStream_t st = PPC_LAUNCH(s);
	const int dyn = (int)sizeof(queue_smem);
	if (s->precision == PPC_FP32_FORCE)
	{
		PPC_CUDA(cudaFuncSetAttribute(k_fused_queue<DIMS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
		pdl(k_fused_queue<DIMS, true>, b, kQueueThreads, dyn, st, s->v, s->cur, opts);
	}
	else
	{
		PPC_CUDA(cudaFuncSetAttribute(k_fused_queue<DIMS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
		pdl(k_fused_queue<DIMS, false>, b, kQueueThreads, dyn, st, s->v, s->cur, opts);
	}
	return PPC_OK;
}

template <int DIMS, bool F32, int FORM>
static int persistent_launch(ppc_state* s, size_t dyn, const persist_args& pa)
{
	auto k = k_step_persistent<DIMS, F32, FORM>;
	PPC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
	int per_sm = 0;
	PPC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kPersistThreads, dyn));
	if (per_sm < 1)
		return cuda_fail(cudaErrorInvalidConfiguration, "persistent step: no block fits an SM");
	// every block must be resident at once (the barriers wait for all of them)
	const int64_t want = ((int64_t)s->total_cap + kPersistThreads - 1) / kPersistThreads;
	const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)per_sm * s->sm_count,
																  std::max<int64_t>(want, s->nreps)));
	cudaLaunchConfig_t cfg {};
	cfg.gridDim = dim3(grid);
	cfg.blockDim = dim3(kPersistThreads);
	cfg.dynamicSmemBytes = dyn;
	cfg.stream = s->stream;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeCooperative;
	at[0].val.cooperative = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	PPC_CUDA(cudaLaunchKernelEx(&cfg, k, s->v, s->cur, pa));
	return PPC_OK;
}

// one mechanics step (fused pass, folded compaction, mesh rebuild) as one
// cooperative launch
int launch_step_persistent(ppc_state* s)
{
	s->ready_recorded = false;
	persist_args pa {};
	pa.bar = s->v.barrier;
	pa.limit = s->wait_limit;
	pa.opts = fused_opts(s);
	pa.springs = s->has_springs ? 1 : 0;
	const bool staged = !s->flat && (s->staged || s->coop);
	size_t dyn = s->queue ? sizeof(queue_smem) : sizeof(flat_smem);
	if (staged)
	{
		pa.cap = s->staged ? std::max(0, (s->tile_smem - kList * kPersistThreads * (int)sizeof(int32_t))
											 / (int)sizeof(float4))
						   : 0;
		dyn = (size_t)pa.cap * sizeof(float4) + (size_t)kList * kPersistThreads * sizeof(int32_t);
	}
	dyn = std::max(dyn, (size_t)kSortCap * sizeof(int32_t)); // the compaction plan's sort buffer
	dyn = std::max(dyn, sizeof(place_smem));				  // the rebuild's tiles
	PPC_CUDA(cudaMemsetAsync(s->v.barrier, 0, sizeof(unsigned), s->stream));
	const bool f32 = s->precision == PPC_FP32_FORCE;
	s->launches++;
	int rc;
#define PPC_PERSIST_FORM(D, FORM)                                                                                      \
	rc = f32 ? persistent_launch<D, true, FORM>(s, dyn, pa) : persistent_launch<D, false, FORM>(s, dyn, pa);
#define PPC_PERSIST(D)                                                                                                 \
	if (staged)                                                                                                        \
	{                                                                                                                  \
		PPC_PERSIST_FORM(D, PERSIST_STAGED)                                                                            \
	}                                                                                                                  \
	else if (s->queue)                                                                                                 \
	{                                                                                                                  \
		PPC_PERSIST_FORM(D, PERSIST_QUEUE)                                                                             \
	}                                                                                                                  \
	else                                                                                                               \
	{                                                                                                                  \
		PPC_PERSIST_FORM(D, PERSIST_FLAT)                                                                              \
	}
	if (s->dims == 1)
	{
		PPC_PERSIST(1)
	}
	else if (s->dims == 2)
	{
		PPC_PERSIST(2)
	}
	else
	{
		PPC_PERSIST(3)
	}
#undef PPC_PERSIST
#undef PPC_PERSIST_FORM
	if (rc != PPC_OK)
		return rc;
	s->cur ^= 1;
	s->vel_dirty = false;
	return PPC_OK;
}

int launch_fused(ppc_state* s)
{
	const int b = blocks_for(s->total_cap, kThreads);
	cudaEvent_t ev_end = nullptr;
	if (s->profiling)
	{
		if (s->prof_used + 2 > s->prof_events.size())
		{
			for (int k = 0; k < 256; k++)
			{
				cudaEvent_t e;
				PPC_CUDA(cudaEventCreate(&e));
				s->prof_events.push_back(e);
			}
		}
		PPC_CUDA(cudaEventRecord(s->prof_events[s->prof_used], s->stream));
		ev_end = s->prof_events[s->prof_used + 1];
		s->prof_used += 2;
	}
	if (s->queue)
	{
		int rc = s->dims == 1 ? queue_dispatch<1>(s) : (s->dims == 2 ? queue_dispatch<2>(s) : queue_dispatch<3>(s));
		if (rc != PPC_OK)
			return rc;
	}
	else if (s->flat)
	{
		int rc = s->dims == 1 ? flat_dispatch<1>(s) : (s->dims == 2 ? flat_dispatch<2>(s) : flat_dispatch<3>(s));
		if (rc != PPC_OK)
			return rc;
	}
	else if (s->staged || s->coop)
	{
		int rc = s->dims == 1 ? staged_dispatch<1>(s) : (s->dims == 2 ? staged_dispatch<2>(s) : staged_dispatch<3>(s));
		if (rc != PPC_OK)
			return rc;
	}
	else if (s->dims == 1)
		fused_dispatch<1>(s, b);
	else if (s->dims == 2)
		fused_dispatch<2>(s, b);
	else
		fused_dispatch<3>(s, b);
	PPC_CHECK_LAUNCH();
	if (ev_end)
		PPC_CUDA(cudaEventRecord(ev_end, s->stream));
	s->cur ^= 1;
	s->vel_dirty = false;
	return PPC_OK;
}

int launch_compact(ppc_state* s, bool phenotype_pass, bool fold, bool produced)
{
	const int springs = s->has_springs ? 1 : 0;
	pdl(k_compact_plan, s->nreps, kThreads, 0, PPC_LAUNCH(s), s->v, phenotype_pass ? 1 : 0, springs, fold ? 1 : 0,
		produced ? 1 : 0);
	if (!fold)
	{
		dim3 g(std::max(1, std::min(64, blocks_for(s->total_cap / std::max(1, s->nreps), kThreads))), s->nreps);
		pdl(k_compact_apply, g, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	}
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_mark_remove(ppc_state* s)
{
	const int b = blocks_for(s->total_cap, kThreads);
	if (s->dims == 1)
		pdl(k_mark_remove<1>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else if (s->dims == 2)
		pdl(k_mark_remove<2>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else
		pdl(k_mark_remove<3>, b, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_divide(ppc_state* s)
{
	const int b = blocks_for(s->total_cap, kThreads);
	const int springs = s->has_springs ? 1 : 0;
	pdl(k_mark_divide, b, kThreads, 0, PPC_LAUNCH(s), s->v);
	pdl(k_divide_plan, s->nreps, kThreads, 0, PPC_LAUNCH(s), s->v, springs);
	dim3 g(std::max(1, std::min(64, blocks_for(s->total_cap / std::max(1, s->nreps), kThreads))), s->nreps);
	if (s->dims == 1)
		pdl(k_divide_apply<1>, g, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else if (s->dims == 2)
		pdl(k_divide_apply<2>, g, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	else
		pdl(k_divide_apply<3>, g, kThreads, 0, PPC_LAUNCH(s), s->v, s->cur);
	pdl(k_divide_finish, blocks_for(s->nreps, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_flag_by_draws(ppc_state* s, double p_divide, double p_death)
{
	const int b = blocks_for(s->total_cap, kThreads);
	pdl(k_flag_by_draws, b, kThreads, 0, PPC_LAUNCH(s), s->v, p_divide, p_death);
	pdl(k_bump_draw_epoch, blocks_for(s->nreps, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_count_flags(ppc_state* s, int32_t r, int32_t flag, int32_t* count)
{
	pdl(k_count_flags, blocks_for(s->reps[r].cap, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v, (int)r, (int)flag,
		count);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_unpack_vec(ppc_state* s, double4* dst, const double* src, int32_t r, int32_t n, int32_t* changed)
{
	if (n == 0)
		return PPC_OK;
	pdl(k_unpack_vec, blocks_for(n * 4, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v, dst, src, s->reps[r].base, n,
		changed);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_pack_vec(ppc_state* s, double* dst, const double4* src, int32_t r, int32_t n)
{
	if (n == 0)
		return PPC_OK;
	pdl(k_pack_vec, blocks_for(n * s->dims, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v, dst, src, s->reps[r].base,
		n);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_unpack_prm(ppc_state* s, int field, const double* src, int32_t r, int32_t n)
{
	if (n == 0)
		return PPC_OK;
	pdl(k_unpack_prm, blocks_for(n, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v, field, src, s->reps[r].base, n);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_pack_prm(ppc_state* s, int field, double* dst, int32_t r, int32_t n)
{
	if (n == 0)
		return PPC_OK;
	pdl(k_pack_prm, blocks_for(n, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v, field, dst, s->reps[r].base, n);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_neighbors_local(ppc_state* s, int32_t r, int32_t n, int32_t* counts, int32_t* lists, int32_t cap)
{
	if (n == 0)
		return PPC_OK;
	pdl(k_neighbors_local, blocks_for(n, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v, s->reps[r].base, n, counts,
																			 lists, cap);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

int launch_springs_local(ppc_state* s, int32_t r, int32_t n, int32_t* rows, int32_t cap, int to_device)
{
	if (n == 0)
		return PPC_OK;
	pdl(k_springs_local, blocks_for(n, kThreads), kThreads, 0, PPC_LAUNCH(s), s->v, s->reps[r].base, n, rows, cap,
																		   to_device);
	PPC_CHECK_LAUNCH();
	return PPC_OK;
}

} // namespace ppc
