// ppc_internal.cuh — device state layout and shared helpers of libppc.
//
// Layout in HBM (one allocation per array, all sized to the total slot
// capacity C = sum of replicate capacities):
//   replicate r owns slots [base_r, base_r + cap_r); its live agents are
//   slots base_r .. base_r + count_r - 1 in the reference's index order.
//   pos4[2][C]   double4 {x, y, z, 0}, double-buffered across the fused step
//   vel[C], vprev[C]  double4 {vx, vy, vz, 0}
//   prm[C]       double4 {radius, repulsion, adhesion, BM repulsion}
//   rmad, ec, arate, drate, pressure, vol, nvol, nrad, sarea, polarity [C] double
//   orient[C]    double4
//   aff[C*D], def, maxatt, scnt [C] int32, springs [C*S] int32
//   movable, flags [C] uint8, ids [C] int64, rid [C] int32 (replicate of slot)
// Mechanics mesh bins, rebuilt each step from the previous order (tiles of
// 2^tshift consecutive voxel keys; agents that leave their tile move on
// per-tile chains):
//   vstart[V+1] exclusive prefix of the voxel counts over the key space of
//   all replicates; key[C] (global voxel index of each slot)
//   sorted[C] slots in voxel-key order (descending slot inside a voxel),
//   skey[C] their keys, spos4[C] double4 {x, y, z, rmad*radius} in that order
//   (with sposf, its single-precision twin, double-buffered: a fused pass
//   that does the rebuild's per-agent work writes the next step's positions
//   into spos4_next / sposf_next, and the host swaps the pairs after the
//   rebuild completes them).
// Because the sorted array follows the key order, the voxels x-1..x+1 of one
// stencil row are one contiguous range [vstart[k-1], vstart[k+2]).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ppc.h"

namespace ppc {

constexpr double simple_pressure_coefficient = 36.64504274775163; // reference: position_solver.cpp:13

// device error bits (folded into a status by the host)
enum : int32_t
{
	ERR_NEIGHBOR_CAPACITY = 1,
	ERR_NONFINITE = 2,
	ERR_OUT_OF_MESH = 4,
	ERR_AGENT_CAPACITY = 8,
	ERR_SPRING_CAPACITY = 16,
	ERR_LIST_CAPACITY = 32,
	ERR_TIMEOUT = 64 // a bounded wait of the persistent step gave up
};

struct rep_info
{
	double mins[3], maxs[3], shape[3];
	int32_t grid[3];
	int32_t base, cap;
	int64_t vox_base;
	int64_t voxels;
	int32_t maxs_int[3], mins_int[3];
	float fmargin;	  // bound on the FP32 distance error of positions relative to mins (um)
	double inv_grid[2]; // 1 / grid[0], 1 / grid[1]: voxel coordinates of a key without integer division
};

// per-replicate device counters
struct rep_counters
{
	int32_t count;		 // live agents
	int32_t nvisit;		 // agents visited by the current removal pass
	int32_t nbad;		 // entries in the removal candidate list
	int32_t ndiv;		 // entries in the division list
	int64_t divisions;	 // environment::divisions_count
	int64_t deaths;		 // environment::deaths_count
	int64_t next_id;	 // id of the next created agent
	int32_t nattach;	 // entries in the spring-attachment candidate list
	int32_t pad;
	int64_t spring_epoch; // spring updates so far: epoch of their counter-based draws
};

// Phenotype columns a caller made resident (ppc_upload_interactions,
// ppc_upload_motility): slot-indexed like the mechanics fields, moved by the
// compaction and set by division; null pointers until uploaded.
struct ix_columns
{
	uint8_t* dead;
	double *dead_phago, *damage_rate, *live_phago, *attack, *fusion, *immuno, *frac; // rates: [C], [C*D], [C*S]
	double *damage, *attack_time, *fluid, *solid, *cyto, *cyto_fluid, *cyto_solid, *nuc_fluid, *nuc_solid,
		*fluid_fraction, *c2n, *target_cyto, *target_nuc, *isub; // [C], isub [C*S]
	int32_t* nuclei;
	int32_t S;		   // internalized substrates per agent
	int32_t halve_sub; // division halves the internalized substrates (compute_internalized_substrates)
};

struct mot_columns
{
	uint8_t *motile, *restrict2d, *rule;
	double *persistence, *speed, *bias, *direction, *vector; // direction, vector: [C*dims]
	int32_t* chemo_index;
	double *chemo_dir, *sens; // sens: [C*S]
	int32_t per_agent;
	int32_t S; // chemotactic sensitivities per agent
};

// everything a kernel needs, passed by value
struct view
{
	int32_t dims, ndefs, nreps, total_cap, scap, ncap;
	double dt;
	int32_t walls;
	int32_t auto_springs; // automated_spring_adhesion: every step updates springs
	const rep_info* reps;
	rep_counters* ctr;
	int32_t* err;
	int32_t* cursor;	// number of binned agents (length of `sorted`)
	int32_t nvox;		// voxels of all replicates
	int32_t tshift;		// a rebuild tile is 2^tshift consecutive voxel keys
	int32_t ntiles;		// rebuild tiles

	double4* pos[2];
	double4* vel;
	double4* vprev;
	double4* prm;
	double* rmad;
	double* ec;
	double* arate;
	double* drate;
	double* pressure;
	double* vol;
	double* nvol;
	double* nrad;
	double* sarea;
	double* polarity;
	double4* orient;
	double* aff;
	int32_t* def;
	int32_t* maxatt;
	int32_t* scnt;
	int32_t* springs;
	uint8_t* movable;
	uint8_t* flags;
	int64_t* ids;
	int32_t* rid;

	int32_t* vstart;	// [nvox + 1] start of each voxel's agents in the key order
	int32_t* key;		// [C] voxel key of each slot at the last rebuild
	int32_t* tmp;		// [C] scratch of the rebuild's large tiles (slots grouped by voxel)
	int2* vsc;			// [C] scratch of the rebuild's large tiles (listed agents)
	int2* tprev;		// [ntiles] start and count of each tile's agents in the key order
	int32_t* tdelta;	// [ntiles] agents entering minus leaving each tile at the pending rebuild
	int32_t* sdelta;	// [ntiles / 1024] the same per 1024 tiles
	int32_t* chead;		// [ntiles * 32] heads of the tiles' mover chains (-1: empty)
	int32_t* cnext;		// [C] next slot of a mover chain
	int2* porder;		// [C] entries of the previous order: (slot, key) of agents kept in their tile
	uint8_t* tfresh;	// [C] 1 where the agent at a position of the key order is new to it
	int32_t* params_changed; // fields other than positions, or slots' agents, changed since the last rebuild
	int32_t* copy_full;	// the current rebuild's k_bin_copy copies every field of every agent
	int32_t* recount;	// the compaction removed agents: the rebuild's count recomputes every entry
	int32_t* order_valid; // 1 once a rebuild has set `sorted` (cleared by uploads)
	int32_t* binned;	  // [replicates] live count at the last rebuild (the slots `sorted` lists)
	int32_t* move_src;	  // [C] tail slot whose agent the next k_bin_count moves into this hole, or -1
	int32_t* moves_pending; // a folded compaction left moves for the next k_bin_count
	int32_t* appended;		// agents were appended (division) since the last rebuild
	uint8_t* sdel;		  // [C*S] spring marked for detachment this step
	int32_t* first_end;	  // [C] INT32_MAX between spring attachment passes
	int32_t* pos_changed; // set by an upload whose positions differ from the resident ones
	int32_t* bin_active;  // the current rebuild runs (a conditional one may find nothing changed)
	unsigned* barrier;	  // [2] grid barrier of the persistent step: arrivals, generation
	int32_t* sorted;
	int32_t* skey;
	double4* spos4;
	// the other buffer of the key-ordered positions (double and single
	// precision): a fused pass that makes the rebuild's entries writes each
	// agent's new position there at its current place, and the rebuild after
	// it completes the pair, which then becomes spos4 / sposf
	double4* spos4_next;
	float4* sposf_next;
	double4* sprm4;	// {radius, repulsion, adhesion, bits: def | movable << 32} in sorted order
	double* saff;	// affinity rows in sorted order
	// FP32-force form: key-ordered copies in single precision
	int32_t f32;
	float4* sposf;	// {x - min, y - min, z - min, rmad*radius}
	float4* sprmf;	// {radius, repulsion, adhesion, bits: def | movable << 16 | springs << 24}
	float* safff;	// affinity rows

	int32_t* ncnt;
	int32_t* nidx;

	int32_t* bad;	  // per replicate: removal candidates (local indices), C entries total at base_r
	int32_t* divl;	  // per replicate: division list, same layout
	int32_t* moves;	  // per replicate: (dst, src) pairs of the compaction, 2*C at 2*base_r
	int32_t* nmoves;  // per replicate move counts

	uint64_t seed;
	uint64_t* draw_epoch; // per replicate draw epoch

	ix_columns ix;
	mot_columns mot;
};

struct buffer
{
	void* p = nullptr;
	size_t bytes = 0;
};

// one device block holding a set of resident columns
struct store_block
{
	void* p = nullptr;
	size_t bytes = 0;
};

// a host-layout unpack or a device-to-host copy queued after the copies or
// packs of the same transfer call
struct pending_unpack
{
	double4* dev;
	const double* src;
	int32_t r, n;
	int32_t* changed;
};

struct pending_copy
{
	void* dst;
	const void* src;
	size_t bytes;
};

// one captured block of fused steps and what its kernels were captured with
struct graph_entry
{
	cudaGraphExec_t exec = nullptr;
	int steps = 0, cur = 0;
	int sbuf = 0, sflip = 0; // key-ordered position buffer at the start, and whether the steps flip it
	bool phenotype = false, lead_bin = false, springs = false;
	bool ready = false; // the last step records ev_ready
	double pdiv = 0, pdeath = 0;
	int64_t launches = 0;
};

} // namespace ppc

struct ppc_state
{
	int device = 0;
	int32_t dims = 3, ndefs = 1, nreps = 1, total_cap = 0, scap = 12, ncap = 64;
	ppc_params params {};
	std::vector<ppc_mesh> meshes;
	std::vector<ppc::rep_info> reps;
	int64_t total_voxels = 0;
	int32_t precision = PPC_FP64;
	uint64_t seed = 0;

	cudaStream_t own_stream = nullptr;
	cudaStream_t stream = nullptr;
	// Host transfers beside the device work: the host-to-device copies of an
	// upload of positions run on `xfer` while the stream finishes the last
	// step's mesh rebuild, and a download right after a step runs there once
	// the step's agent fields are final (ev_ready, recorded after the last
	// step's count kernel, the last one that changes them), beside the rest
	// of the rebuild.
	cudaStream_t xfer = nullptr;
	cudaStream_t h2d_stream = nullptr; // the stream an upload's host copies go to (null: `stream`)
	cudaEvent_t ev_ready = nullptr, ev_h2d = nullptr, ev_stage_free = nullptr, ev_fork = nullptr, ev_join = nullptr;
	bool join_pending = false; // a capture forked the transfer stream for ev_ready
	bool ready_pending = false;	 // ev_ready marks the state a download reads...
	int64_t ready_launches = 0;	 // ...while no kernel has been launched since (launch count then)
	bool ready_recorded = false; // the last rebuild enqueued recorded ev_ready

	ppc::view v {};
	std::vector<ppc::buffer> allocations;

	int cur = 0;				  // which pos4 buffer is current
	int sbuf = 0;				  // flips with each swap of v.spos4/sposf and their _next buffers
	bool vel_dirty = false;		  // some movable agent may have a non-zero velocity
	bool has_springs = false;	  // some agent may have springs
	bool rates_nonzero = false;	  // some attachment/detachment rate is non-zero
	bool bins_valid = false;	  // bins match the current positions
	bool bins_cond = false;		  // ...unless an upload changed them: the device decides (pos_changed)
	bool counts_known = false;	  // host_count holds the device counts (no count-changing work since)
	bool zero_copy = false;		  // pinned host rows are read and written by kernels over the bus
	bool lists_stale = false;	  // a fused step ran since the neighbour lists were built
	int64_t launches = 0;
	int max_grid_blocks = 0;
	int sm_count = 148;

	// staging for host <-> device copies
	void* stage = nullptr;
	size_t stage_bytes = 0;
	size_t stage_used = 0; // bytes of the arena taken by the current transfer call
	std::vector<ppc::pending_unpack> pending_unpacks;
	std::vector<ppc::pending_copy> pending_copies;

	// captured CUDA graphs of blocks of fused steps (ppc_api.cu: replay_steps)
	std::vector<ppc::graph_entry> graphs;
	bool use_graphs = true;

	// fused pass launch shape: one thread per agent with its own pair work
	// (default), or warp-cooperative pair work with candidates read from
	// global memory or from the block's ranges staged in shared memory;
	// threads per block; staging bytes per block
	// host copies of the replicate counts as last read (a download's first guess)
	std::vector<int32_t> host_count;
	std::vector<uint64_t> ix_epoch; // cell-cell interaction calls so far, per replicate
	std::vector<uint64_t> mot_epoch; // motility calls so far, per replicate
	void* ix_scratch = nullptr;		// per-call scratch of the interaction and motility passes
	size_t ix_scratch_bytes = 0;
	ppc::store_block ix_store, mot_store; // resident phenotype columns
	struct gradient_field
	{
		void* p = nullptr;
		int32_t S = 0, grid[3] = { 1, 1, 1 };
		double shape[3] = { 1, 1, 1 };
	};
	std::vector<gradient_field> gradients; // per replicate, for the chemotaxis rules
	ppc::rep_counters* pinned_ctr = nullptr; // pinned landing area of the counters
	int32_t* pinned_err = nullptr;			 // pinned landing area of the device error word
	bool staged = false;
	bool coop = false;
	bool flat = false; // per-thread pass with batched candidate fetches (shape -3)
	bool queue = true; // per-thread pass with the warp's candidates shared out (shape -4, the default)
	bool produce = false; // the fused pass being launched makes the rebuild's entries (FUSED_PRODUCE)
	bool persistent = false;		 // mechanics steps as one cooperative launch each (PPC_STEP_PERSISTENT)
	long long wait_limit = 1LL << 25; // polls of a bounded device wait before it gives up
	bool lost = false;				 // a bounded wait gave up: the state needs a fresh upload
	int tile_threads = 128;
	int tile_smem = 32 * 1024;

	// fused-kernel timing (ppc_set_profiling)
	bool profiling = false;
	std::vector<cudaEvent_t> prof_events; // pairs (start, end)
	size_t prof_used = 0;
};

namespace ppc {

void set_error(const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);

#define PPC_CUDA(call)                                                                                                 \
	do                                                                                                                 \
	{                                                                                                                  \
		cudaError_t e_ = (call);                                                                                       \
		if (e_ != cudaSuccess)                                                                                         \
			return ppc::cuda_fail(e_, #call);                                                                          \
	} while (0)

#define PPC_LAUNCH(s) ((s)->launches++, (s)->stream)

inline int blocks_for(int64_t n, int threads)
{
	int64_t b = (n + threads - 1) / threads;
	return (int)(b < 1 ? 1 : b);
}

// ---- kernel entry points (ppc_kernels.cu) ----
int launch_bin(ppc_state* s, bool conditional, bool ready = false, bool produced = false);
// swaps the key-ordered position buffers (spos4, sposf) with their _next pair
void flip_sorted_positions(ppc_state* s);
int launch_neighbors(ppc_state* s);
int launch_forces(ppc_state* s);
int launch_membrane(ppc_state* s);
int launch_springs(ppc_state* s);
int launch_spring_updates(ppc_state* s);
int launch_positions(ppc_state* s);
int launch_fused(ppc_state* s);
int launch_step_persistent(ppc_state* s);
int launch_compact(ppc_state* s, bool phenotype_pass, bool fold = false, bool produced = false);
int launch_mark_remove(ppc_state* s);
int launch_divide(ppc_state* s);
int launch_flag_by_draws(ppc_state* s, double p_divide, double p_death);
int launch_count_flags(ppc_state* s, int32_t r, int32_t flag, int32_t* count);

// packing between host-layout staging buffers and device arrays
int launch_unpack_vec(ppc_state* s, double4* dst, const double* src, int32_t r, int32_t n, int32_t* changed = nullptr);
int launch_pack_vec(ppc_state* s, double* dst, const double4* src, int32_t r, int32_t n);
int launch_unpack_prm(ppc_state* s, int field, const double* src, int32_t r, int32_t n);
int launch_pack_prm(ppc_state* s, int field, double* dst, int32_t r, int32_t n);
int launch_neighbors_local(ppc_state* s, int32_t r, int32_t n, int32_t* counts, int32_t* lists, int32_t cap);
int launch_springs_local(ppc_state* s, int32_t r, int32_t n, int32_t* rows, int32_t cap, int to_device);

// device copies of the ppc_interactions fields of one replicate (local rows)
struct ix_fields
{
	int32_t n, substrates, replicate, base;
	double dt;
	uint64_t epoch;
	const uint8_t* dead;
	const double *dead_phago, *damage_rate, *live_phago, *attack, *fusion, *immuno, *frac;
	double *damage, *attack_time;
	int32_t* nuclei;
	double *fluid, *solid, *cyto, *cyto_fluid, *cyto_solid, *nuc_fluid, *nuc_solid, *fluid_fraction, *c2n, *target_cyto,
		*target_nuc, *isub;
	int32_t* ncand; // [n] candidate neighbours of each agent
	int32_t* cand;	// [n*ncap] their positions in the agent's neighbour list
	int32_t* status; // [2] capacity error found by the candidate pass, count of agents left for the ordered pass
	int32_t* dep;	 // [n] agents whose interactions depend on an earlier agent's
	int32_t* order;	 // [n] the dependent agents still to walk, in index order
};
int launch_interactions(ppc_state* s, const ix_fields& x);
int mark_fields_changed(ppc_state* s);

// device copies of the ppc_motility fields of one replicate (local rows)
struct mot_fields
{
	int32_t n, replicate, base, per_agent, cur;
	double dt;
	uint64_t epoch;
	const uint8_t *motile, *restrict2d, *rule;
	const double *persistence, *speed, *bias;
	double* direction; // [n*dims], written by a direction rule
	double* vector;	   // [n*dims]
	const int32_t* chemo_index;
	const double *chemo_dir, *sens; // sens: [n*S]
	int32_t S;
	// the replicate's gradient field (null without one): [voxels * gS * 3]
	const double* grad;
	int32_t gS, ggrid[3];
	double gshape[3], gmins[3];
};
int launch_motility(ppc_state* s, const mot_fields& m);

} // namespace ppc

// block-wide exclusive scan of one int per thread; returns the block total
__device__ __forceinline__ int block_exclusive_scan(int x, int& total)
{
	__shared__ int warp_sums[32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int incl = x;
	for (int o = 1; o < 32; o <<= 1)
	{
		int y = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o)
			incl += y;
	}
	if (lane == 31)
		warp_sums[warp] = incl;
	__syncthreads();
	const int nwarps = blockDim.x >> 5;
	if (warp == 0)
	{
		int w = lane < nwarps ? warp_sums[lane] : 0;
		for (int o = 1; o < 32; o <<= 1)
		{
			int y = __shfl_up_sync(0xffffffffu, w, o);
			if (lane >= o)
				w += y;
		}
		if (lane < nwarps)
			warp_sums[lane] = w;
	}
	__syncthreads();
	total = warp_sums[nwarps - 1];
	int excl = incl - x + (warp > 0 ? warp_sums[warp - 1] : 0);
	__syncthreads();
	return excl;
}
