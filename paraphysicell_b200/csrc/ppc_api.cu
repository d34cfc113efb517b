// ppc_api.cu — the extern "C" entry points of libppc (include/ppc.h).
//
// Host side of the device state: allocation, host <-> device transfer in the
// reference's cell_data layout, the reference solver entry points, and the
// fused step with CUDA-graph replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ppc_internal.cuh"

namespace ppc {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char* where)
{
	set_error(std::string(where) + ": " + cudaGetErrorString(e));
	return PPC_ERR_CUDA;
}

namespace {

int fail(int rc, const std::string& msg)
{
	set_error(msg);
	return rc;
}

template <typename T>
int alloc(ppc_state* s, T*& p, size_t count, bool zero = true)
{
	size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
	void* q = nullptr;
	PPC_CUDA(cudaMalloc(&q, bytes));
	if (zero) // on the state's stream (non-blocking: the legacy stream would not order with it)
		PPC_CUDA(cudaMemsetAsync(q, 0, bytes, s->stream));
	s->allocations.push_back({ q, bytes });
	p = static_cast<T*>(q);
	return PPC_OK;
}

#define PPC_TRY(x)                                                                                                     \
	do                                                                                                                 \
	{                                                                                                                  \
		int rc_ = (x);                                                                                                 \
		if (rc_ != PPC_OK)                                                                                             \
			return rc_;                                                                                                \
	} while (0)

int launch_pending(ppc_state* s);

// Staging arena of one transfer call: stage_reset at the start of the call,
// then each field takes its own 256-byte aligned region, so the copy and the
// (un)pack kernel of every field are queued without waiting for the previous
// field's. Growing the arena waits for the queued work (which still reads the
// old buffer) before freeing it.
void stage_reset(ppc_state* s)
{
	s->stage_used = 0;
	s->pending_unpacks.clear();
	s->pending_copies.clear();
}

int stage_take(ppc_state* s, size_t bytes, void** out)
{
	size_t off = (s->stage_used + 255) & ~(size_t)255;
	if (off + bytes > s->stage_bytes)
	{
		const size_t want = std::max(off + bytes, 2 * s->stage_bytes);
		if (s->stage)
		{
			// the deferred unpacks and copies still read the old buffer
			PPC_TRY(launch_pending(s));
			PPC_CUDA(cudaStreamSynchronize(s->stream));
			PPC_CUDA(cudaFree(s->stage));
			s->stage = nullptr;
			s->stage_bytes = 0;
		}
		PPC_CUDA(cudaMalloc(&s->stage, want));
		s->stage_bytes = want;
		off = 0;
	}
	*out = static_cast<char*>(s->stage) + off;
	s->stage_used = off + bytes;
	return PPC_OK;
}

int flush_unpacks(ppc_state* s)
{
	for (const auto& u : s->pending_unpacks)
		PPC_TRY(launch_unpack_vec(s, u.dev, u.src, u.r, u.n, u.changed));
	s->pending_unpacks.clear();
	return PPC_OK;
}

int flush_copies(ppc_state* s)
{
	for (const auto& c : s->pending_copies)
		PPC_CUDA(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, s->stream));
	s->pending_copies.clear();
	return PPC_OK;
}

int launch_pending(ppc_state* s)
{
	PPC_TRY(flush_unpacks(s));
	return flush_copies(s);
}

// status of the device error bits `err`; clears the device word when set
int map_errors(ppc_state* s, int32_t err)
{
	if (err == 0)
		return PPC_OK;
	PPC_CUDA(cudaMemsetAsync(s->v.err, 0, sizeof(int32_t), s->stream));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	if (err & ERR_TIMEOUT)
	{
		s->lost = true;
		return fail(PPC_ERR_TIMEOUT, "a grid barrier of the persistent step gave up waiting; the state must be "
									 "uploaded again");
	}
	if (err & ERR_NONFINITE)
		return fail(PPC_ERR_NONFINITE, "an agent position is NaN or infinite");
	if (err & ERR_OUT_OF_MESH)
		return fail(PPC_ERR_OUT_OF_MESH, "an agent lies outside the mechanics mesh");
	if (err & ERR_NEIGHBOR_CAPACITY)
		return fail(PPC_ERR_CAPACITY, "a neighbour list exceeds the neighbour capacity");
	if (err & ERR_AGENT_CAPACITY)
		return fail(PPC_ERR_CAPACITY, "division exceeds the agent capacity of a replicate");
	if (err & ERR_SPRING_CAPACITY)
		return fail(PPC_ERR_ARG, "spring rows are not symmetric");
	if (err & ERR_LIST_CAPACITY)
		return fail(PPC_ERR_CAPACITY, "removal or division list overflow");
	return fail(PPC_ERR_CUDA, "unknown device error");
}

int device_errors(ppc_state* s)
{
	PPC_CUDA(cudaMemcpyAsync(s->pinned_err, s->v.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	return map_errors(s, *s->pinned_err);
}

// the bins no longer match the positions: the next step rebuilds them
void invalidate_bins(ppc_state* s)
{
	s->bins_valid = false;
	s->bins_cond = false;
}

int finish(ppc_state* s)
{
	PPC_CUDA(cudaGetLastError());
	return device_errors(s);
}

bool valid(ppc_state* s, int32_t r) { return s && r >= 0 && r < s->nreps; }

int read_counters(ppc_state* s, std::vector<rep_counters>& c)
{
	c.resize(s->nreps);
	PPC_CUDA(cudaMemcpyAsync(c.data(), s->v.ctr, sizeof(rep_counters) * s->nreps, cudaMemcpyDeviceToHost, s->stream));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	for (int32_t k = 0; k < s->nreps; k++)
		s->host_count[k] = c[k].count;
	s->counts_known = true;
	return PPC_OK;
}

int release_graph(ppc_state* s)
{
	for (auto& e : s->graphs)
		if (e.exec)
			cudaGraphExecDestroy(e.exec);
	s->graphs.clear();
	return PPC_OK;
}

// ---- host <-> device transfer --------------------------------------------------

template <typename T>
int put_scalar(ppc_state* s, T* dev, const T* host, int32_t base, int32_t n, size_t width, bool defaults, T dflt)
{
	T* dst = dev + (size_t)base * width;
	size_t cnt = (size_t)n * width;
	if (host)
	{
		PPC_CUDA(cudaMemcpyAsync(dst, host, cnt * sizeof(T), cudaMemcpyHostToDevice, s->stream));
	}
	else if (defaults && cnt)
	{
		std::vector<T> tmp(cnt, dflt);
		PPC_CUDA(cudaMemcpyAsync(dst, tmp.data(), cnt * sizeof(T), cudaMemcpyHostToDevice, s->stream));
		PPC_CUDA(cudaStreamSynchronize(s->stream));
	}
	return PPC_OK;
}

template <typename T>
int get_scalar(ppc_state* s, T* host, const T* dev, int32_t base, int32_t n, size_t width)
{
	if (host && n)
		PPC_CUDA(cudaMemcpyAsync(host, dev + (size_t)base * width, (size_t)n * width * sizeof(T), cudaMemcpyDeviceToHost,
								 s->stream));
	return PPC_OK;
}

// the device address of a pinned, mapped host buffer (kernels then read or
// write it directly over the bus, without a staging copy), or null
const void* mapped(const void* host)
{
	cudaPointerAttributes at {};
	if (cudaPointerGetAttributes(&at, host) != cudaSuccess)
	{
		cudaGetLastError();
		return nullptr;
	}
	return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
}

// Host rows (dims doubles per agent) into the double4 device rows. Pinned
// host buffers go through the copy engine into the staging arena (or, in the
// zero-copy transfer mode, are read by the unpack kernel over the bus);
// pageable ones are staged by the copy call itself.
int put_vec(ppc_state* s, double4* dev, const double* host, int32_t r, int32_t n, bool defaults,
			int32_t* changed = nullptr)
{
	if (!host && !defaults)
		return PPC_OK;
	if (n == 0)
		return PPC_OK;
	if (host && s->zero_copy)
		if (const void* d = mapped(host))
			return launch_unpack_vec(s, dev, static_cast<const double*>(d), r, n, changed);
	const size_t bytes = (size_t)n * s->dims * sizeof(double);
	void* st = nullptr;
	PPC_TRY(stage_take(s, bytes, &st));
	if (host)
		PPC_CUDA(cudaMemcpyAsync(st, host, bytes, cudaMemcpyHostToDevice, s->h2d_stream ? s->h2d_stream : s->stream));
	else
		PPC_CUDA(cudaMemsetAsync(st, 0, bytes, s->stream));
	// the unpack waits until the call's other copies are queued, so the copy
	// engine moves the fields back to back
	s->pending_unpacks.push_back({ dev, static_cast<const double*>(st), r, n, changed });
	return PPC_OK;
}

int get_vec(ppc_state* s, double* host, const double4* dev, int32_t r, int32_t n)
{
	if (!host || n == 0)
		return PPC_OK;
	if (s->zero_copy)
		if (const void* d = mapped(host))
			return launch_pack_vec(s, static_cast<double*>(const_cast<void*>(d)), dev, r, n);
	const size_t bytes = (size_t)n * s->dims * sizeof(double);
	void* st = nullptr;
	PPC_TRY(stage_take(s, bytes, &st));
	PPC_TRY(launch_pack_vec(s, static_cast<double*>(st), dev, r, n));
	// the copy waits until the call's other packs are queued
	s->pending_copies.push_back({ host, st, bytes });
	return PPC_OK;
}

int put_prm(ppc_state* s, int field, const double* host, int32_t r, int32_t n, bool defaults, double dflt)
{
	if ((!host && !defaults) || n == 0)
		return PPC_OK;
	const size_t bytes = (size_t)n * sizeof(double);
	void* st = nullptr;
	PPC_TRY(stage_take(s, bytes, &st));
	if (host)
		PPC_CUDA(cudaMemcpyAsync(st, host, bytes, cudaMemcpyHostToDevice, s->stream));
	else
	{
		std::vector<double> tmp(n, dflt);
		PPC_CUDA(cudaMemcpyAsync(st, tmp.data(), bytes, cudaMemcpyHostToDevice, s->stream));
		PPC_CUDA(cudaStreamSynchronize(s->stream)); // tmp leaves scope
	}
	PPC_TRY(launch_unpack_prm(s, field, static_cast<const double*>(st), r, n));
	return PPC_OK;
}

int get_prm(ppc_state* s, int field, double* host, int32_t r, int32_t n)
{
	if (!host || n == 0)
		return PPC_OK;
	const size_t bytes = (size_t)n * sizeof(double);
	void* st = nullptr;
	PPC_TRY(stage_take(s, bytes, &st));
	PPC_TRY(launch_pack_prm(s, field, static_cast<double*>(st), r, n));
	PPC_CUDA(cudaMemcpyAsync(host, st, bytes, cudaMemcpyDeviceToHost, s->stream));
	return PPC_OK;
}

// reference defaults (src/data_storage_phenotype.cpp:62-125,194-214, src/cell.cpp:47-61)
constexpr double kRadius = 8.412710547954228, kNuclearRadius = 5.051670902881889, kSurface = 889.3685284131693;

// true when the view carries no field but positions, velocities, previous
// velocities, pressure and orientation
bool only_kinematic(const ppc_agents* a)
{
	const void* others[] = { a->radius, a->cell_cell_repulsion_strength, a->cell_cell_adhesion_strength,
							 a->relative_maximum_adhesion_distance, a->cell_BM_repulsion_strength,
							 a->attachment_elastic_constant, a->attachment_rate, a->detachment_rate,
							 a->maximum_number_of_attachments, a->cell_adhesion_affinities, a->cell_definition_indices,
							 a->is_movable, a->flags, a->agent_ids, a->total_volume, a->nuclear_volume,
							 a->nuclear_radius, a->surface_area, a->polarity, a->spring_counts, a->springs };
	for (const void* p : others)
		if (p)
			return false;
	return true;
}

int transfer_in(ppc_state* s, int32_t r, const ppc_agents* a, bool defaults)
{
	const rep_info& R = s->reps[r];
	const int32_t n = a->count;
	const int32_t base = R.base;
	const int D = s->ndefs;
	view& v = s->v;
	stage_reset(s);
	if (a->cell_definition_indices)
		for (int32_t i = 0; i < n; i++)
			if (a->cell_definition_indices[i] < 0 || a->cell_definition_indices[i] >= D)
				return fail(PPC_ERR_ARG, "cell definition index out of range");

	// an upload of kinematic fields only (positions, velocities, previous
	// velocities, pressure, orientation) keeps the mesh when the positions it
	// brings are bit-identical to the resident ones
	// (pos_changed is zero after every rebuild: its copy kernel clears it)
	const bool kinematic = !defaults && only_kinematic(a);
	s->ready_pending = false;
	bool pinned = true;
	for (const void* p : { (const void*)a->positions, (const void*)a->velocities,
						   (const void*)a->previous_velocities, (const void*)a->simple_pressure,
						   (const void*)a->orientation })
		if (p && !mapped(p))
			pinned = false;
	// page-locked kinematic rows are copied into the staging arena on the
	// transfer stream, beside whatever the stream still runs (the last step's
	// mesh rebuild); the arena is free once the stream has unpacked the
	// previous upload, and the unpacks wait for the copies
	const bool beside = kinematic && pinned && !s->zero_copy && s->xfer;
	if (beside)
	{
		PPC_CUDA(cudaStreamWaitEvent(s->xfer, s->ev_stage_free, 0));
		s->h2d_stream = s->xfer;
	}
	int rc = put_vec(s, v.pos[s->cur], a->positions, r, n, defaults, kinematic ? v.pos_changed : nullptr);
	if (rc == PPC_OK)
		rc = put_vec(s, v.vel, a->velocities, r, n, defaults);
	if (rc == PPC_OK)
		rc = put_vec(s, v.vprev, a->previous_velocities, r, n, defaults);
	if (rc == PPC_OK)
		rc = put_vec(s, v.orient, a->orientation, r, n, defaults);
	s->h2d_stream = nullptr;
	PPC_TRY(rc);
	if (beside)
	{
		PPC_CUDA(cudaEventRecord(s->ev_h2d, s->xfer));
		PPC_CUDA(cudaStreamWaitEvent(s->stream, s->ev_h2d, 0));
	}
	PPC_TRY(flush_unpacks(s));
	PPC_CUDA(cudaEventRecord(s->ev_stage_free, s->stream));
	PPC_TRY(put_prm(s, 0, a->radius, r, n, defaults, kRadius));
	PPC_TRY(put_prm(s, 1, a->cell_cell_repulsion_strength, r, n, defaults, 10.0));
	PPC_TRY(put_prm(s, 2, a->cell_cell_adhesion_strength, r, n, defaults, 0.4));
	PPC_TRY(put_prm(s, 3, a->cell_BM_repulsion_strength, r, n, defaults, 100.0));
	PPC_TRY(put_scalar(s, v.rmad, a->relative_maximum_adhesion_distance, base, n, 1, defaults, 1.25));
	PPC_TRY(put_scalar(s, v.ec, a->attachment_elastic_constant, base, n, 1, defaults, 0.01));
	PPC_TRY(put_scalar(s, v.arate, a->attachment_rate, base, n, 1, defaults, 0.0));
	PPC_TRY(put_scalar(s, v.drate, a->detachment_rate, base, n, 1, defaults, 0.0));
	PPC_TRY(put_scalar(s, v.pressure, a->simple_pressure, base, n, 1, defaults, 0.0));
	PPC_TRY(put_scalar(s, v.vol, a->total_volume, base, n, 1, defaults, 2494.0));
	PPC_TRY(put_scalar(s, v.nvol, a->nuclear_volume, base, n, 1, defaults, 540.0));
	PPC_TRY(put_scalar(s, v.nrad, a->nuclear_radius, base, n, 1, defaults, kNuclearRadius));
	PPC_TRY(put_scalar(s, v.sarea, a->surface_area, base, n, 1, defaults, kSurface));
	PPC_TRY(put_scalar(s, v.polarity, a->polarity, base, n, 1, defaults, 0.0));
	PPC_TRY(put_scalar(s, v.aff, a->cell_adhesion_affinities, base, n, D, defaults, 1.0));
	PPC_TRY(put_scalar<int32_t>(s, v.def, a->cell_definition_indices, base, n, 1, defaults, 0));
	PPC_TRY(put_scalar<int32_t>(s, v.maxatt, a->maximum_number_of_attachments, base, n, 1, defaults, 12));
	PPC_TRY(put_scalar<uint8_t>(s, v.movable, a->is_movable, base, n, 1, defaults, 1));
	PPC_TRY(put_scalar<uint8_t>(s, v.flags, a->flags, base, n, 1, defaults, 0));

	// ids: given or 0..n-1; the next created agent continues after the largest
	if (a->agent_ids || defaults)
	{
		std::vector<int64_t> ids(n);
		int64_t next = 0;
		for (int32_t i = 0; i < n; i++)
		{
			ids[i] = a->agent_ids ? a->agent_ids[i] : i;
			next = std::max<int64_t>(next, ids[i] + 1);
		}
		PPC_TRY(put_scalar<int64_t>(s, v.ids, ids.data(), base, n, 1, false, 0));
		PPC_CUDA(cudaMemcpyAsync(&v.ctr[r].next_id, &next, sizeof next, cudaMemcpyHostToDevice, s->stream));
		PPC_CUDA(cudaStreamSynchronize(s->stream));
	}

	// springs: host rows hold local indices, device rows hold slots
	if (a->spring_counts || defaults)
	{
		bool any = false;
		if (a->spring_counts)
		{
			for (int32_t i = 0; i < n; i++)
			{
				const int32_t c = a->spring_counts[i];
				if (c < 0 || c > s->scap || c > a->spring_capacity)
					return fail(PPC_ERR_CAPACITY, "spring count exceeds the spring capacity");
				for (int32_t k = 0; k < c; k++)
				{
					const int32_t j = a->springs ? a->springs[(size_t)i * a->spring_capacity + k] : -1;
					if (j < 0 || j >= n)
						return fail(PPC_ERR_ARG, "spring partner index out of range");
				}
				any |= c > 0;
			}
		}
		PPC_TRY(put_scalar<int32_t>(s, v.scnt, a->spring_counts, base, n, 1, true, 0));
		if (any)
		{
			const size_t bytes = (size_t)n * a->spring_capacity * sizeof(int32_t);
			void* st = nullptr;
			PPC_TRY(stage_take(s, bytes, &st));
			PPC_CUDA(cudaMemcpyAsync(st, a->springs, bytes, cudaMemcpyHostToDevice, s->stream));
			PPC_TRY(launch_springs_local(s, r, n, static_cast<int32_t*>(st), a->spring_capacity, 1));
			PPC_CUDA(cudaStreamSynchronize(s->stream));
		}
		s->has_springs = s->has_springs || any;
	}

	if (defaults)
	{
		PPC_CUDA(cudaMemsetAsync(v.ncnt + base, 0, sizeof(int32_t) * std::max(n, 1), s->stream));
		int32_t cnt[2] = { n, n };
		PPC_CUDA(cudaMemcpyAsync(&v.ctr[r].count, cnt, sizeof(int32_t) * 2, cudaMemcpyHostToDevice, s->stream));
		s->host_count[r] = n;
	}

	// host flags that pick kernel variants
	if (a->velocities)
	{
		for (int32_t i = 0; i < n * s->dims && !s->vel_dirty; i++)
			s->vel_dirty = a->velocities[i] != 0.0;
	}
	for (const double* rate : { a->attachment_rate, a->detachment_rate })
		if (rate)
			for (int32_t i = 0; i < n && !s->rates_nonzero; i++)
				s->rates_nonzero = rate[i] != 0.0;
	if (kinematic)
	{
		// the slots still hold the same agents; whether the positions moved is
		// known on the device only: the next rebuild runs there if they did
		if (a->positions && s->bins_valid)
		{
			s->bins_valid = false;
			s->bins_cond = true;
		}
		// page-locked rows are copied by the queued DMA, so the call returns
		// at once and the next step queues behind the copies; pageable rows
		// are waited for, so the caller may reuse them on return
		if (!pinned)
			PPC_CUDA(cudaStreamSynchronize(s->stream));
		return PPC_OK;
	}
	invalidate_bins(s);
	// slots were rewritten: the next rebuild counts by slot
	PPC_CUDA(cudaMemsetAsync(v.order_valid, 0, sizeof(int32_t), s->stream));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	return PPC_OK;
}

// queues the copies of the first n agents of replicate r into the host view
// (no synchronisation)
int copy_out(ppc_state* s, int32_t r, ppc_agents* a, int32_t n)
{
	const int32_t base = s->reps[r].base;
	const int D = s->ndefs;
	view& v = s->v;
	PPC_TRY(get_vec(s, a->positions, v.pos[s->cur], r, n));
	PPC_TRY(get_vec(s, a->velocities, v.vel, r, n));
	PPC_TRY(get_vec(s, a->previous_velocities, v.vprev, r, n));
	PPC_TRY(get_vec(s, a->orientation, v.orient, r, n));
	PPC_TRY(flush_copies(s));
	PPC_TRY(get_prm(s, 0, a->radius, r, n));
	PPC_TRY(get_prm(s, 1, a->cell_cell_repulsion_strength, r, n));
	PPC_TRY(get_prm(s, 2, a->cell_cell_adhesion_strength, r, n));
	PPC_TRY(get_prm(s, 3, a->cell_BM_repulsion_strength, r, n));
	PPC_TRY(get_scalar(s, a->relative_maximum_adhesion_distance, v.rmad, base, n, 1));
	PPC_TRY(get_scalar(s, a->attachment_elastic_constant, v.ec, base, n, 1));
	PPC_TRY(get_scalar(s, a->attachment_rate, v.arate, base, n, 1));
	PPC_TRY(get_scalar(s, a->detachment_rate, v.drate, base, n, 1));
	PPC_TRY(get_scalar(s, a->simple_pressure, v.pressure, base, n, 1));
	PPC_TRY(get_scalar(s, a->total_volume, v.vol, base, n, 1));
	PPC_TRY(get_scalar(s, a->nuclear_volume, v.nvol, base, n, 1));
	PPC_TRY(get_scalar(s, a->nuclear_radius, v.nrad, base, n, 1));
	PPC_TRY(get_scalar(s, a->surface_area, v.sarea, base, n, 1));
	PPC_TRY(get_scalar(s, a->polarity, v.polarity, base, n, 1));
	PPC_TRY(get_scalar(s, a->cell_adhesion_affinities, v.aff, base, n, D));
	PPC_TRY(get_scalar(s, a->cell_definition_indices, v.def, base, n, 1));
	PPC_TRY(get_scalar(s, a->maximum_number_of_attachments, v.maxatt, base, n, 1));
	PPC_TRY(get_scalar(s, a->is_movable, v.movable, base, n, 1));
	PPC_TRY(get_scalar(s, a->flags, v.flags, base, n, 1));
	PPC_TRY(get_scalar(s, a->agent_ids, v.ids, base, n, 1));
	return PPC_OK;
}

int transfer_out_on(ppc_state* s, int32_t r, ppc_agents* a, cudaStream_t main, bool beside)
{
	// Copies as many agents as this host last saw in the replicate, together
	// with the counters and the device error word, and synchronises once; if
	// the device count turns out larger (divisions since), the copies are
	// redone with the true count. Rows between the device count and the
	// previous count, within the host capacity, may be overwritten.
	stage_reset(s);
	const int32_t guess = std::max(0, std::min(s->host_count[r], std::min(a->capacity, s->reps[r].cap)));
	PPC_CUDA(cudaMemcpyAsync(s->pinned_ctr, s->v.ctr, sizeof(rep_counters) * (s->nreps + 1), cudaMemcpyDeviceToHost,
							 s->stream)); // the counters and the error word
	PPC_TRY(copy_out(s, r, a, guess));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	if (beside && *s->pinned_err)
	{
		// the rebuild beside the copies may still set error bits: read the
		// word after the main stream
		s->stream = main;
		PPC_TRY(device_errors(s));
	}
	else
		PPC_TRY(map_errors(s, *s->pinned_err));
	for (int32_t k = 0; k < s->nreps; k++)
		s->host_count[k] = s->pinned_ctr[k].count;
	s->counts_known = true;
	const int32_t n = s->host_count[r];
	a->count = n;
	if (n > a->capacity)
		return fail(PPC_ERR_CAPACITY, "host arrays are smaller than the agent count");
	if (n > guess)
		PPC_TRY(copy_out(s, r, a, n));
	const int32_t base = s->reps[r].base;
	view& v = s->v;
	if (a->spring_counts)
	{
		PPC_TRY(get_scalar(s, a->spring_counts, v.scnt, base, n, 1));
		PPC_CUDA(cudaStreamSynchronize(s->stream));
		int32_t mx = 0;
		for (int32_t i = 0; i < n; i++)
			mx = std::max(mx, a->spring_counts[i]);
		if (mx > a->spring_capacity)
			return fail(PPC_ERR_CAPACITY, "host spring rows are shorter than a spring list");
		if (a->springs && n)
		{
			const size_t bytes = (size_t)n * a->spring_capacity * sizeof(int32_t);
			void* st = nullptr;
			PPC_TRY(stage_take(s, bytes, &st));
			PPC_TRY(launch_springs_local(s, r, n, static_cast<int32_t*>(st), a->spring_capacity, 0));
			PPC_CUDA(cudaMemcpyAsync(a->springs, st, bytes, cudaMemcpyDeviceToHost, s->stream));
		}
	}
	if (n > guess || a->spring_counts)
		PPC_CUDA(cudaStreamSynchronize(s->stream));
	return PPC_OK;
}

// A download right after a step (no kernel launched since) runs on the
// transfer stream once the step's agent fields are final (ev_ready), beside
// the rest of the step's mesh rebuild, which changes none of them; any other
// download runs on the stream.
int transfer_out(ppc_state* s, int32_t r, ppc_agents* a)
{
	const bool beside = s->ready_pending && s->launches == s->ready_launches && s->xfer;
	s->ready_pending = false;
	cudaStream_t main = s->stream;
	if (beside)
	{
		PPC_CUDA(cudaStreamWaitEvent(s->xfer, s->ev_ready, 0));
		s->stream = s->xfer;
	}
	const int rc = transfer_out_on(s, r, a, main, beside);
	s->stream = main;
	return rc;
}

int ensure_bins(ppc_state* s)
{
	if (!s->bins_valid)
	{
		PPC_TRY(launch_bin(s, s->bins_cond));
		s->bins_valid = true;
		s->bins_cond = false;
	}
	return PPC_OK;
}

bool stochastic_springs(ppc_state* s) { return s->params.automated_spring_adhesion && s->rates_nonzero; }

// The fused step recomputes neighbours inside its force pass and does not
// store them; the lists the reference would hold after the step are built
// here when a consumer needs them.
int ensure_lists(ppc_state* s)
{
	if (s->lists_stale)
	{
		PPC_TRY(ensure_bins(s));
		PPC_TRY(launch_neighbors(s));
		s->lists_stale = false;
	}
	return PPC_OK;
}

// one fused mechanics step (+ phenotype container update); `last`: the last
// step of a call, whose agent fields a download may read beside its rebuild
int enqueue_step(ppc_state* s, bool phenotype, double p_divide, double p_death, bool last)
{
	if (s->persistent && !phenotype)
		return launch_step_persistent(s);
	// the compaction right before the rebuild leaves its moves to k_bin_count;
	// in a step without the phenotype update the fused passes -3 and -4 also
	// make the count's entries, which hold unless the compaction removes agents
	const bool produce = !phenotype && (s->flat || s->queue);
	s->produce = produce;
	const int rc_fused = launch_fused(s);
	s->produce = false;
	PPC_TRY(rc_fused);
	PPC_TRY(launch_compact(s, false, !phenotype, produce));
	if (phenotype)
	{
		PPC_TRY(launch_flag_by_draws(s, p_divide, p_death));
		PPC_TRY(launch_divide(s));
		PPC_TRY(launch_mark_remove(s));
		PPC_TRY(launch_compact(s, true, true));
	}
	PPC_TRY(launch_bin(s, false, last, produce));
	return PPC_OK;
}

// one step through the separate entry points, for stochastic spring
// attachment: the spring update needs every agent's neighbour list and its
// attachments must be settled before the springs pull, so the step runs the
// reference's sequence (simulator::simulate_mechanics, src/simulator.cpp:173-192)
int enqueue_step_separate(ppc_state* s, bool phenotype, double p_divide, double p_death, bool last)
{
	PPC_TRY(launch_neighbors(s));
	PPC_TRY(launch_forces(s));
	if (s->params.virtual_wall_at_domain_edges)
		PPC_TRY(launch_membrane(s));
	PPC_TRY(launch_spring_updates(s));
	PPC_TRY(launch_springs(s));
	PPC_TRY(launch_positions(s));
	PPC_TRY(launch_mark_remove(s));
	PPC_TRY(launch_compact(s, false, !phenotype));
	if (phenotype)
	{
		PPC_TRY(launch_flag_by_draws(s, p_divide, p_death));
		PPC_TRY(launch_divide(s));
		PPC_TRY(launch_mark_remove(s));
		PPC_TRY(launch_compact(s, true, true));
	}
	PPC_TRY(launch_bin(s, false, last));
	return PPC_OK;
}

constexpr int kGraphSteps = 10; // steps per replay of a long run's graph
constexpr size_t kGraphCache = 8; // captured graphs kept per state

// Replays `k` fused steps from a captured graph, capturing it on first use.
// A graph is keyed by everything its kernels' variants and arguments depend
// on: the step count, the position buffer it starts from, the phenotype
// update and its probabilities, springs, and whether it starts with the
// conditional mesh rebuild an upload of positions leaves for the device.
int replay_steps(ppc_state* s, int k, bool phenotype, double p_divide, double p_death, bool lead_bin)
{
	graph_entry* hit = nullptr;
	for (auto& e : s->graphs)
		if (e.steps == k && e.cur == s->cur && e.sbuf == s->sbuf && e.phenotype == phenotype && e.pdiv == p_divide && e.pdeath == p_death
			&& e.lead_bin == lead_bin && e.springs == s->has_springs)
			hit = &e;
	if (!hit)
	{
		if (s->graphs.size() >= kGraphCache)
			PPC_TRY(release_graph(s));
		graph_entry e {};
		e.steps = k;
		e.cur = s->cur;
		e.sbuf = s->sbuf;
		e.phenotype = phenotype;
		e.pdiv = p_divide;
		e.pdeath = p_death;
		e.lead_bin = lead_bin;
		e.springs = s->has_springs;
		const int cur0 = s->cur;
		const int64_t l0 = s->launches;
		cudaGraph_t g = nullptr;
		PPC_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
		int rc = lead_bin ? launch_bin(s, true) : PPC_OK;
		for (int q = 0; q < k && rc == PPC_OK; q++)
			rc = enqueue_step(s, phenotype, p_divide, p_death, q == k - 1);
		e.ready = s->ready_recorded;
		if (s->join_pending)
		{
			// the transfer stream's branch rejoins before the capture ends
			s->join_pending = false;
			if (cudaEventRecord(s->ev_join, s->xfer) != cudaSuccess
				|| cudaStreamWaitEvent(s->stream, s->ev_join, 0) != cudaSuccess)
				rc = fail(PPC_ERR_CUDA, "joining the transfer stream into the step graph failed");
		}
		cudaError_t ec = cudaStreamEndCapture(s->stream, &g);
		s->cur = cur0;
		e.sflip = s->sbuf ^ e.sbuf;
		if (e.sflip)
			flip_sorted_positions(s);
		if (rc != PPC_OK)
		{
			if (g)
				cudaGraphDestroy(g);
			return rc;
		}
		if (ec != cudaSuccess)
			return cuda_fail(ec, "cudaStreamEndCapture");
		ec = cudaGraphInstantiate(&e.exec, g, 0);
		cudaGraphDestroy(g);
		if (ec != cudaSuccess)
			return cuda_fail(ec, "cudaGraphInstantiate");
		e.launches = s->launches - l0;
		s->launches = l0;
		s->graphs.push_back(e);
		hit = &s->graphs.back();
	}
	PPC_CUDA(cudaGraphLaunch(hit->exec, s->stream));
	s->launches += hit->launches;
	s->ready_recorded = hit->ready;
	s->cur ^= k & 1;
	if (hit->sflip)
		flip_sorted_positions(s);
	s->vel_dirty = false;
	return PPC_OK;
}

// after a call's last step: a download may run beside its rebuild while no
// other kernel is launched
int mark_ready(ppc_state* s)
{
	s->ready_pending = s->ready_recorded;
	s->ready_launches = s->launches;
	return PPC_OK;
}

int run_steps(ppc_state* s, int32_t steps, bool phenotype, double p_divide, double p_death)
{
	if (steps < 0)
		return fail(PPC_ERR_ARG, "negative step count");
	if (s->lost)
		return fail(PPC_ERR_ARG, "a bounded device wait gave up in an earlier step: upload the state again");
	if (steps > 0)
		s->counts_known = false; // compaction and division change the counts
	s->ready_pending = false;
	s->ready_recorded = false;
	const bool graphs = s->use_graphs && !s->profiling;
	// a rebuild the device decides on (after an upload of positions) rides
	// at the head of the first replayed graph
	bool lead_bin = graphs && steps > 0 && !s->bins_valid && s->bins_cond && !s->vel_dirty && !stochastic_springs(s);
	if (!lead_bin)
		PPC_TRY(ensure_bins(s));
	s->bins_valid = true;
	s->bins_cond = false;
	if (stochastic_springs(s))
	{
		// non-zero attachment or detachment rates
		s->has_springs = true;
		for (int32_t k = 0; k < steps; k++)
			PPC_TRY(enqueue_step_separate(s, phenotype, p_divide, p_death, k == steps - 1));
		s->lists_stale = steps > 0 || s->lists_stale;
		return mark_ready(s);
	}
	int32_t done = 0;
	// the first step after an upload may read non-zero velocities
	while (done < steps && s->vel_dirty)
	{
		PPC_TRY(enqueue_step(s, phenotype, p_divide, p_death, done == steps - 1));
		done++;
	}
	if (graphs)
	{
		while (steps - done >= kGraphSteps)
		{
			PPC_TRY(replay_steps(s, kGraphSteps, phenotype, p_divide, p_death, lead_bin));
			lead_bin = false;
			done += kGraphSteps;
		}
		while (done < steps)
		{
			PPC_TRY(replay_steps(s, 1, phenotype, p_divide, p_death, lead_bin));
			lead_bin = false;
			done++;
		}
	}
	while (done < steps)
	{
		PPC_TRY(enqueue_step(s, phenotype, p_divide, p_death, done == steps - 1));
		done++;
	}
	s->lists_stale = steps > 0 || s->lists_stale;
	return mark_ready(s);
}

// grid of a mesh (validated: positive voxel shapes, maxs >= mins); sizes in
// 64-bit arithmetic, saturated at INT32_MAX per axis and in the product, so
// an oversized mesh is rejected by the caller's voxel limit instead of
// wrapping
void mesh_info(const ppc_mesh& m, rep_info& R)
{
	R.voxels = 1;
	for (int d = 0; d < 3; d++)
	{
		R.mins[d] = m.bounding_box_mins[d];
		R.maxs[d] = m.bounding_box_maxs[d];
		R.mins_int[d] = m.bounding_box_mins[d];
		R.maxs_int[d] = m.bounding_box_maxs[d];
		R.shape[d] = m.voxel_shape[d];
		int64_t g = 1;
		if (d < m.dims && m.voxel_shape[d] > 0)
			g = ((int64_t)m.bounding_box_maxs[d] - (int64_t)m.bounding_box_mins[d] + m.voxel_shape[d] - 1)
				/ m.voxel_shape[d];
		g = std::min<int64_t>(std::max<int64_t>(g, 1), INT32_MAX);
		R.grid[d] = (int32_t)g;
		R.voxels = std::min<int64_t>(R.voxels * g, (int64_t)INT32_MAX + 1);
	}
}

} // namespace
} // namespace ppc

using namespace ppc;

extern "C" {

const char* ppc_last_error(void) { return g_last_error.c_str(); }

int ppc_abi_version(void) { return PPC_ABI_VERSION; }

int ppc_create_batch(const ppc_mesh* meshes, const int32_t* capacities, int32_t replicates, const ppc_params* params,
					 ppc_state** out)
{
	if (!meshes || !capacities || !params || !out || replicates < 1)
		return fail(PPC_ERR_ARG, "null argument or no replicates");
	const int dims = meshes[0].dims;
	if (dims < 1 || dims > 3 || params->cell_definitions_count < 1 || params->mechanics_time_step <= 0)
		return fail(PPC_ERR_ARG, "dims must be 1..3, cell definitions >= 1, time step > 0");
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		return fail(PPC_ERR_NO_DEVICE, "no CUDA device");

	auto* s = new ppc_state;
	s->dims = dims;
	s->ndefs = params->cell_definitions_count;
	s->nreps = replicates;
	s->params = *params;
	int64_t vox = 0;
	int64_t cap = 0;
	for (int32_t r = 0; r < replicates; r++)
	{
		if (meshes[r].dims != dims || capacities[r] < 0)
		{
			delete s;
			return fail(PPC_ERR_ARG, "replicates must share dims; capacities must be >= 0");
		}
		for (int d = 0; d < dims; d++)
			if (meshes[r].voxel_shape[d] <= 0 || meshes[r].bounding_box_maxs[d] < meshes[r].bounding_box_mins[d])
			{
				delete s;
				return fail(PPC_ERR_ARG, "invalid mesh");
			}
		rep_info R {};
		mesh_info(meshes[r], R);
		{
			// positions relative to the box minimum reach about the extent; the
			// FP32 filter tolerates 16 float ulps of it per coordinate
			double ext = 1.0;
			for (int d = 0; d < dims; d++)
				ext = std::max(ext, (double)(R.maxs[d] - R.mins[d]) + 2.0 * R.shape[d]);
			int e2 = 0;
			std::frexp(ext, &e2);
			R.fmargin = (float)std::ldexp(16.0, e2 - 24);
		}
		R.inv_grid[0] = 1.0 / R.grid[0];
		R.inv_grid[1] = 1.0 / R.grid[1];
		R.base = (int32_t)cap;
		R.cap = capacities[r];
		R.vox_base = vox;
		vox += R.voxels;
		cap += capacities[r];
		s->reps.push_back(R);
		s->meshes.push_back(meshes[r]);
	}
	if (cap > INT32_MAX / 2 || vox > INT32_MAX)
	{
		delete s;
		return fail(PPC_ERR_CAPACITY, "agent capacity or voxel count exceeds 32-bit indexing");
	}
	s->total_cap = (int32_t)std::max<int64_t>(cap, 1);
	s->total_voxels = vox;

	cudaGetDevice(&s->device);
	cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device);
	int rc = PPC_OK;
	auto try_ = [&](int x) {
		if (rc == PPC_OK)
			rc = x;
	};
	if (cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking) != cudaSuccess)
		rc = fail(PPC_ERR_CUDA, "cudaStreamCreate failed");
	s->stream = s->own_stream;
	if (rc == PPC_OK
		&& (cudaStreamCreateWithFlags(&s->xfer, cudaStreamNonBlocking) != cudaSuccess
			|| cudaEventCreateWithFlags(&s->ev_ready, cudaEventDisableTiming) != cudaSuccess
			|| cudaEventCreateWithFlags(&s->ev_h2d, cudaEventDisableTiming) != cudaSuccess
			|| cudaEventCreateWithFlags(&s->ev_stage_free, cudaEventDisableTiming) != cudaSuccess
			|| cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) != cudaSuccess
			|| cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming) != cudaSuccess))
		rc = fail(PPC_ERR_CUDA, "cudaStreamCreate or cudaEventCreate failed");

	view& v = s->v;
	const size_t C = s->total_cap;
	v.dims = dims;
	v.ndefs = s->ndefs;
	v.nreps = replicates;
	v.total_cap = s->total_cap;
	v.scap = s->scap;
	v.ncap = s->ncap;
	v.dt = params->mechanics_time_step;
	v.walls = params->virtual_wall_at_domain_edges;
	v.auto_springs = params->automated_spring_adhesion != 0;
	rep_info* reps = nullptr;
	try_(alloc(s, reps, replicates));
	v.reps = reps;
	// the error word sits right after the counters, so one copy brings both
	try_(alloc(s, v.ctr, (size_t)replicates + 1));
	if (rc == PPC_OK)
		v.err = reinterpret_cast<int32_t*>(v.ctr + replicates);
	try_(alloc(s, v.cursor, 1));
	v.nvox = (int32_t)vox;
	{
		// rebuild tiles of about 512 agents at full capacity, 64 to 4096 voxels
		const double want = 512.0 * (double)std::max<int64_t>(vox, 1) / (double)std::max<int64_t>(cap, 1);
		const int sh = (int)std::lround(std::log2(std::max(want, 1.0)));
		v.tshift = std::min(12, std::max(6, sh));
	}
	v.ntiles = (int32_t)((vox + (1 << v.tshift) - 1) >> v.tshift);
	try_(alloc(s, v.pos[0], C));
	try_(alloc(s, v.pos[1], C));
	try_(alloc(s, v.vel, C));
	try_(alloc(s, v.vprev, C));
	try_(alloc(s, v.prm, C));
	try_(alloc(s, v.rmad, C));
	try_(alloc(s, v.ec, C));
	try_(alloc(s, v.arate, C));
	try_(alloc(s, v.drate, C));
	try_(alloc(s, v.pressure, C));
	try_(alloc(s, v.vol, C));
	try_(alloc(s, v.nvol, C));
	try_(alloc(s, v.nrad, C));
	try_(alloc(s, v.sarea, C));
	try_(alloc(s, v.polarity, C));
	try_(alloc(s, v.orient, C));
	try_(alloc(s, v.aff, C * s->ndefs));
	try_(alloc(s, v.def, C));
	try_(alloc(s, v.maxatt, C));
	try_(alloc(s, v.scnt, C));
	try_(alloc(s, v.springs, C * s->scap));
	try_(alloc(s, v.movable, C));
	try_(alloc(s, v.flags, C));
	try_(alloc(s, v.ids, C));
	try_(alloc(s, v.rid, C));
	try_(alloc(s, v.vstart, (size_t)vox + 1));
	try_(alloc(s, v.key, C));
	try_(alloc(s, v.tmp, C));
	try_(alloc(s, v.vsc, C));
	try_(alloc(s, v.tprev, (size_t)v.ntiles));
	try_(alloc(s, v.tdelta, (size_t)v.ntiles));
	try_(alloc(s, v.sdelta, ((size_t)v.ntiles + 1023) / 1024));
	try_(alloc(s, v.chead, (size_t)v.ntiles * 32));
	try_(alloc(s, v.cnext, C));
	try_(alloc(s, v.porder, C));
	try_(alloc(s, v.tfresh, C));
	try_(alloc(s, v.params_changed, 1));
	try_(alloc(s, v.copy_full, 1));
	try_(alloc(s, v.recount, 1));
	if (rc == PPC_OK && cudaMemsetAsync(v.chead, 0xff, sizeof(int32_t) * (size_t)v.ntiles * 32, s->stream) != cudaSuccess)
		rc = fail(PPC_ERR_CUDA, "cudaMemset failed");
	try_(alloc(s, v.order_valid, 1));
	try_(alloc(s, v.binned, replicates));
	try_(alloc(s, v.moves_pending, 1));
	try_(alloc(s, v.appended, 1));
	try_(alloc(s, v.move_src, C)); // -1: no pending move into the slot
	try_(alloc(s, v.sdel, C * s->scap));
	try_(alloc(s, v.first_end, C));
	try_(alloc(s, v.pos_changed, 1));
	try_(alloc(s, v.bin_active, 1));
	try_(alloc(s, v.barrier, 2));
	if (rc == PPC_OK && cudaMemsetAsync(v.first_end, 0x7f, sizeof(int32_t) * std::max<size_t>(C, 1), s->stream) != cudaSuccess)
		rc = fail(PPC_ERR_CUDA, "cudaMemset failed");
	if (rc == PPC_OK && cudaMemsetAsync(v.move_src, 0xff, sizeof(int32_t) * std::max<size_t>(C, 1), s->stream) != cudaSuccess)
		rc = fail(PPC_ERR_CUDA, "cudaMemset failed");
	try_(alloc(s, v.sorted, C));
	try_(alloc(s, v.skey, C));
	try_(alloc(s, v.spos4, C));
	try_(alloc(s, v.spos4_next, C));
	try_(alloc(s, v.sprm4, C));
	try_(alloc(s, v.sposf, C));
	try_(alloc(s, v.sposf_next, C));
	try_(alloc(s, v.sprmf, C));
	try_(alloc(s, v.safff, C * s->ndefs));
	try_(alloc(s, v.saff, C * s->ndefs));
	try_(alloc(s, v.ncnt, C));
	try_(alloc(s, v.nidx, C * s->ncap, false));
	try_(alloc(s, v.bad, C));
	try_(alloc(s, v.divl, C));
	try_(alloc(s, v.moves, 2 * C));
	try_(alloc(s, v.nmoves, replicates));
	try_(alloc(s, v.draw_epoch, replicates));
	s->host_count.assign(replicates, 0);
	if (rc == PPC_OK
		&& cudaHostAlloc(reinterpret_cast<void**>(&s->pinned_ctr), sizeof(rep_counters) * (replicates + 1),
						 cudaHostAllocDefault)
			   != cudaSuccess)
		rc = fail(PPC_ERR_CUDA, "cudaHostAlloc failed");
	if (rc == PPC_OK)
		s->pinned_err = reinterpret_cast<int32_t*>(s->pinned_ctr + replicates);
	if (rc == PPC_OK)
	{
		std::vector<int32_t> rid(C, 0);
		for (int32_t r = 0; r < replicates; r++)
			for (int32_t k = 0; k < s->reps[r].cap; k++)
				rid[s->reps[r].base + k] = r;
		if (cudaMemcpyAsync(v.rid, rid.data(), C * sizeof(int32_t), cudaMemcpyHostToDevice, s->stream) != cudaSuccess
			|| cudaMemcpyAsync(reps, s->reps.data(), sizeof(rep_info) * replicates, cudaMemcpyHostToDevice, s->stream)
				   != cudaSuccess
			|| cudaStreamSynchronize(s->stream) != cudaSuccess)
			rc = fail(PPC_ERR_CUDA, "initial copy failed");
	}
	if (rc != PPC_OK)
	{
		ppc_destroy(s);
		return rc;
	}
	*out = s;
	return PPC_OK;
}

int ppc_create(const ppc_mesh* mesh, const ppc_params* params, int32_t agent_capacity, ppc_state** out)
{
	return ppc_create_batch(mesh, &agent_capacity, 1, params, out);
}

int ppc_destroy(ppc_state* s)
{
	if (!s)
		return PPC_OK;
	if (s->stream)
		cudaStreamSynchronize(s->stream);
	if (s->xfer)
		cudaStreamSynchronize(s->xfer);
	release_graph(s);
	for (auto e : s->prof_events)
		cudaEventDestroy(e);
	for (auto e : { s->ev_ready, s->ev_h2d, s->ev_stage_free, s->ev_fork, s->ev_join })
		if (e)
			cudaEventDestroy(e);
	if (s->xfer)
		cudaStreamDestroy(s->xfer);
	for (auto& b : s->allocations)
		cudaFree(b.p);
	if (s->stage)
		cudaFree(s->stage);
	if (s->ix_scratch)
		cudaFree(s->ix_scratch);
	for (auto& b : { s->ix_store.p, s->mot_store.p })
		if (b)
			cudaFree(b);
	for (auto& g : s->gradients)
		if (g.p)
			cudaFree(g.p);
	if (s->pinned_ctr)
		cudaFreeHost(s->pinned_ctr);
	if (s->own_stream)
		cudaStreamDestroy(s->own_stream);
	delete s;
	return PPC_OK;
}

int ppc_set_stream(ppc_state* s, void* stream)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	release_graph(s);
	s->stream = stream ? static_cast<cudaStream_t>(stream) : s->own_stream;
	return PPC_OK;
}

int ppc_set_precision(ppc_state* s, int32_t precision)
{
	if (!s || (precision != PPC_FP64 && precision != PPC_FP32_FORCE))
		return fail(PPC_ERR_ARG, "precision must be PPC_FP64 or PPC_FP32_FORCE");
	if (precision == PPC_FP32_FORCE && s->ndefs > 65535)
		return fail(PPC_ERR_UNSUPPORTED, "the FP32-force form packs definition indices in 16 bits");
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	s->precision = precision;
	s->v.f32 = precision == PPC_FP32_FORCE ? 1 : 0;
	invalidate_bins(s); // the single-precision copies are written by the binning
	PPC_TRY(mark_fields_changed(s));
	release_graph(s);
	return PPC_OK;
}

int ppc_set_random_seed(ppc_state* s, uint64_t seed)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	s->seed = seed;
	s->v.seed = seed;
	release_graph(s);
	return PPC_OK;
}

int ppc_set_launch_shape(ppc_state* s, int32_t tile_edge, int32_t threads, int32_t smem_bytes)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	if (tile_edge < -4 || tile_edge > 0 || threads < 32 || threads > 256 || threads % 32 != 0 || smem_bytes < 0
		|| smem_bytes > 160 * 1024)
		return fail(PPC_ERR_ARG, "tile edge 0, -1, -2, -3 or -4, threads 32..256 (multiple of 32), smem <= 160 KiB");
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	release_graph(s);
	s->flat = tile_edge == -3;
	s->queue = tile_edge == -4;
	s->staged = tile_edge == 0;
	s->coop = tile_edge == 0 || tile_edge == -2;
	s->tile_threads = threads;
	s->tile_smem = smem_bytes;
	return PPC_OK;
}

int ppc_set_step_form(ppc_state* s, int32_t form)
{
	if (!s || (form != PPC_STEP_KERNELS && form != PPC_STEP_PERSISTENT))
		return fail(PPC_ERR_ARG, "form must be PPC_STEP_KERNELS or PPC_STEP_PERSISTENT");
	int coop = 0;
	if (form == PPC_STEP_PERSISTENT
		&& (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, s->device) != cudaSuccess || !coop))
		return fail(PPC_ERR_UNSUPPORTED, "the device has no cooperative launch");
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	release_graph(s);
	s->persistent = form == PPC_STEP_PERSISTENT;
	return PPC_OK;
}

int ppc_set_wait_limit(ppc_state* s, int64_t polls)
{
	if (!s || polls < 1)
		return fail(PPC_ERR_ARG, "the wait limit must be at least one poll");
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	release_graph(s);
	s->wait_limit = polls;
	return PPC_OK;
}

int ppc_set_host_transfer(ppc_state* s, int32_t mode)
{
	if (!s || (mode != PPC_TRANSFER_COPY_ENGINE && mode != PPC_TRANSFER_ZERO_COPY))
		return fail(PPC_ERR_ARG, "mode must be PPC_TRANSFER_COPY_ENGINE or PPC_TRANSFER_ZERO_COPY");
	s->zero_copy = mode == PPC_TRANSFER_ZERO_COPY;
	return PPC_OK;
}

int ppc_set_neighbor_capacity(ppc_state* s, int32_t per_agent)
{
	if (!s || per_agent < 1)
		return fail(PPC_ERR_ARG, "neighbour capacity must be >= 1");
	if (per_agent == s->ncap)
		return PPC_OK;
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	int32_t* p = nullptr;
	size_t bytes = (size_t)s->total_cap * per_agent * sizeof(int32_t);
	PPC_CUDA(cudaMalloc(&p, bytes));
	for (auto& b : s->allocations)
		if (b.p == s->v.nidx)
		{
			cudaFree(b.p);
			b.p = p;
			b.bytes = bytes;
		}
	s->v.nidx = p;
	s->v.ncap = s->ncap = per_agent;
	PPC_CUDA(cudaMemsetAsync(s->v.ncnt, 0, sizeof(int32_t) * s->total_cap, s->stream));
	release_graph(s);
	return PPC_OK;
}

int ppc_upload(ppc_state* s, int32_t r, const ppc_agents* a)
{
	if (!valid(s, r) || !a || a->count < 0)
		return fail(PPC_ERR_ARG, "invalid state, replicate or agents");
	if (a->count > s->reps[r].cap)
		return fail(PPC_ERR_CAPACITY, "agent count exceeds the replicate's capacity");
	// a fresh upload resets the replicate's counters except the event totals
	// and the spring-draw epoch
	std::vector<rep_counters> all;
	PPC_TRY(read_counters(s, all));
	rep_counters c {};
	c.divisions = all[r].divisions;
	c.deaths = all[r].deaths;
	c.spring_epoch = all[r].spring_epoch; // the draw streams continue, as in the reference's generator
	PPC_CUDA(cudaMemcpyAsync(&s->v.ctr[r], &c, sizeof c, cudaMemcpyHostToDevice, s->stream));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	s->lists_stale = false;
	s->lost = false;
	return transfer_in(s, r, a, true);
}

int ppc_upload_fields(ppc_state* s, int32_t r, const ppc_agents* a)
{
	if (!valid(s, r) || !a)
		return fail(PPC_ERR_ARG, "invalid state, replicate or agents");
	// the count is read from the device unless no count-changing work was
	// queued since it was last read (a download, typically)
	if (!s->counts_known)
	{
		std::vector<rep_counters> c;
		PPC_TRY(read_counters(s, c));
	}
	if (a->count != s->host_count[r])
		return fail(PPC_ERR_ARG, "count differs from the device count");
	return transfer_in(s, r, a, false);
}

int ppc_download(ppc_state* s, int32_t r, ppc_agents* a)
{
	if (!valid(s, r) || !a)
		return fail(PPC_ERR_ARG, "invalid state, replicate or agents");
	PPC_CUDA(cudaGetLastError());
	return transfer_out(s, r, a); // reads the device error word with the counters
}

int ppc_get_count(ppc_state* s, int32_t r, int32_t* count)
{
	if (!valid(s, r) || !count)
		return fail(PPC_ERR_ARG, "invalid state or replicate");
	std::vector<rep_counters> c;
	PPC_TRY(read_counters(s, c));
	*count = c[r].count;
	return finish(s);
}

int ppc_get_event_counts(ppc_state* s, int32_t r, int64_t* divisions, int64_t* deaths)
{
	if (!valid(s, r))
		return fail(PPC_ERR_ARG, "invalid state or replicate");
	std::vector<rep_counters> c;
	PPC_TRY(read_counters(s, c));
	if (divisions)
		*divisions = c[r].divisions;
	if (deaths)
		*deaths = c[r].deaths;
	return PPC_OK;
}

int ppc_synchronize(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	return finish(s);
}

void* ppc_host_alloc(size_t bytes)
{
	void* p = nullptr;
	if (cudaHostAlloc(&p, std::max<size_t>(bytes, 1), cudaHostAllocDefault) != cudaSuccess)
		return nullptr;
	return p;
}

void ppc_host_free(void* p)
{
	if (p)
		cudaFreeHost(p);
}

int ppc_update_mechanics_mesh(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	PPC_TRY(launch_bin(s, false));
	s->bins_valid = true;
	s->bins_cond = false;
	return finish(s);
}

int ppc_update_cell_neighbors(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	PPC_TRY(ensure_bins(s));
	PPC_TRY(launch_neighbors(s));
	s->lists_stale = false;
	return finish(s);
}

int ppc_update_cell_forces(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	PPC_TRY(ensure_lists(s));
	PPC_TRY(launch_forces(s));
	return finish(s);
}

int ppc_update_motility(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	return PPC_OK;
}

int ppc_update_basement_membrane_interactions(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	if (!s->params.virtual_wall_at_domain_edges)
		return PPC_OK;
	PPC_TRY(launch_membrane(s));
	return finish(s);
}

int ppc_update_spring_attachments(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	if (!s->params.automated_spring_adhesion)
		return PPC_OK;
	// detachment and attachment draws (they advance the draw epoch even when
	// every rate is zero, as the reference's loop does), then the pull
	PPC_TRY(ensure_lists(s));
	PPC_TRY(launch_spring_updates(s));
	s->has_springs = s->has_springs || s->rates_nonzero;
	if (s->has_springs)
		PPC_TRY(launch_springs(s));
	return finish(s);
}

int ppc_update_positions(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	PPC_TRY(launch_positions(s));
	invalidate_bins(s);
	return finish(s);
}

int ppc_update_cell_container_for_mechanics(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	s->counts_known = false;
	PPC_TRY(ensure_lists(s));
	PPC_TRY(launch_mark_remove(s));
	PPC_TRY(launch_compact(s, false));
	invalidate_bins(s);
	return finish(s);
}

int ppc_update_cell_container_for_phenotype(ppc_state* s)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	s->counts_known = false;
	PPC_TRY(ensure_lists(s));
	PPC_TRY(launch_divide(s));
	PPC_TRY(launch_mark_remove(s));
	PPC_TRY(launch_compact(s, true));
	invalidate_bins(s);
	return finish(s);
}

int ppc_count_flags(ppc_state* s, int32_t r, int32_t flag, int32_t* count)
{
	if (!valid(s, r) || !count)
		return fail(PPC_ERR_ARG, "invalid arguments");
	int32_t* d = reinterpret_cast<int32_t*>(s->v.err) + 1; // the word after the error word, spare
	PPC_CUDA(cudaMemsetAsync(d, 0, sizeof(int32_t), s->stream));
	PPC_TRY(launch_count_flags(s, r, flag, d));
	PPC_CUDA(cudaMemcpyAsync(s->pinned_err + 1, d, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	*count = s->pinned_err[1];
	return finish(s);
}

int ppc_flag_by_draws(ppc_state* s, double p_divide, double p_death)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	PPC_TRY(launch_flag_by_draws(s, p_divide, p_death));
	return finish(s);
}

// device scratch for the phenotype fields of a per-call entry point, kept
// between calls
static int ensure_field_scratch(ppc_state* s, size_t bytes)
{
	if (bytes <= s->ix_scratch_bytes)
		return PPC_OK;
	if (s->ix_scratch)
	{
		PPC_CUDA(cudaStreamSynchronize(s->stream));
		PPC_CUDA(cudaFree(s->ix_scratch));
		s->ix_scratch = nullptr;
		s->ix_scratch_bytes = 0;
	}
	PPC_CUDA(cudaMalloc(&s->ix_scratch, bytes));
	s->ix_scratch_bytes = bytes;
	return PPC_OK;
}

} // extern "C"

namespace ppc {
namespace {

// one resident column: its device base, the caller's host rows, bytes per
// value and values per agent
struct column
{
	void* dev;
	const void* host;
	size_t elem;
	size_t width;
};

// the interaction columns of `x` paired with the host rows of `f`, in one order
std::vector<column> ix_column_list(const ix_columns& x, const ppc_interactions* f, int D)
{
	const size_t S = (size_t)x.S, d = (size_t)D, e = sizeof(double);
	return {
		{ x.dead, f ? f->dead : nullptr, 1, 1 },
		{ x.dead_phago, f ? f->dead_phagocytosis_rate : nullptr, e, 1 },
		{ x.damage_rate, f ? f->damage_rate : nullptr, e, 1 },
		{ x.live_phago, f ? f->live_phagocytosis_rates : nullptr, e, d },
		{ x.attack, f ? f->attack_rates : nullptr, e, d },
		{ x.fusion, f ? f->fusion_rates : nullptr, e, d },
		{ x.immuno, f ? f->immunogenicities : nullptr, e, d },
		{ x.frac, f ? f->fraction_transferred_when_ingested : nullptr, e, S },
		{ x.damage, f ? f->damage : nullptr, e, 1 },
		{ x.attack_time, f ? f->total_attack_time : nullptr, e, 1 },
		{ x.nuclei, f ? f->number_of_nuclei : nullptr, sizeof(int32_t), 1 },
		{ x.fluid, f ? f->fluid : nullptr, e, 1 },
		{ x.solid, f ? f->solid : nullptr, e, 1 },
		{ x.cyto, f ? f->cytoplasmic : nullptr, e, 1 },
		{ x.cyto_fluid, f ? f->cytoplasmic_fluid : nullptr, e, 1 },
		{ x.cyto_solid, f ? f->cytoplasmic_solid : nullptr, e, 1 },
		{ x.nuc_fluid, f ? f->nuclear_fluid : nullptr, e, 1 },
		{ x.nuc_solid, f ? f->nuclear_solid : nullptr, e, 1 },
		{ x.fluid_fraction, f ? f->fluid_fraction : nullptr, e, 1 },
		{ x.c2n, f ? f->cytoplasmic_to_nuclear_ratio : nullptr, e, 1 },
		{ x.target_cyto, f ? f->target_solid_cytoplasmic : nullptr, e, 1 },
		{ x.target_nuc, f ? f->target_solid_nuclear : nullptr, e, 1 },
		{ x.isub, f ? f->internalized_substrates : nullptr, e, S },
	};
}

std::vector<column> mot_column_list(const mot_columns& m, const ppc_motility* f, int dims)
{
	const size_t e = sizeof(double), d = (size_t)dims;
	return {
		{ m.motile, f ? f->is_motile : nullptr, 1, 1 },
		{ m.restrict2d, f ? f->restrict_to_2d : nullptr, 1, 1 },
		{ m.persistence, f ? f->persistence_time : nullptr, e, 1 },
		{ m.speed, f ? f->migration_speed : nullptr, e, 1 },
		{ m.bias, f ? f->migration_bias : nullptr, e, 1 },
		{ m.direction, f ? f->migration_bias_direction : nullptr, e, d },
		{ m.vector, f ? f->motility_vector : nullptr, e, d },
		{ m.rule, f ? f->direction_rule : nullptr, 1, 1 },
		{ m.chemo_index, f ? f->chemotaxis_index : nullptr, sizeof(int32_t), 1 },
		{ m.chemo_dir, f ? f->chemotaxis_direction : nullptr, e, 1 },
		{ m.sens, f ? f->chemotactic_sensitivities : nullptr, e, (size_t)m.S },
	};
}

// carves the columns out of one zeroed block of C rows; the view changes, so
// captured step graphs are released
int alloc_columns(ppc_state* s, store_block& b, std::vector<std::pair<void**, size_t>> cols)
{
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	PPC_TRY(release_graph(s));
	if (b.p)
	{
		PPC_CUDA(cudaFree(b.p));
		b.p = nullptr;
	}
	size_t total = 0;
	for (auto& c : cols)
		total += (c.second + 255) & ~(size_t)255;
	PPC_CUDA(cudaMalloc(&b.p, std::max<size_t>(total, 1)));
	PPC_CUDA(cudaMemsetAsync(b.p, 0, std::max<size_t>(total, 1), s->stream));
	b.bytes = total;
	char* q = static_cast<char*>(b.p);
	for (auto& c : cols)
	{
		*c.first = q;
		q += (c.second + 255) & ~(size_t)255;
	}
	return PPC_OK;
}

int ensure_ix_store(ppc_state* s, int32_t S)
{
	if (s->ix_store.p && s->v.ix.S == S)
		return PPC_OK;
	const size_t C = s->total_cap, D = s->ndefs, e = sizeof(double);
	ix_columns& x = s->v.ix;
	const int32_t halve = x.halve_sub;
	x = ix_columns {};
	x.S = S;
	x.halve_sub = halve;
	std::vector<std::pair<void**, size_t>> cols = {
		{ (void**)&x.dead, C }, { (void**)&x.nuclei, C * 4 }, { (void**)&x.dead_phago, C * e },
		{ (void**)&x.damage_rate, C * e }, { (void**)&x.live_phago, C * D * e }, { (void**)&x.attack, C * D * e },
		{ (void**)&x.fusion, C * D * e }, { (void**)&x.immuno, C * D * e }, { (void**)&x.frac, C * S * e },
		{ (void**)&x.damage, C * e }, { (void**)&x.attack_time, C * e }, { (void**)&x.fluid, C * e },
		{ (void**)&x.solid, C * e }, { (void**)&x.cyto, C * e }, { (void**)&x.cyto_fluid, C * e },
		{ (void**)&x.cyto_solid, C * e }, { (void**)&x.nuc_fluid, C * e }, { (void**)&x.nuc_solid, C * e },
		{ (void**)&x.fluid_fraction, C * e }, { (void**)&x.c2n, C * e }, { (void**)&x.target_cyto, C * e },
		{ (void**)&x.target_nuc, C * e }, { (void**)&x.isub, C * S * e },
	};
	return alloc_columns(s, s->ix_store, cols);
}

int ensure_mot_store(ppc_state* s, int32_t S)
{
	if (s->mot_store.p && s->v.mot.S == S)
		return PPC_OK;
	const size_t C = s->total_cap, d = s->dims, e = sizeof(double);
	mot_columns& m = s->v.mot;
	const int32_t per_agent = m.per_agent;
	m = mot_columns {};
	m.per_agent = per_agent;
	m.S = S;
	std::vector<std::pair<void**, size_t>> cols = {
		{ (void**)&m.motile, C }, { (void**)&m.restrict2d, C }, { (void**)&m.rule, C },
		{ (void**)&m.persistence, C * e }, { (void**)&m.speed, C * e }, { (void**)&m.bias, C * e },
		{ (void**)&m.direction, C * d * e }, { (void**)&m.vector, C * d * e }, { (void**)&m.chemo_index, C * 4 },
		{ (void**)&m.chemo_dir, C * e }, { (void**)&m.sens, C * (size_t)S * e },
	};
	return alloc_columns(s, s->mot_store, cols);
}

// rows [base, base + n) of the columns from (to_device) or to the host rows
int move_columns(ppc_state* s, const std::vector<column>& cols, int32_t base, int32_t n, bool to_device)
{
	for (const auto& c : cols)
	{
		if (!c.host || c.width == 0 || n == 0)
			continue;
		char* dev = static_cast<char*>(c.dev) + (size_t)base * c.width * c.elem;
		const size_t bytes = (size_t)n * c.width * c.elem;
		if (to_device)
			PPC_CUDA(cudaMemcpyAsync(dev, c.host, bytes, cudaMemcpyHostToDevice, s->stream));
		else
			PPC_CUDA(cudaMemcpyAsync(const_cast<void*>(c.host), dev, bytes, cudaMemcpyDeviceToHost, s->stream));
	}
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	return PPC_OK;
}

int check_ix_fields(const ppc_interactions* f)
{
	const void* all[] = { f->dead, f->dead_phagocytosis_rate, f->damage_rate, f->live_phagocytosis_rates,
						  f->attack_rates, f->fusion_rates, f->immunogenicities, f->damage, f->total_attack_time,
						  f->number_of_nuclei, f->fluid, f->solid, f->cytoplasmic, f->cytoplasmic_fluid,
						  f->cytoplasmic_solid, f->nuclear_fluid, f->nuclear_solid, f->fluid_fraction,
						  f->cytoplasmic_to_nuclear_ratio, f->target_solid_cytoplasmic, f->target_solid_nuclear };
	for (const void* p : all)
		if (!p)
			return fail(PPC_ERR_ARG, "a ppc_interactions field is NULL");
	if (f->substrates > 0 && (!f->internalized_substrates || !f->fraction_transferred_when_ingested))
		return fail(PPC_ERR_ARG, "a ppc_interactions substrate field is NULL");
	return PPC_OK;
}

int check_mot_fields(const ppc_motility* f)
{
	if (!f->is_motile || !f->restrict_to_2d || !f->persistence_time || !f->migration_speed || !f->migration_bias
		|| !f->migration_bias_direction || !f->motility_vector)
		return fail(PPC_ERR_ARG, "a ppc_motility field is NULL");
	if (f->substrates < 0)
		return fail(PPC_ERR_ARG, "negative substrate count");
	if (f->direction_rule
		&& (!f->chemotaxis_index || !f->chemotaxis_direction || (f->substrates > 0 && !f->chemotactic_sensitivities)))
		return fail(PPC_ERR_ARG, "a direction-rule field of ppc_motility is NULL");
	return PPC_OK;
}

// the replicate's live count, read from the device unless already known
int live_count(ppc_state* s, int32_t r, int32_t& n)
{
	if (!s->counts_known)
	{
		std::vector<rep_counters> c;
		PPC_TRY(read_counters(s, c));
	}
	n = s->host_count[r];
	return PPC_OK;
}

} // namespace
} // namespace ppc

extern "C" {

int ppc_upload_interactions(ppc_state* s, int32_t r, const ppc_interactions* f, int32_t compute_internalized_substrates)
{
	if (!valid(s, r) || !f || f->substrates < 0)
		return fail(PPC_ERR_ARG, "invalid arguments");
	int32_t n = 0;
	PPC_TRY(live_count(s, r, n));
	if (f->count != n)
		return fail(PPC_ERR_ARG, "fields.count differs from the replicate's agent count");
	PPC_TRY(check_ix_fields(f));
	if (s->ix_store.p && f->substrates != s->v.ix.S)
		return fail(PPC_ERR_ARG, "substrates differ from the resident interaction fields'");
	PPC_TRY(ensure_ix_store(s, f->substrates));
	if (s->v.ix.halve_sub != (compute_internalized_substrates != 0))
	{
		PPC_CUDA(cudaStreamSynchronize(s->stream));
		PPC_TRY(release_graph(s));
		s->v.ix.halve_sub = compute_internalized_substrates != 0;
	}
	return move_columns(s, ix_column_list(s->v.ix, f, s->ndefs), s->reps[r].base, n, true);
}

int ppc_download_interactions(ppc_state* s, int32_t r, ppc_interactions* f)
{
	if (!valid(s, r) || !f)
		return fail(PPC_ERR_ARG, "invalid arguments");
	if (!s->ix_store.p || f->substrates != s->v.ix.S)
		return fail(PPC_ERR_ARG, "no resident interaction fields with these substrates");
	PPC_CUDA(cudaGetLastError());
	std::vector<rep_counters> c;
	PPC_TRY(read_counters(s, c));
	const int32_t n = c[r].count;
	f->count = n;
	PPC_TRY(check_ix_fields(f));
	return move_columns(s, ix_column_list(s->v.ix, f, s->ndefs), s->reps[r].base, n, false);
}

int ppc_upload_motility(ppc_state* s, int32_t r, const ppc_motility* f)
{
	if (!valid(s, r) || !f)
		return fail(PPC_ERR_ARG, "invalid arguments");
	int32_t n = 0;
	PPC_TRY(live_count(s, r, n));
	if (f->count != n)
		return fail(PPC_ERR_ARG, "fields.count differs from the replicate's agent count");
	PPC_TRY(check_mot_fields(f));
	const int32_t S = f->direction_rule ? f->substrates : (s->mot_store.p ? s->v.mot.S : 0);
	PPC_TRY(ensure_mot_store(s, S));
	if (s->v.mot.per_agent != (f->restrict_per_agent != 0))
	{
		PPC_CUDA(cudaStreamSynchronize(s->stream));
		PPC_TRY(release_graph(s));
		s->v.mot.per_agent = f->restrict_per_agent != 0;
	}
	if (!f->direction_rule && n > 0) // no rules: every agent keeps the caller's direction
		PPC_CUDA(cudaMemsetAsync(s->v.mot.rule + s->reps[r].base, PPC_DIRECTION_NONE, (size_t)n, s->stream));
	return move_columns(s, mot_column_list(s->v.mot, f, s->dims), s->reps[r].base, n, true);
}

int ppc_download_motility(ppc_state* s, int32_t r, ppc_motility* f)
{
	if (!valid(s, r) || !f)
		return fail(PPC_ERR_ARG, "invalid arguments");
	if (!s->mot_store.p)
		return fail(PPC_ERR_ARG, "no resident motility fields");
	PPC_CUDA(cudaGetLastError());
	std::vector<rep_counters> c;
	PPC_TRY(read_counters(s, c));
	const int32_t n = c[r].count;
	f->count = n;
	PPC_TRY(check_mot_fields(f));
	return move_columns(s, mot_column_list(s->v.mot, f, s->dims), s->reps[r].base, n, false);
}

int ppc_update_motility_fields(ppc_state* s, int32_t r, ppc_motility* f)
{
	if (!valid(s, r))
		return fail(PPC_ERR_ARG, "invalid arguments");
	if (f)
		PPC_TRY(ppc_upload_motility(s, r, f)); // fields travel with the call
	else if (!s->mot_store.p)
		return fail(PPC_ERR_ARG, "no resident motility fields: upload them or pass fields");
	int32_t n = 0;
	PPC_TRY(live_count(s, r, n));
	if ((int32_t)s->mot_epoch.size() < s->nreps)
		s->mot_epoch.resize(s->nreps, 0);
	const uint64_t epoch = s->mot_epoch[r]++;
	if (n > 0)
	{
		const int32_t base = s->reps[r].base;
		const mot_columns& mc = s->v.mot;
		const size_t d = (size_t)s->dims;
		mot_fields m {};
		m.n = n;
		m.replicate = r;
		m.base = base;
		m.dt = s->params.mechanics_time_step;
		m.per_agent = mc.per_agent;
		m.cur = s->cur;
		m.epoch = epoch;
		m.motile = mc.motile + base;
		m.restrict2d = mc.restrict2d + base;
		m.rule = mc.rule + base;
		m.persistence = mc.persistence + base;
		m.speed = mc.speed + base;
		m.bias = mc.bias + base;
		m.direction = mc.direction + (size_t)base * d;
		m.vector = mc.vector + (size_t)base * d;
		m.chemo_index = mc.chemo_index + base;
		m.chemo_dir = mc.chemo_dir + base;
		m.S = mc.S;
		m.sens = mc.sens + (size_t)base * mc.S;
		if ((int32_t)s->gradients.size() > r && s->gradients[r].p)
		{
			const auto& g = s->gradients[r];
			m.grad = static_cast<const double*>(g.p);
			m.gS = g.S;
			for (int q = 0; q < 3; q++)
			{
				m.ggrid[q] = g.grid[q];
				m.gshape[q] = g.shape[q];
				m.gmins[q] = s->reps[r].mins[q];
			}
		}
		PPC_TRY(launch_motility(s, m));
		s->vel_dirty = true; // the next fused step reads the velocities
	}
	if (f)
		PPC_TRY(move_columns(s,
							 { { s->v.mot.vector, f->motility_vector, sizeof(double), (size_t)s->dims },
							   { s->v.mot.direction, f->migration_bias_direction, sizeof(double), (size_t)s->dims } },
							 s->reps[r].base, n, false));
	return finish(s);
}

int ppc_upload_gradients(ppc_state* s, int32_t r, const ppc_gradient_field* g)
{
	if (!valid(s, r) || !g || g->substrates < 0 || (g->substrates > 0 && !g->gradients))
		return fail(PPC_ERR_ARG, "invalid gradient field");
	ppc_state::gradient_field f;
	f.S = g->substrates;
	int64_t voxels = 1;
	const ppc_mesh& m = s->meshes[r];
	for (int d = 0; d < 3; d++)
	{
		int64_t n = 1;
		if (d < m.dims)
		{
			if (g->voxel_shape[d] <= 0)
				return fail(PPC_ERR_ARG, "diffusion voxel edges must be positive");
			n = ((int64_t)m.bounding_box_maxs[d] - m.bounding_box_mins[d] + g->voxel_shape[d] - 1) / g->voxel_shape[d];
			f.shape[d] = g->voxel_shape[d];
		}
		f.grid[d] = (int32_t)std::max<int64_t>(1, std::min<int64_t>(n, INT32_MAX));
		voxels *= f.grid[d];
		if (voxels > ((int64_t)1 << 31))
			return fail(PPC_ERR_CAPACITY, "the diffusion mesh has too many voxels");
	}
	if ((int32_t)s->gradients.size() < s->nreps)
		s->gradients.resize(s->nreps);
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	if (s->gradients[r].p)
		PPC_CUDA(cudaFree(s->gradients[r].p));
	s->gradients[r] = ppc_state::gradient_field {};
	const size_t bytes = (size_t)voxels * f.S * 3 * sizeof(double);
	if (bytes)
	{
		PPC_CUDA(cudaMalloc(&f.p, bytes));
		PPC_CUDA(cudaMemcpyAsync(f.p, g->gradients, bytes, cudaMemcpyHostToDevice, s->stream));
		PPC_CUDA(cudaStreamSynchronize(s->stream));
	}
	s->gradients[r] = f;
	return PPC_OK;
}

int ppc_update_cell_cell_interactions(ppc_state* s, int32_t r, ppc_interactions* f)
{
	if (!valid(s, r) || (f && f->substrates < 0))
		return fail(PPC_ERR_ARG, "invalid arguments");
	if (f)
	{
		// fields travel with the call: resident for its duration
		if (s->ix_store.p && f->substrates != s->v.ix.S)
			PPC_TRY(ensure_ix_store(s, f->substrates));
		PPC_TRY(ppc_upload_interactions(s, r, f, s->v.ix.halve_sub));
	}
	else if (!s->ix_store.p)
		return fail(PPC_ERR_ARG, "no resident interaction fields: upload them or pass fields");
	int32_t n = 0;
	PPC_TRY(live_count(s, r, n));
	if ((int32_t)s->ix_epoch.size() < s->nreps)
		s->ix_epoch.resize(s->nreps, 0);
	const uint64_t epoch = s->ix_epoch[r]++;
	if (n == 0)
		return PPC_OK;
	PPC_TRY(ensure_lists(s));
	const size_t nd = (size_t)n;
	PPC_TRY(ensure_field_scratch(s, sizeof(int32_t) * (3 * nd + nd * s->ncap + 2)));
	int32_t* ip = static_cast<int32_t*>(s->ix_scratch);
	const int32_t base = s->reps[r].base;
	const ix_columns& c = s->v.ix;
	const size_t D = s->ndefs, S = c.S;
	ix_fields x {};
	x.n = n;
	x.substrates = c.S;
	x.replicate = r;
	x.base = base;
	x.dt = s->params.mechanics_time_step;
	x.epoch = epoch;
	x.status = ip;
	x.ncand = ip + 2;
	x.dep = ip + 2 + nd;
	x.cand = ip + 2 + 2 * nd;
	x.order = ip + 2 + 2 * nd + nd * s->ncap;
	x.dead = c.dead + base;
	x.dead_phago = c.dead_phago + base;
	x.damage_rate = c.damage_rate + base;
	x.live_phago = c.live_phago + base * D;
	x.attack = c.attack + base * D;
	x.fusion = c.fusion + base * D;
	x.immuno = c.immuno + base * D;
	x.frac = c.frac + base * S;
	x.damage = c.damage + base;
	x.attack_time = c.attack_time + base;
	x.nuclei = c.nuclei + base;
	x.fluid = c.fluid + base;
	x.solid = c.solid + base;
	x.cyto = c.cyto + base;
	x.cyto_fluid = c.cyto_fluid + base;
	x.cyto_solid = c.cyto_solid + base;
	x.nuc_fluid = c.nuc_fluid + base;
	x.nuc_solid = c.nuc_solid + base;
	x.fluid_fraction = c.fluid_fraction + base;
	x.c2n = c.c2n + base;
	x.target_cyto = c.target_cyto + base;
	x.target_nuc = c.target_nuc + base;
	x.isub = c.isub + base * S;
	PPC_CUDA(cudaMemsetAsync(x.status, 0, 2 * sizeof(int32_t), s->stream));
	PPC_TRY(launch_interactions(s, x));
	// the call's status and the device error word, with one synchronisation
	PPC_CUDA(cudaMemcpyAsync(s->pinned_err + 1, x.status, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
	PPC_CUDA(cudaMemcpyAsync(s->pinned_err, s->v.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	PPC_CUDA(cudaGetLastError());
	if (s->pinned_err[1])
		return fail(PPC_ERR_CAPACITY, "a neighbour list exceeds the neighbour capacity: no interaction ran");
	// positions and radii changed: the next mesh update rebuilds the bins; the
	// neighbour lists stay those the interactions used, as in the reference
	invalidate_bins(s);
	if (f)
	{
		std::vector<column> back;
		for (const auto& col : ix_column_list(s->v.ix, f, s->ndefs))
			back.push_back(col);
		PPC_TRY(move_columns(s, back, base, n, false));
		return finish(s);
	}
	return map_errors(s, s->pinned_err[0]);
}

int ppc_step(ppc_state* s, int32_t steps)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	return run_steps(s, steps, false, 0, 0);
}

int ppc_autotune(ppc_state* s, int32_t steps, int32_t* tile_edge, int32_t* threads)
{
	if (!s || steps < 1)
		return fail(PPC_ERR_ARG, "autotune needs a state and steps >= 1");
	struct shape
	{
		int edge, threads, smem;
	};
	const shape cand[] = { { -4, 128, 0 }, { -3, 128, 0 }, { -1, 128, 0 }, { -2, 128, 0 }, { 0, 128, 32 * 1024 },
							 { 0, 64, 16 * 1024 } };
	const int ncand = (int)(sizeof cand / sizeof cand[0]);
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	PPC_CUDA(cudaEventCreate(&e0));
	PPC_CUDA(cudaEventCreate(&e1));
	int best = -1;
	float best_ms = 0.f;
	int rc = PPC_OK;
	for (int k = 0; k < ncand && rc == PPC_OK; k++)
	{
		rc = ppc_set_launch_shape(s, cand[k].edge, cand[k].threads, cand[k].smem);
		if (rc == PPC_OK)
			rc = run_steps(s, steps, false, 0, 0); // warm-up: graph capture of this shape
		if (rc != PPC_OK)
			break;
		float ms = 0.f;
		if (cudaEventRecord(e0, s->stream) != cudaSuccess)
			rc = fail(PPC_ERR_CUDA, "cudaEventRecord failed");
		if (rc == PPC_OK)
			rc = run_steps(s, steps, false, 0, 0);
		if (rc == PPC_OK
			&& (cudaEventRecord(e1, s->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess
				|| cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
			rc = fail(PPC_ERR_CUDA, "timing the candidate shape failed");
		if (rc == PPC_OK && (best < 0 || ms < best_ms))
		{
			best = k;
			best_ms = ms;
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	PPC_TRY(rc);
	PPC_TRY(ppc_set_launch_shape(s, cand[best].edge, cand[best].threads, cand[best].smem));
	if (tile_edge)
		*tile_edge = cand[best].edge;
	if (threads)
		*threads = cand[best].threads;
	return PPC_OK;
}

int ppc_step_with_phenotype(ppc_state* s, int32_t steps, double p_divide, double p_death)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	return run_steps(s, steps, true, p_divide, p_death);
}

int ppc_get_neighbors(ppc_state* s, int32_t r, int32_t* counts, int32_t* lists, int32_t list_capacity)
{
	if (!valid(s, r) || !counts || !lists || list_capacity < 1)
		return fail(PPC_ERR_ARG, "invalid arguments");
	PPC_TRY(ensure_lists(s));
	std::vector<rep_counters> c;
	PPC_TRY(read_counters(s, c));
	const int32_t n = c[r].count;
	if (n == 0)
		return PPC_OK;
	int32_t* d = nullptr;
	const size_t bytes = (size_t)n * (list_capacity + 1) * sizeof(int32_t);
	PPC_CUDA(cudaMalloc(&d, bytes));
	int rc = launch_neighbors_local(s, r, n, d, d + n, list_capacity);
	if (rc == PPC_OK)
	{
		cudaMemcpyAsync(counts, d, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream);
		cudaMemcpyAsync(lists, d + n, (size_t)n * list_capacity * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream);
		cudaStreamSynchronize(s->stream);
	}
	cudaFree(d);
	PPC_TRY(rc);
	for (int32_t i = 0; i < n; i++)
		if (counts[i] > list_capacity || counts[i] > s->ncap)
			return fail(PPC_ERR_CAPACITY, "a neighbour list is longer than the capacity");
	return finish(s);
}

int ppc_get_voxel_count(ppc_state* s, int32_t r, int64_t* voxel_count)
{
	if (!valid(s, r) || !voxel_count)
		return fail(PPC_ERR_ARG, "invalid arguments");
	*voxel_count = s->reps[r].voxels;
	return PPC_OK;
}

int ppc_get_mesh_bins(ppc_state* s, int32_t r, int32_t* voxel_counts, int32_t* agents)
{
	if (!valid(s, r) || !voxel_counts || !agents)
		return fail(PPC_ERR_ARG, "invalid arguments");
	PPC_TRY(ensure_bins(s));
	const rep_info& R = s->reps[r];
	std::vector<int32_t> starts(R.voxels + 1);
	PPC_CUDA(cudaMemcpyAsync(starts.data(), s->v.vstart + R.vox_base, (R.voxels + 1) * 4, cudaMemcpyDeviceToHost,
							 s->stream));
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	const int32_t first = starts[0], n = starts[R.voxels] - starts[0];
	std::vector<int32_t> sorted(std::max(n, 1));
	if (n > 0)
	{
		PPC_CUDA(cudaMemcpyAsync(sorted.data(), s->v.sorted + first, (size_t)n * 4, cudaMemcpyDeviceToHost, s->stream));
		PPC_CUDA(cudaStreamSynchronize(s->stream));
	}
	for (int64_t k = 0; k < R.voxels; k++)
		voxel_counts[k] = starts[k + 1] - starts[k];
	for (int32_t u = 0; u < n; u++)
		agents[u] = sorted[u] - R.base;
	return finish(s);
}

int ppc_get_mesh_position(const ppc_mesh* mesh, const double* position, int32_t* c)
{
	if (!mesh || !position || !c)
		return fail(PPC_ERR_ARG, "null argument");
	rep_info R {};
	mesh_info(*mesh, R);
	for (int d = 0; d < 3; d++)
	{
		c[d] = 0;
		if (d >= mesh->dims)
			continue;
		const double q = (position[d] - R.mins[d]) / R.shape[d];
		c[d] = (q == q && q > 0) ? (q >= R.grid[d] ? R.grid[d] - 1 : (int32_t)q) : 0;
	}
	return PPC_OK;
}

int ppc_get_mesh_index(const ppc_mesh* mesh, const int32_t* c, int32_t* index)
{
	if (!mesh || !c || !index)
		return fail(PPC_ERR_ARG, "null argument");
	rep_info R {};
	mesh_info(*mesh, R);
	*index = c[0] + R.grid[0] * (c[1] + R.grid[1] * c[2]);
	return PPC_OK;
}

int ppc_set_profiling(ppc_state* s, int32_t on)
{
	if (!s)
		return fail(PPC_ERR_ARG, "null state");
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	s->profiling = on != 0;
	s->prof_used = 0;
	return PPC_OK;
}

int ppc_get_profile(ppc_state* s, double* fused_ms, int64_t* fused_launches)
{
	if (!s || !fused_ms || !fused_launches)
		return fail(PPC_ERR_ARG, "null argument");
	PPC_CUDA(cudaStreamSynchronize(s->stream));
	double total = 0;
	for (size_t k = 0; k + 1 < s->prof_used; k += 2)
	{
		float ms = 0;
		PPC_CUDA(cudaEventElapsedTime(&ms, s->prof_events[k], s->prof_events[k + 1]));
		total += ms;
	}
	*fused_ms = total;
	*fused_launches = (int64_t)(s->prof_used / 2);
	return PPC_OK;
}

int ppc_get_launch_count(ppc_state* s, int64_t* launches)
{
	if (!s || !launches)
		return fail(PPC_ERR_ARG, "null argument");
	*launches = s->launches;
	return PPC_OK;
}

} // extern "C"
