/*
 * ppc_oracle.cpp — CPU restatement of paraPhysiCell's mechanics solver.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA path and the
 * CPU baseline of the benchmark; the product never loads it.
 *
 * Compile with -ffp-contract=off (no FMA contraction), like the reference's
 * default x86-64 build (its CMakeLists.txt sets no -march, so GCC emits no
 * FMA). Every function below names the reference lines it restates.
 * See ppc_oracle.h for the two execution modes.
 */
#include "ppc_oracle.h"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <shared_mutex>
#include <vector>

#include "../include/ppc_draws.h"

namespace {

using real_t = double;
using index_t = int32_t;

// reference: src/solver/host/position_solver.cpp:13
constexpr real_t simple_pressure_coefficient = 36.64504274775163;
// reference: src/solver/host/position_solver.cpp:372
constexpr index_t erased_spring = -1;

struct mesh_t
{
	int dims;
	int mins[3], maxs[3], shape[3], grid[3];
	int64_t voxels;
};

struct world
{
	mesh_t mesh;
	ppc_params params;
	index_t ndefs;
	index_t n = 0;
	index_t cap = 0;

	std::vector<real_t> pos, vel, vprev, pressure;
	std::vector<real_t> radius, rep, adh, rmad, bm, ec, arate, drate, aff;
	std::vector<index_t> maxatt, def;
	std::vector<uint8_t> movable, flags;
	std::vector<int64_t> ids;
	std::vector<real_t> vol, nvol, nrad, sarea, polarity, orient;
	std::vector<std::vector<index_t>> neighbors, springs;

	// mechanics mesh bins (reference: src/environment.h:44) and the solver's
	// per-voxel atomic counters (reference: containers_solver.h:19)
	std::unique_ptr<std::vector<index_t>[]> bins;
	std::unique_ptr<std::atomic<index_t>[]> bin_sizes;

	int64_t divisions = 0, deaths = 0, next_id = 0;
	// draw epochs: `epoch` for phenotype draws (flags, division), advanced
	// once per draw-consuming call; `spring_epoch` for the attachment loop
	uint64_t seed = 0, epoch = 0, spring_epoch = 0;
	uint64_t ix_epoch = 0; // cell-cell interaction calls so far
	uint64_t mot_epoch = 0; // motility calls so far
	bool timed = false; // timed mode draws from thread_local mt19937
	bool mot_per_agent = false; // resident motility: restrict_per_agent of the last upload

	std::mutex removal_mtx;
	std::shared_mutex division_mtx;

	// Phenotype columns held beside the mechanics fields once a caller makes
	// them resident (orc_upload_interactions / orc_upload_motility): they
	// move with their agent on removal, and division halves, copies and
	// resets them as cell::divide does (src/cell.cpp:108-163).
	struct ix_store
	{
		bool on = false;
		int S = 0;
		bool halve_substrates = false; // e.m.compute_internalized_substrates
		std::vector<uint8_t> dead;
		std::vector<real_t> dead_phago, damage_rate, live_phago, attack, fusion, immuno, frac, damage, attack_time,
			fluid, solid, cyto, cyto_fluid, cyto_solid, nuc_fluid, nuc_solid, fluid_fraction, c2n, target_cyto,
			target_nuc, isub;
		std::vector<int32_t> nuclei;

		// f(column, values per agent) for every column
		template <typename F>
		void each(F&& f, int D)
		{
			f(dead, 1);
			f(dead_phago, 1);
			f(damage_rate, 1);
			f(live_phago, D);
			f(attack, D);
			f(fusion, D);
			f(immuno, D);
			f(frac, S);
			f(damage, 1);
			f(attack_time, 1);
			f(nuclei, 1);
			for (auto* v : { &fluid, &solid, &cyto, &cyto_fluid, &cyto_solid, &nuc_fluid, &nuc_solid, &fluid_fraction,
							 &c2n, &target_cyto, &target_nuc })
				f(*v, 1);
			f(isub, S);
		}
	} ix;

	struct mot_store
	{
		bool on = false;
		int S = 0; // chemotactic sensitivities per agent
		std::vector<uint8_t> motile, restrict2d, rule;
		std::vector<real_t> persistence, speed, bias, direction, vector, chemo_dir, sens;
		std::vector<int32_t> chemo_index;

		template <typename F>
		void each(F&& f, int dims)
		{
			f(motile, 1);
			f(restrict2d, 1);
			f(rule, 1);
			f(persistence, 1);
			f(speed, 1);
			f(bias, 1);
			f(direction, dims);
			f(vector, dims);
			f(chemo_index, 1);
			f(chemo_dir, 1);
			f(sens, S);
		}
	} mot;

	// substrate gradients of the diffusion mesh (agent::nearest_gradient of
	// the absent paraBioFVM): per voxel, per substrate, x, y, z
	struct gradient_field
	{
		int S = 0, grid[3] = { 1, 1, 1 };
		real_t shape[3] = { 1, 1, 1 };
		std::vector<real_t> g;
	} grad;

	// row `dst` of every resident column takes row `src`'s values
	void copy_rows(index_t dst, index_t src)
	{
		auto cp = [&](auto& col, int width) {
			std::copy_n(col.begin() + (size_t)src * width, width, col.begin() + (size_t)dst * width);
		};
		if (ix.on)
			ix.each(cp, ndefs);
		if (mot.on)
			mot.each(cp, mesh.dims);
	}

	void grow_stores(index_t rows)
	{
		auto rs = [&](auto& col, int width) { col.resize((size_t)rows * width); };
		if (ix.on)
			ix.each(rs, ndefs);
		if (mot.on)
			mot.each(rs, mesh.dims);
	}

	void grow(index_t new_cap)
	{
		if (new_cap <= cap)
			return;
		int d = mesh.dims;
		pos.resize((size_t)new_cap * d);
		vel.resize((size_t)new_cap * d);
		vprev.resize((size_t)new_cap * d);
		orient.resize((size_t)new_cap * d);
		for (auto* v : { &pressure, &radius, &rep, &adh, &rmad, &bm, &ec, &arate, &drate, &vol, &nvol, &nrad, &sarea,
						 &polarity })
			v->resize(new_cap);
		aff.resize((size_t)new_cap * ndefs);
		maxatt.resize(new_cap);
		def.resize(new_cap);
		movable.resize(new_cap);
		flags.resize(new_cap);
		ids.resize(new_cap);
		neighbors.resize(new_cap);
		springs.resize(new_cap);
		cap = new_cap;
		grow_stores(new_cap);
	}
};

thread_local std::mt19937 tl_generator;

// reference: src/random.cpp:16-20 (uniform over [0,1) from the thread's generator)
real_t timed_uniform()
{
	std::uniform_real_distribution<real_t> distribution(0, 1);
	return distribution(tl_generator);
}

/* ---- mesh helpers (paraBioFVM cartesian_mesh, absent; rounding assumed) ---- */

void init_mesh(mesh_t& m, const ppc_mesh& pm)
{
	m.dims = pm.dims;
	m.voxels = 1;
	for (int d = 0; d < 3; d++)
	{
		m.mins[d] = pm.bounding_box_mins[d];
		m.maxs[d] = pm.bounding_box_maxs[d];
		m.shape[d] = pm.voxel_shape[d];
		m.grid[d] = d < pm.dims ? (m.maxs[d] - m.mins[d] + m.shape[d] - 1) / m.shape[d] : 1;
		if (m.grid[d] < 1)
			m.grid[d] = 1;
		m.voxels *= m.grid[d];
	}
}

// common_solver::get_mesh_position (reference: src/solver/host/common_solver.cpp:18-38)
// over cartesian_mesh::voxel_position: truncation of (x - min) / shape; the
// coordinate is clamped into the grid (the reference indexes out of bounds for
// an agent exactly on the upper face of a grid whose extent is a multiple of
// the voxel size).
void mesh_position(const mesh_t& m, const real_t* p, index_t* c)
{
	for (int d = 0; d < 3; d++)
	{
		index_t v = 0;
		if (d < m.dims)
		{
			real_t q = (p[d] - (real_t)m.mins[d]) / (real_t)m.shape[d];
			v = (index_t)q;
			if (!(q == q) || v < 0)
				v = 0;
			if (v >= m.grid[d])
				v = m.grid[d] - 1;
		}
		c[d] = v;
	}
}

// common_solver::get_mesh_index (reference: common_solver.cpp:10-16), x fastest
inline int64_t mesh_index(const mesh_t& m, const index_t* c)
{
	return c[0] + (int64_t)m.grid[0] * (c[1] + (int64_t)m.grid[1] * c[2]);
}

/* ---- position_helper<dims> (reference: src/solver/host/solver_helper.h:47-315) ---- */

template <int dims>
inline real_t distance(const real_t* l, const real_t* r)
{
	if constexpr (dims == 1)
		return std::abs(l[0] - r[0]);
	else if constexpr (dims == 2)
		return std::sqrt((l[0] - r[0]) * (l[0] - r[0]) + (l[1] - r[1]) * (l[1] - r[1]));
	else
		return std::sqrt((l[0] - r[0]) * (l[0] - r[0]) + (l[1] - r[1]) * (l[1] - r[1]) + (l[2] - r[2]) * (l[2] - r[2]));
}

template <int dims>
inline real_t difference_and_distance(const real_t* l, const real_t* r, real_t* diff)
{
	for (int d = 0; d < dims; d++)
		diff[d] = l[d] - r[d];
	if constexpr (dims == 1)
		return std::abs(diff[0]);
	else if constexpr (dims == 2)
		return std::sqrt(diff[0] * diff[0] + diff[1] * diff[1]);
	else
		return std::sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
}

// update_membrane_velocity (reference: solver_helper.h:14-28)
inline void membrane_velocity(real_t position, real_t bounding_box, real_t sign, real_t radius, real_t strength,
							  real_t& velocity)
{
	real_t dist = std::abs(bounding_box - position);
	dist = std::max<real_t>(dist, 0.00001);
	real_t repulsion = 1 - dist / radius;
	repulsion = repulsion < 0 ? 0 : repulsion;
	repulsion *= repulsion * strength * sign;
	velocity += repulsion * dist;
}

/* ---- containers_solver::update_mechanics_mesh (reference: containers_solver.cpp:15-56) ---- */

void rebuild_mesh(world& w)
{
	const mesh_t& m = w.mesh;
#pragma omp for
	for (int64_t v = 0; v < m.voxels; v++)
	{
		w.bins[v].clear();
		w.bin_sizes[v].store(0, std::memory_order_relaxed);
	}

#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		index_t c[3];
		mesh_position(m, w.pos.data() + (size_t)i * m.dims, c);
		w.bin_sizes[mesh_index(m, c)].fetch_add(1, std::memory_order_relaxed);
	}

#pragma omp for
	for (int64_t v = 0; v < m.voxels; v++)
		w.bins[v].resize(w.bin_sizes[v].load(std::memory_order_relaxed));

#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		index_t c[3];
		mesh_position(m, w.pos.data() + (size_t)i * m.dims, c);
		int64_t k = mesh_index(m, c);
		index_t slot = w.bin_sizes[k].fetch_sub(1, std::memory_order_relaxed) - 1;
		w.bins[k][slot] = i;
	}
}

/* ---- common_solver::for_each_in_mech_neighborhood (reference: common_solver.h:77-105) ---- */

template <typename F>
inline void for_each_in_neighborhood(const world& w, const index_t* c, index_t i, F&& f)
{
	const mesh_t& m = w.mesh;
	for (index_t z = -1; z <= 1; z++)
	{
		if (c[2] + z >= m.grid[2] || c[2] + z < 0)
			continue;
		for (index_t y = -1; y <= 1; y++)
		{
			if (c[1] + y >= m.grid[1] || c[1] + y < 0)
				continue;
			for (index_t x = -1; x <= 1; x++)
			{
				if (c[0] + x >= m.grid[0] || c[0] + x < 0)
					continue;
				index_t cc[3] = { c[0] + x, c[1] + y, c[2] + z };
				for (index_t j : w.bins[mesh_index(m, cc)])
					if (j != i)
						f(j);
			}
		}
	}
}

/* ---- position_solver::update_cell_neighbors (reference: position_solver.cpp:79-97,180-195,262-286) ---- */

template <int dims>
void neighbors_internal(world& w)
{
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		if (w.movable[i] == 0)
			continue;
		index_t c[3];
		mesh_position(w.mesh, w.pos.data() + (size_t)i * dims, c);
		const real_t* pi = w.pos.data() + (size_t)i * dims;
		for_each_in_neighborhood(w, c, i, [&](index_t j) {
			const real_t adhesion_distance = w.rmad[i] * w.radius[i] + w.rmad[j] * w.radius[j];
			const real_t dist = distance<dims>(pi, w.pos.data() + (size_t)j * dims);
			if (dist <= adhesion_distance)
				w.neighbors[i].push_back(j);
		});
	}
}

void update_neighbors(world& w)
{
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
		w.neighbors[i].clear();

	if (w.mesh.dims == 1)
		neighbors_internal<1>(w);
	else if (w.mesh.dims == 2)
		neighbors_internal<2>(w);
	else
		neighbors_internal<3>(w);
}

/* ---- position_solver::update_cell_forces (reference: position_solver.cpp:15-77,99-113,158-178,233-260) ---- */

template <int dims>
inline void solve_pair(world& w, index_t lhs, index_t rhs)
{
	real_t diff[dims];
	const real_t dist = std::max<real_t>(
		difference_and_distance<dims>(w.pos.data() + (size_t)lhs * dims, w.pos.data() + (size_t)rhs * dims, diff),
		0.00001);

	real_t repulsion;
	{
		const real_t repulsive_distance = w.radius[lhs] + w.radius[rhs];
		repulsion = 1 - dist / repulsive_distance;
		repulsion = repulsion < 0 ? 0 : repulsion;
		repulsion *= repulsion;
		// the reference adds to both sides from inside `omp for` over lhs
		// (a data race when threaded); run serially this is the serial sum
		w.pressure[lhs] += repulsion * simple_pressure_coefficient;
		w.pressure[rhs] += repulsion * simple_pressure_coefficient;
		repulsion *= std::sqrt(w.rep[lhs] * w.rep[rhs]);
	}

	real_t adhesion;
	{
		const real_t adhesion_distance = w.rmad[lhs] * w.radius[lhs] + w.rmad[rhs] * w.radius[rhs];
		adhesion = 1 - dist / adhesion_distance;
		adhesion *= adhesion;
		const index_t ldef = w.def[lhs], rdef = w.def[rhs];
		adhesion *= std::sqrt(w.adh[lhs] * w.adh[rhs] * w.aff[(size_t)lhs * w.ndefs + rdef]
							  * w.aff[(size_t)rhs * w.ndefs + ldef]);
	}

	const real_t force = (repulsion - adhesion) / dist;
	real_t* v = w.vel.data() + (size_t)lhs * dims;
	for (int d = 0; d < dims; d++)
		v[d] += force * diff[d];
}

template <int dims>
void forces_internal(world& w)
{
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		if (w.movable[i] == 0)
			continue;
		for (index_t j : w.neighbors[i])
			solve_pair<dims>(w, i, j);
	}
}

void update_forces(world& w)
{
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
		w.pressure[i] = 0;

	if (w.mesh.dims == 1)
		forces_internal<1>(w);
	else if (w.mesh.dims == 2)
		forces_internal<2>(w);
	else
		forces_internal<3>(w);
}

/* ---- basement membrane (reference: position_solver.cpp:147-156,214-231,316-335; solver_helper.h:103-110,184-193,288-299) ---- */

void update_membrane(world& w)
{
	if (!w.params.virtual_wall_at_domain_edges)
		return;
	const mesh_t& m = w.mesh;
	const int dims = m.dims;
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		if (w.movable[i] == 0)
			continue;
		const real_t* p = w.pos.data() + (size_t)i * dims;
		real_t* v = w.vel.data() + (size_t)i * dims;
		const real_t r = w.radius[i], s = w.bm[i];
		if (dims == 1)
		{
			// the 1-D helper uses the y maximum for the upper x wall
			// (reference: solver_helper.h:109); kept as is
			membrane_velocity(p[0], m.mins[0], 1, r, s, v[0]);
			membrane_velocity(p[0], m.maxs[1], -1, r, s, v[0]);
		}
		else
		{
			for (int d = 0; d < dims; d++)
			{
				membrane_velocity(p[d], m.mins[d], 1, r, s, v[d]);
				membrane_velocity(p[d], m.maxs[d], -1, r, s, v[d]);
			}
		}
	}
}

/* ---- spring attachments (reference: position_solver.cpp:337-449,451-479) ---- */

template <int dims>
void spring_contract(world& w)
{
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		if (w.movable[i] == 0)
			continue;
		for (std::size_t k = 0; k < w.springs[i].size(); k++)
		{
			const index_t j = w.springs[i][k];
			const index_t idef = w.def[i], jdef = w.def[j];
			const real_t adhesion = std::sqrt(w.ec[i] * w.ec[j] * w.aff[(size_t)i * w.ndefs + jdef]
											  * w.aff[(size_t)j * w.ndefs + idef]);
			real_t difference[dims];
			for (int d = 0; d < dims; d++)
				difference[d] = w.pos[(size_t)j * dims + d] - w.pos[(size_t)i * dims + d];
			for (int d = 0; d < dims; d++)
				w.vel[(size_t)i * dims + d] += adhesion * difference[d];
		}
	}
}

// draws of the attachment loop: timed mode uses the thread's mt19937 like
// the reference; serial mode uses the counter-based stream
inline real_t spring_draw(world& w, uint64_t epoch, index_t i, uint64_t k)
{
	return w.timed ? timed_uniform() : ppc_uniform(w.seed, epoch, 0, (uint64_t)i, k);
}

void spring_attachments_internal(world& w, uint64_t epoch)
{
	const real_t dt = w.params.mechanics_time_step;
	const index_t D = w.ndefs;

	// mark springs for detachment
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		for (index_t k = 0; k < (index_t)w.springs[i].size(); k++)
		{
			if (spring_draw(w, epoch, i, 1024 + (uint64_t)k) <= w.drate[i] * dt)
			{
#pragma omp critical
				{
					const index_t j = w.springs[i][k];
					if (j != erased_spring)
					{
						w.springs[i][k] = erased_spring;
						*std::find(w.springs[j].begin(), w.springs[j].end(), i) = erased_spring;
					}
				}
			}
		}
	}

	// remove marked springs
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		auto it = std::remove(w.springs[i].begin(), w.springs[i].end(), erased_spring);
		w.springs[i].erase(it, w.springs[i].end());
	}

	// attach
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		for (std::size_t k = 0; k < w.neighbors[i].size(); k++)
		{
			const index_t j = w.neighbors[i][k];
			if (j < i)
				continue;
			const real_t affinity_l = w.aff[(size_t)i * D + w.def[j]];
			const real_t prob_l = w.arate[i] * dt * affinity_l;
			const real_t affinity_r = w.aff[(size_t)j * D + w.def[i]];
			const real_t prob_r = w.arate[j] * dt * affinity_r;
			if (spring_draw(w, epoch, i, 4096 + 2 * (uint64_t)k) <= prob_l
				|| spring_draw(w, epoch, i, 4096 + 2 * (uint64_t)k + 1) <= prob_r)
			{
#pragma omp critical
				{
					if ((index_t)w.springs[i].size() < w.maxatt[i] && (index_t)w.springs[j].size() < w.maxatt[j])
					{
						w.springs[i].push_back(j);
						w.springs[j].push_back(i);
					}
				}
			}
		}
	}
}

void update_springs(world& w)
{
	if (!w.params.automated_spring_adhesion)
		return;
	uint64_t epoch = w.spring_epoch;
	spring_attachments_internal(w, epoch);
#pragma omp single
	w.spring_epoch++;

	if (w.mesh.dims == 1)
		spring_contract<1>(w);
	else if (w.mesh.dims == 2)
		spring_contract<2>(w);
	else
		spring_contract<3>(w);
}

/* ---- position_solver::update_positions (reference: position_solver.cpp:481-520) ---- */

void update_positions(world& w)
{
	const int dims = w.mesh.dims;
	const real_t dt = w.params.mechanics_time_step;
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		if (!w.movable[i])
			continue;
		const real_t factor = dt * 1.5;
		const real_t previous_factor = dt * -0.5;
		for (int d = 0; d < dims; d++)
		{
			size_t k = (size_t)i * dims + d;
			w.pos[k] += w.vel[k] * factor + w.vprev[k] * previous_factor;
			w.vprev[k] = w.vel[k];
			w.vel[k] = 0;
		}
	}
}

/* ---- container: create / remove_at (paraBioFVM agent_container_common, absent;
        src/cell_data.cpp:262-313, src/cell.cpp:47-61) ---- */

// appends one agent with the defaults of a freshly constructed cell
index_t create_agent(world& w)
{
	if (w.n == w.cap)
		w.grow(std::max<index_t>(16, w.cap * 2));
	index_t i = w.n++;
	const int dims = w.mesh.dims;
	for (int d = 0; d < dims; d++)
	{
		w.pos[(size_t)i * dims + d] = 0;
		w.vel[(size_t)i * dims + d] = 0;
		w.vprev[(size_t)i * dims + d] = 0;
		w.orient[(size_t)i * dims + d] = 0;
	}
	w.pressure[i] = 0;
	w.flags[i] = PPC_FLAG_NONE;
	w.movable[i] = 1;
	w.neighbors[i].clear();
	w.springs[i].clear();
	w.ids[i] = w.next_id++;
	return i;
}

// cell_data::remove (reference: src/cell_data.cpp:285-313): the last agent's
// fields move into slot i
void remove_at(world& w, index_t i)
{
	index_t last = --w.n;
	if (i == last)
		return;
	const int dims = w.mesh.dims;
	for (int d = 0; d < dims; d++)
	{
		w.pos[(size_t)i * dims + d] = w.pos[(size_t)last * dims + d];
		w.vel[(size_t)i * dims + d] = w.vel[(size_t)last * dims + d];
		w.vprev[(size_t)i * dims + d] = w.vprev[(size_t)last * dims + d];
		w.orient[(size_t)i * dims + d] = w.orient[(size_t)last * dims + d];
	}
	for (auto* v : { &w.pressure, &w.radius, &w.rep, &w.adh, &w.rmad, &w.bm, &w.ec, &w.arate, &w.drate, &w.vol,
					 &w.nvol, &w.nrad, &w.sarea, &w.polarity })
		(*v)[i] = (*v)[last];
	std::memcpy(w.aff.data() + (size_t)i * w.ndefs, w.aff.data() + (size_t)last * w.ndefs, sizeof(real_t) * w.ndefs);
	w.maxatt[i] = w.maxatt[last];
	w.def[i] = w.def[last];
	w.movable[i] = w.movable[last];
	w.flags[i] = w.flags[last];
	w.ids[i] = w.ids[last];
	w.neighbors[i] = std::move(w.neighbors[last]);
	w.springs[i] = std::move(w.springs[last]);
	w.copy_rows(i, last);
}

// reference: containers_solver.cpp:58-68
void remove_attached(index_t to_remove, std::vector<std::vector<index_t>>& attached)
{
	for (index_t s : attached[to_remove])
	{
		auto it = std::find(attached[s].begin(), attached[s].end(), to_remove);
		*it = attached[s].back();
		attached[s].pop_back();
	}
}

// reference: containers_solver.cpp:70-79
void rename_attached(index_t old_index, index_t new_index, std::vector<std::vector<index_t>>& attached)
{
	for (index_t s : attached[old_index])
		*std::find(attached[s].begin(), attached[s].end(), old_index) = new_index;
}

// remove_single (reference: containers_solver.cpp:81-123). Vectors never
// shrink, so reading a slot past the live count reads stale data exactly
// like the reference does.
void remove_single(world& w, index_t i)
{
	const mesh_t& m = w.mesh;
	while (true)
	{
		bool out_of_bounds = false;
		for (int d = 0; d < m.dims; d++)
		{
			real_t x = w.pos[(size_t)i * m.dims + d];
			if (x < m.mins[d] || x > m.maxs[d])
				out_of_bounds = true;
		}
		if (!out_of_bounds && w.flags[i] != PPC_FLAG_TO_REMOVE)
			return;

		std::lock_guard<std::mutex> l(w.removal_mtx);
		if (i >= w.n)
			return;
		if (w.flags[i] == PPC_FLAG_TO_REMOVE)
			w.deaths++;
		remove_attached(i, w.springs);
		rename_attached(w.n - 1, i, w.springs);
		// attached_cells are not modelled: they are only written by the
		// cell-cell interaction and contact code, which is outside this path
		remove_at(w, i);
		if (i == w.n)
			return;
	}
}

// update_cell_container_internal (reference: containers_solver.cpp:125-147)
void compact_mechanics(world& w)
{
	index_t n = w.n;
#pragma omp barrier
#pragma omp for
	for (index_t i = 0; i < n; i++)
		remove_single(w, i);
}

/* ---- division (reference: src/cell.cpp:108-163, interactions_solver.cpp:89-96,
        data_storage_phenotype.cpp:530-550) ---- */

void divide(world& w, index_t p, index_t c, uint64_t epoch)
{
	const int dims = w.mesh.dims;
	remove_attached(p, w.springs);
	w.springs[p].clear();

	real_t walk[3];
	ppc_random_walk(dims, w.seed, epoch, 0, (uint64_t)p, PPC_DRAW_WALK, walk);
	{
		real_t tmp = 0;
		for (int d = 0; d < dims; d++)
			tmp += walk[d] * w.orient[(size_t)p * dims + d];
		for (int d = 0; d < dims; d++)
			walk[d] = (walk[d] - tmp * w.orient[(size_t)p * dims + d] * w.polarity[p]) * w.radius[p];
	}

	// volume.divide() on the fields this path holds, then geometry.update()
	w.vol[p] *= 0.5;
	w.nvol[p] *= 0.5;
	const real_t four_thirds_pi = M_PI * 4.0 / 3.0;
	w.radius[p] = ppc_cbrt(w.vol[p] / four_thirds_pi);
	w.nrad[p] = ppc_cbrt(w.nvol[p] / four_thirds_pi);
	w.sarea[p] = 4.0 * M_PI * w.radius[p] * w.radius[p];

	// resident phenotype columns: molecular.divide() (when substrates are
	// computed), damage and total attack time cleared, volume.divide() on
	// every compartment (data_storage_phenotype.cpp:530-560)
	if (w.ix.on)
	{
		auto& x = w.ix;
		if (x.halve_substrates)
			for (int q = 0; q < x.S; q++)
				x.isub[(size_t)p * x.S + q] *= 0.5;
		x.damage[p] = 0;
		x.attack_time[p] = 0;
		for (auto* v : { &x.fluid, &x.solid, &x.cyto, &x.cyto_fluid, &x.cyto_solid, &x.nuc_fluid, &x.nuc_solid,
						 &x.target_cyto, &x.target_nuc })
			(*v)[p] *= 0.5;
	}

	// new_cell.copy_from(*this): phenotype and definition index; state
	// (velocities, pressure, springs, is_movable) keeps the new-cell defaults
	for (auto* v : { &w.radius, &w.rep, &w.adh, &w.rmad, &w.bm, &w.ec, &w.arate, &w.drate, &w.vol, &w.nvol, &w.nrad,
					 &w.sarea, &w.polarity })
		(*v)[c] = (*v)[p];
	std::memcpy(w.aff.data() + (size_t)c * w.ndefs, w.aff.data() + (size_t)p * w.ndefs, sizeof(real_t) * w.ndefs);
	w.maxatt[c] = w.maxatt[p];
	w.def[c] = w.def[p];
	// the resident phenotype columns are copied (phenotype_t::copy_to); the
	// new cell's state keeps its constructor's defaults (no damage, no
	// attack time, one nucleus: cell_state::set_defaults, src/cell.cpp:36-45)
	w.copy_rows(c, p);
	if (w.ix.on)
	{
		w.ix.damage[c] = 0;
		w.ix.attack_time[c] = 0;
		w.ix.nuclei[c] = 1;
	}
	// assign_orientation() of the new cell draws a fresh direction
	ppc_random_walk(dims, w.seed, epoch, 0, (uint64_t)p, PPC_DRAW_ORIENTATION, w.orient.data() + (size_t)c * dims);

	for (int d = 0; d < dims; d++)
	{
		w.pos[(size_t)c * dims + d] = w.pos[(size_t)p * dims + d] + walk[d];
		w.pos[(size_t)p * dims + d] -= walk[d] * 0.5;
	}
}

// update_cell_container_for_phenotype (reference: containers_solver.cpp:149-188)
void compact_phenotype(world& w)
{
	const index_t n = w.n;
	const uint64_t epoch = w.epoch;
#pragma omp barrier

#pragma omp for
	for (index_t i = 0; i < n; i++)
	{
		if (w.flags[i] == PPC_FLAG_TO_DIVIDE)
		{
			w.flags[i] = PPC_FLAG_NONE;
			index_t c;
			{
				std::unique_lock<std::shared_mutex> l(w.division_mtx);
				c = create_agent(w);
				w.divisions++;
			}
			{
				std::shared_lock<std::shared_mutex> l(w.division_mtx);
				divide(w, i, c, epoch);
			}
		}
	}

#pragma omp for
	for (index_t i = 0; i < n; i++)
		remove_single(w, i);

#pragma omp single
	w.epoch++;
}

// stand-in for the phenotype models that set the flags
void flag_by_draws(world& w, double p_divide, double p_death)
{
	const uint64_t epoch = w.epoch;
#pragma omp for
	for (index_t i = 0; i < w.n; i++)
	{
		if (ppc_uniform(w.seed, epoch, 0, (uint64_t)i, PPC_DRAW_DEATH) < p_death)
			w.flags[i] = PPC_FLAG_TO_REMOVE;
		else if (ppc_uniform(w.seed, epoch, 0, (uint64_t)i, PPC_DRAW_DIVIDE) < p_divide)
			w.flags[i] = PPC_FLAG_TO_DIVIDE;
	}
#pragma omp single
	w.epoch++;
}

/* ---- cell-cell interactions (reference: src/solver/host/interactions_solver.cpp:1-265) ---- */

constexpr real_t ix_zero_threshold = 1e-16; // reference: src/solver/host/solver_helper.h:12

/* ---- motility (reference: src/solver/host/position_solver.cpp:115-145,198-212,288-314,
        solver_helper.h:82-101,160-182,250-287) ---- */

// normalize (reference: src/solver/host/solver_helper.h:30-45)
void normalize_vec(real_t* x, int dims)
{
	real_t length = 0;
	for (int d = 0; d < dims; d++)
		length += x[d] * x[d];
	length = std::sqrt(length);
	for (int d = 0; d < dims; d++)
		x[d] = length > ix_zero_threshold ? x[d] / length : 0;
}

// the gradient of substrate q in the diffusion voxel holding agent i
void nearest_gradient(const world& w, index_t i, int q, real_t* g)
{
	const int dims = w.mesh.dims;
	int c[3] = { 0, 0, 0 };
	for (int d = 0; d < dims; d++)
	{
		const real_t f = (w.pos[(size_t)i * dims + d] - w.mesh.mins[d]) / w.grad.shape[d];
		const int k = f > 0 ? (int)f : 0;
		c[d] = k < w.grad.grid[d] ? k : w.grad.grid[d] - 1;
	}
	const int64_t vox = c[0] + (int64_t)w.grad.grid[0] * (c[1] + (int64_t)w.grad.grid[1] * c[2]);
	for (int d = 0; d < dims; d++)
		g[d] = w.grad.g[(size_t)(vox * w.grad.S + q) * 3 + d];
}

// chemotaxis_function and advanced_chemotaxis_function<normalize>
// (reference: src/original/core/standard_models.cpp:542-583)
void direction_rule(const world& w, const ppc_motility& f, index_t i, int rule)
{
	const int dims = w.mesh.dims;
	real_t* dir = f.migration_bias_direction + (size_t)i * dims;
	if (rule == PPC_DIRECTION_CHEMOTAXIS)
	{
		real_t g[3];
		nearest_gradient(w, i, f.chemotaxis_index[i], g);
		for (int d = 0; d < dims; d++)
			dir[d] = g[d] * f.chemotaxis_direction[i];
	}
	else
	{
		for (int d = 0; d < dims; d++)
			dir[d] = 0;
		for (int q = 0; q < w.grad.S; q++)
		{
			real_t g[3];
			nearest_gradient(w, i, q, g);
			if (rule == PPC_DIRECTION_ADVANCED_CHEMOTAXIS_NORMALIZED)
				normalize_vec(g, dims);
			const real_t wgt = q < f.substrates ? f.chemotactic_sensitivities[(size_t)i * f.substrates + q] : 0.0;
			for (int d = 0; d < dims; d++)
				dir[d] += g[d] * wgt;
		}
	}
	normalize_vec(dir, dims);
}

// update_motility_single for every agent, with the reference's random walk
// from counter-based draws; the direction-update callbacks are not run. The
// reference passes the whole restrict_to_2d array to random_walk, whose bool
// parameter is then always true (position_solver.cpp:131), so every 3-D walk
// lies in the xy-plane; fields.restrict_per_agent = 1 reads each agent's flag
// instead.
void motility(world& w, ppc_motility& f)
{
	const uint64_t epoch = w.mot_epoch++;
	const int dims = w.mesh.dims;
	const real_t dt = w.params.mechanics_time_step;
	for (index_t i = 0; i < w.n; i++)
	{
		if (f.is_motile[i] == 0)
			continue;
		real_t* mv = f.motility_vector + (size_t)i * dims;
		if (ppc_uniform(w.seed, epoch, 0, (uint64_t)i, PPC_DRAW_MOTILITY) < dt / f.persistence_time[i])
		{
			real_t walk[3] = { 0, 0, 0 };
			const bool planar = dims == 3 && (f.restrict_per_agent ? f.restrict_to_2d[i] != 0 : true);
			ppc_random_walk(planar ? 2 : dims, w.seed, epoch, 0, (uint64_t)i, PPC_DRAW_MOTILITY + 1u, walk);
			// update_migration_bias_direction_f runs after the walk is drawn
			// (position_solver.cpp:133-136)
			const int rule = f.direction_rule ? (int)f.direction_rule[i] : (int)PPC_DIRECTION_NONE;
			if (rule != PPC_DIRECTION_NONE && !w.grad.g.empty())
				direction_rule(w, f, i, rule);
			const real_t bias = f.migration_bias[i];
			for (int d = 0; d < dims; d++)
				mv[d] = (1 - bias) * walk[d] + bias * f.migration_bias_direction[(size_t)i * dims + d];
			real_t length;
			if (dims == 1)
				length = std::abs(mv[0]);
			else if (dims == 2)
				length = std::sqrt(mv[0] * mv[0] + mv[1] * mv[1]);
			else
				length = std::sqrt(mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2]);
			const real_t scale = f.migration_speed[i];
			for (int d = 0; d < dims; d++)
				mv[d] = length > ix_zero_threshold ? mv[d] * scale / length : 0;
		}
		for (int d = 0; d < dims; d++)
			w.vel[(size_t)i * dims + d] += mv[d];
	}
}

// physicell::update_geometry (interactions_solver.cpp:89-96)
void ix_geometry(world& w, index_t i)
{
	const real_t four_thirds_pi = M_PI * 4.0 / 3.0;
	w.radius[i] = ppc_cbrt(w.vol[i] / four_thirds_pi);
	w.nrad[i] = ppc_cbrt(w.nvol[i] / four_thirds_pi);
	w.sarea[i] = 4.0 * M_PI * w.radius[i] * w.radius[i];
}

// ingest (interactions_solver.cpp:6-26,64-74,98-112)
void ix_ingest(world& w, ppc_interactions& f, index_t l, index_t r)
{
	f.cytoplasmic_fluid[l] += f.fluid[r];
	f.cytoplasmic_solid[l] += f.solid[r];
	f.fluid[l] += f.fluid[r];
	f.solid[l] += f.solid[r];
	f.cytoplasmic[l] += f.fluid[r] + f.solid[r];
	w.vol[l] += f.fluid[r] + f.solid[r];
	f.fluid_fraction[l] = f.fluid[l] / (w.vol[l] + ix_zero_threshold);
	f.cytoplasmic_to_nuclear_ratio[l] = f.cytoplasmic_solid[l] / (f.nuclear_solid[l] + ix_zero_threshold);
	const index_t S = f.substrates;
	for (index_t q = 0; q < S; q++)
		f.internalized_substrates[(size_t)l * S + q] +=
			f.internalized_substrates[(size_t)r * S + q] * f.fraction_transferred_when_ingested[(size_t)r * S + q];
	ix_geometry(w, l);
	w.flags[r] = PPC_FLAG_TO_REMOVE;
}

// fuse (interactions_solver.cpp:28-53,76-87,114-131)
void ix_fuse(world& w, ppc_interactions& f, index_t l, index_t r)
{
	const int dims = w.mesh.dims;
	const real_t both = w.vol[l] + w.vol[r];
	for (int d = 0; d < dims; d++)
		w.pos[(size_t)l * dims + d] =
			(w.pos[(size_t)l * dims + d] * w.vol[l] + w.pos[(size_t)r * dims + d] * w.vol[r]) / both;

	f.cytoplasmic_fluid[l] += f.cytoplasmic_fluid[r];
	f.nuclear_fluid[l] += f.nuclear_fluid[r];
	f.cytoplasmic_solid[l] += f.cytoplasmic_solid[r];
	f.nuclear_solid[l] += f.nuclear_solid[r];
	f.target_solid_cytoplasmic[l] += f.target_solid_cytoplasmic[r];
	f.target_solid_nuclear[l] += f.target_solid_nuclear[r];
	f.fluid[l] = f.nuclear_fluid[l] + f.cytoplasmic_fluid[l];
	f.solid[l] = f.nuclear_solid[l] + f.cytoplasmic_solid[l];
	w.nvol[l] = f.nuclear_fluid[l] + f.nuclear_solid[l];
	f.cytoplasmic[l] = f.cytoplasmic_fluid[l] + f.cytoplasmic_solid[l];
	w.vol[l] = w.nvol[l] + f.cytoplasmic[l];
	f.fluid_fraction[l] = f.fluid[l] / (w.vol[l] + ix_zero_threshold);
	f.cytoplasmic_to_nuclear_ratio[l] = f.cytoplasmic_solid[l] / (f.nuclear_solid[l] + ix_zero_threshold);

	const index_t S = f.substrates;
	for (index_t q = 0; q < S; q++)
		f.internalized_substrates[(size_t)l * S + q] += f.internalized_substrates[(size_t)r * S + q];
	ix_geometry(w, l);
	f.number_of_nuclei[l] += f.number_of_nuclei[r];
	w.flags[r] = PPC_FLAG_TO_REMOVE;
}

// update_cell_cell_interactions_internal (interactions_solver.cpp:143-251),
// serial; the mutex-guarded flag checks become plain checks. Draw k of agent
// i is uniform(seed, call, 0, i, PPC_DRAW_INTERACTION + k) instead of the
// shared generator's next number.
void cell_cell_interactions(world& w, ppc_interactions& f)
{
	const uint64_t epoch = w.ix_epoch++;
	const index_t n = w.n;
	const index_t D = w.ndefs;
	const real_t dt = w.params.mechanics_time_step;
	for (index_t i = 0; i < n; i++)
	{
		bool attacked_once = false;
		bool phagocytosed_once = false;
		bool fused_once = false;
		if (f.dead[i] == 1)
			continue;
		for (size_t k = 0; k < w.neighbors[i].size(); k++)
		{
			const index_t j = w.neighbors[i][k];
			const index_t dj = w.def[j];
			const real_t r = ppc_uniform(w.seed, epoch, 0, (uint64_t)i, PPC_DRAW_INTERACTION + (uint64_t)k);
			if (f.dead[j] == 1)
			{
				if (r < f.dead_phagocytosis_rate[i] * dt)
				{
					if (w.flags[i] == PPC_FLAG_TO_REMOVE)
						break;
					if (w.flags[j] == PPC_FLAG_TO_REMOVE)
						continue;
					ix_ingest(w, f, i, j);
				}
				continue;
			}
			if (!phagocytosed_once && r < f.live_phagocytosis_rates[(size_t)i * D + dj] * dt)
			{
				if (w.flags[i] == PPC_FLAG_TO_REMOVE)
					break;
				if (w.flags[j] == PPC_FLAG_TO_REMOVE)
					continue;
				ix_ingest(w, f, i, j);
				phagocytosed_once = true;
				continue;
			}
			{
				const real_t attack_r = f.attack_rates[(size_t)i * D + dj];
				const real_t immuno_r = f.immunogenicities[(size_t)j * D + w.def[i]];
				if (!attacked_once && r < attack_r * immuno_r * dt)
				{
					if (w.flags[i] == PPC_FLAG_TO_REMOVE)
						break;
					if (w.flags[j] == PPC_FLAG_TO_REMOVE)
						continue;
					// attack (interactions_solver.cpp:133-141)
					f.damage[j] += f.damage_rate[i] * dt;
					f.total_attack_time[j] += dt;
					attacked_once = true;
					continue;
				}
			}
			if (!fused_once && r < f.fusion_rates[(size_t)i * D + dj] * dt)
			{
				if (w.flags[i] == PPC_FLAG_TO_REMOVE)
					break;
				if (w.flags[j] == PPC_FLAG_TO_REMOVE)
					continue;
				ix_fuse(w, f, i, j);
				fused_once = true;
				continue;
			}
		}
	}
}

// simulator::simulate_mechanics (reference: src/simulator.cpp:157-196) and,
// optionally, simulator::simulate_phenotype (src/simulator.cpp:198-220)
void step_body(world& w, bool with_phenotype, double p_divide, double p_death)
{
	update_forces(w);
	// update_motility: no agent is motile on this path
	update_membrane(w);
	update_springs(w);
	update_positions(w);
	compact_mechanics(w);
	rebuild_mesh(w);
	update_neighbors(w);
	if (with_phenotype)
	{
		flag_by_draws(w, p_divide, p_death);
		compact_phenotype(w);
		rebuild_mesh(w);
		update_neighbors(w);
	}
}

template <typename T>
void put(T* dst, const std::vector<T>& src, size_t count)
{
	if (dst)
		std::memcpy(dst, src.data(), count * sizeof(T));
}

template <typename T>
void get(std::vector<T>& dst, const T* src, size_t count, T dflt)
{
	if (src)
		std::memcpy(dst.data(), src, count * sizeof(T));
	else
		std::fill(dst.begin(), dst.begin() + count, dflt);
}

} // namespace

// ppc_interactions / ppc_motility views of the resident columns
ppc_interactions ix_view(world& w)
{
	auto& x = w.ix;
	ppc_interactions v {};
	v.count = w.n;
	v.substrates = x.S;
	v.dead = x.dead.data();
	v.dead_phagocytosis_rate = x.dead_phago.data();
	v.damage_rate = x.damage_rate.data();
	v.live_phagocytosis_rates = x.live_phago.data();
	v.attack_rates = x.attack.data();
	v.fusion_rates = x.fusion.data();
	v.immunogenicities = x.immuno.data();
	v.fraction_transferred_when_ingested = x.frac.data();
	v.damage = x.damage.data();
	v.total_attack_time = x.attack_time.data();
	v.number_of_nuclei = x.nuclei.data();
	v.fluid = x.fluid.data();
	v.solid = x.solid.data();
	v.cytoplasmic = x.cyto.data();
	v.cytoplasmic_fluid = x.cyto_fluid.data();
	v.cytoplasmic_solid = x.cyto_solid.data();
	v.nuclear_fluid = x.nuc_fluid.data();
	v.nuclear_solid = x.nuc_solid.data();
	v.fluid_fraction = x.fluid_fraction.data();
	v.cytoplasmic_to_nuclear_ratio = x.c2n.data();
	v.target_solid_cytoplasmic = x.target_cyto.data();
	v.target_solid_nuclear = x.target_nuc.data();
	v.internalized_substrates = x.isub.data();
	return v;
}

ppc_motility mot_view(world& w, int32_t per_agent)
{
	auto& m = w.mot;
	ppc_motility v {};
	v.count = w.n;
	v.restrict_per_agent = per_agent ? 1 : (w.mot_per_agent ? 1 : 0);
	v.is_motile = m.motile.data();
	v.restrict_to_2d = m.restrict2d.data();
	v.persistence_time = m.persistence.data();
	v.migration_speed = m.speed.data();
	v.migration_bias = m.bias.data();
	v.migration_bias_direction = m.direction.data();
	v.motility_vector = m.vector.data();
	v.direction_rule = m.rule.data();
	v.chemotaxis_index = m.chemo_index.data();
	v.chemotaxis_direction = m.chemo_dir.data();
	v.chemotactic_sensitivities = m.sens.data();
	v.substrates = m.S;
	return v;
}

template <typename T>
void copy_col(T* dst, const T* src, size_t count)
{
	if (dst && src && count)
		std::memcpy(dst, src, count * sizeof(T));
}

// every column of `src` into `dst` (rows 0..n-1)
void copy_ix(const ppc_interactions& dst, const ppc_interactions& src, index_t n, index_t D)
{
	const size_t N = (size_t)n, S = (size_t)src.substrates;
	copy_col(const_cast<uint8_t*>(dst.dead), src.dead, N);
	copy_col(const_cast<real_t*>(dst.dead_phagocytosis_rate), src.dead_phagocytosis_rate, N);
	copy_col(const_cast<real_t*>(dst.damage_rate), src.damage_rate, N);
	copy_col(const_cast<real_t*>(dst.live_phagocytosis_rates), src.live_phagocytosis_rates, N * D);
	copy_col(const_cast<real_t*>(dst.attack_rates), src.attack_rates, N * D);
	copy_col(const_cast<real_t*>(dst.fusion_rates), src.fusion_rates, N * D);
	copy_col(const_cast<real_t*>(dst.immunogenicities), src.immunogenicities, N * D);
	copy_col(const_cast<real_t*>(dst.fraction_transferred_when_ingested), src.fraction_transferred_when_ingested, N * S);
	copy_col(dst.damage, src.damage, N);
	copy_col(dst.total_attack_time, src.total_attack_time, N);
	copy_col(dst.number_of_nuclei, src.number_of_nuclei, N);
	copy_col(dst.fluid, src.fluid, N);
	copy_col(dst.solid, src.solid, N);
	copy_col(dst.cytoplasmic, src.cytoplasmic, N);
	copy_col(dst.cytoplasmic_fluid, src.cytoplasmic_fluid, N);
	copy_col(dst.cytoplasmic_solid, src.cytoplasmic_solid, N);
	copy_col(dst.nuclear_fluid, src.nuclear_fluid, N);
	copy_col(dst.nuclear_solid, src.nuclear_solid, N);
	copy_col(dst.fluid_fraction, src.fluid_fraction, N);
	copy_col(dst.cytoplasmic_to_nuclear_ratio, src.cytoplasmic_to_nuclear_ratio, N);
	copy_col(dst.target_solid_cytoplasmic, src.target_solid_cytoplasmic, N);
	copy_col(dst.target_solid_nuclear, src.target_solid_nuclear, N);
	copy_col(dst.internalized_substrates, src.internalized_substrates, N * S);
}

void copy_mot(const ppc_motility& dst, const ppc_motility& src, index_t n, int dims)
{
	const size_t N = (size_t)n;
	copy_col(const_cast<uint8_t*>(dst.is_motile), src.is_motile, N);
	copy_col(const_cast<uint8_t*>(dst.restrict_to_2d), src.restrict_to_2d, N);
	copy_col(const_cast<real_t*>(dst.persistence_time), src.persistence_time, N);
	copy_col(const_cast<real_t*>(dst.migration_speed), src.migration_speed, N);
	copy_col(const_cast<real_t*>(dst.migration_bias), src.migration_bias, N);
	copy_col(dst.migration_bias_direction, src.migration_bias_direction, N * dims);
	copy_col(dst.motility_vector, src.motility_vector, N * dims);
	copy_col(const_cast<uint8_t*>(dst.direction_rule), src.direction_rule, N);
	copy_col(const_cast<int32_t*>(dst.chemotaxis_index), src.chemotaxis_index, N);
	copy_col(const_cast<real_t*>(dst.chemotaxis_direction), src.chemotaxis_direction, N);
	copy_col(const_cast<real_t*>(dst.chemotactic_sensitivities), src.chemotactic_sensitivities,
			 N * (size_t)std::min(dst.substrates, src.substrates));
}

struct orc_state
{
	world w;
};

extern "C" {

int orc_create(const ppc_mesh* mesh, const ppc_params* params, orc_state** out)
{
	if (!mesh || !params || !out || mesh->dims < 1 || mesh->dims > 3 || params->cell_definitions_count < 1)
		return PPC_ERR_ARG;
	auto* s = new orc_state;
	init_mesh(s->w.mesh, *mesh);
	s->w.params = *params;
	s->w.ndefs = params->cell_definitions_count;
	s->w.bins = std::make_unique<std::vector<index_t>[]>(s->w.mesh.voxels);
	s->w.bin_sizes = std::make_unique<std::atomic<index_t>[]>(s->w.mesh.voxels);
	*out = s;
	return PPC_OK;
}

void orc_destroy(orc_state* s) { delete s; }

int orc_upload(orc_state* s, const ppc_agents* a)
{
	world& w = s->w;
	const index_t n = a->count;
	const int dims = w.mesh.dims;
	w.grow(std::max<index_t>(n, 1));
	w.n = n;
	get(w.pos, a->positions, (size_t)n * dims, 0.0);
	get(w.vel, a->velocities, (size_t)n * dims, 0.0);
	get(w.vprev, a->previous_velocities, (size_t)n * dims, 0.0);
	get(w.pressure, a->simple_pressure, n, 0.0);
	get(w.radius, a->radius, n, 8.412710547954228);
	get(w.rep, a->cell_cell_repulsion_strength, n, 10.0);
	get(w.adh, a->cell_cell_adhesion_strength, n, 0.4);
	get(w.rmad, a->relative_maximum_adhesion_distance, n, 1.25);
	get(w.bm, a->cell_BM_repulsion_strength, n, 100.0);
	get(w.ec, a->attachment_elastic_constant, n, 0.01);
	get(w.arate, a->attachment_rate, n, 0.0);
	get(w.drate, a->detachment_rate, n, 0.0);
	get(w.maxatt, a->maximum_number_of_attachments, n, 12);
	get(w.aff, a->cell_adhesion_affinities, (size_t)n * w.ndefs, 1.0);
	get(w.def, a->cell_definition_indices, n, 0);
	get(w.movable, a->is_movable, n, (uint8_t)1);
	get(w.flags, a->flags, n, (uint8_t)0);
	get(w.vol, a->total_volume, n, 2494.0);
	get(w.nvol, a->nuclear_volume, n, 540.0);
	get(w.nrad, a->nuclear_radius, n, 5.051670902881889);
	get(w.sarea, a->surface_area, n, 889.3685284131693);
	get(w.polarity, a->polarity, n, 0.0);
	get(w.orient, a->orientation, (size_t)n * dims, 0.0);
	w.next_id = 0;
	for (index_t i = 0; i < n; i++)
	{
		w.ids[i] = a->agent_ids ? a->agent_ids[i] : i;
		w.next_id = std::max<int64_t>(w.next_id, w.ids[i] + 1);
		w.neighbors[i].clear();
		w.springs[i].clear();
		if (a->spring_counts && a->springs)
			for (int32_t k = 0; k < a->spring_counts[i]; k++)
				w.springs[i].push_back(a->springs[(size_t)i * a->spring_capacity + k]);
	}
	return PPC_OK;
}

int orc_download(orc_state* s, ppc_agents* a)
{
	world& w = s->w;
	const index_t n = w.n;
	const int dims = w.mesh.dims;
	a->count = n;
	if (n > a->capacity)
		return PPC_ERR_CAPACITY;
	put(a->positions, w.pos, (size_t)n * dims);
	put(a->velocities, w.vel, (size_t)n * dims);
	put(a->previous_velocities, w.vprev, (size_t)n * dims);
	put(a->simple_pressure, w.pressure, n);
	put(a->radius, w.radius, n);
	put(a->cell_cell_repulsion_strength, w.rep, n);
	put(a->cell_cell_adhesion_strength, w.adh, n);
	put(a->relative_maximum_adhesion_distance, w.rmad, n);
	put(a->cell_BM_repulsion_strength, w.bm, n);
	put(a->attachment_elastic_constant, w.ec, n);
	put(a->attachment_rate, w.arate, n);
	put(a->detachment_rate, w.drate, n);
	put(a->maximum_number_of_attachments, w.maxatt, n);
	put(a->cell_adhesion_affinities, w.aff, (size_t)n * w.ndefs);
	put(a->cell_definition_indices, w.def, n);
	put(a->is_movable, w.movable, n);
	put(a->flags, w.flags, n);
	put(a->agent_ids, w.ids, n);
	put(a->total_volume, w.vol, n);
	put(a->nuclear_volume, w.nvol, n);
	put(a->nuclear_radius, w.nrad, n);
	put(a->surface_area, w.sarea, n);
	put(a->polarity, w.polarity, n);
	put(a->orientation, w.orient, (size_t)n * dims);
	if (a->spring_counts)
	{
		for (index_t i = 0; i < n; i++)
		{
			a->spring_counts[i] = (int32_t)w.springs[i].size();
			if ((int32_t)w.springs[i].size() > a->spring_capacity)
				return PPC_ERR_CAPACITY;
			if (a->springs)
				for (size_t k = 0; k < w.springs[i].size(); k++)
					a->springs[(size_t)i * a->spring_capacity + k] = w.springs[i][k];
		}
	}
	return PPC_OK;
}

int32_t orc_count(orc_state* s) { return s->w.n; }

void orc_event_counts(orc_state* s, int64_t* divisions, int64_t* deaths)
{
	*divisions = s->w.divisions;
	*deaths = s->w.deaths;
}

void orc_set_random_seed(orc_state* s, uint64_t seed) { s->w.seed = seed; }

int64_t orc_voxel_count(orc_state* s) { return s->w.mesh.voxels; }

void orc_update_mechanics_mesh(orc_state* s) { rebuild_mesh(s->w); }
void orc_update_cell_neighbors(orc_state* s) { update_neighbors(s->w); }
void orc_update_cell_forces(orc_state* s) { update_forces(s->w); }
void orc_update_basement_membrane_interactions(orc_state* s) { update_membrane(s->w); }
void orc_update_spring_attachments(orc_state* s) { update_springs(s->w); }
void orc_update_positions(orc_state* s) { update_positions(s->w); }
void orc_update_cell_container_for_mechanics(orc_state* s) { compact_mechanics(s->w); }
void orc_flag_by_draws(orc_state* s, double p_divide, double p_death) { flag_by_draws(s->w, p_divide, p_death); }
void orc_update_cell_container_for_phenotype(orc_state* s) { compact_phenotype(s->w); }
int orc_update_motility_fields(orc_state* s, ppc_motility* f)
{
	if (!f)
	{
		if (!s->w.mot.on)
			return PPC_ERR_ARG;
		ppc_motility view = mot_view(s->w, 0);
		motility(s->w, view);
		return PPC_OK;
	}
	if (f->count != s->w.n)
		return PPC_ERR_ARG;
	motility(s->w, *f);
	return PPC_OK;
}
int orc_update_cell_cell_interactions(orc_state* s, ppc_interactions* f)
{
	if (!f)
	{
		if (!s->w.ix.on)
			return PPC_ERR_ARG;
		ppc_interactions view = ix_view(s->w);
		cell_cell_interactions(s->w, view);
		return PPC_OK;
	}
	if (f->count != s->w.n || f->substrates < 0)
		return PPC_ERR_ARG;
	cell_cell_interactions(s->w, *f);
	return PPC_OK;
}

int orc_upload_interactions(orc_state* s, const ppc_interactions* f, int32_t compute_internalized_substrates)
{
	world& w = s->w;
	if (!f || f->count != w.n || f->substrates < 0 || (w.ix.on && f->substrates != w.ix.S))
		return PPC_ERR_ARG;
	w.ix.on = true;
	w.ix.S = f->substrates;
	w.ix.halve_substrates = compute_internalized_substrates != 0;
	w.grow_stores(std::max(w.cap, 1));
	ppc_interactions v = ix_view(w);
	copy_ix(v, *f, w.n, w.ndefs);
	return PPC_OK;
}

int orc_download_interactions(orc_state* s, ppc_interactions* f)
{
	world& w = s->w;
	if (!f || !w.ix.on || f->substrates != w.ix.S)
		return PPC_ERR_ARG;
	f->count = w.n;
	ppc_interactions v = ix_view(w);
	copy_ix(*f, v, w.n, w.ndefs);
	return PPC_OK;
}

int orc_upload_motility(orc_state* s, const ppc_motility* f)
{
	world& w = s->w;
	if (!f || f->count != w.n)
		return PPC_ERR_ARG;
	const int S = f->direction_rule ? f->substrates : (w.mot.on ? w.mot.S : 0);
	if (w.mot.on && S != w.mot.S)
	{
		w.mot = world::mot_store {};
	}
	w.mot.on = true;
	w.mot.S = S;
	w.mot_per_agent = f->restrict_per_agent != 0;
	w.grow_stores(std::max(w.cap, 1));
	ppc_motility v = mot_view(w, f->restrict_per_agent);
	copy_mot(v, *f, w.n, w.mesh.dims);
	if (!f->direction_rule)
		std::fill(w.mot.rule.begin(), w.mot.rule.begin() + w.n, (uint8_t)PPC_DIRECTION_NONE);
	return PPC_OK;
}

int orc_upload_gradients(orc_state* s, const ppc_gradient_field* g)
{
	world& w = s->w;
	if (!g || g->substrates < 0 || (g->substrates > 0 && !g->gradients))
		return PPC_ERR_ARG;
	world::gradient_field f;
	f.S = g->substrates;
	size_t voxels = 1;
	for (int d = 0; d < 3; d++)
	{
		int n = 1;
		if (d < w.mesh.dims)
		{
			if (g->voxel_shape[d] <= 0)
				return PPC_ERR_ARG;
			n = (w.mesh.maxs[d] - w.mesh.mins[d] + g->voxel_shape[d] - 1) / g->voxel_shape[d];
			f.shape[d] = g->voxel_shape[d];
		}
		f.grid[d] = n < 1 ? 1 : n;
		voxels *= (size_t)f.grid[d];
	}
	f.g.assign(g->gradients, g->gradients + voxels * (size_t)f.S * 3);
	w.grad = std::move(f);
	return PPC_OK;
}

int orc_download_motility(orc_state* s, ppc_motility* f)
{
	world& w = s->w;
	if (!f || !w.mot.on)
		return PPC_ERR_ARG;
	f->count = w.n;
	ppc_motility v = mot_view(w, 0);
	copy_mot(*f, v, w.n, w.mesh.dims);
	return PPC_OK;
}


void orc_step(orc_state* s, int32_t steps, int32_t with_phenotype, double p_divide, double p_death)
{
	s->w.timed = false;
	for (int32_t k = 0; k < steps; k++)
		step_body(s->w, with_phenotype != 0, p_divide, p_death);
}

double orc_time_steps(orc_state* s, int32_t steps, int32_t threads, int32_t with_phenotype, double p_divide,
					  double p_death)
{
	world& w = s->w;
	w.timed = true;
	// reserve room for divisions so that create() rarely reallocates
	auto t0 = std::chrono::high_resolution_clock::now();
#pragma omp parallel num_threads(threads)
	{
		// reference: src/random.cpp:28-49 seeds one generator per thread
		tl_generator.seed((unsigned)(w.seed + 1 + omp_get_thread_num()));
		for (int32_t k = 0; k < steps; k++)
			step_body(w, with_phenotype != 0, p_divide, p_death);
	}
	auto t1 = std::chrono::high_resolution_clock::now();
	w.timed = false;
	return std::chrono::duration<double>(t1 - t0).count();
}

void orc_sincos(const double* theta, int32_t n, double* sn, double* cs)
{
	for (int32_t i = 0; i < n; i++)
		ppc_sincos(theta[i], sn + i, cs + i);
}

void orc_random_walk(int32_t dims, uint64_t seed, uint64_t epoch, uint64_t replicate, uint64_t slot, uint64_t k0,
					 double* w)
{
	ppc_random_walk(dims, seed, epoch, replicate, slot, k0, w);
}

double orc_uniform(uint64_t seed, uint64_t epoch, uint64_t replicate, uint64_t slot, uint64_t k)
{
	return ppc_uniform(seed, epoch, replicate, slot, k);
}

int orc_get_neighbors(orc_state* s, int32_t* counts, int32_t* lists, int32_t list_capacity)
{
	world& w = s->w;
	int rc = PPC_OK;
	for (index_t i = 0; i < w.n; i++)
	{
		counts[i] = (int32_t)w.neighbors[i].size();
		for (size_t k = 0; k < w.neighbors[i].size(); k++)
		{
			if ((int32_t)k >= list_capacity)
			{
				rc = PPC_ERR_CAPACITY;
				break;
			}
			lists[(size_t)i * list_capacity + k] = w.neighbors[i][k];
		}
	}
	return rc;
}

int orc_get_mesh_bins(orc_state* s, int32_t* voxel_counts, int32_t* agents)
{
	world& w = s->w;
	size_t o = 0;
	for (int64_t v = 0; v < w.mesh.voxels; v++)
	{
		voxel_counts[v] = (int32_t)w.bins[v].size();
		for (index_t j : w.bins[v])
			agents[o++] = j;
	}
	return PPC_OK;
}

int orc_get_mesh_position(orc_state* s, const double* position, int32_t* coords3)
{
	mesh_position(s->w.mesh, position, coords3);
	return PPC_OK;
}

} // extern "C"
