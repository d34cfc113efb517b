// ppc_solver.h — C++ host layer over the C ABI (include/ppc.h) with the
// reference's solver interface.
//
// Mirrors the mechanics-path API of paraPhysiCell so that code written
// against it keeps its calls:
//   physicell::b200::position_solver::update_cell_forces(e) etc.
//     (reference: src/solver/host/position_solver.h:7-21)
//   physicell::b200::containers_solver{initialize, update_mechanics_mesh,
//     update_cell_container_for_mechanics, update_cell_container_for_phenotype}
//     (reference: src/solver/host/containers_solver.h:13-27)
//   physicell::b200::solver{position, containers, initialize}
//     (reference: src/solver/solver.h:9-17)
// The state types keep the reference's field names and nesting
// (`e.data.mechanics.cell_cell_adhesion_strength`, `e.data.states.neighbors`,
// `e.cells_in_mechanics_voxels`, ...; reference src/cell_data.h,
// src/environment.h) for the fields the mechanics path uses.
//
// Residency follows the pattern the reference's simulator uses for BioFVM's
// device solver (src/simulator.cpp:95-118), with one state more: after a
// solver call the agents live on the GPU; host code that reads `e.data` calls
// `e.sync_to_host(access::read)` first (both copies are then current and the
// next solver call uploads nothing), host code that also writes it calls
// `e.sync_to_host()` (access::read_write, the default) or, after a read sync,
// `e.host_modified()`, and the next solver call uploads the host data.
//
// Threading: like the reference, every entry point may be called by all
// threads of an enclosing `omp parallel` region (src/simulator.cpp:302) or
// outside any region; inside a region one thread issues the GPU work
// (`omp single`, with its implicit barrier).
//
// Errors: the reference's entry points return nothing and check nothing;
// these throw std::runtime_error with the library's message instead of
// continuing on a failed call.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
	#include <omp.h>
#endif

#include "../../include/ppc.h"

namespace physicell {
namespace b200 {

using real_t = double;
using index_t = int32_t;

inline void check(int rc, const char* what)
{
	if (rc != PPC_OK)
		throw std::runtime_error(std::string(what) + " failed (status " + std::to_string(rc) + "): " + ppc_last_error());
}

// runs f once per OpenMP team (or directly outside a parallel region)
template <typename F>
inline void once_per_team(F&& f)
{
#ifdef _OPENMP
	if (omp_in_parallel())
	{
		std::string err;
	#pragma omp single copyprivate(err)
		{
			try
			{
				f();
			}
			catch (const std::exception& x)
			{
				err = x.what();
			}
		}
		if (!err.empty())
			throw std::runtime_error(err);
		return;
	}
#endif
	f();
}

enum class cell_state_flag : uint8_t
{
	none = PPC_FLAG_NONE,
	to_remove = PPC_FLAG_TO_REMOVE,
	to_divide = PPC_FLAG_TO_DIVIDE
};

// The mechanics fields of the reference's cell_data (src/cell_data.h:59-196).
struct cell_data
{
	index_t agents_count = 0;
	index_t dims = 3;
	index_t cell_definitions_count = 1;

	struct
	{
		std::vector<real_t> positions; // [agents*dims]
		std::vector<real_t> volumes;   // total volume
		std::vector<int64_t> ids;
	} agent_data;
	struct
	{
		std::vector<real_t> nuclear;
	} volumes;
	struct
	{
		std::vector<real_t> radius, nuclear_radius, surface_area, polarity;
	} geometries;
	struct
	{
		std::vector<real_t> cell_cell_adhesion_strength, cell_cell_repulsion_strength, cell_BM_repulsion_strength,
			cell_adhesion_affinities, relative_maximum_adhesion_distance, attachment_elastic_constant,
			attachment_rate, detachment_rate;
		std::vector<index_t> maximum_number_of_attachments;
	} mechanics;
	struct
	{
		std::vector<std::vector<index_t>> neighbors, springs;
		std::vector<real_t> orientation, simple_pressure;
	} states;
	std::vector<real_t> previous_velocities, velocities;
	std::vector<index_t> cell_definition_indices;
	std::vector<uint8_t> is_movable;
	std::vector<cell_state_flag> flags;

	// Appends one agent the way `cell_container::create()` does: zero
	// velocities, is_movable = true, default state, zero-initialised
	// phenotype (reference: src/cell.cpp:47-61, src/phenotype.cpp:6-16).
	index_t add()
	{
		const index_t i = agents_count++;
		for (auto* v : { &agent_data.positions, &previous_velocities, &velocities, &states.orientation })
			v->resize((size_t)agents_count * dims, 0.0);
		for (auto* v : { &agent_data.volumes, &volumes.nuclear, &geometries.radius, &geometries.nuclear_radius,
						 &geometries.surface_area, &geometries.polarity, &mechanics.cell_cell_adhesion_strength,
						 &mechanics.cell_cell_repulsion_strength, &mechanics.cell_BM_repulsion_strength,
						 &mechanics.relative_maximum_adhesion_distance, &mechanics.attachment_elastic_constant,
						 &mechanics.attachment_rate, &mechanics.detachment_rate, &states.simple_pressure })
			v->resize(agents_count, 0.0);
		mechanics.cell_adhesion_affinities.resize((size_t)agents_count * cell_definitions_count, 0.0);
		mechanics.maximum_number_of_attachments.resize(agents_count, 0);
		cell_definition_indices.resize(agents_count, 0);
		is_movable.resize(agents_count, 1);
		flags.resize(agents_count, cell_state_flag::none);
		states.neighbors.resize(agents_count);
		states.springs.resize(agents_count);
		agent_data.ids.resize(agents_count);
		agent_data.ids[i] = next_id++;
		return i;
	}

	int64_t next_id = 0;
};

// The agents of each mechanics voxel, in bin order, as a contiguous index
// table: bins[v] is a read-only range with size(), begin(), end() and
// operator[] like the reference's std::vector<index_t> per voxel
// (environment::cells_in_mechanics_voxels, src/environment.h:44), without
// one heap vector per voxel.
class voxel_bins
{
public:
	struct range
	{
		const index_t* b;
		const index_t* e;
		size_t size() const { return (size_t)(e - b); }
		bool empty() const { return b == e; }
		const index_t* begin() const { return b; }
		const index_t* end() const { return e; }
		index_t operator[](size_t k) const { return b[k]; }
	};
	struct iterator
	{
		const voxel_bins* bins;
		size_t v;
		range operator*() const { return (*bins)[v]; }
		iterator& operator++()
		{
			++v;
			return *this;
		}
		bool operator!=(const iterator& o) const { return v != o.v; }
	};

	size_t size() const { return start.empty() ? 0 : start.size() - 1; }
	range operator[](size_t v) const { return { agents.data() + start[v], agents.data() + start[v + 1] }; }
	iterator begin() const { return { this, 0 }; }
	iterator end() const { return { this, size() }; }

	// voxel_counts[v] agents per voxel, the agents concatenated in voxel order
	void assign(const std::vector<int32_t>& voxel_counts, std::vector<int32_t>&& concatenated)
	{
		start.assign(voxel_counts.size() + 1, 0);
		for (size_t v = 0; v < voxel_counts.size(); v++)
			start[v + 1] = start[v] + voxel_counts[v];
		agents = std::move(concatenated);
	}

private:
	std::vector<int64_t> start;
	std::vector<index_t> agents;
};

enum class access
{
	read,	   // host code only reads e.data: the device copy stays current
	read_write // host code may change e.data: the next solver call uploads it
};

// The mechanics part of the reference's environment (src/environment.h:12-60).
struct environment
{
	// `mesh`: the domain's bounding box and the mechanics voxel shape
	// (30 um by default in the reference, src/environment.h:10)
	environment(const ppc_mesh& mesh, index_t cell_definitions_count, real_t mechanics_time_step = 0.1)
		: mechanics_mesh(mesh), mechanics_time_step(mechanics_time_step), cell_definitions_count(cell_definitions_count)
	{
		data.dims = mesh.dims;
		data.cell_definitions_count = cell_definitions_count;
	}
	environment(const environment&) = delete;
	environment& operator=(const environment&) = delete;
	~environment()
	{
		if (device)
			ppc_destroy(device);
	}

	ppc_mesh mechanics_mesh;
	bool virtual_wall_at_domain_edges = false;
	bool automated_spring_adhesion = true;
	int64_t divisions_count = 0;
	int64_t deaths_count = 0;
	real_t mechanics_time_step;
	index_t cell_definitions_count;
	uint64_t random_seed = 0;

	voxel_bins cells_in_mechanics_voxels; // filled by sync_to_host
	cell_data data;

	// ---- residency ----
	ppc_state* device = nullptr;
	bool device_current = false; // the GPU holds the latest agent data
	bool host_current = true;	 // e.data holds the latest agent data
	index_t capacity = 0;
	int32_t neighbor_capacity = 64; // per-agent list length on the device; grows on demand
	int64_t divisions_base = 0, deaths_base = 0; // events of device states replaced by a larger one

	// the reference's neighbour lists are unbounded vectors: grow the device
	// lists until every list fits
	void update_neighbors_growing()
	{
		int rc = ppc_update_cell_neighbors(device);
		while (rc == PPC_ERR_CAPACITY && neighbor_capacity < (1 << 16))
		{
			neighbor_capacity *= 4;
			check(ppc_set_neighbor_capacity(device, neighbor_capacity), "ppc_set_neighbor_capacity");
			rc = ppc_update_cell_neighbors(device);
		}
		check(rc, "ppc_update_cell_neighbors");
	}

	ppc_params params() const
	{
		ppc_params p {};
		p.mechanics_time_step = mechanics_time_step;
		p.cell_definitions_count = cell_definitions_count;
		p.virtual_wall_at_domain_edges = virtual_wall_at_domain_edges;
		p.automated_spring_adhesion = automated_spring_adhesion;
		return p;
	}

	// (re)creates the device state with room for `want` agents
	void ensure_state(index_t want)
	{
		if (device && want <= capacity)
			return;
		if (device)
		{
			sync_to_host();
			// the new state's event counters start from zero
			divisions_base = divisions_count;
			deaths_base = deaths_count;
			ppc_destroy(device);
			device = nullptr;
		}
		capacity = want < 1024 ? 1024 : want;
		const ppc_params p = params();
		check(ppc_create(&mechanics_mesh, &p, capacity, &device), "ppc_create");
		check(ppc_set_random_seed(device, random_seed), "ppc_set_random_seed");
		check(ppc_set_neighbor_capacity(device, neighbor_capacity), "ppc_set_neighbor_capacity");
		device_current = false;
	}

	ppc_agents view(bool with_springs, std::vector<int32_t>& counts, std::vector<int32_t>& rows)
	{
		ppc_agents a {};
		a.count = data.agents_count;
		a.capacity = data.agents_count;
		a.positions = data.agent_data.positions.data();
		a.velocities = data.velocities.data();
		a.previous_velocities = data.previous_velocities.data();
		a.simple_pressure = data.states.simple_pressure.data();
		a.radius = data.geometries.radius.data();
		a.cell_cell_repulsion_strength = data.mechanics.cell_cell_repulsion_strength.data();
		a.cell_cell_adhesion_strength = data.mechanics.cell_cell_adhesion_strength.data();
		a.relative_maximum_adhesion_distance = data.mechanics.relative_maximum_adhesion_distance.data();
		a.cell_BM_repulsion_strength = data.mechanics.cell_BM_repulsion_strength.data();
		a.attachment_elastic_constant = data.mechanics.attachment_elastic_constant.data();
		a.attachment_rate = data.mechanics.attachment_rate.data();
		a.detachment_rate = data.mechanics.detachment_rate.data();
		a.maximum_number_of_attachments = data.mechanics.maximum_number_of_attachments.data();
		a.cell_adhesion_affinities = data.mechanics.cell_adhesion_affinities.data();
		a.cell_definition_indices = data.cell_definition_indices.data();
		a.is_movable = data.is_movable.data();
		a.flags = reinterpret_cast<uint8_t*>(data.flags.data());
		a.agent_ids = data.agent_data.ids.data();
		a.total_volume = data.agent_data.volumes.data();
		a.nuclear_volume = data.volumes.nuclear.data();
		a.nuclear_radius = data.geometries.nuclear_radius.data();
		a.surface_area = data.geometries.surface_area.data();
		a.polarity = data.geometries.polarity.data();
		a.orientation = data.states.orientation.data();
		a.spring_capacity = 12;
		if (with_springs)
		{
			counts.assign(data.agents_count, 0);
			rows.assign((size_t)data.agents_count * 12, -1);
			for (index_t i = 0; i < data.agents_count; i++)
			{
				const auto& s = data.states.springs[i];
				if (s.size() > 12)
					throw std::runtime_error("more than 12 springs on one agent");
				counts[i] = (int32_t)s.size();
				for (size_t k = 0; k < s.size(); k++)
					rows[(size_t)i * 12 + k] = s[k];
			}
			a.spring_counts = counts.data();
			a.springs = rows.data();
		}
		return a;
	}

	// host -> device when the host holds the latest data; afterwards the device
	// work makes the host copy stale
	void sync_to_device()
	{
		ensure_state(data.agents_count * 2);
		if (!device_current)
		{
			std::vector<int32_t> counts, rows;
			ppc_agents a = view(true, counts, rows);
			check(ppc_upload(device, 0, &a), "ppc_upload");
			device_current = true;
		}
		host_current = false;
	}

	// host code changed e.data after a read-only sync: the next solver call
	// uploads it
	void host_modified() { device_current = false; }

	// device -> host (counterpart of simulator::sync_data_host); also fills
	// states.neighbors and cells_in_mechanics_voxels. With access::read the
	// device copy stays current, so the next solver call uploads nothing.
	void sync_to_host(access mode = access::read_write)
	{
		if (device && device_current && !host_current)
			download_all();
		if (mode == access::read_write)
			device_current = false;
	}

private:
	void download_all()
	{
		int32_t n = 0;
		check(ppc_get_count(device, 0, &n), "ppc_get_count");
		data.agents_count = n;
		const index_t keep = n;
		data.agents_count = 0;
		data.next_id = 0;
		while (data.agents_count < keep)
			data.add();
		std::vector<int32_t> counts, rows;
		ppc_agents a = view(false, counts, rows);
		counts.assign(n, 0);
		rows.assign((size_t)n * 12, -1);
		a.spring_counts = counts.data();
		a.springs = rows.data();
		check(ppc_download(device, 0, &a), "ppc_download");
		for (index_t i = 0; i < n; i++)
		{
			data.states.springs[i].assign(rows.begin() + (size_t)i * 12, rows.begin() + (size_t)i * 12 + counts[i]);
			data.next_id = data.agent_data.ids[i] + 1 > data.next_id ? data.agent_data.ids[i] + 1 : data.next_id;
		}
		for (;;)
		{
			const int32_t cap = neighbor_capacity;
			std::vector<int32_t> nc(n > 0 ? n : 1), nl((size_t)(n > 0 ? n : 1) * cap);
			const int rc = ppc_get_neighbors(device, 0, nc.data(), nl.data(), cap);
			if (rc == PPC_ERR_CAPACITY && neighbor_capacity < (1 << 16))
			{
				neighbor_capacity *= 4;
				check(ppc_set_neighbor_capacity(device, neighbor_capacity), "ppc_set_neighbor_capacity");
				update_neighbors_growing();
				continue;
			}
			check(rc, "ppc_get_neighbors");
			for (index_t i = 0; i < n; i++)
				data.states.neighbors[i].assign(nl.begin() + (size_t)i * cap, nl.begin() + (size_t)i * cap + nc[i]);
			break;
		}
		int64_t voxels = 0;
		check(ppc_get_voxel_count(device, 0, &voxels), "ppc_get_voxel_count");
		std::vector<int32_t> vc(voxels), va(n > 0 ? n : 1);
		check(ppc_get_mesh_bins(device, 0, vc.data(), va.data()), "ppc_get_mesh_bins");
		va.resize(n);
		cells_in_mechanics_voxels.assign(vc, std::move(va));
		check(ppc_get_event_counts(device, 0, &divisions_count, &deaths_count), "ppc_get_event_counts");
		divisions_count += divisions_base;
		deaths_count += deaths_base;
		host_current = true;
	}
};

// reference: src/solver/host/position_solver.h:7-21
class position_solver
{
	template <typename F>
	static void on_device(environment& e, F&& f)
	{
		once_per_team([&] {
			e.sync_to_device();
			f();
		});
	}

public:
	static void update_cell_forces(environment& e)
	{
		on_device(e, [&] { check(ppc_update_cell_forces(e.device), "ppc_update_cell_forces"); });
	}
	static void update_cell_neighbors(environment& e)
	{
		on_device(e, [&] { e.update_neighbors_growing(); });
	}
	static void update_motility(environment& e)
	{
		on_device(e, [&] { check(ppc_update_motility(e.device), "ppc_update_motility"); });
	}
	static void update_basement_membrane_interactions(environment& e)
	{
		on_device(e, [&] {
			check(ppc_update_basement_membrane_interactions(e.device), "ppc_update_basement_membrane_interactions");
		});
	}
	static void update_spring_attachments(environment& e)
	{
		on_device(e, [&] { check(ppc_update_spring_attachments(e.device), "ppc_update_spring_attachments"); });
	}
	static void update_positions(environment& e)
	{
		on_device(e, [&] { check(ppc_update_positions(e.device), "ppc_update_positions"); });
	}
};

// reference: src/solver/host/containers_solver.h:13-27
class containers_solver
{
public:
	void initialize(environment& e)
	{
		once_per_team([&] { e.ensure_state(e.data.agents_count * 2); });
	}
	void update_mechanics_mesh(environment& e)
	{
		once_per_team([&] {
			e.sync_to_device();
			check(ppc_update_mechanics_mesh(e.device), "ppc_update_mechanics_mesh");
		});
	}
	void update_cell_container_for_mechanics(environment& e)
	{
		once_per_team([&] {
			e.sync_to_device();
			check(ppc_update_cell_container_for_mechanics(e.device), "ppc_update_cell_container_for_mechanics");
		});
	}
	// without BioFVM's release_internalized_substrates; the dividing agents
	// are counted on the device, and the state grows (through the host) only
	// when their daughters would exceed its capacity
	void update_cell_container_for_phenotype(environment& e)
	{
		once_per_team([&] {
			e.sync_to_device();
			int32_t dividing = 0, n = 0;
			check(ppc_count_flags(e.device, 0, PPC_FLAG_TO_DIVIDE, &dividing), "ppc_count_flags");
			check(ppc_get_count(e.device, 0, &n), "ppc_get_count");
			if (n + dividing + 1 > e.capacity)
			{
				e.ensure_state(n + dividing + 1);
				e.sync_to_device();
			}
			check(ppc_update_cell_container_for_phenotype(e.device), "ppc_update_cell_container_for_phenotype");
		});
	}
};

// reference: src/solver/solver.h:9-17
class solver
{
public:
	position_solver position;
	containers_solver containers;

	void initialize(environment& e) { containers.initialize(e); }

	// simulator::simulate_mechanics (reference: src/simulator.cpp:157-196)
	// for `steps` steps in one fused, graph-replayed device call
	void simulate_mechanics(environment& e, int32_t steps = 1)
	{
		once_per_team([&] {
			e.sync_to_device();
			check(ppc_step(e.device, steps), "ppc_step");
			check(ppc_synchronize(e.device), "ppc_synchronize");
		});
	}
};

} // namespace b200
} // namespace physicell
