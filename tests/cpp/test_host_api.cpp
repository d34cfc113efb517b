// The reference's unit tests (test/test.cpp), rewritten against the C++ host
// layer (paraphysicell_b200/host/ppc_solver.h) so they run on the GPU path.
// Solver calls sit inside `#pragma omp parallel` exactly as in the
// reference. Prints one PASS/FAIL line per case; exit status 1 on any FAIL.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../paraphysicell_b200/host/ppc_solver.h"

using namespace physicell::b200;

static int failures = 0;

static void report(bool ok, const std::string& name)
{
	std::printf("%s %s\n", ok ? "PASS" : "FAIL", name.c_str());
	failures += ok ? 0 : 1;
}

static ppc_mesh make_mesh(int dims, int maxx, int maxy, int maxz)
{
	ppc_mesh m {};
	m.dims = dims;
	m.bounding_box_maxs[0] = maxx;
	m.bounding_box_maxs[1] = maxy;
	m.bounding_box_maxs[2] = maxz;
	m.voxel_shape[0] = m.voxel_shape[1] = m.voxel_shape[2] = 30;
	return m;
}

// update_cell_for_velocity (reference: test/test.cpp:117-134)
static void update_cell_for_velocity(environment& e, index_t i, index_t offset, index_t dims, index_t def)
{
	auto& d = e.data;
	d.cell_definition_indices[i] = def;
	d.is_movable[i] = 1;
	for (index_t k = 0; k < dims; k++)
		d.agent_data.positions[(size_t)i * dims + k] = 1 + offset + k;
	d.geometries.radius[i] = 4 + offset;
	d.mechanics.cell_cell_adhesion_strength[i] = 5 + offset;
	d.mechanics.cell_cell_repulsion_strength[i] = 6 + offset;
	d.mechanics.relative_maximum_adhesion_distance[i] = 7 + offset;
	for (index_t k = 0; k < 3; k++)
		d.mechanics.cell_adhesion_affinities[(size_t)i * 3 + k] = 8 + k + offset;
}

// host_velocity_solver.simple (reference: test/test.cpp:141-191)
static void velocity_simple(index_t dims)
{
	environment e(make_mesh(dims, 80, 80, 80), 3);
	e.data.add();
	e.data.add();
	e.data.add();
	update_cell_for_velocity(e, 0, 0, dims, 0);
	update_cell_for_velocity(e, 1, 10, dims, 1);
	for (index_t k = 0; k < dims; k++)
		e.data.agent_data.positions[2 * dims + k] = 70;

	containers_solver cs;
	cs.initialize(e);
#pragma omp parallel
	{
		cs.update_mechanics_mesh(e);
		position_solver::update_cell_neighbors(e);
		position_solver::update_cell_forces(e);
	}
	e.sync_to_host();
	const double expected = dims == 3 ? 55.61362893236258 : (dims == 2 ? 69.556601146394243 : 100.15967659502964);
	bool ok = true;
	for (index_t k = 0; k < dims; k++)
	{
		ok = ok && e.data.velocities[k] == expected;
		ok = ok && e.data.velocities[dims + k] == -expected;
		ok = ok && e.data.velocities[2 * dims + k] == 0.0;
	}
	report(ok, "host_velocity_solver.simple dims=" + std::to_string(dims));
}

// host_velocity_solver.complex neighbour counts (reference: test/test.cpp:265-320)
static void velocity_complex(index_t dims)
{
	environment e(make_mesh(dims, 80, 80, 80), 3);
	for (int k = 0; k < 3; k++)
		e.data.add();
	update_cell_for_velocity(e, 0, 0, dims, 0);
	update_cell_for_velocity(e, 1, 10, dims, 1);
	const double xs[3] = { 1, 4, 7 };
	for (index_t i = 0; i < 3; i++)
	{
		e.data.geometries.radius[i] = dims == 1 ? 2 : 4;
		e.data.mechanics.relative_maximum_adhesion_distance[i] = 1;
		for (index_t k = 0; k < dims; k++)
			e.data.agent_data.positions[(size_t)i * dims + k] = xs[i];
	}
	containers_solver cs;
	cs.initialize(e);
#pragma omp parallel
	{
		cs.update_mechanics_mesh(e);
		position_solver::update_cell_neighbors(e);
		position_solver::update_cell_forces(e);
	}
	e.sync_to_host();
	const auto& nb = e.data.states.neighbors;
	report(nb[0].size() == 1 && nb[1].size() == 2 && nb[2].size() == 1,
		   "host_velocity_solver.complex dims=" + std::to_string(dims));
}

// host_neighbors_solver.grid (reference: test/test.cpp:333-400)
static void neighbors_grid(index_t dims, index_t cells, index_t adhesion)
{
	environment e(make_mesh(dims, 200, 200, 200), 3);
	const index_t g = 7;
	const index_t gy = dims >= 2 ? g : 1, gz = dims >= 3 ? g : 1;
	for (index_t z = 0; z < gz; z++)
		for (index_t y = 0; y < gy; y++)
			for (index_t x = 0; x < g; x++)
				for (index_t c = 0; c < cells; c++)
				{
					const index_t i = e.data.add();
					const double centre[3] = { x * 30 + 15.0, y * 30 + 15.0, z * 30 + 15.0 };
					for (index_t k = 0; k < dims; k++)
						e.data.agent_data.positions[(size_t)i * dims + k] = centre[k];
					e.data.geometries.radius[i] = 9;
					e.data.mechanics.relative_maximum_adhesion_distance[i] = adhesion;
				}
	containers_solver cs;
	cs.initialize(e);
#pragma omp parallel
	cs.update_mechanics_mesh(e);
#pragma omp parallel
	position_solver::update_cell_neighbors(e);
	e.sync_to_host();
	bool ok = true;
	for (const auto& bin : e.cells_in_mechanics_voxels)
		ok = ok && (index_t)bin.size() == cells;
	for (index_t i = 0; i < e.data.agents_count; i++)
	{
		index_t c[3] = { 0, 0, 0 };
		for (index_t k = 0; k < dims; k++)
			c[k] = (index_t)(e.data.agent_data.positions[(size_t)i * dims + k] / 30);
		index_t expected = cells - 1;
		if (adhesion == 3)
			for (index_t z = -1; z <= 1; z++)
				for (index_t y = -1; y <= 1; y++)
					for (index_t x = -1; x <= 1; x++)
						if (!(c[0] + x < 0 || c[0] + x >= g || c[1] + y < 0 || c[1] + y >= gy || c[2] + z < 0
							  || c[2] + z >= gz || (x == 0 && y == 0 && z == 0)))
							expected += cells;
		ok = ok && (index_t)e.data.states.neighbors[i].size() == expected;
	}
	report(ok, "host_neighbors_solver.grid dims=" + std::to_string(dims) + " cells=" + std::to_string(cells)
				   + " adhesion=" + std::to_string(adhesion));
}

// cell_container.add_and_remove through the to_remove flag (reference: test/test.cpp:52-115)
static void container_remove()
{
	environment e(make_mesh(1, 80, 0, 0), 3);
	for (int i = 0; i < 4; i++)
	{
		const index_t k = e.data.add();
		e.data.agent_data.volumes[k] = k + 1;
		e.data.velocities[k] = 10 * (k + 1);
	}
	containers_solver cs;
	cs.initialize(e);
	e.data.flags[2] = cell_state_flag::to_remove;
	cs.update_cell_container_for_mechanics(e);
	e.sync_to_host();
	bool ok = e.data.agents_count == 3 && e.data.agent_data.volumes[2] == 4 && e.data.velocities[2] == 40;
	e.data.flags[0] = cell_state_flag::to_remove;
	cs.update_cell_container_for_mechanics(e);
	e.sync_to_host();
	ok = ok && e.data.agents_count == 2 && e.data.agent_data.volumes[0] == 4 && e.data.agent_data.volumes[1] == 2
		 && e.data.velocities[0] == 40 && e.deaths_count == 2;
	const index_t k = e.data.add();
	e.data.agent_data.volumes[k] = 5;
	ok = ok && e.data.agents_count == 3 && e.data.agent_data.volumes[2] == 5;
	report(ok, "cell_container.add_and_remove");
}

// a fused multi-step run through solver::simulate_mechanics equals the
// separate entry points called in simulator order
static void fused_equals_separate()
{
	environment a(make_mesh(3, 600, 600, 600), 1), b(make_mesh(3, 600, 600, 600), 1);
	for (environment* e : { &a, &b })
	{
		unsigned s = 7;
		for (int i = 0; i < 2000; i++)
		{
			const index_t k = e->data.add();
			for (int d = 0; d < 3; d++)
			{
				s = s * 1103515245u + 12345u;
				e->data.agent_data.positions[(size_t)k * 3 + d] = 150 + 300.0 * ((s >> 8) & 0xffff) / 65536.0;
			}
			e->data.geometries.radius[k] = 8.412710547954228;
			e->data.mechanics.cell_cell_repulsion_strength[k] = 10;
			e->data.mechanics.cell_cell_adhesion_strength[k] = 0.4;
			e->data.mechanics.relative_maximum_adhesion_distance[k] = 1.25;
			e->data.mechanics.cell_adhesion_affinities[k] = 1;
		}
	}
	solver sa, sb;
	sa.initialize(a);
	sb.initialize(b);
#pragma omp parallel
	{
		sa.containers.update_mechanics_mesh(a);
		position_solver::update_cell_neighbors(a);
		sb.containers.update_mechanics_mesh(b);
		for (int step = 0; step < 5; step++)
		{
			position_solver::update_cell_forces(a);
			position_solver::update_motility(a);
			position_solver::update_basement_membrane_interactions(a);
			position_solver::update_spring_attachments(a);
			position_solver::update_positions(a);
			sa.containers.update_cell_container_for_mechanics(a);
			sa.containers.update_mechanics_mesh(a);
			position_solver::update_cell_neighbors(a);
		}
		sb.simulate_mechanics(b, 5);
	}
	a.sync_to_host();
	b.sync_to_host();
	const bool ok = a.data.agents_count == b.data.agents_count
					&& std::memcmp(a.data.agent_data.positions.data(), b.data.agent_data.positions.data(),
								   sizeof(double) * a.data.agent_data.positions.size())
						   == 0
					&& a.data.states.neighbors == b.data.states.neighbors;
	report(ok, "solver.simulate_mechanics equals the separate entry points");
}

static void fill_ball(environment& e, int count, unsigned seed)
{
	for (int i = 0; i < count; i++)
	{
		const index_t k = e.data.add();
		for (int d = 0; d < 3; d++)
		{
			seed = seed * 1103515245u + 12345u;
			e.data.agent_data.positions[(size_t)k * 3 + d] = 150 + 300.0 * ((seed >> 8) & 0xffff) / 65536.0;
		}
		e.data.geometries.radius[k] = 8.412710547954228;
		e.data.mechanics.cell_cell_repulsion_strength[k] = 10;
		e.data.mechanics.cell_cell_adhesion_strength[k] = 0.4;
		e.data.mechanics.relative_maximum_adhesion_distance[k] = 1.25;
		e.data.mechanics.cell_adhesion_affinities[k] = 1;
		e.data.agent_data.volumes[k] = 2494;
		e.data.volumes.nuclear[k] = 540;
	}
}

static int64_t launches(environment& e)
{
	int64_t n = 0;
	check(ppc_get_launch_count(e.device, &n), "ppc_get_launch_count");
	return n;
}

// a read-only host sync keeps the device copy current, so the next solver
// call uploads nothing; a read-write sync makes it upload again; the
// trajectory is the same either way
static void residency_read_only()
{
	environment a(make_mesh(3, 600, 600, 600), 1), b(make_mesh(3, 600, 600, 600), 1);
	fill_ball(a, 1500, 11);
	fill_ball(b, 1500, 11);
	solver sa, sb;
	sa.initialize(a);
	sb.initialize(b);
	sa.containers.update_mechanics_mesh(a);
	sb.containers.update_mechanics_mesh(b);
	sa.simulate_mechanics(a, 3);
	sb.simulate_mechanics(b, 3);
	a.sync_to_host(access::read);
	const int64_t l0 = launches(a);
	sa.simulate_mechanics(a, 1);
	const int64_t quiet = launches(a) - l0;
	a.sync_to_host();
	const int64_t l1 = launches(a);
	sa.simulate_mechanics(a, 1);
	const int64_t uploaded = launches(a) - l1;
	sb.simulate_mechanics(b, 2);
	a.sync_to_host(access::read);
	b.sync_to_host(access::read);
	const bool same = a.data.agents_count == b.data.agents_count
					  && std::memcmp(a.data.agent_data.positions.data(), b.data.agent_data.positions.data(),
									 sizeof(double) * a.data.agent_data.positions.size())
							 == 0;
	report(uploaded > quiet && same, "environment.sync_to_host(access::read) keeps the device copy");
}

// flagged divisions through containers_solver with the count taken on the
// device; the state grows when the daughters exceed its capacity
static void phenotype_divisions_grow_the_state()
{
	environment e(make_mesh(3, 600, 600, 600), 1);
	fill_ball(e, 600, 5);
	solver sv;
	sv.initialize(e); // capacity 1200: twice the count
	sv.containers.update_mechanics_mesh(e);
	e.sync_to_host();
	for (index_t i = 0; i < 600; i++)
		e.data.flags[i] = cell_state_flag::to_divide;
#pragma omp parallel
	sv.containers.update_cell_container_for_phenotype(e);
	e.sync_to_host(access::read);
	bool ok = e.data.agents_count == 1200 && e.divisions_count == 600 && e.capacity > 1200;
	int64_t max_id = 0;
	for (index_t i = 0; i < e.data.agents_count; i++)
		max_id = e.data.agent_data.ids[i] > max_id ? e.data.agent_data.ids[i] : max_id;
	ok = ok && max_id == 1199;
	report(ok, "containers_solver.update_cell_container_for_phenotype counts divisions on the device");
}

int main()
{
	try
	{
		for (index_t dims = 1; dims <= 3; dims++)
		{
			velocity_simple(dims);
			velocity_complex(dims);
		}
		for (index_t dims = 1; dims <= 3; dims++)
			for (index_t cells : { 1, 5, 50 })
				for (index_t adhesion : { 1, 3 })
					neighbors_grid(dims, cells, adhesion);
		container_remove();
		fused_equals_separate();
		residency_read_only();
		phenotype_divisions_grow_the_state();
	}
	catch (const std::exception& x)
	{
		std::printf("FAIL exception: %s\n", x.what());
		return 1;
	}
	return failures == 0 ? 0 : 1;
}
