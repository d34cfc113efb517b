/*
 * ppc_oracle.h — CPU oracle for the mechanics timestep (TEST INFRASTRUCTURE).
 *
 * This library restates the reference's mechanics solver
 * (reference: src/solver/host/{common_solver,position_solver,containers_solver}.cpp,
 * solver_helper.h, interactions_solver.cpp, src/cell_data.cpp:262-313,
 * src/cell.cpp:108-163) on the CPU.
 * It exists only to check the CUDA implementation and to time the reference's
 * OpenMP structure as the CPU baseline. Only the tests, the smoke check and
 * the benchmark's CPU-baseline leg may load it; the product never does.
 *
 * Two modes share one implementation:
 *  - serial (orc_* entry points): called outside any OpenMP parallel region,
 *    every orphaned `omp for` runs on one thread, which is how the reference
 *    behaves when its solver is called outside a parallel region
 *    (reference: test/test.cpp:431-432). The result is deterministic: voxel
 *    bins hold agents in descending index order, pressure is the serial sum,
 *    removal follows ascending slots.
 *  - timed (orc_time_steps): the same functions run inside one
 *    `#pragma omp parallel` region around the step loop, like
 *    simulator::run (reference: src/simulator.cpp:302-341), with the reference's
 *    atomics, std::vector bins, per-agent std::vector neighbour lists and the
 *    random draws of the spring-attachment loop from a thread_local mt19937.
 *
 * Parity status: pinned against the reference's known-answer and
 * brute-force tests (test/test.cpp:52-115,141-191,193-320,333-400), which the
 * Python tests re-express. The mesh rounding rules of the absent paraBioFVM
 * dependency (voxel_position truncation, grid_shape ceiling) are assumptions
 * shared by oracle and device and are not pinned by any reference test.
 */
#ifndef PPC_ORACLE_H
#define PPC_ORACLE_H

#include "../include/ppc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

int orc_create(const ppc_mesh* mesh, const ppc_params* params, orc_state** out);
void orc_destroy(orc_state* s);
int orc_upload(orc_state* s, const ppc_agents* a);
int orc_download(orc_state* s, ppc_agents* a);
int32_t orc_count(orc_state* s);
void orc_event_counts(orc_state* s, int64_t* divisions, int64_t* deaths);
void orc_set_random_seed(orc_state* s, uint64_t seed);
int64_t orc_voxel_count(orc_state* s);

/* reference entry points, serial */
void orc_update_mechanics_mesh(orc_state* s);
void orc_update_cell_neighbors(orc_state* s);
void orc_update_cell_forces(orc_state* s);
void orc_update_basement_membrane_interactions(orc_state* s);
void orc_update_spring_attachments(orc_state* s);
void orc_update_positions(orc_state* s);
void orc_update_cell_container_for_mechanics(orc_state* s);
void orc_flag_by_draws(orc_state* s, double p_divide, double p_death);
void orc_update_cell_container_for_phenotype(orc_state* s);
/* interactions_solver::update_cell_cell_interactions; `fields` rows follow
   the oracle's agent order */
int orc_update_cell_cell_interactions(orc_state* s, ppc_interactions* fields);
/* position_solver::update_motility with motile agents */
int orc_update_motility_fields(orc_state* s, ppc_motility* fields);
/* resident phenotype columns (fields == NULL in the two calls above uses
   them): they move with their agent on removal and division halves, copies
   and resets them like cell::divide */
int orc_upload_interactions(orc_state* s, const ppc_interactions* fields, int32_t compute_internalized_substrates);
int orc_download_interactions(orc_state* s, ppc_interactions* fields);
int orc_upload_motility(orc_state* s, const ppc_motility* fields);
int orc_download_motility(orc_state* s, ppc_motility* fields);
/* the gradient field the chemotaxis direction rules read */
int orc_upload_gradients(orc_state* s, const ppc_gradient_field* field);

/* one mechanics step in simulator::simulate_mechanics order, `steps` times;
   with_phenotype adds flag_by_draws + the phenotype container update +
   mesh and neighbour rebuild after each step (simulator::simulate_phenotype) */
void orc_step(orc_state* s, int32_t steps, int32_t with_phenotype, double p_divide, double p_death);

/* same steps inside one OpenMP parallel region with `threads` threads;
   returns the wall time in seconds (std::chrono around the step loop) */
double orc_time_steps(orc_state* s, int32_t steps, int32_t threads, int32_t with_phenotype, double p_divide,
					  double p_death);

/* the draws header's sine/cosine and random walk evaluated on the host, for
   the tests that pin them against libm and the reference's construction */
void orc_sincos(const double* theta, int32_t n, double* sn, double* cs);
void orc_random_walk(int32_t dims, uint64_t seed, uint64_t epoch, uint64_t replicate, uint64_t slot, uint64_t k0,
					 double* w);
double orc_uniform(uint64_t seed, uint64_t epoch, uint64_t replicate, uint64_t slot, uint64_t k);

/* readback */
int orc_get_neighbors(orc_state* s, int32_t* counts, int32_t* lists, int32_t list_capacity);
int orc_get_mesh_bins(orc_state* s, int32_t* voxel_counts, int32_t* agents);
int orc_get_mesh_position(orc_state* s, const double* position, int32_t* coords3);

#ifdef __cplusplus
}
#endif

#endif
