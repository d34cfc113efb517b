/*
 * ppc.h — C ABI of the B200 mechanics timestep of paraPhysiCell.
 *
 * Every entry point replaces one reference solver entry point that takes
 * `physicell::environment&` (reference: src/solver/host/position_solver.h:7-21,
 * src/solver/host/containers_solver.h:13-27, src/solver/solver.h:9-17). The
 * reference functions are `void` and run inside an enclosing `omp parallel`
 * region; these return an int status (PPC_OK on success) and must be called
 * once per simulation step from one host thread (the C++ layer in
 * paraphysicell_b200/host wraps them in `omp single` where needed).
 *
 * Agent state lives in device memory (HBM) inside a `ppc_state` between calls.
 * Host buffers enter through ppc_upload and leave through ppc_download; the
 * struct `ppc_agents` mirrors the structure-of-arrays fields of the reference's
 * `physicell::cell_data` that the mechanics step reads or writes
 * (reference: src/cell_data.h:59-79,137-196). All pointers in `ppc_agents` are
 * plain host pointers; no CUDA or torch types appear in any signature.
 *
 * Threading: a ppc_state is not thread safe; calls on one state must be
 * serialised by the caller. Device work is issued on the state's stream
 * (ppc_set_stream) and every call returns once the work is enqueued, except
 * calls that return data or a status that depends on device results, which
 * synchronise the stream.
 */
#ifndef PPC_H
#define PPC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PPC_ABI_VERSION 2

/* Status codes. The reference has no error reporting (all entry points are
 * void); these are new. */
enum ppc_status
{
	PPC_OK = 0,
	PPC_ERR_ARG = 1,		 /* invalid argument (null handle, bad dims, ...) */
	PPC_ERR_CUDA = 2,		 /* a CUDA runtime call failed */
	PPC_ERR_CAPACITY = 3,	 /* agent, neighbour or spring capacity exceeded */
	PPC_ERR_NONFINITE = 4,	 /* a position is NaN or infinite */
	PPC_ERR_TIMEOUT = 5,	 /* a bounded device wait gave up */
	PPC_ERR_UNSUPPORTED = 6, /* feature not implemented on the device path */
	PPC_ERR_OUT_OF_MESH = 7, /* an agent lies outside the mechanics mesh when binned */
	PPC_ERR_NO_DEVICE = 8	 /* no CUDA device is available */
};

/* Cell state flags (reference: src/cell_data.h:155-160, enum cell_state_flag). */
enum ppc_flag
{
	PPC_FLAG_NONE = 0,
	PPC_FLAG_TO_REMOVE = 1,
	PPC_FLAG_TO_DIVIDE = 2
};

/* Arithmetic used for the pairwise cell-cell forces. */
enum ppc_precision
{
	PPC_FP64 = 0,		/* every operation in FP64, bit-faithful to the reference */
	PPC_FP32_FORCE = 1	/* pair force arithmetic in FP32 with compensated sums;
						   positions, binning, neighbour sets and integration stay FP64 */
};

/*
 * Domain and mechanics mesh. The reference's mechanics mesh shares the
 * bounding box of the diffusion mesh and uses 30 um voxels by default
 * (reference: src/environment.cpp:16, src/environment.h:10). The bounding box
 * is integer, as in the reference's builder (src/builder.cpp:84-105).
 * grid_shape[d] = ceil((max-min)/voxel_shape) for d < dims, 1 otherwise.
 */
typedef struct ppc_mesh
{
	int32_t dims; /* 1, 2 or 3 */
	int32_t bounding_box_mins[3];
	int32_t bounding_box_maxs[3];
	int32_t voxel_shape[3]; /* mechanics voxel edge lengths (um) */
} ppc_mesh;

/* Per-environment switches (reference: src/environment.h:30-46). */
typedef struct ppc_params
{
	double mechanics_time_step;			  /* e.mechanics_time_step (min) */
	int32_t cell_definitions_count;		  /* e.cell_definitions_count */
	int32_t virtual_wall_at_domain_edges; /* e.virtual_wall_at_domain_edges */
	int32_t automated_spring_adhesion;	  /* e.automated_spring_adhesion */
	int32_t reserved;
} ppc_params;

/*
 * Host view of the agents of one simulation (structure of arrays, host memory).
 * Positions, velocities, previous velocities and orientation are AoS by dims,
 * exactly like the reference (`positions[i*dims+d]`). Any pointer may be NULL:
 * on upload the field then takes the reference's default
 * (src/data_storage_phenotype.cpp:120-125,194-214, src/cell.cpp:47-61);
 * on download it is skipped.
 * `count` is the number of agents; `capacity` is how many agents the arrays can
 * hold (used by ppc_download; on upload it must be >= count).
 */
typedef struct ppc_agents
{
	int32_t count;
	int32_t capacity;

	double* positions;			 /* [capacity*dims] */
	double* velocities;			 /* [capacity*dims] */
	double* previous_velocities; /* [capacity*dims] */
	double* simple_pressure;	 /* [capacity] */

	double* radius;								/* geometries.radius */
	double* cell_cell_repulsion_strength;		/* mechanics.* */
	double* cell_cell_adhesion_strength;
	double* relative_maximum_adhesion_distance;
	double* cell_BM_repulsion_strength;
	double* attachment_elastic_constant;
	double* attachment_rate;
	double* detachment_rate;
	int32_t* maximum_number_of_attachments;
	double* cell_adhesion_affinities; /* [capacity*cell_definitions_count], row per agent */

	int32_t* cell_definition_indices;
	uint8_t* is_movable;
	uint8_t* flags; /* enum ppc_flag */
	int64_t* agent_ids;

	/* fields that division reads or writes (reference: src/cell.cpp:108-163) */
	double* total_volume;	/* agent_data.volumes */
	double* nuclear_volume; /* volumes.nuclear */
	double* nuclear_radius;
	double* surface_area;
	double* polarity;
	double* orientation; /* [capacity*dims] */

	/* spring attachments, one row of `spring_capacity` slots per agent
	   (reference: states.springs, vector<vector<index_t>>) */
	int32_t spring_capacity;
	int32_t* spring_counts; /* [capacity] */
	int32_t* springs;		/* [capacity*spring_capacity] */
} ppc_agents;

typedef struct ppc_state ppc_state;

/* ---- lifetime ----------------------------------------------------------- */

/* Creates the device state of one simulation (counterpart of constructing the
 * environment plus `solver::initialize`, reference src/solver/solver.cpp:5 and
 * src/solver/host/containers_solver.cpp:10-13). `agent_capacity` bounds the
 * agent count reachable by division. */
int ppc_create(const ppc_mesh* mesh, const ppc_params* params, int32_t agent_capacity, ppc_state** out);

/* Creates a batch of `replicates` independent simulations advanced together
 * (ensemble form; no reference counterpart: the reference runs one
 * environment per process). meshes[r] and capacities[r] describe replicate r;
 * all replicates share `params`. */
int ppc_create_batch(const ppc_mesh* meshes, const int32_t* capacities, int32_t replicates, const ppc_params* params,
					 ppc_state** out);

int ppc_destroy(ppc_state* s);

/* Sets the CUDA stream (a cudaStream_t passed as void*) used for all device
 * work of this state; NULL selects the state's own stream. */
int ppc_set_stream(ppc_state* s, void* cuda_stream);

/* Arithmetic of the fused force pass (enum ppc_precision). Steps with
 * non-zero spring attachment or detachment rates run the separate FP64
 * kernels whatever the setting. */
int ppc_set_precision(ppc_state* s, int32_t precision);

/* Seed of the counter-based random stream that replaces the reference's
 * per-thread mt19937 (src/random.cpp:8-49) for division directions. */
int ppc_set_random_seed(ppc_state* s, uint64_t seed);

/* Launch shape of the fused force pass, one thread per agent in every shape:
 *  -4 (the default): a warp lays its 32 agents' candidates end to end and
 *     every lane takes every 32nd of them, so the filter and the pair code run
 *     on full warps however unevenly the candidates fall; each agent's lane
 *     adds its own pair terms in its candidate order — best where agents are
 *     sparse (well under one per voxel); `threads` and `smem_bytes` are
 *     ignored (128 threads);
 *  -3: each thread numbers its candidates in the reference's order and
 *     fetches their single-precision positions ten at a time into shared
 *     memory with asynchronous copies, then the FP64 data of the kept ones two
 *     at a time (128 threads);
 *  -1: each thread reads its candidates one at a time from global memory and
 *     runs its own pair code;
 *  -2: the pair code of a warp's kept candidates is spread over the warp's
 *     32 lanes, candidates read from global memory — best where agents are
 *     dense (several per voxel);
 *   0: as -2, with each block's candidate ranges staged in `smem_bytes` of
 *     shared memory (32 KiB is a good budget; a block whose ranges do not fit
 *     reads global memory).
 * `threads` per block 32..256, a multiple of 32 (the fused pass uses at most
 * 128). Results do not depend on the shape; ppc_autotune picks one. */
int ppc_set_launch_shape(ppc_state* s, int32_t tile_edge, int32_t threads, int32_t smem_bytes);

/* How ppc_step runs a mechanics step (ppc_step_with_phenotype and steps with
 * non-zero spring rates always use the separate kernels). */
enum ppc_step_form
{
	PPC_STEP_KERNELS = 0,	 /* the default: the fused pass, the compaction plan and
								the three mesh-rebuild kernels (count, order,
								copy), five launches */
	PPC_STEP_PERSISTENT = 1	 /* one cooperative launch: the same phases over all
								replicates, separated by grid barriers */
};
int ppc_set_step_form(ppc_state* s, int32_t form);

/* Bound of every device-side wait (the persistent step's grid barriers), in
 * polls of about 64 ns each; the default 2^25 is about two seconds. A wait
 * that runs out leaves the step incomplete: the next synchronising call
 * returns PPC_ERR_TIMEOUT, later persistent steps do nothing until then, and
 * ppc_step refuses to run until the state is uploaded again. */
int ppc_set_wait_limit(ppc_state* s, int64_t polls);

/* Autotuner of the launch shape (no counterpart in the reference, whose
 * OpenMP loops have no launch shape): runs 2 x `steps` mechanics steps
 * (ppc_step) with each candidate shape — -4, -3, -1 and -2 with 128 threads,
 * 0 with 128 threads / 32 KiB and with 64 threads / 16 KiB — times the second
 * half of each on the state's stream, and keeps the fastest. The simulation
 * advances by 12 x `steps` steps (the trajectory does not depend on the
 * shape). Writes the chosen shape to `tile_edge` and `threads` when they are
 * not NULL. */
int ppc_autotune(ppc_state* s, int32_t steps, int32_t* tile_edge, int32_t* threads);

/* Neighbour-list capacity per agent for ppc_update_cell_neighbors (default 64). */
int ppc_set_neighbor_capacity(ppc_state* s, int32_t per_agent);

/* ---- host <-> device ---------------------------------------------------- */

/* Replaces the agents of replicate `replicate` (0 for ppc_create states) with
 * the host view. Synchronises the stream. */
int ppc_upload(ppc_state* s, int32_t replicate, const ppc_agents* agents);

/* Copies the agents of replicate `replicate` back to the host view. Sets
 * agents->count; returns PPC_ERR_CAPACITY if it exceeds agents->capacity.
 * Synchronises the stream, once when the count has not grown since the
 * state last reported it (the copies are queued with that count, next to the
 * counters); rows past the new count but within the last reported count and
 * agents->capacity may then be overwritten. */
int ppc_download(ppc_state* s, int32_t replicate, ppc_agents* agents);

/* Overwrites only the fields whose pointers are non-NULL, keeping every other
 * device field; agents->count must equal the device count (read from the
 * device unless a download or upload since the last count-changing call
 * already told it). This is the per-step host sync of a caller that keeps
 * cell_data authoritative on the host. When the view carries only positions,
 * velocities, previous velocities, pressure and orientation (the kinematic
 * fields), the device compares the positions with the resident ones and the
 * next step rebuilds the mechanics mesh only if some differ; if in addition
 * every one of those rows is page-locked (ppc_host_alloc), the call returns
 * once the copies are queued, and the rows must stay unchanged until the next
 * call that synchronises the stream (ppc_download, ppc_synchronize, ...).
 * Otherwise it synchronises the stream. */
int ppc_upload_fields(ppc_state* s, int32_t replicate, const ppc_agents* agents);

int ppc_get_count(ppc_state* s, int32_t replicate, int32_t* count);

/* Waits for the state's queued device work and returns the first error any
 * kernel reported since the last check (e.g. PPC_ERR_NONFINITE from
 * ppc_step, which itself returns as soon as the work is queued). */
int ppc_synchronize(ppc_state* s);

/* How page-locked host rows (ppc_host_alloc) travel in ppc_upload,
 * ppc_upload_fields and ppc_download (pageable rows always take the copy
 * engine through a staging buffer). */
enum ppc_host_transfer
{
	PPC_TRANSFER_COPY_ENGINE = 0, /* the default: DMA copies into a device staging
									 buffer, then a (un)pack kernel */
	PPC_TRANSFER_ZERO_COPY = 1	  /* the (un)pack kernels read and write the host rows
									 over the bus */
};
int ppc_set_host_transfer(ppc_state* s, int32_t mode);

/* Page-locked host memory for fast host <-> device copies (cudaHostAlloc);
 * NULL on failure. */
void* ppc_host_alloc(size_t bytes);
void ppc_host_free(void* p);

/* Counters kept like environment::divisions_count / deaths_count
 * (reference: src/environment.h:34-35). */
int ppc_get_event_counts(ppc_state* s, int32_t replicate, int64_t* divisions, int64_t* deaths);

/* ---- reference entry points --------------------------------------------- */

/* containers_solver::update_mechanics_mesh (reference: src/solver/host/containers_solver.cpp:15-56).
 * Bins agents into mechanics voxels; the order inside a voxel is descending
 * agent index, the order a serial run of the reference produces. */
int ppc_update_mechanics_mesh(ppc_state* s);

/* position_solver::update_cell_neighbors (reference: src/solver/host/position_solver.cpp:262-286).
 * Requires a current mesh. Returns PPC_ERR_CAPACITY if a list overflows the
 * neighbour capacity (the lists are then incomplete). */
int ppc_update_cell_neighbors(ppc_state* s);

/* position_solver::update_cell_forces (reference: src/solver/host/position_solver.cpp:233-260).
 * Uses the neighbour lists of the last ppc_update_cell_neighbors. */
int ppc_update_cell_forces(ppc_state* s);

/* position_solver::update_motility (reference: src/solver/host/position_solver.cpp:288-314)
 * for a state whose agents carry no motility fields: a no-op that always
 * succeeds. Motile agents go through ppc_update_motility_fields. */
int ppc_update_motility(ppc_state* s);

/* Standard rules that set an agent's migration bias direction when it
 * redraws its walk (the reference's update_migration_bias_direction
 * callbacks, set by the builder from the XML: src/builder.cpp:1184-1232). */
enum ppc_direction_rule
{
	PPC_DIRECTION_NONE = 0,		  /* the direction the caller set */
	PPC_DIRECTION_CHEMOTAXIS = 1, /* chemotaxis_function: the gradient of substrate
									 chemotaxis_index times chemotaxis_direction,
									 normalised (src/original/core/standard_models.cpp:542-555) */
	PPC_DIRECTION_ADVANCED_CHEMOTAXIS = 2, /* advanced_chemotaxis_function<false>: the
											  gradients weighted by the chemotactic
											  sensitivities, normalised (:557-583) */
	PPC_DIRECTION_ADVANCED_CHEMOTAXIS_NORMALIZED = 3 /* advanced_chemotaxis_function<true>:
														each gradient normalised first */
};

/* Motility fields of one replicate (reference: cell_data motilities.*,
 * defaults src/data_storage_phenotype.cpp:245-256), host memory, one row per
 * agent in the state's agent order (`count` = the replicate's count). */
typedef struct ppc_motility
{
	int32_t count;
	/* 0: as the reference, every 3-D walk lies in the xy-plane (its
	   random_walk receives the restrict_to_2d array pointer as a bool,
	   src/solver/host/position_solver.cpp:131, which is always true);
	   1: each agent's restrict_to_2d flag decides */
	int32_t restrict_per_agent;
	const uint8_t* is_motile;				 /* [count] */
	const uint8_t* restrict_to_2d;			 /* [count] */
	const double* persistence_time;			 /* [count] */
	const double* migration_speed;			 /* [count] */
	const double* migration_bias;			 /* [count] */
	double* migration_bias_direction;		 /* [count*dims], read, and written by a direction rule */
	double* motility_vector;				 /* [count*dims], read and written */
	/* direction rules (NULL direction_rule: PPC_DIRECTION_NONE for all) */
	const uint8_t* direction_rule;			 /* [count] enum ppc_direction_rule */
	const int32_t* chemotaxis_index;		 /* [count] substrate of PPC_DIRECTION_CHEMOTAXIS */
	const double* chemotaxis_direction;		 /* [count] +1 up the gradient, -1 down */
	const double* chemotactic_sensitivities; /* [count*substrates] weights of the advanced rules */
	int32_t substrates;						 /* columns of chemotactic_sensitivities */
	int32_t reserved;
} ppc_motility;

/* Substrate gradients of one replicate's diffusion mesh, the input of the
 * chemotaxis rules (the reference reads them with agent::nearest_gradient of
 * the absent paraBioFVM library). The diffusion mesh shares the replicate's
 * bounding box; voxel_shape gives its voxel edges, its grid is
 * ceil(extent / voxel_shape) per axis like the mechanics mesh, and an agent's
 * voxel is found by the same truncation. `gradients` holds, per diffusion
 * voxel (x fastest, then y, then z), per substrate, the x, y and z components
 * (3 values even in 1-D and 2-D). */
typedef struct ppc_gradient_field
{
	int32_t substrates;
	int32_t voxel_shape[3];
	const double* gradients; /* [voxels * substrates * 3] */
} ppc_gradient_field;

/* Copies replicate r's gradient field to the device, where the motility pass
 * reads it (replacing any earlier field of that replicate). Synchronises. */
int ppc_upload_gradients(ppc_state* s, int32_t r, const ppc_gradient_field* field);

/* Makes the motility fields of replicate r resident on the device (rows in
 * the state's agent order, `count` = the replicate's count): from then on
 * they move with their agent when the container is compacted, a dividing
 * agent's daughter copies them (phenotype_t::copy_to, src/phenotype.cpp:18-30),
 * and ppc_update_motility_fields(s, r, NULL) uses them without any copy.
 * Synchronises. */
int ppc_upload_motility(ppc_state* s, int32_t r, const ppc_motility* fields);
/* Copies the resident motility fields of replicate r to the host rows and
 * sets fields->count. Synchronises. */
int ppc_download_motility(ppc_state* s, int32_t r, ppc_motility* fields);

/* position_solver::update_motility with motile agents (reference:
 * src/solver/host/position_solver.cpp:115-145,198-212,288-314,
 * solver_helper.h:82-101,160-182,250-287). A motile agent redraws its
 * direction with probability dt/persistence_time — draw 0 of agent i at the
 * n-th call for a replicate is uniform(seed, n, replicate, i,
 * PPC_DRAW_MOTILITY); the walk's angle and z are the next two draws — mixes
 * it with migration_bias_direction by migration_bias, scales it to
 * migration_speed, and adds its motility vector to its resident velocity.
 * Agents with a direction rule (ppc_direction_rule) first set their
 * migration bias direction from the uploaded gradient field, as the
 * reference's callback does right after the walk is drawn; the others keep
 * the direction the caller set. With `fields` NULL the
 * resident fields (ppc_upload_motility) are used and nothing is copied;
 * otherwise `fields` is uploaded (and becomes the resident copy), and the
 * motility vectors and bias directions are written back to it. Synchronizes. */
int ppc_update_motility_fields(ppc_state* s, int32_t replicate, ppc_motility* fields);

/* position_solver::update_basement_membrane_interactions (reference: src/solver/host/position_solver.cpp:316-335). */
int ppc_update_basement_membrane_interactions(ppc_state* s);

/* position_solver::update_spring_attachments (reference: src/solver/host/position_solver.cpp:372-479).
 * Stochastic detachment and attachment (update_spring_attachments_internal)
 * with counter-based draws — agent i's k-th draw of the n-th spring update of
 * a replicate is uniform(seed, n, replicate, i, k) — in the reference's
 * serial order and capacity checks, then spring contraction. Needs the
 * neighbour lists (computed here if stale). ppc_step takes the same route
 * (through these separate entry points) while any rate is non-zero. The
 * attachment candidates of one update (agent-neighbour pairs whose draw
 * succeeds) are listed in a buffer of the replicate's capacity; more return
 * PPC_ERR_CAPACITY. */
int ppc_update_spring_attachments(ppc_state* s);

/* position_solver::update_positions (reference: src/solver/host/position_solver.cpp:481-520). */
int ppc_update_positions(ppc_state* s);

/* containers_solver::update_cell_container_for_mechanics (reference: src/solver/host/containers_solver.cpp:140-147).
 * Removes agents outside the domain bounding box or flagged PPC_FLAG_TO_REMOVE
 * by swap-with-last, in the order a serial run of the reference produces. */
int ppc_update_cell_container_for_mechanics(ppc_state* s);

/* containers_solver::update_cell_container_for_phenotype (reference: src/solver/host/containers_solver.cpp:149-188)
 * without BioFVM's release_internalized_substrates: divides agents flagged
 * PPC_FLAG_TO_DIVIDE (src/cell.cpp:108-163), then removes as above. */
int ppc_update_cell_container_for_phenotype(ppc_state* s);

/* Number of agents of replicate `replicate` whose flag is `flag` (enum
 * ppc_flag), counted on the device (no counterpart in the reference: a host
 * caller sizing the container before a division pass counts this way instead
 * of downloading every flag). Synchronises. */
int ppc_count_flags(ppc_state* s, int32_t replicate, int32_t flag, int32_t* count);

/* Sets PPC_FLAG_TO_REMOVE with probability p_death and otherwise
 * PPC_FLAG_TO_DIVIDE with probability p_divide per agent, from the state's
 * counter-based random stream (stand-in for the reference's phenotype models,
 * src/original/core/standard_models.cpp:478-540). */
int ppc_flag_by_draws(ppc_state* s, double p_divide, double p_death);

/*
 * Phenotype fields of one replicate that cell-cell interactions read or write
 * and that the mechanics state does not hold (reference: cell_data
 * interactions.*, deaths.dead, states.damage/total_attack_time/number_of_nuclei,
 * volumes.*, agent_data.internalized_substrates). Host memory, one row per
 * agent in the state's current agent order (`count` = the replicate's count).
 * Per-definition rows have cell_definitions_count entries; substrate rows have
 * `substrates` entries. The resident total volume, nuclear volume, radius,
 * nuclear radius, surface area, positions and flags are the state's own.
 */
typedef struct ppc_interactions
{
	int32_t count;
	int32_t substrates;

	/* read */
	const uint8_t* dead;						/* [count] deaths.dead */
	const double* dead_phagocytosis_rate;		/* [count] */
	const double* damage_rate;					/* [count] */
	const double* live_phagocytosis_rates;		/* [count*definitions] */
	const double* attack_rates;					/* [count*definitions] */
	const double* fusion_rates;					/* [count*definitions] */
	const double* immunogenicities;				/* [count*definitions] */
	const double* fraction_transferred_when_ingested; /* [count*substrates] */

	/* read and written */
	double* damage;				/* [count] states.damage */
	double* total_attack_time;	/* [count] states.total_attack_time */
	int32_t* number_of_nuclei;	/* [count] states.number_of_nuclei */
	double* fluid;				/* [count] volumes.* */
	double* solid;
	double* cytoplasmic;
	double* cytoplasmic_fluid;
	double* cytoplasmic_solid;
	double* nuclear_fluid;
	double* nuclear_solid;
	double* fluid_fraction;
	double* cytoplasmic_to_nuclear_ratio;
	double* target_solid_cytoplasmic;
	double* target_solid_nuclear;
	double* internalized_substrates; /* [count*substrates] */
} ppc_interactions;

/* Makes the interaction fields of replicate r resident on the device (rows
 * in the state's agent order): from then on they move with their agent when
 * the container is compacted, and division treats them as cell::divide does
 * (src/cell.cpp:108-163): the parent's damage and total attack time are
 * cleared, every volume compartment is halved, the internalized substrates
 * are halved when `compute_internalized_substrates` is non-zero (the
 * reference's e.m.compute_internalized_substrates), and the daughter copies
 * the parent's phenotype with a fresh state (no damage or attack time, one
 * nucleus). ppc_update_cell_cell_interactions(s, r, NULL) then uses them with
 * no copy. All replicates share one substrate count. Synchronises. */
int ppc_upload_interactions(ppc_state* s, int32_t r, const ppc_interactions* fields,
							int32_t compute_internalized_substrates);
/* Copies the resident interaction fields of replicate r to the host rows and
 * sets fields->count. Synchronises. */
int ppc_download_interactions(ppc_state* s, int32_t r, ppc_interactions* fields);

/* interactions_solver::update_cell_cell_interactions (reference:
 * src/solver/host/interactions_solver.cpp:143-265): each live agent walks its
 * neighbour list and, with one uniform draw per neighbour, may ingest a dead
 * neighbour, ingest a live one, attack it or fuse with it (at most one live
 * ingestion, attack and fusion per agent). Draw k of agent i at the n-th call
 * for a replicate is uniform(seed, n, replicate, i, PPC_DRAW_INTERACTION + k).
 * Ingested and fused neighbours get PPC_FLAG_TO_REMOVE; the ingesting or fusing
 * agent's volumes, geometry (and, when fusing, position) change in the
 * resident state. With `fields` NULL the resident interaction fields
 * (ppc_upload_interactions) are used and nothing is copied; otherwise
 * `fields` is uploaded (becoming the resident copy) and written back after
 * the call. The outcome is that of the reference run on one thread (agents in
 * index order). Uses the neighbour lists of the last
 * ppc_update_cell_neighbors (rebuilt here if a fused step ran since); if one
 * of the replicate's lists was cut at the neighbour capacity, nothing changes
 * and PPC_ERR_CAPACITY is returned. Synchronizes. */
int ppc_update_cell_cell_interactions(ppc_state* s, int32_t replicate, ppc_interactions* fields);

/* ---- fused step ----------------------------------------------------------- */
/* ppc_step returns once the work is queued (device errors surface at the
 * next ppc_synchronize or syncing call). Blocks of steps are captured once in
 * a CUDA graph and replayed. */

/* Advances `steps` mechanics steps in the order of simulator::simulate_mechanics
 * (reference: src/simulator.cpp:157-196, without gradient, custom rules,
 * interactions and motility): forces, membrane, springs, positions, container
 * compaction, mesh rebuild. Neighbour lists are recomputed inside the force
 * pass; call ppc_update_cell_neighbors to materialise them. Requires a current
 * mesh (ppc_update_mechanics_mesh once after upload). With `with_phenotype`
 * non-zero, each step is followed by ppc_flag_by_draws(p_divide, p_death) and
 * the phenotype container update, then a mesh rebuild. */
int ppc_step(ppc_state* s, int32_t steps);
int ppc_step_with_phenotype(ppc_state* s, int32_t steps, double p_divide, double p_death);

/* ---- readback of derived structures -------------------------------------- */

/* Neighbour lists of replicate `replicate`: counts[i] and lists[i*list_capacity + k].
 * Synchronises the stream. */
int ppc_get_neighbors(ppc_state* s, int32_t replicate, int32_t* counts, int32_t* lists, int32_t list_capacity);

/* Mechanics mesh bins of replicate `replicate` as CSR over voxels:
 * voxel_counts[v] (size voxel_count) and agents (size count) concatenated in
 * voxel order, each voxel's agents in bin order. Synchronises the stream. */
int ppc_get_mesh_bins(ppc_state* s, int32_t replicate, int32_t* voxel_counts, int32_t* agents);

/* Voxel count of replicate `replicate`'s mechanics mesh. */
int ppc_get_voxel_count(ppc_state* s, int32_t replicate, int64_t* voxel_count);

/* ---- helpers -------------------------------------------------------------- */

/* common_solver::get_mesh_position (reference: src/solver/host/common_solver.cpp:18-38). */
int ppc_get_mesh_position(const ppc_mesh* mesh, const double* position, int32_t* voxel_coords3);

/* common_solver::get_mesh_index (reference: src/solver/host/common_solver.cpp:10-16). */
int ppc_get_mesh_index(const ppc_mesh* mesh, const int32_t* voxel_coords3, int32_t* index);

/* Number of kernel launches this state has issued (for launch accounting). */
int ppc_get_launch_count(ppc_state* s, int64_t* launches);

/* Kernel timing: while on, every launch of the fused force kernel is
 * bracketed by CUDA events on the state's stream (steps then run without
 * graph capture). ppc_get_profile synchronises and returns the summed
 * device time (ms) and the number of timed launches since profiling was
 * switched on. */
int ppc_set_profiling(ppc_state* s, int32_t on);
int ppc_get_profile(ppc_state* s, double* fused_ms, int64_t* fused_launches);

/* ---- binning without allocation ------------------------------------------ */

/* Limits of the fixed scratch of ppc_bin_agents_noalloc (about 5.8 MB of
 * device memory reserved on every GPU that loads the library). */
#define PPC_NOALLOC_MAX_AGENTS 131072
#define PPC_NOALLOC_MAX_VOXELS 1048576

/* Mechanics-mesh binning for callers that cannot allocate device memory.
 * No counterpart in the reference: it is ppc_update_mechanics_mesh followed
 * by ppc_get_mesh_bins without a ppc_state, for code that must not call
 * cudaMalloc (a framework allocator that forbids hidden allocations, a
 * real-time loop that must not block in the driver's allocator).
 * `positions` (count*dims doubles, AoS as in the reference), `voxel_counts`
 * (one int32 per mechanics voxel) and `agents` (count int32) are the caller's
 * device buffers; results match ppc_get_mesh_bins: per-voxel counts and the
 * agents grouped by voxel, descending index inside a voxel. Scratch lives in
 * one fixed device array; sizes above PPC_NOALLOC_MAX_AGENTS or
 * PPC_NOALLOC_MAX_VOXELS return PPC_ERR_CAPACITY (the grid is sized in 64-bit
 * arithmetic, so no mesh extent can wrap it). The in-voxel ordering pass costs
 * c^2 loads for a voxel of c agents: negligible at tissue densities, about a
 * second of GPU time if all PPC_NOALLOC_MAX_AGENTS agents share one voxel.
 * Nothing is allocated. The
 * first call on a device looks the array's address up for that device, so
 * make that first call before any stream capture. All calls share the array:
 * calls whose work overlaps on the GPU race. Work is queued on `cuda_stream`
 * (NULL: the legacy default stream) and the call returns without waiting. */
int ppc_bin_agents_noalloc(const ppc_mesh* mesh, const double* positions, int32_t count, int32_t* voxel_counts,
						   int32_t* agents, void* cuda_stream);

/* Message of the last error on the calling thread ("" if none). */
const char* ppc_last_error(void);

int ppc_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PPC_H */
