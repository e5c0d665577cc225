/*
 * dsmc_b200.h - C ABI of the B200 DSMC timestep (libdsmc_b200.so).
 *
 * Drop-in for the timestep of andeplane/master's DSMC solver
 * (code/base_code/program/dsmc/): the mover with diffuse walls, the cell
 * re-binning ("sort"), the no-time-counter collide and the sampler that
 * System::step (dsmc/system.cpp:22-47) and StatisticsSampler::sample
 * (dsmc/statisticssampler.cpp:42-65) run once per timestep.
 *
 * Conventions: plain C types, caller-owned host buffers that are copied in
 * and out, device memory owned by the context, int status (0 = DSMC_OK), no
 * exceptions across the boundary.  One context per host thread; calls on a
 * context are ordered on its CUDA stream and are not re-entrant.  Units are
 * the reference's reduced units (dsmc/unitconverter.cpp:3-21): length 1 um,
 * mass 1 amu, energy 1.65088e-21 J.  Arrays of voxels use the reference's
 * order, index i*ny*nz + j*nz + k (dsmc/grid.h:139-145).
 */
#ifndef DSMC_B200_H
#define DSMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define DSMC_OK 0
#define DSMC_ERR_ARG 1         /* bad argument or null pointer */
#define DSMC_ERR_IO 2          /* file missing, short or malformed */
#define DSMC_ERR_CUDA 3        /* CUDA runtime error (message in dsmc_last_error) */
#define DSMC_ERR_CAPACITY 4    /* a size limit of this build was exceeded */
#define DSMC_ERR_CONFIG 5      /* voxel/cell configuration rejected (dsmc/system.cpp:221-239) */
#define DSMC_ERR_STATE 6       /* particle state invalid: in solid, non-finite, ... */
#define DSMC_ERR_NOT_FOUND 7   /* ini key missing (dsmc/cinifile.h:61) */
#define DSMC_ERR_NO_DEVICE 8   /* no CUDA device, or the kernels were not built for it */

/* ---- precision of a context ---------------------------------------- */
#define DSMC_PREC_SPLIT32 0    /* int voxel + fp32 offset, fp32 velocity, fp64 tallies */
#define DSMC_PREC_FP64 1       /* the reference's fp64 positions and arithmetic */

/* ---- settings: the fields of Settings (dsmc/settings.h:11-49) ------- */
typedef struct dsmc_settings {
    int timesteps;
    int statistics_interval;
    int atoms_per_molecule;     /* F_N, simulator weight (an int in the reference) */
    int cells_x, cells_y, cells_z;
    int flow_direction;         /* axis of gravity and flux; <0: none */
    int sampling_bins;
    int seed;                   /* reference ini seed */
    int max_molecules_per_node;
    int nx, ny, nz;             /* MPI processor grid of the reference; 1 1 1 here */
    double mass;                /* amu */
    double temperature;         /* K (SI, as the ini) */
    double wall_temperature;    /* K */
    double gravity;             /* reduced acceleration */
    double density;             /* m^-3 (SI, as the ini) */
    double diam;                /* um */
    double Lx, Ly, Lz;          /* um */
    double dt;                  /* reduced time */
    double alpha_n, alpha_t;
    double viscosity;
    int surface_model;          /* wall model (dsmc/system.cpp:345-352): 0 thermal (diffuse),
                                   1 specular, 2 cercignani_lampis (alpha_n, alpha_t) */
    int sample_begin;           /* first step sampled (0: from the start) */
    uint64_t rng_seed;          /* key of the counter-based draws */
    char world[512];            /* world folder (the ini's `world`) */
    int load_previous_state;    /* continue from state_files/ + Tocontinue (dsmc/main.cpp:37-55) */
} dsmc_settings;

/* Fills the reference's Python-driver defaults (dsmcconfig.py:14-77). */
int dsmc_settings_defaults(dsmc_settings *s);
/* Parses a dsmc.ini with the reference's CIniFile rules (dsmc/cinifile.h:28-104):
 * `key = value` lines, getint = (int)strtod, getbool = "true".  Replaces
 * Settings::Settings (dsmc/settings.cpp:3-44). */
int dsmc_settings_load_ini(const char *path, dsmc_settings *s);

/* ---- state files and continuation ----------------------------------- */
/* The reference's particle state file (DSMC_IO::save_state_to_file_binary /
 * load_state_from_file_binary, dsmc/dsmc_io.cpp:82-159, one per rank as
 * state_files/state%04d.bin): int32 N, then per particle rx ry rz vx vy vz as
 * doubles.  Host only.  Read: *n is set to N; DSMC_ERR_CAPACITY if cap < N
 * (r and v may be NULL to ask for N). */
int dsmc_state_file_read(const char *path, int64_t cap, double *r, double *v, int64_t *n);
int dsmc_state_file_write(const char *path, int64_t n, const double *r, const double *v);
/* The reference's Tocontinue counters (dsmc/main.cpp:37-55 reads, :110-112
 * writes): "t steps collisions wall_collisions" as text.  Host only; written
 * with 17 significant digits (the reference writes 6). */
int dsmc_tocontinue_read(const char *path, double *t, uint64_t *steps, uint64_t *collisions,
                         uint64_t *wall_collisions);
int dsmc_tocontinue_write(const char *path, double t, uint64_t steps, uint64_t collisions, uint64_t wall_collisions);

/* ---- world files ---------------------------------------------------- */
typedef struct dsmc_world_header {
    float porosity_global;
    float porosity;
    uint32_t global_nx, global_ny, global_nz;
    uint32_t nx, ny, nz;        /* stored dimensions (3x the rank's block with halo) */
} dsmc_world_header;

/* Reads the header of a world file (dsmc/dsmc_io.cpp:183-220). */
int dsmc_world_read_header(const char *path, dsmc_world_header *h);
/* Reads a single-rank world file and strips the 3x3x3 periodic halo: the
 * outputs hold global_nx*global_ny*global_nz voxels (normals etc. 3 floats
 * each).  Replaces DSMC_IO::read_grid_matrix (dsmc/dsmc_io.cpp:183-220). */
int dsmc_world_read(const char *path, uint8_t *voxels, float *normals, float *tangents1,
                    float *tangents2);
/* Writes world files in the reference layout, one per rank of a px*py*pz
 * grid, each with its 3x3x3 halo (ComplexGeometry::save_to_file,
 * dsmc/complexgeometry.cpp:220-318).  folder/%04d.bin and folder/porosity.txt. */
int dsmc_world_write(const char *folder, uint32_t nx, uint32_t ny, uint32_t nz, const uint8_t *voxels,
                     const float *normals, const float *tangents1, const float *tangents2, int px,
                     int py, int pz);

/* ---- geometry generation -------------------------------------------- */
typedef struct dsmc_sphere_params {
    int nx, ny, nz;
    double radius;              /* box-normalised, e.g. 4 voxels / 64 = 0.0625 */
    int spheres_type;           /* 0: spheres_num spheres; 1: until wanted_porosity */
    int spheres_num;
    double wanted_porosity;
    int seed;                   /* the ini seed; the generator uses -|seed| */
    int inverted;               /* 1: spheres are solid */
    int prevent_overlap;
    int number_of_neighbor_averages;
} dsmc_sphere_params;

/* Packed-sphere geometry with normals, tangents and boundary voxels,
 * identical to ComplexGeometry::create_packed_spheres + make_periodic +
 * calculate_normals + calculate_tangents + find_boundary_points
 * (dsmc/complexgeometry.cpp:401-513, 853-871, 928-1063).  Outputs hold
 * nx*ny*nz voxels.  porosity_out: fraction of empty voxels. */
int dsmc_geometry_packed_spheres(const dsmc_sphere_params *p, uint8_t *voxels, float *normals,
                                 float *tangents1, float *tangents2, float *porosity_out);
/* Normals, tangents and boundary typing of an arbitrary solid mask (0/1),
 * in place (ComplexGeometry::calculate_normals_tangents_and_inner_points,
 * dsmc/complexgeometry.cpp:196-201).  On the CPU. */
int dsmc_geometry_finish(uint32_t nx, uint32_t ny, uint32_t nz, int number_of_neighbor_averages,
                         uint8_t *voxels, float *normals, float *tangents1, float *tangents2);
/* The same stencil on the GPU (device_id), identical output: the normal,
 * tangent and boundary passes of dsmc/complexgeometry.cpp:928-1063 as
 * kernels, the order-dependent removals replayed on the host. */
int dsmc_geometry_finish_gpu(int device_id, uint32_t nx, uint32_t ny, uint32_t nz,
                             int number_of_neighbor_averages, uint8_t *voxels, float *normals,
                             float *tangents1, float *tangents2);

/* dsmc_geometry_finish_gpu without any device allocation, for callers that
 * may not call cudaMalloc (fixed device-memory budgets, or code that must not
 * take the implicit synchronisation of an allocation).  No counterpart in
 * the reference.  Its device-side working buffers are a file-scope array of
 * the library sized for at most 64^3 voxels (13.1 MB kept by every GPU that
 * loads the library until exit); larger grids return DSMC_ERR_CAPACITY.  The
 * first call on a device looks up the array's device address and keeps it
 * (make that call before any stream capture; after a cudaDeviceReset of the
 * device the kept address is stale, so do not call it there again); calls
 * that overlap on one GPU race on the array. */
int dsmc_geometry_finish_gpu_noalloc(int device_id, uint32_t nx, uint32_t ny, uint32_t nz,
                                     int number_of_neighbor_averages, uint8_t *voxels, float *normals,
                                     float *tangents1, float *tangents2);

/* ---- context ---------------------------------------------------------- */
typedef struct dsmc_ctx dsmc_ctx;

/* A context: one GPU, its stream and device buffers, and any number of
 * systems advanced together.  It takes the place of the per-rank process
 * state of the reference's main (dsmc/main.cpp:19-30: one System per MPI
 * rank); precision is DSMC_PREC_SPLIT32 or DSMC_PREC_FP64.  destroy frees
 * everything (the reference never frees its grid, dsmc/dsmc_io.cpp:205-208). */
int dsmc_ctx_create(int device_id, int precision, dsmc_ctx **out);
void dsmc_ctx_destroy(dsmc_ctx *ctx);
/* Message of the last failed call on ctx (or of the last failed context-free
 * call on this thread when ctx is NULL): the text the reference prints before
 * its exit(1) (e.g. dsmc/system.h:137-166) or throws to System::step
 * (dsmc/system.cpp:41-44), here returned with the DSMC_ERR_* code. */
const char *dsmc_last_error(const dsmc_ctx *ctx);
/* Waits until the context's queued work has finished.  No counterpart in the
 * reference, whose calls are synchronous. */
int dsmc_sync(dsmc_ctx *ctx);

/* Adds one system (one geometry and its gas; the reference's System,
 * dsmc/system.cpp:241-382) from a halo-free voxel grid.  Builds the cells as
 * System::setup_cells does (dsmc/system.cpp:432-490) and validates the
 * voxel/cell divisibility (dsmc/system.cpp:221-239).  Returns its id. */
int dsmc_system_add(dsmc_ctx *ctx, const dsmc_settings *s, uint32_t nx, uint32_t ny, uint32_t nz,
                    const uint8_t *voxels, const float *normals, const float *tangents1,
                    const float *tangents2, float porosity_global, int *sys_id);
/* Same, reading s->world/0000.bin as the reference's Grid does
 * (DSMC_IO::read_grid_matrix, dsmc/dsmc_io.cpp:183-220), halo stripped. */
int dsmc_system_add_world(dsmc_ctx *ctx, const dsmc_settings *s, int *sys_id);

/* The active cells of a voxel grid as System::setup_cells builds them
 * (dsmc/system.cpp:432-490): numbered in order of first touch by a k-outer,
 * i-inner voxel sweep, cells without empty voxels dropped; per cell its
 * global index (i*cy*cz + j*cz + k), empty and total voxel counts, volume
 * (Cell::update_volume, dsmc/cell.cpp:27-40) and NTC coefficient.  Host only.
 * cap: capacity of the output arrays (any may be NULL); *num_cells is set. */
int dsmc_cells_layout(const dsmc_settings *s, uint32_t nx, uint32_t ny, uint32_t nz, const uint8_t *voxels,
                      int cap, int32_t *global_index, int32_t *pixels, int32_t *total_pixels, double *volume,
                      double *coeff, int *num_cells);

typedef struct dsmc_system_info {
    int64_t num_particles;
    int num_cells_total;
    int num_active_cells;
    double volume;              /* effective (empty) volume */
    double porosity;
    double atoms_per_molecule;
    double dt;
    int64_t expected_particles; /* density*volume/atoms_per_molecule (dsmc/system.cpp:323) */
    int slots;                  /* particle slots reserved per buffer */
    double volume_global;       /* L_x L_y L_z * porosity_global (dsmc/system.cpp:314) */
} dsmc_system_info;
/* The sizes System::initialize derives for a system (dsmc/system.cpp:241-382)
 * and the slots this library reserves for it. */
int dsmc_system_info_get(dsmc_ctx *ctx, int sys_id, dsmc_system_info *info);

/* One x-slab of a geometry, for a run over several GPUs (the reference's
 * domain decomposition, dsmc/topology.cpp + System::mpi_move,
 * dsmc/system.cpp:49-105, along x): the system owns the active cells with
 * cell x index in [cell_x0, cell_x1) and holds the whole geometry for the
 * mover.  Particle init and dsmc_particles_set keep the particles of the
 * slab's cells (ids stay the geometry-wide indices).  A slab is its
 * context's only system, runs in split precision, and advances one step per
 * dsmc_step; after each step dsmc_exchange_take hands out the particles that
 * ended in another slab's cell and dsmc_exchange_put takes in those that
 * ended in this one, before the next step.  dsmc_particles_get on a slab
 * needs buffers for every id of the geometry and marks the ids it does not
 * hold with cell = -1. */
int dsmc_system_add_slab(dsmc_ctx *ctx, const dsmc_settings *s, uint32_t nx, uint32_t ny, uint32_t nz,
                         const uint8_t *voxels, const float *normals, const float *tangents1, const float *tangents2,
                         float porosity_global, int cell_x0, int cell_x1, int *sys_id);
/* Exchange records are 32 bytes: uint32 voxel (i | j << 11 | k << 22),
 * uint32 x offset (float bits; the top bit flags a non-empty voxel), float y
 * and z offsets in voxel units; float vx, vy, vz, uint32 id.  The owner of a
 * record is the slab holding cell x index i / (nx / cells_x).
 * take: moves the outgoing records into `records` (host memory, or device
 * memory of the context's GPU when device != 0) and sets *n;
 * DSMC_ERR_CAPACITY, with *n set and nothing taken, when cap < *n.
 * put: inserts n records, each in a cell of system sys_id. */
int dsmc_exchange_take(dsmc_ctx *ctx, int64_t cap, void *records, int device, int64_t *n);
int dsmc_exchange_put(dsmc_ctx *ctx, int sys_id, int64_t n, const void *records, int device);

/* Maxwellian velocities and uniform positions in empty voxels, as
 * System::setup_molecules (dsmc/system.cpp:398-430); draws come from one
 * counter-based stream per particle.  n < 0: the reference's count. */
int dsmc_particles_init(dsmc_ctx *ctx, int sys_id, int64_t n);
/* Warm start: replaces a system's particles by n particles (n < 0: the
 * reference's count) drawn from a per-voxel field instead of the uniform
 * Maxwellian at rest of System::setup_molecules (dsmc/system.cpp:398-430):
 * voxel w is chosen with probability weight[w] / sum(weight) over the empty
 * voxels, the position uniformly inside it, the velocity drift[3w..3w+2] plus
 * a Maxwellian of the gas temperature.  weight holds nx*ny*nz floats and
 * drift 3*nx*ny*nz (reduced velocity units), in the geometry's voxel order;
 * device != 0: both are device memory of the context's GPU.  Draws come from
 * one counter-based stream per particle, as dsmc_particles_init's. */
int dsmc_particles_init_field(dsmc_ctx *ctx, int sys_id, int64_t n, const float *weight, const float *drift,
                              int device);
/* Batched dsmc_particles_init / dsmc_particles_init_field for the systems of
 * a multi-system context: the listed systems (count distinct ids, no slabs)
 * get the same particles as from one call each (a system's draws depend only
 * on its seed, count and field), but the context's other particles are
 * staged and all of them re-laid out once, not once per system.  n: count
 * values, n[i] < 0 or n null the reference's count.  _field: weights[i] and
 * drifts[i] as dsmc_particles_init_field's weight and drift for system
 * sys_ids[i], every field checked before any particle is replaced.  A
 * system listed twice is DSMC_ERR_ARG. */
int dsmc_particles_init_many(dsmc_ctx *ctx, int count, const int *sys_ids, const int64_t *n);
int dsmc_particles_init_field_many(dsmc_ctx *ctx, int count, const int *sys_ids, const int64_t *n,
                                   const float *const *weights, const float *const *drifts, int device);
/* No counterpart in the reference (the warm start's training data).
 * Adds one system's per-voxel particle sums {count, sum vx, sum vy, sum vz}
 * (4 floats per voxel, geometry voxel order, 16-byte aligned) to field: the
 * steady fields that the warm-start surrogate learns are these sums over
 * many steps.  device != 0: field is device memory of the context's GPU and
 * the call is asynchronous: the sums are added on the context's stream
 * (dsmc_stream), so read them after a dsmc_sync or an event on that stream;
 * device == 0: a host array, complete when the call returns. */
int dsmc_field_accumulate(dsmc_ctx *ctx, int sys_id, float *field, int device);
/* Replaces a system's particles by n particles in the reference's state-file
 * layout: r[3n], v[3n] fp64 (dsmc/dsmc_io.cpp:82-159).  Particle i gets id i. */
int dsmc_particles_set(dsmc_ctx *ctx, int sys_id, int64_t n, const double *r, const double *v);
/* The system's particle count (System::num_molecules_local, dsmc/system.h:85). */
int dsmc_particles_count(dsmc_ctx *ctx, int sys_id, int64_t *n);
/* Copies the particles out ordered by id (r[3n], v[3n]: the reference's
 * System::r and System::v, dsmc/system.h:74-75; cell: the reference's
 * global cell index of each particle, may be NULL). */
int dsmc_particles_get(dsmc_ctx *ctx, int sys_id, int64_t cap, double *r, double *v, int32_t *cell,
                       int64_t *n);

/* Advances every system by nsteps timesteps: accelerate, move, re-bin,
 * collide and sample, one fused kernel pass per step (System::step +
 * StatisticsSampler::sample, dsmc/main.cpp:57-64). */
int dsmc_step(dsmc_ctx *ctx, int nsteps);

/* The stages of System::step as separate calls, for callers that drive the
 * stage order themselves (all systems of the context):
 *   move     = steps += 1; accelerate (dsmc/system.cpp:133-144) + move with
 *              periodic wrap (dsmc/system.cpp:107-120)
 *   sort     = update_molecule_cells (dsmc/system.cpp:146-157)
 *   collide  = prepare + collide of every active cell (dsmc/system.cpp:122-131)
 *   sample   = the per-cell moment tallies on the sampling cadence */
int dsmc_stage_move(dsmc_ctx *ctx);
int dsmc_stage_sort(dsmc_ctx *ctx);
int dsmc_stage_collide(dsmc_ctx *ctx);
int dsmc_stage_sample(dsmc_ctx *ctx);

typedef struct dsmc_tallies {
    uint64_t step;              /* System::steps */
    uint64_t collisions;        /* System::collisions */
    uint64_t wall_collisions;   /* ColliderBase::num_collisions */
    uint64_t reseeds;           /* particles re-seeded by the mover's find_position */
    uint64_t particle_steps;
    int64_t count_periodic[3];  /* MoleculeMover::count_periodic */
    uint64_t samples;           /* sampled steps in the cell moments */
    uint64_t candidates;        /* NTC candidate pairs */
    double kinetic_energy;      /* current, reduced units (MeasureEnergy) */
    double temperature;         /* current, K (MeasureTemperature) */
    double flux;                /* F_N*count_periodic[flow]/(t - t0) (MeasureNumberFlowRate) */
    double time;                /* t, reduced */
    uint64_t stranded;          /* moves that ended in a cell with no free volume (re-seeded next step) */
} dsmc_tallies;
/* get: the counters and current scalars the reference's sampler reads from
 * System, MoleculeMover and ColliderBase (dsmc/statisticssampler.cpp:45-66,
 * dsmc/statisticalproperty.cpp:21-101).  reset: zeroes the counters, the cell
 * moments and the profiles and restarts the flux window at the current time
 * (as the reference's t0 = t at a run's start, dsmc/main.cpp:51-52). */
int dsmc_tallies_get(dsmc_ctx *ctx, int sys_id, dsmc_tallies *t);
int dsmc_tallies_reset(dsmc_ctx *ctx, int sys_id);

/* The sampler's scalar measurements at the current step, as each
 * Measure*::update computes them (dsmc/statisticalproperty.cpp:21-210) and
 * StatisticsSampler::sample prints them (dsmc/statisticssampler.cpp:45-66).
 * Flow rates count from the last tally reset or continuation; permeability
 * is 0 without a flow direction or gravity. */
typedef struct dsmc_measures {
    uint64_t step;
    double t_ns;                 /* System::t_in_nano_seconds */
    double energy_eV;            /* MeasureEnergy: 1/2 m sum |v|^2 * atoms_per_molecule */
    double temperature_K;        /* MeasureTemperature */
    double number_flow_rate;     /* MeasureNumberFlowRate, reduced units */
    double volumetric_flow_rate; /* MeasureVolumetricFlowRate, reduced units */
    double pressure_Pa;          /* MeasurePressure */
    double permeability_darcy;   /* MeasurePermeability, finalize's unit */
    uint64_t collisions, wall_collisions, molecules;
} dsmc_measures;
int dsmc_measures_get(dsmc_ctx *ctx, int sys_id, dsmc_measures *m);

/* Sampler profiles over the samples since the last tally reset
 * (StatisticsSampler, dsmc/statisticssampler.cpp:22-26): sampling_bins bins
 * in y of {count, sum v_z, sum 1/2 m v_z^2} (MeasureCount,
 * MeasureVelocityDistributionPoiseuille, MeasureTemperatureDistribution,
 * dsmc/statisticalproperty.cpp:229-362) and a v_x histogram over
 * [-4, 4] sqrt(T/m) (MeasureVelocityDistribution, :432-458).
 *
 * dsmc_profile_sums_get: the raw sums, 4*bins doubles: {count, sum v_z,
 * sum 1/2 m v_z^2} per y bin, then the v_x histogram; sums NULL gives only
 * *bins.  Sums of several ranks add up before finishing.
 * dsmc_profiles_finish: finishes sums as the reference's finalize() does
 * (:303-309, 364-371, 393-426, 462-478): count, v_z (m/s), temperature (K)
 * and pressure (Pa) per y bin, v_x bin centres (m/s) and counts.  Host only;
 * any output may be NULL; volume_global from dsmc_system_info.
 * dsmc_profiles_get: both for one system; outputs hold cap >= bins values. */
int dsmc_profile_sums_get(dsmc_ctx *ctx, int sys_id, int cap, double *sums, int *bins);
int dsmc_profiles_finish(const dsmc_settings *s, double volume_global, int bins, const double *sums, double *count,
                         double *velocity_z, double *temperature, double *pressure, double *vx_center,
                         double *vx_count);
int dsmc_profiles_get(dsmc_ctx *ctx, int sys_id, int cap, double *count, double *velocity_z, double *temperature,
                      double *pressure, double *vx_center, double *vx_count, int *bins);

/* Per active cell: global cell index (dsmc/system.h:130-132), particle count,
 * vr_max, selection remainder, and 8 fp64 moment sums over the sampled steps
 * (n, sum vx, vy, vz, sum vx^2, vy^2, vz^2, sum |v|^2).  Any pointer may be NULL. */
int dsmc_cells_get(dsmc_ctx *ctx, int sys_id, int cap, int32_t *global_index, int32_t *count,
                   double *vr_max, double *rest, double *moments, double *volume, int *num_cells);
/* Sets each active cell's Cell::vr_max and Cell::collision_rest
 * (dsmc/cell.h:18-23), in active-cell order. */
int dsmc_cells_set_state(dsmc_ctx *ctx, int sys_id, const double *vr_max, const double *rest);

/* Continuation (dsmc/main.cpp:37-55): the step counter, collisions and wall
 * collisions of an earlier run, typically read from its Tocontinue; the time
 * becomes t and the flux window restarts there (the reference's t0 = t). */
int dsmc_continue_from(dsmc_ctx *ctx, int sys_id, double t, uint64_t steps, uint64_t collisions,
                       uint64_t wall_collisions);

/* Exact checkpoint of a context: every particle record in its own precision
 * with its cell, each cell's (sigma c_r)_max, selection remainder and moment
 * sums, every system's tallies, flux window and draw key, and the step
 * counter -- the fields the reference's state file and Tocontinue leave out
 * (dsmc/dsmc_io.cpp:82-159).  A context set up with the same systems and
 * precision continues from it with the same trajectories as the context that
 * wrote it (the draws are keyed by particle id and step). */
int dsmc_checkpoint_save(dsmc_ctx *ctx, const char *path);
int dsmc_checkpoint_load(dsmc_ctx *ctx, const char *path);

/* No counterpart in the reference, whose cell member lists are vectors that
 * grow (Cell::add_molecule, dsmc/cell.cpp:113-140).
 * Slot capacity policy of the cell-sorted particle buffers: a cell gets
 * ceil(factor * max(expected, present) + pad) slots (default 2.0, 24).  An
 * overflow never loses particles: they spill to an overflow list, the
 * pipeline stops after that step and the host re-lays the buffers out. */
int dsmc_ctx_set_capacity(dsmc_ctx *ctx, double factor, int pad);

/* No counterpart in the reference.
 * Launch shape of the timestep pass: pipelined = 1 when the split-precision
 * production pass (collide_cells, move_cells, place_movers, place_walls) runs
 * dsmc_step (0: the generic cell pass, e.g. fp64 contexts), the grid and
 * block of move_cells, and its per-warp staging ring in particles. */
int dsmc_pass_info(dsmc_ctx *ctx, int *pipelined, int *grid, int *block, int *stage_capacity);

/* Launch tuning of the production pass, for the autotuner
 * (master_b200/autotune.py): the reference has no counterpart (its stages are
 * loops over particles on one core).  blocks_per_sm: resident blocks per SM of
 * collide_cells, move_cells, place_movers, place_walls and sample_cells, each
 * a persistent grid (0: the most that are resident, the default; larger
 * values are clamped to it); ring: move_cells' shared-memory staging ring in
 * particles per warp (0: the smallest that holds the largest cell; larger
 * rings trade resident blocks for staging depth); collide_claim: how
 * collide_cells' warps take chunks of 32 cells after their first (0: a
 * pass-wide counter when each warp has four chunks or more, else a fixed
 * stride; 1: always the stride; 2: always the counter).  Any setting gives
 * the same trajectories: only the work distribution changes.
 * dsmc_tuning_get: the current settings, and in limits the most blocks per SM
 * of each kernel at the current ring and the ring in use. */
typedef struct dsmc_tuning {
    int blocks_per_sm[5];
    int ring;
    int collide_claim;
} dsmc_tuning;
int dsmc_tuning_set(dsmc_ctx *ctx, const dsmc_tuning *t);
int dsmc_tuning_get(dsmc_ctx *ctx, dsmc_tuning *current, dsmc_tuning *limits);

/* Per-kernel timers of the production pass, the device-side counterpart of
 * the reference's stage timers (the Moving / Colliding / Accelerating /
 * Sampling lines of its report, dsmc/system.cpp and dsmc/dsmc_io.cpp).  With
 * timing on, dsmc_step records a CUDA event around each kernel of each pass
 * and waits for the pass to finish; turning it on or off clears the sums.
 * dsmc_pass_times_get returns the summed milliseconds of collide_cells,
 * move_cells, place_movers and place_walls and the number of timed passes. */
int dsmc_ctx_set_timing(dsmc_ctx *ctx, int on);
int dsmc_pass_times_get(dsmc_ctx *ctx, double ms[4], int64_t *passes);

/* Reads the status of the last pass: bit flags of device-side errors
 * (DSMC_EBIT_*) and the number of particles spilled to the overflow list.
 * The reference stops the process where these bits are raised (exit(1) for a
 * particle in a cell with no free volume, dsmc/system.h:137-140); here the
 * pass sets a bit and dsmc_step returns DSMC_ERR_STATE for the fatal ones. */
#define DSMC_EBIT_CELL 1u        /* a particle ended in a cell with no free volume */
#define DSMC_EBIT_FACET 2u       /* facet search found no face of the hit voxel (re-seeded, counted) */
#define DSMC_EBIT_RESEED 4u      /* re-seeding found no empty voxel within its limit */
#define DSMC_EBIT_SPILL_FULL 8u  /* the overflow list itself overflowed */
#define DSMC_EBIT_SMEM 16u       /* a cell held more particles than the staging buffer */
#define DSMC_EBIT_NAN 32u        /* non-finite position or velocity */
#define DSMC_EBIT_STRANDED 64u   /* a move ended inside solid whose cell has no free volume; the
                                    particle stays in its previous cell and is re-seeded next step */
#define DSMC_EBIT_WALL 512u      /* the Cercignani-Lampis sampler accepted nothing within its limit */
/* bits that stop the pipeline (a failed facet search or a stranded particle
 * is re-seeded, counted, and the pipeline goes on) */
#define DSMC_EBIT_FATAL \
    (DSMC_EBIT_CELL | DSMC_EBIT_RESEED | DSMC_EBIT_SPILL_FULL | DSMC_EBIT_SMEM | DSMC_EBIT_NAN | DSMC_EBIT_WALL)
int dsmc_device_status(dsmc_ctx *ctx, uint32_t *error_bits, uint32_t *spill);

/* The CUDA stream (cudaStream_t) the context enqueues its work on, for
 * callers that order or time their own work against it.  No counterpart in
 * the reference. */
void *dsmc_stream(dsmc_ctx *ctx);

/* Raw running counters of one system, without synchronising the device
 * beyond the copy: collisions, wall collisions, reseeds, particle steps,
 * count_periodic[3], samples (8 values, as int64): System::collisions,
 * ColliderBase::num_collisions and MoleculeMover::count_periodic
 * (dsmc/system.h, dsmc/colliderbase.h, dsmc/moleculemover.h:15) as the
 * sampler reads them each statistics_interval. */
int dsmc_counters_get(dsmc_ctx *ctx, int sys_id, int64_t out[8]);

#ifdef __cplusplus
}
#endif
#endif /* DSMC_B200_H */
