/*
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference DSMC
 * timestep and its sampler (andeplane/master code/base_code/program/dsmc/)
 * in fp64, used by the tests as the checker for the GPU kernels.  Nothing
 * in the shipped library includes or links it.  It is pinned against the reference's own
 * routines through the golden fixtures in tests/golden/.
 *
 * Draws come from the same counter-based streams as the kernels (philox.h):
 * one per particle and step for the mover, one per cell and step for the
 * collide, one per particle for initialisation.
 */
#ifndef DSMC_ORACLE_H
#define DSMC_ORACLE_H
#include <stdint.h>

typedef struct oracle_system {
    int n[3];               /* voxels per axis */
    int cells[3];           /* cells per axis */
    double L[3];            /* box lengths */
    double dt;
    double gravity;         /* reduced acceleration along flow_dir */
    int flow_dir;           /* <0: none */
    double wall_s;          /* sqrt(T_wall/m) */
    double sqrt_t_over_m;   /* sqrt(T/m), initial velocities */
    const unsigned char *vox;  /* voxel types, (i*ny + j)*nz + k, no halo */
    const float *nrm, *t1, *t2;
    uint64_t seed;
    int wall_model;         /* 0 thermal, 1 specular, 2 Cercignani-Lampis (dsmc/system.cpp:345-352) */
    double alpha_n, alpha_t;  /* Cercignani-Lampis accommodation */
    double cl_vmax;         /* UnitConverter::velocity_from_SI(1500) */
} oracle_system;

typedef struct oracle_counters {
    long long count_periodic[3];
    unsigned long long wall_hits, reseeds, collisions, candidates;
} oracle_counters;

/* System::setup_molecules velocities and find_position (dsmc/system.cpp:384-430). */
void oracle_init(const oracle_system *s, long n, double *r, double *v);
/* System::accelerate (dsmc/system.cpp:133-144). */
void oracle_accelerate(const oracle_system *s, long n, double *v);
/* System::move: move_molecule per particle then periodic wrap (dsmc/system.cpp:107-120). */
void oracle_move(const oracle_system *s, long n, double *r, double *v, uint32_t step, oracle_counters *c);
/* System::cell_index_from_position (dsmc/system.h:122-132): global cell index. */
int oracle_cell_of(const oracle_system *s, const double *r3);
/* System::setup_cells + Cell::update_volume (dsmc/system.cpp:432-490, dsmc/cell.cpp:27-40).
 * Returns the number of active cells; arrays may be NULL; cell_map[global] = active or -1. */
int oracle_cells_layout(const oracle_system *s, double atoms_per_molecule, double diam, int *cell_map,
                        int *global_index, int *pixels, int *total_pixels, double *volume, double *coeff);
/* Cell lists by counting sort: members of each active cell in particle-index order. */
int oracle_sort(const oracle_system *s, long n, const double *r, const int *cell_map, int num_cells, int *cell_of,
                int *count, int *start, int *members);
/* Cell::prepare + Cell::collide over every active cell (dsmc/cell.cpp:42-111). */
void oracle_collide(const oracle_system *s, int num_cells, const int *global_index, const double *coeff,
                    double *vr_max, double *rest, const int *count, const int *start, const int *members, double *v,
                    uint32_t step, oracle_counters *c);

/* The gas quantities the sampler's measurements read (System::initialize,
 * dsmc/system.cpp:252-314), reduced units. */
typedef struct oracle_gas {
    double mass, diam;
    double density;             /* number density */
    double atoms_per_molecule;
    double volume_global;       /* L_x L_y L_z times the world file's float porosity */
} oracle_gas;

/* One sample of the sampler's profiles added to `sums` (4*bins doubles: per
 * y bin {count, sum v_z, sum 1/2 m v_z^2}, then the v_x histogram over
 * [-4, 4] sqrt(temperature/mass)): MeasureCount,
 * MeasureVelocityDistributionPoiseuille, MeasureTemperatureDistribution and
 * MeasureVelocityDistribution (dsmc/statisticalproperty.cpp:229-458). */
void oracle_sample_profiles(const oracle_system *s, long n, const double *r, const double *v, double mass,
                            double temperature, int bins, double *sums);
/* The scalar measurements of one sample, in the units their files print:
 * energy (eV), temperature (K), number and volumetric flow rate (reduced),
 * pressure (Pa), permeability (darcy); `crossings` is count_periodic along
 * the flow and `elapsed` the time since the run's start
 * (dsmc/statisticalproperty.cpp:21-214). */
void oracle_measures(const oracle_system *s, const oracle_gas *g, long n, const double *v, long long crossings,
                     double elapsed, double out[6]);

#endif
