/*
 * TEST INFRASTRUCTURE: a ctypes-callable driver around the reference's own
 * System / MoleculeMover / Cell classes (andeplane/master
 * code/base_code/program/dsmc/), compiled from the reference sources by
 * oracle/Makefile.  It runs the reference's stage routines one at a time so a
 * test can compare each GPU stage against the reference on the same state and
 * the same draws:
 *
 *   refh_accelerate      -> System::accelerate           (dsmc/system.cpp:133-144)
 *   refh_move            -> MoleculeMover::move_molecule (dsmc/moleculemover.cpp:50-126)
 *                           per particle, then apply_periodic_boundary_conditions
 *                           (dsmc/moleculemover.h:29-38), as System::move
 *                           (dsmc/system.cpp:107-120) does
 *   refh_update_cells    -> System::update_molecule_cells (dsmc/system.cpp:146-157)
 *   refh_collide         -> Cell::prepare + Cell::collide (dsmc/cell.cpp:42-111)
 *                           per active cell, as System::collide
 *                           (dsmc/system.cpp:122-131) does
 *   refh_sample          -> StatisticsSampler::sample (dsmc/statisticssampler.cpp:45-66)
 *
 * The only departures from System::step are the draw source (one stream per
 * particle / per cell, selected with tape_select before each call) and
 * refh_canonicalize_cells, which orders every cell's member list by particle
 * index so the member order no longer depends on history.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#define private public
#define protected public
#include <system.h>
#include <cell.h>
#include <grid.h>
#include <moleculemover.h>
#include <colliderbase.h>
#include <settings.h>
#include <random.h>
#include <cvector.h>
#include <topology.h>
#include <statisticssampler.h>
#include <statisticalproperty.h>
#include <unitconverter.h>
#undef private
#undef protected

extern "C" void tape_select(uint64_t seed, uint32_t stream, uint32_t step, uint32_t tag);

namespace {
const uint32_t kTagMove = 1, kTagCollide = 2;
struct Handle {
    Settings *settings;
    System *system;
};
System *sys_of(void *h) { return static_cast<Handle *>(h)->system; }
}  // namespace

extern "C" {

void *refh_create(const char *ini_path) {
    try {
        Handle *h = new Handle;
        h->settings = new Settings(std::string(ini_path));
        h->system = new System();
        h->system->initialize(h->settings, 0);
        // System::initialize leaves t0 unset; the reference's main sets it
        // to the start time before the first step (dsmc/main.cpp:51-52), and
        // the flow-rate measurement divides by t - t0
        h->system->t0 = h->system->t;
        return h;
    } catch (std::string &e) {
        std::fprintf(stderr, "refh_create: %s\n", e.c_str());
        return nullptr;
    }
}

long refh_num_particles(void *h) { return sys_of(h)->num_molecules_local; }
int refh_num_active_cells(void *h) { return (int)sys_of(h)->active_cells.size(); }
int refh_max_particles(void *h) { return sys_of(h)->MAX_MOLECULE_NUM; }
double refh_dt(void *h) { return sys_of(h)->dt; }
double refh_porosity(void *h) { return sys_of(h)->porosity; }

void refh_grid_dims(void *h, unsigned *out9) {
    Grid *g = sys_of(h)->world_grid;
    unsigned v[9] = {g->nx, g->ny, g->nz, g->global_nx, g->global_ny, g->global_nz,
                     g->nx_per_cpu, g->ny_per_cpu, g->nz_per_cpu};
    std::memcpy(out9, v, sizeof(v));
}

/* Copies the centre (non-halo) block of the world grid: voxel types and the
 * normal / tangent arrays, in the reference's i*ny*nz + j*nz + k order. */
void refh_grid_core(void *h, unsigned char *vox, float *n, float *t1, float *t2) {
    Grid *g = sys_of(h)->world_grid;
    unsigned gx = g->nx_per_cpu, gy = g->ny_per_cpu, gz = g->nz_per_cpu;
    size_t o = 0;
    for (unsigned i = 0; i < gx; ++i)
        for (unsigned j = 0; j < gy; ++j)
            for (unsigned k = 0; k < gz; ++k, ++o) {
                size_t src = (size_t)(i + gx) * g->ny * g->nz + (size_t)(j + gy) * g->nz + (k + gz);
                vox[o] = g->voxels[src];
                for (int a = 0; a < 3; ++a) {
                    n[3 * o + a] = g->normals[3 * src + a];
                    t1[3 * o + a] = g->tangents1[3 * src + a];
                    t2[3 * o + a] = g->tangents2[3 * src + a];
                }
            }
}

void refh_cell_info(void *h, int *global_index, int *pixels, int *total_pixels, double *volume,
                    double *coeff, double *vr_max, double *rest, int *num_molecules) {
    System *s = sys_of(h);
    for (size_t i = 0; i < s->active_cells.size(); ++i) {
        Cell *c = s->active_cells[i];
        global_index[i] = c->index;
        pixels[i] = c->pixels;
        total_pixels[i] = c->total_pixels;
        volume[i] = c->volume;
        coeff[i] = c->collision_coefficient;
        vr_max[i] = c->vr_max;
        rest[i] = c->collision_rest;
        num_molecules[i] = c->num_molecules;
    }
}

void refh_set_cell_state(void *h, const double *vr_max, const double *rest) {
    System *s = sys_of(h);
    for (size_t i = 0; i < s->active_cells.size(); ++i) {
        s->active_cells[i]->vr_max = vr_max[i];
        s->active_cells[i]->collision_rest = rest[i];
    }
}

int refh_cell_index_map(void *h, int *out, int cap) {
    System *s = sys_of(h);
    int n = (int)s->cell_index_map.size();
    for (int i = 0; i < n && i < cap; ++i) out[i] = s->cell_index_map[i];
    return n;
}

/* Replaces the particle state and rebuilds every cell list in particle-index
 * order (System::setup_molecules' add order, dsmc/system.cpp:426-428). */
int refh_set_particles(void *h, long n, const double *r, const double *v) {
    System *s = sys_of(h);
    if (n > s->MAX_MOLECULE_NUM) return -1;
    for (Cell *c : s->active_cells) c->num_molecules = 0;
    for (long i = 0; i < 3 * n; ++i) {
        s->r[i] = r[i];
        s->v[i] = v[i];
    }
    s->num_molecules_local = n;
    s->num_molecules_global = n;
    for (long i = 0; i < n; ++i) {
        Cell *c = s->cell_that_should_contain_molecule((int)i);
        c->add_molecule((int)i, s->molecule_index_in_cell, s->molecule_cell_index);
    }
    return 0;
}

void refh_get_particles(void *h, double *r, double *v, int *cell_global) {
    System *s = sys_of(h);
    long n = s->num_molecules_local;
    for (long i = 0; i < 3 * n; ++i) {
        r[i] = s->r[i];
        v[i] = s->v[i];
    }
    if (cell_global)
        for (long i = 0; i < n; ++i) cell_global[i] = s->molecule_cell_index[i];
}

/* Member list of active cell `cell`; returns its length. */
int refh_cell_members(void *h, int cell, int *out, int cap) {
    Cell *c = sys_of(h)->active_cells.at(cell);
    for (int i = 0; i < c->num_molecules && i < cap; ++i) out[i] = c->molecules[i];
    return c->num_molecules;
}

void refh_canonicalize_cells(void *h) {
    System *s = sys_of(h);
    for (Cell *c : s->active_cells) {
        std::sort(c->molecules.begin(), c->molecules.begin() + c->num_molecules);
        for (int i = 0; i < c->num_molecules; ++i) s->molecule_index_in_cell[c->molecules[i]] = i;
    }
}

/* System::setup_molecules (dsmc/system.cpp:398-430) with one draw stream per
 * particle (id n, step 0, init tag): three next_gauss velocities times
 * sqrt(T/m), then the reference's own find_position. */
int refh_init_particles(void *h, uint64_t seed, long n) {
    System *s = sys_of(h);
    if (n > s->MAX_MOLECULE_NUM) return -1;
    for (Cell *c : s->active_cells) c->num_molecules = 0;
    s->num_molecules_local = n;
    s->num_molecules_global = n;
    const double sqrt_temp_over_mass = std::sqrt(s->temperature / s->settings->mass);
    for (long i = 0; i < n; ++i) {
        tape_select(seed, (uint32_t)i, 0u, 3u);
        s->v[3 * i + 0] = s->rnd->next_gauss() * sqrt_temp_over_mass;
        s->v[3 * i + 1] = s->rnd->next_gauss() * sqrt_temp_over_mass;
        s->v[3 * i + 2] = s->rnd->next_gauss() * sqrt_temp_over_mass;
        s->find_position((int)i);
        Cell *c = s->cell_that_should_contain_molecule((int)i);
        c->add_molecule((int)i, s->molecule_index_in_cell, s->molecule_cell_index);
    }
    return 0;
}

void refh_accelerate(void *h) { sys_of(h)->accelerate(); }

void refh_move(void *h, uint64_t seed, uint32_t step) {
    System *s = sys_of(h);
    CVector system_length(s->length[0], s->length[1], s->length[2]);
    for (int n = 0; n < s->num_molecules_local; ++n) {
        tape_select(seed, (uint32_t)n, step, kTagMove);
        int idx = n;
        s->mover->move_molecule(idx, s->dt, s->rnd, 0);
    }
    for (int n = 0; n < s->num_molecules_local; ++n) {
        int idx = n;
        s->mover->apply_periodic_boundary_conditions(idx, s->r, system_length);
    }
}

void refh_update_cells(void *h) { sys_of(h)->update_molecule_cells(); }

void refh_collide(void *h, uint64_t seed, uint32_t step) {
    System *s = sys_of(h);
    for (size_t i = 0; i < s->active_cells.size(); ++i) {
        Cell *c = s->active_cells[i];
        tape_select(seed, (uint32_t)c->index, step, kTagCollide);
        c->prepare();
        s->collisions += c->collide(s->rnd);
    }
}

void refh_counters(void *h, long *count_periodic3, unsigned long *collisions, unsigned long *wall_collisions) {
    System *s = sys_of(h);
    for (int a = 0; a < 3; ++a) count_periodic3[a] = s->mover->count_periodic[a];
    *collisions = s->collisions;
    *wall_collisions = s->mover->surface_collider->num_collisions;
}

void refh_reset_counters(void *h) {
    System *s = sys_of(h);
    for (int a = 0; a < 3; ++a) s->mover->count_periodic[a] = 0;
    s->collisions = 0;
    s->mover->surface_collider->num_collisions = 0;
}

// The reference's StatisticsSampler (dsmc/statisticssampler.cpp:13-42) over
// the harness's System.  refh_sample advances System::steps and t to `step`
// as System::step does (steps += 1; t += dt, dsmc/system.cpp:24-26) and runs
// StatisticsSampler::sample as dsmc/main.cpp:57-64 does after each step.
void *refh_sampler_create(void *h) { return new StatisticsSampler(sys_of(h)); }
void refh_sample(void *h, void *smp, uint32_t step) {
    System *s = sys_of(h);
    while ((uint32_t)s->steps < step) {
        s->steps += 1;
        s->t += s->dt;
    }
    static_cast<StatisticsSampler *>(smp)->sample();
}
// The current values of the scalar measurements, in the units their file
// lines use: energy (eV), temperature (K), number and volumetric flow rate
// (reduced), pressure (Pa), permeability (darcy).
void refh_measures(void *h, void *smp, double *out6) {
    StatisticsSampler *S = static_cast<StatisticsSampler *>(smp);
    UnitConverter *u = sys_of(h)->unit_converter;
    out6[0] = u->energy_to_eV(S->energy->get_current_value());
    out6[1] = u->temperature_to_SI(S->temperature->get_current_value());
    out6[2] = S->number_flow_rate->get_current_value();
    out6[3] = S->volumetric_flow_rate->get_current_value();
    out6[4] = u->pressure_to_SI(S->pressure->get_current_value());
    out6[5] = u->permeability_to_darcy(S->permeability->get_current_value());
}
// Profile sums: per y bin {MeasureCount, MeasureVelocityDistributionPoiseuille,
// MeasureTemperatureDistribution} sums, then MeasureVelocityDistribution's
// histogram; 4*bins doubles.  Returns bins (negative when cap is short).
int refh_profile_sums(void *smp, int cap, double *out) {
    StatisticsSampler *S = static_cast<StatisticsSampler *>(smp);
    const int b = S->count->value.number_of_bins;
    if (cap < 4 * b) return -b;
    std::vector<unsigned long> c = S->count->get_sum();
    std::vector<double> vz = S->velocity->value.get_sum();
    std::vector<double> e = S->temperature_distribution->value.get_sum();
    std::vector<long> hx = S->velocity_distribution->value.get_sum();
    for (int i = 0; i < b; ++i) {
        out[3 * i] = (double)c[i];
        out[3 * i + 1] = vz[i];
        out[3 * i + 2] = e[i];
        out[3 * b + i] = (double)hx[i];
    }
    return b;
}
// The finished profiles in SI units as each finalize() prints them
// (dsmc/statisticalproperty.cpp:303-309, 364-371, 419-426, 462-478), at full
// precision: v_z, temperature and pressure per y bin, v_x bin centres.
int refh_profiles_finish(void *h, void *smp, int cap, double *vz, double *T, double *P, double *vx_center) {
    System *sys = sys_of(h);
    StatisticsSampler *S = static_cast<StatisticsSampler *>(smp);
    UnitConverter *u = sys->unit_converter;
    const int b = S->count->value.number_of_bins;
    if (cap < b) return -b;
    std::vector<double> a = S->velocity->get_average();
    std::vector<double> t = S->temperature_distribution->get_average();
    std::vector<double> p = S->pressure_distribution->get_average(sys);
    MeasureVelocityDistribution *vd = S->velocity_distribution;
    for (int i = 0; i < b; ++i) {
        vz[i] = u->velocity_to_SI(a[i]);
        T[i] = u->temperature_to_SI(t[i]);
        P[i] = u->pressure_to_SI(p[i]);
        vx_center[i] = u->velocity_to_SI(vd->v_min + (i + 0.5) * vd->bin_size);
    }
    return b;
}

int refh_voxel_index(void *h, const double *r3) { return sys_of(h)->world_grid->get_index_of_voxel(r3); }
int refh_cell_index_of(void *h, long n) { return sys_of(h)->cell_index_from_position((int)n); }

}  // extern "C"
