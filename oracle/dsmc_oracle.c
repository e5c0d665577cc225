/*
 * TEST INFRASTRUCTURE ONLY: plain-C restatement of the reference DSMC
 * timestep in fp64 (see dsmc_oracle.h).  Each routine cites the reference
 * routine it restates (paths inside code/base_code/program/).  Built with
 * -ffp-contract=off so every product and sum rounds on its own, as in the
 * reference's x86-64 build.
 */
#define _DEFAULT_SOURCE
#include "dsmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "philox.h"

enum { EMPTY = 0, WALL = 1, BOUNDARY = 2 };

/* ---- draws ------------------------------------------------------------ */
typedef struct {
    uint64_t seed;
    uint32_t stream, step, tag;
    uint64_t k;
} draws;

static double uni(draws *d) { return oracle_uniform64(d->seed, d->stream, d->step, d->tag, d->k++); }
/* Random::next_gauss (dsmc/random.cpp:21-25), log(1-U) draw first */
static double gauss(draws *d) {
    double u1 = uni(d);
    double u2 = uni(d);
    return sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307 * u2);
}

/* ---- grid --------------------------------------------------------------- */
static int wrap(int c, int n) {
    int x = c % n;
    return x < 0 ? x + n : x;
}
static int type_at(const oracle_system *s, int i, int j, int k) {
    return s->vox[((size_t)wrap(i, s->n[0]) * s->n[1] + wrap(j, s->n[1])) * s->n[2] + wrap(k, s->n[2])];
}
static size_t lin_at(const oracle_system *s, const int u[3]) {
    return ((size_t)wrap(u[0], s->n[0]) * s->n[1] + wrap(u[1], s->n[1])) * s->n[2] + wrap(u[2], s->n[2]);
}
/* Grid::get_index_of_voxel (dsmc/grid.h:139-145) with the float-rounded
 * constants of dsmc/grid.cpp:41-46 (one rank): coordinates relative to the
 * box, in [-n, 2n) for the reference's 3x halo grid. */
static void voxel_of(const oracle_system *s, const double r[3], int u[3]) {
    for (int d = 0; d < 3; ++d) {
        const double scale = (double)(float)((1.0 / s->L[d]) * s->n[d]);
        const double shift = (double)(float)(-0.0 * (1.0 / s->L[d]) * s->n[d] + (double)s->n[d]);
        u[d] = (int)(r[d] * scale + shift) - s->n[d];
    }
}

/* ---- CVector arithmetic of the facet test (dsmc/cvector.h, dsmc/grid.h:14-41) */
typedef struct {
    double x, y, z;
} vec;
static vec mk(double x, double y, double z) {
    vec v = {x, y, z};
    return v;
}
static vec sub(vec a, vec b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static vec add(vec a, vec b) { return mk(b.x + a.x, b.y + a.y, b.z + a.z); }
static vec scl(vec a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static double dot(vec a, vec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static vec cross(vec t, vec o) { return mk(o.y * t.z - o.z * t.y, o.z * t.x - o.x * t.z, o.x * t.y - o.y * t.x); }
static int same_side(vec p1, vec p2, vec a, vec b) {
    vec e = sub(b, a);
    return dot(cross(e, sub(p1, a)), cross(e, sub(p2, a))) >= 0;
}
static int in_square(vec p1, vec p2, vec p3, vec p4, vec pt) {
    vec c = scl(add(add(add(p1, p2), p3), p4), 0.25);
    return same_side(pt, c, p1, p2) && same_side(pt, c, p2, p3) && same_side(pt, c, p3, p4) &&
           same_side(pt, c, p4, p1);
}

/* Grid::get_time_until_collision (dsmc/grid.h:82-137): earliest positive
 * crossing of a face of voxel b whose hit point lies in that face; 0 below
 * 1e-5, else minus 1e-7.  *found = 0 when no face qualifies. */
static double facet_time(const oracle_system *s, const double r[3], const double v[3], const int b[3], int *found) {
    const vec R = mk(r[0] - 0.0, r[1] - 0.0, r[2] - 0.0), V = mk(v[0], v[1], v[2]);
    const double h0 = s->L[0] / s->n[0], h1 = s->L[1] / s->n[1], h2 = s->L[2] / s->n[2];
    const int i = b[0], j = b[1], k = b[2];
    vec P[8];
    P[0] = mk(i * h0, j * h1, k * h2);
    P[1] = mk((i + 1) * h0, j * h1, k * h2);
    P[2] = mk(i * h0, j * h1, (k + 1) * h2);
    P[3] = mk((i + 1) * h0, j * h1, (k + 1) * h2);
    P[4] = mk(i * h0, (j + 1) * h1, k * h2);
    P[5] = mk((i + 1) * h0, (j + 1) * h1, k * h2);
    P[6] = mk(i * h0, (j + 1) * h1, (k + 1) * h2);
    P[7] = mk((i + 1) * h0, (j + 1) * h1, (k + 1) * h2);
    const vec N[6] = {mk(-1, 0, 0), mk(1, 0, 0), mk(0, -1, 0), mk(0, 1, 0), mk(0, 0, -1), mk(0, 0, 1)};
    const int plane[6] = {2, 1, 0, 4, 0, 2};
    const int sq[6][4] = {{4, 0, 2, 6}, {1, 5, 7, 3}, {0, 1, 3, 2}, {5, 4, 6, 7}, {4, 5, 1, 0}, {2, 3, 7, 6}};
    double best = 1e9;
    *found = 0;
    for (int f = 0; f < 6; ++f) {
        const double t = dot(sub(P[plane[f]], R), N[f]) / dot(V, N[f]);
        const int hit = in_square(P[sq[f][0]], P[sq[f][1]], P[sq[f][2]], P[sq[f][3]], add(R, scl(V, t)));
        if (t > 0 && t < best && hit && !isnan(t)) {
            best = t;
            *found = 1;
        }
    }
    if (best < 1e-5) return 0;
    return best - 1e-7;
}

/* System::find_position (dsmc/system.cpp:384-396) with Grid::get_voxel(r, n)
 * (dsmc/grid.cpp:63-69). */
static void find_position(const oracle_system *s, double r[3], draws *d) {
    for (long tries = 0; tries < 100000000L; ++tries) {
        for (int a = 0; a < 3; ++a) r[a] = 0.0 + s->L[a] * uni(d);
        int u[3];
        for (int a = 0; a < 3; ++a) u[a] = (int)((r[a] - 0.0) * (1.0 / s->L[a]) * (double)s->n[a] + (double)s->n[a]) - s->n[a];
        if (type_at(s, u[0], u[1], u[2]) < WALL) return;
    }
}

/* ColliderThermal::collide (dsmc/colliderthermal.cpp:13-46). */
/* Random::bessel_i0 (dsmc/random.cpp:27-40): the modified Bessel function I0
 * by Abramowitz & Stegun (1964) 9.8.1 and 9.8.2, in the reference's nesting. */
static double bessel_i0(double x) {
    const double ax = fabs(x);
    if (ax < 3.75) {
        double y = x / 3.75;
        y *= y;
        return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 + y * (0.360768e-1 +
                                                                                               y * 0.45813e-2)))));
    }
    const double y = 3.75 / ax;
    return (exp(ax) / sqrt(ax)) *
           (0.39894228 +
            y * (0.1328592e-1 +
                 y * (0.225319e-2 +
                      y * (-0.157565e-2 +
                           y * (0.916281e-2 +
                                y * (-0.2057706e-1 + y * (0.2635537e-1 + y * (-0.1647633e-1 + y * 0.392377e-2))))))));
}

/* Random::next_cercignani_lampis_normal_component (dsmc/random.cpp:70-91):
 * rejection sampling; 0 with *ok = 0 when 100000 trials accept nothing. */
static double cl_normal(const oracle_system *s, double v_norm_in, double factor, double max_v_out, draws *d,
                        int *ok) {
    max_v_out /= factor;
    v_norm_in /= factor;
    const double std_dev = sqrt(s->alpha_n / 2);
    const double mu = sqrt(1 - s->alpha_n) * v_norm_in;
    const double k = sqrt(1 - s->alpha_n) / s->alpha_n;
    for (long trial = 0; trial < 100000; ++trial) {
        const double v_out = std_dev * gauss(d) + mu;
        const double u = uni(d);
        const double arg = 2 * k * v_norm_in * v_out;
        const double bb = v_out * exp(-arg) * bessel_i0(arg) / max_v_out;
        if (bb >= u) {
            *ok = 1;
            return v_out * factor;
        }
    }
    *ok = 0;
    return 0;
}

/* ColliderThermal (dsmc/colliderthermal.cpp:13-46), ColliderSpecular
 * (dsmc/colliderspecular.cpp:8-32) or ColliderCercignaniLampis
 * (dsmc/collidercercignanilampis.cpp:13-45): float wall frames, double
 * velocities, as the reference mixes them. */
static void reflect(const oracle_system *s, const int b[3], double v[3], draws *d) {
    if (s->wall_model == 1 || s->wall_model == 2) {
        const size_t q = 3 * lin_at(s, b);
        const float *n = s->nrm + q, *a = s->t1 + q, *t = s->t2 + q;
        if (s->wall_model == 1) {
            const double vn = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
            const double vt1 = a[0] * v[0] + a[1] * v[1] + a[2] * v[2];
            const double vt2 = t[0] * v[0] + t[1] * v[1] + t[2] * v[2];
            for (int k = 0; k < 3; ++k) v[k] = -vn * n[k] + vt1 * a[k] + vt2 * t[k];
            return;
        }
        const double factor = sqrt(2.0) * s->wall_s;
        const double vni = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
        const double vt1i = v[0] * a[0] + v[1] * a[1] + v[2] * a[2];
        const double vt2i = v[0] * t[0] + v[1] * t[1] + v[2] * t[2];
        int ok = 0;
        const double vn = cl_normal(s, vni, factor, s->cl_vmax, d, &ok);
        if (!ok) return;  /* the GPU flags DSMC_EBIT_WALL and keeps the velocity */
        const double sigma = 1 - sqrt(1 - s->alpha_t);
        const double vt1 = gauss(d) * sqrt(s->alpha_t) * s->wall_s + vt1i * (1 - sigma);
        const double vt2 = gauss(d) * sqrt(s->alpha_t) * s->wall_s + vt2i * (1 - sigma);
        for (int k = 0; k < 3; ++k) v[k] = vn * n[k] + vt1 * a[k] + vt2 * t[k];
        return;
    }
    const double vn = s->wall_s * sqrt(-2 * log(uni(d)));
    const double vt1 = s->wall_s * gauss(d);
    const double vt2 = s->wall_s * gauss(d);
    const size_t q = 3 * lin_at(s, b);
    for (int a = 0; a < 3; ++a) v[a] = vn * s->nrm[q + a] + vt1 * s->t1[q + a] + vt2 * s->t2[q + a];
}

static void advance(double r[3], const double v[3], double tau) {
    for (int a = 0; a < 3; ++a) r[a] += v[a] * tau;
}

/* MoleculeMover::move_molecule (dsmc/moleculemover.cpp:50-126), recursion
 * written as a loop over depth. */
static void move_one(const oracle_system *s, double r[3], double v[3], draws *d, oracle_counters *c) {
    double dt = s->dt;
    int u[3];
    for (int depth = 0;; ++depth) {
        double tau = dt;
        voxel_of(s, r, u);
        if (type_at(s, u[0], u[1], u[2]) != EMPTY) {
            c->reseeds++;
            find_position(s, r, d);
            return;
        }
        advance(r, v, tau);
        voxel_of(s, r, u);
        int t = type_at(s, u[0], u[1], u[2]);
        if (t < WALL) return;
        int count = 0;
        while (t != BOUNDARY) {
            if (++count > 100) {
                c->reseeds++;
                find_position(s, r, d);
                return;
            }
            if (t == WALL) {
                tau /= 2;
                advance(r, v, -tau);
                voxel_of(s, r, u);
                t = type_at(s, u[0], u[1], u[2]);
            } else {
                dt -= tau;
                if (dt > 1e-5 && depth < 10) goto next_depth;
                return;
            }
        }
        {
            int b[3] = {u[0], u[1], u[2]};
            count = 0;
            while (t == BOUNDARY) {
                if (++count > 100) {
                    c->reseeds++;
                    find_position(s, r, d);
                    return;
                }
                b[0] = u[0];
                b[1] = u[1];
                b[2] = u[2];
                advance(r, v, -tau);
                int found;
                tau = facet_time(s, r, v, b, &found);
                if (!found) { /* the reference would fly off; the kernels re-seed */
                    c->reseeds++;
                    find_position(s, r, d);
                    return;
                }
                advance(r, v, tau);
                voxel_of(s, r, u);
                t = type_at(s, u[0], u[1], u[2]);
            }
            dt -= tau;
            reflect(s, b, v, d);
            c->wall_hits++;
        }
        if (!(dt > 1e-5 && depth < 10)) return;
    next_depth:;
    }
}

void oracle_init(const oracle_system *s, long n, double *r, double *v) {
    for (long i = 0; i < n; ++i) {
        draws d = {s->seed, (uint32_t)i, 0u, ORACLE_TAG_INIT, 0};
        for (int a = 0; a < 3; ++a) v[3 * i + a] = gauss(&d) * s->sqrt_t_over_m;
        find_position(s, r + 3 * i, &d);
    }
}

void oracle_accelerate(const oracle_system *s, long n, double *v) {
    if (s->flow_dir < 0 || s->gravity == 0) return;
    const double g = s->gravity * s->dt;
    for (long i = 0; i < n; ++i) v[3 * i + s->flow_dir] += g;
}

void oracle_move(const oracle_system *s, long n, double *r, double *v, uint32_t step, oracle_counters *c) {
    for (long i = 0; i < n; ++i) {
        draws d = {s->seed, (uint32_t)i, step, ORACLE_TAG_MOVE, 0};
        move_one(s, r + 3 * i, v + 3 * i, &d, c);
    }
    /* MoleculeMover::apply_periodic_boundary_conditions (dsmc/moleculemover.h:29-38) */
    for (long i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            double *x = r + 3 * i + a;
            if (*x >= s->L[a]) {
                *x -= s->L[a];
                c->count_periodic[a]++;
            } else if (*x < 0) {
                *x += s->L[a];
                c->count_periodic[a]--;
            }
        }
}

int oracle_cell_of(const oracle_system *s, const double *r3) {
    int ci[3];
    for (int a = 0; a < 3; ++a) ci[a] = (int)(r3[a] * (1.0 / s->L[a]) * s->cells[a]);
    return ci[0] * s->cells[1] * s->cells[2] + ci[1] * s->cells[2] + ci[2];
}

int oracle_cells_layout(const oracle_system *s, double apm, double diam, int *cell_map, int *global_index,
                        int *pixels, int *total_pixels, double *volume, double *coeff) {
    const int cx = s->cells[0], cy = s->cells[1], cz = s->cells[2], nc = cx * cy * cz;
    int *first = malloc(sizeof(int) * nc), *order = malloc(sizeof(int) * nc);
    int *tot = calloc(nc, sizeof(int)), *pix = calloc(nc, sizeof(int));
    int touched = 0;
    for (int q = 0; q < nc; ++q) first[q] = -1;
    for (int k = 0; k < s->n[2]; ++k) {
        const int c_z = (int)((float)k / (unsigned)s->n[2] * cz);
        for (int j = 0; j < s->n[1]; ++j) {
            const int c_y = (int)((float)j / (unsigned)s->n[1] * cy);
            for (int i = 0; i < s->n[0]; ++i) {
                const int c_x = (int)((float)i / (unsigned)s->n[0] * cx);
                const int g = c_x * cy * cz + c_y * cz + c_z;
                if (first[g] < 0) {
                    first[g] = touched;
                    order[touched++] = g;
                }
                tot[first[g]]++;
                pix[first[g]] += s->vox[((size_t)i * s->n[1] + j) * s->n[2] + k] < WALL;
            }
        }
    }
    const double system_volume = s->L[0] * s->L[1] * s->L[2];
    int a = 0;
    if (cell_map)
        for (int q = 0; q < nc; ++q) cell_map[q] = -1;
    for (int q = 0; q < touched; ++q) {
        if (pix[q] == 0) continue;
        const double vol = system_volume / (nc) * (float)pix[q] / tot[q];
        if (cell_map) cell_map[order[q]] = a;
        if (global_index) global_index[a] = order[q];
        if (pixels) pixels[a] = pix[q];
        if (total_pixels) total_pixels[a] = tot[q];
        if (volume) volume[a] = vol;
        if (coeff) coeff[a] = 0.5 * apm * M_PI * diam * diam * s->dt / vol;
        ++a;
    }
    free(first);
    free(order);
    free(tot);
    free(pix);
    return a;
}

int oracle_sort(const oracle_system *s, long n, const double *r, const int *cell_map, int num_cells, int *cell_of,
                int *count, int *start, int *members) {
    memset(count, 0, sizeof(int) * num_cells);
    for (long i = 0; i < n; ++i) {
        const int a = cell_map[oracle_cell_of(s, r + 3 * i)];
        if (a < 0) return -1; /* dsmc/system.h:137-140 */
        cell_of[i] = a;
        count[a]++;
    }
    int acc = 0;
    for (int a = 0; a < num_cells; ++a) {
        start[a] = acc;
        acc += count[a];
    }
    int *fill = calloc(num_cells, sizeof(int));
    for (long i = 0; i < n; ++i) members[start[cell_of[i]] + fill[cell_of[i]]++] = (int)i;
    free(fill);
    return 0;
}

/* Cell::collide_molecules (dsmc/cell.cpp:53-73). */
static void scatter(double *v0, double *v1, double vrel, draws *d) {
    const double cmx = 0.5 * (v0[0] + v1[0]), cmy = 0.5 * (v0[1] + v1[1]), cmz = 0.5 * (v0[2] + v1[2]);
    const double cos_th = 1.0 - 2.0 * uni(d);
    const double sin_th = sqrt(1.0 - cos_th * cos_th);
    const double phi = 2 * M_PI * uni(d);
    const double rx = vrel * cos_th, ry = vrel * sin_th * cos(phi), rz = vrel * sin_th * sin(phi);
    v0[0] = cmx + 0.5 * rx;
    v0[1] = cmy + 0.5 * ry;
    v0[2] = cmz + 0.5 * rz;
    v1[0] = cmx - 0.5 * rx;
    v1[1] = cmy - 0.5 * ry;
    v1[2] = cmz - 0.5 * rz;
}

void oracle_collide(const oracle_system *s, int num_cells, const int *global_index, const double *coeff,
                    double *vr_max, double *rest, const int *count, const int *start, const int *members, double *v,
                    uint32_t step, oracle_counters *c) {
    for (int a = 0; a < num_cells; ++a) {
        const int n = count[a];
        /* Cell::prepare (dsmc/cell.cpp:42-51) */
        const double select = coeff[a] * n * (n - 1) * vr_max[a] + rest[a];
        const int pairs = (int)round(select);
        rest[a] = select - pairs;
        if (n < 2) continue;
        draws d = {s->seed, (uint32_t)global_index[a], step, ORACLE_TAG_COLLIDE, 0};
        double crm = vr_max[a];
        const int *m = members + start[a];
        for (int isel = 0; isel < pairs; ++isel) {
            const int ip0 = (int)(uni(&d) * n);
            const int ip1 = ((int)(ip0 + 1 + uni(&d) * (n - 1))) % n;
            double *v0 = v + 3 * (size_t)m[ip0], *v1 = v + 3 * (size_t)m[ip1];
            const double dx = v0[0] - v1[0], dy = v0[1] - v1[1], dz = v0[2] - v1[2];
            const double vrel = sqrt(dx * dx + dy * dy + dz * dz);
            if (vrel > crm) crm = vrel;
            if (vrel > uni(&d) * vr_max[a]) {
                c->collisions++;
                scatter(v0, v1, vrel, &d);
            }
        }
        c->candidates += pairs;
        vr_max[a] = crm;
    }
}

/* ---- sampler ------------------------------------------------------------ */
/* Reduced units of the reference (dsmc/unitconverter.cpp:3-21). */
static const double U_M0 = 1.66053886e-27, U_L0 = 1e-6, U_E0 = 1.65088e-21, U_E0EV = 1.0318e-2,
                    U_KB = 1.3806503e-23;

void oracle_sample_profiles(const oracle_system *s, long n, const double *r, const double *v, double mass,
                            double temperature, int bins, double *sums) {
    /* one sample's per-bin values, summed in particle order, then added to
     * the running sums (StatisticalValue::add_value, dsmc/statisticalvalue.h:38-46) */
    double *cnt = calloc((size_t)bins, sizeof(double));
    double *vz = calloc((size_t)bins, sizeof(double));
    double *ez = calloc((size_t)bins, sizeof(double));
    double *hx = calloc((size_t)bins, sizeof(double));
    const double one_over_ly = 1.0 / s->L[1];
    /* MeasureVelocityDistribution's histogram over [-4, 4] sqrt(T/m)
     * (dsmc/statisticalproperty.cpp:432-438) */
    const double std_dev = sqrt(temperature / mass);
    const double v_min = -4 * std_dev, v_max = 4 * std_dev;
    const double bin_size = (v_max - v_min) / bins;
    for (long i = 0; i < n; ++i) {
        /* MeasureCount, MeasureVelocityDistributionPoiseuille and
         * MeasureTemperatureDistribution bin by y (:229-244, :261-278, :322-338) */
        const int b = (int)(r[3 * i + 1] * one_over_ly * bins);
        cnt[b] += 1.0;
        vz[b] += v[3 * i + 2];
        ez[b] += 0.5 * mass * v[3 * i + 2] * v[3 * i + 2];
        /* the histogram keeps the bin of v_x only, truncated toward zero (:440-452) */
        const int bx = (int)((v[3 * i] - v_min) / bin_size);
        if (bx < 0 || bx > bins - 1) continue;
        hx[bx] += 1.0;
    }
    for (int b = 0; b < bins; ++b) {
        sums[3 * b] += cnt[b];
        sums[3 * b + 1] += vz[b];
        sums[3 * b + 2] += ez[b];
        sums[3 * bins + b] += hx[b];
    }
    free(cnt);
    free(vz);
    free(ez);
    free(hx);
}

void oracle_measures(const oracle_system *s, const oracle_gas *g, long n, const double *v, long long crossings,
                     double elapsed, double out[6]) {
    const double t0 = U_L0 * sqrt(U_M0 / U_E0);
    const double T0 = U_E0 / U_KB;
    const double P0 = U_M0 / (t0 * t0 * U_L0);
    const double perm0 = U_L0 * U_L0;
    /* MeasureEnergy (dsmc/statisticalproperty.cpp:21-41) */
    double ke = 0;
    for (long i = 0; i < n; ++i)
        ke += (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    ke *= 0.5 * g->mass * g->atoms_per_molecule;
    /* System::get_number_of_atoms_global (dsmc/system.cpp:509-511): a long */
    const long atoms = (long)((double)n * g->atoms_per_molecule);
    /* MeasureTemperature (:57-70) */
    const double T = 2.0 / 3.0 * ke / atoms;
    /* MeasureNumberFlowRate (:87-101): cumulative net crossings over the elapsed time */
    const double flux = g->atoms_per_molecule * (double)crossings / elapsed;
    /* MeasureVolumetricFlowRate (:117-131) */
    const double q = flux * (1.0 / g->density);
    /* MeasurePressure (:154-165) */
    const double P = atoms / g->volume_global * T;
    /* MeasurePermeability (:185-214): hard-sphere viscosity at the measured T */
    double area = 1;
    for (int a = 0; a < 3; ++a)
        if (a != s->flow_dir) area *= s->L[a];
    const double visc = 5.0 / (16 * g->diam * g->diam) * sqrt(g->mass * T / M_PI);
    const double k = q * visc / (area * g->mass * g->density * s->gravity);
    out[0] = U_E0EV * ke;      /* UnitConverter::energy_to_eV */
    out[1] = T0 * T;           /* temperature_to_SI */
    out[2] = flux;
    out[3] = q;
    out[4] = P0 * P;           /* pressure_to_SI */
    out[5] = k * perm0 * 1e4;  /* permeability_to_darcy */
}
