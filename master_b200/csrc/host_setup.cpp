// Host-side set-up of the DSMC timestep: settings and ini files, reduced
// units, world files and the packed-sphere geometry generator.
//
// Arithmetic that decides voxel types, normals and tangents follows the
// reference operation by operation (float vs double rounding included), so a
// geometry built here is byte-identical to the reference tool's output.  This
// file must be compiled without floating-point contraction (-ffp-contract=off).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "dsmc_b200.h"
#include "dsmc_internal.h"
#include "dsmc_layout.h"

namespace dsmc {

// ---------------------------------------------------------------------------
// Thread-local error text for calls that have no context.
static thread_local std::string g_thread_error;
void set_thread_error(const std::string &msg) { g_thread_error = msg; }
const char *thread_error() { return g_thread_error.c_str(); }

// ---------------------------------------------------------------------------
// Reduced units (dsmc/unitconverter.cpp:3-21).
Units::Units() {
    m0 = 1.66053886e-27;
    L0 = 1e-6;
    E0 = 1.65088e-21;
    E0ev = 1.0318e-2;
    kb = 1.3806503e-23;
    t0 = L0 * std::sqrt(m0 / E0);
    T0 = E0 / kb;
    v0 = L0 / t0;
    a0 = v0 / t0;
    P0 = m0 / (t0 * t0 * L0);
    number_density0 = 1.0 / (L0 * L0 * L0);
}

// ---------------------------------------------------------------------------
// Park-Miller minimal standard generator with a Bays-Durham shuffle
// ("ran1", Press et al., Numerical Recipes in C, 2nd ed., section 7.1), the
// generator the reference's geometry tool draws sphere centres and tangent
// seeds from (dsmc/random.cpp:43-68).  The geometry is an input of the
// timestep, so the same draws are needed to rebuild the same geometry.
Ran1::Ran1(long seed) : idum(seed), iy(0) { std::memset(iv, 0, sizeof(iv)); }

double Ran1::next() {
    const long IA = 16807, IM = 2147483647, IQ = 127773, IR = 2836, NTAB = 32;
    const long NDIV = 1 + (IM - 1) / NTAB;
    const double AM = 1.0 / IM, RNMX = 1.0 - 1.2e-7;
    if (idum <= 0 || !iy) {
        idum = (-idum < 1) ? 1 : -idum;
        for (long j = NTAB + 7; j >= 0; --j) {
            long k = idum / IQ;
            idum = IA * (idum - k * IQ) - IR * k;
            if (idum < 0) idum += IM;
            if (j < NTAB) iv[j] = idum;
        }
        iy = iv[0];
    }
    long k = idum / IQ;
    idum = IA * (idum - k * IQ) - IR * k;
    if (idum < 0) idum += IM;
    long j = iy / NDIV;
    iy = iv[j];
    iv[j] = idum;
    double temp = AM * iy;
    return temp > RNMX ? RNMX : temp;
}

// ---------------------------------------------------------------------------
// ini files with the reference's CIniFile rules (dsmc/cinifile.h:28-104,
// dsmc/cutil.cpp:3-93): "key = value" split on '=', empty pieces skipped,
// CR removed, spaces trimmed; numbers through strtod.
namespace {
std::string trim_spaces(const std::string &s) {
    size_t e = s.find_last_not_of(' ');
    if (e == std::string::npos) return "";
    size_t b = s.find_first_not_of(' ');
    return s.substr(b, e - b + 1);
}
}  // namespace

bool IniFile::load(const std::string &path) {
    std::ifstream f(path.c_str());
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
        size_t cr = line.find('\r');
        if (cr != std::string::npos) line.erase(cr, 1);
        std::vector<std::string> tok;
        size_t pos = 0;
        while (pos < line.size()) {
            size_t b = line.find_first_not_of('=', pos);
            if (b == std::string::npos) break;
            size_t e = line.find('=', b);
            if (e == std::string::npos) e = line.size();
            tok.push_back(line.substr(b, e - b));
            pos = e;
        }
        if (tok.size() == 2) {
            Item it;
            it.name = trim_spaces(tok[0]);
            it.str = trim_spaces(tok[1]);
            it.num = std::strtod(tok[1].c_str(), nullptr);
            items.push_back(it);
        }
    }
    return true;
}

const IniFile::Item *IniFile::find(const std::string &key) const {
    for (const Item &it : items)
        if (it.name == key) return &it;
    return nullptr;
}

}  // namespace dsmc

using namespace dsmc;

extern "C" {

int dsmc_settings_defaults(dsmc_settings *s) {
    if (!s) return DSMC_ERR_ARG;
    std::memset(s, 0, sizeof(*s));
    // The reference's Python driver defaults (dsmcconfig.py:14-77).
    s->timesteps = 10000;
    s->statistics_interval = 100;
    s->atoms_per_molecule = 1000;
    s->cells_x = s->cells_y = s->cells_z = 10;
    s->flow_direction = 2;
    s->sampling_bins = 128;
    s->seed = -1;
    s->max_molecules_per_node = 1000000;
    s->nx = s->ny = s->nz = 1;
    s->mass = 39.948;
    s->temperature = 300;
    s->wall_temperature = 300;
    s->gravity = 0;
    s->density = 2.4143e25;
    s->diam = 3.62e-4;
    s->Lx = s->Ly = s->Lz = 1;
    s->dt = 0.001;
    s->alpha_n = 0.5;
    s->alpha_t = 0.8;
    s->viscosity = 2.23e-5;
    s->surface_model = 0;
    s->sample_begin = 0;
    s->rng_seed = 0x5eed5eedULL;
    std::snprintf(s->world, sizeof(s->world), "worlds");
    return DSMC_OK;
}

int dsmc_settings_load_ini(const char *path, dsmc_settings *s) {
    if (!path || !s) return DSMC_ERR_ARG;
    IniFile ini;
    if (!ini.load(path)) {
        set_thread_error(std::string("could not load file ") + path);
        return DSMC_ERR_IO;
    }
    dsmc_settings_defaults(s);
    std::string missing;
    auto num = [&](const char *k, double &out) {
        const IniFile::Item *it = ini.find(k);
        if (!it) {
            if (missing.empty()) missing = k;
            return;
        }
        out = it->num;
    };
    auto integer = [&](const char *k, int &out) {
        double d = out;
        num(k, d);
        out = (int)d;
    };
    // Settings::Settings (dsmc/settings.cpp:3-44): every key is required.
    if (const IniFile::Item *it = ini.find("load_previous_state")) s->load_previous_state = it->str == "true";
    else missing = "load_previous_state";
    integer("statistics_interval", s->statistics_interval);
    integer("atoms_per_molecule", s->atoms_per_molecule);
    integer("timesteps", s->timesteps);
    integer("sampling_bins", s->sampling_bins);
    integer("max_molecules_per_node", s->max_molecules_per_node);
    integer("nx", s->nx);
    integer("ny", s->ny);
    integer("nz", s->nz);
    integer("cells_x", s->cells_x);
    integer("cells_y", s->cells_y);
    integer("cells_z", s->cells_z);
    integer("flow_direction", s->flow_direction);
    integer("seed", s->seed);
    num("mass", s->mass);
    num("temperature", s->temperature);
    num("wall_temperature", s->wall_temperature);
    num("gravity", s->gravity);
    num("density", s->density);
    num("diam", s->diam);
    num("Lx", s->Lx);
    num("Ly", s->Ly);
    num("Lz", s->Lz);
    num("alpha_n", s->alpha_n);
    num("alpha_t", s->alpha_t);
    num("dt", s->dt);
    num("viscosity", s->viscosity);
    const IniFile::Item *model = ini.find("surface_interaction_model");
    if (!model) {
        if (missing.empty()) missing = "surface_interaction_model";
    } else if (model->str == "thermal") {
        s->surface_model = DSMC_WALL_THERMAL;
    } else if (model->str == "specular") {
        s->surface_model = DSMC_WALL_SPECULAR;
    } else if (model->str == "cercignani_lampis") {
        s->surface_model = DSMC_WALL_CL;
    } else {
        // "maxwell" is a stub in the reference (dsmc/collidermaxwell.cpp:13-16)
        set_thread_error("surface_interaction_model '" + model->str +
                         "' has no model; thermal, specular and cercignani_lampis are built");
        return DSMC_ERR_CONFIG;
    }
    const IniFile::Item *world = ini.find("world");
    if (!world) {
        if (missing.empty()) missing = "world";
    } else {
        std::snprintf(s->world, sizeof(s->world), "%s", world->str.c_str());
    }
    if (!missing.empty()) {
        set_thread_error("Could not find any parameter '" + missing + "'");
        return DSMC_ERR_NOT_FOUND;
    }
    // Optional keys of this build.
    if (const IniFile::Item *it = ini.find("sample_begin")) s->sample_begin = (int)it->num;
    if (const IniFile::Item *it = ini.find("rng_seed")) s->rng_seed = (uint64_t)std::strtoull(it->str.c_str(), nullptr, 0);
    else s->rng_seed = (uint64_t)(uint32_t)s->seed * 0x9E3779B97F4A7C15ULL + 0x1234567ULL;
    return DSMC_OK;
}

// ---------------------------------------------------------------------------
// World files (dsmc/dsmc_io.cpp:183-220 reads; dsmc/complexgeometry.cpp:220-318 writes).
int dsmc_world_read_header(const char *path, dsmc_world_header *h) {
    if (!path || !h) return DSMC_ERR_ARG;
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        set_thread_error(std::string("Error, could not open file ") + path);
        return DSMC_ERR_IO;
    }
    size_t got = 0;
    got += std::fread(&h->porosity_global, sizeof(float), 1, f);
    got += std::fread(&h->porosity, sizeof(float), 1, f);
    got += std::fread(&h->global_nx, sizeof(uint32_t), 1, f);
    got += std::fread(&h->global_ny, sizeof(uint32_t), 1, f);
    got += std::fread(&h->global_nz, sizeof(uint32_t), 1, f);
    got += std::fread(&h->nx, sizeof(uint32_t), 1, f);
    got += std::fread(&h->ny, sizeof(uint32_t), 1, f);
    got += std::fread(&h->nz, sizeof(uint32_t), 1, f);
    std::fclose(f);
    if (got != 8) {
        set_thread_error(std::string("truncated world header in ") + path);
        return DSMC_ERR_IO;
    }
    if (h->nx == 0 || h->ny == 0 || h->nz == 0 || h->nx % 3 || h->ny % 3 || h->nz % 3) {
        set_thread_error(std::string("world dimensions are not three halo blocks in ") + path);
        return DSMC_ERR_IO;
    }
    return DSMC_OK;
}

int dsmc_world_read(const char *path, uint8_t *voxels, float *normals, float *tangents1, float *tangents2) {
    dsmc_world_header h;
    int rc = dsmc_world_read_header(path, &h);
    if (rc) return rc;
    if (!voxels || !normals || !tangents1 || !tangents2) return DSMC_ERR_ARG;
    const uint64_t bx = h.nx / 3, by = h.ny / 3, bz = h.nz / 3;
    if (bx != h.global_nx || by != h.global_ny || bz != h.global_nz) {
        set_thread_error("world file belongs to a multi-rank decomposition; read it with one rank's block");
        return DSMC_ERR_IO;
    }
    const uint64_t V = (uint64_t)h.nx * h.ny * h.nz;
    FILE *f = std::fopen(path, "rb");
    if (!f) return DSMC_ERR_IO;
    std::fseek(f, 32, SEEK_SET);
    std::vector<uint8_t> vox(V);
    std::vector<float> buf(3 * V);
    bool ok = std::fread(vox.data(), 1, V, f) == V;
    // Keep the centre block: halo block (1,1,1) is the rank's own voxels.
    auto core = [&](uint64_t i, uint64_t j, uint64_t k) {
        return ((i + bx) * h.ny + (j + by)) * h.nz + (k + bz);
    };
    const uint64_t n = bx * by * bz;
    if (ok) {
        uint64_t o = 0;
        for (uint64_t i = 0; i < bx; ++i)
            for (uint64_t j = 0; j < by; ++j)
                for (uint64_t k = 0; k < bz; ++k) voxels[o++] = vox[core(i, j, k)];
    }
    float *dst[3] = {normals, tangents1, tangents2};
    for (int a = 0; a < 3 && ok; ++a) {
        ok = std::fread(buf.data(), sizeof(float), 3 * V, f) == 3 * V;
        if (!ok) break;
        uint64_t o = 0;
        for (uint64_t i = 0; i < bx; ++i)
            for (uint64_t j = 0; j < by; ++j)
                for (uint64_t k = 0; k < bz; ++k, ++o) {
                    uint64_t s = core(i, j, k);
                    dst[a][3 * o + 0] = buf[3 * s + 0];
                    dst[a][3 * o + 1] = buf[3 * s + 1];
                    dst[a][3 * o + 2] = buf[3 * s + 2];
                }
    }
    std::fclose(f);
    (void)n;
    if (!ok) {
        set_thread_error(std::string("truncated world file ") + path);
        return DSMC_ERR_IO;
    }
    return DSMC_OK;
}

int dsmc_world_write(const char *folder, uint32_t nx, uint32_t ny, uint32_t nz, const uint8_t *voxels,
                     const float *normals, const float *tangents1, const float *tangents2, int px, int py,
                     int pz) {
    if (!folder || !voxels || !normals || !tangents1 || !tangents2 || px < 1 || py < 1 || pz < 1)
        return DSMC_ERR_ARG;
    if (nx % px || ny % py || nz % pz) return DSMC_ERR_CONFIG;
    const uint64_t V = (uint64_t)nx * ny * nz;
    uint64_t empty = 0;
    for (uint64_t i = 0; i < V; ++i) empty += voxels[i] == DSMC_VOX_EMPTY;
    const float porosity_global = (float)((double)empty / V);
    const int bx = nx / px, by = ny / py, bz = nz / pz;
    const uint64_t L = (uint64_t)27 * bx * by * bz;
    std::vector<uint8_t> lv(L);
    std::vector<float> ln(3 * L), lt1(3 * L), lt2(3 * L);
    char name[1024];
    for (int rank = 0; rank < px * py * pz; ++rank) {
        // rank index -> (x, y, z) processor coordinates (dsmc/topology.cpp:86-94)
        const int ix = rank / (py * pz), iy = (rank / pz) % py, iz = rank % pz;
        const int ox = ix * bx, oy = iy * by, oz = iz * bz;
        uint64_t o = 0, empty_local = 0, local = 0;
        for (int di = -bx; di < 2 * bx; ++di)
            for (int dj = -by; dj < 2 * by; ++dj)
                for (int dk = -bz; dk < 2 * bz; ++dk, ++o) {
                    const uint64_t i = (uint64_t)((ox + di + 10 * (int)nx) % (int)nx);
                    const uint64_t j = (uint64_t)((oy + dj + 10 * (int)ny) % (int)ny);
                    const uint64_t k = (uint64_t)((oz + dk + 10 * (int)nz) % (int)nz);
                    const uint64_t g = (i * ny + j) * nz + k;
                    lv[o] = voxels[g];
                    for (int a = 0; a < 3; ++a) {
                        ln[3 * o + a] = normals[3 * g + a];
                        lt1[3 * o + a] = tangents1[3 * g + a];
                        lt2[3 * o + a] = tangents2[3 * g + a];
                    }
                    if (di >= 0 && di < bx && dj >= 0 && dj < by && dk >= 0 && dk < bz) {
                        empty_local += voxels[g] == DSMC_VOX_EMPTY;
                        ++local;
                    }
                }
        float porosity = local ? (float)empty_local / local : 0.0f;
        uint32_t dims[6] = {nx, ny, nz, (uint32_t)(3 * bx), (uint32_t)(3 * by), (uint32_t)(3 * bz)};
        std::snprintf(name, sizeof(name), "%s/%04d.bin", folder, rank);
        FILE *f = std::fopen(name, "wb");
        if (!f) {
            set_thread_error(std::string("Could not open ") + name);
            return DSMC_ERR_IO;
        }
        bool ok = std::fwrite(&porosity_global, sizeof(float), 1, f) == 1;
        ok = ok && std::fwrite(&porosity, sizeof(float), 1, f) == 1;
        ok = ok && std::fwrite(dims, sizeof(uint32_t), 6, f) == 6;
        ok = ok && std::fwrite(lv.data(), 1, L, f) == L;
        ok = ok && std::fwrite(ln.data(), sizeof(float), 3 * L, f) == 3 * L;
        ok = ok && std::fwrite(lt1.data(), sizeof(float), 3 * L, f) == 3 * L;
        ok = ok && std::fwrite(lt2.data(), sizeof(float), 3 * L, f) == 3 * L;
        std::fclose(f);
        if (!ok) return DSMC_ERR_IO;
    }
    std::snprintf(name, sizeof(name), "%s/porosity.txt", folder);
    FILE *f = std::fopen(name, "wb");
    if (!f) return DSMC_ERR_IO;
    std::fprintf(f, "%f", porosity_global);
    std::fclose(f);
    return DSMC_OK;
}

// ---------------------------------------------------------------------------
// Geometry (dsmc/complexgeometry.cpp).
int dsmc_geometry_finish(uint32_t nx, uint32_t ny, uint32_t nz, int avg, uint8_t *vox, float *nrm, float *t1,
                         float *t2) {
    if (!vox || !nrm || !t1 || !t2 || nx == 0 || ny == 0 || nz == 0 || avg < 0) return DSMC_ERR_ARG;
    const uint64_t V = (uint64_t)nx * ny * nz;
    const int X = nx, Y = ny, Z = nz;
    std::memset(nrm, 0, 3 * V * sizeof(float));
    std::memset(t1, 0, 3 * V * sizeof(float));
    std::memset(t2, 0, 3 * V * sizeof(float));
    // The reference takes sqrt of float sums, which resolves to the float
    // overload (std::sqrt(float)), then divides in double; both are kept.
    // Normals: minus the first moment of the solid indicator over the 27
    // neighbours; if non-zero, redone over the (2a+1)^3 window; normalised.
    // Voxels are visited in i, j, k order and a solid voxel with no normal and
    // an empty neighbour is emptied in place, so later voxels see the change
    // (calculate_normals, dsmc/complexgeometry.cpp:928-999).
    for (int i = 0; i < X; ++i)
        for (int j = 0; j < Y; ++j)
            for (int k = 0; k < Z; ++k) {
                const uint64_t idx = ((uint64_t)i * Y + j) * Z + k;
                bool any_solid = false, all_solid = true;
                float n0 = 0.f, n1 = 0.f, n2 = 0.f;
                for (int di = -1; di <= 1; ++di)
                    for (int dj = -1; dj <= 1; ++dj)
                        for (int dk = -1; dk <= 1; ++dk) {
                            const uint64_t q = ((uint64_t)((i + di + X) % X) * Y + (j + dj + Y) % Y) * Z +
                                               (k + dk + Z) % Z;
                            const int s = vox[q];
                            if (s > 0) any_solid = true;
                            if (s == 0) all_solid = false;
                            n0 -= s * di;
                            n1 -= s * dj;
                            n2 -= s * dk;
                        }
                const double norm_sq = n0 * n0 + n1 * n1 + n2 * n2;
                if (norm_sq > 0) {
                    n0 = n1 = n2 = 0.f;
                    for (int di = -avg; di <= avg; ++di)
                        for (int dj = -avg; dj <= avg; ++dj)
                            for (int dk = -avg; dk <= avg; ++dk) {
                                const uint64_t q = ((uint64_t)((i + di + X) % X) * Y + (j + dj + Y) % Y) * Z +
                                                   (k + dk + Z) % Z;
                                const int s = vox[q];
                                n0 -= s * di;
                                n1 -= s * dj;
                                n2 -= s * dk;
                            }
                }
                const double norm = (double)std::sqrt((float)(n0 * n0 + n1 * n1 + n2 * n2));
                if (norm > 0) {
                    n0 = (float)(n0 / norm);
                    n1 = (float)(n1 / norm);
                    n2 = (float)(n2 / norm);
                } else if (!any_solid || !all_solid) {
                    vox[idx] = 0;
                }
                nrm[3 * idx + 0] = n0;
                nrm[3 * idx + 1] = n1;
                nrm[3 * idx + 2] = n2;
            }
    // Tangents: a ran1(-1) seed vector per voxel, Gram-Schmidt against the
    // normal, t2 = t1 x n (calculate_tangents, dsmc/complexgeometry.cpp:1001-1046).
    Ran1 rnd(-1);
    for (uint64_t idx = 0; idx < V; ++idx) {
        const float n0 = nrm[3 * idx], n1 = nrm[3 * idx + 1], n2 = nrm[3 * idx + 2];
        float a0 = (float)rnd.next(), a1 = (float)rnd.next(), a2 = (float)rnd.next();
        const double dot = n0 * a0 + n1 * a1 + n2 * a2;
        a0 = (float)(a0 - n0 * dot);
        a1 = (float)(a1 - n1 * dot);
        a2 = (float)(a2 - n2 * dot);
        double norm = (double)std::sqrt((float)(a0 * a0 + a1 * a1 + a2 * a2));
        if (norm > 0) {
            a0 = (float)(a0 / norm);
            a1 = (float)(a1 / norm);
            a2 = (float)(a2 / norm);
        }
        float b0 = a1 * n2 - a2 * n1;
        float b1 = a2 * n0 - a0 * n2;
        float b2 = a0 * n1 - a1 * n0;
        norm = (double)std::sqrt((float)(b0 * b0 + b1 * b1 + b2 * b2));
        if (norm > 0) {
            b0 = (float)(b0 / norm);
            b1 = (float)(b1 / norm);
            b2 = (float)(b2 / norm);
        }
        t1[3 * idx] = a0;
        t1[3 * idx + 1] = a1;
        t1[3 * idx + 2] = a2;
        t2[3 * idx] = b0;
        t2[3 * idx + 1] = b1;
        t2[3 * idx + 2] = b2;
    }
    // Boundary voxels: solid with a non-zero normal (find_boundary_points,
    // dsmc/complexgeometry.cpp:1048-1063).
    for (uint64_t idx = 0; idx < V; ++idx) {
        const double nn = nrm[3 * idx] * nrm[3 * idx] + nrm[3 * idx + 1] * nrm[3 * idx + 1] +
                          nrm[3 * idx + 2] * nrm[3 * idx + 2];
        if (vox[idx] > 0 && nn > 0) vox[idx] = DSMC_VOX_BOUNDARY;
    }
    return DSMC_OK;
}

int dsmc_geometry_packed_spheres(const dsmc_sphere_params *p, uint8_t *vox, float *nrm, float *t1, float *t2,
                                 float *porosity_out) {
    if (!p || !vox || !nrm || !t1 || !t2 || p->nx < 2 || p->ny < 2 || p->nz < 2) return DSMC_ERR_ARG;
    if (p->spheres_type == 1 && !(p->wanted_porosity > 0 && p->wanted_porosity < 1)) return DSMC_ERR_ARG;
    const int X = p->nx, Y = p->ny, Z = p->nz;
    const uint64_t V = (uint64_t)X * Y * Z;
    const bool inverted = p->inverted != 0;
    const double r2 = p->radius * p->radius;
    const float vsx = 1.0 / X, vsy = 1.0 / Y, vsz = 1.0 / Z;
    const int hx = X / 2, hy = Y / 2, hz = Z / 2;
    std::memset(vox, inverted ? 0 : 1, V);
    Ran1 rnd(-std::abs(p->seed));
    std::vector<double> centres;
    // Voxels only ever change to `inverted`, so the empty count of the octant
    // can be kept incrementally; each sphere only visits its bounding box.
    int64_t empty = inverted ? (int64_t)hx * hy * hz : 0;
    const uint64_t max_spheres = 100000000ULL;
    for (uint64_t s = 0;; ++s) {
        if (s > max_spheres) {
            set_thread_error("packed spheres: wanted porosity not reached");
            return DSMC_ERR_CONFIG;
        }
        double x0 = rnd.next() * 0.5, y0 = rnd.next() * 0.5, z0 = rnd.next() * 0.5;
        bool overlap = true;
        while (p->prevent_overlap && overlap) {
            x0 = rnd.next() * 0.5;
            y0 = rnd.next() * 0.5;
            z0 = rnd.next() * 0.5;
            overlap = false;
            for (size_t c = 0; c < centres.size(); c += 3) {
                const double dx = centres[c] - x0, dy = centres[c + 1] - y0, dz = centres[c + 2] - z0;
                if (std::sqrt(dx * dx + dy * dy + dz * dz) < 2 * p->radius) {
                    overlap = true;
                    break;
                }
            }
        }
        centres.push_back(x0);
        centres.push_back(y0);
        centres.push_back(z0);
        auto range = [&](double c, int n, int half, int &lo, int &hi) {
            lo = (int)std::floor((c - p->radius) * n) - 2;
            hi = (int)std::ceil((c + p->radius) * n) + 2;
            if (lo < 0) lo = 0;
            if (hi > half) hi = half;
        };
        int i0, i1, j0, j1, k0, k1;
        range(x0, X, hx, i0, i1);
        range(y0, Y, hy, j0, j1);
        range(z0, Z, hz, k0, k1);
        for (int i = i0; i < i1; ++i)
            for (int j = j0; j < j1; ++j)
                for (int k = k0; k < k1; ++k) {
                    const double x = i / double(X) + vsx / 2.0;
                    const double y = j / double(Y) + vsy / 2.0;
                    const double z = k / double(Z) + vsz / 2.0;
                    const double dx = x - x0, dy = y - y0, dz = z - z0;
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    const uint64_t idx = ((uint64_t)i * Y + j) * Z + k;
                    if (d2 < r2 && vox[idx] != (uint8_t)inverted) {
                        if (vox[idx] == DSMC_VOX_EMPTY) --empty;
                        vox[idx] = (uint8_t)inverted;
                        if (vox[idx] == DSMC_VOX_EMPTY) ++empty;
                    }
                }
        bool done;
        if (p->spheres_type == 0) {
            done = centres.size() / 3 >= (size_t)p->spheres_num;
        } else {
            const double porosity = (double)empty / ((int64_t)hx * hy * hz);
            done = inverted ? (porosity < p->wanted_porosity) : (porosity > p->wanted_porosity);
        }
        if (done) break;
    }
    // Mirror the first octant into all eight (make_periodic, dsmc/complexgeometry.cpp:853-871).
    for (int i = 0; i < X; ++i)
        for (int j = 0; j < Y; ++j)
            for (int k = 0; k < Z; ++k) {
                const int gi = i < X / 2 ? i : X - i - 1;
                const int gj = j < Y / 2 ? j : Y - j - 1;
                const int gk = k < Z / 2 ? k : Z - k - 1;
                vox[((uint64_t)i * Y + j) * Z + k] = vox[((uint64_t)gi * Y + gj) * Z + gk];
            }
    int rc = dsmc_geometry_finish(X, Y, Z, p->number_of_neighbor_averages, vox, nrm, t1, t2);
    if (rc) return rc;
    if (porosity_out) {
        uint64_t e = 0;
        for (uint64_t i = 0; i < V; ++i) e += vox[i] == DSMC_VOX_EMPTY;
        *porosity_out = (float)((double)e / V);
    }
    return DSMC_OK;
}

// ---------------------------------------------------------------------------
// State files and continuation counters (dsmc/dsmc_io.cpp:82-159,
// dsmc/main.cpp:37-55 and 110-112).

int dsmc_state_file_read(const char *path, int64_t cap, double *r, double *v, int64_t *n) {
    if (!path || !n) return DSMC_ERR_ARG;
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        set_thread_error(std::string("Error, could not open file ") + path);
        return DSMC_ERR_IO;
    }
    int32_t N = 0;
    if (std::fread(&N, sizeof(N), 1, f) != 1 || N < 0) {
        std::fclose(f);
        set_thread_error(std::string("state file has no particle count: ") + path);
        return DSMC_ERR_IO;
    }
    *n = N;
    if (!r || !v) {
        std::fclose(f);
        return DSMC_OK;
    }
    if (cap < N) {
        std::fclose(f);
        set_thread_error("output buffers smaller than the state file's particle count");
        return DSMC_ERR_CAPACITY;
    }
    std::vector<double> buf(6 * (size_t)N);
    const bool ok = std::fread(buf.data(), sizeof(double), buf.size(), f) == buf.size();
    std::fclose(f);
    if (!ok) {
        set_thread_error(std::string("state file shorter than its particle count: ") + path);
        return DSMC_ERR_IO;
    }
    for (int64_t k = 0; k < N; ++k)
        for (int d = 0; d < 3; ++d) {
            r[3 * k + d] = buf[6 * k + d];
            v[3 * k + d] = buf[6 * k + 3 + d];
        }
    return DSMC_OK;
}

int dsmc_state_file_write(const char *path, int64_t n, const double *r, const double *v) {
    if (!path || n < 0 || n > 0x7fffffff || (n > 0 && (!r || !v))) return DSMC_ERR_ARG;
    std::vector<double> buf(6 * (size_t)n);
    for (int64_t k = 0; k < n; ++k)
        for (int d = 0; d < 3; ++d) {
            buf[6 * k + d] = r[3 * k + d];
            buf[6 * k + 3 + d] = v[3 * k + d];
        }
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        set_thread_error(std::string("Error, could not open file ") + path);
        return DSMC_ERR_IO;
    }
    const int32_t N = (int32_t)n;
    bool ok = std::fwrite(&N, sizeof(N), 1, f) == 1;
    ok = ok && std::fwrite(buf.data(), sizeof(double), buf.size(), f) == buf.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        set_thread_error(std::string("could not write ") + path);
        return DSMC_ERR_IO;
    }
    return DSMC_OK;
}

int dsmc_tocontinue_read(const char *path, double *t, uint64_t *steps, uint64_t *collisions,
                         uint64_t *wall_collisions) {
    if (!path || !t || !steps || !collisions || !wall_collisions) return DSMC_ERR_ARG;
    std::ifstream in(path);
    if (!in.is_open()) {
        set_thread_error(std::string("could not open ") + path);
        return DSMC_ERR_IO;
    }
    // the reference extracts t, then the three counters as unsigned long
    double tt = 0;
    unsigned long long a = 0, b = 0, c = 0;
    in >> tt >> a >> b >> c;
    if (in.fail()) {
        set_thread_error(std::string("Tocontinue needs 't steps collisions wall_collisions': ") + path);
        return DSMC_ERR_IO;
    }
    *t = tt;
    *steps = a;
    *collisions = b;
    *wall_collisions = c;
    return DSMC_OK;
}

int dsmc_tocontinue_write(const char *path, double t, uint64_t steps, uint64_t collisions, uint64_t wall_collisions) {
    if (!path) return DSMC_ERR_ARG;
    FILE *f = std::fopen(path, "w");
    if (!f) {
        set_thread_error(std::string("could not open ") + path);
        return DSMC_ERR_IO;
    }
    std::fprintf(f, "%.17g %llu %llu %llu", t, (unsigned long long)steps, (unsigned long long)collisions,
                 (unsigned long long)wall_collisions);
    return std::fclose(f) == 0 ? DSMC_OK : DSMC_ERR_IO;
}

}  // extern "C"

int dsmc_profiles_finish(const dsmc_settings *s, double volume_global, int bins, const double *sums, double *count,
                         double *velocity_z, double *temperature, double *pressure, double *vx_center,
                         double *vx_count) {
    if (!s || !sums || bins < 1 || !(s->mass > 0)) return DSMC_ERR_ARG;
    const dsmc::Units u;
    // The average of a bin divides by max(count, 1)
    // (MeasureVelocityDistributionPoiseuille / MeasureTemperatureDistribution
    // ::get_average, dsmc/statisticalproperty.cpp:280-301, 341-362).
    const double volume_per_bin = volume_global / bins;
    for (int b = 0; b < bins; ++b) {
        const double c = sums[3 * b], norm = c > 1 ? c : 1.0;
        const double t_red = sums[3 * b + 2] / norm * (2.0 / 3.0);
        if (count) count[b] = c;
        if (velocity_z) velocity_z[b] = u.velocity_to_SI(sums[3 * b + 1] / norm);
        if (temperature) temperature[b] = u.temperature_to_SI(t_red);
        // MeasurePressureDistribution::get_average (:393-417): the summed count
        // over the bin's volume times the bin temperature, as the reference has it
        if (pressure) pressure[b] = u.pressure_to_SI(c / volume_per_bin * t_red);
    }
    // MeasureVelocityDistribution::finalize (:462-478): bin centres and counts
    const double sd = std::sqrt(u.temperature_from_SI(s->temperature) / s->mass);
    const double v_min = -4 * sd, width = (4 * sd - v_min) / bins;
    for (int b = 0; b < bins; ++b) {
        if (vx_center) vx_center[b] = u.velocity_to_SI(v_min + (b + 0.5) * width);
        if (vx_count) vx_count[b] = sums[3 * bins + b];
    }
    return DSMC_OK;
}
