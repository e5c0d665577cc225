// Kernels and launchers instantiated once per precision policy.  The including
// translation unit defines DSMC_PREC (the policy) and DSMC_PREC_NS (the
// namespace the launchers are placed in).
#pragma once
#include "engine.cuh"
#include "kernels.h"

namespace dsmc {
namespace DSMC_PREC_NS {

typedef DSMC_PREC Prec;
typedef Prec::RecA RecA;
typedef Prec::RecB RecB;
typedef Prec::Particle Particle;

// fp64 position -> record of this precision.  The voxel is the one the
// reference's Grid::get_index_of_voxel assigns (dsmc/grid.h:139-145).
template <class P> struct Maker;
template <> struct Maker<Split32> {
    static __device__ void make(const SysDev &g, const double r[3], const double v[3], uint32_t id,
                                Split32::Particle &p) {
        for (int d = 0; d < 3; ++d) {
            const double x = r[d] * g.ref_scale[d] + g.ref_shift[d];
            const int c = (int)x;
            float o = (float)(x - (double)c);
            if (!(o >= 0.0f)) o = 0.0f;
            if (o >= 1.0f) o = one_minus_ulp();
            p.c[d] = wrap_index(c - g.n[d], g.n[d]);
            p.o[d] = o;
            p.v[d] = (float)v[d];
        }
        p.id = id;
        p.flag = voxel_type(g, p.c[0], p.c[1], p.c[2]) != DSMC_VOX_EMPTY;
    }
    static __device__ void position(const SysDev &g, const Split32::Particle &p, double r[3]) {
        for (int d = 0; d < 3; ++d) r[d] = ((double)p.c[d] + (double)p.o[d]) * g.vox_len[d];
    }
};
template <> struct Maker<Fp64> {
    static __device__ void make(const SysDev &, const double r[3], const double v[3], uint32_t id,
                                Fp64::Particle &p) {
        for (int d = 0; d < 3; ++d) {
            p.r[d] = r[d];
            p.v[d] = v[d];
        }
        p.id = id;
    }
    static __device__ void position(const SysDev &, const Fp64::Particle &p, double r[3]) {
        for (int d = 0; d < 3; ++d) r[d] = p.r[d];
    }
};

__device__ __forceinline__ int particle_cell(const SysDev &g, const Particle &p, unsigned *err) {
    const int cg = Prec::cell_global(g, p);
    const int ac = __ldg(g.cell_map + cg);
    if (ac == DSMC_CELL_SOLID) atomicOr(err, DSMC_EBIT_CELL);
    return ac;  // DSMC_CELL_FOREIGN: another slab's cell, the particle is left out
}

// Flat fp64 state (the reference's state-file layout) -> flat records + cell keys.
__global__ void k_from_fp64(const SysDev *sys, int s, const double *r, const double *v, uint32_t id_base,
                            long long n, RecA *A, RecB *B, int *key, unsigned *hist, unsigned *err) {
    const SysDev &g = sys[s];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double rr[3] = {r[3 * i], r[3 * i + 1], r[3 * i + 2]};
        double vv[3] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        bool finite = true;
        for (int d = 0; d < 3; ++d) finite = finite && isfinite(rr[d]) && isfinite(vv[d]);
        if (!finite) {
            // refused by the caller (DSMC_ERR_STATE); the record is left out
            atomicOr(err, DSMC_EBIT_NAN);
            key[i] = DSMC_CELL_SOLID;
            continue;
        }
        Particle p;
        Maker<Prec>::make(g, rr, vv, id_base + (uint32_t)i, p);
        const int ac = particle_cell(g, p, err);
        Prec::pack(p, A[i], B[i]);
        key[i] = ac;
        if (ac >= 0) atomicAdd(&hist[ac], 1u);
    }
}

// System::setup_molecules (dsmc/system.cpp:398-430): three Box-Muller normals
// (dsmc/random.cpp:21-25) times sqrt(T/m), then find_position's rejection loop
// (dsmc/system.cpp:384-396); stream (id, 0, init) per particle.
__global__ void k_init(const SysDev *sys, int s, double sqrt_t_over_m, long long n, RecA *A, RecB *B, int *key,
                       unsigned *hist, unsigned *err) {
    const SysDev &g = sys[s];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        DrawStream rs;
        rs.init(g.seed, (uint32_t)i, 0u, DSMC_TAG_INIT);
        double v[3], r[3];
        for (int d = 0; d < 3; ++d) {
            const double u1 = rs.uniform64();
            const double u2 = rs.uniform64();
            v[d] = sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307 * u2) * sqrt_t_over_m;
        }
        bool ok = false;
        for (int tries = 0; tries < 100000 && !ok; ++tries) {
            int u[3];
            for (int d = 0; d < 3; ++d) r[d] = 0.0 + g.L[d] * rs.uniform64();
            for (int d = 0; d < 3; ++d)
                u[d] = (int)((r[d] - 0.0) * g.invL[d] * (double)g.n[d] + (double)g.n[d]) - g.n[d];
            ok = voxel_type(g, u[0], u[1], u[2]) < DSMC_VOX_WALL;
        }
        if (!ok) atomicOr(err, DSMC_EBIT_RESEED);
        Particle p;
        Maker<Prec>::make(g, r, v, (uint32_t)i, p);
        const int ac = particle_cell(g, p, err);
        Prec::pack(p, A[i], B[i]);
        key[i] = ac;
        if (ac >= 0) atomicAdd(&hist[ac], 1u);
    }
}

// Warm start from a field: particle i is placed in voxel w with probability
// weight[w] / sum(weight) (inverse of the cumulative weights `cdf`, V + 1
// entries with cdf[0] = 0), uniformly inside it, with velocity drift[w] plus
// a Maxwellian of sqrt(T/m) per component; stream (id, 0, init) per particle.
// The field-free counterpart is k_init (System::setup_molecules).
__global__ void k_init_field(const SysDev *sys, int s, double sqrt_t_over_m, long long n, const double *cdf,
                             const float *drift, long long V, RecA *A, RecB *B, int *key, unsigned *hist,
                             unsigned *err) {
    const SysDev &g = sys[s];
    const double total = cdf[V];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        DrawStream rs;
        rs.init(g.seed, (uint32_t)i, 0u, DSMC_TAG_INIT);
        double v[3], r[3];
        for (int d = 0; d < 3; ++d) {
            const double u1 = rs.uniform64();
            const double u2 = rs.uniform64();
            v[d] = sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307 * u2) * sqrt_t_over_m;
        }
        // the voxel w with cdf[w] <= u < cdf[w + 1]
        const double u = rs.uniform64() * total;
        long long lo = 0, hi = V;
        while (hi - lo > 1) {
            const long long mid = (lo + hi) >> 1;
            if (cdf[mid] <= u) lo = mid; else hi = mid;
        }
        const long long w = lo;
        const int k = (int)(w % g.n[2]), j = (int)((w / g.n[2]) % g.n[1]), ii = (int)(w / ((long long)g.n[1] * g.n[2]));
        const int c[3] = {ii, j, k};
        for (int d = 0; d < 3; ++d) {
            // inside the voxel, away from its faces by a margin of 1e-6 voxel
            const double f = 1e-6 + (1.0 - 2e-6) * rs.uniform64();
            r[d] = ((double)c[d] + f) * g.vox_len[d];
            v[d] += (double)drift[3 * w + d];
        }
        if (voxel_type(g, c[0], c[1], c[2]) != DSMC_VOX_EMPTY) atomicOr(err, DSMC_EBIT_RESEED);
        Particle p;
        Maker<Prec>::make(g, r, v, (uint32_t)i, p);
        const int ac = particle_cell(g, p, err);
        Prec::pack(p, A[i], B[i]);
        key[i] = ac;
        if (ac >= 0) atomicAdd(&hist[ac], 1u);
    }
}

// Per-voxel sums of one system's particles, added to field[voxel] =
// {count, sum vx, sum vy, sum vz} (fp32): the steady fields the warm-start
// surrogate learns, accumulated over many steps.
__global__ void k_field_accumulate(const SysDev *sys, int s, const CellArrays cells, const ParticleArrays parts, int cur,
                                   int cin, float4 *field) {
    const SysDev &g = sys[s];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const RecA *Ain = reinterpret_cast<const RecA *>(parts.A[cur]);
    const RecB *Bin = reinterpret_cast<const RecB *>(parts.B[cur]);
    for (int a = g.active_begin + warp; a < g.active_end; a += nwarps) {
        const int4 m = cells.meta[a];
        const unsigned nb = min(cells.bot[cin][a], (unsigned)m.y);
        const unsigned nt = min(cells.top[cin][a], (unsigned)m.y - nb);
        for (unsigned q = lane; q < nb + nt; q += 32) {
            Particle p;
            const unsigned addr = cell_slot(m.x, m.y, nb, nt, q);
            Prec::unpack(Ain[addr], Bin[addr], p);
            double rr[3];
            Maker<Prec>::position(g, p, rr);
            int c[3];
            for (int d = 0; d < 3; ++d) {
                c[d] = (int)(rr[d] / g.vox_len[d]);
                c[d] = c[d] < 0 ? 0 : (c[d] >= g.n[d] ? g.n[d] - 1 : c[d]);
            }
            float4 *f = field + ((long long)c[0] * g.n[1] + c[1]) * g.n[2] + c[2];
            atomicAdd(&f->x, 1.0f);
            atomicAdd(&f->y, (float)p.v[0]);
            atomicAdd(&f->z, (float)p.v[1]);
            atomicAdd(&f->w, (float)p.v[2]);
        }
    }
}

// Slots of buffer `cur` (cells [c0, c1)) and the overflow list -> flat records.
__global__ void k_gather(const CellArrays cells, const ParticleArrays parts, int cur, int cin, int c0, int c1,
                         unsigned nspill, RecA *A, RecB *B, int *key, unsigned *hist, unsigned long long *cursor,
                         unsigned long long limit, unsigned *err) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const RecA *Ain = reinterpret_cast<const RecA *>(parts.A[cur]);
    const RecB *Bin = reinterpret_cast<const RecB *>(parts.B[cur]);
    for (int a = c0 + warp; a < c1; a += nwarps) {
        const int4 m = cells.meta[a];
        const unsigned nb = min(cells.bot[cin][a], (unsigned)m.y);
        const unsigned nt = min(cells.top[cin][a], (unsigned)m.y - nb);
        const unsigned n = nb + nt;
        unsigned long long at = 0;
        if (lane == 0 && n) at = atomicAdd(cursor, (unsigned long long)n);
        at = __shfl_sync(0xffffffffu, at, 0);
        if (at + n > limit) {
            if (lane == 0) atomicOr(err, DSMC_EBIT_SPILL_FULL);
            continue;
        }
        for (unsigned s = lane; s < n; s += 32) {
            const unsigned addr = cell_slot(m.x, m.y, nb, nt, s);
            A[at + s] = Ain[addr];
            B[at + s] = Bin[addr];
            key[at + s] = a;
        }
        if (lane == 0 && n) atomicAdd(&hist[a], n);
    }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    for (unsigned i = t; i < nspill; i += gridDim.x * blockDim.x) {
        const SpillRec &sr = parts.spill[i];
        if (sr.cell < c0 || sr.cell >= c1) continue;
        const unsigned long long at = atomicAdd(cursor, 1ull);
        if (at >= limit) {
            atomicOr(err, DSMC_EBIT_SPILL_FULL);
            continue;
        }
        if (sizeof(typename Prec::real) == 8) {
            A[at] = *reinterpret_cast<const RecA *>(&sr.ra);
            B[at] = *reinterpret_cast<const RecB *>(&sr.rb);
        } else {
            A[at] = *reinterpret_cast<const RecA *>(&sr.a);
            B[at] = *reinterpret_cast<const RecB *>(&sr.b);
        }
        key[at] = sr.cell;
        atomicAdd(&hist[sr.cell], 1u);
    }
}

// Flat records -> slots of buffer `cur` (counts must start at zero).
__global__ void k_insert(const CellArrays cells, const ParticleArrays parts, int cur, int cin, long long n,
                         const RecA *A, const RecB *B, const int *key, unsigned *err) {
    RecA *Aout = reinterpret_cast<RecA *>(parts.A[cur]);
    RecB *Bout = reinterpret_cast<RecB *>(parts.B[cur]);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int a = key[i];
        if (a < 0) continue;
        const int4 m = cells.meta[a];
        const unsigned slot = atomicAdd(&cells.bot[cin][a], 1u);
        if (slot >= (unsigned)m.y) {
            atomicOr(err, DSMC_EBIT_SPILL_FULL);
            continue;
        }
        Aout[m.x + slot] = A[i];
        Bout[m.x + slot] = B[i];
    }
}

// Slots of one system -> fp64 state ordered by id (dsmc/dsmc_io.cpp:98-113
// layout); r, v and cell may each be null (not written).
__global__ void k_to_fp64(const SysDev *sys, int s, const CellArrays cells, const ParticleArrays parts, int cur,
                          int cin, uint32_t id_base, long long cap, double *r, double *v, int *cell, unsigned *err) {
    const SysDev &g = sys[s];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const RecA *Ain = reinterpret_cast<const RecA *>(parts.A[cur]);
    const RecB *Bin = reinterpret_cast<const RecB *>(parts.B[cur]);
    for (int a = g.active_begin + warp; a < g.active_end; a += nwarps) {
        const int4 m = cells.meta[a];
        const unsigned nb = min(cells.bot[cin][a], (unsigned)m.y);
        const unsigned nt = min(cells.top[cin][a], (unsigned)m.y - nb);
        for (unsigned q = lane; q < nb + nt; q += 32) {
            Particle p;
            const unsigned addr = cell_slot(m.x, m.y, nb, nt, q);
            Prec::unpack(Ain[addr], Bin[addr], p);
            const long long i = (long long)p.id - (long long)id_base;
            if (i < 0 || i >= cap) {
                atomicOr(err, DSMC_EBIT_CELL);
                continue;
            }
            if (r) {
                double rr[3];
                Maker<Prec>::position(g, p, rr);
                for (int d = 0; d < 3; ++d) r[3 * i + d] = rr[d];
            }
            if (v)
                for (int d = 0; d < 3; ++d) v[3 * i + d] = (double)p.v[d];
            if (cell) cell[i] = m.z;
        }
    }
}

// Sum of |v|^2 over each cell's particles (MeasureEnergy's sum,
// dsmc/statisticalproperty.cpp:21-41), one fp64 value per cell.
__global__ void k_cell_energy(const CellArrays cells, const ParticleArrays parts, int cur, int cin, int c0, int c1,
                              double *out) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const RecB *Bin = reinterpret_cast<const RecB *>(parts.B[cur]);
    for (int a = c0 + warp; a < c1; a += nwarps) {
        const int4 m = cells.meta[a];
        const unsigned nb = min(cells.bot[cin][a], (unsigned)m.y);
        const unsigned nt = min(cells.top[cin][a], (unsigned)m.y - nb);
        double e = 0;
        for (unsigned q = lane; q < nb + nt; q += 32) {
            const RecB b = Bin[cell_slot(m.x, m.y, nb, nt, q)];
            const double x = (double)b.x, y = (double)b.y, z = (double)b.z;
            e += x * x + y * y + z * z;
        }
        e = warp_sum_f64(e);
        if (lane == 0) out[a - c0] = e;
    }
}

// ---- launchers --------------------------------------------------------------
static size_t stage_bytes(int cap) { return WarpStage<Prec>::bytes(cap); }

cudaError_t launch_pass(int mode, const PassParams &P, int grid, int block, cudaStream_t st) {
    const size_t smem = stage_bytes(P.smem_cap) * (block / 32);
    switch (mode) {
        case MODE_FUSED:
            pass_kernel<Prec, MODE_FUSED><<<grid, block, smem, st>>>(P);
            break;
        case MODE_INPLACE:
            pass_kernel<Prec, MODE_INPLACE><<<grid, block, smem, st>>>(P);
            break;
        default:
            pass_kernel<Prec, MODE_SORT><<<grid, block, smem, st>>>(P);
            break;
    }
    return cudaGetLastError();
}

template <class K> static int blocks_per_sm(K kernel, int block, size_t smem) {
    // the opt-in limit is a property of the function, shared by every
    // context: raise it to the device maximum, never lower it
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return 0;
    if (smem + fa.sharedSizeBytes > (size_t)optin) return 0;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes) !=
        cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, smem) != cudaSuccess) return 0;
    return nb;
}

int pass_blocks_per_sm(int mode, int block, int smem_cap) {
    const size_t smem = stage_bytes(smem_cap) * (block / 32);
    if (mode == MODE_FUSED) return blocks_per_sm(pass_kernel<Prec, MODE_FUSED>, block, smem);
    if (mode == MODE_INPLACE) return blocks_per_sm(pass_kernel<Prec, MODE_INPLACE>, block, smem);
    return blocks_per_sm(pass_kernel<Prec, MODE_SORT>, block, smem);
}

size_t record_bytes() { return sizeof(RecA) + sizeof(RecB); }

static int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

cudaError_t launch_from_fp64(const SysDev *sys, int s, const double *r, const double *v, uint32_t id_base,
                             long long n, void *A, void *B, int *key, unsigned *hist, unsigned *err,
                             cudaStream_t st) {
    k_from_fp64<<<grid_for(n, 256), 256, 0, st>>>(sys, s, r, v, id_base, n, (RecA *)A, (RecB *)B, key, hist, err);
    return cudaGetLastError();
}

cudaError_t launch_init(const SysDev *sys, int s, double sqrt_t_over_m, long long n, void *A, void *B, int *key,
                        unsigned *hist, unsigned *err, cudaStream_t st) {
    k_init<<<grid_for(n, 128), 128, 0, st>>>(sys, s, sqrt_t_over_m, n, (RecA *)A, (RecB *)B, key, hist, err);
    return cudaGetLastError();
}

cudaError_t launch_init_field(const SysDev *sys, int s, double sqrt_t_over_m, long long n, const double *cdf,
                              const float *drift, long long V, void *A, void *B, int *key, unsigned *hist,
                              unsigned *err, cudaStream_t st) {
    k_init_field<<<grid_for(n, 128), 128, 0, st>>>(sys, s, sqrt_t_over_m, n, cdf, drift, V, (RecA *)A, (RecB *)B, key,
                                                    hist, err);
    return cudaGetLastError();
}

cudaError_t launch_field_accumulate(const SysDev *sys, int s, const CellArrays &cells, const ParticleArrays &parts,
                                    int cur, int cin, float4 *field, cudaStream_t st) {
    k_field_accumulate<<<148 * 8, 256, 0, st>>>(sys, s, cells, parts, cur, cin, field);
    return cudaGetLastError();
}

cudaError_t launch_gather(const CellArrays &cells, const ParticleArrays &parts, int cur, int cin, int c0, int c1,
                          unsigned nspill, void *A, void *B, int *key, unsigned *hist, unsigned long long *cursor,
                          unsigned long long limit, unsigned *err, cudaStream_t st) {
    k_gather<<<148 * 8, 256, 0, st>>>(cells, parts, cur, cin, c0, c1, nspill, (RecA *)A, (RecB *)B, key, hist, cursor,
                                      limit, err);
    return cudaGetLastError();
}

cudaError_t launch_insert(const CellArrays &cells, const ParticleArrays &parts, int cur, int cin, long long n,
                          const void *A, const void *B, const int *key, unsigned *err, cudaStream_t st) {
    k_insert<<<grid_for(n, 256), 256, 0, st>>>(cells, parts, cur, cin, n, (const RecA *)A, (const RecB *)B, key, err);
    return cudaGetLastError();
}

cudaError_t launch_to_fp64(const SysDev *sys, int s, const CellArrays &cells, const ParticleArrays &parts, int cur,
                           int cin, uint32_t id_base, long long cap, double *r, double *v, int *cell, unsigned *err,
                           cudaStream_t st) {
    k_to_fp64<<<148 * 8, 256, 0, st>>>(sys, s, cells, parts, cur, cin, id_base, cap, r, v, cell, err);
    return cudaGetLastError();
}

cudaError_t launch_cell_energy(const CellArrays &cells, const ParticleArrays &parts, int cur, int cin, int c0, int c1,
                               double *out, cudaStream_t st) {
    k_cell_energy<<<148 * 8, 256, 0, st>>>(cells, parts, cur, cin, c0, c1, out);
    return cudaGetLastError();
}

}  // namespace DSMC_PREC_NS
}  // namespace dsmc
