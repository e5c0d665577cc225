// Launchers of the DSMC kernels, one set per precision policy
// (namespaces dsmc::split32 and dsmc::fp64).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dsmc_layout.h"

namespace dsmc {

#define DSMC_DECLARE_LAUNCHERS(NS)                                                                              \
    namespace NS {                                                                                              \
    cudaError_t launch_pass(int mode, const PassParams &P, int grid, int block, cudaStream_t st);               \
    int pass_blocks_per_sm(int mode, int block, int smem_cap);                                                  \
    size_t record_bytes();                                                                                      \
    cudaError_t launch_from_fp64(const SysDev *sys, int s, const double *r, const double *v, uint32_t id_base, \
                                 long long n, void *A, void *B, int *key, unsigned *hist, unsigned *err,        \
                                 cudaStream_t st);                                                              \
    cudaError_t launch_init(const SysDev *sys, int s, double sqrt_t_over_m, long long n, void *A, void *B,     \
                            int *key, unsigned *hist, unsigned *err, cudaStream_t st);                          \
    cudaError_t launch_init_field(const SysDev *sys, int s, double sqrt_t_over_m, long long n, const double *cdf, \
                                  const float *drift, long long V, void *A, void *B, int *key, unsigned *hist,  \
                                  unsigned *err, cudaStream_t st);                                              \
    cudaError_t launch_field_accumulate(const SysDev *sys, int s, const CellArrays &cells,                      \
                                        const ParticleArrays &parts, int cur, int cin, float4 *field,           \
                                        cudaStream_t st);                                                       \
    cudaError_t launch_gather(const CellArrays &cells, const ParticleArrays &parts, int cur, int cin, int c0,   \
                              int c1,                                                                           \
                              unsigned nspill, void *A, void *B, int *key, unsigned *hist,                      \
                              unsigned long long *cursor, unsigned long long limit, unsigned *err,               \
                              cudaStream_t st);                                                                  \
    cudaError_t launch_insert(const CellArrays &cells, const ParticleArrays &parts, int cur, int cin, long long n, \
                              const void *A, const void *B, const int *key, unsigned *err, cudaStream_t st);    \
    cudaError_t launch_to_fp64(const SysDev *sys, int s, const CellArrays &cells, const ParticleArrays &parts, \
                               int cur, int cin, uint32_t id_base, long long cap, double *r, double *v, int *cell, \
                               unsigned *err, cudaStream_t st);                                                 \
    cudaError_t launch_cell_energy(const CellArrays &cells, const ParticleArrays &parts, int cur, int cin, int c0,  \
                                   int c1,                                                                      \
                                   double *out, cudaStream_t st);                                               \
    }

DSMC_DECLARE_LAUNCHERS(split32)
DSMC_DECLARE_LAUNCHERS(fp64)

namespace split32 {
// the production pass (split_pass.cuh)
int fused_capacity(int smem_cap);   // move_cells ring slots per warp; 0: the production pass cannot run
// The ring move_cells runs with: the smallest ring of at least max(ring,
// fused_capacity(smem_cap)) slots (0: none).
int ring_for(int smem_cap, int ring);
// The largest ring this build has.
int max_ring();
int fused_block();                  // threads per block of the production kernels
// Persistent grids of collide_cells, move_cells, place_movers, place_walls
// and sample_cells; 0 when one of them cannot be resident.
// ring: as ring_for.  max_bps (may be null): the most blocks per SM of each.
int fused_grids(int smem_cap, int num_sms, int grids[5], int ring = 0, int max_bps[5] = nullptr);
// ev: null, or five events recorded before each kernel and after the last
// (the sampler, on sampled steps, falls in the collide interval)
cudaError_t launch_fused(const PassParams &P, const int grids[5], cudaStream_t st, cudaEvent_t *ev = nullptr);
// collide_cells (and sample_cells when P.do_sample) alone, in place: the
// collide of a step whose move has not started
cudaError_t launch_collide(const PassParams &P, const int grids[5], cudaStream_t st);
// Records from another slab into system s's cells (occupancy set cin of buffer
// cur): top segments, or the overflow list when a cell is full.
cudaError_t launch_put(const SysDev *sys, int s, const CellArrays &cells, const ParticleArrays &parts, int cur, int cin,
                       long long n, const uint4 *rec, Status *status, cudaStream_t st);
}  // namespace split32

// Slot layout of the cells (cell_layout.cu): meta[a].y = capacity of cell a
// from its free voxels pix[a], its present occupancy and np[system] =
// {particles, free voxels of the system}; meta[a].x = its first slot (the
// capacities of the cells before it).  out = {total slots, largest capacity};
// bsum holds cell_layout_blocks(C) entries.
int cell_layout_blocks(int C);
cudaError_t launch_cell_layout(int4 *meta, const int *pix, const unsigned *present, const double2 *np, double factor,
                               double pad, int C, unsigned long long *bsum, unsigned long long *out, cudaStream_t st);

// Pass modes (engine.cuh PassMode).
enum { PASS_FUSED = 0, PASS_INPLACE = 1, PASS_SORT = 2 };

}  // namespace dsmc
