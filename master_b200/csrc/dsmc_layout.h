// Device-side data layout of the DSMC timestep, shared by host and device code.
//
// One "system" is one voxel geometry with its gas (the reference's System,
// dsmc/system.h:29-120).  Many systems advance together: their active cells
// are concatenated into one cell range, and every kernel walks that range.
//
// Particles live in per-cell slot regions (a bucketed counting sort):
//   active cell a owns slots [base, base + cap) of each particle array
//   (meta[a] = {base, cap, ...}); two segments of them are occupied:
//   the bottom [base, base + bot) and the top [base + cap - top, base + cap).
// Buffers b = 0/1 ping-pong: the fused pass reads buffer `cur` and places
// every moved particle into its new cell's region of buffer `cur ^ 1`.
// Particles that stay in their cell are written to the bottom by the warp
// that owns the cell, without atomics; every other placement takes a top slot
// with an atomic.  The occupancy counts rotate through three sets (in, out,
// and the set the pass clears for the pass after next), so no count a pass
// reads is written during it.
//
// Record formats (structure of arrays, 16-byte vectors):
//   split precision:  A = uint4 {voxel (i | j<<11 | k<<22), ox, oy, oz (fp32 bits)}
//                     B = float4 {vx, vy, vz, id (u32 bits)}
//                     ox,oy,oz in [0,1) voxel units; v in reduced units.
//   fp64 reference:   A = double4 {rx, ry, rz, id}   B = double4 {vx, vy, vz, 0}
//                     the reference's own representation (dsmc/system.h:74-75).
#pragma once
#include <stdint.h>
#include <vector_types.h>

#define DSMC_VOX_EMPTY 0
#define DSMC_VOX_WALL 1
#define DSMC_VOX_BOUNDARY 2

#define DSMC_TAG_MOVE 1u
#define DSMC_TAG_COLLIDE 2u
#define DSMC_TAG_INIT 3u

// error bits reported in Status::error: DSMC_EBIT_* of the public header
#include "dsmc_b200.h"

// cell_map values of cells that are not this system's active cells
#define DSMC_CELL_SOLID (-1)    // no free volume
#define DSMC_CELL_FOREIGN (-2)  // owned by another slab of the geometry

#define DSMC_VOX_PACK(i, j, k) ((uint32_t)(i) | ((uint32_t)(j) << 11) | ((uint32_t)(k) << 22))
#define DSMC_VOX_I(p) ((int)((p)&0x7FFu))
#define DSMC_VOX_J(p) ((int)(((p) >> 11) & 0x7FFu))
#define DSMC_VOX_K(p) ((int)((p) >> 22))

namespace dsmc {

// Slot address of the s-th occupied particle of a cell (bottom, then top).
#ifdef __CUDACC__
__host__ __device__
#endif
inline unsigned cell_slot(int base, int cap, unsigned bot, unsigned top, unsigned s) {
    return s < bot ? (unsigned)base + s : (unsigned)(base + cap) - top + (s - bot);
}

struct SysDev {
    // voxel grid (no halo; periodic index wrap replaces the reference's 27x copy)
    int n[3];                  // voxels per axis
    int cells[3];              // cells per axis
    int vpc[3];                // voxels per cell per axis
    float inv_vpc[3];
    const uint8_t *vox;        // voxel type, index (i*ny + j)*nz + k
    const float *nrm, *t1, *t2;  // 3 floats per voxel, same order
    const int *cell_map;       // global cell (i*cy + j)*cz + k -> active cell id, -1 if solid
    int active_begin, active_end;
    // geometry constants
    double L[3], invL[3];
    double vox_len[3];         // L/n (the reference's Grid::voxel_size, dsmc/grid.cpp:17-19)
    double ref_scale[3];       // (double)(float)(invL*n): Grid::one_over_length_*_times_global_n*
    double ref_shift[3];       // (double)(float)(n):      Grid::constant_* (one rank, origin 0)
    float inv_vox_f[3];        // n/L in fp32 (split-precision mover)
    float L_f[3];
    // physics
    double dt;
    float dt_f;
    double accel_dt;           // gravity*dt along flow_dir
    float accel_dt_f;
    int flow_dir;              // -1: no acceleration
    double wall_s;             // sqrt(T_wall/m) (dsmc/system.cpp:343)
    float wall_s_f;
    // wall model (dsmc/system.cpp:345-352): DSMC_WALL_* and the constants of
    // Random(seed, alpha_n, alpha_t) (dsmc/random.cpp:8-15)
    int wall_model;
    double alpha_t, sqrt_1m_an, sqrt_1m_an_over_an, sqrt_an_over_2, cl_vmax;
    float alpha_t_f, sqrt_1m_an_f, sqrt_1m_an_over_an_f, sqrt_an_over_2_f, cl_vmax_f;
    uint64_t seed;
    int sample_interval;       // sample when step % interval == 0 and step >= sample_begin
    int sample_begin;
    // y-binned profiles of the sampler (dsmc/statisticalproperty.cpp:229-362):
    // per bin {particle count, sum v_z, sum 1/2 m v_z^2} over the samples
    // and the v_x histogram of MeasureVelocityDistribution (bins of width
    // vx_bin from vx_min = -4 sqrt(T/m)), stored after the 3*bins sums;
    // prof_copies copies of these 4*bins sums, each warp adding to one of
    // them (every particle of a sample lands in one of a few bins: with one
    // copy the atomics queue on those few addresses); the host adds them up
    double *prof;
    int prof_bins, prof_copies;
    double mass, vx_min, vx_bin, vx_inv_bin;
};

#define DSMC_WALL_THERMAL 0    // diffuse reflection at the wall temperature
#define DSMC_WALL_SPECULAR 1
#define DSMC_WALL_CL 2         // Cercignani-Lampis

struct SysTally {
    unsigned long long collisions;
    unsigned long long wall_hits;
    unsigned long long reseeds;
    unsigned long long particle_steps;
    long long count_periodic[3];   // net boundary crossings (dsmc/moleculemover.h:29-38)
    unsigned long long samples;    // sampled steps folded into the cell moments
    unsigned long long candidates;
    unsigned long long stranded;   // moves that ended inside solid cells (see DSMC_EBIT_STRANDED)
};

struct Status {
    unsigned int error;        // DSMC_EBIT_* bits
    unsigned int spill;        // particles written to the overflow list this pass
    unsigned int step;         // current step number (the reference's System::steps)
    unsigned int blocks_done;  // end-of-pass counter used to advance `step`
    unsigned int halted;       // non-zero: a pass saw spill/error; later passes do nothing
    unsigned int walls;        // entries in the wall-flight list this pass (production pass)
    unsigned int nout;         // records in the outgoing list (particles that left a slab)
    unsigned int walls_taken;  // wall-flight entries claimed by place_walls' warps this pass
    unsigned int collide_taken;  // cell chunks claimed by collide_cells' warps this pass
};

struct SpillRec {
    uint4 a;
    uint4 b;        // raw bits of B
    double4 ra;     // fp64 records
    double4 rb;
    int cell;
    int pad[3];
};

struct CellArrays {
    int num_cells;             // total active cells over all systems
    const int4 *meta;          // {first slot, slots, the reference's cell index
                               //  (dsmc/system.h:130-132), system}, fixed between relayouts
    double4 *state;            // {vr_max, selection remainder, coefficient, 0} in fp64:
                               //  (sigma*c_r)_max bookkeeping and NTC remainder
                               //  (dsmc/cell.cpp:42-111), 0.5 F_N pi d^2 dt / V_cell
                               //  (dsmc/cell.cpp:27-40)
    unsigned *bot[3];          // bottom-segment occupancy, three rotating sets
    unsigned *top[3];          // top-segment occupancy
    double *mom;               // 8 fp64 per cell: n, sum v (3), sum v^2 (3), sum |v|^2
    unsigned *key;             // per slot: new active cell after a stand-alone move stage
    int2 *room;                // per cell, this pass: {first slot past the cell, top slots free}
};

struct ParticleArrays {
    void *A[2];
    void *B[2];
    SpillRec *spill;
    unsigned spill_cap;
    int2 *walls;               // production pass: {output slot, source cell} of flights that meet a wall
    unsigned walls_cap;
    uint4 *out;                // outgoing list: record k is {A, B} at out[2k], out[2k + 1]
    unsigned out_cap;
};

struct PassParams {
    const SysDev *sys;
    SysTally *tally;
    Status *status;
    CellArrays cells;
    ParticleArrays parts;
    int cur;                   // buffer read this pass
    int cin, cout, cclear;     // count sets: read, written, cleared this pass
    int top_only;              // every placement takes a top slot (generic passes)
    int sorted_in;             // every bottom segment of the input is sorted by id
    int do_collide;            // collide the cells of the pass's input (step - 1's sort)
    int do_move;               // accelerate + move + re-bin (step)
    int do_sample;             // sample after the collide, on the reference's cadence
    int smem_cap;              // staging capacity per warp (particles)
    int advance_step;          // increment Status::step at the end of the pass
    int ring;                  // production pass: move_cells ring slots per warp (0: the smallest that fits)
    int claim;                 // production pass: collide_cells chunk claims (0 auto, 1 stride, 2 counter)
};

}  // namespace dsmc
