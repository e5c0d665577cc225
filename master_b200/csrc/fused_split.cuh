// The production timestep pass for split-precision state: one kernel per
// step that, for every active cell, collides (NTC) and samples the particles
// the previous step sorted into it, then accelerates, moves and re-bins them
// into the next buffer.  One warp per cell at a time, persistent grid.
//
// Work layout: each warp owns chunks of 32 consecutive active cells (chunk c
// goes to warp c mod total warps).  The per-cell bookkeeping of a chunk --
// metadata, occupancy, the NTC selection count, the (sigma c_r)_max state and
// the occupancy written for the next pass -- is done by lane i for cell i,
// with coalesced loads and stores, two chunks ahead of the particle work.
//
// Memory pipeline: the particle records of the warp's next cells stream into
// a per-warp shared-memory ring of R slots with per-lane 16-byte cp.async
// copies, one commit group per cell, up to DEPTH cells ahead of the cell in
// work.  Waits are cp.async.wait_group on the warp's own copies (no spin).
#pragma once
#include "engine.cuh"

namespace dsmc {
namespace fused {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 16-byte global -> shared copy, cached in L2 only (both addresses 16-byte
// aligned: slots are uint4/float4 records).
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most `pending` of this thread's newest commit groups are
// still in flight (0 <= pending <= 4).
__device__ __forceinline__ void cp_async_wait(int pending) {
    switch (pending) {
        case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
        case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
        case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
        case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
        default: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
    }
}
constexpr int DEPTH = 4;  // cells staged ahead of the one in work

struct SmemVel {
    float4 *b;
    __device__ void get(int s, float &x, float &y, float &z) const {
        x = b[s].x;
        y = b[s].y;
        z = b[s].z;
    }
    __device__ void set(int s, float x, float y, float z) const {
        b[s].x = x;
        b[s].y = y;
        b[s].z = z;
    }
};

// A particle that left its voxel, waiting for the general mover with the
// cell it came from.
struct SlowRec {
    uint4 a;
    float4 b;
    int cell;       // active cell it was in
    int global;     // that cell's reference index
    int pad[2];
};

constexpr int QCAP = 32;   // mover queue
constexpr int WCAP = 16;   // wall queue
enum { T_WALL, T_RESEED, T_CROSS0, T_CROSS1, T_CROSS2, T_STRANDED, T_ERR, T_COLL, T_CAND, T_MOVED, TALLY_N };

// Per-chunk cell table: entry i describes cell first + i of the chunk.
struct CellTab {
    int base[32];        // first slot
    int cap[32];         // slots
    unsigned nb[32];     // bottom-segment occupancy (input)
    unsigned nt[32];     // top-segment occupancy (input)
    int glob[32];        // the reference's cell index
    int sys[32];
    int pairs[32];       // NTC candidate pairs this step
    double vr[32];       // (sigma c_r)_max
    double rest[32];     // selection remainder after this step's selection
    int first;           // first active cell of the chunk
    int ncell;           // cells in the chunk; 0: no chunk
};

// Per-warp shared memory: particle ring, two chunk tables, the general-mover
// queue and the collide permutation.
template <int R> struct WarpSmem {
    uint4 A[R];
    float4 B[R];
    CellTab tab[2];
    SlowRec q[QCAP];     // left their voxel: the open-flight mover first
    SlowRec wq[WCAP];    // flight meets a wall: the general mover
    uint4 blk[32];       // Philox blocks 0..31 of the collide stream of the cell in work
    uint16_t perm[R];
    int qn, wqn;
    // the warp's counts since its last flush: wall hits, reseeds, crossings
    // x3, stranded, error bits, collisions, candidates, particles moved
    unsigned wtally[TALLY_N];
};

// Publishes the warp's counts for system `sys` and clears them (lane 0).
template <int R> __device__ void flush_warp(const PassParams &P, WarpSmem<R> &W, int sys, int lane) {
    __syncwarp();
    if (lane == 0 && sys >= 0) {
        SysTally &T = P.tally[sys];
        const unsigned *w = W.wtally;
        if (w[T_COLL]) atomicAdd(&T.collisions, (unsigned long long)w[T_COLL]);
        if (w[T_CAND]) atomicAdd(&T.candidates, (unsigned long long)w[T_CAND]);
        if (w[T_WALL]) atomicAdd(&T.wall_hits, (unsigned long long)w[T_WALL]);
        if (w[T_RESEED]) atomicAdd(&T.reseeds, (unsigned long long)w[T_RESEED]);
        if (w[T_MOVED]) atomicAdd(&T.particle_steps, (unsigned long long)w[T_MOVED]);
        if (w[T_STRANDED]) atomicAdd(&T.stranded, (unsigned long long)w[T_STRANDED]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int c = (int)w[T_CROSS0 + d];
            if (c) atomicAdd((unsigned long long *)&T.count_periodic[d], (unsigned long long)(long long)c);
        }
        if (w[T_ERR]) atomicOr(&P.status->error, w[T_ERR]);
    }
    __syncwarp();
    if (lane < TALLY_N) W.wtally[lane] = 0;
    __syncwarp();
}

// Places one particle per valid lane into a top slot of its new cell
// (warp-aggregated atomics; a slot that could meet the owner's bottom
// segment, i.e. within the cell's input occupancy, spills instead).
__device__ __forceinline__ void insert_top(const PassParams &P, const Split32::Particle &p, bool valid,
                                           unsigned key, int lane, unsigned &err) {
    unsigned *top_out = P.cells.top[P.cout];
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    unsigned slot0 = 0;
    if (valid && lane == leader) slot0 = atomicAdd(&top_out[key], (unsigned)__popc(peers));
    slot0 = __shfl_sync(0xffffffffu, slot0, leader);
    bool spilled = false;
    if (valid) {
        const unsigned j = slot0 + (unsigned)__popc(peers & ((1u << lane) - 1u));
        uint4 ra;
        float4 rb;
        Split32::pack(p, ra, rb);
        const int4 km = P.cells.meta[key];
        const unsigned room = (unsigned)km.y - min((unsigned)km.y, P.cells.bot[P.cin][key] + P.cells.top[P.cin][key]);
        if (j < room) {
            const unsigned dst = (unsigned)(km.x + km.y) - 1u - j;
            reinterpret_cast<uint4 *>(P.parts.A[P.cur ^ 1])[dst] = ra;
            reinterpret_cast<float4 *>(P.parts.B[P.cur ^ 1])[dst] = rb;
        } else {
            spilled = true;
            const unsigned si = atomicAdd(&P.status->spill, 1u);
            if (si < P.parts.spill_cap) {
                SpillRec &sr = P.parts.spill[si];
                sr.a = ra;
                sr.b = *reinterpret_cast<const uint4 *>(&rb);
                sr.cell = (int)key;
            } else {
                err |= DSMC_EBIT_SPILL_FULL;
            }
        }
    }
    // spilled slots are given back: the counter ends at the placed count
    const unsigned over = __ballot_sync(0xffffffffu, spilled) & peers;
    if (valid && lane == leader && over) atomicSub(&top_out[key], (unsigned)__popc(over));
}

__device__ __forceinline__ void tally_moves(unsigned *wtally, const MoveTally &mt, unsigned stranded) {
    const unsigned wh = __reduce_add_sync(0xffffffffu, (unsigned)mt.wall_hits);
    const unsigned rs = __reduce_add_sync(0xffffffffu, (unsigned)mt.reseeds);
    const int c0 = __reduce_add_sync(0xffffffffu, mt.cross[0]);
    const int c1 = __reduce_add_sync(0xffffffffu, mt.cross[1]);
    const int c2 = __reduce_add_sync(0xffffffffu, mt.cross[2]);
    const unsigned sd = __reduce_add_sync(0xffffffffu, stranded);
    const unsigned er = __reduce_or_sync(0xffffffffu, mt.err);
    if ((threadIdx.x & 31) == 0) {
        wtally[T_WALL] += wh;
        wtally[T_RESEED] += rs;
        wtally[T_CROSS0] += (unsigned)c0;
        wtally[T_CROSS1] += (unsigned)c1;
        wtally[T_CROSS2] += (unsigned)c2;
        wtally[T_STRANDED] += sd;
        wtally[T_ERR] |= er;
    }
}

// Runs the general mover on the queued particles, one per lane, and places
// them; its counts go to the warp's shared tally.  All lanes call.
__device__ __noinline__ void drain_wall(const PassParams &P, int sys, SlowRec *q, int *qn_p, unsigned *wtally,
                                         int lane, uint32_t move_step) {
    const SysDev &g = P.sys[sys];
    const int qn = *qn_p;
    const bool valid = lane < qn;
    Split32::Particle p;
    unsigned key = 0xffffffffu;
    MoveTally mt;
    mt.wall_hits = mt.reseeds = 0;
    mt.cross[0] = mt.cross[1] = mt.cross[2] = 0;
    mt.err = 0;
    unsigned stranded = 0;
    if (valid) {
        const SlowRec &r = q[lane];
        Split32::unpack(r.a, r.b, p);
        Split32::move_general(g, p, move_step, mt);
        key = (unsigned)r.cell;
        const int cg = Split32::cell_global(g, p);
        if (cg != r.global) {
            const int ac = __ldg(g.cell_map + cg);
            if (ac < 0) {
                mt.err |= DSMC_EBIT_STRANDED;
                stranded = 1;
            } else {
                key = (unsigned)ac;
            }
        }
    }
    __syncwarp();
    insert_top(P, p, valid, key, lane, mt.err);
    tally_moves(wtally, mt, stranded);
    if (lane == 0) *qn_p = 0;
    __syncwarp();
}

// Particles that left their voxel, one per lane: a flight that ends in an
// empty voxel completes here (Split32::move_open) and the particle takes a
// top slot of its cell; the rest go to the wall queue unchanged, or, when
// more of them than the wall queue holds arrive at once, take the general
// mover right here.  All lanes call.
__device__ __noinline__ void drain_movers(const PassParams &P, int sys, SlowRec *q, int *qn_p, SlowRec *wq,
                                          int *wqn_p, unsigned *wtally, int lane, uint32_t move_step) {
    const SysDev &g = P.sys[sys];
    const int qn = *qn_p;
    const bool valid = lane < qn;
    Split32::Particle p;
    MoveTally mt;
    mt.wall_hits = mt.reseeds = 0;
    mt.cross[0] = mt.cross[1] = mt.cross[2] = 0;
    mt.err = 0;
    unsigned stranded = 0, key = 0xffffffffu;
    int from_cell = 0, from_global = 0;
    bool done = false;
    if (valid) {
        const SlowRec &r = q[lane];
        Split32::unpack(r.a, r.b, p);
        from_cell = r.cell;
        from_global = r.global;
        done = Split32::move_open(g, p, mt);
    }
    const unsigned wall = __ballot_sync(0xffffffffu, valid && !done);
    const int nwall = __popc(wall);
    if (nwall) {
        if (*wqn_p + nwall > WCAP && nwall <= WCAP) drain_wall(P, sys, wq, wqn_p, wtally, lane, move_step);
        if (*wqn_p + nwall <= WCAP) {
            if (valid && !done) wq[*wqn_p + __popc(wall & ((1u << lane) - 1u))] = q[lane];
            __syncwarp();
            if (lane == 0) *wqn_p += nwall;
            __syncwarp();
        } else if (valid && !done) {
            Split32::move_general(g, p, move_step, mt);
            done = true;
        }
    }
    if (done) {
        key = (unsigned)from_cell;
        const int cg = Split32::cell_global(g, p);
        if (cg != from_global) {
            const int ac = __ldg(g.cell_map + cg);
            if (ac < 0) {
                mt.err |= DSMC_EBIT_STRANDED;
                stranded = 1;
            } else {
                key = (unsigned)ac;
            }
        }
    }
    insert_top(P, p, done, key, lane, mt.err);
    tally_moves(wtally, mt, stranded);
    if (lane == 0) *qn_p = 0;
    __syncwarp();
}

// Draws of one collide stream: blocks 0..nblk-1 come from shared memory
// (computed by the warp in parallel), later ones are computed here.  Same
// layout as DrawStream.
struct CachedDraws {
    const uint4 *blk;
    uint32_t nblk, key0, key1, id, step, k;
    uint32_t w2, w3;
    __device__ __forceinline__ void words(uint32_t &a, uint32_t &b) {
        const uint32_t j = k >> 1;
        if ((k & 1u) == 0) {
            uint32_t w[4];
            if (j < nblk) {
                const uint4 c = blk[j];
                w[0] = c.x;
                w[1] = c.y;
                w[2] = c.z;
                w[3] = c.w;
            } else {
                philox4x32_10(id, step, DSMC_TAG_COLLIDE, j, key0, key1, w);
            }
            a = w[0];
            b = w[1];
            w2 = w[2];
            w3 = w[3];
        } else {
            a = w2;
            b = w3;
        }
        ++k;
    }
    template <class T> __device__ __forceinline__ T uniform() {
        uint32_t a, b;
        words(a, b);
        return ((float)(a >> 9) + 0.5f) * (1.0f / 8388608.0f);
    }
};

// The NTC collide of one staged cell.  The warp computes the cell's first
// Philox blocks in parallel and ranks the cell's particles by id (the
// reference's canonical member order); perm[rank] is the ring slot of that
// particle.  Lane 0 then runs the candidate loop.
template <int R>
__device__ __forceinline__ unsigned collide_cell(uint64_t seed, int cell_global, uint32_t step, int n, int pairs,
                                              double *vr_max, float4 *ring_b, int start, uint16_t *perm, uint4 *blk,
                                              int lane) {
    // three draws per candidate and two per collision: at most 5 * pairs
    const uint32_t nblk = (uint32_t)min(32, (5 * pairs + 1) >> 1);
    const uint32_t key0 = (uint32_t)seed, key1 = (uint32_t)(seed >> 32);
    if ((uint32_t)lane < nblk) {
        uint32_t w[4];
        philox4x32_10((uint32_t)cell_global, step, DSMC_TAG_COLLIDE, (uint32_t)lane, key0, key1, w);
        blk[lane] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    if (n <= 32) {
        int sq = start + lane;
        if (sq >= R) sq -= R;
        const uint32_t mine = lane < n ? __float_as_uint(ring_b[sq].w) : 0xffffffffu;
        int rank = 0;
#pragma unroll
        for (int r = 0; r < 32; ++r) rank += __shfl_sync(0xffffffffu, mine, r) < mine;
        if (lane < n) perm[rank] = (uint16_t)sq;
    } else {
        for (int q = lane; q < n; q += 32) {
            int sq = start + q;
            if (sq >= R) sq -= R;
            const uint32_t mine = __float_as_uint(ring_b[sq].w);
            int rank = 0;
            int sr = start;
            for (int r = 0; r < n; ++r) {
                rank += __float_as_uint(ring_b[sr].w) < mine;
                if (++sr == R) sr = 0;
            }
            perm[rank] = (uint16_t)sq;
        }
    }
    __syncwarp();
    unsigned long long col = 0;
    if (lane == 0) {
        CachedDraws rs;
        rs.blk = blk;
        rs.nblk = nblk;
        rs.key0 = key0;
        rs.key1 = key1;
        rs.id = (uint32_t)cell_global;
        rs.step = step;
        rs.k = 0;
        SmemVel vel;
        vel.b = ring_b;
        ntc_loop<float>(rs, n, pairs, *vr_max, vel, perm, col);
    }
    __syncwarp();
    return (unsigned)col;
}

constexpr int FUSED_WARPS = 4;  // warps per block of the pipelined pass

template <int R>
__global__ void __launch_bounds__(32 * FUSED_WARPS, 4) fused_split_kernel(const __grid_constant__ PassParams P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    typedef Split32::Particle Particle;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const volatile Status *vs = P.status;
    if (vs->halted) return;
    const uint32_t step = vs->step;
    const uint32_t move_step = step + 1;

    WarpSmem<R> &W = reinterpret_cast<WarpSmem<R> *>(smem_raw)[wib];
    if (lane == 0) W.qn = W.wqn = 0;
    if (lane < TALLY_N) W.wtally[lane] = 0;

    const uint4 *Ain = reinterpret_cast<const uint4 *>(P.parts.A[P.cur]);
    const float4 *Bin = reinterpret_cast<const float4 *>(P.parts.B[P.cur]);
    uint4 *Aout = reinterpret_cast<uint4 *>(P.parts.A[P.cur ^ 1]);
    float4 *Bout = reinterpret_cast<float4 *>(P.parts.B[P.cur ^ 1]);

    int tsys = -1;  // system of the counts in W.wtally

    const int C = P.cells.num_cells;
    const int nchunks = (C + 31) >> 5;
    const int wstride = gridDim.x * FUSED_WARPS;
    const int chunk0 = blockIdx.x * FUSED_WARPS + wib;

    // Lane i: cell i of chunk `ch` into table b, with this step's NTC
    // selection (Cell::prepare, dsmc/cell.cpp:42-50).
    auto load_tab = [&](int b, int ch) {
        CellTab &T = W.tab[b];
        const int first = ch * 32;
        const int ncell = ch < nchunks ? min(32, C - first) : 0;
        if (lane == 0) {
            T.first = first;
            T.ncell = ncell;
        }
        if (lane < ncell) {
            const int a = first + lane;
            const int4 m = P.cells.meta[a];
            const unsigned nb = min(P.cells.bot[P.cin][a], (unsigned)m.y);
            const unsigned nt = min(P.cells.top[P.cin][a], (unsigned)m.y - nb);
            const double4 st = P.cells.state[a];
            double rest = st.y;
            int pairs = 0;
            if (P.do_collide) {
                pairs = ntc_select(st.z, (int)(nb + nt), st.x, rest);
                if (nb + nt < 2) pairs = 0;
            }
            if (nb + nt > (unsigned)R) atomicOr(&P.status->error, DSMC_EBIT_SMEM);  // the host sizes R above every cap
            T.base[lane] = m.x;
            T.cap[lane] = m.y;
            T.nb[lane] = nb;
            T.nt[lane] = nt;
            T.glob[lane] = m.z;
            T.sys[lane] = m.w;
            T.pairs[lane] = pairs;
            T.vr[lane] = st.x;
            T.rest[lane] = rest;
        }
    };
    // Lane i: occupancy and cell state of cell i of table b for the next pass.
    auto write_tab = [&](int b, unsigned nfs) {
        const CellTab &T = W.tab[b];
        if (lane < T.ncell) {
            const int a = T.first + lane;
            P.cells.bot[P.cout][a] = nfs;
            P.cells.bot[P.cclear][a] = 0;
            P.cells.top[P.cclear][a] = 0;
            if (P.do_collide) *reinterpret_cast<double2 *>(&P.cells.state[a]) = make_double2(T.vr[lane], T.rest[lane]);
        }
    };

    load_tab(0, chunk0);
    load_tab(1, chunk0 + wstride);
    __syncwarp();

    // ring (warp-uniform): slots [tail, tail + used) hold the staged cells,
    // the cell in work first
    int head = 0, tail = 0, used = 0;
    int it = 0, ii = 0;     // next cell to stage: chunk ordinal, cell in chunk
    int ct = 0, ci = 0;     // cell in work
    int ahead = 0;          // cells staged, the one in work included
    unsigned nfs_mine = 0;  // lane i: bottom occupancy written for cell i of the chunk in work

    // Stage cells ahead while the ring has room (warp-uniform control flow:
    // every lane commits one group per staged cell).
    auto stage_ahead = [&]() {
        // (it, ii) moves past a full chunk as soon as its last cell is
        // staged, so ii >= ncell only past the warp's last cell
        while (ahead <= DEPTH && it <= ct + 1) {
            const CellTab &T = W.tab[it & 1];
            if (ii >= T.ncell) return;
            const unsigned nb = T.nb[ii], nt = T.nt[ii];
            const int n = (int)min(nb + nt, (unsigned)R);
            if (used + n > R) return;
            const int base = T.base[ii];
            const int top0 = base + T.cap[ii] - (int)nt;
            for (int q = lane; q < n; q += 32) {
                const int slot = q < (int)nb ? base + q : top0 + (q - (int)nb);
                int r = head + q;
                if (r >= R) r -= R;
                cp_async16(&W.A[r], Ain + slot);
                cp_async16(&W.B[r], Bin + slot);
            }
            cp_async_commit();
            head += n;
            if (head >= R) head -= R;
            used += n;
            ++ahead;
            if (++ii == 32) {
                ++it;
                ii = 0;
            }
        }
    };

    while (true) {
        const CellTab &T = W.tab[ct & 1];
        if (ci >= T.ncell) {
            // chunk finished: publish its cells, load the chunk two ahead
            if (T.ncell > 0) write_tab(ct & 1, nfs_mine);
            if (T.ncell < 32) break;  // that was the warp's last chunk
            __syncwarp();
            load_tab(ct & 1, chunk0 + (ct + 2) * wstride);
            __syncwarp();
            ++ct;
            ci = 0;
            continue;
        }
        stage_ahead();  // the cell in work is staged once this returns
        cp_async_wait(ahead - 1);
        __syncwarp();

        const int a = T.first + ci;
        const int n = (int)min(T.nb[ci] + T.nt[ci], (unsigned)R);
        const int base = T.base[ci];
        const int sys = T.sys[ci];
        const int pairs = T.pairs[ci];
        if (sys != tsys) {
            if (W.qn) drain_movers(P, tsys, W.q, &W.qn, W.wq, &W.wqn, W.wtally, lane, move_step);
            if (W.wqn) drain_wall(P, tsys, W.wq, &W.wqn, W.wtally, lane, move_step);
            if (tsys >= 0) flush_warp(P, W, tsys, lane);
            tsys = sys;
        }
        const SysDev &g = P.sys[sys];

        // ---- collide: Cell::collide (dsmc/cell.cpp:52-111)
        if (pairs > 0) {
            const unsigned col = collide_cell<R>(g.seed, T.glob[ci], step, n, pairs, &W.tab[ct & 1].vr[ci], W.B,
                                                 tail, W.perm, W.blk, lane);
            if (lane == 0) {
                W.wtally[T_COLL] += col;
                W.wtally[T_CAND] += (unsigned)pairs;
            }
        }

        // ---- sample: cell moments in fp64 on the reference's cadence
        if (P.do_sample && g.sample_interval > 0 && step > 0 && (step % (uint32_t)g.sample_interval) == 0 &&
            step >= (uint32_t)g.sample_begin) {
            double m1[3] = {0, 0, 0}, m2[3] = {0, 0, 0};
            for (int q = lane; q < n; q += 32) {
                int r = tail + q;
                if (r >= R) r -= R;
                const float4 b = W.B[r];
                const double x = b.x, y = b.y, z = b.z;
                m1[0] += x;
                m1[1] += y;
                m1[2] += z;
                m2[0] += x * x;
                m2[1] += y * y;
                m2[2] += z * z;
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                m1[q] = warp_sum_f64(m1[q]);
                m2[q] = warp_sum_f64(m2[q]);
            }
            if (lane == 0) {
                double *M = P.cells.mom + 8 * (size_t)a;
                M[0] += (double)n;
                M[1] += m1[0];
                M[2] += m1[1];
                M[3] += m1[2];
                M[4] += m2[0];
                M[5] += m2[1];
                M[6] += m2[2];
                M[7] += m2[0] + m2[1] + m2[2];
                if (a == g.active_begin) atomicAdd(&P.tally[sys].samples, 1ull);
            }
        }

        // ---- accelerate + move.  Particles that stay in their voxel keep
        // their cell and go to its bottom segment, in order, without atomics;
        // the rest queue for the general mover and a top slot.
        unsigned n_fs = 0;
        for (int c0 = 0; c0 < n; c0 += 32) {
            const int q = c0 + lane;
            const bool valid = q < n;
            Particle p;
            bool stay = false;
            if (valid) {
                int r = tail + q;
                if (r >= R) r -= R;
                Split32::unpack(W.A[r], W.B[r], p);
                Split32::accelerate(g, p);
                if (!p.flag) {
                    float x[3];
                    stay = true;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        x[d] = fmaf(p.v[d] * g.inv_vox_f[d], g.dt_f, p.o[d]);
                        stay &= (x[d] >= 0.0f) & (x[d] < 1.0f);
                    }
                    if (stay) {
                        p.o[0] = x[0];
                        p.o[1] = x[1];
                        p.o[2] = x[2];
                    }
                }
            }
            const unsigned fast = __ballot_sync(0xffffffffu, valid && stay);
            const unsigned slow = __ballot_sync(0xffffffffu, valid && !stay);
            if (valid && stay) {
                const unsigned dst = (unsigned)base + n_fs + (unsigned)__popc(fast & ((1u << lane) - 1u));
                uint4 ra;
                float4 rb;
                Split32::pack(p, ra, rb);
                Aout[dst] = ra;
                Bout[dst] = rb;
            }
            n_fs += (unsigned)__popc(fast);
            if (slow) {
                if (W.qn + __popc(slow) > QCAP)
                    drain_movers(P, sys, W.q, &W.qn, W.wq, &W.wqn, W.wtally, lane, move_step);
                if (valid && !stay) {
                    SlowRec &rec = W.q[W.qn + __popc(slow & ((1u << lane) - 1u))];
                    Split32::pack(p, rec.a, rec.b);
                    rec.cell = a;
                    rec.global = T.glob[ci];
                }
                __syncwarp();
                if (lane == 0) W.qn += __popc(slow);
                __syncwarp();
            }
        }
        if (lane == ci) nfs_mine = n_fs;
        if (lane == 0) W.wtally[T_MOVED] += (unsigned)n;
        // free the cell's ring slots once every lane is done with them
        __syncwarp();
        tail += n;
        if (tail >= R) tail -= R;
        used -= n;
        --ahead;
        ++ci;
    }
    if (W.qn) drain_movers(P, tsys, W.q, &W.qn, W.wq, &W.wqn, W.wtally, lane, move_step);
    if (W.wqn) drain_wall(P, tsys, W.wq, &W.wqn, W.wtally, lane, move_step);
    if (tsys >= 0) flush_warp(P, W, tsys, lane);

    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned done = atomicAdd(&P.status->blocks_done, 1u);
        if (done == gridDim.x - 1) {
            __threadfence();
            if (P.advance_step) atomicAdd(&P.status->step, 1u);
            if (atomicAdd(&P.status->spill, 0u) != 0u || (atomicAdd(&P.status->error, 0u) & DSMC_EBIT_FATAL) != 0u)
                atomicExch(&P.status->halted, 1u);
            atomicExch(&P.status->blocks_done, 0u);
        }
    }
}

template <int R> size_t fused_smem_bytes() { return sizeof(WarpSmem<R>) * FUSED_WARPS; }

}  // namespace fused
}  // namespace dsmc
