// The production timestep pass for split-precision state: four kernels per
// step (five on sampled steps) over the active cells, which the previous pass
// left sorted by cell (bottom segment + top segment of each cell's slots,
// counts in the `cin` occupancy set).
//
//   collide_cells  Cell::prepare + Cell::collide (dsmc/cell.cpp:42-111) of
//                  every cell.
//                  Per chunk of 32 consecutive cells lane i selects for cell
//                  i; the warp ranks each colliding cell's particles by id
//                  (the reference's member order) into shared memory, then
//                  every lane runs the candidate loop of its own cell.
//                  Velocities are updated in place in the input buffer.
//   sample_cells   On sampled steps only (the reference's cadence,
//                  dsmc/statisticssampler.cpp:45-66): every cell's fp64
//                  moments and the y-binned profiles.
//   move_cells     System::accelerate + the mover's first flight
//                  (dsmc/system.cpp:133-144, dsmc/moleculemover.cpp:50-126)
//                  for every particle.  A particle that stays inside its
//                  empty voxel goes, moved, to the bottom segment of its cell
//                  in the output buffer; the rest ("movers"), accelerated but
//                  not moved, go to the gap just above: slots
//                  [base + stayers, base + n_in) hold exactly the cell's
//                  movers.  Particle records stream through a per-warp
//                  shared-memory ring with 16-byte cp.async copies.
//   place_movers   A mover whose flight ends in an empty voxel completes it
//                  and takes a top slot of its new cell (warp-aggregated
//                  atomics; the spill list when the cell is full).  Flights
//                  that meet a wall go to a list of (slot, source cell)
//                  pairs.
//   place_walls    The general mover (bisection, facet, diffuse wall) for
//                  the listed flights, then the same placement.  The last
//                  block ends the pass (step counter, halting).
//
// Top slots are taken from the top of the cell down and never below
// base + n_in(cell), so they cannot meet the bottom segment or the gap.
//
// Member order: move_cells writes each cell's stayers in id order, so a
// bottom segment is normally sorted by id and only the few arrivals of the
// top segment are out of order.  The id rank of a member (the reference's
// cell-list order) is then its bottom position plus the arrivals below it,
// which collide_cells and move_cells compute with one shuffle and ballot per
// arrival.  A cell whose bottom segment is not sorted (after a repack or the
// stand-alone stage kernels) is ranked in full and leaves move_cells sorted.
#pragma once
#include "engine.cuh"

namespace dsmc {
namespace pass3 {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 16-byte global -> shared copy, cached in L2 only (both addresses 16-byte
// aligned: slots are uint4/float4 records).
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most `pending` of this thread's newest commit groups are
// still in flight (more than 4 is treated as 4, which waits longer).
__device__ __forceinline__ void cp_async_wait(int pending) {
    switch (pending) {
        case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
        case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
        case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
        case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
        default: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
    }
}

// Input occupancy of active cell a (clamped to its capacity).
__device__ __forceinline__ void input_counts(const PassParams &P, int a, const int4 &m, unsigned &nb, unsigned &nt) {
    nb = min(P.cells.bot[P.cin][a], (unsigned)m.y);
    nt = min(P.cells.top[P.cin][a], (unsigned)m.y - nb);
}
// Slot of member q of a cell: bottom segment, then top segment.
__device__ __forceinline__ int member_slot(int base, int cap, int nb, int nt, int q) {
    return q < nb ? base + q : base + cap - nt + (q - nb);
}

__device__ __forceinline__ unsigned warp_sum(unsigned x) { return __reduce_add_sync(0xffffffffu, x); }
__device__ __forceinline__ int warp_sum(int x) { return __reduce_add_sync(0xffffffffu, x); }

// The system shared by the valid lanes of a warp, or -2 when they differ
// (-1 when no lane is valid).  All lanes call.
__device__ __forceinline__ int common_system(bool valid, int sys) {
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    if (!vm) return -1;
    const int s0 = __shfl_sync(0xffffffffu, sys, __ffs(vm) - 1);
    return __all_sync(0xffffffffu, !valid || sys == s0) ? s0 : -2;
}

// collide_cells' chunks of 32 cells beyond each warp's first go to warps from
// a pass-wide counter when there are many per warp, so that a warp that
// finishes early takes more (a chunk's cost varies with its cells'
// collisions); place_walls' last block zeroes the counter for the next pass.
// Four chunks per warp or more take the counter.  (move_cells, place_movers
// and sample_cells keep a fixed stride: a counter made them no faster or
// slower.)  claim_issue starts a claim (lane 0), claim_take hands its chunk
// to every lane: issued a chunk ahead, the atomic's latency is hidden.
constexpr int CLAIM_MIN_CHUNKS_PER_WARP = 4;
__device__ __forceinline__ unsigned claim_issue(unsigned *counter, int lane) {
    return lane == 0 ? atomicAdd(counter, 1u) : 0u;
}
__device__ __forceinline__ int claim_take(unsigned claimed) { return (int)__shfl_sync(0xffffffffu, claimed, 0); }

// ---- collide_cells ----------------------------------------------------------

constexpr int C_WARPS = 4;
constexpr int PCAP = 512;    // members per warp and batch (>= the largest cell)
constexpr int NTMAX = 8;     // arrivals a lane merges on its own (sorted bottom segments)

struct CollideSmem {
    uint32_t ids[PCAP];  // batch members: ids and slots, cell by cell
    int slot[PCAP];
    int perm[PCAP];      // batch members by id rank within each cell (warp-ranked cells)
    int apos[32 * (NTMAX + 1)];   // lane i: its cell's arrivals in id order: merged rank
    int aslot[32 * (NTMAX + 1)];  //   and slot (rows of NTMAX + 1: no bank conflicts)
};

// Velocities of one cell's members in the input buffer, by id rank.
struct RankVel {
    float4 *b;
    const int *perm;
    __device__ __forceinline__ void get(int r, float &x, float &y, float &z) const {
        const float4 v = b[perm[r]];
        x = v.x;
        y = v.y;
        z = v.z;
    }
    __device__ __forceinline__ void set(int r, float x, float y, float z) const {
        float *q = reinterpret_cast<float *>(b + perm[r]);
        q[0] = x;
        q[1] = y;
        q[2] = z;
    }
};
struct IdentityPerm {
    __device__ __forceinline__ int operator[](int i) const { return i; }
};
// Velocities of a cell's members by slot.
struct SlotVel {
    float4 *b;
    __device__ __forceinline__ void get(int s, float &x, float &y, float &z) const {
        const float4 v = b[s];
        x = v.x;
        y = v.y;
        z = v.z;
    }
    __device__ __forceinline__ void set(int s, float x, float y, float z) const {
        float *q = reinterpret_cast<float *>(b + s);
        q[0] = x;
        q[1] = y;
        q[2] = z;
    }
};
// Slot of the member of id rank r in a cell whose bottom segment is sorted:
// an arrival if one has merged rank r, else the bottom member r minus the
// arrivals below.
struct PickPerm {
    const int *apos, *aslot;
    int nt, base;
    __device__ __forceinline__ int operator[](int r) const {
        int below = 0;
        for (int j = 0; j < nt; ++j) {
            const int p = apos[j];
            if (p == r) return aslot[j];
            below += p < r;
        }
        return base + (r - below);
    }
};

__device__ __forceinline__ void publish_collide(const PassParams &P, int sys, unsigned col, unsigned cand,
                                                bool per_lane) {
    if (per_lane) {
        if (sys >= 0) {
            if (col) atomicAdd(&P.tally[sys].collisions, (unsigned long long)col);
            if (cand) atomicAdd(&P.tally[sys].candidates, (unsigned long long)cand);
        }
        return;
    }
    const unsigned c = warp_sum(col), d = warp_sum(cand);
    if ((threadIdx.x & 31) == 0 && sys >= 0) {
        if (c) atomicAdd(&P.tally[sys].collisions, (unsigned long long)c);
        if (d) atomicAdd(&P.tally[sys].candidates, (unsigned long long)d);
    }
}

// CLAIM: chunks beyond each warp's first come from the counter (chosen by
// the launcher when there are many chunks per warp; a fixed stride measured
// faster with few: packed_64 and packed_128).
template <bool CLAIM>
__global__ void __launch_bounds__(32 * C_WARPS) collide_cells_kernel(const __grid_constant__ PassParams P) {
    __shared__ CollideSmem smem[C_WARPS];
    const int lane = threadIdx.x & 31;
    const volatile Status *vs = P.status;
    if (vs->halted) return;
    const uint32_t step = vs->step;
    CollideSmem &W = smem[threadIdx.x >> 5];
    float4 *Bin = reinterpret_cast<float4 *>(P.parts.B[P.cur]);

    const int C = P.cells.num_cells;
    const int nchunks = (C + 31) >> 5;
    unsigned col = 0, cand = 0;  // this lane's counts for system tsys
    int tsys = -1;

    // A warp's first chunk is its index; with CLAIM the later ones come from
    // the counter, each claimed while the chunk before is in work.
    const int nw = gridDim.x * C_WARPS;
    unsigned nxt = 0;
    for (int ch = blockIdx.x * C_WARPS + (threadIdx.x >> 5); ch < nchunks;
         ch = CLAIM ? nw + claim_take(nxt) : ch + nw) {
        if (CLAIM) nxt = claim_issue(&P.status->collide_taken, lane);  // the next chunk, in flight meanwhile
        const int first = ch * 32;
        const bool mine = lane < C - first;
        const int a = first + lane;
        int4 m = make_int4(0, 0, 0, -1);
        unsigned nb = 0, nt = 0;
        double vr = 0, rest = 0;
        int pairs = 0;
        if (mine) {
            m = P.cells.meta[a];
            input_counts(P, a, m, nb, nt);
            const double4 st = P.cells.state[a];
            vr = st.x;
            rest = st.y;
            if (P.do_collide) {
                pairs = ntc_select(st.z, (int)(nb + nt), vr, rest);
                if (nb + nt < 2) pairs = 0;
                if (nb + nt > (unsigned)PCAP) {  // the host keeps every cap below PCAP
                    atomicOr(&P.status->error, DSMC_EBIT_SMEM);
                    pairs = 0;
                }
            }
        }
        const int n = (int)(nb + nt);
        const int sys = m.w;
        const int csys = common_system(mine, sys);
        if (csys != tsys) {
            publish_collide(P, tsys, col, cand, false);
            col = cand = 0;
            tsys = csys;
        }

        // Rank the colliding cells' members by id, a batch at a time, and
        // run the batch's candidate loops one cell per lane.
        unsigned todo = __ballot_sync(0xffffffffu, pairs > 0);
        while (todo) {
            // the batch: colliding cells, in order, whose members fit PCAP
            unsigned ready = 0;
            {
                int off = 0;
                for (unsigned t2 = todo; t2;) {
                    const int c = __ffs(t2) - 1;
                    const int nc = __shfl_sync(0xffffffffu, n, c);
                    if (off + nc > PCAP) break;  // off > 0 here: nc <= PCAP
                    off += nc;
                    ready |= 1u << c;
                    t2 &= t2 - 1u;
                }
            }
            todo &= ~ready;
            // offsets of the batch cells' members: exclusive prefix over lanes
            const bool rb = (ready >> lane) & 1u;
            const int nr = rb ? n : 0;
            int incl = nr;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int start = incl - nr;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            // ids and slots of every batch member: independent loads
            for (int f0 = 0; f0 < total; f0 += 32) {
                const int f = f0 + lane;
                int c = 0;  // the last lane whose start is <= f: a batch cell holding member f
#pragma unroll
                for (int st = 16; st > 0; st >>= 1) {
                    const int sc = __shfl_sync(0xffffffffu, start, c + st);
                    if (sc <= f) c += st;
                }
                const int k = f - __shfl_sync(0xffffffffu, start, c);
                const int cb = __shfl_sync(0xffffffffu, m.x, c), cc = __shfl_sync(0xffffffffu, m.y, c);
                const int cnb = (int)__shfl_sync(0xffffffffu, nb, c), cnt = __shfl_sync(0xffffffffu, n, c) - cnb;
                if (f < total) W.slot[f] = member_slot(cb, cc, cnb, cnt, k);
            }
            __syncwarp();
            // the members' ids, four loads in flight per lane
            for (int f0 = lane; f0 < total; f0 += 128) {
                uint32_t v[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int f = f0 + 32 * u;
                    v[u] = f < total ? __float_as_uint(Bin[W.slot[f]].w) : 0u;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (f0 + 32 * u < total) W.ids[f0 + 32 * u] = v[u];
            }
            __syncwarp();
            // Cells with a sorted bottom and few arrivals: each lane sorts its
            // cell's arrivals and finds their merged ranks by binary search.
            const bool lp = rb && P.sorted_in && (int)nt <= NTMAX;
            if (lp) {
                uint32_t *ids = W.ids + start;
                int *sl = W.slot + start;
                const int b = (int)nb;
                for (int j = b + 1; j < n; ++j) {
                    const uint32_t id = ids[j];
                    const int s = sl[j];
                    int i = j - 1;
                    while (i >= b && ids[i] > id) {
                        ids[i + 1] = ids[i];
                        sl[i + 1] = sl[i];
                        --i;
                    }
                    ids[i + 1] = id;
                    sl[i + 1] = s;
                }
                int *ap = W.apos + lane * (NTMAX + 1), *as = W.aslot + lane * (NTMAX + 1);
                for (int j = 0; j < (int)nt; ++j) {
                    const uint32_t id = ids[b + j];
                    int lo = 0, hi = b;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (ids[mid] < id) lo = mid + 1;
                        else hi = mid;
                    }
                    ap[j] = lo + j;
                    as[j] = sl[b + j];
                }
            }
            // The other cells: id ranks by the warp, cell by cell.
            const unsigned wr = ready & ~__ballot_sync(0xffffffffu, lp);
            for (unsigned t2 = wr; t2; t2 &= t2 - 1u) {
                const int c = __ffs(t2) - 1;
                const int off = __shfl_sync(0xffffffffu, start, c);
                const int nc = __shfl_sync(0xffffffffu, n, c);
                const int nbc = (int)__shfl_sync(0xffffffffu, nb, c);
                const int ntc = nc - nbc;
                if (nc <= 32) {
                    const uint32_t id = lane < nc ? W.ids[off + lane] : 0xffffffffu;
                    const uint32_t nxt = __shfl_down_sync(0xffffffffu, id, 1);
                    const bool sorted = !__any_sync(0xffffffffu, lane + 1 < nbc && !(id < nxt));
                    int rank = 0;
                    if (sorted) {
                        // bottom position (or the bottom members below an
                        // arrival) plus the arrivals below
                        const unsigned bmask = nbc >= 32 ? 0xffffffffu : (1u << nbc) - 1u;
                        unsigned add = 0, pb = 0;
                        for (int i = 0; i < ntc; ++i) {
                            const uint32_t t = __shfl_sync(0xffffffffu, id, nbc + i);
                            add += t < id;
                            const unsigned bl = __popc(bmask & __ballot_sync(0xffffffffu, id < t));
                            if (lane == nbc + i) pb = bl;
                        }
                        rank = (lane < nbc ? lane : (int)pb) + (int)add;
                    } else {
#pragma unroll
                        for (int r = 0; r < 32; ++r) rank += __shfl_sync(0xffffffffu, id, r) < id;
                    }
                    if (lane < nc) W.perm[off + rank] = W.slot[off + lane];
                } else {
                    const uint32_t *ids = W.ids + off;
                    bool viol = false;
                    for (int q = lane; q + 1 < nbc; q += 32) viol |= !(ids[q] < ids[q + 1]);
                    const bool sorted = !__any_sync(0xffffffffu, viol);
                    for (int q = lane; q < nc; q += 32) {
                        const uint32_t id = ids[q];
                        int rank = 0;
                        if (sorted) {
                            if (q < nbc) {
                                rank = q;
                            } else {  // bottom members below: binary search
                                int lo = 0, hi = nbc;
                                while (lo < hi) {
                                    const int mid = (lo + hi) >> 1;
                                    if (ids[mid] < id) lo = mid + 1;
                                    else hi = mid;
                                }
                                rank = lo;
                            }
                            for (int i = nbc; i < nc; ++i) rank += ids[i] < id;
                        } else {
                            for (int r = 0; r < nc; ++r) rank += ids[r] < id;
                        }
                        W.perm[off + rank] = W.slot[off + q];
                    }
                }
            }
            __syncwarp();
            if (rb) {
                const SysDev &g = P.sys[sys];
                DrawStream rs;
                rs.init(g.seed, (uint32_t)m.z, step, DSMC_TAG_COLLIDE);
                unsigned long long c_ = 0;
                if (lp) {
                    SlotVel vel;
                    vel.b = Bin;
                    PickPerm pick;
                    pick.apos = W.apos + lane * (NTMAX + 1);
                    pick.aslot = W.aslot + lane * (NTMAX + 1);
                    pick.nt = (int)nt;
                    pick.base = m.x;
                    ntc_loop<float>(rs, n, pairs, vr, vel, pick, c_);
                } else {
                    RankVel vel;
                    vel.b = Bin;
                    vel.perm = W.perm + start;
                    ntc_loop<float>(rs, n, pairs, vr, vel, IdentityPerm(), c_);
                }
                col += (unsigned)c_;
                cand += (unsigned)pairs;
            }
            __syncwarp();
        }
        if (mine && P.do_collide)
            *reinterpret_cast<double2 *>(&P.cells.state[a]) = make_double2(vr, rest);

        if (tsys == -2) {  // a chunk that spans systems: per-lane counts
            publish_collide(P, sys, col, cand, true);
            col = cand = 0;
        }
    }
    publish_collide(P, tsys, col, cand, false);
}

// ---- sample_cells -----------------------------------------------------------

constexpr int SHIST = 1024;  // v_x histogram bins a warp counts in shared memory

// Eight per-lane values summed over the warp, transposed: lane l returns the
// sum of slot l >> 2 (lanes 4j..4j+3 hold the sum of slot j).  Each exchange
// halves the slots a lane carries (4, 2, 1, then two plain steps): 9 fp64
// shuffles where eight separate reductions take 40.  All lanes call.
__device__ __forceinline__ double warp_transpose_sum8(const double (&v)[8], int lane) {
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
    double w[4], u[2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
        w[i] = (b4 ? v[i + 4] : v[i]) + __shfl_xor_sync(0xffffffffu, b4 ? v[i] : v[i + 4], 16);
#pragma unroll
    for (int i = 0; i < 2; ++i)
        u[i] = (b3 ? w[i + 2] : w[i]) + __shfl_xor_sync(0xffffffffu, b3 ? w[i] : w[i + 2], 8);
    double t = (b2 ? u[1] : u[0]) + __shfl_xor_sync(0xffffffffu, b2 ? u[0] : u[1], 4);
    t += __shfl_xor_sync(0xffffffffu, t, 2);
    t += __shfl_xor_sync(0xffffffffu, t, 1);
    return t;
}

// The sampler on the reference's cadence (StatisticsSampler::sample,
// dsmc/statisticssampler.cpp:45-66), after collide_cells on sampled steps
// only: every cell's fp64 moments and the y-binned profiles.  A warp takes a
// chunk of 32 cells, their headers one per lane, then each sampled cell with
// its members over the lanes.  Per cell one transposing butterfly sums the
// six velocity moments and the cell's profile sums {v_z, 1/2 m v_z^2} in the
// bin of its first member (members in another bin, rare when the bins are
// no finer than the cells, add their own); lanes 4j then add slot j to the
// cell's moment row or the profile.  Each warp counts the v_x histogram in
// shared memory and adds it to its copy of the sums once per system (every
// particle lands in one of a few bins: one global atomic per particle queued
// on those addresses).
__global__ void __launch_bounds__(32 * C_WARPS) sample_cells_kernel(const __grid_constant__ PassParams P) {
    __shared__ unsigned hist[C_WARPS][SHIST];
    const int lane = threadIdx.x & 31;
    const volatile Status *vs = P.status;
    if (vs->halted) return;
    const uint32_t step = vs->step;
    const float4 *Bin = reinterpret_cast<const float4 *>(P.parts.B[P.cur]);
    const uint4 *Ain = reinterpret_cast<const uint4 *>(P.parts.A[P.cur]);
    unsigned *H = hist[threadIdx.x >> 5];
    for (int b = lane; b < SHIST; b += 32) H[b] = 0;
    __syncwarp();
    int hsys = -1;  // the system whose histogram H holds
    auto flush = [&]() {
        if (hsys >= 0) {
            const SysDev &gh = P.sys[hsys];
            double *pr = profile_copy(gh) + 3 * (size_t)gh.prof_bins;
            for (int b = lane; b < gh.prof_bins; b += 32)
                if (H[b]) {
                    atomicAdd(pr + b, (double)H[b]);
                    H[b] = 0;
                }
            __syncwarp();
        }
    };
    // moment row entry this lane adds: slot j of the butterfly to M[1 + j]
    // (j < 6), lane 1 the count to M[0]; lane 12 also M[7] = the three sums
    // of squares
    const int slot = lane >> 2;
    const int mcol = (lane & 3) == 0 && slot < 6 ? 1 + slot : lane == 1 ? 0 : -1;
    const int C = P.cells.num_cells;
    const int nchunks = (C + 31) >> 5;
    const int nwarps = gridDim.x * C_WARPS;
    for (int ch = blockIdx.x * C_WARPS + (threadIdx.x >> 5); ch < nchunks; ch += nwarps) {
        const int a = ch * 32 + lane;
        int4 m = make_int4(0, 0, 0, -1);
        unsigned nb = 0, nt = 0;
        bool smp = false;
        if (a < C) {
            m = P.cells.meta[a];
            input_counts(P, a, m, nb, nt);
            const SysDev &g = P.sys[m.w];
            smp = g.sample_interval > 0 && step > 0 && (step % (uint32_t)g.sample_interval) == 0 &&
                  step >= (uint32_t)g.sample_begin;
        }
        for (unsigned todo = __ballot_sync(0xffffffffu, smp); todo; todo &= todo - 1u) {
            const int c = __ffs(todo) - 1;
            const int ac = ch * 32 + c;
            const int sys = __shfl_sync(0xffffffffu, m.w, c);
            const int cb = __shfl_sync(0xffffffffu, m.x, c), cc = __shfl_sync(0xffffffffu, m.y, c);
            const int cnb = (int)__shfl_sync(0xffffffffu, nb, c), cnt = (int)__shfl_sync(0xffffffffu, nt, c);
            const int n = cnb + cnt;
            const SysDev &g = P.sys[sys];
            double *M = P.cells.mom + 8 * (size_t)ac;
            const double mold = mcol >= 0 ? M[mcol] : 0.0;  // in flight with the members' loads
            const double m7 = lane == 12 ? M[7] : 0.0;
            const bool local = g.prof_bins <= SHIST;
            if (local && sys != hsys) {
                flush();
                hsys = sys;
            }
            // Σv_x Σv_y Σv_z Σv_x² Σv_y² Σv_z², then Σv_z and Σ 1/2 m v_z² in bin b0
            double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            int b0 = 0;
            unsigned in0 = 0;  // members in bin b0
            for (int q0 = 0; q0 < n; q0 += 32) {
                const int q = q0 + lane;
                const bool ok = q < n;
                int bin = 0;
                double x = 0, y = 0, z = 0;
                if (ok) {
                    const int sl = member_slot(cb, cc, cnb, cnt, q);
                    const float4 b = Bin[sl];
                    x = b.x;
                    y = b.y;
                    z = b.z;
                    bin = profile_bin(g, Split32::y_of(g, Ain[sl]));
                    v[0] += x;
                    v[1] += y;
                    v[2] += z;
                    v[3] += x * x;
                    v[4] += y * y;
                    v[5] += z * z;
                }
                if (q0 == 0) b0 = __shfl_sync(0xffffffffu, bin, 0);
                const bool here = ok && bin == b0;
                const double e = 0.5 * g.mass * z * z;
                if (here) {
                    v[6] += z;
                    v[7] += e;
                }
                in0 += (unsigned)__popc(__ballot_sync(0xffffffffu, here));
                profile_add_warp(g, ok && !here, bin, 1.0, z, e);
                if (ok) {
                    if (local) {
                        const int hb = profile_vx_bin(g, x);
                        if (hb >= 0) atomicAdd(&H[hb], 1u);
                    } else {
                        profile_vx(g, x);
                    }
                }
            }
            const double t = warp_transpose_sum8(v, lane);
            const double sq = __shfl_sync(0xffffffffu, t, 12) + __shfl_sync(0xffffffffu, t, 16) +
                              __shfl_sync(0xffffffffu, t, 20);
            if (mcol >= 0) M[mcol] = mold + (mcol == 0 ? (double)n : t);
            if (lane == 12) M[7] = m7 + sq;
            if (in0) {
                double *pr = profile_copy(g) + 3 * b0;
                if (lane == 2) atomicAdd(pr, (double)in0);
                if (lane == 24) atomicAdd(pr + 1, t);
                if (lane == 28) atomicAdd(pr + 2, t);
            }
            if (lane == 0 && ac == g.active_begin) atomicAdd(&P.tally[sys].samples, 1ull);
        }
    }
    flush();
}

// ---- move_cells -------------------------------------------------------------

constexpr int M_WARPS = 4;
constexpr int DEPTH = 4;  // cells staged ahead of the one in work

struct MoveTab {
    int base[32], cap[32];
    unsigned nb[32], nt[32];
    int sys[32];
    int first, ncell;
};
template <int R> struct MoveSmem {
    uint4 A[R];
    float4 B[R];
    MoveTab tab[2];
    uint16_t pref[R + 2];  // two-pass placement: stayers before each member
};

// accelerate, then the first flight when it stays inside the particle's
// empty voxel (the reference's outcome: r += v dt lands in an empty voxel,
// dsmc/moleculemover.cpp:74-77); false leaves the particle accelerated.
__device__ __forceinline__ bool first_flight(const SysDev &g, Split32::Particle &p) {
    Split32::accelerate(g, p);
    if (p.flag) return false;
    float x[3];
    bool stay = true;
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
    return stay;
}

// A system's constants of the first flight, held in registers.
struct FlightConst {
    float inv_vox[3], dt, accel;
    int flow_dir;
};
__device__ __forceinline__ FlightConst flight_const(const SysDev &g) {
    FlightConst k;
#pragma unroll
    for (int d = 0; d < 3; ++d) k.inv_vox[d] = g.inv_vox_f[d];
    k.dt = g.dt_f;
    k.accel = g.accel_dt_f;
    k.flow_dir = g.flow_dir;
    return k;
}
// first_flight on the packed record itself: the voxel index is never
// unpacked (a stayer changes only its offsets, a mover only its velocity).
// Bit for bit what unpack + first_flight + pack give.
__device__ __forceinline__ bool first_flight_raw(const FlightConst &k, uint4 &a, float4 &b) {
    b.x = k.flow_dir == 0 ? b.x + k.accel : b.x;
    b.y = k.flow_dir == 1 ? b.y + k.accel : b.y;
    b.z = k.flow_dir == 2 ? b.z + k.accel : b.z;
    if (a.y >> 31) return false;  // the voxel is not empty: general mover
    const float x0 = fmaf(b.x * k.inv_vox[0], k.dt, __uint_as_float(a.y));
    const float x1 = fmaf(b.y * k.inv_vox[1], k.dt, __uint_as_float(a.z));
    const float x2 = fmaf(b.z * k.inv_vox[2], k.dt, __uint_as_float(a.w));
    const bool stay = (x0 >= 0.0f) & (x0 < 1.0f) & (x1 >= 0.0f) & (x1 < 1.0f) & (x2 >= 0.0f) & (x2 < 1.0f);
    if (stay) {
        a.y = __float_as_uint(x0);
        a.z = __float_as_uint(x1);
        a.w = __float_as_uint(x2);
    }
    return stay;
}

// One cell of at most 32 * NR members whose bottom segment is sorted by id,
// held in registers (member q = 32 k + lane in p[k]): flight of every member,
// then stayers to the bottom segment in id order and movers to the gap.
// Returns the number of stayers.  All lanes call.
template <int R, int NR>
__device__ __forceinline__ unsigned place_sorted(const FlightConst &fc, const MoveSmem<R> &W, int tail, int base,
                                                 int n, int nb, uint4 *Aout, float4 *Bout, int lane) {
    const unsigned below = (1u << lane) - 1u;
    uint4 ra[NR];
    float4 rb[NR];
    bool stay[NR];
    uint32_t id[NR];
    unsigned fast[NR], slow[NR], bm[NR], add[NR], pb[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
        const int q = 32 * k + lane;
        const bool valid = q < n;
        stay[k] = false;
        if (valid) {
            int r = tail + q;
            if (r >= R) r -= R;
            ra[k] = W.A[r];
            rb[k] = W.B[r];
            stay[k] = first_flight_raw(fc, ra[k], rb[k]);
        }
        id[k] = valid ? __float_as_uint(rb[k].w) : 0xffffffffu;
        fast[k] = __ballot_sync(0xffffffffu, valid && stay[k]);
        slow[k] = __ballot_sync(0xffffffffu, valid && !stay[k]);
        const int nbk = nb - 32 * k;  // bottom members of chunk k
        bm[k] = nbk >= 32 ? 0xffffffffu : nbk <= 0 ? 0u : (1u << nbk) - 1u;
        add[k] = pb[k] = 0;
    }
    // each arrival i: staying arrivals below every member, bottom stayers
    // below the arrival
    for (int i = nb; i < n; ++i) {
        const int li = i & 31;
        const bool hi = NR > 1 && i >= 32;
        const uint32_t t = __shfl_sync(0xffffffffu, hi ? id[NR - 1] : id[0], li);
        const unsigned ts = ((hi ? fast[NR - 1] : fast[0]) >> li) & 1u;
        unsigned bl = 0;
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            add[k] += ts && t < id[k];
            bl += (unsigned)__popc(fast[k] & bm[k] & __ballot_sync(0xffffffffu, id[k] < t));
        }
        if (lane == li) {
            if (hi) pb[NR - 1] = bl;
            else pb[0] = bl;
        }
    }
    unsigned fs_before = 0, mv_before = 0;  // bottom stayers and movers of the earlier chunks
#pragma unroll
    for (int k = 0; k < NR; ++k) {
        const int q = 32 * k + lane;
        if (q < n) {
            const unsigned dst =
                stay[k] ? (unsigned)base + (q < nb ? fs_before + (unsigned)__popc(fast[k] & bm[k] & below) : pb[k]) + add[k]
                        : (unsigned)(base + n) - 1u - mv_before - (unsigned)__popc(slow[k] & below);
            Aout[dst] = ra[k];
            Bout[dst] = rb[k];
        }
        fs_before += (unsigned)__popc(fast[k] & bm[k]);
        mv_before += (unsigned)__popc(slow[k]);
    }
    unsigned nfs = 0;
#pragma unroll
    for (int k = 0; k < NR; ++k) nfs += (unsigned)__popc(fast[k]);
    return nfs;
}

// Two consecutive cells of at most 32 members each with sorted bottom
// segments and one system: place_sorted<R, 1> for both, written as one
// straight-line body so that the two cells' dependency chains interleave.
// nfs[k]: stayers of cell k.  All lanes call.
template <int R>
__device__ __forceinline__ void place_pair(const FlightConst &fc, const MoveSmem<R> &W, int tail, const int base[2],
                                          const int n[2], const int nb[2], uint4 *Aout, float4 *Bout, int lane,
                                          unsigned nfs[2]) {
    const unsigned below = (1u << lane) - 1u;
    uint4 ra[2];
    float4 rb[2];
    bool stay[2];
    uint32_t id[2];
    unsigned fast[2], slow[2], bm[2], add[2], pb[2];
    int t1 = tail + n[0];
    if (t1 >= R) t1 -= R;
    const int tl[2] = {tail, t1};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const bool valid = lane < n[k];
        stay[k] = false;
        if (valid) {
            int r = tl[k] + lane;
            if (r >= R) r -= R;
            ra[k] = W.A[r];
            rb[k] = W.B[r];
            stay[k] = first_flight_raw(fc, ra[k], rb[k]);
        }
        id[k] = valid ? __float_as_uint(rb[k].w) : 0xffffffffu;
        fast[k] = __ballot_sync(0xffffffffu, valid && stay[k]);
        slow[k] = __ballot_sync(0xffffffffu, valid && !stay[k]);
        bm[k] = nb[k] >= 32 ? 0xffffffffu : (1u << nb[k]) - 1u;
        add[k] = pb[k] = 0;
    }
    // arrival j of each cell: staying arrivals below every member, bottom
    // stayers below the arrival (both cells in every iteration)
    const int nt0 = n[0] - nb[0], nt1 = n[1] - nb[1];
    const int ntmax = max(nt0, nt1);
    for (int j = 0; j < ntmax; ++j) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const bool has = j < (k ? nt1 : nt0);
            const int li = (nb[k] + j) & 31;
            const uint32_t t = __shfl_sync(0xffffffffu, id[k], li);
            const unsigned ts = has ? (fast[k] >> li) & 1u : 0u;
            add[k] += ts && t < id[k];
            const unsigned bl = (unsigned)__popc(fast[k] & bm[k] & __ballot_sync(0xffffffffu, id[k] < t));
            if (has && lane == li) pb[k] = bl;
        }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (lane < n[k]) {
            const unsigned dst =
                stay[k] ? (unsigned)base[k] + (lane < nb[k] ? (unsigned)__popc(fast[k] & bm[k] & below) : pb[k]) + add[k]
                        : (unsigned)(base[k] + n[k]) - 1u - (unsigned)__popc(slow[k] & below);
            Aout[dst] = ra[k];
            Bout[dst] = rb[k];
        }
        nfs[k] = (unsigned)__popc(fast[k]);
    }
}

// At most 128 registers (four blocks per SM): the compiler then keeps both
// cells of a pair in flight; left to itself it may pick 96 and five blocks,
// which measured slower.
template <int R>
__global__ void __launch_bounds__(32 * M_WARPS, 4) move_cells_kernel(const __grid_constant__ PassParams P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    typedef Split32::Particle Particle;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const volatile Status *vs = P.status;
    if (vs->halted) return;

    MoveSmem<R> &W = reinterpret_cast<MoveSmem<R> *>(smem_raw)[wib];
    const uint4 *Ain = reinterpret_cast<const uint4 *>(P.parts.A[P.cur]);
    const float4 *Bin = reinterpret_cast<const float4 *>(P.parts.B[P.cur]);
    uint4 *Aout = reinterpret_cast<uint4 *>(P.parts.A[P.cur ^ 1]);
    float4 *Bout = reinterpret_cast<float4 *>(P.parts.B[P.cur ^ 1]);

    const int C = P.cells.num_cells;
    const int nchunks = (C + 31) >> 5;
    const int wstride = gridDim.x * M_WARPS;
    const int chunk0 = blockIdx.x * M_WARPS + wib;

    auto load_tab = [&](int b, int ch) {
        MoveTab &T = W.tab[b];
        const int first = ch * 32;
        const int ncell = ch < nchunks ? min(32, C - first) : 0;
        if (lane == 0) {
            T.first = first;
            T.ncell = ncell;
        }
        if (lane < ncell) {
            const int a = first + lane;
            const int4 m = P.cells.meta[a];
            unsigned nb, nt;
            input_counts(P, a, m, nb, nt);
            if (nb + nt > (unsigned)R) atomicOr(&P.status->error, DSMC_EBIT_SMEM);  // the host sizes R above every cap
            // top slots free for arrivals this pass: above the input occupancy
            P.cells.room[a] = make_int2(m.x + m.y, m.y - (int)(nb + nt));
            T.base[lane] = m.x;
            T.cap[lane] = m.y;
            T.nb[lane] = nb;
            T.nt[lane] = nt;
            T.sys[lane] = m.w;
        }
    };
    // Lane i publishes cell i's bottom occupancy and clears the set the next
    // pass writes.
    auto write_tab = [&](int b, unsigned nfs) {
        const MoveTab &T = W.tab[b];
        if (lane < T.ncell) {
            const int a = T.first + lane;
            P.cells.bot[P.cout][a] = nfs;
            P.cells.bot[P.cclear][a] = 0;
            P.cells.top[P.cclear][a] = 0;
        }
    };

    load_tab(0, chunk0);
    load_tab(1, chunk0 + wstride);
    __syncwarp();

    int head = 0, tail = 0, used = 0;  // ring (warp-uniform)
    int it = 0, ii = 0;                // next cell to stage: chunk ordinal, cell in chunk
    int ct = 0, ci = 0;                // cell in work
    int ahead = 0;                     // cells staged, the one in work included
    unsigned nfs_mine = 0;             // lane i: bottom occupancy of cell i of the chunk in work
    unsigned moved = 0;                // particles moved, system tsys (warp-uniform)
    int tsys = -1;
    FlightConst fc = {};               // constants of system tsys

    auto stage_ahead = [&]() {
        // (it, ii) moves past a full chunk as soon as its last cell is
        // staged, so ii >= ncell only past the warp's last cell
        while (ahead <= DEPTH && it <= ct + 1) {
            const MoveTab &T = W.tab[it & 1];
            if (ii >= T.ncell) return;
            const int nb = (int)T.nb[ii], nt = (int)T.nt[ii];
            const int n = min(nb + nt, R);
            if (used + n > R) return;
            const int base = T.base[ii], cap = T.cap[ii];
            for (int q = lane; q < n; q += 32) {
                const int slot = member_slot(base, cap, nb, nt, q);
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
        const MoveTab &T = W.tab[ct & 1];
        if (ci >= T.ncell) {
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
        // Two small cells of one system with sorted bottoms go together.
        if (P.sorted_in && ahead >= 2 && ci + 1 < T.ncell && T.sys[ci + 1] == T.sys[ci] &&
            T.sys[ci] == tsys && T.nb[ci] + T.nt[ci] <= 32u && T.nb[ci + 1] + T.nt[ci + 1] <= 32u) {
            cp_async_wait(ahead - 2);
            __syncwarp();
            const int pn[2] = {(int)(T.nb[ci] + T.nt[ci]), (int)(T.nb[ci + 1] + T.nt[ci + 1])};
            const int pnb[2] = {(int)T.nb[ci], (int)T.nb[ci + 1]};
            const int pbase[2] = {T.base[ci], T.base[ci + 1]};
            unsigned nfs[2];
            place_pair<R>(fc, W, tail, pbase, pn, pnb, Aout, Bout, lane, nfs);
            if (lane == ci) nfs_mine = nfs[0];
            if (lane == ci + 1) nfs_mine = nfs[1];
            const int m = pn[0] + pn[1];
            moved += (unsigned)m;
            __syncwarp();  // every lane is done with the cells' ring slots
            tail += m;
            if (tail >= R) tail -= R;
            used -= m;
            ahead -= 2;
            ci += 2;
            continue;
        }
        cp_async_wait(ahead - 1);
        __syncwarp();

        const int n = min((int)(T.nb[ci] + T.nt[ci]), R);
        const int base = T.base[ci];
        const int sys = T.sys[ci];
        if (sys != tsys) {
            if (lane == 0 && tsys >= 0 && moved) atomicAdd(&P.tally[tsys].particle_steps, (unsigned long long)moved);
            moved = 0;
            tsys = sys;
            fc = flight_const(P.sys[sys]);
        }
        const SysDev &g = P.sys[sys];

        const int nb = min((int)T.nb[ci], n);
        auto ring = [&](int q) {
            const int r = tail + q;
            return r >= R ? r - R : r;
        };
        auto rid = [&](int q) { return __float_as_uint(W.B[ring(q)].w); };
        bool viol = false;
        if (!P.sorted_in)
            for (int q = lane; q + 1 < nb; q += 32) viol |= !(rid(q) < rid(q + 1));
        const bool sorted = !__any_sync(0xffffffffu, viol);
        const unsigned below = (1u << lane) - 1u;

        // Stayers go to the bottom segment in id order, movers to the gap.
        unsigned n_fs;
        if (sorted && n <= 32) {
            n_fs = place_sorted<R, 1>(fc, W, tail, base, n, nb, Aout, Bout, lane);
        } else if (sorted && n <= 64) {
            n_fs = place_sorted<R, 2>(fc, W, tail, base, n, nb, Aout, Bout, lane);
        } else {
            // pass 1: every member's flight; the record goes back into the
            // ring and pref[q] counts the stayers before member q
            unsigned S = 0;
            for (int c0 = 0; c0 < n; c0 += 32) {
                const int q = c0 + lane;
                const bool valid = q < n;
                bool stay = false;
                if (valid) {
                    const int r = ring(q);
                    Particle p;
                    Split32::unpack(W.A[r], W.B[r], p);
                    stay = first_flight(g, p);
                    Split32::pack(p, W.A[r], W.B[r]);
                }
                const unsigned fast = __ballot_sync(0xffffffffu, valid && stay);
                if (valid) W.pref[q] = (uint16_t)(S + (unsigned)__popc(fast & below));
                S += (unsigned)__popc(fast);
            }
            if (lane == 0) W.pref[n] = (uint16_t)S;
            __syncwarp();
            // pass 2: stayers in id order, movers below the top of the gap
            for (int c0 = 0; c0 < n; c0 += 32) {
                const int q = c0 + lane;
                if (q < n) {
                    const int r = ring(q);
                    const uint32_t id = rid(q);
                    unsigned dst;
                    if (W.pref[q + 1] > W.pref[q]) {
                        unsigned pos;
                        if (sorted) {
                            int lb = q;  // bottom members below this id
                            if (q >= nb) {
                                int lo = 0, hi = nb;
                                while (lo < hi) {
                                    const int mid = (lo + hi) >> 1;
                                    if (rid(mid) < id) lo = mid + 1;
                                    else hi = mid;
                                }
                                lb = lo;
                            }
                            pos = W.pref[lb];
                            for (int i = nb; i < n; ++i) pos += (W.pref[i + 1] > W.pref[i]) && rid(i) < id;
                        } else {
                            pos = 0;
                            for (int i = 0; i < n; ++i) pos += (W.pref[i + 1] > W.pref[i]) && rid(i) < id;
                        }
                        dst = (unsigned)base + pos;
                    } else {
                        dst = (unsigned)(base + n) - 1u - ((unsigned)q - W.pref[q]);
                    }
                    Aout[dst] = W.A[r];
                    Bout[dst] = W.B[r];
                }
            }
            n_fs = S;
        }
        if (lane == ci) nfs_mine = n_fs;
        moved += (unsigned)n;
        __syncwarp();  // every lane is done with the cell's ring slots
        tail += n;
        if (tail >= R) tail -= R;
        used -= n;
        --ahead;
        ++ci;
    }
    if (lane == 0 && tsys >= 0 && moved) atomicAdd(&P.tally[tsys].particle_steps, (unsigned long long)moved);
}

template <int R> constexpr size_t move_smem_bytes() { return sizeof(MoveSmem<R>) * M_WARPS; }

// ---- place_movers -----------------------------------------------------------

constexpr int P_WARPS = 4;
constexpr int W_WARPS = 4;
constexpr int WQ = 32;  // wall-flight entries a warp collects before appending them to the list

struct PlaceSmem {
    int2 q[WQ];  // {output slot, system}
    int qn;
};

struct MoveCounts {
    unsigned wall, reseed, stranded, err;
    int cross[3];
};
__device__ __forceinline__ void counts_reset(MoveCounts &c) {
    c.wall = c.reseed = c.stranded = c.err = 0;
    c.cross[0] = c.cross[1] = c.cross[2] = 0;
}
__device__ __forceinline__ void counts_add(MoveCounts &c, const MoveTally &t) {
    c.wall += (unsigned)t.wall_hits;
    c.reseed += (unsigned)t.reseeds;
    c.err |= t.err;
#pragma unroll
    for (int d = 0; d < 3; ++d) c.cross[d] += t.cross[d];
}
// Publishes the counts for system sys: the warp's sum (all lanes call) or,
// per_lane, each lane's own.
__device__ void counts_publish(const PassParams &P, int sys, MoveCounts &c, bool per_lane) {
    unsigned w = c.wall, r = c.reseed, s = c.stranded, e = c.err;
    int x[3] = {c.cross[0], c.cross[1], c.cross[2]};
    if (!per_lane) {
        w = warp_sum(w);
        r = warp_sum(r);
        s = warp_sum(s);
        e = __reduce_or_sync(0xffffffffu, e);
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = warp_sum(x[d]);
    }
    if ((per_lane || (threadIdx.x & 31) == 0) && sys >= 0) {
        SysTally &T = P.tally[sys];
        if (w) atomicAdd(&T.wall_hits, (unsigned long long)w);
        if (r) atomicAdd(&T.reseeds, (unsigned long long)r);
        if (s) atomicAdd(&T.stranded, (unsigned long long)s);
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (x[d]) atomicAdd((unsigned long long *)&T.count_periodic[d], (unsigned long long)(long long)x[d]);
    }
    if ((per_lane || (threadIdx.x & 31) == 0) && e) atomicOr(&P.status->error, e);
    counts_reset(c);
}

// Places one particle per valid lane into a top slot of cell `key`
// (warp-aggregated atomics).  A slot at or below the cell's input occupancy
// could meet its bottom segment or gap: that particle spills instead, and its
// slot is given back so the counter ends at the number placed.
__device__ __forceinline__ void insert_top(const PassParams &P, const Split32::Particle &p, bool valid,
                                           unsigned key, unsigned &err) {
    const int lane = threadIdx.x & 31;
    unsigned *top_out = P.cells.top[P.cout];
    const int2 rt = valid ? P.cells.room[key] : make_int2(0, 0);  // {first slot past the cell, room}
    const unsigned peers = __match_any_sync(0xffffffffu, valid ? key : 0xffffffffu);
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
        if (j < (unsigned)rt.y) {
            const unsigned dst = (unsigned)rt.x - 1u - j;
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
    const unsigned over = __ballot_sync(0xffffffffu, spilled) & peers;
    if (valid && lane == leader && over) atomicSub(&top_out[key], (unsigned)__popc(over));
}

// Where a particle that completed its flight goes: its new active cell; or,
// when it ended inside solid whose cell has no free volume, its source cell
// (the reference aborts there, dsmc/system.h:134-142; the particle's next
// move re-seeds it, dsmc/moleculemover.cpp:57-60); or, in another slab's
// cell, the outgoing list (`leave`).  False only for the outgoing list.
__device__ __forceinline__ bool new_cell(const SysDev &g, const Split32::Particle &p, int src, unsigned &key,
                                         bool &leave, MoveCounts &cnt, unsigned &err) {
    const int ac = __ldg(g.cell_map + Split32::cell_global(g, p));
    leave = ac == DSMC_CELL_FOREIGN;
    if (ac >= 0) {
        key = (unsigned)ac;
    } else if (!leave) {
        err |= DSMC_EBIT_STRANDED;
        ++cnt.stranded;
        key = (unsigned)src;
    }
    return !leave;
}

// Appends the particles of the valid lanes to the outgoing list (one atomic
// per warp).  All lanes call.
__device__ __forceinline__ void leave_slab(const PassParams &P, const Split32::Particle &p, bool valid, unsigned &err) {
    const int lane = threadIdx.x & 31;
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    if (!vm) return;
    unsigned at = 0;
    if (lane == __ffs(vm) - 1) at = atomicAdd(&P.status->nout, (unsigned)__popc(vm));
    at = __shfl_sync(0xffffffffu, at, __ffs(vm) - 1) + (unsigned)__popc(vm & ((1u << lane) - 1u));
    if (valid) {
        if (at < P.parts.out_cap) {
            uint4 ra;
            float4 rb;
            Split32::pack(p, ra, rb);
            P.parts.out[2 * (size_t)at] = ra;
            P.parts.out[2 * (size_t)at + 1] = *reinterpret_cast<const uint4 *>(&rb);
        } else {
            err |= DSMC_EBIT_SPILL_FULL;
        }
    }
}

// Appends the warp's collected wall flights to the list (one atomic per
// batch).  All lanes call.
__device__ __forceinline__ void flush_walls(const PassParams &P, PlaceSmem &W) {
    const int lane = threadIdx.x & 31;
    const int qn = W.qn;
    unsigned at = 0;
    if (lane == 0 && qn) at = atomicAdd(&P.status->walls, (unsigned)qn);
    at = __shfl_sync(0xffffffffu, at, 0);
    if (lane < qn) {
        if (at + lane < P.parts.walls_cap) P.parts.walls[at + lane] = W.q[lane];
        else atomicOr(&P.status->error, DSMC_EBIT_SPILL_FULL);  // cannot happen: one entry per slot at most
    }
    __syncwarp();
    if (lane == 0) W.qn = 0;
    __syncwarp();
}

__global__ void __launch_bounds__(32 * P_WARPS, 5) place_movers_kernel(const __grid_constant__ PassParams P) {
    __shared__ PlaceSmem smem[P_WARPS];
    const int lane = threadIdx.x & 31;
    const volatile Status *vs = P.status;
    if (vs->halted) return;
    PlaceSmem &W = smem[threadIdx.x >> 5];
    if (lane == 0) W.qn = 0;
    __syncwarp();
    const uint4 *Aout = reinterpret_cast<const uint4 *>(P.parts.A[P.cur ^ 1]);
    const float4 *Bout = reinterpret_cast<const float4 *>(P.parts.B[P.cur ^ 1]);

    MoveCounts cnt;
    counts_reset(cnt);
    int tsys = -1;

    const int C = P.cells.num_cells;
    const int nchunks = (C + 31) >> 5;
    for (int ch = blockIdx.x * P_WARPS + (threadIdx.x >> 5); ch < nchunks; ch += gridDim.x * P_WARPS) {
        const int first = ch * 32;
        const bool mine = lane < C - first;
        // lane i: the movers of cell i sit in output slots [gap, gap + cnt)
        int gap = 0, mv = 0, sys = -1;
        if (mine) {
            const int a = first + lane;
            const int4 m = P.cells.meta[a];
            unsigned nb, nt;
            input_counts(P, a, m, nb, nt);
            const unsigned nfs = min(P.cells.bot[P.cout][a], nb + nt);
            gap = m.x + (int)nfs;
            mv = (int)(nb + nt - nfs);
            sys = m.w;
        }
        // exclusive prefix of the mover counts over the chunk's cells
        int incl = mv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        const int pre = mine ? incl - mv : 0x7fffffff;
        for (int f0 = 0; f0 < total; f0 += 32) {
            const int f = f0 + lane;
            const bool valid = f < total;
            // cell of mover f: the last cell whose prefix is <= f
            int c = 0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                const int pc = __shfl_sync(0xffffffffu, pre, (c + s) & 31);
                if (c + s < 32 && pc <= f) c += s;
            }
            const int slot = __shfl_sync(0xffffffffu, gap, c) + (f - __shfl_sync(0xffffffffu, pre, c));
            const int psys = __shfl_sync(0xffffffffu, sys, c);
            const int src = first + c;  // the mover's cell
            const int csys = common_system(valid, psys);
            if (csys != tsys) {
                counts_publish(P, tsys, cnt, false);
                tsys = csys;
            }
            Split32::Particle p;
            MoveTally mt;
            mt.wall_hits = mt.reseeds = 0;
            mt.cross[0] = mt.cross[1] = mt.cross[2] = 0;
            mt.err = 0;
            bool done = false, place = false, leave = false;
            unsigned key = 0;
            if (valid) {
                Split32::unpack(Aout[slot], Bout[slot], p);
                const SysDev &g = P.sys[psys];
                done = Split32::move_open(g, p, mt);
                if (done) place = new_cell(g, p, src, key, leave, cnt, mt.err);
            }
            // flights that meet a wall stay in their slot for place_walls
            const unsigned wall = __ballot_sync(0xffffffffu, valid && !done);
            if (wall) {
                if (W.qn + __popc(wall) > WQ) flush_walls(P, W);
                if (valid && !done) W.q[W.qn + __popc(wall & ((1u << lane) - 1u))] = make_int2(slot, src);
                __syncwarp();
                if (lane == 0) W.qn += __popc(wall);
                __syncwarp();
            }
            insert_top(P, p, place, key, mt.err);
            leave_slab(P, p, leave, mt.err);
            counts_add(cnt, mt);
            if (tsys == -2) counts_publish(P, psys, cnt, true);
        }
    }
    if (W.qn) flush_walls(P, W);
    counts_publish(P, tsys, cnt, false);
}

// The general mover for every listed wall flight, one per thread, then the
// placement.  The last block ends the pass: it advances the step and halts
// the pipeline if anything spilled or failed.
__global__ void __launch_bounds__(32 * W_WARPS) place_walls_kernel(const __grid_constant__ PassParams P) {
    const int lane = threadIdx.x & 31;
    const volatile Status *vs = P.status;
    if (vs->halted) return;
    const uint32_t move_step = vs->step + 1;
    const unsigned nwalls = min(vs->walls, P.parts.walls_cap);
    const uint4 *Aout = reinterpret_cast<const uint4 *>(P.parts.A[P.cur ^ 1]);
    const float4 *Bout = reinterpret_cast<const float4 *>(P.parts.B[P.cur ^ 1]);
    MoveCounts cnt;
    counts_reset(cnt);
    int tsys = -1;
    // warps claim 32 entries at a time: flights differ widely in length, so
    // a warp that finishes early takes more
    for (;;) {
        unsigned i0 = 0;
        if (lane == 0) i0 = atomicAdd(&P.status->walls_taken, 32u);
        i0 = __shfl_sync(0xffffffffu, i0, 0);
        if (i0 >= nwalls) break;
        const unsigned i = i0 + lane;
        const bool valid = i < nwalls;
        const int2 e = valid ? P.parts.walls[i] : make_int2(0, -1);  // {slot, source cell}
        const int esys = valid ? P.cells.meta[e.y].w : -1;
        const int csys = common_system(valid, esys);
        if (csys != tsys) {
            counts_publish(P, tsys, cnt, false);
            tsys = csys;
        }
        Split32::Particle p;
        MoveTally mt;
        mt.wall_hits = mt.reseeds = 0;
        mt.cross[0] = mt.cross[1] = mt.cross[2] = 0;
        mt.err = 0;
        unsigned key = 0;
        bool place = false, leave = false;
        // the lanes of a warp share their system unless it is mixed; a mixed
        // warp moves its lanes one system at a time
        const int s0 = esys;
        if (valid) Split32::unpack(Aout[e.x], Bout[e.x], p);
        for (unsigned todo = __ballot_sync(0xffffffffu, valid); todo;) {
            const int sys = __shfl_sync(0xffffffffu, s0, __ffs(todo) - 1);
            const bool mine = valid && s0 == sys;
            Split32::move_general_warp(P.sys[sys], p, move_step, mt, mine);
            todo &= ~__ballot_sync(0xffffffffu, mine);
        }
        if (valid) place = new_cell(P.sys[esys], p, e.y, key, leave, cnt, mt.err);
        insert_top(P, p, place, key, mt.err);
        leave_slab(P, p, leave, mt.err);
        counts_add(cnt, mt);
        if (tsys == -2) counts_publish(P, esys, cnt, true);
    }
    counts_publish(P, tsys, cnt, false);

    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned done = atomicAdd(&P.status->blocks_done, 1u);
        if (done == gridDim.x - 1) {
            __threadfence();
            if (P.advance_step) atomicAdd(&P.status->step, 1u);
            if (atomicAdd(&P.status->spill, 0u) != 0u || (atomicAdd(&P.status->error, 0u) & DSMC_EBIT_FATAL) != 0u)
                atomicExch(&P.status->halted, 1u);
            atomicExch(&P.status->walls, 0u);
            atomicExch(&P.status->walls_taken, 0u);
            atomicExch(&P.status->collide_taken, 0u);
            atomicExch(&P.status->blocks_done, 0u);
        }
    }
}

// ---- slab exchange ----------------------------------------------------------

// Records that arrive from another slab (the receiving side of the
// reference's mpi_move, dsmc/system.cpp:49-105): each goes into the top
// segment of its cell, above the bottom segment, or into the overflow list
// (the host then repacks).  A record outside this system's cells is an error.
__global__ void put_records_kernel(const SysDev *sys, int s, const CellArrays cells, const ParticleArrays parts,
                                   int cur, int cin, long long n, const uint4 *rec, Status *status) {
    const SysDev &g = sys[s];
    uint4 *A = reinterpret_cast<uint4 *>(parts.A[cur]);
    float4 *B = reinterpret_cast<float4 *>(parts.B[cur]);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint4 ra = rec[2 * i];
        const uint4 rbits = rec[2 * i + 1];
        const float4 rb = *reinterpret_cast<const float4 *>(&rbits);
        Split32::Particle p;
        Split32::unpack(ra, rb, p);
        if (p.c[0] < 0 || p.c[0] >= g.n[0] || p.c[1] >= g.n[1] || p.c[2] >= g.n[2]) {
            atomicOr(&status->error, DSMC_EBIT_CELL);
            continue;
        }
        const int ac = __ldg(g.cell_map + Split32::cell_global(g, p));
        if (ac < 0) {
            atomicOr(&status->error, DSMC_EBIT_CELL);
            continue;
        }
        const int4 m = cells.meta[ac];
        const unsigned nb = min(cells.bot[cin][ac], (unsigned)m.y);
        const unsigned j = atomicAdd(&cells.top[cin][ac], 1u);
        if (nb + j < (unsigned)m.y) {
            const unsigned dst = (unsigned)(m.x + m.y) - 1u - j;
            A[dst] = ra;
            B[dst] = rb;
        } else {
            atomicSub(&cells.top[cin][ac], 1u);
            const unsigned si = atomicAdd(&status->spill, 1u);
            if (si < parts.spill_cap) {
                SpillRec &sr = parts.spill[si];
                sr.a = ra;
                sr.b = rbits;
                sr.cell = ac;
            } else {
                atomicOr(&status->error, DSMC_EBIT_SPILL_FULL);
            }
        }
    }
}

}  // namespace pass3
}  // namespace dsmc
