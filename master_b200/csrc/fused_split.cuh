// The production timestep pass for split-precision state: one kernel per
// step that, for every active cell, collides (NTC) and samples the particles
// the previous step sorted into it, then accelerates, moves and re-bins them
// into the next buffer.  One warp per cell, persistent grid.
//
// Memory pipeline: each warp double-buffers its cells in shared memory.  While
// it works on cell k, the bulk-copy engine (cp.async.bulk, completion on an
// mbarrier) brings cell k+1's particle records in; cell k+2's metadata is
// loaded into registers at the same time.  Every wait on an mbarrier is
// bounded: on expiry the warp records DSMC_EBIT_TIMEOUT, waits (bounded) for
// its copies in flight and leaves the loop.  No cluster multicast is used.
#pragma once
#include "engine.cuh"

namespace dsmc {
namespace fused {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// global -> shared bulk copy into this CTA's own shared memory (16-byte
// aligned addresses, size a multiple of 16; no cluster is involved).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (int i = 0; i < (1 << 22); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

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

constexpr int QCAP = 32;

template <int CAP> struct WarpSmem {
    uint4 A[2][CAP];
    float4 B[2][CAP];
    double4 cs[2];       // cell state {vr_max, rest, coeff, 0}
    int4 meta[2];        // cell metadata {base, cap, global, sys}
    uint64_t bar[2];
    int n[2];
    int qn;
    int pad;
    unsigned wtally[8];  // wall hits, reseeds, crossings x3, stranded, error bits (drained particles)
    SlowRec q[QCAP];
    uint16_t perm[CAP];
};

struct LaneTally {
    unsigned collisions, candidates, wall_hits, reseeds, moved, stranded;
    int cross[3];
    unsigned err;
    int sys;
};

__device__ __forceinline__ void lane_tally_reset(LaneTally &t) {
    t.collisions = t.candidates = t.wall_hits = t.reseeds = t.moved = t.stranded = 0;
    t.cross[0] = t.cross[1] = t.cross[2] = 0;
    t.err = 0;
}

__device__ __forceinline__ unsigned warp_sum_u32(unsigned x) { return __reduce_add_sync(0xffffffffu, x); }

__device__ void flush_lane_tally(const PassParams &P, LaneTally &t, int lane) {
    const unsigned long long col = warp_sum_u32(t.collisions), cand = warp_sum_u32(t.candidates);
    const unsigned long long wh = warp_sum_u32(t.wall_hits), rs = warp_sum_u32(t.reseeds);
    const unsigned long long mv = warp_sum_u32(t.moved), sd = warp_sum_u32(t.stranded);
    int cr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) cr[d] = __reduce_add_sync(0xffffffffu, t.cross[d]);
    const unsigned err = __reduce_or_sync(0xffffffffu, t.err);
    if (lane == 0 && t.sys >= 0) {
        SysTally &T = P.tally[t.sys];
        if (col) atomicAdd(&T.collisions, col);
        if (cand) atomicAdd(&T.candidates, cand);
        if (wh) atomicAdd(&T.wall_hits, wh);
        if (rs) atomicAdd(&T.reseeds, rs);
        if (mv) atomicAdd(&T.particle_steps, mv);
        if (sd) atomicAdd(&T.stranded, sd);
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (cr[d]) atomicAdd((unsigned long long *)&T.count_periodic[d], (unsigned long long)(long long)cr[d]);
        if (err) atomicOr(&P.status->error, err);
    }
    lane_tally_reset(t);
}

// Folds the drained particles' counts (warp shared tally) into lane 0's
// tally and publishes the warp's counts for its current system.
template <int CAP> __device__ void flush_warp(const PassParams &P, WarpSmem<CAP> &W, LaneTally &t, int lane) {
    __syncwarp();
    if (lane == 0) {
        t.wall_hits += W.wtally[0];
        t.reseeds += W.wtally[1];
        t.cross[0] += (int)W.wtally[2];
        t.cross[1] += (int)W.wtally[3];
        t.cross[2] += (int)W.wtally[4];
        t.stranded += W.wtally[5];
        t.err |= W.wtally[6];
    }
    __syncwarp();
    if (lane < 8) W.wtally[lane] = 0;
    __syncwarp();
    flush_lane_tally(P, t, lane);
}

// Output side of a pass: where a moved particle goes.
struct Sink {
    unsigned *cnt_out;
    uint4 *Aout;
    float4 *Bout;
    const int4 *meta;
    Status *status;
    SpillRec *spill;
    unsigned spill_cap;
};

// Places one particle per valid lane into its new cell of the output buffer
// (warp-aggregated counting-sort insert; overflow goes to the spill list).
__device__ __forceinline__ void insert(const Sink &k, const Split32::Particle &p, bool valid, unsigned key, int lane,
                                       int home, const int4 &home_meta, unsigned &err) {
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    unsigned slot0 = 0;
    if (valid && lane == leader) slot0 = atomicAdd(&k.cnt_out[key], (unsigned)__popc(peers));
    slot0 = __shfl_sync(0xffffffffu, slot0, leader);
    if (!valid) return;
    const unsigned slot = slot0 + (unsigned)__popc(peers & ((1u << lane) - 1u));
    uint4 ra;
    float4 rb;
    Split32::pack(p, ra, rb);
    const int4 km = key == (unsigned)home ? home_meta : k.meta[key];
    if (slot < (unsigned)km.y) {
        const unsigned dst = (unsigned)km.x + slot;
        k.Aout[dst] = ra;
        k.Bout[dst] = rb;
    } else {
        const unsigned si = atomicAdd(&k.status->spill, 1u);
        if (si < k.spill_cap) {
            SpillRec &sr = k.spill[si];
            sr.a = ra;
            sr.b = *reinterpret_cast<const uint4 *>(&rb);
            sr.cell = (int)key;
        } else {
            err |= DSMC_EBIT_SPILL_FULL;
        }
    }
}

// Runs the general mover on the queued particles, one per lane, and places
// them; its counts go to the warp's shared tally.  All lanes call.
__device__ __noinline__ void drain_queue(const SysDev *gp, SlowRec *q, int *qn_p, unsigned *wtally, int lane,
                                         uint32_t move_step, Sink k) {
    const SysDev &g = *gp;
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
    insert(k, p, valid, key, lane, -1, make_int4(0, 0, 0, 0), mt.err);
    const unsigned wh = __reduce_add_sync(0xffffffffu, (unsigned)mt.wall_hits);
    const unsigned rs = __reduce_add_sync(0xffffffffu, (unsigned)mt.reseeds);
    const int c0 = __reduce_add_sync(0xffffffffu, mt.cross[0]);
    const int c1 = __reduce_add_sync(0xffffffffu, mt.cross[1]);
    const int c2 = __reduce_add_sync(0xffffffffu, mt.cross[2]);
    const unsigned sd = __reduce_add_sync(0xffffffffu, stranded);
    const unsigned er = __reduce_or_sync(0xffffffffu, mt.err);
    if (lane == 0) {
        wtally[0] += wh;
        wtally[1] += rs;
        wtally[2] += (unsigned)c0;
        wtally[3] += (unsigned)c1;
        wtally[4] += (unsigned)c2;
        wtally[5] += sd;
        wtally[6] |= er;
        *qn_p = 0;
    }
    __syncwarp();
}

// The NTC collide of one staged cell by lane 0 (ranks by the whole warp).
__device__ __noinline__ unsigned collide_cell(uint64_t seed, int cell_global, uint32_t step, int n, int pairs,
                                              double *vr_max, float4 *SB, uint16_t *perm, int lane) {
    for (int q = lane; q < n; q += 32) {
        const uint32_t mine = __float_as_uint(SB[q].w);
        int rank = 0;
        for (int r = 0; r < n; ++r) rank += __float_as_uint(SB[r].w) < mine;
        perm[rank] = (uint16_t)q;
    }
    __syncwarp();
    unsigned long long col = 0;
    if (lane == 0) {
        SmemVel vel;
        vel.b = SB;
        ntc_run<float>(seed, cell_global, step, n, pairs, *vr_max, vel, perm, col);
    }
    __syncwarp();
    return (unsigned)col;
}

template <int CAP>
__global__ void __launch_bounds__(256, 3) fused_split_kernel(PassParams P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    typedef Split32::Particle Particle;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warps_per_block = blockDim.x >> 5;
    const volatile Status *vs = P.status;
    if (vs->halted) return;
    const uint32_t step = vs->step;
    const uint32_t move_step = step + 1;

    WarpSmem<CAP> &W = reinterpret_cast<WarpSmem<CAP> *>(smem_raw)[wib];
    if (lane == 0) {
        mbar_init(&W.bar[0]);
        mbar_init(&W.bar[1]);
        W.qn = 0;
        fence_mbar_init();
    }
    __syncwarp();

    const uint4 *Ain = reinterpret_cast<const uint4 *>(P.parts.A[P.cur]);
    const float4 *Bin = reinterpret_cast<const float4 *>(P.parts.B[P.cur]);
    unsigned *cnt_in = P.cells.count[P.cur];
    Sink sink;
    sink.cnt_out = P.cells.count[P.cur ^ 1];
    sink.Aout = reinterpret_cast<uint4 *>(P.parts.A[P.cur ^ 1]);
    sink.Bout = reinterpret_cast<float4 *>(P.parts.B[P.cur ^ 1]);
    sink.meta = P.cells.meta;
    sink.status = P.status;
    sink.spill = P.parts.spill;
    sink.spill_cap = P.parts.spill_cap;
    if (lane < 8) W.wtally[lane] = 0;

    LaneTally t;
    lane_tally_reset(t);
    t.sys = -1;

    const int C = P.cells.num_cells;
    const int stride = gridDim.x * warps_per_block;
    int a = blockIdx.x * warps_per_block + wib;

    // Lane 0 stages a cell: metadata into shared memory, then one bulk copy
    // each of its records and its fp64 state.
    int4 m_pf = make_int4(0, 0, 0, 0);  // lane 0: metadata of the cell to issue next
    unsigned n_pf = 0;
    auto load_meta = [&](int cell) {
        if (lane == 0 && cell < C) {
            m_pf = P.cells.meta[cell];
            n_pf = min(min(cnt_in[cell], (unsigned)m_pf.y), (unsigned)CAP);
        }
    };
    auto issue = [&](int stage, int cell) {
        fence_proxy_async();
        W.meta[stage] = m_pf;
        W.n[stage] = (int)n_pf;
        const uint32_t bytes = n_pf * 16u;
        const void *srcA = Ain + m_pf.x, *srcB = Bin + m_pf.x, *srcS = P.cells.state + cell;
        // every operand is 16-byte aligned by construction; a violation is
        // recorded and the transfer skipped rather than issued
        if (!aligned16(srcA) || !aligned16(srcB) || !aligned16(srcS) || !aligned16(&W.A[stage][0]) ||
            !aligned16(&W.B[stage][0]) || !aligned16(&W.cs[stage])) {
            atomicOr(&P.status->error, DSMC_EBIT_ALIGN);
            W.n[stage] = 0;
            mbar_arrive_expect(&W.bar[stage], 0u);
            return;
        }
        mbar_arrive_expect(&W.bar[stage], 2u * bytes + (uint32_t)sizeof(double4));
        bulk_g2s(&W.cs[stage], srcS, (uint32_t)sizeof(double4), &W.bar[stage]);
        if (n_pf) {
            bulk_g2s(&W.A[stage][0], srcA, bytes, &W.bar[stage]);
            bulk_g2s(&W.B[stage][0], srcB, bytes, &W.bar[stage]);
        }
    };
    load_meta(a);
    if (lane == 0 && a < C) issue(0, a);
    load_meta(a + stride);

    uint32_t parity = 0;
    bool ok = true;
    for (int k = 0; a < C; a += stride, ++k) {
        const int s = k & 1;
        const int a_nxt = a + stride;
        if (lane == 0 && a_nxt < C) issue(s ^ 1, a_nxt);
        load_meta(a_nxt + stride);

        if (!mbar_wait(&W.bar[s], (parity >> s) & 1u)) {
            ok = false;
            break;
        }
        parity ^= 1u << s;
        __syncwarp();
        const int4 m = W.meta[s];
        const int n = W.n[s];
        const int sys = m.w;
        if (sys != t.sys) {
            if (W.qn) drain_queue(P.sys + t.sys, W.q, &W.qn, W.wtally, lane, move_step, sink);
            if (t.sys >= 0) flush_warp(P, W, t, lane);
            t.sys = sys;
        }
        const SysDev &g = P.sys[sys];
        uint4 *SA = W.A[s];
        float4 *SB = W.B[s];

        // ---- collide: Cell::prepare + Cell::collide (dsmc/cell.cpp:42-111)
        if (P.do_collide) {
            int pairs = 0;
            if (lane == 0) {
                double4 &cs = W.cs[s];
                pairs = ntc_select(cs.z, n, cs.x, cs.y);
                if (n < 2) pairs = 0;
            }
            pairs = __shfl_sync(0xffffffffu, pairs, 0);
            if (pairs > 0) {
                const unsigned col = collide_cell(g.seed, m.z, step, n, pairs, &W.cs[s].x, SB, W.perm, lane);
                if (lane == 0) {
                    t.collisions += col;
                    t.candidates += (unsigned)pairs;
                }
            }
            if (lane == 0) P.cells.state[a] = W.cs[s];
        }

        // ---- sample: cell moments in fp64 on the reference's cadence
        if (P.do_sample && g.sample_interval > 0 && step > 0 && (step % (uint32_t)g.sample_interval) == 0 &&
            step >= (uint32_t)g.sample_begin) {
            double m1[3] = {0, 0, 0}, m2[3] = {0, 0, 0};
            for (int q = lane; q < n; q += 32) {
                const float4 b = SB[q];
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
        if (lane == 0) cnt_in[a] = 0;

        // ---- accelerate + move; particles that stay in their voxel are
        // placed at once, the rest queue for the general mover
        for (int ch = 0; ch * 32 < n; ++ch) {
            const int q = ch * 32 + lane;
            const bool valid = q < n;
            Particle p;
            bool stay = false;
            if (valid) {
                Split32::unpack(SA[q], SB[q], p);
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
                t.moved += 1;
            }
            const unsigned slow = __ballot_sync(0xffffffffu, valid && !stay);
            if (slow) {
                if (W.qn + __popc(slow) > QCAP) drain_queue(&g, W.q, &W.qn, W.wtally, lane, move_step, sink);
                if (valid && !stay) {
                    SlowRec &r = W.q[W.qn + __popc(slow & ((1u << lane) - 1u))];
                    Split32::pack(p, r.a, r.b);
                    r.cell = a;
                    r.global = m.z;
                }
                __syncwarp();
                if (lane == 0) W.qn += __popc(slow);
                __syncwarp();
            }
            const bool place = valid && stay;
            insert(sink, p, place, place ? (unsigned)a : 0xffffffffu, lane, a, m, t.err);
        }
        __syncwarp();
    }
    if (!ok) {
        if (lane == 0) atomicOr(&P.status->error, DSMC_EBIT_TIMEOUT);
        mbar_wait(&W.bar[0], parity & 1u);
        mbar_wait(&W.bar[1], (parity >> 1) & 1u);
    } else if (W.qn) {
        drain_queue(P.sys + t.sys, W.q, &W.qn, W.wtally, lane, move_step, sink);
    }
    if (t.sys >= 0) flush_warp(P, W, t, lane);

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

template <int CAP> size_t fused_smem_bytes(int warps) { return sizeof(WarpSmem<CAP>) * warps; }

}  // namespace fused
}  // namespace dsmc
