// C ABI of libdsmc_b200: context, systems, particle I/O and the timestep
// pipeline.  Host code only; the kernels are in kernels_split.cu and
// kernels_fp64.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "dsmc_b200.h"
#include "dsmc_internal.h"
#include "dsmc_layout.h"
#include "kernels.h"

namespace dsmc {

template <class T> struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
    cudaError_t ensure(size_t count) { return count <= n && p ? cudaSuccess : alloc(count); }
    // ensure with 1/16 headroom on growth, so that capacities that drift up
    // between repacks do not reallocate every time
    cudaError_t ensure_grow(size_t count) { return count <= n && p ? cudaSuccess : alloc(count + count / 16); }
};

struct SysHost {
    dsmc_settings settings;
    int n[3], cells[3];
    float porosity_global, porosity;
    double volume, atoms_per_molecule;
    int64_t expected;
    int64_t num_particles = 0;
    uint32_t id_count = 0;  // ids handed out: 0 .. id_count-1
    int active_begin = 0, active_end = 0;
    std::vector<int> cell_global;     // per active cell
    std::vector<int> pixels, total_pixels;
    double pixel_sum = 0;             // free voxels over the active cells
    std::vector<double> volume_cell, coeff;
    std::vector<int> cell_map;        // global -> local active index
    DevBuf<uint8_t> vox;
    DevBuf<float> nrm, t1, t2;
    DevBuf<int> cell_map_dev;         // global -> absolute active index
    SysDev dev;
    double t0_reduced = 0;            // time of the last tally reset
    double t_offset = 0;              // t - step * dt after a continuation
    double sqrt_t_over_m = 0;
    double vr_max0 = 0;
    double volume_global = 0;         // L_x L_y L_z * porosity_global (dsmc/system.cpp:314)
    int prof_bins = 0, prof_copies = 1;
    DevBuf<double> prof;              // sampler profiles: copies of {3*bins y-binned sums, v_x histogram}
    size_t prof_len() const { return (size_t)prof_copies * 4 * (size_t)prof_bins; }
    // the copies added up: the 4*bins sums
    cudaError_t prof_sums(std::vector<double> &out, cudaStream_t st) const {
        std::vector<double> all(prof_len());
        cudaError_t e = cudaMemcpyAsync(all.data(), prof.p, all.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        out.assign(4 * (size_t)prof_bins, 0.0);
        for (int c = 0; c < prof_copies; ++c)
            for (size_t i = 0; i < out.size(); ++i) out[i] += all[(size_t)c * out.size() + i];
        return e;
    }
    bool slab = false;                // owns only the cells with x index in [slab_x0, slab_x1)
    int slab_x0 = 0, slab_x1 = 0;
};

}  // namespace dsmc

using namespace dsmc;

struct dsmc_ctx {
    int device = 0;
    int precision = DSMC_PREC_SPLIT32;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    Units units;
    std::vector<std::unique_ptr<SysHost>> systems;

    // device tables
    DevBuf<SysDev> sys_dev;
    DevBuf<SysTally> tally;
    DevBuf<Status> status;
    // cells (all systems)
    int num_cells = 0;
    DevBuf<int4> meta;
    DevBuf<double4> state;
    DevBuf<unsigned> bot[3], top[3], key;  // occupancy sets, rotating per re-binning pass
    DevBuf<int2> room;                      // per cell: top-slot room of the pass in flight
    DevBuf<double> mom;
    DevBuf<int> pix;                 // per cell: free voxels (the capacity's expected share)
    DevBuf<double2> cap_np;          // per system: {particles, free voxels} at the last layout
    DevBuf<unsigned long long> cap_bsum, cap_out;  // layout scan: block sums; {total slots, largest capacity}
    size_t slots = 0;
    int smem_cap = 32;
    // particles
    DevBuf<unsigned char> A0, A1, B0, B1;
    DevBuf<SpillRec> spill;
    unsigned spill_cap = 1u << 16;
    DevBuf<int2> walls;       // wall-flight list of the production pass (one entry per slot at most)
    DevBuf<uint4> out;        // outgoing list of a slab: particles that ended in another slab's cell
    unsigned out_cap = 0;
    bool slab = false;        // the context holds a slab system (its only system)
    int cur = 0;
    int cphase = 0;           // occupancy set the next pass reads
    bool sorted = false;      // every bottom segment is sorted by id (a production pass ran last)
    bool pending = false;     // the last step's collide/sample has not run yet
    bool keys_valid = false;  // a stand-alone move stage left new cell keys
    // the device step counter as the last settle read it, while no pass and
    // no host write has touched it since (dsmc_step then skips its read)
    bool step_known = false;
    unsigned known_step = 0;
    // staging
    DevBuf<unsigned char> fA, fB;
    DevBuf<int> fkey;
    DevBuf<unsigned> hist;
    DevBuf<unsigned long long> cursor;
    DevBuf<double> io_r, io_v;
    DevBuf<int> io_cell;
    DevBuf<double> cell_energy;  // dsmc_tallies_get: per-cell kinetic-energy sums
    // launch shape of the cell pass
    int block = 256;
    int grid = 0;
    int fused_grids[5] = {0, 0, 0, 0, 0};  // production pass (collide, move, place, walls, sample); 0 = not usable
    int fused_max_bps[5] = {0, 0, 0, 0, 0};  // the most resident blocks per SM of each at the current ring
    // launch tuning (dsmc_tuning_set): blocks per SM of each production
    // kernel (0: the most resident), move_cells ring, collide chunk claims
    int tune_bps[5] = {0, 0, 0, 0, 0};
    int tune_ring = 0;
    int tune_claim = 0;
    bool use_pipelined = true;
    // per-kernel timers of the production pass (dsmc_ctx_set_timing)
    bool timing = false;
    cudaEvent_t tev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // dsmc_particles_get: positions are copied out on io_stream while the
    // velocities are converted on `stream`
    cudaStream_t io_stream = nullptr;
    cudaEvent_t io_event = nullptr;
    double tms[4] = {0, 0, 0, 0};
    long long tpasses = 0;
    double cap_factor = 2.0;
    int cap_pad = 24;
    // The production pass as CUDA graphs, one per pass configuration (buffer
    // parity, occupancy set, sorted bottoms, collide, sample); every buffer
    // pointer is baked into the graphs, so any (re)allocation drops them.
    bool use_graphs = true;
    std::map<int, cudaGraphExec_t> graphs;
    void drop_graphs() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }

    size_t rec_half() const { return precision == DSMC_PREC_FP64 ? 32 : 16; }
};

namespace {

int fail(dsmc_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->error = msg;
    else set_thread_error(msg);
    return code;
}

int cuda_fail(dsmc_ctx *ctx, cudaError_t e, const char *what) {
    return fail(ctx, DSMC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                  \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);  \
    } while (0)

bool is_fp64(const dsmc_ctx *ctx) { return ctx->precision == DSMC_PREC_FP64; }

CellArrays cell_arrays(dsmc_ctx *ctx) {
    CellArrays c;
    c.num_cells = ctx->num_cells;
    c.meta = ctx->meta.p;
    c.state = ctx->state.p;
    for (int q = 0; q < 3; ++q) {
        c.bot[q] = ctx->bot[q].p;
        c.top[q] = ctx->top[q].p;
    }
    c.mom = ctx->mom.p;
    c.key = ctx->key.p;
    c.room = ctx->room.p;
    return c;
}

ParticleArrays particle_arrays(dsmc_ctx *ctx) {
    ParticleArrays p;
    p.A[0] = ctx->A0.p;
    p.A[1] = ctx->A1.p;
    p.B[0] = ctx->B0.p;
    p.B[1] = ctx->B1.p;
    p.spill = ctx->spill.p;
    p.spill_cap = ctx->spill_cap;
    p.walls = ctx->walls.p;
    p.walls_cap = (unsigned)std::min<size_t>(ctx->slots, 0xffffffffu);
    p.out = ctx->out.p;
    p.out_cap = ctx->out.p ? ctx->out_cap : 0u;
    return p;
}

int upload_sys_table(dsmc_ctx *ctx) {
    ctx->drop_graphs();  // the table may move
    std::vector<SysDev> t;
    for (auto &s : ctx->systems) t.push_back(s->dev);
    CK(ctx->sys_dev.ensure(std::max<size_t>(t.size(), 1)));
    if (!t.empty())
        CK(cudaMemcpyAsync(ctx->sys_dev.p, t.data(), t.size() * sizeof(SysDev), cudaMemcpyHostToDevice, ctx->stream));
    return DSMC_OK;
}

Status read_status(dsmc_ctx *ctx, cudaError_t *err) {
    Status st;
    std::memset(&st, 0, sizeof(st));
    *err = cudaMemcpyAsync(&st, ctx->status.p, sizeof(Status), cudaMemcpyDeviceToHost, ctx->stream);
    if (*err == cudaSuccess) *err = cudaStreamSynchronize(ctx->stream);
    return st;
}

// Rebuilds every cell table and slot buffer from flat staged particles.
// fA/fB/fkey hold `total` records; hist holds per-cell counts.
// Grids of the production pass: the most resident blocks per SM of each
// kernel, or the tuned count when one is set (never above the most).
void apply_launch_shape(dsmc_ctx *ctx) {
    for (int &gsz : ctx->fused_grids) gsz = 0;
    for (int &b : ctx->fused_max_bps) b = 0;
    if (is_fp64(ctx) || split32::fused_capacity(ctx->smem_cap) <= 0) return;
    if (!split32::fused_grids(ctx->smem_cap, ctx->num_sms, ctx->fused_grids, ctx->tune_ring, ctx->fused_max_bps)) {
        for (int &gsz : ctx->fused_grids) gsz = 0;
        return;
    }
    for (int k = 0; k < 5; ++k)
        if (ctx->tune_bps[k] > 0)
            ctx->fused_grids[k] = std::min(ctx->tune_bps[k], ctx->fused_max_bps[k]) * ctx->num_sms;
}

int relayout(dsmc_ctx *ctx, long long total) {
    ctx->drop_graphs();  // slot buffers and grids may change
    const int C = ctx->num_cells;
    // Capacity per cell: twice the larger of the expected and the present
    // occupancy plus 24 slots by default (Poisson tails beyond it are below
    // 1e-12 per cell and step; an overflow spills and the host repacks).
    // Computed on the device with the cells' first slots (cell_layout.cu).
    const size_t S = std::max<size_t>(ctx->systems.size(), 1);
    std::vector<double2> np(S, double2{0.0, 0.0});
    for (size_t q = 0; q < ctx->systems.size(); ++q)
        np[q] = double2{(double)ctx->systems[q]->num_particles, ctx->systems[q]->pixel_sum};
    CK(ctx->cap_np.ensure(S));
    CK(ctx->cap_bsum.ensure(std::max(cell_layout_blocks(C), 1)));
    CK(ctx->cap_out.ensure(2));
    CK(cudaMemcpyAsync(ctx->cap_np.p, np.data(), S * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_cell_layout(ctx->meta.p, ctx->pix.p, ctx->hist.p, ctx->cap_np.p, ctx->cap_factor, (double)ctx->cap_pad, C,
                          ctx->cap_bsum.p, ctx->cap_out.p, ctx->stream));
    unsigned long long lay[2] = {0, 0};
    CK(cudaMemcpyAsync(lay, ctx->cap_out.p, sizeof(lay), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const size_t slots = (size_t)lay[0];
    const unsigned maxcap = (unsigned)std::max<unsigned long long>(4, lay[1]);
    if (slots >= (size_t)0x7fffffffu) return fail(ctx, DSMC_ERR_CAPACITY, "more than 2^31 particle slots");
    if (maxcap > 4096) return fail(ctx, DSMC_ERR_CAPACITY, "a cell needs more than 4096 slots");
    ctx->smem_cap = (int)((maxcap + 31u) & ~31u);
    ctx->slots = slots;
    const size_t half = ctx->rec_half();
    CK(ctx->A0.ensure_grow(slots * half));
    CK(ctx->A1.ensure_grow(slots * half));
    CK(ctx->B0.ensure_grow(slots * half));
    CK(ctx->B1.ensure_grow(slots * half));
    CK(ctx->key.ensure_grow(slots));
    CK(ctx->walls.ensure_grow(std::max<size_t>(slots, 1)));
    if (C) {
        for (int q = 0; q < 3; ++q) {
            CK(cudaMemsetAsync(ctx->bot[q].p, 0, C * sizeof(unsigned), ctx->stream));
            CK(cudaMemsetAsync(ctx->top[q].p, 0, C * sizeof(unsigned), ctx->stream));
        }
    }
    ctx->cur = 0;
    ctx->cphase = 0;
    ctx->sorted = false;  // the repack inserts in arrival order
    CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(unsigned) * 2, ctx->stream));  // error, spill
    unsigned zero = 0;
    CK(cudaMemcpyAsync(&ctx->status.p->halted, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    if (total > 0) {
        cudaError_t e = is_fp64(ctx)
                            ? fp64::launch_insert(cell_arrays(ctx), particle_arrays(ctx), 0, 0, total, ctx->fA.p,
                                                  ctx->fB.p, ctx->fkey.p, &ctx->status.p->error, ctx->stream)
                            : split32::launch_insert(cell_arrays(ctx), particle_arrays(ctx), 0, 0, total, ctx->fA.p,
                                                     ctx->fB.p, ctx->fkey.p, &ctx->status.p->error, ctx->stream);
        CK(e);
    }
    // Launch shape of the cell pass: a persistent grid at full occupancy.
    const int bps = is_fp64(ctx) ? fp64::pass_blocks_per_sm(PASS_FUSED, ctx->block, ctx->smem_cap)
                                 : split32::pass_blocks_per_sm(PASS_FUSED, ctx->block, ctx->smem_cap);
    if (bps <= 0) return fail(ctx, DSMC_ERR_CUDA, "cell pass cannot be resident (shared memory)");
    const int bps_in = is_fp64(ctx) ? fp64::pass_blocks_per_sm(PASS_INPLACE, ctx->block, ctx->smem_cap)
                                    : split32::pass_blocks_per_sm(PASS_INPLACE, ctx->block, ctx->smem_cap);
    const int bps_so = is_fp64(ctx) ? fp64::pass_blocks_per_sm(PASS_SORT, ctx->block, ctx->smem_cap)
                                    : split32::pass_blocks_per_sm(PASS_SORT, ctx->block, ctx->smem_cap);
    if (bps_in <= 0 || bps_so <= 0) return fail(ctx, DSMC_ERR_CUDA, "stage passes cannot be resident (shared memory)");
    ctx->grid = bps * ctx->num_sms;
    apply_launch_shape(ctx);
    Status st;
    cudaError_t e;
    st = read_status(ctx, &e);
    CK(e);
    if (st.error & DSMC_EBIT_FATAL) return fail(ctx, DSMC_ERR_STATE, "particles could not be placed in cells");
    return DSMC_OK;
}

// Stages every present particle (all systems, or all but `skip`) into fA/fB.
// Every particle of the systems not marked in `skip` (skip.empty(): all)
// into the staging buffer, sized for `extra` more records.
static int stage_present_set(dsmc_ctx *ctx, long long extra, const std::vector<char> &skip, long long *staged) {
    auto skipped = [&](size_t s) { return s < skip.size() && skip[s]; };
    long long present = 0;
    for (size_t s = 0; s < ctx->systems.size(); ++s)
        if (!skipped(s)) present += ctx->systems[s]->num_particles;
    Status st;
    cudaError_t e;
    st = read_status(ctx, &e);
    CK(e);
    const long long total = present + st.spill + extra;
    const size_t half = ctx->rec_half();
    CK(ctx->fA.ensure(std::max<long long>(total, 1) * half));
    CK(ctx->fB.ensure(std::max<long long>(total, 1) * half));
    CK(ctx->fkey.ensure(std::max<long long>(total, 1)));
    CK(ctx->hist.ensure(std::max(ctx->num_cells, 1)));
    CK(ctx->cursor.ensure(1));
    CK(cudaMemsetAsync(ctx->hist.p, 0, std::max(ctx->num_cells, 1) * sizeof(unsigned), ctx->stream));
    CK(cudaMemsetAsync(ctx->cursor.p, 0, sizeof(unsigned long long), ctx->stream));
    *staged = 0;
    if (ctx->A0.p && ctx->num_cells) {
        for (size_t s = 0; s < ctx->systems.size(); ++s) {
            if (skipped(s)) continue;
            SysHost &h = *ctx->systems[s];
            if (h.active_end <= h.active_begin) continue;
            e = is_fp64(ctx) ? fp64::launch_gather(cell_arrays(ctx), particle_arrays(ctx), ctx->cur, ctx->cphase,
                                                   h.active_begin,
                                                   h.active_end, std::min(st.spill, ctx->spill_cap), ctx->fA.p,
                                                   ctx->fB.p, ctx->fkey.p, ctx->hist.p, ctx->cursor.p,
                                                   (unsigned long long)total, &ctx->status.p->error, ctx->stream)
                             : split32::launch_gather(cell_arrays(ctx), particle_arrays(ctx), ctx->cur, ctx->cphase,
                                                      h.active_begin, h.active_end, std::min(st.spill, ctx->spill_cap),
                                                      ctx->fA.p, ctx->fB.p, ctx->fkey.p, ctx->hist.p, ctx->cursor.p,
                                                      (unsigned long long)total, &ctx->status.p->error, ctx->stream);
            CK(e);
        }
        unsigned long long got = 0;
        CK(cudaMemcpyAsync(&got, ctx->cursor.p, sizeof(got), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        *staged = (long long)got;
    }
    return DSMC_OK;
}

int stage_present(dsmc_ctx *ctx, long long extra, int skip, long long *staged) {
    std::vector<char> set;
    if (skip >= 0 && skip < (int)ctx->systems.size()) {
        set.assign(ctx->systems.size(), 0);
        set[skip] = 1;
    }
    return stage_present_set(ctx, extra, set, staged);
}

// Runs the collide + sample of the last step if it is still pending.
int flush_pending(dsmc_ctx *ctx);

// One production pass from its cached graph, captured on first use.
cudaError_t launch_fused_graph(dsmc_ctx *ctx, const PassParams &P) {
    const int key = P.cur | (P.cin << 1) | (P.sorted_in << 3) | (P.do_collide << 4) | (P.do_sample << 5) |
                    (P.do_move << 6);
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        const cudaError_t el = split32::launch_fused(P, ctx->fused_grids, ctx->stream, nullptr);
        e = cudaStreamEndCapture(ctx->stream, &g);
        if (el != cudaSuccess || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return el != cudaSuccess ? el : e;
        }
        cudaGraphExec_t x = nullptr;
        e = cudaGraphInstantiate(&x, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return e;
        it = ctx->graphs.emplace(key, x).first;
    }
    return cudaGraphLaunch(it->second, ctx->stream);
}

PassParams pass_params(dsmc_ctx *ctx, int do_collide, int do_move, int do_sample, int advance) {
    PassParams P;
    P.sys = ctx->sys_dev.p;
    P.tally = ctx->tally.p;
    P.status = ctx->status.p;
    P.cells = cell_arrays(ctx);
    P.parts = particle_arrays(ctx);
    P.cur = ctx->cur;
    P.cin = ctx->cphase;
    P.sorted_in = ctx->sorted ? 1 : 0;
    P.cout = (ctx->cphase + 1) % 3;
    P.cclear = (ctx->cphase + 2) % 3;
    P.do_collide = do_collide;
    P.do_move = do_move;
    P.do_sample = do_sample;
    P.smem_cap = ctx->smem_cap;
    P.advance_step = advance;
    P.ring = ctx->tune_ring;
    P.claim = ctx->tune_claim;
    return P;
}

int launch(dsmc_ctx *ctx, int mode, int do_collide, int do_move, int do_sample, int advance) {
    ctx->step_known = false;
    PassParams P = pass_params(ctx, do_collide, do_move, do_sample, advance);
    cudaError_t e;
    if (mode == PASS_FUSED && ctx->use_pipelined && ctx->fused_grids[1] > 0) {
        P.top_only = 0;
        ctx->sorted = true;  // move_cells leaves every bottom segment sorted
        if (ctx->use_graphs && !ctx->timing && advance) {
            e = launch_fused_graph(ctx, P);
            if (e != cudaSuccess) {  // capture refused: plain launches from here on
                cudaGetLastError();
                ctx->drop_graphs();
                ctx->use_graphs = false;
                e = split32::launch_fused(P, ctx->fused_grids, ctx->stream, nullptr);
            }
        } else {
            e = split32::launch_fused(P, ctx->fused_grids, ctx->stream, ctx->timing ? ctx->tev : nullptr);
        }
        if (e == cudaSuccess && ctx->timing) {
            CK(cudaEventSynchronize(ctx->tev[4]));
            for (int k = 0; k < 4; ++k) {
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, ctx->tev[k], ctx->tev[k + 1]));
                ctx->tms[k] += ms;
            }
            ++ctx->tpasses;
        }
    } else {
        P.top_only = 1;
        if (mode != PASS_INPLACE) ctx->sorted = false;  // the generic passes fill top segments only
        e = is_fp64(ctx) ? fp64::launch_pass(mode, P, ctx->grid, ctx->block, ctx->stream)
                         : split32::launch_pass(mode, P, ctx->grid, ctx->block, ctx->stream);
    }
    CK(e);
    // a re-binning pass rotates the occupancy sets
    if (mode != PASS_INPLACE) ctx->cphase = (ctx->cphase + 1) % 3;
    return DSMC_OK;
}

// Whether the collide of a pass that sees step counter `step` samples any
// system (the cadence of StatisticsSampler::sample; the kernels check it again
// per system).
bool samples_at(const dsmc_ctx *ctx, unsigned step) {
    for (const auto &s : ctx->systems) {
        const SysDev &d = s->dev;
        if (d.sample_interval > 0 && step > 0 && step % (unsigned)d.sample_interval == 0 &&
            step >= (unsigned)d.sample_begin)
            return true;
    }
    return false;
}

// After a batch of passes: find how many ran, fix the buffer parity, and
// repack if one of them spilled.
int settle(dsmc_ctx *ctx, unsigned step_before, int cur_before, int cphase_before, int *ran) {
    cudaError_t e;
    Status st = read_status(ctx, &e);
    CK(e);
    *ran = (int)(st.step - step_before);
    ctx->cur = cur_before ^ (*ran & 1);
    ctx->cphase = (cphase_before + *ran) % 3;
    if (st.error & DSMC_EBIT_FATAL) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "device error bits 0x%x after step %u (1 cell, 4 reseed, 8 spill list, 16 "
                      "staging, 32 non-finite)", st.error, st.step);
        return fail(ctx, DSMC_ERR_STATE, buf);
    }
    if (st.halted && st.spill) {
        long long staged = 0;
        int rc = stage_present(ctx, 0, -1, &staged);
        if (rc) return rc;
        rc = relayout(ctx, staged);  // leaves the step counter as it is
        if (rc) return rc;
    }
    ctx->step_known = true;
    ctx->known_step = st.step;
    return DSMC_OK;
}

int flush_pending(dsmc_ctx *ctx) {
    if (!ctx->pending) return DSMC_OK;
    if (!is_fp64(ctx) && ctx->use_pipelined && ctx->fused_grids[1] > 0) {
        // the production pass's own collide (and, on a sampled step, sampler)
        // kernels, in place: the pending step is the device's step counter
        cudaError_t e;
        const Status st = read_status(ctx, &e);
        CK(e);
        PassParams P = pass_params(ctx, 1, 0, samples_at(ctx, st.step) ? 1 : 0, 0);
        P.top_only = 0;
        CK(split32::launch_collide(P, ctx->fused_grids, ctx->stream));
    } else {
        int rc = launch(ctx, PASS_INPLACE, 1, 0, 1, 0);
        if (rc) return rc;
    }
    ctx->pending = false;
    return DSMC_OK;
}

// Grows b to hold `need` elements (at least doubling, so that n appends cost
// O(n) copies in all), keeping its first `keep` elements.
template <class T> static cudaError_t grow_keep(DevBuf<T> &b, size_t need, size_t keep, cudaStream_t st) {
    if (b.p && need <= b.n) return cudaSuccess;
    const size_t cap = std::max<size_t>(std::max<size_t>(need, 2 * b.n), 1);
    T *p = nullptr;
    cudaError_t e = cudaMalloc(&p, cap * sizeof(T));
    if (e != cudaSuccess) return e;
    if (keep && b.p) {
        e = cudaMemcpyAsync(p, b.p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the copy is done before the old buffer goes
    }
    if (e != cudaSuccess) {
        cudaFree(p);
        return e;
    }
    b.release();
    b.p = p;
    b.n = cap;
    return cudaSuccess;
}

// Appends the cells of the context's last system (just added) after those of
// the systems before it, which keep their cell indices, cell state, moment
// sums, tallies and device cell maps: systems are only ever appended, so
// only the new system's cells are built on the host and uploaded (adding n
// systems one by one costs O(total cells), not O(n * total cells)).
// Occupancy sets are cleared for every cell; the caller re-lays the
// particles out.
int rebuild_cells(dsmc_ctx *ctx) {
    ctx->drop_graphs();
    const int C_old = ctx->num_cells;
    const int si = (int)ctx->systems.size() - 1;
    SysHost &s = *ctx->systems[si];
    const int nc = (int)s.cell_global.size();
    const int C = C_old + nc;
    const size_t Cn = std::max(C, 1);
    CK(grow_keep(ctx->meta, Cn, C_old, ctx->stream));
    CK(grow_keep(ctx->pix, Cn, C_old, ctx->stream));
    CK(grow_keep(ctx->state, Cn, C_old, ctx->stream));
    CK(grow_keep(ctx->mom, 8 * Cn, 8 * (size_t)C_old, ctx->stream));
    for (int q = 0; q < 3; ++q) {
        CK(grow_keep(ctx->bot[q], Cn, 0, ctx->stream));
        CK(grow_keep(ctx->top[q], Cn, 0, ctx->stream));
    }
    CK(grow_keep(ctx->room, Cn, 0, ctx->stream));
    CK(grow_keep(ctx->hist, Cn, 0, ctx->stream));
    CK(grow_keep(ctx->tally, std::max<size_t>(ctx->systems.size(), 1), (size_t)si, ctx->stream));
    CK(cudaMemsetAsync(ctx->tally.p + si, 0, sizeof(SysTally), ctx->stream));
    // the new system's cells
    s.active_begin = C_old;
    s.active_end = C;
    s.pixel_sum = 0;
    std::vector<int4> h_meta(std::max(nc, 1), int4{0, 0, 0, 0});  // {base, cap: set by each layout; global, sys}
    std::vector<int> pix(std::max(nc, 1));
    std::vector<double4> state(std::max(nc, 1));
    for (int c = 0; c < nc; ++c) {
        h_meta[c].z = s.cell_global[c];
        h_meta[c].w = si;
        pix[c] = s.pixels[c];
        s.pixel_sum += s.pixels[c];
        // Cell::vr_max starts at 3*sqrt(T) (dsmc/system.cpp:451,477)
        state[c] = double4{s.vr_max0, 0.0, s.coeff[c], 0.0};
    }
    s.dev.active_begin = s.active_begin;
    s.dev.active_end = s.active_end;
    std::vector<int> map_abs(s.cell_map.size());
    for (size_t g = 0; g < s.cell_map.size(); ++g)
        map_abs[g] = s.cell_map[g] < 0 ? s.cell_map[g] : s.cell_map[g] + s.active_begin;
    CK(s.cell_map_dev.ensure(map_abs.size()));
    CK(cudaMemcpyAsync(s.cell_map_dev.p, map_abs.data(), map_abs.size() * sizeof(int), cudaMemcpyHostToDevice,
                       ctx->stream));
    s.dev.cell_map = s.cell_map_dev.p;
    ctx->num_cells = C;
    if (nc) {
        CK(cudaMemcpyAsync(ctx->meta.p + C_old, h_meta.data(), nc * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->pix.p + C_old, pix.data(), nc * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->state.p + C_old, state.data(), nc * sizeof(double4), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(cudaMemsetAsync(ctx->mom.p + 8 * (size_t)C_old, 0, 8 * (size_t)nc * sizeof(double), ctx->stream));
    }
    if (C)
        for (int q = 0; q < 3; ++q) {
            CK(cudaMemsetAsync(ctx->bot[q].p, 0, C * sizeof(unsigned), ctx->stream));
            CK(cudaMemsetAsync(ctx->top[q].p, 0, C * sizeof(unsigned), ctx->stream));
        }
    CK(cudaStreamSynchronize(ctx->stream));  // the host vectors above are released on return
    return upload_sys_table(ctx);
}

}  // namespace

extern "C" {

const char *dsmc_last_error(const dsmc_ctx *ctx) { return ctx ? ctx->error.c_str() : thread_error(); }

int dsmc_ctx_create(int device_id, int precision, dsmc_ctx **out) {
    if (!out || (precision != DSMC_PREC_SPLIT32 && precision != DSMC_PREC_FP64)) return DSMC_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(nullptr, DSMC_ERR_NO_DEVICE, "no CUDA device");
    if (device_id < 0 || device_id >= ndev) return fail(nullptr, DSMC_ERR_ARG, "device id out of range");
    e = cudaSetDevice(device_id);
    if (e != cudaSuccess) return fail(nullptr, DSMC_ERR_CUDA, cudaGetErrorString(e));
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device_id);
    if (prop.major != 10) return fail(nullptr, DSMC_ERR_NO_DEVICE, "kernels are built for sm_100a (B200) only");
    std::unique_ptr<dsmc_ctx> ctx(new dsmc_ctx);
    ctx->device = device_id;
    ctx->precision = precision;
    ctx->num_sms = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(nullptr, DSMC_ERR_CUDA, cudaGetErrorString(e));
    if (ctx->status.alloc(1) != cudaSuccess) return fail(nullptr, DSMC_ERR_CUDA, "status alloc");
    cudaMemset(ctx->status.p, 0, sizeof(Status));
    if (ctx->spill.alloc(ctx->spill_cap) != cudaSuccess) return fail(nullptr, DSMC_ERR_CUDA, "spill alloc");
    if (ctx->tally.alloc(1) != cudaSuccess) return fail(nullptr, DSMC_ERR_CUDA, "tally alloc");
    cudaMemset(ctx->tally.p, 0, sizeof(SysTally));
    *out = ctx.release();
    return DSMC_OK;
}

void dsmc_ctx_destroy(dsmc_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->drop_graphs();
    for (cudaEvent_t &e : ctx->tev)
        if (e) cudaEventDestroy(e);
    if (ctx->io_event) cudaEventDestroy(ctx->io_event);
    if (ctx->io_stream) cudaStreamDestroy(ctx->io_stream);
    cudaStream_t s = ctx->stream;
    delete ctx;
    cudaStreamDestroy(s);
}

int dsmc_sync(dsmc_ctx *ctx) {
    if (!ctx) return DSMC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    return DSMC_OK;
}

// A system over the whole geometry, or (cx1 >= 0) an x-slab that owns the
// active cells with cell x index in [cx0, cx1).
static int system_add(dsmc_ctx *ctx, const dsmc_settings *s, uint32_t nx, uint32_t ny, uint32_t nz,
                      const uint8_t *voxels, const float *normals, const float *tangents1, const float *tangents2,
                      float porosity_global, int cx0, int cx1, int *sys_id) {
    if (!ctx || !s || !voxels || !normals || !tangents1 || !tangents2 || !sys_id) return DSMC_ERR_ARG;
    const bool slab = cx1 >= 0;
    if (ctx->slab) return fail(ctx, DSMC_ERR_CONFIG, "a slab is its context's only system");
    if (slab) {
        if (!ctx->systems.empty()) return fail(ctx, DSMC_ERR_CONFIG, "a slab is its context's only system");
        if (is_fp64(ctx)) return fail(ctx, DSMC_ERR_CONFIG, "slabs run in split precision");
        if (cx0 < 0 || cx0 >= cx1 || cx1 > s->cells_x)
            return fail(ctx, DSMC_ERR_CONFIG, "slab cell range must satisfy 0 <= x0 < x1 <= cells_x");
    }
    cudaSetDevice(ctx->device);
    if (nx == 0 || ny == 0 || nz == 0 || nx > 2048 || ny > 2048 || nz > 1024)
        return fail(ctx, DSMC_ERR_CAPACITY, "voxel grid limited to 2048 x 2048 x 1024");
    if (s->cells_x <= 0 || s->cells_y <= 0 || s->cells_z <= 0) return fail(ctx, DSMC_ERR_CONFIG, "cells must be > 0");
    if (s->nx != 1 || s->ny != 1 || s->nz != 1)
        return fail(ctx, DSMC_ERR_CONFIG, "one system is one domain: processor grid must be 1 1 1");
    if (s->surface_model < DSMC_WALL_THERMAL || s->surface_model > DSMC_WALL_CL)
        return fail(ctx, DSMC_ERR_CONFIG, "unknown wall model");
    if (s->sampling_bins < 1 || s->sampling_bins > (1 << 20))
        return fail(ctx, DSMC_ERR_CONFIG, "sampling_bins must be in 1 .. 2^20");
    if (s->surface_model == DSMC_WALL_CL && !(s->alpha_n > 0 && s->alpha_n <= 1 && s->alpha_t >= 0 && s->alpha_t <= 1))
        return fail(ctx, DSMC_ERR_CONFIG, "Cercignani-Lampis accommodation needs 0 < alpha_n <= 1, 0 <= alpha_t <= 1");
    // System::validate_number_of_cells (dsmc/system.cpp:221-239).
    if (nx % s->cells_x || ny % s->cells_y || nz % s->cells_z)
        return fail(ctx, DSMC_ERR_CONFIG, "Error: voxel-cell-cpu configuration not good.");
    // Settle pending work and stage the particles already present.
    int rc = flush_pending(ctx);
    if (rc) return rc;
    long long staged = 0;
    rc = stage_present(ctx, 0, -1, &staged);
    if (rc) return rc;

    std::unique_ptr<SysHost> h(new SysHost);
    h->settings = *s;
    h->n[0] = nx;
    h->n[1] = ny;
    h->n[2] = nz;
    h->cells[0] = s->cells_x;
    h->cells[1] = s->cells_y;
    h->cells[2] = s->cells_z;
    const uint64_t V = (uint64_t)nx * ny * nz;
    uint64_t empty = 0;
    for (uint64_t i = 0; i < V; ++i) empty += voxels[i] == DSMC_VOX_EMPTY;
    h->porosity = (float)empty / (float)V;
    h->porosity_global = porosity_global > 0 ? porosity_global : (float)((double)empty / V);
    const Units &u = ctx->units;
    const double L[3] = {s->Lx, s->Ly, s->Lz};
    // System::initialize (dsmc/system.cpp:241-382).
    const double temperature = u.temperature_from_SI(s->temperature);
    const double wall_temperature = u.temperature_from_SI(s->wall_temperature);
    const double density = u.number_density_from_SI(s->density);
    h->atoms_per_molecule = s->atoms_per_molecule;
    h->vr_max0 = 3 * std::sqrt(temperature);
    h->sqrt_t_over_m = std::sqrt(temperature / s->mass);
    double volume = L[0] * L[1] * L[2];
    volume = volume / 1 * h->porosity;
    h->volume = volume;
    h->volume_global = L[0] * L[1] * L[2] * h->porosity_global;
    h->expected = (int64_t)(density * volume / h->atoms_per_molecule);
    {
        int nc = 0;
        int rc2 = dsmc_cells_layout(s, nx, ny, nz, voxels, 0, nullptr, nullptr, nullptr, nullptr, nullptr, &nc);
        if (rc2) return fail(ctx, rc2, thread_error());
        h->cell_global.resize(nc);
        h->pixels.resize(nc);
        h->total_pixels.resize(nc);
        h->volume_cell.resize(nc);
        h->coeff.resize(nc);
        rc2 = dsmc_cells_layout(s, nx, ny, nz, voxels, nc, h->cell_global.data(), h->pixels.data(),
                                h->total_pixels.data(), h->volume_cell.data(), h->coeff.data(), &nc);
        if (rc2) return fail(ctx, rc2, thread_error());
        h->cell_map.assign(s->cells_x * s->cells_y * s->cells_z, DSMC_CELL_SOLID);
        if (slab) {
            // keep the slab's cells; the other active cells are foreign
            const int yz = s->cells_y * s->cells_z;
            int k = 0;
            for (int c = 0; c < nc; ++c) {
                const int cg = h->cell_global[c], x = cg / yz;
                if (x < cx0 || x >= cx1) {
                    h->cell_map[cg] = DSMC_CELL_FOREIGN;
                    continue;
                }
                h->cell_global[k] = cg;
                h->pixels[k] = h->pixels[c];
                h->total_pixels[k] = h->total_pixels[c];
                h->volume_cell[k] = h->volume_cell[c];
                h->coeff[k] = h->coeff[c];
                ++k;
            }
            nc = k;
            h->cell_global.resize(nc);
            h->pixels.resize(nc);
            h->total_pixels.resize(nc);
            h->volume_cell.resize(nc);
            h->coeff.resize(nc);
            h->slab = true;
            h->slab_x0 = cx0;
            h->slab_x1 = cx1;
        }
        for (int c = 0; c < nc; ++c) h->cell_map[h->cell_global[c]] = c;
    }
    // Device geometry.
    CK(h->vox.alloc(V));
    CK(h->nrm.alloc(3 * V));
    CK(h->t1.alloc(3 * V));
    CK(h->t2.alloc(3 * V));
    CK(cudaMemcpyAsync(h->vox.p, voxels, V, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(h->nrm.p, normals, 3 * V * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(h->t1.p, tangents1, 3 * V * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(h->t2.p, tangents2, 3 * V * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    SysDev &d = h->dev;
    std::memset(&d, 0, sizeof(d));
    for (int a = 0; a < 3; ++a) {
        d.n[a] = h->n[a];
        d.cells[a] = h->cells[a];
        d.vpc[a] = h->n[a] / h->cells[a];
        d.inv_vpc[a] = 1.0f / d.vpc[a];
        d.L[a] = L[a];
        d.invL[a] = 1.0 / L[a];
        d.vox_len[a] = L[a] / h->n[a];
        // Grid constants (dsmc/grid.cpp:41-46): float-rounded, one rank.
        d.ref_scale[a] = (double)(float)(d.invL[a] * h->n[a]);
        d.ref_shift[a] = (double)(float)(-0.0 * d.invL[a] * h->n[a] + (double)h->n[a]);
        d.inv_vox_f[a] = (float)(h->n[a] / L[a]);
        d.L_f[a] = (float)L[a];
    }
    d.vox = h->vox.p;
    d.nrm = h->nrm.p;
    d.t1 = h->t1.p;
    d.t2 = h->t2.p;
    d.dt = s->dt;
    d.dt_f = (float)s->dt;
    d.flow_dir = (s->flow_direction < 0 || s->flow_direction > 2 || s->gravity == 0) ? -1 : s->flow_direction;
    d.accel_dt = s->gravity * s->dt;
    d.accel_dt_f = (float)d.accel_dt;
    d.wall_s = std::sqrt(wall_temperature / s->mass);
    d.wall_s_f = (float)d.wall_s;
    d.wall_model = s->surface_model;
    d.alpha_t = s->alpha_t;
    d.sqrt_1m_an = std::sqrt(1 - s->alpha_n);
    d.sqrt_1m_an_over_an = std::sqrt(1 - s->alpha_n) / s->alpha_n;
    d.sqrt_an_over_2 = std::sqrt(s->alpha_n / 2);
    d.cl_vmax = 1500.0 / ctx->units.v0;  // UnitConverter::velocity_from_SI(1500)
    d.alpha_t_f = (float)d.alpha_t;
    d.sqrt_1m_an_f = (float)d.sqrt_1m_an;
    d.sqrt_1m_an_over_an_f = (float)d.sqrt_1m_an_over_an;
    d.sqrt_an_over_2_f = (float)d.sqrt_an_over_2;
    d.cl_vmax_f = (float)d.cl_vmax;
    d.seed = s->rng_seed;
    d.sample_interval = s->statistics_interval;
    d.sample_begin = s->sample_begin;
    // Sampler profiles (dsmc/statisticssampler.cpp:22-26): sampling_bins bins
    // in y, and a v_x histogram over [-4 sigma, 4 sigma], sigma = sqrt(T/m).
    // Up to 64 copies, 16 MB at most, so that a sample's atomics spread.
    h->prof_bins = s->sampling_bins;
    h->prof_copies = (int)std::max<size_t>(1, std::min<size_t>(64, ((size_t)1 << 21) / (4 * (size_t)h->prof_bins)));
    CK(h->prof.alloc(h->prof_len()));
    CK(cudaMemsetAsync(h->prof.p, 0, h->prof_len() * sizeof(double), ctx->stream));
    d.prof = h->prof.p;
    d.prof_bins = h->prof_bins;
    d.prof_copies = h->prof_copies;
    d.mass = s->mass;
    {
        const double sd = std::sqrt(temperature / s->mass);
        d.vx_min = -4 * sd;
        d.vx_bin = (4 * sd - d.vx_min) / h->prof_bins;
        d.vx_inv_bin = 1.0 / d.vx_bin;
    }

    if (slab) {
        // outgoing records: a quarter of the geometry's particles at most
        // per step (an overflow is reported, never written past the end)
        ctx->out_cap = (unsigned)std::min<int64_t>(std::max<int64_t>(h->expected / 4, 1 << 16), 1 << 28);
        CK(ctx->out.alloc(2 * (size_t)ctx->out_cap));
        ctx->slab = true;
    }
    ctx->systems.push_back(std::move(h));
    *sys_id = (int)ctx->systems.size() - 1;
    // The staged keys index the old cell numbering; rebuild with the new
    // system appended at the end, so earlier systems keep their cell ids.
    rc = rebuild_cells(ctx);
    if (rc) return rc;
    CK(ctx->hist.ensure(std::max(ctx->num_cells, 1)));
    CK(cudaMemsetAsync(ctx->hist.p, 0, std::max(ctx->num_cells, 1) * sizeof(unsigned), ctx->stream));
    if (staged > 0) {
        // recount the staged keys into the new histogram
        std::vector<int> keys(staged);
        CK(cudaMemcpyAsync(keys.data(), ctx->fkey.p, staged * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        std::vector<unsigned> hc(ctx->num_cells, 0);
        for (int k : keys)
            if (k >= 0) hc[k]++;
        CK(cudaMemcpyAsync(ctx->hist.p, hc.data(), hc.size() * sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    }
    return relayout(ctx, staged);
}

int dsmc_system_add(dsmc_ctx *ctx, const dsmc_settings *s, uint32_t nx, uint32_t ny, uint32_t nz,
                    const uint8_t *voxels, const float *normals, const float *tangents1, const float *tangents2,
                    float porosity_global, int *sys_id) {
    return system_add(ctx, s, nx, ny, nz, voxels, normals, tangents1, tangents2, porosity_global, 0, -1, sys_id);
}

int dsmc_system_add_slab(dsmc_ctx *ctx, const dsmc_settings *s, uint32_t nx, uint32_t ny, uint32_t nz,
                         const uint8_t *voxels, const float *normals, const float *tangents1, const float *tangents2,
                         float porosity_global, int cell_x0, int cell_x1, int *sys_id) {
    if (cell_x1 < 0) return DSMC_ERR_ARG;
    return system_add(ctx, s, nx, ny, nz, voxels, normals, tangents1, tangents2, porosity_global, cell_x0, cell_x1,
                      sys_id);
}

int dsmc_cells_layout(const dsmc_settings *s, uint32_t nx, uint32_t ny, uint32_t nz, const uint8_t *voxels, int cap,
                      int32_t *global_index, int32_t *pixels, int32_t *total_pixels, double *volume, double *coeff,
                      int *num_cells) {
    if (!s || !voxels || !num_cells || nx == 0 || ny == 0 || nz == 0) return DSMC_ERR_ARG;
    const int cx = s->cells_x, cy = s->cells_y, cz = s->cells_z;
    if (cx <= 0 || cy <= 0 || cz <= 0) return fail(nullptr, DSMC_ERR_CONFIG, "cells must be > 0");
    // System::setup_cells (dsmc/system.cpp:432-490): cells numbered in order of
    // first touch by a k-outer, i-inner voxel sweep; cells with no empty voxel
    // are dropped.
    const int ncells = cx * cy * cz;
    std::vector<int> first(ncells, -1), tot, pix, order;
    for (uint32_t k = 0; k < nz; ++k) {
        const int c_z = (int)((float)k / nz * cz);
        for (uint32_t j = 0; j < ny; ++j) {
            const int c_y = (int)((float)j / ny * cy);
            for (uint32_t i = 0; i < nx; ++i) {
                const int c_x = (int)((float)i / nx * cx);
                const int ci = c_x * cy * cz + c_y * cz + c_z;
                if (first[ci] < 0) {
                    first[ci] = (int)order.size();
                    order.push_back(ci);
                    tot.push_back(0);
                    pix.push_back(0);
                }
                tot[first[ci]]++;
                pix[first[ci]] += voxels[((uint64_t)i * ny + j) * nz + k] < DSMC_VOX_WALL;
            }
        }
    }
    const double system_volume = s->Lx * s->Ly * s->Lz;
    const double apm = s->atoms_per_molecule;
    int n = 0;
    for (size_t c = 0; c < order.size(); ++c) {
        if (pix[c] == 0) continue;
        if (n < cap) {
            // Cell::update_volume (dsmc/cell.cpp:27-40)
            const double vol = system_volume / (ncells) * (float)pix[c] / tot[c];
            if (global_index) global_index[n] = order[c];
            if (pixels) pixels[n] = pix[c];
            if (total_pixels) total_pixels[n] = tot[c];
            if (volume) volume[n] = vol;
            if (coeff) coeff[n] = 0.5 * apm * M_PI * s->diam * s->diam * s->dt / vol;
        }
        ++n;
    }
    *num_cells = n;
    return DSMC_OK;
}

int dsmc_system_add_world(dsmc_ctx *ctx, const dsmc_settings *s, int *sys_id) {
    if (!ctx || !s) return DSMC_ERR_ARG;
    char path[600];
    std::snprintf(path, sizeof(path), "%s/%04d.bin", s->world, 0);
    dsmc_world_header hd;
    int rc = dsmc_world_read_header(path, &hd);
    if (rc) return fail(ctx, rc, thread_error());
    const uint64_t V = (uint64_t)hd.global_nx * hd.global_ny * hd.global_nz;
    std::vector<uint8_t> vox(V);
    std::vector<float> n(3 * V), a(3 * V), b(3 * V);
    rc = dsmc_world_read(path, vox.data(), n.data(), a.data(), b.data());
    if (rc) return fail(ctx, rc, thread_error());
    return dsmc_system_add(ctx, s, hd.global_nx, hd.global_ny, hd.global_nz, vox.data(), n.data(), a.data(), b.data(),
                           hd.porosity_global, sys_id);
}

int dsmc_system_info_get(dsmc_ctx *ctx, int sys_id, dsmc_system_info *info) {
    if (!ctx || !info || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    SysHost &h = *ctx->systems[sys_id];
    info->num_particles = h.num_particles;
    info->num_cells_total = h.cells[0] * h.cells[1] * h.cells[2];
    info->num_active_cells = (int)h.cell_global.size();
    info->volume = h.volume;
    info->volume_global = h.volume_global;
    info->porosity = h.porosity;
    info->atoms_per_molecule = h.atoms_per_molecule;
    info->dt = h.settings.dt;
    info->expected_particles = h.expected;
    info->slots = (int)ctx->slots;
    return DSMC_OK;
}

static int place_particles(dsmc_ctx *ctx, int sys_id, long long n, const double *r, const double *v) {
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    long long staged = 0;
    rc = stage_present(ctx, n, sys_id, &staged);
    if (rc) return rc;
    SysHost &h = *ctx->systems[sys_id];
    const size_t half = ctx->rec_half();
    unsigned char *A = ctx->fA.p + staged * half;
    unsigned char *B = ctx->fB.p + staged * half;
    int *key = ctx->fkey.p + staged;
    cudaError_t e;
    if (r) {
        CK(ctx->io_r.ensure(3 * std::max<long long>(n, 1)));
        CK(ctx->io_v.ensure(3 * std::max<long long>(n, 1)));
        if (n) {
            CK(cudaMemcpyAsync(ctx->io_r.p, r, 3 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaMemcpyAsync(ctx->io_v.p, v, 3 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            e = is_fp64(ctx) ? fp64::launch_from_fp64(ctx->sys_dev.p, sys_id, ctx->io_r.p, ctx->io_v.p, 0, n, A, B, key,
                                                      ctx->hist.p, &ctx->status.p->error, ctx->stream)
                             : split32::launch_from_fp64(ctx->sys_dev.p, sys_id, ctx->io_r.p, ctx->io_v.p, 0, n, A, B,
                                                         key, ctx->hist.p, &ctx->status.p->error, ctx->stream);
            CK(e);
        }
    } else if (n) {
        e = is_fp64(ctx) ? fp64::launch_init(ctx->sys_dev.p, sys_id, h.sqrt_t_over_m, n, A, B, key, ctx->hist.p,
                                             &ctx->status.p->error, ctx->stream)
                         : split32::launch_init(ctx->sys_dev.p, sys_id, h.sqrt_t_over_m, n, A, B, key, ctx->hist.p,
                                                &ctx->status.p->error, ctx->stream);
        CK(e);
    }
    Status st = read_status(ctx, &e);
    CK(e);
    if (st.error & DSMC_EBIT_FATAL) {
        cudaMemsetAsync(ctx->status.p, 0, sizeof(unsigned), ctx->stream);
        return fail(ctx, DSMC_ERR_STATE, (st.error & DSMC_EBIT_NAN)
                                             ? "a particle has a non-finite position or velocity"
                                             : "a particle lies in a solid voxel or a cell with no free volume");
    }
    h.num_particles = n;
    h.id_count = (uint32_t)n;
    if (h.slab) {
        // the slab keeps the particles in its own cells (ids are the global indices)
        const int C = h.active_end - h.active_begin;
        std::vector<unsigned> counts(std::max(C, 1), 0u);
        if (C)
            CK(cudaMemcpyAsync(counts.data(), ctx->hist.p + h.active_begin, C * sizeof(unsigned),
                               cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        long long kept = 0;
        for (int c = 0; c < C; ++c) kept += counts[c];
        h.num_particles = kept;
        if (h.settings.max_molecules_per_node > 0 && kept > h.settings.max_molecules_per_node)
            return fail(ctx, DSMC_ERR_CAPACITY, "the slab holds more than max_molecules_per_node particles");
    }
    return relayout(ctx, staged + n);
}

int dsmc_particles_set(dsmc_ctx *ctx, int sys_id, int64_t n, const double *r, const double *v) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size() || n < 0 || (n && (!r || !v))) return DSMC_ERR_ARG;
    if (n > 0xffffffffLL) return fail(ctx, DSMC_ERR_CAPACITY, "at most 2^32 particles per system");
    return place_particles(ctx, sys_id, n, r, v);
}

int dsmc_particles_init(dsmc_ctx *ctx, int sys_id, int64_t n) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    SysHost &h = *ctx->systems[sys_id];
    if (n < 0) n = h.expected;
    if (n > h.settings.max_molecules_per_node && h.settings.max_molecules_per_node > 0 && !h.slab) {
        char buf[200];
        std::snprintf(buf, sizeof(buf), "Node 0 wants to create %lld molecules (MAX_MOLECULE_NUM=%d)", (long long)n,
                      h.settings.max_molecules_per_node);
        return fail(ctx, DSMC_ERR_CAPACITY, buf);
    }
    return place_particles(ctx, sys_id, n, nullptr, nullptr);
}

// One system of a batched initialisation: its count and, for a warm start,
// its per-voxel field (weight null: System::setup_molecules' uniform
// Maxwellian at rest, dsmc/system.cpp:398-430).
struct InitItem {
    int sys;
    long long n;
    const float *weight, *drift;
};

// The weights of system h's empty voxels (host copy of a host or device
// field) and their sum; the weights of non-empty voxels are ignored.
static int field_weights(dsmc_ctx *ctx, const SysHost &h, const float *weight, int device, std::vector<float> &w,
                         std::vector<uint8_t> &vox) {
    const long long V = (long long)h.n[0] * h.n[1] * h.n[2];
    w.resize(V);
    vox.resize(V);
    if (device) {
        CK(cudaMemcpy(w.data(), weight, V * sizeof(float), cudaMemcpyDeviceToHost));
    } else {
        std::memcpy(w.data(), weight, V * sizeof(float));
    }
    CK(cudaMemcpy(vox.data(), h.vox.p, V, cudaMemcpyDeviceToHost));
    for (long long i = 0; i < V; ++i) {
        const float x = w[i];
        if (!(vox[i] == DSMC_VOX_EMPTY && std::isfinite(x) && x > 0.0f)) w[i] = 0.0f;
    }
    return DSMC_OK;
}

// Replaces the particles of every listed system (distinct, not slabs) by
// freshly drawn ones: one staging of the other systems' particles, the
// draws of each listed system appended in list order, one re-layout.  A
// system's particles depend only on its seed, count and field (one
// counter-based stream per particle id), so the result is that of one call
// per system, without re-laying the whole context out once per system.
static int init_systems(dsmc_ctx *ctx, const std::vector<InitItem> &items, int device) {
    cudaSetDevice(ctx->device);
    std::vector<char> set(ctx->systems.size(), 0);
    long long extra = 0;
    bool any_field = false;
    std::vector<float> w;
    std::vector<uint8_t> vox;
    for (const InitItem &it : items) {
        set[it.sys] = 1;
        extra += it.n;
        if (!it.weight) continue;
        any_field = true;
        // every field is checked before anything is staged
        int rc = field_weights(ctx, *ctx->systems[it.sys], it.weight, device, w, vox);
        if (rc) return rc;
        double total = 0.0;
        for (float x : w) total += (double)x;
        if (!(total > 0.0)) return fail(ctx, DSMC_ERR_STATE, "the weight field is zero in every empty voxel");
    }
    int rc = flush_pending(ctx);
    if (rc) return rc;
    long long staged = 0;
    rc = stage_present_set(ctx, extra, set, &staged);
    if (rc) return rc;
    const size_t half = ctx->rec_half();
    long long at = staged;
    DevBuf<double> dcdf;
    DevBuf<float> ddrift;
    std::vector<double> cdf;
    for (const InitItem &it : items) {
        SysHost &h = *ctx->systems[it.sys];
        unsigned char *A = ctx->fA.p + at * half, *B = ctx->fB.p + at * half;
        int *key = ctx->fkey.p + at;
        cudaError_t e = cudaSuccess;
        if (!it.weight) {
            if (it.n)
                e = is_fp64(ctx) ? fp64::launch_init(ctx->sys_dev.p, it.sys, h.sqrt_t_over_m, it.n, A, B, key,
                                                     ctx->hist.p, &ctx->status.p->error, ctx->stream)
                                 : split32::launch_init(ctx->sys_dev.p, it.sys, h.sqrt_t_over_m, it.n, A, B, key,
                                                        ctx->hist.p, &ctx->status.p->error, ctx->stream);
        } else {
            rc = field_weights(ctx, h, it.weight, device, w, vox);
            if (rc) return rc;
            const long long V = (long long)w.size();
            cdf.resize(V + 1);
            cdf[0] = 0.0;
            for (long long i = 0; i < V; ++i) cdf[i + 1] = cdf[i] + (double)w[i];
            // the host buffers may be reused once an upload from pageable
            // memory returns; the device buffers once the stream has reached
            // the next upload, which follows this system's draws
            CK(dcdf.ensure(V + 1));
            CK(cudaMemcpyAsync(dcdf.p, cdf.data(), (V + 1) * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            const float *drift_dev = it.drift;
            if (!device) {
                CK(ddrift.ensure(3 * V));
                CK(cudaMemcpyAsync(ddrift.p, it.drift, 3 * V * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
                drift_dev = ddrift.p;
            }
            if (it.n)
                e = is_fp64(ctx) ? fp64::launch_init_field(ctx->sys_dev.p, it.sys, h.sqrt_t_over_m, it.n, dcdf.p,
                                                           drift_dev, V, A, B, key, ctx->hist.p,
                                                           &ctx->status.p->error, ctx->stream)
                                 : split32::launch_init_field(ctx->sys_dev.p, it.sys, h.sqrt_t_over_m, it.n, dcdf.p,
                                                              drift_dev, V, A, B, key, ctx->hist.p,
                                                              &ctx->status.p->error, ctx->stream);
        }
        CK(e);
        at += it.n;
    }
    cudaError_t e;
    Status st = read_status(ctx, &e);
    CK(e);
    if (st.error & DSMC_EBIT_FATAL) {
        cudaMemsetAsync(ctx->status.p, 0, sizeof(unsigned), ctx->stream);
        return fail(ctx, DSMC_ERR_STATE,
                    (st.error & DSMC_EBIT_NAN) ? (any_field ? "a drift is not finite" : "a velocity is not finite")
                                               : "a particle landed in a solid voxel or a cell with no free volume");
    }
    for (const InitItem &it : items) {
        SysHost &h = *ctx->systems[it.sys];
        h.num_particles = it.n;
        h.id_count = (uint32_t)it.n;
    }
    return relayout(ctx, at);
}

// The listed systems as InitItems: distinct, not slabs, n < 0 (or no n) the
// reference's count, at most 2^32 particles each.
static int init_items(dsmc_ctx *ctx, int count, const int *sys_ids, const int64_t *n, const float *const *weights,
                      const float *const *drifts, std::vector<InitItem> &items) {
    if (count < 0 || (count && !sys_ids)) return DSMC_ERR_ARG;
    std::vector<char> seen(ctx->systems.size(), 0);
    items.clear();
    for (int i = 0; i < count; ++i) {
        const int s = sys_ids[i];
        if (s < 0 || s >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
        if (seen[s]) return fail(ctx, DSMC_ERR_ARG, "a system is listed twice");
        seen[s] = 1;
        SysHost &h = *ctx->systems[s];
        if (h.slab) return fail(ctx, DSMC_ERR_CONFIG, "a slab is initialised by dsmc_particles_init or _set");
        long long k = n && n[i] >= 0 ? (long long)n[i] : h.expected;
        if (k > 0xffffffffLL) return fail(ctx, DSMC_ERR_CAPACITY, "at most 2^32 particles per system");
        InitItem it{s, k, nullptr, nullptr};
        if (weights) {
            if (!drifts || !weights[i] || !drifts[i]) return DSMC_ERR_ARG;
            it.weight = weights[i];
            it.drift = drifts[i];
        } else if (h.settings.max_molecules_per_node > 0 && k > h.settings.max_molecules_per_node) {
            char buf[200];
            std::snprintf(buf, sizeof(buf), "Node 0 wants to create %lld molecules (MAX_MOLECULE_NUM=%d)", k,
                          h.settings.max_molecules_per_node);
            return fail(ctx, DSMC_ERR_CAPACITY, buf);
        }
        items.push_back(it);
    }
    return DSMC_OK;
}

int dsmc_particles_init_many(dsmc_ctx *ctx, int count, const int *sys_ids, const int64_t *n) {
    if (!ctx) return DSMC_ERR_ARG;
    std::vector<InitItem> items;
    int rc = init_items(ctx, count, sys_ids, n, nullptr, nullptr, items);
    if (rc) return rc;
    return items.empty() ? DSMC_OK : init_systems(ctx, items, 0);
}

// Warm start: n particles drawn from a per-voxel weight and drift field
// instead of System::setup_molecules' uniform Maxwellian at rest
// (dsmc/system.cpp:398-430).  The weights of non-empty voxels are ignored.
int dsmc_particles_init_field(dsmc_ctx *ctx, int sys_id, int64_t n, const float *weight, const float *drift,
                              int device) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size() || !weight || !drift) return DSMC_ERR_ARG;
    return dsmc_particles_init_field_many(ctx, 1, &sys_id, &n, &weight, &drift, device);
}

int dsmc_particles_init_field_many(dsmc_ctx *ctx, int count, const int *sys_ids, const int64_t *n,
                                   const float *const *weights, const float *const *drifts, int device) {
    if (!ctx || (count > 0 && (!weights || !drifts))) return DSMC_ERR_ARG;
    std::vector<InitItem> items;
    int rc = init_items(ctx, count, sys_ids, n, weights, drifts, items);
    if (rc) return rc;
    return items.empty() ? DSMC_OK : init_systems(ctx, items, device);
}

// Per-voxel sums {count, sum vx, sum vy, sum vz} of a system's particles added
// to field (4 floats per voxel in the voxel order of the geometry).
int dsmc_field_accumulate(dsmc_ctx *ctx, int sys_id, float *field, int device) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size() || !field) return DSMC_ERR_ARG;
    if (((uintptr_t)field & 15u) != 0) return fail(ctx, DSMC_ERR_ARG, "the field must be 16-byte aligned");
    SysHost &h = *ctx->systems[sys_id];
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    const long long V = (long long)h.n[0] * h.n[1] * h.n[2];
    DevBuf<float> tmp;
    float *f = field;
    if (!device) {
        CK(tmp.ensure(4 * V));
        CK(cudaMemcpyAsync(tmp.p, field, 4 * V * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        f = tmp.p;
    }
    if (h.active_end > h.active_begin) {
        const cudaError_t e =
            is_fp64(ctx) ? fp64::launch_field_accumulate(ctx->sys_dev.p, sys_id, cell_arrays(ctx), particle_arrays(ctx),
                                                         ctx->cur, ctx->cphase, reinterpret_cast<float4 *>(f),
                                                         ctx->stream)
                         : split32::launch_field_accumulate(ctx->sys_dev.p, sys_id, cell_arrays(ctx),
                                                            particle_arrays(ctx), ctx->cur, ctx->cphase,
                                                            reinterpret_cast<float4 *>(f), ctx->stream);
        CK(e);
    }
    if (!device) {
        CK(cudaMemcpyAsync(field, tmp.p, 4 * V * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return DSMC_OK;
}

// main.cpp:37-55: t, steps, collisions and wall collisions carried over from
// an earlier run; the flux window restarts at t (system.t0 = t).
int dsmc_continue_from(dsmc_ctx *ctx, int sys_id, double t, uint64_t steps, uint64_t collisions,
                       uint64_t wall_collisions) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    if (steps > 0xffffffffULL) return fail(ctx, DSMC_ERR_CAPACITY, "the step counter holds 32 bits");
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    SysHost &h = *ctx->systems[sys_id];
    SysTally T;
    CK(cudaMemcpyAsync(&T, ctx->tally.p + sys_id, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    T.collisions = collisions;
    T.wall_hits = wall_collisions;
    CK(cudaMemcpyAsync(ctx->tally.p + sys_id, &T, sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    const unsigned st = (unsigned)steps;
    ctx->step_known = false;
    CK(cudaMemcpyAsync(&ctx->status.p->step, &st, sizeof(st), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    h.t0_reduced = t;
    h.t_offset = t - (double)steps * h.settings.dt;
    return DSMC_OK;
}

namespace {
const char kCkptMagic[8] = {'D', 'S', 'M', 'C', 'B', '2', '0', '0'};
struct CkptHeader {
    char magic[8];
    uint32_t version, step;
    int32_t precision, num_systems, num_cells, pad;
    uint64_t records;
};
struct CkptSystem {
    int64_t num_particles;
    uint32_t id_count;
    int32_t active_begin, active_end, pad;
    double t0_reduced, t_offset;
    uint64_t rng_seed;
    SysTally tally;
};
}  // namespace

int dsmc_checkpoint_save(dsmc_ctx *ctx, const char *path) {
    if (!ctx || !path) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    long long staged = 0;
    rc = stage_present(ctx, 0, -1, &staged);  // every particle record with its cell key
    if (rc) return rc;
    const int C = ctx->num_cells, S = (int)ctx->systems.size();
    const size_t half = ctx->rec_half();
    std::vector<unsigned char> A(staged * half), B(staged * half);
    std::vector<int> key(staged);
    std::vector<double4> state(C);
    std::vector<double> mom(8 * (size_t)C);
    std::vector<SysTally> tally(S);
    if (staged) {
        CK(cudaMemcpyAsync(A.data(), ctx->fA.p, A.size(), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(B.data(), ctx->fB.p, B.size(), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(key.data(), ctx->fkey.p, staged * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (C) {
        CK(cudaMemcpyAsync(state.data(), ctx->state.p, C * sizeof(double4), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(mom.data(), ctx->mom.p, mom.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (S) CK(cudaMemcpyAsync(tally.data(), ctx->tally.p, S * sizeof(SysTally), cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<std::vector<double>> prof(S);
    for (int s = 0; s < S; ++s) CK(ctx->systems[s]->prof_sums(prof[s], ctx->stream));
    cudaError_t e;
    Status st = read_status(ctx, &e);
    CK(e);
    if (st.nout) return fail(ctx, DSMC_ERR_STATE, "take the outgoing records of the slab before a checkpoint");
    CkptHeader hd;
    std::memset(&hd, 0, sizeof(hd));
    std::memcpy(hd.magic, kCkptMagic, 8);
    hd.version = 2;
    hd.step = st.step;
    hd.precision = ctx->precision;
    hd.num_systems = S;
    hd.num_cells = C;
    hd.records = (uint64_t)staged;
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ctx, DSMC_ERR_IO, std::string("could not open ") + path);
    bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1;
    for (int s = 0; s < S && ok; ++s) {
        const SysHost &h = *ctx->systems[s];
        CkptSystem cs;
        std::memset(&cs, 0, sizeof(cs));
        cs.num_particles = h.num_particles;
        cs.id_count = h.id_count;
        cs.active_begin = h.active_begin;
        cs.active_end = h.active_end;
        cs.t0_reduced = h.t0_reduced;
        cs.t_offset = h.t_offset;
        cs.rng_seed = h.settings.rng_seed;
        cs.tally = tally[s];
        ok = std::fwrite(&cs, sizeof(cs), 1, f) == 1;
    }
    ok = ok && std::fwrite(state.data(), sizeof(double4), C, f) == (size_t)C;
    ok = ok && std::fwrite(mom.data(), sizeof(double), mom.size(), f) == mom.size();
    ok = ok && std::fwrite(A.data(), 1, A.size(), f) == A.size();
    ok = ok && std::fwrite(B.data(), 1, B.size(), f) == B.size();
    ok = ok && std::fwrite(key.data(), sizeof(int), key.size(), f) == key.size();
    for (int s = 0; s < S && ok; ++s) {  // version 2: the sampler profiles, per system {bins, pad, 4*bins doubles}
        const int32_t bp[2] = {ctx->systems[s]->prof_bins, 0};
        ok = std::fwrite(bp, sizeof(bp), 1, f) == 1;
        ok = ok && std::fwrite(prof[s].data(), sizeof(double), prof[s].size(), f) == prof[s].size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(ctx, DSMC_ERR_IO, std::string("could not write ") + path);
    return DSMC_OK;
}

int dsmc_checkpoint_load(dsmc_ctx *ctx, const char *path) {
    if (!ctx || !path) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ctx, DSMC_ERR_IO, std::string("could not open ") + path);
    auto bad = [&](const char *why) {
        std::fclose(f);
        return fail(ctx, DSMC_ERR_CONFIG, std::string(path) + ": " + why);
    };
    CkptHeader hd;
    if (std::fread(&hd, sizeof(hd), 1, f) != 1 || std::memcmp(hd.magic, kCkptMagic, 8) ||
        (hd.version != 1 && hd.version != 2))
        return bad("not a checkpoint of this library");
    const int C = ctx->num_cells, S = (int)ctx->systems.size();
    if (hd.precision != ctx->precision) return bad("written by a context of the other precision");
    if (hd.num_systems != S || hd.num_cells != C) return bad("the context's systems differ from the checkpoint's");
    std::vector<CkptSystem> cs(S);
    if (S && std::fread(cs.data(), sizeof(CkptSystem), S, f) != (size_t)S) return bad("truncated");
    for (int s = 0; s < S; ++s)
        if (cs[s].active_begin != ctx->systems[s]->active_begin || cs[s].active_end != ctx->systems[s]->active_end)
            return bad("the context's cells differ from the checkpoint's");
    const long long R = (long long)hd.records;
    const size_t half = ctx->rec_half();
    std::vector<double4> state(C);
    std::vector<double> mom(8 * (size_t)C);
    std::vector<unsigned char> A(R * half), B(R * half);
    std::vector<int> key(R);
    bool ok = std::fread(state.data(), sizeof(double4), C, f) == (size_t)C;
    ok = ok && std::fread(mom.data(), sizeof(double), mom.size(), f) == mom.size();
    ok = ok && std::fread(A.data(), 1, A.size(), f) == A.size();
    ok = ok && std::fread(B.data(), 1, B.size(), f) == B.size();
    ok = ok && std::fread(key.data(), sizeof(int), key.size(), f) == key.size();
    std::vector<std::vector<double>> prof(S);  // version 1 carries no profiles: they restart from zero
    for (int s = 0; s < S; ++s) prof[s].assign(4 * (size_t)ctx->systems[s]->prof_bins, 0.0);
    for (int s = 0; s < S && ok && hd.version >= 2; ++s) {
        int32_t bp[2];
        ok = std::fread(bp, sizeof(bp), 1, f) == 1;
        if (ok && bp[0] != ctx->systems[s]->prof_bins) return bad("the context's sampling bins differ from the checkpoint's");
        ok = ok && std::fread(prof[s].data(), sizeof(double), prof[s].size(), f) == prof[s].size();
    }
    if (!ok) return bad("truncated");
    std::fclose(f);
    std::vector<unsigned> hist(std::max(C, 1), 0);
    for (long long i = 0; i < R; ++i) {
        if (key[i] < 0 || key[i] >= C) return fail(ctx, DSMC_ERR_CONFIG, "checkpoint record outside the cells");
        ++hist[key[i]];
    }
    ctx->pending = false;  // the saved state had its collide and sample done
    CK(ctx->fA.ensure(std::max<long long>(R, 1) * half));
    CK(ctx->fB.ensure(std::max<long long>(R, 1) * half));
    CK(ctx->fkey.ensure(std::max<long long>(R, 1)));
    CK(ctx->hist.ensure(std::max(C, 1)));
    if (R) {
        CK(cudaMemcpyAsync(ctx->fA.p, A.data(), A.size(), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->fB.p, B.data(), B.size(), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->fkey.p, key.data(), R * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    }
    CK(cudaMemcpyAsync(ctx->hist.p, hist.data(), hist.size() * sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    for (int s = 0; s < S; ++s) {
        SysHost &h = *ctx->systems[s];
        h.num_particles = cs[s].num_particles;
        h.id_count = cs[s].id_count;
        h.t0_reduced = cs[s].t0_reduced;
        h.t_offset = cs[s].t_offset;
        if (h.settings.rng_seed != cs[s].rng_seed) {
            h.settings.rng_seed = cs[s].rng_seed;  // the draws continue the saved streams
            h.dev.seed = cs[s].rng_seed;
        }
    }
    int rc = upload_sys_table(ctx);
    if (rc) return rc;
    rc = relayout(ctx, R);
    if (rc) return rc;
    std::vector<SysTally> tally(S);
    for (int s = 0; s < S; ++s) tally[s] = cs[s].tally;
    if (C) {
        CK(cudaMemcpyAsync(ctx->state.p, state.data(), C * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->mom.p, mom.data(), mom.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    }
    if (S) CK(cudaMemcpyAsync(ctx->tally.p, tally.data(), S * sizeof(SysTally), cudaMemcpyHostToDevice, ctx->stream));
    for (int s = 0; s < S; ++s)
        CK(cudaMemsetAsync(ctx->systems[s]->prof.p, 0, ctx->systems[s]->prof_len() * sizeof(double), ctx->stream));
    for (int s = 0; s < S; ++s)  // the saved sums into the first copy
        CK(cudaMemcpyAsync(ctx->systems[s]->prof.p, prof[s].data(), prof[s].size() * sizeof(double),
                           cudaMemcpyHostToDevice, ctx->stream));
    ctx->step_known = false;
    CK(cudaMemcpyAsync(&ctx->status.p->step, &hd.step, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return DSMC_OK;
}

int dsmc_particles_count(dsmc_ctx *ctx, int sys_id, int64_t *n) {
    if (!ctx || !n || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    *n = ctx->systems[sys_id]->num_particles;
    return DSMC_OK;
}

int dsmc_particles_get(dsmc_ctx *ctx, int sys_id, int64_t cap, double *r, double *v, int32_t *cell, int64_t *n) {
    if (!ctx || !r || !v || !n || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    SysHost &h = *ctx->systems[sys_id];
    *n = h.num_particles;
    // a slab holds some of the geometry's ids: entries run over every id and
    // cell[i] = -1 marks the ids it does not hold
    const long long N = h.slab ? (long long)h.id_count : h.num_particles;
    if (h.slab && !cell) return fail(ctx, DSMC_ERR_ARG, "a slab reports which ids it holds through cell");
    if (cap < N)
        return fail(ctx, DSMC_ERR_CAPACITY, h.slab ? "output buffers smaller than the geometry's id count"
                                                   : "output buffers smaller than the particle count");
    CK(ctx->io_r.ensure(3 * std::max<long long>(N, 1)));
    CK(ctx->io_v.ensure(3 * std::max<long long>(N, 1)));
    CK(ctx->io_cell.ensure(std::max<long long>(N, 1)));
    if (N == 0) return DSMC_OK;
    if (h.slab) CK(cudaMemsetAsync(ctx->io_cell.p, 0xff, N * sizeof(int), ctx->stream));
    if (!ctx->io_stream) {
        CK(cudaStreamCreateWithFlags(&ctx->io_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->io_event, cudaEventDisableTiming));
    }
    // Each record's values go to its id's place, a scatter: the positions
    // (and cells) first, copied out on io_stream while the velocities are
    // converted, so that one conversion overlaps the other's copy.
    auto to_fp64 = [&](double *ro, double *vo, int *co) {
        return is_fp64(ctx) ? fp64::launch_to_fp64(ctx->sys_dev.p, sys_id, cell_arrays(ctx), particle_arrays(ctx),
                                                   ctx->cur, ctx->cphase, 0, N, ro, vo, co, &ctx->status.p->error,
                                                   ctx->stream)
                            : split32::launch_to_fp64(ctx->sys_dev.p, sys_id, cell_arrays(ctx), particle_arrays(ctx),
                                                      ctx->cur, ctx->cphase, 0, N, ro, vo, co, &ctx->status.p->error,
                                                      ctx->stream);
    };
    CK(to_fp64(ctx->io_r.p, nullptr, ctx->io_cell.p));
    CK(cudaEventRecord(ctx->io_event, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->io_stream, ctx->io_event, 0));
    cudaError_t e = cudaMemcpyAsync(r, ctx->io_r.p, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->io_stream);
    if (e == cudaSuccess && cell)
        e = cudaMemcpyAsync(cell, ctx->io_cell.p, N * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->io_stream);
    if (e == cudaSuccess) e = to_fp64(nullptr, ctx->io_v.p, nullptr);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(v, ctx->io_v.p, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    // both streams are done with the caller's buffers before this returns
    const cudaError_t e1 = cudaStreamSynchronize(ctx->io_stream);
    const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    CK(e);
    CK(e1);
    CK(e2);
    return DSMC_OK;
}

int dsmc_step(dsmc_ctx *ctx, int nsteps) {
    if (!ctx || nsteps < 0) return DSMC_ERR_ARG;
    if (ctx->systems.empty() || nsteps == 0) return DSMC_OK;
    cudaSetDevice(ctx->device);
    if (ctx->slab) {
        if (nsteps != 1) return fail(ctx, DSMC_ERR_ARG, "a slab advances one step between exchanges");
        if (!(ctx->use_pipelined && ctx->fused_grids[1] > 0))
            return fail(ctx, DSMC_ERR_CONFIG, "a slab needs the production pass (cells too large for it)");
    }
    ctx->keys_valid = false;
    int left = nsteps;
    while (left > 0) {
        unsigned step0 = ctx->known_step;
        if (!ctx->step_known) {
            cudaError_t e;
            const Status st = read_status(ctx, &e);
            CK(e);
            step0 = st.step;
        }
        const int cur0 = ctx->cur;
        const int cphase0 = ctx->cphase;
        const bool pending0 = ctx->pending;
        // One fused pass per step: collide + sample of the previous step's
        // cells, then accelerate + move + re-bin of this step.
        for (int i = 0; i < left; ++i) {
            const int prologue = (i == 0 && !pending0);
            // pass i collides at step step0 + i (a halted batch runs no later pass)
            const int sample = !prologue && samples_at(ctx, step0 + (unsigned)i);
            int rc = launch(ctx, PASS_FUSED, !prologue, 1, sample, 1);
            if (rc) return rc;
            ctx->cur ^= 1;
        }
        int ran = 0;
        int rc = settle(ctx, step0, cur0, cphase0, &ran);
        if (rc) return rc;
        if (ran <= 0) return fail(ctx, DSMC_ERR_STATE, "timestep pipeline made no progress");
        ctx->pending = true;
        left -= ran;
    }
    return DSMC_OK;
}

int dsmc_exchange_take(dsmc_ctx *ctx, int64_t cap, void *records, int device, int64_t *n) {
    if (!ctx || !n || cap < 0 || (cap > 0 && !records)) return DSMC_ERR_ARG;
    *n = 0;
    if (!ctx->slab) return DSMC_OK;
    cudaSetDevice(ctx->device);
    cudaError_t e;
    Status st = read_status(ctx, &e);
    CK(e);
    if (st.nout > ctx->out_cap)
        return fail(ctx, DSMC_ERR_STATE, "more particles left the slab in one step than its outgoing list holds");
    *n = st.nout;
    if ((int64_t)st.nout > cap) return fail(ctx, DSMC_ERR_CAPACITY, "record buffer smaller than the outgoing count");
    if (st.nout) {
        CK(cudaMemcpyAsync(records, ctx->out.p, 2 * sizeof(uint4) * st.nout,
                           device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
        const unsigned zero = 0;
        CK(cudaMemcpyAsync(&ctx->status.p->nout, &zero, sizeof(zero), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->systems[0]->num_particles -= st.nout;
    }
    return DSMC_OK;
}

int dsmc_exchange_put(dsmc_ctx *ctx, int sys_id, int64_t n, const void *records, int device) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size() || n < 0 || (n > 0 && !records))
        return DSMC_ERR_ARG;
    if (!ctx->slab) return fail(ctx, DSMC_ERR_CONFIG, "records enter a slab system only");
    if (n == 0) return DSMC_OK;
    cudaSetDevice(ctx->device);
    SysHost &h = *ctx->systems[sys_id];
    const uint4 *src = static_cast<const uint4 *>(records);
    DevBuf<uint4> staged;
    if (!device) {
        CK(staged.alloc(2 * (size_t)n));
        CK(cudaMemcpyAsync(staged.p, records, 2 * sizeof(uint4) * n, cudaMemcpyHostToDevice, ctx->stream));
        src = staged.p;
    }
    CK(split32::launch_put(ctx->sys_dev.p, sys_id, cell_arrays(ctx), particle_arrays(ctx), ctx->cur, ctx->cphase, n,
                           src, ctx->status.p, ctx->stream));
    cudaError_t e;
    Status st = read_status(ctx, &e);
    CK(e);
    h.num_particles += n;
    if (st.error & DSMC_EBIT_CELL) return fail(ctx, DSMC_ERR_STATE, "a record lies outside the slab's cells");
    if (st.error & DSMC_EBIT_FATAL) return fail(ctx, DSMC_ERR_STATE, "records could not be placed");
    if (st.spill) {
        // cells without room: repack with the overflow records
        long long staged_n = 0;
        int rc = stage_present(ctx, 0, -1, &staged_n);
        if (rc) return rc;
        return relayout(ctx, staged_n);
    }
    return DSMC_OK;
}

int dsmc_stage_move(dsmc_ctx *ctx) {
    if (!ctx) return DSMC_ERR_ARG;
    if (ctx->slab) return fail(ctx, DSMC_ERR_CONFIG, "a slab moves through dsmc_step and the exchange");
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    rc = launch(ctx, PASS_INPLACE, 0, 1, 0, 1);
    if (rc) return rc;
    ctx->keys_valid = true;
    return DSMC_OK;
}

int dsmc_stage_sort(dsmc_ctx *ctx) {
    if (!ctx) return DSMC_ERR_ARG;
    if (ctx->slab) return fail(ctx, DSMC_ERR_CONFIG, "a slab moves through dsmc_step and the exchange");
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    if (!ctx->keys_valid) return DSMC_OK;  // nothing moved since the last re-bin
    ctx->keys_valid = false;
    cudaError_t e;
    rc = launch(ctx, PASS_SORT, 0, 0, 0, 0);
    if (rc) return rc;
    ctx->cur ^= 1;
    Status st2 = read_status(ctx, &e);
    CK(e);
    if (st2.error & DSMC_EBIT_FATAL) return fail(ctx, DSMC_ERR_STATE, "sort failed");
    if (st2.spill) {
        long long staged = 0;
        rc = stage_present(ctx, 0, -1, &staged);
        if (rc) return rc;
        return relayout(ctx, staged);
    }
    return DSMC_OK;
}

int dsmc_stage_collide(dsmc_ctx *ctx) {
    if (!ctx) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    return launch(ctx, PASS_INPLACE, 1, 0, 0, 0);
}

int dsmc_stage_sample(dsmc_ctx *ctx) {
    if (!ctx) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    return launch(ctx, PASS_INPLACE, 0, 0, 1, 0);
}

int dsmc_tallies_get(dsmc_ctx *ctx, int sys_id, dsmc_tallies *t) {
    if (!ctx || !t || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    SysHost &h = *ctx->systems[sys_id];
    SysTally T;
    CK(cudaMemcpyAsync(&T, ctx->tally.p + sys_id, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    cudaError_t e;
    Status st = read_status(ctx, &e);
    CK(e);
    std::memset(t, 0, sizeof(*t));
    t->step = st.step;
    t->collisions = T.collisions;
    t->wall_collisions = T.wall_hits;
    t->reseeds = T.reseeds;
    t->particle_steps = T.particle_steps;
    for (int a = 0; a < 3; ++a) t->count_periodic[a] = T.count_periodic[a];
    t->samples = T.samples;
    t->candidates = T.candidates;
    t->stranded = T.stranded;
    t->time = st.step * h.settings.dt + h.t_offset;
    // MeasureEnergy / MeasureTemperature (dsmc/statisticalproperty.cpp:21-71)
    // from the current velocities, summed per cell and then in cell order.
    const int C = h.active_end - h.active_begin;
    if (C > 0 && ctx->A0.p) {
        // kept by the context: a sampler reading this every few steps
        // allocates once, not on every read
        DevBuf<double> &ce = ctx->cell_energy;
        CK(ce.ensure(C));
        e = is_fp64(ctx) ? fp64::launch_cell_energy(cell_arrays(ctx), particle_arrays(ctx), ctx->cur, ctx->cphase,
                                                    h.active_begin,
                                                    h.active_end, ce.p, ctx->stream)
                         : split32::launch_cell_energy(cell_arrays(ctx), particle_arrays(ctx), ctx->cur,
                                                       ctx->cphase, h.active_begin, h.active_end, ce.p, ctx->stream);
        CK(e);
        std::vector<double> hc(C);
        CK(cudaMemcpyAsync(hc.data(), ce.p, C * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        double sum = 0;
        for (double x : hc) sum += x;
        t->kinetic_energy = sum * 0.5 * h.settings.mass * h.atoms_per_molecule;
        if (h.num_particles > 0)
            t->temperature = ctx->units.temperature_to_SI(2.0 / 3.0 * t->kinetic_energy /
                                                          (h.num_particles * h.atoms_per_molecule));
    }
    const double elapsed = t->time - h.t0_reduced;
    const int fd = h.settings.flow_direction;
    if (fd >= 0 && fd < 3 && elapsed > 0) t->flux = h.atoms_per_molecule * T.count_periodic[fd] / elapsed;
    return DSMC_OK;
}

int dsmc_measures_get(dsmc_ctx *ctx, int sys_id, dsmc_measures *m) {
    if (!ctx || !m || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    dsmc_tallies t;
    int rc = dsmc_tallies_get(ctx, sys_id, &t);
    if (rc) return rc;
    const SysHost &h = *ctx->systems[sys_id];
    const dsmc_settings &s = h.settings;
    const Units &u = ctx->units;
    // System::get_number_of_atoms_global and the reduced temperature of
    // MeasureTemperature (dsmc/statisticalproperty.cpp:57-68)
    const double atoms = (double)h.num_particles * h.atoms_per_molecule;
    const double T = atoms > 0 ? 2.0 / 3.0 * t.kinetic_energy / atoms : 0.0;
    const double density = u.number_density_from_SI(s.density);
    std::memset(m, 0, sizeof(*m));
    m->step = t.step;
    m->t_ns = u.time_to_SI(t.time) * 1e9;
    m->energy_eV = u.energy_to_eV(t.kinetic_energy);
    m->temperature_K = u.temperature_to_SI(T);
    m->number_flow_rate = t.flux;
    m->volumetric_flow_rate = t.flux * (1.0 / density);  // MeasureVolumetricFlowRate (:118-133)
    if (h.volume_global > 0) m->pressure_Pa = u.pressure_to_SI(atoms / h.volume_global * T);  // MeasurePressure
    const int fd = s.flow_direction;
    if (fd >= 0 && fd < 3 && s.gravity != 0 && density > 0) {
        // MeasurePermeability::update (:180-210): kinetic-theory viscosity of
        // hard spheres, permeability = Q mu / (A m n g)
        const double L[3] = {s.Lx, s.Ly, s.Lz};
        double area = 1;
        for (int a = 0; a < 3; ++a)
            if (a != fd) area *= L[a];
        const double viscosity = 5.0 / (16 * s.diam * s.diam) * std::sqrt(s.mass * T / M_PI);
        const double k = m->volumetric_flow_rate * viscosity / (area * s.mass * density * s.gravity);
        m->permeability_darcy = u.permeability_to_darcy(k);
    }
    m->collisions = t.collisions;
    m->wall_collisions = t.wall_collisions;
    m->molecules = (uint64_t)h.num_particles;
    return DSMC_OK;
}

int dsmc_profile_sums_get(dsmc_ctx *ctx, int sys_id, int cap, double *sums, int *bins) {
    if (!ctx || !bins || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    const SysHost &h = *ctx->systems[sys_id];
    *bins = h.prof_bins;
    if (!sums) return DSMC_OK;
    if (cap < 4 * h.prof_bins) return fail(ctx, DSMC_ERR_CAPACITY, "profile buffer smaller than 4 * sampling_bins");
    std::vector<double> total;
    CK(h.prof_sums(total, ctx->stream));
    std::memcpy(sums, total.data(), total.size() * sizeof(double));
    return DSMC_OK;
}

int dsmc_profiles_get(dsmc_ctx *ctx, int sys_id, int cap, double *count, double *velocity_z, double *temperature,
                      double *pressure, double *vx_center, double *vx_count, int *bins) {
    if (!ctx || !bins || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    int rc = dsmc_profile_sums_get(ctx, sys_id, 0, nullptr, bins);
    if (rc) return rc;
    if (cap < *bins) return fail(ctx, DSMC_ERR_CAPACITY, "profile buffers smaller than sampling_bins");
    const SysHost &h = *ctx->systems[sys_id];
    std::vector<double> sums(4 * (size_t)*bins);
    rc = dsmc_profile_sums_get(ctx, sys_id, (int)sums.size(), sums.data(), bins);
    if (rc) return rc;
    return dsmc_profiles_finish(&h.settings, h.volume_global, *bins, sums.data(), count, velocity_z, temperature,
                                pressure, vx_center, vx_count);
}

int dsmc_tallies_reset(dsmc_ctx *ctx, int sys_id) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    SysHost &h = *ctx->systems[sys_id];
    CK(cudaMemsetAsync(ctx->tally.p + sys_id, 0, sizeof(SysTally), ctx->stream));
    const int C = h.active_end - h.active_begin;
    if (C > 0) CK(cudaMemsetAsync(ctx->mom.p + 8 * (size_t)h.active_begin, 0, 8 * (size_t)C * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(h.prof.p, 0, h.prof_len() * sizeof(double), ctx->stream));
    cudaError_t e;
    Status st = read_status(ctx, &e);
    CK(e);
    h.t0_reduced = st.step * h.settings.dt + h.t_offset;
    return DSMC_OK;
}

int dsmc_cells_get(dsmc_ctx *ctx, int sys_id, int cap, int32_t *global_index, int32_t *count, double *vr_max,
                   double *rest, double *moments, double *volume, int *num_cells) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    SysHost &h = *ctx->systems[sys_id];
    const int C = h.active_end - h.active_begin;
    if (num_cells) *num_cells = C;
    if (cap < C) return fail(ctx, DSMC_ERR_CAPACITY, "output buffers smaller than the active cell count");
    if (C == 0) return DSMC_OK;
    const int a0 = h.active_begin;
    if (global_index) std::memcpy(global_index, h.cell_global.data(), C * sizeof(int32_t));
    if (volume) std::memcpy(volume, h.volume_cell.data(), C * sizeof(double));
    std::vector<unsigned> nb, nt;
    if (count) {
        nb.resize(C);
        nt.resize(C);
        CK(cudaMemcpyAsync(nb.data(), ctx->bot[ctx->cphase].p + a0, C * sizeof(unsigned), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaMemcpyAsync(nt.data(), ctx->top[ctx->cphase].p + a0, C * sizeof(unsigned), cudaMemcpyDeviceToHost,
                           ctx->stream));
    }
    std::vector<double4> st(C);
    std::vector<int4> mt(count ? C : 0);
    if (count) CK(cudaMemcpyAsync(mt.data(), ctx->meta.p + a0, C * sizeof(int4), cudaMemcpyDeviceToHost, ctx->stream));
    if (vr_max || rest)
        CK(cudaMemcpyAsync(st.data(), ctx->state.p + a0, C * sizeof(double4), cudaMemcpyDeviceToHost, ctx->stream));
    if (moments)
        CK(cudaMemcpyAsync(moments, ctx->mom.p + 8 * (size_t)a0, 8 * (size_t)C * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < C; ++q) {
        if (vr_max) vr_max[q] = st[q].x;
        if (rest) rest[q] = st[q].y;
        if (count) {
            const unsigned cap = (unsigned)mt[q].y;
            const unsigned b = std::min(nb[q], cap);
            count[q] = (int32_t)(b + std::min(nt[q], cap - b));
        }
    }
    return DSMC_OK;
}

int dsmc_cells_set_state(dsmc_ctx *ctx, int sys_id, const double *vr_max, const double *rest) {
    if (!ctx || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    SysHost &h = *ctx->systems[sys_id];
    const int C = h.active_end - h.active_begin;
    if (C == 0) return DSMC_OK;
    std::vector<double4> st(C);
    CK(cudaMemcpyAsync(st.data(), ctx->state.p + h.active_begin, C * sizeof(double4), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < C; ++q) {
        if (vr_max) st[q].x = vr_max[q];
        if (rest) st[q].y = rest[q];
    }
    CK(cudaMemcpyAsync(ctx->state.p + h.active_begin, st.data(), C * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return DSMC_OK;
}

void *dsmc_stream(dsmc_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int dsmc_ctx_set_capacity(dsmc_ctx *ctx, double factor, int pad) {
    if (!ctx || !(factor >= 1.0) || pad < 0) return DSMC_ERR_ARG;
    ctx->cap_factor = factor;
    ctx->cap_pad = pad;
    return DSMC_OK;
}

int dsmc_counters_get(dsmc_ctx *ctx, int sys_id, int64_t out[8]) {
    if (!ctx || !out || sys_id < 0 || sys_id >= (int)ctx->systems.size()) return DSMC_ERR_ARG;
    SysTally T;
    CK(cudaMemcpyAsync(&T, ctx->tally.p + sys_id, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    out[0] = (int64_t)T.collisions;
    out[1] = (int64_t)T.wall_hits;
    out[2] = (int64_t)T.reseeds;
    out[3] = (int64_t)T.particle_steps;
    out[4] = T.count_periodic[0];
    out[5] = T.count_periodic[1];
    out[6] = T.count_periodic[2];
    out[7] = (int64_t)T.samples;
    return DSMC_OK;
}

int dsmc_pass_info(dsmc_ctx *ctx, int *pipelined, int *grid, int *block, int *stage_capacity) {
    if (!ctx) return DSMC_ERR_ARG;
    const bool pipe = ctx->use_pipelined && ctx->fused_grids[1] > 0;
    if (pipelined) *pipelined = pipe ? 1 : 0;
    if (grid) *grid = pipe ? ctx->fused_grids[1] : ctx->grid;
    if (block) *block = pipe ? split32::fused_block() : ctx->block;
    if (stage_capacity) *stage_capacity = pipe ? split32::fused_capacity(ctx->smem_cap) : ctx->smem_cap;
    return DSMC_OK;
}

int dsmc_ctx_set_timing(dsmc_ctx *ctx, int on) {
    if (!ctx) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (on) {
        for (cudaEvent_t &e : ctx->tev)
            if (!e) CK(cudaEventCreate(&e));
    }
    ctx->timing = on != 0;
    for (double &t : ctx->tms) t = 0;
    ctx->tpasses = 0;
    return DSMC_OK;
}

int dsmc_pass_times_get(dsmc_ctx *ctx, double ms[4], int64_t *passes) {
    if (!ctx || !ms) return DSMC_ERR_ARG;
    for (int k = 0; k < 4; ++k) ms[k] = ctx->tms[k];
    if (passes) *passes = ctx->tpasses;
    return DSMC_OK;
}

int dsmc_tuning_set(dsmc_ctx *ctx, const dsmc_tuning *t) {
    if (!ctx || !t) return DSMC_ERR_ARG;
    for (int k = 0; k < 5; ++k)
        if (t->blocks_per_sm[k] < 0 || t->blocks_per_sm[k] > 64) return fail(ctx, DSMC_ERR_ARG, "blocks per SM out of range");
    if (t->ring < 0 || t->ring > split32::max_ring()) return fail(ctx, DSMC_ERR_ARG, "ring out of range");
    if (t->collide_claim < 0 || t->collide_claim > 2) return fail(ctx, DSMC_ERR_ARG, "collide_claim is 0, 1 or 2");
    cudaSetDevice(ctx->device);
    int rc = flush_pending(ctx);
    if (rc) return rc;
    for (int k = 0; k < 5; ++k) ctx->tune_bps[k] = t->blocks_per_sm[k];
    ctx->tune_ring = t->ring;
    ctx->tune_claim = t->collide_claim;
    ctx->drop_graphs();  // the grids are baked into the captured passes
    apply_launch_shape(ctx);
    return DSMC_OK;
}

int dsmc_tuning_get(dsmc_ctx *ctx, dsmc_tuning *current, dsmc_tuning *limits) {
    if (!ctx) return DSMC_ERR_ARG;
    if (current) {
        for (int k = 0; k < 5; ++k) current->blocks_per_sm[k] = ctx->tune_bps[k];
        current->ring = ctx->tune_ring;
        current->collide_claim = ctx->tune_claim;
    }
    if (limits) {
        for (int k = 0; k < 5; ++k) limits->blocks_per_sm[k] = ctx->fused_max_bps[k];
        limits->ring = is_fp64(ctx) ? 0 : split32::ring_for(ctx->smem_cap, ctx->tune_ring);
        limits->collide_claim = 2;
    }
    return DSMC_OK;
}

int dsmc_device_status(dsmc_ctx *ctx, uint32_t *error_bits, uint32_t *spill) {
    if (!ctx) return DSMC_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaError_t e;
    Status st = read_status(ctx, &e);
    CK(e);
    if (error_bits) *error_bits = st.error;
    if (spill) *spill = st.spill;
    return DSMC_OK;
}

}  // extern "C"
