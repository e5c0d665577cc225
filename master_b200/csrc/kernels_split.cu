// Split-precision instantiation of the DSMC kernels: int voxel index + fp32
// in-voxel offset, fp32 velocities, fp64 cell bookkeeping and tallies.
#define DSMC_PREC Split32
#define DSMC_PREC_NS split32
#include <algorithm>
#include "kernels_impl.cuh"

#include "split_pass.cuh"

namespace dsmc {
namespace split32 {

// The production pass (split_pass.cuh): collide_cells, move_cells with the
// smallest ring that holds the largest cell, place_movers, place_walls.
template <int R> static cudaError_t launch_move_ring(const PassParams &P, int grid, cudaStream_t st) {
    pass3::move_cells_kernel<R><<<grid, 32 * pass3::M_WARPS, pass3::move_smem_bytes<R>(), st>>>(P);
    return cudaGetLastError();
}
template <int R> static int move_ring_blocks() {
    const size_t smem = pass3::move_smem_bytes<R>();
    // the opt-in limit is a property of the function, shared by every
    // context: raise it to the device maximum, never lower it
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, pass3::move_cells_kernel<R>) != cudaSuccess) return 0;
    if (smem + fa.sharedSizeBytes > (size_t)optin) return 0;
    if (cudaFuncSetAttribute(pass3::move_cells_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes) != cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pass3::move_cells_kernel<R>, 32 * pass3::M_WARPS,
                                                      smem) != cudaSuccess)
        return 0;
    return nb;
}
template <class K> static int static_blocks(K kernel, int threads) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, 0) != cudaSuccess) return 0;
    return nb;
}

// Ring slots per warp of move_cells for cells of at most `smem_cap` slots
// (0: no ring is large enough, or a cell could exceed the collide batch).
int fused_capacity(int smem_cap) {
    static const int rings[] = {64, 96, 128, 160, 192, 224, 256, 320, 384, 448, 512};
    if (smem_cap > pass3::PCAP) return 0;
    for (int r : rings)
        if (smem_cap <= r) return r;
    return 0;
}

int ring_for(int smem_cap, int ring) {
    static const int rings[] = {64, 96, 128, 160, 192, 224, 256, 320, 384, 448, 512};
    const int need = fused_capacity(smem_cap);
    if (need <= 0) return 0;
    const int want = std::max(need, ring);
    for (int r : rings)
        if (want <= r) return r;
    return 0;
}

int max_ring() { return 512; }

int fused_block() { return 32 * pass3::M_WARPS; }

#define DSMC_MOVE_RINGS(X) X(64) X(96) X(128) X(160) X(192) X(224) X(256) X(320) X(384) X(448) X(512)

int fused_grids(int smem_cap, int num_sms, int grids[5], int ring, int max_bps[5]) {
    int bm = 0;
    switch (ring_for(smem_cap, ring)) {
#define X(r) \
    case r: bm = move_ring_blocks<r>(); break;
        DSMC_MOVE_RINGS(X)
#undef X
    }
    const int bc = std::min(static_blocks(pass3::collide_cells_kernel<false>, 32 * pass3::C_WARPS),
                            static_blocks(pass3::collide_cells_kernel<true>, 32 * pass3::C_WARPS));
    const int bp = static_blocks(pass3::place_movers_kernel, 32 * pass3::P_WARPS);
    const int bw = static_blocks(pass3::place_walls_kernel, 32 * pass3::W_WARPS);
    const int bs = static_blocks(pass3::sample_cells_kernel, 32 * pass3::C_WARPS);
    if (bm <= 0 || bc <= 0 || bp <= 0 || bw <= 0 || bs <= 0) return 0;
    grids[0] = bc * num_sms;
    grids[1] = bm * num_sms;
    grids[2] = bp * num_sms;
    grids[3] = bw * num_sms;
    grids[4] = bs * num_sms;
    if (max_bps) {
        max_bps[0] = bc;
        max_bps[1] = bm;
        max_bps[2] = bp;
        max_bps[3] = bw;
        max_bps[4] = bs;
    }
    return 1;
}

// collide_cells with the chunk counter when each warp has many chunks
static void launch_collide_cells(const PassParams &P, int grid, cudaStream_t st) {
    const long long nchunks = (P.cells.num_cells + 31) / 32;
    const bool counter = P.claim == 2 ||
                         (P.claim == 0 && nchunks >= (long long)pass3::CLAIM_MIN_CHUNKS_PER_WARP * grid * pass3::C_WARPS);
    if (counter)
        pass3::collide_cells_kernel<true><<<grid, 32 * pass3::C_WARPS, 0, st>>>(P);
    else
        pass3::collide_cells_kernel<false><<<grid, 32 * pass3::C_WARPS, 0, st>>>(P);
}

cudaError_t launch_fused(const PassParams &P, const int grids[5], cudaStream_t st, cudaEvent_t *ev) {
    if (ev) cudaEventRecord(ev[0], st);
    if (P.do_collide || P.do_sample) {
        launch_collide_cells(P, grids[0], st);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (P.do_sample) {  // sampled steps only: the host knows the cadence
            pass3::sample_cells_kernel<<<grids[4], 32 * pass3::C_WARPS, 0, st>>>(P);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    if (ev) cudaEventRecord(ev[1], st);
    cudaError_t e = cudaErrorInvalidValue;
    switch (ring_for(P.smem_cap, P.ring)) {
#define X(r) \
    case r: e = launch_move_ring<r>(P, grids[1], st); break;
        DSMC_MOVE_RINGS(X)
#undef X
    }
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[2], st);
    pass3::place_movers_kernel<<<grids[2], 32 * pass3::P_WARPS, 0, st>>>(P);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[3], st);
    pass3::place_walls_kernel<<<grids[3], 32 * pass3::W_WARPS, 0, st>>>(P);
    e = cudaGetLastError();
    if (ev) cudaEventRecord(ev[4], st);
    return e;
}

cudaError_t launch_collide(const PassParams &P, const int grids[5], cudaStream_t st) {
    launch_collide_cells(P, grids[0], st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (P.do_sample) {
        pass3::sample_cells_kernel<<<grids[4], 32 * pass3::C_WARPS, 0, st>>>(P);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    // place_walls, whose last block zeroes collide_cells' chunk counter at the
    // end of a full pass, does not run here
    return cudaMemsetAsync(&P.status->collide_taken, 0, sizeof(unsigned), st);
}

cudaError_t launch_put(const SysDev *sys, int s, const CellArrays &cells, const ParticleArrays &parts, int cur, int cin,
                       long long n, const uint4 *rec, Status *status, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int grid = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    pass3::put_records_kernel<<<grid, 256, 0, st>>>(sys, s, cells, parts, cur, cin, n, rec, status);
    return cudaGetLastError();
}

}  // namespace split32
}  // namespace dsmc
