// Split-precision instantiation of the DSMC kernels: int voxel index + fp32
// in-voxel offset, fp32 velocities, fp64 cell bookkeeping and tallies.
#define DSMC_PREC Split32
#define DSMC_PREC_NS split32
#include "kernels_impl.cuh"

#include "fused_split.cuh"

namespace dsmc {
namespace split32 {

// The production pass: the smallest ring that holds the largest cell.
template <int R> static cudaError_t launch_fused_ring(const PassParams &P, int grid, cudaStream_t st) {
    fused::fused_split_kernel<R><<<grid, 32 * fused::FUSED_WARPS, fused::fused_smem_bytes<R>(), st>>>(P);
    return cudaGetLastError();
}
template <int R> static int fused_ring_blocks() {
    const size_t smem = fused::fused_smem_bytes<R>();
    // the opt-in limit is a property of the function, shared by every
    // context: raise it to the device maximum, never lower it
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fused::fused_split_kernel<R>) != cudaSuccess) return 0;
    if (smem + fa.sharedSizeBytes > (size_t)optin) return 0;
    if (cudaFuncSetAttribute(fused::fused_split_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes) != cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fused::fused_split_kernel<R>, 32 * fused::FUSED_WARPS,
                                                      smem) != cudaSuccess)
        return 0;
    return nb;
}

// Ring slots per warp of the production pass for cells of at most
// `smem_cap` slots (0: no ring is large enough).
int fused_capacity(int smem_cap) {
    static const int rings[] = {64, 96, 128, 160, 192, 224, 256};
    for (int r : rings)
        if (smem_cap <= r) return r;
    return 0;
}

int fused_block() { return 32 * fused::FUSED_WARPS; }

#define DSMC_FUSED_RINGS(X) X(64) X(96) X(128) X(160) X(192) X(224) X(256)

int fused_blocks_per_sm(int smem_cap) {
    switch (fused_capacity(smem_cap)) {
#define X(r) \
    case r: return fused_ring_blocks<r>();
        DSMC_FUSED_RINGS(X)
#undef X
    }
    return 0;
}

cudaError_t launch_fused(const PassParams &P, int grid, cudaStream_t st) {
    switch (fused_capacity(P.smem_cap)) {
#define X(r) \
    case r: return launch_fused_ring<r>(P, grid, st);
        DSMC_FUSED_RINGS(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

}  // namespace split32
}  // namespace dsmc
