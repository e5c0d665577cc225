// Split-precision instantiation of the DSMC kernels: int voxel index + fp32
// in-voxel offset, fp32 velocities, fp64 cell bookkeeping and tallies.
#define DSMC_PREC Split32
#define DSMC_PREC_NS split32
#include "kernels_impl.cuh"

#include "fused_split.cuh"

namespace dsmc {
namespace split32 {

// The production pass: smallest staging capacity that holds every cell.
template <int CAP> static cudaError_t launch_fused_cap(const PassParams &P, int grid, cudaStream_t st) {
    const size_t smem = fused::fused_smem_bytes<CAP>(8);
    fused::fused_split_kernel<CAP><<<grid, 256, smem, st>>>(P);
    return cudaGetLastError();
}
template <int CAP> static int fused_cap_blocks() {
    const size_t smem = fused::fused_smem_bytes<CAP>(8);
    // the opt-in limit is a property of the function, shared by every
    // context: raise it to the device maximum, never lower it
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fused::fused_split_kernel<CAP>) != cudaSuccess) return 0;
    if (smem + fa.sharedSizeBytes > (size_t)optin) return 0;
    if (cudaFuncSetAttribute(fused::fused_split_kernel<CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes) != cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fused::fused_split_kernel<CAP>, 256, smem) != cudaSuccess)
        return 0;
    return nb;
}

int fused_capacity(int smem_cap) {
    if (smem_cap <= 64) return 64;
    if (smem_cap <= 96) return 96;
    if (smem_cap <= 128) return 128;
    if (smem_cap <= 192) return 192;
    if (smem_cap <= 256) return 256;
    return 0;
}

int fused_blocks_per_sm(int smem_cap) {
    switch (fused_capacity(smem_cap)) {
        case 64: return fused_cap_blocks<64>();
        case 96: return fused_cap_blocks<96>();
        case 128: return fused_cap_blocks<128>();
        case 192: return fused_cap_blocks<192>();
        case 256: return fused_cap_blocks<256>();
    }
    return 0;
}

cudaError_t launch_fused(const PassParams &P, int grid, cudaStream_t st) {
    switch (fused_capacity(P.smem_cap)) {
        case 64: return launch_fused_cap<64>(P, grid, st);
        case 96: return launch_fused_cap<96>(P, grid, st);
        case 128: return launch_fused_cap<128>(P, grid, st);
        case 192: return launch_fused_cap<192>(P, grid, st);
        case 256: return launch_fused_cap<256>(P, grid, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace split32
}  // namespace dsmc
