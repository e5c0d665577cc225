// Split-precision instantiation of the DSMC kernels: int voxel index + fp32
// in-voxel offset, fp32 velocities, fp64 cell bookkeeping and tallies.
#define DSMC_PREC Split32
#define DSMC_PREC_NS split32
#include "kernels_impl.cuh"
