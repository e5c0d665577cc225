// fp64 instantiation of the DSMC kernels: the reference's own state and
// arithmetic.  Built with -fmad=false so every product and sum is rounded on
// its own, as in the reference's x86-64 build.
#define DSMC_PREC Fp64
#define DSMC_PREC_NS fp64
#include "kernels_impl.cuh"
