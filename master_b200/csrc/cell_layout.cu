// Slot layout of the cells on the device: each active cell's capacity from
// its expected and present occupancy, then the cells' first slots as an
// exclusive scan of the capacities in cell order (systems one after another).
// Replaces a host loop over every cell and the upload of its table.
#include <cuda_runtime.h>

#include "kernels.h"

namespace dsmc {
namespace {

constexpr int LB = 1024;  // cells per block of the first and last kernel

// Capacity of one cell: the larger of the expected occupancy (the system's
// particles spread over its free voxels) and the present one, times `factor`
// plus `pad`, at least 1.  Rounded as the host does it (no fused multiply-add).
__device__ __forceinline__ unsigned cell_capacity(int pix, unsigned present, double2 np, double factor, double pad) {
    const double expect = np.y > 0 ? __ddiv_rn(__dmul_rn(np.x, (double)pix), np.y) : 0.0;
    const double want = fmax(expect, (double)present);
    const unsigned cap = (unsigned)ceil(__dadd_rn(__dmul_rn(factor, want), pad));
    return cap < 1u ? 1u : cap;
}

__device__ __forceinline__ unsigned long long warp_incl_scan(unsigned long long x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Inclusive scan over a block of LB threads; `tot` receives the block's sum.
__device__ unsigned long long block_incl_scan(unsigned long long x, unsigned long long *ws, unsigned long long &tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    x = warp_incl_scan(x, lane);
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) ws[lane] = warp_incl_scan(ws[lane], lane);
    __syncthreads();
    if (w > 0) x += ws[w - 1];
    tot = ws[31];
    __syncthreads();
    return x;
}

// meta[a].y = capacity of cell a; per block the sum of the capacities; the
// largest capacity into out[1].
__global__ void __launch_bounds__(LB) k_capacities(int4 *meta, const int *pix, const unsigned *present,
                                                   const double2 *np, double factor, double pad, int C,
                                                   unsigned long long *bsum, unsigned long long *out) {
    __shared__ unsigned long long ws[32];
    __shared__ unsigned wmax[32];
    const int a = blockIdx.x * LB + threadIdx.x;
    unsigned cap = 0;
    if (a < C) {
        const int sys = meta[a].w;
        cap = cell_capacity(pix[a], present[a], np[sys], factor, pad);
        meta[a].y = (int)cap;
    }
    unsigned long long tot;
    block_incl_scan(cap, ws, tot);
    const unsigned m = __reduce_max_sync(0xffffffffu, cap);
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        const unsigned mb = __reduce_max_sync(0xffffffffu, wmax[threadIdx.x]);
        if (threadIdx.x == 0) {
            bsum[blockIdx.x] = tot;
            atomicMax(out + 1, (unsigned long long)mb);
        }
    }
}

// Exclusive scan of the block sums in place (one block); the total into out[0].
__global__ void __launch_bounds__(LB) k_scan_blocks(unsigned long long *bsum, int nb, unsigned long long *out) {
    __shared__ unsigned long long ws[32];
    const int per = (nb + LB - 1) / LB;
    const int i0 = threadIdx.x * per, i1 = min(i0 + per, nb);
    unsigned long long s = 0;
    for (int i = i0; i < i1; ++i) s += bsum[i];
    unsigned long long tot;
    const unsigned long long incl = block_incl_scan(s, ws, tot);
    unsigned long long run = incl - s;
    for (int i = i0; i < i1; ++i) {
        const unsigned long long v = bsum[i];
        bsum[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) out[0] = tot;
}

// meta[a].x = first slot of cell a: the block's offset plus the capacities
// of the cells before a in its block.
__global__ void __launch_bounds__(LB) k_bases(int4 *meta, int C, const unsigned long long *bsum) {
    __shared__ unsigned long long ws[32];
    const int a = blockIdx.x * LB + threadIdx.x;
    const unsigned cap = a < C ? (unsigned)meta[a].y : 0u;
    unsigned long long tot;
    const unsigned long long incl = block_incl_scan(cap, ws, tot);
    if (a < C) meta[a].x = (int)(bsum[blockIdx.x] + incl - cap);  // the host refuses totals of 2^31 or more
}

}  // namespace

int cell_layout_blocks(int C) { return (C + LB - 1) / LB; }

cudaError_t launch_cell_layout(int4 *meta, const int *pix, const unsigned *present, const double2 *np, double factor,
                               double pad, int C, unsigned long long *bsum, unsigned long long *out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess || C <= 0) return e;
    const int nb = cell_layout_blocks(C);
    k_capacities<<<nb, LB, 0, st>>>(meta, pix, present, np, factor, pad, C, bsum, out);
    k_scan_blocks<<<1, LB, 0, st>>>(bsum, nb, out);
    k_bases<<<nb, LB, 0, st>>>(meta, C, bsum);
    return cudaGetLastError();
}

}  // namespace dsmc
