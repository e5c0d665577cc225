// Surrogate network kernels: a 3-level 3D U-Net that maps a porous voxel
// geometry (solid mask + Knudsen number) to the steady per-voxel density and
// drift of the gas, used to warm-start the DSMC particles.  The reference has
// no counterpart: it always starts from a Maxwellian at rest
// (System::setup_molecules, dsmc/system.cpp:398-430).
//
// Tensors are channels-last bf16 volumes [batch][d0][d1][d2][channels] of a
// cube of edge S (a power of two), addressed with a channel stride and a
// channel offset so that a concatenation is two views of one buffer.  Every
// 3x3x3 convolution pads periodically, as the DSMC geometry is periodic.
//
// Convolutions are implicit GEMMs on the fifth-generation tensor cores
// (tcgen05.mma, bf16 operands, fp32 accumulators in TMEM):
//   forward:  D[voxel][co]  = sum_{tap,ci} X[voxel + off(tap)][ci] W[co][tap][ci]
//   dgrad:    the forward kernel on the flipped, transposed weights
//             Wd[ci][tap][co] = W[co][26 - tap][ci]
//   wgrad:    D[(tap,co)][ci] = sum_u dY[u - off(tap)][co] X[u][ci]
// M tiles of 128 rows, operands staged in shared memory by cp.async in a
// three-stage ring, one elected thread issuing the MMAs, completion tracked
// by tcgen05.commit on an mbarrier per stage.  The epilogue (bias, ReLU, the
// ReLU mask of a gradient, bf16 rounding) runs on the TMEM read-back.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "dsmc_b200.h"
#include "dsmc_internal.h"
#include "dsmc_surrogate.h"
#include "tc05.cuh"

namespace sg {

using bf16 = __nv_bfloat16;

constexpr int kThreads = 128;  // four warps: one TMEM lane quarter each
constexpr int kStages = 3;
constexpr int kChunks = 8;     // 16-byte K chunks per stage (64 bf16 = 4 MMAs of K = 16)
constexpr int kRowBytes = 16;
constexpr int kATileBytes = kChunks * 128 * kRowBytes;  // 128 rows

__device__ unsigned g_error;  // set when a bounded wait ran out

struct Vol {
    const bf16 *p;
    int cs, coff;
};
struct VolOut {
    bf16 *p;
    int cs, coff;
};

struct ConvArgs {
    Vol in;
    int cin;
    const bf16 *w;      // [n][27][cin]
    const float *bias;  // [n] or null
    VolOut out;
    Vol mask;           // multiply output channel c by (mask > 0), or mask.p null
    int relu;
    int S, lg;          // edge and log2(edge)
    long long rows;     // batch * S^3
};

__device__ __forceinline__ int tap_d(int t, int axis) {
    return axis == 0 ? t / 9 - 1 : axis == 1 ? (t / 3) % 3 - 1 : t % 3 - 1;
}

// Linear voxel row of the neighbour at tap t (sign +1: +off, -1: -off).
__device__ __forceinline__ long long neighbour(long long row, int t, int sign, int S, int lg) {
    const long long vol = 1ll << (3 * lg);
    const long long b = row >> (3 * lg);
    const int v = (int)(row & (vol - 1));
    const int m = S - 1;
    const int x0 = (v >> (2 * lg)) & m, x1 = (v >> lg) & m, x2 = v & m;
    const int y0 = (x0 + sign * tap_d(t, 0)) & m;
    const int y1 = (x1 + sign * tap_d(t, 1)) & m;
    const int y2 = (x2 + sign * tap_d(t, 2)) & m;
    return b * vol + ((long long)y0 << (2 * lg)) + ((long long)y1 << lg) + y2;
}

template <int N> struct ConvShape {
    static constexpr int kBTileBytes = kChunks * N * kRowBytes;
    static constexpr int kStageBytes = kATileBytes + kBTileBytes;
    static constexpr int kSmem = kStages * kStageBytes + 64;
    static constexpr uint32_t kCols = N <= 32 ? 32 : N <= 64 ? 64 : 128;
    static constexpr uint32_t kIdesc = tc05::idesc_bf16_f32(128, N, 0, 0);
};

// Forward (and dgrad) 3x3x3 convolution.  One CTA walks M tiles
// blockIdx.x, +gridDim.x, ...; the stage sequence runs across tiles, so the
// loads of a tile's first stages overlap the previous tile's epilogue.
template <int N>
__global__ void __launch_bounds__(kThreads) conv3_kernel(ConvArgs a) {
    using Sh = ConvShape<N>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kStages * Sh::kStageBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + kStages);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    const int cpt = a.cin >> 3;                  // 16-byte chunks per tap
    const int Q = 27 * cpt;                      // chunks of K
    const int nst = (Q + kChunks - 1) / kChunks; // stages per tile
    const int tiles = (int)(a.rows >> 7);
    const int my_tiles = tiles > (int)blockIdx.x ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int G = my_tiles * nst;                // stages of this CTA (32-bit: at most 2^31)
    const int lg = a.lg, msk = a.S - 1;
    const int lg2 = 2 * lg, lg3 = 3 * lg;

    if (warp == 0) {
        tc05::tmem_alloc(tslot, Sh::kCols);
        tc05::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) tc05::mbar_init(&mbar[s], 1);
        tc05::mbar_fence_init();
    }
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    const uint32_t tmem = *tslot;

    // Position of the next stage to load (tile ordinal, stage in tile, ring
    // buffer), advanced one stage per call; no divisions in the loop.
    int ld_t = 0, ld_j = 0, ld_s = 0;
    auto load_next = [&]() {
        unsigned char *As = smem + ld_s * Sh::kStageBytes;
        unsigned char *Bs = As + kATileBytes;
        const long long row = ((long long)blockIdx.x + (long long)ld_t * gridDim.x) * 128 + tid;
        const int q0 = ld_j * kChunks, nq = min(kChunks, Q - q0);
        // this thread's row: sample base and coordinates
        const long long base = (row >> lg3) << lg3;
        const int v = (int)(row - base);
        const int x0 = v >> lg2, x1 = (v >> lg) & msk, x2 = v & msk;
        int t = q0 / cpt, c8 = q0 - t * cpt;
        const bf16 *src = nullptr;
        auto at_tap = [&](int tt) {
            const int y0 = (x0 + tt / 9 - 1) & msk, y1 = (x1 + (tt / 3) % 3 - 1) & msk, y2 = (x2 + tt % 3 - 1) & msk;
            const long long nrow = base + ((long long)y0 << lg2) + ((long long)y1 << lg) + y2;
            src = a.in.p + nrow * a.in.cs + a.in.coff;
        };
        at_tap(t);
        for (int c = 0; c < nq; ++c) {
            tc05::cp_async16(As + c * 2048 + (tid >> 3) * 128 + (tid & 7) * 16, src + c8 * 8);
            if (++c8 == cpt) {
                c8 = 0;
                if (++t < 27) at_tap(t);
            }
        }
        // B: n rows x nq chunks of the weights
        const bf16 *wsrc = a.w + q0 * 8;
        for (int idx = tid; idx < N * nq; idx += kThreads) {
            const int n = idx % N, c = idx / N;
            tc05::cp_async16(Bs + c * (N * 16) + (n >> 3) * 128 + (n & 7) * 16, wsrc + (long long)n * (27 * a.cin) + c * 8);
        }
        if (++ld_j == nst) {
            ld_j = 0;
            ++ld_t;
        }
        if (++ld_s == kStages) ld_s = 0;
    };

    for (int g = 0; g < kStages - 1; ++g) {
        if (g < G) load_next();
        tc05::cp_async_commit();
    }
    int j = 0, s = 0, ti = 0;  // the stage in work: stage in tile, ring buffer, tile ordinal
    int ph_prev = 0;           // parity of the commit of stage g - 1 on its buffer
    int s_prev = kStages - 1;
    uint32_t parity_bits = 0;  // bit b: parity of the next commit on buffer b
    for (int g = 0; g < G; ++g) {
        if (g + kStages - 1 < G) {
            if (g >= 1) {
                // the MMAs of stage g-1 read the buffer the next load reuses
                if (!tc05::mbar_wait(&mbar[s_prev], (uint32_t)ph_prev)) atomicOr(&g_error, 1u);
            }
            load_next();
        }
        tc05::cp_async_commit();
        tc05::cp_async_wait<kStages - 1>();
        tc05::fence_proxy_async_smem();
        __syncthreads();
        const uint32_t my_parity = (parity_bits >> s) & 1u;
        if (tid == 0) {
            tc05::fence_after_sync();
            const uint32_t As = tc05::smem_u32(smem + s * Sh::kStageBytes);
            const uint32_t Bs = As + kATileBytes;
            const int nq = min(kChunks, Q - j * kChunks);
            for (int kk = 0; kk < nq / 2; ++kk) {
                const uint64_t ad = tc05::desc_noswizzle(As + kk * 2 * 2048, 2048, 128);
                const uint64_t bd = tc05::desc_noswizzle(Bs + kk * 2 * (N * 16), N * 16, 128);
                tc05::mma_bf16(tmem, ad, bd, Sh::kIdesc, (j > 0 || kk > 0) ? 1u : 0u);
            }
            tc05::mma_commit(&mbar[s]);
        }
        if (j == nst - 1) {
            // tile complete: wait for its MMAs, then the epilogue
            if (!tc05::mbar_wait(&mbar[s], my_parity)) atomicOr(&g_error, 1u);
            tc05::fence_after_sync();
            const long long tile = (long long)blockIdx.x + (long long)ti * gridDim.x;
            const long long row = tile * 128 + warp * 32 + lane;
            bf16 *dst = a.out.p + row * a.out.cs + a.out.coff;
            const bf16 *mk = a.mask.p ? a.mask.p + row * a.mask.cs + a.mask.coff : nullptr;
#pragma unroll
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tc05::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
                if (a.bias) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] += __ldg(a.bias + c0 + i);
                }
                if (a.relu) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.0f);
                }
                if (mk) {
                    const uint4 m0 = *reinterpret_cast<const uint4 *>(mk + c0);
                    const uint4 m1 = *reinterpret_cast<const uint4 *>(mk + c0 + 8);
                    const bf16 *mb0 = reinterpret_cast<const bf16 *>(&m0);
                    const bf16 *mb1 = reinterpret_cast<const bf16 *>(&m1);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        if (!(__bfloat162float(mb0[i]) > 0.0f)) v[i] = 0.0f;
                        if (!(__bfloat162float(mb1[i]) > 0.0f)) v[8 + i] = 0.0f;
                    }
                }
                uint4 o0, o1;
                __nv_bfloat162 *h0 = reinterpret_cast<__nv_bfloat162 *>(&o0);
                __nv_bfloat162 *h1 = reinterpret_cast<__nv_bfloat162 *>(&o1);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    h0[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                    h1[i] = __floats2bfloat162_rn(v[8 + 2 * i], v[8 + 2 * i + 1]);
                }
                *reinterpret_cast<uint4 *>(dst + c0) = o0;
                *reinterpret_cast<uint4 *>(dst + c0 + 8) = o1;
            }
            tc05::fence_before_sync();
        }
        // advance the stage in work
        ph_prev = (int)my_parity;
        s_prev = s;
        parity_bits ^= 1u << s;
        if (++s == kStages) s = 0;
        if (++j == nst) {
            j = 0;
            ++ti;
        }
    }
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    if (warp == 0) tc05::tmem_dealloc(tmem, Sh::kCols);
}

// ---- weight gradient ---------------------------------------------------------
struct WgradArgs {
    Vol dy;
    int cout;
    Vol x;
    int cin;
    float *dw;       // [cout][27][cin], accumulated
    int S, lg;
    long long rows;  // batch * S^3
    long long kv;    // voxels per CTA (multiple of 64)
};

template <int N> struct WgradShape {
    static constexpr int kBTileBytes = kChunks * N * kRowBytes;
    static constexpr int kStageBytes = kATileBytes + kBTileBytes;
    static constexpr int kSmem = kStages * kStageBytes + 64;
    static constexpr uint32_t kCols = N <= 32 ? 32 : N <= 64 ? 64 : 128;
    static constexpr uint32_t kIdesc = tc05::idesc_bf16_f32(128, N, 1, 1);
};

// D[(tap,co)][ci] over the voxels [blockIdx.y*kv, +kv), rows of the M tile
// blockIdx.x; both operands MN-major (a 16-byte load is 8 consecutive
// channels of one voxel), K = voxels in stages of 64.
template <int N>
__global__ void __launch_bounds__(kThreads) wgrad_kernel(WgradArgs a) {
    using Sh = WgradShape<N>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kStages * Sh::kStageBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + kStages);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m_total = 27 * a.cout;
    const long long u_begin = (long long)blockIdx.y * a.kv;
    const long long u_end = min(a.rows, u_begin + a.kv);
    const int G = (int)((u_end - u_begin) / 64);

    if (warp == 0) {
        tc05::tmem_alloc(tslot, Sh::kCols);
        tc05::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) tc05::mbar_init(&mbar[s], 1);
        tc05::mbar_fence_init();
    }
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    const uint32_t tmem = *tslot;

    // This thread's eight row groups of the M tile: tap offset (negated) and
    // channel offset, fixed for the CTA; -1: a padding group (zeros).
    const int msk = a.S - 1, lg = a.lg, lg2 = 2 * a.lg, lg3 = 3 * a.lg;
    int goff[8], gco[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int m = blockIdx.x * 128 + ((tid >> 6) + 2 * i) * 8;
        if (m < m_total) {
            const int t = m / a.cout;
            gco[i] = m - t * a.cout;
            goff[i] = t;
        } else {
            gco[i] = -1;
            goff[i] = 0;
        }
    }
    int ld_s = 0;
    long long ld_u = u_begin + (tid & 63);  // this thread's voxel of the next stage to load
    auto load_next = [&]() {
        unsigned char *As = smem + ld_s * Sh::kStageBytes;
        unsigned char *Bs = As + kATileBytes;
        const int k = tid & 63;
        const int kg = k >> 3, k8 = k & 7;
        const long long u = ld_u;
        const long long base = (u >> lg3) << lg3;
        const int v = (int)(u - base);
        const int x0 = v >> lg2, x1 = (v >> lg) & msk, x2 = v & msk;
        // A: 8 of the 16 groups of 8 rows (tap, co..co+7) at voxel u - off(tap)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int mg = (tid >> 6) + 2 * i;
            unsigned char *dst = As + kg * 2048 + mg * 128 + k8 * 16;
            if (gco[i] >= 0) {
                const int t = goff[i];
                const int y0 = (x0 - (t / 9 - 1)) & msk, y1 = (x1 - ((t / 3) % 3 - 1)) & msk,
                          y2 = (x2 - (t % 3 - 1)) & msk;
                const long long nrow = base + ((long long)y0 << lg2) + ((long long)y1 << lg) + y2;
                tc05::cp_async16(dst, a.dy.p + nrow * a.dy.cs + a.dy.coff + gco[i]);
            } else {
                tc05::cp_async16_zfill(dst, a.dy.p, 0);
            }
        }
        // B: N/8 groups of 8 input channels at voxel u
        const bf16 *xs = a.x.p + u * a.x.cs + a.x.coff;
        for (int ng = tid >> 6; ng < N / 8; ng += 2)
            tc05::cp_async16(Bs + kg * (N * 16) + ng * 128 + k8 * 16, xs + ng * 8);
        ld_u += 64;
        if (++ld_s == kStages) ld_s = 0;
    };

    for (int g = 0; g < kStages - 1; ++g) {
        if (g < G) load_next();
        tc05::cp_async_commit();
    }
    int s = 0, s_prev = kStages - 1;
    uint32_t parity_bits = 0, ph_prev = 0;
    for (int g = 0; g < G; ++g) {
        if (g + kStages - 1 < G) {
            if (g >= 1) {
                if (!tc05::mbar_wait(&mbar[s_prev], ph_prev)) atomicOr(&g_error, 2u);
            }
            load_next();
        }
        tc05::cp_async_commit();
        tc05::cp_async_wait<kStages - 1>();
        tc05::fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc05::fence_after_sync();
            const uint32_t As = tc05::smem_u32(smem + s * Sh::kStageBytes);
            const uint32_t Bs = As + kATileBytes;
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t ad = tc05::desc_noswizzle(As + kk * 2 * 2048, 2048, 128);
                const uint64_t bd = tc05::desc_noswizzle(Bs + kk * 2 * (N * 16), N * 16, 128);
                tc05::mma_bf16(tmem, ad, bd, Sh::kIdesc, (g > 0 || kk > 0) ? 1u : 0u);
            }
            tc05::mma_commit(&mbar[s]);
        }
        ph_prev = (parity_bits >> s) & 1u;
        s_prev = s;
        parity_bits ^= 1u << s;
        if (++s == kStages) s = 0;
    }
    if (G > 0) {
        // the last stage's commit: buffer s_prev, parity ph_prev
        if (!tc05::mbar_wait(&mbar[s_prev], ph_prev)) atomicOr(&g_error, 2u);
        tc05::fence_after_sync();
        const int m = blockIdx.x * 128 + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc05::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
            if (m < m_total) {
                const int t = m / a.cout, co = m - t * a.cout;
                float *d = a.dw + ((long long)co * 27 + t) * a.cin + c0;
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(d + i, v[i]);
            }
        }
    }
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    if (warp == 0) tc05::tmem_dealloc(tmem, Sh::kCols);
}

// ---- element-wise and small kernels (CUDA cores) -----------------------------

__device__ __forceinline__ long long vox_index(long long b, int x0, int x1, int x2, int lg) {
    return (b << (3 * lg)) + ((long long)x0 << (2 * lg)) + ((long long)x1 << lg) + x2;
}

// 2x2x2 average pool: out[B][S/2] <- in[B][S], C channels (multiple of 8).
__global__ void pool2_kernel(Vol in, VolOut out, int C, int lg_out, long long rows_out) {
    const int C8 = C >> 3;
    const long long total = rows_out * C8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / C8;
        const int c8 = (int)(i - r * C8);
        const int m = (1 << lg_out) - 1;
        const long long b = r >> (3 * lg_out);
        const int v = (int)(r & ((1ll << (3 * lg_out)) - 1));
        const int x0 = v >> (2 * lg_out), x1 = (v >> lg_out) & m, x2 = v & m;
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 8; ++d) {
            const long long src = vox_index(b, 2 * x0 + (d >> 2), 2 * x1 + ((d >> 1) & 1), 2 * x2 + (d & 1),
                                            lg_out + 1);
            const uint4 u = *reinterpret_cast<const uint4 *>(in.p + src * in.cs + in.coff + c8 * 8);
            const bf16 *h = reinterpret_cast<const bf16 *>(&u);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += __bfloat162float(h[k]);
        }
        uint4 o;
        __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
        for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(0.125f * acc[2 * k], 0.125f * acc[2 * k + 1]);
        *reinterpret_cast<uint4 *>(out.p + r * out.cs + out.coff + c8 * 8) = o;
    }
}

// Backward of pool2 fused with the skip gradient and the ReLU mask of the
// pooled activation: out[child] = (skip[child] + dy[parent] / 8) * (act[child] > 0).
__global__ void pool2_bwd_kernel(Vol dy, Vol skip, Vol act, VolOut out, int C, int lg_in, long long rows_in) {
    const int C8 = C >> 3;
    const long long total = rows_in * C8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / C8;
        const int c8 = (int)(i - r * C8);
        const int m = (1 << lg_in) - 1;
        const long long b = r >> (3 * lg_in);
        const int v = (int)(r & ((1ll << (3 * lg_in)) - 1));
        const int x0 = v >> (2 * lg_in), x1 = (v >> lg_in) & m, x2 = v & m;
        const long long p = vox_index(b, x0 >> 1, x1 >> 1, x2 >> 1, lg_in - 1);
        const uint4 ud = *reinterpret_cast<const uint4 *>(dy.p + p * dy.cs + dy.coff + c8 * 8);
        const uint4 ua = *reinterpret_cast<const uint4 *>(act.p + r * act.cs + act.coff + c8 * 8);
        uint4 us = make_uint4(0, 0, 0, 0);
        if (skip.p) us = *reinterpret_cast<const uint4 *>(skip.p + r * skip.cs + skip.coff + c8 * 8);
        const bf16 *hd = reinterpret_cast<const bf16 *>(&ud);
        const bf16 *ha = reinterpret_cast<const bf16 *>(&ua);
        const bf16 *hs = reinterpret_cast<const bf16 *>(&us);
        float o[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float g = __bfloat162float(hs[k]) + 0.125f * __bfloat162float(hd[k]);
            o[k] = __bfloat162float(ha[k]) > 0.0f ? g : 0.0f;
        }
        uint4 w;
        __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&w);
#pragma unroll
        for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(o[2 * k], o[2 * k + 1]);
        *reinterpret_cast<uint4 *>(out.p + r * out.cs + out.coff + c8 * 8) = w;
    }
}

// Nearest 2x upsampling: out[child] = in[parent].
__global__ void up2_kernel(Vol in, VolOut out, int C, int lg_out, long long rows_out) {
    const int C8 = C >> 3;
    const long long total = rows_out * C8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / C8;
        const int c8 = (int)(i - r * C8);
        const int m = (1 << lg_out) - 1;
        const long long b = r >> (3 * lg_out);
        const int v = (int)(r & ((1ll << (3 * lg_out)) - 1));
        const int x0 = v >> (2 * lg_out), x1 = (v >> lg_out) & m, x2 = v & m;
        const long long p = vox_index(b, x0 >> 1, x1 >> 1, x2 >> 1, lg_out - 1);
        *reinterpret_cast<uint4 *>(out.p + r * out.cs + out.coff + c8 * 8) =
            *reinterpret_cast<const uint4 *>(in.p + p * in.cs + in.coff + c8 * 8);
    }
}

// Backward of up2: out[parent] = sum over its 8 children of dy[child],
// times (act[parent] > 0) when act is given (the ReLU of the upsampled input).
__global__ void up2_bwd_kernel(Vol dy, Vol act, VolOut out, int C, int lg_out, long long rows_out) {
    const int C8 = C >> 3;
    const long long total = rows_out * C8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / C8;
        const int c8 = (int)(i - r * C8);
        const int m = (1 << lg_out) - 1;
        const long long b = r >> (3 * lg_out);
        const int v = (int)(r & ((1ll << (3 * lg_out)) - 1));
        const int x0 = v >> (2 * lg_out), x1 = (v >> lg_out) & m, x2 = v & m;
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 8; ++d) {
            const long long src = vox_index(b, 2 * x0 + (d >> 2), 2 * x1 + ((d >> 1) & 1), 2 * x2 + (d & 1),
                                            lg_out + 1);
            const uint4 u = *reinterpret_cast<const uint4 *>(dy.p + src * dy.cs + dy.coff + c8 * 8);
            const bf16 *h = reinterpret_cast<const bf16 *>(&u);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += __bfloat162float(h[k]);
        }
        if (act.p) {
            const uint4 ua = *reinterpret_cast<const uint4 *>(act.p + r * act.cs + act.coff + c8 * 8);
            const bf16 *ha = reinterpret_cast<const bf16 *>(&ua);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (!(__bfloat162float(ha[k]) > 0.0f)) acc[k] = 0.0f;
        }
        uint4 w;
        __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&w);
#pragma unroll
        for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(acc[2 * k], acc[2 * k + 1]);
        *reinterpret_cast<uint4 *>(out.p + r * out.cs + out.coff + c8 * 8) = w;
    }
}

// Per-channel sum of a gradient volume (the bias gradient), fp32 atomics of
// block partial sums.  C <= 128.
__global__ void bias_grad_kernel(Vol dy, int C, long long rows, float *db) {
    __shared__ float part[128];
    for (int c = threadIdx.x; c < C; c += blockDim.x) part[c] = 0.0f;
    __syncthreads();
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;  // rows handled in parallel by a block
    float acc = 0.0f;
    if ((int)threadIdx.x < lanes * C)
        for (long long r = blockIdx.x * (long long)lanes + threadIdx.x / C; r < rows;
             r += (long long)gridDim.x * lanes)
            acc += __bfloat162float(dy.p[r * dy.cs + dy.coff + c]);
    atomicAdd(&part[c], acc);
    __syncthreads();
    for (int k = threadIdx.x; k < C; k += blockDim.x) atomicAdd(&db[k], part[k]);
}

// Input features: channel 0 = 1 in an empty voxel, channel 1 = the sample's
// feature (log10 Knudsen number), channels 2..15 = 0.
__global__ void pack_input_kernel(const uint8_t *solid, const float *feature, bf16 *out, int lg, long long rows) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
         r += (long long)gridDim.x * blockDim.x) {
        const long long b = r >> (3 * lg);
        uint4 o0 = make_uint4(0, 0, 0, 0), o1 = make_uint4(0, 0, 0, 0);
        __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&o0);
        h[0] = __floats2bfloat162_rn(solid[r] ? 0.0f : 1.0f, feature[b]);
        *reinterpret_cast<uint4 *>(out + r * 16) = o0;
        *reinterpret_cast<uint4 *>(out + r * 16 + 8) = o1;
    }
}

// Head: 1x1x1 convolution 16 -> 4 in fp32, out[r][c] = bh[c] + sum_k wh[c][k] e[r][k].
__global__ void head_kernel(Vol e, const float *wh, const float *bh, float *out, long long rows) {
    __shared__ float w[64 + 4];
    if (threadIdx.x < 64) w[threadIdx.x] = wh[threadIdx.x];
    if (threadIdx.x < 4) w[64 + threadIdx.x] = bh[threadIdx.x];
    __syncthreads();
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
         r += (long long)gridDim.x * blockDim.x) {
        float x[16];
        const uint4 u0 = *reinterpret_cast<const uint4 *>(e.p + r * e.cs + e.coff);
        const uint4 u1 = *reinterpret_cast<const uint4 *>(e.p + r * e.cs + e.coff + 8);
        const bf16 *h0 = reinterpret_cast<const bf16 *>(&u0);
        const bf16 *h1 = reinterpret_cast<const bf16 *>(&u1);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            x[k] = __bfloat162float(h0[k]);
            x[8 + k] = __bfloat162float(h1[k]);
        }
        float4 o;
        float *op = &o.x;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float s = w[64 + c];
#pragma unroll
            for (int k = 0; k < 16; ++k) s += w[c * 16 + k] * x[k];
            op[c] = s;
        }
        *reinterpret_cast<float4 *>(out + r * 4) = o;
    }
}

// Masked weighted squared error of the head output and its backward through
// the head: per row r with valid[r] != 0,
//   loss += sum_c cw[c] (out[r][c] - tgt[r][c])^2 / count,
//   dout  = 2 cw (out - tgt) / count,
//   dwh  += dout (x) e[r],  dbh += dout,
//   de[r][k] = (sum_c wh[c][k] dout[c]) * (e[r][k] > 0)   (bf16).
__global__ void loss_head_bwd_kernel(const float *out, const float *tgt, const uint8_t *valid, const float *cw,
                                     float inv_count, Vol e, const float *wh, float *dwh, float *dbh,
                                     VolOut de, double *loss, long long rows, const double *coef, int coef_ch,
                                     int lg) {
    __shared__ float w[64];
    __shared__ float gw[64 + 4];
    __shared__ double ls;
    if (threadIdx.x < 64) w[threadIdx.x] = wh[threadIdx.x];
    if (threadIdx.x < 68) gw[threadIdx.x] = 0.0f;
    if (threadIdx.x == 0) ls = 0.0;
    __syncthreads();
    float lgw[68];
#pragma unroll
    for (int i = 0; i < 68; ++i) lgw[i] = 0.0f;
    double lloss = 0.0;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
         r += (long long)gridDim.x * blockDim.x) {
        float d[4] = {0, 0, 0, 0};
        if (valid[r]) {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float diff = out[r * 4 + c] - tgt[r * 4 + c];
                lloss += (double)(cw[c] * diff * diff * inv_count);
                d[c] = 2.0f * cw[c] * diff * inv_count;
            }
            if (coef) d[coef_ch] += (float)coef[r >> (3 * lg)];
        }
        float x[16];
        const uint4 u0 = *reinterpret_cast<const uint4 *>(e.p + r * e.cs + e.coff);
        const uint4 u1 = *reinterpret_cast<const uint4 *>(e.p + r * e.cs + e.coff + 8);
        const bf16 *h0 = reinterpret_cast<const bf16 *>(&u0);
        const bf16 *h1 = reinterpret_cast<const bf16 *>(&u1);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            x[k] = __bfloat162float(h0[k]);
            x[8 + k] = __bfloat162float(h1[k]);
        }
        float g[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            float s = 0.0f;
#pragma unroll
            for (int c = 0; c < 4; ++c) s += w[c * 16 + k] * d[c];
            g[k] = x[k] > 0.0f ? s : 0.0f;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
#pragma unroll
            for (int k = 0; k < 16; ++k) lgw[c * 16 + k] += d[c] * x[k];
            lgw[64 + c] += d[c];
        }
        uint4 o0, o1;
        __nv_bfloat162 *q0 = reinterpret_cast<__nv_bfloat162 *>(&o0);
        __nv_bfloat162 *q1 = reinterpret_cast<__nv_bfloat162 *>(&o1);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            q0[k] = __floats2bfloat162_rn(g[2 * k], g[2 * k + 1]);
            q1[k] = __floats2bfloat162_rn(g[8 + 2 * k], g[8 + 2 * k + 1]);
        }
        *reinterpret_cast<uint4 *>(de.p + r * de.cs + de.coff) = o0;
        *reinterpret_cast<uint4 *>(de.p + r * de.cs + de.coff + 8) = o1;
    }
    // block reduction of the head gradients and the loss
#pragma unroll
    for (int i = 0; i < 68; ++i) {
        float v = lgw[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&gw[i], v);
    }
    for (int o = 16; o > 0; o >>= 1) lloss += __shfl_xor_sync(0xffffffffu, lloss, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&ls, lloss);
    __syncthreads();
    if (threadIdx.x < 64) atomicAdd(&dwh[threadIdx.x], gw[threadIdx.x]);
    if (threadIdx.x < 4) atomicAdd(&dbh[threadIdx.x], gw[64 + threadIdx.x]);
    if (threadIdx.x == 0) atomicAdd(loss, ls);
}

// Per-sample sums over the valid rows of out[r][ch] - tgt[r][ch] and of the
// valid rows themselves: acc[2b], acc[2b + 1] (fp64 atomics of block sums).
// blockIdx.y = sample.
__global__ void sample_diff_kernel(const float *out, const float *tgt, const uint8_t *valid, int ch,
                                   long long rows_per_sample, double *acc) {
    __shared__ double part[2];
    if (threadIdx.x < 2) part[threadIdx.x] = 0.0;
    __syncthreads();
    const long long b = blockIdx.y;
    double sd = 0.0, sn = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < rows_per_sample;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = b * rows_per_sample + i;
        if (valid[r]) {
            sd += (double)(out[r * 4 + ch] - tgt[r * 4 + ch]);
            sn += 1.0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sd += __shfl_xor_sync(0xffffffffu, sd, o);
        sn += __shfl_xor_sync(0xffffffffu, sn, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&part[0], sd);
        atomicAdd(&part[1], sn);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&acc[2 * b], part[0]);
        atomicAdd(&acc[2 * b + 1], part[1]);
    }
}

// The per-sample mean term: loss += w * sum_b m_b^2 / B with m_b the mean of
// out - tgt over sample b's valid rows; coef[b] = 2 w m_b / (n_b B) is its
// derivative with respect to each of those rows' outputs.
__global__ void sample_flux_finish_kernel(const double *acc, int batch, float w, double *coef, double *loss) {
    double l = 0.0;
    for (int b = threadIdx.x; b < batch; b += blockDim.x) {
        const double n = acc[2 * b + 1] > 0.0 ? acc[2 * b + 1] : 1.0;
        const double m = acc[2 * b] / n;
        coef[b] = 2.0 * (double)w * m / (n * (double)batch);
        l += (double)w * m * m / (double)batch;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// Adam with bias correction on n fp32 parameters.
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// fp32 master weights [cout][27][cin] -> bf16 forward copy (same layout) and
// dgrad copy wd[ci][t][co] = w[co][26 - t][ci].
__global__ void pack_weights_kernel(const float *w, int cout, int cin, bf16 *wf, bf16 *wd) {
    const long long n = (long long)cout * 27 * cin;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int ci = (int)(i % cin);
        const int t = (int)((i / cin) % 27);
        const int co = (int)(i / (27ll * cin));
        const bf16 h = __float2bfloat16_rn(w[i]);
        wf[i] = h;
        if (wd) wd[((long long)ci * 27 + (26 - t)) * cout + co] = h;
    }
}

int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    if (g > 148 * 16) g = 148 * 16;
    return (int)(g < 1 ? 1 : g);
}

template <int N> cudaError_t launch_conv(const ConvArgs &a, cudaStream_t st) {
    using Sh = ConvShape<N>;
    cudaError_t e = cudaFuncSetAttribute(conv3_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::kSmem);
    if (e != cudaSuccess) return e;
    // two resident CTAs per SM, persistent over the M tiles: three or four
    // (as shared memory would allow at N <= 64) measured slower, the gathers
    // of more CTAs contending for L2 (c1c forward 2.0 -> 2.5 ms at four)
    int per_sm = 0, dev = 0, sms = 148;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, conv3_kernel<N>, kThreads, Sh::kSmem);
    if (e != cudaSuccess) return e;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    per_sm = per_sm < 1 ? 1 : (per_sm > 2 ? 2 : per_sm);
    const long long tiles = a.rows >> 7;
    const long long cap = (long long)per_sm * sms;
    const int grid = (int)(tiles < cap ? tiles : cap);
    conv3_kernel<N><<<grid, kThreads, Sh::kSmem, st>>>(a);
    return cudaGetLastError();
}

template <int N> cudaError_t launch_wgrad(const WgradArgs &a0, cudaStream_t st) {
    using Sh = WgradShape<N>;
    cudaError_t e = cudaFuncSetAttribute(wgrad_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::kSmem);
    if (e != cudaSuccess) return e;
    WgradArgs a = a0;
    const int mtiles = (27 * a.cout + 127) / 128;
    // about four CTAs per SM over all M tiles, at least 512 voxels each
    long long per = (a.rows * mtiles) / (148 * 4);
    per = ((per + 63) / 64) * 64;
    if (per < 512) per = 512;
    if (per > a.rows) per = a.rows;
    a.kv = per;
    const long long ks = (a.rows + per - 1) / per;
    dim3 grid(mtiles, (unsigned)ks);
    wgrad_kernel<N><<<grid, kThreads, Sh::kSmem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace sg

using namespace sg;

namespace {

int lg2_of(int S) {
    int lg = 0;
    while ((1 << lg) < S) ++lg;
    return (1 << lg) == S ? lg : -1;
}

int sg_fail(int code, const std::string &msg) {
    dsmc::set_thread_error("surrogate: " + msg);
    return code;
}

int cuda_rc(cudaError_t e) {
    if (e == cudaSuccess) return DSMC_OK;
    return sg_fail(DSMC_ERR_CUDA, cudaGetErrorString(e));
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

extern "C" {

int dsmc_sg_conv3(void *stream, int batch, int S, const uint16_t *in, int in_cs, int in_coff, int cin,
                  const uint16_t *w, const float *bias, int cout, uint16_t *out, int out_cs, int out_coff, int relu,
                  const uint16_t *mask, int mask_cs, int mask_coff) {
    const int lg = lg2_of(S);
    if (lg < 2 || batch < 1 || !in || !w || !out || (((long long)batch << (3 * lg)) & 127))
        return sg_fail(DSMC_ERR_ARG, "conv3: bad shape (S a power of two >= 4, batch*S^3 a multiple of 128) or pointer");
    if (cin % 16 || cin < 16 || cin > 256 || in_cs % 8 || in_coff % 8 || out_cs % 8 || out_coff % 8 ||
        (mask && (mask_cs % 8 || mask_coff % 8 || mask_coff + cout > mask_cs)) || in_coff + cin > in_cs ||
        out_coff + cout > out_cs)
        return sg_fail(DSMC_ERR_ARG, "conv3: channels, strides and offsets must be multiples of 8 (cin of 16)");
    if (!aligned16(in) || !aligned16(w) || !aligned16(out) || (mask && !aligned16(mask)))
        return sg_fail(DSMC_ERR_ARG, "conv3: tensors must be 16-byte aligned");
    ConvArgs a;
    a.in = {reinterpret_cast<const bf16 *>(in), in_cs, in_coff};
    a.cin = cin;
    a.w = reinterpret_cast<const bf16 *>(w);
    a.bias = bias;
    a.out = {reinterpret_cast<bf16 *>(out), out_cs, out_coff};
    a.mask = {reinterpret_cast<const bf16 *>(mask), mask_cs, mask_coff};
    a.relu = relu;
    a.S = S;
    a.lg = lg;
    a.rows = (long long)batch << (3 * lg);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (cout) {
    case 16: return cuda_rc(launch_conv<16>(a, st));
    case 32: return cuda_rc(launch_conv<32>(a, st));
    case 48: return cuda_rc(launch_conv<48>(a, st));
    case 64: return cuda_rc(launch_conv<64>(a, st));
    case 96: return cuda_rc(launch_conv<96>(a, st));
    default: return sg_fail(DSMC_ERR_ARG, "conv3: output channels must be 16, 32, 48, 64 or 96");
    }
}

int dsmc_sg_conv3_wgrad(void *stream, int batch, int S, const uint16_t *dy, int dy_cs, int dy_coff, int cout,
                        const uint16_t *x, int x_cs, int x_coff, int cin, float *dw) {
    const int lg = lg2_of(S);
    if (lg < 2 || batch < 1 || !dy || !x || !dw || (((long long)batch << (3 * lg)) & 63))
        return sg_fail(DSMC_ERR_ARG, "wgrad: bad shape (S a power of two >= 4, batch*S^3 a multiple of 64) or pointer");
    if (cout % 16 || cout < 16 || cout > 256 || dy_cs % 8 || dy_coff % 8 || x_cs % 8 || x_coff % 8 ||
        dy_coff + cout > dy_cs || x_coff + cin > x_cs)
        return sg_fail(DSMC_ERR_ARG, "wgrad: channels, strides and offsets must be multiples of 8 (cout of 16)");
    if (!aligned16(dy) || !aligned16(x)) return sg_fail(DSMC_ERR_ARG, "wgrad: tensors must be 16-byte aligned");
    WgradArgs a;
    a.dy = {reinterpret_cast<const bf16 *>(dy), dy_cs, dy_coff};
    a.cout = cout;
    a.x = {reinterpret_cast<const bf16 *>(x), x_cs, x_coff};
    a.cin = cin;
    a.dw = dw;
    a.S = S;
    a.lg = lg;
    a.rows = (long long)batch << (3 * lg);
    a.kv = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (cin) {
    case 16: return cuda_rc(launch_wgrad<16>(a, st));
    case 32: return cuda_rc(launch_wgrad<32>(a, st));
    case 48: return cuda_rc(launch_wgrad<48>(a, st));
    case 64: return cuda_rc(launch_wgrad<64>(a, st));
    case 96: return cuda_rc(launch_wgrad<96>(a, st));
    default: return sg_fail(DSMC_ERR_ARG, "wgrad: input channels must be 16, 32, 48, 64 or 96");
    }
}

int dsmc_sg_bias_grad(void *stream, int batch, int S, const uint16_t *dy, int dy_cs, int dy_coff, int c,
                      float *db) {
    const int lg = lg2_of(S);
    if (lg < 1 || !dy || !db || c < 1 || c > 128) return sg_fail(DSMC_ERR_ARG, "bias_grad: bad argument");
    const long long rows = (long long)batch << (3 * lg);
    bias_grad_kernel<<<grid_for(rows, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        {reinterpret_cast<const bf16 *>(dy), dy_cs, dy_coff}, c, rows, db);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_pool2(void *stream, int batch, int S, const uint16_t *in, int in_cs, int in_coff, int c, uint16_t *out,
                  int out_cs, int out_coff) {
    const int lg = lg2_of(S);
    if (lg < 1 || c % 8 || !in || !out) return sg_fail(DSMC_ERR_ARG, "pool2: bad argument");
    const long long rows = (long long)batch << (3 * (lg - 1));
    pool2_kernel<<<grid_for(rows * (c / 8), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        {reinterpret_cast<const bf16 *>(in), in_cs, in_coff}, {reinterpret_cast<bf16 *>(out), out_cs, out_coff}, c,
        lg - 1, rows);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_pool2_bwd(void *stream, int batch, int S, const uint16_t *dy, int dy_cs, int dy_coff,
                      const uint16_t *skip, int skip_cs, int skip_coff, const uint16_t *act, int act_cs, int act_coff,
                      int c, uint16_t *out, int out_cs, int out_coff) {
    const int lg = lg2_of(S);
    if (lg < 1 || c % 8 || !dy || !act || !out) return sg_fail(DSMC_ERR_ARG, "pool2_bwd: bad argument");
    const long long rows = (long long)batch << (3 * lg);
    pool2_bwd_kernel<<<grid_for(rows * (c / 8), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        {reinterpret_cast<const bf16 *>(dy), dy_cs, dy_coff}, {reinterpret_cast<const bf16 *>(skip), skip_cs, skip_coff},
        {reinterpret_cast<const bf16 *>(act), act_cs, act_coff}, {reinterpret_cast<bf16 *>(out), out_cs, out_coff}, c,
        lg, rows);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_up2(void *stream, int batch, int S, const uint16_t *in, int in_cs, int in_coff, int c, uint16_t *out,
                int out_cs, int out_coff) {
    const int lg = lg2_of(S);
    if (lg < 1 || c % 8 || !in || !out) return sg_fail(DSMC_ERR_ARG, "up2: bad argument");
    const long long rows = (long long)batch << (3 * lg);
    up2_kernel<<<grid_for(rows * (c / 8), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        {reinterpret_cast<const bf16 *>(in), in_cs, in_coff}, {reinterpret_cast<bf16 *>(out), out_cs, out_coff}, c, lg,
        rows);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_up2_bwd(void *stream, int batch, int S, const uint16_t *dy, int dy_cs, int dy_coff, const uint16_t *act,
                    int act_cs, int act_coff, int c, uint16_t *out, int out_cs, int out_coff) {
    const int lg = lg2_of(S);
    if (lg < 1 || c % 8 || !dy || !out) return sg_fail(DSMC_ERR_ARG, "up2_bwd: bad argument");
    const long long rows = (long long)batch << (3 * (lg - 1));
    up2_bwd_kernel<<<grid_for(rows * (c / 8), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        {reinterpret_cast<const bf16 *>(dy), dy_cs, dy_coff}, {reinterpret_cast<const bf16 *>(act), act_cs, act_coff},
        {reinterpret_cast<bf16 *>(out), out_cs, out_coff}, c, lg - 1, rows);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_pack_input(void *stream, int batch, int S, const uint8_t *solid, const float *feature, uint16_t *out) {
    const int lg = lg2_of(S);
    if (lg < 1 || !solid || !feature || !out) return sg_fail(DSMC_ERR_ARG, "pack_input: bad argument");
    const long long rows = (long long)batch << (3 * lg);
    pack_input_kernel<<<grid_for(rows, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        solid, feature, reinterpret_cast<bf16 *>(out), lg, rows);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_head(void *stream, int batch, int S, const uint16_t *e, int e_cs, int e_coff, const float *wh,
                 const float *bh, float *out) {
    const int lg = lg2_of(S);
    if (lg < 1 || !e || !wh || !bh || !out) return sg_fail(DSMC_ERR_ARG, "head: bad argument");
    const long long rows = (long long)batch << (3 * lg);
    head_kernel<<<grid_for(rows, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        {reinterpret_cast<const bf16 *>(e), e_cs, e_coff}, wh, bh, out, rows);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_loss_head_bwd(void *stream, int batch, int S, const float *out, const float *target,
                          const uint8_t *valid, const float *channel_weight, float inv_count, const uint16_t *e,
                          int e_cs, int e_coff, const float *wh, float *dwh, float *dbh, uint16_t *de, int de_cs,
                          int de_coff, double *loss, const double *sample_coef, int coef_channel) {
    const int lg = lg2_of(S);
    if (lg < 1 || !out || !target || !valid || !channel_weight || !e || !wh || !dwh || !dbh || !de || !loss ||
        coef_channel < 0 || coef_channel > 3)
        return sg_fail(DSMC_ERR_ARG, "loss_head_bwd: bad argument");
    const long long rows = (long long)batch << (3 * lg);
    loss_head_bwd_kernel<<<grid_for(rows, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        out, target, valid, channel_weight, inv_count, {reinterpret_cast<const bf16 *>(e), e_cs, e_coff}, wh, dwh, dbh,
        {reinterpret_cast<bf16 *>(de), de_cs, de_coff}, loss, rows, sample_coef, coef_channel, lg);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_sample_flux_loss(void *stream, int batch, int S, const float *out, const float *target,
                             const uint8_t *valid, int channel, float weight, double *work, double *coef,
                             double *loss) {
    const int lg = lg2_of(S);
    if (lg < 1 || batch < 1 || batch > 1024 || channel < 0 || channel > 3 || !out || !target || !valid || !work ||
        !coef || !loss)
        return sg_fail(DSMC_ERR_ARG, "sample_flux_loss: bad argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(work, 0, 2 * (size_t)batch * sizeof(double), st);
    if (e != cudaSuccess) return cuda_rc(e);
    const long long per = 1ll << (3 * lg);
    dim3 grid((unsigned)std::max<long long>(1, std::min<long long>((per + 255) / 256, 256)), (unsigned)batch);
    sample_diff_kernel<<<grid, 256, 0, st>>>(out, target, valid, channel, per, work);
    sample_flux_finish_kernel<<<1, 256, 0, st>>>(work, batch, weight, coef, loss);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_adam(void *stream, float *param, const float *grad, float *m, float *v, int64_t n, float lr, float beta1,
                 float beta2, float eps, int64_t step) {
    if (!param || !grad || !m || !v || n < 0 || step < 1) return sg_fail(DSMC_ERR_ARG, "adam: bad argument");
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(param, grad, m, v, n, lr, beta1,
                                                                                  beta2, eps, c1, c2);
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_pack_weights(void *stream, const float *w, int cout, int cin, uint16_t *w_fwd, uint16_t *w_dgrad) {
    if (!w || !w_fwd || cout < 1 || cin < 1) return sg_fail(DSMC_ERR_ARG, "pack_weights: bad argument");
    const long long n = (long long)cout * 27 * cin;
    pack_weights_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, cout, cin, reinterpret_cast<bf16 *>(w_fwd), reinterpret_cast<bf16 *>(w_dgrad));
    return cuda_rc(cudaGetLastError());
}

int dsmc_sg_status(unsigned *error_flags, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_error, sizeof(v));
    if (e != cudaSuccess) return cuda_rc(e);
    if (error_flags) *error_flags = v;
    if (clear && v) {
        const unsigned z = 0;
        e = cudaMemcpyToSymbol(g_error, &z, sizeof(z));
        if (e != cudaSuccess) return cuda_rc(e);
    }
    return DSMC_OK;
}

}  // extern "C"
