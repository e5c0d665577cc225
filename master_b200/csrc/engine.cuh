// The DSMC timestep kernels, templated on the precision policy.
//
// One kernel, `pass_kernel`, walks every active cell of every system (one warp
// per cell, persistent grid) and, depending on its mode flags, performs
//   collide (NTC, dsmc/cell.cpp:42-111) -> sample (cell moments)
//   -> accelerate (dsmc/system.cpp:133-144) -> move with diffuse walls
//      (dsmc/moleculemover.cpp:50-126) -> periodic wrap + flux tally
//      (dsmc/moleculemover.h:29-38) -> re-bin into the new cell
//      (dsmc/system.cpp:146-157)
// on the cell's particles.  The fused production pass does all of them in one
// read and one write of every particle.  The same device functions serve the
// stand-alone stage passes.
//
// Included by kernels_split.cu (fp32 state, FMA allowed) and by
// kernels_fp64.cu (the reference's fp64 arithmetic; built with -fmad=false so
// every product and sum rounds as the reference's x86-64 build does).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dsmc_layout.h"
#include "dsmc_philox.cuh"

namespace dsmc {

enum PassMode { MODE_FUSED = 0, MODE_INPLACE = 1, MODE_SORT = 2 };

__device__ __forceinline__ float one_minus_ulp() { return __int_as_float(0x3f7fffff); }

__device__ __forceinline__ int wrap_index(int c, int n) {
    if (c >= 0 && c < n) return c;
    if (c >= -n && c < 2 * n) return c < 0 ? c + n : c - n;
    int x = c % n;
    return x < 0 ? x + n : x;
}

__device__ __forceinline__ uint32_t voxel_linear(const SysDev &g, int i, int j, int k) {
    return ((uint32_t)wrap_index(i, g.n[0]) * (uint32_t)g.n[1] + (uint32_t)wrap_index(j, g.n[1])) *
               (uint32_t)g.n[2] +
           (uint32_t)wrap_index(k, g.n[2]);
}

__device__ __forceinline__ int voxel_type(const SysDev &g, int i, int j, int k) {
    return __ldg(g.vox + voxel_linear(g, i, j, k));
}

struct MoveTally {
    int wall_hits, reseeds;
    int cross[3];
    unsigned err;
};

// ============================================================================
// Split precision: int voxel + fp32 offset in [0,1) voxel units, fp32 velocity.
// ============================================================================
// ---- wall models besides the diffuse wall ----------------------------------
// ColliderSpecular (dsmc/colliderspecular.cpp:8-32) and
// ColliderCercignaniLampis (dsmc/collidercercignanilampis.cpp:13-45) with
// Random::next_cercignani_lampis_normal_component (dsmc/random.cpp:70-91).

// Modified Bessel function I0 by the polynomial approximations of Abramowitz
// & Stegun (1964), eqs. 9.8.1 (|x| < 3.75) and 9.8.2 (|x| >= 3.75), nested as
// the reference's Random::bessel_i0 evaluates them (dsmc/random.cpp:27-40).
template <class real> __device__ __forceinline__ real bessel_i0_as(real x) {
    const real ax = fabs(x);
    if (ax < (real)3.75) {
        real y = x / (real)3.75;
        y *= y;
        return (real)1.0 +
               y * ((real)3.5156229 +
                    y * ((real)3.0899424 +
                         y * ((real)1.2067492 + y * ((real)0.2659732 + y * ((real)0.360768e-1 + y * (real)0.45813e-2)))));
    }
    const real y = (real)3.75 / ax;
    return (exp(ax) / sqrt(ax)) *
           ((real)0.39894228 +
            y * ((real)0.1328592e-1 +
                 y * ((real)0.225319e-2 +
                      y * ((real)-0.157565e-2 +
                           y * ((real)0.916281e-2 +
                                y * ((real)-0.2057706e-1 +
                                     y * ((real)0.2635537e-1 + y * ((real)-0.1647633e-1 + y * (real)0.392377e-2))))))));
}

// Random::next_gauss (dsmc/random.cpp:21-25) on a draw stream: the ln(1-U)
// draw first.
template <class real> __device__ __forceinline__ real gauss_draw(DrawStream &rs) {
    const real u1 = rs.template uniform<real>();
    const real u2 = rs.template uniform<real>();
    return sqrt((real)-2.0 * log((real)1.0 - u1)) * cos((real)6.283185307 * u2);
}

// The reference's rejection sampler loops until it accepts; here it gives up
// after DSMC_CL_TRIALS and the caller records DSMC_EBIT_WALL.
#define DSMC_CL_TRIALS 100000
template <class real>
__device__ __forceinline__ bool cl_normal(real v_norm_in, real factor, real max_v_out, real sqrt_an_over_2,
                                          real sqrt_1m_an, real sqrt_1m_an_over_an, DrawStream &rs, real &out) {
    max_v_out /= factor;
    v_norm_in /= factor;
    const real std_dev = sqrt_an_over_2;
    const real mu = sqrt_1m_an * v_norm_in;
    for (int trial = 0; trial < DSMC_CL_TRIALS; ++trial) {
        const real v_out = std_dev * gauss_draw<real>(rs) + mu;
        const real u = rs.template uniform<real>();
        const real arg = (real)2 * sqrt_1m_an_over_an * v_norm_in * v_out;
        const real b = v_out * exp(-arg) * bessel_i0_as<real>(arg) / max_v_out;
        if (b >= u) {
            out = v_out * factor;
            return true;
        }
    }
    return false;
}

// ---- sampler profiles -------------------------------------------------------
// The calling warp's copy of the system's profile sums.
__device__ __forceinline__ double *profile_copy(const SysDev &g) {
    const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    return g.prof + (size_t)(w % (unsigned)g.prof_copies) * 4 * (size_t)g.prof_bins;
}
// Bin of a y position as MeasureCount and friends take it
// (dsmc/statisticalproperty.cpp:236): int(r_y * (1/L_y) * bins), kept in range.
__device__ __forceinline__ int profile_bin(const SysDev &g, double y) {
    const int b = (int)(y * g.invL[1] * g.prof_bins);
    return min(max(b, 0), g.prof_bins - 1);
}
// Adds per-lane {count, sum v_z, sum 1/2 m v_z^2} to the system's profile,
// one atomic per distinct bin of the warp.  All lanes call.
__device__ __forceinline__ void profile_add_warp(const SysDev &g, bool valid, int bin, double c, double s, double e) {
    unsigned todo = __ballot_sync(0xffffffffu, valid);
    while (todo) {
        const int b = __shfl_sync(0xffffffffu, bin, __ffs(todo) - 1);
        const bool in = valid && bin == b;
        double cc = in ? c : 0.0, ss = in ? s : 0.0, ee = in ? e : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            cc += __shfl_xor_sync(0xffffffffu, cc, o);
            ss += __shfl_xor_sync(0xffffffffu, ss, o);
            ee += __shfl_xor_sync(0xffffffffu, ee, o);
        }
        if ((threadIdx.x & 31) == 0) {
            double *pr = profile_copy(g);
            atomicAdd(pr + 3 * b, cc);
            atomicAdd(pr + 3 * b + 1, ss);
            atomicAdd(pr + 3 * b + 2, ee);
        }
        todo &= ~__ballot_sync(0xffffffffu, in);
    }
}

// MeasureVelocityDistribution::update (dsmc/statisticalproperty.cpp:441-458):
// bin int((v_x - v_min) / width), truncated toward zero, counted when in range.
// The quotient is taken by the reciprocal (within 4.4e-16 of the divided one,
// relatively) unless it lies within 1e-9 of an integer or beyond 1e6, where
// the division itself decides: the bin is the one the division gives.
__device__ __forceinline__ int profile_vx_bin(const SysDev &g, double vx) {
    const double d = vx - g.vx_min;
    double q = d * g.vx_inv_bin;
    const double f = q - floor(q);
    if (f < 1e-9 || f > 1.0 - 1e-9 || fabs(q) > 1e6) q = d / g.vx_bin;
    const int b = (int)q;
    return b >= 0 && b < g.prof_bins ? b : -1;
}
__device__ __forceinline__ void profile_vx(const SysDev &g, double vx) {
    const int b = profile_vx_bin(g, vx);
    if (b >= 0) atomicAdd(profile_copy(g) + 3 * g.prof_bins + b, 1.0);
}

struct Split32 {
    typedef float real;
    typedef uint4 RecA;
    typedef float4 RecB;

    // flag: the particle's voxel is not empty (kept in the sign bit of ox,
    // which is otherwise always clear), so the move needs no lookup to know
    // the start voxel's type.
    struct Particle {
        int c[3];
        float o[3];
        float v[3];
        uint32_t id;
        uint32_t flag;
    };

    static __device__ __forceinline__ void unpack(const uint4 &a, const float4 &b, Particle &p) {
        p.c[0] = DSMC_VOX_I(a.x);
        p.c[1] = DSMC_VOX_J(a.x);
        p.c[2] = DSMC_VOX_K(a.x);
        p.flag = a.y >> 31;
        p.o[0] = __uint_as_float(a.y & 0x7fffffffu);
        p.o[1] = __uint_as_float(a.z);
        p.o[2] = __uint_as_float(a.w);
        p.v[0] = b.x;
        p.v[1] = b.y;
        p.v[2] = b.z;
        p.id = __float_as_uint(b.w);
    }
    static __device__ __forceinline__ void pack(const Particle &p, uint4 &a, float4 &b) {
        a.x = DSMC_VOX_PACK(p.c[0], p.c[1], p.c[2]);
        a.y = __float_as_uint(p.o[0]) | (p.flag << 31);
        a.z = __float_as_uint(p.o[1]);
        a.w = __float_as_uint(p.o[2]);
        b.x = p.v[0];
        b.y = p.v[1];
        b.z = p.v[2];
        b.w = __uint_as_float(p.id);
    }
    // y position of a record in box units (for the sampler's bins)
    static __device__ __forceinline__ double y_of(const SysDev &g, const uint4 &a) {
        return ((double)DSMC_VOX_J(a.x) + (double)__uint_as_float(a.z)) * g.vox_len[1];
    }
    static __device__ __forceinline__ void stage_load(const uint4 *, const float4 *B, size_t i, float v[3],
                                                      uint32_t &id) {
        const float4 b = B[i];
        v[0] = b.x;
        v[1] = b.y;
        v[2] = b.z;
        id = __float_as_uint(b.w);
    }

    // r += w*tau in voxel units, carrying whole voxels into the index.
    static __device__ __forceinline__ void advance(int c[3], float o[3], const float w[3], float tau) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            float x = fmaf(w[d], tau, o[d]);
            if (x >= 1.0f || x < 0.0f) {
                float f = floorf(x);
                c[d] += (int)f;
                x -= f;
                if (x >= 1.0f) x = one_minus_ulp();
            }
            o[d] = x;
        }
    }

    // Grid::get_time_until_collision (dsmc/grid.h:82-137) in voxel units: the
    // earliest positive crossing of a face of voxel cb whose hit point lies on
    // that face (bounds inclusive), faces in the reference's order
    // x-, x+, y-, y+, z-, z+; 0 below 1e-5, else minus 1e-7.  The particle is
    // at whole-voxel offset dc = c - cb plus in-voxel offset o; the distance
    // to a face is formed as (face - dc) - o, exact for the near faces where
    // dc + o itself would round (a particle 2e-8 above a face is not on it).
    static __device__ __forceinline__ float facet_time(const int dc[3], const float o[3], const float w[3], int &axis,
                                                       int &side) {
        float best = 1e9f;
        axis = -1;
        side = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const float t = ((float)(s - dc[a]) - o[a]) / w[a];
                if (!(t > 0.0f && t < best)) continue;
                const int b1 = (a + 1) % 3, b2 = (a + 2) % 3;
                const float h1 = fmaf(w[b1], t, (float)dc[b1] + o[b1]);
                const float h2 = fmaf(w[b2], t, (float)dc[b2] + o[b2]);
                // fp32 hit points on an edge can round just outside the face
                const float eps = 1e-6f;
                if (h1 >= -eps && h1 <= 1.0f + eps && h2 >= -eps && h2 <= 1.0f + eps) {
                    best = t;
                    axis = a;
                    side = s;
                }
            }
        }
        if (axis < 0) return -1.0f;
        return best < 1e-5f ? 0.0f : best - 1e-7f;
    }

    // System::find_position (dsmc/system.cpp:384-396): uniform in the box until
    // the voxel is empty.
    static __device__ __forceinline__ bool reseed(const SysDev &g, Particle &p, DrawStream &rs) {
        for (int tries = 0; tries < 100000; ++tries) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float x = rs.uniform32() * (float)g.n[d];
                int c = (int)x;
                if (c > g.n[d] - 1) c = g.n[d] - 1;
                float o = x - (float)c;
                if (o >= 1.0f) o = one_minus_ulp();
                p.c[d] = c;
                p.o[d] = o;
            }
            if (voxel_type(g, p.c[0], p.c[1], p.c[2]) < DSMC_VOX_WALL) return true;
        }
        return false;
    }

    // The wall model's collide: ColliderThermal::collide
    // (dsmc/colliderthermal.cpp:13-46), ColliderSpecular::collide or
    // ColliderCercignaniLampis::collide.  Returns error bits.
    static __device__ __forceinline__ unsigned reflect(const SysDev &g, uint32_t vlin, float v[3], DrawStream &rs) {
        if (g.wall_model != DSMC_WALL_THERMAL) {
            const float *np = g.nrm + 3 * (size_t)vlin, *ap = g.t1 + 3 * (size_t)vlin, *bp = g.t2 + 3 * (size_t)vlin;
            const float n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2);
            const float a0 = __ldg(ap), a1 = __ldg(ap + 1), a2 = __ldg(ap + 2);
            const float b0 = __ldg(bp), b1 = __ldg(bp + 1), b2 = __ldg(bp + 2);
            const float vni = v[0] * n0 + v[1] * n1 + v[2] * n2;
            const float vt1i = v[0] * a0 + v[1] * a1 + v[2] * a2;
            const float vt2i = v[0] * b0 + v[1] * b1 + v[2] * b2;
            float vn, vt1, vt2;
            if (g.wall_model == DSMC_WALL_SPECULAR) {
                vn = -vni;
                vt1 = vt1i;
                vt2 = vt2i;
            } else {
                const float factor = sqrtf(2.0f) * g.wall_s_f;
                if (!cl_normal<float>(vni, factor, g.cl_vmax_f, g.sqrt_an_over_2_f, g.sqrt_1m_an_f,
                                      g.sqrt_1m_an_over_an_f, rs, vn))
                    return DSMC_EBIT_WALL;
                const float sigma = 1.0f - sqrtf(1.0f - g.alpha_t_f);
                vt1 = gauss_draw<float>(rs) * sqrtf(g.alpha_t_f) * g.wall_s_f + vt1i * (1.0f - sigma);
                vt2 = gauss_draw<float>(rs) * sqrtf(g.alpha_t_f) * g.wall_s_f + vt2i * (1.0f - sigma);
            }
            v[0] = vn * n0 + vt1 * a0 + vt2 * b0;
            v[1] = vn * n1 + vt1 * a1 + vt2 * b1;
            v[2] = vn * n2 + vt1 * a2 + vt2 * b2;
            return 0;
        }
        const float s = g.wall_s_f;
        const float vn = s * sqrtf(-2.0f * logf(rs.uniform32()));
        float u = rs.uniform32();
        float c = rs.uniform32();
        const float g1 = sqrtf(-2.0f * logf(1.0f - u)) * cosf(6.283185307f * c);
        u = rs.uniform32();
        c = rs.uniform32();
        const float g2 = sqrtf(-2.0f * logf(1.0f - u)) * cosf(6.283185307f * c);
        const float vt1 = s * g1, vt2 = s * g2;
        const float *n = g.nrm + 3 * (size_t)vlin;
        const float *a = g.t1 + 3 * (size_t)vlin;
        const float *b = g.t2 + 3 * (size_t)vlin;
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] = vn * __ldg(n + d) + vt1 * __ldg(a + d) + vt2 * __ldg(b + d);
        return 0;
    }

    // MoleculeMover::move_molecule (dsmc/moleculemover.cpp:50-126) with its
    // recursion unrolled into a loop, then the periodic wrap.
    //
    // In the reference every "move back by tau" of the facet loop
    // (dsmc/moleculemover.cpp:95-108) returns the particle to the position it
    // had at the start of the sub-step (the bisection's halvings and the
    // facet move are undone exactly in exact arithmetic).  In fp32 offsets
    // that subtraction drifts by an ulp, which is more than the 1e-7 time
    // units the reference leaves before a face for slow particles, so the
    // sub-step's start position is kept and restored instead.
    static __device__ __noinline__ void move_general(const SysDev &g, Particle &p, uint32_t step, MoveTally &t) {
        DrawStream rs;
        rs.init(g.seed, p.id, step, DSMC_TAG_MOVE);
        float w[3] = {p.v[0] * g.inv_vox_f[0], p.v[1] * g.inv_vox_f[1], p.v[2] * g.inv_vox_f[2]};
        float dt = g.dt_f;
        int here = p.flag ? DSMC_VOX_WALL : DSMC_VOX_EMPTY;  // (non-)emptiness of the current voxel
        for (int depth = 0;; ++depth) {
            if (here != DSMC_VOX_EMPTY) {
                ++t.reseeds;
                if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                here = DSMC_VOX_EMPTY;
                break;
            }
            const int c0[3] = {p.c[0], p.c[1], p.c[2]};
            const float o0[3] = {p.o[0], p.o[1], p.o[2]};
            float tau = dt;
            advance(p.c, p.o, w, tau);
            int vt = voxel_type(g, p.c[0], p.c[1], p.c[2]);
            if (vt == DSMC_VOX_EMPTY) break;
            // Bisect back out of solid (wall) voxels until a boundary voxel.
            bool stop = false, again = false;
            int count = 0;
            while (vt != DSMC_VOX_BOUNDARY) {
                if (++count > 100) {
                    ++t.reseeds;
                    if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                    stop = true;
                    break;
                }
                if (vt == DSMC_VOX_WALL) {
                    tau *= 0.5f;
                    advance(p.c, p.o, w, -tau);
                    vt = voxel_type(g, p.c[0], p.c[1], p.c[2]);
                } else {
                    dt -= tau;
                    again = dt > 1e-5f && depth < 10;
                    stop = !again;
                    break;
                }
            }
            if (stop) break;
            if (again) continue;
            // Back off and stop just short of the first boundary voxel's face.
            int cb[3] = {p.c[0], p.c[1], p.c[2]};
            count = 0;
            while (vt == DSMC_VOX_BOUNDARY) {
                if (++count > 100) {
                    ++t.reseeds;
                    if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                    stop = true;
                    break;
                }
                cb[0] = p.c[0];
                cb[1] = p.c[1];
                cb[2] = p.c[2];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    p.c[a] = c0[a];
                    p.o[a] = o0[a];
                }
                int dc[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) dc[a] = p.c[a] - cb[a];
                const bool outside = (dc[0] | dc[1] | dc[2]) != 0;  // offsets lie in [0, 1)
                int axis, side;
                const float tf = facet_time(dc, p.o, w, axis, side);
                if (tf < 0.0f) {
                    t.err |= DSMC_EBIT_FACET;
                    ++t.reseeds;
                    if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                    stop = true;
                    break;
                }
                tau = tf;
                advance(p.c, p.o, w, tau);
                // fp32 offsets can round onto the face the fp64 reference stops
                // 1e-7 time units short of; put the particle back outside.
                if (outside && tau > 0.0f && p.c[0] == cb[0] && p.c[1] == cb[1] && p.c[2] == cb[2]) {
                    const int cba = axis == 0 ? cb[0] : axis == 1 ? cb[1] : cb[2];  // no run-time index
                    const int out = side == 0 ? cba - 1 : cba + 1;
                    const float oo = side == 0 ? one_minus_ulp() : 0.0f;
                    if (axis == 0) {
                        p.c[0] = out;
                        p.o[0] = oo;
                    } else if (axis == 1) {
                        p.c[1] = out;
                        p.o[1] = oo;
                    } else {
                        p.c[2] = out;
                        p.o[2] = oo;
                    }
                }
                vt = voxel_type(g, p.c[0], p.c[1], p.c[2]);
            }
            if (stop) break;
            here = vt;
            dt -= tau;
            t.err |= reflect(g, voxel_linear(g, cb[0], cb[1], cb[2]), p.v, rs);
            ++t.wall_hits;
#pragma unroll
            for (int d = 0; d < 3; ++d) w[d] = p.v[d] * g.inv_vox_f[d];
            if (!(dt > 1e-5f && depth < 10)) break;
        }
        p.flag = here != DSMC_VOX_EMPTY;
        wrap(g, p, t);
    }

    // move_general as a state machine for a whole warp: every lane runs its
    // own flight, and each turn of the loop issues at most one voxel lookup
    // per lane at one program point, so the warp's lookups travel together
    // instead of one divergent path after another.  The same arithmetic in
    // the same order per particle as move_general.  All lanes call; inactive
    // lanes only keep the loop company.
    static __device__ __forceinline__ void move_general_warp(const SysDev &g, Particle &p, uint32_t step,
                                                             MoveTally &t, bool active) {
        enum { S_START, S_FIRST, S_BISECT, S_FACET, S_REFLECT, S_DONE };
        DrawStream rs;
        rs.init(g.seed, p.id, step, DSMC_TAG_MOVE);
        float w[3] = {p.v[0] * g.inv_vox_f[0], p.v[1] * g.inv_vox_f[1], p.v[2] * g.inv_vox_f[2]};
        float dt = g.dt_f, tau = 0.0f;
        int here = p.flag ? DSMC_VOX_WALL : DSMC_VOX_EMPTY;
        int depth = 0, count = 0, vt = DSMC_VOX_EMPTY;
        int c0[3] = {0, 0, 0}, cb[3] = {0, 0, 0};
        float o0[3] = {0.0f, 0.0f, 0.0f};
        int state = active ? S_START : S_DONE;
        while (__any_sync(0xffffffffu, state != S_DONE)) {
            bool look = false;
            while (state != S_DONE && !look) {
                if (state == S_START) {
                    if (here != DSMC_VOX_EMPTY) {
                        ++t.reseeds;
                        if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                        here = DSMC_VOX_EMPTY;
                        state = S_DONE;
                    } else {
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            c0[a] = p.c[a];
                            o0[a] = p.o[a];
                        }
                        tau = dt;
                        advance(p.c, p.o, w, tau);
                        look = true;
                        state = S_FIRST;
                    }
                } else if (state == S_FIRST) {
                    if (vt == DSMC_VOX_EMPTY) {
                        state = S_DONE;
                    } else {
                        count = 0;
                        state = S_BISECT;
                    }
                } else if (state == S_BISECT) {
                    // bisect back out of solid (wall) voxels until a boundary voxel
                    if (vt == DSMC_VOX_BOUNDARY) {
                        cb[0] = p.c[0];
                        cb[1] = p.c[1];
                        cb[2] = p.c[2];
                        count = 0;
                        state = S_FACET;
                    } else if (++count > 100) {
                        ++t.reseeds;
                        if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                        state = S_DONE;
                    } else if (vt == DSMC_VOX_WALL) {
                        tau *= 0.5f;
                        advance(p.c, p.o, w, -tau);
                        look = true;
                    } else {
                        dt -= tau;
                        if (dt > 1e-5f && depth < 10) {
                            ++depth;
                            state = S_START;
                        } else {
                            state = S_DONE;
                        }
                    }
                } else if (state == S_FACET) {
                    // back off and stop just short of the first boundary voxel's face
                    if (vt != DSMC_VOX_BOUNDARY) {
                        state = S_REFLECT;
                    } else if (++count > 100) {
                        ++t.reseeds;
                        if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                        state = S_DONE;
                    } else {
                        cb[0] = p.c[0];
                        cb[1] = p.c[1];
                        cb[2] = p.c[2];
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            p.c[a] = c0[a];
                            p.o[a] = o0[a];
                        }
                        int dc[3];
#pragma unroll
                        for (int a = 0; a < 3; ++a) dc[a] = p.c[a] - cb[a];
                        const bool outside = (dc[0] | dc[1] | dc[2]) != 0;  // offsets lie in [0, 1)
                        int axis, side;
                        const float tf = facet_time(dc, p.o, w, axis, side);
                        if (tf < 0.0f) {
                            t.err |= DSMC_EBIT_FACET;
                            ++t.reseeds;
                            if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                            state = S_DONE;
                        } else {
                            tau = tf;
                            advance(p.c, p.o, w, tau);
                            if (outside && tau > 0.0f && p.c[0] == cb[0] && p.c[1] == cb[1] && p.c[2] == cb[2]) {
                                const int cba = axis == 0 ? cb[0] : axis == 1 ? cb[1] : cb[2];  // no run-time index
                                const int out = side == 0 ? cba - 1 : cba + 1;
                                const float oo = side == 0 ? one_minus_ulp() : 0.0f;
                                if (axis == 0) {
                                    p.c[0] = out;
                                    p.o[0] = oo;
                                } else if (axis == 1) {
                                    p.c[1] = out;
                                    p.o[1] = oo;
                                } else {
                                    p.c[2] = out;
                                    p.o[2] = oo;
                                }
                            }
                            look = true;
                        }
                    }
                } else {  // S_REFLECT
                    here = vt;
                    dt -= tau;
                    t.err |= reflect(g, voxel_linear(g, cb[0], cb[1], cb[2]), p.v, rs);
                    ++t.wall_hits;
#pragma unroll
                    for (int d = 0; d < 3; ++d) w[d] = p.v[d] * g.inv_vox_f[d];
                    if (!(dt > 1e-5f && depth < 10)) {
                        state = S_DONE;
                    } else {
                        ++depth;
                        state = S_START;
                    }
                }
            }
            if (look) vt = voxel_type(g, p.c[0], p.c[1], p.c[2]);
        }
        if (active) {
            p.flag = here != DSMC_VOX_EMPTY;
            wrap(g, p, t);
        }
    }

    // Periodic wrap, one box length at most, counting net crossings
    // (System::move, dsmc/system.cpp:107-120).
    static __device__ __forceinline__ void wrap(const SysDev &g, Particle &p, MoveTally &t) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (p.c[d] >= g.n[d]) {
                p.c[d] -= g.n[d];
                ++t.cross[d];
            } else if (p.c[d] < 0) {
                p.c[d] += g.n[d];
                --t.cross[d];
            }
            if (!(p.o[d] >= 0.0f && p.o[d] < 1.0f) || !isfinite(p.v[d]) || p.c[d] < 0 || p.c[d] >= g.n[d]) {
                t.err |= DSMC_EBIT_NAN;
                p.c[d] = min(max(p.c[d], 0), g.n[d] - 1);
                p.o[d] = 0.5f;
            }
        }
    }

    // The general mover's outcome when its first flight is all there is: a
    // particle in an empty voxel whose full-dt flight ends in an empty voxel
    // stops there (dsmc/moleculemover.cpp:74-77), then wraps.  Same arithmetic
    // as move_general's first sub-step; false (p untouched) when the flight
    // ends in a wall or boundary voxel or starts outside an empty one.
    static __device__ __forceinline__ bool move_open(const SysDev &g, Particle &p, MoveTally &t) {
        if (p.flag) return false;
        int c[3] = {p.c[0], p.c[1], p.c[2]};
        float o[3] = {p.o[0], p.o[1], p.o[2]};
        const float w[3] = {p.v[0] * g.inv_vox_f[0], p.v[1] * g.inv_vox_f[1], p.v[2] * g.inv_vox_f[2]};
        advance(c, o, w, g.dt_f);
        if (voxel_type(g, c[0], c[1], c[2]) != DSMC_VOX_EMPTY) return false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            p.c[d] = c[d];
            p.o[d] = o[d];
        }
        wrap(g, p, t);
        return true;
    }

    // The whole move.  A particle whose full-dt flight stays inside its
    // (empty) voxel needs no lookup at all: that is the reference's outcome
    // too (r += v*dt lands in an empty voxel, dt = 0; dsmc/moleculemover.cpp:
    // 74-77,122).  Everything else takes the general path.
    // Returns true when the particle left its voxel.
    static __device__ __forceinline__ bool move(const SysDev &g, Particle &p, uint32_t step, MoveTally &t) {
        if (!p.flag) {
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
                return false;
            }
        }
        move_general(g, p, step, t);
        return true;
    }

    // Cell of the particle: whole voxels per cell, so cell = voxel / vpc.
    static __device__ __forceinline__ int cell_global(const SysDev &g, const Particle &p) {
        int ci[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            int c = __float2int_rz(((float)p.c[d] + 0.5f) * g.inv_vpc[d]);
            ci[d] = min(c, g.cells[d] - 1);
        }
        return (ci[0] * g.cells[1] + ci[1]) * g.cells[2] + ci[2];
    }

    static __device__ __forceinline__ void accelerate(const SysDev &g, Particle &p) {
        // per-component selects: a store at a run-time index into p.v would
        // put the particle in local memory
        const int f = g.flow_dir;
        const float a = g.accel_dt_f;
        p.v[0] = f == 0 ? p.v[0] + a : p.v[0];
        p.v[1] = f == 1 ? p.v[1] + a : p.v[1];
        p.v[2] = f == 2 ? p.v[2] + a : p.v[2];
    }
};

// ============================================================================
// fp64 reference arithmetic: absolute fp64 positions as in System::r
// (dsmc/system.h:74), the reference's float-rounded index constants.
// ============================================================================
struct Vec3d {
    double x, y, z;
};
__device__ __forceinline__ Vec3d v3(double x, double y, double z) {
    Vec3d r;
    r.x = x;
    r.y = y;
    r.z = z;
    return r;
}
__device__ __forceinline__ Vec3d v3sub(const Vec3d &a, const Vec3d &b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ Vec3d v3add(const Vec3d &a, const Vec3d &b) { return v3(b.x + a.x, b.y + a.y, b.z + a.z); }
__device__ __forceinline__ Vec3d v3scale(const Vec3d &a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double v3dot(const Vec3d &a, const Vec3d &o) { return a.x * o.x + a.y * o.y + a.z * o.z; }
// CVector::cross (dsmc/cvector.h:148-150): this x o
__device__ __forceinline__ Vec3d v3cross(const Vec3d &t, const Vec3d &o) {
    return v3(o.y * t.z - o.z * t.y, o.z * t.x - o.x * t.z, o.x * t.y - o.y * t.x);
}
// same_side / is_point_within_square (dsmc/grid.h:21-41)
__device__ __forceinline__ bool same_side(const Vec3d &p1, const Vec3d &p2, const Vec3d &a, const Vec3d &b) {
    const Vec3d ba = v3sub(b, a);
    const Vec3d cp1 = v3cross(ba, v3sub(p1, a));
    const Vec3d cp2 = v3cross(ba, v3sub(p2, a));
    return v3dot(cp1, cp2) >= 0;
}
__device__ __forceinline__ bool within_square(const Vec3d &p1, const Vec3d &p2, const Vec3d &p3, const Vec3d &p4,
                                              const Vec3d &pt) {
    const Vec3d c = v3scale(v3add(v3add(v3add(p1, p2), p3), p4), 0.25);
    return same_side(pt, c, p1, p2) && same_side(pt, c, p2, p3) && same_side(pt, c, p3, p4) &&
           same_side(pt, c, p4, p1);
}

struct Fp64 {
    typedef double real;
    typedef double4 RecA;
    typedef double4 RecB;

    struct Particle {
        double r[3];
        double v[3];
        uint32_t id;
    };

    static __device__ __forceinline__ void unpack(const double4 &a, const double4 &b, Particle &p) {
        p.r[0] = a.x;
        p.r[1] = a.y;
        p.r[2] = a.z;
        p.id = (uint32_t)a.w;
        p.v[0] = b.x;
        p.v[1] = b.y;
        p.v[2] = b.z;
    }
    static __device__ __forceinline__ void pack(const Particle &p, double4 &a, double4 &b) {
        a.x = p.r[0];
        a.y = p.r[1];
        a.z = p.r[2];
        a.w = (double)p.id;
        b.x = p.v[0];
        b.y = p.v[1];
        b.z = p.v[2];
        b.w = 0.0;
    }
    static __device__ __forceinline__ double y_of(const SysDev &, const double4 &a) { return a.y; }
    static __device__ __forceinline__ void stage_load(const double4 *A, const double4 *B, size_t i, double v[3],
                                                      uint32_t &id) {
        const double4 b = B[i];
        v[0] = b.x;
        v[1] = b.y;
        v[2] = b.z;
        id = (uint32_t)A[i].w;
    }

    // Grid::get_index_of_voxel (dsmc/grid.h:139-145): i = int(r*float(n/L) +
    // float(halo offset)) in the 3x halo grid; returned here relative to the
    // box (halo offset subtracted, may lie in [-n, 2n)).
    static __device__ __forceinline__ void voxel_of(const SysDev &g, const double r[3], int u[3]) {
#pragma unroll
        for (int d = 0; d < 3; ++d) u[d] = (int)(r[d] * g.ref_scale[d] + g.ref_shift[d]) - g.n[d];
    }
    static __device__ __forceinline__ int type_at(const SysDev &g, const double r[3], int u[3]) {
        voxel_of(g, r, u);
        return voxel_type(g, u[0], u[1], u[2]);
    }
    static __device__ __forceinline__ void do_move(double r[3], const double v[3], double tau) {
#pragma unroll
        for (int d = 0; d < 3; ++d) r[d] += v[d] * tau;
    }

    // Grid::get_time_until_collision (dsmc/grid.h:82-137), operation by operation.
    static __device__ double facet_time(const SysDev &g, const double r[3], const double v[3], const int b[3],
                                        bool &found) {
        const Vec3d R = v3(r[0] - 0.0, r[1] - 0.0, r[2] - 0.0);
        const Vec3d V = v3(v[0], v[1], v[2]);
        const double hx = g.vox_len[0], hy = g.vox_len[1], hz = g.vox_len[2];
        const int i = b[0], j = b[1], k = b[2];
        Vec3d P[8];
        P[0] = v3(i * hx, j * hy, k * hz);
        P[1] = v3((i + 1) * hx, j * hy, k * hz);
        P[2] = v3(i * hx, j * hy, (k + 1) * hz);
        P[3] = v3((i + 1) * hx, j * hy, (k + 1) * hz);
        P[4] = v3(i * hx, (j + 1) * hy, k * hz);
        P[5] = v3((i + 1) * hx, (j + 1) * hy, k * hz);
        P[6] = v3(i * hx, (j + 1) * hy, (k + 1) * hz);
        P[7] = v3((i + 1) * hx, (j + 1) * hy, (k + 1) * hz);
        const Vec3d N[6] = {v3(-1, 0, 0), v3(1, 0, 0), v3(0, -1, 0), v3(0, 1, 0), v3(0, 0, -1), v3(0, 0, 1)};
        const int plane_point[6] = {2, 1, 0, 4, 0, 2};
        const int sq[6][4] = {{4, 0, 2, 6}, {1, 5, 7, 3}, {0, 1, 3, 2}, {5, 4, 6, 7}, {4, 5, 1, 0}, {2, 3, 7, 6}};
        double best = 1e9;
        found = false;
        for (int f = 0; f < 6; ++f) {
            const double tf = v3dot(v3sub(P[plane_point[f]], R), N[f]) / v3dot(V, N[f]);
            const bool hit = within_square(P[sq[f][0]], P[sq[f][1]], P[sq[f][2]], P[sq[f][3]], v3add(R, v3scale(V, tf)));
            if (tf > 0 && tf < best && hit && !isnan(tf)) {
                best = tf;
                found = true;
            }
        }
        if (best < 1e-5) return 0;
        return best - 1e-7;
    }

    // System::find_position (dsmc/system.cpp:384-396) with Grid::get_voxel(r, n)
    // (dsmc/grid.cpp:63-69): all-double index arithmetic.
    static __device__ __forceinline__ bool reseed(const SysDev &g, Particle &p, DrawStream &rs) {
        for (int tries = 0; tries < 100000; ++tries) {
#pragma unroll
            for (int d = 0; d < 3; ++d) p.r[d] = 0.0 + g.L[d] * rs.uniform64();
            int u[3];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                u[d] = (int)((p.r[d] - 0.0) * g.invL[d] * (double)g.n[d] + (double)g.n[d]) - g.n[d];
            if (voxel_type(g, u[0], u[1], u[2]) < DSMC_VOX_WALL) return true;
        }
        return false;
    }

    // ColliderThermal::collide (dsmc/colliderthermal.cpp:13-46).
    static __device__ __forceinline__ unsigned reflect(const SysDev &g, uint32_t vlin, double v[3], DrawStream &rs) {
        if (g.wall_model != DSMC_WALL_THERMAL) {
            // the reference's mix: float wall frames, double velocities
            const float *np = g.nrm + 3 * (size_t)vlin, *ap = g.t1 + 3 * (size_t)vlin, *bp = g.t2 + 3 * (size_t)vlin;
            const float n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2);
            const float a0 = __ldg(ap), a1 = __ldg(ap + 1), a2 = __ldg(ap + 2);
            const float b0 = __ldg(bp), b1 = __ldg(bp + 1), b2 = __ldg(bp + 2);
            if (g.wall_model == DSMC_WALL_SPECULAR) {
                const double vn = n0 * v[0] + n1 * v[1] + n2 * v[2];
                const double vt1 = a0 * v[0] + a1 * v[1] + a2 * v[2];
                const double vt2 = b0 * v[0] + b1 * v[1] + b2 * v[2];
                v[0] = -vn * n0 + vt1 * a0 + vt2 * b0;
                v[1] = -vn * n1 + vt1 * a1 + vt2 * b1;
                v[2] = -vn * n2 + vt1 * a2 + vt2 * b2;
                return 0;
            }
            const double factor = sqrt(2.0) * g.wall_s;
            const double vni = v[0] * n0 + v[1] * n1 + v[2] * n2;
            const double vt1i = v[0] * a0 + v[1] * a1 + v[2] * a2;
            const double vt2i = v[0] * b0 + v[1] * b1 + v[2] * b2;
            double vn;
            if (!cl_normal<double>(vni, factor, g.cl_vmax, g.sqrt_an_over_2, g.sqrt_1m_an, g.sqrt_1m_an_over_an, rs,
                                   vn))
                return DSMC_EBIT_WALL;
            const double sigma = 1 - sqrt(1 - g.alpha_t);
            const double vt1 = gauss_draw<double>(rs) * sqrt(g.alpha_t) * g.wall_s + vt1i * (1 - sigma);
            const double vt2 = gauss_draw<double>(rs) * sqrt(g.alpha_t) * g.wall_s + vt2i * (1 - sigma);
            v[0] = vn * n0 + vt1 * a0 + vt2 * b0;
            v[1] = vn * n1 + vt1 * a1 + vt2 * b1;
            v[2] = vn * n2 + vt1 * a2 + vt2 * b2;
            return 0;
        }
        const double s = g.wall_s;
        const double vn = s * sqrt(-2 * log(rs.uniform64()));
        double u = rs.uniform64();
        double c = rs.uniform64();
        const double g1 = sqrt(-2.0 * log(1.0 - u)) * cos(6.283185307 * c);
        u = rs.uniform64();
        c = rs.uniform64();
        const double g2 = sqrt(-2.0 * log(1.0 - u)) * cos(6.283185307 * c);
        const double vt1 = s * g1, vt2 = s * g2;
        const float *n = g.nrm + 3 * (size_t)vlin;
        const float *a = g.t1 + 3 * (size_t)vlin;
        const float *b = g.t2 + 3 * (size_t)vlin;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float nf = __ldg(n + d), af = __ldg(a + d), bf = __ldg(b + d);
            v[d] = vn * nf + vt1 * af + vt2 * bf;
        }
        return 0;
    }

    static __device__ bool move(const SysDev &g, Particle &p, uint32_t step, MoveTally &t) {
        DrawStream rs;
        rs.init(g.seed, p.id, step, DSMC_TAG_MOVE);
        double dt = g.dt;
        int u[3];
        for (int depth = 0;; ++depth) {
            double tau = dt;
            if (type_at(g, p.r, u) != DSMC_VOX_EMPTY) {
                ++t.reseeds;
                if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                break;
            }
            do_move(p.r, p.v, tau);
            int vt = type_at(g, p.r, u);
            if (vt < DSMC_VOX_WALL) break;
            bool stop = false, again = false;
            int count = 0;
            while (vt != DSMC_VOX_BOUNDARY) {
                if (++count > 100) {
                    ++t.reseeds;
                    if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                    stop = true;
                    break;
                }
                if (vt == DSMC_VOX_WALL) {
                    tau /= 2;
                    do_move(p.r, p.v, -tau);
                    vt = type_at(g, p.r, u);
                } else {
                    dt -= tau;
                    again = dt > 1e-5 && depth < 10;
                    stop = !again;
                    break;
                }
            }
            if (stop) break;
            if (again) continue;
            int b[3] = {u[0], u[1], u[2]};
            count = 0;
            while (vt == DSMC_VOX_BOUNDARY) {
                if (++count > 100) {
                    ++t.reseeds;
                    if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                    stop = true;
                    break;
                }
                b[0] = u[0];
                b[1] = u[1];
                b[2] = u[2];
                do_move(p.r, p.v, -tau);
                bool found;
                tau = facet_time(g, p.r, p.v, b, found);
                if (!found) {
                    t.err |= DSMC_EBIT_FACET;
                    ++t.reseeds;
                    if (!reseed(g, p, rs)) t.err |= DSMC_EBIT_RESEED;
                    stop = true;
                    break;
                }
                do_move(p.r, p.v, tau);
                vt = type_at(g, p.r, u);
            }
            if (stop) break;
            dt -= tau;
            t.err |= reflect(g, voxel_linear(g, b[0], b[1], b[2]), p.v, rs);
            ++t.wall_hits;
            if (!(dt > 1e-5 && depth < 10)) break;
        }
        // MoleculeMover::apply_periodic_boundary_conditions (dsmc/moleculemover.h:29-38)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (p.r[d] >= g.L[d]) {
                p.r[d] -= g.L[d];
                ++t.cross[d];
            } else if (p.r[d] < 0) {
                p.r[d] += g.L[d];
                --t.cross[d];
            }
            if (!isfinite(p.r[d]) || !isfinite(p.v[d])) t.err |= DSMC_EBIT_NAN;
        }
        return true;
    }

    // System::cell_index_from_position (dsmc/system.h:122-132).
    static __device__ __forceinline__ int cell_global(const SysDev &g, const Particle &p) {
        int ci[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            int c = (int)(p.r[d] * g.invL[d] * g.cells[d]);
            ci[d] = min(max(c, 0), g.cells[d] - 1);
        }
        return (ci[0] * g.cells[1] + ci[1]) * g.cells[2] + ci[2];
    }

    static __device__ __forceinline__ void accelerate(const SysDev &g, Particle &p) {
        const int f = g.flow_dir;
        const double a = g.accel_dt;
        p.v[0] = f == 0 ? p.v[0] + a : p.v[0];
        p.v[1] = f == 1 ? p.v[1] + a : p.v[1];
        p.v[2] = f == 2 ? p.v[2] + a : p.v[2];
    }
};

// ============================================================================
// The cell pass.
// ============================================================================
template <class Prec> struct WarpStage {
    typedef typename Prec::real real;
    real *vx, *vy, *vz;
    uint32_t *id;
    uint16_t *perm;
    static __host__ __device__ size_t bytes(int cap) {
        size_t b = (size_t)cap * (3 * sizeof(real) + sizeof(uint32_t) + sizeof(uint16_t));
        return (b + 15) & ~(size_t)15;
    }
    __device__ void bind(unsigned char *base, int cap) {
        vx = reinterpret_cast<real *>(base);
        vy = vx + cap;
        vz = vy + cap;
        id = reinterpret_cast<uint32_t *>(vz + cap);
        perm = reinterpret_cast<uint16_t *>(id + cap);
    }
};

// ---- NTC arithmetic shared by every collide path ----------------------------
// Rounding is spelled out (no contraction) so that the fused pass and the
// stand-alone collide stage produce bit-identical velocities, and the fp64
// bookkeeping rounds as the reference's does.

// Cell::prepare (dsmc/cell.cpp:42-51): pairs = round(coeff N (N-1) vr_max + rest).
__device__ __forceinline__ int ntc_select(double coeff, int n, double vr_max, double &rest) {
    const double select = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(coeff, (double)n), (double)(n - 1)), vr_max), rest);
    const int pairs = (int)round(select);
    rest = __dsub_rn(select, (double)pairs);
    return pairs;
}

// candidate pair (dsmc/cell.cpp:80-82): ip0 = int(U N), ip1 = int(ip0 + 1 + U (N-1)) % N
__device__ __forceinline__ void ntc_pick(float ua, float ub, int n, int &ip0, int &ip1) {
    ip0 = min((int)__fmul_rn(ua, (float)n), n - 1);
    ip1 = ((int)__fadd_rn((float)(ip0 + 1), __fmul_rn(ub, (float)(n - 1)))) % n;
}
__device__ __forceinline__ void ntc_pick(double ua, double ub, int n, int &ip0, int &ip1) {
    ip0 = min((int)__dmul_rn(ua, (double)n), n - 1);
    ip1 = ((int)__dadd_rn((double)(ip0 + 1), __dmul_rn(ub, (double)(n - 1)))) % n;
}

__device__ __forceinline__ float rel_speed(float dx, float dy, float dz) {
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}
__device__ __forceinline__ double rel_speed(double dx, double dy, double dz) {
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// Cell::collide_molecules (dsmc/cell.cpp:53-73): isotropic post-collision
// relative velocity about the centre of mass.
__device__ __forceinline__ void ntc_scatter(float &ax, float &ay, float &az, float &bx, float &by, float &bz,
                                            float vrel, float u_cos, float u_phi) {
    const float cmx = __fmul_rn(0.5f, __fadd_rn(ax, bx));
    const float cmy = __fmul_rn(0.5f, __fadd_rn(ay, by));
    const float cmz = __fmul_rn(0.5f, __fadd_rn(az, bz));
    const float cos_th = __fsub_rn(1.0f, __fmul_rn(2.0f, u_cos));
    const float sin_th = __fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(cos_th, cos_th)));
    const float phi = __fmul_rn(6.2831853071795864769f, u_phi);
    float sp, cp;
    sincosf(phi, &sp, &cp);
    const float rx = __fmul_rn(vrel, cos_th);
    const float ry = __fmul_rn(__fmul_rn(vrel, sin_th), cp);
    const float rz = __fmul_rn(__fmul_rn(vrel, sin_th), sp);
    ax = __fadd_rn(cmx, __fmul_rn(0.5f, rx));
    ay = __fadd_rn(cmy, __fmul_rn(0.5f, ry));
    az = __fadd_rn(cmz, __fmul_rn(0.5f, rz));
    bx = __fsub_rn(cmx, __fmul_rn(0.5f, rx));
    by = __fsub_rn(cmy, __fmul_rn(0.5f, ry));
    bz = __fsub_rn(cmz, __fmul_rn(0.5f, rz));
}
__device__ __forceinline__ void ntc_scatter(double &ax, double &ay, double &az, double &bx, double &by, double &bz,
                                            double vrel, double u_cos, double u_phi) {
    const double cmx = 0.5 * (ax + bx), cmy = 0.5 * (ay + by), cmz = 0.5 * (az + bz);
    const double cos_th = 1.0 - 2.0 * u_cos;
    const double sin_th = sqrt(1.0 - cos_th * cos_th);
    const double phi = 2 * 3.14159265358979323846 * u_phi;
    const double rx = vrel * cos_th;
    const double ry = vrel * sin_th * cos(phi);
    const double rz = vrel * sin_th * sin(phi);
    ax = cmx + 0.5 * rx;
    ay = cmy + 0.5 * ry;
    az = cmz + 0.5 * rz;
    bx = cmx - 0.5 * rx;
    by = cmy - 0.5 * ry;
    bz = cmz - 0.5 * rz;
}

// Cell::collide (dsmc/cell.cpp:75-111) over the members in id order, on
// velocities staged in shared memory.  Run by one lane.  Draws: stream
// (cell, step, collide), three per candidate and two more per collision.
template <class real, class Vel, class Draws, class Perm>
__device__ __forceinline__ void ntc_loop(Draws &rs, int n, int pairs, double &vr_max, Vel vel, Perm perm,
                         unsigned long long &collisions) {
    double crm = vr_max;
    const real vmax = (real)vr_max;
    for (int isel = 0; isel < pairs; ++isel) {
        const real ua = rs.template uniform<real>();
        const real ub = rs.template uniform<real>();
        int ip0, ip1;
        ntc_pick(ua, ub, n, ip0, ip1);
        const int s0 = perm[ip0], s1 = perm[ip1];
        real ax, ay, az, bx, by, bz;
        vel.get(s0, ax, ay, az);
        vel.get(s1, bx, by, bz);
        const real vrel = rel_speed(ax - bx, ay - by, az - bz);
        if ((double)vrel > crm) crm = (double)vrel;
        const real uc = rs.template uniform<real>();
        if (vrel > uc * vmax) {
            ++collisions;
            const real u_cos = rs.template uniform<real>();
            const real u_phi = rs.template uniform<real>();
            ntc_scatter(ax, ay, az, bx, by, bz, vrel, u_cos, u_phi);
            vel.set(s0, ax, ay, az);
            vel.set(s1, bx, by, bz);
        }
    }
    vr_max = crm;
}
template <class real, class Vel>
__device__ void ntc_run(uint64_t seed, int cell_global_index, uint32_t step, int n, int pairs, double &vr_max,
                        Vel vel, const uint16_t *perm, unsigned long long &collisions) {
    DrawStream rs;
    rs.init(seed, (uint32_t)cell_global_index, step, DSMC_TAG_COLLIDE);
    ntc_loop<real>(rs, n, pairs, vr_max, vel, perm, collisions);
}

template <class Prec> struct StageVel {
    typedef typename Prec::real real;
    real *vx, *vy, *vz;
    __device__ void get(int s, real &x, real &y, real &z) const {
        x = vx[s];
        y = vy[s];
        z = vz[s];
    }
    __device__ void set(int s, real x, real y, real z) const {
        vx[s] = x;
        vy[s] = y;
        vz[s] = z;
    }
};

template <class Prec>
__device__ void ntc_collide(const SysDev &g, int cell_global_index, uint32_t step, int n, double coeff,
                            double &vr_max, double &rest, WarpStage<Prec> &st, unsigned long long &collisions,
                            unsigned long long &candidates) {
    const int pairs = ntc_select(coeff, n, vr_max, rest);
    if (n < 2 || pairs <= 0) return;
    StageVel<Prec> vel;
    vel.vx = st.vx;
    vel.vy = st.vy;
    vel.vz = st.vz;
    ntc_run<typename Prec::real>(g.seed, cell_global_index, step, n, pairs, vr_max, vel, st.perm, collisions);
    candidates += (unsigned long long)pairs;
}

struct WarpTally {
    unsigned long long collisions, candidates, wall_hits, reseeds, moved, stranded;
    long long cross[3];
    unsigned err;
    int sys;
};

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ long long warp_sum_i64(long long x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ double warp_sum_f64(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ __forceinline__ void flush_tally(const PassParams &P, WarpTally &w, int lane) {
    // All lanes call; per-lane partial counts are summed, lane 0 publishes.
    const unsigned long long wh = warp_sum_u64(w.wall_hits);
    const unsigned long long rs = warp_sum_u64(w.reseeds);
    const unsigned long long mv = warp_sum_u64(w.moved);
    const unsigned long long sd = warp_sum_u64(w.stranded);
    long long cr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) cr[d] = warp_sum_i64(w.cross[d]);
    unsigned err = __reduce_or_sync(0xffffffffu, w.err);
    if (lane == 0 && w.sys >= 0) {
        SysTally &T = P.tally[w.sys];
        if (w.collisions) atomicAdd(&T.collisions, w.collisions);
        if (w.candidates) atomicAdd(&T.candidates, w.candidates);
        if (wh) atomicAdd(&T.wall_hits, wh);
        if (rs) atomicAdd(&T.reseeds, rs);
        if (mv) atomicAdd(&T.particle_steps, mv);
        if (sd) atomicAdd(&T.stranded, sd);
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (cr[d]) atomicAdd((unsigned long long *)&T.count_periodic[d], (unsigned long long)cr[d]);
        if (err) atomicOr(&P.status->error, err);
    }
    w.collisions = w.candidates = w.wall_hits = w.reseeds = w.moved = w.stranded = 0;
    w.cross[0] = w.cross[1] = w.cross[2] = 0;
    w.err = 0;
}

template <class Prec, int MODE>
__global__ void __launch_bounds__(256) pass_kernel(PassParams P) {
    typedef typename Prec::real real;
    typedef typename Prec::RecA RecA;
    typedef typename Prec::RecB RecB;
    typedef typename Prec::Particle Particle;
    extern __shared__ __align__(16) unsigned char smem[];

    const int lane = threadIdx.x & 31;
    const int warp_in_block = threadIdx.x >> 5;
    const int warps_per_block = blockDim.x >> 5;
    const volatile Status *vs = P.status;
    if (vs->halted) return;
    const uint32_t step = vs->step;
    const uint32_t move_step = step + 1;

    WarpStage<Prec> st;
    st.bind(smem + (size_t)warp_in_block * WarpStage<Prec>::bytes(P.smem_cap), P.smem_cap);

    const RecA *Ain = reinterpret_cast<const RecA *>(P.parts.A[P.cur]);
    const RecB *Bin = reinterpret_cast<const RecB *>(P.parts.B[P.cur]);
    RecA *Aout = reinterpret_cast<RecA *>(P.parts.A[P.cur ^ 1]);
    RecB *Bout = reinterpret_cast<RecB *>(P.parts.B[P.cur ^ 1]);
    RecA *Aio = reinterpret_cast<RecA *>(P.parts.A[P.cur]);
    RecB *Bio = reinterpret_cast<RecB *>(P.parts.B[P.cur]);
    const unsigned *bot_in = P.cells.bot[P.cin];
    const unsigned *top_in = P.cells.top[P.cin];
    unsigned *top_out = P.cells.top[P.cout];

    WarpTally wt;
    wt.collisions = wt.candidates = wt.wall_hits = wt.reseeds = wt.moved = wt.stranded = 0;
    wt.cross[0] = wt.cross[1] = wt.cross[2] = 0;
    wt.err = 0;
    wt.sys = -1;

    const int C = P.cells.num_cells;
    const int stride = gridDim.x * warps_per_block;
    for (int a = blockIdx.x * warps_per_block + warp_in_block; a < C; a += stride) {
        const int4 meta = P.cells.meta[a];
        const int sys = meta.w;
        if (sys != wt.sys) {
            if (wt.sys >= 0) flush_tally(P, wt, lane);
            wt.sys = sys;
        }
        const SysDev &g = P.sys[sys];
        const unsigned nb = min(bot_in[a], (unsigned)meta.y);
        const unsigned nt = min(top_in[a], (unsigned)meta.y - nb);
        int n = (int)(nb + nt);
        if (n > P.smem_cap) {
            wt.err |= DSMC_EBIT_SMEM;
            n = P.smem_cap;
        }
        const bool collide = P.do_collide && MODE != MODE_SORT;
        bool sample = P.do_sample && MODE != MODE_SORT && g.sample_interval > 0 && step > 0 &&
                      (step % (uint32_t)g.sample_interval) == 0 && step >= (uint32_t)g.sample_begin;
        const bool need_order = collide || sample;

        // Stage velocities (and ids) in shared memory.
        if (MODE != MODE_SORT) {
            for (int s = lane; s < n; s += 32) {
                real v[3];
                uint32_t id;
                Prec::stage_load(Ain, Bin, cell_slot(meta.x, meta.y, nb, nt, s), v, id);
                st.vx[s] = v[0];
                st.vy[s] = v[1];
                st.vz[s] = v[2];
                st.id[s] = id;
            }
            __syncwarp();
        }
        if (need_order) {
            // Members in id order: rank = number of smaller ids.
            for (int s = lane; s < n; s += 32) {
                const uint32_t mine = st.id[s];
                int rank = 0;
                for (int q = 0; q < n; ++q) rank += st.id[q] < mine;
                st.perm[rank] = (uint16_t)s;
            }
            __syncwarp();
        }
        if (collide) {
            if (lane == 0) {
                double4 cs = P.cells.state[a];
                ntc_collide<Prec>(g, meta.z, step, n, cs.z, cs.x, cs.y, st, wt.collisions, wt.candidates);
                P.cells.state[a] = cs;
            }
            __syncwarp();
        }
        if (sample) {
            double m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int r0 = 0; r0 < n; r0 += 32) {  // y-binned profiles, member by member
                const int r = r0 + lane;
                const bool ok = r < n;
                int bin = 0;
                double vz = 0;
                if (ok) {
                    const int s = st.perm[r];
                    vz = (double)st.vz[s];
                    bin = profile_bin(g, Prec::y_of(g, Ain[cell_slot(meta.x, meta.y, nb, nt, s)]));
                }
                profile_add_warp(g, ok, bin, 1.0, vz, 0.5 * g.mass * vz * vz);
                if (ok) profile_vx(g, (double)st.vx[st.perm[r]]);
            }
            for (int r = lane; r < n; r += 32) {
                const int s = st.perm[r];
                const double x = (double)st.vx[s], y = (double)st.vy[s], z = (double)st.vz[s];
                m[0] += 1.0;
                m[1] += x;
                m[2] += y;
                m[3] += z;
                m[4] += x * x;
                m[5] += y * y;
                m[6] += z * z;
            }
#pragma unroll
            for (int q = 0; q < 7; ++q) m[q] = warp_sum_f64(m[q]);
            if (lane == 0) {
                double *M = P.cells.mom + 8 * (size_t)a;
#pragma unroll
                for (int q = 0; q < 7; ++q) M[q] += m[q];
                M[7] += m[4] + m[5] + m[6];
                if (a == g.active_begin) atomicAdd(&P.tally[sys].samples, 1ull);
            }
        }
        if (MODE == MODE_FUSED || MODE == MODE_SORT) {
            // this pass writes only top slots; clear the set the pass after next fills
            if (lane == 0) {
                P.cells.bot[P.cclear][a] = 0;
                P.cells.top[P.cclear][a] = 0;
            }
        }

        // Move (or pass through) and place every particle.
        const int chunks = (n + 31) >> 5;
        for (int ch = 0; ch < chunks; ++ch) {
            const int s = ch * 32 + lane;
            const bool valid = s < n;
            Particle p;
            unsigned key = 0xffffffffu;
            const unsigned addr = cell_slot(meta.x, meta.y, nb, nt, (unsigned)s);
            if (valid) {
                RecA ra = Ain[addr];
                RecB rb = Bin[addr];
                Prec::unpack(ra, rb, p);
                if (MODE != MODE_SORT) {
                    p.v[0] = st.vx[s];
                    p.v[1] = st.vy[s];
                    p.v[2] = st.vz[s];
                }
                if (MODE == MODE_SORT) {
                    key = P.cells.key[addr];
                } else if (P.do_move) {
                    Prec::accelerate(g, p);
                    MoveTally mt;
                    mt.wall_hits = mt.reseeds = 0;
                    mt.cross[0] = mt.cross[1] = mt.cross[2] = 0;
                    mt.err = 0;
                    const bool left_voxel = Prec::move(g, p, move_step, mt);
                    wt.wall_hits += mt.wall_hits;
                    wt.reseeds += mt.reseeds;
                    wt.cross[0] += mt.cross[0];
                    wt.cross[1] += mt.cross[1];
                    wt.cross[2] += mt.cross[2];
                    wt.err |= mt.err;
                    wt.moved += 1;
                    const int ac = left_voxel ? __ldg(g.cell_map + Prec::cell_global(g, p)) : a;
                    if (ac < 0) {
                        // The reference aborts here (dsmc/system.h:134-142); the
                        // particle sits in solid and its next move re-seeds it
                        // (dsmc/moleculemover.cpp:57-60), so keep it in this cell.
                        wt.err |= DSMC_EBIT_STRANDED;
                        ++wt.stranded;
                        key = (unsigned)a;
                    } else {
                        key = (unsigned)ac;
                    }
                } else {
                    key = (unsigned)a;
                }
            }
            if (MODE == MODE_INPLACE) {
                if (valid) {
                    RecA ra;
                    RecB rb;
                    Prec::pack(p, ra, rb);
                    if (P.do_move) {
                        Aio[addr] = ra;
                        P.cells.key[addr] = key;
                    }
                    if (P.do_move || collide) Bio[addr] = rb;
                }
            } else {
                // Warp-aggregated counting-sort insert into the new cell's top slots.
                const unsigned peers = __match_any_sync(0xffffffffu, key);
                const int leader = __ffs(peers) - 1;
                const unsigned lower = peers & ((1u << lane) - 1u);
                unsigned slot0 = 0;
                if (valid && lane == leader) slot0 = atomicAdd(&top_out[key], (unsigned)__popc(peers));
                slot0 = __shfl_sync(0xffffffffu, slot0, leader);
                bool spilled = false;
                if (valid) {
                    const unsigned k = slot0 + (unsigned)__popc(lower);
                    RecA ra;
                    RecB rb;
                    Prec::pack(p, ra, rb);
                    const int4 km = key == (unsigned)a ? meta : P.cells.meta[key];
                    // a top slot may not reach the slots the cell's owner can
                    // fill from the bottom (at most its input occupancy)
                    const unsigned room =
                        P.top_only ? (unsigned)km.y
                                   : (unsigned)km.y - min((unsigned)km.y, bot_in[key] + top_in[key]);
                    if (k < room) {
                        const unsigned dst = (unsigned)(km.x + km.y) - 1u - k;
                        Aout[dst] = ra;
                        Bout[dst] = rb;
                    } else {
                        spilled = true;
                        const unsigned si = atomicAdd(&P.status->spill, 1u);
                        if (si < P.parts.spill_cap) {
                            SpillRec &sr = P.parts.spill[si];
                            if (sizeof(real) == 8) {
                                sr.ra = *reinterpret_cast<const double4 *>(&ra);
                                sr.rb = *reinterpret_cast<const double4 *>(&rb);
                            } else {
                                sr.a = *reinterpret_cast<const uint4 *>(&ra);
                                sr.b = *reinterpret_cast<const uint4 *>(&rb);
                            }
                            sr.cell = (int)key;
                        } else {
                            wt.err |= DSMC_EBIT_SPILL_FULL;
                        }
                    }
                }
                // spilled slots are given back, so the counter ends at the
                // number of particles actually placed in the top segment
                const unsigned over = __ballot_sync(0xffffffffu, spilled) & peers;
                if (valid && lane == leader && over) atomicSub(&top_out[key], (unsigned)__popc(over));
            }
        }
    }
    if (wt.sys >= 0) flush_tally(P, wt, lane);

    // End of pass: the last block to finish advances the step and halts the
    // pipeline if anything spilled or failed.
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

}  // namespace dsmc
