/*
 * TEST INFRASTRUCTURE: a link-time stand-in for the reference's random.cpp
 * (dsmc/random.cpp:8-91) that keeps the class Random of dsmc/random.h but
 * feeds the reference's own routines the same draws the GPU kernels take.
 *
 * The reference draws from one sequential ran1 stream per rank
 * (dsmc/random.cpp:43-68).  The GPU draws from counter-based streams, one per
 * particle for the mover and one per cell for the collide.  ref_harness.cpp
 * selects the stream (tape_select) before it hands each particle or cell to
 * the reference's MoleculeMover::move_molecule / Cell::collide, so both sides
 * consume draw 0, 1, 2, ... of the same stream in the same order.
 *
 * next_gauss keeps the reference's Box-Muller form (dsmc/random.cpp:21-25):
 * sqrt(-2 ln(1-U1)) * cos(6.283185307 U2); the U1 draw is taken first.  The
 * Cercignani-Lampis wall's sampler and its Bessel function are restated here
 * (they live in random.cpp) for the wall-model fixtures.
 */
#include <random.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include "philox.h"

namespace {
struct TapeCursor {
    uint64_t seed = 0;
    uint32_t stream = 0, step = 0, tag = 0;
    uint64_t k = 0;
    uint64_t draws_total = 0;
} g_cursor;
}  // namespace

extern "C" void tape_select(uint64_t seed, uint32_t stream, uint32_t step, uint32_t tag) {
    g_cursor.seed = seed;
    g_cursor.stream = stream;
    g_cursor.step = step;
    g_cursor.tag = tag;
    g_cursor.k = 0;
}

extern "C" uint64_t tape_position() { return g_cursor.k; }
extern "C" uint64_t tape_draws_total() { return g_cursor.draws_total; }

Random::Random(long seed, double alpha_n_, double alpha_t_) {
    *idum = seed;
    alpha_n = alpha_n_;
    alpha_t = alpha_t_;
    sqrt_one_minus_alpha = std::sqrt(1 - alpha_n);
    sqrt_one_minus_alpha_over_alpha = std::sqrt(1 - alpha_n) / alpha_n;
    sqrt_alpha_over_two = std::sqrt(alpha_n / 2);
    iy = 0;
    cercignani_lampis_normal_component_trials = 0;
    max_num_trials = 0;
}

double Random::next_double() {
    double u = oracle_uniform64(g_cursor.seed, g_cursor.stream, g_cursor.step, g_cursor.tag, g_cursor.k);
    g_cursor.k++;
    g_cursor.draws_total++;
    return u;
}

double Random::next_gauss() {
    double u1 = next_double();
    double u2 = next_double();
    return std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307 * u2);
}

// Random::bessel_i0 (dsmc/random.cpp:27-40): the modified Bessel function I0
// by the polynomial approximations of Abramowitz & Stegun (1964), eqs. 9.8.1
// and 9.8.2, in the reference's nesting.
inline double Random::bessel_i0(double x) {
    const double ax = std::fabs(x);
    if (ax < 3.75) {
        double y = x / 3.75;
        y *= y;
        return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 + y * (0.360768e-1 +
                                                                                               y * 0.45813e-2)))));
    }
    const double y = 3.75 / ax;
    return (std::exp(ax) / std::sqrt(ax)) *
           (0.39894228 +
            y * (0.1328592e-1 +
                 y * (0.225319e-2 +
                      y * (-0.157565e-2 +
                           y * (0.916281e-2 +
                                y * (-0.2057706e-1 + y * (0.2635537e-1 + y * (-0.1647633e-1 + y * 0.392377e-2))))))));
}

// Random::next_cercignani_lampis_normal_component (dsmc/random.cpp:70-91):
// rejection sampling of the reflected normal velocity.  The reference loops
// until it accepts; the GPU gives up after 100000 trials (DSMC_EBIT_WALL),
// and so does this stand-in.
double Random::next_cercignani_lampis_normal_component(double v_norm_in, double factor, double max_v_out) {
    max_v_out /= factor;
    v_norm_in /= factor;
    const double mu = sqrt_one_minus_alpha * v_norm_in;
    for (long trial = 0; trial < 100000; ++trial) {
        const double v_out = sqrt_alpha_over_two * next_gauss() + mu;
        const double u = next_double();
        const double arg = 2 * sqrt_one_minus_alpha_over_alpha * v_norm_in * v_out;
        const double b = v_out * std::exp(-arg) * bessel_i0(arg) / max_v_out;
        if (b >= u) return v_out * factor;
    }
    std::fprintf(stderr, "tape random: the Cercignani-Lampis sampler accepted nothing in 100000 trials\n");
    std::abort();
}
