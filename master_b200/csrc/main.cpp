// dsmc_b200_main: the reference's solver executable (dsmc/main.cpp) over
// libdsmc_b200.  Reads dsmc.ini from the working directory, sets the system
// up from the ini's world folder, runs `timesteps` steps (System::step +
// StatisticsSampler::sample), prints the run's time analysis in the
// reference's layout, and at the end writes the particle state
// (state_files/state0000.bin) and the Tocontinue counters
// (t steps collisions wall_collisions) as the reference does, and the
// sampler's statistics/ files (energy, temperature, flow rates, pressure and
// permeability per sample; profiles and the v_x histogram at the end).  With
// load_previous_state = true in the ini it continues from those two files
// (dsmc/main.cpp:37-55, dsmc/system.cpp:412-415).
//
//   dsmc_b200_main [--fp64] [--device N]
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/stat.h>
#include <vector>

#include "dsmc_b200.h"

// The statistics files of DSMC_IO (dsmc/dsmc_io.cpp:33-47) with the lines
// each measurement writes (dsmc/statisticalproperty.cpp).
struct Statistics {
    static constexpr int kFiles = 13;
    const char *names[kFiles] = {"energy", "velocity", "velocity_distribution", "number_flow_rate", "permeability",
                                 "density", "linear_density", "num_molecules_file", "pressure", "temperature",
                                 "linear_pressure", "linear_temperature", "volumetric_flow_rate"};
    FILE *f[kFiles] = {};
    double permeability = 0;
    FILE *file(const char *name) {
        for (int i = 0; i < kFiles; ++i)
            if (!std::strcmp(names[i], name)) return f[i];
        return nullptr;
    }
    bool open() {
        mkdir("statistics", 0755);
        for (int i = 0; i < kFiles; ++i) {
            char path[128];
            std::snprintf(path, sizeof(path), "statistics/%s.txt", names[i]);
            if (!(f[i] = std::fopen(path, "w"))) return false;
        }
        return true;
    }
    void record(const dsmc_measures &m) {
        std::fprintf(file("energy"), "%f %E\n", m.t_ns, m.energy_eV);
        std::fprintf(file("temperature"), "%f %f\n", m.t_ns, m.temperature_K);
        std::fprintf(file("number_flow_rate"), "%f %E\n", m.t_ns, m.number_flow_rate);
        std::fprintf(file("volumetric_flow_rate"), "%f %E\n", m.t_ns, m.volumetric_flow_rate);
        std::fprintf(file("pressure"), "%f %E\n", m.t_ns, m.pressure_Pa);
        permeability = m.permeability_darcy;
        // StatisticsSampler::sample's progress line
        std::printf("%llu   t=%gns   T=%gK   Collisions: %llu   Wall collisions: %llu   Pressure: %gPa   Molecules: %llu\n",
                    (unsigned long long)m.step, m.t_ns, m.temperature_K, (unsigned long long)m.collisions,
                    (unsigned long long)m.wall_collisions, m.pressure_Pa, (unsigned long long)m.molecules);
    }
    int finalize(dsmc_ctx *ctx, int sys) {
        int bins = 0;
        int rc = dsmc_profiles_get(ctx, sys, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, &bins);
        if (rc && rc != DSMC_ERR_CAPACITY) return rc;
        std::vector<double> count(bins), vz(bins), T(bins), P(bins), vc(bins), vn(bins);
        if ((rc = dsmc_profiles_get(ctx, sys, bins, count.data(), vz.data(), T.data(), P.data(), vc.data(), vn.data(),
                                    &bins)))
            return rc;
        for (int b = 0; b < bins; ++b) {
            std::fprintf(file("velocity"), "%E ", vz[b]);
            std::fprintf(file("linear_temperature"), "%E ", T[b]);
            std::fprintf(file("linear_pressure"), "%E ", P[b]);
            std::fprintf(file("velocity_distribution"), "%f %ld\n", vc[b], (long)vn[b]);
        }
        std::fprintf(file("permeability"), "%E\n", permeability);
        for (int i = 0; i < kFiles; ++i) {
            if (f[i] && std::fclose(f[i])) rc = DSMC_ERR_IO;
            f[i] = nullptr;
        }
        return rc;
    }
};

static int die(dsmc_ctx *ctx, const char *what, int rc) {
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, dsmc_last_error(ctx));
    if (ctx) dsmc_ctx_destroy(ctx);
    return 1;
}

int main(int argc, char **argv) {
    int device = 0, precision = DSMC_PREC_SPLIT32;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--fp64")) {
            precision = DSMC_PREC_FP64;
        } else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
            device = std::atoi(argv[++i]);
        } else {
            std::fprintf(stderr, "usage: %s [--fp64] [--device N]\n", argv[0]);
            return 2;
        }
    }
    const auto t_start = std::chrono::steady_clock::now();
    std::printf("\nDSMC B200 SOLVER (libdsmc_b200)\n\n");

    dsmc_settings s;
    int rc = dsmc_settings_load_ini("dsmc.ini", &s);
    if (rc) return die(nullptr, "reading dsmc.ini", rc);
    dsmc_ctx *ctx = nullptr;
    if ((rc = dsmc_ctx_create(device, precision, &ctx))) return die(ctx, "creating the context", rc);
    int sys = -1;
    if ((rc = dsmc_system_add_world(ctx, &s, &sys))) return die(ctx, "System::initialize", rc);
    if (s.load_previous_state) {
        double t = 0;
        uint64_t steps = 0, collisions = 0, walls = 0;
        if ((rc = dsmc_tocontinue_read("Tocontinue", &t, &steps, &collisions, &walls))) return die(ctx, "Tocontinue", rc);
        int64_t n = 0;
        if ((rc = dsmc_state_file_read("state_files/state0000.bin", 0, nullptr, nullptr, &n)))
            return die(ctx, "load_state_from_file_binary", rc);
        std::vector<double> r(3 * n), v(3 * n);
        if ((rc = dsmc_state_file_read("state_files/state0000.bin", n, r.data(), v.data(), &n)))
            return die(ctx, "load_state_from_file_binary", rc);
        if ((rc = dsmc_particles_set(ctx, sys, n, r.data(), v.data()))) return die(ctx, "setting the state", rc);
        if ((rc = dsmc_continue_from(ctx, sys, t, steps, collisions, walls))) return die(ctx, "continuing", rc);
    } else if ((rc = dsmc_particles_init(ctx, sys, -1))) {
        return die(ctx, "setup_molecules", rc);
    }
    if ((rc = dsmc_sync(ctx))) return die(ctx, "initialisation", rc);
    const auto t_init = std::chrono::steady_clock::now();

    // per-kernel timers: the counterpart of the reference's stage timers
    if ((rc = dsmc_ctx_set_timing(ctx, 1))) return die(ctx, "timers", rc);
    Statistics stats;
    if (!stats.open()) return die(ctx, "opening statistics/", DSMC_ERR_IO);
    dsmc_tallies t;
    if ((rc = dsmc_tallies_get(ctx, sys, &t))) return die(ctx, "tallies", rc);
    // The reference's loop (dsmc/main.cpp:57-64): System::step, then
    // StatisticsSampler::sample, which records on steps % interval == 0.  The
    // GPU runs the steps between two samples back to back.
    const uint64_t interval = s.statistics_interval > 0 ? (uint64_t)s.statistics_interval : 0;
    uint64_t step = t.step;
    for (long left = s.timesteps; left > 0;) {
        long chunk = left;
        if (interval) chunk = (long)std::min<uint64_t>((uint64_t)left, (step / interval + 1) * interval - step);
        if ((rc = dsmc_step(ctx, (int)chunk))) return die(ctx, "System::step", rc);
        left -= chunk;
        step += chunk;
        if (interval && step % interval == 0) {
            dsmc_measures m;
            if ((rc = dsmc_measures_get(ctx, sys, &m))) return die(ctx, "StatisticsSampler::sample", rc);
            stats.record(m);
        }
    }
    if ((rc = dsmc_sync(ctx))) return die(ctx, "System::step", rc);
    if ((rc = dsmc_tallies_get(ctx, sys, &t))) return die(ctx, "tallies", rc);
    dsmc_system_info info;
    if ((rc = dsmc_system_info_get(ctx, sys, &info))) return die(ctx, "system info", rc);
    double ms[4] = {0, 0, 0, 0};
    int64_t passes = 0;
    dsmc_pass_times_get(ctx, ms, &passes);
    const auto t_end = std::chrono::steady_clock::now();

    const double total = std::chrono::duration<double>(t_end - t_start).count();
    const double init = std::chrono::duration<double>(t_init - t_start).count();
    const double colliding = ms[0] * 1e-3, moving = (ms[1] + ms[2] + ms[3]) * 1e-3;
    auto pct = [&](double x) { return total > 0 ? 100.0 * x / total : 0.0; };
    std::printf("\nProgram finished after %ld seconds. Time analysis:\n", (long)total);
    std::printf("      Moving            : %.2f s ( %.2f%% )   (move_cells, place_movers, place_walls%s)\n", moving,
                pct(moving), passes ? "" : ": not timed for this precision");
    std::printf("      Colliding         : %.2f s ( %.2f%% )   (collide_cells, sampling included)\n", colliding,
                pct(colliding));
    std::printf("      System initialize : %.2f s ( %.2f%% )\n", init, pct(init));
    std::printf("      TOTAL             : %.2f s\n", total);
    std::printf("\n%.2f timesteps / second. \n", s.timesteps / total);
    std::printf("%.2fk atom-timesteps / second. \n", (double)info.num_particles * s.timesteps / (1000.0 * total));
    std::printf("collisions %llu, wall collisions %llu, T = %.3f K\n", (unsigned long long)t.collisions,
                (unsigned long long)t.wall_collisions, t.temperature);

    // StatisticsSampler::finalize (dsmc/statisticssampler.cpp:68-74)
    if ((rc = stats.finalize(ctx, sys))) return die(ctx, "StatisticsSampler::finalize", rc);

    // save_state_to_file_binary (dsmc/dsmc_io.cpp:82-118) and Tocontinue
    std::vector<double> r(3 * info.num_particles), v(3 * info.num_particles);
    int64_t n = 0;
    if ((rc = dsmc_particles_get(ctx, sys, info.num_particles, r.data(), v.data(), nullptr, &n)))
        return die(ctx, "reading the state", rc);
    mkdir("state_files", 0755);
    if ((rc = dsmc_state_file_write("state_files/state0000.bin", n, r.data(), v.data())))
        return die(ctx, "save_state_to_file_binary", rc);
    if ((rc = dsmc_tocontinue_write("Tocontinue", t.time, t.step, t.collisions, t.wall_collisions)))
        return die(ctx, "Tocontinue", rc);
    dsmc_ctx_destroy(ctx);
    return 0;
}
