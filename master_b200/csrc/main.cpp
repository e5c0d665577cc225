// dsmc_b200_main: the reference's solver executable (dsmc/main.cpp) over
// libdsmc_b200.  Reads dsmc.ini from the working directory, sets the system
// up from the ini's world folder, runs `timesteps` steps (System::step +
// StatisticsSampler::sample), prints the run's time analysis in the
// reference's layout, and at the end writes the particle state
// (state_files/state0000.bin) and the Tocontinue counters
// (t steps collisions wall_collisions) as the reference does.  With
// load_previous_state = true in the ini it continues from those two files
// (dsmc/main.cpp:37-55, dsmc/system.cpp:412-415).
//
//   dsmc_b200_main [--fp64] [--device N]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/stat.h>
#include <vector>

#include "dsmc_b200.h"

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
    if ((rc = dsmc_step(ctx, s.timesteps))) return die(ctx, "System::step", rc);
    if ((rc = dsmc_sync(ctx))) return die(ctx, "System::step", rc);
    dsmc_tallies t;
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
