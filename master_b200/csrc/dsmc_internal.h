// Internal declarations shared by the host files of libdsmc_b200.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace dsmc {

void set_thread_error(const std::string &msg);
const char *thread_error();

// Reduced units of the reference (dsmc/unitconverter.cpp:3-21).
struct Units {
    double m0, L0, E0, E0ev, kb, t0, T0, v0, a0, P0, number_density0;
    Units();
    double temperature_from_SI(double T) const { return T / T0; }
    double temperature_to_SI(double T) const { return T0 * T; }
    double number_density_from_SI(double d) const { return d / number_density0; }
    double time_to_SI(double t) const { return t0 * t; }
    double velocity_to_SI(double v) const { return v * v0; }
    double pressure_to_SI(double p) const { return P0 * p; }
    double energy_to_eV(double E) const { return E0ev * E; }
    double permeability_to_darcy(double k) const { return k * L0 * L0 * 1e4; }
};

// Park-Miller + Bays-Durham "ran1" (Numerical Recipes in C, 2nd ed., 7.1).
struct Ran1 {
    long idum, iy, iv[32];
    explicit Ran1(long seed);
    double next();
};

struct IniFile {
    struct Item {
        std::string name, str;
        double num;
    };
    std::vector<Item> items;
    bool load(const std::string &path);
    const Item *find(const std::string &key) const;
};

}  // namespace dsmc
