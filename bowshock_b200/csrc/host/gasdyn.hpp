// Exact relations of compressible flow used to place grids and to check
// results: shock relations (src/validation/gas-dynamics.ts) and the
// Taylor-Maccoll cone solution (src/validation/taylor-maccoll.ts).
#pragma once

#include <string>

namespace bs {

struct NormalShock {
  double pressure_ratio, density_ratio, downstream_mach;
};
struct ObliqueShock {
  double beta, pressure_ratio, density_ratio, downstream_mach;
};
struct ConeFlow {
  double shock_angle, post_shock_mach, post_shock_pressure_ratio, surface_mach,
      surface_pressure_ratio, surface_pressure_coefficient;
};

// Each returns "" on success or the reference's RangeError message.
std::string mach_angle(double mach, double* out);                         // gas-dynamics.ts:11-14
double deflection_angle(double mach, double beta, double gamma);          // :21-26
std::string normal_shock(double mach, double gamma, NormalShock* out);    // :88-96
double max_deflection_wave_angle(double mach, double gamma);              // :70-82
std::string oblique_shock(double mach, double theta, double gamma, ObliqueShock* out);  // :40-67
double stagnation_pressure_ratio(double mach, double gamma);              // :128-130
double prandtl_meyer(double mach, double gamma);                          // :99-104
std::string taylor_maccoll(double mach, double cone, double gamma, double tolerance,
                           ConeFlow* out);                                // taylor-maccoll.ts:153-216

}  // namespace bs
