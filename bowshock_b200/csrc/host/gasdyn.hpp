// Exact relations of compressible flow used to place grids and to check
// results: shock relations (src/validation/gas-dynamics.ts) and the
// Taylor-Maccoll cone solution (src/validation/taylor-maccoll.ts).
#pragma once

#include <string>
#include <vector>

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

// The Taylor-Maccoll flow between the shock and the cone on any ray
// (coneFlowField, taylor-maccoll.ts:227-275): the integration's samples from
// the shock to the cone, V_r between them by cubic Hermite interpolation
// (V_theta is its derivative, V_theta' from the equation).
struct ConeField {
  ConeFlow flow;
  std::vector<double> theta, vr, vt, vtt;
  double lowest = 0;
  // Speed over the maximum speed, and flow angle, on the ray at polar angle `ray`.
  std::string at(double ray, double* speed, double* flow_angle) const;
};
std::string cone_flow_field(double mach, double cone, double gamma, double tolerance, ConeField* out);

// The state behind a normal shock of outward normal (nx, ny) that the free
// stream (rho, u, v, p) meets at relative normal Mach number `mach`, its
// speed along n and the post-shock normal velocity (shockState,
// src/solver/shock-fitting.ts:50-78).
struct ShockState {
  double w[4];  // rho, u, v, p
  double speed, normal_velocity, mach;
};
ShockState shock_state(const double free[4], double gamma, double mach, double nx, double ny);
// The shock consistent with the flow behind it through the u_n + a
// characteristic, p_s + rho a u_n,s = p + rho a u_n, by bisection on the
// relative Mach number; a Mach wave (M = 1) where no stronger shock fits
// (compatibleShock, src/solver/shock-fitting.ts:87-111).
ShockState compatible_shock(const double free[4], double gamma, double nx, double ny, double rho,
                            double a, double p, double un);

}  // namespace bs
