// Shock relations and the Taylor-Maccoll cone solution, in FP64 on the host.
// The algorithms follow src/validation/gas-dynamics.ts and
// src/validation/taylor-maccoll.ts step for step (bisection brackets,
// adaptive RK4 with step doubling), so that grids placed from the cone shock
// angle match the reference's.
#include "gasdyn.hpp"

#include <functional>

#include <algorithm>
#include <cmath>
#include <limits>

namespace bs {

std::string mach_angle(double mach, double* out) {
  if (!(mach >= 1)) return "the Mach angle needs M >= 1";
  *out = std::asin(1 / mach);
  return "";
}

double deflection_angle(double mach, double beta, double gamma) {
  const double s = std::sin(beta);
  const double m2s2 = mach * mach * s * s;
  return std::atan((2 * (m2s2 - 1)) /
                   (std::tan(beta) * (mach * mach * (gamma + std::cos(2 * beta)) + 2)));
}

std::string normal_shock(double mach, double gamma, NormalShock* out) {
  if (!(mach >= 1)) return "a shock needs a supersonic normal Mach number";
  const double m2 = mach * mach;
  out->pressure_ratio = 1 + ((2 * gamma) / (gamma + 1)) * (m2 - 1);
  out->density_ratio = ((gamma + 1) * m2) / ((gamma - 1) * m2 + 2);
  out->downstream_mach = std::sqrt(((gamma - 1) * m2 + 2) / (2 * gamma * m2 - (gamma - 1)));
  return "";
}

double max_deflection_wave_angle(double mach, double gamma) {
  // Golden-section search of the unimodal deflection over [mu, pi/2].
  double a = std::asin(1 / mach);
  double b = M_PI / 2;
  const double r = (std::sqrt(5.0) - 1) / 2;
  for (int k = 0; k < 200 && b - a > 1e-14; k++) {
    const double c = b - r * (b - a);
    const double d = a + r * (b - a);
    if (deflection_angle(mach, c, gamma) < deflection_angle(mach, d, gamma))
      a = c;
    else
      b = d;
  }
  return 0.5 * (a + b);
}

std::string oblique_shock(double mach, double theta, double gamma, ObliqueShock* out) {
  double lo;
  std::string e = mach_angle(mach, &lo);
  if (!e.empty()) return e;
  const double betaMax = max_deflection_wave_angle(mach, gamma);
  if (theta > deflection_angle(mach, betaMax, gamma))
    return "deflection exceeds the detachment angle; the shock is detached";
  double hi = betaMax;
  for (int k = 0; k < 200 && hi - lo > 1e-15; k++) {
    const double mid = 0.5 * (lo + hi);
    if (deflection_angle(mach, mid, gamma) < theta)
      lo = mid;
    else
      hi = mid;
  }
  const double beta = 0.5 * (lo + hi);
  NormalShock n;
  e = normal_shock(mach * std::sin(beta), gamma, &n);
  if (!e.empty()) return e;
  out->beta = beta;
  out->pressure_ratio = n.pressure_ratio;
  out->density_ratio = n.density_ratio;
  out->downstream_mach = n.downstream_mach / std::sin(beta - theta);
  return "";
}

double stagnation_pressure_ratio(double mach, double gamma) {
  return std::pow(1 + 0.5 * (gamma - 1) * mach * mach, gamma / (gamma - 1));
}

double prandtl_meyer(double mach, double gamma) {
  const double k = (gamma + 1) / (gamma - 1);
  const double m = std::sqrt(mach * mach - 1);
  return std::sqrt(k) * std::atan(m / std::sqrt(k)) - std::atan(m);
}

namespace {

// V / V_max for Mach number M, and its inverse (taylor-maccoll.ts:38-45).
double speed_from_mach(double mach, double gamma) {
  return 1 / std::sqrt(1 + 2 / ((gamma - 1) * mach * mach));
}
double mach_from_speed(double speed, double gamma) {
  return std::sqrt(2 / ((gamma - 1) * (1 / (speed * speed) - 1)));
}

// The Taylor-Maccoll equation as a first-order system in theta
// (taylor-maccoll.ts:66-71): d(V_r)/dtheta = V_theta and dV_theta/dtheta.
void tm_derivatives(double theta, double vr, double vt, double gamma, double* dr, double* dt) {
  const double a = 0.5 * (gamma - 1) * (1 - vr * vr - vt * vt);
  *dr = vt;
  *dt = (vr * vt * vt - a * (2 * vr + vt / std::tan(theta))) / (a - vt * vt);
}

void rk4(double theta, double vr, double vt, double h, double gamma, double* r, double* t) {
  double k1r, k1t, k2r, k2t, k3r, k3t, k4r, k4t;
  tm_derivatives(theta, vr, vt, gamma, &k1r, &k1t);
  tm_derivatives(theta + h / 2, vr + (h / 2) * k1r, vt + (h / 2) * k1t, gamma, &k2r, &k2t);
  tm_derivatives(theta + h / 2, vr + (h / 2) * k2r, vt + (h / 2) * k2t, gamma, &k3r, &k3t);
  tm_derivatives(theta + h, vr + h * k3r, vt + h * k3t, gamma, &k4r, &k4t);
  *r = vr + (h / 6) * (k1r + 2 * k2r + 2 * k3r + k4r);
  *t = vt + (h / 6) * (k1t + 2 * k2t + 2 * k3t + k4t);
}

// Integrate from the shock at angle beta towards the axis until V_theta
// vanishes (integrateToCone, taylor-maccoll.ts:78-145). Returns false if no
// cone corresponds to this shock.
bool integrate_to_cone(double mach, double beta, double gamma, double tol, double* cone,
                       double* surface_speed,
                       const std::function<void(double, double, double)>& record = nullptr) {
  NormalShock ns;
  if (!normal_shock(mach * std::sin(beta), gamma, &ns).empty()) return false;
  const double delta = deflection_angle(mach, beta, gamma);
  const double mach2 = ns.downstream_mach / std::sin(beta - delta);
  const double speed = speed_from_mach(mach2, gamma);
  double vr = speed * std::cos(beta - delta);
  double vt = -speed * std::sin(beta - delta);
  double theta = beta;
  double h = -1e-4 * beta;
  if (record) record(theta, vr, vt);
  while (theta > 1e-12) {
    h = std::max(h, -0.5 * theta);
    double fr, ft, hr, ht, r2, t2;
    rk4(theta, vr, vt, h, gamma, &fr, &ft);
    rk4(theta, vr, vt, h / 2, gamma, &hr, &ht);
    rk4(theta + h / 2, hr, ht, h / 2, gamma, &r2, &t2);
    const double err = std::max(std::fabs(r2 - fr), std::fabs(t2 - ft)) / 15;
    if (!(err <= tol)) {
      h /= 2;
      if (std::fabs(h) < 1e-14 * theta) return false;
      continue;
    }
    const double nextR = r2 + (r2 - fr) / 15;
    const double nextT = t2 + (t2 - ft) / 15;
    if (nextT >= 0) {
      if (std::fabs(h) > 1e-12) {
        h /= 2;
        continue;
      }
      const double f = vt / (vt - nextT);
      *cone = theta + f * h;
      *surface_speed = vr + f * (nextR - vr);
      if (record) record(*cone, *surface_speed, 0);
      return true;
    }
    theta += h;
    vr = nextR;
    vt = nextT;
    if (record) record(theta, vr, vt);
    h *= std::min(2.0, 0.9 * std::pow(tol / std::max(err, 1e-300), 0.2));
  }
  return false;
}

}  // namespace

std::string taylor_maccoll(double mach, double cone, double gamma, double tol, ConeFlow* out) {
  if (!(cone > 0)) return "the cone half-angle must be positive";
  double mu;
  std::string e = mach_angle(mach, &mu);
  if (!e.empty()) return e;
  const double nan = std::numeric_limits<double>::quiet_NaN();
  auto cone_at = [&](double beta) {
    if (beta <= mu) return 0.0;
    double c, s;
    return integrate_to_cone(mach, beta, gamma, tol, &c, &s) ? c : nan;
  };
  double lo = mu, hi = mu, previous = 0;
  const double step_up = 0.5 * (M_PI / 180);
  for (;;) {
    hi += step_up;
    const double c = cone_at(hi);
    if (!(hi < M_PI / 2) || std::isnan(c) || c < previous)
      return "the shock detaches: no attached conical solution";
    if (c >= cone) break;
    lo = hi;
    previous = c;
  }
  for (int k = 0; k < 60 && hi - lo > 1e-15; k++) {
    const double mid = 0.5 * (lo + hi);
    if (cone_at(mid) < cone)
      lo = mid;
    else
      hi = mid;
  }
  const double beta = 0.5 * (lo + hi);
  double c, surface_speed;
  if (!integrate_to_cone(mach, beta, gamma, tol, &c, &surface_speed))
    return "integration failed to reach the cone";
  NormalShock ns;
  normal_shock(mach * std::sin(beta), gamma, &ns);
  const double delta = deflection_angle(mach, beta, gamma);
  out->shock_angle = beta;
  out->post_shock_mach = ns.downstream_mach / std::sin(beta - delta);
  out->post_shock_pressure_ratio = ns.pressure_ratio;
  out->surface_mach = mach_from_speed(surface_speed, gamma);
  out->surface_pressure_ratio = (ns.pressure_ratio *
                                 stagnation_pressure_ratio(out->post_shock_mach, gamma)) /
                                stagnation_pressure_ratio(out->surface_mach, gamma);
  out->surface_pressure_coefficient =
      (out->surface_pressure_ratio - 1) / (0.5 * gamma * mach * mach);
  return "";
}

std::string cone_flow_field(double mach, double cone, double gamma, double tol, ConeField* out) {
  std::string e = taylor_maccoll(mach, cone, gamma, tol, &out->flow);
  if (!e.empty()) return e;
  out->theta.clear();
  out->vr.clear();
  out->vt.clear();
  double c, speed;
  if (!integrate_to_cone(mach, out->flow.shock_angle, gamma, tol, &c, &speed,
                         [&](double t, double r, double v) {
                           out->theta.push_back(t);
                           out->vr.push_back(r);
                           out->vt.push_back(v);
                         }))
    return "integration failed to reach the cone";
  // V_theta' at each sample for the Hermite interpolant of V_theta.
  out->vtt.resize(out->theta.size());
  for (size_t k = 0; k < out->theta.size(); k++) {
    double dr;
    tm_derivatives(out->theta[k], out->vr[k], out->vt[k], gamma, &dr, &out->vtt[k]);
  }
  out->lowest = std::min(out->theta.back(), cone);
  return "";
}

std::string ConeField::at(double ray, double* speed, double* flow_angle) const {
  const size_t n = theta.size();
  if (!(ray <= theta[0] + 1e-15 && ray >= lowest - 1e-15)) return "the ray lies outside the conical flow";
  const double polar = std::min(std::max(ray, theta[n - 1]), theta[0]);
  size_t k = 0;
  while (k < n - 2 && theta[k + 1] > polar) k++;
  const double h = theta[k + 1] - theta[k];
  const double t = (polar - theta[k]) / h;
  auto hermite = [&](double f0, double f1, double d0, double d1) {
    return (2 * t * t * t - 3 * t * t + 1) * f0 + (t * t * t - 2 * t * t + t) * h * d0 +
           (-2 * t * t * t + 3 * t * t) * f1 + (t * t * t - t * t) * h * d1;
  };
  const double r = hermite(vr[k], vr[k + 1], vt[k], vt[k + 1]);
  const double v = hermite(vt[k], vt[k + 1], vtt[k], vtt[k + 1]);
  *speed = std::hypot(r, v);
  *flow_angle = polar + std::atan2(v, r);
  return "";
}

ShockState shock_state(const double free[4], double gamma, double mach, double nx, double ny) {
  const double a = std::sqrt(gamma * free[3] / free[0]);
  const double vn = free[1] * nx + free[2] * ny;
  const double speed = mach * a + vn;
  const double m2 = mach * mach;
  const double density_ratio = ((gamma + 1) * m2) / ((gamma - 1) * m2 + 2);
  const double pressure_ratio = 1 + ((2 * gamma) / (gamma + 1)) * (m2 - 1);
  // The relative normal speed is M a ahead of the shock and M a over the
  // density ratio behind it; behind it in the lab frame, along n:
  const double normal_velocity = speed - (mach * a) / density_ratio;
  ShockState s;
  s.w[0] = free[0] * density_ratio;
  s.w[1] = free[1] + (normal_velocity - vn) * nx;
  s.w[2] = free[2] + (normal_velocity - vn) * ny;
  s.w[3] = free[3] * pressure_ratio;
  s.speed = speed;
  s.normal_velocity = normal_velocity;
  s.mach = mach;
  return s;
}

ShockState compatible_shock(const double free[4], double gamma, double nx, double ny, double rho,
                            double a, double p, double un) {
  const double impedance = rho * a;
  const double target = p + impedance * un;
  auto mismatch = [&](double m) {
    const ShockState s = shock_state(free, gamma, m, nx, ny);
    return s.w[3] + impedance * s.normal_velocity - target;
  };
  double mach = 1;
  if (mismatch(1) < 0) {
    double low = 1, high = 2;
    while (mismatch(high) < 0) high *= 2;
    for (int k = 0; k < 100 && high - low > 1e-15 * high; k++) {
      const double mid = 0.5 * (low + high);
      if (mismatch(mid) < 0)
        low = mid;
      else
        high = mid;
    }
    mach = 0.5 * (low + high);
  }
  return shock_state(free, gamma, mach, nx, ny);
}

}  // namespace bs
