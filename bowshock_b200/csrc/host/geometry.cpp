// Nose and body geometry (src/geometry/nose.ts, src/geometry/body.ts).
#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

namespace bs {

namespace {

// Below this ogive parameter the profile is the cone (OGIVE_CONE_LIMIT,
// nose.ts:104).
constexpr double kOgiveConeLimit = 0.001;

struct OgiveArc {
  double stretch, length, rho, xc, y0;
};

// The ogive family's circular arc (ogiveArc, nose.ts:115-127): a nose
// shorter than its radius is the ogive of length R compressed along x.
OgiveArc ogive_arc(double p, double L, double R) {
  OgiveArc a;
  a.stretch = L < R ? R / L : 1;
  a.length = std::max(L, R);
  const double pr = p * R;
  const double k = (2 - p) * a.length;
  a.rho = std::sqrt(((a.length * a.length + R * R) * (k * k + pr * pr)) / (4 * pr * pr));
  a.xc = a.length / p;
  a.y0 = std::sqrt(std::max(0.0, a.rho * a.rho - a.xc * a.xc));
  return a;
}

double ogive_radius(double p, double x, double L, double R) {  // nose.ts:129-139
  if (p < kOgiveConeLimit) return (R * x) / L;
  const OgiveArc a = ogive_arc(p, L, R);
  const double s = x * a.stretch;
  if (s <= 0) return 0;
  const double d = a.xc - s;
  // The cancellation-free form of sqrt(rho^2 - (xc - s)^2) - y0.
  return (s * (2 * a.xc - s)) / (std::sqrt(std::max(0.0, a.rho * a.rho - d * d)) + a.y0);
}

}  // namespace

std::string validate_body(const Body& body) {
  const Nose& n = body.nose;
  if (!(n.length > 0 && n.base_radius > 0)) return "a nose needs a positive length and base radius";
  auto in_range = [](double v, double lo, double hi) { return v >= lo && v <= hi; };
  switch (n.kind) {
    case NOSE_OGIVE:
      if (!in_range(n.parameter, 0, 1)) return "the ogive parameter must lie in [0, 1]";
      break;
    case NOSE_POWER:
      if (!(n.parameter > 0 && n.parameter <= 1))
        return "the power-series exponent must lie in (0, 1]";
      break;
    case NOSE_PARABOLIC:
      if (!in_range(n.parameter, 0, 1)) return "the parabolic parameter must lie in [0, 1]";
      break;
    case NOSE_HAACK:
      if (!in_range(n.parameter, 0, 1.0 / 3.0)) return "the Haack parameter must lie in [0, 1/3]";
      break;
    case NOSE_CONICAL:
    case NOSE_ELLIPSOID:
      break;
    default:
      return "unknown nose shape";
  }
  if (!(body.cylinder_length >= 0)) return "the cylinder length cannot be negative";
  return "";
}

double nose_radius(const Nose& nose, double x) {
  const double L = nose.length, R = nose.base_radius;
  const double t = std::min(std::max(x / L, 0.0), 1.0);
  switch (nose.kind) {
    case NOSE_CONICAL:
      return R * t;
    case NOSE_OGIVE:
      return ogive_radius(nose.parameter, t * L, L, R);
    case NOSE_ELLIPSOID:
      return R * std::sqrt(std::max(0.0, 1 - (1 - t) * (1 - t)));
    case NOSE_POWER:
      return R * std::pow(t, nose.parameter);
    case NOSE_PARABOLIC: {
      const double k = nose.parameter;
      return (R * (2 * t - k * t * t)) / (2 - k);
    }
    default: {  // NOSE_HAACK
      const double theta = std::acos(1 - 2 * t);
      const double s = std::sin(theta);
      const double area = theta - std::sin(2 * theta) / 2 + nose.parameter * s * s * s;
      return R * std::sqrt(std::max(0.0, area) / M_PI);
    }
  }
}

double nose_tip_slope(const Nose& nose) {
  const double L = nose.length, R = nose.base_radius;
  const double inf = std::numeric_limits<double>::infinity();
  switch (nose.kind) {
    case NOSE_CONICAL:
      return R / L;
    case NOSE_OGIVE: {
      if (nose.parameter < kOgiveConeLimit) return R / L;
      const OgiveArc a = ogive_arc(nose.parameter, L, R);
      return (a.xc / a.y0) * a.stretch;
    }
    case NOSE_PARABOLIC:
      return (2 * R) / ((2 - nose.parameter) * L);
    case NOSE_POWER:
      return nose.parameter == 1 ? R / L : inf;
    default:  // ellipsoid, Haack
      return inf;
  }
}

double nose_base_slope(const Nose& nose) {
  const double L = nose.length, R = nose.base_radius;
  switch (nose.kind) {
    case NOSE_CONICAL:
      return R / L;
    case NOSE_OGIVE: {
      if (nose.parameter < kOgiveConeLimit) return R / L;
      const OgiveArc a = ogive_arc(nose.parameter, L, R);
      const double d = a.xc - a.length;
      return (d / std::sqrt(a.rho * a.rho - d * d)) * a.stretch;
    }
    case NOSE_PARABOLIC:
      return (2 * R * (1 - nose.parameter)) / ((2 - nose.parameter) * L);
    case NOSE_POWER:
      return (nose.parameter * R) / L;
    default:
      return 0;
  }
}

double body_length(const Body& b) { return b.nose.length + b.cylinder_length; }

double body_radius(const Body& b, double x) {
  if (x <= 0) return 0;
  return x < b.nose.length ? nose_radius(b.nose, x) : b.nose.base_radius;
}

std::vector<double> body_breakpoints(const Body& b) {
  if (b.cylinder_length > 0) return {0, b.nose.length, body_length(b)};
  return {0, b.nose.length};
}

}  // namespace bs
