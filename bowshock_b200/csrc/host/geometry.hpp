// Nose profiles and bodies of revolution: the host-side geometry from which
// grids are generated. Restates src/geometry/nose.ts and src/geometry/body.ts.
#pragma once

#include <string>
#include <vector>

namespace bs {

enum NoseKind { NOSE_CONICAL = 0, NOSE_OGIVE = 1, NOSE_ELLIPSOID = 2, NOSE_POWER = 3,
                NOSE_PARABOLIC = 4, NOSE_HAACK = 5 };

// Nose (src/geometry/nose.ts:13-40): `parameter` is the ogive parameter, the
// power-series exponent, the parabolic K or the Haack C, as the kind needs.
struct Nose {
  int kind = NOSE_CONICAL;
  double parameter = 0;
  double length = 1;
  double base_radius = 0.5;
};

// Body (src/geometry/body.ts:8-13): a nose followed by a cylinder.
struct Body {
  Nose nose;
  double cylinder_length = 0;
};

// Returns "" or the reference's RangeError message (nose.ts:43-71, body.ts:15-18).
std::string validate_body(const Body& body);
double nose_radius(const Nose& nose, double x);      // nose.ts:74-97
double nose_tip_slope(const Nose& nose);             // nose.ts:145-165
double nose_base_slope(const Nose& nose);            // nose.ts:174-196
double body_length(const Body& body);                // body.ts:20-22
double body_radius(const Body& body, double x);      // body.ts:25-28
std::vector<double> body_breakpoints(const Body& b); // body.ts:31-32

}  // namespace bs
