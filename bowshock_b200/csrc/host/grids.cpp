// Grid generation on the host, in FP64 (src/grid/body-grid.ts,
// src/grid/spacing.ts, src/grid/quality.ts, src/grid/shapes.ts).
#include "grids.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>

#include "gasdyn.hpp"

namespace bs {

GridQuality grid_quality(int ni, int nj, const double* x, const double* y) {
  auto node = [&](int i, int j) { return size_t(i) + size_t(j) * (ni + 1); };
  GridQuality q{M_PI, M_PI, 1, 1, std::numeric_limits<double>::infinity()};
  std::vector<double> width(size_t(ni) * nj), height(size_t(ni) * nj);
  for (int j = 0; j < nj; j++) {
    for (int i = 0; i < ni; i++) {
      const size_t c[4] = {node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)};
      double area = 0;
      for (int k = 0; k < 4; k++) {
        const double ax = x[c[k]], ay = y[c[k]];
        const double bx = x[c[(k + 1) % 4]], by = y[c[(k + 1) % 4]];
        area += 0.5 * (ax * by - bx * ay);
        const double px = x[c[(k + 3) % 4]], py = y[c[(k + 3) % 4]];
        const double cosine = ((bx - ax) * (px - ax) + (by - ay) * (py - ay)) /
                              (std::hypot(bx - ax, by - ay) * std::hypot(px - ax, py - ay));
        const double angle = std::acos(std::max(-1.0, std::min(1.0, cosine)));
        q.min_angle = std::min(q.min_angle, angle);
        if (j == 0) q.min_wall_angle = std::min(q.min_wall_angle, angle);
      }
      q.min_area = std::min(q.min_area, area);
      auto side = [&](int a, int b) { return std::hypot(x[c[b]] - x[c[a]], y[c[b]] - y[c[a]]); };
      const double w = 0.5 * (side(0, 1) + side(3, 2));
      const double h = 0.5 * (side(0, 3) + side(1, 2));
      width[i + size_t(j) * ni] = w;
      height[i + size_t(j) * ni] = h;
      q.max_aspect_ratio = std::max(q.max_aspect_ratio, std::max(w / h, h / w));
    }
  }
  auto ratio = [](double a, double b) { return std::max(a / b, b / a); };
  for (int j = 0; j < nj; j++)
    for (int i = 0; i < ni; i++) {
      const size_t c = i + size_t(j) * ni;
      if (i + 1 < ni) q.max_size_ratio = std::max(q.max_size_ratio, ratio(width[c], width[c + 1]));
      if (j + 1 < nj) q.max_size_ratio = std::max(q.max_size_ratio, ratio(height[c], height[c + ni]));
    }
  return q;
}

std::vector<std::string> quality_failures(const GridQuality& q, const QualityLimits& l) {
  std::vector<std::string> out;
  char buf[160];
  auto deg = [](double r) { return r * 180 / M_PI; };
  if (!(q.min_area > 0)) out.push_back("a cell has non-positive area");
  if (!(q.min_angle >= l.min_angle)) {
    std::snprintf(buf, sizeof buf, "cell angle %.1f deg below %.1f deg", deg(q.min_angle),
                  deg(l.min_angle));
    out.push_back(buf);
  }
  if (!(q.min_wall_angle >= l.min_wall_angle)) {
    std::snprintf(buf, sizeof buf, "wall cell angle %.1f deg below %.1f deg",
                  deg(q.min_wall_angle), deg(l.min_wall_angle));
    out.push_back(buf);
  }
  if (!(q.max_size_ratio <= l.max_size_ratio)) {
    std::snprintf(buf, sizeof buf, "neighbouring cells differ in size by %.2f (limit %g)",
                  q.max_size_ratio, l.max_size_ratio);
    out.push_back(buf);
  }
  if (!(q.max_aspect_ratio <= l.max_aspect_ratio)) {
    std::snprintf(buf, sizeof buf, "cell aspect ratio %.1f above %g", q.max_aspect_ratio,
                  l.max_aspect_ratio);
    out.push_back(buf);
  }
  return out;
}

std::vector<double> column_positions(const std::vector<double>& bp,
                                     const std::function<double(double)>& density, int refinement,
                                     int total, double max_spacing_slope) {
  struct Table {
    double a, b;
    int samples;
    std::vector<double> values;
    std::vector<double> cumulative;
    double at(int n) const { return a + ((b - a) * n) / samples; }
  };
  std::vector<Table> tables;
  for (size_t k = 1; k < bp.size(); k++) {
    Table t;
    t.a = bp[k - 1];
    t.b = bp[k];
    // At least 64 samples per base-grid node, estimated from the ends.
    const double baseNodes = (((density(t.a) + density(t.b)) / 2) * (t.b - t.a)) / refinement;
    t.samples = std::max(2048, 64 * int(std::ceil(baseNodes)));
    t.values.resize(t.samples + 1);
    for (int n = 0; n <= t.samples; n++) t.values[n] = density(t.at(n));
    tables.push_back(std::move(t));
  }
  if (max_spacing_slope > 0) {
    // limitSpacingSlope (src/grid/spacing.ts:84-113): the largest spacing
    // below the given one whose slope is at most the limit, by a forward and
    // a backward pass over all samples in order along the line, on the base
    // grid's spacing (the density divided by the refinement).
    std::vector<double> xs, spacing;
    for (const Table& t : tables)
      for (int n = 0; n <= t.samples; n++) {
        xs.push_back(t.at(n));
        spacing.push_back(refinement / t.values[n]);
      }
    std::vector<double> limited = spacing;
    for (size_t k = 1; k < limited.size(); k++)
      limited[k] = std::min(limited[k], limited[k - 1] + max_spacing_slope * (xs[k] - xs[k - 1]));
    for (size_t k = limited.size() - 1; k-- > 0;)
      limited[k] = std::min(limited[k], limited[k + 1] + max_spacing_slope * (xs[k + 1] - xs[k]));
    size_t k = 0;
    for (Table& t : tables)
      for (int n = 0; n <= t.samples; n++, k++)
        if (limited[k] < spacing[k]) t.values[n] = refinement / limited[k];
  }
  for (Table& t : tables) {
    t.cumulative.assign(t.samples + 1, 0.0);
    for (int n = 1; n <= t.samples; n++)
      t.cumulative[n] =
          t.cumulative[n - 1] + 0.5 * (t.values[n - 1] + t.values[n]) * (t.at(n) - t.at(n - 1));
  }
  // Intervals per breakpoint interval.
  std::vector<int> counts(tables.size());
  if (total <= 0) {
    for (size_t k = 0; k < tables.size(); k++) {
      const double integral = tables[k].cumulative[tables[k].samples];
      counts[k] = refinement * std::max(1, int(std::round(integral / refinement)));
    }
  } else {
    double sum = 0;
    for (const Table& t : tables) sum += t.cumulative[t.samples];
    std::vector<double> share(tables.size());
    int assigned = 0;
    for (size_t k = 0; k < tables.size(); k++) {
      share[k] = total * tables[k].cumulative[tables[k].samples] / sum;
      counts[k] = std::max(1, int(std::floor(share[k])));
      assigned += counts[k];
    }
    // Largest remainders take the intervals left; an excess (from the
    // minimum of one) comes off the largest counts.
    while (assigned < total) {
      size_t best = 0;
      double bestRem = -1;
      for (size_t k = 0; k < tables.size(); k++) {
        const double rem = share[k] - counts[k];
        if (rem > bestRem) {
          bestRem = rem;
          best = k;
        }
      }
      counts[best]++;
      assigned++;
    }
    while (assigned > total) {
      size_t best = 0;
      for (size_t k = 0; k < tables.size(); k++)
        if (counts[k] > counts[best]) best = k;
      counts[best]--;
      assigned--;
    }
  }
  std::vector<double> xs{bp[0]};
  for (size_t k = 0; k < tables.size(); k++) {
    const Table& t = tables[k];
    auto at = [&](int n) { return t.at(n); };
    const double integral = t.cumulative[t.samples];
    const int count = counts[k];
    int n = 0;
    for (int m = 1; m < count; m++) {
      const double target = (integral * m) / count;
      while (t.cumulative[n + 1] < target) n++;
      const double f = (target - t.cumulative[n]) / (t.cumulative[n + 1] - t.cumulative[n]);
      xs.push_back(at(n) + f * (at(n + 1) - at(n)));
    }
    xs.push_back(t.b);
  }
  return xs;
}

std::string body_grid(const Body& body, const BodyGridOptions& o, Grid* out, bool* quality_error) {
  *quality_error = false;
  std::string e = validate_body(body);
  if (!e.empty()) return e;
  const int refinement = o.refinement;
  if (!(o.nj >= 4)) return "a body grid needs at least 4 cells across";
  if (!(refinement >= 1 && (refinement & (refinement - 1)) == 0))
    return "the refinement must be 1, 2, 4, 8, ...";
  if (o.ni > 0 && refinement != 1) return "an exact column count needs refinement 1";
  const double tipSlope = nose_tip_slope(body.nose);
  if (!std::isfinite(tipSlope))
    return "blunt noses (profile vertical at the tip) need the C-topology grid";
  const QualityLimits limits;
  const double maxTipHalfAngle = M_PI / 2 - limits.min_wall_angle;
  const double tipHalfAngle = std::atan(tipSlope);
  if (tipHalfAngle > maxTipHalfAngle) {
    char buf[128];
    std::snprintf(buf, sizeof buf, "tip half-angles above %.1f deg are not supported, got %.1f deg",
                  maxTipHalfAngle * 180 / M_PI, tipHalfAngle * 180 / M_PI);
    return buf;
  }
  ConeFlow cone;
  e = taylor_maccoll(o.mach, tipHalfAngle, o.gamma, 1e-13, &cone);
  if (!e.empty()) return e;
  const double shock = cone.shock_angle;
  const double maxOuterAngle = (shock + M_PI / 2) / 2;
  const double R = body.nose.base_radius;
  const double xEnd = body_length(body);
  const double xStart = -R;
  const double maxStrength = 2 * std::log(limits.max_aspect_ratio);

  struct Across {
    double wall, h, b;
  };
  auto across_for = [&](double angle) {
    return [&, angle](double x) {
      const double wall = body_radius(body, x);
      const double h = 0.5 * R + (x - xStart) * std::tan(angle) - wall;
      return Across{wall, h, std::min(std::log1p(h / R), maxStrength)};
    };
  };
  // Fewest base-grid cells between the tip's conical shock line and the
  // outer boundary, as a fraction of the cells across (body-grid.ts:124-135).
  const std::vector<double> bps = body_breakpoints(body);
  std::vector<double> samples(bps.begin() + 1, bps.end());
  for (int k = 1; k < 1024; k++) samples.push_back((xEnd * k) / 1024);
  auto fraction_above_shock = [&](double angle) {
    auto across = across_for(angle);
    double fewest = std::numeric_limits<double>::infinity();
    for (double x : samples) {
      const Across a = across(x);
      const double eta = std::log1p((std::expm1(a.b) * (x * std::tan(shock) - a.wall)) / a.h) / a.b;
      fewest = std::min(fewest, 1 - eta);
    }
    return fewest;
  };
  const int kCellsAboveShock = 3;  // OUTER_CELLS_ABOVE_SHOCK, body-grid.ts:62
  const int baseNj = std::max(
      o.nj, int(std::ceil(kCellsAboveShock / fraction_above_shock(maxOuterAngle) - 1e-9)));
  auto cells_above_shock = [&](double angle) { return baseNj * fraction_above_shock(angle); };
  double outerAngle = std::min(1.2 * shock, maxOuterAngle);
  if (cells_above_shock(outerAngle) < kCellsAboveShock) {
    double low = outerAngle, high = maxOuterAngle;
    for (int k = 0; k < 50; k++) {
      const double mid = (low + high) / 2;
      if (cells_above_shock(mid) < kCellsAboveShock)
        low = mid;
      else
        high = mid;
    }
    outerAngle = high;
  }
  const int nj = baseNj * refinement;
  auto across = across_for(outerAngle);
  auto density = [&](double x) {
    const Across a = across(x);
    const double spacing = (a.h * a.b * std::exp(a.b / 2)) / (std::expm1(a.b) * nj);
    return 1 / spacing;
  };
  std::vector<double> bpx{xStart};
  bpx.insert(bpx.end(), bps.begin(), bps.end());
  const std::vector<double> xs = column_positions(bpx, density, refinement, o.ni);
  const int ni = int(xs.size()) - 1;
  out->ni = ni;
  out->nj = nj;
  out->i_tip = int(std::find(xs.begin(), xs.end(), 0.0) - xs.begin());
  out->outer_angle = outerAngle;
  out->x.assign(size_t(ni + 1) * (nj + 1), 0);
  out->y.assign(size_t(ni + 1) * (nj + 1), 0);
  for (int j = 0; j <= nj; j++)
    for (int i = 0; i <= ni; i++) {
      const Across a = across(xs[i]);
      const size_t k = i + size_t(j) * (ni + 1);
      out->x[k] = xs[i];
      out->y[k] = a.wall + (a.h * std::expm1((a.b * j) / nj)) / std::expm1(a.b);
    }
  const std::vector<std::string> failures =
      quality_failures(grid_quality(ni, nj, out->x.data(), out->y.data()), limits);
  if (!failures.empty()) {
    *quality_error = true;
    std::string msg = "the generated grid fails its quality checks: ";
    for (size_t k = 0; k < failures.size(); k++) msg += (k ? "; " : "") + failures[k];
    return msg;
  }
  return "";
}

namespace {

// Stretching towards the body along a line of height h (lineStrength,
// src/grid/blunt-grid.ts:547-549): b = ln(1 + h / R), capped by the
// aspect-ratio limit.
double line_strength(double h, double radius, const QualityLimits& q) {
  return std::min(std::log1p(h / radius), 2 * std::log(q.max_aspect_ratio));
}

double stretched_fraction(double b, int j, int nj) {
  return std::expm1((b * j) / nj) / std::expm1(b);
}

}  // namespace

std::string blunt_body_grid(const Body& body, const BluntGridOptions& o, Grid* out,
                            bool* quality_error) {
  *quality_error = false;
  std::string e = validate_body(body);
  if (!e.empty()) return e;
  const int refinement = o.refinement;
  if (!(o.nj >= 4)) return "a body grid needs at least 4 cells across";
  if (!(refinement >= 1 && (refinement & (refinement - 1)) == 0))
    return "the refinement must be 1, 2, 4, 8, ...";
  if (o.ni > 0 && refinement != 1) return "an exact column count needs refinement 1";
  if (!(o.mach > 1)) return "blunt-body grids are for supersonic free streams";
  const QualityLimits limits;
  // Placement constants (DEFAULT_TUNING, blunt-grid.ts:130-137).
  const double kStandoffFactor = 2, kArcRadiusFactor = 2, kTipScaleFactor = 2;
  const double kSmoothing = 0.25, kFanRatio = 1.25, kMaxWidthSlope = 0.5;
  const double kMaxNoseRadius = 10, kMaxShoulderAngle = 15 * M_PI / 180;
  const int kWidthSamples = 4096, kUniformWidthSamples = 1024, kSpacingSamples = 8192;
  const int kWindowSamples = 64, kProfileSamples = 20000;

  const Nose& nose = body.nose;
  const bool sharp = std::isfinite(nose_tip_slope(nose));
  const bool ellipsoid = nose.kind == NOSE_ELLIPSOID;
  const double L = nose.length, R = nose.base_radius;

  // The profile by arc length, sampled in u with x = L u^2 (clustered at the tip).
  auto profile_x = [&](double u) { return L * u * u; };
  auto profile_r = [&](double u) { return nose_radius(nose, profile_x(u)); };
  std::vector<double> u_of(kProfileSamples + 1, 0.0), s_of(kProfileSamples + 1, 0.0);
  for (int k = 1; k <= kProfileSamples; k++) {
    const double u0 = double(k - 1) / kProfileSamples, u1 = double(k) / kProfileSamples;
    u_of[k] = u1;
    s_of[k] = s_of[k - 1] + std::hypot(profile_x(u1) - profile_x(u0), profile_r(u1) - profile_r(u0));
  }
  const double s_nose = s_of[kProfileSamples];
  const double s_end = s_nose + body.cylinder_length;
  // Bisection brackets by bucket of s: bracket_lo[b] is the last sample at or
  // below the bucket's start and bracket_hi[b] the first above its end, so a
  // search started from them ends on the same sample as one over the whole
  // table (the arc length grows strictly with u). An s the bucket arithmetic
  // misplaces fails the bracket test and searches the whole table.
  const int kBuckets = 2048;
  const double bucket_scale = kBuckets / s_nose;
  std::vector<int> bracket_lo(kBuckets), bracket_hi(kBuckets);
  {
    int k = 0;
    for (int b = 0; b < kBuckets; b++) {
      const double start = b / bucket_scale, end = (b + 1) / bucket_scale;
      while (k + 1 < kProfileSamples && s_of[k + 1] <= start) k++;
      bracket_lo[b] = k;
      int h = k + 1;
      while (h < kProfileSamples && s_of[h] <= end) h++;
      bracket_hi[b] = h;
    }
  }
  auto u_at = [&](double s) {
    int low = 0, high = kProfileSamples;
    if (s >= 0 && s < s_nose) {
      const int b = std::min(int(s * bucket_scale), kBuckets - 1);
      if (s_of[bracket_lo[b]] <= s && s < s_of[bracket_hi[b]]) {
        low = bracket_lo[b];
        high = bracket_hi[b];
      }
    }
    while (high - low > 1) {
      const int mid = (low + high) >> 1;
      if (s_of[mid] <= s) low = mid;
      else high = mid;
    }
    const double f = (s - s_of[low]) / (s_of[high] - s_of[low]);
    return u_of[low] + std::min(std::max(f, 0.0), 1.0) / kProfileSamples;
  };
  struct SurfacePoint {
    double x, y, nx, ny;
  };
  // The body point at arc length s and its outward normal.
  // The nose's outward normal at profile parameter u (central difference).
  auto nose_normal = [&](double u, double* nx, double* ny) {
    if (u == 0) {
      *nx = -1;
      *ny = 0;
      return;
    }
    const double eps = 1e-7;
    const double ua = std::max(u - eps, 0.0), ub = std::min(u + eps, 1.0);
    const double tx = profile_x(ub) - profile_x(ua), ty = profile_r(ub) - profile_r(ua);
    const double t = std::hypot(tx, ty);
    *nx = -ty / t;
    *ny = tx / t;
  };
  auto surface = [&](double s) -> SurfacePoint {
    if (s >= s_nose) return {L + (s - s_nose), R, 0, 1};
    const double u = u_at(s);
    SurfacePoint p{profile_x(u), profile_r(u), 0, 0};
    nose_normal(u, &p.nx, &p.ny);
    return p;
  };
  const SurfacePoint shoulder = surface(s_nose * (1 - 1e-9));
  const double shoulder_angle = std::atan2(-shoulder.nx, shoulder.ny);
  if (!(shoulder_angle <= kMaxShoulderAngle))
    return "blunt noses meeting the body at more than 15 deg are not supported";

  // Length scales: the tip's radius of curvature, and the tip scale (the x
  // at which the profile crosses r = x).
  const double x_small = 1e-6 * L;
  const double r_small = nose_radius(nose, x_small);
  const double tip_radius = r_small * r_small / (2 * x_small);
  if (!(tip_radius <= kMaxNoseRadius * R)) return "noses that are nearly flat at the tip are not supported";
  double tip_scale = 0;
  if (!sharp) {
    if (nose_radius(nose, L) > L) {
      tip_scale = L;
    } else {
      double low = 0, high = L;
      for (int k = 0; k < 200; k++) {
        const double mid = 0.5 * (low + high);
        if (nose_radius(nose, mid) > mid) low = mid;
        else high = mid;
      }
      tip_scale = 0.5 * (low + high);
    }
  }
  const double scale = ellipsoid ? std::max(tip_radius, R)
                                 : sharp ? R
                                         : std::max(tip_radius, std::min(R, kTipScaleFactor * tip_scale));

  // Outer boundary: an arc ahead of the tip (standoff from Billig's
  // correlation, billigStandoff, blunt-grid.ts:99-101), then a straight line;
  // or the polyline given, linear between its points and continued by its
  // last segment beyond them.
  const double outer_angle = (M_PI / 2 + std::asin(1 / o.mach)) / 2;
  const double arc_radius = kArcRadiusFactor * scale;
  const double standoff = kStandoffFactor * 0.143 * std::exp(3.24 / (o.mach * o.mach)) * scale;
  const double centre = arc_radius - standoff;
  const double y_join = arc_radius * std::cos(outer_angle);
  const double x_join = centre - arc_radius * std::sin(outer_angle);
  const std::vector<double>& cx = o.outer_x;
  const std::vector<double>& cy = o.outer_y;
  const bool custom = !cx.empty() || !cy.empty();
  if (custom) {
    if (cx.size() != cy.size() || cx.size() < 2 || cy[0] != 0)
      return "the outer boundary needs at least two points, the first on the axis";
    for (size_t k = 0; k < cx.size(); k++)
      if (!std::isfinite(cx[k]) || !std::isfinite(cy[k])) return "the outer boundary must be finite";
    for (size_t k = 1; k < cy.size(); k++)
      if (!(cy[k] > cy[k - 1])) return "the outer boundary must be ordered outwards from the axis";
  }
  auto outer_x = [&](double y) {
    if (!custom)
      return y <= y_join ? centre - std::sqrt(arc_radius * arc_radius - y * y)
                         : x_join + (y - y_join) / std::tan(outer_angle);
    // The segment holding y (the last one at or beyond the last point; the
    // first one below the axis, where the lines ahead of the tip look).
    const size_t n = cy.size() - 1;
    size_t low = 0;
    if (y >= cy[n]) {
      low = n - 1;
    } else {
      size_t high = n;
      while (high - low > 1) {
        const size_t mid = (low + high) >> 1;
        if (cy[mid] <= y) low = mid;
        else high = mid;
      }
    }
    return cx[low] + ((y - cy[low]) / (cy[low + 1] - cy[low])) * (cx[low + 1] - cx[low]);
  };
  bool reaches = false;
  // Distance from the body point at s to the outer boundary along (dx, dy).
  auto length_along = [&](double s, double dx, double dy) {
    const SurfacePoint p = surface(s);
    auto outside = [&](double d) { return p.x + d * dx - outer_x(p.y + d * dy) <= 0; };
    if (outside(0)) {
      reaches = true;
      return R;
    }
    double high = R;
    while (!outside(high)) high *= 2;
    double low = 0;
    for (int k = 0; k < 60; k++) {
      const double mid = (low + high) / 2;
      if (outside(mid)) high = mid;
      else low = mid;
    }
    return high;
  };
  auto width_at = [&](double s) {
    const SurfacePoint p = surface(s);
    return std::min(kSmoothing * length_along(s, p.nx, p.ny), s_end - s);
  };
  // The smoothing window's half-width along the body, tabulated and limited
  // to change by at most kMaxWidthSlope per unit length.
  std::vector<double> width_s, widths;
  const bool uniform = ellipsoid;
  const int nw = uniform ? kUniformWidthSamples : kWidthSamples;
  width_s.resize(nw + 1);
  widths.resize(nw + 1);
  for (int k = 0; k <= nw; k++) {
    width_s[k] = uniform ? k * (s_end / nw) : (s_end * double(k) * k) / (double(nw) * nw);
    widths[k] = width_at(width_s[k]);
  }
  if (reaches) return "the body reaches the outer boundary; the nose is not supported";
  for (int k = 1; k <= nw; k++)
    widths[k] = std::min(widths[k], widths[k - 1] + kMaxWidthSlope * (width_s[k] - width_s[k - 1]));
  for (int k = nw - 1; k >= 0; k--)
    widths[k] = std::min(widths[k], widths[k + 1] + kMaxWidthSlope * (width_s[k + 1] - width_s[k]));
  auto half_width = [&](double s) {
    if (uniform) {
      const double step = s_end / nw;
      const double t = std::min(std::max(s / step, 0.0), double(nw));
      const int k = std::min(int(std::floor(t)), nw - 1);
      return widths[k] + (t - k) * (widths[k + 1] - widths[k]);
    }
    const double t = std::min(std::max(std::sqrt(std::max(s, 0.0) / s_end) * nw, 0.0), double(nw));
    const int k = std::min(int(std::floor(t)), nw - 1);
    const double f = (std::min(std::max(s, 0.0), s_end) - width_s[k]) / (width_s[k + 1] - width_s[k]);
    return widths[k] + std::min(std::max(f, 0.0), 1.0) * (widths[k + 1] - widths[k]);
  };
  // Angle of the body normal to the upstream axis, odd about the tip.
  auto normal_angle = [&](double s) -> double {
    const double a = s < 0 ? -s : s;
    double angle = M_PI / 2;
    if (a < s_nose) {
      // The normal (-ty, tx) / |t| makes the angle atan2(tx, ty) with the
      // upstream axis; atan2 needs no normalised tangent.
      const double u = u_at(a);
      if (u == 0) {
        angle = 0;
      } else {
        const double eps = 1e-7;
        const double ua = std::max(u - eps, 0.0), ub = std::min(u + eps, 1.0);
        angle = std::atan2(profile_x(ub) - profile_x(ua), profile_r(ub) - profile_r(ua));
      }
    }
    return s < 0 ? -angle : angle;
  };
  // A sharp tip's jump in the normal, fanned out geometrically.
  const double tip_jump = sharp ? normal_angle(s_nose * 1e-9) : 0;
  double fan_scale = std::numeric_limits<double>::infinity();
  if (sharp) {
    const double h = length_along(0, -1, 0);
    const double c = 1 / std::log(kFanRatio) / o.nj;
    fan_scale = (h * (-tip_jump + std::sqrt(tip_jump * tip_jump + 4 * c * c))) / 2;
  }
  auto fan = [&](double s) { return tip_jump * -std::expm1(-s / fan_scale); };
  std::function<double(double)> line_angle = [&](double s) -> double {
    if (s == 0) return 0;
    if (s < 0) return -line_angle(-s);
    if (s >= s_end) return M_PI / 2;
    const double w = half_width(s);
    double sum = 0;
    for (int k = 0; k < kWindowSamples; k++) {
      const double t = s - w + (2 * w * (k + 0.5)) / kWindowSamples;
      const double sign = t > 0 ? 1.0 : t < 0 ? -1.0 : 0.0;
      sum += normal_angle(t) - sign * tip_jump;
    }
    return sum / kWindowSamples + fan(s);
  };
  auto turn_rate = [&](double s) {
    const double ew = std::max(std::min(half_width(s) / 4, std::max(fan_scale / 4, s / 8)),
                               s_end / kProfileSamples);
    return (line_angle(s + ew) - line_angle(s - ew)) / (2 * ew);
  };
  struct Line {
    double dx, dy, h;
  };
  auto line = [&](double s) -> Line {
    const double angle = line_angle(s);
    const double dx = -std::cos(angle), dy = std::sin(angle);
    return {dx, dy, length_along(s, dx, dy)};
  };
  const int nj = o.nj * refinement;
  // Spacing along the body: wall cells as long as the geometric mean of
  // their height and the outer cells' height, allowing for the lines'
  // spreading.
  auto spacing = [&](double s) {
    const Line l = line(s);
    const double b = line_strength(l.h, R, limits);
    const double wall_height = (l.h * b) / (std::expm1(b) * nj);
    return (wall_height * std::exp(b / 2)) / std::sqrt(1 + turn_rate(s) * l.h);
  };
  std::vector<double> bps = body.cylinder_length > 0 ? std::vector<double>{0, s_nose, s_end}
                                                     : std::vector<double>{0, s_nose};
  std::vector<double> ss;
  if (ellipsoid) {
    ss = column_positions(bps, [&](double s) { return 1 / spacing(s); }, refinement, o.ni, 0.15);
  } else {
    std::vector<double> dens_s(kSpacingSamples + 1), dens(kSpacingSamples + 1);
    for (int k = 0; k <= kSpacingSamples; k++) {
      dens_s[k] = (s_end * double(k) * k) / (double(kSpacingSamples) * kSpacingSamples);
      dens[k] = 1 / spacing(dens_s[k]);
    }
    auto tabulated = [&](double s) {
      const double t = std::min(
          std::max(std::sqrt(std::max(s, 0.0) / s_end) * kSpacingSamples, 0.0), double(kSpacingSamples));
      const int k = std::min(int(std::floor(t)), kSpacingSamples - 1);
      const double f = (std::min(std::max(s, 0.0), s_end) - dens_s[k]) / (dens_s[k + 1] - dens_s[k]);
      return dens[k] + std::min(std::max(f, 0.0), 1.0) * (dens[k + 1] - dens[k]);
    };
    ss = column_positions(bps, tabulated, refinement, o.ni);
  }
  if (reaches) return "the body reaches the outer boundary; the nose is not supported";
  const int ni = int(ss.size()) - 1;
  out->ni = ni;
  out->nj = nj;
  out->i_tip = 0;
  out->outer_angle = outer_angle;
  out->two_scale = sharp || scale < R;
  out->x.assign(size_t(ni + 1) * (nj + 1), 0);
  out->y.assign(size_t(ni + 1) * (nj + 1), 0);
  for (int i = 0; i <= ni; i++) {
    const SurfacePoint p = surface(ss[i]);
    const Line l = line(ss[i]);
    const double b = line_strength(l.h, R, limits);
    for (int j = 0; j <= nj; j++) {
      const double d = l.h * stretched_fraction(b, j, nj);
      const size_t k = i + size_t(j) * (ni + 1);
      out->x[k] = p.x + d * l.dx;
      out->y[k] = p.y + d * l.dy;
    }
  }
  // The first line lies on the axis ahead of the tip.
  for (int j = 0; j <= nj; j++) out->y[size_t(j) * (ni + 1)] = 0;
  if (!o.gated) return "";
  const std::vector<std::string> failures =
      quality_failures(grid_quality(ni, nj, out->x.data(), out->y.data()), limits);
  if (!failures.empty()) {
    *quality_error = true;
    std::string msg = "the generated grid fails its quality checks: ";
    for (size_t k = 0; k < failures.size(); k++) msg += (k ? "; " : "") + failures[k];
    return msg;
  }
  return "";
}

std::vector<double> sharp_fit_columns(const Body& body, double beta, double x0, int nj, int refinement,
                                      double aspect, double density) {
  const double L = body.nose.length, R = body.nose.base_radius;
  const double x_end = body_length(body);
  auto guess = [&](double x) { return std::max(x * std::tan(beta) - body_radius(body, x), 1e-12 * L); };
  auto spacing = [&](double x) {
    const double h = guess(x);
    const double b = std::min(std::log1p(h / R), 2 * std::log(10.0));
    return (aspect * h * b * std::exp(b / 2)) / (std::expm1(b) * nj);
  };
  const std::vector<double> bp = body.cylinder_length > 0 ? std::vector<double>{x0, L, x_end}
                                                          : std::vector<double>{x0, L};
  return column_positions(bp, [&](double x) { return density / spacing(x); }, refinement, 0);
}

namespace {

// bluntGrid (src/grid/transonic-grid.ts:319-460): the C grid of a blunt nose
// on the spacings of the sharp noses' grid: columns by arc length along the
// body (s.tip at the stagnation point, s.shoulder at the shoulder, at most
// s.nose apart, growing by s.growth along the cylinder), rows by the same
// geometric growth out to a far boundary that is a quarter circle of the far
// radius about the stagnation point continued at the far radius. Each line
// leaves its body point P along the body normal averaged over a window and
// bends to its point Q on the far boundary (Q evenly spaced along it):
// node = P + d (f (1 - f) n + f^2 u), d = |Q - P|, u = (Q - P) / d.
std::string transonic_c_grid(const Body& body, const TransonicSpacing& s, int refinement, int base_nj,
                             double far_radius, double x_end, Grid* out, int* i_shoulder_out) {
  constexpr int kProfileSamples = 20000;
  constexpr double kSmoothing = 0.25, kMaxWidthSlope = 0.5;
  constexpr int kWindowSamples = 64;
  const Nose& nose = body.nose;
  const double L = nose.length, R = nose.base_radius;
  auto profile_x = [&](double u) { return L * u * u; };
  auto profile_r = [&](double u) { return nose_radius(nose, profile_x(u)); };
  std::vector<double> u_of(kProfileSamples + 1, 0.0), s_of(kProfileSamples + 1, 0.0);
  for (int k = 1; k <= kProfileSamples; k++) {
    const double u0 = double(k - 1) / kProfileSamples, u1 = double(k) / kProfileSamples;
    u_of[k] = u1;
    s_of[k] = s_of[k - 1] + std::hypot(profile_x(u1) - profile_x(u0), profile_r(u1) - profile_r(u0));
  }
  const double s_nose = s_of[kProfileSamples];
  const double s_end = s_nose + (x_end - L);
  auto u_at = [&](double arc) {
    int low = 0, high = kProfileSamples;
    while (high - low > 1) {
      const int mid = (low + high) >> 1;
      if (s_of[mid] <= arc) low = mid;
      else high = mid;
    }
    const double f = (arc - s_of[low]) / (s_of[high] - s_of[low]);
    return u_of[low] + std::min(std::max(f, 0.0), 1.0) / kProfileSamples;
  };
  struct P {
    double x, y, nx, ny;
  };
  auto surface = [&](double arc) -> P {
    if (arc >= s_nose) return {L + (arc - s_nose), R, 0, 1};
    const double u = u_at(arc);
    if (u == 0) return {0, 0, -1, 0};
    const double e = 1e-7;
    const double ua = std::max(u - e, 0.0), ub = std::min(u + e, 1.0);
    const double tx = profile_x(ub) - profile_x(ua), ty = profile_r(ub) - profile_r(ua);
    const double t = std::hypot(tx, ty);
    return {profile_x(u), profile_r(u), -ty / t, tx / t};
  };
  if (!(std::abs(surface(s_nose * (1 - 1e-9)).nx) < 1e-3))
    return "blunt noses that do not meet the body tangentially are not supported by the transonic grid yet";
  auto spacing = [&](double arc) {
    return arc >= s_nose ? s.shoulder * R + s.growth * (arc - s_nose)
                         : std::min(std::min(s.tip * R + s.nose_growth * arc,
                                             s.shoulder * R + s.nose_growth * (s_nose - arc)),
                                    s.nose * R);
  };
  const std::vector<double> arcs = column_positions(
      {0.0, s_nose, s_end}, [&](double arc) { return refinement / spacing(arc); }, refinement, 0);
  const int ni = int(arcs.size()) - 1;
  int i_shoulder = -1;
  for (int i = 0; i <= ni && i_shoulder < 0; i++)
    if (arcs[i] == s_nose) i_shoulder = i;
  std::vector<P> points(ni + 1);
  for (int i = 0; i <= ni; i++) points[i] = surface(arcs[i]);
  const double quarter = (M_PI / 2) * far_radius;
  const double far_length = quarter + x_end;
  auto far = [&](double t, double* qx, double* qy) {
    if (t <= quarter) {
      *qx = -far_radius * std::cos(t / far_radius);
      *qy = far_radius * std::sin(t / far_radius);
    } else {
      *qx = t - quarter;
      *qy = far_radius;
    }
  };
  // Angle of the body normal to the upstream axis, odd about the stagnation
  // point, pi / 2 from the shoulder on.
  std::function<double(double)> normal_angle = [&](double arc) -> double {
    if (arc < 0) return -normal_angle(-arc);
    if (arc >= s_nose) return M_PI / 2;
    const P p = surface(arc);
    return std::atan2(p.ny, -p.nx);
  };
  // The normal averaged over a window of half-width the harmonic
  // combination of kSmoothing h and kMaxWidthSlope times the distance to
  // the end of the body.
  auto direction = [&](double arc, double h, double* dx, double* dy) {
    const double a = kSmoothing * h;
    const double c = kMaxWidthSlope * (s_end - arc);
    const double w = a + c > 0 ? (a * c) / (a + c) : 0;
    double angle;
    if (arc == 0 || w == 0) {
      angle = normal_angle(arc);
    } else {
      double sum = 0;
      for (int k = 0; k < kWindowSamples; k++)
        sum += normal_angle(arc - w + (2 * w * (k + 0.5)) / kWindowSamples);
      angle = sum / kWindowSamples;
    }
    *dx = -std::cos(angle);
    *dy = std::sin(angle);
  };
  const int nj = base_nj * refinement;
  const double b = s.growth * base_nj;
  out->ni = ni;
  out->nj = nj;
  out->i_tip = 0;
  out->outer_angle = 0;
  out->two_scale = false;
  out->x.assign(size_t(ni + 1) * (nj + 1), 0);
  out->y.assign(size_t(ni + 1) * (nj + 1), 0);
  for (int i = 0; i <= ni; i++) {
    const P& p = points[i];
    double qx, qy;
    if (i == ni) {
      qx = x_end;
      qy = far_radius;
    } else {
      far((far_length * i) / ni, &qx, &qy);
    }
    const double d = std::hypot(qx - p.x, qy - p.y);
    const double ux = (qx - p.x) / d, uy = (qy - p.y) / d;
    for (int j = 0; j <= nj; j++) {
      const double f = std::expm1((b * j) / nj) / std::expm1(b);
      const double along = f * (1 - f);
      double nx, ny;
      direction(arcs[i], d * f, &nx, &ny);
      const size_t k = i + size_t(j) * (ni + 1);
      out->x[k] = p.x + d * (along * nx + f * f * ux);
      out->y[k] = p.y + d * (along * ny + f * f * uy);
    }
  }
  *i_shoulder_out = i_shoulder;
  return "";
}

}  // namespace

std::string transonic_grid(const Body& body, const TransonicGridOptions& o, Grid* out,
                           TransonicGridInfo* info) {
  std::string e = validate_body(body);
  if (!e.empty()) return e;
  const int refinement = o.refinement;
  if (!(refinement >= 1 && (refinement & (refinement - 1)) == 0))
    return "the refinement must be 1, 2, 4, 8, ...";
  const double R = body.nose.base_radius, L = body.nose.length;
  if (!(o.cylinder > 0)) return "the transonic domain needs a cylinder";
  if (!(o.far_field * R > 4 * std::max(R, L))) return "the far boundaries must lie beyond four nose lengths";
  const TransonicSpacing& s = o.spacing;
  if (!(s.wall > 0 && s.growth > 0 && s.tip > 0 && s.shoulder > 0 && s.nose > 0 && s.nose_growth > 0))
    return "the transonic grid's spacings must be positive";
  const bool blunt = !std::isfinite(nose_tip_slope(body.nose));
  const double wall = s.wall * R, growth = s.growth;
  // Cells across on the base grid: geometric growth from the wall spacing
  // reaches the far radius in this many cells.
  const int base_nj = int(std::ceil(std::log1p(growth * o.far_field * R / wall) / growth - 1e-9));
  const double far_radius = (wall / growth) * std::expm1(growth * base_nj);
  const double x_upstream = -far_radius;
  const double x_end = L + 2 * R * o.cylinder;
  const int nj = base_nj * refinement;
  if (blunt) {
    if (o.nested) return "nested domains are not available on the C grids of blunt noses yet";
    e = transonic_c_grid(body, s, refinement, base_nj, far_radius, x_end, out, &info->i_shoulder);
    if (!e.empty()) return e;
    info->i_tip = 0;
    info->base_nj = base_nj;
    info->far_radius = far_radius;
    info->x_upstream = x_upstream;
    info->x_end = x_end;
    info->c_topology = true;
    return "";
  }
  // Column spacing along x: growing geometrically from the tip and from the
  // shoulder, at most s.nose along the nose.
  const double tip = s.tip * R, shoulder = s.shoulder * R;
  auto spacing = [&](double x) {
    if (x <= 0) return tip + growth * -x;
    if (x >= L) return shoulder + growth * (x - L);
    return std::min(std::min(tip + s.nose_growth * x, shoulder + s.nose_growth * (L - x)), s.nose * R);
  };
  const std::vector<double> xs = column_positions(
      {x_upstream, 0.0, L, x_end}, [&](double x) { return refinement / spacing(x); }, refinement, 0);
  const int ni = int(xs.size()) - 1;
  int i_tip = -1, i_shoulder = -1;
  for (int i = 0; i <= ni; i++) {
    if (i_tip < 0 && xs[i] == 0) i_tip = i;
    if (i_shoulder < 0 && xs[i] == L) i_shoulder = i;
  }
  // Across each line from the wall to the far radius at f = expm1(b j / nj)
  // / expm1(b) of the way, b = growth base_nj; the lines lean, by f^2 of the
  // way, to points evenly spaced along the far boundary.
  const double b = growth * base_nj;
  auto node = [&](int i, int j, double* x_out, double* y_out) {
    const double x = xs[i];
    const double r = body_radius(body, x);
    const double f = std::expm1((b * j) / nj) / std::expm1(b);
    const double x_far = x_upstream + ((x_end - x_upstream) * i) / ni;
    *x_out = x + (x_far - x) * f * f;
    *y_out = r + (far_radius - r) * f;
  };
  out->outer_angle = 0;
  out->two_scale = false;
  info->c_topology = false;
  if (!o.nested) {
    out->ni = ni;
    out->nj = nj;
    out->i_tip = i_tip;
    out->x.assign(size_t(ni + 1) * (nj + 1), 0);
    out->y.assign(size_t(ni + 1) * (nj + 1), 0);
    for (int j = 0; j <= nj; j++)
      for (int i = 0; i <= ni; i++) {
        const size_t k = i + size_t(j) * (ni + 1);
        node(i, j, &out->x[k], &out->y[k]);
      }
    info->i_tip = i_tip;
    info->i_shoulder = i_shoulder;
    info->base_nj = base_nj;
    info->far_radius = far_radius;
    info->x_upstream = x_upstream;
    info->x_end = x_end;
    return "";
  }

  // nestedGrid (:191-303): the grid cut back or continued to the nested far
  // boundaries and cylinder in whole base cells, every node the two domains
  // share the same. Beyond the grid's own columns the spacing grows on
  // geometrically as inside, as vertical lines; beyond its far radius the
  // rows grow on as on the axis, as horizontal lines.
  const double g = growth;
  const double far = (o.nested_far_field == 0 || o.nested_far_field == o.far_field) ? far_radius
                                                                                       : o.nested_far_field * R;
  const double cylinder_end = L + 2 * R * (o.nested_cylinder != 0 ? o.nested_cylinder : o.cylinder);
  if (!(far > 4 * std::max(R, L))) return "the far boundaries must lie beyond four nose lengths";
  if (!(cylinder_end > L)) return "the transonic domain needs a cylinder";
  auto row = [&](double j) { return (wall / g) * std::expm1((g * j) / refinement); };
  const double upstream_step = std::log1p((g * -x_upstream) / tip) / g / (double(i_tip) / refinement);
  const double downstream_step =
      std::log1p((g * (x_end - L)) / shoulder) / g / (double(ni - i_shoulder) / refinement);
  auto x_before = [&](double k) { return -((tip + g * -x_upstream) * std::exp(g * k * upstream_step) - tip) / g; };
  auto x_beyond = [&](double k) {
    return L + ((shoulder + g * (x_end - L)) * std::exp(g * k * downstream_step) - shoulder) / g;
  };
  auto x_at = [&](int i) {
    return i < 0 ? x_before(double(-i) / refinement) : i > ni ? x_beyond(double(i - ni) / refinement) : xs[i];
  };
  int j_hi = nj, i_lo = 0;
  if (far < far_radius) {
    int jb = 1;
    while (row(jb * refinement) < far) jb++;
    j_hi = jb * refinement;
    int m = 0;
    while (xs[(m + 1) * refinement] <= -far) m++;
    i_lo = m * refinement;
  } else if (far > far_radius) {
    j_hi = refinement * int(std::ceil(std::log1p((g * far) / wall) / g - 1e-9));
    int k = 1;
    while (x_before(k) > -far) k++;
    i_lo = -k * refinement;
  }
  int i_hi = ni;
  if (cylinder_end < x_end) {
    int m = i_shoulder / refinement + 1;
    while (xs[m * refinement] < cylinder_end) m++;
    i_hi = m * refinement;
  } else if (cylinder_end > x_end) {
    int k = 1;
    while (x_beyond(k) < cylinder_end) k++;
    i_hi = ni + k * refinement;
  }
  auto x_far = [&](int i) { return x_upstream + ((x_end - x_upstream) * i) / ni; };
  const int nni = i_hi - i_lo;
  out->ni = nni;
  out->nj = j_hi;
  out->i_tip = i_tip - i_lo;
  out->x.assign(size_t(nni + 1) * (j_hi + 1), 0);
  out->y.assign(size_t(nni + 1) * (j_hi + 1), 0);
  for (int j = 0; j <= j_hi; j++)
    for (int ii = 0; ii <= nni; ii++) {
      const int i = ii + i_lo;
      const size_t k = ii + size_t(j) * (nni + 1);
      double x, y;
      if (i >= 0 && i <= ni && j <= nj) {
        node(i, j, &x, &y);
      } else if (j > nj) {
        x = (i < 0 || i > ni) ? x_at(i) : x_far(i);
        y = row(j);
      } else if (i < 0) {
        x = x_at(i);
        y = row(j);
      } else {
        // Beyond the end along x: vertical lines with the end column's rows.
        const double f = std::expm1((g * j) / refinement) / std::expm1((g * nj) / refinement);
        x = x_at(i);
        y = R + (far_radius - R) * f;
      }
      out->x[k] = x;
      out->y[k] = y;
    }
  info->i_tip = i_tip - i_lo;
  info->i_shoulder = i_shoulder - i_lo;
  info->base_nj = j_hi / refinement;
  info->far_radius = row(j_hi);
  info->x_upstream = x_at(i_lo);
  info->x_end = x_at(i_hi);
  return "";
}

std::string ramp_grid(int ni, int nj, double x_min, double x_corner, double x_max, double height,
                      double angle, Grid* out) {
  if (!(x_min < x_corner && x_corner < x_max)) return "the corner must lie inside";
  auto wall = [&](double x) { return x <= x_corner ? 0.0 : (x - x_corner) * std::tan(angle); };
  if (wall(x_max) >= height) return "the ramp reaches the upper boundary";
  const int iCorner = int(std::round((ni * (x_corner - x_min)) / (x_max - x_min)));
  if (iCorner < 1 || iCorner >= ni) return "too few cells to resolve the corner";
  auto x_at = [&](int i) {
    return i <= iCorner ? x_min + ((x_corner - x_min) * i) / iCorner
                        : x_corner + ((x_max - x_corner) * (i - iCorner)) / (ni - iCorner);
  };
  out->ni = ni;
  out->nj = nj;
  out->x.assign(size_t(ni + 1) * (nj + 1), 0);
  out->y.assign(size_t(ni + 1) * (nj + 1), 0);
  for (int j = 0; j <= nj; j++)
    for (int i = 0; i <= ni; i++) {
      const double x = x_at(i), y0 = wall(x);
      const size_t k = i + size_t(j) * (ni + 1);
      out->x[k] = x;
      out->y[k] = y0 + ((height - y0) * j) / nj;
    }
  return "";
}

}  // namespace bs
