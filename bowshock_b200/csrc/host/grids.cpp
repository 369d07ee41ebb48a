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
                                     int total) {
  struct Table {
    double a, b;
    int samples;
    std::vector<double> cumulative;
  };
  std::vector<Table> tables;
  for (size_t k = 1; k < bp.size(); k++) {
    Table t;
    t.a = bp[k - 1];
    t.b = bp[k];
    // At least 64 samples per base-grid node, estimated from the ends.
    const double baseNodes = (((density(t.a) + density(t.b)) / 2) * (t.b - t.a)) / refinement;
    t.samples = std::max(2048, 64 * int(std::ceil(baseNodes)));
    std::vector<double> values(t.samples + 1);
    auto at = [&](int n) { return t.a + ((t.b - t.a) * n) / t.samples; };
    for (int n = 0; n <= t.samples; n++) values[n] = density(at(n));
    t.cumulative.assign(t.samples + 1, 0.0);
    for (int n = 1; n <= t.samples; n++)
      t.cumulative[n] =
          t.cumulative[n - 1] + 0.5 * (values[n - 1] + values[n]) * (at(n) - at(n - 1));
    tables.push_back(std::move(t));
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
    auto at = [&](int n) { return t.a + ((t.b - t.a) * n) / t.samples; };
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
