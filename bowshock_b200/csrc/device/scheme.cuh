// Device-side scheme: gas law, limiters, MUSCL reconstruction, HLLC/Rusanov
// face fluxes and the far-field state, templated on the arithmetic type.
// These are the sm_100a counterparts of src/scheme/{gas,limiters,
// reconstruction,flux}.ts and farFieldState (src/engine-cpu/euler2d.ts:139-165);
// the formulas and their order of operations follow the reference so that the
// FP64 instantiation reproduces the FP64 CPU engine to rounding.
#pragma once

#include <cuda_runtime.h>

#include "bowshock.h"

namespace bsd {

template <class R>
struct Prim {
  R rho, u, v, p;
};

template <class R>
struct Cons {
  R rho, mu, mv, e;
};

template <class R>
__device__ __forceinline__ R dsqrt(R x);
template <>
__device__ __forceinline__ float dsqrt<float>(float x) { return __fsqrt_rn(x); }
template <>
__device__ __forceinline__ double dsqrt<double>(double x) { return __dsqrt_rn(x); }

template <class R>
__device__ __forceinline__ R dmin(R a, R b) { return a < b ? a : b; }
template <class R>
__device__ __forceinline__ R dmax(R a, R b) { return a > b ? a : b; }

// pressureFromConserved2D (src/scheme/gas.ts:51-59).
template <class R>
__device__ __forceinline__ R pressure_of(R rho, R mu, R mv, R e, R gamma) {
  return (gamma - R(1)) * (e - (R(0.5) * (mu * mu + mv * mv)) / rho);
}

template <class R>
__device__ __forceinline__ Prim<R> to_prim(const Cons<R>& q, R gamma) {
  return {q.rho, q.mu / q.rho, q.mv / q.rho, pressure_of(q.rho, q.mu, q.mv, q.e, gamma)};
}

template <class R>
__device__ __forceinline__ Cons<R> to_cons(const Prim<R>& w, R gamma) {
  return {w.rho, w.rho * w.u, w.rho * w.v,
          w.p / (gamma - R(1)) + R(0.5) * w.rho * (w.u * w.u + w.v * w.v)};
}

template <class R>
__device__ __forceinline__ bool is_physical(const Cons<R>& q, R gamma) {
  const Prim<R> w = to_prim(q, gamma);
  // Comparisons with NaN are false; the bounds reject infinities.
  const R big = R(3.0e38);
  return w.rho > R(0) && w.rho < big && w.p > R(0) && w.p < big && fabs(w.u) < big &&
         fabs(w.v) < big;
}

// applyImplicitUpdate (src/engine-cpu/euler2d.ts:816-847) for one cell:
// Q + alpha dQ with alpha halved until density and pressure stay within a
// factor of two of Q's.
template <class R>
__device__ __forceinline__ Cons<R> implicit_update(const Cons<R>& q0, float4 d4, R gamma) {
  const R p0 = pressure_of(q0.rho, q0.mu, q0.mv, q0.e, gamma);
  const R d0 = R(d4.x), d1 = R(d4.y), d2 = R(d4.z), d3 = R(d4.w);
  R alpha = R(1);
  for (int tries = 0; tries < 30; tries++) {
    const R rho1 = q0.rho + alpha * d0;
    const R p1 = pressure_of(rho1, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3, gamma);
    if (rho1 > R(0.5) * q0.rho && rho1 < R(2) * q0.rho && p1 > R(0.5) * p0 && p1 < R(2) * p0) break;
    alpha *= R(0.5);
  }
  return {q0.rho + alpha * d0, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3};
}

// LIMITERS (src/scheme/limiters.ts:24-94).
template <class R>
__device__ __forceinline__ R limit(int limiter, R a, R b) {
  switch (limiter) {
    case BS_LIMITER_FIRST_ORDER:
      return R(0);
    case BS_LIMITER_MINMOD:
      if (a * b <= R(0)) return R(0);
      return fabs(a) < fabs(b) ? a : b;
    case BS_LIMITER_VAN_LEER:
      if (a * b <= R(0)) return R(0);
      return (R(2) * a * b) / (a + b);
    case BS_LIMITER_VAN_ALBADA: {
      const R eps = R(1e-6);
      return (a * (b * b + eps) + b * (a * a + eps)) / (a * a + b * b + R(2) * eps);
    }
    case BS_LIMITER_MONOTONIZED_CENTRAL: {
      if (a * b <= R(0)) return R(0);
      const R sign = a > R(0) ? R(1) : R(-1);
      return sign * dmin(dmin(R(2) * fabs(a), R(2) * fabs(b)), R(0.5) * fabs(a + b));
    }
    default:
      return R(0.5) * (a + b);
  }
}

// The clipped van Albada factor of two difference vectors
// (sharedFactor / sharedScaledFactor, src/scheme/reconstruction.ts:70-136).
template <class R>
__device__ __forceinline__ R van_albada_factor(R aR, R aU, R aV, R aP, R bR, R bU, R bV, R bP) {
  const R ab = aR * bR + aU * bU + aV * bV + aP * bP;
  const R aa = aR * aR + aU * aU + aV * aV + aP * aP;
  const R bb = bR * bR + bU * bU + bV * bV + bP * bP;
  const R eps = R(1e-6);
  return dmax(R(0), (R(2) * (ab + eps)) / (aa + bb + R(2) * eps));
}

// The centre cell's state at its +1 (side = 1) or -1 face
// (reconstructPerVariable / reconstructShared / reconstructSharedScaled,
// src/scheme/reconstruction.ts:50-151).
template <class R>
__device__ __forceinline__ Prim<R> reconstruct(int recon, int limiter, const Prim<R>& pv,
                                               const Prim<R>& c, const Prim<R>& n, R side,
                                               R gamma) {
  if (recon == BS_RECON_PER_VARIABLE) {
    const R h = R(0.5) * side;
    return {c.rho + h * limit(limiter, c.rho - pv.rho, n.rho - c.rho),
            c.u + h * limit(limiter, c.u - pv.u, n.u - c.u),
            c.v + h * limit(limiter, c.v - pv.v, n.v - c.v),
            c.p + h * limit(limiter, c.p - pv.p, n.p - c.p)};
  }
  R factor;
  if (recon == BS_RECON_SHARED) {
    factor = van_albada_factor(c.rho - pv.rho, c.u - pv.u, c.v - pv.v, c.p - pv.p,
                               n.rho - c.rho, n.u - c.u, n.v - c.v, n.p - c.p);
  } else {
    const R rho = dmin(dmin(pv.rho, c.rho), n.rho);
    const R sRho = R(1) / rho;
    const R rhoA2 = gamma * dmin(dmin(pv.p, c.p), n.p);
    const R sU = dsqrt(rho / rhoA2);
    const R sP = R(1) / rhoA2;
    factor = van_albada_factor((c.rho - pv.rho) * sRho, (c.u - pv.u) * sU, (c.v - pv.v) * sU,
                               (c.p - pv.p) * sP, (n.rho - c.rho) * sRho, (n.u - c.u) * sU,
                               (n.v - c.v) * sU, (n.p - c.p) * sP);
  }
  const R k = R(0.25) * side * factor;
  return {c.rho + k * (n.rho - pv.rho), c.u + k * (n.u - pv.u), c.v + k * (n.v - pv.v),
          c.p + k * (n.p - pv.p)};
}

// Flux through a face in its own frame [mass, normal mom., tangential mom.,
// energy] per unit area (src/scheme/flux.ts:34-205).
template <class R>
struct FaceState {
  R rho, un, ut, p;
};

template <class R>
__device__ __forceinline__ R energy_of(const FaceState<R>& w, R gamma) {
  return w.p / (gamma - R(1)) + R(0.5) * w.rho * (w.un * w.un + w.ut * w.ut);
}

template <class R>
__device__ __forceinline__ void physical_flux(const FaceState<R>& w, R gamma, R out[4]) {
  const R mass = w.rho * w.un;
  out[0] = mass;
  out[1] = mass * w.un + w.p;
  out[2] = mass * w.ut;
  out[3] = w.un * (energy_of(w, gamma) + w.p);
}

template <class R>
__device__ __forceinline__ void hllc_flux(const FaceState<R>& l, const FaceState<R>& r, R gamma,
                                          R out[4]) {
  const R energyL = energy_of(l, gamma);
  const R energyR = energy_of(r, gamma);
  // Einfeldt's wave speeds (einfeldtSpeeds, flux.ts:87-107).
  const R aL = dsqrt((gamma * l.p) / l.rho);
  const R aR = dsqrt((gamma * r.p) / r.rho);
  const R wL = dsqrt(l.rho);
  const R wR = dsqrt(r.rho);
  const R unRoe = (wL * l.un + wR * r.un) / (wL + wR);
  const R utRoe = (wL * l.ut + wR * r.ut) / (wL + wR);
  const R hL = (energyL + l.p) / l.rho;
  const R hR = (energyR + r.p) / r.rho;
  const R hRoe = (wL * hL + wR * hR) / (wL + wR);
  const R aRoe =
      dsqrt(dmax((gamma - R(1)) * (hRoe - R(0.5) * (unRoe * unRoe + utRoe * utRoe)), R(0)));
  const R sL = dmin(l.un - aL, unRoe - aRoe);
  const R sR = dmax(r.un + aR, unRoe + aRoe);
  if (sL >= R(0)) {
    physical_flux(l, gamma, out);
    return;
  }
  if (sR <= R(0)) {
    physical_flux(r, gamma, out);
    return;
  }
  const R mL = l.rho * (sL - l.un);
  const R mR = r.rho * (sR - r.un);
  const R sStar = (r.p - l.p + l.un * mL - r.un * mR) / (mL - mR);
  const bool left = sStar >= R(0);
  const FaceState<R> s = left ? l : r;
  const R sK = left ? sL : sR;
  const R energyK = left ? energyL : energyR;
  const R starRho = (s.rho * (sK - s.un)) / (sK - sStar);
  const R starEnergy =
      starRho * (energyK / s.rho + (sStar - s.un) * (sStar + s.p / (s.rho * (sK - s.un))));
  const R mass = s.rho * s.un;
  out[0] = mass + sK * (starRho - s.rho);
  out[1] = mass * s.un + s.p + sK * (starRho * sStar - mass);
  out[2] = mass * s.ut + sK * (starRho - s.rho) * s.ut;
  out[3] = s.un * (energyK + s.p) + sK * (starEnergy - energyK);
}

template <class R>
__device__ __forceinline__ void rusanov_flux(const FaceState<R>& l, const FaceState<R>& r,
                                             R gamma, R out[4]) {
  const R sMax = dmax(fabs(l.un) + dsqrt((gamma * l.p) / l.rho),
                      fabs(r.un) + dsqrt((gamma * r.p) / r.rho));
  const R eL = energy_of(l, gamma), eR = energy_of(r, gamma);
  const R mL = l.rho * l.un, mR = r.rho * r.un;
  out[0] = R(0.5) * (mL + mR) - R(0.5) * sMax * (r.rho - l.rho);
  out[1] = R(0.5) * (mL * l.un + l.p + mR * r.un + r.p) - R(0.5) * sMax * (mR - mL);
  out[2] = R(0.5) * (mL * l.ut + mR * r.ut) - R(0.5) * sMax * (r.rho * r.ut - l.rho * l.ut);
  out[3] = R(0.5) * (l.un * (eL + l.p) + r.un * (eR + r.p)) - R(0.5) * sMax * (eR - eL);
}

// faceFlux2D (src/scheme/flux.ts:342-366): flux per unit area along the unit
// normal (nx, ny), as [mass, x momentum, y momentum, energy].
template <class R>
__device__ __forceinline__ void face_flux(int flux, const Prim<R>& left, const Prim<R>& right,
                                          R nx, R ny, R gamma, R out[4]) {
  const FaceState<R> l{left.rho, left.u * nx + left.v * ny, -left.u * ny + left.v * nx, left.p};
  const FaceState<R> r{right.rho, right.u * nx + right.v * ny, -right.u * ny + right.v * nx,
                       right.p};
  if (flux == BS_FLUX_RUSANOV)
    rusanov_flux(l, r, gamma, out);
  else
    hllc_flux(l, r, gamma, out);
  const R normal = out[1];
  const R tangential = out[2];
  out[1] = normal * nx - tangential * ny;
  out[2] = normal * ny + tangential * nx;
}

// The face's reconstructed left and right states from its 4-cell stencil,
// with the first-order fallback (faceStates, src/engine-cpu/euler2d.ts:1303-1320),
// then the wall mirror (wallMirrored, :1332-1346): wall = -1 on a minimum
// wall side (cell inside on the right), +1 on a maximum one, 0 elsewhere.
template <class R>
__device__ __forceinline__ void face_states(int recon, int limiter, const Prim<R>& wLL,
                                            const Prim<R>& wL, const Prim<R>& wR,
                                            const Prim<R>& wRR, R gamma, int wall, R nx, R ny,
                                            Prim<R>& left, Prim<R>& right) {
  left = reconstruct(recon, limiter, wLL, wL, wR, R(1), gamma);
  right = reconstruct(recon, limiter, wL, wR, wRR, R(-1), gamma);
  if (!(left.rho > R(0) && left.p > R(0) && right.rho > R(0) && right.p > R(0))) {
    left = wL;
    right = wR;
  }
  if (wall != 0) {
    const Prim<R> inside = wall < 0 ? right : left;
    const R un = inside.u * nx + inside.v * ny;
    const Prim<R> mirror{inside.rho, inside.u - R(2) * un * nx, inside.v - R(2) * un * ny,
                         inside.p};
    if (wall < 0) {
      left = mirror;
      right = inside;
    } else {
      left = inside;
      right = mirror;
    }
  }
}

// farFieldState (src/engine-cpu/euler2d.ts:139-165).
template <class R>
__device__ __forceinline__ Prim<R> far_field_state(const Prim<R>& in, const Prim<R>& fr, R nx,
                                                   R ny, R gamma) {
  const R g = R(2) / (gamma - R(1));
  const R aIn = dsqrt((gamma * in.p) / in.rho);
  const R aFree = dsqrt((gamma * fr.p) / fr.rho);
  const R unIn = in.u * nx + in.v * ny;
  const R unFree = fr.u * nx + fr.v * ny;
  const R plus = unIn + aIn > R(0) ? unIn + g * aIn : unFree + g * aFree;
  const R minus = unIn - aIn > R(0) ? unIn - g * aIn : unFree - g * aFree;
  const R un = R(0.5) * (plus + minus);
  const R a = (plus - minus) / (R(2) * g);
  const Prim<R> up = unIn > R(0) ? in : fr;
  const R entropy = up.p / pow(up.rho, gamma);
  const R unUp = up.u * nx + up.v * ny;
  const R rho = pow((a * a) / (gamma * entropy), R(1) / (gamma - R(1)));
  return {rho, up.u + (un - unUp) * nx, up.v + (un - unUp) * ny, (rho * a * a) / gamma};
}

}  // namespace bsd
