// LU-SGS forward and backward sweeps as anti-diagonal wavefronts
// (implicitCorrection's sweeps, src/engine-cpu/euler2d.ts:1058-1102, and
// applyImplicitUpdate, :816-847, fused into the backward sweep).
//
// The forward sweep solves (D + L) dQ* = R cell by cell in the order j, then
// i; cell (i, j) needs only (i - 1, j) and (i, j - 1), both on the previous
// anti-diagonal i + j = d - 1, so every cell of a diagonal is independent and
// the sweep is ni + nj - 1 dependent steps. One CTA owns a case; thread j
// owns grid row j for the whole sweep and walks it along i as d advances:
//   - its west (forward) / east (backward) neighbour is the cell it finished
//     on the previous step, held in registers;
//   - its south / north neighbour is the cell thread j -+ 1 finished on the
//     previous step, exchanged through double-buffered shared memory;
//   - everything that does not depend on dQ (residual, diagonal, state, face
//     metrics) is prefetched one step ahead, so a step's critical path is the
//     exchange, the two neighbour terms and one division.
// One __syncthreads per diagonal orders the exchange.
//
// The operator runs in FP32. The neighbour term is the change of the
// physical flux, F(Q + dQ) - F(Q), exactly as the reference forms it, but
// evaluated in a rearranged form whose every term is proportional to dQ
// (no difference of two O(|F|) numbers), so FP32 rounding is relative to the
// term itself and vanishes with dQ.
#pragma once

#include "layout.cuh"

namespace bsd {

struct SweepArgs {
  const CaseDev* cases;
  const int* case_list;   // blockIdx.x -> case
  const int* active;      // per case (may be null)
  MetricsView m;
  const float4* r32;      // residual of each cell (pass A)
  const float4* q32;      // state of each cell (pass A)
  const float* diag;      // scalar diagonal (pass A)
  float4* dq;             // forward result, then the final correction
  float* cfl;             // per case current CFL number (ramped after the sweep)
  const float* cfl_max;   // per case
  const float* growth;    // per case
  const float* omega;     // per case
  unsigned* status;       // per case
};

template <class R>
struct UpdateArgs {
  StateView<R> q;         // the state, updated by the backward sweep
};

// Change of the physical flux along (nx, ny) of state q (pressure p) for the
// change d, times area/2, less omega lambda A / 2 times d, added to `sum`
// (the neighbour term, src/engine-cpu/euler2d.ts:977-1005).
__device__ __forceinline__ void neighbour_term(float4& sum, const float4 q, const float p,
                                               const float4 d, const float nx, const float ny,
                                               const float area, const float damp_lambda_a,
                                               const float gm1) {
  const float rho = q.x, mx = q.y, my = q.z, e = q.w;
  const float inv = 1.f / rho;
  const float u = mx * inv, v = my * inv;
  const float un = u * nx + v * ny;
  const float rho1 = rho + d.x;
  const float inv1 = 1.f / rho1;
  const float dmn = d.y * nx + d.z * ny;
  // u_n(Q + dQ) - u_n(Q)
  const float dun = (dmn - un * d.x) * inv1;
  // kinetic energy (|m|^2 / 2 rho) change, then pressure change
  const float dk = (rho * (u * d.y + v * d.z - 0.5f * (u * u + v * v) * d.x) +
                    0.5f * (d.y * d.y + d.z * d.z)) * inv1;
  const float dp = gm1 * (d.w - dk);
  const float half = 0.5f * area;
  sum.x += half * dmn - damp_lambda_a * d.x;
  sum.y += half * (d.y * un + (mx + d.y) * dun + dp * nx) - damp_lambda_a * d.y;
  sum.z += half * (d.z * un + (my + d.z) * dun + dp * ny) - damp_lambda_a * d.z;
  sum.w += half * ((d.w + dp) * un + (e + d.w + p + dp) * dun) - damp_lambda_a * d.w;
}

__device__ __forceinline__ float pressure32(const float4 q, float gm1) {
  return gm1 * (q.w - (0.5f * (q.y * q.y + q.z * q.z)) / q.x);
}

__device__ __forceinline__ float radius_q(const float4 q, float p, float gamma, float nx,
                                          float ny) {
  return fabsf((q.y * nx + q.z * ny) / q.x) + __fsqrt_rn((gamma * p) / q.x);
}

// Data of one cell that the sweep step needs and that does not depend on dQ.
struct SweepCell {
  float4 r;     // residual (forward) or dQ* (backward)
  float4 q;
  float4 face_i;  // west (forward) / east (backward) i-face
  float4 face_j;  // south (forward) / north (backward) j-face
  float d;
};

template <class R>
__global__ void __launch_bounds__(512) lusgs_sweep_kernel(const SweepArgs A,
                                                           const UpdateArgs<R> U) {
  extern __shared__ float4 smem[];
  const int c = A.case_list[blockIdx.x];
  if (A.active != nullptr && A.active[c] == 0) return;
  const CaseDev& cd = A.cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int nt = blockDim.x;
  const int j = threadIdx.x;
  const bool row = j < nj;
  const float gamma = float(cd.gamma);
  const float gm1 = gamma - 1.f;
  const float omega = A.omega[c];
  const float half_omega = 0.5f * omega;
  float4* sq = smem;              // [2][nt] state of the cell finished last step
  float4* sd = smem + 2 * nt;     // [2][nt] its dQ
  float* sp = reinterpret_cast<float*>(smem + 4 * nt);  // [2][nt] its pressure
  const int ndiag = ni + nj - 1;
  const int64_t cell0 = cd.cell + int64_t(j) * ni;

  auto fetch_forward = [&](int d, SweepCell& s) {
    const int i = d - j;
    if (!row || i < 0 || i >= ni) return;
    const int64_t k = cell0 + i;
    s.r = A.r32[k];
    s.q = A.q32[k];
    s.d = A.diag[k];
    s.face_i = A.m.iface[cd.iface + i + int64_t(j) * (ni + 1)];
    s.face_j = A.m.jface[cd.jface + i + int64_t(j) * ni];
  };

  // ---- forward sweep: (D + L) dQ* = R -------------------------------------
  float4 wq = make_float4(0, 0, 0, 0), wd = wq;
  float wp = 0;
  SweepCell cur{}, nxt{};
  fetch_forward(0, cur);
  for (int d = 0; d < ndiag; d++) {
    fetch_forward(d + 1, nxt);
    const int i = d - j;
    if (row && i >= 0 && i < ni) {
      const float p = pressure32(cur.q, gm1);
      float4 sum = make_float4(0, 0, 0, 0);
      if (i > 0) {
        const float4 f = cur.face_i;
        const float lam = fmaxf(radius_q(wq, wp, gamma, f.x, f.y), radius_q(cur.q, p, gamma, f.x, f.y)) * f.z;
        neighbour_term(sum, wq, wp, wd, -f.x, -f.y, f.z, half_omega * lam, gm1);
      }
      if (j > 0) {
        const int b = ((d - 1) & 1) * nt + j - 1;
        const float4 q = sq[b], dd = sd[b];
        const float ps = sp[b];
        const float4 f = cur.face_j;
        const float lam = fmaxf(radius_q(q, ps, gamma, f.x, f.y), radius_q(cur.q, p, gamma, f.x, f.y)) * f.z;
        neighbour_term(sum, q, ps, dd, -f.x, -f.y, f.z, half_omega * lam, gm1);
      }
      const float4 dq = make_float4((cur.r.x - sum.x) / cur.d, (cur.r.y - sum.y) / cur.d,
                                    (cur.r.z - sum.z) / cur.d, (cur.r.w - sum.w) / cur.d);
      A.dq[cell0 + i] = dq;
      const int b = (d & 1) * nt + j;
      sq[b] = cur.q;
      sd[b] = dq;
      sp[b] = p;
      wq = cur.q;
      wd = dq;
      wp = p;
    }
    cur = nxt;
    __syncthreads();
  }

  // ---- backward sweep: (D + U) dQ = D dQ*, then the update -----------------
  auto fetch_backward = [&](int d, SweepCell& s) {
    const int i = d - j;
    if (!row || i < 0 || i >= ni) return;
    const int64_t k = cell0 + i;
    s.r = A.dq[k];
    s.q = A.q32[k];
    s.d = A.diag[k];
    s.face_i = A.m.iface[cd.iface + i + 1 + int64_t(j) * (ni + 1)];
    s.face_j = A.m.jface[cd.jface + i + int64_t(j + 1) * ni];
  };
  const R rgamma = R(cd.gamma);
  bool bad = false;
  fetch_backward(ndiag - 1, cur);
  for (int d = ndiag - 1; d >= 0; d--) {
    if (d > 0) fetch_backward(d - 1, nxt);
    const int i = d - j;
    if (row && i >= 0 && i < ni) {
      const float p = pressure32(cur.q, gm1);
      float4 sum = make_float4(0, 0, 0, 0);
      if (i < ni - 1) {
        const float4 f = cur.face_i;
        const float lam = fmaxf(radius_q(cur.q, p, gamma, f.x, f.y), radius_q(wq, wp, gamma, f.x, f.y)) * f.z;
        neighbour_term(sum, wq, wp, wd, f.x, f.y, f.z, half_omega * lam, gm1);
      }
      if (j < nj - 1) {
        const int b = ((d + 1) & 1) * nt + j + 1;
        const float4 q = sq[b], dd = sd[b];
        const float pn = sp[b];
        const float4 f = cur.face_j;
        const float lam = fmaxf(radius_q(cur.q, p, gamma, f.x, f.y), radius_q(q, pn, gamma, f.x, f.y)) * f.z;
        neighbour_term(sum, q, pn, dd, f.x, f.y, f.z, half_omega * lam, gm1);
      }
      const float4 dq = make_float4(cur.r.x - sum.x / cur.d, cur.r.y - sum.y / cur.d,
                                    cur.r.z - sum.z / cur.d, cur.r.w - sum.w / cur.d);
      const int b = (d & 1) * nt + j;
      sq[b] = cur.q;
      sd[b] = dq;
      sp[b] = p;
      wq = cur.q;
      wd = dq;
      wp = p;
      // applyImplicitUpdate: halve the change until density and pressure
      // stay within a factor of two.
      const int64_t k = cell0 + i;
      const Cons<R> q0 = U.q.load(k);
      const R p0 = pressure_of(q0.rho, q0.mu, q0.mv, q0.e, rgamma);
      const R d0 = R(dq.x), d1 = R(dq.y), d2 = R(dq.z), d3 = R(dq.w);
      R alpha = R(1);
      for (int tries = 0; tries < 30; tries++) {
        const R rho1 = q0.rho + alpha * d0;
        const R p1 = pressure_of(rho1, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3, rgamma);
        if (rho1 > R(0.5) * q0.rho && rho1 < R(2) * q0.rho && p1 > R(0.5) * p0 && p1 < R(2) * p0) break;
        alpha *= R(0.5);
      }
      const Cons<R> q1{q0.rho + alpha * d0, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3};
      U.q.store(k, q1);
      if (!is_physical(q1, rgamma)) bad = true;
    }
    cur = nxt;
    __syncthreads();
  }
  if (bad) atomicOr(&A.status[c], STATUS_NON_PHYSICAL);
  if (threadIdx.x == 0) A.cfl[c] = fminf(A.cfl_max[c], A.cfl[c] * A.growth[c]);
}

}  // namespace bsd
