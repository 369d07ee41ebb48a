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

// ---- asynchronous global -> shared copies (cp.async, sm_80 and later) ------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A cell's state as the neighbour term needs it: conserved (rho, mx, my, E)
// and the derived (u, v, a, p) - all independent of dQ, so they are computed
// off the sweep's critical path and handed to the next row with the dQ.
struct NbrState {
  float4 q;
  float4 w;  // u, v, sound speed, pressure
};

__device__ __forceinline__ NbrState derive(const float4 q, float gamma, float gm1) {
  const float inv = __frcp_rn(q.x);
  const float u = q.y * inv, v = q.z * inv;
  const float p = gm1 * (q.w - 0.5f * (q.y * u + q.z * v));
  const float a = __fsqrt_rn(gamma * p * inv);
  return {q, make_float4(u, v, a, p)};
}

// Change of the physical flux along (nx, ny) of state s for the change d,
// times area/2, less (omega lambda A / 2) d, added to `sum` (the neighbour
// term, src/engine-cpu/euler2d.ts:977-1005) - the exact difference
// F(Q + dQ) - F(Q) written so that every term is proportional to dQ. d = 0
// contributes exactly nothing, which stands for an absent neighbour.
__device__ __forceinline__ void neighbour_change(float4& sum, const NbrState& s, const float4 d,
                                                 float nx, float ny, float half_area,
                                                 float damp, float gm1) {
  const float u = s.w.x, v = s.w.y, p = s.w.w;
  const float un = u * nx + v * ny;
  const float inv1 = __frcp_rn(s.q.x + d.x);
  const float dmn = d.y * nx + d.z * ny;
  const float dun = (dmn - un * d.x) * inv1;
  const float dk = (s.q.x * (u * d.y + v * d.z - 0.5f * (u * u + v * v) * d.x) +
                    0.5f * (d.y * d.y + d.z * d.z)) * inv1;
  const float dp = gm1 * (d.w - dk);
  sum.x += half_area * dmn - damp * d.x;
  sum.y += half_area * (d.y * un + (s.q.y + d.y) * dun + dp * nx) - damp * d.y;
  sum.z += half_area * (d.z * un + (s.q.z + d.z) * dun + dp * ny) - damp * d.z;
  sum.w += half_area * ((d.w + dp) * un + (s.q.w + d.w + p + dp) * dun) - damp * d.w;
}

__device__ __forceinline__ float spectral(const NbrState& s, float nx, float ny) {
  return fabsf(s.w.x * nx + s.w.y * ny) + s.w.z;
}

// Shared memory of the sweep kernel for `nt` threads and a prefetch ring of
// `depth` slots: each thread stages the data of its next `depth` cells
// (everything that does not depend on dQ) in its own ring, so global-memory
// latency overlaps the dependent chain of diagonal steps.
__host__ __device__ constexpr size_t sweep_smem_bytes(int nt, int depth) {
  // exchange: q, w, dq (float4), double-buffered; ring: r, q, face_i,
  // face_j (float4) and diag (float) per slot.
  return size_t(nt) * (2 * 3 * 16 + depth * (4 * 16 + 4));
}

// The forward and backward sweeps of every active case, one CTA per case,
// leaving the final correction dQ in A.dq for lusgs_update_kernel.
template <int kSweepDepth>
__global__ void __launch_bounds__(512) lusgs_sweep_kernel(const SweepArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = A.case_list[blockIdx.x];
  if (A.active != nullptr && A.active[c] == 0) return;
  const CaseDev& cd = A.cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int nt = blockDim.x;
  const int j = threadIdx.x;
  const bool row = j < nj;
  const float gamma = float(cd.gamma);
  const float gm1 = gamma - 1.f;
  const float half_omega = 0.5f * A.omega[c];
  const int ndiag = ni + nj - 1;
  const int64_t cell0 = cd.cell + int64_t(j) * ni;
  const int64_t if0 = cd.iface + int64_t(j) * (ni + 1);
  const int64_t jf0 = cd.jface + int64_t(j) * ni;

  float4* xq = reinterpret_cast<float4*>(smem_raw);  // [2][nt] exchange: state
  float4* xw = xq + 2 * nt;                           // [2][nt] derived
  float4* xd = xw + 2 * nt;                           // [2][nt] dQ
  float4* ring_r = xd + 2 * nt;                       // [depth][nt]
  float4* ring_q = ring_r + kSweepDepth * nt;
  float4* ring_fi = ring_q + kSweepDepth * nt;
  float4* ring_fj = ring_fi + kSweepDepth * nt;
  float* ring_d = reinterpret_cast<float*>(ring_fj + kSweepDepth * nt);

  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);

  // One sweep: `dir` +1 forward (neighbours i - 1 and j - 1, faces (i, j)),
  // -1 backward (neighbours i + 1 and j + 1, faces (i + 1, j) and (i, j + 1)).
  for (int pass = 0; pass < 2; pass++) {
    const bool fwd = pass == 0;
    auto cell_at = [&](int step) { return (fwd ? step : ndiag - 1 - step) - j; };
    auto fetch = [&](int step) {
      const int i = cell_at(step);
      if (row && step < ndiag && i >= 0 && i < ni) {
        const int slot = (step % kSweepDepth) * nt + j;
        const int64_t k = cell0 + i;
        cp_async16(&ring_r[slot], fwd ? &A.r32[k] : &A.dq[k]);
        cp_async16(&ring_q[slot], &A.q32[k]);
        cp_async16(&ring_fi[slot], &A.m.iface[if0 + i + (fwd ? 0 : 1)]);
        cp_async16(&ring_fj[slot], &A.m.jface[jf0 + i + (fwd ? 0 : ni)]);
        cp_async4(&ring_d[slot], &A.diag[k]);
      }
      cp_async_commit();
    };
    for (int s = 0; s < kSweepDepth; s++) fetch(s);
    // The neighbour along the row: the cell this thread finished last step.
    NbrState prev{make_float4(1.f, 0.f, 0.f, 1.f), make_float4(0.f, 0.f, 1.f, 1.f)};
    float4 prev_dq = zero;
    for (int step = 0; step < ndiag; step++) {
      cp_async_wait<kSweepDepth - 1>();
      const int d = fwd ? step : ndiag - 1 - step;
      const int i = d - j;
      const bool live = row && i >= 0 && i < ni;
      NbrState self{};
      float4 r = zero, fi = zero, fj = zero;
      float inv_d = 0.f;
      if (live) {
        // Everything here is independent of dQ.
        const int slot = (step % kSweepDepth) * nt + j;
        r = ring_r[slot];
        fi = ring_fi[slot];
        fj = ring_fj[slot];
        inv_d = __frcp_rn(ring_d[slot]);
        self = derive(ring_q[slot], gamma, gm1);
      }
      const float sx = fwd ? -1.f : 1.f;  // the flux leaves the cell being solved
      const float rad_i = live ? spectral(self, fi.x, fi.y) : 0.f;
      const float rad_j = live ? spectral(self, fj.x, fj.y) : 0.f;
      // Neighbour across the j-face: thread j -+ 1's cell of the last step.
      const int nb = fwd ? j - 1 : j + 1;
      const bool has_j = live && (fwd ? j > 0 : j < nj - 1);
      const bool has_i = live && (fwd ? i > 0 : i < ni - 1);
      NbrState other = self;
      float4 other_dq = zero;
      if (has_j) {
        const int b = ((step - 1) & 1) * nt + nb;
        other.q = xq[b];
        other.w = xw[b];
        other_dq = xd[b];
      }
      if (live) {
        const float4 dq_i = has_i ? prev_dq : zero;
        const NbrState& si = has_i ? prev : self;
        const float lam_i = fmaxf(spectral(si, fi.x, fi.y), rad_i) * fi.z;
        const float lam_j = fmaxf(spectral(other, fj.x, fj.y), rad_j) * fj.z;
        float4 sum = zero;
        neighbour_change(sum, si, dq_i, sx * fi.x, sx * fi.y, 0.5f * fi.z, half_omega * lam_i, gm1);
        neighbour_change(sum, other, other_dq, sx * fj.x, sx * fj.y, 0.5f * fj.z,
                         half_omega * lam_j, gm1);
        float4 dq;
        if (fwd) {
          dq = make_float4((r.x - sum.x) * inv_d, (r.y - sum.y) * inv_d, (r.z - sum.z) * inv_d,
                           (r.w - sum.w) * inv_d);
        } else {
          dq = make_float4(r.x - sum.x * inv_d, r.y - sum.y * inv_d, r.z - sum.z * inv_d,
                           r.w - sum.w * inv_d);
        }
        const int b = (step & 1) * nt + j;
        xq[b] = self.q;
        xw[b] = self.w;
        xd[b] = dq;
        A.dq[cell0 + i] = dq;
        prev = self;
        prev_dq = dq;
      }
      __syncthreads();
      fetch(step + kSweepDepth);
    }
    cp_async_wait<0>();
    __syncthreads();
  }
  if (threadIdx.x == 0) A.cfl[c] = fminf(A.cfl_max[c], A.cfl[c] * A.growth[c]);
}

// applyImplicitUpdate (src/engine-cpu/euler2d.ts:816-847) for every cell of
// every active case: Q += alpha dQ with alpha halved until density and
// pressure stay within a factor of two; flags non-physical results.
template <class R>
__global__ void __launch_bounds__(TILE_THREADS) lusgs_update_kernel(const CaseDev* cases,
                                                                    const int2* tiles,
                                                                    const int* active,
                                                                    StateView<R> q,
                                                                    const float4* dq,
                                                                    unsigned* status) {
  const int2 tile = tiles[blockIdx.x];
  const int c = tile.x;
  if (active != nullptr && active[c] == 0) return;
  const CaseDev& cd = cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int tiles_i = (ni + TI - 1) / TI;
  const int i = (tile.y % tiles_i) * TI + threadIdx.x % TI;
  const int j = (tile.y / tiles_i) * TJ + threadIdx.x / TI;
  bool bad = false;
  if (i < ni && j < nj) {
    const R gamma = R(cd.gamma);
    const int64_t k = cd.cell + i + int64_t(j) * ni;
    const Cons<R> q0 = q.load(k);
    const float4 d4 = dq[k];
    const R p0 = pressure_of(q0.rho, q0.mu, q0.mv, q0.e, gamma);
    const R d0 = R(d4.x), d1 = R(d4.y), d2 = R(d4.z), d3 = R(d4.w);
    R alpha = R(1);
    for (int tries = 0; tries < 30; tries++) {
      const R rho1 = q0.rho + alpha * d0;
      const R p1 = pressure_of(rho1, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3, gamma);
      if (rho1 > R(0.5) * q0.rho && rho1 < R(2) * q0.rho && p1 > R(0.5) * p0 && p1 < R(2) * p0) break;
      alpha *= R(0.5);
    }
    const Cons<R> q1{q0.rho + alpha * d0, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3};
    q.store(k, q1);
    bad = !is_physical(q1, gamma);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&status[c], STATUS_NON_PHYSICAL);
}

// Launches the sweep kernel with the deepest prefetch ring that fits the
// shared memory of one CTA (8 slots for up to 384 rows, 4 beyond).
inline cudaError_t launch_sweep(const SweepArgs& A, int n_cases, int max_nj, cudaStream_t stream) {
  const int nt = ((max_nj + 31) / 32) * 32;
  constexpr size_t kLimit = 227 * 1024;
  const size_t deep = sweep_smem_bytes(nt, 8);
  if (deep <= kLimit) {
    cudaError_t e = cudaFuncSetAttribute(lusgs_sweep_kernel<8>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(deep));
    if (e != cudaSuccess) return e;
    lusgs_sweep_kernel<8><<<n_cases, nt, deep, stream>>>(A);
    return cudaGetLastError();
  }
  const size_t shallow = sweep_smem_bytes(nt, 4);
  cudaError_t e = cudaFuncSetAttribute(lusgs_sweep_kernel<4>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(shallow));
  if (e != cudaSuccess) return e;
  lusgs_sweep_kernel<4><<<n_cases, nt, shallow, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace bsd
