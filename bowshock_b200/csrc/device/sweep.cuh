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
  const float4* rec;      // the sweep record of each cell (5 float4, pass A)
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

// Change of the physical flux along (nx, ny) of state q (with u, v, p in
// w) for the change d, times half_area, less damp d, added to `sum` (the
// neighbour term, src/engine-cpu/euler2d.ts:977-1005: half_area = A / 2,
// damp = omega lambda A / 2) - the exact difference F(Q + dQ) - F(Q) written
// so that every term is proportional to dQ. d = 0 contributes exactly
// nothing, which stands for an absent neighbour.
__device__ __forceinline__ void neighbour_change(float4& sum, const float4 q, const float4 w,
                                                 const float4 d, float nx, float ny,
                                                 float half_area, float damp, float gm1) {
  const float u = w.x, v = w.y, p = w.z;
  const float un = u * nx + v * ny;
  const float inv1 = __frcp_rn(q.x + d.x);
  const float dmn = d.y * nx + d.z * ny;
  const float dun = (dmn - un * d.x) * inv1;
  const float dk = (q.x * (u * d.y + v * d.z - 0.5f * (u * u + v * v) * d.x) +
                    0.5f * (d.y * d.y + d.z * d.z)) * inv1;
  const float dp = gm1 * (d.w - dk);
  sum.x += half_area * dmn - damp * d.x;
  sum.y += half_area * (d.y * un + (q.y + d.y) * dun + dp * nx) - damp * d.y;
  sum.z += half_area * (d.z * un + (q.z + d.z) * dun + dp * ny) - damp * d.z;
  sum.w += half_area * ((d.w + dp) * un + (q.w + d.w + p + dp) * dun) - damp * d.w;
}

// Fields of the sweep record (five float4 per cell, written by the residual
// pass): residual; state; (u, v, p, 1/D); west face and south face as
// (nx, ny, A/2, omega lambda A / 2).
enum { REC_R = 0, REC_Q = 1, REC_W = 2, REC_FW = 3, REC_FS = 4, REC_SIZE = 5 };

// Shared memory of the sweep kernel for `nt` threads and a prefetch ring of
// `depth` slots: each thread stages the records of its next `depth` cells in
// its own ring (cp.async), so memory latency overlaps the dependent chain of
// diagonal steps.
__host__ __device__ constexpr size_t sweep_smem_bytes(int nt, int depth) {
  // exchange: state, (u, v, p, 1/D), dQ, south face (float4), double-buffered;
  // ring: the record and dQ* (6 float4) per slot.
  return size_t(nt) * 16 * (2 * 4 + depth * (REC_SIZE + 1));
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
  const float gm1 = float(cd.gamma) - 1.f;
  const int ndiag = ni + nj - 1;
  const int64_t cell0 = cd.cell + int64_t(j) * ni;

  float4* xq = reinterpret_cast<float4*>(smem_raw);  // [2][nt] exchange: state
  float4* xw = xq + 2 * nt;                           // (u, v, p, 1/D)
  float4* xd = xw + 2 * nt;                           // dQ
  float4* xf = xd + 2 * nt;                           // south face record
  float4* ring = xf + 2 * nt;                         // [depth][6][nt]
  auto at = [&](int step, int field) { return ring + ((step % kSweepDepth) * (REC_SIZE + 1) + field) * nt + j; };
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);

  for (int pass = 0; pass < 2; pass++) {
    const bool fwd = pass == 0;
    auto fetch = [&](int step) {
      const int i = (fwd ? step : ndiag - 1 - step) - j;
      if (row && step < ndiag && i >= 0 && i < ni) {
        const float4* src = A.rec + REC_SIZE * (cell0 + i);
#pragma unroll
        for (int f = 0; f < REC_SIZE; f++) cp_async16(at(step, f), src + f);
        if (!fwd) cp_async16(at(step, REC_SIZE), &A.dq[cell0 + i]);
      }
      cp_async_commit();
    };
    for (int s = 0; s < kSweepDepth; s++) fetch(s);
    // The cell this thread finished last step (its neighbour along the row).
    float4 pq = make_float4(1.f, 0.f, 0.f, 1.f), pw = make_float4(0.f, 0.f, 1.f, 1.f);
    float4 pd = zero, pfw = zero;
    for (int step = 0; step < ndiag; step++) {
      cp_async_wait<kSweepDepth - 1>();
      const int d = fwd ? step : ndiag - 1 - step;
      const int i = d - j;
      if (row && i >= 0 && i < ni) {
        const float4 q = *at(step, REC_Q), w = *at(step, REC_W);
        const float4 fw = *at(step, REC_FW), fs = *at(step, REC_FS);
        const float4 base = *at(step, fwd ? REC_R : REC_SIZE);
        const bool has_i = fwd ? i > 0 : i < ni - 1;
        const bool has_j = fwd ? j > 0 : j < nj - 1;
        // Across the j-face: the cell thread j -+ 1 finished last step.
        float4 oq = q, ow = w, od = zero, of = fs;
        if (has_j) {
          const int b = ((step - 1) & 1) * nt + (fwd ? j - 1 : j + 1);
          oq = xq[b];
          ow = xw[b];
          od = xd[b];
          if (!fwd) of = xf[b];
        }
        // Forward: the faces are this cell's west and south faces, the flux
        // leaving through -n; backward: the east neighbour's west face and
        // the north neighbour's south face, through +n.
        const float s = fwd ? -1.f : 1.f;
        const float4 face_i = fwd ? fw : pfw;
        const float4 face_j = fwd ? fs : of;
        float4 sum = zero;
        neighbour_change(sum, has_i ? pq : q, has_i ? pw : w, has_i ? pd : zero, s * face_i.x,
                         s * face_i.y, face_i.z, face_i.w, gm1);
        neighbour_change(sum, oq, ow, od, s * face_j.x, s * face_j.y, face_j.z, face_j.w, gm1);
        const float inv_d = w.w;
        float4 dq;
        if (fwd) {
          dq = make_float4((base.x - sum.x) * inv_d, (base.y - sum.y) * inv_d,
                           (base.z - sum.z) * inv_d, (base.w - sum.w) * inv_d);
        } else {
          dq = make_float4(base.x - sum.x * inv_d, base.y - sum.y * inv_d,
                           base.z - sum.z * inv_d, base.w - sum.w * inv_d);
        }
        const int b = (step & 1) * nt + j;
        xq[b] = q;
        xw[b] = w;
        xd[b] = dq;
        xf[b] = fs;
        A.dq[cell0 + i] = dq;
        pq = q;
        pw = w;
        pd = dq;
        pfw = fw;
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
// shared memory of one CTA.
template <int kDepth>
inline cudaError_t launch_sweep_depth(const SweepArgs& A, int n_cases, int nt, cudaStream_t stream) {
  const size_t bytes = sweep_smem_bytes(nt, kDepth);
  const cudaError_t e = cudaFuncSetAttribute(lusgs_sweep_kernel<kDepth>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (e != cudaSuccess) return e;
  lusgs_sweep_kernel<kDepth><<<n_cases, nt, bytes, stream>>>(A);
  return cudaGetLastError();
}

inline cudaError_t launch_sweep(const SweepArgs& A, int n_cases, int max_nj, cudaStream_t stream) {
  const int nt = ((max_nj + 31) / 32) * 32;
  constexpr size_t kLimit = 227 * 1024;
  if (sweep_smem_bytes(nt, 8) <= kLimit) return launch_sweep_depth<8>(A, n_cases, nt, stream);
  if (sweep_smem_bytes(nt, 6) <= kLimit) return launch_sweep_depth<6>(A, n_cases, nt, stream);
  return launch_sweep_depth<3>(A, n_cases, nt, stream);
}

}  // namespace bsd
