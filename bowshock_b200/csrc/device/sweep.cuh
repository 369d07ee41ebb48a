// LU-SGS forward and backward sweeps as anti-diagonal wavefronts
// (implicitCorrection's sweeps, src/engine-cpu/euler2d.ts:1058-1102), and
// the update that applies the correction (applyImplicitUpdate, :816-847).
//
// The forward sweep solves (D + L) dQ* = R cell by cell in the order j, then
// i; cell (i, j) needs only (i - 1, j) and (i, j - 1), both on the previous
// anti-diagonal, so the sweep is ni + nj - 1 dependent steps. One CTA owns a
// case; thread j of its consumer warps owns grid row j and walks it one
// diagonal per step:
//   - its neighbour along the row is the cell it finished on the previous
//     step (registers); its neighbour across rows is the one the next lane
//     finished, through an exchange row in shared memory that every lane
//     writes and reads, ordered by one named barrier per step among the
//     consumer warps (a __syncwarp for a case of up to 32 rows); on the
//     step's dependent chain one 16-byte store and load cost less than four
//     warp shuffles;
//   - everything a step needs that does not depend on dQ - the residual (or
//     dQ*), 1/D and the constants of the two neighbour terms - is one
//     80-byte record per cell that the residual pass wrote, stored by
//     anti-diagonal (sweep_slot) so that a run of diagonals is one
//     contiguous range;
//   - a producer warp stages those ranges into shared memory by TMA bulk
//     copies, K diagonals at a time into a ring of buffers with full and
//     empty mbarriers, so the consumers' steps carry no copy logic: the K
//     steps of a chunk are unrolled at compile time and have no branch.
// Every wait is bounded: a consumer wait that gives up sets STATUS_TIMEOUT
// (the case's state is then left alone), and the producer lets every copy it
// issued land (bounded) before the CTA leaves.
//
// The operator runs in FP32. The neighbour term is the change of the
// physical flux, F(Q + dQ) - F(Q), exactly as the reference forms it, but
// evaluated in a rearranged form whose every term is proportional to dQ
// (no difference of two O(|F|) numbers), so FP32 rounding is relative to the
// term itself and vanishes with dQ.
#pragma once

#include <algorithm>
#include <type_traits>
#include <utility>

#include "layout.cuh"

namespace bsd {

struct SweepArgs {
  const CaseDev* cases;
  const int* case_list;   // blockIdx.x -> case
  const int* active;      // per case (may be null)
  const float4* rec_f;    // forward records (sweep_slot order, REC_SIZE float4 each)
  float4* rec_b;          // backward records; the forward sweep writes dQ* into field 0
  float4* dq;             // final dQ, one float4 per cell at the case's cell offset (row-major)
  float* cfl;             // per case current CFL number (ramped after the sweep)
  const float* cfl_max;   // per case
  const float* growth;    // per case
  const float* omega;     // per case
  unsigned* status;       // per case
  int buffers;            // chunk buffers (NB, 2..kMaxSweepBuffers)
  int wait_limit;         // polls before a consumer's wait gives up
  int drain_limit;        // polls per copy for the producer's waits
};

// Fields of a record (five float4, written by the residual pass):
//   0: residual (forward) / dQ* (backward, written by the forward sweep)
//   1: (1/D, a.rho, a.u, a.v)     2: (a.H, a.hnx, a.hny, a.hud)
//   3: (b.rho, b.u, b.v, b.H)     4: (b.hnx, b.hny, b.hud, 0)
// for the neighbour along the row (a: west forward, east backward) and the
// one across rows (b: south forward, north backward): its density,
// velocity and total enthalpy per volume H = E + p, the face normal times
// A/2 signed for the direction the flux leaves (-n forward, +n backward),
// and hud = (u, v) . (hnx, hny) - omega lambda A/2. An absent neighbour has
// (1, 0, 0, 0) and (0, 0, 0): with its zero correction it adds exactly
// nothing. REC_SIZE (layout.cuh) is the record's five float4.

constexpr int kMaxSweepWarps = 16;    // nj <= 512
constexpr int kMaxSweepBuffers = 8;
// Header: full[8], empty[8] and the forward-done mbarrier, then the two
// two exchange rows of 32 warps + 2 float4 (row r's correction in slot r + 1,
// slots 0 and the last zero: the rows outside the grid).
__host__ __device__ inline size_t sweep_header_bytes(int warps) { return 256 + 2 * size_t(32 * warps + 2) * 16; }

// ---- TMA bulk copies and mbarriers (sm_90 and later; no multicast) --------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of `bar`; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int limit) {
  for (int k = 0; k < limit; k++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async;\n" ::: "memory");
}

// 1/x by the hardware approximation (rcp.approx.ftz.f32, within about one
// ulp): the LU-SGS operator runs in FP32 and only shapes the path to the
// steady state, whose residual is FP64.
__device__ __forceinline__ float approx_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}


__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// Barrier 1 among the consumer warps only (the producer warp never joins).
__device__ __forceinline__ void consumer_sync(int threads) {
  asm volatile("bar.sync 1, %0;\n" ::"r"(threads) : "memory");
}

// Shared memory of the sweep for chunks of `chunk` diagonals of up to
// `max_len` cells (the longest diagonal, min(ni, nj), of the launch's cases)
// in `buffers` buffers.
__host__ __device__ inline size_t sweep_smem_bytes(int max_len, int warps, int chunk, int buffers) {
  return sweep_header_bytes(warps) + size_t(buffers) * chunk * max_len * 16 * REC_SIZE;
}

// The neighbour term of src/engine-cpu/euler2d.ts:977-1005 - the change of
// the physical flux across the face, F(Q + d) - F(Q), times A/2, less
// omega lambda A/2 d - added to `sum`, for a neighbour stored as (rho, u, v,
// H) and (hnx, hny, hud). With m = rho (u, v), hun = (u, v) . (hnx, hny):
//   dK = (m . d_m - |m|^2/rho d_rho + |d_m|^2 / 2) / (rho + d_rho),
//   dp = (gamma - 1) (d_E - dK),
//   d(A/2 rho u_n) = hdmn = d_m . (hnx, hny),
//   A/2 d(u_n) = hdun = (hdmn - hun d_rho) / (rho + d_rho),
// and the term is (hdmn, d_m hun + (m + d_m) hdun + dp (hnx, hny),
// (d_E + dp) hun + (H + d_E + dp) hdun) - damp d, the damping folded into
// hud = hun - damp. Every term is proportional to d (no difference of two
// O(|F|) numbers), so FP32 rounding is relative to the term and d = 0 adds
// exactly nothing.
__device__ __forceinline__ void add_neighbour(float4& sum, float rho, float u, float v, float H, float hnx,
                                              float hny, float hud, const float4 d, float gm1, float hg) {
  const float mx = rho * u, my = rho * v;
  const float hun = hnx * u + hny * v;
  const float kk2 = mx * u + my * v;  // |m|^2 / rho
  const float inv1 = approx_rcp(rho + d.x);
  const float hdmn = d.y * hnx + d.z * hny;
  const float X = hdmn - hun * d.x;
  const float hdun = X * inv1;
  // 2 dK (rho + d_rho) = d_mx (2 mx + d_mx) + d_my (2 my + d_my) - kk2 d_rho
  float s = d.y * fmaf(2.f, mx, d.y);
  s = fmaf(d.z, fmaf(2.f, my, d.z), s);
  s = fmaf(-kk2, d.x, s);
  const float dp = fmaf(-hg, s * inv1, gm1 * d.w);  // hg = (gamma - 1) / 2
  sum.x += fmaf(hud, d.x, X);
  sum.y += fmaf(d.y, hud, fmaf(mx + d.y, hdun, dp * hnx));
  sum.z += fmaf(d.z, hud, fmaf(my + d.z, hdun, dp * hny));
  sum.w += fmaf(d.w, hud, fmaf(dp, hun, (H + d.w + dp) * hdun));
}

// The forward and backward sweeps of every active case, one CTA per case,
// leaving the final correction dQ in A.dq (row-major). The CTA has P + 1
// warps, P = ceil(nj / 32) of the launch's widest case: warps 0 .. W - 1
// sweep this case's W = ceil(nj / 32) warps of rows, warp P issues the
// copies, and the ones between (for narrower cases) leave at once.
//
// Chunks: a pass's diagonals in sweep order, K per chunk (the last may hold
// fewer); chunk g of the sequence (forward chunks, then backward ones) goes
// to buffer g % NB. Each chunk is one contiguous range of records: forward
// chunk cc holds diagonals [cc K, cc K + n), backward chunk cc the n
// diagonals ending at ndiag - cc K, both in memory order, the backward pass
// visiting its chunk from the top down.
template <int K, bool SOLO>
static __global__ void __launch_bounds__(32 * (kMaxSweepWarps + 1), 1) lusgs_sweep_kernel(const SweepArgs A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int c = A.case_list[blockIdx.x];
  if (A.active != nullptr && A.active[c] == 0) return;
  const CaseDev& cd = A.cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int P = (blockDim.x >> 5) - 1;  // the producer warp
  const int W = SOLO ? 1 : (nj + 31) >> 5;
  const int j = threadIdx.x, w = j >> 5, l = j & 31;
  const int NB = A.buffers;
  const int len_max = min(ni, nj);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);  // [kMaxSweepBuffers]
  uint64_t* empty = full + kMaxSweepBuffers;                // [kMaxSweepBuffers]
  uint64_t* fwd_done = empty + kMaxSweepBuffers;
  const int XS = 32 * P + 2;
  float4* xch = reinterpret_cast<float4*>(smem_raw + 256);  // [2][XS]
  float4* bufs = reinterpret_cast<float4*>(smem_raw + sweep_header_bytes(P));
  for (int k = threadIdx.x; k < 2 * XS; k += blockDim.x) xch[k] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (threadIdx.x == 0) {
    for (int b = 0; b < NB; b++) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], W);
    }
    mbar_init(fwd_done, W);
    mbar_fence_init();
  }
  __syncthreads();
  // Launched behind the residual pass that writes the records: wait for it.
  griddep_wait();
  const int ndiag = ni + nj - 1;
  const int nch = (ndiag + K - 1) / K;
  const int buf_stride = K * len_max * REC_SIZE;

  if (w == P) {
    // Producer: one lane issues every chunk of both passes in order; a
    // buffer is refilled once all W consumer warps have released it, and the
    // backward chunks wait until the forward pass's dQ* is written.
    if (l != 0) return;
    const float4* src_f = A.rec_f + REC_SIZE * cd.slot;
    const float4* src_b = A.rec_b + REC_SIZE * cd.slot;
    int issued = 0;
    for (int g = 0; g < 2 * nch; g++) {
      const int b = g % NB;
      if (g >= NB && !mbar_wait(&empty[b], unsigned(g / NB - 1) & 1u, A.drain_limit)) break;
      if (g == nch) {
        if (!mbar_wait(fwd_done, 0u, A.drain_limit)) break;
        fence_proxy_async();
      }
      const int pass = g / nch, cc = g - pass * nch;
      const int n = min(K, ndiag - cc * K);
      const int dlo = pass == 0 ? cc * K : ndiag - cc * K - n;
      const unsigned lo = diag_cells(ni, nj, dlo), hi = diag_cells(ni, nj, dlo + n);
      const unsigned bytes = (hi - lo) * 16u * REC_SIZE;
      mbar_arrive_expect_tx(&full[b], bytes);
      bulk_load(bufs + size_t(b) * buf_stride, (pass == 0 ? src_f : src_b) + size_t(REC_SIZE) * lo, bytes, &full[b]);
      issued = g + 1;
    }
    // The last NB copies issued are the only ones that can be in flight
    // (each buffer holds one at a time): let them land before leaving.
    for (int g = max(0, issued - NB); g < issued; g++)
      mbar_wait(&full[g % NB], unsigned(g / NB) & 1u, A.drain_limit);
    return;
  }
  if (w >= W) return;

  const float gm1 = float(cd.gamma) - 1.f, hg = 0.5f * gm1;
  float4* rec_b = A.rec_b + REC_SIZE * cd.slot;
  float4* dq_case = A.dq + cd.cell;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  bool failed = false;
  auto run_pass = [&](auto direction) {
    constexpr bool fwd = decltype(direction)::value;
    constexpr int pass = fwd ? 0 : 1;
    float4 pd = zero;  // the lane's previous cell's dQ (zero before its row starts)
    int t = 0;         // step of the pass (exchange parity)
    for (int cc = 0; cc < nch; cc++) {
      const int g = pass * nch + cc;
      const int b = g % NB;
      if (!failed) failed = !__all_sync(0xffffffffu, mbar_wait(&full[b], unsigned(g / NB) & 1u, A.wait_limit));
      const int n = min(K, ndiag - cc * K);
      const int dlo = fwd ? cc * K : ndiag - cc * K - n;
      const unsigned off_lo = diag_cells(ni, nj, dlo);
      int d = fwd ? dlo : dlo + n - 1;
      int boff = fwd ? 0 : int(diag_cells(ni, nj, d) - off_lo);  // d's first record in the chunk
      const float4* buf = bufs + b * buf_stride;
      // The step's records are in registers: the next step's are loaded
      // before this step's exchange store, since shared-memory loads cannot
      // be moved above a shared-memory store, and loaded after it they would
      // put their latency on the step's dependent chain (357 against 309
      // cycles a diagonal on 160 x 80).
      int jlo = max(0, d - ni + 1), jhi = min(d, nj - 1);
      float4 r0, r1, r2, r3, r4;
      {
        const float4* r = buf + REC_SIZE * (boff + min(max(j - jlo, 0), jhi - jlo));
        r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4];
      }
#pragma unroll
      for (int s = 0; s < K; s++) {
        // Steps past the chunk's end (its last) repeat its last diagonal
        // with nothing stored, so every warp meets the same barriers.
        const bool live = s < n;
        // Row j - 1's (forward) / j + 1's (backward) correction of the
        // previous step, from the exchange row (slot r + 1 holds row r).
        const float4 dn = xch[((t & 1) ^ 1) * XS + j + (fwd ? 0 : 2)];
        float4 sum = zero;
        add_neighbour(sum, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w, pd, gm1, hg);
        add_neighbour(sum, r3.x, r3.y, r3.z, r3.w, r4.x, r4.y, r4.z, dn, gm1, hg);
        const float inv_d = r1.x;
        float4 dq;
        if (fwd)
          dq = make_float4((r0.x - sum.x) * inv_d, (r0.y - sum.y) * inv_d, (r0.z - sum.z) * inv_d,
                           (r0.w - sum.w) * inv_d);
        else
          dq = make_float4(fmaf(-sum.x, inv_d, r0.x), fmaf(-sum.y, inv_d, r0.y), fmaf(-sum.z, inv_d, r0.z),
                           fmaf(-sum.w, inv_d, r0.w));
        const bool active = live & (j >= jlo) & (j <= jhi);
        if (active) {
          if (fwd)
            rec_b[size_t(REC_SIZE) * (off_lo + unsigned(boff + j - jlo))] = dq;
          else
            dq_case[unsigned(d - j) + unsigned(j) * unsigned(ni)] = dq;
        }
        pd = active ? dq : pd;
        if (s + 1 < K) {
          // The next diagonal (held in place past the chunk's end) and its records.
          if (s + 1 < n) {
            if (fwd) {
              boff += jhi - jlo + 1;
              d++;
            } else {
              d--;
              boff -= min(d, nj - 1) - max(0, d - ni + 1) + 1;
            }
          }
          jlo = max(0, d - ni + 1);
          jhi = min(d, nj - 1);
          const float4* r = buf + REC_SIZE * (boff + min(max(j - jlo, 0), jhi - jlo));
          r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4];
        }
        xch[(t & 1) * XS + j + 1] = pd;
        if (SOLO)
          __syncwarp();
        else
          consumer_sync(32 * W);
        t++;
      }
      // Every lane's reads of the buffer are done: release it.
      __syncwarp();
      if (l == 0) mbar_arrive(&empty[b]);
    }
    if (fwd) {
      // dQ* written above is read by the backward pass's bulk copies.
      fence_proxy_async();
      __syncwarp();
      if (l == 0) mbar_arrive(fwd_done);
    }
  };
  run_pass(std::true_type{});
  run_pass(std::false_type{});
  if (failed) {
    if (l == 0) atomicOr(&A.status[c], STATUS_TIMEOUT);
    return;
  }
  if (threadIdx.x == 0) A.cfl[c] = fminf(A.cfl_max[c], A.cfl[c] * A.growth[c]);
}

// The update of every cell of every active case, from `src` into `dst` (the
// same arrays, or the other buffer of the state); flags non-physical
// results. A case whose sweep gave up (dQ incomplete) keeps its state.
template <class R>
__global__ void __launch_bounds__(TILE_THREADS) lusgs_update_kernel(const CaseDev* cases,
                                                                    const int2* tiles,
                                                                    const int* active,
                                                                    StateView<R> src,
                                                                    StateView<R> dst,
                                                                    const float4* dq,
                                                                    unsigned* status) {
  const int2 tile = tiles[blockIdx.x];
  const int c = tile.x;
  if (active != nullptr && active[c] == 0) return;
  const bool keep = (status[c] & STATUS_TIMEOUT) != 0;
  const CaseDev& cd = cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int tiles_i = (ni + TI - 1) / TI;
  const int i = (tile.y % tiles_i) * TI + threadIdx.x % TI;
  const int j = (tile.y / tiles_i) * TJ + threadIdx.x / TI;
  bool bad = false;
  if (i < ni && j < nj && int(threadIdx.x) < TI * TJ) {
    const R gamma = R(cd.gamma);
    const int64_t k = cd.cell + i + int64_t(j) * ni;
    const Cons<R> q0 = src.load(k);
    const Cons<R> q1 = keep ? q0 : implicit_update(q0, dq[k], gamma);
    dst.store(k, q1);
    bad = !is_physical(q1, gamma);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&status[c], STATUS_NON_PHYSICAL);
}

// Launch shape of the sweep: diagonals per chunk and chunk buffers.
struct SweepShape {
  int chunk = 0, buffers = 0;
};

// The shape for cases whose longest diagonal is `max_len` cells when
// `cases_in_flight` cases sweep at once: within the shared memory each CTA
// may take (the resident cases, up to 8 per SM, share an SM's), the longest
// chunk of up to `max_chunk` diagonals in at least two buffers, then as many
// buffers as fit, up to four. A chunk's steps are unrolled, so longer chunks
// amortise its wait (one case of 160 x 80 alone: 301 cycles a diagonal with
// K = 16 in two buffers, 313 with K = 8 in three), but fewer buffers copy
// less far ahead, which counts when other kernels load HBM at the same time.
// When not even one diagonal in two buffers fits a CTA's share, the smallest
// shape is taken rather than the largest: a batch that large is bound by
// throughput, and a sweep CTA that fills an SM's shared memory leaves no room
// beside it for the other cases' sweeps or residual passes.
inline SweepShape sweep_shape(int max_len, int warps, int cases_in_flight, int max_chunk = 8) {
  const int per_sm = std::min(8, std::max(1, (cases_in_flight + 147) / 148));
  const size_t budget = size_t(220 * 1024) / per_sm;
  for (int k = 16; k >= 1; k /= 2) {
    if (k > max_chunk || sweep_smem_bytes(max_len, warps, k, 2) > budget) continue;
    int nb = 2;
    while (nb < 4 && sweep_smem_bytes(max_len, warps, k, nb + 1) <= budget) nb++;
    return {k, nb};
  }
  if (sweep_smem_bytes(max_len, warps, 1, 2) <= size_t(220 * 1024)) return {1, 2};
  return {};
}

constexpr int kSweepWaitLimit = 1 << 22;

// Launches `kernel` with the programmatic stream-serialization attribute when
// `pdl` (the kernel must then wait with griddep_wait before it touches what
// the kernel ahead of it in the stream reads or writes).
template <class... Params, class... Args>
inline cudaError_t launch_maybe_pdl(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                                    cudaStream_t stream, bool pdl, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <int K>
inline cudaError_t launch_sweep_k(const SweepArgs& A, int n_cases, int warps, size_t bytes, cudaStream_t stream,
                                  bool pdl) {
  cudaError_t e;
  if (warps == 1) {
    e = cudaFuncSetAttribute(lusgs_sweep_kernel<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (e != cudaSuccess) return e;
    e = launch_maybe_pdl(lusgs_sweep_kernel<K, true>, dim3(n_cases), dim3(64), bytes, stream, pdl, A);
  } else {
    e = cudaFuncSetAttribute(lusgs_sweep_kernel<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (e != cudaSuccess) return e;
    e = launch_maybe_pdl(lusgs_sweep_kernel<K, false>, dim3(n_cases), dim3(32 * (warps + 1)), bytes, stream, pdl, A);
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// `max_nj` and `max_len`: the launch's widest case and longest diagonal;
// `cases_in_flight`: cases of the whole batch sweeping at the same time
// (other lanes included), which sets the shared memory each CTA may take.
// `wait_limit` < 0 keeps the default bound; `pdl`: launched behind the
// residual pass by programmatic dependent launch.
inline cudaError_t launch_sweep(SweepArgs A, int n_cases, int max_nj, int max_len, int cases_in_flight,
                                cudaStream_t stream, int wait_limit = -1, int max_chunk = 8, bool pdl = false) {
  const int warps = (max_nj + 31) / 32;
  if (warps > kMaxSweepWarps || max_nj + max_len > 65536) return cudaErrorInvalidConfiguration;
  const SweepShape shape = sweep_shape(max_len, warps, cases_in_flight, max_chunk);
  if (shape.chunk == 0) return cudaErrorInvalidConfiguration;
  A.buffers = shape.buffers;
  A.wait_limit = wait_limit < 0 ? kSweepWaitLimit : wait_limit;
  A.drain_limit = kSweepWaitLimit;
  const size_t bytes = sweep_smem_bytes(max_len, warps, shape.chunk, shape.buffers);
  switch (shape.chunk) {
    case 16: return launch_sweep_k<16>(A, n_cases, warps, bytes, stream, pdl);
    case 8: return launch_sweep_k<8>(A, n_cases, warps, bytes, stream, pdl);
    case 4: return launch_sweep_k<4>(A, n_cases, warps, bytes, stream, pdl);
    case 2: return launch_sweep_k<2>(A, n_cases, warps, bytes, stream, pdl);
    default: return launch_sweep_k<1>(A, n_cases, warps, bytes, stream, pdl);
  }
}

}  // namespace bsd
