// LU-SGS forward and backward sweeps as anti-diagonal wavefronts
// (implicitCorrection's sweeps, src/engine-cpu/euler2d.ts:1058-1102), and
// the update that applies the correction (applyImplicitUpdate, :816-847).
//
// The forward sweep solves (D + L) dQ* = R cell by cell in the order j, then
// i; cell (i, j) needs only (i - 1, j) and (i, j - 1), both on the previous
// anti-diagonal, so the sweep is ni + nj - 1 dependent steps. One CTA owns a
// case and thread j owns grid row j; the rows are cut into warps of 32, and
// the warps run decoupled, with no CTA-wide barrier in the sweeps:
//   - a warp walks its own rows' cells diagonal by diagonal; the neighbour
//     along the row is the lane's own previous cell (registers), the
//     neighbour across rows is the next lane's previous cell: its dQ by warp
//     shuffle, its state from the records in shared memory;
//   - at a warp edge the neighbour row belongs to the next warp: its state
//     is a ghost row of this warp's records (the residual pass writes that
//     row's records twice), and its dQ arrives through a small ring of
//     shared-memory slots, one per cell column, that the producing lane
//     fills and the consuming lane empties (a slot holds a NaN sentinel
//     while empty, so one 16-byte slot is both the flag and the data);
//   - each warp stages its own records into shared memory by TMA bulk
//     copies, a chunk of diagonals at a time, with a ring of chunk buffers
//     whose mbarriers only that warp waits on.
// The warps of a case therefore form a pipeline whose rate is one warp's
// step, not a CTA barrier's. Every wait is bounded: a wait that gives up sets
// STATUS_TIMEOUT and the kernel drains its copies and leaves.
//
// The operator runs in FP32. The neighbour term is the change of the
// physical flux, F(Q + dQ) - F(Q), exactly as the reference forms it, but
// evaluated in a rearranged form whose every term is proportional to dQ
// (no difference of two O(|F|) numbers), so FP32 rounding is relative to the
// term itself and vanishes with dQ.
#pragma once

#include <algorithm>
#include <type_traits>

#include "layout.cuh"

namespace bsd {

struct SweepArgs {
  const CaseDev* cases;
  const int* case_list;   // blockIdx.x -> case
  const int* active;      // per case (may be null)
  const float4* rec_f;    // forward records (sweep_block_slot layout, 5 float4 per slot)
  float4* rec_b;          // backward records; the forward sweep writes dQ* into field 0
  float4* dq;             // final dQ, one float4 per cell at the case's cell offset (row-major)
  float* cfl;             // per case current CFL number (ramped after the sweep)
  const float* cfl_max;   // per case
  const float* growth;    // per case
  const float* omega;     // per case
  unsigned* status;       // per case
  int chunk;              // diagonals per bulk copy (K)
  int buffers;            // chunk buffers per warp (NB, 2..kMaxSweepBuffers)
  int wait_limit;         // polls before a wait gives up
  int drain_limit;        // polls per copy when draining after a failure
};

// Fields of the records (five float4 per slot, written by the residual pass):
//   forward:  residual | state | (u, v, p, 1/D) | west face | south face
//   backward: dQ*      | state | (u, v, p, 1/D) | east face | north face
// with each face as (nx, ny, A/2, omega lambda A / 2).
enum { REC_R = 0, REC_Q = 1, REC_W = 2, REC_FA = 3, REC_FB = 4, REC_SIZE = 5 };

constexpr int kMaxSweepWarps = 16;    // nj <= 512
constexpr int kMaxSweepBuffers = 4;
constexpr int kEdgeRing = 32;         // slots per warp-edge ring (a power of two)
constexpr unsigned kEdgeEmpty = 0x7f80beefu;  // a NaN no arithmetic produces
// Header: the warps' chunk mbarriers and the abort word.
constexpr size_t kSweepHeader = 8 * kMaxSweepWarps * kMaxSweepBuffers + 128;

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

// ---- the warp-edge rings ----------------------------------------------------
__device__ __forceinline__ uint4 lds_volatile_u4(const float4* p) {
  uint4 v;
  asm volatile("ld.volatile.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(smem_u32(p))
               : "memory");
  return v;
}
__device__ __forceinline__ void sts_volatile_u4(float4* p, uint4 v) {
  asm volatile("st.volatile.shared.v4.u32 [%0], {%1, %2, %3, %4};\n" ::"r"(smem_u32(p)), "r"(v.x),
               "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}
__device__ __forceinline__ bool all_empty(uint4 v) {
  return v.x == kEdgeEmpty && v.y == kEdgeEmpty && v.z == kEdgeEmpty && v.w == kEdgeEmpty;
}
__device__ __forceinline__ bool none_empty(uint4 v) {
  return v.x != kEdgeEmpty && v.y != kEdgeEmpty && v.z != kEdgeEmpty && v.w != kEdgeEmpty;
}
__device__ __forceinline__ bool aborted(const int* abort_word) {
  return *reinterpret_cast<const volatile int*>(abort_word) != 0;
}

// Warp-collective handoffs of one column's dQ at a warp edge. Every lane of
// the warp polls the slot with the same (broadcast) read, so the loop and its
// outcome are the same in every lane and the warp never diverges; only the
// edge lane (`me`) stores. Put: once all four words of the slot read empty
// (the consumer's emptying store has landed in full), the edge lane stores
// its dQ. Get: once none of the four words is empty, the edge lane takes the
// dQ and empties the slot. False if the wait gave up (the limit, or another
// warp's abort).
__device__ __forceinline__ bool warp_edge_put(float4* ring, int i, float4 d, bool me, int limit,
                                              const int* abort_word) {
  float4* s = ring + (i & (kEdgeRing - 1));
  for (int k = 0;; k++) {
    if (all_empty(lds_volatile_u4(s))) break;
    if (k >= limit || ((k & 63) == 63 && aborted(abort_word))) return false;
  }
  if (me)
    sts_volatile_u4(s, make_uint4(__float_as_uint(d.x), __float_as_uint(d.y), __float_as_uint(d.z),
                                  __float_as_uint(d.w)));
  return true;
}
__device__ __forceinline__ bool warp_edge_get(float4* ring, int i, float4& d, bool me, int limit,
                                              const int* abort_word) {
  float4* s = ring + (i & (kEdgeRing - 1));
  uint4 v;
  for (int k = 0;; k++) {
    v = lds_volatile_u4(s);
    if (none_empty(v)) break;
    if (k >= limit || ((k & 63) == 63 && aborted(abort_word))) return false;
  }
  if (me) {
    sts_volatile_u4(s, make_uint4(kEdgeEmpty, kEdgeEmpty, kEdgeEmpty, kEdgeEmpty));
    d = make_float4(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z), __uint_as_float(v.w));
  }
  return true;
}

// Shared memory of the sweep for cases of up to `nj` rows, chunks of `chunk`
// diagonals and `buffers` chunk buffers per warp: the header, two rings per
// warp edge and the warps' chunk buffers (a warp of `rows` rows holds
// rows + 1 record rows per diagonal).
__host__ __device__ inline size_t sweep_smem_bytes(int nj, int chunk, int buffers) {
  const int nw = sweep_warps(nj);
  const size_t rows_sum = size_t(nj) + nw;
  return kSweepHeader + 2 * size_t(nw - 1) * kEdgeRing * 16 + size_t(buffers) * chunk * rows_sum * 16 * REC_SIZE;
}

// The d-independent part of a neighbour's term: its state, the face normal
// (signed for the direction the flux leaves), A/2, omega lambda A/2, its
// normal velocity and the momentum and kinetic-energy weights of dK.
struct NeighbourTerm {
  float4 q;
  float nx, ny, half_area, damp, un, ku, kv, kk, p;
};

__device__ __forceinline__ NeighbourTerm neighbour_term(const float4 q, const float4 w, const float4 f,
                                                        float sgn) {
  NeighbourTerm t;
  t.q = q;
  t.nx = sgn * f.x;
  t.ny = sgn * f.y;
  t.half_area = f.z;
  t.damp = f.w;
  t.un = w.x * t.nx + w.y * t.ny;
  t.ku = q.x * w.x;
  t.kv = q.x * w.y;
  t.kk = q.x * (0.5f * (w.x * w.x + w.y * w.y));
  t.p = w.z;
  return t;
}

// The neighbour term of src/engine-cpu/euler2d.ts:977-1005 - the change of
// the physical flux across the face, F(Q + d) - F(Q), times A/2, less
// omega lambda A/2 d - added to `sum`. The exact difference is written so
// that every term is proportional to d (no difference of two O(|F|)
// numbers), so FP32 rounding is relative to the term and d = 0 adds exactly
// nothing, which stands for an absent neighbour.
__device__ __forceinline__ void add_neighbour(float4& sum, const NeighbourTerm& t, const float4 d,
                                              float gm1) {
  const float inv1 = approx_rcp(t.q.x + d.x);
  const float dmn = d.y * t.nx + d.z * t.ny;
  const float dun = (dmn - t.un * d.x) * inv1;
  const float dk = (t.ku * d.y + t.kv * d.z - t.kk * d.x + 0.5f * (d.y * d.y + d.z * d.z)) * inv1;
  const float dp = gm1 * (d.w - dk);
  sum.x += t.half_area * dmn - t.damp * d.x;
  sum.y += t.half_area * (d.y * t.un + (t.q.y + d.y) * dun + dp * t.nx) - t.damp * d.y;
  sum.z += t.half_area * (d.z * t.un + (t.q.z + d.z) * dun + dp * t.ny) - t.damp * d.z;
  sum.w += t.half_area * ((d.w + dp) * t.un + (t.q.w + d.w + t.p + dp) * dun) - t.damp * d.w;
}

__device__ __forceinline__ float4 shfl4_up(float4 v) {
  return make_float4(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1),
                     __shfl_up_sync(0xffffffffu, v.z, 1), __shfl_up_sync(0xffffffffu, v.w, 1));
}
__device__ __forceinline__ float4 shfl4_down(float4 v) {
  return make_float4(__shfl_down_sync(0xffffffffu, v.x, 1), __shfl_down_sync(0xffffffffu, v.y, 1),
                     __shfl_down_sync(0xffffffffu, v.z, 1), __shfl_down_sync(0xffffffffu, v.w, 1));
}

// The forward and backward sweeps of every active case, one CTA per case and
// one warp per 32 rows, leaving the final correction dQ in A.dq (row-major).
//
// Indexing: a warp of `rows` rows owns a block of records of nT = ni + rows
// diagonals by rows + 1 record rows (sweep_block_slot). Each pass visits the
// block's diagonals in the order of a pass index u = 0 .. nT - 1 (forward:
// the block diagonal; backward: nT - 1 less it); step s = 0 .. nT - 2 works on
// the lane's cell at u = s + 1, whose neighbours are at u = s. Chunk cc of a
// pass holds u in [cc K, cc K + K); the pass's chunks are numbered on from the
// previous pass's (g = pass nch + cc) and cycle through the warp's buffers.
static __global__ void __launch_bounds__(32 * kMaxSweepWarps) lusgs_sweep_kernel(const SweepArgs A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int c = A.case_list[blockIdx.x];
  if (A.active != nullptr && A.active[c] == 0) return;
  const CaseDev& cd = A.cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int nw = sweep_warps(nj);
  const int w = threadIdx.x >> 5;
  const int l = threadIdx.x & 31;
  const int K = A.chunk, NB = A.buffers;
  const float gm1 = float(cd.gamma) - 1.f;

  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);  // [kMaxSweepWarps][kMaxSweepBuffers]
  int* abort_word = reinterpret_cast<int*>(smem_raw + 8 * kMaxSweepWarps * kMaxSweepBuffers);
  float4* rings = reinterpret_cast<float4*>(smem_raw + kSweepHeader);  // [2][nw - 1][kEdgeRing]
  float4* bufs = rings + 2 * (nw - 1) * kEdgeRing;
  const int n_ring_words = 2 * (nw - 1) * kEdgeRing;
  for (int k = threadIdx.x; k < n_ring_words; k += blockDim.x)
    sts_volatile_u4(rings + k, make_uint4(kEdgeEmpty, kEdgeEmpty, kEdgeEmpty, kEdgeEmpty));
  if (threadIdx.x == 0) {
    *abort_word = 0;
    for (int b = 0; b < kMaxSweepWarps * kMaxSweepBuffers; b++) mbar_init(&bars[b], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (w >= nw) return;

  const int rows = sweep_rows(nj, w);
  const int R1 = rows + 1;
  const int nT = ni + rows;
  const int nch = (nT + K - 1) / K;
  const int le = min(l, rows - 1);  // the lane's row for addressing (lanes past the rows idle)
  uint64_t* full = bars + w * kMaxSweepBuffers;
  // This warp's chunk buffers: the warps before it hold rows' + 1 rows each.
  float4* wbuf = bufs + size_t(NB) * K * REC_SIZE * (size_t(32 * w) + w);
  const size_t buf_stride = size_t(K) * R1 * REC_SIZE;
  float4* ring_f_in = w > 0 ? rings + (w - 1) * kEdgeRing : nullptr;            // from warp w - 1
  float4* ring_f_out = w < nw - 1 ? rings + w * kEdgeRing : nullptr;            // to warp w + 1
  float4* ring_b_in = w < nw - 1 ? rings + (nw - 1 + w) * kEdgeRing : nullptr;  // from warp w + 1
  float4* ring_b_out = w > 0 ? rings + (nw - 1 + w - 1) * kEdgeRing : nullptr;  // to warp w - 1
  const int64_t block = cd.slot + sweep_block_base(ni, w);

  // Copies: chunk g of the sequence (forward chunks, then backward ones).
  auto chunk_span = [&](int cc, int& u0, int& n) {
    u0 = cc * K;
    n = min(K, nT - u0);
  };
  auto issue = [&](int g) {
    const int pass = g / nch, cc = g - pass * nch;
    int u0, n;
    chunk_span(cc, u0, n);
    const int t_lo = pass == 0 ? u0 : nT - u0 - n;  // block diagonal of the chunk's first slot row
    const float4* src = (pass == 0 ? A.rec_f : A.rec_b) + REC_SIZE * (block + int64_t(t_lo) * R1);
    const unsigned bytes = unsigned(n) * unsigned(R1) * 16u * REC_SIZE;
    if (l == 0) {
      uint64_t* bar = &full[g % NB];
      mbar_arrive_expect_tx(bar, bytes);
      bulk_load(wbuf + size_t(g % NB) * buf_stride, src, bytes, bar);
    }
  };
  int next = 0;      // next chunk to issue
  int released = 0;  // chunks whose buffers are free again
  int waited = 0;    // chunks waited for
  bool fwd_done = false;
  auto try_issue = [&]() {
    while (next < 2 * nch && next < released + NB && (next < nch || fwd_done)) issue(next++);
  };
  bool failed = false;
  auto wait_chunk = [&](int g) -> bool {
    const bool ok = mbar_wait(&full[g % NB], unsigned(g / NB) & 1u, A.wait_limit);
    if (ok) waited = g + 1;
    return __all_sync(0xffffffffu, ok);
  };
  try_issue();

  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  const int j = 32 * w + le;
  // One pass, its direction a compile-time constant. Steps go chunk by chunk
  // (the chunk holding the lane's own diagonal u = s + 1), so a step needs
  // no division: the neighbours' diagonal u - 1 is the element before (or,
  // at a chunk's first step, the previous chunk's last; forward elements run
  // up a buffer, backward ones down it).
  auto run_pass = [&](auto direction) -> bool {
    constexpr bool fwd = decltype(direction)::value;
    constexpr int pass = fwd ? 0 : 1;
    constexpr float sgn = fwd ? -1.f : 1.f;
    // Block rows: forward, own row l + 1 and the neighbour below at l (row 0
    // is the ghost of the previous warp's last row); backward, own row l and
    // the neighbour above at l + 1 (row `rows` is the ghost of the next
    // warp's first row).
    const int r_own = fwd ? le + 1 : le;
    const int r_nb = fwd ? le : le + 1;
    float4* ring_in = fwd ? ring_f_in : ring_b_in;
    float4* ring_out = fwd ? ring_f_out : ring_b_out;
    const bool edge_in_lane = fwd ? l == 0 : l == 31;
    const bool edge_out_lane = fwd ? l == 31 : l == 0;
    if (!wait_chunk(pass * nch)) return false;
    // The lane's previous cell (its neighbour along the row): state and dQ.
    float4 pq = make_float4(1.f, 0.f, 0.f, 1.f), pw = make_float4(0.f, 0.f, 1.f, 1.f), pd = zero;
    const float4* prev = nullptr;
    for (int cc = 0; cc < nch; cc++) {
      if (cc > 0 && !wait_chunk(pass * nch + cc)) return false;
      const int u0 = cc * K, n = min(K, nT - u0);
      const float4* cur = wbuf + size_t((pass * nch + cc) % NB) * buf_stride;
      for (int u = max(1, u0); u < u0 + n; u++) {
        const int s = u - 1;
        const int e = fwd ? u - u0 : u0 + n - 1 - u;
        const int i = fwd ? s - l : nT - 2 - s - l;
        const bool active = (l < rows) & (i >= 0) & (i < ni);
        const float4* own = cur + size_t(e * R1 + r_own) * REC_SIZE;
        const float4* nb = u > u0 ? cur + size_t((fwd ? e - 1 : e + 1) * R1 + r_nb) * REC_SIZE
                                  : prev + size_t((fwd ? K - 1 : 0) * R1 + r_nb) * REC_SIZE;
        const float4 base = own[REC_R], q = own[REC_Q], wv = own[REC_W], fa = own[REC_FA], fb = own[REC_FB];
        const float4 nq = nb[REC_Q], nwv = nb[REC_W];
        // dQ of the neighbour across rows, finished by the next lane on the
        // previous step, or, for the edge lane, by the other warp: taken from
        // the ring when that lane's cell is on the grid (a warp-uniform test).
        float4 dn = fwd ? shfl4_up(pd) : shfl4_down(pd);
        dn = edge_in_lane ? zero : dn;
        const int i_in = fwd ? s : nT - 2 - s - 31;    // the edge-in lane's column
        const int i_out = fwd ? s - 31 : nT - 2 - s;   // the edge-out lane's column
        bool ok = true;
        if (ring_in != nullptr && i_in >= 0 && i_in < ni)
          ok = warp_edge_get(ring_in, i_in, dn, edge_in_lane, A.wait_limit, abort_word);
        float4 sum = zero;
        add_neighbour(sum, neighbour_term(pq, pw, fa, sgn), pd, gm1);
        add_neighbour(sum, neighbour_term(nq, nwv, fb, sgn), dn, gm1);
        const float inv_d = wv.w;
        float4 dq;
        if (fwd) {
          dq = make_float4((base.x - sum.x) * inv_d, (base.y - sum.y) * inv_d, (base.z - sum.z) * inv_d,
                           (base.w - sum.w) * inv_d);
        } else {
          dq = make_float4(base.x - sum.x * inv_d, base.y - sum.y * inv_d, base.z - sum.z * inv_d,
                           base.w - sum.w * inv_d);
        }
        if (active) {
          if (fwd)
            A.rec_b[REC_SIZE * (block + int64_t(i + le) * R1 + le) + REC_R] = dq;
          else
            A.dq[cd.cell + i + int64_t(j) * ni] = dq;
        }
        if (ok && ring_out != nullptr && i_out >= 0 && i_out < ni)
          ok = warp_edge_put(ring_out, i_out, dq, edge_out_lane, A.wait_limit, abort_word);
        pq = active ? q : pq;
        pw = active ? wv : pw;
        pd = active ? dq : pd;
        if (!ok) return false;  // the same in every lane
        // The neighbours' diagonal u - 1 was the last of the previous chunk:
        // free it, once every lane's reads of it are ordered before the copy
        // that overwrites it.
        if (u == u0) {
          __syncwarp();
          released = pass * nch + cc;
          try_issue();
        }
      }
      prev = cur;
    }
    released = pass * nch + nch;
    if (fwd) {
      // dQ* written above is read by the backward pass's bulk copies.
      fence_proxy_async();
      __syncwarp();
      fwd_done = true;
    }
    try_issue();
    return true;
  };
  failed = !run_pass(std::true_type{}) || !run_pass(std::false_type{});
  if (failed) {
    if (l == 0) {
      atomicExch(abort_word, 1);
      atomicOr(&A.status[c], STATUS_TIMEOUT);
    }
    // Let this warp's copies still in flight land (bounded) before leaving.
    for (int g = waited; g < next; g++) mbar_wait(&full[g % NB], unsigned(g / NB) & 1u, A.drain_limit);
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

// Launch shape of the sweep: diagonals per bulk copy and chunk buffers per
// warp.
struct SweepShape {
  int chunk = 0, buffers = 0;
};

// The shape for cases of up to `nj` rows when `cases_in_flight` cases sweep
// at once: within the shared memory each CTA may take (the resident cases,
// up to 8 per SM, share an SM's), the one whose copies run furthest ahead of
// the diagonal being swept ((buffers - 1) chunk - 1 diagonals), the smaller
// footprint on a tie; chunks of up to `max_chunk` diagonals.
inline SweepShape sweep_shape(int nj, int cases_in_flight, int max_chunk = 8) {
  const int per_sm = std::min(8, std::max(1, (cases_in_flight + 147) / 148));
  for (size_t budget : {size_t(200 * 1024) / per_sm, size_t(200 * 1024)}) {
    SweepShape best;
    int best_lead = -1;
    size_t best_bytes = 0;
    for (int nb = 2; nb <= kMaxSweepBuffers; nb++)
      for (int k = 1; k <= max_chunk; k++) {
        const size_t bytes = sweep_smem_bytes(nj, k, nb);
        if (bytes > budget) continue;
        const int lead = (nb - 1) * k - 1;
        if (lead > best_lead || (lead == best_lead && bytes < best_bytes)) {
          best = {k, nb};
          best_lead = lead;
          best_bytes = bytes;
        }
      }
    if (best.chunk > 0) return best;
  }
  return {};
}

constexpr int kSweepWaitLimit = 1 << 22;

// `cases_in_flight`: cases of the whole batch sweeping at the same time
// (other lanes included), which sets the shared memory each CTA may take.
// `wait_limit` < 0 keeps the default bound.
inline cudaError_t launch_sweep(SweepArgs A, int n_cases, int max_nj, int cases_in_flight,
                                cudaStream_t stream, int wait_limit = -1, int max_chunk = 8) {
  const int nw = sweep_warps(max_nj);
  if (nw > kMaxSweepWarps) return cudaErrorInvalidConfiguration;
  const SweepShape shape = sweep_shape(max_nj, cases_in_flight, max_chunk);
  if (shape.chunk == 0) return cudaErrorInvalidConfiguration;
  A.chunk = shape.chunk;
  A.buffers = shape.buffers;
  A.wait_limit = wait_limit < 0 ? kSweepWaitLimit : wait_limit;
  A.drain_limit = kSweepWaitLimit;
  const size_t bytes = sweep_smem_bytes(max_nj, shape.chunk, shape.buffers);
  const cudaError_t e = cudaFuncSetAttribute(lusgs_sweep_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (e != cudaSuccess) return e;
  lusgs_sweep_kernel<<<n_cases, 32 * nw, bytes, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace bsd
