// The learned warm start's network on the tensor cores: tensor maps and
// launches of the tcgen05 GEMMs (device/umma.cuh), and their C entry points.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "bowshock.h"
#include "common.hpp"
#include "device/umma.cuh"

#define BS_TRY_ST(expr)              \
  do {                               \
    const bs_status s_ = (expr);     \
    if (s_ != BS_OK) return s_;      \
  } while (0)

namespace bsm {

using bsd::umma::kBK;
using bsd::umma::kBM;

// cuTensorMapEncodeTiled from the driver, found through the runtime (the
// library does not link the driver library itself).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// The tensor map of a row-major bf16 matrix (rows x cols, cols contiguous)
// read in tiles of box_rows x 64, 128-byte swizzled; rows past the end read
// as zero.
bs_status make_map(CUtensorMap* map, const void* ptr, int64_t rows, int64_t cols, int box_rows) {
  auto fn = encode_fn();
  if (fn == nullptr) return bs::fail(BS_EXECUTION, "cuTensorMapEncodeTiled is not available");
  if (cols % kBK != 0 || (reinterpret_cast<uintptr_t>(ptr) & 15) != 0)
    return bs::fail(BS_INVALID_ARGUMENT, "a GEMM operand needs 16-byte alignment and K a multiple of 64");
  const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(cols) * 2};
  const cuuint32_t box[2] = {cuuint32_t(kBK), cuuint32_t(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
                        elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return bs::fail(BS_EXECUTION, "cuTensorMapEncodeTiled failed: " + std::to_string(int(r)));
  return BS_OK;
}

// C (m x n) from A (m x k, map a) and B (n x k, map b) with epilogue `epi`,
// K split over `splits` CTAs per tile. n must be a multiple of BN and k of 64.
template <int BN, class Epi>
bs_status gemm(const CUtensorMap& a, const CUtensorMap& b, int m, int n, int k, int splits, const Epi& epi,
               int* error, cudaStream_t stream) {
  if (m <= 0 || n % BN != 0 || k % kBK != 0 || k <= 0 || splits < 1)
    return bs::fail(BS_INVALID_ARGUMENT, "GEMM shape: n a multiple of the tile, k of 64");
  constexpr size_t bytes = bsd::umma::gemm_smem_bytes<BN>();
  static_assert(bytes <= 227 * 1024, "GEMM shared memory");
  auto kernel = bsd::umma::gemm_bf16_tn<BN, Epi>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (e != cudaSuccess) return bs::fail(BS_EXECUTION, std::string("GEMM attribute: ") + cudaGetErrorString(e));
  const int k_chunks = k / kBK;
  const int per_split = (k_chunks + splits - 1) / splits;
  const dim3 grid((m + kBM - 1) / kBM, n / BN, (k_chunks + per_split - 1) / per_split);
  kernel<<<grid, bsd::umma::kThreads, bytes, stream>>>(a, b, m, per_split, k_chunks, epi, error);
  e = cudaGetLastError();
  if (e != cudaSuccess) return bs::fail(BS_EXECUTION, std::string("GEMM launch: ") + cudaGetErrorString(e));
  return BS_OK;
}

template <class Epi>
bs_status gemm_any(const void* a, const void* b, int m, int n, int k, int splits, const Epi& epi, int* error,
                   cudaStream_t stream) {
  const int bn = n % 256 == 0 ? 256 : n % 128 == 0 ? 128 : n % 64 == 0 ? 64 : 0;
  if (bn == 0) return bs::fail(BS_INVALID_ARGUMENT, "GEMM n must be a multiple of 64");
  CUtensorMap ma, mb;
  BS_TRY_ST(make_map(&ma, a, m, k, kBM));
  BS_TRY_ST(make_map(&mb, b, n, k, bn));
  if (bn == 256) return gemm<256>(ma, mb, m, n, k, splits, epi, error, stream);
  if (bn == 128) return gemm<128>(ma, mb, m, n, k, splits, epi, error, stream);
  return gemm<64>(ma, mb, m, n, k, splits, epi, error, stream);
}

}  // namespace bsm

extern "C" {

bs_status bs_gemm_bf16(const void* a, const void* b, float* c, int32_t m, int32_t n, int32_t k, int32_t splits,
                       int32_t accumulate, void* stream) {
  if (a == nullptr || b == nullptr || c == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null pointer");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* d_err = nullptr;
  // Test entry point: a small error word of its own.
  if (cudaMallocAsync(&d_err, sizeof(int), st) != cudaSuccess) return bs::fail(BS_MEMORY_LIMIT, "error word");
  cudaMemsetAsync(d_err, 0, sizeof(int), st);
  bs_status s;
  if (accumulate != 0)
    s = bsm::gemm_any(a, b, m, n, k, splits, bsd::umma::EpiAtomicF32{c, n}, d_err, st);
  else if (splits != 1)
    s = bs::fail(BS_INVALID_ARGUMENT, "split K needs accumulate");
  else
    s = bsm::gemm_any(a, b, m, n, k, 1, bsd::umma::EpiStoreF32{c, n}, d_err, st);
  int h_err = 0;
  cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d_err, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (s != BS_OK) return s;
  if (e != cudaSuccess) return bs::fail(BS_EXECUTION, std::string("GEMM: ") + cudaGetErrorString(e));
  if (h_err != 0) return bs::fail(BS_EXECUTION, "GEMM: a pipeline wait timed out");
  return BS_OK;
}

}  // extern "C"
