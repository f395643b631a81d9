// Host side of the TMA staging: tensor maps encoded through the driver's
// cuTensorMapEncodeTiled, reached with cudaGetDriverEntryPoint (no link against libcuda).
#include <cudaTypedefs.h>
#include <mutex>
#include "mdg_tma.cuh"

namespace mdg {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}
}  // namespace

bool tma_encode_2d_f64(CUtensorMap *m, const void *base, uint64_t cols, uint64_t rows, uint64_t row_bytes,
                       uint32_t box_cols, uint32_t box_rows, std::string *why)
{
  auto bad = [&](const char *w) {
    if (why) *why = w;
    return false;
  };
  if (!m || !base) return bad("tma: null map or table");
  if (reinterpret_cast<uintptr_t>(base) % 16 != 0) return bad("tma: table base not 16-byte aligned");
  if (row_bytes % 16 != 0 || row_bytes < cols * sizeof(double)) return bad("tma: row stride");
  if (box_cols == 0 || box_rows == 0 || box_cols > 256 || box_rows > 256 || (box_cols * sizeof(double)) % 16 != 0)
    return bad("tma: box shape");
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (!fn) return bad("tma: cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {row_bytes};
  const cuuint32_t box[2] = {box_cols, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void *>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return bad("tma: cuTensorMapEncodeTiled failed");
  return true;
}

}  // namespace mdg
