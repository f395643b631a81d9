// Tensor-memory-accelerator (TMA) staging of table tiles into shared memory, sm_100a.
//
// A kernel that stages a tile issues one cp.async.bulk.tensor load per table from one
// thread, the copies complete on an mbarrier in shared memory, and every thread waits on
// that barrier.  Loads only, of this GPU's own memory, without cluster multicast.
//
// Rules the callers keep (checked on the host where the map is encoded):
//   - the table's base address is 16-byte aligned and its row stride a multiple of
//     16 bytes (tables are padded to an even number of FP64 columns);
//   - the innermost start coordinate x of a load is a multiple of 2 FP64 elements (16
//     bytes): callers round the first column down to even and index from the remainder;
//   - the box's inner extent is an even number of FP64 elements, at most 256 per dim;
//   - the destination in shared memory is 128-byte aligned.
// Waits are bounded: a barrier that has not completed after about a second of clock
// cycles reports failure and the caller flags its problem instead of spinning on.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

namespace mdg {

// Tile maps of the 1-D FP64 sweep: the reconstruction table (all RC_NFIELDS rows) and the
// face/zone geometry table (rows 0..GF_TMA_ROWS-1 of GF_NFIELDS), each box TMA_COLS1
// columns wide.  valid = 0: no maps (the kernel reads the tables directly).
struct TmaTables1d {
  CUtensorMap rc;
  CUtensorMap geo;
  int valid;
};
constexpr int TMA_COLS1 = 130;      // columns of a 1-D tile box: 128 (+1 for a rounded-down start)
constexpr int RC_TMA_ROWS = 22;     // every reconstruction field (para_recon and lin_recon)
constexpr int GF_TMA_ROWS = 13;     // GF_AREA .. GF_S00: face and zone geometry, without conn

// Encode a 2-D FP64 tile map over a row-major table of `rows` rows of `cols` elements
// (row stride row_bytes), boxes of box_cols x box_rows.  Returns false with a reason when
// the driver entry point is missing or an alignment rule is broken.
bool tma_encode_2d_f64(CUtensorMap *m, const void *base, uint64_t cols, uint64_t rows, uint64_t row_bytes,
                       uint32_t box_cols, uint32_t box_rows, std::string *why);

#ifdef __CUDACC__
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// Arrive on the barrier announcing tx_bytes of asynchronous copies to come.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned tx_bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(tx_bytes)
               : "memory");
}

// Wait for phase `phase` of the barrier to complete; false after about max_cycles
// clock cycles without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase, long long max_cycles = 2000000000LL)
{
  const long long t0 = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > max_cycles) return false;
  }
}

// 2-D tile load (x: column, y: row of the box's first element) into shared memory,
// completing on bar.  No cluster multicast.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
#endif

}  // namespace mdg
