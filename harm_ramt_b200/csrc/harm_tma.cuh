// Tensor-memory-accelerator (TMA) staging of plane tiles into shared memory
// for the step kernels (sm_100a).
//
// A field block in HBM is a stack of planes of `pitch` doubles x `rows`
// rows (structure of arrays, x1 fastest).  A 3D tensor map over (x1 column,
// x2 row, plane) lets one thread of a block copy a box of
// (columns x rows x planes) into shared memory with one
// cp.async.bulk.tensor instruction; the copy completes on an mbarrier that
// the block's threads wait on.  Rules kept here:
//   * the map covers only this GPU's own buffers, and no load uses cluster
//     multicast;
//   * the innermost coordinate of every copy is even (x * 8 bytes a
//     multiple of 16), the base is 16-byte aligned and the strides are
//     multiples of 16 bytes (pitch is a multiple of 16 doubles);
//   * boxes may start at negative or past-the-end rows and columns: those
//     elements read as zero;
//   * every wait is bounded: a copy that has not landed after TMA_WAIT_LIMIT
//     polls is reported (harm_status.fail_code = FAIL_TMA_TIMEOUT) and the
//     kernel leaves the tile unused.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace harm {

// a copy that did not complete within the wait limit (no reference counterpart)
constexpr int FAIL_TMA_TIMEOUT = 31;
constexpr unsigned TMA_WAIT_LIMIT = 1u << 26;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  // make the initialised barrier visible to the asynchronous (TMA) proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// one 3D box {x, y, z} of the map into shared memory at dst, completing on bar
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar)
{
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// waits for phase `parity` of the barrier; false if it did not complete
// within TMA_WAIT_LIMIT polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
  const uint32_t a = smem_addr(bar);
  for (unsigned it = 0; it < TMA_WAIT_LIMIT; it++) {
    uint32_t done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// host: encodes the 3D tensor map of `nplanes` planes starting at `base`
// (pitch x rows doubles each, `plane` doubles apart), box {bx, by, bz};
// returns false when the driver refuses it (alignment, sizes)
bool tma_encode_planes(CUtensorMap* map, const double* base, int pitch, int rows, int nplanes, long long plane, int bx,
                       int by, int bz);

}  // namespace harm
