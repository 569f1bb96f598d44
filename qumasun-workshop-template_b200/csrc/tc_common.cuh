// Device helpers shared by the tcgen05 kernels (gram_tc.cu, gram_i8.cu):
// mbarrier waits with an iteration limit, 2-D TMA tile loads (no multicast),
// the shared-memory descriptor of a K-major 128-byte-swizzled tile, MMA
// completion commits and TMEM loads, plus the host-side tensor-map encoder.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace qsb {
namespace tc {

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// true when the phase with this parity completed within `limit` polls
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, unsigned limit) {
    for (unsigned i = 0; i < limit; ++i)
        if (bar_try(b, parity)) return true;
    return false;
}
// 2-D tile load into this CTA's shared memory, completion counted on barrier b
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(su32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(su32(b))
        : "memory");
}

// UMMA shared-memory descriptor of a K-major tile stored in 128-byte swizzle
// atoms (8 rows x 128 B): start address >> 4, leading offset 1 (unused for
// swizzled K-major), stride offset 1024 B >> 4 between 8-row groups, descriptor
// version 1, layout SWIZZLE_128B (2).  Advancing K inside the 128-byte row is
// adding the byte offset to the start address.
__device__ __forceinline__ uint64_t sw128_kmajor_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// barrier b gets one arrival once every MMA this thread issued before has completed
__device__ __forceinline__ void umma_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(b))
                 : "memory");
}

// 32 consecutive 32-bit TMEM columns of this warp's 32 lanes (one per thread)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Host: cuTensorMapEncodeTiled through the runtime's driver entry point.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled_fn();

// 2-D map over a K-major operand stored as [cols][ldk] elements of `elem_bytes`
// bytes, box (box_k elements, box_rows rows), 128-byte swizzle.
bool make_kmajor_map(CUtensorMap* map, CUtensorMapDataType dt, int elem_bytes, const void* base, int64_t ldk,
                     int cols, int box_k, int box_rows);

}  // namespace tc
}  // namespace qsb
