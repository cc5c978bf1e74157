// Tensor-memory-accelerator (TMA) tiled loads for the image kernels: host-side
// tensor-map encoding of an NHWC image and the device-side copy into shared
// memory completing on an mbarrier.  Loads only, never multicast.
//
// An image [B, H, W, C] of 4- or 1-byte elements is described as the 3-D
// tensor (C*W, H, B): a box of (bx elements, by rows, 1 image) lands in shared
// memory row by row, bx elements per row.  Requirements checked by
// encode_image(): the base address 16-byte aligned and the row stride C*W*e a
// multiple of 16 bytes; the box's inner extent bx*e a multiple of 16 bytes.
// The inner coordinate of every copy must be a multiple of 16 bytes / e
// (callers round it down); rows and columns outside the image are filled
// with zeros, so callers decide in-image membership themselves.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "tc_sm100.cuh"

namespace cd {
namespace tma {

// Process-wide choice between the persistent TMA-staged kernels and the
// tile-per-CTA kernels for the ops that have both (same results); on by
// default, set by cd_set_persistent_kernels.
bool persistent_enabled();
void set_persistent_enabled(bool on);

// Encodes the map; returns false when the driver entry point is missing or
// the image does not meet the alignment rules above.
bool encode_image(CUtensorMap *map, const void *base, bool bytes, int C, int W, int H, int B, int box_x,
                  int box_y);

__device__ __forceinline__ void load3(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(tc::smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(tc::smem_u32(bar))
        : "memory");
}

// Largest multiple of m (a power of two) not above v, for negative v too.
__host__ __device__ constexpr int floor_to(int v, int m) { return v >= 0 ? v & ~(m - 1) : -((-v + m - 1) & ~(m - 1)); }

}  // namespace tma
}  // namespace cd
