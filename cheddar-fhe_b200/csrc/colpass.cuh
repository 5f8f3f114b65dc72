// Tile geometry shared by the two column-pass kernels of ModUp / ModDown
// (modswitch.cu on the CUDA cores, modswitch_tc.cu with the base conversion
// on the tensor cores): a CTA of 128 threads owns 16 columns of the
// 128 x 512 limb layout; thread t holds rows rg + 8e (e = 0..15) of column
// cl, rg = 2 (t / 32) + (t % 32) / 16, cl = t % 16.  A warp's loads and
// stores cover two rows of 16 consecutive columns (two 64-byte segments).
#pragma once

namespace chd {

constexpr int kTC = 16;          // columns per tile
constexpr int kExRows = 136;     // 128 rows + one padding row per 16 rows

// exchange-buffer index: a 16-word gap every 16 rows keeps both access
// patterns (rows rg + 8k and rows 8j + u) free of bank conflicts
__device__ __forceinline__ int exi(int row, int col) { return (row + (row >> 4)) * kTC + col; }

}  // namespace chd
