// legalize.cuh -- exact greedy legaliser on the GPU (defined in legalize.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace eplace {

struct LegalArgs {
  const float2 *pos;       // [N] clamped continuous positions
  const uint32_t *order;   // [n_order] macros first (sizes in msize), then unit cells
  const uchar2 *msize;     // [n_macro] footprint (w, h) of order[0 .. n_macro)
  uint32_t n_order, n_macro;
  const uint64_t *free0;   // [H * WR] free map with the fixed cells bound (bit set = free)
  uint64_t *work;          // [H * WR + H] map + row summaries when they exceed shared memory
  int W, H, WR;
  int2 *sites;             // [N] anchor site of every cell
  int2 *loc;               // [N] pin location (anchor + (size - 1) / 2), or nullptr
  double *cost;            // [n_order] cost of each placement, in order (summed at the end)
  double *disp;            // [1] total displacement (sequential FP64 sum in order)
  int *status;             // [1] 0 = ok, 1 = no free site for some cell
};

// Shared memory the map of a W-site-wide, H-row chip needs (map + one
// 64-bit summary word per row).
size_t legalize_smem_bytes(int WR, int H);
// Chips wider than 64 words per row are not supported (host legaliser).
bool legalize_supported(int W, int H);
constexpr size_t kLegalMaxSmem = 160 * 1024;

// One CTA of one warp per legalisation; several run concurrently on
// separate streams.
cudaError_t launch_legalize(const LegalArgs &a, cudaStream_t s);

}  // namespace eplace
