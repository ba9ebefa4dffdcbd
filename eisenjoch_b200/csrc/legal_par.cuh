// legal_par.cuh -- parallel exact greedy legaliser on the GPU (legal_par.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace eplace {

// Window capacity (cells per round) and candidate-list capacity per cell.
constexpr uint32_t kLpMaxWindow = 16384;
constexpr int kLpList = 64;
constexpr int kLpPropSteps = 16;  // disturbance propagation passes per round

// Round state, in device memory (one per legalisation in flight).
struct LpState {
  uint32_t pos;       // next order index to place
  uint32_t bcur;      // window size of the current round
  uint32_t stop;      // window cells committed this round
  uint32_t rounds;    // rounds run
  int32_t status;     // 0 ok, 1 no free site for some cell, 2 round cap, 3 tie group beyond the buffer
  uint32_t changed[kLpPropSteps + 1];  // propagation pass i found new disturbed cells
  uint32_t pad_;
};

struct LpArgs {
  const float2 *pos;       // [N] continuous positions (the checkpoint)
  const uint32_t *order;   // [n] legalisation order: macros first, then unit cells, solver order within each
  const uchar2 *fsize;     // [N] footprint (w, h) per cell id, or nullptr when every cell is 1x1
  uint32_t n;              // cells to place
  int W, H, WR;            // chip sites, 64-bit words per row
  const uint64_t *free0;   // [H * WR] free map with the fixed cells bound (bit set = free)
  uint64_t *fm;            // [H * WR] working free map
  int32_t *list;           // [kLpMaxWindow * kLpList] candidate anchors (tile = y * W + x), best first
  int32_t *len;            // [kLpMaxWindow] list lengths
  int32_t *info;           // [kLpMaxWindow] w | h << 8 of the window's cells (written with the lists)
  int32_t *hmark;          // [W * H] lowest window index whose head block covers the site (INT32_MAX: none)
  int32_t *dmark;          // [W * H] lowest disturbed window index whose list covers the site
  uint8_t *dist;           // [kLpMaxWindow] cell must take the serial pass
  uint8_t *fresh;          // [kLpMaxWindow] disturbed in the last pass, lists not marked yet
  int32_t *pick;           // [kLpMaxWindow] anchor chosen by the serial pass
  LpState *st;
  int2 *sites;             // [N] anchor of every cell (out)
  int2 *loc;               // [N] pin location anchor + (size - 1) / 2 (out), or nullptr
  double *cost;            // [n] cost of each placement, by order index (out)
  double *disp;            // [1] total displacement, summed in order (out)
  int32_t *status;         // [1] 0 ok, 1 no free site, else an internal limit (out)
  uint32_t max_rounds;
  cudaGraphConditionalHandle handle;
};

// Chips the device legaliser takes (tile ids and per-site marks sized by
// W x H): up to 4096 x 4096 sites.
inline bool legalize_supported(int W, int H) { return W > 0 && H > 0 && W <= 4096 && H <= 4096; }

// Device bytes of the round buffers (lists, marks, flags) for a W x H chip.
size_t lp_scratch_bytes(int W, int H);

// A legalisation as one CUDA graph: initialisation, a device-side while
// loop over rounds, the displacement sum.  Built once per slot and problem
// load; launched per checkpoint.
struct LpGraph {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  ~LpGraph();
};

// Builds the graph for args `a` (the handle field is filled in).
cudaError_t lp_build_graph(LpArgs a, LpGraph &g, cudaStream_t capture_stream);

}  // namespace eplace
