// init_place.cuh -- the reference's initial placement on the device.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace eplace {

// Draws per thread of the draw kernel; the jump maps are powers of the
// generator step by multiples of it.
constexpr uint32_t kIpSeg = 64;
// Jump maps T^(kIpSeg * 2^m), m = 0 .. kIpJumps - 1, 64 words each: enough
// for 2^kIpJumps * kIpSeg draws (more than any grid the context takes).
constexpr int kIpJumps = 26;

// The jump maps (host-built once per process; see init_place.cu).
const std::vector<uint64_t> &ip_jump_maps();

// Device buffers of one initial placement (sizes in elements).
struct IpBuffers {
  uint32_t *j;        // [n]   j of Fisher-Yates step i (index i)
  uint32_t *cnt;      // [n + 1] steps aimed at each position, then fill cursors
  uint32_t *start;    // [n + 1] exclusive prefix of cnt: position p's steps are entries[start[p], start[p+1])
  uint32_t *entries;  // [n]     steps grouped by target position
  uint32_t *block;    // [(n + 1) / 1024 + 1] scan block totals
  const uint64_t *jump;  // [kIpJumps * 64] jump maps
  const uint32_t *occupied;  // [n_occ] sorted sites taken before the shuffle (fixed logic, pre-bound)
  uint32_t n_occ;
  const uint32_t *unbound;  // [n_unbound] cell ids handed a BEL, in order; nullptr: cells 0 .. n_unbound-1
  uint32_t n_unbound;
  int32_t W;
  int2 *site;   // [N] output: BEL (x, y) of each handed-out cell
  float2 *x, *xp, *look;  // [N] outputs: the same positions as floats (may be nullptr)
};

// Runs the shuffle of the n available BELs with the reference's generator
// and hands the first n_unbound of them out, on stream s (asynchronous).
cudaError_t launch_initial_placement(const IpBuffers &b, uint64_t seed, uint32_t n, cudaStream_t s);

}  // namespace eplace
