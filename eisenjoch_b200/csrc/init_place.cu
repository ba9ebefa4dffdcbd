// init_place.cu -- the reference's initial placement (placer/common.rs:27-117)
// on the device: the free logic BELs (tile order) are shuffled with the
// reference's generator (xorshift64, Fisher-Yates from the end with
// j = (u32)draw % (i + 1), context/rng.rs:19-61) and handed out in order to
// the unbound cells.  The shuffle is sequential as written; here it is
// reformulated so that every handed-out position is found independently,
// giving the same permutation bit for bit:
//
//  * the draws: xorshift64 is linear over GF(2), so thread g starts from
//    T^(g * kIpSeg)(seed), built from the maps T^(kIpSeg * 2^m), and makes
//    its kIpSeg draws; draw k belongs to step i = n - k;
//  * where a final position's element came from: undoing the swaps in
//    reverse order, the element at final position q came from j_q
//    (q >= 1; position 0 starts from 0) and is then carried up to step i
//    whenever a later step i swaps with the position it sits at: while some
//    step i > t has j_i = p, the element sat at p before step i and at i
//    after it (p, t <- i, i for the first such i); the element's start is
//    the last p.  Steps are grouped by j (counting sort) so each lookup
//    scans one short group (about ln(n / p) steps aim at position p).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "init_place.cuh"

namespace eplace {
namespace {

__host__ __device__ __forceinline__ uint64_t xs_step(uint64_t s) {
  s ^= s << 13;
  s ^= s >> 7;
  s ^= s << 17;
  return s;
}

// A GF(2)-linear map of 64-bit words as the images of the unit vectors.
__host__ __device__ __forceinline__ uint64_t gf2_apply(const uint64_t *m, uint64_t v) {
  uint64_t r = 0;
  while (v) {
#ifdef __CUDA_ARCH__
    r ^= m[__ffsll((long long)v) - 1];
#else
    r ^= m[__builtin_ctzll(v)];
#endif
    v &= v - 1;
  }
  return r;
}

void gf2_compose(const uint64_t *a, const uint64_t *b, uint64_t *out) {  // a after b
  uint64_t r[64];
  for (int k = 0; k < 64; ++k) r[k] = gf2_apply(a, b[k]);
  for (int k = 0; k < 64; ++k) out[k] = r[k];
}

// Thread g: its kIpSeg draws, each reduced to the j of its step.
__global__ void k_ip_draws(uint64_t seed, const uint64_t *jump, uint32_t n, uint32_t *j) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t k0 = (uint64_t)g * kIpSeg;
  if (k0 + 1 >= n) return;
  uint64_t s = seed;
  for (int m = 0; m < kIpJumps && (g >> m); ++m)
    if ((g >> m) & 1u) s = gf2_apply(jump + 64 * m, s);
  for (uint32_t r = 1; r <= kIpSeg; ++r) {
    const uint64_t k = k0 + r;  // draw number
    if (k >= n) break;
    s = xs_step(s);
    const uint32_t i = (uint32_t)(n - k);  // its Fisher-Yates step
    j[i] = (uint32_t)s % (i + 1u);
  }
}

__global__ void k_ip_count(const uint32_t *j, uint32_t n, uint32_t *cnt) {
  for (uint32_t i = 1 + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(&cnt[j[i]], 1u);
}

// Exclusive scan of cnt[0, n) into start, 1024 elements per block; block
// totals into block[].
__global__ void __launch_bounds__(1024) k_ip_scan_blocks(const uint32_t *cnt, uint32_t n, uint32_t *start,
                                                         uint32_t *block) {
  __shared__ uint32_t warp_tot[32];
  const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
  const uint32_t v = i < n ? cnt[i] : 0u;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  const uint32_t before = (w ? warp_tot[w - 1] : 0u) + x - v;
  if (i < n) start[i] = before;
  if (threadIdx.x == 1023) block[blockIdx.x] = warp_tot[31];
}

// Exclusive scan of the nb block totals in place (one block).
__global__ void __launch_bounds__(1024) k_ip_scan_top(uint32_t *block, uint32_t nb) {
  __shared__ uint32_t part[1024];
  const uint32_t per = (nb + 1023) / 1024, b0 = threadIdx.x * per;
  uint32_t sum = 0;
  for (uint32_t k = 0; k < per && b0 + k < nb; ++k) sum += block[b0 + k];
  part[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int k = 0; k < 1024; ++k) {
      const uint32_t t = part[k];
      part[k] = run;
      run += t;
    }
  }
  __syncthreads();
  uint32_t run = part[threadIdx.x];
  for (uint32_t k = 0; k < per && b0 + k < nb; ++k) {
    const uint32_t t = block[b0 + k];
    block[b0 + k] = run;
    run += t;
  }
}

__global__ void k_ip_scan_add(uint32_t *start, uint32_t n, const uint32_t *block) {
  const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
  if (i < n) start[i] += block[blockIdx.x];
}

__global__ void k_ip_fill(const uint32_t *j, uint32_t n, const uint32_t *start, uint32_t *cursor,
                          uint32_t *entries) {
  for (uint32_t i = 1 + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = j[i];
    entries[start[p] + atomicAdd(&cursor[p], 1u)] = i;
  }
}

// The k-th free site (tile order) given the sorted taken sites: the least t
// with t - |{o <= t}| = k (it is free: were t taken, t - 1 would do).
__device__ __forceinline__ uint32_t free_site(uint32_t k, const uint32_t *occ, uint32_t n_occ) {
  if (n_occ == 0) return k;
  uint32_t lo = k, hi = k + n_occ;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    uint32_t a = 0, b = n_occ;  // occupied sites <= mid
    while (a < b) {
      const uint32_t c = a + (b - a) / 2;
      if (occ[c] <= mid) a = c + 1;
      else b = c;
    }
    if (mid - a >= k) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// The q-th handed-out BEL: follow its element back to its start.  Each step
// of the walk moves t strictly up (t < n), so the walk ends.
__global__ void k_ip_chase(const uint32_t *j, const uint32_t *start, const uint32_t *entries, IpBuffers b) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= b.n_unbound) return;
  uint32_t p = q ? j[q] : 0u, t = q;
  while (true) {
    uint32_t nxt = 0xffffffffu;
    const uint32_t e0 = start[p], e1 = start[p + 1];
    for (uint32_t e = e0; e < e1; ++e) {
      const uint32_t i = entries[e];
      if (i > t && i < nxt) nxt = i;
    }
    if (nxt == 0xffffffffu) break;
    p = nxt;
    t = nxt;
  }
  const uint32_t site = free_site(p, b.occupied, b.n_occ);
  const uint32_t cell = b.unbound ? b.unbound[q] : q;
  const int2 xy = make_int2((int32_t)(site % (uint32_t)b.W), (int32_t)(site / (uint32_t)b.W));
  b.site[cell] = xy;
  const float2 f = make_float2((float)xy.x, (float)xy.y);
  if (b.x) b.x[cell] = f;
  if (b.xp) b.xp[cell] = f;
  if (b.look) b.look[cell] = f;
}

}  // namespace

const std::vector<uint64_t> &ip_jump_maps() {
  static std::vector<uint64_t> maps;
  static std::once_flag once;
  std::call_once(once, [] {
    uint64_t t[64], acc[64];
    for (int k = 0; k < 64; ++k) {
      t[k] = xs_step(1ull << k);
      acc[k] = 1ull << k;
    }
    for (uint32_t e = kIpSeg; e; e >>= 1) {  // acc = T^kIpSeg
      if (e & 1) gf2_compose(t, acc, acc);
      gf2_compose(t, t, t);
    }
    maps.resize(64 * (size_t)kIpJumps);
    for (int m = 0; m < kIpJumps; ++m) {
      for (int k = 0; k < 64; ++k) maps[64 * m + k] = acc[k];
      gf2_compose(acc, acc, acc);
    }
  });
  return maps;
}

cudaError_t launch_initial_placement(const IpBuffers &b, uint64_t seed, uint32_t n, cudaStream_t s) {
  if (n == 0 || b.n_unbound == 0) return cudaSuccess;
  cudaError_t e;
  // counts of the steps aimed at each position (cnt[n] stays 0), their
  // exclusive prefix (start[p] .. start[p + 1] is position p's group)
  if ((e = cudaMemsetAsync(b.cnt, 0, sizeof(uint32_t) * ((size_t)n + 1), s)) != cudaSuccess) return e;
  const int grid_n = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  if (n > 1) {
    const uint32_t threads = (n - 2) / kIpSeg + 1;  // draws 1 .. n - 1
    k_ip_draws<<<(threads + 255) / 256, 256, 0, s>>>(seed, b.jump, n, b.j);
    k_ip_count<<<grid_n, 256, 0, s>>>(b.j, n, b.cnt);
  }
  const uint32_t m = n + 1, nb = (m + 1023) / 1024;
  k_ip_scan_blocks<<<nb, 1024, 0, s>>>(b.cnt, m, b.start, b.block);
  k_ip_scan_top<<<1, 1024, 0, s>>>(b.block, nb);
  k_ip_scan_add<<<nb, 1024, 0, s>>>(b.start, m, b.block);
  if (n > 1) {
    // the counts again, as fill cursors
    if ((e = cudaMemsetAsync(b.cnt, 0, sizeof(uint32_t) * n, s)) != cudaSuccess) return e;
    k_ip_fill<<<grid_n, 256, 0, s>>>(b.j, n, b.start, b.cnt, b.entries);
  }
  k_ip_chase<<<(b.n_unbound + 255) / 256, 256, 0, s>>>(b.j, b.start, b.entries, b);
  return cudaGetLastError();
}

}  // namespace eplace
