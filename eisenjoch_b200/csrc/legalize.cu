// legalize.cu -- the greedy legaliser of electro_place/mod.rs:206-255 on the
// GPU, with results identical to the reference's exhaustive scan
// (common.rs:294-374: cells in solver order, each onto the free site of
// minimum (bx - x)^2 + (by - y)^2 in FP64, strict '<' so the lowest tile wins
// ties).  Macros (w x h > 1, an extension) go first onto fully free blocks,
// cost measured at the block centre.
//
// The algorithm is sequential by definition.  One warp runs the sequence on
// one SM with the chip's free-site bitmap (one bit per site, 64-bit words,
// plus one summary word per row with a bit per non-empty word) in shared
// memory, or in L2 for chips whose map does not fit:
//  * batches of 32 consecutive unit cells: every lane finds its cell's
//    global-minimum site, the nearest integer point (two per axis only at an
//    exact k + 1/2).  If it is free it is the cell's answer unless an earlier
//    cell takes it first, so the longest prefix of lanes with free, distinct
//    candidates commits at once.  (Removing sites never changes the minimum
//    of a set that still contains it.)
//  * the first lane whose candidate is taken is placed by a warp-parallel
//    exact search: rows outward from the target, 32 rows per step (one per
//    lane), each row's best free site from bit scans (nearest free bit left
//    of or right of the target column, found through the row summary), a
//    warp arg-min over (cost, tile), stopping when the next rows' dy^2
//    exceeds the best cost (a row that far cannot win or tie);
//  * macros: anchor rows the same way, a valid anchor being one whose w x h
//    block is free (AND of the rows' words, AND of w shifted copies).
// Costs are formed with explicit round-to-nearest operations (no FMA
// contraction), so they equal the host's FP64 arithmetic bit for bit, and the
// total displacement is summed in cell order at the end.
#include <cuda_runtime.h>

#include <cstdint>

#include "legalize.cuh"

namespace eplace {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr long long kNoTile = 0x7fffffffffffffffll;

__device__ __forceinline__ double sq(double d) { return __dmul_rn(d, d); }

// lexicographic (cost, tile) minimum across the warp
__device__ __forceinline__ void warp_argmin(double &c, long long &t) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double oc = __shfl_xor_sync(kFull, c, o);
    const long long ot = __shfl_xor_sync(kFull, t, o);
    if (oc < c || (oc == c && ot < t)) {
      c = oc;
      t = ot;
    }
  }
}

// Free map: `fm` holds H rows of WR words, `sum` one word per row whose bit
// j is set while word j of the row has a free site.  Shared-memory maps use
// volatile loads; maps in global memory read through L2 (where the atomics
// of the same warp land).
template <bool kShared>
struct FreeMap {
  uint64_t *fm;
  uint64_t *sum;
  int WR;
  __device__ __forceinline__ uint64_t word(int row, int w) const {
    const uint64_t *p = fm + (size_t)row * WR + w;
    if (kShared) return *reinterpret_cast<const volatile uint64_t *>(p);
    return __ldcg(reinterpret_cast<const unsigned long long *>(p));
  }
  __device__ __forceinline__ uint64_t summary(int row) const {
    if (kShared) return *reinterpret_cast<const volatile uint64_t *>(sum + row);
    return __ldcg(reinterpret_cast<const unsigned long long *>(sum + row));
  }
  __device__ __forceinline__ bool is_free(int row, int x) const { return (word(row, x >> 6) >> (x & 63)) & 1ull; }
  __device__ __forceinline__ void take(int row, int x) const {
    const uint64_t bit = 1ull << (x & 63);
    const unsigned long long old =
        atomicAnd(reinterpret_cast<unsigned long long *>(fm + (size_t)row * WR + (x >> 6)), ~bit);
    if ((old & ~bit) == 0ull) atomicAnd(reinterpret_cast<unsigned long long *>(sum + row), ~(1ull << (x >> 6)));
  }
  // highest free x <= pos in the row, or -1
  __device__ __forceinline__ int free_left(int row, int pos) const {
    if (pos < 0) return -1;
    const int w = pos >> 6;
    const uint64_t v = word(row, w) & (((pos & 63) == 63) ? ~0ull : ((2ull << (pos & 63)) - 1));
    if (v) return (w << 6) + 63 - __clzll(v);
    const uint64_t s = w ? (summary(row) & ((1ull << w) - 1)) : 0ull;
    if (!s) return -1;
    const int j = 63 - __clzll(s);
    return (j << 6) + 63 - __clzll(word(row, j));
  }
  // lowest free x >= pos in the row, or -1 (bits past W are never free)
  __device__ __forceinline__ int free_right(int row, int pos) const {
    if (pos < 0) pos = 0;
    const int w = pos >> 6;
    if (w >= WR) return -1;
    const uint64_t v = word(row, w) & (~0ull << (pos & 63));
    if (v) return (w << 6) + __ffsll(v) - 1;
    const uint64_t s = (w + 1 < 64) ? (summary(row) & (~0ull << (w + 1))) : 0ull;
    if (!s) return -1;
    const int j = __ffsll(s) - 1;
    return (j << 6) + __ffsll(word(row, j)) - 1;
  }
};

// nearest integer(s) to t in [0, n): one, or two when t is exactly k + 1/2
__device__ __forceinline__ int nearest_ints(double t, int n, int &o0, int &o1) {
  const double f = floor(t);
  const int lo = (int)f;
  const double fr = __dsub_rn(t, f);
  int c0, c1 = 0, k;
  if (fr < 0.5) {
    c0 = lo;
    k = 1;
  } else if (fr > 0.5) {
    c0 = lo + 1;
    k = 1;
  } else {
    c0 = lo;
    c1 = lo + 1;
    k = 2;
  }
  int m = 0;
  o0 = o1 = 0;
  if (c0 >= 0 && c0 < n) {
    o0 = c0;
    ++m;
  }
  if (k == 2 && c1 >= 0 && c1 < n) {
    if (m) o1 = c1;
    else o0 = c1;
    ++m;
  }
  return m;
}

// Global-minimum free site of a unit cell (lowest tile among tied ones), or
// -1 when every minimum-cost site is taken or the target is off the grid.
template <class Map>
__device__ __forceinline__ long long fast_candidate(const Map &m, double tx, double ty, int W, int H, double &cost) {
  if (!(tx >= 0.0 && tx <= (double)(W - 1) && ty >= 0.0 && ty <= (double)(H - 1))) return -1;
  int x0, x1, y0, y1;
  const int nx = nearest_ints(tx, W, x0, x1);
  const int ny = nearest_ints(ty, H, y0, y1);
  for (int a = 0; a < ny; ++a) {
    const int yy = a ? y1 : y0;
    for (int b = 0; b < nx; ++b) {
      const int xx = b ? x1 : x0;
      if (m.is_free(yy, xx)) {
        cost = __dadd_rn(sq((double)xx - tx), sq((double)yy - ty));
        return (long long)yy * W + xx;
      }
    }
  }
  return -1;
}

// Row handled by `lane` in step s of an outward search around row c:
// lanes 0..15 take rows c - 16 s - 15 .. c - 16 s, lanes 16..31 rows
// c + 16 s + 1 .. c + 16 s + 16 (step 0 covers c - 15 .. c + 16).
__device__ __forceinline__ int step_row(int c, int s, int lane) {
  return (lane < 16) ? c - 16 * s - 15 + lane : c + 16 * s + lane - 15;
}

// Whether step s >= 1 can still hold a row within reach: its nearest rows are
// c - 16 s and c + 16 s + 1; rows farther out on a side are farther from the
// target (the target row rounds to c), so a side whose nearest row is out of
// range or has dy^2 > best is finished.
__device__ __forceinline__ bool step_live(int c, int s, int nrows, double off, double ty, bool have, double best) {
  const int ra = c - 16 * s, rb = c + 16 * s + 1;
  bool live = false;
  if (ra >= 0) live |= !(have && sq(__dsub_rn(__dadd_rn((double)ra, off), ty)) > best);
  if (rb < nrows) live |= !(have && sq(__dsub_rn(__dadd_rn((double)rb, off), ty)) > best);
  return live;
}

// Warp-parallel exact search for a unit cell.  Returns the tile, or -1.
template <class Map>
__device__ long long row_search(const Map &m, double tx, double ty, int W, int H, int lane, double &best_cost) {
  const int cy = min(max((int)floor(__dadd_rn(ty, 0.5)), 0), H - 1);
  const int fx0 = (int)floor(tx);
  const int lpos = min(fx0, W - 1);
  double best = INFINITY;
  long long bt = -1;
  for (int s = 0;; ++s) {
    if (s >= 1 && !step_live(cy, s, H, 0.0, ty, bt >= 0, best)) break;
    const int row = step_row(cy, s, lane);
    double c = INFINITY;
    long long t = kNoTile;
    if (row >= 0 && row < H) {
      const double dy2 = sq((double)row - ty);
      if (!(bt >= 0 && dy2 > best)) {
        const int l = m.free_left(row, lpos);
        const int r = m.free_right(row, fx0 + 1);
        if (l >= 0) {
          c = __dadd_rn(sq((double)l - tx), dy2);
          t = (long long)row * W + l;
        }
        if (r >= 0 && r < W) {
          const double cc = __dadd_rn(sq((double)r - tx), dy2);
          const long long tt = (long long)row * W + r;
          if (cc < c || (cc == c && tt < t)) {
            c = cc;
            t = tt;
          }
        }
      }
    }
    warp_argmin(c, t);
    if (t != kNoTile && (c < best || (c == best && t < bt))) {
      best = c;
      bt = t;
    }
  }
  best_cost = best;
  return bt;
}

// Valid anchors of a w x h block in anchor row ay, word j: bit a set when
// sites [64 j + a, 64 j + a + w) are free in rows ay .. ay + h - 1.
template <class Map>
__device__ __forceinline__ uint64_t valid_word(const Map &m, int ay, int j, int w, int h, int lastw, int AW) {
  uint64_t mm = ~0ull, mn = ~0ull;
  for (int dy = 0; dy < h; ++dy) {
    mm &= m.word(ay + dy, j);
    mn &= (j + 1 < m.WR) ? m.word(ay + dy, j + 1) : 0ull;
  }
  uint64_t v = mm;
  for (int k = 1; k < w; ++k) v &= (mm >> k) | (mn << (64 - k));
  if (j == lastw && ((AW - 1) & 63) != 63) v &= (2ull << ((AW - 1) & 63)) - 1;
  return v;
}

// Warp-parallel exact search for a w x h macro.  Returns the anchor tile, or -1.
template <class Map>
__device__ long long macro_search(const Map &m, double tx, double ty, int W, int H, int w, int h, int lane,
                                  double &best_cost) {
  best_cost = INFINITY;
  const int AW = W - w + 1, AH = H - h + 1;
  if (AW <= 0 || AH <= 0) return -1;
  const double ox = 0.5 * (w - 1), oy = 0.5 * (h - 1);
  const double ux = __dsub_rn(tx, ox), uy = __dsub_rn(ty, oy);
  const int cy = min(max((int)floor(__dadd_rn(uy, 0.5)), 0), AH - 1);
  const int fa = min(max((int)floor(ux), -1), AW - 1);
  const int lastw = (AW - 1) >> 6;
  double best = INFINITY;
  long long bt = -1;
  for (int s = 0;; ++s) {
    if (s >= 1 && !step_live(cy, s, AH, oy, ty, bt >= 0, best)) break;
    const int ay = step_row(cy, s, lane);
    double c = INFINITY;
    long long t = kNoTile;
    if (ay >= 0 && ay < AH) {
      const double dy2 = sq(__dsub_rn(__dadd_rn((double)ay, oy), ty));
      if (!(bt >= 0 && dy2 > best)) {
        if (fa >= 0) {  // nearest valid anchor <= fa
          int j = fa >> 6;
          uint64_t v =
              valid_word(m, ay, j, w, h, lastw, AW) & (((fa & 63) == 63) ? ~0ull : ((2ull << (fa & 63)) - 1));
          while (!v && --j >= 0) v = valid_word(m, ay, j, w, h, lastw, AW);
          if (v) {
            const int a = (j << 6) + 63 - __clzll(v);
            c = __dadd_rn(sq(__dsub_rn(__dadd_rn((double)a, ox), tx)), dy2);
            t = (long long)ay * W + a;
          }
        }
        if (fa + 1 <= AW - 1) {  // nearest valid anchor >= fa + 1
          const int p = fa + 1;
          int j = p >> 6;
          uint64_t v = valid_word(m, ay, j, w, h, lastw, AW) & (~0ull << (p & 63));
          while (!v && ++j <= lastw) v = valid_word(m, ay, j, w, h, lastw, AW);
          if (v) {
            const int a = (j << 6) + __ffsll(v) - 1;
            const double cc = __dadd_rn(sq(__dsub_rn(__dadd_rn((double)a, ox), tx)), dy2);
            const long long tt = (long long)ay * W + a;
            if (cc < c || (cc == c && tt < t)) {
              c = cc;
              t = tt;
            }
          }
        }
      }
    }
    warp_argmin(c, t);
    if (t != kNoTile && (c < best || (c == best && t < bt))) {
      best = c;
      bt = t;
    }
  }
  best_cost = best;
  return bt;
}

template <bool kShared>
__device__ void legalize_body(const LegalArgs &a, const FreeMap<kShared> &m, int lane) {
  const int W = a.W, H = a.H;
  // Macros, one at a time, in solver order.
  for (uint32_t k = 0; k < a.n_macro; ++k) {
    const uint32_t i = a.order[k];
    const float2 p = a.pos[i];
    const uchar2 sz = a.msize[k];
    const int w = sz.x, h = sz.y;
    double c;
    const long long t = macro_search(m, (double)p.x, (double)p.y, W, H, w, h, lane, c);
    if (t < 0) {
      if (lane == 0) *a.status = 1;
      return;
    }
    const int bx = (int)(t % W), by = (int)(t / W);
    for (int q = lane; q < w * h; q += 32) m.take(by + q / w, bx + q % w);
    if (lane == 0) {
      a.sites[i] = make_int2(bx, by);
      if (a.loc) a.loc[i] = make_int2(bx + (w - 1) / 2, by + (h - 1) / 2);
      a.cost[k] = c;
    }
    __syncwarp();
  }
  // Unit cells in batches of 32 consecutive cells of the order.
  const uint32_t n = a.n_order;
  for (uint32_t base = a.n_macro; base < n; base += 32) {
    const uint32_t k = base + lane;
    const bool live = k < n;
    const uint32_t i = live ? a.order[k] : 0u;
    const float2 p = live ? a.pos[i] : make_float2(0.f, 0.f);
    const double tx = p.x, ty = p.y;
    const int cnt = (int)min(32u, n - base);
    const unsigned in_batch = (cnt == 32) ? kFull : ((1u << cnt) - 1u);
    int cur = 0;
    while (cur < cnt) {
      // fast-path candidates of the remaining lanes against the current map
      double c = 0.0;
      long long cand = -1;
      if (live && lane >= cur) cand = fast_candidate(m, tx, ty, W, H, c);
      // committable: a free candidate that no earlier remaining lane shares
      const unsigned same = __match_any_sync(kFull, cand);
      const unsigned earlier = ((1u << lane) - 1u) & ~((1u << cur) - 1u);
      const bool ok = live && lane >= cur && cand >= 0 && (same & earlier) == 0u;
      const unsigned okmask = __ballot_sync(kFull, ok);
      const unsigned bad = ~okmask & (kFull << cur) & in_batch;
      const int stop = bad ? (__ffs(bad) - 1) : cnt;
      if (lane >= cur && lane < stop) {
        const int cx = (int)(cand % W), cyy = (int)(cand / W);
        m.take(cyy, cx);
        a.sites[i] = make_int2(cx, cyy);
        if (a.loc) a.loc[i] = make_int2(cx, cyy);
        a.cost[k] = c;
      }
      __syncwarp();
      if (stop >= cnt) break;
      // lane `stop`: exact search on the map after the prefix
      const double sx = __shfl_sync(kFull, tx, stop), sy = __shfl_sync(kFull, ty, stop);
      double bc;
      const long long t = row_search(m, sx, sy, W, H, lane, bc);
      if (t < 0) {
        if (lane == 0) *a.status = 1;
        return;
      }
      if (lane == stop) {
        const int bx = (int)(t % W), by = (int)(t / W);
        m.take(by, bx);
        a.sites[i] = make_int2(bx, by);
        if (a.loc) a.loc[i] = make_int2(bx, by);
        a.cost[k] = bc;
      }
      __syncwarp();
      cur = stop + 1;
    }
  }
  // Total displacement, summed in cell order as the sequential loop does.
  __threadfence_block();
  __syncwarp();
  double total = 0.0;
  for (uint32_t base = 0; base < n; base += 32) {
    const uint32_t k = base + lane;
    const double v = (k < n) ? __ldcg(a.cost + k) : 0.0;  // +0.0 leaves a non-negative sum unchanged
#pragma unroll
    for (int l = 0; l < 32; ++l) total = __dadd_rn(total, __shfl_sync(kFull, v, l));
  }
  if (lane == 0) {
    *a.disp = total;
    *a.status = 0;
  }
}

template <bool kShared>
__device__ void init_map(const LegalArgs &a, uint64_t *fm, uint64_t *sum, int lane) {
  const size_t words = (size_t)a.WR * a.H;
  for (size_t q = lane; q < words; q += 32) fm[q] = a.free0[q];
  for (int r = lane; r < a.H; r += 32) {
    uint64_t s = 0;
    for (int j = 0; j < a.WR; ++j)
      if (a.free0[(size_t)r * a.WR + j]) s |= 1ull << j;
    sum[r] = s;
  }
  if (!kShared) __threadfence_block();
  __syncwarp();
}

__global__ void __launch_bounds__(32) k_legalize_smem(const LegalArgs a) {
  extern __shared__ uint64_t smem[];
  const int lane = threadIdx.x;
  uint64_t *fm = smem, *sum = smem + (size_t)a.WR * a.H;
  init_map<true>(a, fm, sum, lane);
  legalize_body<true>(a, FreeMap<true>{fm, sum, a.WR}, lane);
}

__global__ void __launch_bounds__(32) k_legalize_global(const LegalArgs a) {
  const int lane = threadIdx.x;
  uint64_t *fm = a.work, *sum = a.work + (size_t)a.WR * a.H;
  init_map<false>(a, fm, sum, lane);
  legalize_body<false>(a, FreeMap<false>{fm, sum, a.WR}, lane);
}

}  // namespace

size_t legalize_smem_bytes(int WR, int H) { return ((size_t)WR * H + H) * sizeof(uint64_t); }

bool legalize_supported(int W, int H) { return W > 0 && H > 0 && (W + 63) / 64 <= 64; }

cudaError_t launch_legalize(const LegalArgs &a, cudaStream_t s) {
  if (!legalize_supported(a.W, a.H) || a.WR != (a.W + 63) / 64) return cudaErrorInvalidValue;
  const size_t bytes = legalize_smem_bytes(a.WR, a.H);
  if (bytes <= kLegalMaxSmem) {
    static thread_local int attr_dev = -1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (attr_dev != dev) {
      e = cudaFuncSetAttribute(k_legalize_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLegalMaxSmem);
      if (e != cudaSuccess) return e;
      attr_dev = dev;
    }
    k_legalize_smem<<<1, 32, bytes, s>>>(a);
  } else {
    if (!a.work) return cudaErrorInvalidValue;
    k_legalize_global<<<1, 32, 0, s>>>(a);
  }
  return cudaGetLastError();
}

}  // namespace eplace
