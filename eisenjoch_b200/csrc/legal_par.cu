// legal_par.cu -- the greedy legaliser of electro_place/mod.rs:206-255 on the
// whole GPU, with results identical to the reference's exhaustive scan
// (common.rs:294-374): cells in order (macros first, an extension), each onto
// the free anchor of minimum (bx - x)^2 + (by - y)^2 in FP64, ties to the
// lowest tile.
//
// The greedy is sequential, but most of its work is not.  The cells are
// placed in rounds; a round takes a window of the next cells in order and
// the free map as it stands (every earlier cell committed):
//  1. lists (one warp per cell): every free anchor whose cost is at most a
//     threshold tau, sorted by (cost, tile), first kLpList kept.  Whatever
//     the later cells of the window take, a cell's serial choice is the first
//     entry of its list that no earlier window cell took -- the free set only
//     shrinks and everything outside the list costs more.  If every entry is
//     taken, the round ends before that cell.
//  2. disturbance (a few parallel passes): a cell is disturbed when an
//     earlier window cell's head (list entry 0) overlaps its head, or an
//     earlier disturbed cell's list does.  An undisturbed cell's head can be
//     taken by no earlier cell, so it is the serial choice.
//  3. serial pass (one CTA, shared memory): undisturbed heads are entered as
//     taken, then the disturbed cells, in order, take the first entry of
//     their list not taken -- exactly the sequential algorithm restricted to
//     the cells that need it.
//  4. commit the window's prefix up to the first exhausted list; advance.
// Rounds loop on the device (a CUDA-graph while node), no host round trip.
// Each round commits at least one cell (the window's first cell has no
// earlier cell to lose its head to) or stops on a cell with no free anchor,
// and the loop also stops after max_rounds, so it always terminates.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "legal_par.cuh"

namespace eplace {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int32_t kNoMark = 0x7f7f7f7f;   // byte-fill value of the mark arrays
constexpr int kListWarps = 8;             // warps per CTA of the list kernel
constexpr int kCandBuf = 256;             // candidates a warp collects before sorting
constexpr int kListMin = 24;              // threshold search aims at >= this many candidates
constexpr int kSerialThreads = 1024;
constexpr int kChunk = 64;                // disturbed cells staged per chunk

__device__ __forceinline__ double sq(double d) { return __dmul_rn(d, d); }

struct Cell {
  double tx, ty;  // target (the continuous position)
  double ox, oy;  // anchor -> block centre offset, (w - 1) / 2
  int w, h;
  int AW, AH;     // anchor grid
};

__device__ __forceinline__ Cell load_cell(const LpArgs &a, uint32_t cell) {
  Cell c;
  const float2 p = a.pos[cell];
  c.tx = (double)p.x;
  c.ty = (double)p.y;
  const uchar2 s = a.fsize ? a.fsize[cell] : make_uchar2(1, 1);
  c.w = s.x;
  c.h = s.y;
  c.ox = 0.5 * (double)(c.w - 1);
  c.oy = 0.5 * (double)(c.h - 1);
  c.AW = a.W - c.w + 1;
  c.AH = a.H - c.h + 1;
  return c;
}

// Cost of anchor (ax, ay), formed as the host legaliser forms it.
__device__ __forceinline__ double anchor_cost(const Cell &c, int ax, double dy2) {
  const double dx = __dsub_rn(__dadd_rn((double)ax, c.ox), c.tx);
  return __dadd_rn(sq(dx), dy2);
}
__device__ __forceinline__ double row_dy2(const Cell &c, int ay) {
  return sq(__dsub_rn(__dadd_rn((double)ay, c.oy), c.ty));
}

// Word j of anchor row ay: bit b set when the w x h block at anchor
// (64 j + b, ay) is free.  Anchors past AW - 1 are never valid.
__device__ __forceinline__ uint64_t valid_word(const LpArgs &a, const Cell &c, int ay, int j) {
  const int lastw = (c.AW - 1) >> 6;
  if (j > lastw) return 0ull;
  uint64_t m = ~0ull, mn = ~0ull;
  for (int dy = 0; dy < c.h; ++dy) {
    const uint64_t *r = a.fm + (size_t)(ay + dy) * a.WR;
    m &= __ldg(reinterpret_cast<const unsigned long long *>(r + j));
    if (c.w > 1) mn &= (j + 1 < a.WR) ? __ldg(reinterpret_cast<const unsigned long long *>(r + j + 1)) : 0ull;
  }
  uint64_t v = m;
  for (int k = 1; k < c.w; ++k) v &= (m >> k) | (mn << (64 - k));
  if (j == lastw && ((c.AW - 1) & 63) != 63) v &= (2ull << ((c.AW - 1) & 63)) - 1;
  return v;
}

struct Cand {
  unsigned long long key;  // cost bits (costs are >= 0, so the bits order like the values)
  int tile;
  int pad_;
};

__device__ __forceinline__ bool cand_less(const Cand &x, const Cand &y) {
  return x.key < y.key || (x.key == y.key && x.tile < y.tile);
}

// Visits the valid anchors of cell c with cost <= tau.  Without buf it
// returns their number (warp-uniform); with buf it appends them (at most
// cap) and returns the number found.
__device__ int scan_tau(const LpArgs &a, const Cell &c, double tau, int lane, Cand *buf, int cap, int *nbuf) {
  const double r = sqrt(tau);
  const double uy = __dsub_rn(c.ty, c.oy), ux = __dsub_rn(c.tx, c.ox);
  const int ay0 = max(0, (int)floor(uy - r) - 1);
  const int ay1 = min(c.AH - 1, (int)ceil(uy + r) + 1);
  int found = 0;
  for (int ay = ay0 + lane; ay <= ay1; ay += 32) {
    const double dy2 = row_dy2(c, ay);
    if (dy2 > tau) continue;
    const double hx = sqrt(__dsub_rn(tau, dy2));
    // approximate bounds, then exact ones: within a row the anchors with
    // cost <= tau form an interval (the cost is convex in ax)
    // (each loop moves one bound monotonically inside [0, AW - 1], so all
    // four end; the estimate is off by at most a step or two)
    int lo = max(0, (int)ceil(ux - hx)), hi = min(c.AW - 1, (int)floor(ux + hx));
    while (lo > 0 && anchor_cost(c, lo - 1, dy2) <= tau) --lo;
    while (lo <= hi && anchor_cost(c, lo, dy2) > tau) ++lo;
    while (hi < c.AW - 1 && anchor_cost(c, hi + 1, dy2) <= tau) ++hi;
    while (hi >= lo && anchor_cost(c, hi, dy2) > tau) --hi;
    if (lo > hi) continue;
    const int j0 = lo >> 6, j1 = hi >> 6;
    for (int j = j0; j <= j1; ++j) {
      uint64_t v = valid_word(a, c, ay, j);
      if (j == j0) v &= ~0ull << (lo & 63);
      if (j == j1 && (hi & 63) != 63) v &= (2ull << (hi & 63)) - 1;
      if (!buf) {
        found += __popcll(v);
        continue;
      }
      while (v) {
        const int ax = (j << 6) + __ffsll(v) - 1;
        v &= v - 1;
        const double cost = anchor_cost(c, ax, dy2);
        if (cost > tau) continue;  // never: the interval is exact
        const int slot = atomicAdd(nbuf, 1);
        if (slot < cap) {
          buf[slot].key = (unsigned long long)__double_as_longlong(cost);
          buf[slot].tile = ay * a.W + ax;
        }
        ++found;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) found += __shfl_xor_sync(kFull, found, o);
  return found;
}

// Bitonic sort of buf[0..n2) (n2 a power of two, >= 32) by one warp.
__device__ void warp_sort(Cand *buf, int n2, int lane) {
  for (int k = 2; k <= n2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < n2; i += 32) {
        const int p = i ^ j;
        if (p > i) {
          const bool up = (i & k) == 0;
          Cand x = buf[i], y = buf[p];
          if (cand_less(y, x) == up) {
            buf[i] = y;
            buf[p] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Marks the sites of the w x h block at anchor tile t with min(mark, q).
__device__ __forceinline__ void mark_block(int32_t *mark, int W, int t, int w, int h, int32_t q) {
  const int ax = t % W, ay = t / W;
  for (int dy = 0; dy < h; ++dy)
    for (int dx = 0; dx < w; ++dx) atomicMin(&mark[(size_t)(ay + dy) * W + ax + dx], q);
}
__device__ __forceinline__ bool block_marked_below(const int32_t *mark, int W, int t, int w, int h, int32_t q) {
  const int ax = t % W, ay = t / W;
  for (int dy = 0; dy < h; ++dy)
    for (int dx = 0; dx < w; ++dx)
      if (__ldcg(&mark[(size_t)(ay + dy) * W + ax + dx]) < q) return true;
  return false;
}
__device__ __forceinline__ void reset_block(int32_t *mark, int W, int t, int w, int h) {
  const int ax = t % W, ay = t / W;
  for (int dy = 0; dy < h; ++dy)
    for (int dx = 0; dx < w; ++dx) mark[(size_t)(ay + dy) * W + ax + dx] = kNoMark;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
__global__ void k_lp_init(const LpArgs a) {
  const size_t words = (size_t)a.WR * a.H;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x)
    a.fm[i] = a.free0[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    LpState *s = a.st;
    s->pos = 0;
    s->bcur = a.n < 2048u ? a.n : 2048u;
    s->stop = 0;
    s->rounds = 0;
    s->status = 0;
    for (int i = 0; i <= kLpPropSteps; ++i) s->changed[i] = 0;
  }
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < kLpMaxWindow; q += gridDim.x * blockDim.x) {
    a.dist[q] = 0;
    a.fresh[q] = 0;
  }
}

// One warp per window cell: its candidate list against the frozen map, and
// its head block entered in hmark.
__global__ void __launch_bounds__(kListWarps * 32) k_lp_lists(const LpArgs a) {
  __shared__ Cand sbuf[kListWarps][kCandBuf];
  __shared__ int scount[kListWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t q = blockIdx.x * kListWarps + wib;
  const LpState *st = a.st;
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (int i = 1; i <= kLpPropSteps; ++i) a.st->changed[i] = 0;
  const uint32_t bcur = st->bcur, pos = st->pos;
  if (q >= bcur || pos + q >= a.n) return;
  const uint32_t cell = a.order[pos + q];
  const Cell c = load_cell(a, cell);
  Cand *buf = sbuf[wib];
  int32_t *out = a.list + (size_t)q * kLpList;
  if (lane == 0) a.info[q] = c.w | (c.h << 8);
  if (c.AW <= 0 || c.AH <= 0) {
    if (lane == 0) a.len[q] = 0;
    return;
  }
  // Threshold: grow until at least kListMin candidates (or the whole chip),
  // then, if that overshoots the buffer, bisect back into [kListMin, kCandBuf].
  const double span = (double)a.W + (double)a.H;
  const double tau_max = span * span;
  double tau = 2.0, lo = -1.0;
  int cnt = scan_tau(a, c, tau, lane, nullptr, 0, nullptr);
  for (int g = 0; cnt < kListMin && tau < tau_max && g < 64; ++g) {
    lo = tau;
    tau = fmin(tau * 4.0 + 4.0, tau_max);
    cnt = scan_tau(a, c, tau, lane, nullptr, 0, nullptr);
  }
  int lo_cnt = lo < 0.0 ? 0 : -1;  // count at lo when known
  for (int it = 0; cnt > kCandBuf && it < 64; ++it) {
    const double mid = lo < 0.0 ? 0.5 * tau : lo + 0.5 * (tau - lo);
    if (!(mid > lo && mid < tau)) break;
    const int m = scan_tau(a, c, mid, lane, nullptr, 0, nullptr);
    if (m > kCandBuf) {
      tau = mid;
      cnt = m;
    } else if (m >= kListMin) {
      tau = mid;
      cnt = m;
    } else {
      lo = mid;
      lo_cnt = m;
    }
  }
  if (cnt > kCandBuf) {  // a tie group wider than the buffer: fall back to lo
    if (lo >= 0.0) {
      tau = lo;
      cnt = lo_cnt >= 0 ? lo_cnt : scan_tau(a, c, lo, lane, nullptr, 0, nullptr);
    }
    if (cnt == 0 || cnt > kCandBuf) {
      if (lane == 0) {
        a.len[q] = 0;
        atomicMax(&a.st->status, 3);
      }
      return;
    }
  }
  if (cnt == 0) {  // no free anchor anywhere
    if (lane == 0) a.len[q] = 0;
    return;
  }
  if (lane == 0) scount[wib] = 0;
  __syncwarp();
  scan_tau(a, c, tau, lane, buf, kCandBuf, &scount[wib]);
  __syncwarp();
  const int n = min(scount[wib], kCandBuf);
  int n2 = 32;
  while (n2 < n) n2 <<= 1;
  for (int i = n + lane; i < n2; i += 32) {
    buf[i].key = ~0ull;
    buf[i].tile = 0x7fffffff;
  }
  __syncwarp();
  warp_sort(buf, n2, lane);
  const int keep = min(n, kLpList);
  for (int i = lane; i < keep; i += 32) out[i] = buf[i].tile;
  if (lane == 0) a.len[q] = keep;
  // head block into hmark (lanes split the block's rows)
  const int t = buf[0].tile;
  const int ax = t % a.W, ay = t / a.W;
  for (int k = lane; k < c.w * c.h; k += 32)
    atomicMin(&a.hmark[(size_t)(ay + k / c.w) * a.W + ax + k % c.w], (int32_t)q);
}

// Disturbance pass `step`: cells whose head block lies under an earlier
// window cell's head (step 0) or under an earlier disturbed cell's list
// become disturbed and enter their whole list in dmark.
__global__ void k_lp_prop(const LpArgs a, int step) {
  const LpState *st = a.st;
  if (step > 0 && __ldcg(&st->changed[step]) == 0u) return;
  const uint32_t bcur = st->bcur, pos = st->pos;
  bool found = false;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < bcur && pos + q < a.n;
       q += gridDim.x * blockDim.x) {
    const int len = a.len[q];
    if (len <= 0) continue;
    const int inf = a.info[q];
    const uchar2 s = make_uchar2(inf & 255, inf >> 8);
    const int32_t *lst = a.list + (size_t)q * kLpList;
    if (!a.dist[q]) {
      const bool d = step == 0 ? block_marked_below(a.hmark, a.W, lst[0], s.x, s.y, (int32_t)q)
                               : block_marked_below(a.dmark, a.W, lst[0], s.x, s.y, (int32_t)q);
      if (d) {
        a.dist[q] = 1;
        a.fresh[q] = 1;
        found = true;
      }
    }
    if (a.fresh[q]) {
      for (int e = 0; e < len; ++e) mark_block(a.dmark, a.W, lst[e], s.x, s.y, (int32_t)q);
      a.fresh[q] = 0;
    }
  }
  if (found) a.st->changed[step + 1] = 1u;
}

// Sites taken during a round's serial pass, in shared memory: a bitmap of
// the whole chip when it has at most 2^20 sites, else a hash of the taken
// sites (keys tile + 1, 0 = empty), whose load caps the window.
constexpr int kBitmapSites = 1 << 20;

struct TakenBits {
  uint32_t *w;
  int W;
  __device__ __forceinline__ void clear(int tid, int nt, int nsites) {
    for (int i = tid; i < (nsites + 31) / 32; i += nt) w[i] = 0u;
  }
  __device__ __forceinline__ bool block_taken(int t, int bw, int bh) const {
    // a unit cell's block is its one site, whose bit index is the tile
    if (bw == 1 && bh == 1) return (reinterpret_cast<const volatile uint32_t *>(w)[t >> 5] >> (t & 31)) & 1u;
    const int ax = t % W, ay = t / W;
    for (int dy = 0; dy < bh; ++dy) {
      const int s0 = (ay + dy) * W + ax, s1 = s0 + bw - 1;
      const int w0 = s0 >> 5, w1 = s1 >> 5;
      const volatile uint32_t *vw = w;
      if (w0 == w1) {
        const uint32_t m = (bw == 32 ? ~0u : ((1u << bw) - 1u)) << (s0 & 31);
        if (vw[w0] & m) return true;
      } else {
        if (vw[w0] & (~0u << (s0 & 31))) return true;
        if (vw[w1] & ((2u << (s1 & 31)) - 1u)) return true;
      }
    }
    return false;
  }
  __device__ __forceinline__ void put(int t, int bw, int bh) {
    if (bw == 1 && bh == 1) {
      atomicOr(&w[t >> 5], 1u << (t & 31));
      return;
    }
    const int ax = t % W, ay = t / W;
    for (int dy = 0; dy < bh; ++dy)
      for (int dx = 0; dx < bw; ++dx) {
        const int s = (ay + dy) * W + ax + dx;
        atomicOr(&w[s >> 5], 1u << (s & 31));
      }
  }
};

constexpr int kHashBits = 15;
constexpr int kHashLimit = 1 << 14;  // sites entered per round (load factor <= 1/2)

struct TakenHash {
  int *hs;
  int W;
  __device__ __forceinline__ static unsigned slot(int key) { return ((unsigned)key * 2654435761u) >> (32 - kHashBits); }
  __device__ __forceinline__ void clear(int tid, int nt, int) {
    for (int i = tid; i < (1 << kHashBits); i += nt) hs[i] = 0;
  }
  __device__ __forceinline__ bool has(int key) const {
    const unsigned s = slot(key);
    for (int p = 0; p < (1 << kHashBits); ++p) {
      const int v = reinterpret_cast<const volatile int *>(hs)[(s + p) & ((1u << kHashBits) - 1)];
      if (v == key + 1) return true;
      if (v == 0) return false;
    }
    return false;
  }
  __device__ __forceinline__ void add(int key) {
    const unsigned s = slot(key);
    for (int p = 0; p < (1 << kHashBits); ++p) {
      const int prev = atomicCAS(&hs[(s + p) & ((1u << kHashBits) - 1)], 0, key + 1);
      if (prev == 0 || prev == key + 1) return;
    }
  }
  __device__ __forceinline__ bool block_taken(int t, int bw, int bh) const {
    const int ax = t % W, ay = t / W;
    for (int dy = 0; dy < bh; ++dy)
      for (int dx = 0; dx < bw; ++dx)
        if (has((ay + dy) * W + ax + dx)) return true;
    return false;
  }
  __device__ __forceinline__ void put(int t, int bw, int bh) {
    const int ax = t % W, ay = t / W;
    for (int dy = 0; dy < bh; ++dy)
      for (int dx = 0; dx < bw; ++dx) add((ay + dy) * W + ax + dx);
  }
};

// Inclusive block-wide sum of v (all kSerialThreads threads call it); the
// block's total is left in wsum[31].
__device__ __forceinline__ int block_scan(int v, int *wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) wsum[w] = v;
  __syncthreads();
  if (w == 0) {
    int s = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, s, o);
      if (lane >= o) s += t;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  const int r = v + (w ? wsum[w - 1] : 0);
  __syncthreads();
  return r;
}

struct SerialShared {
  uint16_t didx[kLpMaxWindow];
  int lbuf[2][kChunk][kLpList];
  int llen[2][kChunk];
  int linf[2][kChunk];
  int wsum[32];
  int carry, bwin, halt, stop;
};

template <bool kBits>
constexpr size_t serial_smem_bytes() {
  return sizeof(SerialShared) + (kBits ? sizeof(uint32_t) * (kBitmapSites / 32) : sizeof(int) * (1 << kHashBits));
}

// The serial pass of a round (one CTA).
template <bool kBits>
__global__ void __launch_bounds__(kSerialThreads, 1) k_lp_serial(const LpArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SerialShared &S = *reinterpret_cast<SerialShared *>(smem_raw);
  using Taken = typename std::conditional<kBits, TakenBits, TakenHash>::type;
  Taken tk;
  if constexpr (kBits) tk = TakenBits{reinterpret_cast<uint32_t *>(smem_raw + sizeof(SerialShared)), a.W};
  else tk = TakenHash{reinterpret_cast<int *>(smem_raw + sizeof(SerialShared)), a.W};
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t pos = a.st->pos;
  const uint32_t bcur = min(a.st->bcur, a.n - min(pos, a.n));
  const bool all_serial = __ldcg(&a.st->changed[kLpPropSteps]) != 0u;  // propagation did not settle
  tk.clear(tid, kSerialThreads, a.W * a.H);
  if (tid == 0) {
    S.bwin = (int)bcur;
    S.halt = 0;
    S.stop = -1;
    S.carry = 0;
  }
  __syncthreads();
  if constexpr (!kBits) {
    // Window cap: the prefix whose blocks fit the hash's load limit.
    for (uint32_t base = 0; base < bcur; base += kSerialThreads) {
      const uint32_t q = base + tid;
      int sz = 0;
      if (q < bcur) {
        const int inf = a.info[q];
        sz = (inf & 255) * (inf >> 8);
      }
      const int incl = block_scan(sz, S.wsum);
      if (q < bcur && S.carry + incl > kHashLimit) atomicMin(&S.bwin, (int)q);
      __syncthreads();
      if (tid == 0) S.carry += S.wsum[31];
      __syncthreads();
      if (S.bwin < (int)bcur) break;
    }
  }
  const int bwin = S.bwin;
  // Undisturbed heads are taken; disturbed cells are listed in order.
  int nd = 0;
  for (int base = 0; base < bwin; base += kSerialThreads) {
    const int q = base + tid;
    int dis = 0;
    if (q < bwin) {
      const int len = a.len[q];
      dis = (all_serial || a.dist[q] || len <= 0) ? 1 : 0;
      if (!dis) {
        const int inf = a.info[q];
        tk.put(a.list[(size_t)q * kLpList], inf & 255, inf >> 8);
      }
    }
    const int incl = block_scan(dis, S.wsum);
    if (dis) S.didx[nd + incl - 1] = (uint16_t)q;
    nd += S.wsum[31];
    __syncthreads();
  }
  // Stage chunk k of the disturbed cells' lists into buffer k & 1: one warp
  // per cell, the list read as whole 128-byte lines.
  auto stage = [&](int k, int wfirst, int nwarps) {
    const int b = k & 1, c0 = k * kChunk;
    for (int r = warp - wfirst; r < kChunk; r += nwarps) {
      if (c0 + r >= nd) break;
      const int q = S.didx[c0 + r];
      const int len = __ldcg(&a.len[q]);
      for (int e = lane; e < len; e += 32) S.lbuf[b][r][e] = __ldcg(&a.list[(size_t)q * kLpList + e]);
      if (lane == 0) {
        S.llen[b][r] = len;
        S.linf[b][r] = __ldcg(&a.info[q]);
      }
    }
  };
  stage(0, 0, kSerialThreads / 32);
  __syncthreads();
  const int nchunks = (nd + kChunk - 1) / kChunk;
  for (int k = 0; k < nchunks; ++k) {
    if (warp == 0) {
      const int b = k & 1;
      for (int r = 0; r < kChunk && k * kChunk + r < nd; ++r) {
        const int q = S.didx[k * kChunk + r];
        const int len = S.llen[b][r];
        const int inf = S.linf[b][r];
        const int bw = inf & 255, bh = inf >> 8;
        int pick = -1;
        for (int e0 = 0; e0 < len && pick < 0; e0 += 32) {
          const int e = e0 + lane;
          bool ok = false;
          int t = 0;
          if (e < len) {
            t = S.lbuf[b][r][e];
            ok = !tk.block_taken(t, bw, bh);
          }
          const unsigned m = __ballot_sync(kFull, ok);
          if (m) pick = __shfl_sync(kFull, t, __ffs(m) - 1);
        }
        if (pick < 0) {  // list exhausted (or empty): the round ends before q
          if (lane == 0) {
            S.stop = q;
            S.halt = 1;
            if (q == 0) atomicMax(&a.st->status, len <= 0 ? 1 : 3);
          }
          break;
        }
        if (lane == 0) {
          tk.put(pick, bw, bh);
          a.pick[q] = pick;
        }
        __syncwarp();
      }
    } else if (k + 1 < nchunks) {
      stage(k + 1, 1, kSerialThreads / 32 - 1);
    }
    __syncthreads();
    if (S.halt) break;
  }
  __syncthreads();
  if (tid == 0) a.st->stop = (uint32_t)(S.stop >= 0 ? S.stop : bwin);
}

// Commits the round's prefix and clears every mark the round set.
__global__ void k_lp_commit(const LpArgs a) {
  const LpState *st = a.st;
  const uint32_t bcur = st->bcur, pos = st->pos, stop = st->stop;
  const bool all_serial = st->changed[kLpPropSteps] != 0u;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < bcur && pos + q < a.n;
       q += gridDim.x * blockDim.x) {
    const int len = a.len[q];
    const uint32_t cell = a.order[pos + q];
    const int inf = a.info[q];
    const uchar2 s = make_uchar2(inf & 255, inf >> 8);
    const int32_t *lst = a.list + (size_t)q * kLpList;
    if (len > 0) {
      reset_block(a.hmark, a.W, lst[0], s.x, s.y);
      if (a.dist[q])
        for (int e = 0; e < len; ++e) reset_block(a.dmark, a.W, lst[e], s.x, s.y);
    }
    if (q < stop) {
      const int t = (all_serial || a.dist[q]) ? a.pick[q] : lst[0];
      const int ax = t % a.W, ay = t / a.W;
      for (int dy = 0; dy < s.y; ++dy)
        for (int dx = 0; dx < s.x; ++dx) {
          const int x = ax + dx;
          atomicAnd(reinterpret_cast<unsigned long long *>(a.fm + (size_t)(ay + dy) * a.WR + (x >> 6)),
                    ~(1ull << (x & 63)));
        }
      a.sites[cell] = make_int2(ax, ay);
      if (a.loc) a.loc[cell] = make_int2(ax + (s.x - 1) / 2, ay + (s.y - 1) / 2);
      const Cell c = load_cell(a, cell);
      a.cost[pos + q] = anchor_cost(c, ax, row_dy2(c, ay));
    }
    a.dist[q] = 0;
    a.fresh[q] = 0;
  }
}

__global__ void k_lp_advance(const LpArgs a) {
  if (threadIdx.x != 0) return;
  LpState *s = a.st;
  s->pos += s->stop;
  s->rounds += 1;
  const uint32_t left = a.n - min(s->pos, a.n);
  uint32_t b = 2u * s->stop;
  b = max(b, 512u);
  b = min(b, kLpMaxWindow);
  s->bcur = min(b, left);
  if (s->status == 0 && left > 0 && s->rounds >= a.max_rounds) s->status = 2;
  if (left == 0 || s->status != 0) cudaGraphSetConditional(a.handle, 0u);
}

// Total displacement, summed in order as the sequential loop does, and the
// status.
__global__ void k_lp_finish(const LpArgs a) {
  const int lane = threadIdx.x;
  double total = 0.0;
  if (a.st->status == 0) {
    for (uint32_t base = 0; base < a.n; base += 32) {
      const uint32_t k = base + lane;
      const double v = (k < a.n) ? __ldcg(a.cost + k) : 0.0;  // +0.0 leaves a non-negative sum unchanged
#pragma unroll
      for (int l = 0; l < 32; ++l) total = __dadd_rn(total, __shfl_sync(kFull, v, l));
    }
  }
  if (lane == 0) {
    *a.disp = total;
    *a.status = a.st->status;
  }
}

}  // namespace

size_t lp_scratch_bytes(int W, int H) {
  return 2 * sizeof(int32_t) * (size_t)W * H + sizeof(int32_t) * (size_t)kLpMaxWindow * (kLpList + 3) +
         2 * (size_t)kLpMaxWindow;
}

LpGraph::~LpGraph() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
}

cudaError_t lp_build_graph(LpArgs a, LpGraph &g, cudaStream_t cs) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  g.exec = nullptr;
  g.graph = nullptr;
  const bool bits = (size_t)a.W * a.H <= (size_t)kBitmapSites;
  const size_t smem = bits ? serial_smem_bytes<true>() : serial_smem_bytes<false>();
  cudaError_t e = bits ? cudaFuncSetAttribute(k_lp_serial<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                       : cudaFuncSetAttribute(k_lp_serial<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cudaGraph_t graph = nullptr;
  if ((e = cudaGraphCreate(&graph, 0)) != cudaSuccess) return e;
  g.graph = graph;
  // Before the loop: map copy and round state, mark arrays cleared.
  cudaGraphNode_t n_set1, n_set2, n_init, n_loop, n_fin;
  cudaMemsetParams ms = {};
  ms.dst = a.hmark;
  ms.value = 0x7f;
  ms.elementSize = 1;
  ms.width = sizeof(int32_t) * (size_t)a.W * a.H;
  ms.height = 1;
  ms.pitch = ms.width;
  if ((e = cudaGraphAddMemsetNode(&n_set1, graph, nullptr, 0, &ms)) != cudaSuccess) return e;
  ms.dst = a.dmark;
  if ((e = cudaGraphAddMemsetNode(&n_set2, graph, nullptr, 0, &ms)) != cudaSuccess) return e;
  cudaKernelNodeParams kp = {};
  void *args[] = {&a};
  kp.func = (void *)k_lp_init;
  kp.gridDim = dim3(256);
  kp.blockDim = dim3(256);
  kp.kernelParams = args;
  cudaGraphNode_t pre[2] = {n_set1, n_set2};
  if ((e = cudaGraphConditionalHandleCreate(&a.handle, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
    return e;
  if ((e = cudaGraphAddKernelNode(&n_init, graph, pre, 2, &kp)) != cudaSuccess) return e;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = a.handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if ((e = cudaGraphAddNode(&n_loop, graph, &n_init, 1, &cp)) != cudaSuccess) return e;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // The round, captured into the loop body.
  if ((e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return e;
  k_lp_lists<<<kLpMaxWindow / kListWarps, kListWarps * 32, 0, cs>>>(a);
  for (int i = 0; i < kLpPropSteps; ++i) k_lp_prop<<<kLpMaxWindow / 256, 256, 0, cs>>>(a, i);
  if (bits) k_lp_serial<true><<<1, kSerialThreads, smem, cs>>>(a);
  else k_lp_serial<false><<<1, kSerialThreads, smem, cs>>>(a);
  k_lp_commit<<<kLpMaxWindow / 128, 128, 0, cs>>>(a);
  k_lp_advance<<<1, 32, 0, cs>>>(a);
  const cudaError_t launch_err = cudaGetLastError();
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(cs, &captured);
  if (launch_err != cudaSuccess) return launch_err;
  if (e != cudaSuccess) return e;
  // After the loop: displacement and status.
  kp.func = (void *)k_lp_finish;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(32);
  if ((e = cudaGraphAddKernelNode(&n_fin, graph, &n_loop, 1, &kp)) != cudaSuccess) return e;
  return cudaGraphInstantiate(&g.exec, graph, 0);
}

}  // namespace eplace
