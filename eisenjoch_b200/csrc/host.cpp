// host.cpp -- host-side parts of the ElectroPlace path: problem validation,
// the reference's initial placement and pin weights, the exact greedy
// legaliser, integer HPWL and the synthetic netlist generator.
#include <immintrin.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <system_error>
#include <thread>

#include "eplace_internal.h"

namespace eplace {

// ---------------------------------------------------------------------------
// Validation.  The reference Design cannot hold malformed nets; the flat
// arrays can, so they are checked here instead of trusting the caller.
// ---------------------------------------------------------------------------
eplace_status load_problem(const eplace_netlist *nl, const eplace_chip *chip, HostProblem &hp,
                           std::string &msg) {
  if (!nl || !chip) { msg = "null netlist or chip"; return EPLACE_ERR_INVALID; }
  if (chip->width <= 0 || chip->height <= 0) { msg = "chip width/height must be positive"; return EPLACE_ERR_INVALID; }
  hp.W = chip->width;
  hp.H = chip->height;
  hp.BX = chip->bins_x > 0 ? chip->bins_x : chip->width;
  hp.BY = chip->bins_y > 0 ? chip->bins_y : chip->height;
  if (hp.W % hp.BX || hp.H % hp.BY) { msg = "width/height must be multiples of bins_x/bins_y"; return EPLACE_ERR_INVALID; }
  hp.sx = hp.W / hp.BX;
  hp.sy = hp.H / hp.BY;
  if ((int64_t)hp.BX * hp.BY > (1 << 26)) { msg = "bin grid too large"; return EPLACE_ERR_INVALID; }
  hp.N = nl->num_cells;
  hp.F = nl->num_fixed;
  hp.NN = nl->num_nets;
  if (hp.N > (1u << 30) || hp.F > (1u << 30)) { msg = "too many cells"; return EPLACE_ERR_INVALID; }
  if (hp.NN > 0 && (!nl->net_offsets || !nl->pin_cell)) { msg = "missing net arrays"; return EPLACE_ERR_INVALID; }
  if (hp.F > 0 && (!nl->fixed_x || !nl->fixed_y)) { msg = "missing fixed-cell locations"; return EPLACE_ERR_INVALID; }
  hp.P = hp.NN ? nl->net_offsets[hp.NN] : 0;
  if (hp.NN && nl->net_offsets[0] != 0) { msg = "net_offsets[0] must be 0"; return EPLACE_ERR_INVALID; }
  hp.net_off.assign(nl->net_offsets, nl->net_offsets + (hp.NN ? hp.NN + 1 : 0));
  if (hp.NN == 0) hp.net_off.assign(1, 0);
  // Branch-free scans (they vectorise): monotone offsets, largest degree,
  // largest pin cell.
  uint32_t drop = 0, maxdeg = 0;
  for (uint32_t n = 0; n < hp.NN; ++n) {
    const uint32_t a = hp.net_off[n], b = hp.net_off[n + 1];
    drop |= (uint32_t)(b < a);
    maxdeg = std::max(maxdeg, b - a);
  }
  if (drop) { msg = "net_offsets not monotone"; return EPLACE_ERR_INVALID; }
  hp.max_degree = maxdeg;
  hp.pin_cell.assign(nl->pin_cell, nl->pin_cell + hp.P);
  uint32_t maxcell = 0;
  for (uint32_t p = 0; p < hp.P; ++p) maxcell = std::max(maxcell, hp.pin_cell[p]);
  if (hp.P && maxcell >= hp.N + hp.F) { msg = "pin_cell out of range"; return EPLACE_ERR_INVALID; }
  hp.cw.assign(hp.N, 1);
  hp.ch.assign(hp.N, 1);
  if (nl->cell_w) std::copy(nl->cell_w, nl->cell_w + hp.N, hp.cw.begin());
  if (nl->cell_h) std::copy(nl->cell_h, nl->cell_h + hp.N, hp.ch.begin());
  for (uint32_t i = 0; i < hp.N; ++i) {
    if (hp.cw[i] == 0 || hp.ch[i] == 0 || hp.cw[i] > hp.W || hp.ch[i] > hp.H) {
      msg = "cell footprint out of range";
      return EPLACE_ERR_INVALID;
    }
    if (hp.cw[i] * hp.ch[i] > 1) hp.any_macro = true;
  }
  hp.init_x.assign(hp.N, -1);
  hp.init_y.assign(hp.N, -1);
  if (nl->cell_init_x && nl->cell_init_y) {
    for (uint32_t i = 0; i < hp.N; ++i) {
      int32_t x = nl->cell_init_x[i], y = nl->cell_init_y[i];
      if (x < 0) continue;
      if (x >= hp.W || y < 0 || y >= hp.H) { msg = "cell_init out of range"; return EPLACE_ERR_INVALID; }
      hp.init_x[i] = x;
      hp.init_y[i] = y;
    }
  }
  hp.fx.assign(nl->fixed_x, nl->fixed_x + hp.F);
  hp.fy.assign(nl->fixed_y, nl->fixed_y + hp.F);
  hp.f_logic.assign(hp.F, 0);
  if (nl->fixed_on_logic) std::copy(nl->fixed_on_logic, nl->fixed_on_logic + hp.F, hp.f_logic.begin());
  for (uint32_t f = 0; f < hp.F; ++f) {
    if (hp.f_logic[f] && (hp.fx[f] < 0 || hp.fx[f] >= hp.W || hp.fy[f] < 0 || hp.fy[f] >= hp.H)) {
      msg = "fixed cell on a logic BEL outside the chip";
      return EPLACE_ERR_INVALID;
    }
  }
  hp.has_driver.assign(hp.NN, 1);
  if (nl->net_has_driver) std::copy(nl->net_has_driver, nl->net_has_driver + hp.NN, hp.has_driver.begin());
  return EPLACE_OK;
}

// ---------------------------------------------------------------------------
// xorshift64 (context/rng.rs:19-31) and Fisher-Yates (rng.rs:52-61).
// ---------------------------------------------------------------------------
static inline uint64_t xorshift64(uint64_t &s) {
  s ^= s << 13;
  s ^= s >> 7;
  s ^= s << 17;
  return s;
}

// initial_placement (placer/common.rs:27-117).  All movable cells share one
// bucket (tile-major logic BELs, context/buckets.rs:37-43); bound cells keep
// their BEL; the available BELs are shuffled once and handed out in order.
eplace_status initial_placement(const HostProblem &hp, uint64_t seed, std::vector<int32_t> &sx,
                                std::vector<int32_t> &sy, std::string &msg) {
  sx.assign(hp.N, 0);
  sy.assign(hp.N, 0);
  if (hp.N == 0) return EPLACE_OK;
  const int64_t nsites = (int64_t)hp.W * hp.H;
  std::vector<uint8_t> occ((size_t)nsites, 0);
  for (uint32_t f = 0; f < hp.F; ++f)
    if (hp.f_logic[f]) occ[(size_t)hp.fy[f] * hp.W + hp.fx[f]] = 1;
  uint32_t unbound = 0;
  for (uint32_t i = 0; i < hp.N; ++i) {
    if (hp.init_x[i] >= 0) {
      size_t t = (size_t)hp.init_y[i] * hp.W + hp.init_x[i];
      if (occ[t]) {
        msg = "cell " + std::to_string(i);
        return EPLACE_ERR_INITIAL_PLACEMENT;
      }
      occ[t] = 1;
      sx[i] = hp.init_x[i];
      sy[i] = hp.init_y[i];
    } else {
      ++unbound;
    }
  }
  if (unbound == 0) return EPLACE_OK;
  std::vector<int32_t> avail;
  avail.reserve((size_t)nsites);
  for (int64_t t = 0; t < nsites; ++t)
    if (!occ[(size_t)t]) avail.push_back((int32_t)t);
  uint64_t rng = seed ? seed : 1;
  // Fisher-Yates from the end, j = (u32)rng % (i + 1).  The random stream
  // does not depend on the array, so the j of step i - D is drawn D steps
  // early and its element prefetched: the same swaps, with the cache misses
  // of the random accesses overlapped.
  {
    constexpr int D = 16;
    const size_t n = avail.size();
    uint32_t jq[D];
    for (int k = 0; k < D && (size_t)k + 1 < n; ++k) {
      jq[k] = (uint32_t)xorshift64(rng) % (uint32_t)(n - k);  // step i = n - 1 - k
      __builtin_prefetch(&avail[jq[k]], 1);
    }
    int head = 0;
    for (size_t i = n; i-- > 1;) {
      const uint32_t j = jq[head];
      if (i >= (size_t)D + 1) {  // draw for step i - D
        jq[head] = (uint32_t)xorshift64(rng) % (uint32_t)(i - D + 1);
        __builtin_prefetch(&avail[jq[head]], 1);
      }
      head = (head + 1) % D;
      std::swap(avail[i], avail[j]);
    }
  }
  if (unbound > avail.size()) {
    msg = "logic (need " + std::to_string(unbound) + " BELs but only " + std::to_string(avail.size()) +
          " available)";
    return EPLACE_ERR_NO_BELS;
  }
  size_t k = 0;
  for (uint32_t i = 0; i < hp.N; ++i) {
    if (hp.init_x[i] >= 0) continue;
    int32_t t = avail[k++];
    sx[i] = t % hp.W;
    sy[i] = t / hp.W;
  }
  return EPLACE_OK;
}

// compute_pin_weights (placer/common.rs:381-407).
void pin_weights(const HostProblem &hp, std::vector<double> &w) {
  w.assign(hp.N, 0.0);
  for (uint32_t n = 0; n < hp.NN; ++n) {
    uint32_t b = hp.net_off[n], e = hp.net_off[n + 1];
    if (e - b < 2) continue;
    double wt = 1.0 / (double)(e - b);
    for (uint32_t q = b; q < e; ++q)
      if (hp.pin_cell[q] < hp.N) w[hp.pin_cell[q]] += wt;
  }
}

// ---------------------------------------------------------------------------
// Greedy legaliser (electro_place/mod.rs:206-255).
// The reference scans every bucket BEL in chipdb order and keeps the first
// strict minimum of (bx - x)^2 + (by - y)^2 (f64).  The same choice is found
// here in two steps per cell:
//  * fast path: the sites of minimum cost over the whole grid are the
//    nearest integer point(s) to (x, y) (two per axis only when the
//    coordinate is exactly k + 1/2).  If one of them is free it is the
//    answer, and among tied ones the lowest tile wins, as in the scan.
//  * otherwise rows are visited outward from the target; in one row the
//    best free site is the nearest free bit left of or right of floor(x)
//    (64-bit free maps; a per-row summary word, one bit per map word,
//    jumps over full words in one step on rows up to 4096 sites), and a
//    row whose dy^2 already exceeds the best cost cannot win or tie.
// Macros (w*h > 1, an extension) go first onto fully free blocks, cost
// measured at the block centre.
// ---------------------------------------------------------------------------
LegalBase::LegalBase(const HostProblem &hp) : W(hp.W), H(hp.H) {
  WR = (W + 63) / 64;
  free0.assign((size_t)WR * H, ~0ull);
  if (W % 64) {
    const uint64_t tail = (1ull << (W % 64)) - 1;
    for (int32_t y = 0; y < H; ++y) free0[(size_t)y * WR + WR - 1] = tail;
  }
  for (uint32_t f = 0; f < hp.F; ++f)
    if (hp.f_logic[f]) free0[(size_t)hp.fy[f] * WR + (hp.fx[f] >> 6)] &= ~(1ull << (hp.fx[f] & 63));
  if (WR <= 64) {
    sum0.assign(H, 0);
    for (int32_t y = 0; y < H; ++y)
      for (int32_t w = 0; w < WR; ++w)
        if (free0[(size_t)y * WR + w]) sum0[y] |= 1ull << w;
  }
  order.reserve(hp.N);
  for (uint32_t i = 0; i < hp.N; ++i)
    if (hp.cw[i] * hp.ch[i] > 1) order.push_back(i);
  for (uint32_t i = 0; i < hp.N; ++i)
    if (hp.cw[i] * hp.ch[i] == 1) order.push_back(i);
}

Legalizer::Legalizer(const HostProblem &hp, const LegalBase &base) : hp_(hp), base_(base) {
  __builtin_cpu_init();
  // EPLACE_LEGAL_SIMD=0/1 caps the search at the scalar / AVX2 form (all
  // forms give the same bindings; tests compare each with the oracle).
  const char *cap = std::getenv("EPLACE_LEGAL_SIMD");
  const int level = cap ? std::atoi(cap) : 2;
  simd_ = level >= 1 && __builtin_cpu_supports("avx2");
  // The eight-row search keeps tiles in 32 bits: chips below 2^31 sites.
  simd512_ = simd_ && level >= 2 && __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512vl") &&
             (int64_t)hp.W * hp.H < ((int64_t)1 << 31);
  free_.resize(base.free0.size());
  sum_.resize(base.sum0.size());
  lc_.resize(std::max(base.H, 0));
  rc_.resize(std::max(base.H, 0));
}

namespace {
// highest free x <= pos in the row, or -1.  sum (when given) has bit w set
// for each word w of the row with a free site, so a full stretch of words
// is skipped in one step.
inline int32_t free_at_or_left(const uint64_t *row, const uint64_t *sum, int32_t pos) {
  if (pos < 0) return -1;
  int32_t w = pos >> 6;
  uint64_t m = row[w] & (((pos & 63) == 63) ? ~0ull : ((2ull << (pos & 63)) - 1));
  if (m) return (w << 6) + 63 - __builtin_clzll(m);
  if (sum) {
    const uint64_t s = *sum & ((1ull << w) - 1);
    if (!s) return -1;
    const int32_t w2 = 63 - __builtin_clzll(s);
    return (w2 << 6) + 63 - __builtin_clzll(row[w2]);
  }
  while (true) {
    if (--w < 0) return -1;
    m = row[w];
    if (m) return (w << 6) + 63 - __builtin_clzll(m);
  }
}
// lowest free x >= pos in the row, or -1
inline int32_t free_at_or_right(const uint64_t *row, const uint64_t *sum, int32_t pos, int32_t W, int32_t words) {
  if (pos >= W) return -1;
  if (pos < 0) pos = 0;
  int32_t w = pos >> 6;
  uint64_t m = row[w] & (~0ull << (pos & 63));
  if (!m) {
    if (sum) {
      const uint64_t s = (w >= 63) ? 0ull : (*sum & (~0ull << (w + 1)));
      if (!s) return -1;
      w = __builtin_ctzll(s);
      m = row[w];
    } else {
      do {
        if (++w >= words) return -1;
        m = row[w];
      } while (!m);
    }
  }
  const int32_t x = (w << 6) + __builtin_ctzll(m);
  return x < W ? x : -1;
}
inline bool is_free(const uint64_t *fm, int32_t WR, int32_t x, int32_t y) {
  return (fm[(size_t)y * WR + (x >> 6)] >> (x & 63)) & 1;
}
// floor(t), exactly: truncate toward zero and step down for a negative
// fraction (|t| < 2^62, the legaliser's coordinates); anything else goes to
// std::floor.  Built for baseline x86-64, std::floor is a library call, and
// the legaliser takes up to four per cell.
inline double floor_exact(double t) {
  if (!(t > -4.0e18 && t < 4.0e18)) return std::floor(t);
  const double f = (double)(long long)t;
  return f > t ? f - 1.0 : f;
}

// Nearest integer(s) to t in [0, n): one, or two when t is exactly k + 1/2.
inline int nearest_ints(double t, int32_t n, int32_t (&out)[2]) {
  double f = floor_exact(t);
  int32_t lo = (int32_t)f;
  double fr = t - f;
  int k = 0;
  if (fr < 0.5) {
    out[k++] = lo;
  } else if (fr > 0.5) {
    out[k++] = lo + 1;
  } else {
    out[k++] = lo;
    out[k++] = lo + 1;
  }
  int m = 0;
  for (int i = 0; i < k; ++i)
    if (out[i] >= 0 && out[i] < n) out[m++] = out[i];
  return m;
}

// The 3 x 3 block of sites around the unique nearest site (cx, cy) of the
// target.  Every site outside the block is more than 1.5 away from the
// target along one axis, so its cost is at least 2.25 (exact differences,
// monotone rounding); a free site of the block that costs less than that is
// the minimum over the grid.  Visited in tile order with a strict <, so the
// lowest tile wins a tie, as in the reference's scan.  Leaves best / best_t
// at the block's best free site (or unchanged when all nine are taken).
// Bits of columns x0 .. x0 + n - 1 of a row (n <= 57), 0 for columns off
// the grid (the map's bits past W are 0 already).
inline uint64_t window_bits(const uint64_t *row, int32_t x0, int n, int32_t WR) {
  uint64_t m;
  if (x0 >= 0) {
    const int32_t w = x0 >> 6, sh = x0 & 63;
    m = row[w] >> sh;
    if (sh && w + 1 < WR) m |= row[w + 1] << (64 - sh);
  } else {
    m = row[0] << (-x0);
  }
  return m & ((1ull << n) - 1);
}

// The 3 x 3 block around the nearest site (cx, cy), row-major (tile
// order), keeping the first least cost: all nine costs formed and selected
// without branches (a taken or off-grid site counts as infinite).
inline void probe3(const uint64_t *fm, int32_t WR, int32_t W, int32_t H, int32_t cx, int32_t cy, double tx, double ty,
                   double &best, int64_t &best_t, int32_t &bx, int32_t &by) {
  double dx2[3], dy2[3];
  for (int k = 0; k < 3; ++k) {
    const double dx = (double)(cx - 1 + k) - tx, dy = (double)(cy - 1 + k) - ty;
    dx2[k] = dx * dx;
    dy2[k] = dy * dy;
  }
  for (int a = 0; a < 3; ++a) {
    const int32_t y = cy - 1 + a;
    if (y < 0 || y >= H) continue;
    const uint64_t m = window_bits(fm + (size_t)y * WR, cx - 1, 3, WR);
    for (int k = 0; k < 3; ++k) {
      const double cost = ((m >> k) & 1) ? dx2[k] + dy2[a] : INFINITY;
      const bool take = cost < best;
      best = take ? cost : best;
      best_t = take ? (int64_t)y * W + cx - 1 + k : best_t;
      bx = take ? cx - 1 + k : bx;
      by = take ? y : by;
    }
  }
}

// The (2k+1)^2 block around the unique nearest site (cx, cy): in each of
// its rows the nearest free site of the block left of or at floor(tx) and
// right of it (the rest of the row's part in the block costs more).  A site
// outside the block costs at least (k + 1/2)^2; the caller trusts the
// result only below that.  Keeps the lower (cost, tile).
inline void probe_window(const uint64_t *fm, int32_t WR, int32_t W, int32_t H, int32_t cx, int32_t cy, int32_t fx0,
                         int k, double tx, double ty, double &best, int64_t &best_t) {
  const int32_t x0 = cx - k, n = 2 * k + 1, off = fx0 - x0;  // off in [k - 1, k]
  const uint64_t lmask = (2ull << off) - 1;
  auto row = [&](int32_t y) {
    const uint64_t m = window_bits(fm + (size_t)y * WR, x0, n, WR);
    const double dy = (double)y - ty, dy2 = dy * dy;
    const uint64_t ml = m & lmask, mr = m & ~lmask;
    if (ml) {
      const int32_t x = x0 + 63 - __builtin_clzll(ml);
      const double dx = (double)x - tx, c = dx * dx + dy2;
      const int64_t t = (int64_t)y * W + x;
      if (c < best || (c == best && t < best_t)) { best = c; best_t = t; }
    }
    if (mr) {
      const int32_t x = x0 + __builtin_ctzll(mr);
      const double dx = (double)x - tx, c = dx * dx + dy2;
      const int64_t t = (int64_t)y * W + x;
      if (c < best || (c == best && t < best_t)) { best = c; best_t = t; }
    }
  };
  // Rows outward from cy; a side stops once dy^2 exceeds the best cost (no
  // row past it can win or tie).  The (cost, tile) compare makes the order
  // of the rows immaterial.
  row(cy);
  for (int32_t d = 1; d <= k; ++d) {
    const int32_t yd = cy - d, yu = cy + d;
    const double dd = (double)yd - ty, du = (double)yu - ty;
    const bool okd = yd >= 0 && dd * dd <= best, oku = yu < H && du * du <= best;
    if (!okd && !oku) break;  // both sides done: |dy| only grows, best only shrinks
    if (okd) row(yd);
    if (oku) row(yu);
  }
}

// One unit cell's search over the rows (see Legalizer::run).
struct RowSearch {
  const uint64_t *fm;
  const uint64_t *sm;
  int32_t *lc, *rc;
  int32_t W, H, WR;
  double tx, ty;
  int32_t fx0;
  bool cacheable;
  double best;
  int64_t best_t;
};

// The row's two candidates: from the cache when its entry covers fx0, else
// from the bitmap (and then cached).
inline void row_candidates(RowSearch &s, int32_t row, int32_t &l, int32_t &rr) {
  if (s.cacheable && s.lc[row] <= s.fx0 && s.fx0 < s.rc[row]) {
    l = s.lc[row];
    rr = s.rc[row] < s.W ? s.rc[row] : -1;
    return;
  }
  const uint64_t *r = s.fm + (size_t)row * s.WR;
  const uint64_t *rs = s.sm ? s.sm + row : nullptr;
  l = free_at_or_left(r, rs, std::min(s.fx0, s.W - 1));
  rr = free_at_or_right(r, rs, s.fx0 + 1, s.W, s.WR);
  if (s.cacheable) {
    s.lc[row] = l;
    s.rc[row] = rr >= 0 ? rr : s.W;
  }
}

inline void consider(RowSearch &s, double cost, int64_t t) {
  if (cost < s.best || (cost == s.best && t < s.best_t)) {
    s.best = cost;
    s.best_t = t;
  }
}

inline void scan_row(RowSearch &s, int32_t row) {
  const double dy = (double)row - s.ty;
  const double dy2 = dy * dy;
  int32_t l, rr;
  row_candidates(s, row, l, rr);
  if (l >= 0) {
    const double dx = (double)l - s.tx;
    consider(s, dx * dx + dy2, (int64_t)row * s.W + l);
  }
  if (rr >= 0) {
    const double dx = (double)rr - s.tx;
    consider(s, dx * dx + dy2, (int64_t)row * s.W + rr);
  }
}

// Whether a side whose next row is `row` is finished: off the grid, or
// dy^2 above the best cost (no row beyond can win or tie).
inline bool side_done(const RowSearch &s, int32_t row) {
  if (row < 0 || row >= s.H) return true;
  const double dy = (double)row - s.ty;
  return s.best_t >= 0 && dy * dy > s.best;
}

// Rows outward from cy, one at a time.
__attribute__((noinline)) void search_rows(RowSearch &s, int32_t cy) {
  scan_row(s, cy);
  bool up = true, down = true;
  for (int32_t d = 1; up || down; ++d) {
    if (down) {
      if (side_done(s, cy - d)) down = false;
      else scan_row(s, cy - d);
    }
    if (up) {
      if (side_done(s, cy + d)) up = false;
      else scan_row(s, cy + d);
    }
  }
}

// The same search, four consecutive rows per step where they are all on the
// grid (AVX2).  The caches of the four rows are checked together and
// refreshed one by one only where stale; then the eight candidates' costs
// are formed with 256-bit doubles as the scalar code forms them (separate
// multiply and add; the target has no FMA, so nothing is contracted), and
// only when one of them can improve on or tie the best does the block go
// through the scalar comparison with its tile tie-break.  Rows beyond a
// side's stopping row cannot win or tie, so visiting them changes nothing:
// the result is the minimum over all rows, as in the one-row search.
__attribute__((target("avx2"))) inline void rows4(RowSearch &s, int32_t r0) {
  const __m128i fxv = _mm_set1_epi32(s.fx0);
  __m128i l = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s.lc + r0));
  __m128i r = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s.rc + r0));
  // stale: lc > fx0 or rc <= fx0
  const __m128i stale =
      _mm_or_si128(_mm_cmpgt_epi32(l, fxv), _mm_cmpgt_epi32(_mm_add_epi32(fxv, _mm_set1_epi32(1)), r));
  if (_mm_movemask_epi8(stale)) {
    // Refresh only the rows still within reach; a row whose dy^2 exceeds
    // the best cost cannot win or tie, so it leaves the block instead.
    alignas(16) int32_t la[4], ra[4];
    for (int32_t k = 0; k < 4; ++k) {
      const int32_t row = r0 + k;
      const double d = (double)row - s.ty;
      if (s.best_t >= 0 && d * d > s.best) {
        la[k] = -1;
        ra[k] = s.W;
      } else {
        int32_t a, b;
        row_candidates(s, row, a, b);
        la[k] = a;
        ra[k] = b >= 0 ? b : s.W;
      }
    }
    l = _mm_load_si128(reinterpret_cast<const __m128i *>(la));
    r = _mm_load_si128(reinterpret_cast<const __m128i *>(ra));
  }
  const __m256d txv = _mm256_set1_pd(s.tx);
  const __m256d dy = _mm256_sub_pd(_mm256_cvtepi32_pd(_mm_add_epi32(_mm_set1_epi32(r0), _mm_setr_epi32(0, 1, 2, 3))),
                                   _mm256_set1_pd(s.ty));
  const __m256d dy2 = _mm256_mul_pd(dy, dy);
  const __m256d dxl = _mm256_sub_pd(_mm256_cvtepi32_pd(l), txv);
  const __m256d dxr = _mm256_sub_pd(_mm256_cvtepi32_pd(r), txv);
  const __m256d cl = _mm256_add_pd(_mm256_mul_pd(dxl, dxl), dy2);
  const __m256d cr = _mm256_add_pd(_mm256_mul_pd(dxr, dxr), dy2);
  const __m256d okl = _mm256_castsi256_pd(_mm256_cvtepi32_epi64(_mm_cmpgt_epi32(l, _mm_set1_epi32(-1))));
  const __m256d okr = _mm256_castsi256_pd(_mm256_cvtepi32_epi64(_mm_cmplt_epi32(r, _mm_set1_epi32(s.W))));
  const __m256d bv = _mm256_set1_pd(s.best);
  const __m256d le = _mm256_or_pd(_mm256_and_pd(okl, _mm256_cmp_pd(cl, bv, _CMP_LE_OQ)),
                                  _mm256_and_pd(okr, _mm256_cmp_pd(cr, bv, _CMP_LE_OQ)));
  if (!_mm256_movemask_pd(le)) return;
  alignas(32) double al[4], ar[4];
  _mm256_store_pd(al, cl);
  _mm256_store_pd(ar, cr);
  alignas(16) int32_t li[4], ri[4];
  _mm_store_si128(reinterpret_cast<__m128i *>(li), l);
  _mm_store_si128(reinterpret_cast<__m128i *>(ri), r);
  for (int32_t k = 0; k < 4; ++k) {
    const int64_t row = r0 + k;
    if (li[k] >= 0) consider(s, al[k], row * s.W + li[k]);
    if (ri[k] < s.W) consider(s, ar[k], row * s.W + ri[k]);
  }
}

__attribute__((target("avx2"), noinline)) void search_rows4(RowSearch &s, int32_t cy) {
  scan_row(s, cy);
  bool up = true, down = true;
  int32_t dd = 1, du = 1;
  while (up || down) {
    if (down) {
      const int32_t row = cy - dd;
      if (side_done(s, row)) {
        down = false;
      } else if (row >= 3) {
        rows4(s, row - 3);
        dd += 4;
      } else {
        scan_row(s, row);
        dd += 1;
      }
    }
    if (up) {
      const int32_t row = cy + du;
      if (side_done(s, row)) {
        up = false;
      } else if (row + 3 < s.H) {
        rows4(s, row);
        du += 4;
      } else {
        scan_row(s, row);
        du += 1;
      }
    }
  }
}
// The same search with AVX-512, eight consecutive rows per step and no
// branch on the candidates: each of the eight lanes keeps the best
// (cost, tile) of the candidates it has seen, updated with the scalar
// code's comparison (lower cost, then lower tile), and the lanes are merged
// at the end.  Costs are formed as in the scalar code (separate multiply and
// add).  A side stops once dy^2 exceeds the best cost found so far, which
// only ever shrinks, so every row that could win or tie is visited.
struct Lanes8 {
  __m512d bc;   // best cost per lane
  __m256i bt;   // its tile (INT32_MAX: none; the eight-row search runs on chips below 2^31 sites)
  __m256i kw;   // k * W for lane k
  double best;  // minimum over the scalar rows (the lanes keep theirs in bc)
};

// Lane update with the tile order taken from the visiting order, so no tile
// compare is needed.  Rows below the target are visited downward (their
// tiles decrease), rows above it upward (tiles increase), and every row
// below has lower tiles than every row above.  So an upward candidate never
// displaces one of equal cost (its tile is higher: strict <) and a downward
// candidate always does (its tile is lower: <=); within a row the left site
// (the lower tile) comes first upward and last downward.  A lane thus keeps
// the lowest tile among its least-cost candidates, as (cost, tile) order
// asks.
template <bool DOWN>
__attribute__((target("avx512f,avx512vl,avx2"))) inline void lane_keep(Lanes8 &L, __m512d c, __m256i t, __mmask8 ok) {
  const __mmask8 u = ok & _mm512_cmp_pd_mask(c, L.bc, DOWN ? _CMP_LE_OQ : _CMP_LT_OQ);
  L.bc = _mm512_mask_blend_pd(u, L.bc, c);
  L.bt = _mm256_mask_blend_epi32(u, L.bt, t);
}

// Per-search constants of rows8.
struct Rows8K {
  __m256i fxv, fx1v, m1, Wv;  // fx0, fx0 + 1, -1, W in eight lanes
  __m512d txv;
};

// Rows r0 .. r0 + 7: dy holds (r0 + k) - ty and base (r0 + k) W per lane
// (the caller steps both by 8 rows per call, exactly).
template <bool DOWN>
__attribute__((target("avx512f,avx512vl,avx2"))) inline void rows8(RowSearch &s, Lanes8 &L, int32_t r0, __m512d dy,
                                                                 __m256i base, const Rows8K &K) {
  __m256i l = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s.lc + r0));
  __m256i r = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s.rc + r0));
  if (_mm256_cmpgt_epi32_mask(l, K.fxv) | _mm256_cmpgt_epi32_mask(K.fx1v, r)) {
    // Refresh only the rows still within reach (as in rows4).
    const double bnow = std::min(L.best, _mm512_reduce_min_pd(L.bc));
    alignas(32) int32_t la[8], ra[8];
    for (int32_t k = 0; k < 8; ++k) {
      const int32_t row = r0 + k;
      const double d = (double)row - s.ty;
      if (d * d > bnow) {
        la[k] = -1;
        ra[k] = s.W;
      } else {
        int32_t a, b;
        row_candidates(s, row, a, b);
        la[k] = a;
        ra[k] = b >= 0 ? b : s.W;
      }
    }
    l = _mm256_load_si256(reinterpret_cast<const __m256i *>(la));
    r = _mm256_load_si256(reinterpret_cast<const __m256i *>(ra));
  }
  const __m512d dy2 = _mm512_mul_pd(dy, dy);
  const __mmask8 okl = _mm256_cmpgt_epi32_mask(l, K.m1);
  const __m512d dxl = _mm512_sub_pd(_mm512_cvtepi32_pd(l), K.txv);
  const __m512d cl = _mm512_add_pd(_mm512_mul_pd(dxl, dxl), dy2);
  const __m256i tl = _mm256_add_epi32(base, l);
  const __mmask8 okr = _mm256_cmpgt_epi32_mask(K.Wv, r);
  const __m512d dxr = _mm512_sub_pd(_mm512_cvtepi32_pd(r), K.txv);
  const __m512d cr = _mm512_add_pd(_mm512_mul_pd(dxr, dxr), dy2);
  const __m256i tr = _mm256_add_epi32(base, r);
  if (DOWN) {
    lane_keep<true>(L, cr, tr, okr);
    lane_keep<true>(L, cl, tl, okl);
  } else {
    lane_keep<false>(L, cl, tl, okl);
    lane_keep<false>(L, cr, tr, okr);
  }
}

// Whether a row at squared distance d2 from the target can no longer win or
// tie: d2 exceeds the best of the scalar rows or of some lane (no horizontal
// minimum needed).
__attribute__((target("avx512f,avx512vl,avx2"))) inline bool past(const Lanes8 &L, double d2) {
  return d2 > L.best || _mm512_cmp_pd_mask(L.bc, _mm512_set1_pd(d2), _CMP_LT_OQ) != 0;
}

__attribute__((target("avx512f,avx512vl,avx2"), noinline)) void search_rows8(RowSearch &s, int32_t cy) {
  scan_row(s, cy);
  const int32_t W32 = s.W;
  Lanes8 L{_mm512_set1_pd(INFINITY), _mm256_set1_epi32(INT32_MAX),
           _mm256_setr_epi32(0, W32, 2 * W32, 3 * W32, 4 * W32, 5 * W32, 6 * W32, 7 * W32), s.best};
  const Rows8K K{_mm256_set1_epi32(s.fx0), _mm256_set1_epi32(s.fx0 + 1), _mm256_set1_epi32(-1),
                 _mm256_set1_epi32(s.W), _mm512_set1_pd(s.tx)};
  const __m256i iota = _mm256_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7);
  const __m512d tyv = _mm512_set1_pd(s.ty);
  // lanes of the next call each way: rows cy - 8 .. cy - 1 down, cy + 1 ..
  // cy + 8 up, then eight rows further per call
  __m512d dyd = _mm512_sub_pd(_mm512_cvtepi32_pd(_mm256_add_epi32(_mm256_set1_epi32(cy - 8), iota)), tyv);
  __m512d dyu = _mm512_sub_pd(_mm512_cvtepi32_pd(_mm256_add_epi32(_mm256_set1_epi32(cy + 1), iota)), tyv);
  __m256i bsd = _mm256_add_epi32(_mm256_set1_epi32((cy - 8) * W32), L.kw);
  __m256i bsu = _mm256_add_epi32(_mm256_set1_epi32((cy + 1) * W32), L.kw);
  const __m512d step = _mm512_set1_pd(8.0);
  const __m256i stepw = _mm256_set1_epi32(8 * W32);
  bool up = true, down = true;
  int32_t dd = 1, du = 1;
  while (up || down) {
    if (down) {
      const int32_t row = cy - dd;
      const double d = (double)row - s.ty;
      if (row < 0 || past(L, d * d)) {
        down = false;
      } else if (row >= 7) {
        rows8<true>(s, L, row - 7, dyd, bsd, K);
        dyd = _mm512_sub_pd(dyd, step);
        bsd = _mm256_sub_epi32(bsd, stepw);
        dd += 8;
      } else {
        scan_row(s, row);
        L.best = std::min(L.best, s.best);
        dd += 1;
      }
    }
    if (up) {
      const int32_t row = cy + du;
      const double d = (double)row - s.ty;
      if (row >= s.H || past(L, d * d)) {
        up = false;
      } else if (row + 7 < s.H) {
        rows8<false>(s, L, row, dyu, bsu, K);
        dyu = _mm512_add_pd(dyu, step);
        bsu = _mm256_add_epi32(bsu, stepw);
        du += 8;
      } else {
        scan_row(s, row);
        L.best = std::min(L.best, s.best);
        du += 1;
      }
    }
  }
  alignas(64) double cs[8];
  alignas(32) int32_t ts[8];
  _mm512_store_pd(cs, L.bc);
  _mm256_store_si256(reinterpret_cast<__m256i *>(ts), L.bt);
  for (int k = 0; k < 8; ++k)
    if (ts[k] != INT32_MAX) consider(s, cs[k], (int64_t)ts[k]);
}
}  // namespace

eplace_status Legalizer::run(const float *x, const float *y, size_t stride, int32_t *site_x, int32_t *site_y,
                             double *displacement) {
  const int32_t W = hp_.W, H = hp_.H, WR = base_.WR;
  std::copy(base_.free0.begin(), base_.free0.end(), free_.begin());
  std::copy(base_.sum0.begin(), base_.sum0.end(), sum_.begin());
  uint64_t *fm = free_.data();
  uint64_t *sm = sum_.empty() ? nullptr : sum_.data();
  std::fill(lc_.begin(), lc_.end(), INT32_MAX);  // every row's cache entry dead
  int32_t *lc = lc_.data(), *rc = rc_.data();
  double total = 0.0;
  for (uint32_t i : base_.order) {
    const double tx = (double)x[i * stride], ty = (double)y[i * stride];
    const int w = hp_.cw[i], h = hp_.ch[i];
    double best = INFINITY;
    int64_t best_t = -1;
    int32_t bx = -1, by = -1;  // best_t's site when known without a division
    if (w == 1 && h == 1) {
      // fast path: a free site of minimum cost over the whole grid.  With
      // both fractions away from 1/2 the nearest site is unique; otherwise
      // the tied nearest sites are tried in tile order.
      const double flx = floor_exact(tx), fly = floor_exact(ty);
      const double frx = tx - flx, fry = ty - fly;
      const bool inside = tx >= 0.0 && tx <= (double)(W - 1) && ty >= 0.0 && ty <= (double)(H - 1);
      bool resolved = false;
      // The block probes: 3 x 3, then the (2 kWin + 1)^2 block.
      constexpr int kWin = 4;
      if (inside && frx != 0.5 && fry != 0.5) {
        const int32_t nx = (int32_t)flx + (frx > 0.5 ? 1 : 0), ny = (int32_t)fly + (fry > 0.5 ? 1 : 0);
        if (is_free(fm, WR, nx, ny)) {
          const double dx = (double)nx - tx, dy = (double)ny - ty;
          best = dx * dx + dy * dy;
          best_t = (int64_t)ny * W + nx;
          bx = nx;
          by = ny;
          resolved = true;
        } else {
          probe3(fm, WR, W, H, nx, ny, tx, ty, best, best_t, bx, by);
          resolved = best < 2.25;
          // Skip the larger block when the cell's own row is known to have
          // no free site within it (a cell deep in a pile): the row search
          // follows either way.
          const int32_t fx = (int32_t)flx;
          const bool deep = lc[ny] <= fx && fx < rc[ny] && fx - lc[ny] > kWin && rc[ny] - fx > kWin;
          if (!resolved && !deep) {
            probe_window(fm, WR, W, H, nx, ny, fx, kWin, tx, ty, best, best_t);
            bx = -1;
            resolved = best < (kWin + 0.5) * (kWin + 0.5);  // exact product
          }
        }
      } else {
        int32_t xs[2], ys[2];
        const int nx = (tx >= 0.0 && tx <= (double)(W - 1)) ? nearest_ints(tx, W, xs) : 0;
        const int ny = (ty >= 0.0 && ty <= (double)(H - 1)) ? nearest_ints(ty, H, ys) : 0;
        for (int a = 0; a < ny && best_t < 0; ++a)
          for (int b = 0; b < nx; ++b)
            if (is_free(fm, WR, xs[b], ys[a])) {
              const double dx = (double)xs[b] - tx, dy = (double)ys[a] - ty;
              best = dx * dx + dy * dy;
              best_t = (int64_t)ys[a] * W + xs[b];
              bx = xs[b];
              by = ys[a];
              break;
            }
        resolved = best_t >= 0;
      }
      if (!resolved) {
        int32_t cy = (int32_t)floor_exact(ty + 0.5);
        cy = std::min(std::max(cy, 0), H - 1);
        const int32_t fx0 = (int32_t)floor_exact(tx);
        // Per-row candidate cache: (lc, rc) are the nearest free sites left
        // of / right of an earlier query position in this row, with every
        // site strictly between them taken.  For any fx0 with
        // lc <= fx0 < rc they are again this query's two candidates, so a
        // cell of a crowded region (whose neighbours in the order target the
        // same region) reads them instead of searching the bitmap.  A row's
        // entry dies when one of its two sites is taken.
        RowSearch rs{fm, sm, lc, rc, W, H, WR, tx, ty, fx0, fx0 >= 0 && fx0 <= W - 1, best, best_t};
        if (simd512_ && rs.cacheable) search_rows8(rs, cy);
        else if (simd_ && rs.cacheable) search_rows4(rs, cy);
        else search_rows(rs, cy);
        best = rs.best;
        best_t = rs.best_t;
        bx = -1;
      }
    } else {
      // Macro: anchor rows outward from the target anchor row.  In anchor
      // row ay, anchor a is valid when sites [a, a + w) are free in rows
      // ay .. ay + h - 1: AND the rows' free words, then AND w shifted copies
      // (carrying bits in from the next word).  The best anchor of the row is
      // the nearest valid bit left of or right of the target anchor column.
      const double ox = 0.5 * (w - 1), oy = 0.5 * (h - 1);
      const int32_t AW = W - w + 1, AH = H - h + 1;
      if (AW > 0 && AH > 0) {
        const double ux = tx - ox, uy = ty - oy;  // target anchor
        const int32_t cy = std::min(std::max((int32_t)floor_exact(uy + 0.5), 0), AH - 1);
        const int32_t fa = std::min(std::max((int32_t)floor_exact(ux), -1), AW - 1);
        const int32_t lastw = (AW - 1) >> 6;
        auto valid_word = [&](int32_t ay, int32_t j) -> uint64_t {
          uint64_t m = ~0ull, mn = ~0ull;
          for (int dy = 0; dy < h; ++dy) {
            const uint64_t *r = fm + (size_t)(ay + dy) * WR;
            m &= r[j];
            mn &= (j + 1 < WR) ? r[j + 1] : 0ull;
          }
          uint64_t v = m;
          for (int k = 1; k < w; ++k) v &= (m >> k) | (mn << (64 - k));
          if (j == lastw && ((AW - 1) & 63) != 63) v &= (2ull << ((AW - 1) & 63)) - 1;
          return v;
        };
        auto scan_anchor_row = [&](int32_t ay) {
          const double dy = ((double)ay + oy) - ty;
          const double dy2 = dy * dy;
          auto consider = [&](int32_t a) {
            const double dx = ((double)a + ox) - tx, cost = dx * dx + dy2;
            const int64_t t = (int64_t)ay * W + a;
            if (cost < best || (cost == best && t < best_t)) {
              best = cost;
              best_t = t;
            }
          };
          // The word holding fa serves both sides when fa + 1 falls in it too.
          const int32_t jf = fa >> 6;
          const uint64_t vf = fa >= 0 ? valid_word(ay, jf) : 0ull;
          if (fa >= 0) {  // nearest valid anchor <= fa
            int32_t j = jf;
            uint64_t v = vf & (((fa & 63) == 63) ? ~0ull : ((2ull << (fa & 63)) - 1));
            while (true) {
              if (v) {
                consider((j << 6) + 63 - __builtin_clzll(v));
                break;
              }
              if (--j < 0) break;
              v = valid_word(ay, j);
            }
          }
          if (fa + 1 <= AW - 1) {  // nearest valid anchor >= fa + 1
            const int32_t p = fa + 1;
            int32_t j = p >> 6;
            uint64_t v = (fa >= 0 && j == jf ? vf : valid_word(ay, j)) & (~0ull << (p & 63));
            while (true) {
              if (v) {
                consider((j << 6) + __builtin_ctzll(v));
                break;
              }
              if (++j > lastw) break;
              v = valid_word(ay, j);
            }
          }
        };
        scan_anchor_row(cy);
        bool up = true, down = true;
        for (int32_t d = 1; up || down; ++d) {
          if (down) {
            const int32_t row = cy - d;
            if (row < 0) {
              down = false;
            } else {
              const double dy = ((double)row + oy) - ty;
              if (best_t >= 0 && dy * dy > best) down = false;
              else scan_anchor_row(row);
            }
          }
          if (up) {
            const int32_t row = cy + d;
            if (row >= AH) {
              up = false;
            } else {
              const double dy = ((double)row + oy) - ty;
              if (best_t >= 0 && dy * dy > best) up = false;
              else scan_anchor_row(row);
            }
          }
        }
      }
    }
    if (best_t < 0) return EPLACE_ERR_NO_BELS;
    if (bx < 0) {
      bx = (int32_t)(best_t % W);
      by = (int32_t)(best_t / W);
    }
    if (w == 1 && h == 1) {
      // A unit cell takes one site.  When it is one of its row's two cached
      // candidates, the next free site past it (on the same side) becomes
      // the candidate: every site between the two stays taken, so the entry
      // stays valid and the next cell of a pile reads it instead of
      // searching the row again.
      uint64_t *row = fm + (size_t)by * WR;
      row[bx >> 6] &= ~(1ull << (bx & 63));
      if (sm && !row[bx >> 6]) sm[by] &= ~(1ull << (bx >> 6));
      if (lc[by] != INT32_MAX) {
        if (bx == lc[by]) {
          lc[by] = free_at_or_left(row, sm ? sm + by : nullptr, bx - 1);
        } else if (bx == rc[by]) {
          const int32_t r2 = free_at_or_right(row, sm ? sm + by : nullptr, bx + 1, W, WR);
          rc[by] = r2 >= 0 ? r2 : W;
        }
      }
    } else {
      for (int dy = 0; dy < h; ++dy)
        for (int dx = 0; dx < w; ++dx) {
          const int32_t xx = bx + dx;
          uint64_t &word = fm[(size_t)(by + dy) * WR + (xx >> 6)];
          word &= ~(1ull << (xx & 63));
          if (sm && !word) sm[by + dy] &= ~(1ull << (xx >> 6));
          if (xx == lc[by + dy] || xx == rc[by + dy]) lc[by + dy] = INT32_MAX;
        }
    }
    site_x[i] = bx;
    site_y[i] = by;
    total += best;
  }
  if (displacement) *displacement = total;
  return EPLACE_OK;
}

// total_hpwl (metrics/wirelength.rs:10-51): integer bbox of driver + users;
// nets without a driver or without users contribute 0.  A macro's pins sit
// at anchor + (w-1)/2 (integer), which is the BEL itself for a unit cell.
// Pin locations packed per cell, x | y << 16 (the grid fits 16 bits): one
// 4-byte gather per pin from a table that stays in the core's cache.
static const uint32_t *packed_locations(const HostProblem &hp, const int32_t *sx, const int32_t *sy) {
  thread_local std::vector<uint32_t> loc;
  loc.resize((size_t)hp.N + hp.F);
  for (uint32_t c = 0; c < hp.N; ++c)
    loc[c] = (uint32_t)(sx[c] + (hp.cw[c] - 1) / 2) | ((uint32_t)(sy[c] + (hp.ch[c] - 1) / 2) << 16);
  for (uint32_t f = 0; f < hp.F; ++f) loc[hp.N + f] = (uint32_t)hp.fx[f] | ((uint32_t)hp.fy[f] << 16);
  return loc.data();
}

void build_hpwl_table(HostProblem &hp) {
  std::vector<uint32_t> count((size_t)hp.max_degree + 1, 0);
  size_t pins = 0;
  for (uint32_t n = 0; n < hp.NN; ++n) {
    const uint32_t d = hp.net_off[n + 1] - hp.net_off[n];
    if (hp.has_driver[n] && d >= 2) {
      ++count[d];
      pins += d;
    }
  }
  std::vector<size_t> at(count.size(), 0);
  hp.hpwl_runs.clear();
  for (size_t d = 2, k = 0; d < count.size(); ++d) {
    at[d] = k;
    k += count[d] * d;
    if (count[d]) hp.hpwl_runs.emplace_back((uint32_t)d, count[d]);
  }
  hp.hpwl_pins.resize(pins);
  for (uint32_t n = 0; n < hp.NN; ++n) {
    const uint32_t b = hp.net_off[n], d = hp.net_off[n + 1] - b;
    if (!hp.has_driver[n] || d < 2) continue;
    std::copy(hp.pin_cell.begin() + b, hp.pin_cell.begin() + b + d, hp.hpwl_pins.begin() + at[d]);
    at[d] += d;
  }
  hp.hpwl_table = true;
}

int64_t hpwl_host(const HostProblem &hp, const int32_t *sx, const int32_t *sy, int threads) {
  int64_t total = 0;
  if (hp.W > 65536 || hp.H > 65536) {
    // Wide grids: the footprint and binding arrays directly.
    for (uint32_t n = 0; n < hp.NN; ++n) {
      uint32_t b = hp.net_off[n], e = hp.net_off[n + 1];
      if (!hp.has_driver[n] || e - b < 2) continue;
      int32_t x0 = INT32_MAX, x1 = INT32_MIN, y0 = INT32_MAX, y1 = INT32_MIN;
      for (uint32_t q = b; q < e; ++q) {
        uint32_t c = hp.pin_cell[q];
        int32_t lx, ly;
        if (c < hp.N) {
          lx = sx[c] + (hp.cw[c] - 1) / 2;
          ly = sy[c] + (hp.ch[c] - 1) / 2;
        } else {
          lx = hp.fx[c - hp.N];
          ly = hp.fy[c - hp.N];
        }
        x0 = std::min(x0, lx);
        x1 = std::max(x1, lx);
        y0 = std::min(y0, ly);
        y1 = std::max(y1, ly);
      }
      total += (int64_t)(x1 - x0) + (int64_t)(y1 - y0);
    }
    return total;
  }
  const uint32_t *L = packed_locations(hp, sx, sy);
  // bounding box of the d pins at p (d >= 2)
  auto box = [L](const uint32_t *p, uint32_t d) -> int64_t {
    if (d == 2) {
      const uint32_t v0 = L[p[0]], v1 = L[p[1]];
      const int32_t dx = (int32_t)(v0 & 0xffffu) - (int32_t)(v1 & 0xffffu);
      const int32_t dy = (int32_t)(v0 >> 16) - (int32_t)(v1 >> 16);
      return (int64_t)std::abs(dx) + std::abs(dy);
    }
    uint32_t x0 = 0xffffu, x1 = 0, y0 = 0xffffu, y1 = 0;
    for (uint32_t q = 0; q < d; ++q) {
      const uint32_t v = L[p[q]];
      x0 = std::min(x0, v & 0xffffu);
      x1 = std::max(x1, v & 0xffffu);
      y0 = std::min(y0, v >> 16);
      y1 = std::max(y1, v >> 16);
    }
    return (int64_t)(x1 - x0) + (int64_t)(y1 - y0);
  };
  if (hp.hpwl_table) {
    // Nets grouped by degree: the inner trip count repeats from net to net.
    // With threads > 1 the table is cut into that many pieces of about equal
    // pin count, at net boundaries; the sums are integers, so the total does
    // not depend on the cut.
    struct Piece {
      const uint32_t *p;
      uint32_t d, nets;
    };
    const int nt = std::max(1, std::min(threads, 16));
    std::vector<std::vector<Piece>> parts((size_t)nt);
    {
      const size_t per = (hp.hpwl_pins.size() + nt - 1) / nt;
      const uint32_t *p = hp.hpwl_pins.data();
      size_t filled = 0;
      int t = 0;
      for (const auto &run : hp.hpwl_runs) {
        uint32_t d = run.first, left = run.second;
        while (left) {
          const size_t room = (size_t)(t + 1) * per > filled ? (size_t)(t + 1) * per - filled : 0;
          uint32_t take = (uint32_t)std::min<size_t>(left, std::max<size_t>(1, (room + d - 1) / d));
          if (t == nt - 1) take = left;
          parts[(size_t)t].push_back(Piece{p, d, take});
          p += (size_t)take * d;
          filled += (size_t)take * d;
          left -= take;
          if (t < nt - 1 && filled >= (size_t)(t + 1) * per) ++t;
        }
      }
    }
    auto sum = [&](const std::vector<Piece> &ps) {
      int64_t s = 0;
      for (const Piece &pc : ps) {
        const uint32_t *p = pc.p;
        for (uint32_t k = 0; k < pc.nets; ++k, p += pc.d) s += box(p, pc.d);
      }
      return s;
    };
    if (nt == 1) return sum(parts[0]);
    std::vector<int64_t> part((size_t)nt, 0);
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) {
      try {
        th.emplace_back([&, t] { part[(size_t)t] = sum(parts[(size_t)t]); });
      } catch (const std::system_error &) {  // no thread to be had: this one sums the piece
        part[(size_t)t] = sum(parts[(size_t)t]);
      }
    }
    part[0] = sum(parts[0]);
    for (auto &x : th) x.join();
    for (int64_t v : part) total += v;
    return total;
  }
  for (uint32_t n = 0; n < hp.NN; ++n) {
    const uint32_t b = hp.net_off[n], d = hp.net_off[n + 1] - b;
    if (hp.has_driver[n] && d >= 2) total += box(hp.pin_cell.data() + b, d);
  }
  return total;
}

// ---------------------------------------------------------------------------
// Synthetic netlist generator.  Independent splitmix64 streams for macro
// sizes, degrees, pins and pad nets, so the pin count is known from the
// degree stream alone.
//   degree: 2 (p .60), U[3,5] (.25), U[6,20] (.12), U[21,200] (.03), <= cells
//   pins: a uniformly chosen home cluster of `cluster_size` consecutive
//         cells supplies each pin with probability `locality`, otherwise
//         any cell; no cell twice in one net; pin 0 is the driver
//   pads: evenly spaced along the perimeter walk, each joins one uniformly
//         chosen net as a user (appended after the net's cell pins)
// ---------------------------------------------------------------------------
namespace {
struct SplitMix {
  uint64_t s;
  explicit SplitMix(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  uint32_t below(uint32_t n) { return (uint32_t)(next() % n); }
};

uint32_t draw_degree(SplitMix &r, uint32_t ncells) {
  double u = r.uniform();
  uint32_t d;
  if (u < 0.60) d = 2;
  else if (u < 0.85) d = 3 + r.below(3);
  else if (u < 0.97) d = 6 + r.below(15);
  else d = 21 + r.below(180);
  return std::min(d, ncells);
}
}  // namespace

eplace_status synth(const eplace_synth_spec &sp, eplace_synth_info *info, uint8_t *cw, uint8_t *ch,
                    int32_t *fx, int32_t *fy, uint32_t *net_off, uint32_t *pin_cell) {
  if (sp.width <= 0 || sp.height <= 0 || sp.cluster_size == 0) return EPLACE_ERR_INVALID;
  if (sp.num_pads > 0 && sp.width < 2) return EPLACE_ERR_INVALID;
  if (sp.num_nets > 0 && sp.num_cells < 2 && sp.num_pads == 0) return EPLACE_ERR_INVALID;
  const uint32_t N = sp.num_cells, NN = sp.num_nets, F = sp.num_pads;
  SplitMix rdeg(sp.seed ^ 0x1d8e4e27c47d124full);
  SplitMix rpin(sp.seed ^ 0x6a09e667f3bcc909ull);
  SplitMix rmac(sp.seed ^ 0xbb67ae8584caa73bull);
  SplitMix rpad(sp.seed ^ 0x3c6ef372fe94f82bull);
  std::vector<uint32_t> deg(NN), pads_per_net(NN, 0), pad_net(F);
  uint64_t total = 0;
  uint32_t maxdeg = 0;
  for (uint32_t n = 0; n < NN; ++n) {
    deg[n] = N >= 2 ? draw_degree(rdeg, N) : 0;
  }
  for (uint32_t f = 0; f < F; ++f) {
    pad_net[f] = NN ? rpad.below(NN) : 0;
    if (NN) pads_per_net[pad_net[f]]++;
  }
  for (uint32_t n = 0; n < NN; ++n) {
    total += deg[n] + pads_per_net[n];
    maxdeg = std::max(maxdeg, deg[n] + pads_per_net[n]);
  }
  if (total > 0xffffffffull) return EPLACE_ERR_INVALID;
  if (info) {
    info->num_pins = (uint32_t)total;
    info->max_degree = maxdeg;
  }
  if (!net_off) return EPLACE_OK;  // size query
  // footprints
  for (uint32_t i = 0; i < N; ++i) {
    uint8_t s = 1;
    if (sp.macro_fraction > 0 && rmac.uniform() < sp.macro_fraction) {
      uint32_t lo = std::max(1u, sp.macro_min), hi = std::max(lo, sp.macro_max);
      s = (uint8_t)(lo + rmac.below(hi - lo + 1));
    }
    if (cw) cw[i] = s;
    if (ch) ch[i] = s;
  }
  // pads along the perimeter walk
  const int64_t W = sp.width, H = sp.height;
  const int64_t L = (H >= 2) ? 2 * W + 2 * H - 4 : W;
  for (uint32_t f = 0; f < F; ++f) {
    int64_t p = (int64_t)((uint64_t)f * (uint64_t)L / (uint64_t)F);
    int64_t x, y;
    if (p < W) { x = p; y = 0; }
    else if (p < W + H - 1) { x = W - 1; y = p - W + 1; }
    else if (p < 2 * W + H - 2) { x = W - 2 - (p - (W + H - 1)); y = H - 1; }
    else { x = 0; y = H - 2 - (p - (2 * W + H - 2)); }
    fx[f] = (int32_t)x;
    fy[f] = (int32_t)y;
  }
  // nets
  const uint32_t cs = sp.cluster_size;
  const uint32_t nclusters = N ? (N + cs - 1) / cs : 0;
  std::vector<uint32_t> pad_cursor(NN, 0);
  net_off[0] = 0;
  for (uint32_t n = 0; n < NN; ++n) net_off[n + 1] = net_off[n] + deg[n] + pads_per_net[n];
  for (uint32_t n = 0; n < NN; ++n) {
    uint32_t *out = pin_cell + net_off[n];
    uint32_t d = deg[n];
    if (d > 0) {
      uint32_t home = rpin.below(nclusters);
      uint32_t lo = home * cs, sz = std::min(cs, N - lo);
      for (uint32_t k = 0; k < d; ++k) {
        uint32_t c = 0;
        for (int attempt = 0;; ++attempt) {
          bool local = attempt < 64 && rpin.uniform() < sp.locality;
          c = local ? lo + rpin.below(sz) : rpin.below(N);
          bool dup = false;
          for (uint32_t j = 0; j < k; ++j)
            if (out[j] == c) { dup = true; break; }
          if (!dup) break;
        }
        out[k] = c;
      }
    }
  }
  for (uint32_t f = 0; f < F && NN > 0; ++f) {  // with no nets, pads join none
    uint32_t n = pad_net[f];
    pin_cell[net_off[n] + deg[n] + pad_cursor[n]++] = N + f;
  }
  return EPLACE_OK;
}

}  // namespace eplace
