// kernels.cu -- sm_100a kernels of the ElectroPlace iteration.
//
//   k_wa            WA wirelength gradient (placer/common.rs:205-291,
//                   solver/wa.rs:51-101): nets grouped by degree class, a
//                   fixed lane-group width per class (one thread per net up
//                   to a warp per net), deterministic fixed-point scatter.
//   k_scatter       cell -> bin overlap areas (electro_place/density.rs:54-76),
//                   fixed-point atomics (order independent, bit-reproducible).
//   k_density_final FP64 sum / overflow (density.rs:79-86), FP32 charge map
//                   for the transform, resets the accumulator.
//   k_sgemm         FP32 DCT-matrix GEMMs (density.rs:96-166), spectral
//                   Poisson scaling fused into the second GEMM's epilogue.
//   k_step          field gather + penalty + preconditioner + Barzilai-
//                   Borwein + FISTA + clamp + next look-ahead in one
//                   cooperative kernel (density.rs:171-206,
//                   electro_place/mod.rs:131-173, solver/nesterov.rs:41-101,
//                   :199-218).
//   k_hpwl          integer HPWL (metrics/wirelength.rs:10-51).
#include <cooperative_groups.h>

#include "kernels.cuh"

namespace eplace {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr float kLog2e = 1.4426950408889634f;
// Bound on any spin wait: ~2 s at the B200's clock (clock64 counts SM cycles).
constexpr long long kSpinCycles = 4000000000ll;

__device__ __forceinline__ unsigned long long to_fix(float v) {
  return (unsigned long long)__float2ll_rn(v * 4294967296.0f);
}
__device__ __forceinline__ double from_fix(unsigned long long v) {
  return (double)(long long)v * (1.0 / 4294967296.0);
}

struct OpMax {
  __device__ float operator()(float a, float b) const { return fmaxf(a, b); }
};
struct OpMin {
  __device__ float operator()(float a, float b) const { return fminf(a, b); }
};
struct OpAdd {
  __device__ float operator()(float a, float b) const { return a + b; }
};

template <typename Op>
__device__ __forceinline__ float warp_allreduce(float v, Op op) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Deterministic block sum of K doubles (fixed tree for a fixed block size).
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *smem /* [32*K] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum_d(v[k]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) smem[wid * K + k] = v[k];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double t = lane < nw ? smem[lane * K + k] : 0.0;
      v[k] = warp_sum_d(t);
    }
  }
  __syncthreads();
}

// Deterministic sum over the per-block partials part[stride*b + k], b <
// nblocks, for k < K, by the whole block: thread t reads blocks t, t +
// blockDim, ... with L1-bypassing loads (the partials were written by other
// SMs), then a fixed-tree block reduction; every thread gets the result.
template <int K>
__device__ __forceinline__ void sum_partials(const double *part, int stride, unsigned nblocks,
                                             double (&out)[K], double *smem /* [32*K] */) {
  double v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0.0;
  for (unsigned b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += __ldcg(part + (size_t)stride * b + k);
  block_sum<K>(v, smem);
  __shared__ double bc[K];
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) bc[k] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = bc[k];
  __syncthreads();
}

// Per-axis WA terms with max/min shifts.  The reference shifts by the pin
// mean (wa.rs:58); shifting the positive exponentials by the maximum and the
// negative ones by the minimum leaves value and gradient unchanged and keeps
// every exponential in (0, 1], so FP32 cannot overflow.
//   d_max_i = e+_i/S+ (1 + g (u_i - A+/S+)),  u = x - max
//   d_min_i = e-_i/S- (1 - g (v_i - A-/S-)),  v = x - min
// iSp / iSm are 1/S+ and 1/S- (one reciprocal per segment).
__device__ __forceinline__ float wa_pin_grad(float u, float v, float ep, float em, float iSp, float Ap,
                                             float iSm, float Am, float gamma) {
  const float dmax = ep * iSp * (1.0f + gamma * (u - Ap * iSp));
  const float dmin = em * iSm * (1.0f - gamma * (v - Am * iSm));
  return dmax - dmin;
}

// 2^x for x <= 0 (MUFU.EX2; subnormal results flush to zero, harmless here).
__device__ __forceinline__ float ex2(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Segment max / min over the lanes of `mask` (one mask per segment; the
// segments partition the warp).
__device__ __forceinline__ float seg_max(float v, unsigned mask) {
  float r;
  asm volatile("redux.sync.max.f32 %0, %1, %2;" : "=f"(r) : "f"(v), "r"(mask));
  return r;
}
__device__ __forceinline__ float seg_min(float v, unsigned mask) {
  float r;
  asm volatile("redux.sync.min.f32 %0, %1, %2;" : "=f"(r) : "f"(v), "r"(mask));
  return r;
}

// Segment sum over [head, end) with `steps` shuffle rounds (2^steps >= the
// longest segment of the warp), broadcast from the head lane.
__device__ __forceinline__ float seg_sum(float v, int lane, int end, int head, int steps) {
  for (int s = 0, o = 1; s < steps; ++s, o <<= 1) {
    const float u = __shfl_down_sync(kFull, v, o);
    if (lane + o < end) v += u;
  }
  return __shfl_sync(kFull, v, head);
}

// Reduction over the g lanes of an aligned lane group (g a power of two,
// the same on all lanes of the warp); every lane takes part.  Each xor step
// adds a pair in both orders, and FP32 addition commutes, so all lanes of a
// group get the same bits.
template <typename Op>
__device__ __forceinline__ float group_allreduce(float v, int g, Op op) {
  for (int o = g >> 1; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Nets of one degree class: g lanes per net (32 / g nets per warp), lane l
// of a group holding pins l, l + g, ..., l + (np - 1) g of its net in
// registers (pin ids and positions gathered once; np <= P, uniform over the
// warp).  Max/min and the eight exponential sums are reduced over the group;
// the exponentials are kept for the gradient when P <= 4 and recomputed
// otherwise (register budget).  Nets with fewer than two pins contribute
// nothing (wa.rs:58).
template <int P>
__device__ __forceinline__ void wa_group(const WaArgs &a, const WaClass &cl, int g, int pp, int wi, int lane) {
  constexpr bool kKeep = P <= 4;
  const float kg = a.gamma * kLog2e;
  const int gl = lane & (g - 1);
  const int idx = wi * (32 / g) + lane / g;
  const bool valid = idx < cl.nets;
  // The lane's pp (<= P) pin slots in one vector load: no CSR offsets.
  uint32_t cc[P];
#pragma unroll
  for (int k = 0; k < P; ++k) cc[k] = 0xffffffffu;
  if (valid) {
    const uint32_t *sp = a.slots + cl.slot_base + (long long)idx * (g * pp) + gl * pp;
    if (pp == 2) {
      const uint2 v = *reinterpret_cast<const uint2 *>(sp);
      cc[0] = v.x;
      cc[1] = v.y;
    } else if (pp == 4 || P < 8) {
      const uint4 v = *reinterpret_cast<const uint4 *>(sp);
      cc[0] = v.x;
      cc[1] = v.y;
      cc[P > 2 ? 2 : 0] = P > 2 ? v.z : cc[0];
      cc[P > 3 ? 3 : 0] = P > 3 ? v.w : cc[0];
    } else {
      const uint4 v0 = *reinterpret_cast<const uint4 *>(sp), v1 = *reinterpret_cast<const uint4 *>(sp + 4);
      cc[0] = v0.x;
      cc[1] = v0.y;
      cc[P > 2 ? 2 : 0] = P > 2 ? v0.z : cc[0];
      cc[P > 3 ? 3 : 0] = P > 3 ? v0.w : cc[0];
      cc[P > 4 ? 4 : 0] = P > 4 ? v1.x : cc[0];
      cc[P > 5 ? 5 : 0] = P > 5 ? v1.y : cc[0];
      cc[P > 6 ? 6 : 0] = P > 6 ? v1.z : cc[0];
      cc[P > 7 ? 7 : 0] = P > 7 ? v1.w : cc[0];
    }
  }
  float px[P], py[P];
  float mx = -INFINITY, mn = INFINITY, my = -INFINITY, ny = INFINITY;
#pragma unroll
  for (int k = 0; k < P; ++k) {
    const float2 p = (cc[k] != 0xffffffffu) ? a.pos[cc[k]] : make_float2(0.f, 0.f);
    px[k] = p.x;
    py[k] = p.y;
    if (cc[k] != 0xffffffffu) {
      mx = fmaxf(mx, p.x);
      mn = fminf(mn, p.x);
      my = fmaxf(my, p.y);
      ny = fminf(ny, p.y);
    }
  }
  mx = group_allreduce(mx, g, OpMax());
  mn = group_allreduce(mn, g, OpMin());
  my = group_allreduce(my, g, OpMax());
  ny = group_allreduce(ny, g, OpMin());
  float e[kKeep ? P : 1][4];
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < P; ++k) {
    if (cc[k] == 0xffffffffu) continue;
    const float ux = px[k] - mx, vx = px[k] - mn, uy = py[k] - my, vy = py[k] - ny;
    const float epx = ex2(kg * ux), emx = ex2(-kg * vx);
    const float epy = ex2(kg * uy), emy = ex2(-kg * vy);
    if (kKeep) {
      e[kKeep ? k : 0][0] = epx;
      e[kKeep ? k : 0][1] = emx;
      e[kKeep ? k : 0][2] = epy;
      e[kKeep ? k : 0][3] = emy;
    }
    s[0] += epx; s[1] += ux * epx; s[2] += emx; s[3] += vx * emx;
    s[4] += epy; s[5] += uy * epy; s[6] += emy; s[7] += vy * emy;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) s[k] = group_allreduce(s[k], g, OpAdd());
  if (!valid) return;  // every net of a class has two pins or more
  const float ipx = 1.0f / s[0], imx = 1.0f / s[2], ipy = 1.0f / s[4], imy = 1.0f / s[6];
#pragma unroll
  for (int k = 0; k < P; ++k) {
    const uint32_t c = cc[k];
    if (c >= a.N) continue;  // fixed cells and empty slots
    const float ux = px[k] - mx, vx = px[k] - mn, uy = py[k] - my, vy = py[k] - ny;
    float epx, emx, epy, emy;
    if (kKeep) {
      epx = e[kKeep ? k : 0][0];
      emx = e[kKeep ? k : 0][1];
      epy = e[kKeep ? k : 0][2];
      emy = e[kKeep ? k : 0][3];
    } else {
      epx = ex2(kg * ux);
      emx = ex2(-kg * vx);
      epy = ex2(kg * uy);
      emy = ex2(-kg * vy);
    }
    const float gx = wa_pin_grad(ux, vx, epx, emx, ipx, s[1], imx, s[3], a.gamma);
    const float gy = wa_pin_grad(uy, vy, epy, emy, ipy, s[5], imy, s[7], a.gamma);
    atomicAdd(&a.acc[c], pack_grad(__float2ll_rn(gx * a.grad_scale), __float2ll_rn(gy * a.grad_scale)));
  }
}

// A net of more than 224 pins on one warp, three passes over its pins.
__device__ void wa_big_net(const WaArgs &a, int pb, int pe, int lane) {
  const float kg = a.gamma * kLog2e;
  float mx = -INFINITY, mn = INFINITY, my = -INFINITY, ny = INFINITY;
  for (int q = pb + lane; q < pe; q += 32) {
    const float2 p = a.pos[a.pin_cell[q]];
    mx = fmaxf(mx, p.x);
    mn = fminf(mn, p.x);
    my = fmaxf(my, p.y);
    ny = fminf(ny, p.y);
  }
  mx = warp_allreduce(mx, OpMax());
  mn = warp_allreduce(mn, OpMin());
  my = warp_allreduce(my, OpMax());
  ny = warp_allreduce(ny, OpMin());
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int q = pb + lane; q < pe; q += 32) {
    const float2 p = a.pos[a.pin_cell[q]];
    const float ux = p.x - mx, vx = p.x - mn, uy = p.y - my, vy = p.y - ny;
    const float epx = ex2(kg * ux), emx = ex2(-kg * vx);
    const float epy = ex2(kg * uy), emy = ex2(-kg * vy);
    s[0] += epx; s[1] += ux * epx; s[2] += emx; s[3] += vx * emx;
    s[4] += epy; s[5] += uy * epy; s[6] += emy; s[7] += vy * emy;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) s[k] = warp_allreduce(s[k], OpAdd());
  const float ipx = 1.0f / s[0], imx = 1.0f / s[2], ipy = 1.0f / s[4], imy = 1.0f / s[6];
  for (int q = pb + lane; q < pe; q += 32) {
    const uint32_t c = a.pin_cell[q];
    if (c >= a.N) continue;
    const float2 p = a.pos[c];
    const float ux = p.x - mx, vx = p.x - mn, uy = p.y - my, vy = p.y - ny;
    const float gx = wa_pin_grad(ux, vx, ex2(kg * ux), ex2(-kg * vx), ipx, s[1], imx, s[3], a.gamma);
    const float gy = wa_pin_grad(uy, vy, ex2(kg * uy), ex2(-kg * vy), ipy, s[5], imy, s[7], a.gamma);
    atomicAdd(&a.acc[c], pack_grad(__float2ll_rn(gx * a.grad_scale), __float2ll_rn(gy * a.grad_scale)));
  }
}

// Nets are ordered by degree and split into degree classes (WaClass): each
// warp takes 32 / G nets of one class, so the reductions run over a fixed
// group width with no per-lane segment logic.  Warps are visited from the
// heaviest class down.
__global__ void __launch_bounds__(kWaBlock) k_wa(const WaArgs a) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int t = gw; t < a.nwarps; t += nw) {
    const int w = a.nwarps - 1 - t;
    int j = 0;
#pragma unroll
    for (int k = 1; k < kWaClasses; ++k) j += (w >= a.cls[k].first_warp) ? 1 : 0;
    const WaClass &cl = a.cls[j];
    const int wi = w - cl.first_warp;
    switch (j) {
      case 0: case 1: case 2: case 3: case 4: {  // up to 32 pins: 1..8 lanes per net, <= 4 pins per lane
        const int g = j <= 1 ? 1 : (1 << (j - 1));   // kWaGroup
        wa_group<4>(a, cl, g, j == 0 ? 2 : 4, wi, lane);  // kWaSlots
        break;
      }
      case 5: case 6: case 7:  // 33..224 pins: a warp per net, <= 8 slots per lane
        wa_group<8>(a, cl, 32, j == 5 ? 2 : (j == 6 ? 4 : 8), wi, lane);
        break;
      default: {
        const uint32_t n = cl.first_net + wi;
        wa_big_net(a, a.net_off[n], a.net_off[n + 1], lane);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Footprint helpers shared by the scatter and the gather.  Footprint
// [x - w/2, x + w/2] x [y - h/2, y + h/2] in sites; bin b covers
// [b*s, (b+1)*s) (s sites per bin, an integer).  With w = h = s = 1 this is
// cell_bin_overlap / bin_overlap_area (density.rs:20-48).
// The arithmetic is exact in FP32 up to the final product of the two 1-D
// overlaps: a coordinate is split into its integer part i and fraction f
// (both exact), every edge difference is formed as (integer - f), and the
// bin range comes from integer floor / ceiling divisions.  Forming x + w/2
// directly would round once the sum crosses a power of two (at 1024 sites
// the FP32 spacing doubles to 1.2e-4), which shows up as area lost from one
// bin.
// ---------------------------------------------------------------------------
struct Foot {
  float fx, fy;   // fractional parts of the centre, in [0, 1)
  float hw, hh;   // half extents
  int ix, iy;     // integer parts of the centre
  int bx0, bx1, by0, by1;
};

// floor(a / s) for s > 0; a shift when s is a power of two (arithmetic
// shifts floor negative values too), which is the usual bin size.
__device__ __forceinline__ int floor_div(int a, int s) {
  if ((s & (s - 1)) == 0) return a >> (__ffs(s) - 1);
  return a >= 0 ? a / s : -((s - 1 - a) / s);
}
__device__ __forceinline__ int ceil_div(int a, int s) { return -floor_div(-a, s); }

__device__ __forceinline__ Foot make_foot(float2 p, float hw, float hh, int BX, int BY, int sx, int sy) {
  Foot f;
  const float flx = floorf(p.x), fly = floorf(p.y);
  f.ix = (int)flx;
  f.iy = (int)fly;
  f.fx = p.x - flx;
  f.fy = p.y - fly;
  f.hw = hw;
  f.hh = hh;
  // floor(x - hw) = ix + floor(fx - hw), ceil(x + hw) = ix + ceil(fx + hw)
  f.bx0 = max(0, floor_div(f.ix + (int)floorf(f.fx - hw), sx));
  f.bx1 = min(BX, max(0, ceil_div(f.ix + (int)ceilf(f.fx + hw), sx)));
  f.by0 = max(0, floor_div(f.iy + (int)floorf(f.fy - hh), sy));
  f.by1 = min(BY, max(0, ceil_div(f.iy + (int)ceilf(f.fy + hh), sy)));
  return f;
}

// Length of [c - h, c + h] inside [b*s, (b+1)*s), c = i + fr:
// min(h, (b+1)s - c) - max(-h, b s - c), each difference formed exactly.
__device__ __forceinline__ float overlap_1d(int i, float fr, float h, int b, int s) {
  const int k0 = b * s - i;
  const float hi = fminf(h, (float)(k0 + s) - fr);
  const float lo = fmaxf(-h, (float)k0 - fr);
  return fmaxf(hi - lo, 0.0f);
}
__device__ __forceinline__ float overlap_x(const Foot &f, int bx, int s) { return overlap_1d(f.ix, f.fx, f.hw, bx, s); }
__device__ __forceinline__ float overlap_y(const Foot &f, int by, int s) { return overlap_1d(f.iy, f.fy, f.hh, by, s); }

// Unit cells first (a 1x1 footprint covers at most 2 x 2 bins: unrolled, no
// footprint load), then the macros from their own list, so a warp of unit
// cells never waits for one macro's loop.  Fixed-point atomics make the
// order irrelevant.  Without a macro list but with footprints, every cell
// takes the general loop.
__global__ void __launch_bounds__(kScatterBlock) k_scatter(const ScatterArgs a) {
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x, ts = gridDim.x * blockDim.x;
  if (a.half && !a.mflag) {
    for (uint32_t i = t0; i < a.N; i += ts) {
      const float2 hf = a.half[i];
      const Foot f = make_foot(a.pos[i], hf.x, hf.y, a.BX, a.BY, a.isx, a.isy);
      for (int by = f.by0; by < f.by1; ++by) {
        const float oy = overlap_y(f, by, a.isy);
        for (int bx = f.bx0; bx < f.bx1; ++bx) {
          const float ar = overlap_x(f, bx, a.isx) * oy;
          if (ar > 0.0f) atomicAdd(&a.dens[(size_t)by * a.BX + bx], to_fix(ar));
        }
      }
    }
    return;
  }
  for (uint32_t i = t0; i < a.N; i += ts) {
    if (a.mflag && a.mflag[i]) continue;
    const Foot f = make_foot(a.pos[i], 0.5f, 0.5f, a.BX, a.BY, a.isx, a.isy);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int by = f.by0 + (k >> 1), bx = f.bx0 + (k & 1);
      if (by >= f.by1 || bx >= f.bx1) continue;
      const float ar = overlap_x(f, bx, a.isx) * overlap_y(f, by, a.isy);
      if (ar > 0.0f) atomicAdd(&a.dens[(size_t)by * a.BX + bx], to_fix(ar));
    }
  }
  for (uint32_t k = t0; k < a.n_mac; k += ts) {
    const uint32_t i = a.mac_idx[k];
    const float2 hf = a.half[i];
    const Foot f = make_foot(a.pos[i], hf.x, hf.y, a.BX, a.BY, a.isx, a.isy);
    for (int by = f.by0; by < f.by1; ++by) {
      const float oy = overlap_y(f, by, a.isy);
      for (int bx = f.bx0; bx < f.bx1; ++bx) {
        const float ar = overlap_x(f, bx, a.isx) * oy;
        if (ar > 0.0f) atomicAdd(&a.dens[(size_t)by * a.BX + bx], to_fix(ar));
      }
    }
  }
}

__global__ void __launch_bounds__(kFinalBlock) k_density_final(const FinalArgs a) {
  __shared__ double sm[64];
  __shared__ bool last;
  double v[2] = {0.0, 0.0};
  // Groups of four consecutive bins per thread and step: 16-byte loads and
  // stores (when every pointer is aligned for them; a ragged tail, or
  // unaligned caller buffers, take the scalar loop below).
  const int ng = a.vec4 ? (a.nb >> 2) : 0;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, ts = gridDim.x * blockDim.x;
  for (int gi = t0; gi < ng; gi += ts) {
    ulonglong2 *dp = reinterpret_cast<ulonglong2 *>(a.dens) + 2 * gi;
    const ulonglong2 q0 = dp[0], q1 = dp[1];
    dp[0] = make_ulonglong2(0ull, 0ull);
    dp[1] = make_ulonglong2(0ull, 0ull);
    const double d[4] = {from_fix(q0.x), from_fix(q0.y), from_fix(q1.x), from_fix(q1.y)};
    float r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      r[k] = (float)(d[k] - a.c0);
      v[0] += d[k];
      v[1] += fmax(d[k] - a.cap, 0.0);
    }
    if (a.rho) reinterpret_cast<float4 *>(a.rho)[gi] = make_float4(r[0], r[1], r[2], r[3]);
    if (a.rho_hi) {
      __nv_bfloat16 h[4], l[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        h[k] = __float2bfloat16_rn(r[k]);
        l[k] = __float2bfloat16_rn(r[k] - __bfloat162float(h[k]));
      }
      uint2 hv, lv;
      hv.x = (uint32_t)__bfloat16_as_ushort(h[0]) | ((uint32_t)__bfloat16_as_ushort(h[1]) << 16);
      hv.y = (uint32_t)__bfloat16_as_ushort(h[2]) | ((uint32_t)__bfloat16_as_ushort(h[3]) << 16);
      lv.x = (uint32_t)__bfloat16_as_ushort(l[0]) | ((uint32_t)__bfloat16_as_ushort(l[1]) << 16);
      lv.y = (uint32_t)__bfloat16_as_ushort(l[2]) | ((uint32_t)__bfloat16_as_ushort(l[3]) << 16);
      reinterpret_cast<uint2 *>(a.rho_hi)[gi] = hv;
      reinterpret_cast<uint2 *>(a.rho_lo)[gi] = lv;
    }
    if (a.dens_out) {
      reinterpret_cast<double2 *>(a.dens_out)[2 * gi] = make_double2(d[0], d[1]);
      reinterpret_cast<double2 *>(a.dens_out)[2 * gi + 1] = make_double2(d[2], d[3]);
    }
  }
  for (int i = 4 * ng + t0; i < a.nb; i += ts) {
    const double d = from_fix(a.dens[i]);
    a.dens[i] = 0ull;
    const float r = (float)(d - a.c0);
    if (a.rho) a.rho[i] = r;
    if (a.rho_hi) {
      const __nv_bfloat16 h = __float2bfloat16_rn(r);
      a.rho_hi[i] = h;
      a.rho_lo[i] = __float2bfloat16_rn(r - __bfloat162float(h));
    }
    if (a.dens_out) a.dens_out[i] = d;
    v[0] += d;
    v[1] += fmax(d - a.cap, 0.0);
  }
  block_sum<2>(v, sm);
  if (threadIdx.x == 0) {
    a.part[2 * blockIdx.x] = v[0];
    a.part[2 * blockIdx.x + 1] = v[1];
    __threadfence();
    last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double fin[2];
  sum_partials<2>(a.part, 2, gridDim.x, fin, sm);
  if (threadIdx.x == 0) {
    const double s = fin[0], o = fin[1];
    const double ov = (s < 1e-30) ? 0.0 : o / s;  // compute_overlap
    a.sc->overlap = ov;
    a.log[a.sc->iter].overlap = ov;
    *a.ticket = 0u;
  }
}

// ---------------------------------------------------------------------------
// FP32 SIMT GEMM: TM x TN CTA tile (64 x 64 with 256 threads, or 32 x 32 with
// 64 threads when the large tile leaves SMs idle), BK = 16, 4 x 4 outputs per
// thread, double-buffered shared memory.  Bounds are checked on every load
// and store, so any M, N, K works; multiples of 4 take the float4 path.
// Every output sums k = 0 .. K-1 in order whatever the tile, so both tile
// sizes give the same bits.
// ---------------------------------------------------------------------------
constexpr int GK = 16;

// S > 1: split K over a cluster of S CTAs (cluster dims 1 x 1 x S along z).
// CTA rank r sums k in [r K/S, (r+1) K/S) in order, parks its partial tile in
// its shared memory, and after a cluster barrier adds the S partials of a
// TM/S-row slice of the tile in rank order ((p0 + p1) + p2) + ... through
// distributed shared memory, then runs the epilogue on that slice.  The
// order is the same for both tile sizes, so they still give the same bits.
// One output of a SIMT GEMM.  With SPECTRAL: density.rs:114-153, scale
// 4/(WH), x1/2 on the kx = 0 and ky = 0 lines, phi = a / (2(1-cos wx) +
// 2(1-cos wy)), E = phi * w, at the frequencies (ky, kx) the op's layout
// gives the output (row, column); phi is written at its natural place.
template <bool SPECTRAL>
__device__ __forceinline__ void gemm_store(const GemmOp &op, const SpectralArgs &sp, int r, int c, int N, float v) {
  const size_t o = (size_t)r * op.ldc + c;
  if (SPECTRAL) {
    const int ky = op.row_par < 0 ? r : 2 * r + op.row_par;
    const int kx = op.col_split ? (c < N / 2 ? 2 * c : 2 * (c - N / 2) + 1) : c;
    float s = sp.scale;
    if (kx == 0) s *= 0.5f;
    if (ky == 0) s *= 0.5f;
    const float den = sp.gx2[kx] + sp.gy2[ky];
    float phi = 0.0f, ex = 0.0f, ey = 0.0f;
    if (!(den < 1e-30f)) {
      phi = v * s / den;
      ex = phi * sp.wx[kx];
      ey = phi * sp.wy[ky];
    }
    op.C[o] = ex;
    op.C2[o] = ey;
    if (sp.phi) sp.phi[(size_t)ky * N + kx] = phi;
  } else {
    op.C[o] = v;
  }
}

template <bool SPECTRAL, int TM, int TN, int S>
__global__ void __launch_bounds__((TM / 4) * (TN / 4)) k_sgemm(const GemmOp *ops, int M, int N, int K,
                                                               SpectralArgs sp) {
  constexpr int T = (TM / 4) * (TN / 4);
  constexpr int LA = TM * GK / (4 * T), LB = GK * TN / (4 * T);  // float4 loads per thread
  static_assert(S == 1 || (TM % S == 0 && (TM / S) * (TN / 4) == T), "one float4 per thread in the split reduction");
  const GemmOp op = ops[blockIdx.z / S];
  __shared__ __align__(16) float smem[2 * GK * (TM + 4) + 2 * GK * (TN + 4)];
  static_assert(S == 1 || TM * TN <= 2 * GK * (TM + 4) + 2 * GK * (TN + 4), "partial tile fits the staging buffers");
  auto As = reinterpret_cast<float(*)[GK][TM + 4]>(smem);
  auto Bs = reinterpret_cast<float(*)[GK][TN + 4]>(smem + 2 * GK * (TM + 4));
  const int tid = threadIdx.x, tx = tid % (TN / 4), ty = tid / (TN / 4);
  const int bm = blockIdx.y * TM, bn = blockIdx.x * TN;
  const bool vec = ((K & 3) == 0) && ((N & 3) == 0) && ((op.lda & 3) == 0) && ((op.ldb & 3) == 0) &&
                   ((op.a_full & 3) == 0);
  const float am = (float)op.a_mir, bmir = (float)op.b_mir;
  float ra[LA][4], rb[LB][4];
  auto load = [&](int k0) {
#pragma unroll
    for (int l = 0; l < LA; ++l) {
      const int f = tid + l * T;
      const int gr = bm + f / (GK / 4), gk = k0 + (f % (GK / 4)) * 4;
      const float *arow = op.A + (size_t)gr * op.lda;
      if (vec && gr < M && gk + 3 < K) {
        float4 t = *reinterpret_cast<const float4 *>(arow + gk);
        if (op.a_mir) {  // columns a_full-1-gk-j, j = 0..3: the block below, reversed
          const float4 u = *reinterpret_cast<const float4 *>(arow + (op.a_full - 4 - gk));
          t.x += am * u.w; t.y += am * u.z; t.z += am * u.y; t.w += am * u.x;
        }
        ra[l][0] = t.x; ra[l][1] = t.y; ra[l][2] = t.z; ra[l][3] = t.w;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          float v = (gr < M && gk + j < K) ? arow[gk + j] : 0.0f;
          if (op.a_mir && gr < M && gk + j < K) v += am * arow[op.a_full - 1 - (gk + j)];
          ra[l][j] = v;
        }
      }
    }
#pragma unroll
    for (int l = 0; l < LB; ++l) {
      const int f = tid + l * T;
      const int gk = k0 + f / (TN / 4), gc = bn + (f % (TN / 4)) * 4;
      const float *brow = op.B + (size_t)gk * op.ldb;
      const float *bmrow = op.b_mir ? op.B + (size_t)(op.b_full - 1 - gk) * op.ldb : brow;
      if (vec && gk < K && gc + 3 < N) {
        float4 t = *reinterpret_cast<const float4 *>(brow + gc);
        if (op.b_mir) {
          const float4 u = *reinterpret_cast<const float4 *>(bmrow + gc);
          t.x += bmir * u.x; t.y += bmir * u.y; t.z += bmir * u.z; t.w += bmir * u.w;
        }
        rb[l][0] = t.x; rb[l][1] = t.y; rb[l][2] = t.z; rb[l][3] = t.w;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          float v = (gk < K && gc + j < N) ? brow[gc + j] : 0.0f;
          if (op.b_mir && gk < K && gc + j < N) v += bmir * bmrow[gc + j];
          rb[l][j] = v;
        }
      }
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int l = 0; l < LA; ++l) {
      const int f = tid + l * T;
      const int r = f / (GK / 4), k = (f % (GK / 4)) * 4;
#pragma unroll
      for (int j = 0; j < 4; ++j) As[buf][k + j][r] = ra[l][j];
    }
#pragma unroll
    for (int l = 0; l < LB; ++l) {
      const int f = tid + l * T;
      const int k = f / (TN / 4), c = (f % (TN / 4)) * 4;
      *reinterpret_cast<float4 *>(&Bs[buf][k][c]) = make_float4(rb[l][0], rb[l][1], rb[l][2], rb[l][3]);
    }
  };
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  // This CTA's k range (all of K when S == 1; the launcher splits only when
  // S * GK divides K).
  const int kpart = (S == 1) ? K : K / S;
  const int kbeg = (S == 1) ? 0 : (int)(blockIdx.z % S) * kpart;
  const int nk = (kpart + GK - 1) / GK;
  load(kbeg);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < nk; ++kt) {
    const int cur = kt & 1;
    if (kt + 1 < nk) load(kbeg + (kt + 1) * GK);
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      const float4 a4 = *reinterpret_cast<const float4 *>(&As[cur][kk][ty * 4]);
      const float4 b4 = *reinterpret_cast<const float4 *>(&Bs[cur][kk][tx * 4]);
      const float av[4] = {a4.x, a4.y, a4.z, a4.w}, bv[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    if (kt + 1 < nk) {
      store(cur ^ 1);
      __syncthreads();
    }
  }
  if constexpr (S > 1) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    __syncthreads();  // the staging buffers become the partial tile
#pragma unroll
    for (int i = 0; i < 4; ++i)
      *reinterpret_cast<float4 *>(&smem[(ty * 4 + i) * TN + tx * 4]) =
          make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
    cluster.sync();
    const int rank = (int)cluster.block_rank();
    const int lr = rank * (TM / S) + tid / (TN / 4), lc = (tid % (TN / 4)) * 4;
    float4 v = *reinterpret_cast<const float4 *>(cluster.map_shared_rank(&smem[lr * TN + lc], 0));
#pragma unroll
    for (int q = 1; q < S; ++q) {
      const float4 w = *reinterpret_cast<const float4 *>(cluster.map_shared_rank(&smem[lr * TN + lc], q));
      v.x += w.x;
      v.y += w.y;
      v.z += w.z;
      v.w += w.w;
    }
    const float vv[4] = {v.x, v.y, v.z, v.w};
    const int r = bm + lr;
    if (r < M) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int cidx = bn + lc + j;
        if (cidx >= N) continue;
        gemm_store<SPECTRAL>(op, sp, r, cidx, N, vv[j]);
      }
    }
    cluster.sync();  // no CTA leaves while another reads its partial tile
    return;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = bm + ty * 4 + i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int cidx = bn + tx * 4 + j;
      if (cidx >= N) continue;
      gemm_store<SPECTRAL>(op, sp, r, cidx, N, acc[i][j]);
    }
  }
}

// SMs of the current device (cached per device).
int device_sms() {
  static int sms[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!sms[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    sms[dev] = v;
  }
  return sms[dev];
}

// The small tile when the 64 x 64 grid would leave more than half the SMs
// without a CTA (measured: 64 CTAs of 512^3 gain from the small tile, 128
// CTAs do not).
bool sgemm_small_tile(int M, int N, int nb, int K) {
  const long ctas = (long)((N + 63) / 64) * ((M + 63) / 64) * nb * (K % 64 == 0 ? 4 : 1);  // split K: 4 CTAs a tile
  return 2L * ctas < device_sms();
}

// ---------------------------------------------------------------------------
// Grid barrier for the cooperative step kernel.  Every wait is bounded: on
// timeout the block records the error in sc->err and leaves the kernel, so
// the kernel always terminates, no block computes on partial data, and the
// host reports EPLACE_ERR_TIMEOUT (the next run resets the device state).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool grid_barrier(unsigned *bar, DevScalars *sc) {
  // bar[0..1] is one 64-bit arrival count that is never reset inside a run:
  // every launch on it has the same grid and passes whole barriers, so a
  // launch starts at a multiple of gridDim.x, and barrier k of the run is
  // complete when the count reaches (k + 1) * gridDim.x.  The last block's
  // own add releases the others (no reset, no second word to publish).
  // The host zeroes the count at every load and run start.  The wait is
  // bounded (sc->spin_cycles): a block that gives up records sc->err and
  // returns false, and its caller leaves the kernel.
  __shared__ int gave_up;
  __syncthreads();
  if (threadIdx.x == 0) {
    gave_up = 0;
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(bar);
    const long long limit = sc->spin_cycles > 0 ? sc->spin_cycles : kSpinCycles;
    __threadfence();  // this block's writes before its arrival
    const unsigned long long old = atomicAdd(cnt, 1ull);
    const unsigned long long target = old - old % gridDim.x + gridDim.x;
    const long long t0 = clock64();
    while (true) {
      unsigned long long v;
      asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(cnt) : "memory");
      if (v >= target) break;
      if (clock64() - t0 > limit) {
        atomicExch(&sc->err, 1);
        gave_up = 1;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
  }
  __syncthreads();
  return !gave_up;
}

// Field gather of a 1x1 footprint: it touches at most 2 x 2 bins (bins are
// >= 1 site wide); weights first, then all field loads at once, summed in the
// same row-major order as the general loop of gather_cell.
__device__ __forceinline__ float2 gather_unit_foot(const StepArgs &a, const Foot &f) {
  float fx = 0.f, fy = 0.f, wt = 0.f;
  float w[4];
  size_t id[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int by = f.by0 + (k >> 1), bx = f.bx0 + (k & 1);
    const bool in = by < f.by1 && bx < f.bx1;
    w[k] = in ? overlap_x(f, bx, a.isx) * overlap_y(f, by, a.isy) : 0.0f;
    id[k] = (w[k] > 0.0f) ? (size_t)by * a.BX + bx : 0;
  }
  float e[4], h[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    e[k] = (w[k] > 0.0f) ? a.Ex[id[k]] : 0.0f;
    h[k] = (w[k] > 0.0f) ? a.Ey[id[k]] : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (w[k] > 0.0f) {
      fx = fmaf(w[k], e[k], fx);
      fy = fmaf(w[k], h[k], fy);
      wt += w[k];
    }
  float2 g = make_float2(0.f, 0.f);
  if (wt > 1e-10f) {
    g.x = fx / wt;
    g.y = fy / wt;
  }
  return g;
}

// Field gather of a 1x1 cell (no footprint load).
__device__ __forceinline__ float2 gather_unit(const StepArgs &a, float2 p) {
  const Foot f = make_foot(p, 0.5f, 0.5f, a.BX, a.BY, a.isx, a.isy);
  return gather_unit_foot(a, f);
}

// Weighted-mean field gather for one cell, scaled by its area
// (compute_density_gradient, density.rs:171-206).
__device__ __forceinline__ float2 gather_cell(const StepArgs &a, uint32_t i, float2 p) {
  const float2 hf = a.half ? a.half[i] : make_float2(0.5f, 0.5f);
  const Foot f = make_foot(p, hf.x, hf.y, a.BX, a.BY, a.isx, a.isy);
  float fx = 0.f, fy = 0.f, wt = 0.f;
  if (hf.x == 0.5f && hf.y == 0.5f) return gather_unit_foot(a, f);
  // Bins of a row in chunks of 8 with all field loads of a chunk issued
  // before the sums (a macro spans up to 9 bins per axis), so a footprint
  // costs one memory latency per row and chunk instead of one per bin; the
  // sums keep the row-major bin order.
  for (int by = f.by0; by < f.by1; ++by) {
    const float oy = overlap_y(f, by, a.isy);
    for (int b0 = f.bx0; b0 < f.bx1; b0 += 8) {
      float w[8], e[8], h[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int bx = b0 + k;
        w[k] = (bx < f.bx1) ? overlap_x(f, bx, a.isx) * oy : 0.0f;
        const size_t idx = (size_t)by * a.BX + (w[k] > 0.0f ? bx : 0);
        e[k] = (w[k] > 0.0f) ? a.Ex[idx] : 0.0f;
        h[k] = (w[k] > 0.0f) ? a.Ey[idx] : 0.0f;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (w[k] > 0.0f) {
          fx = fmaf(w[k], e[k], fx);
          fy = fmaf(w[k], h[k], fy);
          wt += w[k];
        }
    }
  }
  float2 g = make_float2(0.f, 0.f);
  if (wt > 1e-10f) {
    const float ar = a.area ? a.area[i] : 1.0f;
    g.x = ar * (fx / wt);
    g.y = ar * (fy / wt);
  }
  return g;
}

// g = (g_wl + lam g_den) / max(1, pw + lam area)   (mod.rs:145-156)
// unit: a 1x1 cell, whose area is 1 (no load).
__device__ __forceinline__ float2 combine(const StepArgs &a, uint32_t i, float2 gw, float2 gd,
                                          double lam, bool unit) {
  const double ar = (unit || !a.area) ? 1.0 : (double)a.area[i];
  const double ipc = 1.0 / fmax((double)a.pw[i] + lam * ar, 1.0);
  return make_float2((float)(((double)gw.x + lam * (double)gd.x) * ipc),
                     (float)(((double)gw.y + lam * (double)gd.y) * ipc));
}

// Phase A of the step for one cell, split into its loads and the rest so
// that a thread can have the loads of two cells in flight.
struct CellA {
  float2 gd, gw;     // density field gather, WA gradient
  float2 x, xp, gp;  // for the Barzilai-Borwein dots (after the first penalty)
};

// unit: the cell is 1x1 (the 2 x 2-bin gather, no footprint load).
__device__ __forceinline__ CellA load_a(const StepArgs &a, uint32_t i, bool was_init, bool unit) {
  CellA c;
  c.gd = unit ? gather_unit(a, a.look[i]) : gather_cell(a, i, a.look[i]);
  long long sx, sy;
  unpack_grad(a.acc[i], &sx, &sy);
  c.gw = make_float2((float)((double)sx * a.grad_inv), (float)((double)sy * a.grad_inv));
  if (was_init) {
    c.x = a.x[i];
    c.xp = a.xp[i];
    c.gp = a.gprev[i];
  }
  return c;
}

__device__ __forceinline__ void finish_a(const StepArgs &a, uint32_t i, const CellA &c, bool was_init, double lam,
                                         bool unit, double (&v)[4]) {
  a.acc[i] = 0ull;
  if (was_init) {
    const float2 g = combine(a, i, c.gw, c.gd, lam, unit);
    a.g[i] = g;
    const double dx = (double)c.x.x - c.xp.x, dy = (double)c.x.y - c.xp.y;
    v[0] += dx * dx;
    v[1] += dx * ((double)g.x - c.gp.x);
    v[2] += dy * dy;
    v[3] += dy * ((double)g.y - c.gp.y);
    return;
  }
  a.tmp_wl[i] = c.gw;
  a.tmp_den[i] = c.gd;
  v[0] += (double)c.gw.x * c.gw.x + (double)c.gw.y * c.gw.y;
  v[1] += (double)c.gd.x * c.gd.x + (double)c.gd.y * c.gd.y;
}

// FISTA step (nesterov.rs:41-64), clamp (:67-72), next look-ahead (:95-101)
// clamped to the chip (common.rs:410-415), for one cell.
__device__ __forceinline__ void fista_cell(const StepArgs &a, uint32_t i, float2 x, float2 xp, float2 g, double m,
                                           double mn, const double (&alpha)[2], double (&nrm)[2]) {
  const double yx = (double)x.x + m * ((double)x.x - xp.x);
  const double yy = (double)x.y + m * ((double)x.y - xp.y);
  const double nx = yx - alpha[0] * g.x, ny = yy - alpha[1] * g.y;
  nrm[0] += (nx - x.x) * (nx - x.x);
  nrm[1] += (ny - x.y) * (ny - x.y);
  const float cx = fminf(fmaxf((float)nx, 0.0f), a.maxx);
  const float cy = fminf(fmaxf((float)ny, 0.0f), a.maxy);
  const float px = fminf(fmaxf(x.x, 0.0f), a.maxx);
  const float py = fminf(fmaxf(x.y, 0.0f), a.maxy);
  a.x[i] = make_float2(cx, cy);
  a.xp[i] = make_float2(px, py);
  a.gprev[i] = g;
  const double lx = (double)cx + mn * ((double)cx - px);
  const double ly = (double)cy + mn * ((double)cy - py);
  a.look[i] = make_float2(fminf(fmaxf((float)lx, 0.0f), a.maxx), fminf(fmaxf((float)ly, 0.0f), a.maxy));
}

__global__ void __launch_bounds__(kStepBlock, 2) k_step(const StepArgs a) {
  __shared__ double sm[32 * 4];
  __shared__ bool last;
  const uint32_t tid0 = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gstride = gridDim.x * blockDim.x;
  const int it = a.sc->iter;
  const bool was_init = a.sc->lam_init != 0;
  double lam = a.sc->lam;
  bool lam_init = was_init;
  if (was_init) lam = (lam < 50.0) ? lam * 1.025 : lam + 1.0;  // mod.rs:139-143

  // A bounded wait already gave up in an earlier launch: every block sees the
  // same flag here and leaves before any barrier, so the rest of the
  // interval drains quickly and the host reports EPLACE_ERR_TIMEOUT.
  if (a.sc->err) return;
  if (a.mode == 1) {  // gather only: no barrier is reached
    for (uint32_t i = tid0; i < a.N; i += gstride) a.tmp_den[i] = gather_cell(a, i, a.look[i]);
    return;
  }
  // Modes: 0 = whole step in one cooperative launch (grid barriers between
  // phases); 2, 3, 4 = phase A, the penalty-initialisation pass and phase C
  // as three ordinary launches of the same grid (kernel boundaries replace
  // the barriers, so no block ever waits for another).
  const bool coop = a.mode == 0;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (a.mode == 0 || a.mode == 2) {
    // Phase A: gather, read + clear the WA accumulator, combine.  Two cells
    // per thread and pass (i and i + ustride): every load of both is issued
    // before the first store, so their latencies overlap.  Macros (w*h > 1)
    // are skipped here and done afterwards from their own list, so a warp
    // of unit cells never waits for one macro's multi-bin gather.
    // When the unit cells still fit one pass of pairs on the other threads,
    // the last n_mac threads of the grid take macros only (macro k goes to
    // thread gstride - 1 - k, mod gstride), so a macro's multi-row gather
    // does not queue behind a unit cell in the same thread (200k cells:
    // step 29.1 -> 26.9 us); otherwise (800k) every thread takes unit cells.
    const uint32_t nm =
        (a.n_mac <= gstride / 4 && (uint64_t)a.N <= 2ull * (gstride - a.n_mac)) ? a.n_mac : 0u;
    const uint32_t ustride = gstride - nm;
    if (tid0 < ustride)
      for (uint32_t i0 = tid0; i0 < a.N; i0 += 2 * ustride) {
        const uint32_t i1 = i0 + ustride;
        const bool h1 = i1 < a.N;
        const bool u0 = !a.mflag || !a.mflag[i0];
        const bool u1 = h1 && (!a.mflag || !a.mflag[i1]);
        CellA c0, c1;
        if (u0) c0 = load_a(a, i0, was_init, true);
        if (u1) c1 = load_a(a, i1, was_init, true);
        if (u0) finish_a(a, i0, c0, was_init, lam, true, v);
        if (u1) finish_a(a, i1, c1, was_init, lam, true, v);
      }
    for (uint32_t k = gstride - 1 - tid0; k < a.n_mac; k += gstride) {
      const uint32_t i = a.mac_idx[k];
      const CellA c = load_a(a, i, was_init, false);
      finish_a(a, i, c, was_init, lam, false, v);
    }
    block_sum<4>(v, sm);
    if (threadIdx.x == 0)
      for (int k = 0; k < 4; ++k) a.part[4 * blockIdx.x + k] = v[k];
    if (a.mode == 2) return;
    if (!grid_barrier(a.bar, a.sc)) return;
  }

  // Pass-2 partials: part[] again after a barrier (cooperative), else part_b[].
  double *part2nd = coop ? a.part : a.part_b;
  if (!was_init) {
    // First penalty: 0.1 * |g_wl| / |g_den| when |g_den| > 1e-30 (mod.rs:132-138).
    double nr[2];
    sum_partials<2>(a.part, 4, gridDim.x, nr, sm);
    const double wl = sqrt(nr[0]);
    const double dn = sqrt(nr[1]);
    if (dn > 1e-30) {
      lam = 0.1 * wl / dn;
      lam_init = true;
    }
    if (a.mode == 0 || a.mode == 3) {
      if (coop) if (!grid_barrier(a.bar, a.sc)) return;  // everyone has read part[] before it is reused
      for (int k = 0; k < 4; ++k) v[k] = 0.0;
      for (uint32_t i = tid0; i < a.N; i += gstride) {
        const float2 g = combine(a, i, a.tmp_wl[i], a.tmp_den[i], lam, false);
        a.g[i] = g;
        const float2 x = a.x[i], xp = a.xp[i], gp = a.gprev[i];
        const double dx = (double)x.x - xp.x, dy = (double)x.y - xp.y;
        v[0] += dx * dx;
        v[1] += dx * ((double)g.x - gp.x);
        v[2] += dy * dy;
        v[3] += dy * ((double)g.y - gp.y);
      }
      block_sum<4>(v, sm);
      if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) part2nd[4 * blockIdx.x + k] = v[k];
      if (a.mode == 3) return;
      if (!grid_barrier(a.bar, a.sc)) return;
    }
  } else if (a.mode == 3) {
    return;
  }

  // Barzilai-Borwein per axis after the first iteration (mod.rs:158-166,
  // nesterov.rs:199-218): |dx.dx / dx.dg| clamped to [1e-4, 1], kept when
  // |dx.dg| < 1e-30.
  double t[4];
  sum_partials<4>(was_init ? a.part : part2nd, 4, gridDim.x, t, sm);
  double alpha[2] = {a.sc->step[0], a.sc->step[1]};
  if (it > 0) {
    for (int ax = 0; ax < 2; ++ax) {
      const double dxdx = t[2 * ax], dxdg = t[2 * ax + 1];
      if (!(fabs(dxdg) < 1e-30)) alpha[ax] = fmin(fmax(fabs(dxdx / dxdg), 1e-4), 1.0);
    }
  }
  // FISTA step (nesterov.rs:41-64), clamp (:67-72), next look-ahead
  // (:95-101) clamped to the chip (common.rs:410-415).
  const double m = a.mom[it], mn = a.mom[it + 1];
  double nrm[2] = {0.0, 0.0};
  for (uint32_t i0 = tid0; i0 < a.N; i0 += 2 * gstride) {  // two cells per pass, loads first
    const uint32_t i1 = i0 + gstride;
    const bool h1 = i1 < a.N;
    const float2 x0 = a.x[i0], xp0 = a.xp[i0], g0 = a.g[i0];
    float2 x1 = x0, xp1 = xp0, g1 = g0;
    if (h1) {
      x1 = a.x[i1];
      xp1 = a.xp[i1];
      g1 = a.g[i1];
    }
    fista_cell(a, i0, x0, xp0, g0, m, mn, alpha, nrm);
    if (h1) fista_cell(a, i1, x1, xp1, g1, m, mn, alpha, nrm);
  }
  double w2[2] = {nrm[0], nrm[1]};
  block_sum<2>(w2, sm);
  // Step norms go to a second partials buffer, so no block has to wait for
  // the others to finish reading part[]; the last block to arrive sums them.
  if (threadIdx.x == 0) {
    a.part2[2 * blockIdx.x] = w2[0];
    a.part2[2 * blockIdx.x + 1] = w2[1];
    __threadfence();
    last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double fin[2];
  sum_partials<2>(a.part2, 2, gridDim.x, fin, sm);
  if (threadIdx.x == 0) {
    const double s0 = fin[0], s1 = fin[1];
    IterLog &L = a.log[it];
    L.lam = lam;
    L.step_norm[0] = sqrt(s0);
    L.step_norm[1] = sqrt(s1);
    L.alpha[0] = alpha[0];
    L.alpha[1] = alpha[1];
    a.sc->lam = lam;
    a.sc->lam_init = lam_init ? 1 : 0;
    a.sc->step[0] = alpha[0];
    a.sc->step[1] = alpha[1];
    a.sc->iter = it + 1;
    *a.ticket = 0u;
  }
}

__global__ void __launch_bounds__(kHpwlBlock) k_hpwl(const HpwlArgs a) {
  __shared__ double sm[32];
  double v[1] = {0.0};
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < a.NN; n += gridDim.x * blockDim.x) {
    const uint32_t b = a.net_off[n], e = a.net_off[n + 1];
    if ((a.has_driver && !a.has_driver[n]) || e - b < 2) continue;
    int x0 = INT_MAX, x1 = INT_MIN, y0 = INT_MAX, y1 = INT_MIN;
    for (uint32_t q = b; q < e; ++q) {
      const int2 l = a.loc[a.pin_cell[q]];
      x0 = min(x0, l.x);
      x1 = max(x1, l.x);
      y0 = min(y0, l.y);
      y1 = max(y1, l.y);
    }
    v[0] += (double)((long long)(x1 - x0) + (long long)(y1 - y0));
  }
  // Per-thread partials are integers below 2^53, so the FP64 block sum is exact.
  block_sum<1>(v, sm);
  if (threadIdx.x == 0) atomicAdd(a.total, (unsigned long long)(long long)v[0]);
}

}  // namespace

cudaError_t launch_wa(const WaArgs &a, int grid, cudaStream_t s) {
  if (a.nwarps == 0) return cudaSuccess;
  k_wa<<<grid, kWaBlock, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_scatter(const ScatterArgs &a, int grid, cudaStream_t s) {
  if (a.N == 0) return cudaSuccess;
  k_scatter<<<grid, kScatterBlock, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_density_final(const FinalArgs &a_in, int grid, cudaStream_t s) {
  FinalArgs a = a_in;
  auto al = [](const void *p, uintptr_t m) { return ((uintptr_t)p & (m - 1)) == 0; };
  a.vec4 = al(a.dens, 16) && al(a.rho, 16) && al(a.rho_hi, 8) && al(a.rho_lo, 8) && al(a.dens_out, 16);
  k_density_final<<<grid, kFinalBlock, 0, s>>>(a);
  return cudaGetLastError();
}

// One SIMT GEMM launch: split K four ways over a cluster when 4 * GK
// divides K (every transform of a power-of-two bin grid of at least 64),
// else one CTA per tile.  Which form runs depends on K alone, never on the
// tile, so the tile stays a choice of time only.
constexpr int kSplitK = 4;

template <bool SPECTRAL, int TM, int TN>
cudaError_t sgemm_launch(const GemmOp *ops, int nb, int M, int N, int K, const SpectralArgs &sp, cudaStream_t s) {
  const dim3 tiles((N + TN - 1) / TN, (M + TM - 1) / TM, nb);
  constexpr int T = (TM / 4) * (TN / 4);
  if (K % (kSplitK * GK) != 0) {
    k_sgemm<SPECTRAL, TM, TN, 1><<<tiles, T, 0, s>>>(ops, M, N, K, sp);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tiles.x, tiles.y, tiles.z * kSplitK);
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 1;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = kSplitK;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_sgemm<SPECTRAL, TM, TN, kSplitK>, ops, M, N, K, sp);
}

cudaError_t launch_sgemm(const GemmOp *ops, int nb, int M, int N, int K, cudaStream_t s, int tile) {
  if (tile == 32 || (tile == 0 && sgemm_small_tile(M, N, nb, K)))
    return sgemm_launch<false, 32, 32>(ops, nb, M, N, K, SpectralArgs{}, s);
  return sgemm_launch<false, 64, 64>(ops, nb, M, N, K, SpectralArgs{}, s);
}

cudaError_t launch_sgemm_spectral(const GemmOp *ops, int nb, int M, int N, int K, const SpectralArgs &sp,
                                  cudaStream_t s, int tile) {
  if (tile == 32 || (tile == 0 && sgemm_small_tile(M, N, nb, K)))
    return sgemm_launch<true, 32, 32>(ops, nb, M, N, K, sp, s);
  return sgemm_launch<true, 64, 64>(ops, nb, M, N, K, sp, s);
}

namespace {
__global__ void k_fly_cols(const FlyOp *ops, int H, int W) {
  const FlyOp op = ops[blockIdx.z];
  const int hw = W / 2;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (x >= hw || r >= H) return;
  const float e = op.E[(size_t)r * hw + x], o = op.O[(size_t)r * hw + x];
  op.out[(size_t)r * W + x] = e + o;
  op.out[(size_t)r * W + (W - 1 - x)] = op.sig * (e - o);
}
__global__ void k_fly_rows(const FlyOp *ops, int H, int W) {
  const FlyOp op = ops[blockIdx.z];
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W || y >= H / 2) return;
  const float e = op.E[(size_t)y * W + x], o = op.O[(size_t)y * W + x];
  op.out[(size_t)y * W + x] = e + o;
  op.out[(size_t)(H - 1 - y) * W + x] = op.sig * (e - o);
}
}  // namespace

cudaError_t launch_fly_cols(const FlyOp *ops, int nb, int H, int W, cudaStream_t s) {
  k_fly_cols<<<dim3((W / 2 + 127) / 128, H, nb), 128, 0, s>>>(ops, H, W);
  return cudaGetLastError();
}
cudaError_t launch_fly_rows(const FlyOp *ops, int nb, int H, int W, cudaStream_t s) {
  k_fly_rows<<<dim3((W + 127) / 128, H / 2, nb), 128, 0, s>>>(ops, H, W);
  return cudaGetLastError();
}

int step_max_grid(int device) {
  int sms = 0, occ = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_step, kStepBlock, 0) != cudaSuccess) return 0;
  return sms * occ;
}

cudaError_t launch_step(const StepArgs &a, int grid, cudaStream_t s) {
  void *args[] = {const_cast<StepArgs *>(&a)};
  return cudaLaunchCooperativeKernel((const void *)k_step, dim3(grid), dim3(kStepBlock), args, 0, s);
}
cudaError_t launch_step_split(const StepArgs &a, int grid, cudaStream_t s) {
  for (int mode = 2; mode <= 4; ++mode) {
    StepArgs b = a;
    b.mode = mode;
    k_step<<<grid, kStepBlock, 0, s>>>(b);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_hpwl(const HpwlArgs &a, int grid, cudaStream_t s) {
  k_hpwl<<<grid, kHpwlBlock, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace eplace
