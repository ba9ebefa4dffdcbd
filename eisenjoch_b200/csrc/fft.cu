// fft.cu -- FP32 FFT form of the spectral Poisson solve's transforms (see
// fft.cuh for the maps).  One CTA runs several complex FFTs of length N back
// to back in shared memory (row stages: 1024 points per CTA; column stages:
// four adjacent columns), decimation in time on bit-reversed inputs in
// radix-4 passes, twiddles from FP64-computed tables.  Every bin is loaded
// and stored once per stage, as 16-byte vectors (four positions of a row, or
// the four columns of a CTA at one row), with the lines staged in shared
// memory; the working set of a 1024^2 grid (4 MB per array) stays in L2
// across the three stages.
#include <cmath>

#include "fft.cuh"

namespace eplace {
namespace {

constexpr int kFftThreads = 256;
constexpr int kColLines = 4;  // columns per CTA of the column stages: one 16-byte vector a row
constexpr int kBatch = 4;     // vector loads a thread issues before using them

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ int bitrev(int m, int logN) { return (int)(__brev((unsigned)m) >> (32 - logN)); }

// Padded slot of complex point i of the FFT buffers: one float2 after every
// 16, so that the bit-reversed scatter (consecutive k -> slots N/32 apart)
// and the short strides of the first passes fall on different banks.
__device__ __forceinline__ int pd(int i) { return i + (i >> 4); }

// Spatial position n of a line <-> index of the reordered sequence v:
// v[m] = x[2m], v[N-1-m] = x[2m+1].
__device__ __forceinline__ int vpos(int n, int N) { return (n & 1) ? N - 1 - (n >> 1) : (n >> 1); }

// nf transforms of length N = 2^logN, back to back in s, bit-reversed in,
// natural order out: X[k] = sum_n x[n] e^{-2 pi i k n / N}.  Decimation in
// time; two levels (half sizes h and 2h) per pass as one radix-4 butterfly
// on i0, i0 + h, i0 + 2h, i0 + 3h (the same products and sums as two
// radix-2 levels), after one radix-2 level when logN is odd.
__device__ __forceinline__ void fft_core(float2 *s, int logN, int nf, const float2 *tw) {
  int lh = 0;
  if (logN & 1) {
    const int half = 1 << (logN - 1);
    for (int b = threadIdx.x; b < nf * half; b += blockDim.x) {
      const int i0 = ((b >> (logN - 1)) << logN) + ((b & (half - 1)) << 1);
      const float2 u = s[pd(i0)], t = s[pd(i0 + 1)];
      s[pd(i0)] = make_float2(u.x + t.x, u.y + t.y);
      s[pd(i0 + 1)] = make_float2(u.x - t.x, u.y - t.y);
    }
    lh = 1;
  }
  const int quarter = 1 << (logN - 2);
  for (; lh < logN; lh += 2) {
    const int h = 1 << lh;
    __syncthreads();
    for (int b = threadIdx.x; b < nf * quarter; b += blockDim.x) {
      const int p = b >> (logN - 2);
      const int j = b & (quarter - 1);
      const int pos = j & (h - 1);
      const int i0 = (p << logN) + ((j >> lh) << (lh + 2)) + pos;
      const float2 w1 = tw[pos << (logN - 1 - lh)];  // W_{2h}^pos
      const float2 w2 = tw[pos << (logN - 2 - lh)];  // W_{4h}^pos
      const int j0 = pd(i0), j1 = pd(i0 + h), j2 = pd(i0 + 2 * h), j3 = pd(i0 + 3 * h);
      const float2 x0 = s[j0], x1 = s[j1], x2 = s[j2], x3 = s[j3];
      // level h: (x0, x1), (x2, x3) with W_{2h}^pos
      const float2 t1 = cmul(x1, w1), t3 = cmul(x3, w1);
      const float2 a0 = make_float2(x0.x + t1.x, x0.y + t1.y), a1 = make_float2(x0.x - t1.x, x0.y - t1.y);
      const float2 a2 = make_float2(x2.x + t3.x, x2.y + t3.y), a3 = make_float2(x2.x - t3.x, x2.y - t3.y);
      // level 2h: (a0, a2) with W_{4h}^pos, (a1, a3) with W_{4h}^{pos+h} = -i W_{4h}^pos
      const float2 u2 = cmul(a2, w2);
      const float2 v3 = cmul(a3, make_float2(w2.y, -w2.x));
      s[j0] = make_float2(a0.x + u2.x, a0.y + u2.y);
      s[j2] = make_float2(a0.x - u2.x, a0.y - u2.y);
      s[j1] = make_float2(a1.x + v3.x, a1.y + v3.y);
      s[j3] = make_float2(a1.x - v3.x, a1.y - v3.y);
    }
  }
  __syncthreads();
}

// Sum of v over the CTA in a fixed order (a shuffle tree per warp, then the
// warps in order); the result is valid in thread 0.  red: [2 * warps].
__device__ __forceinline__ void block_sum2(double (&v)[2], double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v[0] += __shfl_down_sync(0xffffffffu, v[0], o);
    v[1] += __shfl_down_sync(0xffffffffu, v[1], o);
  }
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[2 * w] = v[0];
    red[2 * w + 1] = v[1];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    v[0] = v[1] = 0.0;
    for (int k = 0; k < nw; ++k) {
      v[0] += red[2 * k];
      v[1] += red[2 * k + 1];
    }
  }
}

// Index in the line of X'[k] for a stage-2/3 kind (-1: the value is 0).
__device__ __forceinline__ int pre_index(int kind, int k, int N) {
  if (kind == FFT_C3) return k;
  if (kind == FFT_S3) return N - 1 - k;
  return k == 0 ? -1 : N - k;  // FFT_SG
}

// Output sign of position n for the kind: S3 (-1)^n, SG -(-1)^n.
__device__ __forceinline__ float post_sign(int kind, int n) {
  if (kind == FFT_C3) return 1.0f;
  const float alt = (n & 1) ? -1.0f : 1.0f;
  return kind == FFT_S3 ? alt : -alt;
}

// Geometry of a stage: N the transform length, L the lines of the stage,
// lines and FFTs per CTA.
struct FftGeom {
  int N, logN, L, lines, per, ffts;
};

__host__ __device__ inline FftGeom fft_geom(int stage, int W, int H) {
  FftGeom g;
  const bool rows = stage != 1;
  g.N = rows ? W : H;
  g.L = rows ? H : W;
  g.logN = 0;
  while ((1 << g.logN) < g.N) ++g.logN;
  g.per = stage <= 1 ? 2 : 1;  // lines per FFT
  // rows: 1024 points (256 radix-4 butterflies a pass) per CTA; columns:
  // four adjacent columns per CTA, one 16-byte vector per row and array
  g.lines = rows ? g.per * (g.N >= 1024 ? 1 : 1024 / g.N) : kColLines;
  if (g.lines > g.L) g.lines = g.L;
  g.ffts = g.lines / g.per;
  return g;
}

// Complex points of a stage's FFT buffers: stage 1 also runs one inverse FFT
// per column after its forward ones.
__host__ __device__ inline int fft_slots(int stage, const FftGeom &g) {
  return (stage == 1 ? g.lines : g.ffts) * g.N;
}

// Dynamic shared memory of a stage: the FFTs (padded), the twiddles (N/2 +
// N), then (stages 1 and 2) two arrays of the CTA's lines.
__host__ __device__ inline size_t fft_smem(int stage, const FftGeom &g) {
  const int arrays = stage == 0 ? 0 : 2;
  const size_t pts = (size_t)fft_slots(stage, g);
  return sizeof(float2) * (pts + pts / 16 + g.N / 2 + g.N) + sizeof(float) * (size_t)arrays * g.lines * g.N;
}

template <int STAGE>
__global__ void __launch_bounds__(kFftThreads) k_fft(const FftStageArgs a) {
  extern __shared__ float2 s[];
  constexpr bool kRows = STAGE != 1;
  constexpr bool kFwd = STAGE <= 1;
  constexpr int kArrays = kFwd ? 1 : 2;
  const FftGeom G = fft_geom(STAGE, a.W, a.H);
  const int N = G.N, logN = G.logN, nl = G.lines;
  const FftTables tb = kRows ? a.tx : a.ty;
  const int line0 = blockIdx.x * nl;
  float2 *tw = s + pd(fft_slots(STAGE, G));  // [N/2] e^{-2 pi i j / N}
  float2 *tq = tw + N / 2;              // [N]   (cos, sin)(pi k / 2N)
  float *R = reinterpret_cast<float *>(tq + N);  // stages 1 and 2: R[array][line][pos]
  // 16-byte vectors: rows hold 4 consecutive positions of one line, columns
  // the 4 lines of the CTA at one position.
  const int nvec = nl * N / 4;
  auto vec_at = [&](int v, int &l, int &n) -> size_t {  // first element of vector v
    if (kRows) {
      l = v / (N / 4);
      n = (v - l * (N / 4)) * 4;
      return (size_t)(line0 + l) * a.W + n;
    }
    l = 0;
    n = v;
    return (size_t)v * a.W + line0;
  };
  // 1. the lines (all vectors of a thread in flight at once) and the
  // twiddles into shared memory.  Stages 0 and 1 place each value straight
  // at its bit-reversed slot: lines 2p and 2p + 1 are the real and imaginary
  // parts of FFT p, position n of a line goes to v[m], v[m] = x[2m],
  // v[N-1-m] = x[2m+1].
  for (int j = threadIdx.x; j < N / 2; j += kFftThreads) tw[j] = __ldg(tb.tw + j);
  for (int j = threadIdx.x; j < N; j += kFftThreads) tq[j] = __ldg(tb.tq + j);
  __shared__ double red[2 * (kFftThreads / 32)];
  double ov[2] = {0.0, 0.0};  // sum d, sum max(d - cap, 0) (stage 0 from the map)
  if (STAGE == 0 && a.dens) {
    for (int v0 = 0; v0 < nvec; v0 += kBatch * kFftThreads) {
      ulonglong2 q0[kBatch], q1[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int v = v0 + u * kFftThreads + threadIdx.x;
        int l, n;
        const size_t g = vec_at(v < nvec ? v : 0, l, n);
        const ulonglong2 *dp = reinterpret_cast<const ulonglong2 *>(a.dens + g);
        q0[u] = v < nvec ? dp[0] : make_ulonglong2(0ull, 0ull);
        q1[u] = v < nvec ? dp[1] : make_ulonglong2(0ull, 0ull);
      }
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int v = v0 + u * kFftThreads + threadIdx.x;
        if (v >= nvec) break;
        int l, n;
        const size_t g = vec_at(v, l, n);
        ulonglong2 *dp = reinterpret_cast<ulonglong2 *>(a.dens + g);
        dp[0] = make_ulonglong2(0ull, 0ull);
        dp[1] = make_ulonglong2(0ull, 0ull);
        const unsigned long long qq[4] = {q0[u].x, q0[u].y, q1[u].x, q1[u].y};
        float *sf = reinterpret_cast<float *>(s) + (l & 1);
        const int b0 = (l >> 1) << logN;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const double d = (double)(long long)qq[c] * (1.0 / 4294967296.0);
          ov[0] += d;
          ov[1] += fmax(d - a.cap, 0.0);
          sf[2 * pd(b0 + bitrev(vpos(n + c, N), logN))] = (float)(d - a.c0);
        }
      }
    }
  } else {
    const float *src[2] = {a.in_a, a.in_b};
    for (int v0 = 0; v0 < nvec; v0 += kBatch * kFftThreads) {
      float4 q[kArrays][kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int v = v0 + u * kFftThreads + threadIdx.x;
        int l, n;
        const size_t g = vec_at(v < nvec ? v : 0, l, n);
#pragma unroll
        for (int r = 0; r < kArrays; ++r)
          q[r][u] = v < nvec ? __ldg(reinterpret_cast<const float4 *>(src[r] + g)) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int v = v0 + u * kFftThreads + threadIdx.x;
        if (v >= nvec) break;
        int l, n;
        vec_at(v, l, n);
        if (kFwd) {
          const float c4[4] = {q[0][u].x, q[0][u].y, q[0][u].z, q[0][u].w};
          if (kRows) {
            float *sf = reinterpret_cast<float *>(s) + (l & 1);
            const int b0 = (l >> 1) << logN;
#pragma unroll
            for (int c = 0; c < 4; ++c) sf[2 * pd(b0 + bitrev(vpos(n + c, N), logN))] = c4[c];
          } else {
            const int slot = bitrev(vpos(n, N), logN);
            s[pd(slot)] = make_float2(c4[0], c4[1]);
            s[pd(N + slot)] = make_float2(c4[2], c4[3]);
          }
        } else {
#pragma unroll
          for (int r = 0; r < kArrays; ++r) {
            float *d = R + (size_t)r * nl * N;
            if (kRows) {
              *reinterpret_cast<float4 *>(d + (size_t)l * N + n) = q[r][u];
            } else {
              d[0 * N + n] = q[r][u].x;
              d[1 * N + n] = q[r][u].y;
              d[2 * N + n] = q[r][u].z;
              d[3 * N + n] = q[r][u].w;
            }
          }
        }
      }
    }
  }
  __syncthreads();
  // 2. inverse stages: the FFT inputs, bit-reversed.  Line l of array a
  // and of array b (R) -> real and imaginary parts of FFT l.
  auto inv_build = [&]() {
    const float *Ra = R, *Rb = R + (size_t)nl * N;
    for (int e = threadIdx.x; e < nl * N; e += kFftThreads) {
      const int l = e >> logN, k = e & (N - 1);
      const float *ra = Ra + (l << logN), *rb = Rb + (l << logN);
      const int ia = pre_index(a.kind_a, k, N), ib = pre_index(a.kind_b, k, N);
      const float xa = ia >= 0 ? ra[ia] : 0.0f, xb = ib >= 0 ? rb[ib] : 0.0f;
      float2 va, vb;
      if (k == 0) {
        va = make_float2(0.5f * xa, 0.0f);
        vb = make_float2(0.5f * xb, 0.0f);
      } else {
        const int ja = pre_index(a.kind_a, N - k, N), jb = pre_index(a.kind_b, N - k, N);
        const float ya = ja >= 0 ? ra[ja] : 0.0f, yb = jb >= 0 ? rb[jb] : 0.0f;
        const float2 q = tq[k];  // e^{i pi k / 2N} = (q.x, q.y)
        // e^{i theta} (x - i y) / 2
        va = make_float2(0.5f * (q.x * xa + q.y * ya), 0.5f * (q.y * xa - q.x * ya));
        vb = make_float2(0.5f * (q.x * xb + q.y * yb), 0.5f * (q.y * xb - q.x * yb));
      }
      // conj(V_a + i V_b), so that a forward FFT gives the conjugate of the
      // inverse sum
      s[pd((l << logN) + bitrev(k, logN))] = make_float2(va.x - vb.y, -(va.y + vb.x));
    }
  };
  // the inverse outputs, one 16-byte vector per thread and array
  auto inv_out = [&]() {
    for (int v = threadIdx.x; v < nvec; v += kFftThreads) {
      int l0, n0;
      const size_t g = vec_at(v, l0, n0);
      float o[2][4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int l = kRows ? l0 : c, n = kRows ? n0 + c : n0;
        const float2 z = s[pd((l << logN) + vpos(n, N))];
        o[0][c] = z.x * post_sign(a.kind_a, n);
        o[1][c] = -z.y * post_sign(a.kind_b, n);
      }
      *reinterpret_cast<float4 *>(a.out_a + g) = make_float4(o[0][0], o[0][1], o[0][2], o[0][3]);
      *reinterpret_cast<float4 *>(a.out_b + g) = make_float4(o[1][0], o[1][1], o[1][2], o[1][3]);
    }
  };
  if (!kFwd) {
    inv_build();
    __syncthreads();
    fft_core(s, logN, nl, tw);
    inv_out();
    return;
  }
  __syncthreads();
  fft_core(s, logN, G.ffts, tw);
  // 3. forward outputs: stage 0 writes T; stage 1 applies the spectral
  // epilogue, writes phi (when asked), keeps Ex^ and Ey^ of its columns in R
  // and transforms them back along y (Ex: C3, Ey: S3 or SG) before writing.
  float *Rx = R, *Ry = R + (size_t)nl * N;
  for (int v = threadIdx.x; v < nvec; v += kFftThreads) {
    int l0, n0;
    const size_t g = vec_at(v, l0, n0);
    float o[2][4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int l = kRows ? l0 : c, k = kRows ? n0 + c : n0;
      const int b0 = (l >> 1) << logN;
      const float2 z = s[pd(b0 + k)], zc = s[pd(b0 + ((N - k) & (N - 1)))];
      // the line's own spectrum V: (Z[k] + conj Z[N-k]) / 2 for the real
      // part's line, (Z[k] - conj Z[N-k]) / 2i for the imaginary part's
      float vx, vy;
      if ((l & 1) == 0) {
        vx = 0.5f * (z.x + zc.x);
        vy = 0.5f * (z.y - zc.y);
      } else {
        vx = 0.5f * (z.y + zc.y);
        vy = -0.5f * (z.x - zc.x);
      }
      const float2 q = tq[k];
      const float X = q.x * vx + q.y * vy;  // Re(e^{-i pi k / 2N} V[k])
      if (STAGE == 0) {
        o[0][c] = X;
      } else {
        // spectral epilogue at (ky, kx) = (k, line)
        const int kx = line0 + l, ky = k;
        float sc = a.scale;
        if (kx == 0) sc *= 0.5f;
        if (ky == 0) sc *= 0.5f;
        const float den = __ldg(a.gx2 + kx) + __ldg(a.gy2 + ky);
        float ph = 0.0f, ex = 0.0f, ey = 0.0f;
        if (!(den < 1e-30f)) {
          ph = X * sc / den;
          ex = ph * __ldg(a.wx + kx);
          ey = ph * __ldg(a.wy + ky);
        }
        Rx[(l << logN) + ky] = ex;
        Ry[(l << logN) + ky] = ey;
        o[0][c] = ph;
      }
    }
    if (STAGE == 0) *reinterpret_cast<float4 *>(a.out_a + g) = make_float4(o[0][0], o[0][1], o[0][2], o[0][3]);
    if (STAGE == 1 && a.phi) *reinterpret_cast<float4 *>(a.phi + g) = make_float4(o[0][0], o[0][1], o[0][2], o[0][3]);
  }
  if (STAGE == 1) {
    __syncthreads();  // every forward output read before the buffers are reused
    inv_build();
    __syncthreads();
    fft_core(s, logN, nl, tw);
    inv_out();
    return;
  }
  if (STAGE == 0 && a.dens) {
    // the overlap: CTA partials, then the last CTA sums them in CTA order
    __shared__ bool last;
    block_sum2(ov, red);
    if (threadIdx.x == 0) {
      a.part[2 * blockIdx.x] = ov[0];
      a.part[2 * blockIdx.x + 1] = ov[1];
      __threadfence();
      last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t[2] = {0.0, 0.0};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
      t[0] += __ldcg(a.part + 2 * b);
      t[1] += __ldcg(a.part + 2 * b + 1);
    }
    block_sum2(t, red);
    if (threadIdx.x == 0) {
      const double ovl = (t[0] < 1e-30) ? 0.0 : t[1] / t[0];  // compute_overlap
      a.sc->overlap = ovl;
      a.log[a.sc->iter].overlap = ovl;
      *a.ticket = 0u;
    }
  }
}

}  // namespace

bool fft_supported(int W, int H) {
  auto pow2 = [](int n) { return n >= 16 && n <= 1024 && (n & (n - 1)) == 0; };
  return pow2(W) && pow2(H);
}

void fft_tables_host(int N, float2 *tw, float2 *tq) {
  const double pi = 3.14159265358979323846;
  for (int j = 0; j < N / 2; ++j) {
    const double t = 2.0 * pi * j / N;
    tw[j] = make_float2((float)std::cos(t), (float)-std::sin(t));
  }
  for (int k = 0; k < N; ++k) {
    const double t = pi * k / (2.0 * N);
    tq[k] = make_float2((float)std::cos(t), (float)std::sin(t));
  }
}

cudaError_t launch_fft_stage(int stage, const FftStageArgs &a, cudaStream_t s) {
  const FftGeom g = fft_geom(stage, a.W, a.H);
  const int grid = (g.L + g.lines - 1) / g.lines;
  const size_t smem = fft_smem(stage, g);
  // The shared-memory limit is raised to the stage's largest need (a
  // 1024 x 1024 grid) every time: the same value from every thread, so
  // contexts launching from several host threads never lower it under one
  // another's launch.
  const int cap = (int)fft_smem(stage, fft_geom(stage, 1024, 1024));
  cudaError_t e = cudaSuccess;
  switch (stage) {
    case 0:
      e = cudaFuncSetAttribute(k_fft<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
      if (e == cudaSuccess) k_fft<0><<<grid, kFftThreads, smem, s>>>(a);
      break;
    case 1:
      e = cudaFuncSetAttribute(k_fft<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
      if (e == cudaSuccess) k_fft<1><<<grid, kFftThreads, smem, s>>>(a);
      break;
    default:
      e = cudaFuncSetAttribute(k_fft<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
      if (e == cudaSuccess) k_fft<2><<<grid, kFftThreads, smem, s>>>(a);
      break;
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace eplace
