// fft.cuh -- the spectral Poisson solve's transforms as FFTs (FP32).
//
// The linear maps of density.rs:96-166 (the same as the DCT-matrix GEMMs of
// kernels.cu / dct_tc.cu), in three stages per iteration:
//   stage 0  T   = DCT-II along x of rho                        (rows)
//   stage 1  A   = DCT-II along y of T; the spectral scale, Poisson divide
//                  and field weights -> Ex^, Ey^ (and phi); then along y
//                  U = C3 of Ex^, V = S3 (reference field) or SG
//                  (potential-gradient field) of Ey^            (columns)
//   stage 2  Ex  = S3 or SG along x of U;  Ey = C3 along x of V (rows)
// (the 2D transforms are separable, so the inverse may take y before x),
// with, for a line of length N and theta = pi k (n + 1/2) / N,
//   DCT-II  X[k] = sum_n x[n] cos(theta)
//   C3      x[n] = sum_k c_k X[k] cos(theta),  c_0 = 1/2
//   S3      x[n] = sum_k d_k X[k] sin(pi (k + 1)(n + 1/2) / N),  d_{N-1} = 1/2
//   SG      x[n] = -sum_k X[k] sin(theta)
// Each is one N-point complex FFT (Makhoul's reordering):
//   DCT-II: v[m] = x[2m], v[N-1-m] = x[2m+1]; X[k] = Re(e^{-i pi k/2N} V[k]).
//   C3:     V[0] = X[0]/2, V[k] = e^{i pi k/2N} (X[k] - i X[N-k]) / 2;
//           v = sum_k V[k] e^{2 pi i k m / N} is real; x[2m] = v[m],
//           x[2m+1] = v[N-1-m].
//   S3(X)[n] = (-1)^n C3(X reversed)[n];
//   SG(X)[n] = -(-1)^n C3(Y)[n], Y[0] = 0, Y[k] = X[N-k].
// Two real transforms share one complex FFT: two lines of the same array
// (the forward transforms, split by the conjugate symmetry of real inputs)
// or the same line of two arrays (the inverse ones, whose outputs are real).
// O(N log N) per line instead of the GEMMs' O(N^2); FP32 rounding error grows
// with log N instead of N.  Power-of-two grids of 16 .. 1024 bins per axis.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace eplace {

// Twiddles of one transform length N (host-computed in FP64, stored FP32).
struct FftTables {
  const float2 *tw;  // [N/2] e^{-2 pi i j / N}
  const float2 *tq;  // [N]   (cos, sin)(pi k / 2N)
};

// Line transforms of stage 2 and 3 inputs.
enum FftKind { FFT_C3 = 0, FFT_S3 = 1, FFT_SG = 2 };

struct FftStageArgs {
  int W, H;               // bin grid
  const float *in_a, *in_b;
  float *out_a, *out_b;
  FftTables tx, ty;       // length W and length H tables
  int kind_a, kind_b;     // FftKind of the inverse transform of each array (stages 1, 2)
  // stage 1 spectral epilogue (same formula as the GEMM epilogues)
  const float *wx, *gx2, *wy, *gy2;
  float scale;            // 4 / (W H)
  float *phi;             // optional [H][W] potential spectrum
  // Stage 0 straight from the fixed-point density map (the finalise fused
  // in): with dens set, the stage reads the map instead of in_a, forms
  // rho = d - c0, clears the map for the next iteration, and sums the
  // overlap (density.rs:79-86: sum d and sum max(d - cap, 0)) into part[]
  // per CTA; the last CTA to finish writes sc->overlap and the iteration's
  // log entry.
  unsigned long long *dens;
  double cap, c0;
  double *part;           // [2 * CTAs of stage 0]
  unsigned *ticket;
  DevScalars *sc;
  IterLog *log;
};

bool fft_supported(int W, int H);
// Host-side tables for length N: tw [N/2], tq [N].
void fft_tables_host(int N, float2 *tw, float2 *tq);
// One of the three stages (0..2) on stream s.
cudaError_t launch_fft_stage(int stage, const FftStageArgs &a, cudaStream_t s);

}  // namespace eplace
