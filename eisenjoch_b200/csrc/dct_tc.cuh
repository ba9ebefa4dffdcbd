// dct_tc.cuh -- tcgen05 BF16x3 DCT GEMMs: operand tensor maps and epilogues.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace eplace {

constexpr int kTcBN = 64;  // widest CTA tile N (M is 128); N must be a multiple of it

// TMA maps of one GEMM's operands: A (M x K) and B^T (N x K), hi and lo; the
// B maps three times, for the 64-, 32- and 128-column tiles.
struct TcOperandMaps {
  CUtensorMap a_hi, a_lo, b_hi, b_lo, b_hi32, b_lo32, b_hi128, b_lo128;
};

// Up to two GEMMs of the same shape in one launch (blockIdx.z).
struct TcGemmMaps {
  TcOperandMaps op[2];
};

enum TcEpiMode {
  TC_EPI_F32 = 0,       // C row-major FP32
  TC_EPI_SPLIT_T = 1,   // C^T row-major as BF16 hi/lo (next GEMM's B^T)
  TC_EPI_SPECTRAL = 2,  // Poisson scaling -> Ex_hat (hi/lo), Ey_hat (hi2/lo2), row-major
};

struct TcEpiOut {
  float *f32;
  __nv_bfloat16 *hi, *lo, *hi2, *lo2;
};

struct TcGemmEpi {
  int mode;
  TcEpiOut out[2];
  const float *wx, *gx2, *wy, *gy2;  // spectral tables
  float scale;
  float *phi;                        // optional scaled potential spectrum
  int *err;                          // set non-zero when a bounded wait gives up
};

bool tc_shape_ok(int M, int N, int K);
cudaError_t launch_tc_gemm(const TcGemmMaps &maps, const TcGemmEpi &epi, int nbatch, int M, int N, int K,
                           cudaStream_t s);

}  // namespace eplace
