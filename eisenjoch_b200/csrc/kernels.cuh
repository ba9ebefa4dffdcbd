// kernels.cuh -- device-side state of one placement context and the launch
// wrappers of the hot-path kernels (defined in kernels.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace eplace {

// Scalars of the Nesterov loop kept on the device so a whole legalisation
// interval can be replayed as one CUDA graph without host round trips.
struct DevScalars {
  double lam;          // density_penalty (electro_place/mod.rs:100)
  double step[2];      // current step sizes (NesterovSolver::step_size)
  double overlap;      // overlap of the current iteration's density
  int32_t lam_init;    // density_initialized
  int32_t iter;        // index of the next iteration to execute
  int32_t err;         // non-zero: a bounded wait gave up
  int32_t pad_;
  int64_t spin_cycles; // bound of every grid-barrier wait in SM clock cycles (0: the default, ~2 s)
};

// One record per executed iteration (fields of the reference log line).
struct IterLog {
  double overlap;
  double lam;
  double step_norm[2];  // NesterovSolver::step return values
  double alpha[2];      // step sizes used by the FISTA step
};

// Degree classes of the WA kernel over the degree-sorted nets: class j holds
// the nets of degree (kWaDegHi[j-1], kWaDegHi[j]] (class 0 from degree 2;
// nets of fewer pins have no gradient) and runs kWaGroup[j] lanes per net,
// kWaSlots[j] pin slots per lane; the last class (more than 224 pins) runs a
// warp per net over its CSR pins in three passes.
constexpr int kWaClasses = 9;
constexpr int kWaDegHi[kWaClasses] = {2, 4, 8, 16, 32, 64, 128, 224, 0x7fffffff};
constexpr int kWaGroup[kWaClasses] = {1, 1, 2, 4, 8, 32, 32, 32, 32};
// Padded pin table: lane l of a net's group holds that net's pins l, l + G,
// l + 2G, ... in its kWaSlots[j] consecutive slots (one 8-, 16- or 32-byte
// load), unused slots 0xffffffff; a net takes G * kWaSlots[j] slots.
constexpr int kWaSlots[kWaClasses] = {2, 4, 4, 4, 4, 2, 4, 8, 0};

// The WA gradient of a cell is accumulated as one 64-bit integer per cell:
// x and y in fixed point (scale 2^k), packed as gx + 2^32 gy and summed with
// one 64-bit atomic per pin.  Two's-complement sums are exact modulo 2^64,
// so while |sum gx| and |sum gy| stay below 2^31 the low word is the x sum
// and the rest the y sum.  k is chosen per problem from the largest pin
// count of a cell (a pin's gradient is below 2 in magnitude; the bound used
// is 4 per pin), at most 24.
__host__ __device__ inline unsigned long long pack_grad(long long gx, long long gy) {
  return (unsigned long long)gx + ((unsigned long long)gy << 32);
}
__host__ __device__ inline void unpack_grad(unsigned long long v, long long *gx, long long *gy) {
  const int lo = (int)(unsigned)(v & 0xffffffffull);
  *gx = lo;
  *gy = (long long)(v - (unsigned long long)(long long)lo) >> 32;
}

struct WaClass {
  int first_net;        // index into the degree-sorted CSR
  int nets;
  int first_warp;       // warps of the classes before this one
  long long slot_base;  // first slot of the class in the padded pin table (multiple of 4)
};

struct WaArgs {
  WaClass cls[kWaClasses];
  int nwarps;
  const uint32_t *slots;    // padded pin table (kWaSlots)
  const uint32_t *net_off;
  const uint32_t *pin_cell;
  const float2 *pos;        // [N + F]: look-ahead positions, then fixed cells
  unsigned long long *acc;  // [N] packed fixed-point gradient (see pack_grad)
  uint32_t N;
  float gamma;
  float grad_scale;         // 2^k fixed-point scale of the packed gradient
};

struct ScatterArgs {
  const float2 *pos;
  const float2 *half;       // half extents, nullptr => unit cells
  const uint8_t *mflag;     // [N] 1 for a macro, nullptr: no macro list (general loop when half is set)
  const uint32_t *mac_idx;  // [n_mac] the macros' cell ids
  uint32_t n_mac;
  uint32_t N;
  int BX, BY;
  int isx, isy;              // sites per bin along x / y
  unsigned long long *dens; // [BY * BX] fixed point
};

struct FinalArgs {
  unsigned long long *dens;
  int nb;
  double cap;               // capacity per bin (sites per bin)
  double c0;                // constant removed before the transform
  float *rho;               // FP32 charge map (SIMT transform), or nullptr
  __nv_bfloat16 *rho_hi;    // BF16 hi/lo charge map (tensor-core transform), or nullptr
  __nv_bfloat16 *rho_lo;
  double *dens_out;         // optional FP64 copy (stage entry)
  int vec4;                 // set by launch_density_final: every pointer allows 16-byte groups
  double *part;             // [2 * grid]
  unsigned *ticket;
  DevScalars *sc;
  IterLog *log;
};

// C = A B with leading dimensions lda / ldb / ldc.  a_mir = +1 / -1 reads
// A(r, k) as A(r, k) +/- A(r, a_full - 1 - k) (columns folded about the
// middle of a_full); b_mir likewise folds B's rows about the middle of
// b_full.  The spectral epilogue takes output row r as frequency
// ky = 2 r + row_par (row_par < 0: ky = r) and, with col_split, column c as
// kx = 2 c (c < N/2) or 2 (c - N/2) + 1 (even frequencies first).
struct GemmOp {
  const float *A;
  const float *B;
  float *C;
  float *C2;
  int lda, ldb, ldc;
  int a_mir, a_full;
  int b_mir, b_full;
  int row_par, col_split;
};

struct SpectralArgs {
  const float *wx, *gx2;   // [BX]: pi kx / W, 2(1 - cos(pi kx / W))
  const float *wy, *gy2;   // [BY]
  float scale;             // 4 / (W H)
  float *phi;              // optional scaled potential spectrum
};

struct StepArgs {
  uint32_t N;
  int BX, BY;
  int isx, isy;              // sites per bin along x / y
  float maxx, maxy;
  float2 *look;             // [N] (fixed cells follow in the same buffer)
  const float2 *half;       // nullptr => unit cells
  const float *area;
  const uint8_t *mflag;     // [N] 1 for a macro (w*h > 1), nullptr when there are none
  const uint32_t *mac_idx;  // [n_mac] the macros' cell ids, ascending
  uint32_t n_mac;
  const float *pw;
  unsigned long long *acc;  // [N] packed WA accumulator, read then zeroed
  double grad_inv;          // 1 / WaArgs::grad_scale
  const float *Ex, *Ey;
  float2 *x, *xp, *g, *gprev;
  float2 *tmp_wl, *tmp_den; // [N] scratch for the penalty-initialisation phase
  const double *mom;        // momentum per iteration
  DevScalars *sc;
  IterLog *log;
  double *part;             // [4 * grid]
  double *part2;            // [2 * grid] step-norm partials
  double *part_b;           // [4 * grid] pass-2 partials of the split form
  unsigned *bar;            // grid barrier: words 0-1 are one 64-bit arrival count
  unsigned *ticket;
  int mode;                 // 0: full step (cooperative); 1: gather only (tmp_den <- density
                            // gradient); 2/3/4: phase A / penalty-init pass / phase C
};

struct HpwlArgs {
  const uint32_t *net_off;
  const uint32_t *pin_cell;
  const uint8_t *has_driver;
  const int2 *loc;          // [N + F] integer pin locations
  uint32_t NN;
  unsigned long long *total;
};

cudaError_t launch_wa(const WaArgs &a, int grid, cudaStream_t s);
cudaError_t launch_scatter(const ScatterArgs &a, int grid, cudaStream_t s);
cudaError_t launch_density_final(const FinalArgs &a, int grid, cudaStream_t s);
// C[b] = A[b] (M x K) * B[b] (K x N), row-major FP32; batches from ops[0..nb).
// tile: 64 or 32 (CTA tile edge), 0 = pick by grid size.  When 64 divides K
// the sum is split into four K quarters (a cluster of four CTAs per tile)
// added in quarter order; either way both tiles sum every output in the
// same order, so the tile never changes the bits.
cudaError_t launch_sgemm(const GemmOp *ops_dev, int nb, int M, int N, int K, cudaStream_t s, int tile = 0);
// As above with the spectral epilogue: C = Ex_hat, C2 = Ey_hat.
cudaError_t launch_sgemm_spectral(const GemmOp *ops_dev, int nb, int M, int N, int K,
                                  const SpectralArgs &sp, cudaStream_t s, int tile = 0);
// The butterflies that complete a folded transform (see api.cu):
// cols: out[r][x] = E[r][x] + O[r][x], out[r][W-1-x] = sig (E - O), x < W/2,
//       E / O: [H][W/2]; nb products (blockIdx.z), each its own E, O, out, sig.
// rows: out[y][x] = E[y][x] + O[y][x], out[H-1-y][x] = sig (E - O), y < H/2,
//       E / O: [H/2][W].
struct FlyOp {
  const float *E, *O;
  float *out;
  float sig;
};
cudaError_t launch_fly_cols(const FlyOp *ops_dev, int nb, int H, int W, cudaStream_t s);
cudaError_t launch_fly_rows(const FlyOp *ops_dev, int nb, int H, int W, cudaStream_t s);
cudaError_t launch_step(const StepArgs &a, int grid, cudaStream_t s);
// The same step as three ordinary launches (modes 2, 3, 4): no grid barrier,
// safe beside long-running kernels of other streams.
cudaError_t launch_step_split(const StepArgs &a, int grid, cudaStream_t s);
int step_max_grid(int device);
cudaError_t launch_hpwl(const HpwlArgs &a, int grid, cudaStream_t s);

constexpr int kWaBlock = 256;
constexpr int kScatterBlock = 256;
constexpr int kFinalBlock = 256;
constexpr int kStepBlock = 512;
constexpr int kHpwlBlock = 256;

}  // namespace eplace
