// dct_tc.cu -- the DCT-matrix GEMMs of the Poisson solve on the 5th-gen
// tensor cores (tcgen05, sm_100a), BF16 three-term split, FP32 accumulate.
//
// Each GEMM is C = A * B with A (M x K) and B^T (N x K) both K-major in
// global memory, each held as a hi/lo pair of BF16 planes (x = hi + lo,
// hi = bf16(x), lo = bf16(x - hi)).  Per 16-wide K step the CTA issues
//   D += A_hi B_hi + A_hi B_lo + A_lo B_hi
// into one TMEM accumulator (the lo*lo term, ~2^-16 relative, is dropped).
// Tiles: 128 (M) x BN (N) per CTA, K blocks of 64 (one 128-byte swizzle
// atom), a STAGES-deep TMA -> shared-memory ring with mbarriers; thread 0
// issues TMA, thread 32 issues the MMAs, all four warps run the epilogue
// (warp w reads TMEM lanes 32w..32w+31 = tile rows).  No cluster multicast.
//
// Epilogues write the next GEMM's operand directly (split, and transposed
// where the next GEMM needs C^T as its K-major B^T), or the spectral
// Poisson scaling (density.rs:114-153), or the final FP32 field.
//
// Every mbarrier wait is bounded: on timeout the CTA records an error in
// *err, skips the remaining work, waits (bounded again) for the MMAs and
// tensor loads it has in flight, releases its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "dct_tc.cuh"

namespace eplace {
namespace {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr long long kWaitCycles = 4000000000ll;  // ~2 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// K-major, 128-byte swizzled operand tile (rows of 64 BF16 = 128 B, 8-row
// groups 1024 B apart): LBO 16 B (unused for this layout), SBO 1024 B,
// descriptor version 1, layout SWIZZLE_128B (2).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void split_store(__nv_bfloat16 *hi, __nv_bfloat16 *lo, size_t o, float v) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  hi[o] = h;
  lo[o] = __float2bfloat16_rn(v - __bfloat162float(h));
}

template <int BN, int STAGES>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;  // 16 KB
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int TOTAL = STAGE_BYTES * STAGES + 1024 /* align */ + 256 /* barriers */;
};

template <int BN, int STAGES>
__global__ void __launch_bounds__(128, 1)
    k_tc_gemm(const __grid_constant__ TcGemmMaps maps, const TcGemmEpi epi, int M, int N, int K) {
  using S = Smem<BN, STAGES>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + S::STAGE_BYTES * STAGES);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
  __shared__ int failed;
  __shared__ int s_issued;  // stage loads the producer issued

  const int z = blockIdx.z;
  const TcOperandMaps &om = maps.op[z];
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = K / BK;

  if (threadIdx.x == 0) {
    failed = 0;
    s_issued = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0) {
    // TMA producer
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1)) {
        atomicExch(&failed, 1);
        break;
      }
      ++issued;
      uint8_t *st = smem + s * S::STAGE_BYTES;
      mbar_expect_tx(&full[s], S::STAGE_BYTES);
      tma_load_2d(st, &om.a_hi, kb * BK, m0, &full[s]);
      tma_load_2d(st + S::A_BYTES, &om.a_lo, kb * BK, m0, &full[s]);
      const CUtensorMap *bh = BN == 32 ? &om.b_hi32 : (BN == 128 ? &om.b_hi128 : &om.b_hi);
      const CUtensorMap *bl = BN == 32 ? &om.b_lo32 : (BN == 128 ? &om.b_lo128 : &om.b_lo);
      tma_load_2d(st + 2 * S::A_BYTES, bh, kb * BK, n0, &full[s]);
      tma_load_2d(st + 2 * S::A_BYTES + S::B_BYTES, bl, kb * BK, n0, &full[s]);
    }
    s_issued = issued;
  } else if (threadIdx.x == 32) {
    // MMA issuer: M = 128, N = BN, BF16 x BF16 -> FP32, both K-major.
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
    bool ok = true;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(&full[s], (kb / STAGES) & 1)) {
        ok = false;
        atomicExch(&failed, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(smem + s * S::STAGE_BYTES);
      const uint32_t a_hi = base, a_lo = base + S::A_BYTES;
      const uint32_t b_hi = base + 2 * S::A_BYTES, b_lo = b_hi + S::B_BYTES;
#pragma unroll
      for (int k = 0; k < BK / 16; ++k) {
        const uint32_t off = k * 32;  // 16 BF16 along K inside the swizzle atom
        const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
        mma_bf16(tmem, make_desc(a_hi + off), make_desc(b_hi + off), idesc, acc);
        mma_bf16(tmem, make_desc(a_hi + off), make_desc(b_lo + off), idesc, 1u);
        mma_bf16(tmem, make_desc(a_lo + off), make_desc(b_hi + off), idesc, 1u);
      }
      mma_commit(&empty[s]);
    }
    // Also after a timeout: `done` then tracks every MMA issued so far, so
    // the CTA's wait on it below drains them before TMEM is released.
    mma_commit(done);
    (void)ok;
  }
  __syncwarp();
  // Epilogue: warp w owns accumulator rows 32w..32w+31 (TMEM lanes).
  bool ok = mbar_wait(done, 0);
  __syncthreads();
  if (failed) ok = false;
  if (!ok && threadIdx.x == 0) {
    // After a timeout anywhere in the CTA, the loads still in flight (at
    // most the last STAGES issued, one per stage) land before the CTA may
    // leave: bounded waits on their stages' full barriers.
    for (int kb = max(0, s_issued - STAGES); kb < s_issued; ++kb) mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int r = m0 + warp * 32 + lane;
    const TcEpiOut &out = epi.out[z];
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (r >= M) continue;
      if (epi.mode == TC_EPI_F32) {
        float *dst = out.f32 + (size_t)r * N + n0 + c0;
#pragma unroll
        for (int i = 0; i < 32; i += 4)
          *reinterpret_cast<float4 *>(dst + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      } else if (epi.mode == TC_EPI_SPLIT_T) {
        // C^T (N x M) row-major: the next GEMM's K-major B^T.
#pragma unroll
        for (int i = 0; i < 32; ++i) split_store(out.hi, out.lo, (size_t)(n0 + c0 + i) * M + r, v[i]);
      } else {
        // Spectral scaling + Poisson + field spectra (density.rs:114-153),
        // written split and row-major as the A operands of the next GEMMs,
        // 8 BF16 per 16-byte store.
        const int ky = r;
        const float gy2 = epi.gy2[ky], wy = epi.wy[ky];
        const float sy = (ky == 0) ? 0.5f * epi.scale : epi.scale;
#pragma unroll  // constant indices into v[]: it stays in registers
        for (int j = 0; j < 32; j += 8) {
          uint32_t exh[4], exl[4], eyh[4], eyl[4];
#pragma unroll
          for (int i = 0; i < 8; i += 2) {
            float e_x[2], e_y[2];
#pragma unroll
            for (int t = 0; t < 2; ++t) {
              const int kx = n0 + c0 + j + i + t;
              const float s = (kx == 0) ? 0.5f * sy : sy;
              const float den = epi.gx2[kx] + gy2;
              float phi = 0.f;
              if (!(den < 1e-30f)) phi = v[j + i + t] * s / den;
              e_x[t] = phi * epi.wx[kx];
              e_y[t] = phi * wy;
              if (epi.phi) epi.phi[(size_t)ky * N + kx] = phi;
            }
            const __nv_bfloat162 hx = __floats2bfloat162_rn(e_x[0], e_x[1]);
            const __nv_bfloat162 lx = __floats2bfloat162_rn(e_x[0] - __low2float(hx), e_x[1] - __high2float(hx));
            const __nv_bfloat162 hy = __floats2bfloat162_rn(e_y[0], e_y[1]);
            const __nv_bfloat162 ly = __floats2bfloat162_rn(e_y[0] - __low2float(hy), e_y[1] - __high2float(hy));
            exh[i / 2] = *reinterpret_cast<const uint32_t *>(&hx);
            exl[i / 2] = *reinterpret_cast<const uint32_t *>(&lx);
            eyh[i / 2] = *reinterpret_cast<const uint32_t *>(&hy);
            eyl[i / 2] = *reinterpret_cast<const uint32_t *>(&ly);
          }
          const size_t o = (size_t)ky * N + n0 + c0 + j;  // multiple of 8 elements: 16-byte aligned
          *reinterpret_cast<uint4 *>(out.hi + o) = make_uint4(exh[0], exh[1], exh[2], exh[3]);
          *reinterpret_cast<uint4 *>(out.lo + o) = make_uint4(exl[0], exl[1], exl[2], exl[3]);
          *reinterpret_cast<uint4 *>(out.hi2 + o) = make_uint4(eyh[0], eyh[1], eyh[2], eyh[3]);
          *reinterpret_cast<uint4 *>(out.lo2 + o) = make_uint4(eyl[0], eyl[1], eyl[2], eyl[3]);
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(epi.err, 2);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

}  // namespace

bool tc_shape_ok(int M, int N, int K) { return M % BM == 0 && N % kTcBN == 0 && K % BK == 0 && M > 0; }

template <int BN, int STAGES>
cudaError_t launch_cfg(const TcGemmMaps &maps, const TcGemmEpi &epi, int nbatch, int M, int N, int K,
                       cudaStream_t s) {
  using S = Smem<BN, STAGES>;
  // The shared-memory opt-in is per device: set it once on each.
  static std::atomic<bool> attr[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr[dev].load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(k_tc_gemm<BN, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         S::TOTAL);
    if (e != cudaSuccess) return e;
    attr[dev].store(true, std::memory_order_release);
  }
  dim3 grid(N / BN, M / BM, nbatch);
  k_tc_gemm<BN, STAGES><<<grid, 128, S::TOTAL, s>>>(maps, epi, M, N, K);
  return cudaGetLastError();
}

// Tile shape by grid size (measured on 512^2 and 1024^2 bin grids): a grid
// of 128 x 64 tiles that covers at most half the SMs takes 128 x 32 tiles
// (twice the CTAs); one that would need a second wave takes 128 x 128 tiles
// with a 3-deep ring when those fit one wave, else two smaller rings (2
// stages, 97 KB) so that two CTAs share an SM and one's epilogue overlaps
// the other's main loop; in between, 128 x 64 with a 4-deep ring.
// Each output sums its K steps in the same order whatever the tile.
cudaError_t launch_tc_gemm(const TcGemmMaps &maps, const TcGemmEpi &epi, int nbatch, int M, int N, int K,
                           cudaStream_t s) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long ctas = (long)(N / kTcBN) * (M / BM) * nbatch;
  if (2 * ctas <= sms) return launch_cfg<32, 4>(maps, epi, nbatch, M, N, K, s);
  // A grid that 128 x 64 tiles would spread over two waves fits one wave of
  // 128 x 128 tiles: each A tile is loaded half as often (the operand
  // traffic from L2 sets these GEMMs' time), one CTA per SM.
  if (ctas > sms && N % 128 == 0 && ctas / 2 <= sms) return launch_cfg<128, 3>(maps, epi, nbatch, M, N, K, s);
  if (ctas > sms) return launch_cfg<64, 2>(maps, epi, nbatch, M, N, K, s);
  return launch_cfg<64, 4>(maps, epi, nbatch, M, N, K, s);
}

}  // namespace eplace
