// noalloc.cu -- the density stage (cell -> bin overlap map and overlap
// metric) for callers that cannot allocate device memory.
//
// Some callers run where cudaMalloc is not available to them: code inside a
// CUDA-graph capture, a real-time loop that must not allocate or take the
// allocator's locks, or a host application whose device memory is owned and
// handed out by another component.  They own their inputs and outputs
// already; what they cannot do is give this library the working memory the
// density stage needs (the fixed-point accumulation map, the per-block
// partial sums and the completion counter).  For them the scratch lives in
// one file-scope __device__ array, sized for at most kNoAllocMaxBins bins
// (512 x 512).  It is part of the library image: every GPU that loads
// libeplace.so holds it (about 2 MiB) until the process exits.
//
// The kernels are the library's own scatter and finalise kernels; only the
// scratch they are given differs.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>

#include "../../include/eplace.h"
#include "kernels.cuh"

namespace eplace {
namespace {

constexpr size_t kNoAllocMaxBins = 512 * 512;
constexpr int kNoAllocMaxBlocks = 1024;  // finalise grid cap (partials below)

// Layout of the scratch array (byte offsets, each 256-aligned):
//   [0, kMapBytes)                fixed-point bin map, must start at zero
//   [kPartOff, +kPartBytes)       per-block partial sums of the finalise
//   [kTicketOff, +256)            completion counter, must start at zero
//   [kScalOff, +256)              loop scalars the finalise writes into
//   [kLogOff, +256)               one per-iteration log record
constexpr size_t kMapBytes = kNoAllocMaxBins * sizeof(unsigned long long);
constexpr size_t kPartOff = kMapBytes;
constexpr size_t kPartBytes = 2 * kNoAllocMaxBlocks * sizeof(double);
constexpr size_t kTicketOff = kPartOff + kPartBytes;
constexpr size_t kScalOff = kTicketOff + 256;
constexpr size_t kLogOff = kScalOff + 256;
constexpr size_t kScratchBytes = kLogOff + 256;
static_assert(sizeof(DevScalars) <= 256 && sizeof(IterLog) <= 256, "scratch slots too small");

static __device__ __align__(256) unsigned char g_density_scratch[kScratchBytes];

// Device address of g_density_scratch per device.  In host code the symbol
// is only a host-side stand-in, so the address is looked up once per device,
// with that device current, and cached.
std::mutex g_mu;
void *g_addr[128] = {};

eplace_status scratch_for_current_device(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return EPLACE_ERR_NO_DEVICE;
  if (dev < 0 || dev >= 128) return EPLACE_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_density_scratch) != cudaSuccess || !p) return EPLACE_ERR_CUDA;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return EPLACE_OK;
}

}  // namespace
}  // namespace eplace

using namespace eplace;

extern "C" eplace_status eplace_density_noalloc(const float *pos_xy, const float *half_wh, uint32_t num_cells,
                                                int32_t width, int32_t height, int32_t bins_x, int32_t bins_y,
                                                double *density, double *overlap, void *stream) {
  if (width <= 0 || height <= 0 || bins_x <= 0 || bins_y <= 0 || width % bins_x || height % bins_y)
    return EPLACE_ERR_INVALID;
  if ((size_t)bins_x * (size_t)bins_y > kNoAllocMaxBins) return EPLACE_ERR_INVALID;  // over the scratch size
  if (!density || !overlap || (num_cells && !pos_xy)) return EPLACE_ERR_INVALID;
  void *base = nullptr;
  eplace_status st = scratch_for_current_device(&base);
  if (st != EPLACE_OK) return st;
  int sms = 0, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return EPLACE_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char *b = static_cast<unsigned char *>(base);
  const int nb = bins_x * bins_y;
  auto *map = reinterpret_cast<unsigned long long *>(b);
  auto *part = reinterpret_cast<double *>(b + kPartOff);
  auto *ticket = reinterpret_cast<unsigned *>(b + kTicketOff);
  auto *sc = reinterpret_cast<DevScalars *>(b + kScalOff);
  auto *lg = reinterpret_cast<IterLog *>(b + kLogOff);
  // The scratch keeps the previous call's contents: clear the map, the
  // counter and the scalar slot (iteration 0, read by the finalise).
  if (cudaMemsetAsync(map, 0, (size_t)nb * sizeof(unsigned long long), s) != cudaSuccess ||
      cudaMemsetAsync(ticket, 0, 256, s) != cudaSuccess || cudaMemsetAsync(sc, 0, 256, s) != cudaSuccess)
    return EPLACE_ERR_CUDA;
  const float sx = (float)(width / bins_x), sy = (float)(height / bins_y);
  ScatterArgs a{reinterpret_cast<const float2 *>(pos_xy), reinterpret_cast<const float2 *>(half_wh), nullptr,
                nullptr, 0u, num_cells, bins_x, bins_y, sx, sy, 1.0f / sx, 1.0f / sy, map};
  if (num_cells) {
    long long g = ((long long)num_cells + kScatterBlock - 1) / kScatterBlock;
    if (g > (long long)sms * 16) g = (long long)sms * 16;
    if (launch_scatter(a, (int)g, s) != cudaSuccess) return EPLACE_ERR_CUDA;
  }
  long long fg = ((long long)nb + kFinalBlock - 1) / kFinalBlock;
  if (fg > (long long)sms * 2) fg = (long long)sms * 2;
  if (fg > kNoAllocMaxBlocks) fg = kNoAllocMaxBlocks;
  FinalArgs f{map, nb, (double)sx * (double)sy, 0.0, nullptr, nullptr, nullptr, density, 0, part, ticket, sc, lg};
  if (launch_density_final(f, (int)fg, s) != cudaSuccess) return EPLACE_ERR_CUDA;
  if (cudaMemcpyAsync(overlap, &sc->overlap, sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return EPLACE_ERR_CUDA;
  return EPLACE_OK;
}
