// noalloc.cu -- the density stage (cell -> bin overlap map and overlap
// metric) for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a real-time control loop that must
// not take the allocator's locks or stall on it, a host application whose
// device memory is handed out by another component (its own pool, a
// framework's caching allocator) and may not be grown behind its back, or
// code running under a fixed device-memory budget.  They own their inputs
// and outputs already; what they cannot do is give this library the working
// memory the density stage needs (the fixed-point accumulation map, the
// per-block partial sums and the completion counter).  For them the scratch
// lives in one file-scope __device__ array, sized for at most
// kNoAllocMaxBins bins (512 x 512).  It is part of the library image: every
// GPU that loads libeplace.so holds it (about 2 MiB) until the process
// exits.
//
// The kernels are the library's own scatter and finalise kernels; only the
// scratch they are given differs.
#include <cuda.h>
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

// Device address of g_density_scratch.  In host code the symbol is only a
// host-side stand-in, so its device address is looked up with the device
// current (cudaGetSymbolAddress) at set-up and cached per device.  The
// cache entry also records the unique id of the CUDA context it was looked
// up in: after cudaDeviceReset (or any other end of the primary context)
// the module is loaded again, possibly elsewhere, and the next call looks
// the address up again instead of using a stale one.  The driver calls are
// reached through the runtime's entry-point table, so the library does not
// link libcuda directly.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

struct ScratchSlot {
  unsigned long long ctx_id = 0;
  void *addr = nullptr;
};

std::mutex g_mu;
ScratchSlot g_slot[128];
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

// Id of the current context; 0 when no context is current yet.
eplace_status current_context_id(unsigned long long *id) {
  *id = 0;
  if (!g_ctx_current || !g_ctx_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return EPLACE_ERR_CUDA;
    g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    g_ctx_id = reinterpret_cast<CtxGetIdFn>(f2);
  }
  CUcontext c = nullptr;
  if (g_ctx_current(&c) != CUDA_SUCCESS) return EPLACE_ERR_CUDA;
  if (!c) return EPLACE_OK;
  return g_ctx_id(c, id) == CUDA_SUCCESS ? EPLACE_OK : EPLACE_ERR_CUDA;
}

eplace_status scratch_for_current_device(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return EPLACE_ERR_NO_DEVICE;
  if (dev < 0 || dev >= 128) return EPLACE_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> g(g_mu);
  unsigned long long id = 0;
  eplace_status st = current_context_id(&id);
  if (st != EPLACE_OK) return st;
  ScratchSlot &slot = g_slot[dev];
  if (id == 0 || !slot.addr || slot.ctx_id != id) {
    // Set-up: the symbol's device address in the current context (the
    // lookup also creates the device's primary context when none is current
    // yet, so the id is read again afterwards).
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_density_scratch) != cudaSuccess || !p) return EPLACE_ERR_CUDA;
    st = current_context_id(&id);
    if (st != EPLACE_OK) return st;
    if (id == 0) return EPLACE_ERR_CUDA;
    slot.addr = p;
    slot.ctx_id = id;
  }
  *out = slot.addr;
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
  // The kernels read (x, y) and (w/2, h/2) as 8-byte pairs and write
  // doubles: a misaligned pointer would fault the caller's whole context.
  if (((uintptr_t)pos_xy | (uintptr_t)half_wh | (uintptr_t)density | (uintptr_t)overlap) & 7u)
    return EPLACE_ERR_INVALID;
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
  // The scratch keeps the previous call's contents.  A completed call
  // leaves the map at zero (the finalise re-zeroes every bin it reads) and
  // the counter back at zero; the clears below make a call correct also
  // after an earlier call whose kernels did not all run (a launch error part
  // way through), and set the scalar slot the finalise reads (iteration 0).
  if (cudaMemsetAsync(map, 0, (size_t)nb * sizeof(unsigned long long), s) != cudaSuccess ||
      cudaMemsetAsync(ticket, 0, 256, s) != cudaSuccess || cudaMemsetAsync(sc, 0, 256, s) != cudaSuccess)
    return EPLACE_ERR_CUDA;
  const int sx = width / bins_x, sy = height / bins_y;
  ScatterArgs a{reinterpret_cast<const float2 *>(pos_xy), reinterpret_cast<const float2 *>(half_wh), nullptr,
                nullptr, 0u, num_cells, bins_x, bins_y, sx, sy, map};
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
