// api.cu -- C ABI of libeplace.so: context set-up, the device-resident
// ElectroPlace loop (electro_place/mod.rs:65-204) and the stage entry points.
//
// Loop structure.  Every iteration runs on the device without host round
// trips: WA gradient -> density scatter -> density finalise -> 4 DCT GEMM
// launches -> fused gather/penalty/BB/FISTA step.  All loop scalars (penalty,
// step sizes, iteration counter) live on the device, so one legalisation
// interval (legalize_interval iterations) is captured once as a CUDA graph
// and replayed.  After each interval the solver positions are copied to
// pinned host memory; host threads legalise those snapshots (the greedy
// legaliser never feeds back into the positions, only into the choice of the
// best snapshot), while the device runs ahead.  The convergence test reads
// the overlap of the interval's last iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <exception>
#include <thread>
#include <vector>

#include "dct_tc.cuh"
#include "eplace_internal.h"
#include "fft.cuh"
#include "init_place.cuh"
#include "job.h"
#include "kernels.cuh"
#include "legal_par.cuh"

namespace eplace {
namespace {

thread_local std::string g_thread_error;
// Host<->device bytes copied by the library (eplace_result reports each
// call's share; calls running at the same time share the counters).
std::atomic<uint64_t> g_h2d{0}, g_d2h{0};

struct CudaError {
  cudaError_t e;
  std::string where;
};

#define CK(call)                                                           \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) throw CudaError{e_, std::string(#call)};        \
  } while (0)

// Device allocations of a context are stream-ordered (cudaMallocFromPoolAsync
// on the context's stream, from one memory pool per device that keeps what
// it has mapped).  A plain cudaMalloc / cudaFree is a device-wide implicit
// synchronisation point: while the job engine runs many contexts, one job's
// (re)load would otherwise stall every other job's stream.  The stream comes
// from the AllocOn guard of the calling thread; without one, plain
// cudaMalloc (context creation).
thread_local cudaStream_t t_alloc_stream = nullptr;
struct AllocOn {
  cudaStream_t prev;
  explicit AllocOn(cudaStream_t s) : prev(t_alloc_stream) { t_alloc_stream = s; }
  ~AllocOn() { t_alloc_stream = prev; }
};

cudaMemPool_t device_pool() {
  static std::mutex mu;
  static std::vector<cudaMemPool_t> pools;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t mp = nullptr;
    CK(cudaMemPoolCreate(&mp, &props));
    uint64_t keep = ~0ull;  // never trim: freed blocks serve the next loads
    CK(cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[dev] = mp;  // lives until the process exits
  }
  return pools[dev];
}

template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;    // elements in use
  size_t cap = 0;  // elements allocated
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { if (p) cudaFree(p); }
  void release() {
    if (!p) return;
    if (t_alloc_stream) cudaFreeAsync(p, t_alloc_stream);
    else cudaFree(p);
    p = nullptr;
  }
  void alloc(size_t count) {
    release();
    n = cap = 0;
    if (count) {
      if (t_alloc_stream)
        CK(cudaMallocFromPoolAsync((void **)&p, sizeof(T) * count, device_pool(), t_alloc_stream));
      else
        CK(cudaMalloc(&p, sizeof(T) * count));
    }
    n = cap = count;
  }
  // Room for count elements; reallocates only when the capacity is short.
  void ensure(size_t count) {
    if (p && count <= cap) {
      n = count;
      return;
    }
    alloc(count);
  }
  void upload(const T *h, size_t count, cudaStream_t s) {
    if (count) CK(cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    g_h2d += sizeof(T) * count;
  }
  void zero(cudaStream_t s) {
    if (n) CK(cudaMemsetAsync(p, 0, sizeof(T) * n, s));
  }
};

template <typename T>
struct PinBuf {
  T *p = nullptr;
  size_t n = 0;
  PinBuf() = default;
  PinBuf(const PinBuf &) = delete;
  PinBuf &operator=(const PinBuf &) = delete;
  ~PinBuf() { if (p) cudaFreeHost(p); }
  void alloc(size_t count) {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = count;
    if (count) CK(cudaMallocHost(&p, sizeof(T) * count));
  }
};

// Pinned host blocks for checkpoint snapshots, from power-of-two size
// classes carved out of 32 MiB chunks that are never returned: page-locked
// allocation and release are device-wide implicit synchronisation points,
// which the job engine must not hit while other jobs run.  Process-wide.
class PinArena {
 public:
  static PinArena &get() {
    static PinArena *a = new PinArena();  // never destroyed (pinned memory lives until exit)
    return *a;
  }
  // A block of at least `bytes`; *cls receives its class for put().
  void *take(size_t bytes, int *cls) {
    int k = kMinClass;
    while (((size_t)1 << k) < bytes) ++k;
    *cls = k;
    std::lock_guard<std::mutex> g(mu_);
    if (k > kMaxClass) {  // beyond the chunk size: a block of its own
      void *p = nullptr;
      CK(cudaMallocHost(&p, (size_t)1 << k));
      return p;
    }
    auto &fl = free_[k - kMinClass];
    if (fl.empty()) {
      char *chunk = nullptr;
      CK(cudaMallocHost((void **)&chunk, kChunk));
      for (size_t off = 0; off + ((size_t)1 << k) <= kChunk; off += (size_t)1 << k) fl.push_back(chunk + off);
    }
    void *p = fl.back();
    fl.pop_back();
    return p;
  }
  void put(void *p, int cls) {
    if (!p) return;
    std::lock_guard<std::mutex> g(mu_);
    if (cls > kMaxClass) {
      cudaFreeHost(p);
      return;
    }
    free_[cls - kMinClass].push_back(p);
  }

 private:
  static constexpr int kMinClass = 16, kMaxClass = 25;  // 64 KiB .. 32 MiB
  static constexpr size_t kChunk = (size_t)1 << kMaxClass;
  std::mutex mu_;
  std::vector<void *> free_[kMaxClass - kMinClass + 1];
};

// A pinned host block from the arena, grown on demand and kept by its owner.
struct PinBlock {
  void *p = nullptr;
  size_t bytes = 0;
  int cls = 0;
  PinBlock() = default;
  PinBlock(const PinBlock &) = delete;
  PinBlock &operator=(const PinBlock &) = delete;
  ~PinBlock() { PinArena::get().put(p, cls); }
  void reserve(size_t need) {
    if (p && need <= bytes) return;
    PinArena::get().put(p, cls);
    p = PinArena::get().take(std::max<size_t>(need, 1), &cls);
    bytes = (size_t)1 << cls;
  }
};

// A checkpoint's positions in pinned memory (the interval's device-to-host
// copy lands here) and the host legaliser's binding of them.  Kept by the
// context and reused across checkpoints and runs.
struct HostSnap {
  float2 *pos = nullptr;
  size_t cap = 0;  // positions
  int cls = 0;     // PinArena class of pos
  std::vector<int32_t> sx, sy;
  HostSnap() = default;
  HostSnap(const HostSnap &) = delete;
  HostSnap &operator=(const HostSnap &) = delete;
  ~HostSnap() { PinArena::get().put(pos, cls); }
  void reserve(size_t n) {
    if (n <= cap && pos) return;
    PinArena::get().put(pos, cls);
    pos = nullptr;
    pos = (float2 *)PinArena::get().take(sizeof(float2) * std::max<size_t>(n, 1), &cls);
    cap = ((size_t)1 << cls) / sizeof(float2);
  }
};

// What one device legalisation reports back (24 bytes, one copy).
struct LegalOut {
  unsigned long long hpwl;  // HPWL accumulator (k_hpwl)
  double disp;
  int32_t status;           // 0 ok, 1 no free site
  int32_t pad_;
};

// Device resources of one legalisation in flight: its own copy of the
// positions, the binding, the cost of each placement and its stream.
struct LegalSlot {
  DBuf<float2> pos;
  DBuf<int2> sites;
  DBuf<int2> loc;       // [N + F]: pin locations, fixed cells at the end
  DBuf<double> cost;
  DBuf<LegalOut> out;
  PinBuf<LegalOut> hout;
  // round buffers of the parallel legaliser (legal_par.cu)
  DBuf<uint64_t> fm;
  DBuf<int32_t> list, len, info, hmark, dmark, pick;
  DBuf<uint8_t> dist, fresh;
  DBuf<LpState> lst;
  LpGraph graph;        // the whole legalisation: rounds in a device-side loop
  uint64_t gen = ~0ull;  // problem load this slot is prepared for
  cudaStream_t stream = nullptr;
  cudaEvent_t snap = nullptr, start = nullptr, done = nullptr;
  LegalSlot() = default;
  LegalSlot(const LegalSlot &) = delete;
  LegalSlot &operator=(const LegalSlot &) = delete;
  ~LegalSlot() {
    if (snap) cudaEventDestroy(snap);
    if (start) cudaEventDestroy(start);
    if (done) cudaEventDestroy(done);
    if (stream) cudaStreamDestroy(stream);
  }
};

}  // namespace
}  // namespace eplace

using namespace eplace;

struct eplace_ctx {
  HostProblem hp;
  int device = 0;
  cudaStream_t stream = nullptr;
  // Second stream of the iteration: the WA kernel runs on it beside the
  // density -> transform chain (fork / join events, captured into the graph).
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string err;
  int num_sms = 0;
  int64_t spin_cycles = 0;  // bound of the step's barrier waits for the current run (0: kernel default)
  int step_grid = 0;
  std::vector<double> pw_host;
  double total_area = 0.0;

  // problem on device
  DBuf<uint32_t> net_off, pin_cell;
  DBuf<uint8_t> has_driver;
  DBuf<uint32_t> wa_off, wa_pins;  // CSR copy, nets ordered by pin count
  DBuf<uint32_t> wa_slots;         // padded pin table of the degree classes (kWaSlots)
  DBuf<float2> half;
  DBuf<float> area, pw;
  DBuf<uint8_t> mflag;      // [N] 1 for a macro
  DBuf<uint32_t> mac_idx;   // the macros' cell ids
  // The WA pin table is built in pinned memory and uploaded asynchronously;
  // wa_pin_ev marks the end of the last upload from it.
  PinBlock wa_pin;
  cudaEvent_t wa_pin_ev = nullptr;
  uint32_t n_mac = 0;
  // state
  DBuf<float2> look;  // [N + F]
  DBuf<float2> x, xp, g, gprev, tmp_wl, tmp_den;
  DBuf<unsigned long long> acc, dens;
  DBuf<float> rho, T, Exh, Eyh, U, V, Ex, Ey, phi;
  DBuf<float> mB1, mL2, mB3, mL4, mB5, mL6;  // DCT matrices (row-major operands)
  DBuf<float> mB3g, mL6g;                   // potential-gradient field (extension)
  DBuf<float> wx, gx2, wy, gy2;
  DBuf<GemmOp> ops;                         // 0: GEMM1, 1: GEMM2, 2-3: GEMM3, 4-5: GEMM4
  // Folded FP32 transform (grids with bins_x, bins_y multiples of 8): the
  // half matrices (even / odd frequencies of the first or second half of
  // the spatial index), the E / O products of GEMMs 3 and 4, their op
  // tables (12 per field mode) and butterflies (2 + 2 per field mode).
  bool fold = false;
  // FFT form of the transforms (EPLACE_DCT_FP32_FFT on a power-of-two grid):
  // set by every entry that launches the transform; twiddles of length W / H.
  bool fft = false;
  DBuf<float2> fft_twx, fft_tqx, fft_twy, fft_tqy;
  DBuf<float> hB1e, hB1o, hL2e, hL2o, hB3e, hB3o, hB5e, hB5o, hB3ge, hB3go, hL4e, hL4o, hL6e, hL6o, hL6ge, hL6go;
  DBuf<float> f3, f4;
  DBuf<GemmOp> hops;
  DBuf<FlyOp> fops;
  DBuf<double> mom, part, part2, part_b;
  DBuf<DevScalars> sc;
  DBuf<IterLog> log;
  DBuf<unsigned> bar;  // [0..1] grid barrier, [2] finalise ticket, [3] step ticket
  DBuf<int2> loc;
  DBuf<unsigned long long> hp_total;
  size_t log_cap = 0;
  // Bumped whenever a buffer a captured graph points at is reallocated.
  uint64_t buf_epoch = 1;

  // Host resources kept across runs: legaliser base map and per-thread
  // legalisers, the worker pool, pinned snapshot slots and their events, and
  // the CUDA graph of one legalisation interval.
  std::unique_ptr<LegalBase> lbase;
  std::vector<std::unique_ptr<Legalizer>> legal;
  std::unique_ptr<Pool> pool;
  std::vector<std::unique_ptr<HostSnap>> hsnaps;  // all of them
  std::vector<HostSnap *> hsnap_free;             // not held by a run
  std::vector<std::unique_ptr<PinBuf<IterLog>>> logs;
  std::vector<std::unique_ptr<PinBuf<DevScalars>>> scs;
  std::vector<cudaEvent_t> slot_ev;
  size_t slot_log_cap = 0;
  // Device copies of an interval's positions and scalars, one per slot: the
  // loop's stream writes them (device to device, microseconds) and the copy
  // stream moves them to the host while the next interval computes.
  cudaStream_t copy = nullptr;
  std::vector<std::unique_ptr<DBuf<float2>>> snap_pos;
  std::vector<std::unique_ptr<DBuf<DevScalars>>> snap_sc;
  std::vector<cudaEvent_t> snap_ev;
  cudaGraphExec_t gexec = nullptr;
  bool g_valid = false;  // gexec matches the current buffers and settings
  uint64_t g_epoch = 0, g_interval = 0;
  int g_field = -1;
  int g_bx = -1, g_by = -1;  // bin grid gexec was instantiated for
  bool g_tc = false;
  bool g_fft = false;
  float g_gamma = 0.f;

  // Tensor-core (BF16x3) transform: operands as hi/lo BF16 planes, all
  // K-major; *t = transposed (the next GEMM's B^T).
  bool tc_ready = false;
  DBuf<__nv_bfloat16> rho_h, rho_l, Tt_h, Tt_l, Exh_h, Exh_l, Eyh_h, Eyh_l, Ut_h, Ut_l, Vt_h, Vt_l;
  DBuf<__nv_bfloat16> B1t_h, B1t_l, L2_h, L2_l, B3t_h, B3t_l, B5t_h, B5t_l, L4_h, L4_l, L6_h, L6_l;
  DBuf<__nv_bfloat16> B3gt_h, B3gt_l, L6g_h, L6g_l;
  TcGemmMaps tm1{}, tm2{}, tm3[2]{}, tm4[2]{};

  // Device legaliser: cell order, macro footprints and the base free map
  // (from lbase), and the slots of legalisations in flight.
  bool lg_ready = false;
  DBuf<uint32_t> lg_order;
  DBuf<uchar2> lg_fsize;     // [N] footprint per cell (only when some cell is a macro)
  DBuf<uint64_t> lg_free0;
  bool lg_macros = false;
  std::vector<std::unique_ptr<LegalSlot>> lslots;
  int step_grid_full = 0;
  // Step as three ordinary launches instead of one cooperative launch: used
  // whenever other long-running kernels share the device (device legaliser,
  // several jobs at once), where a grid barrier could wait on blocks that
  // cannot become resident.
  bool split_step = false;
  bool shared_device = false;  // set by the job engine: other jobs' kernels run beside this one
  int mat_bx = -1, mat_by = -1;  // bin grid the DCT matrices were built for
  uint64_t load_gen = 0;         // bumped by every (re)load of a problem
  // Launch shapes picked by autotune_launches (none of them changes a bit
  // of any result): grid caps of the WA and scatter kernels in blocks per
  // SM, and the SIMT GEMM tile of each of the four transform GEMMs.
  int wa_blocks_per_sm = 16, sc_blocks_per_sm = 16;
  // Device initial placement (init_place.cu): scratch of the shuffle, the
  // taken sites, the handed-out BELs, and the jump maps (uploaded once).
  DBuf<uint32_t> ip_j, ip_cnt, ip_start, ip_entries, ip_block, ip_occ;
  DBuf<uint64_t> ip_jump;
  DBuf<int2> ip_site;
  std::vector<uint32_t> ip_occ_host;  // sorted taken sites of the pending device placement
  uint64_t ip_n = 0;                  // free logic BELs of the pending device placement
  int gemm_tile[4] = {0, 0, 0, 0};
  WaClass wa_cls[kWaClasses] = {};  // degree classes of the sorted CSR
  int wa_warps = 0;
  int grad_k = 24;  // fixed-point scale 2^k of the packed WA gradient (pack_grad)

  // Device memory this context holds (allocated capacities).
  uint64_t device_bytes() const;

  ~eplace_ctx() {
    if (stream) cudaStreamSynchronize(stream);
    if (copy) cudaStreamSynchronize(copy);
    for (auto &l : lslots)
      if (l && l->stream) cudaStreamSynchronize(l->stream);
    lslots.clear();
    pool.reset();
    if (gexec) cudaGraphExecDestroy(gexec);
    for (auto e : slot_ev) cudaEventDestroy(e);
    for (auto e : snap_ev) cudaEventDestroy(e);
    if (copy) cudaStreamDestroy(copy);
    if (side) cudaStreamSynchronize(side);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (wa_pin_ev) cudaEventDestroy(wa_pin_ev);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

void set_err(eplace_ctx *c, const std::string &m) {
  if (c) c->err = m;
  g_thread_error = m;
}

eplace_status cuda_fail(eplace_ctx *c, const CudaError &e) {
  set_err(c, e.where + ": " + cudaGetErrorString(e.e));
  if (e.e == cudaErrorMemoryAllocation) return EPLACE_ERR_OOM;
  if (e.e == cudaErrorNoDevice || e.e == cudaErrorInsufficientDriver) return EPLACE_ERR_NO_DEVICE;
  return EPLACE_ERR_CUDA;
}

// The WA kernel sees the nets ordered by pin count (stable), so nets of one
// degree class are contiguous: order[i] is the i-th net of that order and
// off[] its offsets (a CSR over the sorted nets).  Net order does not
// change the result: the gradient accumulates in fixed point.
void degree_order(const HostProblem &hp, std::vector<uint32_t> &order, std::vector<uint32_t> &off) {
  // Counting sort by degree (stable: nets of one degree keep their order).
  std::vector<uint32_t> start((size_t)hp.max_degree + 2, 0);
  for (uint32_t n = 0; n < hp.NN; ++n) ++start[hp.net_off[n + 1] - hp.net_off[n] + 1];
  for (size_t d = 1; d < start.size(); ++d) start[d] += start[d - 1];
  order.resize(hp.NN);
  for (uint32_t n = 0; n < hp.NN; ++n) order[start[hp.net_off[n + 1] - hp.net_off[n]]++] = n;
  off.resize((size_t)hp.NN + 1);
  off[0] = 0;
  for (uint32_t i = 0; i < hp.NN; ++i) off[i + 1] = off[i] + (hp.net_off[order[i] + 1] - hp.net_off[order[i]]);
}

// The pins of sorted nets [n0, n1), in sorted-CSR order starting at off[n0]
// (the device reads the sorted CSR only for the last class: nets of more
// than 224 pins).
void sorted_pins(const HostProblem &hp, const std::vector<uint32_t> &order, const std::vector<uint32_t> &off,
                 uint32_t n0, uint32_t n1, std::vector<uint32_t> &pins) {
  pins.resize(off[n1] - off[n0]);
  for (uint32_t i = n0; i < n1; ++i) {
    const uint32_t n = order[i];
    std::copy(hp.pin_cell.begin() + hp.net_off[n], hp.pin_cell.begin() + hp.net_off[n + 1],
              pins.begin() + (off[i] - off[n0]));
  }
}

// The padded pin table of the degree classes: net idx of class j takes
// G * S slots (G = kWaGroup[j], S = kWaSlots[j]) from the class base (a
// multiple of 4 slots, for 16-byte loads); pin q of the net goes to lane
// q % G, slot q / G of that lane, unused slots 0xffffffff.  Sets each
// class's slot_base, writes the table to t (cap slots) and returns its
// length.  A class pads a net of d pins to fewer than 2d slots (2 for 2,
// 4 for 3..4, 8 for 5..8, ..., 256 for 129..224), so 2P + 64 slots always
// suffice.  Three threads fill disjoint runs of classes of about equal size.
size_t build_wa_slots(const HostProblem &hp, const std::vector<uint32_t> &order, WaClass (&cls)[kWaClasses],
                      uint32_t *t, size_t cap) {
  size_t total = 0;
  size_t upto[kWaClasses + 1] = {0};
  for (int j = 0; j < kWaClasses; ++j) {
    total = (total + 3) & ~(size_t)3;
    cls[j].slot_base = (long long)total;
    total += (size_t)cls[j].nets * kWaGroup[j] * kWaSlots[j];
    upto[j + 1] = total;
  }
  const size_t len = std::max<size_t>(total, 4);
  if (len > cap) throw CudaError{cudaErrorInvalidValue, "build_wa_slots: table larger than its bound"};
  auto fill = [&](int j0, int j1) {
    for (int j = j0; j < j1; ++j) {
      const int G = kWaGroup[j], S = kWaSlots[j];
      const size_t b0 = (size_t)cls[j].slot_base;
      std::fill(t + b0, t + upto[j + 1], 0xffffffffu);
      if (S == 0) continue;
      const int gs = __builtin_ctz(G);  // G is a power of two
      for (int idx = 0; idx < cls[j].nets; ++idx) {
        const uint32_t n = order[(uint32_t)(cls[j].first_net + idx)];
        const size_t base = b0 + (size_t)idx * G * S;
        const uint32_t b = hp.net_off[n], d = hp.net_off[n + 1] - b;
        for (uint32_t r = 0; r < d; ++r) t[base + (size_t)(r & (G - 1)) * S + (r >> gs)] = hp.pin_cell[b + r];
      }
    }
  };
  int cut[4] = {0, 0, 0, kWaClasses};
  for (int k = 1; k < 3; ++k) {
    cut[k] = cut[k - 1];
    while (cut[k] < kWaClasses && upto[cut[k]] * 3 < total * k) ++cut[k];
  }
  std::thread t1([&] { fill(cut[1], cut[2]); });
  std::thread t2([&] { fill(cut[2], cut[3]); });
  fill(cut[0], cut[1]);
  t1.join();
  t2.join();
  // the alignment gaps between classes and the tail of a short table
  for (int j = 0; j + 1 < kWaClasses; ++j) std::fill(t + upto[j + 1], t + (size_t)cls[j + 1].slot_base, 0xffffffffu);
  std::fill(t + total, t + len, 0xffffffffu);
  return len;
}

// Fixed-point exponent k of the packed WA gradient: every cell's x and y
// sums must stay below 2^31 in magnitude.  With at most D pins on one cell
// and a bound of 4 per pin, 4 D 2^k < 2^31; k is at most 24.
int grad_scale_log2(const HostProblem &hp) {
  std::vector<uint32_t> pins(hp.N, 0);
  uint32_t d = 1;
  for (uint32_t q = 0; q < hp.P; ++q)
    if (hp.pin_cell[q] < hp.N) d = std::max(d, ++pins[hp.pin_cell[q]]);
  int k = 24;
  while (k > 0 && 4.0 * (double)d * std::ldexp(1.0, k) >= 2147483648.0) --k;
  return k;
}

// Splits the degree-sorted nets into the WA kernel's degree classes and
// numbers the warps (32 / group width nets per warp).  Returns the warps.
int build_wa_classes(const std::vector<uint32_t> &off, WaClass (&cls)[kWaClasses]) {
  const uint32_t NN = (uint32_t)off.size() - 1;
  uint32_t n = 0;
  while (n < NN && off[n + 1] - off[n] < 2) ++n;  // no gradient below two pins
  int warps = 0;
  for (int j = 0; j < kWaClasses; ++j) {
    const uint32_t first = n;
    while (n < NN && off[n + 1] - off[n] <= (uint32_t)kWaDegHi[j]) ++n;
    const int per_warp = 32 / kWaGroup[j];
    cls[j] = WaClass{(int)first, (int)(n - first), warps, 0};
    warps += (int)((n - first + per_warp - 1) / per_warp);
  }
  return warps;
}

// Host copies of the FP32 DCT matrices of one bin grid (rustdct conventions,
// density.rs:211-275).  They depend on the bin grid only, so each is computed
// once per process and kept; uploading a kept set costs only the copy.
struct HostMats {
  std::vector<float> B1, B3, B5, L2, L4, L6, B3g, L6g, wx, gx2, wy, gy2;
  // folded halves (bins_x, bins_y multiples of 8), see fold_matrices
  std::vector<float> B1e, B1o, L2e, L2o, B3e, B3o, B5e, B5o, B3ge, B3go, L4e, L4o, L6e, L6o, L6ge, L6go;
};

// The transform's matrices fold about the middle of their spatial index:
// with theta = pi k (n + 1/2) / N, theta(N - 1 - n) = pi k - theta(n), so
// cos and sin of theta (and of the DST-III's pi (k + 1)(n + 1/2) / N) at
// n and N - 1 - n agree up to the sign s (-1)^k, s = +1 except for the
// potential-gradient field's -sin(theta), where s = -1.  A product over the
// spatial index then splits into the even-k half applied to x(n) + x(N-1-n)
// and the odd-k half applied to x(n) - x(N-1-n), each (N/2) x (N/2); a
// product over k gives E = sum over even k and O = sum over odd k, and the
// outputs n, N - 1 - n are E + O and s (E - O).  Half the multiply-adds.
// Halves kept here (row-major):
//   B1e/o  [x < W/2][m]   = B1[x][2m(+1)]      L2e/o [m][y < H/2]  = L2[2m(+1)][y]
//   B3e/o, B5e/o, B3ge/o  [m][x < W/2] = B[2m(+1)][x]
//   L4e/o, L6e/o, L6ge/o  [y < H/2][m] = L[y][2m(+1)]
void fold_matrices(int W, int H, HostMats &m) {
  const int hw = W / 2, hh = H / 2;
  auto cols = [](const std::vector<float> &M, int n, int rows, int par, std::vector<float> &out) {
    out.resize((size_t)rows * (n / 2));
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < n / 2; ++c) out[(size_t)r * (n / 2) + c] = M[(size_t)r * n + 2 * c + par];
  };  // rows 0..rows-1, every other column from par
  auto rowsel = [](const std::vector<float> &M, int n, int cols, int par, std::vector<float> &out) {
    out.resize((size_t)(n / 2) * cols);
    for (int r = 0; r < n / 2; ++r)
      for (int c = 0; c < cols; ++c) out[(size_t)r * cols + c] = M[(size_t)(2 * r + par) * n + c];
  };  // every other row from par, columns 0..cols-1
  cols(m.B1, W, hw, 0, m.B1e);
  cols(m.B1, W, hw, 1, m.B1o);
  rowsel(m.L2, H, hh, 0, m.L2e);
  rowsel(m.L2, H, hh, 1, m.L2o);
  rowsel(m.B3, W, hw, 0, m.B3e);
  rowsel(m.B3, W, hw, 1, m.B3o);
  rowsel(m.B5, W, hw, 0, m.B5e);
  rowsel(m.B5, W, hw, 1, m.B5o);
  rowsel(m.B3g, W, hw, 0, m.B3ge);
  rowsel(m.B3g, W, hw, 1, m.B3go);
  cols(m.L4, H, hh, 0, m.L4e);
  cols(m.L4, H, hh, 1, m.L4o);
  cols(m.L6, H, hh, 0, m.L6e);
  cols(m.L6, H, hh, 1, m.L6o);
  cols(m.L6g, H, hh, 0, m.L6ge);
  cols(m.L6g, H, hh, 1, m.L6go);
}

bool fold_ok(int W, int H) { return W % 8 == 0 && H % 8 == 0 && W >= 16 && H >= 16; }

void compute_host_mats(int W, int H, HostMats &m) {
  const double pi = 3.14159265358979323846;
  auto &B1 = m.B1, &B3 = m.B3, &B5 = m.B5, &L2 = m.L2, &L4 = m.L4, &L6 = m.L6, &B3g = m.B3g, &L6g = m.L6g;
  for (auto *v : {&B1, &B3, &B5, &B3g}) v->assign((size_t)W * W, 0.f);
  for (auto *v : {&L2, &L4, &L6, &L6g}) v->assign((size_t)H * H, 0.f);
  // GEMM1  T = rho * B1,     B1[x][kx] = cos(pi kx (x + 1/2) / W)        (row DCT-II)
  // GEMM3a U = Ex^ * B3,     B3[kx][x] = sin(pi (kx+1)(x + 1/2) / W), kx = W-1 halved (row DST-III)
  // GEMM3b V = Ey^ * B5,     B5[kx][x] = cos(pi kx (x + 1/2) / W),    kx = 0 halved   (row DCT-III)
  for (int a = 0; a < W; ++a)
    for (int b = 0; b < W; ++b) {
      B1[(size_t)a * W + b] = (float)std::cos(pi * b * (a + 0.5) / W);
      B3[(size_t)a * W + b] = (float)(std::sin(pi * (a + 1) * (b + 0.5) / W) * (a == W - 1 ? 0.5 : 1.0));
      B5[(size_t)a * W + b] = (float)(std::cos(pi * a * (b + 0.5) / W) * (a == 0 ? 0.5 : 1.0));
      // potential-gradient field: B3g[kx][x] = -sin(pi kx (x + 1/2) / W)
      B3g[(size_t)a * W + b] = (float)(-std::sin(pi * a * (b + 0.5) / W));
    }
  // GEMM2  A  = L2 * T,      L2[ky][y] = cos(pi ky (y + 1/2) / H)        (column DCT-II)
  // GEMM4a Ex = L4 * U,      L4[y][ky] = cos(pi ky (y + 1/2) / H), ky = 0 halved   (column DCT-III)
  // GEMM4b Ey = L6 * V,      L6[y][ky] = sin(pi (ky+1)(y + 1/2) / H), ky = H-1 halved (column DST-III)
  for (int a = 0; a < H; ++a)
    for (int b = 0; b < H; ++b) {
      L2[(size_t)a * H + b] = (float)std::cos(pi * a * (b + 0.5) / H);
      L4[(size_t)a * H + b] = (float)(std::cos(pi * b * (a + 0.5) / H) * (b == 0 ? 0.5 : 1.0));
      L6[(size_t)a * H + b] = (float)(std::sin(pi * (b + 1) * (a + 0.5) / H) * (b == H - 1 ? 0.5 : 1.0));
      // potential-gradient field: L6g[y][ky] = -sin(pi ky (y + 1/2) / H)
      L6g[(size_t)a * H + b] = (float)(-std::sin(pi * b * (a + 0.5) / H));
    }
  auto &wx = m.wx, &gx2 = m.gx2, &wy = m.wy, &gy2 = m.gy2;
  wx.assign(W, 0.f);
  gx2.assign(W, 0.f);
  wy.assign(H, 0.f);
  gy2.assign(H, 0.f);
  for (int k = 0; k < W; ++k) {
    double w = pi * k / W;
    wx[k] = (float)w;
    gx2[k] = (float)(2.0 * (1.0 - std::cos(w)));
  }
  for (int k = 0; k < H; ++k) {
    double w = pi * k / H;
    wy[k] = (float)w;
    gy2[k] = (float)(2.0 * (1.0 - std::cos(w)));
  }
}

const HostMats &host_mats(int W, int H) {
  static std::mutex mu;
  static auto *cache = new std::map<std::pair<int, int>, std::unique_ptr<HostMats>>();  // kept for the process
  std::lock_guard<std::mutex> g(mu);
  auto &slot = (*cache)[{W, H}];
  if (!slot) {
    slot.reset(new HostMats());
    compute_host_mats(W, H, *slot);
    if (fold_ok(W, H)) fold_matrices(W, H, *slot);
  }
  return *slot;
}

// DCT matrices as GEMM operands, uploaded from the kept host copies.
void build_matrices(eplace_ctx *c) {
  AllocOn on_stream(c->stream);
  const int W = c->hp.BX, H = c->hp.BY;
  const HostMats &hm = host_mats(W, H);
  const auto &B1 = hm.B1, &B3 = hm.B3, &B5 = hm.B5, &L2 = hm.L2, &L4 = hm.L4, &L6 = hm.L6, &B3g = hm.B3g,
             &L6g = hm.L6g, &wx = hm.wx, &gx2 = hm.gx2, &wy = hm.wy, &gy2 = hm.gy2;
  cudaStream_t s = c->stream;
  c->mB1.ensure(B1.size()); c->mB1.upload(B1.data(), B1.size(), s);
  c->mB3.ensure(B3.size()); c->mB3.upload(B3.data(), B3.size(), s);
  c->mB5.ensure(B5.size()); c->mB5.upload(B5.data(), B5.size(), s);
  c->mL2.ensure(L2.size()); c->mL2.upload(L2.data(), L2.size(), s);
  c->mL4.ensure(L4.size()); c->mL4.upload(L4.data(), L4.size(), s);
  c->mL6.ensure(L6.size()); c->mL6.upload(L6.data(), L6.size(), s);
  c->mB3g.ensure(B3g.size()); c->mB3g.upload(B3g.data(), B3g.size(), s);
  c->mL6g.ensure(L6g.size()); c->mL6g.upload(L6g.data(), L6g.size(), s);
  c->wx.ensure(W); c->wx.upload(wx.data(), W, s);
  c->gx2.ensure(W); c->gx2.upload(gx2.data(), W, s);
  c->wy.ensure(H); c->wy.upload(wy.data(), H, s);
  c->gy2.ensure(H); c->gy2.upload(gy2.data(), H, s);
  // ops[0..5]: reference field; ops[6..11]: potential-gradient field.
  GemmOp ops[12] = {
      {c->rho.p, c->mB1.p, c->T.p, nullptr},
      {c->mL2.p, c->T.p, c->Exh.p, c->Eyh.p},
      {c->Exh.p, c->mB3.p, c->U.p, nullptr},
      {c->Eyh.p, c->mB5.p, c->V.p, nullptr},
      {c->mL4.p, c->U.p, c->Ex.p, nullptr},
      {c->mL6.p, c->V.p, c->Ey.p, nullptr},
      {c->rho.p, c->mB1.p, c->T.p, nullptr},
      {c->mL2.p, c->T.p, c->Exh.p, c->Eyh.p},
      {c->Exh.p, c->mB3g.p, c->U.p, nullptr},
      {c->Eyh.p, c->mB5.p, c->V.p, nullptr},
      {c->mL4.p, c->U.p, c->Ex.p, nullptr},
      {c->mL6g.p, c->V.p, c->Ey.p, nullptr},
  };
  for (auto &o : ops) {  // plain row-major operands, nothing folded
    o.a_mir = o.a_full = o.b_mir = o.b_full = o.col_split = 0;
    o.row_par = -1;
  }
  // leading dimensions: A is M x K, B is K x N, C is M x N
  const int ld[6][3] = {{W, W, W}, {H, W, W}, {W, W, W}, {W, W, W}, {H, W, W}, {H, W, W}};
  for (int k = 0; k < 12; ++k) {
    ops[k].lda = ld[k % 6][0];
    ops[k].ldb = ld[k % 6][1];
    ops[k].ldc = ld[k % 6][2];
  }
  c->ops.ensure(12);
  c->ops.upload(ops, 12, s);
  if (fft_supported(W, H)) {
    std::vector<float2> tw(W / 2), tq(W), uw(H / 2), uq(H);
    fft_tables_host(W, tw.data(), tq.data());
    fft_tables_host(H, uw.data(), uq.data());
    c->fft_twx.ensure(tw.size()); c->fft_twx.upload(tw.data(), tw.size(), s);
    c->fft_tqx.ensure(tq.size()); c->fft_tqx.upload(tq.data(), tq.size(), s);
    c->fft_twy.ensure(uw.size()); c->fft_twy.upload(uw.data(), uw.size(), s);
    c->fft_tqy.ensure(uq.size()); c->fft_tqy.upload(uq.data(), uq.size(), s);
  }
  c->fold = fold_ok(W, H);
  if (c->fold) {
    const int hw = W / 2, hh = H / 2;
    const size_t q = (size_t)H * hw;  // one E or O of GEMM 3 ([H][W/2]); GEMM 4's are [H/2][W], the same size
    DBuf<float> *hb[16] = {&c->hB1e, &c->hB1o, &c->hL2e, &c->hL2o, &c->hB3e, &c->hB3o, &c->hB5e, &c->hB5o,
                           &c->hB3ge, &c->hB3go, &c->hL4e, &c->hL4o, &c->hL6e, &c->hL6o, &c->hL6ge, &c->hL6go};
    const std::vector<float> *hv[16] = {&hm.B1e, &hm.B1o, &hm.L2e, &hm.L2o, &hm.B3e, &hm.B3o, &hm.B5e, &hm.B5o,
                                        &hm.B3ge, &hm.B3go, &hm.L4e, &hm.L4o, &hm.L6e, &hm.L6o, &hm.L6ge, &hm.L6go};
    for (int k = 0; k < 16; ++k) {
      hb[k]->ensure(hv[k]->size());
      hb[k]->upload(hv[k]->data(), hv[k]->size(), s);
    }
    c->f3.ensure(4 * q);
    c->f4.ensure(4 * q);
    float *f3 = c->f3.p, *f4 = c->f4.p;
    auto op = [](const float *A, int lda, const float *B, int ldb, float *C, float *C2, int ldc) {
      GemmOp o{A, B, C, C2, lda, ldb, ldc, 0, 0, 0, 0, -1, 0};
      return o;
    };
    GemmOp h[24];
    for (int fm = 0; fm < 2; ++fm) {
      GemmOp *g = h + 12 * fm;
      // GEMM 1: T = rho B1, columns of rho folded; T's columns even kx first
      g[0] = op(c->rho.p, W, c->hB1e.p, hw, c->T.p, nullptr, W);
      g[0].a_mir = 1;
      g[0].a_full = W;
      g[1] = op(c->rho.p, W, c->hB1o.p, hw, c->T.p + hw, nullptr, W);
      g[1].a_mir = -1;
      g[1].a_full = W;
      // GEMM 2: L2 T + spectral epilogue, rows of T folded; Ex^, Ey^ rows even ky first
      g[2] = op(c->hL2e.p, hh, c->T.p, W, c->Exh.p, c->Eyh.p, W);
      g[2].b_mir = 1;
      g[2].b_full = H;
      g[2].row_par = 0;
      g[2].col_split = 1;
      g[3] = op(c->hL2o.p, hh, c->T.p, W, c->Exh.p + (size_t)hh * W, c->Eyh.p + (size_t)hh * W, W);
      g[3].b_mir = -1;
      g[3].b_full = H;
      g[3].row_par = 1;
      g[3].col_split = 1;
      // GEMM 3: E / O of U = Ex^ B3 (B3g) and V = Ey^ B5
      g[4] = op(c->Exh.p, W, fm ? c->hB3ge.p : c->hB3e.p, hw, f3, nullptr, hw);
      g[5] = op(c->Exh.p + hw, W, fm ? c->hB3go.p : c->hB3o.p, hw, f3 + q, nullptr, hw);
      g[6] = op(c->Eyh.p, W, c->hB5e.p, hw, f3 + 2 * q, nullptr, hw);
      g[7] = op(c->Eyh.p + hw, W, c->hB5o.p, hw, f3 + 3 * q, nullptr, hw);
      // GEMM 4: E / O of Ex = L4 U and Ey = L6 (L6g) V (U, V rows even ky first)
      g[8] = op(c->hL4e.p, hh, c->U.p, W, f4, nullptr, W);
      g[9] = op(c->hL4o.p, hh, c->U.p + (size_t)hh * W, W, f4 + q, nullptr, W);
      g[10] = op(fm ? c->hL6ge.p : c->hL6e.p, hh, c->V.p, W, f4 + 2 * q, nullptr, W);
      g[11] = op(fm ? c->hL6go.p : c->hL6o.p, hh, c->V.p + (size_t)hh * W, W, f4 + 3 * q, nullptr, W);
    }
    c->hops.ensure(24);
    c->hops.upload(h, 24, s);
    FlyOp fl[8];
    for (int fm = 0; fm < 2; ++fm) {
      FlyOp *f = fl + 4 * fm;
      f[0] = FlyOp{f3, f3 + q, c->U.p, fm ? -1.0f : 1.0f};
      f[1] = FlyOp{f3 + 2 * q, f3 + 3 * q, c->V.p, 1.0f};
      f[2] = FlyOp{f4, f4 + q, c->Ex.p, 1.0f};
      f[3] = FlyOp{f4 + 2 * q, f4 + 3 * q, c->Ey.p, fm ? -1.0f : 1.0f};
    }
    c->fops.ensure(8);
    c->fops.upload(fl, 8, s);
  }
  CK(cudaStreamSynchronize(s));
}

void ensure_log(eplace_ctx *c, size_t iters) {
  AllocOn on_stream(c->stream);
  if (c->log_cap >= iters + 2) return;
  c->log_cap = std::max<size_t>(iters + 2, 1024);
  c->log.alloc(c->log_cap);
  c->log.zero(c->stream);
  ++c->buf_epoch;
}

int grid_for(int n, int block, int cap) {
  long long g = ((long long)n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// --- kernel sequence of one iteration ------------------------------------
void launch_wa_stage(eplace_ctx *c, float gamma, cudaStream_t st = nullptr) {
  WaArgs a{};
  std::copy(c->wa_cls, c->wa_cls + kWaClasses, a.cls);
  a.nwarps = c->wa_warps;
  a.slots = c->wa_slots.p;
  a.net_off = c->wa_off.p;
  a.pin_cell = c->wa_pins.p;
  a.pos = c->look.p;
  a.acc = c->acc.p;
  a.N = c->hp.N;
  a.gamma = gamma;
  a.grad_scale = (float)std::ldexp(1.0, c->grad_k);
  CK(launch_wa(a, grid_for(c->wa_warps * 32, kWaBlock, c->num_sms * c->wa_blocks_per_sm), st ? st : c->stream));
}

void launch_scatter_stage(eplace_ctx *c) {
  const HostProblem &hp = c->hp;
  ScatterArgs a{c->look.p, hp.any_macro ? c->half.p : nullptr, hp.any_macro ? c->mflag.p : nullptr,
                hp.any_macro ? c->mac_idx.p : nullptr, hp.any_macro ? c->n_mac : 0u, hp.N, hp.BX, hp.BY,
                hp.sx, hp.sy, c->dens.p};
  CK(launch_scatter(a, grid_for((int)hp.N, kScatterBlock, c->num_sms * c->sc_blocks_per_sm), c->stream));
}

// --- tensor-core transform set-up ------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess) throw CudaError{cudaErrorNotSupported, "cuTensorMapEncodeTiled"};
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2-D map of a row-major BF16 matrix (rows x k), box 64 (k) x box_rows,
// 128-byte swizzle: the K-major operand layout of k_tc_gemm.
CUtensorMap make_map(const __nv_bfloat16 *base, int rows, int k, int box_rows) {
  CUtensorMap m;
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)k * 2};
  cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(base), dims, strides,
                           box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError{cudaErrorInvalidValue, "cuTensorMapEncodeTiled"};
  return m;
}

bool tc_supported(const HostProblem &hp) { return hp.BY % 128 == 0 && hp.BX % kTcBN == 0 && hp.BX % 64 == 0; }

// Host copies of the tensor-core operands (BF16 hi/lo planes of the eight
// transposed DCT matrices) of one bin grid, computed once per process.
struct HostTcMats {
  std::vector<__nv_bfloat16> hi[8], lo[8];  // B1t, B3t, B5t, B3gt, L2, L4, L6, L6g
};

void split_planes(const std::vector<double> &v, std::vector<__nv_bfloat16> &h, std::vector<__nv_bfloat16> &l) {
  h.resize(v.size());
  l.resize(v.size());
  for (size_t i = 0; i < v.size(); ++i) {
    const float f = (float)v[i];
    h[i] = __float2bfloat16_rn(f);
    l[i] = __float2bfloat16_rn(f - __bfloat162float(h[i]));
  }
}

void compute_host_tc(int W, int H, HostTcMats &m) {
  const double pi = 3.14159265358979323846;
  std::vector<double> B1t((size_t)W * W), B3t((size_t)W * W), B5t((size_t)W * W), B3gt((size_t)W * W);
  std::vector<double> L2((size_t)H * H), L4((size_t)H * H), L6((size_t)H * H), L6g((size_t)H * H);
  for (int a = 0; a < W; ++a)      // row a of B^T = output column a
    for (int b = 0; b < W; ++b) {  // b = K index
      B1t[(size_t)a * W + b] = std::cos(pi * a * (b + 0.5) / W);                                    // kx=a, x=b
      B3t[(size_t)a * W + b] = std::sin(pi * (b + 1) * (a + 0.5) / W) * (b == W - 1 ? 0.5 : 1.0);  // x=a, kx=b
      B5t[(size_t)a * W + b] = std::cos(pi * b * (a + 0.5) / W) * (b == 0 ? 0.5 : 1.0);            // x=a, kx=b
      B3gt[(size_t)a * W + b] = -std::sin(pi * b * (a + 0.5) / W);                                  // x=a, kx=b
    }
  for (int a = 0; a < H; ++a)
    for (int b = 0; b < H; ++b) {
      L2[(size_t)a * H + b] = std::cos(pi * a * (b + 0.5) / H);                                     // ky=a, y=b
      L4[(size_t)a * H + b] = std::cos(pi * b * (a + 0.5) / H) * (b == 0 ? 0.5 : 1.0);             // y=a, ky=b
      L6[(size_t)a * H + b] = std::sin(pi * (b + 1) * (a + 0.5) / H) * (b == H - 1 ? 0.5 : 1.0);   // y=a, ky=b
      L6g[(size_t)a * H + b] = -std::sin(pi * b * (a + 0.5) / H);                                   // y=a, ky=b
    }
  const std::vector<double> *src[8] = {&B1t, &B3t, &B5t, &B3gt, &L2, &L4, &L6, &L6g};
  for (int k = 0; k < 8; ++k) split_planes(*src[k], m.hi[k], m.lo[k]);
}

const HostTcMats &host_tc(int W, int H) {
  static std::mutex mu;
  static auto *cache = new std::map<std::pair<int, int>, std::unique_ptr<HostTcMats>>();  // kept for the process
  std::lock_guard<std::mutex> g(mu);
  auto &slot = (*cache)[{W, H}];
  if (!slot) {
    slot.reset(new HostTcMats());
    compute_host_tc(W, H, *slot);
  }
  return *slot;
}

void upload_planes(DBuf<__nv_bfloat16> &hi, DBuf<__nv_bfloat16> &lo, const std::vector<__nv_bfloat16> &h,
                   const std::vector<__nv_bfloat16> &l, cudaStream_t s) {
  hi.ensure(h.size());
  lo.ensure(l.size());
  hi.upload(h.data(), h.size(), s);
  lo.upload(l.data(), l.size(), s);
}

// Uploads the kept hi/lo DCT matrices and builds the operand buffers and the
// tensor maps of the four GEMM launches (two field formulas for the inverse
// transforms).
void setup_tc(eplace_ctx *c) {
  AllocOn on_stream(c->stream);
  if (c->tc_ready) return;
  const int W = c->hp.BX, H = c->hp.BY;
  cudaStream_t s = c->stream;
  const HostTcMats &hm = host_tc(W, H);
  DBuf<__nv_bfloat16> *dh[8] = {&c->B1t_h, &c->B3t_h, &c->B5t_h, &c->B3gt_h, &c->L2_h, &c->L4_h, &c->L6_h, &c->L6g_h};
  DBuf<__nv_bfloat16> *dl[8] = {&c->B1t_l, &c->B3t_l, &c->B5t_l, &c->B3gt_l, &c->L2_l, &c->L4_l, &c->L6_l, &c->L6g_l};
  for (int k = 0; k < 8; ++k) upload_planes(*dh[k], *dl[k], hm.hi[k], hm.lo[k], s);
  const size_t nb = (size_t)W * H;
  for (auto *b : {&c->rho_h, &c->rho_l, &c->Tt_h, &c->Tt_l, &c->Exh_h, &c->Exh_l, &c->Eyh_h, &c->Eyh_l, &c->Ut_h,
                  &c->Ut_l, &c->Vt_h, &c->Vt_l})
    b->ensure(nb);
  auto ops = [&](const DBuf<__nv_bfloat16> &ah, const DBuf<__nv_bfloat16> &al, int mrows, int k,
                 const DBuf<__nv_bfloat16> &bh, const DBuf<__nv_bfloat16> &bl, int nrows) {
    TcOperandMaps m;
    m.a_hi = make_map(ah.p, mrows, k, 128);
    m.a_lo = make_map(al.p, mrows, k, 128);
    m.b_hi = make_map(bh.p, nrows, k, kTcBN);
    m.b_lo = make_map(bl.p, nrows, k, kTcBN);
    m.b_hi32 = make_map(bh.p, nrows, k, 32);
    m.b_lo32 = make_map(bl.p, nrows, k, 32);
    m.b_hi128 = nrows >= 128 ? make_map(bh.p, nrows, k, 128) : m.b_hi;  // used only when N % 128 == 0
    m.b_lo128 = nrows >= 128 ? make_map(bl.p, nrows, k, 128) : m.b_lo;
    return m;
  };
  // GEMM1  T   = rho * B1          A = rho (H x W),  B^T = B1t (W x W)
  c->tm1.op[0] = ops(c->rho_h, c->rho_l, H, W, c->B1t_h, c->B1t_l, W);
  // GEMM2  Coef = L2 * T           A = L2 (H x H),   B^T = T^T (W x H)
  c->tm2.op[0] = ops(c->L2_h, c->L2_l, H, H, c->Tt_h, c->Tt_l, W);
  // GEMM3  U = Ex^ * B3, V = Ey^ * B5 (reference) / U = Ex^ * B3g (gradient)
  c->tm3[0].op[0] = ops(c->Exh_h, c->Exh_l, H, W, c->B3t_h, c->B3t_l, W);
  c->tm3[0].op[1] = ops(c->Eyh_h, c->Eyh_l, H, W, c->B5t_h, c->B5t_l, W);
  c->tm3[1].op[0] = ops(c->Exh_h, c->Exh_l, H, W, c->B3gt_h, c->B3gt_l, W);
  c->tm3[1].op[1] = c->tm3[0].op[1];
  // GEMM4  Ex = L4 * U, Ey = L6 * V (reference) / Ey = L6g * V (gradient)
  c->tm4[0].op[0] = ops(c->L4_h, c->L4_l, H, H, c->Ut_h, c->Ut_l, W);
  c->tm4[0].op[1] = ops(c->L6_h, c->L6_l, H, H, c->Vt_h, c->Vt_l, W);
  c->tm4[1].op[0] = c->tm4[0].op[0];
  c->tm4[1].op[1] = ops(c->L6g_h, c->L6g_l, H, H, c->Vt_h, c->Vt_l, W);
  CK(cudaStreamSynchronize(s));
  c->tc_ready = true;
  ++c->buf_epoch;
}

int *err_ptr(eplace_ctx *c) { return reinterpret_cast<int *>(reinterpret_cast<char *>(c->sc.p) + offsetof(DevScalars, err)); }

void launch_final_stage(eplace_ctx *c, double *dens_out, bool tc = false) {
  const HostProblem &hp = c->hp;
  const int nb = hp.BX * hp.BY;
  const double c0 = c->total_area / (double)nb;
  FinalArgs a{c->dens.p, nb, (double)hp.sx * hp.sy, c0, tc ? nullptr : c->rho.p, tc ? c->rho_h.p : nullptr,
              tc ? c->rho_l.p : nullptr, dens_out, 0, c->part.p, c->bar.p + 2, c->sc.p, c->log.p};
  CK(launch_density_final(a, grid_for((nb + 3) / 4, kFinalBlock, c->num_sms * 4), c->stream));
}

// One of the four GEMM launches of a field solve (density.rs:96-166):
//   0: T = rho * B1 (row DCT-II)          1: Coef = L2 * T + spectral epilogue
//   2: U = Ex^ * B3, V = Ey^ * B5          3: Ex = L4 * U, Ey = L6 * V
// from_dens (FFT form, stage 0): read the fixed-point density map itself,
// with the finalise (charge, map clear, overlap) fused into the stage.
void launch_field_gemm(eplace_ctx *c, int g, float *phi, int field_mode, bool tc, bool from_dens = false) {
  const int W = c->hp.BX, H = c->hp.BY;
  const int fm = field_mode == EPLACE_FIELD_POTENTIAL_GRADIENT ? 1 : 0;
  if (tc) {
    TcGemmEpi e{};
    e.err = err_ptr(c);
    e.wx = c->wx.p;
    e.gx2 = c->gx2.p;
    e.wy = c->wy.p;
    e.gy2 = c->gy2.p;
    e.scale = (float)(4.0 / ((double)W * H));
    switch (g) {
      case 0:
        e.mode = TC_EPI_SPLIT_T;
        e.out[0] = TcEpiOut{nullptr, c->Tt_h.p, c->Tt_l.p, nullptr, nullptr};
        CK(launch_tc_gemm(c->tm1, e, 1, H, W, W, c->stream));
        break;
      case 1:
        e.mode = TC_EPI_SPECTRAL;
        e.phi = phi;
        e.out[0] = TcEpiOut{nullptr, c->Exh_h.p, c->Exh_l.p, c->Eyh_h.p, c->Eyh_l.p};
        CK(launch_tc_gemm(c->tm2, e, 1, H, W, H, c->stream));
        break;
      case 2:
        e.mode = TC_EPI_SPLIT_T;
        e.out[0] = TcEpiOut{nullptr, c->Ut_h.p, c->Ut_l.p, nullptr, nullptr};
        e.out[1] = TcEpiOut{nullptr, c->Vt_h.p, c->Vt_l.p, nullptr, nullptr};
        CK(launch_tc_gemm(c->tm3[fm], e, 2, H, W, W, c->stream));
        break;
      default:
        e.mode = TC_EPI_F32;
        e.out[0] = TcEpiOut{c->Ex.p, nullptr, nullptr, nullptr, nullptr};
        e.out[1] = TcEpiOut{c->Ey.p, nullptr, nullptr, nullptr, nullptr};
        CK(launch_tc_gemm(c->tm4[fm], e, 2, H, W, H, c->stream));
        break;
    }
    return;
  }
  if (c->fft) {
    FftStageArgs a{};
    a.W = W;
    a.H = H;
    a.tx = FftTables{c->fft_twx.p, c->fft_tqx.p};
    a.ty = FftTables{c->fft_twy.p, c->fft_tqy.p};
    const int sn = fm ? FFT_SG : FFT_S3;  // Ex's transform along x, Ey's along y
    switch (g) {
      case 0:
        a.in_a = c->rho.p;
        a.out_a = c->T.p;
        if (from_dens) {
          a.dens = c->dens.p;
          a.cap = (double)c->hp.sx * c->hp.sy;
          a.c0 = c->total_area / ((double)W * H);
          a.part = c->part.p;
          a.ticket = c->bar.p + 2;
          a.sc = c->sc.p;
          a.log = c->log.p;
        }
        break;
      case 1:  // forward along y, spectral, then back along y: U, V
        a.in_a = c->T.p;
        a.out_a = c->U.p;
        a.out_b = c->V.p;
        a.kind_a = FFT_C3;
        a.kind_b = sn;
        a.wx = c->wx.p;
        a.gx2 = c->gx2.p;
        a.wy = c->wy.p;
        a.gy2 = c->gy2.p;
        a.scale = (float)(4.0 / ((double)W * H));
        a.phi = phi;
        break;
      case 2:
        a.in_a = c->U.p;
        a.in_b = c->V.p;
        a.out_a = c->Ex.p;
        a.out_b = c->Ey.p;
        a.kind_a = sn;
        a.kind_b = FFT_C3;
        break;
      default:
        return;  // three stages: the fourth slot launches nothing
    }
    CK(launch_fft_stage(g, a, c->stream));
    return;
  }
  if (c->fold) {
    const GemmOp *h = c->hops.p + 12 * fm;
    const FlyOp *f = c->fops.p + 4 * fm;
    const int hw = W / 2, hh = H / 2;
    switch (g) {
      case 0:
        CK(launch_sgemm(h + 0, 2, H, hw, hw, c->stream, c->gemm_tile[0]));
        break;
      case 1: {
        SpectralArgs sp{c->wx.p, c->gx2.p, c->wy.p, c->gy2.p, (float)(4.0 / ((double)W * H)), phi};
        CK(launch_sgemm_spectral(h + 2, 2, hh, W, hh, sp, c->stream, c->gemm_tile[1]));
        break;
      }
      case 2:
        CK(launch_sgemm(h + 4, 4, H, hw, hw, c->stream, c->gemm_tile[2]));
        CK(launch_fly_cols(f, 2, H, W, c->stream));
        break;
      default:
        CK(launch_sgemm(h + 8, 4, hh, W, hh, c->stream, c->gemm_tile[3]));
        CK(launch_fly_rows(f + 2, 2, H, W, c->stream));
        break;
    }
    return;
  }
  const GemmOp *ops = c->ops.p + (fm ? 6 : 0);
  switch (g) {
    case 0:
      CK(launch_sgemm(ops + 0, 1, H, W, W, c->stream, c->gemm_tile[0]));
      break;
    case 1: {
      SpectralArgs sp{c->wx.p, c->gx2.p, c->wy.p, c->gy2.p, (float)(4.0 / ((double)W * H)), phi};
      CK(launch_sgemm_spectral(ops + 1, 1, H, W, H, sp, c->stream, c->gemm_tile[1]));
      break;
    }
    case 2:
      CK(launch_sgemm(ops + 2, 2, H, W, W, c->stream, c->gemm_tile[2]));
      break;
    default:
      CK(launch_sgemm(ops + 4, 2, H, W, H, c->stream, c->gemm_tile[3]));
      break;
  }
}

void launch_field_stage(eplace_ctx *c, float *phi, int field_mode, bool tc = false, bool from_dens = false) {
  for (int g = 0; g < 4; ++g) launch_field_gemm(c, g, phi, field_mode, tc, from_dens && g == 0);
}

// The FFT form takes the density finalise into its first stage.
bool final_fused(const eplace_ctx *c, bool tc) { return c->fft && !tc; }

// --- launch-shape autotuner ------------------------------------------------
// Picks, by timing on the context's stream, the grid caps of the WA and
// scatter kernels (4, 8, 16 or 32 blocks per SM) and the CTA tile of each
// SIMT GEMM (64 or 32).  Every candidate computes the same bits (fixed-point
// atomics; the GEMM sums each output in order whatever the tile), so the
// choice only moves time.  Results are kept per process for a shape class
// (cells and pins to the next power of two, bin grid, transform) and reused
// by every context of that class.  Runs after reset_state (positions are the
// initial placement), and clears the accumulators it dirtied.  A context on a
// shared device (the job engine) keeps the default shapes: timings taken
// beside other jobs' kernels do not rank the candidates, and the host
// legaliser, not the kernels, bounds the engine's rate.
struct TuneKey {
  int n2, p2, bx, by, tc;
  bool operator<(const TuneKey &o) const {
    return std::tie(n2, p2, bx, by, tc) < std::tie(o.n2, o.p2, o.bx, o.by, o.tc);
  }
};
struct TuneVal {
  int wa, sc, tile[4];
};

void autotune_launches(eplace_ctx *c, float gamma, int field_mode, bool tc) {
  if (c->shared_device) {
    c->wa_blocks_per_sm = 16;
    c->sc_blocks_per_sm = 16;
    std::fill(c->gemm_tile, c->gemm_tile + 4, 0);
    return;
  }
  static std::mutex mu;
  static std::map<TuneKey, TuneVal> *cache = new std::map<TuneKey, TuneVal>();  // process lifetime
  const HostProblem &hp = c->hp;
  auto lg = [](uint64_t v) {
    int k = 0;
    while ((1ull << k) < v) ++k;
    return k;
  };
  const TuneKey key{lg(hp.N), lg(hp.P), hp.BX, hp.BY, tc ? 1 : 0};
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache->find(key);
    if (it != cache->end()) {
      c->wa_blocks_per_sm = it->second.wa;
      c->sc_blocks_per_sm = it->second.sc;
      std::copy(it->second.tile, it->second.tile + 4, c->gemm_tile);
      return;
    }
  }
  cudaStream_t s = c->stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto timed = [&](auto &&launch) {
    launch();  // warm
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
      CK(cudaEventRecord(e0, s));
      launch();
      CK(cudaEventRecord(e1, s));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      best = std::min(best, ms);
    }
    return best;
  };
  TuneVal v{16, 16, {0, 0, 0, 0}};
  try {
    const int cand[4] = {4, 8, 16, 32};
    float bw = 1e30f, bs = 1e30f;
    for (int m : cand) {
      c->wa_blocks_per_sm = m;
      const float t = timed([&] { launch_wa_stage(c, gamma); });
      if (t < bw) {
        bw = t;
        v.wa = m;
      }
      c->sc_blocks_per_sm = m;
      const float u = timed([&] { launch_scatter_stage(c); });
      if (u < bs) {
        bs = u;
        v.sc = m;
      }
    }
    if (!tc && !c->fft) {
      for (int g = 0; g < 4; ++g) {
        float bt = 1e30f;
        for (int tile : {64, 32}) {
          c->gemm_tile[g] = tile;
          const float t = timed([&] { launch_field_gemm(c, g, nullptr, field_mode, false); });
          if (t < bt) {
            bt = t;
            v.tile[g] = tile;
          }
        }
      }
    }
    c->acc.zero(s);
    c->dens.zero(s);
    CK(cudaStreamSynchronize(s));
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->wa_blocks_per_sm = v.wa;
  c->sc_blocks_per_sm = v.sc;
  std::copy(v.tile, v.tile + 4, c->gemm_tile);
  std::lock_guard<std::mutex> g(mu);
  (*cache)[key] = v;
}

StepArgs step_args(eplace_ctx *c) {
  const HostProblem &hp = c->hp;
  StepArgs a{};
  a.N = hp.N;
  a.BX = hp.BX;
  a.BY = hp.BY;
  a.isx = hp.sx;
  a.isy = hp.sy;
  a.maxx = (float)(hp.W - 1);
  a.maxy = (float)(hp.H - 1);
  a.look = c->look.p;
  a.half = hp.any_macro ? c->half.p : nullptr;
  a.area = hp.any_macro ? c->area.p : nullptr;
  a.mflag = hp.any_macro ? c->mflag.p : nullptr;
  a.mac_idx = hp.any_macro ? c->mac_idx.p : nullptr;
  a.n_mac = hp.any_macro ? c->n_mac : 0;
  a.pw = c->pw.p;
  a.acc = c->acc.p;
  a.grad_inv = std::ldexp(1.0, -c->grad_k);
  a.Ex = c->Ex.p;
  a.Ey = c->Ey.p;
  a.x = c->x.p;
  a.xp = c->xp.p;
  a.g = c->g.p;
  a.gprev = c->gprev.p;
  a.tmp_wl = c->tmp_wl.p;
  a.tmp_den = c->tmp_den.p;
  a.mom = c->mom.p;
  a.sc = c->sc.p;
  a.log = c->log.p;
  a.part = c->part.p;
  a.part2 = c->part2.p;
  a.part_b = c->part_b.p;
  a.bar = c->bar.p;
  a.ticket = c->bar.p + 3;
  a.mode = 0;
  return a;
}

void launch_step_stage(eplace_ctx *c) {
  StepArgs a = step_args(c);
  if (c->split_step) CK(launch_step_split(a, c->step_grid, c->stream));
  else CK(launch_step(a, c->step_grid, c->stream));
}

// One iteration.  The WA gradient and the density -> field chain both read
// only the look-ahead positions and write separate buffers, so WA runs on
// the side stream beside scatter / finalise / the four GEMMs; the step joins
// both.  (In a captured graph this is a fork and a join.)
void launch_iteration(eplace_ctx *c, float gamma, int field_mode, bool tc) {
  CK(cudaEventRecord(c->ev_fork, c->stream));
  CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
  launch_wa_stage(c, gamma, c->side);
  CK(cudaEventRecord(c->ev_join, c->side));
  launch_scatter_stage(c);
  const bool fuse = final_fused(c, tc);
  if (!fuse) launch_final_stage(c, nullptr, tc);
  launch_field_stage(c, nullptr, field_mode, tc, fuse);
  CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
  launch_step_stage(c);
}

constexpr int kLaunchesPerIter = 8;  // with the cooperative step; +2 with the split step, -2 with the FFT form

void upload_momentum(eplace_ctx *c, uint64_t iters) {
  AllocOn on_stream(c->stream);
  // FISTA sequence a_0 = 1, a_{k+1} = (1 + sqrt(1 + 4 a_k^2)) / 2; the
  // look-ahead and the step of iteration k both use m_k = (a_k - 1) / a_{k+1}
  // (nesterov.rs:41-64, :75-82; m_0 = 0).
  std::vector<double> m(iters + 2);
  double a = 1.0;
  for (size_t k = 0; k < m.size(); ++k) {
    double an = (1.0 + std::sqrt(1.0 + 4.0 * a * a)) / 2.0;
    m[k] = (a - 1.0) / an;
    a = an;
  }
  if (c->mom.cap < m.size()) {
    c->mom.alloc(std::max<size_t>(m.size(), 1024));
    ++c->buf_epoch;
  }
  c->mom.upload(m.data(), m.size(), c->stream);
}

// Uploads what every device legalisation reads: the cell order (macros
// first), the footprints and the free map with the fixed cells.
void setup_gpu_legal(eplace_ctx *c) {
  AllocOn on_stream(c->stream);
  if (c->lg_ready) return;
  const HostProblem &hp = c->hp;
  if (!c->lbase) c->lbase.reset(new LegalBase(hp));
  const LegalBase &b = *c->lbase;
  c->lg_macros = false;
  std::vector<uchar2> fs(hp.N);
  for (uint32_t i = 0; i < hp.N; ++i) {
    fs[i] = make_uchar2(hp.cw[i], hp.ch[i]);
    c->lg_macros |= hp.cw[i] * hp.ch[i] > 1;
  }
  c->lg_order.ensure(std::max<size_t>(b.order.size(), 1));
  c->lg_order.upload(b.order.data(), b.order.size(), c->stream);
  if (c->lg_macros) {
    c->lg_fsize.ensure(std::max<size_t>(fs.size(), 1));
    c->lg_fsize.upload(fs.data(), fs.size(), c->stream);
  }
  c->lg_free0.ensure(b.free0.size());
  c->lg_free0.upload(b.free0.data(), b.free0.size(), c->stream);
  CK(cudaStreamSynchronize(c->stream));
  c->lg_ready = true;
}

// Sizes slot L for the current problem (capacity reuse) and writes the
// fixed cells' pin locations after a (re)load.
void prepare_slot(eplace_ctx *c, LegalSlot &L) {
  AllocOn on_stream(L.stream);  // synchronised below
  const HostProblem &hp = c->hp;
  if (L.gen == c->load_gen) return;
  const size_t N1 = std::max<size_t>(hp.N, 1);
  L.pos.ensure(N1);
  L.sites.ensure(N1);
  L.loc.ensure((size_t)hp.N + hp.F + 1);
  L.cost.ensure(N1);
  const int WR = (hp.W + 63) / 64;
  const size_t sites = (size_t)hp.W * hp.H;
  L.fm.ensure((size_t)WR * hp.H);
  L.list.ensure((size_t)kLpMaxWindow * kLpList);
  L.len.ensure(kLpMaxWindow);
  L.info.ensure(kLpMaxWindow);
  L.pick.ensure(kLpMaxWindow);
  L.dist.ensure(kLpMaxWindow);
  L.fresh.ensure(kLpMaxWindow);
  L.hmark.ensure(sites);
  L.dmark.ensure(sites);
  L.lst.ensure(1);
  std::vector<int2> floc(hp.F);
  for (uint32_t f = 0; f < hp.F; ++f) floc[f] = make_int2(hp.fx[f], hp.fy[f]);
  if (hp.F) CK(cudaMemcpyAsync(L.loc.p + hp.N, floc.data(), sizeof(int2) * hp.F, cudaMemcpyHostToDevice, L.stream));
  g_h2d += sizeof(int2) * hp.F;
  CK(cudaStreamSynchronize(L.stream));
  // The legalisation graph bakes in this load's buffers.
  LpArgs a{};
  a.pos = L.pos.p;
  a.order = c->lg_order.p;
  a.fsize = c->lg_macros ? c->lg_fsize.p : nullptr;
  a.n = (uint32_t)c->lbase->order.size();
  a.W = hp.W;
  a.H = hp.H;
  a.WR = WR;
  a.free0 = c->lg_free0.p;
  a.fm = L.fm.p;
  a.list = L.list.p;
  a.len = L.len.p;
  a.info = L.info.p;
  a.hmark = L.hmark.p;
  a.dmark = L.dmark.p;
  a.dist = L.dist.p;
  a.fresh = L.fresh.p;
  a.pick = L.pick.p;
  a.st = L.lst.p;
  a.sites = L.sites.p;
  a.loc = L.loc.p;
  a.cost = L.cost.p;
  a.disp = &L.out.p->disp;
  a.status = &L.out.p->status;
  a.max_rounds = a.n + 64;
  CK(lp_build_graph(a, L.graph, L.stream));
  L.gen = c->load_gen;
}

// Allocates one more legalisation slot (lowest stream priority).
LegalSlot *new_legal_slot(eplace_ctx *c) {
  std::unique_ptr<LegalSlot> L(new LegalSlot());
  int prio_lo = 0, prio_hi = 0;
  CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  CK(cudaStreamCreateWithPriority(&L->stream, cudaStreamNonBlocking, prio_lo));
  AllocOn on_stream(L->stream);  // prepare_slot synchronises it
  CK(cudaEventCreateWithFlags(&L->snap, cudaEventDisableTiming));
  CK(cudaEventCreate(&L->start));
  CK(cudaEventCreate(&L->done));
  L->out.alloc(1);
  L->hout.alloc(1);
  prepare_slot(c, *L);
  c->lslots.push_back(std::move(L));
  return c->lslots.back().get();
}

// Legalises slot L's positions and takes the HPWL of the binding, all on
// L's stream, then copies the 24-byte outcome to pinned memory and records
// L.done.  The caller has already ordered the positions before this work.
void launch_gpu_legal(eplace_ctx *c, LegalSlot &L) {
  const HostProblem &hp = c->hp;
  CK(cudaMemsetAsync(L.out.p, 0, sizeof(LegalOut), L.stream));
  CK(cudaEventRecord(L.start, L.stream));
  CK(cudaGraphLaunch(L.graph.exec, L.stream));
  HpwlArgs h{c->net_off.p, c->pin_cell.p, c->has_driver.p, L.loc.p, hp.NN, &L.out.p->hpwl};
  if (hp.NN) CK(launch_hpwl(h, grid_for((int)hp.NN, kHpwlBlock, c->num_sms * 2), L.stream));
  CK(cudaMemcpyAsync(L.hout.p, L.out.p, sizeof(LegalOut), cudaMemcpyDeviceToHost, L.stream));
  g_d2h += sizeof(LegalOut);
  CK(cudaEventRecord(L.done, L.stream));
}

// (Re)targets a context at a validated problem.  Device buffers only grow
// (capacity reuse: no frees, which would synchronise the device); the DCT
// matrices and the tensor-core operands are rebuilt only when the bin grid
// changes; every captured graph is invalidated.
void load_into(eplace_ctx *c, HostProblem &&hp_in) {
  AllocOn on_stream(c->stream);
  const bool same_bins = c->mat_bx == hp_in.BX && c->mat_by == hp_in.BY;
  c->hp = std::move(hp_in);
  const HostProblem &hp = c->hp;
  cudaStream_t s = c->stream;
  // host-side structures of the previous problem
  c->legal.clear();
  c->lbase.reset();
  c->lg_ready = false;
  ++c->load_gen;
  if (c->gexec) {
    c->g_valid = false;  // updated in place by the next capture
  }
  ++c->buf_epoch;
  // Host-side derived arrays are built on two helper threads while this
  // thread uploads the netlist; all CUDA calls stay on this thread.
  std::vector<uint32_t> sorder, soff, spins;
  WaClass cls[kWaClasses];
  int wa_warps = 0;
  const size_t wa_cap = 2 * (size_t)hp.P + 64;
  if (c->wa_pin_ev) CK(cudaEventSynchronize(c->wa_pin_ev));  // the last upload from the block is done
  c->wa_pin.reserve(sizeof(uint32_t) * wa_cap);
  uint32_t *slots = static_cast<uint32_t *>(c->wa_pin.p);
  size_t nslots = 0;
  std::exception_ptr wa_err;
  std::thread t_wa([&] {
    degree_order(hp, sorder, soff);
    wa_warps = build_wa_classes(soff, cls);
    sorted_pins(hp, sorder, soff, (uint32_t)cls[kWaClasses - 1].first_net, hp.NN, spins);
    try {
      nslots = build_wa_slots(hp, sorder, cls, slots, wa_cap);
    } catch (...) {
      wa_err = std::current_exception();
    }
  });
  int grad_k = 24;
  std::thread t_pw([&] { pin_weights(hp, c->pw_host); });
  std::thread t_hp([&] {
    grad_k = grad_scale_log2(hp);
    build_hpwl_table(c->hp);  // its own members only; the others read the rest
  });
  struct Joiner {  // joins the helpers on every exit, an upload error included
    std::thread &a, &b, &d;
    ~Joiner() {
      for (std::thread *t : {&a, &b, &d})
        if (t->joinable()) t->join();
    }
  } joiner{t_wa, t_pw, t_hp};
  c->net_off.ensure(hp.net_off.size());
  c->net_off.upload(hp.net_off.data(), hp.net_off.size(), s);
  c->pin_cell.ensure(std::max<size_t>(hp.P, 1));
  c->pin_cell.upload(hp.pin_cell.data(), hp.P, s);
  c->has_driver.ensure(std::max<size_t>(hp.NN, 1));
  c->has_driver.upload(hp.has_driver.data(), hp.NN, s);
  const size_t N1 = std::max<size_t>(hp.N, 1);
  std::vector<float2> half(hp.N);
  std::vector<float> area(hp.N);
  double tot = 0.0;
  for (uint32_t i = 0; i < hp.N; ++i) {
    half[i] = make_float2(0.5f * hp.cw[i], 0.5f * hp.ch[i]);
    area[i] = (float)(hp.cw[i] * hp.ch[i]);
    tot += area[i];
  }
  c->total_area = tot;
  c->half.ensure(N1);
  c->half.upload(half.data(), hp.N, s);
  c->area.ensure(N1);
  c->area.upload(area.data(), hp.N, s);
  {
    std::vector<uint8_t> mf(hp.N, 0);
    std::vector<uint32_t> mi;
    for (uint32_t i = 0; i < hp.N; ++i)
      if (hp.cw[i] * hp.ch[i] > 1) {
        mf[i] = 1;
        mi.push_back(i);
      }
    c->n_mac = (uint32_t)mi.size();
    c->mflag.ensure(N1);
    c->mflag.upload(mf.data(), hp.N, s);
    c->mac_idx.ensure(std::max<size_t>(mi.size(), 1));
    c->mac_idx.upload(mi.data(), mi.size(), s);
  }
  c->look.ensure((size_t)hp.N + hp.F + 1);
  std::vector<float2> fixed(hp.F);
  for (uint32_t f = 0; f < hp.F; ++f) fixed[f] = make_float2((float)hp.fx[f], (float)hp.fy[f]);
  if (hp.F) CK(cudaMemcpyAsync(c->look.p + hp.N, fixed.data(), sizeof(float2) * hp.F, cudaMemcpyHostToDevice, s));
  g_h2d += sizeof(float2) * hp.F;
  for (auto *b : {&c->x, &c->xp, &c->g, &c->gprev, &c->tmp_wl, &c->tmp_den}) b->ensure(N1);
  c->acc.ensure(N1);
  c->acc.zero(s);
  const size_t nb = (size_t)hp.BX * hp.BY;
  c->dens.ensure(nb);
  c->dens.zero(s);
  if (!same_bins) {
    for (auto *b : {&c->rho, &c->T, &c->Exh, &c->Eyh, &c->U, &c->V, &c->Ex, &c->Ey}) b->ensure(nb);
    build_matrices(c);
    c->mat_bx = hp.BX;
    c->mat_by = hp.BY;
    c->tc_ready = false;
  }
  // Two blocks per SM: enough to stream the cells, few arrivals per grid
  // barrier (the grid must stay co-resident for the cooperative launch).
  c->step_grid = std::max(1, std::min({step_max_grid(c->device), c->num_sms * 2,
                                       grid_for((int)hp.N, kStepBlock, 1 << 30)}));
  c->step_grid_full = c->step_grid;
  c->part.ensure(4 * (size_t)std::max(c->step_grid, c->num_sms * 4) + 8);
  c->part2.ensure(2 * (size_t)c->step_grid + 8);
  c->part_b.ensure(4 * (size_t)c->step_grid + 8);
  c->bar.zero(s);
  c->loc.ensure((size_t)hp.N + hp.F + 1);
  std::vector<int2> floc(hp.F);
  for (uint32_t f = 0; f < hp.F; ++f) floc[f] = make_int2(hp.fx[f], hp.fy[f]);
  if (hp.F) CK(cudaMemcpyAsync(c->loc.p + hp.N, floc.data(), sizeof(int2) * hp.F, cudaMemcpyHostToDevice, s));
  g_h2d += sizeof(int2) * hp.F;
  // The helpers' results last: the work above did not need them.
  t_wa.join();
  {
    std::copy(cls, cls + kWaClasses, c->wa_cls);
    c->wa_warps = wa_warps;
    // The sorted CSR itself is read only by the last class (nets of more
    // than 224 pins); the others read the padded table.
    c->wa_off.ensure(soff.size());
    c->wa_off.upload(soff.data(), soff.size(), s);
    // Only the last class's part of the sorted pin list is uploaded, at its
    // sorted-CSR place; no other class reads it.
    c->wa_pins.ensure(std::max<size_t>(hp.P, 1));
    if (c->wa_cls[kWaClasses - 1].nets > 0 && !spins.empty()) {
      const size_t at = soff[c->wa_cls[kWaClasses - 1].first_net];
      CK(cudaMemcpyAsync(c->wa_pins.p + at, spins.data(), sizeof(uint32_t) * spins.size(), cudaMemcpyHostToDevice, s));
      g_h2d += sizeof(uint32_t) * spins.size();
    }
    if (wa_err) std::rethrow_exception(wa_err);
    c->wa_slots.ensure(nslots);
    c->wa_slots.upload(slots, nslots, s);  // from pinned memory: asynchronous
    if (!c->wa_pin_ev) CK(cudaEventCreateWithFlags(&c->wa_pin_ev, cudaEventDisableTiming));
    CK(cudaEventRecord(c->wa_pin_ev, s));
  }
  t_pw.join();
  std::vector<float> pwf(c->pw_host.begin(), c->pw_host.end());
  c->pw.ensure(N1);
  c->pw.upload(pwf.data(), hp.N, s);
  t_hp.join();
  c->grad_k = grad_k;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int32_t eplace_abi_version(void) { return EPLACE_ABI_VERSION; }

void eplace_cfg_default(eplace_cfg *c) {
  if (!c) return;
  c->seed = 1;
  c->wl_coeff = 0.5;
  c->target_util = 0.7;
  c->timing_driven = 0;
  c->target_density = 1.0;
  c->timing_weight = 0.0;
  c->nesterov_step_size = 0.1;
  c->max_iters = 500;
  c->legalize_interval = 5;
}

void eplace_opts_default(eplace_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->dct_mode = EPLACE_DCT_FP32_FFT;
  o->legal_threads = 0;
  o->use_graphs = 1;
  o->verbose = 0;
  o->max_inflight = 3;
  o->field_mode = EPLACE_FIELD_REFERENCE;
}

size_t eplace_last_error(const eplace_ctx *ctx, char *buf, size_t len) {
  const std::string &m = ctx ? ctx->err : g_thread_error;
  if (buf && len) {
    size_t k = std::min(len - 1, m.size());
    std::memcpy(buf, m.data(), k);
    buf[k] = 0;
  }
  return m.size();
}

eplace_status eplace_ctx_create(const eplace_netlist *nl, const eplace_chip *chip, int32_t device,
                                eplace_ctx **out) {
  if (!out) return EPLACE_ERR_INVALID;
  *out = nullptr;
  std::string msg;
  HostProblem hp;
  eplace_status st = load_problem(nl, chip, hp, msg);
  if (st != EPLACE_OK) {
    set_err(nullptr, msg);
    return st;
  }
  eplace_ctx *c = ctx_new(device, &st);
  if (!c) return st;
  st = ctx_load_problem(c, std::move(hp));
  if (st != EPLACE_OK) {
    g_thread_error = c->err;
    delete c;
    return st;
  }
  *out = c;
  return EPLACE_OK;
}

eplace_status eplace_ctx_load(eplace_ctx *c, const eplace_netlist *nl, const eplace_chip *chip) {
  if (!c) return EPLACE_ERR_INVALID;
  std::string msg;
  HostProblem hp;
  eplace_status st = load_problem(nl, chip, hp, msg);
  if (st != EPLACE_OK) {
    set_err(c, msg);
    return st;
  }
  return ctx_load_problem(c, std::move(hp));
}

void eplace_ctx_destroy(eplace_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  delete ctx;
}

// Validates the run options against this context.
static eplace_status check_modes(eplace_ctx *c, const eplace_opts &o) {
  if (o.dct_mode != EPLACE_DCT_FP32_SIMT && o.dct_mode != EPLACE_DCT_BF16X3_TC && o.dct_mode != EPLACE_DCT_FP32_FFT) {
    set_err(c, "unknown dct_mode");
    return EPLACE_ERR_INVALID;
  }
  if (o.dct_mode == EPLACE_DCT_BF16X3_TC && !tc_supported(c->hp)) {
    set_err(c, "the tensor-core transform needs bins_y % 128 == 0 and bins_x % 64 == 0");
    return EPLACE_ERR_INVALID;
  }
  if (o.field_mode != EPLACE_FIELD_REFERENCE && o.field_mode != EPLACE_FIELD_POTENTIAL_GRADIENT) {
    set_err(c, "unknown field_mode");
    return EPLACE_ERR_INVALID;
  }
  return EPLACE_OK;
}

// Resets the loop state on the device for a new run from positions (sx, sy).
// Host half of the device initial placement (placer/common.rs:27-117): the
// taken sites and the count check of the host form, without the shuffle.
// Returns false when the device form does not apply (a pre-bound cell, or a
// grid beyond 32-bit site indices): the host form runs instead.
static bool ip_device_prepare(eplace_ctx *c, eplace_status &st, std::string &msg) {
  const HostProblem &hp = c->hp;
  st = EPLACE_OK;
  if ((uint64_t)hp.W * hp.H >= (1ull << 31)) return false;
  for (uint32_t i = 0; i < hp.N; ++i)
    if (hp.init_x[i] >= 0) return false;
  std::vector<uint32_t> &occ = c->ip_occ_host;
  occ.clear();
  for (uint32_t f = 0; f < hp.F; ++f)
    if (hp.f_logic[f]) occ.push_back((uint32_t)hp.fy[f] * (uint32_t)hp.W + (uint32_t)hp.fx[f]);
  std::sort(occ.begin(), occ.end());
  occ.erase(std::unique(occ.begin(), occ.end()), occ.end());
  c->ip_n = (uint64_t)hp.W * hp.H - occ.size();
  if (hp.N > c->ip_n) {
    msg = "logic (need " + std::to_string(hp.N) + " BELs but only " + std::to_string(c->ip_n) + " available)";
    st = EPLACE_ERR_NO_BELS;
  }
  return true;
}

// Device half: the shuffle and the hand-out on the context's stream, writing
// x, x_prev and the look-ahead positions (and the integer sites).  Returns
// the kernels it launched.
static int ip_device_launch(eplace_ctx *c, uint64_t seed) {
  const HostProblem &hp = c->hp;
  cudaStream_t s = c->stream;
  AllocOn on_stream(s);  // scratch that grows is allocated in stream order
  const size_t n = c->ip_n;
  if (!c->ip_jump.p) {
    const std::vector<uint64_t> &m = ip_jump_maps();
    c->ip_jump.ensure(m.size());
    c->ip_jump.upload(m.data(), m.size(), s);
  }
  c->ip_j.ensure(std::max<size_t>(n, 1));
  c->ip_cnt.ensure(n + 1);
  c->ip_start.ensure(n + 1);
  c->ip_entries.ensure(std::max<size_t>(n, 1));
  c->ip_block.ensure((n + 1) / 1024 + 2);
  c->ip_occ.ensure(std::max<size_t>(c->ip_occ_host.size(), 1));
  c->ip_occ.upload(c->ip_occ_host.data(), c->ip_occ_host.size(), s);
  c->ip_site.ensure(std::max<size_t>(hp.N, 1));
  IpBuffers b{c->ip_j.p, c->ip_cnt.p, c->ip_start.p, c->ip_entries.p, c->ip_block.p, c->ip_jump.p,
              c->ip_occ.p, (uint32_t)c->ip_occ_host.size(), nullptr, hp.N, hp.W, c->ip_site.p,
              c->x.p, c->xp.p, c->look.p};
  CK(launch_initial_placement(b, seed ? seed : 1, (uint32_t)n, s));
  return n > 1 ? 7 : 4;
}

// sx / sy empty: the positions come from the device initial placement.
// Returns the kernels launched.  Nothing here waits for the device: the
// scalars leave first (a copy from pageable memory waits for the stream's
// earlier work, so it goes before the placement kernels, not after them),
// and every later use of the state is ordered on the same stream.
static int reset_state(eplace_ctx *c, const std::vector<int32_t> &sx, const std::vector<int32_t> &sy,
                       const eplace_cfg *cfg) {
  const HostProblem &hp = c->hp;
  cudaStream_t s = c->stream;
  c->gprev.zero(s);
  c->g.zero(s);
  c->acc.zero(s);
  c->dens.zero(s);
  DevScalars sc{};
  sc.lam = 0.0;
  sc.step[0] = sc.step[1] = cfg->nesterov_step_size;
  sc.overlap = 0.0;
  sc.lam_init = 0;
  sc.iter = 0;
  sc.err = 0;
  sc.spin_cycles = c->spin_cycles;
  c->sc.upload(&sc, 1, s);
  c->bar.zero(s);
  int launches = 0;
  if (sx.empty() && hp.N) {
    launches = ip_device_launch(c, cfg->seed);
  } else {
    std::vector<float2> p(hp.N);
    for (uint32_t i = 0; i < hp.N; ++i) p[i] = make_float2((float)sx[i], (float)sy[i]);
    c->x.upload(p.data(), hp.N, s);
    c->xp.upload(p.data(), hp.N, s);
    CK(cudaMemcpyAsync(c->look.p, p.data(), sizeof(float2) * hp.N, cudaMemcpyHostToDevice, s));
    g_h2d += sizeof(float2) * hp.N;
  }
  return launches;
}

// SM clock cycles of a wait limit given in microseconds (0: the kernel default).
static int64_t wait_cycles(int device, int32_t us) {
  if (us <= 0) return 0;
  int khz = 0;
  if (cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device) != cudaSuccess || khz <= 0) khz = 2000000;
  return (int64_t)us * (int64_t)khz / 1000;
}

namespace {
struct Checkpoint {
  int32_t iter = -1;
  size_t chunk = 0;
  // host legaliser: the snapshot and its binding
  HostSnap *hs = nullptr;
  // device legaliser: the slot holding positions and binding
  int slot = -1;
  bool discard = false;  // its interval ran past convergence
  double disp = 0.0;
  int64_t hpwl = 0;
  double secs = 0.0;  // time of its legalisation + HPWL (host clock, or device events)
  double began = 0.0;  // host legaliser: its start, seconds from the run's start
  eplace_status st = EPLACE_OK;
  std::atomic<bool> done{false};
};
}  // namespace
}  // extern "C"

namespace eplace {

// One place_electro run (electro_place/mod.rs:65-204) on a context, as a
// resumable state machine so that one host thread can drive many runs: the
// blocking entry point loops pump(true) until done(); the job engine calls
// pump(false) on each of its jobs in turn.
//
// Per interval of legalize_interval iterations (one CUDA graph): the
// interval's log and scalars are copied to pinned memory, the positions are
// snapshotted (to pinned memory for the host legaliser, to a device slot for
// the device legaliser), and the checkpoint is legalised concurrently with
// the next intervals.  Checkpoints are folded in iteration order (best =
// first minimum HPWL, common.rs:485-495).
struct JobState {
  enum Phase { kInit, kLoop, kLegal, kDone };
  struct Chunk {
    uint64_t first, last;
  };

  JobState(eplace_ctx *c_, const eplace_cfg &cfg_, const eplace_opts &opts_, eplace_result *res_, Pool *shared)
      : c(c_), cfg(cfg_), opts(opts_), res(res_), shared_pool(shared) {
    t_start = std::chrono::steady_clock::now();
    h2d0 = g_h2d;
    d2h0 = g_d2h;
  }
  ~JobState() {
    drain();
    for (auto &cp : cps) release(cp.get());
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
  bool done() const { return phase == kDone; }

  // Waits until no host legalisation of this job is queued or running and
  // the device legaliser streams are idle (they read this job's buffers).
  void drain() {
    while (outstanding.load(std::memory_order_acquire) != 0) std::this_thread::sleep_for(std::chrono::microseconds(50));
    for (auto &l : c->lslots)
      if (l && l->stream) cudaStreamSynchronize(l->stream);
  }

  void mark(const char *what) {
    marks.emplace_back(what, std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count());
  }

  eplace_status start() {
    const HostProblem &hp = c->hp;
    res->traj_len = 0;
    res->iters = 0;
    res->best_iter = -1;
    res->converged = 0;
    res->hpwl = 0;
    res->overlap = 0.0;
    res->gpu_seconds = 0.0;
    res->gpu_launches = 0;
    phase = kDone;
    if (cfg.legalize_interval == 0) {
      set_err(c, "legalize_interval must be positive");
      return final_st = EPLACE_ERR_INVALID;
    }
    if (!(cfg.wl_coeff > 0) || !std::isfinite(cfg.wl_coeff) || !std::isfinite(cfg.nesterov_step_size)) {
      set_err(c, "wl_coeff / nesterov_step_size must be finite (wl_coeff > 0)");
      return final_st = EPLACE_ERR_INVALID;
    }
    eplace_status mst = check_modes(c, opts);
    if (mst != EPLACE_OK) return final_st = mst;
    tc = opts.dct_mode == EPLACE_DCT_BF16X3_TC;
    c->fft = opts.dct_mode == EPLACE_DCT_FP32_FFT && fft_supported(hp.BX, hp.BY);
    gpu_legal = opts.legal_mode == EPLACE_LEGAL_GPU && legalize_supported(hp.W, hp.H);
    if (!res->bel_tile && hp.N) return final_st = EPLACE_ERR_INVALID;
    std::string msg;
    eplace_status st;
    if (!ip_device_prepare(c, st, msg)) {
      st = initial_placement(hp, cfg.seed, isx, isy, msg);
    }  // else: isx / isy stay empty, the placement is made on the device in reset_state
    mark("initial_placement");
    if (st != EPLACE_OK) {
      set_err(c, msg);
      return final_st = st;
    }
    if (hp.N == 0) return EPLACE_OK;  // mod.rs:80-82
    max_iters = cfg.max_iters;
    interval = cfg.legalize_interval;
    gamma = (float)cfg.wl_coeff;
    try {
      CK(cudaSetDevice(c->device));
      cudaStream_t s = c->stream;
      ensure_log(c, max_iters);
      upload_momentum(c, max_iters);
      if (tc) setup_tc(c);
      const bool want_split = gpu_legal || c->shared_device;
      if (want_split != c->split_step) {
        c->split_step = want_split;
        ++c->buf_epoch;
      }
      c->spin_cycles = wait_cycles(c->device, opts.wait_limit_us);
      ip_launches = reset_state(c, isx, isy, &cfg);
      autotune_launches(c, gamma, opts.field_mode, tc);
      mark("device_reset");
      // Host resources persist in the context across runs.
      if (!c->lbase) c->lbase.reset(new LegalBase(hp));
      if (gpu_legal) {
        setup_gpu_legal(c);
        if (c->legal.empty()) c->legal.emplace_back(new Legalizer(hp, *c->lbase));
      } else {
        if (shared_pool) {
          pool = shared_pool;
        } else {
          int n = opts.legal_threads > 0 ? opts.legal_threads : (int)std::max(1u, std::thread::hardware_concurrency());
          n = std::min(n, 64);
          if (!c->pool || c->pool->size() != n) {
            c->pool.reset();
            c->pool.reset(new Pool(n));
          }
          pool = c->pool.get();
        }
        while ((int)c->legal.size() < pool->size()) c->legal.emplace_back(new Legalizer(hp, *c->lbase));
      }
      CK(cudaEventCreate(&ev0));
      CK(cudaEventCreate(&ev1));
      // Interval boundaries: iterations k with k % interval == 0, plus the last.
      uint64_t k = 0;
      while (k < max_iters) {
        uint64_t last = (k == 0) ? 0 : std::min(max_iters - 1, ((k + interval - 1) / interval) * interval);
        if (last < k) last = max_iters - 1;
        chunks.push_back({k, last});
        k = last + 1;
      }
      // Pinned ring of interval outputs (log and scalars); the positions of
      // a checkpoint the host legalises go to a HostSnap of their own.
      inflight = std::max(1, std::min(opts.max_inflight, 8));
      if ((int)c->logs.size() < inflight || c->slot_log_cap < interval + 1) {
        c->logs.clear();
        c->scs.clear();
        for (auto e : c->slot_ev) cudaEventDestroy(e);
        c->slot_ev.clear();
        c->slot_log_cap = std::max<uint64_t>(interval + 1, 16);
        for (int i = 0; i < inflight; ++i) {
          c->logs.emplace_back(new PinBuf<IterLog>());
          c->logs.back()->alloc(c->slot_log_cap);
          c->scs.emplace_back(new PinBuf<DevScalars>());
          c->scs.back()->alloc(1);
          cudaEvent_t e;
          CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
          c->slot_ev.push_back(e);
        }
      }
      {
        // Device staging of the slots (stream-ordered on the loop's stream);
        // no copy of an earlier run still reads them.
        AllocOn on_stream(s);
        CK(cudaStreamSynchronize(c->copy));
        while ((int)c->snap_sc.size() < inflight) {
          c->snap_pos.emplace_back(new DBuf<float2>());
          c->snap_sc.emplace_back(new DBuf<DevScalars>());
          cudaEvent_t e;
          CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
          c->snap_ev.push_back(e);
        }
        for (int i = 0; i < inflight; ++i) {
          if (!gpu_legal) c->snap_pos[i]->ensure(hp.N);
          c->snap_sc[i]->ensure(1);
        }
      }
      if (!gpu_legal) {
        // Snapshots for the intervals in flight and a few legalisations:
        // pinned allocations here rather than while the loop runs.
        std::vector<HostSnap *> pre;
        for (int i = 0; i < inflight + 2; ++i) pre.push_back(take_snap());
        for (HostSnap *h : pre) give_snap(h);
      }
      for (int i = (int)c->lslots.size() - 1; i >= 0; --i) free_slots.push_back(i);
      // The interval graph is reused while nothing it bakes in has changed:
      // buffers (epoch), interval length, field formula, transform, wl_coeff.
      // A new one is captured, instantiated and uploaded here, so that the
      // thread pumping the loop only launches it.
      use_graph = opts.use_graphs != 0 && interval > 1;
      if (c->gexec && (c->g_epoch != c->buf_epoch || c->g_interval != interval || c->g_field != opts.field_mode ||
                       c->g_tc != tc || c->g_fft != c->fft || c->g_gamma != gamma))
        c->g_valid = false;
      if (use_graph && interval < max_iters) ensure_graph();
      converged_chunk = chunks.size();
      CK(cudaEventRecord(ev0, s));
      phase = kLoop;
    } catch (const CudaError &e) {
      final_st = cuda_fail(c, e);
      return final_st;
    }
    return EPLACE_OK;
  }

  bool slot_available() const { return !free_slots.empty() || (int)c->lslots.size() < kMaxLegalSlots; }
  int acquire_slot() {
    if (free_slots.empty()) {
      new_legal_slot(c);
      return (int)c->lslots.size() - 1;
    }
    const int k = free_slots.back();
    free_slots.pop_back();
    prepare_slot(c, *c->lslots[k]);
    return k;
  }

  // Captures the graph of one interval (`interval` iterations) unless the
  // context holds a current one; on failure (capture not available, e.g.
  // cooperative nodes) the run falls back to plain launches.
  void ensure_graph() {
    if (c->gexec && c->g_valid) return;
    cudaStream_t s = c->stream;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    bool ok = true;
    try {
      for (uint64_t k = 0; k < interval; ++k) launch_iteration(c, gamma, opts.field_mode, tc);
    } catch (const CudaError &) {
      ok = false;
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    ok = ok && ce == cudaSuccess;
    // A stale executable graph of the same shape (same kernels, new
    // pointers and sizes) is updated in place, which is cheaper than a new
    // instantiation.  Only for the bin grid and transform it was made for:
    // those decide which transform kernels run and how they launch (a
    // split-K GEMM is a cluster launch, whose cluster shape an in-place
    // update does not carry), so any other grid gets a new instantiation.
    if (c->gexec && (c->g_bx != c->hp.BX || c->g_by != c->hp.BY || c->g_tc != tc || c->g_fft != c->fft)) {
      cudaGraphExecDestroy(c->gexec);
      c->gexec = nullptr;
    }
    if (ok && c->gexec) {
      cudaGraphExecUpdateResultInfo info{};
      if (cudaGraphExecUpdate(c->gexec, graph, &info) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphExecDestroy(c->gexec);
        c->gexec = nullptr;
      }
    }
    if (ok && !c->gexec && cudaGraphInstantiate(&c->gexec, graph, 0) != cudaSuccess) {
      c->gexec = nullptr;
      ok = false;
    }
    if (!ok) {
      cudaGetLastError();
      if (graph) cudaGraphDestroy(graph);
      if (c->gexec) cudaGraphExecDestroy(c->gexec);
      c->gexec = nullptr;
      c->g_valid = false;
      use_graph = false;
      return;
    }
    cudaGraphDestroy(graph);
    c->g_valid = true;
    CK(cudaGraphUpload(c->gexec, s));
    c->g_epoch = c->buf_epoch;
    c->g_interval = interval;
    c->g_field = opts.field_mode;
    c->g_tc = tc;
    c->g_fft = c->fft;
    c->g_gamma = gamma;
    c->g_bx = c->hp.BX;
    c->g_by = c->hp.BY;
  }

  void launch_chunk(const Chunk &ch) {
    cudaStream_t s = c->stream;
    const uint64_t n = ch.last - ch.first + 1;
    launched_iters += n;
    if (use_graph && n == interval) ensure_graph();
    if (use_graph && n == interval) {
      CK(cudaGraphLaunch(c->gexec, s));
    } else {
      for (uint64_t k = 0; k < n; ++k) launch_iteration(c, gamma, opts.field_mode, tc);
    }
  }

  // A pinned snapshot buffer of at least N positions from the context's
  // free list (allocated when none fits).
  HostSnap *take_snap() {
    const size_t N = c->hp.N;
    auto &fl = c->hsnap_free;
    for (size_t k = 0; k < fl.size(); ++k)
      if (fl[k]->pos && fl[k]->cap >= N) {
        HostSnap *h = fl[k];
        fl.erase(fl.begin() + k);
        return h;
      }
    HostSnap *h;
    if (!fl.empty()) {
      h = fl.back();
      fl.pop_back();
    } else {
      c->hsnaps.emplace_back(new HostSnap());
      h = c->hsnaps.back().get();
    }
    h->reserve(N);
    return h;
  }
  void give_snap(HostSnap *h) {
    if (h) c->hsnap_free.push_back(h);
  }

  void release(Checkpoint *cp) {
    if (!cp) return;
    give_snap(cp->hs);
    cp->hs = nullptr;
    if (cp->slot >= 0) {
      free_slots.push_back(cp->slot);
      cp->slot = -1;
    }
  }

  // Folds finished checkpoints in iteration order; blocking: waits for the
  // next one if it is still being legalised.  Returns whether any was folded.
  bool fold(bool blocking) {
    bool any = false;
    while (fold_next < cps.size() && final_st == EPLACE_OK) {
      Checkpoint *cp = cps[fold_next].get();
      if (cp->chunk >= processed) break;
      if (gpu_legal) {
        if (!cp->discard) {
          LegalSlot &L = *c->lslots[cp->slot];
          if (blocking) {
            CK(cudaEventSynchronize(L.done));
          } else {
            const cudaError_t q = cudaEventQuery(L.done);
            if (q == cudaErrorNotReady) break;
            CK(q);
          }
          const LegalOut &o = *L.hout.p;
          float lms = 0.f;
          if (cudaEventElapsedTime(&lms, L.start, L.done) == cudaSuccess) cp->secs = 1e-3 * lms;
          cp->st = o.status == 0 ? EPLACE_OK : (o.status == 1 ? EPLACE_ERR_NO_BELS : EPLACE_ERR_PLACEMENT_FAILED);
          cp->disp = o.disp;
          cp->hpwl = (int64_t)o.hpwl;
        }
      } else if (!cp->done.load(std::memory_order_acquire)) {
        if (!blocking) break;
        while (!cp->done.load(std::memory_order_acquire)) std::this_thread::sleep_for(std::chrono::microseconds(50));
      }
      ++fold_next;
      any = true;
      if (cp->discard) {
        release(cp);
        continue;
      }
      if (cp->st != EPLACE_OK) {
        final_st = cp->st;
        set_err(c, "logic");
        break;
      }
      const IterLog &L = iterlog[cp->iter];
      if (res->traj && res->traj_len < res->traj_capacity) {
        eplace_traj_entry &t = res->traj[res->traj_len++];
        t.iter = cp->iter;
        t.hpwl = (double)cp->hpwl;
        t.displacement = cp->disp;
        t.step_x = L.step_norm[0];
        t.step_y = L.step_norm[1];
        t.density_penalty = L.lam;
        t.overlap = L.overlap;
      }
      if (opts.verbose) {
        std::fprintf(stderr,
                     "ElectroPlace iter %d: HPWL=%.0f, disp=%.1f, step=(%.4f,%.4f), density_p=%.3f, overlap=%.4f\n",
                     cp->iter, (double)cp->hpwl, cp->disp, L.step_norm[0], L.step_norm[1], L.lam, L.overlap);
      }
      Checkpoint *drop = cp;
      if ((double)cp->hpwl < best_metric) {
        best_metric = (double)cp->hpwl;
        drop = best;
        best = cp;
      }
      release(drop);
    }
    return any;
  }

  // Launches intervals while allowed, reads finished intervals' outputs and
  // folds finished legalisations.  block: wait where the loop has to wait
  // (one interval output per call, as a plain loop would).  Returns whether
  // anything happened.
  bool pump(bool block) {
    if (phase == kDone || phase == kInit) return false;
    bool progressed = false;
    try {
      if (phase == kLoop) progressed |= pump_loop(block);
      if (phase == kLegal) {
        if (final_st == EPLACE_OK) {
          progressed |= fold(false);
          if (block && fold_next < cps.size()) progressed |= fold(true);
        }
        if (final_st != EPLACE_OK || fold_next >= cps.size()) {
          mark("legalisation_done");
          phase = kDone;
          progressed = true;
        }
      }
    } catch (const CudaError &e) {
      final_st = cuda_fail(c, e);
      phase = kDone;
      progressed = true;
    }
    return progressed;
  }

  bool pump_loop(bool block) {
    const HostProblem &hp = c->hp;
    cudaStream_t s = c->stream;
    auto &logs = c->logs;
    auto &scs = c->scs;
    auto &evs = c->slot_ev;
    bool progressed = false;
    while (!stop && next_chunk < chunks.size() && (int)pending.size() < inflight) {
      if (gpu_legal && !slot_available()) {
        if (!pending.empty()) break;  // read the outputs first, then fold
        if (!fold(block) && !block) break;
        if (final_st != EPLACE_OK) {
          stop = true;
          break;
        }
        continue;
      }
      const Chunk &ch = chunks[next_chunk];
      launch_chunk(ch);
      const int slot = slot_rr;
      slot_rr = (slot_rr + 1) % inflight;
      const uint64_t n = ch.last - ch.first + 1;
      HostSnap *hs = nullptr;
      if (gpu_legal) {
        // Snapshot on the device and legalise it on the slot's stream.
        auto cp = std::make_unique<Checkpoint>();
        cp->iter = (int32_t)ch.last;
        cp->chunk = next_chunk;
        cp->slot = acquire_slot();
        LegalSlot &L = *c->lslots[cp->slot];
        CK(cudaStreamWaitEvent(s, L.done, 0));  // a reused slot's last legalisation has finished
        CK(cudaMemcpyAsync(L.pos.p, c->x.p, sizeof(float2) * hp.N, cudaMemcpyDeviceToDevice, s));
        CK(cudaEventRecord(L.snap, s));
        CK(cudaStreamWaitEvent(L.stream, L.snap, 0));
        launch_gpu_legal(c, L);
        cps.push_back(std::move(cp));
      } else {
        hs = take_snap();
        CK(cudaMemcpyAsync(c->snap_pos[slot]->p, c->x.p, sizeof(float2) * hp.N, cudaMemcpyDeviceToDevice, s));
      }
      // The interval's outputs leave on the copy stream: positions and
      // scalars from the slot's device copy (the loop overwrites its own),
      // the log entries from their own places (each iteration has one).
      CK(cudaMemcpyAsync(c->snap_sc[slot]->p, c->sc.p, sizeof(DevScalars), cudaMemcpyDeviceToDevice, s));
      CK(cudaEventRecord(c->snap_ev[slot], s));
      CK(cudaStreamWaitEvent(c->copy, c->snap_ev[slot], 0));
      if (hs) {
        CK(cudaMemcpyAsync(hs->pos, c->snap_pos[slot]->p, sizeof(float2) * hp.N, cudaMemcpyDeviceToHost, c->copy));
        g_d2h += sizeof(float2) * hp.N;
      }
      CK(cudaMemcpyAsync(logs[slot]->p, c->log.p + ch.first, sizeof(IterLog) * n, cudaMemcpyDeviceToHost, c->copy));
      CK(cudaMemcpyAsync(scs[slot]->p, c->snap_sc[slot]->p, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->copy));
      g_d2h += sizeof(IterLog) * n + sizeof(DevScalars);
      CK(cudaEventRecord(evs[slot], c->copy));
      pending.push_back({next_chunk, slot, hs});
      ++next_chunk;
      progressed = true;
    }
    while (!pending.empty()) {
      const size_t ci = pending.front().chunk;
      const int slot = pending.front().slot;
      HostSnap *hs = pending.front().hs;
      if (block) {
        CK(cudaEventSynchronize(evs[slot]));
      } else {
        const cudaError_t q = cudaEventQuery(evs[slot]);
        if (q == cudaErrorNotReady) break;
        CK(q);
      }
      pending.pop_front();
      progressed = true;
      processed = ci + 1;
      if (stop) {  // ran ahead of convergence: discard
        if (gpu_legal) cps[ci]->discard = true;
        give_snap(hs);
        continue;
      }
      const Chunk &ch = chunks[ci];
      if (scs[slot]->p->err) {
        set_err(c, "a bounded device wait timed out");
        final_st = EPLACE_ERR_TIMEOUT;
        stop = true;
        if (gpu_legal) cps[ci]->discard = true;
        give_snap(hs);
        continue;
      }
      const uint64_t n = ch.last - ch.first + 1;
      for (uint64_t k = 0; k < n; ++k) iterlog.push_back(logs[slot]->p[k]);
      iters_done = ch.last + 1;
      const IterLog &L = logs[slot]->p[n - 1];
      last_overlap = L.overlap;
      if (!gpu_legal) {
        // Legalise this checkpoint on the host pool (mod.rs:176-183).
        auto cp = std::make_unique<Checkpoint>();
        cp->iter = (int32_t)ch.last;
        cp->chunk = ci;
        cp->hs = hs;  // the legaliser reads the pinned snapshot in place
        Checkpoint *raw = cp.get();
        cps.push_back(std::move(cp));
        outstanding.fetch_add(1, std::memory_order_acq_rel);
        eplace_ctx *cc = c;
        std::atomic<int> *out = &outstanding;
        const auto ts = t_start;
        pool->submit([raw, cc, out, ts](int tid) {
          const HostProblem &php = cc->hp;
          const auto t0 = std::chrono::steady_clock::now();
          raw->began = std::chrono::duration<double>(t0 - ts).count();
          HostSnap &h = *raw->hs;
          h.sx.resize(php.N);
          h.sy.resize(php.N);
          raw->st = cc->legal[tid]->run(&h.pos[0].x, &h.pos[0].y, 2, h.sx.data(), h.sy.data(), &raw->disp);
          // A lone job's last legalisations finish with cores to spare: the
          // HPWL of a large netlist is summed on four threads there (the job
          // engine's contexts keep one; its cores are busy with other jobs).
          const int hpwl_threads = (!cc->shared_device && php.P >= (1u << 19)) ? 4 : 1;
          if (raw->st == EPLACE_OK) raw->hpwl = hpwl_host(php, h.sx.data(), h.sy.data(), hpwl_threads);
          raw->secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
          raw->done.store(true, std::memory_order_release);
          out->fetch_sub(1, std::memory_order_acq_rel);
        });
      }
      // Convergence (mod.rs:190-195).
      if (ch.last >= 20 && L.overlap < 0.1) {
        stop = true;
        converged_chunk = ci;
      }
      fold(false);
      if (final_st != EPLACE_OK) stop = true;
      if (block) break;
    }
    if (pending.empty() && (stop || next_chunk >= chunks.size())) {
      // The loop is over: everything before ev1 has already completed.
      CK(cudaEventRecord(ev1, s));
      CK(cudaEventSynchronize(ev1));
      mark("device_loop_done");
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ev0, ev1));
      res->gpu_seconds = ms * 1e-3;
      res->gpu_launches = (uint64_t)(kLaunchesPerIter + (c->split_step ? 2 : 0) + (c->fold && !tc && !c->fft ? 2 : 0) -
                                         (final_fused(c, tc) ? 2 : 0)) *
                              launched_iters +
                          (gpu_legal ? 2 * cps.size() : 0) + (uint64_t)ip_launches;
      res->iters = (uint32_t)iters_done;
      res->converged = converged_chunk < chunks.size() ? 1 : 0;
      res->overlap = last_overlap;
      phase = kLegal;
      progressed = true;
    }
    return progressed;
  }

  // Writes the result (final legalisation = the best checkpoint's binding,
  // mod.rs:199) and releases what the run holds.  Call once done() (or after
  // a failed start()).
  eplace_status finish() {
    const HostProblem &hp = c->hp;
    drain();
    if (final_st == EPLACE_OK && hp.N > 0 && phase == kDone) {
      try {
        if (opts.verbose && res->converged)
          std::fprintf(stderr, "ElectroPlace converged at iteration %d (overlap %.4f < 0.1)\n",
                       (int)(iters_done - 1), last_overlap);
        // Legalisation is a pure function of the positions and the fixed
        // cells, so the final binding is the best checkpoint's own.
        std::vector<int32_t> fsx(hp.N), fsy(hp.N);
        std::vector<float> bx(hp.N), by(hp.N);
        if (best && gpu_legal) {
          LegalSlot &L = *c->lslots[best->slot];
          std::vector<int2> sites(hp.N);
          std::vector<float2> pos(hp.N);
          CK(cudaMemcpyAsync(sites.data(), L.sites.p, sizeof(int2) * hp.N, cudaMemcpyDeviceToHost, L.stream));
          CK(cudaMemcpyAsync(pos.data(), L.pos.p, sizeof(float2) * hp.N, cudaMemcpyDeviceToHost, L.stream));
          g_d2h += (sizeof(int2) + sizeof(float2)) * hp.N;
          CK(cudaStreamSynchronize(L.stream));
          for (uint32_t i = 0; i < hp.N; ++i) {
            fsx[i] = sites[i].x;
            fsy[i] = sites[i].y;
            bx[i] = pos[i].x;
            by[i] = pos[i].y;
          }
          res->best_iter = best->iter;
        } else if (best) {
          const HostSnap &h = *best->hs;
          std::copy(h.sx.begin(), h.sx.begin() + hp.N, fsx.begin());
          std::copy(h.sy.begin(), h.sy.begin() + hp.N, fsy.begin());
          for (uint32_t i = 0; i < hp.N; ++i) {
            bx[i] = h.pos[i].x;
            by[i] = h.pos[i].y;
          }
          res->best_iter = best->iter;
        } else {
          if (isx.empty()) {  // the device made the initial placement
            std::vector<int2> site(hp.N);
            CK(cudaMemcpy(site.data(), c->ip_site.p, sizeof(int2) * hp.N, cudaMemcpyDeviceToHost));
            g_d2h += sizeof(int2) * hp.N;
            isx.resize(hp.N);
            isy.resize(hp.N);
            for (uint32_t i = 0; i < hp.N; ++i) {
              isx[i] = site[i].x;
              isy[i] = site[i].y;
            }
          }
          for (uint32_t i = 0; i < hp.N; ++i) {
            bx[i] = (float)isx[i];
            by[i] = (float)isy[i];
          }
          double d = 0.0;
          if (!c->lbase) c->lbase.reset(new LegalBase(hp));
          if (c->legal.empty()) c->legal.emplace_back(new Legalizer(hp, *c->lbase));
          eplace_status ls = c->legal[0]->run(bx.data(), by.data(), fsx.data(), fsy.data(), &d);
          if (ls != EPLACE_OK) {
            final_st = ls;
            set_err(c, "logic");
          }
        }
        if (final_st == EPLACE_OK) {
          for (uint32_t i = 0; i < hp.N; ++i) {
            res->bel_tile[i] = fsy[i] * hp.W + fsx[i];
            if (res->bel_index) res->bel_index[i] = 0;
            if (res->x) res->x[i] = bx[i];
            if (res->y) res->y[i] = by[i];
          }
          res->hpwl = best ? best->hpwl : hpwl_host(hp, fsx.data(), fsy.data());
        }
      } catch (const CudaError &e) {
        final_st = cuda_fail(c, e);
      }
    }
    res->total_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    if (opts.verbose >= 2) {
      std::fprintf(stderr, "eplace_run phases (ms from start):");
      for (auto &m : marks) std::fprintf(stderr, " %s=%.2f", m.first, m.second * 1e3);
      std::fprintf(stderr, " end=%.2f\n", res->total_seconds * 1e3);
      double sum = 0.0, mx = 0.0;
      for (auto &cp : cps) {
        sum += cp->secs;
        mx = std::max(mx, cp->secs);
      }
      std::fprintf(stderr, "eplace_run legalisations: %zu (%s), mean %.2f ms, max %.2f ms, threads %d\n", cps.size(),
                   gpu_legal ? "device" : "host", cps.empty() ? 0.0 : 1e3 * sum / cps.size(), 1e3 * mx,
                   pool ? pool->size() : 0);
      std::fprintf(stderr, "eplace_run checkpoints (iteration: start + length, ms):");
      for (auto &cp : cps) std::fprintf(stderr, " %d:%.1f+%.1f", cp->iter, cp->began * 1e3, cp->secs * 1e3);
      std::fprintf(stderr, "\n");
    }
    res->h2d_bytes = g_h2d - h2d0;
    res->d2h_bytes = g_d2h - d2h0;
    return final_st;
  }

  static constexpr int kMaxLegalSlots = 32;
  eplace_ctx *c;
  eplace_cfg cfg;
  eplace_opts opts;
  eplace_result *res;
  Pool *shared_pool;
  Pool *pool = nullptr;
  Phase phase = kInit;
  std::chrono::steady_clock::time_point t_start;
  uint64_t h2d0 = 0, d2h0 = 0;
  bool tc = false, gpu_legal = false, use_graph = false;
  uint64_t max_iters = 0, interval = 1;
  float gamma = 0.f;
  std::vector<int32_t> isx, isy;
  int ip_launches = 0;  // kernels of the device initial placement
  std::vector<std::pair<const char *, double>> marks;
  std::vector<Chunk> chunks;
  int inflight = 1;
  std::vector<int> free_slots;
  uint64_t launched_iters = 0;
  struct Pending {
    size_t chunk;
    int slot;      // pinned log / scalars slot
    HostSnap *hs;  // the positions, when the host legalises
  };
  std::deque<Pending> pending;
  size_t next_chunk = 0, processed = 0;
  bool stop = false;
  size_t converged_chunk = 0;
  uint64_t iters_done = 0;
  double last_overlap = 0.0;
  std::vector<IterLog> iterlog;
  std::vector<std::unique_ptr<Checkpoint>> cps;
  Checkpoint *best = nullptr;
  double best_metric = INFINITY;
  size_t fold_next = 0;
  int slot_rr = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  eplace_status final_st = EPLACE_OK;
  std::atomic<int> outstanding{0};
};

JobState *job_create(eplace_ctx *c, const eplace_cfg &cfg, const eplace_opts &opts, eplace_result *res,
                     Pool *shared_pool) {
  return new JobState(c, cfg, opts, res, shared_pool);
}
eplace_status job_start(JobState *j) { return j->start(); }
bool job_pump(JobState *j, bool block) { return j->pump(block); }
bool job_done(const JobState *j) { return j->done(); }
eplace_status job_finish(JobState *j) { return j->finish(); }
void job_destroy(JobState *j) { delete j; }
void ctx_set_shared(eplace_ctx *c, bool shared) { c->shared_device = shared; }
uint64_t ctx_device_bytes(const eplace_ctx *c) { return c->device_bytes(); }
int ctx_bins_x(const eplace_ctx *c) { return c->mat_bx; }
int ctx_bins_y(const eplace_ctx *c) { return c->mat_by; }
void set_thread_error(const std::string &m) { set_err(nullptr, m); }
bool problem_tc_supported(const HostProblem &hp) { return tc_supported(hp); }

uint64_t problem_device_bytes(const HostProblem &hp) {
  const uint64_t N = hp.N, F = hp.F, NN = hp.NN, P = hp.P;
  const uint64_t nb = (uint64_t)hp.BX * hp.BY;
  const uint64_t m = (uint64_t)hp.BX * hp.BX + (uint64_t)hp.BY * hp.BY;
  return N * 120 + F * 16 + P * 8 + NN * 16 + nb * 64 + m * 48 + (1u << 20);
}

namespace {
std::mutex g_kept_mu;
std::vector<eplace_ctx *> *g_kept = nullptr;  // never freed: lives until the process exits
constexpr size_t kMaxKept = 4;
}  // namespace

// A kept context of `device`, preferring one whose DCT matrices match the
// bin grid; nullptr if none is kept.
eplace_ctx *take_kept_context(int32_t device, int bx, int by) {
  std::lock_guard<std::mutex> g(g_kept_mu);
  if (!g_kept) return nullptr;
  size_t pick = g_kept->size();
  for (size_t k = 0; k < g_kept->size(); ++k) {
    eplace_ctx *c = (*g_kept)[k];
    if (c->device != device) continue;
    if (pick == g_kept->size()) pick = k;
    if (c->mat_bx == bx && c->mat_by == by) {
      pick = k;
      break;
    }
  }
  if (pick == g_kept->size()) return nullptr;
  eplace_ctx *c = (*g_kept)[pick];
  g_kept->erase(g_kept->begin() + pick);
  return c;
}

void keep_context(eplace_ctx *c) {
  {
    std::lock_guard<std::mutex> g(g_kept_mu);
    if (!g_kept) g_kept = new std::vector<eplace_ctx *>();
    if (g_kept->size() < kMaxKept) {
      g_kept->push_back(c);
      return;
    }
  }
  eplace_ctx_destroy(c);
}

eplace_ctx *ctx_new(int32_t device, eplace_status *st) {
  *st = EPLACE_OK;
  std::unique_ptr<eplace_ctx> c(new eplace_ctx());
  try {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      set_err(nullptr, "no CUDA device");
      *st = EPLACE_ERR_NO_DEVICE;
      return nullptr;
    }
    if (device < 0 || device >= ndev) {
      set_err(nullptr, "device index out of range");
      *st = EPLACE_ERR_INVALID;
      return nullptr;
    }
    c->device = device;
    CK(cudaSetDevice(device));
    int major = 0;
    CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major != 10) {
      set_err(nullptr, "this library is built for sm_100a (B200) only");
      *st = EPLACE_ERR_NO_DEVICE;
      return nullptr;
    }
    // The Nesterov loop's stream gets the highest priority: blocks of its
    // kernels are scheduled ahead of the legaliser's long-running warps.
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    CK(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_hi));
    CK(cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_hi));
    CK(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    c->sc.alloc(1);
    c->bar.alloc(4);
    c->hp_total.alloc(1);
    ensure_log(c.get(), 8);
    CK(cudaStreamSynchronize(c->stream));
  } catch (const CudaError &e) {
    *st = cuda_fail(nullptr, e);
    return nullptr;
  }
  return c.release();
}

eplace_status ctx_load_problem(eplace_ctx *c, HostProblem &&hp) {
  try {
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    for (auto &l : c->lslots)
      if (l && l->stream) CK(cudaStreamSynchronize(l->stream));
    load_into(c, std::move(hp));
    CK(cudaStreamSynchronize(c->stream));
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

}  // namespace eplace

uint64_t eplace_ctx::device_bytes() const {
  uint64_t b = 0;
  auto add = [&b](const auto &buf) { b += (uint64_t)buf.cap * sizeof(*buf.p); };
  add(net_off); add(pin_cell); add(has_driver); add(wa_off); add(wa_slots); add(wa_pins);
  add(half); add(area); add(mflag); add(mac_idx); add(pw); add(look); add(x); add(xp); add(g); add(gprev); add(tmp_wl); add(tmp_den);
  add(acc); add(dens); add(rho); add(T); add(Exh); add(Eyh); add(U); add(V); add(Ex); add(Ey); add(phi);
  add(mB1); add(mL2); add(mB3); add(mL4); add(mB5); add(mL6); add(mB3g); add(mL6g);
  add(wx); add(gx2); add(wy); add(gy2); add(ops); add(mom); add(part); add(part2); add(part_b);
  add(sc); add(log); add(bar); add(loc); add(hp_total);
  for (const auto &d : snap_pos) add(*d);
  for (const auto &d : snap_sc) add(*d);
  add(rho_h); add(rho_l); add(Tt_h); add(Tt_l); add(Exh_h); add(Exh_l); add(Eyh_h); add(Eyh_l);
  add(Ut_h); add(Ut_l); add(Vt_h); add(Vt_l); add(B1t_h); add(B1t_l); add(L2_h); add(L2_l);
  add(B3t_h); add(B3t_l); add(B5t_h); add(B5t_l); add(L4_h); add(L4_l); add(L6_h); add(L6_l);
  add(B3gt_h); add(B3gt_l); add(L6g_h); add(L6g_l); add(lg_order); add(lg_fsize); add(lg_free0);
  for (const auto &l : lslots) {
    add(l->pos); add(l->sites); add(l->loc); add(l->cost); add(l->out); add(l->fm); add(l->list); add(l->len); add(l->info);
    add(l->hmark); add(l->dmark); add(l->pick); add(l->dist); add(l->fresh); add(l->lst);
  }
  return b;
}

extern "C" {

eplace_status eplace_run(eplace_ctx *c, const eplace_cfg *cfg, const eplace_opts *opts_in,
                         eplace_result *res) {
  if (!c || !cfg || !res) return EPLACE_ERR_INVALID;
  eplace_opts opts;
  eplace_opts_default(&opts);
  if (opts_in) opts = *opts_in;
  JobState j(c, *cfg, opts, res, nullptr);
  eplace_status st = job_start(&j);
  if (st != EPLACE_OK) return st;
  while (!j.done()) j.pump(true);
  return j.finish();
}

eplace_status eplace_place(const eplace_netlist *nl, const eplace_chip *chip, const eplace_cfg *cfg,
                           const eplace_opts *opts, int32_t device, eplace_result *res) {
  const uint64_t h2d0 = g_h2d, d2h0 = g_d2h;
  const auto t0 = std::chrono::steady_clock::now();
  // The one-shot call keeps its context between calls (one per device and
  // concurrent caller): the next call re-loads it with its own netlist
  // (eplace_ctx_load semantics), so a stream of one-shot placements
  // allocates, builds DCT matrices and frees only when a design outgrows
  // the kept buffers or the bin grid changes.  Kept contexts live until the
  // process exits.
  std::string msg;
  HostProblem hp;
  eplace_status st = load_problem(nl, chip, hp, msg);
  if (st != EPLACE_OK) {
    set_err(nullptr, msg);
    return st;
  }
  eplace_ctx *c = take_kept_context(device, hp.BX, hp.BY);
  if (!c) {
    c = ctx_new(device, &st);
    if (!c) return st;
  }
  st = ctx_load_problem(c, std::move(hp));
  if (st != EPLACE_OK) {
    g_thread_error = c->err;
    eplace_ctx_destroy(c);
    return st;
  }
  const auto t1 = std::chrono::steady_clock::now();
  st = eplace_run(c, cfg, opts, res);
  if (st != EPLACE_OK) g_thread_error = c->err;
  const auto t2 = std::chrono::steady_clock::now();
  keep_context(c);
  if (opts && opts->verbose >= 2) {
    auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
      return std::chrono::duration<double>(b - a).count() * 1e3;
    };
    std::fprintf(stderr, "eplace_place: load %.2f ms, run %.2f ms\n", ms(t0, t1), ms(t1, t2));
  }
  if (res) {
    res->h2d_bytes = g_h2d - h2d0;
    res->d2h_bytes = g_d2h - d2h0;
    res->total_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return st;
}

eplace_status eplace_profile_stages(eplace_ctx *c, const eplace_cfg *cfg, const eplace_opts *opts_in,
                                    uint32_t reps, double *stage_ms) {
  if (!c || !cfg || !stage_ms || reps == 0) return EPLACE_ERR_INVALID;
  eplace_opts opts;
  eplace_opts_default(&opts);
  if (opts_in) opts = *opts_in;
  eplace_status mst = check_modes(c, opts);
  if (mst != EPLACE_OK) return mst;
  const bool tc = opts.dct_mode == EPLACE_DCT_BF16X3_TC;
  const HostProblem &hp = c->hp;
  if (hp.N == 0) return EPLACE_ERR_INVALID;
  c->fft = opts.dct_mode == EPLACE_DCT_FP32_FFT && fft_supported(hp.BX, hp.BY);
  std::vector<cudaEvent_t> ev(9, nullptr);
  eplace_status st = EPLACE_OK;
  try {
    CK(cudaSetDevice(c->device));
    std::string msg;
    std::vector<int32_t> isx, isy;
    st = initial_placement(hp, cfg->seed, isx, isy, msg);
    if (st != EPLACE_OK) {
      set_err(c, msg);
      return st;
    }
    ensure_log(c, reps);
    upload_momentum(c, reps);
    if (tc) setup_tc(c);
    reset_state(c, isx, isy, cfg);
    autotune_launches(c, (float)cfg->wl_coeff, opts.field_mode, tc);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    const float gamma = (float)cfg->wl_coeff;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    cudaStream_t s = c->stream;
    bool capturing = false;
    // Inside a capture the records become event-record nodes of the graph
    // (cudaEventRecordExternal), which the host can wait on and time.
    auto rec = [&](cudaEvent_t e) {
      CK(capturing ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s));
    };
    auto one_iteration = [&]() {
      rec(ev[0]);
      launch_wa_stage(c, gamma);
      rec(ev[1]);
      launch_scatter_stage(c);
      rec(ev[2]);
      const bool fuse = final_fused(c, tc);  // then the finalise is timed with the first transform stage
      if (!fuse) launch_final_stage(c, nullptr, tc);
      rec(ev[3]);
      for (int g = 0; g < 4; ++g) {
        launch_field_gemm(c, g, nullptr, opts.field_mode, tc, fuse && g == 0);
        rec(ev[4 + g]);
      }
      launch_step_stage(c);
      rec(ev[8]);
    };
    // The iteration is timed as a CUDA graph (event-record nodes between the
    // kernel nodes), as the loop replays it, so host launch latency is not
    // counted; plain launches if capture is not available.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      bool ok = true;
      capturing = true;
      try {
        one_iteration();
      } catch (const CudaError &) {
        ok = false;
      }
      capturing = false;
      if (cudaStreamEndCapture(s, &graph) != cudaSuccess || !ok ||
          cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess) {
        cudaGetLastError();
        gexec = nullptr;
      }
      if (graph) cudaGraphDestroy(graph);
    } else {
      cudaGetLastError();
    }
    for (uint32_t r = 0; r < reps; ++r) {
      if (gexec) {
        const cudaError_t le = cudaGraphLaunch(gexec, s);
        if (le != cudaSuccess) {
          cudaGraphExecDestroy(gexec);
          throw CudaError{le, "cudaGraphLaunch (profile)"};
        }
      } else {
        one_iteration();
      }
      CK(cudaEventSynchronize(ev[8]));
      for (int k = 0; k < 8; ++k) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
        acc[k] += ms;
      }
    }
    if (gexec) cudaGraphExecDestroy(gexec);
    for (int k = 0; k < 8; ++k) stage_ms[k] = acc[k] / reps;
  } catch (const CudaError &e) {
    st = cuda_fail(c, e);
  }
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  return st;
}

// ---------------------------------------------------------------------------
// Stage entry points (host buffers in/out, one kernel family each).
// ---------------------------------------------------------------------------
static void upload_look(eplace_ctx *c, const float *x, const float *y) {
  AllocOn on_stream(c->stream);
  std::vector<float2> p(c->hp.N);
  for (uint32_t i = 0; i < c->hp.N; ++i) p[i] = make_float2(x[i], y[i]);
  if (c->hp.N) CK(cudaMemcpyAsync(c->look.p, p.data(), sizeof(float2) * c->hp.N, cudaMemcpyHostToDevice, c->stream));
}

eplace_status eplace_stage_wa_grad(eplace_ctx *c, double wl_coeff, const float *x, const float *y, float *gx,
                                   float *gy) {
  if (!c || (c->hp.N && (!x || !y || !gx || !gy))) return EPLACE_ERR_INVALID;
  try {
    CK(cudaSetDevice(c->device));
    upload_look(c, x, y);
    c->acc.zero(c->stream);
    launch_wa_stage(c, (float)wl_coeff);
    std::vector<unsigned long long> acc((size_t)c->hp.N);
    if (c->hp.N)
      CK(cudaMemcpyAsync(acc.data(), c->acc.p, sizeof(unsigned long long) * acc.size(), cudaMemcpyDeviceToHost,
                         c->stream));
    c->acc.zero(c->stream);
    CK(cudaStreamSynchronize(c->stream));
    const double inv = std::ldexp(1.0, -c->grad_k);
    for (uint32_t i = 0; i < c->hp.N; ++i) {
      long long sx, sy;
      unpack_grad(acc[i], &sx, &sy);
      gx[i] = (float)((double)sx * inv);
      gy[i] = (float)((double)sy * inv);
    }
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

eplace_status eplace_stage_density(eplace_ctx *c, const float *x, const float *y, double *density,
                                   double *overlap) {
  if (!c || !density || (c->hp.N && (!x || !y))) return EPLACE_ERR_INVALID;
  try {
    CK(cudaSetDevice(c->device));
    const size_t nb = (size_t)c->hp.BX * c->hp.BY;
    DBuf<double> dout;
    dout.alloc(nb);
    DevScalars sc{};
    c->sc.upload(&sc, 1, c->stream);
    upload_look(c, x, y);
    c->dens.zero(c->stream);
    launch_scatter_stage(c);
    launch_final_stage(c, dout.p);
    CK(cudaMemcpyAsync(density, dout.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&sc, c->sc.p, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (overlap) *overlap = sc.overlap;
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

eplace_status eplace_stage_field(eplace_ctx *c, const double *density, int32_t dct_mode, int32_t field_mode,
                                 float *ex, float *ey,
                                 float *phi_hat) {
  if (!c || !density || !ex || !ey) return EPLACE_ERR_INVALID;
  eplace_opts o;
  eplace_opts_default(&o);
  o.dct_mode = dct_mode;
  o.field_mode = field_mode;
  eplace_status mst = check_modes(c, o);
  if (mst != EPLACE_OK) return mst;
  const bool tc = dct_mode == EPLACE_DCT_BF16X3_TC;
  c->fft = dct_mode == EPLACE_DCT_FP32_FFT && fft_supported(c->hp.BX, c->hp.BY);
  try {
    CK(cudaSetDevice(c->device));
    const size_t nb = (size_t)c->hp.BX * c->hp.BY;
    const double c0 = c->total_area / (double)nb;
    std::vector<float> rho(nb);
    for (size_t i = 0; i < nb; ++i) rho[i] = (float)(density[i] - c0);
    if (tc) {
      setup_tc(c);
      std::vector<__nv_bfloat16> h(nb), l(nb);
      for (size_t i = 0; i < nb; ++i) {
        h[i] = __float2bfloat16_rn(rho[i]);
        l[i] = __float2bfloat16_rn(rho[i] - __bfloat162float(h[i]));
      }
      c->rho_h.upload(h.data(), nb, c->stream);
      c->rho_l.upload(l.data(), nb, c->stream);
      DevScalars sc{};
      c->sc.upload(&sc, 1, c->stream);
    } else {
      c->rho.upload(rho.data(), nb, c->stream);
    }
    DBuf<float> phi;
    if (phi_hat) phi.alloc(nb);
    launch_field_stage(c, phi_hat ? phi.p : nullptr, field_mode, tc);
    CK(cudaMemcpyAsync(ex, c->Ex.p, sizeof(float) * nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(ey, c->Ey.p, sizeof(float) * nb, cudaMemcpyDeviceToHost, c->stream));
    if (phi_hat) CK(cudaMemcpyAsync(phi_hat, phi.p, sizeof(float) * nb, cudaMemcpyDeviceToHost, c->stream));
    DevScalars sc{};
    CK(cudaMemcpyAsync(&sc, c->sc.p, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (tc && sc.err) {
      set_err(c, "a bounded device wait timed out in the tensor-core transform");
      return EPLACE_ERR_TIMEOUT;
    }
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

eplace_status eplace_stage_gather(eplace_ctx *c, const float *x, const float *y, const float *ex, const float *ey,
                                  float *gx, float *gy) {
  // The gather is fused into the step kernel; mode 1 of that kernel stops
  // after the gather and leaves the density gradient in its scratch buffer.
  if (!c || !ex || !ey || (c->hp.N && (!x || !y || !gx || !gy))) return EPLACE_ERR_INVALID;
  try {
    CK(cudaSetDevice(c->device));
    const HostProblem &hp = c->hp;
    const size_t nb = (size_t)hp.BX * hp.BY;
    upload_look(c, x, y);
    c->Ex.upload(ex, nb, c->stream);
    c->Ey.upload(ey, nb, c->stream);
    StepArgs a = step_args(c);
    a.mode = 1;
    CK(launch_step(a, c->step_grid, c->stream));
    std::vector<float2> t(hp.N);
    if (hp.N) CK(cudaMemcpyAsync(t.data(), c->tmp_den.p, sizeof(float2) * hp.N, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (uint32_t i = 0; i < hp.N; ++i) {
      gx[i] = t[i].x;
      gy[i] = t[i].y;
    }
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

static std::vector<float2> pack2(const float *a, const float *b, size_t n) {
  std::vector<float2> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = make_float2(a[i], b[i]);
  return v;
}

static void unpack2(const std::vector<float2> &v, float *a, float *b) {
  for (size_t i = 0; i < v.size(); ++i) {
    a[i] = v[i].x;
    b[i] = v[i].y;
  }
}

eplace_status eplace_stage_step(eplace_ctx *c, uint64_t iter, const float *look_x, const float *look_y,
                                const float *gwl_x, const float *gwl_y, const float *ex, const float *ey,
                                float *x, float *y, float *x_prev, float *y_prev, float *gprev_x,
                                float *gprev_y, double *scal, double *out, float *next_look_x,
                                float *next_look_y) {
  const uint32_t N = c ? c->hp.N : 0;
  if (!c || !ex || !ey || !scal || !out) return EPLACE_ERR_INVALID;
  if (N && (!look_x || !look_y || !gwl_x || !gwl_y || !x || !y || !x_prev || !y_prev || !gprev_x || !gprev_y ||
            !next_look_x || !next_look_y))
    return EPLACE_ERR_INVALID;
  try {
    CK(cudaSetDevice(c->device));
    const HostProblem &hp = c->hp;
    const size_t nb = (size_t)hp.BX * hp.BY;
    cudaStream_t s = c->stream;
    ensure_log(c, iter + 2);
    upload_momentum(c, iter + 2);
    upload_look(c, look_x, look_y);
    c->Ex.upload(ex, nb, s);
    c->Ey.upload(ey, nb, s);
    std::vector<unsigned long long> acc((size_t)N);
    const double scale = std::ldexp(1.0, c->grad_k);
    for (uint32_t i = 0; i < N; ++i)
      acc[i] = pack_grad(llrint((double)gwl_x[i] * scale), llrint((double)gwl_y[i] * scale));
    if (N)
      CK(cudaMemcpyAsync(c->acc.p, acc.data(), sizeof(unsigned long long) * acc.size(), cudaMemcpyHostToDevice, s));
    std::vector<float2> vx = pack2(x, y, N), vxp = pack2(x_prev, y_prev, N), vg = pack2(gprev_x, gprev_y, N);
    c->x.upload(vx.data(), N, s);
    c->xp.upload(vxp.data(), N, s);
    c->gprev.upload(vg.data(), N, s);
    DevScalars sc{};
    sc.lam = scal[0];
    sc.lam_init = scal[1] != 0.0;
    sc.step[0] = scal[2];
    sc.step[1] = scal[3];
    sc.iter = (int32_t)iter;
    c->sc.upload(&sc, 1, s);
    c->bar.zero(s);
    launch_step_stage(c);
    std::vector<float2> lk(N);
    if (N) {
      CK(cudaMemcpyAsync(vx.data(), c->x.p, sizeof(float2) * N, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(vxp.data(), c->xp.p, sizeof(float2) * N, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(vg.data(), c->gprev.p, sizeof(float2) * N, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(lk.data(), c->look.p, sizeof(float2) * N, cudaMemcpyDeviceToHost, s));
    }
    IterLog L{};
    CK(cudaMemcpyAsync(&L, c->log.p + iter, sizeof(L), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&sc, c->sc.p, sizeof(sc), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (sc.err) {
      set_err(c, "a bounded device wait timed out");
      return EPLACE_ERR_TIMEOUT;
    }
    unpack2(vx, x, y);
    unpack2(vxp, x_prev, y_prev);
    unpack2(vg, gprev_x, gprev_y);
    unpack2(lk, next_look_x, next_look_y);
    scal[0] = sc.lam;
    scal[1] = sc.lam_init;
    scal[2] = sc.step[0];
    scal[3] = sc.step[1];
    out[0] = L.step_norm[0];
    out[1] = L.step_norm[1];
    out[2] = L.alpha[0];
    out[3] = L.alpha[1];
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

eplace_status eplace_stage_barrier_timeout(eplace_ctx *c, int32_t wait_limit_us, uint32_t phantom) {
  if (!c || wait_limit_us <= 0 || phantom == 0) return EPLACE_ERR_INVALID;
  const HostProblem &hp = c->hp;
  if (hp.N == 0) return EPLACE_ERR_INVALID;
  try {
    CK(cudaSetDevice(c->device));
    if (phantom >= (uint32_t)c->step_grid) {
      set_err(c, "phantom arrivals must be below the step's grid size");
      return EPLACE_ERR_INVALID;
    }
    eplace_cfg cfg;
    eplace_cfg_default(&cfg);
    std::vector<int32_t> isx, isy;
    std::string msg;
    const eplace_status st = initial_placement(hp, cfg.seed, isx, isy, msg);
    if (st != EPLACE_OK) {
      set_err(c, msg);
      return st;
    }
    ensure_log(c, 2);
    upload_momentum(c, 2);
    const int64_t saved = c->spin_cycles;
    c->spin_cycles = wait_cycles(c->device, wait_limit_us);
    reset_state(c, isx, isy, &cfg);
    c->spin_cycles = saved;
    // the arrival count starts `phantom` ahead: the block whose ticket lands
    // in the next multiple of the grid waits for arrivals that never come
    const unsigned long long start = phantom;
    CK(cudaMemcpyAsync(c->bar.p, &start, sizeof(start), cudaMemcpyHostToDevice, c->stream));
    CK(launch_step(step_args(c), c->step_grid, c->stream));
    DevScalars sc{};
    CK(cudaMemcpyAsync(&sc, c->sc.p, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (sc.err) {
      set_err(c, "a bounded device wait timed out");
      return EPLACE_ERR_TIMEOUT;
    }
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

eplace_status eplace_stage_initial_placement(eplace_ctx *c, uint64_t seed, int32_t *sx, int32_t *sy,
                                             int32_t *on_device) {
  if (!c || (c->hp.N && (!sx || !sy))) return EPLACE_ERR_INVALID;
  try {
    CK(cudaSetDevice(c->device));
    const HostProblem &hp = c->hp;
    eplace_status st;
    std::string msg;
    const bool dev = ip_device_prepare(c, st, msg);
    if (on_device) *on_device = dev ? 1 : 0;
    if (!dev) {
      std::vector<int32_t> hx, hy;
      st = initial_placement(hp, seed, hx, hy, msg);
      if (st == EPLACE_OK) {
        std::copy(hx.begin(), hx.end(), sx);
        std::copy(hy.begin(), hy.end(), sy);
      }
    } else if (st == EPLACE_OK && hp.N) {
      ip_device_launch(c, seed);
      std::vector<int2> site(hp.N);
      CK(cudaMemcpyAsync(site.data(), c->ip_site.p, sizeof(int2) * hp.N, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      for (uint32_t i = 0; i < hp.N; ++i) {
        sx[i] = site[i].x;
        sy[i] = site[i].y;
      }
    }
    if (st != EPLACE_OK) set_err(c, msg);
    return st;
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
}

eplace_status eplace_stage_hpwl(eplace_ctx *c, const int32_t *sx, const int32_t *sy, int64_t *hpwl) {
  if (!c || !hpwl || (c->hp.N && (!sx || !sy))) return EPLACE_ERR_INVALID;
  try {
    CK(cudaSetDevice(c->device));
    const HostProblem &hp = c->hp;
    std::vector<int2> l(hp.N);
    for (uint32_t i = 0; i < hp.N; ++i) {
      if (sx[i] < 0 || sx[i] >= hp.W || sy[i] < 0 || sy[i] >= hp.H) {
        set_err(c, "site out of range");
        return EPLACE_ERR_INVALID;
      }
      l[i] = make_int2(sx[i] + (hp.cw[i] - 1) / 2, sy[i] + (hp.ch[i] - 1) / 2);
    }
    if (hp.N) CK(cudaMemcpyAsync(c->loc.p, l.data(), sizeof(int2) * hp.N, cudaMemcpyHostToDevice, c->stream));
    c->hp_total.zero(c->stream);
    HpwlArgs a{c->net_off.p, c->pin_cell.p, c->has_driver.p, c->loc.p, hp.NN, c->hp_total.p};
    if (hp.NN) CK(launch_hpwl(a, grid_for((int)hp.NN, kHpwlBlock, c->num_sms * 8), c->stream));
    unsigned long long t = 0;
    CK(cudaMemcpyAsync(&t, c->hp_total.p, sizeof(t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *hpwl = (int64_t)t;
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

eplace_status eplace_legalize(eplace_ctx *c, const float *x, const float *y, int32_t *sx, int32_t *sy,
                              double *disp) {
  if (!c || (c->hp.N && (!x || !y || !sx || !sy))) return EPLACE_ERR_INVALID;
  if (!c->lbase) c->lbase.reset(new LegalBase(c->hp));
  Legalizer L(c->hp, *c->lbase);
  eplace_status st = L.run(x, y, sx, sy, disp);
  if (st != EPLACE_OK) set_err(c, "logic");
  return st;
}

eplace_status eplace_stage_legalize(eplace_ctx *c, const float *x, const float *y, int32_t *sx, int32_t *sy,
                                    double *disp, int64_t *hpwl) {
  if (!c || (c->hp.N && (!x || !y || !sx || !sy))) return EPLACE_ERR_INVALID;
  const HostProblem &hp = c->hp;
  if (!legalize_supported(hp.W, hp.H)) {
    set_err(c, "the device legaliser supports chips up to 4096 x 4096 sites");
    return EPLACE_ERR_INVALID;
  }
  try {
    CK(cudaSetDevice(c->device));
    if (hp.N == 0) {
      if (disp) *disp = 0.0;
      if (hpwl) *hpwl = hpwl_host(hp, nullptr, nullptr);
      return EPLACE_OK;
    }
    setup_gpu_legal(c);
    LegalSlot *L = c->lslots.empty() ? new_legal_slot(c) : c->lslots[0].get();
    prepare_slot(c, *L);
    std::vector<float2> p = pack2(x, y, hp.N);
    CK(cudaMemcpyAsync(L->pos.p, p.data(), sizeof(float2) * hp.N, cudaMemcpyHostToDevice, L->stream));
    g_h2d += sizeof(float2) * hp.N;
    launch_gpu_legal(c, *L);
    std::vector<int2> s(hp.N);
    CK(cudaMemcpyAsync(s.data(), L->sites.p, sizeof(int2) * hp.N, cudaMemcpyDeviceToHost, L->stream));
    g_d2h += sizeof(int2) * hp.N;
    CK(cudaStreamSynchronize(L->stream));
    const LegalOut &o = *L->hout.p;
    if (o.status != 0) {
      set_err(c, o.status == 1 ? "logic" : "device legaliser stopped at an internal limit");
      return o.status == 1 ? EPLACE_ERR_NO_BELS : EPLACE_ERR_PLACEMENT_FAILED;
    }
    for (uint32_t i = 0; i < hp.N; ++i) {
      sx[i] = s[i].x;
      sy[i] = s[i].y;
    }
    if (disp) *disp = o.disp;
    if (hpwl) *hpwl = (int64_t)o.hpwl;
  } catch (const CudaError &e) {
    return cuda_fail(c, e);
  }
  return EPLACE_OK;
}

eplace_status eplace_legalize_host(const eplace_netlist *nl, const eplace_chip *chip, const float *x, const float *y,
                                   int32_t *sx, int32_t *sy, double *disp) {
  HostProblem hp;
  std::string msg;
  eplace_status st = load_problem(nl, chip, hp, msg);
  if (st != EPLACE_OK) {
    set_err(nullptr, msg);
    return st;
  }
  if (hp.N && (!x || !y || !sx || !sy)) return EPLACE_ERR_INVALID;
  LegalBase base(hp);
  Legalizer L(hp, base);
  st = L.run(x, y, sx, sy, disp);
  if (st != EPLACE_OK) set_err(nullptr, "logic");
  return st;
}

eplace_status eplace_hpwl_host(const eplace_netlist *nl, const eplace_chip *chip, const int32_t *sx,
                               const int32_t *sy, int64_t *hpwl) {
  HostProblem hp;
  std::string msg;
  eplace_status st = load_problem(nl, chip, hp, msg);
  if (st != EPLACE_OK) {
    set_err(nullptr, msg);
    return st;
  }
  if (!hpwl || (hp.N && (!sx || !sy))) return EPLACE_ERR_INVALID;
  build_hpwl_table(hp);
  *hpwl = hpwl_host(hp, sx, sy, hp.P >= (1u << 19) ? 4 : 1);  // as a lone job's checkpoints
  return EPLACE_OK;
}

eplace_status eplace_pin_weights(const eplace_netlist *nl, const eplace_chip *chip, double *weights) {
  HostProblem hp;
  std::string msg;
  eplace_status st = load_problem(nl, chip, hp, msg);
  if (st != EPLACE_OK) {
    set_err(nullptr, msg);
    return st;
  }
  if (hp.N && !weights) return EPLACE_ERR_INVALID;
  std::vector<double> w;
  pin_weights(hp, w);
  std::copy(w.begin(), w.end(), weights);
  return EPLACE_OK;
}

eplace_status eplace_initial_placement_host(const eplace_netlist *nl, const eplace_chip *chip, uint64_t seed,
                                            int32_t *sx, int32_t *sy) {
  HostProblem hp;
  std::string msg;
  eplace_status st = load_problem(nl, chip, hp, msg);
  if (st != EPLACE_OK) {
    set_err(nullptr, msg);
    return st;
  }
  std::vector<int32_t> vx, vy;
  st = initial_placement(hp, seed, vx, vy, msg);
  if (st != EPLACE_OK) {
    set_err(nullptr, msg);
    return st;
  }
  if (hp.N && (!sx || !sy)) return EPLACE_ERR_INVALID;
  std::copy(vx.begin(), vx.end(), sx);
  std::copy(vy.begin(), vy.end(), sy);
  return EPLACE_OK;
}

eplace_status eplace_synth_size(const eplace_synth_spec *spec, eplace_synth_info *info) {
  if (!spec || !info) return EPLACE_ERR_INVALID;
  return synth(*spec, info, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
}

eplace_status eplace_synth_fill(const eplace_synth_spec *spec, uint8_t *cw, uint8_t *ch, int32_t *fx, int32_t *fy,
                                uint32_t *net_off, uint32_t *pin_cell) {
  if (!spec || !net_off || (spec->num_pads && (!fx || !fy))) return EPLACE_ERR_INVALID;
  eplace_synth_info info{};
  return synth(*spec, &info, cw, ch, fx, fy, net_off, pin_cell);
}

}  // extern "C"
