// eplace_internal.h -- declarations shared by the host C++ and CUDA sources
// of libeplace.so.  Nothing here crosses the C ABI.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <sys/resource.h>
#include <sys/syscall.h>
#include <unistd.h>

#include "../../include/eplace.h"

namespace eplace {

// Fixed-point scale of the deterministic accumulators (WA gradient, density
// map): value = int64 / 2^32.  Integer addition is associative, so the sum
// is independent of the order in which atomics land.
constexpr double kFixScale = 4294967296.0;
constexpr double kFixInv = 1.0 / 4294967296.0;

// Host copy of a validated problem.
struct HostProblem {
  int32_t W = 0, H = 0, BX = 0, BY = 0;
  int32_t sx = 1, sy = 1;  // sites per bin along x / y
  uint32_t N = 0, F = 0, NN = 0, P = 0;
  std::vector<uint8_t> cw, ch;          // footprint (sites)
  std::vector<int32_t> init_x, init_y;  // -1 = unbound
  std::vector<int32_t> fx, fy;
  std::vector<uint8_t> f_logic;
  std::vector<uint32_t> net_off, pin_cell;
  std::vector<uint8_t> has_driver;
  bool any_macro = false;
  uint32_t max_degree = 0;
  // The nets that count toward the HPWL (a driver and two pins or more),
  // grouped by degree: their pins back to back in hpwl_pins, and one
  // (degree, nets) pair per group in hpwl_runs.  Until build_hpwl_table
  // sets hpwl_table, hpwl_host walks the plain CSR.
  std::vector<uint32_t> hpwl_pins;
  std::vector<std::pair<uint32_t, uint32_t>> hpwl_runs;
  bool hpwl_table = false;
};

// Validates the C structs and copies them.  Returns EPLACE_OK or
// EPLACE_ERR_INVALID with msg set.
eplace_status load_problem(const eplace_netlist *nl, const eplace_chip *chip, HostProblem &hp,
                           std::string &msg);

// initial_placement (placer/common.rs:27-117) with the reference RNG.
eplace_status initial_placement(const HostProblem &hp, uint64_t seed, std::vector<int32_t> &sx,
                                std::vector<int32_t> &sy, std::string &msg);

// compute_pin_weights (placer/common.rs:381-407).
void pin_weights(const HostProblem &hp, std::vector<double> &w);

// Immutable part of the greedy legaliser, built once per problem: the free
// map of logic sites with only the fixed cells bound, and the cell order
// (macros first, then unit cells, each in solver order).
struct LegalBase {
  explicit LegalBase(const HostProblem &hp);
  int32_t W = 0, H = 0, WR = 0;       // WR: 64-bit words per row
  std::vector<uint64_t> free0;        // per-row bitmaps, bit set = free
  std::vector<uint64_t> sum0;         // per row (WR <= 64): bit w set = word w has a free site
  std::vector<uint32_t> order;
};

// Greedy legaliser (electro_place/mod.rs:206-255) with the reference's
// choice and tie-break.  One instance per thread (owns its working map).
struct Legalizer {
  Legalizer(const HostProblem &hp, const LegalBase &base);
  // Returns EPLACE_OK or EPLACE_ERR_NO_BELS.  Cell i's target is
  // (x[i * stride], y[i * stride]): stride 2 reads interleaved (x, y) pairs.
  eplace_status run(const float *x, const float *y, size_t stride, int32_t *site_x, int32_t *site_y,
                    double *displacement);
  eplace_status run(const float *x, const float *y, int32_t *site_x, int32_t *site_y, double *displacement) {
    return run(x, y, 1, site_x, site_y, displacement);
  }

 private:
  const HostProblem &hp_;
  const LegalBase &base_;
  std::vector<uint64_t> free_, sum_;
  std::vector<int32_t> lc_, rc_;  // per-row candidate cache of the unit-cell search
  bool simd_ = false;             // AVX2 available: the search takes four rows per step
  bool simd512_ = false;          // AVX-512F available: eight rows per step
};

// total_hpwl (metrics/wirelength.rs:10-51) on the host; with threads > 1 the
// degree-grouped table is summed in that many pieces at once.
int64_t hpwl_host(const HostProblem &hp, const int32_t *site_x, const int32_t *site_y, int threads = 1);
// Fills hp.hpwl_pins / hp.hpwl_runs (counting sort by degree, O(pins)).
void build_hpwl_table(HostProblem &hp);

// Synthetic generator (no reference counterpart).
eplace_status synth(const eplace_synth_spec &spec, eplace_synth_info *info, uint8_t *cw,
                    uint8_t *ch, int32_t *fx, int32_t *fy, uint32_t *net_off,
                    uint32_t *pin_cell);

// FIFO worker pool of the host legaliser; one pool may serve many placement
// jobs (the job engine shares one across its contexts).  With nice > 0 the
// workers run below the priority of the threads that feed the device (the
// job engine's scheduler and loaders), which then never wait behind a full
// set of legalisations for a core.
class Pool {
 public:
  explicit Pool(int n, int nice = 0) {
    for (int i = 0; i < n; ++i)
      th_.emplace_back([this, i, nice] {
        if (nice > 0) setpriority(PRIO_PROCESS, (id_t)syscall(SYS_gettid), nice);  // this thread only (Linux)
        loop(i);
      });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }
  void submit(std::function<void(int)> f) {
    {
      std::lock_guard<std::mutex> g(m_);
      q_.push_back(std::move(f));
    }
    cv_.notify_one();
  }
  int size() const { return (int)th_.size(); }
  // Blocks until the queue is empty and no job is running.
  void wait_idle() {
    std::unique_lock<std::mutex> g(m_);
    idle_cv_.wait(g, [this] { return q_.empty() && active_ == 0; });
  }

 private:
  void loop(int id) {
    for (;;) {
      std::function<void(int)> f;
      {
        std::unique_lock<std::mutex> g(m_);
        cv_.wait(g, [this] { return stop_ || !q_.empty(); });
        if (stop_ && q_.empty()) return;
        f = std::move(q_.front());
        q_.pop_front();
        ++active_;
      }
      f(id);
      {
        std::lock_guard<std::mutex> g(m_);
        --active_;
      }
      idle_cv_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::deque<std::function<void(int)>> q_;
  std::mutex m_;
  std::condition_variable cv_, idle_cv_;
  int active_ = 0;
  bool stop_ = false;
};


}  // namespace eplace
