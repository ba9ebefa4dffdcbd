/*
 * eplace.h -- C ABI of the B200 (sm_100a) ElectroPlace hot path.
 *
 * This is the drop-in boundary for the reference placer entry point
 *   pub fn place_electro(ctx: &mut Context, cfg: &ElectroPlaceCfg)
 *       -> Result<(), PlacerError>
 * (crates/nextpnr/src/placer/electro_place/mod.rs:65) and for
 *   impl Placer for PlacerElectro { place, place_cells }
 * (crates/nextpnr/src/placer/electro_place/mod.rs:45-63, trait at
 * crates/nextpnr/src/placer/mod.rs:31-52).
 *
 * The caller flattens its netlist into CSR arrays (movable cells in solver
 * order, i.e. the order of collect_movable_cells, placer/common.rs:155-174),
 * creates a context (device upload), runs, and writes the returned BEL
 * bindings back.  Plain pointers and sizes only; no library types cross the
 * boundary.  All functions return an eplace_status; none aborts or traps.
 * Threading: one context is used by one host thread at a time; distinct
 * contexts are independent.
 */
#ifndef EPLACE_H
#define EPLACE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EPLACE_ABI_VERSION 1

/* Status codes.  1..3 map 1:1 onto PlacerError
 * (crates/nextpnr/src/placer/mod.rs:20-28); the rest are this library's. */
typedef enum {
  EPLACE_OK = 0,
  EPLACE_ERR_NO_BELS = 1,           /* PlacerError::NoBelsAvailable */
  EPLACE_ERR_PLACEMENT_FAILED = 2,  /* PlacerError::PlacementFailed */
  EPLACE_ERR_INITIAL_PLACEMENT = 3, /* PlacerError::InitialPlacementFailed */
  EPLACE_ERR_INVALID = 4,           /* malformed CSR, NaN input, bad sizes */
  EPLACE_ERR_OOM = 5,               /* device/host allocation or admission refused */
  EPLACE_ERR_CUDA = 6,              /* CUDA runtime error (message has details) */
  EPLACE_ERR_TIMEOUT = 7,           /* a bounded device wait gave up */
  EPLACE_ERR_NO_DEVICE = 8,         /* no usable sm_100 device */
  EPLACE_PENDING = 9                /* job engine: the job has not finished yet */
} eplace_status;

/* ElectroPlaceCfg (crates/nextpnr/src/placer/electro_place/config.rs:5-40):
 * the same nine fields in the same order.  target_util, timing_driven and
 * timing_weight are carried but, as in the reference, never read;
 * target_density only shifts the DC term, which the solve zeroes. */
typedef struct {
  uint64_t seed;               /* default 1 */
  double wl_coeff;             /* default 0.5 */
  double target_util;          /* default 0.7 (unused, as in the reference) */
  uint8_t timing_driven;       /* default 0   (unused, as in the reference) */
  double target_density;       /* default 1.0 */
  double timing_weight;        /* default 0.0 (unused, as in the reference) */
  double nesterov_step_size;   /* default 0.1 */
  uint64_t max_iters;          /* default 500 */
  uint64_t legalize_interval;  /* default 5; 0 is rejected (EPLACE_ERR_INVALID) */
} eplace_cfg;

/* Fills the defaults of ElectroPlaceCfg::default() (config.rs:29-40). */
void eplace_cfg_default(eplace_cfg *cfg);

/* Build-only knobs with no reference counterpart. */
typedef enum {
  EPLACE_DCT_FP32_SIMT = 0,    /* FP32 DCT-matrix GEMMs on the CUDA cores */
  EPLACE_DCT_BF16X3_TC = 1,    /* BF16 three-term split GEMMs on tcgen05, FP32 accumulate */
  EPLACE_DCT_FP32_FFT = 2      /* FP32 FFTs (one N-point FFT per line); power-of-two bin grids of
                                  16 .. 1024 per axis, other grids take the FP32 GEMMs */
} eplace_dct_mode;

/* Field formula.  EPLACE_FIELD_REFERENCE reproduces density.rs:149-163
 * exactly: phi_hat(k) * w(k) is fed to DST-III input slot k, which that
 * transform treats as frequency k + 1, so the resulting "field" is not the
 * derivative of the potential and does not push cells apart (the reference
 * loop keeps its overlap well above 0.10 on dense designs).
 * EPLACE_FIELD_POTENTIAL_GRADIENT (extension, not reference-identical) moves
 * each spectrum one slot down and flips the sign, giving d(phi)/dx of the
 * reference's own DCT-III synthesis of phi_hat; with it the unchanged loop
 * spreads cells and reaches overlap < 0.10. */
typedef enum {
  EPLACE_FIELD_REFERENCE = 0,
  EPLACE_FIELD_POTENTIAL_GRADIENT = 1
} eplace_field_mode;

/* Where the periodic legalisations run.  Both give the same bindings, the
 * same displacement and the same HPWL (the reference's greedy choice and
 * tie-break, electro_place/mod.rs:206-255).  EPLACE_LEGAL_HOST: host
 * threads, snapshots copied to pinned memory.  EPLACE_LEGAL_GPU: on the
 * device, concurrent with the Nesterov loop, HPWL on the device; only the
 * best checkpoint's binding is copied back.  The device legaliser places the
 * cells in rounds (candidate lists in parallel, one serial pass over the
 * cells whose lists interact), as one CUDA graph per checkpoint.  Chips
 * larger than 4096 x 4096 sites fall back to EPLACE_LEGAL_HOST. */
typedef enum {
  EPLACE_LEGAL_HOST = 0,
  EPLACE_LEGAL_GPU = 1
} eplace_legal_mode;

typedef struct {
  int32_t dct_mode;            /* eplace_dct_mode; default EPLACE_DCT_FP32_FFT */
  int32_t legal_threads;       /* host legaliser threads; 0 = hardware concurrency */
  int32_t use_graphs;          /* capture each legalise interval as a CUDA graph; default 1 */
  int32_t verbose;             /* 1 = print the reference's per-legalisation trajectory line */
  int32_t max_inflight;        /* intervals launched ahead of the host; default 3 */
  int32_t field_mode;          /* eplace_field_mode; default EPLACE_FIELD_REFERENCE */
  int32_t legal_mode;          /* eplace_legal_mode; default EPLACE_LEGAL_HOST */
  int32_t wait_limit_us;       /* bound of each grid-barrier wait of the step kernel, microseconds;
                                  0 = about 2 s.  A wait that runs out ends the run with
                                  EPLACE_ERR_TIMEOUT; the context stays usable. */
} eplace_opts;

void eplace_opts_default(eplace_opts *opts);

/* Chip: a W x H site grid with one logic BEL (z = 0) per site, tile-major
 * (tile = y*W + x, chipdb/access.rs:118-126).  IO pads sit on separate BELs
 * and never occupy logic sites unless fixed_on_logic says so.  The density
 * grid is bins_x x bins_y (0 => one bin per site, as in the reference,
 * electro_place/mod.rs:71-76); width and height must be multiples of it. */
typedef struct {
  int32_t width, height;
  int32_t bins_x, bins_y;
} eplace_chip;

/* Netlist in CSR form.  Pin ids < num_cells are movable cells (solver
 * order); id num_cells + f is fixed cell f.  Each net lists its driver
 * first, then its users (NetInfo::driver / users, netlist/net.rs:14-67). */
typedef struct {
  uint32_t num_cells;
  uint32_t num_fixed;
  uint32_t num_nets;
  const uint8_t *cell_w, *cell_h;           /* footprint in sites; NULL => all 1x1 */
  const int32_t *cell_init_x, *cell_init_y; /* pre-bound site or -1; NULL => all unbound */
  const int32_t *fixed_x, *fixed_y;         /* BEL location of each fixed cell */
  const uint8_t *fixed_on_logic;            /* 1 => occupies the logic BEL at (x,y); NULL => none */
  const uint32_t *net_offsets;              /* [num_nets + 1], net_offsets[0] == 0 */
  const uint32_t *pin_cell;                 /* [net_offsets[num_nets]] */
  const uint8_t *net_has_driver;            /* NULL => every net's pin 0 drives it */
} eplace_netlist;

/* One line of the reference trajectory log (electro_place/mod.rs:185-188). */
typedef struct {
  int32_t iter;
  int32_t pad_;
  double hpwl;
  double displacement;
  double step_x, step_y;
  double density_penalty;
  double overlap;
} eplace_traj_entry;

/* Result: the side effects place_electro leaves on Context (cell.bel =
 * BelId{tile, index}, context/occupancy.rs:58-82), written into caller
 * buffers.  For a macro the BEL is its lower-left anchor site. */
typedef struct {
  int32_t *bel_tile;           /* [num_cells] out: y*W + x */
  int32_t *bel_index;          /* [num_cells] out: z (always 0), may be NULL */
  float *x, *y;                /* [num_cells] out: best continuous positions, may be NULL */
  eplace_traj_entry *traj;     /* [traj_capacity] out, may be NULL */
  uint32_t traj_capacity;
  /* scalar outputs */
  uint32_t traj_len;
  int64_t hpwl;                /* integer HPWL of the final binding */
  double overlap;              /* overlap of the last executed iteration */
  uint32_t iters;              /* Nesterov iterations executed */
  int32_t best_iter;           /* legalisation checkpoint chosen (-1: initial) */
  uint8_t converged;           /* overlap < 0.1 after >= 20 iterations */
  double gpu_seconds;          /* device time of the Nesterov loop */
  double total_seconds;        /* wall time of eplace_run */
  uint64_t gpu_launches;       /* kernels this library launched for the run */
  uint64_t h2d_bytes;          /* host->device bytes copied for the run */
  uint64_t d2h_bytes;          /* device->host bytes copied for the run */
} eplace_result;

typedef struct eplace_ctx eplace_ctx;

/* Validates and uploads the netlist to `device`; replaces Context set-up. */
eplace_status eplace_ctx_create(const eplace_netlist *nl, const eplace_chip *chip,
                                int32_t device, eplace_ctx **out);
void eplace_ctx_destroy(eplace_ctx *ctx);

/* Re-targets an existing context at another netlist / chip (the next job),
 * keeping its device buffers: they only grow, nothing is freed, and the DCT
 * matrices are rebuilt only when the bin grid changes.  Equivalent to
 * destroy + create, without the allocations.  No reference counterpart
 * (the reference rebuilds its Context per design). */
eplace_status eplace_ctx_load(eplace_ctx *ctx, const eplace_netlist *nl, const eplace_chip *chip);

/* place_electro (electro_place/mod.rs:65-204) on the uploaded netlist.
 * opts may be NULL (defaults). */
eplace_status eplace_run(eplace_ctx *ctx, const eplace_cfg *cfg, const eplace_opts *opts,
                         eplace_result *res);

/* One-shot convenience: load, run, return the result (the host-buffer
 * path).  The call keeps its context for the next one-shot call on the same
 * device (up to four are kept, until the process exits); the next call
 * re-loads it (eplace_ctx_load), so repeated calls do not re-allocate. */
eplace_status eplace_place(const eplace_netlist *nl, const eplace_chip *chip,
                           const eplace_cfg *cfg, const eplace_opts *opts,
                           int32_t device, eplace_result *res);

/* Copies the last error message (of ctx, or of this thread if ctx is NULL)
 * into buf; returns its full length. */
size_t eplace_last_error(const eplace_ctx *ctx, char *buf, size_t len);

int32_t eplace_abi_version(void);

/* ---------------------------------------------------------------------- */
/* Stage entry points: one hot-path kernel each, host buffers in and out. */
/* They run on the context's device and stream and are what the parity    */
/* tests call (teacher forcing: the same inputs the oracle gets).          */
/* ---------------------------------------------------------------------- */

/* WA gradient, replaces add_wa_wirelength_gradient (placer/common.rs:205-291)
 * + wa_axis_grad (solver/wa.rs:51-101).  x, y: [num_cells]. */
eplace_status eplace_stage_wa_grad(eplace_ctx *ctx, double wl_coeff, const float *x,
                                   const float *y, float *gx, float *gy);

/* Density map + overlap, replaces compute_concrete_density / compute_overlap
 * (electro_place/density.rs:54-86).  density: [bins_y * bins_x] row-major. */
eplace_status eplace_stage_density(eplace_ctx *ctx, const float *x, const float *y,
                                   double *density, double *overlap);

/* Field from a density map, replaces compute_density_field
 * (electro_place/density.rs:96-166).  phi_hat (scaled potential spectrum)
 * may be NULL. */
eplace_status eplace_stage_field(eplace_ctx *ctx, const double *density,
                                 int32_t dct_mode, int32_t field_mode, float *ex, float *ey,
                                 float *phi_hat);

/* Field gather, replaces compute_density_gradient (density.rs:171-206). */
eplace_status eplace_stage_gather(eplace_ctx *ctx, const float *x, const float *y,
                                  const float *ex, const float *ey, float *gx, float *gy);

/* One fused iteration tail, teacher-forced: field gather + density-penalty
 * update + combine + preconditioner + Barzilai-Borwein + FISTA step + clamp
 * + next look-ahead.  Replaces electro_place/mod.rs:124-173 with
 * compute_density_gradient (density.rs:171-206), NesterovSolver::step /
 * clamp_positions_range / look_ahead_into (solver/nesterov.rs:41-101) and
 * bb_step_size (:199-218).  look_*: the clamped look-ahead positions the
 * gradients were taken at; gwl_*: the WA gradient there; ex/ey: the field.
 * Solver state (x, y, x_prev, y_prev, gprev_*) is updated in place.
 * scal in/out: {density_penalty, density_initialized, step_x, step_y};
 * out: {step_norm_x, step_norm_y, alpha_x, alpha_y}. */
eplace_status eplace_stage_step(eplace_ctx *ctx, uint64_t iter, const float *look_x,
                                const float *look_y, const float *gwl_x, const float *gwl_y,
                                const float *ex, const float *ey, float *x, float *y,
                                float *x_prev, float *y_prev, float *gprev_x, float *gprev_y,
                                double *scal, double *out, float *next_look_x,
                                float *next_look_y);

/* The failure path of a bounded device wait, on demand.  No counterpart in
 * the reference.  Resets the context's solver state to the initial
 * placement of seed 1 and runs one fused step in its cooperative form (the
 * form with grid barriers) with `phantom` arrivals already counted on the
 * barrier (1 <= phantom < the step's grid size), so one block's wait can
 * never be met and must run out after wait_limit_us (> 0).  Returns
 * EPLACE_ERR_TIMEOUT when the wait ran out, as it must; the context is then
 * usable for the next run, which resets the device state.  Nothing faults
 * or hangs: every wait is bounded. */
eplace_status eplace_stage_barrier_timeout(eplace_ctx *ctx, int32_t wait_limit_us, uint32_t phantom);

/* Integer HPWL of a binding (anchor sites per movable cell), replaces
 * total_hpwl (metrics/wirelength.rs:10-51). */
/* The initial placement (placer/common.rs:27-117) for `seed` on the
 * context's device, as eplace_run makes it: the reference's xorshift64
 * Fisher-Yates shuffle of the free logic BELs, reformulated so that each
 * handed-out BEL is found independently (same permutation, bit for bit, as
 * eplace_initial_placement_host).  Problems with pre-bound cells take the
 * host form; *on_device (optional) tells which ran.  Writes the context's
 * positions (the next run resets them). */
eplace_status eplace_stage_initial_placement(eplace_ctx *ctx, uint64_t seed, int32_t *site_x, int32_t *site_y,
                                             int32_t *on_device);
eplace_status eplace_stage_hpwl(eplace_ctx *ctx, const int32_t *site_x,
                                const int32_t *site_y, int64_t *hpwl);

/* Device time of each kernel of the iteration, measured with CUDA events on
 * the context's stream over `reps` real iterations started from the initial
 * placement of cfg.  The iteration (kernels with event records between them)
 * is replayed as one CUDA graph, as the placement loop runs it, so host
 * launch latency is not counted.  stage_ms[8] = {WA gradient, density scatter, density
 * finalise, DCT GEMM 1, DCT GEMM 2 + spectral, DCT GEMM 3 (x2), DCT GEMM 4
 * (x2), fused gather/step}, mean milliseconds per launch. */
eplace_status eplace_profile_stages(eplace_ctx *ctx, const eplace_cfg *cfg, const eplace_opts *opts,
                                    uint32_t reps, double *stage_ms);

/* Greedy legalisation of continuous positions (electro_place/mod.rs:206-255),
 * host row search with the reference's tie-break. */
eplace_status eplace_legalize(eplace_ctx *ctx, const float *x, const float *y,
                              int32_t *site_x, int32_t *site_y, double *displacement);

/* The same legalisation on the GPU (rounds of parallel candidate lists and a
 * serial pass over the interacting cells; results identical to
 * eplace_legalize), followed by the device HPWL of the binding.  Replaces
 * legalize_electro (electro_place/mod.rs:206-255) + total_hpwl
 * (metrics/wirelength.rs:10-51).  Returns EPLACE_ERR_NO_BELS when a cell
 * finds no free site; EPLACE_ERR_INVALID for chips larger than 4096 x 4096
 * sites. */
eplace_status eplace_stage_legalize(eplace_ctx *ctx, const float *x, const float *y,
                                    int32_t *site_x, int32_t *site_y, double *displacement,
                                    int64_t *hpwl);

/* The same legaliser and the host HPWL without a context (no device needed):
 * host code of the path that callers may run on CPU-only machines. */
eplace_status eplace_legalize_host(const eplace_netlist *nl, const eplace_chip *chip,
                                   const float *x, const float *y, int32_t *site_x,
                                   int32_t *site_y, double *displacement);
eplace_status eplace_hpwl_host(const eplace_netlist *nl, const eplace_chip *chip,
                               const int32_t *site_x, const int32_t *site_y, int64_t *hpwl);
/* The reference's initial placement (placer/common.rs:27-117, xorshift64
 * Fisher-Yates over the free logic BELs), host only. */
eplace_status eplace_initial_placement_host(const eplace_netlist *nl, const eplace_chip *chip,
                                            uint64_t seed, int32_t *site_x, int32_t *site_y);
/* compute_pin_weights (placer/common.rs:381-407) without a context: for each
 * movable cell the sum of 1 / degree (f64, nets in order) over its nets of
 * two pins or more; pads take no weight.  The optimal-transport placer
 * computes the same weights for its preconditioner
 * (opt_trans_place/mod.rs:110), so a port of that placer takes them from
 * here.  weights: [num_cells].  Host only. */
eplace_status eplace_pin_weights(const eplace_netlist *nl, const eplace_chip *chip, double *weights);

/* Density map + overlap without any allocation.  No counterpart in the
 * reference: it is the density stage (eplace_stage_density) for callers
 * that cannot call cudaMalloc -- a real-time loop that must not allocate or
 * wait on the allocator, an application whose device memory is owned and
 * handed out by another component, or code under a fixed device-memory
 * budget.  All pointers are DEVICE pointers the caller owns, each 8-byte
 * aligned (a misaligned one is rejected with EPLACE_ERR_INVALID): pos_xy
 * [2*num_cells] (x0, y0, x1, y1, ...), half_wh [2*num_cells] half extents or
 * NULL for 1x1 cells, density [bins_y*bins_x] (out), overlap [1] (out).
 * stream is a cudaStream_t (NULL = the legacy default stream); the call is
 * asynchronous on it.  The working memory is a fixed array inside the
 * library, sized for at most 512 x 512 bins; larger grids are rejected with
 * EPLACE_ERR_INVALID.  Every GPU that loads the library holds that array
 * (about 2 MiB) until exit.  The first call on a device (and the first after
 * the device's context was destroyed, e.g. by cudaDeviceReset) looks the
 * array's device address up in the current context; make that first call
 * before any stream capture.  All calls share the one array: calls that
 * overlap on the GPU (other streams, other threads) race, so serialise
 * them.  Nothing is allocated or freed. */
eplace_status eplace_density_noalloc(const float *pos_xy, const float *half_wh,
                                     uint32_t num_cells, int32_t width, int32_t height,
                                     int32_t bins_x, int32_t bins_y, double *density,
                                     double *overlap, void *stream);

/* ---------------------------------------------------------------------- */
/* Job engine: many placement jobs on one GPU, continuously batched.       */
/* No reference counterpart (the reference places one design per call).   */
/* Jobs are admitted while fewer than max_jobs run and their estimated     */
/* device footprint fits hbm_budget (a job larger than the budget still    */
/* runs, alone).  Admitted jobs run concurrently: each on a context of its */
/* own (device buffers kept and reused across jobs), its intervals as CUDA */
/* graphs on its own stream, the legalisations on one shared host pool.    */
/* A job's result is the same as eplace_run's on the same input.           */
/* One internal thread drives the device; the calls are thread-safe.       */
/* ---------------------------------------------------------------------- */
typedef struct eplace_server eplace_server;

typedef struct {
  int32_t device;
  int32_t max_jobs;            /* jobs on the device at once; 0 = 16 */
  uint64_t hbm_budget;         /* device bytes jobs may hold; 0 = half the free memory */
  int32_t legal_threads;       /* shared host legaliser threads; 0 = hardware concurrency */
  int32_t reserved;
  eplace_opts opts;            /* run options of every job (a job whose bin grid the tensor-core
                                  transform does not support runs the FP32 transform) */
} eplace_server_cfg;

typedef struct {
  double queued_seconds;       /* submit -> admitted */
  double run_seconds;          /* admitted -> finished */
  double latency_seconds;      /* submit -> finished */
  uint64_t footprint_bytes;    /* admission estimate */
} eplace_job_info;

typedef struct {
  uint64_t submitted, finished, running, queued;
  uint64_t contexts;           /* contexts created (each reused across jobs) */
  uint64_t device_bytes;       /* device memory the contexts hold */
  double admit_seconds;        /* scheduler time spent admitting (load + start) */
  double pump_seconds;         /* scheduler time spent advancing and completing jobs */
  double idle_seconds;         /* scheduler time with nothing to do */
} eplace_server_stats;

void eplace_server_cfg_default(eplace_server_cfg *cfg);
eplace_status eplace_server_create(const eplace_server_cfg *cfg, eplace_server **out);
/* Finishes the running jobs, drops queued ones, frees everything.  Call it
 * after the last eplace_server_wait has returned. */
void eplace_server_destroy(eplace_server *srv);
/* Copies and validates the job's inputs (the caller may free them on
 * return) and queues it.  EPLACE_ERR_INVALID for a malformed netlist. */
eplace_status eplace_server_submit(eplace_server *srv, const eplace_netlist *nl, const eplace_chip *chip,
                                   const eplace_cfg *cfg, uint64_t *job_id);
/* Waits up to timeout_ms (< 0: forever, 0: poll) for the job.  Finished:
 * fills res (buffers as for eplace_run) and info (may be NULL), forgets the
 * job and returns its status (the message via eplace_last_error(NULL, ..)).
 * Not finished: EPLACE_PENDING. */
eplace_status eplace_server_wait(eplace_server *srv, uint64_t job_id, int32_t timeout_ms, eplace_result *res,
                                 eplace_job_info *info);
eplace_status eplace_server_stats_get(eplace_server *srv, eplace_server_stats *out);
/* The admission estimate of a job's device bytes (0 for an invalid netlist). */
uint64_t eplace_footprint(const eplace_netlist *nl, const eplace_chip *chip);

/* ---------------------------------------------------------------------- */
/* Synthetic netlist generator (seeded, deterministic), no reference      */
/* counterpart: the benchmark inputs.  Two calls: sizes, then fill.       */
/* ---------------------------------------------------------------------- */
typedef struct {
  uint64_t seed;
  uint32_t num_cells, num_nets, num_pads;
  int32_t width, height, bins_x, bins_y;
  uint32_t cluster_size;       /* 32 (cfg 1) / 64 (cfg 2+) */
  double locality;             /* 0.6 */
  double macro_fraction;       /* 0.05 for cfg 2+, else 0 */
  uint32_t macro_min, macro_max; /* 2, 8 */
} eplace_synth_spec;

typedef struct {
  uint32_t num_pins;           /* out of eplace_synth_size */
  uint32_t max_degree;
} eplace_synth_info;

eplace_status eplace_synth_size(const eplace_synth_spec *spec, eplace_synth_info *info);
/* Buffers: cell_w/cell_h [num_cells], fixed_x/fixed_y [num_pads],
 * net_offsets [num_nets + 1], pin_cell [num_pins]. */
eplace_status eplace_synth_fill(const eplace_synth_spec *spec, uint8_t *cell_w,
                                uint8_t *cell_h, int32_t *fixed_x, int32_t *fixed_y,
                                uint32_t *net_offsets, uint32_t *pin_cell);

#ifdef __cplusplus
}
#endif
#endif /* EPLACE_H */
