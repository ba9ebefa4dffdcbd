/*
 * eplace_oracle.h -- CPU restatement (FP64) of the reference ElectroPlace loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * sm_100a product path in eisenjoch_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline / reference arm may load it, and only to check or
 * to time the CPU form.  The product library never links or calls it.
 *
 * Every function cites the reference file:line it restates (paths are relative
 * to the reference project root, crates/nextpnr/src/...).
 *
 * Parity status: the reference (Rust) cannot be built here (no cargo/rustc),
 * and its DCT arithmetic lives in the third-party crate rustdct 0.7.1 (on
 * rustfft 6.4.1), which is not vendored.  The transforms below restate
 * rustdct's documented unnormalised DCT-II / DCT-III / DST-III; they are
 * pinned against scipy.fft (tests/golden) and against the reference's own unit
 * tests (WA finite-difference KATs, overlap, HPWL integers, defaults).  No
 * reference test pins a numeric value of the field, so field parity is
 * "unpinned" by the reference itself.
 */
#ifndef EPLACE_ORACLE_H
#define EPLACE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: same numbering as include/eplace.h. */
enum {
  ORC_OK = 0,
  ORC_ERR_NO_BELS = 1,
  ORC_ERR_PLACEMENT_FAILED = 2,
  ORC_ERR_INITIAL_PLACEMENT = 3,
  ORC_ERR_INVALID = 4,
  ORC_ERR_OOM = 5,
};

/* Flat problem description (the same arrays the product C-ABI takes). */
typedef struct {
  int32_t width, height;   /* site grid: one logic BEL per site, tile = y*width + x */
  int32_t bins_x, bins_y;  /* density grid (reference: bins == sites) */
  uint32_t num_cells;      /* movable cells, solver order */
  uint32_t num_fixed;      /* fixed cells (pads / locked cells) */
  uint32_t num_nets;
  const uint8_t *cell_w, *cell_h;            /* NULL => 1x1 */
  const int32_t *cell_init_x, *cell_init_y;  /* NULL or -1 => unplaced */
  const int32_t *fixed_x, *fixed_y;
  const uint8_t *fixed_on_logic;             /* NULL => none occupy logic BELs */
  const uint32_t *net_offsets;               /* [num_nets + 1] */
  const uint32_t *pin_cell;                  /* < num_cells movable, else num_cells + fixed */
  const uint8_t *net_has_driver;             /* NULL => all nets driven by pin 0 */
} orc_problem;

/* ElectroPlaceCfg (electro_place/config.rs:5-40), same field order. */
typedef struct {
  uint64_t seed;
  double wl_coeff;
  double target_util;
  uint8_t timing_driven;
  double target_density;
  double timing_weight;
  double nesterov_step_size;
  uint64_t max_iters;
  uint64_t legalize_interval;
} orc_cfg;

typedef struct {
  int32_t iter;
  double hpwl, displacement, step_x, step_y, density_penalty, overlap;
} orc_traj;

/* --- RNG (context/rng.rs:19-61) --- */
uint64_t orc_rng_next(uint64_t *state);
void orc_rng_shuffle_i32(uint64_t *state, int32_t *a, size_t n);

/* --- set-up (placer/common.rs:27-117, :179-199, :381-407) --- */
int orc_initial_placement(const orc_problem *p, uint64_t seed, int32_t *site_x,
                          int32_t *site_y);
void orc_pin_weights(const orc_problem *p, double *w);

/* --- WA wirelength (solver/wa.rs:17-101, placer/common.rs:205-291) --- */
double orc_wa_axis_value(const double *c, size_t n, double coeff);
void orc_wa_axis_grad(const double *c, size_t n, double coeff, double *grad);
void orc_wa_gradient(const orc_problem *p, const double *x, const double *y,
                     double coeff, double *gx, double *gy);

/* --- density (electro_place/density.rs:20-86) --- */
void orc_density(const orc_problem *p, const double *x, const double *y, double *d);
double orc_overlap(const double *d, size_t n, double capacity);

/* --- 1D transforms, rustdct conventions (density.rs:211-275) --- */
/* backend 0 = direct FP64 sums, 1 = FFT-based (power-of-two lengths) */
void orc_dct2(double *v, size_t n, int backend);
void orc_dct3(double *v, size_t n, int backend);
void orc_dst3(double *v, size_t n, int backend);

/* Field mode: ORC_FIELD_REFERENCE restates density.rs exactly (default).
 * ORC_FIELD_POTENTIAL_GRADIENT is an extension with no reference
 * counterpart: the spectrum is moved one DST-III slot down and negated so
 * the field is d(phi)/dx of the DCT-III synthesis of phi_hat. */
enum { ORC_FIELD_REFERENCE = 0, ORC_FIELD_POTENTIAL_GRADIENT = 1 };
void orc_set_field_mode(int mode);

/* WA exponent shift: ORC_WA_REFERENCE = the pin mean (wa.rs:58, overflows in
 * FP64 on wide nets); ORC_WA_STABLE = per-net max / min (extension: the same
 * value and gradient, never overflows; the shift the CUDA kernel uses). */
enum { ORC_WA_REFERENCE = 0, ORC_WA_STABLE = 1 };
void orc_set_wa_mode(int mode);

/* --- Poisson field (density.rs:96-166) ---
 * phi_hat (optional) receives the scaled potential spectrum.  */
int orc_field(const double *d, int32_t bw, int32_t bh, double target_density,
              int backend, double *ex, double *ey, double *phi_hat);
/* Spatial potential: DCT-III of phi_hat along both axes (debug tap; the
 * reference never forms it). */
int orc_potential(const double *phi_hat, int32_t bw, int32_t bh, int backend,
                  double *phi);

/* --- gather (density.rs:171-206), area-scaled for macros --- */
void orc_gather(const orc_problem *p, const double *x, const double *y,
                const double *ex, const double *ey, double *gx, double *gy);

/* --- legaliser (electro_place/mod.rs:206-255) ---
 * method 0 = brute force in BEL order (reference loop), 1 = ring search
 * (identical result).  Outputs the anchor site per cell; returns status. */
int orc_legalize(const orc_problem *p, const double *x, const double *y,
                 int method, int32_t *site_x, int32_t *site_y,
                 double *displacement);

/* Integer HPWL (metrics/wirelength.rs:10-51) from each movable cell's
 * legalised anchor site.  Macro pins sit at anchor + (w-1)/2. */
int64_t orc_hpwl(const orc_problem *p, const int32_t *site_x, const int32_t *site_y);

/* --- NesterovSolver (solver/nesterov.rs:12-224), one axis --- */
typedef struct {
  double *x, *x_prev;   /* caller-owned [n] */
  size_t n;
  double step_size;
  uint64_t iter;
  double a;
} orc_nesterov;

void orc_nesterov_init(orc_nesterov *s, double *x, double *x_prev, size_t n, double step_size);
void orc_nesterov_set_positions(orc_nesterov *s, const double *v);           /* :128-132 */
double orc_nesterov_momentum(const orc_nesterov *s);                          /* :75-82 */
void orc_nesterov_look_ahead(const orc_nesterov *s, double *y);               /* :95-101 */
double orc_nesterov_step(orc_nesterov *s, const double *grad);                /* :41-64 */
void orc_nesterov_clamp(orc_nesterov *s, double lo, double hi);               /* :67-72 */
void orc_nesterov_adaptive_restart(orc_nesterov *s, const double *grad);      /* :125-139 */
double orc_nesterov_lipschitz(const orc_nesterov *s, const double *pg, const double *cg); /* :171-191 */
int orc_nesterov_bb(const orc_nesterov *s, const double *pg, const double *cg, double *out); /* :199-218 */

/* --- loop body (f)-(i) of electro_place/mod.rs:131-173, teacher-forced ---
 * gwl/gden: [2][n] (x then y), overwritten with the combined gradient.
 * State: both solvers, prev_grad [2][n], penalty.  Returns the two step norms. */
typedef struct {
  orc_nesterov sx, sy;
  double *prev_grad;        /* [2][n] */
  double density_penalty;
  int density_initialized;
} orc_state;

void orc_step(const orc_problem *p, orc_state *st, uint64_t iter, double *g, const double *gden,
              const double *pw, double max_x, double max_y, double *step_norm);

/* --- full loop (electro_place/mod.rs:65-204) --- */
typedef struct {
  int32_t *site_x, *site_y;   /* [num_cells] final legalised anchors */
  double *best_x, *best_y;    /* [num_cells] best continuous positions (may be NULL) */
  orc_traj *traj;             /* [traj_capacity] */
  uint32_t traj_capacity, traj_len;
  int64_t hpwl;
  double final_overlap;
  uint32_t iters;             /* iterations executed */
  int32_t best_iter;
  int converged;
  double overlap_trace_last;
  int32_t first_nonfinite_grad_iter; /* first iteration whose WA gradient had a NaN/inf, or -1 */
} orc_result;

/* dct_backend: 0 direct, 1 FFT.  legal_method: 0 brute, 1 ring.
 * overlap_trace (optional, [max_iters]) receives the per-iteration overlap. */
int orc_place(const orc_problem *p, const orc_cfg *cfg, int dct_backend,
              int legal_method, orc_result *res, double *overlap_trace);

void orc_cfg_default(orc_cfg *cfg);

/* --- benchmark input generator (orc_synth.c; no reference counterpart) --- */
typedef struct {
  uint64_t seed;
  uint32_t num_cells, num_nets, num_pads;
  int32_t width, height, bins_x, bins_y;
  uint32_t cluster_size;
  double locality;
  double macro_fraction;
  uint32_t macro_min, macro_max;
} orc_synth_spec;

/* With net_off == NULL: only *num_pins.  Else fills cw/ch [num_cells] (may
 * be NULL), fx/fy [num_pads], net_off [num_nets + 1], pin_cell [num_pins]. */
int orc_synth(const orc_synth_spec *spec, uint32_t *num_pins, uint8_t *cw, uint8_t *ch, int32_t *fx,
              int32_t *fy, uint32_t *net_off, uint32_t *pin_cell);

#ifdef __cplusplus
}
#endif
#endif
