/*
 * orc_synth.c -- the benchmark input generator, restated for the oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see eplace_oracle.h).  The reference has no
 * generator: its benchmark flow synthesises Verilog with Yosys, which is not
 * available, so the workloads are seeded synthetic netlists.  The CPU
 * reference arm of the benchmark must not load the product library, so the
 * oracle carries its own copy of the generator.  tests/test_host_cpu.py
 * checks that both copies emit the same bytes for the same spec.
 *
 * Distribution (the benchmark configurations' shapes):
 *   net degree 2 (p .60), U[3,5] (.25), U[6,20] (.12), U[21,200] (.03),
 *   capped at the cell count;
 *   pins: a home cluster of `cluster_size` consecutive cells per net; each
 *   pin comes from it with probability `locality` (at most 64 tries), else
 *   uniformly from all cells; no cell twice in a net; pin 0 drives;
 *   footprints: a `macro_fraction` of the cells are square macros with side
 *   U[macro_min, macro_max], the rest 1x1;
 *   pads: evenly spaced along the perimeter walk (x along the bottom, up the
 *   right edge, back along the top, down the left edge), each joins one
 *   uniformly chosen net as a user, after the net's cell pins.
 * Random streams: splitmix64, one stream per purpose, seeded seed ^ const.
 */
#include <stdint.h>
#include <stdlib.h>

#include "eplace_oracle.h"

typedef struct {
  uint64_t s;
} sm64;

static uint64_t sm_next(sm64 *r) {
  uint64_t z = (r->s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

/* 53 random bits in [0, 1). */
static double sm_unit(sm64 *r) { return (double)(sm_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static uint32_t sm_below(sm64 *r, uint32_t n) { return (uint32_t)(sm_next(r) % n); }

static uint32_t degree_of(sm64 *r, uint32_t ncells) {
  double u = sm_unit(r);
  uint32_t d;
  if (u < 0.60)
    d = 2;
  else if (u < 0.85)
    d = 3 + sm_below(r, 3);
  else if (u < 0.97)
    d = 6 + sm_below(r, 15);
  else
    d = 21 + sm_below(r, 180);
  return d < ncells ? d : ncells;
}

/* Perimeter walk position p -> site (x, y), L = 2W + 2H - 4 positions. */
static void perimeter_site(int64_t p, int64_t W, int64_t H, int32_t *x, int32_t *y) {
  int64_t px, py;
  if (p < W) {
    px = p;
    py = 0;
  } else if (p < W + H - 1) {
    px = W - 1;
    py = p - W + 1;
  } else if (p < 2 * W + H - 2) {
    px = W - 2 - (p - (W + H - 1));
    py = H - 1;
  } else {
    px = 0;
    py = H - 2 - (p - (2 * W + H - 2));
  }
  *x = (int32_t)px;
  *y = (int32_t)py;
}

int orc_synth(const orc_synth_spec *sp, uint32_t *num_pins, uint8_t *cw, uint8_t *ch, int32_t *fx,
              int32_t *fy, uint32_t *net_off, uint32_t *pin_cell) {
  if (sp->width <= 0 || sp->height <= 0 || sp->cluster_size == 0) return ORC_ERR_INVALID;
  if (sp->num_pads > 0 && sp->width < 2) return ORC_ERR_INVALID;
  if (sp->num_nets > 0 && sp->num_cells < 2 && sp->num_pads == 0) return ORC_ERR_INVALID;
  const uint32_t N = sp->num_cells, NN = sp->num_nets, F = sp->num_pads;
  sm64 rdeg = {sp->seed ^ 0x1d8e4e27c47d124full};
  sm64 rpin = {sp->seed ^ 0x6a09e667f3bcc909ull};
  sm64 rmac = {sp->seed ^ 0xbb67ae8584caa73bull};
  sm64 rpad = {sp->seed ^ 0x3c6ef372fe94f82bull};
  uint32_t *deg = (uint32_t *)calloc((size_t)NN + 1, sizeof(uint32_t));
  uint32_t *npads = (uint32_t *)calloc((size_t)NN + 1, sizeof(uint32_t));
  uint32_t *pad_net = (uint32_t *)calloc((size_t)F + 1, sizeof(uint32_t));
  if (!deg || !npads || !pad_net) {
    free(deg);
    free(npads);
    free(pad_net);
    return ORC_ERR_OOM;
  }
  for (uint32_t n = 0; n < NN; ++n) deg[n] = N >= 2 ? degree_of(&rdeg, N) : 0;
  for (uint32_t f = 0; f < F; ++f) {
    pad_net[f] = NN ? sm_below(&rpad, NN) : 0;
    if (NN) npads[pad_net[f]]++;
  }
  uint64_t total = 0;
  for (uint32_t n = 0; n < NN; ++n) total += (uint64_t)deg[n] + npads[n];
  int st = ORC_OK;
  if (total > 0xffffffffull) st = ORC_ERR_INVALID;
  if (st == ORC_OK && num_pins) *num_pins = (uint32_t)total;
  if (st != ORC_OK || !net_off) goto done; /* size query */

  for (uint32_t i = 0; i < N; ++i) {
    uint8_t s = 1;
    if (sp->macro_fraction > 0 && sm_unit(&rmac) < sp->macro_fraction) {
      uint32_t lo = sp->macro_min > 1 ? sp->macro_min : 1;
      uint32_t hi = sp->macro_max > lo ? sp->macro_max : lo;
      s = (uint8_t)(lo + sm_below(&rmac, hi - lo + 1));
    }
    if (cw) cw[i] = s;
    if (ch) ch[i] = s;
  }
  {
    const int64_t W = sp->width, H = sp->height;
    const int64_t L = H >= 2 ? 2 * W + 2 * H - 4 : W;
    for (uint32_t f = 0; f < F; ++f)
      perimeter_site((int64_t)((uint64_t)f * (uint64_t)L / (uint64_t)F), W, H, &fx[f], &fy[f]);
  }
  {
    const uint32_t cs = sp->cluster_size;
    const uint32_t nclusters = N ? (N + cs - 1) / cs : 0;
    net_off[0] = 0;
    for (uint32_t n = 0; n < NN; ++n) net_off[n + 1] = net_off[n] + deg[n] + npads[n];
    for (uint32_t n = 0; n < NN; ++n) {
      uint32_t *out = pin_cell + net_off[n];
      if (deg[n] == 0) continue;
      uint32_t lo = sm_below(&rpin, nclusters) * cs;
      uint32_t sz = N - lo < cs ? N - lo : cs;
      for (uint32_t k = 0; k < deg[n]; ++k) {
        uint32_t c = 0;
        for (int attempt = 0;; ++attempt) {
          int local = attempt < 64 && sm_unit(&rpin) < sp->locality;
          c = local ? lo + sm_below(&rpin, sz) : sm_below(&rpin, N);
          int dup = 0;
          for (uint32_t j = 0; j < k && !dup; ++j) dup = out[j] == c;
          if (!dup) break;
        }
        out[k] = c;
      }
    }
    uint32_t *cursor = npads; /* reused: counts pads already appended per net */
    for (uint32_t n = 0; n < NN; ++n) cursor[n] = 0;
    for (uint32_t f = 0; f < F && NN > 0; ++f) { /* with no nets, pads join none */
      uint32_t n = pad_net[f];
      pin_cell[net_off[n] + deg[n] + cursor[n]++] = N + f;
    }
  }
done:
  free(deg);
  free(npads);
  free(pad_net);
  return st;
}
