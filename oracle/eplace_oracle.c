/*
 * eplace_oracle.c -- FP64 CPU restatement of the reference ElectroPlace loop.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker and the timed CPU baseline).
 * The product path (eisenjoch_b200/) never links or calls this file.
 *
 * Reference paths are relative to the reference project root.  Where the
 * reference has no behaviour (macro footprints, bins coarser than sites) the
 * extension is defined so that it reduces exactly to the reference at
 * w = h = 1 and one bin per site; those places say "extension".
 */
#include "eplace_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------ */
/* RNG: xorshift64, seed 0 -> 1 (crates/nextpnr/src/context/rng.rs:19-31)   */
/* ------------------------------------------------------------------------ */
uint64_t orc_rng_next(uint64_t *s) {
  uint64_t x = *s;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  *s = x;
  return x;
}

/* Fisher-Yates from the end, j = (u64 as u32) % (i + 1)  (rng.rs:41-61). */
void orc_rng_shuffle_i32(uint64_t *s, int32_t *a, size_t n) {
  if (n <= 1) return;
  for (size_t i = n - 1; i >= 1; --i) {
    uint32_t r = (uint32_t)orc_rng_next(s);
    size_t j = (size_t)(r % (uint32_t)(i + 1));
    int32_t t = a[i];
    a[i] = a[j];
    a[j] = t;
  }
}

static int cell_w(const orc_problem *p, uint32_t i) { return p->cell_w ? p->cell_w[i] : 1; }
static int cell_h(const orc_problem *p, uint32_t i) { return p->cell_h ? p->cell_h[i] : 1; }

/* ------------------------------------------------------------------------ */
/* initial_placement (crates/nextpnr/src/placer/common.rs:27-117)            */
/* One movable cell type; fixed cells are already bound and consume no RNG.  */
/* Logic BELs are in chipdb order: tile-major, tile = y*W + x                */
/* (context/buckets.rs:37-43, chipdb/access.rs:118-126, :214-217).           */
/* Extension: a macro takes one site here, like a unit cell; its footprint   */
/* only matters for density and legalisation.                                */
/* ------------------------------------------------------------------------ */
int orc_initial_placement(const orc_problem *p, uint64_t seed, int32_t *sx, int32_t *sy) {
  const int64_t nsites = (int64_t)p->width * p->height;
  uint64_t rng = seed ? seed : 1; /* reseed_rng: DeterministicRng::new(seed.max(1)) */
  if (p->num_cells == 0) return ORC_OK;
  uint8_t *occ = (uint8_t *)calloc((size_t)(nsites > 0 ? nsites : 1), 1);
  if (!occ) return ORC_ERR_OOM;
  if (p->fixed_on_logic) {
    for (uint32_t f = 0; f < p->num_fixed; ++f)
      if (p->fixed_on_logic[f]) occ[(int64_t)p->fixed_y[f] * p->width + p->fixed_x[f]] = 1;
  }
  uint32_t n_unplaced = 0;
  for (uint32_t i = 0; i < p->num_cells; ++i) {
    int placed = p->cell_init_x && p->cell_init_x[i] >= 0;
    if (placed) {
      sx[i] = p->cell_init_x[i];
      sy[i] = p->cell_init_y[i];
      int64_t t = (int64_t)sy[i] * p->width + sx[i];
      if (occ[t]) { free(occ); return ORC_ERR_INITIAL_PLACEMENT; }
      occ[t] = 1;
    } else {
      ++n_unplaced;
    }
  }
  if (n_unplaced == 0) { free(occ); return ORC_OK; }
  if (nsites == 0) { free(occ); return ORC_ERR_NO_BELS; }
  int32_t *avail = (int32_t *)malloc(sizeof(int32_t) * (size_t)nsites);
  if (!avail) { free(occ); return ORC_ERR_OOM; }
  size_t na = 0;
  for (int64_t t = 0; t < nsites; ++t)
    if (!occ[t]) avail[na++] = (int32_t)t;
  orc_rng_shuffle_i32(&rng, avail, na);
  if (n_unplaced > na) { free(avail); free(occ); return ORC_ERR_NO_BELS; }
  size_t k = 0;
  for (uint32_t i = 0; i < p->num_cells; ++i) {
    if (p->cell_init_x && p->cell_init_x[i] >= 0) continue;
    int32_t t = avail[k++];
    sx[i] = t % p->width;
    sy[i] = t / p->width;
  }
  free(avail);
  free(occ);
  return ORC_OK;
}

/* compute_pin_weights (placer/common.rs:381-407): sum over pin occurrences
 * of 1/degree, degree = driver + users, nets of degree < 2 skipped. */
void orc_pin_weights(const orc_problem *p, double *w) {
  memset(w, 0, sizeof(double) * p->num_cells);
  for (uint32_t n = 0; n < p->num_nets; ++n) {
    uint32_t b = p->net_offsets[n], e = p->net_offsets[n + 1];
    uint32_t deg = e - b;
    if (deg < 2) continue;
    double wt = 1.0 / (double)deg;
    for (uint32_t k = b; k < e; ++k) {
      uint32_t c = p->pin_cell[k];
      if (c < p->num_cells) w[c] += wt;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* WA wirelength (crates/nextpnr/src/placer/solver/wa.rs)                    */
/* ------------------------------------------------------------------------ */
#define WA_EXP_CLAMP_MIN (-3000.0) /* wa.rs:14 */

static int g_wa_mode = ORC_WA_REFERENCE;

void orc_set_wa_mode(int mode) { g_wa_mode = mode; }

/* The exponent shifts of one axis.  Reference (wa.rs:58, :68, :73): both
 * exponentials are shifted by the pin mean, so exp() overflows once a pin
 * sits more than ~709/coeff sites from it (and S^2 in the gradient at half
 * that).  ORC_WA_STABLE (extension): e+ is shifted by the largest
 * coordinate and e- by the smallest, so every exponent is <= 0 and S >= 1;
 * WA value and gradient are the same functions of the coordinates (the
 * shift cancels in every quotient), only the rounding differs. */
static void wa_shifts(const double *c, size_t n, double *up, double *down) {
  if (g_wa_mode == ORC_WA_STABLE) {
    double lo = c[0], hi = c[0];
    for (size_t i = 1; i < n; ++i) {
      lo = fmin(lo, c[i]);
      hi = fmax(hi, c[i]);
    }
    *up = hi;
    *down = lo;
    return;
  }
  double center = 0.0;
  for (size_t i = 0; i < n; ++i) center += c[i];
  center /= (double)n;
  *up = *down = center;
}

/* wa_axis_value (wa.rs:17-46) */
double orc_wa_axis_value(const double *c, size_t n, double coeff) {
  if (n < 2) return 0.0;
  double up, down;
  wa_shifts(c, n, &up, &down);
  double smax = 0, xmax = 0, smin = 0, xmin = 0;
  for (size_t i = 0; i < n; ++i) {
    double ea = exp(fmax(coeff * (c[i] - up), WA_EXP_CLAMP_MIN));
    smax += ea;
    xmax += c[i] * ea;
    double eb = exp(fmax(coeff * (down - c[i]), WA_EXP_CLAMP_MIN));
    smin += eb;
    xmin += c[i] * eb;
  }
  if (smax < 1e-30 || smin < 1e-30) return 0.0;
  return xmax / smax - xmin / smin;
}

/* wa_axis_grad (wa.rs:51-101): quotient rule, accumulates into grad. */
void orc_wa_axis_grad(const double *c, size_t n, double coeff, double *grad) {
  if (n < 2) return;
  double up, down;
  wa_shifts(c, n, &up, &down);
  double *ea = (double *)malloc(sizeof(double) * n * 2);
  double *eb = ea + n;
  double smax = 0, smin = 0, xmax = 0, xmin = 0;
  for (size_t i = 0; i < n; ++i) {
    ea[i] = exp(fmax(coeff * (c[i] - up), WA_EXP_CLAMP_MIN));
    smax += ea[i];
    xmax += c[i] * ea[i];
    eb[i] = exp(fmax(coeff * (down - c[i]), WA_EXP_CLAMP_MIN));
    smin += eb[i];
    xmin += c[i] * eb[i];
  }
  if (smax < 1e-30 || smin < 1e-30) { free(ea); return; }
  double ism = 1.0 / smax, isn = 1.0 / smin;
  double ism2 = ism * ism, isn2 = isn * isn;
  for (size_t i = 0; i < n; ++i) {
    double dmax = ea[i] * ism + coeff * ea[i] * (c[i] * smax - xmax) * ism2;
    double dmin = eb[i] * isn - coeff * eb[i] * (c[i] * smin - xmin) * isn2;
    grad[i] += dmax - dmin;
  }
  free(ea);
}

/* add_wa_wirelength_gradient (placer/common.rs:205-291): per net, driver
 * then users; movable pins at the solver position, fixed pins at their BEL
 * location (no gradient); nets with < 2 pins skipped; net weight 1. */
void orc_wa_gradient(const orc_problem *p, const double *x, const double *y,
                     double coeff, double *gx, double *gy) {
  uint32_t maxdeg = 0;
  for (uint32_t n = 0; n < p->num_nets; ++n) {
    uint32_t d = p->net_offsets[n + 1] - p->net_offsets[n];
    if (d > maxdeg) maxdeg = d;
  }
  double *px = (double *)malloc(sizeof(double) * (maxdeg + 1) * 4);
  double *py = px + (maxdeg + 1);
  double *ngx = py + (maxdeg + 1);
  double *ngy = ngx + (maxdeg + 1);
  for (uint32_t n = 0; n < p->num_nets; ++n) {
    uint32_t b = p->net_offsets[n], e = p->net_offsets[n + 1];
    size_t k = 0;
    for (uint32_t q = b; q < e; ++q, ++k) {
      uint32_t c = p->pin_cell[q];
      if (c < p->num_cells) {
        px[k] = x[c];
        py[k] = y[c];
      } else {
        px[k] = (double)p->fixed_x[c - p->num_cells];
        py[k] = (double)p->fixed_y[c - p->num_cells];
      }
    }
    if (k < 2) continue;
    memset(ngx, 0, sizeof(double) * k);
    memset(ngy, 0, sizeof(double) * k);
    orc_wa_axis_grad(px, k, coeff, ngx);
    orc_wa_axis_grad(py, k, coeff, ngy);
    k = 0;
    for (uint32_t q = b; q < e; ++q, ++k) {
      uint32_t c = p->pin_cell[q];
      if (c < p->num_cells) {
        gx[c] += 1.0 * ngx[k];
        gy[c] += 1.0 * ngy[k];
      }
    }
  }
  free(px);
}

/* ------------------------------------------------------------------------ */
/* Density ("slither") -- electro_place/density.rs:20-76                     */
/* Cell footprint [x - w/2, x + w/2] x [y - h/2, y + h/2] in site units;     */
/* bin bx covers [bx*sx, (bx+1)*sx).  Reference: w = h = 1, sx = sy = 1.     */
/* ------------------------------------------------------------------------ */
typedef struct {
  double xlo, xhi, ylo, yhi;
  int32_t bxlo, bxhi, bylo, byhi;
} footprint;

static int32_t floor_bin(double v, double s) {
  double f = floor(v / s);
  if (f < 0) return 0;
  if (f > 2147483647.0) return 2147483647;
  return (int32_t)f;
}
static int32_t ceil_bin(double v, double s, int32_t nb) {
  double c = ceil(v / s);
  if (c < 0) c = 0; /* Rust `as usize` saturates at 0 */
  if (c > (double)nb) return nb;
  return (int32_t)c;
}

/* cell_bin_overlap (density.rs:20-37) */
static footprint cell_footprint(const orc_problem *p, uint32_t i, double cx, double cy) {
  footprint f;
  double sx = (double)(p->width / p->bins_x), sy = (double)(p->height / p->bins_y);
  double hw = 0.5 * cell_w(p, i), hh = 0.5 * cell_h(p, i);
  f.xlo = cx - hw;
  f.xhi = cx + hw;
  f.ylo = cy - hh;
  f.yhi = cy + hh;
  f.bxlo = floor_bin(f.xlo, sx);
  f.bxhi = ceil_bin(f.xhi, sx, p->bins_x);
  f.bylo = floor_bin(f.ylo, sy);
  f.byhi = ceil_bin(f.yhi, sy, p->bins_y);
  return f;
}

/* bin_overlap_area (density.rs:40-48) */
static double bin_area(const orc_problem *p, const footprint *f, int32_t bx, int32_t by) {
  double sx = (double)(p->width / p->bins_x), sy = (double)(p->height / p->bins_y);
  double x0 = (double)bx * sx, y0 = (double)by * sy;
  double ox = fmax(fmin(f->xhi, x0 + sx) - fmax(f->xlo, x0), 0.0);
  double oy = fmax(fmin(f->yhi, y0 + sy) - fmax(f->ylo, y0), 0.0);
  return ox * oy;
}

/* compute_concrete_density (density.rs:54-74) */
void orc_density(const orc_problem *p, const double *x, const double *y, double *d) {
  memset(d, 0, sizeof(double) * (size_t)p->bins_x * p->bins_y);
  for (uint32_t i = 0; i < p->num_cells; ++i) {
    footprint f = cell_footprint(p, i, x[i], y[i]);
    for (int32_t by = f.bylo; by < f.byhi; ++by)
      for (int32_t bx = f.bxlo; bx < f.bxhi; ++bx)
        d[(size_t)by * p->bins_x + bx] += bin_area(p, &f, bx, by);
  }
}

/* compute_overlap (density.rs:79-86); capacity 1 in the reference,
 * sites-per-bin (sx*sy) in the extension. */
double orc_overlap(const double *d, size_t n, double capacity) {
  double total = 0.0;
  for (size_t i = 0; i < n; ++i) total += d[i];
  if (total < 1e-30) return 0.0;
  double over = 0.0;
  for (size_t i = 0; i < n; ++i) over += fmax(d[i] - capacity, 0.0);
  return over / total;
}

/* ------------------------------------------------------------------------ */
/* 1D transforms with rustdct 0.7.1's unnormalised conventions               */
/* (the crate is called at density.rs:211-275):                              */
/*   DCT-II : X_k = sum_n x_n cos(pi k (n + 1/2) / N)                        */
/*   DCT-III: X_k = x_0 / 2 + sum_{n>=1} x_n cos(pi n (k + 1/2) / N)         */
/*   DST-III: X_k = (-1)^k x_{N-1} / 2 + sum_{n<N-1} x_n sin(pi (n+1)(k+1/2)/N) */
/* Backend 0 sums directly; backend 1 uses a radix-2 complex FFT (Makhoul's  */
/* reordering), valid for power-of-two N.                                    */
/* ------------------------------------------------------------------------ */
static int is_pow2(size_t n) { return n && !(n & (n - 1)); }

static void dct2_direct(double *v, size_t n) {
  double *o = (double *)malloc(sizeof(double) * n);
  for (size_t k = 0; k < n; ++k) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += v[i] * cos(M_PI * (double)k * ((double)i + 0.5) / (double)n);
    o[k] = s;
  }
  memcpy(v, o, sizeof(double) * n);
  free(o);
}

static void dct3_direct(double *v, size_t n) {
  double *o = (double *)malloc(sizeof(double) * n);
  for (size_t k = 0; k < n; ++k) {
    double s = 0.5 * v[0];
    for (size_t i = 1; i < n; ++i) s += v[i] * cos(M_PI * (double)i * ((double)k + 0.5) / (double)n);
    o[k] = s;
  }
  memcpy(v, o, sizeof(double) * n);
  free(o);
}

static void dst3_direct(double *v, size_t n) {
  double *o = (double *)malloc(sizeof(double) * n);
  for (size_t k = 0; k < n; ++k) {
    double s = ((k & 1) ? -0.5 : 0.5) * v[n - 1];
    for (size_t i = 0; i + 1 < n; ++i)
      s += v[i] * sin(M_PI * (double)(i + 1) * ((double)k + 0.5) / (double)n);
    o[k] = s;
  }
  memcpy(v, o, sizeof(double) * n);
  free(o);
}

/* radix-2 in-place complex FFT, sign = -1 forward, +1 inverse (unscaled) */
static void fft(double *re, double *im, size_t n, int sign) {
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double t = re[i]; re[i] = re[j]; re[j] = t;
      t = im[i]; im[i] = im[j]; im[j] = t;
    }
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    double ang = (double)sign * 2.0 * M_PI / (double)len;
    size_t half = len >> 1;
    for (size_t k = 0; k < half; ++k) {
      double wr = cos(ang * (double)k), wi = sin(ang * (double)k);
      for (size_t i = k; i < n; i += len) {
        size_t j = i + half;
        double xr = re[j] * wr - im[j] * wi;
        double xi = re[j] * wi + im[j] * wr;
        re[j] = re[i] - xr;
        im[j] = im[i] - xi;
        re[i] += xr;
        im[i] += xi;
      }
    }
  }
}

static void dct2_fft(double *v, size_t n) {
  if (n == 1) return;
  double *re = (double *)malloc(sizeof(double) * n * 2), *im = re + n;
  for (size_t i = 0; i < n / 2; ++i) {
    re[i] = v[2 * i];
    re[n - 1 - i] = v[2 * i + 1];
  }
  memset(im, 0, sizeof(double) * n);
  fft(re, im, n, -1);
  for (size_t k = 0; k < n; ++k) {
    double a = M_PI * (double)k / (2.0 * (double)n);
    v[k] = re[k] * cos(a) + im[k] * sin(a);
  }
  free(re);
}

/* DCT-III = (N/2) * inverse(DCT-II); inverse via the reverse Makhoul map */
static void dct3_fft(double *v, size_t n) {
  if (n == 1) { v[0] *= 0.5; return; }
  double *re = (double *)malloc(sizeof(double) * n * 2), *im = re + n;
  for (size_t k = 0; k < n; ++k) {
    double xr = v[k], xi = (k == 0) ? 0.0 : -v[n - k];
    double a = M_PI * (double)k / (2.0 * (double)n);
    double c = cos(a), s = sin(a);
    re[k] = xr * c - xi * s;
    im[k] = xr * s + xi * c;
  }
  fft(re, im, n, +1);
  /* unscaled inverse FFT = N * ifft; result * (N/2) / N = 0.5 */
  for (size_t i = 0; i < n / 2; ++i) {
    v[2 * i] = 0.5 * re[i];
    v[2 * i + 1] = 0.5 * re[n - 1 - i];
  }
  free(re);
}

/* DST-III_k(x) = (-1)^k DCT-III_k(reverse(x)) */
static void dst3_fft(double *v, size_t n) {
  for (size_t i = 0; i < n / 2; ++i) {
    double t = v[i]; v[i] = v[n - 1 - i]; v[n - 1 - i] = t;
  }
  dct3_fft(v, n);
  for (size_t k = 1; k < n; k += 2) v[k] = -v[k];
}

void orc_dct2(double *v, size_t n, int backend) {
  if (backend == 1 && is_pow2(n)) dct2_fft(v, n); else dct2_direct(v, n);
}
void orc_dct3(double *v, size_t n, int backend) {
  if (backend == 1 && is_pow2(n)) dct3_fft(v, n); else dct3_direct(v, n);
}
void orc_dst3(double *v, size_t n, int backend) {
  if (backend == 1 && is_pow2(n)) dst3_fft(v, n); else dst3_direct(v, n);
}

typedef void (*tf1d)(double *, size_t, int);

static void rows(double *d, size_t w, size_t h, tf1d f, int be) {
  for (size_t r = 0; r < h; ++r) f(d + r * w, w, be);
}
static void cols(double *d, size_t w, size_t h, tf1d f, int be) {
  double *buf = (double *)malloc(sizeof(double) * h);
  for (size_t c = 0; c < w; ++c) {
    for (size_t r = 0; r < h; ++r) buf[r] = d[r * w + c];
    f(buf, h, be);
    for (size_t r = 0; r < h; ++r) d[r * w + c] = buf[r];
  }
  free(buf);
}

static int g_field_mode = ORC_FIELD_REFERENCE;

/* compute_density_field (density.rs:96-166) */
int orc_field(const double *d, int32_t bw, int32_t bh, double td, int be,
              double *ex, double *ey, double *phi_hat) {
  size_t W = (size_t)bw, H = (size_t)bh, n = W * H;
  double *rho = (double *)malloc(sizeof(double) * n);
  if (!rho) return ORC_ERR_OOM;
  double sum = 0.0;
  for (size_t i = 0; i < n; ++i) sum += d[i];
  double avg = sum / (double)n;
  double target = td * fmax(avg, 1e-30);
  for (size_t i = 0; i < n; ++i) rho[i] = d[i] - target;
  rows(rho, W, H, orc_dct2, be); /* dct2_2d: rows then columns (:211-229) */
  cols(rho, W, H, orc_dct2, be);
  double scale = 4.0 / ((double)W * (double)H);
  for (size_t ky = 0; ky < H; ++ky)
    for (size_t kx = 0; kx < W; ++kx) {
      double s = scale;
      if (kx == 0) s *= 0.5;
      if (ky == 0) s *= 0.5;
      rho[ky * W + kx] *= s;
    }
  for (size_t ky = 0; ky < H; ++ky) {
    double wy = M_PI * (double)ky / (double)H;
    double wy2 = 2.0 * (1.0 - cos(wy));
    for (size_t kx = 0; kx < W; ++kx) {
      size_t idx = ky * W + kx;
      double wx = M_PI * (double)kx / (double)W;
      double wx2 = 2.0 * (1.0 - cos(wx));
      double den = wx2 + wy2;
      double ph = 0.0;
      if (den < 1e-30) {
        ex[idx] = 0.0;
        ey[idx] = 0.0;
      } else {
        ph = rho[idx] / den;
        ex[idx] = ph * wx;
        ey[idx] = ph * wy;
      }
      if (phi_hat) phi_hat[idx] = ph;
    }
  }
  if (g_field_mode == ORC_FIELD_POTENTIAL_GRADIENT) {
    /* Extension (not reference behaviour): DST-III input slot k is frequency
     * k + 1, so the spectrum of frequency k moves to slot k - 1, and the sign
     * is flipped, giving d(phi)/dx of the DCT-III synthesis of phi_hat. */
    for (size_t ky = 0; ky < H; ++ky) {
      for (size_t kx = 0; kx + 1 < W; ++kx) ex[ky * W + kx] = -ex[ky * W + kx + 1];
      ex[ky * W + W - 1] = 0.0;
    }
    for (size_t ky = 0; ky + 1 < H; ++ky)
      for (size_t kx = 0; kx < W; ++kx) ey[ky * W + kx] = -ey[(ky + 1) * W + kx];
    for (size_t kx = 0; kx < W; ++kx) ey[(H - 1) * W + kx] = 0.0;
  }
  rows(ex, W, H, orc_dst3, be); /* Ex: IDST rows, IDCT cols (:155-158) */
  cols(ex, W, H, orc_dct3, be);
  rows(ey, W, H, orc_dct3, be); /* Ey: IDCT rows, IDST cols (:160-163) */
  cols(ey, W, H, orc_dst3, be);
  free(rho);
  return ORC_OK;
}

void orc_set_field_mode(int mode) { g_field_mode = mode; }

int orc_potential(const double *phi_hat, int32_t bw, int32_t bh, int be, double *phi) {
  size_t W = (size_t)bw, H = (size_t)bh;
  memcpy(phi, phi_hat, sizeof(double) * W * H);
  rows(phi, W, H, orc_dct3, be);
  cols(phi, W, H, orc_dct3, be);
  return ORC_OK;
}

/* compute_density_gradient (density.rs:171-206): weighted mean of the field
 * over the bins the footprint overlaps.  Extension: scaled by the cell area
 * (w*h), which is 1 for every reference cell. */
void orc_gather(const orc_problem *p, const double *x, const double *y,
                const double *ex, const double *ey, double *gx, double *gy) {
  for (uint32_t i = 0; i < p->num_cells; ++i) {
    footprint f = cell_footprint(p, i, x[i], y[i]);
    double fx = 0, fy = 0, wt = 0;
    for (int32_t by = f.bylo; by < f.byhi; ++by)
      for (int32_t bx = f.bxlo; bx < f.bxhi; ++bx) {
        double w = bin_area(p, &f, bx, by);
        if (w > 0.0) {
          size_t idx = (size_t)by * p->bins_x + bx;
          fx += w * ex[idx];
          fy += w * ey[idx];
          wt += w;
        }
      }
    if (wt > 1e-10) {
      double area = (double)(cell_w(p, i) * cell_h(p, i));
      gx[i] += area * (fx / wt);
      gy[i] += area * (fy / wt);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Greedy legaliser (electro_place/mod.rs:206-255).                          */
/* Cells in solver order pick the available logic BEL minimising             */
/* (bx - x)^2 + (by - y)^2 (f64), strict '<' so the first minimum in BEL     */
/* order wins.  Extension: macros (w*h > 1) are legalised first, in solver   */
/* order, onto fully free w x h blocks inside the chip; cost uses the block  */
/* centre anchor + (w-1)/2; ties go to the lowest anchor tile.               */
/* ------------------------------------------------------------------------ */
static int block_free(const uint8_t *occ, int32_t W, int32_t ax, int32_t ay, int w, int h) {
  for (int dy = 0; dy < h; ++dy)
    for (int dx = 0; dx < w; ++dx)
      if (occ[(int64_t)(ay + dy) * W + ax + dx]) return 0;
  return 1;
}

static void block_set(uint8_t *occ, int32_t W, int32_t ax, int32_t ay, int w, int h) {
  for (int dy = 0; dy < h; ++dy)
    for (int dx = 0; dx < w; ++dx) occ[(int64_t)(ay + dy) * W + ax + dx] = 1;
}

/* Exhaustive scan in BEL order (the reference loop, mod.rs:224-237). */
static int legal_brute(const uint8_t *occ, int32_t W, int32_t H, double tx, double ty,
                       int w, int h, int32_t *bx, int32_t *by, double *bc) {
  double best = INFINITY;
  int found = 0;
  double ox = 0.5 * (w - 1), oy = 0.5 * (h - 1);
  for (int32_t ay = 0; ay + h <= H; ++ay)
    for (int32_t ax = 0; ax + w <= W; ++ax) {
      if (w == 1 && h == 1) {
        if (occ[(int64_t)ay * W + ax]) continue;
      } else if (!block_free(occ, W, ax, ay, w, h)) {
        continue;
      }
      double dx = ((double)ax + ox) - tx, dy = ((double)ay + oy) - ty;
      double c = dx * dx + dy * dy;
      if (c < best) {
        best = c;
        *bx = ax;
        *by = ay;
        found = 1;
      }
    }
  *bc = best;
  return found;
}

/* Ring search around the nearest anchor; same minimum and tie-break as the
 * scan.  A ring at Chebyshev radius r from the rounded target holds no site
 * closer than (r - 1/2)^2, so the search stops once (r - 1)^2 > best. */
static int legal_ring(const uint8_t *occ, int32_t W, int32_t H, double tx, double ty,
                      int w, int h, int32_t *bx, int32_t *by, double *bc) {
  double ox = 0.5 * (w - 1), oy = 0.5 * (h - 1);
  int32_t AW = W - w + 1, AH = H - h + 1; /* anchor grid */
  if (AW <= 0 || AH <= 0) return 0;
  int32_t cx = (int32_t)floor(tx - ox + 0.5), cy = (int32_t)floor(ty - oy + 0.5);
  if (cx < 0) cx = 0;
  if (cx >= AW) cx = AW - 1;
  if (cy < 0) cy = 0;
  if (cy >= AH) cy = AH - 1;
  double best = INFINITY;
  int64_t best_t = -1;
  int32_t rmax = AW > AH ? AW : AH;
  for (int32_t r = 0; r <= rmax; ++r) {
    if (best_t >= 0) {
      double lb = (double)(r - 1) * (double)(r - 1);
      if (r >= 1 && lb > best) break;
    }
    int32_t y0 = cy - r, y1 = cy + r, x0 = cx - r, x1 = cx + r;
    for (int32_t ay = (y0 < 0 ? 0 : y0); ay <= (y1 >= AH ? AH - 1 : y1); ++ay) {
      int full_row = (ay == y0 || ay == y1);
      int32_t step = full_row ? 1 : (x1 - x0);
      if (step <= 0) step = 1;
      for (int32_t ax = x0; ax <= x1; ax += step) {
        if (ax < 0 || ax >= AW) continue;
        int64_t t = (int64_t)ay * W + ax;
        if (w == 1 && h == 1) {
          if (occ[t]) continue;
        } else if (!block_free(occ, W, ax, ay, w, h)) {
          continue;
        }
        double dx = ((double)ax + ox) - tx, dy = ((double)ay + oy) - ty;
        double c = dx * dx + dy * dy;
        if (c < best || (c == best && t < best_t)) {
          best = c;
          best_t = t;
        }
      }
    }
  }
  if (best_t < 0) return 0;
  *bx = (int32_t)(best_t % W);
  *by = (int32_t)(best_t / W);
  *bc = best;
  return 1;
}

int orc_legalize(const orc_problem *p, const double *x, const double *y, int method,
                 int32_t *sx, int32_t *sy, double *disp) {
  int32_t W = p->width, H = p->height;
  uint8_t *occ = (uint8_t *)calloc((size_t)W * H + 1, 1);
  if (!occ) return ORC_ERR_OOM;
  if (p->fixed_on_logic)
    for (uint32_t f = 0; f < p->num_fixed; ++f)
      if (p->fixed_on_logic[f]) occ[(int64_t)p->fixed_y[f] * W + p->fixed_x[f]] = 1;
  double total = 0.0;
  int status = ORC_OK;
  for (int pass = 0; pass < 2 && status == ORC_OK; ++pass) {
    for (uint32_t i = 0; i < p->num_cells; ++i) {
      int w = cell_w(p, i), h = cell_h(p, i);
      int is_macro = (w * h > 1);
      if ((pass == 0) != is_macro) continue;
      int32_t bx = 0, by = 0;
      double c = 0;
      int ok = method == 0 ? legal_brute(occ, W, H, x[i], y[i], w, h, &bx, &by, &c)
                           : legal_ring(occ, W, H, x[i], y[i], w, h, &bx, &by, &c);
      if (!ok) { status = ORC_ERR_NO_BELS; break; }
      block_set(occ, W, bx, by, w, h);
      sx[i] = bx;
      sy[i] = by;
      total += c;
    }
  }
  free(occ);
  if (disp) *disp = total;
  return status;
}

/* net_hpwl / total_hpwl (metrics/wirelength.rs:10-51): nets without a
 * driver or without users contribute 0; integer bbox of driver + users. */
int64_t orc_hpwl(const orc_problem *p, const int32_t *sx, const int32_t *sy) {
  int64_t total = 0;
  for (uint32_t n = 0; n < p->num_nets; ++n) {
    uint32_t b = p->net_offsets[n], e = p->net_offsets[n + 1];
    int driven = p->net_has_driver ? p->net_has_driver[n] : 1;
    if (!driven || e - b < 2) continue; /* no driver, or no users */
    int32_t x0 = INT32_MAX, x1 = INT32_MIN, y0 = INT32_MAX, y1 = INT32_MIN;
    for (uint32_t q = b; q < e; ++q) {
      uint32_t c = p->pin_cell[q];
      int32_t lx, ly;
      if (c < p->num_cells) {
        lx = sx[c] + (cell_w(p, c) - 1) / 2;
        ly = sy[c] + (cell_h(p, c) - 1) / 2;
      } else {
        lx = p->fixed_x[c - p->num_cells];
        ly = p->fixed_y[c - p->num_cells];
      }
      if (lx < x0) x0 = lx;
      if (lx > x1) x1 = lx;
      if (ly < y0) y0 = ly;
      if (ly > y1) y1 = ly;
    }
    total += (int64_t)(x1 - x0) + (int64_t)(y1 - y0);
  }
  return total;
}

/* ------------------------------------------------------------------------ */
/* Full loop: place_electro (electro_place/mod.rs:65-204)                    */
/* ------------------------------------------------------------------------ */
void orc_cfg_default(orc_cfg *c) { /* config.rs:29-40 */
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

static double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ------------------------------------------------------------------------ */
/* NesterovSolver (crates/nextpnr/src/placer/solver/nesterov.rs:12-224)      */
/* ------------------------------------------------------------------------ */
void orc_nesterov_init(orc_nesterov *s, double *x, double *xp, size_t n, double step) {
  s->x = x;
  s->x_prev = xp;
  s->n = n;
  s->step_size = step;
  s->iter = 0;
  s->a = 1.0;
  memset(x, 0, sizeof(double) * n);
  memset(xp, 0, sizeof(double) * n);
}

void orc_nesterov_set_positions(orc_nesterov *s, const double *v) {
  memcpy(s->x, v, sizeof(double) * s->n);
  memcpy(s->x_prev, v, sizeof(double) * s->n);
}

/* momentum(): 0 before the first step, else (a - 1) / a_next (:75-82) */
double orc_nesterov_momentum(const orc_nesterov *s) {
  if (s->iter == 0) return 0.0;
  double an = (1.0 + sqrt(1.0 + 4.0 * s->a * s->a)) / 2.0;
  return (s->a - 1.0) / an;
}

void orc_nesterov_look_ahead(const orc_nesterov *s, double *y) {
  double m = orc_nesterov_momentum(s);
  for (size_t i = 0; i < s->n; ++i) y[i] = s->x[i] + m * (s->x[i] - s->x_prev[i]);
}

/* step(): FISTA momentum, y = x + m (x - x_prev) (unclamped), x' = y - step g;
 * returns the L2 norm of x' - x (:41-64). */
double orc_nesterov_step(orc_nesterov *s, const double *g) {
  s->iter += 1;
  double an = (1.0 + sqrt(1.0 + 4.0 * s->a * s->a)) / 2.0;
  double m = (s->a - 1.0) / an;
  s->a = an;
  double n2 = 0.0;
  for (size_t i = 0; i < s->n; ++i) {
    double xo = s->x[i];
    double y = s->x[i] + m * (s->x[i] - s->x_prev[i]);
    double xn = y - s->step_size * g[i];
    s->x_prev[i] = xo;
    s->x[i] = xn;
    double d = xn - xo;
    n2 += d * d;
  }
  return sqrt(n2);
}

void orc_nesterov_clamp(orc_nesterov *s, double lo, double hi) {
  for (size_t i = 0; i < s->n; ++i) {
    s->x[i] = clampd(s->x[i], lo, hi);
    s->x_prev[i] = clampd(s->x_prev[i], lo, hi);
  }
}

/* adaptive_restart (:125-139): restart when grad . (x - x_prev) > 0 */
void orc_nesterov_adaptive_restart(orc_nesterov *s, const double *g) {
  double dot = 0.0;
  for (size_t i = 0; i < s->n; ++i) dot += g[i] * (s->x[i] - s->x_prev[i]);
  if (dot > 0.0) {
    memcpy(s->x_prev, s->x, sizeof(double) * s->n);
    s->iter = 0;
    s->a = 1.0;
  }
}

/* lipschitz_step_size (:171-191) */
double orc_nesterov_lipschitz(const orc_nesterov *s, const double *pg, const double *cg) {
  double dx2 = 0.0, dg2 = 0.0;
  for (size_t i = 0; i < s->n; ++i) {
    double dx = s->x[i] - s->x_prev[i], dg = cg[i] - pg[i];
    dx2 += dx * dx;
    dg2 += dg * dg;
  }
  double dgn = sqrt(dg2);
  return dgn > 1e-30 ? sqrt(dx2) / dgn : s->step_size;
}

/* bb_step_size (:199-218): |dx.dx / dx.dg|, none when |dx.dg| < 1e-30 */
int orc_nesterov_bb(const orc_nesterov *s, const double *pg, const double *cg, double *out) {
  double dxdx = 0.0, dxdg = 0.0;
  for (size_t i = 0; i < s->n; ++i) {
    double dx = s->x[i] - s->x_prev[i], dg = cg[i] - pg[i];
    dxdx += dx * dx;
    dxdg += dx * dg;
  }
  if (fabs(dxdg) < 1e-30) return 0;
  *out = fabs(dxdx / dxdg);
  return 1;
}

/* Loop body (f)-(i), electro_place/mod.rs:131-173.  g holds g_wl on entry
 * and the combined, preconditioned gradient on exit. */
void orc_step(const orc_problem *p, orc_state *st, uint64_t it, double *g, const double *gd,
              const double *pw, double max_x, double max_y, double *step_norm) {
  const size_t n = p->num_cells;
  double *g2[2] = {g, g + n};
  const double *gd2[2] = {gd, gd + n};
  /* density penalty: init 0.1 |g_wl| / |g_den|, then x1.025 below 50, else +1 */
  if (!st->density_initialized) {
    double wl = 0, dn = 0;
    for (int ax = 0; ax < 2; ++ax)
      for (size_t i = 0; i < n; ++i) wl += g2[ax][i] * g2[ax][i];
    for (int ax = 0; ax < 2; ++ax)
      for (size_t i = 0; i < n; ++i) dn += gd2[ax][i] * gd2[ax][i];
    wl = sqrt(wl);
    dn = sqrt(dn);
    if (dn > 1e-30) {
      st->density_penalty = 0.1 * wl / dn;
      st->density_initialized = 1;
    }
  } else if (st->density_penalty < 50.0) {
    st->density_penalty *= 1.025;
  } else {
    st->density_penalty += 1.0;
  }
  const double lam = st->density_penalty;
  for (int ax = 0; ax < 2; ++ax)
    for (size_t i = 0; i < n; ++i) g2[ax][i] += lam * gd2[ax][i];
  /* preconditioner max(1, pw + lam) (mod.rs:151-156); extension: lam * area */
  for (size_t i = 0; i < n; ++i) {
    double area = (double)(cell_w(p, (uint32_t)i) * cell_h(p, (uint32_t)i));
    double pc = fmax(pw[i] + lam * area, 1.0);
    g2[0][i] /= pc;
    g2[1][i] /= pc;
  }
  double *pg[2] = {st->prev_grad, st->prev_grad + n};
  if (it > 0) {
    double bb;
    if (orc_nesterov_bb(&st->sx, pg[0], g2[0], &bb)) st->sx.step_size = clampd(bb, 1e-4, 1.0);
    if (orc_nesterov_bb(&st->sy, pg[1], g2[1], &bb)) st->sy.step_size = clampd(bb, 1e-4, 1.0);
  }
  memcpy(pg[0], g2[0], sizeof(double) * n); /* save_gradients (common.rs:479-482) */
  memcpy(pg[1], g2[1], sizeof(double) * n);
  step_norm[0] = orc_nesterov_step(&st->sx, g2[0]);
  step_norm[1] = orc_nesterov_step(&st->sy, g2[1]);
  orc_nesterov_clamp(&st->sx, 0.0, max_x);
  orc_nesterov_clamp(&st->sy, 0.0, max_y);
}

int orc_place(const orc_problem *p, const orc_cfg *cfg, int be, int lm, orc_result *res,
              double *overlap_trace) {
  const uint32_t n = p->num_cells;
  const double max_x = (double)(p->width - 1), max_y = (double)(p->height - 1);
  const size_t nb = (size_t)p->bins_x * p->bins_y;
  const double cap = (double)(p->width / p->bins_x) * (double)(p->height / p->bins_y);
  res->traj_len = 0;
  res->iters = 0;
  res->best_iter = -1;
  res->converged = 0;
  res->hpwl = 0;
  res->final_overlap = 0.0;
  res->first_nonfinite_grad_iter = -1;
  if (cfg->legalize_interval == 0) return ORC_ERR_INVALID; /* `%` by zero panics */

  /* reseed_rng + initial_placement (mod.rs:66-69) */
  int32_t *isx = (int32_t *)malloc(sizeof(int32_t) * (n + 1) * 2), *isy = isx + n + 1;
  int st = orc_initial_placement(p, cfg->seed, isx, isy);
  if (st != ORC_OK || n == 0) { free(isx); return st; } /* n == 0 => Ok (mod.rs:80-82) */

  double *buf = (double *)calloc((size_t)n * 16 + nb * 3, sizeof(double));
  int32_t *lsx = (int32_t *)malloc(sizeof(int32_t) * (n + 1) * 2), *lsy = lsx + n + 1;
  if (!buf || !lsx) { free(buf); free(lsx); free(isx); return ORC_ERR_OOM; }
  double *xs[2] = {buf, buf + n}, *xps[2] = {buf + 2 * n, buf + 3 * n};
  double *c = buf + 4 * n;        /* [2][n] look-ahead (cell_x, cell_y) */
  double *g = buf + 6 * n;        /* [2][n] */
  double *gd = buf + 8 * n;       /* [2][n] */
  double *best = buf + 12 * n;    /* [2][n] */
  double *pw = buf + 14 * n;
  double *init = buf + 10 * n;    /* [2][n] scratch: initial positions */
  double *d = buf + 16 * (size_t)n, *ex = d + nb, *ey = ex + nb;
  double *prev = (double *)calloc((size_t)n * 2, sizeof(double));
  for (uint32_t i = 0; i < n; ++i) { /* init_positions_from_bels (common.rs:179-199) */
    init[i] = (double)isx[i];
    init[n + i] = (double)isy[i];
  }
  orc_state S;
  orc_nesterov_init(&S.sx, xs[0], xps[0], n, cfg->nesterov_step_size);
  orc_nesterov_init(&S.sy, xs[1], xps[1], n, cfg->nesterov_step_size);
  orc_nesterov_set_positions(&S.sx, init);
  orc_nesterov_set_positions(&S.sy, init + n);
  S.prev_grad = prev; /* NesterovLoopState::new (common.rs:452-462) */
  S.density_penalty = 0.0;
  S.density_initialized = 0;
  memcpy(best, init, sizeof(double) * n * 2);
  orc_pin_weights(p, pw);
  double best_metric = INFINITY;
  double last_overlap = 0.0;

  for (uint64_t it = 0; it < cfg->max_iters; ++it) {
    /* look_ahead_into + clamp_positions (mod.rs:105-107) */
    orc_nesterov_look_ahead(&S.sx, c);
    orc_nesterov_look_ahead(&S.sy, c + n);
    for (uint32_t i = 0; i < n; ++i) {
      c[i] = clampd(c[i], 0.0, max_x);
      c[n + i] = clampd(c[n + i], 0.0, max_y);
    }
    memset(g, 0, sizeof(double) * n * 4); /* g and gd */
    orc_wa_gradient(p, c, c + n, cfg->wl_coeff, g, g + n);
    if (res->first_nonfinite_grad_iter < 0)
      for (size_t k = 0; k < (size_t)n * 2; ++k)
        if (!isfinite(g[k])) {
          res->first_nonfinite_grad_iter = (int32_t)it;
          break;
        }
    orc_density(p, c, c + n, d);
    double overlap = orc_overlap(d, nb, cap);
    last_overlap = overlap;
    if (overlap_trace) overlap_trace[it] = overlap;
    orc_field(d, p->bins_x, p->bins_y, cfg->target_density, be, ex, ey, NULL);
    orc_gather(p, c, c + n, ex, ey, gd, gd + n);
    double snorm[2];
    orc_step(p, &S, it, g, gd, pw, max_x, max_y, snorm);
    res->iters = (uint32_t)(it + 1);
    /* periodic legalisation + convergence (mod.rs:175-196) */
    if (it % cfg->legalize_interval == 0 || it == cfg->max_iters - 1) {
      double disp = 0.0;
      st = orc_legalize(p, S.sx.x, S.sy.x, lm, lsx, lsy, &disp);
      if (st != ORC_OK) break;
      double hp = (double)orc_hpwl(p, lsx, lsy);
      if (hp < best_metric) { /* record_metric (common.rs:485-495) */
        best_metric = hp;
        res->best_iter = (int32_t)it;
        memcpy(best, S.sx.x, sizeof(double) * n);
        memcpy(best + n, S.sy.x, sizeof(double) * n);
      }
      if (res->traj && res->traj_len < res->traj_capacity) {
        orc_traj *t = &res->traj[res->traj_len++];
        t->iter = (int32_t)it;
        t->hpwl = hp;
        t->displacement = disp;
        t->step_x = snorm[0];
        t->step_y = snorm[1];
        t->density_penalty = S.density_penalty;
        t->overlap = overlap;
      }
      if (it >= 20 && overlap < 0.1) {
        res->converged = 1;
        break;
      }
    }
  }
  if (st == ORC_OK) { /* final legalisation of the best snapshot (mod.rs:199) */
    double disp = 0.0;
    st = orc_legalize(p, best, best + n, lm, res->site_x, res->site_y, &disp);
    if (st == ORC_OK) res->hpwl = orc_hpwl(p, res->site_x, res->site_y);
    if (res->best_x) memcpy(res->best_x, best, sizeof(double) * n);
    if (res->best_y) memcpy(res->best_y, best + n, sizeof(double) * n);
  }
  res->final_overlap = last_overlap;
  free(prev);
  free(lsx);
  free(buf);
  free(isx);
  return st;
}
