/*
 * edm_oracle.c — CPU float64 restatement of the ED-MRDT per-timestep path.
 *
 * TEST INFRASTRUCTURE ONLY (see edm_oracle.h).  Every function cites the
 * reference lines it restates (paths within the reference project).  Compiled
 * with -ffp-contract=off so that no multiply-add is fused: the reference's
 * Numba kernels evaluate every float64 expression as separate IEEE operations.
 */
#include "edm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ========================================================================
 * Keyed noise.  Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies
 * with the Weyl key schedule.  Counter = (a, b, step_lo, stream<<16 | step_hi),
 * key = seed.  A 64-bit word x gives the uniform (x >> 11) * 2^-53 in [0,1).
 * ======================================================================== */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
    uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += PHILOX_W0; k1 += PHILOX_W1;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void orc_uniform2(uint64_t seed, int64_t step, int32_t stream, uint64_t a,
                  uint64_t b, double* u0, double* u1) {
  uint32_t ctr[4], key[2], o[4];
  ctr[0] = (uint32_t)a;
  ctr[1] = (uint32_t)b;
  ctr[2] = (uint32_t)((uint64_t)step);
  ctr[3] = ((uint32_t)stream << 16) | (uint32_t)(((uint64_t)step >> 32) & 0xFFFFu);
  key[0] = (uint32_t)seed;
  key[1] = (uint32_t)(seed >> 32);
  orc_philox(ctr, key, o);
  uint64_t x0 = ((uint64_t)o[1] << 32) | o[0];
  uint64_t x1 = ((uint64_t)o[3] << 32) | o[2];
  *u0 = (double)(x0 >> 11) * 0x1p-53;
  *u1 = (double)(x1 >> 11) * 0x1p-53;
}

/* Natural logarithm by the atanh series (Abramowitz & Stegun 4.1.27):
 * q = m 2^e, m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1),
 * ln m = 2 s (1 + s^2/3 + s^4/5 + ... + s^22/23), |s| <= 0.1716.
 * Fixed operation order; the device copy evaluates the same sequence. */
static const double ORC_LN_C[12] = {
    1.0,          1.0 / 3.0,  1.0 / 5.0,  1.0 / 7.0,  1.0 / 9.0,  1.0 / 11.0,
    1.0 / 13.0,   1.0 / 15.0, 1.0 / 17.0, 1.0 / 19.0, 1.0 / 21.0, 1.0 / 23.0};
#define ORC_LN2_HI 6.93147180369123816490e-01
#define ORC_LN2_LO 1.90821492927058770002e-10
#define ORC_SQRT2 1.41421356237309514547e+00

double orc_ln(double q) {
  uint64_t bits;
  memcpy(&bits, &q, 8);
  int e = (int)((bits >> 52) & 0x7FF) - 1023;
  uint64_t mb = (bits & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  double m;
  memcpy(&m, &mb, 8);
  if (m > ORC_SQRT2) {
    m = m * 0.5;
    e += 1;
  }
  double s = (m - 1.0) / (m + 1.0);
  double s2 = s * s;
  double p = ORC_LN_C[11];
  for (int k = 10; k >= 0; --k) p = p * s2 + ORC_LN_C[k];
  double lnm = (2.0 * s) * p;
  double de = (double)e;
  return de * ORC_LN2_HI + (de * ORC_LN2_LO + lnm);
}

/* sin and cos of 2 pi u, u in [0, 1): 4u = k + f with f reduced to
 * [-1/2, 1/2) (both exact), x = f pi/2 in [-pi/4, pi/4), Taylor series of
 * sin to x^17 and cos to x^18 (truncation below 3e-19) in Horner form with
 * a fixed operation order, then the quadrant k.  The device copy evaluates
 * the same sequence. */
static const double ORC_SIN_C[9] = {
    0x1.0000000000000p+0,  -0x1.5555555555555p-3, 0x1.1111111111111p-7,
    -0x1.a01a01a01a01ap-13, 0x1.71de3a556c734p-19, -0x1.ae64567f544e4p-26,
    0x1.6124613a86d09p-33,  -0x1.ae7f3e733b81fp-41, 0x1.952c77030ad4ap-49};
static const double ORC_COS_C[10] = {
    0x1.0000000000000p+0,  -0x1.0000000000000p-1, 0x1.5555555555555p-5,
    -0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-16, -0x1.27e4fb7789f5cp-22,
    0x1.1eed8eff8d898p-29,  -0x1.93974a8c07c9dp-37, 0x1.ae7f3e733b81fp-45,
    -0x1.6827863b97d97p-53};
#define ORC_PI_2 0x1.921fb54442d18p+0

void orc_sincos_2pi(double u, double* c, double* s) {
  double v = u * 4.0;
  int k = (int)v;
  double f = v - (double)k;
  if (f >= 0.5) {
    f = f - 1.0;
    k += 1;
  }
  double x = f * ORC_PI_2;
  double x2 = x * x;
  double ps = ORC_SIN_C[8];
  for (int i = 7; i >= 0; --i) ps = ps * x2 + ORC_SIN_C[i];
  double pc = ORC_COS_C[9];
  for (int i = 8; i >= 0; --i) pc = pc * x2 + ORC_COS_C[i];
  double sn = x * ps;
  switch (k & 3) {
    case 0: *c = pc; *s = sn; break;
    case 1: *c = -sn; *s = pc; break;
    case 2: *c = -pc; *s = -sn; break;
    default: *c = sn; *s = -pc; break;
  }
}

/* Standard normal pair by the Box-Muller transform (Box & Muller 1958) of
 * the key's uniform pair (counter b = 0): r = sqrt(-2 ln(1 - u0)),
 * (z0, z1) = r (cos 2 pi u1, sin 2 pi u1). */
void orc_normal2(uint64_t seed, int64_t step, int32_t stream, uint64_t a,
                 double* z0, double* z1) {
  double u0, u1;
  orc_uniform2(seed, step, stream, a, 0, &u0, &u1);
  double r = sqrt(-2.0 * orc_ln(1.0 - u0));
  double c, s;
  orc_sincos_2pi(u1, &c, &s);
  *z0 = r * c;
  *z1 = r * s;
}

void orc_fill_uniform(uint64_t seed, int64_t step, int32_t stream,
                      const int64_t* a, const int64_t* b, int64_t n,
                      double* out, int32_t two) {
  for (int64_t i = 0; i < n; ++i) {
    double u0, u1;
    orc_uniform2(seed, step, stream, (uint64_t)a[i], b ? (uint64_t)b[i] : 0u, &u0, &u1);
    if (two) {
      out[2 * i] = u0;
      out[2 * i + 1] = u1;
    } else {
      out[i] = u0;
    }
  }
}

void orc_fill_normal(uint64_t seed, int64_t step, int32_t stream,
                     const int64_t* a, int64_t n, double* out, int32_t two) {
  for (int64_t i = 0; i < n; ++i) {
    double z0, z1;
    orc_normal2(seed, step, stream, (uint64_t)a[i], &z0, &z1);
    if (two) {
      out[2 * i] = z0;
      out[2 * i + 1] = z1;
    } else {
      out[i] = z0;
    }
  }
}

/* Keyed Poisson draw (Knuth's product method) used for dark counts, in place
 * of numpy's Generator.poisson; exp(-lambda) comes from the host. */
int64_t orc_poisson_knuth(uint64_t seed, int64_t step, int32_t stream,
                          uint64_t key, double exp_neg_lambda) {
  double p = 1.0;
  int64_t k = 0;
  for (uint64_t t = 0; t < 100000; ++t) {
    double u0, u1;
    orc_uniform2(seed, step, stream, key, t, &u0, &u1);
    p *= u0;
    if (p <= exp_neg_lambda) return k;
    k += 1;
  }
  return k;
}

/* ========================================================================
 * Dynamics.
 * ======================================================================== */
static inline int clampi(int v, int n) {
  if (v >= n) v = n - 1;
  if (v < 0) v = 0;
  return v;
}

/* Python/Numba float `%` (floor-mod): result has the sign of the divisor. */
static inline double py_fmod(double x, double L) {
  double r = fmod(x, L);
  if (r != 0.0) {
    if ((r < 0.0) != (L < 0.0)) r += L;
  } else {
    r = copysign(0.0, L);
  }
  return r;
}

/* dynamics.py:199-216 */
static inline double min_image(double x1, double y1, double x2, double y2,
                               const EdmDynParams* p, double* odx, double* ody) {
  double dx = x1 - x2, dy = y1 - y2;
  if (p->periodic_x) {
    if (dx > 0.5 * p->Lx) dx -= p->Lx;
    else if (dx < -0.5 * p->Lx) dx += p->Lx;
  }
  if (p->periodic_y) {
    if (dy > 0.5 * p->Ly) dy -= p->Ly;
    else if (dy < -0.5 * p->Ly) dy += p->Ly;
  }
  *odx = dx;
  *ody = dy;
  return dx * dx + dy * dy;
}

int orc_dyn_alloc(OrcDyn* s, const EdmDynParams* p, int64_t N) {
  memset(s, 0, sizeof(*s));
  s->N = N;
  s->pos = (double*)calloc((size_t)N * 2, sizeof(double));
  s->species = (int32_t*)calloc((size_t)N, sizeof(int32_t));
  s->alive = (uint8_t*)calloc((size_t)N, 1);
  s->bond = (int32_t*)calloc((size_t)N, sizeof(int32_t));
  s->head = (int32_t*)calloc((size_t)p->nx * p->ny, sizeof(int32_t));
  s->next = (int32_t*)calloc((size_t)N, sizeof(int32_t));
  /* dynamics.py:233 */
  s->max_pairs = N * 30 < 500000 ? N * 30 : 500000;
  s->pairs = (int32_t*)calloc((size_t)(s->max_pairs > 0 ? s->max_pairs : 1) * 2, sizeof(int32_t));
  s->forces = (double*)calloc((size_t)N * 2, sizeof(double));
  if (!s->pos || !s->species || !s->alive || !s->bond || !s->head || !s->next ||
      !s->pairs || !s->forces)
    return -1;
  if (p->adapt_grid >= 0) {  /* dynamics.py:2088-2090: zeros */
    const EdmGrid* A = &p->grid[p->adapt_grid];
    s->adapt_w = (double*)calloc((size_t)A->nx * A->ny, sizeof(double));
    if (!s->adapt_w) return -1;
  }
  return 0;
}

void orc_dyn_free(OrcDyn* s) {
  free(s->pos); free(s->species); free(s->alive); free(s->bond);
  free(s->head); free(s->next); free(s->pairs); free(s->forces); free(s->adapt_w);
  memset(s, 0, sizeof(*s));
}

/* dynamics.py:1667-1703 — sequential float64 accumulation of inv_area. */
static void density_field(const EdmDynParams* p, const OrcDyn* s, int g, double* out) {
  const EdmGrid* G = &p->grid[g];
  memset(out, 0, sizeof(double) * (size_t)G->nx * G->ny);
  double cell_area = G->sx * G->sy;
  double inv_area = cell_area > 0.0 ? 1.0 / cell_area : 0.0;
  for (int64_t i = 0; i < s->N; ++i) {
    if (!s->alive[i]) continue;
    if (s->species[i] != G->sensor) continue;
    int gx = clampi((int)(s->pos[2 * i] / G->sx), G->nx);
    int gy = clampi((int)(s->pos[2 * i + 1] / G->sy), G->ny);
    out[gx * G->ny + gy] += inv_area;
  }
}

/* Hill factor as inlined in every feedback kernel, e.g. dynamics.py:965-976. */
static double hill_at(const EdmDynParams* p, int rule, const double* dens, double x, double y) {
  const EdmRule* R = &p->rule[rule];
  const EdmGrid* G = &p->grid[R->grid];
  int gx = clampi((int)(x / G->sx), G->nx);
  int gy = clampi((int)(y / G->sy), G->ny);
  double rho = dens[gx * G->ny + gy];
  if (R->K_half > 0) {
    double ratio = rho / R->K_half;
    double ratio_n = pow(ratio, R->n_hill);
    if (R->inhibition) return 1.0 / (1.0 + ratio_n);
    double h = ratio_n / (1.0 + ratio_n);
    return R->basal + (1.0 - R->basal) * h;
  }
  return 1.0;
}

/* Adaptation factor 1/(1 + (w/K)^n) (dynamics.py:1077-1083): w is read as
 * adaptation_field[gx, gy] with the feedback grid's (gx, gy), i.e. at flat
 * index gx * ny_adapt + gy of the adaptation array; w = 0 without PIP3. */
static double adapt_at(const EdmDynParams* p, const OrcDyn* s, int rule, double x, double y) {
  const EdmGrid* G = &p->grid[p->rule[rule].grid];
  int gx = clampi((int)(x / G->sx), G->nx);
  int gy = clampi((int)(y / G->sy), G->ny);
  double w = 0.0;
  if (p->adapt_grid >= 0) w = s->adapt_w[gx * p->grid[p->adapt_grid].ny + gy];
  if (p->adapt_K > 0) return 1.0 / (1.0 + pow(w / p->adapt_K, p->adapt_n));
  return 1.0;
}

int orc_dyn_step(const EdmDynParams* p, OrcDyn* s, int64_t step) {
  const int64_t N = s->N;
  const uint64_t seed = p->seed;
  double* pos = s->pos;
  int32_t* sp = s->species;
  uint8_t* alive = s->alive;
  const int nsp = EDM_MAX_SPECIES;

  /* 1. D(x) field (dynamics.py:440-519; sine-x field: D0(1+a sin(2 pi x/wl))) */
  double* Dp = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
  double* gD = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1) * 2);
  for (int64_t i = 0; i < N; ++i) {
    double x = pos[2 * i], y = pos[2 * i + 1];
    double base_D = p->D_base[sp[i]];
    double factor = 1.0, gfx = 0.0, gfy = 0.0;
    if (p->dfield == EDM_DFIELD_REGIONS) {
      for (int reg = 0; reg < p->n_regions; ++reg) {
        double dx_c = x - p->reg_cx[reg];
        double dy_c = y - p->reg_cy[reg];
        double d_sq = dx_c * dx_c + dy_c * dy_c;
        double d = d_sq > 1e-30 ? sqrt(d_sq) : 1e-15;
        double arg = (d - p->reg_r[reg]) / p->smooth_w;
        double sig, dsig;
        if (arg > 100.0) { sig = 0.0; dsig = 0.0; }
        else if (arg < -100.0) { sig = 1.0; dsig = 0.0; }
        else {
          double ea = exp(arg);
          double den = 1.0 + ea;
          sig = 1.0 / den;
          dsig = -ea / (den * den * p->smooth_w);
        }
        double local = 1.0 + (p->reg_f[reg] - 1.0) * sig;
        if (sig > 0.01) {
          factor = local;
          double inv_d = 1.0 / d;
          gfx = (p->reg_f[reg] - 1.0) * dsig * dx_c * inv_d;
          gfy = (p->reg_f[reg] - 1.0) * dsig * dy_c * inv_d;
          break;
        }
      }
      Dp[i] = base_D * factor;
      gD[2 * i] = base_D * gfx;
      gD[2 * i + 1] = base_D * gfy;
    } else if (p->dfield == EDM_DFIELD_SINE_X) {
      double w = 2.0 * M_PI / p->sine_wavelength;
      double ph = w * x;
      Dp[i] = base_D * (1.0 + p->sine_amp * sin(ph));
      gD[2 * i] = base_D * p->sine_amp * w * cos(ph);
      gD[2 * i + 1] = 0.0;
    } else {
      Dp[i] = base_D * factor;
      gD[2 * i] = base_D * gfx;
      gD[2 * i + 1] = base_D * gfy;
    }
  }

  /* 2. cell list, head/next chains (dynamics.py:176-196) */
  const int nx = p->nx, ny = p->ny;
  for (int c = 0; c < nx * ny; ++c) s->head[c] = -1;
  for (int64_t i = 0; i < N; ++i) {
    int cx = clampi((int)(pos[2 * i] / p->cell_sx), nx);
    int cy = clampi((int)(pos[2 * i + 1] / p->cell_sy), ny);
    int c = cx * ny + cy;
    s->next[i] = s->head[c];
    s->head[c] = (int32_t)i;
  }

  /* 3. pairs (dynamics.py:219-278), cap min(30N, 500000) */
  int64_t np_ = 0;
  for (int64_t i = 0; i < N; ++i) {
    double xi = pos[2 * i], yi = pos[2 * i + 1];
    int cxi = clampi((int)(xi / p->cell_sx), nx);
    int cyi = clampi((int)(yi / p->cell_sy), ny);
    for (int dcx = -1; dcx <= 1; ++dcx) {
      for (int dcy = -1; dcy <= 1; ++dcy) {
        int ncx = cxi + dcx, ncy = cyi + dcy;
        if (p->periodic_x) ncx = ((ncx % nx) + nx) % nx;
        else if (ncx < 0 || ncx >= nx) continue;
        if (p->periodic_y) ncy = ((ncy % ny) + ny) % ny;
        else if (ncy < 0 || ncy >= ny) continue;
        int j = s->head[ncx * ny + ncy];
        while (j >= 0) {
          if (j > i) {
            double dx, dy;
            double dsq = min_image(xi, yi, pos[2 * j], pos[2 * j + 1], p, &dx, &dy);
            if (dsq < p->cutoff_sq) {
              if (np_ < s->max_pairs) {
                s->pairs[2 * np_] = (int32_t)i;
                s->pairs[2 * np_ + 1] = j;
                np_++;
              }
            }
          }
          j = s->next[j];
        }
      }
    }
  }
  s->n_pairs = np_;
  const int32_t* pairs = s->pairs;

  /* 4. forces (dynamics.py:665-739, 752-816) */
  double* F = s->forces;
  memset(F, 0, sizeof(double) * (size_t)N * 2);
  if (p->use_wca) {
    for (int64_t q = 0; q < np_; ++q) {
      int i = pairs[2 * q], j = pairs[2 * q + 1];
      if (!alive[i] || !alive[j]) continue;
      double sigma = p->sigma[sp[i] * nsp + sp[j]];
      double eps = p->eps[sp[i] * nsp + sp[j]];
      if (sigma <= 0.0 || eps <= 0.0) continue;
      double dx, dy;
      double dsq = min_image(pos[2 * i], pos[2 * i + 1], pos[2 * j], pos[2 * j + 1], p, &dx, &dy);
      double rcut2 = sigma * sigma * 1.2599210498948732;
      if (dsq >= rcut2 || dsq < 1e-30) continue;
      double inv_r2 = 1.0 / dsq;
      double s2 = sigma * sigma * inv_r2;
      double s6 = s2 * s2 * s2;
      double s12 = s6 * s6;
      double f_over_r = 24.0 * eps * (2.0 * s12 - s6) * inv_r2;
      double fmax = 2400.0 * eps / (sigma * sigma);
      if (f_over_r > fmax) f_over_r = fmax;
      double fx = f_over_r * dx, fy = f_over_r * dy;
      F[2 * i] += fx; F[2 * i + 1] += fy;
      F[2 * j] -= fx; F[2 * j + 1] -= fy;
    }
  }
  if (p->use_harmonic) {
    for (int64_t q = 0; q < np_; ++q) {
      int i = pairs[2 * q], j = pairs[2 * q + 1];
      if (!alive[i] || !alive[j]) continue;
      double sigma = p->sigma[sp[i] * nsp + sp[j]];
      double k = p->kharm[sp[i] * nsp + sp[j]];
      if (sigma <= 0.0 || k <= 0.0) continue;
      double dx, dy;
      double dsq = min_image(pos[2 * i], pos[2 * i + 1], pos[2 * j], pos[2 * j + 1], p, &dx, &dy);
      double s2 = sigma * sigma;
      if (dsq >= s2 || dsq < 1e-30) continue;
      double r = sqrt(dsq);
      double fmag = k * (sigma - r);
      double f_over_r = fmag / r;
      double fx = f_over_r * dx, fy = f_over_r * dy;
      F[2 * i] += fx; F[2 * i + 1] += fy;
      F[2 * j] -= fx; F[2 * j + 1] -= fy;
    }
  }

  /* 5. BD step (dynamics.py:323-406) with keyed normals (dynamics.py:2194) */
  const double dt = p->dt;
  for (int64_t i = 0; i < N; ++i) {
    if (!alive[i]) continue;
    double z0, z1;
    orc_normal2(seed, step, EDM_S_BD_NORMAL, (uint64_t)i, &z0, &z1);
    double Di = Dp[i];
    double sn = sqrt(2.0 * Di * dt);
    double dxt = gD[2 * i] * dt;
    double dyt = gD[2 * i + 1] * dt;
    dxt += sn * z0;
    dyt += sn * z1;
    dxt += Di * F[2 * i] * dt;
    dyt += Di * F[2 * i + 1] * dt;
    double dr2 = dxt * dxt + dyt * dyt;
    if (dr2 > p->max_disp_sq) {
      double dr = sqrt(dr2);
      double scale = p->max_disp / dr;
      dxt *= scale;
      dyt *= scale;
    }
    pos[2 * i] += dxt;
    pos[2 * i + 1] += dyt;
    if (p->periodic_x) pos[2 * i] = py_fmod(pos[2 * i], p->Lx);
    else {
      if (pos[2 * i] < 0.0) pos[2 * i] = -pos[2 * i];
      else if (pos[2 * i] >= p->Lx) pos[2 * i] = 2.0 * p->Lx - pos[2 * i];
    }
    if (p->periodic_y) pos[2 * i + 1] = py_fmod(pos[2 * i + 1], p->Ly);
    else {
      if (pos[2 * i + 1] < 0.0) pos[2 * i + 1] = -pos[2 * i + 1];
      else if (pos[2 * i + 1] >= p->Ly) pos[2 * i + 1] = 2.0 * p->Ly - pos[2 * i + 1];
    }
  }
  free(Dp);
  free(gD);

  /* 6. binding / dissociation (dynamics.py:528-654, 2205-2225) */
  for (int r = 0; r < p->n_bind; ++r) {
    const EdmBind* B = &p->bind[r];
    for (int64_t q = 0; q < np_; ++q) {
      int i = pairs[2 * q], j = pairs[2 * q + 1];
      if (!alive[i] || !alive[j]) continue;
      if (s->bond[i] >= 0 || s->bond[j] >= 0) continue;
      int a, b;
      if (sp[i] == B->ra && sp[j] == B->rb) { a = i; b = j; }
      else if (sp[i] == B->rb && sp[j] == B->ra) { a = j; b = i; }
      else continue;
      double dx, dy;
      double dsq = min_image(pos[2 * i], pos[2 * i + 1], pos[2 * j], pos[2 * j + 1], p, &dx, &dy);
      if (dsq > B->contact_sq) continue;
      double u0, u1;
      orc_uniform2(seed, step, EDM_S_BIND + 2 * r, (uint64_t)i, (uint64_t)j, &u0, &u1);
      if (u0 < B->prob_bind) {
        sp[a] = B->product;
        alive[b] = 0;
        s->bond[a] = b;
        s->bond[b] = a;
        s->counters[EDM_C_BINDINGS]++;
      }
    }
    for (int64_t i = 0; i < N; ++i) {
      if (!alive[i]) continue;
      if (sp[i] != B->product) continue;
      if (s->bond[i] < 0) continue;
      double u0, u1;
      orc_uniform2(seed, step, EDM_S_DISSOC + 2 * r, (uint64_t)i, 0, &u0, &u1);
      if (u0 < B->prob_dissoc) {
        int j = s->bond[i];
        sp[i] = B->ra;
        sp[j] = B->rb;
        alive[j] = 1;
        pos[2 * j] = pos[2 * i];
        pos[2 * j + 1] = pos[2 * i + 1];
        s->bond[i] = -1;
        s->bond[j] = -1;
        s->counters[EDM_C_DISSOC]++;
      }
    }
  }

  /* density scratch: largest grid */
  int64_t gmax = 1;
  for (int g = 0; g < p->n_grids; ++g)
    if ((int64_t)p->grid[g].nx * p->grid[g].ny > gmax) gmax = (int64_t)p->grid[g].nx * p->grid[g].ny;
  double* dens1 = (double*)malloc(sizeof(double) * (size_t)gmax);
  double* dens2 = (double*)malloc(sizeof(double) * (size_t)gmax);

  /* 7a. adaptation field: w += dt/tau_w (rho_PIP3 - w) (dynamics.py:1093-1112, 2227-2242) */
  if (p->adapt_grid >= 0) {
    const EdmGrid* A = &p->grid[p->adapt_grid];
    density_field(p, s, p->adapt_grid, dens1);
    for (int64_t c = 0; c < (int64_t)A->nx * A->ny; ++c)
      s->adapt_w[c] += p->adapt_inv_tau * (dens1[c] - s->adapt_w[c]);
  }

  /* 7b. catalytic passes (dynamics.py:825-983, 2245-2297) */
  for (int c = 0; c < p->n_cat; ++c) {
    const EdmCat* C = &p->cat[c];
    if (C->rule >= 0) density_field(p, s, p->rule[C->rule].grid, dens1);
    for (int64_t q = 0; q < np_; ++q) {
      int i = pairs[2 * q], j = pairs[2 * q + 1];
      if (!alive[i] || !alive[j]) continue;
      int si;
      if (sp[i] == C->enzyme && sp[j] == C->substrate) si = j;
      else if (sp[j] == C->enzyme && sp[i] == C->substrate) si = i;
      else continue;
      double dx, dy;
      double dsq = min_image(pos[2 * i], pos[2 * i + 1], pos[2 * j], pos[2 * j + 1], p, &dx, &dy);
      if (dsq > C->contact_sq) continue;
      double peff = C->prob;
      if (C->rule >= 0) peff = C->prob * hill_at(p, C->rule, dens1, pos[2 * si], pos[2 * si + 1]);
      if (C->rule >= 0 && ((p->adapt_cat_mask >> c) & 1)) peff = peff * adapt_at(p, s, C->rule, pos[2 * si], pos[2 * si + 1]);
      double u0, u1;
      orc_uniform2(seed, step, EDM_S_CAT + c, (uint64_t)i, (uint64_t)j, &u0, &u1);
      if (u0 < peff) {
        sp[si] = C->product;
        s->counters[EDM_C_CATALYTIC]++;
      }
    }
  }

  /* 8. compartment exchanges (dynamics.py:1229-1555, 2300-2434) */
  for (int e = 0; e < p->n_exch; ++e) {
    const EdmExch* X = &p->exch[e];
    int dual = X->rule_on >= 0 && X->rule_on2 >= 0;
    if (dual) {
      density_field(p, s, p->rule[X->rule_on].grid, dens1);
      density_field(p, s, p->rule[X->rule_on2].grid, dens2);
    } else if (X->rule_on >= 0) {
      density_field(p, s, p->rule[X->rule_on].grid, dens1);
    }
    int64_t nrec = 0;
    /* local recruitment: CDF of max(density, 0.01) over the feedback grid (dynamics.py:2356-2371) */
    const EdmGrid* LG = X->rule_on >= 0 ? &p->grid[p->rule[X->rule_on].grid] : NULL;
    int64_t ncdf = 0;
    if (X->local_recruit && LG) {
      ncdf = (int64_t)LG->nx * LG->ny;
      double total = 0.0;
      for (int64_t k = 0; k < ncdf; ++k) {
        total += dens1[k] > 0.01 ? dens1[k] : 0.01;
        dens2[k] = total;
      }
      if (total > 0)
        for (int64_t k = 0; k < ncdf; ++k) dens2[k] /= total;
      else
        for (int64_t k = 0; k < ncdf; ++k) dens2[k] = (k + 1.0) / (double)ncdf;
    }
    for (int64_t i = 0; i < N; ++i) {
      if (nrec >= X->max_recruits) break;
      if (alive[i]) continue;
      if (sp[i] != X->species) continue;
      double ua, ub, px, py;
      orc_uniform2(seed, step, EDM_S_EX_ACCEPT + 4 * e, (uint64_t)i, 0, &ua, &ub);
      orc_uniform2(seed, step, EDM_S_EX_POS + 4 * e, (uint64_t)i, 0, &px, &py);
      double cx = px * p->Lx, cy = py * p->Ly;
      if (ncdf > 0) {  /* dynamics.py:1115-1217 */
        double rl, rl2, o0, o1;
        orc_uniform2(seed, step, EDM_S_EX_LOC + 4 * e, (uint64_t)i, 0, &rl, &rl2);
        orc_normal2(seed, step, EDM_S_EX_OFFSET + e, (uint64_t)i, &o0, &o1);
        int64_t lo = 0, hi = ncdf - 1;
        while (lo < hi) {
          int64_t mid = (lo + hi) / 2;
          if (dens2[mid] < rl) lo = mid + 1;
          else hi = mid;
        }
        int64_t gx = lo / LG->ny, gy = lo % LG->ny;
        cx = py_fmod(((double)gx + 0.5) * LG->sx + o0 * p->recruit_sigma, p->Lx);
        cy = py_fmod(((double)gy + 0.5) * LG->sy + o1 * p->recruit_sigma, p->Ly);
      }
      double peff = X->prob_on;
      if (dual) {
        peff = X->prob_on * hill_at(p, X->rule_on, dens1, cx, cy) * hill_at(p, X->rule_on2, dens2, cx, cy);
      } else if (X->rule_on >= 0) {
        peff = X->prob_on * hill_at(p, X->rule_on, dens1, cx, cy);
      }
      if (ua < peff) {
        alive[i] = 1;
        pos[2 * i] = cx;
        pos[2 * i + 1] = cy;
        nrec++;
      }
    }
    s->counters[EDM_C_RECRUITED] += nrec;
    if (X->rule_off >= 0) density_field(p, s, p->rule[X->rule_off].grid, dens1);
    for (int64_t i = 0; i < N; ++i) {
      if (!alive[i]) continue;
      if (sp[i] != X->species) continue;
      double peff = X->prob_off;
      if (X->rule_off >= 0) peff = X->prob_off * hill_at(p, X->rule_off, dens1, pos[2 * i], pos[2 * i + 1]);
      double u0, u1;
      orc_uniform2(seed, step, EDM_S_EX_DETACH + 4 * e, (uint64_t)i, 0, &u0, &u1);
      if (u0 < peff) {
        alive[i] = 0;
        s->counters[EDM_C_DETACHED]++;
      }
    }
  }

  /* 9. unimolecular conversions (dynamics.py:1565-1657, 2437-2465) */
  for (int v = 0; v < p->n_conv; ++v) {
    const EdmConv* V = &p->conv[v];
    if (V->rule >= 0) density_field(p, s, p->rule[V->rule].grid, dens1);
    for (int64_t i = 0; i < N; ++i) {
      if (!alive[i]) continue;
      if (sp[i] != V->from) continue;
      double peff = V->prob;
      if (V->rule >= 0) peff = V->prob * hill_at(p, V->rule, dens1, pos[2 * i], pos[2 * i + 1]);
      double u0, u1;
      orc_uniform2(seed, step, EDM_S_CONV + v, (uint64_t)i, 0, &u0, &u1);
      if (u0 < peff) {
        sp[i] = V->to;
        s->counters[EDM_C_CONVERTED]++;
      }
    }
  }
  free(dens1);
  free(dens2);
  return 0;
}

/* ========================================================================
 * Photophysics.
 * ======================================================================== */

/* photophysics.py:528-588 */
static void fret_bond(const OrcPhotParams* p, int b, OrcPhot* s) {
  for (int64_t i = 0; i < s->N; ++i) {
    if (!s->has_dye[i] || s->bleached[i]) continue;
    if (s->dye_type[i] != p->bond_donor[b]) continue;
    int partner = s->bond[i];
    if (partner >= 0) {
      if (p->bond_intra[b]) {
        double ratio = p->bond_R0[b] / p->bond_icd[b];
        double r6 = ratio * ratio * ratio * ratio * ratio * ratio;
        s->k_fret[i] = r6 / p->bond_tauD[b];
        s->acc_idx[i] = -1;
      } else if (s->has_dye[partner] && s->dye_type[partner] == p->bond_acceptor[b]) {
        double ratio = p->bond_R0[b] / p->bond_icd[b];
        double r6 = ratio * ratio * ratio * ratio * ratio * ratio;
        s->k_fret[i] = r6 / p->bond_tauD[b];
        s->acc_idx[i] = partner;
      }
    }
  }
}

/* photophysics.py:591-683 (O(N^2) search, as in the reference) */
static void fret_prox(const OrcPhotParams* p, int b, OrcPhot* s) {
  double r2 = p->prox_radius_um[b] * p->prox_radius_um[b];
  for (int64_t i = 0; i < s->N; ++i) {
    if (!s->has_dye[i] || !s->alive[i] || s->bleached[i]) continue;
    if (s->dye_type[i] != p->prox_donor[b]) continue;
    int found = 0;
    for (int64_t j = 0; j < s->N; ++j) {
      if (j == i) continue;
      if (!s->alive[j] || s->species[j] != p->prox_target[b]) continue;
      double dx = s->pos[2 * j] - s->pos[2 * i];
      double dy = s->pos[2 * j + 1] - s->pos[2 * i + 1];
      if (p->periodic_x) {
        if (dx > p->Lx / 2.0) dx -= p->Lx;
        else if (dx < -p->Lx / 2.0) dx += p->Lx;
      }
      if (p->periodic_y) {
        if (dy > p->Ly / 2.0) dy -= p->Ly;
        else if (dy < -p->Ly / 2.0) dy += p->Ly;
      }
      if (dx * dx + dy * dy < r2) {
        found = 1;
        break;
      }
    }
    s->k_fret[i] = found ? p->prox_khigh[b] : p->prox_klow[b];
    s->acc_idx[i] = -1;
  }
}

/* photophysics.py:1021-1114 */
void orc_update_fret_rates(const OrcPhotParams* p, OrcPhot* s) {
  for (int64_t i = 0; i < s->N; ++i) {
    s->k_fret[i] = 0.0;
    s->acc_idx[i] = -1;
  }
  for (int b = 0; b < p->n_bond; ++b) fret_bond(p, b, s);
  for (int b = 0; b < p->n_prox; ++b) fret_prox(p, b, s);
}

/* photophysics.py:486-521 */
static int64_t poisson_draw(double mean, double u_seed) {
  if (mean <= 0.0) return 0;
  uint64_t st = (uint64_t)(int64_t)(u_seed * 9.007199254740992e15);
  if (mean < 30.0) {
    double L = exp(-mean);
    int64_t k = 0;
    double pr = 1.0;
    for (;;) {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      double u = (double)(st >> 11) / 9.007199254740992e15;
      pr *= u;
      if (pr <= L) break;
      k += 1;
      if (k > 10000) break;
    }
    return k;
  }
  st = st * 6364136223846793005ull + 1442695040888963407ull;
  double u1 = (double)(st >> 11) / 9.007199254740992e15;
  st = st * 6364136223846793005ull + 1442695040888963407ull;
  double u2 = (double)(st >> 11) / 9.007199254740992e15;
  if (u1 < 1e-30) u1 = 1e-30;
  double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  double v = mean + sqrt(mean) * z + 0.5;
  int64_t n = (int64_t)v;
  return n > 0 ? n : 0;
}

/* photophysics.py:338-483, 1116-1197 */
int orc_photon_step(const OrcPhotParams* p, OrcPhot* s, int64_t step) {
  orc_update_fret_rates(p, s);
  const uint64_t seed = p->seed;
  int64_t n_ph = 0, arr_idx = 0;
  for (int64_t i = 0; i < s->N; ++i) {
    if (!s->has_dye[i] || !s->alive[i] || s->bleached[i]) continue;
    int dt_ = s->dye_type[i];
    if (dt_ < 0 || dt_ >= p->n_fluoro) continue;
    int s0 = p->ground[dt_], s1 = p->excited[dt_], t1 = p->t1[dt_], bl = p->bl[dt_];
    int cur = s->ctmc[i];
    int pss;
    if (cur == s0 || cur == s1) pss = 0;
    else if (t1 >= 0 && cur == t1) pss = 1;
    else if (bl >= 0 && cur == bl) {
      s->bleached[i] = 1;
      continue;
    } else pss = 0;
    double mean_d, mean_f, tau, T00, T01;
    int has_fret = s->k_fret[i] > 0.0;
    if (has_fret) {
      double tauD = p->tau_all[dt_];
      double kf = s->k_fret[i];
      tau = tauD / (1.0 + kf * tauD);
      double kb = p->k_fret_bound[dt_];
      double frac = 0.0;
      if (kb > 0.0) {
        frac = kf / kb;
        if (frac > 1.0) frac = 1.0;
      }
      mean_d = p->mean_ph[dt_][pss] * (1.0 - frac) + p->mean_ph_fret[dt_][pss] * frac;
      mean_f = p->mean_fret[dt_][pss] * (1.0 - frac) + p->mean_fret_fret[dt_][pss] * frac;
      T00 = p->T_step[dt_][pss][0] * (1.0 - frac) + p->T_step_fret[dt_][pss][0] * frac;
      T01 = p->T_step[dt_][pss][1] * (1.0 - frac) + p->T_step_fret[dt_][pss][1] * frac;
    } else {
      mean_d = p->mean_ph[dt_][pss];
      mean_f = p->mean_fret[dt_][pss];
      tau = p->tau_all[dt_];
      T00 = p->T_step[dt_][pss][0];
      T01 = p->T_step[dt_][pss][1];
    }
    double up, ut, ux;
    orc_uniform2(seed, step, EDM_S_PH_POISSON, (uint64_t)i, 0, &up, &ux);
    orc_uniform2(seed, step, EDM_S_PH_TRANS, (uint64_t)i, 0, &ut, &ux);
    int64_t n_d = poisson_draw(mean_d, up);
    int64_t n_f = 0;
    if (mean_f > 0.0 && has_fret) n_f = poisson_draw(mean_f, up * 0.5 + 0.25);
    for (int64_t j = 0; j < n_d; ++j) {
      if (n_ph >= p->max_photons) break;
      double t_arr;
      if (arr_idx < p->est_photons) {
        double u, uy;
        orc_uniform2(seed, step, EDM_S_PH_ARRIVAL, (uint64_t)arr_idx, 0, &u, &uy);
        arr_idx++;
        if (u < 1e-30) u = 1e-30;
        t_arr = -tau * log(u);
      } else {
        t_arr = tau;
      }
      s->ph_particle[n_ph] = (int32_t)i;
      s->ph_time[n_ph] = t_arr;
      s->ph_channel[n_ph] = (int8_t)dt_;
      s->ph_is_fret[n_ph] = 0;
      n_ph++;
    }
    int acc = s->acc_idx[i];
    if (n_f > 0 && acc >= 0) {
      int acc_t = s->dye_type[acc];
      double tau_a = (acc_t >= 0 && acc_t < p->n_fluoro) ? p->tau_all[acc_t] : tau;
      for (int64_t j = 0; j < n_f; ++j) {
        if (n_ph >= p->max_photons) break;
        double t_arr;
        if (arr_idx < p->est_photons) {
          double u, uy;
          orc_uniform2(seed, step, EDM_S_PH_ARRIVAL, (uint64_t)arr_idx, 0, &u, &uy);
          arr_idx++;
          if (u < 1e-30) u = 1e-30;
          t_arr = -tau_a * log(u);
        } else {
          t_arr = tau_a;
        }
        s->ph_particle[n_ph] = acc;
        s->ph_time[n_ph] = t_arr;
        s->ph_channel[n_ph] = (int8_t)acc_t;
        s->ph_is_fret[n_ph] = 1;
        n_ph++;
      }
    }
    if (ut < T00) s->ctmc[i] = (int8_t)s0;
    else if (ut < T00 + T01) s->ctmc[i] = (int8_t)(t1 >= 0 ? t1 : s0);
    else {
      s->ctmc[i] = (int8_t)(bl >= 0 ? bl : s0);
      s->bleached[i] = 1;
    }
  }
  s->n_photons = n_ph;
  return 0;
}

/* ========================================================================
 * Microscope.
 * ======================================================================== */

/* microscope.py:1069-1157 with 522-631 and 777-803 inlined. */
int orc_process_photons(const EdmScopeParams* sp, uint64_t seed, int64_t step,
                        const double* pos, int64_t N, const int32_t* ph_particle,
                        const double* ph_time, const int8_t* ph_channel,
                        int64_t n_ph, uint32_t* flim, OrcScopeStats* st) {
  if (n_ph == 0) return 0;
  st->n_received += n_ph;
  /* 1. detection efficiency: keyed by photon index */
  int64_t* det = (int64_t*)malloc(sizeof(int64_t) * (size_t)n_ph);
  int64_t nd = 0;
  for (int64_t k = 0; k < n_ph; ++k) {
    double u0, u1;
    orc_uniform2(seed, step, EDM_S_SC_QE, (uint64_t)k, 0, &u0, &u1);
    if (u0 < sp->qe) {
      int32_t pid = ph_particle[k];
      if (pid >= 0 && pid < N) det[nd++] = k;  /* microscope.py:1109-1114 */
    }
  }
  if (nd == 0) {
    free(det);
    return 0;
  }
  /* 2. stable sort of survivors by particle index (argsort mergesort) */
  int64_t* ord = (int64_t*)malloc(sizeof(int64_t) * (size_t)nd);
  int64_t* tmp = (int64_t*)malloc(sizeof(int64_t) * (size_t)nd);
  memcpy(ord, det, sizeof(int64_t) * (size_t)nd);
  for (int64_t width = 1; width < nd; width *= 2) {
    for (int64_t lo = 0; lo < nd; lo += 2 * width) {
      int64_t mid = lo + width < nd ? lo + width : nd;
      int64_t hi = lo + 2 * width < nd ? lo + 2 * width : nd;
      int64_t a = lo, b = mid, o = lo;
      while (a < mid && b < hi) {
        if (ph_particle[ord[b]] < ph_particle[ord[a]]) tmp[o++] = ord[b++];
        else tmp[o++] = ord[a++];
      }
      while (a < mid) tmp[o++] = ord[a++];
      while (b < hi) tmp[o++] = ord[b++];
    }
    memcpy(ord, tmp, sizeof(int64_t) * (size_t)nd);
  }
  /* 3. emitter-centric PSF draw (microscope.py:522-631) */
  const int R = sp->psf_range_px;
  const int maxn = (2 * R + 1) * (2 * R + 1);
  double* cum = (double*)malloc(sizeof(double) * (size_t)maxn);
  int* cpi = (int*)malloc(sizeof(int) * (size_t)maxn);
  int* cpj = (int*)malloc(sizeof(int) * (size_t)maxn);
  int cached_n = 0;
  double cached_total = 0.0;
  int last_pid = -999;
  double last_sigma = -1.0;
  for (int64_t q = 0; q < nd; ++q) {
    int64_t k = ord[q];
    int pid = ph_particle[k];
    int ch = ph_channel[k];
    if (ch < 0) ch = 0;
    if (ch >= sp->n_sigma) ch = 0;
    double sigma = sp->sigma_ch[ch];
    double inv2 = sp->inv_2sig2_ch[ch];
    if (sigma <= 0.0) {
      sigma = sp->sigma_ch[0];
      inv2 = sp->inv_2sig2_ch[0];
    }
    if (pid != last_pid || sigma != last_sigma) {
      double x = pos[2 * pid], y = pos[2 * pid + 1];
      double fx = (x - sp->offset_x) / sp->pixel_size - 0.5;
      double fy = (y - sp->offset_y) / sp->pixel_size - 0.5;
      int i0 = (int)floor(fx + 0.5);
      int j0 = (int)floor(fy + 0.5);
      if (i0 < -R || i0 >= sp->nx + R) continue;
      if (j0 < -R || j0 >= sp->ny + R) continue;
      cached_n = 0;
      cached_total = 0.0;
      for (int di = -R; di <= R; ++di) {
        int ii = i0 + di;
        if (ii < 0 || ii >= sp->nx) continue;
        double pcx = ((double)ii + 0.5) * sp->pixel_size + sp->offset_x;
        double dx = x - pcx;
        for (int dj = -R; dj <= R; ++dj) {
          int jj = j0 + dj;
          if (jj < 0 || jj >= sp->ny) continue;
          double pcy = ((double)jj + 0.5) * sp->pixel_size + sp->offset_y;
          double dy = y - pcy;
          double w = exp(-(dx * dx + dy * dy) * inv2);
          cached_total += w;
          cum[cached_n] = cached_total;
          cpi[cached_n] = ii;
          cpj[cached_n] = jj;
          cached_n++;
        }
      }
      last_pid = pid;
      last_sigma = sigma;
    }
    if (cached_n == 0 || cached_total <= 0.0) continue;
    double ua, ub;
    orc_uniform2(seed, step, EDM_S_SC_ASSIGN, (uint64_t)k, 0, &ua, &ub);
    double u = ua * cached_total;
    int si = cpi[0], sj = cpj[0];
    for (int m = 0; m < cached_n; ++m) {
      if (cum[m] >= u) {
        si = cpi[m];
        sj = cpj[m];
        break;
      }
    }
    /* 4. IRF jitter + TCSPC accumulate (microscope.py:743, 777-803) */
    double z0, z1;
    orc_normal2(seed, step, EDM_S_SC_JITTER, (uint64_t)k, &z0, &z1);
    double t = ph_time[k] + (0.0 + sp->sigma_irf * z0);
    st->n_detected++;
    int chn = ph_channel[k];
    if (chn < 0 || chn >= sp->n_channels) continue;
    if (si < 0 || si >= sp->nx || sj < 0 || sj >= sp->ny) continue;
    if (t < 0.0) t = 0.0;
    int64_t b = (int64_t)(t / sp->bin_width);
    if (b >= sp->n_bins) continue;
    flim[(((int64_t)chn * sp->nx + si) * sp->ny + sj) * sp->n_bins + b] += 1u;
  }
  free(cum); free(cpi); free(cpj); free(ord); free(tmp); free(det);
  return 0;
}

/* microscope.py:850-922 with keyed draws (pixel index q = (ch*nx+i)*ny+j). */
int orc_finalize_frame(const EdmScopeParams* sp, uint64_t seed, int64_t frame,
                       uint32_t* flim, int64_t* n_dark, int64_t* n_ap) {
  int64_t npx = (int64_t)sp->n_channels * sp->nx * sp->ny;
  int64_t tot = 0, tot_ap = 0;
  if (sp->dark_lambda >= 1e-10) {
    for (int64_t q = 0; q < npx; ++q) {
      int64_t n = orc_poisson_knuth(seed, frame, EDM_S_SC_DARK, (uint64_t)q, sp->dark_exp_neg);
      for (int64_t m = 0; m < n; ++m) {
        double u0, u1;
        orc_uniform2(seed, frame, EDM_S_SC_DARK_BIN, (uint64_t)q, (uint64_t)m, &u0, &u1);
        int64_t b = (int64_t)(u0 * (double)sp->n_bins);
        flim[q * sp->n_bins + b] += 1u;
      }
      tot += n;
    }
  }
  if (sp->ap_prob > 0.0) {
    for (int64_t q = 0; q < npx; ++q) {
      int64_t total = 0;
      for (int b = 0; b < sp->n_bins; ++b) total += flim[q * sp->n_bins + b];
      if (total == 0) continue;
      int64_t n = 0;
      for (int64_t m = 0; m < total; ++m) {
        double u0, u1;
        orc_uniform2(seed, frame, EDM_S_SC_AP, (uint64_t)q, (uint64_t)m, &u0, &u1);
        if (u0 < sp->ap_prob) n++;
      }
      for (int64_t m = 0; m < n; ++m) {
        double u0, u1;
        orc_uniform2(seed, frame, EDM_S_SC_AP_BIN, (uint64_t)q, (uint64_t)m, &u0, &u1);
        int64_t b = (int64_t)(u0 * (double)sp->n_bins);
        flim[q * sp->n_bins + b] += 1u;
      }
      tot_ap += n;
    }
  }
  *n_dark = tot;
  *n_ap = tot_ap;
  return 0;
}
