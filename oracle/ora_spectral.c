/* Oracle: random streams and spectral routines.
 * TEST INFRASTRUCTURE ONLY (see ora.h).  FP64 throughout. */
#define _POSIX_C_SOURCE 200112L
#include "ora.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/*******************************************************************************
 * Philox4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11).  Replaces the per-tile Threefry proxy
 * of src/core/htrdr_draw_map.c:429-442: streams are keyed by pixel and
 * realisation so results do not depend on tiling or scheduling.
 ******************************************************************************/
void
ora_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  int r;
  for(r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void
ora_rng_init(struct ora_rng* rng, uint32_t key0, uint32_t key1, uint32_t ctr0, uint32_t ctr1)
{
  memset(rng, 0, sizeof(*rng));
  rng->key[0] = key0; rng->key[1] = key1;
  rng->ctr[0] = ctr0; rng->ctr[1] = ctr1;
}

uint32_t
ora_rng_u32(struct ora_rng* rng)
{
  const uint32_t id = rng->n >> 2;
  uint32_t w;
  if(!rng->blk_valid || rng->blk_id != id) {
    uint32_t c[4];
    c[0] = rng->ctr[0]; c[1] = rng->ctr[1]; c[2] = id; c[3] = 0;
    ora_philox4x32_10(c, rng->key, rng->blk);
    rng->blk_id = id;
    rng->blk_valid = 1;
  }
  w = rng->blk[rng->n & 3];
  rng->n += 1;
  return w;
}

double
ora_rng_canonical_f(struct ora_rng* rng)
{
  return (double)(ora_rng_u32(rng) >> 8) * (1.0 / 16777216.0);
}

double
ora_rng_canonical_d(struct ora_rng* rng)
{
  const uint32_t a = ora_rng_u32(rng) >> 5;
  const uint32_t b = ora_rng_u32(rng) >> 6;
  return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
}

/*******************************************************************************
 * Planck / Wiebelt (src/core/htrdr_spectral.h:56-132)
 ******************************************************************************/
/* Fraction of the black body emission above v = C2/(lambda T): 5-term series
 * for v >= 2, polynomial expansion otherwise (htrdr_spectral.h:56-83). */
double
ora_wiebelt(double v)
{
  const double c15_pi4 = 15.0 / (M_PI * M_PI * M_PI * M_PI);
  double w;
  if(v >= 2.0) {
    int m;
    w = 0.0;
    for(m = 1; m < 6; ++m) {
      const double mv = (double)m * v;
      w += exp(-mv) / (double)(m * m * m * m) * (((mv + 3.0) * mv + 6.0) * mv + 6.0);
    }
    w *= c15_pi4;
  } else {
    const double z0 = 1.0 / 3.0, z1 = 1.0 / 8.0, z2 = 1.0 / 60.0;
    const double z4 = 1.0 / 5040.0, z6 = 1.0 / 272160.0, z8 = 1.0 / 13305600.0;
    const double v2 = v * v;
    const double v4 = v2 * v2;
    const double poly = z0 - z1 * v + z2 * v2 - z4 * v2 * v2 + z6 * v4 * v2 - z8 * v4 * v4;
    w = 1.0 - c15_pi4 * v2 * v * poly;
  }
  return w;
}

/* htrdr_spectral.h:85-99 */
double
ora_blackbody_fraction(double lambda0, double lambda1, double T)
{
  const double C2 = 1.43877735e-2; /* m.K */
  return ora_wiebelt(C2 / lambda1 / T) - ora_wiebelt(C2 / lambda0 / T);
}

/* B_lambda(T) in W/m^2/sr/m (htrdr_spectral.h:101-116) */
double
ora_planck_monochromatic(double lambda, double T)
{
  const double c = 299792458.0, h = 6.62607015e-34, k = 1.380649e-23;
  const double l2 = lambda * lambda;
  const double l5 = l2 * l2 * lambda;
  return (2.0 * h * c * c / l5) / (exp(h * c / (lambda * k * T)) - 1.0);
}

/* Band average of B_lambda (htrdr_spectral.h:118-132) */
double
ora_planck_interval(double lmin, double lmax, double T)
{
  const double T2 = T * T;
  const double sigma = 5.6696e-8;
  return ora_blackbody_fraction(lmin, lmax, T) * sigma * (T2 * T2) / (M_PI * (lmax - lmin));
}

/* htrdr_spectral.h:136-148 */
double
ora_planck(double lmin, double lmax, double T)
{
  return lmin == lmax ? ora_planck_monochromatic(lmin, T) : ora_planck_interval(lmin, lmax, T);
}

/* Bisection on T (src/core/htrdr_spectral.c:31-89) */
int
ora_brightness_temperature(double lmin, double lmax, double radiance, double* temperature)
{
  const size_t MAX_ITER = 100;
  const double eps_T = 1e-4;
  const double eps_B = radiance * 1e-8;
  double T = 0, T0 = 0, T1 = 0, T2 = 200, B0 = 0;
  size_t i;
  for(i = 0; i < MAX_ITER; ++i) {
    if(ora_planck(lmin, lmax, T2) >= radiance) break;
    T2 *= 2;
  }
  if(i >= MAX_ITER) return ORA_RES_BAD_OP;
  for(i = 0; i < MAX_ITER; ++i) {
    double B;
    T = (T1 + T2) * 0.5;
    B = ora_planck(lmin, lmax, T);
    if(B < radiance) T1 = T; else T2 = T;
    if(fabs(T - T0) < eps_T || fabs(B - B0) < eps_B) break;
    T0 = T;
    B0 = B;
  }
  if(i >= MAX_ITER) return ORA_RES_BAD_OP;
  *temperature = T;
  return ORA_RES_OK;
}

/* src/core/htrdr_spectral.c:91-121 */
double
ora_radiance_temperature(double lmin, double lmax, double radiance)
{
  double T = 0;
  double avg = radiance;
  if(lmin != lmax) avg /= (lmax - lmin);
  if(ora_brightness_temperature(lmin, lmax, avg, &T) != ORA_RES_OK) T = 0;
  return T;
}

/*******************************************************************************
 * Planck wavelength sampler (src/core/htrdr_ran_wlen_planck.c)
 ******************************************************************************/
/* First index whose value is >= key (rsys search_lower_bound + cmp_dbl) */
static size_t
lower_bound(const double* a, size_t n, double key)
{
  size_t lo = 0, hi = n;
  while(lo < hi) {
    const size_t mid = lo + (hi - lo) / 2;
    if(a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* htrdr_ran_wlen_planck.c:55-134 */
int
ora_planck_ran_init(struct ora_planck_ran* p, const double range[2], size_t nbands, double Tref)
{
  size_t i;
  double sum = 0;
  memset(p, 0, sizeof(*p));
  p->range[0] = range[0];
  p->range[1] = range[1];
  p->ref_temperature = Tref;
  p->nbands = nbands;
  if(nbands == 0) return ORA_RES_OK; /* continuous sampling */
  p->band_len = (range[1] - range[0]) / (double)nbands;
  p->pdf = malloc(nbands * sizeof(double));
  p->cdf = malloc(nbands * sizeof(double));
  if(!p->pdf || !p->cdf) return ORA_RES_MEM_ERR;
  for(i = 0; i < nbands; ++i) {
    double lo = range[0] + (double)i * p->band_len;
    double hi = lo + p->band_len;
    if(hi > range[1]) hi = range[1];
    p->pdf[i] = ora_blackbody_fraction(lo * 1e-9, hi * 1e-9, Tref);
    sum += p->pdf[i];
  }
  for(i = 0; i < nbands; ++i) {
    p->pdf[i] /= sum;
    p->cdf[i] = i == 0 ? p->pdf[i] : p->pdf[i] + p->cdf[i - 1];
  }
  p->cdf[nbands - 1] = 1.0;
  return ORA_RES_OK;
}

void
ora_planck_ran_release(struct ora_planck_ran* p)
{
  free(p->pdf);
  free(p->cdf);
  p->pdf = p->cdf = NULL;
}

size_t
ora_planck_ran_band(const struct ora_planck_ran* p, double r0)
{
  return lower_bound(p->cdf, p->nbands, nextafter(r0, DBL_MAX));
}

/* Bisection on the black body fraction (htrdr_ran_wlen_planck.c:136-216) */
static double
planck_sample_continue(const struct ora_planck_ran* p, double r, double* pdf)
{
  const size_t MAX_ITER = 100;
  const double eps_l = 1e-15, eps_bf = 1e-6;
  const double r0m = p->range[0] * 1e-9, r1m = p->range[1] * 1e-9;
  const double bf_all = ora_blackbody_fraction(r0m, r1m, p->ref_temperature);
  double lmin = r0m, lmax = r1m, l = 0, lprev = 0, bf = 0, bfprev = 0;
  size_t i;
  for(i = 0; i < MAX_ITER; ++i) {
    l = (lmin + lmax) * 0.5;
    bf = ora_blackbody_fraction(r0m, l, p->ref_temperature);
    if(bf / bf_all < r) lmin = l; else lmax = l;
    if(fabs(lprev - l) < eps_l || fabs(bfprev - bf) < eps_bf) break;
    lprev = l;
    bfprev = bf;
  }
  if(pdf) {
    const double Bl = ora_planck(l, l, p->ref_temperature);
    const double Bm = ora_planck(r0m, r1m, p->ref_temperature);
    *pdf = Bl / (Bm * (r1m - r0m)) * 1e-9;
  }
  return l * 1e9;
}

/* htrdr_ran_wlen_planck.c:218-268 and :359-376 */
double
ora_planck_ran_sample(const struct ora_planck_ran* p, double r0, double r1, double* pdf)
{
  if(p->nbands) {
    const size_t i = ora_planck_ran_band(p, r0);
    const double lo = p->range[0] + (double)i * p->band_len;
    const double hi = lo + p->band_len;
    if(pdf) *pdf = p->pdf[i] * (1.0 / (hi - lo));
    return lo + (hi - lo) * r1;
  }
  if(fabs(p->range[0] - p->range[1]) <= 1e-6) { /* rsys eq_eps */
    if(pdf) *pdf = 1;
    return p->range[0];
  }
  return planck_sample_continue(p, r0, pdf);
}

/*******************************************************************************
 * CIE 1931 XYZ sampler (src/core/htrdr_ran_wlen_cie_xyz.c); analytic fits of
 * C. Wyman, P.-P. Sloan, P. Shirley, "Simple Analytic Approximations to the
 * CIE XYZ Color Matching Functions", JCGT 2(2), 2013.
 ******************************************************************************/
static double
gauss_piece(double lambda, double mu, double s_lo, double s_hi)
{
  const double t = (lambda - mu) * (lambda < mu ? s_lo : s_hi);
  return exp(-0.5 * t * t);
}

double
ora_fit_bar_1931(int channel, double l)
{
  switch(channel) {
    case 0: /* htrdr_ran_wlen_cie_xyz.c:85-92 */
      return 0.362 * gauss_piece(l, 442.0, 0.0624, 0.0374)
           + 1.056 * gauss_piece(l, 599.8, 0.0264, 0.0323)
           - 0.065 * gauss_piece(l, 501.1, 0.0490, 0.0382);
    case 1: /* :94-100 */
      return 0.821 * gauss_piece(l, 568.8, 0.0213, 0.0247)
           + 0.286 * gauss_piece(l, 530.9, 0.0613, 0.0322);
    default: /* :102-108 */
      return 1.217 * gauss_piece(l, 437.0, 0.0845, 0.0278)
           + 0.681 * gauss_piece(l, 459.0, 0.0385, 0.0725);
  }
}

/* htrdr_ran_wlen_cie_xyz.c:57-77 */
static double
trapezoid(double lo, double hi, int channel)
{
  const size_t n = (size_t)(hi - lo) + 1;
  const double dl = (hi - lo) / (double)n;
  double acc = 0;
  size_t i;
  for(i = 0; i < n; ++i) {
    const double f1 = ora_fit_bar_1931(channel, lo + dl * (double)i);
    const double f2 = ora_fit_bar_1931(channel, lo + dl * (double)(i + 1));
    acc += (f1 + f2) * dl * 0.5;
  }
  return acc;
}

/* htrdr_ran_wlen_cie_xyz.c:185-280 */
int
ora_cie_ran_init(struct ora_cie_ran* c, const double range[2], size_t nbands)
{
  int ch;
  size_t i;
  memset(c, 0, sizeof(*c));
  c->range[0] = range[0];
  c->range[1] = range[1];
  c->nbands = nbands;
  c->band_len = (range[1] - range[0]) / (double)nbands;
  for(ch = 0; ch < 3; ++ch) {
    double sum = 0;
    c->cdf[ch] = malloc(nbands * sizeof(double));
    if(!c->cdf[ch]) return ORA_RES_MEM_ERR;
    for(i = 0; i < nbands; ++i) {
      const double lo = range[0] + (double)i * c->band_len;
      double hi = lo + c->band_len;
      if(hi > range[1]) hi = range[1];
      c->cdf[ch][i] = trapezoid(lo, hi, ch);
      sum += c->cdf[ch][i];
    }
    c->rcp_integral[ch] = 1.0 / sum;
    for(i = 0; i < nbands; ++i) {
      c->cdf[ch][i] /= sum;
      if(i) c->cdf[ch][i] += c->cdf[ch][i - 1];
    }
    c->cdf[ch][nbands - 1] = 1.0;
  }
  return ORA_RES_OK;
}

void
ora_cie_ran_release(struct ora_cie_ran* c)
{
  int ch;
  for(ch = 0; ch < 3; ++ch) { free(c->cdf[ch]); c->cdf[ch] = NULL; }
}

size_t
ora_cie_ran_band(const struct ora_cie_ran* c, int channel, double r0)
{
  return lower_bound(c->cdf[channel], c->nbands, nextafter(r0, DBL_MAX));
}

/* Band from the CDF, then the root of the quadratic CDF of the linear
 * interpolant of the fit inside the band (htrdr_ran_wlen_cie_xyz.c:110-183) */
double
ora_cie_ran_sample(const struct ora_cie_ran* c, int ch, double r0, double r1, double* pdf)
{
  const size_t ib = ora_cie_ran_band(c, ch, r0);
  const double lmin = c->range[0] + c->band_len * (double)ib;
  const double lmax = lmin + c->band_len;
  const double fmin = ora_fit_bar_1931(ch, lmin);
  const double fmax = ora_fit_bar_1931(ch, lmax);
  const double a = 0.5 * (fmax - fmin) / c->band_len;
  const double b = (lmax * fmin - lmin * fmax) / c->band_len;
  const double cc = -lmin * fmin + lmin * lmin * a;
  const double d = 0.5 * (fmax + fmin) * c->band_len;
  double delta = b * b - 4 * a * (cc - d * r1);
  double l1, l2, l;
  if(delta < 0 && fabs(delta) <= 1e-6) delta = 0;
  l1 = (-b - sqrt(delta)) / (2 * a);
  l2 = (-b + sqrt(delta)) / (2 * a);
  if(lmin <= l1 && l1 < lmax) l = l1;
  else if(lmin <= l2 && l2 < lmax) l = l2;
  else l = (lmin + lmax) * 0.5;
  if(pdf) *pdf = c->rcp_integral[ch];
  return l;
}
