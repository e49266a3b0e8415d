/*
 * hyrex_oracle.c -- CPU restatement of HyRex, ABCMB's recombination module
 * (abcmb/hyrex/hyrex.py, helium.py, hydrogen.py, recomb_functions.py).
 *
 * TEST INFRASTRUCTURE ONLY: the checker a GPU version of the recombination
 * history is compared against.  Nothing in the product path loads it.
 *
 * The history is built in the reference's seven phases, each writing its own
 * fixed-size buffer and joined the way array_with_padding.concat joins them
 * (abcmb/hyrex/array_with_padding.py: the next buffer starts after the last
 * finite entry, every buffer keeps its length, unused entries are +inf):
 *   1 Saha HeII/III on the grid points with z >= 3600      helium.py:156-233
 *   2 post-Saha HeII expansion (4000 entries)              helium.py:297-373
 *   3 HeII ODE until x_HeII < 1e-4 (4096)                  helium.py:375-565
 *   4 post-Saha H expansion (800)                          hydrogen.py:190-276
 *   5 EMLA with two-photon correction to z = 700 (8192)    hydrogen.py:278-383
 *   6 EMLA + T_m until T_m/T_CMB or T_CMB leave the tables hydrogen.py:385-495
 *   7 three-level atom to lna = 0 (8192)                   hydrogen.py:664-780
 * with the effective rates of recomb_functions.py and the correction
 * function of hydrogen.py:538-575.  Each ODE phase is diffrax's
 * diffeqsolve(Kvaerno3, PIDController(rtol, atol), dt0 = 1e-3, t1 = inf,
 * SaveAt(ts) on the phase's 5e-4 grid, Event(cond)) -- the event is tested
 * at the end of every accepted step and ends the solve there, the grid points
 * up to that time are saved from the cubic Hermite dense output.  The
 * derivatives the post-Saha expansions take with jax.grad are taken here in
 * forward mode (dual numbers) through the same formulas, the table lookups
 * included.  The very-chord Jacobian is a central difference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "abcmb_oracle.h"

/* constants.py */
#define HX_PI 3.14159265358979323846
#define HX_C 29979245800.0
#define HX_HBAR 6.582119569509e-16
#define HX_KB 8.617343e-5
#define HX_MP 938271999.0
#define HX_ME 510998.9461
#define HX_MH (HX_MP + HX_ME + 13.5982860719383)
#define HX_MHE 3.72839e9
#define HX_MU_E (HX_MP * HX_ME / HX_MH)
#define HX_E21 10.198714553953742
#define HX_RYD 13.598286071938324
#define HX_LYA_FREQ (HX_RYD * 3. / 4. / (2. * HX_PI * HX_HBAR))
#define HX_SIGT 6.652458734e-25
#define HX_STEF (HX_PI * HX_PI / (60. * HX_HBAR * HX_HBAR * HX_HBAR * HX_C * HX_C))
#define HX_R2S1S 8.2206

/* recomb_functions.py:16-26 */
#define HX_TR_MIN 0.004
#define HX_TR_MAX 0.4
#define HX_NTR 100
#define HX_TRATIO_MIN 0.1
#define HX_TRATIO_MAX 1.0
#define HX_NTM 40

/* hyrex.py:126-136, helium.py:40, hydrogen.py:53 */
#define HX_SPACING 5.0e-4
#define HX_Z0 8000.
#define HX_Z_HE_EQUIL 3601.
#define HX_Z_TWOG 701.
#define HX_N_POST_HE 4000
#define HX_N_HE_ODE 4096
#define HX_N_POST_H 800
#define HX_N_LATE 8192

/* ---------------------------------------------------------------------- */
/* forward-mode dual numbers for the jax.grad derivatives                  */
/* ---------------------------------------------------------------------- */
typedef struct {
  double v, d;
} dl;

static dl dc(double v) { dl r = {v, 0.}; return r; }
static dl dadd(dl a, dl b) { dl r = {a.v + b.v, a.d + b.d}; return r; }
static dl dsub(dl a, dl b) { dl r = {a.v - b.v, a.d - b.d}; return r; }
static dl dmul(dl a, dl b) { dl r = {a.v * b.v, a.d * b.v + a.v * b.d}; return r; }
static dl ddiv(dl a, dl b) { dl r = {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; return r; }
static dl dexp_(dl a) { double e = exp(a.v); dl r = {e, a.d * e}; return r; }
static dl dsqrt_(dl a) { double s = sqrt(a.v); dl r = {s, a.d / (2. * s)}; return r; }
static dl dsc(dl a, double k) { dl r = {a.v * k, a.d * k}; return r; }          /* a * k */
static dl drs(double k, dl a) { return ddiv(dc(k), a); }                         /* k / a */

/* ---------------------------------------------------------------------- */
/* inputs                                                                  */
/* ---------------------------------------------------------------------- */
typedef struct {
  const oracle_hyrex_tables* tab;
  double logA[2][HX_NTR * HX_NTM];   /* log of the A2s / A2p columns of Alpha_inf */
  double logR[HX_NTR];
  double* swift_x;                   /* kB x the correction table's temperature column */
  /* RecombInputs: T_CMB, n_H, H sampled on the full lna grid (hyrex.py:16-90) */
  int n;
  double l0, l1;
  const double *T, *nH, *H;
  double YHe, omega_b, omega_cdm, Neff;
  double twog_end;                   /* lna where the two-photon phase ends, -log(701) */
} hx_t;

/* RecombInputs.TCMB / nH / H: fast_interp(lna, grid[0], grid[-1], arr)
 * (ABCMBTools.py:268-308), with its derivative in lna (zero where clipped) */
static dl ri_interp(const hx_t* h, const double* arr, dl x) {
  const int n = h->n;
  double i = (x.v - h->l0) / (h->l1 - h->l0) * (double)(n - 1);
  double di = x.d / (h->l1 - h->l0) * (double)(n - 1);
  if (i < 1.e-6) { i = 1.e-6; di = 0.; }
  if (i > (double)(n - 1) - 1.e-6) { i = (double)(n - 1) - 1.e-6; di = 0.; }
  const int il = (int)floor(i);
  const int iu = il + 1 < n - 1 ? il + 1 : n - 1;
  const double wu = i - (double)il;
  dl r = {(1.0 - wu) * arr[il] + wu * arr[iu], di * (arr[iu] - arr[il])};
  return r;
}
static dl ri_T(const hx_t* h, dl l) { return ri_interp(h, h->T, l); }
static dl ri_nH(const hx_t* h, dl l) { return ri_interp(h, h->nH, l); }
static dl ri_H(const hx_t* h, dl l) { return ri_interp(h, h->H, l); }

/* jnp.interp(x, xp, fp) on an increasing uniform axis (clamped) */
static double interp_uniform(double x, double x0, double x1, int n, const double* fp) {
  if (x <= x0) return fp[0];
  if (x >= x1) return fp[n - 1];
  const double step = (x1 - x0) / (double)(n - 1);
  int i = (int)floor((x - x0) / step);
  if (i > n - 2) i = n - 2;
  const double xa = x0 + (double)i * step;
  return fp[i] + (x - xa) / step * (fp[i + 1] - fp[i]);
}

/* jnp.interp(x, xp, arange(n)): the fractional index on a uniform axis */
static double frac_index(double x, double x0, double x1, int n) {
  if (x <= x0) return 0.;
  if (x >= x1) return (double)(n - 1);
  const double step = (x1 - x0) / (double)(n - 1);
  int i = (int)floor((x - x0) / step);
  if (i > n - 2) i = n - 2;
  const double xa = x0 + (double)i * step;
  return (double)i + (x - xa) / step;
}

/* jax.scipy.ndimage.map_coordinates(table, [a, b], order=1), mode constant
 * (out-of-range corners count 0 with weight 0 at the upper edges) */
static double bilinear(const double* t, double a, double b) {
  const int a0 = (int)floor(a), b0 = (int)floor(b);
  const double wa = a - a0, wb = b - b0;
  double s = 0.;
  for (int da = 0; da < 2; ++da)
    for (int db = 0; db < 2; ++db) {
      const int ia = a0 + da, ib = b0 + db;
      const double w = (da ? wa : 1. - wa) * (db ? wb : 1. - wb);
      if (ia < 0 || ia >= HX_NTR || ib < 0 || ib >= HX_NTM) continue;
      s += w * t[ia * HX_NTM + ib];
    }
  return s;
}

/* ---------------------------------------------------------------------- */
/* recomb_functions.py                                                     */
/* ---------------------------------------------------------------------- */
static double alpha_H(double Tm) {                       /* :31-50 */
  const double TK = Tm / HX_KB;
  return 1.0 * 4.309e-13 * pow(1.0e-4 * TK, -0.6166) / (1. + 0.6703 * pow(1.0e-4 * TK, 0.5300));
}

static double beta_H(double T) {                         /* :52-70 */
  const double ldb = 2. * HX_PI * HX_HBAR * HX_C / sqrt(2. * HX_PI * HX_MU_E * T);
  const double il = 1. / ldb;
  return il * il * il * exp(-HX_RYD / 4. / T) * alpha_H(T) / 4.;
}

static double gamma_compton(double xe, double T, double YHe) {   /* :100-125 */
  const double FHe = YHe * HX_MH / HX_MHE / (1 - YHe);
  return xe / (1. + FHe + xe) * 8. * HX_SIGT * (4. * HX_STEF) * T * T * T * T / (3. * HX_ME);
}

static double xe_saha(double T, double nH, double* s_out) {      /* :127-150 */
  const double ge = pow(2. * HX_PI * HX_MU_E * T, 1.5) / pow(2. * HX_PI * HX_HBAR * HX_C, 3.) / nH;
  const double s = ge * exp(-HX_RYD / T);
  *s_out = s;
  return (sqrt(s * s + 4. * s) - s) / 2.;
}

typedef struct {
  double A2s, A2p, B2s, B2p, R2p2s, R2s2p;
} eff_t;

static void effective_coefficients(const hx_t* h, double T, double Tm, eff_t* e) {   /* :152-212 */
  const double ratio = Tm / T;
  const double iT = frac_index(log(T), log(HX_TR_MIN), log(HX_TR_MAX), HX_NTR);
  const double iR = frac_index(ratio, HX_TRATIO_MIN, HX_TRATIO_MAX, HX_NTM);
  e->A2s = exp(bilinear(h->logA[0], iT, iR));
  e->A2p = exp(bilinear(h->logA[1], iT, iR));
  const double E2 = -HX_RYD / 4.;
  const double q = pow(2 * HX_PI * HX_MU_E * T / ((2 * HX_PI * HX_HBAR) * (2 * HX_PI * HX_HBAR)), 1.5) /
                   (HX_C * HX_C * HX_C);
  e->B2s = exp(E2 / T) * q * exp(bilinear(h->logA[0], iT, (double)(HX_NTM - 1)));
  e->B2p = (1. / 3.) * exp(E2 / T) * q * exp(bilinear(h->logA[1], iT, (double)(HX_NTM - 1)));
  e->R2p2s = exp(interp_uniform(log(T), log(HX_TR_MIN), log(HX_TR_MAX), HX_NTR, h->logR));
  e->R2s2p = 3. * e->R2p2s;
}

static double peebles_C(const hx_t* h, double z, double xHII, double H, double nH) {   /* :72-98 */
  const double cl = HX_C / HX_LYA_FREQ;
  const double rate_2p1s_x1s = 8 * HX_PI * H / (3 * (nH * cl * cl * cl));
  const double rate_exc = 3. * rate_2p1s_x1s / 4. + (1. - xHII) * HX_R2S1S / 4.;
  const double rate_ion = (1 - xHII) * beta_H(ri_T(h, dc(log(1 / (1 + z)))).v);
  return rate_exc / (rate_exc + rate_ion);
}

/* ---------------------------------------------------------------------- */
/* hydrogen.py: the effective multilevel atom                              */
/* ---------------------------------------------------------------------- */

/* HyRec-2 correction function (hydrogen.py:538-575) */
static double correction_delta(const hx_t* h, double T) {
  const double* sw = h->tab->swift;
  const int ns = h->tab->n_swift;
  const double* xs = h->swift_x;
  double col[4];
  for (int k = 0; k < 4; ++k) {
    /* jnp.interp on the (increasing) temperature column */
    double v;
    if (T <= xs[0]) v = sw[k + 1];
    else if (T >= xs[ns - 1]) v = sw[(ns - 1) * 5 + k + 1];
    else {
      int lo = 0, hi = ns - 1;
      while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (xs[mid] <= T) lo = mid; else hi = mid;
      }
      v = sw[lo * 5 + k + 1] + (T - xs[lo]) / (xs[hi] - xs[lo]) * (sw[hi * 5 + k + 1] - sw[lo * 5 + k + 1]);
    }
    col[k] = v;
  }
  const double omega_H = h->omega_b * (1 - h->YHe);
  const double omega_cb = h->omega_b + h->omega_cdm;
  return col[0] + (omega_cb - 0.14175) * col[1] + (omega_H - 0.01689) * col[2] + (h->Neff - 3.046) * col[3];
}

/* dx_e/dlna of the effective multilevel atom (hydrogen.py:497-536, the
 * steady-state 2s/2p equations :577-636, Lyman-alpha escape :638-662), as a
 * dual number in x_e */
static dl dxe_dlna_twophoton(const hx_t* h, dl xe, double T, double Tm, double H, double nH, double Delta) {
  eff_t e;
  effective_coefficients(h, T, Tm, &e);
  const dl x1s = dsub(dc(1.), xe);
  const double lam = 2. * HX_PI * HX_HBAR * HX_C / HX_RYD * 4. / 3.;
  const dl RLya = ddiv(dc(8. * HX_PI * H / 3. / nH), dsc(x1s, lam * lam * lam));
  const dl R2p1s = dsc(RLya, 1. / (1. + Delta));
  const double R1s2s = exp(-HX_E21 / T) * HX_R2S1S;
  const dl R1s2p = dsc(R2p1s, 3. * exp(-HX_E21 / T));
  const dl T00 = dc(e.B2s + e.R2s2p + HX_R2S1S);
  const dl T01 = dc(-e.R2p2s);
  const dl T10 = dc(-e.R2s2p);
  const dl T11 = dadd(dc(e.B2p + e.R2p2s), R2p1s);
  const dl xe2n = dsc(dmul(xe, xe), nH);
  const dl S0 = dadd(dsc(xe2n, e.A2s), dsc(x1s, R1s2s));
  const dl S1 = dadd(dsc(xe2n, e.A2p), dmul(x1s, R1s2p));
  /* jnp.linalg.solve of the 2 x 2 system */
  const dl det = dsub(dmul(T00, T11), dmul(T01, T10));
  const dl x2s = ddiv(dsub(dmul(S0, T11), dmul(T01, S1)), det);
  const dl x2p = ddiv(dsub(dmul(T00, S1), dmul(T10, S0)), det);
  const dl num = dsub(dadd(dsc(x2s, e.B2s), dsc(x2p, e.B2p)), dsc(xe2n, e.A2s + e.A2p));
  return dsc(num, 1. / H);
}

/* ---------------------------------------------------------------------- */
/* helium.py                                                               */
/* ---------------------------------------------------------------------- */
static double fHe_of(const hx_t* h) { return h->YHe / (1. - h->YHe) / 3.97153; }

static dl xHeII_post_saha(const hx_t* h, dl lna) {      /* helium.py:235-264 */
  const double fHe = fHe_of(h);
  const dl TK = dsc(ri_T(h, lna), 1. / HX_KB);
  const dl nH = ri_nH(h, lna);
  const dl s = ddiv(dmul(dmul(dsc(TK, 4 * 2.414194e15), dsqrt_(TK)), dexp_(drs(-285325., TK))), nH);
  const dl ops = dadd(dc(1.), s);
  const dl inner = dadd(dc(1.), ddiv(dsc(s, 4. * fHe), dmul(ops, ops)));
  return ddiv(ddiv(dsc(s, 2. * fHe), ops), dadd(dc(1.), dsqrt_(inner)));
}

static dl xH1_saha(const hx_t* h, dl lna) {              /* helium.py:266-295 */
  const dl xHeII = xHeII_post_saha(h, lna);
  const dl TK = dsc(ri_T(h, lna), 1. / HX_KB);
  const dl nH = ri_nH(h, lna);
  const dl s = ddiv(dmul(dmul(dsc(TK, 2.4127161187130e15), dsqrt_(TK)), dexp_(drs(-157801.37882, TK))), nH);
  if (s.v > 1e5) {
    const dl a = ddiv(dadd(dc(1.), xHeII), s);
    const dl b = ddiv(dadd(dadd(dmul(xHeII, xHeII), dsc(xHeII, 3.)), dc(2.)), dmul(s, s));
    return dsub(a, b);
  }
  if (s.v == 0.) return dc(1.);
  const dl u = dadd(dc(1.), ddiv(xHeII, s));
  const dl root = dsqrt_(dadd(dmul(u, u), drs(4., s)));
  return dsub(dc(1.), ddiv(dc(2.), dadd(u, root)));
}

/* dx_HeII/dlna (helium.py:375-453), dual in x_e and lna */
static dl helium_dxHeIIdlna(const hx_t* h, dl xe, dl lna) {
  const double fHe = fHe_of(h);
  const dl T = ri_T(h, lna);
  const dl nH = ri_nH(h, lna);
  const dl H = ri_H(h, lna);
  const dl xH1 = xH1_saha(h, lna);
  const dl xHeII = dsub(xe, dsub(dc(1.), xH1));
  const dl TK = dsc(T, 1. / HX_KB);
  const dl s0 = dsc(ddiv(dmul(dsc(TK, 2.414194e15), dsqrt_(TK)), nH), 4.);
  const dl s = dmul(s0, dexp_(drs(-285325., TK)));
  const dl y2s = ddiv(dexp_(drs(46090., TK)), s0);
  const dl y2p = dsc(ddiv(dexp_(drs(39101., TK)), s0), 3.);
  const dl etacinv = ddiv(dsc(H, 9.15776e22), dmul(nH, xH1));
  static const double gA[7] = {1.976e6, 6.03e6, 1.06e8, 2.18e6, 3.37e7, 1.04e6, 1.51e7};
  static const double gE[7] = {6989., 19754., 21539., 28496., 29224., 32414., 32781.};
  dl g2pinc = ddiv(dc(gA[0]), dsub(dc(1.), dexp_(drs(-gE[0], TK))));
  for (int i = 1; i < 7; ++i) g2pinc = dadd(g2pinc, ddiv(dc(gA[i]), dsub(dexp_(drs(gE[i], TK)), dc(1.))));
  const dl tau2p = dmul(dsc(ddiv(nH, H), 4.277e-8), dsub(dc(fHe), xHeII));
  const dl dnuline = dsc(dmul(g2pinc, tau2p), 1. / (4 * HX_PI * HX_PI));
  const dl tauc = ddiv(dnuline, etacinv);
  const dl enh = dadd(dsqrt_(dadd(dc(1.), dsc(tauc, HX_PI * HX_PI))),
                      ddiv(dsc(tauc, 7.74), dadd(dc(1.), dsc(tauc, 70.))));
  dl pesc = ddiv(enh, tau2p);
  const dl a = dsub(dc(1.), dexp_(dsc(tau2p, -1.023e-7)));
  const dl b = dsub(dsc(dexp_(drs(2947., TK)), 0.964525), dmul(enh, dexp_(drs(-6.14e13, etacinv))));
  pesc = dadd(pesc, ddiv(dmul(a, b), tau2p));
  const dl ydown = dadd(dsc(y2s, 50.94), dmul(dsc(y2p, 1.7989e9), pesc));
  const dl bracket = dsub(dmul(dsub(dc(fHe), xHeII), s), dmul(xHeII, dsub(dadd(xHeII, dc(1.)), xH1)));
  return ddiv(dmul(ydown, bracket), H);
}

/* The two rates whose jax.grad derivatives the post-Saha expansions take,
 * with their forward-mode derivatives: out[0..1] = helium_dxHeIIdlna and its
 * derivative in x_e (at xe_he, lna), out[2..3] = its derivative in lna and
 * xHeII_post_Saha's, out[4..5] = dxe_dlna_twophoton(xe_h, T, Tm = T, H, n_H,
 * Delta = 0) and its derivative in x_e (T, H, n_H from the inputs at lna),
 * out[6] = xHeII_post_Saha.  For tests: the derivatives against finite
 * differences. */
int oracle_hyrex_rates(const oracle_hyrex_tables* tab, int n_grid, const double* TCMB, const double* nH,
                       const double* H, double YHe, double omega_b, double omega_cdm, double Neff, double lna,
                       double xe_he, double xe_h, double* out) {
  hx_t* h = (hx_t*)calloc(1, sizeof(hx_t));
  h->tab = tab;
  for (int i = 0; i < HX_NTR * HX_NTM; ++i) {
    h->logA[0][i] = log(tab->alpha[i * 4 + 0]);
    h->logA[1][i] = log(tab->alpha[i * 4 + 1]);
  }
  for (int i = 0; i < HX_NTR; ++i) h->logR[i] = log(tab->R[i]);
  h->swift_x = (double*)malloc(sizeof(double) * (tab->n_swift > 0 ? tab->n_swift : 1));
  for (int i = 0; i < tab->n_swift; ++i) h->swift_x[i] = HX_KB * tab->swift[i * 5];
  h->n = n_grid;
  h->l0 = -log(1. + HX_Z0);
  h->l1 = h->l0 + (double)(n_grid - 1) * HX_SPACING;
  h->T = TCMB;
  h->nH = nH;
  h->H = H;
  h->YHe = YHe;
  h->omega_b = omega_b;
  h->omega_cdm = omega_cdm;
  h->Neff = Neff;
  const dl a = helium_dxHeIIdlna(h, (dl){xe_he, 1.}, dc(lna));
  const dl b = helium_dxHeIIdlna(h, dc(xe_he), (dl){lna, 1.});
  const dl c = xHeII_post_saha(h, (dl){lna, 1.});
  const double T = ri_T(h, dc(lna)).v, n = ri_nH(h, dc(lna)).v, Hv = ri_H(h, dc(lna)).v;
  const dl d = dxe_dlna_twophoton(h, (dl){xe_h, 1.}, T, T, Hv, n, 0.0);
  out[0] = a.v;
  out[1] = a.d;
  out[2] = b.d;
  out[3] = c.d;
  out[4] = d.v;
  out[5] = d.d;
  out[6] = c.v;
  free(h->swift_x);
  free(h);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Kvaerno3 (Kvaerno, BIT 44 (2004): ESDIRK 3(2), four stages, L-stable    */
/* gamma, stiffly accurate, embedded solution = stage 3)                   */
/* ---------------------------------------------------------------------- */
#define KV3_G 0.43586652150
static double kv3_a[4][4], kv3_c[4], kv3_b[4], kv3_be[4];

static void kv3_init(void) {
  const double g = KV3_G;
  memset(kv3_a, 0, sizeof(kv3_a));
  kv3_a[1][0] = g;
  kv3_a[2][0] = (-4 * g * g + 6 * g - 1) / (4 * g);
  kv3_a[2][1] = (-2 * g + 1) / (4 * g);
  kv3_a[3][0] = (6 * g - 1) / (12 * g);
  kv3_a[3][1] = -1 / ((24 * g - 12) * g);
  kv3_a[3][2] = (-6 * g * g + 6 * g - 1) / (6 * g - 3);
  kv3_c[0] = 0.;
  kv3_c[1] = 2 * g;
  kv3_c[2] = 1.;
  kv3_c[3] = 1.;
  for (int j = 0; j < 3; ++j) kv3_b[j] = kv3_a[3][j];
  kv3_b[3] = g;
  for (int j = 0; j < 2; ++j) kv3_be[j] = kv3_a[2][j];
  kv3_be[2] = g;
  kv3_be[3] = 0.;
}

void oracle_kvaerno3_tableau(double* A16, double* c4, double* b4, double* be4) {
  kv3_init();
  for (int i = 0; i < 4; ++i) {
    for (int j = 0; j < 4; ++j) A16[i * 4 + j] = kv3_a[i][j];
    if (i > 0) A16[i * 4 + i] = KV3_G;
    c4[i] = kv3_c[i];
    b4[i] = kv3_b[i];
    be4[i] = kv3_be[i];
  }
}

typedef void (*hx_rhs)(const hx_t* h, double t, const double* y, double* f);
typedef int (*hx_event)(const hx_t* h, double t, const double* y);

/* diffeqsolve(ODETerm(F), Kvaerno3(), t0, t1 = inf, dt0 = 1e-3, y0,
 * PIDController(rtol, atol), SaveAt(ts = t0 + spacing * (1..n_save)),
 * Event(E), max_steps) for a state of m <= 2 components.  ts_out / ys_out
 * [n_save] (ys_out [n_save][m]) must hold +inf on entry; the saved grid
 * points are written.  Returns an ABCMB_STATUS_* code. */
static int kv3_solve(const hx_t* h, hx_rhs F, hx_event E, int m, double t0, const double* y0, double rtol,
                     double atol, int max_steps, int n_save, double* ts_out, double* ys_out, int* n_saved,
                     int* n_steps) {
  const double g = KV3_G;
  const double err_order = 3.0, safety = 0.9, factormin = 0.2, factormax = 10.0;
  const double coeff1 = 1.0 / err_order;     /* pcoeff 0, icoeff 1, dcoeff 0 */
  const double kappa = 1e-2, small_res = 1e-13;
  const int root_max = 10;
  const double t_first = t0 + HX_SPACING, t_last = t0 + (double)n_save * HX_SPACING;
  const double tstep = (t_last - t_first) / (double)(n_save - 1);
  double y[2], y1[2], Fs[4][2], v[2], r[2], base[2];
  for (int j = 0; j < m; ++j) y[j] = y0[j];
  double t = t0, t1 = t0 + 1e-3;
  F(h, t, y, Fs[0]);
  int isave = 0, nsteps = 0, status = ABCMB_STATUS_OK;
  for (;;) {
    if (nsteps >= max_steps) { status = ABCMB_STATUS_MAX_STEPS; break; }
    nsteps++;
    const double hs = t1 - t;
    const double hg = hs * g;
    /* very chord: Jacobian of F once per step, at the first implicit stage's
     * starting point, by central differences */
    double J[2][2], Minv[2][2];
    {
      double z[2], fp[2], fm[2];
      for (int j = 0; j < m; ++j) z[j] = y[j] + hs * (kv3_a[1][0] + g) * Fs[0][j];
      const double tz = t + kv3_c[1] * hs;
      for (int col = 0; col < m; ++col) {
        const double d = 1e-7 * (fabs(z[col]) > 1e-8 ? fabs(z[col]) : 1e-8);
        double zp[2] = {z[0], m > 1 ? z[1] : 0.}, zm[2] = {z[0], m > 1 ? z[1] : 0.};
        zp[col] += d;
        zm[col] -= d;
        F(h, tz, zp, fp);
        F(h, tz, zm, fm);
        for (int row = 0; row < m; ++row) J[row][col] = (fp[row] - fm[row]) / (2. * d);
      }
      double M[2][2];
      for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b) M[a][b] = (a == b ? 1. : 0.) - hg * J[a][b];
      if (m == 1) {
        Minv[0][0] = 1. / M[0][0];
      } else {
        const double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        Minv[0][0] = M[1][1] / det;
        Minv[0][1] = -M[0][1] / det;
        Minv[1][0] = -M[1][0] / det;
        Minv[1][1] = M[0][0] / det;
      }
    }
    int ok = 1;
    for (int i = 1; i < 4 && ok; ++i) {
      const double ti = t + kv3_c[i] * hs;
      for (int j = 0; j < m; ++j) {
        double acc = 0.;
        for (int k = 0; k < i; ++k) acc += kv3_a[i][k] * Fs[k][j];
        base[j] = y[j] + hs * acc;
        Fs[i][j] = Fs[i - 1][j];                          /* starting guess: previous stage */
      }
      double diffsize = INFINITY, diffsize_prev;
      int conv = 0;
      for (int it = 1; it <= root_max; ++it) {
        for (int j = 0; j < m; ++j) v[j] = base[j] + hg * Fs[i][j];
        double fv[2];
        F(h, ti, v, fv);
        for (int j = 0; j < m; ++j) r[j] = fv[j] - Fs[i][j];
        double ss = 0.;
        double dx[2];
        for (int a = 0; a < m; ++a) {
          dx[a] = 0.;
          for (int b = 0; b < m; ++b) dx[a] += Minv[a][b] * r[b];
        }
        for (int j = 0; j < m; ++j) {
          Fs[i][j] += dx[j];
          const double q = dx[j] / (atol + rtol * fabs(Fs[i][j]));
          ss += q * q;
        }
        diffsize_prev = diffsize;
        diffsize = sqrt(ss / m);
        if (it >= 2) {
          const double rate = diffsize / diffsize_prev;
          const double factor = diffsize * rate / (1. - rate);
          const int small = diffsize < small_res;
          const int diverged = !isfinite(rate) || rate > 2.;
          const int converged = factor > 0. && factor < kappa;
          if (small || converged) { conv = 1; break; }
          if (diverged) break;
        }
      }
      if (!conv) ok = 0;
    }
    double scaled = INFINITY;
    if (ok) {
      double ss = 0.;
      for (int j = 0; j < m; ++j) {
        double acc = 0., acce = 0.;
        for (int k = 0; k < 4; ++k) {
          acc += kv3_b[k] * Fs[k][j];
          acce += (kv3_b[k] - kv3_be[k]) * Fs[k][j];
        }
        y1[j] = y[j] + hs * acc;
        const double err = hs * acce;
        const double sc = atol + rtol * (fabs(y[j]) > fabs(y1[j]) ? fabs(y[j]) : fabs(y1[j]));
        ss += (err / sc) * (err / sc);
      }
      scaled = sqrt(ss / m);
      if (!isfinite(scaled)) scaled = INFINITY;
    }
    const int keep = scaled < 1.0;
    double inv = 1.0 / scaled;
    double factor = safety * pow(inv, coeff1);
    const double fmn = keep ? 1.0 : factormin;
    if (factor < fmn) factor = fmn;
    if (factor > factormax) factor = factormax;
    const double dt_new = hs * factor;
    if (keep) {
      /* SaveAt(ts): the grid points inside the step, cubic Hermite */
      while (isave < n_save) {
        const double ts = (isave == n_save - 1) ? t_last : t_first + (double)isave * tstep;
        if (!(ts <= t1)) break;
        const double th = (ts - t) / hs;
        for (int j = 0; j < m; ++j) {
          const double k0 = hs * Fs[0][j], k1 = hs * Fs[3][j];
          const double a = k0 + k1 + 2. * y[j] - 2. * y1[j];
          const double b = -2. * k0 - k1 - 3. * y[j] + 3. * y1[j];
          ys_out[isave * m + j] = ((a * th + b) * th + k0) * th + y[j];
        }
        ts_out[isave] = ts;
        isave++;
      }
      t = t1;
      for (int j = 0; j < m; ++j) {
        y[j] = y1[j];
        Fs[0][j] = Fs[3][j];                               /* FSAL */
      }
      if (E(h, t, y)) break;                               /* Event: ends at this step */
      if (isave >= n_save) break;                          /* nothing left to save */
    }
    t1 = t + dt_new;
    if (!(hs > 1e-14) || !isfinite(t1)) { status = ABCMB_STATUS_DT_UNDERFLOW; break; }
  }
  *n_saved = isave;
  *n_steps = nsteps;
  return status;
}

/* ---------------------------------------------------------------------- */
/* the ODE phases' right-hand sides and events                             */
/* ---------------------------------------------------------------------- */
static void rhs_HeII(const hx_t* h, double t, const double* y, double* f) {   /* helium.py:455-483 */
  const dl lna = dc(t);
  const dl xe = dadd(dc(y[0]), xH1_saha(h, lna));
  f[0] = helium_dxHeIIdlna(h, xe, lna).v;
}
static int ev_HeII(const hx_t* h, double t, const double* y) {               /* helium.py:531-538 */
  const double xH1 = xH1_saha(h, dc(t)).v;
  return y[0] - (1. - xH1) < 1e-4;
}

static void rhs_twophoton(const hx_t* h, double t, const double* y, double* f) {   /* hydrogen.py:278-313 */
  const double T = ri_T(h, dc(t)).v, nH = ri_nH(h, dc(t)).v, H = ri_H(h, dc(t)).v;
  const double GC = gamma_compton(y[0], T, h->YHe);
  const double Tm = T * (1. - H / GC);
  const double Delta = correction_delta(h, T);
  f[0] = dxe_dlna_twophoton(h, dc(y[0]), T, Tm, H, nH, Delta).v;
}
static int ev_twophoton(const hx_t* h, double t, const double* y) {          /* hydrogen.py:365-367 */
  (void)y;
  return t > h->twog_end;
}

static void rhs_emla(const hx_t* h, double t, const double* y, double* f) {  /* hydrogen.py:385-419 */
  const double T = ri_T(h, dc(t)).v, nH = ri_nH(h, dc(t)).v, H = ri_H(h, dc(t)).v;
  const double GC = gamma_compton(y[0], T, h->YHe);
  f[0] = dxe_dlna_twophoton(h, dc(y[0]), T, y[1], H, nH, 0.0).v;
  f[1] = (-2 * H * y[1] + GC * (T - y[1])) / H;
}
static int ev_emla(const hx_t* h, double t, const double* y) {               /* hydrogen.py:470-478 */
  const double T = ri_T(h, dc(t)).v;
  const double ratio = y[1] / T < T / y[1] ? y[1] / T : T / y[1];
  return T < HX_TR_MIN || ratio < HX_TRATIO_MIN;
}

static void rhs_tla(const hx_t* h, double t, const double* y, double* f) {   /* hydrogen.py:664-702 */
  const double xe = y[0], Tm = y[1];
  const double nH = ri_nH(h, dc(t)).v, T = ri_T(h, dc(t)).v, H = ri_H(h, dc(t)).v;
  const double C = peebles_C(h, exp(-t) - 1.0, xe, H, nH);
  const double dxe_dt = C * (beta_H(Tm) * (1.0 - xe) - alpha_H(Tm) * nH * xe * xe);
  f[0] = dxe_dt / H;
  f[1] = -2.0 * Tm + (gamma_compton(xe, T, h->YHe) / H) * (T - Tm);
}
static int ev_tla(const hx_t* h, double t, const double* y) {                /* hydrogen.py:749-751 */
  (void)h; (void)y;
  return t > 0.0;                                                           /* lna_end = -log(1 + z1), z1 = 0 */
}

/* ---------------------------------------------------------------------- */
/* the whole history                                                       */
/* ---------------------------------------------------------------------- */
typedef struct {
  double* a;      /* the joined array */
  int valid;      /* finite entries so far */
  int len;        /* total length so far (array_with_padding keeps every buffer's length) */
  int cap;
} joined_t;

static int join_append(joined_t* J, const double* seg, int seg_valid, int seg_len) {
  if (J->valid + seg_len > J->cap) return -1;
  for (int i = 0; i < seg_len; ++i) J->a[J->valid + i] = i < seg_valid ? seg[i] : INFINITY;
  J->valid += seg_valid;
  J->len += seg_len;
  return 0;
}

int oracle_hyrex_sizes(int n_grid, int* n_xe, int* n_tm) {
  const double l0 = -log(1. + HX_Z0);
  int n1 = 0;
  for (int i = 0; i < n_grid; ++i)
    if (l0 + (double)i * HX_SPACING <= -log(HX_Z_HE_EQUIL)) n1++;
  *n_xe = n1 + HX_N_POST_HE + HX_N_HE_ODE + HX_N_POST_H + 3 * HX_N_LATE;
  *n_tm = 2 * HX_N_LATE;
  return n1;
}

int oracle_hyrex(const oracle_hyrex_tables* tab, int n_grid, const double* TCMB, const double* nH,
                 const double* H, double YHe, double omega_b, double omega_cdm, double Neff, double* xe_out,
                 double* lna_out, int cap_xe, double* tm_out, double* lna_tm_out, int cap_tm, int* info) {
  kv3_init();
  hx_t* h = (hx_t*)calloc(1, sizeof(hx_t));
  h->tab = tab;
  for (int i = 0; i < HX_NTR * HX_NTM; ++i) {
    h->logA[0][i] = log(tab->alpha[i * 4 + 0]);
    h->logA[1][i] = log(tab->alpha[i * 4 + 1]);
  }
  for (int i = 0; i < HX_NTR; ++i) h->logR[i] = log(tab->R[i]);
  h->swift_x = (double*)malloc(sizeof(double) * (tab->n_swift > 0 ? tab->n_swift : 1));
  for (int i = 0; i < tab->n_swift; ++i) h->swift_x[i] = HX_KB * tab->swift[i * 5];
  h->n = n_grid;
  h->l0 = -log(1. + HX_Z0);
  h->l1 = h->l0 + (double)(n_grid - 1) * HX_SPACING;
  h->T = TCMB;
  h->nH = nH;
  h->H = H;
  h->YHe = YHe;
  h->omega_b = omega_b;
  h->omega_cdm = omega_cdm;
  h->Neff = Neff;
  int n_xe_len, n_tm_len;
  const int n1 = oracle_hyrex_sizes(n_grid, &n_xe_len, &n_tm_len);
  memset(info, 0, sizeof(int) * 16);
  if (cap_xe < n_xe_len || cap_tm < n_tm_len || n1 < 2 || tab->n_swift < 2) {
    free(h->swift_x);
    free(h);
    return ABCMB_ERR_ARG;
  }
  for (int i = 0; i < cap_xe; ++i) xe_out[i] = lna_out[i] = INFINITY;
  for (int i = 0; i < cap_tm; ++i) tm_out[i] = lna_tm_out[i] = INFINITY;
  joined_t X = {xe_out, 0, 0, cap_xe}, L = {lna_out, 0, 0, cap_xe};
  joined_t TM = {tm_out, 0, 0, cap_tm}, LT = {lna_tm_out, 0, 0, cap_tm};
  const int nbuf = HX_N_LATE * 2;
  double* sx = (double*)malloc(sizeof(double) * nbuf * 2);   /* also the (x_e, T_m) pairs of phases 6-7 */
  double* sl = (double*)malloc(sizeof(double) * nbuf);
  const double fHe = fHe_of(h);
  int status = ABCMB_STATUS_OK, nsv = 0, nst = 0;

  /* 1 Saha HeII/III (helium.py:156-233) */
  {
    int k = 0;
    for (; k < n1; ++k) {
      const double l = h->l0 + (double)k * HX_SPACING;
      const double T = ri_T(h, dc(l)).v, nHv = ri_nH(h, dc(l)).v;
      const double TK = T / HX_KB;
      const double s = 2.414194e15 * TK * sqrt(TK) * exp(-631462.7 / TK) / nHv;
      const double xHeIII = 2 * s * fHe / (1 + s + fHe) / (1 + sqrt(1 + 4 * s * fHe / ((1 + s + fHe) * (1 + s + fHe))));
      sx[k] = 1 + fHe + xHeIII;
      sl[k] = l;
      if (xHeIII < 1e-9) { k++; break; }
    }
    join_append(&X, sx, k, n1);
    join_append(&L, sl, k, n1);
    info[0] = k;
  }
  /* 2 post-Saha HeII (helium.py:297-373) */
  {
    const double start = L.a[L.valid - 1] + HX_SPACING;
    int k = 0;
    for (; k < HX_N_POST_HE; ++k) {
      const double l = start + (double)k * HX_SPACING;
      const double xHeII = xHeII_post_saha(h, dc(l)).v;
      const double xH1 = xH1_saha(h, dc(l)).v;
      const double xs = 1 - xH1 + xHeII;
      const dl gx = helium_dxHeIIdlna(h, (dl){xs, 1.}, dc(l));          /* d/dxe */
      const dl gl = xHeII_post_saha(h, (dl){l, 1.});                     /* d/dlna */
      const double x = xs + gl.d / gx.d;
      sx[k] = x;
      sl[k] = l;
      if (fabs(xs - x) > 1e-5) { k++; break; }
    }
    join_append(&X, sx, k, HX_N_POST_HE);
    join_append(&L, sl, k, HX_N_POST_HE);
    info[1] = k;
  }
  /* 3 HeII ODE (helium.py:485-565) */
  {
    const double t0 = L.a[L.valid - 1];
    const double y0[1] = {X.a[X.valid - 1]};
    for (int i = 0; i < HX_N_HE_ODE; ++i) sx[i] = sl[i] = INFINITY;
    status = kv3_solve(h, rhs_HeII, ev_HeII, 1, t0, y0, 1e-6, 1e-9, 4096, HX_N_HE_ODE, sl, sx, &nsv, &nst);
    join_append(&X, sx, nsv, HX_N_HE_ODE);
    join_append(&L, sl, nsv, HX_N_HE_ODE);
    info[2] = nsv;
    info[8] = nst;
    if (status != ABCMB_STATUS_OK) goto done;
  }
  /* 4 post-Saha H (hydrogen.py:190-276) */
  {
    const double start = L.a[L.valid - 1] + HX_SPACING;
    int k = 0;
    for (; k < HX_N_POST_H; ++k) {
      const double l = start + (double)k * HX_SPACING;
      const double T = ri_T(h, dc(l)).v, nHv = ri_nH(h, dc(l)).v, Hv = ri_H(h, dc(l)).v;
      double s;
      const double xs = xe_saha(T, nHv, &s);
      const double dxs = -(HX_RYD / T - 3. / 2.) * xs * xs / (2. * xs + s);
      const dl gx = dxe_dlna_twophoton(h, (dl){xs, 1.}, T, T, Hv, nHv, 0.0);
      const double x = xs + dxs / gx.d;
      sx[k] = x;
      sl[k] = l;
      if (fabs(xs - x) > 1e-5) { k++; break; }
    }
    join_append(&X, sx, k, HX_N_POST_H);
    join_append(&L, sl, k, HX_N_POST_H);
    info[3] = k;
  }
  /* 5 two-photon EMLA to z = 700 (hydrogen.py:315-383) */
  {
    const double t0 = L.a[L.valid - 1];
    const double y0[1] = {X.a[X.valid - 1]};
    h->twog_end = -log(HX_Z_TWOG);
    for (int i = 0; i < HX_N_LATE; ++i) sx[i] = sl[i] = INFINITY;
    status = kv3_solve(h, rhs_twophoton, ev_twophoton, 1, t0, y0, 1e-6, 1e-9, 4096, HX_N_LATE, sl, sx, &nsv, &nst);
    join_append(&X, sx, nsv, HX_N_LATE);
    join_append(&L, sl, nsv, HX_N_LATE);
    info[4] = nsv;
    info[9] = nst;
    if (status != ABCMB_STATUS_OK) goto done;
  }
  /* 6 EMLA with T_m (hydrogen.py:421-495; called with rtol 1e-6, Kvaerno3) */
  {
    double* s2 = sx;
    const double t0 = L.a[L.valid - 1];
    const double x0 = X.a[X.valid - 1];
    const double T0 = ri_T(h, dc(t0)).v;
    const double y0[2] = {x0, T0 * (1. - ri_H(h, dc(t0)).v / gamma_compton(x0, T0, YHe))};
    for (int i = 0; i < HX_N_LATE; ++i) sl[i] = INFINITY;
    for (int i = 0; i < 2 * HX_N_LATE; ++i) s2[i] = INFINITY;
    status = kv3_solve(h, rhs_emla, ev_emla, 2, t0, y0, 1e-6, 1e-9, 4096, HX_N_LATE, sl, s2, &nsv, &nst);
    double* xcol = (double*)malloc(sizeof(double) * HX_N_LATE);
    double* tcol = (double*)malloc(sizeof(double) * HX_N_LATE);
    for (int i = 0; i < HX_N_LATE; ++i) { xcol[i] = s2[2 * i]; tcol[i] = s2[2 * i + 1]; }
    join_append(&X, xcol, nsv, HX_N_LATE);
    join_append(&L, sl, nsv, HX_N_LATE);
    join_append(&TM, tcol, nsv, HX_N_LATE);
    join_append(&LT, sl, nsv, HX_N_LATE);
    free(xcol);
    free(tcol);
    info[5] = nsv;
    info[10] = nst;
    if (status != ABCMB_STATUS_OK) goto done;
  }
  if (LT.valid < 1) { status = ABCMB_STATUS_NONFINITE; goto done; }   /* no T_m point to start from */
  /* 7 three-level atom to lna = 0 (hydrogen.py:704-780) */
  {
    double* s2 = sx;
    const double t0 = LT.a[LT.valid - 1];
    const double y0[2] = {X.a[X.valid - 1], TM.a[TM.valid - 1]};
    for (int i = 0; i < HX_N_LATE; ++i) sl[i] = INFINITY;
    for (int i = 0; i < 2 * HX_N_LATE; ++i) s2[i] = INFINITY;
    status = kv3_solve(h, rhs_tla, ev_tla, 2, t0, y0, 1e-7, 1e-9, 4096, HX_N_LATE, sl, s2, &nsv, &nst);
    double* xcol = (double*)malloc(sizeof(double) * HX_N_LATE);
    double* tcol = (double*)malloc(sizeof(double) * HX_N_LATE);
    for (int i = 0; i < HX_N_LATE; ++i) { xcol[i] = s2[2 * i]; tcol[i] = s2[2 * i + 1]; }
    join_append(&X, xcol, nsv, HX_N_LATE);
    join_append(&L, sl, nsv, HX_N_LATE);
    join_append(&TM, tcol, nsv, HX_N_LATE);
    join_append(&LT, sl, nsv, HX_N_LATE);
    free(xcol);
    free(tcol);
    info[6] = nsv;
    info[11] = nst;
  }
done:
  info[12] = X.len;
  info[13] = TM.len;
  info[14] = status;
  free(sx);
  free(sl);
  free(h->swift_x);
  free(h);
  return status == ABCMB_STATUS_OK ? ABCMB_OK : ABCMB_ERR_SOLVER;
}
