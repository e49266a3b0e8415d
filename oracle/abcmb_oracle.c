/*
 * abcmb_oracle.c -- CPU FP64 restatement of ABCMB's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA kernels are
 * compared against (tests/, __graft_entry__.smoke) and the timed CPU
 * baseline (bench.py cpu_baseline / --impl reference).  Nothing in the
 * product path (abcmb_b200/) loads or calls it.
 *
 * It follows the reference line by line, in plain C with straightforward
 * data structures (dense Jacobian, dense LU with partial pivoting -- the
 * reference builds the Jacobian with JAX autodiff and solves it with a dense
 * LU through lineax):
 *   constants            abcmb/constants.py:8-39
 *   fast_interp          abcmb/ABCMBTools.py:268-308
 *   jnp.interp           numpy.interp semantics (perturbations.py:150,155)
 *   species rho / P      abcmb/species.py:454-1346
 *   background           abcmb/background.py:101-187 (rho_tot, H, aH,
 *                        aH_prime), 321-387 (tau, nH, TCMB), 568-680 (xe, Tm,
 *                        tau_c), hyrex/recomb_functions.py:127-153
 *   background tables    abcmb/background.py:252-319 (conformal-time table,
 *                        Kvaerno5 + PID, dense output), 682-720 (optical
 *                        depth), 552-564 (lna_rec, lna_transfer_start),
 *                        spectrum.py:640-651 (line-of-sight arrays)
 *   start time           abcmb/perturbations.py:119-159, 279
 *   initial conditions   abcmb/perturbations.py:161-199 + species y_ini
 *   RHS                  abcmb/perturbations.py:201-248 + species y_prime
 *   ODE solve            diffrax.diffeqsolve(Kvaerno5, PIDController,
 *                        SaveAt(ts)) as called at perturbations.py:285-312:
 *                        ESDIRK 5(4) tableau of Kvaerno (BIT 44, 2004), the
 *                        "very chord" stage solve (Jacobian once per step),
 *                        the PID step controller, cubic Hermite dense output.
 *   output table         abcmb/perturbations.py:318-404 + output_perturbations
 *   k resampling         interpax CubicSpline (not-a-knot, extrapolating),
 *                        spectrum.py:664-678
 *   sources              abcmb/spectrum.py:681-696
 *   line of sight        abcmb/spectrum.py:638-786 (phi0/1/2 with the large-x
 *                        asymptotic j_l of spectrum.py:48-51)
 *   k quadrature         abcmb/spectrum.py:789-796 (trapezoid)
 *   l spline             abcmb/spectrum.py:594-608
 *   Pk_lin               abcmb/spectrum.py:250-302
 *   lensing              abcmb/spectrum.py:349-572 (Limber C_l^phiphi, the
 *                        correlation-function lensed spectra) with the
 *                        Wigner-d recursion of abcmb/ABCMBTools.py:16-186
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/abcmb_b200.h"
#include "abcmb_oracle.h"

/* ---------------------------------------------------------------------- */
/* constants.py                                                            */
/* ---------------------------------------------------------------------- */
#define C_CM     29979245800.0
#define C_MPC    9.71561e-15
#define H0H      3.24078e-18
#define HBAR     6.582119569509e-16
#define GN       1.18980205e-40
#define MP       938271999.0
#define ME       510998.9461
#define MH       (MP + ME + 13.5982860719383)
#define MHE      3.72839e9
#define SIGT     6.652458734e-25
#define PI       3.14159265358979323846
#define STEF_BOLT (PI * PI / (60. * HBAR * HBAR * HBAR * C_CM * C_CM))
#define RHO_CRIT_UNIT (3. * H0H * H0H / 8. / PI / GN)

/* MassiveNeutrino quadratures (species.py:791-794) */
static const double Q3[3] = {0.913201, 3.37517, 7.79184};
static const double W3[3] = {0.0687359, 3.31435, 2.29911};
static const double Q5[5] = {0.583165, 2.0, 4.0, 7.26582, 13.0};
static const double W5[5] = {0.0081201, 0.689407, 2.8063, 2.05156, 0.12681};

/* ---------------------------------------------------------------------- */
/* interpolation helpers                                                   */
/* ---------------------------------------------------------------------- */

/* ABCMBTools.fast_interp (ABCMBTools.py:268-308). */
double oracle_fast_interp(double x, double xp_min, double xp_max, const double* fp, int n) {
  const double eps = 1.e-6;
  double i = (x - xp_min) / (xp_max - xp_min) * (double)(n - 1);
  if (i < eps) i = eps;
  if (i > (double)(n - 1) - eps) i = (double)(n - 1) - eps;
  int il = (int)floor(i);
  int iu = il + 1 < n - 1 ? il + 1 : n - 1;
  double wu = i - (double)il;
  double wl = 1.0 - wu;
  return wl * fp[il] + wu * fp[iu];
}

/* jnp.interp(x, xp, fp) for increasing xp (numpy semantics, clamped). */
double oracle_np_interp(double x, const double* xp, const double* fp, int n) {
  /* searchsorted(xp, x, side='right') */
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (xp[mid] <= x) lo = mid + 1; else hi = mid;
  }
  int i = lo;
  if (i < 1) i = 1;
  if (i > n - 1) i = n - 1;
  double df = fp[i] - fp[i - 1];
  double dx = xp[i] - xp[i - 1];
  double delta = x - xp[i - 1];
  double f;
  if (fabs(dx) <= 2.220446049250313e-16) f = fp[i - 1];
  else f = fp[i - 1] + (delta / dx) * df;
  if (x < xp[0]) f = fp[0];
  if (x > xp[n - 1]) f = fp[n - 1];
  return f;
}

/* jnp.linspace(a, b, n)[i] */
static double linspace_at(double a, double b, int n, int i) {
  if (i == n - 1) return b;
  return a + (double)i * ((b - a) / (double)(n - 1));
}

/* ---------------------------------------------------------------------- */
/* background                                                              */
/* ---------------------------------------------------------------------- */

typedef struct {
  double lna, a, aH, tau, xe, tau_c, Tm, TCMB, cs2, R;
  double rho_tot, P_tot;
  double rho_cdm, rho_b, rho_g, rho_nu, rho_ncdm, P_ncdm;
  double ncdm_T, ncdm_x, ncdm_fac;  /* N * 4/pi^2 T^4 / hbar^3 / c^3 */
  double eps3[3];
} bgs_t;

static double rho_ncdm_fn(const abcmb_cosmo* c, double lna, double* P_out) {
  double a = exp(lna);
  double T = c->T_nu_massive * c->TCMB0 / a;
  double x = c->m_nu_massive / T;
  double ir = 0., ip = 0.;
  for (int j = 0; j < 5; ++j) {
    double q = Q5[j];
    ir += (1. + exp(-q)) / (q * q) * sqrt(q * q + x * x) * W5[j];
    ip += (1. + exp(-q)) / sqrt(q * q + x * x) * W5[j];
  }
  double T4 = T * T * T * T;
  double rho = c->N_nu_massive * 4. * T4 / (PI * PI) * ir / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
  double P = c->N_nu_massive * 4. / 3. * T4 / (PI * PI) * ip / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
  if (P_out) *P_out = P;
  return rho;
}

/* rho_tot / P_tot (background.py:101-145) in species order. */
static void rho_P_tot(const abcmb_cosmo* c, double lna, double* rho_tot, double* P_tot,
                      double* rcdm, double* rb, double* rg, double* rnu, double* rncdm, double* pncdm) {
  double a = exp(lna);
  double a3 = a * a * a, a4 = a * a * a * a;
  double chb3 = (C_CM * HBAR) * (C_CM * HBAR) * (C_CM * HBAR);
  double rde = c->omega_Lambda * RHO_CRIT_UNIT;
  double rc = c->omega_cdm * RHO_CRIT_UNIT / a3;
  double rbb = c->omega_b * RHO_CRIT_UNIT / a3;
  double T04 = c->TCMB0 * c->TCMB0 * c->TCMB0 * c->TCMB0;
  double r_g = PI * PI / 15. * T04 / a4 / chb3;
  double tn = c->T_nu_massless;
  double r_nu = c->N_nu_massless * 2. * 7. / 8. * PI * PI / 30. * (tn * tn * tn * tn) * T04 / a4;
  r_nu = r_nu / chb3;
  double r_ncdm = 0., p_ncdm = 0.;
  if (c->has_ncdm) r_ncdm = rho_ncdm_fn(c, lna, &p_ncdm);
  double rt = 0., pt = 0.;
  rt += rde; pt += -rde;
  rt += rc;
  rt += rbb;
  rt += r_g; pt += r_g / 3.;
  rt += r_nu; pt += r_nu / 3.;
  if (c->has_ncdm) { rt += r_ncdm; pt += p_ncdm; }
  *rho_tot = rt; *P_tot = pt;
  if (rcdm) *rcdm = rc;
  if (rb) *rb = rbb;
  if (rg) *rg = r_g;
  if (rnu) *rnu = r_nu;
  if (rncdm) *rncdm = r_ncdm;
  if (pncdm) *pncdm = p_ncdm;
}

double oracle_aH(const abcmb_cosmo* c, double lna) {
  double rt, pt;
  rho_P_tot(c, lna, &rt, &pt, 0, 0, 0, 0, 0, 0);
  double H = sqrt(8. * PI * GN * rt / 3.);
  return exp(lna) * H / C_MPC;
}

static double bg_H(const abcmb_cosmo* c, double lna) {
  double rt, pt;
  rho_P_tot(c, lna, &rt, &pt, 0, 0, 0, 0, 0, 0);
  return sqrt(8. * PI * GN * rt / 3.);
}

double oracle_tau(const abcmb_cosmo* c, const double* tables, double lna) {
  return oracle_fast_interp(lna, ABCMB_LNA_TAU_MIN, ABCMB_LNA_TAU_MAX, tables + c->off_tau, ABCMB_NTAU_TAB);
}

double oracle_xe(const abcmb_cosmo* c, const double* tables, double lna) {
  if (lna < c->lna_xe0) return c->xe_first;
  if (lna >= c->lna_xe_last) return c->xe_last;
  return oracle_fast_interp(lna, c->lna_xe0, c->lna_xe_max, tables + c->off_xe, c->n_xe);
}

static double nH_fn(const abcmb_cosmo* c, double lna) {
  double a = exp(lna);
  return (1. - c->YHe) * 3. * c->omega_b * H0H * H0H / 8. / PI / GN / MH / (a * a * a);
}

static double gamma_compton(double xe, double TCMB, double YHe) {
  double FHe = YHe * MH / MHE / (1. - YHe);
  return xe / (1. + FHe + xe) * 8. * SIGT * (4. * STEF_BOLT) * (TCMB * TCMB * TCMB * TCMB) / (3. * ME);
}

double oracle_Tm(const abcmb_cosmo* c, const double* tables, double lna) {
  if (lna < c->lna_tm0) {
    double TCMB = c->TCMB0 / exp(lna);
    double xe = oracle_xe(c, tables, lna);
    return TCMB * (1. - bg_H(c, lna) / gamma_compton(xe, TCMB, c->YHe));
  }
  if (lna >= c->lna_tm_last) return c->tm_last;
  return oracle_fast_interp(lna, c->lna_tm0, c->lna_tm_max, tables + c->off_tm, c->n_tm);
}

double oracle_tau_c(const abcmb_cosmo* c, const double* tables, double lna) {
  double a = exp(lna);
  double ne = nH_fn(c, lna) * oracle_xe(c, tables, lna);
  return 1. / a / ne / SIGT / C_CM * C_MPC;
}

/* All background scalars the RHS needs at one lna. */
static void bg_eval(const abcmb_cosmo* c, const double* tables, double lna, bgs_t* b) {
  b->lna = lna;
  b->a = exp(lna);
  rho_P_tot(c, lna, &b->rho_tot, &b->P_tot, &b->rho_cdm, &b->rho_b, &b->rho_g, &b->rho_nu,
            &b->rho_ncdm, &b->P_ncdm);
  double H = sqrt(8. * PI * GN * b->rho_tot / 3.);
  b->aH = exp(lna) * H / C_MPC;
  b->tau = oracle_tau(c, tables, lna);
  b->xe = oracle_xe(c, tables, lna);
  b->tau_c = oracle_tau_c(c, tables, lna);
  b->Tm = oracle_Tm(c, tables, lna);
  b->TCMB = c->TCMB0 / exp(lna);
  /* Baryon.cs2 (species.py:1163-1196), mean_mass (1198-1220) */
  double denom = (1. + b->xe) * (1. - c->YHe) + MH / MHE * c->YHe;
  double mu = MH / denom;
  b->R = 4. * b->rho_g / 3. / b->rho_b;
  b->cs2 = b->Tm / mu * (5. / 3. - 2. / 3. * mu * b->R / ME / b->aH / b->tau_c * (b->TCMB / b->Tm - 1.));
  if (c->has_ncdm) {
    b->ncdm_T = c->T_nu_massive * c->TCMB0 / b->a;
    b->ncdm_x = c->m_nu_massive / b->ncdm_T;
    double T4 = b->ncdm_T * b->ncdm_T * b->ncdm_T * b->ncdm_T;
    b->ncdm_fac = c->N_nu_massive * 4. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    for (int i = 0; i < 3; ++i) b->eps3[i] = sqrt(Q3[i] * Q3[i] + b->ncdm_x * b->ncdm_x);
  } else {
    b->ncdm_T = b->ncdm_x = b->ncdm_fac = 0.;
    b->eps3[0] = b->eps3[1] = b->eps3[2] = 1.;
  }
}

double oracle_aH_prime(const abcmb_cosmo* c, double lna) {
  double rt, pt;
  rho_P_tot(c, lna, &rt, &pt, 0, 0, 0, 0, 0, 0);
  double aH = oracle_aH(c, lna);
  double a = exp(lna);
  return -4. * PI * GN * a * a / 3. / aH * (rt + 3. * pt) / (C_MPC * C_MPC);
}

/* ---------------------------------------------------------------------- */
/* state layout (model_specs.populate_species)                            */
/* ---------------------------------------------------------------------- */
typedef struct {
  int i_eta, i_cdm, i_b, i_g, i_G, i_nu, i_ncdm;
  int nF, nG, nN, nM, ny;
} layout_t;

static void make_layout(const abcmb_cosmo* c, layout_t* L) {
  L->i_eta = 0;
  L->i_cdm = 1;
  L->i_b = 2;
  L->nF = c->lmax_g + 1;
  L->nG = c->lmax_pol_g + 1;
  L->nN = c->lmax_nu + 1;
  L->nM = c->has_ncdm ? c->lmax_ncdm + 1 : 0;
  L->i_g = 4;
  L->i_G = L->i_g + L->nF;
  L->i_nu = L->i_G + L->nG;
  L->i_ncdm = L->i_nu + L->nN;
  L->ny = L->i_ncdm + 3 * L->nM;
}

/* Species sums entering the metric (perturbations.py:231-236). */
static void species_sums(const abcmb_cosmo* c, const layout_t* L, const bgs_t* b, const double* y,
                         double* srd, double* srt, double* srs) {
  double rd = 0., rt = 0., rs = 0.;
  /* DE: 0 */
  rd += b->rho_cdm * y[L->i_cdm];
  rd += b->rho_b * y[L->i_b];
  rt += (b->rho_b + 0.) * y[L->i_b + 1];
  rd += b->rho_g * y[L->i_g];
  rt += (b->rho_g + b->rho_g / 3.) * y[L->i_g + 1];
  rs += (b->rho_g + b->rho_g / 3.) * y[L->i_g + 2];
  rd += b->rho_nu * y[L->i_nu];
  rt += (b->rho_nu + b->rho_nu / 3.) * y[L->i_nu + 1];
  rs += (b->rho_nu + b->rho_nu / 3.) * y[L->i_nu + 2];
  if (c->has_ncdm) {
    double r0 = 0., r1 = 0., r2 = 0.;
    for (int i = 0; i < 3; ++i) {
      double q = Q3[i], w = W3[i];
      const double* Psi = y + L->i_ncdm + i * L->nM;
      r0 += w * (1. + exp(-q)) * b->eps3[i] / (q * q) * Psi[0];
      r1 += w * (1. + exp(-q)) / q * Psi[1];
      r2 += w * (1. + exp(-q)) / b->eps3[i] * Psi[2];
    }
    double T4 = b->ncdm_T * b->ncdm_T * b->ncdm_T * b->ncdm_T;
    rd += c->N_nu_massive * r0 * 4. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    rt += c->N_nu_massive * r1 * 4. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    rs += c->N_nu_massive * r2 * 8. / 3. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
  }
  *srd = rd; *srt = rt; if (srs) *srs = rs;
}

/* get_derivatives (perturbations.py:201-248) with every species' y_prime. */
static void rhs(const abcmb_cosmo* c, const layout_t* L, double k, const bgs_t* b,
                const double* y, double* f) {
  const double aH = b->aH, a = b->a, tau = b->tau, tau_c = b->tau_c;
  double srd, srt;
  species_sums(c, L, b, y, &srd, &srt, 0);
  double hp = 2. / (aH * aH) * (k * k * y[0] + 4. * PI * GN * a * a / (C_MPC * C_MPC) * srd);
  double etap = 4. * PI * GN * a * a / aH / (k * k) * srt / (C_MPC * C_MPC);
  f[0] = etap;
  /* ColdDarkMatter.y_prime (species.py:583-607) */
  f[L->i_cdm] = -0.5 * hp;
  /* Baryon.y_prime (species.py:1245-1285) */
  {
    double d = y[L->i_b], th = y[L->i_b + 1], thg = y[L->i_g + 1];
    f[L->i_b] = -th / aH - hp / 2.;
    f[L->i_b + 1] = -th + b->cs2 * k * k * d / aH + b->R / tau_c / aH * (thg - th);
  }
  /* Photon.y_prime (species.py:1390-1448) */
  {
    const double* F = y + L->i_g;
    const double* G = y + L->i_G;
    double* fF = f + L->i_g;
    double* fG = f + L->i_G;
    int Fl = L->nF - 1, Gl = L->nG - 1;
    double thb = y[L->i_b + 1];
    double delta = F[0], theta = F[1], sigma = F[2];
    fF[0] = -4. / 3. / aH * theta - 2. / 3. * hp;
    fF[1] = k * k / aH * (delta / 4. - sigma) + (thb - theta) / aH / tau_c;
    fF[2] = 4. / 15. / aH * theta - 3. / 10. * k / aH * F[3] + 2. / 15. * hp + 4. / 5. * etap
            - 9. / 10. / aH / tau_c * sigma + (G[0] + G[2]) / 20. / aH / tau_c;
    fF[3] = k / 7. / aH * (6. * sigma - 4. * F[4]) - F[3] / aH / tau_c;
    for (int l = 4; l < Fl; ++l)
      fF[l] = 1. / (2. * l + 1.) * k / aH * (l * F[l - 1] - (l + 1) * F[l + 1]) - F[l] / aH / tau_c;
    fF[Fl] = k / aH * F[Fl - 1] - (Fl + 1) / aH / tau * F[Fl] - F[Fl] / aH / tau_c;
    double src = (2. * sigma + G[0] + G[2]) / 2. / aH / tau_c;
    for (int l = 0; l < Gl; ++l) {
      double s = (l == 0) ? 1. : (l == 2 ? 0.2 : 0.);
      double gm1 = (l == 0) ? G[Gl] : G[l - 1];   /* G[-1] * 0 (quirk q4) */
      fG[l] = 1. / (2. * l + 1.) * k / aH * (l * gm1 - (l + 1) * G[l + 1]) - G[l] / aH / tau_c + src * s;
    }
    fG[Gl] = k / aH * G[Gl - 1] - (Gl + 1) / aH / tau * G[Gl] - G[Gl] / aH / tau_c;
  }
  /* MasslessNeutrino.y_prime (species.py:707-753) */
  {
    const double* F = y + L->i_nu;
    double* fF = f + L->i_nu;
    int lmax = L->nN - 1;
    double delta = F[0], theta = F[1], sigma = F[2];
    fF[0] = -4. / 3. / aH * theta - 2. / 3. * hp;
    fF[1] = k * k / aH * (delta / 4. - sigma);
    fF[2] = 4. / 15. / aH * theta - 3. / 10. * k / aH * F[3] + 2. / 15. * hp + 4. / 5. * etap;
    fF[3] = 1. / 7. * k / aH * (6. * sigma - 4. * F[4]);
    for (int l = 4; l < lmax; ++l)
      fF[l] = 1. / (2. * l + 1.) * k / aH * (l * F[l - 1] - (l + 1) * F[l + 1]);
    fF[lmax] = k / aH * F[lmax - 1] - (lmax + 1) / aH / tau * F[lmax];
  }
  /* MassiveNeutrino.y_prime (species.py:919-977) */
  if (c->has_ncdm) {
    int lmax = L->nM - 1;
    for (int i = 0; i < 3; ++i) {
      double q = Q3[i];
      double eps = b->eps3[i];
      double dlnf0 = -q / (1 + exp(-q));
      const double* P = y + L->i_ncdm + i * L->nM;
      double* fP = f + L->i_ncdm + i * L->nM;
      fP[0] = -q / eps / aH * P[1] + hp / 6. * dlnf0;
      fP[1] = q * k * k / 3. / eps / aH * (P[0] - 2. * P[2]);
      fP[2] = q * k / 5. / eps / aH * (2. * P[1] / k - 3. * P[3]) - (hp / 15. + 2. * etap / 5.) * dlnf0;
      for (int l = 3; l < lmax; ++l)
        fP[l] = q * k / eps / aH / (2 * l + 1) * (l * P[l - 1] - (l + 1) * P[l + 1]);
      fP[lmax] = q * k / aH / eps * P[lmax - 1] - (lmax + 1) / aH / tau * P[lmax];
    }
  }
}

/* ---------------------------------------------------------------------- */
/* start time and initial conditions                                       */
/* ---------------------------------------------------------------------- */

/* Per-cosmology part of get_starting_time: the 10000-point grids. */
typedef struct {
  double* lna;   /* linspace(-20, -10, 10000) */
  double* f1;    /* tau_c * aH                */
  double* aH;
  double lna1;   /* interp(R_tc, f1, lna)     */
} start_grid_t;

#define NSTART 10000

static void start_grid_init(const abcmb_cosmo* c, const double* tables, double R_tc, start_grid_t* g) {
  g->lna = (double*)malloc(sizeof(double) * NSTART);
  g->f1 = (double*)malloc(sizeof(double) * NSTART);
  g->aH = (double*)malloc(sizeof(double) * NSTART);
  for (int i = 0; i < NSTART; ++i) {
    double l = linspace_at(-20.0, -10.0, NSTART, i);
    g->lna[i] = l;
    g->aH[i] = oracle_aH(c, l);
    g->f1[i] = oracle_tau_c(c, tables, l) * g->aH[i];
  }
  g->lna1 = oracle_np_interp(R_tc, g->f1, g->lna, NSTART);
}

static void start_grid_free(start_grid_t* g) { free(g->lna); free(g->f1); free(g->aH); }

double oracle_start_time(const abcmb_cosmo* c, const double* tables, double k, double R_tc, double R_large) {
  start_grid_t g;
  start_grid_init(c, tables, R_tc, &g);
  double* f2 = (double*)malloc(sizeof(double) * NSTART);
  for (int i = 0; i < NSTART; ++i) f2[i] = k / g.aH[i];
  double lna2 = oracle_np_interp(R_large, f2, g.lna, NSTART);
  double s = g.lna1 < lna2 ? g.lna1 : lna2;
  free(f2);
  start_grid_free(&g);
  return s < -10. ? s : -10.;
}

static double start_time_from_grid(const start_grid_t* g, double k, double R_large, double* f2) {
  for (int i = 0; i < NSTART; ++i) f2[i] = k / g->aH[i];
  double lna2 = oracle_np_interp(R_large, f2, g->lna, NSTART);
  double s = g->lna1 < lna2 ? g->lna1 : lna2;
  return s < -10. ? s : -10.;
}

/* initial_conditions_one_k (perturbations.py:161-199). */
static void initial_conditions(const abcmb_cosmo* c, const layout_t* L, const double* tables,
                               double k, double lna_ini, double* y) {
  double tau_ini = oracle_tau(c, tables, lna_ini);
  double om = c->om, Rn = c->R_nu, Rb = c->R_b;
  memset(y, 0, sizeof(double) * L->ny);
  y[0] = (1. - k * k * tau_ini * tau_ini / 12. / (15. + 4. * Rn) *
                   (5. + 4. * Rn - (16. * Rn * Rn + 280. * Rn + 325) / 10. / (2. * Rn + 15.) * tau_ini * om));
  double kt = k * tau_ini;
  /* CDM */
  y[L->i_cdm] = -(kt * kt) / 4. * (1. - om * tau_ini / 5.);
  /* Baryon */
  y[L->i_b] = -(kt * kt) / 4. * (1. - om * tau_ini / 5.);
  y[L->i_b + 1] = -k * k * k * k * tau_ini * tau_ini * tau_ini / 36. *
                  (1. - 3. * (1. + 5. * Rb - Rn) / 20. / (1. - Rn) * om * tau_ini);
  /* Photon */
  y[L->i_g] = -(kt * kt) / 3. * (1. - om * tau_ini / 5.);
  y[L->i_g + 1] = -k * k * k * k * tau_ini * tau_ini * tau_ini / 36. *
                  (1. - 3. * (1. + 5. * Rb - Rn) / 20. / (1. - Rn) * om * tau_ini);
  /* Massless neutrinos */
  double nd = -(kt * kt) / 3. * (1. - om * tau_ini / 5.);
  double nth = -k * (kt * kt * kt) / 36. / (4. * Rn + 15.) *
               (4. * Rn + 11. + 12. - 3. * (8. * Rn * Rn + 50. * Rn + 275.) / 20. / (2. * Rn + 15.) * tau_ini * om);
  double ns = (kt * kt) / (45. + 12. * Rn) * 2. * (1. + (4. * Rn - 5.) / 4. / (2. * Rn + 15.) * tau_ini * om);
  y[L->i_nu] = nd;
  y[L->i_nu + 1] = nth;
  y[L->i_nu + 2] = ns;
  /* Massive neutrinos (species.py:882-917) */
  if (c->has_ncdm) {
    for (int i = 0; i < 3; ++i) {
      double q = Q3[i];
      double fac = q / (1. + exp(-q));
      double* P = y + L->i_ncdm + i * L->nM;
      P[0] = nd / 4. * fac;
      P[1] = nth / 3. * fac;
      P[2] = ns / 2. * fac;
    }
  }
}

/* ---------------------------------------------------------------------- */
/* Kvaerno5 tableau (Kvaerno, BIT 44 (2004) 489-502; ESDIRK 5(4), 7 stages) */
/* ---------------------------------------------------------------------- */
#define KV_GAMMA 0.26
static const double KV_C[7] = {0.0, 0.52, 1.230333209967908, 0.8957659843500759,
                               0.43639360985864756, 1.0, 1.0};
static const double KV_A[7][7] = {
  {0, 0, 0, 0, 0, 0, 0},
  {0.26, 0, 0, 0, 0, 0, 0},
  {0.13, 0.84033320996790809, 0, 0, 0, 0, 0},
  {0.22371961478320505, 0.47675532319799699, -0.06470895363112615, 0, 0, 0, 0},
  {0.16648564323248321, 0.10450018841591720, 0.03631482272098715, -0.13090704451073998, 0, 0, 0},
  {0.13855640231268224, 0.0, -0.04245337201752043, 0.02446657898003141, 0.61943039072480676, 0, 0},
  {0.13659751177640291, 0.0, -0.05496908796538376, -0.04118626728321046, 0.62993304899016403,
   0.06962479448202728, 0}};

void oracle_kvaerno5_tableau(double* A49, double* c7, double* gamma) {
  for (int i = 0; i < 7; ++i) {
    for (int j = 0; j < 7; ++j) A49[i * 7 + j] = KV_A[i][j];
    if (i > 0) A49[i * 7 + i] = KV_GAMMA;
    c7[i] = KV_C[i];
  }
  *gamma = KV_GAMMA;
}

/* ---------------------------------------------------------------------- */
/* dense linear algebra                                                    */
/* ---------------------------------------------------------------------- */

/* LU with partial pivoting, in place; returns 0 on success. */
static int lu_factor(double* M, int n, int* piv) {
  for (int p = 0; p < n; ++p) {
    int im = p;
    double vm = fabs(M[p * n + p]);
    for (int i = p + 1; i < n; ++i) {
      double v = fabs(M[i * n + p]);
      if (v > vm) { vm = v; im = i; }
    }
    piv[p] = im;
    if (vm == 0.0) return -1;
    if (im != p)
      for (int j = 0; j < n; ++j) { double t = M[p * n + j]; M[p * n + j] = M[im * n + j]; M[im * n + j] = t; }
    double inv = 1.0 / M[p * n + p];
    for (int i = p + 1; i < n; ++i) {
      double m = M[i * n + p] * inv;
      M[i * n + p] = m;
      if (m != 0.0)
        for (int j = p + 1; j < n; ++j) M[i * n + j] -= m * M[p * n + j];
    }
  }
  return 0;
}

static void lu_solve(const double* M, int n, const int* piv, double* b) {
  for (int p = 0; p < n; ++p) {
    if (piv[p] != p) { double t = b[p]; b[p] = b[piv[p]]; b[piv[p]] = t; }
  }
  for (int i = 1; i < n; ++i) {
    double s = b[i];
    for (int j = 0; j < i; ++j) s -= M[i * n + j] * b[j];
    b[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < n; ++j) s -= M[i * n + j] * b[j];
    b[i] = s / M[i * n + i];
  }
}

static double rms_norm(const double* v, int n) {
  double s = 0.;
  for (int i = 0; i < n; ++i) s += v[i] * v[i];
  return sqrt(s / n);
}

/* ---------------------------------------------------------------------- */
/* output table at one save point (perturbations.py:318-404)               */
/* ---------------------------------------------------------------------- */
static void output_fields(const abcmb_cosmo* c, const layout_t* L, const double* tables,
                          double k, double lna, const double* y, double* out) {
  bgs_t b;
  bg_eval(c, tables, lna, &b);
  double srd, srt, srs;
  species_sums(c, L, &b, y, &srd, &srt, &srs);
  double a = b.a, aH = b.aH;
  double eta = y[0];
  double delta_b = y[L->i_b], theta_b = y[L->i_b + 1], theta_g = y[L->i_g + 1];
  out[ABCMB_F_THETA_B_PRIME] = -theta_b + b.cs2 / aH * (k * k * delta_b) + b.R / aH / b.tau_c * (theta_g - theta_b);
  /* delta_m: matter species CDM, Baryon, MassiveNeutrino (is_matter) */
  double rdm = b.rho_cdm * y[L->i_cdm] + b.rho_b * y[L->i_b];
  double rm = b.rho_cdm + b.rho_b;
  double ncdm_d = 0., ncdm_t = 0., ncdm_s = 0.;
  if (c->has_ncdm) {
    double r0 = 0., r1 = 0., r2 = 0.;
    for (int i = 0; i < 3; ++i) {
      double q = Q3[i], w = W3[i];
      const double* Psi = y + L->i_ncdm + i * L->nM;
      r0 += w * (1. + exp(-q)) * b.eps3[i] / (q * q) * Psi[0];
      r1 += w * (1. + exp(-q)) / q * Psi[1];
      r2 += w * (1. + exp(-q)) / b.eps3[i] * Psi[2];
    }
    double T4 = b.ncdm_T * b.ncdm_T * b.ncdm_T * b.ncdm_T;
    double rd_n = c->N_nu_massive * r0 * 4. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    double rt_n = c->N_nu_massive * r1 * 4. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    double rs_n = c->N_nu_massive * r2 * 8. / 3. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    rdm += rd_n;
    rm += b.rho_ncdm;
    double rhoP = b.rho_ncdm + b.P_ncdm;
    ncdm_d = rd_n / b.rho_ncdm;
    ncdm_t = rt_n / rhoP;
    ncdm_s = rs_n / rhoP;
  }
  out[ABCMB_F_DELTA_M] = rdm / rm;
  double hp = 2. / (aH * aH) * (k * k * eta + 4. * PI * GN * a * a / (C_MPC * C_MPC) * srd);
  double etap = 4. * PI * GN * a * a / aH * srt / (C_MPC * C_MPC) / (k * k);
  double alpha = aH * (hp + 6. * etap) / 2. / (k * k);
  double alphap = eta / aH - 2. * alpha - 12. * PI * GN * a * a / aH * srs / (C_MPC * C_MPC) / (k * k);
  out[ABCMB_F_ETA] = eta;
  out[ABCMB_F_H_PRIME] = hp;
  out[ABCMB_F_ETA_PRIME] = etap;
  out[ABCMB_F_ALPHA] = alpha;
  out[ABCMB_F_ALPHA_PRIME] = alphap;
  out[ABCMB_F_CDM_DELTA] = y[L->i_cdm];
  out[ABCMB_F_B_DELTA] = delta_b;
  out[ABCMB_F_B_THETA] = theta_b;
  out[ABCMB_F_G_DELTA] = y[L->i_g];
  out[ABCMB_F_G_THETA] = theta_g;
  out[ABCMB_F_G_SIGMA] = y[L->i_g + 2];
  out[ABCMB_F_G_G0] = y[L->i_G];
  out[ABCMB_F_G_G2] = y[L->i_G + 2];
  out[ABCMB_F_NU_DELTA] = y[L->i_nu];
  out[ABCMB_F_NU_THETA] = y[L->i_nu + 1];
  out[ABCMB_F_NU_SIGMA] = y[L->i_nu + 2];
  out[ABCMB_F_NCDM_DELTA] = ncdm_d;
  out[ABCMB_F_NCDM_THETA] = ncdm_t;
  out[ABCMB_F_NCDM_SIGMA] = ncdm_s;
}

/* ---------------------------------------------------------------------- */
/* one k mode: diffeqsolve(Kvaerno5, PIDController, SaveAt(ts))            */
/* ---------------------------------------------------------------------- */

/* scaled rms error as in PIDController.adapt_step_size */
static double scaled_err(const double* y0, const double* y1, const double* e, int n, double rtol, double atol) {
  double s = 0.;
  for (int i = 0; i < n; ++i) {
    double ym = fabs(y0[i]) > fabs(y1[i]) ? fabs(y0[i]) : fabs(y1[i]);
    double v = e[i] / (atol + ym * rtol);
    s += v * v;
  }
  return sqrt(s / n);
}

typedef struct {
  double* y0; double* y1; double* F;  /* F: 7 x ny stage derivatives */
  double* base; double* v; double* r; double* yerr; double* Jm; int* piv;
  double* col; double* tmp; double* f2;
} work_t;

static void work_alloc(work_t* w, int ny) {
  w->y0 = (double*)calloc(ny, sizeof(double));
  w->y1 = (double*)calloc(ny, sizeof(double));
  w->F = (double*)calloc(7 * ny, sizeof(double));
  w->base = (double*)calloc(ny, sizeof(double));
  w->v = (double*)calloc(ny, sizeof(double));
  w->r = (double*)calloc(ny, sizeof(double));
  w->yerr = (double*)calloc(ny, sizeof(double));
  w->Jm = (double*)calloc((size_t)ny * ny, sizeof(double));
  w->piv = (int*)calloc(ny, sizeof(int));
  w->col = (double*)calloc(ny, sizeof(double));
  w->tmp = (double*)calloc(ny, sizeof(double));
  w->f2 = (double*)calloc(NSTART, sizeof(double));
}

static void work_free(work_t* w) {
  free(w->y0); free(w->y1); free(w->F); free(w->base); free(w->v); free(w->r); free(w->yerr);
  free(w->Jm); free(w->piv); free(w->col); free(w->tmp); free(w->f2);
}

/* Forward-mode sensitivities (tangents) of one k mode with respect to up to
 * ABCMB_MAX_TANGENTS parameter directions.  Direction p is given by two
 * descriptors, the cosmology at theta + eps_p (plus) and at theta - eps_p
 * (minus), with their own tables; the tangent u_p approximates
 * eps_p dy/dtheta_p, the first-order part of (y(plus) - y(minus)) / 2.
 *
 * The right-hand side is linear in y and in the background "basis" (every
 * coefficient of A(lna) is a constant times one background function), so
 *   d/deps [A(lna; theta) y] = (f(plus, lna, y) - f(minus, lna, y)) / 2
 * up to second order in eps: the central difference of the background
 * alone, at the base trajectory's times.  The tangent is the forward-mode
 * derivative of the discrete ESDIRK step with the base's step sizes frozen:
 * each implicit stage's tangent solves (I - h gamma A_i) dF_i =
 * A_i (du + h sum_{j<i} a_ij dF_j) + dA_i Y_i exactly, by chord iterations
 * with the step's Newton matrix until the same very-chord test the primal
 * stage uses is met (the iteration matrix is the primal's, so it converges
 * as fast).  The start time moves with theta: u(t0) = dy0/deps - f(t0, y0)
 * dt0/deps, with y0 = IC(theta, t0(theta)) differenced between the two
 * descriptors; afterwards the stage-1 derivative is the previous step's last
 * stage's (first same as last, like the primal's).  Outputs are the two
 * variants' PerturbationTables at their
 * own save times ts(plus) and ts(minus): the fields of y(ts) +- (u(ts) +
 * y'(ts) (ts(plus) - ts(minus)) / 2), with y' the derivative of the dense
 * output, evaluated with each variant's own background. */
typedef struct {
  int nd;
  double tscale;   /* the tangents' size relative to the state's: atol of the tangent solves x tscale */
  const abcmb_cosmo* cp[ABCMB_MAX_TANGENTS];
  const abcmb_cosmo* cm[ABCMB_MAX_TANGENTS];
  const start_grid_t* sgp[ABCMB_MAX_TANGENTS];
  const start_grid_t* sgm[ABCMB_MAX_TANGENTS];
} tan_ctx_t;

typedef struct {
  double* u0;     /* nd x ny tangent at t0             */
  double* u1;     /* nd x ny tangent at t1             */
  double* dF;     /* nd x 7 x ny stage derivatives     */
  double* Y;      /* ny primal stage value             */
  double* z;      /* ny                                */
  double* q;      /* ny                                */
  double* r;      /* ny                                */
  double* fp;     /* ny                                */
  double* fm;     /* ny                                */
  double* yp;     /* ny                                */
  double* us;     /* ny                                */
  double* yd;     /* ny                                */
} tan_work_t;

static void tan_work_alloc(tan_work_t* t, int ny) {
  t->u0 = (double*)calloc((size_t)ABCMB_MAX_TANGENTS * ny, sizeof(double));
  t->u1 = (double*)calloc((size_t)ABCMB_MAX_TANGENTS * ny, sizeof(double));
  t->dF = (double*)calloc((size_t)ABCMB_MAX_TANGENTS * 7 * ny, sizeof(double));
  t->Y = (double*)calloc(ny, sizeof(double));
  t->z = (double*)calloc(ny, sizeof(double));
  t->q = (double*)calloc(ny, sizeof(double));
  t->r = (double*)calloc(ny, sizeof(double));
  t->fp = (double*)calloc(ny, sizeof(double));
  t->fm = (double*)calloc(ny, sizeof(double));
  t->yp = (double*)calloc(ny, sizeof(double));
  t->us = (double*)calloc(ny, sizeof(double));
  t->yd = (double*)calloc(ny, sizeof(double));
}

static void tan_work_free(tan_work_t* t) {
  free(t->u0); free(t->u1); free(t->dF); free(t->Y); free(t->z); free(t->q); free(t->r);
  free(t->fp); free(t->fm); free(t->yp); free(t->us); free(t->yd);
}

/* dA y at lna for direction p: (f(plus, y) - f(minus, y)) / 2 into out. */
static void tangent_dA(const tan_ctx_t* T, int p, const layout_t* L, const double* tables, double k, double lna,
                       const double* y, tan_work_t* tw, double* out) {
  bgs_t bp, bm;
  bg_eval(T->cp[p], tables, lna, &bp);
  bg_eval(T->cm[p], tables, lna, &bm);
  rhs(T->cp[p], L, k, &bp, y, tw->fp);
  rhs(T->cm[p], L, k, &bm, y, tw->fm);
  for (int e = 0; e < L->ny; ++e) out[e] = 0.5 * (tw->fp[e] - tw->fm[e]);
}

/* Jacobian of the stage root function at lna_lin: M = I - h*gamma*A(lna_lin).
 * A is obtained column by column (the RHS is linear in y), the way JAX
 * materialises the Jacobian from JVPs of basis vectors. */
static void build_newton_matrix(const abcmb_cosmo* c, const layout_t* L, double k, const bgs_t* b,
                                double hg, work_t* w) {
  int n = L->ny;
  for (int j = 0; j < n; ++j) {
    memset(w->col, 0, sizeof(double) * n);
    w->col[j] = 1.0;
    rhs(c, L, k, b, w->col, w->tmp);
    for (int i = 0; i < n; ++i) w->Jm[i * n + j] = (i == j ? 1.0 : 0.0) - hg * w->tmp[i];
  }
}

/* Tangents of one accepted step (the primal's stage derivatives F, its
 * Newton matrix LU and y0 are those of the step).  The tangent iteration is
 * linear with the primal's iteration matrix I - M_lin^-1 M_i, whose
 * spectral radius is small whenever the primal stage converged, but which is
 * far from normal in the tight-coupling era: an error with a stiff
 * component (the initial tangent's start-time term puts one there) can grow
 * by ~25x over the first iteration before it contracts.  So a growing step
 * does not stop the tangent iterations (only a non-finite one does), and
 * they get TANGENT_ROOT_MAX iterations.  ts[0] counts chord iterations,
 * ts[1] stage solves that did not meet the test (the last iterate is kept:
 * the tangent never changes the primal's step sequence). */
#define TANGENT_ROOT_MAX 16
static void tangent_step(const abcmb_cosmo* c, const layout_t* L, const double* tables, double k, double h,
                         double t0, double rtol, double atol, const tan_ctx_t* T, work_t* w, tan_work_t* tw,
                         int32_t* ts) {
  const int n = L->ny;
  const double hg = h * KV_GAMMA;
  const double kappa = 1e-2, small_res = 1e-13;
  const int root_max = TANGENT_ROOT_MAX;
  for (int i = 1; i < 7; ++i) {
    const double ti = t0 + KV_C[i] * h;
    bgs_t bi;
    bg_eval(c, tables, ti, &bi);
    /* the converged primal stage value, as the primal formed it */
    for (int e = 0; e < n; ++e) {
      double acc = 0.;
      for (int j = 0; j < i; ++j) acc += KV_A[i][j] * w->F[j * n + e];
      tw->Y[e] = (w->y0[e] + h * acc) + hg * w->F[i * n + e];
    }
    for (int p = 0; p < T->nd; ++p) {
      double* dF = tw->dF + (size_t)p * 7 * n;
      const double* u0 = tw->u0 + (size_t)p * n;
      for (int e = 0; e < n; ++e) {
        double acc = 0.;
        for (int j = 0; j < i; ++j) acc += KV_A[i][j] * dF[j * n + e];
        tw->z[e] = u0[e] + h * acc;
      }
      /* q = A_i z + dA_i Y_i: the part of the residual the iterations keep */
      rhs(c, L, k, &bi, tw->z, tw->q);
      tangent_dA(T, p, L, tables, k, ti, tw->Y, tw, tw->r);
      for (int e = 0; e < n; ++e) tw->q[e] += tw->r[e];
      double* fi = dF + i * n;
      memcpy(fi, dF + (i - 1) * n, sizeof(double) * n);     /* the previous stage's, like the primal */
      double diffsize = INFINITY, diffsize_prev = INFINITY;
      int conv = 0;
      for (int it = 1; it <= root_max; ++it) {
        rhs(c, L, k, &bi, fi, tw->r);
        /* residual h gamma A_i dF + q - dF, solved as the primal's (sign included) */
        for (int e = 0; e < n; ++e) tw->r[e] = -((hg * tw->r[e] + tw->q[e]) - fi[e]);
        lu_solve(w->Jm, n, w->piv, tw->r);
        double ss = 0.;
        for (int e = 0; e < n; ++e) {
          double fnew = fi[e] - tw->r[e];
          fi[e] = fnew;
          double sc = atol + rtol * fabs(fnew);
          double qq = tw->r[e] / sc;
          ss += qq * qq;
        }
        diffsize_prev = diffsize;
        diffsize = sqrt(ss / n);
        ts[0]++;
        if (it >= 2) {
          double rate = diffsize / diffsize_prev;
          double factor = diffsize * rate / (1. - rate);
          int small = diffsize < small_res;
          int converged = factor > 0. && factor < kappa;
          if (small || converged) { conv = 1; break; }
          if (!isfinite(rate)) break;
        }
      }
      if (!conv) ts[1]++;
    }
  }
  for (int p = 0; p < T->nd; ++p) {
    const double* dF = tw->dF + (size_t)p * 7 * n;
    const double* u0 = tw->u0 + (size_t)p * n;
    double* u1 = tw->u1 + (size_t)p * n;
    for (int e = 0; e < n; ++e) {
      double acc = 0.;
      for (int j = 0; j < 6; ++j) acc += KV_A[6][j] * dF[j * n + e];
      acc += KV_GAMMA * dF[6 * n + e];
      u1[e] = u0[e] + h * acc;
    }
  }
}

/* One k mode from its start time to lna = 0 (perturbations.py:250-316). */
/* Internal numerical differentiation (H. G. Bock 1981): mode 1 records every
 * accepted step of the integration (its end time, and the chord iterations
 * of the six implicit stages, 4 bits each); mode 2 replays a record: the
 * step ends and iteration counts are taken from it instead of the step-size
 * controller and the termination test, and every step is accepted (a
 * non-finite error estimate stops the item). */
typedef struct {
  int mode;        /* 0 none, 1 record, 2 replay */
  double* t1;      /* [cap] step ends      */
  int32_t* it;     /* [cap] iteration bits */
  int cap;
  int n;           /* steps recorded (record: written; replay: read) */
} ind_rec_t;

static void solve_k(const abcmb_cosmo* c, const double* tables, const double* kbuf,
                    const abcmb_pert_settings* s, const start_grid_t* sg, int ik,
                    double* pt, abcmb_kstat* st, work_t* w, const tan_ctx_t* T, tan_work_t* tw,
                    int32_t* tst, ind_rec_t* R) {
  const int ind = R ? R->mode : 0;
  layout_t L;
  make_layout(c, &L);
  const int n = L.ny;
  const double k = kbuf[c->off_k + ik];
  const int nsave = s->n_save;
  const double rtol = k > s->k_split ? s->rtol_large : s->rtol_small;
  const double atol = k > s->k_split ? s->atol_large : s->atol_small;
  const double err_order = 5.0;       /* Kvaerno5.order */
  const double safety = 0.9, factormin = 0.2, factormax = 10.0;
  const double coeff1 = (s->icoeff + s->pcoeff + s->dcoeff) / err_order;
  const double coeff2 = -(s->pcoeff + 2. * s->dcoeff) / err_order;
  const double coeff3 = s->dcoeff / err_order;
  const double kappa = 1e-2;          /* VeryChord kappa          */
  const int root_max = 10;            /* Kvaerno5.root_find_max_steps */
  const double small_res = 1e-13;     /* 10**(2 - precision(float64)) */

  double lna_start = start_time_from_grid(sg, k, s->R_large, w->f2);
  st->lna_start = lna_start;
  st->status = ABCMB_STATUS_OK;
  st->n_accepted = st->n_rejected = st->n_newton = 0;

  initial_conditions(c, &L, tables, k, lna_start, w->y0);

  const double t_end = 0.0;
  double t0 = lna_start;
  double t1 = t0 + s->dt0;
  if (t1 > t_end) t1 = t_end;
  double prev_inv = 1.0, prev_prev_inv = 1.0;
  int isave = 0;
  const double lts = c->lna_transfer_start;
  double* ptc = pt + c->off_pt;
  const int nk = c->nk;
  double outv[ABCMB_NFIELDS];
  double* ysave = w->tmp;  /* reuse */

  /* FSAL: stage 1 derivative at (t0, y0) */
  bgs_t b;
  bg_eval(c, tables, t0, &b);
  rhs(c, &L, k, &b, w->y0, w->F);
  if (T) {
    /* tangents at the start: u = dy0/deps - f(t0, y0) dt0/deps, dF_0 = A u + dA y0 */
    for (int p = 0; p < T->nd; ++p) {
      const double tp = start_time_from_grid(T->sgp[p], k, s->R_large, w->f2);
      const double tm = start_time_from_grid(T->sgm[p], k, s->R_large, w->f2);
      initial_conditions(T->cp[p], &L, tables, k, tp, tw->yp);
      initial_conditions(T->cm[p], &L, tables, k, tm, tw->us);
      const double dt0 = 0.5 * (tp - tm);
      double* u = tw->u0 + (size_t)p * n;
      for (int e = 0; e < n; ++e) u[e] = 0.5 * (tw->yp[e] - tw->us[e]) - w->F[e] * dt0;
      double* dF0 = tw->dF + (size_t)p * 7 * n;
      rhs(c, &L, k, &b, u, dF0);
      tangent_dA(T, p, &L, tables, k, t0, w->y0, tw, tw->q);
      for (int e = 0; e < n; ++e) dF0[e] += tw->q[e];
    }
  }

  int nsteps = 0;
  unsigned itbits = 0u;
  if (ind == 2 && R->n <= 0) st->status = ABCMB_STATUS_NONFINITE;   /* the base failed */
  while (t0 < t_end && st->status == ABCMB_STATUS_OK) {
    if (ind == 2) {
      if (nsteps >= R->n) { st->status = ABCMB_STATUS_NONFINITE; break; }
      t1 = R->t1[nsteps];
      itbits = (unsigned)R->it[nsteps];
      if (!(t1 > t0)) { st->status = ABCMB_STATUS_DT_UNDERFLOW; break; }
    } else {
      if (nsteps >= s->max_steps) { st->status = ABCMB_STATUS_MAX_STEPS; break; }
      itbits = 0u;
    }
    nsteps++;
    const double h = t1 - t0;
    const double hg = h * KV_GAMMA;
    /* VeryChord: one Jacobian per step, linearised at the first implicit stage */
    bgs_t blin;
    bg_eval(c, tables, t0 + KV_C[1] * h, &blin);
    build_newton_matrix(c, &L, k, &blin, hg, w);
    int ok = lu_factor(w->Jm, n, w->piv) == 0;
    for (int i = 1; i < 7 && ok; ++i) {
      double ti = t0 + KV_C[i] * h;
      bgs_t bi;
      bg_eval(c, tables, ti, &bi);
      for (int e = 0; e < n; ++e) {
        double acc = 0.;
        for (int j = 0; j < i; ++j) acc += KV_A[i][j] * w->F[j * n + e];
        w->base[e] = w->y0[e] + h * acc;
      }
      double* fi = w->F + i * n;
      memcpy(fi, w->F + (i - 1) * n, sizeof(double) * n);   /* predictor: previous stage */
      double diffsize = INFINITY, diffsize_prev = INFINITY;
      int conv = 0;
      const int it_replay = (int)((itbits >> (4 * (i - 1))) & 15u);
      for (int it = 1; it <= root_max; ++it) {
        for (int e = 0; e < n; ++e) w->v[e] = w->base[e] + hg * fi[e];
        rhs(c, &L, k, &bi, w->v, w->r);
        /* R = A v - f ; diff = J^{-1} R with J = h*gamma*A_lin - I = -M  => diff = -M^{-1} R */
        for (int e = 0; e < n; ++e) w->r[e] = -(w->r[e] - fi[e]);
        lu_solve(w->Jm, n, w->piv, w->r);
        double ss = 0.;
        for (int e = 0; e < n; ++e) {
          double fnew = fi[e] - w->r[e];
          fi[e] = fnew;
          double sc = atol + rtol * fabs(fnew);
          double q = w->r[e] / sc;
          ss += q * q;
        }
        diffsize_prev = diffsize;
        diffsize = sqrt(ss / n);
        st->n_newton++;
        if (ind == 2) {
          if (it >= it_replay) { conv = 1; break; }
        } else if (it >= 2) {
          double rate = diffsize / diffsize_prev;
          double factor = diffsize * rate / (1. - rate);
          int small = diffsize < small_res;
          int diverged = !isfinite(rate) || rate > 2.;
          int converged = factor > 0. && factor < kappa;
          if (small || converged) {
            if (ind == 1) itbits |= (unsigned)it << (4 * (i - 1));
            conv = 1;
            break;
          }
          if (diverged) break;
        }
      }
      if (!conv) ok = 0;
    }
    double scaled;
    if (ok) {
      /* y1 = z7 = y0 + h sum_j a7j F_j + h gamma F_7 ;  y_err = z7 - z6 */
      for (int e = 0; e < n; ++e) {
        double acc = 0., acce = 0.;
        for (int j = 0; j < 6; ++j) {
          acc += KV_A[6][j] * w->F[j * n + e];
          acce += (KV_A[6][j] - KV_A[5][j]) * w->F[j * n + e];
        }
        acc += KV_GAMMA * w->F[6 * n + e];
        /* b_error = b_sol - b_embedded: the embedded row 6 carries gamma on
         * stage 6, the solution row 7 carries gamma on stage 7 */
        acce += -KV_GAMMA * w->F[5 * n + e] + KV_GAMMA * w->F[6 * n + e];
        w->y1[e] = w->y0[e] + h * acc;
        w->yerr[e] = h * acce;
      }
      scaled = scaled_err(w->y0, w->y1, w->yerr, n, rtol, atol);
      if (!isfinite(scaled)) scaled = INFINITY;
    } else {
      scaled = INFINITY;
    }
    int keep = scaled < 1.0;
    if (ind == 2) {
      keep = isfinite(scaled);
      if (!keep) { st->status = ABCMB_STATUS_NONFINITE; break; }
    }
    double inv = 1.0 / scaled;
    double f1v = (coeff1 == 0.) ? 1. : pow(inv, coeff1);
    double f2v = (coeff2 == 0.) ? 1. : pow(prev_inv, coeff2);
    double f3v = (coeff3 == 0.) ? 1. : pow(prev_prev_inv, coeff3);
    double fmin = keep ? 1.0 : factormin;
    double factor = safety * f1v * f2v * f3v;
    if (factor < fmin) factor = fmin;
    if (factor > factormax) factor = factormax;
    double dt_new = h * factor;
    if (inv == 0. || isinf(inv)) inv = 1.;
    if (keep) {
      if (ind == 1) {
        R->t1[st->n_accepted] = t1;
        R->it[st->n_accepted] = (int32_t)itbits;
      }
      st->n_accepted++;
      if (T) tangent_step(c, &L, tables, k, h, t0, rtol, atol * T->tscale, T, w, tw, tst);
      /* dense output: cubic Hermite on [t0, t1] (ThirdOrderHermitePolynomialInterpolation) */
      const double* fa = w->F;            /* f(t0, y0) */
      const double* fb = w->F + 6 * n;    /* f(t1, y1) */
      while (isave < nsave) {
        double ts = linspace_at(lts, 0.0, nsave, isave);
        if (!(ts <= t1)) break;
        if (ts < t0) { isave++; continue; }   /* cannot happen: start < lts */
        double th = (ts - t0) / h;
        for (int e = 0; e < n; ++e) {
          double y0e = w->y0[e], y1e = w->y1[e];
          double k0 = h * fa[e], k1 = h * fb[e];
          ysave[e] = y0e + th * (k0 + th * ((3. * (y1e - y0e) - 2. * k0 - k1) +
                                            th * (2. * (y0e - y1e) + k0 + k1)));
        }
        output_fields(c, &L, tables, k, ts, ysave, outv);
        for (int f = 0; f < ABCMB_NFIELDS; ++f)
          ptc[((size_t)f * nsave + isave) * nk + ik] = outv[f];
        if (T) {
          /* d/dt of the dense output at ts */
          for (int e = 0; e < n; ++e) {
            double y0e = w->y0[e], y1e = w->y1[e];
            double k0 = h * fa[e], k1 = h * fb[e];
            double a2 = 3. * (y1e - y0e) - 2. * k0 - k1, a3 = 2. * (y0e - y1e) + k0 + k1;
            tw->yd[e] = (k0 + th * (2. * a2 + 3. * th * a3)) / h;
          }
          for (int p = 0; p < T->nd; ++p) {
            const double* u0 = tw->u0 + (size_t)p * n;
            const double* u1 = tw->u1 + (size_t)p * n;
            const double* dF = tw->dF + (size_t)p * 7 * n;
            const double tsp = linspace_at(T->cp[p]->lna_transfer_start, 0.0, nsave, isave);
            const double tsm = linspace_at(T->cm[p]->lna_transfer_start, 0.0, nsave, isave);
            const double dts = 0.5 * (tsp - tsm);
            for (int e = 0; e < n; ++e) {
              double k0 = h * dF[e], k1 = h * dF[6 * n + e];
              double us = u0[e] + th * (k0 + th * ((3. * (u1[e] - u0[e]) - 2. * k0 - k1) +
                                                   th * (2. * (u0[e] - u1[e]) + k0 + k1)));
              tw->us[e] = us + tw->yd[e] * dts;
            }
            for (int sgn = 0; sgn < 2; ++sgn) {
              const abcmb_cosmo* cv = sgn == 0 ? T->cp[p] : T->cm[p];
              for (int e = 0; e < n; ++e) tw->yp[e] = sgn == 0 ? ysave[e] + tw->us[e] : ysave[e] - tw->us[e];
              output_fields(cv, &L, tables, k, sgn == 0 ? tsp : tsm, tw->yp, outv);
              double* ptv = pt + cv->off_pt;
              for (int f = 0; f < ABCMB_NFIELDS; ++f)
                ptv[((size_t)f * nsave + isave) * cv->nk + ik] = outv[f];
            }
          }
        }
        isave++;
      }
      prev_prev_inv = prev_inv;
      prev_inv = inv;
      memcpy(w->y0, w->y1, sizeof(double) * n);
      memcpy(w->F, w->F + 6 * n, sizeof(double) * n);   /* FSAL */
      if (T) {
        for (int p = 0; p < T->nd; ++p) {
          memcpy(tw->u0 + (size_t)p * n, tw->u1 + (size_t)p * n, sizeof(double) * n);
          /* first same as last: a re-evaluation A(t0) u0 + dA(t0) y0 would
           * multiply the stiff components' tolerance-level residue by |A| */
          memcpy(tw->dF + (size_t)p * 7 * n, tw->dF + ((size_t)p * 7 + 6) * n, sizeof(double) * n);
        }
      }
      t0 = t1;
    } else {
      st->n_rejected++;
    }
    if (t0 >= t_end || ind == 2) continue;
    double tn = t0 + dt_new;
    const double tol = 1e-10;
    if (tn > t_end - tol) tn = keep ? t_end : t0 + 0.5 * (t_end - t0);
    t1 = tn;
    if (!(h > 1e-14) || !isfinite(t1)) { st->status = ABCMB_STATUS_DT_UNDERFLOW; break; }
  }
  if (st->status == ABCMB_STATUS_OK && isave < nsave) st->status = ABCMB_STATUS_NONFINITE;
  if (ind == 1) R->n = st->status == ABCMB_STATUS_OK ? st->n_accepted : -1;
}

int oracle_pert_forward(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                        int n_items, const int32_t* items, const abcmb_pert_settings* s,
                        double* pt, abcmb_kstat* kstat, int n_threads) {
  start_grid_t* sg = (start_grid_t*)calloc(n_cosmo, sizeof(start_grid_t));
  int maxny = 0;
  for (int c = 0; c < n_cosmo; ++c) {
    start_grid_init(&cosmo[c], tables, s->R_tc, &sg[c]);
    if (cosmo[c].ny > maxny) maxny = cosmo[c].ny;
  }
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
#pragma omp parallel
  {
    work_t w;
    work_alloc(&w, maxny);
#pragma omp for schedule(dynamic, 1)
    for (int it = 0; it < n_items; ++it) {
      int ci = items[2 * it], ik = items[2 * it + 1];
      solve_k(&cosmo[ci], tables, kbuf, s, &sg[ci], ik, pt, &kstat[it], &w, NULL, NULL, NULL, NULL);
    }
    work_free(&w);
  }
  for (int c = 0; c < n_cosmo; ++c) start_grid_free(&sg[c]);
  free(sg);
  int bad = 0;
  for (int it = 0; it < n_items; ++it) if (kstat[it].status != ABCMB_STATUS_OK) bad = 1;
  return bad ? ABCMB_ERR_SOLVER : ABCMB_OK;
}

/* oracle_pert_forward with forward-mode sensitivities (see tan_ctx_t):
 * items name base cosmologies; dirs[ci][p] = (plus, minus) descriptor
 * indices of direction p of base ci (ABCMB_MAX_TANGENTS x 2 int32 per
 * descriptor, -1 where unused).  Writes the base's and every variant's
 * PerturbationTable; tscale = the tangents' size relative to the state's
 * (the parameter step as a fraction of the parameter): the tangent stage
 * solves use the primal's test with atol x tscale.  tstat[2 it] = tangent
 * chord iterations,
 * tstat[2 it + 1] = tangent stage solves left unconverged. */
int oracle_pert_forward_tangent(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                                int n_items, const int32_t* items, int n_dir, const int32_t* dirs, double tscale,
                                const abcmb_pert_settings* s, double* pt, abcmb_kstat* kstat, int32_t* tstat,
                                int n_threads) {
  if (n_dir < 1 || n_dir > ABCMB_MAX_TANGENTS) return ABCMB_ERR_ARG;
  for (int it = 0; it < n_items; ++it) {
    const int ci = items[2 * it];
    for (int p = 0; p < n_dir; ++p) {
      const int a = dirs[(ci * ABCMB_MAX_TANGENTS + p) * 2], b = dirs[(ci * ABCMB_MAX_TANGENTS + p) * 2 + 1];
      if (a < 0 || b < 0 || a >= n_cosmo || b >= n_cosmo || cosmo[a].ny != cosmo[ci].ny ||
          cosmo[b].ny != cosmo[ci].ny || cosmo[a].nk != cosmo[ci].nk || cosmo[b].nk != cosmo[ci].nk)
        return ABCMB_ERR_ARG;
    }
  }
  start_grid_t* sg = (start_grid_t*)calloc(n_cosmo, sizeof(start_grid_t));
  int maxny = 0;
  for (int c = 0; c < n_cosmo; ++c) {
    start_grid_init(&cosmo[c], tables, s->R_tc, &sg[c]);
    if (cosmo[c].ny > maxny) maxny = cosmo[c].ny;
  }
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
#pragma omp parallel
  {
    work_t w;
    work_alloc(&w, maxny);
    tan_work_t tw;
    tan_work_alloc(&tw, maxny);
#pragma omp for schedule(dynamic, 1)
    for (int it = 0; it < n_items; ++it) {
      int ci = items[2 * it], ik = items[2 * it + 1];
      tan_ctx_t T;
      T.nd = n_dir;
      T.tscale = tscale;
      for (int p = 0; p < n_dir; ++p) {
        const int a = dirs[(ci * ABCMB_MAX_TANGENTS + p) * 2], b = dirs[(ci * ABCMB_MAX_TANGENTS + p) * 2 + 1];
        T.cp[p] = &cosmo[a];
        T.cm[p] = &cosmo[b];
        T.sgp[p] = &sg[a];
        T.sgm[p] = &sg[b];
      }
      tstat[2 * it] = tstat[2 * it + 1] = 0;
      solve_k(&cosmo[ci], tables, kbuf, s, &sg[ci], ik, pt, &kstat[it], &w, &T, &tw, tstat + 2 * it, NULL);
    }
    tan_work_free(&tw);
    work_free(&w);
  }
  for (int c = 0; c < n_cosmo; ++c) start_grid_free(&sg[c]);
  free(sg);
  int bad = 0;
  for (int it = 0; it < n_items; ++it) if (kstat[it].status != ABCMB_STATUS_OK) bad = 1;
  return bad ? ABCMB_ERR_SOLVER : ABCMB_OK;
}

/* oracle_pert_forward by internal numerical differentiation (ind_rec_t):
 * items = n_base base items then n_var variant items; var_base[j] = the
 * base item (0..n_base-1) variant item j replays (same k and state layout,
 * ABCMB_STATUS_BAD_LAYOUT otherwise).  kstat has n_base + n_var entries. */
int oracle_pert_forward_ind(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                            int n_base, int n_var, const int32_t* items, const int32_t* var_base,
                            const abcmb_pert_settings* s, double* pt, abcmb_kstat* kstat, int n_threads) {
  if (n_base < 0 || n_var < 0 || (n_var > 0 && n_base == 0)) return ABCMB_ERR_ARG;
  const int cap = s->max_steps;
  double* rt = (double*)malloc(sizeof(double) * (size_t)(n_base > 0 ? n_base : 1) * cap);
  int32_t* ri = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n_base > 0 ? n_base : 1) * cap);
  int32_t* rn = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n_base > 0 ? n_base : 1));
  start_grid_t* sg = (start_grid_t*)calloc(n_cosmo, sizeof(start_grid_t));
  int maxny = 0;
  for (int c = 0; c < n_cosmo; ++c) {
    start_grid_init(&cosmo[c], tables, s->R_tc, &sg[c]);
    if (cosmo[c].ny > maxny) maxny = cosmo[c].ny;
  }
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel
    {
      work_t w;
      work_alloc(&w, maxny);
#pragma omp for schedule(dynamic, 1)
      for (int j = 0; j < (pass == 0 ? n_base : n_var); ++j) {
        const int it = pass == 0 ? j : n_base + j;
        const int ci = items[2 * it], ik = items[2 * it + 1];
        ind_rec_t R;
        if (pass == 0) {
          R.mode = 1;
          R.t1 = rt + (size_t)j * cap;
          R.it = ri + (size_t)j * cap;
          R.cap = cap;
          R.n = -1;
          solve_k(&cosmo[ci], tables, kbuf, s, &sg[ci], ik, pt, &kstat[it], &w, NULL, NULL, NULL, &R);
          rn[j] = R.n;
        } else {
          const int rb = var_base[j];
          int bad = rb < 0 || rb >= n_base;
          if (!bad) {
            const int cb = items[2 * rb];
            const abcmb_cosmo* a = &cosmo[ci];
            const abcmb_cosmo* b = &cosmo[cb];
            bad = items[2 * rb + 1] != ik || a->ny != b->ny || a->nk != b->nk || a->has_ncdm != b->has_ncdm ||
                  a->lmax_g != b->lmax_g || a->lmax_pol_g != b->lmax_pol_g || a->lmax_nu != b->lmax_nu ||
                  a->lmax_ncdm != b->lmax_ncdm || kbuf[a->off_k + ik] != kbuf[b->off_k + ik];
          }
          if (bad) {
            abcmb_kstat z = {ABCMB_STATUS_BAD_LAYOUT, 0, 0, 0, 0.};
            kstat[it] = z;
            continue;
          }
          R.mode = 2;
          R.t1 = rt + (size_t)rb * cap;
          R.it = ri + (size_t)rb * cap;
          R.cap = cap;
          R.n = rn[rb];
          solve_k(&cosmo[ci], tables, kbuf, s, &sg[ci], ik, pt, &kstat[it], &w, NULL, NULL, NULL, &R);
        }
      }
      work_free(&w);
    }
  }
  for (int c = 0; c < n_cosmo; ++c) start_grid_free(&sg[c]);
  free(sg);
  free(rt);
  free(ri);
  free(rn);
  int bad = 0;
  for (int it = 0; it < n_base + n_var; ++it) if (kstat[it].status != ABCMB_STATUS_OK) bad = 1;
  return bad ? ABCMB_ERR_SOLVER : ABCMB_OK;
}

/* Single-k helpers for unit tests. */
void oracle_rhs(const abcmb_cosmo* c, const double* tables, double k, double lna, const double* y, double* f) {
  layout_t L;
  make_layout(c, &L);
  bgs_t b;
  bg_eval(c, tables, lna, &b);
  rhs(c, &L, k, &b, y, f);
}

void oracle_initial_conditions(const abcmb_cosmo* c, const double* tables, double k, double lna, double* y) {
  layout_t L;
  make_layout(c, &L);
  initial_conditions(c, &L, tables, k, lna, y);
}

void oracle_output_fields(const abcmb_cosmo* c, const double* tables, double k, double lna,
                          const double* y, double* out) {
  layout_t L;
  make_layout(c, &L);
  output_fields(c, &L, tables, k, lna, y, out);
}

/* ---------------------------------------------------------------------- */
/* cubic spline, not-a-knot, extrapolating (interpax / scipy CubicSpline)   */
/* ---------------------------------------------------------------------- */

/* Derivatives s[n] of the not-a-knot spline through (x, y); n >= 4. */
void oracle_spline_slopes(const double* x, const double* y, int n, double* s) {
  double* lo = (double*)malloc(sizeof(double) * n);
  double* di = (double*)malloc(sizeof(double) * n);
  double* up = (double*)malloc(sizeof(double) * n);
  double* b = (double*)malloc(sizeof(double) * n);
  double* dx = (double*)malloc(sizeof(double) * n);
  double* sl = (double*)malloc(sizeof(double) * n);
  for (int i = 0; i < n - 1; ++i) { dx[i] = x[i + 1] - x[i]; sl[i] = (y[i + 1] - y[i]) / dx[i]; }
  /* first row */
  {
    double d = x[2] - x[0];
    di[0] = dx[1]; up[0] = d; lo[0] = 0.;
    b[0] = ((dx[0] + 2. * d) * dx[1] * sl[0] + dx[0] * dx[0] * sl[1]) / d;
  }
  for (int i = 1; i < n - 1; ++i) {
    lo[i] = dx[i];
    di[i] = 2. * (dx[i - 1] + dx[i]);
    up[i] = dx[i - 1];
    b[i] = 3. * (dx[i] * sl[i - 1] + dx[i - 1] * sl[i]);
  }
  {
    double d = x[n - 1] - x[n - 3];
    lo[n - 1] = d; di[n - 1] = dx[n - 3]; up[n - 1] = 0.;
    b[n - 1] = (dx[n - 2] * dx[n - 2] * sl[n - 3] + (2. * d + dx[n - 2]) * dx[n - 3] * sl[n - 2]) / d;
  }
  /* Thomas algorithm */
  for (int i = 1; i < n; ++i) {
    double m = lo[i] / di[i - 1];
    di[i] -= m * up[i - 1];
    b[i] -= m * b[i - 1];
  }
  s[n - 1] = b[n - 1] / di[n - 1];
  for (int i = n - 2; i >= 0; --i) s[i] = (b[i] - up[i] * s[i + 1]) / di[i];
  free(lo); free(di); free(up); free(b); free(dx); free(sl);
}

/* Evaluate the spline with slopes s at xq (extrapolating with end pieces). */
double oracle_spline_eval(const double* x, const double* y, const double* s, int n, double xq) {
  /* i = clip(searchsorted(x, xq, 'right'), 1, n-1) - 1 */
  int lo = 0, hi = n;
  while (lo < hi) { int mid = (lo + hi) >> 1; if (x[mid] <= xq) lo = mid + 1; else hi = mid; }
  int i = lo;
  if (i < 1) i = 1;
  if (i > n - 1) i = n - 1;
  i -= 1;
  double dx = x[i + 1] - x[i];
  double sl = (y[i + 1] - y[i]) / dx;
  double t = (s[i] + s[i + 1] - 2. * sl) / dx;
  double c3 = t / dx;
  double c2 = (sl - s[i]) / dx - t;
  double c1 = s[i];
  double c0 = y[i];
  double u = xq - x[i];
  return ((c3 * u + c2) * u + c1) * u + c0;
}

/* ---------------------------------------------------------------------- */
/* Bessel lookups (spectrum.py:48-109, 719-753)                            */
/* ---------------------------------------------------------------------- */
static double jasym(double l, double x) {
  double nu = l + 0.5;
  double r = sqrt(x * x - nu * nu);
  double Q = r - nu * PI / 2 + nu * asin(nu / x);
  double J = sqrt(2 / PI / r) * cos(Q - PI / 4);
  return sqrt(PI / 2 / x) * J;
}

double oracle_phi(int which, const oracle_bessel* B, int idx, double x) {
  double l = (double)B->l_tab[idx];
  double xmin = B->xmin[which][idx], xmax = B->xmax[which][idx];
  const double* col = B->phi[which] + (size_t)idx * B->n_x;
  if (x < xmin) return 0.;
  if (x >= xmax) {
    if (which == 0) return jasym(l, x);
    if (which == 1) return l / x * jasym(l, x) - jasym(l + 1, x);
    return ((3 * l * (l - 1) - 2 * x * x) * jasym(l, x) + 6 * x * jasym(l + 1, x)) / 2 / (x * x);
  }
  return oracle_fast_interp(x, xmin, xmax, col, B->n_x);
}

/* ---------------------------------------------------------------------- */
/* SpectrumSolver.get_Cl                                                   */
/* ---------------------------------------------------------------------- */

/* Transfer sources S[4][n_lna][nkt] for one cosmology (spectrum.py:640-696). */
void oracle_sources(const abcmb_cosmo* c, const double* tables, const double* kbuf, const double* pt,
                    const double* kt, int nkt, int n_save, const abcmb_los_settings* ls, double* S) {
  const int nk = c->nk;
  const int nl = n_save - 1;
  const double* kp = kbuf + c->off_k;
  const double* los = tables + c->off_los;
  const double* ptc = pt + c->off_pt;
  double* lk = (double*)malloc(sizeof(double) * nk);
  double* lkt = (double*)malloc(sizeof(double) * nkt);
  for (int i = 0; i < nk; ++i) lk[i] = log10(kp[i]);
  for (int i = 0; i < nkt; ++i) lkt[i] = log10(kt[i]);
  static const int fields[10] = {ABCMB_F_G_DELTA, ABCMB_F_B_THETA, ABCMB_F_THETA_B_PRIME, ABCMB_F_G_SIGMA,
                                 ABCMB_F_G_G0, ABCMB_F_G_G2, ABCMB_F_ETA, ABCMB_F_ETA_PRIME,
                                 ABCMB_F_ALPHA, ABCMB_F_ALPHA_PRIME};
#pragma omp parallel
  {
    double* sl = (double*)malloc(sizeof(double) * nk);
    double* val = (double*)malloc(sizeof(double) * 10 * nkt);
#pragma omp for schedule(static)
    for (int il = 0; il < nl; ++il) {
      for (int f = 0; f < 10; ++f) {
        const double* col = ptc + ((size_t)fields[f] * n_save + il) * nk;
        oracle_spline_slopes(lk, col, nk, sl);
        for (int j = 0; j < nkt; ++j) val[f * nkt + j] = oracle_spline_eval(lk, col, sl, nk, lkt[j]);
      }
      double g = los[1 * nl + il], gp = los[2 * nl + il], aH = los[3 * nl + il];
      double em = los[4 * nl + il], aHd = los[5 * nl + il];
      for (int j = 0; j < nkt; ++j) {
        double k = kt[j];
        double dg = val[0 * nkt + j], thb = val[1 * nkt + j], thbp = val[2 * nkt + j], sg = val[3 * nkt + j];
        double G0 = val[4 * nkt + j], G2 = val[5 * nkt + j], eta = val[6 * nkt + j], etap = val[7 * nkt + j];
        double al = val[8 * nkt + j], alp = val[9 * nkt + j];
        double sT0 = ls->scale_sw * g * (dg / 4. + aH * alp)
                     + ls->scale_isw * (g * (eta - aH * alp - 2. * aH * al)
                                        + 2. * em * (aH * etap - aHd * al - aH * aH * alp))
                     + ls->scale_dop * (aH * (g * ((thbp / (k * k)) + alp) + gp * ((thb / (k * k)) + al)));
        double sT1 = ls->scale_isw * em * ((aH * alp + 2. * aH * al - eta) * k);
        double sT2 = ls->scale_pol * g * (2 * sg + G0 + G2) / 8.;
        double sE = sqrt(6.) * g * (2 * sg + G0 + G2) / 8.;
        S[((size_t)0 * nl + il) * nkt + j] = sT0;
        S[((size_t)1 * nl + il) * nkt + j] = sT1;
        S[((size_t)2 * nl + il) * nkt + j] = sT2;
        S[((size_t)3 * nl + il) * nkt + j] = sE;
      }
    }
    free(sl); free(val);
  }
  free(lk); free(lkt);
}

/* Transfer functions Delta_T(l,k), Delta_E(l,k) for tabulated l index idx. */
static void los_one_ell(const abcmb_cosmo* c, const double* tables, const double* S, const double* kt, int nkt,
                        int n_save, double lna_first, double lna_last_delta, const oracle_bessel* B, int idx,
                        double* T, double* E) {
  const int nl = n_save - 1;
  const double* los = tables + c->off_los;
  const double tau0 = c->tau0;
  double l = (double)B->l_tab[idx];
  double ef = sqrt(3. / 8. * (l + 2) * (l + 1) * l * (l - 1));
  (void)lna_first;
  for (int j = 0; j < nkt; ++j) {
    double k = kt[j];
    double a0 = 0., a1 = 0., a2 = 0., aE = 0.;
    for (int il = 0; il < nl; ++il) {
      double w = il == 0 ? 0.5 * lna_last_delta : lna_last_delta;
      double tau = los[0 * nl + il], aH = los[3 * nl + il];
      double chi = (tau0 - tau) * k;
      double p0 = oracle_phi(0, B, idx, chi);
      double p1 = oracle_phi(1, B, idx, chi);
      double p2 = oracle_phi(2, B, idx, chi);
      double eps = p0 / (chi * chi) * ef;
      double inv_aH = 1.0 / aH;
      a0 = a0 + w * S[((size_t)0 * nl + il) * nkt + j] * inv_aH * p0;
      a1 = a1 + w * S[((size_t)1 * nl + il) * nkt + j] * inv_aH * p1;
      a2 = a2 + w * S[((size_t)2 * nl + il) * nkt + j] * inv_aH * p2;
      aE = aE + w * S[((size_t)3 * nl + il) * nkt + j] * inv_aH * eps;
    }
    T[j] = a0 + a1 + a2;
    E[j] = aE;
  }
}

static double trapz(const double* y, const double* x, int n) {
  double s = 0.;
  for (int i = 0; i < n - 1; ++i) s += (x[i + 1] - x[i]) * (y[i] + y[i + 1]) / 2.;
  return s;
}

int oracle_los_forward(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                       const double* pt, const double* kt, const abcmb_los_settings* ls, int n_save,
                       const oracle_bessel* B, double* cl_raw, double* cl, int n_threads) {
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  const int nkt = ls->nkt;
  const int nl = n_save - 1;
  const int n_ell_tab = ls->idx_max - ls->idx_min + 1;
  const int n_out = ls->l_max - ls->l_min + 1;
  double* S = (double*)malloc(sizeof(double) * 4 * (size_t)nl * nkt);
  for (int ci = 0; ci < n_cosmo; ++ci) {
    const abcmb_cosmo* c = &cosmo[ci];
    oracle_sources(c, tables, kbuf, pt, kt, nkt, n_save, ls, S);
    double lts = c->lna_transfer_start;
    double dl = linspace_at(lts, 0., n_save, n_save - 1) - linspace_at(lts, 0., n_save, n_save - 2);
    double* raw = cl_raw + (size_t)ci * n_ell_tab * 3;
#pragma omp parallel
    {
      double* T = (double*)malloc(sizeof(double) * nkt);
      double* E = (double*)malloc(sizeof(double) * nkt);
      double* itg = (double*)malloc(sizeof(double) * nkt * 3);
#pragma omp for schedule(dynamic, 1)
      for (int ie = 0; ie < n_ell_tab; ++ie) {
        int idx = ls->idx_min + ie;
        los_one_ell(c, tables, S, kt, nkt, n_save, lts, dl, B, idx, T, E);
        for (int j = 0; j < nkt; ++j) {
          double k = kt[j];
          double pr = 4. * PI * c->A_s * pow(k / ls->k_pivot, c->n_s - 1.);
          itg[j] = pr * T[j] * T[j] / k;
          itg[nkt + j] = pr * T[j] * E[j] / k;
          itg[2 * nkt + j] = pr * E[j] * E[j] / k;
        }
        raw[ie * 3 + 0] = trapz(itg, kt, nkt);
        raw[ie * 3 + 1] = trapz(itg + nkt, kt, nkt);
        raw[ie * 3 + 2] = trapz(itg + 2 * nkt, kt, nkt);
      }
      free(T); free(E); free(itg);
    }
    /* spline over tabulated l onto integer l (spectrum.py:597-608) */
    double* lx = (double*)malloc(sizeof(double) * n_ell_tab);
    double* yy = (double*)malloc(sizeof(double) * n_ell_tab);
    double* sl = (double*)malloc(sizeof(double) * n_ell_tab);
    for (int ie = 0; ie < n_ell_tab; ++ie) lx[ie] = (double)B->l_tab[ls->idx_min + ie];
    for (int X = 0; X < 3; ++X) {
      for (int ie = 0; ie < n_ell_tab; ++ie) yy[ie] = raw[ie * 3 + X];
      oracle_spline_slopes(lx, yy, n_ell_tab, sl);
      for (int o = 0; o < n_out; ++o)
        cl[((size_t)ci * 3 + X) * n_out + o] = oracle_spline_eval(lx, yy, sl, n_ell_tab, (double)(ls->l_min + o));
    }
    free(lx); free(yy); free(sl);
  }
  free(S);
  return ABCMB_OK;
}

/* SpectrumSolver.Pk_lin (spectrum.py:268-302) */
int oracle_pk_lin(int n_cosmo, const abcmb_cosmo* cosmo, const double* kbuf, const double* pt, int n_save,
                  double k_pivot, int n_kout, const double* kout, int n_z, const double* z, double* pk) {
  for (int ci = 0; ci < n_cosmo; ++ci) {
    const abcmb_cosmo* c = &cosmo[ci];
    const int nk = c->nk;
    const double* kp = kbuf + c->off_k;
    const double* dm = pt + c->off_pt + (size_t)ABCMB_F_DELTA_M * n_save * nk;
    double* lna = (double*)malloc(sizeof(double) * n_save);
    double* colv = (double*)malloc(sizeof(double) * n_save);
    double* dml = (double*)malloc(sizeof(double) * nk);
    for (int i = 0; i < n_save; ++i) lna[i] = linspace_at(c->lna_transfer_start, 0., n_save, i);
    for (int iz = 0; iz < n_z; ++iz) {
      double l = -log(1. + z[iz]);
      for (int ik = 0; ik < nk; ++ik) {
        for (int i = 0; i < n_save; ++i) colv[i] = dm[(size_t)i * nk + ik];
        dml[ik] = oracle_np_interp(l, lna, colv, n_save);
      }
      for (int j = 0; j < n_kout; ++j) {
        double k = kout[j];
        double d = oracle_np_interp(k, kp, dml, nk);
        double prim = c->A_s * pow(k / k_pivot, c->n_s - 1.) * (2 * PI * PI / (k * k * k));
        pk[((size_t)ci * n_z + iz) * n_kout + j] = d * d * prim;
      }
    }
    free(lna); free(colv); free(dml);
  }
  return ABCMB_OK;
}

/* ---------------------------------------------------------------------- */
/* lensing (spectrum.py:349-572, ABCMBTools.py:16-186)                     */
/* ---------------------------------------------------------------------- */

static double nan_to_zero(double x) { return isnan(x) ? 0. : x; }

static double factorial_int(int n) {
  double f = 1.;
  for (int i = 2; i <= n; ++i) f *= (double)i;
  return f;
}

static double ipow(double x, int p) {
  double r = 1.;
  for (int i = 0; i < p; ++i) r *= x;
  return r;
}

/* ABCMBTools.wigner_d_matrix (ABCMBTools.py:16-65) for one mu: d^l_{mn}(mu)
 * for l = m..l_end into out[l - m].  The recursion variable is normalised by
 * sqrt((2l+1)/2); the coefficients' 0/0 at l = 0 (d00) become 0 exactly as
 * jnp.nan_to_num does there (no coefficient is ever infinite). */
void oracle_wigner_d(int m, int n, double mu, int l_end, double* out) {
  double beta = acos(mu);
  double norm = sqrt((2. * m + 1.) / 2.) * sqrt(factorial_int(2 * m) / (factorial_int(m + n) * factorial_int(m - n)));
  double D = norm * ipow(cos(beta / 2.), m + n) * ipow(-sin(beta / 2.), m - n);
  double Dm1 = 0.;
  for (int l = m; l <= l_end; ++l) {
    double L = (double)l;
    out[l - m] = D * sqrt(2. / (2. * L + 1.));
    double normA = sqrt((2. * L + 3.) / (2. * L + 1.));
    double normC = sqrt((2. * L + 3.) / (2. * L - 1.));
    double denom = sqrt((L + 1.) * (L + 1.) - (double)(m * m)) * sqrt((L + 1.) * (L + 1.) - (double)(n * n));
    double A = nan_to_zero(normA * (L + 1.) * (2. * L + 1.) / denom);
    double B = nan_to_zero(-A * m * n / L / (L + 1.));
    double C = nan_to_zero(-normC * sqrt(L * L - (double)(m * m)) * sqrt(L * L - (double)(n * n)) / denom * (L + 1.) / L);
    double Dn = A * mu * D + B * D + C * Dm1;
    Dm1 = D;
    D = Dn;
  }
}

/* d^l_{mn}(mu) on ells 2..l_lens as the d00/d1n/d2n/d3n/d4n wrappers return
 * them (ABCMBTools.py:67-186): rows for m < 2 drop the patched l < 2, rows
 * for m > 2 are zero below l = m.  row[l - 2]. */
static void wigner_row(int m, int n, double mu, int l_lens, double* row, double* tmp) {
  oracle_wigner_d(m, n, mu, l_lens, tmp);
  for (int l = 2; l <= l_lens; ++l) row[l - 2] = (l >= m) ? tmp[l - m] : 0.;
}

/* SpectrumSolver.lensing_Cl (spectrum.py:386-435) with
 * lensing_power_spectrum (:349-384) and Pk_lin (:268-302). */
static void lensing_cl(const abcmb_cosmo* c, const abcmb_lens_cosmo* lc, const double* tables, const double* kbuf,
                       const double* pt, const abcmb_lens_settings* s, double* clpp) {
  const int n_lna = s->n_lna, n_save = s->n_save, nk = c->nk, L = s->l_lens;
  const double* kp = kbuf + c->off_k;
  const double* dm = pt + c->off_pt + (size_t)ABCMB_F_DELTA_M * n_save * nk;
  double* ptl = (double*)malloc(sizeof(double) * n_save);
  double* col = (double*)malloc(sizeof(double) * n_save);
  double* dml = (double*)malloc(sizeof(double) * (size_t)n_lna * nk);   /* delta_m(lna_i) per PT k */
  double* fac = (double*)malloc(sizeof(double) * n_lna);                /* everything but Pk/k     */
  double* chi = (double*)malloc(sizeof(double) * n_lna);
  double* x = (double*)malloc(sizeof(double) * n_lna);
  for (int i = 0; i < n_save; ++i) ptl[i] = linspace_at(c->lna_transfer_start, 0., n_save, i);
  const double chi_rec = c->tau0 - oracle_tau(c, tables, lc->lna_rec);
  const double lna_floor = linspace_at(lc->lna_rec, 0., n_lna, n_lna - 2);
  const double Omega_m = lc->omega_m / (c->h * c->h);
  const double Omega_L = c->omega_Lambda / (c->h * c->h);
  for (int i = 0; i < n_lna; ++i) {
    double lna = linspace_at(lc->lna_rec, 0., n_lna, i);
    x[i] = lna;
    double ls = lna < 0. ? lna : lna_floor;
    double chs = c->tau0 - oracle_tau(c, tables, ls);
    chi[i] = chs;
    double window = (chi_rec - chs) / chi_rec / chs;
    double aH = oracle_aH(c, ls);
    double a = exp(ls);
    double z = 1. / a - 1.;
    double zp3 = (1. + z) * (1. + z) * (1. + z);
    double Om = (Omega_m * zp3) / ((Omega_m * zp3) + Omega_L);
    double aH2 = aH * aH;
    fac[i] = lna < 0. ? chs / aH * window * window * (9. / 8. / (PI * PI) * (Om * Om) * (aH2 * aH2)) : 0.;
    double lnap = -log(1. + z);
    for (int j = 0; j < nk; ++j) {
      for (int t = 0; t < n_save; ++t) col[t] = dm[(size_t)t * nk + j];
      dml[(size_t)i * nk + j] = oracle_np_interp(lnap, ptl, col, n_save);
    }
  }
#pragma omp parallel for schedule(static)
  for (int l = 2; l <= L; ++l) {
    double acc = 0., yprev = 0.;
    for (int i = 0; i < n_lna; ++i) {
      double k = ((double)l + 0.5) / chi[i];
      double d = oracle_np_interp(k, kp, dml + (size_t)i * nk, nk);
      double Pk = d * d * (c->A_s * pow(k / s->k_pivot, c->n_s - 1.) * (2 * PI * PI / (k * k * k)));
      double y = fac[i] * Pk / k;
      if (i > 0) acc += (x[i] - x[i - 1]) * (y + yprev);
      yprev = y;
    }
    double lh = (double)l + 0.5;
    clpp[l - 2] = 8. * PI * PI / (lh * lh * lh) * (0.5 * acc);
  }
  free(ptl); free(col); free(dml); free(fac); free(chi); free(x);
}

enum { W00, W11, W1M1, W2M2, W22, W20, W31, W3M3, W3M1, W40, W4M4, W4M2, NWROW };
static const int WROW_M[NWROW] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 4, 4, 4};
static const int WROW_N[NWROW] = {0, 1, -1, -2, 2, 0, 1, -3, -1, 0, -4, -2};

/* SpectrumSolver.lensed_Cls (spectrum.py:437-572) for one cosmology, one mu
 * row of the 12 distinct d matrices at a time. */
static void lensed_cls(const abcmb_lens_settings* s, const double* mu, const double* w, const double* clpp,
                       const double* cl_unl, double* cl_out) {
  const int L = s->l_lens, nl = L - 1, n_mu = s->n_mu;
  const double* ClTT = cl_unl;
  const double* ClTE = cl_unl + nl;
  const double* ClEE = cl_unl + 2 * nl;
  double* Cgl = (double*)malloc(sizeof(double) * n_mu);
  double* Cgl2 = (double*)malloc(sizeof(double) * n_mu);
  /* lensing angular correlation functions (spectrum.py:497-506) */
#pragma omp parallel
  {
    double* r11 = (double*)malloc(sizeof(double) * nl);
    double* r1m1 = (double*)malloc(sizeof(double) * nl);
    double* tmp = (double*)malloc(sizeof(double) * (L + 2));
#pragma omp for schedule(static)
    for (int im = 0; im < n_mu; ++im) {
      wigner_row(1, 1, mu[im], L, r11, tmp);
      wigner_row(1, -1, mu[im], L, r1m1, tmp);
      double a = 0., b = 0.;
      for (int l = 2; l <= L; ++l) {
        double c0 = (2. * l + 1) * l * (l + 1) * clpp[l - 2];
        a += c0 * r11[l - 2];
        b += c0 * r1m1[l - 2];
      }
      Cgl[im] = 1. / 4. / PI * a;
      Cgl2[im] = 1. / 4. / PI * b;
    }
    free(r11); free(r1m1); free(tmp);
  }
  int nthr = 1;
#ifdef _OPENMP
  nthr = omp_get_max_threads();
#endif
  double* acc = (double*)calloc((size_t)nthr * 3 * nl, sizeof(double));
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* my = acc + (size_t)tid * 3 * nl;
    double* d = (double*)malloc(sizeof(double) * NWROW * nl);
    double* tmp = (double*)malloc(sizeof(double) * (L + 2));
#pragma omp for schedule(static)
    for (int im = 0; im < n_mu; ++im) {
      for (int r = 0; r < NWROW; ++r) wigner_row(WROW_M[r], WROW_N[r], mu[im], L, d + (size_t)r * nl, tmp);
      const double sigma2 = Cgl[n_mu - 1] - Cgl[im];
      const double cg = Cgl2[im];
      double ksi = 0., ksip = 0., ksim = 0., ksix = 0.;
      for (int l = 2; l <= L; ++l) {
        const int i = l - 2;
        const double llp1 = (double)l * (l + 1);
        const double X000 = exp(-llp1 * sigma2 / 4);
        const double X000p = -llp1 / 4. * X000;
        const double X220 = 1. / 4. * sqrt((double)(l + 2) * (l - 1) * l * (l + 1)) * exp(-(llp1 - 2) * sigma2 / 4.);
        const double X022 = exp(-(llp1 - 4) * sigma2 / 4);
        const double X022p = -(llp1 - 4) / 4 * X022;
        const double X121 = -1. / 2. * sqrt((double)(l + 2) * (l - 1)) * exp(-(llp1 - 8. / 3.) * sigma2 / 4.);
        const double X132 = -1. / 2. * sqrt((double)(l + 3) * (l - 2)) * exp(-(llp1 - 20. / 3.) * sigma2 / 4.);
        const double X242 = 1. / 4. * sqrt((double)(l + 4) * (l + 3) * (l - 2) * (l - 3)) *
                            exp(-(llp1 - 10.) * sigma2 / 4.);
        const double d00 = d[W00 * nl + i], d11 = d[W11 * nl + i], d1m1 = d[W1M1 * nl + i];
        const double d2m2 = d[W2M2 * nl + i], d22 = d[W22 * nl + i], d20 = d[W20 * nl + i];
        const double d31 = d[W31 * nl + i], d3m3 = d[W3M3 * nl + i], d3m1 = d[W3M1 * nl + i];
        const double d40 = d[W40 * nl + i], d4m4 = d[W4M4 * nl + i], d4m2 = d[W4M2 * nl + i];
        const double tl = 2. * l + 1;
        ksi += tl * ClTT[i] * (X000 * X000 * d00 + 8. / l / (l + 1) * cg * X000p * X000p * d1m1 +
                               cg * cg * (X000p * X000p * d00 + X220 * X220 * d2m2));
        ksip += tl * ClEE[i] * (X022 * X022 * d22 + 2 * cg * X132 * X121 * d31 +
                                cg * cg * (X022p * X022p * d22 + X242 * X220 * d40));
        ksim += tl * ClEE[i] * (X022 * X022 * d2m2 + cg * (X121 * X121 * d1m1 + X132 * X132 * d3m3) +
                                1. / 2. * cg * cg * (2 * X022p * X022p * d2m2 + X220 * X220 * d00 + X242 * X242 * d4m4));
        ksix += tl * ClTE[i] * (X022 * X000 * d20 + cg * 2 * X000p / sqrt(llp1) * (X121 * d11 + X132 * d3m1) +
                                1. / 2. * cg * cg * ((2 * X022p * X000p + X220 * X220) * d20 + X220 * X242 * d4m2));
      }
      ksi *= 1. / 4. / PI; ksip *= 1. / 4. / PI; ksim *= 1. / 4. / PI; ksix *= 1. / 4. / PI;
      /* Gauss-Legendre quadrature back to C_l (spectrum.py:563-570) */
      for (int i = 0; i < nl; ++i) {
        my[i] += ksi * d[W00 * nl + i] * w[im];
        my[nl + i] += ksix * d[W20 * nl + i] * w[im];
        my[2 * nl + i] += (ksip * d[W22 * nl + i] + ksim * d[W2M2 * nl + i]) * w[im];
      }
    }
    free(d); free(tmp);
  }
  const int n_out = s->l_max - 1;
  for (int i = 0; i < n_out; ++i) {
    double tt = 0., te = 0., ee = 0.;
    for (int t = 0; t < nthr; ++t) {
      tt += acc[(size_t)t * 3 * nl + i];
      te += acc[(size_t)t * 3 * nl + nl + i];
      ee += acc[(size_t)t * 3 * nl + 2 * nl + i];
    }
    cl_out[i] = 2 * PI * tt;
    cl_out[n_out + i] = 2 * PI * te;
    cl_out[2 * n_out + i] = 1. / 2. * 2 * PI * ee;
  }
  free(acc); free(Cgl); free(Cgl2);
}

/* The lensing branch of get_Cl (spectrum.py:603-612): C_l^phiphi, then the
 * lensed spectra on ells 2..l_max. */
int oracle_lens_forward(int n_cosmo, const abcmb_cosmo* cosmo, const abcmb_lens_cosmo* lens, const double* tables,
                        const double* kbuf, const double* pt, const double* mu, const double* w,
                        const double* cl_unl, const abcmb_lens_settings* s, double* clpp, double* cl,
                        int n_threads) {
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  if (s->l_max < 2 || s->l_lens < s->l_max || s->n_mu < 2 || s->n_lna < 3) return ABCMB_ERR_ARG;
  const int nl = s->l_lens - 1;
  for (int ci = 0; ci < n_cosmo; ++ci) {
    lensing_cl(&cosmo[ci], &lens[ci], tables, kbuf, pt, s, clpp + (size_t)ci * nl);
    lensed_cls(s, mu, w, clpp + (size_t)ci * nl, cl_unl + (size_t)ci * 3 * nl, cl + (size_t)ci * 3 * (s->l_max - 1));
  }
  return ABCMB_OK;
}

/* ---------------------------------------------------------------------- */
/* background producer: conformal-time table, optical depth, visibility    */
/* ---------------------------------------------------------------------- */

/* Dense output of a scalar solve: the accepted points (s_j, y_j, f_j) in the
 * solver's own time s = d t (d = -1 for a backward solve, as diffrax flips
 * time), f = dy/ds. */
typedef struct {
  int n;
  double* s;
  double* y;
  double* f;
} dense_t;

typedef double (*bg_rhs_fn)(const abcmb_cosmo* c, const double* tables, double lna);

static double rhs_dtau(const abcmb_cosmo* c, const double* tables, double lna) {
  (void)tables;
  return 1. / oracle_aH(c, lna);                               /* background.py:231-250 */
}

static double rhs_dkappa(const abcmb_cosmo* c, const double* tables, double lna) {
  return -1. / oracle_tau_c(c, tables, lna) / oracle_aH(c, lna); /* background.py:704 */
}

/* diffeqsolve(ODETerm(f), Kvaerno5(), t0, t1, dt0, y0, PIDController(...),
 * SaveAt(dense=True), max_steps) for a right-hand side f(t) that does not
 * depend on y (background.py:286-297, 708-719).  With a constant Jacobian
 * of zero the very-chord iteration of every implicit stage returns f(t_i)
 * (its second iteration finds a zero update), so each stage derivative is f
 * at the stage time; the step, error estimate, PID controller and end
 * clipping are those of solve_k.  Returns an ABCMB_STATUS_* code; *nsteps =
 * step attempts, d->n = accepted points (including the initial one). */
static int quad_solve(bg_rhs_fn f, double scale, const abcmb_cosmo* c, const double* tables, double t0,
                      double t1, double y0, double dt0, double rtol, double atol, double pcoeff, double icoeff,
                      double dcoeff, int max_steps, dense_t* d, int* nsteps_out) {
  const double dir = t1 < t0 ? -1. : 1.;
  const double err_order = 5.0, safety = 0.9, factormin = 0.2, factormax = 10.0;
  const double coeff1 = (icoeff + pcoeff + dcoeff) / err_order;
  const double coeff2 = -(pcoeff + 2. * dcoeff) / err_order;
  const double coeff3 = dcoeff / err_order;
  const double s_end = dir * t1;
  double s0 = dir * t0;
  double s1 = s0 + dir * dt0;
  if (s1 > s_end) s1 = s_end;
  double y = y0;
  double F[7];
  F[0] = dir * scale * f(c, tables, dir * s0);
  double prev_inv = 1.0, prev_prev_inv = 1.0;
  int status = ABCMB_STATUS_OK, nsteps = 0;
  d->n = 1;
  d->s[0] = s0; d->y[0] = y; d->f[0] = F[0];
  while (s0 < s_end) {
    if (nsteps >= max_steps) { status = ABCMB_STATUS_MAX_STEPS; break; }
    nsteps++;
    const double h = s1 - s0;
    for (int i = 1; i < 7; ++i) F[i] = dir * scale * f(c, tables, dir * (s0 + KV_C[i] * h));
    double acc = 0., acce = 0.;
    for (int j = 0; j < 6; ++j) {
      acc += KV_A[6][j] * F[j];
      acce += (KV_A[6][j] - KV_A[5][j]) * F[j];
    }
    acc += KV_GAMMA * F[6];
    acce += -KV_GAMMA * F[5] + KV_GAMMA * F[6];
    const double y1 = y + h * acc;
    const double err = h * acce;
    const double sc_y = fabs(y) > fabs(y1) ? fabs(y) : fabs(y1);
    double scaled = fabs(err / (atol + rtol * sc_y));
    if (!isfinite(scaled)) scaled = INFINITY;
    const int keep = scaled < 1.0;
    double inv = 1.0 / scaled;
    double f1v = (coeff1 == 0.) ? 1. : pow(inv, coeff1);
    double f2v = (coeff2 == 0.) ? 1. : pow(prev_inv, coeff2);
    double f3v = (coeff3 == 0.) ? 1. : pow(prev_prev_inv, coeff3);
    double fmn = keep ? 1.0 : factormin;
    double factor = safety * f1v * f2v * f3v;
    if (factor < fmn) factor = fmn;
    if (factor > factormax) factor = factormax;
    const double dt_new = h * factor;
    if (inv == 0. || isinf(inv)) inv = 1.;
    if (keep) {
      d->s[d->n] = s1; d->y[d->n] = y1; d->f[d->n] = F[6];
      d->n++;
      prev_prev_inv = prev_inv;
      prev_inv = inv;
      y = y1;
      F[0] = F[6];                                        /* FSAL */
      s0 = s1;
    }
    if (s0 >= s_end) break;
    double sn = s0 + dt_new;
    if (sn > s_end - 1e-10) sn = keep ? s_end : s0 + 0.5 * (s_end - s0);
    s1 = sn;
    if (!(h > 1e-14) || !isfinite(s1)) { status = ABCMB_STATUS_DT_UNDERFLOW; break; }
  }
  *nsteps_out = nsteps;
  return status;
}

/* sol.evaluate(t) and its t-derivative: the cubic Hermite interpolation
 * (ThirdOrderHermitePolynomialInterpolation, coefficients [a, b, k0, y0] in
 * the step fraction, k = h f) of the step interval holding t, chosen as
 * DenseInterpolation does: the first point s_i >= s (searchsorted, side
 * left) closes the interval, clipped to the first and last intervals. */
static double dense_eval(const dense_t* d, double dir, double t, double* dydt) {
  const double s = dir * t;
  int lo = 0, hi = d->n;                         /* first index with s_i >= s */
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (d->s[mid] < s) lo = mid + 1; else hi = mid;
  }
  int j = lo - 1;
  if (j < 0) j = 0;
  if (j > d->n - 2) j = d->n - 2;
  const double h = d->s[j + 1] - d->s[j];
  const double y0 = d->y[j], y1 = d->y[j + 1];
  const double k0 = h * d->f[j], k1 = h * d->f[j + 1];
  const double a = k0 + k1 + 2. * y0 - 2. * y1;
  const double b = -2. * k0 - k1 - 3. * y0 + 3. * y1;
  const double th = (s - d->s[j]) / h;
  if (dydt) *dydt = dir * ((3. * a * th + 2. * b) * th + k0) / h;
  return ((a * th + b) * th + k0) * th + y0;
}

/* d x_e / d lna as jax.grad takes it through BG.xe (background.py:593-603)
 * and fast_interp (ABCMBTools.py:300-308): zero outside the table and where
 * the index is clipped. */
static double xe_slope(const abcmb_cosmo* c, const double* tables, double lna) {
  if (lna < c->lna_xe0 || lna >= c->lna_xe_last) return 0.;
  const int n = c->n_xe;
  const double di = 1. / (c->lna_xe_max - c->lna_xe0) * (double)(n - 1);
  double i = (lna - c->lna_xe0) * di;
  if (!(i > 1.e-6 && i < (double)(n - 1) - 1.e-6)) return 0.;
  int il = (int)floor(i);
  int iu = il + 1 < n - 1 ? il + 1 : n - 1;
  const double* fp = tables + c->off_xe;
  return (fp[iu] - fp[il]) * di;
}

/* omega_r (main.py:581-586): every species' density at a = e^-23 times a^4. */
static double omega_r_of(const abcmb_cosmo* c) {
  const double lna = -23.0, a = exp(lna);
  double rt, pt;
  rho_P_tot(c, lna, &rt, &pt, 0, 0, 0, 0, 0, 0);
  return rt * a * a * a * a / RHO_CRIT_UNIT;
}

/* One cosmology of abcmb_bg_forward: conformal-time table and tau0
 * (background.py:252-319, 88-89), optical depth (682-720), lna_rec and
 * lna_transfer_start (552-564), the line-of-sight arrays of Cl_one_ell
 * (spectrum.py:640-651). */
static int bg_one(abcmb_cosmo* c, double* tables, const abcmb_bg_settings* s, abcmb_bgstat* st,
                  dense_t* dt, dense_t* dk) {
  memset(st, 0, sizeof(*st));
  const double lna_cut = -16.1;
  const double tscale = H0H / C_MPC;                 /* H0_over_h / c_Mpc_over_s */
  const double sq_or = sqrt(omega_r_of(c));
  /* conformal time: analytic before lna_cut, Kvaerno5 after */
  const double tau_cut = exp(lna_cut) / tscale / sq_or;
  int st_tau = quad_solve(rhs_dtau, 1.0, c, tables, lna_cut, 0.0, tau_cut, 1e-5, 1e-8, 1e-8, 0., 1., 0.,
                          s->max_steps_tau, dt, &st->n_steps_tau);
  int st_kap = quad_solve(rhs_dkappa, 1.0, c, tables, 0.0, -10.0, 0.0, -1e-3, 1e-10, 1e-10, 0.4, 0.3, 0.,
                          s->max_steps_kappa, dk, &st->n_steps_kappa);
  st->n_accepted_kappa = dk->n - 1;
  st->status = st_tau != ABCMB_STATUS_OK ? st_tau : st_kap;
  if (st->status != ABCMB_STATUS_OK) return st->status;
  double* tab = tables + c->off_tau;
  for (int i = 0; i < ABCMB_NTAU_TAB; ++i) {
    const double l = linspace_at(ABCMB_LNA_TAU_MIN, ABCMB_LNA_TAU_MAX, ABCMB_NTAU_TAB, i);
    const double ap = exp(l) / tscale / sq_or;
    double v = l > lna_cut ? dense_eval(dt, 1., l, 0) : ap;
    tab[i] = isfinite(v) ? v : ap;
  }
  c->tau0 = oracle_tau(c, tables, 0.);
  st->tau0 = c->tau0;
  /* visibility maximum (first index of the max) on linspace(-8, -4, 1500) */
  int imax = 0;
  double vmax = -INFINITY;
  for (int i = 0; i < 1500; ++i) {
    const double l = linspace_at(-8.0, -4.0, 1500, i);
    const double g = exp(-dense_eval(dk, -1., l, 0)) / oracle_tau_c(c, tables, l);
    if (g > vmax) { vmax = g; imax = i; }
  }
  st->lna_rec = linspace_at(-8.0, -4.0, 1500, imax);
  st->kappa_rec = dense_eval(dk, -1., st->lna_rec, 0);
  /* first lna of linspace(-15, -6, 5000) minimising (aH tau_c - 0.008)^2 */
  int imin = 0;
  double vmin = INFINITY;
  for (int i = 0; i < 5000; ++i) {
    const double l = linspace_at(-15.0, -6.0, 5000, i);
    const double q = oracle_aH(c, l) * oracle_tau_c(c, tables, l) - 0.008;
    if (q * q < vmin) { vmin = q * q; imin = i; }
  }
  c->lna_transfer_start = linspace_at(-15.0, -6.0, 5000, imin);
  st->lna_transfer_start = c->lna_transfer_start;
  /* the six 1-D arrays of Cl_one_ell on PT.lna[:-1] */
  const int nl = s->n_save - 1;
  double* los = tables + c->off_los;
  for (int i = 0; i < nl; ++i) {
    const double l = linspace_at(c->lna_transfer_start, 0.0, s->n_save, i);
    const double aH = oracle_aH(c, l);
    const double tc = oracle_tau_c(c, tables, l);
    double em = 0., g = 0., gp = 0.;
    if (!(l < -10.)) {
      double dkap;
      const double kap = dense_eval(dk, -1., l, &dkap);
      em = exp(-kap);
      g = em / tc;
      gp = g * (-dkap - 2. + xe_slope(c, tables, l) / oracle_xe(c, tables, l));
    }
    los[0 * nl + i] = oracle_tau(c, tables, l);
    los[1 * nl + i] = g;
    los[2 * nl + i] = gp;
    los[3 * nl + i] = aH;
    los[4 * nl + i] = em;
    los[5 * nl + i] = oracle_aH_prime(c, l) * aH;
  }
  return ABCMB_STATUS_OK;
}

/* The optical-depth solve alone with its right-hand side scaled by
 * rhs_scale: how far the reference's step sequence moves under a rounding-
 * level change of the integrand.  Returns the status; *nsteps = attempts,
 * *kappa_end = kappa(-10). */

int oracle_kappa_solve(const abcmb_cosmo* c, const double* tables, double rhs_scale, int max_steps,
                       int* nsteps, double* kappa_end) {
  dense_t d;
  d.s = (double*)malloc(sizeof(double) * 3 * (size_t)(max_steps + 1));
  d.y = d.s + max_steps + 1;
  d.f = d.y + max_steps + 1;
  int st = quad_solve(rhs_dkappa, rhs_scale, c, tables, 0.0, -10.0, 0.0, -1e-3, 1e-10, 1e-10, 0.4, 0.3, 0.,
                      max_steps, &d, nsteps);
  *kappa_end = d.y[d.n - 1];
  free(d.s);
  return st;
}

int oracle_bg_forward(int n_cosmo, abcmb_cosmo* cosmo, double* tables, const abcmb_bg_settings* s,
                      abcmb_bgstat* stat, int n_threads) {
  if (n_cosmo <= 0 || !cosmo || !tables || !s || !stat || s->n_save < 3 || s->max_steps_tau < 1 ||
      s->max_steps_kappa < 1)
    return ABCMB_ERR_ARG;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#else
  (void)n_threads;
#endif
  int bad = 0;
#pragma omp parallel reduction(+ : bad)
  {
    dense_t dt, dk;
    const int nt = s->max_steps_tau + 1, nk = s->max_steps_kappa + 1;
    dt.s = (double*)malloc(sizeof(double) * 3 * nt); dt.y = dt.s + nt; dt.f = dt.y + nt;
    dk.s = (double*)malloc(sizeof(double) * 3 * nk); dk.y = dk.s + nk; dk.f = dk.y + nk;
#pragma omp for schedule(dynamic, 1)
    for (int ci = 0; ci < n_cosmo; ++ci)
      if (bg_one(&cosmo[ci], tables, s, &stat[ci], &dt, &dk) != ABCMB_STATUS_OK) bad++;
    free(dt.s);
    free(dk.s);
  }
  return bad ? ABCMB_ERR_SOLVER : ABCMB_OK;
}

/* sizeof of the C-ABI records, so tests can check the Python layouts. */
int oracle_sizeof(int which) {
  switch (which) {
    case 0: return (int)sizeof(abcmb_cosmo);
    case 1: return (int)sizeof(abcmb_pert_settings);
    case 2: return (int)sizeof(abcmb_kstat);
    case 3: return (int)sizeof(abcmb_los_settings);
    case 4: return (int)sizeof(abcmb_lens_cosmo);
    case 5: return (int)sizeof(abcmb_lens_settings);
    case 6: return (int)sizeof(abcmb_bg_settings);
    case 7: return (int)sizeof(abcmb_bgstat);
  }
  return -1;
}
