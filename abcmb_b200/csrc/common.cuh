// common.cuh -- device-side background cosmology shared by the kernels.
//
// Every function here restates one evaluator of the reference in FP64:
//   fast_interp                 abcmb/ABCMBTools.py:268-308
//   species rho / P             abcmb/species.py:454-1346
//   aH, aH_prime                abcmb/background.py:147-208
//   tau, nH, TCMB               abcmb/background.py:321-387
//   xe, Tm, tau_c               abcmb/background.py:568-680
//   Gamma_compton               abcmb/hyrex/recomb_functions.py:127-153
//   Baryon.cs2, mean_mass       abcmb/species.py:1163-1220
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/abcmb_b200.h"

namespace abcmb {

// constants.py
constexpr double C_CM = 29979245800.0;
constexpr double C_MPC = 9.71561e-15;
constexpr double H0H = 3.24078e-18;
constexpr double HBAR = 6.582119569509e-16;
constexpr double GN = 1.18980205e-40;
constexpr double MP = 938271999.0;
constexpr double ME = 510998.9461;
constexpr double MH = MP + ME + 13.5982860719383;
constexpr double MHE = 3.72839e9;
constexpr double SIGT = 6.652458734e-25;
constexpr double PI = 3.14159265358979323846;
constexpr double STEF_BOLT = PI * PI / (60. * HBAR * HBAR * HBAR * C_CM * C_CM);
constexpr double RHO_CRIT_UNIT = 3. * H0H * H0H / 8. / PI / GN;
constexpr double CHB3 = (C_CM * HBAR) * (C_CM * HBAR) * (C_CM * HBAR);
constexpr double HB3C3 = (HBAR * HBAR * HBAR) * (C_CM * C_CM * C_CM);

// MassiveNeutrino quadratures (species.py:791-794)
static __constant__ double Q3[3] = {0.913201, 3.37517, 7.79184};
static __constant__ double W3[3] = {0.0687359, 3.31435, 2.29911};
static __constant__ double Q5[5] = {0.583165, 2.0, 4.0, 7.26582, 13.0};
static __constant__ double W5[5] = {0.0081201, 0.689407, 2.8063, 2.05156, 0.12681};

__device__ __forceinline__ double fast_interp(double x, double xp_min, double xp_max,
                                              const double* __restrict__ fp, int n) {
  const double eps = 1.e-6;
  double i = (x - xp_min) / (xp_max - xp_min) * (double)(n - 1);
  i = fmin(fmax(i, eps), (double)(n - 1) - eps);
  int il = (int)floor(i);
  int iu = min(il + 1, n - 1);
  double wu = i - (double)il;
  double wl = 1.0 - wu;
  return wl * __ldg(fp + il) + wu * __ldg(fp + iu);
}

// fast_interp on a table held in shared memory (no read-only-cache loads).
__device__ __forceinline__ double fast_interp_smem(double x, double xp_min, double xp_max, const double* fp, int n) {
  const double eps = 1.e-6;
  double i = (x - xp_min) / (xp_max - xp_min) * (double)(n - 1);
  i = fmin(fmax(i, eps), (double)(n - 1) - eps);
  int il = (int)floor(i);
  int iu = min(il + 1, n - 1);
  double wu = i - (double)il;
  double wl = 1.0 - wu;
  return wl * fp[il] + wu * fp[iu];
}

// jnp.linspace(a, b, n)[i]
__device__ __forceinline__ double linspace_at(double a, double b, int n, int i) {
  return (i == n - 1) ? b : a + (double)i * ((b - a) / (double)(n - 1));
}

struct Rho {
  double tot, P, cdm, b, g, nu, ncdm, Pncdm;
};

__device__ __forceinline__ void rho_ncdm(const abcmb_cosmo& c, double a, double& rho, double& P) {
  double T = c.T_nu_massive * c.TCMB0 / a;
  double x = c.m_nu_massive / T;
  double ir = 0., ip = 0.;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    double q = Q5[j];
    double e = sqrt(q * q + x * x);
    ir += (1. + exp(-q)) / (q * q) * e * W5[j];
    ip += (1. + exp(-q)) / e * W5[j];
  }
  double T4 = T * T * T * T;
  rho = c.N_nu_massive * 4. * T4 / (PI * PI) * ir / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
  P = c.N_nu_massive * 4. / 3. * T4 / (PI * PI) * ip / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
}

__device__ __forceinline__ Rho rho_all(const abcmb_cosmo& c, double a) {
  Rho r;
  double a3 = a * a * a, a4 = a3 * a;
  double rde = c.omega_Lambda * RHO_CRIT_UNIT;
  r.cdm = c.omega_cdm * RHO_CRIT_UNIT / a3;
  r.b = c.omega_b * RHO_CRIT_UNIT / a3;
  double T04 = c.TCMB0 * c.TCMB0 * c.TCMB0 * c.TCMB0;
  r.g = PI * PI / 15. * T04 / a4 / CHB3;
  double tn = c.T_nu_massless;
  r.nu = c.N_nu_massless * 2. * 7. / 8. * PI * PI / 30. * (tn * tn * tn * tn) * T04 / a4 / CHB3;
  r.ncdm = 0.;
  r.Pncdm = 0.;
  if (c.has_ncdm) rho_ncdm(c, a, r.ncdm, r.Pncdm);
  r.tot = rde + r.cdm + r.b + r.g + r.nu + r.ncdm;
  r.P = -rde + r.g / 3. + r.nu / 3. + r.Pncdm;
  return r;
}

__device__ __forceinline__ double aH_of(const abcmb_cosmo& c, double lna) {
  double a = exp(lna);
  Rho r = rho_all(c, a);
  return a * sqrt(8. * PI * GN * r.tot / 3.) / C_MPC;
}

__device__ __forceinline__ double tau_of(const abcmb_cosmo& c, const double* __restrict__ tables, double lna) {
  return fast_interp(lna, ABCMB_LNA_TAU_MIN, ABCMB_LNA_TAU_MAX, tables + c.off_tau, ABCMB_NTAU_TAB);
}

__device__ __forceinline__ double xe_of(const abcmb_cosmo& c, const double* __restrict__ tables, double lna) {
  if (lna < c.lna_xe0) return c.xe_first;
  if (lna >= c.lna_xe_last) return c.xe_last;
  return fast_interp(lna, c.lna_xe0, c.lna_xe_max, tables + c.off_xe, c.n_xe);
}

__device__ __forceinline__ double nH_of(const abcmb_cosmo& c, double a) {
  return (1. - c.YHe) * 3. * c.omega_b * H0H * H0H / 8. / PI / GN / MH / (a * a * a);
}

__device__ __forceinline__ double gamma_compton(double xe, double TCMB, double YHe) {
  double FHe = YHe * MH / MHE / (1. - YHe);
  return xe / (1. + FHe + xe) * 8. * SIGT * (4. * STEF_BOLT) * (TCMB * TCMB * TCMB * TCMB) / (3. * ME);
}

// Device copy of the Bessel tables (abcmb/bessel_tab).
struct BesselDev {
  int n_l, n_x;
  const int32_t* l_tab;
  const double* xmin;   // [3][n_l]
  const double* xmax;   // [3][n_l]
  const double* phi;    // [3][n_l][n_x]
};

// Every background scalar the perturbation equations use at one lna.
struct BG {
  double a, aH, tau, itau_c, cs2, R;   // itau_c = 1 / tau_c
  double iaH;                          // 1 / aH
  double rho_cdm, rho_b, rho_g, rho_nu, rho_ncdm, P_ncdm;
  double ncdm_fac;   // N * 4/pi^2 * T^4 / hbar^3 / c^3
  double eps[3];     // sqrt(q^2 + (m/T)^2) for the 3 perturbation q-bins
};

// fast_interp index of one table (ABCMBTools.py:300-307): lower node and weight
__device__ __forceinline__ void lerp_index(double x, double xp_min, double xp_max, int n, int& il, int& iu,
                                           double& wu) {
  double i = (x - xp_min) / (xp_max - xp_min) * (double)(n - 1);
  i = fmin(fmax(i, 1.e-6), (double)(n - 1) - 1.e-6);
  il = (int)floor(i);
  iu = min(il + 1, n - 1);
  wu = i - (double)il;
}

// Quadrature constants of MassiveNeutrino.rho / P (species.py:835-877),
// w_j (1 + e^{-q_j}) / q_j^2 and w_j (1 + e^{-q_j}), evaluated in FP64.
static __constant__ double R5[5] = {0.03720333831716864, 0.19567702290257588, 0.17860619858834093,
                                    0.038888252814630056, 0.0007503567256353378};
static __constant__ double P5[5] = {0.012652164020403861, 0.7827080916103035, 2.857699177413455,
                                    2.052994097538504, 0.1268102866323721};

// Constant factors of bg_eval, folded at compile time (a division by a
// constant at run time costs a full FP64 division sequence).
constexpr double BG_RHOG = PI * PI / 15. / CHB3;
constexpr double BG_RHONU = (2. * 7. / 8. * PI * PI / 30.) / CHB3;
constexpr double BG_NCDM = 1. / (PI * PI) / HB3C3;
constexpr double BG_NH = 3. * H0H * H0H / 8. / PI / GN / MH;
constexpr double BG_ITAUC = SIGT * C_CM / C_MPC;           // 1/tau_c = n_e a sigma_T c (in Mpc units)
constexpr double BG_IMH = 1. / MH;
constexpr double BG_IME = 1. / ME;
constexpr double BG_ICMPC = 1. / C_MPC;
constexpr double BG_TAU_SCALE = (double)(ABCMB_NTAU_TAB - 1) / (ABCMB_LNA_TAU_MAX - ABCMB_LNA_TAU_MIN);

// Per-cosmology constants of bg_eval, computed once per (cosmology, k) item:
// the x_e and T_m table scales (n - 1) / (lna_max - lna_0) of fast_interp and
// R a = (4/3) rho_g a^4 / (rho_b a^3).
struct BGK {
  double sxe, stm, rfac;
};
__device__ __forceinline__ BGK bg_constants(const abcmb_cosmo& c) {
  BGK k;
  k.sxe = (double)(c.n_xe - 1) / (c.lna_xe_max - c.lna_xe0);
  k.stm = (double)(c.n_tm - 1) / (c.lna_tm_max - c.lna_tm0);
  const double T04 = c.TCMB0 * c.TCMB0 * c.TCMB0 * c.TCMB0;
  k.rfac = 4. / 3. * BG_RHOG * T04 / (c.omega_b * RHO_CRIT_UNIT);
  return k;
}

// fast_interp index with a precomputed scale
__device__ __forceinline__ void lerp_index_scaled(double x, double xp_min, double scale, int n, int& il, int& iu,
                                                  double& wu) {
  double i = (x - xp_min) * scale;
  i = fmin(fmax(i, 1.e-6), (double)(n - 1) - 1.e-6);
  il = (int)floor(i);
  iu = min(il + 1, n - 1);
  wu = i - (double)il;
}

// Every background scalar at one lna.  Same formulas as the reference; the
// three table reads are issued before the density sums so their latencies
// overlap, powers of 1/a replace repeated divisions, and constants are
// folded (this changes only rounding).
__device__ __forceinline__ void bg_eval(const abcmb_cosmo& c, const BGK& K, const double* __restrict__ tables,
                                        double lna, BG& b) {
  int t0, t1, x0, x1, m0, m1;
  double tw, xw, mw;
  {
    double i = (lna - ABCMB_LNA_TAU_MIN) * BG_TAU_SCALE;
    i = fmin(fmax(i, 1.e-6), (double)(ABCMB_NTAU_TAB - 1) - 1.e-6);
    t0 = (int)floor(i);
    t1 = min(t0 + 1, ABCMB_NTAU_TAB - 1);
    tw = i - (double)t0;
  }
  lerp_index_scaled(lna, c.lna_xe0, K.sxe, c.n_xe, x0, x1, xw);
  lerp_index_scaled(lna, c.lna_tm0, K.stm, c.n_tm, m0, m1, mw);
  const double* tt = tables + c.off_tau;
  const double* tx = tables + c.off_xe;
  const double* tm = tables + c.off_tm;
  const double ta = __ldg(tt + t0), tb = __ldg(tt + t1);
  const double xa = __ldg(tx + x0), xb = __ldg(tx + x1);
  const double ma = __ldg(tm + m0), mb = __ldg(tm + m1);
  const double a = exp(lna);
  const double ia = 1. / a;
  const double ia2 = ia * ia, ia3 = ia2 * ia, ia4 = ia2 * ia2;
  b.a = a;
  const double T04 = c.TCMB0 * c.TCMB0 * c.TCMB0 * c.TCMB0;
  const double tn = c.T_nu_massless;
  const double rde = c.omega_Lambda * RHO_CRIT_UNIT;
  b.rho_cdm = c.omega_cdm * RHO_CRIT_UNIT * ia3;
  b.rho_b = c.omega_b * RHO_CRIT_UNIT * ia3;
  b.rho_g = BG_RHOG * T04 * ia4;
  b.rho_nu = c.N_nu_massless * BG_RHONU * (tn * tn * tn * tn) * T04 * ia4;
  b.rho_ncdm = 0.;
  b.P_ncdm = 0.;
  double x = 0.;
  b.ncdm_fac = 0.;
  if (c.has_ncdm) {
    const double T = c.T_nu_massive * c.TCMB0 * ia;
    x = c.m_nu_massive / T;
    double ir = 0., ip = 0.;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const double e2 = Q5[j] * Q5[j] + x * x;
      const double ie = rsqrt(e2);
      ir = fma(R5[j], e2 * ie, ir);
      ip = fma(P5[j], ie, ip);
    }
    const double T4 = T * T * T * T;
    const double f = c.N_nu_massive * T4 * BG_NCDM;
    b.rho_ncdm = 4. * f * ir;
    b.P_ncdm = 4. / 3. * f * ip;
    b.ncdm_fac = 4. * f;
  }
  const double tot = rde + b.rho_cdm + b.rho_b + b.rho_g + b.rho_nu + b.rho_ncdm;
  const double H = sqrt(8. * PI * GN / 3. * tot);
  b.aH = a * H * BG_ICMPC;
  b.tau = (1. - tw) * ta + tw * tb;
  const double xe = (lna < c.lna_xe0) ? c.xe_first : (lna >= c.lna_xe_last) ? c.xe_last : (1. - xw) * xa + xw * xb;
  const double ne = (1. - c.YHe) * c.omega_b * BG_NH * ia3 * xe;
  b.itau_c = ne * a * BG_ITAUC;
  const double TCMB = c.TCMB0 * ia;
  double Tm;
  if (lna < c.lna_tm0) Tm = TCMB * (1. - H / gamma_compton(xe, TCMB, c.YHe));
  else if (lna >= c.lna_tm_last) Tm = c.tm_last;
  else Tm = (1. - mw) * ma + mw * mb;
  const double denom = (1. + xe) * (1. - c.YHe) + MH / MHE * c.YHe;
  const double mu = MH / denom;
  b.R = K.rfac * ia;
  const double iaH = 1. / b.aH;
  b.iaH = iaH;
  b.cs2 = Tm * denom * BG_IMH * (5. / 3. - 2. / 3. * mu * b.R * BG_IME * iaH * b.itau_c * (TCMB / Tm - 1.));
  if (c.has_ncdm) {
#pragma unroll
    for (int i = 0; i < 3; ++i) b.eps[i] = sqrt(Q3[i] * Q3[i] + x * x);
  } else {
    b.eps[0] = b.eps[1] = b.eps[2] = 1.;
  }
}

}  // namespace abcmb
