// hyrex.cu -- the recombination history of HyRex on the GPU
// (abcmb/hyrex/hyrex.py, helium.py, hydrogen.py, recomb_functions.py).
//
// One warp per cosmology follows the reference's seven phases, each in its
// fixed-size buffer joined the way array_with_padding.concat joins them (the
// next buffer starts after the last finite entry, every buffer keeps its
// length, the rest stays +inf):
//   1 Saha HeII/III on the grid points with z >= 3600      helium.py:156-233
//   2 post-Saha HeII expansion (4000 entries)              helium.py:297-373
//   3 HeII ODE until x_HeII < 1e-4 (4096)                  helium.py:375-565
//   4 post-Saha H expansion (800)                          hydrogen.py:190-276
//   5 EMLA with two-photon correction to z = 700 (8192)    hydrogen.py:278-383
//   6 EMLA + T_m until T_CMB or T_m/T_CMB leave the tables hydrogen.py:385-495
//   7 three-level atom to lna = 0 (8192)                   hydrogen.py:664-780
// The ODE phases are diffrax's diffeqsolve(Kvaerno3, PIDController(rtol,
// atol), dt0 = 1e-3, t1 = inf, SaveAt(ts) on the phase's 5e-4 grid,
// Event(cond)): the event is tested at accepted step ends and ends the solve
// there; the grid points up to that time come from the cubic Hermite dense
// output.  The jax.grad derivatives of the post-Saha expansions are taken in
// forward mode (dual numbers) through the same formulas and table lookups;
// the very-chord Jacobian is a central difference.  The reference runs this
// module on the CPU (main.py:220); here every cosmology of a batch runs at
// once.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>
#include <cmath>

#include "common.cuh"

namespace abcmb {

// constants.py
constexpr double HX_KB = 8.617343e-5;
constexpr double HX_MU_E = 938271999.0 * ME / MH;
constexpr double HX_E21 = 10.198714553953742;
constexpr double HX_RYD = 13.598286071938324;
constexpr double HX_LYA_FREQ = HX_RYD * 3. / 4. / (2. * PI * HBAR);
constexpr double HX_STEF = PI * PI / (60. * HBAR * HBAR * HBAR * C_CM * C_CM);
constexpr double HX_R2S1S = 8.2206;
// recomb_functions.py:16-26
constexpr double HX_TR_MIN = 0.004, HX_TR_MAX = 0.4, HX_TRATIO_MIN = 0.1, HX_TRATIO_MAX = 1.0;
constexpr int HX_NTR = 100, HX_NTM = 40;
// hyrex.py:126-136, helium.py:40, hydrogen.py:53
constexpr double HX_SPACING = 5.0e-4;
constexpr int HX_N_POST_HE = 4000, HX_N_HE_ODE = 4096, HX_N_POST_H = 800, HX_N_LATE = 8192;

struct HyrexTablesDev {
  const double* logA2s;   // [NTR * NTM] log of Alpha_inf column 0
  const double* logA2p;   // column 1
  const double* logR;     // [NTR]
  const double* swift;    // [n_swift * 5]
  const double* swift_x;  // [n_swift] kB x temperature column
  int n_swift;
};

struct Kv3 {
  double a[4][4], c[4], b[4], be[4], g;
};

// forward-mode dual numbers
struct dl {
  double v, d;
};
__device__ __forceinline__ dl dc(double v) { return {v, 0.}; }
__device__ __forceinline__ dl dadd(dl a, dl b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ dl dsub(dl a, dl b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ dl dmul(dl a, dl b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ dl ddiv(dl a, dl b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
__device__ __forceinline__ dl dexp_(dl a) {
  const double e = exp(a.v);
  return {e, a.d * e};
}
__device__ __forceinline__ dl dsqrt_(dl a) {
  const double s = sqrt(a.v);
  return {s, a.d / (2. * s)};
}
__device__ __forceinline__ dl dsc(dl a, double k) { return {a.v * k, a.d * k}; }
__device__ __forceinline__ dl drs(double k, dl a) { return ddiv(dc(k), a); }

struct Hx {
  HyrexTablesDev t;
  int n;
  double l0, l1;
  const double *T, *nH, *H;
  double YHe, omega_b, omega_cdm, Neff;
};

// RecombInputs lookups: fast_interp(lna, grid[0], grid[-1], arr) with its lna derivative
__device__ dl ri_interp(const Hx& h, const double* arr, dl x) {
  const int n = h.n;
  double i = (x.v - h.l0) / (h.l1 - h.l0) * (double)(n - 1);
  double di = x.d / (h.l1 - h.l0) * (double)(n - 1);
  if (i < 1.e-6) { i = 1.e-6; di = 0.; }
  if (i > (double)(n - 1) - 1.e-6) { i = (double)(n - 1) - 1.e-6; di = 0.; }
  const int il = (int)floor(i);
  const int iu = min(il + 1, n - 1);
  const double wu = i - (double)il;
  const double a = __ldg(arr + il), b = __ldg(arr + iu);
  return {(1.0 - wu) * a + wu * b, di * (b - a)};
}
__device__ __forceinline__ dl ri_T(const Hx& h, dl l) { return ri_interp(h, h.T, l); }
__device__ __forceinline__ dl ri_nH(const Hx& h, dl l) { return ri_interp(h, h.nH, l); }
__device__ __forceinline__ dl ri_H(const Hx& h, dl l) { return ri_interp(h, h.H, l); }

// jnp.interp on a uniform increasing axis (clamped), value and fractional index
__device__ double interp_uniform(double x, double x0, double x1, int n, const double* fp) {
  if (x <= x0) return __ldg(fp);
  if (x >= x1) return __ldg(fp + n - 1);
  const double step = (x1 - x0) / (double)(n - 1);
  int i = min((int)floor((x - x0) / step), n - 2);
  const double xa = x0 + (double)i * step;
  return __ldg(fp + i) + (x - xa) / step * (__ldg(fp + i + 1) - __ldg(fp + i));
}
__device__ double frac_index(double x, double x0, double x1, int n) {
  if (x <= x0) return 0.;
  if (x >= x1) return (double)(n - 1);
  const double step = (x1 - x0) / (double)(n - 1);
  int i = min((int)floor((x - x0) / step), n - 2);
  const double xa = x0 + (double)i * step;
  return (double)i + (x - xa) / step;
}
// map_coordinates(table, [a, b], order=1), constant mode
__device__ double bilinear(const double* t, double a, double b) {
  const int a0 = (int)floor(a), b0 = (int)floor(b);
  const double wa = a - a0, wb = b - b0;
  double s = 0.;
  for (int da = 0; da < 2; ++da)
    for (int db = 0; db < 2; ++db) {
      const int ia = a0 + da, ib = b0 + db;
      if (ia < 0 || ia >= HX_NTR || ib < 0 || ib >= HX_NTM) continue;
      s += (da ? wa : 1. - wa) * (db ? wb : 1. - wb) * __ldg(t + ia * HX_NTM + ib);
    }
  return s;
}

// recomb_functions.py
__device__ double alpha_H(double Tm) {
  const double TK = Tm / HX_KB;
  return 1.0 * 4.309e-13 * pow(1.0e-4 * TK, -0.6166) / (1. + 0.6703 * pow(1.0e-4 * TK, 0.5300));
}
__device__ double beta_H(double T) {
  const double ldb = 2. * PI * HBAR * C_CM / sqrt(2. * PI * HX_MU_E * T);
  const double il = 1. / ldb;
  return il * il * il * exp(-HX_RYD / 4. / T) * alpha_H(T) / 4.;
}
__device__ double gamma_compton_hx(double xe, double T, double YHe) {
  const double FHe = YHe * MH / MHE / (1 - YHe);
  return xe / (1. + FHe + xe) * 8. * SIGT * (4. * HX_STEF) * T * T * T * T / (3. * ME);
}
__device__ double xe_saha(double T, double nH, double& s_out) {
  const double ge = pow(2. * PI * HX_MU_E * T, 1.5) / pow(2. * PI * HBAR * C_CM, 3.) / nH;
  const double s = ge * exp(-HX_RYD / T);
  s_out = s;
  return (sqrt(s * s + 4. * s) - s) / 2.;
}

struct Eff {
  double A2s, A2p, B2s, B2p, R2p2s, R2s2p;
};
__device__ void effective_coefficients(const Hx& h, double T, double Tm, Eff& e) {
  const double iT = frac_index(log(T), log(HX_TR_MIN), log(HX_TR_MAX), HX_NTR);
  const double iR = frac_index(Tm / T, HX_TRATIO_MIN, HX_TRATIO_MAX, HX_NTM);
  e.A2s = exp(bilinear(h.t.logA2s, iT, iR));
  e.A2p = exp(bilinear(h.t.logA2p, iT, iR));
  const double E2 = -HX_RYD / 4.;
  const double q = pow(2 * PI * HX_MU_E * T / ((2 * PI * HBAR) * (2 * PI * HBAR)), 1.5) / (C_CM * C_CM * C_CM);
  e.B2s = exp(E2 / T) * q * exp(bilinear(h.t.logA2s, iT, (double)(HX_NTM - 1)));
  e.B2p = (1. / 3.) * exp(E2 / T) * q * exp(bilinear(h.t.logA2p, iT, (double)(HX_NTM - 1)));
  e.R2p2s = exp(interp_uniform(log(T), log(HX_TR_MIN), log(HX_TR_MAX), HX_NTR, h.t.logR));
  e.R2s2p = 3. * e.R2p2s;
}
// HyRec-2 correction function (hydrogen.py:538-575)
__device__ double correction_delta(const Hx& h, double T) {
  const double* sw = h.t.swift;
  const double* xs = h.t.swift_x;
  const int ns = h.t.n_swift;
  int lo = 0, hi = ns - 1;
  const bool below = T <= xs[0], above = T >= xs[ns - 1];
  if (!below && !above)
    while (hi - lo > 1) {
      const int mid = (lo + hi) / 2;
      if (xs[mid] <= T) lo = mid;
      else hi = mid;
    }
  double col[4];
  for (int k = 0; k < 4; ++k) {
    if (below) col[k] = sw[k + 1];
    else if (above) col[k] = sw[(ns - 1) * 5 + k + 1];
    else col[k] = sw[lo * 5 + k + 1] + (T - xs[lo]) / (xs[hi] - xs[lo]) * (sw[hi * 5 + k + 1] - sw[lo * 5 + k + 1]);
  }
  const double omega_H = h.omega_b * (1 - h.YHe);
  const double omega_cb = h.omega_b + h.omega_cdm;
  return col[0] + (omega_cb - 0.14175) * col[1] + (omega_H - 0.01689) * col[2] + (h.Neff - 3.046) * col[3];
}

// dx_e/dlna of the effective multilevel atom (hydrogen.py:497-536, 577-662), dual in x_e
__device__ dl dxe_dlna_twophoton(const Hx& h, dl xe, double T, double Tm, double H, double nH, double Delta) {
  Eff e;
  effective_coefficients(h, T, Tm, e);
  const dl x1s = dsub(dc(1.), xe);
  const double lam = 2. * PI * HBAR * C_CM / HX_RYD * 4. / 3.;
  const dl RLya = ddiv(dc(8. * PI * H / 3. / nH), dsc(x1s, lam * lam * lam));
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
  const dl det = dsub(dmul(T00, T11), dmul(T01, T10));
  const dl x2s = ddiv(dsub(dmul(S0, T11), dmul(T01, S1)), det);
  const dl x2p = ddiv(dsub(dmul(T00, S1), dmul(T10, S0)), det);
  const dl num = dsub(dadd(dsc(x2s, e.B2s), dsc(x2p, e.B2p)), dsc(xe2n, e.A2s + e.A2p));
  return dsc(num, 1. / H);
}

// helium.py
__device__ __forceinline__ double fHe_of(const Hx& h) { return h.YHe / (1. - h.YHe) / 3.97153; }

__device__ dl xHeII_post_saha(const Hx& h, dl lna) {
  const double fHe = fHe_of(h);
  const dl TK = dsc(ri_T(h, lna), 1. / HX_KB);
  const dl nH = ri_nH(h, lna);
  const dl s = ddiv(dmul(dmul(dsc(TK, 4 * 2.414194e15), dsqrt_(TK)), dexp_(drs(-285325., TK))), nH);
  const dl ops = dadd(dc(1.), s);
  const dl inner = dadd(dc(1.), ddiv(dsc(s, 4. * fHe), dmul(ops, ops)));
  return ddiv(ddiv(dsc(s, 2. * fHe), ops), dadd(dc(1.), dsqrt_(inner)));
}

__device__ dl xH1_saha(const Hx& h, dl lna) {
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

__constant__ double HE_GA[7] = {1.976e6, 6.03e6, 1.06e8, 2.18e6, 3.37e7, 1.04e6, 1.51e7};
__constant__ double HE_GE[7] = {6989., 19754., 21539., 28496., 29224., 32414., 32781.};

__device__ dl helium_dxHeIIdlna(const Hx& h, dl xe, dl lna) {
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
  dl g2pinc = ddiv(dc(HE_GA[0]), dsub(dc(1.), dexp_(drs(-HE_GE[0], TK))));
  for (int i = 1; i < 7; ++i) g2pinc = dadd(g2pinc, ddiv(dc(HE_GA[i]), dsub(dexp_(drs(HE_GE[i], TK)), dc(1.))));
  const dl tau2p = dmul(dsc(ddiv(nH, H), 4.277e-8), dsub(dc(fHe), xHeII));
  const dl dnuline = dsc(dmul(g2pinc, tau2p), 1. / (4 * PI * PI));
  const dl tauc = ddiv(dnuline, etacinv);
  const dl enh = dadd(dsqrt_(dadd(dc(1.), dsc(tauc, PI * PI))), ddiv(dsc(tauc, 7.74), dadd(dc(1.), dsc(tauc, 70.))));
  dl pesc = ddiv(enh, tau2p);
  const dl a = dsub(dc(1.), dexp_(dsc(tau2p, -1.023e-7)));
  const dl b = dsub(dsc(dexp_(drs(2947., TK)), 0.964525), dmul(enh, dexp_(drs(-6.14e13, etacinv))));
  pesc = dadd(pesc, ddiv(dmul(a, b), tau2p));
  const dl ydown = dadd(dsc(y2s, 50.94), dmul(dsc(y2p, 1.7989e9), pesc));
  const dl bracket = dsub(dmul(dsub(dc(fHe), xHeII), s), dmul(xHeII, dsub(dadd(xHeII, dc(1.)), xH1)));
  return ddiv(dmul(ydown, bracket), H);
}

// the ODE phases: right-hand sides and events
enum { PH_HE = 0, PH_TWOG = 1, PH_EMLA = 2, PH_TLA = 3 };

// Each right-hand side splits into the quantities that depend on lna alone
// (the RecombInputs lookups, the Saha fractions, the rates of the radiation
// temperature) and the arithmetic in the state.  A step evaluates the first
// part once per distinct stage time, on separate lanes at the step's start;
// its Jacobian columns and chord iterations then run only the second part.
// Both parts apply the reference's operations in the reference's order.
constexpr int HX_NC = 16;

__device__ __forceinline__ double gamma_compton_f(double xe, double T, double FHe) {
  return xe / (1. + FHe + xe) * 8. * SIGT * (4. * HX_STEF) * T * T * T * T / (3. * ME);
}

// the lna-only quantities of phase ph at lna = t
__device__ void phase_cache(const Hx& h, int ph, double t, double* c) {
  const dl lna = dc(t);
  const double T = ri_T(h, lna).v, nH = ri_nH(h, lna).v, H = ri_H(h, lna).v;
  if (ph == PH_HE) {                                                   // helium.py:455-483
    const double xH1 = xH1_saha(h, lna).v;
    const double TK = T * (1. / HX_KB);
    const double s0 = TK * 2.414194e15 * sqrt(TK) / nH * 4.;
    const double etacinv = H * 9.15776e22 / (nH * xH1);
    double g2pinc = HE_GA[0] / (1. - exp(-HE_GE[0] / TK));
    for (int i = 1; i < 7; ++i) g2pinc = g2pinc + HE_GA[i] / (exp(HE_GE[i] / TK) - 1.);
    c[0] = xH1;
    c[1] = nH / H * 4.277e-8;
    c[2] = g2pinc;
    c[3] = etacinv;
    c[4] = s0 * exp(-285325. / TK);                  // s
    c[5] = exp(46090. / TK) / s0 * 50.94;            // y2s 50.94
    c[6] = exp(39101. / TK) / s0 * 3. * 1.7989e9;    // y2p 1.7989e9
    c[7] = exp(2947. / TK) * 0.964525;
    c[8] = exp(-6.14e13 / etacinv);
    c[9] = H;
    c[10] = fHe_of(h);
    return;
  }
  c[0] = T;
  c[1] = nH;
  c[2] = H;
  c[14] = h.YHe * MH / MHE / (1 - h.YHe);             // gamma_compton's FHe
  if (ph == PH_TLA) {                                                  // hydrogen.py:664-702
    const double z = exp(-t) - 1.0;
    const double cl = C_CM / HX_LYA_FREQ;
    const double r21 = 8 * PI * H / (3 * (nH * cl * cl * cl));
    c[3] = 3. * r21 / 4.;
    c[4] = beta_H(ri_T(h, dc(log(1 / (1 + z)))).v);
    return;
  }
  // effective_coefficients' temperature-only rates (hydrogen.py:497-536)
  const double iT = frac_index(log(T), log(HX_TR_MIN), log(HX_TR_MAX), HX_NTR);
  const double E2 = -HX_RYD / 4.;
  const double q = pow(2 * PI * HX_MU_E * T / ((2 * PI * HBAR) * (2 * PI * HBAR)), 1.5) / (C_CM * C_CM * C_CM);
  const double B2s = exp(E2 / T) * q * exp(bilinear(h.t.logA2s, iT, (double)(HX_NTM - 1)));
  const double B2p = (1. / 3.) * exp(E2 / T) * q * exp(bilinear(h.t.logA2p, iT, (double)(HX_NTM - 1)));
  const double R2p2s = exp(interp_uniform(log(T), log(HX_TR_MIN), log(HX_TR_MAX), HX_NTR, h.t.logR));
  const double R2s2p = 3. * R2p2s;
  const double Delta = ph == PH_TWOG ? correction_delta(h, T) : 0.0;
  const double eE21 = exp(-HX_E21 / T);
  c[3] = iT;
  c[4] = B2s;
  c[5] = B2p;
  c[6] = R2p2s;
  c[7] = R2s2p;
  c[8] = 8. * PI * H / 3. / nH;
  c[9] = 1. / (1. + Delta);
  c[10] = eE21 * HX_R2S1S;                           // R1s2s
  c[11] = 3. * eE21;
  c[12] = B2s + R2s2p + HX_R2S1S;
  c[13] = B2p + R2p2s;
  c[15] = 1. / H;
}

// dx_e/dlna of the effective multilevel atom in x_e and T_m, from the cache
__device__ double twophoton_x(const Hx& h, const double* c, double xe, double Tm) {
  const double T = c[0], nH = c[1];
  const double iR = frac_index(Tm / T, HX_TRATIO_MIN, HX_TRATIO_MAX, HX_NTM);
  const double A2s = exp(bilinear(h.t.logA2s, c[3], iR));
  const double A2p = exp(bilinear(h.t.logA2p, c[3], iR));
  const double x1s = 1. - xe;
  const double lam = 2. * PI * HBAR * C_CM / HX_RYD * 4. / 3.;
  const double RLya = c[8] / (x1s * (lam * lam * lam));
  const double R2p1s = RLya * c[9];
  const double R1s2p = R2p1s * c[11];
  const double T00 = c[12], T01 = -c[6], T10 = -c[7];
  const double T11 = c[13] + R2p1s;
  const double xe2n = xe * xe * nH;
  const double S0 = xe2n * A2s + x1s * c[10];
  const double S1 = xe2n * A2p + x1s * R1s2p;
  const double det = T00 * T11 - T01 * T10;
  const double x2s = (S0 * T11 - T01 * S1) / det;
  const double x2p = (T00 * S1 - T10 * S0) / det;
  const double num = x2s * c[4] + x2p * c[5] - xe2n * (A2s + A2p);
  return num * c[15];
}

// the right-hand side of phase ph at the cached time
__device__ void phase_rhs_c(const Hx& h, int ph, const double* c, const double* y, double* f) {
  if (ph == PH_HE) {                                                   // helium.py:455-483
    const double xH1 = c[0], fHe = c[10];
    const double xe = y[0] + xH1;
    const double xHeII = xe - (1. - xH1);
    const double tau2p = c[1] * (fHe - xHeII);
    const double dnuline = c[2] * tau2p * (1. / (4 * PI * PI));
    const double tauc = dnuline / c[3];
    const double enh = sqrt(1. + tauc * (PI * PI)) + tauc * 7.74 / (1. + tauc * 70.);
    double pesc = enh / tau2p;
    const double a = 1. - exp(tau2p * -1.023e-7);
    const double b = c[7] - enh * c[8];
    pesc = pesc + a * b / tau2p;
    const double ydown = c[5] + c[6] * pesc;
    const double bracket = (fHe - xHeII) * c[4] - xHeII * (xHeII + 1. - xH1);
    f[0] = ydown * bracket / c[9];
    return;
  }
  const double T = c[0], nH = c[1], H = c[2];
  if (ph == PH_TLA) {                                                  // hydrogen.py:664-702
    const double xe = y[0], Tm = y[1];
    const double rate_exc = c[3] + (1. - xe) * HX_R2S1S / 4.;
    const double rate_ion = (1 - xe) * c[4];
    const double C = rate_exc / (rate_exc + rate_ion);
    const double dxe_dt = C * (beta_H(Tm) * (1.0 - xe) - alpha_H(Tm) * nH * xe * xe);
    f[0] = dxe_dt / H;
    f[1] = -2.0 * Tm + (gamma_compton_f(xe, T, c[14]) / H) * (T - Tm);
    return;
  }
  const double GC = gamma_compton_f(y[0], T, c[14]);
  if (ph == PH_TWOG) {                                                 // hydrogen.py:278-313
    const double Tm = T * (1. - H / GC);
    f[0] = twophoton_x(h, c, y[0], Tm);
  } else {                                                             // hydrogen.py:385-419
    f[0] = twophoton_x(h, c, y[0], y[1]);
    f[1] = (-2 * H * y[1] + GC * (T - y[1])) / H;
  }
}

__device__ void phase_rhs(const Hx& h, int ph, double t, const double* y, double* f) {
  double c[HX_NC];
  phase_cache(h, ph, t, c);
  phase_rhs_c(h, ph, c, y, f);
}

// the phase's end condition at an accepted step end t (c: the cache at t)
__device__ bool phase_event(int ph, double t, const double* c, const double* y) {
  if (ph == PH_HE) return y[0] - (1. - c[0]) < 1e-4;                        // helium.py:531-538
  if (ph == PH_TWOG) return t > -log(701.);                                  // hydrogen.py:365-367
  if (ph == PH_EMLA) {                                                       // hydrogen.py:470-478
    const double T = c[0];
    const double ratio = fmin(y[1] / T, T / y[1]);
    return T < HX_TR_MIN || ratio < HX_TRATIO_MIN;
  }
  return t > 0.0;                                                            // hydrogen.py:749-751
}

// diffeqsolve(Kvaerno3, PIDController(rtol, atol), dt0 = 1e-3, t1 = inf,
// SaveAt(ts = t0 + spacing * (1..n_save)), Event, max_steps) for m <= 2
// components; the saved points go to ts_a[i] (and ts_b[i]), y_a[i], y_b[i]
// (y_b / ts_b only for m = 2).  At most n_save points are written.
// Every lane of the history's warp runs the solver with the same values;
// lanes 0-3 evaluate the lna-only part of the right-hand side at the three
// implicit stage times and at the step end into sc (4 x HX_NC doubles of
// the warp's shared memory), the 2m right-hand sides of the
// central-difference Jacobian are evaluated by lanes 0 .. 2m-1 at once, and
// an accepted step's save points are written one per lane.
__device__ int kv3_solve(const Hx& h, const Kv3& K, int ph, int m, double t0, const double* y0, double rtol,
                         double atol, int max_steps, int n_save, double* ts_a, double* ts_b, double* y_a,
                         double* y_b, int& n_saved, int& n_steps, int lane, double* sc) {
  const double g = K.g;
  const double coeff1 = 1.0 / 3.0;       // pcoeff 0, icoeff 1, dcoeff 0, error order 3
  const double t_first = t0 + HX_SPACING, t_last = t0 + (double)n_save * HX_SPACING;
  const double tstep = (t_last - t_first) / (double)(n_save - 1);
  double y[2] = {y0[0], m > 1 ? y0[1] : 0.}, y1[2] = {0., 0.}, Fs[4][2], base[2], v[2];
  double t = t0, t1 = t0 + 1e-3;
  phase_rhs(h, ph, t, y, Fs[0]);
  int isave = 0, nsteps = 0, status = ABCMB_STATUS_OK;
  for (;;) {
    if (nsteps >= max_steps) { status = ABCMB_STATUS_MAX_STEPS; break; }
    ++nsteps;
    const double hs = t1 - t;
    const double hg = hs * g;
    __syncwarp();                                   // the previous step's reads of sc are done
    if (lane < 4) phase_cache(h, ph, lane < 3 ? t + K.c[lane + 1] * hs : t1, sc + lane * HX_NC);
    __syncwarp();
    // stage 1's base and first chord argument: its right-hand side runs on
    // lane 2m beside the Jacobian's columns (both at t + c_1 hs)
    double v1[2] = {0., 0.}, fv1[2] = {0., 0.};
    for (int j = 0; j < m; ++j) {
      double acc = 0.;
      acc += K.a[1][0] * Fs[0][j];
      base[j] = y[j] + hs * acc;
      Fs[1][j] = Fs[0][j];                                        // starting guess: previous stage
      v1[j] = base[j] + hg * Fs[1][j];
    }
    double Minv[2][2];
    {
      double J[2][2], z[2];
      for (int j = 0; j < m; ++j) z[j] = y[j] + hs * (K.a[1][0] + g) * Fs[0][j];
      // lane 2 col + 0 / 1: the + / - evaluation of column col
      double fl[2] = {0., 0.};
      {
        // one call site for all 2m + 1 lanes, so they run it together
        const int col = lane >> 1;
        double zz[2] = {v1[0], v1[1]};
        if (col < m) {
          const double d = 1e-7 * fmax(fabs(z[col]), 1e-8);
          zz[0] = z[0];
          zz[1] = m > 1 ? z[1] : 0.;
          if (lane & 1) zz[col] -= d;
          else zz[col] += d;
        }
        if (lane <= 2 * m) phase_rhs_c(h, ph, sc, zz, fl);
      }
      for (int row = 0; row < m; ++row) fv1[row] = __shfl_sync(0xffffffffu, fl[row], 2 * m);
      for (int col = 0; col < m; ++col) {
        const double d = 1e-7 * fmax(fabs(z[col]), 1e-8);
        for (int row = 0; row < m; ++row) {
          const double fp = __shfl_sync(0xffffffffu, fl[row], 2 * col);
          const double fm = __shfl_sync(0xffffffffu, fl[row], 2 * col + 1);
          J[row][col] = (fp - fm) / (2. * d);
        }
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
    bool ok = true;
    for (int i = 1; i < 4 && ok; ++i) {
      const double* ci = sc + (i - 1) * HX_NC;          // the cache at t + c_i hs
      if (i > 1)
        for (int j = 0; j < m; ++j) {
          double acc = 0.;
          for (int k = 0; k < i; ++k) acc += K.a[i][k] * Fs[k][j];
          base[j] = y[j] + hs * acc;
          Fs[i][j] = Fs[i - 1][j];                                // starting guess: previous stage
        }
      double diffsize = INFINITY, diffsize_prev;
      bool conv = false;
      for (int it = 1; it <= 10; ++it) {
        double fv[2], r[2], dx[2];
        for (int j = 0; j < m; ++j) v[j] = base[j] + hg * Fs[i][j];
        if (i == 1 && it == 1) {
          fv[0] = fv1[0];
          fv[1] = fv1[1];
        } else {
          phase_rhs_c(h, ph, ci, v, fv);
        }
        for (int j = 0; j < m; ++j) r[j] = fv[j] - Fs[i][j];
        double ss = 0.;
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
          if (diffsize < 1e-13 || (factor > 0. && factor < 1e-2)) { conv = true; break; }
          if (!isfinite(rate) || rate > 2.) break;
        }
      }
      if (!conv) ok = false;
    }
    double scaled = INFINITY;
    if (ok) {
      double ss = 0.;
      for (int j = 0; j < m; ++j) {
        double acc = 0., acce = 0.;
        for (int k = 0; k < 4; ++k) {
          acc += K.b[k] * Fs[k][j];
          acce += (K.b[k] - K.be[k]) * Fs[k][j];
        }
        y1[j] = y[j] + hs * acc;
        const double err = hs * acce;
        const double sc = atol + rtol * fmax(fabs(y[j]), fabs(y1[j]));
        ss += (err / sc) * (err / sc);
      }
      scaled = sqrt(ss / m);
      if (!isfinite(scaled)) scaled = INFINITY;
    }
    const bool keep = scaled < 1.0;
    const double factor = fmin(fmax(0.9 * pow(1.0 / scaled, coeff1), keep ? 1.0 : 0.2), 10.0);
    const double dt_new = hs * factor;
    if (keep) {
      // the save points this step covers (ts <= t1, a prefix of the
      // increasing grid from isave on), 32 candidates at a time, one per lane
      for (;;) {
        const int js = isave + lane;
        double ts = 0.;
        bool in = false;
        if (js < n_save) {
          ts = (js == n_save - 1) ? t_last : t_first + (double)js * tstep;
          in = ts <= t1;
        }
        const unsigned out = ~__ballot_sync(0xffffffffu, in);
        const int cnt = out ? __ffs(out) - 1 : 32;
        if (lane < cnt) {
          const double th = (ts - t) / hs;
          for (int j = 0; j < m; ++j) {
            const double k0 = hs * Fs[0][j], k1 = hs * Fs[3][j];
            const double a = k0 + k1 + 2. * y[j] - 2. * y1[j];
            const double b = -2. * k0 - k1 - 3. * y[j] + 3. * y1[j];
            const double val = ((a * th + b) * th + k0) * th + y[j];
            if (j == 0) y_a[js] = val;
            else y_b[js] = val;
          }
          ts_a[js] = ts;
          if (ts_b) ts_b[js] = ts;
        }
        isave += cnt;
        if (cnt < 32) break;
      }
      t = t1;
      for (int j = 0; j < m; ++j) {
        y[j] = y1[j];
        Fs[0][j] = Fs[3][j];
      }
      if (phase_event(ph, t, sc + 3 * HX_NC, y)) break;
      if (isave >= n_save) break;
    }
    t1 = t + dt_new;
    if (!(hs > 1e-14) || !isfinite(t1)) { status = ABCMB_STATUS_DT_UNDERFLOW; break; }
  }
  n_saved = isave;
  n_steps = nsteps;
  return status;
}

struct HyrexArgs {
  int n_cosmo, n_grid, cap_xe, cap_tm, n1;
  const double *T, *nH, *H;
  const abcmb_hyrex_params* params;
  double *xe, *lna_xe, *tm, *lna_tm;
  int32_t* info;
  HyrexTablesDev tabs;
  Kv3 K;
};

__global__ void hyrex_fill_kernel(double* a, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = INFINITY;
}

// One history per warp: the scalar path runs on every lane with the same
// values; the grid-point phases (Saha, post-Saha) take 32 points at a time,
// one per lane, the ODE phases split their Jacobian evaluations and their
// saved points across lanes.  The operations per point are those of the
// one-thread formulation (the same steps and phase lengths; the last bits
// may differ where the compiler contracts a product into an FMA).
__global__ void __launch_bounds__(32) hyrex_kernel(HyrexArgs A) {
  const int ci = blockIdx.x;
  if (ci >= A.n_cosmo) return;                    // the whole warp
  const int lane = threadIdx.x;
  const unsigned FULL = 0xffffffffu;
  Hx h;
  h.t = A.tabs;
  h.n = A.n_grid;
  h.l0 = -log(1. + 8000.);
  h.l1 = h.l0 + (double)(A.n_grid - 1) * HX_SPACING;
  h.T = A.T + (size_t)ci * A.n_grid;
  h.nH = A.nH + (size_t)ci * A.n_grid;
  h.H = A.H + (size_t)ci * A.n_grid;
  const abcmb_hyrex_params P = A.params[ci];
  h.YHe = P.YHe;
  h.omega_b = P.omega_b;
  h.omega_cdm = P.omega_cdm;
  h.Neff = P.Neff;
  double* X = A.xe + (size_t)ci * A.cap_xe;
  double* L = A.lna_xe + (size_t)ci * A.cap_xe;
  double* TM = A.tm + (size_t)ci * A.cap_tm;
  double* LT = A.lna_tm + (size_t)ci * A.cap_tm;
  int32_t* info = A.info + (size_t)ci * 16;
  int32_t inf[16] = {0};
  const double fHe = fHe_of(h);
  int xv = 0, xlen = 0, tv = 0, tlen = 0;     // finite entries / joined length of x_e and T_m
  int status = ABCMB_STATUS_OK, nsv = 0, nst = 0;
  __shared__ double sc[4 * HX_NC];                // the ODE phases' per-step caches
  // 1 Saha HeII/III: up to and including the first point with x_HeIII < 1e-9
  {
    int k = 0;
    for (int k0 = 0; k0 < A.n1; k0 += 32) {
      const int kk = k0 + lane;
      bool stop = false;
      double xval = 0., lval = 0.;
      if (kk < A.n1) {
        const double l = h.l0 + (double)kk * HX_SPACING;
        const double T = ri_T(h, dc(l)).v, nHv = ri_nH(h, dc(l)).v;
        const double TK = T / HX_KB;
        const double s = 2.414194e15 * TK * sqrt(TK) * exp(-631462.7 / TK) / nHv;
        const double xHeIII = 2 * s * fHe / (1 + s + fHe) / (1 + sqrt(1 + 4 * s * fHe / ((1 + s + fHe) * (1 + s + fHe))));
        stop = xHeIII < 1e-9;
        xval = 1 + fHe + xHeIII;
        lval = l;
      }
      const unsigned hit = __ballot_sync(FULL, stop);
      const int cnt = hit ? __ffs(hit) : min(32, A.n1 - k0);   // the stopping point is kept
      if (lane < cnt) {
        X[xv + kk] = xval;
        L[xv + kk] = lval;
      }
      k = k0 + cnt;
      if (hit) break;
    }
    __syncwarp();
    xv += k;
    xlen += A.n1;
    inf[0] = k;
  }
  // 2 post-Saha HeII: up to and including the first point where the
  // expansion moves x_e by more than 1e-5
  {
    const double start = L[xv - 1] + HX_SPACING;
    int k = 0;
    for (int k0 = 0; k0 < HX_N_POST_HE; k0 += 32) {
      const int kk = k0 + lane;
      bool stop = false;
      double xval = 0., lval = 0.;
      if (kk < HX_N_POST_HE) {
        const double l = start + (double)kk * HX_SPACING;
        const double xHeII = xHeII_post_saha(h, dc(l)).v;
        const double xH1 = xH1_saha(h, dc(l)).v;
        const double xs = 1 - xH1 + xHeII;
        const dl gx = helium_dxHeIIdlna(h, dl{xs, 1.}, dc(l));
        const dl gl = xHeII_post_saha(h, dl{l, 1.});
        const double x = xs + gl.d / gx.d;
        stop = fabs(xs - x) > 1e-5;
        xval = x;
        lval = l;
      }
      const unsigned hit = __ballot_sync(FULL, stop);
      const int cnt = hit ? __ffs(hit) : min(32, HX_N_POST_HE - k0);   // the stopping point is kept
      if (lane < cnt) {
        X[xv + kk] = xval;
        L[xv + kk] = lval;
      }
      k = k0 + cnt;
      if (hit) break;
    }
    __syncwarp();
    xv += k;
    xlen += HX_N_POST_HE;
    inf[1] = k;
  }
  // 3 HeII ODE
  {
    const double t0 = L[xv - 1];
    const double y0[1] = {X[xv - 1]};
    status = kv3_solve(h, A.K, PH_HE, 1, t0, y0, 1e-6, 1e-9, 4096, HX_N_HE_ODE, L + xv, nullptr, X + xv, nullptr,
                       nsv, nst, lane, sc);
    __syncwarp();
    xv += nsv;
    xlen += HX_N_HE_ODE;
    inf[2] = nsv;
    inf[8] = nst;
  }
  // 4 post-Saha H (same stopping rule as phase 2)
  if (status == ABCMB_STATUS_OK) {
    const double start = L[xv - 1] + HX_SPACING;
    int k = 0;
    for (int k0 = 0; k0 < HX_N_POST_H; k0 += 32) {
      const int kk = k0 + lane;
      bool stop = false;
      double xval = 0., lval = 0.;
      if (kk < HX_N_POST_H) {
        const double l = start + (double)kk * HX_SPACING;
        const double T = ri_T(h, dc(l)).v, nHv = ri_nH(h, dc(l)).v, Hv = ri_H(h, dc(l)).v;
        double s;
        const double xs = xe_saha(T, nHv, s);
        const double dxs = -(HX_RYD / T - 3. / 2.) * xs * xs / (2. * xs + s);
        const dl gx = dxe_dlna_twophoton(h, dl{xs, 1.}, T, T, Hv, nHv, 0.0);
        const double x = xs + dxs / gx.d;
        stop = fabs(xs - x) > 1e-5;
        xval = x;
        lval = l;
      }
      const unsigned hit = __ballot_sync(FULL, stop);
      const int cnt = hit ? __ffs(hit) : min(32, HX_N_POST_H - k0);   // the stopping point is kept
      if (lane < cnt) {
        X[xv + kk] = xval;
        L[xv + kk] = lval;
      }
      k = k0 + cnt;
      if (hit) break;
    }
    __syncwarp();
    xv += k;
    xlen += HX_N_POST_H;
    inf[3] = k;
  }
  // 5 two-photon EMLA to z = 700
  if (status == ABCMB_STATUS_OK) {
    const double t0 = L[xv - 1];
    const double y0[1] = {X[xv - 1]};
    status = kv3_solve(h, A.K, PH_TWOG, 1, t0, y0, 1e-6, 1e-9, 4096, HX_N_LATE, L + xv, nullptr, X + xv, nullptr,
                       nsv, nst, lane, sc);
    __syncwarp();
    xv += nsv;
    xlen += HX_N_LATE;
    inf[4] = nsv;
    inf[9] = nst;
  }
  // 6 EMLA with T_m
  if (status == ABCMB_STATUS_OK) {
    const double t0 = L[xv - 1];
    const double x0 = X[xv - 1];
    const double T0 = ri_T(h, dc(t0)).v;
    const double y0[2] = {x0, T0 * (1. - ri_H(h, dc(t0)).v / gamma_compton_hx(x0, T0, h.YHe))};
    status = kv3_solve(h, A.K, PH_EMLA, 2, t0, y0, 1e-6, 1e-9, 4096, HX_N_LATE, L + xv, LT + tv, X + xv, TM + tv,
                       nsv, nst, lane, sc);
    __syncwarp();
    xv += nsv;
    xlen += HX_N_LATE;
    tv += nsv;
    tlen += HX_N_LATE;
    inf[5] = nsv;
    inf[10] = nst;
  }
  if (status == ABCMB_STATUS_OK && tv < 1) status = ABCMB_STATUS_NONFINITE;   // no T_m point to start from
  // 7 three-level atom to lna = 0
  if (status == ABCMB_STATUS_OK) {
    const double t0 = LT[tv - 1];
    const double y0[2] = {X[xv - 1], TM[tv - 1]};
    status = kv3_solve(h, A.K, PH_TLA, 2, t0, y0, 1e-7, 1e-9, 4096, HX_N_LATE, L + xv, LT + tv, X + xv, TM + tv,
                       nsv, nst, lane, sc);
    __syncwarp();
    xv += nsv;
    xlen += HX_N_LATE;
    tv += nsv;
    tlen += HX_N_LATE;
    inf[6] = nsv;
    inf[11] = nst;
  }
  inf[12] = xlen;
  inf[13] = tlen;
  inf[14] = status;
  inf[15] = xv;
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < 16; ++j) info[j] = inf[j];
  }
}

// ------------------------------------------------------------------------
// tables (once per device) and the launcher
// ------------------------------------------------------------------------
namespace {
struct HyrexCache {
  bool ready = false;
  void* mem = nullptr;
  HyrexTablesDev dev{};
};
std::mutex g_hx_mu;
std::vector<HyrexCache> g_hx;
}  // namespace

int hyrex_sizes(int n_grid, int* n_xe, int* n_tm) {
  const double l0 = -std::log(1. + 8000.);
  int n1 = 0;
  for (int i = 0; i < n_grid; ++i)
    if (l0 + (double)i * HX_SPACING <= -std::log(3601.)) n1++;
  *n_xe = n1 + HX_N_POST_HE + HX_N_HE_ODE + HX_N_POST_H + 3 * HX_N_LATE;
  *n_tm = 2 * HX_N_LATE;
  return n1;
}

cudaError_t hyrex_upload_tables(const double* alpha, const double* R, const double* swift, int n_swift) {
  int d = 0;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_hx_mu);
  if ((int)g_hx.size() <= d) g_hx.resize(d + 1);
  HyrexCache& c = g_hx[d];
  const size_t nA = (size_t)HX_NTR * HX_NTM;
  std::vector<double> host(2 * nA + HX_NTR + 5 * (size_t)n_swift + n_swift);
  for (size_t i = 0; i < nA; ++i) {
    host[i] = std::log(alpha[i * 4 + 0]);
    host[nA + i] = std::log(alpha[i * 4 + 1]);
  }
  for (int i = 0; i < HX_NTR; ++i) host[2 * nA + i] = std::log(R[i]);
  double* sw = host.data() + 2 * nA + HX_NTR;
  std::memcpy(sw, swift, sizeof(double) * 5 * (size_t)n_swift);
  for (int i = 0; i < n_swift; ++i) sw[5 * (size_t)n_swift + i] = HX_KB * swift[i * 5];
  if (c.mem) cudaFree(c.mem);
  c.mem = nullptr;
  c.ready = false;
  e = cudaMalloc(&c.mem, host.size() * sizeof(double));
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(c.mem, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  const double* base = static_cast<const double*>(c.mem);
  c.dev.logA2s = base;
  c.dev.logA2p = base + nA;
  c.dev.logR = base + 2 * nA;
  c.dev.swift = base + 2 * nA + HX_NTR;
  c.dev.swift_x = base + 2 * nA + HX_NTR + 5 * (size_t)n_swift;
  c.dev.n_swift = n_swift;
  c.ready = true;
  return cudaSuccess;
}

bool hyrex_tables_ready() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lk(g_hx_mu);
  return (int)g_hx.size() > d && g_hx[d].ready;
}

// RecombInputs on the device (Background.TCMB, nH, H at lna_axis_full,
// background.py:147-166, 349-387; hyrex.py:16-90): one thread per
// (grid point, cosmology); H = sqrt(8 pi G rho_tot / 3) in 1/s from the same
// species densities the perturbation kernels use (rho_all).
__global__ void hyrex_inputs_kernel(int n_cosmo, int n_grid, const abcmb_cosmo* __restrict__ cosmo, double* T,
                                    double* nH, double* H) {
  const int ci = blockIdx.y;
  if (ci >= n_cosmo) return;
  const abcmb_cosmo& c = cosmo[ci];
  // the grid values of numpy's arange (which jnp.arange uses for concrete
  // arguments): start + i * ((start + step) - start)
  const double l0 = -log(1. + 8000.);
  const double dl = (l0 + HX_SPACING) - l0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_grid; i += gridDim.x * blockDim.x) {
    const double a = exp(l0 + (double)i * dl);
    const size_t o = (size_t)ci * n_grid + i;
    T[o] = c.TCMB0 / a;
    nH[o] = nH_of(c, a);
    const Rho r = rho_all(c, a);
    H[o] = sqrt(8. * PI * GN * r.tot / 3.);
  }
}

cudaError_t launch_hyrex_inputs(int n_cosmo, int n_grid, const abcmb_cosmo* cosmo, double* T, double* nH, double* H,
                                cudaStream_t stream) {
  dim3 g((n_grid + 255) / 256, n_cosmo);
  hyrex_inputs_kernel<<<g, 256, 0, stream>>>(n_cosmo, n_grid, cosmo, T, nH, H);
  return cudaGetLastError();
}

cudaError_t launch_hyrex(int n_cosmo, int n_grid, const double* T, const double* nH, const double* H,
                         const abcmb_hyrex_params* params, double* xe, double* lna_xe, double* tm, double* lna_tm,
                         int32_t* info, cudaStream_t stream) {
  int d = 0;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) return e;
  HyrexArgs A{};
  {
    std::lock_guard<std::mutex> lk(g_hx_mu);
    if ((int)g_hx.size() <= d || !g_hx[d].ready) return cudaErrorInvalidValue;
    A.tabs = g_hx[d].dev;
  }
  A.n_cosmo = n_cosmo;
  A.n_grid = n_grid;
  A.n1 = hyrex_sizes(n_grid, &A.cap_xe, &A.cap_tm);
  A.T = T;
  A.nH = nH;
  A.H = H;
  A.params = params;
  A.xe = xe;
  A.lna_xe = lna_xe;
  A.tm = tm;
  A.lna_tm = lna_tm;
  A.info = info;
  // Kvaerno3 tableau (Kvaerno, BIT 44 (2004)): ESDIRK 3(2), stiffly accurate,
  // the embedded solution is stage 3
  const double g = 0.43586652150;
  Kv3& K = A.K;
  std::memset(&K, 0, sizeof(K));
  K.g = g;
  K.a[1][0] = g;
  K.a[2][0] = (-4 * g * g + 6 * g - 1) / (4 * g);
  K.a[2][1] = (-2 * g + 1) / (4 * g);
  K.a[3][0] = (6 * g - 1) / (12 * g);
  K.a[3][1] = -1 / ((24 * g - 12) * g);
  K.a[3][2] = (-6 * g * g + 6 * g - 1) / (6 * g - 3);
  K.c[1] = 2 * g;
  K.c[2] = 1.;
  K.c[3] = 1.;
  for (int j = 0; j < 3; ++j) K.b[j] = K.a[3][j];
  K.b[3] = g;
  K.be[0] = K.a[2][0];
  K.be[1] = K.a[2][1];
  K.be[2] = g;
  K.be[3] = 0.;
  const int64_t nx = (int64_t)n_cosmo * A.cap_xe, nt = (int64_t)n_cosmo * A.cap_tm;
  hyrex_fill_kernel<<<296, 256, 0, stream>>>(xe, nx);
  hyrex_fill_kernel<<<296, 256, 0, stream>>>(lna_xe, nx);
  hyrex_fill_kernel<<<296, 256, 0, stream>>>(tm, nt);
  hyrex_fill_kernel<<<296, 256, 0, stream>>>(lna_tm, nt);
  hyrex_kernel<<<n_cosmo, 32, 0, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace abcmb
