// lens.cu -- lensed CMB spectra: SpectrumSolver.lensing_Cl and lensed_Cls
// (abcmb/spectrum.py:349-572) with the reduced Wigner-d recursions of
// abcmb/ABCMBTools.py:16-186.
//
// The reference materialises 13 d matrices of n_mu x n_l doubles (about
// 1.3 GB at l_lens = 3000).  Here every three-term recursion runs in
// registers, one thread per quadrature node mu, sequentially in l; nothing of
// size n_mu x n_l is ever stored.
//   lens_coef_kernel    l-only tables: the recursion coefficients A, B, C of
//                       each (m, n) and the l factors of the X functions
//   limber_prep_kernel  per Limber point: chi, the l-independent part of the
//                       integrand, the lna bracket Pk_lin uses on PT.lna
//   limber_kernel       C_l^phiphi, one thread per l (trapezoid in lna)
//   lens_cgl_kernel     C_gl(mu), C_gl2(mu)              (d11, d1-1)
//   lens_ksi_kernel     xi, xi+, xi-, xi_x at every mu   (all 12 recursions)
//   lens_cl_kernel      sum over mu of xi d w for every l: per-block sums
//                       through a shared-memory transpose (deterministic)
//   lens_final_kernel   fixed-order sum of the block partials
// Every kernel is launched once per call for the whole batch (grid.y or the
// flat index runs over the cosmologies).
#include "common.cuh"

namespace abcmb {

namespace {

constexpr int NPAIR = 12;
// the (m, n) of the d matrices lensed_Cls uses (spectrum.py:478-495); d-11,
// d02 and d-24 are the aliases d1-1, d20 and d4-2 there
enum { P00, P11, P1M1, P2M2, P22, P20, P31, P3M3, P3M1, P40, P4M4, P4M2 };
__constant__ int PAIR_M[NPAIR] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 4, 4, 4};
__constant__ int PAIR_N[NPAIR] = {0, 1, -1, -2, 2, 0, 1, -3, -1, 0, -4, -2};

// l factors: nrm = sqrt(2/(2l+1)) (the d normalisation), 2l+1, l(l+1), the
// square-root prefactors of X220, X121, X132, X242, 8/l/(l+1), 2/sqrt(l(l+1))
enum { LC_NRM, LC_TL, LC_LLP1, LC_S220, LC_S121, LC_S132, LC_S242, LC_C8, LC_C2, LC_N = 10 };
// Limber point record
enum { SC_CHI, SC_FAC, SC_ILO, SC_T, SC_MODE, SC_X, SC_N = 8 };

constexpr int CGL_THREADS = 128;
constexpr int KSI_THREADS = 128;
constexpr int CL_THREADS = 256;
constexpr int CL_CHUNK = CL_THREADS / 32;   // multipoles per transpose (one per warp)

__device__ __forceinline__ double nan_to_zero(double x) { return isnan(x) ? 0. : x; }

// sqrt((2m+1)/2) sqrt((2m)! / ((m+n)! (m-n)!)) (ABCMBTools.py:40-43)
__device__ double base_norm(int m, int n) {
  double f2m = 1., fp = 1., fm = 1.;
  for (int i = 2; i <= 2 * m; ++i) f2m *= (double)i;
  for (int i = 2; i <= m + n; ++i) fp *= (double)i;
  for (int i = 2; i <= m - n; ++i) fm *= (double)i;
  return sqrt((2. * m + 1.) / 2.) * sqrt(f2m / (fp * fm));
}

// d^m_{mn} in the normalised recursion variable: norm cos(b/2)^(m+n) (-sin(b/2))^(m-n)
__device__ double base_val(int m, int n, double cb, double sb) {
  double v = base_norm(m, n);
  for (int i = 0; i < m + n; ++i) v *= cb;
  for (int i = 0; i < m - n; ++i) v *= sb;
  return v;
}

// D_{l+1} = (A mu + B) D_l + C D_{l-1}
struct Rec {
  double d, p;
  __device__ __forceinline__ void init(double base) { d = base; p = 0.; }
  __device__ __forceinline__ void adv(const double* __restrict__ c, double mu) {
    double n = fma(fma(__ldg(c), mu, __ldg(c + 1)), d, __ldg(c + 2) * p);
    p = d;
    d = n;
  }
};

__global__ void lens_coef_kernel(int L, double* __restrict__ rc, double* __restrict__ lc) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l > L) return;
  const double x = (double)l;
  for (int p = 0; p < NPAIR; ++p) {
    const int m = PAIR_M[p], n = PAIR_N[p];
    double A = 0., B = 0., C = 0.;
    if (l >= m) {
      const double normA = sqrt((2. * x + 3.) / (2. * x + 1.));
      const double normC = sqrt((2. * x + 3.) / (2. * x - 1.));
      const double denom = sqrt((x + 1.) * (x + 1.) - (double)(m * m)) * sqrt((x + 1.) * (x + 1.) - (double)(n * n));
      A = nan_to_zero(normA * (x + 1.) * (2. * x + 1.) / denom);
      B = nan_to_zero(-A * m * n / x / (x + 1.));
      C = nan_to_zero(-normC * sqrt(x * x - (double)(m * m)) * sqrt(x * x - (double)(n * n)) / denom * (x + 1.) / x);
    }
    double* r = rc + ((int64_t)l * NPAIR + p) * 3;
    r[0] = A;
    r[1] = B;
    r[2] = C;
  }
  double* q = lc + (int64_t)l * LC_N;
  const double llp1 = x * (x + 1.);
  q[LC_NRM] = sqrt(2. / (2. * x + 1.));
  q[LC_TL] = 2. * x + 1.;
  q[LC_LLP1] = llp1;
  q[LC_S220] = l >= 2 ? 0.25 * sqrt((x + 2.) * (x - 1.) * x * (x + 1.)) : 0.;
  q[LC_S121] = l >= 2 ? -0.5 * sqrt((x + 2.) * (x - 1.)) : 0.;
  q[LC_S132] = l >= 2 ? -0.5 * sqrt((x + 3.) * (x - 2.)) : 0.;
  q[LC_S242] = l >= 3 ? 0.25 * sqrt((x + 4.) * (x + 3.) * (x - 2.) * (x - 3.)) : 0.;
  q[LC_C8] = l >= 1 ? 8. / x / (x + 1.) : 0.;
  q[LC_C2] = l >= 1 ? 2. / sqrt(llp1) : 0.;
  q[LC_N - 1] = 0.;
}

// Per Limber point i of linspace(lna_rec, 0, n_lna) (spectrum.py:419-433):
// chi at lna_safe, the integrand without Pk/k (zero at lna = 0, the masked
// end point), and the bracket jnp.interp(lna', PT.lna, .) uses in Pk_lin with
// lna' = -log(1 + z) recomputed from z as the reference does.
__global__ void limber_prep_kernel(int n_cosmo, const abcmb_cosmo* __restrict__ cosmo,
                                   const abcmb_lens_cosmo* __restrict__ lens, const double* __restrict__ tables,
                                   int n_lna, int n_save, double* __restrict__ sc) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_cosmo * n_lna) return;
  const int ci = g / n_lna, i = g % n_lna;
  const abcmb_cosmo& c = cosmo[ci];
  const abcmb_lens_cosmo& lz = lens[ci];
  const double lna = linspace_at(lz.lna_rec, 0., n_lna, i);
  const double lna_floor = linspace_at(lz.lna_rec, 0., n_lna, n_lna - 2);
  const double ls = lna < 0. ? lna : lna_floor;
  const double chi_rec = c.tau0 - tau_of(c, tables, lz.lna_rec);
  const double chs = c.tau0 - tau_of(c, tables, ls);
  const double window = (chi_rec - chs) / chi_rec / chs;
  const double aH = aH_of(c, ls);
  const double a = exp(ls);
  const double z = 1. / a - 1.;
  const double Omega_m = lz.omega_m / (c.h * c.h);
  const double Omega_L = c.omega_Lambda / (c.h * c.h);
  const double zp3 = (1. + z) * (1. + z) * (1. + z);
  const double Om = (Omega_m * zp3) / ((Omega_m * zp3) + Omega_L);
  const double aH2 = aH * aH;
  const double fac = lna < 0. ? chs / aH * window * window * (9. / 8. / (PI * PI) * (Om * Om) * (aH2 * aH2)) : 0.;
  // jnp.interp(lnap, PT.lna, .) on PT.lna = linspace(lna_transfer_start, 0, n_save)
  const double lnap = -log(1. + z);
  const double lts = c.lna_transfer_start;
  int lo = 0, hi = n_save;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (linspace_at(lts, 0., n_save, mid) <= lnap) lo = mid + 1; else hi = mid;
  }
  const int il = min(max(lo, 1), n_save - 1);
  const double x0 = linspace_at(lts, 0., n_save, il - 1), x1 = linspace_at(lts, 0., n_save, il);
  const double dx = x1 - x0;
  double mode = fabs(dx) <= 2.220446049250313e-16 ? 3. : 0.;
  if (lnap < linspace_at(lts, 0., n_save, 0)) mode = 1.;
  if (lnap > 0.) mode = 2.;
  double* r = sc + (int64_t)g * SC_N;
  r[SC_CHI] = chs;
  r[SC_FAC] = fac;
  r[SC_ILO] = (double)il;
  r[SC_T] = (lnap - x0) / dx;
  r[SC_MODE] = mode;
  r[SC_X] = lna;
}

// delta_m at lna' for PT k column j (Pk_lin's first jnp.interp)
__device__ __forceinline__ double dm_lna(const double* __restrict__ dm, int nk, int n_save, int il, double t, int mode,
                                         int j) {
  if (mode == 1) return __ldg(dm + j);
  if (mode == 2) return __ldg(dm + (int64_t)(n_save - 1) * nk + j);
  const double f0 = __ldg(dm + (int64_t)(il - 1) * nk + j);
  if (mode == 3) return f0;
  const double f1 = __ldg(dm + (int64_t)il * nk + j);
  return f0 + t * (f1 - f0);
}

// C_l^phiphi for l = 2..L, one thread per l (spectrum.py:386-435)
__global__ void limber_kernel(const abcmb_cosmo* __restrict__ cosmo, const double* __restrict__ kbuf,
                              const double* __restrict__ pt, const double* __restrict__ sc, int n_lna, int n_save,
                              int L, double k_pivot, double* __restrict__ clpp) {
  const int ci = blockIdx.y;
  const int l = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  if (l > L) return;
  const abcmb_cosmo& c = cosmo[ci];
  const int nk = c.nk;
  const double* kp = kbuf + c.off_k;
  const double* dm = pt + c.off_pt + (int64_t)ABCMB_F_DELTA_M * n_save * nk;
  const double* scc = sc + (int64_t)ci * n_lna * SC_N;
  const double lh = (double)l + 0.5;
  const double kmin = __ldg(kp), kmax = __ldg(kp + nk - 1);
  double acc = 0., yprev = 0., xprev = 0.;
  for (int i = 0; i < n_lna; ++i) {
    const double* r = scc + (int64_t)i * SC_N;
    const double chs = __ldg(r + SC_CHI), fac = __ldg(r + SC_FAC), t = __ldg(r + SC_T), x = __ldg(r + SC_X);
    const int il = (int)__ldg(r + SC_ILO), mode = (int)__ldg(r + SC_MODE);
    const double k = lh / chs;
    // jnp.interp(k, PT.k, delta_m_lna)
    double d;
    if (k < kmin) {
      d = dm_lna(dm, nk, n_save, il, t, mode, 0);
    } else if (k > kmax) {
      d = dm_lna(dm, nk, n_save, il, t, mode, nk - 1);
    } else {
      int lo = 0, hi = nk;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(kp + mid) <= k) lo = mid + 1; else hi = mid;
      }
      const int j = min(max(lo, 1), nk - 1);
      const double k0 = __ldg(kp + j - 1), k1 = __ldg(kp + j);
      const double d0 = dm_lna(dm, nk, n_save, il, t, mode, j - 1);
      const double dk = k1 - k0;
      d = fabs(dk) <= 2.220446049250313e-16 ? d0 : d0 + ((k - k0) / dk) * (dm_lna(dm, nk, n_save, il, t, mode, j) - d0);
    }
    const double Pk = d * d * (c.A_s * pow(k / k_pivot, c.n_s - 1.) * (2 * PI * PI / (k * k * k)));
    const double y = fac * Pk / k;
    if (i > 0) acc += (x - xprev) * (y + yprev);
    yprev = y;
    xprev = x;
  }
  clpp[(int64_t)ci * (L - 1) + (l - 2)] = 8. * PI * PI / (lh * lh * lh) * (0.5 * acc);
}

// C_gl and C_gl2 (spectrum.py:497-503): one thread per mu node
__global__ void __launch_bounds__(CGL_THREADS) lens_cgl_kernel(int n_mu, int L, const double* __restrict__ mu,
                                                               const double* __restrict__ rc,
                                                               const double* __restrict__ lc,
                                                               const double* __restrict__ clpp,
                                                               double* __restrict__ cgl) {
  const int ci = blockIdx.y;
  const int im = blockIdx.x * blockDim.x + threadIdx.x;
  if (im >= n_mu) return;
  const double x = mu[im];
  const double hb = 0.5 * acos(x);
  const double cb = cos(hb), sb = -sin(hb);
  Rec r11, r1m1;
  r11.init(base_val(1, 1, cb, sb));
  r1m1.init(base_val(1, -1, cb, sb));
  r11.adv(rc + ((int64_t)1 * NPAIR + P11) * 3, x);
  r1m1.adv(rc + ((int64_t)1 * NPAIR + P1M1) * 3, x);
  const double* cp = clpp + (int64_t)ci * (L - 1);
  double a = 0., b = 0.;
  for (int l = 2; l <= L; ++l) {
    const double* q = lc + (int64_t)l * LC_N;
    const double c0 = __ldg(q + LC_TL) * __ldg(q + LC_LLP1) * __ldg(cp + l - 2) * __ldg(q + LC_NRM);
    a = fma(c0, r11.d, a);
    b = fma(c0, r1m1.d, b);
    const double* rl = rc + (int64_t)l * NPAIR * 3;
    r11.adv(rl + P11 * 3, x);
    r1m1.adv(rl + P1M1 * 3, x);
  }
  double* o = cgl + ((int64_t)ci * n_mu + im) * 2;
  o[0] = a * (1. / (4. * PI));
  o[1] = b * (1. / (4. * PI));
}

// xi, xi+, xi-, xi_x at every mu (spectrum.py:505-561).  The X functions
// exp(-(l(l+1) - c) sigma2 / 4) are exp(-l(l+1) sigma2 / 4) exp(c sigma2 / 4):
// one exponential per (mu, l).  The d normalisation sqrt(2/(2l+1)) is common
// to every term at one l and folded into the l coefficient.
__global__ void __launch_bounds__(KSI_THREADS) lens_ksi_kernel(int n_mu, int L, const double* __restrict__ mu,
                                                               const double* __restrict__ rc,
                                                               const double* __restrict__ lc,
                                                               const double* __restrict__ cl_unl,
                                                               const double* __restrict__ cgl,
                                                               double* __restrict__ ksi_out) {
  const int ci = blockIdx.y;
  const int im = blockIdx.x * blockDim.x + threadIdx.x;
  if (im >= n_mu) return;
  const double x = mu[im];
  const double hb = 0.5 * acos(x);
  const double cb = cos(hb), sb = -sin(hb);
  const double* cg = cgl + (int64_t)ci * n_mu * 2;
  const double sigma2 = cg[(int64_t)(n_mu - 1) * 2] - cg[(int64_t)im * 2];
  const double C2 = cg[(int64_t)im * 2 + 1];
  const double C22 = C2 * C2;
  const double e2 = exp(2. * sigma2 / 4.), e4 = exp(4. * sigma2 / 4.), e83 = exp(8. / 3. * sigma2 / 4.);
  const double e203 = exp(20. / 3. * sigma2 / 4.), e10 = exp(10. * sigma2 / 4.);
  const int nl = L - 1;
  const double* cTT = cl_unl + (int64_t)ci * 3 * nl;
  const double* cTE = cTT + nl;
  const double* cEE = cTT + 2 * nl;

  Rec d00, d11, d1m1, d2m2, d22, d20, d31, d3m3, d3m1, d40, d4m4, d4m2;
  d00.init(base_val(0, 0, cb, sb));
  d00.adv(rc + P00 * 3, x);                                  // l = 0 -> 1
  d11.init(base_val(1, 1, cb, sb));
  d1m1.init(base_val(1, -1, cb, sb));
  {
    const double* r1 = rc + (int64_t)1 * NPAIR * 3;           // l = 1 -> 2
    d00.adv(r1 + P00 * 3, x);
    d11.adv(r1 + P11 * 3, x);
    d1m1.adv(r1 + P1M1 * 3, x);
  }
  d2m2.init(base_val(2, -2, cb, sb));
  d22.init(base_val(2, 2, cb, sb));
  d20.init(base_val(2, 0, cb, sb));
  d31.init(0.); d3m3.init(0.); d3m1.init(0.);
  d40.init(0.); d4m4.init(0.); d4m2.init(0.);

  double ksi = 0., ksip = 0., ksim = 0., ksix = 0.;
  for (int l = 2; l <= L; ++l) {
    const double* q = lc + (int64_t)l * LC_N;
    const double llp1 = __ldg(q + LC_LLP1);
    const double tln = __ldg(q + LC_TL) * __ldg(q + LC_NRM);
    const double E = exp(-llp1 * sigma2 / 4.);
    const double X000 = E;
    const double X000p = -llp1 / 4. * E;
    const double X220 = __ldg(q + LC_S220) * E * e2;
    const double X022 = E * e4;
    const double X022p = -(llp1 - 4.) / 4. * X022;
    const double X121 = __ldg(q + LC_S121) * E * e83;
    const double X132 = __ldg(q + LC_S132) * E * e203;
    const double X242 = __ldg(q + LC_S242) * E * e10;
    const double tt = tln * __ldg(cTT + l - 2), te = tln * __ldg(cTE + l - 2), ee = tln * __ldg(cEE + l - 2);
    const double X000p2 = X000p * X000p, X022p2 = X022p * X022p, X2202 = X220 * X220;
    ksi += tt * (X000 * X000 * d00.d + __ldg(q + LC_C8) * C2 * X000p2 * d1m1.d +
                 C22 * (X000p2 * d00.d + X2202 * d2m2.d));
    ksip += ee * (X022 * X022 * d22.d + 2. * C2 * X132 * X121 * d31.d + C22 * (X022p2 * d22.d + X242 * X220 * d40.d));
    ksim += ee * (X022 * X022 * d2m2.d + C2 * (X121 * X121 * d1m1.d + X132 * X132 * d3m3.d) +
                  0.5 * C22 * (2. * X022p2 * d2m2.d + X2202 * d00.d + X242 * X242 * d4m4.d));
    ksix += te * (X022 * X000 * d20.d + C2 * X000p * __ldg(q + LC_C2) * (X121 * d11.d + X132 * d3m1.d) +
                  0.5 * C22 * ((2. * X022p * X000p + X2202) * d20.d + X220 * X242 * d4m2.d));
    if (l == L) break;
    const double* rl = rc + (int64_t)l * NPAIR * 3;
    d00.adv(rl + P00 * 3, x);
    d11.adv(rl + P11 * 3, x);
    d1m1.adv(rl + P1M1 * 3, x);
    d2m2.adv(rl + P2M2 * 3, x);
    d22.adv(rl + P22 * 3, x);
    d20.adv(rl + P20 * 3, x);
    if (l >= 3) {
      d31.adv(rl + P31 * 3, x);
      d3m3.adv(rl + P3M3 * 3, x);
      d3m1.adv(rl + P3M1 * 3, x);
    } else {
      d31.init(base_val(3, 1, cb, sb));
      d3m3.init(base_val(3, -3, cb, sb));
      d3m1.init(base_val(3, -1, cb, sb));
    }
    if (l >= 4) {
      d40.adv(rl + P40 * 3, x);
      d4m4.adv(rl + P4M4 * 3, x);
      d4m2.adv(rl + P4M2 * 3, x);
    } else if (l == 3) {
      d40.init(base_val(4, 0, cb, sb));
      d4m4.init(base_val(4, -4, cb, sb));
      d4m2.init(base_val(4, -2, cb, sb));
    }
  }
  double* o = ksi_out + ((int64_t)ci * n_mu + im) * 4;
  o[0] = ksi * (1. / (4. * PI));
  o[1] = ksip * (1. / (4. * PI));
  o[2] = ksim * (1. / (4. * PI));
  o[3] = ksix * (1. / (4. * PI));
}

// sum_mu w xi d^l for l = 2..l_max (spectrum.py:563-570).  Each thread runs
// the d00, d20, d22, d2-2 recursions of its node; every CL_CHUNK multipoles
// the block transposes its contributions through shared memory and warp w
// reduces multipole l0 + w over the block's nodes.
__global__ void __launch_bounds__(CL_THREADS) lens_cl_kernel(int n_mu, int l_max, const double* __restrict__ mu,
                                                             const double* __restrict__ w,
                                                             const double* __restrict__ rc,
                                                             const double* __restrict__ lc,
                                                             const double* __restrict__ ksi,
                                                             double* __restrict__ partial) {
  __shared__ double sb[CL_CHUNK * 3 * CL_THREADS];
  const int ci = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int im = blockIdx.x * CL_THREADS + tid;
  const bool valid = im < n_mu;
  const double x = valid ? mu[im] : 0.;
  const double wq = valid ? w[im] : 0.;
  const double* kq = ksi + ((int64_t)ci * n_mu + (valid ? im : 0)) * 4;
  const double a = valid ? kq[0] * wq : 0., cp = valid ? kq[1] * wq : 0.;
  const double cm = valid ? kq[2] * wq : 0., b = valid ? kq[3] * wq : 0.;
  const double hb = 0.5 * acos(x);
  const double cb = cos(hb), sbh = -sin(hb);
  Rec d00, d20, d22, d2m2;
  d00.init(base_val(0, 0, cb, sbh));
  d00.adv(rc + P00 * 3, x);
  d00.adv(rc + ((int64_t)NPAIR + P00) * 3, x);
  d20.init(base_val(2, 0, cb, sbh));
  d22.init(base_val(2, 2, cb, sbh));
  d2m2.init(base_val(2, -2, cb, sbh));
  const int nout = l_max - 1;
  const int nblk = gridDim.x;
  for (int l0 = 2; l0 <= l_max; l0 += CL_CHUNK) {
    for (int j = 0; j < CL_CHUNK; ++j) {
      const int l = l0 + j;
      double* s = sb + (j * 3) * CL_THREADS + tid;
      if (l <= l_max) {
        s[0] = a * d00.d;
        s[CL_THREADS] = b * d20.d;
        s[2 * CL_THREADS] = cp * d22.d + cm * d2m2.d;
        if (l < l_max) {
          const double* rl = rc + (int64_t)l * NPAIR * 3;
          d00.adv(rl + P00 * 3, x);
          d20.adv(rl + P20 * 3, x);
          d22.adv(rl + P22 * 3, x);
          d2m2.adv(rl + P2M2 * 3, x);
        }
      } else {
        s[0] = 0.;
        s[CL_THREADS] = 0.;
        s[2 * CL_THREADS] = 0.;
      }
    }
    __syncthreads();
    const int l = l0 + wid;
    if (l <= l_max) {
      const double nrm = __ldg(lc + (int64_t)l * LC_N + LC_NRM);
#pragma unroll
      for (int X = 0; X < 3; ++X) {
        const double* s = sb + (wid * 3 + X) * CL_THREADS;
        double v = 0.;
#pragma unroll
        for (int r = 0; r < CL_THREADS / 32; ++r) v += s[lane + 32 * r];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) partial[(((int64_t)ci * nblk + blockIdx.x) * 3 + X) * nout + (l - 2)] = v * nrm;
      }
    }
    __syncthreads();
  }
}

__global__ void lens_final_kernel(int n_cosmo, int nblk, int l_max, const double* __restrict__ partial,
                                  double* __restrict__ cl) {
  const int nout = l_max - 1;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_cosmo * 3 * nout) return;
  const int ci = g / (3 * nout), X = (g / nout) % 3, i = g % nout;
  double s = 0.;
  for (int bk = 0; bk < nblk; ++bk) s += partial[(((int64_t)ci * nblk + bk) * 3 + X) * nout + i];
  cl[g] = (X == 2 ? 0.5 : 1.) * (2. * PI) * s;
}

int64_t al256(int64_t b) { return (b + 255) / 256 * 256; }

}  // namespace

int64_t lens_workspace_bytes(int n_cosmo, const abcmb_lens_settings& s) {
  const int L = s.l_lens;
  const int nblk = (s.n_mu + CL_THREADS - 1) / CL_THREADS;
  int64_t b = 0;
  b += al256((int64_t)(L + 1) * NPAIR * 3 * 8);             // recursion coefficients
  b += al256((int64_t)(L + 1) * LC_N * 8);                  // l factors
  b += al256((int64_t)n_cosmo * s.n_lna * SC_N * 8);        // Limber points
  b += al256((int64_t)n_cosmo * s.n_mu * 2 * 8);            // C_gl, C_gl2
  b += al256((int64_t)n_cosmo * s.n_mu * 4 * 8);            // xi, xi+, xi-, xi_x
  b += al256((int64_t)n_cosmo * nblk * 3 * (s.l_max - 1) * 8);  // block partials
  return b;
}

cudaError_t launch_lens(int n_cosmo, const abcmb_cosmo* cosmo, const abcmb_lens_cosmo* lens, const double* tables,
                        const double* kbuf, const double* pt, const double* mu, const double* w,
                        const double* cl_unl, const abcmb_lens_settings& s, double* clpp, double* cl, void* ws,
                        cudaStream_t stream) {
  const int L = s.l_lens;
  const int nblk = (s.n_mu + CL_THREADS - 1) / CL_THREADS;
  char* p = static_cast<char*>(ws);
  double* rc = reinterpret_cast<double*>(p); p += al256((int64_t)(L + 1) * NPAIR * 3 * 8);
  double* lc = reinterpret_cast<double*>(p); p += al256((int64_t)(L + 1) * LC_N * 8);
  double* sc = reinterpret_cast<double*>(p); p += al256((int64_t)n_cosmo * s.n_lna * SC_N * 8);
  double* cgl = reinterpret_cast<double*>(p); p += al256((int64_t)n_cosmo * s.n_mu * 2 * 8);
  double* ksi = reinterpret_cast<double*>(p); p += al256((int64_t)n_cosmo * s.n_mu * 4 * 8);
  double* partial = reinterpret_cast<double*>(p);

  lens_coef_kernel<<<(L + 1 + 127) / 128, 128, 0, stream>>>(L, rc, lc);
  const int npts = n_cosmo * s.n_lna;
  limber_prep_kernel<<<(npts + 127) / 128, 128, 0, stream>>>(n_cosmo, cosmo, lens, tables, s.n_lna, s.n_save, sc);
  limber_kernel<<<dim3((L - 1 + 127) / 128, n_cosmo), 128, 0, stream>>>(cosmo, kbuf, pt, sc, s.n_lna, s.n_save, L,
                                                                        s.k_pivot, clpp);
  lens_cgl_kernel<<<dim3((s.n_mu + CGL_THREADS - 1) / CGL_THREADS, n_cosmo), CGL_THREADS, 0, stream>>>(
      s.n_mu, L, mu, rc, lc, clpp, cgl);
  lens_ksi_kernel<<<dim3((s.n_mu + KSI_THREADS - 1) / KSI_THREADS, n_cosmo), KSI_THREADS, 0, stream>>>(
      s.n_mu, L, mu, rc, lc, cl_unl, cgl, ksi);
  lens_cl_kernel<<<dim3(nblk, n_cosmo), CL_THREADS, 0, stream>>>(s.n_mu, s.l_max, mu, w, rc, lc, ksi, partial);
  const int nout = n_cosmo * 3 * (s.l_max - 1);
  lens_final_kernel<<<(nout + 255) / 256, 256, 0, stream>>>(n_cosmo, nblk, s.l_max, partial, cl);
  return cudaGetLastError();
}

}  // namespace abcmb
