// bg.cu -- the background tables the perturbation and line-of-sight kernels
// read, produced on the GPU from the x_e / T_m history:
//
//   conformal time        abcmb/background.py:252-319
//                         (BackgroundPreRecomb._tabulate_conformal_time),
//                         tau0 = BG.tau(0.) at :89
//   optical depth         abcmb/background.py:682-720 (_tabulate_optical_depth),
//                         expmkappa :722-742, visibility :744-768
//   lna_rec, transfer start   abcmb/background.py:552-564
//   line-of-sight arrays  abcmb/spectrum.py:640-651 (tau, g, g' = jax.grad of
//                         the visibility, aH, exp(-kappa), aH_dot)
//
// One block per cosmology.  Warp 0 integrates the conformal time while warp 1
// integrates the optical depth, each with diffrax's Kvaerno5 step, embedded
// error estimate and PID controller.  Both right-hand sides are independent
// of the state, so every implicit stage derivative is the right-hand side at
// the stage time: lanes 1-6 evaluate the six stage times of a step at once
// and the step itself is a few FMAs.  The accepted points (s, y, f) are the
// nodes of the cubic Hermite dense output (ThirdOrderHermitePolynomial-
// Interpolation) and go to the workspace.  The whole block then evaluates
// the outputs: the 10 000-point conformal-time table, the visibility maximum
// on 1500 points, the transfer start on 5000 points and the six arrays on
// the n_save - 1 line-of-sight points.
#include "common.cuh"

namespace abcmb {

constexpr int BG_THREADS = 256;
constexpr double BG_LNA_CUT = -16.1;   // background.py:272

// Kvaerno5 (Kvaerno, BIT 44 (2004) 489-502): stage times, and the rows of
// the tableau a state-independent step needs -- row 6 (embedded solution,
// gamma on stage 6) and row 7 (solution, gamma on stage 7).
static __constant__ double QC[7] = {0.0, 0.52, 1.230333209967908, 0.8957659843500759,
                                    0.43639360985864756, 1.0, 1.0};
static __constant__ double QA6[6] = {0.13855640231268224, 0.0, -0.04245337201752043, 0.02446657898003141,
                                     0.61943039072480676, 0.0};
static __constant__ double QA7[6] = {0.13659751177640291, 0.0, -0.05496908796538376, -0.04118626728321046,
                                     0.62993304899016403, 0.06962479448202728};
constexpr double QG = 0.26;

// tau_c = 1 / (a n_e sigma_T c) in Mpc (background.py:659-680)
__device__ __forceinline__ double bg_tau_c(const abcmb_cosmo& c, const double* tables, double lna) {
  const double a = exp(lna);
  const double ne = nH_of(c, a) * xe_of(c, tables, lna);
  return 1. / a / ne / SIGT / C_CM * C_MPC;
}

// d(aH)/dlna from the second Friedmann equation (background.py:189-208)
__device__ __forceinline__ double aH_prime_of(const abcmb_cosmo& c, double lna) {
  const double a = exp(lna);
  const Rho r = rho_all(c, a);
  return -4. * PI * GN * a * a / 3. / aH_of(c, lna) * (r.tot + 3. * r.P) / (C_MPC * C_MPC);
}

// d x_e / d lna as jax.grad takes it through BG.xe and fast_interp
// (background.py:593-603, ABCMBTools.py:300-308): zero outside the table and
// where the index is clipped.
__device__ __forceinline__ double xe_slope(const abcmb_cosmo& c, const double* tables, double lna) {
  if (lna < c.lna_xe0 || lna >= c.lna_xe_last) return 0.;
  const int n = c.n_xe;
  const double di = 1. / (c.lna_xe_max - c.lna_xe0) * (double)(n - 1);
  const double i = (lna - c.lna_xe0) * di;
  if (!(i > 1.e-6 && i < (double)(n - 1) - 1.e-6)) return 0.;
  const int il = (int)floor(i);
  const int iu = min(il + 1, n - 1);
  const double* fp = tables + c.off_xe;
  return (__ldg(fp + iu) - __ldg(fp + il)) * di;
}

// dtau/dlna = 1/aH (which 0) or dkappa/dlna = -1/(tau_c aH) (which 1)
__device__ __forceinline__ double quad_rhs(int which, const abcmb_cosmo& c, const double* tables, double lna) {
  return which == 0 ? 1. / aH_of(c, lna) : -1. / bg_tau_c(c, tables, lna) / aH_of(c, lna);
}

struct DenseNodes {
  double* s;   // solver time s = dir * t of each accepted point
  double* y;
  double* f;   // dy/ds
};

// diffeqsolve(ODETerm(f), Kvaerno5(), t0, t1, dt0, y0, PIDController(rtol,
// atol, pcoeff, icoeff, dcoeff), SaveAt(dense=True), max_steps) for a
// state-independent f, run by one warp (every lane follows the same control
// flow and holds the same scalars; lane 0 stores the nodes).  Backward solves
// run in s = -t with the negated right-hand side, as diffrax flips time.
// Returns an ABCMB_STATUS_* code; at most max_steps + 1 nodes are written.
__device__ int quad_solve_warp(int which, const abcmb_cosmo& c, const double* tables, double t0, double t1,
                               double y0, double dt0, double rtol, double atol, double pcoeff, double icoeff,
                               double dcoeff, int max_steps, DenseNodes d, int& nsteps_out, int& npts_out,
                               int lane) {
  const unsigned FULL = 0xffffffffu;
  const double dir = t1 < t0 ? -1. : 1.;
  const double err_order = 5.0, safety = 0.9, factormin = 0.2, factormax = 10.0;
  const double coeff1 = (icoeff + pcoeff + dcoeff) / err_order;
  const double coeff2 = -(pcoeff + 2. * dcoeff) / err_order;
  const double coeff3 = dcoeff / err_order;
  const double s_end = dir * t1;
  double s0 = dir * t0;
  double s1 = fmin(s0 + dir * dt0, s_end);
  double y = y0;
  double F0 = dir * quad_rhs(which, c, tables, dir * s0);
  double prev_inv = 1.0, prev_prev_inv = 1.0;
  int status = ABCMB_STATUS_OK, nsteps = 0, npts = 1;
  if (lane == 0) {
    d.s[0] = s0;
    d.y[0] = y;
    d.f[0] = F0;
  }
  while (s0 < s_end) {
    if (nsteps >= max_steps) { status = ABCMB_STATUS_MAX_STEPS; break; }
    ++nsteps;
    const double h = s1 - s0;
    double fl = 0.;
    if (lane >= 1 && lane <= 6) fl = dir * quad_rhs(which, c, tables, dir * (s0 + QC[lane] * h));
    double F[7];
    F[0] = F0;
#pragma unroll
    for (int i = 1; i < 7; ++i) F[i] = __shfl_sync(FULL, fl, i);
    double acc = 0., acce = 0.;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      acc += QA7[j] * F[j];
      acce += (QA7[j] - QA6[j]) * F[j];
    }
    acc += QG * F[6];
    acce += -QG * F[5] + QG * F[6];
    const double y1 = y + h * acc;
    const double err = h * acce;
    double scaled = fabs(err / (atol + rtol * fmax(fabs(y), fabs(y1))));
    if (!isfinite(scaled)) scaled = INFINITY;
    const bool keep = scaled < 1.0;
    double inv = 1.0 / scaled;
    const double f1v = (coeff1 == 0.) ? 1. : pow(inv, coeff1);
    const double f2v = (coeff2 == 0.) ? 1. : pow(prev_inv, coeff2);
    const double f3v = (coeff3 == 0.) ? 1. : pow(prev_prev_inv, coeff3);
    const double factor = fmin(fmax(safety * f1v * f2v * f3v, keep ? 1.0 : factormin), factormax);
    const double dt_new = h * factor;
    if (inv == 0. || isinf(inv)) inv = 1.;
    if (keep) {
      if (lane == 0) {                      // npts <= nsteps <= max_steps: inside the max_steps + 1 nodes
        d.s[npts] = s1;
        d.y[npts] = y1;
        d.f[npts] = F[6];
      }
      ++npts;
      prev_prev_inv = prev_inv;
      prev_inv = inv;
      y = y1;
      F0 = F[6];                            // FSAL
      s0 = s1;
    }
    if (s0 >= s_end) break;
    double sn = s0 + dt_new;
    if (sn > s_end - 1e-10) sn = keep ? s_end : s0 + 0.5 * (s_end - s0);
    s1 = sn;
    if (!(h > 1e-14) || !isfinite(s1)) { status = ABCMB_STATUS_DT_UNDERFLOW; break; }
  }
  nsteps_out = nsteps;
  npts_out = npts;
  return status;
}

// sol.evaluate(t) (and d/dt): the cubic Hermite polynomial, coefficients
// [a, b, k0, y0] in the step fraction with k = h f, of the interval that
// DenseInterpolation picks -- the first node s_i >= s (searchsorted, side
// left) closes it, clipped to the first and last intervals.  Plain loads:
// the nodes were written by this kernel.
__device__ double dense_eval(const DenseNodes& d, int n, double dir, double t, double* dydt) {
  const double s = dir * t;
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (d.s[mid] < s) lo = mid + 1;
    else hi = mid;
  }
  const int j = max(0, min(lo - 1, n - 2));
  const double h = d.s[j + 1] - d.s[j];
  const double y0 = d.y[j], y1 = d.y[j + 1];
  const double k0 = h * d.f[j], k1 = h * d.f[j + 1];
  const double a = k0 + k1 + 2. * y0 - 2. * y1;
  const double b = -2. * k0 - k1 - 3. * y0 + 3. * y1;
  const double th = (s - d.s[j]) / h;
  if (dydt) *dydt = dir * ((3. * a * th + 2. * b) * th + k0) / h;
  return ((a * th + b) * th + k0) * th + y0;
}

// fast_interp on the conformal-time table this kernel wrote (plain loads)
__device__ __forceinline__ double tau_from_table(const double* tab, double lna) {
  double i = (lna - ABCMB_LNA_TAU_MIN) / (ABCMB_LNA_TAU_MAX - ABCMB_LNA_TAU_MIN) * (double)(ABCMB_NTAU_TAB - 1);
  i = fmin(fmax(i, 1.e-6), (double)(ABCMB_NTAU_TAB - 1) - 1.e-6);
  const int il = (int)floor(i);
  const int iu = min(il + 1, ABCMB_NTAU_TAB - 1);
  const double wu = i - (double)il;
  return (1.0 - wu) * tab[il] + wu * tab[iu];
}

// (value, index) reductions that keep the first index of the extremum, as
// jnp.argmax / jnp.argmin do
__device__ __forceinline__ void keep_better(bool want_max, double& v, int& i, double v2, int i2) {
  const bool better = want_max ? (v2 > v) : (v2 < v);
  if (better || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

__device__ int block_arg_extremum(bool want_max, double v, int i, double* sv, int* si) {
  const unsigned FULL = 0xffffffffu;
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_down_sync(FULL, v, o);
    const int i2 = __shfl_down_sync(FULL, i, o);
    keep_better(want_max, v, i, v2, i2);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();                          // sv / si free from any earlier use
  if (lane == 0) {
    sv[wid] = v;
    si[wid] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < BG_THREADS / 32; ++w) keep_better(want_max, v, i, sv[w], si[w]);
    si[0] = i;
  }
  __syncthreads();
  return si[0];
}

struct BgArgs {
  int n_cosmo;
  abcmb_cosmo* cosmo;
  double* tables;
  abcmb_bg_settings s;
  abcmb_bgstat* stat;
  double* nodes;        // per cosmology: 3 (max_steps_tau + 1) + 3 (max_steps_kappa + 1) doubles
  int32_t* solve;       // per cosmology: status, step attempts, dense points of both solves (8 ints)
};

// omega_r (main.py:581-586) and tau_approx's scale (background.py:274-276)
__device__ __forceinline__ void early_radiation(const abcmb_cosmo& c, double& sq_or, double& tscale) {
  const double a_early = exp(-23.0);
  const double omega_r = rho_all(c, a_early).tot * a_early * a_early * a_early * a_early / RHO_CRIT_UNIT;
  sq_or = sqrt(omega_r);
  tscale = H0H / C_MPC;
}

// The two solves of every cosmology: one two-warp block per cosmology (the
// conformal-time solve on warp 0, the optical-depth solve on warp 1), so a
// whole batch runs in one wave; the dense-output nodes go to the workspace,
// the statuses and counts to A.solve.
__global__ void __launch_bounds__(64) bg_solve_kernel(BgArgs A) {
  const int ci = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const abcmb_cosmo c = A.cosmo[ci];
  const int cap_t = A.s.max_steps_tau + 1, cap_k = A.s.max_steps_kappa + 1;
  double* nb = A.nodes + (size_t)ci * 3 * (size_t)(cap_t + cap_k);
  double sq_or, tscale;
  early_radiation(c, sq_or, tscale);
  int ns = 0, np = 0, st;
  if (wid == 0) {
    const DenseNodes Dt{nb, nb + cap_t, nb + 2 * cap_t};
    st = quad_solve_warp(0, c, A.tables, BG_LNA_CUT, 0.0, exp(BG_LNA_CUT) / tscale / sq_or, 1e-5, 1e-8, 1e-8, 0.,
                         1., 0., A.s.max_steps_tau, Dt, ns, np, lane);
  } else {
    double* nk = nb + 3 * (size_t)cap_t;
    const DenseNodes Dk{nk, nk + cap_k, nk + 2 * cap_k};
    st = quad_solve_warp(1, c, A.tables, 0.0, -10.0, 0.0, -1e-3, 1e-10, 1e-10, 0.4, 0.3, 0.,
                         A.s.max_steps_kappa, Dk, ns, np, lane);
  }
  if (lane == 0) {
    int32_t* o = A.solve + (size_t)ci * 8 + 3 * wid;
    o[0] = st;
    o[1] = ns;
    o[2] = np;
  }
}

// Everything after the solves: the conformal-time table, the visibility
// peak and lna_rec, lna_transfer_start and the six line-of-sight arrays; one
// 256-thread block per cosmology.
__global__ void __launch_bounds__(BG_THREADS) bg_kernel(BgArgs A) {
  const int ci = blockIdx.x;
  const int tid = threadIdx.x;
  const abcmb_cosmo c = A.cosmo[ci];
  const int cap_t = A.s.max_steps_tau + 1, cap_k = A.s.max_steps_kappa + 1;
  double* nb = A.nodes + (size_t)ci * 3 * (size_t)(cap_t + cap_k);
  const DenseNodes Dt{nb, nb + cap_t, nb + 2 * cap_t};
  double* nk = nb + 3 * (size_t)cap_t;
  const DenseNodes Dk{nk, nk + cap_k, nk + 2 * cap_k};
  __shared__ double red_v[BG_THREADS / 32];
  __shared__ int red_i[BG_THREADS / 32];
  __shared__ double sh_lts;

  double sq_or, tscale;
  early_radiation(c, sq_or, tscale);
  // the two solves' results (bg_solve_kernel, earlier on the stream)
  const int32_t* sv = A.solve + (size_t)ci * 8;
  const int sh_status[2] = {sv[0], sv[3]}, sh_steps[2] = {sv[1], sv[4]};
  const int status = sh_status[0] != ABCMB_STATUS_OK ? sh_status[0] : sh_status[1];
  const int npt = sv[2], npk = sv[5];
  if (status != ABCMB_STATUS_OK || npt < 2 || npk < 2) {
    if (tid == 0) {
      abcmb_bgstat r{};
      r.status = status != ABCMB_STATUS_OK ? status : ABCMB_STATUS_NONFINITE;
      r.n_steps_tau = sh_steps[0];
      r.n_steps_kappa = sh_steps[1];
      r.n_accepted_kappa = npk - 1;
      A.stat[ci] = r;
    }
    return;                                 // block-uniform: every thread read the same solve record
  }

  // conformal-time table: analytic before lna_cut, dense solution after
  double* tab = A.tables + c.off_tau;
  for (int i = tid; i < ABCMB_NTAU_TAB; i += BG_THREADS) {
    const double l = linspace_at(ABCMB_LNA_TAU_MIN, ABCMB_LNA_TAU_MAX, ABCMB_NTAU_TAB, i);
    const double ap = exp(l) / tscale / sq_or;
    const double v = l > BG_LNA_CUT ? dense_eval(Dt, npt, 1., l, nullptr) : ap;
    tab[i] = isfinite(v) ? v : ap;
  }
  // visibility maximum on linspace(-8, -4, 1500)
  double bv = -INFINITY;
  int bi = 0x7fffffff;
  for (int i = tid; i < 1500; i += BG_THREADS) {
    const double l = linspace_at(-8.0, -4.0, 1500, i);
    const double g = exp(-dense_eval(Dk, npk, -1., l, nullptr)) / bg_tau_c(c, A.tables, l);
    keep_better(true, bv, bi, g, i);
  }
  const int irec = block_arg_extremum(true, bv, bi, red_v, red_i);
  // first minimum of (aH tau_c - 0.008)^2 on linspace(-15, -6, 5000)
  bv = INFINITY;
  bi = 0x7fffffff;
  for (int i = tid; i < 5000; i += BG_THREADS) {
    const double l = linspace_at(-15.0, -6.0, 5000, i);
    const double q = aH_of(c, l) * bg_tau_c(c, A.tables, l) - 0.008;
    keep_better(false, bv, bi, q * q, i);
  }
  const int its = block_arg_extremum(false, bv, bi, red_v, red_i);   // its __syncthreads publish tab too
  if (tid == 0) {
    const double lts = linspace_at(-15.0, -6.0, 5000, its);
    const double lrec = linspace_at(-8.0, -4.0, 1500, irec);
    const double tau0 = tau_from_table(tab, 0.0);
    sh_lts = lts;
    A.cosmo[ci].tau0 = tau0;
    A.cosmo[ci].lna_transfer_start = lts;
    abcmb_bgstat r{};
    r.status = ABCMB_STATUS_OK;
    r.n_steps_tau = sh_steps[0];
    r.n_steps_kappa = sh_steps[1];
    r.n_accepted_kappa = npk - 1;
    r.tau0 = tau0;
    r.lna_rec = lrec;
    r.lna_transfer_start = lts;
    r.kappa_rec = dense_eval(Dk, npk, -1., lrec, nullptr);
    A.stat[ci] = r;
  }
  __syncthreads();
  // the six 1-D arrays of Cl_one_ell on PT.lna[:-1] = linspace(lts, 0, n_save)[:-1]
  const double lts = sh_lts;
  const int nl = A.s.n_save - 1;
  double* los = A.tables + c.off_los;
  for (int i = tid; i < nl; i += BG_THREADS) {
    const double l = linspace_at(lts, 0.0, A.s.n_save, i);
    const double aH = aH_of(c, l);
    const double tc = bg_tau_c(c, A.tables, l);
    double em = 0., g = 0., gp = 0.;
    if (!(l < -10.)) {                      // expmkappa = 0 below lna = -10 (background.py:738-742)
      double dkap;
      const double kap = dense_eval(Dk, npk, -1., l, &dkap);
      em = exp(-kap);
      g = em / tc;
      gp = g * (-dkap - 2. + xe_slope(c, A.tables, l) / xe_of(c, A.tables, l));
    }
    los[0 * nl + i] = tau_from_table(tab, l);
    los[1 * nl + i] = g;
    los[2 * nl + i] = gp;
    los[3 * nl + i] = aH;
    los[4 * nl + i] = em;
    los[5 * nl + i] = aH_prime_of(c, l) * aH;
  }
}

static int64_t bg_nodes_bytes(int n_cosmo, const abcmb_bg_settings& s) {
  return (int64_t)n_cosmo * 3 * ((int64_t)s.max_steps_tau + 1 + (int64_t)s.max_steps_kappa + 1) * 8;
}

int64_t bg_workspace_bytes(int n_cosmo, const abcmb_bg_settings& s) {
  return (bg_nodes_bytes(n_cosmo, s) + 255) / 256 * 256 + (int64_t)n_cosmo * 8 * 4;
}

cudaError_t launch_bg(int n_cosmo, abcmb_cosmo* cosmo, double* tables, const abcmb_bg_settings& s,
                      abcmb_bgstat* stat, void* ws, cudaStream_t stream) {
  char* w = static_cast<char*>(ws);
  BgArgs A{n_cosmo, cosmo, tables, s, stat, reinterpret_cast<double*>(w),
           reinterpret_cast<int32_t*>(w + (bg_nodes_bytes(n_cosmo, s) + 255) / 256 * 256)};
  bg_solve_kernel<<<n_cosmo, 64, 0, stream>>>(A);
  bg_kernel<<<n_cosmo, BG_THREADS, 0, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace abcmb
