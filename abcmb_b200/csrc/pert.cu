// pert.cu -- batched perturbation integration, one warp per (cosmology, k).
//
// Restates PerturbationEvolver.evolution_one_k (abcmb/perturbations.py:250-316):
// diffrax.diffeqsolve(ODETerm(get_derivatives), Kvaerno5(),
// PIDController(pcoeff, icoeff, dcoeff, rtol, atol), SaveAt(ts=lna), dt0=1e-2,
// max_steps) followed by make_output_table (perturbations.py:318-404).
//
// Work distribution: a persistent grid; each warp pops (cosmology, k) items
// from a device queue (the host orders them most-expensive first) and keeps
// the whole integration state of its item in shared memory.
//
// Linear algebra: the RHS is linear in y, f = A(lna) y.  The stage root find
// ("very chord": one Jacobian per step, linearised at the first implicit
// stage) needs solves with M = I - h*gamma*A(t_lin).  M is not factored
// densely: every hierarchy's l >= 4 tail is a tridiagonal chain that couples
// to the rest of the system only through its l = 3 element, so the tails are
// eliminated bottom-up (pivots >= 1: the free-streaming couplings have
// opposite signs and the damping is non-negative) and fold into one diagonal
// entry each of a dense "core" block holding eta, delta_c, delta_b, theta_b
// and l <= 3 of every hierarchy (16 unknowns, 28 with massive neutrinos).
// The core is inverted once per step by a warp-parallel Gauss-Jordan with
// partial pivoting; every chord iteration then costs two chain sweeps and a
// core mat-vec instead of a dense LU solve.
#include "common.cuh"

namespace abcmb {

constexpr int WARP = 32;
constexpr int MAX_CORE = 28;
constexpr int NCHAIN = 6;            // F, G, N, Psi(q0), Psi(q1), Psi(q2)
constexpr int NSTART = 10000;        // get_starting_time grid

// Kvaerno5 tableau (Kvaerno, BIT 44 (2004) 489-502), ESDIRK 5(4), 7 stages.
constexpr double KV_G = 0.26;
__constant__ double KV_C[7] = {0.0, 0.52, 1.230333209967908, 0.8957659843500759,
                               0.43639360985864756, 1.0, 1.0};
__constant__ double KV_A[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.26, 0, 0, 0, 0, 0},
    {0.13, 0.84033320996790809, 0, 0, 0, 0},
    {0.22371961478320505, 0.47675532319799699, -0.06470895363112615, 0, 0, 0},
    {0.16648564323248321, 0.10450018841591720, 0.03631482272098715, -0.13090704451073998, 0, 0},
    {0.13855640231268224, 0.0, -0.04245337201752043, 0.02446657898003141, 0.61943039072480676, 0},
    {0.13659751177640291, 0.0, -0.05496908796538376, -0.04118626728321046, 0.62993304899016403,
     0.06962479448202728}};

struct Layout {
  int ny, nc, nchain, ntail;
  int i_g, i_G, i_nu, i_ncdm, nM;
  int ch_start[NCHAIN];   // state index of the l = 4 element
  int ch_L[NCHAIN];       // l_max of the chain
  int ch_off[NCHAIN + 1]; // prefix offsets of the tails
};

__device__ __forceinline__ void make_layout(const abcmb_cosmo& c, Layout& L) {
  L.i_g = 4;
  L.i_G = L.i_g + c.lmax_g + 1;
  L.i_nu = L.i_G + c.lmax_pol_g + 1;
  L.i_ncdm = L.i_nu + c.lmax_nu + 1;
  L.nM = c.has_ncdm ? c.lmax_ncdm + 1 : 0;
  L.ny = L.i_ncdm + 3 * L.nM;
  L.nchain = c.has_ncdm ? 6 : 3;
  L.nc = 4 * (1 + L.nchain);
  L.ch_start[0] = L.i_g + 4;   L.ch_L[0] = c.lmax_g;
  L.ch_start[1] = L.i_G + 4;   L.ch_L[1] = c.lmax_pol_g;
  L.ch_start[2] = L.i_nu + 4;  L.ch_L[2] = c.lmax_nu;
  for (int b = 0; b < 3; ++b) {
    L.ch_start[3 + b] = L.i_ncdm + b * L.nM + 4;
    L.ch_L[3 + b] = c.lmax_ncdm;
  }
  L.ch_off[0] = 0;
  for (int ch = 0; ch < NCHAIN; ++ch)
    L.ch_off[ch + 1] = L.ch_off[ch] + (ch < L.nchain ? L.ch_L[ch] - 3 : 0);
  L.ntail = L.ch_off[L.nchain];
}

// state index of core unknown ci (groups of four: [eta,dc,db,thb], F0-3, G0-3, N0-3, Psi_b 0-3)
__device__ __forceinline__ int core_state(const Layout& L, int ci) {
  int g = ci >> 2, o = ci & 3;
  if (g == 0) return o;
  if (g == 1) return L.i_g + o;
  if (g == 2) return L.i_G + o;
  if (g == 3) return L.i_nu + o;
  return L.i_ncdm + (g - 4) * L.nM + o;
}

// tail element t -> chain, l
__device__ __forceinline__ void tail_elem(const Layout& L, int t, int& ch, int& l) {
  ch = 0;
#pragma unroll
  for (int j = 1; j < NCHAIN; ++j)
    if (t >= L.ch_off[j]) ch = j;
  l = 4 + (t - L.ch_off[ch]);
}

// Per-warp shared-memory arrays.
struct WarpMem {
  double* y0;     // ny
  double* y1;     // ny
  double* F;      // 7 * ny stage derivatives
  double* base;   // ny
  double* v;      // ny
  double* r;      // ny
  double* tA;     // ny  tail coefficient of v[e-1] (per unit chain speed)
  double* tG;     // ny  tail coefficient of v[e+1]
  double* invd;   // ny  tail pivots
  double* mult;   // ny  upward-sweep multipliers
  double* sub;    // ny  tail sub-diagonal of M
  double* Ac;     // ncm * cs   A_core(t) of the current stage
  double* Mc;     // ncm * cs   (I - h g A_core(t_lin))^-1 after inversion
  double* wv;     // 2 * ncm    metric functionals w_h, w_eta
  double* vc;     // ncm        gathered core vector
  double* ch;     // 4 * NCHAIN chain speed, damping, trunc, M_{3,4} inv_d_4
  int* perm;      // ncm
  int ncm, cs;    // core capacity (16 or 28) and row stride
};

__host__ __device__ inline size_t warp_mem_doubles(int max_ny, int ncm) {
  return (size_t)17 * max_ny + 2 * (size_t)ncm * (ncm + 1) + 3 * ncm + 4 * NCHAIN + ncm / 2 + 2;
}

__device__ __forceinline__ void carve(double* p, int max_ny, int ncm, WarpMem& m) {
  m.ncm = ncm;
  m.cs = ncm + 1;
  m.y0 = p; p += max_ny;
  m.y1 = p; p += max_ny;
  m.F = p; p += 7 * max_ny;
  m.base = p; p += max_ny;
  m.v = p; p += max_ny;
  m.r = p; p += max_ny;
  m.tA = p; p += max_ny;
  m.tG = p; p += max_ny;
  m.invd = p; p += max_ny;
  m.mult = p; p += max_ny;
  m.sub = p; p += max_ny;
  m.Ac = p; p += ncm * m.cs;
  m.Mc = p; p += ncm * m.cs;
  m.wv = p; p += 2 * ncm;
  m.vc = p; p += ncm;
  m.ch = p; p += 4 * NCHAIN;
  m.perm = reinterpret_cast<int*>(p);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// A_core(t) and the chain scalars at one time.  Lane r builds row r.
// ---------------------------------------------------------------------------
__device__ void build_core(const abcmb_cosmo& c, const Layout& L, double k, const BG& b,
                           WarpMem& m, int lane) {
  const int nc = L.nc;
  const double aH = b.aH, tc = b.tau_c;
  const double iaH = 1. / aH;
  const double kap = 1. / aH / tc;                         // 1/(aH tau_c)
  const double Ca2 = 4. * PI * GN * b.a * b.a / (C_MPC * C_MPC);
  const double whf = 2. / (aH * aH) * Ca2;                  // h' per rho*delta
  const double wef = Ca2 / aH / (k * k);                    // eta' per (rho+P) theta
  // metric functionals (perturbations.py:238-239)
  if (lane < nc) {
    double wh = 0., we = 0.;
    int g = lane >> 2, o = lane & 3;
    if (g == 0) {
      if (o == 0) wh = 2. / (aH * aH) * k * k;
      if (o == 1) wh = whf * b.rho_cdm;
      if (o == 2) wh = whf * b.rho_b;
      if (o == 3) we = wef * b.rho_b;
    } else if (g == 1) {
      if (o == 0) wh = whf * b.rho_g;
      if (o == 1) we = wef * (b.rho_g + b.rho_g / 3.);
    } else if (g == 3) {
      if (o == 0) wh = whf * b.rho_nu;
      if (o == 1) we = wef * (b.rho_nu + b.rho_nu / 3.);
    } else if (g >= 4) {
      int bb = g - 4;
      double q = Q3[bb], w = W3[bb];
      if (o == 0) wh = whf * b.ncdm_fac * (w * (1. + exp(-q)) * b.eps[bb] / (q * q));
      if (o == 1) we = wef * b.ncdm_fac * (w * (1. + exp(-q)) / q);
    }
    m.wv[lane] = wh;
    m.wv[m.ncm + lane] = we;
  }
  // chain scalars: speed s, damping, truncation 1/(aH tau)
  if (lane < L.nchain) {
    double s, d;
    if (lane == 0 || lane == 1) { s = k * iaH; d = kap; }
    else if (lane == 2) { s = k * iaH; d = 0.; }
    else { s = Q3[lane - 3] * k / b.eps[lane - 3] * iaH; d = 0.; }
    m.ch[lane] = s;
    m.ch[NCHAIN + lane] = d;
  }
  if (lane == 0) m.ch[2 * NCHAIN] = 1. / aH / b.tau;
  __syncwarp();
  if (lane < nc) {
    double* row = m.Ac + lane * m.cs;
    double uh = 0., ue = 0.;
    int g = lane >> 2, o = lane & 3;
    for (int j = 0; j < nc; ++j) row[j] = 0.;
    const double k2 = k * k;
    if (g == 0) {
      if (o == 0) ue = 1.;
      if (o == 1) uh = -0.5;
      if (o == 2) { uh = -0.5; row[3] = -iaH; }
      if (o == 3) { row[3] = -1. - b.R * kap; row[2] = b.cs2 * k2 * iaH; row[5] = b.R * kap; }
    } else if (g == 1) {            // photon temperature F0..F3
      if (o == 0) { uh = -2. / 3.; row[5] = -4. / 3. * iaH; }
      if (o == 1) { row[4] = k2 / 4. * iaH; row[6] = -k2 * iaH; row[3] = kap; row[5] = -kap; }
      if (o == 2) {
        uh = 2. / 15.; ue = 4. / 5.;
        row[5] = 4. / 15. * iaH; row[7] = -3. / 10. * k * iaH; row[6] = -9. / 10. * kap;
        row[8] = kap / 20.; row[10] = kap / 20.;
      }
      if (o == 3) { row[6] = 6. / 7. * k * iaH; row[7] = -kap; }
    } else if (g == 2) {            // photon polarisation G0..G3
      if (o == 0) { row[9] = -k * iaH; row[8] = -kap + kap / 2.; row[6] = kap; row[10] = kap / 2.; }
      if (o == 1) { row[8] = k / 3. * iaH; row[10] = -2. * k / 3. * iaH; row[9] = -kap; }
      if (o == 2) {
        row[9] = 2. * k / 5. * iaH; row[11] = -3. * k / 5. * iaH; row[10] = -kap + 0.2 * kap / 2.;
        row[6] = 0.2 * kap; row[8] = 0.2 * kap / 2.;
      }
      if (o == 3) { row[10] = 3. * k / 7. * iaH; row[11] = -kap; }
    } else if (g == 3) {            // massless neutrinos N0..N3
      if (o == 0) { uh = -2. / 3.; row[13] = -4. / 3. * iaH; }
      if (o == 1) { row[12] = k2 / 4. * iaH; row[14] = -k2 * iaH; }
      if (o == 2) { uh = 2. / 15.; ue = 4. / 5.; row[13] = 4. / 15. * iaH; row[15] = -3. / 10. * k * iaH; }
      if (o == 3) { row[14] = 6. / 7. * k * iaH; }
    } else {                        // massive neutrino q-bin Psi0..Psi3
      int bb = g - 4, i0 = 4 * g;
      double q = Q3[bb], eps = b.eps[bb];
      double dl = -q / (1. + exp(-q));
      if (o == 0) { uh = dl / 6.; row[i0 + 1] = -q / eps * iaH; }
      if (o == 1) { row[i0 + 0] = q * k2 / 3. / eps * iaH; row[i0 + 2] = -2. * q * k2 / 3. / eps * iaH; }
      if (o == 2) {
        uh = -dl / 15.; ue = -2. / 5. * dl;
        row[i0 + 1] = 2. * q / 5. / eps * iaH; row[i0 + 3] = -3. * q * k / 5. / eps * iaH;
      }
      if (o == 3) { row[i0 + 2] = 3. * q * k / 7. / eps * iaH; }
    }
    if (uh != 0. || ue != 0.)
      for (int j = 0; j < nc; ++j) row[j] += uh * m.wv[j] + ue * m.wv[m.ncm + j];
  }
  __syncwarp();
}

// f = A(t) v, written to out (core rows by lanes < nc, tails round robin).
// Requires build_core for t.  v, out in shared memory; out may alias nothing.
__device__ void apply_A(const Layout& L, const WarpMem& m, const double* v, double* out, int lane) {
  const int nc = L.nc;
  if (lane < nc) m.vc[lane] = v[core_state(L, lane)];
  __syncwarp();
  if (lane < nc) {
    const double* row = m.Ac + lane * m.cs;
    double acc = 0.;
    for (int j = 0; j < nc; ++j) acc = fma(row[j], m.vc[j], acc);
    int g = lane >> 2;
    if ((lane & 3) == 3 && g >= 1) {      // l = 3 row couples to the chain's l = 4
      int chn = g - 1;
      acc += -4. / 7. * m.ch[chn] * v[L.ch_start[chn]];
    }
    out[core_state(L, lane)] = acc;
  }
  const double trunc = m.ch[2 * NCHAIN];
  for (int t = lane; t < L.ntail; t += WARP) {
    int chn, l;
    tail_elem(L, t, chn, l);
    int e = L.ch_start[chn] + (l - 4);
    double s = m.ch[chn], d = m.ch[NCHAIN + chn];
    int Lc = L.ch_L[chn];
    double fv;
    if (l == Lc) fv = s * v[e - 1] - (d + (double)(Lc + 1) * trunc) * v[e];
    else fv = s * (m.tA[e] * v[e - 1] - m.tG[e] * v[e + 1]) - d * v[e];
    out[e] = fv;
  }
  __syncwarp();
}

// Factor M = I - hg A(t_lin): tails (lanes < nchain) then the core inverse.
__device__ void factor_newton(const Layout& L, WarpMem& m, double hg, int lane) {
  const int nc = L.nc;
  // M_core = I - hg A_core
  if (lane < nc) {
    double* row = m.Mc + lane * m.cs;
    const double* arow = m.Ac + lane * m.cs;
    for (int j = 0; j < nc; ++j) row[j] = (j == lane ? 1. : 0.) - hg * arow[j];
  }
  __syncwarp();
  const double trunc = m.ch[2 * NCHAIN];
  if (lane < L.nchain) {
    const int chn = lane;
    const double s = m.ch[chn], d = m.ch[NCHAIN + chn];
    const int Lc = L.ch_L[chn];
    const int e4 = L.ch_start[chn];
    double inv_next = 0., sub_next = 0.;
    for (int l = Lc; l >= 4; --l) {
      int e = e4 + (l - 4);
      double diag, sup, sb;
      if (l == Lc) {
        diag = 1. + hg * (d + (double)(Lc + 1) * trunc);
        sup = 0.;
        sb = -hg * s;
      } else {
        diag = 1. + hg * d;
        sup = hg * s * m.tG[e];
        sb = -hg * s * m.tA[e];
      }
      double dd = diag - sup * sub_next * inv_next;
      double inv = 1. / dd;
      m.invd[e] = inv;
      m.mult[e] = sup * inv_next;
      m.sub[e] = sb;
      inv_next = inv;
      sub_next = sb;
    }
    // fold the tail into the l = 3 diagonal entry of the core
    const double M34 = hg * (4. / 7.) * s;
    const int cc = 4 * (chn + 1) + 3;
    m.Mc[cc * m.cs + cc] -= M34 * sub_next * inv_next;
    m.ch[3 * NCHAIN + chn] = M34 * inv_next;
  }
  __syncwarp();
  // in-place Gauss-Jordan inverse of the core with partial (row) pivoting
  const int CS = m.cs;
  for (int p = 0; p < nc; ++p) {
    double val = (lane >= p && lane < nc) ? fabs(m.Mc[lane * CS + p]) : -1.;
    int idx = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, val, o);
      int oi = __shfl_xor_sync(0xffffffffu, idx, o);
      if (ov > val || (ov == val && oi < idx)) { val = ov; idx = oi; }
    }
    const int q = idx;
    if (lane == 0) m.perm[p] = q;
    if (q != p && lane < nc) {
      double a = m.Mc[p * CS + lane], bq = m.Mc[q * CS + lane];
      m.Mc[p * CS + lane] = bq;
      m.Mc[q * CS + lane] = a;
    }
    __syncwarp();
    const double pinv = 1. / m.Mc[p * CS + p];
    __syncwarp();
    if (lane < nc) m.Mc[p * CS + lane] = (lane == p ? 1. : m.Mc[p * CS + lane]) * pinv;
    __syncwarp();
    if (lane < nc && lane != p) {
      double* row = m.Mc + lane * CS;
      const double* prow = m.Mc + p * CS;
      double f = row[p];
      row[p] = 0.;
      for (int j = 0; j < nc; ++j) row[j] = fma(-f, prow[j], row[j]);
    }
    __syncwarp();
  }
  for (int p = nc - 1; p >= 0; --p) {
    int q = m.perm[p];
    if (q != p && lane < nc) {
      double* row = m.Mc + lane * CS;
      double a = row[p];
      row[p] = row[q];
      row[q] = a;
    }
    __syncwarp();
  }
}

// Solve M x = r in place (r holds the right-hand side on entry).
__device__ void solve_newton(const Layout& L, WarpMem& m, double* r, int lane) {
  const int nc = L.nc;
  // upward sweeps of the tails; the l = 3 right-hand side picks up the tail
  if (lane < L.nchain) {
    const int chn = lane;
    const int e4 = L.ch_start[chn];
    const int Lc = L.ch_L[chn];
    double nxt = r[e4 + (Lc - 4)];
    for (int l = Lc - 1; l >= 4; --l) {
      int e = e4 + (l - 4);
      double val = r[e] - m.mult[e] * nxt;
      r[e] = val;
      nxt = val;
    }
    const int cc = 4 * (chn + 1) + 3;
    m.vc[cc] = r[core_state(L, cc)] - m.ch[3 * NCHAIN + chn] * nxt;
  }
  if (lane < nc && !((lane & 3) == 3 && (lane >> 2) >= 1)) m.vc[lane] = r[core_state(L, lane)];
  __syncwarp();
  double xc = 0.;
  if (lane < nc) {
    const double* row = m.Mc + lane * m.cs;
    for (int j = 0; j < nc; ++j) xc = fma(row[j], m.vc[j], xc);
  }
  __syncwarp();
  if (lane < nc) r[core_state(L, lane)] = xc;
  __syncwarp();
  if (lane < L.nchain) {
    const int chn = lane;
    const int e4 = L.ch_start[chn];
    const int Lc = L.ch_L[chn];
    double prev = r[e4 - 1];
    for (int l = 4; l <= Lc; ++l) {
      int e = e4 + (l - 4);
      double x = (r[e] - m.sub[e] * prev) * m.invd[e];
      r[e] = x;
      prev = x;
    }
  }
  __syncwarp();
}

// Fields of make_output_table at one save point from the interpolated state ys.
__device__ void write_fields(const abcmb_cosmo& c, const Layout& L, const double* tables, double k, double lna,
                             const double* ys, double* pt, int n_save, int isave, int ik, int lane) {
  BG b;
  bg_eval(c, tables, lna, b);
  const double a = b.a, aH = b.aH;
  double srd = b.rho_cdm * ys[1] + b.rho_b * ys[2] + b.rho_g * ys[L.i_g] + b.rho_nu * ys[L.i_nu];
  double srt = (b.rho_b + 0.) * ys[3] + (b.rho_g + b.rho_g / 3.) * ys[L.i_g + 1] +
               (b.rho_nu + b.rho_nu / 3.) * ys[L.i_nu + 1];
  double srs = (b.rho_g + b.rho_g / 3.) * ys[L.i_g + 2] + (b.rho_nu + b.rho_nu / 3.) * ys[L.i_nu + 2];
  double rdm = b.rho_cdm * ys[1] + b.rho_b * ys[2];
  double rm = b.rho_cdm + b.rho_b;
  double nd = 0., nt = 0., ns = 0.;
  if (c.has_ncdm) {
    double r0 = 0., r1 = 0., r2 = 0.;
    for (int i = 0; i < 3; ++i) {
      double q = Q3[i], w = W3[i];
      const double* P = ys + L.i_ncdm + i * L.nM;
      r0 += w * (1. + exp(-q)) * b.eps[i] / (q * q) * P[0];
      r1 += w * (1. + exp(-q)) / q * P[1];
      r2 += w * (1. + exp(-q)) / b.eps[i] * P[2];
    }
    double T = c.T_nu_massive * c.TCMB0 / a;
    double T4 = T * T * T * T;
    double rd = c.N_nu_massive * r0 * 4. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    double rt = c.N_nu_massive * r1 * 4. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    double rs = c.N_nu_massive * r2 * 8. / 3. / (PI * PI) * T4 / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
    srd += rd; srt += rt; srs += rs;
    rdm += rd; rm += b.rho_ncdm;
    double rhoP = b.rho_ncdm + b.P_ncdm;
    nd = rd / b.rho_ncdm; nt = rt / rhoP; ns = rs / rhoP;
  }
  if (lane < ABCMB_NFIELDS) {
    const double eta = ys[0];
    const double hp = 2. / (aH * aH) * (k * k * eta + 4. * PI * GN * a * a / (C_MPC * C_MPC) * srd);
    const double etap = 4. * PI * GN * a * a / aH * srt / (C_MPC * C_MPC) / (k * k);
    const double alpha = aH * (hp + 6. * etap) / 2. / (k * k);
    double val = 0.;
    switch (lane) {
      case ABCMB_F_DELTA_M: val = rdm / rm; break;
      case ABCMB_F_THETA_B_PRIME:
        val = -ys[3] + b.cs2 / aH * (k * k * ys[2]) + b.R / aH / b.tau_c * (ys[L.i_g + 1] - ys[3]);
        break;
      case ABCMB_F_ETA: val = eta; break;
      case ABCMB_F_H_PRIME: val = hp; break;
      case ABCMB_F_ETA_PRIME: val = etap; break;
      case ABCMB_F_ALPHA: val = alpha; break;
      case ABCMB_F_ALPHA_PRIME:
        val = eta / aH - 2. * alpha - 12. * PI * GN * a * a / aH * srs / (C_MPC * C_MPC) / (k * k);
        break;
      case ABCMB_F_CDM_DELTA: val = ys[1]; break;
      case ABCMB_F_B_DELTA: val = ys[2]; break;
      case ABCMB_F_B_THETA: val = ys[3]; break;
      case ABCMB_F_G_DELTA: val = ys[L.i_g]; break;
      case ABCMB_F_G_THETA: val = ys[L.i_g + 1]; break;
      case ABCMB_F_G_SIGMA: val = ys[L.i_g + 2]; break;
      case ABCMB_F_G_G0: val = ys[L.i_G]; break;
      case ABCMB_F_G_G2: val = ys[L.i_G + 2]; break;
      case ABCMB_F_NU_DELTA: val = ys[L.i_nu]; break;
      case ABCMB_F_NU_THETA: val = ys[L.i_nu + 1]; break;
      case ABCMB_F_NU_SIGMA: val = ys[L.i_nu + 2]; break;
      case ABCMB_F_NCDM_DELTA: val = nd; break;
      case ABCMB_F_NCDM_THETA: val = nt; break;
      case ABCMB_F_NCDM_SIGMA: val = ns; break;
    }
    pt[c.off_pt + ((int64_t)lane * n_save + isave) * c.nk + ik] = val;
  }
}

// get_starting_time grids, one block row per cosmology (perturbations.py:119-159).
__global__ void start_grid_kernel(int n_cosmo, const abcmb_cosmo* __restrict__ cosmo,
                                  const double* __restrict__ tables, double* __restrict__ aHg,
                                  double* __restrict__ f1g) {
  const int ci = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= n_cosmo || i >= NSTART) return;
  const abcmb_cosmo& c = cosmo[ci];
  double lna = linspace_at(-20.0, -10.0, NSTART, i);
  double a = exp(lna);
  double aH = aH_of(c, lna);
  double xe = xe_of(c, tables, lna);
  double tc = 1. / a / (nH_of(c, a) * xe) / SIGT / C_CM * C_MPC;
  aHg[(int64_t)ci * NSTART + i] = aH;
  f1g[(int64_t)ci * NSTART + i] = tc * aH;
}

// jnp.interp(x, xp, fp) with xp increasing; xp_i = scale / den[i] when den != null.
__device__ double np_interp_lna(double x, const double* xp, const double* den, double scale) {
  auto X = [&](int i) { return den ? scale / den[i] : xp[i]; };
  int lo = 0, hi = NSTART;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (X(mid) <= x) lo = mid + 1; else hi = mid;
  }
  int i = min(max(lo, 1), NSTART - 1);
  double x0 = X(i - 1), x1 = X(i);
  double f0 = linspace_at(-20.0, -10.0, NSTART, i - 1), f1 = linspace_at(-20.0, -10.0, NSTART, i);
  double dx = x1 - x0;
  double f = (fabs(dx) <= 2.220446049250313e-16) ? f0 : f0 + ((x - x0) / dx) * (f1 - f0);
  if (x < X(0)) f = -20.0;
  if (x > X(NSTART - 1)) f = -10.0;
  return f;
}

__global__ void start_lna1_kernel(int n_cosmo, const double* __restrict__ f1g, double R_tc,
                                  double* __restrict__ lna1) {
  int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= n_cosmo) return;
  lna1[ci] = np_interp_lna(R_tc, f1g + (int64_t)ci * NSTART, nullptr, 0.);
}

struct PertArgs {
  int n_cosmo, n_items, max_ny, ncm;
  const abcmb_cosmo* cosmo;
  const double* tables;
  const double* kbuf;
  const int32_t* items;
  double* pt;
  abcmb_kstat* kstat;
  const double* aHg;
  const double* lna1;
  int* queue;
  abcmb_pert_settings s;
};

__global__ void __launch_bounds__(128) pert_kernel(PertArgs P) {
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  WarpMem m;
  carve(smem + (size_t)wib * warp_mem_doubles(P.max_ny, P.ncm), P.max_ny, P.ncm, m);
  const abcmb_pert_settings& S = P.s;
  const double err_order = 5.0, safety = 0.9, factormin = 0.2, factormax = 10.0;
  const double coeff1 = (S.icoeff + S.pcoeff + S.dcoeff) / err_order;
  const double coeff2 = -(S.pcoeff + 2. * S.dcoeff) / err_order;
  const double coeff3 = S.dcoeff / err_order;
  const double kappa = 1e-2, small_res = 1e-13;
  const int root_max = 10;

  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(P.queue, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= P.n_items) break;
    const int ci = P.items[2 * item], ik = P.items[2 * item + 1];
    const abcmb_cosmo& c = P.cosmo[ci];
    Layout L;
    make_layout(c, L);
    const int n = L.ny;
    const double k = P.kbuf[c.off_k + ik];
    const double rtol = k > S.k_split ? S.rtol_large : S.rtol_small;
    const double atol = k > S.k_split ? S.atol_large : S.atol_small;
    const int nsave = S.n_save;
    const double lts = c.lna_transfer_start;

    // start time (perturbations.py:274-279)
    double lna2 = np_interp_lna(S.R_large, nullptr, P.aHg + (int64_t)ci * NSTART, k);
    double lna_start = fmin(fmin(P.lna1[ci], lna2), -10.);

    // tail coefficients
    for (int t = lane; t < L.ntail; t += WARP) {
      int chn, l;
      tail_elem(L, t, chn, l);
      int e = L.ch_start[chn] + (l - 4);
      m.tA[e] = (double)l / (2. * l + 1.);
      m.tG[e] = (double)(l + 1) / (2. * l + 1.);
    }
    // initial conditions (perturbations.py:161-199 + species y_ini)
    for (int e = lane; e < n; e += WARP) m.y0[e] = 0.;
    __syncwarp();
    if (lane == 0) {
      const double tau_ini = tau_of(c, P.tables, lna_start);
      const double om = c.om, Rn = c.R_nu, Rb = c.R_b;
      const double kt = k * tau_ini;
      m.y0[0] = (1. - k * k * tau_ini * tau_ini / 12. / (15. + 4. * Rn) *
                          (5. + 4. * Rn - (16. * Rn * Rn + 280. * Rn + 325) / 10. / (2. * Rn + 15.) * tau_ini * om));
      m.y0[1] = -(kt * kt) / 4. * (1. - om * tau_ini / 5.);
      m.y0[2] = -(kt * kt) / 4. * (1. - om * tau_ini / 5.);
      const double thb = -k * k * k * k * tau_ini * tau_ini * tau_ini / 36. *
                         (1. - 3. * (1. + 5. * Rb - Rn) / 20. / (1. - Rn) * om * tau_ini);
      m.y0[3] = thb;
      m.y0[L.i_g] = -(kt * kt) / 3. * (1. - om * tau_ini / 5.);
      m.y0[L.i_g + 1] = thb;
      const double nd = -(kt * kt) / 3. * (1. - om * tau_ini / 5.);
      const double nth = -k * (kt * kt * kt) / 36. / (4. * Rn + 15.) *
                         (4. * Rn + 11. + 12. - 3. * (8. * Rn * Rn + 50. * Rn + 275.) / 20. / (2. * Rn + 15.) * tau_ini * om);
      const double ns = (kt * kt) / (45. + 12. * Rn) * 2. * (1. + (4. * Rn - 5.) / 4. / (2. * Rn + 15.) * tau_ini * om);
      m.y0[L.i_nu] = nd;
      m.y0[L.i_nu + 1] = nth;
      m.y0[L.i_nu + 2] = ns;
      if (c.has_ncdm) {
        for (int i = 0; i < 3; ++i) {
          double q = Q3[i];
          double fac = q / (1. + exp(-q));
          double* Pb = m.y0 + L.i_ncdm + i * L.nM;
          Pb[0] = nd / 4. * fac;
          Pb[1] = nth / 3. * fac;
          Pb[2] = ns / 2. * fac;
        }
      }
    }
    __syncwarp();

    double t0 = lna_start;
    double t1 = fmin(t0 + S.dt0, 0.0);
    double prev_inv = 1.0, prev_prev_inv = 1.0;
    int isave = 0, nsteps = 0, nacc = 0, nrej = 0, nnewton = 0, status = ABCMB_STATUS_OK;
    BG b;
    bg_eval(c, P.tables, t0, b);
    build_core(c, L, k, b, m, lane);
    apply_A(L, m, m.y0, m.F, lane);         // FSAL stage 1

    while (t0 < 0.0) {
      if (nsteps >= S.max_steps) { status = ABCMB_STATUS_MAX_STEPS; break; }
      ++nsteps;
      const double h = t1 - t0;
      const double hg = h * KV_G;
      bool ok = true;
      for (int i = 1; i < 7 && ok; ++i) {
        const double ti = t0 + KV_C[i] * h;
        if (i != 6) {                  // stages 6 and 7 share t0 + h
          bg_eval(c, P.tables, ti, b);
          build_core(c, L, k, b, m, lane);
        }
        if (i == 1) factor_newton(L, m, hg, lane);
        double* fi = m.F + i * n;
        for (int e = lane; e < n; e += WARP) {
          double acc = 0.;
          for (int j = 0; j < i; ++j) acc = fma(KV_A[i][j], m.F[j * n + e], acc);
          m.base[e] = m.y0[e] + h * acc;
          fi[e] = m.F[(i - 1) * n + e];
        }
        __syncwarp();
        double diffsize = INFINITY, diffsize_prev;
        bool conv = false;
        for (int it = 1; it <= root_max; ++it) {
          for (int e = lane; e < n; e += WARP) m.v[e] = m.base[e] + hg * fi[e];
          __syncwarp();
          apply_A(L, m, m.v, m.r, lane);
          for (int e = lane; e < n; e += WARP) m.r[e] = m.r[e] - fi[e];
          __syncwarp();
          solve_newton(L, m, m.r, lane);
          double ss = 0.;
          for (int e = lane; e < n; e += WARP) {
            double x = m.r[e];
            double fnew = fi[e] + x;
            fi[e] = fnew;
            double q = x / (atol + rtol * fabs(fnew));
            ss += q * q;
          }
          ss = warp_sum(ss);
          __syncwarp();
          diffsize_prev = diffsize;
          diffsize = sqrt(ss / n);
          ++nnewton;
          if (it >= 2) {
            double rate = diffsize / diffsize_prev;
            double factor = diffsize * rate / (1. - rate);
            bool small = diffsize < small_res;
            bool diverged = !isfinite(rate) || rate > 2.;
            bool converged = factor > 0. && factor < kappa;
            if (small || converged) { conv = true; break; }
            if (diverged) break;
          }
        }
        if (!conv) ok = false;
      }
      double scaled = INFINITY;
      if (ok) {
        double ss = 0.;
        for (int e = lane; e < n; e += WARP) {
          double acc = 0., acce = 0.;
#pragma unroll
          for (int j = 0; j < 6; ++j) {
            double fj = m.F[j * n + e];
            acc = fma(KV_A[6][j], fj, acc);
            acce = fma(KV_A[6][j] - KV_A[5][j], fj, acce);
          }
          acc = fma(KV_G, m.F[6 * n + e], acc);
          acce += -KV_G * m.F[5 * n + e] + KV_G * m.F[6 * n + e];
          double y0e = m.y0[e];
          double y1e = y0e + h * acc;
          m.y1[e] = y1e;
          double err = h * acce;
          double q = err / (atol + fmax(fabs(y0e), fabs(y1e)) * rtol);
          ss += q * q;
        }
        ss = warp_sum(ss);
        scaled = sqrt(ss / n);
        if (!isfinite(scaled)) scaled = INFINITY;
      }
      __syncwarp();
      const bool keep = scaled < 1.0;
      double inv = 1.0 / scaled;
      double f1v = (coeff1 == 0.) ? 1. : pow(inv, coeff1);
      double f2v = (coeff2 == 0.) ? 1. : pow(prev_inv, coeff2);
      double f3v = (coeff3 == 0.) ? 1. : pow(prev_prev_inv, coeff3);
      double factor = fmin(fmax(safety * f1v * f2v * f3v, keep ? 1.0 : factormin), factormax);
      double dt_new = h * factor;
      if (inv == 0. || isinf(inv)) inv = 1.;
      if (keep) {
        ++nacc;
        // cubic Hermite dense output on [t0, t1] at every save point it covers
        while (isave < nsave) {
          double ts = linspace_at(lts, 0.0, nsave, isave);
          if (!(ts <= t1)) break;
          double th = (ts - t0) / h;
          for (int e = lane; e < n; e += WARP) {
            double y0e = m.y0[e], y1e = m.y1[e];
            double k0 = h * m.F[e], k1 = h * m.F[6 * n + e];
            m.v[e] = y0e + th * (k0 + th * ((3. * (y1e - y0e) - 2. * k0 - k1) + th * (2. * (y0e - y1e) + k0 + k1)));
          }
          __syncwarp();
          write_fields(c, L, P.tables, k, ts, m.v, P.pt, nsave, isave, ik, lane);
          __syncwarp();
          ++isave;
        }
        prev_prev_inv = prev_inv;
        prev_inv = inv;
        for (int e = lane; e < n; e += WARP) {
          m.y0[e] = m.y1[e];
          m.F[e] = m.F[6 * n + e];
        }
        __syncwarp();
        t0 = t1;
      } else {
        ++nrej;
      }
      if (t0 >= 0.0) break;
      double tn = t0 + dt_new;
      if (tn > 0.0 - 1e-10) tn = keep ? 0.0 : t0 + 0.5 * (0.0 - t0);
      t1 = tn;
      if (!(h > 1e-14) || !isfinite(t1)) { status = ABCMB_STATUS_DT_UNDERFLOW; break; }
    }
    if (status == ABCMB_STATUS_OK && isave < nsave) status = ABCMB_STATUS_NONFINITE;
    if (lane == 0) {
      abcmb_kstat st;
      st.status = status;
      st.n_accepted = nacc;
      st.n_rejected = nrej;
      st.n_newton = nnewton;
      st.lna_start = lna_start;
      P.kstat[item] = st;
    }
    __syncwarp();
  }
}

}  // namespace abcmb

// ---------------------------------------------------------------------------
// host launcher (called from capi.cu)
// ---------------------------------------------------------------------------
namespace abcmb {

int64_t pert_workspace_bytes(int n_cosmo) {
  int64_t b = 256;                                        // queue counter
  b += ((int64_t)n_cosmo * 8 + 255) / 256 * 256;          // lna1
  b += 2 * (((int64_t)n_cosmo * NSTART * 8 + 255) / 256 * 256);  // aH and f1 grids
  return b;
}

size_t pert_smem_per_warp(int max_ny, int ncm) { return warp_mem_doubles(max_ny, ncm) * sizeof(double); }

cudaError_t launch_pert(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                        int n_items, const int32_t* items, const abcmb_pert_settings& s, double* pt,
                        abcmb_kstat* kstat, void* ws, cudaStream_t stream, int warps_per_block,
                        int* grid_out) {
  char* w = static_cast<char*>(ws);
  int* queue = reinterpret_cast<int*>(w);
  w += 256;
  double* lna1 = reinterpret_cast<double*>(w);
  w += ((int64_t)n_cosmo * 8 + 255) / 256 * 256;
  double* aHg = reinterpret_cast<double*>(w);
  w += ((int64_t)n_cosmo * NSTART * 8 + 255) / 256 * 256;
  double* f1g = reinterpret_cast<double*>(w);
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  dim3 g1((NSTART + 255) / 256, n_cosmo);
  start_grid_kernel<<<g1, 256, 0, stream>>>(n_cosmo, cosmo, tables, aHg, f1g);
  start_lna1_kernel<<<(n_cosmo + 127) / 128, 128, 0, stream>>>(n_cosmo, f1g, s.R_tc, lna1);
  PertArgs A;
  A.n_cosmo = n_cosmo;
  A.n_items = n_items;
  A.max_ny = s.max_ny;
  A.ncm = s.any_ncdm ? 28 : 16;
  A.cosmo = cosmo;
  A.tables = tables;
  A.kbuf = kbuf;
  A.items = items;
  A.pt = pt;
  A.kstat = kstat;
  A.aHg = aHg;
  A.lna1 = lna1;
  A.queue = queue;
  A.s = s;
  const int threads = 32 * warps_per_block;
  const size_t smem = (size_t)warps_per_block * pert_smem_per_warp(s.max_ny, A.ncm);
  e = cudaFuncSetAttribute(pert_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pert_kernel, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int grid = nsm * per_sm;
  int need = (n_items + warps_per_block - 1) / warps_per_block;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  if (grid_out) *grid_out = grid;
  pert_kernel<<<grid, threads, smem, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace abcmb
