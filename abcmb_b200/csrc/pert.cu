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
// densely: every hierarchy's l >= 3 tail is a tridiagonal chain that couples
// to the rest of the system only through its l = 2 element, so the tails are
// eliminated bottom-up (pivots >= 1: the free-streaming couplings have
// opposite signs and the damping is non-negative) and fold into one diagonal
// entry each of a dense "core" block holding eta, delta_c, delta_b, theta_b
// and l <= 2 of every hierarchy (13 unknowns, 22 with massive neutrinos).
// The core is inverted once per step by a warp-parallel Gauss-Jordan with
// partial pivoting; every chord iteration then costs two chain sweeps and a
// core mat-vec instead of a dense LU solve.
#include "common.cuh"

namespace abcmb {

constexpr int WARP = 32;
constexpr int NCHAIN = 6;            // F, G, N, Psi(q0), Psi(q1), Psi(q2)
constexpr int NSV = 18;              // saved background: 16 BG values, the save-index tag, 1/aH
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

// Scalar layout of one item's state vector (kept in registers; the per-chain
// arrays live in shared memory, see WarpMem::chs / chL).
struct Layout {
  int ny, nc, nchain, ntail;
  int i_g, i_G, i_nu, i_ncdm, nM;
  int lg, lp, lnu, lm;
};

__device__ __forceinline__ void make_layout(const abcmb_cosmo& c, Layout& L) {
  L.lg = c.lmax_g;
  L.lp = c.lmax_pol_g;
  L.lnu = c.lmax_nu;
  L.lm = c.lmax_ncdm;
  L.i_g = 4;
  L.i_G = L.i_g + c.lmax_g + 1;
  L.i_nu = L.i_G + c.lmax_pol_g + 1;
  L.i_ncdm = L.i_nu + c.lmax_nu + 1;
  L.nM = c.has_ncdm ? c.lmax_ncdm + 1 : 0;
  L.ny = L.i_ncdm + 3 * L.nM;
  L.nchain = c.has_ncdm ? 6 : 3;
  L.nc = 4 + 3 * L.nchain;
  L.ntail = (L.lg - 2) + (L.lp - 2) + (L.lnu - 2) + (c.has_ncdm ? 3 * (L.lm - 2) : 0);
}

// chain ch: state index of its l = 3 element (first tail element), its
// l_max, its offset in the tail enumeration
__device__ __forceinline__ void chain_info(const Layout& L, int ch, int& start, int& lmax, int& off) {
  if (ch == 0) { start = L.i_g + 3; lmax = L.lg; off = 0; }
  else if (ch == 1) { start = L.i_G + 3; lmax = L.lp; off = L.lg - 2; }
  else if (ch == 2) { start = L.i_nu + 3; lmax = L.lnu; off = (L.lg - 2) + (L.lp - 2); }
  else {
    const int b = ch - 3;
    start = L.i_ncdm + b * L.nM + 3;
    lmax = L.lm;
    off = (L.lg - 2) + (L.lp - 2) + (L.lnu - 2) + b * (L.lm - 2);
  }
}

// state index of core unknown ci: [eta, dc, db, thb], then l = 0..2 of the
// chains F, G, N, Psi(q0), Psi(q1), Psi(q2) in groups of three
__device__ __forceinline__ int core_state(const Layout& L, int ci) {
  if (ci < 4) return ci;
  const int g = (ci - 4) / 3, o = (ci - 4) % 3;
  if (g == 0) return L.i_g + o;
  if (g == 1) return L.i_G + o;
  if (g == 2) return L.i_nu + o;
  return L.i_ncdm + (g - 3) * L.nM + o;
}

// core index of chain ch's l = 2 row (the row its tail hangs off)
__device__ __forceinline__ int chain_core_l2(int ch) { return 4 + 3 * ch + 2; }

// tail slot t -> chain, l, state index, l_max
__device__ __forceinline__ void tail_elem(const Layout& L, int t, int& ch, int& l, int& e, int& lmax) {
  ch = 0;
  int start = 0, off = 0;
  for (int j = 0; j < L.nchain; ++j) {
    int s, lm, o;
    chain_info(L, j, s, lm, o);
    if (t >= o) { ch = j; start = s; lmax = lm; off = o; }
  }
  l = 3 + (t - off);
  e = start + (l - 3);
}

// Per-warp shared-memory arrays, addressed from one base pointer so that the
// kernel keeps two registers instead of one pointer per array.
struct WarpMem {
  double* p;      // base of this warp's region
  int my, ncm, cs;
  __device__ __forceinline__ double* y0() const { return p; }                 // ny
  __device__ __forceinline__ double* F() const { return p + my; }             // 7 ny stage derivatives
  __device__ __forceinline__ double* base() const { return p + 8 * my; }      // ny stage base
  __device__ __forceinline__ double* y1() const { return base(); }            // the step's result reuses base
  __device__ __forceinline__ double* v() const { return p + 9 * my; }         // ny
  __device__ __forceinline__ double* r() const { return p + 10 * my; }        // ny
  __device__ __forceinline__ double* invd() const { return p + 11 * my; }     // tail pivots
  __device__ __forceinline__ double* mult() const { return p + 12 * my; }     // upward-sweep multipliers
  __device__ __forceinline__ double* sub() const { return p + 13 * my; }      // tail sub-diagonal of M
  __device__ __forceinline__ double* Mc() const { return p + 14 * my; }       // ncm x cs core inverse
  __device__ __forceinline__ double* vc() const { return Mc() + ncm * cs; }   // gathered core vector
  __device__ __forceinline__ double* SB() const { return vc() + ncm; }        // NSLOT x NB basis
  __device__ __forceinline__ double* m3() const { return SB() + 6 * 32; }     // M_{2,3} / d_3 per chain
  __device__ __forceinline__ double* SV() const { return m3() + NCHAIN; }     // background at the next save time
  __device__ __forceinline__ int* cmap() const { return reinterpret_cast<int*>(SV() + NSV); }
  __device__ __forceinline__ int* perm() const { return cmap() + ncm; }      // pivot row of column k
  __device__ __forceinline__ int* iperm() const { return perm() + ncm; }     // column whose pivot row is j
  __device__ __forceinline__ int* rstate() const { return iperm() + ncm; }   // 5 ncm
  __device__ __forceinline__ int* chs() const { return rstate() + 5 * ncm; }  // 8
  __device__ __forceinline__ int* chL() const { return chs() + 8; }           // 8
  __device__ __forceinline__ int* tinfo() const { return chL() + 8; }         // max_ny
};

// Static sparsity of the core rows, shared by the block (filled once).
constexpr int MAXC = 22;
constexpr int LMAXT = 63;           // largest hierarchy l_max the kernel supports
// Byte-sized index tables: with ny = 100 the 3-blocks/SM instantiation needs
// 3 x (4 x 18 320 B of warp scratch + this table + 1 KB reserved) to fit in
// the SM's 228 KB, which leaves this table about 2.4 KB.
struct RowTab {
  int8_t n[MAXC];
  uint8_t bid[MAXC * 5];     // basis slot (< NB)
  uint8_t col[MAXC * 5];     // core column (< MAXC)
  int8_t tch[MAXC];          // chain hanging off the row, -1 for none
  double cst[MAXC * 5];
  double uh[MAXC], ue[MAXC], tco[MAXC];
  double ncdm_w[9];   // massive-neutrino bin weights of stage_basis and write_fields
  // tail coefficients of v[l-1] and v[l+1] per unit chain speed, by l:
  // l / (2l+1) and (l+1) / (2l+1); slot 1 holds the l = 3 pair of the F and
  // N hierarchies (6/7, 4/7: their l = 2 slot stores sigma = F_2 / 2)
  double ta[LMAXT + 1], tg[LMAXT + 1];
};

// Background "basis" of one time: every coefficient of A(lna) is a constant
// times one of these.  Slots: 0 = t0, 1..5 = t0 + c_i h for c = 0.52,
// 1.2303, 0.8958, 0.4364, 1 (stages 6 and 7 share slot 5).
constexpr int NB = 32;
constexpr int NSLOT = 6;
enum {
  B_ONE = 0, B_IAH, B_KIAH, B_K2IAH, B_KAP, B_RKAP, B_CS2K2IAH,
  B_NCDM = 7,        // 3 per bin: q/(eps aH), q k/(eps aH), q k^2/(eps aH)
  B_TRUNC = 16,      // 1/(aH tau)
  B_WH = 17,         // 8 weights of h': eta, dc, db, F0, N0, Psi0 x 3
  B_WE = 25,         // 6 weights of eta': thb, F1, N1, kPsi1 x 3
};
__device__ __forceinline__ int chain_speed_bid(int chn) { return chn < 3 ? B_KIAH : B_NCDM + 3 * (chn - 3) + 1; }

__host__ __device__ inline size_t warp_mem_doubles(int max_ny, int ncm) {
  const size_t ints = (size_t)ncm * 8 + (size_t)max_ny + 16;
  return (size_t)14 * max_ny + (size_t)ncm * (ncm + 1) + (size_t)ncm + NSLOT * NB + NCHAIN + NSV + (ints + 1) / 2;
}

__device__ __forceinline__ void carve(double* p, int max_ny, int ncm, WarpMem& m) {
  m.p = p;
  m.my = max_ny;
  m.ncm = ncm;
  m.cs = ncm + 1;
}

// 1/s for s > 0: an FP32 seed refined by two Newton steps (relative error
// ~1e-15); used for the tolerance scales of the norms, far cheaper than an
// FP64 division.  Values outside the FP32 range take the division.
__device__ __forceinline__ double pos_rcp(double s) {
  if (!(s > 1e-30 && s < 1e30)) return 1. / s;
  double r = (double)__frcp_rn((float)s);
  r = r * fma(-s, r, 2.);
  r = r * fma(-s, r, 2.);
  return r;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// Background basis at one time (one lane per time; abcmb/background.py and
// species.py evaluators through bg_eval).
// ---------------------------------------------------------------------------
// BG <-> shared memory (the background of a save point computed ahead)
__device__ __forceinline__ void bg_store(const BG& b, double* s) {
  s[0] = b.a; s[1] = b.aH; s[2] = b.tau; s[3] = b.itau_c; s[4] = b.cs2; s[5] = b.R;
  s[6] = b.rho_cdm; s[7] = b.rho_b; s[8] = b.rho_g; s[9] = b.rho_nu; s[10] = b.rho_ncdm; s[11] = b.P_ncdm;
  s[12] = b.ncdm_fac; s[13] = b.eps[0]; s[14] = b.eps[1]; s[15] = b.eps[2];
  s[17] = b.iaH;                        // s[16] is the save-index tag
}
__device__ __forceinline__ void bg_load(const double* s, BG& b) {
  b.a = s[0]; b.aH = s[1]; b.tau = s[2]; b.itau_c = s[3]; b.cs2 = s[4]; b.R = s[5];
  b.rho_cdm = s[6]; b.rho_b = s[7]; b.rho_g = s[8]; b.rho_nu = s[9]; b.rho_ncdm = s[10]; b.P_ncdm = s[11];
  b.ncdm_fac = s[12]; b.eps[0] = s[13]; b.eps[1] = s[14]; b.eps[2] = s[15];
  b.iaH = s[17];
}

// The basis values of one background state b into B[0..NB) (B may be a
// register array: every index is a compile-time constant).  ik2 = 1/k^2 of
// the item; ncdm_w the block table's massive-neutrino bin weights
// w_b (1 + e^-q_b) / q_b^2 and / q_b (constants, not recomputed here).
template <typename Arr>
__device__ __forceinline__ void basis_values(const BG& b, double k, double ik2, const double* __restrict__ ncdm_w,
                                             Arr& B) {
  const double iaH = b.iaH;
  const double kap = iaH * b.itau_c;                         // 1/(aH tau_c)
  B[B_ONE] = 1.;
  B[B_IAH] = iaH;
  B[B_KIAH] = k * iaH;
  B[B_K2IAH] = k * k * iaH;
  B[B_KAP] = kap;
  B[B_RKAP] = b.R * kap;
  B[B_CS2K2IAH] = b.cs2 * k * k * iaH;
#pragma unroll
  for (int bb = 0; bb < 3; ++bb) {
    double s = Q3[bb] * rsqrt(b.eps[bb] * b.eps[bb]) * iaH;  // q/(eps aH)
    B[B_NCDM + 3 * bb] = s;
    B[B_NCDM + 3 * bb + 1] = s * k;
    B[B_NCDM + 3 * bb + 2] = s * k * k;
  }
  B[B_TRUNC] = iaH / b.tau;
  // metric functionals (perturbations.py:238-239)
  const double Ca2 = (4. * PI * GN / (C_MPC * C_MPC)) * b.a * b.a;
  const double whf = 2. * iaH * iaH * Ca2;
  const double wef = Ca2 * iaH * ik2;
  B[B_WH + 0] = 2. * iaH * iaH * k * k;
  B[B_WH + 1] = whf * b.rho_cdm;
  B[B_WH + 2] = whf * b.rho_b;
  B[B_WH + 3] = whf * b.rho_g;
  B[B_WH + 4] = whf * b.rho_nu;
  B[B_WE + 0] = wef * b.rho_b;
  B[B_WE + 1] = wef * ((4. / 3.) * b.rho_g);
  B[B_WE + 2] = wef * ((4. / 3.) * b.rho_nu);
#pragma unroll
  for (int bb = 0; bb < 3; ++bb) {
    B[B_WH + 5 + bb] = whf * b.ncdm_fac * (ncdm_w[3 * bb] * b.eps[bb]);
    B[B_WE + 3 + bb] = wef * b.ncdm_fac * ncdm_w[3 * bb + 1];
  }
  B[31] = 0.;
}

// Background basis of one stage time; with sv != null the same lane instead
// stores the full background of a save time (lanes 0-4 stage times, lane 5
// the next save point: one instruction stream, no divergence).
__device__ __noinline__ void stage_basis(const abcmb_cosmo& c, const BGK& K, const double* __restrict__ tables,
                                         double k, double ik2, const double* __restrict__ ncdm_w, double lna, double* B,
                                         double* sv) {
  BG b;
  bg_eval(c, K, tables, lna, b);
  if (sv) {
    bg_store(b, sv);
    return;
  }
  basis_values(b, k, ik2, ncdm_w, B);
}

// Change of the basis along one parameter direction at lna: half the
// difference of the plus and minus descriptors' bases (the central
// difference of the background alone, at the base trajectory's time).
__device__ __noinline__ void stage_basis_diff(const abcmb_cosmo& cp, const abcmb_cosmo& cm,
                                              const double* __restrict__ tables, double k, double ik2,
                                              const double* __restrict__ ncdm_w, double lna, double* Bd) {
  BG b;
  double Bp[NB], Bm[NB];
  bg_eval(cp, bg_constants(cp), tables, lna, b);
  basis_values(b, k, ik2, ncdm_w, Bp);
  bg_eval(cm, bg_constants(cm), tables, lna, b);
  basis_values(b, k, ik2, ncdm_w, Bm);
#pragma unroll
  for (int j = 0; j < NB; ++j) Bd[j] = 0.5 * (Bp[j] - Bm[j]);
}

// Sparse description of one core row of A: up to five terms
// cst * basis[bid] * y[col] plus the metric terms uh * h' + ue * eta' and,
// for the l = 2 row of a hierarchy, the coupling tcoef * speed * y[l = 3].
struct RowDesc {
  int n;
  int col[5];      // core index
  int bid[5];
  double cst[5];
  double uh, ue;
  int tchain;      // chain whose tail hangs off this (l = 2) row, or -1
  double tcoef;    // coefficient of that tail's l = 3 element, per unit chain speed
};

// Core rows (core indices: 0 eta, 1 dc, 2 db, 3 thb, 4-6 F0-2, 7-9 G0-2,
// 10-12 N0-2, 13+3b..15+3b Psi0-2 of q-bin b).
__device__ __noinline__ void make_row(int r, RowDesc& d) {
  d.n = 0;
  d.uh = 0.;
  d.ue = 0.;
  d.tchain = -1;
  d.tcoef = 0.;
  auto add = [&](int col, int bid, double cst) {
    d.col[d.n] = col;
    d.bid[d.n] = bid;
    d.cst[d.n] = cst;
    ++d.n;
  };
  if (r < 4) {
    if (r == 0) d.ue = 1.;                                        // eta' (perturbations.py:239)
    if (r == 1) d.uh = -0.5;                                      // CDM (species.py:607)
    if (r == 2) { d.uh = -0.5; add(3, B_IAH, -1.); }              // Baryon (species.py:1282)
    if (r == 3) {                                                 // species.py:1283
      add(3, B_ONE, -1.); add(3, B_RKAP, -1.); add(2, B_CS2K2IAH, 1.); add(5, B_RKAP, 1.);
    }
    return;
  }
  const int g = (r - 4) / 3, o = (r - 4) % 3;
  if (g == 0) {                                                   // Photon F (species.py:1432-1434)
    if (o == 0) { d.uh = -2. / 3.; add(5, B_IAH, -4. / 3.); }
    if (o == 1) { add(4, B_K2IAH, 0.25); add(6, B_K2IAH, -1.); add(3, B_KAP, 1.); add(5, B_KAP, -1.); }
    if (o == 2) {
      d.uh = 2. / 15.; d.ue = 4. / 5.;
      add(5, B_IAH, 4. / 15.); add(6, B_KAP, -9. / 10.); add(7, B_KAP, 1. / 20.); add(9, B_KAP, 1. / 20.);
      d.tchain = 0; d.tcoef = -3. / 10.;
    }
  } else if (g == 1) {                                            // Photon G (species.py:1443-1445)
    if (o == 0) { add(8, B_KIAH, -1.); add(7, B_KAP, -0.5); add(6, B_KAP, 1.); add(9, B_KAP, 0.5); }
    if (o == 1) { add(7, B_KIAH, 1. / 3.); add(9, B_KIAH, -2. / 3.); add(8, B_KAP, -1.); }
    if (o == 2) {
      add(8, B_KIAH, 2. / 5.); add(9, B_KAP, -0.9); add(6, B_KAP, 0.2); add(7, B_KAP, 0.1);
      d.tchain = 1; d.tcoef = -3. / 5.;
    }
  } else if (g == 2) {                                            // MasslessNeutrino (species.py:742-744)
    if (o == 0) { d.uh = -2. / 3.; add(11, B_IAH, -4. / 3.); }
    if (o == 1) { add(10, B_K2IAH, 0.25); add(12, B_K2IAH, -1.); }
    if (o == 2) { d.uh = 2. / 15.; d.ue = 4. / 5.; add(11, B_IAH, 4. / 15.); d.tchain = 2; d.tcoef = -3. / 10.; }
  } else {                                                        // MassiveNeutrino (species.py:962-964)
    const int bb = g - 3, i0 = 13 + 3 * bb, bs = B_NCDM + 3 * bb;
    const double q = Q3[bb];
    const double dl = -q / (1. + exp(-q));
    if (o == 0) { d.uh = dl / 6.; add(i0 + 1, bs, -1.); }
    if (o == 1) { add(i0 + 0, bs + 2, 1. / 3.); add(i0 + 2, bs + 2, -2. / 3.); }
    if (o == 2) {
      d.uh = -dl / 15.; d.ue = -2. / 5. * dl; add(i0 + 1, bs, 2. / 5.);
      d.tchain = 3 + bb; d.tcoef = -3. / 5.;
    }
  }
}

// h' and eta' of the state v (perturbations.py:238-239) with basis B.
__device__ __forceinline__ void metric(const Layout& L, const double* B, const double* v, bool ncdm, double& hp,
                                       double& etap) {
  // sums split into independent partial sums: short dependency chains
  hp = fma(B[B_WH], v[0], B[B_WH + 1] * v[1]) + fma(B[B_WH + 2], v[2], fma(B[B_WH + 3], v[L.i_g], B[B_WH + 4] * v[L.i_nu]));
  etap = fma(B[B_WE], v[3], B[B_WE + 1] * v[L.i_g + 1]) + B[B_WE + 2] * v[L.i_nu + 1];
  if (ncdm) {
    const double* p0 = v + L.i_ncdm;
    const int nM = L.nM;
    hp += fma(B[B_WH + 5], p0[0], fma(B[B_WH + 6], p0[nM], B[B_WH + 7] * p0[2 * nM]));
    etap += fma(B[B_WE + 3], p0[1], fma(B[B_WE + 4], p0[nM + 1], B[B_WE + 5] * p0[2 * nM + 1]));
  }
}

// out = A(t) v for the time whose basis is B (get_derivatives, perturbations.py:201-248).
// One core row of A at one stage time, kept in registers for all chord
// iterations of that stage (unused terms have coefficient 0 and index 0).
struct CoreRow {
  double c[5];      // cst * basis[bid]
  int s[5];         // state index of each term
  double tc;        // coefficient of the hanging tail's l = 3 element
  int ts;           // its state index
  double uh, ue;
  int out;          // state index of the row
};

__device__ __forceinline__ void core_row_at(const Layout& L, const RowTab& R, const WarpMem& m, const double* B,
                                            int lane, CoreRow& cr) {
  const int r = lane < L.nc ? lane : 0;
  const int nt = R.n[r];
#pragma unroll
  for (int t = 0; t < 5; ++t) {
    cr.c[t] = t < nt ? R.cst[r * 5 + t] * B[R.bid[r * 5 + t]] : 0.;
    cr.s[t] = t < nt ? m.rstate()[r * 5 + t] : 0;
  }
  const int tc = R.tch[r];
  cr.tc = tc >= 0 ? R.tco[r] * B[chain_speed_bid(tc)] : 0.;
  cr.ts = tc >= 0 ? m.chs()[tc] : 0;
  cr.uh = R.uh[r];
  cr.ue = R.ue[r];
  cr.out = m.cmap()[r];
}

#ifndef PERT_APPLY_ATTR
#define PERT_APPLY_ATTR
#endif
// out = A v - fsub (fsub may be null): the RHS, or the chord residual directly.
// B (a basis slot), v, out and fsub are disjoint regions of the warp's
// scratch in every call (fsub may be null).
__device__ PERT_APPLY_ATTR void apply_A(const Layout& L, const WarpMem& m, const RowTab& R, const CoreRow& cr,
                                       const double* __restrict__ B, const double* __restrict__ v,
                                       double* __restrict__ out, const double* __restrict__ fsub,
                                       bool ncdm, int lane) {
  double hp, etap;
  metric(L, B, v, ncdm, hp, etap);
  if (lane < L.nc) {
    double acc = cr.uh * hp + cr.ue * etap;
#pragma unroll
    for (int t = 0; t < 5; ++t) acc = fma(cr.c[t], v[cr.s[t]], acc);
    acc = fma(cr.tc, v[cr.ts], acc);
    out[cr.out] = fsub ? acc - fsub[cr.out] : acc;
  }
  const double trunc = B[B_TRUNC];
  for (int t = lane; t < L.ntail; t += WARP) {
    const int info = m.tinfo()[t];
    const int e = info & 0xFFF, chn = (info >> 12) & 7;
    const double s = B[chain_speed_bid(chn)];
    const double d = chn < 2 ? B[B_KAP] : 0.;
    double fv;
    if ((info >> 15) & 1) fv = s * v[e - 1] - (d + (double)(m.chL()[chn] + 1) * trunc) * v[e];
    else {
      const int li = info >> 16;
      fv = s * (R.ta[li] * v[e - 1] - R.tg[li] * v[e + 1]) - d * v[e];
    }
    out[e] = fsub ? fv - fsub[e] : fv;
  }
  __syncwarp();
}

// Factor M = I - hg A(t_lin) (basis B): tails bottom-up, then the core inverse.
// The Gauss-Jordan sweep of factor_newton on the NC x NC core in shared
// memory, one row per lane.  NC is a compile-time size (13, or 22 with
// massive neutrinos) so the row loops unroll; the row a lane updates and the
// pivot row are disjoint, declared __restrict__, so all loads of a pivot step
// issue before its stores.
template <int NC>
__device__ __forceinline__ void gauss_jordan(WarpMem& m, int lane) {
  const unsigned FULL = 0xffffffffu;
  const int CS = m.cs;
  double* Mc = m.Mc();
  unsigned used = 0u;
  for (int p = 0; p < NC; ++p) {
    const bool elig = lane < NC && !((used >> lane) & 1u);
    const unsigned key = elig ? (unsigned)(__double_as_longlong(fabs(Mc[lane * CS + p])) >> 32) : 0u;
    const unsigned kmax = __reduce_max_sync(FULL, key);
    const unsigned hit = __ballot_sync(FULL, elig && key == kmax);
    const int q = __ffs(hit) - 1;
    used |= 1u << q;
    if (lane == 0) {
      m.perm()[p] = q;
      m.iperm()[q] = p;
    }
    const double pinv = __drcp_rn(Mc[q * CS + p]);          // == 1. / pivot, correctly rounded
    __syncwarp();
    if (lane < NC) Mc[q * CS + lane] = (lane == p ? 1. : Mc[q * CS + lane]) * pinv;
    __syncwarp();
    if (lane < NC && lane != q) {
      double* __restrict__ row = Mc + lane * CS;
      const double* __restrict__ prow = Mc + q * CS;
      const double f = row[p];
      double pr[NC], rw[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        pr[c] = prow[c];
        rw[c] = (c == p) ? 0. : row[c];
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) row[c] = fma(-f, pr[c], rw[c]);
    }
    __syncwarp();
  }
}

__device__ void factor_newton(const Layout& L, WarpMem& m, const RowTab& R, const double* B, double hg,
                              bool ncdm, int lane) {
  const int nc = L.nc;
  const int CS = m.cs;
  if (lane < nc) {
    double* row = m.Mc() + lane * CS;
    for (int j = 0; j < nc; ++j) row[j] = 0.;
    const int nt = R.n[lane];
#pragma unroll
    for (int t = 0; t < 5; ++t)
      if (t < nt) row[R.col[lane * 5 + t]] -= hg * R.cst[lane * 5 + t] * B[R.bid[lane * 5 + t]];
    const double ruh = R.uh[lane], rue = R.ue[lane];
    // metric columns (core indices): h' <- eta, dc, db, F0, N0, Psi0_b ; eta' <- thb, F1, N1, kPsi1_b
    if (ruh != 0.) {
      const double u = hg * ruh;
      row[0] -= u * B[B_WH]; row[1] -= u * B[B_WH + 1]; row[2] -= u * B[B_WH + 2];
      row[4] -= u * B[B_WH + 3]; row[10] -= u * B[B_WH + 4];
      if (ncdm) for (int bb = 0; bb < 3; ++bb) row[13 + 3 * bb] -= u * B[B_WH + 5 + bb];
    }
    if (rue != 0.) {
      const double u = hg * rue;
      row[3] -= u * B[B_WE]; row[5] -= u * B[B_WE + 1]; row[11] -= u * B[B_WE + 2];
      if (ncdm) for (int bb = 0; bb < 3; ++bb) row[14 + 3 * bb] -= u * B[B_WE + 3 + bb];
    }
    row[lane] += 1.;
  }
  __syncwarp();
  const double trunc = B[B_TRUNC];
  if (lane < L.nchain) {
    // tail l = 3..L_c eliminated bottom-up; pivots stay >= 1
    const int chn = lane;
    const double s = B[chain_speed_bid(chn)];
    const double d = chn < 2 ? B[B_KAP] : 0.;
    const int Lc = m.chL()[chn];
    const int e3 = m.chs()[chn];
    double inv_next = 0., sub_next = 0.;
    for (int l = Lc; l >= 3; --l) {
      int e = e3 + (l - 3);
      double diag, sup, sb;
      if (l == Lc) {
        diag = 1. + hg * (d + (double)(Lc + 1) * trunc);
        sup = 0.;
        sb = -hg * s;
      } else {
        diag = 1. + hg * d;
        const int li = (l == 3 && (chn == 0 || chn == 2)) ? 1 : l;
        sup = hg * s * R.tg[li];
        sb = -hg * s * R.ta[li];
      }
      double inv = pos_rcp(diag - sup * sub_next * inv_next);    // pivots are >= 1
      m.invd()[e] = inv;
      m.mult()[e] = sup * inv_next;
      m.sub()[e] = sb;
      inv_next = inv;
      sub_next = sb;
    }
    // fold the tail into the l = 2 diagonal entry of the core
    const int cc = chain_core_l2(chn);
    const double M23 = -hg * R.tco[cc] * s;
    m.Mc()[cc * CS + cc] -= M23 * sub_next * inv_next;
    m.m3()[chn] = M23 * inv_next;
  }
  __syncwarp();
  // In-place Gauss-Jordan inverse of the core with partial pivoting and no
  // row exchanges: the pivot of column p is the not-yet-used row q_p of
  // largest |M[.][p]| (compared on the high 32 bits of the IEEE pattern,
  // monotonic in magnitude; ties -> lowest row), recorded in perm[p] and left
  // in place.  Afterwards A^{-1}[i][j] = Mc[q_i][k] with q_k = j, which
  // solve_newton applies as x_i = sum_k Mc[q_i][k] b[q_k].
  if (nc == 13) gauss_jordan<13>(m, lane);
  else gauss_jordan<MAXC>(m, lane);
}

// sum_j a[j] b[j] over a compile-time length, in four independent partial sums
template <int N>
__device__ __forceinline__ double core_dot(const double* __restrict__ a, const double* __restrict__ b) {
  double s0 = 0., s1 = 0., s2 = 0., s3 = 0.;
#pragma unroll
  for (int j = 0; j + 3 < N; j += 4) {
    s0 = fma(a[j], b[j], s0);
    s1 = fma(a[j + 1], b[j + 1], s1);
    s2 = fma(a[j + 2], b[j + 2], s2);
    s3 = fma(a[j + 3], b[j + 3], s3);
  }
#pragma unroll
  for (int j = N & ~3; j < N; ++j) s0 = fma(a[j], b[j], s0);
  return (s0 + s1) + (s2 + s3);
}

// Solve M x = r in place (r holds the right-hand side on entry); vcb is the
// warp buffer of the gathered core vector (ncm doubles).
__device__ void solve_newton(const Layout& L, WarpMem& m, double* r, int lane, double* vcb) {
  const int nc = L.nc;
  // upward sweeps of the tails (l = L-1 .. 3); the l = 2 right-hand side
  // picks up the tail.  Two elements per trip so the loads run ahead.
  const double* mult = m.mult();
  if (lane < L.nchain) {
    const int chn = lane;
    const int e3 = m.chs()[chn];
    int e = e3 + (m.chL()[chn] - 3);
    double nxt = r[e];
    --e;
    for (; e - 1 >= e3; e -= 2) {
      const double ra = r[e], ma = mult[e], rb = r[e - 1], mb = mult[e - 1];
      const double va = ra - ma * nxt;
      const double vb = rb - mb * va;
      r[e] = va;
      r[e - 1] = vb;
      nxt = vb;
    }
    if (e >= e3) {
      nxt = r[e] - mult[e] * nxt;
      r[e] = nxt;
    }
    const int cc = chain_core_l2(chn);
    vcb[m.iperm()[cc]] = r[m.cmap()[cc]] - m.m3()[chn] * nxt;
  }
  // every other core row gathers its right-hand side directly
  // (vc is stored permuted: the entry for core row j goes to slot iperm[j])
  if (lane < nc && !(lane >= 4 && (lane - 4) % 3 == 2)) vcb[m.iperm()[lane]] = r[m.cmap()[lane]];
  __syncwarp();
  double xc = 0.;
  if (lane < nc) {
    // x_i = sum_k Mc[q_i][k] b[q_k] (pivot rows left in place, see
    // factor_newton); vc already holds b[q_k] in slot k
    const double* row = m.Mc() + m.perm()[lane] * m.cs;
    const double* vc = vcb;
    xc = nc == 13 ? core_dot<13>(row, vc) : core_dot<MAXC>(row, vc);
  }
  __syncwarp();
  if (lane < nc) r[m.cmap()[lane]] = xc;
  __syncwarp();
  if (lane < L.nchain) {
    const double* sub = m.sub();
    const double* invd = m.invd();
    const int chn = lane;
    const int e3 = m.chs()[chn];
    const int eL = e3 + (m.chL()[chn] - 3);
    double prev = r[e3 - 1];
    int e = e3;
    for (; e + 1 <= eL; e += 2) {
      const double ra = r[e], sa = sub[e], ia = invd[e], rb = r[e + 1], sb = sub[e + 1], ib = invd[e + 1];
      const double xa = (ra - sa * prev) * ia;
      const double xb = (rb - sb * xa) * ib;
      r[e] = xa;
      r[e + 1] = xb;
      prev = xb;
    }
    if (e <= eL) r[e] = (r[e] - sub[e] * prev) * invd[e];
  }
  __syncwarp();
}

// Fields of make_output_table at one save point from the interpolated state ys.
// Massive-neutrino perturbation sums of write_fields: 4/pi^2 / (hbar c)^3
constexpr double NCDM_K = 4. / (PI * PI) / (HBAR * HBAR * HBAR) / (C_CM * C_CM * C_CM);
constexpr double G4C = 4. * PI * GN / (C_MPC * C_MPC);

// PerturbationTable fields at one save point (make_output_table,
// perturbations.py:318-404, with each species' output_perturbations).  Lane f
// (< ABCMB_NFIELDS) writes field f.  Reciprocals are taken once (1/aH, 1/k^2,
// the massive-neutrino bin constants come from the block table) so the metric
// fields are products rather than chains of divisions; output-only, the
// integration never reads them.
__device__ __noinline__ void write_fields(const abcmb_cosmo& c, const Layout& L, const double* tables, double k, double lna,
                             const double* ys, double* pt, int n_save, int isave, int ik, int lane,
                             const double* sv, const double* ncdm_w) {
  BG b;
  if (sv) bg_load(sv, b);               // computed ahead for this save point
  else bg_eval(c, bg_constants(c), tables, lna, b);
  const double a = b.a, aH = b.aH;
  const double iaH = b.iaH;
  const double ik2 = 1. / (k * k);
  double srd = b.rho_cdm * ys[1] + b.rho_b * ys[2] + b.rho_g * ys[L.i_g] + b.rho_nu * ys[L.i_nu];
  const double pg = (4. / 3.) * b.rho_g, pn = (4. / 3.) * b.rho_nu;   // rho + P of photons, massless nu
  double srt = b.rho_b * ys[3] + pg * ys[L.i_g + 1] + pn * ys[L.i_nu + 1];
  double srs = pg * ys[L.i_g + 2] + pn * ys[L.i_nu + 2];
  double rdm = b.rho_cdm * ys[1] + b.rho_b * ys[2];
  double rm = b.rho_cdm + b.rho_b;
  double nd = 0., nt = 0., ns = 0.;
  if (c.has_ncdm) {
    // ncdm_w[3 i + {0,1,2}] = w_i (1 + e^-q_i) / q_i^2, / q_i, * 1
    double r0 = 0., r1 = 0., r2 = 0.;
    for (int i = 0; i < 3; ++i) {
      const double* P = ys + L.i_ncdm + i * L.nM;
      r0 += ncdm_w[3 * i] * b.eps[i] * P[0];
      r1 += ncdm_w[3 * i + 1] * P[1];
      r2 += ncdm_w[3 * i + 2] / b.eps[i] * P[2];
    }
    const double T = c.T_nu_massive * c.TCMB0 / a;
    const double f = c.N_nu_massive * NCDM_K * (T * T) * (T * T);
    const double rd = f * r0, rt = f * r1, rs = (2. / 3.) * f * r2;
    srd += rd; srt += rt; srs += rs;
    rdm += rd; rm += b.rho_ncdm;
    const double irhoP = 1. / (b.rho_ncdm + b.P_ncdm);
    nd = rd / b.rho_ncdm; nt = rt * irhoP; ns = rs * irhoP;
  }
  if (lane < ABCMB_NFIELDS) {
    const double eta = ys[0];
    const double a2 = a * a;
    const double hp = 2. * (iaH * iaH) * (k * k * eta + G4C * a2 * srd);
    const double etap = G4C * a2 * iaH * srt * ik2;
    const double alpha = aH * (hp + 6. * etap) * 0.5 * ik2;
    double val = 0.;
    switch (lane) {
      case ABCMB_F_DELTA_M: val = rdm / rm; break;
      case ABCMB_F_THETA_B_PRIME:
        val = -ys[3] + b.cs2 * iaH * (k * k * ys[2]) + b.R * iaH * b.itau_c * (ys[L.i_g + 1] - ys[3]);
        break;
      case ABCMB_F_ETA: val = eta; break;
      case ABCMB_F_H_PRIME: val = hp; break;
      case ABCMB_F_ETA_PRIME: val = etap; break;
      case ABCMB_F_ALPHA: val = alpha; break;
      case ABCMB_F_ALPHA_PRIME:
        val = eta * iaH - 2. * alpha - 3. * G4C * a2 * iaH * srs * ik2;
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

// Adiabatic initial conditions (perturbations.py:161-199 + species y_ini)
// of descriptor c at lna: the nonzero entries of y, written by one lane
// (y zeroed beforehand).
__device__ __noinline__ void write_ic(const abcmb_cosmo& c, const Layout& L, const double* __restrict__ tables,
                                      double k, double lna, double* y) {
  const double tau_ini = tau_of(c, tables, lna);
  const double om = c.om, Rn = c.R_nu, Rb = c.R_b;
  const double kt = k * tau_ini;
  y[0] = (1. - k * k * tau_ini * tau_ini / 12. / (15. + 4. * Rn) *
                   (5. + 4. * Rn - (16. * Rn * Rn + 280. * Rn + 325) / 10. / (2. * Rn + 15.) * tau_ini * om));
  y[1] = -(kt * kt) / 4. * (1. - om * tau_ini / 5.);
  y[2] = -(kt * kt) / 4. * (1. - om * tau_ini / 5.);
  const double thb = -k * k * k * k * tau_ini * tau_ini * tau_ini / 36. *
                     (1. - 3. * (1. + 5. * Rb - Rn) / 20. / (1. - Rn) * om * tau_ini);
  y[3] = thb;
  y[L.i_g] = -(kt * kt) / 3. * (1. - om * tau_ini / 5.);
  y[L.i_g + 1] = thb;
  const double nd = -(kt * kt) / 3. * (1. - om * tau_ini / 5.);
  const double nth = -k * (kt * kt * kt) / 36. / (4. * Rn + 15.) *
                     (4. * Rn + 11. + 12. - 3. * (8. * Rn * Rn + 50. * Rn + 275.) / 20. / (2. * Rn + 15.) * tau_ini * om);
  const double ns = (kt * kt) / (45. + 12. * Rn) * 2. * (1. + (4. * Rn - 5.) / 4. / (2. * Rn + 15.) * tau_ini * om);
  y[L.i_nu] = nd;
  y[L.i_nu + 1] = nth;
  y[L.i_nu + 2] = ns;
  if (c.has_ncdm) {
    for (int i = 0; i < 3; ++i) {
      double q = Q3[i];
      double fac = q / (1. + exp(-q));
      double* Pb = y + L.i_ncdm + i * L.nM;
      Pb[0] = nd / 4. * fac;
      Pb[1] = nth / 3. * fac;
      Pb[2] = ns / 2. * fac;
    }
  }
}

// ---------------------------------------------------------------------------
// Forward-mode sensitivities (abcmb_pert_forward_tangent)
// ---------------------------------------------------------------------------
// The tangent u_q of the discrete Kvaerno5 step along parameter direction q
// is integrated by the warp that integrates the base item, one direction
// after another once a step is accepted.  Each implicit stage i's tangent
// derivative solves (I - h gamma A_i) dF_i = A_i z + dA_i Y_i with
// z = u0 + h sum_{j<i} a_ij dF_j and Y_i the converged primal stage value,
// by chord iterations with the step's own factorisation (the primal's
// iteration matrix); dA_i is A with the basis replaced by its change along
// q (A is linear in the basis): half the difference of the plus and minus
// descriptors' bases at t_i.  Only u0 and the stage-1 derivative (the last
// stage's of the previous step, first-same-as-last like the primal's: a
// re-evaluation A(t0) u0 + dA(t0) y0 would multiply the stiff components'
// tolerance-level residue by |A|) persist per direction; the other stage
// derivatives and the work vectors are reused by the next direction, which
// keeps the shared memory per warp (and so the resident warps per SM) close
// to the forward kernel's.
//
// The tangent iteration is linear with the primal's iteration matrix
// I - M_lin^-1 M_i: its spectral radius is small whenever the primal stage
// converged, but it is far from normal in the tight-coupling era, so an
// error with a stiff component (the initial tangent's start-time term puts
// one there) can grow ~25x over the first iteration before it contracts.  A
// growing step therefore does not stop the tangent iterations (only a
// non-finite one does); they get TANGENT_ROOT_MAX iterations and the last
// iterate is kept (the tangents never change the primal's step sequence).
constexpr int ND_MAX = ABCMB_MAX_TANGENTS;
constexpr int TANGENT_ROOT_MAX = 16;

// Per-warp tangent scratch, after the primal's WarpMem: per direction u0
// and the stage-1 derivative f0; shared by the directions: the seven stage
// derivatives dF, q (the constant part of a stage's residual; u1 once the
// stages are done), r (residual and solve vector; a variant's state at a
// save point), yd (dy/dt of the dense output), yv (a variant's state), the
// basis changes at the five stage times, the variants' backgrounds at a save
// point, the solve's gathered core vector and the variants' descriptor
// indices.
struct TanMem {
  double* p;
  int my, nd, ncm;
  __device__ __forceinline__ double* u0(int q) const { return p + q * my; }
  __device__ __forceinline__ double* f0(int q) const { return p + nd * my + q * my; }
  __device__ __forceinline__ double* dF() const { return p + 2 * nd * my; }
  __device__ __forceinline__ double* qv() const { return dF() + 7 * my; }
  __device__ __forceinline__ double* rv() const { return qv() + my; }
  __device__ __forceinline__ double* yd() const { return rv() + my; }
  __device__ __forceinline__ double* yv() const { return yd() + my; }
  __device__ __forceinline__ double* bd(int slot) const { return yv() + my + (slot - 1) * NB; }
  __device__ __forceinline__ double* sv(int j) const { return yv() + my + 5 * NB + j * NSV; }
  __device__ __forceinline__ double* vc() const { return sv(2); }
  __device__ __forceinline__ int* vix() const { return reinterpret_cast<int*>(vc() + ncm); }   // 2 ND_MAX ints
  // the item's tangent chord iterations and unconverged stage solves
  __device__ __forceinline__ int* cnt() const { return vix() + 2 * ND_MAX; }
};

__host__ __device__ inline size_t tan_mem_doubles(int max_ny, int ncm, int nd) {
  if (nd <= 0) return 0;
  return (size_t)nd * 2 * (size_t)max_ny + 11 * (size_t)max_ny + 5 * NB + 2 * NSV + (size_t)ncm + ND_MAX + 1;
}

// out = A(B) z + A(Bd) Y for one direction: the part of a stage's tangent
// residual the chord iterations keep (Bd the basis change).
__device__ __forceinline__ void tan_const(const Layout& L, const WarpMem& m, const RowTab& R, const CoreRow& cr,
                                          const double* __restrict__ B, const double* __restrict__ Bd,
                                          const double* __restrict__ z, const double* __restrict__ Y,
                                          double* __restrict__ out, bool ncdm, int lane) {
  double hp, ep, hpd, epd;
  metric(L, B, z, ncdm, hp, ep);
  metric(L, Bd, Y, ncdm, hpd, epd);
  if (lane < L.nc) {
    const int r = lane;
    const int nt = R.n[r];
    const int tch = R.tch[r];
    double acc = cr.uh * hp + cr.ue * ep;
    double accd = cr.uh * hpd + cr.ue * epd;
#pragma unroll
    for (int u = 0; u < 5; ++u) {
      acc = fma(cr.c[u], z[cr.s[u]], acc);
      const double cd = u < nt ? R.cst[r * 5 + u] * Bd[R.bid[r * 5 + u]] : 0.;
      accd = fma(cd, Y[cr.s[u]], accd);
    }
    acc = fma(cr.tc, z[cr.ts], acc);
    const double tcd = tch >= 0 ? R.tco[r] * Bd[chain_speed_bid(tch)] : 0.;
    accd = fma(tcd, Y[cr.ts], accd);
    out[cr.out] = acc + accd;
  }
  const double trunc = B[B_TRUNC], trd = Bd[B_TRUNC];
  for (int u = lane; u < L.ntail; u += WARP) {
    const int info = m.tinfo()[u];
    const int e = info & 0xFFF, chn = (info >> 12) & 7;
    const int sb = chain_speed_bid(chn);
    const double sp = B[sb], sd = Bd[sb];
    const double d = chn < 2 ? B[B_KAP] : 0., dd = chn < 2 ? Bd[B_KAP] : 0.;
    double fv, fvd;
    if ((info >> 15) & 1) {
      const double lc1 = (double)(m.chL()[chn] + 1);
      fv = sp * z[e - 1] - (d + lc1 * trunc) * z[e];
      fvd = sd * Y[e - 1] - (dd + lc1 * trd) * Y[e];
    } else {
      const int li = info >> 16;
      const double ta = R.ta[li], tg = R.tg[li];
      fv = sp * (ta * z[e - 1] - tg * z[e + 1]) - d * z[e];
      fvd = sd * (ta * Y[e - 1] - tg * Y[e + 1]) - dd * Y[e];
    }
    out[e] = fv + fvd;
  }
  __syncwarp();
}

// r = h gamma A(B) F + q - F: the residual of a stage's tangent derivative F.
__device__ __forceinline__ void tan_resid(const Layout& L, const WarpMem& m, const RowTab& R, const CoreRow& cr,
                                          const double* __restrict__ B, const double* __restrict__ F,
                                          const double* __restrict__ q, double* __restrict__ r, double hg,
                                          bool ncdm, int lane) {
  double hp, ep;
  metric(L, B, F, ncdm, hp, ep);
  if (lane < L.nc) {
    double acc = cr.uh * hp + cr.ue * ep;
#pragma unroll
    for (int u = 0; u < 5; ++u) acc = fma(cr.c[u], F[cr.s[u]], acc);
    acc = fma(cr.tc, F[cr.ts], acc);
    const int o = cr.out;
    r[o] = fma(hg, acc, q[o]) - F[o];
  }
  const double trunc = B[B_TRUNC];
  for (int u = lane; u < L.ntail; u += WARP) {
    const int info = m.tinfo()[u];
    const int e = info & 0xFFF, chn = (info >> 12) & 7;
    const double sp = B[chain_speed_bid(chn)];
    const double d = chn < 2 ? B[B_KAP] : 0.;
    double fv;
    if ((info >> 15) & 1) fv = sp * F[e - 1] - (d + (double)(m.chL()[chn] + 1) * trunc) * F[e];
    else {
      const int li = info >> 16;
      fv = sp * (R.ta[li] * F[e - 1] - R.tg[li] * F[e + 1]) - d * F[e];
    }
    r[e] = fma(hg, fv, q[e]) - F[e];
  }
  __syncwarp();
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
  // forward-mode sensitivities (nd = 0: none)
  int nd;
  double tscale;           // tangent size relative to the state's (atol of the tangent solves x tscale)
  const int32_t* dirs;     // [n_cosmo][ND_MAX][2] (plus, minus) descriptors
  int32_t* tstat;          // [n_items][2] or null
  // internal numerical differentiation: the base items' accepted steps (end
  // time, chord iterations of the six implicit stages, 4 bits each),
  // recorded by one launch and replayed by the variants' launch
  double* rec_t1;          // [n_base][rec_cap]
  int32_t* rec_it;         // [n_base][rec_cap]
  int32_t* rec_n;          // [n_base] accepted steps, -1 if the base item failed
  int rec_cap;
  int n_base;              // replay: the record launch's items
  const int32_t* base_items;
  const int32_t* var_base; // replay: [n_items] index of each variant item's base item
};

__device__ __forceinline__ TanMem tan_mem(const WarpMem& m, const PertArgs& P) {
  TanMem t;
  t.p = m.p + warp_mem_doubles(P.max_ny, P.ncm);
  t.my = P.max_ny;
  t.nd = P.nd;
  t.ncm = P.ncm;
  return t;
}

// Optional per-phase cycle accounting, compiled in only with
// -DABCMB_PHASE_CLOCKS (python -m abcmb_b200.build --phase-clocks): every
// warp adds the clock64() cycles it spends in each phase of its steps to its
// own slot of g_pert_phase with reductions whose result nobody waits for;
// abcmb_pert_phase_clocks sums the slots.  Phases: 0 stage-time background,
// 1 Newton-matrix factorisation, 2 stage set-up, 3 residual (apply_A),
// 4 structured solve, 5 chord update and convergence test, 6 error estimate
// and step-size control, 7 the rest (dense output and PerturbationTable
// writes, item start and end, queue); the tangent kernel adds 8 the basis
// changes, 9 the stages' constant parts (primal stage values, z, A z +
// dA Y), 10 the tangent chord iterations, 11 the variants' tables.
#ifdef ABCMB_PHASE_CLOCKS
constexpr int PHASE_N = 12;
constexpr int PHASE_SLOTS = 8192;
__device__ unsigned long long g_pert_phase[PHASE_SLOTS * PHASE_N];
#define PERT_PHASE(k)                                                                      \
  do {                                                                                    \
    const long long ph_now = clock64();                                                   \
    if (lane == 0 && ph_slot) atomicAdd(ph_slot + (k), (unsigned long long)(ph_now - ph_t)); \
    ph_t = ph_now;                                                                        \
  } while (0)
#else
#define PERT_PHASE(k) \
  do {                \
  } while (0)
#endif
#ifdef ABCMB_PHASE_CLOCKS
#define PERT_PHASE_BEGIN()                                                                                    \
  const int ph_index = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);                                 \
  unsigned long long* ph_slot = ph_index < PHASE_SLOTS ? g_pert_phase + (size_t)ph_index * PHASE_N : nullptr; \
  long long ph_t = clock64()
#define PERT_PHASE_RESET() ph_t = clock64()
#else
#define PERT_PHASE_BEGIN() \
  do {                     \
  } while (0)
#define PERT_PHASE_RESET() \
  do {                     \
  } while (0)
#endif

// Direction q of one accepted step [t0, t0 + h] (the primal's stage
// derivatives F, y0, y1, factorisation and basis slots are the step's):
// the basis changes at the five stage times (lanes 0-4), the stage-1
// derivative, stages 1..6 by chord iterations, u1, then the variants'
// PerturbationTables at every save point of the step, each at its own save
// time: the fields of y(ts) +- (u_q(ts) + y'(ts) (ts_plus - ts_minus) / 2)
// with the variant's own background; finally u0 <- u1.  isave0 is the first
// save index the step covers (the primal writes its own fields afterwards).
// atol_t is the primal's atol scaled by the tangents' relative size.
__device__ __noinline__ void tangent_pass(const Layout& L, WarpMem& m, const RowTab& R, const PertArgs& P, int q,
                                          double k, double ik2, double t0, double h, double rtol, double atol_t,
                                          double inv_n, double lts, int isave0, int ik, int lane) {
  const TanMem t = tan_mem(m, P);
  PERT_PHASE_BEGIN();
  int titer = 0, tunconv = 0;
  const int n = L.ny;
  const bool ncdm = L.nM > 0;
  const double hg = h * KV_G;
  const double kappa = 1e-2, small_res = 1e-13;
  const abcmb_cosmo& cp = P.cosmo[t.vix()[2 * q]];
  const abcmb_cosmo& cm = P.cosmo[t.vix()[2 * q + 1]];
  double* __restrict__ dF = t.dF();
  if (lane < 5) stage_basis_diff(cp, cm, P.tables, k, ik2, R.ncdm_w, t0 + KV_C[lane + 1] * h, t.bd(lane + 1));
  CoreRow cr;
  for (int e = lane; e < n; e += WARP) dF[e] = t.f0(q)[e];     // the stage-1 derivative (FSAL)
  __syncwarp();
  PERT_PHASE(8);
  for (int i = 1; i < 7; ++i) {
    const int slot = (i == 6) ? 5 : i;
    const double* B = m.SB() + slot * NB;
    core_row_at(L, R, m, B, lane, cr);
    {
      // the converged primal stage value Y_i (into v), formed as the primal
      // formed it; z (into r); the predictor dF_i = dF_{i-1}
      const double* __restrict__ Fr = m.F();
      const double* __restrict__ y0 = m.y0();
      const double* __restrict__ u0 = t.u0(q);
      double* __restrict__ vw = m.v();
      double* __restrict__ z = t.rv();
      for (int e = lane; e < n; e += WARP) {
        double acc = 0., acc2 = 0., tc = 0., tc2 = 0.;
        int j = 0;
        for (; j + 1 < i; j += 2) {
          acc = fma(KV_A[i][j], Fr[j * n + e], acc);
          acc2 = fma(KV_A[i][j + 1], Fr[(j + 1) * n + e], acc2);
          tc = fma(KV_A[i][j], dF[j * n + e], tc);
          tc2 = fma(KV_A[i][j + 1], dF[(j + 1) * n + e], tc2);
        }
        if (j < i) {
          acc = fma(KV_A[i][j], Fr[j * n + e], acc);
          tc = fma(KV_A[i][j], dF[j * n + e], tc);
        }
        const double be = y0[e] + h * (acc + acc2);
        vw[e] = be + hg * Fr[i * n + e];
        z[e] = u0[e] + h * (tc + tc2);
        dF[i * n + e] = dF[(i - 1) * n + e];
      }
    }
    __syncwarp();
    tan_const(L, m, R, cr, B, t.bd(slot), t.rv(), m.v(), t.qv(), ncdm, lane);
    PERT_PHASE(9);
    double* __restrict__ fi = dF + i * n;
    double dsz = INFINITY;
    bool conv = false;
    for (int it = 1; it <= TANGENT_ROOT_MAX; ++it) {
      tan_resid(L, m, R, cr, B, fi, t.qv(), t.rv(), hg, ncdm, lane);
      solve_newton(L, m, t.rv(), lane, t.vc());
      double ss = 0.;
      {
        const double* __restrict__ rr = t.rv();
        for (int e = lane; e < n; e += WARP) {
          const double x = rr[e];
          const double fnew = fi[e] + x;
          fi[e] = fnew;
          const double qq = x * pos_rcp(atol_t + rtol * fabs(fnew));
          ss += qq * qq;
        }
      }
      ss = warp_sum(ss);
      __syncwarp();
      const double dp = dsz;
      const double d = sqrt(ss * inv_n);
      dsz = d;
      ++titer;
      if (it >= 2) {
        // the primal's very-chord termination test (division-free form); no
        // divergence stop but a non-finite size
        const bool small = d < small_res;
        const bool converged = d > 0. && d < dp && d * d < kappa * (dp - d);
        if (small || converged) {
          conv = true;
          break;
        }
        if (!isfinite(d)) break;
      }
    }
    if (!conv) ++tunconv;
    PERT_PHASE(10);
  }
  {
    // u1 = u0 + h (sum_j a_7j dF_j + gamma dF_7) into q
    const double* __restrict__ u0 = t.u0(q);
    double* __restrict__ u1 = t.qv();
    for (int e = lane; e < n; e += WARP) {
      double acc = 0., accb = 0.;
#pragma unroll
      for (int j = 0; j < 6; j += 2) {
        acc = fma(KV_A[6][j], dF[j * n + e], acc);
        accb = fma(KV_A[6][j + 1], dF[(j + 1) * n + e], accb);
      }
      acc = fma(KV_G, dF[6 * n + e], acc + accb);
      u1[e] = u0[e] + h * acc;
    }
  }
  __syncwarp();
  // the variants' tables at the save points of this step
  const int nsave = P.s.n_save;
  const double t1 = t0 + h;
  for (int is = isave0; is < nsave; ++is) {
    const double ts = linspace_at(lts, 0.0, nsave, is);
    if (!(ts <= t1)) break;
    const double th = (ts - t0) / h;
    const double tsp = linspace_at(cp.lna_transfer_start, 0.0, nsave, is);
    const double tsm = linspace_at(cm.lna_transfer_start, 0.0, nsave, is);
    const double dts = 0.5 * (tsp - tsm);
    if (lane < 2) {
      const abcmb_cosmo& cv = lane ? cm : cp;
      BG b;
      bg_eval(cv, bg_constants(cv), P.tables, lane ? tsm : tsp, b);
      bg_store(b, t.sv(lane));
    }
    {
      const double* __restrict__ y0 = m.y0();
      const double* __restrict__ y1 = m.y1();
      const double* __restrict__ Fr = m.F();
      const double* __restrict__ u0 = t.u0(q);
      const double* __restrict__ u1 = t.qv();
      double* __restrict__ yp = t.yv();
      double* __restrict__ ym = t.rv();
      for (int e = lane; e < n; e += WARP) {
        const double y0e = y0[e], y1e = y1[e];
        const double k0 = h * Fr[e], k1 = h * Fr[6 * n + e];
        const double a2 = 3. * (y1e - y0e) - 2. * k0 - k1, a3 = 2. * (y0e - y1e) + k0 + k1;
        const double ys = y0e + th * (k0 + th * (a2 + th * a3));
        const double yd = (k0 + th * (2. * a2 + 3. * th * a3)) / h;
        const double u0e = u0[e], u1e = u1[e];
        const double g0 = h * dF[e], g1 = h * dF[6 * n + e];
        const double us = u0e + th * (g0 + th * ((3. * (u1e - u0e) - 2. * g0 - g1) + th * (2. * (u0e - u1e) + g0 + g1)));
        const double ut = us + yd * dts;
        yp[e] = ys + ut;
        ym[e] = ys - ut;
      }
    }
    __syncwarp();
    write_fields(cp, L, P.tables, k, tsp, t.yv(), P.pt, nsave, is, ik, lane, t.sv(0), R.ncdm_w);
    write_fields(cm, L, P.tables, k, tsm, t.rv(), P.pt, nsave, is, ik, lane, t.sv(1), R.ncdm_w);
    __syncwarp();
  }
  {
    const double* __restrict__ u1 = t.qv();
    double* __restrict__ u0 = t.u0(q);
    for (int e = lane; e < n; e += WARP) u0[e] = u1[e];
    double* __restrict__ f0 = t.f0(q);
    for (int e = lane; e < n; e += WARP) f0[e] = dF[6 * n + e];   // first same as last
    if (lane == 0) {
      t.cnt()[0] += titer;
      t.cnt()[1] += tunconv;
    }
  }
  __syncwarp();
  PERT_PHASE(11);
}

// The tangents at an item's start: u = dy0/deps - f(t0, y0) dt0/deps from
// the variants' initial conditions at their own start times (plus into q,
// minus into r), the stage-1 derivative A(t0) u + dA(t0) y0 (the basis
// change at t0 into bd(1)), the counters cleared.
__device__ __noinline__ void tangent_init(const Layout& L, const WarpMem& m, const RowTab& R, const PertArgs& P,
                                          int ci, double k, double ik2, double lna_start, int lane) {
  const TanMem tm = tan_mem(m, P);
  const int n = L.ny, nd = tm.nd;
  if (lane < 2 * nd) tm.vix()[lane] = P.dirs[(ci * ND_MAX + (lane >> 1)) * 2 + (lane & 1)];
  if (lane < 2) tm.cnt()[lane] = 0;
  __syncwarp();
  for (int q = 0; q < nd; ++q) {
    for (int e = lane; e < n; e += WARP) tm.qv()[e] = tm.rv()[e] = 0.;
    __syncwarp();
    if (lane < 2) {
      const int v = tm.vix()[2 * q + lane];
      const double l2 = np_interp_lna(P.s.R_large, nullptr, P.aHg + (int64_t)v * NSTART, k);
      const double tv = fmin(fmin(P.lna1[v], l2), -10.);
      write_ic(P.cosmo[v], L, P.tables, k, tv, lane ? tm.rv() : tm.qv());
      tm.sv(0)[lane] = tv;
    }
    if (lane == 2)
      stage_basis_diff(P.cosmo[tm.vix()[2 * q]], P.cosmo[tm.vix()[2 * q + 1]], P.tables, k, ik2, R.ncdm_w,
                       lna_start, tm.bd(1));
    __syncwarp();
    const double dt0 = 0.5 * (tm.sv(0)[0] - tm.sv(0)[1]);
    for (int e = lane; e < n; e += WARP) tm.u0(q)[e] = 0.5 * (tm.qv()[e] - tm.rv()[e]) - m.F()[e] * dt0;
    __syncwarp();
    CoreRow cr;
    core_row_at(L, R, const_cast<WarpMem&>(m), m.SB(), lane, cr);
    tan_const(L, m, R, cr, m.SB(), tm.bd(1), tm.u0(q), m.y0(), tm.f0(q), L.nM > 0, lane);
  }
}

// Two instantiations of the same kernel, differing only in the register cap:
// 2 blocks of 4 warps per SM (250 registers, no spills: the shortest time per
// item) and 3 blocks per SM (168 registers, 12 warps: the shared-memory limit
// at ny = 100, the most items per second once the queue is long).
constexpr int PERT_BLOCKS_LATENCY = 2;
constexpr int PERT_BLOCKS_THROUGHPUT = 3;
constexpr int PERT_THREADS_MAX = 128;
// queue length per warp (at 2 blocks/SM) from which the throughput variant wins
constexpr int PERT_THROUGHPUT_ITEMS_PER_WARP = 16;



// IND: 0 = the adaptive integration; 1 = the same, recording every accepted
// step (end time and the chord-iteration count of each implicit stage) of
// the item into the record buffers; 2 = replay: the item (a variant of a base
// cosmology) takes its base item's recorded step ends and per-stage chord
// iteration counts instead of the step-size controller and the termination
// test, so every variant follows one fixed discrete map and the central
// difference of two variants is a smooth function of the parameter step
// (internal numerical differentiation, Bock 1981: no step-sequence noise).
template <bool TAN, int IND = 0>
__device__ __forceinline__ void pert_body(const PertArgs& P) {
  extern __shared__ double smem[];
  __shared__ RowTab R;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  if (threadIdx.x < MAXC) {
    RowDesc d;
    make_row(threadIdx.x, d);
    const int r = threadIdx.x;
    R.n[r] = d.n;
    R.tch[r] = d.tchain;
    R.tco[r] = d.tcoef;
    R.uh[r] = d.uh;
    R.ue[r] = d.ue;
    for (int t = 0; t < 5; ++t) {
      R.bid[r * 5 + t] = t < d.n ? d.bid[t] : 0;
      R.col[r * 5 + t] = t < d.n ? d.col[t] : 0;
      R.cst[r * 5 + t] = t < d.n ? d.cst[t] : 0.;
    }
  }
  if (threadIdx.x < 3) {
    const int i = threadIdx.x;
    const double q = Q3[i], wq = W3[i] * (1. + exp(-q));
    R.ncdm_w[3 * i] = wq / (q * q);
    R.ncdm_w[3 * i + 1] = wq / q;
    R.ncdm_w[3 * i + 2] = wq;
  }
  for (int l = threadIdx.x; l <= LMAXT; l += blockDim.x) {
    R.ta[l] = (l == 1) ? 6. / 7. : (double)l / (2. * l + 1.);
    R.tg[l] = (l == 1) ? 4. / 7. : (double)(l + 1) / (2. * l + 1.);
  }
  __syncthreads();
  WarpMem m;
  carve(smem + (size_t)wib * (warp_mem_doubles(P.max_ny, P.ncm) + tan_mem_doubles(P.max_ny, P.ncm, TAN ? P.nd : 0)),
        P.max_ny, P.ncm, m);
#ifdef ABCMB_PHASE_CLOCKS
  const int ph_index = blockIdx.x * (blockDim.x >> 5) + wib;
  unsigned long long* ph_slot = ph_index < PHASE_SLOTS ? g_pert_phase + (size_t)ph_index * PHASE_N : nullptr;
  long long ph_t = clock64();
#endif
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
    const double inv_n = 1. / (double)n;
    const bool ncdm = c.has_ncdm != 0;
    // a descriptor this launch cannot hold is reported, never indexed
    {
      const int lmx = max(max(L.lg, L.lp), max(L.lnu, ncdm ? L.lm : 4));
      const int lmn = min(min(L.lg, L.lp), min(L.lnu, ncdm ? L.lm : 4));
      bool bad = n > P.max_ny || L.nc > P.ncm || lmx > LMAXT || lmn < 4 || n != c.ny;
      if constexpr (TAN) {
        // every variant shares the base's state layout and k grid
        for (int j = 0; j < 2 * P.nd; ++j) {
          const int v = P.dirs[(ci * ND_MAX + (j >> 1)) * 2 + (j & 1)];
          bad = bad || v < 0 || v >= P.n_cosmo;
          if (!bad) {
            const abcmb_cosmo& cv = P.cosmo[v];
            bad = cv.ny != c.ny || cv.nk != c.nk || cv.has_ncdm != c.has_ncdm || cv.lmax_g != c.lmax_g ||
                  cv.lmax_pol_g != c.lmax_pol_g || cv.lmax_nu != c.lmax_nu || cv.lmax_ncdm != c.lmax_ncdm;
          }
        }
      }
      if constexpr (IND == 2) {
        // a variant replays a base item of the same k and state layout
        const int rb = P.var_base[item];
        bad = bad || rb < 0 || rb >= P.n_base;
        if (!bad) {
          const int cb = P.base_items[2 * rb];
          bad = cb < 0 || cb >= P.n_cosmo || P.base_items[2 * rb + 1] != ik;
          if (!bad) {
            const abcmb_cosmo& cv = P.cosmo[cb];
            bad = cv.ny != c.ny || cv.nk != c.nk || cv.has_ncdm != c.has_ncdm || cv.lmax_g != c.lmax_g ||
                  cv.lmax_pol_g != c.lmax_pol_g || cv.lmax_nu != c.lmax_nu || cv.lmax_ncdm != c.lmax_ncdm ||
                  ik < 0 || ik >= c.nk || P.kbuf[cv.off_k + ik] != P.kbuf[c.off_k + ik];
          }
        }
      }
      if (bad) {
        if (lane == 0) {
          abcmb_kstat st{ABCMB_STATUS_BAD_LAYOUT, 0, 0, 0, 0.};
          P.kstat[item] = st;
          if (TAN && P.tstat) P.tstat[2 * item] = P.tstat[2 * item + 1] = 0;
          if (IND == 1) P.rec_n[item] = -1;
        }
        continue;
      }
    }
    const double k = P.kbuf[c.off_k + ik];
    const double ik2 = 1. / (k * k);
    const BGK K = bg_constants(c);
    const double rtol = k > S.k_split ? S.rtol_large : S.rtol_small;
    const double atol = k > S.k_split ? S.atol_large : S.atol_small;
    const int nsave = S.n_save;
    const double lts = c.lna_transfer_start;

    // start time (perturbations.py:274-279)
    const double lna2 = np_interp_lna(S.R_large, nullptr, P.aHg + (int64_t)ci * NSTART, k);
    const double lna_start = fmin(fmin(P.lna1[ci], lna2), -10.);

    // per-item structure: tail coefficients, core map, this lane's core row
    for (int t = lane; t < L.ntail; t += WARP) {
      int chn, l, e, lmax = 0;
      tail_elem(L, t, chn, l, e, lmax);
      // F3' and N3' carry 6/7 on their l = 2 slot (which holds sigma = F_2 / 2;
      // species.py:745 and 1435): table slot 1; every other l uses slot l
      const int li = (l == 3 && (chn == 0 || chn == 2)) ? 1 : l;
      m.tinfo()[t] = e | (chn << 12) | ((l == lmax) ? (1 << 15) : 0) | (li << 16);
    }
    if (lane < NCHAIN) {
      int s, lm, o;
      chain_info(L, lane, s, lm, o);
      m.chs()[lane] = s;
      m.chL()[lane] = lm;
    }
    if (lane < L.nc) {
      m.cmap()[lane] = core_state(L, lane);
#pragma unroll
      for (int t = 0; t < 5; ++t) m.rstate()[lane * 5 + t] = core_state(L, t < R.n[lane] ? R.col[lane * 5 + t] : 0);
    }
    // initial conditions (perturbations.py:161-199 + species y_ini)
    for (int e = lane; e < n; e += WARP) m.y0()[e] = 0.;
    __syncwarp();
    if (lane == 0) {
      write_ic(c, L, P.tables, k, lna_start, m.y0());
      stage_basis(c, K, P.tables, k, ik2, R.ncdm_w, lna_start, m.SB(), nullptr);
      m.SV()[16] = -1.;                                      // no save background computed yet
    }
    __syncwarp();

    double t0 = lna_start;
    double t1 = fmin(t0 + S.dt0, 0.0);
    double prev_inv = 1.0, prev_prev_inv = 1.0;
    int isave = 0, nsteps = 0, nacc = 0, nrej = 0, nnewton = 0, status = ABCMB_STATUS_OK;
    unsigned itbits = 0u;            // chord iterations of the step's stages (record / replay)
    int rbase = 0, rn = 0;           // replay: the base item and its recorded steps
    if constexpr (IND == 2) {
      rbase = P.var_base[item];
      rn = P.rec_n[rbase];
      if (rn <= 0) status = ABCMB_STATUS_NONFINITE;      // the base item failed: nothing to replay
    }
    CoreRow cr;
    core_row_at(L, R, m, m.SB(), lane, cr);
    apply_A(L, m, R, cr, m.SB(), m.y0(), m.F(), nullptr, ncdm, lane);   // FSAL stage 1
    if constexpr (TAN) tangent_init(L, m, R, P, ci, k, ik2, lna_start, lane);

    while (t0 < 0.0 && status == ABCMB_STATUS_OK) {
      PERT_PHASE(7);
      if constexpr (IND == 2) {
        if (nsteps >= rn) { status = ABCMB_STATUS_NONFINITE; break; }
        t1 = P.rec_t1[(int64_t)rbase * P.rec_cap + nsteps];
        itbits = (unsigned)P.rec_it[(int64_t)rbase * P.rec_cap + nsteps];
        if (!(t1 > t0)) { status = ABCMB_STATUS_DT_UNDERFLOW; break; }
      } else {
        if (nsteps >= S.max_steps) { status = ABCMB_STATUS_MAX_STEPS; break; }
        itbits = 0u;
      }
      ++nsteps;
      const double h = t1 - t0;
      const double hg = h * KV_G;
      // background of the five distinct stage times, one lane each
      {
        // lanes 0-4: the five distinct stage times; lane 5: the next save
        // point if this step's candidate end covers it
        const double tsn = isave < nsave ? linspace_at(lts, 0.0, nsave, isave) : 1.0;
        const bool want_sv = lane == NSLOT - 1 && tsn <= t1 && (double)isave != m.SV()[16];
        if (lane < NSLOT - 1 || want_sv)
          stage_basis(c, K, P.tables, k, ik2, R.ncdm_w, want_sv ? tsn : t0 + KV_C[lane + 1] * h, m.SB() + (lane + 1) * NB,
                      want_sv ? m.SV() : nullptr);
        if (want_sv) m.SV()[16] = (double)isave;
      }
      __syncwarp();
      PERT_PHASE(0);
      factor_newton(L, m, R, m.SB() + NB, hg, ncdm, lane);
      PERT_PHASE(1);
      bool ok = true;
      for (int i = 1; i < 7 && ok; ++i) {
        const double* B = m.SB() + (i == 6 ? 5 : i) * NB;
        double* fi = m.F() + i * n;
        {
          // F rows 0..i-1 are read, row i (fi), base and v written: disjoint
          const double* __restrict__ Fr = m.F();
          const double* __restrict__ y0 = m.y0();
          double* __restrict__ bw = m.base();
          double* __restrict__ fw = fi;
          double* __restrict__ vw = m.v();
          for (int e = lane; e < n; e += WARP) {
            double acc = 0., acc2 = 0.;
            int j = 0;
            for (; j + 1 < i; j += 2) {
              acc = fma(KV_A[i][j], Fr[j * n + e], acc);
              acc2 = fma(KV_A[i][j + 1], Fr[(j + 1) * n + e], acc2);
            }
            if (j < i) acc = fma(KV_A[i][j], Fr[j * n + e], acc);
            const double be = y0[e] + h * (acc + acc2);
            const double fe = Fr[(i - 1) * n + e];              // predictor: the previous stage's f
            bw[e] = be;
            fw[e] = fe;
            vw[e] = be + hg * fe;                               // first chord argument
          }
        }
        if (i != 6) core_row_at(L, R, m, B, lane, cr);       // stage 7 shares stage 6's time
        __syncwarp();
        PERT_PHASE(2);
        double diffsize = INFINITY, diffsize_prev;
        bool conv = false;
        const int it_replay = (int)((itbits >> (4 * (i - 1))) & 15u);
        for (int it = 1; it <= root_max; ++it) {
          apply_A(L, m, R, cr, B, m.v(), m.r(), fi, ncdm, lane);    // residual A v - f
          PERT_PHASE(3);
          solve_newton(L, m, m.r(), lane, m.vc());
          PERT_PHASE(4);
          double ss = 0.;
          {
            // disjoint regions of the warp's scratch: no load waits on a store
            const double* __restrict__ rr = m.r();
            const double* __restrict__ bb = m.base();
            double* __restrict__ ff = fi;
            double* __restrict__ vv = m.v();
            for (int e = lane; e < n; e += WARP) {
              double x = rr[e];
              double fnew = ff[e] + x;
              ff[e] = fnew;
              vv[e] = bb[e] + hg * fnew;                        // the next iteration's argument
              if constexpr (IND != 2) {                         // a replay needs no termination test
                double q = x * pos_rcp(atol + rtol * fabs(fnew));
                ss += q * q;
              }
            }
          }
          if constexpr (IND != 2) ss = warp_sum(ss);
          __syncwarp();
          if constexpr (IND != 2) {
            diffsize_prev = diffsize;
            diffsize = sqrt(ss * inv_n);
          }
          ++nnewton;
          PERT_PHASE(5);
          if constexpr (IND == 2) {
            if (it >= it_replay) {
              conv = true;
              break;
            }
          } else if (it >= 2) {
            // optimistix very-chord termination, without divisions:
            // rate = d/dp; converged <=> 0 < rate < 1 and d rate / (1 - rate) < kappa
            //                        <=> 0 < d < dp and d^2 < kappa (dp - d);
            // diverged <=> rate not finite or rate > 2 <=> !(d <= 2 dp)
            const double d = diffsize, dp = diffsize_prev;
            const bool small = d < small_res;
            const bool converged = d > 0. && d < dp && d * d < kappa * (dp - d);
            const bool diverged = !(d <= 2. * dp);
            if (small || converged) {
              if constexpr (IND == 1) itbits |= (unsigned)it << (4 * (i - 1));
              conv = true;
              break;
            }
            if (diverged) break;
          }
        }
        if (!conv) ok = false;
      }
      double scaled = INFINITY;
      if (ok) {
        double ss = 0.;
        const double* __restrict__ Fr = m.F();
        const double* __restrict__ y0 = m.y0();
        double* __restrict__ y1 = m.y1();
        for (int e = lane; e < n; e += WARP) {
          double acc = 0., acce = 0., accb = 0., acceb = 0.;
#pragma unroll
          for (int j = 0; j < 6; j += 2) {
            const double fa = Fr[j * n + e], fb = Fr[(j + 1) * n + e];
            acc = fma(KV_A[6][j], fa, acc);
            acce = fma(KV_A[6][j] - KV_A[5][j], fa, acce);
            accb = fma(KV_A[6][j + 1], fb, accb);
            acceb = fma(KV_A[6][j + 1] - KV_A[5][j + 1], fb, acceb);
          }
          acc = fma(KV_G, Fr[6 * n + e], acc + accb);
          acce = (acce + acceb) + (-KV_G * Fr[5 * n + e] + KV_G * Fr[6 * n + e]);
          double y0e = y0[e];
          double y1e = y0e + h * acc;
          y1[e] = y1e;
          if constexpr (IND == 2) {
            // a replay takes the step: only a non-finite state stops it
            if (!isfinite(y1e)) ss = INFINITY;
          } else {
            double err = h * acce;
            double q = err * pos_rcp(atol + fmax(fabs(y0e), fabs(y1e)) * rtol);
            ss += q * q;
          }
        }
        if constexpr (IND == 2) {
          scaled = __any_sync(0xffffffffu, ss != 0.) ? INFINITY : 0.;
        } else {
          ss = warp_sum(ss);
          scaled = sqrt(ss * inv_n);
        }
        if (!isfinite(scaled)) scaled = INFINITY;
      }
      __syncwarp();
      bool keep = scaled < 1.0;
      if constexpr (IND == 2) {
        // the base accepted this step: the variant takes it (scaled is 0, or
        // infinite for a non-finite state, which stops the item)
        if (!keep) status = ABCMB_STATUS_NONFINITE;
      }
      double inv = 1.0 / scaled;
      double f1v = (coeff1 == 0.) ? 1. : pow(inv, coeff1);
      double f2v = (coeff2 == 0.) ? 1. : pow(prev_inv, coeff2);
      double f3v = (coeff3 == 0.) ? 1. : pow(prev_prev_inv, coeff3);
      double factor = fmin(fmax(safety * f1v * f2v * f3v, keep ? 1.0 : factormin), factormax);
      double dt_new = h * factor;
      if (inv == 0. || isinf(inv)) inv = 1.;
      PERT_PHASE(6);
      if (keep) {
        if constexpr (IND == 1) {
          if (lane == 0) {
            P.rec_t1[(int64_t)item * P.rec_cap + nacc] = t1;
            P.rec_it[(int64_t)item * P.rec_cap + nacc] = (int32_t)itbits;
          }
        }
        ++nacc;
        if constexpr (TAN) {
          for (int q = 0; q < P.nd; ++q)
            tangent_pass(L, m, R, P, q, k, ik2, t0, h, rtol, atol * P.tscale, inv_n, lts, isave, ik, lane);
          PERT_PHASE_RESET();
        }
        // cubic Hermite dense output on [t0, t1] at every save point it covers
        while (isave < nsave) {
          double ts = linspace_at(lts, 0.0, nsave, isave);
          if (!(ts <= t1)) break;
          double th = (ts - t0) / h;
          {
            const double* __restrict__ y0 = m.y0();
            const double* __restrict__ y1 = m.y1();
            const double* __restrict__ Fr = m.F();
            double* __restrict__ vv = m.v();
            for (int e = lane; e < n; e += WARP) {
              double y0e = y0[e], y1e = y1[e];
              double k0 = h * Fr[e], k1 = h * Fr[6 * n + e];
              vv[e] = y0e + th * (k0 + th * ((3. * (y1e - y0e) - 2. * k0 - k1) + th * (2. * (y0e - y1e) + k0 + k1)));
            }
          }
          __syncwarp();
          write_fields(c, L, P.tables, k, ts, m.v(), P.pt, nsave, isave, ik, lane,
                       m.SV()[16] == (double)isave ? m.SV() : nullptr, R.ncdm_w);
          __syncwarp();
          ++isave;
        }
        prev_prev_inv = prev_inv;
        prev_inv = inv;
        for (int e = lane; e < n; e += WARP) {
          m.y0()[e] = m.y1()[e];
          m.F()[e] = m.F()[6 * n + e];
        }
        m.SB()[lane] = m.SB()[5 * NB + lane];                  // basis at the new t0
        __syncwarp();
        t0 = t1;
      } else {
        ++nrej;
      }
      if (t0 >= 0.0 || IND == 2) continue;
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
      if (IND == 1) P.rec_n[item] = status == ABCMB_STATUS_OK ? nacc : -1;
      if (TAN && P.tstat) {
        const int* cnt = tan_mem(m, P).cnt();
        P.tstat[2 * item] = cnt[0];
        P.tstat[2 * item + 1] = cnt[1];
      }
    }
    __syncwarp();
  }
}

}  // namespace abcmb

// ---------------------------------------------------------------------------
// host launcher (called from capi.cu)
// ---------------------------------------------------------------------------
namespace abcmb {

template <int MIN_BLOCKS>
__global__ void __launch_bounds__(PERT_THREADS_MAX, MIN_BLOCKS) pert_kernel(PertArgs P) {
  pert_body<false>(P);
}

// The record (IND = 1) and replay (IND = 2) integrations of abcmb_pert_forward_ind.
template <int MIN_BLOCKS, int IND>
__global__ void __launch_bounds__(PERT_THREADS_MAX, MIN_BLOCKS) pert_kernel_ind(PertArgs P) {
  pert_body<false, IND>(P);
}

// The same integration with the tangents; shared memory (not registers)
// limits its occupancy, so the register cap stays off.
__global__ void __launch_bounds__(PERT_THREADS_MAX, 1) pert_kernel_tangent(PertArgs P) {
  pert_body<true>(P);
}

int pert_phase_clocks(unsigned long long* out, int reset) {
#ifdef ABCMB_PHASE_CLOCKS
  static unsigned long long h[PHASE_SLOTS * PHASE_N];
  cudaError_t e = cudaMemcpyFromSymbol(h, g_pert_phase, sizeof(h));
  if (e != cudaSuccess) return -2;
  for (int k = 0; k < PHASE_N; ++k) out[k] = 0;
  for (int i = 0; i < PHASE_SLOTS; ++i)
    for (int k = 0; k < PHASE_N; ++k) out[k] += h[(size_t)i * PHASE_N + k];
  if (reset) {
    static const unsigned long long zero[PHASE_SLOTS * PHASE_N] = {};
    e = cudaMemcpyToSymbol(g_pert_phase, zero, sizeof(zero));
    if (e != cudaSuccess) return -2;
  }
  return 0;
#else
  (void)out;
  (void)reset;
  return -1;
#endif
}

// launch choices set through the C ABI (capi.cu): 0 = automatic
int pert_variant();
int pert_tangent_warps();

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
  PertArgs A{};
  A.n_cosmo = n_cosmo;
  A.n_items = n_items;
  A.max_ny = s.max_ny;
  A.ncm = s.any_ncdm ? 22 : 13;
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
  A.nd = 0;
  A.tscale = 1.;
  A.dirs = nullptr;
  A.tstat = nullptr;
  if (warps_per_block < 1 || 32 * warps_per_block > PERT_THREADS_MAX) return cudaErrorInvalidConfiguration;
  const int threads = 32 * warps_per_block;
  const size_t smem = (size_t)warps_per_block * pert_smem_per_warp(s.max_ny, A.ncm);
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // a long queue (many items per warp) favours more resident warps; a short
  // one is bounded by its slowest items and favours the uncapped registers
  const int variant = pert_variant();
  const bool throughput =
      variant == 2 ||
      (variant == 0 &&
       (int64_t)n_items >= (int64_t)PERT_THROUGHPUT_ITEMS_PER_WARP * nsm * PERT_BLOCKS_LATENCY * warps_per_block);
  const void* fn = throughput ? (const void*)pert_kernel<PERT_BLOCKS_THROUGHPUT>
                              : (const void*)pert_kernel<PERT_BLOCKS_LATENCY>;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int grid = nsm * per_sm;
  int need = (n_items + warps_per_block - 1) / warps_per_block;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  if (grid_out) *grid_out = grid;
  if (throughput) pert_kernel<PERT_BLOCKS_THROUGHPUT><<<grid, threads, smem, stream>>>(A);
  else pert_kernel<PERT_BLOCKS_LATENCY><<<grid, threads, smem, stream>>>(A);
  return cudaGetLastError();
}

int64_t pert_ind_workspace_bytes(int n_cosmo, int n_base, int max_steps) {
  int64_t b = pert_workspace_bytes(n_cosmo) + 256;                   // + the replay's queue counter
  b += ((int64_t)n_base * max_steps * 8 + 255) / 256 * 256;          // recorded step ends
  b += ((int64_t)n_base * max_steps * 4 + 255) / 256 * 256;          // recorded chord iterations
  b += ((int64_t)n_base * 4 + 255) / 256 * 256;                      // recorded step counts
  return b;
}

// abcmb_pert_forward_ind: the base items (the first n_base of items) are
// integrated recording their accepted steps, then the variant items replay
// their base item's steps; both launches in stream order on one queue each.
cudaError_t launch_pert_ind(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                            int n_base, int n_var, const int32_t* items, const int32_t* var_base,
                            const abcmb_pert_settings& s, double* pt, abcmb_kstat* kstat, void* ws,
                            cudaStream_t stream, int warps_per_block, int* grid_out) {
  if (warps_per_block < 1 || 32 * warps_per_block > PERT_THREADS_MAX) return cudaErrorInvalidConfiguration;
  char* w = static_cast<char*>(ws);
  int* queue = reinterpret_cast<int*>(w);
  w += 256;
  double* lna1 = reinterpret_cast<double*>(w);
  w += ((int64_t)n_cosmo * 8 + 255) / 256 * 256;
  double* aHg = reinterpret_cast<double*>(w);
  w += ((int64_t)n_cosmo * NSTART * 8 + 255) / 256 * 256;
  double* f1g = reinterpret_cast<double*>(w);
  w += ((int64_t)n_cosmo * NSTART * 8 + 255) / 256 * 256;
  int* queue2 = reinterpret_cast<int*>(w);
  w += 256;
  double* rec_t1 = reinterpret_cast<double*>(w);
  w += ((int64_t)n_base * s.max_steps * 8 + 255) / 256 * 256;
  int32_t* rec_it = reinterpret_cast<int32_t*>(w);
  w += ((int64_t)n_base * s.max_steps * 4 + 255) / 256 * 256;
  int32_t* rec_n = reinterpret_cast<int32_t*>(w);
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(queue2, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  dim3 g1((NSTART + 255) / 256, n_cosmo);
  start_grid_kernel<<<g1, 256, 0, stream>>>(n_cosmo, cosmo, tables, aHg, f1g);
  start_lna1_kernel<<<(n_cosmo + 127) / 128, 128, 0, stream>>>(n_cosmo, f1g, s.R_tc, lna1);
  PertArgs A{};
  A.n_cosmo = n_cosmo;
  A.max_ny = s.max_ny;
  A.ncm = s.any_ncdm ? 22 : 13;
  A.cosmo = cosmo;
  A.tables = tables;
  A.kbuf = kbuf;
  A.pt = pt;
  A.aHg = aHg;
  A.lna1 = lna1;
  A.s = s;
  A.nd = 0;
  A.tscale = 1.;
  A.rec_t1 = rec_t1;
  A.rec_it = rec_it;
  A.rec_n = rec_n;
  A.rec_cap = s.max_steps;
  A.n_base = n_base;
  A.base_items = items;
  A.var_base = var_base;
  const int threads = 32 * warps_per_block;
  const size_t smem = (size_t)warps_per_block * pert_smem_per_warp(s.max_ny, A.ncm);
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int variant = pert_variant();
  for (int pass = 0; pass < 2; ++pass) {
    const int n_items = pass == 0 ? n_base : n_var;
    if (n_items == 0) continue;
    A.n_items = n_items;
    A.items = pass == 0 ? items : items + 2 * (int64_t)n_base;
    A.kstat = pass == 0 ? kstat : kstat + n_base;
    A.queue = pass == 0 ? queue : queue2;
    const bool throughput =
        variant == 2 ||
        (variant == 0 &&
         (int64_t)n_items >= (int64_t)PERT_THROUGHPUT_ITEMS_PER_WARP * nsm * PERT_BLOCKS_LATENCY * warps_per_block);
    const void* fn;
    if (pass == 0)
      fn = throughput ? (const void*)pert_kernel_ind<PERT_BLOCKS_THROUGHPUT, 1>
                      : (const void*)pert_kernel_ind<PERT_BLOCKS_LATENCY, 1>;
    else
      fn = throughput ? (const void*)pert_kernel_ind<PERT_BLOCKS_THROUGHPUT, 2>
                      : (const void*)pert_kernel_ind<PERT_BLOCKS_LATENCY, 2>;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int grid = nsm * per_sm;
    const int need = (n_items + warps_per_block - 1) / warps_per_block;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    if (grid_out) *grid_out = grid;
    void* args[] = {&A};
    e = cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, smem, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

size_t pert_tangent_smem_per_warp(int max_ny, int ncm, int nd) {
  return (warp_mem_doubles(max_ny, ncm) + tan_mem_doubles(max_ny, ncm, nd)) * sizeof(double);
}

// abcmb_pert_forward_tangent: the items are base cosmologies; warps per
// block is chosen (1..4) for the most resident warps per SM, since the
// per-warp shared memory (the tangents' stage derivatives) sets occupancy.
cudaError_t launch_pert_tangent(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                                int n_items, const int32_t* items, int nd, const int32_t* dirs, double tscale,
                                const abcmb_pert_settings& s, double* pt, abcmb_kstat* kstat, int32_t* tstat,
                                void* ws, cudaStream_t stream, int* grid_out, int* warps_out) {
  if (nd < 1 || nd > ND_MAX) return cudaErrorInvalidValue;
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
  PertArgs A{};
  A.n_cosmo = n_cosmo;
  A.n_items = n_items;
  A.max_ny = s.max_ny;
  A.ncm = s.any_ncdm ? 22 : 13;
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
  A.nd = nd;
  A.tscale = tscale;
  A.dirs = dirs;
  A.tstat = tstat;
  const size_t per_warp = pert_tangent_smem_per_warp(s.max_ny, A.ncm, nd);
  const void* fn = (const void*)pert_kernel_tangent;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  int best_w = 0, best_blocks = 0, best_total = 0;
  const int fixed_w = pert_tangent_warps();
  for (int wpb = PERT_THREADS_MAX / 32; wpb >= 1; --wpb) {
    if (fixed_w > 0 && wpb != fixed_w) continue;
    const size_t smem = (size_t)wpb * per_warp;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * wpb, smem) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (per_sm * wpb > best_total) {
      best_total = per_sm * wpb;
      best_w = wpb;
      best_blocks = per_sm;
    }
  }
  if (best_total < 1) return cudaErrorInvalidConfiguration;
  const size_t smem = (size_t)best_w * per_warp;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int grid = nsm * best_blocks;
  const int need = (n_items + best_w - 1) / best_w;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  if (grid_out) *grid_out = grid;
  if (warps_out) *warps_out = best_w;
  pert_kernel_tangent<<<grid, 32 * best_w, smem, stream>>>(A);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// vector-Jacobian product with respect to the gradient parameters
// ---------------------------------------------------------------------------
constexpr int VJP_THREADS = 256;

// theta_bar[b][p] = <pt_bar(base b), (PT(plus) - PT(minus)) / (2 step)>
// over the base descriptor's whole PerturbationTable (fields x saves x k):
// one block per (direction, base), a fixed-order block reduction (the same
// result on every run).  A plus / minus descriptor outside the batch or of
// another table shape gives NaN.
__global__ void __launch_bounds__(VJP_THREADS) pert_vjp_theta_kernel(int n_cosmo, const abcmb_cosmo* __restrict__ cosmo,
                                                                     const double* __restrict__ pt,
                                                                     const double* __restrict__ pt_bar, int n_save,
                                                                     const int32_t* __restrict__ base, int n_dir,
                                                                     const int32_t* __restrict__ dirs,
                                                                     const double* __restrict__ step,
                                                                     double* __restrict__ theta_bar) {
  __shared__ double red[VJP_THREADS];
  const int q = blockIdx.x, b = blockIdx.y;
  const int cb = base[b];
  const int cp = dirs[(b * n_dir + q) * 2], cm = dirs[(b * n_dir + q) * 2 + 1];
  const bool ok = cb >= 0 && cb < n_cosmo && cp >= 0 && cp < n_cosmo && cm >= 0 && cm < n_cosmo &&
                  cosmo[cp].nk == cosmo[cb].nk && cosmo[cm].nk == cosmo[cb].nk;
  double acc = 0.;
  if (ok) {
    const int64_t n = (int64_t)ABCMB_NFIELDS * n_save * cosmo[cb].nk;
    const double* __restrict__ g = pt_bar + cosmo[cb].off_pt;
    const double* __restrict__ xp = pt + cosmo[cp].off_pt;
    const double* __restrict__ xm = pt + cosmo[cm].off_pt;
    for (int64_t j = threadIdx.x; j < n; j += VJP_THREADS) acc = fma(g[j], xp[j] - xm[j], acc);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = VJP_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) theta_bar[b * n_dir + q] = ok ? red[0] / (2. * step[b * n_dir + q]) : NAN;
}

cudaError_t launch_pert_vjp_theta(int n_cosmo, const abcmb_cosmo* cosmo, const double* pt, const double* pt_bar,
                                  int n_save, int n_base, const int32_t* base, int n_dir, const int32_t* dirs,
                                  const double* step, double* theta_bar, cudaStream_t stream) {
  dim3 g(n_dir, n_base);
  pert_vjp_theta_kernel<<<g, VJP_THREADS, 0, stream>>>(n_cosmo, cosmo, pt, pt_bar, n_save, base, n_dir, dirs, step,
                                                        theta_bar);
  return cudaGetLastError();
}

}  // namespace abcmb
