// los.cu -- line-of-sight C_l projection (SpectrumSolver.get_Cl).
//
// Cosmologies are processed in chunks of up to LOS_CHUNK; five launches per
// chunk:
//   spline_prep   not-a-knot cubic-spline factorisation in log10 k of the
//                 perturbation k grid (interpax CubicSpline, spectrum.py:664)
//                 and the interval of every transfer k;
//   spline_slopes the spline slopes of the 10 source fields on every lna row;
//   sources       the splined fields at the transfer k and the T0/T1/T2/E
//                 sources (spectrum.py:681-696);
//   los           one CTA per (tabulated l, k tile, cosmology): the l column
//                 of the phi0/phi1/phi2 Bessel tables is staged in shared
//                 memory and the four lna integrals of every transfer k are
//                 accumulated (spectrum.py:755-786), then the block reduces
//                 its share of the k trapezoid (spectrum.py:789-796);
//   cl_final      fixed-order sum of the tile partials and the cubic spline
//                 over tabulated l onto the integer ells (spectrum.py:597-608).
#include "common.cuh"

namespace abcmb {

constexpr int NSRC_FIELDS = 10;
__constant__ int SRC_FIELDS[NSRC_FIELDS] = {ABCMB_F_G_DELTA, ABCMB_F_B_THETA, ABCMB_F_THETA_B_PRIME,
                                            ABCMB_F_G_SIGMA, ABCMB_F_G_G0, ABCMB_F_G_G2, ABCMB_F_ETA,
                                            ABCMB_F_ETA_PRIME, ABCMB_F_ALPHA, ABCMB_F_ALPHA_PRIME};


// Thomas factors of the not-a-knot system for x[0..n): di (modified
// diagonal inverse), up, lo multipliers; plus x itself.
struct SplineFac {
  double* x;      // n
  double* dinv;   // n  1 / modified diagonal
  double* mlo;    // n  elimination multipliers
  double* up;     // n  super-diagonal
};

// Not-a-knot right-hand side row i (scipy CubicSpline / interpax).
__device__ __forceinline__ double nak_rhs(const double* x, const double* y, int n, int i) {
  if (i == 0) {
    double dx0 = x[1] - x[0], dx1 = x[2] - x[1];
    double s0 = (y[1] - y[0]) / dx0, s1 = (y[2] - y[1]) / dx1;
    double d = x[2] - x[0];
    return ((dx0 + 2. * d) * dx1 * s0 + dx0 * dx0 * s1) / d;
  }
  if (i == n - 1) {
    double dxa = x[n - 2] - x[n - 3], dxb = x[n - 1] - x[n - 2];
    double sa = (y[n - 2] - y[n - 3]) / dxa, sb = (y[n - 1] - y[n - 2]) / dxb;
    double d = x[n - 1] - x[n - 3];
    return (dxb * dxb * sa + (2. * d + dxb) * dxa * sb) / d;
  }
  double dxm = x[i] - x[i - 1], dxp = x[i + 1] - x[i];
  double sm = (y[i] - y[i - 1]) / dxm, sp = (y[i + 1] - y[i]) / dxp;
  return 3. * (dxp * sm + dxm * sp);
}

// Factorise the not-a-knot tridiagonal matrix (one thread; n sequential steps).
__device__ void nak_factor(const double* x, int n, double* dinv, double* mlo, double* up) {
  double di_prev = 0., up_prev = 0.;
  for (int i = 0; i < n; ++i) {
    double lo, di, u;
    if (i == 0) { di = x[2] - x[1]; u = x[2] - x[0]; lo = 0.; }
    else if (i == n - 1) { lo = x[n - 1] - x[n - 3]; di = x[n - 2] - x[n - 3]; u = 0.; }
    else { lo = x[i + 1] - x[i]; di = 2. * ((x[i] - x[i - 1]) + (x[i + 1] - x[i])); u = x[i] - x[i - 1]; }
    double m = 0.;
    if (i > 0) { m = lo * di_prev; di -= m * up_prev; }
    mlo[i] = m;
    up[i] = u;
    dinv[i] = 1. / di;
    di_prev = dinv[i];
    up_prev = u;
  }
}

// Slopes s of the not-a-knot spline through (x, y) using the factorisation.
__device__ void nak_solve(const double* x, const double* y, int n, const double* dinv, const double* mlo,
                          const double* up, double* s) {
  double bprev = 0.;
  for (int i = 0; i < n; ++i) {
    double bi = nak_rhs(x, y, n, i) - mlo[i] * bprev;
    s[i] = bi;
    bprev = bi;
  }
  double snext = s[n - 1] * dinv[n - 1];
  s[n - 1] = snext;
  for (int i = n - 2; i >= 0; --i) {
    snext = (s[i] - up[i] * snext) * dinv[i];
    s[i] = snext;
  }
}

__device__ __forceinline__ double spline_piece(double y0, double y1, double s0, double s1, double dx, double u) {
  double sl = (y1 - y0) / dx;
  double t = (s0 + s1 - 2. * sl) / dx;
  double c3 = t / dx;
  double c2 = (sl - s0) / dx - t;
  return ((c3 * u + c2) * u + s0) * u + y0;
}

// i = clip(searchsorted(x, xq, 'right'), 1, n-1) - 1
__device__ __forceinline__ int spline_interval(const double* x, int n, double xq) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (x[mid] <= xq) lo = mid + 1; else hi = mid;
  }
  return min(max(lo, 1), n - 1) - 1;
}

// Chunked launches: every kernel below covers a chunk of up to LOS_CHUNK
// cosmologies (blockIdx.z, or blockIdx.x for the one-block-per-cosmology
// kernels); per-cosmology scratch lives at a fixed stride in the workspace.
constexpr int LOS_CHUNK = 8;

struct LosScratch {
  double* xk;        // [C][max_nk] log10 of the perturbation k grid
  double* dinv;      // [C][max_nk] not-a-knot factorisation
  double* mlo;
  double* up;
  int* kidx;         // [C][nkt] spline interval of every transfer k
  double* slopes;    // [C][NSRC_FIELDS][nl][max_nk]
  void* S;           // [C][4][nl][nkt] sources (double or float)
  double* partial;   // [C][n_ell_tab][ntile][6]
  double* lscr;      // [C][16 n_ell_tab] l-spline scratch
  double* te;        // null, or [C][n_ell_tab][2][nkt]: T and E of every (l, k) (the adjoint reads them)
  int max_nk;
};

__global__ void spline_prep_kernel(const abcmb_cosmo* __restrict__ cosmo, int c0, const double* __restrict__ kbuf,
                                   const double* __restrict__ kt, int nkt, LosScratch W) {
  // one block per cosmology: threads fill x = log10(PT.k), thread 0
  // factorises, all threads locate the transfer k
  const int cz = blockIdx.x;
  const abcmb_cosmo& c = cosmo[c0 + cz];
  const int nk = c.nk;
  const double* kp = kbuf + c.off_k;
  double* xk = W.xk + (int64_t)cz * W.max_nk;
  for (int i = threadIdx.x; i < nk; i += blockDim.x) xk[i] = log10(kp[i]);
  __syncthreads();
  if (threadIdx.x == 0)
    nak_factor(xk, nk, W.dinv + (int64_t)cz * W.max_nk, W.mlo + (int64_t)cz * W.max_nk, W.up + (int64_t)cz * W.max_nk);
  for (int j = threadIdx.x; j < nkt; j += blockDim.x) W.kidx[(int64_t)cz * nkt + j] = spline_interval(xk, nk, log10(kt[j]));
}

__global__ void spline_slopes_kernel(const abcmb_cosmo* __restrict__ cosmo, int c0, const double* __restrict__ pt,
                                     int n_save, int nl, LosScratch W) {
  const int cz = blockIdx.y;
  const abcmb_cosmo& c = cosmo[c0 + cz];
  const int col = blockIdx.x * blockDim.x + threadIdx.x;    // f * nl + il
  if (col >= NSRC_FIELDS * nl) return;
  const int nk = c.nk;
  const int f = col / nl, il = col % nl;
  const double* y = pt + c.off_pt + ((int64_t)SRC_FIELDS[f] * n_save + il) * nk;
  const int64_t o = (int64_t)cz * W.max_nk;
  nak_solve(W.xk + o, y, nk, W.dinv + o, W.mlo + o, W.up + o,
            W.slopes + ((int64_t)cz * NSRC_FIELDS * nl + col) * W.max_nk);
}

template <typename SrcT>
__global__ void sources_kernel(const abcmb_cosmo* __restrict__ cosmo, int c0, const double* __restrict__ tables,
                               const double* __restrict__ pt, int n_save, int nl, const double* __restrict__ kt,
                               int nkt, abcmb_los_settings ls, LosScratch W) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int il = blockIdx.y;
  const int cz = blockIdx.z;
  if (j >= nkt) return;
  const abcmb_cosmo& c = cosmo[c0 + cz];
  const int nk = c.nk;
  const double* ptc = pt + c.off_pt;
  const double* los = tables + c.off_los;
  const double* xk = W.xk + (int64_t)cz * W.max_nk;
  const double* slopes = W.slopes + (int64_t)cz * NSRC_FIELDS * nl * W.max_nk;
  const double k = kt[j];
  const int i = W.kidx[(int64_t)cz * nkt + j];
  const double dx = xk[i + 1] - xk[i];
  const double u = log10(k) - xk[i];
  double v[NSRC_FIELDS];
#pragma unroll
  for (int f = 0; f < NSRC_FIELDS; ++f) {
    const double* y = ptc + ((int64_t)SRC_FIELDS[f] * n_save + il) * nk;
    const double* s = slopes + ((int64_t)f * nl + il) * W.max_nk;
    v[f] = spline_piece(y[i], y[i + 1], s[i], s[i + 1], dx, u);
  }
  const double dg = v[0], thb = v[1], thbp = v[2], sg = v[3], G0 = v[4], G2 = v[5];
  const double eta = v[6], etap = v[7], al = v[8], alp = v[9];
  const double g = los[1 * nl + il], gp = los[2 * nl + il], aH = los[3 * nl + il];
  const double em = los[4 * nl + il], aHd = los[5 * nl + il];
  double sT0 = ls.scale_sw * g * (dg / 4. + aH * alp) +
               ls.scale_isw * (g * (eta - aH * alp - 2. * aH * al) + 2. * em * (aH * etap - aHd * al - aH * aH * alp)) +
               ls.scale_dop * (aH * (g * ((thbp / (k * k)) + alp) + gp * ((thb / (k * k)) + al)));
  double sT1 = ls.scale_isw * em * ((aH * alp + 2. * aH * al - eta) * k);
  double sT2 = ls.scale_pol * g * (2 * sg + G0 + G2) / 8.;
  double sE = sqrt(6.) * g * (2 * sg + G0 + G2) / 8.;
  const int64_t plane = (int64_t)nl * nkt;
  SrcT* S = static_cast<SrcT*>(W.S) + (int64_t)cz * 4 * plane;
  const int64_t o = (int64_t)il * nkt + j;
  S[o] = (SrcT)sT0;
  S[plane + o] = (SrcT)sT1;
  S[2 * plane + o] = (SrcT)sT2;
  S[3 * plane + o] = (SrcT)sE;
}

// Large-x asymptotic spherical Bessel j_l (spectrum.py:48-51):
//   r = sqrt(x^2 - nu^2), Q = r - nu pi/2 + nu asin(nu/x),
//   j = sqrt(2/(pi r)) cos(Q - pi/4) sqrt(pi/(2x)) = cos(Q - pi/4) / sqrt(r x)
// with nu = l + 1/2 and 1/x supplied by the caller (no division).
__device__ __forceinline__ double jasym(double nu, double nusq, double x, double ix) {
  const double r = sqrt(fma(x, x, -nusq));
  const double Q = r - nu * (PI / 2) + nu * asin(nu * ix);
  return rsqrt(r * x) * cos(Q - PI / 4);
}

// fast_interp (ABCMBTools.py:268-308) with the scale (n-1)/(xp_max-xp_min)
// precomputed; the table is in shared memory.
__device__ __forceinline__ double lerp_tab(double x, double xmin, double scale, const double* fp, int n) {
  const double eps = 1.e-6;
  double i = (x - xmin) * scale;
  i = fmin(fmax(i, eps), (double)(n - 1) - eps);
  const int il = (int)i;
  const int iu = min(il + 1, n - 1);
  const double wu = i - (double)il;
  return (1.0 - wu) * fp[il] + wu * fp[iu];
}

constexpr int LOS_TX = 256;   // transfer k per CTA (one per thread column)
constexpr int LOS_TY = 3;     // lna segments: thread row y sums segment y
constexpr int LOS_THREADS = LOS_TX * LOS_TY;

// Kahan-compensated accumulator for the FP32 path.
struct KahanF {
  float s, c;
  __device__ void add(float v) {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// One CTA per (tabulated l, 256-wide transfer-k tile, cosmology of the
// chunk).  The l column of the three Bessel tables and the per-lna factors
// (tau0 - tau, its reciprocal, w / aH) sit in shared memory; each thread
// column owns one transfer k and each of the LOS_TY thread rows sums every
// LOS_TY-th lna point; the rows' sums are added in row order.  Shared memory (~148 KB) admits one CTA per SM: 24 resident warps.
template <int PREC>
__global__ void __launch_bounds__(LOS_THREADS, 1) los_kernel(const abcmb_cosmo* __restrict__ cosmo, int c0,
                                                             const double* __restrict__ tables, int nl, int n_save,
                                                             const double* __restrict__ kt, int nkt, BesselDev B,
                                                             int idx_min, double k_pivot, LosScratch W) {
  extern __shared__ double sm[];
  const int ie = blockIdx.x, tile = blockIdx.y, cz = blockIdx.z;
  const int n_ell = gridDim.x, ntile = gridDim.y;
  const int idx = idx_min + ie;
  const int nx = B.n_x;
  double* ph0 = sm;
  double* ph1 = ph0 + nx;
  double* ph2 = ph1 + nx;
  double* sdt = ph2 + nx;          // tau0 - tau_i
  double* sidt = sdt + nl;         // 1 / (tau0 - tau_i)
  double* swa = sidt + nl;         // w_i / aH_i
  double* seg = swa + nl;          // [LOS_TY - 1][4][LOS_TX] segment sums of rows 1..
  const int tid = threadIdx.y * LOS_TX + threadIdx.x;
  const abcmb_cosmo& c = cosmo[c0 + cz];
  const double* los = tables + c.off_los;
  for (int i = tid; i < nx; i += LOS_THREADS) {
    ph0[i] = B.phi[((int64_t)0 * B.n_l + idx) * nx + i];
    ph1[i] = B.phi[((int64_t)1 * B.n_l + idx) * nx + i];
    ph2[i] = B.phi[((int64_t)2 * B.n_l + idx) * nx + i];
  }
  const double lts = c.lna_transfer_start;
  const double delta_lna = linspace_at(lts, 0., n_save, n_save - 1) - linspace_at(lts, 0., n_save, n_save - 2);
  for (int i = tid; i < nl; i += LOS_THREADS) {
    const double d = c.tau0 - los[i];
    sdt[i] = d;
    sidt[i] = 1.0 / d;
    swa[i] = ((i == 0) ? 0.5 * delta_lna : delta_lna) * (1.0 / los[3 * nl + i]);
  }
  __syncthreads();
  const double l = (double)B.l_tab[idx];
  const double x0min = B.xmin[idx], x0max = B.xmax[idx];
  const double x1min = B.xmin[B.n_l + idx], x1max = B.xmax[B.n_l + idx];
  const double x2min = B.xmin[2 * B.n_l + idx], x2max = B.xmax[2 * B.n_l + idx];
  const double s0 = (double)(nx - 1) / (x0max - x0min);
  const double s1 = (double)(nx - 1) / (x1max - x1min);
  const double s2 = (double)(nx - 1) / (x2max - x2min);
  const double ef = sqrt(3. / 8. * (l + 2) * (l + 1) * l * (l - 1));
  const double nu0 = l + 0.5, nu1 = l + 1.5;
  const double nu0sq = nu0 * nu0, nu1sq = nu1 * nu1;
  const double c2 = 3 * l * (l - 1);
  const int j = tile * LOS_TX + threadIdx.x;
  const int iy = threadIdx.y;
  double a0 = 0., a1 = 0., a2 = 0., aE = 0.;
  double k = 0.;
  if (j < nkt) {
    k = kt[j];
    const double invk = 1.0 / k;
    const int64_t plane = (int64_t)nl * nkt;
    KahanF f0{0.f, 0.f}, f1{0.f, 0.f}, f2{0.f, 0.f}, fE{0.f, 0.f};
    // row iy takes lna points iy, iy + LOS_TY, ...: the costly early points
    // (large k chi: asymptotic j_l) are shared evenly between the rows
    for (int il = iy; il < nl; il += LOS_TY) {
      const double chi = sdt[il] * k;
      const double ichi = sidt[il] * invk;
      // phi0/phi1/phi2 (spectrum.py:719-753): 0 below the table, table
      // lerp inside, asymptotic j_l above; only the taken branch is evaluated
      double p0;
      if (chi < x0min) p0 = 0.;
      else if (chi >= x0max) p0 = jasym(nu0, nu0sq, chi, ichi);
      else p0 = lerp_tab(chi, x0min, s0, ph0, nx);
      const bool as1 = chi >= x1max, as2 = chi >= x2max;
      double jl = 0., jl1 = 0.;
      if (as1 || as2) {
        jl = (chi >= x0max) ? p0 : jasym(nu0, nu0sq, chi, ichi);
        jl1 = jasym(nu1, nu1sq, chi, ichi);
      }
      double p1, p2;
      if (chi < x1min) p1 = 0.;
      else if (as1) p1 = l * ichi * jl - jl1;
      else p1 = lerp_tab(chi, x1min, s1, ph1, nx);
      const double ichi2 = ichi * ichi;
      if (chi < x2min) p2 = 0.;
      else if (as2) p2 = ((c2 - 2 * chi * chi) * jl + 6 * chi * jl1) * 0.5 * ichi2;
      else p2 = lerp_tab(chi, x2min, s2, ph2, nx);
      const double eps = p0 * ichi2 * ef;
      const double wa = swa[il];
      const int64_t o = (int64_t)il * nkt + j;
      if (PREC == 0) {
        const double* S = static_cast<const double*>(W.S) + (int64_t)cz * 4 * plane;
        a0 = fma(wa * S[o], p0, a0);
        a1 = fma(wa * S[plane + o], p1, a1);
        a2 = fma(wa * S[2 * plane + o], p2, a2);
        aE = fma(wa * S[3 * plane + o], eps, aE);
      } else {
        const float* S = static_cast<const float*>(W.S) + (int64_t)cz * 4 * plane;
        const float wf = (float)wa;
        f0.add(wf * S[o] * (float)p0);
        f1.add(wf * S[plane + o] * (float)p1);
        f2.add(wf * S[2 * plane + o] * (float)p2);
        fE.add(wf * S[3 * plane + o] * (float)eps);
      }
    }
    if (PREC != 0) {
      a0 = (double)f0.s - (double)f0.c;
      a1 = (double)f1.s - (double)f1.c;
      a2 = (double)f2.s - (double)f2.c;
      aE = (double)fE.s - (double)fE.c;
    }
  }
  if (iy > 0) {
    double* sg = seg + (int64_t)(iy - 1) * 4 * LOS_TX + threadIdx.x;
    sg[0] = a0;
    sg[LOS_TX] = a1;
    sg[2 * LOS_TX] = a2;
    sg[3 * LOS_TX] = aE;
  }
  __syncthreads();
  if (iy != 0) return;
  double contrib[6] = {0., 0., 0., 0., 0., 0.};
  if (j < nkt) {
    for (int y = 1; y < LOS_TY; ++y) {
      const double* sg = seg + (int64_t)(y - 1) * 4 * LOS_TX + threadIdx.x;
      a0 += sg[0];
      a1 += sg[LOS_TX];
      a2 += sg[2 * LOS_TX];
      aE += sg[3 * LOS_TX];
    }
    const double T = a0 + a1 + a2;
    const double E = aE;
    if (W.te) {
      double* te = W.te + (((int64_t)cz * n_ell + ie) * 2) * nkt;
      te[j] = T;
      te[nkt + j] = E;
    }
    const double pr = 4. * PI * c.A_s * pow(k / k_pivot, c.n_s - 1.) / k;
    // trapezoid weight of node j
    double wj;
    if (nkt == 1) wj = 0.;
    else if (j == 0) wj = 0.5 * (kt[1] - kt[0]);
    else if (j == nkt - 1) wj = 0.5 * (kt[nkt - 1] - kt[nkt - 2]);
    else wj = 0.5 * (kt[j + 1] - kt[j - 1]);
    contrib[0] = wj * pr * T * T;
    contrib[1] = wj * pr * T * E;
    contrib[2] = wj * pr * E * E;
    // n_s enters only the primordial factor (k/k_pivot)^(n_s-1): d/dn_s = ln(k/k_pivot)
    const double lk = log(k / k_pivot);
    contrib[3] = contrib[0] * lk;
    contrib[4] = contrib[1] * lk;
    contrib[5] = contrib[2] * lk;
  }
  // reduction over the LOS_TX columns (fixed order: deterministic); rows
  // y > 0 have returned, so only named warps of row 0 take part
  __shared__ double red[6][LOS_TX / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int X = 0; X < 6; ++X) {
    double v = contrib[X];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[X][wid] = v;
  }
  asm volatile("bar.sync 1, %0;" ::"r"(LOS_TX));
  if (threadIdx.x < 6) {
    double s = 0.;
    for (int w = 0; w < LOS_TX / 32; ++w) s += red[threadIdx.x][w];
    W.partial[(((int64_t)cz * n_ell + ie) * ntile + tile) * 6 + threadIdx.x] = s;
  }
}

__global__ void cl_final_kernel(int c0, int n_ell_tab, int ntile, BesselDev B, int idx_min, int l_min, int n_out,
                                LosScratch W, double* __restrict__ cl_raw, double* __restrict__ cl,
                                double* __restrict__ dcl_dns) {
  // one block per cosmology of the chunk; scratch: x[n], y[6][n], s[6][n],
  // dinv, mlo, up (n = n_ell_tab); series 3..5 are dC/dn_s
  const int cz = blockIdx.x, ci = c0 + cz;
  const double* partial = W.partial + (int64_t)cz * n_ell_tab * ntile * 6;
  cl_raw += (int64_t)ci * n_ell_tab * 3;
  cl += (int64_t)ci * 3 * n_out;
  if (dcl_dns) dcl_dns += (int64_t)ci * 3 * n_out;
  const int n = n_ell_tab;
  const int nser = dcl_dns ? 6 : 3;
  double* x = W.lscr + (int64_t)cz * 16 * n;
  double* y = x + n;
  double* s = y + 6 * n;
  double* dinv = s + 6 * n;
  double* mlo = dinv + n;
  double* up = mlo + n;
  for (int i = threadIdx.x; i < n * nser; i += blockDim.x) {
    int ie = i / nser, X = i % nser;
    double acc = 0.;
    for (int t = 0; t < ntile; ++t) acc += partial[((int64_t)ie * ntile + t) * 6 + X];
    if (X < 3) cl_raw[ie * 3 + X] = acc;
    y[X * n + ie] = acc;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (double)B.l_tab[idx_min + i];
  __syncthreads();
  if (threadIdx.x == 0) nak_factor(x, n, dinv, mlo, up);
  __syncthreads();
  if (threadIdx.x < nser) nak_solve(x, y + threadIdx.x * n, n, dinv, mlo, up, s + threadIdx.x * n);
  __syncthreads();
  for (int i = threadIdx.x; i < nser * n_out; i += blockDim.x) {
    int X = i / n_out, o = i % n_out;
    double xq = (double)(l_min + o);
    int iv = spline_interval(x, n, xq);
    double v = spline_piece(y[X * n + iv], y[X * n + iv + 1], s[X * n + iv], s[X * n + iv + 1],
                            x[iv + 1] - x[iv], xq - x[iv]);
    if (X < 3) cl[(int64_t)X * n_out + o] = v;
    else dcl_dns[(int64_t)(X - 3) * n_out + o] = v;
  }
}

// The l spline of cl_final_kernel on C_l already summed at the tabulated l
// (cl_raw [n_cosmo][n_ell_tab][3]): one block per cosmology, scratch in
// dynamic shared memory (13 n_ell_tab doubles).  Same operations as
// cl_final_kernel, so the results are identical to the single-call path.
__global__ void cl_spline_kernel(const double* __restrict__ cl_raw, int n_ell_tab, BesselDev B, int idx_min,
                                 int l_min, int n_out, double* __restrict__ cl) {
  extern __shared__ double sp[];
  const int ci = blockIdx.x;
  const int n = n_ell_tab;
  double* x = sp;
  double* y = x + n;
  double* s = y + 3 * n;
  double* dinv = s + 3 * n;
  double* mlo = dinv + n;
  double* up = mlo + n;
  const double* raw = cl_raw + (int64_t)ci * n * 3;
  for (int i = threadIdx.x; i < n * 3; i += blockDim.x) y[(i % 3) * n + i / 3] = raw[i];
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (double)B.l_tab[idx_min + i];
  __syncthreads();
  if (threadIdx.x == 0) nak_factor(x, n, dinv, mlo, up);
  __syncthreads();
  if (threadIdx.x < 3) nak_solve(x, y + threadIdx.x * n, n, dinv, mlo, up, s + threadIdx.x * n);
  __syncthreads();
  double* out = cl + (int64_t)ci * 3 * n_out;
  for (int i = threadIdx.x; i < 3 * n_out; i += blockDim.x) {
    const int X = i / n_out, o = i % n_out;
    const double xq = (double)(l_min + o);
    const int iv = spline_interval(x, n, xq);
    out[(int64_t)X * n_out + o] = spline_piece(y[X * n + iv], y[X * n + iv + 1], s[X * n + iv], s[X * n + iv + 1],
                                               x[iv + 1] - x[iv], xq - x[iv]);
  }
}

// jnp.interp(x, xp, fp) for increasing xp
__device__ double np_interp(double x, const double* xp, const double* fp, int n, int stride) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (xp[mid] <= x) lo = mid + 1; else hi = mid;
  }
  int i = min(max(lo, 1), n - 1);
  double df = fp[(int64_t)i * stride] - fp[(int64_t)(i - 1) * stride];
  double dx = xp[i] - xp[i - 1];
  double delta = x - xp[i - 1];
  double f = (fabs(dx) <= 2.220446049250313e-16) ? fp[(int64_t)(i - 1) * stride]
                                                  : fp[(int64_t)(i - 1) * stride] + (delta / dx) * df;
  if (x < xp[0]) f = fp[0];
  if (x > xp[n - 1]) f = fp[(int64_t)(n - 1) * stride];
  return f;
}

__global__ void pk_lin_kernel(const abcmb_cosmo* __restrict__ cosmo, const double* __restrict__ kbuf,
                              const double* __restrict__ pt, int n_save, double k_pivot, int n_kout,
                              const double* __restrict__ kout, int n_z, const double* __restrict__ z,
                              double* __restrict__ pk, double* __restrict__ lna_scratch) {
  // one block per (cosmology, z); lna grid in shared memory
  extern __shared__ double slna[];
  const int ci = blockIdx.x, iz = blockIdx.y;
  const abcmb_cosmo& c = cosmo[ci];
  for (int i = threadIdx.x; i < n_save; i += blockDim.x)
    slna[i] = linspace_at(c.lna_transfer_start, 0., n_save, i);
  __syncthreads();
  const double lna = -log(1. + z[iz]);
  const double* dm = pt + c.off_pt + (int64_t)ABCMB_F_DELTA_M * n_save * c.nk;
  const double* kp = kbuf + c.off_k;
  const int nk = c.nk;
  for (int j = threadIdx.x; j < n_kout; j += blockDim.x) {
    double k = kout[j];
    // jnp.interp(k, PT.k, delta_m_lna) needs delta_m_lna at the two bracketing k
    int lo = 0, hi = nk;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (kp[mid] <= k) lo = mid + 1; else hi = mid;
    }
    int i = min(max(lo, 1), nk - 1);
    double d0 = np_interp(lna, slna, dm + (i - 1), n_save, nk);
    double d1 = np_interp(lna, slna, dm + i, n_save, nk);
    double dx = kp[i] - kp[i - 1];
    double d = (fabs(dx) <= 2.220446049250313e-16) ? d0 : d0 + ((k - kp[i - 1]) / dx) * (d1 - d0);
    if (k < kp[0]) d = np_interp(lna, slna, dm, n_save, nk);
    if (k > kp[nk - 1]) d = np_interp(lna, slna, dm + (nk - 1), n_save, nk);
    double prim = c.A_s * pow(k / k_pivot, c.n_s - 1.) * (2 * PI * PI / (k * k * k));
    pk[((int64_t)ci * n_z + iz) * n_kout + j] = d * d * prim;
  }
  (void)lna_scratch;
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// adjoint (vector-Jacobian product) of the line of sight
// ---------------------------------------------------------------------------
// d piece / d(y0, y1, s0, s1) of spline_piece at offset u in an interval dx
struct PieceGrad {
  double y0, y1, s0, s1;
};
__device__ __forceinline__ PieceGrad piece_grad(double dx, double u) {
  const double idx = 1.0 / dx;
  const double u2 = u * u, u3 = u2 * u;
  const double dsl = -2. * u3 * idx * idx + 3. * u2 * idx;   // d piece / d slope (y1 - y0) / dx
  PieceGrad g;
  g.y1 = dsl * idx;
  g.y0 = 1. - g.y1;
  g.s0 = u3 * idx * idx - 2. * u2 * idx + u;
  g.s1 = u3 * idx * idx - u2 * idx;
  return g;
}

// ybar += R^T z, R the not-a-knot right-hand side operator of nak_rhs
__device__ void nak_rhs_adjoint(const double* x, int n, const double* z, double* ybar, int64_t ystride) {
  for (int i = 0; i < n; ++i) {
    const double zi = z[i];
    if (i == 0) {
      const double dx0 = x[1] - x[0], dx1 = x[2] - x[1], d = x[2] - x[0];
      const double c0 = zi * (dx0 + 2. * d) * dx1 / d / dx0;   // via s0 = (y1 - y0) / dx0
      const double c1 = zi * dx0 * dx0 / d / dx1;              // via s1 = (y2 - y1) / dx1
      ybar[0] -= c0;
      ybar[ystride] += c0 - c1;
      ybar[2 * ystride] += c1;
    } else if (i == n - 1) {
      const double dxa = x[n - 2] - x[n - 3], dxb = x[n - 1] - x[n - 2], d = x[n - 1] - x[n - 3];
      const double ca = zi * dxb * dxb / d / dxa;
      const double cb = zi * (2. * d + dxb) * dxa / d / dxb;
      ybar[(int64_t)(n - 3) * ystride] -= ca;
      ybar[(int64_t)(n - 2) * ystride] += ca - cb;
      ybar[(int64_t)(n - 1) * ystride] += cb;
    } else {
      const double dxm = x[i] - x[i - 1], dxp = x[i + 1] - x[i];
      const double cm = zi * 3. * dxp / dxm, cp = zi * 3. * dxm / dxp;
      ybar[(int64_t)(i - 1) * ystride] -= cm;
      ybar[(int64_t)i * ystride] += cm - cp;
      ybar[(int64_t)(i + 1) * ystride] += cp;
    }
  }
}

// z = T^{-T} sbar in place, T = L U the factorisation of nak_factor
// (L unit lower with sub-diagonal mlo, U upper with diagonal 1/dinv and
// super-diagonal up): U^T w = sbar forward, then L^T z = w backward.
__device__ void nak_solve_transposed(int n, const double* dinv, const double* mlo, const double* up, double* v,
                                     int64_t vstride) {
  double wprev = 0.;
  for (int i = 0; i < n; ++i) {
    const double w = (v[(int64_t)i * vstride] - (i > 0 ? up[i - 1] * wprev : 0.)) * dinv[i];
    v[(int64_t)i * vstride] = w;
    wprev = w;
  }
  double znext = v[(int64_t)(n - 1) * vstride];
  for (int i = n - 2; i >= 0; --i) {
    znext = v[(int64_t)i * vstride] - mlo[i + 1] * znext;
    v[(int64_t)i * vstride] = znext;
  }
}

// C_l cotangent at the integer ells -> at the tabulated l (transposed l
// spline), and the A_s / n_s cotangents.  One block, three threads.
__global__ void cl_spline_adjoint_kernel(int ci, int n_ell_tab, int ntile, BesselDev B, int idx_min, int l_min,
                                         int n_out, const double* __restrict__ cl_bar, const double* __restrict__ cl_raw,
                                         const abcmb_cosmo* __restrict__ cosmo, LosScratch W,
                                         double* __restrict__ rbar, double* __restrict__ param_bar) {
  const int n = n_ell_tab;
  double* x = W.lscr;
  double* dinv = x + n;
  double* mlo = dinv + n;
  double* up = mlo + n;
  double* sb = up + n;                      // 3 n
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (double)B.l_tab[idx_min + i];
  __syncthreads();
  if (threadIdx.x == 0) nak_factor(x, n, dinv, mlo, up);
  __syncthreads();
  if (threadIdx.x < 3) {
    const int X = threadIdx.x;
    double* yb = rbar + X;                  // rbar [n][3]
    double* s = sb + X * n;
    for (int i = 0; i < n; ++i) {
      yb[(int64_t)i * 3] = 0.;
      s[i] = 0.;
    }
    const double* cb = cl_bar + (int64_t)ci * 3 * n_out + (int64_t)X * n_out;
    for (int o = 0; o < n_out; ++o) {
      const double xq = (double)(l_min + o);
      const int iv = spline_interval(x, n, xq);
      const PieceGrad g = piece_grad(x[iv + 1] - x[iv], xq - x[iv]);
      const double c = cb[o];
      yb[(int64_t)iv * 3] += c * g.y0;
      yb[(int64_t)(iv + 1) * 3] += c * g.y1;
      s[iv] += c * g.s0;
      s[iv + 1] += c * g.s1;
    }
    nak_solve_transposed(n, dinv, mlo, up, s, 1);
    nak_rhs_adjoint(x, n, s, yb, 3);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // C_raw is linear in A_s; dC_raw/dn_s is the ln(k/k_pivot)-weighted quadrature (series 3..5)
    const double* raw = cl_raw + (int64_t)ci * n * 3;
    double as = 0., ns = 0.;
    for (int ie = 0; ie < n; ++ie) {
      for (int X = 0; X < 3; ++X) {
        double d = 0.;
        for (int t = 0; t < ntile; ++t) d += W.partial[((int64_t)ie * ntile + t) * 6 + 3 + X];
        as += rbar[ie * 3 + X] * raw[ie * 3 + X];
        ns += rbar[ie * 3 + X] * d;
      }
    }
    param_bar[2 * ci] = as / cosmo[ci].A_s;
    param_bar[2 * ci + 1] = ns;
  }
}

// T, E (stored by los_kernel) -> their cotangents in place:
// Tbar = w_k pr_k (2 Cbar_TT T + Cbar_TE E), Ebar = w_k pr_k (Cbar_TE T + 2 Cbar_EE E)
__global__ void te_adjoint_kernel(const abcmb_cosmo* __restrict__ cosmo, int ci, int n_ell, const double* __restrict__ kt,
                                  int nkt, double k_pivot, const double* __restrict__ rbar, double* __restrict__ te) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int ie = blockIdx.y;
  if (j >= nkt) return;
  const abcmb_cosmo& c = cosmo[ci];
  const double k = kt[j];
  const double pr = 4. * PI * c.A_s * pow(k / k_pivot, c.n_s - 1.) / k;
  double wj;
  if (nkt == 1) wj = 0.;
  else if (j == 0) wj = 0.5 * (kt[1] - kt[0]);
  else if (j == nkt - 1) wj = 0.5 * (kt[nkt - 1] - kt[nkt - 2]);
  else wj = 0.5 * (kt[j + 1] - kt[j - 1]);
  const double f = wj * pr;
  double* t = te + ((int64_t)ie * 2) * nkt;
  const double T = t[j], E = t[nkt + j];
  const double btt = rbar[ie * 3], bte = rbar[ie * 3 + 1], bee = rbar[ie * 3 + 2];
  t[j] = f * (2. * btt * T + bte * E);
  t[nkt + j] = f * (bte * T + 2. * bee * E);
}

// Source cotangents: Sbar_X(i, k) = sum_l Xbar(l, k) w_i / aH_i phi_X(l, k chi_i)
// (the line-of-sight sum taken over l instead of lna).  Thread per transfer
// k, ADJ_TAU lna points per block; the Bessel columns are read through L1.
constexpr int ADJ_TAU = 8;
__global__ void __launch_bounds__(128) los_adjoint_kernel(const abcmb_cosmo* __restrict__ cosmo, int ci,
                                                          const double* __restrict__ tables, int nl, int n_save,
                                                          const double* __restrict__ kt, int nkt, BesselDev B,
                                                          int idx_min, int n_ell, const double* __restrict__ te,
                                                          double* __restrict__ sbar) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * ADJ_TAU;
  if (j >= nkt) return;
  const abcmb_cosmo& c = cosmo[ci];
  const double* los = tables + c.off_los;
  const double lts = c.lna_transfer_start;
  const double delta_lna = linspace_at(lts, 0., n_save, n_save - 1) - linspace_at(lts, 0., n_save, n_save - 2);
  double dt[ADJ_TAU], idt[ADJ_TAU], wa[ADJ_TAU];
#pragma unroll
  for (int u = 0; u < ADJ_TAU; ++u) {
    const int i = min(i0 + u, nl - 1);
    dt[u] = c.tau0 - los[i];
    idt[u] = 1.0 / dt[u];
    wa[u] = (i0 + u < nl) ? ((i == 0) ? 0.5 * delta_lna : delta_lna) * (1.0 / los[3 * nl + i]) : 0.;
  }
  const double k = kt[j], invk = 1.0 / k;
  const int nx = B.n_x;
  double a0[ADJ_TAU], a1[ADJ_TAU], a2[ADJ_TAU], aE[ADJ_TAU];
#pragma unroll
  for (int u = 0; u < ADJ_TAU; ++u) a0[u] = a1[u] = a2[u] = aE[u] = 0.;
  for (int ie = 0; ie < n_ell; ++ie) {
    const int idx = idx_min + ie;
    const double Tb = te[((int64_t)ie * 2) * nkt + j], Eb = te[((int64_t)ie * 2 + 1) * nkt + j];
    const double l = (double)B.l_tab[idx];
    const double x0min = B.xmin[idx], x0max = B.xmax[idx];
    const double x1min = B.xmin[B.n_l + idx], x1max = B.xmax[B.n_l + idx];
    const double x2min = B.xmin[2 * B.n_l + idx], x2max = B.xmax[2 * B.n_l + idx];
    const double s0 = (double)(nx - 1) / (x0max - x0min);
    const double s1 = (double)(nx - 1) / (x1max - x1min);
    const double s2 = (double)(nx - 1) / (x2max - x2min);
    const double* ph0 = B.phi + ((int64_t)0 * B.n_l + idx) * nx;
    const double* ph1 = B.phi + ((int64_t)1 * B.n_l + idx) * nx;
    const double* ph2 = B.phi + ((int64_t)2 * B.n_l + idx) * nx;
    const double ef = sqrt(3. / 8. * (l + 2) * (l + 1) * l * (l - 1));
    const double nu0 = l + 0.5, nu1 = l + 1.5, nu0sq = nu0 * nu0, nu1sq = nu1 * nu1;
    const double c2 = 3 * l * (l - 1);
#pragma unroll
    for (int u = 0; u < ADJ_TAU; ++u) {
      const double chi = dt[u] * k;
      const double ichi = idt[u] * invk;
      double p0;
      if (chi < x0min) p0 = 0.;
      else if (chi >= x0max) p0 = jasym(nu0, nu0sq, chi, ichi);
      else p0 = lerp_tab(chi, x0min, s0, ph0, nx);
      const bool as1 = chi >= x1max, as2 = chi >= x2max;
      double jl = 0., jl1 = 0.;
      if (as1 || as2) {
        jl = (chi >= x0max) ? p0 : jasym(nu0, nu0sq, chi, ichi);
        jl1 = jasym(nu1, nu1sq, chi, ichi);
      }
      double p1, p2;
      if (chi < x1min) p1 = 0.;
      else if (as1) p1 = l * ichi * jl - jl1;
      else p1 = lerp_tab(chi, x1min, s1, ph1, nx);
      const double ichi2 = ichi * ichi;
      if (chi < x2min) p2 = 0.;
      else if (as2) p2 = ((c2 - 2 * chi * chi) * jl + 6 * chi * jl1) * 0.5 * ichi2;
      else p2 = lerp_tab(chi, x2min, s2, ph2, nx);
      const double eps = p0 * ichi2 * ef;
      const double tw = Tb * wa[u], ew = Eb * wa[u];
      a0[u] = fma(tw, p0, a0[u]);
      a1[u] = fma(tw, p1, a1[u]);
      a2[u] = fma(tw, p2, a2[u]);
      aE[u] = fma(ew, eps, aE[u]);
    }
  }
  const int64_t plane = (int64_t)nl * nkt;
#pragma unroll
  for (int u = 0; u < ADJ_TAU; ++u) {
    if (i0 + u < nl) {
      const int64_t o = (int64_t)(i0 + u) * nkt + j;
      sbar[o] = a0[u];
      sbar[plane + o] = a1[u];
      sbar[2 * plane + o] = a2[u];
      sbar[3 * plane + o] = aE[u];
    }
  }
}

// PT cotangent of one (source field, lna row) column: the transposed source
// combination (sources_kernel) and the transposed k spline (spline_slopes /
// spline_piece), accumulated in a fixed order.
__global__ void spline_adjoint_kernel(const abcmb_cosmo* __restrict__ cosmo, int ci, const double* __restrict__ tables,
                                      int n_save, int nl, const double* __restrict__ kt, int nkt,
                                      abcmb_los_settings ls, LosScratch W, const double* __restrict__ sbar,
                                      double* __restrict__ pt_bar) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;    // f * nl + il
  if (col >= NSRC_FIELDS * nl) return;
  const abcmb_cosmo& c = cosmo[ci];
  const int nk = c.nk;
  const int f = col / nl, il = col % nl;
  const double* los = tables + c.off_los;
  const double g = los[1 * nl + il], gp = los[2 * nl + il], aH = los[3 * nl + il];
  const double em = los[4 * nl + il], aHd = los[5 * nl + il];
  const double* xk = W.xk;
  double* yb = pt_bar + c.off_pt + ((int64_t)SRC_FIELDS[f] * n_save + il) * nk;
  double* s = W.slopes + (int64_t)col * W.max_nk;
  for (int m = 0; m < nk; ++m) {
    yb[m] = 0.;
    s[m] = 0.;
  }
  const int64_t plane = (int64_t)nl * nkt;
  for (int j = 0; j < nkt; ++j) {
    const double k = kt[j];
    const int64_t o = (int64_t)il * nkt + j;
    const double b0 = sbar[o], b1 = sbar[plane + o], b2 = sbar[2 * plane + o], bE = sbar[3 * plane + o];
    // d(sT0, sT1, sT2, sE) / d field f (sources_kernel)
    double fb;
    switch (f) {
      case 0: fb = b0 * (ls.scale_sw * g / 4.); break;                                          // delta_g
      case 1: fb = b0 * (ls.scale_dop * aH * gp / (k * k)); break;                              // theta_b
      case 2: fb = b0 * (ls.scale_dop * aH * g / (k * k)); break;                               // theta_b'
      case 3: fb = b2 * (ls.scale_pol * g * 2. / 8.) + bE * (sqrt(6.) * g * 2. / 8.); break;    // sigma_g
      case 4:
      case 5: fb = b2 * (ls.scale_pol * g / 8.) + bE * (sqrt(6.) * g / 8.); break;              // G0, G2
      case 6: fb = b0 * (ls.scale_isw * g) - b1 * (ls.scale_isw * em * k); break;               // eta
      case 7: fb = b0 * (ls.scale_isw * 2. * em * aH); break;                                   // eta'
      case 8:                                                                                   // alpha
        fb = b0 * (-ls.scale_isw * 2. * g * aH - ls.scale_isw * 2. * em * aHd + ls.scale_dop * aH * gp) +
             b1 * (ls.scale_isw * em * 2. * aH * k);
        break;
      default:                                                                                  // alpha'
        fb = b0 * (ls.scale_sw * g * aH - ls.scale_isw * g * aH - ls.scale_isw * 2. * em * aH * aH +
                   ls.scale_dop * aH * g) +
             b1 * (ls.scale_isw * em * aH * k);
        break;
    }
    const int m = W.kidx[j];
    const PieceGrad pg = piece_grad(xk[m + 1] - xk[m], log10(k) - xk[m]);
    yb[m] += fb * pg.y0;
    yb[m + 1] += fb * pg.y1;
    s[m] += fb * pg.s0;
    s[m + 1] += fb * pg.s1;
  }
  nak_solve_transposed(nk, W.dinv, W.mlo, W.up, s, 1);
  nak_rhs_adjoint(xk, nk, s, yb, 1);
}

static int64_t al256(int64_t b) { return (b + 255) / 256 * 256; }

struct LosLayout {
  int chunk, max_nk, nkt, n_ell_tab, nl, ntile;
  int64_t o_xk, o_dinv, o_mlo, o_up, o_kidx, o_slopes, o_S, o_partial, o_lscr, total;
};

static LosLayout los_layout(int n_cosmo, int max_nk, int nkt, int n_ell_tab, int n_save, int precision) {
  LosLayout L{};
  L.chunk = n_cosmo < LOS_CHUNK ? (n_cosmo > 0 ? n_cosmo : 1) : LOS_CHUNK;
  L.max_nk = max_nk;
  L.nkt = nkt;
  L.n_ell_tab = n_ell_tab;
  L.nl = n_save - 1;
  L.ntile = (nkt + LOS_TX - 1) / LOS_TX;
  const int64_t C = L.chunk;
  int64_t b = 0;
  L.o_xk = b;      b += al256(C * max_nk * 8);
  L.o_dinv = b;    b += al256(C * max_nk * 8);
  L.o_mlo = b;     b += al256(C * max_nk * 8);
  L.o_up = b;      b += al256(C * max_nk * 8);
  L.o_kidx = b;    b += al256(C * nkt * 4);
  L.o_slopes = b;  b += al256(C * NSRC_FIELDS * L.nl * max_nk * 8);
  L.o_S = b;       b += al256(C * 4 * L.nl * nkt * (precision ? 4 : 8));
  L.o_partial = b; b += al256(C * n_ell_tab * L.ntile * 6 * 8);
  L.o_lscr = b;    b += al256(C * 16 * n_ell_tab * 8);
  L.total = b;
  return L;
}

int64_t los_workspace_bytes(int n_cosmo, int max_nk, int nkt, int n_ell_tab, int n_save, int precision) {
  return los_layout(n_cosmo, max_nk, nkt, n_ell_tab, n_save, precision).total;
}

cudaError_t launch_los(int n_cosmo, const abcmb_cosmo* cosmo_dev, const abcmb_cosmo* cosmo_host,
                       const double* tables, const double* kbuf, const double* pt, const double* kt,
                       const abcmb_los_settings& ls, int n_save, const BesselDev& B, double* cl_raw,
                       double* cl, double* dcl_dns, void* ws, cudaStream_t stream) {
  const int nkt = ls.nkt;
  const int n_ell_tab = ls.idx_max - ls.idx_min + 1;
  const int n_out = ls.l_max - ls.l_min + 1;
  int max_nk = 0;
  for (int c = 0; c < n_cosmo; ++c) max_nk = cosmo_host[c].nk > max_nk ? cosmo_host[c].nk : max_nk;
  const LosLayout L = los_layout(n_cosmo, max_nk, nkt, n_ell_tab, n_save, ls.precision);
  const int nl = L.nl;
  char* w = static_cast<char*>(ws);
  LosScratch W;
  W.xk = reinterpret_cast<double*>(w + L.o_xk);
  W.dinv = reinterpret_cast<double*>(w + L.o_dinv);
  W.mlo = reinterpret_cast<double*>(w + L.o_mlo);
  W.up = reinterpret_cast<double*>(w + L.o_up);
  W.kidx = reinterpret_cast<int*>(w + L.o_kidx);
  W.slopes = reinterpret_cast<double*>(w + L.o_slopes);
  W.S = w + L.o_S;
  W.partial = reinterpret_cast<double*>(w + L.o_partial);
  W.lscr = reinterpret_cast<double*>(w + L.o_lscr);
  W.te = nullptr;
  W.max_nk = max_nk;
  const size_t smem = (size_t)(3 * B.n_x + 3 * nl + (LOS_TY - 1) * 4 * LOS_TX) * sizeof(double);
  cudaError_t e;
  if (ls.precision == 0) {
    e = cudaFuncSetAttribute(los_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  } else {
    e = cudaFuncSetAttribute(los_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  if (e != cudaSuccess) return e;
  for (int c0 = 0; c0 < n_cosmo; c0 += L.chunk) {
    const int nc = (n_cosmo - c0) < L.chunk ? (n_cosmo - c0) : L.chunk;
    spline_prep_kernel<<<nc, 256, 0, stream>>>(cosmo_dev, c0, kbuf, kt, nkt, W);
    spline_slopes_kernel<<<dim3((NSRC_FIELDS * nl + 127) / 128, nc), 128, 0, stream>>>(cosmo_dev, c0, pt, n_save, nl, W);
    dim3 gs((nkt + 127) / 128, nl, nc);
    if (ls.precision == 0)
      sources_kernel<double><<<gs, 128, 0, stream>>>(cosmo_dev, c0, tables, pt, n_save, nl, kt, nkt, ls, W);
    else
      sources_kernel<float><<<gs, 128, 0, stream>>>(cosmo_dev, c0, tables, pt, n_save, nl, kt, nkt, ls, W);
    dim3 gl(n_ell_tab, L.ntile, nc);
    dim3 bl(LOS_TX, LOS_TY);
    if (ls.precision == 0)
      los_kernel<0><<<gl, bl, smem, stream>>>(cosmo_dev, c0, tables, nl, n_save, kt, nkt, B, ls.idx_min, ls.k_pivot, W);
    else
      los_kernel<1><<<gl, bl, smem, stream>>>(cosmo_dev, c0, tables, nl, n_save, kt, nkt, B, ls.idx_min, ls.k_pivot, W);
    cl_final_kernel<<<nc, 256, 0, stream>>>(c0, n_ell_tab, L.ntile, B, ls.idx_min, ls.l_min, n_out, W, cl_raw, cl,
                                            dcl_dns);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

struct LosVjpLayout {
  LosLayout f;
  int n_out;
  int64_t o_te, o_raw, o_cl, o_rbar, total;
};

static LosVjpLayout los_vjp_layout(int n_cosmo, int max_nk, int nkt, int n_ell_tab, int n_save, int n_out) {
  LosVjpLayout L{};
  L.f = los_layout(1, max_nk, nkt, n_ell_tab, n_save, 0);
  L.n_out = n_out;
  int64_t b = L.f.total;
  L.o_te = b;   b += al256((int64_t)n_ell_tab * 2 * nkt * 8);
  L.o_raw = b;  b += al256((int64_t)n_cosmo * n_ell_tab * 3 * 8);
  L.o_cl = b;   b += al256((int64_t)n_cosmo * 3 * n_out * 8);
  L.o_rbar = b; b += al256((int64_t)n_ell_tab * 3 * 8);
  L.total = b;
  return L;
}

int64_t los_vjp_workspace_bytes(int n_cosmo, int max_nk, int nkt, int n_ell_tab, int n_save, int n_out) {
  return los_vjp_layout(n_cosmo, max_nk, nkt, n_ell_tab, n_save, n_out).total;
}

// Vector-Jacobian product of launch_los (FP64), one cosmology after another:
// the forward pieces again (storing T and E), then the adjoint kernels.
cudaError_t launch_los_vjp(int n_cosmo, const abcmb_cosmo* cosmo_dev, const abcmb_cosmo* cosmo_host,
                           const double* tables, const double* kbuf, const double* pt, const double* kt,
                           const abcmb_los_settings& ls, int n_save, const BesselDev& B, const double* cl_bar,
                           double* pt_bar, double* param_bar, void* ws, cudaStream_t stream) {
  const int nkt = ls.nkt;
  const int n_ell_tab = ls.idx_max - ls.idx_min + 1;
  const int n_out = ls.l_max - ls.l_min + 1;
  int max_nk = 0;
  for (int c = 0; c < n_cosmo; ++c) max_nk = cosmo_host[c].nk > max_nk ? cosmo_host[c].nk : max_nk;
  const LosVjpLayout L = los_vjp_layout(n_cosmo, max_nk, nkt, n_ell_tab, n_save, n_out);
  const int nl = L.f.nl;
  char* w = static_cast<char*>(ws);
  LosScratch W;
  W.xk = reinterpret_cast<double*>(w + L.f.o_xk);
  W.dinv = reinterpret_cast<double*>(w + L.f.o_dinv);
  W.mlo = reinterpret_cast<double*>(w + L.f.o_mlo);
  W.up = reinterpret_cast<double*>(w + L.f.o_up);
  W.kidx = reinterpret_cast<int*>(w + L.f.o_kidx);
  W.slopes = reinterpret_cast<double*>(w + L.f.o_slopes);
  W.S = w + L.f.o_S;
  W.partial = reinterpret_cast<double*>(w + L.f.o_partial);
  W.lscr = reinterpret_cast<double*>(w + L.f.o_lscr);
  W.te = reinterpret_cast<double*>(w + L.o_te);
  W.max_nk = max_nk;
  double* raw = reinterpret_cast<double*>(w + L.o_raw);
  double* clf = reinterpret_cast<double*>(w + L.o_cl);
  double* rbar = reinterpret_cast<double*>(w + L.o_rbar);
  const size_t smem = (size_t)(3 * B.n_x + 3 * nl + (LOS_TY - 1) * 4 * LOS_TX) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(los_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  for (int ci = 0; ci < n_cosmo; ++ci) {
    const abcmb_cosmo& ch = cosmo_host[ci];
    e = cudaMemsetAsync(pt_bar + ch.off_pt, 0, (size_t)ABCMB_NFIELDS * n_save * ch.nk * sizeof(double), stream);
    if (e != cudaSuccess) return e;
    // forward, one cosmology (chunk of one: scratch index 0)
    spline_prep_kernel<<<1, 256, 0, stream>>>(cosmo_dev, ci, kbuf, kt, nkt, W);
    spline_slopes_kernel<<<dim3((NSRC_FIELDS * nl + 127) / 128, 1), 128, 0, stream>>>(cosmo_dev, ci, pt, n_save, nl, W);
    sources_kernel<double><<<dim3((nkt + 127) / 128, nl, 1), 128, 0, stream>>>(cosmo_dev, ci, tables, pt, n_save, nl,
                                                                              kt, nkt, ls, W);
    los_kernel<0><<<dim3(n_ell_tab, L.f.ntile, 1), dim3(LOS_TX, LOS_TY), smem, stream>>>(
        cosmo_dev, ci, tables, nl, n_save, kt, nkt, B, ls.idx_min, ls.k_pivot, W);
    cl_final_kernel<<<1, 256, 0, stream>>>(ci, n_ell_tab, L.f.ntile, B, ls.idx_min, ls.l_min, n_out, W, raw, clf,
                                           nullptr);
    // adjoint
    cl_spline_adjoint_kernel<<<1, 32, 0, stream>>>(ci, n_ell_tab, L.f.ntile, B, ls.idx_min, ls.l_min, n_out, cl_bar,
                                                   raw, cosmo_dev, W, rbar, param_bar);
    te_adjoint_kernel<<<dim3((nkt + 127) / 128, n_ell_tab), 128, 0, stream>>>(cosmo_dev, ci, n_ell_tab, kt, nkt,
                                                                               ls.k_pivot, rbar, W.te);
    double* sbar = static_cast<double*>(W.S);
    los_adjoint_kernel<<<dim3((nkt + 127) / 128, (nl + ADJ_TAU - 1) / ADJ_TAU), 128, 0, stream>>>(
        cosmo_dev, ci, tables, nl, n_save, kt, nkt, B, ls.idx_min, n_ell_tab, W.te, sbar);
    spline_adjoint_kernel<<<(NSRC_FIELDS * nl + 127) / 128, 128, 0, stream>>>(cosmo_dev, ci, tables, n_save, nl, kt,
                                                                               nkt, ls, W, sbar, pt_bar);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_cl_spline(int n_cosmo, const double* cl_raw, int idx_min, int n_ell_tab, int l_min, int l_max,
                             const BesselDev& B, double* cl, cudaStream_t stream) {
  const size_t smem = (size_t)13 * n_ell_tab * sizeof(double);
  cl_spline_kernel<<<n_cosmo, 256, smem, stream>>>(cl_raw, n_ell_tab, B, idx_min, l_min, l_max - l_min + 1, cl);
  return cudaGetLastError();
}

cudaError_t launch_pk_lin(int n_cosmo, const abcmb_cosmo* cosmo, const double* kbuf, const double* pt,
                          int n_save, double k_pivot, int n_kout, const double* kout, int n_z, const double* z,
                          double* pk, cudaStream_t stream) {
  dim3 g(n_cosmo, n_z);
  pk_lin_kernel<<<g, 256, n_save * sizeof(double), stream>>>(cosmo, kbuf, pt, n_save, k_pivot, n_kout, kout, n_z,
                                                              z, pk, nullptr);
  return cudaGetLastError();
}

}  // namespace abcmb
