/*
 * abcmb_b200.h -- C ABI of the B200 implementation of ABCMB's hot path:
 * the per-k linear Einstein-Boltzmann hierarchy integration
 * (abcmb/perturbations.py + abcmb/species.py) and the line-of-sight C_l
 * projection (abcmb/spectrum.py).
 *
 * Every entry point takes plain pointers and sizes.  Device pointers are
 * marked "dev"; the caller (XLA, torch, or any CUDA client) owns every
 * buffer.  All calls are stream ordered and return 0 on success or a
 * negative ABCMB_ERR_* code; per-k solver failures are reported through the
 * per-item status array (ABCMB_STATUS_*), mirroring diffrax raising when
 * max_steps is hit (abcmb/perturbations.py:304-312, docs/FAQ.rst:42-47).
 *
 * Data layout shared by every entry point
 * ---------------------------------------
 *  - abcmb_cosmo[n_cosmo]: one descriptor per cosmology (parameters after
 *    Model.add_derived_parameters, abcmb/main.py:368-612; background scalars;
 *    state layout from model_specs.populate_species, abcmb/model_specs.py:84-118;
 *    offsets into the shared table / k / output buffers).
 *  - tables (double): per cosmology the conformal-time table (10000 values on
 *    lna in [-33, 0], abcmb/background.py:59,252-319), the x_e and T_m HyRex
 *    tables with their inf padding already replaced by the last value
 *    (abcmb/background.py:544-550), and the six 1-D line-of-sight arrays on
 *    PT.lna[:-1] (tau, g, dg/dlna, aH, exp(-kappa), d(aH)/dtau;
 *    abcmb/spectrum.py:640-651).
 *  - PT output (double): per cosmology ABCMB_NFIELDS fields x n_save x nk,
 *    field-major, each field laid out [save][k] like the (Nlna, Nk) arrays
 *    of PerturbationTable (abcmb/perturbations.py:406-450).
 */
#ifndef ABCMB_B200_H
#define ABCMB_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ABCMB_B200_VERSION 100   /* 1.0.0 */

/* ---- error codes (return values) ---- */
#define ABCMB_OK                 0
#define ABCMB_ERR_ARG           -1   /* bad argument / unsupported layout   */
#define ABCMB_ERR_CUDA          -2   /* a CUDA runtime call failed          */
#define ABCMB_ERR_WORKSPACE     -3   /* workspace too small                 */
#define ABCMB_ERR_TABLES        -4   /* Bessel tables not uploaded          */
#define ABCMB_ERR_SOLVER        -5   /* at least one item has status != OK  */

/* ---- per-k status codes ---- */
#define ABCMB_STATUS_OK          0
#define ABCMB_STATUS_MAX_STEPS   1   /* diffrax RESULTS.max_steps_reached     */
#define ABCMB_STATUS_NONFINITE   2   /* NaN/Inf in the state or the error     */
#define ABCMB_STATUS_DT_UNDERFLOW 3  /* step size collapsed below 1e-14       */
#define ABCMB_STATUS_BAD_LAYOUT  4   /* descriptor outside the launch's limits
                                        (ny > max_ny, l_max outside 4..63)   */

/* ---- PerturbationTable field indices (abcmb/perturbations.py:393-404) ---- */
enum {
  ABCMB_F_DELTA_M = 0,        /* delta_m                                  */
  ABCMB_F_THETA_B_PRIME,      /* theta_b_prime                            */
  ABCMB_F_ETA,                /* metric_eta                               */
  ABCMB_F_H_PRIME,            /* metric_h_prime                           */
  ABCMB_F_ETA_PRIME,          /* metric_eta_prime                         */
  ABCMB_F_ALPHA,              /* metric_alpha                             */
  ABCMB_F_ALPHA_PRIME,        /* metric_alpha_prime                       */
  ABCMB_F_CDM_DELTA,          /* species_perturbations["ColdDarkMatter"]  */
  ABCMB_F_B_DELTA,            /* ["Baryon"]["delta"]                      */
  ABCMB_F_B_THETA,            /* ["Baryon"]["theta"]                      */
  ABCMB_F_G_DELTA,            /* ["Photon"]["delta"]                      */
  ABCMB_F_G_THETA,            /* ["Photon"]["theta"]                      */
  ABCMB_F_G_SIGMA,            /* ["Photon"]["sigma"]                      */
  ABCMB_F_G_G0,               /* ["Photon"]["G0"]                         */
  ABCMB_F_G_G2,               /* ["Photon"]["G2"]                         */
  ABCMB_F_NU_DELTA,           /* ["MasslessNeutrino"]["delta"]            */
  ABCMB_F_NU_THETA,           /* ["MasslessNeutrino"]["theta"]            */
  ABCMB_F_NU_SIGMA,           /* ["MasslessNeutrino"]["sigma"]            */
  ABCMB_F_NCDM_DELTA,         /* ["MassiveNeutrino"]["delta"] (0 if absent) */
  ABCMB_F_NCDM_THETA,         /* ["MassiveNeutrino"]["theta"]             */
  ABCMB_F_NCDM_SIGMA,         /* ["MassiveNeutrino"]["sigma"]             */
  ABCMB_NFIELDS
};

/* Fixed background grids of the reference. */
#define ABCMB_NTAU_TAB   10000    /* lna_tau_tab = linspace(-33, 0, 10000)  */
#define ABCMB_LNA_TAU_MIN (-33.0)
#define ABCMB_LNA_TAU_MAX (0.0)
#define ABCMB_NLOS_ARR   6        /* tau, g, g', aH, exp(-kappa), aH_dot    */

/*
 * One cosmology.  Parameters are the derived dict of
 * Model.add_derived_parameters (abcmb/main.py:368-612); background scalars
 * are fields of abcmb.background.Background.
 */
typedef struct abcmb_cosmo {
  /* parameters */
  double h, omega_b, omega_cdm, omega_Lambda, A_s, n_s, TCMB0, YHe;
  double N_nu_massless, T_nu_massless, N_nu_massive, T_nu_massive, m_nu_massive;
  double R_nu, R_b, om;
  /* background scalars */
  double tau0;                /* BG.tau0 = BG.tau(0.)                        */
  double lna_transfer_start;  /* BG.lna_transfer_start                        */
  /* x_e table: fast_interp(lna, lna_xe0, lna_xe0 + n_xe*dx, xe) with n_xe the
   * padded length (abcmb/background.py:593-603) */
  double lna_xe0, lna_xe_max, lna_xe_last, xe_first, xe_last;
  /* T_m table (abcmb/background.py:647-657) */
  double lna_tm0, lna_tm_max, lna_tm_last, tm_last;
  /* offsets (in doubles) into the shared table buffer */
  int64_t off_tau;            /* ABCMB_NTAU_TAB values                        */
  int64_t off_xe;             /* n_xe values                                  */
  int64_t off_tm;             /* n_tm values                                  */
  int64_t off_los;            /* ABCMB_NLOS_ARR x (n_save-1) values           */
  /* offsets into the k buffer and the PT output buffer (doubles) */
  int64_t off_k;              /* nk perturbation wavenumbers, increasing      */
  int64_t off_pt;             /* ABCMB_NFIELDS x n_save x nk                  */
  int32_t n_xe, n_tm;
  /* state layout: y = [eta | d_cdm | d_b, th_b | F_0..F_lg | G_0..G_lp |
   *                    N_0..N_lnu | (Psi_0..Psi_lm) x 3 bins]            */
  int32_t lmax_g, lmax_pol_g, lmax_nu, lmax_ncdm, has_ncdm, ny;
  int32_t nk;
  int32_t pad_;
} abcmb_cosmo;

/* Perturbation solver settings (specs dict, abcmb/model_specs.py:55-69). */
typedef struct abcmb_pert_settings {
  double R_tc, R_large;             /* start-time thresholds              */
  double k_split;                   /* k_split_PE                         */
  double rtol_small, rtol_large;    /* rtol_{small,large}_k_PE            */
  double atol_small, atol_large;    /* atol_{small,large}_k_PE            */
  double pcoeff, icoeff, dcoeff;    /* PIDController coefficients         */
  double dt0;                       /* first step (perturbations.py:306)  */
  int32_t max_steps;                /* max_steps_PE                       */
  int32_t n_save;                   /* 500 save points                    */
  int32_t max_ny;                   /* largest state size in the batch    */
  int32_t any_ncdm;                 /* 1 if any cosmology has massive nu  */
} abcmb_pert_settings;

/* Per-k solver statistics. */
typedef struct abcmb_kstat {
  int32_t status;        /* ABCMB_STATUS_*            */
  int32_t n_accepted;
  int32_t n_rejected;
  int32_t n_newton;      /* chord iterations          */
  double lna_start;      /* integration start         */
} abcmb_kstat;

/* Line-of-sight / C_l settings (SpectrumSolver, abcmb/spectrum.py:180-248). */
typedef struct abcmb_los_settings {
  double k_pivot;
  double scale_sw, scale_isw, scale_dop, scale_pol;
  int32_t l_min, l_max;          /* output ells = l_min..l_max (l_min == 2)   */
  int32_t idx_min, idx_max;      /* bessel_l_tab indices covered             */
  int32_t nkt;                   /* transfer k grid length                   */
  int32_t precision;             /* 0 = FP64, 1 = FP32 + compensated sums    */
  int32_t n_save;                /* PT save points (500)                     */
  int32_t pad_;
} abcmb_los_settings;

/* ------------------------------------------------------------------------ */
/* Library information                                                      */
/* ------------------------------------------------------------------------ */

/* Version number (ABCMB_B200_VERSION). */
int abcmb_version(void);

/* Human readable message for the last error on the calling thread. */
const char* abcmb_last_error(void);

/* ------------------------------------------------------------------------ */
/* Bessel tables (abcmb/bessel_tab, loaded at import by spectrum.py:20-46). */
/* ------------------------------------------------------------------------ */

/*
 * Upload the tabulated spherical-Bessel functions once per device.  host
 * arrays: l_tab[n_l] (int32), for n = 0,1,2: x range xmin_n[n_l], xmax_n[n_l]
 * (column min/max of xphi<n>.txt) and values phi_n[n_l * n_x] laid out
 * column-major as [l][x] (i.e. the transpose of phi<n>.txt).  Replaces the
 * module-level device_put of spectrum.py:29-46.
 */
int abcmb_upload_bessel(int n_l, int n_x, const int32_t* l_tab,
                        const double* xmin0, const double* xmax0, const double* phi0,
                        const double* xmin1, const double* xmax1, const double* phi1,
                        const double* xmin2, const double* xmax2, const double* phi2);

/* ------------------------------------------------------------------------ */
/* Background tables: Background / BackgroundPreRecomb (background.py)      */
/* ------------------------------------------------------------------------ */

/* Settings of abcmb_bg_forward. */
typedef struct abcmb_bg_settings {
  int32_t n_save;           /* PT save points (500): the line-of-sight arrays
                               are written on linspace(lna_transfer_start, 0,
                               n_save)[:-1] (spectrum.py:638-651)            */
  int32_t max_steps_tau;    /* step attempts of the conformal-time solve
                               (diffeqsolve's default 4096,
                               background.py:285-296)                        */
  int32_t max_steps_kappa;  /* step attempts of the optical-depth solve
                               (the reference passes 2048,
                               background.py:708-719)                        */
  int32_t pad_;
} abcmb_bg_settings;

/* Per-cosmology result of abcmb_bg_forward. */
typedef struct abcmb_bgstat {
  int32_t status;           /* ABCMB_STATUS_* of both solves (MAX_STEPS when
                               either reached its limit, as diffrax raises) */
  int32_t n_steps_tau;      /* step attempts of the conformal-time solve     */
  int32_t n_steps_kappa;    /* step attempts of the optical-depth solve      */
  int32_t n_accepted_kappa;
  double tau0;              /* BG.tau0 = BG.tau(0.) (background.py:89)       */
  double lna_rec;           /* BG.lna_rec (background.py:554-557)            */
  double lna_transfer_start;/* BG.lna_transfer_start (background.py:561-564) */
  double kappa_rec;         /* optical depth at lna_rec                      */
} abcmb_bgstat;

/* Bytes of device workspace abcmb_bg_forward needs (the dense-output nodes
 * of both solves, (max_steps + 1) x 3 doubles each per cosmology, and 32
 * bytes per cosmology for the solves' statuses and counts). */
int64_t abcmb_bg_workspace_size(int n_cosmo, const abcmb_bg_settings* settings);

/*
 * Everything the perturbation and line-of-sight kernels read about the
 * background that the reference derives from the x_e history, for every
 * cosmology of the batch, from the descriptor parameters and the x_e / T_m
 * tables already in tables_dev:
 *  - the conformal-time table (ABCMB_NTAU_TAB values at off_tau): dtau/dlna =
 *    1/aH integrated from lna = -16.1 (analytic radiation-era value before)
 *    to 0 by Kvaerno5 + PIDController(rtol = atol = 1e-8), dt0 = 1e-5, dense
 *    output (BackgroundPreRecomb._tabulate_conformal_time,
 *    background.py:252-319), and tau0 = BG.tau(0.);
 *  - the optical depth: dkappa/dlna = -1/(tau_c aH) from 0 down to -10 by
 *    Kvaerno5 + PIDController(pcoeff 0.4, icoeff 0.3, rtol = atol = 1e-10),
 *    dt0 = -1e-3, dense output (Background._tabulate_optical_depth,
 *    background.py:682-720);
 *  - lna_rec and lna_transfer_start (background.py:554-564);
 *  - the six line-of-sight arrays at off_los: tau, g, dg/dlna (the derivative
 *    of the visibility through the dense optical-depth solution, as jax.grad
 *    takes it), aH, exp(-kappa), d(aH)/dtau (spectrum.py:640-651).
 * Both right-hand sides are independent of the state, so each implicit stage
 * of the very-chord solve settles on f(t_i) at its first iteration; the
 * kernels take f(t_i) directly.
 *   cosmo_dev  [n_cosmo]  in: parameters, x_e / T_m fields and offsets;
 *                         out: tau0 and lna_transfer_start
 *   tables_dev            in: x_e and T_m tables; out: tau table, LOS arrays
 *   stat_dev   [n_cosmo]  per-cosmology status and scalars
 * Replaces: the pre-recombination conformal-time table and the
 * Background.__init__ steps after reionisation (background.py:88-89,
 * 552-564) for the shipped species.
 */
int abcmb_bg_forward(int n_cosmo, abcmb_cosmo* cosmo_dev, double* tables_dev,
                     const abcmb_bg_settings* settings, abcmb_bgstat* stat_dev,
                     void* workspace_dev, int64_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Recombination: HyRex (abcmb/hyrex/hyrex.py recomb_model.get_history)      */
/* ------------------------------------------------------------------------ */

/* Parameters HyRex reads (params dict entries). */
typedef struct abcmb_hyrex_params {
  double YHe, omega_b, omega_cdm, Neff;
} abcmb_hyrex_params;

/*
 * Upload HyRex's tables once per device (host arrays, as the reference's
 * abcmb/hyrex/tabs files hold them): alpha [100 x 40 x 4] (Alpha_inf.dat,
 * recomb_functions.py:11-24), R [100] (R_inf.dat), swift [n_swift x 5]
 * (fit_swift.dat, hydrogen.py:53).  A second upload replaces the first:
 * make it only while no abcmb_hyrex_forward launch is in flight.
 */
int abcmb_upload_hyrex_tables(const double* alpha, const double* R, const double* swift, int n_swift);

/* Lengths of HyRex's padded output arrays for a grid of n_grid points
 * (the buffers the seven phases keep, joined by array_with_padding.concat);
 * returns the number of grid points with z >= 3600, or -1. */
int abcmb_hyrex_sizes(int n_grid, int* n_xe, int* n_tm);

/*
 * RecombInputs of every cosmology on the device (what HyRex reads from the
 * background: Background.TCMB, nH and H, abcmb/background.py:147-166,
 * 349-387, sampled on lna_axis_full, abcmb/hyrex/hyrex.py:16-90, 131):
 *   cosmo_dev [n_cosmo]   descriptors; only the background parameters are
 *                         read (h ... om, has_ncdm): no tables needed
 *   T_dev, nH_dev, H_dev [n_cosmo x n_grid]  T_CMB (eV), n_H (cm^-3), H (1/s)
 *                         at numpy.arange(-log(8001), 0, 5e-4)
 * The inputs of abcmb_hyrex_forward, without the host sampling.
 */
int abcmb_hyrex_inputs(int n_cosmo, int n_grid, const abcmb_cosmo* cosmo_dev, double* T_dev, double* nH_dev,
                       double* H_dev, void* stream);

/*
 * The recombination history of every cosmology (recomb_model.get_history,
 * abcmb/hyrex/hyrex.py:146-206, with helium.py and hydrogen.py):
 *   T_dev, nH_dev, H_dev [n_cosmo x n_grid]  RecombInputs: T_CMB (eV), n_H
 *                    (cm^-3) and H (1/s) on lna_axis_full =
 *                    arange(-log(8001), 0, 5e-4) (hyrex.py:16-90, 131)
 *   params_dev [n_cosmo]
 *   xe_dev, lna_xe_dev [n_cosmo x n_xe], tm_dev, lna_tm_dev [n_cosmo x n_tm]
 *                    the reference's outputs (xe_full, lna_full, Tm, lna_Tm)
 *                    before reionisation, +inf after the last valid entry
 *   info_dev [n_cosmo x 16] int32: valid entries of the seven phases,
 *                    steps of the four ODE phases, joined lengths, status,
 *                    valid x_e entries
 * Replaces: the CPU HyRex run of Model (main.py:220).
 */
int abcmb_hyrex_forward(int n_cosmo, int n_grid, const double* T_dev, const double* nH_dev, const double* H_dev,
                        const abcmb_hyrex_params* params_dev, double* xe_dev, double* lna_xe_dev, double* tm_dev,
                        double* lna_tm_dev, int32_t* info_dev, void* stream);

/* ------------------------------------------------------------------------ */
/* Perturbations: PerturbationEvolver.full_evolution (perturbations.py:75)  */
/* ------------------------------------------------------------------------ */

/*
 * Bytes of device workspace abcmb_pert_forward needs for n_cosmo cosmologies
 * and n_items (cosmology, k) work items.
 */
int64_t abcmb_pert_workspace_size(int n_cosmo, int n_items);

/*
 * Integrate every (cosmology, k) item from its start time to lna = 0 and
 * write the PerturbationTable fields at the n_save points
 * linspace(lna_transfer_start, 0, n_save) of each cosmology.
 *   cosmo_dev   [n_cosmo]            descriptors (device copy)
 *   tables_dev                       shared table buffer
 *   k_dev                            shared k buffer (abcmb_cosmo.off_k)
 *   items_dev   [n_items] int32 x2   (cosmology index, k index) pairs, in the
 *                                    order the persistent queue hands them out
 *   pt_dev                           PT output buffer (abcmb_cosmo.off_pt)
 *   kstat_dev   [n_items]            per-item statistics / status
 *   workspace_dev, workspace_bytes   scratch (abcmb_pert_workspace_size)
 *   stream                           cudaStream_t
 * Replaces: PerturbationEvolver.full_evolution -> evolution_one_k ->
 * diffrax.diffeqsolve (perturbations.py:75-117, 250-316) and
 * make_output_table (perturbations.py:318-404).
 */
int abcmb_pert_forward(int n_cosmo, const abcmb_cosmo* cosmo_dev,
                       const double* tables_dev, const double* k_dev,
                       int n_items, const int32_t* items_dev,
                       const abcmb_pert_settings* settings,
                       double* pt_dev, abcmb_kstat* kstat_dev,
                       void* workspace_dev, int64_t workspace_bytes,
                       void* stream);

/*
 * abcmb_pert_forward with forward-mode sensitivities: the PerturbationTable
 * of a base cosmology and its first-order change along up to
 * ABCMB_MAX_TANGENTS parameter directions, in one integration.  The
 * reference differentiates through the same integration with jax.jacfwd /
 * jax.grad (abcmb/main.py:111 adjoint=diffrax.ForwardMode,
 * abcmb/perturbations.py:285-312, docs/FAQ.rst:24-28); here the tangents
 * ride along the primal's accepted steps.
 *
 * Direction p of base cosmology ci is given by two more descriptors of the
 * batch, the cosmology at theta + eps_p ("plus") and at theta - eps_p
 * ("minus"), each with its own tables and PerturbationTable slot and no
 * work items of its own: dir_dev[(ci * ABCMB_MAX_TANGENTS + p) * 2 + {0, 1}]
 * = (plus, minus) descriptor indices (same state layout and k grid as ci).
 * Because the right-hand side is linear in y and in the background basis,
 * the change of A(lna) along p is the central difference of the background
 * between plus and minus at the base's own times; the tangent u_p of the
 * discrete Kvaerno5 step (step sizes frozen, each implicit stage's tangent
 * solved to the primal's very-chord test with the primal's Newton matrix)
 * starts from the central difference of the initial conditions at the two
 * variants' start times.  Written outputs: the base's table (bit-identical
 * to abcmb_pert_forward's), and each variant's table at its own save times
 * as the fields of y(ts) +- (u_p(ts) + y'(ts) dts_p), dts_p the half
 * difference of the variants' save times, with the variant's background.
 * The line of sight over all descriptors then gives the C_l of every
 * variant, and (C_l(plus) - C_l(minus)) / 2 eps_p the derivative.
 *   items_dev   [n_items] (base cosmology, k) pairs
 *   n_dir       1..ABCMB_MAX_TANGENTS
 *   tangent_scale  the tangents' size relative to the state's: the
 *               parameter step as a fraction of the parameter (eps_p /
 *               theta_p, e.g. 1e-4).  The tangent stage solves use the
 *               primal's very-chord test with atol scaled by it, so they
 *               stop at the same relative accuracy as the primal instead of
 *               iterating at rounding level.
 *   tstat_dev   [n_items x 2] int32 (optional): tangent chord iterations,
 *               tangent stage solves left unconverged after the primal's
 *               iteration limit (the last iterate is kept; the tangents
 *               never change the primal's step sequence)
 * Workspace: abcmb_pert_workspace_size(n_cosmo, n_items) (start-time grids
 * of every descriptor).
 */
#define ABCMB_MAX_TANGENTS 4
int abcmb_pert_forward_tangent(int n_cosmo, const abcmb_cosmo* cosmo_dev,
                               const double* tables_dev, const double* k_dev,
                               int n_items, const int32_t* items_dev,
                               int n_dir, const int32_t* dir_dev, double tangent_scale,
                               const abcmb_pert_settings* settings,
                               double* pt_dev, abcmb_kstat* kstat_dev, int32_t* tstat_dev,
                               void* workspace_dev, int64_t workspace_bytes,
                               void* stream);

/*
 * abcmb_pert_forward for finite-difference variants by internal numerical
 * differentiation (H. G. Bock, "Numerical treatment of inverse problems in
 * chemical reaction kinetics", 1981): the variants replay their base item's
 * discretisation instead of choosing their own.  Central differences of
 * whole adaptive solves (what the reference's finite-difference checks of
 * its jax gradients compute) pick up the noise of the variants' different
 * step sequences; a replayed variant takes exactly its base item's accepted
 * step ends and the number of chord iterations of each stage, so plus and
 * minus are one smooth discrete map evaluated at two parameter points and
 * their difference converges to the derivative of the base's integration
 * (the quantity jax.jacfwd through diffrax computes, abcmb/main.py:111).
 *   items_dev     [n_base_items + n_var_items] int32 x2 (cosmology, k index):
 *                 first the base items, then the variant items
 *   var_base_dev  [n_var_items] int32: index (0..n_base_items-1) of the base
 *                 item each variant item replays; the variant must have the
 *                 base's state layout and the same k (ABCMB_STATUS_BAD_LAYOUT
 *                 otherwise)
 *   kstat_dev     [n_base_items + n_var_items]; a variant whose base failed
 *                 reports ABCMB_STATUS_NONFINITE; variants report no rejected
 *                 steps
 * The base items are integrated exactly as abcmb_pert_forward does (same
 * tables, same step counts) while their accepted steps are recorded, then
 * the variants replay them: two launches in stream order.  Workspace:
 * abcmb_pert_ind_workspace_size(n_cosmo, n_base_items, settings.max_steps)
 * (12 bytes per base item and step allowed).
 */
int64_t abcmb_pert_ind_workspace_size(int n_cosmo, int n_base_items, int max_steps);
int abcmb_pert_forward_ind(int n_cosmo, const abcmb_cosmo* cosmo_dev,
                           const double* tables_dev, const double* k_dev,
                           int n_base_items, int n_var_items, const int32_t* items_dev,
                           const int32_t* var_base_dev,
                           const abcmb_pert_settings* settings,
                           double* pt_dev, abcmb_kstat* kstat_dev,
                           void* workspace_dev, int64_t workspace_bytes,
                           void* stream);

/*
 * Vector-Jacobian product of the perturbation integration with respect to
 * the gradient parameters: the cotangent of a PerturbationTable
 * contracted with the table's derivative columns, which
 * abcmb_pert_forward_ind (or _tangent, or whole-solve differences) leaves
 * in the variants' tables.  What jax.grad of a loss of the PerturbationTable
 * returns for the background parameters in the reference (the
 * PerturbationTable is differentiable in params through diffeqsolve,
 * abcmb/perturbations.py:285-312, abcmb/main.py:111).
 *   pt_dev        the batch's PerturbationTables after the gradient launch
 *   pt_bar_dev    a buffer shaped like pt_dev; only the base descriptors'
 *                 slots are read (dL/dPT of each base cosmology)
 *   base_dev      [n_base] descriptor index of each base cosmology
 *   dir_dev       [n_base][n_dir][2] (plus, minus) descriptor of direction p
 *   step_dev      [n_base][n_dir] the parameter step eps of direction p
 *                 (plus = theta + eps, minus = theta - eps)
 *   theta_bar_dev [n_base][n_dir] out: <pt_bar, (PT(+) - PT(-)) / (2 eps)>,
 *                 NaN where a descriptor is out of range or of another table
 *                 shape
 * Deterministic (fixed-order reductions).  A_s and n_s do not enter the
 * perturbations (their cotangent at this level is zero).  Cotangents with
 * respect to individual background-table entries need the discrete
 * adjoint of the integration, which this library does not provide.
 */
int abcmb_pert_vjp_theta(int n_cosmo, const abcmb_cosmo* cosmo_dev, const double* pt_dev, const double* pt_bar_dev,
                         int n_save, int n_base, const int32_t* base_dev, int n_dir, const int32_t* dir_dev,
                         const double* step_dev, double* theta_bar_dev, void* stream);

/*
 * abcmb_pert_forward for callers that cannot allocate device memory (no
 * cudaMalloc, no workspace of their own: e.g. code inside a framework that
 * owns every device byte).  No counterpart in the reference.  Same inputs,
 * outputs and results as abcmb_pert_forward (the same warps per block from
 * abcmb_set_pert_warps_per_block; abcmb_last_pert_grid reports its launch
 * too), but the scratch lives in a
 * library-owned static device array (about 1.2 MiB per device, held until
 * the process exits), so:
 *   - n_cosmo must not exceed ABCMB_PERT_NOALLOC_MAX_COSMO
 *     (ABCMB_ERR_WORKSPACE otherwise);
 *   - calls whose kernels may overlap on the GPU (unordered streams) race on
 *     the shared array: order them on one stream;
 *   - the first call on a device looks up the array's address with that
 *     device current: make it before any stream capture.
 */
#define ABCMB_PERT_NOALLOC_MAX_COSMO 8
int abcmb_pert_forward_noalloc(int n_cosmo, const abcmb_cosmo* cosmo_dev,
                               const double* tables_dev, const double* k_dev,
                               int n_items, const int32_t* items_dev,
                               const abcmb_pert_settings* settings,
                               double* pt_dev, abcmb_kstat* kstat_dev,
                               void* stream);

/* ------------------------------------------------------------------------ */
/* Spectrum: SpectrumSolver.get_Cl (spectrum.py:574-614)                   */
/* ------------------------------------------------------------------------ */

/* Bytes of device workspace abcmb_los_forward needs. */
int64_t abcmb_los_workspace_size(int n_cosmo, int max_nk, int nkt, int n_ell_tab,
                                 int n_save, int precision);

/*
 * For every cosmology: k-resample the PT source fields onto the transfer k
 * grid (cubic spline in log10 k), form the T0/T1/T2/E sources, run the
 * line-of-sight integral for every tabulated l in [idx_min, idx_max], do the
 * k quadrature, and spline C_l onto the integer ells l_min..l_max.
 *   cosmo_host [n_cosmo]   optional host copy of the descriptors (NULL: the
 *                          call reads them back and synchronises the stream;
 *                          pass it to keep the call asynchronous/capturable)
 *   kt_dev     [nkt]                            transfer k grid
 *   cl_raw_dev [n_cosmo x n_ell_tab x 3]        C_l at tabulated l (TT,TE,EE)
 *   cl_dev     [n_cosmo x 3 x (l_max-l_min+1)]  ClTT, ClTE, ClEE at integer l
 *   dcl_dns_dev (optional, NULL to skip) same layout as cl_dev: dC_l/dn_s,
 *              exact because n_s enters only the primordial factor of the k
 *              quadrature (spectrum.py:789-791); dC_l/dA_s = C_l / A_s.
 * Replaces: get_Cl, Cl_one_ell (spectrum.py:574-797).
 */
int abcmb_los_forward(int n_cosmo, const abcmb_cosmo* cosmo_dev,
                      const abcmb_cosmo* cosmo_host,
                      const double* tables_dev, const double* k_dev,
                      const double* pt_dev, const double* kt_dev,
                      const abcmb_los_settings* settings,
                      double* cl_raw_dev, double* cl_dev, double* dcl_dns_dev,
                      void* workspace_dev, int64_t workspace_bytes,
                      void* stream);

/*
 * Vector-Jacobian product of abcmb_los_forward (FP64): given cl_bar, the
 * cotangent of cl (same layout), writes
 *   pt_bar_dev     cotangent of the PerturbationTable (layout of pt; the ten
 *                  fields the line of sight reads get their cotangent on the
 *                  lna rows it uses, everything else 0)
 *   param_bar_dev  [n_cosmo x 2] cotangents of A_s and n_s.
 * The background arrays and the transfer k grid are held fixed.  The
 * hand-written adjoint of Cl_one_ell / get_Cl (spectrum.py:574-797): the
 * transposed l spline, the k-quadrature and line-of-sight sums taken in
 * reverse (over l instead of lna), the transposed source combination and
 * the transposed not-a-knot k spline.  cosmo_host is required.
 */
int64_t abcmb_los_vjp_workspace_size(int n_cosmo, int max_nk, const abcmb_los_settings* settings);
int abcmb_los_vjp(int n_cosmo, const abcmb_cosmo* cosmo_dev, const abcmb_cosmo* cosmo_host,
                  const double* tables_dev, const double* k_dev, const double* pt_dev,
                  const double* kt_dev, const abcmb_los_settings* settings,
                  const double* cl_bar_dev, double* pt_bar_dev, double* param_bar_dev,
                  void* workspace_dev, int64_t workspace_bytes, void* stream);

/*
 * The last stage of abcmb_los_forward on its own: the cubic spline in l of
 * C_l given at the tabulated l (spectrum.py:597-608) onto the integer ells
 * l_min..l_max (l_min == 2), for callers that assemble cl_raw themselves --
 * e.g. one cosmology whose tabulated l were shared out over several GPUs and
 * gathered.  Same arithmetic as abcmb_los_forward's own spline.
 *   cl_raw_dev [n_cosmo x n_ell_tab x 3]  C_l at bessel_l_tab[idx_min + i]
 *   cl_dev     [n_cosmo x 3 x (l_max-l_min+1)]
 */
int abcmb_cl_spline(int n_cosmo, const double* cl_raw_dev, int idx_min, int n_ell_tab,
                    int l_min, int l_max, double* cl_dev, void* stream);

/*
 * Linear matter power spectrum P(k, z) (SpectrumSolver.Pk_lin,
 * spectrum.py:268-302): delta_m interpolated linearly in lna to z, then
 * linearly in k (clamped), times the primordial spectrum.
 *   kout_dev [n_kout], z_dev [n_z], pk_dev [n_cosmo x n_z x n_kout]
 */
int abcmb_pk_lin(int n_cosmo, const abcmb_cosmo* cosmo_dev, const double* k_dev,
                 const double* pt_dev, int n_save, double k_pivot,
                 int n_kout, const double* kout_dev, int n_z, const double* z_dev,
                 double* pk_dev, void* stream);

/* ------------------------------------------------------------------------ */
/* Lensing: SpectrumSolver.lensing_Cl / lensed_Cls (spectrum.py:349-572)    */
/* ------------------------------------------------------------------------ */

/* Per-cosmology lensing inputs. */
typedef struct abcmb_lens_cosmo {
  double lna_rec;     /* BG.lna_rec: argmax of the visibility on
                         linspace(-8, -4, 1500) (abcmb/background.py:555-557) */
  double omega_m;     /* params["omega_m"] (abcmb/main.py:569-574)           */
} abcmb_lens_cosmo;

/* Lensing settings (SpectrumSolver.__init__, abcmb/spectrum.py:219-236). */
typedef struct abcmb_lens_settings {
  double k_pivot;
  int32_t l_max;      /* lensed output ells 2..l_max                          */
  int32_t l_lens;     /* lensing_ellmax = l_max + 500: unlensed input and
                         C_l^phiphi on ells 2..l_lens                         */
  int32_t n_mu;       /* quadrature nodes: the l_lens + 70 Gauss-Legendre
                         nodes plus mu = 1 with weight 0, mu ascending        */
  int32_t n_lna;      /* Limber quadrature points (500, spectrum.py:419)     */
  int32_t n_save;     /* PT save points (500)                                */
  int32_t max_nk;     /* largest perturbation k grid in the batch            */
} abcmb_lens_settings;

/* Bytes of device workspace abcmb_lens_forward needs. */
int64_t abcmb_lens_workspace_size(int n_cosmo, const abcmb_lens_settings* settings);

/*
 * Lensed TT, TE, EE (no BB, like the reference) for every cosmology:
 * C_l^phiphi in the Limber approximation (lensing_Cl, spectrum.py:386-435,
 * with lensing_power_spectrum :349-384 and Pk_lin :268-302), the lensing
 * correlation functions on the mu nodes from the Wigner-d recursions
 * (lensed_Cls :437-572; ABCMBTools.wigner_d_matrix and d00..d4n,
 * ABCMBTools.py:16-186, evaluated on the fly rather than stored), and the
 * Gauss-Legendre quadrature back to C_l.
 *   lens_dev        [n_cosmo]                    lna_rec, omega_m
 *   mu_dev, w_dev   [n_mu]                       nodes and weights
 *   cl_unlensed_dev [n_cosmo x 3 x (l_lens-1)]   unlensed TT, TE, EE on
 *                   ells 2..l_lens (abcmb_los_forward with l_max = l_lens)
 *   clpp_dev        [n_cosmo x (l_lens-1)]       C_l^phiphi on 2..l_lens
 *   cl_dev          [n_cosmo x 3 x (l_max-1)]    lensed TT, TE, EE
 * Replaces: the lensing branch of get_Cl (spectrum.py:603-612).
 */
int abcmb_lens_forward(int n_cosmo, const abcmb_cosmo* cosmo_dev,
                       const abcmb_lens_cosmo* lens_dev,
                       const double* tables_dev, const double* k_dev,
                       const double* pt_dev,
                       const double* mu_dev, const double* w_dev,
                       const double* cl_unlensed_dev,
                       const abcmb_lens_settings* settings,
                       double* clpp_dev, double* cl_dev,
                       void* workspace_dev, int64_t workspace_bytes,
                       void* stream);

/* ------------------------------------------------------------------------ */
/* Tuning and diagnostics                                                   */
/* ------------------------------------------------------------------------ */

/* Warps per block of the perturbation kernel (1..4; default 4). */
int abcmb_set_pert_warps_per_block(int warps);

/* Instantiation of the perturbation kernel: 0 = chosen by queue length
 * (default), 1 = two blocks per SM (no register cap: shortest time per
 * item), 2 = three blocks per SM (168 registers: most resident warps).
 * Either gives the same results bit for bit (every item is one warp's
 * independent computation). */
int abcmb_set_pert_variant(int variant);

/* Warps per block of the tangent kernel: 0 = the count with the most
 * resident warps per SM (default), else 1..4. */
int abcmb_set_pert_tangent_warps_per_block(int warps);

/* Cycles the perturbation kernels' warps spent per phase since the last
 * reset, summed over warps: cycles[12] = stage-time background, Newton-matrix
 * factorisation, stage set-up, residual, structured solve, chord update and
 * convergence test, error estimate and step-size control, the rest; and in
 * the tangent kernel the basis changes, the tangent stages' constant parts,
 * the tangent chord iterations, the variants' tables.  Only a
 * library built with ABCMB_PHASE_CLOCKS counts (python -m abcmb_b200.build
 * --phase-clocks); others return ABCMB_ERR_ARG.  reset != 0 zeroes the
 * counters after reading. */
int abcmb_pert_phase_clocks(uint64_t* cycles, int reset);

/* Grid size (blocks) of the last perturbation launch on this process. */
int abcmb_last_pert_grid(void);

/* Measured FP64 FMA rate of the current device in TFLOP/s (best of 5 runs
 * of `iters` x 128 independent FMAs per thread): the peak the perturbation
 * kernel's roofline is quoted against. */
int abcmb_probe_fp64_tflops(double* tflops, int iters, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ABCMB_B200_H */
