/*
 * abcmb_oracle.h -- CPU FP64 restatement of ABCMB's hot path.
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels and the timed
 * CPU baseline.  The product library never includes or links this.
 */
#ifndef ABCMB_ORACLE_H
#define ABCMB_ORACLE_H
#include <stdint.h>
#include "../include/abcmb_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Tabulated spherical-Bessel functions (abcmb/bessel_tab). */
typedef struct oracle_bessel {
  int n_l, n_x;
  const int32_t* l_tab;
  const double* xmin[3];
  const double* xmax[3];
  const double* phi[3];   /* [l][x] */
} oracle_bessel;

double oracle_fast_interp(double x, double xp_min, double xp_max, const double* fp, int n);
double oracle_np_interp(double x, const double* xp, const double* fp, int n);
double oracle_aH(const abcmb_cosmo* c, double lna);
double oracle_aH_prime(const abcmb_cosmo* c, double lna);
double oracle_tau(const abcmb_cosmo* c, const double* tables, double lna);
double oracle_xe(const abcmb_cosmo* c, const double* tables, double lna);
double oracle_Tm(const abcmb_cosmo* c, const double* tables, double lna);
double oracle_tau_c(const abcmb_cosmo* c, const double* tables, double lna);
double oracle_start_time(const abcmb_cosmo* c, const double* tables, double k, double R_tc, double R_large);
void oracle_kvaerno5_tableau(double* A49, double* c7, double* gamma);
void oracle_rhs(const abcmb_cosmo* c, const double* tables, double k, double lna, const double* y, double* f);
void oracle_initial_conditions(const abcmb_cosmo* c, const double* tables, double k, double lna, double* y);
void oracle_output_fields(const abcmb_cosmo* c, const double* tables, double k, double lna,
                          const double* y, double* out);
int oracle_pert_forward(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                        int n_items, const int32_t* items, const abcmb_pert_settings* s,
                        double* pt, abcmb_kstat* kstat, int n_threads);
int oracle_pert_forward_tangent(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                                int n_items, const int32_t* items, int n_dir, const int32_t* dirs, double tscale,
                                const abcmb_pert_settings* s, double* pt, abcmb_kstat* kstat, int32_t* tstat,
                                int n_threads);
int oracle_pert_forward_ind(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                            int n_base, int n_var, const int32_t* items, const int32_t* var_base,
                            const abcmb_pert_settings* s, double* pt, abcmb_kstat* kstat, int n_threads);
void oracle_spline_slopes(const double* x, const double* y, int n, double* s);
double oracle_spline_eval(const double* x, const double* y, const double* s, int n, double xq);
double oracle_phi(int which, const oracle_bessel* B, int idx, double x);
void oracle_sources(const abcmb_cosmo* c, const double* tables, const double* kbuf, const double* pt,
                    const double* kt, int nkt, int n_save, const abcmb_los_settings* ls, double* S);
int oracle_los_forward(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                       const double* pt, const double* kt, const abcmb_los_settings* ls, int n_save,
                       const oracle_bessel* B, double* cl_raw, double* cl, int n_threads);
int oracle_sizeof(int which);
void oracle_wigner_d(int m, int n, double mu, int l_end, double* out);
int oracle_lens_forward(int n_cosmo, const abcmb_cosmo* cosmo, const abcmb_lens_cosmo* lens, const double* tables,
                        const double* kbuf, const double* pt, const double* mu, const double* w,
                        const double* cl_unl, const abcmb_lens_settings* s, double* clpp, double* cl,
                        int n_threads);
int oracle_bg_forward(int n_cosmo, abcmb_cosmo* cosmo, double* tables, const abcmb_bg_settings* s,
                      abcmb_bgstat* stat, int n_threads);
int oracle_kappa_solve(const abcmb_cosmo* c, const double* tables, double rhs_scale, int max_steps,
                       int* nsteps, double* kappa_end);
/* HyRex tables (abcmb/hyrex/tabs): Alpha_inf [100 x 40 x 4], R_inf [100],
 * fit_swift [n_swift x 5]. */
typedef struct oracle_hyrex_tables {
  const double* alpha;
  const double* R;
  const double* swift;
  int n_swift;
} oracle_hyrex_tables;
void oracle_kvaerno3_tableau(double* A16, double* c4, double* b4, double* be4);
int oracle_hyrex_sizes(int n_grid, int* n_xe, int* n_tm);
int oracle_hyrex(const oracle_hyrex_tables* tab, int n_grid, const double* TCMB, const double* nH,
                 const double* H, double YHe, double omega_b, double omega_cdm, double Neff, double* xe_out,
                 double* lna_out, int cap_xe, double* tm_out, double* lna_tm_out, int cap_tm, int* info);
int oracle_hyrex_rates(const oracle_hyrex_tables* tab, int n_grid, const double* TCMB, const double* nH,
                       const double* H, double YHe, double omega_b, double omega_cdm, double Neff, double lna,
                       double xe_he, double xe_h, double* out);
int oracle_pk_lin(int n_cosmo, const abcmb_cosmo* cosmo, const double* kbuf, const double* pt, int n_save,
                  double k_pivot, int n_kout, const double* kout, int n_z, const double* z, double* pk);

#ifdef __cplusplus
}
#endif
#endif
