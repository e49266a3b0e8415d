// capi.cu -- the extern "C" entry points of include/abcmb_b200.h.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace abcmb {
int64_t pert_workspace_bytes(int n_cosmo);
int pert_phase_clocks(unsigned long long* out, int reset);
cudaError_t launch_pert(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                        int n_items, const int32_t* items, const abcmb_pert_settings& s, double* pt,
                        abcmb_kstat* kstat, void* ws, cudaStream_t stream, int warps_per_block, int* grid_out);
cudaError_t launch_pert_tangent(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                                int n_items, const int32_t* items, int nd, const int32_t* dirs, double tscale,
                                const abcmb_pert_settings& s, double* pt, abcmb_kstat* kstat, int32_t* tstat,
                                void* ws, cudaStream_t stream, int* grid_out, int* warps_out);
int64_t pert_ind_workspace_bytes(int n_cosmo, int n_base, int max_steps);
cudaError_t launch_pert_ind(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                            int n_base, int n_var, const int32_t* items, const int32_t* var_base,
                            const abcmb_pert_settings& s, double* pt, abcmb_kstat* kstat, void* ws,
                            cudaStream_t stream, int warps_per_block, int* grid_out);
cudaError_t launch_pert_vjp_theta(int n_cosmo, const abcmb_cosmo* cosmo, const double* pt, const double* pt_bar,
                                  int n_save, int n_base, const int32_t* base, int n_dir, const int32_t* dirs,
                                  const double* step, double* theta_bar, cudaStream_t stream);
int64_t los_workspace_bytes(int n_cosmo, int max_nk, int nkt, int n_ell_tab, int n_save, int precision);
cudaError_t launch_los(int n_cosmo, const abcmb_cosmo* cosmo_dev, const abcmb_cosmo* cosmo_host,
                       const double* tables, const double* kbuf, const double* pt, const double* kt,
                       const abcmb_los_settings& ls, int n_save, const BesselDev& B, double* cl_raw,
                       double* cl, double* dcl_dns, void* ws, cudaStream_t stream);
cudaError_t launch_pk_lin(int n_cosmo, const abcmb_cosmo* cosmo, const double* kbuf, const double* pt,
                          int n_save, double k_pivot, int n_kout, const double* kout, int n_z, const double* z,
                          double* pk, cudaStream_t stream);
cudaError_t launch_cl_spline(int n_cosmo, const double* cl_raw, int idx_min, int n_ell_tab, int l_min, int l_max,
                             const BesselDev& B, double* cl, cudaStream_t stream);
int64_t los_vjp_workspace_bytes(int n_cosmo, int max_nk, int nkt, int n_ell_tab, int n_save, int n_out);
cudaError_t launch_los_vjp(int n_cosmo, const abcmb_cosmo* cosmo_dev, const abcmb_cosmo* cosmo_host,
                           const double* tables, const double* kbuf, const double* pt, const double* kt,
                           const abcmb_los_settings& ls, int n_save, const BesselDev& B, const double* cl_bar,
                           double* pt_bar, double* param_bar, void* ws, cudaStream_t stream);
int64_t lens_workspace_bytes(int n_cosmo, const abcmb_lens_settings& s);
cudaError_t launch_hyrex_inputs(int n_cosmo, int n_grid, const abcmb_cosmo* cosmo, double* T, double* nH, double* H,
                                cudaStream_t stream);
int64_t bg_workspace_bytes(int n_cosmo, const abcmb_bg_settings& s);
int hyrex_sizes(int n_grid, int* n_xe, int* n_tm);
cudaError_t hyrex_upload_tables(const double* alpha, const double* R, const double* swift, int n_swift);
bool hyrex_tables_ready();
cudaError_t launch_hyrex(int n_cosmo, int n_grid, const double* T, const double* nH, const double* H,
                         const abcmb_hyrex_params* params, double* xe, double* lna_xe, double* tm, double* lna_tm,
                         int32_t* info, cudaStream_t stream);
cudaError_t launch_bg(int n_cosmo, abcmb_cosmo* cosmo, double* tables, const abcmb_bg_settings& s,
                      abcmb_bgstat* stat, void* ws, cudaStream_t stream);
cudaError_t launch_lens(int n_cosmo, const abcmb_cosmo* cosmo, const abcmb_lens_cosmo* lens, const double* tables,
                        const double* kbuf, const double* pt, const double* mu, const double* w,
                        const double* cl_unl, const abcmb_lens_settings& s, double* clpp, double* cl, void* ws,
                        cudaStream_t stream);
}  // namespace abcmb

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(ABCMB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Bessel tables, resident once per device (spectrum.py loads them once at import).
struct BesselCache {
  bool ready = false;
  abcmb::BesselDev dev{};
  void* mem = nullptr;
};
std::mutex g_mu;
std::vector<BesselCache> g_bessel;

BesselCache* bessel_for_current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if ((int)g_bessel.size() <= d) g_bessel.resize(d + 1);
  return &g_bessel[d];
}

int g_warps_per_block = 4;
int g_last_grid = 0;
int g_pert_variant = 0;        // 0 automatic, 1 two blocks/SM, 2 three blocks/SM
int g_pert_tangent_warps = 0;  // 0 automatic (most resident warps), else warps per block

}  // namespace

namespace abcmb {
// error message for abcmb_last_error from entry points in other files
void set_last_error(const std::string& msg) { g_last_error = msg; }
// the launch configuration every perturbation entry point shares: warps per
// block (abcmb_set_pert_warps_per_block) and the grid of the last launch
// (abcmb_last_pert_grid)
int pert_warps_per_block() { return g_warps_per_block; }
int pert_variant() { return g_pert_variant; }
int pert_tangent_warps() { return g_pert_tangent_warps; }
void set_last_pert_grid(int grid) { g_last_grid = grid; }
}  // namespace abcmb

extern "C" {

int abcmb_version(void) { return ABCMB_B200_VERSION; }

const char* abcmb_last_error(void) { return g_last_error.c_str(); }

int abcmb_upload_bessel(int n_l, int n_x, const int32_t* l_tab, const double* xmin0, const double* xmax0,
                        const double* phi0, const double* xmin1, const double* xmax1, const double* phi1,
                        const double* xmin2, const double* xmax2, const double* phi2) {
  if (n_l <= 0 || n_x <= 1 || !l_tab || !phi0 || !phi1 || !phi2) return fail(ABCMB_ERR_ARG, "bad Bessel table");
  BesselCache* bc = bessel_for_current_device();
  if (!bc) return fail(ABCMB_ERR_CUDA, "cudaGetDevice failed");
  std::lock_guard<std::mutex> lk(g_mu);
  if (bc->mem) {
    cudaFree(bc->mem);
    bc->mem = nullptr;
    bc->ready = false;
  }
  const size_t nl = (size_t)n_l, nx = (size_t)n_x;
  const size_t bytes = 256 + nl * 4 + 6 * nl * 8 + 3 * nl * nx * 8 + 256;
  void* mem = nullptr;
  cudaError_t e = cudaMalloc(&mem, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_upload_bessel cudaMalloc");
  char* p = static_cast<char*>(mem);
  int32_t* dl = reinterpret_cast<int32_t*>(p);
  p += (nl * 4 + 255) / 256 * 256;
  double* dxmin = reinterpret_cast<double*>(p);
  p += 3 * nl * 8;
  double* dxmax = reinterpret_cast<double*>(p);
  p += 3 * nl * 8;
  double* dphi = reinterpret_cast<double*>(p);
  const double* xmins[3] = {xmin0, xmin1, xmin2};
  const double* xmaxs[3] = {xmax0, xmax1, xmax2};
  const double* phis[3] = {phi0, phi1, phi2};
  e = cudaMemcpy(dl, l_tab, nl * 4, cudaMemcpyHostToDevice);
  for (int n = 0; n < 3 && e == cudaSuccess; ++n) {
    e = cudaMemcpy(dxmin + n * nl, xmins[n], nl * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dxmax + n * nl, xmaxs[n], nl * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dphi + n * nl * nx, phis[n], nl * nx * 8, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(mem);
    return cuda_fail(e, "abcmb_upload_bessel cudaMemcpy");
  }
  bc->mem = mem;
  bc->dev = abcmb::BesselDev{n_l, n_x, dl, dxmin, dxmax, dphi};
  bc->ready = true;
  return ABCMB_OK;
}

int abcmb_upload_hyrex_tables(const double* alpha, const double* R, const double* swift, int n_swift) {
  if (!alpha || !R || !swift || n_swift < 2) return fail(ABCMB_ERR_ARG, "abcmb_upload_hyrex_tables: bad argument");
  cudaError_t e = abcmb::hyrex_upload_tables(alpha, R, swift, n_swift);
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_upload_hyrex_tables");
  return ABCMB_OK;
}

int abcmb_hyrex_sizes(int n_grid, int* n_xe, int* n_tm) {
  if (n_grid < 2 || !n_xe || !n_tm) return -1;
  return abcmb::hyrex_sizes(n_grid, n_xe, n_tm);
}

int abcmb_hyrex_inputs(int n_cosmo, int n_grid, const abcmb_cosmo* cosmo_dev, double* T_dev, double* nH_dev,
                       double* H_dev, void* stream) {
  if (n_cosmo <= 0 || n_grid < 2 || !cosmo_dev || !T_dev || !nH_dev || !H_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_hyrex_inputs: null argument or empty grid");
  cudaError_t e = abcmb::launch_hyrex_inputs(n_cosmo, n_grid, cosmo_dev, T_dev, nH_dev, H_dev,
                                             static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_hyrex_inputs");
  return ABCMB_OK;
}

int abcmb_hyrex_forward(int n_cosmo, int n_grid, const double* T_dev, const double* nH_dev, const double* H_dev,
                        const abcmb_hyrex_params* params_dev, double* xe_dev, double* lna_xe_dev, double* tm_dev,
                        double* lna_tm_dev, int32_t* info_dev, void* stream) {
  if (n_cosmo <= 0 || !T_dev || !nH_dev || !H_dev || !params_dev || !xe_dev || !lna_xe_dev || !tm_dev ||
      !lna_tm_dev || !info_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_hyrex_forward: null argument or n_cosmo <= 0");
  int nx = 0, nt = 0;
  if (n_grid < 2 || abcmb::hyrex_sizes(n_grid, &nx, &nt) < 2)
    return fail(ABCMB_ERR_ARG, "abcmb_hyrex_forward: the grid needs at least two points with z >= 3600");
  if (!abcmb::hyrex_tables_ready()) return fail(ABCMB_ERR_TABLES, "abcmb_hyrex_forward: tables not uploaded");
  cudaError_t e = abcmb::launch_hyrex(n_cosmo, n_grid, T_dev, nH_dev, H_dev, params_dev, xe_dev, lna_xe_dev, tm_dev,
                                      lna_tm_dev, info_dev, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_hyrex_forward");
  return ABCMB_OK;
}

// the two solves' step limits: positive and small enough that the node
// buffers stay a modest workspace (diffrax accepts any positive max_steps)
constexpr int BG_MAX_STEPS_LIMIT = 1 << 20;

static bool bg_settings_ok(const abcmb_bg_settings* s) {
  return s && s->n_save >= 3 && s->max_steps_tau >= 1 && s->max_steps_kappa >= 1 &&
         s->max_steps_tau <= BG_MAX_STEPS_LIMIT && s->max_steps_kappa <= BG_MAX_STEPS_LIMIT;
}

int64_t abcmb_bg_workspace_size(int n_cosmo, const abcmb_bg_settings* settings) {
  if (n_cosmo <= 0 || !bg_settings_ok(settings)) return -1;
  return abcmb::bg_workspace_bytes(n_cosmo, *settings);
}

int abcmb_bg_forward(int n_cosmo, abcmb_cosmo* cosmo_dev, double* tables_dev, const abcmb_bg_settings* settings,
                     abcmb_bgstat* stat_dev, void* workspace_dev, int64_t workspace_bytes, void* stream) {
  if (n_cosmo <= 0 || !cosmo_dev || !tables_dev || !stat_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_bg_forward: null argument or n_cosmo <= 0");
  if (!bg_settings_ok(settings))
    return fail(ABCMB_ERR_ARG, "abcmb_bg_forward: settings need n_save >= 3 and 1 <= max_steps <= 2^20");
  const int64_t need = abcmb::bg_workspace_bytes(n_cosmo, *settings);
  if (!workspace_dev || workspace_bytes < need) return fail(ABCMB_ERR_WORKSPACE, "abcmb_bg_forward: workspace");
  cudaError_t e = abcmb::launch_bg(n_cosmo, cosmo_dev, tables_dev, *settings, stat_dev, workspace_dev,
                                   static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_bg_forward");
  return ABCMB_OK;
}

int64_t abcmb_pert_workspace_size(int n_cosmo, int n_items) {
  (void)n_items;
  return abcmb::pert_workspace_bytes(n_cosmo);
}

int abcmb_pert_forward(int n_cosmo, const abcmb_cosmo* cosmo_dev, const double* tables_dev, const double* k_dev,
                       int n_items, const int32_t* items_dev, const abcmb_pert_settings* settings, double* pt_dev,
                       abcmb_kstat* kstat_dev, void* workspace_dev, int64_t workspace_bytes, void* stream) {
  if (n_cosmo <= 0 || n_items < 0 || !cosmo_dev || !tables_dev || !k_dev || !settings || !pt_dev || !kstat_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward: null argument");
  if (settings->max_ny <= 0 || settings->n_save < 2 || settings->max_steps <= 0)
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward: settings.max_ny / n_save / max_steps");
  if (workspace_bytes < abcmb::pert_workspace_bytes(n_cosmo) || !workspace_dev)
    return fail(ABCMB_ERR_WORKSPACE, "abcmb_pert_forward: workspace too small");
  if (n_items == 0) return ABCMB_OK;
  cudaError_t e = abcmb::launch_pert(n_cosmo, cosmo_dev, tables_dev, k_dev, n_items, items_dev, *settings, pt_dev,
                                     kstat_dev, workspace_dev, static_cast<cudaStream_t>(stream), g_warps_per_block,
                                     &g_last_grid);
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_pert_forward");
  return ABCMB_OK;
}

int abcmb_pert_forward_tangent(int n_cosmo, const abcmb_cosmo* cosmo_dev, const double* tables_dev,
                               const double* k_dev, int n_items, const int32_t* items_dev, int n_dir,
                               const int32_t* dir_dev, double tangent_scale, const abcmb_pert_settings* settings,
                               double* pt_dev,
                               abcmb_kstat* kstat_dev, int32_t* tstat_dev, void* workspace_dev,
                               int64_t workspace_bytes, void* stream) {
  if (n_cosmo <= 0 || n_items < 0 || !cosmo_dev || !tables_dev || !k_dev || !settings || !pt_dev || !kstat_dev ||
      !dir_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward_tangent: null argument");
  if (n_dir < 1 || n_dir > ABCMB_MAX_TANGENTS)
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward_tangent: n_dir must be 1..ABCMB_MAX_TANGENTS");
  if (!(tangent_scale > 0. && tangent_scale <= 1.))
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward_tangent: tangent_scale must be in (0, 1]");
  if (settings->max_ny <= 0 || settings->n_save < 2 || settings->max_steps <= 0)
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward_tangent: settings.max_ny / n_save / max_steps");
  if (workspace_bytes < abcmb::pert_workspace_bytes(n_cosmo) || !workspace_dev)
    return fail(ABCMB_ERR_WORKSPACE, "abcmb_pert_forward_tangent: workspace too small");
  if (n_items == 0) return ABCMB_OK;
  int warps = 0;
  cudaError_t e = abcmb::launch_pert_tangent(n_cosmo, cosmo_dev, tables_dev, k_dev, n_items, items_dev, n_dir,
                                             dir_dev, tangent_scale, *settings, pt_dev, kstat_dev, tstat_dev,
                                             workspace_dev,
                                             static_cast<cudaStream_t>(stream), &g_last_grid, &warps);
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_pert_forward_tangent");
  return ABCMB_OK;
}

int64_t abcmb_pert_ind_workspace_size(int n_cosmo, int n_base_items, int max_steps) {
  if (n_cosmo <= 0 || n_base_items < 0 || max_steps <= 0)
    return fail(ABCMB_ERR_ARG, "abcmb_pert_ind_workspace_size: bad argument");
  return abcmb::pert_ind_workspace_bytes(n_cosmo, n_base_items, max_steps);
}

int abcmb_pert_forward_ind(int n_cosmo, const abcmb_cosmo* cosmo_dev, const double* tables_dev, const double* k_dev,
                           int n_base_items, int n_var_items, const int32_t* items_dev, const int32_t* var_base_dev,
                           const abcmb_pert_settings* settings, double* pt_dev, abcmb_kstat* kstat_dev,
                           void* workspace_dev, int64_t workspace_bytes, void* stream) {
  if (n_cosmo <= 0 || n_base_items < 0 || n_var_items < 0 || !cosmo_dev || !tables_dev || !k_dev || !settings ||
      !pt_dev || !kstat_dev || (n_base_items + n_var_items > 0 && !items_dev) || (n_var_items > 0 && !var_base_dev))
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward_ind: null argument");
  if (settings->max_ny <= 0 || settings->n_save < 2 || settings->max_steps <= 0)
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward_ind: settings.max_ny / n_save / max_steps");
  if (n_var_items > 0 && n_base_items == 0)
    return fail(ABCMB_ERR_ARG, "abcmb_pert_forward_ind: variant items without base items");
  if (!workspace_dev ||
      workspace_bytes < abcmb::pert_ind_workspace_bytes(n_cosmo, n_base_items, settings->max_steps))
    return fail(ABCMB_ERR_WORKSPACE, "abcmb_pert_forward_ind: workspace too small");
  if (n_base_items + n_var_items == 0) return ABCMB_OK;
  cudaError_t e = abcmb::launch_pert_ind(n_cosmo, cosmo_dev, tables_dev, k_dev, n_base_items, n_var_items, items_dev,
                                         var_base_dev, *settings, pt_dev, kstat_dev, workspace_dev,
                                         static_cast<cudaStream_t>(stream), g_warps_per_block, &g_last_grid);
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_pert_forward_ind");
  return ABCMB_OK;
}

int abcmb_pert_vjp_theta(int n_cosmo, const abcmb_cosmo* cosmo_dev, const double* pt_dev, const double* pt_bar_dev,
                         int n_save, int n_base, const int32_t* base_dev, int n_dir, const int32_t* dir_dev,
                         const double* step_dev, double* theta_bar_dev, void* stream) {
  if (n_cosmo <= 0 || n_base < 0 || !cosmo_dev || !pt_dev || !pt_bar_dev || !theta_bar_dev ||
      (n_base > 0 && (!base_dev || !dir_dev || !step_dev)))
    return fail(ABCMB_ERR_ARG, "abcmb_pert_vjp_theta: null argument");
  if (n_dir < 1 || n_dir > 65535 || n_save < 2) return fail(ABCMB_ERR_ARG, "abcmb_pert_vjp_theta: n_dir / n_save");
  if (n_base == 0) return ABCMB_OK;
  if (n_base > 65535) return fail(ABCMB_ERR_ARG, "abcmb_pert_vjp_theta: at most 65535 base cosmologies per call");
  cudaError_t e = abcmb::launch_pert_vjp_theta(n_cosmo, cosmo_dev, pt_dev, pt_bar_dev, n_save, n_base, base_dev, n_dir,
                                               dir_dev, step_dev, theta_bar_dev, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_pert_vjp_theta");
  return ABCMB_OK;
}

int64_t abcmb_los_workspace_size(int n_cosmo, int max_nk, int nkt, int n_ell_tab, int n_save, int precision) {
  return abcmb::los_workspace_bytes(n_cosmo, max_nk, nkt, n_ell_tab, n_save, precision);
}

int abcmb_los_forward(int n_cosmo, const abcmb_cosmo* cosmo_dev, const abcmb_cosmo* cosmo_host,
                      const double* tables_dev, const double* k_dev, const double* pt_dev, const double* kt_dev,
                      const abcmb_los_settings* settings, double* cl_raw_dev, double* cl_dev, double* dcl_dns_dev,
                      void* workspace_dev, int64_t workspace_bytes, void* stream) {
  if (n_cosmo <= 0 || !cosmo_dev || !tables_dev || !k_dev || !pt_dev || !kt_dev || !settings || !cl_raw_dev ||
      !cl_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_los_forward: null argument");
  const abcmb_los_settings& ls = *settings;
  if (ls.l_min != 2) return fail(ABCMB_ERR_ARG, "abcmb_los_forward: get_Cl indexes [ells-2], l_min must be 2");
  if (ls.idx_max - ls.idx_min + 1 < 4 || ls.nkt < 2) return fail(ABCMB_ERR_ARG, "abcmb_los_forward: sizes");
  BesselCache* bc = bessel_for_current_device();
  if (!bc || !bc->ready) return fail(ABCMB_ERR_TABLES, "abcmb_los_forward: Bessel tables not uploaded");
  if (ls.idx_min < 0 || ls.idx_max >= bc->dev.n_l) return fail(ABCMB_ERR_ARG, "abcmb_los_forward: l index range");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the launcher needs the per-cosmology sizes on the host: use the caller's
  // host copy (no synchronisation, graph-capturable) or read them back
  std::vector<abcmb_cosmo> host(n_cosmo);
  cudaError_t e = cudaSuccess;
  if (cosmo_host) {
    std::memcpy(host.data(), cosmo_host, sizeof(abcmb_cosmo) * n_cosmo);
  } else {
    e = cudaMemcpyAsync(host.data(), cosmo_dev, sizeof(abcmb_cosmo) * n_cosmo, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "abcmb_los_forward descriptor read");
  }
  int max_nk = 0;
  for (const auto& c : host) max_nk = c.nk > max_nk ? c.nk : max_nk;
  const int n_save = ls.n_save;
  if (n_save < 3) return fail(ABCMB_ERR_ARG, "abcmb_los_forward: n_save");
  int64_t need = abcmb::los_workspace_bytes(n_cosmo, max_nk, ls.nkt, ls.idx_max - ls.idx_min + 1, n_save, ls.precision);
  if (!workspace_dev || workspace_bytes < need) return fail(ABCMB_ERR_WORKSPACE, "abcmb_los_forward: workspace");
  e = abcmb::launch_los(n_cosmo, cosmo_dev, host.data(), tables_dev, k_dev, pt_dev, kt_dev, ls, n_save, bc->dev,
                        cl_raw_dev, cl_dev, dcl_dns_dev, workspace_dev, st);
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_los_forward");
  return ABCMB_OK;
}

int abcmb_pk_lin(int n_cosmo, const abcmb_cosmo* cosmo_dev, const double* k_dev, const double* pt_dev, int n_save,
                 double k_pivot, int n_kout, const double* kout_dev, int n_z, const double* z_dev, double* pk_dev,
                 void* stream) {
  if (n_cosmo <= 0 || n_kout <= 0 || n_z <= 0 || !cosmo_dev || !k_dev || !pt_dev || !kout_dev || !z_dev || !pk_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_pk_lin: bad argument");
  cudaError_t e = abcmb::launch_pk_lin(n_cosmo, cosmo_dev, k_dev, pt_dev, n_save, k_pivot, n_kout, kout_dev, n_z,
                                       z_dev, pk_dev, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_pk_lin");
  return ABCMB_OK;
}

int64_t abcmb_los_vjp_workspace_size(int n_cosmo, int max_nk, const abcmb_los_settings* settings) {
  if (n_cosmo <= 0 || max_nk < 4 || !settings) return fail(ABCMB_ERR_ARG, "abcmb_los_vjp_workspace_size: bad argument");
  const abcmb_los_settings& ls = *settings;
  return abcmb::los_vjp_workspace_bytes(n_cosmo, max_nk, ls.nkt, ls.idx_max - ls.idx_min + 1, ls.n_save,
                                        ls.l_max - ls.l_min + 1);
}

int abcmb_los_vjp(int n_cosmo, const abcmb_cosmo* cosmo_dev, const abcmb_cosmo* cosmo_host, const double* tables_dev,
                  const double* k_dev, const double* pt_dev, const double* kt_dev, const abcmb_los_settings* settings,
                  const double* cl_bar_dev, double* pt_bar_dev, double* param_bar_dev, void* workspace_dev,
                  int64_t workspace_bytes, void* stream) {
  if (n_cosmo <= 0 || !cosmo_dev || !cosmo_host || !tables_dev || !k_dev || !pt_dev || !kt_dev || !settings ||
      !cl_bar_dev || !pt_bar_dev || !param_bar_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_los_vjp: null argument");
  const abcmb_los_settings& ls = *settings;
  if (ls.l_min != 2 || ls.idx_max - ls.idx_min + 1 < 4 || ls.nkt < 2 || ls.n_save < 3 || ls.l_max < ls.l_min)
    return fail(ABCMB_ERR_ARG, "abcmb_los_vjp: settings");
  if (ls.precision != 0) return fail(ABCMB_ERR_ARG, "abcmb_los_vjp: the adjoint is FP64 (precision 0)");
  BesselCache* bc = bessel_for_current_device();
  if (!bc || !bc->ready) return fail(ABCMB_ERR_TABLES, "abcmb_los_vjp: Bessel tables not uploaded");
  if (ls.idx_min < 0 || ls.idx_max >= bc->dev.n_l) return fail(ABCMB_ERR_ARG, "abcmb_los_vjp: l index range");
  int max_nk = 0;
  for (int c = 0; c < n_cosmo; ++c) max_nk = cosmo_host[c].nk > max_nk ? cosmo_host[c].nk : max_nk;
  if (max_nk < 4) return fail(ABCMB_ERR_ARG, "abcmb_los_vjp: k grid");
  const int64_t need = abcmb::los_vjp_workspace_bytes(n_cosmo, max_nk, ls.nkt, ls.idx_max - ls.idx_min + 1, ls.n_save,
                                                      ls.l_max - ls.l_min + 1);
  if (!workspace_dev || workspace_bytes < need) return fail(ABCMB_ERR_WORKSPACE, "abcmb_los_vjp: workspace");
  cudaError_t e = abcmb::launch_los_vjp(n_cosmo, cosmo_dev, cosmo_host, tables_dev, k_dev, pt_dev, kt_dev, ls,
                                        ls.n_save, bc->dev, cl_bar_dev, pt_bar_dev, param_bar_dev, workspace_dev,
                                        static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_los_vjp");
  return ABCMB_OK;
}

int abcmb_cl_spline(int n_cosmo, const double* cl_raw_dev, int idx_min, int n_ell_tab, int l_min, int l_max,
                    double* cl_dev, void* stream) {
  if (n_cosmo <= 0 || n_cosmo > 65535 || !cl_raw_dev || !cl_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_cl_spline: bad argument");
  if (l_min != 2 || l_max < l_min || n_ell_tab < 4)
    return fail(ABCMB_ERR_ARG, "abcmb_cl_spline: need l_min == 2 <= l_max and at least 4 tabulated l");
  BesselCache* bc = bessel_for_current_device();
  if (!bc || !bc->ready) return fail(ABCMB_ERR_TABLES, "abcmb_cl_spline: Bessel tables not uploaded");
  if (idx_min < 0 || idx_min + n_ell_tab > bc->dev.n_l) return fail(ABCMB_ERR_ARG, "abcmb_cl_spline: l index range");
  cudaError_t e = abcmb::launch_cl_spline(n_cosmo, cl_raw_dev, idx_min, n_ell_tab, l_min, l_max, bc->dev, cl_dev,
                                          static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_cl_spline");
  return ABCMB_OK;
}

static bool lens_settings_ok(int n_cosmo, const abcmb_lens_settings* s) {
  return s && n_cosmo > 0 && n_cosmo <= 65535 && s->l_max >= 2 && s->l_lens >= s->l_max && s->n_mu >= 2 &&
         s->n_lna >= 3 && s->n_save >= 2 && s->max_nk >= 1;
}

int64_t abcmb_lens_workspace_size(int n_cosmo, const abcmb_lens_settings* settings) {
  if (!lens_settings_ok(n_cosmo, settings)) return fail(ABCMB_ERR_ARG, "abcmb_lens_workspace_size: bad settings");
  return abcmb::lens_workspace_bytes(n_cosmo, *settings);
}

int abcmb_lens_forward(int n_cosmo, const abcmb_cosmo* cosmo_dev, const abcmb_lens_cosmo* lens_dev,
                       const double* tables_dev, const double* k_dev, const double* pt_dev, const double* mu_dev,
                       const double* w_dev, const double* cl_unlensed_dev, const abcmb_lens_settings* settings,
                       double* clpp_dev, double* cl_dev, void* workspace_dev, int64_t workspace_bytes,
                       void* stream) {
  if (!cosmo_dev || !lens_dev || !tables_dev || !k_dev || !pt_dev || !mu_dev || !w_dev || !cl_unlensed_dev ||
      !clpp_dev || !cl_dev)
    return fail(ABCMB_ERR_ARG, "abcmb_lens_forward: null argument");
  if (!lens_settings_ok(n_cosmo, settings))
    return fail(ABCMB_ERR_ARG, "abcmb_lens_forward: settings (need 2 <= l_max <= l_lens, n_mu >= 2, n_lna >= 3)");
  const int64_t need = abcmb::lens_workspace_bytes(n_cosmo, *settings);
  if (!workspace_dev || workspace_bytes < need) return fail(ABCMB_ERR_WORKSPACE, "abcmb_lens_forward: workspace");
  cudaError_t e = abcmb::launch_lens(n_cosmo, cosmo_dev, lens_dev, tables_dev, k_dev, pt_dev, mu_dev, w_dev,
                                     cl_unlensed_dev, *settings, clpp_dev, cl_dev, workspace_dev,
                                     static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "abcmb_lens_forward");
  return ABCMB_OK;
}

/* Tuning knob: warps per block of the perturbation kernel (1..4; the
 * kernel is compiled for at most 128 threads per block). */
int abcmb_set_pert_warps_per_block(int w) {
  if (w < 1 || w > 4) return fail(ABCMB_ERR_ARG, "warps per block must be 1..4");
  g_warps_per_block = w;
  return ABCMB_OK;
}

/* Tuning knob: which instantiation of the perturbation kernel runs (0 =
 * by queue length, 1 = two blocks per SM, 2 = three blocks per SM). */
int abcmb_set_pert_variant(int v) {
  if (v < 0 || v > 2) return fail(ABCMB_ERR_ARG, "perturbation kernel variant must be 0, 1 or 2");
  g_pert_variant = v;
  return ABCMB_OK;
}

/* Tuning knob: warps per block of the tangent kernel (0 = the count with the
 * most resident warps, else 1..4). */
int abcmb_set_pert_tangent_warps_per_block(int w) {
  if (w < 0 || w > 4) return fail(ABCMB_ERR_ARG, "tangent warps per block must be 0..4");
  g_pert_tangent_warps = w;
  return ABCMB_OK;
}

/* Per-phase cycle counts of the perturbation kernel (a library built with
 * ABCMB_PHASE_CLOCKS only). */
int abcmb_pert_phase_clocks(uint64_t* cycles, int reset) {
  if (!cycles) return fail(ABCMB_ERR_ARG, "abcmb_pert_phase_clocks: null argument");
  const int rc = abcmb::pert_phase_clocks(reinterpret_cast<unsigned long long*>(cycles), reset);
  if (rc == -1) return fail(ABCMB_ERR_ARG, "abcmb_pert_phase_clocks: library built without ABCMB_PHASE_CLOCKS");
  if (rc != 0) return fail(ABCMB_ERR_CUDA, "abcmb_pert_phase_clocks: device read");
  return ABCMB_OK;
}

/* Grid size of the last perturbation launch (diagnostics). */
int abcmb_last_pert_grid(void) { return g_last_grid; }

}  // extern "C"
