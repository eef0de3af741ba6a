// mcrt_b200.cu -- C ABI of the B200 photon-packet engine (include/mcrt_b200.h).
//
// Host side: one context per device holds the model in the transport layout
// of mcrt_device.cuh, the FP64 device tallies, and launches the transport
// kernels (mcrt_fp64.cu / mcrt_mixed.cu) and the Lucy temperature kernels
// below.  Nothing here falls back to the CPU: every call that cannot run on
// the GPU returns an error code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "mcrt_device.cuh"

namespace mcrt {
// transport launchers (mcrt_fp64.cu, mcrt_mixed.cu)
cudaError_t launch_transport_fp64(const LaunchParams& p, int grid, cudaStream_t s);
cudaError_t launch_transport_mixed(const LaunchParams& p, int grid, cudaStream_t s);
cudaError_t launch_diffusion_finalize(const DevModel& m, const int32_t* ndiff, const double* tdust0, double* tdust,
                                      double nphot, cudaStream_t s);
int transport_fp64_blocks_per_sm();
cudaError_t launch_transport_sched_fp64(const LaunchParams& p, int grid, cudaStream_t s);
int transport_sched_fp64_blocks_per_sm();
cudaError_t launch_peel_fp64(const LaunchParams& p, unsigned long long* next_item, int grid, cudaStream_t s);
int peel_fp64_blocks_per_sm();
cudaError_t launch_peel_mixed(const LaunchParams& p, unsigned long long* next_item, int grid, cudaStream_t s);
int peel_mixed_blocks_per_sm();
int transport_mixed_blocks_per_sm();
cudaError_t launch_wave_init(const WaveArgs& w, cudaStream_t s);
cudaError_t launch_wave_event_fp64(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s);
cudaError_t launch_wave_walk_fp64(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s);
int wave_event_fp64_blocks_per_sm();
int wave_walk_fp64_blocks_per_sm();
cudaError_t launch_wave_event_mixed(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s);
cudaError_t launch_wave_walk_mixed(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s);
int wave_event_mixed_blocks_per_sm();
int wave_walk_mixed_blocks_per_sm();
cudaError_t launch_wave_tail_fp64(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s);
cudaError_t launch_wave_tail_mixed(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s);
int wave_tail_fp64_blocks_per_sm();
int wave_tail_mixed_blocks_per_sm();
cudaError_t launch_batch_fp64(const LaunchParams* params, const BatchItem* items, int64_t nitems,
                              unsigned long long* item_next, unsigned long long* chunk_next, int32_t event_batch,
                              int grid, cudaStream_t s);
cudaError_t launch_batch_mixed(const LaunchParams* params, const BatchItem* items, int64_t nitems,
                               unsigned long long* item_next, unsigned long long* chunk_next, int32_t event_batch,
                               int grid, cudaStream_t s);
int batch_fp64_blocks_per_sm();
int batch_mixed_blocks_per_sm();
cudaError_t launch_setemiss(const SetemissArgs& a, double* tmp, cudaStream_t s);
}  // namespace mcrt

using namespace mcrt;

struct mcrt_ctx {
  mcrt_config cfg{};
  int device = 0;
  int nsm = 148;
  int precision = MCRT_PREC_FP64;
  int schedule = MCRT_SCHED_WAVE;
  int event_batch = 16;
  int wave_batch = 4;
  // wavefront pool
  int64_t wave_pool = 1 << 21;
  int64_t wave_jobs = 0;              // peel-off job queue capacity asked for (0: default)
  int64_t wave_tail = -1;             // tail launch at <= this many live packets (<0: 8 per tail lane, 0: never)
  // device-driven wavefront loop (mcrt_set_wave_loop): the graph captured
  // for the last packet range and the launch parameters it was captured with
  int32_t wave_device_loop = 1;
  cudaGraph_t wl_graph = nullptr;
  cudaGraphExec_t wl_exec = nullptr;
  cudaStream_t wl_body = nullptr;
  LaunchParams wl_params;
  WaveArgs wl_w;
  unsigned long long wl_tail = 0, wl_max = 0;
  int64_t wl_npk = 0;
  int64_t *d_block0 = nullptr, *h_block0 = nullptr;   // the iteration's first random block, read by the graph
  WaveCtl* h_ctl = nullptr;
  int64_t wave_cap = 0;
  WaveRec *d_recs = nullptr;
  int32_t *d_walkq = nullptr, *d_evq = nullptr;
  WaveCtl *d_wctl = nullptr;
  unsigned long long *h_wctl = nullptr;   // pinned: n_front, n_back, packets started, peel jobs, walks, crossings
  int64_t last_waves = 0;
  // device time per kernel class of the last wavefront run: walk, event, tail, peel-off
  cudaEvent_t kt_ev[4][2] = {};
  bool kt_pending[4] = {};
  double kt_ms[4] = {};
  int64_t kt_walks = 0, kt_walk_cross = 0, kt_launch[4] = {};
  // path-replay adjoint buffers (mcrt_adjoint)
  AdjointArgs adj{};
  int64_t adj_rec_used = 0;
  int64_t adj_npk_cap = 0;
  unsigned long long *d_adj_nlist = nullptr;
  void *d_adj_tmp = nullptr;
  size_t adj_tmp_bytes = 0;
  int64_t adj_chunk = (int64_t)1 << 25;   // packets per adjoint chunk (halved when its records reach 2^31)
  double* d_adj_sum = nullptr;        // [ncell*10 + 1] gradient and objective summed over chunks
  int64_t adj_sort_cap = 0;           // capacity of the sorted copies (skey, sc) and the sort scratch
  // control variate of the replay (mcrt_set_adjoint_baseline)
  int32_t cv_nfb = 0, cv_ndir = 1;
  int64_t cv_pilot = 0;
  double cv_min_count = 16.0;
  int64_t cv_cap = 0;                 // entries of cv_tab / cv_sum / cv_cnt
  double *cv_tab = nullptr, *cv_sum = nullptr, *cv_cnt = nullptr;
  bool have_grid = false, have_tables = false;
  bool have_acc = false;              // ravearr / Ldint / hdisk uploaded (accretion packets)
  bool have_isrf = false;             // ISRF sampling table uploaded (external-illumination packets)
  bool have_draine = false;           // small-grain emission spectra uploaded
  bool have_sg = false;               // the grid holds small-grain components (ids 5-8)
  int32_t imean_max = 0;              // largest imean of the grid (0: none given)
  int32_t *d_imean = nullptr;
  std::string err;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  int64_t ncell = 0, nsed = 0, npsed = 0, nimg = 0;
  int64_t uploads = 0;                // grid, table and log-buffer changes so far (batch graphs hold their pointers)
  DevModel dm{};
  DevTallies dt{};
  std::vector<void*> allocs;         // device buffers owned by the context
  // model buffers
  double *d_walls = nullptr;
  CellRec *d_cells = nullptr;
  CellRecF *d_cellsf = nullptr;       // FP32 cells of the mixed walk
  unsigned char *d_walk32 = nullptr;  // FP32 walk tables: tcone | pplane
  double *d_tdust = nullptr, *d_vcell = nullptr;
  double *d_tdust0 = nullptr;         // tdust at the start of the iteration (read by the transport)
  double last_nphot_diff = 1.0;
  DevModel last_m{};                  // model view of the last run (mcrt_refresh_diffusion)
  bool have_last_run = false;
  double last_ns = 0.0;               // stellar packets of the whole iteration of the last run
  double *d_dens_thermal = nullptr;   // [ncell] density of the thermal component (tfinal)
  int32_t *d_idust3 = nullptr;        // [ncell] its opacity species (0 = none)
  int32_t *d_diffus = nullptr;
  // gas velocity field (tfinal's adiabatic and advective terms)
  bool have_vel = false;
  double *d_vel = nullptr;            // [3][ncell] vrarr, vthetarr, divvarr
  int32_t *d_tflag = nullptr;         // [ncell] bit 0: disk ids 1/2/9, bit 1: ids 4/10 (tfinal's gradient rules)
  double *d_rave = nullptr;           // [nrg] cell-centre radii (ravearr or the wall midpoints)
  std::vector<int32_t> h_diffus;      // diffusion flags (convergence statistics)
  bool h_diffus_stale = false;        // mcrt_setdiffus changed d_diffus without copying it here
  void *d_scratch = nullptr;          // grow-only scratch of the per-iteration calls (tfinal, download)
  size_t scratch_bytes = 0;
  // tables
  int32_t *d_nlambda = nullptr;
  double *d_tabs = nullptr;
  int64_t *d_jump = nullptr;
  // tallies
  void *d_tally = nullptr;
  size_t tally_bytes = 0;
  unsigned long long *d_next = nullptr;    // [0] packets, [1] peel jobs, [2] peel items
  PeelJob *d_jobs = nullptr;
  int64_t job_cap = 0;
  double *d_job_nub = nullptr;        // [job_cap] packet frequency per job (filter-band images)
  int64_t job_nub_cap = 0;
  int64_t nimgb = 0;                  // filter-band image size (0: off)
  int64_t nims = 0;                   // nested image size per Stokes parameter (0: off)
  float *d_levels = nullptr;          // [sparse_nlev] nested image half sizes
  int32_t *d_nfpts = nullptr;         // [nfilt] points per filter curve
  int64_t chunk_packets = 1 << 20;
  int32_t *d_err = nullptr;
  mcrt_packet_log *d_log = nullptr;
  int64_t nlog = 0;
  double prev_sig = -1.0;
  cudaEvent_t marks[16] = {};
  void *d_flush = nullptr;
  int64_t off_Tint = 0, off_kappap = 0;   // offsets of Tint/kappap in d_tabs (tfinal)
  int64_t off_kappar = -1;              // offset of kappar in d_tabs (setdiffus), -1 when not uploaded
  double *d_sd_tdave = nullptr;         // setdiffus: [ncell] tdave, [nrg*ntg] marks, [ncell] flags out
  uint8_t *d_sd_mark = nullptr;
  int32_t *d_sd_out = nullptr;
  std::vector<double> h_rarr;
  std::vector<int32_t> species_grid;  // per species: first species with a bit-identical wavelength column
  double* noalloc_scratch = nullptr;   // device address of g_tfinal_scratch (mcrt_update_temperature_noalloc)
  // watchdogs (mcrt_set_limits)
  int64_t walk_limit = 50000000;       // crossings of one walk before it is given up as a geometry failure
  int64_t wave_limit = 400000000;      // waves of one wavefront loop before the call returns MCRT_ERR_TIMEOUT
  double geom_fraction = 1.0e-6;       // lost packets (geometry failures) per packet that make a run return MCRT_ERR_GEOM
  unsigned long long* h_geom = nullptr;   // pinned: the geometry-failure counter before and after a run
};

namespace {

int fail(mcrt_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <class T>
int dalloc(mcrt_ctx* ctx, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "cudaMalloc(%zu): %s", n * sizeof(T), cudaGetErrorString(e));
  ctx->allocs.push_back(q);
  *p = (T*)q;
  return MCRT_OK;
}

void dfree(mcrt_ctx* ctx, void* p) {
  if (!p) return;
  auto it = std::find(ctx->allocs.begin(), ctx->allocs.end(), p);
  if (it != ctx->allocs.end()) ctx->allocs.erase(it);
  cudaFree(p);
}

// Scratch of the calls a driver makes every iteration (the temperature
// update, the tally download): one buffer that only grows, so after the
// first iteration they allocate and free nothing (cudaFree would also wait
// for the whole device).  One user at a time: each call finishes with it
// before it returns.
template <class T>
int scratch(mcrt_ctx* ctx, T** p, size_t n) {
  const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  if (ctx->scratch_bytes < bytes) {
    if (ctx->d_scratch) dfree(ctx, ctx->d_scratch);
    ctx->d_scratch = nullptr;
    ctx->scratch_bytes = 0;
    const int rc = dalloc(ctx, (char**)&ctx->d_scratch, bytes);
    if (rc) return rc;
    ctx->scratch_bytes = bytes;
  }
  *p = static_cast<T*>(ctx->d_scratch);
  return MCRT_OK;
}

int64_t mulmod_h(int64_t a, int64_t b, int64_t m) {
  return (int64_t)(((unsigned __int128)a * (unsigned __int128)b) % (unsigned __int128)m);
}

void zetainit_h(double* inczeta) {   // random.f90:227-245
  for (int i = 0; i < MCRT_IZMAX; ++i) inczeta[i] = 0.0;
  for (int j = MCRT_IZMAX; j >= 1; --j) {
    double temp = 1.0 / (double)(j * j * j * j);
    for (int i = MCRT_IZMAX; i >= j; --i) inczeta[i - 1] += temp;
  }
}

const bool kIsSg[MCRT_NDG2] = {false, false, false, false, true, true, true, true, false, false};  // grid_mod_5.f90:20

}  // namespace

// ---------------------------------------------------------------- tfinal --
namespace mcrt {

__device__ __forceinline__ double p4(double x) { double x2 = x * x; return x2 * x2; }

// dusttemp (dusttemp_5.f90:8-152).
// The emission side of dusttemp's balance at table temperature i:
// Tint^4 kappa_P plus, with a gas velocity field, the adiabatic term
// (k/4/sigt/2.3/mH)/kappa_V/11605^3 * Tint*divv/rstar/rsol and the advective
// term (3k/8/sigt/2.3/mH)/kappa_V/11605^3 * (vr gradtr + vthet gradtt)/
// rstar/rsol (dusttemp_5.f90:42-53).  The factors of Tint and the constant
// term are formed once per cell (dust_vel); the oracle forms them the same way.
struct DustVel {
  double adi, adv;           // adiabatic term per unit Tint; advective term
  bool on;
};
__device__ __forceinline__ DustVel dust_vel(double kv, double rstar, double divv, double vgrad) {
  constexpr double kB = 1.3806503e-16, sigt = 5.670400e-5, mH = 1.67262158e-24, rsol = 6.9598e10;
  const double p3 = 11605.0 * 11605.0 * 11605.0;
  const double c1 = kB / 4.0 / sigt / 2.3 / mH, c2 = kB * 3.0 / 8.0 / sigt / 2.3 / mH;
  DustVel v;
  v.adi = __ddiv_rn(__ddiv_rn(__dmul_rn(__ddiv_rn(__ddiv_rn(c1, kv), p3), divv), rstar), rsol);
  v.adv = __ddiv_rn(__ddiv_rn(__dmul_rn(__ddiv_rn(__ddiv_rn(c2, kv), p3), vgrad), rstar), rsol);
  v.on = true;
  return v;
}
__device__ __forceinline__ double kappa_T(const double* Tint, const double* kp, int i, double kv, double rstar,
                                          const DustVel& v) {
  const double emi = __dmul_rn(p4(Tint[i]), kp[i]);
  if (!v.on) return emi;
  return __dadd_rn(__dadd_rn(emi, __dmul_rn(v.adi, Tint[i])), v.adv);
}

__device__ double dusttemp_dev(const double* Tint, const double* kp, int nT, double kv, double na, int nphot,
                               double mcell, double rstar, double tstar, const DustVel& v = DustVel{0.0, 0.0, false}) {
  const double Tmax = 199999.0, T01 = 0.1 / 11605.0;
  double Td = T01;
  if (!(mcell > 0.0)) return Td;
  double abs_ = p4(tstar) * (na * 3.1415926535897932384626433 * rstar * rstar) / ((double)nphot * kv);
  abs_ = abs_ * (6.9598e10 * 6.9598e10) / p4(mcell);
  if (na == 0.0) return T01;
  double minkap = kappa_T(Tint, kp, 0, kv, rstar, v), maxkap = minkap;
  int mini = 1, maxi = 1;
  for (int i = 1; i <= nT; ++i) {
    const double k = kappa_T(Tint, kp, i - 1, kv, rstar, v);
    if (minkap > k) { minkap = k; mini = i; }
    if (maxkap < k) { maxkap = k; maxi = i; }
  }
  if (maxkap < abs_) Td = fmax(fmin(Tint[maxi - 1], Tmax / 11605.0), T01);
  if (minkap > abs_) Td = fmax(fmin(Tint[mini - 1], Tmax / 11605.0), T01);
  if (mini < maxi) {
    for (int i = mini; i <= maxi - 1; ++i) {
      const double kl = kappa_T(Tint, kp, i - 1, kv, rstar, v), ku = kappa_T(Tint, kp, i, kv, rstar, v);
      if (kl < abs_ && ku >= abs_) {
        const double Tl = Tint[i - 1], Tu = Tint[i];
        Td = Tl + (Tu - Tl) / (ku - kl) * (abs_ - kl);
        return fmax(fmin(Td, Tmax / 11605.0), T01);
      }
    }
  } else {
    for (int i = maxi; i <= mini - 1; ++i) {
      const double kl = kappa_T(Tint, kp, i - 1, kv, rstar, v), ku = kappa_T(Tint, kp, i, kv, rstar, v);
      if (kl > abs_ && ku <= abs_) {
        const double Tl = Tint[i - 1], Tu = Tint[i];
        Td = Tl + (Tu - Tl) / (ku - kl) * (abs_ - kl);
        return fmax(fmin(Td, Tmax / 11605.0), T01);
      }
    }
  }
  return Td;
}

struct TfinalArgs {
  int nrg, ntg, npg, nT, nphot, maxii;
  double rstar, tstar;
  const double *Tint, *kappap, *kappav, *dtauabs, *vcell, *dens, *tdust;
  const int32_t *idust3, *diffus;
  const double *told;   // tdave of the previous iteration
  double *tnew;         // scratch: new upper-hemisphere values
  double *tdave;        // result
  // gas velocity field (null vr: at rest) and the pass scratch of its
  // temperature gradients
  const double *vr, *vth, *divv;        // [ncell]
  const double *rarr, *thetarr, *rave;  // walls; cell-centre radii [nrg-1]
  const int32_t *tflag;                 // [ncell] bit 0: densarr ids 1, 2 or 9 > 0; bit 1: ids 4 or 10 > 0
  double *tsm;                          // [nrg*ntg] smoothed temperature (phi slice 1)
  double *gtr, *gtt, *gtr2, *gtt2;      // [nrg*ntg] gradients, raw and smoothed
  double *acc;                          // [ncell] sum of passes 11..maxii
};

// tfinal_5_test1.f90:206-256: upper-hemisphere cells of phi slice 1.  The
// thermal component of the cell (id) fixes the species; the mirror cell
// ntg-it contributes its density of the same component (zero if absent).
__global__ void tfinal_cells(TfinalArgs a) {
  const int nu = (a.ntg - 1) / 2;
  const int64_t n = (int64_t)(a.nrg - 1) * nu;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % (a.nrg - 1)) + 1;
    const int it = (int)(k / (a.nrg - 1)) + 1;
    const int itm = a.ntg - it;
    const int64_t c = (ir - 1) + (int64_t)a.nrg * (it - 1);
    const int64_t cm = (ir - 1) + (int64_t)a.nrg * (itm - 1);
    double td = 0.1 / 11605.0;
    const int sp = a.idust3[c];
    if (sp > 0) {
      if (!a.diffus[c]) {
        const double dm = (a.idust3[cm] == sp) ? a.dens[cm] : 0.0;
        const double m1 = pow(a.dens[c] * a.vcell[c], 0.25);
        const double m2 = pow(dm * a.vcell[c], 0.25);
        const double* kp = a.kappap + (int64_t)a.nT * (sp - 1);
        const double t1 = dusttemp_dev(a.Tint, kp, a.nT, a.kappav[sp - 1], a.dtauabs[c], a.nphot, m1, a.rstar, a.tstar);
        const double t2 = dusttemp_dev(a.Tint, kp, a.nT, a.kappav[sp - 1], a.dtauabs[cm], a.nphot, m2, a.rstar, a.tstar);
        td = (t1 + t2) / 2.0;
      } else {
        td = (a.tdust[c] + a.tdust[cm]) / 2.0;
      }
      if (td * 11605.0 >= 199999.0) td = 199999.0 / 11605.0;
    }
    a.tnew[c] = td;
  }
}

// tfinal_5_test1.f90:267-293: mirror to the lower hemisphere and the other
// phi slices, then the average over passes 11..20 (all passes give the same
// value for a zero velocity field; the sum is formed term by term as in the
// reference).  Cells outside the loops keep their previous value.
__global__ void tfinal_mirror(TfinalArgs a) {
  const int64_t n = (int64_t)a.nrg * a.ntg * a.npg;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % a.nrg) + 1;
    const int it = (int)((k / a.nrg) % a.ntg) + 1;
    const int ip = (int)(k / ((int64_t)a.nrg * a.ntg)) + 1;
    double v = a.told[k];
    if (ir <= a.nrg - 1 && it <= a.ntg - 1 && (ip == 1 || (a.npg > 2 && ip <= a.npg - 1))) {
      const int src_it = (it >= (a.ntg + 1) / 2) ? a.ntg - it : it;
      v = a.tnew[(ir - 1) + (int64_t)a.nrg * (src_it - 1)];
    }
    if (a.maxii > 10) {
      double acc = 0.0;
      for (int i = 0; i < a.maxii - 10; ++i) acc += v;
      v = acc / (double)(a.maxii - 10);
    }
    a.tdave[k] = v;
  }
}

// ---- tfinal with a gas velocity field: the passes of tfinal_5_test1.f90
// (maxii of them, averaged over passes 11..maxii when maxii > 10).  Every
// pass smooths the temperature over 31 x 31 cells, forms the radial and
// polar gradients, smooths them over 31 radial cells, and solves dusttemp
// with the adiabatic and advective terms cell by cell.  The kernels work on
// phi slice 1 (the model is axisymmetric in this part of the reference).

// Box limits of the reference (width w each side, clipped to 1..n-1).
__device__ __forceinline__ void tf_box(int i, int w, int n, int& lo, int& hi) {
  if (i > w && i < n - w) { lo = i - w; hi = i + w; }
  else if (i <= w) { lo = 1; hi = i + w; }
  else { lo = i - w; hi = n - 1; }
}

// tfinal_5_test1.f90:65-106: smoothed temperature of every cell.
__global__ void tfv_smooth(TfinalArgs a) {
  const double T01 = 0.1 / 11605.0;
  const int64_t n = (int64_t)a.nrg * a.ntg;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % a.nrg) + 1, it = (int)(k / a.nrg) + 1;
    if (ir > a.nrg - 1 || it > a.ntg - 1) { a.tsm[k] = 0.0; continue; }
    int r1, r2, t1, t2;
    tf_box(ir, 15, a.nrg, r1, r2);
    tf_box(it, 15, a.ntg, t1, t2);
    double tot = 0.0;
    int nsm = 0;
    for (int iir = r1; iir <= r2; ++iir)
      for (int iit = t1; iit <= t2; ++iit) {
        const double v = a.tdave[(iir - 1) + (int64_t)a.nrg * (iit - 1)];
        if (v > T01) { ++nsm; tot = __dadd_rn(tot, v); }
      }
    if (nsm > 0) tot = __ddiv_rn(tot, (double)nsm);
    if (a.tdave[(ir - 1) + (int64_t)a.nrg * (it - 1)] == T01) tot = T01;
    a.tsm[k] = tot;
  }
}

// tfinal_5_test1.f90:108-135: the raw gradients of cell (ir,it) before the
// outer-edge copy; zero in disk cells.
__device__ __forceinline__ void tfv_grad_cell(const TfinalArgs& a, int ir, int it, double& gr, double& gt) {
  const int nrg = a.nrg;
  auto T = [&](int i, int j) { return a.tsm[(i - 1) + (int64_t)nrg * (j - 1)]; };
  const double rad = a.rave[ir - 1];
  const double dr = __dsub_rn(a.rarr[ir], a.rarr[ir - 1]);
  const double dt = __dsub_rn(a.thetarr[it], a.thetarr[it - 1]);
  gr = __ddiv_rn(__dsub_rn(T(ir + 1, it), T(ir, it)), dr);
  if (it <= 15) gr = __ddiv_rn(__dsub_rn(T(ir + 1, 16), T(ir, 16)), dr);
  gt = __ddiv_rn(__ddiv_rn(__dsub_rn(T(ir, it + 1), T(ir, it)), dt), rad);
  if (it <= 15) gt = __ddiv_rn(__ddiv_rn(__dsub_rn(T(ir, 17), T(ir, 16)), rad), __dsub_rn(a.thetarr[16], a.thetarr[15]));
}

__global__ void tfv_grad(TfinalArgs a, int first_pass) {
  const int64_t n = (int64_t)a.nrg * a.ntg;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % a.nrg) + 1, it = (int)(k / a.nrg) + 1;
    double gr = 0.0, gt = 0.0;
    if (!first_pass && ir <= a.nrg - 1 && it <= a.ntg - 1) {
      const int src = a.nrg - 17;               // ir >= nrg-widthr-1 copies row nrg-widthr-2 (its final value)
      if (ir >= a.nrg - 16) {
        tfv_grad_cell(a, src, it, gr, gt);
        if (a.tflag[(src - 1) + (int64_t)a.nrg * (it - 1)] & 1) { gr = 0.0; gt = 0.0; }
      } else {
        tfv_grad_cell(a, ir, it, gr, gt);
      }
      if (a.tflag[k] & 1) { gr = 0.0; gt = 0.0; }
    }
    a.gtr[k] = gr;
    a.gtt[k] = gt;
  }
}

// tfinal_5_test1.f90:145-194: gradients smoothed over 31 radial cells; in
// cells of densarr ids 4/10 the radial one is the mean of the negative ones.
__global__ void tfv_smooth_grad(TfinalArgs a) {
  const int64_t n = (int64_t)a.nrg * a.ntg;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % a.nrg) + 1, it = (int)(k / a.nrg) + 1;
    double gr = 0.0, gt = 0.0;
    if (ir <= a.nrg - 1 && it <= a.ntg - 1) {
      int r1, r2;
      tf_box(ir, 15, a.nrg, r1, r2);
      const int64_t row = (int64_t)a.nrg * (it - 1);
      if (a.tflag[k] & 2) {
        int nsm = 0;
        for (int iir = r1; iir <= r2; ++iir) {
          const double v = a.gtr[(iir - 1) + row];
          if (v < 0.0) { ++nsm; gr = __dadd_rn(gr, v); }
        }
        if (nsm > 0) gr = __ddiv_rn(gr, (double)nsm);
      } else {
        for (int iir = r1; iir <= r2; ++iir) gr = __dadd_rn(gr, a.gtr[(iir - 1) + row]);
        gr = __ddiv_rn(__ddiv_rn(gr, (double)(r2 - r1 + 1)), 1.0);
      }
      for (int iir = r1; iir <= r2; ++iir) gt = __dadd_rn(gt, a.gtt[(iir - 1) + row]);
      gt = __ddiv_rn(__ddiv_rn(gt, (double)(r2 - r1 + 1)), 1.0);
    }
    a.gtr2[k] = gr;
    a.gtt2[k] = gt;
  }
}

// tfinal_5_test1.f90:206-243 with the velocity terms: the upper-hemisphere
// cells of slice 1, in place in tdave (each reads only its own cells).
__global__ void tfv_cells(TfinalArgs a) {
  const int nu = (a.ntg - 1) / 2;
  const int64_t n = (int64_t)(a.nrg - 1) * nu;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % (a.nrg - 1)) + 1;
    const int it = (int)(k / (a.nrg - 1)) + 1;
    const int itm = a.ntg - it;
    const int64_t c = (ir - 1) + (int64_t)a.nrg * (it - 1);
    const int64_t cm = (ir - 1) + (int64_t)a.nrg * (itm - 1);
    double td = 0.1 / 11605.0;
    const int sp = a.idust3[c];
    if (sp > 0) {
      if (!a.diffus[c]) {
        const double dm = (a.idust3[cm] == sp) ? a.dens[cm] : 0.0;
        const double m1 = pow(a.dens[c] * a.vcell[c], 0.25);
        const double m2 = pow(dm * a.vcell[c], 0.25);
        const double* kp = a.kappap + (int64_t)a.nT * (sp - 1);
        const double gr = a.gtr2[c], gt = a.gtt2[c];
        const double kv = a.kappav[sp - 1];
        const DustVel v1 = dust_vel(kv, a.rstar, a.divv[c], __dadd_rn(__dmul_rn(a.vr[c], gr), __dmul_rn(a.vth[c], gt)));
        const DustVel v2 = dust_vel(kv, a.rstar, a.divv[cm], __dadd_rn(__dmul_rn(a.vr[cm], gr), __dmul_rn(a.vth[cm], gt)));
        const double t1 = dusttemp_dev(a.Tint, kp, a.nT, a.kappav[sp - 1], a.dtauabs[c], a.nphot, m1, a.rstar, a.tstar, v1);
        const double t2 = dusttemp_dev(a.Tint, kp, a.nT, a.kappav[sp - 1], a.dtauabs[cm], a.nphot, m2, a.rstar, a.tstar, v2);
        td = (t1 + t2) / 2.0;
      } else {
        td = (a.tdust[c] + a.tdust[cm]) / 2.0;
      }
      if (td * 11605.0 >= 199999.0) td = 199999.0 / 11605.0;
    }
    a.tdave[c] = td;
  }
}

// tfinal_5_test1.f90:267-288: mirror to the lower hemisphere and the other
// phi slices (in place), and the pass sum of passes 11..maxii.
__global__ void tfv_mirror(TfinalArgs a, int accumulate, int first_acc) {
  const int64_t n = (int64_t)a.nrg * a.ntg * a.npg;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % a.nrg) + 1;
    const int it = (int)((k / a.nrg) % a.ntg) + 1;
    const int ip = (int)(k / ((int64_t)a.nrg * a.ntg)) + 1;
    double v = a.tdave[k];
    if (ir <= a.nrg - 1 && it <= a.ntg - 1 && (ip == 1 || (a.npg > 2 && ip <= a.npg - 1))) {
      const int src_it = (it >= (a.ntg + 1) / 2) ? a.ntg - it : it;
      if (src_it != it || ip != 1) v = a.tdave[(ir - 1) + (int64_t)a.nrg * (src_it - 1)];
    }
    if (ip != 1 || it >= (a.ntg + 1) / 2) a.tdave[k] = v;      // upper cells of slice 1 are the sources
    if (accumulate) a.acc[k] = first_acc ? v : __dadd_rn(a.acc[k], v);
  }
}

__global__ void tfv_average(TfinalArgs a, int passes) {
  const int64_t n = (int64_t)a.nrg * a.ntg * a.npg;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    a.tdave[k] = a.acc[k] / (double)passes;
}

// gridset_5_model13new.f90:1855-1866: tdust for the next iteration
__global__ void tdust_from_tdave(int64_t n, const double* tdave, const int32_t* diffus, const int32_t* idust3,
                                 const CellRec* cells, double* tdust) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    double t = diffus[k] ? 0.1 / 11605.0 : tdave[k];
    if (cell_n(cells[k].meta) == 0) t = 0.1 / 11605.0;
    tdust[k] = t;
  }
}

// ---- setdiffus (setdiffus_5.f90:1-132) -------------------------------------
struct SetdiffusArgs {
  int nrg, ntg, npg, nT, iter;
  int nr0, nr1;                 // radii ir = nr0..nr1 are marched (rarr(ir) < rmaxd, ir <= nrg-1)
  double rmincgs;
  const double *rarr, *thetarr, *hdisk, *kappav, *kappar, *lTint;
  const double* tdave;          // [ncell] temperature of the last tfinal
  const CellRec* cells;
  uint8_t* mark;                // [nrg*ntg] theta cell it of radius ir starts a diffusion run
};

// chiR (dust_5.f90:112-141): the Rosseland table of species sp interpolated
// in log T; an index outside the table is clamped to its end intervals.
__device__ double chiR_dev(const double* lTint, const double* kappar, int nT, double T, int sp) {
  const double lT = log(T);
  int k = (int)__ddiv_rn(__dmul_rn((double)(nT - 1), __dsub_rn(lT, lTint[0])), __dsub_rn(lTint[nT - 1], lTint[0])) + 1;
  k = min(max(k, 1), nT - 1);
  const double f = __ddiv_rn(__dsub_rn(lT, lTint[k - 1]), __dsub_rn(lTint[k], lTint[k - 1]));
  const double* kr = kappar + (int64_t)nT * (sp - 1);
  return __dadd_rn(__dmul_rn(__dsub_rn(1.0, f), kr[k - 1]), __dmul_rn(f, kr[k]));
}

// One thread per (ir, it) of the upper hemisphere: the march toward the
// pole (setdiffus_5.f90:57-94) that sums the Rosseland optical depth of the
// thermal components of slice ip = 1 until it reaches 1, then the mean-free
// path test against h/20.  mark = 1 where cell it starts a diffusion run.
__global__ void setdiffus_mark(SetdiffusArgs a) {
  const int nt = (a.ntg - 1) / 2 - 1;          // it = 2..(ntg-1)/2
  const int64_t n = (int64_t)(a.nr1 - a.nr0 + 1) * (nt > 0 ? nt : 0);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const int ir = a.nr0 + (int)(q / nt);
    const int it = 2 + (int)(q % nt);
    const double rad = a.rarr[ir - 1];
    const double zmr = a.hdisk[ir - 1];
    double tau = 0.0, tau1 = 0.0;
    int itt = it;
    while (tau < 1.0 && itt > 1) {
      const double dt = __dsub_rn(a.thetarr[itt], a.thetarr[itt - 1]);
      tau1 = tau;
      const int64_t c = (ir - 1) + (int64_t)a.nrg * (itt - 1);
      double tt = a.tdave[c];
      if (a.iter < 2) tt = fmax(tt, 50.0 / 11605.0);
      const CellRec r = a.cells[c];
      for (int k = 0; k < cell_n(r.meta); ++k) {
        const int id = cell_id(r.meta, k);      // findopac(.,id) = id
        if ((id >= 5 && id <= 8) || !(r.rho[k] > 0.0)) continue;   // small grains are not thermal
        double t = __dmul_rn(a.kappav[id - 1], a.rmincgs);
        t = __dmul_rn(t, chiR_dev(a.lTint, a.kappar, a.nT, tt, id));
        t = __dmul_rn(__dmul_rn(__dmul_rn(t, r.rho[k]), dt), rad);
        tau = __dadd_rn(tau, t);
      }
      itt = itt - 1;
    }
    double lmfp1;
    if (tau > 1.0)
      lmfp1 = __dmul_rn(__ddiv_rn(__dmul_rn(rad, __dsub_rn(a.thetarr[itt + 1], a.thetarr[itt])), __dsub_rn(tau, tau1)),
                        __dsub_rn(1.0, tau1));
    else
      lmfp1 = __dmul_rn(rad, __dsub_rn(a.thetarr[itt + 1], a.thetarr[itt]));
    const double lmfp = __dadd_rn(__dmul_rn(rad, __dsub_rn(a.thetarr[it], a.thetarr[itt + 1])), lmfp1);
    a.mark[(ir - 1) + (int64_t)a.nrg * (it - 1)] = (tau >= 1.0 && lmfp < zmr / 20.0) ? 1 : 0;
  }
}

// One thread per cell: a marked cell flags itself and every cell between it
// and the midplane (setdiffus_5.f90:96-101, diffdir -2), the lower
// hemisphere mirrors the upper one with diffdir +2 (:106-111), slice 1 is
// copied to every phi slice (:113-121); cells without a thermal component
// stay off (they have no temperature to diffuse).  Then gridset's reset
// (gridset_5_model13new.f90:1855-1866): tdust = tdave, 0.1 K in diffusion
// cells and in empty cells.  The cell records' flag bits, the flag array and
// both tdust copies are rewritten; out (optional) receives diffus | diffdir << 8.
__global__ void setdiffus_apply(SetdiffusArgs a, int massd_pos, CellRec* cells, int32_t* diffus, double* tdust,
                                double* tdust0, int32_t* out) {
  const int64_t n = (int64_t)a.nrg * a.ntg * a.npg;
  const int half = (a.ntg - 1) / 2;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % a.nrg) + 1;
    const int it = (int)((k / a.nrg) % a.ntg) + 1;
    const int ip = (int)(k / ((int64_t)a.nrg * a.ntg)) + 1;
    int on = 0, dd = 0;
    if (massd_pos && ir <= a.nrg - 1 && it <= a.ntg - 1 && ip <= (a.npg > 2 ? a.npg - 1 : 1)) {
      int src = it, sgn = -2;
      if (it >= (a.ntg + 1) / 2) { src = a.ntg - it; sgn = 2; }
      if (src >= 2 && src <= half)
        for (int j = 2; j <= src && !on; ++j) on = a.mark[(ir - 1) + (int64_t)a.nrg * (j - 1)];
      dd = on ? sgn : 0;
    }
    CellRec r = cells[k];
    if (!cell_thermal(r.flags)) { on = 0; dd = 0; }
    r.flags = (r.flags & ~31u) | (uint32_t)on | ((uint32_t)(dd + 8) << 1);
    cells[k].flags = r.flags;
    diffus[k] = on;
    double t = on ? 0.1 / 11605.0 : a.tdave[k];
    if (cell_n(r.meta) == 0) t = 0.1 / 11605.0;
    tdust[k] = t;
    tdust0[k] = t;
    if (out) out[k] = on | (dd << 8);
  }
}

// Convergence sums of tfinal_5_test1.f90:307-332 accumulated on the device:
// out[0..2] sums of |dT/T|, out[3..5] sums of (dT/T)^2, out[6..8] counts.
__global__ void tfinal_stats(int nrg, int ntg, const double* told, const double* tnew, const double* rarr,
                             double autors, const int32_t* diffus, double* out) {
  const int nu = (ntg - 1) / 2;
  const int64_t n = (int64_t)(nrg - 1) * nu;
  const double T01 = 0.1 / 11605.0;
  double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(k % (nrg - 1)) + 1;
    const int it = (int)(k / (nrg - 1)) + 1;
    const int64_t c = (ir - 1) + (int64_t)nrg * (it - 1);
    const double to = told[c], tn = tnew[c];
    const double d = (tn - to) / tn;
    if (tn != to && tn > T01 && to > T01) { a[0] += fabs(d); a[3] += d * d; a[6] += 1.0; }
    if (!diffus[c] && tn > T01 && to > T01) { a[1] += fabs(d); a[4] += d * d; a[7] += 1.0; }
    if (rarr[ir - 1] / autors < 5.0 && tn > T01 && to > T01) { a[2] += fabs(d); a[5] += d * d; a[8] += 1.0; }
  }
  for (int i = 0; i < 9; ++i) {
    double v = a[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(out + i, v);
  }
}

// Scratch of mcrt_update_temperature_noalloc: previous field, new upper
// hemisphere, result, and the nine convergence sums.  A file-scope device
// array, so that entry point needs no allocation; every process that loads
// the library holds it (3*524288+16 doubles, 12 MiB) on each device it uses.
constexpr int64_t kNoAllocMaxCells = 524288;
static __device__ __align__(256) double g_tfinal_scratch[3 * kNoAllocMaxCells + 16];

// Sorted adjoint records: the range [start, end) of each packet's records
// and the list of packets that have any (keys ~0 mark jobs without a
// contribution and sort last).
__global__ void adjoint_ranges(const unsigned long long* key, int64_t n, int64_t* start, int64_t* end, int32_t* list,
                               unsigned long long* nlist) {
  const unsigned long long none = ~0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = key[i];
    if (k == none) continue;
    const unsigned long long p = k >> kAdjEvBits;
    if (i == 0 || (key[i - 1] >> kAdjEvBits) != p) {
      start[p] = i;
      list[atomicAdd(nlist, 1ull)] = (int32_t)p;
    }
    if (i == n - 1 || key[i + 1] == none || (key[i + 1] >> kAdjEvBits) != p) end[p] = i + 1;
  }
}

// dst[i] += src[i]; kind 0: f64 -> f64, 1: i64 -> u64, 2: f32 -> f64, 3: i32 -> i32
__global__ void add_tally(int kind, const void* src, void* dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    switch (kind) {
      case 0: ((double*)dst)[i] += ((const double*)src)[i]; break;
      case 1: ((unsigned long long*)dst)[i] += (unsigned long long)((const long long*)src)[i]; break;
      case 2: ((double*)dst)[i] += (double)((const float*)src)[i]; break;
      default: ((int32_t*)dst)[i] += ((const int32_t*)src)[i]; break;
    }
  }
}

__global__ void add_counters(unsigned long long* cnt, unsigned long long waves, unsigned long long launches) {
  cnt[MCRT_C_WAVES] += waves;
  cnt[MCRT_C_LAUNCHES] += launches;
}

// Device-driven wavefront loop (a CUDA-graph WHILE node whose body is event
// launch, wave_loop_mid, walk launch, wave_loop_cond): the decisions the
// host loop of run_iteration_impl takes after each walk launch.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The loop kernels also time the launches between them: each adds the time
// since the previous stamp to its kernel class (the launch gaps included).
__global__ void wave_loop_start(WaveCtl* c) { c->t_last = global_ns(); }

__global__ void wave_loop_mid(WaveCtl* c) {
  const unsigned long long t = global_ns();
  c->ev_ns += t - c->t_last;
  c->t_last = t;
  c->n_front = 0;
  c->n_back = 0;
  c->walk_fetch = 0;
}

// pad1 counts waves, pad2 flags a loop stopped by the wave limit (its
// packets in flight are abandoned: the tail launch finds none).  Ends the
// loop when no packet is live, or hands the rest to the tail launch once
// every packet has started and at most tail_live are live.
__global__ void wave_loop_cond(WaveCtl* c, const unsigned long long* next, int64_t npk, unsigned long long tail_live,
                               unsigned long long max_waves, cudaGraphConditionalHandle h) {
  const unsigned long long t = global_ns();
  c->walk_ns += t - c->t_last;
  c->t_last = t;
  c->walks += c->n_walk;
  const unsigned long long live = c->n_front + c->n_back;
  const unsigned long long waves = c->pad1 + 1;
  c->pad1 = waves;
  c->n_walk = 0;                      // for the next event launch or the tail
  c->ev_fetch = 0;
  bool go = live > 0;
  if (go && tail_live > 0 && (int64_t)next[0] >= npk && live <= tail_live) go = false;
  if (go && waves >= max_waves) {
    go = false;
    c->pad2 = 1;
    c->n_front = 0;
    c->n_back = 0;
  }
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

__global__ void wave_loop_finish(unsigned long long* cnt, WaveCtl* c) {
  c->tail_ns += global_ns() - c->t_last;
  cnt[MCRT_C_WAVES] += c->pad1;
  cnt[MCRT_C_LAUNCHES] += 4 * c->pad1 + 5;    // + wave_init, wave_loop_start, tail, diffusion_finalize, this
}

// Captures on stream s (in capture mode) the device-driven wavefront loop of
// one packet range: loop reset, wave_init, the WHILE node whose body (event
// launch, wave_loop_mid, walk launch, wave_loop_cond) is captured on stream
// bs, the tail launch (no work when the loop ended with no live packet) and
// wave_loop_finish.  The kernels' arguments are fixed at capture.
cudaError_t capture_wave_loop(const LaunchParams& P, const WaveArgs& W, unsigned long long* next,
                              unsigned long long* cnt, int64_t npk, unsigned long long tail_live,
                              unsigned long long max_waves, bool mixed, int nsm, cudaStream_t s, cudaStream_t bs) {
  const int egrid = nsm * (mixed ? wave_event_mixed_blocks_per_sm() : wave_event_fp64_blocks_per_sm());
  const int wgrid = nsm * (mixed ? wave_walk_mixed_blocks_per_sm() : wave_walk_fp64_blocks_per_sm());
  const int tgrid = nsm * (mixed ? wave_tail_mixed_blocks_per_sm() : wave_tail_fp64_blocks_per_sm());
  cudaError_t e;
  if ((e = cudaMemsetAsync(next, 0, 4 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(W.ctl, 0, sizeof(WaveCtl), s)) != cudaSuccess) return e;
  if ((e = launch_wave_init(W, s)) != cudaSuccess) return e;
  wave_loop_start<<<1, 1, 0, s>>>(W.ctl);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if ((e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd)) != cudaSuccess) return e;
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cn;
  if ((e = cudaGraphAddNode(&cn, g, deps, nd, &cp)) != cudaSuccess) return e;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return e;
  cudaError_t eb = mixed ? launch_wave_event_mixed(P, W, egrid, bs) : launch_wave_event_fp64(P, W, egrid, bs);
  if (eb == cudaSuccess) {
    wave_loop_mid<<<1, 1, 0, bs>>>(W.ctl);
    eb = cudaGetLastError();
  }
  if (eb == cudaSuccess) eb = mixed ? launch_wave_walk_mixed(P, W, wgrid, bs) : launch_wave_walk_fp64(P, W, wgrid, bs);
  if (eb == cudaSuccess) {
    wave_loop_cond<<<1, 1, 0, bs>>>(W.ctl, next, npk, tail_live, max_waves, h);
    eb = cudaGetLastError();
  }
  cudaGraph_t bout = nullptr;
  e = cudaStreamEndCapture(bs, &bout);
  if (eb != cudaSuccess) return eb;
  if (e != cudaSuccess) return e;
  if ((e = cudaStreamUpdateCaptureDependencies(s, &cn, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess) return e;
  LaunchParams T = P;
  T.fetch_off = 1;
  if ((e = mixed ? launch_wave_tail_mixed(T, W, tgrid, s) : launch_wave_tail_fp64(T, W, tgrid, s)) != cudaSuccess) return e;
  wave_loop_finish<<<1, 1, 0, s>>>(cnt, W.ctl);
  return cudaGetLastError();
}

// diskflux (flux_test.f90:14-82) on the REAL arrays the download produces
// (the FP64 device sums rounded to FP32), in the reference's FP32 order of
// operations; the intrinsics keep the compiler from fusing any of them.
// SED: dst[10][n] = si sq su sv, their relative errors, nums, aveinc.
__global__ void diskflux_sed(const double* sed, int64_t n, float rnorm, float* dst) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    float v[10];
    for (int a = 0; a < 10; ++a) v[a] = (float)sed[a * n + k];
    const float si = v[0], nums = v[8];
    float e[4] = {0.f, 0.f, 0.f, 0.f};
    float aveinc = v[9];
    if (nums > 1.0f) {
      const float nm1 = __fsub_rn(nums, 1.0f);
      for (int a = 0; a < 4; ++a) {         // sqrt((x2 - x**2/nums)/(nums-1.)*nums)/si
        const float x = v[a], x2 = v[4 + a];
        const float var = __fmul_rn(__fdiv_rn(__fsub_rn(x2, __fdiv_rn(__fmul_rn(x, x), nums)), nm1), nums);
        e[a] = __fdiv_rn(__fsqrt_rn(var), si);
      }
      e[0] = __fadd_rn(e[0], __fdiv_rn(1.0f, nums));
      aveinc = __fdiv_rn(aveinc, nums);
    }
    for (int a = 0; a < 4; ++a) {
      dst[a * n + k] = __fdiv_rn(v[a], rnorm);
      dst[(4 + a) * n + k] = e[a];
    }
    dst[8 * n + k] = nums;
    dst[9 * n + k] = aveinc;
  }
}

// Peeled SED: dst[9][n] = ti tq tu tv, their relative errors, numt.
__global__ void diskflux_psed(const double* ps, int64_t n, float inorm, float* dst) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    float v[9];
    for (int a = 0; a < 9; ++a) v[a] = (float)ps[a * n + k];
    const float numt = v[8];
    for (int a = 0; a < 4; ++a) {
      float e = 0.f;
      if (numt > 1.0f) {                    // sqrt((x2*numt/x**2-1.)/(numt-1.))
        const float x = v[a], x2 = v[4 + a];
        e = __fsqrt_rn(__fdiv_rn(__fsub_rn(__fdiv_rn(__fmul_rn(x2, numt), __fmul_rn(x, x)), 1.0f), __fsub_rn(numt, 1.0f)));
      }
      dst[a * n + k] = __fdiv_rn(v[a], inorm);
      dst[(4 + a) * n + k] = e;
    }
    dst[8 * n + k] = numt;
  }
}

__global__ void diskflux_img(const double* img, int64_t n, float inorm, float* dst) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    dst[k] = __fdiv_rn((float)img[k], inorm);
}

__global__ void to_float(const double* src, float* dst, int64_t n) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    dst[k] = (float)src[k];
}

}  // namespace mcrt

// ------------------------------------------------------------------ API --
extern "C" {

const char* mcrt_version(void) { return "mcrt-b200 1.0 (sm_100a)"; }

// message of the last failed context-free call (mcrt_setemiss) of this thread
static thread_local std::string g_free_err;

const char* mcrt_last_error(mcrt_ctx* ctx) {
  if (ctx) return ctx->err.c_str();
  return g_free_err.empty() ? "null context" : g_free_err.c_str();
}

int mcrt_create(const mcrt_config* cfg, int device, mcrt_ctx** out) {
  mcrt_ctx* ctx = nullptr;
  if (!cfg || !out) return MCRT_ERR_ARG;
  *out = nullptr;
  if (cfg->nrg < 3 || cfg->ntg < 2 || cfg->npg < 2 || cfg->nopac < 1 || cfg->nfreq < 1 || cfg->nmu < 1 ||
      cfg->nph < 1 || cfg->nap < 1 || cfg->npeel < 0 || cfg->nxhst < 1 || cfg->nT < 2 || cfg->nnu < 2 ||
      cfg->nhnu < 2 || cfg->nlammax < 1)
    return MCRT_ERR_ARG;
  ctx = new mcrt_ctx();
  ctx->cfg = *cfg;
  ctx->device = device;
  CK(cudaSetDevice(device));
  CK(cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device));
  CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&ctx->ev0));
  CK(cudaEventCreate(&ctx->ev1));
  const mcrt_config& c = *cfg;
  ctx->ncell = (int64_t)c.nrg * c.ntg * c.npg;
  ctx->nsed = (int64_t)c.nfreq * c.nmu * c.nph * c.nap * MCRT_NO;
  ctx->npsed = (int64_t)c.nfreq * c.npeel * c.nap * MCRT_NO;
  ctx->nimg = c.output_imcube ? (int64_t)c.npeel * c.nxhst * c.nxhst * c.nfreq : 0;
  if (c.output_imfilt && (c.nfilt < 1 || c.nfilt > 4096 || c.nwfiltmax < 2)) {
    *out = ctx;
    return fail(ctx, MCRT_ERR_ARG, "output_imfilt needs 1 <= nfilt <= 4096 and nwfiltmax >= 2");
  }
  ctx->nimgb = c.output_imfilt ? (int64_t)c.npeel * c.nxhst * c.nxhst * c.nfilt : 0;
  if (c.output_imsparse && (c.sparse_dim < 1 || c.sparse_nnu < 1 || c.sparse_nlev < 1 || c.sparse_nlev > 64 ||
                            !(c.sparse_lognu_max > c.sparse_lognu_min))) {
    *out = ctx;
    return fail(ctx, MCRT_ERR_ARG, "output_imsparse needs sparse_dim, sparse_nnu >= 1, 1 <= sparse_nlev <= 64 "
                                   "and sparse_lognu_max > sparse_lognu_min");
  }
  ctx->nims = c.output_imsparse ? (int64_t)c.sparse_dim * c.sparse_dim * c.sparse_nnu * c.sparse_nlev * c.npeel : 0;
  // one tally allocation: cell ints, cell doubles, SED, peeled SED, images,
  // filter-band images, scalars, counters
  const int64_t n_int = 5 * ctx->ncell;
  const int64_t n_dbl = 2 * ctx->ncell + 10 * ctx->nsed + 9 * ctx->npsed + 4 * ctx->nimg + 8 * ctx->nimgb + 4 * ctx->nims +
                        MCRT_NSCALARS;
  ctx->tally_bytes = (size_t)n_dbl * 8 + (size_t)MCRT_NCOUNTERS * 8 + (size_t)((n_int * 4 + 7) / 8) * 8;
  int rc = dalloc(ctx, (char**)&ctx->d_tally, ctx->tally_bytes);
  if (rc) { *out = ctx; return rc; }
  char* base = (char*)ctx->d_tally;
  double* d = (double*)base;
  DevTallies& t = ctx->dt;
  t.dtauabs = d; d += ctx->ncell;
  t.fuvmean = d; d += ctx->ncell;
  t.sed = d; d += 10 * ctx->nsed;
  t.psed = d; d += 9 * ctx->npsed;
  t.img = d; d += 4 * ctx->nimg;
  t.imgb = d; d += 8 * ctx->nimgb;
  t.ims = d; d += 4 * ctx->nims;
  t.scal = d; d += MCRT_NSCALARS;
  t.cnt = (unsigned long long*)d;
  int32_t* ip = (int32_t*)(t.cnt + MCRT_NCOUNTERS);
  t.nabs = ip; ip += ctx->ncell;
  t.dbig = ip; ip += ctx->ncell;
  t.dsg = ip; ip += ctx->ncell;
  t.killed = ip; ip += ctx->ncell;
  t.ndiff = ip;
  if ((rc = dalloc(ctx, &ctx->d_next, 4))) { *out = ctx; return rc; }
  if ((rc = dalloc(ctx, &ctx->d_err, 4))) { *out = ctx; return rc; }
  CK(cudaMemset(ctx->d_tally, 0, ctx->tally_bytes));
  *out = ctx;
  return MCRT_OK;
}

void mcrt_destroy(mcrt_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->wl_exec) cudaGraphExecDestroy(ctx->wl_exec);
  if (ctx->wl_graph) cudaGraphDestroy(ctx->wl_graph);
  if (ctx->wl_body) cudaStreamDestroy(ctx->wl_body);
  if (ctx->h_block0) cudaFreeHost(ctx->h_block0);
  if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
  if (ctx->h_wctl) cudaFreeHost(ctx->h_wctl);
  if (ctx->h_geom) cudaFreeHost(ctx->h_geom);
  for (auto& p : ctx->kt_ev)
    for (auto& e : p) if (e) cudaEventDestroy(e);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  for (auto& e : ctx->marks) if (e) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int mcrt_set_precision(mcrt_ctx* ctx, int32_t mode) {
  if (!ctx) return MCRT_ERR_ARG;
  if (mode != MCRT_PREC_FP64 && mode != MCRT_PREC_MIXED) return fail(ctx, MCRT_ERR_ARG, "unknown precision %d", mode);
  ctx->precision = mode;
  return MCRT_OK;
}

int mcrt_set_schedule(mcrt_ctx* ctx, int32_t schedule, int32_t event_batch) {
  if (!ctx) return MCRT_ERR_ARG;
  if (schedule != MCRT_SCHED_PACKET && schedule != MCRT_SCHED_WARP && schedule != MCRT_SCHED_WAVE)
    return fail(ctx, MCRT_ERR_ARG, "unknown schedule %d", schedule);
  if (event_batch < 1 || event_batch > 32) return fail(ctx, MCRT_ERR_ARG, "event_batch must be 1..32");
  ctx->schedule = schedule;
  if (schedule == MCRT_SCHED_WAVE) ctx->wave_batch = event_batch;
  else ctx->event_batch = event_batch;
  return MCRT_OK;
}

int mcrt_set_wave_pool(mcrt_ctx* ctx, int64_t slots, int64_t peel_jobs, int64_t tail_packets) {
  if (!ctx) return MCRT_ERR_ARG;
  if (slots < 32 || slots > ((int64_t)1 << 30)) return fail(ctx, MCRT_ERR_ARG, "wave pool must hold 32..2^30 slots");
  if (peel_jobs != 0 && (peel_jobs < 2 * slots || peel_jobs > ((int64_t)1 << 32)))
    return fail(ctx, MCRT_ERR_ARG, "peel-off job queue must hold 2 x slots .. 2^32 jobs (or 0 for the default)");
  ctx->wave_pool = slots;
  ctx->wave_jobs = peel_jobs;
  ctx->wave_tail = tail_packets;
  return MCRT_OK;
}

int mcrt_upload_grid(mcrt_ctx* ctx, const mcrt_grid* g) {
  if (!ctx || !g) return MCRT_ERR_ARG;
  {
    char msg[256];
    const int rc = mcrt_check_grid(&ctx->cfg, g, msg, (int32_t)sizeof msg);
    if (rc) return fail(ctx, rc, "mcrt_upload_grid: %s", msg);
  }
  ++ctx->uploads;
  CK(cudaSetDevice(ctx->device));
  const mcrt_config& c = ctx->cfg;
  const int nrg = c.nrg, ntg = c.ntg, npg = c.npg;
  const int64_t ncell = ctx->ncell;
  // transport layout: one CellRec per cell with the non-zero components
  std::vector<CellRec> cells(ncell);
  std::vector<int> slot_species;
  std::vector<double> dens_th(ncell, 0.0);
  std::vector<int32_t> idust3(ncell, 0), diffus(ncell, 0);
  bool has_sg = false;
  for (int64_t k = 0; k < ncell; ++k) {
    CellRec& r = cells[k];
    std::memset(&r, 0, sizeof r);
    int n = 0;
    int nth = 0;
    for (int id = 1; id <= MCRT_NDG2; ++id) {
      const double rho = g->densarr[k + ncell * (id - 1)];
      if (!(rho > 0.0)) continue;
      const int sp = g->findopac[k + ncell * (id - 1)];
      if (id > 8) return fail(ctx, MCRT_ERR_UNSUPPORTED, "gas-opacity component %d is outside the built scope", id);
      if (sp != id) return fail(ctx, MCRT_ERR_UNSUPPORTED, "findopac(.,%d)=%d: dust components must map to their own species", id, sp);
      if (sp < 1 || sp > c.nopac) return fail(ctx, MCRT_ERR_ARG, "findopac out of range");
      if (n >= kMaxComp) return fail(ctx, MCRT_ERR_UNSUPPORTED, "more than %d non-zero density components in a cell", kMaxComp);
      int s = -1;
      for (size_t q = 0; q < slot_species.size(); ++q) if (slot_species[q] == sp) s = (int)q;
      if (s < 0) {
        if ((int)slot_species.size() >= kMaxSlot) return fail(ctx, MCRT_ERR_UNSUPPORTED, "more than %d opacity species", kMaxSlot);
        slot_species.push_back(sp);
        s = (int)slot_species.size() - 1;
      }
      r.rho[n] = rho;
      r.meta |= (uint32_t)s << (2 + 7 * n);
      r.meta |= (uint32_t)(id - 1) << (5 + 7 * n);
      ++n;
      if (!kIsSg[id - 1]) { ++nth; dens_th[k] = rho; idust3[k] = id; } else has_sg = true;
    }
    r.meta |= (uint32_t)n;
    if (nth > 1) return fail(ctx, MCRT_ERR_UNSUPPORTED, "cell with %d thermal components (tfinal allows one)", nth);
    diffus[k] = g->diffus[k] ? 1 : 0;
    const int dd = g->diffdir ? g->diffdir[k] : 0;
    if (diffus[k] && dd != 2 && dd != -2)
      return fail(ctx, MCRT_ERR_UNSUPPORTED, "radial/phi diffusion (diffdir=%d, emit_common_2.f90:91-199,374) is outside the built scope", dd);
    if (diffus[k] && nth == 0) return fail(ctx, MCRT_ERR_ARG, "diffusion cell without a thermal component");
    if (dd < -8 || dd > 7) return fail(ctx, MCRT_ERR_ARG, "diffdir out of range");
    r.flags = (uint32_t)diffus[k] | ((uint32_t)(dd + 8) << 1) | (nth > 0 ? 32u : 0u);
  }
  if (slot_species.empty()) slot_species.push_back(1);
  // walls: rarr r2arr | thetarr costarr tan2arr | phiarr aarr barr, each
  // padded by one element.  The reference reads one past the last wall when a
  // peel-off steps to ir=nrg or a walk reaches it=ntg before testgrid
  // (testgrid.f90:92-93, peeloff_3d_2_test.f90:119-121); the pad makes those
  // reads defined: a sphere at 4 r2arr(nrg), a cone beyond the south pole.
  std::vector<double> walls;
  auto addp = [&](const double* a, int n, double pad) { walls.insert(walls.end(), a, a + n); walls.push_back(pad); };
  addp(g->rarr, nrg, 2.0 * g->rarr[nrg - 1]);
  addp(g->r2arr, nrg, 4.0 * g->r2arr[nrg - 1]);
  addp(g->thetarr, ntg, g->thetarr[ntg - 1]);
  addp(g->costarr, ntg, g->costarr[ntg - 1] - 1.0);
  addp(g->tan2arr, ntg, 0.0);
  addp(g->sintarr ? g->sintarr : g->tan2arr, ntg, 0.0);
  addp(g->phiarr, npg, g->phiarr[npg - 1]);
  addp(g->aarr, npg, g->aarr[npg - 1]);
  addp(g->barr, npg, g->barr[npg - 1]);
  // disk-accretion emission tables (initpacc_4.f90:28-36), [nrg-1] each;
  // optional: absent, accretion packets are refused at run time
  const bool acc = g->ravearr && g->Ldint && g->hdisk;
  if (acc) {
    for (int i = 1; i < nrg - 1; ++i)
      if (!(g->Ldint[i] >= g->Ldint[i - 1])) return fail(ctx, MCRT_ERR_ARG, "Ldint must be non-decreasing");
    for (int i = 0; i < nrg - 1; ++i)
      if (!(g->hdisk[i] >= 0.0) || !(g->ravearr[i] > 0.0)) return fail(ctx, MCRT_ERR_ARG, "ravearr/hdisk must be positive");
  }
  // FP32 walk tables (mixed build): cells with FP32 densities; per theta
  // wall (mu, mu^2) with the plane (tan2arr = -1) and the poles (tan2arr =
  // 0, skipped by thetaface.f90) flagged; per phi wall the plane (A, B).
  std::vector<CellRecF> cellsf(ncell);
  for (int64_t k = 0; k < ncell; ++k) {
    for (int i = 0; i < kMaxComp; ++i) cellsf[k].rho[i] = (float)cells[k].rho[i];
    cellsf[k].meta = cells[k].meta;
  }
  std::vector<float2> tcone(ntg + 1), pplane(npg + 1);
  for (int j = 0; j <= ntg; ++j) {
    const double mu = j < ntg ? g->costarr[j] : g->costarr[ntg - 1] - 1.0;
    const double t2 = j < ntg ? g->tan2arr[j] : 0.0;
    tcone[j].x = (float)mu;
    tcone[j].y = t2 < 0.0 ? -1.0f : (t2 == 0.0 ? 2.0f : (float)(mu * mu));
  }
  for (int j = 0; j <= npg; ++j) {
    pplane[j].x = (float)(j < npg ? g->aarr[j] : g->aarr[npg - 1]);
    pplane[j].y = (float)(j < npg ? g->barr[j] : g->barr[npg - 1]);
  }
  const size_t w32_cone = 0, w32_plane = (size_t)(ntg + 1) * sizeof(float2);
  std::vector<unsigned char> walk32(w32_plane + (size_t)(npg + 1) * sizeof(float2), 0);
  std::memcpy(walk32.data() + w32_cone, tcone.data(), tcone.size() * sizeof(float2));
  std::memcpy(walk32.data() + w32_plane, pplane.data(), pplane.size() * sizeof(float2));
  const std::vector<double> zeros(nrg > 1 ? nrg - 1 : 1, 0.0);
  addp(acc ? g->ravearr : zeros.data(), nrg - 1, 0.0);
  addp(acc ? g->Ldint : zeros.data(), nrg - 1, 1.0);
  addp(acc ? g->hdisk : zeros.data(), nrg - 1, 0.0);
  ctx->have_acc = acc;
  ctx->h_rarr.assign(g->rarr, g->rarr + nrg);
  if (!ctx->have_grid) {
    int rc;
    if ((rc = dalloc(ctx, &ctx->d_walls, walls.size()))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_cells, ncell))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_cellsf, ncell))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_walk32, walk32.size()))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_tdust, ncell))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_tdust0, ncell))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_vcell, ncell))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_dens_thermal, 2 * ncell))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_idust3, ncell))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_diffus, ncell))) return rc;
  }
  CK(cudaMemcpyAsync(ctx->d_walls, walls.data(), walls.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_cells, cells.data(), ncell * sizeof(CellRec), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_cellsf, cellsf.data(), ncell * sizeof(CellRecF), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_walk32, walk32.data(), walk32.size(), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_tdust, g->tdust, ncell * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_tdust0, g->tdust, ncell * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_vcell, g->vcell, ncell * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_dens_thermal, dens_th.data(), ncell * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_idust3, idust3.data(), ncell * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_diffus, diffus.data(), ncell * 4, cudaMemcpyHostToDevice, ctx->stream));
  ctx->h_diffus = diffus;
  // velocity field and tfinal's per-cell gradient rules
  const bool vel = g->vrarr && g->vthetarr && g->divvarr;
  if (!vel && (g->vrarr || g->vthetarr || g->divvarr))
    return fail(ctx, MCRT_ERR_ARG, "mcrt_upload_grid: vrarr, vthetarr and divvarr come together (or none)");
  if (vel) {
    if (nrg < 19 || ntg < 18)
      return fail(ctx, MCRT_ERR_UNSUPPORTED, "a velocity field needs nrg >= 19 and ntg >= 18 (tfinal's 15-cell windows)");
    std::vector<int32_t> tflag(ncell, 0);
    for (int64_t k = 0; k < ncell; ++k) {
      auto rho = [&](int id) { return g->densarr[k + ncell * (id - 1)]; };
      if (rho(1) + rho(2) + rho(9) > 0.0) tflag[k] |= 1;
      if (rho(4) + rho(10) > 0.0) tflag[k] |= 2;
    }
    std::vector<double> rave(nrg, 0.0);
    for (int i = 0; i < nrg - 1; ++i) rave[i] = g->ravearr ? g->ravearr[i] : 0.5 * (g->rarr[i] + g->rarr[i + 1]);
    int rc2;
    if (!ctx->d_vel && ((rc2 = dalloc(ctx, &ctx->d_vel, 3 * ncell)) || (rc2 = dalloc(ctx, &ctx->d_tflag, ncell)) ||
                        (rc2 = dalloc(ctx, &ctx->d_rave, nrg))))
      return rc2;
    CK(cudaMemcpyAsync(ctx->d_vel, g->vrarr, ncell * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_vel + ncell, g->vthetarr, ncell * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_vel + 2 * ncell, g->divvarr, ncell * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_tflag, tflag.data(), ncell * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_rave, rave.data(), nrg * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));     // the host vectors go out of scope
  }
  ctx->have_vel = vel;
  // small-grain emission level per cell (imean), optional
  int32_t imax = 0;
  if (g->imean) {
    for (int64_t k = 0; k < ncell; ++k) {
      if (g->imean[k] < 1) return fail(ctx, MCRT_ERR_ARG, "imean(%lld) = %d: rows of the Draine table start at 1",
                                       (long long)k, g->imean[k]);
      imax = std::max(imax, g->imean[k]);
    }
    int rc3;
    if (!ctx->d_imean && (rc3 = dalloc(ctx, &ctx->d_imean, ncell))) return rc3;
    CK(cudaMemcpyAsync(ctx->d_imean, g->imean, ncell * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  ctx->imean_max = imax;
  ctx->have_sg = has_sg;
  CK(cudaStreamSynchronize(ctx->stream));
  DevModel& m = ctx->dm;
  m.imean = g->imean ? ctx->d_imean : nullptr;
  const double* w = ctx->d_walls;
  m.rarr = w; w += nrg + 1;
  m.r2arr = w; w += nrg + 1;
  m.thetarr = w; w += ntg + 1;
  m.costarr = w; w += ntg + 1;
  m.tan2arr = w; w += ntg + 1;
  m.sintarr = w; w += ntg + 1;
  m.phiarr = w; w += npg + 1;
  m.aarr = w; w += npg + 1;
  m.barr = w; w += npg + 1;
  m.ravearr = w; w += nrg;
  m.Ldint = w; w += nrg;
  m.hdisk = w;
  m.cells = ctx->d_cells;
  m.cellsf = ctx->d_cellsf;
  m.tcone = reinterpret_cast<const float2*>(ctx->d_walk32 + w32_cone);
  m.pplane = reinterpret_cast<const float2*>(ctx->d_walk32 + w32_plane);
  m.tdust = ctx->d_tdust0;
  m.vcell = ctx->d_vcell;
  m.nslot = (int)slot_species.size();
  for (int s = 0; s < kMaxSlot; ++s) m.slot_species[s] = s < m.nslot ? slot_species[s] : 1;
  ctx->have_grid = true;
  return MCRT_OK;
}

int mcrt_check_grid(const mcrt_config* c, const mcrt_grid* g, char* msg, int32_t msg_len) {
  auto bad = [&](int code, const char* fmt, auto... a) {
    if (msg && msg_len > 0) {
      if constexpr (sizeof...(a) == 0) snprintf(msg, (size_t)msg_len, "%s", fmt);
      else snprintf(msg, (size_t)msg_len, fmt, a...);
    }
    return code;
  };
  if (msg && msg_len > 0) msg[0] = 0;
  if (!c || !g) return bad(MCRT_ERR_ARG, "missing config or grid");
  const int nrg = c->nrg, ntg = c->ntg, npg = c->npg;
  if (nrg < 3 || ntg < 2 || npg < 2) return bad(MCRT_ERR_ARG, "grid of %d x %d x %d walls is too small", nrg, ntg, npg);
  if (!g->rarr || !g->r2arr || !g->thetarr || !g->costarr || !g->tan2arr || !g->phiarr || !g->aarr || !g->barr ||
      !g->densarr || !g->findopac || !g->diffus || !g->tdust || !g->vcell || !g->sintarr)
    return bad(MCRT_ERR_ARG, "missing array");
  for (int i = 0; i < nrg; ++i) {
    if (!(std::isfinite(g->rarr[i]) && g->rarr[i] > 0.0) || !(std::isfinite(g->r2arr[i])))
      return bad(MCRT_ERR_ARG, "rarr(%d) = %g is not a finite positive radius", i + 1, g->rarr[i]);
    if (i > 0 && !(g->rarr[i] > g->rarr[i - 1])) return bad(MCRT_ERR_ARG, "rarr is not increasing at %d", i + 1);
  }
  for (int i = 0; i < ntg; ++i) {
    if (!(std::isfinite(g->thetarr[i]) && std::isfinite(g->costarr[i]) && std::isfinite(g->tan2arr[i])))
      return bad(MCRT_ERR_ARG, "theta wall %d is not finite", i + 1);
    if (i > 0 && !(g->thetarr[i] > g->thetarr[i - 1])) return bad(MCRT_ERR_ARG, "thetarr is not increasing at %d", i + 1);
  }
  for (int i = 0; i < npg; ++i) {
    if (!(std::isfinite(g->phiarr[i]) && std::isfinite(g->aarr[i]) && std::isfinite(g->barr[i])))
      return bad(MCRT_ERR_ARG, "phi wall %d is not finite", i + 1);
    if (i > 0 && !(g->phiarr[i] > g->phiarr[i - 1])) return bad(MCRT_ERR_ARG, "phiarr is not increasing at %d", i + 1);
  }
  const int64_t ncell = (int64_t)nrg * ntg * npg;
  for (const double* v : {g->vrarr, g->vthetarr, g->divvarr})
    if (v)
      for (int64_t k = 0; k < ncell; ++k)
        if (!std::isfinite(v[k])) return bad(MCRT_ERR_ARG, "velocity field entry %lld is not finite", (long long)k + 1);
  for (int64_t k = 0; k < ncell; ++k) {
    bool dust = false;
    for (int id = 0; id < MCRT_NDG2; ++id) {
      const double rho = g->densarr[k + ncell * id];
      if (!(std::isfinite(rho) && rho >= 0.0))
        return bad(MCRT_ERR_ARG, "densarr(cell %lld, component %d) = %g is not a finite non-negative density",
                   (long long)k + 1, id + 1, rho);
      dust = dust || rho > 0.0;
    }
    if (!(std::isfinite(g->tdust[k]) && g->tdust[k] >= 0.0))
      return bad(MCRT_ERR_ARG, "tdust(cell %lld) = %g is not a finite non-negative temperature", (long long)k + 1,
                 g->tdust[k]);
    if (!std::isfinite(g->vcell[k]) || (dust && !(g->vcell[k] > 0.0)))
      return bad(MCRT_ERR_ARG, "vcell(cell %lld) = %g: a cell with dust needs a finite positive volume", (long long)k + 1,
                 g->vcell[k]);
  }
  return MCRT_OK;
}

int mcrt_set_limits(mcrt_ctx* ctx, int64_t walk_crossings, int64_t waves, double geom_fraction) {
  if (!ctx) return MCRT_ERR_ARG;
  ctx->walk_limit = walk_crossings > 0 ? walk_crossings : 50000000;
  ctx->wave_limit = waves > 0 ? waves : 400000000;
  ctx->geom_fraction = geom_fraction;
  return MCRT_OK;
}

int mcrt_upload_tables(mcrt_ctx* ctx, const mcrt_tables* t) {
  if (!ctx || !t) return MCRT_ERR_ARG;
  ++ctx->uploads;
  CK(cudaSetDevice(ctx->device));
  const mcrt_config& c = ctx->cfg;
  if (!t->nlambda || !t->nudust || !t->kappad || !t->adust || !t->gdust || !t->pldust || !t->kappav || !t->kapint ||
      !t->lTint || !t->Tint || !t->nuint || !t->kappap || !t->atmosnu || !t->hnuint || !t->lognu || !t->loghnu ||
      !t->aperture2 || !t->u || (c.npeel > 0 && (!t->coste_arr || !t->sinte_arr || !t->cospe_arr || !t->sinpe_arr)))
    return fail(ctx, MCRT_ERR_ARG, "mcrt_upload_tables: missing array");
  if (c.limb != 0 && !t->limb_prob) return fail(ctx, MCRT_ERR_ARG, "limb=1 needs limb_prob");
  for (int i = 0; i < c.nopac; ++i)
    if (t->nlambda[i] < 2 || t->nlambda[i] > c.nlammax) return fail(ctx, MCRT_ERR_ARG, "nlambda(%d) out of range", i + 1);
  const int64_t nl = (int64_t)c.nlammax * c.nopac;
  const int64_t nk = (int64_t)c.nT * c.nnu * c.nopac;
  std::vector<double> tab;
  std::vector<int64_t> off;
  auto add = [&](const double* p, int64_t n) { off.push_back((int64_t)tab.size()); tab.insert(tab.end(), p, p + n); };
  std::vector<double> sini(c.nmu), inczeta(MCRT_IZMAX), zero(c.npeel > 0 ? 0 : 1, 0.0);
  for (int i = 0; i < c.nmu; ++i) sini[i] = std::sqrt(1.0 - t->u[i] * t->u[i]);
  zetainit_h(inczeta.data());
  std::vector<double> limb(100, 0.0);
  if (t->limb_prob) limb.assign(t->limb_prob, t->limb_prob + 100);
  add(t->nudust, nl); add(t->kappad, nl); add(t->adust, nl); add(t->gdust, nl); add(t->pldust, nl);   // 0-4
  add(t->kappav, c.nopac); add(t->kapint, nk); add(t->lTint, c.nT); add(t->nuint, c.nnu);              // 5-8
  add(t->atmosnu, c.nhnu); add(t->hnuint, c.nhnu); add(t->lognu, c.nhnu); add(t->loghnu, c.nhnu);      // 9-12
  add(limb.data(), 100); add(inczeta.data(), MCRT_IZMAX);                                              // 13-14
  add(t->aperture2, c.nap); add(t->u, c.nmu); add(sini.data(), c.nmu);                                 // 15-17
  const int np = std::max(c.npeel, 1);
  std::vector<double> pz(np, 0.0);
  add(c.npeel ? t->coste_arr : pz.data(), np); add(c.npeel ? t->sinte_arr : pz.data(), np);            // 18-19
  add(c.npeel ? t->cospe_arr : pz.data(), np); add(c.npeel ? t->sinpe_arr : pz.data(), np);            // 20-21
  add(t->Tint, c.nT); add(t->kappap, (int64_t)c.nT * c.nopac);                                          // 22-23
  // tabulated scattering matrices: the table and, per (species, wavelength)
  // row, the rejection bound max(S11 + |S12|) over the cosine bins, which
  // bounds the sampling probability (S11 I + S12 (cos2i Q +- sin2i U)) / I
  // for any polarisation; it replaces stokes6's running `peak`
  const bool mueller = t->mueller != nullptr && t->narr > 0;
  if (mueller) {
    if (t->narr < 2 || t->narr > 1000000) return fail(ctx, MCRT_ERR_ARG, "narr must be 2..1e6");
    const int64_t nrow = nl, nb = t->narr;
    std::vector<double> peak(nrow, 0.0);
    for (int64_t r = 0; r < nrow; ++r)
      for (int64_t i = 0; i < nb; ++i) {
        const double* e = t->mueller + 6 * (i + nb * r);
        for (int k = 0; k < 6; ++k)
          if (!std::isfinite(e[k])) return fail(ctx, MCRT_ERR_ARG, "mueller table holds a non-finite value");
        if (!(e[0] >= 0.0)) return fail(ctx, MCRT_ERR_ARG, "mueller S11 must be non-negative");
        peak[r] = std::max(peak[r], e[0] + std::fabs(e[1]));
      }
    add(t->mueller, 6 * nb * nrow);                                                                    // 24
    add(peak.data(), nrow);                                                                            // 25
  }
  // ISRF sampling table of external-illumination packets (isrf_cdf.f90):
  // cdf_i, logcdf_i, logfreq_i, as the driver's isrf_mod holds them
  const bool isrf = t->isrf != nullptr && t->nisrf > 0;
  const int isrf_at = isrf ? (int)off.size() : -1;
  if (isrf) {
    if (t->nisrf < 2 || t->nisrf > 1000000) return fail(ctx, MCRT_ERR_ARG, "nisrf must be 2..1e6");
    for (int i = 1; i < t->nisrf; ++i)
      if (!(t->isrf[i] >= t->isrf[i - 1])) return fail(ctx, MCRT_ERR_ARG, "isrf cdf must be non-decreasing");
    add(t->isrf, 3 * (int64_t)t->nisrf);
  }
  // small-grain emission spectra (draine_cdf.f90): cdf_d, logcdf_d
  // (nemit x ndraine) and logfreq_d (ndraine), as draine_mod holds them
  const bool draine = t->draine != nullptr && t->nemit > 0 && t->ndraine > 0;
  const int draine_at = draine ? (int)off.size() : -1;
  if (draine) {
    if (t->nemit > 1000 || t->ndraine < 2 || t->ndraine > 1000000)
      return fail(ctx, MCRT_ERR_ARG, "nemit must be 1..1000 and ndraine 2..1e6");
    const int64_t nn = 2 * (int64_t)t->nemit * t->ndraine + t->ndraine;
    for (int64_t i = 0; i < nn; ++i)
      if (!std::isfinite(t->draine[i])) return fail(ctx, MCRT_ERR_ARG, "draine table entry %lld is not finite", (long long)i);
    add(t->draine, nn);
  }
  // filter curves of the filter-band images (filt_nu.f90): filtwave and
  // filtphi per filter over nwfiltmax points, of which nwfilt-1 are used
  const bool filt = c.output_imfilt && t->nwfilt && t->filtwave && t->filtphi;
  if (c.output_imfilt && !filt) return fail(ctx, MCRT_ERR_ARG, "output_imfilt needs nwfilt, filtwave and filtphi");
  const int filt_at = filt ? (int)off.size() : -1;
  std::vector<int32_t> nfpts;
  if (filt) {
    for (int f = 0; f < c.nfilt; ++f) {
      const int nf = t->nwfilt[f] - 1;
      if (nf < 1 || nf > c.nwfiltmax) return fail(ctx, MCRT_ERR_ARG, "nwfilt(%d) = %d: a curve needs 1..nwfiltmax points", f + 1, t->nwfilt[f]);
      const double* fw = t->filtwave + (int64_t)c.nwfiltmax * f;
      const double* fp = t->filtphi + (int64_t)c.nwfiltmax * f;
      for (int i = 0; i < nf; ++i) {
        if (!std::isfinite(fw[i]) || !std::isfinite(fp[i])) return fail(ctx, MCRT_ERR_ARG, "filter %d holds a non-finite value", f + 1);
        if (i > 0 && fw[i] < fw[i - 1]) return fail(ctx, MCRT_ERR_ARG, "filtwave of filter %d must be non-decreasing in frequency", f + 1);
      }
      nfpts.push_back(nf);
    }
    add(t->filtwave, (int64_t)c.nwfiltmax * c.nfilt);
    add(t->filtphi, (int64_t)c.nwfiltmax * c.nfilt);
  }
  // Rosseland table (setdiffus), optional; after the blocks read by fixed index
  const int kappar_at = t->kappar ? (int)off.size() : -1;
  if (t->kappar) add(t->kappar, (int64_t)c.nT * c.nopac);
  // jump tables a^(2^30 * 2^k)
  std::vector<int64_t> jump(128);
  int64_t j1 = 1033780774, j2 = 1494757890;   // a1w, a2w (ecuyer_cote_mod.f90:14-15)
  for (int k = 0; k < 64; ++k) {
    jump[k] = j1;
    jump[64 + k] = j2;
    j1 = mulmod_h(j1, j1, 2147483563);
    j2 = mulmod_h(j2, j2, 2147483399);
  }
  // digit tables A^(j * 2^(14 c)), A = a^(2^30): [gen][c][j]
  jump.resize(128 + 6 * (size_t)kJumpDigit);
  for (int gen = 0; gen < 2; ++gen) {
    const int64_t mod = gen == 0 ? 2147483563 : 2147483399;
    int64_t base = jump[64 * gen];                       // A
    int64_t* T = jump.data() + 128 + (size_t)gen * 3 * kJumpDigit;
    for (int cdig = 0; cdig < 3; ++cdig) {
      int64_t* Tc = T + (size_t)cdig * kJumpDigit;
      Tc[0] = 1;
      for (int j = 1; j < kJumpDigit; ++j) Tc[j] = mulmod_h(Tc[j - 1], base, mod);
      base = mulmod_h(Tc[kJumpDigit - 1], base, mod);   // A^(2^(14 (c+1)))
    }
  }
  int rc;
  if (ctx->have_tables) { dfree(ctx, ctx->d_tabs); dfree(ctx, ctx->d_nlambda); dfree(ctx, ctx->d_jump); }
  if (ctx->d_nfpts) { dfree(ctx, ctx->d_nfpts); ctx->d_nfpts = nullptr; }
  if (ctx->d_levels) { dfree(ctx, ctx->d_levels); ctx->d_levels = nullptr; }
  if (c.output_imsparse) {
    if (!t->sparse_levels) return fail(ctx, MCRT_ERR_ARG, "output_imsparse needs sparse_levels");
    for (int l = 0; l < c.sparse_nlev; ++l)
      if (!(t->sparse_levels[l] > 0.0f) || !std::isfinite(t->sparse_levels[l]) ||
          (l > 0 && !(t->sparse_levels[l] > t->sparse_levels[l - 1])))
        return fail(ctx, MCRT_ERR_ARG, "sparse_levels must be positive and ascending");
    if ((rc = dalloc(ctx, &ctx->d_levels, (size_t)c.sparse_nlev))) return rc;
    CK(cudaMemcpyAsync(ctx->d_levels, t->sparse_levels, (size_t)c.sparse_nlev * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (filt) {
    if ((rc = dalloc(ctx, &ctx->d_nfpts, nfpts.size()))) return rc;
    CK(cudaMemcpyAsync(ctx->d_nfpts, nfpts.data(), nfpts.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  if ((rc = dalloc(ctx, &ctx->d_tabs, tab.size()))) return rc;
  if ((rc = dalloc(ctx, &ctx->d_nlambda, c.nopac))) return rc;
  if ((rc = dalloc(ctx, &ctx->d_jump, jump.size()))) return rc;
  CK(cudaMemcpyAsync(ctx->d_tabs, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_nlambda, t->nlambda, c.nopac * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_jump, jump.data(), jump.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  DevModel& m = ctx->dm;
  const double* b = ctx->d_tabs;
  m.nudust = b + off[0]; m.kappad = b + off[1]; m.adust = b + off[2]; m.gdust = b + off[3]; m.pldust = b + off[4];
  m.kappav = b + off[5]; m.kapint = b + off[6]; m.lTint = b + off[7]; m.nuint = b + off[8];
  m.atmosnu = b + off[9]; m.hnuint = b + off[10]; m.lognu = b + off[11]; m.loghnu = b + off[12];
  m.limb_prob = b + off[13]; m.inczeta = b + off[14];
  m.aperture2 = b + off[15]; m.u = b + off[16]; m.sini = b + off[17];
  m.coste = b + off[18]; m.sinte = b + off[19]; m.cospe = b + off[20]; m.sinpe = b + off[21];
  m.mueller = mueller ? b + off[24] : nullptr;
  m.mpeak = mueller ? b + off[25] : nullptr;
  m.narr = mueller ? t->narr : 0;
  m.dct = mueller ? 2.0 / (double)t->narr : 0.0;
  m.nisrf = isrf ? t->nisrf : 0;
  m.isrf_cdf = isrf ? b + off[isrf_at] : nullptr;
  m.isrf_logcdf = isrf ? m.isrf_cdf + t->nisrf : nullptr;
  m.isrf_logfreq = isrf ? m.isrf_cdf + 2 * (int64_t)t->nisrf : nullptr;
  ctx->have_isrf = isrf;
  m.nemit = draine ? t->nemit : 0;
  m.ndraine = draine ? t->ndraine : 0;
  m.draine_cdf = draine ? b + off[draine_at] : nullptr;
  m.draine_logcdf = draine ? m.draine_cdf + (int64_t)t->nemit * t->ndraine : nullptr;
  m.draine_logfreq = draine ? m.draine_cdf + 2 * (int64_t)t->nemit * t->ndraine : nullptr;
  ctx->have_draine = draine;
  m.nfpts = filt ? ctx->d_nfpts : nullptr;
  m.sparse_levels = c.output_imsparse ? ctx->d_levels : nullptr;
  m.filtwave = filt ? b + off[filt_at] : nullptr;
  m.filtphi = filt ? b + off[filt_at + 1] : nullptr;
  m.nlambda = ctx->d_nlambda;
  m.jump1 = ctx->d_jump;
  m.jump2 = ctx->d_jump + 64;
  m.jdig1 = ctx->d_jump + 128;
  m.jdig2 = ctx->d_jump + 128 + 3 * kJumpDigit;
  // species that share a wavelength column (same length, same values bit for
  // bit) share opacset's bracket search
  ctx->species_grid.assign(c.nopac, 0);
  for (int id = 0; id < c.nopac; ++id) {
    ctx->species_grid[id] = id;
    for (int k = 0; k < id; ++k) {
      if (ctx->species_grid[k] != k || t->nlambda[k] != t->nlambda[id]) continue;
      if (std::memcmp(t->nudust + (int64_t)c.nlammax * k, t->nudust + (int64_t)c.nlammax * id,
                      (size_t)t->nlambda[id] * 8) == 0) { ctx->species_grid[id] = k; break; }
    }
  }
  ctx->have_tables = true;
  ctx->off_Tint = off[22];
  ctx->off_kappap = off[23];
  ctx->off_kappar = kappar_at >= 0 ? off[kappar_at] : -1;
  return MCRT_OK;
}

int mcrt_reset_tallies(mcrt_ctx* ctx) {
  if (!ctx) return MCRT_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemsetAsync(ctx->d_tally, 0, ctx->tally_bytes, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return MCRT_OK;
}

int mcrt_enable_packet_log(mcrt_ctx* ctx, int64_t max_packets) {
  if (!ctx || max_packets < 0) return MCRT_ERR_ARG;
  ++ctx->uploads;                     // the log buffer is replaced
  CK(cudaSetDevice(ctx->device));
  if (ctx->d_log) { dfree(ctx, ctx->d_log); ctx->d_log = nullptr; }
  ctx->nlog = max_packets;
  if (max_packets > 0) {
    int rc = dalloc(ctx, &ctx->d_log, (size_t)max_packets);
    if (rc) return rc;
    CK(cudaMemset(ctx->d_log, 0, (size_t)max_packets * sizeof(mcrt_packet_log)));
  }
  return MCRT_OK;
}

int mcrt_download_packet_log(mcrt_ctx* ctx, mcrt_packet_log* out, int64_t n) {
  if (!ctx || !out || n < 0 || n > ctx->nlog) return MCRT_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpy(out, ctx->d_log, (size_t)n * sizeof(mcrt_packet_log), cudaMemcpyDeviceToHost));
  return MCRT_OK;
}

// Grow the adjoint's job records to hold at least `need`, keeping the ones
// written so far (the host calls it between launches).
static int adjoint_grow(mcrt_ctx* ctx, int64_t need) {
  AdjointArgs& A = ctx->adj;
  const int64_t cap = std::max<int64_t>(need, 2 * A.rec_cap);
  unsigned long long* rk = nullptr;
  double* rcv = nullptr;
  int rc;
  if ((rc = dalloc(ctx, &rk, cap)) || (rc = dalloc(ctx, &rcv, cap))) return rc;
  const int64_t used = ctx->adj_rec_used;
  CK(cudaMemsetAsync(rk, 0xff, (size_t)cap * 8, ctx->stream));
  CK(cudaMemsetAsync(rcv, 0, (size_t)cap * 8, ctx->stream));
  if (used > 0) {
    CK(cudaMemcpyAsync(rk, A.rec_key, (size_t)used * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(rcv, A.rec_c, (size_t)used * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  dfree(ctx, A.rec_key);
  dfree(ctx, A.rec_c);
  A.rec_key = rk;
  A.rec_c = rcv;
  A.rec_cap = cap;
  return MCRT_OK;
}

// adj_mode 0: an ordinary iteration; 1: the adjoint's forward pass (wave
// schedule, no tail launch so that every peel-off goes through the peel-off
// kernel, records in ctx->adj); 2: the adjoint's replay (warp schedule over
// ctx->adj's packet list, no peel-offs).
// Validated launch parameters of packets lo..hi of an np-packet iteration:
// the packet split (newdisktherm_5_fuv.f90:158-191), generator seeds
// (set_all_seeds), the model and tally views of the context.
static int make_params(mcrt_ctx* ctx, int64_t np, int64_t lo, int64_t hi, int32_t iter, int32_t ipeel, int32_t seed1,
                       int32_t seed2, int32_t generator, LaunchParams& P) {
  if (!ctx) return MCRT_ERR_ARG;
  if (!ctx->have_grid || !ctx->have_tables) return fail(ctx, MCRT_ERR_STATE, "upload the grid and tables first");
  if (np < 1 || lo < 1 || hi > np || lo > hi) return fail(ctx, MCRT_ERR_ARG, "bad packet range %lld..%lld of %lld", (long long)lo, (long long)hi, (long long)np);
  if (generator < 1 || generator > 32) return fail(ctx, MCRT_ERR_ARG, "generator %d not in 1..32", generator);
  if (seed1 < 1 || seed1 >= 2147483563 || seed2 < 1 || seed2 >= 2147483399) return fail(ctx, MCRT_ERR_ARG, "seeds out of range");
  const mcrt_config& c = ctx->cfg;
  if (c.ilucy != 1) return fail(ctx, MCRT_ERR_UNSUPPORTED, "ilucy=0 (Bjorkman-Wood) stops in the reference (emit_common_2.f90:59-61)");
  CK(cudaSetDevice(ctx->device));
  // packet split (newdisktherm_5_fuv.f90:158-191)
  int64_t npout = (int64_t)(c.isrf_frac * (double)np);
  double rn = c.isrf_frac * (double)np;
  if (rn - (double)npout > 0.5) npout++;
  int64_t ns = (int64_t)((double)np * (1.0 - c.accfrac - c.isrf_frac));
  rn = (double)(float)np * (1.0 - c.accfrac - c.isrf_frac);
  if (rn - (double)ns > 0.5) ns++;
  int64_t npacc = (int64_t)((double)np * c.accfrac);
  int64_t npaccstar = (int64_t)(c.accfrac2 * (double)np);
  const int64_t nsum = ns + npacc + npout;
  if (nsum != np) ns = ns + np - nsum;
  if (npacc > 1 && !ctx->have_acc)
    return fail(ctx, MCRT_ERR_ARG, "accretion packets (accfrac > 0) need ravearr, Ldint and hdisk in mcrt_upload_grid");
  if (ctx->have_sg && !ctx->have_draine)
    return fail(ctx, MCRT_ERR_UNSUPPORTED, "the grid has small-grain components (ids 5-8): upload the Draine spectra (mcrt_tables.draine)");
  if (ctx->have_sg && std::max(ctx->imean_max, 2) > ctx->dm.nemit)
    return fail(ctx, MCRT_ERR_ARG, "imean selects Draine row %d of %d", std::max(ctx->imean_max, 2), ctx->dm.nemit);
  if (npout > 0 && !ctx->have_isrf)
    return fail(ctx, MCRT_ERR_ARG, "external-illumination packets (isrf_frac > 0) need the isrf table in mcrt_upload_tables");
  if (c.output_imfilt && ipeel == 1 && !ctx->dm.filtwave)
    return fail(ctx, MCRT_ERR_ARG, "filter-band images (output_imfilt) need nwfilt, filtwave and filtphi in mcrt_upload_tables");
  if (c.output_imsparse && ipeel == 1 && !ctx->dm.sparse_levels)
    return fail(ctx, MCRT_ERR_ARG, "nested images (output_imsparse) need sparse_levels in mcrt_upload_tables");
  // generator seeds (set_all_seeds)
  int64_t g1 = seed1, g2 = seed2;
  for (int g = 2; g <= generator; ++g) { g1 = mulmod_h(2082007225, g1, 2147483563); g2 = mulmod_h(784306273, g2, 2147483399); }
  std::memset(&P, 0, sizeof P);
  P.m = ctx->dm;
  DevModel& m = P.m;
  m.nrg = c.nrg; m.ntg = c.ntg; m.npg = c.npg; m.nopac = c.nopac; m.nlammax = c.nlammax; m.nT = c.nT; m.nnu = c.nnu;
  m.nhnu = c.nhnu; m.nfreq = c.nfreq; m.nmu = c.nmu; m.nph = c.nph; m.nap = c.nap; m.npeel = c.npeel; m.nxhst = c.nxhst;
  m.output_imcube = c.output_imcube; m.partial_peeloff = c.partial_peeloff; m.limb = c.limb; m.iplanckst = c.iplanckst;
  m.idust = c.idust; m.iffuv = c.iffuv; m.ispot = c.ispot; m.nspot = c.nspot;
  m.ncell = ctx->ncell; m.nsed = ctx->nsed; m.npsed = ctx->npsed; m.nimg = ctx->nimg;
  m.output_imfilt = c.output_imfilt ? 1 : 0; m.nfilt = c.nfilt; m.nwfiltmax = c.nwfiltmax; m.nimgb = ctx->nimgb;
  m.output_imsparse = c.output_imsparse ? 1 : 0; m.sparse_dim = c.sparse_dim; m.sparse_nlev = c.sparse_nlev;
  m.sparse_nnu = c.sparse_nnu; m.sparse_lognu_min = c.sparse_lognu_min; m.sparse_lognu_max = c.sparse_lognu_max;
  m.nims = ctx->nims;
  m.rstar = c.rstar; m.rmincgs = c.rstar * 6.9598e10; m.tstar = c.tstar; m.tshock = c.tshock; m.fspot = c.fspot;
  m.rmaxi = c.rmaxi; m.fractxh = 2.0 * c.rmaxi / (double)c.nxhst; m.numin = c.numin; m.lnurat = c.lnurat;
  m.ifuv_ori = c.ifuv_ori;
  m.cspot1 = c.cspot1; m.sspot1 = c.sspot1; m.scspot1 = c.scspot1; m.ssspot1 = c.ssspot1;
  m.cspot2 = c.cspot2; m.sspot2 = c.sspot2; m.scspot2 = c.scspot2; m.ssspot2 = c.ssspot2; m.csprad = c.csprad;
  for (int s = 0; s < kMaxSlot; ++s) {      // slot -> first slot on the same wavelength grid
    m.slot_grid[s] = s;
    if (s >= m.nslot) continue;
    for (int k = 0; k < s; ++k)
      if (ctx->species_grid[m.slot_species[k] - 1] == ctx->species_grid[m.slot_species[s] - 1]) { m.slot_grid[s] = k; break; }
  }
  P.t = ctx->dt;
  P.np = np; P.lo = lo; P.hi = hi;
  if (iter < 1) return fail(ctx, MCRT_ERR_ARG, "iter must be >= 1");
  P.block0 = (int64_t)(iter - 1) * np;
  P.ns = ns; P.npacc = npacc; P.npaccstar = npaccstar;
  P.ipeel = ipeel ? 1 : 0;
  P.nphot_diff = (double)ns * (double)(hi - lo + 1) / (double)np;
  ctx->last_nphot_diff = P.nphot_diff;
  ctx->last_ns = (double)ns;
  P.ips = (c.rddust > 100.0) ? 1 : 0;
  P.g1 = (int32_t)g1; P.g2 = (int32_t)g2;
  P.next = ctx->d_next;
  P.log = ctx->d_log;
  P.nlog = ctx->nlog;
  P.err = ctx->d_err;
  P.event_batch = ctx->event_batch;
  P.walk_limit = ctx->walk_limit;
  return MCRT_OK;
}

// The wavefront loop of one packet range as one graph launch (no peel-off
// queue, no adjoint): the loop's decisions run on the device
// (capture_wave_loop), so the host waits once instead of after every walk
// launch.  The graph is captured again when the launch parameters change;
// the iteration enters through block0_dev, which the graph's first node
// copies from pinned host memory.  Kernel times come from the loop's own
// %globaltimer stamps.
static int run_wave_device_loop(mcrt_ctx* ctx, const LaunchParams& P, const WaveArgs& W, int64_t npk,
                                unsigned long long tail_live, bool mixed) {
  if (!ctx->d_block0) {
    int rc = dalloc(ctx, &ctx->d_block0, 1);
    if (rc) return rc;
    CK(cudaHostAlloc((void**)&ctx->h_block0, sizeof(int64_t), cudaHostAllocDefault));
    CK(cudaHostAlloc((void**)&ctx->h_ctl, sizeof(WaveCtl), cudaHostAllocDefault));
    CK(cudaStreamCreateWithFlags(&ctx->wl_body, cudaStreamNonBlocking));
  }
  LaunchParams K = P;
  K.block0 = 0;
  K.block0_dev = ctx->d_block0;
  const unsigned long long max_waves = (unsigned long long)ctx->wave_limit;
  const bool same = ctx->wl_exec && std::memcmp(&K, &ctx->wl_params, sizeof K) == 0 &&
                    std::memcmp(&W, &ctx->wl_w, sizeof W) == 0 && ctx->wl_tail == tail_live &&
                    ctx->wl_max == max_waves && ctx->wl_npk == npk;
  if (!same) {
    if (ctx->wl_exec) cudaGraphExecDestroy(ctx->wl_exec);
    if (ctx->wl_graph) cudaGraphDestroy(ctx->wl_graph);
    ctx->wl_exec = nullptr;
    ctx->wl_graph = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ec = cudaMemcpyAsync(ctx->d_block0, ctx->h_block0, sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream);
    if (ec == cudaSuccess)
      ec = capture_wave_loop(K, W, ctx->d_next, ctx->dt.cnt, npk, tail_live, max_waves, mixed, ctx->nsm, ctx->stream,
                             ctx->wl_body);
    cudaGraph_t gr = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &gr);
    if (ec != cudaSuccess || ee != cudaSuccess) {
      if (gr) cudaGraphDestroy(gr);
      return fail(ctx, MCRT_ERR_CUDA, "wave loop graph capture: %s", cudaGetErrorString(ec != cudaSuccess ? ec : ee));
    }
    ctx->wl_graph = gr;
    CK(cudaGraphInstantiate(&ctx->wl_exec, gr, 0));
    ctx->wl_params = K;
    ctx->wl_w = W;
    ctx->wl_tail = tail_live;
    ctx->wl_max = max_waves;
    ctx->wl_npk = npk;
  }
  *ctx->h_block0 = P.block0;
  CK(cudaGraphLaunch(ctx->wl_exec, ctx->stream));
  CK(cudaMemcpyAsync(ctx->h_ctl, ctx->d_wctl, sizeof(WaveCtl), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const WaveCtl& c = *ctx->h_ctl;
  ctx->last_waves = (int64_t)c.pad1;
  ctx->kt_ms[0] = 1e-6 * (double)c.walk_ns;      // walk, event, tail (kernel classes of wave_stats)
  ctx->kt_ms[1] = 1e-6 * (double)c.ev_ns;
  ctx->kt_ms[2] = 1e-6 * (double)c.tail_ns;
  ctx->kt_launch[0] = ctx->kt_launch[1] = (int64_t)c.pad1;
  ctx->kt_launch[2] = 1;
  ctx->kt_walks = (int64_t)c.walks;
  ctx->h_wctl[5] = c.walk_cross;
  if (c.pad2)                          // the packets in flight were abandoned; the context stays usable
    return fail(ctx, MCRT_ERR_TIMEOUT, "wavefront loop stopped after %llu waves with packets in flight", c.pad1);
  return MCRT_OK;
}

static int run_iteration_impl(mcrt_ctx* ctx, int64_t np, int64_t lo, int64_t hi, int32_t iter, int32_t ipeel,
                              int32_t seed1, int32_t seed2, int32_t generator, int adj_mode) {
  LaunchParams P;
  std::memset(&P, 0, sizeof P);         // padding too: the device loop compares launch parameters bytewise
  {
    const int rc0 = make_params(ctx, np, lo, hi, iter, ipeel, seed1, seed2, generator, P);
    if (rc0) return rc0;
  }
  const mcrt_config& c = ctx->cfg;
  const int64_t npk = hi - lo + 1;
  const bool mixed = ctx->precision == MCRT_PREC_MIXED;
  const bool wave = adj_mode == 1 || (adj_mode == 0 && ctx->schedule == MCRT_SCHED_WAVE);
  const bool warp = !wave && (adj_mode == 2 || ctx->schedule == MCRT_SCHED_WARP || mixed);   // the mixed build has no per-thread kernel
  if (adj_mode) {
    P.adj = ctx->adj;
    P.adj.mode = adj_mode;
  }
  // peel-offs go through the job queue and the peel-off kernel
  const bool queue = P.ipeel && (warp || wave) && ctx->dm.nslot <= kJobSlots && c.npeel > 0;
  const int64_t wave_slots = wave ? std::min<int64_t>(ctx->wave_pool, npk) : 0;
  if (queue) {
    // the wavefront loop drains the queue once fewer than one wave of jobs
    // (at most one per slot) is left
    // The tail launch of the wavefront loop cannot drain the queue while it
    // runs: the remaining interactions of its packets (the heavy-tailed
    // histories of optically thick regions, several per live packet) must
    // fit, else their peel-offs are walked inline.
    const bool exact = wave && ctx->wave_jobs > 0;    // capacity set by mcrt_set_wave_pool
    const int64_t want = exact ? std::max<int64_t>(ctx->wave_jobs, 2 * wave_slots)
                         : wave ? std::min<int64_t>(std::max<int64_t>(16 * wave_slots, 8 * ctx->chunk_packets),
                                                    (int64_t)1 << 26)
                                : 8 * ctx->chunk_packets;
    if (ctx->job_cap < want || (exact && ctx->job_cap != want)) {
      if (ctx->d_jobs) dfree(ctx, ctx->d_jobs);
      ctx->d_jobs = nullptr;
      ctx->job_cap = 0;
      int rc = dalloc(ctx, &ctx->d_jobs, (size_t)want);
      if (rc) return rc;
      ctx->job_cap = want;
    }
    if ((ctx->cfg.output_imfilt || ctx->cfg.output_imsparse) && ctx->job_nub_cap != ctx->job_cap) {   // each job's frequency
      if (ctx->d_job_nub) dfree(ctx, ctx->d_job_nub);
      ctx->d_job_nub = nullptr;
      ctx->job_nub_cap = 0;
      int rc = dalloc(ctx, &ctx->d_job_nub, (size_t)ctx->job_cap);
      if (rc) return rc;
      ctx->job_nub_cap = ctx->job_cap;
    }
  }
  if (wave && ctx->wave_cap < wave_slots) {
    if (ctx->d_recs) dfree(ctx, ctx->d_recs);
    if (ctx->d_walkq) dfree(ctx, ctx->d_walkq);
    if (ctx->d_evq) dfree(ctx, ctx->d_evq);
    ctx->d_recs = nullptr; ctx->d_walkq = ctx->d_evq = nullptr;
    ctx->wave_cap = 0;
    int rc;
    if ((rc = dalloc(ctx, &ctx->d_recs, (size_t)wave_slots)) || (rc = dalloc(ctx, &ctx->d_walkq, (size_t)wave_slots)) ||
        (rc = dalloc(ctx, &ctx->d_evq, (size_t)wave_slots)))
      return rc;
    ctx->wave_cap = wave_slots;
  }
  if (wave && !ctx->d_wctl) {
    int rc = dalloc(ctx, &ctx->d_wctl, 1);
    if (rc) return rc;
    CK(cudaHostAlloc((void**)&ctx->h_wctl, 6 * sizeof(unsigned long long), cudaHostAllocDefault));
    for (auto& p : ctx->kt_ev)
      for (auto& e : p) CK(cudaEventCreate(&e));
  }
  P.jobs = queue ? ctx->d_jobs : nullptr;
  P.job_nub = (queue && (ctx->cfg.output_imfilt || ctx->cfg.output_imsparse)) ? ctx->d_job_nub : nullptr;
  P.njobs = ctx->d_next + 1;
  P.job_cap = ctx->job_cap;
  const int peel_grid = ctx->nsm * (mixed ? peel_mixed_blocks_per_sm() : peel_fp64_blocks_per_sm());
  int64_t launches = 0;                     // kernels this call launches (MCRT_C_LAUNCHES)
  bool devloop = false;                     // the wavefront loop ran as one graph launch
  // device time per kernel class (wavefront schedule): events around each
  // launch, read back at the next host synchronisation
  enum { KT_WALK = 0, KT_EVENT = 1, KT_TAIL = 2, KT_PEEL = 3 };
  if (wave) {
    for (int k = 0; k < 4; ++k) { ctx->kt_ms[k] = 0.0; ctx->kt_pending[k] = false; ctx->kt_launch[k] = 0; }
    ctx->kt_walks = ctx->kt_walk_cross = 0;
  }
  auto kt_begin = [&](int k) -> int {
    if (!wave) return MCRT_OK;
    if (ctx->kt_pending[k]) {             // the class ran again before a host synchronisation: keep its time
      float f = 0.f;
      CK(cudaEventSynchronize(ctx->kt_ev[k][1]));
      CK(cudaEventElapsedTime(&f, ctx->kt_ev[k][0], ctx->kt_ev[k][1]));
      ctx->kt_ms[k] += f;
      ctx->kt_pending[k] = false;
    }
    CK(cudaEventRecord(ctx->kt_ev[k][0], ctx->stream));
    return MCRT_OK;
  };
  auto kt_end = [&](int k) -> int {
    if (!wave) return MCRT_OK;
    CK(cudaEventRecord(ctx->kt_ev[k][1], ctx->stream));
    ctx->kt_pending[k] = true;
    ++ctx->kt_launch[k];
    return MCRT_OK;
  };
  auto kt_collect = [&]() -> int {        // after a host synchronisation
    for (int k = 0; k < 4; ++k) {
      if (!ctx->kt_pending[k]) continue;
      float f = 0.f;
      CK(cudaEventElapsedTime(&f, ctx->kt_ev[k][0], ctx->kt_ev[k][1]));
      ctx->kt_ms[k] += f;
      ctx->kt_pending[k] = false;
    }
    return MCRT_OK;
  };
  // njobs_now: jobs in the queue at this launch (adjoint record bookkeeping)
  auto launch_peel = [&](int64_t njobs_now) -> int {
    ++launches;
    if (adj_mode == 1) {
      const int64_t n = std::min<int64_t>(njobs_now, ctx->job_cap);
      if (ctx->adj_rec_used + n > ctx->adj.rec_cap) {   // grow the records (no kernel writes them now)
        int rc = adjoint_grow(ctx, ctx->adj_rec_used + n);
        if (rc) return rc;
        P.adj.rec_key = ctx->adj.rec_key;
        P.adj.rec_c = ctx->adj.rec_c;
        P.adj.rec_cap = ctx->adj.rec_cap;
      }
      P.adj.rec_base = ctx->adj_rec_used;
      ctx->adj_rec_used += n;
    }
    int rc = kt_begin(KT_PEEL);
    if (rc) return rc;
    cudaError_t e = mixed ? launch_peel_mixed(P, ctx->d_next + 2, peel_grid, ctx->stream)
                          : launch_peel_fp64(P, ctx->d_next + 2, peel_grid, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "peel-off launch: %s", cudaGetErrorString(e));
    return kt_end(KT_PEEL);
  };
  if (!ctx->h_geom) CK(cudaHostAlloc((void**)&ctx->h_geom, 2 * sizeof(unsigned long long), cudaHostAllocDefault));
  CK(cudaMemcpyAsync(ctx->h_geom, ctx->dt.cnt + MCRT_C_GEOM_FAIL, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  if (wave) {
    // Wavefront loop: event launch (emission / interactions / exits up to
    // the next walk), walk launch (every queued walk to its next event).
    // The host reads the queue sizes after every walk launch and drains the
    // peel-off job queue before it can overflow.  Once every packet of the
    // range has started and few are left in flight, one tail launch
    // finishes them without per-wave synchronisation.
    WaveArgs W{};
    W.recs = ctx->d_recs;
    W.walkq = ctx->d_walkq;
    W.evq = ctx->d_evq;
    W.ctl = ctx->d_wctl;
    W.slots = wave_slots;
    W.walk_batch = ctx->wave_batch;
    const int egrid = ctx->nsm * (mixed ? wave_event_mixed_blocks_per_sm() : wave_event_fp64_blocks_per_sm());
    const int wgrid = ctx->nsm * (mixed ? wave_walk_mixed_blocks_per_sm() : wave_walk_fp64_blocks_per_sm());
    const int tgrid = ctx->nsm * (mixed ? wave_tail_mixed_blocks_per_sm() : wave_tail_fp64_blocks_per_sm());
    const unsigned long long tail_live = adj_mode ? 0ull
                                         : ctx->wave_tail < 0 ? (unsigned long long)tgrid * kTransportBlock * 8ull
                                                              : (unsigned long long)ctx->wave_tail;
    devloop = ctx->wave_device_loop != 0 && !queue && adj_mode == 0;
    if (devloop) {
      int rc = run_wave_device_loop(ctx, P, W, npk, tail_live, mixed);
      if (rc) return rc;
    } else {
    CK(cudaMemsetAsync(ctx->d_next, 0, 4 * sizeof(unsigned long long), ctx->stream));
    cudaError_t e = launch_wave_init(W, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "wave init: %s", cudaGetErrorString(e));
    ++launches;
    // every wave advances each live packet by at least one event, and a
    // packet ends after at most 1e8 events (the event watchdog)
    const int64_t max_waves = ctx->wave_limit;
    int64_t waves = 0;
    // h: n_front, n_back, packets started, peel jobs, walks of this wave, walk crossings so far
    unsigned long long* h = ctx->h_wctl;
    int rc;
    for (;;) {
      CK(cudaMemsetAsync(&ctx->d_wctl->n_walk, 0, 2 * sizeof(unsigned long long), ctx->stream));
      if ((rc = kt_begin(KT_EVENT))) return rc;
      e = mixed ? launch_wave_event_mixed(P, W, egrid, ctx->stream) : launch_wave_event_fp64(P, W, egrid, ctx->stream);
      if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "wave event launch: %s", cudaGetErrorString(e));
      if ((rc = kt_end(KT_EVENT))) return rc;
      CK(cudaMemsetAsync(&ctx->d_wctl->n_front, 0, 3 * sizeof(unsigned long long), ctx->stream));
      if ((rc = kt_begin(KT_WALK))) return rc;
      e = mixed ? launch_wave_walk_mixed(P, W, wgrid, ctx->stream) : launch_wave_walk_fp64(P, W, wgrid, ctx->stream);
      if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "wave walk launch: %s", cudaGetErrorString(e));
      if ((rc = kt_end(KT_WALK))) return rc;
      ++waves;
      launches += 2;
      CK(cudaMemcpyAsync(h, &ctx->d_wctl->n_front, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaMemcpyAsync(h + 2, ctx->d_next, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaMemcpyAsync(h + 4, &ctx->d_wctl->n_walk, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      if ((rc = kt_collect())) return rc;
      ctx->kt_walks += (int64_t)h[4];
      const unsigned long long live = h[0] + h[1];
#ifdef MCRT_WAVE_TRACE
      fprintf(stderr, "wave %lld live %llu interactions %llu started %llu jobs %llu\n", (long long)waves, live, h[0],
              h[2], h[3]);
#endif
      if (live == 0) break;
      if (waves >= max_waves)                // the packets in flight are abandoned; the context stays usable
        return fail(ctx, MCRT_ERR_TIMEOUT, "wavefront loop stopped after %lld waves with %llu packets in flight",
                    (long long)waves, live);
      const bool tail = tail_live > 0 && (int64_t)h[2] >= npk && live <= tail_live;
      if (queue && ((int64_t)h[3] + wave_slots > ctx->job_cap || (tail && h[3] > 0))) {
        CK(cudaMemsetAsync(ctx->d_next + 2, 0, sizeof(unsigned long long), ctx->stream));
        if ((rc = launch_peel((int64_t)h[3]))) return rc;
        CK(cudaMemsetAsync(ctx->d_next + 1, 0, sizeof(unsigned long long), ctx->stream));
      }
      if (tail) {
        LaunchParams T = P;
        T.fetch_off = 1;
        CK(cudaMemsetAsync(&ctx->d_wctl->n_walk, 0, 2 * sizeof(unsigned long long), ctx->stream));
        if ((rc = kt_begin(KT_TAIL))) return rc;
        e = mixed ? launch_wave_tail_mixed(T, W, tgrid, ctx->stream) : launch_wave_tail_fp64(T, W, tgrid, ctx->stream);
        if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "wave tail launch: %s", cudaGetErrorString(e));
        if ((rc = kt_end(KT_TAIL))) return rc;
        ++launches;
        break;
      }
    }
    if (queue) {
      CK(cudaMemcpyAsync(h + 3, ctx->d_next + 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      CK(cudaMemsetAsync(ctx->d_next + 2, 0, sizeof(unsigned long long), ctx->stream));
      if ((rc = launch_peel((int64_t)h[3]))) return rc;
    }
    CK(cudaMemcpyAsync(h + 5, &ctx->d_wctl->walk_cross, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       ctx->stream));
    ctx->last_waves = waves;
    }
  }
  int per_sm = wave ? 1 : ctx->precision == MCRT_PREC_FP64
                              ? (warp ? transport_sched_fp64_blocks_per_sm() : transport_fp64_blocks_per_sm())
                              : transport_mixed_blocks_per_sm();
  const int full_grid = ctx->nsm * std::max(per_sm, 1);
  const int64_t chunk = queue ? ctx->chunk_packets : npk;
  for (int64_t c_lo = lo; !wave && c_lo <= hi; c_lo += chunk) {
    const int64_t c_hi = std::min(hi, c_lo + chunk - 1);
    P.lo = c_lo;
    P.hi = c_hi;
    CK(cudaMemsetAsync(ctx->d_next, 0, 4 * sizeof(unsigned long long), ctx->stream));
    const int64_t want = (c_hi - c_lo + 1 + kTransportBlock - 1) / kTransportBlock;
    const int grid = (int)std::min<int64_t>(full_grid, std::max<int64_t>(want, 1));
    cudaError_t e = ctx->precision == MCRT_PREC_FP64
                        ? (warp ? launch_transport_sched_fp64(P, grid, ctx->stream) : launch_transport_fp64(P, grid, ctx->stream))
                        : launch_transport_mixed(P, grid, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "transport launch: %s", cudaGetErrorString(e));
    ++launches;
    if (queue) {
      int rc = launch_peel(0);
      if (rc) return rc;
    }
  }
  P.lo = lo;
  P.hi = hi;
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  cudaError_t ef = launch_diffusion_finalize(P.m, ctx->dt.ndiff, ctx->d_tdust0, ctx->d_tdust, P.nphot_diff, ctx->stream);
  if (ef != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "diffusion finalize: %s", cudaGetErrorString(ef));
  // diffusion_finalize and add_counters (the graph's wave_loop_finish
  // counts its waves and launches, diffusion_finalize included)
  launches += devloop ? 1 : 2;
  add_counters<<<1, 1, 0, ctx->stream>>>(ctx->dt.cnt, (unsigned long long)(wave && !devloop ? ctx->last_waves : 0),
                                         (unsigned long long)launches);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ctx->h_geom + 1, ctx->dt.cnt + MCRT_C_GEOM_FAIL, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaEventSynchronize(ctx->ev1));
  CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->last_ms = ms;
  ctx->last_m = P.m;
  ctx->have_last_run = true;
  if (wave) {
    int rc = kt_collect();
    if (rc) return rc;
    ctx->kt_walk_cross = (int64_t)ctx->h_wctl[5];
  }
  CK(cudaGetLastError());
  // packets lost to geometry failures (the reference stops the run on one):
  // the tallies hold every other packet; above the set fraction the call
  // reports it
  const unsigned long long lost = ctx->h_geom[1] - ctx->h_geom[0];
  if (ctx->geom_fraction >= 0.0 && (double)lost > ctx->geom_fraction * (double)npk)
    return fail(ctx, MCRT_ERR_GEOM, "%llu of %lld packets lost to geometry failures (limit %g per packet)", lost,
                (long long)npk, ctx->geom_fraction);
  return MCRT_OK;
}

int mcrt_run_iteration(mcrt_ctx* ctx, int64_t np, int64_t lo, int64_t hi, int32_t iter, int32_t ipeel,
                       int32_t seed1, int32_t seed2, int32_t generator) {
  return run_iteration_impl(ctx, np, lo, hi, iter, ipeel, seed1, seed2, generator, 0);
}

namespace {

// per-packet record arrays for a chunk of npk packets (kept between calls)
int adjoint_buffers(mcrt_ctx* ctx, int64_t npk) {
  AdjointArgs& A = ctx->adj;
  int rc;
  if (ctx->adj_npk_cap < npk) {
    for (void* q : {(void*)A.rec_key, (void*)A.rec_c, (void*)A.start, (void*)A.end, (void*)A.list})
      if (q) dfree(ctx, q);
    A.rec_key = nullptr; A.rec_c = nullptr; A.start = nullptr; A.end = nullptr;
    A.list = nullptr; ctx->adj_npk_cap = 0;
    const int64_t cap = std::max<int64_t>(16 * npk, 1 << 16);
    unsigned long long* rk;
    double* rcv;
    int64_t *st, *en;
    int32_t* ls;
    if ((rc = dalloc(ctx, &rk, cap)) || (rc = dalloc(ctx, &rcv, cap)) || (rc = dalloc(ctx, &st, npk)) ||
        (rc = dalloc(ctx, &en, npk)) || (rc = dalloc(ctx, &ls, npk)))
      return rc;
    A.rec_key = rk; A.rec_c = rcv; A.start = st; A.end = en; A.list = ls;
    A.rec_cap = cap;
    ctx->adj_npk_cap = npk;
    ctx->adj_sort_cap = 0;
  }
  return MCRT_OK;
}

// One chunk lo..hi of the packet range: forward pass, record sort, replay.
// The chunk's gradient and objective are left in A.grad / A.obj (zeroed
// here).  *too_many: the chunk holds 2^31 records or more (the device sort
// takes a 32-bit count); nothing is sorted or replayed then.
int adjoint_chunk(mcrt_ctx* ctx, int64_t np, int64_t lo, int64_t hi, int32_t iter, int32_t seed1, int32_t seed2,
                  int32_t generator, double* total_ms_out, bool* too_many) {
  AdjointArgs& A = ctx->adj;
  const int64_t ncell = ctx->ncell;
  const int64_t npk = hi - lo + 1;
  int rc;
  *too_many = false;
  if ((rc = adjoint_buffers(ctx, npk))) return rc;
  CK(cudaMemsetAsync(A.grad, 0, (size_t)ncell * 10 * 8, ctx->stream));
  CK(cudaMemsetAsync(A.obj, 0, 8, ctx->stream));
  CK(cudaMemsetAsync(A.rec_key, 0xff, (size_t)A.rec_cap * 8, ctx->stream));
  CK(cudaMemsetAsync(A.rec_c, 0, (size_t)A.rec_cap * 8, ctx->stream));
  CK(cudaMemsetAsync((void*)A.start, 0, (size_t)npk * 8, ctx->stream));
  CK(cudaMemsetAsync((void*)A.end, 0, (size_t)npk * 8, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_adj_nlist, 0, 8, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream));
  ctx->adj_rec_used = 0;
  double total_ms = 0.0;
  // forward pass: the iteration with its peel-offs, records and -C*tau terms
  if ((rc = run_iteration_impl(ctx, np, lo, hi, iter, 1, seed1, seed2, generator, 1))) return rc;
  total_ms += ctx->last_ms;
  int32_t herr = 0;
  CK(cudaMemcpy(&herr, ctx->d_err, 4, cudaMemcpyDeviceToHost));
  if (herr) return fail(ctx, MCRT_ERR_ARG, "adjoint: peel-off record capacity exceeded");
  // records by (packet, event); the range of each packet; the packet list
  const int64_t nrec = ctx->adj_rec_used;
  cudaEvent_t e0 = ctx->ev0, e1 = ctx->ev1;
  CK(cudaEventRecord(e0, ctx->stream));
  if (nrec > INT32_MAX) {               // before any buffer changes: the caller halves the chunk
    *too_many = true;
    return MCRT_OK;
  }
  if (nrec > ctx->adj_sort_cap) {      // sorted copies and scratch for nrec records
    for (void* q : {(void*)A.skey, (void*)A.sc, ctx->d_adj_tmp})
      if (q) dfree(ctx, q);
    const int64_t cap32 = std::min<int64_t>(std::max<int64_t>(nrec, 2 * ctx->adj_sort_cap), INT32_MAX);
    A.skey = nullptr; A.sc = nullptr; ctx->d_adj_tmp = nullptr;
    ctx->adj_sort_cap = 0;
    unsigned long long* sk;
    double* scv;
    if ((rc = dalloc(ctx, &sk, cap32)) || (rc = dalloc(ctx, &scv, cap32))) return rc;
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, A.rec_key, sk, A.rec_c, scv, (int)cap32));
    if ((rc = dalloc(ctx, (char**)&ctx->d_adj_tmp, std::max<size_t>(tmp, 1)))) return rc;
    ctx->adj_tmp_bytes = tmp;
    A.skey = sk;
    A.sc = scv;
    ctx->adj_sort_cap = cap32;
  }
  if (nrec > 0) {
    size_t tmp = ctx->adj_tmp_bytes;
    CK(cub::DeviceRadixSort::SortPairs(ctx->d_adj_tmp, tmp, A.rec_key, (unsigned long long*)A.skey, A.rec_c,
                                       (double*)A.sc, (int)nrec, 0, 64, ctx->stream));
    adjoint_ranges<<<(int)std::min<int64_t>((nrec + 255) / 256, 8192), 256, 0, ctx->stream>>>(
        A.skey, nrec, (int64_t*)A.start, (int64_t*)A.end, (int32_t*)A.list, ctx->d_adj_nlist);
    CK(cudaGetLastError());
  }
  unsigned long long nlist = 0;
  CK(cudaMemcpyAsync(&nlist, ctx->d_adj_nlist, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaEventRecord(e1, ctx->stream));
  CK(cudaEventSynchronize(e1));
  float sort_ms = 0.f;
  CK(cudaEventElapsedTime(&sort_ms, e0, e1));
  total_ms += sort_ms;
  // replay pass: the packets with peel-off records, scoring their segments
  A.nlist = (int64_t)nlist;
  if (nlist > 0) {
    if ((rc = run_iteration_impl(ctx, np, lo, hi, iter, 0, seed1, seed2, generator, 2))) return rc;
    total_ms += ctx->last_ms;
  }
  *total_ms_out += total_ms;
  return MCRT_OK;
}

__global__ void add_doubles(const double* src, double* dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] += src[i];
}

// The control variate from a learning replay: the mean A per bin, 0 where
// fewer than min_count segments started in the bin.
__global__ void cv_table(const double* sum, const double* cnt, double min_count, double* tab, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    tab[i] = cnt[i] >= min_count ? sum[i] / cnt[i] : 0.0;
}

// Chunks of lo..hi; with `sum` the chunk gradients and objectives are added
// into sum[ncell*10 + 1].
int adjoint_range(mcrt_ctx* ctx, int64_t np, int64_t lo, int64_t hi, int32_t iter, int32_t seed1, int32_t seed2,
                  int32_t generator, double* sum, double* total_ms) {
  AdjointArgs& A = ctx->adj;
  const int64_t ncell = ctx->ncell;
  int rc;
  int64_t chunk = std::min<int64_t>(hi - lo + 1, ctx->adj_chunk);
  for (int64_t c_lo = lo; c_lo <= hi;) {
    const int64_t c_hi = std::min(hi, c_lo + chunk - 1);
    bool too_many = false;
    if ((rc = adjoint_chunk(ctx, np, c_lo, c_hi, iter, seed1, seed2, generator, total_ms, &too_many))) return rc;
    if (too_many) {
      if (c_hi == c_lo) return fail(ctx, MCRT_ERR_ARG, "adjoint: one packet with 2^31 peel-off records");
      chunk = std::max<int64_t>(1, (c_hi - c_lo + 1) / 2);
      continue;
    }
    if (sum) {
      add_doubles<<<256, 256, 0, ctx->stream>>>(A.grad, sum, ncell * 10);
      add_doubles<<<1, 32, 0, ctx->stream>>>(A.obj, sum + ncell * 10, 1);
      CK(cudaGetLastError());
    }
    c_lo = c_hi + 1;
  }
  return MCRT_OK;
}

}  // namespace

int mcrt_set_adjoint_chunk(mcrt_ctx* ctx, int64_t packets) {
  if (!ctx || packets < 1 || packets >= ((int64_t)1 << 31)) return MCRT_ERR_ARG;
  ctx->adj_chunk = packets;
  return MCRT_OK;
}

int mcrt_set_wave_loop(mcrt_ctx* ctx, int32_t device_loop) {
  if (!ctx || (device_loop != 0 && device_loop != 1)) return MCRT_ERR_ARG;
  ctx->wave_device_loop = device_loop;
  return MCRT_OK;
}

int mcrt_set_adjoint_baseline(mcrt_ctx* ctx, int32_t nfb, int32_t ndir, int64_t pilot_packets, double min_count) {
  if (!ctx) return MCRT_ERR_ARG;
  if (nfb == 0) { ctx->cv_nfb = 0; return MCRT_OK; }
  if (nfb < 0 || nfb > 1000 || (ndir != 1 && ndir != 4) || pilot_packets < 1 || !(min_count >= 1.0))
    return fail(ctx, MCRT_ERR_ARG, "adjoint baseline: need 1 <= nfb <= 1000, ndir 1 or 4, pilot >= 1, min_count >= 1");
  ctx->cv_nfb = nfb;
  ctx->cv_ndir = ndir;
  ctx->cv_pilot = pilot_packets;
  ctx->cv_min_count = min_count;
  return MCRT_OK;
}

int mcrt_adjoint(mcrt_ctx* ctx, int64_t np, int64_t lo, int64_t hi, int32_t iter, int32_t seed1, int32_t seed2,
                 int32_t generator, const double* lam_psed, const double* lam_img, double* grad, double* objective) {
  if (!ctx || !lam_psed || !grad || !objective) return MCRT_ERR_ARG;
  if (!ctx->have_grid || !ctx->have_tables) return fail(ctx, MCRT_ERR_STATE, "upload the grid and tables first");
  if (np < 1 || lo < 1 || hi > np || lo > hi) return fail(ctx, MCRT_ERR_ARG, "bad packet range");
  const mcrt_config& c = ctx->cfg;
  if (c.npeel < 1) return fail(ctx, MCRT_ERR_ARG, "the adjoint differentiates peeled outputs: npeel must be >= 1");
  if (ctx->dm.nslot > kJobSlots) return fail(ctx, MCRT_ERR_UNSUPPORTED, "adjoint needs at most %d opacity species", kJobSlots);
  CK(cudaSetDevice(ctx->device));
  const int64_t ncell = ctx->ncell;
  AdjointArgs& A = ctx->adj;
  int rc;
  // buffers (kept between calls; re-sized for larger ranges)
  if (!A.grad) {
    double *lp, *gr, *ob, *li = nullptr;
    if ((rc = dalloc(ctx, &lp, (size_t)std::max<int64_t>(ctx->npsed, 1))) || (rc = dalloc(ctx, &gr, (size_t)ncell * 10)) ||
        (rc = dalloc(ctx, &ob, 1)) || (ctx->nimg > 0 && (rc = dalloc(ctx, &li, (size_t)ctx->nimg))) ||
        (rc = dalloc(ctx, &ctx->d_adj_nlist, 1)))
      return rc;
    A.lam_psed = lp; A.grad = gr; A.obj = ob; A.lam_img = li;
  }
  CK(cudaMemcpyAsync((void*)A.lam_psed, lam_psed, (size_t)ctx->npsed * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (ctx->nimg > 0) {
    if (lam_img) CK(cudaMemcpyAsync((void*)A.lam_img, lam_img, (size_t)ctx->nimg * 8, cudaMemcpyHostToDevice, ctx->stream));
    else CK(cudaMemsetAsync((void*)A.lam_img, 0, (size_t)ctx->nimg * 8, ctx->stream));
  }
  if (!ctx->d_adj_sum && (rc = dalloc(ctx, &ctx->d_adj_sum, (size_t)ncell * 10 + 1))) return rc;
  CK(cudaMemsetAsync(ctx->d_adj_sum, 0, ((size_t)ncell * 10 + 1) * 8, ctx->stream));
  double total_ms = 0.0;
  A.vtab = nullptr; A.vsum = nullptr; A.vcnt = nullptr; A.all = 0;
  if (ctx->cv_nfb > 0) {
    // Control variate: a learning replay of cv_pilot packets on another
    // generator (independent of lo..hi) gives the mean A per bin; the
    // replay of lo..hi then weights every segment's score by A - mean.
    const int64_t nv = ncell * ctx->cv_nfb * ctx->cv_ndir;
    if (ctx->cv_cap < nv) {
      for (double* q : {ctx->cv_tab, ctx->cv_sum, ctx->cv_cnt})
        if (q) dfree(ctx, q);
      ctx->cv_tab = ctx->cv_sum = ctx->cv_cnt = nullptr;
      ctx->cv_cap = 0;
      if ((rc = dalloc(ctx, &ctx->cv_tab, nv)) || (rc = dalloc(ctx, &ctx->cv_sum, nv)) || (rc = dalloc(ctx, &ctx->cv_cnt, nv)))
        return rc;
      ctx->cv_cap = nv;
    }
    CK(cudaMemsetAsync(ctx->cv_sum, 0, (size_t)nv * 8, ctx->stream));
    CK(cudaMemsetAsync(ctx->cv_cnt, 0, (size_t)nv * 8, ctx->stream));
    A.nfb = ctx->cv_nfb;
    A.ndir = ctx->cv_ndir;
    A.lnumin = log(c.numin);
    A.lnurat = c.lnurat;
    A.vsum = ctx->cv_sum;
    A.vcnt = ctx->cv_cnt;
    A.all = 1;
    rc = adjoint_range(ctx, ctx->cv_pilot, 1, ctx->cv_pilot, iter, seed1, seed2, generator % 32 + 1, nullptr, &total_ms);
    A.vsum = nullptr; A.vcnt = nullptr;
    if (rc) { A.all = 0; return rc; }
    cv_table<<<256, 256, 0, ctx->stream>>>(ctx->cv_sum, ctx->cv_cnt, ctx->cv_min_count, ctx->cv_tab, nv);
    CK(cudaGetLastError());
    A.vtab = ctx->cv_tab;
  }
  // Packets are independent here (diffusion heating is frozen), so the
  // gradient and the objective of lo..hi are the sums over chunks; a chunk
  // whose records would reach 2^31 is redone in halves.
  rc = adjoint_range(ctx, np, lo, hi, iter, seed1, seed2, generator, ctx->d_adj_sum, &total_ms);
  A.vtab = nullptr; A.all = 0;
  if (rc) return rc;
  ctx->last_ms = total_ms;
  CK(cudaMemcpyAsync(grad, ctx->d_adj_sum, (size_t)ncell * 10 * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(objective, ctx->d_adj_sum + ncell * 10, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return MCRT_OK;
}

int mcrt_mark(mcrt_ctx* ctx, int32_t slot) {
  if (!ctx || slot < 0 || slot >= 16) return MCRT_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  if (!ctx->marks[slot]) CK(cudaEventCreate(&ctx->marks[slot]));
  CK(cudaEventRecord(ctx->marks[slot], ctx->stream));
  return MCRT_OK;
}

int mcrt_elapsed_ms(mcrt_ctx* ctx, int32_t a, int32_t b, double* ms) {
  if (!ctx || !ms || a < 0 || a >= 16 || b < 0 || b >= 16 || !ctx->marks[a] || !ctx->marks[b]) return MCRT_ERR_ARG;
  CK(cudaEventSynchronize(ctx->marks[b]));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, ctx->marks[a], ctx->marks[b]));
  *ms = f;
  return MCRT_OK;
}

int mcrt_flush_l2(mcrt_ctx* ctx) {
  if (!ctx) return MCRT_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  const size_t bytes = (size_t)256 << 20;
  if (!ctx->d_flush) { int rc = dalloc(ctx, (char**)&ctx->d_flush, bytes); if (rc) return rc; }
  CK(cudaMemsetAsync(ctx->d_flush, ctx->marks[15] ? 1 : 0, bytes, ctx->stream));
  return MCRT_OK;
}

int mcrt_synchronize(mcrt_ctx* ctx) {
  if (!ctx) return MCRT_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  return MCRT_OK;
}

int mcrt_wave_stats(mcrt_ctx* ctx, double* kernel_ms, int64_t* counts) {
  if (!ctx || !kernel_ms || !counts) return MCRT_ERR_ARG;
  for (int k = 0; k < 4; ++k) {
    kernel_ms[k] = ctx->kt_ms[k];
    counts[k] = ctx->kt_launch[k];
  }
  counts[4] = ctx->kt_walks;
  counts[5] = ctx->kt_walk_cross;
  return MCRT_OK;
}

int mcrt_last_kernel_ms(mcrt_ctx* ctx, double* ms) {
  if (!ctx || !ms) return MCRT_ERR_ARG;
  *ms = ctx->last_ms;
  return MCRT_OK;
}

int mcrt_download_tallies(mcrt_ctx* ctx, mcrt_tallies* out) {
  if (!ctx || !out) return MCRT_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  const DevTallies& t = ctx->dt;
  const int64_t nc = ctx->ncell;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
    if (!dst) return MCRT_OK;
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return MCRT_OK;
  };
  int rc;
  if ((rc = cp(out->nabs, t.nabs, nc * 4)) || (rc = cp(out->dbig, t.dbig, nc * 4)) || (rc = cp(out->dsg, t.dsg, nc * 4)) ||
      (rc = cp(out->killed, t.killed, nc * 4)) || (rc = cp(out->dtauabs, t.dtauabs, nc * 8)) ||
      (rc = cp(out->fuvmean, t.fuvmean, nc * 8)) || (rc = cp(out->scalars, t.scal, MCRT_NSCALARS * 8)) ||
      (rc = cp(out->counters, t.cnt, MCRT_NCOUNTERS * 8)))
    return rc;
  // FP64 device sums -> the reference's REAL arrays
  float* sed[10] = {out->si, out->sq, out->su, out->sv, out->si2, out->sq2, out->su2, out->sv2, out->nums, out->aveinc};
  float* ps[9] = {out->ti, out->tq, out->tu, out->tv, out->ti2, out->tq2, out->tu2, out->tv2, out->numt};
  float* im[4] = {out->image_m_i, out->image_m_q, out->image_m_u, out->image_m_v};
  float* ib[8] = {out->image_b_i, out->image_b_q, out->image_b_u, out->image_b_v,
                  out->image_b_d, out->image_b_s, out->image_b_e, out->image_b_o};
  int64_t nmax = std::max(std::max(std::max(ctx->nsed, ctx->nimgb), ctx->nims), std::max(ctx->npsed, ctx->nimg));
  float* d_f = nullptr;
  if ((rc = scratch(ctx, &d_f, nmax))) return rc;
  std::vector<std::pair<float*, std::pair<const double*, int64_t>>> jobs;
  for (int k = 0; k < 10; ++k) jobs.push_back({sed[k], {t.sed + k * ctx->nsed, ctx->nsed}});
  for (int k = 0; k < 9; ++k) jobs.push_back({ps[k], {t.psed + k * ctx->npsed, ctx->npsed}});
  for (int k = 0; k < 4; ++k) jobs.push_back({im[k], {t.img + k * ctx->nimg, ctx->nimg}});
  for (int k = 0; k < 8; ++k) jobs.push_back({ib[k], {t.imgb + k * ctx->nimgb, ctx->nimgb}});
  float* is[4] = {out->image_ms_i, out->image_ms_q, out->image_ms_u, out->image_ms_v};
  for (int k = 0; k < 4; ++k) jobs.push_back({is[k], {t.ims + k * ctx->nims, ctx->nims}});
  for (auto& j : jobs) {
    if (!j.first || j.second.second == 0) continue;
    const int64_t n = j.second.second;
    to_float<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, ctx->stream>>>(j.second.first, d_f, n);
    if ((rc = cp(j.first, d_f, n * 4))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return MCRT_OK;
}

int mcrt_diskflux(mcrt_ctx* ctx, int64_t np, double ltot_lsol, int32_t ipeel, mcrt_tallies* out) {
  if (!ctx || !out) return MCRT_ERR_ARG;
  if (np < 1 || !(ltot_lsol > 0.0) || !std::isfinite(ltot_lsol))
    return fail(ctx, MCRT_ERR_ARG, "mcrt_diskflux: np must be positive and ltot/lsol finite and positive");
  // the counts, FP64 cell tallies, scalars and counters as downloaded
  mcrt_tallies rest = *out;
  for (float** f : {&rest.si, &rest.sq, &rest.su, &rest.sv, &rest.si2, &rest.sq2, &rest.su2, &rest.sv2, &rest.nums,
                    &rest.aveinc, &rest.ti, &rest.tq, &rest.tu, &rest.tv, &rest.ti2, &rest.tq2, &rest.tu2, &rest.tv2,
                    &rest.numt, &rest.image_m_i, &rest.image_m_q, &rest.image_m_u, &rest.image_m_v,
                    &rest.image_b_i, &rest.image_b_q, &rest.image_b_u, &rest.image_b_v,
                    &rest.image_b_d, &rest.image_b_s, &rest.image_b_e, &rest.image_b_o,
                    &rest.image_ms_i, &rest.image_ms_q, &rest.image_ms_u, &rest.image_ms_v})
    *f = nullptr;
  int rc = mcrt_download_tallies(ctx, &rest);
  if (rc) return rc;
  const mcrt_config& c = ctx->cfg;
  const double rnp = (double)np;
  const float rnorm = (float)(rnp / (double)c.nmu / (double)c.nph / ltot_lsol);   // flux_test.f90:20-21
  const float inorm = (float)(rnp / ltot_lsol);
  const bool peel = ipeel == 1;
  const int64_t nsed = ctx->nsed, npsed = ctx->npsed, nimg = (peel && c.output_imcube) ? ctx->nimg : 0;
  const int64_t nimgb = (peel && c.output_imfilt) ? ctx->nimgb : 0;
  float* d_f = nullptr;
  if ((rc = dalloc(ctx, &d_f, std::max<int64_t>({10 * nsed, 9 * npsed, 4 * nimg, nimgb, 1})))) return rc;
  auto grid = [](int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 4096); };
  auto get = [&](float* dst, const float* src, int64_t n) -> int {
    if (!dst) return MCRT_OK;
    cudaError_t e = cudaMemcpyAsync(dst, src, n * 4, cudaMemcpyDeviceToHost, ctx->stream);
    return e == cudaSuccess ? MCRT_OK : fail(ctx, MCRT_ERR_CUDA, "mcrt_diskflux copy: %s", cudaGetErrorString(e));
  };
  const DevTallies& t = ctx->dt;
  float* sed[10] = {out->si, out->sq, out->su, out->sv, out->si2, out->sq2, out->su2, out->sv2, out->nums, out->aveinc};
  float* ps[9] = {out->ti, out->tq, out->tu, out->tv, out->ti2, out->tq2, out->tu2, out->tv2, out->numt};
  float* im[4] = {out->image_m_i, out->image_m_q, out->image_m_u, out->image_m_v};
  float* ib[8] = {out->image_b_i, out->image_b_q, out->image_b_u, out->image_b_v,
                  out->image_b_d, out->image_b_s, out->image_b_e, out->image_b_o};
  diskflux_sed<<<grid(nsed), 256, 0, ctx->stream>>>(t.sed, nsed, rnorm, d_f);
  for (int a = 0; a < 10 && !rc; ++a) rc = get(sed[a], d_f + a * nsed, nsed);
  if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? MCRT_OK : fail(ctx, MCRT_ERR_CUDA, "mcrt_diskflux sync");
  if (!rc && peel) {
    diskflux_psed<<<grid(npsed), 256, 0, ctx->stream>>>(t.psed, npsed, inorm, d_f);
    for (int a = 0; a < 9 && !rc; ++a) rc = get(ps[a], d_f + a * npsed, npsed);
    if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? MCRT_OK : fail(ctx, MCRT_ERR_CUDA, "mcrt_diskflux sync");
    for (int a = 0; a < 4 && !rc && nimg > 0; ++a) {
      diskflux_img<<<grid(nimg), 256, 0, ctx->stream>>>(t.img + a * nimg, nimg, inorm, d_f);
      rc = get(im[a], d_f, nimg);
      if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? MCRT_OK : fail(ctx, MCRT_ERR_CUDA, "mcrt_diskflux sync");
    }
    for (int a = 0; a < 8 && !rc && nimgb > 0; ++a) {      // flux_test.f90:64-73
      if (!ib[a]) continue;
      diskflux_img<<<grid(nimgb), 256, 0, ctx->stream>>>(t.imgb + a * nimgb, nimgb, inorm, d_f);
      rc = get(ib[a], d_f, nimgb);
      if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? MCRT_OK : fail(ctx, MCRT_ERR_CUDA, "mcrt_diskflux sync");
    }
  } else if (!rc) {                          // ipeel /= 1: the peeled arrays as downloaded (flux_test.f90:44)
    mcrt_tallies pe{};
    pe.ti = out->ti; pe.tq = out->tq; pe.tu = out->tu; pe.tv = out->tv;
    pe.ti2 = out->ti2; pe.tq2 = out->tq2; pe.tu2 = out->tu2; pe.tv2 = out->tv2; pe.numt = out->numt;
    pe.image_m_i = out->image_m_i; pe.image_m_q = out->image_m_q;
    pe.image_m_u = out->image_m_u; pe.image_m_v = out->image_m_v;
    pe.image_b_i = out->image_b_i; pe.image_b_q = out->image_b_q; pe.image_b_u = out->image_b_u;
    pe.image_b_v = out->image_b_v; pe.image_b_d = out->image_b_d; pe.image_b_s = out->image_b_s;
    pe.image_b_e = out->image_b_e; pe.image_b_o = out->image_b_o;
    rc = mcrt_download_tallies(ctx, &pe);
  }
  if (!rc && (out->image_ms_i || out->image_ms_q || out->image_ms_u || out->image_ms_v)) {
    mcrt_tallies ms{};                       // nested images: not normalised by flux_test.f90
    ms.image_ms_i = out->image_ms_i; ms.image_ms_q = out->image_ms_q;
    ms.image_ms_u = out->image_ms_u; ms.image_ms_v = out->image_ms_v;
    rc = mcrt_download_tallies(ctx, &ms);
  }
  cudaError_t le = cudaGetLastError();
  if (!rc && le != cudaSuccess) rc = fail(ctx, MCRT_ERR_CUDA, "mcrt_diskflux: %s", cudaGetErrorString(le));
  dfree(ctx, d_f);
  return rc;
}

int mcrt_accumulate_tallies(mcrt_ctx* ctx, const mcrt_tallies* in) {
  if (!ctx || !in) return MCRT_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  const DevTallies& t = ctx->dt;
  const int64_t nc = ctx->ncell;
  const int64_t nmax = std::max<int64_t>(std::max<int64_t>(std::max<int64_t>(nc, MCRT_NCOUNTERS),
                                                            std::max(ctx->nimgb, ctx->nims)),
                                         std::max(ctx->nsed, std::max(ctx->npsed, ctx->nimg)));
  void* d_in = nullptr;
  int rc = dalloc(ctx, (char**)&d_in, (size_t)nmax * 8);
  if (rc) return rc;
  const int grid = (int)std::min<int64_t>((nmax + 255) / 256, 4096);
  // one host array: copy it to the staging buffer and add it to its device tally
  auto add = [&](const void* h, int kind, void* dst, int64_t n) -> int {
    if (!h || n == 0) return MCRT_OK;
    const size_t esz = (kind == 2) ? 4 : (kind == 3 ? 4 : 8);
    cudaError_t e = cudaMemcpyAsync(d_in, h, (size_t)n * esz, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "accumulate copy: %s", cudaGetErrorString(e));
    add_tally<<<grid, 256, 0, ctx->stream>>>(kind, d_in, dst, n);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "accumulate launch: %s", cudaGetErrorString(e));
    e = cudaStreamSynchronize(ctx->stream);     // the staging buffer is reused by the next array
    if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "accumulate: %s", cudaGetErrorString(e));
    return MCRT_OK;
  };
  // kinds: 0 f64 -> f64, 1 i64 -> u64, 2 f32 -> f64, 3 i32 -> i32
  const float* sed[10] = {in->si, in->sq, in->su, in->sv, in->si2, in->sq2, in->su2, in->sv2, in->nums, in->aveinc};
  const float* ps[9] = {in->ti, in->tq, in->tu, in->tv, in->ti2, in->tq2, in->tu2, in->tv2, in->numt};
  const float* im[4] = {in->image_m_i, in->image_m_q, in->image_m_u, in->image_m_v};
  if ((rc = add(in->nabs, 3, t.nabs, nc)) || (rc = add(in->dbig, 3, t.dbig, nc)) || (rc = add(in->dsg, 3, t.dsg, nc)) ||
      (rc = add(in->killed, 3, t.killed, nc)) || (rc = add(in->dtauabs, 0, t.dtauabs, nc)) ||
      (rc = add(in->fuvmean, 0, t.fuvmean, nc)) || (rc = add(in->scalars, 0, t.scal, MCRT_NSCALARS)) ||
      (rc = add(in->counters, 1, t.cnt, MCRT_NCOUNTERS))) {
    dfree(ctx, d_in);
    return rc;
  }
  for (int k = 0; k < 10 && !rc; ++k) rc = add(sed[k], 2, t.sed + k * ctx->nsed, ctx->nsed);
  for (int k = 0; k < 9 && !rc; ++k) rc = add(ps[k], 2, t.psed + k * ctx->npsed, ctx->npsed);
  for (int k = 0; k < 4 && !rc; ++k) rc = add(im[k], 2, t.img + k * ctx->nimg, ctx->nimg);
  const float* ib[8] = {in->image_b_i, in->image_b_q, in->image_b_u, in->image_b_v,
                        in->image_b_d, in->image_b_s, in->image_b_e, in->image_b_o};
  for (int k = 0; k < 8 && !rc; ++k) rc = add(ib[k], 2, t.imgb + k * ctx->nimgb, ctx->nimgb);
  const float* is[4] = {in->image_ms_i, in->image_ms_q, in->image_ms_u, in->image_ms_v};
  for (int k = 0; k < 4 && !rc; ++k) rc = add(is[k], 2, t.ims + k * ctx->nims, ctx->nims);
  dfree(ctx, d_in);
  return rc;
}

int mcrt_device_tallies_view(mcrt_ctx* ctx, mcrt_device_tallies* out) {
  if (!ctx || !out) return MCRT_ERR_ARG;
  const int64_t nc = ctx->ncell;
  out->f64 = ctx->dt.dtauabs;                 // first member of the allocation
  out->n_f64 = 2 * nc + 10 * ctx->nsed + 9 * ctx->npsed + 4 * ctx->nimg + 8 * ctx->nimgb + 4 * ctx->nims + MCRT_NSCALARS;
  out->u64 = (uint64_t*)ctx->dt.cnt;
  out->n_u64 = MCRT_NCOUNTERS;
  out->i32 = ctx->dt.nabs;
  out->n_i32 = 5 * nc;                        // nabs, dbig, dsg, killed, ndiff
  return MCRT_OK;
}

int mcrt_refresh_diffusion(mcrt_ctx* ctx) {
  if (!ctx) return MCRT_ERR_ARG;
  if (!ctx->have_last_run) return fail(ctx, MCRT_ERR_STATE, "mcrt_refresh_diffusion before any mcrt_run_iteration");
  CK(cudaSetDevice(ctx->device));
  cudaError_t e = launch_diffusion_finalize(ctx->last_m, ctx->dt.ndiff, ctx->d_tdust0, ctx->d_tdust,
                                            std::max(ctx->last_ns, 1.0), ctx->stream);
  if (e != cudaSuccess) return fail(ctx, MCRT_ERR_CUDA, "diffusion refresh: %s", cudaGetErrorString(e));
  CK(cudaStreamSynchronize(ctx->stream));
  return MCRT_OK;
}

int mcrt_setdiffus(mcrt_ctx* ctx, int32_t iter, double massd, double rmaxd, const double* tdave, int32_t* diffus,
                   int32_t* diffdir, int64_t* dcount) {
  if (!ctx || !tdave) return MCRT_ERR_ARG;
  if (!ctx->have_grid || !ctx->have_tables) return fail(ctx, MCRT_ERR_STATE, "upload the grid and tables first");
  if (!ctx->have_acc) return fail(ctx, MCRT_ERR_STATE, "mcrt_setdiffus needs the disk scale heights (mcrt_grid.hdisk)");
  if (ctx->off_kappar < 0) return fail(ctx, MCRT_ERR_STATE, "mcrt_setdiffus needs the Rosseland table (mcrt_tables.kappar)");
  if (!std::isfinite(massd) || !std::isfinite(rmaxd)) return fail(ctx, MCRT_ERR_ARG, "massd and rmaxd must be finite");
  const mcrt_config& c = ctx->cfg;
  const int64_t nc = ctx->ncell;
  for (int64_t k = 0; k < nc; ++k)
    if (!(tdave[k] > 0.0) || !std::isfinite(tdave[k]))
      return fail(ctx, MCRT_ERR_ARG, "tdave(%lld) = %g is not a positive temperature", (long long)k + 1, tdave[k]);
  CK(cudaSetDevice(ctx->device));
  int rc;
  if (!ctx->d_sd_tdave) {
    if ((rc = dalloc(ctx, &ctx->d_sd_tdave, nc))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_sd_mark, (size_t)c.nrg * c.ntg))) return rc;
    if ((rc = dalloc(ctx, &ctx->d_sd_out, nc))) return rc;
  }
  SetdiffusArgs a{};
  a.nrg = c.nrg; a.ntg = c.ntg; a.npg = c.npg; a.nT = c.nT; a.iter = iter;
  // the march starts at the first dust cell, or two cells further out when
  // the grid starts at the star rather than at the dust radius (setdiffus_5.f90:44-48)
  a.nr0 = (c.rddust == ctx->h_rarr[0]) ? 1 : 3;
  int ir = a.nr0;
  while (ir <= c.nrg - 1 && ctx->h_rarr[ir - 1] < rmaxd) ++ir;
  a.nr1 = ir - 1;
  a.rmincgs = c.rstar * 6.9598e10;
  a.rarr = ctx->dm.rarr; a.thetarr = ctx->dm.thetarr; a.hdisk = ctx->dm.hdisk;
  a.kappav = ctx->dm.kappav; a.kappar = ctx->d_tabs + ctx->off_kappar; a.lTint = ctx->dm.lTint;
  a.tdave = ctx->d_sd_tdave; a.cells = ctx->d_cells; a.mark = ctx->d_sd_mark;
  CK(cudaMemcpyAsync(ctx->d_sd_tdave, tdave, nc * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_sd_mark, 0, (size_t)c.nrg * c.ntg, ctx->stream));
  const bool disk = massd > 0.0;
  if (disk && a.nr1 >= a.nr0 && (c.ntg - 1) / 2 >= 2) setdiffus_mark<<<148, 128, 0, ctx->stream>>>(a);
  setdiffus_apply<<<512, 256, 0, ctx->stream>>>(a, disk ? 1 : 0, ctx->d_cells, ctx->d_diffus, ctx->d_tdust,
                                                ctx->d_tdust0, ctx->d_sd_out);
  CK(cudaGetLastError());
  if (!diffus && !diffdir && !dcount) {     // nothing to return: no wait; tfinal copies the flags it needs
    ctx->h_diffus_stale = true;
    return MCRT_OK;
  }
  std::vector<int32_t> out(nc);
  CK(cudaMemcpyAsync(out.data(), ctx->d_sd_out, nc * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  int64_t cnt = 0;
  for (int64_t k = 0; k < nc; ++k) {
    const int on = out[k] & 1;
    ctx->h_diffus[k] = on;
    cnt += on;
    if (diffus) diffus[k] = on;
    if (diffdir) diffdir[k] = out[k] >> 8;
  }
  ctx->h_diffus_stale = false;
  if (dcount) *dcount = cnt;
  return MCRT_OK;
}

int mcrt_update_temperature(mcrt_ctx* ctx, int32_t nphot, int32_t iter, double* tdave, int32_t* converge, double* sig) {
  if (!ctx || !tdave || !converge) return MCRT_ERR_ARG;
  if (!ctx->have_grid || !ctx->have_tables) return fail(ctx, MCRT_ERR_STATE, "upload the grid and tables first");
  if (nphot < 1) return fail(ctx, MCRT_ERR_ARG, "nphot must be positive");
  CK(cudaSetDevice(ctx->device));
  const mcrt_config& c = ctx->cfg;
  const int64_t nc = ctx->ncell;
  const int64_t n2 = (int64_t)c.nrg * c.ntg;
  double* d_td = nullptr;
  int rc;
  if ((rc = scratch(ctx, &d_td, 3 * nc + (ctx->have_vel ? nc + 5 * n2 : 0)))) return rc;
  CK(cudaMemcpyAsync(d_td, tdave, nc * 8, cudaMemcpyHostToDevice, ctx->stream));
  TfinalArgs a{};
  a.nrg = c.nrg; a.ntg = c.ntg; a.npg = c.npg; a.nT = c.nT; a.nphot = nphot; a.maxii = iter > 3 ? 20 : 1;
  a.rstar = c.rstar; a.tstar = c.tstarave;
  a.Tint = ctx->d_tabs + ctx->off_Tint;
  a.kappap = ctx->d_tabs + ctx->off_kappap;
  a.kappav = ctx->dm.kappav;
  a.dtauabs = ctx->dt.dtauabs; a.vcell = ctx->d_vcell; a.dens = ctx->d_dens_thermal; a.tdust = ctx->d_tdust;
  a.idust3 = ctx->d_idust3; a.diffus = ctx->d_diffus;
  a.told = d_td; a.tnew = d_td + nc; a.tdave = d_td + 2 * nc;
  std::vector<double> old(tdave, tdave + nc);
  if (!ctx->have_vel) {
    tfinal_cells<<<256, 128, 0, ctx->stream>>>(a);
    tfinal_mirror<<<512, 256, 0, ctx->stream>>>(a);
  } else {
    // the passes work in place on tdave, starting from the previous field
    a.vr = ctx->d_vel; a.vth = ctx->d_vel + nc; a.divv = ctx->d_vel + 2 * nc;
    a.rarr = ctx->dm.rarr; a.thetarr = ctx->dm.thetarr; a.rave = ctx->d_rave; a.tflag = ctx->d_tflag;
    a.acc = d_td + 3 * nc;
    a.tsm = a.acc + nc; a.gtr = a.tsm + n2; a.gtt = a.gtr + n2; a.gtr2 = a.gtt + n2; a.gtt2 = a.gtr2 + n2;
    CK(cudaMemcpyAsync(a.tdave, d_td, nc * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    for (int ii = 1; ii <= a.maxii; ++ii) {
      tfv_smooth<<<256, 128, 0, ctx->stream>>>(a);
      tfv_grad<<<256, 128, 0, ctx->stream>>>(a, ii == 1 ? 1 : 0);
      tfv_smooth_grad<<<256, 128, 0, ctx->stream>>>(a);
      tfv_cells<<<256, 128, 0, ctx->stream>>>(a);
      tfv_mirror<<<512, 256, 0, ctx->stream>>>(a, (a.maxii > 10 && ii > 10) ? 1 : 0, ii == 11 ? 1 : 0);
    }
    if (a.maxii > 10) tfv_average<<<512, 256, 0, ctx->stream>>>(a, a.maxii - 10);
  }
  tdust_from_tdave<<<512, 256, 0, ctx->stream>>>(nc, a.tdave, ctx->d_diffus, ctx->d_idust3, ctx->d_cells, ctx->d_tdust);
  CK(cudaMemcpyAsync(ctx->d_tdust0, ctx->d_tdust, nc * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(tdave, a.tdave, nc * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (ctx->h_diffus_stale) {           // the flags of the last mcrt_setdiffus, for the statistics below
    CK(cudaMemcpyAsync(ctx->h_diffus.data(), ctx->d_diffus, nc * 4, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->h_diffus_stale = false;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  // convergence statistics (tfinal_5_test1.f90:307-348)
  const double T01 = 0.1 / 11605.0;
  double s[3] = {0, 0, 0}, s2[3] = {0, 0, 0};
  int64_t n[3] = {0, 0, 0};
  for (int ir = 1; ir <= c.nrg - 1; ++ir) {
    for (int it = 1; it <= (c.ntg - 1) / 2; ++it) {
      const int64_t k = (ir - 1) + (int64_t)c.nrg * (it - 1);
      const double told = old[k], tnew = tdave[k];
      const double d = (tnew - told) / tnew;
      if (tnew != told && tnew > T01 && told > T01) { s[0] += std::fabs(d); s2[0] += d * d; n[0]++; }
      if (!ctx->h_diffus[k] && tnew > T01 && told > T01) { s[1] += std::fabs(d); s2[1] += d * d; n[1]++; }
      if (ctx->h_rarr[ir - 1] / c.autors < 5.0 && tnew > T01 && told > T01) { s[2] += std::fabs(d); s2[2] += d * d; n[2]++; }
    }
  }
  double sg[3];
  for (int k = 0; k < 3; ++k) {
    const double av = s[k] / (double)n[k], av2 = s2[k] / (double)n[k];
    sg[k] = std::sqrt(av2 - av * av);
    if (sig) sig[k] = sg[k];
  }
  // convergence when sigma changes by less than 25% between iterations
  if (*converge == 0 && ctx->prev_sig > 0.0 && std::fabs(ctx->prev_sig - sg[0]) / sg[0] < 0.25) *converge = 1;
  ctx->prev_sig = sg[0];
  return MCRT_OK;
}

// Allocation-free temperature update.  The device address of the
// file-scope scratch array is looked up once per device (with that device
// current) on the first call made on it; that first call must therefore not
// be made while a stream is being captured.
int mcrt_update_temperature_noalloc(mcrt_ctx* ctx, int32_t nphot, int32_t iter, double* tdave, int32_t* converge,
                                    double* sig) {
  if (!ctx || !tdave || !converge) return MCRT_ERR_ARG;
  if (!ctx->have_grid || !ctx->have_tables) return fail(ctx, MCRT_ERR_STATE, "upload the grid and tables first");
  if (nphot < 1) return fail(ctx, MCRT_ERR_ARG, "nphot must be positive");
  const mcrt_config& c = ctx->cfg;
  const int64_t nc = ctx->ncell;
  if (nc > kNoAllocMaxCells)
    return fail(ctx, MCRT_ERR_ARG, "mcrt_update_temperature_noalloc: %lld cells exceed its fixed scratch of %lld cells",
                (long long)nc, (long long)kNoAllocMaxCells);
  if (ctx->have_vel)
    return fail(ctx, MCRT_ERR_UNSUPPORTED,
                "mcrt_update_temperature_noalloc: a gas velocity field needs the pass buffers of mcrt_update_temperature");
  CK(cudaSetDevice(ctx->device));
  // the scratch array's device address, looked up once per context with the
  // context's device current (a new context, e.g. after a device reset,
  // looks it up again)
  if (!ctx->noalloc_scratch) CK(cudaGetSymbolAddress((void**)&ctx->noalloc_scratch, g_tfinal_scratch));
  double* base = ctx->noalloc_scratch;
  double* d_told = base;
  double* d_tnew = base + kNoAllocMaxCells;
  double* d_res = base + 2 * kNoAllocMaxCells;
  double* d_stats = base + 3 * kNoAllocMaxCells;
  CK(cudaMemcpyAsync(d_told, tdave, nc * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(d_stats, 0, 9 * sizeof(double), ctx->stream));
  TfinalArgs a{};
  a.nrg = c.nrg; a.ntg = c.ntg; a.npg = c.npg; a.nT = c.nT; a.nphot = nphot; a.maxii = iter > 3 ? 20 : 1;
  a.rstar = c.rstar; a.tstar = c.tstarave;
  a.Tint = ctx->d_tabs + ctx->off_Tint;
  a.kappap = ctx->d_tabs + ctx->off_kappap;
  a.kappav = ctx->dm.kappav;
  a.dtauabs = ctx->dt.dtauabs; a.vcell = ctx->d_vcell; a.dens = ctx->d_dens_thermal; a.tdust = ctx->d_tdust;
  a.idust3 = ctx->d_idust3; a.diffus = ctx->d_diffus;
  a.told = d_told; a.tnew = d_tnew; a.tdave = d_res;
  tfinal_cells<<<256, 128, 0, ctx->stream>>>(a);
  tfinal_mirror<<<512, 256, 0, ctx->stream>>>(a);
  tfinal_stats<<<128, 256, 0, ctx->stream>>>(c.nrg, c.ntg, d_told, d_res, ctx->dm.rarr, c.autors, ctx->d_diffus, d_stats);
  tdust_from_tdave<<<512, 256, 0, ctx->stream>>>(nc, d_res, ctx->d_diffus, ctx->d_idust3, ctx->d_cells, ctx->d_tdust);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ctx->d_tdust0, ctx->d_tdust, nc * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(tdave, d_res, nc * 8, cudaMemcpyDeviceToHost, ctx->stream));
  double st[9];
  CK(cudaMemcpyAsync(st, d_stats, 9 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  double sg[3];
  for (int k = 0; k < 3; ++k) {
    const double av = st[k] / st[6 + k], av2 = st[3 + k] / st[6 + k];
    sg[k] = std::sqrt(av2 - av * av);
    if (sig) sig[k] = sg[k];
  }
  if (*converge == 0 && ctx->prev_sig > 0.0 && std::fabs(ctx->prev_sig - sg[0]) / sg[0] < 0.25) *converge = 1;
  ctx->prev_sig = sg[0];
  return MCRT_OK;
}

}  // extern "C"


// ---------------------------------------------------------------- batch --
// Many models in one launch (mcrt_batch.cuh), one CUDA graph per packet-count
// vector: parameter upload, tally reset, the batch kernel, the diffusion
// finalisation of every model.
struct mcrt_batch {
  std::vector<mcrt_ctx*> ctx;
  int device = 0;
  int precision = MCRT_PREC_FP64;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  LaunchParams* h_params = nullptr;       // pinned: read by the graph's upload node
  LaunchParams* d_params = nullptr;
  BatchItem* d_items = nullptr;
  int64_t nitems = 0, items_cap = 0;
  unsigned long long* d_counters = nullptr;   // [1 + items_cap]: item counter, per-item packet counters
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<int64_t> graph_np;
  std::vector<int64_t> graph_uploads;         // each context's upload count at capture
  int graph_key[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // schedule: MCRT_BATCH_PERSISTENT (one launch over (model, chunk) items) or
  // MCRT_BATCH_WAVE (each model's wavefront loop as a WHILE node, the models
  // as parallel branches of one graph)
  int mode = MCRT_BATCH_PERSISTENT;
  // persistent tuning: blocks per SM (0: occupancy maximum), event batch, items per warp
  int blocks_per_sm = 0, event_batch = 16, items_per_warp = 4;
  // wavefront tuning: in-flight packet slots per model
  int64_t wave_slots = (int64_t)1 << 18;
  struct Wave {
    WaveRec* recs = nullptr;
    int32_t* walkq = nullptr;
    int32_t* evq = nullptr;
    WaveCtl* ctl = nullptr;
    unsigned long long* next = nullptr;     // [4] packet counter (and unused job counters)
    int64_t cap = 0;
  };
  std::vector<Wave> wave;
  std::vector<cudaStream_t> branch;           // capture streams of the parallel branches
  cudaStream_t body_stream = nullptr;
  cudaEvent_t e_fork = nullptr, e_join = nullptr;
  int64_t* h_block0 = nullptr;                // pinned [n]: (iter-1)*np[i], uploaded by the graph
  int64_t* d_block0 = nullptr;
  double last_ms = 0.0;
  std::string err;
};

namespace {

int bfail(mcrt_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  return code;
}

#define BK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return bfail(b, MCRT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

int batch_max_blocks(const mcrt_batch* b) {
  return b->precision == MCRT_PREC_MIXED ? batch_mixed_blocks_per_sm() : batch_fp64_blocks_per_sm();
}

void batch_drop_graph(mcrt_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_np.clear();
  b->graph_uploads.clear();
}

int batch_wave_buffers(mcrt_batch* b, int i, int64_t slots) {
  mcrt_batch::Wave& w = b->wave[i];
  if (w.cap >= slots && w.ctl) return MCRT_OK;
  for (void* q : {(void*)w.recs, (void*)w.walkq, (void*)w.evq, (void*)w.ctl, (void*)w.next})
    if (q) cudaFree(q);
  w = mcrt_batch::Wave{};
  BK(cudaMalloc(&w.recs, (size_t)slots * sizeof(WaveRec)));
  BK(cudaMalloc(&w.walkq, (size_t)slots * sizeof(int32_t)));
  BK(cudaMalloc(&w.evq, (size_t)slots * sizeof(int32_t)));
  BK(cudaMalloc(&w.ctl, sizeof(WaveCtl)));
  BK(cudaMalloc(&w.next, 4 * sizeof(unsigned long long)));
  w.cap = slots;
  return MCRT_OK;
}

// One branch per model, captured on its own stream: tally and loop reset,
// wave_init, the WHILE node (event, mid, walk, cond), the tail launch (no
// work when the loop ended with no live packet), diffusion finalisation and
// the wave counters.  Kernel arguments are fixed at capture; the iteration
// enters through block0_dev.
cudaError_t batch_capture_wave_branch(mcrt_batch* b, int i, int64_t npk, cudaStream_t s) {
  mcrt_ctx* c = b->ctx[i];
  mcrt_batch::Wave& w = b->wave[i];
  const bool mixed = b->precision == MCRT_PREC_MIXED;
  const LaunchParams& P = b->h_params[i];
  WaveArgs W{};
  W.recs = w.recs;
  W.walkq = w.walkq;
  W.evq = w.evq;
  W.ctl = w.ctl;
  W.slots = std::min<int64_t>(b->wave_slots, npk);
  W.walk_batch = c->wave_batch > 0 ? c->wave_batch : 8;
  const int tgrid = b->nsm * (mixed ? wave_tail_mixed_blocks_per_sm() : wave_tail_fp64_blocks_per_sm());
  const unsigned long long tail_live = (unsigned long long)tgrid * kTransportBlock * 8ull;
  cudaError_t e;
  if ((e = cudaMemsetAsync(c->d_tally, 0, c->tally_bytes, s)) != cudaSuccess) return e;
  // the tail launch takes over once every packet has started, so the loop
  // needs a few thousand waves at most; the limit only bounds a fault
  if ((e = capture_wave_loop(P, W, w.next, c->dt.cnt, npk, tail_live, 1000000ull, mixed, b->nsm, s, b->body_stream)) !=
      cudaSuccess)
    return e;
  return launch_diffusion_finalize(P.m, c->dt.ndiff, c->d_tdust0, c->d_tdust, P.nphot_diff, s);
}

int batch_build_wave(mcrt_batch* b, const int64_t* np) {
  const int n = (int)b->ctx.size();
  batch_drop_graph(b);
  if ((int)b->wave.size() < n) b->wave.resize(n);
  for (int i = 0; i < n; ++i) {
    const int rc = batch_wave_buffers(b, i, std::min<int64_t>(b->wave_slots, np[i]));
    if (rc) return rc;
  }
  while ((int)b->branch.size() < n) {
    cudaStream_t s;
    BK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->branch.push_back(s);
  }
  BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemcpyAsync(b->d_block0, b->h_block0, (size_t)n * sizeof(int64_t), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaEventRecord(b->e_fork, b->stream);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    cudaStream_t s = b->branch[i];
    e = cudaStreamWaitEvent(s, b->e_fork, 0);
    if (e == cudaSuccess) e = batch_capture_wave_branch(b, i, np[i], s);
    if (e == cudaSuccess) e = cudaEventRecord(b->e_join, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->e_join, 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
  if (e != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return bfail(b, MCRT_ERR_CUDA, "batch wave graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : ee));
  }
  b->graph = g;
  BK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return MCRT_OK;
}

// items: each model's range cut into chunks, about items_per_warp items per
// warp of the launch over the batch's total packet count
int batch_build_graph(mcrt_batch* b, const int64_t* np) {
  const int n = (int)b->ctx.size();
  const int bps = b->blocks_per_sm > 0 ? std::min(b->blocks_per_sm, batch_max_blocks(b)) : batch_max_blocks(b);
  const int grid = b->nsm * std::max(bps, 1);
  int64_t total = 0;
  for (int i = 0; i < n; ++i) total += np[i];
  const int64_t nwarps = (int64_t)grid * (kTransportBlock / 32);
  const int64_t chunk = std::max<int64_t>(256, (total + nwarps * b->items_per_warp - 1) / (nwarps * b->items_per_warp));
  std::vector<BatchItem> items;
  for (int i = 0; i < n; ++i)
    for (int64_t lo = 1; lo <= np[i]; lo += chunk) {
      BatchItem it{};
      it.model = i;
      it.lo = lo;
      it.hi = std::min(np[i], lo + chunk - 1);
      items.push_back(it);
    }
  batch_drop_graph(b);
  if ((int64_t)items.size() > b->items_cap) {
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_counters) cudaFree(b->d_counters);
    b->d_items = nullptr;
    b->d_counters = nullptr;
    b->items_cap = 0;
    BK(cudaMalloc(&b->d_items, items.size() * sizeof(BatchItem)));
    BK(cudaMalloc(&b->d_counters, (items.size() + 1) * sizeof(unsigned long long)));
    b->items_cap = (int64_t)items.size();
  }
  b->nitems = (int64_t)items.size();
  BK(cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice));
  BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemcpyAsync(b->d_params, b->h_params, (size_t)n * sizeof(LaunchParams), cudaMemcpyHostToDevice,
                                  b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_counters, 0, (size_t)(b->nitems + 1) * sizeof(unsigned long long), b->stream);
  for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaMemsetAsync(b->ctx[i]->d_tally, 0, b->ctx[i]->tally_bytes, b->stream);
  if (e == cudaSuccess)
    e = b->precision == MCRT_PREC_MIXED
            ? launch_batch_mixed(b->d_params, b->d_items, b->nitems, b->d_counters, b->d_counters + 1, b->event_batch,
                                 grid, b->stream)
            : launch_batch_fp64(b->d_params, b->d_items, b->nitems, b->d_counters, b->d_counters + 1, b->event_batch,
                                grid, b->stream);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    mcrt_ctx* c = b->ctx[i];
    e = launch_diffusion_finalize(b->h_params[i].m, c->dt.ndiff, c->d_tdust0, c->d_tdust, b->h_params[i].nphot_diff,
                                  b->stream);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
  if (e != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return bfail(b, MCRT_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : ee));
  }
  b->graph = g;
  BK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return MCRT_OK;
}

}  // namespace

int mcrt_batch_create(mcrt_ctx* const* ctxs, int32_t n, mcrt_batch** out) {
  if (!ctxs || n < 1 || !out) return MCRT_ERR_ARG;
  *out = nullptr;
  auto* b = new mcrt_batch();
  for (int i = 0; i < n; ++i) {
    mcrt_ctx* c = ctxs[i];
    if (!c) { delete b; return MCRT_ERR_ARG; }
    if (!c->have_grid || !c->have_tables) { delete b; return MCRT_ERR_STATE; }
    if (i > 0 && (c->device != ctxs[0]->device || c->precision != ctxs[0]->precision)) { delete b; return MCRT_ERR_ARG; }
    b->ctx.push_back(c);
  }
  b->device = ctxs[0]->device;
  b->precision = ctxs[0]->precision;
  b->nsm = ctxs[0]->nsm;
  *out = b;
  BK(cudaSetDevice(b->device));
  BK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  BK(cudaEventCreate(&b->e0));
  BK(cudaEventCreate(&b->e1));
  BK(cudaHostAlloc((void**)&b->h_params, (size_t)n * sizeof(LaunchParams), cudaHostAllocDefault));
  BK(cudaMalloc(&b->d_params, (size_t)n * sizeof(LaunchParams)));
  BK(cudaHostAlloc((void**)&b->h_block0, (size_t)n * sizeof(int64_t), cudaHostAllocDefault));
  BK(cudaMalloc(&b->d_block0, (size_t)n * sizeof(int64_t)));
  BK(cudaStreamCreateWithFlags(&b->body_stream, cudaStreamNonBlocking));
  BK(cudaEventCreateWithFlags(&b->e_fork, cudaEventDisableTiming));
  BK(cudaEventCreateWithFlags(&b->e_join, cudaEventDisableTiming));
  return MCRT_OK;
}

int mcrt_batch_run_iteration(mcrt_batch* b, const int64_t* np, int32_t iter, int32_t seed1, int32_t seed2,
                             int32_t generator) {
  if (!b || !np) return MCRT_ERR_ARG;
  BK(cudaSetDevice(b->device));
  const int n = (int)b->ctx.size();
  const bool wave = b->mode == MCRT_BATCH_WAVE;
  for (int i = 0; i < n; ++i)
    if (np[i] < 1) return bfail(b, MCRT_ERR_ARG, "model %d: np must be >= 1", i);
  // the graph holds every launch argument but the iteration's block offsets
  const int key[8] = {b->mode, b->blocks_per_sm, b->event_batch, b->items_per_warp, (int)b->wave_slots,
                      seed1, seed2, generator};
  bool fresh = b->exec && (int)b->graph_np.size() == n && std::equal(b->graph_np.begin(), b->graph_np.end(), np) &&
               std::equal(key, key + 8, b->graph_key);
  for (int i = 0; fresh && i < n; ++i) fresh = b->graph_uploads[i] == b->ctx[i]->uploads;
  if (wave && !fresh) {
    if ((int)b->wave.size() < n) b->wave.resize(n);
    for (int i = 0; i < n; ++i) {
      const int rc = batch_wave_buffers(b, i, std::min<int64_t>(b->wave_slots, np[i]));
      if (rc) return rc;
    }
  }
  for (int i = 0; i < n; ++i) {
    mcrt_ctx* c = b->ctx[i];
    if (c->precision != b->precision) return bfail(b, MCRT_ERR_ARG, "model %d changed precision", i);
    BK(cudaStreamSynchronize(c->stream));      // its uploads are complete
    LaunchParams P{};
    const int rc = make_params(c, np[i], 1, np[i], iter, 0, seed1, seed2, generator, P);
    if (rc) return bfail(b, rc, "model %d: %s", i, c->err.c_str());
    P.jobs = nullptr;
    P.event_batch = b->event_batch;
    if (wave) {
      P.next = b->wave[i].next;
      P.block0_dev = b->d_block0 + i;
    }
    b->h_params[i] = P;
    b->h_block0[i] = P.block0;
    c->last_m = P.m;
    c->have_last_run = true;
  }
  if (!fresh) {
    const int rc = wave ? batch_build_wave(b, np) : batch_build_graph(b, np);
    if (rc) return rc;
    b->graph_np.assign(np, np + n);
    for (int i = 0; i < n; ++i) b->graph_uploads.push_back(b->ctx[i]->uploads);
    std::copy(key, key + 8, b->graph_key);
  }
  BK(cudaEventRecord(b->e0, b->stream));
  BK(cudaGraphLaunch(b->exec, b->stream));
  BK(cudaEventRecord(b->e1, b->stream));
  BK(cudaEventSynchronize(b->e1));
  float ms = 0.f;
  BK(cudaEventElapsedTime(&ms, b->e0, b->e1));
  b->last_ms = ms;
  for (int i = 0; i < n; ++i) b->ctx[i]->last_ms = ms;
  if (wave) {   // a loop stopped by the wave limit is an error
    for (int i = 0; i < n; ++i) {
      unsigned long long flag = 0;
      BK(cudaMemcpy(&flag, &b->wave[i].ctl->pad2, sizeof flag, cudaMemcpyDeviceToHost));
      if (flag) return bfail(b, MCRT_ERR_CUDA, "model %d: wavefront loop did not finish", i);
    }
  }
  return MCRT_OK;
}

// Autotuner.  Times one iteration of sample_packets per model for: both
// schedules at their defaults (the persistent one kept only if 10 % faster);
// then, for the chosen one, a coordinate search
// -- persistent: items per warp, event batch, one block per SM fewer;
// wavefront: in-flight slots per model (the packet queue size) within a
// quarter of the free device memory.
int mcrt_batch_tune(mcrt_batch* b, int64_t sample_packets, int32_t* chosen) {
  if (!b || sample_packets < 1) return MCRT_ERR_ARG;
  const int n = (int)b->ctx.size();
  std::vector<int64_t> np(n, sample_packets);
  const int maxb = batch_max_blocks(b);
  struct Cand { int mode, bps, eb, ipw; int64_t slots; };
  auto apply = [&](const Cand& c) {
    b->mode = c.mode; b->blocks_per_sm = c.bps; b->event_batch = c.eb; b->items_per_warp = c.ipw; b->wave_slots = c.slots;
  };
  auto time_it = [&](const Cand& c, double* ms) -> int {
    apply(c);
    const int rc = mcrt_batch_run_iteration(b, np.data(), 1, 12345678, 87654321, 1);
    *ms = b->last_ms;
    return rc;
  };
  size_t freeb = 0, totalb = 0;
  BK(cudaMemGetInfo(&freeb, &totalb));
  const int64_t per_slot = (int64_t)sizeof(WaveRec) + 8;
  auto slots_fit = [&](int64_t slots) {
    int64_t need = 0;
    for (int i = 0; i < n; ++i) need += std::min<int64_t>(slots, np[i]) * per_slot;
    return need <= (int64_t)(freeb / 4);
  };
  Cand best{MCRT_BATCH_WAVE, maxb, 16, 2, (int64_t)1 << 16};
  double tbest = 1e300;
  int rc = time_it(best, &tbest);
  if (rc) return rc;
  {
    // The persistent form runs the warp schedule, about half the wavefront's
    // per-packet rate once waves fill; on a sample it wins only by skipping
    // the waves' fixed cost, which shrinks as the packet counts grow, so it
    // must win by 10 % to be kept.
    Cand p = best;
    p.mode = MCRT_BATCH_PERSISTENT;
    double t = 0.0;
    if ((rc = time_it(p, &t))) return rc;
    if (t < 0.9 * tbest) { tbest = t; best = p; }
  }
  if (best.mode == MCRT_BATCH_PERSISTENT) {
    for (int dim = 0; dim < 3; ++dim) {
      const std::vector<int> vals = dim == 0 ? std::vector<int>{1, 4, 8} : dim == 1 ? std::vector<int>{8, 12, 24}
                                                                                     : std::vector<int>{maxb - 1};
      for (int v : vals) {
        if (v < 1) continue;
        Cand c = best;
        (dim == 0 ? c.ipw : dim == 1 ? c.eb : c.bps) = v;
        double t = 0.0;
        if ((rc = time_it(c, &t))) return rc;
        if (t < tbest) { tbest = t; best = c; }
      }
    }
  } else {
    for (int64_t slots : {(int64_t)1 << 14, (int64_t)1 << 18, (int64_t)1 << 20}) {
      if (!slots_fit(slots)) continue;
      Cand c = best;
      c.slots = slots;
      double t = 0.0;
      if ((rc = time_it(c, &t))) return rc;
      if (t < tbest) { tbest = t; best = c; }
    }
  }
  apply(best);
  batch_drop_graph(b);
  if (chosen) {
    chosen[0] = best.mode; chosen[1] = best.bps; chosen[2] = best.eb; chosen[3] = best.ipw;
    chosen[4] = (int32_t)best.slots;
  }
  return MCRT_OK;
}

int mcrt_batch_set_schedule(mcrt_batch* b, int32_t mode, int64_t wave_slots) {
  if (!b || (mode != MCRT_BATCH_PERSISTENT && mode != MCRT_BATCH_WAVE) || wave_slots < 64 ||
      wave_slots > ((int64_t)1 << 30))
    return MCRT_ERR_ARG;
  b->mode = mode;
  b->wave_slots = wave_slots;
  return MCRT_OK;
}

int mcrt_batch_set_tuning(mcrt_batch* b, int32_t blocks_per_sm, int32_t event_batch, int32_t items_per_warp) {
  if (!b || blocks_per_sm < 0 || event_batch < 1 || event_batch > 32 || items_per_warp < 1) return MCRT_ERR_ARG;
  b->blocks_per_sm = blocks_per_sm;
  b->event_batch = event_batch;
  b->items_per_warp = items_per_warp;
  return MCRT_OK;
}

int mcrt_batch_last_ms(mcrt_batch* b, double* ms) {
  if (!b || !ms) return MCRT_ERR_ARG;
  *ms = b->last_ms;
  return MCRT_OK;
}

const char* mcrt_batch_last_error(mcrt_batch* b) { return b ? b->err.c_str() : "null batch"; }

void mcrt_batch_destroy(mcrt_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  for (auto& w : b->wave)
    for (void* q : {(void*)w.recs, (void*)w.walkq, (void*)w.evq, (void*)w.ctl, (void*)w.next})
      if (q) cudaFree(q);
  for (cudaStream_t s : b->branch) cudaStreamDestroy(s);
  if (b->body_stream) cudaStreamDestroy(b->body_stream);
  if (b->e_fork) cudaEventDestroy(b->e_fork);
  if (b->e_join) cudaEventDestroy(b->e_join);
  if (b->d_block0) cudaFree(b->d_block0);
  if (b->h_block0) cudaFreeHost(b->h_block0);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_counters) cudaFree(b->d_counters);
  if (b->d_params) cudaFree(b->d_params);
  if (b->h_params) cudaFreeHost(b->h_params);
  if (b->e0) cudaEventDestroy(b->e0);
  if (b->e1) cudaEventDestroy(b->e1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// ------------------------------------------------------------- setemiss --
// The emission tables of dustinit (dust_5.f90:486-494 grids, setemiss
// dust_5.f90:507-699) on the GPU; mcrt_setemiss.cuh holds the kernels.
namespace {
int sfail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_free_err = buf;
  return code;
}
}  // namespace

int mcrt_setemiss(int32_t device, int32_t nopac, int32_t ndg, int32_t nlammax, const int32_t* nlambda,
                  const double* nudust, const double* kappad, const double* adust, int32_t nT, int32_t nnu,
                  double* lTint, double* Tint, double* nuint, double* kapint, double* kappap, double* kappar,
                  int64_t* qsimp_misses, double* device_ms) {
  g_free_err.clear();
  if (!nlambda || !nudust || !kappad || !adust || !lTint || !Tint || !nuint || !kapint || !kappap || !kappar)
    return sfail(MCRT_ERR_ARG, "mcrt_setemiss: null array");
  if (nopac < 1 || nopac > 65535 || nlammax < 2 || ndg < 0 || ndg > nopac)
    return sfail(MCRT_ERR_ARG, "mcrt_setemiss: nopac %d, nlammax %d, ndg %d out of range", nopac, nlammax, ndg);
  if (nT < 21 || nnu < 2 || nnu > 3072)
    return sfail(MCRT_ERR_ARG, "mcrt_setemiss: nT must be >= 21 (smoothing window) and nnu in 2..3072");
  for (int id = 0; id < nopac; ++id) {
    const int n = nlambda[id];
    if (n < 2 || n > nlammax) return sfail(MCRT_ERR_ARG, "mcrt_setemiss: nlambda(%d)=%d out of range", id + 1, n);
    const double* nud = nudust + (int64_t)nlammax * id;
    for (int k = 1; k < n; ++k)
      if (!(nud[k] < nud[k - 1]))
        return sfail(MCRT_ERR_ARG, "mcrt_setemiss: nudust(:,%d) must decrease strictly", id + 1);
  }
  // temperature grid 0.1 K .. 2e5 K (log-spaced, in eV) and frequency grid
  // numax/1024 .. numax = 32 in units of kT (dust_5.f90:353-362, 486-494)
  const double Tmin = 0.1, Tmax = 200000.0, numax = 32.0, numin = numax / 1024.0;
  for (int i = 1; i <= nT; ++i) {
    lTint[i - 1] = std::log(Tmin / 11605.0) + (double)(i - 1) * std::log(Tmax / Tmin) / (double)(nT - 1);
    Tint[i - 1] = std::exp(lTint[i - 1]);
  }
  for (int i = 1; i <= nnu; ++i) nuint[i - 1] = numin + (double)(i - 1) * (numax - numin) / (double)(nnu - 1);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return sfail(MCRT_ERR_CUDA, "mcrt_setemiss: cudaSetDevice: %s", cudaGetErrorString(e));
  const size_t nl = (size_t)nlammax * nopac, nk = (size_t)nT * nnu * nopac, np_ = (size_t)nT * nopac;
  const size_t ngas = (size_t)(nopac - ndg);
  // one allocation, every piece 256-byte aligned: sizes first, then offsets
  const size_t sizes[11] = {nl * 8, nl * 8, nl * 8, (size_t)nopac * 4, (size_t)nT * 8, (size_t)nnu * 8,
                            nk * 8, np_ * 8, np_ * 8, 8, ngas * nT * 8 + 8};
  size_t bytes = 0;
  for (size_t z : sizes) bytes += (z + 255) / 256 * 256;
  char* buf = nullptr;
  e = cudaMalloc(&buf, bytes);
  if (e != cudaSuccess) return sfail(MCRT_ERR_CUDA, "mcrt_setemiss: cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  size_t off = 0;
  int piece = 0;
  bool layout_ok = true;
  auto take = [&](size_t n) {        // the pieces in the order of `sizes`
    layout_ok = layout_ok && piece < 11 && n == sizes[piece];
    char* p = buf + off;
    off += (sizes[piece < 11 ? piece : 10] + 255) / 256 * 256;
    ++piece;
    return p;
  };
  double* d_nud = (double*)take(nl * 8);
  double* d_kd = (double*)take(nl * 8);
  double* d_ad = (double*)take(nl * 8);
  int32_t* d_nl = (int32_t*)take((size_t)nopac * 4);
  double* d_T = (double*)take((size_t)nT * 8);
  double* d_nu = (double*)take((size_t)nnu * 8);
  double* d_ki = (double*)take(nk * 8);
  double* d_kp = (double*)take(np_ * 8);
  double* d_kr = (double*)take(np_ * 8);
  unsigned long long* d_miss = (unsigned long long*)take(8);
  double* d_tmp = (double*)take(ngas * nT * 8 + 8);
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = MCRT_OK;
  auto chk = [&](cudaError_t x, const char* what) {
    if (x != cudaSuccess && rc == MCRT_OK) rc = sfail(MCRT_ERR_CUDA, "mcrt_setemiss: %s: %s", what, cudaGetErrorString(x));
    return rc == MCRT_OK;
  };
  if (!layout_ok || off > bytes) rc = sfail(MCRT_ERR_CUDA, "mcrt_setemiss: internal buffer layout");
  if (rc == MCRT_OK && chk(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream") &&
      chk(cudaEventCreate(&e0), "event") && chk(cudaEventCreate(&e1), "event") &&
      chk(cudaMemcpyAsync(d_nud, nudust, nl * 8, cudaMemcpyHostToDevice, s), "upload") &&
      chk(cudaMemcpyAsync(d_kd, kappad, nl * 8, cudaMemcpyHostToDevice, s), "upload") &&
      chk(cudaMemcpyAsync(d_ad, adust, nl * 8, cudaMemcpyHostToDevice, s), "upload") &&
      chk(cudaMemcpyAsync(d_nl, nlambda, (size_t)nopac * 4, cudaMemcpyHostToDevice, s), "upload") &&
      chk(cudaMemcpyAsync(d_T, Tint, (size_t)nT * 8, cudaMemcpyHostToDevice, s), "upload") &&
      chk(cudaMemcpyAsync(d_nu, nuint, (size_t)nnu * 8, cudaMemcpyHostToDevice, s), "upload") &&
      chk(cudaMemsetAsync(d_miss, 0, 8, s), "memset") && chk(cudaEventRecord(e0, s), "event")) {
    SetemissArgs a{};
    a.nopac = nopac; a.ndg = ndg; a.nlammax = nlammax; a.nT = nT; a.nnu = nnu;
    a.nlambda = d_nl; a.nudust = d_nud; a.kappad = d_kd; a.adust = d_ad; a.Tint = d_T; a.nuint = d_nu;
    a.kapint = d_ki; a.kappap = d_kp; a.kappar = d_kr; a.misses = d_miss;
    unsigned long long miss = 0;
    float ms = 0.f;
    if (chk(launch_setemiss(a, d_tmp, s), "launch") && chk(cudaEventRecord(e1, s), "event") &&
        chk(cudaMemcpyAsync(kapint, d_ki, nk * 8, cudaMemcpyDeviceToHost, s), "download") &&
        chk(cudaMemcpyAsync(kappap, d_kp, np_ * 8, cudaMemcpyDeviceToHost, s), "download") &&
        chk(cudaMemcpyAsync(kappar, d_kr, np_ * 8, cudaMemcpyDeviceToHost, s), "download") &&
        chk(cudaMemcpyAsync(&miss, d_miss, 8, cudaMemcpyDeviceToHost, s), "download") &&
        chk(cudaStreamSynchronize(s), "synchronize") && chk(cudaEventElapsedTime(&ms, e0, e1), "timing")) {
      if (qsimp_misses) *qsimp_misses = (int64_t)miss;
      if (device_ms) *device_ms = ms;
    }
  }
  if (s) cudaStreamSynchronize(s);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  cudaFree(buf);
  return rc;
}


// -------------------------------------------------------- density model --
// One thread per (r, theta) cell: the disk law, the Ulrich envelope, the
// polynomial cavity, the disk's ownership of a cell and the cell volume for
// every phi plane, plus the disk law's analytic log-derivatives.
namespace {

constexpr double kPi = 3.1415926535897932384626433;
constexpr double kRsun = 6.9598e10, kMsun = 1.989e33, kGN = 6.67428e-8;

struct DensityArgs {
  mcrt_density_params p;
  int32_t nrg, ntg, npg, has_clump;
  const double *rarr, *thetarr, *clump;
  double *dens, *vcell, *dlog;
  double rho0, z1, rhoe0, c1e, dlog_b_const;   // cell-independent parts, from the host
};

// the positive root of mu0^3 + (rx-1) mu0 - rx mu = 0 (zerod.f90), in [1e-12, 1]
__device__ double ulrich_mu0(double mu, double rx) {
  const double a2 = rx - 1.0, a3 = -rx * mu;
  const double q = (-3.0 * a2) / 9.0, r = (27.0 * a3) / 54.0;
  const double q3 = q * q * q;
  double out;
  if (q3 - r * r >= 0.0) {
    const double qh = sqrt(q);
    const double th = acos(fmin(fmax(r / sqrt(q3), -1.0), 1.0));
    out = HUGE_VAL;
    const double roots[3] = {-2.0 * qh * cos(th / 3.0), -2.0 * qh * cos((th + 2.0 * kPi) / 3.0),
                             -2.0 * qh * cos((th + 4.0 * kPi) / 3.0)};
    for (double x : roots)
      if (x > 0.0 && x < out) out = x;
  } else {
    const double fac = sqrt(r * r - q3) + fabs(r);
    const double f3 = pow(fac, 1.0 / 3.0);
    const double sg = r > 0.0 ? 1.0 : (r < 0.0 ? -1.0 : 0.0);
    out = -sg * (f3 + q / f3);
  }
  return fmin(fmax(out, 1e-12), 1.0);
}

__global__ void model_density(DensityArgs a) {
  const int nr = a.nrg - 1, nt = a.ntg - 1, npc = a.npg - 1;
  const int64_t n = (int64_t)nr * nt;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const int ir = (int)(c % nr), it = (int)(c / nr);
    const mcrt_density_params& p = a.p;
    const double rave = 0.5 * (a.rarr[ir] + a.rarr[ir + 1]);
    const double thave = 0.5 * (a.thetarr[it] + a.thetarr[it + 1]);
    const double wcyl = rave * sin(thave), zp = rave * fabs(cos(thave));
    // disk (setup_wave.f90:60-88): rho0 (1 - sqrt(R*/w)) w^-a exp(-z^2/2h^2), h = z1 w^b
    const double h = a.z1 * pow(wcyl, p.b_exp);
    double rho_d = a.rho0 * (1.0 - sqrt(1.0 / wcyl)) * pow(wcyl, -p.a_exp) * exp(-0.5 * ((zp / h) * (zp / h)));
    if (!(rave > p.rddust && wcyl <= p.rmaxd && wcyl > 1.0) || !(rho_d > 1e-300)) rho_d = 0.0;
    // Ulrich envelope (densenv.f90:37-43), floor rhoamb outside the dust radius
    const double mu = zp / rave, rx = rave / p.rc;
    const double mu0 = ulrich_mu0(mu, rx);
    const double factor = 1.0 / ((mu / mu0) + 2.0 * mu0 * mu0 / rx);
    double rho_e = a.rhoe0 * pow(rx, -1.5) * factor / sqrt(1.0 + mu / mu0);
    rho_e = rave > p.rddust ? fmax(rho_e, p.rhoamb) : 0.0;
    // polynomial cavity (densenv.f90:76-90)
    const double zup = a.c1e * pow(wcyl, p.ex1);
    const bool inhole = zp > zup;
    const double rho_c = (inhole && rave > p.rddust && rave < p.rmax) ? p.rhoconst1 : 0.0;
    if (inhole || rave >= p.rmax) rho_e = 0.0;
    const double dr3 = a.rarr[ir + 1] * a.rarr[ir + 1] * a.rarr[ir + 1] - a.rarr[ir] * a.rarr[ir] * a.rarr[ir];
    const double dcost = cos(a.thetarr[it + 1]) - cos(a.thetarr[it]);
    const double rmincgs = p.rstar * kRsun;
    const double vol = -(dr3 * dcost) * (2.0 * kPi / npc) / 3.0 * (rmincgs * rmincgs * rmincgs);
    for (int ip = 0; ip < npc; ++ip) {
      const int64_t cell = ir + (int64_t)a.nrg * (it + (int64_t)a.ntg * ip);
      const int64_t ncell = (int64_t)a.nrg * a.ntg * a.npg;
      const double re = a.has_clump ? rho_e * a.clump[ir + (int64_t)nr * (it + (int64_t)nt * ip)] : rho_e;
      // the disk owns the cell where it is denser (gridset_5_model13new.f90:1217-1224)
      const bool disk = rho_d > re + rho_c;
      a.dens[cell + ncell * 1] = disk ? rho_d : 0.0;
      a.dens[cell + ncell * 2] = disk ? 0.0 : re;
      a.dens[cell + ncell * 3] = disk ? 0.0 : rho_c;
      a.vcell[cell] = vol;
    }
    if (a.dlog) {
      double d0 = 0.0, d1 = 0.0, d2 = 0.0;
      if (rho_d > 0.0) {
        const double zh2 = (zp / h) * (zp / h);
        d0 = 1.0;                                             // log Mdisk
        d1 = a.dlog_b_const + zh2 * (log(wcyl) - log(100.0 * p.autors));   // b
        d2 = zh2 - 1.0;                                       // log h100
      }
      a.dlog[c] = d0;
      a.dlog[c + n] = d1;
      a.dlog[c + 2 * n] = d2;
    }
  }
}

}  // namespace

int mcrt_model_density(int32_t device, const mcrt_density_params* p, int32_t nrg, int32_t ntg, int32_t npg,
                       const double* rarr, const double* thetarr, const double* clump, double* densarr,
                       double* vcell, double* dlog_disk) {
  g_free_err.clear();
  if (!p || !rarr || !thetarr || !densarr || !vcell) return sfail(MCRT_ERR_ARG, "mcrt_model_density: null array");
  if (nrg < 3 || ntg < 2 || npg < 2) return sfail(MCRT_ERR_ARG, "mcrt_model_density: grid too small");
  if (!(p->rstar > 0) || !(p->autors > 0) || !(p->rddust > 1.0) || !(p->rmaxd > p->rddust) || !(p->rmax > p->rddust) ||
      !(p->massd >= 0) || !(p->h100_au > 0) || !(p->rc > 0) || !(p->massc > 0) || !(p->rate >= 0) ||
      !(p->thet1_deg > 0 && p->thet1_deg < 90))
    return sfail(MCRT_ERR_ARG, "mcrt_model_density: parameters out of range");
  for (int i = 1; i < nrg; ++i)
    if (!(rarr[i] > rarr[i - 1])) return sfail(MCRT_ERR_ARG, "mcrt_model_density: rarr must increase");
  for (int i = 1; i < ntg; ++i)
    if (!(thetarr[i] > thetarr[i - 1])) return sfail(MCRT_ERR_ARG, "mcrt_model_density: thetarr must increase");
  DensityArgs a{};
  a.p = *p;
  a.nrg = nrg; a.ntg = ntg; a.npg = npg; a.has_clump = clump ? 1 : 0;
  // cell-independent parts: disk normalisation to Mdisk over [rddust, rmaxd]
  // (setup_wave.f90:60-88), the envelope constant (envset.f90:157-160) and
  // the cavity shape (envset.f90:182-189)
  const double b = p->b_exp, pp = p->b_exp - p->a_exp;
  const double rmincgs = p->rstar * kRsun;
  a.z1 = p->h100_au * p->autors / std::pow(100.0 * p->autors, b);
  const double cst = std::pow(2.0 * kPi, 1.5) * rmincgs * rmincgs * (rmincgs * a.z1);
  const double R = p->rmaxd, r = p->rddust;
  const double A = std::pow(R, pp + 2.0) - std::pow(r, pp + 2.0), B = std::pow(R, pp + 1.5) - std::pow(r, pp + 1.5);
  const double I = 1.0 / (pp + 2.0) * A - 1.0 / (pp + 1.5) * B;
  a.rho0 = p->massd * kMsun / cst / I;
  const double dA = std::pow(R, pp + 2.0) * std::log(R) - std::pow(r, pp + 2.0) * std::log(r);
  const double dB = std::pow(R, pp + 1.5) * std::log(R) - std::pow(r, pp + 1.5) * std::log(r);
  const double dI = dA / (pp + 2.0) - A / ((pp + 2.0) * (pp + 2.0)) - dB / (pp + 1.5) + B / ((pp + 1.5) * (pp + 1.5));
  a.dlog_b_const = std::log(100.0 * p->autors) - dI / I;
  const double rdcgs = p->rc * rmincgs;
  const double cenv = 1.0 / 3.15576e7 * std::sqrt(kMsun) / (4.0 * kPi) / std::sqrt(kGN);
  a.rhoe0 = cenv * p->rate / std::sqrt(p->massc) / std::pow(rdcgs, 1.5);
  const double r1max = p->rmax * std::tan(p->thet1_deg * kPi / 180.0);
  a.c1e = p->rmax / std::pow(r1max, p->ex1);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return sfail(MCRT_ERR_CUDA, "mcrt_model_density: cudaSetDevice: %s", cudaGetErrorString(e));
  const int64_t nr = nrg - 1, nt = ntg - 1, npc = npg - 1;
  const size_t ncell = (size_t)nrg * ntg * npg;
  const size_t sz[6] = {(size_t)nrg * 8, (size_t)ntg * 8, clump ? (size_t)(nr * nt * npc) * 8 : 8, ncell * 10 * 8,
                        ncell * 8, dlog_disk ? (size_t)(nr * nt * 3) * 8 : 8};
  size_t bytes = 0;
  for (size_t z : sz) bytes += (z + 255) / 256 * 256;
  char* buf = nullptr;
  e = cudaMalloc(&buf, bytes);
  if (e != cudaSuccess) return sfail(MCRT_ERR_CUDA, "mcrt_model_density: cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  char* ptr[6];
  size_t off = 0;
  for (int k = 0; k < 6; ++k) { ptr[k] = buf + off; off += (sz[k] + 255) / 256 * 256; }
  a.rarr = (double*)ptr[0]; a.thetarr = (double*)ptr[1]; a.clump = clump ? (double*)ptr[2] : nullptr;
  a.dens = (double*)ptr[3]; a.vcell = (double*)ptr[4]; a.dlog = dlog_disk ? (double*)ptr[5] : nullptr;
  int rc = MCRT_OK;
  auto chk = [&](cudaError_t x, const char* what) {
    if (x != cudaSuccess && rc == MCRT_OK) rc = sfail(MCRT_ERR_CUDA, "mcrt_model_density: %s: %s", what, cudaGetErrorString(x));
    return rc == MCRT_OK;
  };
  if (chk(cudaMemcpy(ptr[0], rarr, sz[0], cudaMemcpyHostToDevice), "upload") &&
      chk(cudaMemcpy(ptr[1], thetarr, sz[1], cudaMemcpyHostToDevice), "upload") &&
      (!clump || chk(cudaMemcpy(ptr[2], clump, sz[2], cudaMemcpyHostToDevice), "upload")) &&
      chk(cudaMemset(ptr[3], 0, sz[3]), "memset") && chk(cudaMemset(ptr[4], 0, sz[4]), "memset")) {
    const int grid = (int)std::min<int64_t>((nr * nt + 255) / 256, 4096);
    model_density<<<grid, 256>>>(a);
    if (chk(cudaGetLastError(), "launch") && chk(cudaDeviceSynchronize(), "kernel") &&
        chk(cudaMemcpy(densarr, ptr[3], sz[3], cudaMemcpyDeviceToHost), "download") &&
        chk(cudaMemcpy(vcell, ptr[4], sz[4], cudaMemcpyDeviceToHost), "download"))
      if (dlog_disk) chk(cudaMemcpy(dlog_disk, ptr[5], sz[5], cudaMemcpyDeviceToHost), "download");
  }
  cudaFree(buf);
  return rc;
}
