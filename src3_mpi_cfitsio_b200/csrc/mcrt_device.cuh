// mcrt_device.cuh -- device-side data layout of the B200 photon-packet engine.
//
// The model lives in HBM in a transport-friendly layout built once per
// upload by the host (mcrt_b200.cu):
//   * walls (rarr/r2arr/costarr/tan2arr/phiarr/aarr/barr) as plain FP64
//     vectors (a few KB, L1/L2 resident);
//   * one CellRec per cell (Fortran linear order over nrg x ntg x npg) with
//     the non-zero density components of densarr(ir,it,ip,1:10) in id order
//     and their opacity-species slot (findopac mapped to a compact slot of
//     the species the model actually references), so a crossing reads one
//     32-byte record instead of 10 strided densarr/findopac pairs;
//   * per-species dust tables (nudust, kappad, adust, gdust, pldust) and the
//     normalised emissivity CDFs kapint(nT,nnu,species).
// Tallies are FP64 on the device (the reference's REAL tallies are produced
// by the download) and are updated with atomics.
#pragma once
#include <cstdint>
#include <cstddef>

#include "../../include/mcrt_b200.h"

namespace mcrt {

constexpr int kMaxComp = 3;   // non-zero density components per cell
constexpr int kMaxSlot = 8;   // distinct opacity species referenced by the grid
constexpr int kTransportBlock = 128;  // threads per transport block
constexpr int kJumpBits = 14;         // block-index digit of the jump tables
constexpr int kJumpDigit = 1 << kJumpBits;

struct __align__(16) CellRec {
  double rho[kMaxComp];       // densarr of the non-zero components, id order
  uint32_t meta;              // bits 0-1: n; per comp k: slot (3 bits) at 2+7k, id-1 (4 bits) at 5+7k
  uint32_t flags;             // bit 0: diffus; bits 1-4: diffdir+8; bit 5: has a thermal component
};
static_assert(sizeof(CellRec) == 32, "CellRec must stay 32 bytes");

// The same cell for the FP32 walk of the mixed build: densities rounded to
// FP32, the component word of CellRec.  16 bytes, one vector load.
struct __align__(16) CellRecF {
  float rho[kMaxComp];
  uint32_t meta;
};
static_assert(sizeof(CellRecF) == 16, "CellRecF must stay 16 bytes");

__host__ __device__ inline int cell_n(uint32_t meta) { return (int)(meta & 3u); }
__host__ __device__ inline int cell_slot(uint32_t meta, int k) { return (int)((meta >> (2 + 7 * k)) & 7u); }
__host__ __device__ inline int cell_id(uint32_t meta, int k) { return (int)((meta >> (5 + 7 * k)) & 15u) + 1; }
__host__ __device__ inline bool cell_diffus(uint32_t flags) { return (flags & 1u) != 0; }
__host__ __device__ inline int cell_diffdir(uint32_t flags) { return (int)((flags >> 1) & 15u) - 8; }
__host__ __device__ inline bool cell_thermal(uint32_t flags) { return (flags & 32u) != 0; }

struct DevTallies {
  int32_t *nabs, *dbig, *dsg, *killed;     // [ncell]
  double *dtauabs, *fuvmean;               // [ncell]
  double *sed;                             // [10][nsed]
  double *psed;                            // [9][npsed]
  double *img;                             // [4][nimg]
  double *imgb;                            // [8][nimgb] filter-band images: I Q U V, I by origin d s e o
  double *ims;                             // [4][nims] nested images I Q U V, [dim,dim,nnu,nlev,npeel]
  double *scal;                            // [MCRT_NSCALARS]
  unsigned long long *cnt;                 // [MCRT_NCOUNTERS]
  int32_t *ndiff;                          // [ncell] diffusion absorptions per surface cell
};

struct DevModel {
  // sizes
  int nrg, ntg, npg, nopac, nlammax, nT, nnu, nhnu;
  int nfreq, nmu, nph, nap, npeel, nxhst;
  int nslot;
  int output_imcube, partial_peeloff, limb, iplanckst, idust, iffuv, ispot, nspot;
  int64_t ncell, nsed, npsed, nimg;
  // scalars
  double rstar, rmincgs, tstar, tshock, fspot, rmaxi, fractxh, numin, lnurat, ifuv_ori;
  double cspot1, sspot1, scspot1, ssspot1, cspot2, sspot2, scspot2, ssspot2, csprad;
  // walls
  const double *rarr, *r2arr, *thetarr, *costarr, *tan2arr, *phiarr, *aarr, *barr, *sintarr;
  // disk-accretion emission (initpacc): cell-centre radii, luminosity CDF, scale heights [nrg-1]
  const double *ravearr, *Ldint, *hdisk;
  // FP32 walk (mixed build): per theta wall (mu, mu^2) with mu = cos(theta)
  // in FP32 (mu^2 = -1: the theta = 90 deg plane, 2: a pole no ray crosses);
  // per phi wall (A, B) of the plane A x + B y = 0
  const float2 *tcone, *pplane;
  const CellRecF *cellsf;
  // cells
  const CellRec *cells;
  const double *tdust, *vcell;              // tdust: start-of-iteration values
  // species: slot -> species (1-based) and the species tables
  int slot_species[kMaxSlot];
  int slot_grid[kMaxSlot];          // first slot whose species has the same wavelength grid (opacset shares its bracket)
  const int32_t *nlambda;
  const double *nudust, *kappad, *adust, *gdust, *pldust, *kappav;
  const double *kapint, *lTint, *nuint;
  // tabulated scattering (stokes6): [nopac][nlammax][narr][6] and the
  // per-row rejection bound; mueller == nullptr selects dustmat
  const double *mueller, *mpeak;
  int narr;
  double dct;
  // external illumination: the ISRF sampling table (isrf_mod after isrf_cdf.f90)
  const double *isrf_cdf, *isrf_logcdf, *isrf_logfreq;
  int nisrf;
  // small-grain emission: the Draine spectra (draine_mod after
  // draine_cdf.f90), [nemit][ndraine] Fortran order, and the per-cell row
  // (imean; nullptr: row 2 in the first iteration, row 1 afterwards)
  const double *draine_cdf, *draine_logcdf, *draine_logfreq;
  int nemit, ndraine;
  const int32_t *imean;
  // star
  const double *atmosnu, *hnuint, *lognu, *loghnu, *limb_prob;
  const double *inczeta;                     // [MCRT_IZMAX]
  // observer
  const double *aperture2, *u, *sini, *coste, *sinte, *cospe, *sinpe;
  // random-number jump tables: a^(2^30 * 2^k) mod m, k = 0..63; and per
  // generator three digit tables A^(j * 2^(14 c)), A = a^(2^30), c = 0..2,
  // j < 2^14 ([3][kJumpDigit]), so a block index below 2^42 jumps in three
  // multiplications
  const int64_t *jump1, *jump2;
  const int64_t *jdig1, *jdig2;
  // filter-band images (output_imfilt): per filter the number of points
  // used (nwfilt - 1) and the curves filtwave (Hz, non-decreasing), filtphi
  // [nfilt][nwfiltmax]
  int output_imfilt, nfilt, nwfiltmax;
  int64_t nimgb;
  const int32_t *nfpts;
  const double *filtwave, *filtphi;
  // nested images (output_imsparse): sparse_nlev square images of
  // sparse_dim^2 pixels with half sizes sparse_levels (ascending), sparse_nnu
  // bins in log10(frequency) over [lognu_min, lognu_max]
  int output_imsparse, sparse_dim, sparse_nlev, sparse_nnu;
  float sparse_lognu_min, sparse_lognu_max;
  int64_t nims;
  const float *sparse_levels;
};

// One peel-off request: the packet's state at an emission, scattering or
// absorption, walked to every inclination by the peel-off kernel
// (peeloff_3d_2_test.f90:7-347 called from newdisktherm_5_fuv.f90:378-413
// and propagate_5_fuv.f90:84-89, 163-169).
constexpr int kJobSlots = 4;   // species slots carried in a job
struct __align__(16) PeelJob {
  double x, y, z, rs, rt;         // position
  double si, sq, su, sv;          // Stokes (si is the un-weighted I of a direct peel-off)
  double d0, d1, d2, d3, d4;      // packet direction cost,sint,cosp,sinp,phi; direct: cosb,sinb,coslp,sinlp
  double kapd[kJobSlots];         // opacity per species slot at the packet's frequency
  double g, pl;                   // phase-function parameters of the scattering species; with a
                                  // tabulated matrix: g = wavelength weight f, pl = table row
  int32_t r, t, p;                // cell
  uint32_t bits;                  // onw | iflag<<1 | direct<<2 | (i_orig)<<3 | (inub-1)<<8
  int32_t pkt, ev;                // packet index in its launch range, event index (0 = emission, k = interaction k)
};

// Wavefront schedule: one in-flight packet per pool slot, kept in HBM
// between the walk kernel and the event kernel.  Fields come in 16-byte
// groups (two doubles, or four 32-bit integers) that one kernel reads or
// writes together, so every record access is a 16-byte vector load or
// store.  The walk part (first 208 bytes) is what the walk kernels read and
// write.  `spec` holds per species slot the columns kapd, albedo, g, pl of
// the packet's current frequency.
struct __align__(16) WaveRec {
  // walk part
  double x, y, z, rs, rt, vx, vy, vz;                 // ray start point and direction
  double tsum, tau;
  double ifuv;
  int64_t ray_steps;
  int32_t r, t, p, rbits;                             // ray cell; rbits: onw | peel << 1
  int32_t ev, status, ncross, exitflag;
  int32_t s1, s2, ndraws, pad0;                       // random stream
  int32_t ir, it, ip, on_wall;                        // packet cell
  double xp, yp, zp, rsq, rtot, pad1;                 // packet position
  // event part
  double ux, uy, uz, cost, sint, cosp, sinp, phi;
  double sip, sqp, sup, svp, nub, xpold, ypold, zpold;
  int64_t nev, iphot, kfetch, pad2;
  int32_t iflag, i_orig, nscat, nabsev;
  int32_t nstar, ndiffev, iscat, iint;
  int32_t first, slot_s, prev_r, prev_t;
  int32_t prev_p, peel_ctx, peelid, peel_idust2;
  double cosb, sinb, lp, peel_si, coslp, sinlp;       // peel-off state
  double spec[4 * kMaxSlot];                          // [slot][kapd, albedo, g, pl]
};
static_assert(sizeof(WaveRec) % 16 == 0, "WaveRec must keep 16-byte alignment");
static_assert(offsetof(WaveRec, tsum) % 16 == 0 && offsetof(WaveRec, ifuv) % 16 == 0 && offsetof(WaveRec, r) % 16 == 0 &&
                  offsetof(WaveRec, s1) % 16 == 0 && offsetof(WaveRec, xp) % 16 == 0 && offsetof(WaveRec, ux) % 16 == 0 &&
                  offsetof(WaveRec, sip) % 16 == 0 && offsetof(WaveRec, nev) % 16 == 0 &&
                  offsetof(WaveRec, iflag) % 16 == 0 && offsetof(WaveRec, cosb) % 16 == 0 &&
                  offsetof(WaveRec, spec) % 16 == 0,
              "WaveRec groups must start on 16-byte boundaries");

// Queue counters of the wavefront loop.  The event queue is filled from both
// ends by the walk kernel: interactions from the front, every other event
// from the back, so the event kernel's warps see one kind of event at a time.
struct WaveCtl {
  unsigned long long n_front, n_back, walk_fetch;         // zeroed before each walk launch
  unsigned long long walk_cross;                          // crossings stepped by walk launches (whole loop)
  unsigned long long n_walk, ev_fetch, pad1, pad2;        // zeroed before each event launch
  // device-driven loop (CUDA-graph WHILE node): %globaltimer stamp of the
  // last loop kernel, device time of the event launches, walk launches and
  // the tail [ns], walks queued over the loop
  unsigned long long t_last, ev_ns, walk_ns, tail_ns, walks, pad3, pad4, pad5;
};

struct WaveArgs {
  WaveRec* recs;        // [slots]
  int32_t* walkq;       // [slots] slots to walk (event kernel -> walk kernel)
  int32_t* evq;         // [slots] slots with a pending event (walk kernel -> event kernel)
  WaveCtl* ctl;
  int64_t slots;
  int32_t walk_batch;   // idle lanes of a warp before the walk kernel fetches new walks
  int32_t pad_;
};

// Path-replay adjoint (mcrt_adjoint).  mode 0: off.  mode 1, forward pass:
// the peel-off kernel records every job's weighted contribution C (one
// record per job: key = packet << 24 | event) and re-walks each contributing
// ray to scatter -C * tau per (cell, component).  mode 2, replay pass: the
// warp-scheduled loop replays the packets that have records on the same
// streams and scores their segments with A, the sum of their later
// peel-offs' C.
struct AdjointArgs {
  int32_t mode;
  int32_t pad_;
  const double* lam_psed;          // [npsed] weights of ti
  const double* lam_img;           // [nimg] weights of image_m_i, or nullptr
  double* grad;                    // [10][ncell] dL/dlog(rho) per component id
  double* obj;                     // objective
  unsigned long long* rec_key;     // [rec_cap] forward: written per job (~0: none)
  double* rec_c;                   // [rec_cap]
  int64_t rec_base;                // record of job 0 of this peel-off launch
  int64_t rec_cap;
  const int32_t* list;             // replay: packets with records
  int64_t nlist;
  const int64_t* start;            // replay: sorted record range [start, end) per packet
  const int64_t* end;
  const unsigned long long* skey;  // replay: sorted records
  const double* sc;
  // Replay control variate: each segment's score is weighted by A - B with
  // B = vtab[(cell*nfb + frequency bin)*ndir + direction class] of the
  // segment's start state (nullptr: B = 0).  vsum/vcnt (learning replay):
  // A and 1 added per segment start.  all != 0: every packet of the range is
  // replayed, not only those with records (B also weights packets whose A
  // is zero).
  const double* vtab;
  double* vsum;
  double* vcnt;
  int32_t nfb, ndir;
  int32_t all, pad2_;
  double lnumin, lnurat;           // frequency bins: nfb log-uniform bins of [numin, numin*exp(lnurat)]
};
constexpr int kAdjEvBits = 24;    // event index bits of a record key

// Arguments of the emission-table kernels (mcrt_setemiss.cuh).
struct SetemissArgs {
  int32_t nopac, ndg, nlammax, nT, nnu, pad_;
  const int32_t* nlambda;       // [nopac]
  const double* nudust;         // (nlammax, nopac), descending nu per species
  const double* kappad;
  const double* adust;
  const double* Tint;           // [nT] temperature grid [eV]
  const double* nuint;          // [nnu] frequency grid in units of kT
  double* kapint;               // (nT, nnu, nopac) out: normalised cumulative
  double* kappap;               // (nT, nopac) out: Planck mean
  double* kappar;               // (nT, nopac) out: Rosseland mean
  unsigned long long* misses;   // qsimp integrals that hit the level limit
};

// One work item of the batch kernel (mcrt_batch.cuh): a chunk of one model's
// packet range.
struct BatchItem {
  int32_t model;
  int32_t pad_;
  int64_t lo, hi;             // 1-based packet range of the chunk
};

struct LaunchParams {
  DevModel m;
  DevTallies t;
  int64_t np, lo, hi;           // iteration size and this launch's packet range
  int64_t block0;               // first random block of the iteration: (iter-1)*np
  const int64_t *block0_dev;    // non-null: block0 read from device memory (graphs replayed over iterations)
  int64_t ns, npacc, npaccstar; // packet split (newdisktherm_5_fuv.f90:158-191)
  int32_t ipeel, ips;
  int32_t event_batch;          // warp scheduler: lanes that must wait before events run
  int32_t fetch_off;            // 1: a finished packet starts no new packet (wavefront tail launch)
  double nphot_diff;            // nphot of emit_common's surface heating (ns of this shard)
  int32_t g1, g2;               // generator initial seeds
  unsigned long long *next;     // dynamic packet counter
  PeelJob *jobs;                // peel-off job queue (nullptr: peel inline)
  double *job_nub;              // [job_cap] packet frequency per job (filter-band and nested images only)
  unsigned long long *njobs;    // jobs queued
  int64_t job_cap;
  mcrt_packet_log *log;
  int64_t nlog;
  int64_t log_off;              // log entry of the launch's k-th packet: k + log_off
  int32_t *err;                 // device error flags
  int64_t walk_limit;           // crossings after which a walk is given up (geometry failure)
  AdjointArgs adj;
};

}  // namespace mcrt
