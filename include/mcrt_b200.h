/*
 * mcrt_b200.h -- C ABI of the B200 Monte Carlo photon-packet engine.
 *
 * The engine replaces the per-packet loop of the Fortran routine
 *   subroutine disk(converge,iter,i1)          newdisktherm_5_fuv.f90:1-663
 * (emission -> propagate -> tauint cell walk -> scatter / absorb+reemit ->
 * peel-off -> SED and image tallies), the rank reduction of its tallies
 * (newdisktherm_5_fuv.f90:520-604) and the Lucy temperature update
 *   subroutine tfinal(nphot,iter,converge)     tfinal_5_test1.f90:1-447
 *   function   dusttemp(...)                   dusttemp_5.f90:8-152
 * One GPU replaces all MPI ranks.  The Fortran driver keeps building the
 * model (gridset, dustinit, atmosinit) and writing FITS output; it hands the
 * module arrays it already owns to this library through the structs below.
 *
 * Conventions at the boundary are the reference's own:
 *   - arrays are Fortran column-major with the reference's dimensions,
 *     e.g. densarr(nrg,ntg,npg,ndg+2) is passed as a flat pointer whose
 *     element (ir,it,ip,id) (1-based) sits at
 *     (ir-1) + nrg*((it-1) + ntg*((ip-1) + npg*(id-1)));
 *   - lengths are in stellar radii, frequencies in eV (lambda[um] = 1.2398/nu),
 *     temperatures in the reference's "eV units" (Kelvin / 11605);
 *   - Fortran LOGICAL arrays are passed as int32 (0 = .false.).
 * All pointers are caller-owned; the library copies inputs to the GPU on
 * upload and copies tallies out on download and keeps no host pointer after
 * a call returns.  Errors are return codes, never process exits; a message is
 * available from mcrt_last_error().  A context is bound to one CUDA device
 * and is not re-entrant (one host thread per context).
 */
#ifndef MCRT_B200_H
#define MCRT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ---- */
#define MCRT_OK               0
#define MCRT_ERR_ARG          1   /* bad argument / inconsistent sizes          */
#define MCRT_ERR_CUDA         2   /* CUDA runtime error (message has details)    */
#define MCRT_ERR_UNSUPPORTED  3   /* model feature outside the built scope       */
#define MCRT_ERR_GEOM         4   /* packets lost to geometry failures (mcrt_set_limits) */
#define MCRT_ERR_TIMEOUT      5   /* wave-loop watchdog ended a run (mcrt_set_limits)    */
#define MCRT_ERR_STATE        6   /* call order violated (e.g. run before upload)*/

/* ---- fixed reference dimensions ---- */
#define MCRT_NDG2   10    /* ndg+2 density components per cell, grid_mod_5.f90:15 */
#define MCRT_NO      8    /* SED components, tts_mod_5.f90:30                      */
#define MCRT_IZMAX 145    /* zeta-series terms of bbfreq, random.f90:12            */

/* ---- scheduling of the transport kernels ---- */
#define MCRT_SCHED_PACKET  0   /* one thread runs one packet start to finish         */
#define MCRT_SCHED_WARP    1   /* lanes step rays in lockstep, events run in batches */
#define MCRT_SCHED_WAVE    2   /* wavefront: walk kernel and event kernel alternate  */
                               /* over a pool of in-flight packets kept in HBM       */

/* ---- arithmetic of the transport kernels ---- */
#define MCRT_PREC_FP64   0   /* everything in FP64 (event-for-event with the oracle) */
#define MCRT_PREC_MIXED  1   /* FP32 walk and scattering; FP64 sphere roots, tau sums, tallies */

/*
 * Run configuration: the scalars of tts_mod/grid_mod/dust_mod/spot_mod that
 * the packet loop reads.  Field names follow the reference's variables.
 */
typedef struct mcrt_config {
  /* grid wall counts (grid_mod_5.f90:10); cells are (nrg-1)x(ntg-1)x(npg-1) */
  int32_t nrg, ntg, npg;
  /* dust tables (dust_mod_5.f90:7-16): species, table lengths */
  int32_t nopac, nlammax, nT, nnu;
  /* stellar atmosphere CDF length (atmos_interp_mod.f90:5) */
  int32_t nhnu;
  /* SED / peel-off / image binning (tts_mod_5.f90:19-62) */
  int32_t nfreq, nmu, nph, nap, npeel, nxhst;
  /* switches */
  int32_t output_imcube;     /* image_m_* cube on (IMCUBE=YES)                */
  int32_t partial_peeloff;   /* tts_mod_5.f90:34                              */
  int32_t limb;              /* 0 uniform, 1 Eddington limb darkening         */
  int32_t iplanckst;         /* 1: star emits a Planck spectrum               */
  int32_t idust;             /* 0 Rayleigh, 1 dustmat phase matrix (setup.f90:152) */
  int32_t ilucy;             /* must be 1: Lucy reemission (emit_common_2.f90:59) */
  int32_t iffuv;             /* FUV mean-intensity tally and FUV-only packets */
  int32_t ispot, nspot;      /* hot spots (spot_mod.f90)                       */
  int32_t pad0;
  /* physics scalars */
  double rstar;              /* stellar radius [Rsun]                          */
  double tstar;              /* stellar temperature [K/11605]                  */
  double tstarave;           /* tstarave [K/11605] (dusttemp normalisation)    */
  double tshock;             /* hot-spot temperature [K/11605]                 */
  double fspot;              /* hot-spot area fraction                         */
  double accfrac, accfrac2;  /* disk-accretion and hot-spot packet fractions   */
  double isrf_frac;          /* external-illumination packet fraction          */
  double rddust;             /* disk inner dust radius [R*] (point-source switch) */
  double rmaxi;              /* image half size [R*]                           */
  double numin, lnurat;      /* SED frequency grid: numin [eV], log(numax/numin) */
  double autors;             /* AU -> R* (setup.f90:45)                        */
  double ifuv_ori;           /* FUV packet energy (newdisktherm_5_fuv.f90:206) */
  /* spot geometry (spotset.f90) */
  double cspot1, sspot1, scspot1, ssspot1;
  double cspot2, sspot2, scspot2, ssspot2;
  double csprad;
  /* Filter-band images (output_imfilt, peeloff_3d_2_test.f90:245-285): the
   * number of filter curves nfilt (the reference's nbnd, tts_mod_5.f90:62)
   * and the leading dimension nwfiltmax of mcrt_tables.filtwave/filtphi
   * (filt_mod.f90:10-14).  output_imfilt = 0 leaves the images off. */
  int32_t output_imfilt, nfilt, nwfiltmax, pad_filt;
  /* Multi-wavelength nested ("sparse") images (output_imsparse,
   * peeloff_3d_2_test.f90:302-309, type_nested_image.f90:75-101): per
   * inclination and Stokes parameter, sparse_nlev nested square images of
   * sparse_dim^2 pixels (half sizes mcrt_tables.sparse_levels) times
   * sparse_nnu bins in log10(frequency [Hz]) from sparse_lognu_min to
   * sparse_lognu_max -- the values nested_image_setup receives
   * (initarr_2_new.f90:170-190), in the reference's single precision. */
  int32_t output_imsparse, sparse_dim, sparse_nlev, sparse_nnu;
  float   sparse_lognu_min, sparse_lognu_max;
} mcrt_config;

/*
 * Spherical-polar grid and per-cell model (grid_mod_5.f90:29-63, gridset).
 */
typedef struct mcrt_grid {
  const double  *rarr, *r2arr;                          /* [nrg]            */
  const double  *thetarr, *costarr, *sintarr, *tan2arr; /* [ntg]; tan2arr=-1 flags theta=90 */
  const double  *phiarr, *aarr, *barr;                  /* [npg]            */
  const double  *densarr;     /* [nrg,ntg,npg,10] g/cm^3                    */
  const int32_t *findopac;    /* [nrg,ntg,npg,10] opacity species, 1-based  */
  const int32_t *diffus;      /* [nrg,ntg,npg] LOGICAL                      */
  const int32_t *diffdir;     /* [nrg,ntg,npg]                              */
  const double  *tdust;       /* [nrg,ntg,npg] [K/11605]                    */
  const double  *vcell;       /* [nrg,ntg,npg] cm^3                         */
  const double  *ravearr;     /* [nrg-1] (accretion emission)               */
  const double  *Ldint;       /* [nrg-1] accretion luminosity CDF           */
  const double  *hdisk;       /* [nrg-1] disk scale height                  */
  /* Gas velocity field (gridset_5_model13new.f90:1383-1480), optional: all
   * three NULL is a gas at rest.  With it, tfinal adds the adiabatic
   * (Tint*divv) and advective (vr*dT/dr + vtheta*dT/dtheta) terms of
   * dusttemp (dusttemp_5.f90:42-53) and forms the temperature gradients
   * from 31x31-cell smoothings over its passes (tfinal_5_test1.f90:61-200). */
  const double  *vrarr;       /* [nrg,ntg,npg] cm/s                         */
  const double  *vthetarr;    /* [nrg,ntg,npg] cm/s                         */
  const double  *divvarr;     /* [nrg,ntg,npg] cm/s per stellar radius      */
  /* Small-grain (VSG/PAH) emission level per cell, optional: the row of the
   * Draine emissivity table (mcrt_tables.draine) a small grain absorbing in
   * the cell re-emits from, the reference's imean (int_mean.f90:67-80).
   * Iteration 1 uses row 2 whatever imean holds, as the reference's first
   * iteration does (emit_common_2.f90:35-39).  NULL: row 1 afterwards, which
   * is what the reference's int_mean gives: its jmean tally is switched off
   * (usejmean = .False., tauint_3d_2_fuv.f90:27), so every cell's intensity
   * ratio is 0 and locates below uratio_arr(1). */
  const int32_t *imean;       /* [nrg,ntg,npg], 1..nemit                    */
} mcrt_grid;

/*
 * Dust, atmosphere and observer tables (dust_mod_5.f90, atmos_interp_mod.f90,
 * tts_mod_5.f90:36-47, setup.f90:115-195).
 */
typedef struct mcrt_tables {
  const int32_t *nlambda;                     /* [nopac]                     */
  const double  *nudust, *kappad, *adust, *gdust, *pldust; /* [nlammax,nopac] */
  const double  *kappav;                      /* [nopac]                     */
  const double  *kapint;                      /* [nT,nnu,nopac] normalised   */
  const double  *lTint, *Tint;                /* [nT]                        */
  const double  *nuint;                       /* [nnu]                       */
  const double  *kappap, *kappar;             /* [nT,nopac]                  */
  const double  *atmosnu, *hnuint, *lognu, *loghnu;        /* [nhnu]         */
  const double  *aperture2;                   /* [nap] squared apertures     */
  const double  *u;                           /* [nmu] SED cos(theta) bins   */
  const double  *coste_arr, *sinte_arr, *cospe_arr, *sinpe_arr; /* [npeel]   */
  const double  *limb_prob;                   /* [100] Eddington CDF (samptabl.f90:1-23), limb=1 only */
  /* Tabulated scattering matrices (stokes6.f90, stokespeel6.f90, tab_mod.f90),
   * optional; NULL selects the analytic dustmat phase matrix.
   * mueller(6,narr,nlammax,nopac): S11 S12 S22 S33 S34 S44 (Bohren & Huffman
   * sign of S34) on narr cosine bins, bin i centred on -1+(i-0.5)*2/narr as
   * reatab.f90 resamples them, for every species and wavelength node of
   * nudust; S11 normalised like reatab (sum of S11*dct/2 over the bins = 1).
   * A scattering interpolates two wavelength nodes with opacset's weights. */
  const double  *mueller;
  int32_t        narr, pad_mueller;
  /* External illumination (ISRF packets, isrf_frac > 0), optional: the
   * sampling table that isrf_cdf.f90 leaves in isrf_mod, isrf(nisrf,3) =
   * cdf_i, logcdf_i, logfreq_i (frequencies in eV, the first row as that
   * routine sets it: cdf 0, log cdf -99, log freq 0).  NULL when unused. */
  const double  *isrf;
  int32_t        nisrf, pad_isrf;
  /* Small-grain (VSG/PAH) emission spectra, needed when a cell holds a
   * small-grain component (ids 5-8): the tables draine_cdf.f90 leaves in
   * draine_mod, concatenated as cdf_d(nemit,ndraine), logcdf_d(nemit,ndraine)
   * and logfreq_d(ndraine), frequencies ascending in eV (the first entries
   * as that routine sets them: cdf 0, log cdf -10, log freq 0).  A small
   * grain re-emits from row imean of the cell (rep_draine_new.f90).  NULL
   * when the model has no small grains. */
  const double  *draine;
  int32_t        nemit, ndraine;
  /* Filter curves of the filter-band images (filt_mod.f90, read by
   * filt_nu.f90), needed when output_imfilt = 1: filtwave(nwfiltmax,nfilt)
   * frequencies in Hz, ascending within each curve, filtphi(nwfiltmax,nfilt)
   * the normalised responses, and nwfilt(nfilt) the reference's line counts
   * (a curve uses its first nwfilt-1 points, filt_nu.f90:30). */
  const int32_t *nwfilt;
  const double  *filtwave, *filtphi;
  /* Half sizes of the nested images [R*], ascending, as find_levels
   * (type_nested_image.f90:62-73) leaves them in image%levels; needed when
   * output_imsparse = 1. */
  const float   *sparse_levels;                                     /* [sparse_nlev] */
} mcrt_tables;

/*
 * Tallies of one iteration (caller-owned; any pointer may be NULL to skip it).
 * Types and shapes are the reference's (tts_mod_5.f90, grid_mod_5.f90).
 */
typedef struct mcrt_tallies {
  int32_t *nabs, *dbig, *dsg, *killed;        /* [nrg,ntg,npg]               */
  double  *dtauabs, *fuvmean;                 /* [nrg,ntg,npg]               */
  float   *si, *sq, *su, *sv, *si2, *sq2, *su2, *sv2, *nums, *aveinc; /* [nfreq,nmu,nph,nap,8] */
  float   *ti, *tq, *tu, *tv, *ti2, *tq2, *tu2, *tv2, *numt;          /* [nfreq,npeel,nap,8]    */
  float   *image_m_i, *image_m_q, *image_m_u, *image_m_v;             /* [npeel,nxhst,nxhst,nfreq] */
  double  *scalars;   /* [MCRT_NSCALARS], see MCRT_S_* below                 */
  int64_t *counters;  /* [MCRT_NCOUNTERS], see MCRT_C_* below                */
  /* Filter-band images (output_imfilt = 1): Stokes I, Q, U, V and Stokes I
   * by origin (d disk, s star, e envelope, o outflow: i_orig 2, 1, 3, 4),
   * tts_mod_5.f90:67-68 */
  float   *image_b_i, *image_b_q, *image_b_u, *image_b_v;             /* [npeel,nxhst,nxhst,nfilt] */
  float   *image_b_d, *image_b_s, *image_b_e, *image_b_o;             /* [npeel,nxhst,nxhst,nfilt] */
  /* Nested images (output_imsparse = 1), image_ms_i..v of tts_mod_5.f90:76
   * held dense: [sparse_dim, sparse_dim, sparse_nnu, sparse_nlev, npeel]
   * (pixel ix fastest); the driver inserts the non-zero pixels into its
   * smart images for nested_image_write. */
  float   *image_ms_i, *image_ms_q, *image_ms_u, *image_ms_v;
} mcrt_tallies;

/* scalars[] of one iteration (the reference's module scalars) */
#define MCRT_S_FLUX     0   /* flux   (propagate_5_fuv.f90:265)  */
#define MCRT_S_SFLUX    1   /* sflux                             */
#define MCRT_S_NSCAT    2   /* nscat                             */
#define MCRT_S_TOT      3   /* tot    (propagate_5_fuv.f90:72)   */
#define MCRT_S_SCOUNT   4   /* scount (propagate_5_fuv.f90:320)  */
#define MCRT_S_DSCOUNT  5   /* dscount                           */
#define MCRT_S_AFLUX    6   /* aflux  (tauint_3d_2_fuv.f90:185)  */
#define MCRT_S_ABFLUX   7   /* abflux (propagate_5_fuv.f90:210)  */
#define MCRT_NSCALARS   8

/* counters[] (device-side work statistics, not reference outputs) */
#define MCRT_C_PACKETS       0  /* packets run                          */
#define MCRT_C_CROSSINGS     1  /* cell crossings of the transport walk */
#define MCRT_C_INTERACTIONS  2  /* scatterings + absorptions            */
#define MCRT_C_SCATTERS      3
#define MCRT_C_PEELS         4  /* peel-off walks started               */
#define MCRT_C_PEEL_CROSS    5  /* cell crossings of peel-off walks     */
#define MCRT_C_PEEL_BINNED   6  /* peel-offs that reached an image/SED  */
#define MCRT_C_GEOM_FAIL     7  /* packets dropped: no wall found       */
#define MCRT_C_RESETS        8  /* testgrid random re-locations         */
#define MCRT_C_KILLED        9  /* packets killed after 10000 events    */
#define MCRT_C_EXITED       10  /* packets that left the grid           */
#define MCRT_C_STARHITS     11  /* packets absorbed + re-emitted by the star */
#define MCRT_C_PEEL_RESETS  12  /* testgrid re-locations inside queued peel-off walks */
#define MCRT_C_PEEL_JOBS    13  /* peel-off jobs queued for the peel-off kernel */
#define MCRT_C_WAVES        14  /* walk/event launch pairs of the wavefront schedule */
#define MCRT_C_LAUNCHES     15  /* kernels launched by mcrt_run_iteration calls */
#define MCRT_NCOUNTERS      16

/* Per-packet summary used by the parity tests (event-for-event checks). */
typedef struct mcrt_packet_log {
  int64_t  iphot;
  int32_t  nscat, nabs, ncross, nstar;   /* event counts                  */
  int32_t  status;                        /* 0 exited, 1 killed, 2 fuv-drop, 3 geometry failure */
  int32_t  ir, it, ip;                    /* last cell                      */
  int32_t  ndraws;                        /* random numbers consumed        */
  int32_t  iflag, i_orig, pad;
  double   nub, cost, phi, sip, sqp, sup, svp, xp, yp, zp;
} mcrt_packet_log;

typedef struct mcrt_ctx mcrt_ctx;

/* Create a context on CUDA device `device` for the sizes in *cfg.
 * Replaces the rank set-up of newtts.f90:36-207 for the packet engine. */
int mcrt_create(const mcrt_config *cfg, int device, mcrt_ctx **out);

/* Upload the grid/model arrays that gridset fills every iteration
 * (newdisktherm_5_fuv.f90:89 -> gridset_5_model13new.f90). */
int mcrt_upload_grid(mcrt_ctx *ctx, const mcrt_grid *grid);

/* diskflux (flux_test.f90:1-143): the tallies as mcrt_download_tallies
 * gives them, with the reference's output normalisation applied on the
 * device in its FP32 order of operations: the SED si..sv divided by
 * np/nmu/nph/(ltot/lsol), and where nums > 1 the relative errors
 * si2 = sqrt((si2 - si^2/nums)/(nums-1)*nums)/si + 1/nums (sq2..sv2 the
 * same without the 1/nums term, relative to si), aveinc/nums (errors 0
 * elsewhere); with ipeel = 1 the peeled SED ti..tv and the image cubes
 * divided by np/(ltot/lsol), and where numt > 1 the relative errors
 * ti2 = sqrt((ti2*numt/ti^2 - 1)/(numt-1)) (0 elsewhere).  As in the
 * reference a peeled Stokes sum of 0 gives a NaN error.  np is the
 * iteration's packet count, ltot_lsol the driver's ltot/lsol.  The
 * filter-band images (image_b_*) are not built. */
int mcrt_diskflux(mcrt_ctx *ctx, int64_t np, double ltot_lsol, int32_t ipeel, mcrt_tallies *out);

/* Check a grid before it is uploaded, on the host only (no device, no
 * context): the walls finite and increasing, every density finite and
 * non-negative, every temperature finite and non-negative, every cell with
 * dust of finite positive volume.  The reference reads these from its
 * parameter files and would run on with a NaN (gridset_5_model13new.f90);
 * here a bad value is refused with MCRT_ERR_ARG and the first offending
 * entry named in `msg` (msg_len bytes, may be NULL).  mcrt_upload_grid
 * runs the same check before any CUDA call. */
int mcrt_check_grid(const mcrt_config *cfg, const mcrt_grid *grid, char *msg, int32_t msg_len);

/* Watchdogs of the packet loop (no reference counterpart: the reference
 * stops the program on a geometry failure, testgrid.f90 / tauint, and has
 * no time limit).
 *   walk_crossings: crossings of one walk after which the walk is given up
 *                   and its packet dropped as a geometry failure (<= 0:
 *                   the default 5e7);
 *   waves:          walk/event launch pairs of one wavefront loop after
 *                   which mcrt_run_iteration stops and returns
 *                   MCRT_ERR_TIMEOUT, abandoning the packets in flight
 *                   (<= 0: the default 4e8); the context stays usable;
 *   geom_fraction:  mcrt_run_iteration returns MCRT_ERR_GEOM when more
 *                   than this fraction of its packets was lost to
 *                   geometry failures (default 1e-6; < 0: never).  The
 *                   tallies hold every other packet and the counter
 *                   MCRT_C_GEOM_FAIL the losses.
 * Takes effect at the next run. */
int mcrt_set_limits(mcrt_ctx *ctx, int64_t walk_crossings, int64_t waves, double geom_fraction);

/* Upload dust, atmosphere and observer tables (dustinit dust_5.f90:345-504,
 * atmosinit starbarb_2.f90:3-122, setup.f90:115-195). */
int mcrt_upload_tables(mcrt_ctx *ctx, const mcrt_tables *tab);

/* Select FP64 or mixed-precision transport (MCRT_PREC_*). */
int mcrt_set_precision(mcrt_ctx *ctx, int32_t mode);

/* Select the kernel schedule (MCRT_SCHED_*; default MCRT_SCHED_WAVE) and
 * its batch size (1..32): for the warp schedule, how many lanes of a warp
 * must wait for an event before the warp stops stepping rays to run them
 * (default 16); for the wavefront schedule, how many lanes of a walk warp
 * must be idle before it takes new walks from the queue (default 4).  Every
 * packet's history, and so every tally up to the order of floating-point
 * additions, is independent of either choice.  No reference counterpart
 * (the reference runs one packet per MPI rank thread). */
int mcrt_set_schedule(mcrt_ctx *ctx, int32_t schedule, int32_t event_batch);

/* Wavefront schedule sizes.  `slots`: in-flight packet slots (default
 * 2,097,152; 744 bytes of device memory each).  `peel_jobs`: capacity of the
 * peel-off job queue in jobs (192 bytes each, 200 with filter-band or nested
 * images; 0 = default, 16 x slots
 * within [8,388,608, 67,108,864]; else at least 2 x slots); the loop runs
 * the peel-off kernel whenever fewer than `slots` free jobs remain and
 * before the tail launch, whose peel-offs beyond the capacity are walked
 * inline.
 * `tail_packets`: once every packet of the range has started and at most
 * this many are in flight, one launch of the warp-scheduled loop finishes
 * them (negative = default, 8 per lane of that launch; 0 = never, waves to
 * the end).  Takes effect at the next mcrt_run_iteration.  No reference
 * counterpart. */
int mcrt_set_wave_pool(mcrt_ctx *ctx, int64_t slots, int64_t peel_jobs, int64_t tail_packets);

/* Zero the tallies of one iteration (initarr_2_new.f90:79-119). */
int mcrt_reset_tallies(mcrt_ctx *ctx);

/* Run packets iphot_lo..iphot_hi (1-based, inclusive) of an iteration of
 * np packets: the loop `do iphot=1,np` of newdisktherm_5_fuv.f90:220-491.
 * Packet iphot of iteration iter draws from block (iter-1)*np + iphot-1
 * of L'Ecuyer-Cote generator `generator` seeded by (seed1,seed2) as
 * user_set_all does (user_set_generator.f90:250-273,
 * ecuyer_cote_mod.f90:297-395); blocks are 2^30 draws apart.
 * ipeel=1 peels each emission/interaction off to every inclination.
 * Tallies accumulate on the device until mcrt_reset_tallies. */
int mcrt_run_iteration(mcrt_ctx *ctx, int64_t np, int64_t iphot_lo,
                       int64_t iphot_hi, int32_t iter, int32_t ipeel,
                       int32_t seed1, int32_t seed2, int32_t generator);

/* Copy the tallies to caller-owned arrays (the reduced values of
 * newdisktherm_5_fuv.f90:520-604 for a single GPU). */
int mcrt_download_tallies(mcrt_ctx *ctx, mcrt_tallies *out);

/* Add a tally set (host arrays, the layout mcrt_download_tallies writes)
 * into this context's device tallies: the summing half of the rank
 * reduction newdisktherm_5_fuv.f90:520-604 when the ranks reduce on the host
 * (download, sum across processes, mcrt_reset_tallies, accumulate the sum).
 * NULL members are skipped.  The diffusion absorption counts are not part of
 * mcrt_tallies; reduce through mcrt_device_tallies_view to include them. */
int mcrt_accumulate_tallies(mcrt_ctx *ctx, const mcrt_tallies *in);

/* The device tally buffer as three contiguous segments, for an in-place
 * all-reduce across GPUs (NCCL sum) -- the MPI_ALLREDUCE block of
 * newdisktherm_5_fuv.f90:520-604 without a host round trip.  Sum every
 * segment over the ranks, then call mcrt_refresh_diffusion and
 * mcrt_update_temperature.  Pointers are device addresses owned by the
 * context and valid until mcrt_destroy. */
typedef struct mcrt_device_tallies {
  double   *f64;  int64_t n_f64;  /* dtauabs, fuvmean, SEDs, peeled SEDs, images, scalars */
  uint64_t *u64;  int64_t n_u64;  /* counters                                            */
  int32_t  *i32;  int64_t n_i32;  /* nabs, dbig, dsg, killed, diffusion absorption counts */
} mcrt_device_tallies;
int mcrt_device_tallies_view(mcrt_ctx *ctx, mcrt_device_tallies *out);

/* Path-replay adjoint of the peeled outputs for packets lo..hi of an
 * np-packet iteration (with peel-offs).  Objective
 *   L = sum_k lam_psed[k] * ti[k] + sum_p lam_img[p] * image_m_i[p]
 * (peeled SED and monochromatic image, Stokes I; lam_img may be NULL).
 * Writes *objective = L of this run and grad[ncell*10] = dL/dlog(rho) per
 * cell and density component id (Fortran order (nrg,ntg,npg,10)), the
 * derivative of this run's estimate with its random numbers held fixed:
 * peel-off rays contribute -C*tau, and the packet's own path segments their
 * score (interaction density minus tau) times the peel-off contribution
 * that follows them.  Two passes: the forward run (peel-off kernel records
 * each job's weighted contribution) and a replay of the contributing
 * packets on the same streams.  Diffusion surfaces keep their
 * start-of-iteration temperature during both passes.  The device tallies
 * after the call hold both passes (reset before the next iteration).
 * Gradients of parameters of a density law follow by the chain rule over
 * grad.  No reference counterpart (the reference has no derivatives). */
int mcrt_adjoint(mcrt_ctx *ctx, int64_t np, int64_t iphot_lo, int64_t iphot_hi, int32_t iter,
                 int32_t seed1, int32_t seed2, int32_t generator,
                 const double *lam_psed, const double *lam_img, double *grad, double *objective);
/* Packets per adjoint chunk (default 2^25).  No reference counterpart.  The
 * adjoint runs its range in chunks: forward pass, record sort and replay
 * per chunk, with the gradient and objective summed.  Packets are
 * independent in the adjoint because diffusion heating is frozen, so the
 * sums equal a single pass.  A chunk whose peel-off records would reach 2^31
 * (the device sort's 32-bit count) is redone in halves; optically thick
 * models without diffusion cells can need that.  Every chunk's forward pass
 * ends with its own tail of long-lived packets, so large chunks are faster. */
int mcrt_set_adjoint_chunk(mcrt_ctx *ctx, int64_t packets);
/* Who drives the wavefront loop of mcrt_run_iteration.  No reference
 * counterpart.  1 (default): the device, as one CUDA-graph launch per
 * iteration whose WHILE node runs the event and walk launches and decides
 * on the device when to hand over to the tail launch; the host waits once.
 * It applies to iterations without peel-off jobs and outside the adjoint;
 * the graph is captured on the first such call and again whenever the
 * launch parameters change (packet range, seeds, grid or table uploads,
 * schedule settings), so the first call after a change also pays the
 * capture.  0: the host reads the queue sizes after every walk launch (as
 * peeled iterations and the adjoint always do).  Results do not depend on
 * it. */
int mcrt_set_wave_loop(mcrt_ctx *ctx, int32_t device_loop);
/* Control variate of the adjoint's replay.  No reference counterpart.  A
 * segment's score (delta at the interaction minus the optical depth of the
 * segment, per cell and component) has zero mean given the segment's start,
 * so it may be weighted by A - B instead of A, for any B fixed before the
 * segment: the gradient stays unbiased, and its variance drops where B is
 * close to A (the peel-off contributions still ahead of the packet).  With
 * nfb > 0, mcrt_adjoint first replays `pilot_packets` packets of another
 * generator (generator % 32 + 1, independent of the range) and tabulates
 * the mean A per (cell, frequency bin, direction class); bins with fewer
 * than `min_count` segment starts get B = 0.  Frequency bins: nfb
 * log-uniform bins of the SED's range (numin, lnurat); direction classes
 * (ndir = 4): radially outward or inward x moving away from or toward the
 * midplane (ndir = 1: none).  The replay then covers every packet of the
 * range, not only those with peel-off records.  Device memory: three
 * arrays of ncell*nfb*ndir doubles.  nfb = 0 switches it off (default). */
int mcrt_set_adjoint_baseline(mcrt_ctx *ctx, int32_t nfb, int32_t ndir, int64_t pilot_packets, double min_count);

/* Recompute the diffusion cells' end-of-iteration temperature of the last
 * mcrt_run_iteration from the (reduced) diffusion absorption counts and the
 * whole iteration's stellar packet count -- the single-process result of
 * emit_common_2.f90:260-339; each rank's packets were emitted with its own
 * counts, as each MPI rank heats a private copy in the reference. */
int mcrt_refresh_diffusion(mcrt_ctx *ctx);

/* The diffusion region of the next iteration: setdiffus(iter)
 * (setdiffus_5.f90:1-132, called from gridset_5_model13new.f90:1842 at the
 * start of every iteration) followed by gridset's temperature reset
 * (gridset_5_model13new.f90:1855-1866), on the device.  For each radius from
 * the dust radius out to rmaxd [R*], each theta cell of the upper hemisphere
 * marches toward the pole summing kappav*R* x chiR(tdave) x rho x dtheta x r
 * over its thermal components (tdave floored at 50 K when iter < 2); a cell
 * whose march reaches tau = 1 within h/20 (hdisk) of photon path starts a
 * diffusion run down to the midplane (diffdir -2), mirrored below it (+2) and
 * copied to every phi slice.  massd <= 0 (no disk) clears the region.  The
 * context's cell flags and start-of-iteration tdust are rewritten (tdust =
 * tdave, 0.1 K in diffusion and empty cells) for the next mcrt_run_iteration.
 * Needs mcrt_grid.hdisk and mcrt_tables.kappar.  tdave [nrg,ntg,npg] (every
 * entry positive) is read; diffus, diffdir [nrg,ntg,npg] and dcount (the
 * reference's count of diffusion cells) may be NULL; with all three NULL the
 * call returns without waiting for the device.  Cells without a thermal
 * component are never flagged (diffusion emission needs a temperature). */
int mcrt_setdiffus(mcrt_ctx *ctx, int32_t iter, double massd, double rmaxd,
                   const double *tdave, int32_t *diffus, int32_t *diffdir,
                   int64_t *dcount);

/* Lucy temperature update on the device: tfinal(nphot,iter,converge)
 * (tfinal_5_test1.f90:1-447) with dusttemp (dusttemp_5.f90:8-152).
 * tdave [nrg,ntg,npg] is read (previous iteration) and overwritten.
 * *converge is 0 ('no') or 1 ('yes') on entry and may be set to 1.
 * sig[0..2] receive the three convergence statistics of tfinal_5_test1.f90:346-348. */
int mcrt_update_temperature(mcrt_ctx *ctx, int32_t nphot, int32_t iter,
                            double *tdave, int32_t *converge, double *sig);

/* Allocation-free variant of mcrt_update_temperature (no counterpart in the
 * reference).  For callers that cannot allocate device memory while they
 * run, e.g. a Fortran driver stepping the Lucy loop inside a memory pool it
 * sized up front, or code that must not trigger cudaMalloc's implicit device
 * synchronisation between iterations.  Same inputs, outputs and result as
 * mcrt_update_temperature (sig to summation order), but the scratch lives in
 * a fixed 12 MiB device array inside the library, so models are limited to
 * nrg*ntg*npg <= 524288 cells (larger ones return MCRT_ERR_ARG).  The first
 * call on each context looks the array's device address up (with the
 * context's device current; a context created after a device reset looks
 * it up again) and should come before any stream capture.  All calls in the
 * process share the array: calls that overlap on a GPU (two contexts on one
 * device, or two host threads) race.  Models with a gas velocity field
 * (mcrt_grid.vrarr...) need pass buffers it does not have and are refused
 * with MCRT_ERR_UNSUPPORTED. */
int mcrt_update_temperature_noalloc(mcrt_ctx *ctx, int32_t nphot, int32_t iter,
                                    double *tdave, int32_t *converge, double *sig);

/* Parity support: record a mcrt_packet_log for the first `max_packets`
 * packets of the next mcrt_run_iteration (0 disables). */
int mcrt_enable_packet_log(mcrt_ctx *ctx, int64_t max_packets);
int mcrt_download_packet_log(mcrt_ctx *ctx, mcrt_packet_log *out, int64_t n);

/* Device time of the last mcrt_run_iteration's transport kernels [ms]. */
int mcrt_last_kernel_ms(mcrt_ctx *ctx, double *ms);

/* Per-kernel breakdown of the last wavefront-schedule run (zeros after a
 * run with another schedule): kernel_ms[4] = summed device time [ms] of the
 * walk, event, tail and peel-off launches (CUDA events on the engine's
 * stream); counts[6] = launches of each of those four, walks stepped by the
 * walk launches, cell crossings stepped by the walk launches.  No reference
 * counterpart (profiling aid). */
int mcrt_wave_stats(mcrt_ctx *ctx, double *kernel_ms, int64_t *counts);

/* Measurement support: record CUDA event `slot` (0..15) on the context's
 * stream, and the device time between two recorded events [ms]. */
int mcrt_mark(mcrt_ctx *ctx, int32_t slot);
int mcrt_elapsed_ms(mcrt_ctx *ctx, int32_t slot_a, int32_t slot_b, double *ms);

/* Overwrite a 256 MiB device buffer on the context's stream so that the next
 * launch starts with a cold L2 (timing hygiene between benchmark steps). */
int mcrt_flush_l2(mcrt_ctx *ctx);

/* Block until all work queued on the context's stream has finished. */
int mcrt_synchronize(mcrt_ctx *ctx);

const char *mcrt_last_error(mcrt_ctx *ctx);   /* NULL: the last failed context-free call of this thread */
void mcrt_destroy(mcrt_ctx *ctx);

/* Parameters of the density law of mcrt_model_density (lengths in stellar
 * radii unless noted). */
typedef struct mcrt_density_params {
  double rstar;        /* stellar radius [Rsun] */
  double autors;       /* AU in stellar radii (214.94 / rstar, setup.f90:45) */
  double rddust;       /* dust destruction radius = inner disk and envelope edge */
  double rmax;         /* outer grid radius */
  double rmaxd;        /* outer disk radius */
  double massd;        /* disk mass [Msun] */
  double a_exp, b_exp; /* disk density and flaring exponents */
  double h100_au;      /* disk scale height at 100 AU [AU] */
  double rate;         /* envelope infall rate [Msun/yr] */
  double rc;           /* centrifugal radius */
  double massc;        /* central mass [Msun] */
  double rhoamb;       /* ambient density floor [g/cm^3] */
  double thet1_deg;    /* cavity opening angle at rmax [deg] */
  double ex1;          /* cavity shape exponent */
  double rhoconst1;    /* cavity density [g/cm^3] */
} mcrt_density_params;

/* Density grid on the GPU: the disk + Ulrich envelope + polynomial cavity
 * model of gridset for one parameter set.  Replaces the density part of
 * gridset_5_model13new.f90: the disk (setup_wave.f90:60-88, scale height
 * setup.f90:96-99), the Ulrich envelope (envset.f90:157-160, densenv.f90:37-43;
 * the mu0 cubic of zerod.f90), the polynomial cavity (envset.f90:182-189,
 * densenv.f90:76-90), the disk's ownership of the cells where it is denser
 * than the envelope and cavity gas (gridset_5_model13new.f90:1217-1224) and
 * the cell volumes (:1147-1150).  In: walls rarr[nrg], thetarr[ntg]
 * (stellar radii, radians); `clump` (may be NULL) multiplies the envelope
 * per cell, Fortran (nrg-1, ntg-1, npg-1).  Out: densarr Fortran
 * (nrg, ntg, npg, 10) with components 2 (disk), 3 (envelope), 4 (cavity);
 * vcell (nrg, ntg, npg) [cm^3]; dlog_disk (may be NULL) Fortran
 * (nrg-1, ntg-1, 3) = d log rho_disk / d (log Mdisk, b, log h100) per cell,
 * analytic, zero outside the disk.  No context needed; runs on `device`. */
int mcrt_model_density(int32_t device, const mcrt_density_params *p, int32_t nrg, int32_t ntg, int32_t npg,
                       const double *rarr, const double *thetarr, const double *clump, double *densarr,
                       double *vcell, double *dlog_disk);

/* Emission tables on the GPU: replaces the temperature and frequency grids
 * of dustinit (dust_5.f90:486-494) and setemiss (dust_5.f90:507-699; the
 * reference splits the species over its MPI ranks and reduces).  No context
 * needed; runs on `device`.  In: the dust tables in the mcrt_tables layout
 * (nudust/kappad/adust Fortran (nlammax, nopac), nu strictly decreasing in
 * each column; nlambda[nopac]); ndg = the number of dust species (ids above
 * it are gas opacities, whose Planck mean is smoothed as the reference
 * does); nT >= 21, nnu <= 3072 (the reference: 500, 513).  Out (host
 * arrays): lTint[nT], Tint[nT], nuint[nnu], kapint (nT, nnu, nopac),
 * kappap and kappar (nT, nopac), ready for mcrt_upload_tables;
 * *qsimp_misses (may be NULL) = interval integrals that hit the 20-level
 * limit (the reference counts and ignores them); *device_ms (may be NULL) =
 * kernel time.  Allocates and frees its own device memory. */
int mcrt_setemiss(int32_t device, int32_t nopac, int32_t ndg, int32_t nlammax, const int32_t *nlambda,
                  const double *nudust, const double *kappad, const double *adust, int32_t nT, int32_t nnu,
                  double *lTint, double *Tint, double *nuint, double *kapint, double *kappap, double *kappar,
                  int64_t *qsimp_misses, double *device_ms);

/* ---- batched models (no reference counterpart) ----------------------------
 * The reference runs one model per MPI job (newdisktherm_5_fuv.f90, the
 * `disk` loop at :220-491 inside the Lucy iterations).  A batch runs one Lucy
 * iteration of many models in ONE graph launch.  Each model keeps its own context
 * (grid, tables, tallies, temperature); the packets of model i use block
 * (iter-1)*np[i] + iphot-1 of the generator's stream, so every model's
 * histories are those of mcrt_run_iteration(ctx[i], np[i], 1, np[i], iter, 0,
 * ...) and its tallies equal that call's up to FP64 summation order.  One
 * iteration is one CUDA graph launch: parameter upload, tally reset, the
 * packet loop, each model's diffusion-heating finalisation (the graph is
 * re-captured when np[], the seeds, the tuning or a context's grid, tables
 * or packet log change).  Two schedules: MCRT_BATCH_PERSISTENT runs every
 * model's packets in one persistent launch (blocks take (model, chunk)
 * items); MCRT_BATCH_WAVE runs each model's wavefront loop (the default
 * single-model schedule) on the device as a CUDA-graph WHILE node, the
 * models as parallel branches of the one graph.  No peel-offs (ipeel=0: the
 * temperature iterations; run the final peel-off iteration per context).
 * All contexts must be on one device with one precision and have their grid
 * and tables uploaded; they must outlive the batch. */
typedef struct mcrt_batch mcrt_batch;
#define MCRT_BATCH_PERSISTENT 0  /* one persistent launch over (model, packet chunk) work items */
#define MCRT_BATCH_WAVE       1  /* every model's wavefront loop on the device (graph WHILE node), models in parallel branches */
int mcrt_batch_create(mcrt_ctx *const *ctxs, int32_t n, mcrt_batch **out);
/* Resets each model's tallies, then one iteration of every model (np[i]
 * packets, n entries).  Blocks until done; the device time is read with
 * mcrt_batch_last_ms.  Follow with mcrt_update_temperature per context. */
int mcrt_batch_run_iteration(mcrt_batch *b, const int64_t *np, int32_t iter, int32_t seed1, int32_t seed2,
                             int32_t generator);
/* Autotuner: times one iteration of `sample_packets` per model for both
 * schedules at their defaults, keeps the faster (the persistent one only if
 * it wins by 10 %: its advantage on small samples shrinks as packet counts
 * grow; sample at a tenth of the production count or more) and searches its
 * knobs --
 * persistent: work items per warp (chunk size of the item queue), the warp
 * schedule's event batch, blocks per SM; wavefront: in-flight packet slots
 * per model (the packet queue size).  chosen[5] (may be NULL) = (schedule,
 * blocks per SM, event batch, items per warp, wave slots).  The tuning runs
 * overwrite the models' tallies. */
int mcrt_batch_tune(mcrt_batch *b, int64_t sample_packets, int32_t *chosen);
/* Schedule of the batch (MCRT_BATCH_PERSISTENT or MCRT_BATCH_WAVE) and, for
 * the wavefront, the in-flight packet slots per model (64..2^30). */
int mcrt_batch_set_schedule(mcrt_batch *b, int32_t mode, int64_t wave_slots);
/* Persistent schedule by hand: blocks_per_sm 0 = occupancy maximum,
 * event_batch 1..32, items_per_warp >= 1. */
int mcrt_batch_set_tuning(mcrt_batch *b, int32_t blocks_per_sm, int32_t event_batch, int32_t items_per_warp);
int mcrt_batch_last_ms(mcrt_batch *b, double *ms);
const char *mcrt_batch_last_error(mcrt_batch *b);
void mcrt_batch_destroy(mcrt_batch *b);

/* Library version string. */
const char *mcrt_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MCRT_B200_H */
