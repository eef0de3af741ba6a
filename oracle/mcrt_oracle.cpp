// mcrt_oracle.cpp -- CPU restatement of the reference's photon-packet loop.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker the parity tests, the
// smoke test and the CPU-baseline leg of bench.py compare the CUDA engine
// against.  The engine never links, loads or calls it.
//
// It restates, routine by routine and in FP64, the Fortran hot path of
// evc9pu/src3_mpi_cfitsio (paths relative to src3_mpi_cfitsio/):
//   packet loop       newdisktherm_5_fuv.f90:220-491
//   propagate         propagate_5_fuv.f90:1-326
//   tauint            tauint_3d_2_fuv.f90:5-210
//   radface/thetaface/phiface/closest_wall  radface.f90, thetaface.f90,
//                     phiface.f90, closest_wall.f90
//   testgrid          testgrid.f90:1-128
//   stokes, dustmat   stokes.f90:1-340, dustmat.f90:1-70
//   peeloff           peeloff_3d_2_test.f90:7-347
//   findangle3        findangle3.f90:1-70
//   stokespeel        stokespeel.f90:1-328
//   emission          initpspot.f90, initp_common.f90, initp_ps.f90,
//                     initpabs.f90, samptabl.f90, starbarb_2.f90:124-153
//   reemission        emit_common_2.f90:24-81, reemit.f90,
//                     lucydustfreq_2_test.f90:19-160, select_dust_2.f90
//   opacity           dust_5.f90:9-109 (opacset)
//   RNG               ecuyer_cote_mod.f90:252-293 (random_large_integer),
//                     random_standard_uniform_mod.f90:16-46, random.f90:197-250
//   temperature       tfinal_5_test1.f90:1-447, dusttemp_5.f90:8-152,
//                     dust_5.f90:144-172 (KapP)
//
// Per-packet random streams: packet iphot of iteration iter draws from block
// (iter-1)*np + iphot-1 of the L'Ecuyer-Cote generator selected by
// user_set_all(seed1,seed2,generator);
// block b starts at a^(b*2^30) times the generator's initial seed, the state
// reinitialize_current_generator(1) moves to (ecuyer_cote_mod.f90:335-337).
// Packet 1 therefore draws the same numbers as the first packet of a
// single-rank reference run.
//
// Parity status: the random-number arithmetic is pinned to the reference's
// own jump constants (a1w, a1vw, ecuyer_cote_mod.f90:14-15) and to an
// independent big-integer evaluation of the recurrences; the transport is
// pinned to analytic known answers (tests/).  The Fortran itself cannot be
// compiled here (no Fortran compiler, no cfitsio, no parameter files), so
// event-level parity with the unmodified reference is unpinned.
//
// Deliberate, documented deviations from undefined reference behaviour:
//   * SED cos(theta)/phi bins that fall one past the last bin (cost=-1,
//     phi=2pi exactly) are clamped into the last bin;
//   * findangle3 leaves ri1 unset when sint1 or sin(scattering angle) is
//     below 1e-8; ri1 = 0 is used there;
//   * geometry failures that stop the Fortran program drop the packet and
//     are counted instead.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/mcrt_b200.h"

namespace {

constexpr double PI = 3.1415926535897932384626433;   // constants.f90:6
constexpr double R2P = 2.0 * PI;
constexpr double RSOL = 6.9598e10;
constexpr double SIGT = 5.670400e-5;
constexpr double KB = 1.3806503e-16;
constexpr double MHY = 1.67262158e-24;
constexpr double HUGE_D = 1.7976931348623157e308;   // huge(1d0)

// ------------------------------------------------------------------ RNG --
constexpr int64_t M1 = 2147483563, M2 = 2147483399;
constexpr int64_t A1W = 1033780774, A2W = 1494757890;    // a^(2^30)
constexpr int64_t A1VW = 2082007225, A2VW = 784306273;   // a^(2^50)

int64_t mulmod(int64_t a, int64_t s, int64_t m) {
  return (int64_t)(((unsigned __int128)a * (unsigned __int128)s) % (unsigned __int128)m);
}
int64_t powmod(int64_t a, int64_t e, int64_t m) {
  int64_t r = 1 % m, b = a % m;
  while (e > 0) {
    if (e & 1) r = mulmod(r, b, m);
    b = mulmod(b, b, m);
    e >>= 1;
  }
  return r;
}

struct Rng {
  int32_t s1 = 1, s2 = 1;
  int64_t ndraws = 0;
  // random_large_integer (ecuyer_cote_mod.f90:252-293) * 1/M1
  // (random_standard_uniform_mod.f90:339)
  double ran() {
    int32_t k = s1 / 53668;
    s1 = 40014 * (s1 - k * 53668) - k * 12211;
    if (s1 < 0) s1 += (int32_t)M1;
    k = s2 / 52774;
    s2 = 40692 * (s2 - k * 52774) - k * 3791;
    if (s2 < 0) s2 += (int32_t)M2;
    int32_t z = s1 - s2;
    if (z < 1) z += (int32_t)(M1 - 1);
    ++ndraws;
    return (double)z * 4.656613057e-10;
  }
};

// rep_draine_new.f90: a small-grain re-emission frequency from row im of the
// Draine spectra: locate3 (bisection over the columns of row im, in the
// direction the row runs), then linear in log10 cdf and log10 nu.  The
// tables: cdf_d(nemit,ndraine), logcdf_d(nemit,ndraine), logfreq_d(ndraine).
double rep_draine(const mcrt_tables* t, int im, Rng& rng) {
  const double xran = rng.ran();
  const int ne = t->nemit, nd = t->ndraine;
  const double* cdf = t->draine;
  const double* lcdf = cdf + (int64_t)ne * nd;
  const double* lfrq = cdf + 2 * (int64_t)ne * nd;
  auto at = [&](const double* a, int j) { return a[(im - 1) + (int64_t)ne * (j - 1)]; };
  int jl = 0, ju = nd + 1;
  while (ju - jl > 1) {                           // locate3.f90:8-22
    const int jm = (ju + jl) / 2;
    if ((at(cdf, nd) > at(cdf, 1)) == (xran > at(cdf, jm))) jl = jm;
    else ju = jm;
  }
  int ifreq = jl;
  if (ifreq == nd) ifreq = ifreq - 1;
  if (ifreq == 0) ifreq = 1;
  const double logfreq = (std::log10(xran) - at(lcdf, ifreq)) / (at(lcdf, ifreq + 1) - at(lcdf, ifreq)) *
                             (lfrq[ifreq] - lfrq[ifreq - 1]) +
                         lfrq[ifreq - 1];
  return std::pow(10.0, logfreq);
}

// set_all_seeds (ecuyer_cote_mod.f90:350-395) for `generator`, then `block`
// applications of reinitialize_current_generator(1).
Rng stream(int32_t seed1, int32_t seed2, int32_t generator, int64_t block) {
  int64_t g1 = seed1, g2 = seed2;
  for (int g = 2; g <= generator; ++g) {
    g1 = mulmod(A1VW, g1, M1);
    g2 = mulmod(A2VW, g2, M2);
  }
  Rng r;
  r.s1 = (int32_t)mulmod(powmod(A1W, block, M1), g1, M1);
  r.s2 = (int32_t)mulmod(powmod(A2W, block, M2), g2, M2);
  return r;
}

// ------------------------------------------------------------- helpers ---
// locate (nr_2.f:131-154): bisection; j with xx(j) < x <= xx(j+1) for an
// ascending table, xx(j) >= x > xx(j+1) for a descending one; 1-based.
int locate(const double* xx, int n, double x) {
  int jl = 0, ju = n + 1;
  const bool asc = xx[n - 1] > xx[0];
  while (ju - jl > 1) {
    int jm = (ju + jl) / 2;
    if (asc == (x > xx[jm - 1])) jl = jm; else ju = jm;
  }
  if (jl == 0 && x == xx[0]) jl = 1;
  return jl;
}

double check(double x) {       // check.f90: clamp a cosine to [-1,1]
  if (x > 1.0) return 1.0;
  if (x < -1.0) return -1.0;
  return x;
}

// closest_wall.f90: keep the largest negative root and the two smallest
// non-negative roots.
struct Walls {
  double tn1, tp1, tp2;
  int in1, ip1, ip2;
  void reset() { tn1 = -HUGE_D; tp1 = HUGE_D; tp2 = HUGE_D; in1 = ip1 = ip2 = 0; }
  void insert(double t, int i) {
    if (t < 0.0) {
      if (t > tn1) { tn1 = t; in1 = i; }
    } else {
      if (t < tp1) { tp2 = tp1; ip2 = ip1; tp1 = t; ip1 = i; }
      else if (t < tp2) { tp2 = t; ip2 = i; }
    }
  }
  void next(bool on_wall, double& t, int& i) const {
    if (on_wall) {
      if (std::fabs(tn1) < std::fabs(tp1)) { t = tp1; i = ip1; }
      else { t = tp2; i = ip2; }
    } else { t = tp1; i = ip1; }
  }
};

// ------------------------------------------------------------- model -----
struct Model {
  mcrt_config c;
  const mcrt_grid* g;
  const mcrt_tables* t;
  int nrg, ntg, npg;
  int64_t ncell;             // nrg*ntg*npg
  double inczeta[MCRT_IZMAX];
  bool is_sg[MCRT_NDG2];
  double rmincgs;
  // walls padded by one element: the reference reads one past the last wall
  // when a peel-off steps to ir=nrg or a walk reaches it=ntg before testgrid
  // re-locates (testgrid.f90:92-93); the pad makes those reads defined.
  std::vector<double> rarr, r2arr, thetarr, costarr, tan2arr, phiarr, aarr, barr;
  void pad_walls() {
    auto padv = [](std::vector<double>& v, const double* a, int n, double pad) { v.assign(a, a + n); v.push_back(pad); };
    padv(rarr, g->rarr, nrg, 2.0 * g->rarr[nrg - 1]);
    padv(r2arr, g->r2arr, nrg, 4.0 * g->r2arr[nrg - 1]);
    padv(thetarr, g->thetarr, ntg, g->thetarr[ntg - 1]);
    padv(costarr, g->costarr, ntg, g->costarr[ntg - 1] - 1.0);
    padv(tan2arr, g->tan2arr, ntg, 0.0);
    padv(sintarr, g->sintarr, ntg, 0.0);
    padv(phiarr, g->phiarr, npg, g->phiarr[npg - 1]);
    padv(aarr, g->aarr, npg, g->aarr[npg - 1]);
    padv(barr, g->barr, npg, g->barr[npg - 1]);
  }

  // Diffusion surface bookkeeping (emit_common_2.f90:201-372): the number of
  // diffusion absorptions so far at each surface cell; the k-th one heats the
  // cell to T^4 = T0^4 + k dT^4, the recursion of emit_common_2.f90:260-272.
  std::atomic<int32_t>* ndiff = nullptr;
  double nphot_diff = 1.0;
  std::vector<double> sintarr;
  int iter = 1;              // the iteration (small grains re-emit from Draine row 2 in the first)

  int64_t cidx(int ir, int it, int ip) const {
    return (int64_t)(ir - 1) + (int64_t)nrg * ((it - 1) + (int64_t)ntg * (ip - 1));
  }
  double dens(int ir, int it, int ip, int id) const { return g->densarr[cidx(ir, it, ip) + ncell * (id - 1)]; }
  int fopac(int ir, int it, int ip, int id) const { return g->findopac[cidx(ir, it, ip) + ncell * (id - 1)]; }
};

void zetainit(double* inczeta) {  // random.f90:227-245
  for (int i = 0; i < MCRT_IZMAX; ++i) inczeta[i] = 0.0;
  for (int j = MCRT_IZMAX; j >= 1; --j) {
    double temp = 1.0 / (double)(j * j * j * j);
    for (int i = MCRT_IZMAX; i >= j; --i) inczeta[i - 1] += temp;
  }
}

// --------------------------------------------------------------- tallies -
struct Tally {
  int64_t ncell = 0, nsed = 0, npsed = 0;
  std::vector<int64_t> nabs, dbig, dsg, killed;
  std::vector<double> dtauabs, fuvmean;
  std::vector<double> sed[10];     // si sq su sv si2 sq2 su2 sv2 nums aveinc
  std::vector<double> psed[9];     // ti tq tu tv ti2 tq2 tu2 tv2 numt
  double scal[MCRT_NSCALARS] = {0};
  int64_t cnt[MCRT_NCOUNTERS] = {0};
  void init(int64_t nc, int64_t ns, int64_t np) {
    ncell = nc; nsed = ns; npsed = np;
    nabs.assign(nc, 0); dbig.assign(nc, 0); dsg.assign(nc, 0); killed.assign(nc, 0);
    dtauabs.assign(nc, 0.0); fuvmean.assign(nc, 0.0);
    for (auto& v : sed) v.assign(ns, 0.0);
    for (auto& v : psed) v.assign(np, 0.0);
  }
};

struct Images {       // shared across threads, atomic adds
  std::vector<double> im[4];
  std::vector<double> imb[8];   // filter-band images: I Q U V, then I by origin d s e o
  std::vector<double> ims[4];   // nested images, I Q U V, dense [dim,dim,nnu,nlev,npeel]
};

// math_binning.f90 ipos_sp: bin of x among nbin equal bins of [xmin,xmax]
// in single precision; 0 below the range, nbin+1 above it.
int ipos_sp(float xmin, float xmax, float x, int nbin) {
  if (xmax > xmin) {
    if (x < xmin) return 0;
    if (x > xmax) return nbin + 1;
  } else {
    if (x < xmax) return 0;
    if (x > xmin) return nbin + 1;
  }
  const float frac = (x - xmin) / (xmax - xmin);
  return (int)(frac * (float)nbin) + 1;
}

// math_binning.f90 locate_sp: jl with xx(jl) <= x < xx(jl+1) (1-based) by
// bisection, 1 at xx(1), n-1 at xx(n), -1 outside the table.
int locate_sp(const float* xx, int n, float x) {
  const bool ascnd = xx[n - 1] >= xx[0];
  int jl = 0, ju = n + 1;
  while (ju - jl > 1) {
    const int jm = (ju + jl) / 2;
    if (ascnd == (x >= xx[jm - 1])) jl = jm; else ju = jm;
  }
  if (x == xx[0]) return 1;
  if (x == xx[n - 1]) return n - 1;
  if (x > xx[n - 1] || x < xx[0]) return -1;
  return jl;
}

void atomic_add(double& x, double v) {
  std::atomic_ref<double> a(x);
  double old = a.load(std::memory_order_relaxed);
  while (!a.compare_exchange_weak(old, old + v, std::memory_order_relaxed)) {}
}

// ------------------------------------------------------------- packet ----
// Path-replay adjoint of the peeled outputs (engine's mcrt_adjoint, restated
// sequentially).  Objective L = sum lam_psed * ti + sum lam_img * image_m_i
// (Stokes I).  With the random numbers held fixed, dL/dlog(rho[c,id]) is
//   sum over peel-offs   -C * tau[c,id] along the peel ray
// + sum over segments k  A_k * (delta(c,id = interaction cell, species) - tau[c,id] along k)
// where C is a peel-off's weighted contribution and A_k the summed C of the
// packet's peel-offs after segment k (at interactions k, k+1, ...).  Pass 1
// runs the packet with peel-offs, pass 2 replays it (same stream, no
// peel-offs) and scores the segments.
struct Adjoint {
  const double* lam_psed = nullptr;   // [npsed] weights of ti
  const double* lam_img = nullptr;    // [nimg] weights of image_m_i
  std::vector<double>* grad = nullptr;   // [ncell*10] this thread's sums
  double obj = 0.0;
  bool record = false, replay = false;
  double A = 0.0;
  std::vector<std::pair<int, double>> ev;   // (event index, C) of the packet, in event order
  size_t pos = 0;
  std::vector<std::pair<int64_t, double>> cross;   // crossings of the current peel ray: (cell, length)
  // Control variate: a segment's score is weighted by A - B instead of A,
  // with B = vtab[cell, frequency bin] of the segment's start state, a
  // table fixed before the run (the score of a segment has zero mean given
  // its start, so any such B leaves the estimate unbiased).  vsum/vcnt, if
  // set, collect A per (cell, bin) at segment starts to build such a table.
  const double* vtab = nullptr;
  double* vsum = nullptr;
  double* vcnt = nullptr;
  int nfb = 1, ndir = 1;
  double lnumin = 0.0, lnurat = 1.0;
  double B = 0.0;
  double W() const { return A - B; }
};

struct Packet {
  const Model* m;
  Tally* T;
  Images* I;
  Rng rng;
  int ipeel;
  Adjoint* adj = nullptr;
  // taunum_mod / stokes_mod / tts_mod state
  double xp, yp, zp, rsq, rtot, ux, uy, uz, tau;
  double cost, sint, cosp, sinp, phi, sip, sqp, sup, svp;
  double nub, cosb, sinb, lp, ifuv;
  bool on_wall;
  int iflag, exitflag, i_orig;
  int geom_fail;
  // opacset outputs (dust_mod) and kapd (opacin_mod) for all species
  std::vector<double> kappa, albedo, g, pl, g2, onemg2, g2p1, twog, kapd;
  // statistics
  int32_t nscat = 0, nabsev = 0, ncross = 0, nstar = 0, ndiffev = 0;

  double ran() { return rng.ran(); }

  // ---------------------------------------------------------- opacset
  // dust_5.f90:9-109 for every species (the gas-mixing block :64-87 only
  // concerns gas-opacity species, which the supported models do not use).
  void opacset(double nu) {
    const mcrt_tables* t = m->t;
    const int nl = m->c.nlammax;
    for (int id = 0; id < m->c.nopac; ++id) {
      const double* nud = t->nudust + (int64_t)nl * id;
      const double* kd = t->kappad + (int64_t)nl * id;
      const double* ad = t->adust + (int64_t)nl * id;
      const double* gd = t->gdust + (int64_t)nl * id;
      const double* pd = t->pldust + (int64_t)nl * id;
      const int n = t->nlambda[id];
      if (nu >= nud[0]) {
        g[id] = gd[0]; pl[id] = pd[0]; kappa[id] = kd[0]; albedo[id] = ad[0];
      } else if (nu <= nud[n - 1]) {
        g[id] = gd[n - 1]; pl[id] = pd[n - 1]; kappa[id] = kd[n - 1]; albedo[id] = ad[n - 1];
      } else {
        int i0 = 1, i1 = n;
        while (i1 - i0 > 1) {
          int i = (i1 + i0) / 2;
          if (nu <= nud[i - 1]) i0 = i; else i1 = i;
        }
        double f = (nu - nud[i1 - 1]) / (nud[i0 - 1] - nud[i1 - 1]);
        double fm1 = 1.0 - f;
        g[id] = fm1 * gd[i1 - 1] + f * gd[i0 - 1];
        pl[id] = fm1 * pd[i1 - 1] + f * pd[i0 - 1];
        kappa[id] = fm1 * kd[i1 - 1] + f * kd[i0 - 1];
        albedo[id] = fm1 * ad[i1 - 1] + f * ad[i0 - 1];
      }
      g2[id] = g[id] * g[id];
      g2p1[id] = g2[id] + 1.0;
      onemg2[id] = 1.0 - g2[id];
      twog[id] = 2.0 * g[id];
    }
  }
  // The three call sites compute kapd with different association orders.
  void kapd_disk() {        // newdisktherm_5_fuv.f90:258-261, 338-340
    for (int id = 0; id < m->c.nopac; ++id) kapd[id] = kappa[id] * m->rmincgs * m->t->kappav[id];
  }
  void kapd_propagate() {   // propagate_5_fuv.f90:157-159
    for (int id = 0; id < m->c.nopac; ++id) kapd[id] = kappa[id] * m->c.rstar * RSOL * m->t->kappav[id];
  }
  void kapd_tauint() {      // tauint_3d_2_fuv.f90:199-201
    for (int id = 0; id < m->c.nopac; ++id) kapd[id] = kappa[id] * RSOL * m->c.rstar * m->t->kappav[id];
  }
  bool is_fuv(double nu) const { return nu <= 13.6 && nu >= 6.0; }

  // ------------------------------------------------------- frequencies
  double bbfreq(double teff) {     // random.f90:197-225
    double z0 = m->inczeta[MCRT_IZMAX - 1] * ran();
    double z1 = ran(), z2 = ran(), z3 = ran(), z4 = ran();
    int i = 1;
    while (z0 > m->inczeta[i - 1]) ++i;
    return -std::log(z1 * z2 * z3 * z4) * teff / (double)i;
  }
  double atmosfreq() {             // starbarb_2.f90:124-153
    const mcrt_tables* t = m->t;
    double xi = ran();
    int i = locate(t->hnuint, m->c.nhnu, xi);
    i = std::min(std::max(i, 1), m->c.nhnu - 1);   // a CDF that does not span [0,1) cannot index outside the table
    if (i > 1) {
      double logatm = t->lognu[i - 1] + (t->lognu[i] - t->lognu[i - 1]) / (t->loghnu[i] - t->loghnu[i - 1]) *
                                            (std::log10(xi) - t->loghnu[i - 1]);
      return std::pow(10.0, logatm);
    }
    return t->atmosnu[i - 1] + (t->atmosnu[i] - t->atmosnu[i - 1]) / (t->hnuint[i] - t->hnuint[i - 1]) * (xi - t->hnuint[i - 1]);
  }
  double lucydustfreq(double T0, int idust2) {   // lucydustfreq_2_test.f90:19-160
    const mcrt_tables* t = m->t;
    const int nT = m->c.nT, nnu = m->c.nnu;
    const double Tmax = 199999.0;
    if (T0 >= Tmax / 11605.0) return bbfreq(T0);
    double lT0 = std::log(T0);
    double xi = ran();
    int j = (int)((double)(nT - 1) * (lT0 - t->lTint[0]) / (t->lTint[nT - 1] - t->lTint[0])) + 1;
    j = std::min(std::max(j, 1), nT - 1);   // out-of-range j is undefined in the reference
    double f = (lT0 - t->lTint[j - 1]) / (t->lTint[j] - t->lTint[j - 1]);
    if (f < 0.0) f = 0.0;
    if (f > 1.0) f = 1.0;
    const double* K = t->kapint + (int64_t)nT * nnu * (idust2 - 1);
    auto kap = [&](int jj, int ii) { return K[(jj - 1) + (int64_t)nT * (ii - 1)]; };
    int i0 = 1, i1 = nnu;
    double P0 = (1.0 - f) * kap(j, i0) + f * kap(j + 1, i0);
    if (xi < P0) {
      if (P0 > 0.0) return T0 * xi * t->nuint[0] / P0;
      return T0 * t->nuint[0];
    }
    double P1 = (1.0 - f) * kap(j, i1) + f * kap(j + 1, i1);
    if (P1 > 1.0) P1 = 1.0;
    if (xi >= P1) {
      if (P1 < 1.0) {
        if (xi < 1.0) return T0 * t->nuint[nnu - 1] * (1.0 - P1) / (1.0 - xi);
        return T0 * t->nuint[nnu - 1];
      }
      return T0 * t->nuint[nnu - 1];
    }
    double P = 0.0;
    while (i1 - i0 > 1) {
      int i = (i0 + i1) / 2;
      P = (1.0 - f) * kap(j, i) + f * kap(j + 1, i);
      if (P > 1.0) P = 1.0;
      if (P < P0) { P0 = P; i0 = i; }
      if (P > P1) { P1 = P; i1 = 1; }
      if (P > xi) { i1 = i; P1 = P; } else { i0 = i; P0 = P; }
    }
    if (xi < P0) f = 0.0;
    else if (xi > P1) f = 1.0;
    else if (P0 <= 0.0) f = 0.5;
    else if (P1 <= 0.0) { /* f keeps its value */ }
    else if (xi <= 0.0) { /* f keeps its value */ }
    else f = std::log(xi / P0) / std::log(P1 / P0);
    return T0 * t->nuint[i0 - 1] * std::pow(t->nuint[i1 - 1] / t->nuint[i0 - 1], f);
  }

  // --------------------------------------------------------- emission
  void initp_sample() {            // initp_common.f90:1-29
    if (m->c.limb == 0) {
      cost = std::sqrt(ran());
    } else {                       // darkening, samptabl.f90:29-65
      double xr = ran();
      const double* prob = m->t->limb_prob;
      const int ntab = 100;
      const double delmu = 1.0 / (double)ntab;
      int n = std::min(std::max(locate(prob, ntab, xr), 1), ntab - 1);
      double xmu1 = delmu * (double)(n + 1);
      cost = xmu1 - (prob[n] - xr) / (prob[n] - prob[n - 1]) * delmu;
    }
    sint = std::sqrt(1.0 - cost * cost);
    phi = R2P * ran();
    cosp = std::cos(phi);
    sinp = std::sin(phi);
  }
  void initp_transform() {         // initp_common.f90:31-94
    if (std::fabs(cosb) < 0.9999999) {
      double costi = cost * cosb - sint * sinb * cosp;
      if (std::fabs(costi) > 1.0) {
        if (costi > 1.0) costi = 1.0;
        if (cost < -1.0) costi = -1.0;
      }
      double sinti = std::sqrt(1.0 - costi * costi);
      double phinew;
      if (sinti > 0.0000001) {
        double cospn = (cost - costi * cosb) / (sinti * sinb);
        if (std::fabs(cospn) > 1.0) cospn = (cospn < 0.0) ? -1.0 : 1.0;
        if (phi < PI) {
          phinew = std::acos(cospn);
          if (phinew > PI) phinew = PI;
        } else {
          phinew = R2P - std::acos(cospn);
          if (phinew < PI) phinew = PI;
        }
      } else {
        phinew = 0.0;
      }
      phi = phinew;
      cost = costi;
      sint = sinti;
    } else {
      if (cosb < 0.0) cost = -cost;
    }
    phi = phi + lp;
    if (phi > R2P) phi = phi - R2P;
    if (phi < 0.0) phi = phi + R2P;
    sinp = std::sin(phi);
    cosp = std::cos(phi);
  }
  // initpout.f90:1-68 with rep_isrf.f90: a point on the outer sphere
  // (uniform cosb and longitude), an inward direction with cos = -xi in the
  // local frame, rotated by initp_transform; the frequency from the ISRF cdf
  // table, interpolated linearly in log10(cdf) and log10(nu).
  void initpout() {
    sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
    double xran = ran();
    cosb = 1.0 - 2.0 * xran;
    sinb = std::sqrt(1.0 - cosb * cosb);
    xran = ran();
    cost = -xran;
    sint = std::sqrt(1.0 - cost * cost);
    xran = ran();
    phi = R2P * xran;
    cosp = std::cos(phi);
    sinp = std::sin(phi);
    xran = ran();
    lp = R2P * xran;
    initp_transform();
    xran = ran();
    const int n = m->t->nisrf;
    const double* cdf = m->t->isrf;
    const double* lcdf = cdf + n;
    const double* lfrq = cdf + 2 * n;
    int ifreq = locate(cdf, n, xran);
    if (ifreq == n) ifreq = n - 1;
    if (ifreq == 0) ifreq = 1;
    const double logfreq = lfrq[ifreq - 1] + (std::log10(xran) - lcdf[ifreq - 1]) / (lcdf[ifreq] - lcdf[ifreq - 1]) *
                                                 (lfrq[ifreq] - lfrq[ifreq - 1]);
    nub = std::pow(10.0, logfreq);
  }

  void initpspot(int ispotph) {    // initpspot.f90:3-175
    const mcrt_config& c = m->c;
    sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
    for (;;) {                     // label 100
      for (;;) {
        double xr = ran();
        cosb = 1.0 - 2.0 * xr;
        sinb = std::sqrt(1.0 - cosb * cosb);
        if (cosb != 0.0 && std::fabs(cosb) < 1.0) break;
      }
      lp = R2P * ran();
      double cphi = std::cos(lp), sphi = std::sin(lp);
      double sthet = sinb, cthet = cosb;
      if (c.ispot == 1) {
        double dotsp1 = c.scspot1 * sthet * cphi + c.ssspot1 * sthet * sphi + c.cspot1 * cthet;
        double dotsp2 = c.scspot2 * sthet * cphi + c.ssspot2 * sthet * sphi + c.cspot2 * cthet;
        if (c.nspot == 1) {
          if (ispotph == 1 && dotsp1 < c.csprad) continue;
        } else {
          if (ispotph == 1 && dotsp1 < c.csprad && dotsp2 < c.csprad) continue;
        }
        if (c.fspot < 1.0) {
          double dellon = (lp < PI) ? lp : R2P - lp;
          double costhp = c.cspot1 * cosb + c.sspot1 * sinb * std::cos(dellon);
          if (costhp > c.csprad) ispotph = 1;
          if (c.nspot == 2) {
            dellon = (lp < PI) ? PI - lp : lp - PI;
            costhp = c.cspot2 * cosb + c.sspot2 * sinb * std::cos(dellon);
            if (costhp > c.csprad) ispotph = 1;
          }
        }
      }
      break;
    }
    initp_sample();
    initp_transform();
    if (c.fspot == 1.0) {
      nub = (c.iplanckst == 0) ? atmosfreq() : bbfreq(c.tshock);
    } else if (ispotph == 0) {
      nub = (c.iplanckst == 0) ? atmosfreq() : bbfreq(c.tstar);
    } else {
      nub = bbfreq(c.tshock);
    }
  }
  void initp_ps(int ispotph) {     // initp_common.f90 / initp_ps: point source
    const mcrt_config& c = m->c;
    sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
    for (;;) {
      double xr = ran();
      cosb = check(1.0 - 2.0 * xr);
      sinb = check(std::sqrt(1.0 - cosb * cosb));
      if (cosb != 0.0) break;
    }
    cost = cosb;
    sint = sinb;
    lp = R2P * ran();
    phi = lp;
    sinp = check(std::sin(phi));
    cosp = check(std::cos(phi));
    if (ispotph == 0) nub = (c.iplanckst == 0) ? atmosfreq() : bbfreq(c.tstar);
    else nub = bbfreq(c.tshock);
  }
  void initpabs() {                // initpabs.f90:1-44
    sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
    cosb = zp / rtot;
    sinb = std::sqrt(1.0 - cosb * cosb);
    lp = std::atan2(yp, xp);
    initp_sample();
    initp_transform();
    ux = sint * cosp;
    uy = sint * sinp;
    uz = cost;
    nub = atmosfreq();
  }

  // ------------------------------------------------------------- grid
  // testgrid.f90:1-128
  void testgrid(double& x, double& y, double& z, double& rs, double& rt, int& ir, int& it, int& ip, bool& onw) {
    const int nrg = m->nrg, ntg = m->ntg, npg = m->npg;
    const double tol = 1.0e-4;
    double cb = check(z / rt);
    double ph = std::atan2(y, x);
    if (ph < 0.0) ph = ph + R2P;
    bool reset = false;
    const double* r2 = m->r2arr.data();
    const double* ca = m->costarr.data();
    const double* pa = m->phiarr.data();
    if ((rs - r2[0]) / (r2[1] - r2[0]) < -tol || (rs - r2[nrg - 2]) / (r2[nrg - 1] - r2[nrg - 2]) > 1.0 + tol) {
      const double third = (double)(1.0f / 3.0f);
      double r1 = m->rarr[0], rn = m->rarr[nrg - 1];
      rt = std::pow(ran() * (std::pow(rn, 3.0) - std::pow(r1, 3.0)) + std::pow(r1, 3.0), third);
      reset = true;
    }
    if ((cb - ca[0]) / (ca[1] - ca[0]) < -tol || (cb - ca[ntg - 2]) / (ca[ntg - 1] - ca[ntg - 2]) > 1.0 + tol) {
      cb = ran() * (ca[ntg - 1] - ca[0]) + ca[0];
      reset = true;
    }
    if ((ph - pa[0]) / (pa[1] - pa[0]) < -tol || (ph - pa[npg - 2]) / (pa[npg - 1] - pa[npg - 2]) > 1.0 + tol) {
      ph = ran() * (pa[npg - 1] - pa[0]) + pa[0];
      reset = true;
    }
    if (reset) {
      double s = std::sqrt(1.0 - cb * cb);
      x = rt * s * std::cos(ph);
      y = rt * s * std::sin(ph);
      z = rt * cb;
      rs = rt * rt;
      onw = false;
      T->cnt[MCRT_C_RESETS]++;
    }
    if (ir < 1 || ir > nrg) ir = locate(r2, nrg, rs);
    if (it < 1 || it > ntg) it = locate(ca, ntg, cb);
    if (ip < 1 || ip > npg) ip = locate(pa, npg, ph);
    double rfrac = (rs - r2[ir - 1]) / (r2[ir] - r2[ir - 1]);
    double tfrac = (cb - ca[it - 1]) / (ca[it] - ca[it - 1]);
    double pfrac = (ph - pa[ip - 1]) / (pa[ip] - pa[ip - 1]);
    bool phierr = false;
    if (pfrac < -tol || pfrac > 1.0 + tol) {
      double d1 = ph - pa[ip - 1];
      if (d1 > PI) d1 -= R2P;
      if (d1 < -PI) d1 += R2P;
      double d2 = ph - pa[ip];
      if (d2 > PI) d2 -= R2P;
      if (d2 < -PI) d2 += R2P;
      phierr = std::fabs(d1) > tol && std::fabs(d2) > tol;
    }
    if (rfrac < -tol || rfrac > 1.0 + tol) ir = locate(r2, nrg, rs);
    if (tfrac < -tol || tfrac > 1.0 + tol) it = locate(ca, ntg, cb);
    if (phierr) ip = locate(pa, npg, ph);
  }

  // radface/thetaface/phiface into the wall selector
  void faces(Walls& w, double vx, double vy, double vz, double x, double y, double z, int ir, int it, int ip) const {
    // radface.f90
    double bb = 2.0 * (x * vx + y * vy + vz * z);
    double cc = x * x + y * y + z * z - m->r2arr[ir - 1];
    double descr = bb * bb - 4.0 * cc;
    if (descr > 0.0) {
      descr = std::sqrt(descr);
      w.insert((-bb + descr) * 0.5, 1);
      w.insert((-bb - descr) * 0.5, 1);
    }
    cc = x * x + y * y + z * z - m->r2arr[ir];
    descr = bb * bb - 4.0 * cc;
    if (descr > 0.0) {
      descr = std::sqrt(descr);
      w.insert((-bb + descr) * 0.5, 2);
      w.insert((-bb - descr) * 0.5, 2);
    }
    // thetaface.f90
    if (m->ntg > 2) {
      double t1 = m->tan2arr[it - 1], t2 = m->tan2arr[it];
      double tmp1 = x * vx + y * vy, tmp2 = vx * vx + vy * vy, tmp3 = x * x + y * y;
      double ta, tb;
      int i1, i2;
      if (t2 < t1) { ta = t2; tb = t1; i1 = 4; i2 = 3; }
      else { ta = t1; tb = t2; i1 = 3; i2 = 4; }
      if (ta < 0.0) {
        if (vz != 0.0) w.insert(-z / vz, i1);
      } else {
        double b2 = 2.0 * (tmp1 - ta * vz * z);
        double aa = tmp2 - ta * vz * vz;
        double c2 = tmp3 - z * z * ta;
        if (std::fabs(aa) > 1.0e-10) {
          double d = b2 * b2 - 4.0 * aa * c2;
          if (d > 0.0 && ta != 0.0) {
            d = std::sqrt(d);
            w.insert((-b2 + d) * 0.5 / aa, i1);
            w.insert((-b2 - d) * 0.5 / aa, i1);
          }
        } else {
          if (std::fabs(b2) > 1.0e-10) w.insert(-c2 / b2, i1);
        }
      }
      double b2 = 2.0 * (tmp1 - tb * vz * z);
      double aa = tmp2 - tb * vz * vz;
      double c2 = tmp3 - z * z * tb;
      if (std::fabs(aa) > 1.0e-10) {
        double d = b2 * b2 - 4.0 * aa * c2;
        if (d > 0.0 && tb != 0.0) {
          d = std::sqrt(d);
          w.insert((-b2 + d) * 0.5 / aa, i2);
          w.insert((-b2 - d) * 0.5 / aa, i2);
        }
      } else {
        if (std::fabs(b2) > 1.0e-10) w.insert(-c2 / b2, i2);
      }
    }
    // phiface.f90 (C=D=0 planes through the z axis)
    if (m->npg > 2 && m->ntg > 2) {
      double A1 = m->aarr[ip - 1], B1 = m->barr[ip - 1], A2 = m->aarr[ip], B2 = m->barr[ip];
      double d1 = (A1 * vx + B1 * vy + 0.0 * vz);
      if (d1 != 0.0) w.insert(-(A1 * x + B1 * y + 0.0 * z + 0.0) / d1, 5);
      double d2 = (A2 * vx + B2 * vy + 0.0 * vz);
      if (d2 != 0.0) w.insert(-(A2 * x + B2 * y + 0.0 * z + 0.0) / d2, 6);
    }
  }

  double cell_opac(int ir, int it, int ip) const {     // tauint_3d_2_fuv.f90:59-65
    double opac = 0.0;
    for (int id = 1; id <= MCRT_NDG2; ++id) {
      double d = m->dens(ir, it, ip, id);
      if (d > 0.0) opac = opac + kapd[m->fopac(ir, it, ip, id) - 1] * d;
    }
    return opac;
  }

  void tally_abs(int ir, int it, int ip, double len) {   // tauint_3d_2_fuv.f90:83-98, 122-144
    int64_t c = m->cidx(ir, it, ip);
    if (adj && adj->replay && adj->W() != 0.0) {
      for (int id = 1; id <= MCRT_NDG2; ++id) {
        const double d = m->dens(ir, it, ip, id);
        if (d > 0.0) (*adj->grad)[c + m->ncell * (id - 1)] -= adj->W() * (kapd[m->fopac(ir, it, ip, id) - 1] * d * len);
      }
    }
    for (int id = 1; id <= MCRT_NDG2; ++id) {
      double d = m->dens(ir, it, ip, id);
      if (!m->is_sg[id - 1] && d > 0.0) {
        int id2 = m->fopac(ir, it, ip, id) - 1;
        T->dtauabs[c] = T->dtauabs[c] + len * kapd[id2] * d * (1.0 - albedo[id2]);
      }
    }
    if (m->c.iffuv) T->fuvmean[c] = T->fuvmean[c] + len * (m->c.rstar * RSOL) * ifuv / m->g->vcell[c];
  }

  // tauint_3d_2_fuv.f90:5-210; returns false on a geometry failure
  bool tauint(int& ir, int& it, int& ip) {
    const int nrg = m->nrg, npg = m->npg;
    double tsum = 0.0;
    for (;;) {
      testgrid(xp, yp, zp, rsq, rtot, ir, it, ip, on_wall);
      Walls w;
      w.reset();
      faces(w, ux, uy, uz, xp, yp, zp, ir, it, ip);
      double dt;
      int iface;
      w.next(on_wall, dt, iface);
      if (dt < 0.0 || dt == HUGE_D || iface < 1 || iface > 6) return false;
      double opac = cell_opac(ir, it, ip);
      double dtau = opac * dt;
      if (tsum + dtau > tau) {
        double ds = (tau - tsum) / opac;
        tally_abs(ir, it, ip, ds);
        xp = xp + ds * ux;
        yp = yp + ds * uy;
        zp = zp + ds * uz;
        rsq = xp * xp + yp * yp + zp * zp;
        rtot = std::sqrt(rsq);
        on_wall = false;
        return true;
      }
      tally_abs(ir, it, ip, dt);
      switch (iface) {
        case 1: ir = ir - 1; break;
        case 2: ir = ir + 1; break;
        case 3: it = it - 1; break;
        case 4: it = it + 1; break;
        case 5: ip = ip - 1; break;
        case 6: ip = ip + 1; break;
      }
      if (ip == 0) ip = npg - 1;
      if (ip == npg) ip = 1;
      xp = xp + dt * ux;
      yp = yp + dt * uy;
      zp = zp + dt * uz;
      on_wall = true;
      rsq = xp * xp + yp * yp + zp * zp;
      rtot = std::sqrt(rsq);
      tsum = tsum + dtau;
      ++ncross;
      T->cnt[MCRT_C_CROSSINGS]++;
      if (ir == nrg) { exitflag = 1; return true; }
      if (ir == 0) {
        T->scal[MCRT_S_AFLUX] += 1.0;
        ++nstar;
        T->cnt[MCRT_C_STARHITS]++;
        rtot = std::sqrt(rsq);
        initpabs();
        opacset(nub);
        ifuv = is_fuv(nub) ? m->c.ifuv_ori : 0.0;
        i_orig = 1;
        iflag = 0;
        kapd_tauint();
        ir = 1;
        tsum = 0.0;
      }
      if (ncross > 200000000) return false;   // watchdog
    }
  }

  // --------------------------------------------- tabulated scattering
  // stokes6.f90 / stokespeel6.f90 with the tables of tab_mod.f90 per species
  // and wavelength node (the reference keeps one table, reatab.f90, and its
  // stokes6 indexes s11arr(narr,4) with one subscript, so it does not
  // compile; this restatement and the engine share one definition):
  //   row      = species x wavelength node a of opacset's bracket, weight f
  //              of node a-1 (the interpolation of kappa, albedo, g);
  //   itab     = int((1+bmu)/dct)+1 within 1..narr (stokes6.f90:62);
  //   rejection bound = max over the row of S11+|S12| (max of the two rows
  //              when interpolating), which bounds the sampling probability
  //              for any polarisation; stokes6's running `peak` is not kept.
  void mueller_row(double nu, int id, int& row, double& f) const {
    const mcrt_tables* t = m->t;
    const int nl = m->c.nlammax;
    const double* nud = t->nudust + (int64_t)nl * id;
    const int n = t->nlambda[id];
    int a;
    if (nu >= nud[0]) { a = 0; f = 0.0; }
    else if (nu <= nud[n - 1]) { a = n - 1; f = 0.0; }
    else {
      int i0 = 1, i1 = n;
      while (i1 - i0 > 1) {
        int i = (i1 + i0) / 2;
        if (nu <= nud[i - 1]) i0 = i; else i1 = i;
      }
      a = i1 - 1;
      const int b = i0 - 1;
      f = (nu - nud[a]) / (nud[b] - nud[a]);
    }
    row = a + nl * id;
  }
  double mueller_el(int row, double f, int itab, int k) const {
    const double* tab = m->t->mueller;
    const int narr = m->t->narr;
    const double va = tab[6 * ((int64_t)(itab - 1) + (int64_t)narr * row) + k];
    if (f == 0.0) return va;
    const double vb = tab[6 * ((int64_t)(itab - 1) + (int64_t)narr * (row - 1)) + k];
    return (1.0 - f) * va + f * vb;
  }
  int mueller_bin(double bmu) const {
    const int narr = m->t->narr;
    return std::min(std::max((int)((1.0 + bmu) / (2.0 / (double)narr)) + 1, 1), narr);
  }
  double mueller_peak(int row, double f) const {
    auto rowpeak = [&](int r) {
      double pk = 0.0;
      const double* tab = m->t->mueller;
      for (int i = 0; i < m->t->narr; ++i) {
        const double* e = tab + 6 * ((int64_t)i + (int64_t)m->t->narr * r);
        pk = std::max(pk, e[0] + std::fabs(e[1]));
      }
      return pk;
    };
    return f == 0.0 ? rowpeak(row) : std::max(rowpeak(row), rowpeak(row - 1));
  }
  // stokes6.f90:174-201 (i1 > pi) and :286-306 (i1 < pi)
  void mueller6(int row, double f, int itab, bool upper, double s11, double s12, double c2i, double s2i,
                double sini2, double cosi2, double* A) const {
    const double sin2i2 = 2.0 * sini2 * cosi2, cos2i2 = 2.0 * cosi2 * cosi2 - 1.0;
    const double sin2 = sin2i2 * s2i, cos2 = cos2i2 * c2i;
    const double sin2cos1 = sin2i2 * c2i, cos2sin1 = cos2i2 * s2i;
    const double s22 = mueller_el(row, f, itab, 2), s33 = mueller_el(row, f, itab, 3);
    const double s34 = mueller_el(row, f, itab, 4), s44 = mueller_el(row, f, itab, 5);
    // A: a11 a12 a13 a21 a22 a23 a24 a31 a32 a33 a34 a42 a43 a44
    A[0] = s11; A[1] = s12 * c2i; A[3] = s12 * cos2i2;
    A[4] = s22 * cos2 - s33 * sin2;
    A[9] = -s22 * sin2 + s33 * cos2;
    A[10] = s34 * cos2i2;
    A[12] = -s34 * c2i;
    A[13] = s44;
    if (upper) {
      A[2] = s12 * s2i; A[5] = s22 * cos2sin1 + s33 * sin2cos1; A[6] = s34 * sin2i2;
      A[7] = -s12 * sin2i2; A[8] = -s22 * sin2cos1 - s33 * cos2sin1; A[11] = s34 * s2i;
    } else {
      A[2] = -s12 * s2i; A[5] = -s22 * cos2sin1 - s33 * sin2cos1; A[6] = -s34 * sin2i2;
      A[7] = s12 * sin2i2; A[8] = s22 * sin2cos1 + s33 * cos2sin1; A[11] = -s34 * s2i;
    }
  }
  void stokes6(int id) {          // stokes6.f90:1-336, id 0-based species
    int row;
    double f;
    mueller_row(nub, id, row, f);
    const double peak = mueller_peak(row, f);
    const double costp = cost, sintp = sint, phip = phi;
    double bmu, s11, s12, sinbt, a, ci, si_, c2i, s2i;
    int itab;
    bool upper;
    for (;;) {
      bmu = 1.0 - 2.0 * ran();
      itab = mueller_bin(bmu);
      s11 = mueller_el(row, f, itab, 0);
      s12 = mueller_el(row, f, itab, 1);
      const double cosb2 = bmu * bmu;
      sinbt = std::sqrt(1.0 - cosb2);
      const double ri1 = R2P * ran();
      upper = ri1 > PI;
      const double ang = upper ? R2P - ri1 : ri1;
      ci = std::cos(ang);
      si_ = std::sin(ang);
      s2i = 2.0 * si_ * ci;
      c2i = 2.0 * ci * ci - 1.0;
      const double a12 = s12 * c2i;
      const double a13 = upper ? s12 * s2i : -s12 * s2i;
      const double rprob = (s11 * sip + a12 * sqp + a13 * sup) / sip;
      if (peak * ran() > rprob) continue;
      a = rprob;
      break;
    }
    if (bmu == 1.0) return;
    double sini2, cosi2 = 0.0;
    if (bmu == -1.0) {
      si_ = 1.0; sini2 = 1.0; ci = 0.0; cosi2 = 0.0;
      cost = -costp; sint = sintp;
    } else {
      cost = costp * bmu + sintp * sinbt * ci;
      if (std::fabs(cost) < 1.0) {
        sint = std::fabs(std::sqrt(1.0 - cost * cost));
        sini2 = si_ * sintp / sint;
        const double bott = sint * sinbt;
        cosi2 = costp / bott - cost * bmu / bott;
      } else {
        sint = 0.0; sini2 = 0.0;
        if (cost >= 1.0) { cosi2 = -1.0; cost = 1.0; }
        if (cost <= -1.0) { cosi2 = 1.0; cost = -1.0; }
      }
    }
    double cosdph = -cosi2 * ci + sini2 * si_ * bmu;
    if (std::fabs(cosdph) > 1.0) cosdph = (cosdph > 1.0) ? 1.0 : -1.0;
    phi = upper ? phip + std::acos(cosdph) : phip - std::acos(cosdph);
    if (phi > R2P) phi = phi - R2P;
    if (phi < 0.0) phi = phi + R2P;
    double A[14];
    mueller6(row, f, itab, upper, s11, s12, c2i, s2i, sini2, cosi2, A);
    const double nsi = (A[0] * sip + A[1] * sqp + A[2] * sup) / a;
    const double nsq = (A[3] * sip + A[4] * sqp + A[5] * sup + A[6] * svp) / a;
    const double nsu = (A[7] * sip + A[8] * sqp + A[9] * sup + A[10] * svp) / a;
    const double nsv = (A[11] * sqp + A[12] * sup + A[13] * svp) / a;
    sip = nsi; sqp = nsq; sup = nsu; svp = nsv;
    cosp = std::cos(phi);
    sinp = std::sin(phi);
  }
  void stokespeel6(double& s_i, double& s_q, double& s_u, double& s_v, double cst, double snt, double ri1,
                   double bmu, double costp, double sintp, int id) const {   // stokespeel6.f90:1-321
    int row;
    double f;
    mueller_row(nub, id, row, f);
    const int itab = mueller_bin(bmu);
    const double s11 = mueller_el(row, f, itab, 0), s12 = mueller_el(row, f, itab, 1);
    const double cosb2 = bmu * bmu;
    const double sinbt = std::sqrt(1.0 - cosb2);
    const bool upper = ri1 > PI;
    const double ang = upper ? R2P - ri1 : ri1;
    double ci = std::cos(ang), si_ = std::sin(ang);
    const double s2i = 2.0 * si_ * ci, c2i = 2.0 * ci * ci - 1.0;
    if (bmu == 1.0) return;
    double sini2, cosi2 = 0.0;
    if (bmu == -1.0) { si_ = 1.0; sini2 = 1.0; ci = 0.0; cosi2 = 0.0; }
    else if (std::fabs(cst) < 1.0) {
      sini2 = si_ * sintp / snt;
      const double bott = snt * sinbt;
      cosi2 = costp / bott - cst * bmu / bott;
    } else {
      sini2 = 0.0;
      if (cst >= 1.0) cosi2 = -1.0;
      if (cst <= -1.0) cosi2 = 1.0;
    }
    double A[14];
    mueller6(row, f, itab, upper, s11, s12, c2i, s2i, sini2, cosi2, A);
    const double ni = (A[0] * s_i + A[1] * s_q + A[2] * s_u);
    const double nq = (A[3] * s_i + A[4] * s_q + A[5] * s_u + A[6] * s_v);
    const double nu_ = (A[7] * s_i + A[8] * s_q + A[9] * s_u + A[10] * s_v);
    const double nv = (A[11] * s_q + A[12] * s_u + A[13] * s_v);
    s_i = ni; s_q = nq; s_u = nu_; s_v = nv;
  }
  void scatter(int id) { if (m->t->mueller && m->t->narr > 0) stokes6(id); else stokes(id); }
  void peel_matrix(double& s_i, double& s_q, double& s_u, double& s_v, double cst, double snt, double ri1,
                   double bmu, double costp, double sintp, int id) const {
    if (m->t->mueller && m->t->narr > 0) stokespeel6(s_i, s_q, s_u, s_v, cst, snt, ri1, bmu, costp, sintp, id);
    else stokespeel(s_i, s_q, s_u, s_v, cst, snt, ri1, bmu, costp, sintp, id);
  }

  // ---------------------------------------------------------- scattering
  void dustmat(double bmu, double cosb2, int id, double& p1, double& p2, double& p3, double& p4) const {
    // dustmat.f90:343-412
    double temp = g2p1[id] - twog[id] * bmu;
    p1 = 1.5 * onemg2[id] / (2.0 + g2[id]) * (1.0 + cosb2) / (temp * std::sqrt(temp));
    p2 = -pl[id] * p1 * (1.0 - cosb2) / (1.0 + cosb2);
    p3 = p1 * 2.0 * bmu / (1.0 + cosb2);
    p4 = 0.0;
  }
  double peak_of(int id) const {   // stokes.f90:54-70
    double temp;
    if (g[id] > 0.0) temp = g2p1[id] - twog[id];
    else temp = g2p1[id] + twog[id];
    double pk = 1.5 * (onemg2[id]) / (2.0 + g2[id]) * 2.0 / temp / std::sqrt(temp);
    return pk * 1.01;
  }

  void stokes(int id) {            // stokes.f90:1-340, id 0-based species
    const double costp = cost, sintp = sint, phip = phi;
    double peak = peak_of(id);
    double bmu, cosb2, sinbt, p1, p2, p3, p4;
    double a11, a12, a13, a21, a22, a23, a24, a31, a32, a33, a34, a42, a43, a44, a, rprob;
    for (;;) {
      double xr = ran();
      bmu = 1.0 - 2.0 * xr;
      cosb2 = bmu * bmu;
      double b = cosb2 - 1.0;
      if (m->c.idust == 0) {
        p1 = 0.75 * (1.0 + cosb2); p2 = 0.75 * b * 1.0; p3 = 0.75 * (2.0 * bmu); p4 = 0.0;
        peak = 1.501;
      } else {
        dustmat(bmu, cosb2, id, p1, p2, p3, p4);
      }
      sinbt = std::sqrt(1.0 - cosb2);
      double ri1 = R2P * ran();
      if (ri1 > PI) {
        double ri3 = R2P - ri1;
        double cosi3 = std::cos(ri3), sini3 = std::sin(ri3);
        double sin2i3 = 2.0 * sini3 * cosi3, cos2i3 = 2.0 * cosi3 * cosi3 - 1.0;
        a11 = p1; a12 = p2 * cos2i3; a13 = p2 * sin2i3;
        rprob = (a11 * sip + a12 * sqp + a13 * sup) / sip;
        if (rprob > peak) peak = rprob;
        double xr2 = ran();
        if (peak * xr2 > rprob) continue;
        a = rprob;
        double sini2, cosi2 = 0.0;
        if (bmu == 1.0) return;
        else if (bmu == -1.0) {
          sini3 = 1.0; sini2 = 1.0; cosi3 = 0.0; cosi2 = 0.0;
          cost = -costp; sint = sintp;
        } else {
          cost = costp * bmu + sintp * sinbt * cosi3;
          if (std::fabs(cost) < 1.0) {
            sint = std::fabs(std::sqrt(1.0 - cost * cost));
            sini2 = sini3 * sintp / sint;
            double bott = sint * sinbt;
            cosi2 = costp / bott - cost * bmu / bott;
          } else {
            sint = 0.0; sini2 = 0.0;
            if (cost >= 1.0) cosi2 = -1.0;
            if (cost <= -1.0) cosi2 = 1.0;
          }
        }
        double cosdph = -cosi2 * cosi3 + sini2 * sini3 * bmu;
        if (std::fabs(cosdph) > 1.0) cosdph = (cosdph > 1.0) ? 1.0 : -1.0;
        phi = phip + std::acos(cosdph);
        if (phi > R2P) phi = phi - R2P;
        if (phi < 0.0) phi = phi + R2P;
        double sin2i2 = 2.0 * sini2 * cosi2, cos2i2 = 2.0 * cosi2 * cosi2 - 1.0;
        double sin2 = sin2i2 * sin2i3, cos2 = cos2i2 * cos2i3;
        double sin2cos1 = sin2i2 * cos2i3, cos2sin1 = cos2i2 * sin2i3;
        a21 = p2 * cos2i2; a22 = p1 * cos2 - p3 * sin2; a23 = p1 * cos2sin1 + p3 * sin2cos1; a24 = -p4 * sin2i2;
        a31 = -p2 * sin2i2; a32 = -p1 * sin2cos1 - p3 * cos2sin1; a33 = -p1 * sin2 + p3 * cos2; a34 = -p4 * cos2i2;
        a42 = -p4 * sin2i3; a43 = p4 * cos2i3; a44 = p3;
      } else {
        double cosi1 = std::cos(ri1), sini1 = std::sin(ri1);
        double sin2i1 = 2.0 * sini1 * cosi1, cos2i1 = 2.0 * cosi1 * cosi1 - 1.0;
        a11 = p1; a12 = p2 * cos2i1; a13 = -p2 * sin2i1;
        rprob = (a11 * sip + a12 * sqp + a13 * sup) / sip;
        if (rprob > peak) peak = rprob;
        double xr2 = ran();
        if (peak * xr2 > rprob) continue;
        a = rprob;
        double sini2, cosi2 = 0.0;
        if (bmu == 1.0) return;
        else if (bmu == -1.0) {
          sini1 = 1.0; sini2 = 1.0; cosi1 = 0.0; cosi2 = 0.0;
          cost = -costp; sint = sintp;
        } else {
          cost = costp * bmu + sintp * sinbt * cosi1;
          if (std::fabs(cost) < 1.0) {
            sint = std::fabs(std::sqrt(1.0 - cost * cost));
            sini2 = sini1 * sintp / sint;
            double bott = sint * sinbt;
            cosi2 = costp / bott - cost * bmu / bott;
          } else {
            sint = 0.0; sini2 = 0.0;
            if (cost >= 1.0) cosi2 = -1.0;
            if (cost <= -1.0) cosi2 = 1.0;
          }
        }
        double cosdph = -cosi1 * cosi2 + sini1 * sini2 * bmu;
        if (std::fabs(cosdph) > 1.0) cosdph = (cosdph > 1.0) ? 1.0 : -1.0;
        phi = phip - std::acos(cosdph);
        if (phi > R2P) phi = phi - R2P;
        if (phi < 0.0) phi = phi + R2P;
        double sin2i2 = 2.0 * sini2 * cosi2, cos2i2 = 2.0 * cosi2 * cosi2 - 1.0;
        double sin2 = sin2i2 * sin2i1, cos2 = cos2i2 * cos2i1;
        double sin2cos1 = sin2i2 * cos2i1, cos2sin1 = cos2i2 * sin2i1;
        a21 = p2 * cos2i2; a22 = p1 * cos2 - p3 * sin2; a23 = -p1 * cos2sin1 - p3 * sin2cos1; a24 = p4 * sin2i2;
        a31 = p2 * sin2i2; a32 = p1 * sin2cos1 + p3 * cos2sin1; a33 = -p1 * sin2 + p3 * cos2; a34 = -p4 * cos2i2;
        a42 = p4 * sin2i1; a43 = p4 * cos2i1; a44 = p3;
      }
      break;
    }
    double si = (a11 * sip + a12 * sqp + a13 * sup) / a;
    double sq = (a21 * sip + a22 * sqp + a23 * sup + a24 * svp) / a;
    double su = (a31 * sip + a32 * sqp + a33 * sup + a34 * svp) / a;
    double sv = (a42 * sqp + a43 * sup + a44 * svp) / a;
    sip = si; sqp = sq; sup = su; svp = sv;
    cosp = std::cos(phi);
    sinp = std::sin(phi);
  }

  // ----------------------------------------------------------- peel-off
  // findangle3.f90 with phi2 = phie = 0 (reapar_4_test1.f90:425)
  static void findangle3(double cost1, double sint1, double phi1, double cosp1, double sinp1, double cost2,
                         double sint2, double phi2, double cosp2, double sinp2, double& costnew,
                         double& sintnew, double& ri1) {
    costnew = cost1 * cost2 + (sint1 * sint2 * (cosp1 * cosp2 + sinp1 * sinp2));
    costnew = check(costnew);
    sintnew = std::sqrt(1.0 - costnew * costnew);
    ri1 = 0.0;
    if (sint1 > 1.0e-8) {
      if (sintnew > 1.0e-8) {
        double cosx = (cost2 - (cost1 * costnew)) / (sint1 * sintnew);
        cosx = check(cosx);
        double x = std::acos(cosx);
        if (phi2 > phi1) {
          double diff = phi2 - phi1;
          ri1 = (diff > PI) ? x : R2P - x;
        } else {
          double diff = phi1 - phi2;
          ri1 = (diff > PI) ? R2P - x : x;
        }
      }
    }
  }

  // stokespeel.f90:1-328 (rotate+multiply without normalisation)
  void stokespeel(double& s_i, double& s_q, double& s_u, double& s_v, double cost_e, double sint_e, double ri1,
                  double bmu, double costp, double sintp, int id) const {
    double p1, p2, p3, p4;
    double cosb2 = bmu * bmu;
    double b = cosb2 - 1.0;
    if (m->c.idust == 0) {
      p1 = 0.75 * (1.0 + cosb2); p2 = 0.75 * b * 1.0; p3 = 0.75 * (2.0 * bmu); p4 = 0.0;
    } else {
      dustmat(bmu, cosb2, id, p1, p2, p3, p4);
    }
    double sinbt = std::sqrt(1.0 - cosb2);
    double a11, a12, a13, a21, a22, a23, a24, a31, a32, a33, a34, a42, a43, a44;
    double cost = cost_e, sint = sint_e;
    if (ri1 > PI) {
      double ri3 = R2P - ri1;
      double cosi3 = std::cos(ri3), sini3 = std::sin(ri3);
      double sin2i3 = 2.0 * sini3 * cosi3, cos2i3 = 2.0 * cosi3 * cosi3 - 1.0;
      a11 = p1; a12 = p2 * cos2i3; a13 = p2 * sin2i3;
      double sini2, cosi2 = 0.0;
      if (bmu == 1.0) return;
      else if (bmu == -1.0) { sini3 = 1.0; sini2 = 1.0; cosi3 = 0.0; cosi2 = 0.0; }
      else {
        if (std::fabs(cost) < 1.0) {
          sini2 = sini3 * sintp / sint;
          double bott = sint * sinbt;
          cosi2 = costp / bott - cost * bmu / bott;
        } else {
          sint = 0.0; sini2 = 0.0;
          if (cost >= 1.0) cosi2 = -1.0;
          if (cost <= -1.0) cosi2 = 1.0;
        }
      }
      double sin2i2 = 2.0 * sini2 * cosi2, cos2i2 = 2.0 * cosi2 * cosi2 - 1.0;
      double sin2 = sin2i2 * sin2i3, cos2 = cos2i2 * cos2i3;
      double sin2cos1 = sin2i2 * cos2i3, cos2sin1 = cos2i2 * sin2i3;
      a21 = p2 * cos2i2; a22 = p1 * cos2 - p3 * sin2; a23 = p1 * cos2sin1 + p3 * sin2cos1; a24 = -p4 * sin2i2;
      a31 = -p2 * sin2i2; a32 = -p1 * sin2cos1 - p3 * cos2sin1; a33 = -p1 * sin2 + p3 * cos2; a34 = -p4 * cos2i2;
      a42 = -p4 * sin2i3; a43 = p4 * cos2i3; a44 = p3;
    } else {
      double cosi1 = std::cos(ri1), sini1 = std::sin(ri1);
      double sin2i1 = 2.0 * sini1 * cosi1, cos2i1 = 2.0 * cosi1 * cosi1 - 1.0;
      a11 = p1; a12 = p2 * cos2i1; a13 = -p2 * sin2i1;
      double sini2, cosi2 = 0.0;
      if (bmu == 1.0) return;
      else if (bmu == -1.0) { sini1 = 1.0; sini2 = 1.0; cosi1 = 0.0; cosi2 = 0.0; }
      else {
        if (std::fabs(cost) < 1.0) {
          sini2 = sini1 * sintp / sint;
          double bott = sint * sinbt;
          cosi2 = costp / bott - cost * bmu / bott;
        } else {
          sini2 = 0.0;
          if (cost >= 1.0) cosi2 = -1.0;
          if (cost <= -1.0) cosi2 = 1.0;
        }
      }
      double sin2i2 = 2.0 * sini2 * cosi2, cos2i2 = 2.0 * cosi2 * cosi2 - 1.0;
      double sin2 = sin2i2 * sin2i1, cos2 = cos2i2 * cos2i1;
      double sin2cos1 = sin2i2 * cos2i1, cos2sin1 = cos2i2 * sin2i1;
      a21 = p2 * cos2i2; a22 = p1 * cos2 - p3 * sin2; a23 = -p1 * cos2sin1 - p3 * sin2cos1; a24 = p4 * sin2i2;
      a31 = p2 * sin2i2; a32 = p1 * sin2cos1 + p3 * cos2sin1; a33 = -p1 * sin2 + p3 * cos2; a34 = -p4 * cos2i2;
      a42 = p4 * sin2i1; a43 = p4 * cos2i1; a44 = p3;
    }
    double si = (a11 * s_i + a12 * s_q + a13 * s_u);
    double sq = (a21 * s_i + a22 * s_q + a23 * s_u + a24 * s_v);
    double su = (a31 * s_i + a32 * s_q + a33 * s_u + a34 * s_v);
    double sv = (a42 * s_q + a43 * s_u + a44 * s_v);
    s_i = si; s_q = sq; s_u = su; s_v = sv;
  }

  int freq_bin(double nu) const {  // propagate_5_fuv.f90:273, peeloff :289
    double v = (double)m->c.nfreq * std::log(nu / m->c.numin) / m->c.lnurat;
    int ib;
    if (!(v > -2.0e9)) ib = 0;
    else if (v > 2.0e9) ib = m->c.nfreq;
    else ib = (int)v + 1;
    return std::min(std::max(ib, 1), m->c.nfreq);
  }

  // peeloff_3d_2_test.f90:7-347
  void peeloff(double s_i, int ir, int it, int ip, int idust2, int peelid) {
    const mcrt_config& c = m->c;
    const mcrt_tables* t = m->t;
    const int nrg = m->nrg, npg = m->npg;
    T->cnt[MCRT_C_PEELS]++;
    bool onw = on_wall;
    double x1 = xp, y1 = yp, z1 = zp, rs1 = rsq, rt1 = rtot;
    double q_i = s_i, q_q = sqp, q_u = sup, q_v = svp;
    double tsum = 0.0;
    const double cospe = t->cospe_arr[peelid - 1], sinpe = t->sinpe_arr[peelid - 1];
    const double coste = t->coste_arr[peelid - 1], sinte = t->sinte_arr[peelid - 1];
    const double ux1 = sinte * cospe, uy1 = sinte * sinpe, uz1 = coste;
    // adjoint pass 1: the peel walk draws (testgrid re-locations) from a
    // copy of the stream, as the engine's peel-off kernel uses its own
    const Rng saved = rng;
    struct Restore { Packet* p; const Rng& r; bool on; ~Restore() { if (on) p->rng = r; } } restore{this, saved, adj != nullptr};
    if (adj) adj->cross.clear();
    if (onw) {
      bool inner = std::fabs(rs1 - m->r2arr[ir - 1]) < std::fabs(rs1 - m->r2arr[ir]);
      bool outwards = ux1 * x1 + uy1 * y1 + uz1 * z1 > 0.0;
      if (inner && !outwards) {
        if (ir == 1) return;
        ir = ir - 1;
      }
      if (!inner && outwards) ir = ir + 1;
    }
    int64_t steps = 0;
    for (;;) {
      testgrid(x1, y1, z1, rs1, rt1, ir, it, ip, onw);
      Walls w;
      w.reset();
      faces(w, ux1, uy1, uz1, x1, y1, z1, ir, it, ip);
      double dt;
      int iface;
      w.next(onw, dt, iface);
      if (dt == HUGE_D || iface < 1 || iface > 6) { T->cnt[MCRT_C_GEOM_FAIL]++; return; }
      double opac = cell_opac(ir, it, ip);
      tsum = tsum + opac * dt;
      if (adj) adj->cross.emplace_back(m->cidx(ir, it, ip), dt);
      if (tsum > 25.0) return;
      switch (iface) {
        case 1: ir = ir - 1; break;
        case 2: ir = ir + 1; break;
        case 3: it = it - 1; break;
        case 4: it = it + 1; break;
        case 5: ip = ip - 1; break;
        case 6: ip = ip + 1; break;
      }
      if (ip == 0) ip = npg - 1;
      if (ip == npg) ip = 1;
      x1 = x1 + dt * ux1;
      y1 = y1 + dt * uy1;
      z1 = z1 + dt * uz1;
      onw = true;
      rs1 = x1 * x1 + y1 * y1 + z1 * z1;
      rt1 = std::sqrt(rs1);
      T->cnt[MCRT_C_PEEL_CROSS]++;
      if (ir == nrg) break;
      if (ir == 0) return;
      if (++steps > 100000000) { T->cnt[MCRT_C_GEOM_FAIL]++; return; }
    }
    T->cnt[MCRT_C_PEEL_BINNED]++;
    double factor = std::exp(-tsum);
    q_i = q_i * factor; q_q = q_q * factor; q_u = q_u * factor; q_v = q_v * factor;
    if (iflag == 1) {
      double bmu, sinbm, ri1;
      findangle3(cost, sint, phi, cosp, sinp, coste, sinte, 0.0, cospe, sinpe, bmu, sinbm, ri1);
      peel_matrix(q_i, q_q, q_u, q_v, coste, sinte, ri1, bmu, cost, sint, m->fopac(ir, it, ip, idust2) - 1);
    }
    double yimage = z1 * sinte - y1 * coste * sinpe - x1 * coste * cospe;
    double ximage = y1 * cospe - x1 * sinpe;
    const double fractxh = 2.0 * c.rmaxi / (double)c.nxhst;
    double vx = (ximage + c.rmaxi) / fractxh, vy = (yimage + c.rmaxi) / fractxh;
    double rho2 = ximage * ximage + yimage * yimage;
    int inub = freq_bin(nub);
    int64_t img_k = -1;
    int64_t e_list[64];
    int ne = 0;
    if (c.output_imcube && vx > -1.0e9 && vx < 1.0e9 && vy > -1.0e9 && vy < 1.0e9) {
      int ix = (int)vx + 1, iy = (int)vy + 1;
      if (ix <= c.nxhst && iy <= c.nxhst && ix > 0 && iy > 0) {
        int64_t k = (int64_t)(peelid - 1) + (int64_t)c.npeel * ((ix - 1) + (int64_t)c.nxhst * ((iy - 1) + (int64_t)c.nxhst * (inub - 1)));
        img_k = k;
        atomic_add(I->im[0][k], q_i);
        atomic_add(I->im[1][k], q_q);
        atomic_add(I->im[2][k], q_u);
        atomic_add(I->im[3][k], q_v);
      }
    }
    // filter-band images (peeloff_3d_2_test.f90:242-285): freq = 2.9979e14/wave,
    // wave = 1.2398/nub; a filter whose open range (filtwave(1), filtwave(nf))
    // holds freq adds the Stokes vector times filtphi at the last point below
    // freq, found by the reference's linear scan; I also goes to the image of
    // the packet's origin (s star, d disk, e envelope, o outflow)
    if (c.output_imfilt && !I->imb[0].empty() && vx > -1.0e9 && vx < 1.0e9 && vy > -1.0e9 && vy < 1.0e9) {
      int ix = (int)vx + 1, iy = (int)vy + 1;
      if (ix <= c.nxhst && iy <= c.nxhst && ix > 0 && iy > 0) {
        const double wave = 1.2398 / nub;
        const double freq = 2.9979e14 / wave;
        for (int ifilt = 1; ifilt <= c.nfilt; ++ifilt) {
          const int nf = t->nwfilt[ifilt - 1] - 1;
          const double* fw = t->filtwave + (int64_t)c.nwfiltmax * (ifilt - 1);
          if (freq > fw[0] && freq < fw[nf - 1]) {
            int iw = 1;
            while (freq > fw[iw - 1]) iw = iw + 1;
            iw = iw - 1;
            const double wt = t->filtphi[(int64_t)c.nwfiltmax * (ifilt - 1) + iw - 1];
            const int64_t k = (int64_t)(peelid - 1) + (int64_t)c.npeel * ((ix - 1) + (int64_t)c.nxhst * ((iy - 1) + (int64_t)c.nxhst * (ifilt - 1)));
            atomic_add(I->imb[0][k], q_i * wt);
            atomic_add(I->imb[1][k], q_q * wt);
            atomic_add(I->imb[2][k], q_u * wt);
            atomic_add(I->imb[3][k], q_v * wt);
            const int oi = i_orig == 1 ? 5 : (i_orig == 2 ? 4 : (i_orig == 3 ? 6 : (i_orig == 4 ? 7 : -1)));
            if (oi >= 0) atomic_add(I->imb[oi][k], q_i * wt);
          }
        }
      }
    }
    // nested images (peeloff_3d_2_test.f90:302-309 -> nested_image_bin,
    // type_nested_image.f90:75-101): single-precision position and
    // log10(frequency); the level is the smallest whose half size exceeds
    // max(|x|,|y|); a pixel outside the image (only at a level's exact edge)
    // is dropped
    if (c.output_imsparse && !I->ims[0].empty()) {
      const float xr = (float)ximage, yr = (float)yimage;
      const float lnu = (float)std::log10(2.9979e14 / (1.2398 / nub));
      const float* lev = t->sparse_levels;
      const int nl = c.sparse_nlev;
      const float r = std::max(std::fabs(xr), std::fabs(yr));
      if (!(r > lev[nl - 1])) {
        int l = locate_sp(lev, nl, r);
        l = (l < 0) ? 1 : std::min(l + 1, nl);   // a single level met exactly at its edge stays that level
        const int ix = ipos_sp(-lev[l - 1], lev[l - 1], xr, c.sparse_dim);
        const int iy = ipos_sp(-lev[l - 1], lev[l - 1], yr, c.sparse_dim);
        const int inu = ipos_sp(c.sparse_lognu_min, c.sparse_lognu_max, lnu, c.sparse_nnu);
        if (inu >= 1 && inu <= c.sparse_nnu && ix >= 1 && ix <= c.sparse_dim && iy >= 1 && iy <= c.sparse_dim) {
          const int64_t k = (int64_t)(ix - 1) + (int64_t)c.sparse_dim * ((iy - 1) + (int64_t)c.sparse_dim *
                            ((inu - 1) + (int64_t)c.sparse_nnu * ((l - 1) + (int64_t)nl * (peelid - 1))));
          atomic_add(I->ims[0][k], q_i);
          atomic_add(I->ims[1][k], q_q);
          atomic_add(I->ims[2][k], q_u);
          atomic_add(I->ims[3][k], q_v);
        }
      }
    }
    int i_inter = (iflag == 1) ? 2 : ((i_orig == 1) ? 1 : 3);
    int indx[3] = {1, 1 + i_orig, 5 + i_inter};
    for (int ia = 1; ia <= c.nap; ++ia) {
      if (rho2 < t->aperture2[ia - 1]) {
        for (int k = 0; k < 3; ++k) {
          int64_t e = (inub - 1) + (int64_t)c.nfreq * ((peelid - 1) + (int64_t)c.npeel * ((ia - 1) + (int64_t)c.nap * (indx[k] - 1)));
          if (ne < 64) e_list[ne++] = e;
          T->psed[0][e] += q_i; T->psed[1][e] += q_q; T->psed[2][e] += q_u; T->psed[3][e] += q_v;
          T->psed[4][e] += q_i * q_i; T->psed[5][e] += q_q * q_q; T->psed[6][e] += q_u * q_u; T->psed[7][e] += q_v * q_v;
          T->psed[8][e] += 1.0;
        }
      }
    }
    if (adj && adj->record) adjoint_peel(q_i, img_k, e_list, ne);
  }

  void peel_all(double s_i, int ir, int it, int ip, int idust2) {
    for (int peelid = 1; peelid <= m->c.npeel; ++peelid) peeloff(s_i, ir, it, ip, idust2, peelid);
  }

  // isotrp.f90:1-36
  void isotrp(double sux, double suy, double suz, double& vx, double& vy, double& vz) {
    double r2 = 2.0, mur = 0.0, x = 0.0, y = 0.0, z = 0.0;
    while (r2 * r2 > std::fabs(mur)) {
      x = ran(); x = x + x - 1.0;
      y = ran(); y = y + y - 1.0;
      z = ran(); z = z + z - 1.0;
      mur = x * sux + y * suy + z * suz;
      r2 = x * x + y * y + z * z;
    }
    double r = std::sqrt(r2);
    if (mur < 0.0) r = -r;
    vx = x / r; vy = y / r; vz = z / r;
  }

  // select_dust with mask = is_thermal (emit_common_2.f90:346)
  int select_thermal(int ir, int it, int ip) {
    double xran = ran();
    int nn = 0, idust2 = 0;
    for (int id = 1; id <= MCRT_NDG2; ++id)
      if (!m->is_sg[id - 1] && m->dens(ir, it, ip, id) > 0.0) { ++nn; idust2 = id; }
    if (nn == 1) return idust2;
    double opac = 0.0;
    for (int id = 1; id <= MCRT_NDG2; ++id)
      if (!m->is_sg[id - 1]) opac = opac + kapd[m->fopac(ir, it, ip, id) - 1] * m->dens(ir, it, ip, id);
    if (opac == 0.0) return 0;
    double frac = 0.0;
    for (int id = 1; id <= MCRT_NDG2; ++id) {
      if (m->is_sg[id - 1]) continue;
      frac = frac + kapd[m->fopac(ir, it, ip, id) - 1] * m->dens(ir, it, ip, id) / opac;
      if (xran <= frac + 1.0e-10) return id;
    }
    return 0;
  }

  // emit_common_2.f90:201-372, vertical diffusion (|diffdir| = 2) without
  // accretion photons (nacc = 0).  Moves the packet to the diffusion
  // surface, heats the surface cell and emits isotropically from it.
  // Returns false on a geometry failure.  ir/it/idust2 are updated like the
  // reference's by-reference arguments.
  bool emit_diffusion(int& ir, int& it, int& ip, int& idust2) {
    const mcrt_grid* g = m->g;
    const double Tmax = 199999.0;
    const int dd = g->diffdir[m->cidx(ir, it, ip)];
    if (dd == -2) {
      while (it >= 1 && g->diffus[m->cidx(ir, it, ip)]) it = it - 1;
      if (it < 1) return false;
      it = it + 1;
    } else {
      while (it <= m->ntg - 1 && g->diffus[m->cidx(ir, it, ip)]) it = it + 1;
      if (it > m->ntg - 1) return false;
    }
    cosb = zp / rtot;
    sinb = std::sqrt(1.0 - cosb * cosb);
    const double cosbnew = 1.00001 * m->costarr[it - 1];
    const double sinbnew = std::sqrt(1.0 - cosbnew * cosbnew);
    xp = xp * sinbnew / sinb;
    yp = yp * sinbnew / sinb;
    zp = rtot * cosbnew;
    const double mu0 = m->costarr[it - 1], sth = m->sintarr[it - 1];
    double sux, suy, suz;
    if (mu0 > 0.0) { sux = -mu0 * xp / sth / rtot; suy = -mu0 * yp / sth / rtot; suz = sth; }
    else { sux = mu0 * xp / sth / rtot; suy = mu0 * yp / sth / rtot; suz = -sth; }
    isotrp(sux, suy, suz, ux, uy, uz);
    cost = uz;
    sint = std::sqrt(1.0 - cost * cost);
    cosp = ux / sint;
    sinp = uy / sint;
    phi = std::atan2(sinp, cosp);
    if (m->costarr[it - 1] < 0.0) it = it - 1;
    const double dA = PI * sth * (m->rarr[ir] * m->rarr[ir] - m->rarr[ir - 1] * m->rarr[ir - 1]);
    double T4s = m->c.tstar * m->c.tstar;
    T4s = T4s * T4s;
    const int64_t cs = m->cidx(ir, it, ip);
    int nth = 0;
    for (int id = 1; id <= MCRT_NDG2; ++id) if (!m->is_sg[id - 1] && m->dens(ir, it, ip, id) > 0.0) ++nth;
    if (nth == 0) return false;
    // adjoint evaluations freeze the surface at its start-of-iteration
    // temperature (a replay must see the forward pass's heating)
    const int32_t k = adj ? 0 : m->ndiff[cs].fetch_add(nth) + nth;
    double T4d = g->tdust[cs] * g->tdust[cs];
    T4d = T4d * T4d;
    const double T4 = T4d + (double)k * (4.0 * PI * T4s / (m->nphot_diff * dA));
    const double tsurf = std::min(Tmax / 11605.0, std::pow(T4, 0.25));
    idust2 = select_thermal(ir, it, ip);
    if (idust2 == 0) return false;
    double T4b = tsurf * tsurf;
    T4b = T4b * T4b;
    const double T4eff = 0.0;   // 4 pi T4s nacc/(dA nphot) with nacc = 0
    const double mu = ux * sux + uy * suy + uz * suz;
    const double T = std::min(std::pow(T4b + 0.75 * mu * T4eff, 0.25), Tmax / 11605.0);
    nub = bbfreq(T);
    if (g->diffdir[cs] == -2) it = it - 1; else it = it + 1;
    return true;
  }

  // select_dust_2.f90:1-84 with mask = is_any; returns 1-based id or 0
  int select_dust(int ir, int it, int ip) {
    double xran = ran();
    int nn = 0, idust2 = 0;
    for (int id = 1; id <= MCRT_NDG2; ++id)
      if (!m->is_sg[id - 1] && m->dens(ir, it, ip, id) > 0.0) { ++nn; idust2 = id; }
    if (nn == 1) return idust2;
    double opac = 0.0;
    for (int id = 1; id <= MCRT_NDG2; ++id) opac = opac + kapd[m->fopac(ir, it, ip, id) - 1] * m->dens(ir, it, ip, id);
    if (opac == 0.0) return 0;
    double frac = 0.0;
    for (int id = 1; id <= MCRT_NDG2; ++id) {
      frac = frac + kapd[m->fopac(ir, it, ip, id) - 1] * m->dens(ir, it, ip, id) / opac;
      if (xran <= frac + 1.0e-10) return id;
    }
    return 0;
  }

  // initpacc_4.f90:19-99 with emit_common: a disk-accretion packet.  The
  // radius comes once from the luminosity CDF Ldint (locate, cell centre
  // ravearr); the azimuth (rantheta, random.f90:23-42) and the height
  // hdisk*gasdev (random.f90:119-138, polar Box-Muller keeping its second
  // deviate) are redrawn until the point lies in a cell with thermal dust
  // (initpacc_4.f90:22, goto 11).  Two choices of this restatement, shared
  // with the engine: gasdev's saved deviate belongs to the packet (the
  // reference carries it from one packet to the next of a rank's single
  // stream; packets here use independent streams), and a point outside the
  // grid is redrawn (the reference would index past its arrays).  The
  // reference's dsg/dbig/nabs rules (:83-97) reduce to dbig and nabs for the
  // selected thermal component.  Returns idust2, or 0 on failure.
  int accretion_emission(int* ii) {
    const mcrt_grid* g = m->g;
    const int nrg = m->nrg;
    const double xi = ran();
    int r0 = locate(g->Ldint, nrg - 1, xi);
    r0 = std::min(std::max(r0, 1), nrg - 1);
    const double rp = g->ravearr[r0 - 1], hd = g->hdisk[r0 - 1];
    bool have_g = false, found = false;
    double gsave = 0.0;
    int ir = 0, it = 0, ip = 0;
    for (int tries = 0; tries < 1000000 && !found; ++tries) {
      double x = 0.0, y = 0.0, r2 = 2.0;
      while (r2 > 1.0) {
        x = ran(); x = x + x - 1.0;
        y = ran(); y = y + y - 1.0;
        r2 = x * x + y * y;
      }
      const double rr = std::sqrt(r2);
      const double st = y / rr, ct = x / rr;
      xp = rp * ct;
      yp = rp * st;
      double gd;
      if (!have_g) {
        double v1, v2, q;
        do {
          v1 = 2.0 * ran() - 1.0;
          v2 = 2.0 * ran() - 1.0;
          q = v1 * v1 + v2 * v2;
        } while (!(q < 1.0 && q > 0.0));
        const double fac = std::sqrt(-2.0 * std::log(q) / q);
        gsave = v1 * fac;
        gd = v2 * fac;
        have_g = true;
      } else {
        gd = gsave;
        have_g = false;
      }
      zp = hd * gd;
      sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
      rsq = xp * xp + yp * yp + zp * zp;
      rtot = std::sqrt(rsq);
      ir = locate(m->r2arr.data(), nrg, rsq);
      cosb = zp / rtot;
      it = locate(m->costarr.data(), m->ntg, cosb);
      lp = std::atan2(yp, xp);
      if (lp < 0.0) lp = lp + R2P;
      ip = locate(m->phiarr.data(), m->npg, lp);
      if (ir < 1 || ir > nrg - 1 || it < 1 || it > m->ntg - 1 || ip < 1 || ip > m->npg - 1) continue;
      double th = 0.0;
      for (int id = 1; id <= MCRT_NDG2; ++id) if (!m->is_sg[id - 1]) th += m->dens(ir, it, ip, id);
      found = th > 0.0;
    }
    if (!found) return 0;
    int idust2 = select_thermal(ir, it, ip);
    if (idust2 == 0) return 0;
    const int64_t cc = m->cidx(ir, it, ip);
    T->dbig[cc]++;
    T->nabs[cc]++;
    ii[0] = ir; ii[1] = it; ii[2] = ip;
    if (!m->g->diffus[cc]) {               // emit_common, thermal branch: reemit.f90 + lucydustfreq
      const double tave = m->g->tdust[cc];
      sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
      cost = 1.0 - 2.0 * ran();
      sint = std::sqrt(1.0 - cost * cost);
      phi = R2P * ran();
      cosp = std::cos(phi);
      sinp = std::sin(phi);
      nub = lucydustfreq(tave, m->fopac(ir, it, ip, idust2));
      uy = sint * sinp;
      ux = sint * cosp;
      uz = cost;
    } else {
      ++ndiffev;
      if (!emit_diffusion(ir, it, ip, idust2)) return 0;
      ii[1] = it;
    }
    return idust2;
  }

  // ------------------------------------------------------------ adjoint
  // Replay: before the walk that follows interaction k (k = nscat + nabsev;
  // 0 after the emission), drop the peel-offs of event k from A.
  void adjoint_advance(const int* ii) {
    if (!adj || !adj->replay) return;
    const int k = nscat + nabsev;
    while (adj->pos < adj->ev.size() && adj->ev[adj->pos].first <= k) adj->A -= adj->ev[adj->pos++].second;
    if (adj->vtab || adj->vsum) {
      int fb = (int)((double)adj->nfb * (std::log(nub) - adj->lnumin) / adj->lnurat);
      fb = std::min(std::max(fb, 0), adj->nfb - 1);
      int db = 0;
      if (adj->ndir == 4) {     // outward / inward radially, away from / toward the midplane
        const double ux_ = sint * cosp, uy_ = sint * sinp, uz_ = cost;
        db = (ux_ * xp + uy_ * yp + uz_ * zp > 0.0 ? 1 : 0) + (uz_ * zp > 0.0 ? 2 : 0);
      }
      const int64_t v = (m->cidx(ii[0], ii[1], ii[2]) * adj->nfb + fb) * adj->ndir + db;
      if (adj->vtab) adj->B = adj->vtab[v];
      if (adj->vsum) { adj->vsum[v] += adj->A; adj->vcnt[v] += 1.0; }
    }
  }
  // Replay: the interaction density kapd*rho of the selected component at
  // the end of the segment.
  void adjoint_interaction(int ir, int it, int ip, int idust2) {
    if (!adj || !adj->replay || adj->W() == 0.0) return;
    (*adj->grad)[m->cidx(ir, it, ip) + m->ncell * (idust2 - 1)] += adj->W();
  }
  // Pass 1: weighted contribution of one binned peel-off and its -C*tau
  // terms along the recorded ray.
  void adjoint_peel(double q_i, int64_t img_k, const int64_t* e_list, int ne) {
    const double* lp = adj->lam_psed;
    double C = 0.0;
    for (int j = 0; j < ne; ++j) C += lp[e_list[j]] * q_i;
    if (img_k >= 0 && adj->lam_img) C += adj->lam_img[img_k] * q_i;
    adj->obj += C;
    const int k = nscat + nabsev;
    if (!adj->ev.empty() && adj->ev.back().first == k) adj->ev.back().second += C;
    else adj->ev.emplace_back(k, C);
    if (C == 0.0) return;
    for (const auto& cr : adj->cross) {
      const int64_t c = cr.first;
      for (int id = 1; id <= MCRT_NDG2; ++id) {
        const double d = m->g->densarr[c + m->ncell * (id - 1)];
        if (d > 0.0) (*adj->grad)[c + m->ncell * (id - 1)] -= C * (kapd[m->g->findopac[c + m->ncell * (id - 1)] - 1] * d * cr.second);
      }
    }
  }

  // ----------------------------------------------------------- packet
  // newdisktherm_5_fuv.f90:220-491 for one packet, then propagate
  int run(int64_t iphot, int64_t np, int64_t ns, int64_t npacc, int64_t npaccstar, int ips) {
    const mcrt_config& c = m->c;
    on_wall = false;
    int ii[3] = {0, 0, 0};
    if (iphot < npacc) {                    // disk accretion, newdisktherm_5_fuv.f90:238-287
      const int idust2 = accretion_emission(ii);
      if (idust2 == 0) return 3;
      opacset(nub);
      kapd_disk();
      iflag = 0;
      i_orig = 2;
      if (ipeel == 1) peel_all(sip, ii[0], ii[1], ii[2], idust2);
    } else if (iphot <= npacc + ns) {
      if (iphot < npacc + npaccstar) {
        if (ips == 0) initpspot(1); else initp_ps(1);
        if (ran() < 0.5) nub = 1.2398 / 0.06 + ran() * (1.2398 / 0.015 - 1.2398 / 0.06);
      } else {
        if (ips == 0) initpspot(0); else initp_ps(0);
      }
      i_orig = 1;
      opacset(nub);
      kapd_disk();
      double coslp = std::cos(lp), sinlp = std::sin(lp);
      double rmin = m->rarr[0];
      zp = cosb * rmin;
      double rp = sinb * rmin;
      xp = rp * coslp;
      yp = rp * sinlp;
      rsq = zp * zp + rp * rp;
      rtot = std::sqrt(rsq);
      ux = sint * cosp;
      uy = sint * sinp;
      uz = cost;
      iflag = 0;
      ii[0] = 1;
      on_wall = true;
      double thetb = std::acos(cosb);
      ii[1] = locate(m->thetarr.data(), m->ntg, thetb);
      ii[2] = locate(m->phiarr.data(), m->npg, lp);
      if (ipeel == 1 && !c.partial_peeloff) {
        for (int peelid = 1; peelid <= c.npeel; ++peelid) {
          const double coste = m->t->coste_arr[peelid - 1], sinte = m->t->sinte_arr[peelid - 1];
          const double cospe = m->t->cospe_arr[peelid - 1], sinpe = m->t->sinpe_arr[peelid - 1];
          if (ips == 0) {
            double cosnorm = cosb * coste + (sinb * sinte * (cospe * coslp + sinpe * sinlp));
            double sipnew;
            if (c.limb == 0) sipnew = 4.0 * sip * cosnorm;
            else sipnew = 12.0 / 5.0 * sip * (cosnorm + cosnorm * cosnorm);
            if (cosnorm > 0.0) peeloff(sipnew, ii[0], ii[1], ii[2], 0, peelid);
          } else {
            peeloff(sip * 2.0, ii[0], ii[1], ii[2], 0, peelid);
          }
        }
      }
    } else {                                 // external illumination, newdisktherm_5_fuv.f90:416-460
      initpout();
      on_wall = true;
      i_orig = 5;
      opacset(nub);
      kapd_disk();
      const double coslp = std::cos(lp), sinlp = std::sin(lp);
      const double rmax = m->rarr[m->nrg - 1];
      zp = cosb * rmax * 0.999999;
      const double rp = sinb * rmax * 0.999999;
      xp = rp * coslp;
      yp = rp * sinlp;
      rsq = zp * zp + rp * rp;
      rtot = std::sqrt(rsq);
      ux = sint * cosp;
      uy = sint * sinp;
      uz = cost;
      iflag = 0;
      ii[0] = m->nrg - 1;
      ii[1] = locate(m->thetarr.data(), m->ntg, std::acos(cosb));
      ii[2] = locate(m->phiarr.data(), m->npg, lp);
      // no peel-off of the direct light: it is the sky background
    }
    ifuv = is_fuv(nub) ? c.ifuv_ori : 0.0;
    return propagate(ii);
  }

  // propagate_5_fuv.f90:1-326.  Returns the packet status.
  int propagate(int* ii) {
    const mcrt_config& c = m->c;
    const mcrt_tables* t = m->t;
    double xpold = xp, ypold = yp, zpold = zp;
    iflag = 0;
    exitflag = 0;
    int iscat = 0, iint = 0, idust2 = 0;
    int64_t nev = 0;
    adjoint_advance(ii);
    tau = -std::log(ran());
    if (!tauint(ii[0], ii[1], ii[2])) return 3;
    int ir = ii[0], it = ii[1], ip = ii[2];
    if (exitflag != 1) {
      idust2 = select_dust(ir, it, ip);
      if (idust2 == 0) return 3;
      adjoint_interaction(ir, it, ip, idust2);
      T->scal[MCRT_S_TOT] += 1.0;
      for (;;) {
        int fo = m->fopac(ir, it, ip, idust2) - 1;
        T->cnt[MCRT_C_INTERACTIONS]++;
        if (ran() <= albedo[fo]) {          // scattered
          iflag = 1;
          ++iscat;
          ++iint;
          ++nscat;
          T->cnt[MCRT_C_SCATTERS]++;
          if (ipeel == 1) peel_all(sip, ii[0], ii[1], ii[2], idust2);
          scatter(fo);
        } else {                            // absorbed + re-emitted
          ++nabsev;
          int64_t cc = m->cidx(ir, it, ip);
          if (m->is_sg[idust2 - 1]) T->dsg[cc]++; else T->dbig[cc]++;
          if (idust2 == 1 || idust2 == 2 || idust2 == 5 || idust2 == 6 || idust2 == 9) i_orig = 2;
          else if (idust2 == 3 || idust2 == 7) i_orig = 3;
          else i_orig = 4;
          if (!m->g->diffus[cc]) T->nabs[cc]++;
          if (!m->g->diffus[cc] && m->is_sg[idust2 - 1]) {
            // emit_common, small grains (emit_common_2.f90:32-50): a frequency
            // from the Draine spectrum of the cell's intensity level, then
            // emit_sg.f90; the opacset there is repeated below
            const int im = m->iter == 1 ? 2 : (m->g->imean ? m->g->imean[cc] : 1);
            nub = rep_draine(m->t, im, rng);
            sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
            cost = 1.0 - 2.0 * ran();
            sint = std::sqrt(1.0 - cost * cost);
            phi = R2P * ran();
            cosp = std::cos(phi);
            sinp = std::sin(phi);
            uy = sint * sinp;
            ux = sint * cosp;
            uz = cost;
          } else if (!m->g->diffus[cc]) {
            // emit_common, non-diffusion thermal branch (emit_common_2.f90:52-81)
            double tave = m->g->tdust[cc];
            // reemit.f90
            sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
            cost = 1.0 - 2.0 * ran();
            sint = std::sqrt(1.0 - cost * cost);
            phi = R2P * ran();
            cosp = std::cos(phi);
            sinp = std::sin(phi);
            nub = lucydustfreq(tave, m->fopac(ir, it, ip, idust2));
            uy = sint * sinp;
            ux = sint * cosp;
            uz = cost;
          } else {
            ++ndiffev;
            if (!emit_diffusion(ir, it, ip, idust2)) return 3;
            ii[1] = it;
          }
          iflag = 0;
          opacset(nub);
          ifuv = is_fuv(nub) ? c.ifuv_ori : 0.0;
          kapd_propagate();
          if (ipeel == 1 && !c.partial_peeloff) peel_all(sip, ii[0], ii[1], ii[2], idust2);
          ++iint;
        }
        adjoint_advance(ii);
        tau = -std::log(ran());
        xpold = xp; ypold = yp; zpold = zp;
        ux = sint * cosp;
        uy = sint * sinp;
        uz = cost;
        int prev[3] = {ii[0], ii[1], ii[2]};
        if (!tauint(ii[0], ii[1], ii[2])) return 3;
        ir = ii[0]; it = ii[1]; ip = ii[2];
        if (exitflag == 1) break;
        if (ii[0] != prev[0] || ii[1] != prev[1] || ii[2] != prev[2]) iint = 0;
        if (c.iffuv && !is_fuv(nub)) return 2;
        if (iint > 10000 || ++nev > 100000000) {   // + total-event watchdog
          T->killed[m->cidx(ii[0], ii[1], ii[2])]++;
          T->scal[MCRT_S_ABFLUX] += 1.0;
          T->cnt[MCRT_C_KILLED]++;
          return 1;
        }
        idust2 = select_dust(ir, it, ip);
        if (idust2 == 0) return 3;
        adjoint_interaction(ir, it, ip, idust2);
      }
    }
    // exit: bin into the SED arrays (propagate_5_fuv.f90:231-320)
    T->cnt[MCRT_C_EXITED]++;
    int itb = (int)((double)c.nmu * (1.0 - cost) / 2.0) + 1;
    itb = std::min(std::max(itb, 1), c.nmu);
    if (phi < 0.0) phi = phi + R2P;
    int ipb = (int)((double)c.nph * phi / R2P) + 1;
    ipb = std::min(std::max(ipb, 1), c.nph);
    double ub = t->u[itb - 1];
    double sini = std::sqrt(1.0 - ub * ub);
    double x = ypold * cosp - xpold * sinp;
    double y = zpold * sini - ypold * ub * sinp - xpold * ub * cosp;
    double rho2 = x * x + y * y;
    if (rho2 < t->aperture2[c.nap - 1] * 1.0001) {
      T->scal[MCRT_S_FLUX] += 1.0;
      if (iflag == 1) {
        T->scal[MCRT_S_SFLUX] += 1.0;
        T->scal[MCRT_S_NSCAT] += iscat;
      }
    }
    int inub = freq_bin(nub);
    int i_inter = (iflag == 1) ? 2 : ((i_orig == 1) ? 1 : 3);
    int indx[3] = {1, 1 + i_orig, 5 + i_inter};
    for (int ia = 1; ia <= c.nap; ++ia) {
      if (rho2 < t->aperture2[ia - 1]) {
        if (!(iflag == 0 && i_orig == 5)) {
          for (int k = 0; k < 3; ++k) {
            int64_t e = (inub - 1) + (int64_t)c.nfreq * ((itb - 1) + (int64_t)c.nmu * ((ipb - 1) + (int64_t)c.nph * ((ia - 1) + (int64_t)c.nap * (indx[k] - 1))));
            T->sed[0][e] += sip; T->sed[1][e] += sqp; T->sed[2][e] += sup; T->sed[3][e] += svp;
            T->sed[4][e] += sip * sip; T->sed[5][e] += sqp * sqp; T->sed[6][e] += sup * sup; T->sed[7][e] += svp * svp;
            T->sed[8][e] += 1.0;
            T->sed[9][e] += std::fabs(cost);
          }
        }
      }
    }
    if (iflag == 1) T->scal[MCRT_S_SCOUNT] += 1.0;
    return 0;
  }
};

template <class S, class D>
void put(D* dst, const std::vector<S>& src) {
  if (!dst) return;
  for (size_t i = 0; i < src.size(); ++i) dst[i] = (D)src[i];
}

}  // namespace

extern "C" {

// Run packets iphot_lo..iphot_hi of an iteration of np packets
// (newdisktherm_5_fuv.f90:158-491) on `nthreads` host threads; the tallies
// of all threads are summed (the MPI_ALLREDUCE of :520-604).
int oracle_run(const mcrt_config* cfg, const mcrt_grid* grid, const mcrt_tables* tab, int64_t np,
               int64_t iphot_lo, int64_t iphot_hi, int32_t iter, int32_t ipeel, int32_t seed1,
               int32_t seed2, int32_t generator, int32_t nthreads, mcrt_tallies* out,
               mcrt_packet_log* log, int64_t nlog, double* tdust_out) {
  if (iter < 1) return MCRT_ERR_ARG;
  const int64_t block0 = (int64_t)(iter - 1) * np;
  Model m;
  m.c = *cfg;
  m.iter = iter;
  m.g = grid;
  m.t = tab;
  m.nrg = cfg->nrg; m.ntg = cfg->ntg; m.npg = cfg->npg;
  m.ncell = (int64_t)m.nrg * m.ntg * m.npg;
  zetainit(m.inczeta);
  const bool sg[MCRT_NDG2] = {false, false, false, false, true, true, true, true, false, false};  // grid_mod_5.f90:20
  for (int i = 0; i < MCRT_NDG2; ++i) m.is_sg[i] = sg[i];
  m.rmincgs = cfg->rstar * RSOL;
  m.pad_walls();
  if (cfg->ilucy != 1) return MCRT_ERR_UNSUPPORTED;
  for (int64_t c = 0; c < m.ncell; ++c)
    if (grid->diffus[c] && (grid->diffdir[c] != 2 && grid->diffdir[c] != -2)) return MCRT_ERR_UNSUPPORTED;
  std::vector<std::atomic<int32_t>> ndiff(m.ncell);
  for (auto& a : ndiff) a.store(0);
  m.ndiff = ndiff.data();

  // packet split (newdisktherm_5_fuv.f90:158-191)
  int64_t npout = (int64_t)(cfg->isrf_frac * (double)np);
  double rn = cfg->isrf_frac * (double)np;
  if (rn - (double)npout > 0.5) npout++;
  int64_t ns = (int64_t)((double)np * (1.0 - cfg->accfrac - cfg->isrf_frac));
  rn = (double)(float)np * (1.0 - cfg->accfrac - cfg->isrf_frac);
  if (rn - (double)ns > 0.5) ns++;
  int64_t npacc = (int64_t)((double)np * cfg->accfrac);
  int64_t npaccstar = (int64_t)(cfg->accfrac2 * (double)np);
  int64_t nsum = ns + npacc + npout;
  if (nsum != np) ns = ns + np - nsum;
  if (npout > 0 && (!tab->isrf || tab->nisrf < 2)) return MCRT_ERR_ARG;   // external packets need the ISRF table
  if (npacc > 1 && (!grid->ravearr || !grid->Ldint || !grid->hdisk)) return MCRT_ERR_ARG;
  // emit_common receives nphot = ns of the (rank's) run; a shard uses its share
  m.nphot_diff = (double)ns * (double)(iphot_hi - iphot_lo + 1) / (double)np;
  int ips = (cfg->rddust > 100.0) ? 1 : 0;

  const int64_t nsed = (int64_t)cfg->nfreq * cfg->nmu * cfg->nph * cfg->nap * MCRT_NO;
  const int64_t npsed = (int64_t)cfg->nfreq * cfg->npeel * cfg->nap * MCRT_NO;
  const int64_t nimg = (int64_t)cfg->npeel * cfg->nxhst * cfg->nxhst * cfg->nfreq;
  Images img;
  for (auto& v : img.im) v.assign(cfg->output_imcube ? nimg : 0, 0.0);
  const int64_t nimgb = (int64_t)cfg->npeel * cfg->nxhst * cfg->nxhst * cfg->nfilt;
  if (cfg->output_imfilt && (cfg->nfilt < 1 || !tab->nwfilt || !tab->filtwave || !tab->filtphi)) return MCRT_ERR_ARG;
  for (auto& v : img.imb) v.assign(cfg->output_imfilt ? nimgb : 0, 0.0);
  const int64_t nims = (int64_t)cfg->sparse_dim * cfg->sparse_dim * cfg->sparse_nnu * cfg->sparse_nlev * cfg->npeel;
  if (cfg->output_imsparse && (cfg->sparse_dim < 1 || cfg->sparse_nnu < 1 || cfg->sparse_nlev < 1 || !tab->sparse_levels))
    return MCRT_ERR_ARG;
  for (auto& v : img.ims) v.assign(cfg->output_imsparse ? nims : 0, 0.0);
  int nt = std::max(1, (int)nthreads);
  std::vector<Tally> tl(nt);
  for (auto& t : tl) t.init(m.ncell, nsed, npsed);
  std::atomic<int64_t> next(iphot_lo);
  const int64_t chunk = 64;
  auto worker = [&](int tid) {
    Tally& T = tl[tid];
    Packet p;
    p.m = &m; p.T = &T; p.I = &img; p.ipeel = ipeel;
    const int no = cfg->nopac;
    for (auto* v : {&p.kappa, &p.albedo, &p.g, &p.pl, &p.g2, &p.onemg2, &p.g2p1, &p.twog, &p.kapd}) v->assign(no, 0.0);
    for (;;) {
      int64_t lo = next.fetch_add(chunk);
      if (lo > iphot_hi) break;
      int64_t hi = std::min(lo + chunk - 1, iphot_hi);
      for (int64_t iphot = lo; iphot <= hi; ++iphot) {
        p.rng = stream(seed1, seed2, generator, block0 + iphot - 1);
        p.nscat = p.nabsev = p.ncross = p.nstar = p.ndiffev = 0;
        int st = p.run(iphot, np, ns, npacc, npaccstar, ips);
        T.cnt[MCRT_C_PACKETS]++;
        if (st == 3) T.cnt[MCRT_C_GEOM_FAIL]++;
        int64_t li = iphot - iphot_lo;
        if (log && li < nlog) {
          mcrt_packet_log& L = log[li];
          L.iphot = iphot; L.nscat = p.nscat; L.nabs = p.nabsev; L.ncross = p.ncross; L.nstar = p.nstar;
          L.status = st; L.ir = 0; L.it = 0; L.ip = 0; L.ndraws = (int32_t)p.rng.ndraws;
          L.iflag = p.iflag; L.i_orig = p.i_orig; L.pad = p.ndiffev;
          L.nub = p.nub; L.cost = p.cost; L.phi = p.phi; L.sip = p.sip; L.sqp = p.sqp; L.sup = p.sup; L.svp = p.svp;
          L.xp = p.xp; L.yp = p.yp; L.zp = p.zp;
        }
      }
    }
  };
  std::vector<std::thread> th;
  for (int i = 1; i < nt; ++i) th.emplace_back(worker, i);
  worker(0);
  for (auto& t : th) t.join();
  Tally& S = tl[0];
  for (int i = 1; i < nt; ++i) {
    Tally& o = tl[i];
    for (int64_t c = 0; c < m.ncell; ++c) {
      S.nabs[c] += o.nabs[c]; S.dbig[c] += o.dbig[c]; S.dsg[c] += o.dsg[c]; S.killed[c] += o.killed[c];
      S.dtauabs[c] += o.dtauabs[c]; S.fuvmean[c] += o.fuvmean[c];
    }
    for (int k = 0; k < 10; ++k) for (int64_t e = 0; e < nsed; ++e) S.sed[k][e] += o.sed[k][e];
    for (int k = 0; k < 9; ++k) for (int64_t e = 0; e < npsed; ++e) S.psed[k][e] += o.psed[k][e];
    for (int k = 0; k < MCRT_NSCALARS; ++k) S.scal[k] += o.scal[k];
    for (int k = 0; k < MCRT_NCOUNTERS; ++k) S.cnt[k] += o.cnt[k];
  }
  if (out) {
    put(out->nabs, S.nabs); put(out->dbig, S.dbig); put(out->dsg, S.dsg); put(out->killed, S.killed);
    put(out->dtauabs, S.dtauabs); put(out->fuvmean, S.fuvmean);
    float* sd[10] = {out->si, out->sq, out->su, out->sv, out->si2, out->sq2, out->su2, out->sv2, out->nums, out->aveinc};
    for (int k = 0; k < 10; ++k) put(sd[k], S.sed[k]);
    float* pd[9] = {out->ti, out->tq, out->tu, out->tv, out->ti2, out->tq2, out->tu2, out->tv2, out->numt};
    for (int k = 0; k < 9; ++k) put(pd[k], S.psed[k]);
    float* im[4] = {out->image_m_i, out->image_m_q, out->image_m_u, out->image_m_v};
    for (int k = 0; k < 4; ++k) put(im[k], img.im[k]);
    float* ib[8] = {out->image_b_i, out->image_b_q, out->image_b_u, out->image_b_v,
                    out->image_b_d, out->image_b_s, out->image_b_e, out->image_b_o};
    for (int k = 0; k < 8; ++k) put(ib[k], img.imb[k]);
    float* is[4] = {out->image_ms_i, out->image_ms_q, out->image_ms_u, out->image_ms_v};
    for (int k = 0; k < 4; ++k) put(is[k], img.ims[k]);
    if (out->scalars) for (int k = 0; k < MCRT_NSCALARS; ++k) out->scalars[k] = S.scal[k];
    if (out->counters) for (int k = 0; k < MCRT_NCOUNTERS; ++k) out->counters[k] = S.cnt[k];
  }
  // End-of-iteration tdust of the diffusion cells (emit_common_2.f90:260-339,
  // nacc = 0): the surface cell of a column with N diffusion absorptions
  // holds min(Tmax,(T0^4+N dT^4)^(1/4)); interior cells whose neighbour
  // toward the surface holds a thermal component take the same value.
  if (tdust_out) {
    const int nrg = m.nrg, ntg = m.ntg, npg = m.npg;
    auto thermal = [&](int r, int t, int p) {
      for (int id = 1; id <= MCRT_NDG2; ++id) if (!m.is_sg[id - 1] && m.dens(r, t, p, id) > 0.0) return true;
      return false;
    };
    for (int ip = 1; ip <= npg; ++ip)
      for (int it = 1; it <= ntg; ++it)
        for (int ir = 1; ir <= nrg; ++ir) {
          const int64_t c = m.cidx(ir, it, ip);
          double t = grid->tdust[c];
          if (grid->diffus[c]) {
            const int dd = grid->diffdir[c];
            int is = it, iwall;
            if (dd == -2) { while (is - 1 >= 1 && grid->diffus[m.cidx(ir, is - 1, ip)]) --is; iwall = is; }
            else { while (is + 1 <= ntg - 1 && grid->diffus[m.cidx(ir, is + 1, ip)]) ++is; iwall = is + 1; }
            const int64_t cs = m.cidx(ir, is, ip);
            const int32_t N = ndiff[cs].load();
            bool gets = false;
            if (N > 0) {
              if (is == it) gets = thermal(ir, is, ip);
              else if (dd == -2) gets = thermal(ir, it - 1, ip);
              else gets = thermal(ir, it + 1, ip);
            }
            if (gets) {
              const double sth = m.sintarr[iwall - 1];
              const double dA = PI * sth * (m.rarr[ir] * m.rarr[ir] - m.rarr[ir - 1] * m.rarr[ir - 1]);
              double T4s = cfg->tstar * cfg->tstar;
              T4s = T4s * T4s;
              const double t0 = grid->tdust[cs];
              double T4d = t0 * t0;
              T4d = T4d * T4d;
              const double T4 = T4d + (double)N * (4.0 * PI * T4s / (m.nphot_diff * dA));
              t = std::min(199999.0 / 11605.0, std::pow(T4, 0.25));
            }
          }
          tdust_out[c] = t;
        }
  }
  return MCRT_OK;
}

// First n uniforms of packet block `block` (1-based iphot = block+1).
void oracle_rng(int32_t seed1, int32_t seed2, int32_t generator, int64_t block, int32_t n, double* out, int32_t* seeds) {
  Rng r = stream(seed1, seed2, generator, block);
  if (seeds) { seeds[0] = r.s1; seeds[1] = r.s2; }
  for (int i = 0; i < n; ++i) out[i] = r.ran();
}

// bbfreq's cumulative zeta table (random.f90:227-245).
void oracle_inczeta(double* out) { zetainit(out); }

// -------------------------------------------------------------- tfinal --
// KapP (dust_5.f90:144-172)
static double kapP(const mcrt_config* c, const mcrt_tables* t, double T, int idust3) {
  const int nT = c->nT;
  double lT = std::log(T);
  int k = (int)((double)(nT - 1) * (lT - t->lTint[0]) / (t->lTint[nT - 1] - t->lTint[0])) + 1;
  const double* kp = t->kappap + (int64_t)nT * (idust3 - 1);
  if (k < 1) return kp[0];
  if (k > nT - 1) return kp[nT - 1];
  double f = (lT - t->lTint[k - 1]) / (t->lTint[k] - t->lTint[k - 1]);
  return (1.0 - f) * kp[k - 1] + f * kp[k];
}

// dusttemp (dusttemp_5.f90:8-152).  kappaT(i) = emission + adiabatic +
// advective term (:42-53); with vel == false (a gas at rest) only the
// emission term, as the other two are exact zeros then.
static double dusttemp(const mcrt_config* c, const mcrt_tables* t, double na, int nphot, int idust3, double mcell,
                       double gradtr, double gradtt, double divv, double vr, double vthet, bool vel = false) {
  const int nT = c->nT;
  const double Tmax = 199999.0;
  const double rstar = c->rstar, tstar = c->tstarave;
  std::vector<double> kappaT(nT);
  const double* kp = t->kappap + (int64_t)nT * (idust3 - 1);
  const double kv = t->kappav[idust3 - 1];
  // Tint**4 etc. are integer powers in Fortran: x2=x*x, x4=x2*x2
  auto p4 = [](double x) { double x2 = x * x; return x2 * x2; };
  const double p3 = 11605.0 * 11605.0 * 11605.0;
  const double c1 = KB / 4.0 / SIGT / 2.3 / MHY, c2 = KB * 3.0 / 8.0 / SIGT / 2.3 / MHY;
  // the factor of Tint in the adiabatic term and the advective term, formed
  // once per cell
  const double adi = c1 / kv / p3 * divv / rstar / RSOL;
  const double adv = c2 / kv / p3 * (vr * gradtr + vthet * gradtt) / rstar / RSOL;
  for (int i = 0; i < nT; ++i) {
    const double emi = p4(t->Tint[i]) * kp[i];
    kappaT[i] = vel ? emi + adi * t->Tint[i] + adv : emi;
  }
  double Td = 0.1 / 11605.0;
  if (mcell > 0.0) {
    double abs_ = p4(tstar) * (na * PI * rstar * rstar) / ((double)nphot * kv);
    abs_ = abs_ * (RSOL * RSOL) / p4(mcell);
    if (na == 0.0) return 0.1 / 11605.0;
    double minkap = kappaT[0], maxkap = kappaT[0];
    int mini = 1, maxi = 1;
    for (int i = 1; i <= nT; ++i) {
      if (minkap > kappaT[i - 1]) { minkap = kappaT[i - 1]; mini = i; }
      if (maxkap < kappaT[i - 1]) { maxkap = kappaT[i - 1]; maxi = i; }
    }
    if (maxkap < abs_) Td = std::max(std::min(t->Tint[maxi - 1], Tmax / 11605.0), 0.1 / 11605.0);
    if (minkap > abs_) Td = std::max(std::min(t->Tint[mini - 1], Tmax / 11605.0), 0.1 / 11605.0);
    if (mini < maxi) {
      for (int i = mini; i <= maxi - 1; ++i) {
        if (kappaT[i - 1] < abs_ && kappaT[i] >= abs_) {
          double kl = kappaT[i - 1], ku = kappaT[i], Tl = t->Tint[i - 1], Tu = t->Tint[i];
          Td = Tl + (Tu - Tl) / (ku - kl) * (abs_ - kl);
          Td = std::max(std::min(Td, Tmax / 11605.0), 0.1 / 11605.0);
          break;
        }
      }
    } else {
      for (int i = maxi; i <= mini - 1; ++i) {
        if (kappaT[i - 1] > abs_ && kappaT[i] <= abs_) {
          double kl = kappaT[i - 1], ku = kappaT[i], Tl = t->Tint[i - 1], Tu = t->Tint[i];
          Td = Tl + (Tu - Tl) / (ku - kl) * (abs_ - kl);
          Td = std::max(std::min(Td, Tmax / 11605.0), 0.1 / 11605.0);
          break;
        }
      }
    }
  }
  return Td;
}

// tfinal (tfinal_5_test1.f90:1-447) for axisymmetric models; with a gas
// velocity field every pass smooths the temperature, forms and smooths its
// gradients and adds dusttemp's adiabatic and advective terms.
int oracle_tfinal(const mcrt_config* c, const mcrt_grid* g, const mcrt_tables* t, const double* dtauabs,
                  const double* tdust_now, int32_t nphot, int32_t iter, double* tdave, int32_t* converge,
                  double* sig_out) {
  if (!tdust_now) tdust_now = g->tdust;
  const int nrg = c->nrg, ntg = c->ntg, npg = c->npg;
  const int64_t ncell = (int64_t)nrg * ntg * npg;
  auto ci = [&](int ir, int it, int ip) { return (int64_t)(ir - 1) + (int64_t)nrg * ((it - 1) + (int64_t)ntg * (ip - 1)); };
  auto dens = [&](int ir, int it, int ip, int id) { return g->densarr[ci(ir, it, ip) + ncell * (id - 1)]; };
  const bool sg[MCRT_NDG2] = {false, false, false, false, true, true, true, true, false, false};
  const double Tmax = 199999.0, T01 = 0.1 / 11605.0;
  std::vector<double> old(tdave, tdave + ncell), iter_acc(ncell, 0.0);
  int maxii = (iter > 3) ? 20 : 1;
  // gas velocity field: the temperature gradients of every pass
  // (tfinal_5_test1.f90:61-200) feed dusttemp's advective term
  const bool vel = g->vrarr && g->vthetarr && g->divvarr;
  const int64_t n2 = (int64_t)nrg * ntg;
  std::vector<double> tsm(vel ? n2 : 0), gtr(vel ? n2 : 0), gtt(vel ? n2 : 0), gtr2(vel ? n2 : 0), gtt2(vel ? n2 : 0);
  auto c2d = [&](int ir, int it) { return (int64_t)(ir - 1) + (int64_t)nrg * (it - 1); };
  auto box = [](int i, int w, int n, int& lo, int& hi) {
    if (i > w && i < n - w) { lo = i - w; hi = i + w; }
    else if (i <= w) { lo = 1; hi = i + w; }
    else { lo = i - w; hi = n - 1; }
  };
  auto rave = [&](int ir) { return g->ravearr ? g->ravearr[ir - 1] : 0.5 * (g->rarr[ir - 1] + g->rarr[ir]); };
  for (int ii = 1; ii <= maxii; ++ii) {
    const int ip = 1;
    if (vel) {
      std::fill(tsm.begin(), tsm.end(), 0.0);
      for (int ir = 1; ir <= nrg - 1; ++ir)
        for (int it = 1; it <= ntg - 1; ++it) {
          int r1, r2, t1, t2;
          box(ir, 15, nrg, r1, r2);
          box(it, 15, ntg, t1, t2);
          double tot = 0.0;
          int nsm = 0;
          for (int iir = r1; iir <= r2; ++iir)
            for (int iit = t1; iit <= t2; ++iit)
              if (tdave[ci(iir, iit, 1)] > T01) { ++nsm; tot += tdave[ci(iir, iit, 1)]; }
          if (nsm > 0) tot = tot / (double)nsm;
          tsm[c2d(ir, it)] = (tdave[ci(ir, it, 1)] == T01) ? T01 : tot;
        }
      auto T = [&](int i, int j) { return tsm[c2d(i, j)]; };
      auto disk = [&](int ir, int it) { return dens(ir, it, 1, 1) + dens(ir, it, 1, 2) + dens(ir, it, 1, 9) > 0.0; };
      for (int ir = 1; ir <= nrg - 1; ++ir) {
        const double rad = rave(ir), dr = g->rarr[ir] - g->rarr[ir - 1];
        for (int it = 1; it <= ntg - 1; ++it) {
          const double dt = g->thetarr[it] - g->thetarr[it - 1];
          double gr = 0.0, gt = 0.0;
          if (ii > 1) {
            gr = (T(ir + 1, it) - T(ir, it)) / dr;
            if (it <= 15) gr = (T(ir + 1, 16) - T(ir, 16)) / dr;
            if (ir >= nrg - 16) gr = gtr[c2d(nrg - 17, it)];
            if (disk(ir, it)) gr = 0.0;
            gt = (T(ir, it + 1) - T(ir, it)) / dt / rad;
            if (it <= 15) gt = (T(ir, 17) - T(ir, 16)) / rad / (g->thetarr[16] - g->thetarr[15]);
            if (ir >= nrg - 16) gt = gtt[c2d(nrg - 17, it)];
            if (disk(ir, it)) gt = 0.0;
          }
          gtr[c2d(ir, it)] = gr;
          gtt[c2d(ir, it)] = gt;
        }
      }
      for (int ir = 1; ir <= nrg - 1; ++ir)
        for (int it = 1; it <= ntg - 1; ++it) {
          int r1, r2;
          box(ir, 15, nrg, r1, r2);
          double gr = 0.0, gt = 0.0;
          if (dens(ir, it, 1, 4) + dens(ir, it, 1, 10) > 0.0) {
            int nsm = 0;
            for (int iir = r1; iir <= r2; ++iir)
              if (gtr[c2d(iir, it)] < 0.0) { ++nsm; gr += gtr[c2d(iir, it)]; }
            if (nsm > 0) gr = gr / (double)nsm;
          } else {
            for (int iir = r1; iir <= r2; ++iir) gr += gtr[c2d(iir, it)];
            gr = gr / (double)(r2 - r1 + 1) / 1.0;
          }
          for (int iir = r1; iir <= r2; ++iir) gt += gtt[c2d(iir, it)];
          gt = gt / (double)(r2 - r1 + 1) / 1.0;
          gtr2[c2d(ir, it)] = gr;
          gtt2[c2d(ir, it)] = gt;
        }
    }
    for (int ir = 1; ir <= nrg - 1; ++ir) {
      for (int it = 1; it <= (ntg - 1) / 2; ++it) {
        double td = T01;
        int itm = ntg - it;
        for (int id = 1; id <= MCRT_NDG2; ++id) {
          if (!sg[id - 1] && dens(ir, it, ip, id) > 0.0) {
            int idust3 = g->findopac[ci(ir, it, ip) + ncell * (id - 1)];
            if (!g->diffus[ci(ir, it, ip)]) {
              double m1 = std::pow(dens(ir, it, ip, id) * g->vcell[ci(ir, it, ip)], 0.25);
              double m2 = std::pow(dens(ir, itm, ip, id) * g->vcell[ci(ir, it, ip)], 0.25);
              const double gr = vel ? gtr2[c2d(ir, it)] : 0.0, gt = vel ? gtt2[c2d(ir, it)] : 0.0;
              const int64_t a = ci(ir, it, ip), b = ci(ir, itm, ip);
              double t1 = dusttemp(c, t, dtauabs[a], nphot, idust3, m1, gr, gt, vel ? g->divvarr[a] : 0.0,
                                   vel ? g->vrarr[a] : 0.0, vel ? g->vthetarr[a] : 0.0, vel);
              int idust3b = g->findopac[ci(ir, itm, ip) + ncell * (id - 1)];
              double t2 = dusttemp(c, t, dtauabs[b], nphot, idust3b, m2, gr, gt, vel ? g->divvarr[b] : 0.0,
                                   vel ? g->vrarr[b] : 0.0, vel ? g->vthetarr[b] : 0.0, vel);
              td = (t1 + t2) / 2.0;
            } else {
              td = (tdust_now[ci(ir, it, ip)] + tdust_now[ci(ir, itm, ip)]) / 2.0;
            }
            if (td * 11605.0 >= Tmax) td = Tmax / 11605.0;
          }
        }
        tdave[ci(ir, it, ip)] = td;
      }
    }
    for (int ir = 1; ir <= nrg - 1; ++ir)
      for (int it = (ntg + 1) / 2; it <= ntg - 1; ++it) tdave[ci(ir, it, 1)] = tdave[ci(ir, ntg - it, 1)];
    if (npg > 2)
      for (int ir = 1; ir <= nrg - 1; ++ir)
        for (int it = 1; it <= ntg - 1; ++it)
          for (int ipp = 2; ipp <= npg - 1; ++ipp) tdave[ci(ir, it, ipp)] = tdave[ci(ir, it, 1)];
    if (maxii > 10 && ii > 10) for (int64_t k = 0; k < ncell; ++k) iter_acc[k] += tdave[k];
  }
  if (maxii > 10) for (int64_t k = 0; k < ncell; ++k) tdave[k] = iter_acc[k] / (double)(maxii - 10);
  double s[3] = {0, 0, 0}, s2[3] = {0, 0, 0};
  int64_t n[3] = {0, 0, 0};
  for (int ir = 1; ir <= nrg - 1; ++ir) {
    for (int it = 1; it <= (ntg - 1) / 2; ++it) {
      double told = old[ci(ir, it, 1)], tnew = tdave[ci(ir, it, 1)];
      double d = (tnew - told) / tnew;
      if (tnew != told && tnew > T01 && told > T01) { s[0] += std::fabs(d); s2[0] += d * d; n[0]++; }
      if (!g->diffus[ci(ir, it, 1)] && tnew > T01 && told > T01) { s[1] += std::fabs(d); s2[1] += d * d; n[1]++; }
      if (g->rarr[ir - 1] / c->autors < 5.0 && tnew > T01 && told > T01) { s[2] += std::fabs(d); s2[2] += d * d; n[2]++; }
    }
  }
  for (int k = 0; k < 3; ++k) {
    double a = s[k] / (double)n[k], b = s2[k] / (double)n[k];
    if (sig_out) sig_out[k] = std::sqrt(b - a * a);
  }
  (void)converge;
  return MCRT_OK;
}

// setdiffus (setdiffus_5.f90:1-132) as the reference writes it: clear the
// flags; for ir from nr0 while rarr(ir) < rmaxd (and ir <= nrg-1), for it =
// (ntg-1)/2 down to 2, march toward the pole over slice 1 summing
// kapd(V) x chiR(tt) x densarr x dtheta x rad of the thermal components
// (tt = tdave, floored at 50 K when iter < 2) until tau reaches 1; if
// tau >= 1 and the path to tau = 1 is below hdisk/20, flag it..(ntg-1)/2
// with diffdir -2.  Mirror into the lower hemisphere (diffdir +2), copy slice
// 1 to the other phi slices, then gridset's reset (gridset_5_model13new.f90:
// 1855-1866): tdust = tdave, 0.1 K in diffusion cells and in empty cells.
// kapd holds kappav x R* (setup_wave.f90:50).  chiR (dust_5.f90:112-141)
// clamps an index outside the table to its end intervals where the
// reference stops.  Cells without a thermal component are left unflagged.
int oracle_setdiffus(const mcrt_config* c, const mcrt_grid* g, const mcrt_tables* t, int32_t iter, double massd,
                     double rmaxd, const double* tdave, int32_t* diffus, int32_t* diffdir, double* tdust) {
  const int nrg = c->nrg, ntg = c->ntg, npg = c->npg, nT = c->nT;
  const int64_t ncell = (int64_t)nrg * ntg * npg;
  auto ci = [&](int ir, int it, int ip) { return (int64_t)(ir - 1) + (int64_t)nrg * ((it - 1) + (int64_t)ntg * (ip - 1)); };
  auto dens = [&](int ir, int it, int ip, int id) { return g->densarr[ci(ir, it, ip) + ncell * (id - 1)]; };
  auto fop = [&](int ir, int it, int ip, int id) { return g->findopac[ci(ir, it, ip) + ncell * (id - 1)]; };
  const bool thermal[MCRT_NDG2] = {true, true, true, true, false, false, false, false, true, true};
  auto chiR = [&](double T, int sp) {
    const double lT = std::log(T);
    int k = (int)((double)(nT - 1) * (lT - t->lTint[0]) / (t->lTint[nT - 1] - t->lTint[0])) + 1;
    k = std::min(std::max(k, 1), nT - 1);
    const double f = (lT - t->lTint[k - 1]) / (t->lTint[k] - t->lTint[k - 1]);
    const double* kr = t->kappar + (int64_t)nT * (sp - 1);
    return (1.0 - f) * kr[k - 1] + f * kr[k];
  };
  const double rmincgs = c->rstar * 6.9598e10;
  std::fill(diffus, diffus + ncell, 0);
  std::fill(diffdir, diffdir + ncell, 0);
  if (massd > 0.0) {
    const int nr0 = (c->rddust == g->rarr[0]) ? 1 : 3;
    int ir = nr0;
    double rad = g->rarr[ir - 1];
    while (rad < rmaxd && ir <= nrg - 1) {
      const double zmr = g->hdisk[ir - 1];
      for (int it = (ntg - 1) / 2; it >= 2; --it) {
        double tau = 0.0, tau1 = 0.0;
        int itt = it;
        while (tau < 1.0 && itt > 1) {
          const double dt = g->thetarr[itt] - g->thetarr[itt - 1];
          tau1 = tau;
          double tt = tdave[ci(ir, itt, 1)];
          if (iter < 2) tt = std::max(tt, 50.0 / 11605.0);
          for (int id = 1; id <= MCRT_NDG2; ++id) {
            if (!thermal[id - 1] || !(dens(ir, itt, 1, id) > 0.0)) continue;
            const int sp = fop(ir, itt, 1, id);
            tau = tau + (t->kappav[sp - 1] * rmincgs) * chiR(tt, sp) * dens(ir, itt, 1, id) * dt * rad;
          }
          itt = itt - 1;
        }
        double lmfp1;
        if (tau > 1.0) lmfp1 = rad * (g->thetarr[itt + 1] - g->thetarr[itt]) / (tau - tau1) * (1.0 - tau1);
        else lmfp1 = rad * (g->thetarr[itt + 1] - g->thetarr[itt]);
        const double lmfp = rad * (g->thetarr[it] - g->thetarr[itt + 1]) + lmfp1;
        if (tau >= 1.0 && lmfp < zmr / 20.0)
          for (int it1 = it; it1 <= (ntg - 1) / 2; ++it1) { diffus[ci(ir, it1, 1)] = 1; diffdir[ci(ir, it1, 1)] = -2; }
      }
      ir = ir + 1;
      rad = g->rarr[ir - 1];
    }
    for (int ir2 = 1; ir2 <= nrg - 1; ++ir2)
      for (int it = (ntg + 1) / 2; it <= ntg - 1; ++it) {
        diffus[ci(ir2, it, 1)] = diffus[ci(ir2, ntg - it, 1)];
        diffdir[ci(ir2, it, 1)] = -diffdir[ci(ir2, ntg - it, 1)];
      }
    if (npg > 2)
      for (int ir2 = 1; ir2 <= nrg - 1; ++ir2)
        for (int it = 1; it <= ntg - 1; ++it)
          for (int ip = 2; ip <= npg - 1; ++ip) {
            diffus[ci(ir2, it, ip)] = diffus[ci(ir2, it, 1)];
            diffdir[ci(ir2, it, ip)] = diffdir[ci(ir2, it, 1)];
          }
  }
  for (int64_t k = 0; k < ncell; ++k) {
    bool th = false, any = false;
    for (int id = 1; id <= MCRT_NDG2; ++id) {
      const double rho = g->densarr[k + ncell * (id - 1)];
      if (rho > 0.0) { any = true; if (thermal[id - 1]) th = true; }
    }
    if (!th) { diffus[k] = 0; diffdir[k] = 0; }
    tdust[k] = (diffus[k] || !any) ? 0.1 / 11605.0 : tdave[k];
  }
  return 0;
}

}  // extern "C"


// Path-replay adjoint (see struct Adjoint): packets lo..hi of an np-packet
// iteration with peel-offs, objective and dL/dlog(rho) per (cell, component
// id) summed into grad[ncell*10] (Fortran order (nrg,ntg,npg,10)), objective
// into *obj.  Test infrastructure: the FP64 reference of mcrt_adjoint.
// With `vtab` (ncell x nfb, cell-major) every segment's score is weighted
// by A - vtab[cell, bin] (Adjoint::vtab) and every packet is replayed; with
// `vsum`/`vcnt` (same shape) the replay adds A and 1 per segment start.  The
// frequency bins split [numin, numin*e^lnurat] (the SED's range) into nfb
// log-uniform bins.
extern "C" int oracle_adjoint_cv(const mcrt_config* cfg, const mcrt_grid* grid, const mcrt_tables* tab, int64_t np,
                                 int64_t iphot_lo, int64_t iphot_hi, int32_t iter, int32_t seed1, int32_t seed2,
                                 int32_t generator, int32_t nthreads, const double* lam_psed, const double* lam_img,
                                 double* grad, double* obj, const double* vtab, int32_t nfb, double* vsum,
                                 double* vcnt) {
  if (iter < 1 || !lam_psed || !grad || !obj || nfb == 0 || ((vsum != nullptr) != (vcnt != nullptr)))
    return MCRT_ERR_ARG;
  const int64_t block0 = (int64_t)(iter - 1) * np;
  Model m;
  m.c = *cfg;
  m.iter = iter;
  m.g = grid;
  m.t = tab;
  m.nrg = cfg->nrg; m.ntg = cfg->ntg; m.npg = cfg->npg;
  m.ncell = (int64_t)m.nrg * m.ntg * m.npg;
  zetainit(m.inczeta);
  const bool sg[MCRT_NDG2] = {false, false, false, false, true, true, true, true, false, false};
  for (int i = 0; i < MCRT_NDG2; ++i) m.is_sg[i] = sg[i];
  m.rmincgs = cfg->rstar * RSOL;
  m.pad_walls();
  if (cfg->ilucy != 1) return MCRT_ERR_UNSUPPORTED;
  std::vector<std::atomic<int32_t>> ndiff(m.ncell);
  for (auto& a : ndiff) a.store(0);
  m.ndiff = ndiff.data();
  int64_t npout = (int64_t)(cfg->isrf_frac * (double)np);
  double rn = cfg->isrf_frac * (double)np;
  if (rn - (double)npout > 0.5) npout++;
  int64_t ns = (int64_t)((double)np * (1.0 - cfg->accfrac - cfg->isrf_frac));
  rn = (double)(float)np * (1.0 - cfg->accfrac - cfg->isrf_frac);
  if (rn - (double)ns > 0.5) ns++;
  int64_t npacc = (int64_t)((double)np * cfg->accfrac);
  int64_t npaccstar = (int64_t)(cfg->accfrac2 * (double)np);
  if (ns + npacc + npout != np) ns = ns + np - (ns + npacc + npout);
  if (npout > 0 && (!tab->isrf || tab->nisrf < 2)) return MCRT_ERR_ARG;   // external packets need the ISRF table
  m.nphot_diff = (double)ns * (double)(iphot_hi - iphot_lo + 1) / (double)np;
  const int ips = (cfg->rddust > 100.0) ? 1 : 0;
  const int64_t nsed = (int64_t)cfg->nfreq * cfg->nmu * cfg->nph * cfg->nap * MCRT_NO;
  const int64_t npsed = (int64_t)cfg->nfreq * cfg->npeel * cfg->nap * MCRT_NO;
  const int64_t nimg = (int64_t)cfg->npeel * cfg->nxhst * cfg->nxhst * cfg->nfreq;
  Images img;
  for (auto& v : img.im) v.assign(cfg->output_imcube ? nimg : 0, 0.0);
  const int nt = std::max(1, (int)nthreads);
  std::vector<Tally> tl(nt);
  for (auto& t : tl) t.init(m.ncell, nsed, npsed);
  std::vector<std::vector<double>> gl(nt, std::vector<double>(m.ncell * MCRT_NDG2, 0.0));
  std::vector<double> objs(nt, 0.0);
  const int ndir = nfb < 0 ? 4 : 1;
  if (nfb < 0) nfb = -nfb;
  const int64_t nv = vsum ? m.ncell * nfb * ndir : 0;
  std::vector<std::vector<double>> vs(nt, std::vector<double>(nv, 0.0)), vc(nt, std::vector<double>(nv, 0.0));
  const bool all = vtab || vsum;       // the control variate scores packets without peel-offs too
  std::atomic<int64_t> next(iphot_lo);
  auto worker = [&](int tid) {
    Packet p;
    Adjoint A;
    A.lam_psed = lam_psed;
    A.lam_img = cfg->output_imcube ? lam_img : nullptr;
    A.grad = &gl[tid];
    A.vtab = vtab;
    A.nfb = nfb;
    A.ndir = ndir;
    A.lnumin = std::log(cfg->numin);
    A.lnurat = cfg->lnurat;
    if (vsum) { A.vsum = vs[tid].data(); A.vcnt = vc[tid].data(); }
    p.m = &m; p.T = &tl[tid]; p.I = &img; p.adj = &A;
    for (auto* v : {&p.kappa, &p.albedo, &p.g, &p.pl, &p.g2, &p.onemg2, &p.g2p1, &p.twog, &p.kapd}) v->assign(cfg->nopac, 0.0);
    for (;;) {
      const int64_t lo = next.fetch_add(64);
      if (lo > iphot_hi) break;
      const int64_t hi = std::min(lo + 63, iphot_hi);
      for (int64_t iphot = lo; iphot <= hi; ++iphot) {
        // pass 1: the packet with its peel-offs
        A.ev.clear();
        A.record = true; A.replay = false;
        p.ipeel = 1;
        p.rng = stream(seed1, seed2, generator, block0 + iphot - 1);
        p.nscat = p.nabsev = p.ncross = p.nstar = p.ndiffev = 0;
        p.run(iphot, np, ns, npacc, npaccstar, ips);
        double R = 0.0;
        for (const auto& e : A.ev) R += e.second;
        if (R == 0.0 && !all) continue;
        // pass 2: replay on the same stream, scoring the segments
        A.record = false; A.replay = true;
        A.A = R; A.pos = 0; A.B = 0.0;
        p.ipeel = 0;
        p.rng = stream(seed1, seed2, generator, block0 + iphot - 1);
        p.nscat = p.nabsev = p.ncross = p.nstar = p.ndiffev = 0;
        p.run(iphot, np, ns, npacc, npaccstar, ips);
        A.replay = false;
      }
    }
    objs[tid] = A.obj;
  };
  std::vector<std::thread> th;
  for (int i = 1; i < nt; ++i) th.emplace_back(worker, i);
  worker(0);
  for (auto& t : th) t.join();
  for (int64_t k = 0; k < m.ncell * MCRT_NDG2; ++k) {
    double s = 0.0;
    for (int i = 0; i < nt; ++i) s += gl[i][k];
    grad[k] = s;
  }
  double o = 0.0;
  for (int i = 0; i < nt; ++i) o += objs[i];
  *obj = o;
  for (int64_t k = 0; k < nv; ++k) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < nt; ++i) { a += vs[i][k]; b += vc[i][k]; }
    vsum[k] += a;
    vcnt[k] += b;
  }
  return MCRT_OK;
}

extern "C" int oracle_adjoint(const mcrt_config* cfg, const mcrt_grid* grid, const mcrt_tables* tab, int64_t np,
                              int64_t iphot_lo, int64_t iphot_hi, int32_t iter, int32_t seed1, int32_t seed2,
                              int32_t generator, int32_t nthreads, const double* lam_psed, const double* lam_img,
                              double* grad, double* obj) {
  return oracle_adjoint_cv(cfg, grid, tab, np, iphot_lo, iphot_hi, iter, seed1, seed2, generator, nthreads, lam_psed,
                           lam_img, grad, obj, nullptr, 1, nullptr, nullptr);
}

// ===================================================================
// setemiss: the emission tables of the Lucy reemission (oracle restatement)
// -------------------------------------------------------------------
// dust_5.f90:486-494 (the temperature and frequency grids), dust_5.f90:507-
// 699 (setemiss: per species and temperature, the cumulative integral of
// kappa_abs * B_nu and the Rosseland integral of dB_nu/dT / chi over 513
// frequency intervals, each interval integrated by qsimp; the normalised
// cumulative table, the Planck mean and the Rosseland mean; the 21-point
// smoothing of the Planck mean of gas opacities, ids > ndg), dust_5.f90:784-
// 831 (the integrands kappaB, chidB), mathsubs.f90:4-47 (Bnu, dBnu),
// mathsubs.f90:79-113 (expm1 by the Abramowitz & Stegun 4.2.45 expansion
// below ln 2), nr_2.f:209-254 (qsimp/trapzd: trapezoid refinement with the
// Simpson combination, relative tolerance 1e-5, at most 20 levels; the
// Numerical Recipes algorithm, restated from its definition) and
// dust_5.f90:9-55 (opacset's interpolation of kappa and albedo in nu).
// ===================================================================
namespace setemiss_oracle {

double expm1_as(double x) {
  static const double c[7] = {0.9999999995, 0.4999999206, 0.1666653019, 0.0416573475,
                              0.0083013598, 0.0013298820, 0.0001413161};
  if (std::fabs(x) > 0.6931472) return std::exp(x) - 1.0;
  double s = 0.0;
  for (int i = 6; i >= 0; --i) s = x * (c[i] + s);
  return s;
}

const double kNorm = 0.1539897;   // 15/pi^4 as the reference writes it

double planck(double nu, double T) {
  const double x = nu / T;
  if (x == 0.0) return 0.0;
  return kNorm * x * x * x / expm1_as(x);
}

double dplanck(double nu, double T) {
  const double x = nu / T;
  if (x == 0.0) return 0.0;
  return -(kNorm * x * x * x * x) / (4.0 * expm1_as(x) * expm1_as(-x));
}

// kappa and albedo of one species at nu (linear in nu between the bracketing
// nodes of the descending nudust column, clamped at the ends)
void interp(const double* nud, const double* kd, const double* ad, int n, double nu, double& kap, double& alb) {
  if (nu >= nud[0]) { kap = kd[0]; alb = ad[0]; return; }
  if (nu <= nud[n - 1]) { kap = kd[n - 1]; alb = ad[n - 1]; return; }
  int i0 = 1, i1 = n;
  while (i1 - i0 > 1) {
    const int i = (i1 + i0) / 2;
    if (nu <= nud[i - 1]) i0 = i; else i1 = i;
  }
  const double f = (nu - nud[i1 - 1]) / (nud[i0 - 1] - nud[i1 - 1]);
  const double fm1 = 1.0 - f;
  kap = fm1 * kd[i1 - 1] + f * kd[i0 - 1];
  alb = fm1 * ad[i1 - 1] + f * ad[i0 - 1];
}

// trapezoid refinement on [0, 1] with the Simpson combination; `miss` is set
// when 20 levels do not reach the tolerance
template <class F>
double qsimp(const F& fn, bool& miss) {
  double st = 0.0, ost = -1.0e30, os = -1.0e30, s = 0.0;
  for (int j = 1; j <= 20; ++j) {
    if (j == 1) {
      st = 0.5 * (1.0 - 0.0) * (fn(0.0) + fn(1.0));
    } else {
      const long it = 1L << (j - 2);
      const double tnm = (double)it;
      const double del = (1.0 - 0.0) / tnm;
      double x = 0.0 + 0.5 * del, sum = 0.0;
      for (long k = 0; k < it; ++k) { sum = sum + fn(x); x = x + del; }
      st = 0.5 * (st + (1.0 - 0.0) * sum / tnm);
    }
    s = (4.0 * st - ost) / 3.0;
    if (std::fabs(s - os) < 1.0e-5 * std::fabs(os)) return s;
    os = s;
    ost = st;
  }
  miss = true;
  return s;
}

void one(int i, int id, int nT, int nnu, int nlammax, const int32_t* nlambda, const double* nudust,
         const double* kappad, const double* adust, const double* Tint, const double* nuint, double* kapint,
         double* kappap, double* kappar, int64_t* misses) {
  const double* nud = nudust + (int64_t)nlammax * id;
  const double* kd = kappad + (int64_t)nlammax * id;
  const double* ad = adust + (int64_t)nlammax * id;
  const int n = nlambda[id];
  const double T = Tint[i];
  double nu1 = 0.0, k1 = 0.0, a1 = 0.0;
  interp(nud, kd, ad, n, nu1, k1, a1);
  double chi1 = k1, kap1 = (1.0 - a1) * k1;
  double cum = 0.0, ross = 0.0;
  int64_t miss = 0;
  for (int j = 1; j <= nnu; ++j) {
    const double nu0 = nu1;
    nu1 = nuint[j - 1] * T;
    const double dnu = nu1 - nu0;
    const double dx = dnu / T;
    const double chi0 = chi1, kap0 = kap1;
    interp(nud, kd, ad, n, nu1, k1, a1);
    chi1 = k1;
    kap1 = (1.0 - a1) * k1;
    double ik = 0.0, ic = 0.0;
    if (nu0 / T < 50.0) {
      bool m1 = false, m2 = false;
      ik = qsimp([&](double f) { return ((1.0 - f) * kap0 + f * kap1) * planck(nu0 + f * dnu, T); }, m1);
      ic = qsimp([&](double f) { return dplanck(nu0 + f * dnu, T) / ((1.0 - f) * chi0 + f * chi1); }, m2);
      miss += (m1 ? 1 : 0) + (m2 ? 1 : 0);
    }
    if (j == 1) { cum = dx * ik; ross = dx * ic; }
    else { cum = dx * ik + cum; ross = dx * ic + ross; }
    kapint[i + (int64_t)nT * ((j - 1) + (int64_t)nnu * id)] = cum;
  }
  kappar[i + (int64_t)nT * id] = 1.0 / ross;
  const double top = kapint[i + (int64_t)nT * ((nnu - 1) + (int64_t)nnu * id)];
  kappap[i + (int64_t)nT * id] = top;
  for (int j = 1; j <= nnu - 1; ++j) {
    double& v = kapint[i + (int64_t)nT * ((j - 1) + (int64_t)nnu * id)];
    v = v / top;
  }
  kapint[i + (int64_t)nT * ((nnu - 1) + (int64_t)nnu * id)] = 1.0;
  misses[0] += miss;
}

// two passes of the 21-point box average of the Planck mean (ids > ndg)
void smooth(int nT, double* kp) {
  const int ns = 10;
  std::vector<double> out(nT);
  for (int pass = 0; pass < 2; ++pass) {
    for (int i = 1; i <= nT; ++i) {
      int lo, hi;
      if (i > ns && i <= nT - ns) { lo = i - ns; hi = i + ns; }
      else if (i <= ns) { lo = 1; hi = 2 * i + 1; }
      else { lo = 2 * i - nT; hi = nT; }
      double s = 0.0;
      for (int k = lo; k <= hi; ++k) s = s + kp[k - 1];
      out[i - 1] = s / (double)(hi - lo + 1);
    }
    for (int i = 0; i < nT; ++i) kp[i] = out[i];
  }
}

}  // namespace setemiss_oracle

extern "C" int oracle_setemiss(int32_t nopac, int32_t ndg, int32_t nlammax, const int32_t* nlambda,
                               const double* nudust, const double* kappad, const double* adust, int32_t nT,
                               int32_t nnu, double* lTint, double* Tint, double* nuint, double* kapint,
                               double* kappap, double* kappar, int64_t* qsimp_misses, int32_t threads) {
  using namespace setemiss_oracle;
  if (nopac < 1 || nT < 21 || nnu < 2 || nlammax < 2 || ndg < 0 || ndg > nopac) return 1;   // 21: the smoothing window
  const double Tmin = 0.1, Tmax = 200000.0, numax = 32.0, numin = numax / 1024.0;
  for (int i = 1; i <= nT; ++i) {
    lTint[i - 1] = std::log(Tmin / 11605.0) + (double)(i - 1) * std::log(Tmax / Tmin) / (double)(nT - 1);
    Tint[i - 1] = std::exp(lTint[i - 1]);
  }
  for (int i = 1; i <= nnu; ++i) nuint[i - 1] = numin + (double)(i - 1) * (numax - numin) / (double)(nnu - 1);
  const int64_t work = (int64_t)nT * nopac;
  const int nth = std::max(1, threads);
  std::atomic<int64_t> next{0};
  std::vector<int64_t> miss(nth, 0);
  std::vector<std::thread> th;
  for (int t = 0; t < nth; ++t)
    th.emplace_back([&, t]() {
      for (;;) {
        const int64_t w = next.fetch_add(1);
        if (w >= work) break;
        one((int)(w % nT), (int)(w / nT), nT, nnu, nlammax, nlambda, nudust, kappad, adust, Tint, nuint, kapint,
            kappap, kappar, &miss[t]);
      }
    });
  for (auto& x : th) x.join();
  for (int id = ndg; id < nopac; ++id) smooth(nT, kappap + (int64_t)nT * id);
  int64_t m = 0;
  for (auto v : miss) m += v;
  if (qsimp_misses) *qsimp_misses = m;
  return 0;
}

// rep_draine on its own: n frequencies from row im of the Draine spectra,
// drawn from block 0 of generator 1 of (seed1, seed2).  Test infrastructure.
extern "C" int oracle_rep_draine(const mcrt_tables* tab, int32_t im, int64_t n, int32_t seed1, int32_t seed2,
                                 double* out) {
  if (!tab || !tab->draine || im < 1 || im > tab->nemit || tab->ndraine < 2 || !out) return MCRT_ERR_ARG;
  Rng rng = stream(seed1, seed2, 1, 0);
  for (int64_t i = 0; i < n; ++i) out[i] = rep_draine(tab, im, rng);
  return MCRT_OK;
}
