// mcrt_transport.cuh -- FP64 photon-packet transport kernel for sm_100a.
//
// One persistent kernel runs the whole packet life of the reference's loop
// `do iphot=1,np` (newdisktherm_5_fuv.f90:220-491): emission, the cell walk
// (tauint_3d_2_fuv.f90:5-210), interactions (propagate_5_fuv.f90:76-218),
// peel-off walks (peeloff_3d_2_test.f90:7-347) and the exit binning
// (propagate_5_fuv.f90:231-320).  Threads fetch packets from a global counter,
// so a lane whose packet leaves the grid early starts the next packet instead
// of idling behind a long-lived one.
//
// The arithmetic is written in the reference's operation order; compiled
// with --fmad=false the FP64 kernel performs the same IEEE operations as the
// CPU oracle, and differs from it only by the last-place behaviour of the
// transcendental functions (log, exp, sin, cos, acos, atan2, pow).
//
// Per-thread opacity state (kapd, albedo, g, pl of the species slots the
// model references) lives in shared memory, indexed [slot][thread], so the
// data-dependent slot lookups of a crossing do not spill to local memory.
#pragma once
#include "mcrt_device.cuh"

namespace mcrt {

constexpr double PI = 3.1415926535897932384626433;
constexpr double R2P = 2.0 * PI;
constexpr double RSOL = 6.9598e10;
constexpr double HUGE_D = 1.7976931348623157e308;
constexpr int kBlock = kTransportBlock;
// watchdog: a packet is killed after this many interactions in total (the
// reference only kills after 10000 in one cell, propagate_5_fuv.f90:208-213)
constexpr int64_t kMaxEvents = 100000000;
constexpr int kMaxAccTries = 1000000;   // accretion emission redraws before the packet is dropped

// --------------------------------------------------------------- RNG ----
struct Rng {
  int32_t s1, s2;
  int32_t ndraws;
  // random_large_integer (ecuyer_cote_mod.f90:252-293), Schrage steps
  __device__ __forceinline__ double ran() {
    int32_t k = s1 / 53668;
    s1 = 40014 * (s1 - k * 53668) - k * 12211;
    if (s1 < 0) s1 += 2147483563;
    k = s2 / 52774;
    s2 = 40692 * (s2 - k * 52774) - k * 3791;
    if (s2 < 0) s2 += 2147483399;
    int32_t z = s1 - s2;
    if (z < 1) z += 2147483562;
    ++ndraws;
    return (double)z * 4.656613057e-10;
  }
};

__device__ __forceinline__ int64_t mulmod(int64_t a, int64_t b, int64_t m) {
  return (int64_t)(((unsigned long long)a * (unsigned long long)b) % (unsigned long long)m);
}

// a*b mod m for 0 <= a, b < m < 2^31, exactly: the FP64 quotient estimate is
// within one of floor(a*b/m) (its relative error is ~3*2^-53 of a value
// below 2^31), and the remainder is corrected in exact 64-bit integers.
__device__ __forceinline__ int64_t mulmod31(int64_t a, int64_t b, int64_t mod, double inv) {
  const int64_t q = (int64_t)(__dmul_rn(__dmul_rn((double)a, (double)b), inv));
  int64_t r = a * b - q * mod;
  if (r < 0) r += mod;
  else if (r >= mod) r -= mod;
  return r;
}

// Block `b` of the generator seeded (g1,g2): a^(b*2^30) * g mod m
// (reinitialize_current_generator(1) b times).  Below 2^42 blocks: the
// three 14-bit digits of b index the tables A^(j*2^(14c)); otherwise the
// binary powers a^(2^30*2^k).  Exact modular arithmetic either way.
__device__ __forceinline__ Rng rng_block(const DevModel& m, int32_t g1, int32_t g2, int64_t b) {
  constexpr int64_t M1 = 2147483563, M2 = 2147483399;
  int64_t r1 = g1, r2 = g2;
  if (m.jdig1 && b >= 0 && b < ((int64_t)1 << (3 * kJumpBits))) {
    const double i1 = 1.0 / (double)M1, i2 = 1.0 / (double)M2;
    const int d0 = (int)(b & (kJumpDigit - 1)), d1 = (int)((b >> kJumpBits) & (kJumpDigit - 1));
    const int d2 = (int)(b >> (2 * kJumpBits));
    const int64_t a0 = __ldg(m.jdig1 + d0), a1 = __ldg(m.jdig1 + kJumpDigit + d1), a2 = __ldg(m.jdig1 + 2 * kJumpDigit + d2);
    const int64_t c0 = __ldg(m.jdig2 + d0), c1 = __ldg(m.jdig2 + kJumpDigit + d1), c2 = __ldg(m.jdig2 + 2 * kJumpDigit + d2);
    r1 = mulmod31(mulmod31(mulmod31(r1, a0, M1, i1), a1, M1, i1), a2, M1, i1);
    r2 = mulmod31(mulmod31(mulmod31(r2, c0, M2, i2), c1, M2, i2), c2, M2, i2);
  } else {
    for (int k = 0; b != 0; ++k, b >>= 1) {
      if (b & 1) {
        r1 = mulmod(r1, m.jump1[k], M1);
        r2 = mulmod(r2, m.jump2[k], M2);
      }
    }
  }
  Rng r;
  r.s1 = (int32_t)r1;
  r.s2 = (int32_t)r2;
  r.ndraws = 0;
  return r;
}

// ------------------------------------------------------------ helpers ---
__device__ __forceinline__ double chk(double x) { return x > 1.0 ? 1.0 : (x < -1.0 ? -1.0 : x); }

// locate (nr_2.f:131-154), 1-based result
__device__ __forceinline__ int locate(const double* xx, int n, double x) {
  int jl = 0, ju = n + 1;
  const bool asc = xx[n - 1] > xx[0];
  while (ju - jl > 1) {
    int jm = (ju + jl) >> 1;
    if (asc == (x > xx[jm - 1])) jl = jm; else ju = jm;
  }
  if (jl == 0 && x == xx[0]) jl = 1;
  return jl;
}

// closest_wall.f90 selector
struct Walls {
  double tn1, tp1, tp2;
  int ip1, ip2;
  __device__ __forceinline__ void reset() { tn1 = -HUGE_D; tp1 = HUGE_D; tp2 = HUGE_D; ip1 = 0; ip2 = 0; }
  __device__ __forceinline__ void insert(double t, int i) {
    if (t < 0.0) {
      if (t > tn1) tn1 = t;
    } else if (t < tp1) {
      tp2 = tp1; ip2 = ip1; tp1 = t; ip1 = i;
    } else if (t < tp2) {
      tp2 = t; ip2 = i;
    }
  }
  __device__ __forceinline__ void next(bool on_wall, double& t, int& i) const {
    if (on_wall && !(fabs(tn1) < fabs(tp1))) { t = tp2; i = ip2; }
    else { t = tp1; i = ip1; }
  }
};

#ifdef MCRT_MIXED
// --------------------------------------------------- FP32 cell walk ----
// The mixed build walks a ray in the closest-approach form: a point of the
// ray is c + q u, with c the point nearest the origin (c . u = 0) and q the
// signed distance from it.  Every face of the spherical-polar grid is then a
// root in q that depends on the ray and the wall only, never on the current
// position, so the on-wall cancellation of radface/thetaface/phiface
// (|x|^2 - R^2 -> 0 on the wall just crossed) does not arise:
//   sphere R:  q = +-sqrt(R^2 - p^2), p^2 = |c|^2 (inward half first);
//   cone mu:   (c_z + u_z q)^2 = mu^2 (p^2 + q^2) on the nappe sign(z) = sign(mu);
//   plane A x + B y = 0:  q = -(A c_x + B c_y) / (A u_x + B u_y).
// Each dimension's next crossing is kept and only the dimension just
// crossed is solved again, and the roots of the theta cell's two cones are
// kept too (a theta crossing shares one wall with the new cell), so a
// crossing costs one sphere root or one cone root.  The walk state, the
// cone and plane roots and the opacity sums are FP32.  q and p^2 are FP64,
// and so is every sphere root: an FP32 square root refined by one Newton
// step on the FP64 residual (R^2 - p^2 - s^2), accurate to ~1e-14 of the
// radius, which resolves the disk rim's refined cells (~1.6e-6 of their
// radius wide).  The cumulative optical depth, its comparison with the
// sampled tau and the tallies are FP64.
struct QRay {
  double q, p2, q0;            // current q, squared impact parameter, q of the walk's start point
  double qr, qt, qp;           // next crossing per dimension (r, theta, phi); HUGE_D: none
  float cx, cy, cz, ux, uy, uz, p2f, pabs;
  float ta1, ta2, tb1, tb2;    // roots of the theta cell's upper (t-1) and lower (t) cone; -inf: none
  int sr, st, sp;              // index step of the pending crossing per dimension
  int nphi;                    // phi crossings of this walk (a line turns by less than pi)
  bool lzpos;                  // the azimuth grows along the ray (L_z > 0)
};
#endif

// Shared per-thread species state: S[q][slot][tid], q = kapd, albedo, g,
// pl.  Kernels reserve a fifth column of kMaxSlot doubles per thread: the
// mixed build keeps the FP32 walk columns there (Packet::sfb).
constexpr int kSpecCols = 5;
struct SpecState {
  double* base;
  int tid;
  __device__ __forceinline__ double& kapd(int s) const { return base[(0 * kMaxSlot + s) * kBlock + tid]; }
  __device__ __forceinline__ double& alb(int s) const { return base[(1 * kMaxSlot + s) * kBlock + tid]; }
  __device__ __forceinline__ double& g(int s) const { return base[(2 * kMaxSlot + s) * kBlock + tid]; }
  __device__ __forceinline__ double& pl(int s) const { return base[(3 * kMaxSlot + s) * kBlock + tid]; }
};

enum KapdOrder { KAPD_DISK = 0, KAPD_PROPAGATE = 1, KAPD_TAUINT = 2 };

// Filter-band images (peeloff_3d_2_test.f90:242-285) of one peel-off that
// reached image coordinates (vx, vy) (pixel units from the image corner):
// freq = 2.9979e14 / wave with wave = 1.2398 / nub, as the reference forms
// them; every filter whose open range (filtwave(1), filtwave(nf)) holds freq
// adds the Stokes vector times filtphi(iw), iw the last point below freq
// (the reference's linear scan; a binary search finds the same point on a
// non-decreasing curve), and Stokes I to the image of the packet's origin
// (i_orig 1 star, 2 disk, 3 envelope, 4 outflow).
__device__ __forceinline__ void bin_filters(const DevModel& m, const DevTallies& T, int id, double vx, double vy,
                                            double nub, int i_orig, double qi, double qq, double qu, double qv) {
  if (!m.output_imfilt || !(vx > -1.0e9 && vx < 1.0e9 && vy > -1.0e9 && vy < 1.0e9)) return;
  const int ix = (int)vx + 1, iy = (int)vy + 1;
  if (ix > m.nxhst || iy > m.nxhst || ix <= 0 || iy <= 0) return;
  const double wave = 1.2398 / nub;
  const double freq = 2.9979e14 / wave;
  const int oi = i_orig == 1 ? 5 : (i_orig == 2 ? 4 : (i_orig == 3 ? 6 : (i_orig == 4 ? 7 : -1)));
  for (int f = 0; f < m.nfilt; ++f) {
    const int nf = __ldg(m.nfpts + f);
    const double* fw = m.filtwave + (int64_t)m.nwfiltmax * f;
    if (!(freq > __ldg(fw) && freq < __ldg(fw + nf - 1))) continue;
    int lo = 0, hi = nf - 1;                 // first point with fw >= freq lies in (0, nf-1]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(fw + mid) >= freq) hi = mid; else lo = mid;
    }
    const double wt = __ldg(m.filtphi + (int64_t)m.nwfiltmax * f + hi - 1);
    const int64_t k = (int64_t)(id - 1) + (int64_t)m.npeel * ((ix - 1) + (int64_t)m.nxhst * ((iy - 1) + (int64_t)m.nxhst * f));
    atomicAdd(T.imgb + k, qi * wt);
    atomicAdd(T.imgb + m.nimgb + k, qq * wt);
    atomicAdd(T.imgb + 2 * m.nimgb + k, qu * wt);
    atomicAdd(T.imgb + 3 * m.nimgb + k, qv * wt);
    if (oi >= 0) atomicAdd(T.imgb + oi * m.nimgb + k, qi * wt);
  }
}

// math_binning.f90 ipos_sp / locate_sp in single precision, each rounding
// explicit so that the bins are the reference's bit for bit.
__device__ __forceinline__ int ipos_sp(float xmin, float xmax, float x, int nbin) {
  if (xmax > xmin) {
    if (x < xmin) return 0;
    if (x > xmax) return nbin + 1;
  } else {
    if (x < xmax) return 0;
    if (x > xmin) return nbin + 1;
  }
  const float frac = __fdiv_rn(__fsub_rn(x, xmin), __fsub_rn(xmax, xmin));
  return (int)__fmul_rn(frac, (float)nbin) + 1;
}
__device__ __forceinline__ int locate_sp(const float* xx, int n, float x) {
  const bool ascnd = __ldg(xx + n - 1) >= __ldg(xx);
  int jl = 0, ju = n + 1;
  while (ju - jl > 1) {
    const int jm = (ju + jl) >> 1;
    if (ascnd == (x >= __ldg(xx + jm - 1))) jl = jm; else ju = jm;
  }
  if (x == __ldg(xx)) return 1;
  if (x == __ldg(xx + n - 1)) return n - 1;
  if (x > __ldg(xx + n - 1) || x < __ldg(xx)) return -1;
  return jl;
}

// Nested multi-wavelength images (peeloff_3d_2_test.f90:302-309 calling
// nested_image_bin, type_nested_image.f90:75-101) of one peel-off at image
// position (ximage, yimage): position and log10(frequency) in single
// precision as the reference passes them; the level is the smallest whose
// half size exceeds max(|x|,|y|); the four Stokes images share the pixel.
// A pixel beyond the image (a position exactly on a level's edge, where
// ipos gives dim+1) is dropped.
__device__ __forceinline__ void bin_nested(const DevModel& m, const DevTallies& T, int id, double ximage,
                                           double yimage, double nub, double qi, double qq, double qu, double qv) {
  if (!m.output_imsparse) return;
  const float xr = (float)ximage, yr = (float)yimage;
  const float* lev = m.sparse_levels;
  const int nl = m.sparse_nlev;
  const float r = fmaxf(fabsf(xr), fabsf(yr));
  if (r > __ldg(lev + nl - 1)) return;
  int l = locate_sp(lev, nl, r);
  l = (l < 0) ? 1 : min(l + 1, nl);     // a single level met exactly at its edge stays that level
  const float h = __ldg(lev + l - 1);
  const int ix = ipos_sp(-h, h, xr, m.sparse_dim), iy = ipos_sp(-h, h, yr, m.sparse_dim);
  const float lnu = (float)log10(2.9979e14 / (1.2398 / nub));
  const int inu = ipos_sp(m.sparse_lognu_min, m.sparse_lognu_max, lnu, m.sparse_nnu);
  if (inu < 1 || inu > m.sparse_nnu || ix < 1 || ix > m.sparse_dim || iy < 1 || iy > m.sparse_dim) return;
  const int64_t k = (int64_t)(ix - 1) + (int64_t)m.sparse_dim * ((iy - 1) + (int64_t)m.sparse_dim *
                    ((inu - 1) + (int64_t)m.sparse_nnu * ((l - 1) + (int64_t)nl * (id - 1))));
  atomicAdd(T.ims + k, qi);
  atomicAdd(T.ims + m.nims + k, qq);
  atomicAdd(T.ims + 2 * m.nims + k, qu);
  atomicAdd(T.ims + 3 * m.nims + k, qv);
}

struct Packet {
  const DevModel& m;
  const DevTallies& T;
  SpecState sp;
  Rng rng;
  double xp, yp, zp, rsq, rtot, ux, uy, uz, tau;
  double cost, sint, cosp, sinp, phi, sip, sqp, sup, svp, nub, ifuv;
  double cosb, sinb, lp;
  int ir, it, ip;
  bool on_wall;
  int iflag, i_orig, exitflag;
  int nscat, nabsev, ncross, nstar, ndiffev;
  unsigned long long c_cross, c_peel, c_pcross, c_pbin, c_reset;
  bool spec_dirty = false;      // opacset rewrote the species columns (the wavefront event kernel saves them then)

  // sbase: kSpecCols columns of kMaxSlot doubles per thread (the species
  // state and, in the mixed build, the FP32 walk columns in the last one);
  // fbase, if given, holds the FP32 walk columns instead.
  __device__ Packet(const DevModel& mm, const DevTallies& tt, double* sbase, float* fbase = nullptr)
      : m(mm), T(tt) {
    sp.base = sbase;
    sp.tid = threadIdx.x;
    c_cross = c_peel = c_pcross = c_pbin = c_reset = 0;
#ifdef MCRT_MIXED
    sfb = fbase ? fbase : reinterpret_cast<float*>(sbase + 4 * kMaxSlot * kBlock);
#else
    (void)fbase;
#endif
  }

  __device__ __forceinline__ double ran() { return rng.ran(); }

  // opacset (dust_5.f90:9-109) for the referenced species, then kapd with
  // the association order of the calling site.
  // opacset (dust_5.f90:9-55) for the species of every slot.  Slots whose
  // species share a wavelength column (slot_grid) reuse the bracket and the
  // interpolation weight of the first such slot: the same search over the
  // same values gives the same result.
  __device__ void opacset(double nu, int order) {
    spec_dirty = true;
    int a = 0, b = 0, have = -1;
    double f = 0.0;
    for (int s = 0; s < m.nslot; ++s) {
      const int id = m.slot_species[s] - 1;
      const int nl = m.nlammax;
      if (m.slot_grid[s] != have) {
        const double* nud = m.nudust + (int64_t)nl * id;
        const int n = m.nlambda[id];
        if (nu >= __ldg(nud)) { a = 0; b = 0; f = 0.0; }
        else if (nu <= __ldg(nud + n - 1)) { a = n - 1; b = n - 1; f = 0.0; }
        else {
          int i0 = 1, i1 = n;
          while (i1 - i0 > 1) {
            int i = (i1 + i0) >> 1;
            if (nu <= __ldg(nud + i - 1)) i0 = i; else i1 = i;
          }
          a = i1 - 1; b = i0 - 1;
          f = (nu - __ldg(nud + a)) / (__ldg(nud + b) - __ldg(nud + a));
        }
        have = m.slot_grid[s];
      }
      const double* kd = m.kappad + (int64_t)nl * id;
      const double* ad = m.adust + (int64_t)nl * id;
      const double* gd = m.gdust + (int64_t)nl * id;
      const double* pd = m.pldust + (int64_t)nl * id;
      double kap, alb, gg, pll;
      if (a == b) {
        kap = __ldg(kd + a); alb = __ldg(ad + a); gg = __ldg(gd + a); pll = __ldg(pd + a);
      } else {
        const double fm1 = 1.0 - f;
        gg = fm1 * __ldg(gd + a) + f * __ldg(gd + b);
        pll = fm1 * __ldg(pd + a) + f * __ldg(pd + b);
        kap = fm1 * __ldg(kd + a) + f * __ldg(kd + b);
        alb = fm1 * __ldg(ad + a) + f * __ldg(ad + b);
      }
      const double kv = __ldg(m.kappav + id);
      double kd_;
      if (order == KAPD_DISK) kd_ = kap * m.rmincgs * kv;
      else if (order == KAPD_PROPAGATE) kd_ = kap * m.rstar * RSOL * kv;
      else kd_ = kap * RSOL * m.rstar * kv;
      sp.kapd(s) = kd_;
      sp.alb(s) = alb;
      sp.g(s) = gg;
      sp.pl(s) = pll;
    }
  }

  __device__ __forceinline__ static bool is_fuv(double nu) { return nu <= 13.6 && nu >= 6.0; }

  // ------------------------------------------------------ frequencies
  __device__ double bbfreq(double teff) {          // random.f90:197-225
    double z0 = __ldg(m.inczeta + MCRT_IZMAX - 1) * ran();
    double z1 = ran(), z2 = ran(), z3 = ran(), z4 = ran();
    int i = 1;
    while (z0 > __ldg(m.inczeta + i - 1)) ++i;
    return -log(z1 * z2 * z3 * z4) * teff / (double)i;
  }
  __device__ double atmosfreq() {                  // starbarb_2.f90:124-153
    double xi = ran();
    int i = locate(m.hnuint, m.nhnu, xi);
    i = min(max(i, 1), m.nhnu - 1);   // a CDF that does not span [0,1) cannot index outside the table
    if (i > 1) {
      double logatm = m.lognu[i - 1] + (m.lognu[i] - m.lognu[i - 1]) / (m.loghnu[i] - m.loghnu[i - 1]) *
                                           (log10(xi) - m.loghnu[i - 1]);
      return pow(10.0, logatm);
    }
    return m.atmosnu[i - 1] + (m.atmosnu[i] - m.atmosnu[i - 1]) / (m.hnuint[i] - m.hnuint[i - 1]) * (xi - m.hnuint[i - 1]);
  }
  __device__ double lucydustfreq(double T0, int idust2) {   // lucydustfreq_2_test.f90:19-160
    const int nT = m.nT, nnu = m.nnu;
    const double Tmax = 199999.0;
    if (T0 >= Tmax / 11605.0) return bbfreq(T0);
    double lT0 = log(T0);
    double xi = ran();
    const double l1 = __ldg(m.lTint), ln = __ldg(m.lTint + nT - 1);
    int j = (int)((double)(nT - 1) * (lT0 - l1) / (ln - l1)) + 1;
    j = min(max(j, 1), nT - 1);
    double f = (lT0 - __ldg(m.lTint + j - 1)) / (__ldg(m.lTint + j) - __ldg(m.lTint + j - 1));
    if (f < 0.0) f = 0.0;
    if (f > 1.0) f = 1.0;
    const double* K = m.kapint + (int64_t)nT * nnu * (idust2 - 1);
    auto kap = [&](int jj, int ii) { return __ldg(K + (jj - 1) + (int64_t)nT * (ii - 1)); };
    int i0 = 1, i1 = nnu;
    double P0 = (1.0 - f) * kap(j, i0) + f * kap(j + 1, i0);
    if (xi < P0) {
      if (P0 > 0.0) return T0 * xi * __ldg(m.nuint) / P0;
      return T0 * __ldg(m.nuint);
    }
    double P1 = (1.0 - f) * kap(j, i1) + f * kap(j + 1, i1);
    if (P1 > 1.0) P1 = 1.0;
    if (xi >= P1) {
      if (P1 < 1.0 && xi < 1.0) return T0 * __ldg(m.nuint + nnu - 1) * (1.0 - P1) / (1.0 - xi);
      return T0 * __ldg(m.nuint + nnu - 1);
    }
    while (i1 - i0 > 1) {
      int i = (i0 + i1) >> 1;
      double P = (1.0 - f) * kap(j, i) + f * kap(j + 1, i);
      if (P > 1.0) P = 1.0;
      if (P < P0) { P0 = P; i0 = i; }
      if (P > P1) { P1 = P; i1 = 1; }
      if (P > xi) { i1 = i; P1 = P; } else { i0 = i; P0 = P; }
    }
    if (xi < P0) f = 0.0;
    else if (xi > P1) f = 1.0;
    else if (P0 <= 0.0) f = 0.5;
    else if (P1 <= 0.0 || xi <= 0.0) { }
    else f = log(xi / P0) / log(P1 / P0);
    return T0 * __ldg(m.nuint + i0 - 1) * pow(__ldg(m.nuint + i1 - 1) / __ldg(m.nuint + i0 - 1), f);
  }

  // ---------------------------------------------------------- emission
  __device__ void initp_sample() {                 // initp_common.f90:1-29
    if (m.limb == 0) {
      cost = sqrt(ran());
    } else {                                       // samptabl.f90:29-65
      double xr = ran();
      int n = min(max(locate(m.limb_prob, 100, xr), 1), 99);
      const double delmu = 1.0 / 100.0;
      double xmu1 = delmu * (double)(n + 1);
      cost = xmu1 - (m.limb_prob[n] - xr) / (m.limb_prob[n] - m.limb_prob[n - 1]) * delmu;
    }
    sint = sqrt(1.0 - cost * cost);
    phi = R2P * ran();
    cosp = cos(phi);
    sinp = sin(phi);
  }
  __device__ void initp_transform() {              // initp_common.f90:31-94
    if (fabs(cosb) < 0.9999999) {
      double costi = cost * cosb - sint * sinb * cosp;
      if (fabs(costi) > 1.0) {
        if (costi > 1.0) costi = 1.0;
        if (cost < -1.0) costi = -1.0;
      }
      double sinti = sqrt(1.0 - costi * costi);
      double phinew;
      if (sinti > 0.0000001) {
        double cospn = (cost - costi * cosb) / (sinti * sinb);
        if (fabs(cospn) > 1.0) cospn = (cospn < 0.0) ? -1.0 : 1.0;
        if (phi < PI) {
          phinew = acos(cospn);
          if (phinew > PI) phinew = PI;
        } else {
          phinew = R2P - acos(cospn);
          if (phinew < PI) phinew = PI;
        }
      } else {
        phinew = 0.0;
      }
      phi = phinew;
      cost = costi;
      sint = sinti;
    } else if (cosb < 0.0) {
      cost = -cost;
    }
    phi = phi + lp;
    if (phi > R2P) phi = phi - R2P;
    if (phi < 0.0) phi = phi + R2P;
    sinp = sin(phi);
    cosp = cos(phi);
  }
  __device__ void initpspot(int ispotph) {         // initpspot.f90:3-175
    sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
    for (;;) {
      for (;;) {
        double xr = ran();
        cosb = 1.0 - 2.0 * xr;
        sinb = sqrt(1.0 - cosb * cosb);
        if (cosb != 0.0 && fabs(cosb) < 1.0) break;
      }
      lp = R2P * ran();
      if (m.ispot == 1) {
        double cphi = cos(lp), sphi = sin(lp);
        double dotsp1 = m.scspot1 * sinb * cphi + m.ssspot1 * sinb * sphi + m.cspot1 * cosb;
        double dotsp2 = m.scspot2 * sinb * cphi + m.ssspot2 * sinb * sphi + m.cspot2 * cosb;
        if (m.nspot == 1) {
          if (ispotph == 1 && dotsp1 < m.csprad) continue;
        } else {
          if (ispotph == 1 && dotsp1 < m.csprad && dotsp2 < m.csprad) continue;
        }
        if (m.fspot < 1.0) {
          double dellon = (lp < PI) ? lp : R2P - lp;
          double costhp = m.cspot1 * cosb + m.sspot1 * sinb * cos(dellon);
          if (costhp > m.csprad) ispotph = 1;
          if (m.nspot == 2) {
            dellon = (lp < PI) ? PI - lp : lp - PI;
            costhp = m.cspot2 * cosb + m.sspot2 * sinb * cos(dellon);
            if (costhp > m.csprad) ispotph = 1;
          }
        }
      }
      break;
    }
    initp_sample();
    initp_transform();
    if (m.fspot == 1.0) nub = (m.iplanckst == 0) ? atmosfreq() : bbfreq(m.tshock);
    else if (ispotph == 0) nub = (m.iplanckst == 0) ? atmosfreq() : bbfreq(m.tstar);
    else nub = bbfreq(m.tshock);
  }
  __device__ void initp_ps(int ispotph) {          // initp_ps (initp_common.f90 family)
    sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
    for (;;) {
      double xr = ran();
      cosb = chk(1.0 - 2.0 * xr);
      sinb = chk(sqrt(1.0 - cosb * cosb));
      if (cosb != 0.0) break;
    }
    cost = cosb;
    sint = sinb;
    lp = R2P * ran();
    phi = lp;
    sinp = chk(sin(phi));
    cosp = chk(cos(phi));
    if (ispotph == 0) nub = (m.iplanckst == 0) ? atmosfreq() : bbfreq(m.tstar);
    else nub = bbfreq(m.tshock);
  }
  // External illumination (initpout.f90:1-68): an unpolarised packet on the
  // sphere of the grid's outer radius (cosb uniform, longitude lp uniform),
  // heading inward with cos(theta) = -xi in the local frame (isotropic in a
  // volume), rotated to the grid frame by initp_transform; the frequency
  // from the ISRF table (rep_isrf.f90: locate in the cdf, then linear in
  // log10 cdf and log10 nu between the bracketing rows).
  __device__ void initpout() {
    sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
    double xran = ran();
    cosb = 1.0 - 2.0 * xran;
    sinb = sqrt(1.0 - cosb * cosb);
    xran = ran();
    cost = -xran;
    sint = sqrt(1.0 - cost * cost);
    xran = ran();
    phi = R2P * xran;
    cosp = cos(phi);
    sinp = sin(phi);
    xran = ran();
    lp = R2P * xran;
    initp_transform();
    xran = ran();
    const int n = m.nisrf;
    int i = locate(m.isrf_cdf, n, xran);
    if (i == n) i = n - 1;
    if (i == 0) i = 1;
    const double* lc = m.isrf_logcdf;
    const double* lf = m.isrf_logfreq;
    const double lg = lf[i - 1] + (log10(xran) - lc[i - 1]) / (lc[i] - lc[i - 1]) * (lf[i] - lf[i - 1]);
    nub = pow(10.0, lg);
  }

  // Small-grain re-emission frequency (rep_draine_new.f90): locate3 in row
  // im of the cumulative spectra (bisection over the columns, in the
  // direction the row runs), then linear in log10 cdf and log10 nu between
  // the bracketing columns.
  __device__ double rep_draine(int im) {
    const double xran = ran();
    const int ne = m.nemit, nd = m.ndraine;
    const double* cd = m.draine_cdf + (im - 1);
    auto cdf = [&](int j) { return __ldg(cd + (int64_t)(j - 1) * ne); };
    const bool asc = cdf(nd) > cdf(1);
    int jl = 0, ju = nd + 1;
    while (ju - jl > 1) {
      const int jm = (ju + jl) >> 1;
      if (asc == (xran > cdf(jm))) jl = jm; else ju = jm;
    }
    int i = jl;
    if (i == nd) i = i - 1;
    if (i == 0) i = 1;
    const double* lc = m.draine_logcdf + (im - 1);
    const double* lf = m.draine_logfreq;
    const double c0 = __ldg(lc + (int64_t)(i - 1) * ne), c1 = __ldg(lc + (int64_t)i * ne);
    const double lg = (log10(xran) - c0) / (c1 - c0) * (__ldg(lf + i) - __ldg(lf + i - 1)) + __ldg(lf + i - 1);
    return pow(10.0, lg);
  }

  __device__ void initpabs() {                     // initpabs.f90:1-44
    sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
    cosb = zp / rtot;
    sinb = sqrt(1.0 - cosb * cosb);
    lp = atan2(yp, xp);
    initp_sample();
    initp_transform();
    ux = sint * cosp;
    uy = sint * sinp;
    uz = cost;
    nub = atmosfreq();
  }

  // -------------------------------------------------------------- grid
  // testgrid.f90:1-128 (the FP64 walk).  For npg == 2 the phi checks can
  // never fire (phi in [0,2pi) against phiarr = [0,2pi]), so atan2 is only
  // evaluated when a re-location needs it.
  __device__ void testgrid(double& x, double& y, double& z, double& rs, double& rt, int& r, int& t, int& p, bool& onw) {
    const int nrg = m.nrg, ntg = m.ntg, npg = m.npg;
    const double tol = 1.0e-4;
    const double* r2 = m.r2arr;
    const double* ca = m.costarr;
    const double* pa = m.phiarr;
    double cb = chk(z / rt);
    const bool need_phi = npg > 2;
    double ph = 0.0;
    if (need_phi) {
      ph = atan2(y, x);
      if (ph < 0.0) ph = ph + R2P;
    }
    bool reset = false;
    if ((rs - __ldg(r2)) / (__ldg(r2 + 1) - __ldg(r2)) < -tol ||
        (rs - __ldg(r2 + nrg - 2)) / (__ldg(r2 + nrg - 1) - __ldg(r2 + nrg - 2)) > 1.0 + tol) {
      const double third = (double)(1.0f / 3.0f);
      const double r1 = m.rarr[0], rn = m.rarr[nrg - 1];
      rt = pow(ran() * (pow(rn, 3.0) - pow(r1, 3.0)) + pow(r1, 3.0), third);
      reset = true;
    }
    if ((cb - __ldg(ca)) / (__ldg(ca + 1) - __ldg(ca)) < -tol ||
        (cb - __ldg(ca + ntg - 2)) / (__ldg(ca + ntg - 1) - __ldg(ca + ntg - 2)) > 1.0 + tol) {
      cb = ran() * (__ldg(ca + ntg - 1) - __ldg(ca)) + __ldg(ca);
      reset = true;
    }
    if (need_phi && ((ph - pa[0]) / (pa[1] - pa[0]) < -tol || (ph - pa[npg - 2]) / (pa[npg - 1] - pa[npg - 2]) > 1.0 + tol)) {
      ph = ran() * (pa[npg - 1] - pa[0]) + pa[0];
      reset = true;
    }
    if (reset) {
      if (!need_phi) {
        ph = atan2(y, x);
        if (ph < 0.0) ph = ph + R2P;
      }
      double s = sqrt(1.0 - cb * cb);
      x = rt * s * cos(ph);
      y = rt * s * sin(ph);
      z = rt * cb;
      rs = rt * rt;
      onw = false;
      ++c_reset;
    }
    if (r < 1 || r > nrg) r = locate(r2, nrg, rs);
    if (t < 1 || t > ntg) t = locate(ca, ntg, cb);
    if (p < 1 || p > npg) {
      if (!need_phi) { ph = atan2(y, x); if (ph < 0.0) ph = ph + R2P; }
      p = locate(pa, npg, ph);
    }
    const double rfrac = (rs - __ldg(r2 + r - 1)) / (__ldg(r2 + r) - __ldg(r2 + r - 1));
    const double tfrac = (cb - __ldg(ca + t - 1)) / (__ldg(ca + t) - __ldg(ca + t - 1));
    bool phierr = false;
    if (need_phi) {
      const double pfrac = (ph - pa[p - 1]) / (pa[p] - pa[p - 1]);
      if (pfrac < -tol || pfrac > 1.0 + tol) {
        double d1 = ph - pa[p - 1];
        if (d1 > PI) d1 -= R2P;
        if (d1 < -PI) d1 += R2P;
        double d2 = ph - pa[p];
        if (d2 > PI) d2 -= R2P;
        if (d2 < -PI) d2 += R2P;
        phierr = fabs(d1) > tol && fabs(d2) > tol;
      }
    }
    if (rfrac < -tol || rfrac > 1.0 + tol) r = locate(r2, nrg, rs);
    if (tfrac < -tol || tfrac > 1.0 + tol) t = locate(ca, ntg, cb);
    if (phierr) p = locate(pa, npg, ph);
  }

  // radface / thetaface / phiface (radface.f90, thetaface.f90, phiface.f90)
  __device__ __forceinline__ void faces(Walls& w, double vx, double vy, double vz, double x, double y, double z,
                                        int r, int t, int p) const {
    const double bb = 2.0 * (x * vx + y * vy + vz * z);
    const double rr = x * x + y * y + z * z;
    double cc = rr - __ldg(m.r2arr + r - 1);
    double descr = bb * bb - 4.0 * cc;
    if (descr > 0.0) {
      descr = sqrt(descr);
      w.insert((-bb + descr) * 0.5, 1);
      w.insert((-bb - descr) * 0.5, 1);
    }
    cc = rr - __ldg(m.r2arr + r);
    descr = bb * bb - 4.0 * cc;
    if (descr > 0.0) {
      descr = sqrt(descr);
      w.insert((-bb + descr) * 0.5, 2);
      w.insert((-bb - descr) * 0.5, 2);
    }
    if (m.ntg > 2) {
      const double t1 = __ldg(m.tan2arr + t - 1), t2 = __ldg(m.tan2arr + t);
      const double tmp1 = x * vx + y * vy, tmp2 = vx * vx + vy * vy, tmp3 = x * x + y * y;
      double ta, tb;
      int i1, i2;
      if (t2 < t1) { ta = t2; tb = t1; i1 = 4; i2 = 3; }
      else { ta = t1; tb = t2; i1 = 3; i2 = 4; }
      if (ta < 0.0) {
        if (vz != 0.0) w.insert(-z / vz, i1);
      } else {
        const double b2 = 2.0 * (tmp1 - ta * vz * z);
        const double aa = tmp2 - ta * vz * vz;
        const double c2 = tmp3 - z * z * ta;
        if (fabs(aa) > 1.0e-10) {
          double d = b2 * b2 - 4.0 * aa * c2;
          if (d > 0.0 && ta != 0.0) {
            d = sqrt(d);
            w.insert((-b2 + d) * 0.5 / aa, i1);
            w.insert((-b2 - d) * 0.5 / aa, i1);
          }
        } else if (fabs(b2) > 1.0e-10) {
          w.insert(-c2 / b2, i1);
        }
      }
      const double b2 = 2.0 * (tmp1 - tb * vz * z);
      const double aa = tmp2 - tb * vz * vz;
      const double c2 = tmp3 - z * z * tb;
      if (fabs(aa) > 1.0e-10) {
        double d = b2 * b2 - 4.0 * aa * c2;
        if (d > 0.0 && tb != 0.0) {
          d = sqrt(d);
          w.insert((-b2 + d) * 0.5 / aa, i2);
          w.insert((-b2 - d) * 0.5 / aa, i2);
        }
      } else if (fabs(b2) > 1.0e-10) {
        w.insert(-c2 / b2, i2);
      }
    }
    if (m.npg > 2 && m.ntg > 2) {
      const double A1 = __ldg(m.aarr + p - 1), B1 = __ldg(m.barr + p - 1);
      const double A2 = __ldg(m.aarr + p), B2 = __ldg(m.barr + p);
      const double d1 = (A1 * vx + B1 * vy + 0.0 * vz);
      if (d1 != 0.0) w.insert(-(A1 * x + B1 * y + 0.0 * z + 0.0) / d1, 5);
      const double d2 = (A2 * vx + B2 * vy + 0.0 * vz);
      if (d2 != 0.0) w.insert(-(A2 * x + B2 * y + 0.0 * z + 0.0) / d2, 6);
    }
  }

  __device__ __forceinline__ int64_t cidx(int r, int t, int p) const {
    return (int64_t)(r - 1) + (int64_t)m.nrg * ((t - 1) + (int64_t)m.ntg * (p - 1));
  }

  __device__ __forceinline__ double cell_opac(const CellRec& c) const {   // tauint_3d_2_fuv.f90:59-65
    const int n = cell_n(c.meta);
    double opac = 0.0;
    for (int k = 0; k < n; ++k) opac = opac + sp.kapd(cell_slot(c.meta, k)) * c.rho[k];
    return opac;
  }

  __device__ __forceinline__ void tally_abs(int64_t ci, const CellRec& c, double len) {  // tauint_3d_2_fuv.f90:83-98
    const int n = cell_n(c.meta);
    double add = 0.0;
    bool any = false;
    for (int k = 0; k < n; ++k) {
      const int id = cell_id(c.meta, k);
      if (id >= 5 && id <= 8) continue;     // is_sg
      const int s = cell_slot(c.meta, k);
      const double v = len * sp.kapd(s) * c.rho[k] * (1.0 - sp.alb(s));
      add = any ? add + v : v;
      any = true;
    }
    if (any) atomicAdd(T.dtauabs + ci, add);
    if (m.iffuv) atomicAdd(T.fuvmean + ci, len * (m.rstar * RSOL) * ifuv / __ldg(m.vcell + ci));
  }

  __device__ __forceinline__ void step_index(int iface, int& r, int& t, int& p) const {
    switch (iface) {
      case 1: r = r - 1; break;
      case 2: r = r + 1; break;
      case 3: t = t - 1; break;
      case 4: t = t + 1; break;
      case 5: p = p - 1; break;
      default: p = p + 1; break;
    }
    if (p == 0) p = m.npg - 1;
    if (p == m.npg) p = 1;
  }

#ifndef MCRT_TALLY_WARP_AGG
#define MCRT_TALLY_WARP_AGG 0
#endif
#ifdef MCRT_MIXED
  // ------------------------------------------------ FP32 walk (QRay)
  // FP32 opacity columns of the walk: kapd and kapd*(1-albedo) per slot.
  float* sfb = nullptr;                                  // [2][kMaxSlot][kBlock] in shared memory
  __device__ __forceinline__ float& kf(int s) const { return sfb[s * kBlock + threadIdx.x]; }
  __device__ __forceinline__ float& kaf(int s) const { return sfb[(kMaxSlot + s) * kBlock + threadIdx.x]; }
  __device__ __forceinline__ void walk_columns() {
    for (int s = 0; s < m.nslot; ++s) {
      kf(s) = (float)sp.kapd(s);
      kaf(s) = (float)__dmul_rn(sp.kapd(s), __dsub_rn(1.0, sp.alb(s)));
    }
  }
  // Opacity and thermal absorption coefficient of a cell at the walk's
  // frequency (tauint_3d_2_fuv.f90:59-65, :83-90; small grains, ids 5-8,
  // take no part in the absorption tally).
  __device__ __forceinline__ void cell_coefs(const CellRecF& c, float& opac, float& absc) const {
    const int n = cell_n(c.meta);
    opac = 0.0f;
    absc = 0.0f;
    for (int k = 0; k < n; ++k) {
      const int s = cell_slot(c.meta, k);
      opac = __fmaf_rn(kf(s), c.rho[k], opac);
      const int id = cell_id(c.meta, k);
      if (id < 5 || id > 8) absc = __fmaf_rn(kaf(s), c.rho[k], absc);
    }
  }
  __device__ __forceinline__ void tally_absf(int64_t ci, float absc, double len) {
#if MCRT_TALLY_WARP_AGG
    // Lanes of the warp that tally the same cell add their pieces first and
    // one of them issues the atomic (the sum order differs from one atomic
    // per lane only in rounding).
    const double v = absc > 0.0f ? __dmul_rn(len, (double)absc) : 0.0;
    const unsigned grp = __match_any_sync(__activemask(), (unsigned long long)ci);
    const int lane = threadIdx.x & 31;
    if (grp == (1u << lane)) {
      if (v != 0.0) atomicAdd(T.dtauabs + ci, v);
    } else {
      double sum = 0.0;
      for (unsigned b = grp; b; b &= b - 1u) sum = __dadd_rn(sum, __shfl_sync(grp, v, __ffs(b) - 1));
      if (lane == __ffs(grp) - 1 && sum != 0.0) atomicAdd(T.dtauabs + ci, sum);
    }
#else
    if (absc > 0.0f) atomicAdd(T.dtauabs + ci, __dmul_rn(len, (double)absc));
#endif
    if (m.iffuv) atomicAdd(T.fuvmean + ci, len * (m.rstar * RSOL) * ifuv / __ldg(m.vcell + ci));
  }

  // Next sphere crossing of cell r: the inner wall while the ray still
  // approaches the origin (q < 0) and passes inside it, else the outer wall.
  // sqrt(R^2 - p^2): an FP32 reciprocal-square-root seed and one Newton step
  // on the FP64 residual, the same instructions for every wall.
  __device__ __forceinline__ void qnext_r(QRay& g, int r) const {
    const double a2 = __ldg(m.r2arr + r - 1);
    const bool inner = g.q < 0.0 && g.p2 < a2;
    const double d = fmax(__dsub_rn(inner ? a2 : __ldg(m.r2arr + r), g.p2), 0.0);
    const float df = (float)d;
    double s = 0.0;
    if (df > 0.0f) {
      const float s0 = __fmul_rn(df, rsqrtf(df));
      s = (double)s0;
      s = __dadd_rn(s, (double)__fmul_rn((float)__fma_rn(-s, s, d), __fdividef(0.5f, s0)));
    }
    g.qr = inner ? -s : s;
    g.sr = inner ? -1 : 1;
  }

  // Roots of cone wall w on its own nappe (-inf: none).
  __device__ __forceinline__ void cone_roots(const QRay& g, int w, float& q1, float& q2) const {
    const float2 c = __ldg(m.tcone + w);
    q1 = -HUGE_VALF;
    q2 = -HUGE_VALF;
    if (c.y > 1.5f) return;                               // pole (tan2arr = 0): never crossed
    if (c.y < 0.0f) {                                     // the theta = 90 deg plane z = 0
      if (g.uz != 0.0f) q1 = -__fdividef(g.cz, g.uz);
      return;
    }
    const float A = __fmaf_rn(g.uz, g.uz, -c.y);
    const float B = __fmul_rn(g.cz, g.uz);
    const float cz2 = __fmul_rn(g.cz, g.cz);
    const float D = __fmaf_rn(g.p2f, A, cz2);             // discriminant / mu^2
    if (!(D > 0.0f)) return;
    const float sq = __fmul_rn(fabsf(c.x), __fmul_rn(D, rsqrtf(D)));
    const float den = B >= 0.0f ? __fsub_rn(-B, sq) : __fsub_rn(sq, B);   // no cancellation
    const float C = __fmaf_rn(-c.y, g.p2f, cz2);
    const float r1 = __fdividef(den, A), r2 = __fdividef(C, den);
    // a root on the other nappe (z of opposite sign to mu) is not this wall
    if (__fmul_rn(__fmaf_rn(g.uz, r1, g.cz), c.x) > 0.0f) q1 = r1;
    if (__fmul_rn(__fmaf_rn(g.uz, r2, g.cz), c.x) > 0.0f) q2 = r2;
  }

  // Next cone crossing from the cached roots.  A root within `win` of the
  // current point counts only if the ray moves towards that wall there
  // (mu grows toward the upper wall), which settles the crossings that FP32
  // rounding cannot order, such as the wall a walk starts next to or has
  // just crossed.
  __device__ __forceinline__ void qpick_t(QRay& g) const {
    const float qf = (float)g.q;
    const float win = __fmul_rn(1.0e-5f, __fadd_rn(fabsf(qf), g.pabs));
    const float dmu = __fmaf_rn(g.uz, g.p2f, -__fmul_rn(g.cz, qf));   // d mu / dq has this sign
    const bool up = dmu > 0.0f, down = dmu < 0.0f;
    float best = HUGE_VALF;
    int st = 0;
    auto take = [&](float qi, bool toward, int step) {
      const bool ok = qi > qf + win || (qi >= qf - win && toward);
      if (ok && qi < best) { best = qi; st = step; }
    };
    take(g.ta1, up, -1);
    take(g.ta2, up, -1);
    take(g.tb1, down, 1);
    take(g.tb2, down, 1);
    g.qt = st != 0 ? fmax((double)best, g.q) : HUGE_D;
    g.st = st;
  }

  // After a theta crossing into cell t by `step`: the wall just crossed is
  // one of the new cell's walls (its roots are kept), the other is solved.
  __device__ __forceinline__ void qnext_t(QRay& g, int t, int step) const {
    if (step > 0) {
      g.ta1 = g.tb1; g.ta2 = g.tb2;
      cone_roots(g, t, g.tb1, g.tb2);
    } else {
      g.tb1 = g.ta1; g.tb2 = g.ta2;
      cone_roots(g, t - 1, g.ta1, g.ta2);
    }
    qpick_t(g);
  }

  // Next phi-plane crossing of cell p.  A line's azimuth sweeps
  // monotonically (the sense of L_z = c_x u_y - c_y u_x) toward the azimuth
  // of its direction, which it reaches at q -> +inf; so the wall ahead (p,
  // or p-1 when the azimuth falls) is crossed exactly when the direction's
  // azimuth lies beyond it, the sign of A u_x + B u_y with A = sin(phi_w),
  // B = -cos(phi_w).  The decision needs no position, so it holds for rays
  // that pass the z axis closer than FP32 resolves (where every plane's root
  // is within rounding of the current point); the root only orders the
  // crossing among the other faces.  A line turns by less than pi about the
  // axis, so a walk takes at most one turn of crossings.
  __device__ __forceinline__ void qnext_p(QRay& g, int p) const {
    g.qp = HUGE_D;
    g.sp = 0;
    if (m.npg <= 2 || m.ntg <= 2 || g.nphi >= m.npg) return;
    const int w = g.lzpos ? p : p - 1;
    const float2 ab = __ldg(m.pplane + w);
    const float den = __fmaf_rn(ab.x, g.ux, __fmul_rn(ab.y, g.uy));
    if (!(g.lzpos ? den < 0.0f : den > 0.0f)) return;
    const float qi = -__fdividef(__fmaf_rn(ab.x, g.cx, __fmul_rn(ab.y, g.cy)), den);
    g.qp = fmax((double)qi, g.q);
    g.sp = g.lzpos ? 1 : -1;
  }

  // The point of the walk at q: start + (q - q0) u, and its r^2 and r.
  // Written with explicit rounding intrinsics, which the compiler neither
  // contracts nor reassociates, so every schedule that inlines it forms the
  // same bits (the FP32 walk helpers below are written the same way).
  __device__ __forceinline__ static void qpos(double x0, double y0, double z0, double vx, double vy, double vz,
                                              double q, double q0, double& x, double& y, double& z, double& rs,
                                              double& rt) {
    const double d = __dsub_rn(q, q0);
    x = __fma_rn(d, vx, x0);
    y = __fma_rn(d, vy, y0);
    z = __fma_rn(d, vz, z0);
    rs = __fma_rn(z, z, __fma_rn(y, y, __dmul_rn(x, x)));
    rt = __dsqrt_rn(rs);
  }

  // Set up the walk of the ray from (x,y,z) along (vx,vy,vz) in cell
  // (r,t,p).  testgrid's role (testgrid.f90:1-128) is played here, once per
  // walk: an index that disagrees with the start point beyond 1e-4 of the
  // cell is re-located; a start point outside the grid is clamped to its
  // first or last cell (counted as a reset).
  __device__ __forceinline__ void qbegin(QRay& g, double x, double y, double z, double vx, double vy, double vz, int& r,
                                         int& t, int& p) {
    const double q0 = __fma_rn(z, vz, __fma_rn(y, vy, __dmul_rn(x, vx)));
    const double cx = __fma_rn(-q0, vx, x), cy = __fma_rn(-q0, vy, y), cz = __fma_rn(-q0, vz, z);
    g.q = q0;
    g.q0 = q0;
    g.p2 = __fma_rn(cz, cz, __fma_rn(cy, cy, __dmul_rn(cx, cx)));
    g.p2f = (float)g.p2;
    g.pabs = __fsqrt_rn(g.p2f);
    g.cx = (float)cx; g.cy = (float)cy; g.cz = (float)cz;
    g.ux = (float)vx; g.uy = (float)vy; g.uz = (float)vz;
    // the sense of rotation of the FP32 line the roots are solved on: its
    // L_z from the FP32 values, exact in FP64 (a product of two floats is)
    g.lzpos = __dsub_rn(__dmul_rn((double)g.cx, (double)g.uy), __dmul_rn((double)g.cy, (double)g.ux)) > 0.0;
    g.nphi = 0;
    const int nrg = m.nrg, ntg = m.ntg, npg = m.npg;
    const double tol = 1.0e-4;
    const double rs = x * x + y * y + z * z;
    bool moved = false;
    {
      const bool bad = r < 1 || r > nrg - 1;
      const double a = bad ? 0.0 : __ldg(m.r2arr + r - 1), b = bad ? 0.0 : __ldg(m.r2arr + r);
      if (bad || rs - a < -tol * (b - a) || rs - b > tol * (b - a)) {
        const int r0 = locate(m.r2arr, nrg, rs);
        r = min(max(r0, 1), nrg - 1);
        moved = moved || r0 < 1 || r0 > nrg - 1;
      }
    }
    if (ntg > 2) {
      const double cb = chk(z / sqrt(rs));
      const bool bad = t < 1 || t > ntg - 1;
      const double a = bad ? 0.0 : __ldg(m.costarr + t - 1), b = bad ? 0.0 : __ldg(m.costarr + t);
      if (bad || cb - a > tol * (a - b) || b - cb > tol * (a - b)) {
        const int t0 = locate(m.costarr, ntg, cb);
        t = min(max(t0, 1), ntg - 1);
        moved = moved || t0 < 1 || t0 > ntg - 1;
      }
    }
    if (npg > 2) {
      double ph = atan2(y, x);
      if (ph < 0.0) ph = ph + R2P;
      const bool bad = p < 1 || p > npg - 1;
      const double a = bad ? 0.0 : __ldg(m.phiarr + p - 1), b = bad ? 0.0 : __ldg(m.phiarr + p);
      if (bad || ph - a < -tol * (b - a) || ph - b > tol * (b - a)) {
        const int p0 = locate(m.phiarr, npg, ph);
        p = min(max(p0, 1), npg - 1);
      }
    }
    if (moved) ++c_reset;
    qnext_r(g, r);
    if (ntg > 2) {
      cone_roots(g, t - 1, g.ta1, g.ta2);
      cone_roots(g, t, g.tb1, g.tb2);
      qpick_t(g);
    } else {
      g.qt = HUGE_D;
      g.st = 0;
    }
    qnext_p(g, p);
  }
#endif

  // tauint_3d_2_fuv.f90:5-210.  false = geometry failure.
  __device__ bool tauint() {
    double tsum = 0.0;
    for (int guard = 0; guard < 50000000; ++guard) {
      testgrid(xp, yp, zp, rsq, rtot, ir, it, ip, on_wall);
      Walls w;
      w.reset();
      faces(w, ux, uy, uz, xp, yp, zp, ir, it, ip);
      double dt;
      int iface;
      w.next(on_wall, dt, iface);
      if (dt < 0.0 || dt == HUGE_D || iface < 1 || iface > 6) return false;
      const int64_t ci = cidx(ir, it, ip);
      const CellRec c = m.cells[ci];
      const double opac = cell_opac(c);
      const double dtau = opac * dt;
      if (tsum + dtau > tau) {
        const double ds = (tau - tsum) / opac;
        tally_abs(ci, c, ds);
        xp = xp + ds * ux;
        yp = yp + ds * uy;
        zp = zp + ds * uz;
        rsq = xp * xp + yp * yp + zp * zp;
        rtot = sqrt(rsq);
        on_wall = false;
        return true;
      }
      tally_abs(ci, c, dt);
      step_index(iface, ir, it, ip);
      xp = xp + dt * ux;
      yp = yp + dt * uy;
      zp = zp + dt * uz;
      on_wall = true;
      rsq = xp * xp + yp * yp + zp * zp;
      rtot = sqrt(rsq);
      tsum = tsum + dtau;
      ++ncross;
      ++c_cross;
      if (ir == m.nrg) { exitflag = 1; return true; }
      if (ir == 0) {
        atomicAdd(T.scal + MCRT_S_AFLUX, 1.0);
        ++nstar;
        rtot = sqrt(rsq);
        initpabs();
        opacset(nub, KAPD_TAUINT);
        ifuv = is_fuv(nub) ? m.ifuv_ori : 0.0;
        i_orig = 1;
        iflag = 0;
        ir = 1;
        tsum = 0.0;
      }
    }
    return false;
  }

  // ------------------------------------------- tabulated scattering
  // Table row of the species in slot s at the wavelength node a of
  // frequency nu, and the weight f of node a-1: opacset's bracket and
  // weights (dust_5.f90:9-109), so the matrix is interpolated in wavelength
  // exactly as kappa, albedo and g are.
  __device__ void mueller_row(double nu, int s, int& row, double& f) const {
    const int id = m.slot_species[s] - 1;
    const int nl = m.nlammax;
    const double* nud = m.nudust + (int64_t)nl * id;
    const int n = m.nlambda[id];
    int a;
    if (nu >= __ldg(nud)) { a = 0; f = 0.0; }
    else if (nu <= __ldg(nud + n - 1)) { a = n - 1; f = 0.0; }
    else {
      int i0 = 1, i1 = n;
      while (i1 - i0 > 1) {
        const int i = (i1 + i0) >> 1;
        if (nu <= __ldg(nud + i - 1)) i0 = i; else i1 = i;
      }
      a = i1 - 1;
      const int b = i0 - 1;
      f = (nu - __ldg(nud + a)) / (__ldg(nud + b) - __ldg(nud + a));
    }
    row = a + nl * id;
  }
  // matrix element k (S11 S12 S22 S33 S34 S44) in cosine bin itab
  __device__ __forceinline__ double mueller_el(int row, double f, int itab, int k) const {
    const double va = __ldg(m.mueller + 6 * ((int64_t)(itab - 1) + (int64_t)m.narr * row) + k);
    if (f == 0.0) return va;
    const double vb = __ldg(m.mueller + 6 * ((int64_t)(itab - 1) + (int64_t)m.narr * (row - 1)) + k);
    return (1.0 - f) * va + f * vb;
  }
  // itab = int((1+bmu)/dct)+1 (stokes6.f90:62), kept inside the table
  __device__ __forceinline__ int mueller_bin(double bmu) const {
    return min(max((int)((1.0 + bmu) / m.dct) + 1, 1), m.narr);
  }
  // Rejection bound of the interpolated row: the per-row max(S11 + |S12|)
  // bounds (S11 I + S12 (cos2i Q +- sin2i U)) / I for any polarisation, and
  // a linear interpolation of two rows by the larger of their bounds.
  __device__ __forceinline__ double mueller_peak(int row, double f) const {
    return f == 0.0 ? __ldg(m.mpeak + row) : fmax(__ldg(m.mpeak + row), __ldg(m.mpeak + row - 1));
  }

  // The six-element matrix product of stokes6.f90:174-201 (i1 > pi) and
  // :286-306 (i1 < pi), Bohren & Huffman sign of S34.
  struct Mueller6 { double a11, a12, a13, a21, a22, a23, a24, a31, a32, a33, a34, a42, a43, a44; };
  __device__ __forceinline__ Mueller6 mueller6(int row, double f, int itab, bool upper, double s11, double s12,
                                               double c2i, double s2i, double sini2, double cosi2) const {
    const double sin2i2 = 2.0 * sini2 * cosi2, cos2i2 = 2.0 * cosi2 * cosi2 - 1.0;
    const double sin2 = sin2i2 * s2i, cos2 = cos2i2 * c2i;
    const double sin2cos1 = sin2i2 * c2i, cos2sin1 = cos2i2 * s2i;
    const double s22 = mueller_el(row, f, itab, 2), s33 = mueller_el(row, f, itab, 3);
    const double s34 = mueller_el(row, f, itab, 4), s44 = mueller_el(row, f, itab, 5);
    Mueller6 A;
    A.a11 = s11;
    A.a12 = s12 * c2i;
    A.a21 = s12 * cos2i2;
    A.a22 = s22 * cos2 - s33 * sin2;
    A.a33 = -s22 * sin2 + s33 * cos2;
    A.a34 = s34 * cos2i2;
    A.a43 = -s34 * c2i;
    A.a44 = s44;
    if (upper) {
      A.a13 = s12 * s2i;
      A.a23 = s22 * cos2sin1 + s33 * sin2cos1;
      A.a24 = s34 * sin2i2;
      A.a31 = -s12 * sin2i2;
      A.a32 = -s22 * sin2cos1 - s33 * cos2sin1;
      A.a42 = s34 * s2i;
    } else {
      A.a13 = -s12 * s2i;
      A.a23 = -s22 * cos2sin1 - s33 * sin2cos1;
      A.a24 = -s34 * sin2i2;
      A.a31 = s12 * sin2i2;
      A.a32 = s22 * sin2cos1 + s33 * cos2sin1;
      A.a42 = -s34 * s2i;
    }
    return A;
  }

  // stokes6.f90:1-336: scattering with the tabulated matrix of the species
  // in slot s, by rejection under the row's bound.
  __device__ void stokes6(int s) {
    int row;
    double f;
    mueller_row(nub, s, row, f);
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
      sinbt = sqrt(1.0 - cosb2);
      const double ri1 = R2P * ran();
      upper = ri1 > PI;
      const double ang = upper ? R2P - ri1 : ri1;
      ci = cos(ang);
      si_ = sin(ang);
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
      if (fabs(cost) < 1.0) {
        sint = fabs(sqrt(1.0 - cost * cost));
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
    if (fabs(cosdph) > 1.0) cosdph = (cosdph > 1.0) ? 1.0 : -1.0;
    phi = upper ? phip + acos(cosdph) : phip - acos(cosdph);
    if (phi > R2P) phi = phi - R2P;
    if (phi < 0.0) phi = phi + R2P;
    const Mueller6 A = mueller6(row, f, itab, upper, s11, s12, c2i, s2i, sini2, cosi2);
    const double nsi = (A.a11 * sip + A.a12 * sqp + A.a13 * sup) / a;
    const double nsq = (A.a21 * sip + A.a22 * sqp + A.a23 * sup + A.a24 * svp) / a;
    const double nsu = (A.a31 * sip + A.a32 * sqp + A.a33 * sup + A.a34 * svp) / a;
    const double nsv = (A.a42 * sqp + A.a43 * sup + A.a44 * svp) / a;
    sip = nsi; sqp = nsq; sup = nsu; svp = nsv;
    cosp = cos(phi);
    sinp = sin(phi);
  }

  // stokespeel6.f90:1-321: the peel-off weight matrix of the tabulated row
  // (row, f) for scattering angle bmu (no normalisation).
  __device__ void stokespeel6(double& qi, double& qq, double& qu, double& qv, double cst, double snt, double ri1,
                              double bmu, double costp, double sintp, int row, double f) const {
    const int itab = mueller_bin(bmu);
    const double s11 = mueller_el(row, f, itab, 0), s12 = mueller_el(row, f, itab, 1);
    const double cosb2 = bmu * bmu;
    const double sinbt = sqrt(1.0 - cosb2);
    const bool upper = ri1 > PI;
    const double ang = upper ? R2P - ri1 : ri1;
    double ci = cos(ang), si_ = sin(ang);
    const double s2i = 2.0 * si_ * ci, c2i = 2.0 * ci * ci - 1.0;
    if (bmu == 1.0) return;
    double sini2, cosi2 = 0.0;
    if (bmu == -1.0) { si_ = 1.0; sini2 = 1.0; ci = 0.0; cosi2 = 0.0; }
    else if (fabs(cst) < 1.0) {
      sini2 = si_ * sintp / snt;
      const double bott = snt * sinbt;
      cosi2 = costp / bott - cst * bmu / bott;
    } else {
      sini2 = 0.0;
      if (cst >= 1.0) cosi2 = -1.0;
      if (cst <= -1.0) cosi2 = 1.0;
    }
    const Mueller6 A = mueller6(row, f, itab, upper, s11, s12, c2i, s2i, sini2, cosi2);
    const double ni = (A.a11 * qi + A.a12 * qq + A.a13 * qu);
    const double nq = (A.a21 * qi + A.a22 * qq + A.a23 * qu + A.a24 * qv);
    const double nu_ = (A.a31 * qi + A.a32 * qq + A.a33 * qu + A.a34 * qv);
    const double nv = (A.a42 * qq + A.a43 * qu + A.a44 * qv);
    qi = ni; qq = nq; qu = nu_; qv = nv;
  }

  // scattering of the species in slot s: tabulated matrix (stokes6) when the
  // model has one, else the analytic phase matrix (stokes)
  __device__ __forceinline__ void scatter(int s) {
    if (m.mueller) stokes6(s); else stokes(s);
  }
  __device__ __forceinline__ void peel_matrix(double& qi, double& qq, double& qu, double& qv, double cst, double snt,
                                              double ri1, double bmu, double costp, double sintp, int s) const {
    if (m.mueller) {
      int row;
      double f;
      mueller_row(nub, s, row, f);
      stokespeel6(qi, qq, qu, qv, cst, snt, ri1, bmu, costp, sintp, row, f);
    } else {
      stokespeel(qi, qq, qu, qv, cst, snt, ri1, bmu, costp, sintp, s);
    }
  }

  // ------------------------------------------------------- scattering
  __device__ __forceinline__ void dustmat(double bmu, double cosb2, int s, double& p1, double& p2, double& p3) const {
    const double gg = sp.g(s);
    const double g2 = gg * gg;
    const double temp = (g2 + 1.0) - (2.0 * gg) * bmu;
    p1 = 1.5 * (1.0 - g2) / (2.0 + g2) * (1.0 + cosb2) / (temp * sqrt(temp));
    p2 = -sp.pl(s) * p1 * (1.0 - cosb2) / (1.0 + cosb2);
    p3 = p1 * 2.0 * bmu / (1.0 + cosb2);
  }

  // Rotation/phase-matrix product shared by stokes and stokespeel
  // (stokes.f90:183-216 and :284-317; stokespeel.f90:193-210, :293-309).
  struct Mat { double a11, a12, a13, a21, a22, a23, a31, a32, a33, a43, a44; };

#ifdef MCRT_MIXED
  // FP32 scattering: the same rejection sampling and rotations in float
  __device__ __forceinline__ void dustmat_f(float bmu, float cosb2, int s, float& p1, float& p2, float& p3) const {
    const float gg = (float)sp.g(s);
    const float g2 = gg * gg;
    const float temp = (g2 + 1.0f) - (2.0f * gg) * bmu;
    p1 = 1.5f * (1.0f - g2) / (2.0f + g2) * (1.0f + cosb2) / (temp * sqrtf(temp));
    p2 = -(float)sp.pl(s) * p1 * (1.0f - cosb2) / (1.0f + cosb2);
    p3 = p1 * 2.0f * bmu / (1.0f + cosb2);
  }

  __device__ void stokes(int s) {
    const float PIf = 3.14159265358979f, R2Pf = 6.28318530717959f;
    const float costp = (float)cost, sintp = (float)sint, phip = (float)phi;
    const float fsi = (float)sip, fsq = (float)sqp, fsu = (float)sup, fsv = (float)svp;
    const float gg = (float)sp.g(s);
    const float g2 = gg * gg;
    float peak;
    {
      const float temp = (gg > 0.0f) ? (g2 + 1.0f) - (2.0f * gg) : (g2 + 1.0f) + (2.0f * gg);
      peak = 1.5f * (1.0f - g2) / (2.0f + g2) * 2.0f / temp / sqrtf(temp) * 1.01f;
    }
    float bmu, cosb2, sinbt, p1, p2, p3, a, ci, si_, c2i, s2i;
    bool upper;
    for (;;) {
      bmu = 1.0f - 2.0f * (float)ran();
      cosb2 = bmu * bmu;
      if (m.idust == 0) {
        p1 = 0.75f * (1.0f + cosb2); p2 = 0.75f * (cosb2 - 1.0f); p3 = 0.75f * (2.0f * bmu);
        peak = 1.501f;
      } else {
        dustmat_f(bmu, cosb2, s, p1, p2, p3);
      }
      sinbt = sqrtf(fmaxf(0.0f, 1.0f - cosb2));
      const float ri1 = R2Pf * (float)ran();
      upper = ri1 > PIf;
      const float ang = upper ? R2Pf - ri1 : ri1;
      sincosf(ang, &si_, &ci);
      s2i = 2.0f * si_ * ci;
      c2i = 2.0f * ci * ci - 1.0f;
      const float a12 = p2 * c2i;
      const float a13 = upper ? p2 * s2i : -p2 * s2i;
      const float rprob = (p1 * fsi + a12 * fsq + a13 * fsu) / fsi;
      if (rprob > peak) peak = rprob;
      if (peak * (float)ran() > rprob) continue;
      a = rprob;
      break;
    }
    if (bmu == 1.0f) return;
    float sini2, cosi2 = 0.0f, ncost, nsint;
    if (bmu == -1.0f) {
      si_ = 1.0f; sini2 = 1.0f; ci = 0.0f; cosi2 = 0.0f;
      ncost = -costp; nsint = sintp;
    } else {
      ncost = costp * bmu + sintp * sinbt * ci;
      if (fabsf(ncost) < 1.0f) {
        nsint = sqrtf(1.0f - ncost * ncost);
        sini2 = si_ * sintp / nsint;
        const float bott = nsint * sinbt;
        cosi2 = costp / bott - ncost * bmu / bott;
      } else {
        nsint = 0.0f; sini2 = 0.0f;
        if (ncost >= 1.0f) cosi2 = -1.0f;
        if (ncost <= -1.0f) cosi2 = 1.0f;
      }
    }
    float cosdph = -cosi2 * ci + sini2 * si_ * bmu;
    cosdph = fminf(1.0f, fmaxf(-1.0f, cosdph));
    float nphi = upper ? phip + acosf(cosdph) : phip - acosf(cosdph);
    if (nphi > R2Pf) nphi = nphi - R2Pf;
    if (nphi < 0.0f) nphi = nphi + R2Pf;
    const float sin2i2 = 2.0f * sini2 * cosi2, cos2i2 = 2.0f * cosi2 * cosi2 - 1.0f;
    const float sin2 = sin2i2 * s2i, cos2 = cos2i2 * c2i;
    const float sin2cos1 = sin2i2 * c2i, cos2sin1 = cos2i2 * s2i;
    const float a11 = p1, a12 = p2 * c2i, a21 = p2 * cos2i2, a22 = p1 * cos2 - p3 * sin2;
    const float a33 = -p1 * sin2 + p3 * cos2, a44 = p3;
    float a13, a23, a31, a32;
    if (upper) {
      a13 = p2 * s2i; a23 = p1 * cos2sin1 + p3 * sin2cos1; a31 = -p2 * sin2i2; a32 = -p1 * sin2cos1 - p3 * cos2sin1;
    } else {
      a13 = -p2 * s2i; a23 = -p1 * cos2sin1 - p3 * sin2cos1; a31 = p2 * sin2i2; a32 = p1 * sin2cos1 + p3 * cos2sin1;
    }
    const float ia = 1.0f / a;
    sip = (double)((a11 * fsi + a12 * fsq + a13 * fsu) * ia);
    sqp = (double)((a21 * fsi + a22 * fsq + a23 * fsu) * ia);
    sup = (double)((a31 * fsi + a32 * fsq + a33 * fsu) * ia);
    svp = (double)((a44 * fsv) * ia);
    // the walk's face roots assume |u| = 1 to FP64 precision: rebuild the
    // direction from cos(theta) and phi in FP64
    cost = (double)ncost;
    sint = (nsint == 0.0f) ? 0.0 : sqrt(fmax(0.0, 1.0 - cost * cost));
    phi = (double)nphi;
    sincos(phi, &sinp, &cosp);
    (void)nsint;
  }

  __device__ void stokespeel(double& qi, double& qq, double& qu, double& qv, double cst, double snt, double ri1d,
                             double bmud, double costpd, double sintpd, int s) const {
    const float PIf = 3.14159265358979f, R2Pf = 6.28318530717959f;
    const float bmu = (float)bmud, cstf = (float)cst, sntf = (float)snt, costp = (float)costpd, sintp = (float)sintpd;
    float p1, p2, p3;
    const float cosb2 = bmu * bmu;
    if (m.idust == 0) { p1 = 0.75f * (1.0f + cosb2); p2 = 0.75f * (cosb2 - 1.0f); p3 = 0.75f * (2.0f * bmu); }
    else dustmat_f(bmu, cosb2, s, p1, p2, p3);
    const float sinbt = sqrtf(fmaxf(0.0f, 1.0f - cosb2));
    const float ri1 = (float)ri1d;
    const bool upper = ri1 > PIf;
    const float ang = upper ? R2Pf - ri1 : ri1;
    float ci, si_;
    sincosf(ang, &si_, &ci);
    const float s2i = 2.0f * si_ * ci, c2i = 2.0f * ci * ci - 1.0f;
    if (bmu == 1.0f) return;
    float sini2, cosi2 = 0.0f;
    if (bmu == -1.0f) { si_ = 1.0f; sini2 = 1.0f; ci = 0.0f; cosi2 = 0.0f; }
    else if (fabsf(cstf) < 1.0f) {
      sini2 = si_ * sintp / sntf;
      const float bott = sntf * sinbt;
      cosi2 = costp / bott - cstf * bmu / bott;
    } else {
      sini2 = 0.0f;
      if (cstf >= 1.0f) cosi2 = -1.0f;
      if (cstf <= -1.0f) cosi2 = 1.0f;
    }
    const float sin2i2 = 2.0f * sini2 * cosi2, cos2i2 = 2.0f * cosi2 * cosi2 - 1.0f;
    const float sin2 = sin2i2 * s2i, cos2 = cos2i2 * c2i;
    const float sin2cos1 = sin2i2 * c2i, cos2sin1 = cos2i2 * s2i;
    const float a11 = p1, a12 = p2 * c2i, a21 = p2 * cos2i2, a22 = p1 * cos2 - p3 * sin2;
    const float a33 = -p1 * sin2 + p3 * cos2, a44 = p3;
    float a13, a23, a31, a32;
    if (upper) {
      a13 = p2 * s2i; a23 = p1 * cos2sin1 + p3 * sin2cos1; a31 = -p2 * sin2i2; a32 = -p1 * sin2cos1 - p3 * cos2sin1;
    } else {
      a13 = -p2 * s2i; a23 = -p1 * cos2sin1 - p3 * sin2cos1; a31 = p2 * sin2i2; a32 = p1 * sin2cos1 + p3 * cos2sin1;
    }
    const float fi = (float)qi, fq = (float)qq, fu = (float)qu, fv = (float)qv;
    qi = (double)(a11 * fi + a12 * fq + a13 * fu);
    qq = (double)(a21 * fi + a22 * fq + a23 * fu);
    qu = (double)(a31 * fi + a32 * fq + a33 * fu);
    qv = (double)(a44 * fv);
  }
#else
  __device__ void stokes(int s) {                  // stokes.f90:1-340 (p4 = 0)
    const double costp = cost, sintp = sint, phip = phi;
    const double gg = sp.g(s);
    const double g2 = gg * gg;
    double peak;
    {
      double temp = (gg > 0.0) ? (g2 + 1.0) - (2.0 * gg) : (g2 + 1.0) + (2.0 * gg);
      peak = 1.5 * (1.0 - g2) / (2.0 + g2) * 2.0 / temp / sqrt(temp);
      peak = peak * 1.01;
    }
    double bmu, cosb2, sinbt, p1, p2, p3, a, ci, si_, c2i, s2i;
    bool upper;
    for (;;) {
      bmu = 1.0 - 2.0 * ran();
      cosb2 = bmu * bmu;
      if (m.idust == 0) {
        p1 = 0.75 * (1.0 + cosb2); p2 = 0.75 * (cosb2 - 1.0) * 1.0; p3 = 0.75 * (2.0 * bmu);
        peak = 1.501;
      } else {
        dustmat(bmu, cosb2, s, p1, p2, p3);
      }
      sinbt = sqrt(1.0 - cosb2);
      const double ri1 = R2P * ran();
      upper = ri1 > PI;
      const double ang = upper ? R2P - ri1 : ri1;
      ci = cos(ang);
      si_ = sin(ang);
      s2i = 2.0 * si_ * ci;
      c2i = 2.0 * ci * ci - 1.0;
      const double a12 = p2 * c2i;
      const double a13 = upper ? p2 * s2i : -p2 * s2i;
      const double rprob = (p1 * sip + a12 * sqp + a13 * sup) / sip;
      if (rprob > peak) peak = rprob;
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
      if (fabs(cost) < 1.0) {
        sint = fabs(sqrt(1.0 - cost * cost));
        sini2 = si_ * sintp / sint;
        const double bott = sint * sinbt;
        cosi2 = costp / bott - cost * bmu / bott;
      } else {
        sint = 0.0; sini2 = 0.0;
        if (cost >= 1.0) cosi2 = -1.0;
        if (cost <= -1.0) cosi2 = 1.0;
      }
    }
    double cosdph = upper ? -cosi2 * ci + sini2 * si_ * bmu : -ci * cosi2 + si_ * sini2 * bmu;
    if (fabs(cosdph) > 1.0) cosdph = (cosdph > 1.0) ? 1.0 : -1.0;
    phi = upper ? phip + acos(cosdph) : phip - acos(cosdph);
    if (phi > R2P) phi = phi - R2P;
    if (phi < 0.0) phi = phi + R2P;
    const double sin2i2 = 2.0 * sini2 * cosi2, cos2i2 = 2.0 * cosi2 * cosi2 - 1.0;
    const double sin2 = sin2i2 * s2i, cos2 = cos2i2 * c2i;
    const double sin2cos1 = sin2i2 * c2i, cos2sin1 = cos2i2 * s2i;
    // p4 = 0 in dustmat and the Rayleigh branch, so a24=a34=a42=a43=0
    double a11 = p1, a12 = p2 * c2i, a13, a21 = p2 * cos2i2, a22 = p1 * cos2 - p3 * sin2, a23, a31, a32;
    const double a33 = -p1 * sin2 + p3 * cos2, a44 = p3;
    if (upper) {
      a13 = p2 * s2i;
      a23 = p1 * cos2sin1 + p3 * sin2cos1;
      a31 = -p2 * sin2i2;
      a32 = -p1 * sin2cos1 - p3 * cos2sin1;
    } else {
      a13 = -p2 * s2i;
      a23 = -p1 * cos2sin1 - p3 * sin2cos1;
      a31 = p2 * sin2i2;
      a32 = p1 * sin2cos1 + p3 * cos2sin1;
    }
    const double a24 = 0.0 * sin2i2, a34 = 0.0 * cos2i2, a42 = 0.0 * s2i, a43 = 0.0 * c2i;
    const double nsi = (a11 * sip + a12 * sqp + a13 * sup) / a;
    const double nsq = (a21 * sip + a22 * sqp + a23 * sup + a24 * svp) / a;
    const double nsu = (a31 * sip + a32 * sqp + a33 * sup + a34 * svp) / a;
    const double nsv = (a42 * sqp + a43 * sup + a44 * svp) / a;
    sip = nsi; sqp = nsq; sup = nsu; svp = nsv;
    cosp = cos(phi);
    sinp = sin(phi);
  }

  // stokespeel.f90:1-328 (no normalisation), sign conventions as stokes
  __device__ void stokespeel(double& qi, double& qq, double& qu, double& qv, double cst, double snt, double ri1,
                             double bmu, double costp, double sintp, int s) const {
    double p1, p2, p3;
    const double cosb2 = bmu * bmu;
    if (m.idust == 0) {
      p1 = 0.75 * (1.0 + cosb2); p2 = 0.75 * (cosb2 - 1.0) * 1.0; p3 = 0.75 * (2.0 * bmu);
    } else {
      dustmat(bmu, cosb2, s, p1, p2, p3);
    }
    const double sinbt = sqrt(1.0 - cosb2);
    const bool upper = ri1 > PI;
    const double ang = upper ? R2P - ri1 : ri1;
    double ci = cos(ang), si_ = sin(ang);
    const double s2i = 2.0 * si_ * ci, c2i = 2.0 * ci * ci - 1.0;
    if (bmu == 1.0) return;
    double sini2, cosi2 = 0.0;
    if (bmu == -1.0) { si_ = 1.0; sini2 = 1.0; ci = 0.0; cosi2 = 0.0; }
    else if (fabs(cst) < 1.0) {
      sini2 = si_ * sintp / snt;
      const double bott = snt * sinbt;
      cosi2 = costp / bott - cst * bmu / bott;
    } else {
      sini2 = 0.0;
      if (cst >= 1.0) cosi2 = -1.0;
      if (cst <= -1.0) cosi2 = 1.0;
    }
    const double sin2i2 = 2.0 * sini2 * cosi2, cos2i2 = 2.0 * cosi2 * cosi2 - 1.0;
    const double sin2 = sin2i2 * s2i, cos2 = cos2i2 * c2i;
    const double sin2cos1 = sin2i2 * c2i, cos2sin1 = cos2i2 * s2i;
    double a13, a23, a31, a32;
    const double a11 = p1, a12 = p2 * c2i, a21 = p2 * cos2i2, a22 = p1 * cos2 - p3 * sin2;
    const double a33 = -p1 * sin2 + p3 * cos2, a44 = p3;
    if (upper) {
      a13 = p2 * s2i; a23 = p1 * cos2sin1 + p3 * sin2cos1; a31 = -p2 * sin2i2; a32 = -p1 * sin2cos1 - p3 * cos2sin1;
    } else {
      a13 = -p2 * s2i; a23 = -p1 * cos2sin1 - p3 * sin2cos1; a31 = p2 * sin2i2; a32 = p1 * sin2cos1 + p3 * cos2sin1;
    }
    const double a24 = 0.0 * sin2i2, a34 = 0.0 * cos2i2, a42 = 0.0 * s2i, a43 = 0.0 * c2i;
    const double ni = (a11 * qi + a12 * qq + a13 * qu);
    const double nq = (a21 * qi + a22 * qq + a23 * qu + a24 * qv);
    const double nu_ = (a31 * qi + a32 * qq + a33 * qu + a34 * qv);
    const double nv = (a42 * qq + a43 * qu + a44 * qv);
    qi = ni; qq = nq; qu = nu_; qv = nv;
  }
#endif

  __device__ __forceinline__ int freq_bin(double nu) const {
    const double v = (double)m.nfreq * log(nu / m.numin) / m.lnurat;
    int ib;
    if (!(v > -2.0e9)) ib = 0;
    else if (v > 2.0e9) ib = m.nfreq;
    else ib = (int)v + 1;
    return min(max(ib, 1), m.nfreq);
  }

  // ------------------------------------------------------- peel-off
  // peeloff_3d_2_test.f90:7-347 for one direction
  __device__ void peeloff(double s_i, int r, int t, int p, int idust2, int peelid) {
    ++c_peel;
    bool onw = on_wall;
    double x1 = xp, y1 = yp, z1 = zp, rs1 = rsq, rt1 = rtot;
    const double cospe = __ldg(m.cospe + peelid - 1), sinpe = __ldg(m.sinpe + peelid - 1);
    const double coste = __ldg(m.coste + peelid - 1), sinte = __ldg(m.sinte + peelid - 1);
    const double ux1 = sinte * cospe, uy1 = sinte * sinpe, uz1 = coste;
    if (onw) {
      const bool inner = fabs(rs1 - __ldg(m.r2arr + r - 1)) < fabs(rs1 - __ldg(m.r2arr + r));
      const bool outwards = ux1 * x1 + uy1 * y1 + uz1 * z1 > 0.0;
      if (inner && !outwards) {
        if (r == 1) return;
        r = r - 1;
      }
      if (!inner && outwards) r = r + 1;
    }
    double tsum = 0.0;
    for (int guard = 0;; ++guard) {
      if (guard > 10000000) return;
      testgrid(x1, y1, z1, rs1, rt1, r, t, p, onw);
      Walls w;
      w.reset();
      faces(w, ux1, uy1, uz1, x1, y1, z1, r, t, p);
      double dt;
      int iface;
      w.next(onw, dt, iface);
      if (dt == HUGE_D || iface < 1 || iface > 6) return;
      const CellRec c = m.cells[cidx(r, t, p)];
      tsum = tsum + cell_opac(c) * dt;
      if (tsum > 25.0) return;
      step_index(iface, r, t, p);
      x1 = x1 + dt * ux1;
      y1 = y1 + dt * uy1;
      z1 = z1 + dt * uz1;
      onw = true;
      rs1 = x1 * x1 + y1 * y1 + z1 * z1;
      rt1 = sqrt(rs1);
      ++c_pcross;
      if (r == m.nrg) break;
      if (r == 0) return;
    }
    ++c_pbin;
    const double factor = exp(-tsum);
    double qi = s_i * factor, qq = sqp * factor, qu = sup * factor, qv = svp * factor;
    if (iflag == 1) {
      // findangle3.f90 with phi2 = phie = 0 (reapar_4_test1.f90:425)
      double costnew = cost * coste + (sint * sinte * (cosp * cospe + sinp * sinpe));
      costnew = chk(costnew);
      const double sintnew = sqrt(1.0 - costnew * costnew);
      double ri1 = 0.0;
      if (sint > 1.0e-8 && sintnew > 1.0e-8) {
        double cosx = (coste - (cost * costnew)) / (sint * sintnew);
        cosx = chk(cosx);
        const double x = acos(cosx);
        if (0.0 > phi) ri1 = (0.0 - phi > PI) ? x : R2P - x;
        else ri1 = (phi - 0.0 > PI) ? R2P - x : x;
      }
      // species of the final walk cell, as the reference indexes findopac
      int sslot = 0;
      const CellRec cf = m.cells[cidx(r, t, p)];
      const int n = cell_n(cf.meta);
      bool found = false;
      for (int k = 0; k < n; ++k)
        if (cell_id(cf.meta, k) == idust2) { sslot = cell_slot(cf.meta, k); found = true; }
      if (!found) sslot = idust2slot(idust2);
      peel_matrix(qi, qq, qu, qv, coste, sinte, ri1, costnew, cost, sint, sslot);
    }
    const double yimage = z1 * sinte - y1 * coste * sinpe - x1 * coste * cospe;
    const double ximage = y1 * cospe - x1 * sinpe;
    const double vx = (ximage + m.rmaxi) / m.fractxh, vy = (yimage + m.rmaxi) / m.fractxh;
    const double rho2 = ximage * ximage + yimage * yimage;
    const int inub = freq_bin(nub);
    if (m.output_imcube && vx > -1.0e9 && vx < 1.0e9 && vy > -1.0e9 && vy < 1.0e9) {
      const int ix = (int)vx + 1, iy = (int)vy + 1;
      if (ix <= m.nxhst && iy <= m.nxhst && ix > 0 && iy > 0) {
        const int64_t k = (int64_t)(peelid - 1) + (int64_t)m.npeel * ((ix - 1) + (int64_t)m.nxhst * ((iy - 1) + (int64_t)m.nxhst * (inub - 1)));
        atomicAdd(T.img + k, qi);
        atomicAdd(T.img + m.nimg + k, qq);
        atomicAdd(T.img + 2 * m.nimg + k, qu);
        atomicAdd(T.img + 3 * m.nimg + k, qv);
      }
    }
    bin_filters(m, T, peelid, vx, vy, nub, i_orig, qi, qq, qu, qv);
    bin_nested(m, T, peelid, ximage, yimage, nub, qi, qq, qu, qv);
    const int i_inter = (iflag == 1) ? 2 : ((i_orig == 1) ? 1 : 3);
    const int indx[3] = {1, 1 + i_orig, 5 + i_inter};
    for (int ia = 1; ia <= m.nap; ++ia) {
      if (rho2 < __ldg(m.aperture2 + ia - 1)) {
        for (int k = 0; k < 3; ++k) {
          const int64_t e = (inub - 1) + (int64_t)m.nfreq * ((peelid - 1) + (int64_t)m.npeel * ((ia - 1) + (int64_t)m.nap * (indx[k] - 1)));
          double* P = T.psed + e;
          atomicAdd(P, qi); atomicAdd(P + m.npsed, qq); atomicAdd(P + 2 * m.npsed, qu); atomicAdd(P + 3 * m.npsed, qv);
          atomicAdd(P + 4 * m.npsed, qi * qi); atomicAdd(P + 5 * m.npsed, qq * qq);
          atomicAdd(P + 6 * m.npsed, qu * qu); atomicAdd(P + 7 * m.npsed, qv * qv);
          atomicAdd(P + 8 * m.npsed, 1.0);
        }
      }
    }
  }

  // isotrp.f90:1-36
  __device__ void isotrp(double sux, double suy, double suz) {
    double r2 = 2.0, mur = 0.0, x = 0.0, y = 0.0, z = 0.0;
    while (r2 * r2 > fabs(mur)) {
      x = ran(); x = x + x - 1.0;
      y = ran(); y = y + y - 1.0;
      z = ran(); z = z + z - 1.0;
      mur = x * sux + y * suy + z * suz;
      r2 = x * x + y * y + z * z;
    }
    double r = sqrt(r2);
    if (mur < 0.0) r = -r;
    ux = x / r; uy = y / r; uz = z / r;
  }

  // select_dust with mask = is_thermal (emit_common_2.f90:346)
  __device__ int select_thermal(const CellRec& c) {
    const double xran = ran();
    const int n = cell_n(c.meta);
    int nn = 0, kk = -1;
    for (int k = 0; k < n; ++k) {
      const int id = cell_id(c.meta, k);
      if (!(id >= 5 && id <= 8)) { ++nn; kk = k; }
    }
    if (nn == 1) return kk;
    double opac = 0.0;
    for (int k = 0; k < n; ++k) {
      const int id = cell_id(c.meta, k);
      if (!(id >= 5 && id <= 8)) opac = opac + sp.kapd(cell_slot(c.meta, k)) * c.rho[k];
    }
    if (opac == 0.0) return -1;
    double frac = 0.0;
    for (int k = 0; k < n; ++k) {
      const int id = cell_id(c.meta, k);
      if (id >= 5 && id <= 8) continue;
      frac = frac + sp.kapd(cell_slot(c.meta, k)) * c.rho[k] / opac;
      if (xran <= frac + 1.0e-10) return k;
    }
    return -1;
  }

  // emit_common_2.f90:201-372, vertical diffusion (|diffdir| = 2) without
  // accretion photons (nacc = 0): move the packet to the diffusion surface,
  // heat the surface cell and emit isotropically from it.  The k-th
  // diffusion absorption at a surface cell (atomic counter) heats it to
  // T^4 = T0^4 + k dT^4, the reference's recursion of :260-272.
  __device__ bool emit_diffusion(const LaunchParams& P) {
    const double Tmax = 199999.0;
    const int dd = cell_diffdir(m.cells[cidx(ir, it, ip)].flags);
    if (dd == -2) {
      while (it >= 1 && cell_diffus(m.cells[cidx(ir, it, ip)].flags)) it = it - 1;
      if (it < 1) return false;
      it = it + 1;
    } else {
      while (it <= m.ntg - 1 && cell_diffus(m.cells[cidx(ir, it, ip)].flags)) it = it + 1;
      if (it > m.ntg - 1) return false;
    }
    cosb = zp / rtot;
    sinb = sqrt(1.0 - cosb * cosb);
    const double cosbnew = 1.00001 * m.costarr[it - 1];
    const double sinbnew = sqrt(1.0 - cosbnew * cosbnew);
    xp = xp * sinbnew / sinb;
    yp = yp * sinbnew / sinb;
    zp = rtot * cosbnew;
    const double mu0 = m.costarr[it - 1], sth = m.sintarr[it - 1];
    double sux, suy, suz;
    if (mu0 > 0.0) { sux = -mu0 * xp / sth / rtot; suy = -mu0 * yp / sth / rtot; suz = sth; }
    else { sux = mu0 * xp / sth / rtot; suy = mu0 * yp / sth / rtot; suz = -sth; }
    isotrp(sux, suy, suz);
    cost = uz;
    sint = sqrt(1.0 - cost * cost);
    cosp = ux / sint;
    sinp = uy / sint;
    phi = atan2(sinp, cosp);
    if (m.costarr[it - 1] < 0.0) it = it - 1;
    const double dA = PI * sth * (m.rarr[ir] * m.rarr[ir] - m.rarr[ir - 1] * m.rarr[ir - 1]);
    double T4s = m.tstar * m.tstar;
    T4s = T4s * T4s;
    const int64_t cs = cidx(ir, it, ip);
    const CellRec c = m.cells[cs];
    int nth = 0;
    for (int k = 0; k < cell_n(c.meta); ++k) { const int id = cell_id(c.meta, k); if (!(id >= 5 && id <= 8)) ++nth; }
    if (nth == 0) return false;
    // adjoint evaluations freeze the surface at its start-of-iteration
    // temperature (a replay must see the forward pass's heating)
    const int32_t k = P.adj.mode ? 0 : atomicAdd(T.ndiff + cs, nth) + nth;
    const double t0 = __ldg(m.tdust + cs);
    double T4d = t0 * t0;
    T4d = T4d * T4d;
    const double T4 = T4d + (double)k * (4.0 * PI * T4s / (P.nphot_diff * dA));
    const double tsurf = fmin(Tmax / 11605.0, pow(T4, 0.25));
    if (select_thermal(c) < 0) return false;
    double T4b = tsurf * tsurf;
    T4b = T4b * T4b;
    const double T4eff = 0.0;
    const double mu = ux * sux + uy * suy + uz * suz;
    const double T = fmin(pow(T4b + 0.75 * mu * T4eff, 0.25), Tmax / 11605.0);
    nub = bbfreq(T);
    if (cell_diffdir(c.flags) == -2) it = it - 1; else it = it + 1;
    return true;
  }

  // slot of a species id whose component is absent in the lookup cell
  __device__ __forceinline__ int idust2slot(int idust2) const {
    for (int s = 0; s < m.nslot; ++s)
      if (m.slot_species[s] == idust2) return s;
    return 0;
  }

  // select_dust_2.f90 with mask = is_any; returns component index k (or -1)
  __device__ int select_dust(const CellRec& c) {
    const double xran = ran();
    const int n = cell_n(c.meta);
    int nn = 0, kk = -1;
    for (int k = 0; k < n; ++k) {
      const int id = cell_id(c.meta, k);
      if (!(id >= 5 && id <= 8)) { ++nn; kk = k; }
    }
    if (nn == 1) return kk;
    double opac = 0.0;
    for (int k = 0; k < n; ++k) opac = opac + sp.kapd(cell_slot(c.meta, k)) * c.rho[k];
    if (opac == 0.0) return -1;
    double frac = 0.0;
    for (int k = 0; k < n; ++k) {
      frac = frac + sp.kapd(cell_slot(c.meta, k)) * c.rho[k] / opac;
      if (xran <= frac + 1.0e-10) return k;
    }
    return -1;
  }

  // ------------------------------------------------------------ packet
  // emit_common (emit_common_2.f90:1-384) for the absorbing / emitting cell
  // ci and its thermal component in species slot `slot`: Lucy reemission
  // at the cell's temperature (reemit.f90 + lucydustfreq), or, in a
  // diffusion cell, emission from the diffusion surface.  false = geometry
  // failure.
  __device__ bool emit_common(const LaunchParams& P, int64_t ci, const CellRec& c, int slot) {
    const int id = m.slot_species[slot];    // dust components use their own species (findopacid_5.f90)
    if (!cell_diffus(c.flags) && id >= 5 && id <= 8) {
      // small grains (emit_common_2.f90:32-50): a frequency from the Draine
      // spectrum of the cell's intensity level, then emit_sg.f90 (an
      // unpolarised packet in a random direction).  The opacset the
      // reference calls here is repeated by propagate right after.
      const bool first = (P.block0_dev ? *P.block0_dev : P.block0) == 0;   // iteration 1
      const int im = first ? 2 : (m.imean ? __ldg(m.imean + ci) : 1);
      nub = rep_draine(im);
      sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
      cost = 1.0 - 2.0 * ran();
      sint = sqrt(1.0 - cost * cost);
      phi = R2P * ran();
      cosp = cos(phi);
      sinp = sin(phi);
      uy = sint * sinp;
      ux = sint * cosp;
      uz = cost;
      return true;
    }
    if (!cell_diffus(c.flags)) {
      const double tave = __ldg(m.tdust + ci);
      sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;    // reemit.f90
      cost = 1.0 - 2.0 * ran();
      sint = sqrt(1.0 - cost * cost);
      phi = R2P * ran();
      cosp = cos(phi);
      sinp = sin(phi);
      nub = lucydustfreq(tave, m.slot_species[slot]);
      uy = sint * sinp;
      ux = sint * cosp;
      uz = cost;
      return true;
    }
    ++ndiffev;
    return emit_diffusion(P);
  }

  // initpacc_4.f90:19-81: a disk-accretion emission point.  The radius is
  // drawn once from the luminosity CDF Ldint (cell centre ravearr); the
  // azimuth (rantheta, random.f90:23-42) and the height hdisk * gasdev
  // (random.f90:119-138, Box-Muller polar form with its saved second
  // deviate) are redrawn until the point lies in a cell with thermal dust.
  // The saved deviate lives in the packet: packets draw from independent
  // streams here, where the reference passes it from one packet to the
  // next of its rank's single stream.  Points outside the grid are redrawn
  // (the reference would index past its arrays).  Returns the thermal
  // component index in the cell record, or -1 after kMaxAccTries draws.
  __device__ int initpacc(int64_t& ci) {
    const double xi = ran();
    int r0 = locate(m.Ldint, m.nrg - 1, xi);
    r0 = min(max(r0, 1), m.nrg - 1);
    const double rp = __ldg(m.ravearr + r0 - 1);
    const double hd = __ldg(m.hdisk + r0 - 1);
    bool have_g = false;
    double gsave = 0.0;
    for (int tries = 0; tries < kMaxAccTries; ++tries) {
      double x = 0.0, y = 0.0, r2 = 2.0;
      while (r2 > 1.0) {
        x = ran(); x = x + x - 1.0;
        y = ran(); y = y + y - 1.0;
        r2 = x * x + y * y;
      }
      const double rr = sqrt(r2);
      const double st = y / rr, ct = x / rr;
      xp = rp * ct;
      yp = rp * st;
      double g;
      if (!have_g) {
        double v1, v2, q;
        do {
          v1 = 2.0 * ran() - 1.0;
          v2 = 2.0 * ran() - 1.0;
          q = v1 * v1 + v2 * v2;
        } while (!(q < 1.0 && q > 0.0));
        const double fac = sqrt(-2.0 * log(q) / q);
        gsave = v1 * fac;
        g = v2 * fac;
        have_g = true;
      } else {
        g = gsave;
        have_g = false;
      }
      zp = hd * g;
      sip = 1.0; sqp = 0.0; sup = 0.0; svp = 0.0;
      rsq = xp * xp + yp * yp + zp * zp;
      rtot = sqrt(rsq);
      ir = locate(m.r2arr, m.nrg, rsq);
      cosb = zp / rtot;
      it = locate(m.costarr, m.ntg, cosb);
      lp = atan2(yp, xp);
      if (lp < 0.0) lp = lp + R2P;
      ip = locate(m.phiarr, m.npg, lp);
      if (ir < 1 || ir > m.nrg - 1 || it < 1 || it > m.ntg - 1 || ip < 1 || ip > m.npg - 1) continue;
      ci = cidx(ir, it, ip);
      const CellRec c = m.cells[ci];
      if (!cell_thermal(c.flags)) continue;
      return select_thermal(c);
    }
    return -1;
  }

  // initpacc_4.f90:83-99 after the position: tallies of the emitting cell
  // and emit_common.  The selected component is a thermal one with non-zero
  // density, so dbig and nabs count every accretion packet.  Returns idust2
  // (1-based component id), or -1 on failure.
  __device__ int accretion_emission(const LaunchParams& P) {
    int64_t ci = 0;
    const int k = initpacc(ci);
    if (k < 0) return -1;
    const CellRec c = m.cells[ci];
    atomicAdd(T.dbig + ci, 1);
    atomicAdd(T.nabs + ci, 1);
    if (!emit_common(P, ci, c, cell_slot(c.meta, k))) return -1;
    return cell_id(c.meta, k);
  }

  __device__ int run(int64_t iphot, const LaunchParams& P) {
    on_wall = false;
    nscat = nabsev = ncross = nstar = ndiffev = 0;
    if (iphot > P.npacc + P.ns) return 3;   // external illumination: rejected at launch
    if (iphot < P.npacc) {                  // disk accretion, newdisktherm_5_fuv.f90:238-287
      const int idust2 = accretion_emission(P);
      if (idust2 < 0) return 3;
      opacset(nub, KAPD_DISK);
      iflag = 0;
      i_orig = 2;
      if (P.ipeel == 1)
        for (int peelid = 1; peelid <= m.npeel; ++peelid) peeloff(sip, ir, it, ip, idust2, peelid);
      ifuv = is_fuv(nub) ? m.ifuv_ori : 0.0;
      return propagate(P);
    }
    if (iphot < P.npacc + P.npaccstar) {
      if (P.ips == 0) initpspot(1); else initp_ps(1);
      if (ran() < 0.5) nub = 1.2398 / 0.06 + ran() * (1.2398 / 0.015 - 1.2398 / 0.06);
    } else {
      if (P.ips == 0) initpspot(0); else initp_ps(0);
    }
    i_orig = 1;
    opacset(nub, KAPD_DISK);
    const double coslp = cos(lp), sinlp = sin(lp);
    const double rmin = m.rarr[0];
    zp = cosb * rmin;
    const double rp = sinb * rmin;
    xp = rp * coslp;
    yp = rp * sinlp;
    rsq = zp * zp + rp * rp;
    rtot = sqrt(rsq);
    ux = sint * cosp;
    uy = sint * sinp;
    uz = cost;
    iflag = 0;
    ir = 1;
    on_wall = true;
    it = locate(m.thetarr, m.ntg, acos(cosb));
    ip = locate(m.phiarr, m.npg, lp);
    if (P.ipeel == 1 && !m.partial_peeloff) {
      for (int peelid = 1; peelid <= m.npeel; ++peelid) {
        if (P.ips == 0) {
          const double coste = __ldg(m.coste + peelid - 1), sinte = __ldg(m.sinte + peelid - 1);
          const double cospe = __ldg(m.cospe + peelid - 1), sinpe = __ldg(m.sinpe + peelid - 1);
          const double cosnorm = cosb * coste + (sinb * sinte * (cospe * coslp + sinpe * sinlp));
          const double sipnew = (m.limb == 0) ? 4.0 * sip * cosnorm : 12.0 / 5.0 * sip * (cosnorm + cosnorm * cosnorm);
          if (cosnorm > 0.0) peeloff(sipnew, ir, it, ip, 0, peelid);
        } else {
          peeloff(sip * 2.0, ir, it, ip, 0, peelid);
        }
      }
    }
    ifuv = is_fuv(nub) ? m.ifuv_ori : 0.0;
    return propagate(P);
  }

  // propagate_5_fuv.f90:1-326
  __device__ int propagate(const LaunchParams& P) {
    double xpold = xp, ypold = yp, zpold = zp;
    iflag = 0;
    exitflag = 0;
    int iscat = 0, iint = 0;
    int64_t nev = 0;
    tau = -log(ran());
    if (!tauint()) return 3;
    if (exitflag != 1) {
      CellRec c = m.cells[cidx(ir, it, ip)];
      int k = select_dust(c);
      if (k < 0) return 3;
      atomicAdd(T.scal + MCRT_S_TOT, 1.0);
      for (;;) {
        const int slot = cell_slot(c.meta, k);
        const int idust2 = cell_id(c.meta, k);
        if (ran() <= sp.alb(slot)) {               // scattered
          iflag = 1;
          ++iscat;
          ++iint;
          ++nscat;
          if (P.ipeel == 1)
            for (int peelid = 1; peelid <= m.npeel; ++peelid) peeloff(sip, ir, it, ip, idust2, peelid);
          scatter(slot);
        } else {                                    // absorbed + re-emitted
          ++nabsev;
          const int64_t ci = cidx(ir, it, ip);
          if (idust2 >= 5 && idust2 <= 8) atomicAdd(T.dsg + ci, 1); else atomicAdd(T.dbig + ci, 1);
          if (idust2 == 1 || idust2 == 2 || idust2 == 5 || idust2 == 6 || idust2 == 9) i_orig = 2;
          else if (idust2 == 3 || idust2 == 7) i_orig = 3;
          else i_orig = 4;
          if (!cell_diffus(c.flags)) atomicAdd(T.nabs + ci, 1);
          if (!emit_common(P, ci, c, slot)) return 3;
          iflag = 0;
          opacset(nub, KAPD_PROPAGATE);
          ifuv = is_fuv(nub) ? m.ifuv_ori : 0.0;
          if (P.ipeel == 1 && !m.partial_peeloff)
            for (int peelid = 1; peelid <= m.npeel; ++peelid) peeloff(sip, ir, it, ip, idust2, peelid);
          ++iint;
        }
        tau = -log(ran());
        xpold = xp; ypold = yp; zpold = zp;
        ux = sint * cosp;
        uy = sint * sinp;
        uz = cost;
        const int pr = ir, pt = it, pp = ip;
        if (!tauint()) return 3;
        if (exitflag == 1) break;
        if (ir != pr || it != pt || ip != pp) iint = 0;
        if (m.iffuv && !is_fuv(nub)) return 2;
        if (iint > 10000 || ++nev > kMaxEvents) {
          atomicAdd(T.killed + cidx(ir, it, ip), 1);
          atomicAdd(T.scal + MCRT_S_ABFLUX, 1.0);
          return 1;
        }
        c = m.cells[cidx(ir, it, ip)];
        k = select_dust(c);
        if (k < 0) return 3;
      }
    }
    // exit binning (propagate_5_fuv.f90:231-320)
    int itb = (int)((double)m.nmu * (1.0 - cost) / 2.0) + 1;
    itb = min(max(itb, 1), m.nmu);
    if (phi < 0.0) phi = phi + R2P;
    int ipb = (int)((double)m.nph * phi / R2P) + 1;
    ipb = min(max(ipb, 1), m.nph);
    const double ub = __ldg(m.u + itb - 1);
    const double sini = __ldg(m.sini + itb - 1);
    const double x = ypold * cosp - xpold * sinp;
    const double y = zpold * sini - ypold * ub * sinp - xpold * ub * cosp;
    const double rho2 = x * x + y * y;
    if (rho2 < __ldg(m.aperture2 + m.nap - 1) * 1.0001) {
      atomicAdd(T.scal + MCRT_S_FLUX, 1.0);
      if (iflag == 1) {
        atomicAdd(T.scal + MCRT_S_SFLUX, 1.0);
        atomicAdd(T.scal + MCRT_S_NSCAT, (double)iscat);
      }
    }
    const int inub = freq_bin(nub);
    const int i_inter = (iflag == 1) ? 2 : ((i_orig == 1) ? 1 : 3);
    const int indx[3] = {1, 1 + i_orig, 5 + i_inter};
    for (int ia = 1; ia <= m.nap; ++ia) {
      if (rho2 < __ldg(m.aperture2 + ia - 1) && !(iflag == 0 && i_orig == 5)) {
        for (int kk = 0; kk < 3; ++kk) {
          const int64_t e = (inub - 1) + (int64_t)m.nfreq * ((itb - 1) + (int64_t)m.nmu * ((ipb - 1) + (int64_t)m.nph * ((ia - 1) + (int64_t)m.nap * (indx[kk] - 1))));
          double* S = T.sed + e;
          const int64_t ns = m.nsed;
          atomicAdd(S, sip); atomicAdd(S + ns, sqp); atomicAdd(S + 2 * ns, sup); atomicAdd(S + 3 * ns, svp);
          atomicAdd(S + 4 * ns, sip * sip); atomicAdd(S + 5 * ns, sqp * sqp);
          atomicAdd(S + 6 * ns, sup * sup); atomicAdd(S + 7 * ns, svp * svp);
          atomicAdd(S + 8 * ns, 1.0); atomicAdd(S + 9 * ns, fabs(cost));
        }
      }
    }
    if (iflag == 1) atomicAdd(T.scal + MCRT_S_SCOUNT, 1.0);
    return 0;
  }
};

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Persistent transport kernel: every thread fetches packets until the
// launch's range is exhausted.
__global__ void __launch_bounds__(kBlock) transport_fp64(LaunchParams P) {
  __shared__ double spec[5 * kMaxSlot * kBlock];
  Packet pk(P.m, P.t, spec);
  const int64_t n = P.hi - P.lo + 1;
  unsigned long long c_pkt = 0, c_int = 0, c_sca = 0, c_geo = 0, c_kil = 0, c_exit = 0, c_star = 0;
  for (;;) {
    const unsigned long long k = atomicAdd(P.next, 1ull);
    if ((int64_t)k >= n) break;
    const int64_t iphot = P.lo + (int64_t)k;
    pk.rng = rng_block(P.m, P.g1, P.g2, P.block0 + iphot - 1);
    const int st = pk.run(iphot, P);
    ++c_pkt;
    c_int += pk.nscat + pk.nabsev;
    c_sca += pk.nscat;
    c_star += pk.nstar;
    if (st == 3) ++c_geo;
    if (st == 1) ++c_kil;
    if (st == 0) ++c_exit;
    if (P.log && (int64_t)k < P.nlog) {
      mcrt_packet_log& L = P.log[k];
      L.iphot = iphot; L.nscat = pk.nscat; L.nabs = pk.nabsev; L.ncross = pk.ncross; L.nstar = pk.nstar;
      L.status = st; L.ir = 0; L.it = 0; L.ip = 0; L.ndraws = pk.rng.ndraws;
      L.iflag = pk.iflag; L.i_orig = pk.i_orig; L.pad = pk.ndiffev;
      L.nub = pk.nub; L.cost = pk.cost; L.phi = pk.phi; L.sip = pk.sip; L.sqp = pk.sqp; L.sup = pk.sup; L.svp = pk.svp;
      L.xp = pk.xp; L.yp = pk.yp; L.zp = pk.zp;
    }
  }
  // warp-aggregated statistics
  unsigned long long v[12] = {c_pkt, pk.c_cross, c_int, c_sca, pk.c_peel, pk.c_pcross, pk.c_pbin, c_geo,
                              pk.c_reset, c_kil, c_exit, c_star};
  for (int i = 0; i < 12; ++i) {
    unsigned long long s = warp_sum(v[i]);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(P.t.cnt + i, s);
  }
}

// End-of-iteration dust temperature of the diffusion cells: the state the
// reference's per-packet updates leave behind (emit_common_2.f90:260-339 with
// nacc = 0): the surface cell of a column that saw N diffusion absorptions
// holds min(Tmax, (T0^4 + N dT^4)^(1/4)); the interior cells whose
// neighbour toward the surface holds a thermal component take that value.
__global__ void diffusion_finalize(DevModel m, const int32_t* ndiff, const double* tdust0, double* tdust,
                                   double nphot) {
  const int64_t n = (int64_t)m.nrg * m.ntg * m.npg;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    double t = tdust0[c];
    const uint32_t fl = m.cells[c].flags;
    if (cell_diffus(fl)) {
      const int ir = (int)(c % m.nrg) + 1;
      const int it = (int)((c / m.nrg) % m.ntg) + 1;
      const int ip = (int)(c / ((int64_t)m.nrg * m.ntg)) + 1;
      auto ci = [&](int r, int tt, int p) { return (int64_t)(r - 1) + (int64_t)m.nrg * ((tt - 1) + (int64_t)m.ntg * (p - 1)); };
      const int dd = cell_diffdir(fl);
      int is = it, iwall;
      if (dd == -2) {
        while (is - 1 >= 1 && cell_diffus(m.cells[ci(ir, is - 1, ip)].flags)) --is;
        iwall = is;
      } else {
        while (is + 1 <= m.ntg - 1 && cell_diffus(m.cells[ci(ir, is + 1, ip)].flags)) ++is;
        iwall = is + 1;
      }
      const int64_t cs = ci(ir, is, ip);
      const int32_t N = ndiff[cs];
      bool gets = false;
      if (N > 0) {
        if (is == it) gets = cell_thermal(m.cells[cs].flags);
        else if (dd == -2) gets = cell_thermal(m.cells[ci(ir, it - 1, ip)].flags);
        else gets = cell_thermal(m.cells[ci(ir, it + 1, ip)].flags);
      }
      if (gets) {
        const double sth = m.sintarr[iwall - 1];
        const double dA = PI * sth * (m.rarr[ir] * m.rarr[ir] - m.rarr[ir - 1] * m.rarr[ir - 1]);
        double T4s = m.tstar * m.tstar;
        T4s = T4s * T4s;
        const double t0 = tdust0[cs];
        double T4d = t0 * t0;
        T4d = T4d * T4d;
        const double T4 = T4d + (double)N * (4.0 * PI * T4s / (nphot * dA));
        t = fmin(199999.0 / 11605.0, pow(T4, 0.25));
      }
    }
    tdust[c] = t;
  }
}

}  // namespace mcrt
