// mcrt_setemiss.cuh -- emission tables of the Lucy reemission on the GPU.
//
// The reference builds these once per run in setemiss (dust_5.f90:507-699),
// splitting the species over its MPI ranks: for every opacity species and
// each of nT=500 temperatures it integrates, over 513 frequency intervals of
// x = h nu / kT, the absorption opacity times the normalised Planck function
// (the cumulative table kapint that lucydustfreq samples) and dB_nu/dT over
// the total opacity (the Rosseland mean kappar); the last cumulative value is
// the Planck mean kappap.  Each interval is integrated by qsimp (trapezoid
// refinement with the Simpson combination, relative tolerance 1e-5, at most
// 20 levels; nr_2.f:209-254), the opacities are linear in nu between the
// interval's end points (kappaB/chidB, dust_5.f90:784-831), B_nu and dB_nu/dT
// use the reference's expm1 (the Abramowitz & Stegun 4.2.45 expansion below
// ln 2, mathsubs.f90:4-47, 79-113).
//
// Here one block takes one (temperature, species) pair: its threads
// integrate the 513 intervals independently (the rare interval that needs
// more than 10 refinement levels is finished by the whole block), then one
// thread forms the cumulative sums in the reference's order (so the tables
// do not depend on the thread count) and the block normalises.  The second kernel smooths the
// Planck mean of gas opacities (species > ndg) as the reference does.  This
// translation unit is compiled without FMA contraction, so the arithmetic
// follows the reference's operation for operation; exp() is the only
// function evaluated.
#pragma once
#include <cstdint>

#include "mcrt_device.cuh"

namespace mcrt {

namespace setemiss {

__device__ __forceinline__ double expm1_as(double x) {
  if (fabs(x) > 0.6931472) return exp(x) - 1.0;
  // A&S 4.2.45 coefficients, innermost (x^7) first
  double s = 0.0;
  s = x * (0.0001413161 + s);
  s = x * (0.0013298820 + s);
  s = x * (0.0083013598 + s);
  s = x * (0.0416573475 + s);
  s = x * (0.1666653019 + s);
  s = x * (0.4999999206 + s);
  s = x * (0.9999999995 + s);
  return s;
}

__device__ __forceinline__ double planck(double nu, double T) {
  const double x = nu / T;
  if (x == 0.0) return 0.0;
  return 0.1539897 * x * x * x / expm1_as(x);
}

__device__ __forceinline__ double dplanck(double nu, double T) {
  const double x = nu / T;
  if (x == 0.0) return 0.0;
  return -(0.1539897 * x * x * x * x) / (4.0 * expm1_as(x) * expm1_as(-x));
}

__device__ __forceinline__ void interp(const double* nud, const double* kd, const double* ad, int n, double nu,
                                       double& kap, double& alb) {
  if (nu >= __ldg(nud)) { kap = __ldg(kd); alb = __ldg(ad); return; }
  if (nu <= __ldg(nud + n - 1)) { kap = __ldg(kd + n - 1); alb = __ldg(ad + n - 1); return; }
  int i0 = 1, i1 = n;
  while (i1 - i0 > 1) {
    const int i = (i1 + i0) >> 1;
    if (nu <= __ldg(nud + i - 1)) i0 = i; else i1 = i;
  }
  const double f = (nu - __ldg(nud + i1 - 1)) / (__ldg(nud + i0 - 1) - __ldg(nud + i1 - 1));
  const double fm1 = 1.0 - f;
  kap = fm1 * __ldg(kd + i1 - 1) + f * __ldg(kd + i0 - 1);
  alb = fm1 * __ldg(ad + i1 - 1) + f * __ldg(ad + i0 - 1);
}

// qsimp on [0, 1] as a resumable state: `level` trapezoid levels done, `st`
// the last trapezoid sum, `os`/`ost` the previous Simpson and trapezoid
// values (both -1e30 before the first level), `s` the current estimate.
struct QSimp {
  double st, ost, os, s;
  int level;
  bool done;
  __device__ __forceinline__ void init() { st = 0.0; ost = -1.0e30; os = -1.0e30; s = 0.0; level = 0; done = false; }
  // the Simpson combination and the convergence test after a level
  __device__ __forceinline__ void finish_level() {
    s = (4.0 * st - ost) / 3.0;
    if (fabs(s - os) < 1.0e-5 * fabs(os)) { done = true; return; }
    os = s;
    ost = st;
  }
};

// levels up to `upto` in this thread, with the reference's point recurrence
template <class F>
__device__ void qsimp_serial(const F& fn, QSimp& q, int upto) {
  while (!q.done && q.level < upto) {
    const int j = ++q.level;
    if (j == 1) {
      q.st = 0.5 * 1.0 * (fn(0.0) + fn(1.0));
    } else {
      const long long it = 1LL << (j - 2);
      const double tnm = (double)it;
      const double del = 1.0 / tnm;
      double x = 0.5 * del, sum = 0.0;
      for (long long k = 0; k < it; ++k) { sum = sum + fn(x); x = x + del; }
      q.st = 0.5 * (q.st + 1.0 * sum / tnm);
    }
    q.finish_level();
  }
}

// One interval's end-point opacities (opacset at nuint(j-1) T and nuint(j) T;
// nu = 0 below the first node) and its width in nu and in x.
struct Interval {
  double nu0, dnu, dx, T, kap0, kap1, chi0, chi1;
  __device__ __forceinline__ void set(const SetemissArgs& a, const double* nud, const double* kd, const double* ad,
                                      int n, int j, double Tj) {
    T = Tj;
    nu0 = j == 0 ? 0.0 : a.nuint[j - 1] * T;
    const double nu1 = a.nuint[j] * T;
    double k0, a0, k1, a1;
    interp(nud, kd, ad, n, nu0, k0, a0);
    interp(nud, kd, ad, n, nu1, k1, a1);
    chi0 = k0; kap0 = (1.0 - a0) * k0; chi1 = k1; kap1 = (1.0 - a1) * k1;
    dnu = nu1 - nu0;
    dx = dnu / T;
  }
  // kappaB (which = 0) and chidB (which = 1) of dust_5.f90:784-831
  __device__ __forceinline__ double eval(int which, double f) const {
    if (which == 0) return ((1.0 - f) * kap0 + f * kap1) * planck(nu0 + f * dnu, T);
    return dplanck(nu0 + f * dnu, T) / ((1.0 - f) * chi0 + f * chi1);
  }
};

}  // namespace setemiss

// Integrals that have not converged after kSerialLevels levels (a few in a
// thousand: mostly Rosseland integrands across a steep opacity change) are
// finished by the whole block, level by level, each level's points spread
// over the threads and summed by a fixed tree.  Up to there every interval
// follows the reference's sequence of points and sums exactly.
constexpr int kSerialLevels = 10;
constexpr int kDeferCap = 32;
constexpr int kSetemissBlock = 128;

// grid (nT, nopac); dynamic shared memory 2 * nnu doubles
__global__ void __launch_bounds__(kSetemissBlock) setemiss_tables(SetemissArgs a) {
  extern __shared__ double sm[];
  double* cum = sm;              // [nnu] dx * kappaB integral, then the cumulative sum
  double* ros = sm + a.nnu;      // [nnu] dx * chidB integral
  __shared__ setemiss::QSimp dq[kDeferCap];
  __shared__ int dj[kDeferCap], dwhich[kDeferCap];
  __shared__ int ndefer;
  __shared__ double red[kSetemissBlock];
  __shared__ int level_done;
  const int i = blockIdx.x, id = blockIdx.y;
  const int nnu = a.nnu, nT = a.nT;
  const double* nud = a.nudust + (int64_t)a.nlammax * id;
  const double* kd = a.kappad + (int64_t)a.nlammax * id;
  const double* ad = a.adust + (int64_t)a.nlammax * id;
  const int n = a.nlambda[id];
  const double T = a.Tint[i];
  if (threadIdx.x == 0) ndefer = 0;
  __syncthreads();
  unsigned long long miss = 0;
  for (int j = threadIdx.x; j < nnu; j += blockDim.x) {
    setemiss::Interval v;
    v.set(a, nud, kd, ad, n, j, T);
    double res[2] = {0.0, 0.0};
    if (v.nu0 / T < 50.0) {
      for (int which = 0; which < 2; ++which) {
        setemiss::QSimp q;
        q.init();
        setemiss::qsimp_serial([&](double f) { return v.eval(which, f); }, q, kSerialLevels);
        if (!q.done) {
          const int slot = atomicAdd(&ndefer, 1);
          if (slot < kDeferCap) {            // the block finishes it below
            dq[slot] = q;
            dj[slot] = j;
            dwhich[slot] = which;
            continue;
          }
          setemiss::qsimp_serial([&](double f) { return v.eval(which, f); }, q, 20);
        }
        if (!q.done) ++miss;
        res[which] = q.s;
      }
    }
    cum[j] = v.dx * res[0];
    ros[j] = v.dx * res[1];
  }
  __syncthreads();
  const int nd = min(ndefer, kDeferCap);
  for (int e = 0; e < nd; ++e) {
    setemiss::Interval v;
    v.set(a, nud, kd, ad, n, dj[e], T);
    const int which = dwhich[e];
    for (;;) {
      const int j = dq[e].level + 1;
      if (j > 20) break;
      const long long it = 1LL << (j - 2);
      const double del = 1.0 / (double)it;
      double part = 0.0;
      for (long long k = threadIdx.x; k < it; k += blockDim.x) part = part + v.eval(which, ((double)k + 0.5) * del);
      red[threadIdx.x] = part;
      __syncthreads();
      for (int w = kSetemissBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        __syncthreads();
      }
      if (threadIdx.x == 0) {
        setemiss::QSimp& q = dq[e];
        q.level = j;
        q.st = 0.5 * (q.st + 1.0 * red[0] / (double)it);
        q.finish_level();
        level_done = q.done ? 1 : 0;
      }
      __syncthreads();
      if (level_done) break;
    }
    if (threadIdx.x == 0) {
      if (!dq[e].done) ++miss;
      (which == 0 ? cum : ros)[dj[e]] = v.dx * dq[e].s;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {      // the reference's summation order
    double c = cum[0], r = ros[0];
    for (int j = 1; j < nnu; ++j) {
      c = cum[j] + c;
      cum[j] = c;
      r = ros[j] + r;
    }
    a.kappar[i + (int64_t)nT * id] = 1.0 / r;
    a.kappap[i + (int64_t)nT * id] = cum[nnu - 1];
  }
  __syncthreads();
  const double top = cum[nnu - 1];
  for (int j = threadIdx.x; j < nnu; j += blockDim.x)
    a.kapint[i + (int64_t)nT * (j + (int64_t)nnu * id)] = j == nnu - 1 ? 1.0 : cum[j] / top;
  for (int o = 16; o > 0; o >>= 1) miss += __shfl_down_sync(0xffffffffu, miss, o);
  if ((threadIdx.x & 31) == 0 && miss) atomicAdd(a.misses, miss);
}

// Two passes of the 21-point box average of the Planck mean of the gas
// species (ids ndg+1..nopac), the window shrinking symmetrically at the ends
// (dust_5.f90:623-663).  One thread per species; `tmp` holds nT doubles per
// species.
__global__ void setemiss_smooth(double* kappap, double* tmp, int nT, int ndg, int nopac) {
  const int id = ndg + blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= nopac) return;
  double* kp = kappap + (int64_t)nT * id;
  double* out = tmp + (int64_t)nT * (id - ndg);
  const int ns = 10;
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

}  // namespace mcrt
