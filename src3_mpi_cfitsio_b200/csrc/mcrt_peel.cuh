// mcrt_peel.cuh -- peel-off kernel: walks every queued peel-off job to every
// inclination (peeloff_3d_2_test.f90:7-347 with findangle3.f90 and
// stokespeel.f90).
//
// The transport kernel queues one job per emission / scattering / absorption
// that the reference peels off; this kernel turns the queue into
// (job, inclination) work items.  Every lane of a warp walks one item, one
// cell crossing per loop iteration, in the same step code; binning and the
// start of the next item are batched like the transport kernel's events.
// A peel-off walk draws a random number only when testgrid must re-locate a
// position outside the grid (testgrid.f90:48-73), which a walk that starts
// inside the grid and stops at its boundary cannot reach; such draws come
// from a private stream here and are counted (MCRT_C_PEEL_RESETS).
#pragma once
#include "mcrt_transport.cuh"

namespace mcrt {

struct PeelLane {
  Packet pk;        // walk helpers (testgrid, faces, cell_opac, stokespeel, binning index)
  Ray ray;
  int state;        // 0 walk, 1 bin, 2 need item, 3 done, 5 adjoint re-walk
  int dir;
  unsigned long long item;
  double si;        // I weight of this direction
  int64_t steps;
  PeelJob J;
  double nub;       // the packet's frequency (filter-band images only)
  double adjC;      // adjoint forward pass: weighted contribution of the binned ray
  Rng rng0;         // stream state at the walk's start (the re-walk repeats it)

  __device__ PeelLane(const DevModel& m, const DevTallies& t, double* sbase) : pk(m, t, sbase) {
    state = 2;
    pk.rng.s1 = 1234567;
    pk.rng.s2 = 7654321;
    pk.rng.ndraws = 0;
  }

  // Start item k; false if the item produces no walk (direct peel-off away
  // from the observer, or a start on the stellar surface heading inward).
  __device__ bool start(const LaunchParams& P, unsigned long long k) {
    const DevModel& m = pk.m;
    const unsigned long long jid = k / (unsigned long long)m.npeel;
    dir = (int)(k % (unsigned long long)m.npeel) + 1;
    J = P.jobs[jid];
    nub = P.job_nub ? P.job_nub[jid] : 0.0;
    const double cospe = __ldg(m.cospe + dir - 1), sinpe = __ldg(m.sinpe + dir - 1);
    const double coste = __ldg(m.coste + dir - 1), sinte = __ldg(m.sinte + dir - 1);
    if (J.bits & 4u) {             // direct stellar peel-off (newdisktherm_5_fuv.f90:378-411)
      if (P.ips == 0) {
        const double cosnorm = J.d0 * coste + (J.d1 * sinte * (cospe * J.d2 + sinpe * J.d3));
        si = (m.limb == 0) ? 4.0 * J.si * cosnorm : 12.0 / 5.0 * J.si * (cosnorm + cosnorm * cosnorm);
        if (!(cosnorm > 0.0)) return false;
      } else {
        si = J.si * 2.0;
      }
    } else {
      si = J.si;
    }
    ++pk.c_peel;
    rng0 = pk.rng;
    for (int s = 0; s < kJobSlots && s < m.nslot; ++s) pk.sp.kapd(s) = J.kapd[s];
    return set_ray();
  }

  // The ray of (J, dir) at its start (peeloff_3d_2_test.f90:91-122); false
  // if it ends at once.
  __device__ bool set_ray() {
    const DevModel& m = pk.m;
    const double cospe = __ldg(m.cospe + dir - 1), sinpe = __ldg(m.sinpe + dir - 1);
    const double coste = __ldg(m.coste + dir - 1), sinte = __ldg(m.sinte + dir - 1);
    ray.x = J.x; ray.y = J.y; ray.z = J.z; ray.rs = J.rs; ray.rt = J.rt;
    ray.r = J.r; ray.t = J.t; ray.p = J.p; ray.onw = (J.bits & 1u) != 0; ray.peel = true; ray.tsum = 0.0;
#ifdef MCRT_MIXED
    ray.qready = false;
#endif
    ray.vx = sinte * cospe;
    ray.vy = sinte * sinpe;
    ray.vz = coste;
    steps = 0;
    if (ray.onw) {                 // peeloff_3d_2_test.f90:109-122
      const bool inner = fabs(ray.rs - __ldg(m.r2arr + ray.r - 1)) < fabs(ray.rs - __ldg(m.r2arr + ray.r));
      const bool outwards = ray.vx * ray.x + ray.vy * ray.y + ray.vz * ray.z > 0.0;
      if (inner && !outwards) {
        if (ray.r == 1) return false;
        ray.r = ray.r - 1;
      }
      if (!inner && outwards) ray.r = ray.r + 1;
    }
    return true;
  }

  // one crossing (peeloff_3d_2_test.f90:133-214); sets state 1 (bin) or 2
  // (done, no bin).  In the adjoint re-walk (state 5) the same crossings
  // scatter -C * tau per (cell, component) and the walk ends in state 2.
#ifdef MCRT_MIXED
  // Mixed build: the FP32 walk (QRay).  The bin reads the start point: the
  // image coordinates are projections along the peel-off direction.
  __device__ __forceinline__ void step(const LaunchParams& P) {
    const DevModel& m = pk.m;
    Ray& R = ray;
    QRay& g = R.g;
    if (!R.qready) {
      for (int s = 0; s < kJobSlots && s < m.nslot; ++s) pk.kf(s) = (float)J.kapd[s];
      pk.qbegin(g, R.x, R.y, R.z, R.vx, R.vy, R.vz, R.r, R.t, R.p);
      R.qready = true;
    }
    double qn = g.qr;
    int d = 0;
    if (g.qt < qn) { qn = g.qt; d = 1; }
    if (g.qp < qn) { qn = g.qp; d = 2; }
    if (!(qn < HUGE_D) || ++steps > P.walk_limit) { state = 2; return; }
    const float dt = (float)(qn - g.q);
    const int64_t ci = pk.cidx(R.r, R.t, R.p);
    const CellRecF c = m.cellsf[ci];
    float opac = 0.0f;
    const int n = cell_n(c.meta);
    for (int k = 0; k < n; ++k) opac = __fmaf_rn(pk.kf(cell_slot(c.meta, k)), c.rho[k], opac);
    R.tsum = __dadd_rn(R.tsum, (double)__fmul_rn(opac, dt));
    if (R.tsum > 25.0) { state = 2; return; }
    if (state == 5) {
      for (int k = 0; k < n; ++k)
        atomicAdd(P.adj.grad + ci + m.ncell * (cell_id(c.meta, k) - 1),
                  -(adjC * (double)(pk.kf(cell_slot(c.meta, k)) * c.rho[k] * dt)));
    }
    g.q = qn;
    R.onw = true;
    if (d == 0) {
      R.r += g.sr;
    } else if (d == 1) {
      R.t += g.st;
      if (R.t < 1 || R.t > m.ntg - 1) { state = 2; return; }   // no cell beyond a non-pole theta wall
    } else {
      R.p += g.sp;
      ++g.nphi;
      if (R.p == 0) R.p = m.npg - 1;
      if (R.p == m.npg) R.p = 1;
    }
    if (state != 5) ++pk.c_pcross;
    if (R.r == m.nrg) { state = (state == 5) ? 2 : 1; return; }
    if (R.r == 0) { state = 2; return; }
    if (d == 0) pk.qnext_r(g, R.r);
    else if (d == 1) pk.qnext_t(g, R.t, g.st);
    else pk.qnext_p(g, R.p);
  }
#else
  __device__ __forceinline__ void step(const LaunchParams& P) {
    const DevModel& m = pk.m;
    Ray& R = ray;
    pk.testgrid(R.x, R.y, R.z, R.rs, R.rt, R.r, R.t, R.p, R.onw);
    Walls w;
    w.reset();
    pk.faces(w, R.vx, R.vy, R.vz, R.x, R.y, R.z, R.r, R.t, R.p);
    double dt;
    int iface;
    w.next(R.onw, dt, iface);
    if (dt == HUGE_D || iface < 1 || iface > 6 || ++steps > P.walk_limit) { state = 2; return; }
    const int64_t ci = pk.cidx(R.r, R.t, R.p);
    const CellRec c = m.cells[ci];
    R.tsum = R.tsum + pk.cell_opac(c) * dt;
    if (R.tsum > 25.0) { state = 2; return; }
    if (state == 5) {
      const int n = cell_n(c.meta);
      for (int k = 0; k < n; ++k)
        atomicAdd(P.adj.grad + ci + m.ncell * (cell_id(c.meta, k) - 1),
                  -(adjC * (pk.sp.kapd(cell_slot(c.meta, k)) * c.rho[k] * dt)));
    }
    pk.step_index(iface, R.r, R.t, R.p);
    R.x = R.x + dt * R.vx;
    R.y = R.y + dt * R.vy;
    R.z = R.z + dt * R.vz;
    R.onw = true;
    R.rs = R.x * R.x + R.y * R.y + R.z * R.z;
    R.rt = sqrt(R.rs);
    if (state != 5) ++pk.c_pcross;
    if (R.r == m.nrg) { state = (state == 5) ? 2 : 1; return; }
    if (R.r == 0) { state = 2; return; }
  }
#endif

  // peeloff_3d_2_test.f90:217-345
  __device__ void bin(const LaunchParams& P) {
    const DevModel& m = pk.m;
    const int id = dir;
    ++pk.c_pbin;
    const double cospe = __ldg(m.cospe + id - 1), sinpe = __ldg(m.sinpe + id - 1);
    const double coste = __ldg(m.coste + id - 1), sinte = __ldg(m.sinte + id - 1);
    const double factor = exp(-ray.tsum);
    double qi = si * factor, qq = J.sq * factor, qu = J.su * factor, qv = J.sv * factor;
    const bool scattered = (J.bits & 2u) != 0;
    if (scattered) {
      const double cost = J.d0, sint = J.d1, cosp = J.d2, sinp = J.d3, phi = J.d4;
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
      if (m.mueller) {       // the job carries the table row and wavelength weight
        pk.stokespeel6(qi, qq, qu, qv, coste, sinte, ri1, costnew, cost, sint, (int)J.pl, J.g);
      } else {
        pk.sp.g(0) = J.g;
        pk.sp.pl(0) = J.pl;
        pk.stokespeel(qi, qq, qu, qv, coste, sinte, ri1, costnew, cost, sint, 0);
      }
    }
    const double x1 = ray.x, y1 = ray.y, z1 = ray.z;
    const double yimage = z1 * sinte - y1 * coste * sinpe - x1 * coste * cospe;
    const double ximage = y1 * cospe - x1 * sinpe;
    const double vx = (ximage + m.rmaxi) / m.fractxh, vy = (yimage + m.rmaxi) / m.fractxh;
    const double rho2 = ximage * ximage + yimage * yimage;
    const int inub = (int)(J.bits >> 8) + 1;
    const int i_orig = (int)((J.bits >> 3) & 31u);
    const DevTallies& T = pk.T;
    const bool adj = P.adj.mode == 1;
    adjC = 0.0;
    if (m.output_imcube && vx > -1.0e9 && vx < 1.0e9 && vy > -1.0e9 && vy < 1.0e9) {
      const int ix = (int)vx + 1, iy = (int)vy + 1;
      if (ix <= m.nxhst && iy <= m.nxhst && ix > 0 && iy > 0) {
        const int64_t k = (int64_t)(id - 1) + (int64_t)m.npeel * ((ix - 1) + (int64_t)m.nxhst * ((iy - 1) + (int64_t)m.nxhst * (inub - 1)));
        if (adj && P.adj.lam_img) adjC += P.adj.lam_img[k] * qi;
        atomicAdd(T.img + k, qi);
        atomicAdd(T.img + m.nimg + k, qq);
        atomicAdd(T.img + 2 * m.nimg + k, qu);
        atomicAdd(T.img + 3 * m.nimg + k, qv);
      }
    }
    bin_filters(m, T, id, vx, vy, nub, i_orig, qi, qq, qu, qv);
    bin_nested(m, T, id, ximage, yimage, nub, qi, qq, qu, qv);
    const int i_inter = scattered ? 2 : ((i_orig == 1) ? 1 : 3);
    const int indx[3] = {1, 1 + i_orig, 5 + i_inter};
    for (int ia = 1; ia <= m.nap; ++ia) {
      if (rho2 < __ldg(m.aperture2 + ia - 1)) {
        for (int k = 0; k < 3; ++k) {
          const int64_t e = (inub - 1) + (int64_t)m.nfreq * ((id - 1) + (int64_t)m.npeel * ((ia - 1) + (int64_t)m.nap * (indx[k] - 1)));
          if (adj) adjC += P.adj.lam_psed[e] * qi;
          double* Q = T.psed + e;
          atomicAdd(Q, qi); atomicAdd(Q + m.npsed, qq); atomicAdd(Q + 2 * m.npsed, qu); atomicAdd(Q + 3 * m.npsed, qv);
          atomicAdd(Q + 4 * m.npsed, qi * qi); atomicAdd(Q + 5 * m.npsed, qq * qq);
          atomicAdd(Q + 6 * m.npsed, qu * qu); atomicAdd(Q + 7 * m.npsed, qv * qv);
          atomicAdd(Q + 8 * m.npsed, 1.0);
        }
      }
    }
  }
};

// Persistent peel-off kernel over the (job, inclination) items queued by the
// preceding transport launch (the job count is read on the device).
#ifndef MCRT_PEEL_MIN_BLOCKS
#define MCRT_PEEL_MIN_BLOCKS 1
#endif
__global__ void __launch_bounds__(kBlock, MCRT_PEEL_MIN_BLOCKS) peel_sched(LaunchParams P, unsigned long long* next_item) {
  __shared__ double spec[5 * kMaxSlot * kBlock];
  PeelLane L(P.m, P.t, spec);
  const unsigned FULL = 0xffffffffu;
  const int batch = P.event_batch > 0 ? P.event_batch : 16;
  unsigned long long njobs = *P.njobs;
  if ((int64_t)njobs > P.job_cap) njobs = (unsigned long long)P.job_cap;
  const unsigned long long nitems = njobs * (unsigned long long)P.m.npeel;
  for (;;) {
    const bool stepping = L.state == 0 || L.state == 5;
    const bool pending = L.state == 1 || L.state == 2;
    const unsigned s = __ballot_sync(FULL, stepping);
    const unsigned e = __ballot_sync(FULL, pending);
    if (s == 0u && e == 0u) break;
    if (s == 0u || __popc(e) >= batch) {
      if (pending) {
        if (L.state == 1) {
          L.bin(P);
          L.state = 2;
          if (P.adj.mode == 1 && L.adjC != 0.0) {
            // adjoint forward pass: record the job's contribution, then walk
            // the ray again (same stream state) to scatter -C * tau
            const unsigned long long jid = L.item / (unsigned long long)P.m.npeel;
            const int64_t r = P.adj.rec_base + (int64_t)jid;
            if (r < P.adj.rec_cap) {
              P.adj.rec_key[r] = ((unsigned long long)L.J.pkt << kAdjEvBits) | (unsigned long long)L.J.ev;
              atomicAdd(P.adj.rec_c + r, L.adjC);
            } else {
              atomicAdd(P.err, 1);
            }
            atomicAdd(P.adj.obj, L.adjC);
            L.pk.rng = L.rng0;
            if (L.set_ray()) L.state = 5;
          }
        }
        while (L.state == 2) {
          const unsigned long long k = atomicAdd(next_item, 1ull);
          if (k >= nitems) { L.state = 3; break; }
          L.item = k;
          if (L.start(P, k)) L.state = 0;
        }
      }
    } else if (stepping) {
      L.step(P);
    }
  }
  unsigned long long v[4] = {L.pk.c_peel, L.pk.c_pcross, L.pk.c_pbin, L.pk.c_reset};
  const int slot[4] = {MCRT_C_PEELS, MCRT_C_PEEL_CROSS, MCRT_C_PEEL_BINNED, MCRT_C_PEEL_RESETS};
  for (int i = 0; i < 4; ++i) {
    unsigned long long x = warp_sum(v[i]);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(P.t.cnt + slot[i], x);
  }
}

}  // namespace mcrt
