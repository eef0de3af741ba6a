// mcrt_sched.cuh -- warp-scheduled photon-packet transport for sm_100a.
//
// The same physics as the per-thread kernel of mcrt_transport.cuh (the
// reference's packet loop, newdisktherm_5_fuv.f90:220-491), reorganised for
// SIMT execution:
//
//  * every lane holds one packet and, at any moment, either one ray to step
//    (the packet's own walk, tauint_3d_2_fuv.f90:34-208, or one peel-off walk,
//    peeloff_3d_2_test.f90:126-215) or a pending event;
//  * ray stepping is one shared code path: each loop iteration advances every
//    stepping lane by one cell crossing, so the hot loop stays small and the
//    warp stays converged whether a lane walks its packet or a peel-off;
//  * events (emission, interaction, peel-off binning, exit binning) are
//    deferred until at least `event_batch` lanes of the warp wait (or no lane
//    has a ray), then run together, so the long scattering / reemission code
//    runs with many lanes active instead of one.
//
// Each lane executes its packet's steps in the reference's order, so every
// packet consumes its random stream exactly as the per-thread kernel and the
// CPU oracle do (event-for-event parity is unchanged).
#pragma once
#include "mcrt_transport.cuh"

namespace mcrt {

enum Ev : int {
  EV_NONE = 0,       // stepping a ray
  EV_FETCH,          // start the next packet
  EV_PROP_START,     // propagate entry: first tau, packet walk
  EV_AFTER_WALK,     // packet walk stopped at an interaction point
  EV_PEEL_NEXT,      // next direction of the current peel-off sequence
  EV_PEEL_BIN,       // a peel-off walk left the grid
  EV_SCATTER_DONE,   // peel-offs of a scattering done: stokes, next tau
  EV_ABSORB_DONE,    // peel-offs of an absorption done: next tau
  EV_NEXT_TAU,       // sample tau, resume the packet walk
  EV_EXIT,           // packet left the grid: SED binning
  EV_FINISH,         // packet finished (status set)
  EV_STAR,           // packet walk reached the stellar surface (wavefront walk only)
  EV_DONE            // no packets left for this lane
};
enum PeelCtx : int { PC_DIRECT = 0, PC_SCATTER = 1, PC_ABSORB = 2, PC_ACCRETION = 3 };

struct Ray {
  double x, y, z, rs, rt, vx, vy, vz, tsum;   // mixed build: x..rt = the walk's start point
  int r, t, p;
  bool onw, peel;
#ifdef MCRT_MIXED
  bool qready;                                 // g set up for this walk
  QRay g;
#endif
};

struct Lane {
  Packet pk;
  Ray ray;
  int ev, status;
  int iscat, iint, first, slot_s;
  int prev_r, prev_t, prev_p;
  int64_t nev, iphot, kfetch;
  double xpold, ypold, zpold;
  int peel_ctx, peelid, peel_idust2;
  double peel_si, coslp, sinlp;
  unsigned long long c_pkt, c_int, c_sca, c_geo, c_kil, c_exit, c_star, c_jobs;
  // the integer-valued scalar tallies (MCRT_S_*), counted per lane and added
  // once per warp when the kernel ends: every exit and first interaction
  // otherwise adds to the same few addresses
  unsigned long long s_cnt[MCRT_NSCALARS];
  int64_t ray_steps;
  double adjA;                      // replay: summed C of the packet's peel-offs still ahead
  double adjB;                      // replay: the control variate of the current segment
  int64_t adj_pos, adj_end;         // replay: the packet's next record

  __device__ Lane(const DevModel& m, const DevTallies& t, double* sbase, float* fbase = nullptr) : pk(m, t, sbase, fbase) {
#ifdef MCRT_MIXED
    ray.qready = false;
#endif
    ev = EV_FETCH;
    status = 0;
    c_pkt = c_int = c_sca = c_geo = c_kil = c_exit = c_star = c_jobs = 0;
#pragma unroll
    for (int i = 0; i < MCRT_NSCALARS; ++i) s_cnt[i] = 0;
  }

  __device__ __forceinline__ void ray_from_packet(bool peel) {
    ray.x = pk.xp; ray.y = pk.yp; ray.z = pk.zp; ray.rs = pk.rsq; ray.rt = pk.rtot;
    ray.r = pk.ir; ray.t = pk.it; ray.p = pk.ip; ray.onw = pk.on_wall; ray.peel = peel;
    ray.tsum = 0.0;
    ray_steps = 0;
#ifdef MCRT_MIXED
    ray.qready = false;
#endif
  }
#ifdef MCRT_MIXED
  // The packet at the walk's current point: start + (q - q0) u in FP64.
  __device__ __forceinline__ void packet_from_ray() {
    Packet::qpos(ray.x, ray.y, ray.z, ray.vx, ray.vy, ray.vz, ray.g.q, ray.g.q0, pk.xp, pk.yp, pk.zp, pk.rsq, pk.rtot);
    pk.ir = ray.r; pk.it = ray.t; pk.ip = ray.p; pk.on_wall = ray.onw;
  }
#else
  __device__ __forceinline__ void packet_from_ray() {
    pk.xp = ray.x; pk.yp = ray.y; pk.zp = ray.z; pk.rsq = ray.rs; pk.rtot = ray.rt;
    pk.ir = ray.r; pk.it = ray.t; pk.ip = ray.p; pk.on_wall = ray.onw;
  }
#endif
  __device__ __forceinline__ void start_walk() {
    ray_from_packet(false);
    ray.vx = pk.ux; ray.vy = pk.uy; ray.vz = pk.uz;
    ev = EV_NONE;
  }

  // Stellar-surface hit inside the packet walk: re-emission from the surface
  // with the sampled tau kept (tauint_3d_2_fuv.f90:184-206).  The packet
  // position has been copied from the ray.
  __device__ void star_reemit() {
    const DevModel& m = pk.m;
    ++s_cnt[MCRT_S_AFLUX];
    ++pk.nstar;
    pk.rtot = sqrt(pk.rsq);
    pk.initpabs();
    pk.opacset(pk.nub, KAPD_TAUINT);
    pk.ifuv = Packet::is_fuv(pk.nub) ? m.ifuv_ori : 0.0;
    pk.i_orig = 1;
    pk.iflag = 0;
    pk.ir = 1;
    const double tsave = 0.0;
    ray_from_packet(false);
    ray.vx = pk.ux; ray.vy = pk.uy; ray.vz = pk.uz;
    ray.tsum = tsave;
  }

  // ---------------------------------------------------------- ray step
  // One cell crossing of the current ray: tauint_3d_2_fuv.f90:36-206 for the
  // packet walk, peeloff_3d_2_test.f90:133-214 for a peel-off walk.  With
  // kStarEvent the stellar-surface hit ends the step with EV_STAR instead of
  // re-emitting in place, so that the walk needs only the opacity and
  // albedo columns of the species state (kapd, alb).
#ifdef MCRT_MIXED
  // Mixed build: one crossing of the FP32 walk (QRay, mcrt_transport.cuh)
  // with the same outcomes as the FP64 step below.  A ray's peel-off bin
  // reads the start point: the image coordinates are projections along the
  // peel-off direction, the same for every point of the ray.  With
  // kStarEvent (the walk kernel) the walk is set up by the record load and
  // the packet position is formed by the record save (wave_save_qwalk), so
  // the start point is not held through the walk.
  template <bool kStarEvent = false>
  __device__ __forceinline__ void step(const LaunchParams& P) {
    const DevModel& m = pk.m;
    Ray& R = ray;
    QRay& g = R.g;
    if (!kStarEvent && !R.qready) {
      pk.walk_columns();
      pk.qbegin(g, R.x, R.y, R.z, R.vx, R.vy, R.vz, R.r, R.t, R.p);
      R.qready = true;
    }
    double qn = g.qr;
    int d = 0;
    if (g.qt < qn) { qn = g.qt; d = 1; }
    if (g.qp < qn) { qn = g.qp; d = 2; }
    if (!(qn < HUGE_D) || ++ray_steps > P.walk_limit) {
      if (!R.peel) { if (!kStarEvent) packet_from_ray(); status = 3; ev = EV_FINISH; }
      else ev = EV_PEEL_NEXT;
      return;
    }
    const double dt = __dsub_rn(qn, g.q);
    const int64_t ci = pk.cidx(R.r, R.t, R.p);
    const CellRecF c = m.cellsf[ci];
    float opac, absc;
    pk.cell_coefs(c, opac, absc);
    if (!R.peel) {
      const double dtau = (double)__fmul_rn(opac, (float)dt);
      // The walk piece in this cell: to the interaction point if the
      // sampled tau is reached here (tauint :69-111), else the whole crossing.
      const bool hit = __dadd_rn(R.tsum, dtau) > pk.tau;
      const double len = hit ? __ddiv_rn(__dsub_rn(pk.tau, R.tsum), (double)opac) : dt;
      pk.tally_absf(ci, absc, len);
      if (P.adj.mode == 2) adjoint_scoref(P, ci, c, (float)len);
      if (hit) {
        g.q = __dadd_rn(g.q, len);
        R.onw = false;
        if (!kStarEvent) packet_from_ray();
        ev = EV_AFTER_WALK;
        return;
      }
      R.tsum = __dadd_rn(R.tsum, dtau);
    } else {
      R.tsum = __dadd_rn(R.tsum, (double)__fmul_rn(opac, (float)dt));
      if (R.tsum > 25.0) { ev = EV_PEEL_NEXT; return; }
    }
    g.q = qn;
    R.onw = true;
    if (d == 0) {
      R.r += g.sr;
    } else if (d == 1) {
      R.t += g.st;
      if (R.t < 1 || R.t > m.ntg - 1) {       // a theta wall that is not a pole was left: no cell beyond
        if (!R.peel) { if (!kStarEvent) packet_from_ray(); status = 3; ev = EV_FINISH; }
        else ev = EV_PEEL_NEXT;
        return;
      }
    } else {
      R.p += g.sp;
      ++g.nphi;
      if (R.p == 0) R.p = m.npg - 1;
      if (R.p == m.npg) R.p = 1;
    }
    if (!R.peel) {
      ++pk.ncross;
      ++pk.c_cross;
      if (R.r == m.nrg) { pk.exitflag = 1; if (!kStarEvent) packet_from_ray(); ev = EV_EXIT; return; }
      if (R.r == 0) {                 // star hit: re-emission, tau kept (tauint_3d_2_fuv.f90:184-206)
        if (!kStarEvent) packet_from_ray();
        if (kStarEvent) { ev = EV_STAR; return; }
        star_reemit();
        return;
      }
    } else {
      ++pk.c_pcross;
      if (R.r == m.nrg) { ev = EV_PEEL_BIN; return; }
      if (R.r == 0) { ev = EV_PEEL_NEXT; return; }
    }
    if (d == 0) pk.qnext_r(g, R.r);
    else if (d == 1) pk.qnext_t(g, R.t, g.st);
    else pk.qnext_p(g, R.p);
  }

  // Replay: -A * tau of a walk piece in cell ci, per component (FP32 cell).
  __device__ __forceinline__ void adjoint_scoref(const LaunchParams& P, int64_t ci, const CellRecF& c, float len) {
    const double w = adjA - adjB;
    if (w == 0.0) return;
    const int n = cell_n(c.meta);
    for (int k = 0; k < n; ++k) {
      const int id = cell_id(c.meta, k);
      atomicAdd(P.adj.grad + ci + pk.m.ncell * (id - 1), -(w * (double)(pk.kf(cell_slot(c.meta, k)) * c.rho[k] * len)));
    }
  }
#else
  template <bool kStarEvent = false>
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
    const bool bad = dt == HUGE_D || iface < 1 || iface > 6 || ++ray_steps > P.walk_limit;
    if (!R.peel) {
      if (bad || dt < 0.0) { packet_from_ray(); status = 3; ev = EV_FINISH; return; }
    } else if (bad) {
      ev = EV_PEEL_NEXT;
      return;
    }
    const int64_t ci = pk.cidx(R.r, R.t, R.p);
    const CellRec c = m.cells[ci];
    const double opac = pk.cell_opac(c);
    double dtau = 0.0;
    if (!R.peel) {
      dtau = opac * dt;
      if (R.tsum + dtau > pk.tau) {
        const double ds = (pk.tau - R.tsum) / opac;
        pk.tally_abs(ci, c, ds);
        if (P.adj.mode == 2) adjoint_score(P, ci, c, ds);
        R.x = R.x + ds * R.vx;
        R.y = R.y + ds * R.vy;
        R.z = R.z + ds * R.vz;
        R.rs = R.x * R.x + R.y * R.y + R.z * R.z;
        R.rt = sqrt(R.rs);
        R.onw = false;
        packet_from_ray();
        ev = EV_AFTER_WALK;
        return;
      }
      pk.tally_abs(ci, c, dt);
      if (P.adj.mode == 2) adjoint_score(P, ci, c, dt);
    } else {
      R.tsum = R.tsum + opac * dt;
      if (R.tsum > 25.0) { ev = EV_PEEL_NEXT; return; }
    }
    pk.step_index(iface, R.r, R.t, R.p);
    R.x = R.x + dt * R.vx;
    R.y = R.y + dt * R.vy;
    R.z = R.z + dt * R.vz;
    R.onw = true;
    R.rs = R.x * R.x + R.y * R.y + R.z * R.z;
    R.rt = sqrt(R.rs);
    if (!R.peel) {
      R.tsum = R.tsum + dtau;
      ++pk.ncross;
      ++pk.c_cross;
      if (R.r == m.nrg) { pk.exitflag = 1; packet_from_ray(); ev = EV_EXIT; return; }
      if (R.r == 0) {                 // star hit: re-emission, tau kept (tauint_3d_2_fuv.f90:184-206)
        packet_from_ray();
        if (kStarEvent) { ev = EV_STAR; return; }
        star_reemit();
      }
    } else {
      ++pk.c_pcross;
      if (R.r == m.nrg) { ev = EV_PEEL_BIN; return; }
      if (R.r == 0) { ev = EV_PEEL_NEXT; return; }
    }
  }
#endif

  // ------------------------------------------------------------ adjoint
  // Replay: -A * tau of a walk piece of length len in cell ci, per component.
  __device__ __forceinline__ void adjoint_score(const LaunchParams& P, int64_t ci, const CellRec& c, double len) {
    const double w = adjA - adjB;
    if (w == 0.0) return;
    const int n = cell_n(c.meta);
    for (int k = 0; k < n; ++k) {
      const int id = cell_id(c.meta, k);
      atomicAdd(P.adj.grad + ci + pk.m.ncell * (id - 1), -(w * (pk.sp.kapd(cell_slot(c.meta, k)) * c.rho[k] * len)));
    }
  }
  // Replay: before the walk that follows event k (0 = emission, else the
  // k-th interaction), drop that event's peel-offs from A.
  __device__ __forceinline__ void adjoint_advance(const LaunchParams& P) {
    if (P.adj.mode != 2) return;
    const unsigned long long k = (unsigned long long)(pk.nscat + pk.nabsev);
    const unsigned long long mask = (1ull << kAdjEvBits) - 1ull;
    while (adj_pos < adj_end && (P.adj.skey[adj_pos] & mask) <= k) adjA -= P.adj.sc[adj_pos++];
    if (P.adj.vtab || P.adj.vsum) {   // the control variate's (cell, frequency, direction) bin
      int fb = (int)((double)P.adj.nfb * (log(pk.nub) - P.adj.lnumin) / P.adj.lnurat);
      fb = min(max(fb, 0), P.adj.nfb - 1);
      int db = 0;
      if (P.adj.ndir == 4) {          // outward / inward radially, away from / toward the midplane
        const double ux = pk.sint * pk.cosp, uy = pk.sint * pk.sinp, uz = pk.cost;
        db = (ux * pk.xp + uy * pk.yp + uz * pk.zp > 0.0 ? 1 : 0) + (uz * pk.zp > 0.0 ? 2 : 0);
      }
      const int64_t v = (pk.cidx(pk.ir, pk.it, pk.ip) * P.adj.nfb + fb) * P.adj.ndir + db;
      if (P.adj.vtab) adjB = P.adj.vtab[v];
      if (P.adj.vsum) { atomicAdd(P.adj.vsum + v, adjA); atomicAdd(P.adj.vcnt + v, 1.0); }
    }
  }

  // Queue a peel-off job for the peel kernel; false if the queue is full
  // (the lane then walks the peel-offs itself).
  __device__ bool push_job(const LaunchParams& P, int ctx, int idust2) {
    const DevModel& m = pk.m;
    if (!P.jobs || m.nslot > kJobSlots) return false;
    const unsigned long long j = atomicAdd(P.njobs, 1ull);
    if ((int64_t)j >= P.job_cap) return false;
    PeelJob J;
    J.x = pk.xp; J.y = pk.yp; J.z = pk.zp; J.rs = pk.rsq; J.rt = pk.rtot;
    J.si = pk.sip; J.sq = pk.sqp; J.su = pk.sup; J.sv = pk.svp;
    if (ctx == PC_DIRECT) { J.d0 = pk.cosb; J.d1 = pk.sinb; J.d2 = coslp; J.d3 = sinlp; J.d4 = 0.0; }
    else { J.d0 = pk.cost; J.d1 = pk.sint; J.d2 = pk.cosp; J.d3 = pk.sinp; J.d4 = pk.phi; }
    for (int s = 0; s < kJobSlots; ++s) J.kapd[s] = s < m.nslot ? pk.sp.kapd(s) : 0.0;
    const int ss = (pk.iflag == 1) ? pk.idust2slot(idust2) : 0;
    if (m.mueller) {         // tabulated matrix: the row and wavelength weight instead of g, pl
      int row = 0;
      double f = 0.0;
      if (pk.iflag == 1) pk.mueller_row(pk.nub, ss, row, f);
      J.g = f;
      J.pl = (double)row;
    } else {
      J.g = pk.sp.g(ss);
      J.pl = pk.sp.pl(ss);
    }
    J.r = pk.ir; J.t = pk.it; J.p = pk.ip;
    J.pkt = (int32_t)kfetch;
    J.ev = min(pk.nscat + pk.nabsev, (1 << kAdjEvBits) - 1);
    J.bits = (pk.on_wall ? 1u : 0u) | ((pk.iflag == 1 ? 1u : 0u) << 1) | ((ctx == PC_DIRECT ? 1u : 0u) << 2) |
             ((uint32_t)pk.i_orig << 3) | ((uint32_t)(pk.freq_bin(pk.nub) - 1) << 8);
    P.jobs[j] = J;
    if (P.job_nub) P.job_nub[j] = pk.nub;
    ++c_jobs;
    return true;
  }

  // ---------------------------------------------------------- peel-off
  // Set up the walk of peel-off direction `peelid` from the packet's
  // position (peeloff_3d_2_test.f90:91-122); false if it ends at once.
  __device__ bool peel_setup(int id) {
    const DevModel& m = pk.m;
    ++pk.c_peel;
    ray_from_packet(true);
    const double cospe = __ldg(m.cospe + id - 1), sinpe = __ldg(m.sinpe + id - 1);
    const double coste = __ldg(m.coste + id - 1), sinte = __ldg(m.sinte + id - 1);
    ray.vx = sinte * cospe;
    ray.vy = sinte * sinpe;
    ray.vz = coste;
    if (ray.onw) {
      const bool inner = fabs(ray.rs - __ldg(m.r2arr + ray.r - 1)) < fabs(ray.rs - __ldg(m.r2arr + ray.r));
      const bool outwards = ray.vx * ray.x + ray.vy * ray.y + ray.vz * ray.z > 0.0;
      if (inner && !outwards) {
        if (ray.r == 1) return false;
        ray.r = ray.r - 1;
      }
      if (!inner && outwards) ray.r = ray.r + 1;
    }
    ev = EV_NONE;
    return true;
  }

  // peeloff_3d_2_test.f90:217-345: weight, scattering rotation, binning
  __device__ void peel_bin() {
    const DevModel& m = pk.m;
    const int id = peelid;
    ++pk.c_pbin;
    const double cospe = __ldg(m.cospe + id - 1), sinpe = __ldg(m.sinpe + id - 1);
    const double coste = __ldg(m.coste + id - 1), sinte = __ldg(m.sinte + id - 1);
    const double factor = exp(-ray.tsum);
    double qi = peel_si * factor, qq = pk.sqp * factor, qu = pk.sup * factor, qv = pk.svp * factor;
    if (pk.iflag == 1) {
      double costnew = pk.cost * coste + (pk.sint * sinte * (pk.cosp * cospe + pk.sinp * sinpe));
      costnew = chk(costnew);
      const double sintnew = sqrt(1.0 - costnew * costnew);
      double ri1 = 0.0;
      if (pk.sint > 1.0e-8 && sintnew > 1.0e-8) {
        double cosx = (coste - (pk.cost * costnew)) / (pk.sint * sintnew);
        cosx = chk(cosx);
        const double x = acos(cosx);
        if (0.0 > pk.phi) ri1 = (0.0 - pk.phi > PI) ? x : R2P - x;
        else ri1 = (pk.phi - 0.0 > PI) ? R2P - x : x;
      }
      pk.peel_matrix(qi, qq, qu, qv, coste, sinte, ri1, costnew, pk.cost, pk.sint, pk.idust2slot(peel_idust2));
    }
    const double x1 = ray.x, y1 = ray.y, z1 = ray.z;
    const double yimage = z1 * sinte - y1 * coste * sinpe - x1 * coste * cospe;
    const double ximage = y1 * cospe - x1 * sinpe;
    const double vx = (ximage + m.rmaxi) / m.fractxh, vy = (yimage + m.rmaxi) / m.fractxh;
    const double rho2 = ximage * ximage + yimage * yimage;
    const int inub = pk.freq_bin(pk.nub);
    if (m.output_imcube && vx > -1.0e9 && vx < 1.0e9 && vy > -1.0e9 && vy < 1.0e9) {
      const int ix = (int)vx + 1, iy = (int)vy + 1;
      if (ix <= m.nxhst && iy <= m.nxhst && ix > 0 && iy > 0) {
        const int64_t k = (int64_t)(id - 1) + (int64_t)m.npeel * ((ix - 1) + (int64_t)m.nxhst * ((iy - 1) + (int64_t)m.nxhst * (inub - 1)));
        atomicAdd(pk.T.img + k, qi);
        atomicAdd(pk.T.img + m.nimg + k, qq);
        atomicAdd(pk.T.img + 2 * m.nimg + k, qu);
        atomicAdd(pk.T.img + 3 * m.nimg + k, qv);
      }
    }
    bin_filters(m, pk.T, id, vx, vy, pk.nub, pk.i_orig, qi, qq, qu, qv);
    bin_nested(m, pk.T, id, ximage, yimage, pk.nub, qi, qq, qu, qv);
    const int i_inter = (pk.iflag == 1) ? 2 : ((pk.i_orig == 1) ? 1 : 3);
    const int indx[3] = {1, 1 + pk.i_orig, 5 + i_inter};
    for (int ia = 1; ia <= m.nap; ++ia) {
      if (rho2 < __ldg(m.aperture2 + ia - 1)) {
        for (int k = 0; k < 3; ++k) {
          const int64_t e = (inub - 1) + (int64_t)m.nfreq * ((id - 1) + (int64_t)m.npeel * ((ia - 1) + (int64_t)m.nap * (indx[k] - 1)));
          double* Q = pk.T.psed + e;
          atomicAdd(Q, qi); atomicAdd(Q + m.npsed, qq); atomicAdd(Q + 2 * m.npsed, qu); atomicAdd(Q + 3 * m.npsed, qv);
          atomicAdd(Q + 4 * m.npsed, qi * qi); atomicAdd(Q + 5 * m.npsed, qq * qq);
          atomicAdd(Q + 6 * m.npsed, qu * qu); atomicAdd(Q + 7 * m.npsed, qv * qv);
          atomicAdd(Q + 8 * m.npsed, 1.0);
        }
      }
    }
  }

  // ----------------------------------------------------------- events
  __device__ void events(const LaunchParams& P) {
    const DevModel& m = pk.m;
    for (;;) {
      switch (ev) {
        case EV_NONE:
        case EV_DONE:
          return;
        case EV_FETCH: {
          if (P.fetch_off) { ev = EV_DONE; return; }
          const unsigned long long k = atomicAdd(P.next, 1ull);
          if (P.adj.mode == 2) {          // replay: the packets that have peel-off records (or all)
            if ((int64_t)k >= (P.adj.all ? P.hi - P.lo + 1 : P.adj.nlist)) { ev = EV_DONE; return; }
            kfetch = P.adj.all ? (int64_t)k : (int64_t)P.adj.list[k];
            adj_pos = P.adj.start[kfetch];
            adj_end = P.adj.end[kfetch];
            adjA = 0.0;
            adjB = 0.0;
            for (int64_t r = adj_pos; r < adj_end; ++r) adjA += P.adj.sc[r];
          } else {
            if ((int64_t)k >= P.hi - P.lo + 1) { ev = EV_DONE; return; }
            kfetch = (int64_t)k;
          }
          iphot = P.lo + kfetch;
          pk.rng = rng_block(m, P.g1, P.g2, (P.block0_dev ? *P.block0_dev : P.block0) + iphot - 1);
          pk.on_wall = false;
          pk.nscat = pk.nabsev = pk.ncross = pk.nstar = pk.ndiffev = 0;
          status = 0;
          if (iphot > P.npacc + P.ns) {     // external illumination, newdisktherm_5_fuv.f90:416-460
            pk.initpout();
            pk.on_wall = true;
            pk.i_orig = 5;
            pk.opacset(pk.nub, KAPD_DISK);
            coslp = cos(pk.lp);
            sinlp = sin(pk.lp);
            const double rmax = m.rarr[m.nrg - 1];
            pk.zp = pk.cosb * rmax * 0.999999;
            const double rp = pk.sinb * rmax * 0.999999;
            pk.xp = rp * coslp;
            pk.yp = rp * sinlp;
            pk.rsq = pk.zp * pk.zp + rp * rp;
            pk.rtot = sqrt(pk.rsq);
            pk.ux = pk.sint * pk.cosp;
            pk.uy = pk.sint * pk.sinp;
            pk.uz = pk.cost;
            pk.iflag = 0;
            pk.ir = m.nrg - 1;
            pk.it = locate(m.thetarr, m.ntg, acos(pk.cosb));
            pk.ip = locate(m.phiarr, m.npg, pk.lp);
            ev = EV_PROP_START;        // no peel-off of the direct light (the sky background)
            break;
          }
          if (iphot < P.npacc) {            // disk accretion, newdisktherm_5_fuv.f90:238-287
            const int idust2 = pk.accretion_emission(P);
            if (idust2 < 0) { status = 3; ev = EV_FINISH; break; }
            pk.opacset(pk.nub, KAPD_DISK);
            pk.iflag = 0;
            pk.i_orig = 2;
            if (P.ipeel == 1 && !push_job(P, PC_ACCRETION, idust2)) {
              peel_ctx = PC_ACCRETION; peelid = 0; peel_idust2 = idust2;
              ev = EV_PEEL_NEXT;
            } else {
              ev = EV_PROP_START;
            }
            break;
          }
          // newdisktherm_5_fuv.f90:295-366
          if (iphot < P.npacc + P.npaccstar) {
            if (P.ips == 0) pk.initpspot(1); else pk.initp_ps(1);
            if (pk.ran() < 0.5) pk.nub = 1.2398 / 0.06 + pk.ran() * (1.2398 / 0.015 - 1.2398 / 0.06);
          } else {
            if (P.ips == 0) pk.initpspot(0); else pk.initp_ps(0);
          }
          pk.i_orig = 1;
          pk.opacset(pk.nub, KAPD_DISK);
          coslp = cos(pk.lp);
          sinlp = sin(pk.lp);
          const double rmin = m.rarr[0];
          pk.zp = pk.cosb * rmin;
          const double rp = pk.sinb * rmin;
          pk.xp = rp * coslp;
          pk.yp = rp * sinlp;
          pk.rsq = pk.zp * pk.zp + rp * rp;
          pk.rtot = sqrt(pk.rsq);
          pk.ux = pk.sint * pk.cosp;
          pk.uy = pk.sint * pk.sinp;
          pk.uz = pk.cost;
          pk.iflag = 0;
          pk.ir = 1;
          pk.on_wall = true;
          pk.it = locate(m.thetarr, m.ntg, acos(pk.cosb));
          pk.ip = locate(m.phiarr, m.npg, pk.lp);
          if (P.ipeel == 1 && !m.partial_peeloff && !push_job(P, PC_DIRECT, 0)) {
            peel_ctx = PC_DIRECT;
            peelid = 0;
            peel_idust2 = 0;
            ev = EV_PEEL_NEXT;
          } else {
            ev = EV_PROP_START;
          }
          break;
        }
        case EV_PEEL_NEXT: {
          bool started = false;
          while (!started) {
            ++peelid;
            if (peelid > m.npeel) break;
            if (peel_ctx == PC_DIRECT) {
              if (P.ips == 0) {
                const double coste = __ldg(m.coste + peelid - 1), sinte = __ldg(m.sinte + peelid - 1);
                const double cospe = __ldg(m.cospe + peelid - 1), sinpe = __ldg(m.sinpe + peelid - 1);
                const double cosnorm = pk.cosb * coste + (pk.sinb * sinte * (cospe * coslp + sinpe * sinlp));
                peel_si = (m.limb == 0) ? 4.0 * pk.sip * cosnorm : 12.0 / 5.0 * pk.sip * (cosnorm + cosnorm * cosnorm);
                if (!(cosnorm > 0.0)) continue;
              } else {
                peel_si = pk.sip * 2.0;
              }
            } else {
              peel_si = pk.sip;
            }
            started = peel_setup(peelid);
          }
          if (started) return;
          ev = (peel_ctx == PC_DIRECT || peel_ctx == PC_ACCRETION) ? EV_PROP_START
               : (peel_ctx == PC_SCATTER ? EV_SCATTER_DONE : EV_ABSORB_DONE);
          break;
        }
        case EV_PEEL_BIN:
          peel_bin();
          ev = EV_PEEL_NEXT;
          break;
        case EV_PROP_START:            // newdisktherm_5_fuv.f90:480-489, propagate_5_fuv.f90:34-55
          pk.ifuv = Packet::is_fuv(pk.nub) ? m.ifuv_ori : 0.0;
          xpold = pk.xp; ypold = pk.yp; zpold = pk.zp;
          pk.iflag = 0;
          pk.exitflag = 0;
          iscat = 0;
          iint = 0;
          nev = 0;
          first = 1;
          adjoint_advance(P);
          pk.tau = -log(pk.ran());
          start_walk();
          return;
        case EV_AFTER_WALK: {          // propagate_5_fuv.f90:56-78, 198-216
          if (!first) {
            if (pk.ir != prev_r || pk.it != prev_t || pk.ip != prev_p) iint = 0;
            if (m.iffuv && !Packet::is_fuv(pk.nub)) { status = 2; ev = EV_FINISH; break; }
            if (iint > 10000 || ++nev > kMaxEvents) {
              atomicAdd(pk.T.killed + pk.cidx(pk.ir, pk.it, pk.ip), 1);
              ++s_cnt[MCRT_S_ABFLUX];
              status = 1;
              ev = EV_FINISH;
              break;
            }
          }
          const int64_t ci = pk.cidx(pk.ir, pk.it, pk.ip);
          const CellRec c = m.cells[ci];
          const int k = pk.select_dust(c);
          if (k < 0) { status = 3; ev = EV_FINISH; break; }
          if (P.adj.mode == 2 && adjA != adjB)   // replay: the interaction density at the segment's end
            atomicAdd(P.adj.grad + ci + m.ncell * (cell_id(c.meta, k) - 1), adjA - adjB);
          if (first) { ++s_cnt[MCRT_S_TOT]; first = 0; }
          const int slot = cell_slot(c.meta, k);
          const int idust2 = cell_id(c.meta, k);
          if (pk.ran() <= pk.sp.alb(slot)) {     // scattered
            pk.iflag = 1;
            ++iscat;
            ++iint;
            ++pk.nscat;
            slot_s = slot;
            if (P.ipeel == 1 && !push_job(P, PC_SCATTER, idust2)) {
              peel_ctx = PC_SCATTER; peelid = 0; peel_idust2 = idust2;
              ev = EV_PEEL_NEXT;
            } else {
              ev = EV_SCATTER_DONE;
            }
          } else {                                // absorbed + re-emitted
            ++pk.nabsev;
            if (idust2 >= 5 && idust2 <= 8) atomicAdd(pk.T.dsg + ci, 1); else atomicAdd(pk.T.dbig + ci, 1);
            if (idust2 == 1 || idust2 == 2 || idust2 == 5 || idust2 == 6 || idust2 == 9) pk.i_orig = 2;
            else if (idust2 == 3 || idust2 == 7) pk.i_orig = 3;
            else pk.i_orig = 4;
            if (!cell_diffus(c.flags)) atomicAdd(pk.T.nabs + ci, 1);
            if (!pk.emit_common(P, ci, c, slot)) { status = 3; ev = EV_FINISH; break; }
            pk.iflag = 0;
            pk.opacset(pk.nub, KAPD_PROPAGATE);
            pk.ifuv = Packet::is_fuv(pk.nub) ? m.ifuv_ori : 0.0;
            if (P.ipeel == 1 && !m.partial_peeloff && !push_job(P, PC_ABSORB, idust2)) {
              peel_ctx = PC_ABSORB; peelid = 0; peel_idust2 = idust2;
              ev = EV_PEEL_NEXT;
            } else {
              ev = EV_ABSORB_DONE;
            }
          }
          break;
        }
        case EV_SCATTER_DONE:
          pk.scatter(slot_s);
          ev = EV_NEXT_TAU;
          break;
        case EV_ABSORB_DONE:
          ++iint;
          ev = EV_NEXT_TAU;
          break;
        case EV_NEXT_TAU:              // propagate_5_fuv.f90:177-193
          adjoint_advance(P);
          pk.tau = -log(pk.ran());
          xpold = pk.xp; ypold = pk.yp; zpold = pk.zp;
          pk.ux = pk.sint * pk.cosp;
          pk.uy = pk.sint * pk.sinp;
          pk.uz = pk.cost;
          prev_r = pk.ir; prev_t = pk.it; prev_p = pk.ip;
          start_walk();
          return;
        case EV_STAR:                  // tauint_3d_2_fuv.f90:184-206, walk resumes
          star_reemit();
          ev = EV_NONE;
          return;
        case EV_EXIT:                  // propagate_5_fuv.f90:231-320
          exit_bin();
          status = 0;
          ev = EV_FINISH;
          break;
        case EV_FINISH:
          ++c_pkt;
          c_int += pk.nscat + pk.nabsev;
          c_sca += pk.nscat;
          c_star += pk.nstar;
          if (status == 3) ++c_geo;
          if (status == 1) ++c_kil;
          if (status == 0) ++c_exit;
          if (P.log && kfetch + P.log_off < P.nlog) {
            mcrt_packet_log& L = P.log[kfetch + P.log_off];
            L.iphot = iphot; L.nscat = pk.nscat; L.nabs = pk.nabsev; L.ncross = pk.ncross; L.nstar = pk.nstar;
            L.status = status; L.ir = 0; L.it = 0; L.ip = 0; L.ndraws = pk.rng.ndraws;
            L.iflag = pk.iflag; L.i_orig = pk.i_orig; L.pad = pk.ndiffev;
            L.nub = pk.nub; L.cost = pk.cost; L.phi = pk.phi; L.sip = pk.sip; L.sqp = pk.sqp; L.sup = pk.sup;
            L.svp = pk.svp; L.xp = pk.xp; L.yp = pk.yp; L.zp = pk.zp;
          }
          ev = EV_FETCH;
          break;
        default:
          ev = EV_DONE;
          return;
      }
    }
  }

  __device__ void exit_bin() {
    const DevModel& m = pk.m;
    int itb = (int)((double)m.nmu * (1.0 - pk.cost) / 2.0) + 1;
    itb = min(max(itb, 1), m.nmu);
    if (pk.phi < 0.0) pk.phi = pk.phi + R2P;
    int ipb = (int)((double)m.nph * pk.phi / R2P) + 1;
    ipb = min(max(ipb, 1), m.nph);
    const double ub = __ldg(m.u + itb - 1);
    const double sini = __ldg(m.sini + itb - 1);
    const double x = ypold * pk.cosp - xpold * pk.sinp;
    const double y = zpold * sini - ypold * ub * pk.sinp - xpold * ub * pk.cosp;
    const double rho2 = x * x + y * y;
    const DevTallies& T = pk.T;
    if (rho2 < __ldg(m.aperture2 + m.nap - 1) * 1.0001) {
      ++s_cnt[MCRT_S_FLUX];
      if (pk.iflag == 1) {
        ++s_cnt[MCRT_S_SFLUX];
        s_cnt[MCRT_S_NSCAT] += (unsigned long long)iscat;
      }
    }
    const int inub = pk.freq_bin(pk.nub);
    const int i_inter = (pk.iflag == 1) ? 2 : ((pk.i_orig == 1) ? 1 : 3);
    const int indx[3] = {1, 1 + pk.i_orig, 5 + i_inter};
    for (int ia = 1; ia <= m.nap; ++ia) {
      if (rho2 < __ldg(m.aperture2 + ia - 1) && !(pk.iflag == 0 && pk.i_orig == 5)) {
        for (int kk = 0; kk < 3; ++kk) {
          const int64_t e = (inub - 1) + (int64_t)m.nfreq * ((itb - 1) + (int64_t)m.nmu * ((ipb - 1) + (int64_t)m.nph * ((ia - 1) + (int64_t)m.nap * (indx[kk] - 1))));
          double* S = T.sed + e;
          const int64_t ns = m.nsed;
          atomicAdd(S, pk.sip); atomicAdd(S + ns, pk.sqp); atomicAdd(S + 2 * ns, pk.sup); atomicAdd(S + 3 * ns, pk.svp);
          atomicAdd(S + 4 * ns, pk.sip * pk.sip); atomicAdd(S + 5 * ns, pk.sqp * pk.sqp);
          atomicAdd(S + 6 * ns, pk.sup * pk.sup); atomicAdd(S + 7 * ns, pk.svp * pk.svp);
          atomicAdd(S + 8 * ns, 1.0); atomicAdd(S + 9 * ns, fabs(pk.cost));
        }
      }
    }
    if (pk.iflag == 1) ++s_cnt[MCRT_S_SCOUNT];
  }
};

// The lanes' integer-valued scalar tallies into the FP64 scalars, one atomic
// per warp and scalar (integers below 2^53: the sums are exact in any order).
__device__ __forceinline__ void flush_scalars(const LaunchParams& P, const Lane& L) {
  for (int i = 0; i < MCRT_NSCALARS; ++i) {
    const unsigned long long x = warp_sum(L.s_cnt[i]);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(P.t.scal + i, (double)x);
  }
}

// Warp-scheduled persistent kernel.  All 32 lanes of a warp stay in the loop
// until every lane is out of packets, so the warp votes are well defined.
#ifndef MCRT_SCHED_MIN_BLOCKS
#define MCRT_SCHED_MIN_BLOCKS 2
#endif
// The warp-scheduled loop of one Lane over the packets of P (all 32 lanes
// of the warp stay in the loop until every lane is out of packets, so the
// warp votes are well defined), then its counters into P's tallies.
__device__ __forceinline__ void warp_loop(Lane& L, const LaunchParams& P) {
  const unsigned FULL = 0xffffffffu;
  const int batch = P.event_batch > 0 ? P.event_batch : 12;
  for (;;) {
    const bool stepping = (L.ev == EV_NONE);
    const bool pending = (L.ev != EV_NONE && L.ev != EV_DONE);
    const unsigned s = __ballot_sync(FULL, stepping);
    const unsigned e = __ballot_sync(FULL, pending);
    if (s == 0u && e == 0u) break;
    if (s == 0u || __popc(e) >= batch) {
      if (pending) L.events(P);
    } else if (stepping) {
      L.step(P);
    }
  }
  unsigned long long v[14] = {L.c_pkt, L.pk.c_cross, L.c_int, L.c_sca, L.pk.c_peel, L.pk.c_pcross, L.pk.c_pbin,
                              L.c_geo, L.pk.c_reset, L.c_kil, L.c_exit, L.c_star, 0ull, L.c_jobs};
  for (int i = 0; i < 14; ++i) {
    unsigned long long x = warp_sum(v[i]);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(P.t.cnt + i, x);
  }
  flush_scalars(P, L);
}

// Warp-scheduled persistent kernel.
__global__ void __launch_bounds__(kBlock, MCRT_SCHED_MIN_BLOCKS) transport_sched(LaunchParams P) {
  __shared__ double spec[5 * kMaxSlot * kBlock];
  Lane L(P.m, P.t, spec);
  warp_loop(L, P);
}

}  // namespace mcrt
