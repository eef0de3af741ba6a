// mcrt_wave.cuh -- wavefront photon-packet transport for sm_100a.
//
// The packet loop of the reference (newdisktherm_5_fuv.f90:220-491 with
// propagate_5_fuv.f90 and tauint_3d_2_fuv.f90) split into two kernels that
// alternate over a pool of in-flight packets kept in HBM (WaveRec):
//
//  * wave_event runs every pending event of a packet -- emission of a new
//    packet, interaction (scattering / absorption + reemission, diffusion),
//    stellar-surface reemission, exit binning, peel-off setup and binning --
//    up to the point where the packet needs its next walk, and queues it for
//    the walk kernel;
//  * wave_walk steps queued walks cell by cell until each reaches its next
//    event and queues it for the event kernel.  Its code is only the cell
//    walk (testgrid, face distances, cell opacity, absorption tally), so it
//    stays resident in the instruction cache, uses far fewer registers than
//    the event code and runs many more warps per SM.  A lane whose walk ends
//    writes the packet back and takes the next queued walk, so lanes stay
//    busy however the walk lengths vary.
//
// Each packet's own steps run in the reference's order on its own random
// substream, exactly as in the other schedules; only the interleaving of
// different packets (and so the order of the FP64 tally atomics) differs.
#pragma once
#include "mcrt_sched.cuh"

namespace mcrt {

// ------------------------------------------------------------ record I/O
// Every access is a 16-byte vector load or store of one group of WaveRec.
__device__ __forceinline__ double2 rd2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ void wr2(double* p, double a, double b) { *reinterpret_cast<double2*>(p) = make_double2(a, b); }
__device__ __forceinline__ int4 rd4(const int32_t* p) { return *reinterpret_cast<const int4*>(p); }
__device__ __forceinline__ void wr4(int32_t* p, int a, int b, int c, int d) {
  *reinterpret_cast<int4*>(p) = make_int4(a, b, c, d);
}

// The ray cell, the walk state and the random stream.
__device__ __forceinline__ void wave_load_state(Lane& L, const WaveRec& R) {
  Packet& k = L.pk;
  const double2 tt = rd2(&R.tsum);
  L.ray.tsum = tt.x;
  k.tau = tt.y;
  const double2 fs = rd2(&R.ifuv);
  k.ifuv = fs.x;
  L.ray_steps = __double_as_longlong(fs.y);
  const int4 e = rd4(&R.ev);
  L.ev = e.x; L.status = e.y; k.ncross = e.z; k.exitflag = e.w;
  const int4 g = rd4(&R.s1);
  k.rng.s1 = g.x; k.rng.s2 = g.y; k.rng.ndraws = g.z;
}

__device__ __forceinline__ void wave_load_raygeom(Lane& L, const WaveRec& R) {
  Ray& y = L.ray;
  double2 a = rd2(&R.x), b = rd2(&R.z), c = rd2(&R.rt), d = rd2(&R.vy);
  y.x = a.x; y.y = a.y; y.z = b.x; y.rs = b.y; y.rt = c.x; y.vx = c.y; y.vy = d.x; y.vz = d.y;
  const int4 q = rd4(&R.r);
  y.r = q.x; y.t = q.y; y.p = q.z;
  y.onw = (q.w & 1) != 0;
  y.peel = (q.w & 2) != 0;
#ifdef MCRT_MIXED
  y.qready = false;
#endif
}

__device__ __forceinline__ void wave_load_pos(Lane& L, const WaveRec& R) {
  Packet& k = L.pk;
  const int4 c = rd4(&R.ir);
  k.ir = c.x; k.it = c.y; k.ip = c.z;
  k.on_wall = c.w != 0;
  const double2 a = rd2(&R.xp), b = rd2(&R.zp), d = rd2(&R.rtot);
  k.xp = a.x; k.yp = a.y; k.zp = b.x; k.rsq = b.y; k.rtot = d.x;
}

__device__ __forceinline__ void wave_save_pos(const Lane& L, WaveRec& R) {
  const Packet& k = L.pk;
  wr4(&R.ir, k.ir, k.it, k.ip, k.on_wall ? 1 : 0);
  wr2(&R.xp, k.xp, k.yp);
  wr2(&R.zp, k.zp, k.rsq);
  wr2(&R.rtot, k.rtot, 0.0);
}

// The walk kernel of the FP64 build reads the ray part only: every way a
// packet walk ends (interaction point, exit, stellar surface, geometry
// failure) first copies the ray into the packet position (packet_from_ray),
// and a peel-off walk never changes it, so the packet position is written
// back after packet walks and never read by the walk kernel.
__device__ __forceinline__ void wave_load_ray(Lane& L, const WaveRec& R, int nslot) {
  wave_load_raygeom(L, R);
  wave_load_state(L, R);
  Packet& k = L.pk;
  for (int s = 0; s < nslot; ++s) {
    const double2 a = rd2(&R.spec[4 * s]);
    k.sp.kapd(s) = a.x;
    k.sp.alb(s) = a.y;
  }
}

__device__ __forceinline__ void wave_save_ray(const Lane& L, WaveRec& R) {
  const Ray& y = L.ray;
  const Packet& k = L.pk;
  wr2(&R.x, y.x, y.y);
  wr2(&R.z, y.z, y.rs);
  wr2(&R.rt, y.rt, y.vx);
  wr2(&R.vy, y.vy, y.vz);
  wr2(&R.tsum, y.tsum, k.tau);
  wr2(&R.ifuv, k.ifuv, __longlong_as_double(L.ray_steps));
  wr4(&R.r, y.r, y.t, y.p, (y.onw ? 1 : 0) | (y.peel ? 2 : 0));
  wr4(&R.ev, L.ev, L.status, k.ncross, k.exitflag);
  wr4(&R.s1, k.rng.s1, k.rng.s2, k.rng.ndraws, 0);
}

__device__ __forceinline__ void wave_load_walk(Lane& L, const WaveRec& R, int nslot) {
  wave_load_ray(L, R, nslot);
  wave_load_pos(L, R);
}

__device__ __forceinline__ void wave_save_walk(const Lane& L, WaveRec& R) {
  wave_save_ray(L, R);
  wave_save_pos(L, R);
}

// Direction, Stokes vector, frequency, the event bookkeeping.
__device__ __forceinline__ void wave_load_core(Lane& L, const WaveRec& R) {
  Packet& k = L.pk;
  double2 a = rd2(&R.ux), b = rd2(&R.uz), c = rd2(&R.sint), d = rd2(&R.sinp);
  k.ux = a.x; k.uy = a.y; k.uz = b.x; k.cost = b.y; k.sint = c.x; k.cosp = c.y; k.sinp = d.x; k.phi = d.y;
  a = rd2(&R.sip); b = rd2(&R.sup); c = rd2(&R.nub); d = rd2(&R.ypold);
  k.sip = a.x; k.sqp = a.y; k.sup = b.x; k.svp = b.y; k.nub = c.x; L.xpold = c.y; L.ypold = d.x; L.zpold = d.y;
  const longlong2 n0 = *reinterpret_cast<const longlong2*>(&R.nev);
  const longlong2 n1 = *reinterpret_cast<const longlong2*>(&R.kfetch);
  L.nev = n0.x; L.iphot = n0.y; L.kfetch = n1.x;
  int4 q = rd4(&R.iflag);
  k.iflag = q.x; k.i_orig = q.y; k.nscat = q.z; k.nabsev = q.w;
  q = rd4(&R.nstar);
  k.nstar = q.x; k.ndiffev = q.y; L.iscat = q.z; L.iint = q.w;
  q = rd4(&R.first);
  L.first = q.x; L.slot_s = q.y; L.prev_r = q.z; L.prev_t = q.w;
  q = rd4(&R.prev_p);
  L.prev_p = q.x; L.peel_ctx = q.y; L.peelid = q.z; L.peel_idust2 = q.w;
}

__device__ __forceinline__ void wave_load_peelstate(Lane& L, const WaveRec& R) {
  Packet& k = L.pk;
  const double2 a = rd2(&R.cosb), b = rd2(&R.lp), c = rd2(&R.coslp);
  k.cosb = a.x; k.sinb = a.y; k.lp = b.x; L.peel_si = b.y; L.coslp = c.x; L.sinlp = c.y;
}

__device__ __forceinline__ void wave_load_spec(Lane& L, const WaveRec& R, int nslot) {
  Packet& k = L.pk;
  for (int s = 0; s < nslot; ++s) {
    const double2 a = rd2(&R.spec[4 * s]), b = rd2(&R.spec[4 * s + 2]);
    k.sp.kapd(s) = a.x;
    k.sp.alb(s) = a.y;
    k.sp.g(s) = b.x;
    k.sp.pl(s) = b.y;
  }
}

// The event part as the tail kernel resumes it (the walk part comes with
// wave_load_walk): core, peel-off state, and the g and pl columns.
__device__ __forceinline__ void wave_load_event(Lane& L, const WaveRec& R, int nslot) {
  wave_load_core(L, R);
  wave_load_peelstate(L, R);
  Packet& k = L.pk;
  for (int s = 0; s < nslot; ++s) {
    const double2 b = rd2(&R.spec[4 * s + 2]);
    k.sp.g(s) = b.x;
    k.sp.pl(s) = b.y;
  }
}

__device__ __forceinline__ void wave_save_core(const Lane& L, WaveRec& R, int nslot) {
  const Packet& k = L.pk;
  wr2(&R.ux, k.ux, k.uy);
  wr2(&R.uz, k.uz, k.cost);
  wr2(&R.sint, k.sint, k.cosp);
  wr2(&R.sinp, k.sinp, k.phi);
  wr2(&R.sip, k.sip, k.sqp);
  wr2(&R.sup, k.sup, k.svp);
  wr2(&R.nub, k.nub, L.xpold);
  wr2(&R.ypold, L.ypold, L.zpold);
  *reinterpret_cast<longlong2*>(&R.nev) = make_longlong2(L.nev, L.iphot);
  *reinterpret_cast<longlong2*>(&R.kfetch) = make_longlong2(L.kfetch, 0);
  wr4(&R.iflag, k.iflag, k.i_orig, k.nscat, k.nabsev);
  wr4(&R.nstar, k.nstar, k.ndiffev, L.iscat, L.iint);
  wr4(&R.first, L.first, L.slot_s, L.prev_r, L.prev_t);
  wr4(&R.prev_p, L.prev_p, L.peel_ctx, L.peelid, L.peel_idust2);
  for (int s = 0; s < nslot; ++s) {
    wr2(&R.spec[4 * s], k.sp.kapd(s), k.sp.alb(s));
    wr2(&R.spec[4 * s + 2], k.sp.g(s), k.sp.pl(s));
  }
}

__device__ __forceinline__ void wave_save_peelstate(const Lane& L, WaveRec& R) {
  const Packet& k = L.pk;
  wr2(&R.cosb, k.cosb, k.sinb);
  wr2(&R.lp, k.lp, L.peel_si);
  wr2(&R.coslp, L.coslp, L.sinlp);
}

#ifdef MCRT_MIXED
// The mixed walk kernel's record I/O: the walk is set up in its
// closest-approach form straight from the record (start point, direction,
// FP32 opacity columns), and the save writes only what a walk changes; the
// packet position at the walk's end is start + (q - q0) u with the start
// point and direction read again from the record, which the walk kernel
// never writes.  The random stream is not used by the mixed walk.
__device__ __forceinline__ void wave_load_qwalk(Lane& L, const WaveRec& R, int nslot) {
  Ray& y = L.ray;
  Packet& k = L.pk;
  const int4 q = rd4(&R.r);
  y.r = q.x; y.t = q.y; y.p = q.z;
  y.onw = (q.w & 1) != 0;
  y.peel = (q.w & 2) != 0;
  const double2 tt = rd2(&R.tsum);
  y.tsum = tt.x;
  k.tau = tt.y;
  y.qready = true;
  const double2 fs = rd2(&R.ifuv);
  k.ifuv = fs.x;
  L.ray_steps = __double_as_longlong(fs.y);
  const int4 e = rd4(&R.ev);
  L.ev = e.x; L.status = e.y; k.ncross = e.z; k.exitflag = e.w;
  for (int s = 0; s < nslot; ++s) {
    const double2 a = rd2(&R.spec[4 * s]);
    k.kf(s) = (float)a.x;
    k.kaf(s) = (float)__dmul_rn(a.x, __dsub_rn(1.0, a.y));
  }
  const double2 a = rd2(&R.x), b = rd2(&R.z), c = rd2(&R.rt), d = rd2(&R.vy);
  k.qbegin(y.g, a.x, a.y, b.x, c.y, d.x, d.y, y.r, y.t, y.p);
}

__device__ __forceinline__ void wave_save_qwalk(const Lane& L, WaveRec& R) {
  const Ray& y = L.ray;
  const Packet& k = L.pk;
  wr2(&R.tsum, y.tsum, k.tau);
  wr2(&R.ifuv, k.ifuv, __longlong_as_double(L.ray_steps));
  wr4(&R.r, y.r, y.t, y.p, (y.onw ? 1 : 0) | (y.peel ? 2 : 0));
  wr4(&R.ev, L.ev, L.status, k.ncross, k.exitflag);
  if (!y.peel) {
    const double2 a = rd2(&R.x), b = rd2(&R.z), c = rd2(&R.rt), d = rd2(&R.vy);
    double x, yy, z, rs, rt;
    Packet::qpos(a.x, a.y, b.x, c.y, d.x, d.y, y.g.q, y.g.q0, x, yy, z, rs, rt);
    wr4(&R.ir, y.r, y.t, y.p, y.onw ? 1 : 0);
    wr2(&R.xp, x, yy);
    wr2(&R.zp, z, rs);
    wr2(&R.rtot, rt, 0.0);
  }
}
#endif

// The event kernel loads by event: the ray geometry only for a peel-off bin
// (every other event starts a new ray), the peel-off state only in peeled
// iterations (it is set and used within one visit otherwise), and the
// species columns not for a packet that exits or ends (the next packet's
// emission sets them).  Its save writes every group a later walk or event
// reads.

__device__ __forceinline__ void flush_counters(const LaunchParams& P, const Lane& L) {
  unsigned long long v[14] = {L.c_pkt, L.pk.c_cross, L.c_int, L.c_sca, L.pk.c_peel, L.pk.c_pcross, L.pk.c_pbin,
                              L.c_geo, L.pk.c_reset, L.c_kil, L.c_exit, L.c_star, 0ull, L.c_jobs};
  for (int i = 0; i < 14; ++i) {
    unsigned long long x = warp_sum(v[i]);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(P.t.cnt + i, x);
  }
  flush_scalars(P, L);
}

// Queue position of this lane among the lanes of `mask` that push to one
// counter: one atomic per warp.
__device__ __forceinline__ unsigned long long warp_push(unsigned mask, bool mine, unsigned long long* counter) {
  const int lane = threadIdx.x & 31;
  unsigned long long base = 0;
  if (mask) {
    const int leader = __ffs(mask) - 1;
    if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
  }
  return mine ? base + (unsigned long long)__popc(mask & ((1u << lane) - 1u)) : 0ull;
}

// The lines of a packet record into L2 (the pool is far larger than L2, so
// a record read otherwise waits for HBM).
__device__ __forceinline__ void prefetch_record(const WaveRec* rec) {
  const char* p = reinterpret_cast<const char*>(rec);
#pragma unroll
  for (int o = 0; o < (int)sizeof(WaveRec); o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + o));
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p + sizeof(WaveRec) - 1));
}

// ------------------------------------------------------------ kernels
// Marks the first `slots` pool entries as waiting for a packet and queues
// them for the first event launch.
__global__ void wave_init(WaveArgs W) {
  const int64_t n = W.slots;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    W.recs[i].ev = EV_FETCH;
    W.evq[n - 1 - i] = (int32_t)i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    WaveCtl& c = *W.ctl;
    c.n_front = 0;
    c.n_back = (unsigned long long)n;
    c.walk_fetch = 0;
    c.walk_cross = 0;
    c.n_walk = 0;
    c.ev_fetch = 0;
  }
}

// Events of every queued packet up to its next walk (or to the end of the
// packet range for this slot).  One queued packet per thread at a time; the
// queue order keeps interactions and the other events in separate warps.
// Prefetching the next round's record into L2 (off: measured 6 % slower on
// the 1e8-packet 2-D iteration, the extra queue read and prefetch
// instructions cost more than the HBM latency they hide).
#ifndef MCRT_EVENT_PREFETCH
#define MCRT_EVENT_PREFETCH 0
#endif
#ifndef MCRT_EVENT_MIN_BLOCKS
#define MCRT_EVENT_MIN_BLOCKS 1
#endif
__global__ void __launch_bounds__(kBlock, MCRT_EVENT_MIN_BLOCKS) wave_event(LaunchParams P, WaveArgs W) {
  __shared__ double spec[5 * kMaxSlot * kBlock];
  Lane L(P.m, P.t, spec);
  const int nslot = P.m.nslot;
  const unsigned long long nf = W.ctl->n_front, nb = W.ctl->n_back;
  const unsigned long long n = nf + nb;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long first = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long rounds = (n + stride - 1) / stride;
  for (unsigned long long r = 0; r < rounds; ++r) {      // uniform trip count: warp votes stay defined
    const unsigned long long k = first + r * stride;
#if MCRT_EVENT_PREFETCH
    {   // the record of this thread's next round into L2 while this round runs
      const unsigned long long k2 = k + stride;
      if (k2 < n) prefetch_record(W.recs + (k2 < nf ? W.evq[k2] : W.evq[W.slots - 1 - (int64_t)(k2 - nf)]));
    }
#endif
    bool walk = false;
    int32_t slot = -1;
    if (k < n) {
      slot = k < nf ? W.evq[k] : W.evq[W.slots - 1 - (int64_t)(k - nf)];
      WaveRec& R = W.recs[slot];
      const int ev = R.ev;
      const bool peeled = P.ipeel != 0;
      if (ev != EV_FETCH) {
        wave_load_state(L, R);
        if (ev == EV_PEEL_BIN) wave_load_raygeom(L, R);
        wave_load_pos(L, R);
        wave_load_core(L, R);
        if (peeled) wave_load_peelstate(L, R);
        if (ev != EV_EXIT && ev != EV_FINISH) wave_load_spec(L, R, nslot);
      }
      L.ev = ev;
      L.pk.spec_dirty = false;
      L.events(P);
      if (L.ev == EV_NONE) {
        wave_save_walk(L, R);
        // the species columns change only with the frequency (opacset):
        // a scattering or a peel-off event leaves the record's copy valid
        wave_save_core(L, R, L.pk.spec_dirty ? nslot : 0);
        if (peeled) wave_save_peelstate(L, R);
        walk = true;
      }
    }
    const unsigned mask = __ballot_sync(0xffffffffu, walk);
    const unsigned long long pos = warp_push(mask, walk, &W.ctl->n_walk);
    if (walk) W.walkq[pos] = slot;
  }
  flush_counters(P, L);
}

#ifndef MCRT_WALK_MIN_BLOCKS
#define MCRT_WALK_MIN_BLOCKS 4
#endif

// Cell walk of every queued packet (or inline peel-off ray) to its next
// event.  Lanes take new walks from the queue in warp batches of at least
// `walk_batch` idle lanes.
__global__ void __launch_bounds__(kBlock, MCRT_WALK_MIN_BLOCKS) wave_walk(LaunchParams P, WaveArgs W) {
#ifdef MCRT_MIXED
  __shared__ float specf[2 * kMaxSlot * kBlock];   // the FP32 walk columns (the only species state it reads)
  Lane L(P.m, P.t, nullptr, specf);
#else
  __shared__ double spec[2 * kMaxSlot * kBlock];   // kapd and alb columns only (step<true> reads no others)
  Lane L(P.m, P.t, spec);
#endif
  const int nslot = P.m.nslot;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned long long nw = W.ctl->n_walk;
  const int batch = W.walk_batch > 0 ? min(W.walk_batch, 32) : 8;
  bool have = false, drained = nw == 0;
  int32_t slot = -1;
  for (;;) {
    const unsigned idle = __ballot_sync(FULL, !have);
    if (!drained && idle && (__popc(idle) >= batch || idle == FULL)) {
      const int cnt = __popc(idle);
      const int leader = __ffs(idle) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(&W.ctl->walk_fetch, (unsigned long long)cnt);
      base = __shfl_sync(FULL, base, leader);
      if (base + (unsigned long long)cnt >= nw) drained = true;
      if (!have) {
        const unsigned long long k = base + (unsigned long long)__popc(idle & ((1u << lane) - 1u));
        if (k < nw) {
          slot = W.walkq[k];
#ifdef MCRT_MIXED
          wave_load_qwalk(L, W.recs[slot], nslot);
#else
          wave_load_ray(L, W.recs[slot], nslot);
#endif
          have = true;
        }
      }
    }
    if (__ballot_sync(FULL, have) == 0u) {
      if (drained) break;
      continue;
    }
    bool done = false;
    if (have) {
      L.step<true>(P);
      done = L.ev != EV_NONE;
      if (done) {
        WaveRec& R = W.recs[slot];
#ifdef MCRT_MIXED
        wave_save_qwalk(L, R);
#else
        wave_save_ray(L, R);
        if (!L.ray.peel) wave_save_pos(L, R);
#endif
      }
    }
    // queue the ended walks (about half of the steps end none: a walk
    // averages ~44 crossings)
    if (__any_sync(FULL, done)) {
      const bool front = done && L.ev == EV_AFTER_WALK;
      const bool back = done && !front;
      const unsigned mf = __ballot_sync(FULL, front);
      const unsigned mb = __ballot_sync(FULL, back);
      const unsigned long long pf = warp_push(mf, front, &W.ctl->n_front);
      const unsigned long long pb = warp_push(mb, back, &W.ctl->n_back);
      if (front) W.evq[pf] = slot;
      if (back) W.evq[W.slots - 1 - (int64_t)pb] = slot;
      if (done) have = false;
    }
  }
  {
    const unsigned long long x = warp_sum(L.pk.c_cross);
    if (lane == 0 && x) atomicAdd(&W.ctl->walk_cross, x);
  }
  flush_counters(P, L);
}

// Tail of the wavefront loop: once every packet of the range has started and
// few remain in flight, one launch finishes them with the warp schedule of
// transport_sched (each lane runs its packet's walks and events back to
// back, no per-wave synchronisation), so the long-lived packets of optically
// thick regions cost their own latency instead of one wave per event.  The
// live packets are the event queue of the last walk launch; a lane whose
// packet ends takes the next one.  Requires P.fetch_off = 1.
__global__ void __launch_bounds__(kBlock, MCRT_SCHED_MIN_BLOCKS) wave_tail(LaunchParams P, WaveArgs W) {
  __shared__ double spec[5 * kMaxSlot * kBlock];
  Lane L(P.m, P.t, spec);
  const int nslot = P.m.nslot;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned long long nf = W.ctl->n_front, nb = W.ctl->n_back;
  const unsigned long long n = nf + nb;
  const int batch = P.event_batch > 0 ? P.event_batch : 16;
  L.ev = EV_DONE;
  bool exhausted = n == 0;
  for (;;) {
    if (!exhausted) {
      const unsigned idle = __ballot_sync(FULL, L.ev == EV_DONE);
      if (idle) {
        const int cnt = __popc(idle);
        const int leader = __ffs(idle) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(&W.ctl->ev_fetch, (unsigned long long)cnt);
        base = __shfl_sync(FULL, base, leader);
        if (base + (unsigned long long)cnt >= n) exhausted = true;
        if (L.ev == EV_DONE) {
          const unsigned long long k = base + (unsigned long long)__popc(idle & ((1u << lane) - 1u));
          if (k < n) {
            const int32_t slot = k < nf ? W.evq[k] : W.evq[W.slots - 1 - (int64_t)(k - nf)];
            const WaveRec& R = W.recs[slot];
            wave_load_walk(L, R, nslot);
            wave_load_event(L, R, nslot);
          }
        }
      }
    }
    const bool stepping = (L.ev == EV_NONE);
    const bool pending = (L.ev != EV_NONE && L.ev != EV_DONE);
    const unsigned s = __ballot_sync(FULL, stepping);
    const unsigned e = __ballot_sync(FULL, pending);
    if (s == 0u && e == 0u) {
      if (exhausted) break;
      continue;
    }
    if (s == 0u || __popc(e) >= batch) {
      if (pending) L.events(P);
    } else if (stepping) {
      L.step(P);
    }
  }
  flush_counters(P, L);
}

}  // namespace mcrt
