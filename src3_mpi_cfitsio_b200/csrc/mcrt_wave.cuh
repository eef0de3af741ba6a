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
// The walk kernel reads the ray part only: every way a packet walk ends
// (interaction point, exit, stellar surface, geometry failure) first copies
// the ray into the packet position (packet_from_ray), and a peel-off walk
// never changes it, so the packet position is written back after packet
// walks and never read by the walk kernel.
__device__ __forceinline__ void wave_load_ray(Lane& L, const WaveRec& R, int nslot) {
  Ray& y = L.ray;
  y.x = R.x; y.y = R.y; y.z = R.z; y.rs = R.rs; y.rt = R.rt;
  y.vx = R.vx; y.vy = R.vy; y.vz = R.vz; y.tsum = R.tsum;
  y.r = R.r; y.t = R.t; y.p = R.p;
  y.onw = (R.rbits & 1) != 0;
  y.peel = (R.rbits & 2) != 0;
#ifdef MCRT_MIXED
  y.qready = false;                 // every loaded walk sets up its own closest-approach form
#endif
  Packet& k = L.pk;
  k.tau = R.tau; k.ifuv = R.ifuv;
  L.ray_steps = R.ray_steps;
  k.rng.s1 = R.s1; k.rng.s2 = R.s2; k.rng.ndraws = R.ndraws;
  L.ev = R.ev; L.status = R.status;
  k.ncross = R.ncross; k.exitflag = R.exitflag;
  for (int s = 0; s < nslot; ++s) {
    k.sp.kapd(s) = R.spec[s];
    k.sp.alb(s) = R.spec[kMaxSlot + s];
  }
}

__device__ __forceinline__ void wave_load_pos(Lane& L, const WaveRec& R) {
  Packet& k = L.pk;
  k.on_wall = R.on_wall != 0;
  k.ir = R.ir; k.it = R.it; k.ip = R.ip;
  k.xp = R.xp; k.yp = R.yp; k.zp = R.zp; k.rsq = R.rsq; k.rtot = R.rtot;
}

__device__ __forceinline__ void wave_save_ray(const Lane& L, WaveRec& R) {
  const Ray& y = L.ray;
  R.x = y.x; R.y = y.y; R.z = y.z; R.rs = y.rs; R.rt = y.rt;
  R.vx = y.vx; R.vy = y.vy; R.vz = y.vz; R.tsum = y.tsum;
  R.r = y.r; R.t = y.t; R.p = y.p;
  R.rbits = (y.onw ? 1 : 0) | (y.peel ? 2 : 0);
  const Packet& k = L.pk;
  R.tau = k.tau; R.ifuv = k.ifuv;
  R.ray_steps = L.ray_steps;
  R.s1 = k.rng.s1; R.s2 = k.rng.s2; R.ndraws = k.rng.ndraws;
  R.ev = L.ev; R.status = L.status;
  R.ncross = k.ncross; R.exitflag = k.exitflag;
}

__device__ __forceinline__ void wave_save_pos(const Lane& L, WaveRec& R) {
  const Packet& k = L.pk;
  R.on_wall = k.on_wall ? 1 : 0;
  R.ir = k.ir; R.it = k.it; R.ip = k.ip;
  R.xp = k.xp; R.yp = k.yp; R.zp = k.zp; R.rsq = k.rsq; R.rtot = k.rtot;
}

__device__ __forceinline__ void wave_load_walk(Lane& L, const WaveRec& R, int nslot) {
  wave_load_ray(L, R, nslot);
  wave_load_pos(L, R);
}

__device__ __forceinline__ void wave_save_walk(const Lane& L, WaveRec& R) {
  wave_save_ray(L, R);
  wave_save_pos(L, R);
}

__device__ __forceinline__ void wave_load_event(Lane& L, const WaveRec& R, int nslot) {
  Packet& k = L.pk;
  k.ux = R.ux; k.uy = R.uy; k.uz = R.uz;
  k.cost = R.cost; k.sint = R.sint; k.cosp = R.cosp; k.sinp = R.sinp; k.phi = R.phi;
  k.sip = R.sip; k.sqp = R.sqp; k.sup = R.sup; k.svp = R.svp; k.nub = R.nub;
  k.cosb = R.cosb; k.sinb = R.sinb; k.lp = R.lp;
  L.xpold = R.xpold; L.ypold = R.ypold; L.zpold = R.zpold;
  L.peel_si = R.peel_si; L.coslp = R.coslp; L.sinlp = R.sinlp;
  L.nev = R.nev; L.iphot = R.iphot; L.kfetch = R.kfetch;
  k.iflag = R.iflag; k.i_orig = R.i_orig; k.nscat = R.nscat; k.nabsev = R.nabsev;
  k.nstar = R.nstar; k.ndiffev = R.ndiffev;
  L.iscat = R.iscat; L.iint = R.iint; L.first = R.first; L.slot_s = R.slot_s;
  L.prev_r = R.prev_r; L.prev_t = R.prev_t; L.prev_p = R.prev_p;
  L.peel_ctx = R.peel_ctx; L.peelid = R.peelid; L.peel_idust2 = R.peel_idust2;
  for (int s = 0; s < nslot; ++s) {
    k.sp.g(s) = R.spec[2 * kMaxSlot + s];
    k.sp.pl(s) = R.spec[3 * kMaxSlot + s];
  }
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
  y.r = R.r; y.t = R.t; y.p = R.p;
  y.onw = (R.rbits & 1) != 0;
  y.peel = (R.rbits & 2) != 0;
  y.tsum = R.tsum;
  y.qready = true;
  k.tau = R.tau; k.ifuv = R.ifuv;
  L.ray_steps = R.ray_steps;
  L.ev = R.ev; L.status = R.status;
  k.ncross = R.ncross; k.exitflag = R.exitflag;
  for (int s = 0; s < nslot; ++s) {
    const double kd = R.spec[s];
    k.kf(s) = (float)kd;
    k.kaf(s) = (float)__dmul_rn(kd, __dsub_rn(1.0, R.spec[kMaxSlot + s]));
  }
  k.qbegin(y.g, R.x, R.y, R.z, R.vx, R.vy, R.vz, y.r, y.t, y.p);
}

__device__ __forceinline__ void wave_save_qwalk(const Lane& L, WaveRec& R) {
  const Ray& y = L.ray;
  const Packet& k = L.pk;
  R.tsum = y.tsum;
  R.r = y.r; R.t = y.t; R.p = y.p;
  R.rbits = (y.onw ? 1 : 0) | (y.peel ? 2 : 0);
  R.ray_steps = L.ray_steps;
  R.ev = L.ev; R.status = L.status;
  R.ncross = k.ncross; R.exitflag = k.exitflag;
  if (!y.peel) {
    double x, yy, z, rs, rt;
    Packet::qpos(R.x, R.y, R.z, R.vx, R.vy, R.vz, y.g.q, y.g.q0, x, yy, z, rs, rt);
    R.xp = x; R.yp = yy; R.zp = z; R.rsq = rs; R.rtot = rt;
    R.on_wall = y.onw ? 1 : 0;
    R.ir = y.r; R.it = y.t; R.ip = y.p;
  }
}
#endif

// The event kernel loads by event: the ray geometry only for a peel-off bin
// (every other event starts a new ray), the peel-off state only in peeled
// iterations (it is set and used within one visit otherwise), and the
// species columns not for a packet that exits or ends (the next packet's
// emission sets them).  Its save writes every group a later walk or event
// reads.
__device__ __forceinline__ void wave_load_state(Lane& L, const WaveRec& R) {
  Packet& k = L.pk;
  k.tau = R.tau; k.ifuv = R.ifuv;
  L.ray_steps = R.ray_steps;
  k.rng.s1 = R.s1; k.rng.s2 = R.s2; k.rng.ndraws = R.ndraws;
  L.ev = R.ev; L.status = R.status;
  k.ncross = R.ncross; k.exitflag = R.exitflag;
}

__device__ __forceinline__ void wave_load_raygeom(Lane& L, const WaveRec& R) {
  Ray& y = L.ray;
  y.x = R.x; y.y = R.y; y.z = R.z; y.rs = R.rs; y.rt = R.rt;
  y.vx = R.vx; y.vy = R.vy; y.vz = R.vz; y.tsum = R.tsum;
  y.r = R.r; y.t = R.t; y.p = R.p;
  y.onw = (R.rbits & 1) != 0;
  y.peel = (R.rbits & 2) != 0;
#ifdef MCRT_MIXED
  y.qready = false;
#endif
}

__device__ __forceinline__ void wave_load_core(Lane& L, const WaveRec& R) {
  Packet& k = L.pk;
  k.ux = R.ux; k.uy = R.uy; k.uz = R.uz;
  k.cost = R.cost; k.sint = R.sint; k.cosp = R.cosp; k.sinp = R.sinp; k.phi = R.phi;
  k.sip = R.sip; k.sqp = R.sqp; k.sup = R.sup; k.svp = R.svp; k.nub = R.nub;
  L.xpold = R.xpold; L.ypold = R.ypold; L.zpold = R.zpold;
  L.nev = R.nev; L.iphot = R.iphot; L.kfetch = R.kfetch;
  k.iflag = R.iflag; k.i_orig = R.i_orig; k.nscat = R.nscat; k.nabsev = R.nabsev;
  k.nstar = R.nstar; k.ndiffev = R.ndiffev;
  L.iscat = R.iscat; L.iint = R.iint; L.first = R.first; L.slot_s = R.slot_s;
  L.prev_r = R.prev_r; L.prev_t = R.prev_t; L.prev_p = R.prev_p;
}

__device__ __forceinline__ void wave_load_peelstate(Lane& L, const WaveRec& R) {
  Packet& k = L.pk;
  k.cosb = R.cosb; k.sinb = R.sinb; k.lp = R.lp;
  L.peel_si = R.peel_si; L.coslp = R.coslp; L.sinlp = R.sinlp;
  L.peel_ctx = R.peel_ctx; L.peelid = R.peelid; L.peel_idust2 = R.peel_idust2;
}

__device__ __forceinline__ void wave_load_spec(Lane& L, const WaveRec& R, int nslot) {
  Packet& k = L.pk;
  for (int s = 0; s < nslot; ++s) {
    k.sp.kapd(s) = R.spec[s];
    k.sp.alb(s) = R.spec[kMaxSlot + s];
    k.sp.g(s) = R.spec[2 * kMaxSlot + s];
    k.sp.pl(s) = R.spec[3 * kMaxSlot + s];
  }
}

__device__ __forceinline__ void wave_save_core(const Lane& L, WaveRec& R, int nslot) {
  const Packet& k = L.pk;
  R.ux = k.ux; R.uy = k.uy; R.uz = k.uz;
  R.cost = k.cost; R.sint = k.sint; R.cosp = k.cosp; R.sinp = k.sinp; R.phi = k.phi;
  R.sip = k.sip; R.sqp = k.sqp; R.sup = k.sup; R.svp = k.svp; R.nub = k.nub;
  R.xpold = L.xpold; R.ypold = L.ypold; R.zpold = L.zpold;
  R.nev = L.nev; R.iphot = L.iphot; R.kfetch = L.kfetch;
  R.iflag = k.iflag; R.i_orig = k.i_orig; R.nscat = k.nscat; R.nabsev = k.nabsev;
  R.nstar = k.nstar; R.ndiffev = k.ndiffev;
  R.iscat = L.iscat; R.iint = L.iint; R.first = L.first; R.slot_s = L.slot_s;
  R.prev_r = L.prev_r; R.prev_t = L.prev_t; R.prev_p = L.prev_p;
  for (int s = 0; s < nslot; ++s) {
    R.spec[s] = k.sp.kapd(s);
    R.spec[kMaxSlot + s] = k.sp.alb(s);
    R.spec[2 * kMaxSlot + s] = k.sp.g(s);
    R.spec[3 * kMaxSlot + s] = k.sp.pl(s);
  }
}

__device__ __forceinline__ void wave_save_peelstate(const Lane& L, WaveRec& R) {
  const Packet& k = L.pk;
  R.cosb = k.cosb; R.sinb = k.sinb; R.lp = k.lp;
  R.peel_si = L.peel_si; R.coslp = L.coslp; R.sinlp = L.sinlp;
  R.peel_ctx = L.peel_ctx; R.peelid = L.peelid; R.peel_idust2 = L.peel_idust2;
}

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
      L.events(P);
      if (L.ev == EV_NONE) {
        wave_save_walk(L, R);
        wave_save_core(L, R, nslot);
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
