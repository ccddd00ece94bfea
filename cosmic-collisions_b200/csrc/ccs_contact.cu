// ccs_contact.cu -- the contact step, warp-cooperative.
//
// src/glsl-sim.js:362-512, simFS({gravity: 'mesh'}): contacts from the 27
// hashed cells around each particle, the mesh gather, the P3M add, settle /
// kick, heat and kick/drift.
//
// A warp owns 32 consecutive particles (neighbours in Morton order).  Their
// neighbour searches have different lengths, and walking them lane by lane
// leaves most of each warp idle.  So the warp works in three stages that keep
// its lanes busy:
//   1. cells: the warp walks the 27 offsets in lockstep; each lane applies its
//      nearest-point test, loads its cell's seats, applies the reference's
//      quantised seat cull to each (where the seat sat at the rebuild, to a
//      fifteenth of a cell: beyond reach, the reference never fetches it)
//      and appends the seats that pass to a per-warp queue in shared memory
//      (a cell's seats fill from the front, so the walk over them stops at
//      the first seat that is empty in every lane's cell);
//   2. candidates: 32 or 64 queued seats at a time, one or two per lane: load
//      the neighbour's position; a pair inside the link radius adds to its
//      owner's count (a shared-memory integer atomic), and a touching one goes
//      on its owner's list;
//   3. contacts: each owner, in its own lane, walks its list of touching
//      neighbours -- the spring-dashpot, its heat and the conduction -- with
//      the sums in registers, so no floating-point atomics are needed (a list
//      holds kTCap; the rare contact past that is worked out in stage 2 and
//      added to the owner's shared slots atomically).
// The pair set and the neighbour counts are decided with exact arithmetic and
// integer counts; force, dissipation and heat flow are summed in the order the
// list was filled, to tolerance.
//
// The seat tables are rebuilt every second step (src/nbody.js:554), so the
// step after a rebuild walks the same tables again.  The rebuilding step's
// walk records what the next one needs (SimArgs::walk 1): for each warp, every
// seat the cull keeps in the cells within cell + mu of an owner, each with its
// owner and which of the owner's 27 cells it came from.  They go through the
// stage-2 queue (tagged whether their cell passed the nearest-point test, as
// only those are this step's candidates), and each 64 the queue drains are
// copied to the record with two contiguous stores.  The next step
// (walk 2) replays that record in place of stage 1, 32 entries at a time, with
// the reference's decisions recomputed: the seat's cell must be one of the
// 27 around where the owner is now and pass its nearest-point test, and then
// the pair the link test.  The quantised cull is not repeated: it can only
// drop a seat whose particle is beyond the link radius while every particle
// has moved less than SEAT_SLACK a less the quantisation's half-diagonal
// since the rebuild.  The record holds every pair the walk can find when the
// owner has moved at most mu and every particle at most D, mu + D within that
// same margin (the host sets both, and checks the margin is there).  Owners
// that moved further walk as the reference does; owners that changed cell
// replay and walk the cells their new neighbourhood adds; a warp whose record
// did not fit, and every warp when any particle moved further than D, walks.
#include "ccs_device.cuh"
#include "ccs_grid.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kQCap = 32 * kSeats + 64;      // seat candidates: one stage-1 round plus what is left
constexpr int kTCap = 16;                    // touching neighbours listed per owner
// a queue entry: particle | owner lane << 18, and when the walk records, the owner's cell it came from << 23
// and whether that cell passed the owner's nearest-point test (kNearCell); the record keeps the first three
constexpr uint32_t kNearCell = 1u << 28, kRecEntry = kNearCell - 1u;
inline int blocks_for(long n, int b) { return (int)((n + b - 1) / b); }
}  // namespace

// a load of state that other CTAs of the same launch may have written (COH, the ensemble's persistent round:
// a plain load, ordered after the producer's release by the consumer's fence) or that no CTA of the launch
// writes (the step's own kernels: the read-only path)
template <bool COH, class T>
__device__ __forceinline__ T ldr(const T *p) {
  if constexpr (COH) return *p;
  else return __ldg(p);
}

struct ContactWarp {
  float4 P[32];        // owner position, tag
  float4 V[32];        // owner velocity, temperature
  float4 C0[32];       // lower corner of the owner's cell (exact), mass ratio
  float ci[32];        // owner heat capacity
  float fx[32], fy[32], fz[32], lost[32], flow[32];   // contacts past an owner's list, added here
  int nb[32];          // neighbours inside the link radius, per owner
  int tn[32];          // touching neighbours listed, per owner
  uint32_t tl[kTCap][32];   // the touching neighbours of owner o: tl[k][o]
  uint32_t near[32];   // walk 2: per owner, its record's cells that its walk would take now (near_cells)
  uint32_t q[kQCap];   // particle index | owner << 18
};

// one touching pair's spring-dashpot, dissipation and conduction (src/glsl-sim.js:433-446)
struct Contact {
  f3 push;
  float lost, flow;
};
template <bool COH>
__device__ __forceinline__ Contact contact_of(const ccs_uniforms &u, const SimArgs &a, float4 Po, float4 Vo, float ri,
                                              float ci, uint32_t j, float r) {
  const float4 Pj = ldr<COH>(a.pos + j);
  const float4 Vj = ldr<COH>(a.vel + j);
  const float rj = __ldg(a.mat + j);
  const f3 nrm = (xyz(Pj) - xyz(Po)) * fdiv(1.0f, fmaxf(r, 1e-6f));
  const float ov = u.touch - r;
  const float cij = u.C * fsqrt(fdiv(2.0f * ri * rj, ri + rj));   // the dashpot for this pair's reduced mass
  const float vn = dot(xyz(Vj) - xyz(Vo), nrm);
  const float fs = u.K * ov - cij * vn;
  const float fn = fmaxf(fs, 0.0f);                                // no tension
  const float cj = rj * (is_iron(Pj.w) ? u.cpIron : 1.0f);
  Contact c;
  c.push = nrm * (-fn);
  c.lost = fs >= 0.0f ? cij * vn * vn : u.K * ov * vn;
  c.flow = (Vj.w - Vo.w) * fdiv(2.0f * ci * cj, ci + cj);         // heat crosses the contact
  return c;
}

// a pair inside the link radius: its owner's count; a touching one onto its owner's list (past the list's
// end, rarely, its contact is worked out here and added to the owner's shared slots).  PAIRS: the pair is
// also written to its owner's row of the pair read-out (the warp's first particle is `base`)
template <bool PAIRS, bool COH>
__device__ __forceinline__ void take_near(const ccs_uniforms &u, const SimArgs &a, ContactWarp &w, uint32_t e,
                                          float r2, int base) {
  const int o = (int)(e >> 18);
  const int slot = atomicAdd(&w.nb[o], 1);
  const float r = __fsqrt_rn(r2);
  const bool touch = xsub(u.touch, r) > 0.0f;
  if (PAIRS && slot < a.pairCap)
    a.pairs[(size_t)(base + o) * a.pairCap + slot] = (e & 0x3FFFFu) | (touch ? 0x80000000u : 0u);
  if (touch) {
    const int k = atomicAdd(&w.tn[o], 1);
    if (k < kTCap) {
      w.tl[k][o] = e & 0x3FFFFu;
    } else {
      const Contact c = contact_of<COH>(u, a, w.P[o], w.V[o], w.C0[o].w, w.ci[o], e & 0x3FFFFu, r);
      atomicAdd(&w.fx[o], c.push.x);
      atomicAdd(&w.fy[o], c.push.y);
      atomicAdd(&w.fz[o], c.push.z);
      atomicAdd(&w.lost[o], c.lost);
      atomicAdd(&w.flow[o], c.flow);
    }
  }
}

// stage 2: queued seats, two per lane when there are 64 (two position loads in flight), else one
// (lanes >= n idle); pairs inside the link radius are counted, touching ones listed for their owner.
// MODE 1: the entries are first copied to the warp's record (rec from rbase, rc entries so far), and only
// those tagged as in a cell past the nearest-point test are candidates
template <bool PAIRS, int MODE, bool COH>
__device__ __forceinline__ void drain_candidates(const ccs_uniforms &u, const SimArgs &a, ContactWarp &w, int base,
                                                 int n, int lane, int first, size_t rbase, int &rc) {
  if (lane < n) {
    const bool two = n == 64;
    const uint32_t e0 = w.q[base + lane];
    const uint32_t e1 = two ? w.q[base + 32 + lane] : 0u;
    if (MODE == 1) {
      if (rc + lane < kRecWarp) a.rec[rbase + rc + lane] = e0 & kRecEntry;
      if (two && rc + 32 + lane < kRecWarp) a.rec[rbase + rc + 32 + lane] = e1 & kRecEntry;
    }
    const float4 Pj0 = ldr<COH>(a.pos + (e0 & 0x3FFFFu));
    const float4 Pj1 = two ? ldr<COH>(a.pos + (e1 & 0x3FFFFu)) : Pj0;
    const float4 Po0 = w.P[(e0 >> 18) & 31u];
    const f3 d0 = xsub3(xyz(Pj0), xyz(Po0));
    const float r20 = xdot(d0, d0);
    if ((MODE != 1 || (e0 & kNearCell)) && r20 < u.link2) take_near<PAIRS, COH>(u, a, w, e0 & 0x7FFFFFu, r20, first);
    if (two) {
      const float4 Po1 = w.P[(e1 >> 18) & 31u];
      const f3 d1 = xsub3(xyz(Pj1), xyz(Po1));
      const float r21 = xdot(d1, d1);
      if ((MODE != 1 || (e1 & kNearCell)) && r21 < u.link2) take_near<PAIRS, COH>(u, a, w, e1 & 0x7FFFFFu, r21, first);
    }
  }
  if (MODE == 1) rc += n;
  __syncwarp();   // every lane has read its entries before the queue is written again
}

// the stencil-split P3M's gravity at a particle: each of its 8 nodes' pull carried from the node's centre
// of mass to the particle by the node's tidal tensor and the pull's second gradient (second order), the
// strays' pull back and the other box's as the reference gives them, and the particle's own pair sum
// (ccs_split.cu)
__device__ __forceinline__ f3 gravity_tide(const ccs_uniforms &u, const SimArgs &a, int me, f3 p) {
  f3 grav = mk(0.0f, 0.0f, 0.0f), g;
  const int box = box_of(u, p, g);
  if (box >= 0) {
    const float4 *F = box == 0 ? a.forceA : a.forceB, *T0 = box == 0 ? a.tideA0 : a.tideB0,
                 *T1 = box == 0 ? a.tideA1 : a.tideB1, *M = box == 0 ? a.fineA : a.fineB,
                 *T2 = box == 0 ? a.tideA2 : a.tideB2;
    const float fx = floorf(g.x), fy = floorf(g.y), fz = floorf(g.z);
    const f3 t = mk(g.x - fx, g.y - fy, g.z - fz);
    const int bx = (int)fx, by = (int)fy, bz = (int)fz;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      const float wgt = (ox ? t.x : 1.0f - t.x) * (oy ? t.y : 1.0f - t.y) * (oz ? t.z : 1.0f - t.z);
      const int c = fine_index(min(bx + ox, 63), min(by + oy, 63), min(bz + oz, 63));
      const float4 m = __ldg(M + c);
      if (!(m.w > 0.0f)) continue;   // a node nothing was deposited on (a corner past the mesh's edge)
      const f3 d = p - xyz(m) * fdiv(1.0f, m.w);
      const float4 f = __ldg(F + c), t0 = __ldg(T0 + c), t1 = __ldg(T1 + c);
      const float4 g0 = __ldg(T2 + c), g1 = __ldg(T2 + kFine + 1 + c), g2 = __ldg(T2 + 2 * (kFine + 1) + c);
      const float xx = d.x * d.x, yy = d.y * d.y, zz = d.z * d.z, xy = d.x * d.y, xz = d.x * d.z, yz = d.y * d.z;
      const f3 Td = mk(t0.x * d.x + t0.w * d.y + t1.x * d.z + 0.5f * (g0.x * xx + g1.z * yy + g2.x * zz) +
                           g1.x * xy + g1.y * xz + g0.w * yz,
                       t0.w * d.x + t0.y * d.y + t1.y * d.z + 0.5f * (g1.x * xx + g0.y * yy + g2.y * zz) +
                           g1.z * xy + g0.w * xz + g1.w * yz,
                       t1.x * d.x + t1.y * d.y + t0.z * d.z + 0.5f * (g1.y * xx + g1.w * yy + g0.z * zz) +
                           g0.w * xy + g2.x * xz + g2.y * yz);
      grav = grav + (xyz(f) + Td) * wgt;
    }
    grav = grav - xyz(__ldg(F + kFine)) * u.Gm;   // the strays in neither box pull back
    if (u.boxB > 0.5f) {
      const float4 mA = __ldg(a.monoA), mB = __ldg(a.monoB);
      grav = grav + (box == 0 ? cross_at(u, mB, mA) : cross_at(u, mA, mB));
    }
  } else {
    grav = mass_at(u, p, __ldg(a.monoA));
    if (u.boxB > 0.5f) grav = grav + mass_at(u, p, __ldg(a.monoB));
  }
  return grav + xyz(__ldg(a.ppAll + me));
}

// a particle's gravity (the mesh gather and the pairwise add, or the field), settle/kick, heat and kick/drift
// from its contact sums: the end of the contact step, and all of a split mesh step's tail (TIDE: the
// stencil-split P3M's gravity instead of the reference's gather and loose-list add)
template <bool FIELD, bool TIDE = false>
__device__ __forceinline__ void finish_particle(const ccs_uniforms &u, const SimArgs &a, int me, float4 P, float4 V,
                                                float ri, float ci, f3 push, float lost, float flow, float nb,
                                                unsigned *recMax = nullptr) {
  const f3 p = xyz(P);
  const float body = P.w;
  f3 grav = mk(0.0f, 0.0f, 0.0f), g;
  if (FIELD) {
    grav = ld3(u.gField);   // SIM_GRAV_FIELD, src/glsl-sim.js:490-492: the whole of gravity
  } else if (TIDE) {
    grav = gravity_tide(u, a, me, p);
  } else {
    // SIM_GRAV_MESH, src/glsl-sim.js:469-488
    const int box = box_of(u, p, g);
    if (box >= 0) {
      const float4 *F = box == 0 ? a.forceA : a.forceB;
      const float fx = floorf(g.x), fy = floorf(g.y), fz = floorf(g.z);
      const f3 t = mk(g.x - fx, g.y - fy, g.z - fz);
      const int bx = (int)fx, by = (int)fy, bz = (int)fz;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
        const float wgt = (ox ? t.x : 1.0f - t.x) * (oy ? t.y : 1.0f - t.y) * (oz ? t.z : 1.0f - t.z);
        const float4 f = __ldg(F + fine_index(min(bx + ox, 63), min(by + oy, 63), min(bz + oz, 63)));
        grav = grav + xyz(f) * wgt;
      }
      grav = grav - xyz(__ldg(F + kFine)) * u.Gm;   // the strays in neither box pull back
      if (u.boxB > 0.5f) {
        const float4 mA = __ldg(a.monoA), mB = __ldg(a.monoB);
        grav = grav + (box == 0 ? cross_at(u, mB, mA) : cross_at(u, mA, mB));
      }
    } else {
      grav = mass_at(u, p, __ldg(a.monoA));
      if (u.boxB > 0.5f) grav = grav + mass_at(u, p, __ldg(a.monoB));
    }
    const int seat = a.ppSlot[me];
    if (seat >= 0) {
#pragma unroll
      for (int s = 0; s < 4; ++s) grav = grav + xyz(__ldg(a.ppForce + (size_t)s * a.cap + seat));
    }
  }
  // SIM_POST, src/glsl-sim.js:493-511
  const float dt = u.dt;
  f3 v = xyz(V) + push * (fdiv(u.invM, ri) * dt) + grav * u.gdt;
  const bool tgt = body < 3.5f;
  const f3 vr = cross(tgt ? ld3(u.spin0) : ld3(u.spin1), p - (tgt ? ld3(u.cen0) : ld3(u.cen1)));
  if (u.settle > 0.5f) {   // damp everything but the spin, and let nothing run
    const f3 dv = (v - vr) * u.damp;
    const float sp = fsqrt(dot(dv, dv));
    v = vr + dv * fminf(1.0f, fdiv(u.creep, fmaxf(sp, 1e-9f)));
  }
  if (u.kick > 0.5f) v = (tgt ? ld3(u.bulk0) : ld3(u.bulk1)) + vr;
  const float Q = u.settle > 0.5f ? 0.0f : a.q[me] + (lost + fdiv(flow * u.kappa, u.tK)) * dt;
  // simFS({frozen: true}), src/glsl-sim.js:523-526: the material that does not move
  if (FIELD && u.frozen >= 0.0f && fabsf(xsub(body, u.frozen)) < 0.5f) v = mk(0.0f, 0.0f, 0.0f);
  const f3 pn = p + v * dt;
  if (recMax) {   // the walk recorded: how far any particle moves before the record is replayed
    const f3 dd = pn - p;
    const unsigned live = __activemask();
    const unsigned m = __reduce_max_sync(live, __float_as_uint(dot(dd, dd)));   // >= 0 (NaN above all)
    if ((threadIdx.x & 31) == __ffs(live) - 1) atomicMax(recMax, m);
  }
  a.posO[me] = make_float4(pn.x, pn.y, pn.z, body);
  a.velO[me] = make_float4(v.x, v.y, v.z, fdiv(u.tK * Q, ci));
  a.auxO[me] = make_float4(grav.x, grav.y, grav.z, nb);
  a.qO[me] = Q;
}

// the cells that pass the owner's nearest-point test (src/glsl-sim.js:415-418) from where it is now (its
// cell's corner c0x, c0y, c0z), with the arithmetic of the walk's own test, as bits e_x + 3 e_y + 9 e_z
// over the 27 cells around another cell of the owner's, the one it had when its record was made, d cells
// off this one (each of dx, dy, dz in -1..1): a cell outside the 27 around the present one has no bit
__device__ __forceinline__ uint32_t near_cells(const ccs_uniforms &u, f3 p, float c0x, float c0y, float c0z, int dx,
                                               int dy, int dz) {
  const float cell = u.cell;
  float sx[3], sy[3], sz[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float off = xmul((float)(d - 1), cell);
    const float lx = xadd(c0x, off), ly = xadd(c0y, off), lz = xadd(c0z, off);
    const float qx = xsub(clampf(p.x, lx, xadd(lx, cell)), p.x);
    const float qy = xsub(clampf(p.y, ly, xadd(ly, cell)), p.y);
    const float qz = xsub(clampf(p.z, lz, xadd(lz, cell)), p.z);
    sx[d] = xmul(qx, qx);
    sy[d] = xmul(qy, qy);
    sz[d] = xmul(qz, qz);
  }
  // the record's cell e (0..2 an axis) is the present frame's o = e + d
  float tx[3], ty[3], tz[3];
  bool vx[3], vy[3], vz[3];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const int ox = e + dx, oy = e + dy, oz = e + dz;
    vx[e] = ox >= 0 && ox <= 2;
    vy[e] = oy >= 0 && oy <= 2;
    vz[e] = oz >= 0 && oz <= 2;
    tx[e] = ox <= 0 ? sx[0] : ox == 1 ? sx[1] : sx[2];
    ty[e] = oy <= 0 ? sy[0] : oy == 1 ? sy[1] : sy[2];
    tz[e] = oz <= 0 ? sz[0] : oz == 1 ? sz[1] : sz[2];
  }
  uint32_t m = 0;
#pragma unroll
  for (int ez = 0; ez < 3; ++ez)
#pragma unroll
    for (int ey = 0; ey < 3; ++ey)
#pragma unroll
      for (int ex = 0; ex < 3; ++ex)
        if (vx[ex] && vy[ey] && vz[ez] && !(xadd(xadd(tx[ex], ty[ey]), tz[ez]) > u.link2))
          m |= 1u << (ex + 3 * ey + 9 * ez);
  return m;
}

// one record entry (particle | owner << 18 | the owner's cell it came from << 23): the walk's decisions
// for it -- the cell one of the owner's 27 now, past the nearest-point test (near, the owner's bits), the
// pair inside the link radius
template <bool PAIRS, bool COH>
__device__ __forceinline__ void replay_entry(const ccs_uniforms &u, const SimArgs &a, ContactWarp &w, uint32_t e,
                                             float4 Pj, int first) {
  const int o = (int)((e >> 18) & 31u);
  if (!((w.near[o] >> ((e >> 23) & 31u)) & 1u)) return;
  const f3 d = xsub3(xyz(Pj), xyz(w.P[o]));
  const float r2 = xdot(d, d);
  if (r2 < u.link2) take_near<PAIRS, COH>(u, a, w, e & 0x7FFFFFu, r2, first);
}

// W warps per CTA (8 or 4: the autotuner's choice; 4 CTAs of 8 or 8 of 4 share an SM); FIELD: the crater
// page's constant gravity and frozen material in place of the mesh gather and the pairwise add.
// The uniforms come by value: every field is then an operand from the constant bank, where through a pointer
// each was a load and a register held across the walk (5.7 % of the launch's time at 262k).
// SPLIT: stop at the contact sums (a mesh step whose mesh runs beside the contact walk; k_contact_tail ends it).
// MODE: 0 the walk; 1 the walk and its record for the next step; 2 the next step, which replays the record
// (SimArgs::walk).
// One CTA's 32 W particles from a.first + blk 32 W: the contact step's body, shared by the kernel below
// (blk = blockIdx.x) and the ensemble's persistent round (k_ensemble_round, one of its work items).  ws: the W
// warps' shared-memory slots; spc: 16 floats of shared memory.  COH: the state it reads (positions,
// velocities, seats, the record) may have been written by other CTAs of the same launch.
template <int W, bool FIELD, bool SPLIT, bool PAIRS, int MODE, bool COH>
__device__ __forceinline__ void contact_block(const ccs_uniforms &u, const SimArgs &a, int blk, ContactWarp *ws,
                                              float *spc) {
  constexpr int kThreads = 32 * W;
  constexpr unsigned kAll = 0xFFFFFFFFu;
  // spc: seatPos(q) * uCell, exact
  if (threadIdx.x < 16) spc[threadIdx.x] = xmul(__fdiv_rn((float)threadIdx.x + 0.5f, 15.0f), u.cell);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  ContactWarp &w = ws[wid];
  const int me = a.first + blk * kThreads + threadIdx.x;
  const int first = me - lane;   // the warp's first particle (the pair read-out's rows)
  const bool live = me < u.N;
  const float cell = u.cell;
  float4 P = make_float4(0, 0, 0, 0), V = make_float4(0, 0, 0, 0);
  float ri = 1.0f;
  if (live) {
    P = a.pos[me];
    V = a.vel[me];
    ri = a.mat[me];
  }
  const f3 p = xyz(P);
  const float body = P.w;
  const float ci = ri * (is_iron(body) ? u.cpIron : 1.0f);
  float gx, gy, gz;
  int cx, cy, cz;
  cell_of(u, p, gx, gy, gz, cx, cy, cz);
  const float c0x = xmul((float)cx, cell), c0y = xmul((float)cy, cell), c0z = xmul((float)cz, cell);
  // MODE 2: how this lane's owner finds its pairs -- 0 its record; 1 its record, and a walk of the cells its
  // new cell adds (ecx, ecy, ecz: its cell when the record was made); 2 the walk.  The warp's record: rn
  // entries from rec[first / 32 * kRecWarp] (more than kRecWarp: it did not fit, and the warp walks)
  int how = 2, ecx = cx, ecy = cy, ecz = cz, rn = 0;
  const size_t rbase = (size_t)(first >> 5) * kRecWarp;
  if (MODE == 2) {
    rn = ldr<COH>(a.recN + (first >> 5));
    if (live && rn <= kRecWarp && __uint_as_float(ldr<COH>(a.recMax)) <= a.recAll2) {
      const float4 Pe = ldr<COH>(a.recP + me);
      const float mx = p.x - Pe.x, my = p.y - Pe.y, mz = p.z - Pe.z;
      if (mx * mx + my * my + mz * mz <= a.recMove2) {
        float ex, ey, ez;
        cell_of(u, xyz(Pe), ex, ey, ez, ecx, ecy, ecz);
        how = (ecx == cx && ecy == cy && ecz == cz) ? 0 : 1;
      }
    }
    w.near[lane] = how < 2 ? near_cells(u, p, c0x, c0y, c0z, ecx - cx, ecy - cy, ecz - cz) : 0u;
    if (rn > kRecWarp) rn = 0;
  }
  w.P[lane] = P;
  w.V[lane] = V;
  w.C0[lane] = make_float4(c0x, c0y, c0z, ri);
  w.ci[lane] = ci;
  w.fx[lane] = w.fy[lane] = w.fz[lane] = w.lost[lane] = w.flow[lane] = 0.0f;
  w.nb[lane] = 0;
  w.tn[lane] = 0;
  __syncthreads();   // spc, and every owner slot
  if (MODE == 2) {
    if (a.recStats) {   // a diagnostic: how many owners took each way
      const unsigned b0 = __ballot_sync(kAll, live && how == 0), b1 = __ballot_sync(kAll, live && how == 1),
                     b2 = __ballot_sync(kAll, live && how == 2);
      if (lane == 0) {
        atomicAdd(a.recStats + 0, (unsigned)__popc(b0));
        atomicAdd(a.recStats + 1, (unsigned)__popc(b1));
        atomicAdd(a.recStats + 2, (unsigned)__popc(b2));
      }
    }
    // the replay: the warp's record 128 entries at a time, four a lane (four position loads in flight),
    // the next 128 entries loaded while these are worked; the entries of owners that walk find no bits in near
    constexpr int kPer = 4;
    uint32_t e[kPer];
#pragma unroll
    for (int q = 0; q < kPer; ++q) e[q] = lane + 32 * q < rn ? ldr<COH>(a.rec + rbase + lane + 32 * q) : 0u;
#pragma unroll 1
    for (int b = 0; b < rn; b += 32 * kPer) {
      float4 Pj[kPer];
#pragma unroll
      for (int q = 0; q < kPer; ++q)
        Pj[q] = b + lane + 32 * q < rn ? ldr<COH>(a.pos + (e[q] & 0x3FFFFu)) : make_float4(0, 0, 0, 0);
      uint32_t en[kPer];
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int k = b + 32 * kPer + lane + 32 * q;
        en[q] = k < rn ? ldr<COH>(a.rec + rbase + k) : 0u;
      }
#pragma unroll
      for (int q = 0; q < kPer; ++q)
        if (b + lane + 32 * q < rn) replay_entry<PAIRS, COH>(u, a, w, e[q], Pj[q], first);
#pragma unroll
      for (int q = 0; q < kPer; ++q) e[q] = en[q];
    }
    __syncwarp();
  }
  const int sh = u.GShift;
  const uint32_t gm = (uint32_t)u.GMask;
  const uint4 *seats = reinterpret_cast<const uint4 *>(a.seats);
  int qn = 0;   // queue fill (warp-uniform)
  int rc = 0;   // MODE 1: entries of the warp's record (warp-uniform)
  // stage 1: the 27 neighbour cells in the reference's order, the warp in lockstep (MODE 2: the lanes whose
  // owners walk, over the cells they walk; none, and no walk, in most warps)
  const bool walks = live && how > 0;
  if (MODE != 2 || __any_sync(kAll, walks)) {
#pragma unroll 1
  for (int dz = 0; dz < 3; ++dz) {
    const int z = cz + dz - 1;
    const float lz = xadd(c0z, xmul((float)(dz - 1), cell));
    const float qz = xsub(clampf(p.z, lz, xadd(lz, cell)), p.z), qz2 = xmul(qz, qz);
    const uint32_t wz = (uint32_t)(z >> sh) << (sh - 2);      // the z period skews y by a quarter
#pragma unroll 1
    for (int dy = 0; dy < 3; ++dy) {
      const int y = cy + dy - 1;
      const float ly = xadd(c0y, xmul((float)(dy - 1), cell));
      const float qy = xsub(clampf(p.y, ly, xadd(ly, cell)), p.y), qy2 = xmul(qy, qy);
      const uint32_t zz = ((uint32_t)z + ((uint32_t)(y >> sh) << (sh - 1))) & gm;   // the y period skews z by half
      const uint32_t row = (zz >> u.SXShift) << sh, col = (zz & (uint32_t)u.SXMask) << sh;
#pragma unroll 1
      for (int dx = 0; dx < 3; ++dx) {
        const int x = cx + dx - 1;
        const float lx = xadd(c0x, xmul((float)(dx - 1), cell));
        const float qx = xsub(clampf(p.x, lx, xadd(lx, cell)), p.x);
        const float d2 = xadd(xadd(xmul(qx, qx), qy2), qz2);
        const bool nearCell = !(d2 > u.link2);   // the nearest-point test
        bool walk = live;
        if (MODE == 2)   // a lane that moved to another cell walks only the cells its old one did not have
          walk = walks && (how == 2 || abs(x - ecx) > 1 || abs(y - ecy) > 1 || abs(z - ecz) > 1);
        // MODE 1 loads the cells a little further out too, for the record (their seats are not this step's)
        const bool load = walk && (MODE == 1 ? !(d2 > a.recLink2) : nearCell);
        const uint32_t tag = MODE == 1 ? ((uint32_t)(dx + 3 * dy + 9 * dz) << 23) | (nearCell ? kNearCell : 0u) : 0u;
        uint4 s0 = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty), s1 = s0;
        if (load) {
          const uint32_t yy = ((uint32_t)y + ((uint32_t)(x >> sh) << (sh - 1)) + wz) & gm;   // the x period skews y by half
          const uint32_t h = (row + yy) * (uint32_t)u.AW + col + ((uint32_t)x & gm);
          const uint4 *cp = seats + (size_t)h * 2;
          s0 = ldr<COH>(cp);       // both halves of the cell: one 32-byte sector, one round trip
          s1 = ldr<COH>(cp + 1);
        }
        {
          const uint32_t sv[kSeats] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
#pragma unroll
          for (int k = 0; k < kSeats; ++k) {
            // a cell's seats fill from the front: the walk ends at the first seat empty in every lane's cell
            if (!__any_sync(kAll, !(sv[k] & 0x80000000u))) break;
            bool seat = !(sv[k] & 0x80000000u) && (int)(sv[k] & 0x3FFFFu) != me;
            if (seat) {   // the quantised cull: where the seat sat at the rebuild, against this particle now
              const f3 dq = mk(xsub(xadd(lx, spc[(sv[k] >> 18) & 15u]), p.x),
                               xsub(xadd(ly, spc[(sv[k] >> 22) & 15u]), p.y),
                               xsub(xadd(lz, spc[(sv[k] >> 26) & 15u]), p.z));
              seat = !(xdot(dq, dq) > u.reach2);
            }
            const unsigned bal = __ballot_sync(kAll, seat);
            if (seat) w.q[qn + __popc(bal & ((1u << lane) - 1u))] = (sv[k] & 0x3FFFFu) | ((uint32_t)lane << 18) | tag;
            qn += __popc(bal);
          }
        }
        __syncwarp();
        while (qn >= 64) {
          qn -= 64;
          drain_candidates<PAIRS, MODE, COH>(u, a, w, qn, 64, lane, first, rbase, rc);
        }
      }
    }
  }
  }
  if (qn >= 32) {
    qn -= 32;
    drain_candidates<PAIRS, MODE, COH>(u, a, w, qn, 32, lane, first, rbase, rc);
  }
  if (qn > 0) drain_candidates<PAIRS, MODE, COH>(u, a, w, 0, qn, lane, first, rbase, rc);
  __syncwarp();
  if (MODE == 1) {
    if (lane == 0) a.recN[first >> 5] = min(rc, kRecWarp + 1);
    if (live) a.recP[me] = P;
  }
  if (!live) return;
  // stage 3: each owner's touching neighbours in its own lane, the sums in registers
  f3 push = mk(w.fx[lane], w.fy[lane], w.fz[lane]);
  float lost = w.lost[lane], flow = w.flow[lane];
  const float nb = (float)w.nb[lane];
  const int nt = min(w.tn[lane], kTCap);
#pragma unroll 4
  for (int k = 0; k < nt; ++k) {   // unrolled: the next contacts' loads are in flight with this one's math
    const uint32_t j = w.tl[k][lane];
    const float4 Pj = ldr<COH>(a.pos + j);
    const f3 d = xsub3(xyz(Pj), p);
    const Contact c = contact_of<COH>(u, a, P, V, ri, ci, j, __fsqrt_rn(xdot(d, d)));
    push = push + c.push;
    lost += c.lost;
    flow += c.flow;
  }
  if (SPLIT) {   // a split mesh step: the sums wait in part for the tail, which runs after the mesh
    a.part[me] = make_float4(push.x, push.y, push.z, nb);
    a.part2[me] = make_float2(lost, flow);
    return;
  }
  finish_particle<FIELD>(u, a, me, P, V, ri, ci, push, lost, flow, nb, MODE == 1 ? a.recMax : nullptr);
}

template <int W, bool FIELD, bool SPLIT = false, bool PAIRS = false, int MODE = 0>
__global__ void __launch_bounds__(32 * W, 32 / W) k_contact_step(const ccs_uniforms u, const SimArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ float spc[16];
  contact_block<W, FIELD, SPLIT, PAIRS, MODE, false>(u, a, blockIdx.x, reinterpret_cast<ContactWarp *>(smem_raw),
                                                     spc);
}

// the tail of a split mesh step, one thread a particle: the contact sums the contact walk left in part, then
// the same gravity, settle/kick, heat and kick/drift as the whole step's (and, after a walk that recorded,
// the displacement its record is good for)
template <bool TIDE>
__global__ void __launch_bounds__(256) k_contact_tail(const ccs_uniforms u, const SimArgs a) {
  const int me = a.first + blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= u.N) return;
  const float4 P = a.pos[me], V = a.vel[me];
  const float ri = a.mat[me];
  const float ci = ri * (is_iron(P.w) ? u.cpIron : 1.0f);
  const float4 s = a.part[me];
  const float2 s2 = a.part2[me];
  finish_particle<false, TIDE>(u, a, me, P, V, ri, ci, mk(s.x, s.y, s.z), s2.x, s2.y, s.w,
                               a.walk == 1 ? a.recMax : nullptr);
}

size_t contact_smem_bytes(int warps) { return sizeof(ContactWarp) * warps; }

// ---------------------------------------------------------------------------
// The ensemble's persistent round: every member's kEnsSteps steps (contact grid on even steps, contact step
// on each) in one launch of as many CTAs as the device holds at once.  Each member's work is a chain of
// segments numbered by one ticket counter (EnsMember, EnsState): a CTA takes the next ticket of a member
// whose current segment is ready (the segment before it finished), does that work item, and counts it done
// after a fence.  A ticket only ever waits for tickets taken before it, by CTAs that are running and wait for
// nothing later, so the round finishes whether or not every CTA is resident.  Every wait is bounded by
// %globaltimer (limitNs): when one runs out the CTA raises kStatusEnsemble and the abort flag, and every CTA
// leaves at its next pick.  State the round writes (positions, velocities, seats, the walk's record) is read
// with plain loads after the fence that follows each wait (contact_block<..., COH = true>); the read-only
// path is kept for what only the kernels before the launch wrote (the mesh force, the pairwise pass).
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int seg_of(const EnsMember &I, int t) {
  int s = 0;
  while (s < I.nseg - 1 && t >= I.end[s]) ++s;
  return s;
}
__device__ __forceinline__ int seg_items(const EnsMember &I, int s) { return I.end[s] - (s ? I.end[s - 1] : 0); }
__device__ __forceinline__ bool seg_ready(const EnsMember &I, const EnsState &S, int s) {
  return s == 0 || *(volatile const int *)&S.done[s - 1] >= seg_items(I, s - 1);
}

// thread 0: the next work item (member, segment, item in the segment); member -1 when every member's work has
// been taken or the round aborted.  Members are tried in the priority order L.order (largest first), from the
// first one whose work is not all taken (L.front, a hint every CTA moves on): each CTA works for the earliest
// member with a ready segment, so a few members are under way at a time -- their state stays in L2 -- and the
// gaps at one member's step boundaries go to the next.
__device__ int4 ens_pick(const EnsLaunch &L) {
  const int M = L.members;
  const unsigned long long t0 = gtime();
  for (;;) {
    if (*(volatile int *)L.abort) return make_int4(-1, 0, 0, 0);
    bool left = false;
    for (int k = *(volatile int *)L.front; k < M; ++k) {
      const int m = L.order[k];
      const EnsMember &I = L.info[m];
      EnsState &S = L.state[m];
      int t = *(volatile int *)&S.next;
      if (t >= I.total) {
        if (!left) atomicMax(L.front, k + 1);   // every member before it is taken too
        continue;
      }
      left = true;
      if (!seg_ready(I, S, seg_of(I, t))) continue;   // its next segment waits: work for another member
      t = atomicAdd(&S.next, 1);
      if (t >= I.total) continue;
      const int s = seg_of(I, t);
      if (t == 0) S.t0 = gtime();
      // the ticket may lie past a segment boundary another CTA crossed meanwhile: wait for the segment before
      while (!seg_ready(I, S, s)) {
        if (*(volatile int *)L.abort) return make_int4(-1, 0, 0, 0);
        if (gtime() - t0 > L.limitNs) {
          atomicOr(L.status, kStatusEnsemble);
          atomicExch(L.abort, 1);
          return make_int4(-1, 0, 0, 0);
        }
        __nanosleep(100);
      }
      return make_int4(m, s, t - (s ? I.end[s - 1] : 0), 0);
    }
    if (!left) return make_int4(-1, 0, 0, 0);
    if (gtime() - t0 > L.limitNs) {
      atomicOr(L.status, kStatusEnsemble);
      atomicExch(L.abort, 1);
      return make_int4(-1, 0, 0, 0);
    }
    __nanosleep(200);
  }
}
}  // namespace

// 3 CTAs of 8 warps an SM: the walk's three forms and the grid in one kernel keep 80 registers without
// spilling (at 64 registers it spilled, and ran slower).  Work items are a CTA's: warp-sized items, each warp
// picking its own, took four times the picks and ran slower; CTAs of 4 warps 4 % slower than of 8.
__global__ void __launch_bounds__(32 * kEnsWarps, 24 / kEnsWarps) k_ensemble_round(const EnsLaunch L) {
  constexpr int W = kEnsWarps;
  extern __shared__ __align__(16) unsigned char smem_raw[];   // the contact step's W warp slots
  __shared__ float spc[16];
  __shared__ __align__(16) unsigned char argRaw[sizeof(EnsStepArgs)];   // the item's step, copied in
  __shared__ int4 pick;
  const EnsStepArgs &A = *reinterpret_cast<const EnsStepArgs *>(argRaw);
  int held = -1;   // the (member, step) whose arguments argRaw holds
  for (;;) {
    if (threadIdx.x == 0) {
      pick = ens_pick(L);
      __threadfence();   // with the barrier: what the finished segments wrote is seen by the whole CTA
    }
    __syncthreads();
    const int4 p = pick;
    if (p.x < 0) break;
    const EnsMember &I = L.info[p.x];
    const int step = I.step[p.y];
    if (p.x * L.steps + step != held) {   // items in a row mostly share their step
      held = p.x * L.steps + step;
      const int *src = reinterpret_cast<const int *>(L.args + held);
      int *dst = reinterpret_cast<int *>(argRaw);
      for (int k = threadIdx.x; k < (int)(sizeof(EnsStepArgs) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
      __syncthreads();
    }
    if (I.grid[p.y]) {
#pragma unroll 1
      for (int r = 0; r < kEnsGridItem / (32 * W); ++r)
        grid_particle(A.u, p.z * kEnsGridItem + r * 32 * W + (int)threadIdx.x, A.gpos, A.gseats, A.ghk,
                      A.gseatsOld, A.ghkOld, A.gstatus, A.grecMax);
    } else {
      ContactWarp *ws = reinterpret_cast<ContactWarp *>(smem_raw);
      if (A.a.walk == 1)
        contact_block<W, false, false, false, 1, true>(A.u, A.a, p.z, ws, spc);
      else if (A.a.walk == 2)
        contact_block<W, false, false, false, 2, true>(A.u, A.a, p.z, ws, spc);
      else
        contact_block<W, false, false, false, 0, true>(A.u, A.a, p.z, ws, spc);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();   // this item's writes before its count
      const int d = atomicAdd(&L.state[p.x].done[p.y], 1) + 1;
      if (d == seg_items(I, p.y) && p.y == I.nseg - 1) {   // the member's last item: its round's time
        const unsigned long long t = gtime() - *(volatile unsigned long long *)&L.state[p.x].t0;
        atomicAdd(L.acc + p.x, t);
        atomicAdd(L.acc + L.members + p.x, 1ull);
      }
    }
  }
}

namespace {
size_t ensemble_smem() { return contact_smem_bytes(kEnsWarps); }
}  // namespace

int ensemble_round_ctas() {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_ensemble_round, 32 * kEnsWarps, ensemble_smem()) !=
          cudaSuccess ||
      per <= 0)
    per = 1;
  return per * sm_count();
}

int launch_ensemble_round(const EnsLaunch &L, int ctas, cudaStream_t st) {
  k_ensemble_round<<<ctas, 32 * kEnsWarps, ensemble_smem(), st>>>(L);
  return 1;
}

namespace {
template <int W, bool FIELD, bool SPLIT, bool PAIRS, int MODE>
cudaError_t set_smem() {
  return cudaFuncSetAttribute(k_contact_step<W, FIELD, SPLIT, PAIRS, MODE>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)contact_smem_bytes(W));
}
template <int W, bool FIELD, bool SPLIT, bool PAIRS>
cudaError_t set_modes() {
  cudaError_t e = set_smem<W, FIELD, SPLIT, PAIRS, 0>();
  if (e == cudaSuccess) e = set_smem<W, FIELD, SPLIT, PAIRS, 1>();
  if (e == cudaSuccess) e = set_smem<W, FIELD, SPLIT, PAIRS, 2>();
  return e;
}
// one launch of the contact step over [a.first, a.first + count) in the walk a.walk names
template <int W, bool FIELD, bool SPLIT, bool PAIRS>
void launch_walk(const ccs_uniforms &u, const SimArgs &a, int count, cudaStream_t st) {
  const dim3 grid(blocks_for(count, 32 * W)), block(32 * W);
  const size_t smem = contact_smem_bytes(W);
  if (a.walk == 1)
    k_contact_step<W, FIELD, SPLIT, PAIRS, 1><<<grid, block, smem, st>>>(u, a);
  else if (a.walk == 2)
    k_contact_step<W, FIELD, SPLIT, PAIRS, 2><<<grid, block, smem, st>>>(u, a);
  else
    k_contact_step<W, FIELD, SPLIT, PAIRS, 0><<<grid, block, smem, st>>>(u, a);
}
}  // namespace

cudaError_t init_kernels() {
  cudaError_t e = set_modes<8, false, false, false>();
  if (e == cudaSuccess) e = set_modes<4, false, false, false>();
  if (e == cudaSuccess) e = set_modes<8, true, false, false>();
  if (e == cudaSuccess) e = set_modes<4, true, false, false>();
  if (e == cudaSuccess) e = set_modes<8, false, true, false>();
  if (e == cudaSuccess) e = set_modes<4, false, true, false>();
  if (e == cudaSuccess) e = set_modes<4, false, false, true>();
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_ensemble_round, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ensemble_smem());
  return e;
}

int launch_simulate_range(const ccs_uniforms &u, int N, SimArgs a, cudaStream_t st, int warps, bool field, int first,
                          int count) {
  (void)N;
  a.first = first;
  if (count <= 0) return 0;
  if (warps == 4 && field)
    launch_walk<4, true, false, false>(u, a, count, st);
  else if (warps == 4)
    launch_walk<4, false, false, false>(u, a, count, st);
  else if (field)
    launch_walk<8, true, false, false>(u, a, count, st);
  else
    launch_walk<8, false, false, false>(u, a, count, st);
  return 1;
}

int launch_simulate(const ccs_uniforms &u, int N, const SimArgs &a, cudaStream_t st, int warps, bool field) {
  return launch_simulate_range(u, N, a, st, warps, field, 0, N);
}

int launch_contacts_only(const ccs_uniforms &u, int N, const SimArgs &a, cudaStream_t st, int warps) {
  if (N <= 0) return 0;
  if (warps == 4)
    launch_walk<4, false, true, false>(u, a, N, st);
  else
    launch_walk<8, false, true, false>(u, a, N, st);
  return 1;
}

// the read-out never records (it is not a step); after a step that recorded it replays as the next step will
int launch_contact_pairs(const ccs_uniforms &u, int N, const SimArgs &a, cudaStream_t st) {
  if (N <= 0) return 0;
  SimArgs b = a;
  if (b.walk == 1) b.walk = 0;
  b.recStats = nullptr;
  launch_walk<4, false, false, true>(u, b, N, st);
  return 1;
}

int launch_contact_tail(const ccs_uniforms &u, int N, const SimArgs &a, cudaStream_t st, bool tide) {
  if (N <= 0) return 0;
  if (tide)
    k_contact_tail<true><<<blocks_for(N, 256), 256, 0, st>>>(u, a);
  else
    k_contact_tail<false><<<blocks_for(N, 256), 256, 0, st>>>(u, a);
  return 1;
}

}  // namespace ccs
