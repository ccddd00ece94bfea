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
//      and appends the seats that pass to a per-warp queue in shared memory;
//   2. candidates: 32 queued seats at a time, one per lane: load the
//      neighbour's position and keep the pairs inside the link radius;
//   3. neighbours: 32 at a time: the neighbour count, and for touching pairs
//      the spring-dashpot, its heat and the conduction, added into the
//      owner's slots.
// The pair set and the neighbour counts are decided with exact arithmetic and
// integer counts; force, dissipation and heat flow are summed in whatever
// order the shared-memory atomics land, to tolerance.
#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kQCap = 32 * kSeats + 64;      // seat candidates: one stage-1 round plus what is left
constexpr int kNCap = 64;                    // neighbours: one stage-2 round plus what is left
inline int blocks_for(long n, int b) { return (int)((n + b - 1) / b); }
}  // namespace

struct ContactWarp {
  float4 P[32];        // owner position, tag
  float4 V[32];        // owner velocity, temperature
  float4 C0[32];       // lower corner of the owner's cell (exact), mass ratio
  float ci[32];        // owner heat capacity
  float fx[32], fy[32], fz[32], lost[32], flow[32];   // what the contacts add up, per owner
  int nb[32];
  uint32_t q[kQCap];   // particle index | owner << 18
  uint2 nq[kNCap];     // x: particle index | owner << 18; y: r^2 bits
};

__device__ __forceinline__ void drain_neighbours(const ccs_uniforms &u, const SimArgs &a, ContactWarp &w, int base,
                                                 int n, int lane) {
  if (lane < n) {
    const uint2 e = w.nq[base + lane];
    const uint32_t sv = e.x;
    const int o = (int)(e.x >> 18);
    const float r2 = __uint_as_float(e.y);
    const float4 Po = w.P[o], C0 = w.C0[o];
    {
      atomicAdd(&w.nb[o], 1);
      const float r = __fsqrt_rn(r2);
      if (xsub(u.touch, r) > 0.0f) {
        const uint32_t j = sv & 0x3FFFFu;
        const float4 Pj = __ldg(a.pos + j);
        const float4 Vj = __ldg(a.vel + j);
        const float rj = __ldg(a.mat + j);
        const float4 Vo = w.V[o];
        const float ri = C0.w, ci = w.ci[o];
        const f3 nrm = (xyz(Pj) - xyz(Po)) * fdiv(1.0f, fmaxf(r, 1e-6f));
        const float ov = u.touch - r;
        const float cij = u.C * fsqrt(fdiv(2.0f * ri * rj, ri + rj));   // the dashpot for this pair's reduced mass
        const float vn = dot(xyz(Vj) - xyz(Vo), nrm);
        const float fs = u.K * ov - cij * vn;
        const float fn = fmaxf(fs, 0.0f);                                // no tension
        atomicAdd(&w.fx[o], -nrm.x * fn);
        atomicAdd(&w.fy[o], -nrm.y * fn);
        atomicAdd(&w.fz[o], -nrm.z * fn);
        atomicAdd(&w.lost[o], fs >= 0.0f ? cij * vn * vn : u.K * ov * vn);
        const float cj = rj * (is_iron(Pj.w) ? u.cpIron : 1.0f);
        atomicAdd(&w.flow[o], (Vj.w - Vo.w) * fdiv(2.0f * ci * cj, ci + cj));   // heat crosses the contact
      }
    }
  }
  __syncwarp();
}

// stage 2: queued seats, two per lane when there are 64 (two position loads in flight), else one
// (lanes >= n idle); pairs inside the link radius go on to stage 3
__device__ __forceinline__ void push_near(const ccs_uniforms &u, const SimArgs &a, ContactWarp &w,
                                          bool near, uint32_t e, float r2, int lane, int &nn) {
  const unsigned bal = __ballot_sync(0xFFFFFFFFu, near);
  if (near) w.nq[nn + __popc(bal & ((1u << lane) - 1u))] = make_uint2(e, __float_as_uint(r2));
  nn += __popc(bal);
  __syncwarp();
  if (nn >= 32) {
    nn -= 32;
    drain_neighbours(u, a, w, nn, 32, lane);
  }
}

__device__ __forceinline__ void drain_candidates(const ccs_uniforms &u, const SimArgs &a, ContactWarp &w, int base,
                                                 int n, int lane, int &nn) {
  const bool two = n == 64;
  bool near0 = false, near1 = false;
  uint32_t e0 = 0u, e1 = 0u;
  float r20 = 0.0f, r21 = 0.0f;
  if (lane < n) {
    e0 = w.q[base + lane];
    if (two) e1 = w.q[base + 32 + lane];
    const float4 Pj0 = __ldg(a.pos + (e0 & 0x3FFFFu));
    const float4 Pj1 = two ? __ldg(a.pos + (e1 & 0x3FFFFu)) : Pj0;
    const float4 Po0 = w.P[e0 >> 18];
    const f3 d0 = xsub3(xyz(Pj0), xyz(Po0));
    r20 = xdot(d0, d0);
    near0 = r20 < u.link2;
    if (two) {
      const float4 Po1 = w.P[e1 >> 18];
      const f3 d1 = xsub3(xyz(Pj1), xyz(Po1));
      r21 = xdot(d1, d1);
      near1 = r21 < u.link2;
    }
  }
  __syncwarp();   // every lane has read its entries before the queue is written again
  push_near(u, a, w, near0, e0, r20, lane, nn);
  if (two) push_near(u, a, w, near1, e1, r21, lane, nn);
}

// W warps per CTA (8 or 4: the autotuner's choice; 4 CTAs of 8 or 8 of 4 share an SM); FIELD: the crater
// page's constant gravity and frozen material in place of the mesh gather and the pairwise add
template <int W, bool FIELD>
__global__ void __launch_bounds__(32 * W, 32 / W) k_contact_step(const ccs_uniforms *__restrict__ U,
                                                                 const SimArgs a) {
  constexpr int kThreads = 32 * W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ float spc[16];   // seatPos(q) * uCell, exact
  const ccs_uniforms &u = *U;
  if (threadIdx.x < 16) spc[threadIdx.x] = xmul(__fdiv_rn((float)threadIdx.x + 0.5f, 15.0f), u.cell);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  ContactWarp &w = reinterpret_cast<ContactWarp *>(smem_raw)[wid];
  const int me = blockIdx.x * kThreads + threadIdx.x;
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
  w.P[lane] = P;
  w.V[lane] = V;
  w.C0[lane] = make_float4(c0x, c0y, c0z, ri);
  w.ci[lane] = ci;
  w.fx[lane] = w.fy[lane] = w.fz[lane] = w.lost[lane] = w.flow[lane] = 0.0f;
  w.nb[lane] = 0;
  __syncthreads();   // spc, and every owner slot
  const int sh = u.GShift;
  const uint32_t gm = (uint32_t)u.GMask;
  const uint4 *seats = reinterpret_cast<const uint4 *>(a.seats);
  int qn = 0, nn = 0;   // queue fills (warp-uniform)
  // stage 1: the 27 neighbour cells in the reference's order, the warp in lockstep
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
        uint4 s0 = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty), s1 = s0;
        if (live && !(xadd(xadd(xmul(qx, qx), qy2), qz2) > u.link2)) {   // the nearest-point test
          const uint32_t yy = ((uint32_t)y + ((uint32_t)(x >> sh) << (sh - 1)) + wz) & gm;   // the x period skews y by half
          const uint32_t h = (row + yy) * (uint32_t)u.AW + col + ((uint32_t)x & gm);
          const uint4 *cp = seats + (size_t)h * 2;
          s0 = __ldg(cp);       // both halves of the cell: one 32-byte sector, one round trip
          s1 = __ldg(cp + 1);
        }
        const bool more = __any_sync(0xFFFFFFFFu, !(s0.w & 0x80000000u));   // any cell with more than four?
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          if (half && !more) break;
          const uint4 s = half ? s1 : s0;
          const uint32_t sv[4] = {s.x, s.y, s.z, s.w};
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            bool seat = !(sv[k] & 0x80000000u) && (int)(sv[k] & 0x3FFFFu) != me;
            if (seat) {   // the quantised cull: where the seat sat at the rebuild, against this particle now
              const f3 dq = mk(xsub(xadd(lx, spc[(sv[k] >> 18) & 15u]), p.x),
                               xsub(xadd(ly, spc[(sv[k] >> 22) & 15u]), p.y),
                               xsub(xadd(lz, spc[(sv[k] >> 26) & 15u]), p.z));
              seat = !(xdot(dq, dq) > u.reach2);
            }
            const unsigned bal = __ballot_sync(0xFFFFFFFFu, seat);
            if (seat) w.q[qn + __popc(bal & ((1u << lane) - 1u))] = (sv[k] & 0x3FFFFu) | ((uint32_t)lane << 18);
            qn += __popc(bal);
          }
        }
        __syncwarp();
        while (qn >= 64) {
          qn -= 64;
          drain_candidates(u, a, w, qn, 64, lane, nn);
        }
      }
    }
  }
  if (qn >= 32) {
    qn -= 32;
    drain_candidates(u, a, w, qn, 32, lane, nn);
  }
  if (qn > 0) drain_candidates(u, a, w, 0, qn, lane, nn);
  if (nn > 0) drain_neighbours(u, a, w, 0, nn, lane);
  __syncwarp();
  if (!live) return;
  const f3 push = mk(w.fx[lane], w.fy[lane], w.fz[lane]);
  const float lost = w.lost[lane], flow = w.flow[lane], nb = (float)w.nb[lane];
  f3 grav = mk(0.0f, 0.0f, 0.0f), g;
  if (FIELD) {
    grav = ld3(u.gField);   // SIM_GRAV_FIELD, src/glsl-sim.js:490-492: the whole of gravity
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
  a.posO[me] = make_float4(pn.x, pn.y, pn.z, body);
  a.velO[me] = make_float4(v.x, v.y, v.z, fdiv(u.tK * Q, ci));
  a.auxO[me] = make_float4(grav.x, grav.y, grav.z, nb);
  a.qO[me] = Q;
}

size_t contact_smem_bytes(int warps) { return sizeof(ContactWarp) * warps; }

cudaError_t init_kernels() {
  const cudaFuncAttribute smem = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(k_contact_step<8, false>, smem, (int)contact_smem_bytes(8));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_contact_step<4, false>, smem, (int)contact_smem_bytes(4));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_contact_step<8, true>, smem, (int)contact_smem_bytes(8));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_contact_step<4, true>, smem, (int)contact_smem_bytes(4));
  return e;
}

int launch_simulate(const ccs_uniforms *u, int N, const SimArgs &a, cudaStream_t st, int warps, bool field) {
  if (warps == 4 && field)
    k_contact_step<4, true><<<blocks_for(N, 128), 128, contact_smem_bytes(4), st>>>(u, a);
  else if (warps == 4)
    k_contact_step<4, false><<<blocks_for(N, 128), 128, contact_smem_bytes(4), st>>>(u, a);
  else if (field)
    k_contact_step<8, true><<<blocks_for(N, 256), 256, contact_smem_bytes(8), st>>>(u, a);
  else
    k_contact_step<8, false><<<blocks_for(N, 256), 256, contact_smem_bytes(8), st>>>(u, a);
  return 1;
}

}  // namespace ccs
