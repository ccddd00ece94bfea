// ccs_step.cu -- the per-particle kernels of the step: the contact grid, the
// contact step (contacts + mesh gather + P3M add + kick/drift), the books'
// read-outs (diag) and the rigid carry of the approach.
#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kBlock = 256;
inline int blocks_for(long n, int b = kBlock) { return (int)((n + b - 1) / b); }
}  // namespace

__global__ void k_fill_u32(uint32_t *p, size_t n, uint32_t v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) p[i] = v;
}
int launch_fill_u32(uint32_t *p, size_t n, uint32_t v, cudaStream_t st) {
  if (n == 0) return 0;
  int g = (int)((n + kBlock - 1) / kBlock);
  if (g > 148 * 16) g = 148 * 16;
  k_fill_u32<<<g, kBlock, 0, st>>>(p, n, v);
  return 1;
}

// ---------------------------------------------------------------------------
// contact grid: src/glsl-sim.js:112-149 (SLOT_VS) with src/nbody.js:379-399.
// The reference fills seat k of every hashed cell with the lowest particle
// index above seat k-1 -- eight depth-peeled point passes.  Here every
// particle inserts its seat word into its cell's eight ascending seats with
// compare-and-swap, carrying any displaced word further down; a word that
// falls off the end is unseated.  Each seat only ever decreases, so the final
// cell holds exactly the eight lowest indices in ascending order -- the depth
// peel's result -- whatever order the threads arrive in.  The same launch
// retires the previous table by clearing the cells it touched, so the next
// rebuild finds it empty without a memset of the 2 x G^3 x 32-byte tables.
//
// Lock-free, and bounded: a thread gives up after kMaxRetries failed swaps
// (only a degenerate pile -- e.g. non-finite positions all hashing to one
// cell -- comes near it), drops the word it carries and raises kStatusGrid in
// the status word the host reads at its next synchronisation (CCS_E_KERNEL).
// ---------------------------------------------------------------------------
constexpr int kMaxRetries = 1 << 20;

__device__ __forceinline__ void seat_insert(uint32_t *cell, uint32_t w, unsigned *status) {
  uint32_t wi = w & 0x3FFFFu;
  int retries = 0;
#pragma unroll 1
  for (int k = 0; k < kSeats; ++k) {
    uint32_t cur = __ldcg(cell + k);
    while (true) {
      if ((cur & 0x80000000u) != 0u || (cur & 0x3FFFFu) > wi) {
        const uint32_t prev = atomicCAS(cell + k, cur, w);
        if (prev != cur) {
          if (++retries > kMaxRetries) {
            atomicOr(status, kStatusGrid);
            return;
          }
          cur = prev;
          continue;
        }
        if (cur & 0x80000000u) return;   // took an empty seat
        w = cur;                         // displaced a higher index: carry it on
        wi = w & 0x3FFFFu;
      }
      break;
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_contact_grid(const ccs_uniforms *__restrict__ U,
                                                         const float4 *__restrict__ pos, uint32_t *seats,
                                                         uint32_t *__restrict__ hk, uint32_t *seatsOld,
                                                         const uint32_t *__restrict__ hkOld, unsigned *status) {
  const ccs_uniforms &u = *U;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= u.N) return;
  const uint32_t old = hkOld[i];
  if (old != kNoCell) {
    uint4 *c = reinterpret_cast<uint4 *>(seatsOld + (size_t)old * kSeats);
    const uint4 e = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
    c[0] = e;
    c[1] = e;
  }
  const float4 P = pos[i];
  float gx, gy, gz;
  int cx, cy, cz;
  cell_of(u, xyz(P), gx, gy, gz, cx, cy, cz);
  const uint32_t qx = (uint32_t)clampf(xmul(xsub(gx, (float)cx), 15.0f), 0.0f, 14.0f);
  const uint32_t qy = (uint32_t)clampf(xmul(xsub(gy, (float)cy), 15.0f), 0.0f, 14.0f);
  const uint32_t qz = (uint32_t)clampf(xmul(xsub(gz, (float)cz), 15.0f), 0.0f, 14.0f);
  const uint32_t w = (uint32_t)i | (qx << 18) | (qy << 22) | (qz << 26) | 0x40000000u;
  const uint32_t h = hash_cell(u, cx, cy, cz);
  hk[i] = h;
  seat_insert(seats + (size_t)h * kSeats, w, status);
}

int launch_contact_grid(const ccs_uniforms *u, int N, const float4 *pos, uint32_t *seats, uint32_t *hk,
                        uint32_t *seatsOld, const uint32_t *hkOld, unsigned *status, cudaStream_t st) {
  k_contact_grid<<<blocks_for(N), kBlock, 0, st>>>(u, pos, seats, hk, seatsOld, hkOld, status);
  return 1;
}

// ---------------------------------------------------------------------------
// the contact step: src/glsl-sim.js:362-512, simFS({gravity: 'mesh'}).
// One thread per particle.  The per-axis parts of the 27-cell walk -- each
// neighbour cell's lower corner, the squared distance to its nearest face and
// the pieces of its hash -- are worked out once, so a cell costs two adds for
// the nearest-point test and a few integer ops for its seat address.  A cell's
// first four seats arrive in one 16-byte load (the next four only when the
// fourth is taken), their positions are loaded together, and the quantised
// seat cull of the reference -- which only saves it a fetch -- is applied to
// the pairs inside the link radius, where it can change the outcome.  The
// pair set and the neighbour count are decided with exact arithmetic.
// ---------------------------------------------------------------------------
struct Contacts {
  f3 push;
  float nb, lost, flow;
};

struct Near {               // what every neighbour cell's visit needs
  f3 p, v;
  float ri, ci, Ti;
  int me;
};

__device__ __forceinline__ void contact(const ccs_uniforms &u, const SimArgs &a, const Near &s, float4 Pj,
                                        uint32_t j, float r, Contacts &c) {
  const float4 Vj = __ldg(a.vel + j);
  const float rj = __ldg(a.mat + j);
  const f3 d = xyz(Pj) - s.p;
  const f3 n = d * fdiv(1.0f, fmaxf(r, 1e-6f));
  const float ov = u.touch - r;
  const float cij = u.C * fsqrt(fdiv(2.0f * s.ri * rj, s.ri + rj));   // the dashpot for this pair's reduced mass
  const float vn = dot(xyz(Vj) - s.v, n);
  const float fs = u.K * ov - cij * vn;
  c.push = c.push - n * fmaxf(fs, 0.0f);                               // no tension
  c.lost += fs >= 0.0f ? cij * vn * vn : u.K * ov * vn;
  const float cj = rj * (is_iron(Pj.w) ? u.cpIron : 1.0f);
  c.flow += (Vj.w - s.Ti) * fdiv(2.0f * s.ci * cj, s.ci + cj);        // heat crosses the contact
}

__device__ __forceinline__ void four_seats(const ccs_uniforms &u, const SimArgs &a, const float *spc, const Near &s,
                                           f3 lo, uint4 w, Contacts &c) {
  const uint32_t sv[4] = {w.x, w.y, w.z, w.w};
  float4 Pj[4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (!(sv[k] & 0x80000000u)) Pj[k] = __ldg(a.pos + (sv[k] & 0x3FFFFu));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (sv[k] & 0x80000000u) break;                                   // seats are packed: the rest are empty
    const uint32_t j = sv[k] & 0x3FFFFu;
    if ((int)j == s.me) continue;
    const f3 d = xsub3(xyz(Pj[k]), s.p);
    const float r2 = xdot(d, d);
    if (!(r2 < u.link2)) continue;
    // where it sat at the rebuild, to a fifteenth of a cell: beyond reach, the reference never fetched it
    const f3 dq = mk(xsub(xadd(lo.x, spc[(sv[k] >> 18) & 15u]), s.p.x), xsub(xadd(lo.y, spc[(sv[k] >> 22) & 15u]), s.p.y),
                     xsub(xadd(lo.z, spc[(sv[k] >> 26) & 15u]), s.p.z));
    if (xdot(dq, dq) > u.reach2) continue;
    c.nb += 1.0f;
    const float r = __fsqrt_rn(r2);
    if (xsub(u.touch, r) > 0.0f) contact(u, a, s, Pj[k], j, r, c);
  }
}

#ifndef CCS_SIM_MIN_BLOCKS
#define CCS_SIM_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(kBlock, CCS_SIM_MIN_BLOCKS) k_simulate(const ccs_uniforms *__restrict__ U, const SimArgs a) {
  __shared__ float spc[16];   // seatPos(q) * uCell, exact
  const ccs_uniforms &u = *U;
  if (threadIdx.x < 16) spc[threadIdx.x] = xmul(__fdiv_rn((float)threadIdx.x + 0.5f, 15.0f), u.cell);
  __syncthreads();
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= u.N) return;
  const float4 P = a.pos[me], V = a.vel[me];
  Near s;
  s.p = xyz(P);
  s.v = xyz(V);
  s.me = me;
  const float body = P.w;
  s.ri = a.mat[me];
  s.ci = s.ri * (is_iron(body) ? u.cpIron : 1.0f);
  s.Ti = V.w;
  const f3 p = s.p;
  const float cell = u.cell;
  Contacts c{mk(0.0f, 0.0f, 0.0f), 0.0f, 0.0f, 0.0f};
  float gx, gy, gz;
  int cx, cy, cz;
  cell_of(u, p, gx, gy, gz, cx, cy, cz);
  // per axis, for the offsets -1, 0, +1: the neighbour cell's lower corner and the
  // square of the distance to its nearest point (src/glsl-sim.js:414-418), exact
  float lo[3][3], q2[3][3];
  {
    const float pc[3] = {p.x, p.y, p.z};
    const int cc[3] = {cx, cy, cz};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const float c0 = xmul((float)cc[ax], cell);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float l = xadd(c0, xmul((float)(d - 1), cell));
        const float q = xsub(clampf(pc[ax], l, xadd(l, cell)), pc[ax]);
        lo[ax][d] = l;
        q2[ax][d] = xmul(q, q);
      }
    }
  }
  // the pieces of hashAt (src/glsl-sim.js:84-90) for each offset
  const int sh = u.GShift;
  const uint32_t gm = (uint32_t)u.GMask;
  uint32_t hx[3], wx[3], wy[3], wz[3], by[3], bz[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int x = cx + d - 1, y = cy + d - 1, z = cz + d - 1;
    hx[d] = (uint32_t)x & gm;
    wx[d] = (uint32_t)(x >> sh) << (sh - 1);   // the x period skews y by half a period
    wz[d] = (uint32_t)(z >> sh) << (sh - 2);   // the z period skews y by a quarter
    wy[d] = (uint32_t)(y >> sh) << (sh - 1);   // the y period skews z by half
    by[d] = (uint32_t)y;
    bz[d] = (uint32_t)z;
  }
  const uint4 *seats = reinterpret_cast<const uint4 *>(a.seats);
  const float link2 = u.link2;
#pragma unroll 1
  for (int dz = 0; dz < 3; dz++)
#pragma unroll 1
    for (int dy = 0; dy < 3; dy++) {
      const float qyz = dy == 0 ? q2[1][0] : dy == 1 ? q2[1][1] : q2[1][2];
      const float qz = dz == 0 ? q2[2][0] : dz == 1 ? q2[2][1] : q2[2][2];
      const float loy = dy == 0 ? lo[1][0] : dy == 1 ? lo[1][1] : lo[1][2];
      const float loz = dz == 0 ? lo[2][0] : dz == 1 ? lo[2][1] : lo[2][2];
      const uint32_t byy = dy == 0 ? by[0] : dy == 1 ? by[1] : by[2];
      const uint32_t wyy = dy == 0 ? wy[0] : dy == 1 ? wy[1] : wy[2];
      const uint32_t bzz = dz == 0 ? bz[0] : dz == 1 ? bz[1] : bz[2];
      const uint32_t wzz = dz == 0 ? wz[0] : dz == 1 ? wz[1] : wz[2];
      const uint32_t z = (bzz + wyy) & gm;
      const uint32_t rowz = ((z >> u.SXShift) << sh), colz = (z & (uint32_t)u.SXMask) << sh;
#pragma unroll 1
      for (int dx = 0; dx < 3; dx++) {
        // nearest-point test: (qx^2 + qy^2) + qz^2 > link^2 skips the cell
        const float qx = dx == 0 ? q2[0][0] : dx == 1 ? q2[0][1] : q2[0][2];
        if (xadd(xadd(qx, qyz), qz) > link2) continue;
        const uint32_t wxx = dx == 0 ? wx[0] : dx == 1 ? wx[1] : wx[2];
        const uint32_t hxx = dx == 0 ? hx[0] : dx == 1 ? hx[1] : hx[2];
        const float lox = dx == 0 ? lo[0][0] : dx == 1 ? lo[0][1] : lo[0][2];
        const uint32_t y = (byy + wxx + wzz) & gm;
        const uint32_t h = (rowz + y) * (uint32_t)u.AW + colz + hxx;
        const uint4 *cellp = seats + (size_t)h * 2;
        const uint4 w0 = __ldg(cellp);
        const f3 lc = mk(lox, loy, loz);
        four_seats(u, a, spc, s, lc, w0, c);
        if (!(w0.w & 0x80000000u)) four_seats(u, a, spc, s, lc, __ldg(cellp + 1), c);
      }
    }
  f3 v = s.v;
  const float ri = s.ri, ci = s.ci;
  // SIM_GRAV_MESH, src/glsl-sim.js:469-488
  f3 grav = mk(0.0f, 0.0f, 0.0f), g;
  const int box = box_of(u, p, g);
  if (box >= 0) {
    const float4 *F = box == 0 ? a.forceA : a.forceB;
    const float fx = floorf(g.x), fy = floorf(g.y), fz = floorf(g.z);
    const f3 t = mk(g.x - fx, g.y - fy, g.z - fz);
    const int bx = (int)fx, by = (int)fy, bz = (int)fz;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      const float w = (ox ? t.x : 1.0f - t.x) * (oy ? t.y : 1.0f - t.y) * (oz ? t.z : 1.0f - t.z);
      const float4 f = __ldg(F + fine_index(min(bx + ox, 63), min(by + oy, 63), min(bz + oz, 63)));
      grav = grav + xyz(f) * w;
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
  // SIM_POST, src/glsl-sim.js:493-511
  const float dt = u.dt;
  v = v + c.push * (fdiv(u.invM, ri) * dt) + grav * u.gdt;
  const bool tgt = body < 3.5f;
  const f3 vr = cross(tgt ? ld3(u.spin0) : ld3(u.spin1), p - (tgt ? ld3(u.cen0) : ld3(u.cen1)));
  if (u.settle > 0.5f) {   // damp everything but the spin, and let nothing run
    const f3 dv = (v - vr) * u.damp;
    const float sp = fsqrt(dot(dv, dv));
    v = vr + dv * fminf(1.0f, fdiv(u.creep, fmaxf(sp, 1e-9f)));
  }
  if (u.kick > 0.5f) v = (tgt ? ld3(u.bulk0) : ld3(u.bulk1)) + vr;
  const float Q = u.settle > 0.5f ? 0.0f : a.q[me] + (c.lost + fdiv(c.flow * u.kappa, u.tK)) * dt;
  const f3 pn = p + v * dt;
  a.posO[me] = make_float4(pn.x, pn.y, pn.z, body);
  a.velO[me] = make_float4(v.x, v.y, v.z, fdiv(u.tK * Q, ci));
  a.auxO[me] = make_float4(grav.x, grav.y, grav.z, c.nb);
  a.qO[me] = Q;
}

int launch_simulate_lanes(const ccs_uniforms *u, int N, const SimArgs &a, cudaStream_t st) {
  k_simulate<<<blocks_for(N), kBlock, 0, st>>>(u, a);
  return 1;
}

// ---------------------------------------------------------------------------
// diag: src/glsl-sim.js:608-667 -- the potential at the particle, whether it
// holds a seat (+2 off the mesh), the seats its cell has taken, its heat
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_diag(const ccs_uniforms *__restrict__ U, const DiagArgs a) {
  const ccs_uniforms &u = *U;
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= u.N) return;
  const f3 p = xyz(a.pos[me]);
  float gx, gy, gz;
  int cx, cy, cz;
  cell_of(u, p, gx, gy, gz, cx, cy, cz);
  const uint32_t h = hash_cell(u, cx, cy, cz);
  const uint4 *seats = reinterpret_cast<const uint4 *>(a.seats);
  const uint4 s0 = seats[(size_t)h * 2], s1 = seats[(size_t)h * 2 + 1];
  const uint32_t sv[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
  float seated = 0.0f, taken = 0.0f;
#pragma unroll
  for (int k = 0; k < kSeats; ++k) {
    if (sv[k] & 0x80000000u) break;
    taken += 1.0f;
    if ((int)(sv[k] & 0x3FFFFu) == me) seated = 1.0f;
  }
  float phi = 0.0f, off = 0.0f;
  f3 g;
  const int box = box_of(u, p, g);
  if (box >= 0) {
    const float4 *F = box == 0 ? a.forceA : a.forceB;
    const float fx = floorf(g.x), fy = floorf(g.y), fz = floorf(g.z);
    const f3 t = mk(g.x - fx, g.y - fy, g.z - fz);
    const int bx = (int)fx, by = (int)fy, bz = (int)fz;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      const float w = (ox ? t.x : 1.0f - t.x) * (oy ? t.y : 1.0f - t.y) * (oz ? t.z : 1.0f - t.z);
      phi += F[fine_index(min(bx + ox, 63), min(by + oy, 63), min(bz + oz, 63))].w * w;
    }
    if (u.boxB > 0.5f) phi += box == 0 ? pot_at(u, p, *a.monoB) : pot_at(u, p, *a.monoA);
  } else {
    phi = pot_at(u, p, *a.monoA);
    if (u.boxB > 0.5f) phi += pot_at(u, p, *a.monoB);
    off = 2.0f;
  }
  const int seat = a.ppSlot[me];
  if (seat >= 0)
    for (int s = 0; s < 4; ++s) phi += a.ppForce[(size_t)s * a.cap + seat].w;
  a.diag[me] = make_float4(phi, seated + off, taken, a.q[me]);
}

int launch_diag(const ccs_uniforms *u, int N, const DiagArgs &a, cudaStream_t st) {
  k_diag<<<blocks_for(N), kBlock, 0, st>>>(u, a);
  return 1;
}

// ---------------------------------------------------------------------------
// rigid carry: src/glsl-sim.js:537-570 (matrices column-major), exact
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_rigid(const ccs_uniforms *__restrict__ U, const float4 *__restrict__ pos,
                                                  const float4 *__restrict__ vel, const float4 *__restrict__ aux,
                                                  const float *__restrict__ q, float4 *__restrict__ posO,
                                                  float4 *__restrict__ velO, float4 *__restrict__ auxO,
                                                  float *__restrict__ qO) {
  const ccs_uniforms &u = *U;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= u.N) return;
  const float4 P = pos[i];
  const bool tgt = P.w < 3.5f;
  const float *m = tgt ? u.rot0 : u.rot1;
  const f3 bulk = tgt ? ld3(u.bulk0) : ld3(u.bulk1), cen = tgt ? ld3(u.cen0) : ld3(u.cen1);
  const f3 w = tgt ? ld3(u.spin0) : ld3(u.spin1);
  const f3 d = xsub3(xyz(P), cen);
  const f3 arm = mk(xadd(xadd(xmul(m[0], d.x), xmul(m[3], d.y)), xmul(m[6], d.z)),
                    xadd(xadd(xmul(m[1], d.x), xmul(m[4], d.y)), xmul(m[7], d.z)),
                    xadd(xadd(xmul(m[2], d.x), xmul(m[5], d.y)), xmul(m[8], d.z)));
  const f3 np = mk(xadd(xadd(cen.x, arm.x), xmul(bulk.x, u.rdt)), xadd(xadd(cen.y, arm.y), xmul(bulk.y, u.rdt)),
                   xadd(xadd(cen.z, arm.z), xmul(bulk.z, u.rdt)));
  const f3 sw = mk(xsub(xmul(w.y, arm.z), xmul(w.z, arm.y)), xsub(xmul(w.z, arm.x), xmul(w.x, arm.z)),
                   xsub(xmul(w.x, arm.y), xmul(w.y, arm.x)));
  posO[i] = make_float4(np.x, np.y, np.z, P.w);
  velO[i] = make_float4(xadd(bulk.x, sw.x), xadd(bulk.y, sw.y), xadd(bulk.z, sw.z), vel[i].w);
  auxO[i] = aux[i];
  qO[i] = q[i];
}

int launch_rigid(const ccs_uniforms *u, int N, const float4 *pos, const float4 *vel, const float4 *aux,
                 const float *q, float4 *posO, float4 *velO, float4 *auxO, float *qO, cudaStream_t st) {
  k_rigid<<<blocks_for(N), kBlock, 0, st>>>(u, pos, vel, aux, q, posO, velO, auxO, qO);
  return 1;
}

}  // namespace ccs
