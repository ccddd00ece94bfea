// ccs_kernels.cu -- the sm_100a kernels of the simulation step.
//
// One kernel per pass of the reference's step (src/glsl-sim.js), re-designed
// for the B200 rather than translated from fragment shaders:
//   contact grid   -- one pass of lock-free sorted insertion into 32-byte cells
//                     (replaces the 8-pass depth peel, src/glsl-sim.js:112-156)
//   simulate       -- contacts + mesh gather + P3M add + kick/drift, one thread
//                     per particle over float4 state (src/glsl-sim.js:362-512)
//   deposit        -- cloud-in-cell with warp reduce-scatter before the L2
//                     atomics (replaces additive point blending, :158-219)
//   coarse/mono    -- 4^3 sums plus a deterministic tree for the monopole
//   far            -- block-to-block far field from a shared-memory copy of
//                     the coarse mesh (:252-295)
//   cell           -- one CTA per occupied coarse block, neighbour blocks
//                     staged through shared memory (:296-352)
//   pp gather/force-- shared-memory tiled all-pairs over the loose list
//                     (:669-754)
// Compiled with -fmad=false and IEEE div/sqrt: see ccs_device.cuh.
#include <climits>

#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kBlock = 256;
inline int blocks_for(long n, int b = kBlock) { return (int)((n + b - 1) / b); }
}  // namespace

// ---------------------------------------------------------------------------
// utility fill
// ---------------------------------------------------------------------------
__global__ void k_fill_u32(uint32_t *p, size_t n, uint32_t v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
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
// peel's result -- independent of the order threads arrive in.  The same
// launch retires the previous table by clearing the cells it touched, so the
// next rebuild finds it empty without a 2 x G^3 x 32-byte memset.
// ---------------------------------------------------------------------------
// Lock-free, and bounded: a thread gives up after kMaxRetries failed swaps
// (only a degenerate pile -- e.g. non-finite positions all hashing to one cell
// -- comes near it), drops the word it carries and raises kStatusGrid in the
// status word the host reads at its next synchronisation (CCS_E_KERNEL).
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
  const float gx = P.x * u.invCell, gy = P.y * u.invCell, gz = P.z * u.invCell;
  const float fx = floorf(gx), fy = floorf(gy), fz = floorf(gz);
  const uint32_t qx = (uint32_t)clampf((gx - fx) * 15.0f, 0.0f, 14.0f);
  const uint32_t qy = (uint32_t)clampf((gy - fy) * 15.0f, 0.0f, 14.0f);
  const uint32_t qz = (uint32_t)clampf((gz - fz) * 15.0f, 0.0f, 14.0f);
  const uint32_t w = (uint32_t)i | (qx << 18) | (qy << 22) | (qz << 26) | 0x40000000u;
  const uint32_t h = hash_cell(u, (int)fx, (int)fy, (int)fz);
  hk[i] = h;
  seat_insert(seats + (size_t)h * kSeats, w, status);
}

int launch_contact_grid(const ccs_uniforms *u, int N, const float4 *pos, uint32_t *seats, uint32_t *hk,
                        uint32_t *seatsOld, const uint32_t *hkOld, unsigned *status, cudaStream_t st) {
  k_contact_grid<<<blocks_for(N), kBlock, 0, st>>>(u, pos, seats, hk, seatsOld, hkOld, status);
  return 1;
}

// ---------------------------------------------------------------------------
// simulate: src/glsl-sim.js:362-512, simFS({gravity: 'mesh'})
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t seat_of(const uint4 &s0, const uint4 &s1, int k) {
  const uint4 &s = k < 4 ? s0 : s1;
  const int h = k & 3;
  return h == 0 ? s.x : h == 1 ? s.y : h == 2 ? s.z : s.w;
}

__global__ void __launch_bounds__(kBlock) k_simulate(const ccs_uniforms *__restrict__ U, const SimArgs a) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  const ccs_uniforms &u = *U;
  if (me >= u.N) return;
  const float4 P = a.pos[me], V = a.vel[me];
  f3 p = xyz(P), v = xyz(V);
  const float body = P.w;
  const float ri = a.mat[me];
  const float cpIron = u.cpIron;
  const float ci = ri * (modg(body, 4.0f) < 0.5f ? cpIron : 1.0f);
  const float Ti = V.w;
  const float cell = u.cell, link2 = u.link2, reach2 = u.reach2, touch = u.touch, K = u.K, Cd = u.C;
  f3 push = mk(0.0f, 0.0f, 0.0f);
  float nb = 0.0f, lost = 0.0f, flow = 0.0f;
  const int cx = (int)floorf(p.x * u.invCell), cy = (int)floorf(p.y * u.invCell), cz = (int)floorf(p.z * u.invCell);
  const f3 c0 = mk((float)cx * cell, (float)cy * cell, (float)cz * cell);
  const uint4 *seats = reinterpret_cast<const uint4 *>(a.seats);
#pragma unroll 1
  for (int dz = -1; dz <= 1; dz++)
#pragma unroll 1
    for (int dy = -1; dy <= 1; dy++)
#pragma unroll 1
      for (int dx = -1; dx <= 1; dx++) {
        const f3 lo = mk(c0.x + (float)dx * cell, c0.y + (float)dy * cell, c0.z + (float)dz * cell);
        const f3 q = mk(clampf(p.x, lo.x, lo.x + cell), clampf(p.y, lo.y, lo.y + cell),
                        clampf(p.z, lo.z, lo.z + cell)) - p;
        if (dot(q, q) > link2) continue;
        const uint32_t h = hash_cell(u, cx + dx, cy + dy, cz + dz);
        const uint4 s0 = __ldg(seats + (size_t)h * 2);
        const uint4 s1 = (s0.w & 0x80000000u) ? make_uint4(kEmpty, kEmpty, kEmpty, kEmpty) : __ldg(seats + (size_t)h * 2 + 1);
#pragma unroll
        for (int k = 0; k < kSeats; ++k) {
          const uint32_t sv = seat_of(s0, s1, k);
          if (sv & 0x80000000u) break;
          const int j = (int)(sv & 0x3FFFFu);
          if (j == me) continue;
          const f3 sp = mk(((float)((sv >> 18) & 15u) + 0.5f) / 15.0f, ((float)((sv >> 22) & 15u) + 0.5f) / 15.0f,
                           ((float)((sv >> 26) & 15u) + 0.5f) / 15.0f);
          const f3 dq = (lo + sp * cell) - p;
          if (dot(dq, dq) > reach2) continue;
          const float4 Pj = __ldg(a.pos + j);
          const f3 d = xyz(Pj) - p;
          const float r2 = dot(d, d);
          if (r2 < link2) {
            const float r = sqrtf(r2);
            const f3 n = d / fmaxf(r, 1e-6f);
            const float ov = touch - r;
            if (ov > 0.0f) {
              const float4 Vj = __ldg(a.vel + j);
              const float rj = __ldg(a.mat + j);
              const float cij = Cd * sqrtf(2.0f * ri * rj / (ri + rj));
              const float vn = dot(xyz(Vj) - v, n);
              const float fs = K * ov - cij * vn, fn = fmaxf(fs, 0.0f), on = fs >= 0.0f ? 1.0f : 0.0f;
              push = push - n * fn;
              lost += cij * vn * vn * on + K * ov * vn * (1.0f - on);
              const float cj = rj * (modg(Pj.w, 4.0f) < 0.5f ? cpIron : 1.0f);
              flow += (Vj.w - Ti) * (2.0f * ci * cj / (ci + cj));
            }
            nb += 1.0f;
          }
        }
      }
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
      const float wx = ox ? t.x : 1.0f - t.x, wy = oy ? t.y : 1.0f - t.y, wz = oz ? t.z : 1.0f - t.z;
      const int ax = min(bx + ox, 63), ay = min(by + oy, 63), az = min(bz + oz, 63);
      const float4 f = __ldg(F + fine_index(ax, ay, az));
      grav = grav + xyz(f) * (wx * wy * wz);
    }
    grav = grav - xyz(__ldg(F + kFine)) * u.Gm;
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
  const float sc = u.invM / ri, dt = u.dt, gdt = u.gdt;
  v = mk(v.x + (push.x * sc * dt + grav.x * gdt), v.y + (push.y * sc * dt + grav.y * gdt),
         v.z + (push.z * sc * dt + grav.z * gdt));
  const bool tgt = body < 3.5f;
  const f3 spin = tgt ? ld3(u.spin0) : ld3(u.spin1);
  const f3 cen = tgt ? ld3(u.cen0) : ld3(u.cen1);
  const f3 vr = cross(spin, p - cen);
  if (u.settle > 0.5f) {
    const f3 dv = (v - vr) * u.damp;
    const float sp = sqrtf(dot(dv, dv));
    v = vr + dv * fminf(1.0f, u.creep / fmaxf(sp, 1e-9f));
  }
  if (u.kick > 0.5f) v = (tgt ? ld3(u.bulk0) : ld3(u.bulk1)) + vr;
  const float Q = u.settle > 0.5f ? 0.0f : a.q[me] + (lost + flow * u.kappa / u.tK) * dt;
  p = p + v * dt;
  a.posO[me] = make_float4(p.x, p.y, p.z, body);
  a.velO[me] = make_float4(v.x, v.y, v.z, u.tK * Q / ci);
  a.auxO[me] = make_float4(grav.x, grav.y, grav.z, nb);
  a.qO[me] = Q;
}

int launch_simulate(const ccs_uniforms *u, int N, const SimArgs &a, cudaStream_t st) {
  k_simulate<<<blocks_for(N), kBlock, 0, st>>>(u, a);
  return 1;
}

// ---------------------------------------------------------------------------
// deposit: src/glsl-sim.js:168-211 (DEP_VS) with src/nbody.js:402-416.
// Each particle's eight cloud-in-cell corners carry (w m x, w m); particles in
// the other box are left out; a stray (in neither) adds its pull toward last
// time's monopole into the scratch texel.  Lanes of a warp whose particles
// share a base cell (the common case in Morton order) first reduce-scatter
// their 32 values (8 corners x 4 components) with 31 shuffles, so a warp
// issues 32 scalar L2 atomics instead of 256 vector ones; mixed warps fall
// back to per-lane float4 atomics.  Summation order is unspecified, as the
// reference's blending order is.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void reduce_scatter32(float (&v)[32], int lane) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int j = 0; j < s; ++j) {
      const float send = upper ? v[j] : v[j + s];
      const float keep = upper ? v[j + s] : v[j];
      v[j] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, s);
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_deposit(const ccs_uniforms *__restrict__ U, int box,
                                                    const float4 *__restrict__ pos, const float *__restrict__ mat,
                                                    const float4 *__restrict__ monoPrev, float4 *fine) {
  const ccs_uniforms &u = *U;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  bool in = false, stray = false;
  int bx = 0, by = 0, bz = 0;
  f3 t = mk(0, 0, 0), p = mk(0, 0, 0);
  float mr = 0.0f;
  float4 sw = make_float4(0, 0, 0, 0);
  if (i < u.N) {
    const float4 P = pos[i];
    p = xyz(P);
    mr = mat[i];
    f3 g;
    const int mine = box_of(u, p, g);
    if (mine == box) {
      in = true;
      const float fx = floorf(g.x), fy = floorf(g.y), fz = floorf(g.z);
      t = mk(g.x - fx, g.y - fy, g.z - fz);
      bx = (int)fx; by = (int)fy; bz = (int)fz;
    } else if (mine < 0) {
      stray = true;
      const float4 mono = *monoPrev;
      const f3 r = xyz(mono) / fmaxf(mono.w, 1e-6f) - p;
      const float inv = isqrt(dot(r, r) + u.eps2Mesh);
      const f3 w = r * (mr * inv * inv * inv);
      sw = make_float4(w.x, w.y, w.z, mr);
    }
  }
  // the strays' reaction: one float4 atomic per warp
  if (__any_sync(0xFFFFFFFFu, stray)) {
    float4 s = sw;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      s.x += __shfl_xor_sync(0xFFFFFFFFu, s.x, o);
      s.y += __shfl_xor_sync(0xFFFFFFFFu, s.y, o);
      s.z += __shfl_xor_sync(0xFFFFFFFFu, s.z, o);
      s.w += __shfl_xor_sync(0xFFFFFFFFu, s.w, o);
    }
    if (lane == 0) atomicAdd(fine + kFine, s);
  }
  const unsigned inMask = __ballot_sync(0xFFFFFFFFu, in);
  if (inMask == 0u) return;
  const int key = in ? (bz << 16) | (by << 8) | bx : -1 - lane;
  const int key0 = __shfl_sync(0xFFFFFFFFu, key, __ffs(inMask) - 1);
  const bool uniform = __all_sync(0xFFFFFFFFu, !in || key == key0) && __popc(inMask) > 1;
  float v[32];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
    const float wx = ox ? t.x : 1.0f - t.x, wy = oy ? t.y : 1.0f - t.y, wz = oz ? t.z : 1.0f - t.z;
    const bool ok = in && bx + ox <= 63 && by + oy <= 63 && bz + oz <= 63;
    const float w = ok ? wx * wy * wz * mr : 0.0f;
    v[4 * k + 0] = ok ? p.x * w : 0.0f;
    v[4 * k + 1] = ok ? p.y * w : 0.0f;
    v[4 * k + 2] = ok ? p.z * w : 0.0f;
    v[4 * k + 3] = ok ? 1.0f * w : 0.0f;
  }
  if (uniform) {
    reduce_scatter32(v, lane);
    const int k = lane >> 2, comp = lane & 3;
    const int b0 = key0 & 0xFF, b1 = (key0 >> 8) & 0xFF, b2 = key0 >> 16;
    const int cx = b0 + (k & 1), cy = b1 + ((k >> 1) & 1), cz = b2 + (k >> 2);
    if (cx <= 63 && cy <= 63 && cz <= 63 && v[0] != 0.0f)
      atomicAdd(reinterpret_cast<float *>(fine + fine_index(cx, cy, cz)) + comp, v[0]);
  } else if (in) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int cx = bx + (k & 1), cy = by + ((k >> 1) & 1), cz = bz + (k >> 2);
      if (cx > 63 || cy > 63 || cz > 63) continue;
      atomicAdd(fine + fine_index(cx, cy, cz), make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]));
    }
  }
}

int launch_deposit(const ccs_uniforms *u, int N, int box, const float4 *pos, const float *mat, const float4 *monoPrev,
                   float4 *fine, cudaStream_t st) {
  k_deposit<<<blocks_for(N), kBlock, 0, st>>>(u, box, pos, mat, monoPrev, fine);
  return 1;
}

// ---------------------------------------------------------------------------
// coarse and monopole: src/glsl-sim.js:222-251.  16 blocks x 256 threads, one
// thread per coarse block summing its 4^3 fine cells in the reference's loop
// order; the monopole is a fixed-shape tree over the 4096 sums finished by the
// last block to arrive (deterministic, unlike the single serial fragment).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_coarse(const float4 *__restrict__ fine, float4 *__restrict__ coarse,
                                                   float4 *partial, unsigned *counter, float4 *mono) {
  __shared__ float4 red[kBlock];
  __shared__ bool last;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int cx = b & 15, cy = (b >> 4) & 15, cz = b >> 8;
  float4 s = make_float4(0, 0, 0, 0);
  for (int z = 0; z < 4; z++)
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) {
        const float4 f = fine[fine_index(cx * 4 + x, cy * 4 + y, cz * 4 + z)];
        s.x += f.x; s.y += f.y; s.z += f.z; s.w += f.w;
      }
  coarse[b] = s;
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      float4 a = red[threadIdx.x];
      const float4 c = red[threadIdx.x + o];
      a.x += c.x; a.y += c.y; a.z += c.z; a.w += c.w;
      red[threadIdx.x] = a;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = red[0];
    __threadfence();
    const unsigned n = atomicAdd(counter, 1u);
    last = (n == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    float4 m = make_float4(0, 0, 0, 0);
    for (int k = 0; k < (int)gridDim.x; ++k) {
      const float4 c = __ldcg(partial + k);
      m.x += c.x; m.y += c.y; m.z += c.z; m.w += c.w;
    }
    *mono = m;
    *counter = 0u;
  }
}

int launch_coarse(const MeshBuf &m, cudaStream_t st) {
  k_coarse<<<kCoarse / kBlock, kBlock, 0, st>>>(m.fine, m.coarse, m.partial, m.counter, m.mono);
  return 1;
}

// ---------------------------------------------------------------------------
// far field: src/glsl-sim.js:263-295.  Each CTA copies the 4096 coarse sums
// (64 KB) into shared memory once; each thread owns one block and walks all
// 4096 in the reference's order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_far(const float4 *__restrict__ coarse, float4 *__restrict__ farA,
                                                float4 *__restrict__ farT0, float4 *__restrict__ farT1) {
  extern __shared__ float4 sc[];
  for (int k = threadIdx.x; k < kCoarse; k += blockDim.x) sc[k] = coarse[k];
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int cx = b & 15, cy = (b >> 4) & 15, cz = b >> 8;
  const float4 mc = sc[b];
  if (!(mc.w > 0.0f)) {
    farA[b] = farT0[b] = farT1[b] = make_float4(0, 0, 0, 0);
    return;
  }
  const f3 x = xyz(mc) / mc.w;
  f3 acc = mk(0, 0, 0), td = mk(0, 0, 0), to = mk(0, 0, 0);
  float pot = 0.0f;
  for (int kz = 0; kz < 16; kz++)
    for (int ky = 0; ky < 16; ky++)
      for (int kx = 0; kx < 16; kx++) {
        const int dm = max(abs(kx - cx), max(abs(ky - cy), abs(kz - cz)));
        if (dm <= 2) continue;
        const float4 m = sc[coarse_index(kx, ky, kz)];
        if (!(m.w > 0.0f)) continue;
        const f3 r = xyz(m) / m.w - x;
        const float inv2 = 1.0f / dot(r, r), inv = sqrtf(inv2), inv3 = inv * inv2, inv5 = inv3 * inv2;
        acc = acc + r * (m.w * inv3);
        pot -= m.w * inv;
        td = td + mk(m.w * (3.0f * r.x * r.x * inv5 - inv3), m.w * (3.0f * r.y * r.y * inv5 - inv3),
                     m.w * (3.0f * r.z * r.z * inv5 - inv3));
        to = to + mk(m.w * (3.0f * (r.x * r.y) * inv5), m.w * (3.0f * (r.x * r.z) * inv5),
                     m.w * (3.0f * (r.y * r.z) * inv5));
      }
  farA[b] = make_float4(acc.x, acc.y, acc.z, pot);
  farT0[b] = make_float4(td.x, td.y, td.z, to.x);
  farT1[b] = make_float4(to.y, to.z, 0.0f, 0.0f);
}

cudaError_t init_kernels() {
  return cudaFuncSetAttribute(k_far, cudaFuncAttributeMaxDynamicSharedMemorySize, kCoarse * (int)sizeof(float4));
}

int launch_far(const MeshBuf &m, cudaStream_t st) {
  k_far<<<kCoarse / kBlock, kBlock, kCoarse * sizeof(float4), st>>>(m.coarse, m.farA, m.farT0, m.farT1);
  return 1;
}

// ---------------------------------------------------------------------------
// cell gravity: src/glsl-sim.js:303-352.  One 64-thread CTA per coarse block
// (a fine cell can hold mass only if its block does); for each of the 125
// neighbour blocks in the reference's order the CTA stages the block's 64
// fine cells in shared memory and every thread sums them for its own cell.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(64) k_cell(const ccs_uniforms *__restrict__ U, const float4 *__restrict__ fine,
                                             const float4 *__restrict__ coarse, const float4 *__restrict__ farA,
                                             const float4 *__restrict__ farT0, const float4 *__restrict__ farT1,
                                             float4 *__restrict__ force) {
  __shared__ float4 nb[64];
  const int blk = blockIdx.x;
  const int ccx = blk & 15, ccy = (blk >> 4) & 15, ccz = blk >> 8;
  const int tx = threadIdx.x & 3, ty = (threadIdx.x >> 2) & 3, tz = threadIdx.x >> 4;
  const int c = fine_index(ccx * 4 + tx, ccy * 4 + ty, ccz * 4 + tz);
  if (blk == 0 && threadIdx.x == 0) force[kFine] = fine[kFine];   // the scratch texel, carried through
  const float4 mb = coarse[blk];
  if (!(mb.w > 0.0f)) {
    force[c] = make_float4(0, 0, 0, 0);
    return;
  }
  const float4 mc = fine[c];
  const bool occ = mc.w > 0.0f;
  const f3 x = occ ? xyz(mc) / mc.w : mk(0, 0, 0);
  const float eps2 = U->eps2Cell, Gm = U->Gm;
  f3 acc = mk(0, 0, 0);
  float pot = 0.0f;
  for (int kz = -2; kz <= 2; kz++)
    for (int ky = -2; ky <= 2; ky++)
      for (int kx = -2; kx <= 2; kx++) {
        const int kx_ = ccx + kx, ky_ = ccy + ky, kz_ = ccz + kz;
        if (kx_ < 0 || ky_ < 0 || kz_ < 0 || kx_ > 15 || ky_ > 15 || kz_ > 15) continue;
        const float4 m = coarse[coarse_index(kx_, ky_, kz_)];
        if (!(m.w > 0.0f)) continue;
        __syncthreads();
        nb[threadIdx.x] = fine[fine_index(kx_ * 4 + tx, ky_ * 4 + ty, kz_ * 4 + tz)];
        __syncthreads();
        if (occ) {
          const bool self = (kx == 0 && ky == 0 && kz == 0);
#pragma unroll 4
          for (int f = 0; f < 64; ++f) {
            if (self && f == (int)threadIdx.x) continue;
            const float4 mf = nb[f];
            if (!(mf.w > 0.0f)) continue;
            const f3 r = xyz(mf) / mf.w - x;
            const float inv = isqrt(dot(r, r) + eps2);
            acc = acc + r * (mf.w * inv * inv * inv);
            pot -= mf.w * inv;
          }
        }
      }
  if (!occ) {
    force[c] = make_float4(0, 0, 0, 0);
    return;
  }
  const float4 fa = farA[blk], t0 = farT0[blk], t1 = farT1[blk];
  const f3 d = x - xyz(mb) / mb.w;
  const f3 Td = mk(t0.x * d.x + t0.w * d.y + t1.x * d.z, t0.w * d.x + t0.y * d.y + t1.y * d.z,
                   t1.x * d.x + t1.y * d.y + t0.z * d.z);
  acc = acc + (xyz(fa) + Td);
  pot += fa.w - dot(xyz(fa), d) - 0.5f * dot(d, Td);
  force[c] = make_float4(acc.x * Gm, acc.y * Gm, acc.z * Gm, pot * Gm);
}

int launch_cell(const ccs_uniforms *u, const MeshBuf &m, cudaStream_t st) {
  k_cell<<<kCoarse, 64, 0, st>>>(u, m.fine, m.coarse, m.farA, m.farT0, m.farT1, m.force);
  return 1;
}

// ---------------------------------------------------------------------------
// P3M: src/glsl-sim.js:676-754 (PPGATHER_FS, PPFORCE_FS)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_pp_gather(const ccs_uniforms *__restrict__ U,
                                                      const float4 *__restrict__ pos, const float *__restrict__ mat,
                                                      const int *__restrict__ index, int cap,
                                                      float4 *__restrict__ list, float *__restrict__ box) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= cap) return;
  const int i = index[s];
  if (i < 0) {
    list[s] = make_float4(0, 0, 0, 0);
    box[s] = -1.0f;
    return;
  }
  const float4 P = pos[i];
  f3 g;
  box[s] = (float)box_of(*U, xyz(P), g);
  list[s] = make_float4(P.x, P.y, P.z, mat[i]);
}

int launch_pp_gather(const ccs_uniforms *u, const float4 *pos, const float *mat, const int *index, int cap,
                     float4 *list, float *box, cudaStream_t st) {
  k_pp_gather<<<blocks_for(cap), kBlock, 0, st>>>(u, pos, mat, index, cap, list, box);
  return 1;
}

constexpr int kPPTile = 128;
__global__ void __launch_bounds__(kPPTile) k_pp_force(const ccs_uniforms *__restrict__ U,
                                                      const float4 *__restrict__ list, const float *__restrict__ box,
                                                      int cap, const float2 *__restrict__ tab,
                                                      float4 *__restrict__ force) {
  __shared__ float4 sq[kPPTile];
  __shared__ float sb[kPPTile];
  __shared__ float2 stab[64];
  const ccs_uniforms &u = *U;
  const int count = u.ppCount;
  const int slice = blockIdx.y;
  const int me = blockIdx.x * kPPTile + threadIdx.x;
  const int share = (count + 3) >> 2, j0 = slice * share, j1 = min(j0 + share, count);
  float4 *o = force + (size_t)slice * cap + me;
  if (blockIdx.x * kPPTile >= count) {   // the whole tile is past the list
    if (me < cap) *o = make_float4(0, 0, 0, 0);
    return;
  }
  if (threadIdx.x < 64) stab[threadIdx.x] = tab[threadIdx.x];
  const float4 P = me < cap ? list[me] : make_float4(0, 0, 0, 0);
  const bool active = me < count && P.w != 0.0f;
  const float myBox = me < cap ? box[me] : -1.0f;
  const float cut = u.cut, a2 = u.a2, cut2 = cut * cut, a = sqrtf(a2), cut08 = 0.8f * cut;
  f3 acc = mk(0, 0, 0);
  float pot = 0.0f;
  for (int base = j0; base < j1; base += kPPTile) {
    __syncthreads();
    const int j = base + threadIdx.x;
    if (j < j1) { sq[threadIdx.x] = list[j]; sb[threadIdx.x] = box[j]; }
    __syncthreads();
    if (!active) continue;
    const int n = min(kPPTile, j1 - base);
    for (int jj = 0; jj < n; ++jj) {
      if (base + jj == me) continue;
      const float4 Q = sq[jj];
      const f3 d = xyz(Q) - xyz(P);
      const float r2 = dot(d, d);
      if (r2 >= cut2) continue;
      const float r = sqrtf(r2);
      const float xx = clampf(r / cut * 64.0f - 0.5f, 0.0f, 63.0f);
      const int k = (int)xx, k1 = min(k + 1, 63);
      const float tt = xx - (float)k;
      const float invN = isqrt(r2 + a2);
      const float ts = clampf((r - cut) / (cut08 - cut), 0.0f, 1.0f);
      const float taper = ts * ts * (3.0f - 2.0f * ts);
      const float same = (myBox >= 0.0f && sb[jj] == myBox) ? 1.0f : 0.0f;
      const float2 ta = stab[k], tb = stab[k1];
      const float Tx = (ta.x * (1.0f - tt) + tb.x * tt) * same;
      const float Ty = (ta.y * (1.0f - tt) + tb.y * tt) * same;
      const float fn = invN * invN * invN * r - Tx / fmaxf(r2, a2), mj = Q.w;
      acc = acc + (d / fmaxf(r, 1e-6f)) * (mj * fn * taper);
      pot += mj * (-invN - Ty / fmaxf(r, a)) * taper;
    }
  }
  if (me < cap) *o = active ? make_float4(acc.x * u.Gm, acc.y * u.Gm, acc.z * u.Gm, pot * u.Gm) : make_float4(0, 0, 0, 0);
}

int launch_pp_force(const ccs_uniforms *u, const float4 *list, const float *box, int cap, const float2 *tab,
                    float4 *force, cudaStream_t st) {
  dim3 grid((cap + kPPTile - 1) / kPPTile, 4);
  k_pp_force<<<grid, kPPTile, 0, st>>>(u, list, box, cap, tab, force);
  return 1;
}

// ---------------------------------------------------------------------------
// diag: src/glsl-sim.js:608-667
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_diag(const ccs_uniforms *__restrict__ U, const DiagArgs a) {
  const ccs_uniforms &u = *U;
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= u.N) return;
  const f3 p = xyz(a.pos[me]);
  const int cx = (int)floorf(p.x * u.invCell), cy = (int)floorf(p.y * u.invCell), cz = (int)floorf(p.z * u.invCell);
  const uint32_t h = hash_cell(u, cx, cy, cz);
  const uint4 *seats = reinterpret_cast<const uint4 *>(a.seats);
  const uint4 s0 = seats[(size_t)h * 2], s1 = seats[(size_t)h * 2 + 1];
  float seated = 0.0f, taken = 0.0f;
#pragma unroll
  for (int k = 0; k < kSeats; ++k) {
    const uint32_t sv = seat_of(s0, s1, k);
    if (sv & 0x80000000u) break;
    taken += 1.0f;
    if ((int)(sv & 0x3FFFFu) == me) seated = 1.0f;
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
      const float wx = ox ? t.x : 1.0f - t.x, wy = oy ? t.y : 1.0f - t.y, wz = oz ? t.z : 1.0f - t.z;
      phi += F[fine_index(min(bx + ox, 63), min(by + oy, 63), min(bz + oz, 63))].w * (wx * wy * wz);
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
// rigid carry: src/glsl-sim.js:537-570 (matrices column-major)
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
  const f3 spin = tgt ? ld3(u.spin0) : ld3(u.spin1);
  const f3 d = xyz(P) - cen;
  const f3 arm = mk(m[0] * d.x + m[3] * d.y + m[6] * d.z, m[1] * d.x + m[4] * d.y + m[7] * d.z,
                    m[2] * d.x + m[5] * d.y + m[8] * d.z);
  const f3 np = (cen + arm) + bulk * u.rdt;
  const f3 nv = bulk + cross(spin, arm);
  posO[i] = make_float4(np.x, np.y, np.z, P.w);
  velO[i] = make_float4(nv.x, nv.y, nv.z, vel[i].w);
  auxO[i] = aux[i];
  qO[i] = q[i];
}

int launch_rigid(const ccs_uniforms *u, int N, const float4 *pos, const float4 *vel, const float4 *aux,
                 const float *q, float4 *posO, float4 *velO, float4 *auxO, float *qO, cudaStream_t st) {
  k_rigid<<<blocks_for(N), kBlock, 0, st>>>(u, pos, vel, aux, q, posO, velO, auxO, qO);
  return 1;
}

// ---------------------------------------------------------------------------
// permute: src/glsl-sim.js:578-602 (PERM_FS) plus the CPU-side mat/home
// permutation of src/nbody.js:932-941, all as one gather on the device
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_permute(int N, const int32_t *__restrict__ perm,
                                                    const float4 *__restrict__ pos, const float4 *__restrict__ vel,
                                                    const float4 *__restrict__ aux, const float *__restrict__ q,
                                                    const float *__restrict__ mat, const float4 *__restrict__ home,
                                                    float4 *posO, float4 *velO, float4 *auxO, float *qO, float *matO,
                                                    float4 *homeO) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int s = perm[i];
  posO[i] = pos[s];
  velO[i] = vel[s];
  auxO[i] = aux[s];
  qO[i] = q[s];
  matO[i] = mat[s];
  if (home) homeO[i] = home[s];
}

int launch_permute(int N, const int32_t *perm, const float4 *pos, const float4 *vel, const float4 *aux,
                   const float *q, const float *mat, const float4 *home, float4 *posO, float4 *velO, float4 *auxO,
                   float *qO, float *matO, float4 *homeO, cudaStream_t st) {
  k_permute<<<blocks_for(N), kBlock, 0, st>>>(N, perm, pos, vel, aux, q, mat, home, posO, velO, auxO, qO, matO,
                                              homeO);
  return 1;
}

// ---------------------------------------------------------------------------
// Morton keys (src/nbody.js:878-882): 7 bits an axis over +-6 R of the
// largest body's core, computed in binary64 as the reference's JavaScript
// does, interleaved x -> bit 3k, y -> 3k+1, z -> 3k+2.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_morton_keys(int N, const float4 *__restrict__ pos, double cx, double cy,
                                                        double cz, uint32_t *__restrict__ keys,
                                                        int32_t *__restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float4 P = pos[i];
  const double c[3] = {cx, cy, cz};
  const double pv[3] = {(double)P.x, (double)P.y, (double)P.z};
  uint32_t m[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double v = floor((pv[k] - c[k] + 6.0) / 12.0 * 128.0);
    m[k] = (uint32_t)fmin(127.0, fmax(0.0, v));
  }
  uint32_t key = 0;
#pragma unroll
  for (int k = 0; k < 7; ++k)
    key |= ((m[0] >> k) & 1u) << (3 * k) | ((m[1] >> k) & 1u) << (3 * k + 1) | ((m[2] >> k) & 1u) << (3 * k + 2);
  keys[i] = key;
  idx[i] = i;
}

int launch_morton_keys(int N, const float4 *pos, double cx, double cy, double cz, uint32_t *keys, int32_t *idx,
                       cudaStream_t st) {
  k_morton_keys<<<blocks_for(N), kBlock, 0, st>>>(N, pos, cx, cy, cz, keys, idx);
  return 1;
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort, 7 bits a pass (128 bins).  Per pass: a per-tile
// histogram, one exclusive scan over the (bin, tile) matrix in bin-major
// order, then a scatter in which each tile's single warp walks its keys in
// order and ranks equal digits with __match_any_sync -- so equal keys keep
// their order (the stability a counting sort gives the reference).
// ---------------------------------------------------------------------------
constexpr int kRadixBits = 7, kRadixBins = 1 << kRadixBits, kRadixTile = 2048;

size_t radix_hist_words(int N) { return (size_t)kRadixBins * ((N + kRadixTile - 1) / kRadixTile) + 1; }

__global__ void __launch_bounds__(kBlock) k_radix_hist(int N, int shift, const uint32_t *__restrict__ keys,
                                                       uint32_t *__restrict__ hist, int tiles) {
  __shared__ uint32_t h[kRadixBins];
  for (int b = threadIdx.x; b < kRadixBins; b += blockDim.x) h[b] = 0;
  __syncthreads();
  const int base = blockIdx.x * kRadixTile;
  for (int k = threadIdx.x; k < kRadixTile; k += blockDim.x) {
    const int i = base + k;
    if (i < N) atomicAdd(&h[(keys[i] >> shift) & (kRadixBins - 1)], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kRadixBins; b += blockDim.x) hist[(size_t)b * tiles + blockIdx.x] = h[b];
}

__global__ void __launch_bounds__(1024) k_radix_scan(uint32_t *hist, int n) {
  // exclusive scan of n words by one CTA (n <= 128 * 128 for N <= 2^18)
  __shared__ uint32_t carry;
  __shared__ uint32_t warpSums[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const uint32_t v = i < n ? hist[i] : 0u;
    uint32_t x = v;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t s = lane < (int)(blockDim.x >> 5) ? warpSums[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
        if (lane >= o) s += y;
      }
      warpSums[lane] = s;
    }
    __syncthreads();
    const uint32_t before = (wid > 0 ? warpSums[wid - 1] : 0u) + carry;
    if (i < n) hist[i] = before + x - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + x;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(32) k_radix_scatter(int N, int shift, const uint32_t *__restrict__ keys,
                                                      const int32_t *__restrict__ vals,
                                                      const uint32_t *__restrict__ hist, int tiles,
                                                      uint32_t *__restrict__ keysO, int32_t *__restrict__ valsO) {
  __shared__ uint32_t off[kRadixBins];
  const int lane = threadIdx.x;
  for (int b = lane; b < kRadixBins; b += 32) off[b] = hist[(size_t)b * tiles + blockIdx.x];
  __syncwarp();
  const int base = blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixTile; r += 32) {
    const int i = base + r + lane;
    const bool ok = i < N;
    const uint32_t key = ok ? keys[i] : 0u;
    const uint32_t d = ok ? (key >> shift) & (kRadixBins - 1) : kRadixBins;   // sentinel bin for padding
    const unsigned act = __ballot_sync(0xFFFFFFFFu, ok);
    if (act == 0u) break;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
    const unsigned lower = peers & ((1u << lane) - 1u);
    if (ok) {
      const uint32_t dst = off[d] + __popc(lower);
      keysO[dst] = key;
      valsO[dst] = vals[i];
    }
    __syncwarp();
    if (ok && lower == 0u) off[d] += __popc(peers);
    __syncwarp();
  }
}

int launch_radix_sort(int N, int bits, uint32_t *keys, int32_t *vals, uint32_t *keysTmp, int32_t *valsTmp,
                      uint32_t *hist, cudaStream_t st) {
  const int tiles = (N + kRadixTile - 1) / kRadixTile;
  int launched = 0;
  uint32_t *ka = keys, *kb = keysTmp;
  int32_t *va = vals, *vb = valsTmp;
  const int passes = (bits + kRadixBits - 1) / kRadixBits;
  for (int p = 0; p < passes; ++p) {
    const int shift = p * kRadixBits;
    k_radix_hist<<<tiles, kBlock, 0, st>>>(N, shift, ka, hist, tiles);
    k_radix_scan<<<1, 1024, 0, st>>>(hist, kRadixBins * tiles);
    k_radix_scatter<<<tiles, 32, 0, st>>>(N, shift, ka, va, hist, tiles, kb, vb);
    launched += 3;
    uint32_t *tk = ka; ka = kb; kb = tk;
    int32_t *tv = va; va = vb; vb = tv;
  }
  if (ka != keys) {   // an odd number of passes leaves the result in the scratch pair
    cudaMemcpyAsync(keys, ka, sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(vals, va, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, st);
  }
  return launched;
}

__global__ void k_invert_perm(int N, const int32_t *__restrict__ perm, int32_t *__restrict__ into) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) into[perm[i]] = i;
}
int launch_invert_perm(int N, const int32_t *perm, int32_t *into, cudaStream_t st) {
  k_invert_perm<<<blocks_for(N), kBlock, 0, st>>>(N, perm, into);
  return 1;
}

// ---------------------------------------------------------------------------
// books: the binary64 sums of src/nbody.js:837-850, as per-block partials
// reduced in a fixed order by the last block (deterministic).
// ---------------------------------------------------------------------------
constexpr int kBooks = CCS_BOOKS;
size_t books_partial_doubles(int N) { return (size_t)kBooks * blocks_for(N) + 8; }

__global__ void __launch_bounds__(kBlock) k_books(int N, double mref, const float4 *__restrict__ pos,
                                                  const float4 *__restrict__ vel, const float *__restrict__ mat,
                                                  const float4 *__restrict__ diag, int withDiag,
                                                  double *__restrict__ partial, double *__restrict__ out) {
  __shared__ double red[kBooks][kBlock / 32];
  __shared__ bool last;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[kBooks];
#pragma unroll
  for (int k = 0; k < kBooks; ++k) v[k] = 0.0;
  if (i < N) {
    const double m = mref * (double)mat[i];
    const float4 P = pos[i], V = vel[i];
    const double bx = P.x, by = P.y, bz = P.z, bu = V.x, bv = V.y, bw = V.z;
    v[0] = m;
    v[1] = m * bu; v[2] = m * bv; v[3] = m * bw;
    v[4] = m * (by * bw - bz * bv); v[5] = m * (bz * bu - bx * bw); v[6] = m * (bx * bv - by * bu);
    v[7] = 0.5 * m * (bu * bu + bv * bv + bw * bw);
    if (withDiag) {
      const float4 D = diag[i];
      const double flag = D.y;
      const bool off = flag >= 2.0;
      v[8] = (off ? 1.0 : 0.5) * m * (double)D.x;
      v[9] = 0.5 * (double)D.w;
      v[10] = (flag - (off ? 2.0 : 0.0) < 0.5) ? 1.0 : 0.0;
      v[11] = D.z >= 7.5f ? 1.0 : 0.0;
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kBooks; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
    if (lane == 0) red[k][wid] = x;
  }
  __syncthreads();
  if (threadIdx.x < kBooks) {
    double s = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) s += red[threadIdx.x][w];
    partial[(size_t)blockIdx.x * kBooks + threadIdx.x] = s;
  }
  __syncthreads();
  unsigned *counter = reinterpret_cast<unsigned *>(partial + (size_t)gridDim.x * kBooks);
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x < kBooks) {
    __threadfence();
    double s = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) s += __ldcg(partial + (size_t)b * kBooks + threadIdx.x);
    out[threadIdx.x] = s;
  }
  if (last && threadIdx.x == 0) *counter = 0u;
}

int launch_books(int N, double mref, const float4 *pos, const float4 *vel, const float *mat, const float4 *diag,
                 double *partial, double *out, int withDiag, cudaStream_t st) {
  k_books<<<blocks_for(N), kBlock, 0, st>>>(N, mref, pos, vel, mat, diag, withDiag, partial, out);
  return 1;
}

}  // namespace ccs
