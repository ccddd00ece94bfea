// ccs_step.cu -- the per-particle kernels around the contact step: the contact
// grid (seat tables), the books' read-outs (diag) and the rigid carry of the
// approach.
#include <atomic>

#include "ccs_device.cuh"
#include "ccs_grid.cuh"
#include "ccs_internal.h"

namespace ccs {

int sm_count() {
  constexpr int kDevices = 64;
  static std::atomic<int> cache[kDevices];   // zero until the device's first lookup
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices) return 148;
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v > 0) return v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
  cache[dev].store(v, std::memory_order_relaxed);
  return v;
}

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
  const int cap = sm_count() * 16;
  if (g > cap) g = cap;
  k_fill_u32<<<g, kBlock, 0, st>>>(p, n, v);
  return 1;
}

// ---------------------------------------------------------------------------
// contact grid: src/glsl-sim.js:112-149 (SLOT_VS) with src/nbody.js:379-399,
// one thread per particle (grid_particle, ccs_grid.cuh: CAS insertion into the
// cell's eight ascending seats, the retired table's touched cells cleared)
// ---------------------------------------------------------------------------
// the uniforms by value: constant-bank operands, no load at the head of each warp's chain
__global__ void __launch_bounds__(kBlock) k_contact_grid(const ccs_uniforms u, const float4 *__restrict__ pos,
                                                         uint32_t *seats, uint32_t *__restrict__ hk,
                                                         uint32_t *seatsOld, const uint32_t *__restrict__ hkOld,
                                                         unsigned *status, unsigned *recMax) {
  grid_particle(u, blockIdx.x * blockDim.x + threadIdx.x, pos, seats, hk, seatsOld, hkOld, status, recMax);
}

int launch_contact_grid(const ccs_uniforms &u, int N, const float4 *pos, uint32_t *seats, uint32_t *hk,
                        uint32_t *seatsOld, const uint32_t *hkOld, unsigned *status, unsigned *recMax,
                        cudaStream_t st) {
  k_contact_grid<<<blocks_for(N), kBlock, 0, st>>>(u, pos, seats, hk, seatsOld, hkOld, status, recMax);
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
  if (u.ppSplit > 0) {
    phi += a.ppAll[me].w;   // the stencil-split P3M: every particle's own pair sum
  } else {
    const int seat = a.ppSlot[me];
    if (seat >= 0)
      for (int s = 0; s < 4; ++s) phi += a.ppForce[(size_t)s * a.cap + seat].w;
  }
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
