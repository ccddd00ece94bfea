// ccs_step.cu -- the per-particle kernels around the contact step: the contact
// grid (seat tables), the books' read-outs (diag) and the rigid carry of the
// approach.
#include <atomic>

#include "ccs_device.cuh"
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
// contact grid: src/glsl-sim.js:112-149 (SLOT_VS) with src/nbody.js:379-399.
// The reference fills seat k of every hashed cell with the lowest particle
// index above seat k-1 -- eight depth-peeled point passes.  Here every
// particle inserts its seat word into its cell's eight ascending seats with
// compare-and-swap, carrying any displaced word further down; a word that
// falls off the end is unseated.  Each seat only ever decreases, so the final
// cell holds exactly the eight lowest indices in ascending order -- the depth
// peel's result -- whatever order the threads arrive in.  A particle whose
// warp holds r lower indices in the same cell starts at seat r: those r end
// in the seats before its own whenever it is seated, and one with r >= 8 is
// unseated at once.  In Morton order most cell-mates share a warp, so most
// inserts take their seat at the first swap.  The same launch
// retires the previous table by clearing the cells it touched, so the next
// rebuild finds it empty without a memset of the 2 x G^3 x 32-byte tables.
//
// Lock-free, and bounded: a thread gives up after kMaxRetries failed swaps
// (only a degenerate pile -- e.g. non-finite positions all hashing to one
// cell -- comes near it), drops the word it carries and raises kStatusGrid in
// the status word the host reads at its next synchronisation (CCS_E_KERNEL).
// ---------------------------------------------------------------------------
constexpr int kMaxRetries = 1 << 20;

// Each seat is first tried as if it were empty: the swap checks the guess and, when it fails, returns the
// seat's word -- one round trip a seat where a read and then a swap would take two.
__device__ __forceinline__ void seat_insert(uint32_t *cell, uint32_t w, unsigned *status, int start) {
  uint32_t wi = w & 0x3FFFFu;
  int retries = 0;
#pragma unroll 1
  for (int k = start; k < kSeats; ++k) {
    uint32_t cur = kEmpty;
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

// the uniforms by value: constant-bank operands, no load at the head of each warp's chain
__global__ void __launch_bounds__(kBlock) k_contact_grid(const ccs_uniforms u, const float4 *__restrict__ pos,
                                                         uint32_t *seats, uint32_t *__restrict__ hk,
                                                         uint32_t *seatsOld, const uint32_t *__restrict__ hkOld,
                                                         unsigned *status, unsigned *recMax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (recMax && i == 0) *recMax = 0u;   // the displacement the contact walk's record is good for, from none
  const bool live = i < u.N;
  float4 P = make_float4(0, 0, 0, 0);
  if (live) P = pos[i];
  float gx, gy, gz;
  int cx, cy, cz;
  cell_of(u, xyz(P), gx, gy, gz, cx, cy, cz);
  const uint32_t h = live ? hash_cell(u, cx, cy, cz) : 0xFFFFFFFFu;
  // the lanes that share this cell hold ascending indices: the lower ones end in the seats before this one's
  const unsigned mates = __match_any_sync(0xFFFFFFFFu, h);
  if (!live) return;
  const int start = __popc(mates & ((1u << (threadIdx.x & 31)) - 1u));
  const uint32_t old = hkOld[i];
  if (old != kNoCell) {
    uint4 *c = reinterpret_cast<uint4 *>(seatsOld + (size_t)old * kSeats);
    const uint4 e = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
    c[0] = e;
    c[1] = e;
  }
  const uint32_t qx = (uint32_t)clampf(xmul(xsub(gx, (float)cx), 15.0f), 0.0f, 14.0f);
  const uint32_t qy = (uint32_t)clampf(xmul(xsub(gy, (float)cy), 15.0f), 0.0f, 14.0f);
  const uint32_t qz = (uint32_t)clampf(xmul(xsub(gz, (float)cz), 15.0f), 0.0f, 14.0f);
  const uint32_t w = (uint32_t)i | (qx << 18) | (qy << 22) | (qz << 26) | 0x40000000u;
  hk[i] = h;
  if (start < kSeats) seat_insert(seats + (size_t)h * kSeats, w, status, start);
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
