// ccs_grid.cuh -- one particle's part of the contact grid (src/glsl-sim.js:112-149, SLOT_VS, with
// src/nbody.js:379-399), shared by the grid kernel (ccs_step.cu) and the ensemble's persistent round
// (ccs_contact.cu).
//
// The reference fills seat k of every hashed cell with the lowest particle index above seat k-1 -- eight
// depth-peeled point passes.  Here every particle inserts its seat word into its cell's eight ascending
// seats with compare-and-swap, carrying any displaced word further down; a word that falls off the end is
// unseated.  Each seat only ever decreases, so the final cell holds exactly the eight lowest indices in
// ascending order -- the depth peel's result -- whatever order the threads arrive in.  A particle whose warp
// holds r lower indices in the same cell starts at seat r: those r end in the seats before its own whenever
// it is seated, and one with r >= 8 is unseated at once.  In Morton order most cell-mates share a warp, so
// most inserts take their seat at the first swap.  The same pass retires the previous table by clearing the
// cells it touched, so the next rebuild finds it empty without a memset of the 2 x G^3 x 32-byte tables.
//
// Lock-free, and bounded: a thread gives up after kMaxRetries failed swaps (only a degenerate pile -- e.g.
// non-finite positions all hashing to one cell -- comes near it), drops the word it carries and raises
// kStatusGrid in the status word the host reads at its next synchronisation (CCS_E_KERNEL).
#pragma once
#include "ccs_device.cuh"

namespace ccs {

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

// particle i's seat (every lane of the warp calls it: the cell-mates are found with one match.any).
// recMax, if not null, is zeroed by particle 0: the displacement the contact walk's record is good for,
// from none.
__device__ __forceinline__ void grid_particle(const ccs_uniforms &u, int i, const float4 *pos, uint32_t *seats,
                                              uint32_t *hk, uint32_t *seatsOld, const uint32_t *hkOld,
                                              unsigned *status, unsigned *recMax) {
  if (recMax && i == 0) *recMax = 0u;
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

}  // namespace ccs
