// ccs_split.cu -- the stencil-split P3M: pairs of mesh nodes far apart are left to the mesh, everything
// nearer is summed particle by particle, exactly.
//
// The reference corrects only the loose list (src/nbody.js:851-870), and only against the mesh's
// placement-averaged pair table (src/glsl-sim.js:700-754), so a particle inside a body keeps the mesh's
// near field: a cell-centre sum softened by FH^2/2 at every distance (src/glsl-sim.js:303-352), a few per
// cent off Newton.  This form splits the interaction exactly instead.  A particle's cloud-in-cell weights
// w_i(k) over its 8 nodes and a source's w_j(l) over its 8 make a partition of unity over node pairs
// (k, l); the mesh keeps the pairs of nodes more than S cells apart in every axis' Chebyshev sense
// (k_cell_tide, unsoftened, with the tidal tensor and the pull's second gradient so the gather is second
// order in the offset from each node's centre of mass), and this pass keeps the rest, each particle pair
// weighted by
//   W_ij = sum over (k, l) with |k - l|_inf <= S of w_i(k) w_j(l) = prod over axes of W_a(D_a, t_ia, t_ja),
// D_a = b_ja - b_ia the base nodes' offset: 1 for |D| <= S - 1, (1 - t_j) + t_i t_j for D = S,
// (1 - t_i) + t_i t_j for D = -S, t_i (1 - t_j) for D = S + 1, (1 - t_i) t_j for D = -S - 1, 0 beyond.
// Each pair is Newton softened at the particle radius a (the reference's own pairwise softening,
// src/glsl-sim.js:745).  Both particles must read the same box; a particle in neither gets the boxes'
// monopoles as before.
//
// Layout: particles are sorted (stable radix sort) by key = box * 64^3 + their base node's fine index,
// so a row of nodes (fixed y, z) is one contiguous range; start[key] is the first sorted position with a
// key >= key.  The work is cut into items of one occupied target node's particles: 64 at a time while 64
// remain, then 32, then the rest.  A warp takes an item and walks the (2S + 3)^2 rows of source nodes
// around the node, staging 64 of their sources at a time in shared memory with the per-axis weight factors
// already reduced to W_a = P_a + Q_a t_ia and the mass folded in (the offset D is the same for every
// target of the node), so a pair costs the three factors' FMAs, two products and the softened Newton term.
// An item of 64 gives each lane two targets; of 32, one; of fewer, each target L lanes (the largest power
// of two that fits), which take every L-th source and add up by shuffles -- most occupied nodes outside
// the bodies hold a few particles whose stencils reach thousands of sources, and a target a lane would
// leave most lanes idle there.  Items are taken heaviest first (a counting sort by the log2 of a lane's
// share of the pairs) from one counter by a persistent grid, so the last items are short.  Sums run in a
// fixed order per item (rows, then sorted order, then the shuffle tree): deterministic.
//
// Nodes holding at least symMin particles (16 by default: the bodies and most of their surfaces) are "big",
// and a pair of particles in two big nodes is evaluated once, by the node of the lower key, its reaction
// added to the other particle (Newton's third law: the weight, the softened distance and the pull are the
// same both ways).  A big node's work is cut into CTA items of up to 256 targets (64 a warp, two a lane) and
// one z slab of its stencil, taken heaviest first by a persistent grid (k_pp_split_both, whose warps then
// take the small nodes' items, so those fill the first phase's tail): the CTA stages 64 sources at a time; a
// source chunk of big nodes of higher key (or the node itself, from the item's first target on, each pair
// once) is walked by each lane in a rotating order, so the reaction owed to each source travels with it from
// lane to lane (one shuffle a component a step) and is complete after 32 steps; the warps add theirs in
// shared memory and the CTA adds the chunk's to the sources' sums with one vector atomic a source.  Small
// nodes in a big node's stencil are sources one way only, and small nodes' own items take every source one
// way, so every pair is counted once in each direction (k_split_finish writes the big nodes' sums out).  The
// big nodes' sums are float atomics: summed in any order.  symMin = 0 takes every node one way (the form
// above, k_pp_split: deterministic).  The items count the pairs they take, one way and both ways.
#include <algorithm>

#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kBlock = 256;
inline int blocks_for(long n, int b = kBlock) { return (int)((n + b - 1) / b); }
constexpr int kSplitWarps = 4;       // a CTA of the pair kernel: warps that each take their own items
constexpr int kSplitStage = 64;      // sources a warp stages at a time
constexpr int kSplitClasses = 32;    // cost classes of the items (log2 of a lane's pairs)
// the pass's scratch (split_work_bytes): counters (the small nodes' items' and, kCtrBig on, the big nodes'),
// the small items as made and in the order they are taken, the big items likewise, then the big nodes'
// particles' sums (sorted order)
constexpr int kCtrTmp = 0, kCtrTaken = 1, kCtrCount = 32, kCtrStart = 64, kCtrFill = 96, kCtrBig = 128;
// after both lists' counters (kCtrBig + kCtrFill + 31 = 255), two 64-bit counts: the pairs the items take one
// way and both ways
constexpr int kCtrPairs = 256;
constexpr int kCtrInts = 264;   // a multiple of 4, so the items that follow stay 16-byte aligned
static_assert(kCtrBig + kCtrFill + 32 <= kCtrPairs && kCtrPairs + 4 <= kCtrInts && kCtrInts % 4 == 0,
              "the counters do not overlap, and the items after them are 16-byte aligned");
inline size_t item_cap(int N) { return 2 * (size_t)N + (size_t)N / 64 + 64; }
constexpr int kSymWarps = 4;                    // a big item's CTA
constexpr int kSymTargets = 64 * kSymWarps;     // its targets: two a lane
constexpr int kSymStage = 64;                   // sources staged at a time
// the big nodes' items: with at least kSymMinNode particles a big node, at most N / kSymMinNode big nodes of
// count / 256 + 1 chunks each, one item a chunk and z slab of the stencil (2 S + 3 <= 9 slabs)
inline size_t big_cap(int N) { return 9 * ((size_t)N / kSymMinNode + (size_t)N / kSymTargets + 64); }
struct SplitWork {
  int *ctr;
  int4 *tmp, *items, *tmpBig, *itemsBig;
  float4 *acc;
};
inline SplitWork split_work(void *work, int N) {
  SplitWork w;
  w.ctr = static_cast<int *>(work);
  w.tmp = reinterpret_cast<int4 *>(w.ctr + kCtrInts);
  w.items = w.tmp + item_cap(N);
  w.tmpBig = w.items + item_cap(N);
  w.itemsBig = w.tmpBig + big_cap(N);
  w.acc = reinterpret_cast<float4 *>(w.itemsBig + big_cap(N));
  return w;
}
}  // namespace

// per particle: the box it reads and its base node (exact: the gather's own box_of and floor), as one key
__global__ void __launch_bounds__(kBlock) k_split_keys(const ccs_uniforms *__restrict__ U,
                                                       const float4 *__restrict__ pos, uint32_t *__restrict__ keys,
                                                       int32_t *__restrict__ vals) {
  const ccs_uniforms &u = *U;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= u.N) return;
  f3 g;
  const int box = box_of(u, xyz(pos[i]), g);
  uint32_t key = (uint32_t)kSplitKeys;
  if (box >= 0) key = (uint32_t)box * kFine + fine_index((int)floorf(g.x), (int)floorf(g.y), (int)floorf(g.z));
  keys[i] = key;
  vals[i] = i;
}

// start[x] = the first sorted position whose key is >= x, for x in [0, kSplitKeys + 1]: a lower bound each
__global__ void __launch_bounds__(kBlock) k_split_starts(int N, const uint32_t *__restrict__ keys,
                                                         int *__restrict__ start) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x > kSplitKeys + 1) return;
  int lo = 0, hi = N;   // keys[lo - 1] < x <= keys[hi]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (keys[mid] < (uint32_t)x) lo = mid + 1;
    else hi = mid;
  }
  start[x] = lo;
}

// the sorted sources (position, mass; fractional place in the base node, base node) and the occupied target
// nodes (the first sorted position of each key in a box)
__global__ void __launch_bounds__(kBlock) k_split_sources(const ccs_uniforms *__restrict__ U,
                                                          const uint32_t *__restrict__ keys,
                                                          const int32_t *__restrict__ vals,
                                                          const float4 *__restrict__ pos,
                                                          const float *__restrict__ mat, float4 *__restrict__ src,
                                                          float4 *__restrict__ srcT, int *__restrict__ cells,
                                                          int *__restrict__ nCells) {
  const ccs_uniforms &u = *U;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= u.N) return;
  const uint32_t key = keys[k];
  const int i = vals[k];
  const float4 P = pos[i];
  f3 g = mk(0, 0, 0);
  if (key < (uint32_t)kSplitKeys) box_of(u, xyz(P), g);
  src[k] = make_float4(P.x, P.y, P.z, mat[i]);
  srcT[k] = make_float4(g.x - floorf(g.x), g.y - floorf(g.y), g.z - floorf(g.z), __int_as_float((int)key));
  if (key < (uint32_t)kSplitKeys && (k == 0 || keys[k - 1] != key)) cells[atomicAdd(nCells, 1)] = k;
}

// the weight factor of one axis for a base-node offset D: W_a = alpha + beta t_i + gamma t_j + delta t_i t_j
__device__ __forceinline__ float4 split_coef(int D, int S) {
  if (D <= S - 1 && D >= 1 - S) return make_float4(1.0f, 0.0f, 0.0f, 0.0f);
  if (D == S) return make_float4(1.0f, 0.0f, -1.0f, 1.0f);
  if (D == -S) return make_float4(1.0f, -1.0f, 0.0f, 1.0f);
  if (D == S + 1) return make_float4(0.0f, 1.0f, 0.0f, -1.0f);
  if (D == -S - 1) return make_float4(0.0f, 0.0f, 1.0f, -1.0f);
  return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// per occupied target node: its items (first target, targets) and each item's cost class, from the number
// of sources in the node's stencil and how many of them one lane of the item's warp takes
template <int S>
__global__ void __launch_bounds__(kBlock) k_split_items(const int *__restrict__ start, const int *__restrict__ cells,
                                                        const int *__restrict__ nCells,
                                                        const float4 *__restrict__ srcT, int *__restrict__ ctr,
                                                        int4 *__restrict__ tmp, int4 *__restrict__ tmpBig,
                                                        int symMin) {
  constexpr int R = S + 1;
  const int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= *nCells) return;
  const int k0 = cells[ci];
  const int key = __float_as_int(srcT[k0].w);
  const int k1 = start[key + 1];
  const int box = key / kFine, node = key - box * kFine;
  const int bx = node & 63, by = (node >> 6) & 63, bz = node >> 12;
  const int x0 = max(bx - R, 0), x1 = min(bx + R, 63);
  if (symMin > 0 && k1 - k0 >= symMin) {
    // a big node: items of up to kSymTargets targets, one a z slab of the stencil, each costed by the sources
    // it takes (big nodes of higher key, about half of its own, every small node)
    for (int dz = -R; dz <= R; ++dz) {
      const int z = bz + dz;
      if (z < 0 || z > 63) continue;
      long both = 0, one = 0;   // the slab's sources other than the node itself: big of higher key, small
      bool own = false;
      for (int y = max(by - R, 0); y <= min(by + R, 63); ++y) {
        const int rowKey = box * kFine + fine_index(0, y, z);
        for (int x = x0; x <= x1; ++x) {
          const int X = rowKey + x, n = start[X + 1] - start[X];
          if (X == key) own = true;
          else if (n > 0 && n < symMin) one += n;
          else if (n > 0 && X > key) both += n;
        }
      }
      if (both + one == 0 && !(own && k1 - k0 > 1)) continue;
      for (int f = k0; f < k1; f += kSymTargets) {
        const int nt = min(kSymTargets, k1 - f);
        // targets f .. f + nt - 1 each meet the node's particles after them once
        const long mine = own ? (long)nt * (k1 - 1 - f) - (long)nt * (nt - 1) / 2 : 0;
        const long pairsBoth = (long)nt * both + mine, pairsOne = (long)nt * one;
        const long share = (pairsBoth + pairsOne) / 64;   // a lane's pairs, as the small items count them
        const int cls = 31 - __clz((int)min(max(share, 1L), (long)INT_MAX));
        tmpBig[atomicAdd(ctr + kCtrBig + kCtrTmp, 1)] = make_int4(f, nt, cls, dz);
        atomicAdd(ctr + kCtrBig + kCtrCount + cls, 1);
        atomicAdd(reinterpret_cast<unsigned long long *>(ctr + kCtrPairs), (unsigned long long)pairsOne);
        atomicAdd(reinterpret_cast<unsigned long long *>(ctr + kCtrPairs + 2), (unsigned long long)pairsBoth);
      }
    }
    return;
  }
  long sources = 0;
  for (int z = max(bz - R, 0); z <= min(bz + R, 63); ++z)
    for (int y = max(by - R, 0); y <= min(by + R, 63); ++y) {
      const int rowKey = box * kFine + fine_index(0, y, z);
      sources += start[rowKey + x1 + 1] - start[rowKey + x0];
    }
  for (int f = k0; f < k1;) {
    const int left = k1 - f;
    const int nt = left >= 64 ? 64 : left >= 32 ? 32 : left;
    const int L = nt >= 32 ? 1 : 1 << (31 - __clz(32 / nt));   // lanes a target: nt * L <= 32
    const long share = (nt == 64 ? 2 * sources : sources) / L;
    const int cls = 31 - __clz((int)min(max(share, 1L), (long)INT_MAX));
    tmp[atomicAdd(ctr + kCtrTmp, 1)] = make_int4(f, nt, cls, L);
    atomicAdd(ctr + kCtrCount + cls, 1);
    atomicAdd(reinterpret_cast<unsigned long long *>(ctr + kCtrPairs), (unsigned long long)nt * sources);
    f += nt;
  }
}

// the items' places, heaviest class first
__global__ void __launch_bounds__(32) k_split_order(int *__restrict__ ctr) {
  const int c = threadIdx.x;   // one lane a class; lane 0 the heaviest
  const int cls = kSplitClasses - 1 - c;
  const int n = ctr[kCtrCount + cls];
  int incl = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (c >= o) incl += v;
  }
  ctr[kCtrStart + cls] = incl - n;
  ctr[kCtrFill + cls] = 0;
}

__global__ void __launch_bounds__(kBlock) k_split_scatter(int *__restrict__ ctr, const int4 *__restrict__ tmp,
                                                          int4 *__restrict__ items) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ctr[kCtrTmp]) return;
  const int4 t = tmp[i];
  items[ctr[kCtrStart + t.z] + atomicAdd(ctr + kCtrFill + t.z, 1)] = t;
}

// one source's part of a pair: its position, and its weight factors for the item's node with its mass in
// the x factor (sP: x, y, z, P_z; sW: P_x m, Q_x m, P_y, Q_y; sQ: Q_z)
struct SplitStage {
  float4 P[kSplitStage];
  float4 W[kSplitStage];
  float Q[kSplitStage];
};

// the one-way items (each warp its own; stage: kSplitWarps warps' staging)
template <int S>
__device__ __forceinline__ void split_small(const ccs_uniforms *__restrict__ U, const int *__restrict__ start,
                                            const float4 *__restrict__ src, const float4 *__restrict__ srcT,
                                            const int32_t *__restrict__ vals, int *__restrict__ ctr,
                                            const int4 *__restrict__ items, float4 *__restrict__ out,
                                            SplitStage *stage) {
  constexpr int R = S + 1;   // the stencil's reach in nodes
  constexpr unsigned kAll = 0xFFFFFFFFu;
  SplitStage &sg = stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const float a2 = U->a2, Gm = U->Gm;
  const float selfInv = rsqrtf(a2);   // a target meets itself with W = 1 and d = 0: only this potential
  const int nItems = ctr[kCtrTmp];
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(ctr + kCtrTaken, 1);
    it = __shfl_sync(kAll, it, 0);
    if (it >= nItems) break;
    const int4 item = items[it];
    const int first = item.x, nt = item.y, L = item.w;
    const bool two = nt == 64;
    const int tgt = two ? lane : lane / L, phase = two ? 0 : lane % L;
    const bool va = tgt < nt;
    const int ta = first + tgt, tc = ta + 32;
    const float4 Pa = va ? src[ta] : make_float4(0, 0, 0, 0), Pc = two ? src[tc] : Pa;
    const float4 Ta = va ? srcT[ta] : make_float4(0, 0, 0, 0), Tc = two ? srcT[tc] : Ta;
    const int key = __float_as_int(srcT[first].w);
    const int box = key / kFine, node = key - box * kFine;
    const int bx = node & 63, by = (node >> 6) & 63, bz = node >> 12;
    float ax = 0, ay = 0, az = 0, pa = 0, cx = 0, cy = 0, cz = 0, pc = 0;
#pragma unroll 1
    for (int dz = -R; dz <= R; ++dz) {
      const int z = bz + dz;
      if (z < 0 || z > 63) continue;
      const float4 cz4 = split_coef(dz, S);
#pragma unroll 1
      for (int dy = -R; dy <= R; ++dy) {
        const int y = by + dy;
        if (y < 0 || y > 63) continue;
        const float4 cy4 = split_coef(dy, S);
        const int x0 = max(bx - R, 0), x1 = min(bx + R, 63);
        const int rowKey = box * kFine + fine_index(0, y, z);
        const int s0 = start[rowKey + x0], s1 = start[rowKey + x1 + 1];
#pragma unroll 1
        for (int c0 = s0; c0 < s1; c0 += kSplitStage) {
          const int cn = min(kSplitStage, s1 - c0);
          __syncwarp();   // the previous chunk's readers are done
          for (int j = lane; j < cn; j += 32) {
            const float4 P = src[c0 + j], T = srcT[c0 + j];
            const float4 cx4 = split_coef((__float_as_int(T.w) & 63) - bx, S);
            sg.P[j] = make_float4(P.x, P.y, P.z, cz4.x + cz4.z * T.z);
            sg.W[j] = make_float4((cx4.x + cx4.z * T.x) * P.w, (cx4.y + cx4.w * T.x) * P.w, cy4.x + cy4.z * T.y,
                                  cy4.y + cy4.w * T.y);
            sg.Q[j] = cz4.y + cz4.w * T.z;
          }
          __syncwarp();
          if (two) {
#pragma unroll 4
            for (int j = 0; j < cn; ++j) {
              const float4 P = sg.P[j], Wc = sg.W[j];
              const float Qz = sg.Q[j];
              {
                const float w = (Wc.x + Wc.y * Ta.x) * (Wc.z + Wc.w * Ta.y) * (P.w + Qz * Ta.z);
                const float dx = P.x - Pa.x, dy_ = P.y - Pa.y, dz_ = P.z - Pa.z;
                const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
                const float pw = w * inv, s = pw * (inv * inv);
                ax = fmaf(dx, s, ax);
                ay = fmaf(dy_, s, ay);
                az = fmaf(dz_, s, az);
                pa -= pw;
              }
              {
                const float w = (Wc.x + Wc.y * Tc.x) * (Wc.z + Wc.w * Tc.y) * (P.w + Qz * Tc.z);
                const float dx = P.x - Pc.x, dy_ = P.y - Pc.y, dz_ = P.z - Pc.z;
                const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
                const float pw = w * inv, s = pw * (inv * inv);
                cx = fmaf(dx, s, cx);
                cy = fmaf(dy_, s, cy);
                cz = fmaf(dz_, s, cz);
                pc -= pw;
              }
            }
          } else if (va) {
#pragma unroll 4
            for (int j = phase; j < cn; j += L) {
              const float4 P = sg.P[j], Wc = sg.W[j];
              const float Qz = sg.Q[j];
              const float w = (Wc.x + Wc.y * Ta.x) * (Wc.z + Wc.w * Ta.y) * (P.w + Qz * Ta.z);
              const float dx = P.x - Pa.x, dy_ = P.y - Pa.y, dz_ = P.z - Pa.z;
              const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
              const float pw = w * inv, s = pw * (inv * inv);
              ax = fmaf(dx, s, ax);
              ay = fmaf(dy_, s, ay);
              az = fmaf(dz_, s, az);
              pa -= pw;
            }
          }
        }
      }
    }
    if (!two && L > 1) {   // a target's lanes add up their shares (the lanes of a target are consecutive)
      for (int o = L >> 1; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(kAll, ax, o);
        ay += __shfl_xor_sync(kAll, ay, o);
        az += __shfl_xor_sync(kAll, az, o);
        pa += __shfl_xor_sync(kAll, pa, o);
      }
    }
    if (va && phase == 0) out[vals[ta]] = make_float4(ax * Gm, ay * Gm, az * Gm, fmaf(Pa.w, selfInv, pa) * Gm);
    if (two) out[vals[tc]] = make_float4(cx * Gm, cy * Gm, cz * Gm, fmaf(Pc.w, selfInv, pc) * Gm);
  }
}

template <int S>
__global__ void __launch_bounds__(32 * kSplitWarps, 8) k_pp_split(const ccs_uniforms *__restrict__ U,
                                                                  const int *__restrict__ start,
                                                                  const float4 *__restrict__ src,
                                                                  const float4 *__restrict__ srcT,
                                                                  const int32_t *__restrict__ vals,
                                                                  int *__restrict__ ctr,
                                                                  const int4 *__restrict__ items,
                                                                  float4 *__restrict__ out) {
  __shared__ SplitStage stage[kSplitWarps];
  split_small<S>(U, start, src, srcT, vals, ctr, items, out, stage);
}

struct SymShared {   // a big item's CTA: its staged chunk
  float4 P[kSymStage];   // position, the z factor's constant part
  float4 W[kSymStage];   // the x factor (constant, slope) and the y factor's; one way: x times mass
  float2 Q[kSymStage];   // the z factor's slope, the source's mass
  float4 R[kSymStage];   // the chunk's reactions, summed over the warps
  int item;
};

// the big nodes' items (see the file's head): a CTA of kSymWarps warps, warp w's targets first + 64 w + lane
// and + 32, over one z slab of the stencil
template <int S>
__device__ __forceinline__ void split_big(const ccs_uniforms *__restrict__ U, const int *__restrict__ start,
                                          const float4 *__restrict__ src, const float4 *__restrict__ srcT,
                                          int *__restrict__ ctr, const int4 *__restrict__ items,
                                          float4 *__restrict__ acc, int symMin, SymShared &sh) {
  constexpr int R = S + 1;
  constexpr unsigned kAll = 0xFFFFFFFFu;
  float4 *sP = sh.P, *sW = sh.W, *sR = sh.R;
  float2 *sQ = sh.Q;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, tid = threadIdx.x;
  const float a2 = U->a2;
  const int nItems = ctr[kCtrBig + kCtrTmp];
  for (;;) {
    __syncthreads();   // the previous item's last chunk is done
    if (tid == 0) sh.item = atomicAdd(ctr + kCtrBig + kCtrTaken, 1);
    __syncthreads();
    const int it = sh.item;
    if (it >= nItems) break;
    const int4 item = items[it];
    const int first = item.x, nt = item.y, dz = item.w;
    const int ta = first + 64 * wid + lane, tc = ta + 32;
    const bool va = 64 * wid + lane < nt, vc = 64 * wid + lane + 32 < nt;
    // an absent target has no mass: it owes no reaction, and its own sums are never written
    const float4 Pa = va ? src[ta] : make_float4(0, 0, 0, 0), Pc = vc ? src[tc] : make_float4(0, 0, 0, 0);
    const float4 Ta = va ? srcT[ta] : make_float4(0, 0, 0, 0), Tc = vc ? srcT[tc] : make_float4(0, 0, 0, 0);
    const int key = __float_as_int(srcT[first].w);
    const int box = key / kFine, node = key - box * kFine;
    const int bx = node & 63, by = (node >> 6) & 63, bz = node >> 12;
    const int z = bz + dz;
    const float4 cz4 = split_coef(dz, S);
    const int x0 = max(bx - R, 0), x1 = min(bx + R, 63);
    float ax = 0, ay = 0, az = 0, pa = 0, cx = 0, cy = 0, cz = 0, pc = 0;
#pragma unroll 1
    for (int dy = -R; dy <= R; ++dy) {
      const int y = by + dy;
      if (y < 0 || y > 63) continue;
      const float4 cy4 = split_coef(dy, S);
      const int rowKey = box * kFine + fine_index(0, y, z);
      // the row's nodes in runs of one kind: 1 both ways (big, higher key; the node itself), 2 one way (small),
      // 0 none (big, lower key: it takes these pairs); empty nodes join the run they sit in
      int x = x0;
#pragma unroll 1
      while (x <= x1) {
        int X = rowKey + x;
        if (start[X + 1] == start[X]) {
          ++x;
          continue;
        }
        const int n0 = start[X + 1] - start[X];
        const int kind = X == key ? 1 : n0 < symMin ? 2 : X > key ? 1 : 0;
        const int r0 = X == key ? first : start[X];
        int xe = x + 1;
        while (xe <= x1) {
          const int Y = rowKey + xe, n = start[Y + 1] - start[Y];
          if (Y == key) break;   // the node itself starts a run of its own, at the item's first target
          if (n > 0 && (n < symMin ? 2 : Y > key ? 1 : 0) != kind) break;
          ++xe;
        }
        const int r1 = start[rowKey + xe];
        const int maskEnd = X == key ? first + nt : 0;   // chunks before it hold the item's own targets
        x = xe;
        if (kind == 0) continue;
#pragma unroll 1
        for (int c0 = r0; c0 < r1; c0 += kSymStage) {
          const int cn = min(kSymStage, r1 - c0);
          __syncthreads();   // the previous chunk's readers, and its reactions' flush, are done
          if (tid < kSymStage) {
            if (tid < cn) {
              const float4 P = src[c0 + tid], T = srcT[c0 + tid];
              const float4 cx4 = split_coef((__float_as_int(T.w) & 63) - bx, S);
              const float mx = kind == 2 ? P.w : 1.0f;   // one way: the mass in the x factor, as k_pp_split
              sP[tid] = make_float4(P.x, P.y, P.z, cz4.x + cz4.z * T.z);
              sW[tid] = make_float4((cx4.x + cx4.z * T.x) * mx, (cx4.y + cx4.w * T.x) * mx, cy4.x + cy4.z * T.y,
                                    cy4.y + cy4.w * T.y);
              sQ[tid] = make_float2(cz4.y + cz4.w * T.z, P.w);
            } else {   // past the chunk's end: no weight, no mass
              sP[tid] = make_float4(0, 0, 0, 0);
              sW[tid] = make_float4(0, 0, 0, 0);
              sQ[tid] = make_float2(0, 0);
            }
            sR[tid] = make_float4(0, 0, 0, 0);
          }
          __syncthreads();
          if (kind == 2) {
#pragma unroll 4
            for (int j = 0; j < cn; ++j) {
              const float4 P = sP[j], Wc = sW[j];
              const float Qz = sQ[j].x;
              {
                const float w = (Wc.x + Wc.y * Ta.x) * (Wc.z + Wc.w * Ta.y) * (P.w + Qz * Ta.z);
                const float dx = P.x - Pa.x, dy_ = P.y - Pa.y, dz_ = P.z - Pa.z;
                const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
                const float pw = w * inv, s = pw * (inv * inv);
                ax = fmaf(dx, s, ax);
                ay = fmaf(dy_, s, ay);
                az = fmaf(dz_, s, az);
                pa -= pw;
              }
              {
                const float w = (Wc.x + Wc.y * Tc.x) * (Wc.z + Wc.w * Tc.y) * (P.w + Qz * Tc.z);
                const float dx = P.x - Pc.x, dy_ = P.y - Pc.y, dz_ = P.z - Pc.z;
                const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
                const float pw = w * inv, s = pw * (inv * inv);
                cx = fmaf(dx, s, cx);
                cy = fmaf(dy_, s, cy);
                cz = fmaf(dz_, s, cz);
                pc -= pw;
              }
            }
          } else {
            // both ways: each lane meets the chunk's 32-source halves in a rotating order, the reaction it owes a
            // source carried with that source from lane to lane; a chunk holding the item's own targets counts
            // each pair once (the source after the target in sorted order)
            const bool masked = c0 < maskEnd;
#pragma unroll 1
            for (int h = 0; h < 2 && 32 * h < cn; ++h) {
              float rx = 0, ry = 0, rz = 0, rp = 0;
#pragma unroll 4
              for (int k = 0; k < 32; ++k) {
                const int s = 32 * h + ((lane + k) & 31);
                const float4 P = sP[s], Wc = sW[s];
                const float2 QM = sQ[s];
                float wa = (Wc.x + Wc.y * Ta.x) * (Wc.z + Wc.w * Ta.y) * (P.w + QM.x * Ta.z);
                float wc = (Wc.x + Wc.y * Tc.x) * (Wc.z + Wc.w * Tc.y) * (P.w + QM.x * Tc.z);
                if (masked) {
                  if (c0 + s <= ta) wa = 0.0f;
                  if (c0 + s <= tc) wc = 0.0f;
                }
                {
                  const float dx = P.x - Pa.x, dy_ = P.y - Pa.y, dz_ = P.z - Pa.z;
                  const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
                  const float pw = wa * inv, s3 = pw * (inv * inv);
                  const float sj = s3 * QM.y, si = s3 * Pa.w;
                  ax = fmaf(dx, sj, ax);
                  ay = fmaf(dy_, sj, ay);
                  az = fmaf(dz_, sj, az);
                  pa = fmaf(-pw, QM.y, pa);
                  rx = fmaf(-dx, si, rx);
                  ry = fmaf(-dy_, si, ry);
                  rz = fmaf(-dz_, si, rz);
                  rp = fmaf(-pw, Pa.w, rp);
                }
                {
                  const float dx = P.x - Pc.x, dy_ = P.y - Pc.y, dz_ = P.z - Pc.z;
                  const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
                  const float pw = wc * inv, s3 = pw * (inv * inv);
                  const float sj = s3 * QM.y, si = s3 * Pc.w;
                  cx = fmaf(dx, sj, cx);
                  cy = fmaf(dy_, sj, cy);
                  cz = fmaf(dz_, sj, cz);
                  pc = fmaf(-pw, QM.y, pc);
                  rx = fmaf(-dx, si, rx);
                  ry = fmaf(-dy_, si, ry);
                  rz = fmaf(-dz_, si, rz);
                  rp = fmaf(-pw, Pc.w, rp);
                }
                // the next step's source for this lane is the one lane + 1 has now: take its reaction along
                const int from = (lane + 1) & 31;
                rx = __shfl_sync(kAll, rx, from);
                ry = __shfl_sync(kAll, ry, from);
                rz = __shfl_sync(kAll, rz, from);
                rp = __shfl_sync(kAll, rp, from);
              }
              // after 32 steps each source's reaction is back at the lane of its own slot
              const int s = 32 * h + lane;
              if (s < cn) {
                atomicAdd(&sR[s].x, rx);
                atomicAdd(&sR[s].y, ry);
                atomicAdd(&sR[s].z, rz);
                atomicAdd(&sR[s].w, rp);
              }
            }
            __syncthreads();
            if (tid < cn) atomicAdd(acc + c0 + tid, sR[tid]);
          }
        }
      }
    }
    if (va) atomicAdd(acc + ta, make_float4(ax, ay, az, pa));
    if (vc) atomicAdd(acc + tc, make_float4(cx, cy, cz, pc));
  }
}

// both ways: the big nodes' CTA items first (heaviest first), then each warp takes the small nodes' one-way
// items, which fill the tail of the first phase
template <int S>
__global__ void __launch_bounds__(32 * kSymWarps, 6) k_pp_split_both(const ccs_uniforms *__restrict__ U,
                                                                     const int *__restrict__ start,
                                                                     const float4 *__restrict__ src,
                                                                     const float4 *__restrict__ srcT,
                                                                     const int32_t *__restrict__ vals,
                                                                     int *__restrict__ ctr,
                                                                     const int4 *__restrict__ items,
                                                                     const int4 *__restrict__ itemsBig,
                                                                     float4 *__restrict__ acc,
                                                                     float4 *__restrict__ out, int symMin) {
  static_assert(kSymWarps == kSplitWarps, "one CTA shape for both phases");
  __shared__ SymShared sh;
  __shared__ SplitStage stage[kSplitWarps];
  split_big<S>(U, start, src, srcT, ctr, itemsBig, acc, symMin, sh);
  split_small<S>(U, start, src, srcT, vals, ctr, items, out, stage);
}

// the big nodes' particles: their sums out, x Gm (the small nodes' are written by the one-way items)
__global__ void __launch_bounds__(kBlock) k_split_finish(const ccs_uniforms *__restrict__ U, int N,
                                                         const int *__restrict__ start,
                                                         const float4 *__restrict__ srcT,
                                                         const int32_t *__restrict__ vals,
                                                         const float4 *__restrict__ acc, float4 *__restrict__ out,
                                                         int symMin) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int key = __float_as_int(srcT[k].w);
  if (key >= kSplitKeys || start[key + 1] - start[key] < symMin) return;
  const float Gm = U->Gm;
  const float4 s = acc[k];
  out[vals[k]] = make_float4(s.x * Gm, s.y * Gm, s.z * Gm, s.w * Gm);
}

size_t split_start_ints() { return (size_t)kSplitKeys + 2; }

const void *split_pair_counts(const void *work) { return static_cast<const int *>(work) + kCtrPairs; }

size_t split_work_bytes(int N) {
  return sizeof(int) * kCtrInts + 2 * sizeof(int4) * (item_cap(N) + big_cap(N)) + sizeof(float4) * (size_t)N;
}

int launch_pp_split(const ccs_uniforms *U, int N, int S, const float4 *pos, const float *mat, uint32_t *keys,
                    int32_t *vals, uint32_t *keysTmp, int32_t *valsTmp, uint32_t *hist, int *start, float4 *src,
                    float4 *srcT, int *cells, int *nCells, void *work, float4 *out, int symMin, cudaStream_t st) {
  int launched = 0;
  const SplitWork w = split_work(work, N);
  k_split_keys<<<blocks_for(N), kBlock, 0, st>>>(U, pos, keys, vals);
  launched += 1 + launch_radix_sort(N, 20, keys, vals, keysTmp, valsTmp, hist, st);
  k_split_starts<<<blocks_for(kSplitKeys + 2), kBlock, 0, st>>>(N, keys, start);
  cudaMemsetAsync(nCells, 0, sizeof(int), st);
  cudaMemsetAsync(w.ctr, 0, sizeof(int) * kCtrInts, st);
  k_split_sources<<<blocks_for(N), kBlock, 0, st>>>(U, keys, vals, pos, mat, src, srcT, cells, nCells);
  cudaMemsetAsync(out, 0, sizeof(float4) * N, st);   // particles in neither box get no pairs
  if (symMin > 0) cudaMemsetAsync(w.acc, 0, sizeof(float4) * N, st);
  if (S == 1)
    k_split_items<1><<<blocks_for(N), kBlock, 0, st>>>(start, cells, nCells, srcT, w.ctr, w.tmp, w.tmpBig, symMin);
  else if (S == 2)
    k_split_items<2><<<blocks_for(N), kBlock, 0, st>>>(start, cells, nCells, srcT, w.ctr, w.tmp, w.tmpBig, symMin);
  else
    k_split_items<3><<<blocks_for(N), kBlock, 0, st>>>(start, cells, nCells, srcT, w.ctr, w.tmp, w.tmpBig, symMin);
  k_split_order<<<1, 32, 0, st>>>(w.ctr);
  k_split_scatter<<<blocks_for((long)item_cap(N)), kBlock, 0, st>>>(w.ctr, w.tmp, w.items);
  launched += 6;
  if (symMin > 0) {
    k_split_order<<<1, 32, 0, st>>>(w.ctr + kCtrBig);
    k_split_scatter<<<blocks_for((long)big_cap(N)), kBlock, 0, st>>>(w.ctr + kCtrBig, w.tmpBig, w.itemsBig);
    launched += 2;
  }
  if (symMin > 0) {
    const int gs = sm_count() * 6;
    if (S == 1)
      k_pp_split_both<1><<<gs, 32 * kSymWarps, 0, st>>>(U, start, src, srcT, vals, w.ctr, w.items, w.itemsBig,
                                                        w.acc, out, symMin);
    else if (S == 2)
      k_pp_split_both<2><<<gs, 32 * kSymWarps, 0, st>>>(U, start, src, srcT, vals, w.ctr, w.items, w.itemsBig,
                                                        w.acc, out, symMin);
    else
      k_pp_split_both<3><<<gs, 32 * kSymWarps, 0, st>>>(U, start, src, srcT, vals, w.ctr, w.items, w.itemsBig,
                                                        w.acc, out, symMin);
    k_split_finish<<<blocks_for(N), kBlock, 0, st>>>(U, N, start, srcT, vals, w.acc, out, symMin);
    return launched + 2;
  }
  const int grid = sm_count() * 8;
  if (S == 1)
    k_pp_split<1><<<grid, 32 * kSplitWarps, 0, st>>>(U, start, src, srcT, vals, w.ctr, w.items, out);
  else if (S == 2)
    k_pp_split<2><<<grid, 32 * kSplitWarps, 0, st>>>(U, start, src, srcT, vals, w.ctr, w.items, out);
  else
    k_pp_split<3><<<grid, 32 * kSplitWarps, 0, st>>>(U, start, src, srcT, vals, w.ctr, w.items, out);
  return launched + 1;
}

// the kernels one split pair pass launches (the sort's count included)
int pp_split_launches(int symMin) { return 7 + 3 * 3 + (symMin > 0 ? 3 : 0); }

}  // namespace ccs
