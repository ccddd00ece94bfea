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
// the pass's scratch (split_work_bytes): counters, then the items as made, then in the order they are taken
constexpr int kCtrTmp = 0, kCtrTaken = 1, kCtrCount = 32, kCtrStart = 64, kCtrFill = 96, kCtrInts = 128;
inline size_t item_cap(int N) { return 2 * (size_t)N + (size_t)N / 64 + 64; }
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
                                                        int4 *__restrict__ tmp) {
  constexpr int R = S + 1;
  const int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= *nCells) return;
  const int k0 = cells[ci];
  const int key = __float_as_int(srcT[k0].w);
  const int k1 = start[key + 1];
  const int box = key / kFine, node = key - box * kFine;
  const int bx = node & 63, by = (node >> 6) & 63, bz = node >> 12;
  const int x0 = max(bx - R, 0), x1 = min(bx + R, 63);
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

template <int S>
__global__ void __launch_bounds__(32 * kSplitWarps, 8) k_pp_split(const ccs_uniforms *__restrict__ U,
                                                                  const int *__restrict__ start,
                                                                  const float4 *__restrict__ src,
                                                                  const float4 *__restrict__ srcT,
                                                                  const int32_t *__restrict__ vals,
                                                                  int *__restrict__ ctr,
                                                                  const int4 *__restrict__ items,
                                                                  float4 *__restrict__ out) {
  constexpr int R = S + 1;   // the stencil's reach in nodes
  constexpr unsigned kAll = 0xFFFFFFFFu;
  __shared__ SplitStage stage[kSplitWarps];
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

size_t split_start_ints() { return (size_t)kSplitKeys + 2; }

size_t split_work_bytes(int N) { return sizeof(int) * kCtrInts + 2 * sizeof(int4) * item_cap(N); }

int launch_pp_split(const ccs_uniforms *U, int N, int S, const float4 *pos, const float *mat, uint32_t *keys,
                    int32_t *vals, uint32_t *keysTmp, int32_t *valsTmp, uint32_t *hist, int *start, float4 *src,
                    float4 *srcT, int *cells, int *nCells, void *work, float4 *out, cudaStream_t st) {
  int launched = 0;
  int *ctr = static_cast<int *>(work);
  int4 *tmp = reinterpret_cast<int4 *>(ctr + kCtrInts), *items = tmp + item_cap(N);
  k_split_keys<<<blocks_for(N), kBlock, 0, st>>>(U, pos, keys, vals);
  launched += 1 + launch_radix_sort(N, 20, keys, vals, keysTmp, valsTmp, hist, st);
  k_split_starts<<<blocks_for(kSplitKeys + 2), kBlock, 0, st>>>(N, keys, start);
  cudaMemsetAsync(nCells, 0, sizeof(int), st);
  cudaMemsetAsync(ctr, 0, sizeof(int) * kCtrInts, st);
  k_split_sources<<<blocks_for(N), kBlock, 0, st>>>(U, keys, vals, pos, mat, src, srcT, cells, nCells);
  cudaMemsetAsync(out, 0, sizeof(float4) * N, st);   // particles in neither box get no pairs
  if (S == 1)
    k_split_items<1><<<blocks_for(N), kBlock, 0, st>>>(start, cells, nCells, srcT, ctr, tmp);
  else if (S == 2)
    k_split_items<2><<<blocks_for(N), kBlock, 0, st>>>(start, cells, nCells, srcT, ctr, tmp);
  else
    k_split_items<3><<<blocks_for(N), kBlock, 0, st>>>(start, cells, nCells, srcT, ctr, tmp);
  k_split_order<<<1, 32, 0, st>>>(ctr);
  k_split_scatter<<<blocks_for((long)item_cap(N)), kBlock, 0, st>>>(ctr, tmp, items);
  const int grid = sm_count() * 8;
  if (S == 1)
    k_pp_split<1><<<grid, 32 * kSplitWarps, 0, st>>>(U, start, src, srcT, vals, ctr, items, out);
  else if (S == 2)
    k_pp_split<2><<<grid, 32 * kSplitWarps, 0, st>>>(U, start, src, srcT, vals, ctr, items, out);
  else
    k_pp_split<3><<<grid, 32 * kSplitWarps, 0, st>>>(U, start, src, srcT, vals, ctr, items, out);
  return launched + 6;
}

// the kernels one split pair pass launches (the sort's count included)
int pp_split_launches() { return 7 + 3 * 3; }

}  // namespace ccs
