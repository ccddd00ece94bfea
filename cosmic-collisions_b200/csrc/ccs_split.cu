// ccs_split.cu -- the stencil-split P3M: pairs of mesh nodes far apart are left to the mesh, everything
// nearer is summed particle by particle, exactly.
//
// The reference corrects only the loose list (src/nbody.js:851-870), and only against the mesh's
// placement-averaged pair table (src/glsl-sim.js:700-754), so a particle inside a body keeps the mesh's
// near field: a cell-centre sum softened by FH^2/2 at every distance (src/glsl-sim.js:303-352), a few per
// cent off Newton.  This form splits the interaction exactly instead.  A particle's cloud-in-cell weights
// w_i(k) over its 8 nodes and a source's w_j(l) over its 8 make a partition of unity over node pairs
// (k, l); the mesh keeps the pairs of nodes more than S cells apart in every axis' Chebyshev sense
// (k_cell_tide, unsoftened, with the tidal tensor so the gather is first order in the offset from each
// node's centre of mass), and this pass keeps the rest, each particle pair weighted by
//   W_ij = sum over (k, l) with |k - l|_inf <= S of w_i(k) w_j(l) = prod over axes of W_a(D_a, t_ia, t_ja),
// D_a = b_ja - b_ia the base nodes' offset: 1 for |D| <= S - 1, (1 - t_j) + t_i t_j for D = S,
// (1 - t_i) + t_i t_j for D = -S, t_i (1 - t_j) for D = S + 1, (1 - t_i) t_j for D = -S - 1, 0 beyond.
// Each pair is Newton softened at the particle radius a (the reference's own pairwise softening,
// src/glsl-sim.js:745).  Both particles must read the same box; a particle in neither gets the boxes'
// monopoles as before.
//
// Layout: particles are sorted (stable radix sort) by key = box * 64^3 + their base node's fine index,
// so a row of nodes (fixed y, z) is one contiguous range; start[key] is the first sorted position with a
// key >= key.  A CTA takes one occupied target node (its particles are the targets, up to 256 a round, two
// a thread) and walks the (2S + 3)^2 rows of source nodes around it, staging each row's sources in shared
// memory with their per-axis weight factors already reduced to W_a = P_a + Q_a t_ia (the offset D is the
// same for every target of the node), so a pair costs the three factors' FMAs, a product and the softened
// Newton term.  Sums run in a fixed order (rows, then sorted order): deterministic.
#include <algorithm>

#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kBlock = 256;
inline int blocks_for(long n, int b = kBlock) { return (int)((n + b - 1) / b); }
constexpr int kSplitThreads = 128;   // a CTA of the pair kernel; two targets a thread
constexpr int kSplitChunk = 256;     // sources staged at a time
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

template <int S>
__global__ void __launch_bounds__(kSplitThreads) k_pp_split(const ccs_uniforms *__restrict__ U,
                                                            const int *__restrict__ start,
                                                            const int *__restrict__ cells,
                                                            const int *__restrict__ nCells,
                                                            const float4 *__restrict__ src,
                                                            const float4 *__restrict__ srcT,
                                                            const int32_t *__restrict__ vals,
                                                            float4 *__restrict__ out) {
  constexpr int R = S + 1;   // the stencil's reach in nodes
  __shared__ float4 sP[kSplitChunk];   // x, y, z, m
  __shared__ float4 sW[kSplitChunk];   // P_x, Q_x, P_y, Q_y: W_a = P_a + Q_a t_ia
  __shared__ float2 sZ[kSplitChunk];   // P_z, Q_z
  const float a2 = U->a2, Gm = U->Gm;
  const float selfInv = rsqrtf(a2);   // a target meets itself with W = 1 and d = 0: only this potential
  const int n = *nCells;
  for (int ci = blockIdx.x; ci < n; ci += gridDim.x) {
    const int k0 = cells[ci];
    const int key = __float_as_int(srcT[k0].w);
    const int box = key / kFine, node = key - box * kFine;
    const int bx = node & 63, by = (node >> 6) & 63, bz = node >> 12;
    const int k1 = start[key + 1];
    for (int tb = k0; tb < k1; tb += 2 * kSplitThreads) {
      const int ta = tb + threadIdx.x, tc = ta + kSplitThreads;
      const bool va = ta < k1, vc = tc < k1;
      const float4 Pa = va ? src[ta] : make_float4(0, 0, 0, 0), Pc = vc ? src[tc] : make_float4(0, 0, 0, 0);
      const float4 Ta = va ? srcT[ta] : make_float4(0, 0, 0, 0), Tc = vc ? srcT[tc] : make_float4(0, 0, 0, 0);
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
          for (int c0 = s0; c0 < s1; c0 += kSplitChunk) {
            const int cn = min(kSplitChunk, s1 - c0);
            __syncthreads();   // the previous chunk's readers are done
            for (int j = threadIdx.x; j < cn; j += kSplitThreads) {
              const float4 P = src[c0 + j], T = srcT[c0 + j];
              const int D = (__float_as_int(T.w) & 63) - bx;
              const float4 cx4 = split_coef(D, S);
              sP[j] = P;
              sW[j] = make_float4(cx4.x + cx4.z * T.x, cx4.y + cx4.w * T.x, cy4.x + cy4.z * T.y,
                                  cy4.y + cy4.w * T.y);
              sZ[j] = make_float2(cz4.x + cz4.z * T.z, cz4.y + cz4.w * T.z);
            }
            __syncthreads();
#pragma unroll 4
            for (int j = 0; j < cn; ++j) {
              const float4 P = sP[j], Wc = sW[j];
              const float2 Wz = sZ[j];
              {
                const float w = (Wc.x + Wc.y * Ta.x) * (Wc.z + Wc.w * Ta.y) * (Wz.x + Wz.y * Ta.z) * P.w;
                const float dx = P.x - Pa.x, dy_ = P.y - Pa.y, dz_ = P.z - Pa.z;
                const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
                const float s = w * inv * inv * inv;
                ax = fmaf(dx, s, ax);
                ay = fmaf(dy_, s, ay);
                az = fmaf(dz_, s, az);
                pa = fmaf(-w, inv, pa);
              }
              {
                const float w = (Wc.x + Wc.y * Tc.x) * (Wc.z + Wc.w * Tc.y) * (Wz.x + Wz.y * Tc.z) * P.w;
                const float dx = P.x - Pc.x, dy_ = P.y - Pc.y, dz_ = P.z - Pc.z;
                const float inv = rsqrtf(fmaf(dz_, dz_, fmaf(dy_, dy_, fmaf(dx, dx, a2))));
                const float s = w * inv * inv * inv;
                cx = fmaf(dx, s, cx);
                cy = fmaf(dy_, s, cy);
                cz = fmaf(dz_, s, cz);
                pc = fmaf(-w, inv, pc);
              }
            }
          }
        }
      }
      if (va) out[vals[ta]] = make_float4(ax * Gm, ay * Gm, az * Gm, fmaf(Pa.w, selfInv, pa) * Gm);
      if (vc) out[vals[tc]] = make_float4(cx * Gm, cy * Gm, cz * Gm, fmaf(Pc.w, selfInv, pc) * Gm);
    }
  }
}

size_t split_start_ints() { return (size_t)kSplitKeys + 2; }

int launch_pp_split(const ccs_uniforms *U, int N, int S, const float4 *pos, const float *mat, uint32_t *keys,
                    int32_t *vals, uint32_t *keysTmp, int32_t *valsTmp, uint32_t *hist, int *start, float4 *src,
                    float4 *srcT, int *cells, int *nCells, float4 *out, cudaStream_t st) {
  int launched = 0;
  k_split_keys<<<blocks_for(N), kBlock, 0, st>>>(U, pos, keys, vals);
  launched += 1 + launch_radix_sort(N, 20, keys, vals, keysTmp, valsTmp, hist, st);
  k_split_starts<<<blocks_for(kSplitKeys + 2), kBlock, 0, st>>>(N, keys, start);
  cudaMemsetAsync(nCells, 0, sizeof(int), st);
  k_split_sources<<<blocks_for(N), kBlock, 0, st>>>(U, keys, vals, pos, mat, src, srcT, cells, nCells);
  cudaMemsetAsync(out, 0, sizeof(float4) * N, st);   // particles in neither box get no pairs
  const int grid = sm_count() * 16;
  if (S == 1)
    k_pp_split<1><<<grid, kSplitThreads, 0, st>>>(U, start, cells, nCells, src, srcT, vals, out);
  else if (S == 2)
    k_pp_split<2><<<grid, kSplitThreads, 0, st>>>(U, start, cells, nCells, src, srcT, vals, out);
  else
    k_pp_split<3><<<grid, kSplitThreads, 0, st>>>(U, start, cells, nCells, src, srcT, vals, out);
  return launched + 3;
}

// the kernels one split pair pass launches (the sort's count included)
int pp_split_launches() { return 4 + 3 * 3; }

}  // namespace ccs
