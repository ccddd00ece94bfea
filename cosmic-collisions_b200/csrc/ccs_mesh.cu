// ccs_mesh.cu -- the 64^3 particle mesh of one box: cloud-in-cell deposit,
// coarse sums and the monopole, the block-to-block far field, and the gravity
// at every occupied fine cell (src/glsl-sim.js:158-352).
#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kBlock = 256;
inline int blocks_for(long n, int b = kBlock) { return (int)((n + b - 1) / b); }
}  // namespace

// ---------------------------------------------------------------------------
// deposit: src/glsl-sim.js:168-211 (DEP_VS) with src/nbody.js:402-416.
// Each particle's eight cloud-in-cell corners carry (w m x, w m); particles in
// the other box are left out; a stray (in neither) adds its pull toward last
// time's monopole into the scratch texel.  The lanes of a warp are grouped by
// base cell (Morton order keeps a warp's particles in one or a few): a group
// reduce-scatters its 32 values (8 corners x 4 components) over the warp with
// 31 shuffles and issues 32 scalar L2 atomics instead of 8 vector ones a lane;
// lone lanes, and lanes past the fourth group, add their own corners with
// float4 atomics.  The box a particle is in and its base cell are
// exact; the summation order is unspecified, as the reference's blending is.
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
      bx = (int)fx;
      by = (int)fy;
      bz = (int)fz;
    } else if (mine < 0) {
      stray = true;
      const float4 mono = *monoPrev;
      const f3 r = xyz(mono) * fdiv(1.0f, fmaxf(mono.w, 1e-6f)) - p;
      const float inv = rsqrtf(dot(r, r) + u.eps2Mesh);
      const f3 w = r * (mr * inv * inv * inv);
      sw = make_float4(w.x, w.y, w.z, mr);
    }
  }
  if (__any_sync(0xFFFFFFFFu, stray)) {   // the strays' reaction: one float4 atomic per warp
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
  // the warp's lanes grouped by base cell (Morton order keeps a warp's particles in a few): each group of
  // two or more reduce-scatters its 8 corners x 4 components over the warp (the others adding zeros) and
  // issues 32 scalar atomics; a lone lane, and what is left after kDepGroups groups, adds its own corners
  constexpr int kDepGroups = 4;
  unsigned todo = inMask, lone = 0u;
#pragma unroll 1
  for (int g = 0; g < kDepGroups && todo; ++g) {
    const int key0 = __shfl_sync(0xFFFFFFFFu, key, __ffs(todo) - 1);
    const bool member = in && key == key0;
    const unsigned gm = __ballot_sync(0xFFFFFFFFu, member);
    todo &= ~gm;
    if (__popc(gm) == 1) {   // a lone lane: its own atomics below
      lone |= gm;
      continue;
    }
    float v[32];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      const bool ok = member && bx + ox <= 63 && by + oy <= 63 && bz + oz <= 63;
      const float w = ok ? (ox ? t.x : 1.0f - t.x) * (oy ? t.y : 1.0f - t.y) * (oz ? t.z : 1.0f - t.z) * mr : 0.0f;
      v[4 * k + 0] = p.x * w;
      v[4 * k + 1] = p.y * w;
      v[4 * k + 2] = p.z * w;
      v[4 * k + 3] = w;
    }
    reduce_scatter32(v, lane);
    const int k = lane >> 2, comp = lane & 3;
    const int cx = (key0 & 0xFF) + (k & 1), cy = ((key0 >> 8) & 0xFF) + ((k >> 1) & 1), cz = (key0 >> 16) + (k >> 2);
    if (cx <= 63 && cy <= 63 && cz <= 63 && v[0] != 0.0f)
      atomicAdd(reinterpret_cast<float *>(fine + fine_index(cx, cy, cz)) + comp, v[0]);
  }
  if (((todo | lone) >> lane) & 1u) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      const int cx = bx + ox, cy = by + oy, cz = bz + oz;
      if (cx > 63 || cy > 63 || cz > 63) continue;
      const float w = (ox ? t.x : 1.0f - t.x) * (oy ? t.y : 1.0f - t.y) * (oz ? t.z : 1.0f - t.z) * mr;
      atomicAdd(fine + fine_index(cx, cy, cz), make_float4(p.x * w, p.y * w, p.z * w, w));
    }
  }
}

int launch_deposit(const ccs_uniforms *u, int N, int box, const float4 *pos, const float *mat, const float4 *monoPrev,
                   float4 *fine, cudaStream_t st) {
  k_deposit<<<blocks_for(N), kBlock, 0, st>>>(u, box, pos, mat, monoPrev, fine);
  return 1;
}

// ---------------------------------------------------------------------------
// the stencil-split P3M's node moments: each fine cell's second moment about its own centre of mass, from
// the particles' cloud-in-cell weights, Q = sum w m (x - X)(x - X)^T as two planes of kFine + 1 float4,
// (Qxx, Qyy, Qzz, Qxy) and (Qxz, Qyz).  With them the split form's mesh carries each node's quadrupole as a
// source, the reaction to the second-order gather's pull on the node's spread (without it that pull has
// no counterpart, and momentum drifts).  After the deposit (the centres of mass); the same grouping by
// base cell as the deposit, its 8 corners x 6 moments reduce-scattered over the warp in two rounds.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_node_moments(const ccs_uniforms *__restrict__ U, int box,
                                                         const float4 *__restrict__ pos,
                                                         const float *__restrict__ mat,
                                                         const float4 *__restrict__ fine, float4 *fineQ) {
  const ccs_uniforms &u = *U;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  bool in = false;
  int bx = 0, by = 0, bz = 0;
  f3 t = mk(0, 0, 0), p = mk(0, 0, 0);
  float mr = 0.0f;
  if (i < u.N) {
    p = xyz(pos[i]);
    mr = mat[i];
    f3 g;
    if (box_of(u, p, g) == box) {
      in = true;
      const float fx = floorf(g.x), fy = floorf(g.y), fz = floorf(g.z);
      t = mk(g.x - fx, g.y - fy, g.z - fz);
      bx = (int)fx;
      by = (int)fy;
      bz = (int)fz;
    }
  }
  const unsigned inMask = __ballot_sync(0xFFFFFFFFu, in);
  if (inMask == 0u) return;
  // corner k's moments of this particle (zero where the corner is past the mesh or the lane is out)
  auto corner = [&](int k, bool on, float (&m6)[6]) {
    const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
    const bool ok = on && bx + ox <= 63 && by + oy <= 63 && bz + oz <= 63;
    float w = 0.0f;
    f3 d = mk(0, 0, 0);
    if (ok) {
      w = (ox ? t.x : 1.0f - t.x) * (oy ? t.y : 1.0f - t.y) * (oz ? t.z : 1.0f - t.z) * mr;
      const float4 c = __ldg(fine + fine_index(bx + ox, by + oy, bz + oz));
      d = p - xyz(c) * fdiv(1.0f, c.w);
    }
    m6[0] = w * d.x * d.x; m6[1] = w * d.y * d.y; m6[2] = w * d.z * d.z;
    m6[3] = w * d.x * d.y; m6[4] = w * d.x * d.z; m6[5] = w * d.y * d.z;
  };
  const int key = in ? (bz << 16) | (by << 8) | bx : -1 - lane;
  constexpr int kGroups = 4;
  unsigned todo = inMask, lone = 0u;
#pragma unroll 1
  for (int gi = 0; gi < kGroups && todo; ++gi) {
    const int key0 = __shfl_sync(0xFFFFFFFFu, key, __ffs(todo) - 1);
    const bool member = in && key == key0;
    const unsigned gm = __ballot_sync(0xFFFFFFFFu, member);
    todo &= ~gm;
    if (__popc(gm) == 1) {
      lone |= gm;
      continue;
    }
#pragma unroll
    for (int half = 0; half < 2; ++half) {   // corners 4 half .. 4 half + 3, 8 slots a corner (6 used)
      float v[32];
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        float m6[6];
        corner(4 * half + kk, member, m6);
#pragma unroll
        for (int c = 0; c < 8; ++c) v[8 * kk + c] = c < 6 ? m6[c] : 0.0f;
      }
      reduce_scatter32(v, lane);
      const int k = 4 * half + (lane >> 3), comp = lane & 7;
      const int cx = (key0 & 0xFF) + (k & 1), cy = ((key0 >> 8) & 0xFF) + ((k >> 1) & 1), cz = (key0 >> 16) + (k >> 2);
      if (comp < 6 && cx <= 63 && cy <= 63 && cz <= 63 && v[0] != 0.0f)
        atomicAdd(reinterpret_cast<float *>(fineQ + (size_t)(comp >> 2) * (kFine + 1) + fine_index(cx, cy, cz)) +
                      (comp & 3),
                  v[0]);
    }
  }
  if (((todo | lone) >> lane) & 1u) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      const int cx = bx + ox, cy = by + oy, cz = bz + oz;
      if (cx > 63 || cy > 63 || cz > 63) continue;
      float m6[6];
      corner(k, true, m6);
      const int fi = fine_index(cx, cy, cz);
      atomicAdd(fineQ + fi, make_float4(m6[0], m6[1], m6[2], m6[3]));
      atomicAdd(reinterpret_cast<float *>(fineQ + kFine + 1 + fi) + 0, m6[4]);
      atomicAdd(reinterpret_cast<float *>(fineQ + kFine + 1 + fi) + 1, m6[5]);
    }
  }
}

int launch_node_moments(const ccs_uniforms *u, int N, int box, const float4 *pos, const float *mat,
                        const MeshBuf &m, cudaStream_t st) {
  cudaMemsetAsync(m.fineQ, 0, sizeof(float4) * 2 * (kFine + 1), st);
  k_node_moments<<<blocks_for(N), kBlock, 0, st>>>(u, box, pos, mat, m.fine, m.fineQ);
  return 1;
}

// ---------------------------------------------------------------------------
// coarse and monopole: src/glsl-sim.js:222-251.  One warp per coarse block:
// its lanes load the block's 4^3 fine cells together into shared memory, and
// lane 0 sums them in the reference's loop order (bit for bit).  The same warp
// writes the block's occupied fine cells, in that loop order, as (centre of
// mass, mass) plus their place in the block -- the source list the cell pass
// walks instead of all 64 cells of every neighbour block -- and appends an
// occupied block to the list the cell pass visits.  The monopole is a
// fixed-shape tree over the 4096 sums finished by the last CTA to arrive
// (deterministic, unlike the reference's single serial fragment).
// ---------------------------------------------------------------------------
constexpr int kCoarseWarps = 8;

__global__ void __launch_bounds__(32 * kCoarseWarps) k_coarse(const float4 *__restrict__ fine,
                                                              float4 *__restrict__ coarse, float4 *partial,
                                                              unsigned *counter, float4 *mono,
                                                              float4 *__restrict__ occ, uint8_t *__restrict__ occIdx,
                                                              int *__restrict__ occN, int *__restrict__ occBlocks,
                                                              int *__restrict__ occCount) {
  __shared__ float4 cells[kCoarseWarps][64];
  __shared__ float4 red[kCoarseWarps];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int b = blockIdx.x * kCoarseWarps + wid;
  const int cx = b & 15, cy = (b >> 4) & 15, cz = b >> 8;
  int n = 0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {   // cell c = (z * 4 + y) * 4 + x: the reference's loop order
    const int c = 32 * h + lane;
    const float4 f = fine[fine_index(cx * 4 + (c & 3), cy * 4 + ((c >> 2) & 3), cz * 4 + (c >> 4))];
    cells[wid][c] = f;
    const bool here = f.w > 0.0f;
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, here);
    if (here) {
      const int at = n + __popc(bal & ((1u << lane) - 1u));
      const float iw = fdiv(1.0f, f.w);
      occ[b * 64 + at] = make_float4(f.x * iw, f.y * iw, f.z * iw, f.w);
      occIdx[b * 64 + at] = (uint8_t)c;
    }
    n += __popc(bal);
  }
  __syncwarp();
  float4 s = make_float4(0, 0, 0, 0);
  if (lane == 0) {
    for (int c = 0; c < 64; ++c) {
      const float4 f = cells[wid][c];
      s.x = xadd(s.x, f.x);
      s.y = xadd(s.y, f.y);
      s.z = xadd(s.z, f.z);
      s.w = xadd(s.w, f.w);
    }
    occN[b] = n;
    if (n) occBlocks[atomicAdd(occCount, 1)] = b;   // the cell pass visits these only
    coarse[b] = s;
    red[wid] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float4 a = red[0];
    for (int w = 1; w < kCoarseWarps; ++w) {
      const float4 c = red[w];
      a.x += c.x; a.y += c.y; a.z += c.z; a.w += c.w;
    }
    partial[blockIdx.x] = a;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {   // the CTA partials in a fixed tree: each thread a fixed stride of them, then halving
    __shared__ float4 tree[32 * kCoarseWarps];
    __threadfence();
    float4 m = make_float4(0, 0, 0, 0);
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
      const float4 c = __ldcg(partial + k);
      m.x += c.x; m.y += c.y; m.z += c.z; m.w += c.w;
    }
    tree[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) {
        float4 a = tree[threadIdx.x];
        const float4 c = tree[threadIdx.x + o];
        a.x += c.x; a.y += c.y; a.z += c.z; a.w += c.w;
        tree[threadIdx.x] = a;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      *mono = tree[0];
      *counter = 0u;
    }
  }
}

int launch_coarse(const MeshBuf &m, cudaStream_t st) {
  k_coarse<<<kCoarse / kCoarseWarps, 32 * kCoarseWarps, 0, st>>>(m.fine, m.coarse, m.partial, m.counter, m.mono,
                                                                 m.occ, m.occIdx, m.occN, m.occBlocks, m.occCount);
  return 1;
}

// ---------------------------------------------------------------------------
// far field: src/glsl-sim.js:263-295.  The occupied blocks are listed once in
// ascending order (k_occ_list); a persistent grid of warps takes the occupied
// target blocks, and a warp's lanes split that list of sources (i, i + 32,
// ...) and reduce the ten sums.  Empty blocks' outputs are cleared before.
// Occupancy (mass > 0) and the "more than two away" test are exact.
// ---------------------------------------------------------------------------
constexpr int kFarWarps = 8;

__global__ void __launch_bounds__(1024) k_occ_list(const float4 *__restrict__ coarse, int *__restrict__ list,
                                                   int *__restrict__ count) {
  __shared__ int warpSum[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  bool occ[4];
  int n = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    occ[k] = __ldg(coarse + 4 * t + k).w > 0.0f;
    n += occ[k];
  }
  int x = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warpSum[w] = x;
  __syncthreads();
  if (w == 0) {
    int v = warpSum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, v, o);
      if (lane >= o) v += y;
    }
    warpSum[lane] = v;
  }
  __syncthreads();
  int at = x - n + (w > 0 ? warpSum[w - 1] : 0);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (occ[k]) list[at++] = 4 * t + k;
  if (t == 1023) *count = at;
}

__global__ void __launch_bounds__(32 * kFarWarps) k_far(const float4 *__restrict__ coarse,
                                                       const int *__restrict__ targets,
                                                       const int *__restrict__ nTargets,
                                                       const int *__restrict__ sources,
                                                       const int *__restrict__ nSources, float4 *__restrict__ farA,
                                                       float4 *__restrict__ farT0, float4 *__restrict__ farT1) {
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kFarWarps + (threadIdx.x >> 5), warps = gridDim.x * kFarWarps;
  const int nt = *nTargets, ns = *nSources;
  for (int ti = warp; ti < nt; ti += warps) {
    const int b = targets[ti];
    const float4 mc = __ldg(coarse + b);
    const int cx = b & 15, cy = (b >> 4) & 15, cz = b >> 8;
    const f3 x = xyz(mc) * fdiv(1.0f, mc.w);
    float s[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) s[k] = 0.0f;
    for (int i = lane; i < ns; i += 32) {
      const int k = __ldg(sources + i);
      const int kx = k & 15, ky = (k >> 4) & 15, kz = k >> 8;
      if (max(abs(kx - cx), max(abs(ky - cy), abs(kz - cz))) <= 2) continue;
      const float4 m = __ldg(coarse + k);
      const f3 r = xyz(m) * fdiv(1.0f, m.w) - x;
      const float inv = rsqrtf(dot(r, r)), inv2 = inv * inv, inv3 = inv * inv2, inv5 = inv3 * inv2;
      const float a3 = m.w * inv3, a5 = 3.0f * m.w * inv5;
      s[0] += r.x * a3; s[1] += r.y * a3; s[2] += r.z * a3;
      s[3] -= m.w * inv;
      s[4] += a5 * r.x * r.x - a3; s[5] += a5 * r.y * r.y - a3; s[6] += a5 * r.z * r.z - a3;
      s[7] += a5 * r.x * r.y; s[8] += a5 * r.x * r.z; s[9] += a5 * r.y * r.z;
    }
#pragma unroll
    for (int k = 0; k < 10; ++k)
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) s[k] += __shfl_xor_sync(0xFFFFFFFFu, s[k], o);
    if (lane == 0) {
      farA[b] = make_float4(s[0], s[1], s[2], s[3]);
      farT0[b] = make_float4(s[4], s[5], s[6], s[7]);
      farT1[b] = make_float4(s[8], s[9], 0.0f, 0.0f);
    }
  }
}

int launch_far(const MeshBuf &m, cudaStream_t st) {
  const int sms = sm_count();
  cudaMemsetAsync(m.farA, 0, sizeof(float4) * kCoarse, st);
  cudaMemsetAsync(m.farT0, 0, sizeof(float4) * kCoarse, st);
  cudaMemsetAsync(m.farT1, 0, sizeof(float4) * kCoarse, st);
  k_occ_list<<<1, 1024, 0, st>>>(m.coarse, m.occAsc, m.occAscN);
  k_far<<<2 * sms, 32 * kFarWarps, 0, st>>>(m.coarse, m.occBlocks, m.occCount, m.occAsc, m.occAscN, m.farA, m.farT0,
                                             m.farT1);
  return 2;
}

// ---------------------------------------------------------------------------
// cell gravity: src/glsl-sim.js:303-352.  Every occupied coarse block the
// coarse pass listed is split into kCellChunks work items, one CTA each: the
// item reads how many occupied cells each of the 5^3 blocks around its block
// holds (a warp scan gives where each one's cells start in the
// neighbourhood's list), takes its share of that list -- centre of mass and
// mass, as the coarse pass listed them, block by block in the reference's
// order -- into shared memory, and sums it onto each of the block's occupied
// cells with SPLIT threads a cell (every SPLIT-th source; 2, 4 or 8, the
// autotuner's choice).  The partial sums of a chunk are added in a fixed
// order and written out; the last of the block's CTAs to finish adds the
// chunks in chunk order, carries the block's far field to each cell by the
// tidal tensor and writes the force (the force mesh is cleared before, so
// empty cells read zero).  The result is deterministic for a given SPLIT.
// A block near the bodies sees about 1,500 occupied cells while only some 60
// blocks are occupied at all, so splitting a block's sources over CTAs is
// what keeps the SMs busy.  A cell skips itself.  Cell-on-cell pulls are fast
// arithmetic (rsqrt, FMA).
// ---------------------------------------------------------------------------
namespace {
constexpr int kCellBatch = 1024;

template <int SPLIT>
__global__ void __launch_bounds__(64 * SPLIT) k_cell(const ccs_uniforms *__restrict__ U,
                                                     const float4 *__restrict__ fine,
                                                     const float4 *__restrict__ coarse,
                                                     const float4 *__restrict__ occ,
                                                     const uint8_t *__restrict__ occIdx,
                                                     const int *__restrict__ occN,
                                                     const int *__restrict__ occBlocks,
                                                     const int *__restrict__ occCount,
                                                     const float4 *__restrict__ farA,
                                                     const float4 *__restrict__ farT0,
                                                     const float4 *__restrict__ farT1, float4 *__restrict__ force,
                                                     float4 *__restrict__ cellPart, int *__restrict__ cellDone) {
  constexpr int kCellThreads = 64 * SPLIT;
  __shared__ int nbK[128], nbOff[129];
  __shared__ float4 src[kCellBatch];
  __shared__ uint8_t sidx[kCellBatch];   // a source's place in its block; 255 for another block's cells
  __shared__ float4 part[SPLIT][64];
  __shared__ int last;
  const int t = threadIdx.x, cellT = t & 63, q = t >> 6, lane = t & 31;
  if (blockIdx.x == 0 && t == 0) force[kFine] = fine[kFine];   // the scratch texel, carried through
  const float eps2 = U->eps2Cell, Gm = U->Gm;
  const int items = *occCount * kCellChunks;
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const int bi = it / kCellChunks, chunk = it % kCellChunks;
    const int blk = occBlocks[bi];
    const int ccx = blk & 15, ccy = (blk >> 4) & 15, ccz = blk >> 8;
    if (t < 32) {   // the 125 neighbour blocks (o = kx + 5 ky + 25 kz: the reference's loop order), 4 a lane
      int n[4], run = 0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int o = lane * 4 + r;
        const int kx = ccx + o % 5 - 2, ky = ccy + (o / 5) % 5 - 2, kz = ccz + o / 25 - 2;
        const bool in = o < 125 && kx >= 0 && ky >= 0 && kz >= 0 && kx <= 15 && ky <= 15 && kz <= 15;
        const int k = in ? coarse_index(kx, ky, kz) : 0;
        nbK[o] = k;
        n[r] = in ? __ldg(occN + k) : 0;
        run += n[r];
      }
      int incl = run;   // where each lane's four start: an exclusive scan over the lanes
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += y;
      }
      int at = incl - run;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        nbOff[lane * 4 + r] = at;
        at += n[r];
      }
      if (lane == 31) nbOff[128] = at;
    }
    // the cellT-th occupied cell of the block, so the busy lanes sit together
    const int nOwn = __ldg(occN + blk);
    const bool mine = cellT < nOwn;
    const float4 tc = mine ? __ldg(occ + (size_t)blk * 64 + cellT) : make_float4(0, 0, 0, 0);
    const int tl = mine ? (int)__ldg(occIdx + (size_t)blk * 64 + cellT) : -1;
    const f3 x = xyz(tc);
    f3 acc = mk(0, 0, 0);
    float pot = 0.0f;
    __syncthreads();
    const int total = nbOff[125];
    const int c0 = (int)((long long)total * chunk / kCellChunks);
    const int c1 = (int)((long long)total * (chunk + 1) / kCellChunks);
    for (int b0 = c0; b0 < c1; b0 += kCellBatch) {
      const int b1 = min(b0 + kCellBatch, c1);
      // this chunk's sources in [b0, b1), a thread an entry: the neighbour block holding entry e is the
      // last o with nbOff[o] <= e (a binary search over the 126 starts); every load independent
      for (int e = b0 + t; e < b1; e += kCellThreads) {
        int lo = 0, hi = 125;   // nbOff[lo] <= e < nbOff[hi]
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (nbOff[mid] <= e) lo = mid;
          else hi = mid;
        }
        const int k = nbK[lo], i = e - nbOff[lo];
        src[e - b0] = __ldg(occ + (size_t)k * 64 + i);
        sidx[e - b0] = k == blk ? __ldg(occIdx + (size_t)k * 64 + i) : (uint8_t)255;
      }
      __syncthreads();
      if (mine) {
        const int n = b1 - b0;
#pragma unroll 4
        for (int i = q; i < n; i += SPLIT) {
          if ((int)sidx[i] == tl) continue;   // a cell does not pull itself
          const float4 mf = src[i];
          const f3 r = xyz(mf) - x;
          const float inv = rsqrtf(dot(r, r) + eps2);
          acc = acc + r * (mf.w * inv * inv * inv);
          pot -= mf.w * inv;
        }
      }
      __syncthreads();
    }
    part[q][cellT] = make_float4(acc.x, acc.y, acc.z, pot);
    __syncthreads();
    float4 *out = cellPart + ((size_t)bi * kCellChunks + chunk) * 64;
    if (mine && q == 0) {
#pragma unroll
      for (int k = 1; k < SPLIT; ++k) {
        const float4 p = part[k][cellT];
        acc = acc + mk(p.x, p.y, p.z);
        pot += p.w;
      }
      __stcg(out + cellT, make_float4(acc.x, acc.y, acc.z, pot));
    }
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(cellDone + bi, 1) == kCellChunks - 1;
    __syncthreads();
    if (last) {   // every chunk of this block is in: add them in chunk order, then the far field
      __threadfence();
      if (mine && q == 0) {
        const float4 *pb = cellPart + (size_t)bi * kCellChunks * 64;
        float4 s = __ldcg(pb + cellT);
#pragma unroll
        for (int c = 1; c < kCellChunks; ++c) {
          const float4 p = __ldcg(pb + (size_t)c * 64 + cellT);
          s.x += p.x;
          s.y += p.y;
          s.z += p.z;
          s.w += p.w;
        }
        f3 a3 = mk(s.x, s.y, s.z);
        float pt = s.w;
        const float4 mb = coarse[blk];
        const float4 fa = farA[blk], t0 = farT0[blk], t1 = farT1[blk];
        const f3 d = x - xyz(mb) * fdiv(1.0f, mb.w);
        const f3 Td = mk(t0.x * d.x + t0.w * d.y + t1.x * d.z, t0.w * d.x + t0.y * d.y + t1.y * d.z,
                         t1.x * d.x + t1.y * d.y + t0.z * d.z);
        a3 = a3 + (xyz(fa) + Td);
        pt += fa.w - dot(xyz(fa), d) - 0.5f * dot(d, Td);
        force[fine_index(ccx * 4 + (tl & 3), ccy * 4 + ((tl >> 2) & 3), ccz * 4 + (tl >> 4))] =
            make_float4(a3.x * Gm, a3.y * Gm, a3.z * Gm, pt * Gm);
      }
      if (t == 0) cellDone[bi] = 0;   // ready for the next pass
    }
    __syncthreads();   // the shared arrays are the next item's
  }
}
}  // namespace

// ---------------------------------------------------------------------------
// cell gravity of the stencil-split P3M (ccs_split.cu): the same work items, sources and chunk reduction as
// k_cell, but a source cell within S cells of the target cell in every axis (the stencil, itself included)
// is left to the pair pass, the rest is summed unsoftened (the pair pass takes everything near, so no
// softening is needed to keep the sum finite), and each cell also gets its tidal tensor -- the gradient of
// the pull, the near sources' exactly and the block's far field's as the block carries it -- so that the
// gather can carry each node's pull from its centre of mass to the particle, and the pull's second gradient
// for the second-order term.  Outputs (x Gm): force = (pull, potential) at the cell's centre of mass, tide0 =
// (Txx, Tyy, Tzz, Txy), tide1 = (Txz, Tyz), and tide2's three planes (Gxxx Gyyy Gzzz Gxyz), (Gxxy Gxxz Gxyy
// Gyyz), (Gxzz Gyzz), G_abc = d2 F_a / dx_b dx_c.
// The far field is k_far_cell's, added after: each far block's pull evaluated at the cell itself, with the
// block's quadrupole (the reference carries a block's monopole field from the block's centre of mass by its
// tidal tensor, which at a few blocks' distance is off by a per cent or two).
// ---------------------------------------------------------------------------
namespace {
// one source at r from the cell (r = source - cell, a5 = 3 M / r^5, a7 = 15 M / r^7): its second gradient
// of the pull, G_abc = a7 r_a r_b r_c - a5 (d_ab r_c + d_ac r_b + d_bc r_a), onto g0 = (Gxxx Gyyy Gzzz Gxyz),
// g1 = (Gxxy Gxxz Gxyy Gyyz), g2 = (Gxzz Gyzz)
__device__ __forceinline__ void add_tide2(float4 &g0, float4 &g1, float2 &g2, f3 r, float a5, float a7) {
  const float xx = r.x * r.x, yy = r.y * r.y, zz = r.z * r.z;
  g0.x += r.x * (a7 * xx - 3.0f * a5);
  g0.y += r.y * (a7 * yy - 3.0f * a5);
  g0.z += r.z * (a7 * zz - 3.0f * a5);
  g0.w += a7 * r.x * r.y * r.z;
  g1.x += r.y * (a7 * xx - a5);
  g1.y += r.z * (a7 * xx - a5);
  g1.z += r.x * (a7 * yy - a5);
  g1.w += r.z * (a7 * yy - a5);
  g2.x += r.x * (a7 * zz - a5);
  g2.y += r.y * (a7 * zz - a5);
}
__device__ __forceinline__ float4 add4(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

template <int SPLIT>
__global__ void __launch_bounds__(64 * SPLIT) k_cell_tide(const ccs_uniforms *__restrict__ U, int S,
                                                          const float4 *__restrict__ fine,
                                                          const float4 *__restrict__ coarse,
                                                          const float4 *__restrict__ occ,
                                                          const uint8_t *__restrict__ occIdx,
                                                          const int *__restrict__ occN,
                                                          const int *__restrict__ occBlocks,
                                                          const int *__restrict__ occCount,
                                                          const float4 *__restrict__ farA,
                                                          const float4 *__restrict__ farT0,
                                                          const float4 *__restrict__ farT1,
                                                          const float4 *__restrict__ fineQ,
                                                          float4 *__restrict__ force, float4 *__restrict__ tide0,
                                                          float4 *__restrict__ tide1, float4 *__restrict__ tide2,
                                                          float4 *__restrict__ cellPart, int *__restrict__ cellDone) {
  constexpr int kCellThreads = 64 * SPLIT;
  constexpr int kRows = 5;               // partial rows a cell: pull + potential, the tide (2), G (2 + 1 in row 2's zw)
  constexpr int kBatch = 512;
  __shared__ int nbK[128], nbOff[129];
  __shared__ float4 src[kBatch];
  __shared__ float4 sq0[kBatch];         // a source's second moment about its centre of mass: Qxx Qyy Qzz Qxy
  __shared__ float2 sq1[kBatch];         // Qxz Qyz
  __shared__ int sfc[kBatch];            // a source's fine cell, x | y << 6 | z << 12
  __shared__ float4 part[kRows][SPLIT][64];
  __shared__ int last;
  const int t = threadIdx.x, cellT = t & 63, q = t >> 6, lane = t & 31;
  if (blockIdx.x == 0 && t == 0) force[kFine] = fine[kFine];   // the scratch texel, carried through
  const float Gm = U->Gm, eps2 = 1e-6f * U->eps2Mesh;
  const int items = *occCount * kCellChunks;
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const int bi = it / kCellChunks, chunk = it % kCellChunks;
    const int blk = occBlocks[bi];
    const int ccx = blk & 15, ccy = (blk >> 4) & 15, ccz = blk >> 8;
    if (t < 32) {   // the 125 neighbour blocks and where each one's occupied cells start (as k_cell)
      int n[4], run = 0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int o = lane * 4 + r;
        const int kx = ccx + o % 5 - 2, ky = ccy + (o / 5) % 5 - 2, kz = ccz + o / 25 - 2;
        const bool in = o < 125 && kx >= 0 && ky >= 0 && kz >= 0 && kx <= 15 && ky <= 15 && kz <= 15;
        const int k = in ? coarse_index(kx, ky, kz) : 0;
        nbK[o] = k;
        n[r] = in ? __ldg(occN + k) : 0;
        run += n[r];
      }
      int incl = run;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += y;
      }
      int at = incl - run;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        nbOff[lane * 4 + r] = at;
        at += n[r];
      }
      if (lane == 31) nbOff[128] = at;
    }
    const int nOwn = __ldg(occN + blk);
    const bool mine = cellT < nOwn;
    const float4 tc = mine ? __ldg(occ + (size_t)blk * 64 + cellT) : make_float4(0, 0, 0, 0);
    const int tl = mine ? (int)__ldg(occIdx + (size_t)blk * 64 + cellT) : 0;
    const int tx = ccx * 4 + (tl & 3), ty = ccy * 4 + ((tl >> 2) & 3), tz = ccz * 4 + (tl >> 4);
    const f3 x = xyz(tc);
    f3 acc = mk(0, 0, 0);
    float pot = 0.0f, txx = 0.0f, tyy = 0.0f, tzz = 0.0f, txy = 0.0f, txz = 0.0f, tyz = 0.0f;
    float4 g0 = make_float4(0, 0, 0, 0), g1 = g0;
    float2 g2 = make_float2(0, 0);
    __syncthreads();
    const int total = nbOff[125];
    const int c0 = (int)((long long)total * chunk / kCellChunks);
    const int c1 = (int)((long long)total * (chunk + 1) / kCellChunks);
    for (int b0 = c0; b0 < c1; b0 += kBatch) {
      const int b1 = min(b0 + kBatch, c1);
      for (int e = b0 + t; e < b1; e += kCellThreads) {
        int lo = 0, hi = 125;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (nbOff[mid] <= e) lo = mid;
          else hi = mid;
        }
        const int k = nbK[lo], i = e - nbOff[lo];
        src[e - b0] = __ldg(occ + (size_t)k * 64 + i);
        const int ix = __ldg(occIdx + (size_t)k * 64 + i);
        const int fx = (k & 15) * 4 + (ix & 3), fy = (k >> 4 & 15) * 4 + ((ix >> 2) & 3), fz = (k >> 8) * 4 + (ix >> 4);
        sfc[e - b0] = fx | (fy << 6) | (fz << 12);
        const int fi = fine_index(fx, fy, fz);
        sq0[e - b0] = __ldg(fineQ + fi);
        const float4 q1 = __ldg(fineQ + kFine + 1 + fi);
        sq1[e - b0] = make_float2(q1.x, q1.y);
      }
      __syncthreads();
      if (mine) {
        const int n = b1 - b0;
#pragma unroll 2
        for (int i = q; i < n; i += SPLIT) {
          const int f = sfc[i];
          const int cheb = max(abs((f & 63) - tx), max(abs(((f >> 6) & 63) - ty), abs((f >> 12) - tz)));
          if (cheb <= S) continue;   // the pair pass's
          const float4 mf = src[i];
          const f3 r = xyz(mf) - x;
          // unsoftened beyond the stencil; eps2 (a thousandth of a cell, squared) only keeps two centres of mass
          // that happen to coincide finite
          const float inv = rsqrtf(dot(r, r) + eps2), inv2 = inv * inv, a3 = mf.w * inv * inv2, a5 = 3.0f * a3 * inv2;
          acc = acc + r * a3;
          pot -= mf.w * inv;
          txx += a5 * r.x * r.x - a3;
          tyy += a5 * r.y * r.y - a3;
          tzz += a5 * r.z * r.z - a3;
          txy += a5 * r.x * r.y;
          txz += a5 * r.x * r.z;
          tyz += a5 * r.y * r.z;
          add_tide2(g0, g1, g2, r, a5, 5.0f * a5 * inv2);
          // the source's spread about its centre of mass as a quadrupole (the reaction to the second-order
          // gather's pull on a node's spread): a = -3 Q r / r^5 + 7.5 (r Q r) r / r^7 - 1.5 tr(Q) r / r^5
          const float4 q0 = sq0[i];
          const float2 q1 = sq1[i];
          const f3 Qr = mk(q0.x * r.x + q0.w * r.y + q1.x * r.z, q0.w * r.x + q0.y * r.y + q1.y * r.z,
                           q1.x * r.x + q1.y * r.y + q0.z * r.z);
          const float rQr = dot(r, Qr), tr = q0.x + q0.y + q0.z, inv5 = inv2 * inv2 * inv;
          const float cq = 7.5f * rQr * inv5 * inv2 - 1.5f * tr * inv5;
          acc = acc + r * cq - Qr * (3.0f * inv5);
          pot -= 0.5f * (3.0f * rQr * inv5 - tr * inv2 * inv);
        }
      }
      __syncthreads();
    }
    part[0][q][cellT] = make_float4(acc.x, acc.y, acc.z, pot);
    part[1][q][cellT] = make_float4(txx, tyy, tzz, txy);
    part[2][q][cellT] = make_float4(txz, tyz, g2.x, g2.y);
    part[3][q][cellT] = g0;
    part[4][q][cellT] = g1;
    __syncthreads();
    float4 *out = cellPart + ((size_t)bi * kCellChunks + chunk) * 64 * kRows;
    if (mine && q == 0) {
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        float4 sr = part[r][0][cellT];
#pragma unroll
        for (int k = 1; k < SPLIT; ++k) sr = add4(sr, part[r][k][cellT]);
        __stcg(out + 64 * r + cellT, sr);
      }
    }
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(cellDone + bi, 1) == kCellChunks - 1;
    __syncthreads();
    if (last) {   // every chunk is in: add them in chunk order, then the block's far field and its tide
      __threadfence();
      if (mine && q == 0) {
        const float4 *pb = cellPart + (size_t)bi * kCellChunks * 64 * kRows;
        float4 s[kRows];
#pragma unroll
        for (int r = 0; r < kRows; ++r) s[r] = __ldcg(pb + 64 * r + cellT);
#pragma unroll 1
        for (int c = 1; c < kCellChunks; ++c) {
#pragma unroll
          for (int r = 0; r < kRows; ++r) s[r] = add4(s[r], __ldcg(pb + (size_t)c * 64 * kRows + 64 * r + cellT));
        }
        const int fi = fine_index(tx, ty, tz);
        force[fi] = make_float4(s[0].x * Gm, s[0].y * Gm, s[0].z * Gm, s[0].w * Gm);
        tide0[fi] = make_float4(s[1].x * Gm, s[1].y * Gm, s[1].z * Gm, s[1].w * Gm);
        tide1[fi] = make_float4(s[2].x * Gm, s[2].y * Gm, 0.0f, 0.0f);
        tide2[fi] = make_float4(s[3].x * Gm, s[3].y * Gm, s[3].z * Gm, s[3].w * Gm);
        tide2[kFine + 1 + fi] = make_float4(s[4].x * Gm, s[4].y * Gm, s[4].z * Gm, s[4].w * Gm);
        tide2[2 * (kFine + 1) + fi] = make_float4(s[2].z * Gm, s[2].w * Gm, 0.0f, 0.0f);
      }
      if (t == 0) cellDone[bi] = 0;
    }
    __syncthreads();
  }
}
}  // namespace

// each occupied block's second moment about its centre of mass, from its occupied cells' own moments and
// their centres of mass (parallel axes): Q = sum (m (x - X)(x - X)^T + Q_cell), q0 = (Qxx, Qyy, Qzz, Qxy), q1 =
// (Qxz, Qyz).  A warp a block, the lanes over its (up to 64) cells.
__global__ void __launch_bounds__(256) k_block_quad(const float4 *__restrict__ coarse,
                                                    const float4 *__restrict__ occ,
                                                    const uint8_t *__restrict__ occIdx,
                                                    const int *__restrict__ occN,
                                                    const int *__restrict__ occBlocks,
                                                    const int *__restrict__ occCount,
                                                    const float4 *__restrict__ fineQ, float4 *__restrict__ q0,
                                                    float4 *__restrict__ q1) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (w >= *occCount) return;
  const int b = occBlocks[w];
  const float4 mb = coarse[b];
  const f3 X = xyz(mb) * fdiv(1.0f, mb.w);
  float s[6] = {0, 0, 0, 0, 0, 0};
  const int n = occN[b];
  const int bx = b & 15, by = (b >> 4) & 15, bz = b >> 8;
  for (int c = lane; c < n; c += 32) {
    const float4 e = occ[(size_t)b * 64 + c];
    const f3 d = xyz(e) - X;
    const int ix = occIdx[(size_t)b * 64 + c];
    const int fi = fine_index(bx * 4 + (ix & 3), by * 4 + ((ix >> 2) & 3), bz * 4 + (ix >> 4));
    const float4 Q0 = fineQ[fi], Q1 = fineQ[kFine + 1 + fi];   // the cell's own spread, by parallel axes
    s[0] += e.w * d.x * d.x + Q0.x; s[1] += e.w * d.y * d.y + Q0.y; s[2] += e.w * d.z * d.z + Q0.z;
    s[3] += e.w * d.x * d.y + Q0.w; s[4] += e.w * d.x * d.z + Q1.x; s[5] += e.w * d.y * d.z + Q1.y;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s[k] += __shfl_xor_sync(0xFFFFFFFFu, s[k], o);
  if (lane == 0) {
    q0[b] = make_float4(s[0], s[1], s[2], s[3]);
    q1[b] = make_float4(s[4], s[5], 0.0f, 0.0f);
  }
}

// the far field of the stencil-split P3M: at every occupied cell's centre of mass, the pull, potential and
// tide of every occupied block more than two blocks from the cell's own (the blocks the near field leaves
// out), each block as its monopole at its centre of mass plus its quadrupole; added to the near field.
// A thread a cell: work items are (occupied block, its n-th occupied cell), the sources the ascending list
// of occupied blocks, staged in shared memory a batch at a time.
constexpr int kFarCellBatch = 256;
__global__ void __launch_bounds__(256) k_far_cell(const ccs_uniforms *__restrict__ U,
                                                  const float4 *__restrict__ coarse, const float4 *__restrict__ q0,
                                                  const float4 *__restrict__ q1, const float4 *__restrict__ occ,
                                                  const uint8_t *__restrict__ occIdx, const int *__restrict__ occN,
                                                  const int *__restrict__ occBlocks, const int *__restrict__ occCount,
                                                  const int *__restrict__ occAsc, const int *__restrict__ occAscN,
                                                  float4 *__restrict__ force, float4 *__restrict__ tide0,
                                                  float4 *__restrict__ tide1, float4 *__restrict__ tide2) {
  __shared__ float4 sM[kFarCellBatch], sQ0[kFarCellBatch];
  __shared__ float2 sQ1[kFarCellBatch];
  __shared__ int sB[kFarCellBatch];
  const float Gm = U->Gm;
  const int nb = *occCount, ns = *occAscN;
  const int items = nb * 64;
  // every CTA walks the same rounds of 256 items (a block's 64 cell slots, four blocks a round), so the
  // staging barriers are uniform; slots past a block's occupied cells idle
  for (int base = blockIdx.x * 256; base < items; base += gridDim.x * 256) {
    const int it = base + threadIdx.x;
    const int bi = it >> 6, c = it & 63;
    const bool live = it < items && c < occN[occBlocks[min(bi, nb - 1)]];
    int blk = 0, tl = 0;
    f3 x = mk(0, 0, 0);
    if (live) {
      blk = occBlocks[bi];
      const float4 e = occ[(size_t)blk * 64 + c];
      x = xyz(e);
      tl = occIdx[(size_t)blk * 64 + c];
    }
    const int bx = blk & 15, by = (blk >> 4) & 15, bz = blk >> 8;
    float ax = 0, ay = 0, az = 0, pot = 0, txx = 0, tyy = 0, tzz = 0, txy = 0, txz = 0, tyz = 0;
    float4 g0 = make_float4(0, 0, 0, 0), g1 = g0;
    float2 g2 = make_float2(0, 0);
    for (int s0 = 0; s0 < ns; s0 += kFarCellBatch) {
      const int sn = min(kFarCellBatch, ns - s0);
      __syncthreads();
      for (int j = threadIdx.x; j < sn; j += blockDim.x) {
        const int k = occAsc[s0 + j];
        const float4 m = coarse[k];
        const float iw = fdiv(1.0f, m.w);
        sM[j] = make_float4(m.x * iw, m.y * iw, m.z * iw, m.w);
        sQ0[j] = q0[k];
        const float4 t = q1[k];
        sQ1[j] = make_float2(t.x, t.y);
        sB[j] = k;
      }
      __syncthreads();
      if (live) {
        for (int j = 0; j < sn; ++j) {
          const int k = sB[j];
          if (max(abs((k & 15) - bx), max(abs(((k >> 4) & 15) - by), abs((k >> 8) - bz))) <= 2) continue;
          const float4 m = sM[j], Q0 = sQ0[j];
          const float2 Q1 = sQ1[j];
          const f3 r = xyz(m) - x;   // from the cell to the block
          const float r2 = dot(r, r), inv = rsqrtf(r2), inv2 = inv * inv, inv3 = inv * inv2, inv5 = inv3 * inv2;
          const float a3 = m.w * inv3, a5 = 3.0f * a3 * inv2;
          // monopole: pull, potential, tide
          ax += r.x * a3; ay += r.y * a3; az += r.z * a3;
          pot -= m.w * inv;
          txx += a5 * r.x * r.x - a3; tyy += a5 * r.y * r.y - a3; tzz += a5 * r.z * r.z - a3;
          txy += a5 * r.x * r.y; txz += a5 * r.x * r.z; tyz += a5 * r.y * r.z;
          add_tide2(g0, g1, g2, r, a5, 5.0f * a5 * inv2);   // the monopole's second gradient
          // quadrupole: a = -3 Q r / r^5 + 7.5 (r Q r) r / r^7 - 1.5 tr(Q) r / r^5,
          // potential -0.5 (3 r Q r / r^5 - tr(Q) / r^3)
          const f3 Qr = mk(Q0.x * r.x + Q0.w * r.y + Q1.x * r.z, Q0.w * r.x + Q0.y * r.y + Q1.y * r.z,
                           Q1.x * r.x + Q1.y * r.y + Q0.z * r.z);
          const float rQr = dot(r, Qr), tr = Q0.x + Q0.y + Q0.z;
          const float c1 = 7.5f * rQr * inv5 * inv2 - 1.5f * tr * inv5;
          ax += c1 * r.x - 3.0f * inv5 * Qr.x;
          ay += c1 * r.y - 3.0f * inv5 * Qr.y;
          az += c1 * r.z - 3.0f * inv5 * Qr.z;
          pot -= 0.5f * (3.0f * rQr * inv5 - tr * inv3);
        }
      }
    }
    if (live) {
      const int fi = fine_index((blk & 15) * 4 + (tl & 3), ((blk >> 4) & 15) * 4 + ((tl >> 2) & 3),
                                (blk >> 8) * 4 + (tl >> 4));
      const float4 f = force[fi], t0 = tide0[fi], t1 = tide1[fi];
      force[fi] = make_float4(f.x + ax * Gm, f.y + ay * Gm, f.z + az * Gm, f.w + pot * Gm);
      tide0[fi] = make_float4(t0.x + txx * Gm, t0.y + tyy * Gm, t0.z + tzz * Gm, t0.w + txy * Gm);
      tide1[fi] = make_float4(t1.x + txz * Gm, t1.y + tyz * Gm, 0.0f, 0.0f);
      float4 *G0 = tide2 + fi, *G1 = tide2 + kFine + 1 + fi, *G2 = tide2 + 2 * (kFine + 1) + fi;
      const float4 h0 = *G0, h1 = *G1, h2 = *G2;
      *G0 = make_float4(h0.x + g0.x * Gm, h0.y + g0.y * Gm, h0.z + g0.z * Gm, h0.w + g0.w * Gm);
      *G1 = make_float4(h1.x + g1.x * Gm, h1.y + g1.y * Gm, h1.z + g1.z * Gm, h1.w + g1.w * Gm);
      *G2 = make_float4(h2.x + g2.x * Gm, h2.y + g2.y * Gm, 0.0f, 0.0f);
    }
  }
}

int launch_cell_tide(const ccs_uniforms *u, int S, const MeshBuf &m, cudaStream_t st) {
  const int sms = sm_count();
  cudaMemsetAsync(m.force, 0, sizeof(float4) * kFine, st);
  k_cell_tide<4><<<sms * 8, 256, 0, st>>>(u, S, m.fine, m.coarse, m.occ, m.occIdx, m.occN, m.occBlocks, m.occCount,
                                          m.farA, m.farT0, m.farT1, m.fineQ, m.force, m.tide0, m.tide1, m.tide2,
                                          m.cellPartT, m.cellDone);
  k_block_quad<<<kCoarse / 8, 256, 0, st>>>(m.coarse, m.occ, m.occIdx, m.occN, m.occBlocks, m.occCount, m.fineQ,
                                            m.quad0, m.quad1);
  k_far_cell<<<sms * 4, 256, 0, st>>>(u, m.coarse, m.quad0, m.quad1, m.occ, m.occIdx, m.occN, m.occBlocks,
                                      m.occCount, m.occAsc, m.occAscN, m.force, m.tide0, m.tide1, m.tide2);
  return 3;
}

int launch_cell(const ccs_uniforms *u, const MeshBuf &m, cudaStream_t st, int split) {
  const int sms = sm_count();
  // a persistent grid over (block, chunk) items: four CTAs of 512 threads fill an SM, more of smaller ones
  const int grid = sms * (split == 2 ? 16 : split == 4 ? 8 : 4);
  cudaMemsetAsync(m.force, 0, sizeof(float4) * kFine, st);
  if (split == 2)
    k_cell<2><<<grid, 128, 0, st>>>(u, m.fine, m.coarse, m.occ, m.occIdx, m.occN, m.occBlocks, m.occCount, m.farA,
                                    m.farT0, m.farT1, m.force, m.cellPart, m.cellDone);
  else if (split == 8)
    k_cell<8><<<grid, 512, 0, st>>>(u, m.fine, m.coarse, m.occ, m.occIdx, m.occN, m.occBlocks, m.occCount, m.farA,
                                    m.farT0, m.farT1, m.force, m.cellPart, m.cellDone);
  else
    k_cell<4><<<grid, 256, 0, st>>>(u, m.fine, m.coarse, m.occ, m.occIdx, m.occN, m.occBlocks, m.occCount, m.farA,
                                    m.farT0, m.farT1, m.force, m.cellPart, m.cellDone);
  return 1;
}

}  // namespace ccs
