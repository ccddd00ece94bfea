// ccs_fof.cu -- the analysis of src/nbody.js:646-893 (fof) on the device.
//
// The reference runs it in a Web Worker on the state it reads back every 360
// steps; at 262k particles the host restatement (ccs_fof) takes about half a
// second, several times the steps between two analyses.  Here the same
// analysis runs where the state already is:
//   * groups: friends within 2.4 radii, found over an exact cell list (cells
//     of side 2.4 a hashed into 2^20 buckets exactly as the host does, sorted
//     by (bucket, index) with the library's stable radix sort), joined with a
//     lock-free union-find that hooks the larger root under the smaller, so a
//     group's label is its smallest index; the contacts' spring energy is
//     summed on the way;
//   * group sizes and the two largest (ties to the smaller label);
//   * every sum the report needs -- group moments, the body's centre walk,
//     the shell / hot / impactor statistics and the density histogram, the
//     spin, the orbit budget, the books -- as binary64 per-CTA partials in a
//     fixed order (deterministic; the host adds the partials in order);
//   * the loose list by an ordered compaction.
// The host assembles the report from the sums with the formulas of ccs_fof.
// Binary64 sums are added in a different order than the host's loops, so the
// report agrees with ccs_fof to rounding; the groups, the loose list and the
// Morton order are the same.
#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {
namespace fof {

constexpr int kBlock = 256;
constexpr uint32_t kUnionTries = 1u << 20;   // a union's retries before it gives up (status bit)

__device__ __forceinline__ int hash3(int x, int y, int z) {
  return ((int)((uint32_t)x * 73856093u) ^ (int)((uint32_t)y * 19349663u) ^ (int)((uint32_t)z * 83492791u)) &
         (kFofBuckets - 1);
}

// (x*x + y*y) + z*z rounded once per operation, never fused: the host's arithmetic
__device__ __forceinline__ double sq3(double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

__device__ __forceinline__ void cell3(const float4 P, double inv, int &x, int &y, int &z) {
  x = (int)floor((double)P.x * inv);
  y = (int)floor((double)P.y * inv);
  z = (int)floor((double)P.z * inv);
}

__global__ void k_keys(int N, const float4 *__restrict__ pos, double inv, uint32_t *__restrict__ keys,
                       int32_t *__restrict__ vals, int *__restrict__ parent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int x, y, z;
  cell3(pos[i], inv, x, y, z);
  keys[i] = (uint32_t)hash3(x, y, z);
  vals[i] = i;
  parent[i] = i;
}

// bucket ranges over the sorted keys; start was filled with -1 (an empty bucket)
__global__ void k_ranges(int N, const uint32_t *__restrict__ keys, int *__restrict__ start, int *__restrict__ end) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  const uint32_t k = keys[s];
  if (s == 0 || keys[s - 1] != k) start[k] = s;
  if (s == N - 1 || keys[s + 1] != k) end[k] = s + 1;
}

__device__ __forceinline__ int find(const int *parent, int x) {
  int p = __ldcg(parent + x);
  while (p != x) {   // parents only ever move to smaller indices: at most N steps
    x = p;
    p = __ldcg(parent + x);
  }
  return x;
}

__device__ __forceinline__ bool unite(int *parent, int a, int b) {
  for (uint32_t it = 0; it < kUnionTries; ++it) {
    a = find(parent, a);
    b = find(parent, b);
    if (a == b) return true;
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(parent + a, a, b) == a) return true;   // the larger root hooked under the smaller
  }
  return false;
}

// friends within L of each particle, over the 27 buckets around its cell; the spring energy of its touching pairs
__global__ void __launch_bounds__(kBlock) k_pairs(int N, const float4 *__restrict__ pos, double inv, double L2,
                                                  double touch, double spring, const int32_t *__restrict__ order,
                                                  const int *__restrict__ start, const int *__restrict__ end,
                                                  int *parent, double *__restrict__ elasticPart, unsigned *status) {
  __shared__ double red[kBlock / 32];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const double touch2 = touch * touch;
  double el = 0.0;
  bool ok = true;
  if (s < N) {
    const int i = order[s];
    const float4 Pi = pos[i];
    int cx, cy, cz;
    cell3(Pi, inv, cx, cy, cz);
    const double px = Pi.x, py = Pi.y, pz = Pi.z;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int k = hash3(cx + dx, cy + dy, cz + dz);
          const int b = start[k];
          if (b < 0) continue;
          const int e = end[k];
          for (int t = b; t < e; ++t) {
            const int j = order[t];
            if (j <= i) continue;
            const float4 Pj = pos[j];
            const double ex = (double)Pj.x - px, ey = (double)Pj.y - py, ez = (double)Pj.z - pz;
            const double e2 = sq3(ex, ey, ez);   // who is a friend is decided as the host decides it
            if (e2 >= L2) continue;
            ok = unite(parent, i, j) && ok;
            if (e2 < touch2) {
              const double ov = touch - sqrt(e2);
              el += 0.5 * spring * ov * ov;
            }
          }
        }
  }
  if (!ok) atomicOr(status, kStatusFof);
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) el += __shfl_xor_sync(0xFFFFFFFFu, el, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = el;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) t += red[w];
    elasticPart[blockIdx.x] = t;
  }
}

// label = the group's smallest index; sizes counted per label
__global__ void k_labels(int N, int *parent, int *__restrict__ size) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int r = find(parent, i);
  parent[i] = r;
  atomicAdd(size + r, 1);
}

// per CTA the two largest groups, as (size << 32 | ~label): the larger key wins, ties to the smaller label
__device__ __forceinline__ void top2_push(unsigned long long v, unsigned long long &a, unsigned long long &b) {
  if (v > a) {
    b = a;
    a = v;
  } else if (v > b && v != a) {
    b = v;
  }
}

__global__ void __launch_bounds__(kBlock) k_top2(int N, const int *__restrict__ parent, const int *__restrict__ size,
                                                 unsigned long long *__restrict__ out) {
  __shared__ unsigned long long ta[kBlock], tb[kBlock];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long a = 0, b = 0;
  if (i < N && parent[i] == i) a = ((unsigned long long)size[i] << 32) | (unsigned long long)(0xFFFFFFFFu - (uint32_t)i);
  ta[threadIdx.x] = a;
  tb[threadIdx.x] = b;
  __syncthreads();
  for (int o = kBlock / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      unsigned long long x = ta[threadIdx.x], y = tb[threadIdx.x];
      top2_push(ta[threadIdx.x + o], x, y);
      top2_push(tb[threadIdx.x + o], x, y);
      ta[threadIdx.x] = x;
      tb[threadIdx.x] = y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = ta[0];
    out[2 * blockIdx.x + 1] = tb[0];
  }
}

// ---------------------------------------------------------------------------
// the sums: one pass = up to kTerms binary64 terms per particle, each CTA's
// sum written to part[block * kTerms + term] in a fixed order
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool iron_tag(double w) { return w - 4.0 * floor(w / 4.0) < 0.5; }

__global__ void __launch_bounds__(kBlock) k_sums(FofSumArgs a, double *__restrict__ part) {
  __shared__ double red[kBlock / 32][kFofTerms];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double t[kFofTerms];
#pragma unroll
  for (int k = 0; k < kFofTerms; ++k) t[k] = 0.0;
  if (i < a.N) {
    const float4 P = a.pos[i], V = a.vel[i];
    const double m = a.mref * (double)a.mat[i];
    const double x = P.x, y = P.y, z = P.z, w = P.w, vx = V.x, vy = V.y, vz = V.z;
    const int lab = a.label[i];
    switch (a.pass) {
      case kFofGroup:
        if (lab == a.g) {
          t[0] = 1.0;
          t[1] = m;
          t[2] = m * x; t[3] = m * y; t[4] = m * z;
          t[5] = m * vx; t[6] = m * vy; t[7] = m * vz;
          if (w >= 3.5) { t[8] = m; t[9] = m * x; t[10] = m * y; t[11] = m * z; }
          if (iron_tag(w)) t[12] = m;
        }
        break;
      case kFofCore:
        if (lab == a.g) {
          const double qx = x - a.c[0], qy = y - a.c[1], qz = z - a.c[2];
          if (sq3(qx, qy, qz) < a.r2) { t[0] = m; t[1] = m * x; t[2] = m * y; t[3] = m * z; }
        }
        break;
      case kFofShape:
        if (lab == a.g) {
          const double sx = x - a.c[0], sy = y - a.c[1], sz = z - a.c[2];
          const double r2s = sq3(sx, sy, sz), Th = V.w;
          if (r2s > a.r2) { const double Tt = fmin(Th, 12000.0), wt = Tt * Tt; t[0] = wt * Tt; t[1] = wt; }
          if (Th > 1200.0) {
            double wh = fmin(Th, 12000.0);
            wh *= wh;
            t[3] = wh; t[4] = wh * x; t[5] = wh * y; t[6] = wh * z; t[7] = wh * r2s;
          }
          if (w >= 3.5) {
            const double ex = x - a.d[0], ey = y - a.d[1], ez = z - a.d[2];
            t[2] = m * (ex * ex + ey * ey + ez * ez);
          }
        }
        break;
      case kFofProper1:
      case kFofProper2:
      case kFofProper3: {
        const double d0 = x - a.c[0], d1 = y - a.c[1], d2 = z - a.c[2];
        if (lab == a.g && !(sq3(d0, d1, d2) > a.r2)) {
          if (a.pass == kFofProper1) {
            t[0] = m; t[1] = m * vx; t[2] = m * vy; t[3] = m * vz;
          } else if (a.pass == kFofProper2) {
            const double ux = vx - a.d[0], uy = vy - a.d[1], uz = vz - a.d[2];
            t[0] = m * (d1 * uz - d2 * uy);
            t[1] = m * (d2 * ux - d0 * uz);
            t[2] = m * (d0 * uy - d1 * ux);
          } else {
            const double along = d0 * a.d[0] + d1 * a.d[1] + d2 * a.d[2];
            t[0] = m * (d0 * d0 + d1 * d1 + d2 * d2 - along * along);
          }
        }
        break;
      }
      case kFofOrbit:
        if (lab != a.g) {
          // bound or not, decided with the host's roundings
          const double r = sqrt(sq3(x - a.c[0], y - a.c[1], z - a.c[2]));
          const double dv2 = sq3(vx - a.d[0], vy - a.d[1], vz - a.d[2]);
          if (__dsub_rn(__dmul_rn(0.5, dv2), a.s0 / fmax(r, a.s1)) < 0.0) {
            const double x0 = x - a.c[0], y0 = y - a.c[1], z0 = z - a.c[2];
            const double wx = vx - a.d[0], wy = vy - a.d[1], wz = vz - a.d[2];
            t[0] = m;
            t[2] = m * (y0 * wz - z0 * wy);
            t[3] = m * (z0 * wx - x0 * wz);
            t[4] = m * (x0 * wy - y0 * wx);
          } else {
            t[1] = m;
          }
        }
        break;
      case kFofBooks: {
        const float4 D = a.diag[i];
        t[0] = m;
        t[1] = m * vx; t[2] = m * vy; t[3] = m * vz;
        t[4] = m * (y * vz - z * vy);
        t[5] = m * (z * vx - x * vz);
        t[6] = m * (x * vy - y * vx);
        t[7] = 0.5 * m * (vx * vx + vy * vy + vz * vz);
        const double flag = D.y;
        const bool off = flag >= 2.0;
        t[8] = (off ? 1.0 : 0.5) * m * (double)D.x;
        t[9] = 0.5 * (double)D.w;
        if (iron_tag(w)) t[10] = m;
        if (flag - (off ? 2.0 : 0.0) < 0.5) t[11] = 1.0;
        if (D.z >= 7.5f) t[12] = 1.0;
        break;
      }
      default:
        break;
    }
  }
#pragma unroll
  for (int k = 0; k < kFofTerms; ++k) {
    double v = t[k];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kFofTerms) {
    double v = 0.0;
    for (int wd = 0; wd < kBlock / 32; ++wd) v += red[wd][threadIdx.x];
    part[(size_t)blockIdx.x * kFofTerms + threadIdx.x] = v;
  }
}

// the density histogram of a group: NBIN shells of width dr about its centre, per-CTA bins
__global__ void __launch_bounds__(kBlock) k_hist(FofSumArgs a, double dr, double *__restrict__ part) {
  __shared__ double bins[kFofBins];
  for (int k = threadIdx.x; k < kFofBins; k += blockDim.x) bins[k] = 0.0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.N && a.label[i] == a.g) {
    const float4 P = a.pos[i];
    const double sx = P.x - a.c[0], sy = P.y - a.c[1], sz = P.z - a.c[2];
    const double bi = sqrt(sq3(sx, sy, sz)) / dr;
    atomicAdd(bins + (bi < kFofBins - 1 ? (int)bi : kFofBins - 1), a.mref * (double)a.mat[i]);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kFofBins; k += blockDim.x) part[(size_t)blockIdx.x * kFofBins + k] = bins[k];
}

// ---------------------------------------------------------------------------
// the loose list: beyond 1.3 radii of the planet (and of a big second body)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double far2(const float4 P, const double *c) {
  const double ex = P.x - c[0], ey = P.y - c[1], ez = P.z - c[2];
  return sq3(ex, ey, ez);
}

__device__ __forceinline__ bool is_loose(const FofLooseArgs &a, const float4 P) {
  return far2(P, a.comA) > 1.69 * a.RA * a.RA && !(a.bigB && far2(P, a.comB) <= 1.69 * a.RB * a.RB);
}

// pass 0: per-CTA counts of the loose (and their distances, compacted in no order, for the cut);
// pass 1: per-CTA counts of the loose at least `least` away; pass 2: those in index order, the first `len`
__global__ void __launch_bounds__(kBlock) k_loose(FofLooseArgs a, int pass, const int *__restrict__ offs,
                                                  int *__restrict__ counts, double *__restrict__ dist,
                                                  int *__restrict__ nDist, int32_t *__restrict__ list) {
  __shared__ int warpN[kBlock / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  bool in = false;
  double d2 = 0.0;
  if (i < a.N) {
    const float4 P = a.pos[i];
    if (is_loose(a, P)) {
      d2 = far2(P, a.comA);
      in = pass == 0 || d2 >= a.least;   // least is 0 when every loose particle fits
    }
  }
  const unsigned bal = __ballot_sync(0xFFFFFFFFu, in);
  if (lane == 0) warpN[w] = __popc(bal);
  __syncthreads();
  if (pass < 2) {
    if (pass == 0 && in && dist) dist[atomicAdd(nDist, 1)] = d2;
    if (threadIdx.x == 0) {
      int n = 0;
      for (int k = 0; k < kBlock / 32; ++k) n += warpN[k];
      counts[blockIdx.x] = n;
    }
    return;
  }
  int before = offs[blockIdx.x];
  for (int k = 0; k < w; ++k) before += warpN[k];
  const int at = before + __popc(bal & ((1u << lane) - 1u));
  if (in && at < a.len) list[at] = i;
}

// exclusive scan of n <= 1024 * 64 counts by one CTA; offs[n] = the total
__global__ void __launch_bounds__(1024) k_scan(const int *__restrict__ counts, int n, int *__restrict__ offs) {
  __shared__ int warpSum[32];
  const int per = (n + 1023) / 1024;
  const int e0 = threadIdx.x * per, e1 = min(e0 + per, n);
  int s = 0;
  for (int e = e0; e < e1; ++e) s += counts[e];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = s;
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
  int run = x - s + (w > 0 ? warpSum[w - 1] : 0);
  for (int e = e0; e < e1; ++e) {
    offs[e] = run;
    run += counts[e];
  }
  if (threadIdx.x == 1023) offs[n] = run;
}

__global__ void k_remap(int n, const int32_t *__restrict__ into, int32_t *list) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) list[k] = into[list[k]];
}

inline int grid(long n) { return (int)((n + kBlock - 1) / kBlock); }

}  // namespace fof

int fof_blocks(int N) { return fof::grid(N); }

int launch_fof_groups(int N, const float4 *pos, double a, double touch, double spring, uint32_t *keys, int32_t *vals,
                      uint32_t *keysTmp, int32_t *valsTmp, uint32_t *hist, int *start, int *end, int *parent,
                      int *size, double *elasticPart, unsigned long long *top, unsigned *status, cudaStream_t st) {
  const double L = 2.4 * a, inv = 1.0 / L;
  const int g = fof::grid(N);
  int n = 0;
  fof::k_keys<<<g, fof::kBlock, 0, st>>>(N, pos, inv, keys, vals, parent);
  ++n;
  n += launch_radix_sort(N, 20, keys, vals, keysTmp, valsTmp, hist, st);
  cudaMemsetAsync(start, 0xFF, sizeof(int) * kFofBuckets, st);
  fof::k_ranges<<<g, fof::kBlock, 0, st>>>(N, keys, start, end);
  fof::k_pairs<<<g, fof::kBlock, 0, st>>>(N, pos, inv, L * L, touch, spring, vals, start, end, parent, elasticPart,
                                          status);
  cudaMemsetAsync(size, 0, sizeof(int) * N, st);
  fof::k_labels<<<g, fof::kBlock, 0, st>>>(N, parent, size);
  fof::k_top2<<<g, fof::kBlock, 0, st>>>(N, parent, size, top);
  return n + 4;
}

int launch_fof_sums(const FofSumArgs &a, double *part, cudaStream_t st) {
  fof::k_sums<<<fof::grid(a.N), fof::kBlock, 0, st>>>(a, part);
  return 1;
}

int launch_fof_hist(const FofSumArgs &a, double dr, double *part, cudaStream_t st) {
  fof::k_hist<<<fof::grid(a.N), fof::kBlock, 0, st>>>(a, dr, part);
  return 1;
}

int launch_fof_loose(const FofLooseArgs &a, int pass, int *counts, int *offs, double *dist, int *nDist,
                     int32_t *list, cudaStream_t st) {
  const int g = fof::grid(a.N);
  if (pass == 0) {
    fof::k_loose<<<g, fof::kBlock, 0, st>>>(a, 0, nullptr, counts, dist, nDist, nullptr);
    return 1;
  }
  fof::k_loose<<<g, fof::kBlock, 0, st>>>(a, 1, nullptr, counts, nullptr, nullptr, nullptr);
  fof::k_scan<<<1, 1024, 0, st>>>(counts, g, offs);
  fof::k_loose<<<g, fof::kBlock, 0, st>>>(a, 2, offs, counts, nullptr, nullptr, list);
  return 3;
}

int launch_fof_remap(int n, const int32_t *into, int32_t *list, cudaStream_t st) {
  if (n <= 0) return 0;
  fof::k_remap<<<fof::grid(n), fof::kBlock, 0, st>>>(n, into, list);
  return 1;
}

}  // namespace ccs
