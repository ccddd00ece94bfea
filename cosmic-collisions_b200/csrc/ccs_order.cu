// ccs_order.cu -- relabelling and bookkeeping kernels: the permutation of
// applyPerm, the Morton order of the analysis computed on the device, the
// stable radix sort behind it, and the binary64 conservation books.
#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kBlock = 256;
inline int blocks_for(long n, int b = kBlock) { return (int)((n + b - 1) / b); }
}  // namespace

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
    const double v = floor(__dmul_rn(__ddiv_rn(__dadd_rn(__dsub_rn(pv[k], c[k]), 6.0), 12.0), 128.0));
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

namespace ccs {

// ---------------------------------------------------------------------------
// FP64 direct sum: the exact pull at chosen particles, for the force-error
// measurement and for the learned correction's training labels.  Targets are
// tiled 128 to a CTA and the sources split across gridDim.y chunks staged in
// shared memory; chunks add into the result with double atomics.  Newton is
// softened at eps (the P3M pass's own softening), the self term left out.
// ---------------------------------------------------------------------------
constexpr int kDsTile = 128;

__global__ void __launch_bounds__(kDsTile) k_direct_sum(int N, const float4 *__restrict__ pos,
                                                        const float *__restrict__ mat, double mref, double eps2,
                                                        const int32_t *__restrict__ idx, int nt, int chunk,
                                                        double *__restrict__ acc, double *__restrict__ pot) {
  __shared__ double sx[kDsTile], sy[kDsTile], sz[kDsTile], sm[kDsTile];
  const int t = blockIdx.x * kDsTile + threadIdx.x;
  const int i = t < nt ? idx[t] : -1;
  double xi = 0, yi = 0, zi = 0;
  if (i >= 0) {
    const float4 P = pos[i];
    xi = P.x; yi = P.y; zi = P.z;
  }
  const int j0 = blockIdx.y * chunk, j1 = min(j0 + chunk, N);
  double ax = 0, ay = 0, az = 0, ph = 0;
  for (int base = j0; base < j1; base += kDsTile) {
    __syncthreads();
    const int j = base + threadIdx.x;
    if (j < j1) {
      const float4 Q = pos[j];
      sx[threadIdx.x] = Q.x; sy[threadIdx.x] = Q.y; sz[threadIdx.x] = Q.z;
      sm[threadIdx.x] = mref * (double)mat[j];
    }
    __syncthreads();
    const int n = min(kDsTile, j1 - base);
    if (i < 0) continue;
    for (int k = 0; k < n; ++k) {
      if (base + k == i) continue;
      const double dx = sx[k] - xi, dy = sy[k] - yi, dz = sz[k] - zi;
      const double r2 = dx * dx + dy * dy + dz * dz + eps2;
      const double inv = 1.0 / sqrt(r2), w = sm[k] * inv * inv * inv;
      ax += dx * w; ay += dy * w; az += dz * w;
      ph -= sm[k] * inv;
    }
  }
  if (i >= 0) {
    atomicAdd(acc + 3 * t, ax);
    atomicAdd(acc + 3 * t + 1, ay);
    atomicAdd(acc + 3 * t + 2, az);
    atomicAdd(pot + t, ph);
  }
}

int launch_direct_sum(int N, const float4 *pos, const float *mat, double mref, double eps, const int32_t *idx,
                      int nt, double *acc, double *pot, cudaStream_t st) {
  const int chunks = 32;
  const int chunk = (N + chunks - 1) / chunks;
  cudaMemsetAsync(acc, 0, sizeof(double) * 3 * nt, st);
  cudaMemsetAsync(pot, 0, sizeof(double) * nt, st);
  dim3 g((nt + kDsTile - 1) / kDsTile, chunks);
  k_direct_sum<<<g, kDsTile, 0, st>>>(N, pos, mat, mref, eps * eps, idx, nt, chunk, acc, pot);
  return 1;
}

}  // namespace ccs
