// ccs_nn.cu -- the learned form of the P3M pairwise correction.
//
// The reference subtracts, for every loose pair inside the cut, the mesh's own
// force between two particles as a function of distance alone: the placement-
// averaged table of src/nbody.js:48-109 (meshPairTable).  Where the two
// particles share no cloud-in-cell node (certainly once they are two cells
// apart along an axis) the mesh's pair force is the node-to-node Newton force
// with CELL_FS's 0.5 FH^2 softening, exactly; where they share nodes (possible
// out to 2 sqrt(3) cells) it depends on the direction against the grid axes
// and on where the particles sit in their cells, and the table keeps only its
// average.  A small network learns that part:
//
//   R(d, s) = M(d, s) - d / (|d|^2 + 1/2)^(3/2) ~ MLP(d, s - 1/2),
//   6 -> 64 -> 64 -> 3, SiLU, BF16 weights, FP32 accumulation,
//
// d the pair offset in mesh cells (source - target), s the source's fractional
// position in its cell, M the mesh's force on the target from a unit source
// (cells^-2).  The learned pass corrects a loose pair inside half the plain
// cut by m_j (N_a(d) - d/(r^2 + FH^2/2)^(3/2) - R(d, s)/FH^2) taper; the
// potential keeps the table's.
//
// Labels are the mesh arithmetic of meshPairTable's field() for the isolated
// pair -- cloud-in-cell deposit, node centres of mass, node-to-node Newton
// with 0.5 FH^2 softening and the own node left out, cloud-in-cell gather --
// in binary64 on the device (k_nn_label), less the softened Newton force.
// Training pairs are drawn from a running impact's particles
// (k_nn_sample_state).
//
// The three layers run on the 5th-generation tensor cores: 128 pairs per
// tile are the MMA's M, operands are staged in shared memory in the
// no-swizzle K-major layout, accumulators live in tensor memory.  Training
// runs forward, backward and the weight gradients on the tensor cores too:
// the weight gradients are MMAs over the tile's 128 rows with the activations
// stored transposed, two layers stacked into one M = 128 operand, and a row
// of ones that turns the same MMA into the bias gradients.
//
// The input goes in as a high and a low BF16 part (both multiplied by the
// same BF16 weights), so the offset keeps about 16 bits through layer 1.
#include <algorithm>

#include "ccs_device.cuh"
#include "ccs_internal.h"
#include "ccs_umma.cuh"

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

namespace ccs {
namespace nn {

using namespace umma;

constexpr int kIn = 6, kH = 64, kOut = 3;
constexpr int kRows = 128;                    // pairs per tile (the MMA's M)
constexpr int kOnes = 12;                     // input column that is 1 on live rows (bias gradient of layer 1)
// flat parameter order: W1[64][6] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH, kParams = oB3 + kOut;
static_assert(kParams == CCS_NN_PARAMS, "parameter count");
constexpr int kStride = 4808;                 // per-CTA partials: the gradient, then the squared error
// the operand image: BF16 halves, each matrix in the canonical layout, then the FP32 biases
constexpr int iW1 = 0, iW2 = iW1 + 64 * 16, iW2T = iW2 + 64 * 64, iW3 = iW2T + 64 * 64, iW3T = iW3 + 16 * 64,
              kImgHalves = iW3T + 64 * 16;
constexpr int kImgBytes = kImgHalves * 2;     // 22528
constexpr int bB1 = kImgBytes, bB2 = bB1 + 256, bB3 = bB2 + 256, kImgTotal = bB3 + 16;   // 23056
static_assert(kImgTotal % 16 == 0, "image copies in 16-byte pieces");

// training kernel's shared memory (bytes)
constexpr int tX = 0, tA1 = 4096, tA2 = 20480, tDY = 36864, tDH2 = 40960, tW = 57344, tGA = tW + kImgBytes,
              tGB = tGA + 32768, tGA2 = tGB + 36864, tXT = tGA2 + 32768, tBias = tXT + 4096,
              tMisc = tBias + (kImgTotal - kImgBytes), kTrainSmem = tMisc + 64;
static_assert(tGA == 79872 && tMisc % 16 == 0, "layout");
// forward kernel's shared memory; padded so that at most 3 CTAs (3 x 128 TMEM columns) share an SM
constexpr int fX = 0, fA1 = 4096, fA2 = 20480, fW = 36864, fBias = fW + kImgBytes,
              fMisc = fBias + (kImgTotal - kImgBytes), kFwdSmem = 65536;
static_assert(fMisc + 64 <= kFwdSmem, "layout");

constexpr uint32_t kWaitLimit = 1u << 22;     // polls of an mbarrier before a kernel gives up

__device__ __forceinline__ float silu(float h) { return __fdividef(h, 1.0f + __expf(-h)); }
__device__ __forceinline__ float silu_grad(float h) {
  const float s = __fdividef(1.0f, 1.0f + __expf(-h));
  return s * (1.0f + h * (1.0f - s));
}

// a row of 16 input columns: the high and low BF16 parts of the 6 features, the ones column, zeros
__device__ __forceinline__ void input_row(const float (&x)[kIn], bool live, uint16_t (&b)[16]) {
#pragma unroll
  for (int f = 0; f < kIn; ++f) {
    const uint16_t hi = bf16_bits(x[f]);
    b[f] = hi;
    b[kIn + f] = bf16_bits(x[f] - bf16_value(hi));
  }
  b[kOnes] = live ? (uint16_t)0x3F80 : (uint16_t)0;   // 1.0
  b[13] = b[14] = b[15] = 0;
}

// one K-major row of n BF16 values (n a multiple of 8) into a canonical operand with K = n
template <int n>
__device__ __forceinline__ void store_row(uint8_t *base, int r, const uint16_t (&v)[n]) {
#pragma unroll
  for (int c = 0; c < n / 8; ++c) {
    uint4 w;
    w.x = pack2(v[8 * c + 0], v[8 * c + 1]);
    w.y = pack2(v[8 * c + 2], v[8 * c + 3]);
    w.z = pack2(v[8 * c + 4], v[8 * c + 5]);
    w.w = pack2(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4 *>(base + canon(r, 8 * c, n)) = w;
  }
}

// rows r0.. of a K = 128 operand at column `col` (the transposed store of a tile row)
template <int n>
__device__ __forceinline__ void store_col(uint8_t *base, int r0, int col, const uint16_t (&v)[n]) {
#pragma unroll
  for (int k = 0; k < n; ++k) *reinterpret_cast<uint16_t *>(base + canon(r0 + k, col, 128)) = v[k];
}

// ---------------------------------------------------------------------------
// labels: meshPairTable's field() (src/nbody.js:60-91) for the isolated pair,
// binary64.  Coordinates are in mesh cells with the deposit's half-cell shift
// (g of GLSL_BOX), so corners are floor(g) + {0,1}; only differences of node
// centres enter, so a record (d, s) places the source at s and the target at
// s - d.  The target alone feels no force (all its nodes sit at its own
// position), so the pair's field is the mesh force M.
// ---------------------------------------------------------------------------
__device__ void pair_field(double px, double py, double pz, double qx, double qy, double qz, double out[3]) {
  int kx[16], ky[16], kz[16];
  double m[16], cx[16], cy[16], cz[16], pw[8];
  int nn = 0;
  const double P[2][3] = {{px, py, pz}, {qx, qy, qz}};
  for (int part = 0; part < 2; ++part) {
    const double *p = P[part];
    const double fx = floor(p[0]), fy = floor(p[1]), fz = floor(p[2]);
    const double t0 = p[0] - fx, t1 = p[1] - fy, t2 = p[2] - fz;
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      const int ax = (int)fx + ox, ay = (int)fy + oy, az = (int)fz + oz;
      const double w = ((ox ? t0 : 1.0 - t0) * (oy ? t1 : 1.0 - t1)) * (oz ? t2 : 1.0 - t2);
      if (part == 0) pw[k] = w;
      int n = -1;
      for (int j = 0; j < nn; ++j)
        if (kx[j] == ax && ky[j] == ay && kz[j] == az) { n = j; break; }
      if (n < 0) {
        n = nn++;
        kx[n] = ax; ky[n] = ay; kz[n] = az;
        m[n] = 0.0; cx[n] = 0.0; cy[n] = 0.0; cz[n] = 0.0;
      }
      m[n] += w;
      cx[n] += w * p[0];
      cy[n] += w * p[1];
      cz[n] += w * p[2];
    }
  }
  for (int j = 0; j < nn; ++j) {   // a node of zero weight (a particle exactly on a cell face) carries nothing
    if (m[j] > 0.0) {
      cx[j] /= m[j];
      cy[j] /= m[j];
      cz[j] /= m[j];
    }
  }
  out[0] = out[1] = out[2] = 0.0;
  for (int k = 0; k < 8; ++k) {   // the target's nodes are the first eight
    if (!(m[k] > 0.0)) continue;
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    for (int o = 0; o < nn; ++o) {
      if (o == k || !(m[o] > 0.0)) continue;
      const double rx = cx[o] - cx[k], ry = cy[o] - cy[k], rz = cz[o] - cz[k];
      const double inv = 1.0 / sqrt(((rx * rx + ry * ry) + rz * rz) + 0.5);
      const double inv3 = (inv * inv) * inv;
      f0 += (rx * m[o]) * inv3;
      f1 += (ry * m[o]) * inv3;
      f2 += (rz * m[o]) * inv3;
    }
    out[0] += pw[k] * f0;
    out[1] += pw[k] * f1;
    out[2] += pw[k] * f2;
  }
}

// the network's target: the isolated pair's mesh force less the node-softened Newton force
// d / (r^2 + 1/2)^(3/2) (cells, the 0.5 FH^2 softening of CELL_FS), which it equals when the two
// particles share no node
__global__ void k_nn_label(const float4 *__restrict__ D, const float4 *__restrict__ S, long n,
                           float4 *__restrict__ L) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float4 d = D[k], s = S[k];
  if (d.w == 0.0f) {
    L[k] = make_float4(0, 0, 0, 0);
    return;
  }
  const double qx = s.x, qy = s.y, qz = s.z, dx = d.x, dy = d.y, dz = d.z;
  double o[3];
  pair_field(qx - dx, qy - dy, qz - dz, qx, qy, qz, o);
  const double q = 1.0 / sqrt((dx * dx + dy * dy + dz * dz) + 0.5), b = q * q * q;
  L[k] = make_float4((float)(o[0] - dx * b), (float)(o[1] - dy * b), (float)(o[2] - dz * b), 0.0f);
}

// ---------------------------------------------------------------------------
// training pairs
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mix32(uint32_t x) {   // integer finaliser ("lowbias32")
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ float unit(uint32_t &st) {   // uniform in (0, 1): never a cell face
  st = mix32(st + 0x9E3779B9u);
  return ((float)(st >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// pairs of a running impact's particles inside the cut, both in box 0: half drawn
// uniformly over the body, half among Morton neighbours (index within +-128),
// which covers the close pairs.  A record that finds no pair in 256 draws is
// written dead (w = 0) and is masked out of training.
__global__ void k_nn_sample_state(const ccs_uniforms *__restrict__ U, const float4 *__restrict__ pos, int N,
                                  long count, uint32_t seed, float cutG, float4 *__restrict__ D,
                                  float4 *__restrict__ S) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const ccs_uniforms &u = *U;
  uint32_t st = mix32(seed ^ mix32((uint32_t)k * 0x85EBCA6Bu + 0x27D4EB2Fu));
  const float cut2 = cutG * cutG;
  for (int attempt = 0; attempt < 256; ++attempt) {
    st = mix32(st + 0x632BE5ABu);
    const int j = (int)(st % (uint32_t)N);
    st = mix32(st + 0x85157AF5u);
    const int i = (k & 1) ? j + (int)(st % 257u) - 128 : (int)(st % (uint32_t)N);
    if (i < 0 || i >= N || i == j) continue;
    f3 gj, gi;
    if (box_of(u, xyz(pos[j]), gj) != 0 || box_of(u, xyz(pos[i]), gi) != 0) continue;
    const f3 d = gj - gi;
    const float r2 = dot(d, d);
    if (!(r2 < cut2) || r2 == 0.0f) continue;
    D[k] = make_float4(d.x, d.y, d.z, 1.0f);
    S[k] = make_float4(gj.x - floorf(gj.x), gj.y - floorf(gj.y), gj.z - floorf(gj.z), 0.0f);
    return;
  }
  D[k] = make_float4(0, 0, 0, 0);
  S[k] = make_float4(0, 0, 0, 0);
}

// synthetic pairs: the source uniform in its cell; the offset uniform in the ball
// (even records) or uniform in distance with a uniform direction (odd records)
__global__ void k_nn_sample_uniform(long count, uint32_t seed, float cutG, float4 *__restrict__ D,
                                    float4 *__restrict__ S) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  uint32_t st = mix32(seed ^ mix32((uint32_t)k * 0xC2B2AE35u + 0x165667B1u));
  const float sx = unit(st), sy = unit(st), sz = unit(st);
  float dx, dy, dz;
  if (k & 1) {
    const float r = cutG * fmaxf(unit(st), 1e-4f);
    const float z = 2.0f * unit(st) - 1.0f, ph = 6.2831853f * unit(st), rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    dx = r * rr * cosf(ph);
    dy = r * rr * sinf(ph);
    dz = r * z;
  } else {
    do {
      dx = (2.0f * unit(st) - 1.0f) * cutG;
      dy = (2.0f * unit(st) - 1.0f) * cutG;
      dz = (2.0f * unit(st) - 1.0f) * cutG;
    } while (dx * dx + dy * dy + dz * dz >= cutG * cutG || dx * dx + dy * dy + dz * dz == 0.0f);
  }
  D[k] = make_float4(dx, dy, dz, 1.0f);
  S[k] = make_float4(sx, sy, sz, 0.0f);
}

// ---------------------------------------------------------------------------
// features of a row
// ---------------------------------------------------------------------------
struct RecordRows {   // training / evaluation records: d in cells, s in [0,1)
  const float4 *D, *S;
  long first, n;
  __device__ long count() const { return n; }
  __device__ bool load(long row, float (&x)[kIn]) const {
    const float4 d = D[first + row], s = S[first + row];
    x[0] = d.x; x[1] = d.y; x[2] = d.z;
    x[3] = s.x - 0.5f; x[4] = s.y - 0.5f; x[5] = s.z - 0.5f;
    return d.w != 0.0f;
  }
};

struct LoosePairs {   // (target, source) pairs of the loose list
  const ccs_uniforms *U;
  const float4 *list;
  const int2 *pairs;
  const int *total;
  __device__ long count() const { return *total; }
  __device__ bool load(long row, float (&x)[kIn]) const {
    const ccs_uniforms &u = *U;
    const int2 pr = pairs[row];
    const f3 pi = xyz(list[pr.x]), pj = xyz(list[pr.y]);
    const f3 d = (pj - pi) * u.invH;
    f3 g;
    box_of(u, pj, g);
    x[0] = d.x; x[1] = d.y; x[2] = d.z;
    x[3] = g.x - floorf(g.x) - 0.5f; x[4] = g.y - floorf(g.y) - 0.5f; x[5] = g.z - floorf(g.z) - 0.5f;
    return true;
  }
};

// the operand image and biases into shared memory (16-byte pieces)
__device__ __forceinline__ void load_image(const uint8_t *__restrict__ img, uint8_t *w, uint8_t *bias) {
  const uint4 *src = reinterpret_cast<const uint4 *>(img);
  for (int i = threadIdx.x; i < kImgBytes / 16; i += blockDim.x) reinterpret_cast<uint4 *>(w)[i] = src[i];
  for (int i = threadIdx.x; i < (kImgTotal - kImgBytes) / 16; i += blockDim.x)
    reinterpret_cast<uint4 *>(bias)[i] = src[kImgBytes / 16 + i];
}

// issue (one thread) n K-steps of an MMA whose A has K = kA and B has K = kB columns
__device__ __forceinline__ void mma_k(uint32_t d, uint32_t a, int kA, uint32_t b, int kB, uint32_t idesc, int steps,
                                      bool accumulate) {
  for (int s = 0; s < steps; ++s)
    mma(d, sdesc(a + 256u * s, kA), sdesc(b + 256u * s, kB), idesc, (accumulate || s > 0) ? 1u : 0u);
}

// ---------------------------------------------------------------------------
// inference: pairs in, the mesh's pair force (cells^-2) out.  128 threads, one
// per tile row (= TMEM lane); a persistent loop over tiles.
// ---------------------------------------------------------------------------
template <class Rows>
__global__ void __launch_bounds__(kRows, 1) k_nn_forward(Rows rows, const uint8_t *__restrict__ img,
                                                         float4 *__restrict__ out, unsigned *status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int t = threadIdx.x, warp = t >> 5;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + fMisc);
  uint32_t *slot = reinterpret_cast<uint32_t *>(sm + fMisc + 8);
  const float *b1 = reinterpret_cast<const float *>(sm + fBias), *b2 = b1 + 64, *b3 = b2 + 64;
  const long n = rows.count(), tiles = (n + kRows - 1) / kRows;
  if (blockIdx.x >= tiles) return;   // no tile for this CTA: nothing loaded, nothing allocated
  load_image(img, sm + fW, sm + fBias);
  if (t == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(slot, 128);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tm = *slot, lane = tm + ((uint32_t)(warp * 32) << 16);
  const uint32_t base = smem_u32(sm);
  uint32_t phase = 0;
  bool ok = true;
  for (long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const long row = tile * kRows + t;
    float x[kIn] = {0, 0, 0, 0, 0, 0};
    bool live = row < n && rows.load(row, x);
    uint16_t xb[16];
    input_row(x, live, xb);
    store_row<16>(sm + fX, t, xb);
    fence_async_smem();
    __syncthreads();
    // layer 1 -> TMEM columns [0, 64)
    if (t == 0) {
      fence_after();
      mma_k(tm, base + fX, 16, base + fW + 2 * iW1, 16, idesc_bf16(128, 64), 1, false);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    fence_after();
    {
      float h[64];
      tmem_load<64>(lane, h);
      uint16_t a[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) a[j] = bf16_bits(silu(h[j] + b1[j]));
      store_row<64>(sm + fA1, t, a);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    // layer 2 -> [64, 128)
    if (t == 0) {
      fence_after();
      mma_k(tm + 64, base + fA1, 64, base + fW + 2 * iW2, 64, idesc_bf16(128, 64), 4, false);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    fence_after();
    {
      float h[64];
      tmem_load<64>(lane + 64, h);
      uint16_t a[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) a[j] = bf16_bits(silu(h[j] + b2[j]));
      store_row<64>(sm + fA2, t, a);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    // layer 3 -> [0, 16) (layer 1's columns, read by every lane above)
    if (t == 0) {
      fence_after();
      mma_k(tm, base + fA2, 64, base + fW + 2 * iW3, 64, idesc_bf16(128, 16), 4, false);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    fence_after();
    float y[16];
    tmem_load<16>(lane, y);
    if (live) out[row] = make_float4(y[0] + b3[0], y[1] + b3[1], y[2] + b3[2], 0.0f);
    fence_before();
    __syncthreads();
  }
  if (!ok) {
    if (t == 0) atomicOr(status, kStatusNN);
    mbar_wait(bar, phase ^ 1u, kWaitLimit);   // the phase that timed out: let its MMA land before the columns go
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tm, 128);
}

// ---------------------------------------------------------------------------
// training: forward, backward and the weight gradients of `tiles` tiles per
// CTA; the CTA's summed gradient and squared error go to partial[blockIdx.x].
// TMEM: [0,64) layer 1 / dA1, [64,128) layer 2 / dA2, [128,144) the output,
// [256,400) the stacked gradient of layers 2 and 3 (+ bias column 384),
// [400,416) the gradient of layer 1 (+ bias column 412).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRows, 1) k_nn_train(RecordRows recs, const float4 *__restrict__ L, long rowsInBatch,
                                                       int tiles, float gscale, const uint8_t *__restrict__ img,
                                                       float *__restrict__ partial, unsigned *status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int t = threadIdx.x, warp = t >> 5;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + tMisc);
  uint32_t *slot = reinterpret_cast<uint32_t *>(sm + tMisc + 8);
  float *sLoss = reinterpret_cast<float *>(sm + tMisc + 16);
  const float *b1 = reinterpret_cast<const float *>(sm + tBias), *b2 = b1 + 64, *b3 = b2 + 64;
  // zero everything (padding rows and columns stay zero), then the weights and the ones row
  for (int i = t; i < kTrainSmem / 16; i += kRows) reinterpret_cast<uint4 *>(sm)[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  load_image(img, sm + tW, sm + tBias);
  *reinterpret_cast<uint16_t *>(sm + tGB + canon(128, t, 128)) = 0x3F80;   // B row 128: ones
  if (t == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(slot, 512);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tm = *slot, lane = tm + ((uint32_t)(warp * 32) << 16);
  const uint32_t base = smem_u32(sm);
  uint32_t phase = 0;
  bool ok = true;
  float sq = 0.0f;
  for (int k = 0; k < tiles && ok; ++k) {
    const long row = ((long)blockIdx.x * tiles + k) * kRows + t;
    float x[kIn] = {0, 0, 0, 0, 0, 0};
    const bool live = row < rowsInBatch && recs.load(row, x);
    const float4 lab = live ? L[recs.first + row] : make_float4(0, 0, 0, 0);
    uint16_t xb[16];
    input_row(x, live, xb);
    store_row<16>(sm + tX, t, xb);
    store_col<16>(sm + tXT, 0, t, xb);
    fence_async_smem();
    __syncthreads();
    // forward 1
    if (t == 0) {
      fence_after();
      mma_k(tm, base + tX, 16, base + tW + 2 * iW1, 16, idesc_bf16(128, 64), 1, false);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    fence_after();
    float h1[64], h2[64];
    tmem_load<64>(lane, h1);
    {
      uint16_t a[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) {
        h1[j] += b1[j];
        a[j] = bf16_bits(silu(h1[j]));
      }
      store_row<64>(sm + tA1, t, a);
      store_col<64>(sm + tGB, 0, t, a);   // A1^T: B rows 0..63
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    // forward 2
    if (t == 0) {
      fence_after();
      mma_k(tm + 64, base + tA1, 64, base + tW + 2 * iW2, 64, idesc_bf16(128, 64), 4, false);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    fence_after();
    tmem_load<64>(lane + 64, h2);
    {
      uint16_t a[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) {
        h2[j] += b2[j];
        a[j] = bf16_bits(silu(h2[j]));
      }
      store_row<64>(sm + tA2, t, a);
      store_col<64>(sm + tGB, 64, t, a);   // A2^T: B rows 64..127
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    // forward 3
    if (t == 0) {
      fence_after();
      mma_k(tm + 128, base + tA2, 64, base + tW + 2 * iW3, 64, idesc_bf16(128, 16), 4, false);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    fence_after();
    {
      float y[16];
      tmem_load<16>(lane + 128, y);
      uint16_t dy[16];
      const float lb[3] = {lab.x, lab.y, lab.z};
#pragma unroll
      for (int c = 0; c < 16; ++c) dy[c] = 0;
#pragma unroll
      for (int c = 0; c < kOut; ++c) {
        const float e = live ? y[c] + b3[c] - lb[c] : 0.0f;
        sq += e * e;
        dy[c] = bf16_bits(e * gscale);
      }
      store_row<16>(sm + tDY, t, dy);
      uint16_t dy3[3] = {dy[0], dy[1], dy[2]};
      store_col<3>(sm + tGA, 64, t, dy3);   // dY^T: A rows 64..66
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    // backward through layer 3: dA2 = dY W3 -> [64, 128)
    if (t == 0) {
      fence_after();
      mma_k(tm + 64, base + tDY, 16, base + tW + 2 * iW3T, 16, idesc_bf16(128, 64), 1, false);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    fence_after();
    {
      float g[64];
      tmem_load<64>(lane + 64, g);
      uint16_t dh[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) dh[j] = bf16_bits(g[j] * silu_grad(h2[j]));
      store_row<64>(sm + tDH2, t, dh);
      store_col<64>(sm + tGA, 0, t, dh);   // dH2^T: A rows 0..63
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    // backward through layer 2: dA1 = dH2 W2 -> [0, 64)
    if (t == 0) {
      fence_after();
      mma_k(tm, base + tDH2, 64, base + tW + 2 * iW2T, 64, idesc_bf16(128, 64), 4, false);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    fence_after();
    {
      float g[64];
      tmem_load<64>(lane, g);
      uint16_t dh[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) dh[j] = bf16_bits(g[j] * silu_grad(h1[j]));
      store_col<64>(sm + tGA2, 0, t, dh);   // dH1^T: A rows 0..63
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    // weight gradients over the tile's rows, accumulated over the CTA's tiles
    if (t == 0) {
      fence_after();
      mma_k(tm + 256, base + tGA, 128, base + tGB, 128, idesc_bf16(128, 144), 8, k > 0);
      mma_k(tm + 400, base + tGA2, 128, base + tXT, 128, idesc_bf16(128, 16), 8, k > 0);
      commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, kWaitLimit));
    phase ^= 1;
  }
  if (ok) {
    fence_after();
    float *P = partial + (size_t)blockIdx.x * kStride;
    // lanes 0..63: dW2 (columns 0..63) and db2 (column 128); lanes 64..66: dW3 (64..127) and db3 (128)
#pragma unroll 1
    for (int c = 0; c < 9; ++c) {
      float g[16];
      tmem_load<16>(lane + 256 + 16 * c, g);
      if (c < 4 && t < 64) {
#pragma unroll
        for (int i = 0; i < 16; ++i) P[oW2 + t * 64 + 16 * c + i] = g[i];
      } else if (c >= 4 && c < 8 && t >= 64 && t < 64 + kOut) {
#pragma unroll
        for (int i = 0; i < 16; ++i) P[oW3 + (t - 64) * 64 + 16 * (c - 4) + i] = g[i];
      } else if (c == 8 && t < 64) {
        P[oB2 + t] = g[0];
      } else if (c == 8 && t >= 64 && t < 64 + kOut) {
        P[oB3 + t - 64] = g[0];
      }
    }
    float g2[16];
    tmem_load<16>(lane + 400, g2);
    if (t < 64) {
#pragma unroll
      for (int f = 0; f < kIn; ++f) P[oW1 + t * kIn + f] = g2[f] + g2[kIn + f];
      P[oB1 + t] = g2[kOnes];
    }
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) sq += __shfl_xor_sync(0xFFFFFFFFu, sq, s);
    if ((t & 31) == 0) sLoss[warp] = sq;
    __syncthreads();
    if (t == 0) P[kParams] = (sLoss[0] + sLoss[1]) + (sLoss[2] + sLoss[3]);
  } else {
    if (t == 0) atomicOr(status, kStatusNN);
    mbar_wait(bar, phase ^ 1u, kWaitLimit);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tm, 512);
}

// ---------------------------------------------------------------------------
// the optimiser: sums the CTAs' partial gradients in order, takes an Adam
// step on the FP32 master weights (or only writes the gradient), and rewrites
// the BF16 operand image
// ---------------------------------------------------------------------------
__device__ __forceinline__ void set_half(uint8_t *img, int sub, uint32_t off, float w) {
  *reinterpret_cast<uint16_t *>(img + 2 * sub + off) = bf16_bits(w);
}

__device__ void write_image(uint8_t *img, int p, float w) {
  if (p < oB1) {
    const int o = p / kIn, f = p % kIn;
    set_half(img, iW1, canon(o, f, 16), w);
    set_half(img, iW1, canon(o, kIn + f, 16), w);   // the low input parts see the same weight
  } else if (p < oW2) {
    reinterpret_cast<float *>(img + bB1)[p - oB1] = w;
  } else if (p < oB2) {
    const int o = (p - oW2) / kH, i = (p - oW2) % kH;
    set_half(img, iW2, canon(o, i, 64), w);
    set_half(img, iW2T, canon(i, o, 64), w);
  } else if (p < oW3) {
    reinterpret_cast<float *>(img + bB2)[p - oB2] = w;
  } else if (p < oB3) {
    const int c = (p - oW3) / kH, i = (p - oW3) % kH;
    set_half(img, iW3, canon(c, i, 64), w);
    set_half(img, iW3T, canon(i, c, 16), w);
  } else {
    reinterpret_cast<float *>(img + bB3)[p - oB3] = w;
  }
}

__global__ void k_nn_adam(const float *__restrict__ partial, int nPart, float *__restrict__ params,
                          float *__restrict__ m1, float *__restrict__ m2, float lr, float c1, float c2, int update,
                          float *__restrict__ gradOut, float lossScale, float *__restrict__ lossOut,
                          uint8_t *__restrict__ img) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == kParams) {
    float s = 0.0f;
    for (int c = 0; c < nPart; ++c) s += partial[(size_t)c * kStride + kParams];
    if (lossOut) *lossOut = s * lossScale;
    return;
  }
  if (p > kParams) return;
  float g = 0.0f;
  for (int c = 0; c < nPart; ++c) g += partial[(size_t)c * kStride + p];
  if (gradOut) gradOut[p] = g;
  if (!update) return;
  const float b1 = 0.9f, b2 = 0.999f;
  const float a = b1 * m1[p] + (1.0f - b1) * g, v = b2 * m2[p] + (1.0f - b2) * g * g;
  m1[p] = a;
  m2[p] = v;
  const float w = params[p] - lr * (a * c1) / (sqrtf(v * c2) + 1e-8f);
  params[p] = w;
  write_image(img, p, w);
}

__global__ void k_nn_image(const float *__restrict__ params, uint8_t *__restrict__ img) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kParams) write_image(img, p, params[p]);
}

// ---------------------------------------------------------------------------
// the learned P3M pass over the loose list (the pass of src/glsl-sim.js:
// 676-754 with the table's force replaced by the network's inside half the
// cut): pairs inside half the cut are enumerated in (target, source) order,
// the network evaluates the mesh part of every one, and each target's pairs --
// those and the list members out to the full cut, with the table -- are summed
// by one warp.
// ---------------------------------------------------------------------------
// count pass (pairs == nullptr) and fill pass: one warp per target, the lanes test 32 consecutive sources
// at a time; ballot prefix sums keep each target's pairs in ascending source order
__global__ void __launch_bounds__(256) k_nn_pp_pairs(const ccs_uniforms *__restrict__ U,
                                                     const float4 *__restrict__ list, int cap,
                                                     const int *__restrict__ offs, int *__restrict__ counts,
                                                     int2 *__restrict__ pairs) {
  const int lane = threadIdx.x & 31, warps = (gridDim.x * blockDim.x) >> 5;
  const ccs_uniforms &u = *U;
  const int count = u.ppCount;
  const float cutN = xmul(0.5f, u.cut), cut2 = xmul(cutN, cutN);
  // a warp per target, the grid striding over the list's length (read on the device)
  for (int me = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; me < min(count, cap); me += warps) {
  const float4 P = list[me];
  const bool active = P.w != 0.0f;
  int n = 0;
  const int at = pairs ? offs[me] : 0;
  if (active) {
    for (int j0 = 0; j0 < count; j0 += 32) {
      const int j = j0 + lane;
      bool near = false;
      if (j < count && j != me) {
        const f3 d = xsub3(xyz(list[j]), xyz(P));
        near = xdot(d, d) < cut2;
      }
      const unsigned bal = __ballot_sync(0xFFFFFFFFu, near);
      if (pairs && near) pairs[at + n + __popc(bal & ((1u << lane) - 1u))] = make_int2(me, j);
      n += __popc(bal);
    }
  }
  if (!pairs && lane == 0) counts[me] = n;
  }
}

// exclusive scan of the targets' pair counts: offs[0..count], total = offs[count]
__global__ void __launch_bounds__(1024) k_nn_pp_scan(const ccs_uniforms *__restrict__ U,
                                                     const int *__restrict__ counts, int *__restrict__ offs,
                                                     int *__restrict__ total) {
  __shared__ int warpSum[32];
  const int E = U->ppCount;
  const int per = (E + 1023) / 1024;
  const int e0 = threadIdx.x * per, e1 = min(e0 + per, E);
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
  if (threadIdx.x == 1023) {
    offs[E] = run;
    *total = run;
  }
}

// one warp per target: the lanes take every 32nd of its pairs inside half the cut (the network's model of
// the mesh's pull, blended into the table's by tau_in from 0.8 of the half cut out to it), then every 32nd
// list member between the half cut and the cut (the plain pass's table, tapered to the cut); a fixed
// shuffle tree adds the lanes
__global__ void __launch_bounds__(256) k_nn_pp_reduce(const ccs_uniforms *__restrict__ U,
                                                      const float4 *__restrict__ list, const float *__restrict__ box,
                                                      int cap, const float2 *__restrict__ tab,
                                                      const int2 *__restrict__ pairs, const int *__restrict__ offs,
                                                      const float4 *__restrict__ mesh, float4 *__restrict__ force) {
  const int lane = threadIdx.x & 31, warps = (gridDim.x * blockDim.x) >> 5;
  const ccs_uniforms &u = *U;
  const int count = u.ppCount;
  // a warp per target, the grid striding over the list's length; only the list's seats are ever read
  for (int me = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; me < min(count, cap); me += warps) {
  float4 o = make_float4(0, 0, 0, 0);
  const float4 P = list[me];
  if (P.w != 0.0f) {
    const float myBox = box[me];
    const float cut = u.cut, cutN = xmul(0.5f, cut), a2 = u.a2, a = fsqrt(a2);
    const float cut2 = xmul(cut, cut), cutN2 = xmul(cutN, cutN);
    const float binScale = fdiv(64.0f, cut), inScale = fdiv(1.0f, 0.8f * cutN - cutN),
                outScale = fdiv(1.0f, 0.8f * cut - cut);
    const float invH2 = u.invH * u.invH, eps2Cell = u.eps2Cell;
    f3 acc = mk(0, 0, 0);
    float pot = 0.0f;
    // a pair's pull and potential: Newton softened at a, less the mesh's own as the network (weight tin) and
    // the table (the rest) model it, tapered to the cut
    auto pair = [&](const float4 Q, const f3 d, float r2, float tin, const float4 R, float bj) {
      const float r = fsqrt(r2);
      const float invN = rsqrtf(r2 + a2);
      const float to = clampf((r - cut) * outScale, 0.0f, 1.0f);
      const float tout = to * to * (3.0f - 2.0f * to);
      f3 f = d * (invN * invN * invN * tout);
      float Ty = 0.0f;
      if (myBox >= 0.0f && bj == myBox) {
        const float xx = clampf(r * binScale - 0.5f, 0.0f, 63.0f);
        const int k = (int)xx, k1 = min(k + 1, 63);
        const float tt = xx - (float)k;
        const float2 ta = tab[k], tb = tab[k1];
        const float Tx = ta.x + (tb.x - ta.x) * tt;
        Ty = ta.y + (tb.y - ta.y) * tt;
        const f3 table = d * (fdiv(1.0f, fmaxf(r, 1e-6f)) * fdiv(Tx, fmaxf(r2, a2)));
        f = f - table * ((1.0f - tin) * tout);
        if (tin > 0.0f) {
          const float qn = rsqrtf(r2 + eps2Cell);
          f = f - (d * (qn * qn * qn) + mk(R.x, R.y, R.z) * invH2) * tin;
        }
      }
      acc = acc + f * Q.w;
      pot += Q.w * (-invN - fdiv(Ty, fmaxf(r, a))) * tout;
    };
    const int q0 = offs[me], q1 = offs[me + 1];
    for (int q = q0 + lane; q < q1; q += 32) {   // inside half the cut: the network's pairs
      const int j = pairs[q].y;
      const float4 Q = list[j];
      const f3 d = xsub3(xyz(Q), xyz(P));
      const float r2 = xdot(d, d);
      const float ti = clampf((fsqrt(r2) - cutN) * inScale, 0.0f, 1.0f);
      pair(Q, d, r2, ti * ti * (3.0f - 2.0f * ti), mesh[q], box[j]);
    }
    for (int j = lane; j < count; j += 32) {     // between half the cut and the cut: the table
      if (j == me) continue;
      const float4 Q = list[j];
      const f3 d = xsub3(xyz(Q), xyz(P));
      const float r2 = xdot(d, d);
      if (r2 < cutN2 || r2 >= cut2) continue;
      pair(Q, d, r2, 0.0f, make_float4(0, 0, 0, 0), box[j]);
    }
#pragma unroll
    for (int sh = 16; sh >= 1; sh >>= 1) {
      acc.x += __shfl_xor_sync(0xFFFFFFFFu, acc.x, sh);
      acc.y += __shfl_xor_sync(0xFFFFFFFFu, acc.y, sh);
      acc.z += __shfl_xor_sync(0xFFFFFFFFu, acc.z, sh);
      pot += __shfl_xor_sync(0xFFFFFFFFu, pot, sh);
    }
    o = make_float4(acc.x * u.Gm, acc.y * u.Gm, acc.z * u.Gm, pot * u.Gm);
  }
  if (lane < 4) force[(size_t)lane * cap + me] = lane == 0 ? o : make_float4(0, 0, 0, 0);
  }
}

int forward_grid() { return 3 * sm_count(); }

}  // namespace nn

// ---------------------------------------------------------------------------
// launchers used by the engine
// ---------------------------------------------------------------------------
size_t nn_pp_count_ints() { return (size_t)CCS_PP_CAP + 1; }

int launch_pp_nn(const ccs_uniforms *u, const float4 *list, const float *box, int cap, const float2 *tab,
                 const uint8_t *img, int *counts, int *offs, int *total, int2 *pairs, float4 *mesh, float4 *force,
                 unsigned *status, cudaStream_t st) {
  // grids striding over the list's length on the device, so a captured launch serves any length
  const int g = std::min((cap * 32 + 255) / 256, 8 * (nn::forward_grid() / 3));
  nn::k_nn_pp_pairs<<<g, 256, 0, st>>>(u, list, cap, nullptr, counts, nullptr);
  nn::k_nn_pp_scan<<<1, 1024, 0, st>>>(u, counts, offs, total);
  nn::k_nn_pp_pairs<<<g, 256, 0, st>>>(u, list, cap, offs, counts, pairs);
  nn::LoosePairs rows{u, list, pairs, total};
  nn::k_nn_forward<nn::LoosePairs><<<nn::forward_grid(), nn::kRows, nn::kFwdSmem, st>>>(rows, img, mesh, status);
  nn::k_nn_pp_reduce<<<g, 256, 0, st>>>(u, list, box, cap, tab, pairs, offs, mesh, force);
  return 5;
}

cudaError_t init_nn_kernels() {
  cudaError_t e = cudaFuncSetAttribute(nn::k_nn_forward<nn::LoosePairs>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       nn::kFwdSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(nn::k_nn_forward<nn::RecordRows>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           nn::kFwdSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(nn::k_nn_train, cudaFuncAttributeMaxDynamicSharedMemorySize, nn::kTrainSmem);
}

int launch_nn_sample_state(const ccs_uniforms *u, const float4 *pos, int N, long count, uint32_t seed, float cutG,
                           float4 *D, float4 *S, cudaStream_t st) {
  if (count <= 0) return 0;
  nn::k_nn_sample_state<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(u, pos, N, count, seed, cutG, D, S);
  return 1;
}

}  // namespace ccs

// ---------------------------------------------------------------------------
// the network object and its C ABI
// ---------------------------------------------------------------------------
using namespace ccs;

struct ccs_nn {
  int device = 0;
  cudaStream_t st = nullptr;
  std::string err;
  float *params = nullptr, *m1 = nullptr, *m2 = nullptr, *partial = nullptr, *grad = nullptr, *loss = nullptr;
  uint8_t *img = nullptr;
  unsigned *status = nullptr;
  float4 *D = nullptr, *S = nullptr, *L = nullptr, *out = nullptr;
  long capPairs = 0, nPairs = 0;
  int partCap = 0, steps = 0;
};

namespace {

std::mutex g_nnInit;
bool g_nnInitDone[64] = {};

#define NN_TRY(nn, call)                                                  \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      (nn)->err = std::string(#call) + ": " + cudaGetErrorString(e_);     \
      return CCS_E_CUDA;                                                  \
    }                                                                     \
  } while (0)

template <class T>
int nn_alloc(ccs_nn *nn, T **p, size_t count) {
  if (*p) { cudaFree(*p); *p = nullptr; }
  if (count == 0) count = 1;
  if (cudaMalloc((void **)p, sizeof(T) * count) != cudaSuccess) {
    nn->err = "cudaMalloc failed";
    *p = nullptr;
    return CCS_E_NOMEM;
  }
  return CCS_OK;
}

int nn_check(ccs_nn *nn) {
  cudaError_t e = cudaStreamSynchronize(nn->st);
  if (e != cudaSuccess) {
    nn->err = std::string("stream: ") + cudaGetErrorString(e);
    return CCS_E_CUDA;
  }
  unsigned s = 0;
  if (cudaMemcpy(&s, nn->status, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return CCS_E_CUDA;
  if (s) {
    nn->err = "a tensor-core wait gave up";
    return CCS_E_KERNEL;
  }
  return CCS_OK;
}

int ensure_pool(ccs_nn *nn, long need) {
  if (need <= nn->capPairs) return CCS_OK;
  long cap = std::max(need, nn->capPairs * 2);
  float4 *D = nullptr, *S = nullptr, *L = nullptr;
  if (cudaMalloc(&D, 16 * (size_t)cap) != cudaSuccess || cudaMalloc(&S, 16 * (size_t)cap) != cudaSuccess ||
      cudaMalloc(&L, 16 * (size_t)cap) != cudaSuccess) {
    cudaFree(D); cudaFree(S); cudaFree(L);
    nn->err = "cudaMalloc of the pair pool failed";
    return CCS_E_NOMEM;
  }
  if (nn->nPairs) {
    NN_TRY(nn, cudaMemcpyAsync(D, nn->D, 16 * (size_t)nn->nPairs, cudaMemcpyDeviceToDevice, nn->st));
    NN_TRY(nn, cudaMemcpyAsync(S, nn->S, 16 * (size_t)nn->nPairs, cudaMemcpyDeviceToDevice, nn->st));
    NN_TRY(nn, cudaMemcpyAsync(L, nn->L, 16 * (size_t)nn->nPairs, cudaMemcpyDeviceToDevice, nn->st));
    NN_TRY(nn, cudaStreamSynchronize(nn->st));
  }
  cudaFree(nn->D); cudaFree(nn->S); cudaFree(nn->L);
  nn->D = D; nn->S = S; nn->L = L;
  nn->capPairs = cap;
  return CCS_OK;
}

int ensure_partials(ccs_nn *nn, int parts) {
  if (parts <= nn->partCap) return CCS_OK;
  int rc = nn_alloc(nn, &nn->partial, (size_t)parts * nn::kStride);
  if (rc) return rc;
  nn->partCap = parts;
  return CCS_OK;
}

// host records (d.xyz, s.xyz) into device float4 pairs at [at, at + n)
int upload_records(ccs_nn *nn, const float *rec6, long n, float4 *D, float4 *S) {
  std::vector<float> d(4 * (size_t)n), s(4 * (size_t)n);
  for (long k = 0; k < n; ++k) {
    d[4 * k + 0] = rec6[6 * k + 0]; d[4 * k + 1] = rec6[6 * k + 1]; d[4 * k + 2] = rec6[6 * k + 2];
    d[4 * k + 3] = 1.0f;
    s[4 * k + 0] = rec6[6 * k + 3]; s[4 * k + 1] = rec6[6 * k + 4]; s[4 * k + 2] = rec6[6 * k + 5];
    s[4 * k + 3] = 0.0f;
  }
  NN_TRY(nn, cudaMemcpyAsync(D, d.data(), 16 * (size_t)n, cudaMemcpyHostToDevice, nn->st));
  NN_TRY(nn, cudaMemcpyAsync(S, s.data(), 16 * (size_t)n, cudaMemcpyHostToDevice, nn->st));
  NN_TRY(nn, cudaStreamSynchronize(nn->st));
  return CCS_OK;
}

// scratch records of the host-facing calls live after the pool's end
int scratch(ccs_nn *nn, long n, float4 **D, float4 **S, float4 **L) {
  int rc = ensure_pool(nn, nn->nPairs + n);
  if (rc) return rc;
  *D = nn->D + nn->nPairs;
  *S = nn->S + nn->nPairs;
  *L = nn->L + nn->nPairs;
  return CCS_OK;
}

// one training pass (or gradient) over rows [first, first + rows) of the given arrays
int run_batch(ccs_nn *nn, const float4 *D, const float4 *S, const float4 *L, long first, long rows, int tilesPerCta,
              int update, float lr, float *gradOut, float *lossOut) {
  const long tiles = (rows + nn::kRows - 1) / nn::kRows;
  const int grid = (int)((tiles + tilesPerCta - 1) / tilesPerCta);
  int rc = ensure_partials(nn, grid);
  if (rc) return rc;
  nn::RecordRows recs{D, S, first, rows};
  const float gscale = 2.0f / (3.0f * (float)rows);
  nn::k_nn_train<<<grid, nn::kRows, nn::kTrainSmem, nn->st>>>(recs, L, rows, tilesPerCta, gscale, nn->img,
                                                              nn->partial, nn->status);
  float c1 = 1.0f, c2 = 1.0f;
  if (update) {
    ++nn->steps;
    c1 = (float)(1.0 / (1.0 - std::pow(0.9, nn->steps)));
    c2 = (float)(1.0 / (1.0 - std::pow(0.999, nn->steps)));
  }
  nn::k_nn_adam<<<(nn::kParams + 256) / 256, 256, 0, nn->st>>>(nn->partial, grid, nn->params, nn->m1, nn->m2, lr, c1,
                                                                c2, update, gradOut, 1.0f / (3.0f * (float)rows),
                                                                lossOut, nn->img);
  NN_TRY(nn, cudaGetLastError());
  return CCS_OK;
}

}  // namespace

namespace ccs {

// the engine-side half (ccs_api.cu) draws the records; this labels them and grows the pool
int nn_reserve(ccs_nn *nn, int64_t count, float4 **D, float4 **S, cudaStream_t *st) {
  int rc = ensure_pool(nn, nn->nPairs + count);
  if (rc) return rc;
  *D = nn->D + nn->nPairs;
  *S = nn->S + nn->nPairs;
  *st = nn->st;
  return CCS_OK;
}

int nn_commit(ccs_nn *nn, int64_t count) {
  float4 *D = nn->D + nn->nPairs, *S = nn->S + nn->nPairs, *L = nn->L + nn->nPairs;
  if (count) {
    nn::k_nn_label<<<(unsigned)((count + 255) / 256), 256, 0, nn->st>>>(D, S, count, L);
    NN_TRY(nn, cudaGetLastError());
  }
  int rc = nn_check(nn);
  if (rc) return rc;
  nn->nPairs += count;
  return CCS_OK;
}

const uint8_t *nn_image(const ccs_nn *nn) { return nn->img; }
int nn_device(const ccs_nn *nn) { return nn->device; }

}  // namespace ccs

extern "C" {

int ccs_nn_create(int device, uint32_t seed, ccs_nn **out) {
  if (!out) return CCS_E_ARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return CCS_E_CUDA;
  ccs_nn *nn = new ccs_nn();
  nn->device = device;
  {
    std::lock_guard<std::mutex> lk(g_nnInit);
    if (device >= 0 && device < 64 && !g_nnInitDone[device]) {
      if (init_nn_kernels() != cudaSuccess) {
        delete nn;
        return CCS_E_CUDA;
      }
      g_nnInitDone[device] = true;
    }
  }
  int rc = CCS_OK;
  if (cudaStreamCreateWithFlags(&nn->st, cudaStreamNonBlocking) != cudaSuccess) rc = CCS_E_CUDA;
  rc |= nn_alloc(nn, &nn->params, nn::kParams);
  rc |= nn_alloc(nn, &nn->m1, nn::kParams);
  rc |= nn_alloc(nn, &nn->m2, nn::kParams);
  rc |= nn_alloc(nn, &nn->grad, nn::kParams);
  rc |= nn_alloc(nn, &nn->loss, 1 << 16);
  rc |= nn_alloc(nn, &nn->img, nn::kImgTotal);
  rc |= nn_alloc(nn, &nn->status, 1);
  if (rc) {
    ccs_nn_destroy(nn);
    return rc < 0 ? rc : CCS_E_NOMEM;
  }
  // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights from a mulberry32 stream, zero biases
  std::vector<float> p(nn::kParams, 0.0f);
  uint32_t a = seed;
  auto rnd = [&a]() {
    a += 0x6D2B79F5u;
    uint32_t t = a;
    t = (t ^ (t >> 15)) * (t | 1u);
    t ^= t + (t ^ (t >> 7)) * (t | 61u);
    return (double)((t ^ (t >> 14)) >> 0) / 4294967296.0;
  };
  for (int k = 0; k < nn::kH * nn::kIn; ++k) p[nn::oW1 + k] = (float)((2.0 * rnd() - 1.0) / std::sqrt(6.0));
  for (int k = 0; k < nn::kH * nn::kH; ++k) p[nn::oW2 + k] = (float)((2.0 * rnd() - 1.0) / 8.0);
  for (int k = 0; k < nn::kOut * nn::kH; ++k) p[nn::oW3 + k] = (float)((2.0 * rnd() - 1.0) / 8.0);
  rc = ccs_nn_set_params(nn, p.data());
  if (rc) {
    ccs_nn_destroy(nn);
    return rc;
  }
  *out = nn;
  return CCS_OK;
}

int ccs_nn_destroy(ccs_nn *nn) {
  if (!nn) return CCS_OK;
  cudaSetDevice(nn->device);
  if (nn->st) cudaStreamSynchronize(nn->st);
  cudaFree(nn->params); cudaFree(nn->m1); cudaFree(nn->m2); cudaFree(nn->grad); cudaFree(nn->loss);
  cudaFree(nn->partial); cudaFree(nn->img); cudaFree(nn->status);
  cudaFree(nn->D); cudaFree(nn->S); cudaFree(nn->L); cudaFree(nn->out);
  if (nn->st) cudaStreamDestroy(nn->st);
  delete nn;
  return CCS_OK;
}

const char *ccs_nn_last_error(const ccs_nn *nn) { return nn ? nn->err.c_str() : "null network"; }

int ccs_nn_set_params(ccs_nn *nn, const float *params) {
  if (!nn || !params) return CCS_E_ARG;
  cudaSetDevice(nn->device);
  NN_TRY(nn, cudaMemcpyAsync(nn->params, params, 4 * (size_t)nn::kParams, cudaMemcpyHostToDevice, nn->st));
  NN_TRY(nn, cudaMemsetAsync(nn->m1, 0, 4 * (size_t)nn::kParams, nn->st));
  NN_TRY(nn, cudaMemsetAsync(nn->m2, 0, 4 * (size_t)nn::kParams, nn->st));
  NN_TRY(nn, cudaMemsetAsync(nn->img, 0, nn::kImgTotal, nn->st));
  NN_TRY(nn, cudaMemsetAsync(nn->status, 0, 4, nn->st));
  nn::k_nn_image<<<(nn::kParams + 255) / 256, 256, 0, nn->st>>>(nn->params, nn->img);
  NN_TRY(nn, cudaGetLastError());
  nn->steps = 0;
  return nn_check(nn);
}

int ccs_nn_get_params(ccs_nn *nn, float *params) {
  if (!nn || !params) return CCS_E_ARG;
  cudaSetDevice(nn->device);
  NN_TRY(nn, cudaMemcpyAsync(params, nn->params, 4 * (size_t)nn::kParams, cudaMemcpyDeviceToHost, nn->st));
  return nn_check(nn);
}

int ccs_nn_clear(ccs_nn *nn) {
  if (!nn) return CCS_E_ARG;
  nn->nPairs = 0;
  return CCS_OK;
}

int64_t ccs_nn_pool_size(const ccs_nn *nn) { return nn ? (int64_t)nn->nPairs : -1; }

int ccs_nn_sample_uniform(ccs_nn *nn, int64_t count, uint32_t seed) {
  if (!nn || count < 0) return CCS_E_ARG;
  cudaSetDevice(nn->device);
  int rc = ensure_pool(nn, nn->nPairs + count);
  if (rc) return rc;
  if (count) {
    float4 *D = nn->D + nn->nPairs, *S = nn->S + nn->nPairs, *L = nn->L + nn->nPairs;
    const unsigned g = (unsigned)((count + 255) / 256);
    nn::k_nn_sample_uniform<<<g, 256, 0, nn->st>>>(count, seed, (float)(CCS_NN_CUT_CELLS), D, S);
    nn::k_nn_label<<<g, 256, 0, nn->st>>>(D, S, count, L);
    NN_TRY(nn, cudaGetLastError());
  }
  rc = nn_check(nn);
  if (rc) return rc;
  nn->nPairs += count;
  return CCS_OK;
}

int ccs_nn_read_pool(ccs_nn *nn, int64_t first, int64_t n, float *rec6, float *label3) {
  if (!nn || first < 0 || n < 0 || first + n > nn->nPairs) return CCS_E_ARG;
  cudaSetDevice(nn->device);
  std::vector<float4> d((size_t)n), s((size_t)n), l((size_t)n);
  NN_TRY(nn, cudaMemcpyAsync(d.data(), nn->D + first, 16 * (size_t)n, cudaMemcpyDeviceToHost, nn->st));
  NN_TRY(nn, cudaMemcpyAsync(s.data(), nn->S + first, 16 * (size_t)n, cudaMemcpyDeviceToHost, nn->st));
  NN_TRY(nn, cudaMemcpyAsync(l.data(), nn->L + first, 16 * (size_t)n, cudaMemcpyDeviceToHost, nn->st));
  int rc = nn_check(nn);
  if (rc) return rc;
  for (long k = 0; k < n; ++k) {
    if (rec6) {
      rec6[6 * k + 0] = d[k].x; rec6[6 * k + 1] = d[k].y; rec6[6 * k + 2] = d[k].z;
      rec6[6 * k + 3] = s[k].x; rec6[6 * k + 4] = s[k].y; rec6[6 * k + 5] = s[k].z;
      if (d[k].w == 0.0f) rec6[6 * k + 0] = rec6[6 * k + 1] = rec6[6 * k + 2] = NAN;   // a dead record
    }
    if (label3) {
      label3[3 * k + 0] = l[k].x; label3[3 * k + 1] = l[k].y; label3[3 * k + 2] = l[k].z;
    }
  }
  return CCS_OK;
}

int ccs_nn_labels(ccs_nn *nn, const float *rec6, int64_t n, float *label3) {
  if (!nn || n < 0 || (n && (!rec6 || !label3))) return CCS_E_ARG;
  if (!n) return CCS_OK;
  cudaSetDevice(nn->device);
  float4 *D, *S, *L;
  int rc = scratch(nn, n, &D, &S, &L);
  if (!rc) rc = upload_records(nn, rec6, n, D, S);
  if (rc) return rc;
  nn::k_nn_label<<<(unsigned)((n + 255) / 256), 256, 0, nn->st>>>(D, S, n, L);
  NN_TRY(nn, cudaGetLastError());
  std::vector<float4> l((size_t)n);
  NN_TRY(nn, cudaMemcpyAsync(l.data(), L, 16 * (size_t)n, cudaMemcpyDeviceToHost, nn->st));
  rc = nn_check(nn);
  if (rc) return rc;
  for (long k = 0; k < n; ++k) {
    label3[3 * k + 0] = l[k].x; label3[3 * k + 1] = l[k].y; label3[3 * k + 2] = l[k].z;
  }
  return CCS_OK;
}

int ccs_nn_forward(ccs_nn *nn, const float *rec6, int64_t n, float *out3) {
  if (!nn || n < 0 || (n && (!rec6 || !out3))) return CCS_E_ARG;
  if (!n) return CCS_OK;
  cudaSetDevice(nn->device);
  float4 *D, *S, *L;
  int rc = scratch(nn, n, &D, &S, &L);
  if (!rc) rc = upload_records(nn, rec6, n, D, S);
  if (rc) return rc;
  nn::RecordRows rows{D, S, 0, n};
  const long tiles = (n + nn::kRows - 1) / nn::kRows;
  const int grid = (int)std::min<long>(tiles, nn::forward_grid());
  nn::k_nn_forward<nn::RecordRows><<<grid, nn::kRows, nn::kFwdSmem, nn->st>>>(rows, nn->img, L, nn->status);
  NN_TRY(nn, cudaGetLastError());
  std::vector<float4> l((size_t)n);
  NN_TRY(nn, cudaMemcpyAsync(l.data(), L, 16 * (size_t)n, cudaMemcpyDeviceToHost, nn->st));
  rc = nn_check(nn);
  if (rc) return rc;
  for (long k = 0; k < n; ++k) {
    out3[3 * k + 0] = l[k].x; out3[3 * k + 1] = l[k].y; out3[3 * k + 2] = l[k].z;
  }
  return CCS_OK;
}

int ccs_nn_grad(ccs_nn *nn, const float *rec6, const float *label3, int64_t n, float *grad, float *loss) {
  if (!nn || n <= 0 || !rec6 || !label3 || !grad) return CCS_E_ARG;
  cudaSetDevice(nn->device);
  float4 *D, *S, *L;
  int rc = scratch(nn, n, &D, &S, &L);
  if (!rc) rc = upload_records(nn, rec6, n, D, S);
  if (rc) return rc;
  std::vector<float> l(4 * (size_t)n);
  for (long k = 0; k < n; ++k) {
    l[4 * k + 0] = label3[3 * k + 0]; l[4 * k + 1] = label3[3 * k + 1]; l[4 * k + 2] = label3[3 * k + 2];
    l[4 * k + 3] = 0.0f;
  }
  NN_TRY(nn, cudaMemcpyAsync(L, l.data(), 16 * (size_t)n, cudaMemcpyHostToDevice, nn->st));
  rc = run_batch(nn, D, S, L, 0, n, 1, 0, 0.0f, nn->grad, nn->loss);
  if (rc) return rc;
  NN_TRY(nn, cudaMemcpyAsync(grad, nn->grad, 4 * (size_t)nn::kParams, cudaMemcpyDeviceToHost, nn->st));
  float lv = 0.0f;
  NN_TRY(nn, cudaMemcpyAsync(&lv, nn->loss, 4, cudaMemcpyDeviceToHost, nn->st));
  rc = nn_check(nn);
  if (rc) return rc;
  if (loss) *loss = lv;
  return CCS_OK;
}

int ccs_nn_train(ccs_nn *nn, int64_t first, int64_t n, int epochs, int tilesPerCta, float lr, float *epochLoss) {
  if (!nn || first < 0 || n <= 0 || first + n > nn->nPairs || epochs <= 0 || tilesPerCta <= 0 || !(lr > 0.0f))
    return CCS_E_ARG;
  cudaSetDevice(nn->device);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, nn->device);
  const long batch = (long)sms * tilesPerCta * nn::kRows;
  const long perEpoch = (n + batch - 1) / batch;
  const long total = perEpoch * epochs;
  if (total > (1 << 16)) {
    nn->err = "more than 65536 optimiser steps in one call";
    return CCS_E_RANGE;
  }
  long step = 0;
  for (int e = 0; e < epochs; ++e) {
    for (long b = 0; b < perEpoch; ++b, ++step) {
      const long at = first + b * batch, rows = std::min(batch, first + n - at);
      // cosine decay to 5 % of the initial rate over the call
      const double frac = total > 1 ? (double)step / (double)(total - 1) : 1.0;
      const float lrs = (float)(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * frac))));
      int rc = run_batch(nn, nn->D, nn->S, nn->L, at, rows, tilesPerCta, 1, lrs, nullptr, nn->loss + step);
      if (rc) return rc;
    }
  }
  int rc = nn_check(nn);
  if (rc) return rc;
  if (epochLoss) {
    std::vector<float> l((size_t)total);
    NN_TRY(nn, cudaMemcpy(l.data(), nn->loss, 4 * (size_t)total, cudaMemcpyDeviceToHost));
    for (int e = 0; e < epochs; ++e) {
      double s = 0.0;
      for (long b = 0; b < perEpoch; ++b) s += l[(size_t)(e * perEpoch + b)];
      epochLoss[e] = (float)(s / (double)perEpoch);
    }
  }
  return CCS_OK;
}

}  // extern "C"
