// ccs_pp.cu -- the P3M pairwise correction for the loose list
// (src/glsl-sim.js:669-754, src/nbody.js:509-528).
//
// The reference gathers the list into a 128x64 texture and runs 4 x 8192
// fragments, each walking a quarter of the list.  Here the list is tiled two
// ways: a work item is 128 seats (i) against one chunk (j) of one quarter,
// with the chunk staged in shared memory; chunks are 128 entries wide for a
// full list (4096 items instead of 32K threads walking 2048 pairs each) and
// narrower for a short one (down to 16), so the few hundred entries a
// mid-impact list holds still spread over dozens of CTAs.  A persistent grid
// takes the items, counted from the list's length on the device.  A second
// kernel sums each quarter's chunks in a fixed order: the four slices the
// contact step adds are the reference's four slices, and the result is
// deterministic.  The cut-off test and the box comparison are exact; the
// force arithmetic is fast (FMA, rsqrt).
#include <algorithm>

#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {

namespace {
constexpr int kBlock = 256;
inline int blocks_for(long n, int b = kBlock) { return (int)((n + b - 1) / b); }
constexpr int kPPI = 128;                                  // seats per CTA
constexpr int kPPJ = 128;                                  // list entries per chunk
constexpr int kMaxChunks = (CCS_PP_CAP / 4 + kPPJ - 1) / kPPJ;   // chunks per quarter at full capacity
}  // namespace

size_t pp_partial_float4s() { return (size_t)4 * kMaxChunks * CCS_PP_CAP; }

__global__ void __launch_bounds__(kBlock) k_pp_gather(const ccs_uniforms *__restrict__ U,
                                                      const float4 *__restrict__ pos, const float *__restrict__ mat,
                                                      const int *__restrict__ index, int cap,
                                                      float4 *__restrict__ list, float *__restrict__ box) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= cap) return;
  const int i = index[s];
  if (i < 0) {
    list[s] = make_float4(0, 0, 0, 0);
    box[s] = -1.0f;
    return;
  }
  const float4 P = pos[i];
  f3 g;
  box[s] = (float)box_of(*U, xyz(P), g);
  list[s] = make_float4(P.x, P.y, P.z, mat[i]);
}

int launch_pp_gather(const ccs_uniforms *u, const float4 *pos, const float *mat, const int *index, int cap,
                     float4 *list, float *box, cudaStream_t st) {
  k_pp_gather<<<blocks_for(cap), kBlock, 0, st>>>(u, pos, mat, index, cap, list, box);
  return 1;
}

// a quarter's chunk width: eight chunks or so a quarter, 16 to kPPJ entries wide, so that a short list
// spreads over many CTAs and a long one keeps kPPJ (at most kMaxChunks chunks either way)
__device__ __forceinline__ int pp_chunk_width(int share) {
  const int w = ((share + 7) / 8 + 15) / 16 * 16;
  return min(max(w, 16), kPPJ);
}

// one pair's correction (PPFORCE_FS, src/glsl-sim.js:738-750): the softened Newton force less the mesh's own
// (the table, zeroed unless both read the same box), tapered to zero at the cut, added to (acc, pot)
struct PPConst {
  float cut, a2, cut2, a, binScale, taperScale;
  __device__ __forceinline__ explicit PPConst(const ccs_uniforms &u)
      : cut(u.cut), a2(u.a2), cut2(xmul(u.cut, u.cut)), a(fsqrt(u.a2)), binScale(fdiv(64.0f, u.cut)),
        taperScale(fdiv(1.0f, 0.8f * u.cut - u.cut)) {}
};
__device__ __forceinline__ void pp_pair(const PPConst &c, float4 P, float myBox, float4 Q, float qBox,
                                        const float2 *stab, f3 &acc, float &pot) {
  const f3 d = xsub3(xyz(Q), xyz(P));
  const float r2 = xdot(d, d);
  if (r2 >= c.cut2) return;
  const float r = fsqrt(r2);
  const float xx = clampf(r * c.binScale - 0.5f, 0.0f, 63.0f);
  const int k = (int)xx, k1 = min(k + 1, 63);
  const float tt = xx - (float)k;
  const float invN = rsqrtf(r2 + c.a2);
  const float ts = clampf((r - c.cut) * c.taperScale, 0.0f, 1.0f);
  const float taper = ts * ts * (3.0f - 2.0f * ts);
  const float same = (myBox >= 0.0f && qBox == myBox) ? 1.0f : 0.0f;
  const float2 ta = stab[k], tb = stab[k1];
  const float Tx = (ta.x + (tb.x - ta.x) * tt) * same;
  const float Ty = (ta.y + (tb.y - ta.y) * tt) * same;
  const float fn = invN * invN * invN * r - fdiv(Tx, fmaxf(r2, c.a2));
  const float mj = Q.w;
  acc = acc + d * (fdiv(1.0f, fmaxf(r, 1e-6f)) * mj * fn * taper);
  pot += mj * (-invN - fdiv(Ty, fmaxf(r, c.a))) * taper;
}

// a persistent grid over (seat tile, quarter, chunk) work items, counted from the list's length on the
// device, so a captured launch serves any length
__global__ void __launch_bounds__(kPPI) k_pp_pairs(const ccs_uniforms *__restrict__ U,
                                                   const float4 *__restrict__ list, const float *__restrict__ box,
                                                   int cap, const float2 *__restrict__ tab,
                                                   float4 *__restrict__ part) {
  __shared__ float4 sq[kPPJ];
  __shared__ float sb[kPPJ];
  __shared__ float2 stab[CCS_PP_BINS];
  const ccs_uniforms &u = *U;
  const int count = u.ppCount;
  const int share = (count + 3) >> 2;
  const int jw = pp_chunk_width(share);
  const int nCh = share > 0 ? (share + jw - 1) / jw : 0;
  const int items = (count + kPPI - 1) / kPPI * 4 * nCh;
  if (threadIdx.x < CCS_PP_BINS) stab[threadIdx.x] = tab[threadIdx.x];
  const PPConst c(u);
  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int tile = item / (4 * nCh), rest = item % (4 * nCh);
    const int slice = rest / nCh, chunk = rest % nCh;
    const int s0 = slice * share, s1 = min(s0 + share, count);
    const int j0 = s0 + chunk * jw, j1 = min(j0 + jw, s1);
    if (j0 >= j1) continue;   // past the end of a short last quarter: never read by the reduction
    const int me = tile * kPPI + threadIdx.x;
    __syncthreads();   // the previous item's reads of the chunk are done
    if (j0 + (int)threadIdx.x < j1) {
      sq[threadIdx.x] = list[j0 + threadIdx.x];
      sb[threadIdx.x] = box[j0 + threadIdx.x];
    }
    __syncthreads();
    const float4 P = me < count ? list[me] : make_float4(0, 0, 0, 0);
    const bool active = me < count && P.w != 0.0f;
    const float myBox = me < count ? box[me] : -1.0f;
    f3 acc = mk(0, 0, 0);
    float pot = 0.0f;
    if (active) {
      const int n = j1 - j0;
#pragma unroll 4
      for (int jj = 0; jj < n; ++jj) {
        if (j0 + jj == me) continue;
        pp_pair(c, P, myBox, sq[jj], sb[jj], stab, acc, pot);
      }
    }
    if (me < count) part[((size_t)slice * kMaxChunks + chunk) * cap + me] = make_float4(acc.x, acc.y, acc.z, pot);
  }
}

__global__ void __launch_bounds__(kBlock) k_pp_reduce(const ccs_uniforms *__restrict__ U,
                                                      const float4 *__restrict__ list,
                                                      const float4 *__restrict__ part, int cap,
                                                      float4 *__restrict__ force) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  const int slice = blockIdx.y;
  const ccs_uniforms &u = *U;
  const int count = u.ppCount;
  if (me >= count) return;   // only the list's seats are ever read
  float4 o = make_float4(0, 0, 0, 0);
  if (list[me].w != 0.0f) {
    const int share = (count + 3) >> 2;
    const int jw = pp_chunk_width(share);
    const int s0 = slice * share, s1 = min(s0 + share, count);
    const int nChunks = s1 > s0 ? (s1 - s0 + jw - 1) / jw : 0;
    for (int c = 0; c < nChunks; ++c) {
      const float4 v = part[((size_t)slice * kMaxChunks + c) * cap + me];
      o.x += v.x; o.y += v.y; o.z += v.z; o.w += v.w;
    }
    o = make_float4(o.x * u.Gm, o.y * u.Gm, o.z * u.Gm, o.w * u.Gm);
  }
  force[(size_t)slice * cap + me] = o;
}

// the same correction over a list of any length (the reference caps it at 8,192): one thread a member, the
// whole list staged kPPJ entries at a time and walked in list order, so no partial sums are kept; out[s] is
// Gm x (pull, potential), the four slices of the capped pass in one
__global__ void __launch_bounds__(kPPI) k_pp_list(const ccs_uniforms u, const float4 *__restrict__ list,
                                                  const float *__restrict__ box, int n,
                                                  const float2 *__restrict__ tab, float4 *__restrict__ out) {
  __shared__ float4 sq[kPPJ];
  __shared__ float sb[kPPJ];
  __shared__ float2 stab[CCS_PP_BINS];
  if (threadIdx.x < CCS_PP_BINS) stab[threadIdx.x] = tab[threadIdx.x];
  const PPConst c(u);
  const int me = blockIdx.x * kPPI + threadIdx.x;
  const float4 P = me < n ? list[me] : make_float4(0, 0, 0, 0);
  const bool active = me < n && P.w != 0.0f;
  const float myBox = me < n ? box[me] : -1.0f;
  f3 acc = mk(0, 0, 0);
  float pot = 0.0f;
  for (int j0 = 0; j0 < n; j0 += kPPJ) {
    __syncthreads();   // the previous chunk's reads are done
    if (j0 + (int)threadIdx.x < n) {
      sq[threadIdx.x] = list[j0 + threadIdx.x];
      sb[threadIdx.x] = box[j0 + threadIdx.x];
    }
    __syncthreads();
    if (active) {
      const int m = min(kPPJ, n - j0);
#pragma unroll 4
      for (int jj = 0; jj < m; ++jj) {
        if (j0 + jj == me) continue;
        pp_pair(c, P, myBox, sq[jj], sb[jj], stab, acc, pot);
      }
    }
  }
  if (me < n) out[me] = active ? make_float4(acc.x * u.Gm, acc.y * u.Gm, acc.z * u.Gm, pot * u.Gm)
                               : make_float4(0, 0, 0, 0);
}

int launch_pp_list(const ccs_uniforms &u, const float4 *list, const float *box, int n, const float2 *tab,
                   float4 *out, cudaStream_t st) {
  if (n <= 0) return 0;
  k_pp_list<<<(n + kPPI - 1) / kPPI, kPPI, 0, st>>>(u, list, box, n, tab, out);
  return 1;
}

int launch_pp_force(const ccs_uniforms *u, const float4 *list, const float *box, int cap, const float2 *tab,
                    float4 *part, float4 *force, cudaStream_t st) {
  const int sms = sm_count();
  // enough CTAs for a full list's items to take a few rounds; a short list's take one
  const int full = (cap + kPPI - 1) / kPPI * 4 * kMaxChunks;
  k_pp_pairs<<<std::min(full, sms * 8), kPPI, 0, st>>>(u, list, box, cap, tab, part);
  dim3 g2(blocks_for(cap), 4);
  k_pp_reduce<<<g2, kBlock, 0, st>>>(u, list, part, cap, force);
  return 2;
}

}  // namespace ccs

// ---------------------------------------------------------------------------
// The pairwise pass without allocation: ccs_pp_force_static.
//
// Some callers cannot call cudaMalloc at the point they need this pass: a
// host that runs the step inside a device-memory budget owned by someone
// else (a JavaScript or game engine's arena, a framework's caching pool),
// code that must not trigger the device-wide synchronisation cudaMalloc and
// cudaFree imply, or a loop that may not fail on an out-of-memory halfway
// through a frame.  They hand over the list, the boxes, the table and the
// output in memory they already own; the pass's only scratch -- the partial
// sums of the 2-D tiling -- lives here, in a file-scope device array sized for
// lists of up to CCS_PP_STATIC_MAX entries (2 MiB, held by every GPU that
// loads the library until the process exits).  Its uniforms live in a second
// static device struct, written on the caller's stream by a one-thread kernel
// that takes them by value (no host staging buffer, pageable or pinned, is
// read by the GPU).  Every call shares both: two calls that overlap on the GPU
// (different streams, or another thread) race and must be ordered by the
// caller.  Nothing in the scratch has to start at zero -- every partial the
// reduction reads is written earlier in the same call.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {
constexpr int kStaticMaxDevices = 64;
constexpr size_t kStaticScratch = (size_t)4 * ccs::kMaxChunks * CCS_PP_STATIC_MAX;   // float4 partials: 2 MiB
}  // namespace

static __device__ __align__(256) float4 g_pp_scratch[kStaticScratch];
static __device__ __align__(256) ccs_uniforms g_pp_uniforms;

namespace {
// the call's uniforms into the static struct, in stream order before the pass that reads them (device code
// names the array itself; only host code needs its looked-up address)
__global__ void k_pp_static_uniforms(const ccs_uniforms u) { g_pp_uniforms = u; }

std::mutex g_pp_static_mutex;
float4 *g_pp_scratch_at[kStaticMaxDevices] = {};
ccs_uniforms *g_pp_uniforms_at[kStaticMaxDevices] = {};
}  // namespace

extern "C" int ccs_pp_force_static(const float *list4, const float *box, int n, const float *tab2, float cut,
                                   float a2, float gm, float *force4, void *stream) {
  if (n < 0 || (n > 0 && (!list4 || !box || !tab2 || !force4))) return CCS_E_ARG;
  if (n > CCS_PP_STATIC_MAX) return CCS_E_RANGE;
  if (n == 0) return CCS_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kStaticMaxDevices) return CCS_E_CUDA;
  {
    // set-up, once per device, with that device current: the arrays' device addresses (in host code
    // their names stand for host-side shadows, never for device memory)
    std::lock_guard<std::mutex> lock(g_pp_static_mutex);
    if (!g_pp_scratch_at[dev]) {
      void *s = nullptr, *u = nullptr;
      if (cudaGetSymbolAddress(&s, g_pp_scratch) != cudaSuccess || !s) return CCS_E_CUDA;
      if (cudaGetSymbolAddress(&u, g_pp_uniforms) != cudaSuccess || !u) return CCS_E_CUDA;
      g_pp_uniforms_at[dev] = static_cast<ccs_uniforms *>(u);
      g_pp_scratch_at[dev] = static_cast<float4 *>(s);
    }
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ccs_uniforms u{};
  u.cut = cut;
  u.a2 = a2;
  u.Gm = gm;
  u.ppCount = n;
  k_pp_static_uniforms<<<1, 1, 0, st>>>(u);
  ccs::launch_pp_force(g_pp_uniforms_at[dev], reinterpret_cast<const float4 *>(list4), box, n,
                       reinterpret_cast<const float2 *>(tab2), g_pp_scratch_at[dev],
                       reinterpret_cast<float4 *>(force4), st);
  return cudaGetLastError() == cudaSuccess ? CCS_OK : CCS_E_CUDA;
}
