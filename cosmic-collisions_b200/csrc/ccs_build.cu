// ccs_build.cu -- the builder's overlap relaxation on the device.
//
// relax() of src/bodies.js:97-146: a pile of particles laid in Fibonacci
// shells is relaxed, with no inertia, by pushing every pair closer than
// 0.96 diameters apart by half its overlap, sweep after sweep over a cell
// grid of side 2.2 radii that is rebuilt every fourth sweep, each particle
// held inside the body's spheroid.  The reference sweeps the particles one by
// one in index order (Gauss-Seidel): a particle moves its later neighbours at
// once.  Here a sweep is 27 phases, one for each class of cells with the
// same coordinates modulo 3; within a phase every cell of the class is one
// thread, which walks its particles in index order exactly as the reference
// walks them.  Two cells of a class are three apart on some axis, so the
// particles one thread reads and moves (its own cell and the 26 around it)
// are never another's in the same phase: the sweep is race-free and
// deterministic.  Every pair is still pushed once a sweep, from the cell of
// its lower index, in binary64 with binary32 storage as the reference does;
// only the order in which the pushes happen differs, so the pile comes out
// equivalent (the same overlap statistics), not bit-identical.
#include <cmath>
#include <vector>

#include "ccs_device.cuh"
#include "ccs_internal.h"

namespace ccs {
namespace {

constexpr int kBlock = 256;
constexpr int kSweeps = 10, kRegrid = 4;   // RELAX_SWEEPS, RELAX_REGRID of src/bodies.js:97

struct RelaxGrid {
  double lo[3], cs;
  int g[3];   // cells along x, y, z; a cell is (x * gy + y) * gz + z
};

__device__ __forceinline__ int relax_axis(double v, const RelaxGrid &G, int k) {
  const double c = floor((v - G.lo[k]) / G.cs) + 1.0;
  return (int)fmin(fmax(c, 0.0), (double)(G.g[k] - 1));
}

__global__ void k_relax_cells(int n, const float *__restrict__ p, RelaxGrid G, uint32_t *__restrict__ keys,
                              int32_t *__restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int cx = relax_axis(p[3 * i], G, 0), cy = relax_axis(p[3 * i + 1], G, 1), cz = relax_axis(p[3 * i + 2], G, 2);
  keys[i] = (uint32_t)((cx * G.g[1] + cy) * G.g[2] + cz);
  vals[i] = i;
}

// where each cell's particles start and end in the sorted order (start = -1: an empty cell)
__global__ void k_relax_ranges(int n, const uint32_t *__restrict__ keys, int *__restrict__ start,
                               int *__restrict__ end) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t k = keys[s];
  if (s == 0 || keys[s - 1] != k) start[k] = s;
  if (s == n - 1 || keys[s + 1] != k) end[k] = s + 1;
}

// one phase: every cell whose coordinates are (r0, r1, r2) modulo 3, a thread each
__global__ void k_relax_phase(int r0, int r1, int r2, RelaxGrid G, float *p, const int32_t *__restrict__ order,
                              const int *__restrict__ start, const int *__restrict__ end, double D, double iA2,
                              double iC2) {
  const int nx = (G.g[0] - r0 + 2) / 3, ny = (G.g[1] - r1 + 2) / 3, nz = (G.g[2] - r2 + 2) / 3;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * ny * nz) return;
  const int cx = r0 + 3 * (t / (ny * nz)), cy = r1 + 3 * ((t / nz) % ny), cz = r2 + 3 * (t % nz);
  const int nc = G.g[0] * G.g[1] * G.g[2], gyz = G.g[1] * G.g[2];
  const int cell = (cx * G.g[1] + cy) * G.g[2] + cz;
  const int b = start[cell];
  if (b < 0) return;
  const int e = end[cell];
  const double D2 = D * D;
  for (int si = b; si < e; ++si) {
    const int i = order[si];
    double x = p[3 * i], y = p[3 * i + 1], z = p[3 * i + 2];
    for (int o = 0; o < 27; ++o) {   // the reference's offset order
      const int cc = cell + (o % 3 - 1) * gyz + ((o / 3) % 3 - 1) * G.g[2] + (o / 9 - 1);
      if (cc < 0 || cc >= nc) continue;
      const int bs = start[cc];
      if (bs < 0) continue;
      const int es = end[cc];
      for (int s = bs; s < es; ++s) {
        const int j = order[s];
        if (j <= i) continue;
        double dx = (double)p[3 * j] - x, dy = (double)p[3 * j + 1] - y, dz = (double)p[3 * j + 2] - z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 >= D2) continue;
        double d = sqrt(d2);
        if (d == 0.0) d = 1e-9;
        const double mv = 0.5 * (D - d) / d;
        dx *= mv;
        dy *= mv;
        dz *= mv;
        x -= dx;
        y -= dy;
        z -= dz;
        p[3 * j] = (float)((double)p[3 * j] + dx);
        p[3 * j + 1] = (float)((double)p[3 * j + 1] + dy);
        p[3 * j + 2] = (float)((double)p[3 * j + 2] + dz);
      }
    }
    const double qq = (x * x + z * z) * iA2 + y * y * iC2;   // held inside the body's own spheroid
    if (qq > 1.0) {
      const double f = 1.0 / sqrt(qq);
      x *= f;
      y *= f;
      z *= f;
    }
    p[3 * i] = (float)x;
    p[3 * i + 1] = (float)y;
    p[3 * i + 2] = (float)z;
  }
}

inline int grid_for(long n) { return (int)((n + kBlock - 1) / kBlock); }

}  // namespace

int relax_device(int device, float *p, int n, double a, double A, double C, std::string *err) {
  if (cudaSetDevice(device) != cudaSuccess) {
    if (err) *err = "relax: no such device";
    return CCS_E_CUDA;
  }
  const double D = 2 * a * 0.96, cs = 2.2 * a;
  RelaxGrid G;
  double hi[3] = {-1e9, -1e9, -1e9};
  for (int k = 0; k < 3; ++k) G.lo[k] = 1e9;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      const double v = p[3 * i + k];
      G.lo[k] = v < G.lo[k] ? v : G.lo[k];
      hi[k] = v > hi[k] ? v : hi[k];
    }
  G.cs = cs;
  for (int k = 0; k < 3; ++k) G.g[k] = (int)std::floor((hi[k] - G.lo[k]) / cs) + 3;
  const long nc = (long)G.g[0] * G.g[1] * G.g[2];
  int bits = 1;
  while ((1L << bits) < nc) ++bits;
  if (bits > 30) {
    if (err) *err = "relax: the pile's cell grid is too large";
    return CCS_E_RANGE;
  }
  float *dp = nullptr;
  uint32_t *keys = nullptr, *keysTmp = nullptr, *hist = nullptr;
  int32_t *vals = nullptr, *valsTmp = nullptr;
  int *start = nullptr, *end = nullptr;
  cudaStream_t st = nullptr;
  auto release = [&] {
    cudaFree(dp); cudaFree(keys); cudaFree(keysTmp); cudaFree(hist); cudaFree(vals); cudaFree(valsTmp);
    cudaFree(start); cudaFree(end);
    if (st) cudaStreamDestroy(st);
  };
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&dp, sizeof(float) * 3 * (size_t)n) != cudaSuccess ||
      cudaMalloc(&keys, 4 * (size_t)n) != cudaSuccess || cudaMalloc(&keysTmp, 4 * (size_t)n) != cudaSuccess ||
      cudaMalloc(&vals, 4 * (size_t)n) != cudaSuccess || cudaMalloc(&valsTmp, 4 * (size_t)n) != cudaSuccess ||
      cudaMalloc(&hist, 4 * radix_hist_words(n)) != cudaSuccess ||
      cudaMalloc(&start, sizeof(int) * (size_t)nc) != cudaSuccess ||
      cudaMalloc(&end, sizeof(int) * (size_t)nc) != cudaSuccess) {
    release();
    if (err) *err = "relax: device allocation failed";
    return CCS_E_NOMEM;
  }
  cudaMemcpyAsync(dp, p, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, st);
  const double iA2 = 1 / (A * A), iC2 = 1 / (C * C);
  for (int sweep = 0; sweep < kSweeps; ++sweep) {
    if (sweep % kRegrid == 0) {   // the pile barely moves: the grid keeps for four sweeps
      k_relax_cells<<<grid_for(n), kBlock, 0, st>>>(n, dp, G, keys, vals);
      launch_radix_sort(n, bits, keys, vals, keysTmp, valsTmp, hist, st);
      cudaMemsetAsync(start, 0xFF, sizeof(int) * (size_t)nc, st);
      k_relax_ranges<<<grid_for(n), kBlock, 0, st>>>(n, keys, start, end);
    }
    for (int r = 0; r < 27; ++r) {
      const int r0 = r % 3, r1 = (r / 3) % 3, r2 = r / 9;
      const long cells = (long)((G.g[0] - r0 + 2) / 3) * ((G.g[1] - r1 + 2) / 3) * ((G.g[2] - r2 + 2) / 3);
      k_relax_phase<<<grid_for(cells), kBlock, 0, st>>>(r0, r1, r2, G, dp, vals, start, end, D, iA2, iC2);
    }
  }
  cudaMemcpyAsync(p, dp, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToHost, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  const cudaError_t l = cudaGetLastError();
  release();
  if (e != cudaSuccess || l != cudaSuccess) {
    if (err) *err = std::string("relax: ") + cudaGetErrorString(e != cudaSuccess ? e : l);
    return CCS_E_CUDA;
  }
  return CCS_OK;
}

}  // namespace ccs
