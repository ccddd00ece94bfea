// ccs_device.cuh -- device-side helpers shared by the step kernels.
//
// Float semantics: this library is compiled with -fmad=false and IEEE divide
// and square root, so every expression below rounds once per operation in the
// order written -- the GLSL expressions of src/glsl-sim.js evaluated left to
// right.  dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z and inversesqrt(x) =
// 1/sqrt(x), both correctly rounded.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "ccs_internal.h"

namespace ccs {

struct f3 { float x, y, z; };
__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ f3 ld3(const float *p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ float isqrt(float x) { return 1.0f / sqrtf(x); }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float modg(float x, float y) { return x - y * floorf(x / y); }  // GLSL mod

__device__ __forceinline__ int fine_index(int x, int y, int z) { return (z * 64 + y) * 64 + x; }
__device__ __forceinline__ int coarse_index(int x, int y, int z) { return (z * 16 + y) * 16 + x; }

// hashAt of src/glsl-sim.js:84-90: the wrap-skewed hash of a contact cell,
// returned as the atlas texel's linear index ay * AW + ax.
__device__ __forceinline__ uint32_t hash_cell(const ccs_uniforms &u, int cx, int cy, int cz) {
  const int s = u.GShift;
  const int px = cx >> s, py = cy >> s, pz = cz >> s;  // arithmetic: the wrap period
  uint32_t y = (uint32_t)cy + ((uint32_t)px << (s - 1)) + ((uint32_t)pz << (s - 2));
  uint32_t z = (uint32_t)cz + ((uint32_t)py << (s - 1));
  const uint32_t m = (uint32_t)u.GMask;
  const uint32_t x = (uint32_t)cx & m;
  y &= m;
  z &= m;
  const uint32_t ax = ((z & (uint32_t)u.SXMask) << s) + x;
  const uint32_t ay = ((z >> u.SXShift) << s) + y;
  return ay * (uint32_t)u.AW + ax;
}

// boxOf of src/glsl-sim.js:29-36
__device__ __forceinline__ int box_of(const ccs_uniforms &u, f3 p, f3 &g) {
  const f3 gA = mk((p.x + u.LA[0]) * u.invH - 0.5f, (p.y + u.LA[1]) * u.invH - 0.5f, (p.z + u.LA[2]) * u.invH - 0.5f);
  const f3 gB = mk((p.x + u.LB[0]) * u.invH - 0.5f, (p.y + u.LB[1]) * u.invH - 0.5f, (p.z + u.LB[2]) * u.invH - 0.5f);
  bool inA = gA.x >= 0.0f && gA.y >= 0.0f && gA.z >= 0.0f && gA.x <= 63.0f && gA.y <= 63.0f && gA.z <= 63.0f;
  bool inB = u.boxB > 0.5f && gB.x >= 0.0f && gB.y >= 0.0f && gB.z >= 0.0f && gB.x <= 63.0f && gB.y <= 63.0f &&
             gB.z <= 63.0f;
  if (inA && inB) {
    const float dA = fmaxf(fabsf(gA.x - 31.5f), fmaxf(fabsf(gA.y - 31.5f), fabsf(gA.z - 31.5f)));
    const float dB = fmaxf(fabsf(gB.x - 31.5f), fmaxf(fabsf(gB.y - 31.5f), fabsf(gB.z - 31.5f)));
    inA = dA <= dB;
    inB = !inA;
  }
  g = inA ? gA : gB;
  return inA ? 0 : inB ? 1 : -1;
}

// GLSL_MASS of src/glsl-sim.js:57-66
__device__ __forceinline__ f3 mass_at(const ccs_uniforms &u, f3 p, float4 mono) {
  const f3 r = xyz(mono) / fmaxf(mono.w, 1e-6f) - p;
  const float inv = isqrt(dot(r, r) + u.eps2Mesh);
  return r * (u.Gm * mono.w * inv * inv * inv);
}
__device__ __forceinline__ float pot_at(const ccs_uniforms &u, f3 p, float4 mono) {
  const f3 r = xyz(mono) / fmaxf(mono.w, 1e-6f) - p;
  return -u.Gm * mono.w * isqrt(dot(r, r) + u.eps2Mesh);
}
__device__ __forceinline__ f3 cross_at(const ccs_uniforms &u, float4 other, float4 mine) {
  const f3 d = xyz(other) / fmaxf(other.w, 1e-6f) - xyz(mine) / fmaxf(mine.w, 1e-6f);
  const float inv = isqrt(dot(d, d) + u.eps2Mesh);
  return d * (u.Gm * other.w * inv * inv * inv);
}

}  // namespace ccs
