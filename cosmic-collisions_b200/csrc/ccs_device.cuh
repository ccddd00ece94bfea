// ccs_device.cuh -- device-side helpers shared by the step kernels.
//
// Two kinds of arithmetic live side by side:
//  * exact -- every operation that decides an integer outcome (a particle's
//    cell, its seat word, the seat and cell culls, the contact test, the box a
//    particle reads, a pair inside or beyond the P3M cut) is written with the
//    _rn intrinsics, which are never fused, so it rounds once per operation in
//    the order the reference's GLSL is written: dot(a,b) = (a.x*b.x +
//    a.y*b.y) + a.z*b.z.  These outcomes match the CPU oracle bit for bit.
//  * fast -- forces, heat and potentials use FMA, rsqrtf and __fdividef; they
//    match the oracle to tolerance (1e-5 of the field's scale).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "ccs_internal.h"

namespace ccs {

struct f3 { float x, y, z; };
__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ f3 ld3(const float *p) { return {p[0], p[1], p[2]}; }
// fast (fusable) vector arithmetic
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ float fsqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
// exact (never fused, IEEE round-to-nearest) arithmetic
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ f3 xsub3(f3 a, f3 b) { return {xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z)}; }
__device__ __forceinline__ float xdot(f3 a, f3 b) {
  return xadd(xadd(xmul(a.x, b.x), xmul(a.y, b.y)), xmul(a.z, b.z));
}
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
// GLSL mod(x, 4.0) < 0.5 for a material tag: exact (division by 4 is a power of two)
__device__ __forceinline__ bool is_iron(float tag) {
  return xsub(tag, xmul(4.0f, floorf(xmul(tag, 0.25f)))) < 0.5f;
}

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

// the contact cell of a position: floor(p * uInvCell), exact
__device__ __forceinline__ void cell_of(const ccs_uniforms &u, f3 p, float &gx, float &gy, float &gz, int &cx,
                                        int &cy, int &cz) {
  gx = xmul(p.x, u.invCell);
  gy = xmul(p.y, u.invCell);
  gz = xmul(p.z, u.invCell);
  cx = (int)floorf(gx);
  cy = (int)floorf(gy);
  cz = (int)floorf(gz);
}

// boxOf of src/glsl-sim.js:29-36, exact: it decides which mesh a particle reads
__device__ __forceinline__ int box_of(const ccs_uniforms &u, f3 p, f3 &g) {
  const f3 gA = mk(xsub(xmul(xadd(p.x, u.LA[0]), u.invH), 0.5f), xsub(xmul(xadd(p.y, u.LA[1]), u.invH), 0.5f),
                   xsub(xmul(xadd(p.z, u.LA[2]), u.invH), 0.5f));
  const f3 gB = mk(xsub(xmul(xadd(p.x, u.LB[0]), u.invH), 0.5f), xsub(xmul(xadd(p.y, u.LB[1]), u.invH), 0.5f),
                   xsub(xmul(xadd(p.z, u.LB[2]), u.invH), 0.5f));
  bool inA = gA.x >= 0.0f && gA.y >= 0.0f && gA.z >= 0.0f && gA.x <= 63.0f && gA.y <= 63.0f && gA.z <= 63.0f;
  bool inB = u.boxB > 0.5f && gB.x >= 0.0f && gB.y >= 0.0f && gB.z >= 0.0f && gB.x <= 63.0f && gB.y <= 63.0f &&
             gB.z <= 63.0f;
  if (inA && inB) {
    const float dA = fmaxf(fabsf(xsub(gA.x, 31.5f)), fmaxf(fabsf(xsub(gA.y, 31.5f)), fabsf(xsub(gA.z, 31.5f))));
    const float dB = fmaxf(fabsf(xsub(gB.x, 31.5f)), fmaxf(fabsf(xsub(gB.y, 31.5f)), fabsf(xsub(gB.z, 31.5f))));
    inA = dA <= dB;
    inB = !inA;
  }
  g = inA ? gA : gB;
  return inA ? 0 : inB ? 1 : -1;
}

// GLSL_MASS of src/glsl-sim.js:57-66 (fast)
__device__ __forceinline__ f3 mass_at(const ccs_uniforms &u, f3 p, float4 mono) {
  const float iw = fdiv(1.0f, fmaxf(mono.w, 1e-6f));
  const f3 r = xyz(mono) * iw - p;
  const float inv = rsqrtf(dot(r, r) + u.eps2Mesh);
  return r * (u.Gm * mono.w * inv * inv * inv);
}
__device__ __forceinline__ float pot_at(const ccs_uniforms &u, f3 p, float4 mono) {
  const float iw = fdiv(1.0f, fmaxf(mono.w, 1e-6f));
  const f3 r = xyz(mono) * iw - p;
  return -u.Gm * mono.w * rsqrtf(dot(r, r) + u.eps2Mesh);
}
__device__ __forceinline__ f3 cross_at(const ccs_uniforms &u, float4 other, float4 mine) {
  const f3 d = xyz(other) * fdiv(1.0f, fmaxf(other.w, 1e-6f)) - xyz(mine) * fdiv(1.0f, fmaxf(mine.w, 1e-6f));
  const float inv = rsqrtf(dot(d, d) + u.eps2Mesh);
  return d * (u.Gm * other.w * inv * inv * inv);
}

}  // namespace ccs
