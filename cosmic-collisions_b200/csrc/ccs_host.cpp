// ccs_host.cpp -- the CPU side of the engine: the body builder, the mesh
// pair table and the friends-of-friends analysis.
//
// These are the reference's JavaScript routines (binary64 arithmetic, results
// stored to Float32Array) restated in C++ so that a host without a JS engine
// can build a run and read its books:
//   mulberry32          src/math.js:8-15
//   maclaurin, turn     src/bodies.js:152-169
//   ball, relax         src/bodies.js:23-146
//   build               src/nbody.js:114-250
//   approachTime        src/nbody.js:578-590
//   meshPairTable       src/nbody.js:56-108
//   fof                 src/nbody.js:646-893
// Compiled with -ffp-contract=off so every binary64 operation rounds once, in
// the order the JavaScript evaluates it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ccstep.h"

namespace ccs {
// the same relaxation on a GPU (ccs_build.cu)
int relax_device(int device, float *p, int n, double a, double A, double C, std::string *err);
}  // namespace ccs

namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kFL = 6.0, kFH = 2.0 * kFL / 64.0;
constexpr double kJam = 0.96, kEkg = 6.256e7, kCpRock = 1200.0;

// mulberry32: the seeded random of src/math.js:8-15
struct Mulberry {
  uint32_t s;
  explicit Mulberry(uint32_t seed) : s(seed) {}
  double operator()() {
    s += 0x6D2B79F5u;
    uint32_t t = (s ^ (s >> 15)) * (1u | s);
    t = (t + (t ^ (t >> 7)) * (61u | t)) ^ t;
    return (double)(t ^ (t >> 14)) / 4294967296.0;
  }
};

// JavaScript's Math.round: halves go up
double js_round(double x) {
  const double f = std::floor(x);
  return x - f >= 0.5 ? f + 1.0 : f;
}

double maclaurin_rhs(double e) {
  const double s2 = 1 - e * e;
  return 2 * std::sqrt(s2) / (e * e * e) * (3 - 2 * e * e) * std::asin(e) - 6 * s2 / (e * e);
}

// the Maclaurin spheroid's eccentricity for a spin of f of breakup
double maclaurin(double f) {
  const double want = 4.0 / 3.0 * f * f;
  if (want < 1e-6) return 0;
  double lo = 0.01, hi = 0.93;
  if (want >= maclaurin_rhs(hi)) return hi;
  for (int i = 0; i < 60; ++i) {
    const double m = 0.5 * (lo + hi);
    (maclaurin_rhs(m) < want ? lo : hi) = m;
  }
  return 0.5 * (lo + hi);
}

// overlap removal sweeps, src/bodies.js:97-146 (confine = the body's spheroid)
void relax(std::vector<float> &p, int n, double a, double A, double C) {
  const int sweeps = 10;
  const double D = 2 * a * 0.96, cs = 2.2 * a, iA2 = 1 / (A * A), iC2 = 1 / (C * C);
  double lo[3] = {1e9, 1e9, 1e9}, hi[3] = {-1e9, -1e9, -1e9};
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      const double v = p[3 * i + k];
      lo[k] = v < lo[k] ? v : lo[k];
      hi[k] = v > hi[k] ? v : hi[k];
    }
  const int gx = (int)std::floor((hi[0] - lo[0]) / cs) + 3;
  const int gy = (int)std::floor((hi[1] - lo[1]) / cs) + 3;
  const int gz = (int)std::floor((hi[2] - lo[2]) / cs) + 3;
  const int nc = gx * gy * gz;
  std::vector<int> start(nc + 1), order(n), cell(n);
  auto axis = [&](double v, int k, int g) {
    const double c = std::floor((v - lo[k]) / cs) + 1;
    return (int)std::min(std::max(c, 0.0), (double)(g - 1));
  };
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    if (sweep % 4 == 0) {   // the pile barely moves: the grid keeps for four sweeps
      std::fill(start.begin(), start.end(), 0);
      for (int i = 0; i < n; ++i) {
        cell[i] = (axis(p[3 * i], 0, gx) * gy + axis(p[3 * i + 1], 1, gy)) * gz + axis(p[3 * i + 2], 2, gz);
        start[cell[i] + 1]++;
      }
      for (int k = 0; k < nc; ++k) start[k + 1] += start[k];
      for (int i = 0; i < n; ++i) order[start[cell[i]]++] = i;
      for (int k = nc; k > 0; --k) start[k] = start[k - 1];
      start[0] = 0;
    }
    for (int i = 0; i < n; ++i) {
      double x = p[3 * i], y = p[3 * i + 1], z = p[3 * i + 2];
      for (int o = 0; o < 27; ++o) {
        const int cc = cell[i] + (o % 3 - 1) * gy * gz + ((o / 3) % 3 - 1) * gz + (o / 9 - 1);
        if (cc < 0 || cc >= nc) continue;
        for (int s = start[cc]; s < start[cc + 1]; ++s) {
          const int j = order[s];
          if (j <= i) continue;
          double dx = p[3 * j] - x, dy = p[3 * j + 1] - y, dz = p[3 * j + 2] - z;
          const double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 >= D * D) continue;
          double d = std::sqrt(d2);
          if (d == 0) d = 1e-9;
          const double mv = 0.5 * (D - d) / d;
          dx *= mv; dy *= mv; dz *= mv;
          x -= dx; y -= dy; z -= dz;
          p[3 * j] = (float)(p[3 * j] + dx);
          p[3 * j + 1] = (float)(p[3 * j + 1] + dy);
          p[3 * j + 2] = (float)(p[3 * j + 2] + dz);
        }
      }
      const double qq = (x * x + z * z) * iA2 + y * y * iC2;
      if (qq > 1.0) {
        const double f = 1 / std::sqrt(qq);
        x *= f; y *= f; z *= f;
      }
      p[3 * i] = (float)x; p[3 * i + 1] = (float)y; p[3 * i + 2] = (float)z;
    }
  }
}

// the onion of Fibonacci shells, src/bodies.js:23-76; returns the shell
// bounds (ascending, 0 .. n)
std::vector<int> ball(int n, double s, double a, Mulberry &rng, double e, std::vector<float> &out, int device,
                      int *rc) {
  constexpr int NB = 256;
  const double R = std::cbrt(3 * n * s * s * s / (16 * kPi));
  const double ae = R / std::pow(1 - e * e, 1.0 / 6), ce = ae * std::sqrt(1 - e * e);
  const double vp = s * s * s / 4, unit = 3 * vp / (4 * kPi), jit = 0.06 * s;
  double h = s * std::sqrt(1.0 / 3);
  const int K = std::max(1, (int)js_round(ce / h));
  const double GA = kPi * (3 - std::sqrt(5.0));
  h = ce / K;
  struct Shell { double A, C, want; std::vector<double> cum; };
  std::vector<Shell> shells;
  double total = 0;
  int kept = 0;
  for (int j = 0; j < K; ++j) {
    const double A = ae - j * h, C = ce - j * h;
    if (C - h * 0.5 < h) break;
    Shell sh;
    sh.A = A - h * 0.5;
    sh.C = C - h * 0.5;
    sh.cum.assign(NB + 1, 0.0);
    for (int b = 0; b < NB; ++b) {
      const double be = (b + 0.5) * kPi / NB - kPi / 2, cb = std::cos(be), sb = std::sin(be);
      sh.cum[b + 1] = sh.cum[b] + sh.A * cb * std::sqrt(sh.C * sh.C * cb * cb + sh.A * sh.A * sb * sb);
    }
    sh.want = (A * A * C - (A - h) * (A - h) * (C - h)) / unit;
    total += sh.want;
    shells.push_back(std::move(sh));
    kept = j + 1;
  }
  const double As = ae - kept * h, Cs = ce - kept * h;
  total += std::max(As * As * Cs, 0.0) / unit;
  out.assign((size_t)3 * n, 0.0f);
  std::vector<int> bounds{n};
  int i = n;
  double acc = 0;
  for (const Shell &sh : shells) {
    acc += sh.want * n / total;
    const int m = (int)std::min(std::min(js_round(acc), (double)n) - (n - i), (double)i);
    const int lo = i - m;
    const double phi0 = rng() * 2 * kPi;
    const double flip = rng() < 0.5 ? -1 : 1;
    int bb = 0;
    for (int q = 0; q < m; ++q) {
      const double u = (q + 0.5) / m * sh.cum[NB];
      while (bb < NB - 1 && sh.cum[bb + 1] < u) ++bb;
      const double lat = (bb + (u - sh.cum[bb]) / (sh.cum[bb + 1] - sh.cum[bb])) * kPi / NB - kPi / 2;
      const double phi = phi0 + q * GA, rc = sh.A * std::cos(lat);
      float *o = &out[(size_t)3 * (lo + q)];
      const double x = rc * std::cos(phi);
      o[0] = (float)(x + (rng() - 0.5) * jit);
      const double y = flip * sh.C * std::sin(lat);
      o[1] = (float)(y + (rng() - 0.5) * jit);
      const double z = rc * std::sin(phi);
      o[2] = (float)(z + (rng() - 0.5) * jit);
    }
    i = lo;
    bounds.push_back(lo);
  }
  const double lam = std::cbrt(i * vp / std::max(4.0 / 3 * kPi * As * As * Cs, 1e-12));
  for (int k = 0; k < i; ++k) {   // the seed: the last few anywhere inside the leftover's shape
    double ux, uy, uz;
    do {
      ux = rng() * 2 - 1;
      uy = rng() * 2 - 1;
      uz = rng() * 2 - 1;
    } while (ux * ux + uy * uy + uz * uz > 1);
    out[3 * k] = (float)(ux * As * lam);
    out[3 * k + 1] = (float)(uy * Cs * lam);
    out[3 * k + 2] = (float)(uz * As * lam);
  }
  bounds.push_back(0);
  std::reverse(bounds.begin(), bounds.end());
  if (device < 0) relax(out, n, a, ae - h * 0.5, ce - h * 0.5);
  else *rc = ccs::relax_device(device, out.data(), n, a, ae - h * 0.5, ce - h * 0.5, nullptr);
  return bounds;
}

double approach_time(const double relr[3], const double relv[3], double M, double touch) {
  double r[3] = {relr[0], relr[1], relr[2]}, v[3] = {relv[0], relv[1], relv[2]}, t = 0;
  const double h = 0.01 / 8;
  double a[3];
  auto acc = [&]() {
    const double f = -M * std::pow(r[0] * r[0] + r[1] * r[1] + r[2] * r[2], -1.5);
    for (int k = 0; k < 3; ++k) a[k] = r[k] * f;
  };
  acc();
  while (std::hypot(std::hypot(r[0], r[1]), r[2]) > touch && t < 200) {
    for (int k = 0; k < 3; ++k) v[k] += a[k] * h * 0.5;
    for (int k = 0; k < 3; ++k) r[k] += v[k] * h;
    acc();
    for (int k = 0; k < 3; ++k) v[k] += a[k] * h * 0.5;
    t += h;
  }
  return t;
}

int closest_bound(const std::vector<int> &bounds, double target) {
  int best = 0;
  for (int c : bounds)
    if (std::fabs(c - target) < std::fabs(best - target)) best = c;
  return best;
}

}  // namespace

static int make_bodies(const ccs_build_opt *opt, ccs_sim *sim, float *pos, float *vel, float *matR, float *home,
                       int device) {
  if (!opt || !sim || !pos || !vel || !matR) return CCS_E_ARG;
  const int N = opt->N;
  if (N < 64 || N > CCS_MAX_N) return CCS_E_RANGE;
  if (!(opt->rest > 0 && opt->rest < 1) || !(opt->dens > 0) || !(opt->q > 0)) return CCS_E_ARG;
  const int W = N >= 131072 ? 512 : N >= 32768 ? 256 : 128, H = N / W;
  const double rhoR = opt->rhoR > 0 ? opt->rhoR : 2.5;
  const double mT = opt->mTarget > 0 ? opt->mTarget : 1.0;
  const double rhoCrust = opt->rhoCrust > 0 ? opt->rhoCrust : 1.0;
  const double dens = opt->dens;
  auto core_volume = [&](double f) { return f / (rhoR - f * (rhoR - 1)); };
  const double coreV = core_volume(opt->core);
  const double coreV2 = core_volume(opt->coreImp >= 0 ? opt->coreImp : opt->core);
  const double V1 = mT, V2 = opt->q / dens, vp = (V1 + V2) / N;
  const double s = std::cbrt(16 * kPi * vp / 3);
  const double a = kJam * s / (2 * std::sqrt(2.0));
  int n1 = (int)js_round(N * V1 / (V1 + V2)), n2 = N - n1;
  if (opt->n2 > 0) { n2 = opt->n2; n1 = N - n2; }
  else if (n2 < 16) { n2 = 16; n1 = N - n2; }
  if (n1 < 16 || n2 < 1) return CCS_E_ARG;
  const double R1 = std::cbrt(V1), R2 = std::cbrt(V2), Rsum = R1 + R2;
  const double e1 = maclaurin(std::fabs(opt->spin0)), e2 = maclaurin(std::fabs(opt->spin1));
  Mulberry rng(1234567u);
  std::vector<float> b1, b2;
  int rc = CCS_OK;
  const std::vector<int> bd1 = ball(n1, s, a, rng, e1, b1, device, &rc);
  if (rc) return rc;
  const std::vector<int> bd2 = ball(n2, s, a, rng, e2, b2, device, &rc);
  if (rc) return rc;
  std::vector<unsigned char> lay((size_t)N);
  auto layers = [&](int off, int n, const std::vector<int> &bounds, double densB, double cv) {
    const int nCore = closest_bound(bounds, cv * n);
    int nCrust = n - bounds[bounds.size() - 2];
    if (opt->crustFrac > 0) nCrust = n - closest_bound(bounds, std::pow(1 - opt->crustFrac, 3) * n);
    double sum = 0;
    for (int j = 0; j < n; ++j) {
      const int layer = j < nCore ? 0 : j >= n - nCrust ? 2 : 1;
      lay[(size_t)off + j] = (unsigned char)layer;
      matR[off + j] = (float)(densB * (layer == 0 ? rhoR : layer == 2 ? rhoCrust : 1));
      sum += matR[off + j];
    }
    return sum;
  };
  const double sum1 = layers(0, n1, bd1, 1, coreV);
  double sum2 = layers(n1, n2, bd2, dens, coreV2);
  const double mref = mT / sum1;
  if (opt->mImp > 0) {
    const double k2 = opt->mImp / (mref * sum2);
    for (int j = n1; j < N; ++j) matR[j] = (float)(matR[j] * k2);
    sum2 *= k2;
  }
  const double M1 = mT, M2 = mref * sum2, M = M1 + M2;
  // the encounter, walked back from contact to the start line
  const double vesc = std::sqrt(2 * M / Rsum), vc = opt->vfac * vesc;
  const double bc = Rsum * std::sin(opt->angle * kPi / 180);
  const double D = Rsum + 3.7;
  const double vD = std::sqrt(std::max(vc * vc - 2 * M * (1 / Rsum - 1 / D), 0.04));
  const double bD = std::min(bc * vc / vD, D * 0.95);
  const double xD = -std::sqrt(D * D - bD * bD);
  const double inc = opt->incl * kPi / 180, bY = bD * std::sin(inc), bZ = bD * std::cos(inc);
  const double c1[3] = {-xD * M2 / M, -bY * M2 / M, -bZ * M2 / M};
  const double c2[3] = {xD + c1[0], bY + c1[1], bZ + c1[2]};
  for (int i = 0; i < N; ++i) {
    const bool imp = i >= n1;
    const float *b = imp ? &b2[(size_t)3 * (i - n1)] : &b1[(size_t)3 * i];
    const double *c = imp ? c2 : c1;
    for (int k = 0; k < 3; ++k) pos[4 * i + k] = (float)(b[k] + c[k]);
    pos[4 * i + 3] = (float)(lay[(size_t)i] + (imp ? 4 : 0));
  }
  std::memset(vel, 0, sizeof(float) * 4 * (size_t)N);
  if (home) {
    Mulberry hr(99u);
    const double off[3] = {1.5, 0.7, -1.1};
    for (int i = 0; i < N; ++i) {
      const bool imp = i >= n1;
      const float *b = imp ? &b2[(size_t)3 * (i - n1)] : &b1[(size_t)3 * i];
      for (int k = 0; k < 3; ++k) home[4 * i + k] = imp ? (float)(b[k] + off[k]) : b[k];
      home[4 * i + 3] = (float)hr();
    }
  }
  // the contact spring, the dashpot and the step, src/nbody.js:202-206
  const double vref = std::max(1.5, vc);
  const double k = 4 * mref * vref * vref / (a * a);
  const double dt = 0.35 / std::sqrt(2 * k / (mref * std::min(1.0, dens)));
  const double lnE = std::log(opt->rest), zeta = -lnE / std::sqrt(kPi * kPi + lnE * lnE);
  const double cd = 2 * zeta * std::sqrt(k * mref / 2);
  std::memset(sim, 0, sizeof *sim);
  sim->N = N; sim->W = W; sim->H = H; sim->n1 = n1; sim->n2 = n2; sim->G = N >= 65536 ? 128 : 64;
  sim->m = mref; sim->a = a; sim->cell = 2.6 * a; sim->dt = dt; sim->k = k; sim->c = cd; sim->creep = 0.12;
  sim->R1 = R1; sim->R2 = R2;
  sim->Re1 = R1 / std::pow(1 - e1 * e1, 1.0 / 6);
  sim->Re2 = R2 / std::pow(1 - e2 * e2, 1.0 / 6);
  sim->M1 = M1; sim->M2 = M2; sim->M = M; sim->vc = vc; sim->vesc = vesc;
  sim->spin0[1] = opt->spin0;
  sim->spin1[1] = opt->spin1 * std::sqrt(dens);
  for (int kk = 0; kk < 3; ++kk) { sim->cen0[kk] = c1[kk]; sim->cen1[kk] = c2[kk]; }
  sim->relr[0] = xD; sim->relr[1] = bY; sim->relr[2] = bZ;
  sim->relv[0] = vD;
  sim->t = -approach_time(sim->relr, sim->relv, M, sim->Re1 + sim->Re2 + 2 * a);
  sim->settleLeft = sim->settleTotal = (int)std::ceil(0.6 / dt);
  sim->phase = 0;
  sim->impactT = -1;
  sim->damp = std::exp(-dt * 12);
  sim->boxOn[0] = 1;
  sim->tK = 0.5 * kEkg / kCpRock / mref;
  sim->kappa = 0.3;
  return CCS_OK;
}

extern "C" int ccs_make_bodies(const ccs_build_opt *opt, ccs_sim *sim, float *pos, float *vel, float *matR,
                               float *home) {
  return make_bodies(opt, sim, pos, vel, matR, home, -1);
}

extern "C" int ccs_make_bodies_device(int device, const ccs_build_opt *opt, ccs_sim *sim, float *pos, float *vel,
                                      float *matR, float *home) {
  if (device < 0) return CCS_E_ARG;
  return make_bodies(opt, sim, pos, vel, matR, home, device);
}

// ---------------------------------------------------------------------------
// meshPairTable, src/nbody.js:56-108: the mesh's own pull between two
// particles by distance, its arithmetic repeated on a handful of nodes
// ---------------------------------------------------------------------------
namespace {
struct Node { int x, y, z; double m, cx, cy, cz, fx, fy, fz, pot; };

void cic_corners(const double p[3], int key[8][3], double w[8]) {
  double fl[3], t[3];
  for (int k = 0; k < 3; ++k) {
    const double g = (p[k] + kFL) / kFH - 0.5;
    fl[k] = std::floor(g);
    t[k] = g - fl[k];
  }
  for (int k = 0; k < 8; ++k) {
    const int o[3] = {k & 1, (k >> 1) & 1, k >> 2};
    for (int d = 0; d < 3; ++d) key[k][d] = (int)fl[d] + o[d];
    w[k] = (o[0] ? t[0] : 1 - t[0]) * (o[1] ? t[1] : 1 - t[1]) * (o[2] ? t[2] : 1 - t[2]);
  }
}

void node_field(const double (*parts)[3], int np, const double at[3], double out[4]) {
  std::vector<Node> nodes;   // in first-touched order, as the reference's Map
  auto find = [&](const int key[3]) -> int {
    for (size_t q = 0; q < nodes.size(); ++q)
      if (nodes[q].x == key[0] && nodes[q].y == key[1] && nodes[q].z == key[2]) return (int)q;
    return -1;
  };
  for (int i = 0; i < np; ++i) {
    int key[8][3];
    double w[8];
    cic_corners(parts[i], key, w);
    for (int k = 0; k < 8; ++k) {
      int f = find(key[k]);
      if (f < 0) {
        nodes.push_back(Node{key[k][0], key[k][1], key[k][2], 0, 0, 0, 0, 0, 0, 0, 0});
        f = (int)nodes.size() - 1;
      }
      Node &n = nodes[(size_t)f];
      n.m += w[k];
      n.cx += w[k] * parts[i][0];
      n.cy += w[k] * parts[i][1];
      n.cz += w[k] * parts[i][2];
    }
  }
  for (Node &n : nodes) { n.cx /= n.m; n.cy /= n.m; n.cz /= n.m; }
  const double eps2 = 0.5 * kFH * kFH;
  for (Node &c : nodes)
    for (const Node &o : nodes) {
      if (&o == &c) continue;
      const double rx = o.cx - c.cx, ry = o.cy - c.cy, rz = o.cz - c.cz;
      const double inv = 1 / std::sqrt(rx * rx + ry * ry + rz * rz + eps2), inv3 = inv * inv * inv;
      c.fx += rx * o.m * inv3;
      c.fy += ry * o.m * inv3;
      c.fz += rz * o.m * inv3;
      c.pot -= o.m * inv;
    }
  out[0] = out[1] = out[2] = out[3] = 0;
  int key[8][3];
  double w[8];
  cic_corners(at, key, w);
  for (int k = 0; k < 8; ++k) {
    const int f = find(key[k]);
    if (f < 0) continue;
    const Node &n = nodes[(size_t)f];
    out[0] += w[k] * n.fx;
    out[1] += w[k] * n.fy;
    out[2] += w[k] * n.fz;
    out[3] += w[k] * n.pot;
  }
}
}  // namespace

extern "C" int ccs_pair_table(int bins, double cut, float *f, float *pt) {
  if (bins <= 0 || !(cut > 0) || !f || !pt) return CCS_E_ARG;
  Mulberry rng(777u);
  const int per = 80;
  for (int b = 0; b < bins; ++b) {
    const double r = (b + 0.5) / bins * cut;
    double sf = 0, sp = 0;
    for (int s = 0; s < per; ++s) {
      double p[3];
      for (int k = 0; k < 3; ++k) p[k] = (rng() - 0.5) * kFH;
      const double z = 2 * rng() - 1;
      const double ph = rng() * 6.2831853;
      const double rr = std::sqrt(1 - z * z);
      const double u[3] = {rr * std::cos(ph), rr * std::sin(ph), z};
      const double parts[2][3] = {{p[0], p[1], p[2]}, {p[0] + u[0] * r, p[1] + u[1] * r, p[2] + u[2] * r}};
      double both[4], alone[4];
      node_field(parts, 2, p, both);
      node_field(parts, 1, p, alone);
      sf += (both[0] - alone[0]) * u[0] + (both[1] - alone[1]) * u[1] + (both[2] - alone[2]) * u[2];
      sp += both[3] - alone[3];
    }
    f[b] = (float)(sf / per * r * r);
    pt[b] = (float)(sp / per * r);
  }
  return CCS_OK;
}

// ---------------------------------------------------------------------------
// fof, src/nbody.js:646-893
// ---------------------------------------------------------------------------
namespace {

struct Group {
  int n = 0;
  double mass = 0, com[3] = {}, core[3] = {}, vel[3] = {}, imp = 0, iron = 0, R = 0, Redge = 0, Tsurf = 0;
  double hotCom[3] = {}, hotR = 0, impMass = 0, impCom[3] = {}, impRms = 0;
};

struct UnionFind {
  std::vector<int> up;
  explicit UnionFind(int n) : up((size_t)n) {
    for (int i = 0; i < n; ++i) up[(size_t)i] = i;
  }
  int root(int x) {
    while (up[(size_t)x] != x) {
      up[(size_t)x] = up[(size_t)up[(size_t)x]];
      x = up[(size_t)x];
    }
    return x;
  }
};

inline int fof_hash(int x, int y, int z, int mask) {
  return ((int)((uint32_t)x * 73856093u) ^ (int)((uint32_t)y * 19349663u) ^ (int)((uint32_t)z * 83492791u)) & mask;
}

Group group_stats(int N, double mref, const float *P, const float *V, const float *R, const std::vector<int> &rootOf,
                  int root, std::vector<int> &members) {
  Group g;
  members.clear();
  double x = 0, y = 0, z = 0, vx = 0, vy = 0, vz = 0, ix = 0, iy = 0, iz = 0;
  for (int t = 0; t < N; ++t) {
    if (rootOf[(size_t)t] != root) continue;
    const double m = mref * R[t], w = P[4 * t + 3];
    members.push_back(t);
    g.mass += m;
    x += m * P[4 * t]; y += m * P[4 * t + 1]; z += m * P[4 * t + 2];
    vx += m * V[4 * t]; vy += m * V[4 * t + 1]; vz += m * V[4 * t + 2];
    if (w >= 3.5) { g.impMass += m; ix += m * P[4 * t]; iy += m * P[4 * t + 1]; iz += m * P[4 * t + 2]; }
    if (w - 4 * std::floor(w / 4) < 0.5) g.iron += m;
  }
  g.n = (int)members.size();
  const double mass = g.mass, imp = g.impMass, Rg = std::cbrt(mass);
  g.com[0] = x / mass; g.com[1] = y / mass; g.com[2] = z / mass;
  g.impCom[0] = imp > 0 ? ix / imp : 0;
  g.impCom[1] = imp > 0 ? iy / imp : 0;
  g.impCom[2] = imp > 0 ? iz / imp : 0;
  // the body's own centre: from the material it is mostly made of, walked to
  // the centroid within 0.9 of its radius three times
  const double tm = mass - imp;
  double core[3];
  if (imp > tm) for (int k = 0; k < 3; ++k) core[k] = g.impCom[k];
  else { core[0] = (x - ix) / tm; core[1] = (y - iy) / tm; core[2] = (z - iz) / tm; }
  const double rc2 = 0.9 * 0.9 * Rg * Rg;
  for (int it = 0; it < 3; ++it) {
    double sm = 0, s0 = 0, s1 = 0, s2 = 0;
    for (int t : members) {
      const double qx = P[4 * t] - core[0], qy = P[4 * t + 1] - core[1], qz = P[4 * t + 2] - core[2];
      if (qx * qx + qy * qy + qz * qz < rc2) {
        const double m = mref * R[t];
        sm += m; s0 += m * P[4 * t]; s1 += m * P[4 * t + 1]; s2 += m * P[4 * t + 2];
      }
    }
    if (sm > 0) { core[0] = s0 / sm; core[1] = s1 / sm; core[2] = s2 / sm; }
  }
  std::memcpy(g.core, core, sizeof core);
  constexpr int NBIN = 96;
  const double shell = 0.64 * Rg * Rg, dr = 3 * Rg / NBIN;
  double Ts = 0, ws = 0, irms = 0, hs = 0, hx = 0, hy = 0, hz = 0, hr2 = 0, hist[NBIN] = {};
  for (int t : members) {
    const double m = mref * R[t];
    const double sx = P[4 * t] - core[0], sy = P[4 * t + 1] - core[1], sz = P[4 * t + 2] - core[2];
    const double r2s = sx * sx + sy * sy + sz * sz, Th = V[4 * t + 3];
    if (r2s > shell) { const double Tt = std::min(Th, 12000.0), wt = Tt * Tt; Ts += wt * Tt; ws += wt; }
    if (Th > 1200) {
      double wh = std::min(Th, 12000.0);
      wh *= wh;
      hs += wh; hx += wh * P[4 * t]; hy += wh * P[4 * t + 1]; hz += wh * P[4 * t + 2]; hr2 += wh * r2s;
    }
    if (P[4 * t + 3] >= 3.5) {
      const double ex = P[4 * t] - g.impCom[0], ey = P[4 * t + 1] - g.impCom[1], ez = P[4 * t + 2] - g.impCom[2];
      irms += m * (ex * ex + ey * ey + ez * ez);
    }
    const double bi = std::sqrt(r2s) / dr;
    hist[bi < NBIN - 1 ? (int)bi : NBIN - 1] += m;
  }
  std::memcpy(g.hotCom, core, sizeof core);
  g.hotR = Rg;
  if (hs > 0) {
    g.hotCom[0] = hx / hs; g.hotCom[1] = hy / hs; g.hotCom[2] = hz / hs;
    const double ox = g.hotCom[0] - core[0], oy = g.hotCom[1] - core[1], oz = g.hotCom[2] - core[2];
    g.hotR = std::sqrt(std::max(hr2 / hs - (ox * ox + oy * oy + oz * oz), 0.0));
  }
  if (g.n >= 2000) {   // where the body ends: the first shell under a third of the mantle's density
    const double Rb = std::cbrt(std::max(imp, tm));
    double rho[NBIN], refS = 0;
    int refN = 0;
    for (int b = 0; b < NBIN; ++b) {
      const double rm = (b + 0.5) * dr;
      rho[b] = hist[b] / (rm * rm * dr);
      if (rm > 0.6 * Rb && rm < 0.85 * Rb) { refS += rho[b]; ++refN; }
    }
    g.Redge = Rg;
    for (int b = 0; b < NBIN; ++b)
      if ((b + 0.5) * dr > 0.85 * Rb && refN > 0 && rho[b] < 0.35 * refS / refN) { g.Redge = b * dr; break; }
  }
  g.vel[0] = vx / mass; g.vel[1] = vy / mass; g.vel[2] = vz / mass;
  g.imp = imp / mass;
  g.iron /= mass;
  g.R = Rg;
  g.Tsurf = ws > 0 ? Ts / ws : 0;
  g.impRms = imp > 0 ? std::sqrt(irms / imp) : 0;
  return g;
}

}  // namespace

extern "C" int ccs_fof(int N, double mref, double a, const float *P, const float *V, const float *R, const float *D,
                       double spring, double touch, int cap, int sort, ccs_report *rep, int32_t *list,
                       int32_t *perm) {
  if (N <= 0 || !P || !V || !R || !D || !rep || (cap > 0 && !list) || cap < 0 || (sort && !perm)) return CCS_E_ARG;
  const double L = 2.4 * a, L2 = L * L, inv = 1 / L, touch2 = touch * touch;
  const int T = 1 << 20, TM = T - 1;
  // counting sort into hashed cells
  std::vector<int> cx((size_t)N), cy((size_t)N), cz((size_t)N), key((size_t)N), cnt((size_t)T + 1, 0);
  for (int i = 0; i < N; ++i) {
    cx[(size_t)i] = (int)std::floor(P[4 * i] * inv);
    cy[(size_t)i] = (int)std::floor(P[4 * i + 1] * inv);
    cz[(size_t)i] = (int)std::floor(P[4 * i + 2] * inv);
    key[(size_t)i] = fof_hash(cx[(size_t)i], cy[(size_t)i], cz[(size_t)i], TM);
    cnt[(size_t)key[(size_t)i] + 1]++;
  }
  for (int k = 0; k < T; ++k) cnt[(size_t)k + 1] += cnt[(size_t)k];
  std::vector<int> fill(cnt.begin(), cnt.begin() + T), order((size_t)N);
  for (int i = 0; i < N; ++i) order[(size_t)fill[(size_t)key[(size_t)i]]++] = i;
  // friends within 2.4 radii are one group; the contacts' spring energy on the way
  UnionFind uf(N);
  double elastic = 0;
  for (int i = 0; i < N; ++i) {
    const double px = P[4 * i], py = P[4 * i + 1], pz = P[4 * i + 2];
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int k = fof_hash(cx[(size_t)i] + dx, cy[(size_t)i] + dy, cz[(size_t)i] + dz, TM);
          for (int s = cnt[(size_t)k]; s < cnt[(size_t)k + 1]; ++s) {
            const int j = order[(size_t)s];
            if (j <= i) continue;
            const double ex = P[4 * j] - px, ey = P[4 * j + 1] - py, ez = P[4 * j + 2] - pz;
            const double e2 = ex * ex + ey * ey + ez * ez;
            if (e2 >= L2) continue;
            const int ri = uf.root(i), rj = uf.root(j);
            if (ri != rj) uf.up[(size_t)ri] = rj;
            if (e2 < touch2) {
              const double ov = touch - std::sqrt(e2);
              elastic += 0.5 * spring * ov * ov;
            }
          }
        }
  }
  std::vector<int> rootOf((size_t)N), size((size_t)N, 0);
  for (int i = 0; i < N; ++i) {
    rootOf[(size_t)i] = uf.root(i);
    size[(size_t)rootOf[(size_t)i]]++;
  }
  int g1 = -1, g2 = -1;
  for (int i = 0; i < N; ++i) {
    if (size[(size_t)i] <= 0) continue;
    if (g1 < 0 || size[(size_t)i] > size[(size_t)g1]) { g2 = g1; g1 = i; }
    else if (g2 < 0 || size[(size_t)i] > size[(size_t)g2]) g2 = i;
  }
  std::vector<int> members;
  members.reserve((size_t)N);
  const Group A = group_stats(N, mref, P, V, R, rootOf, g1, members);
  const bool hasB = g2 >= 0;
  const Group B = hasB ? group_stats(N, mref, P, V, R, rootOf, g2, members) : Group();
  // the planet's spin over the body proper, within 1.15 of its own radius
  const double rb = 1.15 * std::cbrt(std::max(A.impMass, A.mass - A.impMass)), rb2 = rb * rb;
  auto proper = [&](int i, double &dx0, double &dy0, double &dz0) {
    dx0 = P[4 * i] - A.core[0];
    dy0 = P[4 * i + 1] - A.core[1];
    dz0 = P[4 * i + 2] - A.core[2];
    return rootOf[(size_t)i] == g1 && !(dx0 * dx0 + dy0 * dy0 + dz0 * dz0 > rb2);
  };
  double bm = 0, bv[3] = {0, 0, 0}, d0, d1, d2;
  for (int i = 0; i < N; ++i) {
    if (!proper(i, d0, d1, d2)) continue;
    const double m = mref * R[i];
    bm += m;
    for (int k = 0; k < 3; ++k) bv[k] += m * V[4 * i + k];
  }
  if (bm > 0) for (int k = 0; k < 3; ++k) bv[k] /= bm;
  double Lx = 0, Ly = 0, Lz = 0, I = 0;
  for (int i = 0; i < N; ++i) {
    if (!proper(i, d0, d1, d2)) continue;
    const double m = mref * R[i];
    const double ux = V[4 * i] - bv[0], uy = V[4 * i + 1] - bv[1], uz = V[4 * i + 2] - bv[2];
    Lx += m * (d1 * uz - d2 * uy);
    Ly += m * (d2 * ux - d0 * uz);
    Lz += m * (d0 * uy - d1 * ux);
  }
  const double Lm = std::sqrt(Lx * Lx + Ly * Ly + Lz * Lz);
  const double lx = Lx / (Lm + 1e-30), ly = Ly / (Lm + 1e-30), lz = Lz / (Lm + 1e-30);
  const double tilt = std::acos(std::max(-1.0, std::min(1.0, ly))) * 180 / kPi;
  for (int i = 0; i < N; ++i) {
    if (!proper(i, d0, d1, d2)) continue;
    const double m = mref * R[i], along = d0 * lx + d1 * ly + d2 * lz;
    I += m * (d0 * d0 + d1 * d1 + d2 * d2 - along * along);
  }
  const double day = Lm > 1e-9 ? 2 * kPi * I / Lm * 805 / 3600 : INFINITY;
  auto energy = [&](double x, double y, double z, double vx, double vy, double vz) {
    const double r = std::sqrt((x - A.com[0]) * (x - A.com[0]) + (y - A.com[1]) * (y - A.com[1]) +
                               (z - A.com[2]) * (z - A.com[2]));
    const double dv2 = (vx - A.vel[0]) * (vx - A.vel[0]) + (vy - A.vel[1]) * (vy - A.vel[1]) +
                       (vz - A.vel[2]) * (vz - A.vel[2]);
    return 0.5 * dv2 - A.mass / std::max(r, A.R);
  };
  // the disk: what is bound in orbit about the planet, and the Moon it makes
  double orbit = 0, esc = 0, J[3] = {0, 0, 0};
  for (int i = 0; i < N; ++i) {
    if (rootOf[(size_t)i] == g1) continue;
    const double m = mref * R[i];
    if (energy(P[4 * i], P[4 * i + 1], P[4 * i + 2], V[4 * i], V[4 * i + 1], V[4 * i + 2]) < 0) {
      orbit += m;
      const double x0 = P[4 * i] - A.com[0], y0 = P[4 * i + 1] - A.com[1], z0 = P[4 * i + 2] - A.com[2];
      const double wx = V[4 * i] - A.vel[0], wy = V[4 * i + 1] - A.vel[1], wz = V[4 * i + 2] - A.vel[2];
      J[0] += m * (y0 * wz - z0 * wy);
      J[1] += m * (z0 * wx - x0 * wz);
      J[2] += m * (x0 * wy - y0 * wx);
    } else {
      esc += m;
    }
  }
  const double jD = orbit > 0 ? std::sqrt(J[0] * J[0] + J[1] * J[1] + J[2] * J[2]) / (orbit * std::sqrt(A.mass * 2.9)) : 0;
  const double moon = std::min(std::max(0.0, orbit * (1.9 * jD - 1.1 - 1.9 * 0.05)), 0.95 * orbit);
  std::memset(rep, 0, sizeof *rep);
  if (hasB && B.n >= std::max(8.0, N / 1000.0)) {
    const double dAB = std::sqrt((B.com[0] - A.com[0]) * (B.com[0] - A.com[0]) +
                                 (B.com[1] - A.com[1]) * (B.com[1] - A.com[1]) +
                                 (B.com[2] - A.com[2]) * (B.com[2] - A.com[2]));
    if (dAB > A.R + B.R + 2 * a) {
      rep->hasSecond = 1;
      rep->secMass = B.mass;
      rep->secDist = dAB;
      rep->secBound = energy(B.com[0], B.com[1], B.com[2], B.vel[0], B.vel[1], B.vel[2]) < 0;
      rep->secImp = B.imp;
      rep->secIron = B.iron;
      std::memcpy(rep->secCom, B.com, sizeof B.com);
      std::memcpy(rep->secCore, B.core, sizeof B.core);
      std::memcpy(rep->secVel, B.vel, sizeof B.vel);
      rep->secR = B.R;
    }
  }
  // the books
  double Mt = 0, p[3] = {0, 0, 0}, Jx = 0, Jy = 0, Jz = 0, ke = 0, pe = 0, Q = 0, ironAll = 0;
  int unseated = 0, full = 0;
  for (int i = 0; i < N; ++i) {
    const double m = mref * R[i];
    const double bx = P[4 * i], by = P[4 * i + 1], bz = P[4 * i + 2], bu = V[4 * i], bvv = V[4 * i + 1],
                 bw = V[4 * i + 2];
    Mt += m;
    p[0] += m * bu; p[1] += m * bvv; p[2] += m * bw;
    const double w = P[4 * i + 3];
    if (w - 4 * std::floor(w / 4.0) < 0.5) ironAll += m;
    Jx += m * (by * bw - bz * bvv);
    Jy += m * (bz * bu - bx * bw);
    Jz += m * (bx * bvv - by * bu);
    ke += 0.5 * m * (bu * bu + bvv * bvv + bw * bw);
    const double flag = D[4 * i + 1];
    const bool off = flag >= 2;
    pe += (off ? 1 : 0.5) * m * D[4 * i];
    Q += 0.5 * D[4 * i + 3];
    if (flag - (off ? 2 : 0) < 0.5) ++unseated;
    if (D[4 * i + 2] >= 7.5) ++full;
  }
  // the loose list: beyond 1.3 radii of the planet (and of a big second body),
  // the farthest first when there is more than the pairwise pass can take
  const bool bigB = hasB && B.mass > 0.05;
  auto far2 = [&](const Group &b, int i) {
    const double ex = P[4 * i] - b.com[0], ey = P[4 * i + 1] - b.com[1], ez = P[4 * i + 2] - b.com[2];
    return ex * ex + ey * ey + ez * ez;
  };
  auto loose = [&](int i) { return far2(A, i) > 1.69 * A.R * A.R && !(bigB && far2(B, i) <= 1.69 * B.R * B.R); };
  int nLoose = 0;
  for (int i = 0; i < N; ++i) nLoose += loose(i);
  double least = 0;
  if (nLoose > cap) {
    std::vector<double> ds;
    ds.reserve((size_t)nLoose);
    for (int i = 0; i < N; ++i)
      if (loose(i)) ds.push_back(far2(A, i));
    std::sort(ds.begin(), ds.end());
    least = ds[(size_t)(nLoose - cap)];
  }
  const int len = std::min(nLoose, cap);
  int wr = 0;
  for (int i = 0; i < N && wr < len; ++i)
    if (loose(i) && far2(A, i) >= least) list[wr++] = i;
  if (sort) {
    // the spatial order: a Morton key of 7 bits an axis over the largest body's box
    constexpr int KB = 1 << 21;
    std::vector<int> keys((size_t)N), bins((size_t)KB + 1, 0), into((size_t)N);
    for (int i = 0; i < N; ++i) {
      int m[3];
      for (int k = 0; k < 3; ++k) {
        const double v = std::floor(((double)P[4 * i + k] - A.core[k] + 6) / 12 * 128);
        m[k] = (int)std::min(127.0, std::max(0.0, v));
      }
      int mk = 0;
      for (int k = 0; k < 7; ++k)
        mk |= ((m[0] >> k) & 1) << (3 * k) | ((m[1] >> k) & 1) << (3 * k + 1) | ((m[2] >> k) & 1) << (3 * k + 2);
      keys[(size_t)i] = mk;
      bins[(size_t)mk + 1]++;
    }
    for (int k = 0; k < KB; ++k) bins[(size_t)k + 1] += bins[(size_t)k];
    for (int i = 0; i < N; ++i) {
      const int dst = bins[(size_t)keys[(size_t)i]]++;
      perm[dst] = i;
      into[(size_t)i] = dst;
    }
    for (int i = 0; i < len; ++i) list[i] = into[(size_t)list[i]];
  }
  rep->largest = A.mass; rep->largestImp = A.imp; rep->largestIron = A.iron; rep->day = day; rep->tilt = tilt;
  rep->axis[0] = lx; rep->axis[1] = ly; rep->axis[2] = lz;
  std::memcpy(rep->bodyVel, bv, sizeof bv);
  rep->orbit = orbit; rep->escape = esc;
  std::memcpy(rep->com, A.com, sizeof A.com);
  std::memcpy(rep->core, A.core, sizeof A.core);
  std::memcpy(rep->vel, A.vel, sizeof A.vel);
  rep->R = A.R; rep->Redge = A.Redge; rep->Tsurf = A.Tsurf;
  std::memcpy(rep->hotCom, A.hotCom, sizeof A.hotCom);
  rep->hotR = A.hotR; rep->impMass = A.impMass;
  std::memcpy(rep->impCom, A.impCom, sizeof A.impCom);
  rep->impRms = A.impRms;
  rep->M = Mt; rep->iron = ironAll / Mt;
  rep->drift = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) / Mt;
  rep->L = std::sqrt(Jx * Jx + Jy * Jy + Jz * Jz);
  rep->KE = ke; rep->PE = pe; rep->EL = elastic; rep->Q = Q;
  rep->unseated = (double)unseated / N; rep->full = (double)full / N;
  rep->jD = jD; rep->moon = moon;
  rep->ppCount = len; rep->ppLoose = nLoose;
  return CCS_OK;
}
