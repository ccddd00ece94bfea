/*
 * ccs_oracle.c -- CPU oracle for the cosmic-collisions simulation step.
 *
 * TEST INFRASTRUCTURE ONLY (see ccs_oracle.h).  Each function cites the
 * reference file:line it restates; paths are relative to the reference tree.
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fno-fast-math -fopenmp).
 */
#include "ccs_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FL 6.0
#define FH (2.0 * FL / 64.0)
#define PP_CUT (5.0 * FH)
#define SEAT_SLACK 0.6
#define JAM 0.96
#define E_KG 6.256e7
#define CP_ROCK 1200.0
#define CP_IRON 450.0
#define PI 3.141592653589793

void orc_engine_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------ */
/* binary32 vector helpers: one rounding per operation                 */
/* ------------------------------------------------------------------ */
typedef struct { float x, y, z; } v3;
static inline v3 V3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmuls(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline v3 vdivs(v3 a, float s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline float vdot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline float isqrt(float x) { return 1.0f / sqrtf(x); }   /* GLSL inversesqrt */
static inline v3 vcross(v3 a, v3 b) {
  return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline v3 ld3(const float *p) { return V3(p[0], p[1], p[2]); }
static inline float fmodg(float x, float y) { return x - y * floorf(x / y); } /* GLSL mod */
static inline float fclampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

/* JS Math.round: nearest, halves toward +infinity */
static double js_round(double x) {
  double r = floor(x);
  if (x - r >= 0.5) r += 1.0;
  return r;
}

/* ------------------------------------------------------------------ */
/* src/math.js:8-15 mulberry32                                         */
/* ------------------------------------------------------------------ */
double orc_mulberry(uint32_t *state) {
  uint32_t s = *state + 0x6D2B79F5u;
  *state = s;
  uint32_t t = (s ^ (s >> 15)) * (1u | s);
  t = (t + (t ^ (t >> 7)) * (61u | t)) ^ t;
  return (double)(t ^ (t >> 14)) / 4294967296.0;
}

/* ------------------------------------------------------------------ */
/* src/bodies.js:152-160 maclaurin, 162-169 turn                       */
/* ------------------------------------------------------------------ */
double orc_maclaurin_g(double e) {
  double s2 = 1 - e * e;
  return 2 * sqrt(s2) / (e * e * e) * (3 - 2 * e * e) * asin(e) - 6 * s2 / (e * e);
}
double orc_maclaurin(double f) {
  double want = 4.0 / 3.0 * f * f;
  if (want < 1e-6) return 0;
  double lo = 0.01, hi = 0.93;
  if (want >= orc_maclaurin_g(hi)) return hi;
  for (int i = 0; i < 60; i++) {
    double m = 0.5 * (lo + hi);
    if (orc_maclaurin_g(m) < want) lo = m; else hi = m;
  }
  return 0.5 * (lo + hi);
}
void orc_turn(const double w[3], double dt, double o[9]) {
  double m = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  if (m < 1e-12) { double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}; memcpy(o, I, sizeof I); return; }
  double x = w[0] / m, y = w[1] / m, z = w[2] / m, th = m * dt, c = cos(th), s = sin(th), t = 1 - c;
  o[0] = t * x * x + c;     o[1] = t * x * y + s * z; o[2] = t * x * z - s * y;
  o[3] = t * x * y - s * z; o[4] = t * y * y + c;     o[5] = t * y * z + s * x;
  o[6] = t * x * z + s * y; o[7] = t * y * z - s * x; o[8] = t * z * z + c;
}

/* ------------------------------------------------------------------ */
/* src/bodies.js:97-146 relax                                          */
/* ------------------------------------------------------------------ */
void orc_relax(float *p, int n, double a, double A, double C, int sweeps) {
  double D = 2 * a * 0.96, cs = 2.2 * a, iA2 = 1 / (A * A), iC2 = 1 / (C * C);
  int nSweeps = sweeps > 0 ? sweeps : 10;
  double lo[3] = {1e9, 1e9, 1e9}, hi[3] = {-1e9, -1e9, -1e9};
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      double v = p[i * 3 + k];
      if (v < lo[k]) lo[k] = v;
      if (v > hi[k]) hi[k] = v;
    }
  int gx = (int)floor((hi[0] - lo[0]) / cs) + 3, gy = (int)floor((hi[1] - lo[1]) / cs) + 3,
      gz = (int)floor((hi[2] - lo[2]) / cs) + 3;
  int nc = gx * gy * gz;
  int *start = (int *)calloc((size_t)nc + 1, sizeof(int));
  int *order = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int *cell = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int sweep = 0; sweep < nSweeps; sweep++) {
    if (sweep % 4 == 0) {
      memset(start, 0, sizeof(int) * ((size_t)nc + 1));
      for (int i = 0; i < n; i++) {
        double fx = floor((p[i * 3] - lo[0]) / cs) + 1, fy = floor((p[i * 3 + 1] - lo[1]) / cs) + 1,
               fz = floor((p[i * 3 + 2] - lo[2]) / cs) + 1;
        int cx = (int)fmin(fmax(fx, 0), gx - 1), cy = (int)fmin(fmax(fy, 0), gy - 1),
            cz = (int)fmin(fmax(fz, 0), gz - 1);
        cell[i] = (cx * gy + cy) * gz + cz;
        start[cell[i] + 1]++;
      }
      for (int k = 0; k < nc; k++) start[k + 1] += start[k];
      for (int i = 0; i < n; i++) order[start[cell[i]]++] = i;
      for (int k = nc; k > 0; k--) start[k] = start[k - 1];
      start[0] = 0;
    }
    for (int i = 0; i < n; i++) {
      int c = cell[i];
      double x = p[i * 3], y = p[i * 3 + 1], z = p[i * 3 + 2];
      for (int o = 0; o < 27; o++) {
        int cc = c + ((o % 3) - 1) * gy * gz + (((o / 3) % 3) - 1) * gz + ((o / 9) - 1);
        if (cc < 0 || cc >= nc) continue;
        for (int q = start[cc]; q < start[cc + 1]; q++) {
          int j = order[q];
          if (j <= i) continue;
          double dx = p[j * 3] - x, dy = p[j * 3 + 1] - y, dz = p[j * 3 + 2] - z;
          double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 >= D * D) continue;
          double d = sqrt(d2);
          if (d == 0) d = 1e-9;
          double ov = D - d, mv = 0.5 * ov / d;
          dx *= mv; dy *= mv; dz *= mv;
          x -= dx; y -= dy; z -= dz;
          p[j * 3] = (float)(p[j * 3] + dx);
          p[j * 3 + 1] = (float)(p[j * 3 + 1] + dy);
          p[j * 3 + 2] = (float)(p[j * 3 + 2] + dz);
        }
      }
      double qq = (x * x + z * z) * iA2 + y * y * iC2;
      if (qq > 1.0) { double f = 1 / sqrt(qq); x *= f; y *= f; z *= f; }
      p[i * 3] = (float)x; p[i * 3 + 1] = (float)y; p[i * 3 + 2] = (float)z;
    }
  }
  free(start); free(order); free(cell);
}

/* ------------------------------------------------------------------ */
/* src/bodies.js:23-76 ball                                            */
/* ------------------------------------------------------------------ */
typedef struct { double A, C, want; double cum[257]; } shell_t;

int orc_ball(int n, double s, double a, uint32_t *rng, double e, float *out, int *bounds) {
  enum { NB = 256 };
  double R = cbrt(3 * n * s * s * s / (16 * PI));
  double ae = R / pow(1 - e * e, 1.0 / 6), ce = ae * sqrt(1 - e * e);
  double vp = s * s * s / 4, unit = 3 * vp / (4 * PI), jit = 0.06 * s;
  double h = s * sqrt(1.0 / 3);
  int K = (int)js_round(ce / h);
  if (K < 1) K = 1;
  double GA = PI * (3 - sqrt(5.0));
  h = ce / K;
  shell_t *sh = (shell_t *)malloc(sizeof(shell_t) * (size_t)K);
  int nsh = 0, kept = 0;
  double total = 0;
  for (int j = 0; j < K; j++) {
    double A = ae - j * h, C = ce - j * h;
    if (C - h * 0.5 < h) break;
    double Am = A - h * 0.5, Cm = C - h * 0.5;
    sh[nsh].cum[0] = 0;
    for (int b = 0; b < NB; b++) {
      double be = (b + 0.5) * PI / NB - PI / 2, cb = cos(be), sb = sin(be);
      sh[nsh].cum[b + 1] = sh[nsh].cum[b] + Am * cb * sqrt(Cm * Cm * cb * cb + Am * Am * sb * sb);
    }
    double want = (A * A * C - (A - h) * (A - h) * (C - h)) / unit;
    sh[nsh].A = Am; sh[nsh].C = Cm; sh[nsh].want = want;
    nsh++;
    total += want;
    kept = j + 1;
  }
  double As = ae - kept * h, Cs = ce - kept * h;
  total += fmax(As * As * Cs, 0) / unit;
  int nb = 0;
  bounds[nb++] = n;
  int i = n;
  double acc = 0;
  for (int j = 0; j < nsh; j++) {
    acc += sh[j].want * n / total;
    double r = js_round(acc);
    int mm = (int)fmin(fmin(r, n) - (n - i), i);
    int lo = i - mm;
    double phi0 = orc_mulberry(rng) * 2 * PI;
    double flip = orc_mulberry(rng) < 0.5 ? -1 : 1;
    int bb = 0;
    for (int q = 0; q < mm; q++) {
      double u = (q + 0.5) / mm * sh[j].cum[NB];
      while (bb < NB - 1 && sh[j].cum[bb + 1] < u) bb++;
      double lat = (bb + (u - sh[j].cum[bb]) / (sh[j].cum[bb + 1] - sh[j].cum[bb])) * PI / NB - PI / 2;
      double phi = phi0 + q * GA, rc = sh[j].A * cos(lat);
      int o = (lo + q) * 3;
      out[o] = (float)(rc * cos(phi) + (orc_mulberry(rng) - 0.5) * jit);
      out[o + 1] = (float)(flip * sh[j].C * sin(lat) + (orc_mulberry(rng) - 0.5) * jit);
      out[o + 2] = (float)(rc * sin(phi) + (orc_mulberry(rng) - 0.5) * jit);
    }
    i = lo;
    bounds[nb++] = lo;
  }
  double lam = cbrt(i * vp / fmax(4.0 / 3 * PI * As * As * Cs, 1e-12));
  for (int k = 0; k < i; k++) {
    double ux, uy, uz, u2;
    do {
      ux = orc_mulberry(rng) * 2 - 1; uy = orc_mulberry(rng) * 2 - 1; uz = orc_mulberry(rng) * 2 - 1;
      u2 = ux * ux + uy * uy + uz * uz;
    } while (u2 > 1);
    out[k * 3] = (float)(ux * As * lam);
    out[k * 3 + 1] = (float)(uy * Cs * lam);
    out[k * 3 + 2] = (float)(uz * As * lam);
  }
  bounds[nb++] = 0;
  for (int x = 0, y = nb - 1; x < y; x++, y--) { int t = bounds[x]; bounds[x] = bounds[y]; bounds[y] = t; }
  orc_relax(out, n, a, ae - h * 0.5, ce - h * 0.5, 10);
  free(sh);
  return nb;
}

/* ------------------------------------------------------------------ */
/* src/nbody.js:578-590 approachTime                                   */
/* ------------------------------------------------------------------ */
double orc_approach_time(const double relr[3], const double relv[3], double M, double touch) {
  double r[3] = {relr[0], relr[1], relr[2]}, v[3] = {relv[0], relv[1], relv[2]}, h = 0.01 / 8, t = 0;
  double a[3];
#define ACC()                                                    \
  do {                                                           \
    double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];         \
    double f = -M * pow(d2, -1.5);                               \
    a[0] = r[0] * f; a[1] = r[1] * f; a[2] = r[2] * f;           \
  } while (0)
  ACC();
  while (hypot(hypot(r[0], r[1]), r[2]) > touch && t < 200) {
    for (int k = 0; k < 3; k++) v[k] += a[k] * h * 0.5;
    for (int k = 0; k < 3; k++) r[k] += v[k] * h;
    ACC();
    for (int k = 0; k < 3; k++) v[k] += a[k] * h * 0.5;
    t += h;
  }
#undef ACC
  return t;
}

/* ------------------------------------------------------------------ */
/* src/nbody.js:114-250 build (+ documented extensions)                */
/* ------------------------------------------------------------------ */
static int nearest_bound(const int *bounds, int nb, double target) {
  /* bounds.reduce(..., 0): the first bound closest to target, starting from 0 */
  int best = 0;
  for (int i = 0; i < nb; i++)
    if (fabs(bounds[i] - target) < fabs(best - target)) best = bounds[i];
  return best;
}

int orc_build(const orc_opt *opt, orc_sim *sim, float *pos, float *vel, float *matR, float *home) {
  int N = opt->N;
  int W = N >= 131072 ? 512 : N >= 32768 ? 256 : 128, H = N / W;
  double q = opt->q, dens = opt->dens, coreF = opt->core;
  double RHO_R = opt->rhoR > 0 ? opt->rhoR : 2.5;
  double mT = opt->mTarget > 0 ? opt->mTarget : 1.0;
  double rhoCrust = opt->rhoCrust > 0 ? opt->rhoCrust : 1.0;
  double coreV = coreF / (RHO_R - coreF * (RHO_R - 1));
  double coreF2 = opt->coreImp >= 0 ? opt->coreImp : coreF;
  double coreV2 = coreF2 / (RHO_R - coreF2 * (RHO_R - 1));
  double V1 = mT, V2 = q / dens;
  double vp = (V1 + V2) / N;
  double s = cbrt(16 * PI * vp / 3);
  double a = JAM * s / (2 * sqrt(2.0));
  int n1 = (int)js_round(N * V1 / (V1 + V2)), n2 = N - n1;
  if (opt->n2 > 0) { n2 = opt->n2; n1 = N - n2; }
  else if (n2 < 16) { n2 = 16; n1 = N - n2; }
  double R1 = cbrt(V1), R2 = cbrt(V2), Rsum = R1 + R2;
  double w0[3] = {0, opt->spin0, 0}, w1[3] = {0, opt->spin1 * sqrt(dens), 0};
  double e1 = orc_maclaurin(fabs(opt->spin0)), e2 = orc_maclaurin(fabs(opt->spin1));
  double Re1 = R1 / pow(1 - e1 * e1, 1.0 / 6), Re2 = R2 / pow(1 - e2 * e2, 1.0 / 6);

  uint32_t rng = 1234567u;
  float *b1 = (float *)malloc(sizeof(float) * 3 * (size_t)n1), *b2 = (float *)malloc(sizeof(float) * 3 * (size_t)n2);
  int *bd1 = (int *)malloc(sizeof(int) * ((size_t)n1 + 3)), *bd2 = (int *)malloc(sizeof(int) * ((size_t)n2 + 3));
  int nb1 = orc_ball(n1, s, a, &rng, e1, b1, bd1);
  int nb2 = orc_ball(n2, s, a, &rng, e2, b2, bd2);
  unsigned char *lay = (unsigned char *)malloc((size_t)N);
  double sums[2];
  for (int body = 0; body < 2; body++) {
    int off = body ? n1 : 0, n = body ? n2 : n1, nb = body ? nb2 : nb1;
    const int *bounds = body ? bd2 : bd1;
    double densB = body ? dens : 1, cv = body ? coreV2 : coreV;
    int nCore = nearest_bound(bounds, nb, cv * n);
    int nCrust = n - bounds[nb - 2];
    if (opt->crustFrac > 0) {
      double inside = pow(1 - opt->crustFrac, 3);
      nCrust = n - nearest_bound(bounds, nb, inside * n);
    }
    double sum = 0;
    for (int j = 0; j < n; j++) {
      int layer = j < nCore ? 0 : j >= n - nCrust ? 2 : 1;
      lay[off + j] = (unsigned char)layer;
      matR[off + j] = (float)(densB * (layer == 0 ? RHO_R : layer == 2 ? rhoCrust : 1));
      sum += matR[off + j];
    }
    sums[body] = sum;
  }
  double sum1 = sums[0], sum2 = sums[1];
  double mref = mT / sum1;
  if (opt->mImp > 0) {
    double k2 = opt->mImp / (mref * sum2);
    for (int jj = n1; jj < N; jj++) matR[jj] = (float)(matR[jj] * k2);
    sum2 *= k2;
  }
  double M1 = mT, M2 = mref * sum2, M = M1 + M2;
  double vesc = sqrt(2 * M / Rsum), vc = opt->vfac * vesc;
  double bc = Rsum * sin(opt->angle * PI / 180);
  double D = Rsum + 3.7;
  double vD = sqrt(fmax(vc * vc - 2 * M * (1 / Rsum - 1 / D), 0.04));
  double bD = fmin(bc * vc / vD, D * 0.95);
  double xD = -sqrt(D * D - bD * bD);
  double inc = opt->incl * PI / 180, bY = bD * sin(inc), bZ = bD * cos(inc);
  double c1[3] = {-xD * M2 / M, -bY * M2 / M, -bZ * M2 / M};
  double c2[3] = {xD + c1[0], bY + c1[1], bZ + c1[2]};
  for (int i = 0; i < n1; i++) {
    int o = i * 4;
    pos[o] = (float)(b1[i * 3] + c1[0]); pos[o + 1] = (float)(b1[i * 3 + 1] + c1[1]);
    pos[o + 2] = (float)(b1[i * 3 + 2] + c1[2]); pos[o + 3] = (float)lay[i];
  }
  for (int i = 0; i < n2; i++) {
    int o = (n1 + i) * 4;
    pos[o] = (float)(b2[i * 3] + c2[0]); pos[o + 1] = (float)(b2[i * 3 + 1] + c2[1]);
    pos[o + 2] = (float)(b2[i * 3 + 2] + c2[2]); pos[o + 3] = (float)(lay[n1 + i] + 4);
  }
  memset(vel, 0, sizeof(float) * 4 * (size_t)N);
  if (home) {
    uint32_t hr = 99u;
    for (int i = 0; i < n1; i++) {
      int o = i * 4;
      home[o] = b1[i * 3]; home[o + 1] = b1[i * 3 + 1]; home[o + 2] = b1[i * 3 + 2];
      home[o + 3] = (float)orc_mulberry(&hr);
    }
    for (int i = 0; i < n2; i++) {
      int o = (n1 + i) * 4;
      home[o] = (float)(b2[i * 3] + 1.5); home[o + 1] = (float)(b2[i * 3 + 1] + 0.7);
      home[o + 2] = (float)(b2[i * 3 + 2] - 1.1); home[o + 3] = (float)orc_mulberry(&hr);
    }
  }
  double vref = fmax(1.5, vc);
  double k = 4 * mref * vref * vref / (a * a);
  double dt = 0.35 / sqrt(2 * k / (mref * fmin(1, dens)));
  double lnE = log(opt->rest), zeta = -lnE / sqrt(PI * PI + lnE * lnE);
  double cd = 2 * zeta * sqrt(k * mref / 2);
  int G = N >= 65536 ? 128 : 64;
  int settle = (int)ceil(0.6 / dt);

  memset(sim, 0, sizeof *sim);
  sim->N = N; sim->W = W; sim->H = H; sim->n1 = n1; sim->n2 = n2; sim->G = G;
  sim->m = mref; sim->a = a; sim->cell = 2.6 * a; sim->dt = dt; sim->k = k; sim->c = cd; sim->creep = 0.12;
  sim->R1 = R1; sim->R2 = R2; sim->Re1 = Re1; sim->Re2 = Re2; sim->M1 = M1; sim->M2 = M2; sim->M = M;
  sim->vc = vc; sim->vesc = vesc;
  memcpy(sim->spin0, w0, sizeof w0); memcpy(sim->spin1, w1, sizeof w1);
  memcpy(sim->cen0, c1, sizeof c1); memcpy(sim->cen1, c2, sizeof c2);
  sim->relr[0] = xD; sim->relr[1] = bY; sim->relr[2] = bZ;
  sim->relv[0] = vD; sim->relv[1] = 0; sim->relv[2] = 0;
  sim->t = -orc_approach_time(sim->relr, sim->relv, M, Re1 + Re2 + 2 * a);
  sim->phase = 0; sim->settleLeft = settle; sim->settleTotal = settle; sim->impactT = -1; sim->stepNo = 0;
  sim->damp = exp(-dt * 12); sim->soft = 0;
  sim->boxOn[0] = 1; sim->boxOn[1] = 0;
  sim->tK = 0.5 * E_KG / CP_ROCK / mref;
  sim->kappa = 0.3;
  free(b1); free(b2); free(bd1); free(bd2); free(lay);
  return 0;
}

/* ------------------------------------------------------------------ */
/* src/nbody.js:56-108 meshPairTable                                   */
/* ------------------------------------------------------------------ */
typedef struct { int key[3]; double m, x, y, z, fx, fy, fz, pot; } node_t;

static void corners(const double p[3], int key[8][3], double w[8]) {
  double g[3], fl[3], t[3];
  for (int k = 0; k < 3; k++) {
    g[k] = (p[k] + FL) / FH - 0.5;
    fl[k] = floor(g[k]);
    t[k] = g[k] - fl[k];
  }
  for (int k = 0; k < 8; k++) {
    int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
    key[k][0] = (int)fl[0] + ox; key[k][1] = (int)fl[1] + oy; key[k][2] = (int)fl[2] + oz;
    w[k] = (ox ? t[0] : 1 - t[0]) * (oy ? t[1] : 1 - t[1]) * (oz ? t[2] : 1 - t[2]);
  }
}

static void pair_field(const double parts[][3], int np, const double at[3], double out[4]) {
  node_t nodes[16];
  int nn = 0;
  double eps2 = 0.5 * FH * FH;
  for (int i = 0; i < np; i++) {
    int key[8][3]; double w[8];
    corners(parts[i], key, w);
    for (int k = 0; k < 8; k++) {
      int f = -1;
      for (int q = 0; q < nn; q++)
        if (nodes[q].key[0] == key[k][0] && nodes[q].key[1] == key[k][1] && nodes[q].key[2] == key[k][2]) { f = q; break; }
      if (f < 0) {
        f = nn++;
        memset(&nodes[f], 0, sizeof nodes[f]);
        memcpy(nodes[f].key, key[k], sizeof key[k]);
      }
      nodes[f].m += w[k]; nodes[f].x += w[k] * parts[i][0]; nodes[f].y += w[k] * parts[i][1]; nodes[f].z += w[k] * parts[i][2];
    }
  }
  /* a node of zero weight (a particle exactly on a cell face) carries nothing; the table's random
   * placings never make one */
  for (int q = 0; q < nn; q++)
    if (nodes[q].m > 0) { nodes[q].x /= nodes[q].m; nodes[q].y /= nodes[q].m; nodes[q].z /= nodes[q].m; }
  for (int c = 0; c < nn; c++)
    for (int o = 0; o < nn; o++) {
      if (o == c || !(nodes[o].m > 0) || !(nodes[c].m > 0)) continue;
      double rx = nodes[o].x - nodes[c].x, ry = nodes[o].y - nodes[c].y, rz = nodes[o].z - nodes[c].z;
      double inv = 1 / sqrt(rx * rx + ry * ry + rz * rz + eps2), inv3 = inv * inv * inv;
      nodes[c].fx += rx * nodes[o].m * inv3; nodes[c].fy += ry * nodes[o].m * inv3; nodes[c].fz += rz * nodes[o].m * inv3;
      nodes[c].pot -= nodes[o].m * inv;
    }
  out[0] = out[1] = out[2] = out[3] = 0;
  int key[8][3]; double w[8];
  corners(at, key, w);
  for (int k = 0; k < 8; k++) {
    int f = -1;
    for (int q = 0; q < nn; q++)
      if (nodes[q].key[0] == key[k][0] && nodes[q].key[1] == key[k][1] && nodes[q].key[2] == key[k][2]) { f = q; break; }
    if (f < 0) continue;
    out[0] += w[k] * nodes[f].fx; out[1] += w[k] * nodes[f].fy; out[2] += w[k] * nodes[f].fz; out[3] += w[k] * nodes[f].pot;
  }
}

/* The label of the learned correction: the mesh's force on a target from a
 * unit source, field() of meshPairTable (src/nbody.js:60-91) for the isolated
 * pair, both minus alone, in mesh cells: d = source - target in cells, s the
 * source's position in its cell (the GLSL_BOX g with its half-cell shift, as
 * the deposit uses it).  The pair is placed mid-mesh; out in cells^-2. */
void orc_nn_label(const double d[3], const double s[3], double out[3]) {
  double q[3], p[3], both[4], alone[4];
  for (int k = 0; k < 3; k++) {
    q[k] = (s[k] + 32.0 + 0.5) * FH - FL;
    p[k] = q[k] - d[k] * FH;
  }
  const double two[2][3] = {{p[0], p[1], p[2]}, {q[0], q[1], q[2]}};
  const double one[1][3] = {{p[0], p[1], p[2]}};
  pair_field(two, 2, p, both);
  pair_field(one, 1, p, alone);
  for (int k = 0; k < 3; k++) out[k] = (both[k] - alone[k]) * (FH * FH);
}

void orc_pair_table(int bins, double cut, float *f, float *pt) {
  uint32_t rng = 777u;
  int per = 80;
  for (int b = 0; b < bins; b++) {
    double r = (b + 0.5) / bins * cut, sf = 0, sp = 0;
    for (int s = 0; s < per; s++) {
      double p[3];
      p[0] = (orc_mulberry(&rng) - 0.5) * FH; p[1] = (orc_mulberry(&rng) - 0.5) * FH; p[2] = (orc_mulberry(&rng) - 0.5) * FH;
      double z = 2 * orc_mulberry(&rng) - 1, ph = orc_mulberry(&rng) * 6.2831853, rr = sqrt(1 - z * z);
      double u[3] = {rr * cos(ph), rr * sin(ph), z};
      double q[3] = {p[0] + u[0] * r, p[1] + u[1] * r, p[2] + u[2] * r};
      double both2[2][3] = {{p[0], p[1], p[2]}, {q[0], q[1], q[2]}};
      double both[4], alone[4];
      pair_field(both2, 2, p, both);
      pair_field(both2, 1, p, alone);
      sf += (both[0] - alone[0]) * u[0] + (both[1] - alone[1]) * u[1] + (both[2] - alone[2]) * u[2];
      sp += both[3] - alone[3];
    }
    f[b] = (float)(sf / per * r * r);
    pt[b] = (float)(sp / per * r);
  }
}

/* ------------------------------------------------------------------ */
/* uniforms: src/nbody.js:255-336 setStaticUniforms, 342-350 boxes,     */
/* 545-550 soften                                                      */
/* ------------------------------------------------------------------ */
void orc_make_uni(const orc_sim *s, orc_uni *u) {
  memset(u, 0, sizeof *u);
  u->N = s->N; u->W = s->W;
  u->G = s->G; u->SX = s->G == 128 ? 16 : 8;
  u->GShift = s->G == 128 ? 7 : 6; u->SXShift = u->SX == 16 ? 4 : 3;
  u->GMask = u->G - 1; u->SXMask = u->SX - 1;
  u->AW = u->SX * u->G; u->AH = (u->G / u->SX) * u->G;
  u->invCell = (float)(1 / s->cell); u->cell = (float)s->cell;
  u->link2 = (float)(s->cell * s->cell);
  u->reach2 = (float)pow(s->cell + SEAT_SLACK * s->a, 2);
  u->touch = (float)(2 * s->a);
  u->K = (float)s->k; u->C = (float)s->c; u->invM = (float)(1 / s->m);
  u->damp = (float)s->damp; u->creep = (float)s->creep; u->tK = (float)s->tK; u->kappa = (float)s->kappa;
  u->cpIron = (float)(CP_IRON / CP_ROCK);
  u->dt = (float)s->dt;
  for (int k = 0; k < 3; k++) {
    u->spin0[k] = (float)s->spin0[k]; u->spin1[k] = (float)s->spin1[k];
    u->bulk0[k] = (float)s->bulk0[k]; u->bulk1[k] = (float)s->bulk1[k];
    u->cen0[k] = (float)s->cen0[k]; u->cen1[k] = (float)s->cen1[k];
  }
  u->invH = (float)(1 / FH); u->eps2Mesh = (float)(FH * FH); u->eps2Cell = (float)(0.5 * FH * FH);
  u->Gm = (float)s->m;
  u->cut = (float)PP_CUT; u->a2 = (float)(s->a * s->a);
  u->frozen = -1.0f;   /* simFS without frozen: nothing is held */
  /* uLA, uLB, uBoxB keep GL's initial zeros until boxes() first runs */
}
void orc_boxes(const orc_sim *s, orc_uni *u) {
  for (int i = 0; i < 2; i++) {
    double dt = s->t - s->boxT[i];
    float *L = i ? u->LB : u->LA;
    for (int k = 0; k < 3; k++) L[k] = (float)(FL - s->boxCen[i][k] - s->boxVel[i][k] * dt);
  }
  u->boxB = s->boxOn[1] ? 1.0f : 0.0f;
}
void orc_soften(orc_sim *s) {
  s->soft = 1;
  s->k *= 0.5; s->c *= sqrt(0.5); s->dt *= sqrt(2.0);
  s->damp = exp(-s->dt * 12);
}

/* ------------------------------------------------------------------ */
/* src/glsl-sim.js:79-91 hashAt; 112-149 SLOT_VS                        */
/* ------------------------------------------------------------------ */
void orc_hash(const orc_uni *u, int cx, int cy, int cz, int *ax, int *ay) {
  int px = cx >> u->GShift, py = cy >> u->GShift, pz = cz >> u->GShift;   /* arithmetic shifts */
  uint32_t y = (uint32_t)cy + ((uint32_t)px << (u->GShift - 1)) + ((uint32_t)pz << (u->GShift - 2));
  uint32_t z = (uint32_t)cz + ((uint32_t)py << (u->GShift - 1));
  uint32_t x = (uint32_t)cx & (uint32_t)u->GMask;
  y &= (uint32_t)u->GMask; z &= (uint32_t)u->GMask;
  *ax = (int)(((z & (uint32_t)u->SXMask) << u->GShift) + x);
  *ay = (int)(((z >> u->SXShift) << u->GShift) + y);
}

uint32_t orc_cell_of(const orc_uni *u, const float p[3], uint32_t *word, int idx) {
  float g[3];
  int c[3];
  uint32_t q[3];
  for (int k = 0; k < 3; k++) {
    g[k] = p[k] * u->invCell;
    float f = floorf(g[k]);
    c[k] = (int)f;
    float fr = g[k] - f;
    q[k] = (uint32_t)fclampf(fr * 15.0f, 0.0f, 14.0f);
  }
  int ax, ay;
  orc_hash(u, c[0], c[1], c[2], &ax, &ay);
  if (word) *word = (uint32_t)idx | (q[0] << 18) | (q[1] << 22) | (q[2] << 26) | 0x40000000u;
  return (uint32_t)ay * (uint32_t)u->AW + (uint32_t)ax;
}

void orc_slots(const orc_uni *u, const float *pos4, uint32_t *seats) {
  size_t nc = (size_t)u->AW * (size_t)u->AH * ORC_SEATS;
  for (size_t k = 0; k < nc; k++) seats[k] = ORC_EMPTY;
  /* the depth-peel keeps, for seat k, the lowest index above seat k-1: in
   * index order that is "the first eight to arrive" */
  for (int i = 0; i < u->N; i++) {
    uint32_t w;
    uint32_t h = orc_cell_of(u, pos4 + (size_t)i * 4, &w, i);
    uint32_t *s = seats + (size_t)h * ORC_SEATS;
    for (int k = 0; k < ORC_SEATS; k++)
      if (s[k] == ORC_EMPTY) { s[k] = w; break; }
  }
}

/* ------------------------------------------------------------------ */
/* src/glsl-sim.js:25-37 boxOf                                         */
/* ------------------------------------------------------------------ */
int orc_box_of(const orc_uni *u, const float p[3], float g[3]) {
  float gA[3], gB[3];
  int inA = 1, inB = u->boxB > 0.5f;
  for (int k = 0; k < 3; k++) {
    gA[k] = (p[k] + u->LA[k]) * u->invH - 0.5f;
    gB[k] = (p[k] + u->LB[k]) * u->invH - 0.5f;
    if (!(gA[k] >= 0.0f && gA[k] <= 63.0f)) inA = 0;
    if (!(gB[k] >= 0.0f && gB[k] <= 63.0f)) inB = 0;
  }
  if (inA && inB) {
    float dA = fmaxf(fabsf(gA[0] - 31.5f), fmaxf(fabsf(gA[1] - 31.5f), fabsf(gA[2] - 31.5f)));
    float dB = fmaxf(fabsf(gB[0] - 31.5f), fmaxf(fabsf(gB[1] - 31.5f), fabsf(gB[2] - 31.5f)));
    inA = dA <= dB;
    inB = !inA;
  }
  for (int k = 0; k < 3; k++) g[k] = inA ? gA[k] : gB[k];
  return inA ? 0 : inB ? 1 : -1;
}

static inline int fine_index(int x, int y, int z) { return (z * 64 + y) * 64 + x; }
static inline int coarse_index(int x, int y, int z) { return (z * 16 + y) * 16 + x; }

/* ------------------------------------------------------------------ */
/* src/glsl-sim.js:168-211 DEP_VS (+ the clear, src/nbody.js:402-416)  */
/* ------------------------------------------------------------------ */
void orc_deposit(const orc_uni *u, int box, const float *pos4, const float *mat, const float mono[4], float *fine) {
  memset(fine, 0, sizeof(float) * 4 * (ORC_FINE + 1));
  int N = u->N, pow2 = N > 0 && (N & (N - 1)) == 0;
  for (int v = 0; v < N; v++) {
    int i = pow2 ? (int)(((uint32_t)v * 40503u) & (uint32_t)(N - 1)) : v;   /* the reference's draw order */
    v3 p = ld3(pos4 + (size_t)i * 4);
    float pp[3] = {p.x, p.y, p.z}, g[3];
    float mr = mat[i];
    int mine = orc_box_of(u, pp, g);
    if (mine != box) {
      if (mine >= 0) continue;
      v3 r = vsub(vdivs(V3(mono[0], mono[1], mono[2]), fmaxf(mono[3], 1e-6f)), p);
      float inv = isqrt(vdot(r, r) + u->eps2Mesh);
      v3 w = vmuls(r, mr * inv * inv * inv);
      float *s = fine + 4 * ORC_FINE;
      s[0] += w.x; s[1] += w.y; s[2] += w.z; s[3] += mr;
      continue;
    }
    float f[3], t[3];
    for (int k = 0; k < 3; k++) { f[k] = floorf(g[k]); t[k] = g[k] - f[k]; }
    for (int k = 0; k < 8; k++) {
      int o[3] = {k & 1, (k >> 1) & 1, k >> 2};
      int c[3];
      float w3[3];
      for (int d = 0; d < 3; d++) { c[d] = (int)f[d] + o[d]; w3[d] = o[d] ? t[d] : 1.0f - t[d]; }
      if (c[0] > 63 || c[1] > 63 || c[2] > 63) continue;
      float w = w3[0] * w3[1] * w3[2] * mr;
      float *d = fine + 4 * fine_index(c[0], c[1], c[2]);
      d[0] += p.x * w; d[1] += p.y * w; d[2] += p.z * w; d[3] += 1.0f * w;
    }
  }
}

/* src/glsl-sim.js:222-251 COARSE_FS, MONO_FS */
void orc_coarse(const float *fine, float *coarse, float mono[4]) {
  for (int cz = 0; cz < 16; cz++)
    for (int cy = 0; cy < 16; cy++)
      for (int cx = 0; cx < 16; cx++) {
        float s[4] = {0, 0, 0, 0};
        for (int z = 0; z < 4; z++)
          for (int y = 0; y < 4; y++)
            for (int x = 0; x < 4; x++) {
              const float *f = fine + 4 * fine_index(cx * 4 + x, cy * 4 + y, cz * 4 + z);
              s[0] += f[0]; s[1] += f[1]; s[2] += f[2]; s[3] += f[3];
            }
        memcpy(coarse + 4 * coarse_index(cx, cy, cz), s, sizeof s);
      }
  /* MONO_FS sums the 64x64 coarse atlas row by row: texel (x, y) holds
   * block (x & 15, y & 15, (y >> 4) * 4 + (x >> 4)) */
  float s[4] = {0, 0, 0, 0};
  for (int y = 0; y < 64; y++)
    for (int x = 0; x < 64; x++) {
      const float *c = coarse + 4 * coarse_index(x & 15, y & 15, (y >> 4) * 4 + (x >> 4));
      s[0] += c[0]; s[1] += c[1]; s[2] += c[2]; s[3] += c[3];
    }
  memcpy(mono, s, sizeof s);
}

/* src/glsl-sim.js:263-295 FAR_FS */
void orc_far(const float *coarse, float *farA, float *farT0, float *farT1) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int b = 0; b < ORC_COARSE; b++) {
    int cx = b & 15, cy = (b >> 4) & 15, cz = b >> 8;
    const float *mc = coarse + 4 * b;
    float *A = farA + 4 * b, *T0 = farT0 + 4 * b, *T1 = farT1 + 4 * b;
    memset(A, 0, 16); memset(T0, 0, 16); memset(T1, 0, 16);
    if (mc[3] <= 0.0f) continue;
    v3 x = vdivs(ld3(mc), mc[3]);
    v3 acc = V3(0, 0, 0), td = V3(0, 0, 0), to = V3(0, 0, 0);
    float pot = 0.0f;
    for (int kz = 0; kz < 16; kz++)
      for (int ky = 0; ky < 16; ky++)
        for (int kx = 0; kx < 16; kx++) {
          int dx = abs(kx - cx), dy = abs(ky - cy), dz = abs(kz - cz);
          int dm = dx > dy ? dx : dy;
          if (dz > dm) dm = dz;
          if (dm <= 2) continue;
          const float *m = coarse + 4 * coarse_index(kx, ky, kz);
          if (m[3] <= 0.0f) continue;
          v3 r = vsub(vdivs(ld3(m), m[3]), x);
          float inv2 = 1.0f / vdot(r, r), inv = sqrtf(inv2), inv3 = inv * inv2, inv5 = inv3 * inv2;
          acc = vadd(acc, vmuls(r, m[3] * inv3));
          pot -= m[3] * inv;
          v3 rr = V3(3.0f * r.x * r.x * inv5 - inv3, 3.0f * r.y * r.y * inv5 - inv3, 3.0f * r.z * r.z * inv5 - inv3);
          td = vadd(td, V3(m[3] * rr.x, m[3] * rr.y, m[3] * rr.z));
          v3 ro = V3(3.0f * (r.x * r.y) * inv5, 3.0f * (r.x * r.z) * inv5, 3.0f * (r.y * r.z) * inv5);
          to = vadd(to, V3(m[3] * ro.x, m[3] * ro.y, m[3] * ro.z));
        }
    A[0] = acc.x; A[1] = acc.y; A[2] = acc.z; A[3] = pot;
    T0[0] = td.x; T0[1] = td.y; T0[2] = td.z; T0[3] = to.x;
    T1[0] = to.y; T1[1] = to.z; T1[2] = 0; T1[3] = 0;
  }
}

/* src/glsl-sim.js:303-352 CELL_FS */
void orc_cell(const orc_uni *u, const float *fine, const float *coarse, const float *farA,
              const float *farT0, const float *farT1, float *force) {
  memcpy(force + 4 * ORC_FINE, fine + 4 * ORC_FINE, 16);   /* the scratch row, carried through */
#pragma omp parallel for schedule(dynamic, 256)
  for (int ci = 0; ci < ORC_FINE; ci++) {
    int c[3] = {ci & 63, (ci >> 6) & 63, ci >> 12};
    const float *mc = fine + 4 * ci;
    float *o = force + 4 * ci;
    if (mc[3] <= 0.0f) { o[0] = o[1] = o[2] = o[3] = 0.0f; continue; }
    v3 x = vdivs(ld3(mc), mc[3]);
    int cc[3] = {c[0] >> 2, c[1] >> 2, c[2] >> 2};
    v3 acc = V3(0, 0, 0);
    float pot = 0.0f;
    for (int kz = -2; kz <= 2; kz++)
      for (int ky = -2; ky <= 2; ky++)
        for (int kx = -2; kx <= 2; kx++) {
          int k[3] = {cc[0] + kx, cc[1] + ky, cc[2] + kz};
          if (k[0] < 0 || k[1] < 0 || k[2] < 0 || k[0] > 15 || k[1] > 15 || k[2] > 15) continue;
          const float *m = coarse + 4 * coarse_index(k[0], k[1], k[2]);
          if (m[3] <= 0.0f) continue;
          for (int fz = 0; fz < 4; fz++)
            for (int fy = 0; fy < 4; fy++)
              for (int fx = 0; fx < 4; fx++) {
                int f[3] = {k[0] * 4 + fx, k[1] * 4 + fy, k[2] * 4 + fz};
                if (f[0] == c[0] && f[1] == c[1] && f[2] == c[2]) continue;
                const float *mf = fine + 4 * fine_index(f[0], f[1], f[2]);
                if (mf[3] <= 0.0f) continue;
                v3 r = vsub(vdivs(ld3(mf), mf[3]), x);
                float inv = isqrt(vdot(r, r) + u->eps2Cell);
                acc = vadd(acc, vmuls(r, mf[3] * inv * inv * inv));
                pot -= mf[3] * inv;
              }
        }
    int ca = coarse_index(cc[0], cc[1], cc[2]);
    const float *mb = coarse + 4 * ca, *fa = farA + 4 * ca, *t0 = farT0 + 4 * ca, *t1 = farT1 + 4 * ca;
    v3 d = vsub(x, vdivs(ld3(mb), mb[3]));
    v3 Td = V3(t0[0] * d.x + t0[3] * d.y + t1[0] * d.z,
               t0[3] * d.x + t0[1] * d.y + t1[1] * d.z,
               t1[0] * d.x + t1[1] * d.y + t0[2] * d.z);
    acc = vadd(acc, vadd(ld3(fa), Td));
    pot += fa[3] - vdot(ld3(fa), d) - 0.5f * vdot(d, Td);
    o[0] = acc.x * u->Gm; o[1] = acc.y * u->Gm; o[2] = acc.z * u->Gm; o[3] = pot * u->Gm;
  }
}

/* ------------------------------------------------------------------ */
/* The stencil-split P3M (no counterpart in the reference; the library's ccs_set_pp_split).  The cell pass  */
/* of CELL_FS (src/glsl-sim.js:303-352) with the node pairs within S cells (Chebyshev) left out, no         */
/* softening, and the tidal tensor summed beside the pull; then every particle's pairs inside the stencil,  */
/* each weighted by its share of cloud-in-cell node pairs within S; then the gather, first order from each  */
/* node's centre of mass.                                                                                    */
/* ------------------------------------------------------------------ */
static v3 mass_at(const orc_uni *u, v3 p, const float *mono);
static v3 cross_at(const orc_uni *u, const float *other, const float *mine);

/* each fine cell's second moment about its own centre of mass (fine, after orc_deposit), from the particles'
 * cloud-in-cell weights: Q = sum w m (x - X)(x - X)^T, two planes of (64^3 + 1) float4, (Qxx Qyy Qzz Qxy) and
 * (Qxz Qyz) -- the split form's node quadrupoles (binary64 sums, stored as binary32) */
void orc_node_moments(const orc_uni *u, int box, const float *pos4, const float *mat, const float *fine,
                      float *fineQ) {
  double *q = (double *)calloc((size_t)ORC_FINE * 6, sizeof(double));
  for (int i = 0; i < u->N; i++) {
    float pp[3] = {pos4[4 * (size_t)i], pos4[4 * (size_t)i + 1], pos4[4 * (size_t)i + 2]}, g[3];
    if (orc_box_of(u, pp, g) != box) continue;
    float f[3], t[3];
    for (int k = 0; k < 3; k++) { f[k] = floorf(g[k]); t[k] = g[k] - f[k]; }
    for (int k = 0; k < 8; k++) {
      int o[3] = {k & 1, (k >> 1) & 1, k >> 2}, c[3];
      double w = mat[i];
      for (int d = 0; d < 3; d++) { c[d] = (int)f[d] + o[d]; w *= o[d] ? t[d] : 1.0 - t[d]; }
      if (c[0] > 63 || c[1] > 63 || c[2] > 63) continue;
      int ci = fine_index(c[0], c[1], c[2]);
      const float *m = fine + 4 * (size_t)ci;
      double d[3] = {pp[0] - (double)m[0] / m[3], pp[1] - (double)m[1] / m[3], pp[2] - (double)m[2] / m[3]};
      double *Q = q + 6 * (size_t)ci;
      Q[0] += w * d[0] * d[0]; Q[1] += w * d[1] * d[1]; Q[2] += w * d[2] * d[2];
      Q[3] += w * d[0] * d[1]; Q[4] += w * d[0] * d[2]; Q[5] += w * d[1] * d[2];
    }
  }
  memset(fineQ, 0, sizeof(float) * 8 * (ORC_FINE + 1));
  for (int ci = 0; ci < ORC_FINE; ci++) {
    const double *Q = q + 6 * (size_t)ci;
    float *a = fineQ + 4 * (size_t)ci, *b = fineQ + 4 * ((size_t)ORC_FINE + 1 + ci);
    a[0] = (float)Q[0]; a[1] = (float)Q[1]; a[2] = (float)Q[2]; a[3] = (float)Q[3];
    b[0] = (float)Q[4]; b[1] = (float)Q[5];
  }
  free(q);
}

/* one source's second moment Q (Qxx Qyy Qzz Qxy Qxz Qyz) at offset r from the cell (r = source - cell): its
 * quadrupole pull a = -3 Q r / r^5 + 7.5 (r Q r) r / r^7 - 1.5 tr(Q) r / r^5 and potential
 * -0.5 (3 r Q r / r^5 - tr(Q) / r^3), added to acc and pot */
static void add_quad(double *acc, double *pot, const double *r, const double *Q, double inv) {
  double inv2 = inv * inv, inv3 = inv * inv2, inv5 = inv3 * inv2;
  double Qr[3] = {Q[0] * r[0] + Q[3] * r[1] + Q[4] * r[2], Q[3] * r[0] + Q[1] * r[1] + Q[5] * r[2],
                  Q[4] * r[0] + Q[5] * r[1] + Q[2] * r[2]};
  double rQr = r[0] * Qr[0] + r[1] * Qr[1] + r[2] * Qr[2], tr = Q[0] + Q[1] + Q[2];
  double c1 = 7.5 * rQr * inv5 * inv2 - 1.5 * tr * inv5;
  for (int a = 0; a < 3; a++) acc[a] += c1 * r[a] - 3.0 * inv5 * Qr[a];
  *pot -= 0.5 * (3.0 * rQr * inv5 - tr * inv3);
}

/* one source of mass M at offset r from the cell's centre of mass (r = source - cell): the second gradient
 * of its pull at the cell, G_abc = d2 F_a / dx_b dx_c = M (15 r_a r_b r_c / r^7 - 3 (d_ab r_c + d_ac r_b +
 * d_bc r_a) / r^5), added to G = (Gxxx Gyyy Gzzz Gxyz, Gxxy Gxxz Gxyy Gyyz, Gxzz Gyzz); a5 = 3 M / r^5 and
 * a7 = 15 M / r^7 */
static void add_tide2(double *G, double rx, double ry, double rz, double a5, double a7) {
  G[0] += a7 * rx * rx * rx - 3.0 * a5 * rx;
  G[1] += a7 * ry * ry * ry - 3.0 * a5 * ry;
  G[2] += a7 * rz * rz * rz - 3.0 * a5 * rz;
  G[3] += a7 * rx * ry * rz;
  G[4] += a7 * rx * rx * ry - a5 * ry;
  G[5] += a7 * rx * rx * rz - a5 * rz;
  G[6] += a7 * rx * ry * ry - a5 * rx;
  G[7] += a7 * ry * ry * rz - a5 * rz;
  G[8] += a7 * rx * rz * rz - a5 * rx;
  G[9] += a7 * ry * rz * rz - a5 * ry;
}

void orc_cell_tide(const orc_uni *u, int S, const float *fine, const float *coarse, const float *fineQ,
                   float *force, float *tide0, float *tide1, float *tide2) {
  const float eps2 = 1e-6f * u->eps2Mesh;   /* keeps two coinciding centres of mass finite, as the library's */
  memcpy(force + 4 * ORC_FINE, fine + 4 * ORC_FINE, 16);
  /* each occupied block's centre of mass and second moment, from its occupied cells at their centres of mass */
  double *bq = (double *)calloc((size_t)ORC_COARSE * 10, sizeof(double));   /* X[3], M, Q[6] */
  for (int b = 0; b < ORC_COARSE; b++) {
    const float *m = coarse + 4 * b;
    double *q = bq + 10 * b;
    if (m[3] <= 0.0f) continue;
    q[0] = m[0] / m[3]; q[1] = m[1] / m[3]; q[2] = m[2] / m[3]; q[3] = m[3];
    int bx = b & 15, by = (b >> 4) & 15, bz = b >> 8;
    for (int c = 0; c < 64; c++) {
      const float *f = fine + 4 * fine_index(bx * 4 + (c & 3), by * 4 + ((c >> 2) & 3), bz * 4 + (c >> 4));
      if (f[3] <= 0.0f) continue;
      double d[3] = {f[0] / f[3] - q[0], f[1] / f[3] - q[1], f[2] / f[3] - q[2]};
      q[4] += f[3] * d[0] * d[0]; q[5] += f[3] * d[1] * d[1]; q[6] += f[3] * d[2] * d[2];
      q[7] += f[3] * d[0] * d[1]; q[8] += f[3] * d[0] * d[2]; q[9] += f[3] * d[1] * d[2];
      if (fineQ) {   /* the cell's own spread, by parallel axes */
        size_t fi = (size_t)fine_index(bx * 4 + (c & 3), by * 4 + ((c >> 2) & 3), bz * 4 + (c >> 4));
        const float *a = fineQ + 4 * fi, *b = fineQ + 4 * ((size_t)ORC_FINE + 1 + fi);
        q[4] += a[0]; q[5] += a[1]; q[6] += a[2]; q[7] += a[3]; q[8] += b[0]; q[9] += b[1];
      }
    }
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (int ci = 0; ci < ORC_FINE; ci++) {
    int c[3] = {ci & 63, (ci >> 6) & 63, ci >> 12};
    const float *mc = fine + 4 * ci;
    float *o = force + 4 * ci, *T0 = tide0 + 4 * ci, *T1 = tide1 + 4 * ci;
    if (mc[3] <= 0.0f) {
      o[0] = o[1] = o[2] = o[3] = 0.0f;
      continue;
    }
    v3 x = vdivs(ld3(mc), mc[3]);
    int cc[3] = {c[0] >> 2, c[1] >> 2, c[2] >> 2};
    double acc[3] = {0, 0, 0}, pot = 0, T[6] = {0, 0, 0, 0, 0, 0};   /* Txx Tyy Tzz Txy Txz Tyz */
    double G[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    /* near: the fine cells of the 5^3 blocks around, beyond the stencil, unsoftened */
    for (int kz = -2; kz <= 2; kz++)
      for (int ky = -2; ky <= 2; ky++)
        for (int kx = -2; kx <= 2; kx++) {
          int k[3] = {cc[0] + kx, cc[1] + ky, cc[2] + kz};
          if (k[0] < 0 || k[1] < 0 || k[2] < 0 || k[0] > 15 || k[1] > 15 || k[2] > 15) continue;
          const float *m = coarse + 4 * coarse_index(k[0], k[1], k[2]);
          if (m[3] <= 0.0f) continue;
          for (int fz = 0; fz < 4; fz++)
            for (int fy = 0; fy < 4; fy++)
              for (int fx = 0; fx < 4; fx++) {
                int f[3] = {k[0] * 4 + fx, k[1] * 4 + fy, k[2] * 4 + fz};
                int dx = abs(f[0] - c[0]), dy = abs(f[1] - c[1]), dz = abs(f[2] - c[2]);
                int cheb = dx > dy ? (dx > dz ? dx : dz) : (dy > dz ? dy : dz);
                if (cheb <= S) continue;
                const float *mf = fine + 4 * fine_index(f[0], f[1], f[2]);
                if (mf[3] <= 0.0f) continue;
                v3 r = vsub(vdivs(ld3(mf), mf[3]), x);
                double rx = r.x, ry = r.y, rz = r.z, M = mf[3];
                double inv = 1.0 / sqrt(rx * rx + ry * ry + rz * rz + eps2), inv2 = inv * inv;
                double a3 = M * inv * inv2, a5 = 3.0 * a3 * inv2;
                acc[0] += rx * a3; acc[1] += ry * a3; acc[2] += rz * a3;
                pot -= M * inv;
                T[0] += a5 * rx * rx - a3; T[1] += a5 * ry * ry - a3; T[2] += a5 * rz * rz - a3;
                T[3] += a5 * rx * ry; T[4] += a5 * rx * rz; T[5] += a5 * ry * rz;
                add_tide2(G, rx, ry, rz, a5, 5.0 * a5 * inv2);
                if (fineQ) {   /* the source's spread as a quadrupole */
                  size_t fi = (size_t)fine_index(f[0], f[1], f[2]);
                  const float *qa = fineQ + 4 * fi, *qb = fineQ + 4 * ((size_t)ORC_FINE + 1 + fi);
                  double Q[6] = {qa[0], qa[1], qa[2], qa[3], qb[0], qb[1]}, rr[3] = {rx, ry, rz};
                  add_quad(acc, &pot, rr, Q, inv);
                }
              }
        }
    /* far: every occupied block more than two from the cell's own, monopole + quadrupole, at the cell */
    for (int b = 0; b < ORC_COARSE; b++) {
      const double *q = bq + 10 * b;
      if (q[3] <= 0.0) continue;
      int bx = b & 15, by = (b >> 4) & 15, bz = b >> 8;
      int dx = abs(bx - cc[0]), dy = abs(by - cc[1]), dz = abs(bz - cc[2]);
      if ((dx > dy ? (dx > dz ? dx : dz) : (dy > dz ? dy : dz)) <= 2) continue;
      double r[3] = {q[0] - x.x, q[1] - x.y, q[2] - x.z};
      double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2], inv = 1.0 / sqrt(r2), inv2 = inv * inv;
      double inv3 = inv * inv2, inv5 = inv3 * inv2, M = q[3], a3 = M * inv3, a5 = 3.0 * a3 * inv2;
      acc[0] += r[0] * a3; acc[1] += r[1] * a3; acc[2] += r[2] * a3;
      pot -= M * inv;
      T[0] += a5 * r[0] * r[0] - a3; T[1] += a5 * r[1] * r[1] - a3; T[2] += a5 * r[2] * r[2] - a3;
      T[3] += a5 * r[0] * r[1]; T[4] += a5 * r[0] * r[2]; T[5] += a5 * r[1] * r[2];
      add_tide2(G, r[0], r[1], r[2], a5, 5.0 * a5 * inv2);
      double Qr[3] = {q[4] * r[0] + q[7] * r[1] + q[8] * r[2], q[7] * r[0] + q[5] * r[1] + q[9] * r[2],
                      q[8] * r[0] + q[9] * r[1] + q[6] * r[2]};
      double rQr = r[0] * Qr[0] + r[1] * Qr[1] + r[2] * Qr[2], tr = q[4] + q[5] + q[6];
      double c1 = 7.5 * rQr * inv5 * inv2 - 1.5 * tr * inv5;
      for (int a = 0; a < 3; a++) acc[a] += c1 * r[a] - 3.0 * inv5 * Qr[a];
      pot -= 0.5 * (3.0 * rQr * inv5 - tr * inv3);
    }
    o[0] = (float)(acc[0] * u->Gm); o[1] = (float)(acc[1] * u->Gm); o[2] = (float)(acc[2] * u->Gm);
    o[3] = (float)(pot * u->Gm);
    T0[0] = (float)(T[0] * u->Gm); T0[1] = (float)(T[1] * u->Gm); T0[2] = (float)(T[2] * u->Gm);
    T0[3] = (float)(T[3] * u->Gm);
    T1[0] = (float)(T[4] * u->Gm); T1[1] = (float)(T[5] * u->Gm); T1[2] = T1[3] = 0.0f;
    if (tide2) {   /* three planes of (64^3 + 1) float4, as the library's */
      for (int k = 0; k < 10; k++) tide2[(size_t)(k >> 2) * 4 * (ORC_FINE + 1) + 4 * (size_t)ci + (k & 3)] = (float)(G[k] * u->Gm);
      tide2[2 * 4 * (size_t)(ORC_FINE + 1) + 4 * (size_t)ci + 2] = 0.0f;
      tide2[2 * 4 * (size_t)(ORC_FINE + 1) + 4 * (size_t)ci + 3] = 0.0f;
    }
  }
  free(bq);
}

static double split_w(int D, int S, double ti, double tj) {
  if (D <= S - 1 && D >= 1 - S) return 1.0;
  if (D == S) return (1.0 - tj) + ti * tj;
  if (D == -S) return (1.0 - ti) + ti * tj;
  if (D == S + 1) return ti * (1.0 - tj);
  if (D == -S - 1) return (1.0 - ti) * tj;
  return 0.0;
}

void orc_pp_split(const orc_uni *u, int S, const float *pos4, const float *mat, float *out4) {
  const int N = u->N;
  int *box = (int *)malloc(sizeof(int) * N), *b = (int *)malloc(sizeof(int) * 3 * N);
  double *t = (double *)malloc(sizeof(double) * 3 * N);
  for (int i = 0; i < N; i++) {
    float p[3] = {pos4[4 * (size_t)i], pos4[4 * (size_t)i + 1], pos4[4 * (size_t)i + 2]}, g[3];
    box[i] = orc_box_of(u, p, g);
    for (int k = 0; k < 3; k++) {
      float f = floorf(g[k]);
      b[3 * i + k] = (int)f;
      t[3 * i + k] = (double)(g[k] - f);
    }
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < N; i++) {
    float *o = out4 + 4 * (size_t)i;
    o[0] = o[1] = o[2] = o[3] = 0.0f;
    if (box[i] < 0) continue;
    double acc[3] = {0, 0, 0}, pot = 0;
    const double px = pos4[4 * (size_t)i], py = pos4[4 * (size_t)i + 1], pz = pos4[4 * (size_t)i + 2];
    for (int j = 0; j < N; j++) {
      if (j == i || box[j] != box[i]) continue;
      int D0 = b[3 * j] - b[3 * i], D1 = b[3 * j + 1] - b[3 * i + 1], D2 = b[3 * j + 2] - b[3 * i + 2];
      if (abs(D0) > S + 1 || abs(D1) > S + 1 || abs(D2) > S + 1) continue;
      double W = split_w(D0, S, t[3 * i], t[3 * j]) * split_w(D1, S, t[3 * i + 1], t[3 * j + 1]) *
                 split_w(D2, S, t[3 * i + 2], t[3 * j + 2]);
      double dx = pos4[4 * (size_t)j] - px, dy = pos4[4 * (size_t)j + 1] - py, dz = pos4[4 * (size_t)j + 2] - pz;
      double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz + (double)u->a2);
      double w = mat[j] * W;
      acc[0] += dx * w * inv * inv * inv; acc[1] += dy * w * inv * inv * inv; acc[2] += dz * w * inv * inv * inv;
      pot -= w * inv;
    }
    o[0] = (float)(acc[0] * u->Gm); o[1] = (float)(acc[1] * u->Gm); o[2] = (float)(acc[2] * u->Gm);
    o[3] = (float)(pot * u->Gm);
  }
  free(box); free(b); free(t);
}

void orc_gather_split(const orc_uni *u, const float *pos4, const float *fineA, const float *forceA,
                      const float *tideA0, const float *tideA1, const float *tideA2, const float *fineB,
                      const float *forceB, const float *tideB0, const float *tideB1, const float *tideB2,
                      const float *monoA, const float *monoB, const float *ppAll, float *grav4) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < u->N; i++) {
    v3 p = ld3(pos4 + 4 * (size_t)i), grav = V3(0, 0, 0);
    float pp[3] = {p.x, p.y, p.z}, g[3];
    int box = orc_box_of(u, pp, g);
    if (box >= 0) {
      const float *F = box == 0 ? forceA : forceB, *M = box == 0 ? fineA : fineB;
      const float *T0 = box == 0 ? tideA0 : tideB0, *T1 = box == 0 ? tideA1 : tideB1;
      const float *T2 = box == 0 ? tideA2 : tideB2;
      float f[3], t[3];
      int cf[3];
      for (int k = 0; k < 3; k++) { f[k] = floorf(g[k]); t[k] = g[k] - f[k]; cf[k] = (int)f[k]; }
      for (int k = 0; k < 8; k++) {
        int o[3] = {k & 1, (k >> 1) & 1, k >> 2}, at[3];
        float w3[3];
        for (int d = 0; d < 3; d++) {
          w3[d] = o[d] ? t[d] : 1.0f - t[d];
          at[d] = cf[d] + o[d] < 63 ? cf[d] + o[d] : 63;
        }
        size_t c = (size_t)fine_index(at[0], at[1], at[2]);
        const float *m = M + 4 * c, *fv = F + 4 * c, *t0 = T0 + 4 * c, *t1 = T1 + 4 * c;
        if (!(m[3] > 0.0f)) continue;
        v3 d = vsub(p, vdivs(ld3(m), m[3]));
        v3 Td = V3(t0[0] * d.x + t0[3] * d.y + t1[0] * d.z,
                   t0[3] * d.x + t0[1] * d.y + t1[1] * d.z,
                   t1[0] * d.x + t1[1] * d.y + t0[2] * d.z);
        if (T2) {   /* second order: half the pull's second gradient along d, twice */
          const float *g0 = T2 + 4 * c, *g1 = T2 + 4 * ((size_t)(ORC_FINE + 1) + c), *g2 = T2 + 4 * (2 * (size_t)(ORC_FINE + 1) + c);
          float xx = d.x * d.x, yy = d.y * d.y, zz = d.z * d.z, xy = d.x * d.y, xz = d.x * d.z, yz = d.y * d.z;
          Td = vadd(Td, V3(0.5f * (g0[0] * xx + g1[2] * yy + g2[0] * zz) + g1[0] * xy + g1[1] * xz + g0[3] * yz,
                           0.5f * (g1[0] * xx + g0[1] * yy + g2[1] * zz) + g1[2] * xy + g0[3] * xz + g1[3] * yz,
                           0.5f * (g1[1] * xx + g1[3] * yy + g0[2] * zz) + g0[3] * xy + g2[0] * xz + g2[1] * yz));
        }
        grav = vadd(grav, vmuls(vadd(ld3(fv), Td), w3[0] * w3[1] * w3[2]));
      }
      grav = vsub(grav, vmuls(ld3(F + 4 * ORC_FINE), u->Gm));
      if (u->boxB > 0.5f) grav = vadd(grav, box == 0 ? cross_at(u, monoB, monoA) : cross_at(u, monoA, monoB));
    } else {
      grav = mass_at(u, p, monoA);
      if (u->boxB > 0.5f) grav = vadd(grav, mass_at(u, p, monoB));
    }
    grav = vadd(grav, ld3(ppAll + 4 * (size_t)i));
    float *o = grav4 + 4 * (size_t)i;
    o[0] = grav.x; o[1] = grav.y; o[2] = grav.z; o[3] = 0.0f;
  }
}

/* ------------------------------------------------------------------ */
/* src/glsl-sim.js:676-754 PPGATHER_FS, PPFORCE_FS                      */
/* ------------------------------------------------------------------ */
void orc_pp_gather(const orc_uni *u, const float *pos4, const float *mat, const int *index, int cap,
                   float *list4, float *box) {
  for (int s = 0; s < cap; s++) {
    int i = index[s];
    if (i < 0) { list4[4 * s] = list4[4 * s + 1] = list4[4 * s + 2] = list4[4 * s + 3] = 0.0f; box[s] = -1.0f; continue; }
    float p[3] = {pos4[4 * (size_t)i], pos4[4 * (size_t)i + 1], pos4[4 * (size_t)i + 2]}, g[3];
    box[s] = (float)orc_box_of(u, p, g);
    list4[4 * s] = p[0]; list4[4 * s + 1] = p[1]; list4[4 * s + 2] = p[2]; list4[4 * s + 3] = mat[i];
  }
}

static inline float smoothstepf(float e0, float e1, float x) {
  float t = fclampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

void orc_pp_force(const orc_uni *u, const float *list4, const float *box, int count, int cap,
                  const float *tab, float *force) {
  int share = (count + 3) >> 2;
#pragma omp parallel for schedule(dynamic, 64)
  for (int w = 0; w < 4 * cap; w++) {
    int slice = w / cap, me = w % cap;
    float *o = force + 4 * (size_t)w;
    int j0 = slice * share, j1 = j0 + share < count ? j0 + share : count;
    const float *P = list4 + 4 * me;
    if (me >= count || P[3] == 0.0f) { o[0] = o[1] = o[2] = o[3] = 0.0f; continue; }
    float myBox = box[me];
    v3 acc = V3(0, 0, 0);
    float pot = 0.0f, cut2 = u->cut * u->cut, a = sqrtf(u->a2);
    for (int j = j0; j < j1; j++) {
      if (j == me) continue;
      const float *Q = list4 + 4 * j;
      v3 d = vsub(ld3(Q), ld3(P));
      float r2 = vdot(d, d);
      if (r2 >= cut2) continue;
      float r = sqrtf(r2);
      float x = fclampf(r / u->cut * 64.0f - 0.5f, 0.0f, 63.0f);
      int k = (int)x, k1 = k + 1 < 63 ? k + 1 : 63;
      float t = x - (float)k;
      float invN = isqrt(r2 + u->a2);
      float taper = smoothstepf(u->cut, 0.8f * u->cut, r);
      float same = (myBox >= 0.0f && box[j] == myBox) ? 1.0f : 0.0f;
      float Tx = (tab[2 * k] * (1.0f - t) + tab[2 * k1] * t) * same;
      float Ty = (tab[2 * k + 1] * (1.0f - t) + tab[2 * k1 + 1] * t) * same;
      float fn = invN * invN * invN * r - Tx / fmaxf(r2, u->a2), mj = Q[3];
      acc = vadd(acc, vmuls(vdivs(d, fmaxf(r, 1e-6f)), mj * fn * taper));
      pot += mj * (-invN - Ty / fmaxf(r, a)) * taper;
    }
    o[0] = acc.x * u->Gm; o[1] = acc.y * u->Gm; o[2] = acc.z * u->Gm; o[3] = pot * u->Gm;
  }
}

/* ------------------------------------------------------------------ */
/* src/glsl-sim.js:57-66 GLSL_MASS                                     */
/* ------------------------------------------------------------------ */
static v3 mass_at(const orc_uni *u, v3 p, const float *mono) {
  v3 r = vsub(vdivs(ld3(mono), fmaxf(mono[3], 1e-6f)), p);
  float inv = isqrt(vdot(r, r) + u->eps2Mesh);
  return vmuls(r, u->Gm * mono[3] * inv * inv * inv);
}
static float pot_at(const orc_uni *u, v3 p, const float *mono) {
  v3 r = vsub(vdivs(ld3(mono), fmaxf(mono[3], 1e-6f)), p);
  return -u->Gm * mono[3] * isqrt(vdot(r, r) + u->eps2Mesh);
}
static v3 cross_at(const orc_uni *u, const float *other, const float *mine) {
  v3 d = vsub(vdivs(ld3(other), fmaxf(other[3], 1e-6f)), vdivs(ld3(mine), fmaxf(mine[3], 1e-6f)));
  float inv = isqrt(vdot(d, d) + u->eps2Mesh);
  return vmuls(d, u->Gm * other[3] * inv * inv * inv);
}

/* ------------------------------------------------------------------ */
/* src/glsl-sim.js:362-512 simFS({gravity:'mesh'})                      */
/* ------------------------------------------------------------------ */
void orc_sim_pass(const orc_uni *u, const float *pos4, const float *vel4, const float *mat, const float *qa,
                  const uint32_t *seats, const float *forceA, const float *monoA, const float *forceB,
                  const float *monoB, const int *ppslot, const float *ppforce, int cap,
                  float *pos_o, float *vel_o, float *aux_o, float *q_o) {
#pragma omp parallel for schedule(static)
  for (int me = 0; me < u->N; me++) {
    const float *P = pos4 + 4 * (size_t)me, *V = vel4 + 4 * (size_t)me;
    v3 p = ld3(P), v = ld3(V);
    float body = P[3];
    float ri = mat[me];
    float ci = ri * (fmodg(body, 4.0f) < 0.5f ? u->cpIron : 1.0f);
    float Ti = V[3];
    v3 push = V3(0, 0, 0);
    float nb = 0.0f, lost = 0.0f, flow = 0.0f;
    int c[3] = {(int)floorf(p.x * u->invCell), (int)floorf(p.y * u->invCell), (int)floorf(p.z * u->invCell)};
    v3 c0 = V3((float)c[0] * u->cell, (float)c[1] * u->cell, (float)c[2] * u->cell);
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          v3 lo = V3(c0.x + (float)dx * u->cell, c0.y + (float)dy * u->cell, c0.z + (float)dz * u->cell);
          v3 hi = V3(lo.x + u->cell, lo.y + u->cell, lo.z + u->cell);
          v3 q = vsub(V3(fclampf(p.x, lo.x, hi.x), fclampf(p.y, lo.y, hi.y), fclampf(p.z, lo.z, hi.z)), p);
          if (vdot(q, q) > u->link2) continue;
          int ax, ay;
          orc_hash(u, c[0] + dx, c[1] + dy, c[2] + dz, &ax, &ay);
          const uint32_t *s = seats + ((size_t)ay * u->AW + ax) * ORC_SEATS;
          for (int k = 0; k < ORC_SEATS; k++) {
            uint32_t sv = s[k];
            if (sv & 0x80000000u) break;
            int j = (int)(sv & 0x3FFFFu);
            if (j == me) continue;
            v3 sp = V3(((float)((sv >> 18) & 15u) + 0.5f) / 15.0f, ((float)((sv >> 22) & 15u) + 0.5f) / 15.0f,
                       ((float)((sv >> 26) & 15u) + 0.5f) / 15.0f);
            v3 dq = vsub(vadd(lo, vmuls(sp, u->cell)), p);
            if (vdot(dq, dq) > u->reach2) continue;
            const float *Pj = pos4 + 4 * (size_t)j;
            v3 d = vsub(ld3(Pj), p);
            float r2 = vdot(d, d);
            if (r2 < u->link2) {
              float r = sqrtf(r2);
              v3 n = vdivs(d, fmaxf(r, 1e-6f));
              float ov = u->touch - r;
              if (ov > 0.0f) {
                const float *Vj = vel4 + 4 * (size_t)j;
                float rj = mat[j];
                float cij = u->C * sqrtf(2.0f * ri * rj / (ri + rj));
                float vn = vdot(vsub(ld3(Vj), v), n);
                float fs = u->K * ov - cij * vn, fn = fmaxf(fs, 0.0f), on = fs >= 0.0f ? 1.0f : 0.0f;
                push = vsub(push, vmuls(n, fn));
                lost += cij * vn * vn * on + u->K * ov * vn * (1.0f - on);
                float cj = rj * (fmodg(Pj[3], 4.0f) < 0.5f ? u->cpIron : 1.0f);
                flow += (Vj[3] - Ti) * (2.0f * ci * cj / (ci + cj));
              }
              nb += 1.0f;
            }
          }
        }
    /* SIM_GRAV_FIELD (src/glsl-sim.js:490-492) or SIM_GRAV_MESH */
    v3 grav = V3(0, 0, 0);
    float pp[3] = {p.x, p.y, p.z}, g[3];
    int box = u->field > 0.5f ? -2 : orc_box_of(u, pp, g);
    if (box == -2) {
      grav = ld3(u->gField);
    } else if (box >= 0) {
      const float *F = box == 0 ? forceA : forceB;
      float f[3], t[3];
      int cf[3];
      for (int k = 0; k < 3; k++) { f[k] = floorf(g[k]); t[k] = g[k] - f[k]; cf[k] = (int)f[k]; }
      for (int k = 0; k < 8; k++) {
        int o[3] = {k & 1, (k >> 1) & 1, k >> 2}, at[3];
        float w3[3];
        for (int d = 0; d < 3; d++) {
          w3[d] = o[d] ? t[d] : 1.0f - t[d];
          at[d] = cf[d] + o[d] < 63 ? cf[d] + o[d] : 63;
        }
        const float *fv = F + 4 * fine_index(at[0], at[1], at[2]);
        grav = vadd(grav, vmuls(ld3(fv), w3[0] * w3[1] * w3[2]));
      }
      grav = vsub(grav, vmuls(ld3(F + 4 * ORC_FINE), u->Gm));
      if (u->boxB > 0.5f) grav = vadd(grav, box == 0 ? cross_at(u, monoB, monoA) : cross_at(u, monoA, monoB));
    } else {
      grav = mass_at(u, p, monoA);
      if (u->boxB > 0.5f) grav = vadd(grav, mass_at(u, p, monoB));
    }
    int seat = box == -2 ? -1 : ppslot[me];
    if (seat >= 0)
      for (int s = 0; s < 4; s++) grav = vadd(grav, ld3(ppforce + 4 * ((size_t)s * cap + seat)));
    /* SIM_POST */
    float sc = u->invM / ri;
    v = V3(v.x + (push.x * sc * u->dt + grav.x * u->gdt), v.y + (push.y * sc * u->dt + grav.y * u->gdt),
           v.z + (push.z * sc * u->dt + grav.z * u->gdt));
    const float *spin = body < 3.5f ? u->spin0 : u->spin1, *cen = body < 3.5f ? u->cen0 : u->cen1;
    v3 vr = vcross(ld3(spin), vsub(p, ld3(cen)));
    if (u->settle > 0.5f) {
      v3 dv = vmuls(vsub(v, vr), u->damp);
      float sp = sqrtf(vdot(dv, dv));
      v = vadd(vr, vmuls(dv, fminf(1.0f, u->creep / fmaxf(sp, 1e-9f))));
    }
    if (u->kick > 0.5f) v = vadd(ld3(body < 3.5f ? u->bulk0 : u->bulk1), vr);
    float Q = u->settle > 0.5f ? 0.0f : qa[me] + (lost + flow * u->kappa / u->tK) * u->dt;
    if (u->frozen >= 0.0f && fabsf(body - u->frozen) < 0.5f) v = V3(0, 0, 0);   /* src/glsl-sim.js:523-526 */
    p = vadd(p, vmuls(v, u->dt));
    float *po = pos_o + 4 * (size_t)me, *vo = vel_o + 4 * (size_t)me, *ao = aux_o + 4 * (size_t)me;
    po[0] = p.x; po[1] = p.y; po[2] = p.z; po[3] = body;
    vo[0] = v.x; vo[1] = v.y; vo[2] = v.z; vo[3] = u->tK * Q / ci;
    ao[0] = grav.x; ao[1] = grav.y; ao[2] = grav.z; ao[3] = nb;
    q_o[me] = Q;
  }
}

/* src/glsl-sim.js:415-450: the same 27-cell walk, seat cull and link test as orc_sim_pass, recording the
 * pairs instead of summing their forces */
void orc_contact_pairs(const orc_uni *u, const float *pos4, const uint32_t *seats, int cap, int32_t *counts,
                       uint32_t *pairs) {
#pragma omp parallel for schedule(static)
  for (int me = 0; me < u->N; me++) {
    const float *P = pos4 + 4 * (size_t)me;
    v3 p = ld3(P);
    int n = 0;
    uint32_t *row = pairs + (size_t)me * cap;
    for (int k = 0; k < cap; k++) row[k] = 0xFFFFFFFFu;
    int c[3] = {(int)floorf(p.x * u->invCell), (int)floorf(p.y * u->invCell), (int)floorf(p.z * u->invCell)};
    v3 c0 = V3((float)c[0] * u->cell, (float)c[1] * u->cell, (float)c[2] * u->cell);
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          v3 lo = V3(c0.x + (float)dx * u->cell, c0.y + (float)dy * u->cell, c0.z + (float)dz * u->cell);
          v3 hi = V3(lo.x + u->cell, lo.y + u->cell, lo.z + u->cell);
          v3 q = vsub(V3(fclampf(p.x, lo.x, hi.x), fclampf(p.y, lo.y, hi.y), fclampf(p.z, lo.z, hi.z)), p);
          if (vdot(q, q) > u->link2) continue;
          int ax, ay;
          orc_hash(u, c[0] + dx, c[1] + dy, c[2] + dz, &ax, &ay);
          const uint32_t *s = seats + ((size_t)ay * u->AW + ax) * ORC_SEATS;
          for (int k = 0; k < ORC_SEATS; k++) {
            uint32_t sv = s[k];
            if (sv & 0x80000000u) break;
            int j = (int)(sv & 0x3FFFFu);
            if (j == me) continue;
            v3 sp = V3(((float)((sv >> 18) & 15u) + 0.5f) / 15.0f, ((float)((sv >> 22) & 15u) + 0.5f) / 15.0f,
                       ((float)((sv >> 26) & 15u) + 0.5f) / 15.0f);
            v3 dq = vsub(vadd(lo, vmuls(sp, u->cell)), p);
            if (vdot(dq, dq) > u->reach2) continue;
            v3 d = vsub(ld3(pos4 + 4 * (size_t)j), p);
            float r2 = vdot(d, d);
            if (r2 < u->link2) {
              float r = sqrtf(r2);
              if (n < cap) row[n] = (uint32_t)j | (u->touch - r > 0.0f ? 0x80000000u : 0u);
              n++;
            }
          }
        }
    counts[me] = n;
  }
}

/* src/glsl-sim.js:608-667 DIAG_FS */
void orc_diag(const orc_uni *u, const float *pos4, const float *qa, const uint32_t *seats,
              const float *forceA, const float *monoA, const float *forceB, const float *monoB,
              const int *ppslot, const float *ppforce, int cap, float *diag4) {
#pragma omp parallel for schedule(static)
  for (int me = 0; me < u->N; me++) {
    v3 p = ld3(pos4 + 4 * (size_t)me);
    float pp[3] = {p.x, p.y, p.z}, g[3];
    uint32_t h = orc_cell_of(u, pp, NULL, me);
    const uint32_t *s = seats + (size_t)h * ORC_SEATS;
    float seated = 0.0f, taken = 0.0f;
    for (int k = 0; k < ORC_SEATS; k++) {
      if (s[k] & 0x80000000u) break;
      taken += 1.0f;
      if ((int)(s[k] & 0x3FFFFu) == me) seated = 1.0f;
    }
    float phi = 0.0f, off = 0.0f;
    int box = orc_box_of(u, pp, g);
    if (box >= 0) {
      const float *F = box == 0 ? forceA : forceB;
      float f[3], t[3];
      int cf[3];
      for (int k = 0; k < 3; k++) { f[k] = floorf(g[k]); t[k] = g[k] - f[k]; cf[k] = (int)f[k]; }
      for (int k = 0; k < 8; k++) {
        int o[3] = {k & 1, (k >> 1) & 1, k >> 2}, at[3];
        float w3[3];
        for (int d = 0; d < 3; d++) {
          w3[d] = o[d] ? t[d] : 1.0f - t[d];
          at[d] = cf[d] + o[d] < 63 ? cf[d] + o[d] : 63;
        }
        phi += F[4 * fine_index(at[0], at[1], at[2]) + 3] * (w3[0] * w3[1] * w3[2]);
      }
      if (u->boxB > 0.5f) phi += box == 0 ? pot_at(u, p, monoB) : pot_at(u, p, monoA);
    } else {
      phi = pot_at(u, p, monoA);
      if (u->boxB > 0.5f) phi += pot_at(u, p, monoB);
      off = 2.0f;
    }
    int seat = ppslot[me];
    if (seat >= 0)
      for (int sl = 0; sl < 4; sl++) phi += ppforce[4 * ((size_t)sl * cap + seat) + 3];
    float *o = diag4 + 4 * (size_t)me;
    o[0] = phi; o[1] = seated + off; o[2] = taken; o[3] = qa[me];
  }
}

/* src/glsl-sim.js:537-570 RIGID_FS (matrices column-major, as uniformMatrix3fv) */
void orc_rigid(int N, const float *pos4, const float *vel4, const float bulk0[3], const float bulk1[3],
               const float cen0[3], const float cen1[3], const float spin0[3], const float spin1[3],
               const float rot0[9], const float rot1[9], float dt, float *pos_o, float *vel_o) {
  for (int i = 0; i < N; i++) {
    const float *P = pos4 + 4 * (size_t)i;
    int tgt = P[3] < 3.5f;
    const float *bulk = tgt ? bulk0 : bulk1, *cen = tgt ? cen0 : cen1, *m = tgt ? rot0 : rot1, *spin = tgt ? spin0 : spin1;
    v3 d = vsub(ld3(P), ld3(cen));
    v3 arm = V3(m[0] * d.x + m[3] * d.y + m[6] * d.z, m[1] * d.x + m[4] * d.y + m[7] * d.z,
                m[2] * d.x + m[5] * d.y + m[8] * d.z);
    v3 np = vadd(vadd(ld3(cen), arm), vmuls(ld3(bulk), dt));
    v3 nv = vadd(ld3(bulk), vcross(ld3(spin), arm));
    float *po = pos_o + 4 * (size_t)i, *vo = vel_o + 4 * (size_t)i;
    po[0] = np.x; po[1] = np.y; po[2] = np.z; po[3] = P[3];
    vo[0] = nv.x; vo[1] = nv.y; vo[2] = nv.z; vo[3] = vel4[4 * (size_t)i + 3];
  }
}

/* src/nbody.js:875-886 Morton key (binary64) and stable counting sort */
void orc_morton(int N, const float *P, const double core[3], int32_t *keys, int32_t *perm, int32_t *into) {
  int KB = 1 << 21;
  int32_t *bins = (int32_t *)calloc((size_t)KB + 1, sizeof(int32_t));
  for (int i = 0; i < N; i++) {
    int m[3];
    for (int k = 0; k < 3; k++) {
      double v = floor(((double)P[i * 4 + k] - core[k] + 6) / 12 * 128);
      m[k] = (int)fmin(127, fmax(0, v));
    }
    int mk = 0;
    for (int k = 0; k < 7; k++)
      mk |= ((m[0] >> k) & 1) << (3 * k) | ((m[1] >> k) & 1) << (3 * k + 1) | ((m[2] >> k) & 1) << (3 * k + 2);
    keys[i] = mk;
    bins[mk + 1]++;
  }
  for (int k = 0; k < KB; k++) bins[k + 1] += bins[k];
  for (int i = 0; i < N; i++) {
    int dst = bins[keys[i]]++;
    perm[dst] = i;
    if (into) into[i] = dst;
  }
  free(bins);
}

/* ------------------------------------------------------------------ */
/* the engine (src/nbody.js:376-636)                                   */
/* ------------------------------------------------------------------ */
typedef struct {
  float *fine, *coarse, mono[4], *farA, *farT0, *farT1, *force;
} orc_mesh;

struct orc_engine {
  orc_sim sim;
  orc_uni u;
  int N, cap, meshEvery, ppCount;
  int field;
  double gField[3], frozen, fieldInvM, fieldCpIron;
  float *pos, *vel, *aux, *q, *pos2, *vel2, *aux2, *q2, *mat;
  uint32_t *seats;
  orc_mesh pm[2];
  int *ppIndex, *ppSlot;
  float *ppList, *ppBox, *ppForce, tab[2 * ORC_PP_BINS];
};

static void mesh_alloc(orc_mesh *m) {
  m->fine = (float *)calloc(4 * (ORC_FINE + 1), sizeof(float));
  m->force = (float *)calloc(4 * (ORC_FINE + 1), sizeof(float));
  m->coarse = (float *)calloc(4 * ORC_COARSE, sizeof(float));
  m->farA = (float *)calloc(4 * ORC_COARSE, sizeof(float));
  m->farT0 = (float *)calloc(4 * ORC_COARSE, sizeof(float));
  m->farT1 = (float *)calloc(4 * ORC_COARSE, sizeof(float));
  memset(m->mono, 0, sizeof m->mono);
}
static void mesh_free(orc_mesh *m) {
  free(m->fine); free(m->force); free(m->coarse); free(m->farA); free(m->farT0); free(m->farT1);
}

orc_engine *orc_engine_new(const orc_sim *sim, const float *pos4, const float *vel4, const float *mat) {
  orc_engine *e = (orc_engine *)calloc(1, sizeof *e);
  e->sim = *sim;
  e->N = sim->N;
  e->cap = ORC_PP_CAP;
  e->meshEvery = 8;
  size_t N = (size_t)sim->N;
  e->pos = (float *)malloc(16 * N); e->vel = (float *)malloc(16 * N);
  e->aux = (float *)calloc(4 * N, 4); e->q = (float *)calloc(N, 4);
  e->pos2 = (float *)calloc(4 * N, 4); e->vel2 = (float *)calloc(4 * N, 4);
  e->aux2 = (float *)calloc(4 * N, 4); e->q2 = (float *)calloc(N, 4);
  e->mat = (float *)malloc(4 * N);
  memcpy(e->pos, pos4, 16 * N); memcpy(e->vel, vel4, 16 * N); memcpy(e->mat, mat, 4 * N);
  orc_make_uni(&e->sim, &e->u);
  e->seats = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)e->u.AW * e->u.AH * ORC_SEATS);
  for (size_t k = 0; k < (size_t)e->u.AW * e->u.AH * ORC_SEATS; k++) e->seats[k] = ORC_EMPTY;
  mesh_alloc(&e->pm[0]); mesh_alloc(&e->pm[1]);
  e->ppIndex = (int *)malloc(sizeof(int) * ORC_PP_CAP);
  e->ppSlot = (int *)malloc(sizeof(int) * N);
  for (int k = 0; k < ORC_PP_CAP; k++) e->ppIndex[k] = -1;
  for (size_t k = 0; k < N; k++) e->ppSlot[k] = -1;
  e->ppList = (float *)calloc(4 * ORC_PP_CAP, 4);
  e->ppBox = (float *)calloc(ORC_PP_CAP, 4);
  e->ppForce = (float *)calloc(16 * ORC_PP_CAP, 4);
  float f[ORC_PP_BINS], p[ORC_PP_BINS];
  orc_pair_table(ORC_PP_BINS, PP_CUT, f, p);
  for (int k = 0; k < ORC_PP_BINS; k++) { e->tab[2 * k] = f[k]; e->tab[2 * k + 1] = p[k]; }
  return e;
}
void orc_engine_free(orc_engine *e) {
  if (!e) return;
  free(e->pos); free(e->vel); free(e->aux); free(e->q); free(e->pos2); free(e->vel2); free(e->aux2); free(e->q2);
  free(e->mat); free(e->seats); mesh_free(&e->pm[0]); mesh_free(&e->pm[1]);
  free(e->ppIndex); free(e->ppSlot); free(e->ppList); free(e->ppBox); free(e->ppForce);
  free(e);
}
orc_sim *orc_engine_sim(orc_engine *e) { return &e->sim; }

static void refresh_static(orc_engine *e) {
  /* setStaticUniforms keeps the per-pass values; only the static ones change */
  orc_uni keep = e->u;
  orc_make_uni(&e->sim, &e->u);
  e->u.gdt = keep.gdt; e->u.settle = keep.settle; e->u.kick = keep.kick;
  e->u.field = keep.field; e->u.frozen = keep.frozen; memcpy(e->u.gField, keep.gField, 12);
  e->u.invM = keep.invM; e->u.cpIron = keep.cpIron;
  memcpy(e->u.LA, keep.LA, sizeof keep.LA); memcpy(e->u.LB, keep.LB, sizeof keep.LB); e->u.boxB = keep.boxB;
  memcpy(e->u.bulk0, keep.bulk0, 12); memcpy(e->u.bulk1, keep.bulk1, 12);
  memcpy(e->u.cen0, keep.cen0, 12); memcpy(e->u.cen1, keep.cen1, 12);
}

static void pass_slots(orc_engine *e) { orc_slots(&e->u, e->pos, e->seats); }

static void pass_mesh_box(orc_engine *e, int b) {
  orc_mesh *m = &e->pm[b];
  orc_deposit(&e->u, b, e->pos, e->mat, m->mono, m->fine);
  orc_coarse(m->fine, m->coarse, m->mono);
  orc_far(m->coarse, m->farA, m->farT0, m->farT1);
  orc_cell(&e->u, m->fine, m->coarse, m->farA, m->farT0, m->farT1, m->force);
}
static void pass_mesh(orc_engine *e) {
  pass_mesh_box(e, 0);
  if (e->sim.boxOn[1]) pass_mesh_box(e, 1);
}
static void pass_pp(orc_engine *e) {
  if (!e->ppCount) return;
  orc_pp_gather(&e->u, e->pos, e->mat, e->ppIndex, e->cap, e->ppList, e->ppBox);
  orc_pp_force(&e->u, e->ppList, e->ppBox, e->ppCount, e->cap, e->tab, e->ppForce);
}
static void swap_state(orc_engine *e) {
  float *t;
  t = e->pos; e->pos = e->pos2; e->pos2 = t;
  t = e->vel; e->vel = e->vel2; e->vel2 = t;
  t = e->aux; e->aux = e->aux2; e->aux2 = t;
  t = e->q; e->q = e->q2; e->q2 = t;
}
static void pass_sim(orc_engine *e, int settle, int kick, double gdt) {
  orc_sim *s = &e->sim;
  e->u.settle = settle ? 1.0f : 0.0f;
  e->u.kick = kick ? 1.0f : 0.0f;
  e->u.gdt = (float)gdt;
  for (int k = 0; k < 3; k++) {
    e->u.bulk0[k] = (float)s->bulk0[k]; e->u.bulk1[k] = (float)s->bulk1[k];
    e->u.cen0[k] = (float)s->cen0[k]; e->u.cen1[k] = (float)s->cen1[k];
  }
  orc_sim_pass(&e->u, e->pos, e->vel, e->mat, e->q, e->seats, e->pm[0].force, e->pm[0].mono, e->pm[1].force,
               e->pm[1].mono, e->ppSlot, e->ppForce, e->cap, e->pos2, e->vel2, e->aux2, e->q2);
  swap_state(e);
}

void orc_engine_set_field(orc_engine *e, int on, const double g[3], double frozen, double invM, double cpIron) {
  /* the crater page's setStaticUniforms: uGField, uFrozen, uInvM = 1, uCpIron = 1 (chicxulub.html:700-710) */
  e->field = on;
  orc_make_uni(&e->sim, &e->u);
  if (on) {
    e->u.field = 1.0f;
    for (int k = 0; k < 3; k++) e->u.gField[k] = (float)g[k];
    e->u.frozen = frozen < 0 ? -1.0f : (float)frozen;
    e->u.invM = (float)invM;
    e->u.cpIron = (float)cpIron;
  }
}

void orc_engine_step(orc_engine *e, int settle, int kick) {
  orc_sim *s = &e->sim;
  if (e->field) {   /* chicxulub.html:763-766: step(settle) { if (stepNo++ % 2 === 0) passSlots(); passSim(settle, dt) } */
    int n = s->stepNo++;
    if (n % 2 == 0) pass_slots(e);
    pass_sim(e, settle, kick, s->dt);
    return;
  }
  if (!settle && !kick && !s->soft && s->t - s->impactT > 1.5) { orc_soften(s); refresh_static(e); }
  int n = s->stepNo++;
  if (n % 2 == 0) pass_slots(e);
  int mesh = n % e->meshEvery == 0;
  if (mesh) { orc_boxes(s, &e->u); pass_mesh(e); pass_pp(e); }
  pass_sim(e, settle, kick, mesh ? e->meshEvery * s->dt : 0);
}

/* src/nbody.js:571-636 centres, rigidStep */
void orc_engine_rigid_step(orc_engine *e, double dtF) {
  orc_sim *s = &e->sim;
  double *r = s->relr, *v = s->relv, M = s->M, M1 = s->M1, M2 = s->M2;
  double r0[3] = {r[0], r[1], r[2]};
  int n = 8;
  double h = dtF / n, a[3];
  double cen[2][3] = {{-r0[0] * M2 / M, -r0[1] * M2 / M, -r0[2] * M2 / M}, {r0[0] * M1 / M, r0[1] * M1 / M, r0[2] * M1 / M}};
#define ACC()                                                    \
  do {                                                           \
    double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];         \
    double f = -M * pow(d2, -1.5);                               \
    a[0] = r[0] * f; a[1] = r[1] * f; a[2] = r[2] * f;           \
  } while (0)
  ACC();
  for (int i = 0; i < n; i++) {
    for (int k = 0; k < 3; k++) v[k] += a[k] * h * 0.5;
    for (int k = 0; k < 3; k++) r[k] += v[k] * h;
    ACC();
    for (int k = 0; k < 3; k++) v[k] += a[k] * h * 0.5;
  }
#undef ACC
  double mv[3] = {(r[0] - r0[0]) / dtF, (r[1] - r0[1]) / dtF, (r[2] - r0[2]) / dtF};
  for (int k = 0; k < 3; k++) { s->bulk0[k] = -mv[k] * M2 / M; s->bulk1[k] = mv[k] * M1 / M; }
  double R0[9], R1[9];
  orc_turn(s->spin0, dtF, R0);
  orc_turn(s->spin1, dtF, R1);
  float fb0[3], fb1[3], fc0[3], fc1[3], fs0[3], fs1[3], fr0[9], fr1[9];
  for (int k = 0; k < 3; k++) {
    fb0[k] = (float)s->bulk0[k]; fb1[k] = (float)s->bulk1[k]; fc0[k] = (float)cen[0][k]; fc1[k] = (float)cen[1][k];
    fs0[k] = (float)s->spin0[k]; fs1[k] = (float)s->spin1[k];
  }
  for (int k = 0; k < 9; k++) { fr0[k] = (float)R0[k]; fr1[k] = (float)R1[k]; }
  orc_rigid(s->N, e->pos, e->vel, fb0, fb1, fc0, fc1, fs0, fs1, fr0, fr1, (float)dtF, e->pos2, e->vel2);
  memcpy(e->aux2, e->aux, 16 * (size_t)s->N);
  memcpy(e->q2, e->q, 4 * (size_t)s->N);
  swap_state(e);
  s->t += dtF;
  if (hypot(hypot(r[0], r[1]), r[2]) <= s->Re1 + s->Re2 + 2 * s->a) {
    for (int k = 0; k < 3; k++) { s->bulk0[k] = -v[k] * M2 / M; s->bulk1[k] = v[k] * M1 / M; }
    for (int k = 0; k < 3; k++) { s->cen0[k] = -r[k] * M2 / M; s->cen1[k] = r[k] * M1 / M; }
    s->boxOn[0] = 1;
    for (int k = 0; k < 3; k++) { s->boxCen[0][k] = s->cen0[k]; s->boxVel[0][k] = s->bulk0[k]; }
    s->boxT[0] = s->t;
    s->boxOn[1] = 0;
    s->stepNo = 0;
    orc_engine_step(e, 0, 1);
    s->t += s->dt;
    s->phase = 2;
    s->impactT = s->t;
  }
}

/* src/nbody.js:957-966 setPP */
void orc_engine_set_pp(orc_engine *e, const int *list, int n) {
  for (int k = 0; k < e->N; k++) e->ppSlot[k] = -1;
  for (int k = 0; k < n; k++) e->ppSlot[list[k]] = k;
  for (int k = 0; k < e->cap; k++) e->ppIndex[k] = k < n ? list[k] : -1;
  e->ppCount = n;
  if (n) pass_pp(e);
}
void orc_engine_prime_mono(orc_engine *e, int box, const float mono[4]) { memcpy(e->pm[box].mono, mono, 16); }

/* src/nbody.js:932-954 applyPerm; src/glsl-sim.js:578-602 PERM_FS */
void orc_engine_apply_perm(orc_engine *e, const int32_t *perm) {
  size_t N = (size_t)e->N;
  float *R = (float *)malloc(4 * N);
  for (size_t i = 0; i < N; i++) {
    size_t s = (size_t)perm[i];
    R[i] = e->mat[s];
    memcpy(e->pos2 + 4 * i, e->pos + 4 * s, 16);
    memcpy(e->vel2 + 4 * i, e->vel + 4 * s, 16);
    memcpy(e->aux2 + 4 * i, e->aux + 4 * s, 16);
    e->q2[i] = e->q[s];
  }
  memcpy(e->mat, R, 4 * N);
  free(R);
  swap_state(e);
  pass_slots(e);
}

/* src/nbody.js:488-507 passDiag */
void orc_engine_diag(orc_engine *e, float *diag4) {
  orc_boxes(&e->sim, &e->u);
  pass_slots(e);
  pass_mesh(e);
  pass_pp(e);
  orc_diag(&e->u, e->pos, e->q, e->seats, e->pm[0].force, e->pm[0].mono, e->pm[1].force, e->pm[1].mono, e->ppSlot,
           e->ppForce, e->cap, diag4);
}

const void *orc_engine_buf(orc_engine *e, int which, long *bytes) {
  long N = e->N;
  switch (which) {
    case 0: *bytes = 16 * N; return e->pos;
    case 1: *bytes = 16 * N; return e->vel;
    case 2: *bytes = 16 * N; return e->aux;
    case 3: *bytes = 4 * N; return e->q;
    case 4: *bytes = 4 * N; return e->mat;
    case 5: *bytes = 4L * e->u.AW * e->u.AH * ORC_SEATS; return e->seats;
    case 6: *bytes = 16L * (ORC_FINE + 1); return e->pm[0].fine;
    case 7: *bytes = 16L * (ORC_FINE + 1); return e->pm[0].force;
    case 8: *bytes = 16; return e->pm[0].mono;
    case 9: *bytes = 16L * ORC_COARSE; return e->pm[0].coarse;
    case 10: *bytes = 16L * ORC_COARSE; return e->pm[0].farA;
    case 11: *bytes = 16L * (ORC_FINE + 1); return e->pm[1].fine;
    case 12: *bytes = 16L * (ORC_FINE + 1); return e->pm[1].force;
    case 13: *bytes = 16; return e->pm[1].mono;
    case 14: *bytes = 16L * ORC_PP_CAP; return e->ppList;
    case 15: *bytes = 64L * ORC_PP_CAP; return e->ppForce;
    case 16: *bytes = 4L * ORC_PP_CAP; return e->ppBox;
    case 17: *bytes = 4 * N; return e->ppSlot;
    default: *bytes = 0; return NULL;
  }
}

/* ------------------------------------------------------------------ */
/* src/nbody.js:646-893 fof: groups, body stats, books, loose list,    */
/* Morton order                                                        */
/* ------------------------------------------------------------------ */
typedef struct {
  int n;
  double mass, com[3], core[3], vel[3], imp, iron, R, Redge, Tsurf, hotCom[3], hotR, impMass, impCom[3], impRms;
} grp_t;

static int uf_find(int *uf, int x) {
  while (uf[x] != x) { uf[x] = uf[uf[x]]; x = uf[x]; }
  return x;
}

static void grp_stats(int N, double mref, const float *P, const float *V, const float *R, int *uf, int root,
                      int *members, grp_t *g) {
  int n = 0;
  double mass = 0, x = 0, y = 0, z = 0, vx = 0, vy = 0, vz = 0, imp = 0, iron = 0, ix = 0, iy = 0, iz = 0;
  for (int t = 0; t < N; t++)
    if (uf_find(uf, t) == root) {
      double m = mref * R[t], w = P[t * 4 + 3];
      members[n++] = t;
      mass += m;
      x += m * P[t * 4]; y += m * P[t * 4 + 1]; z += m * P[t * 4 + 2];
      vx += m * V[t * 4]; vy += m * V[t * 4 + 1]; vz += m * V[t * 4 + 2];
      if (w >= 3.5) { imp += m; ix += m * P[t * 4]; iy += m * P[t * 4 + 1]; iz += m * P[t * 4 + 2]; }
      if (w - 4 * floor(w / 4) < 0.5) iron += m;
    }
  double gx = x / mass, gy = y / mass, gz = z / mass, Rg = cbrt(mass);
  double icx = imp > 0 ? ix / imp : 0, icy = imp > 0 ? iy / imp : 0, icz = imp > 0 ? iz / imp : 0;
  double tm = mass - imp, core[3];
  if (imp > tm) { core[0] = icx; core[1] = icy; core[2] = icz; }
  else { core[0] = (x - ix) / tm; core[1] = (y - iy) / tm; core[2] = (z - iz) / tm; }
  double rc2 = 0.9 * 0.9 * Rg * Rg;
  for (int it = 0; it < 3; it++) {
    double sm = 0, sx0 = 0, sy0 = 0, sz0 = 0;
    for (int s = 0; s < n; s++) {
      int t = members[s];
      double qx = P[t * 4] - core[0], qy = P[t * 4 + 1] - core[1], qz = P[t * 4 + 2] - core[2];
      if (qx * qx + qy * qy + qz * qz < rc2) {
        double m = mref * R[t];
        sm += m; sx0 += m * P[t * 4]; sy0 += m * P[t * 4 + 1]; sz0 += m * P[t * 4 + 2];
      }
    }
    if (sm > 0) { core[0] = sx0 / sm; core[1] = sy0 / sm; core[2] = sz0 / sm; }
  }
  enum { NBIN = 96 };
  double shell = 0.64 * Rg * Rg, Ts = 0, ws = 0, irms = 0;
  double dr = 3 * Rg / NBIN, hist[NBIN], hs = 0, hx = 0, hy = 0, hz = 0, hr2 = 0;
  memset(hist, 0, sizeof hist);
  for (int s = 0; s < n; s++) {
    int t = members[s];
    double m = mref * R[t];
    double sx = P[t * 4] - core[0], sy = P[t * 4 + 1] - core[1], sz = P[t * 4 + 2] - core[2];
    double r2s = sx * sx + sy * sy + sz * sz;
    double Th = V[t * 4 + 3];
    if (r2s > shell) { double Tt = fmin(Th, 12000), wt = Tt * Tt; Ts += wt * Tt; ws += wt; }
    if (Th > 1200) {
      double wh = fmin(Th, 12000);
      wh *= wh;
      hs += wh; hx += wh * P[t * 4]; hy += wh * P[t * 4 + 1]; hz += wh * P[t * 4 + 2]; hr2 += wh * r2s;
    }
    if (P[t * 4 + 3] >= 3.5) {
      double ex = P[t * 4] - icx, ey = P[t * 4 + 1] - icy, ez = P[t * 4 + 2] - icz;
      irms += m * (ex * ex + ey * ey + ez * ez);
    }
    double bi = sqrt(r2s) / dr;
    hist[bi < NBIN - 1 ? (int)bi : NBIN - 1] += m;
  }
  double hot[3] = {core[0], core[1], core[2]}, hotR = Rg;
  if (hs > 0) {
    hot[0] = hx / hs; hot[1] = hy / hs; hot[2] = hz / hs;
    double ox = hot[0] - core[0], oy = hot[1] - core[1], oz = hot[2] - core[2];
    hotR = sqrt(fmax(hr2 / hs - (ox * ox + oy * oy + oz * oz), 0));
  }
  double Redge = 0;
  if (n >= 2000) {
    double Rb = cbrt(fmax(imp, tm)), rho[NBIN], refS = 0;
    int refN = 0;
    for (int bq = 0; bq < NBIN; bq++) {
      double rm = (bq + 0.5) * dr;
      rho[bq] = hist[bq] / (rm * rm * dr);
      if (rm > 0.6 * Rb && rm < 0.85 * Rb) { refS += rho[bq]; refN++; }
    }
    Redge = Rg;
    for (int bq = 0; bq < NBIN; bq++)
      if ((bq + 0.5) * dr > 0.85 * Rb && refN > 0 && rho[bq] < 0.35 * refS / refN) { Redge = bq * dr; break; }
  }
  g->n = n; g->mass = mass;
  g->com[0] = gx; g->com[1] = gy; g->com[2] = gz;
  memcpy(g->core, core, sizeof core);
  g->vel[0] = vx / mass; g->vel[1] = vy / mass; g->vel[2] = vz / mass;
  g->imp = imp / mass; g->iron = iron / mass; g->R = Rg; g->Redge = Redge;
  g->Tsurf = ws > 0 ? Ts / ws : 0;
  memcpy(g->hotCom, hot, sizeof hot); g->hotR = hotR;
  g->impMass = imp; g->impCom[0] = icx; g->impCom[1] = icy; g->impCom[2] = icz;
  g->impRms = imp > 0 ? sqrt(irms / imp) : 0;
}

static double far2(const grp_t *b, const float *P, int i) {
  double ex = P[i * 4] - b->com[0], ey = P[i * 4 + 1] - b->com[1], ez = P[i * 4 + 2] - b->com[2];
  return ex * ex + ey * ey + ez * ez;
}
static int cmp_double(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return x < y ? -1 : x > y ? 1 : 0;
}

void orc_fof(int N, double mref, double a, const float *P, const float *V, const float *R, const float *D,
             double spring, double touch, int cap, int sort, orc_report *rep, int32_t *list, int32_t *perm) {
  double L = 2.4 * a, L2 = L * L, inv = 1 / L, touch2 = touch * touch, elastic = 0;
  int T = 1 << 20, TM = T - 1;
  int *cx = (int *)malloc(4 * (size_t)N), *cy = (int *)malloc(4 * (size_t)N), *cz = (int *)malloc(4 * (size_t)N);
  int *key = (int *)malloc(4 * (size_t)N), *cnt = (int *)calloc((size_t)T + 1, 4);
  for (int i = 0; i < N; i++) {
    int qx = (int)floor(P[i * 4] * inv), qy = (int)floor(P[i * 4 + 1] * inv), qz = (int)floor(P[i * 4 + 2] * inv);
    cx[i] = qx; cy[i] = qy; cz[i] = qz;
    int k = ((int)((uint32_t)qx * 73856093u) ^ (int)((uint32_t)qy * 19349663u) ^ (int)((uint32_t)qz * 83492791u)) & TM;
    key[i] = k;
    cnt[k + 1]++;
  }
  for (int k = 0; k < T; k++) cnt[k + 1] += cnt[k];
  int *fill = (int *)malloc(4 * (size_t)T), *order = (int *)malloc(4 * (size_t)N);
  memcpy(fill, cnt, 4 * (size_t)T);
  for (int i = 0; i < N; i++) order[fill[key[i]]++] = i;
  int *uf = (int *)malloc(4 * (size_t)N);
  for (int i = 0; i < N; i++) uf[i] = i;
  for (int i = 0; i < N; i++) {
    double px = P[i * 4], py = P[i * 4 + 1], pz = P[i * 4 + 2];
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int k = ((int)((uint32_t)(cx[i] + dx) * 73856093u) ^ (int)((uint32_t)(cy[i] + dy) * 19349663u) ^
                   (int)((uint32_t)(cz[i] + dz) * 83492791u)) & TM;
          for (int s = cnt[k]; s < cnt[k + 1]; s++) {
            int j = order[s];
            if (j <= i) continue;
            double ex = P[j * 4] - px, ey = P[j * 4 + 1] - py, ez = P[j * 4 + 2] - pz;
            double e2 = ex * ex + ey * ey + ez * ez;
            if (e2 < L2) {
              int ri = uf_find(uf, i), rj = uf_find(uf, j);
              if (ri != rj) uf[ri] = rj;
              if (e2 < touch2) { double ov = touch - sqrt(e2); elastic += 0.5 * spring * ov * ov; }
            }
          }
        }
  }
  int *size = (int *)calloc((size_t)N, 4);
  for (int i = 0; i < N; i++) size[uf_find(uf, i)]++;
  int g1 = -1, g2 = -1;
  for (int i = 0; i < N; i++)
    if (size[i] > 0) {
      if (g1 < 0 || size[i] > size[g1]) { g2 = g1; g1 = i; }
      else if (g2 < 0 || size[i] > size[g2]) g2 = i;
    }
  int *members = (int *)malloc(4 * (size_t)N);
  grp_t A, B;
  grp_stats(N, mref, P, V, R, uf, g1, members, &A);
  int hasB = g2 >= 0;
  if (hasB) grp_stats(N, mref, P, V, R, uf, g2, members, &B);
  double ib = 1.15 * cbrt(fmax(A.impMass, A.mass - A.impMass));
  double rb2 = ib * ib, cx0 = A.core[0], cy0 = A.core[1], cz0 = A.core[2];
  double bm = 0, bvx = 0, bvy = 0, bvz = 0;
  for (int i = 0; i < N; i++)
    if (uf_find(uf, i) == g1) {
      double dx0 = P[i * 4] - cx0, dy0 = P[i * 4 + 1] - cy0, dz0 = P[i * 4 + 2] - cz0;
      if (dx0 * dx0 + dy0 * dy0 + dz0 * dz0 > rb2) continue;
      double m = mref * R[i];
      bm += m; bvx += m * V[i * 4]; bvy += m * V[i * 4 + 1]; bvz += m * V[i * 4 + 2];
    }
  if (bm > 0) { bvx /= bm; bvy /= bm; bvz /= bm; }
  double Lx = 0, Ly = 0, Lz = 0, I = 0;
  for (int i = 0; i < N; i++)
    if (uf_find(uf, i) == g1) {
      double dx0 = P[i * 4] - cx0, dy0 = P[i * 4 + 1] - cy0, dz0 = P[i * 4 + 2] - cz0;
      if (dx0 * dx0 + dy0 * dy0 + dz0 * dz0 > rb2) continue;
      double m = mref * R[i];
      double ux = V[i * 4] - bvx, uy = V[i * 4 + 1] - bvy, uz = V[i * 4 + 2] - bvz;
      Lx += m * (dy0 * uz - dz0 * uy); Ly += m * (dz0 * ux - dx0 * uz); Lz += m * (dx0 * uy - dy0 * ux);
    }
  double Lm = sqrt(Lx * Lx + Ly * Ly + Lz * Lz), lx = Lx / (Lm + 1e-30), ly = Ly / (Lm + 1e-30), lz = Lz / (Lm + 1e-30);
  double tilt = acos(fmax(-1, fmin(1, ly))) * 180 / PI;
  for (int i = 0; i < N; i++)
    if (uf_find(uf, i) == g1) {
      double dx0 = P[i * 4] - cx0, dy0 = P[i * 4 + 1] - cy0, dz0 = P[i * 4 + 2] - cz0;
      if (dx0 * dx0 + dy0 * dy0 + dz0 * dz0 > rb2) continue;
      double m = mref * R[i];
      double along = dx0 * lx + dy0 * ly + dz0 * lz;
      I += m * (dx0 * dx0 + dy0 * dy0 + dz0 * dz0 - along * along);
    }
  double day = Lm > 1e-9 ? 2 * PI * I / Lm * 805 / 3600 : INFINITY;
#define ENERGY(x, y, z, vx, vy, vz)                                                                            \
  (0.5 * (((vx) - A.vel[0]) * ((vx) - A.vel[0]) + ((vy) - A.vel[1]) * ((vy) - A.vel[1]) +                     \
          ((vz) - A.vel[2]) * ((vz) - A.vel[2])) -                                                             \
   A.mass / fmax(sqrt(((x) - A.com[0]) * ((x) - A.com[0]) + ((y) - A.com[1]) * ((y) - A.com[1]) +            \
                      ((z) - A.com[2]) * ((z) - A.com[2])),                                                    \
                 A.R))
  double orbit = 0, esc = 0, Dx = 0, Dy = 0, Dz = 0;
  for (int i = 0; i < N; i++)
    if (uf_find(uf, i) != g1) {
      double m = mref * R[i];
      if (ENERGY((double)P[i * 4], (double)P[i * 4 + 1], (double)P[i * 4 + 2], (double)V[i * 4], (double)V[i * 4 + 1],
                 (double)V[i * 4 + 2]) < 0) {
        orbit += m;
        double dx0 = P[i * 4] - A.com[0], dy0 = P[i * 4 + 1] - A.com[1], dz0 = P[i * 4 + 2] - A.com[2];
        double wx = V[i * 4] - A.vel[0], wy = V[i * 4 + 1] - A.vel[1], wz = V[i * 4 + 2] - A.vel[2];
        Dx += m * (dy0 * wz - dz0 * wy); Dy += m * (dz0 * wx - dx0 * wz); Dz += m * (dx0 * wy - dy0 * wx);
      } else esc += m;
    }
  double jD = orbit > 0 ? sqrt(Dx * Dx + Dy * Dy + Dz * Dz) / (orbit * sqrt(A.mass * 2.9)) : 0;
  double moon = fmin(fmax(0, orbit * (1.9 * jD - 1.1 - 1.9 * 0.05)), 0.95 * orbit);
  memset(rep, 0, sizeof *rep);
  if (hasB && B.n >= fmax(8, N / 1000.0)) {
    double dAB = sqrt((B.com[0] - A.com[0]) * (B.com[0] - A.com[0]) + (B.com[1] - A.com[1]) * (B.com[1] - A.com[1]) +
                      (B.com[2] - A.com[2]) * (B.com[2] - A.com[2]));
    if (dAB > A.R + B.R + 2 * a) {
      rep->hasSecond = 1;
      rep->secMass = B.mass; rep->secDist = dAB;
      rep->secBound = ENERGY(B.com[0], B.com[1], B.com[2], B.vel[0], B.vel[1], B.vel[2]) < 0;
      rep->secImp = B.imp; rep->secIron = B.iron;
      memcpy(rep->secCom, B.com, 24); memcpy(rep->secCore, B.core, 24); memcpy(rep->secVel, B.vel, 24);
      rep->secR = B.R;
    }
  }
#undef ENERGY
  double Mt = 0, px = 0, py = 0, pz = 0, Jx = 0, Jy = 0, Jz = 0, ke = 0, pe = 0, Q = 0, ironAll = 0;
  int unseated = 0, full = 0;
  for (int i = 0; i < N; i++) {
    double m = mref * R[i];
    double bx = P[i * 4], by = P[i * 4 + 1], bz = P[i * 4 + 2], bu = V[i * 4], bv = V[i * 4 + 1], bw = V[i * 4 + 2];
    Mt += m; px += m * bu; py += m * bv; pz += m * bw;
    if (P[i * 4 + 3] - 4 * floor(P[i * 4 + 3] / 4.0) < 0.5) ironAll += m;
    Jx += m * (by * bw - bz * bv); Jy += m * (bz * bu - bx * bw); Jz += m * (bx * bv - by * bu);
    ke += 0.5 * m * (bu * bu + bv * bv + bw * bw);
    double flag = D[i * 4 + 1];
    int off = flag >= 2;
    pe += (off ? 1 : 0.5) * m * D[i * 4];
    Q += 0.5 * D[i * 4 + 3];
    if (flag - (off ? 2 : 0) < 0.5) unseated++;
    if (D[i * 4 + 2] >= 7.5) full++;
  }
  int bigB = hasB && B.mass > 0.05, nLoose = 0;
#define LOOSE(i) (far2(&A, P, (i)) > 1.69 * A.R * A.R && !(bigB && far2(&B, P, (i)) <= 1.69 * B.R * B.R))
  for (int i = 0; i < N; i++)
    if (LOOSE(i)) nLoose++;
  double least = 0;
  if (nLoose > cap) {
    double *ds = (double *)malloc(8 * (size_t)nLoose);
    int q = 0;
    for (int i = 0; i < N; i++)
      if (LOOSE(i)) ds[q++] = far2(&A, P, i);
    qsort(ds, (size_t)nLoose, 8, cmp_double);
    least = ds[nLoose - cap];
    free(ds);
  }
  int len = nLoose < cap ? nLoose : cap, wr = 0;
  for (int i = 0; i < N && wr < len; i++)
    if (LOOSE(i) && far2(&A, P, i) >= least) list[wr++] = i;
#undef LOOSE
  if (sort && perm) {
    int32_t *keys = (int32_t *)malloc(4 * (size_t)N), *into = (int32_t *)malloc(4 * (size_t)N);
    orc_morton(N, P, A.core, keys, perm, into);
    for (int i = 0; i < len; i++) list[i] = into[list[i]];
    free(keys); free(into);
  }
  rep->largest = A.mass; rep->largestImp = A.imp; rep->largestIron = A.iron; rep->day = day; rep->tilt = tilt;
  rep->axis[0] = lx; rep->axis[1] = ly; rep->axis[2] = lz;
  rep->bodyVel[0] = bvx; rep->bodyVel[1] = bvy; rep->bodyVel[2] = bvz;
  rep->orbit = orbit; rep->escape = esc;
  memcpy(rep->com, A.com, 24); memcpy(rep->core, A.core, 24); memcpy(rep->vel, A.vel, 24);
  rep->R = A.R; rep->Redge = A.Redge; rep->Tsurf = A.Tsurf; memcpy(rep->hotCom, A.hotCom, 24); rep->hotR = A.hotR;
  rep->impMass = A.impMass; memcpy(rep->impCom, A.impCom, 24); rep->impRms = A.impRms;
  rep->M = Mt; rep->iron = ironAll / Mt; rep->drift = sqrt(px * px + py * py + pz * pz) / Mt;
  rep->L = sqrt(Jx * Jx + Jy * Jy + Jz * Jz);
  rep->KE = ke; rep->PE = pe; rep->EL = elastic; rep->Q = Q;
  rep->unseated = (double)unseated / N; rep->full = (double)full / N;
  rep->jD = jD; rep->moon = moon;
  rep->ppCount = len; rep->ppLoose = nLoose;
  free(cx); free(cy); free(cz); free(key); free(cnt); free(fill); free(order); free(uf); free(size); free(members);
}

/* ------------------------------------------------------------------ */
/* FP64 direct sum (the gravity checker of the error sweep)            */
/* ------------------------------------------------------------------ */
void orc_direct_sum(int N, const float *P, const double *m, double eps, int nt, const int32_t *idx, double *acc,
                    double *pot) {
  double e2 = eps * eps;
#pragma omp parallel for schedule(dynamic, 8)
  for (int t = 0; t < nt; t++) {
    int i = idx[t];
    double xi = P[4 * (size_t)i], yi = P[4 * (size_t)i + 1], zi = P[4 * (size_t)i + 2];
    double ax = 0, ay = 0, az = 0, ph = 0;
    for (int j = 0; j < N; j++) {
      if (j == i) continue;
      double dx = P[4 * (size_t)j] - xi, dy = P[4 * (size_t)j + 1] - yi, dz = P[4 * (size_t)j + 2] - zi;
      double r2 = dx * dx + dy * dy + dz * dz + e2;
      double inv = 1.0 / sqrt(r2), inv3 = inv * inv * inv * m[j];
      ax += dx * inv3; ay += dy * inv3; az += dz * inv3;
      ph -= m[j] * inv;
    }
    acc[3 * t] = ax; acc[3 * t + 1] = ay; acc[3 * t + 2] = az;
    pot[t] = ph;
  }
}
