/*
 * ccs_oracle.h -- CPU oracle for the cosmic-collisions simulation step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * giant-impact step (src/glsl-sim.js shaders, src/nbody.js engine, src/bodies.js
 * builder, src/math.js RNG), pass by pass, used as the checker for the CUDA
 * library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it; the product never does.
 *
 * Parity status: UNPINNED against the reference's own outputs.  The reference
 * is GLSL run through WebGL2 plus JavaScript; neither a graphics stack nor a JS
 * engine exists on these machines, and the reference ships no tests or golden
 * vectors.  The oracle is pinned instead by known-answer checks taken from the
 * reference's own text (units, wrap length, Maclaurin peak, pair-table limits)
 * and by invariants (mesh net force ~ 0, conservation books).
 *
 * Float semantics: every GLSL expression is evaluated left to right with one
 * IEEE-754 binary32 rounding per operation (compiled with -ffp-contract=off),
 * dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z, inversesqrt(x) = 1/sqrt(x) with
 * correctly rounded sqrt and divide, mix(x,y,t) = x*(1-t) + y*t.  Host-side
 * JavaScript arithmetic is IEEE binary64, Float32Array stores round to binary32.
 */
#ifndef CCS_ORACLE_H
#define CCS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_SEATS 8            /* CC.SLOTS, src/shell.js:131 */
#define ORC_EMPTY 0xBF800000u  /* -1.0f: an empty seat, src/nbody.js:385 */
#define ORC_MESH 64            /* 64^3 mesh, src/nbody.js:37 */
#define ORC_FINE (64 * 64 * 64) /* fine cells; index ORC_FINE is the scratch texel */
#define ORC_COARSE 4096        /* 16^3 coarse blocks */
#define ORC_PP_CAP 8192        /* src/nbody.js:38 */
#define ORC_PP_BINS 64

/* Every per-run and per-pass uniform, already rounded to binary32 as
 * gl.uniform1f would round it (src/nbody.js:255-336, 342-350, 458-484). */
typedef struct {
  int N, W;
  int G, GShift, GMask, SX, SXShift, SXMask, AW, AH;   /* src/gl.js:73-75 */
  float invCell, cell, link2, reach2, touch;
  float K, C, invM, damp, creep, tK, kappa, cpIron;
  float dt, gdt, settle, kick;
  float bulk0[3], bulk1[3], cen0[3], cen1[3], spin0[3], spin1[3];
  float invH, eps2Mesh, eps2Cell, Gm;                   /* eps2Mesh: FH^2; eps2Cell: 0.5 FH^2 */
  float LA[3], LB[3], boxB;
  float cut, a2;
  float field, gField[3], frozen;   /* the crater page's field step: src/glsl-sim.js:466-468, 490-492, 517-533 */
} orc_uni;

/* The run's scalars (the JS `sim` object), binary64. */
typedef struct {
  int N, W, H, n1, n2, G, settleLeft, settleTotal, stepNo, soft, phase; /* phase 0 settle,1 approach,2 full */
  double m, a, cell, dt, k, c, creep, damp, tK, kappa;
  double R1, R2, Re1, Re2, M1, M2, M, vc, vesc, t, impactT;
  double spin0[3], spin1[3], cen0[3], cen1[3], bulk0[3], bulk1[3];
  double relr[3], relv[3];
  int boxOn[2];
  double boxCen[2][3], boxVel[2][3], boxT[2];
} orc_sim;

/* Options of build(opt) (src/nbody.js:114), plus documented extensions that
 * default to the reference's fixed values. */
typedef struct {
  int N;
  double q, dens, core, coreImp, spin0, spin1, angle, incl, vfac, rest;
  int n2;          /* >0: impactor particle count */
  double mImp;     /* >0: impactor mass, M_earth */
  /* extensions (0 = the reference's value) */
  double mTarget;  /* target mass, M_earth (reference: 1) */
  double rhoR;     /* core over mantle density (reference: 2.5) */
  double rhoCrust; /* crust over mantle density (reference: 1) */
  double crustFrac;/* crust = outer fraction of radius (reference: the outer shell) */
} orc_opt;

/* ---- src/math.js, src/bodies.js ---- */
double orc_mulberry(uint32_t *state);
double orc_maclaurin(double f);
double orc_maclaurin_g(double e);
void orc_turn(const double w[3], double dt, double out[9]);
/* returns the number of shell bounds written to bounds (<= n+2) */
int orc_ball(int n, double s, double a, uint32_t *rng, double e, float *out, int *bounds);
void orc_relax(float *p, int n, double a, double A, double C, int sweeps);
double orc_approach_time(const double relr[3], const double relv[3], double M, double touch);
/* build(): fills sim and the four particle arrays (pos4, vel4 N*4; mat N; home4 N*4) */
int orc_build(const orc_opt *opt, orc_sim *sim, float *pos4, float *vel4, float *mat, float *home4);
void orc_pair_table(int bins, double cut, float *f, float *p);
void orc_nn_label(const double d[3], const double s[3], double out[3]);   /* learned-correction label */

/* ---- uniforms ---- */
void orc_make_uni(const orc_sim *sim, orc_uni *u);
void orc_boxes(const orc_sim *sim, orc_uni *u);                 /* boxes(), src/nbody.js:342-350 */
void orc_soften(orc_sim *sim);                                  /* src/nbody.js:545-550 */

/* ---- the passes (src/glsl-sim.js) ---- */
void orc_hash(const orc_uni *u, int cx, int cy, int cz, int *ax, int *ay);
uint32_t orc_cell_of(const orc_uni *u, const float p[3], uint32_t *word, int idx);
void orc_slots(const orc_uni *u, const float *pos4, uint32_t *seats);     /* seats: AW*AH*8 */
int orc_box_of(const orc_uni *u, const float p[3], float g[3]);
void orc_deposit(const orc_uni *u, int box, const float *pos4, const float *mat, const float mono[4], float *fine);
void orc_coarse(const float *fine, float *coarse, float mono[4]);
void orc_far(const float *coarse, float *farA, float *farT0, float *farT1);
void orc_cell(const orc_uni *u, const float *fine, const float *coarse, const float *farA,
              const float *farT0, const float *farT1, float *force);
/* the stencil-split P3M (the library's ccs_set_pp_split; no counterpart in the reference): the cell pass
 * without the node pairs within S cells, unsoftened, with tides, and the far field at each cell from every
 * block more than two away as its monopole and quadrupole (force, tide0 = Txx Tyy Tzz Txy, tide1 = Txz
 * Tyz, tide2 = the pull's second gradient, three planes of (64^3 + 1) float4: Gxxx Gyyy Gzzz Gxyz, Gxxy
 * Gxxz Gxyy Gyyz, Gxzz Gyzz -- the near sources' and the far blocks' monopoles'; all x Gm; tide2 may be
 * NULL); every particle's pairs inside the stencil (out4: pull, potential x Gm); the gather from each
 * node's centre of mass, second order (first order where tideA2 / tideB2 is NULL), plus the particle's
 * pairs (grav4) */
void orc_cell_tide(const orc_uni *u, int S, const float *fine, const float *coarse, const float *fineQ,
                   float *force, float *tide0, float *tide1, float *tide2);
/* each cell's second moment about its centre of mass (after orc_deposit): fineQ, two planes of (64^3 + 1)
 * float4 (Qxx Qyy Qzz Qxy), (Qxz Qyz); given to orc_cell_tide, the near cells act as quadrupoles and the
 * blocks' quadrupoles include the cells' own (NULL: monopoles at their centres of mass) */
void orc_node_moments(const orc_uni *u, int box, const float *pos4, const float *mat, const float *fine,
                      float *fineQ);
void orc_pp_split(const orc_uni *u, int S, const float *pos4, const float *mat, float *out4);
void orc_gather_split(const orc_uni *u, const float *pos4, const float *fineA, const float *forceA,
                      const float *tideA0, const float *tideA1, const float *tideA2, const float *fineB,
                      const float *forceB, const float *tideB0, const float *tideB1, const float *tideB2,
                      const float *monoA, const float *monoB, const float *ppAll, float *grav4);
void orc_pp_gather(const orc_uni *u, const float *pos4, const float *mat, const int *index, int cap,
                   float *list4, float *box);
void orc_pp_force(const orc_uni *u, const float *list4, const float *box, int count, int cap,
                  const float *tab, float *force);
void orc_sim_pass(const orc_uni *u, const float *pos4, const float *vel4, const float *mat, const float *q,
                  const uint32_t *seats, const float *forceA, const float *monoA, const float *forceB,
                  const float *monoB, const int *ppslot, const float *ppforce, int cap,
                  float *pos_o, float *vel_o, float *aux_o, float *q_o);
/* the contact-pair sets of simFS's loop (src/glsl-sim.js:415-450), walked as orc_sim_pass walks them: per
 * owner, every neighbour inside the link radius as its index with bit 31 set when the two touch; counts (N)
 * the owner's neighbours, pairs (N x cap) the first cap of them in walk order, the rest 0xFFFFFFFF */
void orc_contact_pairs(const orc_uni *u, const float *pos4, const uint32_t *seats, int cap, int32_t *counts,
                       uint32_t *pairs);
void orc_diag(const orc_uni *u, const float *pos4, const float *q, const uint32_t *seats,
              const float *forceA, const float *monoA, const float *forceB, const float *monoB,
              const int *ppslot, const float *ppforce, int cap, float *diag4);
void orc_rigid(int N, const float *pos4, const float *vel4, const float bulk0[3], const float bulk1[3],
               const float cen0[3], const float cen1[3], const float spin0[3], const float spin1[3],
               const float rot0[9], const float rot1[9], float dt, float *pos_o, float *vel_o);
void orc_morton(int N, const float *pos4, const double core[3], int32_t *keys, int32_t *perm, int32_t *into);

/* ---- the engine: state, schedule, phases (src/nbody.js:376-636) ---- */
typedef struct orc_engine orc_engine;
orc_engine *orc_engine_new(const orc_sim *sim, const float *pos4, const float *vel4, const float *mat);
void orc_engine_free(orc_engine *e);
orc_sim *orc_engine_sim(orc_engine *e);
void orc_engine_step(orc_engine *e, int settle, int kick);
/* the crater page's field-gravity step and schedule (chicxulub.html:700-710, 763-766); on = 0: the impact's */
void orc_engine_set_field(orc_engine *e, int on, const double g[3], double frozen, double invM, double cpIron);
void orc_engine_rigid_step(orc_engine *e, double dtF);
void orc_engine_set_pp(orc_engine *e, const int *list, int n);
void orc_engine_prime_mono(orc_engine *e, int box, const float mono[4]);
void orc_engine_apply_perm(orc_engine *e, const int32_t *perm);
void orc_engine_diag(orc_engine *e, float *diag4);
/* read a buffer: 0 pos4, 1 vel4, 2 aux4, 3 q, 4 mat, 5 seats, 6 fineA, 7 forceA, 8 monoA,
 * 9 coarseA, 10 farA, 11 fineB, 12 forceB, 13 monoB, 14 pplist4, 15 ppforce, 16 ppbox, 17 ppslot */
const void *orc_engine_buf(orc_engine *e, int which, long *bytes);
void orc_engine_set_threads(int n);

/* ---- the FP64 direct-sum gravity oracle ----
 * acceleration and potential at the targets idx[0..nt), from all N particles
 * (mass m[j], G = 1), Newton softened at eps (the P3M pass's own softening,
 * src/glsl-sim.js:745), the self term excluded; acc: nt*3, pot: nt */
void orc_direct_sum(int N, const float *pos4, const double *m, double eps, int nt, const int32_t *idx,
                    double *acc, double *pot);

/* ---- the analysis (src/nbody.js:646-893) ---- */
typedef struct {
  double largest, largestImp, largestIron, day, tilt, axis[3], bodyVel[3], orbit, escape;
  int hasSecond;
  double secMass, secDist, secImp, secIron, secCom[3], secCore[3], secVel[3], secR;
  int secBound;
  double com[3], core[3], vel[3], R, Redge, Tsurf, hotCom[3], hotR, impMass, impCom[3], impRms;
  double M, iron, drift, L, KE, PE, EL, Q, unseated, full, jD, moon;
  int ppCount, ppLoose;
} orc_report;
/* list: capacity cap; perm (may be NULL when sort == 0): N entries */
void orc_fof(int N, double mref, double a, const float *P, const float *V, const float *R, const float *D,
             double spring, double touch, int cap, int sort, orc_report *rep, int32_t *list, int32_t *perm);

#ifdef __cplusplus
}
#endif
#endif
