/*
 * ccstep.h -- C ABI of the B200 simulation step for cosmic-collisions.
 *
 * This library is a drop-in for the engine object `CC.nbody` that
 * src/nbody.js:1095-1118 hands the pages (index.html, src/view.js).  Each entry
 * point below names the reference function it replaces.  All functions return
 * an int status (CCS_OK, CCS_NOT_READY, or a negative CCS_E_* code); no C++
 * exception crosses this boundary.  A handle belongs to one host thread at a
 * time.  The handle owns every device buffer; the caller owns every host array
 * it passes.  Particle arrays are row-major: pos4/vel4/aux4/home4 are N x 4
 * float (x, y, z, w), mat and q are N floats -- the reference's RGBA32F / R32F
 * textures laid out by texel index i = y * W + x.
 *
 * Units are the reference's: G = M_earth = R_earth = 1 (src/nbody.js:7-10).
 */
#ifndef CCSTEP_H
#define CCSTEP_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCS_OK 0
#define CCS_NOT_READY 1      /* an async read-back is still in flight (src/nbody.js:1012-1013) */
#define CCS_E_ARG (-1)       /* bad argument, size or pointer */
#define CCS_E_CUDA (-2)      /* a CUDA call failed; ccs_last_error() says which */
#define CCS_E_STATE (-3)     /* call out of order (nothing built, nothing pending, ...) */
#define CCS_E_NOMEM (-4)     /* host or device allocation failed */
#define CCS_E_RANGE (-5)     /* size beyond a documented maximum */
#define CCS_E_KERNEL (-6)    /* a kernel reported an error through its status word */

#define CCS_SEATS 8          /* body-particles a contact cell holds: CC.SLOTS, src/shell.js:131 */
#define CCS_PP_CAP 8192      /* loose-list capacity: PP_CAP, src/nbody.js:38 */
#define CCS_PP_BINS 64       /* mesh pair table bins: src/nbody.js:109 */
#define CCS_MAX_N 262144     /* the 18-bit seat index: src/glsl-sim.js:96-109, CC.N_CHOICES */
#define CCS_SEAT_EMPTY 0xBF800000u /* -1.0f, the cleared seat (src/nbody.js:385) */

typedef struct ccs_handle ccs_handle;

/* The per-pass uniforms, rounded to binary32 as gl.uniform* rounds them
 * (src/nbody.js:255-336 setStaticUniforms, 342-350 boxes, 458-484 passSim). */
typedef struct {
  int N, W;
  int G, GShift, GMask, SX, SXShift, SXMask, AW, AH; /* contact grid, src/gl.js:73-75 */
  float invCell, cell, link2, reach2, touch;
  float K, C, invM, damp, creep, tK, kappa, cpIron;
  float dt, gdt, settle, kick;
  float bulk0[3], bulk1[3], cen0[3], cen1[3], spin0[3], spin1[3];
  float invH, eps2Mesh, eps2Cell, Gm;               /* eps2Mesh = FH^2, eps2Cell = FH^2/2 */
  float LA[3], LB[3], boxB;                         /* the two mesh boxes, src/glsl-sim.js:25-37 */
  float cut, a2;                                    /* P3M cut-off and particle radius^2 */
  float field, gField[3];                           /* 1: constant gravity gField (SIM_GRAV_FIELD) */
  float frozen;                                     /* the material held still (uFrozen); < 0: none */
  int ppCount;                                      /* loose-list length (pp.count) */
  float rot0[9], rot1[9], rdt;                      /* rigid carry (src/glsl-sim.js:537-570) */
  int ppSplit;                                      /* 0: the reference's loose-list pass; S > 0: the stencil-split P3M */
} ccs_uniforms;

/* The run's scalars: the fields of the reference's `sim` object
 * (src/nbody.js:212-234) that the step, the phases and the pages read. */
typedef struct {
  int N, W, H, n1, n2, G, settleLeft, settleTotal, stepNo, soft, phase; /* phase: 0 settle, 1 approach, 2 full */
  double m, a, cell, dt, k, c, creep, damp, tK, kappa;
  double R1, R2, Re1, Re2, M1, M2, M, vc, vesc, t, impactT;
  double spin0[3], spin1[3], cen0[3], cen1[3], bulk0[3], bulk1[3];
  double relr[3], relv[3];                          /* impactor relative to target (sim.rel) */
  int boxOn[2];                                     /* sim.boxes[b].on */
  double boxCen[2][3], boxVel[2][3], boxT[2];       /* sim.boxes[b].cen/vel/t */
} ccs_sim;

/* build(opt) options (src/nbody.js:114, index.html:250).  The last four fields
 * are extensions the reference fixes; 0 keeps the reference's value.
 * coreImp < 0 means "undefined" (use core). */
typedef struct {
  int N;
  double q, dens, core, coreImp, spin0, spin1, angle, incl, vfac, rest;
  int n2;
  double mImp;
  double mTarget;   /* target mass in M_earth (reference: 1) */
  double rhoR;      /* core/mantle density ratio (reference: 2.5, src/nbody.js:118) */
  double rhoCrust;  /* crust/mantle density ratio (reference: 1, src/nbody.js:155) */
  double crustFrac; /* crust = outer fraction of radius (reference: the outermost shell) */
} ccs_build_opt;

/* The analysis report of fof() (src/nbody.js:888-892), binary64. */
typedef struct {
  double largest, largestImp, largestIron, day, tilt, axis[3], bodyVel[3], orbit, escape;
  int hasSecond;
  double secMass, secDist, secImp, secIron, secCom[3], secCore[3], secVel[3], secR;
  int secBound;
  double com[3], core[3], vel[3], R, Redge, Tsurf, hotCom[3], hotR, impMass, impCom[3], impRms;
  double M, iron, drift, L, KE, PE, EL, Q, unseated, full, jD, moon;
  int ppCount, ppLoose;
} ccs_report;

/* Headless device buffers in place of the GL textures src/view.js reads
 * (sim.src.pos/vel/aux/q, sim.mat, sim.home: src/view.js:216-220,566-569). */
typedef struct {
  void *pos4, *vel4, *aux4, *q, *mat, *home4;
  void *force[2], *mono[2];                         /* pm[b].force (64^3 + scratch), pm[b].mono */
  void *stream;                                     /* the cudaStream_t every kernel runs on */
} ccs_device_buffers;

/* ---- lifecycle: CC.nbody.init (src/nbody.js:1032-1092) ---- */
int ccs_create(int device, ccs_handle **out);
int ccs_destroy(ccs_handle *h);
const char *ccs_last_error(const ccs_handle *h);
int ccs_version(void);

/* ---- building a run ---- */
/* Host-side builder: build() of src/nbody.js:114-250 with ball/relax/maclaurin
 * of src/bodies.js:23-160 and mulberry of src/math.js:8-15.  Fills sim and the
 * particle arrays (pos4, vel4, home4: N*4 floats; mat: N floats). */
int ccs_make_bodies(const ccs_build_opt *opt, ccs_sim *sim, float *pos4, float *vel4, float *mat, float *home4);
/* The same builder with relax() (src/bodies.js:97-146) on GPU `device`: the
 * shells, layers, masses, encounter and every other output are the host
 * builder's; the ten sweeps run as 27 race-free phases of cells a sweep, each
 * cell's particles walked in index order, so the relaxed pile is equivalent
 * to the host's (the same overlap statistics, each particle within a small
 * fraction of a radius) but not bit-identical.  Allocates device memory for
 * the call's duration. */
int ccs_make_bodies_device(int device, const ccs_build_opt *opt, ccs_sim *sim, float *pos4, float *vel4, float *mat,
                           float *home4);
/* Upload a run: the texture uploads and setStaticUniforms of src/nbody.js:208-249.
 * home4 may be NULL. */
int ccs_build(ccs_handle *h, const ccs_sim *sim, const float *pos4, const float *vel4, const float *mat,
              const float *home4);
/* The live run scalars (CC.nbody.sim): the caller may advance sim->t as the
 * frame loop does (index.html:372).  After changing static fields (k, c, dt,
 * damp, spins ...) call ccs_set_static (setStaticUniforms, src/nbody.js:255). */
ccs_sim *ccs_sim_ptr(ccs_handle *h);
int ccs_set_static(ccs_handle *h);
int ccs_get_uniforms(ccs_handle *h, ccs_uniforms *out);
/* meshEvery setter, src/nbody.js:1115 (default 8) */
int ccs_set_mesh_every(ccs_handle *h, int n);

/* The field-gravity step of the crater page: simFS({gravity: 'field',
 * frozen: true}) (src/glsl-sim.js:466-468, 490-492, 517-533) on the page's
 * schedule (chicxulub.html:763-766: the contact grid on even steps, the
 * contact step with uGDt = dt on every step, no mesh, no pairwise pass, no
 * soften).  g is the constant acceleration (uGField); particles whose tag is
 * within 0.5 of `frozen` are held still (a negative value holds none); invM
 * and cpIron replace the impact's 1/m and cp_iron/cp_rock (the crater page
 * sets both to 1: its spring is per unit mass and all its material is rock).
 * on = 0 returns to the impact's mesh step.  Applies from the next step. */
int ccs_set_field(ccs_handle *h, int on, const double g[3], double frozen, double invM, double cpIron);

/* ---- the step: src/nbody.js:551-558 step(settle, kick) ---- */
int ccs_step(ccs_handle *h, int settle, int kick);
/* n frame-loop steps: { step(false,false); sim.t += sim.dt } (index.html:372),
 * replayed from captured CUDA graphs in blocks of meshEvery steps. */
int ccs_steps(ccs_handle *h, int n);
/* settleSome(n), src/nbody.js:561-566 */
int ccs_settle_some(ccs_handle *h, int n);
/* rigidStep(dtF), src/nbody.js:591-636: CPU two-body leapfrog + GPU rigid carry,
 * and the first-touch kick step */
int ccs_rigid_step(ccs_handle *h, double dtF);

/* ---- the analysis hand-off: applyReport (src/nbody.js:912-966) ---- */
/* setPP: the loose list (particle indices), then its pairwise pass at once */
int ccs_set_pp(ccs_handle *h, const int32_t *list, int n, int loose);
/* placeBoxes' priming of a box's mono texel (src/nbody.js:368-370) */
int ccs_prime_mono(ccs_handle *h, int box, const float mono[4]);
/* One mesh box as placeBoxes leaves it (sim.boxes[b], src/nbody.js:361-374). */
typedef struct {
  int on;            /* the box is up: box 0 rides the largest body, box 1 a separating second body */
  double cen[3];     /* the body's core at the look (r.core / r.second.core) */
  double vel[3];     /* the body's velocity: boxes() carries the centre on at it (src/nbody.js:342-344) */
  double t;          /* the time of the look */
  int primeMono;     /* 1: the box has just gone up; mono is its first monopole (src/nbody.js:366-370) */
  float mono[4];     /* sum of m x and of m, in particle masses (read when primeMono is 1) */
} ccs_box;
/* placeBoxes(r): both boxes at once, validated (on is 0 or 1; every value finite; |cen| within 1e6 R_earth)
 * before anything changes; CCS_E_ARG otherwise.  Takes effect at the next mesh step. */
int ccs_set_boxes(ccs_handle *h, const ccs_box boxes[2]);
/* applyPerm(perm): state, mat and home gathered by perm, then fresh contact cells */
int ccs_apply_perm(ccs_handle *h, const int32_t *perm);
/* The Morton order of src/nbody.js:871-887 computed on the device (keys in
 * binary64, stable radix sort), applied as applyPerm.  perm_out and into_out
 * (N int32 each) may be NULL; into_out renames a loose list. */
int ccs_sort_morton(ccs_handle *h, const double core[3], int32_t *perm_out, int32_t *into_out);
/* analyze(): passDiag (src/nbody.js:488-507) and the asynchronous read-back of
 * diag, pos and vel (src/nbody.js:977-993) into pinned staging ... */
int ccs_diag_async(ccs_handle *h);
/* ... collected without blocking (src/nbody.js:1011-1025): CCS_NOT_READY until
 * the copy has landed.  P, V, D: N*4 floats each (any may be NULL). */
int ccs_poll(ccs_handle *h, float *P, float *V, float *D);
/* The host analysis, fof() of src/nbody.js:646-893 (CPU, binary64): groups,
 * books, loose list (cap entries) and, with sort, the Morton permutation. */
int ccs_fof(int N, double mref, double a, const float *P, const float *V, const float *R, const float *D,
            double spring, double touch, int cap, int sort, ccs_report *rep, int32_t *list, int32_t *perm);
/* The same analysis on the device, on the engine's current state (it runs the
 * diag pass first, as analyze() reads diag): the groups over an exact cell
 * list with a lock-free union-find, every sum in binary64, the loose list by
 * an ordered compaction and, with sort, the Morton order of ccs_sort_morton's
 * key.  Same report, loose list (cap <= CCS_PP_CAP) and permutation as
 * ccs_fof on the read-back state, the report's sums to rounding (they are
 * added in another order); a tie between the two largest groups' sizes goes
 * to the group holding the smaller index. */
int ccs_fof_device(ccs_handle *h, double spring, double touch, int cap, int sort, ccs_report *rep, int32_t *list,
                   int32_t *perm);
/* The mesh's own pair force and potential by distance, meshPairTable of
 * src/nbody.js:56-108 (host, binary64 -> binary32). */
int ccs_pair_table(int bins, double cut, float *f, float *p);

/* ---- read-outs ---- */
int ccs_read_state(ccs_handle *h, float *pos4, float *vel4, float *aux4, float *q, float *mat);
int ccs_write_state(ccs_handle *h, const float *pos4, const float *vel4, const float *aux4, const float *q,
                    const float *mat);
int ccs_device_ptrs(ccs_handle *h, ccs_device_buffers *out);
/* Conservation books on the device in binary64 (the sums of src/nbody.js:837-850):
 * out[0] M, [1..3] momentum, [4..6] angular momentum about the origin, [7] KE,
 * [8] PE (needs a diag pass), [9] Q/2, [10] unseated fraction, [11] full fraction */
#define CCS_BOOKS 12
int ccs_books(ccs_handle *h, int with_diag, double out[CCS_BOOKS]);
/* The exact pull, for the force-error measurement and the learned correction's
 * labels (no counterpart in the reference, which has no direct sum): binary64
 * acceleration (n*3) and potential (n) at the particles idx[0..n), from all N,
 * Newton softened at the particle radius a (the P3M pass's softening,
 * src/glsl-sim.js:745), self term excluded, G = 1. */
int ccs_direct_sum(ccs_handle *h, const int32_t *idx, int n, double *acc3, double *pot);
/* The P3M pairwise correction of PPFORCE_FS (src/glsl-sim.js:700-754) over a
 * list of any length n <= N (particle indices), without the reference's
 * 8,192 cap (PP_CAP, src/nbody.js:38): for each member, the sum over every
 * other member inside the cut, the four slices of the capped pass added
 * together, x Gm, as (pull xyz, potential) in force4 (n x 4 floats), at the
 * current positions with the boxes and table the step's pass uses.  The run
 * is not changed.  For measuring the uncapped form of the reference's method
 * (the gravity sweep's loose list exceeds the cap); allocates scratch for the
 * call. */
int ccs_pp_list_force(ccs_handle *h, const int32_t *list, int n, float *force4);

/* The P3M pairwise pass with no allocation at all, for callers that may not
 * call cudaMalloc (a host running inside a device-memory budget it does not
 * own, or code that must not pay cudaMalloc's device-wide synchronisation).
 * No counterpart in the reference.  Every pointer is caller-owned device
 * memory: list4 (n x float4: position, mass ratio; 0 mass = empty seat), box
 * (n floats: the box each entry reads, -1 for neither), tab2 (64 x 2 floats:
 * the mesh pair table of ccs_pair_table), force4 (out: 4 x n float4, the four
 * quarter-list slices, slice-major, as the contact step adds them).  cut, a2
 * and gm are the uniforms uCut, uA2, uGm.  stream is a cudaStream_t (NULL:
 * the legacy default stream).  n may not exceed CCS_PP_STATIC_MAX
 * (CCS_E_RANGE otherwise).  The scratch is one static 2 MiB device array
 * shared by all calls: calls that overlap on the GPU race.  The first call on
 * a device looks the array up on that device; make it before any stream
 * capture. */
#define CCS_PP_STATIC_MAX 2048
int ccs_pp_force_static(const float *list4, const float *box, int n, const float *tab2, float cut, float a2,
                        float gm, float *force4, void *stream);

/* ---- the learned pairwise correction ----
 * No counterpart in the reference.  The plain pass subtracts the mesh's pair
 * force as the placement-averaged table of meshPairTable (src/nbody.js:48-109;
 * PPFORCE_FS's T.f, src/glsl-sim.js:738-750).  Here the mesh's pair force is
 * the node-softened Newton force d / (r^2 + FH^2/2)^(3/2) (what it is exactly
 * when the two particles share no mesh node) plus a network R(d, s) for
 * the rest: d the pair offset in mesh cells (source - target), s the source's
 * position in its cell; 6 -> 64 -> 64 -> 3 with SiLU, BF16 weights, FP32
 * accumulation, run and trained on the tensor cores.  With a network
 * attached, the P3M pass of an engine models the mesh's pull on the loose
 * pairs inside CCS_NN_CUT_CELLS cells (half the plain pass's 5) by
 * d/(r^2 + FH^2/2)^(3/2) + R(d, s)/FH^2 instead of the table (blended into
 * the table by a smoothstep from 0.8 of those cells out to them) and keeps the
 * table beyond, out to the plain cut; the potential keeps the table's.
 * Detaching it restores the plain pass.  Flat parameter order:
 * W1[64][6] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]. */
#define CCS_NN_PARAMS 4803
#define CCS_NN_CUT_CELLS 2.5
typedef struct ccs_nn ccs_nn;
int ccs_nn_create(int device, uint32_t seed, ccs_nn **out);
int ccs_nn_destroy(ccs_nn *nn);   /* detach it from every engine first */
const char *ccs_nn_last_error(const ccs_nn *nn);
int ccs_nn_set_params(ccs_nn *nn, const float *params);   /* also resets the optimiser */
int ccs_nn_get_params(ccs_nn *nn, float *params);
/* The pair pool the network trains on: records (d in cells, s in [0,1)) with
 * their labels, the mesh arithmetic of meshPairTable's field() for the
 * isolated pair in binary64 less the softened Newton force (cells^-2, unit
 * masses). */
int ccs_nn_clear(ccs_nn *nn);
int64_t ccs_nn_pool_size(const ccs_nn *nn);
/* count pairs of the engine's particles inside the cut, both in box 0; odd
 * records pair Morton neighbours (index within 128), even ones any two */
int ccs_nn_sample_state(ccs_nn *nn, ccs_handle *h, int64_t count, uint32_t seed);
/* count synthetic pairs: s uniform, d uniform in the ball or in distance */
int ccs_nn_sample_uniform(ccs_nn *nn, int64_t count, uint32_t seed);
/* records n x 6 floats (NaN offsets mark a dead record), labels n x 3 */
int ccs_nn_read_pool(ccs_nn *nn, int64_t first, int64_t n, float *rec6, float *label3);
/* Adam on the mean squared error over pool records [first, first + n):
 * batches of (SMs x tilesPerCta x 128) pairs, cosine decay from lr to lr/20;
 * epochLoss (epochs floats, may be NULL) gets each epoch's mean loss */
int ccs_nn_train(ccs_nn *nn, int64_t first, int64_t n, int epochs, int tilesPerCta, float lr, float *epochLoss);
/* host records in, the network's output (n x 3) / the label (n x 3) out */
int ccs_nn_forward(ccs_nn *nn, const float *rec6, int64_t n, float *out3);
int ccs_nn_labels(ccs_nn *nn, const float *rec6, int64_t n, float *label3);
/* the gradient (CCS_NN_PARAMS floats) and loss of the mean squared error over
 * n host records, through the training kernel, without a step */
int ccs_nn_grad(ccs_nn *nn, const float *rec6, const float *label3, int64_t n, float *grad, float *loss);
/* attach (or, with NULL, detach) a network to an engine's P3M pass */
int ccs_set_pp_nn(ccs_handle *h, ccs_nn *nn);

/* ---- the stencil-split P3M: gravity to a stated accuracy ----
 * No counterpart in the reference.  The reference's pairwise pass corrects
 * only the loose list (src/nbody.js:851-870, capped at PP_CAP) against the
 * mesh's placement-averaged pair table (src/glsl-sim.js:700-754), so
 * particles inside a body keep the mesh's near field, a cell-centre sum
 * softened by FH^2/2 at every distance: a few per cent off Newton.  With
 * S = 1, 2 or 3 the split form hands every pair of mesh nodes within S cells
 * of each other (Chebyshev) to an exact pairwise sum over every particle --
 * each particle pair weighted by the share of its cloud-in-cell node pairs
 * that lie inside the stencil, so mesh and pairs partition the interaction
 * exactly -- and keeps the rest on the mesh, unsoftened, gathered to first
 * order from each node's centre of mass by the node's tidal tensor.  Pairs
 * are Newton softened at the particle radius, the reference's own pairwise
 * softening (src/glsl-sim.js:745); particles in neither box keep the boxes'
 * monopoles.  The loose list is not used while the form is on.  S = 0
 * returns to the reference's pass.  Applies from the next mesh step;
 * allocates its buffers on first use (about 220 MB plus 80 B a particle). */
int ccs_set_pp_split(ccs_handle *h, int S);
/* The split form's pair pass takes the pairs between two mesh nodes that
 * each hold at least minNode particles once, adding each pair's reaction to
 * the other particle (Newton's third law), in float atomics; smaller nodes
 * take every pair one way, in a fixed order.  minNode = 0 takes every pair
 * one way (deterministic); otherwise at least 16 (CCS_E_ARG).  Default 16.
 * No counterpart in the reference. */
int ccs_set_pp_split_sym(ccs_handle *h, int minNode);
/* The split form's last pair pass, counted: counts[0] the (target, source)
 * pair evaluations taken one way, counts[1] those taken once for both
 * particles (each a force on both); waits for the pass.  Zeros before the
 * form's first pass; CCS_E_STATE before the form was ever switched on.  No
 * counterpart in the reference. */
int ccs_pp_split_pairs(ccs_handle *h, uint64_t counts[2]);

/* ---- launch shapes by measurement ----
 * No counterpart in the reference (WebGL fixes its own shapes).  Times the
 * contact step at 8 and 4 warps per CTA and the cell gravity at 2, 4 and 8
 * threads per fine cell, `reps` launches each, on the run's current state
 * (the contact step writes only the spare state buffers; the cell gravity
 * rewrites the last mesh step's force from the same inputs), keeps the fastest
 * of each for this run and for every later run of the same particle count and
 * grid in the process.  reps = 0 measures nothing: it applies what an earlier
 * call measured for this size (or the defaults 8 and 4).  choice (may be NULL)
 * gets {warps, threads per cell}.  Tune a state that has taken a mesh step. */
int ccs_autotune(ccs_handle *h, int reps, int choice[2]);

/* ---- the batched ensemble ----
 * No counterpart in the reference, which runs one impact per page.  An
 * ensemble advances several engines (impacts of any sizes, on one device)
 * together: up to four rounds of meshEvery steps are one CUDA graph holding
 * every member's steps as a parallel branch, replayed with one launch.  The members
 * stay ordinary engines (their own streams, buffers and read-outs); work a
 * caller queues on a member is ordered before and after the ensemble's
 * rounds.  Members must outlive the ensemble, share one meshEvery, and sit at
 * a block boundary (stepNo % meshEvery == 0) when ccs_ensemble_steps is
 * called; n is a multiple of meshEvery. */
typedef struct ccs_ensemble ccs_ensemble;
int ccs_ensemble_create(ccs_handle *const *members, int count, ccs_ensemble **out);
int ccs_ensemble_destroy(ccs_ensemble *e);
const char *ccs_ensemble_last_error(const ccs_ensemble *e);
int ccs_ensemble_steps(ccs_ensemble *e, int n);
int ccs_ensemble_sync(ccs_ensemble *e);   /* waits for the rounds; reports any member's kernel status */
/* The ensemble's launch shapes by measurement: every combination of the
 * contact step's CTA width (8, 4 warps) and the cell gravity's threads per
 * cell (2, 4, 8) is applied to all members and timed over `rounds` real
 * rounds of the ensemble after one round that captures its graph (the
 * members advance: 6 x (rounds + 1) x meshEvery steps when rounds <= 4); the
 * fastest aggregate is kept.  Shapes that win for one run alone
 * can lose when many runs share the GPU, which is why the ensemble measures
 * its own.  choice (may be NULL) gets {warps, threads per cell}. */
int ccs_ensemble_autotune(ccs_ensemble *e, int rounds, int choice[2]);
/* The ensemble's persistent form (on = 1; 0 returns to the branch form).  No
 * counterpart in the reference.  Each round of 8 steps is then one launch of
 * a persistent kernel over every member: after the members' mesh chains for
 * the round's mesh step (parallel branches, as before), the launch runs every
 * member's contact grids and contact steps of the round, as many CTAs as the
 * device holds at once taking work items from per-member queues (a member's
 * next step starts as soon as its own previous one is finished; members never
 * wait for one another).  The rounds stay CUDA graphs, four to a replay.  The
 * members must run the impact's step with the reference's P3M (no field
 * step, stencil-split or learned pass; CCS_E_STATE) and meshEvery 8.  Every
 * wait in the kernel is bounded (2 s); one that runs out abandons the round,
 * and ccs_ensemble_sync reports CCS_E_KERNEL. */
int ccs_ensemble_set_persistent(ccs_ensemble *e, int on);
/* Per member (count = the members), the mean time of one step inside the
 * persistent rounds since the last call, in ms: from the member's first work
 * item to its last in each round (%globaltimer), over 8; -1 for a member no
 * persistent round has run.  Waits for the rounds; resets the sums. */
int ccs_ensemble_step_ms(ccs_ensemble *e, double *ms, int count);
/* persistent rounds launched (one kernel launch each) */
int64_t ccs_ensemble_launch_count(const ccs_ensemble *e);
/* The bound on every wait of the persistent round, in ns (default 2e9).  A
 * bound shorter than the round's ordinary waits abandons the round: the way
 * the time-out path is tested without a hang.  Also clears the ensemble's
 * status word. */
int ccs_ensemble_set_wait_ns(ccs_ensemble *e, uint64_t ns);

/* The contact-pair sets of the current state, read out for checking: the
 * contact step's own walk over the current seat table (the 27 cells, the
 * seat cull, the link test, src/glsl-sim.js:415-450), with each pair inside
 * the link radius written to its owner's row as the neighbour's index, bit 31
 * set when the two touch (2a - r > 0).  counts (N) gets each owner's
 * neighbour count; pairs (N x cap) its first min(count, cap) pairs in no
 * particular order, the rest 0xFFFFFFFF.  The run does not advance.  No
 * counterpart in the reference, whose pairs live only inside simFS's loop.
 * Allocates device memory for the call's duration. */
int ccs_contact_pairs(ccs_handle *h, int cap, int32_t *counts, uint32_t *pairs);

/* Internal buffers, for tests and the console checks of index.html:531-556:
 * which = CCS_BUF_* below; bytes must equal the buffer's size. */
enum {
  CCS_BUF_SEATS = 5, CCS_BUF_FINE_A = 6, CCS_BUF_FORCE_A = 7, CCS_BUF_MONO_A = 8, CCS_BUF_COARSE_A = 9,
  CCS_BUF_FAR_A = 10, CCS_BUF_FINE_B = 11, CCS_BUF_FORCE_B = 12, CCS_BUF_MONO_B = 13, CCS_BUF_PP_LIST = 14,
  CCS_BUF_PP_FORCE = 15, CCS_BUF_PP_BOX = 16, CCS_BUF_PP_SLOT = 17, CCS_BUF_DIAG = 18, CCS_BUF_CELL_OF = 19,
  CCS_BUF_TIDE0_A = 20, CCS_BUF_TIDE1_A = 21, CCS_BUF_PP_ALL = 22,  /* the stencil-split P3M's (ccs_set_pp_split) */
  /* the contact walk's record (ccs_set_contact_walk): 3 uint32 -- particles
   * whose step replayed the record, replayed it and walked the cells a new
   * cell added, walked -- counted while the mode is 2; (N + 31) / 32 int32 --
   * seats recorded per warp of 32 particles by the last step that rebuilt the
   * grid (1537: more than fit) */
  CCS_BUF_WALK_STATS = 23, CCS_BUF_WALK_COUNT = 24,
  /* the stencil-split P3M's second gradient of the pull at each cell of box A:
   * three planes of 64^3 + 1 float4 (Gxxx Gyyy Gzzz Gxyz), (Gxxy Gxxz Gxyy
   * Gyyz), (Gxzz Gyzz) */
  CCS_BUF_TIDE2_A = 25,
  /* ... and each cell's second moment about its centre of mass: two planes
   * of 64^3 + 1 float4 (Qxx Qyy Qzz Qxy), (Qxz Qyz) */
  CCS_BUF_FINEQ_A = 26
};
int ccs_read_buffer(ccs_handle *h, int which, void *dst, size_t bytes);

/* ---- single passes: CC.nbody.passes (src/nbody.js:1105) ---- */
int ccs_pass_slots(ccs_handle *h);
int ccs_pass_mesh(ccs_handle *h);            /* boxes() + passMesh() */
int ccs_pass_pp(ccs_handle *h);
int ccs_pass_sim(ccs_handle *h, int settle, int kick, double gdt);
int ccs_pass_diag(ccs_handle *h);

/* ---- host-buffer step (the plugin call a host without device memory makes):
 * upload pos/vel/q from host arrays, run nsteps frame-loop steps, read
 * pos/vel/aux/q back.  Any output pointer may be NULL. ---- */
int ccs_advance_host(ccs_handle *h, const float *pos4, const float *vel4, const float *q, int nsteps,
                     float *pos4_out, float *vel4_out, float *aux4_out, float *q_out);

/* ---- checkpoint and restore (no counterpart in the reference: its runTo
 * replays a run from the build, index.html:592-600) ----
 * A run's whole state at a step whose successor rebuilds everything derived
 * from it -- the contact grid, the mesh and the pairwise pass: stepNo a
 * multiple of meshEvery for the impact's step, an even stepNo for the field
 * step; elsewhere ccs_checkpoint_save returns CCS_E_STATE.  Restored into any
 * handle, the run continues as the saved one would (to the rounding of the
 * float atomics that sum contacts and deposits).  Layout, little-endian:
 * this header; the ccs_sim struct (simBytes); pos4, vel4, aux4 (16 B a
 * particle each), q, mat (4 B each), home4 (16 B); the loose list (4 B x
 * ppCount); the caller's own bytes (extraBytes, e.g. its analysis state).
 * checksum = the CRC-32 of zlib (IEEE 802.3 polynomial, reflected, initial
 * and final value 0xFFFFFFFF) of everything after the header. */
#define CCS_CKPT_MAGIC "CCSCKPT1"
#define CCS_CKPT_VERSION 1u
typedef struct {
  char magic[8];
  uint32_t version, headerBytes, simBytes, flags;   /* flags: 2 = the field step is on */
  int32_t N, meshEvery, ppCount, ppLoose;
  double field[6];                                  /* ccs_set_field's g[3], frozen, invM, cpIron */
  float monoA[4], monoB[4];                         /* the boxes' monopoles (the strays' pull, src/glsl-sim.js:196-206) */
  uint64_t extraBytes, payloadBytes, checksum;      /* payloadBytes: everything after the header */
} ccs_checkpoint_header;
int ccs_checkpoint_size(ccs_handle *h, size_t extraBytes, size_t *bytes);
int ccs_checkpoint_save(ccs_handle *h, const void *extra, size_t extraBytes, void *buf, size_t cap);
/* rebuilds the handle's run from buf (as ccs_build does) and restores the rest */
int ccs_checkpoint_load(ccs_handle *h, const void *buf, size_t bytes);

/* ---- timing helpers for the benchmark ---- */
int ccs_sync(ccs_handle *h);
/* CUDA-graph replay of steps on (1, the default) or off (0: every kernel
 * launched directly), for comparing the two paths and for debugging */
int ccs_set_graphs(ccs_handle *h, int on);
/* How the contact step finds its pairs (src/glsl-sim.js:415-450) on the step
 * after a grid rebuild, which walks the same seat tables.  1 (the default):
 * the rebuilding step's walk records, per particle, the seats its cull kept
 * in the cells within the link radius and a margin; the next step replays
 * that record (every decision of the walk recomputed, the pair sets and the
 * neighbour counts the same) for the particles that moved less than the
 * margin, and walks the seat tables for the others and for every particle
 * after any call that moves or reorders them between the two steps (state
 * writes, permutations, rigid steps, checkpoint loads, passes run by hand).
 * 0: every step walks the seat tables.  2: as 1, and the replaying steps
 * count how each particle found its pairs (CCS_BUF_WALK_STATS; the counts
 * start from zero when this mode is set). */
int ccs_set_contact_walk(ccs_handle *h, int mode);
/* average device time (ms) of the kernels named by `kernel` launched since the
 * last reset, measured with CUDA events on the handle's stream; kernel ids:
 * 0 contact step (simulate), 1 contact grid, 2 deposit, 3 cell, 4 P3M force,
 * 5 and 6 the two halves of a split mesh step (the contact walk, which stops
 * at the contact sums, and the tail: gravity, settle/kick, heat, kick/drift).
 * `enable` is a mask of the ids to time (bit k for id k; CCS_TIME_ALL for all,
 * 0 for none): each timed launch records two events, which widen the gap
 * before and after it by a microsecond or two.  Timing ids 5 or 6 runs mesh
 * steps split and in order on the handle's stream; timing any of ids 1-4
 * runs them whole. */
#define CCS_TIME_ALL 0x7F
int ccs_timing(ccs_handle *h, int enable);
/* time the contact step on every `every`-th launch only (1, the default: on
 * every launch), so that a long run carries its events on a sample */
int ccs_timing_every(ccs_handle *h, int every);
int ccs_timing_read(ccs_handle *h, int kernel, double *total_ms, int *launches);
/* kernels launched by this handle since creation (the benchmark's gpu_launches) */
int64_t ccs_launch_count(ccs_handle *h);

#ifdef __cplusplus
}
#endif
#endif
