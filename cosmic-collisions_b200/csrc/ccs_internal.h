// ccs_internal.h -- the handle and the kernel launchers shared by the API.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/ccstep.h"

namespace ccs {

constexpr uint32_t kEmpty = CCS_SEAT_EMPTY;   // -1.0f bit pattern: an empty seat
constexpr uint32_t kNoCell = 0xFFFFFFFFu;     // no cell recorded for this particle
constexpr int kFine = 64 * 64 * 64;           // 64^3 mesh; index kFine is the scratch texel
constexpr int kSplitKeys = 2 * kFine;         // the stencil-split pair pass's sort keys: (box, base node); this one: neither box
constexpr int kSymMinNode = 16;               // the least node size ccs_set_pp_split_sym accepts (its items' room)
constexpr int kCoarse = 4096;                 // 16^3 blocks
constexpr int kCellChunks = 8;                // CTAs of the cell pass per occupied block, each a source chunk
constexpr int kSeats = CCS_SEATS;
constexpr unsigned kStatusGrid = 1u;          // a contact-cell insertion gave up (degenerate pile)
constexpr unsigned kStatusNN = 2u;            // a tensor-core wait of the learned P3M pass gave up
constexpr unsigned kStatusFof = 4u;           // a union of the device analysis gave up its retries
constexpr int kRecWarp = 1536;                // seats a grid step's contact walk records per warp for the next step

// the analysis on the device (ccs_fof.cu): src/nbody.js:646-893
constexpr int kFofBuckets = 1 << 20;          // hashed cells of side 2.4 a, as the host restatement hashes them
constexpr int kFofTerms = 13;                 // binary64 terms one sum pass adds per particle
constexpr int kFofBins = 96;                  // shells of the density histogram
enum FofPass { kFofGroup = 0, kFofCore, kFofShape, kFofProper1, kFofProper2, kFofProper3, kFofOrbit, kFofBooks };
struct FofSumArgs {
  int N, pass, g;                             // g: the group label the pass is about
  double mref, r2, s0, s1;
  double c[3], d[3];                          // a centre and a second vector, by pass
  const float4 *pos, *vel, *diag;
  const float *mat;
  const int *label;
};
struct FofLooseArgs {
  int N, len, bigB;
  double RA, RB, least;
  double comA[3], comB[3];
  const float4 *pos;
};
int fof_blocks(int N);
int launch_fof_groups(int N, const float4 *pos, double a, double touch, double spring, uint32_t *keys, int32_t *vals,
                      uint32_t *keysTmp, int32_t *valsTmp, uint32_t *hist, int *start, int *end, int *parent,
                      int *size, double *elasticPart, unsigned long long *top, unsigned *status, cudaStream_t st);
int launch_fof_sums(const FofSumArgs &a, double *part, cudaStream_t st);
int launch_fof_hist(const FofSumArgs &a, double dr, double *part, cudaStream_t st);
int launch_fof_loose(const FofLooseArgs &a, int pass, int *counts, int *offs, double *dist, int *nDist,
                     int32_t *list, cudaStream_t st);
int launch_fof_remap(int n, const int32_t *into, int32_t *list, cudaStream_t st);

// One gravity mesh box: the textures of meshBox(), src/nbody.js:1050-1068,
// as plain float4 arrays.  fine/force hold 64^3 cells in [z][y][x] order
// plus the scratch texel at index 64^3 (the atlas row y = 512 of the reference).
struct MeshBuf {
  float4 *fine = nullptr, *force = nullptr;
  float4 *coarse = nullptr, *farA = nullptr, *farT0 = nullptr, *farT1 = nullptr;
  float4 *mono = nullptr;
  float4 *partial = nullptr;   // per-block partial sums for the monopole
  unsigned *counter = nullptr; // last-block-done counter of the coarse pass
  float4 *occ = nullptr;       // per coarse block: its occupied fine cells (centre of mass, mass), 64 slots
  uint8_t *occIdx = nullptr;   // ... and their place in the block
  int *occN = nullptr;         // ... and how many there are
  int *occBlocks = nullptr;    // the occupied coarse blocks (any order) ...
  int *occCount = nullptr;     // ... and how many
  int *occAsc = nullptr;       // the occupied coarse blocks in ascending order ...
  int *occAscN = nullptr;      // ... and how many
  float4 *cellPart = nullptr;  // the cell pass's partial sums: [listed block][source chunk][cell]
  int *cellDone = nullptr;     // per listed block: the chunks done (the last one adds them up)
  // the stencil-split P3M's mesh (allocated when that form is switched on): each cell's tidal tensor, the
  // pull's second gradient (tide2: three planes of kFine + 1), and the cell pass's partial sums of pull,
  // potential, tide and second gradient: [listed block][source chunk][5][cell]
  float4 *tide0 = nullptr, *tide1 = nullptr, *tide2 = nullptr, *cellPartT = nullptr;
  float4 *fineQ = nullptr;   // each cell's second moment about its centre of mass: two planes of kFine + 1
  float4 *quad0 = nullptr, *quad1 = nullptr;   // each block's second moment about its centre of mass
};

// Arguments of the contact step (simFS, src/glsl-sim.js:354-512).
struct SimArgs {
  const float4 *pos, *vel;
  const float *mat, *q;
  const uint32_t *seats;
  const float4 *forceA, *monoA, *forceB, *monoB;
  const int *ppSlot;
  const float4 *ppForce;
  int cap;
  float4 *posO, *velO, *auxO;
  float *qO;
  int first = 0;   // the launch's first particle (a launch over a range of them)
  float4 *part = nullptr;   // a split mesh step's contact sums: push, neighbour count
  float2 *part2 = nullptr;  // and dissipation, heat flow
  uint32_t *pairs = nullptr;  // the contact-pair read-out: per owner pairCap words, neighbour | touching << 31
  int pairCap = 0;
  // the stencil-split P3M's gather: each box's tides and deposit (centres of mass), and each particle's pairs
  const float4 *tideA0 = nullptr, *tideA1 = nullptr, *tideB0 = nullptr, *tideB1 = nullptr;
  const float4 *tideA2 = nullptr, *tideB2 = nullptr;   // the second gradient's three planes (kFine + 1 apart)
  const float4 *fineA = nullptr, *fineB = nullptr, *ppAll = nullptr;
  // the contact walk's record (ccs_contact.cu).  walk 1, a step that rebuilt the grid: the walk also writes,
  // per warp, every seat its cull kept in the cells within recLink2 of an owner (rec[warp * kRecWarp + k],
  // particle | owner lane << 18 | the owner's cell it came from << 23), how many (recN[warp]; kRecWarp + 1
  // when they did not fit), where each owner was (recP), and the largest squared displacement of the
  // step's kick/drift (recMax, the bits of a float; the grid zeroes it).  walk 2, the next step (same
  // seats): owners that moved less than sqrt(recMove2) replay the record instead of walking the seat
  // tables, while recMax is at most recAll2.  walk 0: the walk alone
  uint32_t *rec = nullptr;
  int *recN = nullptr;
  float4 *recP = nullptr;
  unsigned *recMax = nullptr;
  unsigned *recStats = nullptr;   // walk 2, optional: owners that replayed, replayed and walked new cells, walked
  int walk = 0;
  float recLink2 = 0.0f, recMove2 = 0.0f, recAll2 = 0.0f;
};

// The ensemble's persistent round (k_ensemble_round, ccs_contact.cu): every member's steps of one round of
// kEnsSteps in one launch.  Each member's round is a chain of segments -- on an even step the contact grid's,
// then each step's contact step -- cut into work items (kEnsGridItem particles for the grid, kEnsContactItem
// for the contact step) numbered by one ticket counter per member; a segment's items start once the segment
// before it is finished.  The mesh and the pairwise pass of the round's mesh step run before the launch.
constexpr int kEnsSteps = 8;          // steps a persistent round holds (the ensemble's meshEvery)
constexpr int kEnsSegs = 2 * kEnsSteps;
constexpr int kEnsWarps = 8;          // the contact step's CTA width in the round (8 warps: 2.06e9 against 1.98e9 with 4)
constexpr int kEnsContactItem = 32 * kEnsWarps;   // particles of a contact-step work item (one CTA's)
constexpr int kEnsGridItem = 512;     // particles of a grid work item
constexpr unsigned kStatusEnsemble = 8u;   // a wait of the ensemble's persistent round ran out
struct EnsStepArgs {                  // one member's step
  ccs_uniforms u;
  SimArgs a;                          // the contact step's (the walk in a.walk)
  // the contact grid's, on a step that rebuilds it: as launch_contact_grid takes them
  const float4 *gpos;
  uint32_t *gseats, *ghk, *gseatsOld;
  const uint32_t *ghkOld;
  unsigned *gstatus, *grecMax;
};
struct EnsMember {                    // a member's round: its segments (fixed by its size)
  int nseg, total;                    // segments, work items
  int end[kEnsSegs];                  // segment s holds tickets [s ? end[s - 1] : 0, end[s])
  int step[kEnsSegs];                 // the step it belongs to
  int grid[kEnsSegs];                 // 1: the contact grid; 0: the contact step
};
struct EnsState {                     // a member's counters in one launch, zeroed before it
  int next;                           // the next ticket
  int done[kEnsSegs];                 // work items finished, per segment
  int pad;
  unsigned long long t0;              // %globaltimer when its first item was taken
};
struct EnsLaunch {
  int members, steps;                 // steps = kEnsSteps
  const EnsStepArgs *args;            // [member][step]
  const EnsMember *info;              // [member]
  EnsState *state;                    // [member]
  int *abort;                         // set when a wait runs out: every CTA leaves
  unsigned *status;                   // kStatusEnsemble when a wait ran out
  unsigned long long *acc;            // per member: ns its rounds took (acc[m]) and rounds (acc[members + m])
  const int *order;                   // the members in priority order (largest first)
  int *front;                         // in this launch: the first place in `order` whose work is not all taken
  unsigned long long limitNs;         // the longest a CTA waits for work before it gives up
};
// the round's launch: `ctas` CTAs (ensemble_round_ctas(): the device's resident count)
int launch_ensemble_round(const EnsLaunch &L, int ctas, cudaStream_t st);
int ensemble_round_ctas();

struct DiagArgs {
  const float4 *pos;
  const float *q;
  const uint32_t *seats;
  const float4 *forceA, *monoA, *forceB, *monoB;
  const int *ppSlot;
  const float4 *ppForce;
  int cap;
  float4 *diag;
  const float4 *ppAll = nullptr;   // the stencil-split P3M's per-particle pair sums (uniform ppSplit > 0)
};

// per-device kernel attributes (dynamic shared memory limits); call once per
// device before the first launch and never during a stream capture
cudaError_t init_kernels();
// the current device's multiprocessor count, looked up once per device (safe from any thread)
int sm_count();

// kernel launchers (ccs_kernels.cu); all enqueue on `st` and return the
// number of kernels launched.
int launch_fill_u32(uint32_t *p, size_t n, uint32_t v, cudaStream_t st);
// u by value (the kernel's first argument, as for the contact step); recMax, if not null, is zeroed for the
// contact walk that records (SimArgs::walk 1)
int launch_contact_grid(const ccs_uniforms &u, int N, const float4 *pos, uint32_t *seats, uint32_t *hk,
                        uint32_t *seatsOld, const uint32_t *hkOld, unsigned *status, unsigned *recMax,
                        cudaStream_t st);
// warps: CTA width of the contact step, 8 or 4; u by value (the kernel's first argument); every contact-step
// launcher runs the walk a.walk names (0 the walk, 1 the walk and its record, 2 the record's replay)
int launch_simulate(const ccs_uniforms &u, int N, const SimArgs &a, cudaStream_t st, int warps = 8,
                    bool field = false);
// a split mesh step: the contact walk alone (its sums into a.part, a.part2), then, after the mesh and the
// pairwise pass, the tail that turns them and the gravity into the step's outputs
int launch_contacts_only(const ccs_uniforms &u, int N, const SimArgs &a, cudaStream_t st, int warps);
// tide: the stencil-split P3M's gather (second order from each node's centre of mass, the particle's pairs)
int launch_contact_tail(const ccs_uniforms &u, int N, const SimArgs &a, cudaStream_t st, bool tide = false);
// the contact step with its pair sets written out (a.pairs, a.pairCap): the same walk, outputs to a's buffers
int launch_contact_pairs(const ccs_uniforms &u, int N, const SimArgs &a, cudaStream_t st);
// the contact step for particles [first, first + count) only; first a multiple of 256
int launch_simulate_range(const ccs_uniforms &u, int N, SimArgs a, cudaStream_t st, int warps, bool field, int first,
                          int count);
int launch_deposit(const ccs_uniforms *u, int N, int box, const float4 *pos, const float *mat, const float4 *monoPrev,
                   float4 *fine, cudaStream_t st);
int launch_coarse(const MeshBuf &m, cudaStream_t st);
int launch_far(const MeshBuf &m, cudaStream_t st);
// split: threads per fine cell in the cell-gravity sums, 2, 4 or 8
int launch_cell(const ccs_uniforms *u, const MeshBuf &m, cudaStream_t st, int split = 4);
// the stencil-split P3M (S = 1, 2, 3 nodes): the cell pass without the stencil's node pairs, with tides
int launch_cell_tide(const ccs_uniforms *u, int S, const MeshBuf &m, cudaStream_t st);
// ... after the deposit of box `box`: each cell's second moment about its centre of mass (m.fineQ)
int launch_node_moments(const ccs_uniforms *u, int N, int box, const float4 *pos, const float *mat,
                        const MeshBuf &m, cudaStream_t st);
// ... and the pair pass over every particle inside it: sort by (box, base node), then the stencil's pairs;
// out gets each particle's (pull, potential) x Gm
// (work: split_work_bytes(N) of scratch for the pair pass's items and counters)
size_t split_start_ints();
size_t split_work_bytes(int N);
// where the last pass left its two 64-bit counts: pair evaluations one way, and both ways (each once)
const void *split_pair_counts(const void *work);
// symMin: nodes of at least this many particles take their pairs with each other once, both ways (0: never)
int launch_pp_split(const ccs_uniforms *U, int N, int S, const float4 *pos, const float *mat, uint32_t *keys,
                    int32_t *vals, uint32_t *keysTmp, int32_t *valsTmp, uint32_t *hist, int *start, float4 *src,
                    float4 *srcT, int *cells, int *nCells, void *work, float4 *out, int symMin, cudaStream_t st);
int pp_split_launches(int symMin);
int launch_pp_gather(const ccs_uniforms *u, const float4 *pos, const float *mat, const int *index, int cap,
                     float4 *list, float *box, cudaStream_t st);
// the pairwise partials of the P3M pass: 4 quarters x chunks x cap float4
size_t pp_partial_float4s();
int launch_pp_force(const ccs_uniforms *u, const float4 *list, const float *box, int cap, const float2 *tab,
                    float4 *part, float4 *force, cudaStream_t st);
// the same correction over a gathered list of any length n (no cap), the four slices in one: out[s] = Gm x
// (pull, potential) of member s
int launch_pp_list(const ccs_uniforms &u, const float4 *list, const float *box, int n, const float2 *tab,
                   float4 *out, cudaStream_t st);
// the learned P3M pass (ccs_nn.cu): count / scan / fill the pairs inside half
// the cut, the network on the tensor cores, the per-target sums
size_t nn_pp_count_ints();
int launch_pp_nn(const ccs_uniforms *u, const float4 *list, const float *box, int cap, const float2 *tab,
                 const uint8_t *img, int *counts, int *offs, int *total, int2 *pairs, float4 *mesh, float4 *force,
                 unsigned *status, cudaStream_t st);
int launch_nn_sample_state(const ccs_uniforms *u, const float4 *pos, int N, long count, uint32_t seed, float cutG,
                           float4 *D, float4 *S, cudaStream_t st);
cudaError_t init_nn_kernels();
// the network object's engine-facing half: room for count records in its pool,
// then label them and count them in; its operand image; its device
int nn_reserve(ccs_nn *nn, int64_t count, float4 **D, float4 **S, cudaStream_t *st);
int nn_commit(ccs_nn *nn, int64_t count);
const uint8_t *nn_image(const ccs_nn *nn);
int nn_device(const ccs_nn *nn);
int launch_diag(const ccs_uniforms *u, int N, const DiagArgs &a, cudaStream_t st);
int launch_rigid(const ccs_uniforms *u, int N, const float4 *pos, const float4 *vel, const float4 *aux,
                 const float *q, float4 *posO, float4 *velO, float4 *auxO, float *qO, cudaStream_t st);
int launch_permute(int N, const int32_t *perm, const float4 *pos, const float4 *vel, const float4 *aux,
                   const float *q, const float *mat, const float4 *home, float4 *posO, float4 *velO, float4 *auxO,
                   float *qO, float *matO, float4 *homeO, cudaStream_t st);
int launch_morton_keys(int N, const float4 *pos, double cx, double cy, double cz, uint32_t *keys, int32_t *idx,
                       cudaStream_t st);
// stable LSD radix sort of (key, value) pairs on `bits` key bits; tmp buffers
// hold N entries each, hist holds radix_hist_words(N) words
size_t radix_hist_words(int N);
// the builder's overlap relaxation of n points (x, y, z binary32) on the device: ccs_build.cu
int relax_device(int device, float *p, int n, double a, double A, double C, std::string *err);
int launch_radix_sort(int N, int bits, uint32_t *keys, int32_t *vals, uint32_t *keysTmp, int32_t *valsTmp,
                      uint32_t *hist, cudaStream_t st);
int launch_invert_perm(int N, const int32_t *perm, int32_t *into, cudaStream_t st);
int launch_direct_sum(int N, const float4 *pos, const float *mat, double mref, double eps, const int32_t *idx,
                      int nt, double *acc, double *pot, cudaStream_t st);
int launch_books(int N, double mref, const float4 *pos, const float4 *vel, const float *mat, const float4 *diag,
                 double *partial, double *out, int withDiag, cudaStream_t st);
size_t books_partial_doubles(int N);

}  // namespace ccs
