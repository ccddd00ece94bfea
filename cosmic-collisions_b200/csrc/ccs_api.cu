// ccs_api.cu -- the C ABI: the engine of src/nbody.js on the B200.
//
// The handle owns the device state (the reference's textures as flat arrays),
// runs the step schedule of src/nbody.js:551-558 (contact grid every 2nd step,
// mesh + P3M every 8th, gravity as one impulse), the phases (settle, rigid
// approach, kick) and the analysis hand-off.  The contact step and the
// contact grid take a step's uniforms by value, set in their captured graph
// nodes before each replay; the mesh and pairwise kernels read them from
// device memory.  `ccs_steps` replays captured CUDA graphs of whole 8-step
// blocks, whose device uniform slots one memcpy node refreshes each replay,
// and `ccs_step` one step's graph, whose root kernel writes its uniforms on
// a mesh step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "ccs_internal.h"

using namespace ccs;

namespace {

constexpr double kFL = 6.0;
constexpr double kFH = 2.0 * kFL / 64.0;
constexpr double kPPCut = 5.0 * kFH;
constexpr double kSeatSlack = 0.6;
constexpr double kCpIron = 450.0, kCpRock = 1200.0;
constexpr int kRing = 256;        // per-step uniform slots of the direct path
constexpr int kMaxBlock = 16;     // largest meshEvery a captured block supports
constexpr int kTimedKernels = 7;  // simulate, contact grid, deposit, cell, P3M force, contact walk, contact tail

struct GraphKey {
  int boxB, pp, seatCur, cur, meshEvery, ping, field;
  bool operator<(const GraphKey &o) const {
    return std::memcmp(this, &o, sizeof *this) < 0;
  }
};

// a captured node of a kernel whose first argument is the uniforms by value (the contact step, the contact
// grid): every replay sets them; its other arguments stay as captured (the template graph owns their storage)
struct CapturedNode {
  cudaGraphNode_t node = nullptr;
  int nargs = 0, step = 0;   // the kernel's argument count; the step of the graph it belongs to
};
struct UniNode {
  CapturedNode c;
  cudaKernelNodeParams kp = {};
};

struct GraphSlot {
  cudaGraphExec_t exec = nullptr;
  ccs_uniforms *dev = nullptr;   // meshEvery slots on the device
  ccs_uniforms *host = nullptr;  // pinned staging the memcpy node reads at replay
  cudaEvent_t done = nullptr;    // recorded after the last replay
  bool used = false;
  cudaGraph_t graph = nullptr;   // the template, kept for its nodes' arguments
  cudaGraphNode_t put = nullptr; // a step graph's k_put_uniforms node, given each replay's uniforms
  std::vector<UniNode> uni;      // the nodes that take the uniforms by value, in capture order
};

// one step's launches captured as a graph (ccs_step): its schedule, the buffers it reads and writes
struct StepKey {
  int slots, mesh, boxB, pp, nn, seatCur, cur, ping, field, timed, walk;
  bool operator<(const StepKey &o) const {
    return std::memcmp(this, &o, sizeof *this) < 0;
  }
};

}  // namespace

struct ccs_handle {
  int device = 0;
  cudaStream_t st = nullptr;
  std::string err;
  bool built = false;
  ccs_sim sim{};
  ccs_uniforms stat{};                  // setStaticUniforms
  float LA[3] = {0, 0, 0}, LB[3] = {0, 0, 0}, boxB = 0.0f;   // what boxes() last set
  int N = 0, meshEvery = 8;
  // the crater page's field-gravity step (ccs_set_field)
  bool field = false;
  double gField[3] = {0, 0, 0}, frozen = -1, fieldInvM = 1, fieldCpIron = 1;
  // per-step uniform ring (direct launches)
  ccs_uniforms *uniDev = nullptr;
  int uniNext = 0;
  // particle state, double-buffered (sim.src / sim.dst)
  float4 *pos[2] = {}, *vel[2] = {}, *aux[2] = {};
  float *q[2] = {};
  int cur = 0;
  float *mat = nullptr, *matTmp = nullptr;
  float4 *home = nullptr, *homeTmp = nullptr;
  float4 *part = nullptr;   // a split mesh step's contact sums (SimArgs::part, part2)
  float2 *part2 = nullptr;
  // the contact walk's record (SimArgs::rec ...): made by a step that rebuilt the grid, replayed by the next.
  // recValid: the last step made it and nothing has moved or reordered the particles since
  uint32_t *rec = nullptr;
  int *recN = nullptr;
  float4 *recP = nullptr;
  unsigned *recMax = nullptr, *recStats = nullptr;
  int walkMode = 1;   // ccs_set_contact_walk
  bool recValid = false;
  // contact grid: two seat tables used in turn, and the cell each particle went to
  uint32_t *seats[2] = {}, *hk[2] = {};
  int seatCur = 0;
  size_t ncell = 0;
  MeshBuf pm[2];
  // P3M
  int *ppIndex = nullptr, *ppSlot = nullptr;
  float4 *ppList = nullptr, *ppForce = nullptr, *ppPart = nullptr;
  float *ppBox = nullptr;
  float2 *tab = nullptr;
  int ppCount = 0, ppLoose = 0;
  // the stencil-split P3M (ccs_set_pp_split): the stencil S (0: the reference's loose-list pass), the pair
  // pass's sorted sources, start offsets and occupied target nodes, and every particle's pair sum
  int ppSplit = 0;
  int splitSymMin = 16;    // ccs_set_pp_split_sym: nodes this full take their mutual pairs once, both ways
  int *splitStart = nullptr, *splitCells = nullptr, *splitNCells = nullptr;
  unsigned char *splitWork = nullptr;   // the pair pass's items and counters (split_work_bytes)
  float4 *splitSrc = nullptr, *splitSrcT = nullptr, *ppAll = nullptr;
  // the learned form of the P3M pass (borrowed network; pair buffers sized for the list)
  ccs_nn *nn = nullptr;
  int *nnCounts = nullptr, *nnOffs = nullptr, *nnTotal = nullptr;
  int2 *nnPairs = nullptr;
  float4 *nnMesh = nullptr;
  long nnPairCap = 0;
  float4 *diag = nullptr;
  unsigned *status = nullptr;           // kernel status word (kStatus* bits), sticky until the next build
  // Morton sort scratch
  uint32_t *keys = nullptr, *keysTmp = nullptr, *hist = nullptr;
  int32_t *vals = nullptr, *valsTmp = nullptr, *into = nullptr, *permDev = nullptr;
  // asynchronous read-back
  float *stageP = nullptr, *stageV = nullptr, *stageD = nullptr;
  cudaEvent_t readEv = nullptr;
  bool pending = false;
  // books
  double *booksPartial = nullptr, *booksOut = nullptr;
  // the analysis on the device (allocated on first use)
  int *fofParent = nullptr, *fofSize = nullptr, *fofStart = nullptr, *fofEnd = nullptr, *fofCounts = nullptr,
      *fofOffs = nullptr, *fofNDist = nullptr;
  int32_t *fofList = nullptr;
  double *fofPart = nullptr, *fofElastic = nullptr, *fofDist = nullptr;
  unsigned long long *fofTop = nullptr;
  // graphs
  std::map<GraphKey, GraphSlot> graphs;
  std::map<StepKey, GraphSlot> stepGraphs;
  std::vector<CapturedNode> *uniCapture = nullptr;   // while capturing: where by-value launches record their node
  int captureStep = 0;                               // the step of the graph being captured
  bool uniCaptureLost = false;                       // a node that could not be identified
  // ccs_advance_host's read-back of its last step's first half, overlapping the second half's contact step
  cudaStream_t cst = nullptr;
  // a mesh step's grid and pairwise passes, beside its mesh passes (forked from st and joined back)
  cudaStream_t side = nullptr;
  cudaEvent_t forkEv = nullptr, joinEv = nullptr;
  bool inEnsemble = false;   // captured as an ensemble member: its steps are already a parallel branch
  cudaEvent_t halfEv = nullptr, copyEv = nullptr, inEv = nullptr;
  int ping = 0;
  bool useGraphs = true;
  // launch shapes chosen by ccs_autotune: contact-step warps per CTA, cell-gravity threads per cell
  int tuneWarps = 4, tuneSplit = 4;
  // timing of chosen kernels with events on the stream
  int timing = 0;                       // ccs_timing's mask of kernel ids
  int timingEvery = 1;                  // ccs_timing_every: the contact step timed on every n-th launch
  int64_t timingSeq = 0;                // contact-step launches while it is being timed
  std::vector<cudaEvent_t> evPool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> evRecs;
  size_t evNext = 0;
  double tAcc[kTimedKernels] = {};
  int tCount[kTimedKernels] = {};
  int64_t launches = 0;
};

namespace {

#define CUDA_TRY(h, call)                                                                        \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      (h)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                             \
      return CCS_E_CUDA;                                                                         \
    }                                                                                            \
  } while (0)

template <class T>
int dev_alloc(ccs_handle *h, T **p, size_t count) {
  if (*p) { cudaFree(*p); *p = nullptr; }
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * count);
  if (e != cudaSuccess) {
    h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    *p = nullptr;
    return CCS_E_NOMEM;
  }
  return CCS_OK;
}

template <class T>
void dev_free(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

int check_launch(ccs_handle *h) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    h->err = std::string("kernel launch: ") + cudaGetErrorString(e);
    return CCS_E_CUDA;
  }
  return CCS_OK;
}

// the kernels' status word, read where the host synchronises anyway
int check_status(ccs_handle *h) {
  if (!h->status) return CCS_OK;
  unsigned st = 0;
  cudaError_t e = cudaMemcpy(&st, h->status, sizeof st, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    h->err = std::string("status read: ") + cudaGetErrorString(e);
    return CCS_E_CUDA;
  }
  if (st & kStatusGrid) {
    h->err = "contact grid: an insertion gave up after its retry bound (a degenerate pile of particles, "
             "e.g. non-finite positions)";
    return CCS_E_KERNEL;
  }
  if (st & kStatusNN) {
    h->err = "learned P3M pass: a tensor-core wait gave up";
    return CCS_E_KERNEL;
  }
  return CCS_OK;
}

// setStaticUniforms, src/nbody.js:255-336: every per-run value rounded to binary32
void make_static(ccs_handle *h) {
  const ccs_sim &s = h->sim;
  ccs_uniforms &u = h->stat;
  std::memset(&u, 0, sizeof u);
  u.N = s.N;
  u.W = s.W;
  u.G = s.G;
  u.SX = s.G == 128 ? 16 : 8;
  u.GShift = s.G == 128 ? 7 : 6;
  u.SXShift = u.SX == 16 ? 4 : 3;
  u.GMask = u.G - 1;
  u.SXMask = u.SX - 1;
  u.AW = u.SX * u.G;
  u.AH = (u.G / u.SX) * u.G;
  u.invCell = (float)(1.0 / s.cell);
  u.cell = (float)s.cell;
  u.link2 = (float)(s.cell * s.cell);
  u.reach2 = (float)std::pow(s.cell + kSeatSlack * s.a, 2);
  u.touch = (float)(2 * s.a);
  u.K = (float)s.k;
  u.C = (float)s.c;
  u.invM = (float)(1.0 / s.m);
  u.damp = (float)s.damp;
  u.creep = (float)s.creep;
  u.tK = (float)s.tK;
  u.kappa = (float)s.kappa;
  u.cpIron = (float)(kCpIron / kCpRock);
  u.dt = (float)s.dt;
  for (int k = 0; k < 3; ++k) {
    u.spin0[k] = (float)s.spin0[k];
    u.spin1[k] = (float)s.spin1[k];
  }
  u.invH = (float)(1.0 / kFH);
  u.eps2Mesh = (float)(kFH * kFH);
  u.eps2Cell = (float)(0.5 * kFH * kFH);
  u.Gm = (float)s.m;
  u.cut = (float)kPPCut;
  u.a2 = (float)(s.a * s.a);
  u.frozen = -1.0f;
  if (h->field) {   // the crater page's setStaticUniforms, chicxulub.html:700-710
    u.field = 1.0f;
    for (int k = 0; k < 3; ++k) u.gField[k] = (float)h->gField[k];
    u.frozen = h->frozen < 0 ? -1.0f : (float)h->frozen;
    u.invM = (float)h->fieldInvM;
    u.cpIron = (float)h->fieldCpIron;
  }
}

// boxes(), src/nbody.js:342-350
void set_boxes(ccs_handle *h) {
  const ccs_sim &s = h->sim;
  for (int i = 0; i < 2; ++i) {
    const double dt = s.t - s.boxT[i];
    float *L = i ? h->LB : h->LA;
    for (int k = 0; k < 3; ++k) L[k] = (float)(kFL - s.boxCen[i][k] - s.boxVel[i][k] * dt);
  }
  h->boxB = s.boxOn[1] ? 1.0f : 0.0f;
}

// the uniforms of one pass: statics + the boxes as last set + passSim's own
ccs_uniforms pass_uniforms(const ccs_handle *h, int settle, int kick, double gdt) {
  ccs_uniforms u = h->stat;
  std::memcpy(u.LA, h->LA, sizeof u.LA);
  std::memcpy(u.LB, h->LB, sizeof u.LB);
  u.boxB = h->boxB;
  u.settle = settle ? 1.0f : 0.0f;
  u.kick = kick ? 1.0f : 0.0f;
  u.gdt = (float)gdt;
  for (int k = 0; k < 3; ++k) {
    u.bulk0[k] = (float)h->sim.bulk0[k];
    u.bulk1[k] = (float)h->sim.bulk1[k];
    u.cen0[k] = (float)h->sim.cen0[k];
    u.cen1[k] = (float)h->sim.cen1[k];
  }
  u.ppCount = h->ppCount;
  u.ppSplit = h->field ? 0 : h->ppSplit;
  return u;
}

// soften(), src/nbody.js:545-550
void soften(ccs_handle *h) {
  ccs_sim &s = h->sim;
  s.soft = 1;
  s.k *= 0.5;
  s.c *= std::sqrt(0.5);
  s.dt *= std::sqrt(2.0);
  s.damp = std::exp(-s.dt * 12);
  make_static(h);
}

// a ring slot holding u on the device (direct path)
// a pass's uniforms into the next ring slot, as a kernel's by-value argument: in stream order with the
// kernels that read them, with no copy engine, pinned staging or host wait in between
__global__ void k_put_uniforms(const ccs_uniforms u, ccs_uniforms *dst) {
  static_assert(sizeof(ccs_uniforms) % 4 == 0, "uniforms are whole words");
  const uint32_t *s = reinterpret_cast<const uint32_t *>(&u);
  uint32_t *d = reinterpret_cast<uint32_t *>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(ccs_uniforms) / 4); i += blockDim.x) d[i] = s[i];
}

int push_uniforms(ccs_handle *h, const ccs_uniforms &u, const ccs_uniforms **dev) {
  const int slot = h->uniNext;
  h->uniNext = (h->uniNext + 1) % kRing;
  k_put_uniforms<<<1, 128, 0, h->st>>>(u, h->uniDev + slot);
  h->launches += 1;
  *dev = h->uniDev + slot;
  return CCS_OK;
}

// timing brackets around chosen kernels
// whether this launch of `kernel` is timed: its mask bit, and for the contact step every timingEvery-th launch
bool time_this(const ccs_handle *h, int kernel) {
  if (!((h->timing >> kernel) & 1)) return false;
  return kernel != 0 || h->timingEvery <= 1 || h->timingSeq % h->timingEvery == 0;
}

void time_begin(ccs_handle *h, int kernel, cudaEvent_t *b, cudaEvent_t *e) {
  *b = *e = nullptr;
  if (!time_this(h, kernel)) return;
  if (h->evNext + 2 > h->evPool.size()) {
    for (int k = 0; k < 256; ++k) {
      cudaEvent_t ev;
      if (cudaEventCreate(&ev) == cudaSuccess) h->evPool.push_back(ev);
    }
  }
  if (h->evNext + 2 > h->evPool.size()) return;
  *b = h->evPool[h->evNext++];
  *e = h->evPool[h->evNext++];
  cudaEventRecord(*b, h->st);
  h->evRecs.push_back({kernel, {*b, *e}});
}
void time_end(ccs_handle *h, cudaEvent_t e) {
  if (e) cudaEventRecord(e, h->st);
}
void time_collect(ccs_handle *h) {
  if (h->evRecs.empty()) return;
  cudaStreamSynchronize(h->st);
  for (auto &r : h->evRecs) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, r.second.first, r.second.second) == cudaSuccess) {
      h->tAcc[r.first] += ms;
      h->tCount[r.first] += 1;
    }
  }
  h->evRecs.clear();
  h->evNext = 0;
}

// ---- the passes, each enqueued on h->st reading uniforms at U ----

// while a graph is being captured: the node just added (the capture's one sink) takes the uniforms by value
void record_uniform_node(ccs_handle *h, int nargs) {
  if (!h->uniCapture) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(h->st, &cs, nullptr, nullptr, &deps, &nd) == cudaSuccess &&
      cs == cudaStreamCaptureStatusActive && nd == 1)
    h->uniCapture->push_back(CapturedNode{deps[0], nargs, h->captureStep});
  else
    h->uniCaptureLost = true;
}

void pass_slots(ccs_handle *h, const ccs_uniforms &u) {
  const int nxt = h->seatCur ^ 1;
  cudaEvent_t b, e;
  time_begin(h, 1, &b, &e);
  h->launches += launch_contact_grid(u, h->N, h->pos[h->cur], h->seats[nxt], h->hk[nxt], h->seats[h->seatCur],
                                     h->hk[h->seatCur], h->status, h->recMax, h->st);
  record_uniform_node(h, 8);
  time_end(h, e);
  h->seatCur = nxt;
}

void pass_mesh_box(ccs_handle *h, const ccs_uniforms *U, int b) {
  MeshBuf &m = h->pm[b];
  cudaMemsetAsync(m.fine, 0, sizeof(float4) * (kFine + 1), h->st);
  cudaEvent_t eb, ee;
  time_begin(h, 2, &eb, &ee);
  h->launches += launch_deposit(U, h->N, b, h->pos[h->cur], h->mat, m.mono, m.fine, h->st);
  if (h->ppSplit) h->launches += launch_node_moments(U, h->N, b, h->pos[h->cur], h->mat, m, h->st);
  time_end(h, ee);
  cudaMemsetAsync(m.occCount, 0, sizeof(int), h->st);
  h->launches += launch_coarse(m, h->st);
  h->launches += launch_far(m, h->st);
  time_begin(h, 3, &eb, &ee);
  if (h->ppSplit)
    h->launches += launch_cell_tide(U, h->ppSplit, m, h->st);
  else
    h->launches += launch_cell(U, m, h->st, h->tuneSplit);
  time_end(h, ee);
}

void pass_mesh(ccs_handle *h, const ccs_uniforms *U, int boxB) {
  pass_mesh_box(h, U, 0);
  if (boxB) pass_mesh_box(h, U, 1);
}

void pass_pp(ccs_handle *h, const ccs_uniforms *U, int count) {
  if (h->ppSplit) {   // the stencil-split P3M: every particle's pairs inside the stencil
    cudaEvent_t b, e;
    time_begin(h, 4, &b, &e);
    h->launches += launch_pp_split(U, h->N, h->ppSplit, h->pos[h->cur], h->mat, h->keys, h->vals, h->keysTmp,
                                   h->valsTmp, h->hist, h->splitStart, h->splitSrc, h->splitSrcT, h->splitCells,
                                   h->splitNCells, h->splitWork, h->ppAll, h->splitSymMin, h->st);
    time_end(h, e);
    return;
  }
  if (!count) return;
  h->launches += launch_pp_gather(U, h->pos[h->cur], h->mat, h->ppIndex, CCS_PP_CAP, h->ppList, h->ppBox, h->st);
  cudaEvent_t b, e;
  time_begin(h, 4, &b, &e);
  if (h->nn)
    h->launches += launch_pp_nn(U, h->ppList, h->ppBox, CCS_PP_CAP, h->tab, nn_image(h->nn),
                                h->nnCounts, h->nnOffs, h->nnTotal, h->nnPairs, h->nnMesh, h->ppForce, h->status,
                                h->st);
  else
    h->launches += launch_pp_force(U, h->ppList, h->ppBox, CCS_PP_CAP, h->tab, h->ppPart, h->ppForce, h->st);
  time_end(h, e);
}

// the contact step's arguments: state `s` in, the other buffers out
SimArgs sim_args(const ccs_handle *h) {
  const int s = h->cur, d = h->cur ^ 1;
  SimArgs a;
  a.pos = h->pos[s];
  a.vel = h->vel[s];
  a.mat = h->mat;
  a.q = h->q[s];
  a.seats = h->seats[h->seatCur];
  a.forceA = h->pm[0].force;
  a.monoA = h->pm[0].mono;
  a.forceB = h->pm[1].force;
  a.monoB = h->pm[1].mono;
  a.ppSlot = h->ppSlot;
  a.ppForce = h->ppForce;
  a.cap = CCS_PP_CAP;
  a.posO = h->pos[d];
  a.velO = h->vel[d];
  a.auxO = h->aux[d];
  a.qO = h->q[d];
  a.part = h->part;
  a.part2 = h->part2;
  a.tideA0 = h->pm[0].tide0;
  a.tideA1 = h->pm[0].tide1;
  a.tideB0 = h->pm[1].tide0;
  a.tideB1 = h->pm[1].tide1;
  a.tideA2 = h->pm[0].tide2;
  a.tideB2 = h->pm[1].tide2;
  a.fineA = h->pm[0].fine;
  a.fineB = h->pm[1].fine;
  a.ppAll = h->ppAll;
  a.rec = h->rec;
  a.recN = h->recN;
  a.recP = h->recP;
  a.recMax = h->recMax;
  a.recStats = h->walkMode == 2 ? h->recStats : nullptr;
  // The record holds every pair the next step's walk can find while the owner has moved at most mu and
  // every particle at most D since the rebuild, mu + D below the margin by which the cull's reach (cell +
  // SEAT_SLACK a) exceeds the link radius (cell) plus the seat's quantisation (half the diagonal of a
  // fifteenth of a cell), less rounding.  Without that margin nothing is recorded or replayed.
  const double margin = kSeatSlack * h->sim.a - std::sqrt(3.0) / 30.0 * h->sim.cell - 1e-4 * h->sim.cell;
  if (margin > 0.0) {
    const double mu = 0.35 * margin, D = 0.55 * margin;
    a.recLink2 = (float)((h->sim.cell + mu) * (h->sim.cell + mu));
    a.recMove2 = (float)(0.95 * mu * 0.95 * mu);
    a.recAll2 = (float)(0.95 * D * 0.95 * D);
  }
  a.walk = 0;
  return a;
}

// the walk a step's contact step runs (SimArgs::walk): a step that rebuilds the grid records, the next one
// replays what was recorded, while the record is good (ccs_set_contact_walk 1 or 2)
int step_walk(const ccs_handle *h, bool slots) {
  if (!h->walkMode || !h->rec) return 0;
  if (kSeatSlack * h->sim.a - std::sqrt(3.0) / 30.0 * h->sim.cell - 1e-4 * h->sim.cell <= 0.0) return 0;
  return slots ? 1 : (h->recValid ? 2 : 0);
}

void pass_sim(ccs_handle *h, const ccs_uniforms &u, int walk = 0) {
  SimArgs a = sim_args(h);
  a.walk = walk;
  if (h->ppSplit && !h->field && h->part && h->part2) {   // the stencil-split P3M's contact step: walk + tail
    h->launches += launch_contacts_only(u, h->N, a, h->st, h->tuneWarps);
    h->launches += launch_contact_tail(u, h->N, a, h->st, true);
    h->cur ^= 1;
    return;
  }
  cudaEvent_t b, e;
  time_begin(h, 0, &b, &e);
  h->launches += launch_simulate(u, h->N, a, h->st, h->tuneWarps, h->field);
  record_uniform_node(h, 2);
  time_end(h, e);
  if (h->timing & 1) ++h->timingSeq;
  h->cur ^= 1;
}

void pass_diag_kernel(ccs_handle *h, const ccs_uniforms *U) {
  DiagArgs a;
  a.pos = h->pos[h->cur];
  a.q = h->q[h->cur];
  a.seats = h->seats[h->seatCur];
  a.forceA = h->pm[0].force;
  a.monoA = h->pm[0].mono;
  a.forceB = h->pm[1].force;
  a.monoB = h->pm[1].mono;
  a.ppSlot = h->ppSlot;
  a.ppForce = h->ppForce;
  a.cap = CCS_PP_CAP;
  a.diag = h->diag;
  a.ppAll = h->ppAll;
  h->launches += launch_diag(U, h->N, a, h->st);
}

// the step's schedule decided on the host (src/nbody.js:551-558); returns the
// uniforms of this step and what the step runs
struct StepPlan {
  ccs_uniforms u;
  bool slots, mesh;
  int walk;   // SimArgs::walk of its contact step
};
StepPlan plan_step(ccs_handle *h, int settle, int kick) {
  ccs_sim &s = h->sim;
  StepPlan p;
  if (h->field) {   // chicxulub.html:763-766: the grid every 2nd step, the field every step
    const int n = s.stepNo++;
    p.slots = n % 2 == 0;
    p.mesh = false;
    p.u = pass_uniforms(h, settle, kick, s.dt);
    p.walk = step_walk(h, p.slots);
    h->recValid = p.walk == 1;
    return p;
  }
  if (!settle && !kick && !s.soft && s.t - s.impactT > 1.5) soften(h);
  const int n = s.stepNo++;
  p.slots = n % 2 == 0;
  p.mesh = n % h->meshEvery == 0;
  if (p.mesh) set_boxes(h);
  p.u = pass_uniforms(h, settle, kick, p.mesh ? h->meshEvery * s.dt : 0.0);
  p.walk = step_walk(h, p.slots);
  h->recValid = p.walk == 1;
  return p;
}

// the kernels a captured block launches (a block's device uniforms come by one memcpy node, not a kernel;
// a single step's graph adds its uniforms kernel on a mesh step)
int block_launches(const ccs_handle *h, const StepPlan *plans, int M, bool split = false) {
  int per = 0;
  for (int k = 0; k < M; ++k) {
    if (h->ppSplit && !h->field) {                  // the stencil-split P3M: walk + tail every step
      per += 2 + (plans[k].slots ? 1 : 0);
      if (plans[k].mesh) per += 8 * (1 + (plans[k].u.boxB > 0.5f)) + pp_split_launches(h->splitSymMin);
      continue;
    }
    per += 1;                                       // contact step
    if (plans[k].slots) per += 1;                   // contact grid
    if (plans[k].mesh) {
      per += 5 * (1 + (plans[k].u.boxB > 0.5f));    // deposit, coarse, occupied list, far, cell per box
      if (plans[k].u.ppCount) per += h->nn ? 6 : 3; // gather, then pairs + reduce (or the learned pass's five)
      if (split) per += 1;                          // the contact step as its walk and its tail
    }
  }
  return per;
}

// whether a captured mesh step splits its contact step (needs the side stream and the sums buffers; the
// field step has no mesh)
bool can_split(const ccs_handle *h) { return h->side && h->part && h->part2 && !h->field; }

// what a step runs before its contact step: the grid, and the mesh and the pairwise pass on mesh steps.
// The three read the positions and write disjoint buffers, so on a mesh step the grid and the pairwise pass
// run on the side stream beside the mesh chain (deposit, coarse, far, cell), and the contact step waits for
// both.  While kernels are being timed one by one, or when the step is an ensemble member's (the members'
// steps are parallel branches already), they run in order on st.
void enqueue_pre(ccs_handle *h, const StepPlan &p, const ccs_uniforms *U) {
  if (!p.mesh || !h->side || h->timing || h->inEnsemble) {
    if (p.slots) pass_slots(h, p.u);
    if (p.mesh) {
      pass_mesh(h, U, p.u.boxB > 0.5f);
      pass_pp(h, U, p.u.ppCount);
    }
    return;
  }
  cudaEventRecord(h->forkEv, h->st);
  cudaStreamWaitEvent(h->side, h->forkEv, 0);
  const cudaStream_t main = h->st;
  h->st = h->side;
  if (p.slots) pass_slots(h, p.u);
  pass_pp(h, U, p.u.ppCount);
  h->st = main;
  pass_mesh(h, U, p.u.boxB > 0.5f);
  cudaEventRecord(h->joinEv, h->side);
  cudaStreamWaitEvent(h->st, h->joinEv, 0);
}

// one step's launches.  A mesh step splits its contact step: the grid and then the contact walk run on the
// side stream beside the mesh chain and the pairwise pass, which the walk does not read; the particles'
// gravity, settle/kick, heat and kick/drift (the tail) run after both.  Steps whose kernels are timed one
// by one, and ensemble members' steps (parallel branches already), run the contact step whole.
void enqueue_step(ccs_handle *h, const StepPlan &p, const ccs_uniforms *U) {
  if (h->ppSplit && !h->field && h->part && h->part2) {
    // the stencil-split P3M: every step's contact step as its walk and its tail, whose gravity is the
    // second-order gather plus the particle's own pair sum.  On a mesh step the grid and the walk run on the
    // side stream beside the mesh chain and the pair pass (unless kernels are timed or the step is an
    // ensemble member's), as in the reference form's split mesh step.
    const bool fork = p.mesh && h->side && !h->inEnsemble && !h->timing;
    const cudaStream_t main = h->st;
    if (fork) {
      cudaEventRecord(h->forkEv, h->st);
      cudaStreamWaitEvent(h->side, h->forkEv, 0);
      h->st = h->side;
    }
    if (p.slots) pass_slots(h, p.u);
    SimArgs a = sim_args(h);
    a.walk = p.walk;
    cudaEvent_t b, e;
    time_begin(h, 5, &b, &e);
    h->launches += launch_contacts_only(p.u, h->N, a, h->st, h->tuneWarps);
    record_uniform_node(h, 2);
    time_end(h, e);
    h->st = main;
    if (p.mesh) {
      pass_mesh(h, U, p.u.boxB > 0.5f);
      pass_pp(h, U, p.u.ppCount);
    }
    if (fork) {
      cudaEventRecord(h->joinEv, h->side);
      cudaStreamWaitEvent(h->st, h->joinEv, 0);
    }
    time_begin(h, 6, &b, &e);
    h->launches += launch_contact_tail(p.u, h->N, a, h->st, true);
    record_uniform_node(h, 2);
    time_end(h, e);
    h->cur ^= 1;
    return;
  }
  if (p.mesh && can_split(h) && !h->inEnsemble && (h->timing & (3 << 5))) {
    // the split mesh step with its two halves timed (kernel ids 5 and 6): everything in order on st, so
    // each half sits alone between its events
    if (p.slots) pass_slots(h, p.u);
    SimArgs a = sim_args(h);
    a.walk = p.walk;
    cudaEvent_t b, e;
    time_begin(h, 5, &b, &e);
    h->launches += launch_contacts_only(p.u, h->N, a, h->st, h->tuneWarps);
    time_end(h, e);
    pass_mesh(h, U, p.u.boxB > 0.5f);
    pass_pp(h, U, p.u.ppCount);
    time_begin(h, 6, &b, &e);
    h->launches += launch_contact_tail(p.u, h->N, a, h->st);
    time_end(h, e);
    h->cur ^= 1;
    return;
  }
  if (!p.mesh || !can_split(h) || h->timing || h->inEnsemble) {
    enqueue_pre(h, p, U);
    pass_sim(h, p.u, p.walk);
    return;
  }
  cudaEventRecord(h->forkEv, h->st);
  cudaStreamWaitEvent(h->side, h->forkEv, 0);
  const cudaStream_t main = h->st;
  h->st = h->side;
  if (p.slots) pass_slots(h, p.u);
  SimArgs a = sim_args(h);   // the table the grid has just filled
  a.walk = p.walk;
  h->launches += launch_contacts_only(p.u, h->N, a, h->st, h->tuneWarps);
  record_uniform_node(h, 2);
  h->st = main;
  pass_mesh(h, U, p.u.boxB > 0.5f);
  pass_pp(h, U, p.u.ppCount);
  cudaEventRecord(h->joinEv, h->side);
  cudaStreamWaitEvent(h->st, h->joinEv, 0);
  h->launches += launch_contact_tail(p.u, h->N, a, h->st);
  record_uniform_node(h, 2);
  h->cur ^= 1;
}

// after a capture: the contact-step nodes it recorded, with their captured arguments
int resolve_uniform_nodes(ccs_handle *h, const std::vector<CapturedNode> &nodes, std::vector<UniNode> &out) {
  if (h->uniCaptureLost) {
    h->uniCaptureLost = false;
    h->err = "graph capture: a node taking the uniforms was not identified";
    return CCS_E_CUDA;
  }
  out.resize(nodes.size());
  for (size_t i = 0; i < nodes.size(); ++i) {
    out[i].c = nodes[i];
    CUDA_TRY(h, cudaGraphKernelNodeGetParams(nodes[i].node, &out[i].kp));
  }
  return CCS_OK;
}

// a node of an instantiated graph given this replay's uniforms (replays already enqueued keep theirs)
int set_node_uniforms(ccs_handle *h, cudaGraphExec_t exec, const UniNode &n, const ccs_uniforms &u) {
  constexpr int kMaxArgs = 8;
  if (n.c.nargs < 1 || n.c.nargs > kMaxArgs) return CCS_E_STATE;
  ccs_uniforms v = u;
  void *args[kMaxArgs];
  args[0] = &v;
  for (int i = 1; i < n.c.nargs; ++i) args[i] = n.kp.kernelParams[i];
  cudaKernelNodeParams kp = n.kp;
  kp.kernelParams = args;
  kp.extra = nullptr;
  CUDA_TRY(h, cudaGraphExecKernelNodeSetParams(exec, n.c.node, &kp));
  return CCS_OK;
}

void free_graph_slot(GraphSlot &g);

// one step replayed from a captured graph, so a step costs one cudaGraphLaunch.  The contact step and the
// contact grid take the step's uniforms as their by-value first argument, set in their nodes before each
// replay; the mesh and pairwise kernels read them from device memory, written on a mesh step by the
// graph's root node, k_put_uniforms, whose by-value argument is set the same way (no copy engine or
// pinned staging on the step's path).  Graphs are keyed by what the step runs and by the buffers it
// touches.  When the contact step is being timed (ccs_timing bit 0), or its caller launches it
// (simOutside), the graph stops before it and the contact step is launched directly, between its two
// events when timed (events recorded by a graph's nodes do not time).
int step_graph(ccs_handle *h, const StepPlan &p, bool simOutside = false) {
  const bool timed = (time_this(h, 0) && !h->ppSplit) || simOutside;
  const bool pre = p.mesh;   // kernels that read the uniforms from device memory (the mesh and pairwise passes)
  if (timed && !p.slots && !p.mesh) {   // nothing to replay: the contact step alone, launched directly
    if (!simOutside) pass_sim(h, p.u, p.walk);
    return check_launch(h);
  }
  const StepKey key{(int)p.slots, (int)p.mesh, (int)(p.u.boxB > 0.5f), h->ppCount > 0, h->nn != nullptr,
                    h->seatCur, h->cur, h->ping, (int)h->field, (int)timed, p.walk};
  GraphSlot &g = h->stepGraphs[key];
  const int seatCur0 = h->seatCur, cur0 = h->cur;
  if (!g.exec) {
    if (pre && !g.dev) CUDA_TRY(h, cudaMalloc(&g.dev, sizeof(ccs_uniforms)));
    if (!g.done) CUDA_TRY(h, cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
    const int timing = h->timing;
    const int64_t l0 = h->launches;
    cudaGraph_t graph;
    std::vector<CapturedNode> uniNodes;
    CUDA_TRY(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    h->timing = 0;
    h->uniCapture = &uniNodes;
    h->captureStep = 0;
    if (pre) k_put_uniforms<<<1, 128, 0, h->st>>>(p.u, g.dev);   // the graph's root
    if (timed) enqueue_pre(h, p, g.dev);
    else enqueue_step(h, p, g.dev);
    h->uniCapture = nullptr;
    cudaError_t ce = cudaStreamEndCapture(h->st, &graph);
    h->timing = timing;
    h->launches = l0;
    h->seatCur = seatCur0;
    h->cur = cur0;
    if (ce != cudaSuccess) {
      h->uniCaptureLost = false;
      h->err = std::string("step graph capture: ") + cudaGetErrorString(ce);
      return CCS_E_CUDA;
    }
    g.put = nullptr;
    if (pre) {
      size_t roots = 1;
      ce = cudaGraphGetRootNodes(graph, &g.put, &roots);
      if (ce == cudaSuccess && roots != 1) ce = cudaErrorInvalidValue;
    }
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&g.exec, graph, 0);
    if (ce != cudaSuccess) {
      cudaGraphDestroy(graph);
      h->uniCaptureLost = false;
      h->err = std::string("step graph instantiate: ") + cudaGetErrorString(ce);
      g.exec = nullptr;
      return CCS_E_CUDA;
    }
    g.graph = graph;
    int rc = resolve_uniform_nodes(h, uniNodes, g.uni);
    if (rc) {
      free_graph_slot(g);
      h->stepGraphs.erase(key);
      return rc;
    }
  } else {
    // this replay's uniforms into the root node's argument, the grid's and the contact step's
    if (g.put) {
      ccs_uniforms u = p.u;
      ccs_uniforms *dst = g.dev;
      void *args[] = {&u, &dst};
      cudaKernelNodeParams kp = {};
      kp.func = reinterpret_cast<void *>(k_put_uniforms);
      kp.gridDim = dim3(1);
      kp.blockDim = dim3(128);
      kp.kernelParams = args;
      CUDA_TRY(h, cudaGraphExecKernelNodeSetParams(g.exec, g.put, &kp));
    }
    for (const UniNode &n : g.uni) {
      const int rc = set_node_uniforms(h, g.exec, n, p.u);
      if (rc) return rc;
    }
  }
  CUDA_TRY(h, cudaGraphLaunch(g.exec, h->st));
  h->seatCur = seatCur0 ^ (p.slots ? 1 : 0);
  h->launches += block_launches(h, &p, 1, !timed && can_split(h)) + (pre ? 1 : 0);   // and the uniforms node
  if (simOutside) {
    --h->launches;            // the caller launches the contact step
  } else if (timed) {
    --h->launches;            // pass_sim counts its own
    pass_sim(h, p.u, p.walk);
  } else {
    h->cur = cur0 ^ 1;
    if (h->timing & 1) ++h->timingSeq;   // a contact step that was not this sample's
  }
  CUDA_TRY(h, cudaEventRecord(g.done, h->st));
  g.used = true;
  h->ping ^= 1;
  return check_launch(h);
}

int do_step(ccs_handle *h, int settle, int kick) {
  StepPlan p = plan_step(h, settle, kick);
  if (h->useGraphs && (h->timing & ~1) == 0) return step_graph(h, p);   // timing beyond the contact step: direct
  const ccs_uniforms *U;
  int rc = push_uniforms(h, p.u, &U);
  if (rc) return rc;
  enqueue_step(h, p, U);
  return check_launch(h);
}

void free_graph_slot(GraphSlot &g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  if (g.dev) cudaFree(g.dev);
  if (g.host) cudaFreeHost(g.host);
  if (g.done) cudaEventDestroy(g.done);
}

void free_graphs(ccs_handle *h) {
  for (auto &kv : h->graphs) free_graph_slot(kv.second);
  h->graphs.clear();
  for (auto &kv : h->stepGraphs) free_graph_slot(kv.second);
  h->stepGraphs.clear();
}

// one block of meshEvery frame-loop steps, starting at stepNo % meshEvery == 0,
// replayed from a captured graph
int graph_block(ccs_handle *h) {
  const int M = h->meshEvery;
  GraphKey key{(int)(h->boxB > 0.5f), h->ppCount > 0, h->seatCur, h->cur, M, h->ping, (int)h->field};
  // plan the block's steps on the host (the boxes are set at its first step)
  ccs_uniforms us[kMaxBlock];
  StepPlan plans[kMaxBlock];
  for (int k = 0; k < M; ++k) {
    plans[k] = plan_step(h, 0, 0);
    us[k] = plans[k].u;
    h->sim.t += h->sim.dt;   // the frame loop's clock, index.html:372
  }
  key.boxB = (int)(us[0].boxB > 0.5f);
  GraphSlot &g = h->graphs[key];
  const int seatCur0 = h->seatCur, cur0 = h->cur;
  if (!g.exec) {
    CUDA_TRY(h, cudaMalloc(&g.dev, sizeof(ccs_uniforms) * M));
    CUDA_TRY(h, cudaMallocHost(&g.host, sizeof(ccs_uniforms) * M));
    CUDA_TRY(h, cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
    std::memcpy(g.host, us, sizeof(ccs_uniforms) * M);
    cudaGraph_t graph;
    const int timing = h->timing;
    const int64_t l0 = h->launches;
    std::vector<CapturedNode> uniNodes;
    CUDA_TRY(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    h->timing = 0;
    h->uniCapture = &uniNodes;
    cudaMemcpyAsync(g.dev, g.host, sizeof(ccs_uniforms) * M, cudaMemcpyHostToDevice, h->st);
    for (int k = 0; k < M; ++k) {
      h->captureStep = k;
      enqueue_step(h, plans[k], g.dev + k);
    }
    h->uniCapture = nullptr;
    cudaError_t ce = cudaStreamEndCapture(h->st, &graph);
    h->timing = timing;
    h->launches = l0;
    // capture ran the buffer rotation once on the host; restore it for the replay
    h->seatCur = seatCur0;
    h->cur = cur0;
    if (ce != cudaSuccess) {
      h->uniCaptureLost = false;
      h->err = std::string("graph capture: ") + cudaGetErrorString(ce);
      free_graph_slot(g);
      h->graphs.erase(key);
      return CCS_E_CUDA;
    }
    ce = cudaGraphInstantiate(&g.exec, graph, 0);
    if (ce != cudaSuccess) {
      cudaGraphDestroy(graph);
      h->uniCaptureLost = false;
      h->err = std::string("graph instantiate: ") + cudaGetErrorString(ce);
      g.exec = nullptr;
      free_graph_slot(g);
      h->graphs.erase(key);
      return CCS_E_CUDA;
    }
    g.graph = graph;
    int rc = resolve_uniform_nodes(h, uniNodes, g.uni);
    int want = M;
    for (int k = 0; k < M; ++k)
      want += (plans[k].slots ? 1 : 0) +
              (h->ppSplit && !h->field ? 1 : (plans[k].mesh && can_split(h) ? 1 : 0));
    if (rc == CCS_OK && (int)g.uni.size() != want) {
      h->err = "graph capture: a contact-step node per step and a grid node per even step expected";
      rc = CCS_E_CUDA;
    }
    if (rc) {
      free_graph_slot(g);
      h->graphs.erase(key);
      return rc;
    }
  } else {
    for (const UniNode &n : g.uni) {   // each step's uniforms into its grid's and contact step's argument
      const int rc = set_node_uniforms(h, g.exec, n, us[n.c.step]);
      if (rc) return rc;
    }
  }
  if (g.used) CUDA_TRY(h, cudaEventSynchronize(g.done));
  std::memcpy(g.host, us, sizeof(ccs_uniforms) * M);
  CUDA_TRY(h, cudaGraphLaunch(g.exec, h->st));
  CUDA_TRY(h, cudaEventRecord(g.done, h->st));
  g.used = true;
  h->ping ^= 1;
  // a block does 4 grid rebuilds (the table parity returns) and M swaps
  h->cur = cur0 ^ (M & 1);
  h->seatCur = seatCur0 ^ (((M + 1) / 2) & 1);
  h->launches += block_launches(h, plans, M, can_split(h));
  return CCS_OK;
}

int ensure_built(ccs_handle *h) {
  if (!h || !h->built) {
    if (h) h->err = "no run built (ccs_build)";
    return CCS_E_STATE;
  }
  return CCS_OK;
}

// pair buffers of the learned pass, sized for the worst case of an n-entry list (every pair inside the cut)
int ensure_nn_buffers(ccs_handle *h, int n) {
  if (!h->nn) return CCS_OK;
  int rc = CCS_OK;
  if (!h->nnCounts) {
    free_graphs(h);
    rc |= dev_alloc(h, &h->nnCounts, nn_pp_count_ints());
    rc |= dev_alloc(h, &h->nnOffs, nn_pp_count_ints());
    rc |= dev_alloc(h, &h->nnTotal, 1);
    if (rc) return CCS_E_NOMEM;
  }
  const long need = std::max<long>(1, (long)n * (long)(n - 1));
  if (need > h->nnPairCap) {
    free_graphs(h);   // captured launches hold the old pointers
    rc |= dev_alloc(h, &h->nnPairs, (size_t)need);
    rc |= dev_alloc(h, &h->nnMesh, (size_t)need);
    if (rc) {
      h->nnPairCap = 0;
      return CCS_E_NOMEM;
    }
    h->nnPairCap = need;
  }
  return CCS_OK;
}

// the stencil-split P3M's buffers: each box's tides and tide partials, the pair pass's sort and sums
int ensure_split_buffers(ccs_handle *h) {
  if (h->ppAll) return CCS_OK;
  const size_t N = (size_t)h->N;
  int rc = 0;
  for (int b = 0; b < 2; ++b) {
    MeshBuf &m = h->pm[b];
    rc |= dev_alloc(h, &m.tide0, kFine + 1);
    rc |= dev_alloc(h, &m.tide1, kFine + 1);
    rc |= dev_alloc(h, &m.tide2, 3 * (size_t)(kFine + 1));
    rc |= dev_alloc(h, &m.fineQ, 2 * (size_t)(kFine + 1));
    rc |= dev_alloc(h, &m.cellPartT, (size_t)kCoarse * kCellChunks * 64 * 5);
    rc |= dev_alloc(h, &m.quad0, kCoarse);
    rc |= dev_alloc(h, &m.quad1, kCoarse);
  }
  rc |= dev_alloc(h, &h->splitStart, split_start_ints());
  rc |= dev_alloc(h, &h->splitCells, N);
  rc |= dev_alloc(h, &h->splitNCells, 1);
  rc |= dev_alloc(h, &h->splitWork, split_work_bytes(h->N));
  rc |= dev_alloc(h, &h->splitSrc, N);
  rc |= dev_alloc(h, &h->splitSrcT, N);
  rc |= dev_alloc(h, &h->ppAll, N);
  if (rc) {
    for (int b = 0; b < 2; ++b) {
      dev_free(h->pm[b].tide0); dev_free(h->pm[b].tide1); dev_free(h->pm[b].cellPartT);
      dev_free(h->pm[b].quad0); dev_free(h->pm[b].quad1); dev_free(h->pm[b].tide2); dev_free(h->pm[b].fineQ);
    }
    dev_free(h->splitStart); dev_free(h->splitCells); dev_free(h->splitNCells); dev_free(h->splitSrc);
    dev_free(h->splitSrcT); dev_free(h->ppAll); dev_free(h->splitWork);
    return CCS_E_NOMEM;
  }
  for (int b = 0; b < 2; ++b) {
    CUDA_TRY(h, cudaMemsetAsync(h->pm[b].tide0, 0, sizeof(float4) * (kFine + 1), h->st));
    CUDA_TRY(h, cudaMemsetAsync(h->pm[b].tide1, 0, sizeof(float4) * (kFine + 1), h->st));
    CUDA_TRY(h, cudaMemsetAsync(h->pm[b].tide2, 0, sizeof(float4) * 3 * (kFine + 1), h->st));
  }
  CUDA_TRY(h, cudaMemsetAsync(h->ppAll, 0, sizeof(float4) * N, h->st));
  CUDA_TRY(h, cudaMemsetAsync(h->splitWork, 0, split_work_bytes(h->N), h->st));   // no pass counted yet
  return CCS_OK;
}

void free_state(ccs_handle *h) {
  free_graphs(h);
  for (int b = 0; b < 2; ++b) {
    dev_free(h->pos[b]); dev_free(h->vel[b]); dev_free(h->aux[b]); dev_free(h->q[b]);
    dev_free(h->seats[b]); dev_free(h->hk[b]);
    MeshBuf &m = h->pm[b];
    dev_free(m.fine); dev_free(m.force); dev_free(m.coarse); dev_free(m.farA); dev_free(m.farT0);
    dev_free(m.farT1); dev_free(m.mono); dev_free(m.partial); dev_free(m.counter);
    dev_free(m.occ); dev_free(m.occIdx); dev_free(m.occN); dev_free(m.occBlocks); dev_free(m.occCount);
    dev_free(m.occAsc); dev_free(m.occAscN); dev_free(m.cellPart); dev_free(m.cellDone);
    dev_free(m.tide0); dev_free(m.tide1); dev_free(m.cellPartT); dev_free(m.quad0); dev_free(m.quad1);
    dev_free(m.tide2); dev_free(m.fineQ);
  }
  dev_free(h->splitStart); dev_free(h->splitCells); dev_free(h->splitNCells); dev_free(h->splitSrc);
  dev_free(h->splitSrcT); dev_free(h->ppAll); dev_free(h->splitWork);
  dev_free(h->mat); dev_free(h->matTmp); dev_free(h->home); dev_free(h->homeTmp);
  dev_free(h->part); dev_free(h->part2);
  dev_free(h->rec); dev_free(h->recN); dev_free(h->recP); dev_free(h->recMax); dev_free(h->recStats);
  h->recValid = false;
  dev_free(h->ppIndex); dev_free(h->ppSlot); dev_free(h->ppList); dev_free(h->ppForce); dev_free(h->ppBox);
  dev_free(h->ppPart);
  dev_free(h->nnCounts); dev_free(h->nnOffs); dev_free(h->nnTotal); dev_free(h->nnPairs); dev_free(h->nnMesh);
  h->nnPairCap = 0;
  dev_free(h->tab); dev_free(h->diag);
  dev_free(h->keys); dev_free(h->keysTmp); dev_free(h->hist); dev_free(h->vals); dev_free(h->valsTmp);
  dev_free(h->into); dev_free(h->permDev);
  dev_free(h->fofParent); dev_free(h->fofSize); dev_free(h->fofStart); dev_free(h->fofEnd); dev_free(h->fofCounts);
  dev_free(h->fofOffs); dev_free(h->fofNDist); dev_free(h->fofList); dev_free(h->fofPart); dev_free(h->fofElastic);
  dev_free(h->fofDist); dev_free(h->fofTop);
  dev_free(h->booksPartial); dev_free(h->booksOut); dev_free(h->status);
  if (h->stageP) cudaFreeHost(h->stageP);
  if (h->stageV) cudaFreeHost(h->stageV);
  if (h->stageD) cudaFreeHost(h->stageD);
  h->stageP = h->stageV = h->stageD = nullptr;
  h->built = false;
  h->pending = false;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int ccs_version(void) { return 1; }

const char *ccs_last_error(const ccs_handle *h) { return h ? h->err.c_str() : "null handle"; }

int ccs_create(int device, ccs_handle **out) {
  if (!out) return CCS_E_ARG;
  *out = nullptr;
  ccs_handle *h = new (std::nothrow) ccs_handle();
  if (!h) return CCS_E_NOMEM;
  h->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return CCS_E_CUDA;
  }
  if (cudaMalloc(&h->uniDev, sizeof(ccs_uniforms) * kRing) != cudaSuccess) {
    cudaStreamDestroy(h->st);
    delete h;
    return CCS_E_NOMEM;
  }
  if (init_kernels() != cudaSuccess) {
    h->err = "kernel attributes could not be set";
  }
  cudaEventCreateWithFlags(&h->readEv, cudaEventDisableTiming);
  // without them a mesh step's passes run one after another on st
  if (cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->forkEv, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->joinEv, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (h->side) cudaStreamDestroy(h->side);
    if (h->forkEv) cudaEventDestroy(h->forkEv);
    h->side = nullptr;
    h->forkEv = nullptr;
    h->joinEv = nullptr;
  }
  *out = h;
  return CCS_OK;
}

int ccs_destroy(ccs_handle *h) {
  if (!h) return CCS_E_ARG;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->st);
  free_state(h);
  for (auto ev : h->evPool) cudaEventDestroy(ev);
  if (h->readEv) cudaEventDestroy(h->readEv);
  if (h->halfEv) cudaEventDestroy(h->halfEv);
  if (h->copyEv) cudaEventDestroy(h->copyEv);
  if (h->inEv) cudaEventDestroy(h->inEv);
  if (h->cst) cudaStreamDestroy(h->cst);
  if (h->forkEv) cudaEventDestroy(h->forkEv);
  if (h->joinEv) cudaEventDestroy(h->joinEv);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->uniDev) cudaFree(h->uniDev);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return CCS_OK;
}

int ccs_build(ccs_handle *h, const ccs_sim *sim, const float *pos4, const float *vel4, const float *mat,
              const float *home4) {
  if (!h || !sim || !pos4 || !vel4 || !mat) return CCS_E_ARG;
  if (sim->N <= 0 || sim->N > CCS_MAX_N) {
    h->err = "N must be in 1..262144 (the 18-bit seat index)";
    return CCS_E_RANGE;
  }
  if (sim->G != 64 && sim->G != 128) {
    h->err = "G must be 64 or 128";
    return CCS_E_ARG;
  }
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->st);
  free_state(h);
  h->sim = *sim;
  h->N = sim->N;
  const size_t N = (size_t)h->N;
  int rc = 0;
  for (int b = 0; b < 2; ++b) {
    rc |= dev_alloc(h, &h->pos[b], N); rc |= dev_alloc(h, &h->vel[b], N);
    rc |= dev_alloc(h, &h->aux[b], N); rc |= dev_alloc(h, &h->q[b], N);
  }
  rc |= dev_alloc(h, &h->mat, N); rc |= dev_alloc(h, &h->matTmp, N);
  rc |= dev_alloc(h, &h->home, N); rc |= dev_alloc(h, &h->homeTmp, N);
  rc |= dev_alloc(h, &h->part, N); rc |= dev_alloc(h, &h->part2, N);
  // recN: a count for every warp of the contact step's last CTA (up to 8 warps of 32), also the warps wholly
  // past N, which write (and read) a count of nothing
  rc |= dev_alloc(h, &h->rec, (N + 31) / 32 * kRecWarp); rc |= dev_alloc(h, &h->recN, (N + 255) / 256 * 8);
  if (h->recN) cudaMemset(h->recN, 0, sizeof(int) * ((N + 255) / 256 * 8));   // no warp has a record yet
  rc |= dev_alloc(h, &h->recP, N);
  rc |= dev_alloc(h, &h->recMax, 1); rc |= dev_alloc(h, &h->recStats, 3);
  make_static(h);
  h->ncell = (size_t)h->stat.AW * (size_t)h->stat.AH;
  for (int b = 0; b < 2; ++b) {
    rc |= dev_alloc(h, &h->seats[b], h->ncell * kSeats);
    rc |= dev_alloc(h, &h->hk[b], N);
    MeshBuf &m = h->pm[b];
    rc |= dev_alloc(h, &m.fine, kFine + 1); rc |= dev_alloc(h, &m.force, kFine + 1);
    rc |= dev_alloc(h, &m.coarse, kCoarse); rc |= dev_alloc(h, &m.farA, kCoarse);
    rc |= dev_alloc(h, &m.farT0, kCoarse); rc |= dev_alloc(h, &m.farT1, kCoarse);
    rc |= dev_alloc(h, &m.mono, 1); rc |= dev_alloc(h, &m.partial, kCoarse); rc |= dev_alloc(h, &m.counter, 1);
    rc |= dev_alloc(h, &m.occ, (size_t)kCoarse * 64); rc |= dev_alloc(h, &m.occIdx, (size_t)kCoarse * 64);
    rc |= dev_alloc(h, &m.occN, kCoarse);
    rc |= dev_alloc(h, &m.occBlocks, kCoarse); rc |= dev_alloc(h, &m.occCount, 1);
    rc |= dev_alloc(h, &m.occAsc, kCoarse); rc |= dev_alloc(h, &m.occAscN, 1);
    rc |= dev_alloc(h, &m.cellPart, (size_t)kCoarse * kCellChunks * 64); rc |= dev_alloc(h, &m.cellDone, kCoarse);
  }
  rc |= dev_alloc(h, &h->ppIndex, CCS_PP_CAP); rc |= dev_alloc(h, &h->ppSlot, N);
  rc |= dev_alloc(h, &h->ppList, CCS_PP_CAP); rc |= dev_alloc(h, &h->ppForce, 4 * CCS_PP_CAP);
  rc |= dev_alloc(h, &h->ppBox, CCS_PP_CAP); rc |= dev_alloc(h, &h->tab, CCS_PP_BINS);
  rc |= dev_alloc(h, &h->ppPart, pp_partial_float4s());
  rc |= dev_alloc(h, &h->diag, N);
  rc |= dev_alloc(h, &h->keys, N); rc |= dev_alloc(h, &h->keysTmp, N); rc |= dev_alloc(h, &h->vals, N);
  rc |= dev_alloc(h, &h->valsTmp, N); rc |= dev_alloc(h, &h->into, N); rc |= dev_alloc(h, &h->permDev, N);
  rc |= dev_alloc(h, &h->hist, radix_hist_words(h->N));
  rc |= dev_alloc(h, &h->booksPartial, books_partial_doubles(h->N));
  rc |= dev_alloc(h, &h->booksOut, CCS_BOOKS);
  rc |= dev_alloc(h, &h->status, 1);
  if (rc) { free_state(h); return CCS_E_NOMEM; }
  if (cudaMallocHost(&h->stageP, 16 * N) != cudaSuccess || cudaMallocHost(&h->stageV, 16 * N) != cudaSuccess ||
      cudaMallocHost(&h->stageD, 16 * N) != cudaSuccess) {
    free_state(h);
    h->err = "pinned staging allocation failed";
    return CCS_E_NOMEM;
  }
  cudaStream_t st = h->st;
  CUDA_TRY(h, cudaMemcpyAsync(h->pos[0], pos4, 16 * N, cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaMemcpyAsync(h->vel[0], vel4, 16 * N, cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaMemcpyAsync(h->mat, mat, 4 * N, cudaMemcpyHostToDevice, st));
  if (home4) CUDA_TRY(h, cudaMemcpyAsync(h->home, home4, 16 * N, cudaMemcpyHostToDevice, st));
  else CUDA_TRY(h, cudaMemsetAsync(h->home, 0, 16 * N, st));
  for (int b = 0; b < 2; ++b) {
    CUDA_TRY(h, cudaMemsetAsync(h->aux[b], 0, 16 * N, st));
    CUDA_TRY(h, cudaMemsetAsync(h->q[b], 0, 4 * N, st));
    if (b) {
      CUDA_TRY(h, cudaMemsetAsync(h->pos[b], 0, 16 * N, st));
      CUDA_TRY(h, cudaMemsetAsync(h->vel[b], 0, 16 * N, st));
    }
    h->launches += launch_fill_u32(h->seats[b], h->ncell * kSeats, kEmpty, st);
    h->launches += launch_fill_u32(h->hk[b], N, kNoCell, st);
    MeshBuf &m = h->pm[b];
    CUDA_TRY(h, cudaMemsetAsync(m.fine, 0, sizeof(float4) * (kFine + 1), st));
    CUDA_TRY(h, cudaMemsetAsync(m.force, 0, sizeof(float4) * (kFine + 1), st));
    CUDA_TRY(h, cudaMemsetAsync(m.coarse, 0, sizeof(float4) * kCoarse, st));
    CUDA_TRY(h, cudaMemsetAsync(m.farA, 0, sizeof(float4) * kCoarse, st));
    CUDA_TRY(h, cudaMemsetAsync(m.farT0, 0, sizeof(float4) * kCoarse, st));
    CUDA_TRY(h, cudaMemsetAsync(m.farT1, 0, sizeof(float4) * kCoarse, st));
    CUDA_TRY(h, cudaMemsetAsync(m.mono, 0, sizeof(float4), st));
    CUDA_TRY(h, cudaMemsetAsync(m.counter, 0, sizeof(unsigned), st));
    CUDA_TRY(h, cudaMemsetAsync(m.occN, 0, sizeof(int) * kCoarse, st));
    CUDA_TRY(h, cudaMemsetAsync(m.occCount, 0, sizeof(int), st));
    CUDA_TRY(h, cudaMemsetAsync(m.occAscN, 0, sizeof(int), st));
    CUDA_TRY(h, cudaMemsetAsync(m.cellDone, 0, sizeof(int) * kCoarse, st));
    CUDA_TRY(h, cudaMemsetAsync(m.force, 0, sizeof(float4) * (kFine + 1), st));
  }
  h->launches += launch_fill_u32((uint32_t *)h->ppIndex, CCS_PP_CAP, 0xFFFFFFFFu, st);
  h->launches += launch_fill_u32((uint32_t *)h->ppSlot, N, 0xFFFFFFFFu, st);
  CUDA_TRY(h, cudaMemsetAsync(h->ppList, 0, sizeof(float4) * CCS_PP_CAP, st));
  CUDA_TRY(h, cudaMemsetAsync(h->ppForce, 0, sizeof(float4) * 4 * CCS_PP_CAP, st));
  CUDA_TRY(h, cudaMemsetAsync(h->ppBox, 0, sizeof(float) * CCS_PP_CAP, st));
  CUDA_TRY(h, cudaMemsetAsync(h->booksPartial, 0, sizeof(double) * books_partial_doubles(h->N), st));
  CUDA_TRY(h, cudaMemsetAsync(h->status, 0, sizeof(unsigned), st));
  CUDA_TRY(h, cudaMemsetAsync(h->recMax, 0xFF, sizeof(unsigned), st));   // no record yet (a NaN: replay nothing)
  CUDA_TRY(h, cudaMemsetAsync(h->recStats, 0, 3 * sizeof(unsigned), st));
  h->recValid = false;
  float f[CCS_PP_BINS], p[CCS_PP_BINS];
  ccs_pair_table(CCS_PP_BINS, kPPCut, f, p);
  float2 tab[CCS_PP_BINS];
  for (int k = 0; k < CCS_PP_BINS; ++k) tab[k] = make_float2(f[k], p[k]);
  CUDA_TRY(h, cudaMemcpyAsync(h->tab, tab, sizeof tab, cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  h->cur = 0;
  h->seatCur = 0;
  h->ppCount = h->ppLoose = 0;
  h->LA[0] = h->LA[1] = h->LA[2] = 0;
  h->LB[0] = h->LB[1] = h->LB[2] = 0;
  h->boxB = 0;
  h->built = true;
  if (h->ppSplit) {
    rc = ensure_split_buffers(h);
    if (rc) return rc;
    CUDA_TRY(h, cudaStreamSynchronize(st));
  }
  return check_launch(h);
}

ccs_sim *ccs_sim_ptr(ccs_handle *h) { return h ? &h->sim : nullptr; }

int ccs_set_static(ccs_handle *h) {
  int rc = ensure_built(h);
  if (rc) return rc;
  make_static(h);
  return CCS_OK;
}

int ccs_get_uniforms(ccs_handle *h, ccs_uniforms *out) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!out) return CCS_E_ARG;
  *out = pass_uniforms(h, 0, 0, 0.0);
  return CCS_OK;
}

int ccs_set_mesh_every(ccs_handle *h, int n) {
  if (!h || n < 1 || n > kMaxBlock) return CCS_E_ARG;
  h->meshEvery = n;
  h->recValid = false;
  return CCS_OK;
}

int ccs_set_field(ccs_handle *h, int on, const double g[3], double frozen, double invM, double cpIron) {
  if (!h || (on && (!g || !(invM > 0) || !(cpIron > 0)))) return CCS_E_ARG;
  h->field = on != 0;
  h->recValid = false;
  if (on) {
    for (int k = 0; k < 3; ++k) h->gField[k] = g[k];
    h->frozen = frozen;
    h->fieldInvM = invM;
    h->fieldCpIron = cpIron;
  }
  make_static(h);
  return CCS_OK;
}

int ccs_step(ccs_handle *h, int settle, int kick) {
  int rc = ensure_built(h);
  if (rc) return rc;
  cudaSetDevice(h->device);
  return do_step(h, settle, kick);
}

int ccs_steps(ccs_handle *h, int n) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (n < 0) return CCS_E_ARG;
  cudaSetDevice(h->device);
  while (n > 0) {
    const bool aligned = h->sim.stepNo % h->meshEvery == 0;
    const bool graphOk = h->useGraphs && !h->timing && aligned && n >= h->meshEvery && h->meshEvery % 2 == 0;
    if (graphOk) {
      rc = graph_block(h);
      if (rc) return rc;
      n -= h->meshEvery;
    } else {
      rc = do_step(h, 0, 0);
      if (rc) return rc;
      h->sim.t += h->sim.dt;
      --n;
    }
  }
  return check_launch(h);
}

}  // extern "C"

// ---- the autotuner: launch shapes by measurement on the run's own state ----
namespace {
std::mutex g_tuneMu;
std::map<std::pair<int, int>, std::pair<int, int>> g_tuned;   // (N, G) -> (warps, split)

// mean device time (ms) of `reps` launches of f on the handle's stream, after one warm launch
template <class F>
int time_launches(ccs_handle *h, int reps, F f, float *ms) {
  cudaEvent_t a, b;
  CUDA_TRY(h, cudaEventCreate(&a));
  CUDA_TRY(h, cudaEventCreate(&b));
  f();
  cudaEventRecord(a, h->st);
  for (int r = 0; r < reps; ++r) f();
  cudaEventRecord(b, h->st);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) {
    h->err = std::string("autotune timing: ") + cudaGetErrorString(e);
    return CCS_E_CUDA;
  }
  *ms = t / (float)reps;
  return CCS_OK;
}
}  // namespace

extern "C" {

int ccs_autotune(ccs_handle *h, int reps, int choice[2]) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (reps < 0) return CCS_E_ARG;
  cudaSetDevice(h->device);
  const std::pair<int, int> key(h->N, h->sim.G);
  int warps = 8, split = 4;
  if (reps == 0) {
    std::lock_guard<std::mutex> lk(g_tuneMu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      warps = it->second.first;
      split = it->second.second;
    }
  } else {
    CUDA_TRY(h, cudaStreamSynchronize(h->st));
    const ccs_uniforms tu = pass_uniforms(h, 0, 0, 0.0);
    const ccs_uniforms *U;
    rc = push_uniforms(h, tu, &U);
    if (rc) return rc;
    const int timing = h->timing;
    h->timing = 0;
    const int64_t l0 = h->launches;
    // the contact step into the spare buffers (no state changes), at each CTA width
    const SimArgs a = sim_args(h);
    float best = 1e30f;
    for (int w : {8, 4}) {
      float ms = 0.0f;
      rc = time_launches(h, reps, [&] { launch_simulate(tu, h->N, a, h->st, w, h->field); }, &ms);
      if (rc) break;
      if (ms < best) { best = ms; warps = w; }
    }
    // the cell gravity of box 0 over the last mesh step's inputs (it rewrites the same force), at each split
    best = 1e30f;
    for (int sp : {2, 4, 8}) {
      if (rc) break;
      float ms = 0.0f;
      rc = time_launches(h, reps, [&] { launch_cell(U, h->pm[0], h->st, sp); }, &ms);
      if (rc) break;
      if (ms < best) { best = ms; split = sp; }
    }
    if (!rc) launch_cell(U, h->pm[0], h->st, split);
    h->timing = timing;
    h->launches = l0;
    if (rc) return rc;
    CUDA_TRY(h, cudaStreamSynchronize(h->st));
    std::lock_guard<std::mutex> lk(g_tuneMu);
    g_tuned[key] = std::make_pair(warps, split);
  }
  if (warps != h->tuneWarps || split != h->tuneSplit) {
    CUDA_TRY(h, cudaStreamSynchronize(h->st));
    free_graphs(h);   // captured blocks hold the old shapes
    h->tuneWarps = warps;
    h->tuneSplit = split;
  }
  if (choice) {
    choice[0] = warps;
    choice[1] = split;
  }
  return check_launch(h);
}

}  // extern "C"

// ---- the batched ensemble: every member's block from one graph ----
namespace {
struct EnsembleGraph {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;             // the template, kept for its contact-step nodes' arguments
  std::vector<ccs_uniforms *> dev, host;   // per member: meshEvery uniform slots, and their pinned staging
  std::vector<UniNode> uni;                // every member's by-value nodes, member by member, in capture order
  std::vector<int> member;                 // the member each of them belongs to
  cudaEvent_t done = nullptr;
  bool used = false;
  // the persistent form: every round's step arguments ([round][member][step]) and their pinned staging, and
  // each round's counters ([round][member], with the round's abort flag after them)
  EnsStepArgs *args = nullptr, *argsHost = nullptr;
  unsigned char *state = nullptr;
  size_t stateBytes = 0;
};
}  // namespace

struct ccs_ensemble {
  int device = 0, M = 8;
  std::vector<ccs_handle *> m;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr, after = nullptr;
  std::vector<cudaEvent_t> join, ready;
  std::map<std::pair<int, std::vector<GraphKey>>, EnsembleGraph> graphs;   // (rounds, members' keys)
  std::string err;
  // the persistent form (ccs_ensemble_set_persistent): each round one launch of k_ensemble_round
  bool persistent = false;
  int ctas = 0;                          // its CTAs: the device's resident count
  EnsMember *info = nullptr;             // per member: its round's segments
  int *order = nullptr;                  // the members in priority order: largest first
  unsigned long long *acc = nullptr;     // per member: ns and rounds (EnsLaunch::acc)
  unsigned *status = nullptr;            // kStatusEnsemble
  int64_t launches = 0;                  // persistent rounds launched
  unsigned long long waitNs = 2000000000ull;   // the longest a CTA of the round waits (ccs_ensemble_set_wait_ns)
};

constexpr int kEnsRounds = 4;   // rounds of meshEvery steps one ensemble graph holds

namespace {
void free_ensemble_graph(EnsembleGraph &g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  for (auto p : g.dev) cudaFree(p);
  for (auto p : g.host) cudaFreeHost(p);
  if (g.args) cudaFree(g.args);
  if (g.argsHost) cudaFreeHost(g.argsHost);
  if (g.state) cudaFree(g.state);
  if (g.done) cudaEventDestroy(g.done);
  g = EnsembleGraph();
}

void free_ensemble_graphs(ccs_ensemble *e) {
  for (auto &kv : e->graphs) free_ensemble_graph(kv.second);
  e->graphs.clear();
}

#define ENS_TRY(e, call)                                                                         \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      (e)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                             \
      return CCS_E_CUDA;                                                                         \
    }                                                                                            \
  } while (0)

// the persistent form: R rounds, each the members' mesh chains for the round's mesh step (parallel branches,
// as in the branch form) and then one launch of k_ensemble_round over every member's steps of the round

size_t ens_state_slice(int n) { return (sizeof(EnsState) * n + 255) / 256 * 256 + 256; }   // + the abort flag

int ensemble_block_persistent(ccs_ensemble *e, int R) {
  const int n = (int)e->m.size(), M = kEnsSteps * R;
  for (ccs_handle *h : e->m)
    if (h->field || h->ppSplit || h->nn || h->meshEvery != kEnsSteps) {
      e->err = "persistent ensemble: a member left the impact's step with the reference's P3M and meshEvery 8";
      return CCS_E_STATE;
    }
  std::vector<GraphKey> keys(n);
  std::vector<std::vector<StepPlan>> plans(n, std::vector<StepPlan>(M));
  std::vector<int> seat0(n), cur0(n);
  for (int i = 0; i < n; ++i) {
    ccs_handle *h = e->m[i];
    for (int k = 0; k < M; ++k) {
      plans[i][k] = plan_step(h, 0, 0);
      h->sim.t += h->sim.dt;   // the frame loop's clock, index.html:372
      if (plans[i][k].mesh != (k % kEnsSteps == 0) || plans[i][k].slots != (k % 2 == 0)) {
        e->err = "persistent ensemble: a member's schedule is not the 8-step cycle";
        return CCS_E_STATE;
      }
    }
    keys[i] = GraphKey{(int)(plans[i][0].u.boxB > 0.5f), h->ppCount > 0, h->seatCur, h->cur, -kEnsSteps, 0, 0};
    seat0[i] = h->seatCur;
    cur0[i] = h->cur;
  }
  const size_t nArgs = (size_t)R * n * kEnsSteps, slice = ens_state_slice(n);
  EnsembleGraph &g = e->graphs[std::make_pair(R, keys)];
  if (!g.exec) {
    g.stateBytes = slice * R;
    ENS_TRY(e, cudaMalloc(&g.args, sizeof(EnsStepArgs) * nArgs));
    ENS_TRY(e, cudaMallocHost(&g.argsHost, sizeof(EnsStepArgs) * nArgs));
    ENS_TRY(e, cudaMalloc(&g.state, g.stateBytes));
    ENS_TRY(e, cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
    cudaGraph_t graph;
    ENS_TRY(e, cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(g.args, g.argsHost, sizeof(EnsStepArgs) * nArgs, cudaMemcpyHostToDevice, e->st);
    cudaMemsetAsync(g.state, 0, g.stateBytes, e->st);
    for (int r = 0; r < R; ++r) {
      cudaEventRecord(e->fork, e->st);
      for (int i = 0; i < n; ++i) {   // the round's mesh step: mesh and pairwise pass from the round's positions
        ccs_handle *h = e->m[i];
        const int timing = h->timing;
        const int64_t l0 = h->launches;
        h->timing = 0;
        h->cur = cur0[i];
        cudaStreamWaitEvent(h->st, e->fork, 0);
        const StepPlan &p = plans[i][(size_t)r * kEnsSteps];
        const ccs_uniforms *U = &g.args[((size_t)r * n + i) * kEnsSteps].u;
        pass_mesh(h, U, p.u.boxB > 0.5f);
        pass_pp(h, U, p.u.ppCount);
        cudaEventRecord(e->join[i], h->st);
        cudaStreamWaitEvent(e->st, e->join[i], 0);
        h->timing = timing;
        h->launches = l0;
      }
      EnsLaunch L;
      L.members = n;
      L.steps = kEnsSteps;
      L.args = g.args + (size_t)r * n * kEnsSteps;
      L.info = e->info;
      L.state = reinterpret_cast<EnsState *>(g.state + slice * r);
      L.abort = reinterpret_cast<int *>(g.state + slice * r + slice - 256);
      L.front = L.abort + 1;
      L.status = e->status;
      L.acc = e->acc;
      L.order = e->order;
      L.limitNs = e->waitNs;
      launch_ensemble_round(L, e->ctas, e->st);
    }
    cudaError_t ce = cudaStreamEndCapture(e->st, &graph);
    if (ce == cudaSuccess) {
      ce = cudaGraphInstantiate(&g.exec, graph, 0);
      if (ce != cudaSuccess) {
        g.exec = nullptr;
        cudaGraphDestroy(graph);
      } else {
        g.graph = graph;
      }
    }
    if (ce != cudaSuccess) {
      e->err = std::string("persistent ensemble capture: ") + cudaGetErrorString(ce);
      free_ensemble_graph(g);
      e->graphs.erase(std::make_pair(R, keys));
      return CCS_E_CUDA;
    }
  }
  if (g.used) ENS_TRY(e, cudaEventSynchronize(g.done));   // the last replay has read the staging
  for (int i = 0; i < n; ++i) {
    ccs_handle *h = e->m[i];
    for (int K = 0; K < M; ++K) {
      const StepPlan &p = plans[i][K];
      const int seatB = seat0[i] ^ (((K + 1) / 2) & 1);   // the table the step finds: a rebuild every 2nd step
      h->cur = cur0[i] ^ (K & 1);
      h->seatCur = p.slots ? seatB ^ 1 : seatB;
      EnsStepArgs &A = g.argsHost[((size_t)(K / kEnsSteps) * n + i) * kEnsSteps + K % kEnsSteps];
      A.u = p.u;
      A.a = sim_args(h);
      A.a.walk = p.walk;
      A.gpos = h->pos[h->cur];
      A.gseats = h->seats[seatB ^ 1];
      A.ghk = h->hk[seatB ^ 1];
      A.gseatsOld = h->seats[seatB];
      A.ghkOld = h->hk[seatB];
      A.gstatus = h->status;
      A.grecMax = h->recMax;
    }
    h->cur = cur0[i];
    h->seatCur = seat0[i];
  }
  for (int i = 0; i < n; ++i) {   // after whatever each member has queued
    ENS_TRY(e, cudaEventRecord(e->ready[i], e->m[i]->st));
    ENS_TRY(e, cudaStreamWaitEvent(e->st, e->ready[i], 0));
  }
  ENS_TRY(e, cudaGraphLaunch(g.exec, e->st));
  g.used = true;
  ENS_TRY(e, cudaEventRecord(g.done, e->st));
  ENS_TRY(e, cudaEventRecord(e->after, e->st));
  e->launches += R;
  for (int i = 0; i < n; ++i) {   // and whatever they queue next comes after it
    ccs_handle *h = e->m[i];
    ENS_TRY(e, cudaStreamWaitEvent(h->st, e->after, 0));
    h->cur = cur0[i] ^ (M & 1);
    h->seatCur = seat0[i] ^ (((M + 1) / 2) & 1);
    for (int r = 0; r < R; ++r) {   // the mesh chain's kernels (the round's steps are the ensemble's launch)
      const StepPlan &p = plans[i][(size_t)r * kEnsSteps];
      h->launches += 5 * (1 + (p.u.boxB > 0.5f)) + (p.u.ppCount ? 3 : 0);
    }
  }
  return CCS_OK;
}

// R rounds: every member's next R x meshEvery steps, one graph launch
int ensemble_block(ccs_ensemble *e, int R) {
  if (e->persistent) return ensemble_block_persistent(e, R);
  const int n = (int)e->m.size(), M = e->M * R;
  std::vector<GraphKey> keys(n);
  std::vector<std::vector<StepPlan>> plans(n, std::vector<StepPlan>(M));
  std::vector<int> seat0(n), cur0(n);
  for (int i = 0; i < n; ++i) {
    ccs_handle *h = e->m[i];
    for (int k = 0; k < M; ++k) {
      plans[i][k] = plan_step(h, 0, 0);
      h->sim.t += h->sim.dt;   // the frame loop's clock, index.html:372
    }
    keys[i] = GraphKey{(int)(plans[i][0].u.boxB > 0.5f), h->ppCount > 0, h->seatCur, h->cur, e->M, h->ping,
                       (int)h->field};
    seat0[i] = h->seatCur;
    cur0[i] = h->cur;
  }
  EnsembleGraph &g = e->graphs[std::make_pair(R, keys)];
  if (!g.exec) {
    g.dev.assign(n, nullptr);
    g.host.assign(n, nullptr);
    for (int i = 0; i < n; ++i) {
      ENS_TRY(e, cudaMalloc(&g.dev[i], sizeof(ccs_uniforms) * M));
      ENS_TRY(e, cudaMallocHost(&g.host[i], sizeof(ccs_uniforms) * M));
    }
    ENS_TRY(e, cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
    cudaGraph_t graph;
    std::vector<CapturedNode> uniNodes;
    std::vector<int> member;
    bool lost = false;
    ENS_TRY(e, cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    cudaEventRecord(e->fork, e->st);
    for (int i = 0; i < n; ++i) {   // every member's block on its own stream: parallel branches
      ccs_handle *h = e->m[i];
      const int timing = h->timing;
      const int64_t l0 = h->launches;
      h->timing = 0;
      cudaStreamWaitEvent(h->st, e->fork, 0);
      cudaMemcpyAsync(g.dev[i], g.host[i], sizeof(ccs_uniforms) * M, cudaMemcpyHostToDevice, h->st);
      h->uniCapture = &uniNodes;
      h->inEnsemble = true;
      for (int k = 0; k < M; ++k) {
        h->captureStep = k;
        enqueue_step(h, plans[i][k], g.dev[i] + k);
      }
      h->inEnsemble = false;
      h->uniCapture = nullptr;
      member.resize(uniNodes.size(), i);
      lost = lost || h->uniCaptureLost;
      h->uniCaptureLost = false;
      cudaEventRecord(e->join[i], h->st);
      cudaStreamWaitEvent(e->st, e->join[i], 0);
      h->timing = timing;
      h->launches = l0;
      h->seatCur = seat0[i];   // capture ran the buffer rotation on the host; the replay redoes it
      h->cur = cur0[i];
    }
    cudaError_t ce = cudaStreamEndCapture(e->st, &graph);
    if (ce != cudaSuccess) {
      e->err = std::string("ensemble capture: ") + cudaGetErrorString(ce);
      free_ensemble_graph(g);
      e->graphs.erase(std::make_pair(R, keys));
      return CCS_E_CUDA;
    }
    ce = cudaGraphInstantiate(&g.exec, graph, 0);
    if (ce != cudaSuccess) {
      cudaGraphDestroy(graph);
      e->err = std::string("ensemble instantiate: ") + cudaGetErrorString(ce);
      g.exec = nullptr;
      free_ensemble_graph(g);
      e->graphs.erase(std::make_pair(R, keys));
      return CCS_E_CUDA;
    }
    g.graph = graph;
    int rc = lost ? CCS_E_CUDA : resolve_uniform_nodes(e->m[0], uniNodes, g.uni);
    g.member = member;
    size_t want = 0;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < M; ++k) want += plans[i][k].slots ? 2 : 1;
    if (rc == CCS_OK && g.uni.size() != want) rc = CCS_E_CUDA;
    if (rc) {
      e->err = "ensemble capture: a contact-step node per member step and a grid node per even step expected";
      free_ensemble_graph(g);
      e->graphs.erase(std::make_pair(R, keys));
      return rc;
    }
  } else {
    for (size_t j = 0; j < g.uni.size(); ++j) {   // each member step's uniforms into its by-value nodes
      const int i = g.member[j];
      const int rc = set_node_uniforms(e->m[i], g.exec, g.uni[j], plans[i][g.uni[j].c.step].u);
      if (rc) {
        e->err = e->m[i]->err;
        return rc;
      }
    }
  }
  if (g.used) ENS_TRY(e, cudaEventSynchronize(g.done));
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < M; ++k) g.host[i][k] = plans[i][k].u;
  for (int i = 0; i < n; ++i) {   // after whatever each member has queued
    ENS_TRY(e, cudaEventRecord(e->ready[i], e->m[i]->st));
    ENS_TRY(e, cudaStreamWaitEvent(e->st, e->ready[i], 0));
  }
  ENS_TRY(e, cudaGraphLaunch(g.exec, e->st));
  g.used = true;   // the next use of this graph waits for this replay before it rewrites the staging
  ENS_TRY(e, cudaEventRecord(g.done, e->st));
  ENS_TRY(e, cudaEventRecord(e->after, e->st));
  for (int i = 0; i < n; ++i) {   // and whatever they queue next comes after it
    ccs_handle *h = e->m[i];
    ENS_TRY(e, cudaStreamWaitEvent(h->st, e->after, 0));
    h->ping ^= 1;
    h->cur = cur0[i] ^ (M & 1);
    h->seatCur = seat0[i] ^ (((M + 1) / 2) & 1);
    h->launches += block_launches(h, plans[i].data(), M);
  }
  return CCS_OK;
}
}  // namespace

extern "C" {

int ccs_ensemble_create(ccs_handle *const *members, int count, ccs_ensemble **out) {
  if (!out || !members || count <= 0) return CCS_E_ARG;
  *out = nullptr;
  for (int i = 0; i < count; ++i) {
    if (!members[i] || !members[i]->built) return CCS_E_STATE;
    if (members[i]->device != members[0]->device || members[i]->meshEvery != members[0]->meshEvery ||
        members[i]->meshEvery % 2)
      return CCS_E_ARG;
    for (int j = 0; j < i; ++j)
      if (members[j] == members[i]) return CCS_E_ARG;
  }
  cudaSetDevice(members[0]->device);
  ccs_ensemble *e = new (std::nothrow) ccs_ensemble();
  if (!e) return CCS_E_NOMEM;
  e->device = members[0]->device;
  e->M = members[0]->meshEvery;
  e->m.assign(members, members + count);
  e->join.assign(count, nullptr);
  e->ready.assign(count, nullptr);
  bool ok = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->after, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; ok && i < count; ++i)
    ok = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&e->ready[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    ccs_ensemble_destroy(e);
    return CCS_E_CUDA;
  }
  *out = e;
  return CCS_OK;
}

int ccs_ensemble_destroy(ccs_ensemble *e) {
  if (!e) return CCS_OK;
  cudaSetDevice(e->device);
  if (e->st) cudaStreamSynchronize(e->st);
  free_ensemble_graphs(e);
  for (auto ev : e->join) if (ev) cudaEventDestroy(ev);
  for (auto ev : e->ready) if (ev) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->after) cudaEventDestroy(e->after);
  if (e->st) cudaStreamDestroy(e->st);
  if (e->info) cudaFree(e->info);
  if (e->order) cudaFree(e->order);
  if (e->acc) cudaFree(e->acc);
  if (e->status) cudaFree(e->status);
  delete e;
  return CCS_OK;
}

const char *ccs_ensemble_last_error(const ccs_ensemble *e) { return e ? e->err.c_str() : "null ensemble"; }

int ccs_ensemble_steps(ccs_ensemble *e, int n) {
  if (!e || n < 0 || n % e->M) return CCS_E_ARG;
  for (ccs_handle *h : e->m)
    if (h->sim.stepNo % e->M || h->meshEvery != e->M || h->timing) {
      e->err = "every member must sit at a block boundary (stepNo % meshEvery == 0) with timing off";
      return CCS_E_STATE;
    }
  cudaSetDevice(e->device);
  for (int blocks = n / e->M; blocks > 0;) {
    const int R = blocks < kEnsRounds ? blocks : kEnsRounds;
    int rc = ensemble_block(e, R);
    if (rc) return rc;
    blocks -= R;
  }
  return CCS_OK;
}

int ccs_ensemble_autotune(ccs_ensemble *e, int rounds, int choice[2]) {
  if (!e || rounds <= 0) return CCS_E_ARG;
  for (ccs_handle *h : e->m)
    if (h->sim.stepNo % e->M || h->timing) {
      e->err = "every member must sit at a block boundary (stepNo % meshEvery == 0) with timing off";
      return CCS_E_STATE;
    }
  cudaSetDevice(e->device);
  const int R = rounds < kEnsRounds ? rounds : kEnsRounds;
  int bestW = 8, bestS = 4;
  double best = 1e300;
  cudaEvent_t a = nullptr, b = nullptr;
  ENS_TRY(e, cudaEventCreate(&a));
  ENS_TRY(e, cudaEventCreate(&b));
  int rc = CCS_OK;
  for (int w : {8, 4}) {
    for (int sp : {2, 4, 8}) {
      for (ccs_handle *h : e->m) {
        if (h->tuneWarps != w || h->tuneSplit != sp) {
          cudaStreamSynchronize(h->st);
          free_graphs(h);
          h->tuneWarps = w;
          h->tuneSplit = sp;
        }
      }
      ENS_TRY(e, cudaStreamSynchronize(e->st));
      free_ensemble_graphs(e);
      rc = ensemble_block(e, R);   // captures this shape's graph
      if (rc) break;
      ENS_TRY(e, cudaEventRecord(a, e->st));
      for (int r = 0; r < rounds; r += R) {
        rc = ensemble_block(e, R);
        if (rc) break;
      }
      if (rc) break;
      ENS_TRY(e, cudaEventRecord(b, e->st));
      ENS_TRY(e, cudaEventSynchronize(b));
      float ms = 0.0f;
      ENS_TRY(e, cudaEventElapsedTime(&ms, a, b));
      if (ms < best) {
        best = ms;
        bestW = w;
        bestS = sp;
      }
    }
    if (rc) break;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  for (ccs_handle *h : e->m) {
    if (h->tuneWarps != bestW || h->tuneSplit != bestS) {
      cudaStreamSynchronize(h->st);
      free_graphs(h);
      h->tuneWarps = bestW;
      h->tuneSplit = bestS;
    }
  }
  ENS_TRY(e, cudaStreamSynchronize(e->st));
  free_ensemble_graphs(e);
  if (choice) {
    choice[0] = bestW;
    choice[1] = bestS;
  }
  return CCS_OK;
}

int ccs_ensemble_sync(ccs_ensemble *e) {
  if (!e) return CCS_E_ARG;
  cudaSetDevice(e->device);
  ENS_TRY(e, cudaStreamSynchronize(e->st));
  if (e->status) {
    unsigned st = 0;
    ENS_TRY(e, cudaMemcpy(&st, e->status, sizeof st, cudaMemcpyDeviceToHost));
    if (st & kStatusEnsemble) {
      e->err = "persistent ensemble round: a wait for work ran out (the round was abandoned)";
      return CCS_E_KERNEL;
    }
  }
  for (ccs_handle *h : e->m) {
    int rc = check_status(h);
    if (rc) {
      e->err = h->err;
      return rc;
    }
  }
  return CCS_OK;
}

int ccs_ensemble_set_persistent(ccs_ensemble *e, int on) {
  if (!e || (on != 0 && on != 1)) return CCS_E_ARG;
  cudaSetDevice(e->device);
  if (on) {
    if (e->M != kEnsSteps) {
      e->err = "persistent ensemble: meshEvery must be 8";
      return CCS_E_STATE;
    }
    for (ccs_handle *h : e->m)
      if (h->field || h->ppSplit || h->nn) {
        e->err = "persistent ensemble: members run the impact's step with the reference's P3M (no field step, "
                 "stencil-split or learned pass)";
        return CCS_E_STATE;
      }
  }
  ENS_TRY(e, cudaStreamSynchronize(e->st));
  free_ensemble_graphs(e);
  e->persistent = on != 0;
  if (!on || e->info) return CCS_OK;
  const int n = (int)e->m.size();
  std::vector<EnsMember> info(n);
  long total = 0;
  for (int i = 0; i < n; ++i) {   // the round's chain: grid, contact step on even steps; contact step on odd
    EnsMember &I = info[i];
    constexpr int kItem = kEnsContactItem;
    const int N = e->m[i]->N, gi = (N + kEnsGridItem - 1) / kEnsGridItem, ci = (N + kItem - 1) / kItem;
    I.nseg = 0;
    int t = 0;
    for (int k = 0; k < kEnsSteps; ++k) {
      if (k % 2 == 0) {
        t += gi;
        I.end[I.nseg] = t;
        I.step[I.nseg] = k;
        I.grid[I.nseg++] = 1;
      }
      t += ci;
      I.end[I.nseg] = t;
      I.step[I.nseg] = k;
      I.grid[I.nseg++] = 0;
    }
    I.total = t;
    total += N;
  }
  (void)total;
  e->ctas = ensemble_round_ctas();
  std::vector<int> order(n);   // largest first (ties in member order): the longest chains start first
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e->m[a]->N > e->m[b]->N; });
  ENS_TRY(e, cudaMalloc(&e->info, sizeof(EnsMember) * n));
  ENS_TRY(e, cudaMalloc(&e->order, sizeof(int) * n));
  ENS_TRY(e, cudaMalloc(&e->acc, sizeof(unsigned long long) * 2 * n));
  ENS_TRY(e, cudaMalloc(&e->status, sizeof(unsigned)));
  ENS_TRY(e, cudaMemcpy(e->info, info.data(), sizeof(EnsMember) * n, cudaMemcpyHostToDevice));
  ENS_TRY(e, cudaMemcpy(e->order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  ENS_TRY(e, cudaMemset(e->acc, 0, sizeof(unsigned long long) * 2 * n));
  ENS_TRY(e, cudaMemset(e->status, 0, sizeof(unsigned)));
  return CCS_OK;
}

int ccs_ensemble_step_ms(ccs_ensemble *e, double *ms, int count) {
  if (!e || !ms || count != (int)e->m.size()) return CCS_E_ARG;
  if (!e->acc) return CCS_E_STATE;
  cudaSetDevice(e->device);
  const int n = (int)e->m.size();
  ENS_TRY(e, cudaStreamSynchronize(e->st));
  std::vector<unsigned long long> acc(2 * n);
  ENS_TRY(e, cudaMemcpy(acc.data(), e->acc, sizeof(unsigned long long) * 2 * n, cudaMemcpyDeviceToHost));
  ENS_TRY(e, cudaMemset(e->acc, 0, sizeof(unsigned long long) * 2 * n));
  for (int i = 0; i < n; ++i)
    ms[i] = acc[n + i] ? (double)acc[i] / (double)acc[n + i] / kEnsSteps * 1e-6 : -1.0;
  return CCS_OK;
}

int64_t ccs_ensemble_launch_count(const ccs_ensemble *e) { return e ? e->launches : -1; }

int ccs_ensemble_set_wait_ns(ccs_ensemble *e, uint64_t ns) {
  if (!e || ns == 0) return CCS_E_ARG;
  cudaSetDevice(e->device);
  ENS_TRY(e, cudaStreamSynchronize(e->st));
  free_ensemble_graphs(e);   // the bound is an argument of the captured launches
  e->waitNs = ns;
  if (e->status) ENS_TRY(e, cudaMemset(e->status, 0, sizeof(unsigned)));
  return CCS_OK;
}

int ccs_settle_some(ccs_handle *h, int n) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (n < 0) return CCS_E_ARG;
  ccs_sim &s = h->sim;
  n = n < s.settleLeft ? n : s.settleLeft;
  for (int i = 0; i < n; ++i) {
    rc = do_step(h, 1, 0);
    if (rc) return rc;
  }
  s.settleLeft -= n;
  if (s.settleLeft == 0 && s.phase == 0) s.phase = 1;
  return CCS_OK;
}

static void turn_matrix(const double w[3], double dt, float o[9]) {
  const double m = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  if (m < 1e-12) {
    const float I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::memcpy(o, I, sizeof I);
    return;
  }
  const double x = w[0] / m, y = w[1] / m, z = w[2] / m, th = m * dt, c = std::cos(th), s = std::sin(th), t = 1 - c;
  const double r[9] = {t * x * x + c,     t * x * y + s * z, t * x * z - s * y,
                       t * x * y - s * z, t * y * y + c,     t * y * z + s * x,
                       t * x * z + s * y, t * y * z - s * x, t * z * z + c};
  for (int k = 0; k < 9; ++k) o[k] = (float)r[k];
}

int ccs_rigid_step(ccs_handle *h, double dtF) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!(dtF > 0)) return CCS_E_ARG;
  cudaSetDevice(h->device);
  h->recValid = false;   // the particles move without a contact step
  ccs_sim &s = h->sim;
  double *r = s.relr, *v = s.relv;
  const double M = s.M, M1 = s.M1, M2 = s.M2;
  const double r0[3] = {r[0], r[1], r[2]};
  const int n = 8;
  const double hh = dtF / n;
  double a[3];
  auto acc = [&]() {
    const double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const double f = -M * std::pow(d2, -1.5);
    a[0] = r[0] * f; a[1] = r[1] * f; a[2] = r[2] * f;
  };
  const double cen[2][3] = {{-r0[0] * M2 / M, -r0[1] * M2 / M, -r0[2] * M2 / M},
                            {r0[0] * M1 / M, r0[1] * M1 / M, r0[2] * M1 / M}};
  acc();
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) v[k] += a[k] * hh * 0.5;
    for (int k = 0; k < 3; ++k) r[k] += v[k] * hh;
    acc();
    for (int k = 0; k < 3; ++k) v[k] += a[k] * hh * 0.5;
  }
  const double mv[3] = {(r[0] - r0[0]) / dtF, (r[1] - r0[1]) / dtF, (r[2] - r0[2]) / dtF};
  for (int k = 0; k < 3; ++k) {
    s.bulk0[k] = -mv[k] * M2 / M;
    s.bulk1[k] = mv[k] * M1 / M;
  }
  ccs_uniforms u = pass_uniforms(h, 0, 0, 0.0);
  for (int k = 0; k < 3; ++k) {
    u.cen0[k] = (float)cen[0][k];
    u.cen1[k] = (float)cen[1][k];
  }
  turn_matrix(s.spin0, dtF, u.rot0);
  turn_matrix(s.spin1, dtF, u.rot1);
  u.rdt = (float)dtF;
  const ccs_uniforms *U;
  rc = push_uniforms(h, u, &U);
  if (rc) return rc;
  const int src = h->cur, dst = h->cur ^ 1;
  h->launches += launch_rigid(U, h->N, h->pos[src], h->vel[src], h->aux[src], h->q[src], h->pos[dst], h->vel[dst],
                              h->aux[dst], h->q[dst], h->st);
  h->cur = dst;
  s.t += dtF;
  if (std::hypot(std::hypot(r[0], r[1]), r[2]) <= s.Re1 + s.Re2 + 2 * s.a) {   // the equators touch
    for (int k = 0; k < 3; ++k) {
      s.bulk0[k] = -v[k] * M2 / M;
      s.bulk1[k] = v[k] * M1 / M;
      s.cen0[k] = -r[k] * M2 / M;
      s.cen1[k] = r[k] * M1 / M;
      s.boxCen[0][k] = s.cen0[k];
      s.boxVel[0][k] = s.bulk0[k];
    }
    s.boxOn[0] = 1;
    s.boxT[0] = s.t;
    s.boxOn[1] = 0;
    s.stepNo = 0;
    rc = do_step(h, 0, 1);
    if (rc) return rc;
    s.t += s.dt;
    s.phase = 2;
    s.impactT = s.t;
  }
  return check_launch(h);
}

int ccs_set_pp(ccs_handle *h, const int32_t *list, int n, int loose) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (n < 0 || n > CCS_PP_CAP || (n > 0 && !list)) return CCS_E_ARG;
  rc = ensure_nn_buffers(h, n);
  if (rc) return rc;
  for (int k = 0; k < n; ++k)
    if (list[k] < 0 || list[k] >= h->N) {
      h->err = "loose-list index out of range";
      return CCS_E_ARG;
    }
  cudaSetDevice(h->device);
  std::vector<int32_t> slot((size_t)h->N, -1), index(CCS_PP_CAP, -1);
  for (int k = 0; k < n; ++k) {
    slot[(size_t)list[k]] = k;
    index[(size_t)k] = list[k];
  }
  // synchronous copies: the vectors die with this call
  CUDA_TRY(h, cudaMemcpyAsync(h->ppSlot, slot.data(), 4 * (size_t)h->N, cudaMemcpyHostToDevice, h->st));
  CUDA_TRY(h, cudaMemcpyAsync(h->ppIndex, index.data(), 4 * (size_t)CCS_PP_CAP, cudaMemcpyHostToDevice, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  h->ppCount = n;
  h->ppLoose = loose;
  if (n) {
    const ccs_uniforms *U;
    rc = push_uniforms(h, pass_uniforms(h, 0, 0, 0.0), &U);
    if (rc) return rc;
    pass_pp(h, U, n);
  }
  return check_launch(h);
}

int ccs_set_pp_nn(ccs_handle *h, ccs_nn *nn) {
  if (!h) return CCS_E_ARG;
  if (nn && nn_device(nn) != h->device) {
    h->err = "the network lives on another device";
    return CCS_E_ARG;
  }
  cudaSetDevice(h->device);
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  free_graphs(h);   // the captured P3M launches change
  h->nn = nn;
  if (nn && h->built) return ensure_nn_buffers(h, h->ppCount);
  return CCS_OK;
}

int ccs_nn_sample_state(ccs_nn *nn, ccs_handle *h, int64_t count, uint32_t seed) {
  if (!nn || !h || count < 0) return CCS_E_ARG;
  int rc = ensure_built(h);
  if (rc) return rc;
  if (nn_device(nn) != h->device) {
    h->err = "the network lives on another device";
    return CCS_E_ARG;
  }
  cudaSetDevice(h->device);
  const ccs_uniforms *U;
  rc = push_uniforms(h, pass_uniforms(h, 0, 0, 0.0), &U);   // the boxes where they are now
  if (rc) return rc;
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  float4 *D, *S;
  cudaStream_t st;
  rc = nn_reserve(nn, count, &D, &S, &st);
  if (rc) return rc;
  launch_nn_sample_state(U, h->pos[h->cur], h->N, (long)count, seed, (float)CCS_NN_CUT_CELLS, D, S, st);
  return nn_commit(nn, count);
}

int ccs_prime_mono(ccs_handle *h, int box, const float mono[4]) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (box < 0 || box > 1 || !mono) return CCS_E_ARG;
  float4 m = make_float4(mono[0], mono[1], mono[2], mono[3]);
  CUDA_TRY(h, cudaMemcpyAsync(h->pm[box].mono, &m, sizeof m, cudaMemcpyHostToDevice, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  return CCS_OK;
}

int ccs_set_boxes(ccs_handle *h, const ccs_box boxes[2]) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!boxes) return CCS_E_ARG;
  for (int b = 0; b < 2; ++b) {   // everything checked before anything changes
    const ccs_box &x = boxes[b];
    bool ok = (x.on == 0 || x.on == 1) && (x.primeMono == 0 || x.primeMono == 1) && std::isfinite(x.t);
    for (int k = 0; k < 3; ++k)
      ok = ok && std::isfinite(x.cen[k]) && std::isfinite(x.vel[k]) && std::fabs(x.cen[k]) < 1e6;
    if (x.primeMono)
      for (int k = 0; k < 4; ++k) ok = ok && std::isfinite(x.mono[k]);
    if (!ok) {
      h->err = "ccs_set_boxes: box " + std::to_string(b) + " has a flag other than 0/1 or a non-finite value";
      return CCS_E_ARG;
    }
  }
  for (int b = 0; b < 2; ++b) {
    const ccs_box &x = boxes[b];
    h->sim.boxOn[b] = x.on;
    for (int k = 0; k < 3; ++k) {
      h->sim.boxCen[b][k] = x.cen[k];
      h->sim.boxVel[b][k] = x.vel[k];
    }
    h->sim.boxT[b] = x.t;
    if (x.primeMono) {
      rc = ccs_prime_mono(h, b, x.mono);
      if (rc) return rc;
    }
  }
  return CCS_OK;
}

static int apply_perm_device(ccs_handle *h, const int32_t *permDev) {
  const int s = h->cur, d = h->cur ^ 1;
  h->recValid = false;   // the record names particles by their old places
  h->launches += launch_permute(h->N, permDev, h->pos[s], h->vel[s], h->aux[s], h->q[s], h->mat, h->home, h->pos[d],
                                h->vel[d], h->aux[d], h->q[d], h->matTmp, h->homeTmp, h->st);
  std::swap(h->mat, h->matTmp);
  std::swap(h->home, h->homeTmp);
  h->cur = d;
  // the old cells name particles by their old places: fresh ones
  pass_slots(h, pass_uniforms(h, 0, 0, 0.0));
  return check_launch(h);
}

int ccs_apply_perm(ccs_handle *h, const int32_t *perm) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!perm) return CCS_E_ARG;
  cudaSetDevice(h->device);
  std::vector<char> seen((size_t)h->N, 0);
  for (int i = 0; i < h->N; ++i) {
    if (perm[i] < 0 || perm[i] >= h->N || seen[(size_t)perm[i]]) {
      h->err = "perm is not a permutation of 0..N-1";
      return CCS_E_ARG;
    }
    seen[(size_t)perm[i]] = 1;
  }
  CUDA_TRY(h, cudaMemcpyAsync(h->permDev, perm, 4 * (size_t)h->N, cudaMemcpyHostToDevice, h->st));
  rc = apply_perm_device(h, h->permDev);
  if (rc) return rc;
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  return CCS_OK;
}

// passDiag, src/nbody.js:488-507
static int diag_pass(ccs_handle *h) {
  set_boxes(h);
  const ccs_uniforms du = pass_uniforms(h, 0, 0, 0.0);
  const ccs_uniforms *U;
  int rc = push_uniforms(h, du, &U);
  if (rc) return rc;
  pass_slots(h, du);
  pass_mesh(h, U, h->boxB > 0.5f);
  pass_pp(h, U, h->ppCount);
  pass_diag_kernel(h, U);
  return check_launch(h);
}

int ccs_sort_morton(ccs_handle *h, const double core[3], int32_t *perm_out, int32_t *into_out) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!core) return CCS_E_ARG;
  cudaSetDevice(h->device);
  h->recValid = false;
  const int N = h->N;
  h->launches += launch_morton_keys(N, h->pos[h->cur], core[0], core[1], core[2], h->keys, h->vals, h->st);
  h->launches += launch_radix_sort(N, 21, h->keys, h->vals, h->keysTmp, h->valsTmp, h->hist, h->st);
  CUDA_TRY(h, cudaMemcpyAsync(h->permDev, h->vals, 4 * (size_t)N, cudaMemcpyDeviceToDevice, h->st));
  h->launches += launch_invert_perm(N, h->permDev, h->into, h->st);
  if (perm_out) CUDA_TRY(h, cudaMemcpyAsync(perm_out, h->permDev, 4 * (size_t)N, cudaMemcpyDeviceToHost, h->st));
  if (into_out) CUDA_TRY(h, cudaMemcpyAsync(into_out, h->into, 4 * (size_t)N, cudaMemcpyDeviceToHost, h->st));
  rc = apply_perm_device(h, h->permDev);
  if (rc) return rc;
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  return CCS_OK;
}

}  // extern "C"

// ---- fof of src/nbody.js:646-893 on the device; the report assembled as ccs_fof assembles it ----
namespace {
struct DevGroup {
  int n = 0;
  double mass = 0, com[3] = {}, core[3] = {}, vel[3] = {}, imp = 0, iron = 0, R = 0, Redge = 0, Tsurf = 0;
  double hotCom[3] = {}, hotR = 0, impMass = 0, impCom[3] = {}, impRms = 0;
};

int fof_sum(ccs_handle *h, const FofSumArgs &a, double out[kFofTerms]) {
  h->launches += launch_fof_sums(a, h->fofPart, h->st);
  const int nb = fof_blocks(a.N);
  std::vector<double> part((size_t)nb * kFofTerms);
  CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->fofPart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  for (int k = 0; k < kFofTerms; ++k) out[k] = 0.0;
  for (int b = 0; b < nb; ++b)
    for (int k = 0; k < kFofTerms; ++k) out[k] += part[(size_t)b * kFofTerms + k];
  return CCS_OK;
}

int fof_group(ccs_handle *h, FofSumArgs a, int g, DevGroup &G) {
  double t[kFofTerms];
  a.g = g;
  a.pass = kFofGroup;
  int rc = fof_sum(h, a, t);
  if (rc) return rc;
  G.n = (int)t[0];
  G.mass = t[1];
  G.impMass = t[8];
  G.iron = t[12];
  const double mass = G.mass, imp = G.impMass, Rg = std::cbrt(mass);
  for (int k = 0; k < 3; ++k) {
    G.com[k] = t[2 + k] / mass;
    G.impCom[k] = imp > 0 ? t[9 + k] / imp : 0;
  }
  const double tm = mass - imp;
  double core[3];
  if (imp > tm) for (int k = 0; k < 3; ++k) core[k] = G.impCom[k];
  else for (int k = 0; k < 3; ++k) core[k] = (t[2 + k] - t[9 + k]) / tm;
  a.pass = kFofCore;
  a.r2 = 0.9 * 0.9 * Rg * Rg;
  for (int it = 0; it < 3; ++it) {
    for (int k = 0; k < 3; ++k) a.c[k] = core[k];
    double c[kFofTerms];
    rc = fof_sum(h, a, c);
    if (rc) return rc;
    if (c[0] > 0) for (int k = 0; k < 3; ++k) core[k] = c[1 + k] / c[0];
  }
  std::memcpy(G.core, core, sizeof core);
  const double shell = 0.64 * Rg * Rg, dr = 3 * Rg / kFofBins;
  a.pass = kFofShape;
  a.r2 = shell;
  for (int k = 0; k < 3; ++k) { a.c[k] = core[k]; a.d[k] = G.impCom[k]; }
  double sh[kFofTerms];
  rc = fof_sum(h, a, sh);
  if (rc) return rc;
  const double Ts = sh[0], ws = sh[1], irms = sh[2], hs = sh[3], hx = sh[4], hy = sh[5], hz = sh[6], hr2 = sh[7];
  std::memcpy(G.hotCom, core, sizeof core);
  G.hotR = Rg;
  if (hs > 0) {
    G.hotCom[0] = hx / hs; G.hotCom[1] = hy / hs; G.hotCom[2] = hz / hs;
    const double ox = G.hotCom[0] - core[0], oy = G.hotCom[1] - core[1], oz = G.hotCom[2] - core[2];
    G.hotR = std::sqrt(std::max(hr2 / hs - (ox * ox + oy * oy + oz * oz), 0.0));
  }
  if (G.n >= 2000) {   // where the body ends: the first shell under a third of the mantle's density
    h->launches += launch_fof_hist(a, dr, h->fofPart, h->st);
    const int nb = fof_blocks(a.N);
    std::vector<double> part((size_t)nb * kFofBins);
    CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->fofPart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, h->st));
    CUDA_TRY(h, cudaStreamSynchronize(h->st));
    double hist[kFofBins] = {};
    for (int b = 0; b < nb; ++b)
      for (int k = 0; k < kFofBins; ++k) hist[k] += part[(size_t)b * kFofBins + k];
    const double Rb = std::cbrt(std::max(imp, tm));
    double rho[kFofBins], refS = 0;
    int refN = 0;
    for (int b = 0; b < kFofBins; ++b) {
      const double rm = (b + 0.5) * dr;
      rho[b] = hist[b] / (rm * rm * dr);
      if (rm > 0.6 * Rb && rm < 0.85 * Rb) { refS += rho[b]; ++refN; }
    }
    G.Redge = Rg;
    for (int b = 0; b < kFofBins; ++b)
      if ((b + 0.5) * dr > 0.85 * Rb && refN > 0 && rho[b] < 0.35 * refS / refN) { G.Redge = b * dr; break; }
  }
  for (int k = 0; k < 3; ++k) G.vel[k] = t[5 + k] / mass;
  G.imp = imp / mass;
  G.iron /= mass;
  G.R = Rg;
  G.Tsurf = ws > 0 ? Ts / ws : 0;
  G.impRms = imp > 0 ? std::sqrt(irms / imp) : 0;
  return CCS_OK;
}

int ensure_fof_buffers(ccs_handle *h) {
  if (h->fofParent) return CCS_OK;
  const int N = h->N, nb = fof_blocks(N);
  int rc = CCS_OK;
  rc |= dev_alloc(h, &h->fofParent, N); rc |= dev_alloc(h, &h->fofSize, N);
  rc |= dev_alloc(h, &h->fofStart, kFofBuckets); rc |= dev_alloc(h, &h->fofEnd, kFofBuckets);
  rc |= dev_alloc(h, &h->fofCounts, nb); rc |= dev_alloc(h, &h->fofOffs, nb + 1); rc |= dev_alloc(h, &h->fofNDist, 1);
  rc |= dev_alloc(h, &h->fofList, CCS_PP_CAP); rc |= dev_alloc(h, &h->fofPart, (size_t)nb * kFofBins);
  rc |= dev_alloc(h, &h->fofElastic, nb); rc |= dev_alloc(h, &h->fofDist, N); rc |= dev_alloc(h, &h->fofTop, 2 * nb);
  return rc ? CCS_E_NOMEM : CCS_OK;
}
}  // namespace

extern "C" {

int ccs_fof_device(ccs_handle *h, double spring, double touch, int cap, int sort, ccs_report *rep, int32_t *list,
                   int32_t *perm) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!rep || cap < 0 || cap > CCS_PP_CAP || (cap > 0 && !list) || (sort && !perm)) return CCS_E_ARG;
  cudaSetDevice(h->device);
  if (sort) h->recValid = false;
  rc = ensure_fof_buffers(h);
  if (rc) return rc;
  rc = diag_pass(h);   // the read-outs the books need, as the reference's analysis reads them
  if (rc) return rc;
  const int N = h->N, nb = fof_blocks(N);
  const double mref = h->sim.m, a = h->sim.a;
  const float4 *P = h->pos[h->cur], *V = h->vel[h->cur];
  // groups
  h->launches += launch_fof_groups(N, P, a, touch, spring, h->keys, h->vals, h->keysTmp, h->valsTmp, h->hist,
                                   h->fofStart, h->fofEnd, h->fofParent, h->fofSize, h->fofElastic, h->fofTop,
                                   h->status, h->st);
  std::vector<unsigned long long> top(2 * (size_t)nb);
  std::vector<double> el((size_t)nb);
  CUDA_TRY(h, cudaMemcpyAsync(top.data(), h->fofTop, 8 * top.size(), cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaMemcpyAsync(el.data(), h->fofElastic, 8 * el.size(), cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  rc = check_status(h);
  if (rc) return rc;
  unsigned long long t1 = 0, t2 = 0;
  for (unsigned long long v : top) {
    if (v > t1) { t2 = t1; t1 = v; }
    else if (v > t2 && v != t1) t2 = v;
  }
  double elastic = 0;
  for (double v : el) elastic += v;
  const int g1 = t1 ? (int)(0xFFFFFFFFu - (uint32_t)(t1 & 0xFFFFFFFFu)) : -1;
  const int g2 = t2 ? (int)(0xFFFFFFFFu - (uint32_t)(t2 & 0xFFFFFFFFu)) : -1;
  FofSumArgs base{};
  base.N = N;
  base.mref = mref;
  base.pos = P;
  base.vel = V;
  base.diag = h->diag;
  base.mat = h->mat;
  base.label = h->fofParent;
  DevGroup A, B;
  rc = fof_group(h, base, g1, A);
  if (rc) return rc;
  const bool hasB = g2 >= 0;
  if (hasB) {
    rc = fof_group(h, base, g2, B);
    if (rc) return rc;
  }
  // the planet's spin over the body proper, within 1.15 of its own radius
  const double rb = 1.15 * std::cbrt(std::max(A.impMass, A.mass - A.impMass)), rb2 = rb * rb;
  FofSumArgs pa = base;
  pa.g = g1;
  pa.r2 = rb2;
  for (int k = 0; k < 3; ++k) pa.c[k] = A.core[k];
  double t[kFofTerms];
  pa.pass = kFofProper1;
  if ((rc = fof_sum(h, pa, t))) return rc;
  const double bm = t[0];
  double bv[3] = {t[1], t[2], t[3]};
  if (bm > 0) for (int k = 0; k < 3; ++k) bv[k] /= bm;
  pa.pass = kFofProper2;
  for (int k = 0; k < 3; ++k) pa.d[k] = bv[k];
  if ((rc = fof_sum(h, pa, t))) return rc;
  const double Lx = t[0], Ly = t[1], Lz = t[2];
  const double Lm = std::sqrt(Lx * Lx + Ly * Ly + Lz * Lz);
  const double lx = Lx / (Lm + 1e-30), ly = Ly / (Lm + 1e-30), lz = Lz / (Lm + 1e-30);
  const double tilt = std::acos(std::max(-1.0, std::min(1.0, ly))) * 180 / 3.141592653589793;
  pa.pass = kFofProper3;
  pa.d[0] = lx; pa.d[1] = ly; pa.d[2] = lz;
  if ((rc = fof_sum(h, pa, t))) return rc;
  const double I = t[0];
  const double day = Lm > 1e-9 ? 2 * 3.141592653589793 * I / Lm * 805 / 3600 : INFINITY;
  // the disk: what is bound in orbit about the planet, and the Moon it makes
  FofSumArgs oa = base;
  oa.pass = kFofOrbit;
  oa.g = g1;
  oa.s0 = A.mass;
  oa.s1 = A.R;
  for (int k = 0; k < 3; ++k) { oa.c[k] = A.com[k]; oa.d[k] = A.vel[k]; }
  if ((rc = fof_sum(h, oa, t))) return rc;
  const double orbit = t[0], esc = t[1], J[3] = {t[2], t[3], t[4]};
  const double jD = orbit > 0 ? std::sqrt(J[0] * J[0] + J[1] * J[1] + J[2] * J[2]) / (orbit * std::sqrt(A.mass * 2.9)) : 0;
  const double moon = std::min(std::max(0.0, orbit * (1.9 * jD - 1.1 - 1.9 * 0.05)), 0.95 * orbit);
  std::memset(rep, 0, sizeof *rep);
  auto energy = [&](const double *x, const double *v) {
    const double r = std::sqrt((x[0] - A.com[0]) * (x[0] - A.com[0]) + (x[1] - A.com[1]) * (x[1] - A.com[1]) +
                               (x[2] - A.com[2]) * (x[2] - A.com[2]));
    const double dv2 = (v[0] - A.vel[0]) * (v[0] - A.vel[0]) + (v[1] - A.vel[1]) * (v[1] - A.vel[1]) +
                       (v[2] - A.vel[2]) * (v[2] - A.vel[2]);
    return 0.5 * dv2 - A.mass / std::max(r, A.R);
  };
  if (hasB && B.n >= std::max(8.0, N / 1000.0)) {
    const double dAB = std::sqrt((B.com[0] - A.com[0]) * (B.com[0] - A.com[0]) +
                                 (B.com[1] - A.com[1]) * (B.com[1] - A.com[1]) +
                                 (B.com[2] - A.com[2]) * (B.com[2] - A.com[2]));
    if (dAB > A.R + B.R + 2 * a) {
      rep->hasSecond = 1;
      rep->secMass = B.mass;
      rep->secDist = dAB;
      rep->secBound = energy(B.com, B.vel) < 0;
      rep->secImp = B.imp;
      rep->secIron = B.iron;
      std::memcpy(rep->secCom, B.com, sizeof B.com);
      std::memcpy(rep->secCore, B.core, sizeof B.core);
      std::memcpy(rep->secVel, B.vel, sizeof B.vel);
      rep->secR = B.R;
    }
  }
  // the books
  FofSumArgs ba = base;
  ba.pass = kFofBooks;
  if ((rc = fof_sum(h, ba, t))) return rc;
  const double Mt = t[0], p[3] = {t[1], t[2], t[3]}, Jx = t[4], Jy = t[5], Jz = t[6];
  // the loose list: beyond 1.3 radii of the planet (and of a big second body), the farthest first over the cap
  FofLooseArgs la{};
  la.N = N;
  la.pos = P;
  la.bigB = hasB && B.mass > 0.05;
  la.RA = A.R;
  la.RB = B.R;
  for (int k = 0; k < 3; ++k) { la.comA[k] = A.com[k]; la.comB[k] = B.com[k]; }
  CUDA_TRY(h, cudaMemsetAsync(h->fofNDist, 0, sizeof(int), h->st));
  h->launches += launch_fof_loose(la, 0, h->fofCounts, h->fofOffs, h->fofDist, h->fofNDist, nullptr, h->st);
  std::vector<int> counts((size_t)nb);
  CUDA_TRY(h, cudaMemcpyAsync(counts.data(), h->fofCounts, 4 * (size_t)nb, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  int nLoose = 0;
  for (int c : counts) nLoose += c;
  double least = 0;
  if (nLoose > cap) {
    std::vector<double> ds((size_t)nLoose);
    CUDA_TRY(h, cudaMemcpyAsync(ds.data(), h->fofDist, 8 * (size_t)nLoose, cudaMemcpyDeviceToHost, h->st));
    CUDA_TRY(h, cudaStreamSynchronize(h->st));
    std::nth_element(ds.begin(), ds.begin() + (nLoose - cap), ds.end());
    least = ds[(size_t)(nLoose - cap)];
  }
  const int len = std::min(nLoose, cap);
  la.len = len;
  la.least = least;
  if (len > 0) h->launches += launch_fof_loose(la, 1, h->fofCounts, h->fofOffs, nullptr, nullptr, h->fofList, h->st);
  if (sort) {   // the spatial order: a Morton key of 7 bits an axis over the largest body's box
    h->launches += launch_morton_keys(N, P, A.core[0], A.core[1], A.core[2], h->keys, h->vals, h->st);
    h->launches += launch_radix_sort(N, 21, h->keys, h->vals, h->keysTmp, h->valsTmp, h->hist, h->st);
    h->launches += launch_invert_perm(N, h->vals, h->into, h->st);
    h->launches += launch_fof_remap(len, h->into, h->fofList, h->st);
    CUDA_TRY(h, cudaMemcpyAsync(perm, h->vals, 4 * (size_t)N, cudaMemcpyDeviceToHost, h->st));
  }
  if (len > 0) CUDA_TRY(h, cudaMemcpyAsync(list, h->fofList, 4 * (size_t)len, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
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
  rep->M = Mt; rep->iron = t[10] / Mt;
  rep->drift = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) / Mt;
  rep->L = std::sqrt(Jx * Jx + Jy * Jy + Jz * Jz);
  rep->KE = t[7]; rep->PE = t[8]; rep->EL = elastic; rep->Q = t[9];
  rep->unseated = t[11] / N; rep->full = t[12] / N;
  rep->jD = jD; rep->moon = moon;
  rep->ppCount = len; rep->ppLoose = nLoose;
  return check_launch(h);
}

int ccs_diag_async(ccs_handle *h) {
  int rc = ensure_built(h);
  if (rc) return rc;
  cudaSetDevice(h->device);
  rc = diag_pass(h);
  if (rc) return rc;
  const size_t b = 16 * (size_t)h->N;
  CUDA_TRY(h, cudaMemcpyAsync(h->stageD, h->diag, b, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaMemcpyAsync(h->stageP, h->pos[h->cur], b, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaMemcpyAsync(h->stageV, h->vel[h->cur], b, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaEventRecord(h->readEv, h->st));
  h->pending = true;
  return CCS_OK;
}

int ccs_poll(ccs_handle *h, float *P, float *V, float *D) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!h->pending) {
    h->err = "no read-back pending";
    return CCS_E_STATE;
  }
  const cudaError_t q = cudaEventQuery(h->readEv);
  if (q == cudaErrorNotReady) return CCS_NOT_READY;
  if (q != cudaSuccess) {
    h->err = std::string("read-back: ") + cudaGetErrorString(q);
    return CCS_E_CUDA;
  }
  const size_t b = 16 * (size_t)h->N;
  if (P) std::memcpy(P, h->stageP, b);
  if (V) std::memcpy(V, h->stageV, b);
  if (D) std::memcpy(D, h->stageD, b);
  h->pending = false;
  return check_status(h);
}

int ccs_read_state(ccs_handle *h, float *pos4, float *vel4, float *aux4, float *q, float *mat) {
  int rc = ensure_built(h);
  if (rc) return rc;
  cudaSetDevice(h->device);
  const size_t N = (size_t)h->N;
  if (pos4) CUDA_TRY(h, cudaMemcpyAsync(pos4, h->pos[h->cur], 16 * N, cudaMemcpyDeviceToHost, h->st));
  if (vel4) CUDA_TRY(h, cudaMemcpyAsync(vel4, h->vel[h->cur], 16 * N, cudaMemcpyDeviceToHost, h->st));
  if (aux4) CUDA_TRY(h, cudaMemcpyAsync(aux4, h->aux[h->cur], 16 * N, cudaMemcpyDeviceToHost, h->st));
  if (q) CUDA_TRY(h, cudaMemcpyAsync(q, h->q[h->cur], 4 * N, cudaMemcpyDeviceToHost, h->st));
  if (mat) CUDA_TRY(h, cudaMemcpyAsync(mat, h->mat, 4 * N, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  return check_status(h);
}

int ccs_write_state(ccs_handle *h, const float *pos4, const float *vel4, const float *aux4, const float *q,
                    const float *mat) {
  int rc = ensure_built(h);
  if (rc) return rc;
  cudaSetDevice(h->device);
  h->recValid = false;
  const size_t N = (size_t)h->N;
  if (pos4) CUDA_TRY(h, cudaMemcpyAsync(h->pos[h->cur], pos4, 16 * N, cudaMemcpyHostToDevice, h->st));
  if (vel4) CUDA_TRY(h, cudaMemcpyAsync(h->vel[h->cur], vel4, 16 * N, cudaMemcpyHostToDevice, h->st));
  if (aux4) CUDA_TRY(h, cudaMemcpyAsync(h->aux[h->cur], aux4, 16 * N, cudaMemcpyHostToDevice, h->st));
  if (q) CUDA_TRY(h, cudaMemcpyAsync(h->q[h->cur], q, 4 * N, cudaMemcpyHostToDevice, h->st));
  if (mat) CUDA_TRY(h, cudaMemcpyAsync(h->mat, mat, 4 * N, cudaMemcpyHostToDevice, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  return CCS_OK;
}

int ccs_device_ptrs(ccs_handle *h, ccs_device_buffers *out) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!out) return CCS_E_ARG;
  out->pos4 = h->pos[h->cur];
  out->vel4 = h->vel[h->cur];
  out->aux4 = h->aux[h->cur];
  out->q = h->q[h->cur];
  out->mat = h->mat;
  out->home4 = h->home;
  for (int b = 0; b < 2; ++b) {
    out->force[b] = h->pm[b].force;
    out->mono[b] = h->pm[b].mono;
  }
  out->stream = (void *)h->st;
  return CCS_OK;
}

int ccs_books(ccs_handle *h, int with_diag, double out[CCS_BOOKS]) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!out) return CCS_E_ARG;
  cudaSetDevice(h->device);
  if (with_diag) {
    rc = diag_pass(h);
    if (rc) return rc;
  }
  h->launches += launch_books(h->N, h->sim.m, h->pos[h->cur], h->vel[h->cur], h->mat, h->diag, h->booksPartial,
                              h->booksOut, with_diag, h->st);
  CUDA_TRY(h, cudaMemcpyAsync(out, h->booksOut, sizeof(double) * CCS_BOOKS, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  out[10] /= h->N;
  out[11] /= h->N;
  if (!with_diag) out[8] = out[9] = out[10] = out[11] = 0.0;
  return check_launch(h);
}

int ccs_direct_sum(ccs_handle *h, const int32_t *idx, int n, double *acc3, double *pot) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (n <= 0 || !idx || !acc3 || !pot) return CCS_E_ARG;
  for (int k = 0; k < n; ++k)
    if (idx[k] < 0 || idx[k] >= h->N) {
      h->err = "direct sum: index out of range";
      return CCS_E_ARG;
    }
  cudaSetDevice(h->device);
  int32_t *dIdx = nullptr;
  double *dAcc = nullptr, *dPot = nullptr;
  if (cudaMalloc(&dIdx, 4 * (size_t)n) != cudaSuccess || cudaMalloc(&dAcc, 24 * (size_t)n) != cudaSuccess ||
      cudaMalloc(&dPot, 8 * (size_t)n) != cudaSuccess) {
    cudaFree(dIdx); cudaFree(dAcc); cudaFree(dPot);
    h->err = "direct sum: device allocation failed";
    return CCS_E_NOMEM;
  }
  cudaMemcpyAsync(dIdx, idx, 4 * (size_t)n, cudaMemcpyHostToDevice, h->st);
  h->launches += launch_direct_sum(h->N, h->pos[h->cur], h->mat, h->sim.m, h->sim.a, dIdx, n, dAcc, dPot, h->st);
  cudaMemcpyAsync(acc3, dAcc, 24 * (size_t)n, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(pot, dPot, 8 * (size_t)n, cudaMemcpyDeviceToHost, h->st);
  const cudaError_t e = cudaStreamSynchronize(h->st);
  cudaFree(dIdx); cudaFree(dAcc); cudaFree(dPot);
  if (e != cudaSuccess) {
    h->err = std::string("direct sum: ") + cudaGetErrorString(e);
    return CCS_E_CUDA;
  }
  return check_launch(h);
}

int ccs_pp_list_force(ccs_handle *h, const int32_t *list, int n, float *force4) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (n < 0 || n > h->N || (n > 0 && (!list || !force4))) return CCS_E_ARG;
  for (int k = 0; k < n; ++k)
    if (list[k] < 0 || list[k] >= h->N) {
      h->err = "pairwise list: index out of range";
      return CCS_E_ARG;
    }
  if (n == 0) return CCS_OK;
  cudaSetDevice(h->device);
  const ccs_uniforms u = pass_uniforms(h, 0, 0, 0.0);   // the boxes and constants the step's pass uses
  int32_t *dIdx = nullptr;
  float4 *dList = nullptr, *dOut = nullptr;
  float *dBox = nullptr;
  ccs_uniforms *dU = nullptr;
  if (cudaMalloc(&dIdx, sizeof(int32_t) * n) != cudaSuccess || cudaMalloc(&dList, sizeof(float4) * n) != cudaSuccess ||
      cudaMalloc(&dOut, sizeof(float4) * n) != cudaSuccess || cudaMalloc(&dBox, sizeof(float) * n) != cudaSuccess ||
      cudaMalloc(&dU, sizeof(ccs_uniforms)) != cudaSuccess) {
    cudaFree(dIdx); cudaFree(dList); cudaFree(dOut); cudaFree(dBox); cudaFree(dU);
    h->err = "pairwise list: device allocation failed";
    return CCS_E_NOMEM;
  }
  cudaMemcpyAsync(dIdx, list, sizeof(int32_t) * n, cudaMemcpyHostToDevice, h->st);
  cudaMemcpyAsync(dU, &u, sizeof u, cudaMemcpyHostToDevice, h->st);
  h->launches += launch_pp_gather(dU, h->pos[h->cur], h->mat, dIdx, n, dList, dBox, h->st);
  h->launches += launch_pp_list(u, dList, dBox, n, h->tab, dOut, h->st);
  cudaMemcpyAsync(force4, dOut, sizeof(float4) * n, cudaMemcpyDeviceToHost, h->st);
  const cudaError_t e = cudaStreamSynchronize(h->st);
  cudaFree(dIdx); cudaFree(dList); cudaFree(dOut); cudaFree(dBox); cudaFree(dU);
  if (e != cudaSuccess) {
    h->err = std::string("pairwise list: ") + cudaGetErrorString(e);
    return CCS_E_CUDA;
  }
  return check_launch(h);
}

int ccs_read_buffer(ccs_handle *h, int which, void *dst, size_t bytes) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!dst) return CCS_E_ARG;
  cudaSetDevice(h->device);
  const void *src = nullptr;
  size_t n = 0;
  const size_t N = (size_t)h->N;
  switch (which) {
    case CCS_BUF_SEATS: src = h->seats[h->seatCur]; n = 4 * h->ncell * kSeats; break;
    case CCS_BUF_FINE_A: src = h->pm[0].fine; n = 16 * (size_t)(kFine + 1); break;
    case CCS_BUF_FORCE_A: src = h->pm[0].force; n = 16 * (size_t)(kFine + 1); break;
    case CCS_BUF_MONO_A: src = h->pm[0].mono; n = 16; break;
    case CCS_BUF_COARSE_A: src = h->pm[0].coarse; n = 16 * (size_t)kCoarse; break;
    case CCS_BUF_FAR_A: src = h->pm[0].farA; n = 16 * (size_t)kCoarse; break;
    case CCS_BUF_FINE_B: src = h->pm[1].fine; n = 16 * (size_t)(kFine + 1); break;
    case CCS_BUF_FORCE_B: src = h->pm[1].force; n = 16 * (size_t)(kFine + 1); break;
    case CCS_BUF_MONO_B: src = h->pm[1].mono; n = 16; break;
    case CCS_BUF_PP_LIST: src = h->ppList; n = 16 * (size_t)CCS_PP_CAP; break;
    case CCS_BUF_PP_FORCE: src = h->ppForce; n = 64 * (size_t)CCS_PP_CAP; break;
    case CCS_BUF_PP_BOX: src = h->ppBox; n = 4 * (size_t)CCS_PP_CAP; break;
    case CCS_BUF_PP_SLOT: src = h->ppSlot; n = 4 * N; break;
    case CCS_BUF_DIAG: src = h->diag; n = 16 * N; break;
    case CCS_BUF_CELL_OF: src = h->hk[h->seatCur]; n = 4 * N; break;
    case CCS_BUF_TIDE0_A: src = h->pm[0].tide0; n = 16 * (size_t)(kFine + 1); break;
    case CCS_BUF_TIDE1_A: src = h->pm[0].tide1; n = 16 * (size_t)(kFine + 1); break;
    case CCS_BUF_PP_ALL: src = h->ppAll; n = 16 * N; break;
    case CCS_BUF_WALK_STATS: src = h->recStats; n = 12; break;
    case CCS_BUF_WALK_COUNT: src = h->recN; n = 4 * ((N + 31) / 32); break;
    case CCS_BUF_TIDE2_A: src = h->pm[0].tide2; n = 16 * 3 * (size_t)(kFine + 1); break;
    case CCS_BUF_FINEQ_A: src = h->pm[0].fineQ; n = 16 * 2 * (size_t)(kFine + 1); break;
    default: h->err = "unknown buffer"; return CCS_E_ARG;
  }
  if (!src) {
    h->err = "that buffer exists only in the stencil-split P3M (ccs_set_pp_split)";
    return CCS_E_STATE;
  }
  if (bytes != n) {
    h->err = "buffer size mismatch: expected " + std::to_string(n);
    return CCS_E_ARG;
  }
  CUDA_TRY(h, cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  return check_status(h);
}

int ccs_pass_slots(ccs_handle *h) {
  int rc = ensure_built(h);
  if (rc) return rc;
  h->recValid = false;   // passes run by hand neither record nor replay
  pass_slots(h, pass_uniforms(h, 0, 0, 0.0));
  return check_launch(h);
}

int ccs_pass_mesh(ccs_handle *h) {
  int rc = ensure_built(h);
  if (rc) return rc;
  h->recValid = false;
  set_boxes(h);
  const ccs_uniforms *U;
  rc = push_uniforms(h, pass_uniforms(h, 0, 0, 0.0), &U);
  if (rc) return rc;
  pass_mesh(h, U, h->boxB > 0.5f);
  return check_launch(h);
}

int ccs_pass_pp(ccs_handle *h) {
  int rc = ensure_built(h);
  if (rc) return rc;
  h->recValid = false;
  const ccs_uniforms *U;
  rc = push_uniforms(h, pass_uniforms(h, 0, 0, 0.0), &U);
  if (rc) return rc;
  pass_pp(h, U, h->ppCount);
  return check_launch(h);
}

int ccs_pass_sim(ccs_handle *h, int settle, int kick, double gdt) {
  int rc = ensure_built(h);
  if (rc) return rc;
  h->recValid = false;
  pass_sim(h, pass_uniforms(h, settle, kick, gdt));
  return check_launch(h);
}

int ccs_pass_diag(ccs_handle *h) {
  int rc = ensure_built(h);
  if (rc) return rc;
  return diag_pass(h);
}

// the last step of a host-buffer call: its contact step in two halves, the first half's outputs read back on
// a second stream while the second half runs (the copies over PCIe are most of such a call's time)
static int ensure_copy_stream(ccs_handle *h) {
  if (!h->cst) {
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->cst, cudaStreamNonBlocking));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->halfEv, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->copyEv, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->inEv, cudaEventDisableTiming));
  }
  return CCS_OK;
}

// inputsOnCopyStream: vel and q are still arriving on the copy stream (the grid, the mesh and the pairwise pass
// need only the positions), and the contact step waits for them
static int last_step_overlapped(ccs_handle *h, float *pos4_out, float *vel4_out, float *aux4_out, float *q_out,
                                bool inputsOnCopyStream) {
  int rc = ensure_copy_stream(h);
  if (rc) return rc;
  StepPlan p = plan_step(h, 0, 0);
  rc = step_graph(h, p, true);   // the grid, the mesh and the pairwise pass
  if (rc) return rc;
  if (inputsOnCopyStream) CUDA_TRY(h, cudaStreamWaitEvent(h->st, h->inEv, 0));
  SimArgs a = sim_args(h);
  a.walk = p.walk;
  const int N = h->N, half = std::min(N, (N / 2 + 255) / 256 * 256), d = h->cur ^ 1;
  h->launches += launch_simulate_range(p.u, N, a, h->st, h->tuneWarps, h->field, 0, half);
  CUDA_TRY(h, cudaEventRecord(h->halfEv, h->st));
  h->launches += launch_simulate_range(p.u, N, a, h->st, h->tuneWarps, h->field, half, N - half);
  CUDA_TRY(h, cudaStreamWaitEvent(h->cst, h->halfEv, 0));
  auto read = [&](cudaStream_t st, int i0, int n) -> int {
    if (n <= 0) return CCS_OK;
    const size_t o4 = 4 * (size_t)i0, b4 = 16 * (size_t)n;
    if (pos4_out) CUDA_TRY(h, cudaMemcpyAsync(pos4_out + o4, h->pos[d] + i0, b4, cudaMemcpyDeviceToHost, st));
    if (vel4_out) CUDA_TRY(h, cudaMemcpyAsync(vel4_out + o4, h->vel[d] + i0, b4, cudaMemcpyDeviceToHost, st));
    if (aux4_out) CUDA_TRY(h, cudaMemcpyAsync(aux4_out + o4, h->aux[d] + i0, b4, cudaMemcpyDeviceToHost, st));
    if (q_out) CUDA_TRY(h, cudaMemcpyAsync(q_out + i0, h->q[d] + i0, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    return CCS_OK;
  };
  if ((rc = read(h->cst, 0, half))) return rc;
  if ((rc = read(h->st, half, N - half))) return rc;
  CUDA_TRY(h, cudaEventRecord(h->copyEv, h->cst));
  CUDA_TRY(h, cudaStreamWaitEvent(h->st, h->copyEv, 0));
  h->cur = d;
  h->sim.t += h->sim.dt;   // the frame loop's clock, as ccs_steps keeps it
  return CCS_OK;
}

int ccs_advance_host(ccs_handle *h, const float *pos4, const float *vel4, const float *q, int nsteps, float *pos4_out,
                     float *vel4_out, float *aux4_out, float *q_out) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (nsteps < 0) return CCS_E_ARG;
  cudaSetDevice(h->device);
  if (pos4 || vel4 || q) h->recValid = false;   // a new state: nothing recorded for it
  const size_t N = (size_t)h->N;
  const bool reads = pos4_out || vel4_out || aux4_out || q_out;
  const bool overlapped = nsteps > 0 && reads && h->useGraphs && h->timing == 0 && !h->ppSplit;
  // a one-step call: velocities and heat come over on the copy stream while the step's grid and mesh run
  const bool split = overlapped && nsteps == 1;
  if (split && (rc = ensure_copy_stream(h))) return rc;
  if (split) CUDA_TRY(h, cudaEventRecord(h->inEv, h->st));   // the copy stream starts after what came before
  if (split) CUDA_TRY(h, cudaStreamWaitEvent(h->cst, h->inEv, 0));
  cudaStream_t vs = split ? h->cst : h->st;
  if (pos4) CUDA_TRY(h, cudaMemcpyAsync(h->pos[h->cur], pos4, 16 * N, cudaMemcpyHostToDevice, h->st));
  if (vel4) CUDA_TRY(h, cudaMemcpyAsync(h->vel[h->cur], vel4, 16 * N, cudaMemcpyHostToDevice, vs));
  if (q) CUDA_TRY(h, cudaMemcpyAsync(h->q[h->cur], q, 4 * N, cudaMemcpyHostToDevice, vs));
  if (split) CUDA_TRY(h, cudaEventRecord(h->inEv, h->cst));
  if (overlapped) {
    rc = ccs_steps(h, nsteps - 1);
    if (rc) return rc;
    rc = last_step_overlapped(h, pos4_out, vel4_out, aux4_out, q_out, split);
    if (rc) return rc;
    CUDA_TRY(h, cudaStreamSynchronize(h->st));
    return check_launch(h);
  }
  rc = ccs_steps(h, nsteps);
  if (rc) return rc;
  if (pos4_out) CUDA_TRY(h, cudaMemcpyAsync(pos4_out, h->pos[h->cur], 16 * N, cudaMemcpyDeviceToHost, h->st));
  if (vel4_out) CUDA_TRY(h, cudaMemcpyAsync(vel4_out, h->vel[h->cur], 16 * N, cudaMemcpyDeviceToHost, h->st));
  if (aux4_out) CUDA_TRY(h, cudaMemcpyAsync(aux4_out, h->aux[h->cur], 16 * N, cudaMemcpyDeviceToHost, h->st));
  if (q_out) CUDA_TRY(h, cudaMemcpyAsync(q_out, h->q[h->cur], 4 * N, cudaMemcpyDeviceToHost, h->st));
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  return check_launch(h);
}

// ---- checkpoint and restore ----
namespace {
// CRC-32 (IEEE 802.3: reflected polynomial 0xEDB88320, initial and final 0xFFFFFFFF), byte-table driven
uint64_t crc32(const unsigned char *p, size_t n) {
  static uint32_t table[256];
  static std::once_flag once;
  std::call_once(once, [] {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      table[i] = c;
    }
  });
  uint32_t c = 0xFFFFFFFFu;
  for (size_t i = 0; i < n; ++i) c = table[(c ^ p[i]) & 0xFFu] ^ (c >> 8);
  return c ^ 0xFFFFFFFFu;
}
size_t ckpt_payload(int N, int pp, size_t extra) {
  return sizeof(ccs_sim) + (size_t)N * (16 + 16 + 16 + 4 + 4 + 16) + 4 * (size_t)pp + extra;
}
bool ckpt_boundary(const ccs_handle *h) {
  return h->field ? h->sim.stepNo % 2 == 0 : h->sim.stepNo % h->meshEvery == 0;
}
}  // namespace

int ccs_checkpoint_size(ccs_handle *h, size_t extraBytes, size_t *bytes) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!bytes) return CCS_E_ARG;
  *bytes = sizeof(ccs_checkpoint_header) + ckpt_payload(h->N, h->ppCount, extraBytes);
  return CCS_OK;
}

int ccs_checkpoint_save(ccs_handle *h, const void *extra, size_t extraBytes, void *buf, size_t cap) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!buf || (extraBytes && !extra)) return CCS_E_ARG;
  const size_t N = (size_t)h->N, total = sizeof(ccs_checkpoint_header) + ckpt_payload(h->N, h->ppCount, extraBytes);
  if (cap < total) {
    h->err = "checkpoint buffer too small (ccs_checkpoint_size)";
    return CCS_E_ARG;
  }
  if (!ckpt_boundary(h)) {
    h->err = "a checkpoint is taken where the next step rebuilds the grid and the mesh (stepNo % meshEvery == 0)";
    return CCS_E_STATE;
  }
  cudaSetDevice(h->device);
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  ccs_checkpoint_header hd;
  std::memset(&hd, 0, sizeof hd);
  std::memcpy(hd.magic, CCS_CKPT_MAGIC, 8);
  hd.version = CCS_CKPT_VERSION;
  hd.headerBytes = sizeof hd;
  hd.simBytes = sizeof(ccs_sim);
  hd.flags = h->field ? 2u : 0u;
  hd.N = h->N;
  hd.meshEvery = h->meshEvery;
  hd.ppCount = h->ppCount;
  hd.ppLoose = h->ppLoose;
  for (int k = 0; k < 3; ++k) hd.field[k] = h->gField[k];
  hd.field[3] = h->frozen;
  hd.field[4] = h->fieldInvM;
  hd.field[5] = h->fieldCpIron;
  CUDA_TRY(h, cudaMemcpy(hd.monoA, h->pm[0].mono, 16, cudaMemcpyDeviceToHost));
  CUDA_TRY(h, cudaMemcpy(hd.monoB, h->pm[1].mono, 16, cudaMemcpyDeviceToHost));
  hd.extraBytes = extraBytes;
  hd.payloadBytes = total - sizeof hd;
  unsigned char *p = static_cast<unsigned char *>(buf) + sizeof hd, *p0 = p;
  std::memcpy(p, &h->sim, sizeof(ccs_sim));
  p += sizeof(ccs_sim);
  const int c = h->cur;
  CUDA_TRY(h, cudaMemcpy(p, h->pos[c], 16 * N, cudaMemcpyDeviceToHost)); p += 16 * N;
  CUDA_TRY(h, cudaMemcpy(p, h->vel[c], 16 * N, cudaMemcpyDeviceToHost)); p += 16 * N;
  CUDA_TRY(h, cudaMemcpy(p, h->aux[c], 16 * N, cudaMemcpyDeviceToHost)); p += 16 * N;
  CUDA_TRY(h, cudaMemcpy(p, h->q[c], 4 * N, cudaMemcpyDeviceToHost)); p += 4 * N;
  CUDA_TRY(h, cudaMemcpy(p, h->mat, 4 * N, cudaMemcpyDeviceToHost)); p += 4 * N;
  CUDA_TRY(h, cudaMemcpy(p, h->home, 16 * N, cudaMemcpyDeviceToHost)); p += 16 * N;
  if (h->ppCount) CUDA_TRY(h, cudaMemcpy(p, h->ppIndex, 4 * (size_t)h->ppCount, cudaMemcpyDeviceToHost));
  p += 4 * (size_t)h->ppCount;
  if (extraBytes) std::memcpy(p, extra, extraBytes);
  p += extraBytes;
  hd.checksum = crc32(p0, (size_t)(p - p0));
  std::memcpy(buf, &hd, sizeof hd);
  return CCS_OK;
}

int ccs_checkpoint_load(ccs_handle *h, const void *buf, size_t bytes) {
  if (!h || !buf) return CCS_E_ARG;
  h->recValid = false;
  ccs_checkpoint_header hd;
  if (bytes < sizeof hd) {
    h->err = "checkpoint: shorter than its header";
    return CCS_E_ARG;
  }
  std::memcpy(&hd, buf, sizeof hd);
  if (std::memcmp(hd.magic, CCS_CKPT_MAGIC, 8) != 0 || hd.version != CCS_CKPT_VERSION ||
      hd.headerBytes != sizeof hd || hd.simBytes != sizeof(ccs_sim)) {
    h->err = "checkpoint: not a version-1 checkpoint of this library's layout";
    return CCS_E_ARG;
  }
  if (hd.N <= 0 || hd.N > CCS_MAX_N || hd.ppCount < 0 || hd.ppCount > CCS_PP_CAP || hd.meshEvery < 1 ||
      hd.meshEvery > kMaxBlock || hd.payloadBytes != ckpt_payload(hd.N, hd.ppCount, hd.extraBytes) ||
      bytes < sizeof hd + hd.payloadBytes) {
    h->err = "checkpoint: sizes do not add up";
    return CCS_E_ARG;
  }
  const unsigned char *p = static_cast<const unsigned char *>(buf) + sizeof hd;
  if (crc32(p, hd.payloadBytes) != hd.checksum) {
    h->err = "checkpoint: checksum mismatch";
    return CCS_E_ARG;
  }
  ccs_sim sim;
  std::memcpy(&sim, p, sizeof sim);
  if (sim.N != hd.N) {
    h->err = "checkpoint: sizes do not add up";
    return CCS_E_ARG;
  }
  const size_t N = (size_t)hd.N;
  // the arrays are copied out of the (possibly unaligned) buffer before they are used
  std::vector<float> pos(4 * N), vel(4 * N), aux(4 * N), q(N), mat(N), home(4 * N);
  std::vector<int32_t> list((size_t)hd.ppCount);
  const unsigned char *a = p + sizeof sim;
  std::memcpy(pos.data(), a, 16 * N); a += 16 * N;
  std::memcpy(vel.data(), a, 16 * N); a += 16 * N;
  std::memcpy(aux.data(), a, 16 * N); a += 16 * N;
  std::memcpy(q.data(), a, 4 * N); a += 4 * N;
  std::memcpy(mat.data(), a, 4 * N); a += 4 * N;
  std::memcpy(home.data(), a, 16 * N); a += 16 * N;
  if (hd.ppCount) std::memcpy(list.data(), a, 4 * (size_t)hd.ppCount);
  int rc = ccs_build(h, &sim, pos.data(), vel.data(), mat.data(), home.data());
  if (rc) return rc;
  rc = ccs_write_state(h, nullptr, nullptr, aux.data(), q.data(), nullptr);
  if (rc) return rc;
  h->meshEvery = hd.meshEvery;
  rc = ccs_set_field(h, (hd.flags & 2u) != 0, hd.field, hd.field[3], hd.field[4] > 0 ? hd.field[4] : 1.0,
                     hd.field[5] > 0 ? hd.field[5] : 1.0);
  if (rc) return rc;
  if ((rc = ccs_prime_mono(h, 0, hd.monoA)) || (rc = ccs_prime_mono(h, 1, hd.monoB))) return rc;
  return ccs_set_pp(h, list.data(), hd.ppCount, hd.ppLoose);
}

int ccs_sync(ccs_handle *h) {
  if (!h) return CCS_E_ARG;
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  int rc = check_launch(h);
  return rc ? rc : (h->built ? check_status(h) : CCS_OK);
}

int ccs_contact_pairs(ccs_handle *h, int cap, int32_t *counts, uint32_t *pairs) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (cap < 1 || cap > 1024 || !counts || !pairs) return CCS_E_ARG;
  cudaSetDevice(h->device);
  const size_t N = (size_t)h->N;
  uint32_t *dp = nullptr;
  rc = dev_alloc(h, &dp, N * (size_t)cap);
  if (rc) return rc;
  SimArgs a = sim_args(h);   // the current state in, the spare buffers out (the run does not advance)
  a.walk = step_walk(h, false);   // the walk the next step runs when it does not rebuild the grid
  a.pairs = dp;
  a.pairCap = cap;
  CUDA_TRY(h, cudaMemsetAsync(dp, 0xFF, sizeof(uint32_t) * N * (size_t)cap, h->st));
  h->launches += launch_contact_pairs(pass_uniforms(h, 0, 0, 0.0), h->N, a, h->st);
  std::vector<float4> aux(N);
  cudaError_t e = cudaMemcpyAsync(pairs, dp, sizeof(uint32_t) * N * (size_t)cap, cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(aux.data(), a.auxO, sizeof(float4) * N, cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(dp);
  if (e != cudaSuccess) {
    h->err = std::string("ccs_contact_pairs: ") + cudaGetErrorString(e);
    return CCS_E_CUDA;
  }
  for (size_t i = 0; i < N; ++i) counts[i] = (int32_t)aux[i].w;
  return check_launch(h);
}

int ccs_set_pp_split(ccs_handle *h, int S) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (S < 0 || S > 3) {
    h->err = "ccs_set_pp_split: the stencil is 0 (off) or 1..3 mesh cells";
    return CCS_E_ARG;
  }
  if (S == h->ppSplit) return CCS_OK;
  cudaSetDevice(h->device);
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  free_graphs(h);   // captured steps hold the other form's kernels
  if (S) {
    rc = ensure_split_buffers(h);
    if (rc) return rc;
    CUDA_TRY(h, cudaStreamSynchronize(h->st));
  }
  h->ppSplit = S;
  return CCS_OK;
}

int ccs_pp_split_pairs(ccs_handle *h, uint64_t counts[2]) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (!counts) return CCS_E_ARG;
  if (!h->splitWork) return CCS_E_STATE;
  cudaSetDevice(h->device);
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  CUDA_TRY(h, cudaMemcpy(counts, split_pair_counts(h->splitWork), 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return CCS_OK;
}

int ccs_set_pp_split_sym(ccs_handle *h, int minNode) {
  int rc = ensure_built(h);
  if (rc) return rc;
  if (minNode < 0 || (minNode > 0 && minNode < kSymMinNode)) {
    h->err = "ccs_set_pp_split_sym: 0 (every pair one way) or at least 16 particles a node";
    return CCS_E_ARG;
  }
  if (minNode == h->splitSymMin) return CCS_OK;
  cudaSetDevice(h->device);
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  free_graphs(h);   // captured pair passes hold the threshold as an argument
  h->splitSymMin = minNode;
  return CCS_OK;
}

int ccs_set_graphs(ccs_handle *h, int on) {
  if (!h || (on != 0 && on != 1)) return CCS_E_ARG;
  h->useGraphs = on != 0;
  return CCS_OK;
}

int ccs_set_contact_walk(ccs_handle *h, int mode) {
  if (!h || mode < 0 || mode > 2) return CCS_E_ARG;
  if (mode == h->walkMode) return CCS_OK;
  cudaSetDevice(h->device);
  CUDA_TRY(h, cudaStreamSynchronize(h->st));
  free_graphs(h);   // captured steps hold the other walk's kernels and arguments
  h->walkMode = mode;
  h->recValid = false;
  if (mode == 2 && h->recStats) CUDA_TRY(h, cudaMemsetAsync(h->recStats, 0, 3 * sizeof(unsigned), h->st));
  return CCS_OK;
}

int ccs_timing_every(ccs_handle *h, int every) {
  if (!h || every < 1) return CCS_E_ARG;
  h->timingEvery = every;
  h->timingSeq = 0;
  return CCS_OK;
}

int ccs_timing(ccs_handle *h, int enable) {
  if (!h) return CCS_E_ARG;
  time_collect(h);
  h->timing = enable & ((1 << kTimedKernels) - 1);
  h->timingSeq = 0;
  for (int k = 0; k < kTimedKernels; ++k) {
    h->tAcc[k] = 0;
    h->tCount[k] = 0;
  }
  return CCS_OK;
}

int ccs_timing_read(ccs_handle *h, int kernel, double *total_ms, int *launches) {
  if (!h || kernel < 0 || kernel >= kTimedKernels || !total_ms || !launches) return CCS_E_ARG;
  time_collect(h);
  *total_ms = h->tAcc[kernel];
  *launches = h->tCount[kernel];
  return CCS_OK;
}

int64_t ccs_launch_count(ccs_handle *h) { return h ? h->launches : -1; }

}  // extern "C"
