/*
 * ccstep_napi.c -- the Node-API binding of libccstep: the calls the reference's engine object CC.nbody
 * (src/nbody.js:1095-1118) needs, one JavaScript function per C-ABI entry point, so that nbody_b200.js can
 * keep src/nbody.js's shape with the GL passes replaced.  Node-API version 8; built by binding.gyp where
 * node's headers exist.
 *
 * Conventions: a run is an external value wrapping its ccs_handle (destroyed with it); particle arrays are
 * Float32Array / Int32Array views the caller owns (N x 4 for pos/vel/aux/home, N for mat/q); the run's
 * scalars (`sim`) and the analysis report cross as plain objects; a negative status throws an Error
 * carrying ccs_last_error's text, so no status needs checking on the JavaScript side; CCS_NOT_READY comes
 * back as the number 1 (poll).
 */
#include <node_api.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ccstep.h"

#define MAXARGS 10

typedef struct {
  napi_value argv[MAXARGS];
  size_t argc;
} args_t;

static int get_args(napi_env env, napi_callback_info info, args_t *a) {
  a->argc = MAXARGS;
  return napi_get_cb_info(env, info, &a->argc, a->argv, NULL, NULL) == napi_ok;
}

static napi_value throw_rc(napi_env env, ccs_handle *h, int rc, const char *what) {
  char msg[512];
  const char *detail = h ? ccs_last_error(h) : "";
  snprintf(msg, sizeof msg, "%s failed (%d): %s", what, rc, detail ? detail : "");
  napi_throw_error(env, NULL, msg);
  return NULL;
}

static napi_value num(napi_env env, double v) {
  napi_value r;
  napi_create_double(env, v, &r);
  return r;
}

static napi_value status(napi_env env, ccs_handle *h, int rc, const char *what) {
  if (rc < 0) return throw_rc(env, h, rc, what);
  return num(env, rc);
}

static ccs_handle *handle_of(napi_env env, napi_value v) {
  void *p = NULL;
  if (napi_get_value_external(env, v, &p) != napi_ok) napi_throw_type_error(env, NULL, "not a ccstep run");
  return (ccs_handle *)p;
}

static double get_f64(napi_env env, napi_value v) {
  double d = 0;
  napi_get_value_double(env, v, &d);
  return d;
}

static int get_i32(napi_env env, napi_value v) {
  int32_t i = 0;
  napi_get_value_int32(env, v, &i);
  return i;
}

static int get_bool(napi_env env, napi_value v) {
  bool b = false;
  if (napi_get_value_bool(env, v, &b) != napi_ok) return get_i32(env, v) != 0;
  return b;
}

/* a typed array's data (NULL for null/undefined), with its element count */
static void *typed(napi_env env, napi_value v, size_t *len) {
  napi_valuetype t;
  napi_typeof(env, v, &t);
  if (len) *len = 0;
  if (t == napi_null || t == napi_undefined) return NULL;
  napi_typedarray_type tt;
  size_t n = 0, off = 0;
  void *data = NULL;
  napi_value ab;
  if (napi_get_typedarray_info(env, v, &tt, &n, &data, &ab, &off) != napi_ok) {
    napi_throw_type_error(env, NULL, "expected a typed array");
    return NULL;
  }
  if (len) *len = n;
  return data;
}

static napi_value new_typed(napi_env env, napi_typedarray_type t, size_t n, size_t elem, void **data) {
  napi_value ab, arr;
  napi_create_arraybuffer(env, n * elem, data, &ab);
  napi_create_typedarray(env, t, n, ab, 0, &arr);
  return arr;
}

static napi_value prop(napi_env env, napi_value obj, const char *name) {
  napi_value v;
  napi_get_named_property(env, obj, name, &v);
  return v;
}

static void set_num(napi_env env, napi_value obj, const char *name, double v) {
  napi_set_named_property(env, obj, name, num(env, v));
}

static void set_vec(napi_env env, napi_value obj, const char *name, const double *v, int n) {
  napi_value arr;
  napi_create_array_with_length(env, n, &arr);
  for (int k = 0; k < n; ++k) napi_set_element(env, arr, k, num(env, v[k]));
  napi_set_named_property(env, obj, name, arr);
}

static void get_vec(napi_env env, napi_value obj, const char *name, double *v, int n) {
  napi_value arr = prop(env, obj, name), e;
  napi_valuetype t;
  napi_typeof(env, arr, &t);
  if (t != napi_object) return;
  for (int k = 0; k < n; ++k) {
    napi_get_element(env, arr, k, &e);
    v[k] = get_f64(env, e);
  }
}

/* ---- the run's scalars (the reference's `sim`, src/nbody.js:212-234) as a plain object ---- */
#define SIM_INTS(X) X(N) X(W) X(H) X(n1) X(n2) X(G) X(settleLeft) X(settleTotal) X(stepNo) X(soft) X(phase)
#define SIM_DBLS(X) X(m) X(a) X(cell) X(dt) X(k) X(c) X(creep) X(damp) X(tK) X(kappa) X(R1) X(R2) X(Re1) X(Re2) \
  X(M1) X(M2) X(M) X(vc) X(vesc) X(t) X(impactT)
#define SIM_VECS(X) X(spin0) X(spin1) X(cen0) X(cen1) X(bulk0) X(bulk1) X(relr) X(relv)

static napi_value sim_to_obj(napi_env env, const ccs_sim *s) {
  napi_value o;
  napi_create_object(env, &o);
#define PUT(f) set_num(env, o, #f, s->f);
  SIM_INTS(PUT) SIM_DBLS(PUT)
#undef PUT
#define PUTV(f) set_vec(env, o, #f, s->f, 3);
  SIM_VECS(PUTV)
#undef PUTV
  napi_value boxes;
  napi_create_array_with_length(env, 2, &boxes);
  for (int b = 0; b < 2; ++b) {   /* sim.boxes[b] = {on, cen, vel, t} */
    napi_value x;
    napi_create_object(env, &x);
    napi_value on;
    napi_get_boolean(env, s->boxOn[b] != 0, &on);
    napi_set_named_property(env, x, "on", on);
    set_vec(env, x, "cen", s->boxCen[b], 3);
    set_vec(env, x, "vel", s->boxVel[b], 3);
    set_num(env, x, "t", s->boxT[b]);
    napi_set_element(env, boxes, b, x);
  }
  napi_set_named_property(env, o, "boxes", boxes);
  return o;
}

static void obj_to_sim(napi_env env, napi_value o, ccs_sim *s) {
#define GETI(f) s->f = get_i32(env, prop(env, o, #f));
#define GETD(f) s->f = get_f64(env, prop(env, o, #f));
  SIM_INTS(GETI) SIM_DBLS(GETD)
#undef GETI
#undef GETD
#define GETV(f) get_vec(env, o, #f, s->f, 3);
  SIM_VECS(GETV)
#undef GETV
  napi_value boxes = prop(env, o, "boxes"), x;
  napi_valuetype t;
  napi_typeof(env, boxes, &t);
  if (t != napi_object) return;
  for (int b = 0; b < 2; ++b) {
    napi_get_element(env, boxes, b, &x);
    s->boxOn[b] = get_bool(env, prop(env, x, "on"));
    get_vec(env, x, "cen", s->boxCen[b], 3);
    get_vec(env, x, "vel", s->boxVel[b], 3);
    s->boxT[b] = get_f64(env, prop(env, x, "t"));
  }
}

/* ---- the analysis report (fof's, src/nbody.js:888-892) ---- */
#define REP_DBLS(X) X(largest) X(largestImp) X(largestIron) X(day) X(tilt) X(orbit) X(escape) X(secMass) X(secDist) \
  X(secImp) X(secIron) X(secR) X(R) X(Redge) X(Tsurf) X(hotR) X(impMass) X(impRms) X(M) X(iron) X(drift) X(L) X(KE) \
  X(PE) X(EL) X(Q) X(unseated) X(full) X(jD) X(moon)
#define REP_VECS(X) X(axis) X(bodyVel) X(secCom) X(secCore) X(secVel) X(com) X(core) X(vel) X(hotCom) X(impCom)

static napi_value report_to_obj(napi_env env, const ccs_report *r) {
  napi_value o;
  napi_create_object(env, &o);
#define PUT(f) set_num(env, o, #f, r->f);
  REP_DBLS(PUT)
#undef PUT
#define PUTV(f) set_vec(env, o, #f, r->f, 3);
  REP_VECS(PUTV)
#undef PUTV
  set_num(env, o, "hasSecond", r->hasSecond);
  set_num(env, o, "secBound", r->secBound);
  set_num(env, o, "ppCount", r->ppCount);
  set_num(env, o, "ppLoose", r->ppLoose);
  return o;
}

/* ---- lifecycle: CC.nbody.init ---- */
static void finalize_run(napi_env env, void *data, void *hint) {
  (void)env;
  (void)hint;
  ccs_destroy((ccs_handle *)data);
}

static napi_value Create(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = NULL;
  int rc = ccs_create(a.argc > 0 ? get_i32(env, a.argv[0]) : 0, &h);
  if (rc < 0) return throw_rc(env, h, rc, "ccs_create");
  napi_value ext;
  napi_create_external(env, h, finalize_run, NULL, &ext);
  return ext;
}

/* makeBodies(opt) -> {sim, pos, vel, mat, home}: build(opt)'s initial conditions (src/nbody.js:114-250) */
static napi_value MakeBodies(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  napi_value o = a.argv[0];
  ccs_build_opt opt;
  memset(&opt, 0, sizeof opt);
  opt.N = get_i32(env, prop(env, o, "N"));
#define GETO(f) opt.f = get_f64(env, prop(env, o, #f));
  GETO(q) GETO(dens) GETO(core) GETO(spin0) GETO(spin1) GETO(angle) GETO(incl) GETO(vfac) GETO(rest) GETO(mImp)
  GETO(mTarget) GETO(rhoR) GETO(rhoCrust) GETO(crustFrac)
#undef GETO
  napi_value ci = prop(env, o, "coreImp");
  napi_valuetype t;
  napi_typeof(env, ci, &t);
  opt.coreImp = t == napi_number ? get_f64(env, ci) : -1.0;
  opt.n2 = get_i32(env, prop(env, o, "n2"));
  if (opt.N <= 0 || opt.N > CCS_MAX_N) {
    napi_throw_range_error(env, NULL, "N must be in 1..262144");
    return NULL;
  }
  void *pos, *vel, *mat, *home;
  napi_value P = new_typed(env, napi_float32_array, 4 * (size_t)opt.N, 4, &pos);
  napi_value V = new_typed(env, napi_float32_array, 4 * (size_t)opt.N, 4, &vel);
  napi_value M = new_typed(env, napi_float32_array, (size_t)opt.N, 4, &mat);
  napi_value Hm = new_typed(env, napi_float32_array, 4 * (size_t)opt.N, 4, &home);
  ccs_sim sim;
  int rc = ccs_make_bodies(&opt, &sim, (float *)pos, (float *)vel, (float *)mat, (float *)home);
  if (rc < 0) return throw_rc(env, NULL, rc, "ccs_make_bodies");
  napi_value out;
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "sim", sim_to_obj(env, &sim));
  napi_set_named_property(env, out, "pos", P);
  napi_set_named_property(env, out, "vel", V);
  napi_set_named_property(env, out, "mat", M);
  napi_set_named_property(env, out, "home", Hm);
  return out;
}

/* build(h, sim, pos, vel, mat, home?): the texture uploads and setStaticUniforms (src/nbody.js:208-249) */
static napi_value Build(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  ccs_sim sim;
  memset(&sim, 0, sizeof sim);
  obj_to_sim(env, a.argv[1], &sim);
  size_t np, nv, nm;
  float *pos = typed(env, a.argv[2], &np), *vel = typed(env, a.argv[3], &nv), *mat = typed(env, a.argv[4], &nm);
  float *home = a.argc > 5 ? typed(env, a.argv[5], NULL) : NULL;
  if (!pos || !vel || !mat || np != 4 * (size_t)sim.N || nv != np || nm != (size_t)sim.N) {
    napi_throw_range_error(env, NULL, "build: pos/vel must be N x 4 and mat N floats");
    return NULL;
  }
  return status(env, h, ccs_build(h, &sim, pos, vel, mat, home), "ccs_build");
}

/* getSim(h) -> object; setSim(h, object) writes the live scalars back (the page's sim.t += sim.dt) */
static napi_value GetSim(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_sim *s = ccs_sim_ptr(handle_of(env, a.argv[0]));
  if (!s) return NULL;
  return sim_to_obj(env, s);
}
static napi_value SetSim(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_sim *s = ccs_sim_ptr(handle_of(env, a.argv[0]));
  if (s) obj_to_sim(env, a.argv[1], s);
  return NULL;
}

#define SIMPLE(Name, call, what)                                   \
  static napi_value Name(napi_env env, napi_callback_info info) {  \
    args_t a;                                                      \
    get_args(env, info, &a);                                       \
    ccs_handle *h = handle_of(env, a.argv[0]);                     \
    return status(env, h, call, what);                             \
  }

SIMPLE(SetStatic, ccs_set_static(h), "ccs_set_static")
SIMPLE(Step, ccs_step(h, get_bool(env, a.argv[1]), get_bool(env, a.argv[2])), "ccs_step")
SIMPLE(Steps, ccs_steps(h, get_i32(env, a.argv[1])), "ccs_steps")
SIMPLE(SettleSome, ccs_settle_some(h, get_i32(env, a.argv[1])), "ccs_settle_some")
SIMPLE(RigidStep, ccs_rigid_step(h, get_f64(env, a.argv[1])), "ccs_rigid_step")
SIMPLE(SetMeshEvery, ccs_set_mesh_every(h, get_i32(env, a.argv[1])), "ccs_set_mesh_every")
SIMPLE(SetPPSplit, ccs_set_pp_split(h, get_i32(env, a.argv[1])), "ccs_set_pp_split")
SIMPLE(SetPPSplitSym, ccs_set_pp_split_sym(h, get_i32(env, a.argv[1])), "ccs_set_pp_split_sym")
SIMPLE(SetContactWalk, ccs_set_contact_walk(h, get_i32(env, a.argv[1])), "ccs_set_contact_walk")
SIMPLE(DiagAsync, ccs_diag_async(h), "ccs_diag_async")
SIMPLE(PassSlots, ccs_pass_slots(h), "ccs_pass_slots")
SIMPLE(PassMesh, ccs_pass_mesh(h), "ccs_pass_mesh")
SIMPLE(PassPP, ccs_pass_pp(h), "ccs_pass_pp")
SIMPLE(PassSim, ccs_pass_sim(h, get_bool(env, a.argv[1]), get_bool(env, a.argv[2]), get_f64(env, a.argv[3])),
       "ccs_pass_sim")
SIMPLE(PassDiag, ccs_pass_diag(h), "ccs_pass_diag")
SIMPLE(Sync, ccs_sync(h), "ccs_sync")

/* setPP(h, Int32Array list, loose): the loose list, then its pairwise pass (src/nbody.js:957-966) */
static napi_value SetPP(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  size_t n = 0;
  int32_t *list = typed(env, a.argv[1], &n);
  return status(env, h, ccs_set_pp(h, list, (int)n, a.argc > 2 ? get_i32(env, a.argv[2]) : (int)n), "ccs_set_pp");
}

/* setBoxes(h, [box0, box1]), box = {on, cen[3], vel[3], t, mono?[4]}: placeBoxes (src/nbody.js:361-374) */
static napi_value SetBoxes(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  ccs_box boxes[2];
  memset(boxes, 0, sizeof boxes);
  for (int b = 0; b < 2; ++b) {
    napi_value x, mono;
    napi_get_element(env, a.argv[1], b, &x);
    boxes[b].on = get_bool(env, prop(env, x, "on"));
    get_vec(env, x, "cen", boxes[b].cen, 3);
    get_vec(env, x, "vel", boxes[b].vel, 3);
    boxes[b].t = get_f64(env, prop(env, x, "t"));
    mono = prop(env, x, "mono");
    napi_valuetype t;
    napi_typeof(env, mono, &t);
    if (t == napi_object) {
      double m[4] = {0, 0, 0, 0};
      get_vec(env, x, "mono", m, 4);
      boxes[b].primeMono = 1;
      for (int k = 0; k < 4; ++k) boxes[b].mono[k] = (float)m[k];
    }
  }
  return status(env, h, ccs_set_boxes(h, boxes), "ccs_set_boxes");
}

/* applyPerm(h, Int32Array perm): PERM_FS and a fresh grid (src/nbody.js:932-954) */
static napi_value ApplyPerm(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  return status(env, h, ccs_apply_perm(h, typed(env, a.argv[1], NULL)), "ccs_apply_perm");
}

/* sortMorton(h, core[3]) -> {perm, into}: the analysis's Morton order (src/nbody.js:871-887) on the device */
static napi_value SortMorton(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  napi_value holder;
  napi_create_object(env, &holder);
  napi_set_named_property(env, holder, "c", a.argv[1]);
  double core[3] = {0, 0, 0};
  get_vec(env, holder, "c", core, 3);
  const int N = ccs_sim_ptr(h)->N;
  void *perm, *into;
  napi_value P = new_typed(env, napi_int32_array, (size_t)N, 4, &perm);
  napi_value I = new_typed(env, napi_int32_array, (size_t)N, 4, &into);
  int rc = ccs_sort_morton(h, core, (int32_t *)perm, (int32_t *)into);
  if (rc < 0) return throw_rc(env, h, rc, "ccs_sort_morton");
  napi_value out;
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "perm", P);
  napi_set_named_property(env, out, "into", I);
  return out;
}

/* poll(h, P, V, D) -> 0 landed, 1 not yet (collect()'s fence poll, src/nbody.js:1011-1013) */
static napi_value Poll(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  return status(env, h, ccs_poll(h, typed(env, a.argv[1], NULL), typed(env, a.argv[2], NULL),
                                  typed(env, a.argv[3], NULL)), "ccs_poll");
}

/* fof(N, mref, a, P, V, R, D, spring, touch, cap, sort) -> {report, list, perm}: the worker's analysis */
static napi_value Fof(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  const int N = get_i32(env, a.argv[0]), cap = get_i32(env, a.argv[9]), sort = get_bool(env, a.argv[10]);
  ccs_report rep;
  void *list, *perm = NULL;
  napi_value L = new_typed(env, napi_int32_array, (size_t)(cap > 0 ? cap : 1), 4, &list);
  napi_value Pm;
  napi_get_null(env, &Pm);
  if (sort) Pm = new_typed(env, napi_int32_array, (size_t)N, 4, &perm);
  int rc = ccs_fof(N, get_f64(env, a.argv[1]), get_f64(env, a.argv[2]), typed(env, a.argv[3], NULL),
                   typed(env, a.argv[4], NULL), typed(env, a.argv[5], NULL), typed(env, a.argv[6], NULL),
                   get_f64(env, a.argv[7]), get_f64(env, a.argv[8]), cap, sort, &rep, (int32_t *)list,
                   (int32_t *)perm);
  if (rc < 0) return throw_rc(env, NULL, rc, "ccs_fof");
  napi_value out;
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "report", report_to_obj(env, &rep));
  napi_set_named_property(env, out, "list", L);
  set_num(env, out, "count", rep.ppCount);
  napi_set_named_property(env, out, "perm", Pm);
  return out;
}

/* fofDevice(h, spring, touch, cap, sort) -> {report, list, perm}: the same analysis on the device */
static napi_value FofDevice(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  const int N = ccs_sim_ptr(h)->N, cap = get_i32(env, a.argv[3]), sort = get_bool(env, a.argv[4]);
  ccs_report rep;
  void *list, *perm = NULL;
  napi_value L = new_typed(env, napi_int32_array, (size_t)(cap > 0 ? cap : 1), 4, &list);
  napi_value Pm;
  napi_get_null(env, &Pm);
  if (sort) Pm = new_typed(env, napi_int32_array, (size_t)N, 4, &perm);
  int rc = ccs_fof_device(h, get_f64(env, a.argv[1]), get_f64(env, a.argv[2]), cap, sort, &rep, (int32_t *)list,
                          (int32_t *)perm);
  if (rc < 0) return throw_rc(env, h, rc, "ccs_fof_device");
  napi_value out;
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "report", report_to_obj(env, &rep));
  napi_set_named_property(env, out, "list", L);
  set_num(env, out, "count", rep.ppCount);
  napi_set_named_property(env, out, "perm", Pm);
  return out;
}

/* pairTable(bins, cut) -> {f, p}: meshPairTable (src/nbody.js:48-109) */
static napi_value PairTable(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  const int bins = get_i32(env, a.argv[0]);
  void *f, *p;
  napi_value F = new_typed(env, napi_float32_array, (size_t)bins, 4, &f);
  napi_value P = new_typed(env, napi_float32_array, (size_t)bins, 4, &p);
  int rc = ccs_pair_table(bins, get_f64(env, a.argv[1]), (float *)f, (float *)p);
  if (rc < 0) return throw_rc(env, NULL, rc, "ccs_pair_table");
  napi_value out;
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "f", F);
  napi_set_named_property(env, out, "p", P);
  return out;
}

/* readState(h, pos, vel, aux, q, mat): the state into caller-owned arrays (any may be null) */
static napi_value ReadState(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  return status(env, h, ccs_read_state(h, typed(env, a.argv[1], NULL), typed(env, a.argv[2], NULL),
                                        typed(env, a.argv[3], NULL), typed(env, a.argv[4], NULL),
                                        typed(env, a.argv[5], NULL)), "ccs_read_state");
}

/* books(h, withDiag) -> Float64Array(12): the device's binary64 books (src/nbody.js:837-850) */
static napi_value Books(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  void *out;
  napi_value B = new_typed(env, napi_float64_array, CCS_BOOKS, 8, &out);
  int rc = ccs_books(h, a.argc > 1 ? get_bool(env, a.argv[1]) : 1, (double *)out);
  if (rc < 0) return throw_rc(env, h, rc, "ccs_books");
  return B;
}

/* deviceBuffers(h) -> {pos, vel, aux, q, mat, home, force, mono, stream} as BigInt addresses: the headless
 * stand-ins for the textures src/view.js reads (src/view.js:216-220, 566-569), for a CUDA interop consumer */
static napi_value DeviceBuffers(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  ccs_device_buffers d;
  int rc = ccs_device_ptrs(h, &d);
  if (rc < 0) return throw_rc(env, h, rc, "ccs_device_ptrs");
  napi_value out, v;
  napi_create_object(env, &out);
#define PTR(name, p)                                            \
  napi_create_bigint_uint64(env, (uint64_t)(uintptr_t)(p), &v); \
  napi_set_named_property(env, out, name, v);
  PTR("pos", d.pos4) PTR("vel", d.vel4) PTR("aux", d.aux4) PTR("q", d.q) PTR("mat", d.mat) PTR("home", d.home4)
  PTR("forceA", d.force[0]) PTR("forceB", d.force[1]) PTR("monoA", d.mono[0]) PTR("monoB", d.mono[1])
  PTR("stream", d.stream)
#undef PTR
  return out;
}

/* advanceHost(h, pos, vel, q, nsteps, posOut, velOut, auxOut, qOut): one call from host arrays to host arrays */
static napi_value AdvanceHost(napi_env env, napi_callback_info info) {
  args_t a;
  get_args(env, info, &a);
  ccs_handle *h = handle_of(env, a.argv[0]);
  return status(env, h, ccs_advance_host(h, typed(env, a.argv[1], NULL), typed(env, a.argv[2], NULL),
                                          typed(env, a.argv[3], NULL), get_i32(env, a.argv[4]),
                                          typed(env, a.argv[5], NULL), typed(env, a.argv[6], NULL),
                                          typed(env, a.argv[7], NULL), typed(env, a.argv[8], NULL)),
                "ccs_advance_host");
}

NAPI_MODULE_INIT() {
  napi_property_descriptor d[] = {
#define FN(name, f) {name, NULL, f, NULL, NULL, NULL, napi_default, NULL},
      FN("create", Create) FN("makeBodies", MakeBodies) FN("build", Build) FN("getSim", GetSim)
      FN("setSim", SetSim) FN("setStatic", SetStatic) FN("step", Step) FN("steps", Steps)
      FN("settleSome", SettleSome) FN("rigidStep", RigidStep) FN("setMeshEvery", SetMeshEvery)
      FN("setPPSplit", SetPPSplit) FN("setPPSplitSym", SetPPSplitSym) FN("setContactWalk", SetContactWalk)
      FN("setPP", SetPP) FN("setBoxes", SetBoxes) FN("applyPerm", ApplyPerm)
      FN("sortMorton", SortMorton) FN("diagAsync", DiagAsync) FN("poll", Poll) FN("fof", Fof)
      FN("fofDevice", FofDevice) FN("pairTable", PairTable) FN("readState", ReadState) FN("books", Books)
      FN("deviceBuffers", DeviceBuffers) FN("advanceHost", AdvanceHost) FN("passSlots", PassSlots)
      FN("passMesh", PassMesh) FN("passPP", PassPP) FN("passSim", PassSim) FN("passDiag", PassDiag)
      FN("sync", Sync)
#undef FN
  };
  napi_define_properties(env, exports, sizeof d / sizeof *d, d);
  return exports;
}
