// nbody_b200.js -- CC.nbody on the B200 step.  The engine object src/nbody.js hands the pages
// (src/nbody.js:1095-1118), with its GL passes, textures and Worker replaced by libccstep through the
// Node-API binding (ccstep_napi.c); the pages (index.html's frame loop and runTo, src/view.js's readers)
// keep calling the same methods.  Built where node and its headers are: `node-gyp rebuild` in this folder.
(function () {
'use strict';
var B = require('./build/Release/ccstep.node');
var CC = global.CC || (global.CC = {});
var N_CHOICES = CC.N_CHOICES || [16384, 32768, 65536, 131072, 262144];   // src/shell.js:132
var T_UNIT = 805, V_UNIT = 7.91, E_KG = 6.256e7, CP_ROCK = 1200, CP_IRON = 450, L_EM = 0.1163, JAM = 0.96;
var PP_CAP = 8192, ANALYZE_EVERY = 360;

var h = null, device = 0, report = null, ref = null, gen = 0, analyses = 0, analyzedAt = 0;
var pending = null, asyncRead = true, meshEvery = 8, matR = null, homeArr = null, N = 0;
var P = null, V = null, D = null;

function meanK(r) { return r.Q / r.M * E_KG / (CP_ROCK + r.iron * (CP_IRON - CP_ROCK)); }

// the run's scalars: every read and write goes through the engine, so `sim.t += sim.dt` works as on the page
var sim = new Proxy({}, {
  get: function (_, k) {
    if (!h) return undefined;
    if (k === 'matR') return matR;
    if (k === 'home') return homeArr;
    if (k === 'ref') return ref;
    if (k === 'gen') return gen;
    return B.getSim(h)[k];
  },
  set: function (_, k, v) {
    var s = B.getSim(h);
    s[k] = v;
    B.setSim(h, s);
    if (['k', 'c', 'dt', 'damp', 'creep', 'tK', 'kappa', 'spin0', 'spin1'].indexOf(k) >= 0) B.setStatic(h);
    return true;
  }
});

// init(): the GPU resources (src/nbody.js:1030-1092) -- here one engine on `device`
function init(o) { device = (o && o.device) || 0; h = B.create(device); return CC.nbody; }

// build(opt): the initial conditions and their upload (src/nbody.js:114-250)
function build(opt) {
  var n2 = opt.n2 || 0, mImp = opt.mImp || 0;
  var r = B.makeBodies({N: N_CHOICES[opt.nIdx], q: opt.q, dens: opt.dens, core: opt.core, coreImp: opt.coreImp,
                        spin0: opt.spin0, spin1: opt.spin1, angle: opt.angle, incl: opt.incl, vfac: opt.vfac,
                        rest: opt.rest, n2: n2, mImp: mImp, mTarget: 0, rhoR: 0, rhoCrust: 0, crustFrac: 0});
  B.build(h, r.sim, r.pos, r.vel, r.mat, r.home);
  N = r.sim.N; matR = r.mat; homeArr = r.home;
  P = new Float32Array(4 * N); V = new Float32Array(4 * N); D = new Float32Array(4 * N);
  report = null; ref = null; pending = null; analyses = 0; analyzedAt = 0; gen++;
  if (CC.setSim) CC.setSim(sim);
  return sim;
}

// step(settle, kick): src/nbody.js:551-558
function step(settle, kick) { B.step(h, !!settle, !!kick); }
function steps(n) { B.steps(h, n); }                         // the frame loop's n steps, graph-replayed
function settleSome(n) {                                     // src/nbody.js:561-566
  var before = sim.settleLeft;
  B.settleSome(h, n);
  if (before > 0 && sim.settleLeft === 0) analyzedAt = sim.stepNo;
}
function rigidStep(dtF) { B.rigidStep(h, dtF); }            // src/nbody.js:591-636

// placeBoxes(r): src/nbody.js:361-374
function placeBoxes(r, t) {
  var s = B.getSim(h), b1 = s.boxes[1];
  var boxes = [{on: true, cen: r.core, vel: r.bodyVel, t: t}, {on: b1.on, cen: b1.cen, vel: b1.vel, t: b1.t}];
  if (r.hasSecond && r.secMass > 0.05) {
    var d = Math.max(Math.abs(r.secCore[0] - r.core[0]), Math.abs(r.secCore[1] - r.core[1]),
                     Math.abs(r.secCore[2] - r.core[2])), far = 6.0 - 1.3 * Math.cbrt(r.secMass);
    if (!b1.on && d > far) {
      var w = r.secMass / s.m, c = r.secCore;
      boxes[1].on = true;
      boxes[1].mono = [c[0] * w, c[1] * w, c[2] * w, w];
    } else if (b1.on && d < far - 0.5) boxes[1].on = false;
    boxes[1].cen = r.secCore; boxes[1].vel = r.secVel; boxes[1].t = t;
  } else boxes[1].on = false;
  B.setBoxes(h, boxes);
}

// applyReport: src/nbody.js:912-928
function applyReport(res, t) {
  var r = res.report, s = B.getSim(h);
  report = r;
  placeBoxes(r, t);
  var going = s.phase === 2 || s.bulk0[0] !== 0 || s.bulk0[1] !== 0 || s.bulk0[2] !== 0;
  if (!ref && going) ref = {E: r.KE + r.PE + r.EL, EQ: r.KE + r.PE + r.EL + r.Q, L: r.L, scale: r.KE - r.PE};
  if (res.perm) {                                            // applyPerm: src/nbody.js:932-954
    B.applyPerm(h, res.perm);
    var m = new Float32Array(N), hm = new Float32Array(4 * N);
    for (var i = 0; i < N; i++) {
      var j = res.perm[i];
      m[i] = matR[j];
      for (var k = 0; k < 4; k++) hm[4 * i + k] = homeArr[4 * j + k];
    }
    matR = m; homeArr = hm;
  }
  B.setPP(h, res.list.subarray(0, res.count), r.ppLoose);   // setPP: src/nbody.js:957-966
  if (CC.setReport) CC.setReport(r);
}

// analyze(sync): passDiag and the read-back (src/nbody.js:967-1009); collect(): the fence poll and the
// analysis (src/nbody.js:1011-1025) -- the C restatement of the Worker's fof, or on the device
function analyze(sync) {
  if (pending && !sync) return;
  var s = B.getSim(h), sort = false;
  if (sync) gen++;
  analyzedAt = s.stepNo;
  if (s.phase === 2) sort = analyses++ % 8 === 0;
  B.diagAsync(h);
  pending = {gen: gen, sort: sort, t: s.t};
  if (sync || !asyncRead) { while (B.poll(h, P, V, D) === 1) {} finish(); }
}
function finish() {
  var s = B.getSim(h), p = pending;
  pending = null;
  if (!p || p.gen !== gen) return;                           // a stale analysis is dropped (src/nbody.js:969, 1016)
  applyReport(B.fof(N, s.m, s.a, P, V, matR, D, s.k, 2 * s.a, PP_CAP, p.sort), p.t);
}
function collect() { if (pending && B.poll(h, P, V, D) === 0) finish(); }

CC.nbody = {
  init: init, build: build, step: step, steps: steps, settleSome: settleSome, rigidStep: rigidStep,
  analyze: analyze, collect: collect,
  sortNow: function () { analyses = 0; analyze(true); return report; },
  // a pass's GLSL program swapped for a variant (src/nbody.js:1099-1104) has no counterpart: the passes are
  // compiled CUDA; the passes themselves stay callable for timing in place
  setProg: function () { throw new Error('setProg: the B200 step has no GLSL programs to swap'); },
  passes: { slots: function () { B.passSlots(h); }, mesh: function () { B.passMesh(h); },
            pp: function () { B.passPP(h); }, sim: function (s, k, g) { B.passSim(h, !!s, !!k, g || 0); },
            diag: function () { B.passDiag(h); } },
  get sim() { return sim; },
  get report() { return report; },
  get pending() { return pending; },
  get analyzedAt() { return analyzedAt; },
  get pm() { var d = B.deviceBuffers(h); return [{force: d.forceA, mono: d.monoA}, {force: d.forceB, mono: d.monoB}]; },
  get grid() { return {G: B.getSim(h).G}; },
  get progs() { return {}; },
  get pp() { return {count: report ? report.ppCount : 0, loose: report ? report.ppLoose : 0}; },
  get state() { return {analyzing: false, pending: !!pending, worker: false, analyses: analyses,
                        analyzedAt: analyzedAt, stepNo: h ? B.getSim(h).stepNo : 0, waitStatus: null}; },
  set meshEvery(n) { meshEvery = n; B.setMeshEvery(h, n); },
  set asyncRead(v) { asyncRead = !!v; },
  // the device buffers src/view.js reads as textures (src/view.js:216-220, 566-569), for CUDA interop
  get buffers() { return B.deviceBuffers(h); },
  // the stencil-split P3M (no counterpart in the reference): S = 1..3, or 0 for the reference's pass
  set ppSplit(S) { B.setPPSplit(h, S); },
  set contactWalk(mode) { B.setContactWalk(h, mode); },
  books: function (withDiag) { return B.books(h, withDiag !== false); },
  T_UNIT: T_UNIT, V_UNIT: V_UNIT, E_KG: E_KG, CP_ROCK: CP_ROCK, CP_IRON: CP_IRON, L_EM: L_EM, JAM: JAM,
  PP_CAP: PP_CAP, meanK: meanK, ANALYZE_EVERY: ANALYZE_EVERY
};
module.exports = CC.nbody;
})();
