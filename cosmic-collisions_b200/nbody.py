"""The engine object of the giant-impact pages, on the B200.

`NBody` mirrors `CC.nbody` of src/nbody.js:1095-1118 -- the same method names
(snake_case, with the reference's camelCase names as aliases), the same
argument meaning and the same order of work -- over the C ABI of
libccstep.so.  The physics runs in the library's sm_100a kernels; this module
is the host glue the reference keeps in JavaScript: the analysis cadence, the
worker hand-off and applyReport (src/nbody.js:895-1025).

Errors: every failing library call raises `CCSError` (the reference throws
`Error` from its GL helpers, src/gl.js:15,24,47,62); a stale analysis is
dropped by generation (src/nbody.js:969,1016) exactly as the reference does.
"""
import ctypes as C
import json
import math
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _lib as L
from ._lib import CCSError, check, lib, ptr

FL = 6.0
PP_CAP = L.PP_CAP
PHASES = ("settle", "approach", "full")


def mean_k(r):
    """meanK(r), src/nbody.js:30: the mean temperature rise the heat makes, K."""
    return r.Q / r.M * NBody.E_KG / (NBody.CP_ROCK + r.iron * (NBody.CP_IRON - NBody.CP_ROCK))


class NBody:
    """CC.nbody on one GPU.  One instance per run; not thread-safe."""

    T_UNIT = 805
    V_UNIT = 7.91
    E_KG = 6.256e7
    CP_ROCK = 1200
    CP_IRON = 450
    L_EM = 0.1163
    JAM = 0.96
    PP_CAP = PP_CAP
    meanK = staticmethod(mean_k)

    def __init__(self, device=0):
        self._h = C.c_void_p()
        check(lib().ccs_create(int(device), C.byref(self._h)), what="ccs_create")
        self.device = device
        self.report = None
        self.ref = None
        self.gen = 0
        self.analyses = 0
        self.analyzed_at = 0
        self.pending = None
        self.async_read = True
        self.device_fof = False   # True: the analysis runs on the device (ccs_fof_device), synchronously
        self._worker = ThreadPoolExecutor(max_workers=1)
        self._job = None
        self._opt = None
        self._mat = None
        self.com1 = [0.0, 0.0, 0.0]
        self.pp = {"count": 0, "loose": 0}

    # ---- lifecycle ---------------------------------------------------------
    def close(self):
        if self._h:
            self._worker.shutdown(wait=True)
            lib().ccs_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        return check(rc, self._h, what)

    @property
    def handle(self):
        return self._h

    # ---- build(opt): src/nbody.js:114-250 -----------------------------------
    def build(self, opt=None, relax_on_device=False, **kw):
        """Build a run from options (a BuildOpt or keywords of make_opt) and upload it.  relax_on_device:
        the builder's overlap relaxation on this engine's GPU (equivalent to the host's, not identical)."""
        if opt is None:
            opt = L.make_opt(**kw)
        elif isinstance(opt, dict):
            opt = L.make_opt(**opt)
        self._opt = opt
        sim, pos, vel, mat, home = L.make_bodies(opt, self.device if relax_on_device else None)
        self.upload(sim, pos, vel, mat, home)
        return self.sim

    def upload(self, sim, pos, vel, mat, home=None):
        """Upload a run built elsewhere (ICs from any generator)."""
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        mat = np.ascontiguousarray(mat, np.float32)
        home = None if home is None else np.ascontiguousarray(home, np.float32)
        self._check(lib().ccs_build(self._h, C.byref(sim), ptr(pos), ptr(vel), ptr(mat), ptr(home)), "ccs_build")
        self._mat = mat.copy()
        self.gen += 1
        self.report = None
        self.ref = None
        self.pending = None
        self._job = None
        self.analyses = 0
        self.analyzed_at = 0
        self.pp = {"count": 0, "loose": 0}

    def set_field(self, g, frozen=-1.0, invM=1.0, cpIron=1.0):
        """The crater page's field-gravity step (simFS({gravity: 'field', frozen: true}), chicxulub.html:235,
        700-710, 763-766): constant gravity g, the material tagged `frozen` held still (negative: none),
        the contact grid every 2nd step and no mesh.  invM and cpIron are 1 on that page."""
        gg = np.ascontiguousarray(g, np.float64)
        self._check(lib().ccs_set_field(self._h, 1, ptr(gg), float(frozen), float(invM), float(cpIron)),
                    "ccs_set_field")

    def clear_field(self):
        """Back to the giant impact's mesh step."""
        self._check(lib().ccs_set_field(self._h, 0, None, -1.0, 1.0, 1.0), "ccs_set_field")

    # ---- checkpoint and restore (ccs_checkpoint_*) ---------------------------
    def save(self, path=None):
        """Checkpoint the run with this mirror's own analysis state (the energy reference, the cadence,
        the last report) as the format's extra bytes.  Only where the next step rebuilds the grid and the
        mesh (stepNo a multiple of meshEvery; even in the field step).  Returns the bytes; writes them to
        path too when given."""
        mine = {"ref": self.ref, "analyses": self.analyses, "analyzed_at": self.analyzed_at, "com1": self.com1,
                "pp": self.pp, "report": bytes(self.report).hex() if self.report is not None else None}
        extra = json.dumps(mine).encode()
        n = C.c_size_t()
        self._check(lib().ccs_checkpoint_size(self._h, len(extra), C.byref(n)), "ccs_checkpoint_size")
        buf = C.create_string_buffer(n.value)
        self._check(lib().ccs_checkpoint_save(self._h, extra, len(extra), buf, n.value), "ccs_checkpoint_save")
        data = buf.raw
        if path is not None:
            with open(path, "wb") as f:
                f.write(data)
        return data

    def load(self, src):
        """Restore a checkpoint (bytes or a path) into this engine: the run, and the mirror's analysis
        state when the checkpoint carries it."""
        from . import checkpoint
        if isinstance(src, (str, os.PathLike)):
            with open(src, "rb") as f:
                src = f.read()
        data = bytes(src)
        self._check(lib().ccs_checkpoint_load(self._h, data, len(data)), "ccs_checkpoint_load")
        ck = checkpoint.read(data, verify=False)
        self._mat = ck["mat"]
        self.gen += 1
        self.pending = None
        self._job = None
        self.report = None
        self.ref = None
        self.analyses = self.analyzed_at = 0
        self.pp = {"count": int(ck["ppCount"]), "loose": int(ck["ppLoose"])}
        try:
            mine = json.loads(ck["extra"].decode()) if ck["extra"] else {}
        except (UnicodeDecodeError, ValueError):
            mine = {}
        if mine:
            self.ref = mine.get("ref")
            self.analyses = int(mine.get("analyses", 0))
            self.analyzed_at = int(mine.get("analyzed_at", 0))
            self.com1 = list(mine.get("com1", self.com1))
            if mine.get("report"):
                self.report = L.Report.from_buffer_copy(bytes.fromhex(mine["report"]))

    @property
    def sim(self):
        """The live run scalars (a ctypes view: writes go straight to the engine)."""
        return lib().ccs_sim_ptr(self._h).contents

    @property
    def phase(self):
        return PHASES[self.sim.phase]

    def set_static(self):
        self._check(lib().ccs_set_static(self._h), "ccs_set_static")

    def uniforms(self):
        u = L.Uniforms()
        self._check(lib().ccs_get_uniforms(self._h, C.byref(u)), "ccs_get_uniforms")
        return u

    @property
    def mesh_every(self):
        return self._mesh_every if hasattr(self, "_mesh_every") else 8

    @mesh_every.setter
    def mesh_every(self, n):
        self._check(lib().ccs_set_mesh_every(self._h, int(n)), "ccs_set_mesh_every")
        self._mesh_every = int(n)

    # ---- the step and the phases: src/nbody.js:551-636 -----------------------
    def step(self, settle=False, kick=False):
        self._check(lib().ccs_step(self._h, int(bool(settle)), int(bool(kick))), "ccs_step")

    def steps(self, n):
        """n frame-loop steps: step(false, false); sim.t += sim.dt (index.html:372)."""
        self._check(lib().ccs_steps(self._h, int(n)), "ccs_steps")

    def settle_some(self, n):
        before = self.sim.settleLeft
        self._check(lib().ccs_settle_some(self._h, int(n)), "ccs_settle_some")
        if before > 0 and self.sim.settleLeft == 0:
            self.analyzed_at = self.sim.stepNo   # the settle's steps are not the analysis's to count

    def rigid_step(self, dtF):
        self._check(lib().ccs_rigid_step(self._h, float(dtF)), "ccs_rigid_step")

    def sync(self):
        self._check(lib().ccs_sync(self._h), "ccs_sync")

    # ---- the passes (CC.nbody.passes) --------------------------------------
    def pass_slots(self):
        self._check(lib().ccs_pass_slots(self._h), "ccs_pass_slots")

    def pass_mesh(self):
        self._check(lib().ccs_pass_mesh(self._h), "ccs_pass_mesh")

    def pass_pp(self):
        self._check(lib().ccs_pass_pp(self._h), "ccs_pass_pp")

    def pass_sim(self, settle=False, kick=False, gdt=0.0):
        self._check(lib().ccs_pass_sim(self._h, int(bool(settle)), int(bool(kick)), float(gdt)), "ccs_pass_sim")

    def pass_diag(self):
        self._check(lib().ccs_pass_diag(self._h), "ccs_pass_diag")

    # ---- state read-outs ---------------------------------------------------
    def read_state(self):
        N = self.sim.N
        pos = np.empty((N, 4), np.float32)
        vel = np.empty((N, 4), np.float32)
        aux = np.empty((N, 4), np.float32)
        q = np.empty(N, np.float32)
        mat = np.empty(N, np.float32)
        self._check(lib().ccs_read_state(self._h, ptr(pos), ptr(vel), ptr(aux), ptr(q), ptr(mat)), "ccs_read_state")
        return {"pos": pos, "vel": vel, "aux": aux, "q": q, "mat": mat}

    def write_state(self, pos=None, vel=None, aux=None, q=None, mat=None):
        arr = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (pos, vel, aux, q, mat)]
        self._check(lib().ccs_write_state(self._h, *[ptr(a) for a in arr]), "ccs_write_state")
        if mat is not None:
            self._mat = arr[4].copy()

    def buffer(self, name):
        """An internal buffer (seats, meshes, P3M list ...) as a numpy array."""
        N = self.sim.N
        u = self.uniforms()
        sizes = {"seats": (u.AW * u.AH * L.SEATS, np.uint32), "fineA": ((L.FINE + 1) * 4, np.float32),
                 "forceA": ((L.FINE + 1) * 4, np.float32), "monoA": (4, np.float32),
                 "coarseA": (L.COARSE * 4, np.float32), "farA": (L.COARSE * 4, np.float32),
                 "fineB": ((L.FINE + 1) * 4, np.float32), "forceB": ((L.FINE + 1) * 4, np.float32),
                 "monoB": (4, np.float32), "pplist": (PP_CAP * 4, np.float32),
                 "ppforce": (PP_CAP * 16, np.float32), "ppbox": (PP_CAP, np.float32), "ppslot": (N, np.int32),
                 "diag": (N * 4, np.float32), "cellof": (N, np.uint32),
                 "tide0A": ((L.FINE + 1) * 4, np.float32), "tide1A": ((L.FINE + 1) * 4, np.float32),
                 "ppall": (N * 4, np.float32), "walkstats": (3, np.uint32), "walkcount": ((N + 31) // 32, np.int32),
                 "tide2A": (3 * (L.FINE + 1) * 4, np.float32), "fineQA": (2 * (L.FINE + 1) * 4, np.float32)}
        n, dt = sizes[name]
        a = np.empty(n, dt)
        self._check(lib().ccs_read_buffer(self._h, L.BUF[name], ptr(a), a.nbytes), "ccs_read_buffer")
        if name == "seats":
            return a.reshape(-1, L.SEATS)
        if dt == np.float32 and name not in ("ppbox",):
            return a.reshape(-1, 4)
        return a

    def device_buffers(self):
        d = L.DeviceBuffers()
        self._check(lib().ccs_device_ptrs(self._h, C.byref(d)), "ccs_device_ptrs")
        return d

    def direct_sum(self, idx):
        """The exact pull (binary64 direct sum, softening a) at particles idx: (acc n x 3, pot n)."""
        idx = np.ascontiguousarray(idx, np.int32)
        acc = np.zeros((len(idx), 3), np.float64)
        pot = np.zeros(len(idx), np.float64)
        self._check(lib().ccs_direct_sum(self._h, ptr(idx), len(idx), ptr(acc), ptr(pot)), "ccs_direct_sum")
        return acc, pot

    def pp_list_force(self, lst):
        """ccs_pp_list_force: the reference's pairwise correction over a list of any length (no 8,192 cap), per
        member Gm x (pull xyz, potential), n x 4; the run is not changed."""
        lst = np.ascontiguousarray(lst, np.int32)
        out = np.zeros((len(lst), 4), np.float32)
        self._check(lib().ccs_pp_list_force(self._h, ptr(lst) if len(lst) else None, len(lst),
                                            ptr(out) if len(lst) else None), "ccs_pp_list_force")
        return out

    def books(self, with_diag=True):
        """The conservation books on the device in binary64 (src/nbody.js:837-850)."""
        out = np.zeros(L.BOOKS, np.float64)
        self._check(lib().ccs_books(self._h, int(bool(with_diag)), ptr(out)), "ccs_books")
        keys = ["M", "px", "py", "pz", "Lx", "Ly", "Lz", "KE", "PE", "Q", "unseated", "full"]
        return dict(zip(keys, out.tolist()))

    # ---- the analysis: src/nbody.js:895-1025 --------------------------------
    def analyze(self, sync=False):
        if self._job is not None and not sync:
            return
        s = self.sim
        if sync:
            self.gen += 1   # whatever the worker is still computing is for the state before this call
        self.analyzed_at = s.stepNo
        sort = False
        if s.phase == 2:   # `sim.phase === 'full' && analyses++ % 8 === 0`
            sort = self.analyses % 8 == 0
            self.analyses += 1
        if self.device_fof:
            r, lst, perm = self.fof_device(sort)
            self._apply_report(r, lst, perm, s.t)
            return
        self._check(lib().ccs_diag_async(self._h), "ccs_diag_async")
        if not sync and self.async_read:
            self.pending = {"gen": self.gen, "sort": sort, "t": s.t}
            return
        P, V, D = self._wait_read()
        r, lst, perm = L.fof(s.N, s.m, s.a, P, V, self._mat, D, s.k, 2 * s.a, PP_CAP, sort)
        self._apply_report(r, lst, perm, s.t)

    def fof_device(self, sort=False, cap=PP_CAP):
        """The worker's fof (src/nbody.js:646-893) on the device over the current state:
        (report, loose list, Morton permutation or None).  The state is not moved."""
        s = self.sim
        rep = L.Report()
        lst = np.zeros(max(cap, 1), np.int32)
        perm = np.zeros(s.N, np.int32) if sort else None
        self._check(lib().ccs_fof_device(self._h, s.k, 2 * s.a, int(cap), 1 if sort else 0, C.byref(rep), ptr(lst),
                                         ptr(perm)), "ccs_fof_device")
        return rep, lst[:rep.ppCount].copy(), perm

    def _wait_read(self):
        N = self.sim.N
        P = np.empty((N, 4), np.float32)
        V = np.empty((N, 4), np.float32)
        D = np.empty((N, 4), np.float32)
        self.sync()
        rc = self._check(lib().ccs_poll(self._h, ptr(P), ptr(V), ptr(D)), "ccs_poll")
        if rc != L.CCS_OK:
            raise CCSError("read-back not complete after a stream synchronize")
        return P, V, D

    def collect(self):
        """The frame loop's poll (src/nbody.js:1011-1025): the read-back when it has landed, to the
        worker; the worker's report when it is done, applied if it is still current."""
        if self._job is not None and self._job[0].done():
            fut, gen, t = self._job
            self._job = None
            r, lst, perm = fut.result()
            if gen == self.gen:
                self._apply_report(r, lst, perm, t)
        if self.pending is None:
            return
        N = self.sim.N
        P = np.empty((N, 4), np.float32)
        V = np.empty((N, 4), np.float32)
        D = np.empty((N, 4), np.float32)
        rc = self._check(lib().ccs_poll(self._h, ptr(P), ptr(V), ptr(D)), "ccs_poll")
        if rc == L.CCS_NOT_READY:
            return
        p, self.pending = self.pending, None
        if p["gen"] != self.gen:
            return
        s = self.sim
        args = (s.N, s.m, s.a, P, V, self._mat.copy(), D, s.k, 2 * s.a, PP_CAP, p["sort"])
        self._job = (self._worker.submit(L.fof, *args), p["gen"], p["t"])

    @property
    def state(self):
        return {"analyzing": self._job is not None, "pending": self.pending is not None, "worker": True,
                "analyses": self.analyses, "analyzedAt": self.analyzed_at, "stepNo": self.sim.stepNo}

    def sort_now(self):
        self.analyses = 0
        self.analyze(True)
        return self.report

    def _apply_report(self, r, lst, perm, t):
        """applyReport, src/nbody.js:912-928."""
        self.report = r
        self.com1 = list(r.com)
        self._place_boxes(r, t)
        s = self.sim
        going = s.phase == 2 or any(s.bulk0[k] != 0 for k in range(3))
        if self.ref is None and going:
            self.ref = {"E": r.KE + r.PE + r.EL, "EQ": r.KE + r.PE + r.EL + r.Q, "L": r.L, "scale": r.KE - r.PE}
        if perm is not None:
            self.apply_perm(perm)
        self.set_pp(lst, r.ppLoose)

    def _place_boxes(self, r, t):
        """placeBoxes, src/nbody.js:361-374: the two boxes from a look, handed over in one ccs_set_boxes."""
        s = self.sim
        boxes = (L.Box * 2)()
        a, b = boxes[0], boxes[1]
        a.on, a.t = 1, t
        for k in range(3):
            a.cen[k], a.vel[k] = r.core[k], r.bodyVel[k]
        b.on = s.boxOn[1]
        b.t = s.boxT[1]
        for k in range(3):
            b.cen[k], b.vel[k] = s.boxCen[1][k], s.boxVel[1][k]
        if r.hasSecond and r.secMass > 0.05:
            d = max(abs(r.secCore[k] - r.core[k]) for k in range(3))
            far = FL - 1.3 * math.pow(r.secMass, 1.0 / 3.0)
            if not s.boxOn[1] and d > far:
                b.on = 1
                w = r.secMass / s.m
                c = r.secCore
                b.primeMono = 1
                for k, v in enumerate((c[0] * w, c[1] * w, c[2] * w, w)):
                    b.mono[k] = v
            elif s.boxOn[1] and d < far - 0.5:
                b.on = 0
            for k in range(3):
                b.cen[k], b.vel[k] = r.secCore[k], r.secVel[k]
            b.t = t
        else:
            b.on = 0
        self._check(lib().ccs_set_boxes(self._h, boxes), "ccs_set_boxes")

    def set_boxes(self, boxes):
        """Both mesh boxes at once: a sequence of two dicts with on, cen, vel, t and optionally mono (the
        first monopole of a box that has just gone up)."""
        arr = (L.Box * 2)()
        for b, d in zip(arr, boxes):
            b.on = int(d["on"])
            b.t = float(d.get("t", self.sim.t))
            for k in range(3):
                b.cen[k] = float(d["cen"][k])
                b.vel[k] = float(d.get("vel", (0.0, 0.0, 0.0))[k])
            if d.get("mono") is not None:
                b.primeMono = 1
                for k in range(4):
                    b.mono[k] = float(d["mono"][k])
        self._check(lib().ccs_set_boxes(self._h, arr), "ccs_set_boxes")

    def set_pp_split(self, S):
        """The stencil-split P3M (ccs_set_pp_split): every pair of mesh nodes within S cells (1..3) summed
        particle by particle, the rest on the mesh to second order; 0 returns to the reference's pass."""
        self._check(lib().ccs_set_pp_split(self._h, int(S)), "ccs_set_pp_split")

    def pp_split_pairs(self):
        """ccs_pp_split_pairs: the last split pair pass's pair evaluations (one way, both ways)."""
        out = np.zeros(2, np.uint64)
        self._check(lib().ccs_pp_split_pairs(self._h, ptr(out)), "ccs_pp_split_pairs")
        return int(out[0]), int(out[1])

    def set_pp_split_sym(self, min_node):
        """ccs_set_pp_split_sym: nodes of at least min_node particles take their mutual pairs once, both ways
        (default 16); 0: every pair one way."""
        self._check(lib().ccs_set_pp_split_sym(self._h, int(min_node)), "ccs_set_pp_split_sym")

    def set_contact_walk(self, mode):
        """How the step after a grid rebuild finds its contact pairs (ccs_set_contact_walk): 1 (the default)
        replays the rebuilding step's record where it is good, 0 walks the seat tables every step, 2 is 1
        counting how each particle found its pairs (buffer "walkstats": replayed, replayed and walked the
        cells a new cell added, walked)."""
        self._check(lib().ccs_set_contact_walk(self._h, int(mode)), "ccs_set_contact_walk")

    def contact_pairs(self, cap=64):
        """The contact-pair sets of the current state (ccs_contact_pairs): (counts, pairs), pairs an N x cap
        array of neighbour indices with bit 31 set for touching pairs, unused slots 0xFFFFFFFF."""
        N = self.sim.N
        counts = np.zeros(N, np.int32)
        pairs = np.zeros((N, cap), np.uint32)
        self._check(lib().ccs_contact_pairs(self._h, int(cap), ptr(counts), ptr(pairs)), "ccs_contact_pairs")
        return counts, pairs

    def prime_mono(self, box, mono):
        m = np.ascontiguousarray(mono, np.float32)
        self._check(lib().ccs_prime_mono(self._h, int(box), ptr(m)), "ccs_prime_mono")

    def apply_perm(self, perm):
        """applyPerm, src/nbody.js:932-954: state, mat and home in the new order, fresh cells."""
        perm = np.ascontiguousarray(perm, np.int32)
        self._check(lib().ccs_apply_perm(self._h, ptr(perm)), "ccs_apply_perm")
        self._mat = self._mat[perm]

    def sort_morton(self, core):
        """The Morton order computed on the device and applied; returns (perm, into)."""
        N = self.sim.N
        c = np.ascontiguousarray(core, np.float64)
        perm = np.empty(N, np.int32)
        into = np.empty(N, np.int32)
        self._check(lib().ccs_sort_morton(self._h, ptr(c), ptr(perm), ptr(into)), "ccs_sort_morton")
        self._mat = self._mat[perm]
        return perm, into

    def set_pp(self, lst, loose=None):
        """setPP, src/nbody.js:957-966: the loose list, then its pairwise pass."""
        lst = np.ascontiguousarray(lst, np.int32)
        n = len(lst)
        self._check(lib().ccs_set_pp(self._h, ptr(lst) if n else None, n, int(loose if loose is not None else n)),
                    "ccs_set_pp")
        self.pp = {"count": n, "loose": int(loose if loose is not None else n)}

    def autotune(self, reps=8):
        """ccs_autotune: measure the contact step's CTA width and the cell gravity's threads per cell on this run's
        state (reps > 0) or apply what an earlier run of the same size measured (reps = 0); returns the choice."""
        ch = (C.c_int * 2)()
        self._check(lib().ccs_autotune(self._h, int(reps), ch), "ccs_autotune")
        return {"warps": ch[0], "cell_split": ch[1]}

    def set_pp_nn(self, net):
        """Attach a LearnedCorrection to the P3M pass (None: back to the plain table).  The network must outlive
        the attachment."""
        self._check(lib().ccs_set_pp_nn(self._h, net.handle if net is not None else None), "ccs_set_pp_nn")
        self.nn = net

    # ---- the scripted driver: window.__impact.runTo, index.html:592-600 ------
    def run_to(self, t, analyze_every=360):
        s = self.sim
        if s.t > t and self._opt is not None:
            self.build(self._opt)
        while self.sim.phase == 0:
            self.settle_some(64)
        while self.sim.phase == 1 and self.sim.t < t:
            self.rigid_step(0.01)
        while self.sim.phase == 2 and self.sim.t < t:
            s = self.sim
            left = analyze_every - (s.stepNo - self.analyzed_at)
            # steps that cannot pass t even if soften() grows dt by sqrt(2)
            safe = int((t - s.t) / (s.dt * (1.0 if s.soft else math.sqrt(2.0)))) - 1
            n = max(1, min(left, safe))
            if n > 1:
                self.steps(n)
            else:
                self.step(False, False)
                self.sim.t += self.sim.dt
            if self.sim.stepNo - self.analyzed_at >= analyze_every:
                self.analyze(True)
        self.analyze(True)
        return self.sim.t

    # reference spellings
    settleSome = settle_some
    rigidStep = rigid_step
    sortNow = sort_now
    runTo = run_to

    @property
    def analyzedAt(self):
        return self.analyzed_at


class Ensemble:
    """ccs_ensemble: several engines advanced together, each round of meshEvery steps one CUDA graph with every
    member's block as a parallel branch.  The members stay usable engines and must outlive the ensemble."""

    def __init__(self, members):
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.handle.value for m in self.members])
        h = C.c_void_p()
        rc = lib().ccs_ensemble_create(arr, len(self.members), C.byref(h))
        if rc != 0:
            raise L.CCSError("ccs_ensemble_create failed: %s" % L.CCS_E.get(rc, rc))
        self._h = h

    def _check(self, rc, what):
        if rc != 0:
            raise L.CCSError("%s failed: %s %s" % (what, L.CCS_E.get(rc, rc),
                                                   lib().ccs_ensemble_last_error(self._h).decode()))

    def steps(self, n):
        """n frame-loop steps of every member (n a multiple of meshEvery; members at a block boundary)."""
        self._check(lib().ccs_ensemble_steps(self._h, int(n)), "ccs_ensemble_steps")

    def sync(self):
        self._check(lib().ccs_ensemble_sync(self._h), "ccs_ensemble_sync")

    def set_persistent(self, on=True):
        """ccs_ensemble_set_persistent: each round of 8 steps as one persistent launch over every member (after
        the members' mesh chains), work items taken from per-member queues; off: the branch form."""
        self._check(lib().ccs_ensemble_set_persistent(self._h, 1 if on else 0), "ccs_ensemble_set_persistent")

    def step_ms(self):
        """ccs_ensemble_step_ms: per member, the mean ms of one step inside the persistent rounds since the last
        call (-1 where none ran); waits for the rounds and resets the sums."""
        import numpy as np
        out = np.zeros(len(self.members), np.float64)
        self._check(lib().ccs_ensemble_step_ms(self._h, out.ctypes.data_as(C.c_void_p), len(self.members)),
                    "ccs_ensemble_step_ms")
        return out

    def launch_count(self):
        """persistent rounds launched (one kernel launch each)"""
        return int(lib().ccs_ensemble_launch_count(self._h))

    def set_wait_ns(self, ns):
        """ccs_ensemble_set_wait_ns: the bound on every wait of the persistent round (default 2 s)."""
        self._check(lib().ccs_ensemble_set_wait_ns(self._h, int(ns)), "ccs_ensemble_set_wait_ns")

    def autotune(self, rounds=4):
        """ccs_ensemble_autotune: every launch-shape combination on all members, timed over real rounds (the
        members advance); the fastest aggregate is kept.  Returns the choice."""
        ch = (C.c_int * 2)()
        self._check(lib().ccs_ensemble_autotune(self._h, int(rounds), ch), "ccs_ensemble_autotune")
        return {"warps": ch[0], "cell_split": ch[1]}

    def close(self):
        if self._h:
            lib().ccs_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
