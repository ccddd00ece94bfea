"""ctypes front of the CPU oracle (oracle/ccs_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module;
the product never does.  Parity against the reference's own outputs is
UNPINNED (the reference is WebGL2 GLSL + JavaScript, neither of which can run
on these machines); see ccs_oracle.h.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libccs_oracle.so")

SEATS = 8
EMPTY = 0xBF800000
FINE = 64 * 64 * 64
COARSE = 4096
PP_CAP = 8192
PP_BINS = 64
FL = 6.0
FH = 2 * FL / 64
PP_CUT = 5 * FH


def build():
    """Compile the oracle with its Makefile (gcc; no reference sources are involved)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Uni(C.Structure):
    _fields_ = [("N", C.c_int), ("W", C.c_int),
                ("G", C.c_int), ("GShift", C.c_int), ("GMask", C.c_int), ("SX", C.c_int),
                ("SXShift", C.c_int), ("SXMask", C.c_int), ("AW", C.c_int), ("AH", C.c_int),
                ("invCell", C.c_float), ("cell", C.c_float), ("link2", C.c_float), ("reach2", C.c_float),
                ("touch", C.c_float),
                ("K", C.c_float), ("C", C.c_float), ("invM", C.c_float), ("damp", C.c_float),
                ("creep", C.c_float), ("tK", C.c_float), ("kappa", C.c_float), ("cpIron", C.c_float),
                ("dt", C.c_float), ("gdt", C.c_float), ("settle", C.c_float), ("kick", C.c_float),
                ("bulk0", C.c_float * 3), ("bulk1", C.c_float * 3), ("cen0", C.c_float * 3),
                ("cen1", C.c_float * 3), ("spin0", C.c_float * 3), ("spin1", C.c_float * 3),
                ("invH", C.c_float), ("eps2Mesh", C.c_float), ("eps2Cell", C.c_float), ("Gm", C.c_float),
                ("LA", C.c_float * 3), ("LB", C.c_float * 3), ("boxB", C.c_float),
                ("cut", C.c_float), ("a2", C.c_float),
                ("field", C.c_float), ("gField", C.c_float * 3), ("frozen", C.c_float)]


class Sim(C.Structure):
    _fields_ = [("N", C.c_int), ("W", C.c_int), ("H", C.c_int), ("n1", C.c_int), ("n2", C.c_int),
                ("G", C.c_int), ("settleLeft", C.c_int), ("settleTotal", C.c_int), ("stepNo", C.c_int),
                ("soft", C.c_int), ("phase", C.c_int),
                ("m", C.c_double), ("a", C.c_double), ("cell", C.c_double), ("dt", C.c_double),
                ("k", C.c_double), ("c", C.c_double), ("creep", C.c_double), ("damp", C.c_double),
                ("tK", C.c_double), ("kappa", C.c_double),
                ("R1", C.c_double), ("R2", C.c_double), ("Re1", C.c_double), ("Re2", C.c_double),
                ("M1", C.c_double), ("M2", C.c_double), ("M", C.c_double), ("vc", C.c_double),
                ("vesc", C.c_double), ("t", C.c_double), ("impactT", C.c_double),
                ("spin0", C.c_double * 3), ("spin1", C.c_double * 3), ("cen0", C.c_double * 3),
                ("cen1", C.c_double * 3), ("bulk0", C.c_double * 3), ("bulk1", C.c_double * 3),
                ("relr", C.c_double * 3), ("relv", C.c_double * 3),
                ("boxOn", C.c_int * 2),
                ("boxCen", (C.c_double * 3) * 2), ("boxVel", (C.c_double * 3) * 2), ("boxT", C.c_double * 2)]


class Opt(C.Structure):
    _fields_ = [("N", C.c_int),
                ("q", C.c_double), ("dens", C.c_double), ("core", C.c_double), ("coreImp", C.c_double),
                ("spin0", C.c_double), ("spin1", C.c_double), ("angle", C.c_double), ("incl", C.c_double),
                ("vfac", C.c_double), ("rest", C.c_double),
                ("n2", C.c_int), ("mImp", C.c_double),
                ("mTarget", C.c_double), ("rhoR", C.c_double), ("rhoCrust", C.c_double),
                ("crustFrac", C.c_double)]


class Report(C.Structure):
    _fields_ = [("largest", C.c_double), ("largestImp", C.c_double), ("largestIron", C.c_double),
                ("day", C.c_double), ("tilt", C.c_double), ("axis", C.c_double * 3),
                ("bodyVel", C.c_double * 3), ("orbit", C.c_double), ("escape", C.c_double),
                ("hasSecond", C.c_int),
                ("secMass", C.c_double), ("secDist", C.c_double), ("secImp", C.c_double),
                ("secIron", C.c_double), ("secCom", C.c_double * 3), ("secCore", C.c_double * 3),
                ("secVel", C.c_double * 3), ("secR", C.c_double),
                ("secBound", C.c_int),
                ("com", C.c_double * 3), ("core", C.c_double * 3), ("vel", C.c_double * 3),
                ("R", C.c_double), ("Redge", C.c_double), ("Tsurf", C.c_double),
                ("hotCom", C.c_double * 3), ("hotR", C.c_double), ("impMass", C.c_double),
                ("impCom", C.c_double * 3), ("impRms", C.c_double),
                ("M", C.c_double), ("iron", C.c_double), ("drift", C.c_double), ("L", C.c_double),
                ("KE", C.c_double), ("PE", C.c_double), ("EL", C.c_double), ("Q", C.c_double),
                ("unseated", C.c_double), ("full", C.c_double), ("jD", C.c_double), ("moon", C.c_double),
                ("ppCount", C.c_int), ("ppLoose", C.c_int)]


def make_opt(N, q=0.1, dens=0.75, core=0.325, coreImp=None, spin0=0.18, spin1=0.20, angle=45.0,
             incl=50.0, vfac=1.05, rest=0.3, n2=0, mImp=0.0, mTarget=0.0, rhoR=0.0, rhoCrust=0.0,
             crustFrac=0.0):
    """build(opt) options; defaults are the giant-impact page's S (index.html:177-178)."""
    return Opt(N, q, dens, core, -1.0 if coreImp is None else coreImp, spin0, spin1, angle, incl, vfac,
               rest, n2, mImp, mTarget, rhoR, rhoCrust, crustFrac)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_mulberry.restype = C.c_double
        L.orc_mulberry.argtypes = [C.POINTER(C.c_uint32)]
        L.orc_maclaurin.restype = C.c_double
        L.orc_maclaurin.argtypes = [C.c_double]
        L.orc_maclaurin_g.restype = C.c_double
        L.orc_maclaurin_g.argtypes = [C.c_double]
        L.orc_turn.argtypes = [P, C.c_double, P]
        L.orc_ball.restype = C.c_int
        L.orc_ball.argtypes = [C.c_int, C.c_double, C.c_double, C.POINTER(C.c_uint32), C.c_double, P, P]
        L.orc_relax.argtypes = [P, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int]
        L.orc_approach_time.restype = C.c_double
        L.orc_approach_time.argtypes = [P, P, C.c_double, C.c_double]
        L.orc_build.restype = C.c_int
        L.orc_build.argtypes = [C.POINTER(Opt), C.POINTER(Sim), P, P, P, P]
        L.orc_pair_table.argtypes = [C.c_int, C.c_double, P, P]
        L.orc_make_uni.argtypes = [C.POINTER(Sim), C.POINTER(Uni)]
        L.orc_boxes.argtypes = [C.POINTER(Sim), C.POINTER(Uni)]
        L.orc_soften.argtypes = [C.POINTER(Sim)]
        L.orc_hash.argtypes = [C.POINTER(Uni), C.c_int, C.c_int, C.c_int, P, P]
        L.orc_cell_of.restype = C.c_uint32
        L.orc_cell_of.argtypes = [C.POINTER(Uni), P, P, C.c_int]
        L.orc_slots.argtypes = [C.POINTER(Uni), P, P]
        L.orc_box_of.restype = C.c_int
        L.orc_box_of.argtypes = [C.POINTER(Uni), P, P]
        L.orc_deposit.argtypes = [C.POINTER(Uni), C.c_int, P, P, P, P]
        L.orc_coarse.argtypes = [P, P, P]
        L.orc_far.argtypes = [P, P, P, P]
        L.orc_cell.argtypes = [C.POINTER(Uni), P, P, P, P, P, P]
        L.orc_pp_gather.argtypes = [C.POINTER(Uni), P, P, P, C.c_int, P, P]
        L.orc_pp_force.argtypes = [C.POINTER(Uni), P, P, C.c_int, C.c_int, P, P]
        L.orc_sim_pass.argtypes = [C.POINTER(Uni)] + [P] * 11 + [C.c_int] + [P] * 4
        L.orc_diag.argtypes = [C.POINTER(Uni)] + [P] * 9 + [C.c_int, P]
        L.orc_contact_pairs.argtypes = [C.POINTER(Uni), P, P, C.c_int, P, P]
        L.orc_cell_tide.argtypes = [C.POINTER(Uni), C.c_int] + [P] * 7
        L.orc_node_moments.argtypes = [C.POINTER(Uni), C.c_int] + [P] * 4
        L.orc_pp_split.argtypes = [C.POINTER(Uni), C.c_int, P, P, P]
        L.orc_gather_split.argtypes = [C.POINTER(Uni)] + [P] * 15
        L.orc_rigid.argtypes = [C.c_int] + [P] * 10 + [C.c_float, P, P]
        L.orc_morton.argtypes = [C.c_int, P, P, P, P, P]
        L.orc_engine_new.restype = P
        L.orc_engine_new.argtypes = [C.POINTER(Sim), P, P, P]
        L.orc_engine_free.argtypes = [P]
        L.orc_engine_sim.restype = C.POINTER(Sim)
        L.orc_engine_sim.argtypes = [P]
        L.orc_engine_step.argtypes = [P, C.c_int, C.c_int]
        L.orc_engine_set_field.argtypes = [P, C.c_int, P, C.c_double, C.c_double, C.c_double]
        L.orc_engine_rigid_step.argtypes = [P, C.c_double]
        L.orc_engine_set_pp.argtypes = [P, P, C.c_int]
        L.orc_engine_prime_mono.argtypes = [P, C.c_int, P]
        L.orc_engine_apply_perm.argtypes = [P, P]
        L.orc_engine_diag.argtypes = [P, P]
        L.orc_engine_buf.restype = P
        L.orc_engine_buf.argtypes = [P, C.c_int, C.POINTER(C.c_long)]
        L.orc_engine_set_threads.argtypes = [C.c_int]
        L.orc_fof.argtypes = [C.c_int, C.c_double, C.c_double, P, P, P, P, C.c_double, C.c_double, C.c_int,
                              C.c_int, C.POINTER(Report), P, P]
        L.orc_direct_sum.argtypes = [C.c_int, P, P, C.c_double, C.c_int, P, P, P]
        L.orc_nn_label.argtypes = [P, P, P]
        _lib = L
    return _lib


def ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def set_threads(n):
    lib().orc_engine_set_threads(int(n))


def mulberry_seq(seed, n):
    s = C.c_uint32(seed)
    return np.array([lib().orc_mulberry(C.byref(s)) for _ in range(n)])


def maclaurin(f):
    return lib().orc_maclaurin(f)


def maclaurin_g(e):
    return lib().orc_maclaurin_g(e)


def turn(w, dt):
    w = np.asarray(w, np.float64)
    out = np.zeros(9, np.float64)
    lib().orc_turn(ptr(w), dt, ptr(out))
    return out


def build_run(opt):
    """build(opt): returns (sim, pos4, vel4, mat, home4)."""
    N = opt.N
    sim = Sim()
    pos = np.zeros((N, 4), np.float32)
    vel = np.zeros((N, 4), np.float32)
    mat = np.zeros(N, np.float32)
    home = np.zeros((N, 4), np.float32)
    rc = lib().orc_build(C.byref(opt), C.byref(sim), ptr(pos), ptr(vel), ptr(mat), ptr(home))
    assert rc == 0
    return sim, pos, vel, mat, home


def pair_table(bins=PP_BINS, cut=PP_CUT):
    f = np.zeros(bins, np.float32)
    p = np.zeros(bins, np.float32)
    lib().orc_pair_table(bins, cut, ptr(f), ptr(p))
    return f, p


def make_uni(sim):
    u = Uni()
    lib().orc_make_uni(C.byref(sim), C.byref(u))
    return u


def slots(u, pos4):
    seats = np.empty(u.AW * u.AH * SEATS, np.uint32)
    lib().orc_slots(C.byref(u), ptr(np.ascontiguousarray(pos4, np.float32)), ptr(seats))
    return seats.reshape(-1, SEATS)


def cell_ids(u, pos4):
    pos4 = np.ascontiguousarray(pos4, np.float32)
    N = pos4.shape[0]
    out = np.empty(N, np.uint32)
    words = np.empty(N, np.uint32)
    w = C.c_uint32()
    for i in range(N):
        out[i] = lib().orc_cell_of(C.byref(u), pos4[i].ctypes.data_as(C.c_void_p), C.byref(w), i)
        words[i] = w.value
    return out, words


def morton(pos4, core):
    pos4 = np.ascontiguousarray(pos4, np.float32)
    N = pos4.shape[0]
    keys = np.empty(N, np.int32)
    perm = np.empty(N, np.int32)
    into = np.empty(N, np.int32)
    core = np.asarray(core, np.float64)
    lib().orc_morton(N, ptr(pos4), ptr(core), ptr(keys), ptr(perm), ptr(into))
    return keys, perm, into


def nn_labels(rec):
    """The learned correction's labels (cells^-2) of records (d.xyz, s.xyz): orc_nn_label per record."""
    rec = np.asarray(rec, np.float64)
    out = np.empty((len(rec), 3))
    o = np.empty(3)
    for k in range(len(rec)):
        d = np.ascontiguousarray(rec[k, :3])
        s = np.ascontiguousarray(rec[k, 3:6])
        lib().orc_nn_label(ptr(d), ptr(s), ptr(o))
        out[k] = o
    return out


def contact_pairs(u, pos4, seats, cap=64):
    """The contact-pair sets of simFS's loop: (counts, pairs N x cap; index | touching << 31)."""
    pos4 = np.ascontiguousarray(pos4, np.float32)
    seats = np.ascontiguousarray(seats, np.uint32)
    N = pos4.shape[0]
    counts = np.zeros(N, np.int32)
    pairs = np.zeros((N, cap), np.uint32)
    lib().orc_contact_pairs(C.byref(u), ptr(pos4), ptr(seats), int(cap), ptr(counts), ptr(pairs))
    return counts, pairs


def cell_tide(u, S, fine, coarse, fineQ=None):
    """The stencil-split P3M's cell pass, near and far: (force, tide0, tide1), each (64^3 + 1) x 4, and
    tide2, the pull's second gradient, 3 x (64^3 + 1) x 4 (the library's three planes).  fineQ (node_moments):
    the near cells act as quadrupoles and the blocks' quadrupoles include the cells' own."""
    force = np.zeros((FINE + 1, 4), np.float32)
    t0 = np.zeros((FINE + 1, 4), np.float32)
    t1 = np.zeros((FINE + 1, 4), np.float32)
    t2 = np.zeros((3, FINE + 1, 4), np.float32)
    a = [np.ascontiguousarray(x, np.float32) for x in (fine, coarse)]
    q = None if fineQ is None else np.ascontiguousarray(fineQ, np.float32)
    lib().orc_cell_tide(C.byref(u), int(S), *[ptr(x) for x in a], ptr(q), ptr(force), ptr(t0), ptr(t1), ptr(t2))
    return force, t0, t1, t2


def node_moments(u, box, pos4, mat, fine):
    """Each fine cell's second moment about its centre of mass: 2 x (64^3 + 1) x 4 (Qxx Qyy Qzz Qxy; Qxz Qyz)."""
    out = np.zeros((2, FINE + 1, 4), np.float32)
    a = [np.ascontiguousarray(x, np.float32) for x in (pos4, mat, fine)]
    lib().orc_node_moments(C.byref(u), int(box), *[ptr(x) for x in a], ptr(out))
    return out


def pp_split(u, S, pos4, mat):
    """The stencil-split P3M's pairs: every particle's (pull, potential) x Gm, N x 4."""
    pos4 = np.ascontiguousarray(pos4, np.float32)
    out = np.zeros((len(pos4), 4), np.float32)
    lib().orc_pp_split(C.byref(u), int(S), ptr(pos4), ptr(np.ascontiguousarray(mat, np.float32)), ptr(out))
    return out


def gather_split(u, pos4, meshA, meshB, monoA, monoB, ppall):
    """The stencil-split P3M's gravity at every particle; meshA/meshB = (fine, force, tide0, tide1[, tide2]):
    with tide2 the second-order gather, without it the first-order one."""
    pos4 = np.ascontiguousarray(pos4, np.float32)
    out = np.zeros((len(pos4), 4), np.float32)

    def mesh(m):
        m = [np.ascontiguousarray(x, np.float32) for x in m]
        return [m[0], m[1], m[2], m[3], m[4] if len(m) > 4 else None]
    arrs = mesh(meshA) + mesh(meshB) + [np.ascontiguousarray(x, np.float32) for x in (monoA, monoB, ppall)]
    lib().orc_gather_split(C.byref(u), ptr(pos4), *[None if x is None else ptr(x) for x in arrs], ptr(out))
    return out


def box_of(u, p):
    """GLSL_BOX boxOf for one position: (box, g as float32[3])."""
    p = np.ascontiguousarray(p, np.float32)
    g = np.empty(3, np.float32)
    b = lib().orc_box_of(C.byref(u), ptr(p), ptr(g))
    return b, g


def direct_sum(pos4, masses, eps, idx):
    """FP64 direct-sum acceleration and potential at particles idx (G = 1, softening eps, no self term)."""
    pos4 = np.ascontiguousarray(pos4, np.float32)
    m = np.ascontiguousarray(masses, np.float64)
    idx = np.ascontiguousarray(idx, np.int32)
    acc = np.zeros((len(idx), 3), np.float64)
    pot = np.zeros(len(idx), np.float64)
    lib().orc_direct_sum(len(pos4), ptr(pos4), ptr(m), float(eps), len(idx), ptr(idx), ptr(acc), ptr(pot))
    return acc, pot


def fof(N, mref, a, P, V, R, D, spring, touch, cap=PP_CAP, sort=False):
    rep = Report()
    lst = np.zeros(cap, np.int32)
    perm = np.zeros(N, np.int32) if sort else None
    lib().orc_fof(N, mref, a, ptr(np.ascontiguousarray(P, np.float32)), ptr(np.ascontiguousarray(V, np.float32)),
                  ptr(np.ascontiguousarray(R, np.float32)), ptr(np.ascontiguousarray(D, np.float32)),
                  spring, touch, cap, 1 if sort else 0, C.byref(rep), ptr(lst), ptr(perm))
    return rep, lst[:rep.ppCount].copy(), perm


BUF = {"pos": 0, "vel": 1, "aux": 2, "q": 3, "mat": 4, "seats": 5, "fineA": 6, "forceA": 7, "monoA": 8,
       "coarseA": 9, "farA": 10, "fineB": 11, "forceB": 12, "monoB": 13, "pplist": 14, "ppforce": 15,
       "ppbox": 16, "ppslot": 17}
_DT = {"seats": np.uint32, "ppslot": np.int32}


class Engine:
    """The reference's step schedule on the CPU: src/nbody.js:376-636."""

    def __init__(self, sim, pos4, vel4, mat):
        self.h = lib().orc_engine_new(C.byref(sim), ptr(np.ascontiguousarray(pos4, np.float32)),
                                      ptr(np.ascontiguousarray(vel4, np.float32)),
                                      ptr(np.ascontiguousarray(mat, np.float32)))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_engine_free(self.h)
            self.h = None

    @property
    def sim(self):
        return lib().orc_engine_sim(self.h).contents

    def step(self, settle=False, kick=False):
        lib().orc_engine_step(self.h, int(settle), int(kick))

    def set_field(self, g, frozen=-1.0, invM=1.0, cpIron=1.0, on=True):
        gg = np.ascontiguousarray(g, np.float64)
        lib().orc_engine_set_field(self.h, int(on), ptr(gg), float(frozen), float(invM), float(cpIron))

    def rigid_step(self, dtF):
        lib().orc_engine_rigid_step(self.h, dtF)

    def set_pp(self, lst):
        lst = np.ascontiguousarray(lst, np.int32)
        lib().orc_engine_set_pp(self.h, ptr(lst), len(lst))

    def prime_mono(self, box, mono):
        m = np.ascontiguousarray(mono, np.float32)
        lib().orc_engine_prime_mono(self.h, box, ptr(m))

    def apply_perm(self, perm):
        p = np.ascontiguousarray(perm, np.int32)
        lib().orc_engine_apply_perm(self.h, ptr(p))

    def diag(self):
        N = self.sim.N
        d = np.zeros((N, 4), np.float32)
        lib().orc_engine_diag(self.h, ptr(d))
        return d

    def buf(self, name):
        n = C.c_long()
        p = lib().orc_engine_buf(self.h, BUF[name], C.byref(n))
        dt = _DT.get(name, np.float32)
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(n.value,)).view(dt).copy()
        if name in ("pos", "vel", "aux", "fineA", "forceA", "coarseA", "farA", "fineB", "forceB", "pplist",
                    "monoA", "monoB", "ppforce"):
            arr = arr.reshape(-1, 4)
        if name == "seats":
            arr = arr.reshape(-1, SEATS)
        return arr
