"""ctypes binding of libccstep.so (include/ccstep.h).

The library is the product: there is no CPU fallback.  Loading fails loudly
when the shared object is missing or does not export the ABI.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libccstep.so")

CCS_OK = 0
CCS_NOT_READY = 1
CCS_E = {-1: "CCS_E_ARG", -2: "CCS_E_CUDA", -3: "CCS_E_STATE", -4: "CCS_E_NOMEM", -5: "CCS_E_RANGE",
         -6: "CCS_E_KERNEL"}
SEATS = 8
PP_CAP = 8192
PP_BINS = 64
MAX_N = 262144
SEAT_EMPTY = 0xBF800000
BOOKS = 12
FINE = 64 * 64 * 64
COARSE = 4096

BUF = {"seats": 5, "fineA": 6, "forceA": 7, "monoA": 8, "coarseA": 9, "farA": 10, "fineB": 11, "forceB": 12,
       "monoB": 13, "pplist": 14, "ppforce": 15, "ppbox": 16, "ppslot": 17, "diag": 18, "cellof": 19,
       "tide0A": 20, "tide1A": 21, "ppall": 22, "walkstats": 23, "walkcount": 24, "tide2A": 25, "fineQA": 26}

# every symbol include/ccstep.h declares
EXPORTS = ["ccs_version", "ccs_last_error", "ccs_create", "ccs_destroy", "ccs_make_bodies", "ccs_make_bodies_device",
           "ccs_build",
           "ccs_sim_ptr", "ccs_set_static", "ccs_get_uniforms", "ccs_set_mesh_every", "ccs_step", "ccs_steps",
           "ccs_settle_some", "ccs_rigid_step", "ccs_set_pp", "ccs_prime_mono", "ccs_apply_perm",
           "ccs_sort_morton", "ccs_diag_async", "ccs_poll", "ccs_fof", "ccs_pair_table", "ccs_read_state",
           "ccs_write_state", "ccs_device_ptrs", "ccs_books", "ccs_read_buffer", "ccs_pass_slots",
           "ccs_pass_mesh", "ccs_pass_pp", "ccs_pass_sim", "ccs_pass_diag", "ccs_advance_host", "ccs_sync",
           "ccs_timing", "ccs_timing_read", "ccs_launch_count", "ccs_direct_sum", "ccs_pp_force_static",
           "ccs_nn_create", "ccs_nn_destroy", "ccs_nn_last_error", "ccs_nn_set_params", "ccs_nn_get_params",
           "ccs_nn_clear", "ccs_nn_pool_size", "ccs_nn_sample_state", "ccs_nn_sample_uniform", "ccs_nn_read_pool",
           "ccs_nn_train", "ccs_nn_forward", "ccs_nn_labels", "ccs_nn_grad", "ccs_set_pp_nn", "ccs_autotune",
           "ccs_ensemble_create", "ccs_ensemble_destroy", "ccs_ensemble_last_error", "ccs_ensemble_steps",
           "ccs_ensemble_sync", "ccs_ensemble_autotune", "ccs_fof_device", "ccs_set_field",
           "ccs_checkpoint_size", "ccs_checkpoint_save", "ccs_checkpoint_load", "ccs_timing_every",
           "ccs_set_boxes", "ccs_set_graphs", "ccs_contact_pairs", "ccs_set_pp_split",
           "ccs_set_contact_walk", "ccs_ensemble_set_persistent", "ccs_ensemble_step_ms",
           "ccs_ensemble_launch_count", "ccs_ensemble_set_wait_ns", "ccs_pp_list_force",
           "ccs_set_pp_split_sym", "ccs_pp_split_pairs"]
NN_PARAMS = 4803
NN_CUT_CELLS = 2.5


class Uniforms(C.Structure):
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
                ("field", C.c_float), ("gField", C.c_float * 3), ("frozen", C.c_float),
                ("ppCount", C.c_int),
                ("rot0", C.c_float * 9), ("rot1", C.c_float * 9), ("rdt", C.c_float), ("ppSplit", C.c_int)]


class Sim(C.Structure):
    """The run's scalars: the reference's `sim` object (src/nbody.js:212-234)."""
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


class BuildOpt(C.Structure):
    _fields_ = [("N", C.c_int),
                ("q", C.c_double), ("dens", C.c_double), ("core", C.c_double), ("coreImp", C.c_double),
                ("spin0", C.c_double), ("spin1", C.c_double), ("angle", C.c_double), ("incl", C.c_double),
                ("vfac", C.c_double), ("rest", C.c_double),
                ("n2", C.c_int), ("mImp", C.c_double),
                ("mTarget", C.c_double), ("rhoR", C.c_double), ("rhoCrust", C.c_double),
                ("crustFrac", C.c_double)]


class Report(C.Structure):
    """fof()'s report, src/nbody.js:888-892."""
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


class Box(C.Structure):
    """One mesh box as placeBoxes leaves it (sim.boxes[b], src/nbody.js:361-374)."""
    _fields_ = [("on", C.c_int), ("cen", C.c_double * 3), ("vel", C.c_double * 3), ("t", C.c_double),
                ("primeMono", C.c_int), ("mono", C.c_float * 4)]


class DeviceBuffers(C.Structure):
    _fields_ = [("pos4", C.c_void_p), ("vel4", C.c_void_p), ("aux4", C.c_void_p), ("q", C.c_void_p),
                ("mat", C.c_void_p), ("home4", C.c_void_p), ("force", C.c_void_p * 2), ("mono", C.c_void_p * 2),
                ("stream", C.c_void_p)]


class CCSError(RuntimeError):
    pass


_lib = None


def lib():
    """Load libccstep.so; raise if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CCSError("libccstep.so is not built: run `python cosmic-collisions_b200/build.py` "
                       "(or __graft_entry__.build()); there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    for name in EXPORTS:
        if not hasattr(L, name):
            raise CCSError("libccstep.so does not export " + name)
    P, H, I, D = C.c_void_p, C.c_void_p, C.c_int, C.c_double
    sig = {
        "ccs_version": (I, []),
        "ccs_last_error": (C.c_char_p, [H]),
        "ccs_create": (I, [I, C.POINTER(C.c_void_p)]),
        "ccs_destroy": (I, [H]),
        "ccs_make_bodies": (I, [C.POINTER(BuildOpt), C.POINTER(Sim), P, P, P, P]),
        "ccs_make_bodies_device": (I, [I, C.POINTER(BuildOpt), C.POINTER(Sim), P, P, P, P]),
        "ccs_build": (I, [H, C.POINTER(Sim), P, P, P, P]),
        "ccs_sim_ptr": (C.POINTER(Sim), [H]),
        "ccs_set_static": (I, [H]),
        "ccs_get_uniforms": (I, [H, C.POINTER(Uniforms)]),
        "ccs_set_mesh_every": (I, [H, I]),
        "ccs_step": (I, [H, I, I]),
        "ccs_steps": (I, [H, I]),
        "ccs_settle_some": (I, [H, I]),
        "ccs_rigid_step": (I, [H, D]),
        "ccs_set_pp": (I, [H, P, I, I]),
        "ccs_prime_mono": (I, [H, I, P]),
        "ccs_set_boxes": (I, [H, C.POINTER(Box)]),
        "ccs_apply_perm": (I, [H, P]),
        "ccs_sort_morton": (I, [H, P, P, P]),
        "ccs_diag_async": (I, [H]),
        "ccs_poll": (I, [H, P, P, P]),
        "ccs_fof": (I, [I, D, D, P, P, P, P, D, D, I, I, C.POINTER(Report), P, P]),
        "ccs_pair_table": (I, [I, D, P, P]),
        "ccs_read_state": (I, [H, P, P, P, P, P]),
        "ccs_write_state": (I, [H, P, P, P, P, P]),
        "ccs_device_ptrs": (I, [H, C.POINTER(DeviceBuffers)]),
        "ccs_books": (I, [H, I, P]),
        "ccs_read_buffer": (I, [H, I, P, C.c_size_t]),
        "ccs_pass_slots": (I, [H]),
        "ccs_pass_mesh": (I, [H]),
        "ccs_pass_pp": (I, [H]),
        "ccs_pass_sim": (I, [H, I, I, D]),
        "ccs_pass_diag": (I, [H]),
        "ccs_advance_host": (I, [H, P, P, P, I, P, P, P, P]),
        "ccs_sync": (I, [H]),
        "ccs_timing": (I, [H, I]),
        "ccs_timing_read": (I, [H, I, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
        "ccs_launch_count": (C.c_int64, [H]),
        "ccs_direct_sum": (I, [H, P, I, P, P]),
        "ccs_pp_force_static": (I, [P, P, I, P, C.c_float, C.c_float, C.c_float, P, P]),
        "ccs_nn_create": (I, [I, C.c_uint32, C.POINTER(C.c_void_p)]),
        "ccs_nn_destroy": (I, [H]),
        "ccs_nn_last_error": (C.c_char_p, [H]),
        "ccs_nn_set_params": (I, [H, P]),
        "ccs_nn_get_params": (I, [H, P]),
        "ccs_nn_clear": (I, [H]),
        "ccs_nn_pool_size": (C.c_int64, [H]),
        "ccs_nn_sample_state": (I, [H, H, C.c_int64, C.c_uint32]),
        "ccs_nn_sample_uniform": (I, [H, C.c_int64, C.c_uint32]),
        "ccs_nn_read_pool": (I, [H, C.c_int64, C.c_int64, P, P]),
        "ccs_nn_train": (I, [H, C.c_int64, C.c_int64, I, I, C.c_float, P]),
        "ccs_nn_forward": (I, [H, P, C.c_int64, P]),
        "ccs_nn_labels": (I, [H, P, C.c_int64, P]),
        "ccs_nn_grad": (I, [H, P, P, C.c_int64, P, P]),
        "ccs_set_pp_nn": (I, [H, H]),
        "ccs_autotune": (I, [H, I, P]),
        "ccs_ensemble_create": (I, [P, I, C.POINTER(C.c_void_p)]),
        "ccs_ensemble_destroy": (I, [H]),
        "ccs_ensemble_last_error": (C.c_char_p, [H]),
        "ccs_ensemble_steps": (I, [H, I]),
        "ccs_ensemble_sync": (I, [H]),
        "ccs_ensemble_autotune": (I, [H, I, P]),
        "ccs_fof_device": (I, [H, D, D, I, I, C.POINTER(Report), P, P]),
        "ccs_set_field": (I, [H, I, P, D, D, D]),
        "ccs_checkpoint_size": (I, [H, C.c_size_t, C.POINTER(C.c_size_t)]),
        "ccs_checkpoint_save": (I, [H, P, C.c_size_t, P, C.c_size_t]),
        "ccs_checkpoint_load": (I, [H, P, C.c_size_t]),
        "ccs_timing_every": (I, [H, I]),
        "ccs_set_graphs": (I, [H, I]),
        "ccs_contact_pairs": (I, [H, I, P, P]),
        "ccs_set_pp_split": (I, [H, I]),
        "ccs_set_contact_walk": (I, [H, I]),
        "ccs_ensemble_set_persistent": (I, [H, I]),
        "ccs_ensemble_step_ms": (I, [H, P, I]),
        "ccs_ensemble_launch_count": (C.c_int64, [H]),
        "ccs_ensemble_set_wait_ns": (I, [H, C.c_uint64]),
        "ccs_pp_list_force": (I, [H, P, I, P]),
        "ccs_set_pp_split_sym": (I, [H, I]),
        "ccs_pp_split_pairs": (I, [H, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def ptr(a):
    """A numpy array's data pointer (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the library must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def check(rc, h=None, what=""):
    if rc in (CCS_OK, CCS_NOT_READY):
        return rc
    msg = lib().ccs_last_error(h).decode() if h else ""
    raise CCSError("%s failed: %s %s" % (what, CCS_E.get(rc, rc), msg))


def make_opt(N, q=0.1, dens=0.75, core=0.325, coreImp=None, spin0=0.18, spin1=0.20, angle=45.0, incl=50.0,
             vfac=1.05, rest=0.3, n2=0, mImp=0.0, mTarget=0.0, rhoR=0.0, rhoCrust=0.0, crustFrac=0.0):
    """build(opt) options; defaults are the giant-impact page's S (index.html:177-178)."""
    return BuildOpt(int(N), q, dens, core, -1.0 if coreImp is None else coreImp, spin0, spin1, angle, incl, vfac,
                    rest, int(n2), mImp, mTarget, rhoR, rhoCrust, crustFrac)


def make_bodies(opt, device=None):
    """Host builder (src/nbody.js:114-250): (sim, pos4, vel4, mat, home4).  With a device index the
    overlap relaxation runs on that GPU (ccs_make_bodies_device)."""
    N = opt.N
    sim = Sim()
    pos = np.zeros((N, 4), np.float32)
    vel = np.zeros((N, 4), np.float32)
    mat = np.zeros(N, np.float32)
    home = np.zeros((N, 4), np.float32)
    if device is None:
        check(lib().ccs_make_bodies(C.byref(opt), C.byref(sim), ptr(pos), ptr(vel), ptr(mat), ptr(home)),
              what="ccs_make_bodies")
    else:
        check(lib().ccs_make_bodies_device(int(device), C.byref(opt), C.byref(sim), ptr(pos), ptr(vel), ptr(mat),
                                           ptr(home)), what="ccs_make_bodies_device")
    return sim, pos, vel, mat, home


def pair_table(bins=PP_BINS, cut=5 * 12.0 / 64):
    f = np.zeros(bins, np.float32)
    p = np.zeros(bins, np.float32)
    check(lib().ccs_pair_table(bins, cut, ptr(f), ptr(p)), what="ccs_pair_table")
    return f, p


def fof(N, mref, a, P, V, R, D, spring, touch, cap=PP_CAP, sort=False):
    """Host analysis fof() (src/nbody.js:646-893): (report, loose list, perm or None)."""
    rep = Report()
    lst = np.zeros(max(cap, 1), np.int32)
    perm = np.zeros(N, np.int32) if sort else None
    check(lib().ccs_fof(N, mref, a, ptr(np.ascontiguousarray(P, np.float32)),
                        ptr(np.ascontiguousarray(V, np.float32)), ptr(np.ascontiguousarray(R, np.float32)),
                        ptr(np.ascontiguousarray(D, np.float32)), spring, touch, cap, 1 if sort else 0,
                        C.byref(rep), ptr(lst), ptr(perm)), what="ccs_fof")
    return rep, lst[:rep.ppCount].copy(), perm
