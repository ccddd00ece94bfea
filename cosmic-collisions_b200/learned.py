"""The learned pairwise correction: a BF16 network of the mesh's pair force.

No counterpart in the reference, which subtracts the placement-averaged table
of meshPairTable (src/nbody.js:48-109) inside PPFORCE_FS (src/glsl-sim.js:
738-750).  Here the mesh's pair force is the node-softened Newton force (what
it is exactly when the two particles share no mesh node) plus a network
R(d, s) -- d the pair offset in mesh cells, s the source's position in its
cell -- for the part that depends on direction and placement where they share
nodes; with it attached to an engine the P3M pass corrects loose pairs
inside NN_CUT_CELLS cells (half the plain cut) by m_j (N_a(d) - that) taper.  Everything runs on the device:
labels (binary64 mesh arithmetic of the isolated pair), sampling, training
(forward, backward and weight gradients on the tensor cores, Adam) and
inference inside the P3M pass.
"""
import ctypes as C

import numpy as np

from ._lib import NN_CUT_CELLS, NN_PARAMS, CCSError, check, lib, ptr

# flat parameter layout of include/ccstep.h
SLICES = {"W1": (0, (64, 6)), "b1": (384, (64,)), "W2": (448, (64, 64)), "b2": (4544, (64,)),
          "W3": (4608, (3, 64)), "b3": (4800, (3,))}


def unpack(params):
    """Flat parameters -> dict of named arrays (views)."""
    return {k: params[o:o + int(np.prod(shape))].reshape(shape) for k, (o, shape) in SLICES.items()}


class LearnedCorrection:
    """Owns one network and its training pool on a device (ccs_nn)."""

    def __init__(self, device=0, seed=2024):
        h = C.c_void_p()
        rc = lib().ccs_nn_create(int(device), int(seed) & 0xFFFFFFFF, C.byref(h))
        if rc != 0:
            raise CCSError("ccs_nn_create failed: %d" % rc)
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def _check(self, rc, what):
        if rc in (0, 1):
            return rc
        msg = lib().ccs_nn_last_error(self._h).decode() if self._h else ""
        raise CCSError("%s failed: %s %s" % (what, rc, msg))

    def close(self):
        if self._h:
            lib().ccs_nn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters -------------------------------------------------------
    def params(self):
        p = np.empty(NN_PARAMS, np.float32)
        self._check(lib().ccs_nn_get_params(self._h, ptr(p)), "ccs_nn_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.shape == (NN_PARAMS,)
        self._check(lib().ccs_nn_set_params(self._h, ptr(p)), "ccs_nn_set_params")

    # ---- the pool ---------------------------------------------------------
    def clear(self):
        self._check(lib().ccs_nn_clear(self._h), "ccs_nn_clear")

    def pool_size(self):
        return int(lib().ccs_nn_pool_size(self._h))

    def sample_state(self, nbody, count, seed):
        """count pairs of an engine's current particles inside the cut (both in box 0)."""
        self._check(lib().ccs_nn_sample_state(self._h, nbody.handle, int(count), int(seed) & 0xFFFFFFFF),
                    "ccs_nn_sample_state")

    def sample_uniform(self, count, seed):
        self._check(lib().ccs_nn_sample_uniform(self._h, int(count), int(seed) & 0xFFFFFFFF),
                    "ccs_nn_sample_uniform")

    def read_pool(self, first, n):
        rec = np.empty((n, 6), np.float32)
        lab = np.empty((n, 3), np.float32)
        self._check(lib().ccs_nn_read_pool(self._h, int(first), int(n), ptr(rec), ptr(lab)), "ccs_nn_read_pool")
        return rec, lab

    # ---- training and evaluation -------------------------------------------
    def train(self, first, n, epochs, tiles_per_cta=4, lr=2e-3):
        loss = np.empty(epochs, np.float32)
        self._check(lib().ccs_nn_train(self._h, int(first), int(n), int(epochs), int(tiles_per_cta),
                                       float(lr), ptr(loss)), "ccs_nn_train")
        return loss

    def forward(self, rec):
        rec = np.ascontiguousarray(rec, np.float32)
        out = np.empty((len(rec), 3), np.float32)
        self._check(lib().ccs_nn_forward(self._h, ptr(rec), len(rec), ptr(out)), "ccs_nn_forward")
        return out

    def labels(self, rec):
        rec = np.ascontiguousarray(rec, np.float32)
        out = np.empty((len(rec), 3), np.float32)
        self._check(lib().ccs_nn_labels(self._h, ptr(rec), len(rec), ptr(out)), "ccs_nn_labels")
        return out

    def grad(self, rec, lab):
        rec = np.ascontiguousarray(rec, np.float32)
        lab = np.ascontiguousarray(lab, np.float32)
        g = np.empty(NN_PARAMS, np.float32)
        loss = C.c_float()
        self._check(lib().ccs_nn_grad(self._h, ptr(rec), ptr(lab), len(rec), ptr(g), C.byref(loss)), "ccs_nn_grad")
        return g, float(loss.value)


def softened_newton(rec):
    """d / (r^2 + 1/2)^1.5 in cells^-2: the mesh's pair force when the two particles share no node (the
    0.5 FH^2 softening of CELL_FS); the network learns the isolated pair's mesh force less this."""
    d = np.asarray(rec, np.float64)[:, :3]
    return d / (((d * d).sum(1) + 0.5) ** 1.5)[:, None]


def table_model(rec, f_table, a_cells, cut_cells=5.0):
    """The plain pass's model of the mesh pair force in cells^-2: T.f / max(r^2, a^2) along d (PPFORCE_FS,
    src/glsl-sim.js:738-744), the pair table's force column read over 64 bins to the cut."""
    d = np.asarray(rec, np.float64)[:, :3]
    r = np.sqrt((d * d).sum(1))
    n = len(f_table)
    xx = np.clip(r / cut_cells * n - 0.5, 0.0, n - 1.0)
    k = xx.astype(int)
    k1 = np.minimum(k + 1, n - 1)
    f = np.asarray(f_table, np.float64)
    T = f[k] + (f[k1] - f[k]) * (xx - k)
    return d * (T / np.maximum(r * r, a_cells * a_cells) / np.maximum(r, 1e-300))[:, None]


__all__ = ["LearnedCorrection", "unpack", "softened_newton", "table_model", "NN_CUT_CELLS", "NN_PARAMS"]
