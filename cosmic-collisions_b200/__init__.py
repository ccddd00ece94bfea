"""B200-native simulation step of cosmic-collisions.

The product is libccstep.so (hand-written sm_100a CUDA behind the C ABI of
include/ccstep.h); this package holds its sources (csrc/), its build script and
the host-side mirror of the reference engine object `CC.nbody`
(src/nbody.js:1095-1118).  Import it as ``cosmic_collisions_b200``.
"""
from ._lib import CCSError, lib, make_bodies, make_opt, fof, pair_table  # noqa: F401
from .nbody import Ensemble, NBody, mean_k  # noqa: F401
