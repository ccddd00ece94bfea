"""The C ABI: the library loads without a GPU and exports every entry point
include/ccstep.h declares (no compute is called here)."""
import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ccstep.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ccs_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_abi():
    names = declared_functions()
    assert "ccs_step" in names and "ccs_create" in names and len(names) >= 30


def test_library_exports_every_declared_symbol(ccmod):
    lib = ccmod.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header(ccmod):
    from cosmic_collisions_b200 import _lib
    assert sorted(_lib.EXPORTS) == declared_functions()


def test_struct_sizes_match_the_oracle(ccmod, orc):
    # the uniforms' common prefix is laid out identically in the library and the oracle
    from cosmic_collisions_b200 import _lib
    names = [f[0] for f in orc.Uni._fields_]
    assert names == [f[0] for f in _lib.Uniforms._fields_][:len(names)]
    assert C.sizeof(orc.Sim) == C.sizeof(_lib.Sim)
    assert [f[0] for f in orc.Sim._fields_] == [f[0] for f in _lib.Sim._fields_]
    assert C.sizeof(orc.Report) == C.sizeof(_lib.Report)


def test_version_and_errors_without_gpu(ccmod):
    lib = ccmod.lib()
    assert lib.ccs_version() == 1
    assert lib.ccs_destroy(None) == -1                       # CCS_E_ARG on a null handle
    assert lib.ccs_step(None, 0, 0) == -3                    # CCS_E_STATE: nothing built
    assert lib.ccs_last_error(None) == b"null handle"
    # host-side entry points validate their arguments before any work
    assert lib.ccs_pair_table(0, 1.0, None, None) == -1
    opt = ccmod.make_opt(16)
    sim = ccmod._lib.Sim()
    a = np.zeros(64, np.float32)
    assert lib.ccs_make_bodies(C.byref(opt), C.byref(sim), a.ctypes.data_as(C.c_void_p),
                               a.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p), None) == -5
