"""The allocation-free P3M pass, ccs_pp_force_static, against the handle's own.

ccs_pp_force_static exists for callers that may not call cudaMalloc (a host
running inside a device-memory budget it does not own, or one that must not pay
the device-wide synchronisation cudaMalloc/cudaFree bring).  They pass their own
device buffers; the pass's scratch is a static device array shared by every
call.  This test gives it the list, boxes and table the handle's pass used
(ccs_set_pp), calls it twice in a row on the same buffers, and checks both
outputs against the handle's four slices to the tolerance the other parity
tests use (1e-5 of the field's scale).  It sits in a file of its own, collected
last, and needs nothing the earlier tests leave behind.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _handle_pass(cc, n):
    from cosmic_collisions_b200 import configs
    sim, pos, vel, mat = configs.gravity_sweep(N=16384)
    nb = cc.NBody(0)
    nb.upload(sim, pos, vel, mat)
    nb.pass_mesh()                                   # boxes(): the boxes the list is gathered against
    r = np.linalg.norm(pos[:, :3].astype(np.float64), axis=1)
    lst = np.flatnonzero(r > 1.3)[:n].astype(np.int32)
    assert len(lst) == n
    nb.set_pp(lst)                                   # the existing entry point: gather + pairwise pass
    return nb


def test_static_pass_matches_the_handle_pass_twice(ccmod):
    import torch
    n = 2000
    nb = _handle_pass(ccmod, n)
    try:
        u = nb.uniforms()
        want = nb.buffer("ppforce").reshape(4, ccmod._lib.PP_CAP, 4)[:, :n].astype(np.float64)
        assert np.abs(want[..., :3]).max() > 0
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
        lst4 = dev(nb.buffer("pplist")[:n])
        box = dev(nb.buffer("ppbox")[:n])
        f, p = ccmod.pair_table()
        tab = dev(np.stack([f, p], 1))
        out = torch.empty((4, n, 4), dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        P = lambda t: C.c_void_p(t.data_ptr())
        lib = ccmod.lib()
        scale = np.abs(want).max()
        for call in range(2):
            out.fill_(float("nan"))
            rc = lib.ccs_pp_force_static(P(lst4), P(box), n, P(tab), u.cut, u.a2, u.Gm, P(out), C.c_void_p(stream))
            assert rc == 0, rc
            torch.cuda.synchronize()
            got = out.cpu().numpy().astype(np.float64)
            assert np.all(np.isfinite(got)), call
            assert np.abs(got - want).max() <= TOL * scale, call
    finally:
        nb.close()


def test_static_pass_rejects_a_list_beyond_its_maximum(ccmod):
    import torch
    lib = ccmod.lib()
    t = torch.zeros(16, dtype=torch.float32, device="cuda")
    P = C.c_void_p(t.data_ptr())
    assert lib.ccs_pp_force_static(P, P, 2049, P, 0.9375, 1e-4, 1e-5, P, None) == -5   # CCS_E_RANGE
    assert lib.ccs_pp_force_static(None, None, 10, None, 0.9375, 1e-4, 1e-5, None, None) == -1   # CCS_E_ARG
    assert lib.ccs_pp_force_static(P, P, 0, P, 0.9375, 1e-4, 1e-5, P, None) == 0   # nothing to do
