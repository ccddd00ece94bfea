"""Boundary calls added beside the step: placeBoxes as one validated call (ccs_set_boxes), the graph switch,
and the two halves of a split mesh step against the step launched whole.

A mesh step whose contact step is split (the contact walk beside the mesh chain, then the tail that adds
gravity and integrates) runs the same per-particle code as the whole step; the float atomics of the deposit
sum in an unspecified order, so the two agree to the state tolerance of the other parity tests (1e-5 of the
field's scale), and the neighbour counts exactly.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def scaled_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return 0.0 if s == 0 else float(np.abs(a - b).max() / s)


def settled(orc, N=16384, steps=8):
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(N))
    e = orc.Engine(sim, pos, vel, mat)
    for _ in range(steps):
        e.step(True, False)
    s = orc.Sim.from_buffer_copy(bytes(e.sim))
    com = (e.buf("pos")[:, :3].astype(np.float64) * e.buf("mat")[:, None]).sum(0) / e.buf("mat").sum()
    s.boxOn[0] = 1
    for k in range(3):
        s.boxCen[0][k] = com[k]
    s.boxT[0] = s.t
    s.phase, s.stepNo, s.impactT = 2, 0, s.t
    vel = e.buf("vel")
    rng = np.random.default_rng(5)
    vel[:, :3] += rng.normal(scale=0.05, size=(len(vel), 3)).astype(np.float32)
    return s, e.buf("pos"), vel, e.buf("mat")


def test_set_boxes_validates_then_sets(ccmod, orc):
    s, pos, vel, mat = settled(orc)
    nb = ccmod.NBody(0)
    try:
        nb.upload(ccmod._lib.Sim.from_buffer_copy(bytes(s)), pos, vel, mat)
        before = bytes(nb.sim)
        with pytest.raises(ccmod.CCSError):
            nb.set_boxes([{"on": 1, "cen": (0.0, math.nan, 0.0)}, {"on": 0, "cen": (0, 0, 0)}])
        with pytest.raises(ccmod.CCSError):
            nb.set_boxes([{"on": 2, "cen": (0, 0, 0)}, {"on": 0, "cen": (0, 0, 0)}])
        assert bytes(nb.sim) == before                     # a refused call changes nothing
        nb.set_boxes([{"on": 1, "cen": (0.1, 0.2, 0.3), "vel": (1.0, 0.0, 0.0), "t": 2.5},
                      {"on": 1, "cen": (4.0, 0.0, 0.0), "vel": (0.0, -1.0, 0.0), "t": 2.5,
                       "mono": (400.0, 0.0, 0.0, 100.0)}])
        sm = nb.sim
        assert (sm.boxOn[0], sm.boxOn[1]) == (1, 1)
        assert list(sm.boxCen[1]) == [4.0, 0.0, 0.0] and list(sm.boxVel[0]) == [1.0, 0.0, 0.0]
        assert sm.boxT[0] == sm.boxT[1] == 2.5
        assert np.array_equal(nb.buffer("monoB")[0], np.array([400.0, 0.0, 0.0, 100.0], np.float32))
    finally:
        nb.close()


def test_split_mesh_step_matches_whole(ccmod, orc):
    """The same mesh step three ways from one state: split beside the mesh (graphs off, no timing: the
    direct path), split in order with both halves timed, and whole (timing the deposit runs it whole)."""
    s, pos, vel, mat = settled(orc)
    lib = ccmod.lib()
    outs = []
    for mask in (0, 0x60, 0x04):
        nb = ccmod.NBody(0)
        try:
            nb.upload(ccmod._lib.Sim.from_buffer_copy(bytes(s)), pos, vel, mat)
            assert lib.ccs_set_graphs(nb.handle, 0) == 0
            assert lib.ccs_timing(nb.handle, mask) == 0
            nb.step(False, False)                          # step 0: grid + mesh + contacts + kick/drift
            nb.sync()
            if mask == 0x60:
                for kid in (5, 6):
                    tot, cnt = C.c_double(), C.c_int()
                    assert lib.ccs_timing_read(nb.handle, kid, C.byref(tot), C.byref(cnt)) == 0
                    assert cnt.value == 1 and tot.value > 0, kid
            outs.append(nb.read_state())
        finally:
            nb.close()
    whole = outs[2]
    for got in outs[:2]:
        assert np.array_equal(got["aux"][:, 3], whole["aux"][:, 3])
        for name in ("pos", "vel", "aux"):
            assert scaled_err(got[name][:, :3], whole[name][:, :3]) < TOL, name
        assert scaled_err(got["q"], whole["q"]) < TOL


def test_graphs_off_and_on_agree(ccmod, orc):
    s, pos, vel, mat = settled(orc)
    lib = ccmod.lib()
    outs = []
    for graphs in (1, 0):
        nb = ccmod.NBody(0)
        try:
            nb.upload(ccmod._lib.Sim.from_buffer_copy(bytes(s)), pos, vel, mat)
            assert lib.ccs_set_graphs(nb.handle, graphs) == 0
            for _ in range(9):
                nb.step(False, False)
                nb.sim.t += nb.sim.dt
            outs.append(nb.read_state())
        finally:
            nb.close()
    assert scaled_err(outs[0]["pos"][:, :3], outs[1]["pos"][:, :3]) < 1e-4
    assert scaled_err(outs[0]["vel"][:, :3], outs[1]["vel"][:, :3]) < 1e-4
    assert lib.ccs_set_graphs(None, 1) != 0
