"""The crater page's field-gravity step on the GPU against the oracle.

simFS({gravity: 'field', frozen: true}) (src/glsl-sim.js:466-468, 490-492,
517-533) on the page's schedule (chicxulub.html:763-766): the contact grid on
even steps, the contact step with constant gravity on every step, no mesh.
The scene is a seeded patch of ground in the page's units with a frozen wall
and floor and an impactor on its way in.  As for the impact's step: the
neighbour counts are exact, the state is within 1e-5 of its scale after one
step and within 1e-4 after a dozen (float atomics sum the contacts in any
order); the frozen material does not move at all, and the gravity each
particle reports is the field exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scaled_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return 0.0 if s == 0 else float(np.abs(a - b).max() / s)


def test_field_step_matches_oracle(ccmod, orc):
    from cosmic_collisions_b200 import configs as cf
    sim, pos, vel, mat = cf.crater_patch(16384)
    e = orc.Engine(orc.Sim.from_buffer_copy(bytes(sim)), pos, vel, mat)
    e.set_field(cf.CRATER_G, cf.MAT_FROZEN)
    nb = ccmod.NBody(0)
    try:
        nb.upload(sim, pos, vel, mat)
        nb.set_field(cf.CRATER_G, cf.MAT_FROZEN)
        frozen = pos[:, 3] == cf.MAT_FROZEN
        g32 = np.array(cf.CRATER_G, np.float32)
        # one settle step and one free step from the same state: exact pair sets, state to 1e-5
        for settle in (True, False):
            if not settle:
                nb.write_state(pos=e.buf("pos"), vel=e.buf("vel"), q=e.buf("q"))
            nb.step(settle, False)
            e.step(settle, False)
            got = nb.read_state()
            assert np.array_equal(got["aux"][:, 3], e.buf("aux")[:, 3])
            assert got["aux"][:, 3].mean() > 5
            assert np.array_equal(got["aux"][:, :3], np.broadcast_to(g32, (len(pos), 3)))
            assert np.array_equal(e.buf("aux")[:, :3], got["aux"][:, :3])
            for name, a, b in (("pos", got["pos"][:, :3], e.buf("pos")[:, :3]),
                               ("vel", got["vel"][:, :3], e.buf("vel")[:, :3]),
                               ("T", got["vel"][:, 3], e.buf("vel")[:, 3]), ("q", got["q"], e.buf("q"))):
                assert scaled_err(a, b) < 1e-5, (name, settle)
        # a dozen more, the last eight replayed from a captured graph
        for _ in range(4):
            nb.step(False, False)
            e.step(False, False)
        nb.steps(8)
        for _ in range(8):
            e.step(False, False)
        got = nb.read_state()
        assert nb.sim.stepNo == e.sim.stepNo == 14
        for name, a, b in (("pos", got["pos"][:, :3], e.buf("pos")[:, :3]),
                           ("vel", got["vel"][:, :3], e.buf("vel")[:, :3])):
            assert scaled_err(a, b) < 1e-4, name
        # the wall and the floor stay exactly where they were; everything else falls or flies
        assert np.array_equal(got["pos"][frozen], pos[frozen])
        assert not np.any(got["vel"][frozen, :3])
        assert np.mean(got["pos"][~frozen, 1] != pos[~frozen, 1]) > 0.99
        imp = pos[:, 3] == cf.MAT_IMPACTOR
        assert got["pos"][imp, 1].mean() < pos[imp, 1].mean()
        # and back to the impact's step: the mesh gather returns
        nb.clear_field()
        assert nb.uniforms().field == 0.0
    finally:
        nb.close()
