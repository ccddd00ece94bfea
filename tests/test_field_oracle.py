"""The oracle's field-gravity step (the crater page's simFS({gravity: 'field', frozen: true}),
src/glsl-sim.js:466-468, 490-492, 517-533; schedule chicxulub.html:763-766), on the CPU.

What the shader states outright: the gravity a particle reports is the field,
the frozen material keeps its place and has no velocity, the rest moves, the
contact grid is rebuilt on even steps only, and switching the field off
restores the impact's mesh step.
"""
import numpy as np


def test_field_step_on_the_oracle(orc):
    from cosmic_collisions_b200 import configs as cf
    sim, pos, vel, mat = cf.crater_patch(16384)
    e = orc.Engine(orc.Sim.from_buffer_copy(bytes(sim)), pos, vel, mat)
    e.set_field(cf.CRATER_G, cf.MAT_FROZEN)
    frozen = pos[:, 3] == cf.MAT_FROZEN
    assert 0.1 < frozen.mean() < 0.5
    e.step(True, False)
    seats0 = e.buf("seats").copy()
    e.step(False, False)
    assert np.array_equal(e.buf("seats"), seats0)          # odd step: the grid keeps
    e.step(False, False)
    g32 = np.array(cf.CRATER_G, np.float32)
    aux = e.buf("aux")
    assert np.array_equal(aux[:, :3], np.broadcast_to(g32, (len(pos), 3)))
    assert aux[:, 3].mean() > 5                                 # the lattice touches
    P, V = e.buf("pos"), e.buf("vel")
    assert np.array_equal(P[frozen], pos[frozen])
    assert not np.any(V[frozen, :3])
    assert np.mean(P[~frozen, 1] != pos[~frozen, 1]) > 0.99
    imp = pos[:, 3] == cf.MAT_IMPACTOR
    assert np.all(V[imp, 1] < 0)                                # the impactor keeps coming down
    assert e.sim.stepNo == 3
    e.set_field(cf.CRATER_G, on=False)
    e.step(False, False)                                        # step 3: no mesh yet, no field either
    assert not np.any(e.buf("aux")[:, :3])
