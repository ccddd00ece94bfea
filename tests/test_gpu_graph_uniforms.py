"""Captured graphs replay with each step's own uniforms.

The contact step and the contact grid take the step's uniforms as a by-value
argument, which a graph fixes at capture; before every replay the library sets
them again in those nodes (cudaGraphExecKernelNodeSetParams).  Settle, kick and
full steps share a graph (the phase flags are uniforms, not part of the key),
so a run that alternates them replays each graph with different uniforms: a
node left with its captured uniforms would keep damping, or keep kicking, and
the run would leave the same steps launched directly by an O(1) fraction of
the velocities' scale.  Timing the grid kernel (ccs_timing bit 1) makes every
step launch directly, which gives the reference run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scaled_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return 0.0 if s == 0 else float(np.abs(a - b).max() / s)


def test_graph_replays_take_each_steps_uniforms(ccmod):
    from cosmic_collisions_b200 import configs
    opt = configs.small_impact_opt(16384)
    runs = [ccmod.NBody(0) for _ in range(3)]   # graphs; direct; direct again (the run-to-run spread)
    try:
        for nb in runs:
            nb.build(opt)
            nb.settle_some(24)
            nb.sync()
        st = runs[0].read_state()
        for nb in runs[1:]:
            nb.write_state(pos=st["pos"], vel=st["vel"], aux=st["aux"], q=st["q"])
            ccmod.lib().ccs_timing(nb.handle, 0x2)   # time the grid: every launch direct
        pattern = [(1, 0), (0, 0), (1, 0), (0, 1), (0, 0), (1, 0), (0, 0), (0, 0)]
        for nb in runs:
            for k in range(24):   # one step at a time: each step's graph, replayed as the pattern comes round
                settle, kick = pattern[k % len(pattern)]
                nb.step(bool(settle), bool(kick))
                nb.sim.t += nb.sim.dt
            nb.steps(16)          # then whole 8-step blocks from their graphs, replayed once more
            nb.sync()
        got, ref, ref2 = (nb.read_state() for nb in runs)
        assert [nb.sim.stepNo for nb in runs] == [runs[0].sim.stepNo] * 3
        for k in ("pos", "vel"):
            spread = scaled_err(ref2[k][:, :3], ref[k][:, :3])
            err = scaled_err(got[k][:, :3], ref[k][:, :3])
            print("%s: graphs vs direct %.3e, direct vs direct %.3e" % (k, err, spread))
            assert err <= max(1e-4, 30 * spread), k
    finally:
        for nb in runs:
            nb.close()
