"""The contact walk's record and replay (ccs_set_contact_walk) against the oracle's walk.

The seat tables are rebuilt every second step (src/nbody.js:554); the step in between walks the same tables
again.  The rebuilding step records, per particle, the seats its cull kept; the next step replays that record,
with the walk's decisions recomputed (src/glsl-sim.js:415-450), wherever the particle has moved little enough
for the record to hold all its pairs, and walks the seat tables elsewhere.  Whichever way each particle goes,
its pair set and neighbour count are the oracle walk's over the same seats, and the step is the walking
step's to tolerance (the contacts are summed in another order):
1. one body moved further than its particles' records allow (they walk), the other less (they replay, and
   those that changed cell walk the cells their new cell adds);
2. one body moved further than any record allows: every particle walks;
3. a state written between the two steps: the record is not used.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-5


def settled(orc, N=16384, steps=8):
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(N))
    e = orc.Engine(sim, pos, vel, mat)
    for _ in range(steps):
        e.step(True, False)
    return orc.Sim.from_buffer_copy(bytes(e.sim)), e.buf("pos"), e.buf("vel"), e.buf("mat")


def moving_state(orc, target_move, impactor_move):
    """A settled 16k state on the impact's schedule whose first step is a kick: every particle takes its
    body's bulk velocity (no spin), which moves the target's particles `target_move` and the impactor's
    `impactor_move` radii in the step, each body in its own direction.  The record lets its owner have moved
    about 0.15 of a radius, and every particle about 0.23."""
    osim, pos, vel, mat = settled(orc)
    assert (pos[:, 3] < 3.5).sum() > 1000 and (pos[:, 3] > 3.5).sum() > 1000     # both bodies
    com = (pos[:, :3].astype(np.float64) * mat[:, None]).sum(0) / mat.sum()
    osim.boxOn[0] = 1
    for k in range(3):
        osim.boxCen[0][k] = com[k]
    osim.boxT[0] = osim.t
    osim.phase = 2
    osim.impactT = osim.t
    osim.stepNo = 0
    d0 = np.array([0.6, -0.48, 0.64])
    d1 = np.array([-0.36, 0.8, 0.48])
    for k in range(3):
        osim.spin0[k] = osim.spin1[k] = 0.0
        osim.bulk0[k] = d0[k] * target_move * osim.a / osim.dt
        osim.bulk1[k] = d1[k] * impactor_move * osim.a / osim.dt
    return osim, pos, vel, mat


def two_steps(ccmod, osim, pos, vel, mat, mode, write_between=False):
    """Two scheduled steps, the first a kick that rebuilds the grid, under contact-walk mode `mode`: the
    state after each, the seats the second walks, its pair sets (read out before it runs), the walk counts
    and the seats recorded per warp of 32 particles."""
    nb = ccmod.NBody(0)
    try:
        nb.upload(ccmod._lib.Sim.from_buffer_copy(bytes(osim)), pos, vel, mat)
        nb.set_contact_walk(mode)
        nb.step(False, True)
        mid = nb.read_state()
        if write_between:
            nb.write_state(pos=mid["pos"])
        seats = nb.buffer("seats")
        pairs = nb.contact_pairs(64)
        nb.step(False, False)
        end = nb.read_state()
        stats = nb.buffer("walkstats") if mode == 2 else None
        recorded = nb.buffer("walkcount")
    finally:
        nb.close()
    return mid, end, seats, pairs, stats, recorded


def check_against_oracle_and_walk(orc, osim, run, walk):
    mid, end, seats, (gc, gp), stats, recorded = run
    mid_w, end_w, seats_w, (wc, wp), _, _ = walk
    assert np.array_equal(seats, seats_w)
    assert np.array_equal(mid["pos"], mid_w["pos"])
    u = orc.make_uni(osim)
    oc, op = orc.contact_pairs(u, mid["pos"], seats, 64)
    assert oc.mean() > 5
    assert np.array_equal(gc, oc) and oc.max() <= 64
    assert np.array_equal(np.sort(gp, axis=1), np.sort(op, axis=1))
    assert np.array_equal(wc, oc)
    assert np.array_equal(end["aux"][:, 3], end_w["aux"][:, 3])        # every neighbour count of the step
    assert np.array_equal(end["aux"][:, 3], oc.astype(np.float32))
    dv = end["vel"][:, :3].astype(np.float64) - mid["vel"][:, :3]
    dvw = end_w["vel"][:, :3].astype(np.float64) - mid["vel"][:, :3]
    rms = np.sqrt((dvw ** 2).sum(1).mean())
    rel = np.linalg.norm(dv - dvw, axis=1) / np.maximum(np.linalg.norm(dvw, axis=1), rms)
    assert np.median(rel) < REL and np.percentile(rel, 99.9) < 10 * REL, (np.median(rel), rel.max())
    assert np.abs(end["pos"][:, :3] - end_w["pos"][:, :3]).max() <= 1e-5 * np.abs(end_w["pos"][:, :3]).max()
    return stats, recorded


def test_replay_matches_the_walk_for_every_way(ccmod, orc):
    osim, pos, vel, mat = moving_state(orc, 0.2, 0.05)
    run = two_steps(ccmod, osim, pos, vel, mat, 2)
    walk = two_steps(ccmod, osim, pos, vel, mat, 0)
    stats, recorded = check_against_oracle_and_walk(orc, osim, run, walk)
    print("replayed / replayed and walked new cells / walked:", stats.tolist(),
          "seats recorded per particle: mean %.1f, per warp max %d" % (recorded.mean() / 32, recorded.max()))
    assert stats.sum() == osim.N
    target = int((pos[:, 3] < 3.5).sum())
    assert stats[2] == target                 # the target's particles moved too far for their records
    assert stats[0] > 0 and stats[1] > 0      # the impactor's replayed, some of them walking a new cell's
    assert stats[0] + stats[1] == osim.N - target


def test_a_particle_moved_too_far_makes_every_particle_walk(ccmod, orc):
    osim, pos, vel, mat = moving_state(orc, 0.4, 0.05)
    run = two_steps(ccmod, osim, pos, vel, mat, 2)
    walk = two_steps(ccmod, osim, pos, vel, mat, 0)
    stats, _ = check_against_oracle_and_walk(orc, osim, run, walk)
    assert stats.tolist() == [0, 0, osim.N]


def test_a_state_written_between_the_steps_is_walked(ccmod, orc):
    osim, pos, vel, mat = moving_state(orc, 0.2, 0.05)
    run = two_steps(ccmod, osim, pos, vel, mat, 2, write_between=True)
    walk = two_steps(ccmod, osim, pos, vel, mat, 0, write_between=True)
    stats, _ = check_against_oracle_and_walk(orc, osim, run, walk)
    assert stats.tolist() == [0, 0, 0]       # the second step did not replay: it walked with the record off
