"""The batched ensemble and the autotuner on the GPU.

* ccs_autotune measures launch shapes without moving the run: the state is
  bit-for-bit the same after it, and the chosen shapes step the run as the
  defaults do (to the spread of two lone runs: float atomics sum in any order);
* an ensemble round (one graph with every member's block as a branch) steps
  each member as ccs_steps steps it alone, for members of different sizes, and
  the members stay usable engines afterwards.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def settled(ccmod, N, steps=64):
    from cosmic_collisions_b200 import configs
    nb = ccmod.NBody(0)
    nb.build(configs.small_impact_opt(N))
    nb.settle_some(steps)
    nb.steps(8)
    nb.sync()
    return nb


def twin_spread(ccmod, sizes, lone, steps, prepare=None):
    """Per size, how far two lone runs of the same start drift apart in `steps` steps (float atomics sum in
    any order): a second lone twin of each size against the first one in `lone`."""
    out = {}
    for N, first in zip(sizes, lone):
        if N in out:
            continue
        twin = settled(ccmod, N)
        try:
            if prepare:
                prepare(twin)
            twin.steps(steps)
            twin.sync()
            st, s0 = twin.read_state(), first.read_state()
            out[N] = {k: np.abs(st[k][:, :3] - s0[k][:, :3]).max() for k in ("pos", "vel")}
        finally:
            twin.close()
    return out


def spread_ok(a, b, lone, scale):
    return np.abs(a - b).max() <= max(30 * lone, 2e-3 * scale)


def test_autotune_measures_without_moving_the_run(ccmod):
    runs = [settled(ccmod, 16384) for _ in range(3)]
    try:
        before = runs[0].read_state()
        choice = runs[0].autotune(reps=4)
        after = runs[0].read_state()
        assert choice["warps"] in (4, 8) and choice["cell_split"] in (2, 4, 8)
        for k in ("pos", "vel", "q"):
            assert np.array_equal(before[k], after[k])
        again = runs[1].autotune(reps=0)              # the same size: what was measured, no timing
        assert again == choice
        for nb in runs:
            nb.steps(16)
        st = [nb.read_state() for nb in runs]
    finally:
        for nb in runs:
            nb.close()
    for k in ("pos", "vel"):
        ref = st[2][k][:, :3].astype(np.float64)      # default shapes
        lone = np.abs(st[1][k][:, :3] - ref).max()    # tuned: the same shapes as run 0
        assert spread_ok(st[0][k][:, :3], ref, max(lone, 1e-7), np.abs(ref).max()), k


def test_ensemble_round_steps_members_as_alone(ccmod):
    sizes = [16384, 32768, 16384]
    members = [settled(ccmod, N) for N in sizes]
    lone = [settled(ccmod, N) for N in sizes]
    lone2 = settled(ccmod, 16384)
    try:
        ens = ccmod.Ensemble(members)
        ens.steps(16)
        ens.sync()
        for nb in lone + [lone2]:
            nb.steps(16)
            nb.sync()
        assert [nb.sim.stepNo for nb in members] == [nb.sim.stepNo for nb in lone]
        l2 = lone2.read_state()
        for a, b in zip(members, lone):
            sa, sb = a.read_state(), b.read_state()
            for k in ("pos", "vel"):
                ref = sb[k][:, :3].astype(np.float64)
                scale = np.abs(ref).max()
                diff = np.abs(sa[k][:, :3] - ref).max()
                spread = np.abs(l2[k][:, :3] - lone[0].read_state()[k][:, :3]).max()
                print("member N=%d %s: ensemble vs lone %.3e, lone vs lone %.3e, scale %.3e"
                      % (a.sim.N, k, diff, spread, scale))
                # float atomics sum in any order, and concurrency moves the order more than a rerun alone
                # does; a member that read another's buffers would be off by O(1) of the scale
                assert diff <= max(30 * spread, 2e-3 * scale), k
        # the members stay engines: a direct step, then another round
        members[0].step(False, False)
        members[0].sim.t += members[0].sim.dt
        with pytest.raises(ccmod.CCSError):
            ens.steps(8)                              # member 0 is off the block boundary
        for _ in range(7):
            members[0].step(False, False)
            members[0].sim.t += members[0].sim.dt
        ens.steps(8)
        ens.sync()
        for nb in members:
            assert np.isfinite(nb.read_state()["pos"]).all()
        ens.close()
    finally:
        for nb in members + lone + [lone2]:
            nb.close()


def test_ensemble_autotune_picks_a_shape_and_steps(ccmod):
    members = [settled(ccmod, N) for N in (16384, 32768)]
    try:
        ens = ccmod.Ensemble(members)
        before = [nb.sim.stepNo for nb in members]
        choice = ens.autotune(rounds=1)
        ens.sync()
        assert choice["warps"] in (4, 8) and choice["cell_split"] in (2, 4, 8)
        # one capture round and one timed round for each of the six shapes
        assert [nb.sim.stepNo - b for nb, b in zip(members, before)] == [6 * 2 * 8] * 2
        ens.steps(8)
        ens.sync()
        for nb in members:
            assert np.isfinite(nb.read_state()["pos"]).all()
        ens.close()
    finally:
        for nb in members:
            nb.close()


def test_persistent_round_steps_members_as_alone(ccmod):
    """The persistent form: each round one launch over every member's grids and contact steps (after the
    members' mesh chains), work items from per-member queues.  Members of different sizes step as they do
    alone, to the same spread as the branch form; every member's step time inside the rounds is reported."""
    sizes = [16384, 32768, 16384, 65536]
    members = [settled(ccmod, N) for N in sizes]
    lone = [settled(ccmod, N) for N in sizes]
    try:
        ens = ccmod.Ensemble(members)
        ens.set_persistent(True)
        ens.steps(16)
        ens.sync()
        assert ens.launch_count() == 2                  # one persistent launch a round
        ms = ens.step_ms()
        assert np.all(ms > 0) and np.all(ms < 50), ms
        for nb in lone:
            nb.steps(16)
            nb.sync()
        assert [nb.sim.stepNo for nb in members] == [nb.sim.stepNo for nb in lone]
        spread = twin_spread(ccmod, sizes, lone, 16)
        for a, b in zip(members, lone):
            sa, sb = a.read_state(), b.read_state()
            for k in ("pos", "vel"):
                ref = sb[k][:, :3].astype(np.float64)
                scale = np.abs(ref).max()
                diff = np.abs(sa[k][:, :3] - ref).max()
                sp = spread[a.sim.N][k]
                print("persistent member N=%d %s: vs lone %.3e, lone vs lone %.3e, scale %.3e"
                      % (a.sim.N, k, diff, sp, scale))
                assert diff <= max(30 * sp, 2e-3 * scale), k
            assert np.isfinite(sa["aux"]).all()
        # back to the branch form and on again: the members stay engines throughout
        ens.set_persistent(False)
        ens.steps(8)
        ens.set_persistent(True)
        ens.steps(8)
        ens.sync()
        for nb in members:
            assert np.isfinite(nb.read_state()["pos"]).all()
        ens.close()
    finally:
        for nb in members + lone:
            nb.close()


def test_persistent_round_first_step_counts_as_alone(ccmod):
    """After one persistent round the neighbour counts (the contact-pair sets' sizes, decided with exact
    arithmetic) of almost every particle equal a lone run's: the rounds' launches find the pairs the
    reference's walk finds.  (Float atomics in the mesh deposit move positions in the last bits, which can
    move a pair across the link radius in a handful of particles over 8 steps.)"""
    members = [settled(ccmod, N) for N in (16384, 32768)]
    lone = [settled(ccmod, N) for N in (16384, 32768)]
    try:
        ens = ccmod.Ensemble(members)
        ens.set_persistent(True)
        ens.steps(8)
        ens.sync()
        for nb in lone:
            nb.steps(8)
            nb.sync()
        for a, b in zip(members, lone):
            ca, cb = a.read_state()["aux"][:, 3], b.read_state()["aux"][:, 3]
            same = np.mean(ca == cb)
            print("N=%d: neighbour counts equal for %.5f of particles" % (a.sim.N, same))
            assert same > 0.999
        ens.close()
    finally:
        for nb in members + lone:
            nb.close()


def test_persistent_round_wait_bound_reports_and_leaves_the_device_usable(ccmod):
    """Every wait of the persistent round is bounded.  A bound far shorter than the round's ordinary waits for
    work (1 us) makes CTAs give up: the round is abandoned, the kernel ends, ccs_ensemble_sync reports
    CCS_E_KERNEL, and the device goes on working (a fresh engine steps and matches its twin)."""
    members = [settled(ccmod, N) for N in (16384, 16384)]
    try:
        ens = ccmod.Ensemble(members)
        ens.set_persistent(True)
        ens.set_wait_ns(1000)
        ens.steps(8)
        with pytest.raises(ccmod.CCSError, match="CCS_E_KERNEL|wait"):
            ens.sync()
        ens.close()
    finally:
        for nb in members:
            nb.close()
    a, b = settled(ccmod, 16384), settled(ccmod, 16384)
    try:
        a.steps(8)
        b.steps(8)
        sa, sb = a.read_state(), b.read_state()
        assert np.isfinite(sa["pos"]).all()
        assert np.abs(sa["pos"][:, :3] - sb["pos"][:, :3]).max() <= 1e-3
    finally:
        a.close()
        b.close()


def test_persistent_round_with_the_second_box_up(ccmod):
    """Members whose second mesh box is up (one box on each body: the gather from box B, the cross pull
    between the boxes, each particle reading the box whose centre is nearer) step in the persistent rounds
    as their lone twins do, to the same spread as the other ensemble tests."""
    def two_boxes(nb):
        s = nb.sim
        nb.set_boxes([{"on": 1, "cen": tuple(s.cen0), "t": s.t}, {"on": 1, "cen": tuple(s.cen1), "t": s.t}])

    sizes = [16384, 32768]
    members = [settled(ccmod, N) for N in sizes]
    lone = [settled(ccmod, N) for N in sizes]
    try:
        for nb in members + lone:
            two_boxes(nb)
        ens = ccmod.Ensemble(members)
        ens.set_persistent(True)
        ens.steps(16)
        ens.sync()
        for nb in lone:
            nb.steps(16)
            nb.sync()
        assert all(nb.uniforms().boxB > 0.5 for nb in members)
        spread = twin_spread(ccmod, sizes, lone, 16, prepare=two_boxes)
        for a, b in zip(members, lone):
            sa, sb = a.read_state(), b.read_state()
            for k in ("pos", "vel"):
                ref = sb[k][:, :3].astype(np.float64)
                scale = np.abs(ref).max()
                diff = np.abs(sa[k][:, :3] - ref).max()
                sp = spread[a.sim.N][k]
                print("two boxes, persistent member N=%d %s: vs lone %.3e, lone vs lone %.3e, scale %.3e"
                      % (a.sim.N, k, diff, sp, scale))
                assert diff <= max(30 * sp, 2e-3 * scale), k
        ens.close()
    finally:
        for nb in members + lone:
            nb.close()
