"""The learned pairwise correction on the GPU against its CPU oracle.

* labels: the device's binary64 mesh arithmetic of the isolated pair less the
  node-softened Newton force equals the oracle's (orc_nn_label, the
  restatement of meshPairTable's field(), src/nbody.js:60-91);
* the network's forward pass and its gradients, both through the tensor-core
  kernels, equal the numpy oracle's with the BF16 roundings at the same places;
* training on the device converges on synthetic pairs, and on pairs drawn
  from the impact the trained network's error where the two particles share
  a mesh node is below the placement-averaged pair table's; the learned pass
  at half the cut is within 1 % of the plain pass at the full cut on the
  loose list (its run-to-run spread);
* the learned P3M pass over a loose list equals the oracle's pass.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import nn_oracle as NO

pytestmark = pytest.mark.gpu


def records(n, seed, rmax=2.5):
    rng = np.random.default_rng(seed)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    r = rmax * rng.random(n) ** (1.0 / 3.0)
    return np.concatenate([u * r[:, None], rng.random((n, 3))], axis=1).astype(np.float32)


def shares_a_node(rec):
    """Whether the target's and the source's cloud-in-cell nodes overlap: the target's cell (floor(s - d))
    within one cell of the source's (cell 0) along every axis."""
    rec = np.asarray(rec, np.float64)
    return (np.abs(np.floor(rec[:, 3:6] - rec[:, :3])) <= 1).all(axis=1)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def net(ccmod):
    from cosmic_collisions_b200.learned import LearnedCorrection
    n = LearnedCorrection(0, seed=11)
    yield n
    n.close()


def test_labels_match_the_oracle(net, orc):
    rec = records(512, 1)
    got = net.labels(rec)
    mesh = orc.nn_labels(rec)
    want = NO.target(rec, mesh)
    # float32 of a binary64 difference: rounding relative to the mesh force itself
    assert np.abs(got - want).max() <= 2e-7 * np.abs(mesh).max() + 1e-9
    share = shares_a_node(rec)
    assert np.abs(want[share]).max() > 1e-2         # where the two share a mesh node there is something to learn
    assert np.abs(want[~share]).max() < 1e-5        # apart, the mesh's pair force is the softened Newton force


def test_forward_matches_the_oracle(net):
    p = net.params()
    rec = records(1000, 2)
    got = net.forward(rec)
    want = NO.forward(p, rec)
    assert got.shape == want.shape
    assert rel_l2(got, want) < 1e-2
    assert np.abs(got - want).max() < 3e-2 * np.abs(want).max()


def test_gradient_matches_the_oracle(net):
    p = net.params()
    rec = records(1000, 3)                          # 7 full tiles and a ragged one
    lab = (np.random.default_rng(4).normal(size=(1000, 3)) * 0.1).astype(np.float32)
    g, loss = net.grad(rec, lab)
    gw, lw = NO.grad(p, rec, lab)
    assert abs(loss - lw) <= 1e-3 * lw
    for name, (o, shape) in NO.SL.items():
        n = int(np.prod(shape))
        assert rel_l2(g[o:o + n], gw[o:o + n]) < 3e-2, name
    assert rel_l2(g, gw) < 2e-2


def test_training_learns_the_mesh_pair_force(net, orc):
    p0 = net.params()
    try:
        net.clear()
        net.sample_uniform(262144, seed=5)
        net.sample_uniform(16384, seed=6)           # held out
        prec, plab = net.read_pool(0, 262144)
        assert np.isfinite(prec).all() and np.isfinite(plab).all()
        loss = net.train(0, 262144, epochs=80, tiles_per_cta=1, lr=3e-3)
        assert np.isfinite(loss).all() and np.isfinite(net.params()).all()
        rec, lab = net.read_pool(262144, 16384)
        y = net.forward(rec)
        r = np.linalg.norm(rec[:, :3], axis=1)
        near = shares_a_node(rec) & (r > 0.1)
        mesh = lab + NO.softened_newton(rec)        # the isolated pair's mesh force
        f, _ = orc.pair_table()
        tab = NO.table_model(rec, f, 0.075)         # the plain pass's model (a = 0.075 cells at 262k)
        rms = lambda v: float(np.sqrt((v ** 2).sum(1).mean()))
        e_net, e_tab = rms((y - lab)[near]), rms((mesh - tab)[near])
        print("loss %.3e -> %.3e; pairs sharing a node: label rms %.3e, table error %.3e, network error %.3e"
              % (loss[0], loss[-1], rms(lab[near]), e_tab, e_net))
        assert loss[-1] < loss[0] / 5
        assert e_net < 2 * e_tab          # synthetic pairs, uniform in the ball: training converges
    finally:
        net.set_params(p0)
        net.clear()


@pytest.fixture(scope="module")
def impact_net(ccmod):
    """A network trained as the benchmark trains it: pairs drawn from the full impact at 262,144 particles
    at full-phase steps 0, 1000 and 3000 (4 M each), 24 epochs at a learning rate of 4e-3; a held-out draw
    from the last snapshot.  Returns (network, held-out records, labels, the run's particle radius in
    cells)."""
    from cosmic_collisions_b200 import configs
    from cosmic_collisions_b200.learned import LearnedCorrection
    n = LearnedCorrection(0, seed=2024)
    nb = ccmod.NBody(0)
    try:
        nb.build(ccmod.make_opt(**configs.full_impact_opt(262144)))
        while nb.sim.phase == 0:
            nb.settle_some(64)
        nb.analyze(True)
        while nb.sim.phase == 1:
            nb.rigid_step(0.01)
        done = 0
        for k, snap in enumerate((0, 1000, 3000)):
            while done < snap:
                step = min(360, snap - done)
                nb.steps(step)
                done += step
                nb.analyze(True)
            n.sample_state(nb, 4_000_000, seed=1000 + k)
        n.sample_state(nb, 262_144, seed=9999)
        a_cells = nb.sim.a / (12.0 / 64.0)
    finally:
        nb.close()
    n.train(0, 12_000_000, epochs=24, tiles_per_cta=1, lr=4e-3)
    rec, lab = n.read_pool(12_000_000, 262_144)
    live = np.isfinite(rec[:, 0])
    yield n, rec[live], lab[live], a_cells
    n.close()


def test_network_beats_the_table_on_impact_pairs(impact_net, orc):
    """Where the two particles share a mesh node -- the only place the mesh's pair force is not the
    node-softened Newton force -- the trained network's error is below the placement-averaged table's
    (meshPairTable, src/nbody.js:48-109) on held-out pairs of the impact."""
    net, rec, lab, a_cells = impact_net
    y = net.forward(rec)
    near = shares_a_node(rec)
    mesh = lab + NO.softened_newton(rec)
    f, _ = orc.pair_table()
    tab = NO.table_model(rec, f, a_cells)
    rms = lambda v: float(np.sqrt((v ** 2).sum(1).mean()))
    e_net, e_tab = rms((y - lab)[near]), rms((mesh - tab)[near])
    print("held-out impact pairs sharing a node: %d; table error %.4e, network error %.4e (%.1f %% lower)"
          % (near.sum(), e_tab, e_net, 100 * (1 - e_net / e_tab)))
    assert near.sum() > 10000
    assert e_net < 0.8 * e_tab       # measured: about a third below the table


def test_learned_pass_is_no_worse_than_the_plain_pass(impact_net, ccmod):
    """On the gravity sweep, the loose list's force error (against the binary64 direct sum) with the learned
    pass -- the network's model of the mesh's pull inside half the cut, the table beyond -- is no worse than
    the plain pass's (the table everywhere), to 1 %.  The network is trained on pairs drawn from a simulated
    impact whose float-atomic mesh sums differ in the last bits from run to run, so the trained network, and
    the learned pass's median error with it, varies by about 0.2 % between runs (measured 5.772e-3 and
    5.792e-3 against the plain pass's 5.782e-3); the bound holds that spread and no more."""
    from cosmic_collisions_b200 import configs
    net = impact_net[0]
    N = 262144
    sim, pos, vel, mat = configs.gravity_sweep(N=N)
    out = {}
    for learned in (False, True):
        nb = ccmod.NBody(0)
        try:
            nb.upload(sim, pos, vel, mat)
            if learned:
                nb.set_pp_nn(net)
            nb.pass_slots()
            nb.pass_diag()
            D = nb.buffer("diag")
            s = nb.sim
            rep, lst, _ = ccmod.fof(s.N, s.m, s.a, pos, vel, mat, D, s.k, 2 * s.a)
            nb.set_pp(lst, rep.ppLoose)
            nb.pass_sim(False, False, 0.0)
            g = nb.read_state()["aux"][:, :3].astype(np.float64)
            idx = np.sort(np.asarray(lst, np.int64)[::8]).astype(np.int32)     # a sample of the loose list
            ref, _ = nb.direct_sum(idx)
            if learned:
                nb.set_pp_nn(None)
        finally:
            nb.close()
        out[learned] = float(np.median(np.linalg.norm(g[idx] - ref, axis=1) / np.linalg.norm(ref, axis=1)))
    print("loose-list median force error: plain %.4e, learned inside 2.5 cells %.4e" % (out[False], out[True]))
    assert out[True] <= 1.01 * out[False]


def test_learned_pass_matches_the_oracle(net, ccmod, orc):
    osim, pos, vel, mat, home = orc.build_run(orc.make_opt(16384))
    rng = np.random.default_rng(8)
    pos = pos.copy()
    sel = np.sort(rng.choice(osim.N, 600, replace=False)).astype(np.int32)
    pos[sel, :3] *= np.float32(1.6)                 # spread out: pairs inside and beyond the cut
    com = (pos[:, :3].astype(np.float64) * mat[:, None]).sum(0) / mat.sum()
    osim.boxOn[0] = 1
    for k in range(3):
        osim.boxCen[0][k] = com[k]
    osim.boxT[0] = osim.t
    nb = ccmod.NBody(0)
    try:
        nb.upload(ccmod._lib.Sim.from_buffer_copy(bytes(osim)), pos, vel, mat, home)
        nb.pass_mesh()                              # boxes()
        nb.set_pp_nn(net)
        nb.set_pp(sel)
        got = nb.buffer("ppforce")
        lst = nb.buffer("pplist")
        box = nb.buffer("ppbox")
        lu = ccmod._lib.Uniforms()
        ccmod._lib.check(ccmod._lib.lib().ccs_get_uniforms(nb.handle, C.byref(lu)), nb.handle, "uniforms")
        nb.set_pp_nn(None)
        nb.set_pp(sel)
        plain = nb.buffer("ppforce")
    finally:
        nb.close()
    u = orc.Uni.from_buffer_copy(bytes(lu))
    f, pt = orc.pair_table()
    tab = np.stack([f, pt], 1).astype(np.float32)
    n = len(sel)
    want = NO.pp_nn(u, lst[:n], box[:n], n, tab, net.params(), orc.box_of)
    g0 = got.reshape(4, -1, 4)
    assert np.abs(g0[1:]).max() == 0.0              # one slice
    acc = g0[0, :n, :3].astype(np.float64)
    scale = np.abs(want[:, :3]).max()
    assert scale > 0
    # the network's BF16 activations round the same way on both sides except at ties the FP32 sums
    # land on differently: a few 1e-3 of the learned term, far below the Newton term
    assert np.abs(acc - want[:, :3]).max() < 5e-3 * scale
    assert np.abs(g0[0, :n, 3] - want[:, 3]).max() < 1e-4 * np.abs(want[:, 3]).max()
    # detached, the plain pass is back: four slices again
    assert np.abs(plain.reshape(4, -1, 4)[1:]).max() > 0
