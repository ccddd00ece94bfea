"""The sm_100a library against the CPU oracle on the same seeded inputs.

Bit-exact (integer, index and byte work, and what decides it): the contact
grid (every seat word), the neighbour counts of the contact step, the coarse
sums given the same fine mesh, the P3M list and box gather, the loose-list
maps, the rigid carry, the permutation and the Morton order, the diag seat
counts.  To tolerance -- 1e-5 of the field's scale, per the target "forces and
state within 1e-5 relative after one step" -- every floating-point field: the
kernels use FMA and fast reciprocals where the oracle rounds every operation,
and the cloud-in-cell deposit sums in an unspecified order (as the
reference's additive blending does).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def to_lib_sim(cc, osim):
    return cc._lib.Sim.from_buffer_copy(bytes(osim))


def scaled_err(a, b):
    """max |a - b| over the field's largest magnitude."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return 0.0 if s == 0 else float(np.abs(a - b).max() / s)


@pytest.fixture(scope="module")
def nb(ccmod):
    n = ccmod.NBody(0)
    yield n
    n.close()


def oracle_state(orc, N=16384, settle_steps=24, **kw):
    """A settled state from the oracle's own engine: (sim, pos, vel, mat, q)."""
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(N, **kw))
    e = orc.Engine(sim, pos, vel, mat)
    for _ in range(settle_steps):
        e.step(True, False)
    s = orc.Sim.from_buffer_copy(bytes(e.sim))
    return s, e.buf("pos"), e.buf("vel"), e.buf("mat"), e.buf("q")


def with_motion(pos, vel, seed=1, scale=0.3):
    """Give the particles velocities so the dashpot and the heat have work."""
    rng = np.random.default_rng(seed)
    v = vel.copy()
    v[:, :3] += rng.normal(scale=scale, size=(len(v), 3)).astype(np.float32)
    v[:, 3] = rng.uniform(300, 3000, size=len(v)).astype(np.float32)   # temperatures, for the heat flow
    return v


def uni_for(orc, osim):
    return orc.make_uni(osim)


@pytest.mark.parametrize("N", [16384, 262144])
def test_contact_grid_is_exact(nb, ccmod, orc, N):
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(N))
    nb.upload(to_lib_sim(ccmod, sim), pos, vel, mat, home)
    nb.pass_slots()
    got = nb.buffer("seats")
    u = uni_for(orc, sim)
    want = orc.slots(u, pos)
    assert got.shape == want.shape
    assert np.array_equal(got, want)
    # a second rebuild into the other table (which the first one retired) is exact too
    pos2 = pos.copy()
    pos2[:, :3] += np.float32(0.3) * np.float32(sim.a)
    nb.write_state(pos=pos2)
    nb.pass_slots()
    assert np.array_equal(nb.buffer("seats"), orc.slots(u, pos2))
    nb.pass_slots()
    assert np.array_equal(nb.buffer("seats"), orc.slots(u, pos2))


@pytest.mark.parametrize("order", ["scattered", "by_cell"])
def test_contact_grid_overfull_cells(nb, ccmod, orc, order):
    # a dense blob overfills cells: the eight lowest indices keep the seats.  "by_cell" numbers each cell's
    # particles consecutively, so a warp holds up to 32 of one cell's particles and most start past seat 0
    # or are unseated at once
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(16384))
    rng = np.random.default_rng(4)
    pos = pos.copy()
    pos[:, :3] = rng.normal(scale=0.1, size=(len(pos), 3)).astype(np.float32)
    if order == "by_cell":
        key = np.floor(pos[:, :3] / np.float32(uni_for(orc, sim).cell)).astype(np.int64)
        pos = pos[np.lexsort((key[:, 0], key[:, 1], key[:, 2]))]
    nb.upload(to_lib_sim(ccmod, sim), pos, vel, mat)
    nb.pass_slots()
    want = orc.slots(uni_for(orc, sim), pos)
    got = nb.buffer("seats")
    assert (want[:, 7] != orc.EMPTY).sum() > 100
    assert np.array_equal(got, want)


@pytest.mark.parametrize("settle,kick", [(0, 0), (1, 0), (0, 1)])
def test_contact_step(nb, ccmod, orc, settle, kick):
    osim, pos, vel, mat, q = oracle_state(orc)
    vel = with_motion(pos, vel)
    q = np.random.default_rng(3).uniform(0, 1e-4, size=len(q)).astype(np.float32)
    osim.bulk0[0], osim.bulk1[2] = 0.2, -0.3
    nb.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
    nb.write_state(q=q)
    nb.pass_slots()
    gc, gp = nb.contact_pairs(64)            # the pair sets of this state, before the step moves it
    nb.pass_sim(settle, kick, 0.0)
    got = nb.read_state()
    # the oracle: same seats, zero meshes, gdt = 0
    u = uni_for(orc, osim)
    u.settle, u.kick, u.gdt = float(settle), float(kick), 0.0
    for k in range(3):
        u.bulk0[k], u.bulk1[k] = osim.bulk0[k], osim.bulk1[k]
        u.cen0[k], u.cen1[k] = osim.cen0[k], osim.cen1[k]
    seats = orc.slots(u, pos)
    N = osim.N
    zf = np.zeros(((orc.FINE + 1), 4), np.float32)
    z4 = np.zeros(4, np.float32)
    slot = np.full(N, -1, np.int32)
    ppf = np.zeros((4 * orc.PP_CAP, 4), np.float32)
    po, vo, ao, qo = (np.zeros((N, 4), np.float32), np.zeros((N, 4), np.float32), np.zeros((N, 4), np.float32),
                      np.zeros(N, np.float32))
    P = orc.ptr
    orc.lib().orc_sim_pass(C.byref(u), P(pos), P(vel), P(mat), P(q), P(seats), P(zf), P(z4), P(zf), P(z4), P(slot),
                           P(ppf), orc.PP_CAP, P(po), P(vo), P(ao), P(qo))
    # the pair set: every particle counts the same neighbours
    assert np.array_equal(got["aux"][:, 3], ao[:, 3])
    assert ao[:, 3].mean() > 5          # the contact loop found neighbours
    # ... and the same ones: every owner's neighbours and which of them touch, as sets
    oc, op = orc.contact_pairs(u, pos, seats, 64)
    assert np.array_equal(gc, oc) and gc.max() <= 64
    assert np.array_equal(np.sort(gp, axis=1), np.sort(op, axis=1))
    assert (op[op != 0xFFFFFFFF] >> 31).sum() > 0          # touching pairs among them
    assert np.array_equal(got["pos"][:, 3], po[:, 3])
    for name, a, b in (("pos", got["pos"][:, :3], po[:, :3]), ("vel", got["vel"][:, :3], vo[:, :3]),
                       ("T", got["vel"][:, 3], vo[:, 3]), ("q", got["q"], qo)):
        assert scaled_err(a, b) < TOL, name
    # the velocity change of the step is what the contacts did: compare that too
    dv1 = got["vel"][:, :3].astype(np.float64) - vel[:, :3]
    dv2 = vo[:, :3].astype(np.float64) - vel[:, :3]
    assert scaled_err(dv1, dv2) < 1e-4
    assert np.abs(qo).max() > 0 or settle


def test_contact_step_crowded_particle(nb, ccmod, orc):
    """A particle touching more neighbours than the kernel lists per owner (16): twenty on a sphere of 1.5
    radii around it, away from the bodies (those past a cell's eight seats unseated, as always).  The contacts past the list are worked out as they are found and
    added atomically; counts exact, state to tolerance, as for every other particle."""
    osim, pos, vel, mat, q = oracle_state(orc, settle_steps=4)
    vel = with_motion(pos, vel, scale=0.05)
    a = osim.a
    c = np.array([3.0, 3.0, 3.0])
    k = np.arange(20) + 0.5
    z = 1 - 2 * k / 20
    phi = np.pi * (3 - np.sqrt(5)) * k
    ring = np.stack([np.sqrt(1 - z * z) * np.cos(phi), np.sqrt(1 - z * z) * np.sin(phi), z], 1) * 1.5 * a
    pos = pos.copy()
    pos[0, :3] = c
    pos[1:21, :3] = c + ring            # the lowest indices, so every one of them holds a seat
    nb.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
    nb.write_state(q=q)
    nb.pass_slots()
    nb.pass_sim(0, 0, 0.0)
    got = nb.read_state()
    u = uni_for(orc, osim)
    u.settle, u.kick, u.gdt = 0.0, 0.0, 0.0
    for kk in range(3):
        u.bulk0[kk], u.bulk1[kk] = osim.bulk0[kk], osim.bulk1[kk]
        u.cen0[kk], u.cen1[kk] = osim.cen0[kk], osim.cen1[kk]
    seats = orc.slots(u, pos)
    N = osim.N
    zf = np.zeros(((orc.FINE + 1), 4), np.float32)
    z4 = np.zeros(4, np.float32)
    slot = np.full(N, -1, np.int32)
    ppf = np.zeros((4 * orc.PP_CAP, 4), np.float32)
    po, vo, ao, qo = (np.zeros((N, 4), np.float32), np.zeros((N, 4), np.float32), np.zeros((N, 4), np.float32),
                      np.zeros(N, np.float32))
    P = orc.ptr
    orc.lib().orc_sim_pass(C.byref(u), P(pos), P(vel), P(mat), P(q), P(seats), P(zf), P(z4), P(zf), P(z4), P(slot),
                           P(ppf), orc.PP_CAP, P(po), P(vo), P(ao), P(qo))
    assert ao[0, 3] > 16          # more touching neighbours than a list holds (a cell's ninth is unseated)
    assert np.array_equal(got["aux"][:, 3], ao[:, 3])
    for name, x, y in (("pos", got["pos"][:, :3], po[:, :3]), ("vel", got["vel"][:, :3], vo[:, :3]),
                       ("q", got["q"], qo)):
        assert scaled_err(x, y) < TOL, name
    dv1 = got["vel"][0, :3].astype(np.float64) - vel[0, :3]
    dv2 = vo[0, :3].astype(np.float64) - vel[0, :3]
    assert np.abs(dv1 - dv2).max() <= 1e-4 * np.abs(dv2).max()   # the crowded particle's own kick


def set_box(sim, cen, vel=(0.0, 0.0, 0.0), on_b=False, cen_b=(0.0, 0.0, 0.0)):
    sim.boxOn[0] = 1
    sim.boxOn[1] = 1 if on_b else 0
    for k in range(3):
        sim.boxCen[0][k] = cen[k]
        sim.boxVel[0][k] = vel[k]
        sim.boxCen[1][k] = cen_b[k]
    sim.boxT[0] = sim.t
    sim.boxT[1] = sim.t


def test_mesh_chain(nb, ccmod, orc):
    osim, pos, vel, mat, q = oracle_state(orc)
    com = (pos[:, :3].astype(np.float64) * mat[:, None]).sum(0) / mat.sum()
    set_box(osim, com)
    nb.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
    nb.pass_mesh()
    fine = nb.buffer("fineA")
    coarse = nb.buffer("coarseA")
    farA = nb.buffer("farA")
    force = nb.buffer("forceA")
    mono = nb.buffer("monoA")[0]
    u = uni_for(orc, osim)
    orc.lib().orc_boxes(C.byref(osim), C.byref(u))
    P = orc.ptr
    # the deposit: to tolerance (summation order is unspecified)
    ofine = np.zeros((orc.FINE + 1, 4), np.float32)
    z4 = np.zeros(4, np.float32)
    orc.lib().orc_deposit(C.byref(u), 0, P(pos), P(mat), P(z4), P(ofine))
    m = ofine[:, 3]
    assert (m > 0).sum() > 500
    assert scaled_err(fine[:, 3], m) < TOL
    for k in range(3):
        assert scaled_err(fine[:, k], ofine[:, k]) < TOL
    # given the same fine mesh the coarse sums are exact, far and cell gravity to tolerance
    oc = np.zeros((orc.COARSE, 4), np.float32)
    om = np.zeros(4, np.float32)
    orc.lib().orc_coarse(P(fine), P(oc), P(om))
    assert np.array_equal(coarse.view(np.uint32), oc.view(np.uint32))
    assert scaled_err(mono, om) < 1e-6
    fa, t0, t1 = (np.zeros((orc.COARSE, 4), np.float32) for _ in range(3))
    orc.lib().orc_far(P(oc), P(fa), P(t0), P(t1))
    assert np.array_equal(farA == 0, fa == 0)          # the same blocks are occupied
    for k in range(4):
        assert scaled_err(farA[:, k], fa[:, k]) < TOL
    of = np.zeros((orc.FINE + 1, 4), np.float32)
    orc.lib().orc_cell(C.byref(u), P(fine), P(oc), P(fa), P(t0), P(t1), P(of))
    assert np.array_equal(force[:, 3] == 0, of[:, 3] == 0)
    for k in range(4):
        assert scaled_err(force[:, k], of[:, k]) < TOL
    # per occupied cell too: the pull each cell feels, relative to its own size
    occ = of[:-1, 3] != 0
    g1, g2 = force[:-1][occ, :3].astype(np.float64), of[:-1][occ, :3].astype(np.float64)
    rel = np.linalg.norm(g1 - g2, axis=1) / np.linalg.norm(g2, axis=1)
    assert np.median(rel) < 1e-5 and np.percentile(rel, 99) < 1e-4


def test_pp(nb, ccmod, orc):
    osim, pos, vel, mat, q = oracle_state(orc)
    rng = np.random.default_rng(8)
    # spread a third of the body out as loose material so pairs fall inside and beyond the cut
    pos = pos.copy()
    sel = rng.choice(osim.N, 5000, replace=False)
    pos[sel, :3] *= np.float32(2.5)
    com = (pos[:, :3].astype(np.float64) * mat[:, None]).sum(0) / mat.sum()
    set_box(osim, com, on_b=True, cen_b=com + np.array([4.0, 0.0, 0.0]))
    nb.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
    nb.pass_mesh()                                  # sets the box uniforms (boxes())
    lst = np.sort(sel).astype(np.int32)
    nb.set_pp(lst)
    u = uni_for(orc, osim)
    orc.lib().orc_boxes(C.byref(osim), C.byref(u))
    index = np.full(orc.PP_CAP, -1, np.int32)
    index[:len(lst)] = lst
    ol = np.zeros((orc.PP_CAP, 4), np.float32)
    ob = np.zeros(orc.PP_CAP, np.float32)
    P = orc.ptr
    orc.lib().orc_pp_gather(C.byref(u), P(pos), P(mat), P(index), orc.PP_CAP, P(ol), P(ob))
    f, p = orc.pair_table()
    tab = np.stack([f, p], 1).astype(np.float32).copy()
    of = np.zeros((4 * orc.PP_CAP, 4), np.float32)
    orc.lib().orc_pp_force(C.byref(u), P(ol), P(ob), len(lst), orc.PP_CAP, P(tab), P(of))
    assert np.array_equal(nb.buffer("pplist").view(np.uint32), ol.view(np.uint32))
    assert np.array_equal(nb.buffer("ppbox"), ob)
    assert set(np.unique(ob[:len(lst)])) >= {0.0}
    got = nb.buffer("ppforce")
    for k in range(4):
        assert scaled_err(got[:, k], of[:, k]) < TOL
    assert np.abs(of[:, :3]).max() > 0
    # each member's correction summed over the four slices, relative to its own size
    s1 = got.reshape(4, orc.PP_CAP, 4).sum(0)[:len(lst), :3].astype(np.float64)
    s2 = of.reshape(4, orc.PP_CAP, 4).sum(0)[:len(lst), :3].astype(np.float64)
    big = np.linalg.norm(s2, axis=1) > 1e-3 * np.linalg.norm(s2, axis=1).max()
    rel = np.linalg.norm(s1 - s2, axis=1)[big] / np.linalg.norm(s2, axis=1)[big]
    assert np.median(rel) < 1e-5
    slot = nb.buffer("ppslot")
    want = np.full(osim.N, -1, np.int32)
    want[lst] = np.arange(len(lst))
    assert np.array_equal(slot, want)


def test_pp_list_beyond_the_cap_matches_the_oracle(nb, ccmod, orc):
    """The reference's pairwise correction over a list longer than its 8,192 cap (ccs_pp_list_force, the
    uncapped form the gravity sweep reports): 12,000 members, against the oracle's PPFORCE_FS restatement
    run with the cap lifted (orc_pp_force with cap = the list's length), each member's four slices summed;
    and over a list inside the cap, against the capped pass of the step itself."""
    osim, pos, vel, mat, q = oracle_state(orc)
    rng = np.random.default_rng(9)
    pos = pos.copy()
    n = 12000
    assert n > orc.PP_CAP and n < osim.N
    sel = rng.choice(osim.N, n, replace=False)
    pos[sel, :3] *= np.float32(2.0)
    com = (pos[:, :3].astype(np.float64) * mat[:, None]).sum(0) / mat.sum()
    set_box(osim, com, on_b=True, cen_b=com + np.array([4.0, 0.0, 0.0]))
    nb.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
    nb.pass_mesh()                                  # sets the box uniforms (boxes())
    lst = np.sort(sel).astype(np.int32)
    got = nb.pp_list_force(lst).astype(np.float64)
    u = uni_for(orc, osim)
    orc.lib().orc_boxes(C.byref(osim), C.byref(u))
    P = orc.ptr
    ol = np.zeros((n, 4), np.float32)
    ob = np.zeros(n, np.float32)
    orc.lib().orc_pp_gather(C.byref(u), P(pos), P(mat), P(lst), n, P(ol), P(ob))
    f, p = orc.pair_table()
    tab = np.stack([f, p], 1).astype(np.float32).copy()
    of = np.zeros((4 * n, 4), np.float32)
    orc.lib().orc_pp_force(C.byref(u), P(ol), P(ob), n, n, P(tab), P(of))
    want = of.reshape(4, n, 4).astype(np.float64).sum(0)   # x Gm already
    assert np.abs(want[:, :3]).max() > 0
    assert scaled_err(got, want) < TOL
    big = np.linalg.norm(want[:, :3], axis=1) > 1e-3 * np.linalg.norm(want[:, :3], axis=1).max()
    rel = np.linalg.norm(got[:, :3] - want[:, :3], axis=1)[big] / np.linalg.norm(want[:, :3], axis=1)[big]
    print("uncapped list of %d: per-member median rel %.2e, p99.9 %.2e" % (n, np.median(rel),
                                                                           np.percentile(rel, 99.9)))
    assert np.median(rel) < 1e-5 and np.percentile(rel, 99.9) < 1e-4
    # inside the cap: the same members as the step's own (capped, four-slice) pass
    short = lst[:5000]
    nb.set_pp(short)
    slices = nb.buffer("ppforce").reshape(4, ccmod._lib.PP_CAP, 4)[:, :len(short)].astype(np.float64).sum(0)
    assert scaled_err(nb.pp_list_force(short).astype(np.float64), slices) < TOL


def test_rigid_carry_is_exact(nb, ccmod, orc):
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(16384))
    sim.phase = 1
    nb.upload(to_lib_sim(ccmod, sim), pos, vel, mat, home)
    e = orc.Engine(sim, pos, vel, mat)
    for _ in range(3):
        nb.rigid_step(0.01)
        e.rigid_step(0.01)
    got = nb.read_state()
    assert np.array_equal(got["pos"].view(np.uint32), e.buf("pos").view(np.uint32))
    assert np.array_equal(got["vel"].view(np.uint32), e.buf("vel").view(np.uint32))
    s1, s2 = nb.sim, e.sim
    assert s1.t == s2.t and list(s1.relr) == list(s2.relr) and list(s1.bulk0) == list(s2.bulk0)


def test_permutation_and_morton_order(nb, ccmod, orc):
    osim, pos, vel, mat, q = oracle_state(orc, settle_steps=4)
    nb.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
    core = np.array([0.05, -0.02, 0.01])
    perm, into = nb.sort_morton(core)
    keys, operm, ointo = orc.morton(pos, core)
    assert np.array_equal(perm, operm)
    assert np.array_equal(into, ointo)
    st = nb.read_state()
    assert np.array_equal(st["pos"], pos[operm])
    assert np.array_equal(st["mat"], mat[operm])
    # a host-given permutation (applyPerm) gathers the same way and rebuilds the cells
    rng = np.random.default_rng(0)
    p2 = rng.permutation(osim.N).astype(np.int32)
    nb.apply_perm(p2)
    st2 = nb.read_state()
    assert np.array_equal(st2["pos"], st["pos"][p2])
    assert np.array_equal(nb.buffer("seats"), orc.slots(uni_for(orc, osim), st2["pos"]))


def test_full_steps_to_tolerance(nb, ccmod, orc):
    """The whole schedule (src/nbody.js:551-558): 16 steps from the same state, gravity on."""
    osim, pos, vel, mat, q = oracle_state(orc, settle_steps=8)
    com = (pos[:, :3].astype(np.float64) * mat[:, None]).sum(0) / mat.sum()
    set_box(osim, com)
    osim.phase = 2
    osim.impactT = osim.t
    osim.stepNo = 0
    vel = with_motion(pos, vel, scale=0.05)
    nb.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
    e = orc.Engine(osim, pos, vel, mat)
    for k in range(9):
        nb.step(False, False)
        e.step(False, False)
        if k == 0:
            # one step (grid + mesh + contacts + kick/drift): state and forces to 1e-5 of scale
            got = nb.read_state()
            for name, a, b in (("pos", got["pos"][:, :3], e.buf("pos")[:, :3]),
                               ("vel", got["vel"][:, :3], e.buf("vel")[:, :3]),
                               ("grav", got["aux"][:, :3], e.buf("aux")[:, :3]), ("q", got["q"], e.buf("q"))):
                assert scaled_err(a, b) < TOL, name
            assert np.array_equal(got["aux"][:, 3], e.buf("aux")[:, 3])
            g1 = got["aux"][:, :3].astype(np.float64)
            g2 = e.buf("aux")[:, :3].astype(np.float64)
            rel = np.linalg.norm(g1 - g2, axis=1) / np.linalg.norm(g2, axis=1)
            assert np.median(rel) < 1e-5
    # nine steps, two of them mesh steps: the trajectories stay together
    got = nb.read_state()
    for name, a, b in (("pos", got["pos"][:, :3], e.buf("pos")[:, :3]), ("vel", got["vel"][:, :3], e.buf("vel")[:, :3])):
        err = scaled_err(a, b)
        assert err < 1e-4, (name, err)
    assert np.array_equal(nb.buffer("seats") & 0x3FFFF, e.buf("seats") & 0x3FFFF)


def test_diag_and_books(nb, ccmod, orc):
    osim, pos, vel, mat, q = oracle_state(orc, settle_steps=8)
    com = (pos[:, :3].astype(np.float64) * mat[:, None]).sum(0) / mat.sum()
    set_box(osim, com)
    vel = with_motion(pos, vel, scale=0.05)
    nb.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
    e = orc.Engine(osim, pos, vel, mat)
    nb.pass_diag()
    d1 = nb.buffer("diag")
    d2 = e.diag()
    assert np.array_equal(d1[:, 1:], d2[:, 1:])       # seated, taken, Q: exact
    assert scaled_err(d1[:, 0], d2[:, 0]) < TOL       # potential: through the deposit
    b = nb.books(with_diag=False)
    m = osim.m * mat.astype(np.float64)
    v = vel[:, :3].astype(np.float64)
    p = pos[:, :3].astype(np.float64)
    assert abs(b["M"] - m.sum()) < 1e-12
    assert np.allclose([b["px"], b["py"], b["pz"]], (m[:, None] * v).sum(0), rtol=1e-12, atol=1e-15)
    assert np.allclose([b["Lx"], b["Ly"], b["Lz"]], (m[:, None] * np.cross(p, v)).sum(0), rtol=1e-12, atol=1e-15)
    assert abs(b["KE"] - 0.5 * (m * (v * v).sum(1)).sum()) < 1e-12 * max(1, b["KE"])


def test_async_readback(nb, ccmod, orc):
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(16384))
    nb.upload(to_lib_sim(ccmod, sim), pos, vel, mat, home)
    lib = ccmod.lib()
    N = sim.N
    P = np.zeros((N, 4), np.float32)
    assert lib.ccs_poll(nb.handle, None, None, None) == -3            # nothing pending
    assert lib.ccs_diag_async(nb.handle) == 0
    rc = lib.ccs_poll(nb.handle, P.ctypes.data_as(C.c_void_p), None, None)
    while rc == 1:                                                      # CCS_NOT_READY until the copy lands
        rc = lib.ccs_poll(nb.handle, P.ctypes.data_as(C.c_void_p), None, None)
    assert rc == 0
    assert np.array_equal(P, pos)


def test_graph_blocks_match_direct_steps(ccmod, orc):
    """ccs_steps replays captured 8-step graphs; the same steps launched one by one agree to tolerance."""
    osim, pos, vel, mat, q = oracle_state(orc, settle_steps=8)
    com = (pos[:, :3].astype(np.float64) * mat[:, None]).sum(0) / mat.sum()
    set_box(osim, com)
    osim.phase, osim.stepNo, osim.impactT = 2, 0, osim.t
    a, b = ccmod.NBody(0), ccmod.NBody(0)
    try:
        for n in (a, b):
            n.upload(to_lib_sim(ccmod, osim), pos, vel, mat)
        a.steps(24)
        for _ in range(24):
            b.step(False, False)
            b.sim.t += b.sim.dt
        sa, sb = a.read_state(), b.read_state()
        assert a.sim.t == b.sim.t and a.sim.stepNo == b.sim.stepNo == 24
        # 24 steps, 3 of them mesh steps whose deposits sum in different orders
        assert scaled_err(sa["pos"][:, :3], sb["pos"][:, :3]) < 1e-4
        assert scaled_err(sa["vel"][:, :3], sb["vel"][:, :3]) < 1e-4
        assert np.array_equal(a.buffer("seats") & 0x3FFFF, b.buffer("seats") & 0x3FFFF)
    finally:
        a.close()
        b.close()


def test_errors_are_loud(nb, ccmod, orc):
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(16384))
    nb.upload(to_lib_sim(ccmod, sim), pos, vel, mat, home)
    with pytest.raises(ccmod.CCSError):
        nb.set_pp(np.array([sim.N + 5], np.int32))
    with pytest.raises(ccmod.CCSError):
        nb.apply_perm(np.zeros(sim.N, np.int32))           # not a permutation
    bad = to_lib_sim(ccmod, sim)
    bad.N = 262145
    with pytest.raises(ccmod.CCSError):
        nb.upload(bad, np.zeros((262145, 4), np.float32), np.zeros((262145, 4), np.float32),
                  np.ones(262145, np.float32))
