"""Pins the CPU oracle against what the reference states about itself.

The reference ships no tests and no golden vectors, and its step (WebGL2 GLSL)
and host code (JavaScript) cannot run on these machines, so the oracle's
parity with the reference is pinned by the known answers its sources state in
their own text, and by the invariants its console checks assert.  Each test
names the line it takes its number from.
"""
import math

import numpy as np
import pytest

FH = 12.0 / 64


def test_mulberry_is_deterministic_uniform(orc):
    # src/math.js:8-15: mulberry32, [0, 1), seeded
    a = orc.mulberry_seq(1234567, 20000)
    b = orc.mulberry_seq(1234567, 20000)
    assert np.array_equal(a, b)
    assert a.min() >= 0.0 and a.max() < 1.0
    assert abs(a.mean() - 0.5) < 0.01
    assert not np.array_equal(a[:100], orc.mulberry_seq(99, 100))


def test_maclaurin_peak(orc):
    # src/bodies.js:150-151: "The right side peaks at 0.449 (e ~ 0.93)"
    es = np.linspace(0.5, 0.99, 2000)
    g = np.array([orc.maclaurin_g(e) for e in es])
    assert abs(g.max() - 0.449) < 6e-4
    assert abs(es[g.argmax()] - 0.93) < 0.01


@pytest.mark.parametrize("f", [0.05, 0.18, 0.2, 0.3, 0.45, 0.55])
def test_maclaurin_solves_its_equation(orc, f):
    # src/bodies.js:148-151: e solves (4/3) f^2 = g(e); f <= 0.55 stays on the sequence
    e = orc.maclaurin(f)
    assert 0 < e <= 0.93
    assert abs(orc.maclaurin_g(e) - 4.0 / 3.0 * f * f) < 1e-9


def test_spin_days():
    # index.html:183-185: 0.18 of breakup is a young planet's ~8-hour day; 0.55 is the 2.6-hour Earth
    day = lambda f: 2 * math.pi / f * 805 / 3600
    assert 7.5 < day(0.18) < 8.5
    assert abs(day(0.55) - 2.6) < 0.1


def test_units_and_escape():
    # src/nbody.js:7-10: time unit sqrt(R^3/GM) = 805 s, velocity 7.91 km/s, escape speed off Earth sqrt 2
    G, M, R = 6.674e-11, 5.972e24, 6.371e6
    assert abs(math.sqrt(R ** 3 / (G * M)) - 805) < 3
    assert abs(math.sqrt(G * M / R) / 1000 - 7.91) < 0.02
    assert abs(math.sqrt(2 * 1 / 1) - math.sqrt(2)) < 1e-15


def test_wrap_length_at_131k(orc):
    # src/glsl-sim.js:69: "The wrap is 5.9 R_earth at 131k"
    sim = orc.build_run(orc.make_opt(131072))[0]
    assert sim.G == 128
    assert abs(sim.cell * sim.G - 5.9) < 0.05


def test_near_block_width():
    # src/glsl-sim.js:297: the 5^3 coarse neighbourhood "is 3.75 R_earth wide"
    assert 5 * 4 * FH == 3.75


@pytest.mark.parametrize("N,a,dt", [(16384, 0.0357, 2.55e-3), (262144, 0.01415, 1.01e-3)])
def test_build_scales(orc, N, a, dt):
    # src/nbody.js:125-128, 202-204 at the page's defaults (index.html:177)
    sim = orc.build_run(orc.make_opt(N))[0]
    assert abs(sim.a - a) / a < 2e-3
    assert abs(sim.dt - dt) / dt < 5e-3
    # src/nbody.js:531: "a particle moves under 0.2 radii a step" at the reference speed
    assert max(1.5, sim.vc) * sim.dt / sim.a < 0.2
    assert sim.N == sim.n1 + sim.n2
    assert sim.G == (128 if N >= 65536 else 64)


def test_build_masses(orc):
    # src/nbody.js:161-167: Earth weighs 1; the impactor follows from its density and count
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(16384))
    m = sim.m * mat.astype(np.float64)
    assert abs(m[:sim.n1].sum() - 1.0) < 1e-6
    assert abs(m.sum() - sim.M) < 1e-6
    layers = pos[:, 3]
    assert set(np.unique(layers[:sim.n1])) <= {0.0, 1.0, 2.0}
    assert set(np.unique(layers[sim.n1:])) <= {4.0, 5.0, 6.0}
    assert np.all(vel == 0)
    # the iron is 2.5 times the mantle's density (src/nbody.js:118)
    assert np.allclose(mat[:sim.n1][layers[:sim.n1] == 0], 2.5)


def test_pair_table_limits(orc):
    # src/nbody.js:53-55: force x r^2 and potential x r "go to 1 and -1 where the mesh is Newton's"
    f, p = orc.pair_table()
    assert abs(f[-1] - 1.0) < 0.05 and abs(p[-1] + 1.0) < 0.02
    assert f[0] < 0.01                      # a pair in one cell: the mesh gives it ~nothing
    assert np.all(np.diff(f[:16]) > 0)      # the mesh's share grows with distance ...
    assert f[8] < f[24] < f[40] < f[63]     # ... up to the sampling noise of 80 placings a bin


def test_seat_word_is_a_normal_float():
    # src/glsl-sim.js:96-102: index in 18 bits, place in 12, bit 30 set -> a normal float; -1 is empty
    idx = np.array([0, 1, 262143], np.uint32)
    for q in range(15):
        w = idx | np.uint32(q << 18) | np.uint32(q << 22) | np.uint32(q << 26) | np.uint32(0x40000000)
        f = w.view(np.float32)
        assert np.all(np.isfinite(f)) and np.all(np.abs(f) >= np.finfo(np.float32).tiny)
        assert np.all((w & 0x80000000) == 0)
    assert np.array([-1.0], np.float32).view(np.uint32)[0] == 0xBF800000


def test_hash_is_a_bijection_within_a_period(orc):
    # src/glsl-sim.js:84-90: inside one period the hash is the identity layout of the atlas
    sim = orc.build_run(orc.make_opt(16384))[0]
    u = orc.make_uni(sim)
    import ctypes as C
    seen = set()
    ax, ay = C.c_int(), C.c_int()
    G = u.G
    for z in range(0, G, 3):
        for y in range(0, G, 5):
            for x in range(G):
                orc.lib().orc_hash(C.byref(u), x, y, z, C.byref(ax), C.byref(ay))
                seen.add((ax.value, ay.value))
    n = len(range(0, G, 3)) * len(range(0, G, 5)) * G
    assert len(seen) == n
    # the next period in x lands half a period up in y (src/glsl-sim.js:73-74)
    orc.lib().orc_hash(C.byref(u), G + 3, 7, 9, C.byref(ax), C.byref(ay))
    a2, b2 = C.c_int(), C.c_int()
    orc.lib().orc_hash(C.byref(u), 3, 7 + G // 2, 9, C.byref(a2), C.byref(b2))
    assert (ax.value, ay.value) == (a2.value, b2.value)
    # a quarter for the period in z
    orc.lib().orc_hash(C.byref(u), 3, 7, 9 + G, C.byref(ax), C.byref(ay))
    orc.lib().orc_hash(C.byref(u), 3, 7 + G // 4, 9, C.byref(a2), C.byref(b2))
    assert (ax.value, ay.value) == (a2.value, b2.value)


def test_seats_are_the_eight_lowest(orc):
    # src/glsl-sim.js:112-117 + src/nbody.js:379-399: the depth peel seats the lowest index above the last
    rng = np.random.default_rng(5)
    sim = orc.build_run(orc.make_opt(16384))[0]
    u = orc.make_uni(sim)
    N = 16384
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.normal(scale=0.12, size=(N, 3))   # dense: many cells overfill
    u.N = N
    seats = orc.slots(u, pos)
    cells, _ = orc.cell_ids(u, pos)
    order = np.argsort(cells, kind="stable")
    cs = cells[order]
    starts = np.flatnonzero(np.r_[True, cs[1:] != cs[:-1]])
    ends = np.r_[starts[1:], len(cs)]
    overfull = 0
    for s, e in zip(starts, ends):
        members = order[s:e]                       # ascending index within a cell (stable sort)
        got = seats[cs[s]]
        want = members[:8]
        assert np.array_equal(got[:len(want)] & 0x3FFFF, want)
        assert np.all(got[len(want):] == orc.EMPTY)
        overfull += e - s > 8
    assert overfull > 0
    assert (seats[:, 0] != orc.EMPTY).sum() == len(starts)


def test_mesh_net_force_vanishes(orc):
    # index.html:531-556 (meshCheck): the mesh's cells exert no net force on each other
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(16384))
    e = orc.Engine(sim, pos, vel, mat)
    e.step(True, False)             # step 0: boxes + mesh
    fine = e.buf("fineA")[:-1]
    force = e.buf("forceA")[:-1]
    m = fine[:, 3].astype(np.float64)
    occ = m > 0
    F = force[occ, :3].astype(np.float64) * (m[occ] * sim.m)[:, None]
    net = np.linalg.norm(F.sum(0))
    assert net / np.linalg.norm(F, axis=1).sum() < 1e-4


def test_morton_order(orc):
    # src/nbody.js:871-887: 7 bits an axis about the core, x -> bit 3k, stable counting sort
    rng = np.random.default_rng(2)
    N = 5000
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.uniform(-7, 7, size=(N, 3))
    core = np.array([0.3, -0.2, 0.1])
    keys, perm, into = orc.morton(pos, core)
    m = np.clip(np.floor((pos[:, :3].astype(np.float64) - core + 6) / 12 * 128), 0, 127).astype(np.int64)
    want = np.zeros(N, np.int64)
    for k in range(7):
        for ax in range(3):
            want |= ((m[:, ax] >> k) & 1) << (3 * k + ax)
    assert np.array_equal(keys, want)
    assert np.array_equal(perm, np.lexsort((np.arange(N), keys)))
    assert np.array_equal(into[perm], np.arange(N))


def test_contact_pair_sets_match_the_step_counts(orc):
    """The oracle's pair read-out walks simFS's loop as its step does: every owner's pair count is the
    step's neighbour count, the touching pairs lie inside the contact distance, and no particle pairs with
    itself."""
    import ctypes as C
    N = 16384
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(N))
    u = orc.make_uni(sim)
    seats = orc.slots(u, pos)
    counts, pairs = orc.contact_pairs(u, pos, seats, 64)
    zf = np.zeros(((orc.FINE + 1), 4), np.float32)
    z4 = np.zeros(4, np.float32)
    slot = np.full(N, -1, np.int32)
    ppf = np.zeros((4 * orc.PP_CAP, 4), np.float32)
    q = np.zeros(N, np.float32)
    po, vo, ao, qo = (np.zeros((N, 4), np.float32), np.zeros((N, 4), np.float32), np.zeros((N, 4), np.float32),
                      np.zeros(N, np.float32))
    P = orc.ptr
    orc.lib().orc_sim_pass(C.byref(u), P(pos), P(vel), P(mat), P(q), P(seats), P(zf), P(z4), P(zf), P(z4), P(slot),
                           P(ppf), orc.PP_CAP, P(po), P(vo), P(ao), P(qo))
    assert np.array_equal(counts, ao[:, 3].astype(np.int32))
    assert counts.max() <= 64 and counts.mean() > 5
    own = np.repeat(np.arange(N), 64).reshape(N, 64)
    live = pairs != 0xFFFFFFFF
    j = (pairs & 0x3FFFF).astype(np.int64)
    assert not np.any(live & (j == own))
    d = np.linalg.norm(pos[j[live], :3].astype(np.float64) - pos[own[live], :3], axis=1)
    touch = (pairs[live] >> 31) == 1
    assert touch.any() and np.all(d[touch] < 2 * sim.a * (1 + 1e-6)) and np.all(d[~touch] >= 2 * sim.a * (1 - 1e-6))
