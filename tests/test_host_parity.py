"""The library's host-side code against the oracle, bit for bit: the body
builder (src/nbody.js:114-250, src/bodies.js), the mesh pair table
(src/nbody.js:56-108) and the analysis fof (src/nbody.js:646-893)."""
import numpy as np
import pytest

SIM_FIELDS = ["N", "W", "H", "n1", "n2", "G", "settleLeft", "settleTotal", "stepNo", "soft", "phase", "m", "a",
              "cell", "dt", "k", "c", "creep", "damp", "tK", "kappa", "R1", "R2", "Re1", "Re2", "M1", "M2", "M",
              "vc", "vesc", "t", "impactT"]
VEC_FIELDS = ["spin0", "spin1", "cen0", "cen1", "bulk0", "bulk1", "relr", "relv"]

CASES = {
    "page-default-16k": dict(N=16384),
    "page-default-65k": dict(N=65536),
    # the small giant impact of the plain-method configuration: 0.9 + 0.1 M_earth, 1,638 impactor particles,
    # 7.8 / 3.3 g/cc, 45 degrees at 1.0 v_esc
    "small-impact-16k": dict(N=16384, q=0.1, dens=1.0, core=0.32, spin0=0.18, spin1=0.2, angle=45, incl=0,
                             vfac=1.0, rest=0.3, n2=1638, mImp=0.1, mTarget=0.9, rhoR=7.8 / 3.3),
    # the full impact's layering: crust of 2.7 g/cc on the outer 5 % of radius
    "crust-impact-32k": dict(N=32768, q=0.1, dens=1.0, core=0.3, angle=45, incl=0, vfac=1.0, mImp=0.1,
                             mTarget=0.9, rhoR=7.8 / 3.3, rhoCrust=2.7 / 3.3, crustFrac=0.05),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_builder_matches_oracle(ccmod, orc, case):
    kw = CASES[case]
    s1, p1, v1, m1, h1 = ccmod.make_bodies(ccmod.make_opt(**kw))
    s2, p2, v2, m2, h2 = orc.build_run(orc.make_opt(**kw))
    for a, b in ((p1, p2), (v1, v2), (m1, m2), (h1, h2)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    for f in SIM_FIELDS:
        assert getattr(s1, f) == getattr(s2, f), f
    for f in VEC_FIELDS:
        assert list(getattr(s1, f)) == list(getattr(s2, f)), f


def test_builder_configuration_masses(ccmod):
    s, p, v, m, h = ccmod.make_bodies(ccmod.make_opt(**CASES["small-impact-16k"]))
    assert (s.n1, s.n2) == (16384 - 1638, 1638)
    w = s.m * m.astype(np.float64)
    assert abs(w[:s.n1].sum() - 0.9) < 1e-6 and abs(w[s.n1:].sum() - 0.1) < 1e-6
    s, p, v, m, h = ccmod.make_bodies(ccmod.make_opt(**CASES["crust-impact-32k"]))
    lay = p[:s.n1, 3]
    assert np.allclose(m[:s.n1][lay == 2], 2.7 / 3.3)
    # the crust is the outer 5 % of radius: about 1 - 0.95^3 of the target's particles
    assert abs((lay == 2).mean() - (1 - 0.95 ** 3)) < 0.03


def test_pair_table_matches_oracle(ccmod, orc):
    f1, p1 = ccmod.pair_table()
    f2, p2 = orc.pair_table()
    assert np.array_equal(f1, f2) and np.array_equal(p1, p2)


def _evolved(orc, N=16384, steps=40):
    sim, pos, vel, mat, home = orc.build_run(orc.make_opt(N))
    e = orc.Engine(sim, pos, vel, mat)
    for _ in range(steps):
        e.step(True, False)
    return e


REPORT_FIELDS = ["largest", "largestImp", "largestIron", "day", "tilt", "orbit", "escape", "hasSecond", "secMass",
                 "secDist", "secImp", "secIron", "secR", "secBound", "R", "Redge", "Tsurf", "hotR", "impMass",
                 "impRms", "M", "iron", "drift", "L", "KE", "PE", "EL", "Q", "unseated", "full", "jD", "moon",
                 "ppCount", "ppLoose"]


@pytest.mark.parametrize("sort", [False, True])
def test_fof_matches_oracle(ccmod, orc, sort):
    e = _evolved(orc)
    s = e.sim
    D = e.diag()
    P, V, R = e.buf("pos"), e.buf("vel"), e.buf("mat")
    r1, l1, q1 = ccmod.fof(s.N, s.m, s.a, P, V, R, D, s.k, 2 * s.a, 8192, sort)
    r2, l2, q2 = orc.fof(s.N, s.m, s.a, P, V, R, D, s.k, 2 * s.a, 8192, sort)
    for f in REPORT_FIELDS:
        assert getattr(r1, f) == getattr(r2, f), f
    for f in ("axis", "bodyVel", "com", "core", "vel", "hotCom", "impCom", "secCom", "secCore", "secVel"):
        assert list(getattr(r1, f)) == list(getattr(r2, f)), f
    assert np.array_equal(l1, l2)
    if sort:
        assert np.array_equal(q1, q2)
        assert np.array_equal(np.sort(q1), np.arange(s.N))


def test_fof_loose_list_cap(ccmod, orc):
    # more loose material than the pass can take: the farthest first, in index order (src/nbody.js:863-870)
    rng = np.random.default_rng(11)
    N = 20000
    P = np.zeros((N, 4), np.float32)
    P[:12000, :3] = rng.normal(scale=0.3, size=(12000, 3))
    P[12000:, :3] = rng.uniform(-5, 5, size=(8000, 3))
    P[:, 3] = 1
    V = np.zeros((N, 4), np.float32)
    R = np.ones(N, np.float32)
    D = np.zeros((N, 4), np.float32)
    D[:, 1] = 1
    r1, l1, _ = ccmod.fof(N, 1.0 / N, 0.01, P, V, R, D, 1.0, 0.02, cap=3000)
    r2, l2, _ = orc.fof(N, 1.0 / N, 0.01, P, V, R, D, 1.0, 0.02, cap=3000)
    assert r1.ppLoose > 3000 and r1.ppCount == 3000
    assert np.array_equal(l1, l2)
    assert np.all(np.diff(l1) > 0)
