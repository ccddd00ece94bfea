"""The analysis on the device (ccs_fof_device) against the host fof (ccs_fof) on the same state.

The worker's fof (src/nbody.js:646-893) restated twice: ccs_fof on the host
(itself checked against the oracle in test_host_parity.py) and ccs_fof_device
on the state where it lies.  The device analysis runs the diag pass itself;
the host one is then given that same diag buffer and the read-back state, so
both see identical inputs.  Integer work -- the loose list, its length, the
second-body flags, the Morton permutation -- must be equal.  The report's
sums are binary64 added in another order: 1e-9 relative, with an absolute
floor of 1e-12 for the fields that are a small difference of large terms.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["largest", "largestImp", "largestIron", "day", "tilt", "axis", "bodyVel", "orbit", "escape",
          "secMass", "secDist", "secImp", "secIron", "secCom", "secCore", "secVel", "secR",
          "com", "core", "vel", "R", "Redge", "Tsurf", "hotCom", "hotR", "impMass", "impCom", "impRms",
          "M", "iron", "drift", "L", "KE", "PE", "EL", "Q", "unseated", "full", "jD", "moon"]


def both(cc, nb, sort, cap):
    t0 = time.perf_counter()
    dev = nb.fof_device(sort, cap)
    t1 = time.perf_counter()
    D = nb.buffer("diag").reshape(-1, 4)[:nb.sim.N]   # the read-outs the device analysis used
    st = nb.read_state()
    s = nb.sim
    t2 = time.perf_counter()
    host = cc.fof(s.N, s.m, s.a, st["pos"], st["vel"], st["mat"], D, s.k, 2 * s.a, cap, sort)
    t3 = time.perf_counter()
    print(f"N={s.N} sort={sort} cap={cap}: device {1e3 * (t1 - t0):.1f} ms, host {1e3 * (t3 - t2):.1f} ms, "
          f"loose {host[0].ppLoose}")
    return dev, host


def compare(dev, host):
    rd, ld, qd = dev
    rh, lh, qh = host
    assert (rd.ppLoose, rd.ppCount) == (rh.ppLoose, rh.ppCount)
    assert np.array_equal(ld, lh)
    if qh is not None:
        assert np.array_equal(qd, qh)
    assert (rd.hasSecond, rd.secBound) == (rh.hasSecond, rh.secBound)
    for f in FIELDS:
        a = np.atleast_1d(np.array(getattr(rd, f), np.float64))
        b = np.atleast_1d(np.array(getattr(rh, f), np.float64))
        same_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
        with np.errstate(invalid="ignore"):
            ok = same_inf | (np.abs(a - b) <= 1e-9 * np.abs(b) + 1e-12)
        assert ok.all(), (f, a, b)


@pytest.fixture(scope="module")
def impact(ccmod):
    from cosmic_collisions_b200 import configs
    nb = ccmod.NBody(0)
    nb.build(configs.small_impact_opt(16384))
    yield nb
    nb.close()


def test_two_bodies_before_contact(ccmod, impact):
    """Right after the build: planet and impactor apart, so the second body is reported."""
    dev, host = both(ccmod, impact, True, ccmod.NBody.PP_CAP)
    assert host[0].hasSecond == 1
    compare(dev, host)


@pytest.mark.parametrize("sort,cap", [(False, None), (True, None), (True, 64)])
def test_after_the_impact(ccmod, impact, sort, cap):
    """After first touch and the full phase: debris, a disk and a loose list (capped, too: the farthest first)."""
    if impact.sim.t < 2.0:
        impact.run_to(2.0)
    cap = ccmod.NBody.PP_CAP if cap is None else cap
    dev, host = both(ccmod, impact, sort, cap)
    if cap == 64:
        assert host[0].ppLoose > cap
    compare(dev, host)


def test_gravity_sweep_many_loose(ccmod):
    """The Plummer sphere in a uniform 10 % background: more loose particles than the pairwise pass takes."""
    from cosmic_collisions_b200 import configs
    sim, pos, vel, mat = configs.gravity_sweep(N=131072)
    nb = ccmod.NBody(0)
    try:
        nb.upload(sim, pos, vel, mat)
        nb.pass_slots()
        dev, host = both(ccmod, nb, True, ccmod.NBody.PP_CAP)
    finally:
        nb.close()
    assert host[0].ppLoose > ccmod.NBody.PP_CAP
    compare(dev, host)


def test_device_analysis_in_the_run(ccmod):
    """runTo with the analysis on the device keeps the books as the host analysis does."""
    from cosmic_collisions_b200 import configs
    out = []
    for device_fof in (False, True):
        nb = ccmod.NBody(0)
        try:
            nb.device_fof = device_fof
            nb.build(configs.small_impact_opt(16384))
            nb.run_to(2.0)
            r = nb.report
            out.append((nb.sim.stepNo, r.largest, r.L, r.KE + r.PE + r.EL + r.Q, r.KE - r.PE))
        finally:
            nb.close()
    (s0, m0, L0, e0, k0), (s1, m1, L1, e1, k1) = out
    assert s0 == s1
    assert abs(m1 - m0) <= 0.02 * m0
    assert abs(L1 - L0) <= 0.01 * L0
    assert abs(e1 - e0) <= 0.01 * k0
