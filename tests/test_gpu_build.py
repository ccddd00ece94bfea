"""The builder's overlap relaxation on the GPU (ccs_make_bodies_device) against the host builder.

relax() of src/bodies.js:97-146 sweeps the particles one by one in index
order; the device runs each sweep as 27 race-free phases of cells, so the
same pushes happen in another order and the pile comes out equivalent, not
bit-identical.  Everything else the builder makes -- the run's scalars, the
layers and masses, the tags, the velocities, the home positions -- must be
identical.  The relaxed piles are compared as a relaxation is meant to be
assessed: each particle ends within a small fraction of a radius of where the
host puts it, and the overlaps left (pairs closer than 0.96 diameters) have
the same count, mean and worst case to within a few tens of per cent.
"""
import time

import numpy as np
import pytest
from scipy.spatial import cKDTree

pytestmark = pytest.mark.gpu


def overlaps(P, a):
    D = 2 * a * 0.96
    pairs = cKDTree(P).query_pairs(D, output_type="ndarray")
    d = np.linalg.norm(P[pairs[:, 0]] - P[pairs[:, 1]], axis=1)
    ov = (D - d) / a
    return len(ov), float(ov.mean()) if len(ov) else 0.0, float(ov.max()) if len(ov) else 0.0


@pytest.mark.parametrize("N", [16384, 262144])
def test_device_relax_matches_host(ccmod, N):
    from cosmic_collisions_b200 import _lib as L, configs
    opt = L.make_opt(**configs.full_impact_opt(N))
    t0 = time.perf_counter()
    sh, ph, vh, mh, hh = L.make_bodies(opt)
    t1 = time.perf_counter()
    sd, pd, vd, md, hd = L.make_bodies(opt, 0)
    t2 = time.perf_counter()
    print(f"N={N}: host builder {t1 - t0:.2f} s, with the device relaxation {t2 - t1:.2f} s")
    assert bytes(sh) == bytes(sd)
    assert np.array_equal(mh, md) and np.array_equal(vh, vd)
    assert np.array_equal(hh[:, 3], hd[:, 3])          # home: the relaxed ball's own frame, and its seed
    assert np.abs(hh[:, :3] - hd[:, :3]).max() < 0.5 * sh.a * 10
    assert np.array_equal(ph[:, 3], pd[:, 3])
    a = sh.a
    for lo, hi in ((0, sh.n1), (sh.n1, sh.N)):
        Ph, Pd = ph[lo:hi, :3].astype(np.float64), pd[lo:hi, :3].astype(np.float64)
        disp = np.linalg.norm(Pd - Ph, axis=1) / a
        nh, mh_, wh = overlaps(Ph, a)
        nd, md_, wd = overlaps(Pd, a)
        print(f"  body {lo}-{hi}: displacement median {np.median(disp):.4f} a, p99 {np.percentile(disp, 99):.4f} a; "
              f"overlaps host {nh} mean {mh_:.4f} worst {wh:.4f}, device {nd} mean {md_:.4f} worst {wd:.4f}")
        assert np.median(disp) < 0.05 and np.percentile(disp, 99) < 0.5
        assert 0.75 * nh <= nd <= 1.33 * nh
        assert 0.75 * mh_ <= md_ <= 1.33 * mh_
        assert wd <= 1.5 * wh + 0.01
