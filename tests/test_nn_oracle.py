"""The learned correction's CPU oracle, checked on its own (no GPU).

* Labels: the isolated pair's mesh force (meshPairTable's field(),
  src/nbody.js:60-91) tends to the node-softened Newton force far out, and
  its placement average reproduces the reference's pair table (the same
  arithmetic averaged over random placings, src/nbody.js:93-106).
* The network's backward formulas: the oracle's gradient (with its BF16
  roundings switched off) matches central finite differences of its loss.
"""
import numpy as np

from oracle import nn_oracle as NO
from oracle import oracle as O


def test_label_is_newton_softened_far_out():
    rng = np.random.default_rng(3)
    rec = np.zeros((64, 6))
    u = rng.normal(size=(64, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    r = 4.5
    rec[:, :3] = u * r
    rec[:, 3:] = rng.random((64, 3))
    lab = O.nn_labels(rec)
    along = (lab * u).sum(1) * r * r
    # node softening 0.5 cell^2 and the cloud-in-cell spread: within a few per cent of Newton at 4.5 cells
    assert np.all(np.abs(along - 1.0) < 0.08)
    perp = lab - (lab * u).sum(1)[:, None] * u
    assert np.abs(perp).max() < 0.05 * np.abs(lab).max()


def test_label_placement_average_is_the_pair_table():
    f, p = O.pair_table()
    rng = np.random.default_rng(5)
    cut = 5.0
    for b in (6, 20, 40):
        r = (b + 0.5) / 64 * cut
        n = 400
        u = rng.normal(size=(n, 3))
        u /= np.linalg.norm(u, axis=1)[:, None]
        rec = np.concatenate([u * r, rng.random((n, 3))], axis=1)
        lab = O.nn_labels(rec)
        mean = ((lab * u).sum(1) * r * r).mean()
        # the table is an 80-placing average (src/nbody.js:94); the spread of single placings sets the bound
        spread = ((lab * u).sum(1) * r * r).std()
        assert abs(mean - f[b]) < 4 * spread / np.sqrt(80) + 4 * spread / np.sqrt(n) + 1e-6, (b, mean, f[b], spread)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    p = np.zeros(NO.PARAMS)
    P = NO.SL
    p[P["W1"][0]:P["b1"][0]] = rng.uniform(-0.4, 0.4, 384)
    p[P["b1"][0]:P["W2"][0]] = rng.uniform(-0.1, 0.1, 64)
    p[P["W2"][0]:P["b2"][0]] = rng.uniform(-0.125, 0.125, 4096)
    p[P["b2"][0]:P["W3"][0]] = rng.uniform(-0.1, 0.1, 64)
    p[P["W3"][0]:P["b3"][0]] = rng.uniform(-0.125, 0.125, 192)
    p[P["b3"][0]:] = rng.uniform(-0.1, 0.1, 3)
    rec = np.concatenate([rng.uniform(-2, 2, (40, 3)), rng.random((40, 3))], axis=1)
    lab = rng.normal(size=(40, 3)) * 0.3
    g, loss = NO.grad(p, rec, lab, exact=True)
    for k in rng.choice(NO.PARAMS, 60, replace=False):
        h = 1e-5
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        lp = NO.grad(pp, rec, lab, exact=True)[1]
        lm = NO.grad(pm, rec, lab, exact=True)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(fd), (k, fd, g[k])


def test_bf16_rounding_is_round_to_nearest_even():
    # BF16 keeps 7 fraction bits: the spacing at 1 is 2^-7
    x = np.array([1.0, 1 + 2 ** -8, 1 + 2 ** -8 + 2 ** -10, 1 + 3 * 2 ** -8, -3.14159, 0.0], np.float32)
    b = NO.bf16(x)
    assert b[0] == 1.0
    assert b[1] == 1.0                    # a tie goes to the even fraction (0)
    assert b[2] == 1 + 2 ** -7            # above the tie rounds up
    assert b[3] == 1 + 2 ** -6            # a tie between fractions 1 and 2 goes to 2
    assert b[4] == -3.140625 and b[5] == 0.0
