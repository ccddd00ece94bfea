"""A whole run on the CPU oracle: the host logic of src/nbody.js around the
oracle's step -- settle, the rigid approach, the full phase with a synchronous
analysis every 360 steps (window.__impact.runTo, index.html:592-600), and
applyReport's placeBoxes / applyPerm / setPP (src/nbody.js:912-966).  Test
infrastructure: it drives the checker, never the product.
"""
import math

import numpy as np

from oracle import oracle as O

FL = 6.0


class OracleRun:
    def __init__(self, opt):
        sim, pos, vel, mat, home = O.build_run(O.make_opt(**opt))
        self.e = O.Engine(sim, pos, vel, mat)
        self.analyzed_at = 0
        self.analyses = 0
        self.report = None
        self.ref = None

    @property
    def sim(self):
        return self.e.sim

    def settle_some(self, n):
        s = self.sim
        n = min(n, s.settleLeft)
        for _ in range(n):
            self.e.step(True, False)
        s.settleLeft -= n
        if s.settleLeft == 0:
            s.phase = 1
            self.analyzed_at = s.stepNo

    def analyze(self):
        s = self.sim
        self.analyzed_at = s.stepNo
        sort = False
        if s.phase == 2:
            sort = self.analyses % 8 == 0
            self.analyses += 1
        D = self.e.diag()
        r, lst, perm = O.fof(s.N, s.m, s.a, self.e.buf("pos"), self.e.buf("vel"), self.e.buf("mat"), D, s.k,
                             2 * s.a, O.PP_CAP, sort)
        self.report = r
        t = s.t
        # placeBoxes
        s.boxOn[0] = 1
        for k in range(3):
            s.boxCen[0][k] = r.core[k]
            s.boxVel[0][k] = r.bodyVel[k]
        s.boxT[0] = t
        if r.hasSecond and r.secMass > 0.05:
            d = max(abs(r.secCore[k] - r.core[k]) for k in range(3))
            far = FL - 1.3 * math.pow(r.secMass, 1.0 / 3.0)
            if not s.boxOn[1] and d > far:
                s.boxOn[1] = 1
                w = r.secMass / s.m
                self.e.prime_mono(1, np.array([r.secCore[0] * w, r.secCore[1] * w, r.secCore[2] * w, w], np.float32))
            elif s.boxOn[1] and d < far - 0.5:
                s.boxOn[1] = 0
            for k in range(3):
                s.boxCen[1][k] = r.secCore[k]
                s.boxVel[1][k] = r.secVel[k]
            s.boxT[1] = t
        else:
            s.boxOn[1] = 0
        going = s.phase == 2 or any(s.bulk0[k] != 0 for k in range(3))
        if self.ref is None and going:
            self.ref = {"E": r.KE + r.PE + r.EL, "EQ": r.KE + r.PE + r.EL + r.Q, "L": r.L, "scale": r.KE - r.PE}
        if perm is not None:
            self.e.apply_perm(perm)
        self.e.set_pp(lst)

    def run_to(self, t):
        while self.sim.phase == 0:
            self.settle_some(64)
        while self.sim.phase == 1 and self.sim.t < t:
            self.e.rigid_step(0.01)
        while self.sim.phase == 2 and self.sim.t < t:
            self.e.step(False, False)
            self.sim.t += self.sim.dt
            if self.sim.stepNo - self.analyzed_at >= 360:
                self.analyze()
        self.analyze()
        return self.sim.t
