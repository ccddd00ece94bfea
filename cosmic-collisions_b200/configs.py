"""The workloads the step is run and measured on.

Each impact is a set of build(opt) options (src/nbody.js:114, with the
documented extensions mTarget / rhoR / rhoCrust / crustFrac for masses and
layers the reference fixes).  The gravity sweep is a particle set made here
(a Plummer sphere plus uniform debris), since it is not an impact.  All
inputs are synthetic and seeded.
"""
import math

import numpy as np

from . import _lib as L

DAY_8H = 2 * math.pi * 805 / (8 * 3600)   # an 8-hour day as a fraction of breakup spin (T = 805 s)


def small_impact_opt(N=16384):
    """The plain small giant impact: 0.9 + 0.1 M_earth, 1,638 impactor particles, iron core to 0.55 R
    (7.8 g/cc) under 3.3 g/cc silicate, 45 degrees at 1.0 v_esc, the page's default contact constants."""
    rhoR = 7.8 / 3.3
    coreV = 0.55 ** 3
    core = coreV * rhoR / (1 + coreV * (rhoR - 1))   # core volume fraction -> mass fraction
    return dict(N=N, q=0.1, dens=1.0, core=core, spin0=0.18, spin1=0.2, angle=45.0, incl=0.0, vfac=1.0, rest=0.3,
                n2=max(16, round(N * 1638 / 16384)), mImp=0.1, mTarget=0.9, rhoR=rhoR)


def full_impact_opt(N=262144, case="A"):
    """The full plain giant impact.  Case A: 0.9 + 0.1 M_earth at 45 degrees and 1.0 v_esc; target with
    core mass fraction 0.3 and a 2.7 g/cc crust on the outer 5 % of radius, spun to an 8-hour day.  Case B:
    a 0.15 M_earth impactor at 30 degrees and 1.4 v_esc (a hit & run: the second mesh box goes up)."""
    opt = dict(N=N, q=0.1, dens=1.0, core=0.3, spin0=DAY_8H, spin1=0.2, angle=45.0, incl=0.0, vfac=1.0, rest=0.3,
               mImp=0.1, mTarget=0.9, rhoR=7.8 / 3.3, rhoCrust=2.7 / 3.3, crustFrac=0.05)
    if case == "B":
        opt.update(q=0.15, mImp=0.15, angle=30.0, vfac=1.4)
    return opt


def _mulberry(seed):
    s = seed & 0xFFFFFFFF

    def nxt():
        nonlocal s
        s = (s + 0x6D2B79F5) & 0xFFFFFFFF
        t = ((s ^ (s >> 15)) * (1 | s)) & 0xFFFFFFFF
        t = ((t + (((t ^ (t >> 7)) * (61 | t)) & 0xFFFFFFFF)) & 0xFFFFFFFF) ^ t
        return ((t ^ (t >> 14)) & 0xFFFFFFFF) / 4294967296.0
    return nxt


def gravity_sweep(N=262144, debris=0.1, scale=1.0, seed=2024):
    """The gravity-only correctness sweep: N equal-mass particles totalling 1 M_earth, (1 - debris) of them
    in a Plummer sphere of scale radius `scale` R_earth (radius by inverse CDF, resampled until inside
    the +-6 R_earth box), the rest uniform in the box.  Returns (sim, pos4, vel4, mat) ready for
    NBody.upload; sim.a is the particle radius the builder gives N particles of one Earth volume."""
    rng = np.random.default_rng(seed)
    n_pl = N - int(round(N * debris))
    pos = np.zeros((N, 4), np.float32)
    k = 0
    while k < n_pl:
        m = n_pl - k
        u = rng.uniform(1e-12, 1.0, size=m)
        r = scale / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        z = rng.uniform(-1.0, 1.0, size=m)
        ph = rng.uniform(0.0, 2 * np.pi, size=m)
        rr = np.sqrt(1 - z * z)
        x = np.stack([r * rr * np.cos(ph), r * rr * np.sin(ph), r * z], 1)
        x = x[np.all(np.abs(x) < 6.0, axis=1)]
        pos[k:k + len(x), :3] = x
        k += len(x)
    pos[n_pl:, :3] = rng.uniform(-6.0, 6.0, size=(N - n_pl, 3))
    pos[:, 3] = 1.0                       # mantle, target body
    vel = np.zeros((N, 4), np.float32)
    mat = np.ones(N, np.float32)
    s = L.Sim()
    vp = 1.0 / N
    sgrid = (16 * math.pi * vp / 3) ** (1.0 / 3.0)
    a = 0.96 * sgrid / (2 * math.sqrt(2))
    s.N, s.W = N, 512 if N >= 131072 else 256 if N >= 32768 else 128
    s.H = N // s.W
    s.n1, s.n2 = N, 0
    s.G = 128 if N >= 65536 else 64
    s.m, s.a, s.cell = 1.0 / N, a, 2.6 * a
    vref = 1.5
    s.k = 4 * s.m * vref * vref / (a * a)
    s.dt = 0.35 / math.sqrt(2 * s.k / s.m)
    s.c, s.creep, s.damp = 0.0, 0.12, math.exp(-s.dt * 12)
    s.tK, s.kappa = 0.5 * 6.256e7 / 1200.0 / s.m, 0.3
    s.M1 = s.M = 1.0
    s.phase, s.impactT = 2, 0.0
    s.boxOn[0] = 1                        # the first box on the sphere's centre
    return s, pos, vel, mat


# the crater page's units: chicxulub.html:156-157
CRATER_L, CRATER_T, CRATER_V = 1e4, 10.0, 1000.0     # metres, seconds, m/s
CRATER_G = (0.0, -9.81 * CRATER_T * CRATER_T / CRATER_L, 0.0)
MAT_FROZEN, MAT_BASEMENT, MAT_PLATFORM, MAT_IMPACTOR = 0, 1, 2, 4


def crater_patch(N=16384, R=1.0, D=0.6, froz=0.08, sed=0.15, imp_frac=0.04, v_imp=2.0, angle=45.0, rest=0.3,
                 rho_t=2650.0, rho_i=2630.0, seed=20260827):
    """A patch of ground for the field-gravity step, in the crater page's units (10 km, 10 s): a cylinder
    of radius R and depth D filled with a jittered face-centred lattice -- its outer wall and floor
    (thickness froz) frozen, a platform layer over the top `sed`, basement below -- and an impactor ball
    (imp_frac of the particles, same spacing) one diameter above the surface, coming in at `angle` from the
    horizontal at v_imp.  The contact constants follow the page's formulas (chicxulub.html:626-633: the
    spring per unit mass for max(2.5, v_imp / 4), the dashpot for the restitution, creep 0.10).  Seeded
    synthetic input standing in for the page's own builder (its lattice fill and relax are page code).
    Returns (sim, pos4, vel4, mat) for NBody.upload, then NBody.set_field(CRATER_G, MAT_FROZEN)."""
    rng = np.random.default_rng(seed)
    n2 = max(16, int(round(N * imp_frac)))
    n1 = N - n2
    s = (math.pi * R * R * D * 4.0 / n1) ** (1.0 / 3.0)       # FCC cube side for n1 points in the cylinder
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])

    def fcc(lo, hi):
        ax = [np.arange(math.floor(lo[k] / s), math.ceil(hi[k] / s) + 1) for k in range(3)]
        g = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 1, 3)
        return ((g + base[None]) * s).reshape(-1, 3)

    pts = fcc((-R, -D, -R), (R, 0.0, R))
    pts = pts[(pts[:, 0] ** 2 + pts[:, 2] ** 2 <= R * R) & (pts[:, 1] <= 0.0) & (pts[:, 1] >= -D)]
    while len(pts) < n1:                                       # a little denser until the box holds n1
        s *= 0.99
        pts = fcc((-R, -D, -R), (R, 0.0, R))
        pts = pts[(pts[:, 0] ** 2 + pts[:, 2] ** 2 <= R * R) & (pts[:, 1] <= 0.0) & (pts[:, 1] >= -D)]
    pts = pts[np.sort(rng.choice(len(pts), n1, replace=False))]   # vacancies spread through the rock
    pts = pts + (rng.random(pts.shape) - 0.5) * (0.1 * s)
    a = 0.96 * s / (2 * math.sqrt(2))                          # JAM * s / (2 sqrt 2)
    r_imp = (n2 * s ** 3 / 4.0 * 3.0 / (4.0 * math.pi)) ** (1.0 / 3.0) * 1.05
    ball = fcc((-r_imp,) * 3, (r_imp,) * 3)
    ball = ball[np.sum(ball * ball, 1) <= r_imp * r_imp]
    while len(ball) < n2:
        r_imp *= 1.02
        ball = fcc((-r_imp,) * 3, (r_imp,) * 3)
        ball = ball[np.sum(ball * ball, 1) <= r_imp * r_imp]
    ball = ball[np.argsort(np.sum(ball * ball, 1), kind="stable")[:n2]]
    th = math.radians(angle)
    d = np.array([-math.cos(th) * math.sqrt(0.5), -math.sin(th), -math.cos(th) * math.sqrt(0.5)])
    d /= np.linalg.norm(d)
    c2 = -d * (2.2 * r_imp + 2 * a) + np.array([0.0, r_imp, 0.0])
    pos = np.zeros((N, 4), np.float32)
    vel = np.zeros((N, 4), np.float32)
    mat = np.ones(N, np.float32)
    pos[:n1, :3] = pts
    wall = (pts[:, 0] ** 2 + pts[:, 2] ** 2 > (R - froz) ** 2) | (pts[:, 1] < -(D - froz))
    pos[:n1, 3] = np.where(wall, MAT_FROZEN, np.where(pts[:, 1] > -sed, MAT_PLATFORM, MAT_BASEMENT))
    pos[n1:, :3] = ball + c2
    pos[n1:, 3] = MAT_IMPACTOR
    vel[n1:, :3] = d * v_imp
    mat[n1:] = rho_i / rho_t
    sim = L.Sim()
    sim.N, sim.W = N, 512 if N >= 131072 else 256 if N >= 32768 else 128
    sim.H = N // sim.W
    sim.n1, sim.n2 = n1, n2
    sim.G = 128 if N >= 65536 else 64
    sim.m = math.pi * R * R * D / n1 * CRATER_L ** 3 * rho_t   # kilograms a particle stands for
    sim.a, sim.cell = a, 2.6 * a
    vref = max(2.5, 0.25 * v_imp)
    sim.k = 4 * vref * vref / (a * a)
    sim.dt = 0.35 / math.sqrt(2 * sim.k / min(1.0, rho_i / rho_t))
    ln_e = math.log(rest)
    zeta = -ln_e / math.sqrt(math.pi * math.pi + ln_e * ln_e)
    sim.c = 2 * zeta * math.sqrt(sim.k / 2)
    sim.creep, sim.damp = 0.10, math.exp(-sim.dt * 12)
    sim.tK, sim.kappa = 0.5 * 6.256e7 / 1200.0, 0.3
    sim.settleLeft = sim.settleTotal = int(math.ceil(0.5 / sim.dt))
    sim.t = -float(np.linalg.norm(c2)) / v_imp
    return sim, pos, vel, mat


def ensemble_opts(count=64, seed=7):
    """A batch of impacts of uneven size: N uniform over the page's counts (src/shell.js:132), impactor
    mass log-uniform over 0.02-1 M_earth, angle uniform over 0-75 degrees, speed uniform over 1.0-2.6
    v_esc; layering as in the full impact."""
    rng = _mulberry(seed)
    counts = [16384, 32768, 65536, 131072, 262144]
    out = []
    for _ in range(count):
        N = counts[min(4, int(rng() * 5))]
        mimp = math.exp(math.log(0.02) + rng() * (math.log(1.0) - math.log(0.02)))
        opt = full_impact_opt(N)
        opt.update(q=mimp, mImp=mimp, angle=rng() * 75.0, vfac=1.0 + rng() * 1.6)
        out.append(opt)
    return out
