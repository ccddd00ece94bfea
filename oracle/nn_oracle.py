"""CPU oracle of the learned pairwise correction -- test infrastructure only.

It restates in numpy what the library's tensor-core kernels compute, with the
BF16 roundings at the same places, so the device's forward pass, its
gradients and the learned P3M pass can be checked against it:

  input   x = (d.xyz in cells, s.xyz - 1/2); each feature as a high and a low
          BF16 part, both through the same BF16 first-layer weights;
  layers  h1 = x W1^T + b1, a1 = bf16(silu(h1)); h2 = a1 W2^T + b2,
          a2 = bf16(silu(h2)); y = a2 W3^T + b3 (FP32 biases, FP32 sums);
  loss    mean over rows and components of (y - label)^2;
  back    dy = bf16(2 e / (3 n)); dH2 = bf16((dy W3) * silu'(h2));
          dH1 = bf16((dH2 W2) * silu'(h1)); weight gradients are sums over rows
          of the BF16 operands (FP32 on the device, binary64 here).

The network's target is the isolated pair's mesh force (meshPairTable's
field(), src/nbody.js:60-91; orc_nn_label) less the node-softened Newton
force d / (r^2 + 1/2)^1.5 in cells (softened_newton).  The learned P3M pass
follows src/glsl-sim.js:676-754 with the table's model of the mesh's pull
replaced by the network's inside half the cut: acc += m_j (N_a(d) tau_out -
same * (tau_in (d / (r^2 + FH^2/2)^1.5 + y(d, s) / FH^2) + (1 - tau_in)
tau_out T(r))), tau_in the smoothstep from 0.8 of the half cut to it, tau_out
the plain pass's taper to the full cut; pot is the plain pass's; times Gm;
one slice.
"""
import numpy as np

PARAMS = 4803
SL = {"W1": (0, (64, 6)), "b1": (384, (64,)), "W2": (448, (64, 64)), "b2": (4544, (64,)), "W3": (4608, (3, 64)),
      "b3": (4800, (3,))}


def unpack(p):
    return {k: np.asarray(p[o:o + int(np.prod(s))], np.float32).reshape(s) for k, (o, s) in SL.items()}


def bf16(x):
    """Round float32 to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(x.shape)


def silu(h):
    return h / (1.0 + np.exp(-h))


def silu_grad(h):
    s = 1.0 / (1.0 + np.exp(-h))
    return s * (1.0 + h * (1.0 - s))


def _ident(x):
    return np.asarray(x, np.float64)


def features(rec, exact=False):
    rec = np.asarray(rec, np.float32)
    x = np.concatenate([rec[:, :3], rec[:, 3:6] - np.float32(0.5)], axis=1).astype(np.float32)
    if exact:
        return x.astype(np.float64)
    hi = bf16(x)
    lo = bf16(x - hi)
    return hi.astype(np.float64) + lo.astype(np.float64)


def forward(params, rec, keep=False, exact=False):
    """exact=True: no BF16 rounding anywhere (binary64 throughout), for checking the formulas themselves."""
    P = unpack(params)
    rb = _ident if exact else (lambda v: bf16(np.asarray(v, np.float32)).astype(np.float64))
    x = features(rec, exact)
    W1, W2, W3 = (rb(P[k]) for k in ("W1", "W2", "W3"))
    h1 = x @ W1.T + P["b1"]
    a1 = rb(silu(h1))
    h2 = a1 @ W2.T + P["b2"]
    a2 = rb(silu(h2))
    y = a2 @ W3.T + P["b3"]
    if keep:
        return y, (x, h1, a1, h2, a2, W1, W2, W3)
    return y


def grad(params, rec, lab, exact=False):
    """(flat gradient, loss) of the mean squared error over the records."""
    n = len(rec)
    rb = _ident if exact else (lambda v: bf16(np.asarray(v, np.float32)).astype(np.float64))
    y, (x, h1, a1, h2, a2, W1, W2, W3) = forward(params, rec, keep=True, exact=exact)
    e = y - np.asarray(lab, np.float64)
    loss = float((e * e).sum() / (3.0 * n))
    gs = 2.0 / (3.0 * n)
    dy = rb(e * gs)
    dH2 = rb((dy @ W3) * silu_grad(h2))
    dH1 = rb((dH2 @ W2) * silu_grad(h1))
    g = np.zeros(PARAMS)
    g[SL["W1"][0]:SL["b1"][0]] = (dH1.T @ x).ravel()
    g[SL["b1"][0]:SL["W2"][0]] = dH1.sum(0)
    g[SL["W2"][0]:SL["b2"][0]] = (dH2.T @ a1).ravel()
    g[SL["b2"][0]:SL["W3"][0]] = dH2.sum(0)
    g[SL["W3"][0]:SL["b3"][0]] = (dy.T @ a2).ravel()
    g[SL["b3"][0]:] = dy.sum(0)
    return g, loss


def softened_newton(rec):
    """d / (r^2 + 1/2)^1.5 in cells: the mesh's pair force when the two particles share no mesh node."""
    d = np.asarray(rec, np.float64)[:, :3]
    return d / (((d * d).sum(1) + 0.5) ** 1.5)[:, None]


def table_model(rec, f, a_cells):
    """The plain pass's model of the mesh pair force in cells^-2: T.f / max(r^2, a^2) along d (PPFORCE_FS,
    src/glsl-sim.js:738-744), the table's force column read over 64 bins to 5 cells."""
    d = np.asarray(rec, np.float64)[:, :3]
    r = np.sqrt((d * d).sum(1))
    xx = np.clip(r * (64.0 / 5.0) - 0.5, 0.0, 63.0)
    k = xx.astype(int)
    k1 = np.minimum(k + 1, 63)
    f = np.asarray(f, np.float64)
    T = f[k] + (f[k1] - f[k]) * (xx - k)
    return d * (T / np.maximum(r * r, a_cells * a_cells) / np.maximum(r, 1e-300))[:, None]


def target(rec, mesh):
    """The network's label: the mesh force (orc_nn_label) less the softened Newton force."""
    return np.asarray(mesh, np.float64) - softened_newton(rec)


def pp_nn(u, list4, box, count, tab, params, box_of):
    """The learned P3M pass over a loose list of `count` entries: force slice 0 (count x 4, binary64).
    The network's model of the mesh's pull replaces the pair table's inside half the cut (weight tau_in,
    smoothstep from 0.8 of the half cut to the half cut); beyond it the pass is the plain one (the table,
    tapered to the full cut as PPFORCE_FS does, src/glsl-sim.js:738-750).
    u: the oracle's uniforms; box_of(u, p) -> (box, g) the oracle's GLSL_BOX."""
    list4 = np.asarray(list4, np.float32)
    cut = np.float32(u.cut)
    cutN = np.float32(np.float32(0.5) * cut)
    cutN2 = np.float32(cutN * cutN)
    cut2 = np.float32(cut * cut)
    a2 = float(u.a2)
    a = np.sqrt(a2)
    invH = float(u.invH)
    out = np.zeros((count, 4))
    g = [box_of(u, list4[j, :3])[1] for j in range(count)]

    def smooth(e0, e1, x):
        t = min(max((x - e0) / (e1 - e0), 0.0), 1.0)
        return t * t * (3.0 - 2.0 * t)

    for i in range(count):
        P = list4[i]
        if P[3] == 0.0:
            continue
        js, recs, inner = [], [], []
        for j in range(count):
            if j == i:
                continue
            d = (list4[j, :3] - P[:3]).astype(np.float32)
            r2 = np.float32(np.float32(np.float32(d[0] * d[0]) + np.float32(d[1] * d[1])) + np.float32(d[2] * d[2]))
            if r2 >= cut2:
                continue
            js.append(j)
            inner.append(r2 < cutN2)
            dc = (list4[j, :3].astype(np.float64) - P[:3]) * invH
            s = g[j] - np.floor(g[j])
            recs.append([dc[0], dc[1], dc[2], s[0], s[1], s[2]])
        if not js:
            continue
        y = forward(params, np.asarray(recs, np.float32))
        acc = np.zeros(3)
        pot = 0.0
        for q, j in enumerate(js):
            Q = list4[j].astype(np.float64)
            d = Q[:3] - P[:3].astype(np.float64)
            r2 = float(d @ d)
            r = np.sqrt(r2)
            invN = 1.0 / np.sqrt(r2 + a2)
            tau_out = smooth(float(cut), 0.8 * float(cut), r)
            tau_in = smooth(float(cutN), 0.8 * float(cutN), r) if inner[q] else 0.0
            same = box[i] >= 0 and box[j] == box[i]
            f = d * invN ** 3 * tau_out
            Ty = 0.0
            if same:
                xx = min(max(r * 64.0 / cut - 0.5, 0.0), 63.0)
                k = int(xx)
                k1 = min(k + 1, 63)
                Tx = tab[k, 0] + (tab[k1, 0] - tab[k, 0]) * (xx - k)
                Ty = tab[k, 1] + (tab[k1, 1] - tab[k, 1]) * (xx - k)
                table = d / max(r, 1e-6) * Tx / max(r2, a2)
                learned = d / (r2 + float(u.eps2Cell)) ** 1.5 + y[q] * invH * invH
                f = f - tau_in * learned - (1.0 - tau_in) * tau_out * table
            acc += f * Q[3]
            pot += Q[3] * (-invN - Ty / max(r, a)) * tau_out
        out[i, :3] = acc * u.Gm
        out[i, 3] = pot * u.Gm
    return out
