"""CPU oracle of the learned directional proposal (test infrastructure only).

A float64 numpy restatement of the network the CUDA library runs: the multiresolution hash-grid
encoding (Müller et al. 2022: 16 levels, 2 features, 2^18-entry tables, dense indexing while the
level's grid fits, spatial hash otherwise, trilinear interpolation), the 48→64→64→64→64 ReLU MLP,
the 8-lobe von Mises–Fisher mixture decoded from its first 40 outputs, the mixture's negative
log-likelihood and its exact gradient back through the MLP into the grid features.

Grid cell indices and corner weights are computed in float32, as the device does, so both pick
the same cells; everything after that is float64.
"""
from __future__ import annotations

import numpy as np

LEVELS, FEATURES, LOG2T = 16, 2, 18
TABLE = 1 << LOG2T
NIN, NHID, NOUT, LOBES = 48, 64, 64, 8
OFF_W1 = 0
OFF_B1 = OFF_W1 + NHID * NIN
OFF_W2 = OFF_B1 + NHID
OFF_B2 = OFF_W2 + NHID * NHID
OFF_W3 = OFF_B2 + NHID
OFF_B3 = OFF_W3 + NHID * NHID
OFF_W4 = OFF_B3 + NHID
OFF_B4 = OFF_W4 + NOUT * NHID
NPARAMS = OFF_B4 + NOUT
LOGK_MIN, LOGK_MAX = -6.0, 7.0


def level_scales():
    """16 · 2^(7l/15) rounded: the device's fixed resolution table."""
    return [np.float32(round(16 * 2 ** (7 * l / 15))) for l in range(LEVELS)]


def grid_index(level, x, y, z, res):
    r1 = int(res) + 1
    if r1 ** 3 <= TABLE:
        i = (x + y * r1 + z * r1 * r1) & 0xFFFFFFFF
    else:
        i = ((x * 1) ^ ((y * 2654435761) & 0xFFFFFFFF) ^ ((z * 805459861) & 0xFFFFFFFF)) & 0xFFFFFFFF
    return level * TABLE + (i & (TABLE - 1))


def unit(p, box_min, box_max):
    inv = np.float32(1.0) / (np.asarray(box_max, np.float32) - np.asarray(box_min, np.float32))
    u = (np.asarray(p, np.float32) - np.asarray(box_min, np.float32)) * inv
    return np.clip(u, np.float32(0.0), np.float32(1.0)).astype(np.float32)


def corners(level, u, scales):
    res = scales[level]
    pos = (u * res).astype(np.float32)
    f0 = np.floor(pos)
    f = (pos - f0).astype(np.float32)
    i0 = f0.astype(np.int64)
    out = []
    for k in range(8):
        d = (k & 1, (k >> 1) & 1, (k >> 2) & 1)
        idx = grid_index(level, int(i0[0] + d[0]), int(i0[1] + d[1]), int(i0[2] + d[2]), res)
        w = 1.0
        for a in range(3):
            w *= float(f[a]) if d[a] else 1.0 - float(f[a])
        out.append((idx, w))
    return out


def encode(grid, p, n, wo, box_min, box_max, scales):
    u = unit(p, box_min, box_max)
    x = np.zeros(NIN)
    cs = []
    for l in range(LEVELS):
        c = corners(l, u, scales)
        cs.append(c)
        for idx, w in c:
            x[2 * l] += w * grid[2 * idx]
            x[2 * l + 1] += w * grid[2 * idx + 1]
    x[32:35] = n
    x[35:38] = wo
    return x, cs


def forward(P, x):
    P = np.asarray(P, np.float64)
    W1 = P[OFF_W1:OFF_B1].reshape(NHID, NIN)
    W2 = P[OFF_W2:OFF_B2].reshape(NHID, NHID)
    W3 = P[OFF_W3:OFF_B3].reshape(NHID, NHID)
    W4 = P[OFF_W4:OFF_B4].reshape(NOUT, NHID)
    h1 = np.maximum(W1 @ x + P[OFF_B1:OFF_W2], 0.0)
    h2 = np.maximum(W2 @ h1 + P[OFF_B2:OFF_W3], 0.0)
    h3 = np.maximum(W3 @ h2 + P[OFF_B3:OFF_W4], 0.0)
    o = W4 @ h3 + P[OFF_B4:]
    return h1, h2, h3, o


def decode(o):
    raw = o[:40].reshape(LOBES, 5)
    m = raw[:, :3]
    ln = np.linalg.norm(m, axis=1) + 1e-6
    mu = m / ln[:, None]
    kappa = np.exp(np.clip(raw[:, 3], LOGK_MIN, LOGK_MAX))
    lg = raw[:, 4] - raw[:, 4].max()
    w = np.exp(lg)
    w /= w.sum()
    return mu, kappa, w, ln


def vmf(mu, kappa, d):
    return kappa / (2.0 * np.pi * -np.expm1(-2.0 * kappa)) * np.exp(kappa * (mu @ d - 1.0))


def nll_and_grad(o, d):
    """−log q(d) and its gradient with respect to the network outputs."""
    mu, kappa, w, ln = decode(o)
    v = vmf(mu, kappa, d)
    q = max(float(w @ v), 1e-20)
    r = w * v / q
    g = np.zeros(NOUT)
    raw = o[:40].reshape(LOBES, 5)
    for k in range(LOBES):
        g[5 * k + 4] = w[k] - r[k]
        if LOGK_MIN < raw[k, 3] < LOGK_MAX:
            kap = kappa[k]
            dlogv = 1.0 / kap - 2.0 / np.expm1(2.0 * kap) + (mu[k] @ d - 1.0)
            g[5 * k + 3] = -r[k] * dlogv * kap
        mw = mu[k] @ d
        g[5 * k:5 * k + 3] = -r[k] * kappa[k] / ln[k] * (d - mw * mu[k])
    return -np.log(q), g


def gradients(P, grid, samples, box_min, box_max):
    """Σ c·(−log q) over samples (rows of 13: p, n, wo, d, c) → (loss, dP, {grid index: grad})."""
    scales = level_scales()
    P = np.asarray(P, np.float64)
    W = [P[OFF_W1:OFF_B1].reshape(NHID, NIN), P[OFF_W2:OFF_B2].reshape(NHID, NHID),
         P[OFF_W3:OFF_B3].reshape(NHID, NHID), P[OFF_W4:OFF_B4].reshape(NOUT, NHID)]
    offs = [(OFF_W1, OFF_B1, NHID, NIN), (OFF_W2, OFF_B2, NHID, NHID), (OFF_W3, OFF_B3, NHID, NHID),
            (OFF_W4, OFF_B4, NOUT, NHID)]
    dP = np.zeros(NPARAMS)
    dgrid = {}
    loss = 0.0
    for s in np.asarray(samples, np.float64):
        p, n, wo, d, c = s[0:3], s[3:6], s[6:9], s[9:12], s[12]
        x, cs = encode(grid, p.astype(np.float32), n, wo, box_min, box_max, scales)
        h1, h2, h3, o = forward(P, x)
        l, go = nll_and_grad(o, d)
        loss += c * l
        delta = c * go
        acts = [x, h1, h2, h3]
        for layer in (3, 2, 1, 0):
            ow, ob, no, ni = offs[layer]
            a = acts[layer]
            dP[ow:ow + no * ni] += np.outer(delta, a).ravel()
            dP[ob:ob + no] += delta
            din = W[layer].T @ delta
            if layer > 0:
                din = din * (acts[layer] > 0)
            delta = din
        for lvl in range(LEVELS):
            for idx, wgt in cs[lvl]:
                for f in range(2):
                    key = 2 * idx + f
                    dgrid[key] = dgrid.get(key, 0.0) + wgt * delta[2 * lvl + f]
    return loss, dP, dgrid


def outputs(P, grid, queries, box_min, box_max):
    """Network outputs (first 40) for query rows (p, n, wo)."""
    scales = level_scales()
    out = []
    for q in np.asarray(queries, np.float64):
        x, _ = encode(grid, q[0:3].astype(np.float32), q[3:6], q[6:9], box_min, box_max, scales)
        out.append(forward(P, x)[3][:40])
    return np.array(out)
