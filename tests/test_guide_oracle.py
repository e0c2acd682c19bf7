"""The proposal network's CPU oracle checks itself: its analytic gradients (mixture NLL → MLP →
hash grid) agree with central finite differences in float64, and the vMF mixture it decodes
integrates to one over the sphere."""
import numpy as np

import guide_oracle as go

BOX_MIN = np.array([-1.0, -1.0, -1.0], np.float32)
BOX_MAX = np.array([1.0, 1.0, 1.0], np.float32)


def _setup(seed=0):
    rng = np.random.default_rng(seed)
    P = rng.normal(0.0, 0.15, go.NPARAMS)
    grid = np.zeros(go.LEVELS * go.TABLE * 2)
    s = []
    for _ in range(3):
        p = rng.uniform(-0.9, 0.9, 3)
        n = rng.normal(size=3)
        wo = rng.normal(size=3)
        d = rng.normal(size=3)
        s.append(np.concatenate([p, n / np.linalg.norm(n), wo / np.linalg.norm(wo), d / np.linalg.norm(d),
                                 [rng.uniform(0.5, 1.5)]]))
    s = np.array(s)
    # non-zero features in the cells these samples touch
    scales = go.level_scales()
    for row in s:
        _, cs = go.encode(grid, row[:3].astype(np.float32), row[3:6], row[6:9], BOX_MIN, BOX_MAX, scales)
        for lvl in cs:
            for idx, _ in lvl:
                grid[2 * idx:2 * idx + 2] = rng.uniform(-0.5, 0.5, 2)
    return P, grid, s


def test_mlp_gradient_matches_finite_differences():
    P, grid, s = _setup(1)
    _, dP, _ = go.gradients(P, grid, s, BOX_MIN, BOX_MAX)
    rng = np.random.default_rng(2)
    picks = list(rng.choice(go.NPARAMS, 40, replace=False)) + [go.OFF_B4 + k for k in range(40)]
    h = 1e-6
    for i in picks:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (go.gradients(Pp, grid, s, BOX_MIN, BOX_MAX)[0] - go.gradients(Pm, grid, s, BOX_MIN, BOX_MAX)[0]) / (2 * h)
        assert abs(fd - dP[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, dP[i])


def test_grid_gradient_matches_finite_differences():
    P, grid, s = _setup(3)
    _, _, dg = go.gradients(P, grid, s, BOX_MIN, BOX_MAX)
    h = 1e-6
    for key in list(dg)[:: max(1, len(dg) // 30)]:
        gp, gm = grid.copy(), grid.copy()
        gp[key] += h
        gm[key] -= h
        fd = (go.gradients(P, gp, s, BOX_MIN, BOX_MAX)[0] - go.gradients(P, gm, s, BOX_MIN, BOX_MAX)[0]) / (2 * h)
        assert abs(fd - dg[key]) <= 1e-5 * max(1.0, abs(fd)), (key, fd, dg[key])


def test_mixture_integrates_to_one():
    rng = np.random.default_rng(4)
    o = rng.normal(0.0, 1.0, go.NOUT)
    o[3:40:5] = rng.uniform(-3.0, 4.0, 8)  # log κ from broad to peaked
    mu, kappa, w, _ = go.decode(o)
    # stratified quadrature over the sphere in (cos θ, φ)
    n = 1200
    ct = (np.arange(n) + 0.5) / n * 2.0 - 1.0
    ph = (np.arange(2 * n) + 0.5) / (2 * n) * 2.0 * np.pi
    C, F = np.meshgrid(ct, ph, indexing="ij")
    st = np.sqrt(1.0 - C * C)
    d = np.stack([st * np.cos(F), st * np.sin(F), C], axis=-1).reshape(-1, 3)
    dens = sum(w[k] * go.vmf(mu[k][None, :], kappa[k], d.T).ravel() for k in range(go.LOBES))
    integral = dens.mean() * 4.0 * np.pi
    assert abs(integral - 1.0) < 2e-3, integral
