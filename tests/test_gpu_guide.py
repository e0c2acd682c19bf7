"""The learned directional proposal's network on the GPU against its float64 CPU oracle
(oracle/guide_oracle.py): the FP32 SIMT forward pass, the tcgen05 tensor-core forward pass (FP16
operands, FP32 accumulation), the gradients of the mixture's negative log-likelihood with
respect to the MLP and the hash grid, and Adam training lowering that loss.

Tolerances: FP32 forward vs float64 oracle 1e-4 relative (norm); tensor cores vs FP32 3e-2
relative (FP16 inputs, activations and weights carry ~11-bit mantissas through four layers);
gradients 1e-3 relative (norm) and per element 1e-3 of the largest.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOX_MIN = np.array([-1.0, -1.0, -1.0], np.float32)
BOX_MAX = np.array([1.0, 1.0, 1.0], np.float32)


def _fp(a):
    return np.ascontiguousarray(a, np.float32).ctypes.data_as(C.POINTER(C.c_float))


def _lib(pe):
    return pe._capi.load()


def _reset(pe, device, seed):
    pe._capi.check(_lib(pe).pe_device_guide_reset(device.handle, seed, _fp(BOX_MIN), _fp(BOX_MAX)))


def _params(pe, device):
    mlp = np.zeros(pe._capi.PE_GUIDE_MLP_PARAMS, np.float32)
    grid = np.zeros(pe._capi.PE_GUIDE_GRID_PARAMS, np.float32)
    pe._capi.check(_lib(pe).pe_device_guide_get(device.handle, _fp(mlp), _fp(grid)))
    return mlp, grid


def _set(pe, device, mlp, grid):
    pe._capi.check(_lib(pe).pe_device_guide_set(device.handle, _fp(mlp), _fp(grid)))


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _queries(rng, n):
    p = rng.uniform(-0.95, 0.95, (n, 3))
    nrm = _unit(rng.normal(size=(n, 3)))
    wo = _unit(rng.normal(size=(n, 3)))
    return np.concatenate([p, nrm, wo], axis=1).astype(np.float32)


def _eval(pe, device, q, tc):
    out = np.zeros((len(q), 40), np.float32)
    pe._capi.check(_lib(pe).pe_device_guide_eval(device.handle, _fp(q), len(q), 1 if tc else 0, _fp(out)))
    return out


@pytest.fixture()
def trained_like(pe, device):
    """A network with grid features and weights of trained magnitude (seeded)."""
    _reset(pe, device, 7)
    mlp, grid = _params(pe, device)
    rng = np.random.default_rng(3)
    grid = rng.uniform(-0.5, 0.5, grid.shape).astype(np.float32)
    mlp = (mlp + rng.normal(0.0, 0.05, mlp.shape)).astype(np.float32)
    _set(pe, device, mlp, grid)
    return mlp, grid


def test_fp32_forward_matches_oracle(pe, device, trained_like):
    import guide_oracle as go
    mlp, grid = trained_like
    q = _queries(np.random.default_rng(1), 64)
    mine = _eval(pe, device, q, tc=False)
    ref = go.outputs(mlp, grid, q, BOX_MIN, BOX_MAX)
    err = np.linalg.norm(mine - ref) / np.linalg.norm(ref)
    assert err < 1e-4, err


def test_tensor_core_forward_matches_fp32(pe, device, trained_like):
    q = _queries(np.random.default_rng(2), 1000)   # 8 tiles of 128, the last one partial
    tc = _eval(pe, device, q, tc=True)
    fp = _eval(pe, device, q, tc=False)
    assert np.all(np.isfinite(tc))
    err = np.linalg.norm(tc - fp) / np.linalg.norm(fp)
    assert err < 3e-2, err
    # row by row as well: no tile or lane mixes up its rows
    row_err = np.linalg.norm(tc - fp, axis=1) / np.maximum(np.linalg.norm(fp, axis=1), 1e-6)
    assert np.max(row_err) < 1e-1, np.max(row_err)


def _samples(rng, n):
    q = _queries(rng, n)
    d = _unit(rng.normal(size=(n, 3)))
    c = rng.uniform(0.1, 2.0, (n, 1))
    return np.concatenate([q, d, c], axis=1).astype(np.float32)


def test_gradients_match_oracle(pe, device, trained_like):
    import guide_oracle as go
    mlp, grid = trained_like
    s = _samples(np.random.default_rng(5), 48)
    gm = np.zeros_like(mlp)
    gg = np.zeros(pe._capi.PE_GUIDE_GRID_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    pe._capi.check(_lib(pe).pe_device_guide_grad(device.handle, _fp(s), len(s), 0.0, _fp(gm), _fp(gg), _fp(loss)))
    ref_loss, ref_gm, ref_gg = go.gradients(mlp, grid, s, BOX_MIN, BOX_MAX)
    assert abs(loss[0] - ref_loss) <= 1e-4 * abs(ref_loss) + 1e-4, (loss[0], ref_loss)
    err = np.linalg.norm(gm - ref_gm) / np.linalg.norm(ref_gm)
    assert err < 1e-3, err
    assert np.max(np.abs(gm - ref_gm)) < 1e-3 * np.max(np.abs(ref_gm))
    keys = np.array(sorted(ref_gg), np.int64)
    ref = np.array([ref_gg[k] for k in keys])
    err_g = np.linalg.norm(gg[keys] - ref) / np.linalg.norm(ref)
    assert err_g < 1e-3, err_g
    # nothing outside the touched cells
    mask = np.ones(gg.shape, bool)
    mask[keys] = False
    assert np.all(gg[mask] == 0.0)


def test_training_fits_a_direction_field(pe, device):
    """Samples whose directions cluster around a position-dependent direction: Adam on the
    device must lower the mixture's negative log-likelihood well below that of the initial,
    broad mixture, and the fitted density must favour the true direction."""
    _reset(pe, device, 11)
    rng = np.random.default_rng(9)

    def batch(n):
        p = rng.uniform(-0.9, 0.9, (n, 3))
        target = _unit(np.stack([np.sign(p[:, 0]) + 0.2, 0.5 + p[:, 1], np.cos(3 * p[:, 2])], axis=1))
        d = _unit(target + rng.normal(0.0, 0.15, target.shape))
        nrm = np.tile([0.0, 1.0, 0.0], (n, 1))
        wo = np.tile([0.0, 0.0, 1.0], (n, 1))
        c = np.ones((n, 1))
        return np.concatenate([p, nrm, wo, d, c], axis=1).astype(np.float32), target

    losses = []
    for it in range(300):
        s, _ = batch(4096)
        loss = np.zeros(1, np.float32)
        pe._capi.check(_lib(pe).pe_device_guide_grad(device.handle, _fp(s), len(s), 5e-3, None, None, _fp(loss)))
        losses.append(loss[0] / len(s))
    first, last = np.mean(losses[:5]), np.mean(losses[-5:])
    assert last < first - 1.0, (first, last)
    # density along the true direction vs a random one, from the tensor-core outputs
    s, target = batch(512)
    out = _eval(pe, device, s[:, :9], tc=True)
    import guide_oracle as go
    hit = np.mean([go.vmf(*go.decode(o)[:2], t) @ go.decode(o)[2] for o, t in zip(out.astype(np.float64), target)])
    assert hit > 1.0, hit   # uniform density is 1/(4π) ≈ 0.08
