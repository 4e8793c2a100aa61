"""Particle -> grid deposition on the GPU against the reference's outputs
(tests/golden/deposit.npz) and its ledger and uniform-field properties.

Tolerances: cell masses to 1e-12 of the largest cell mass and the outside mass to rtol 1e-12
(the GPU adds each particle's share by FP64 atomics, so only the order of the additions
differs from the reference; a particle's weights round like the reference's but for CUDA's
exp / acos / atan2 in the cell geometry); trilinear counts exactly; the float32 fields to 1e-6
of their largest value, as the reference's own Numba-against-readable test; the mass ledger
(grid + outside = sum m) to 1e-12.
"""

import numpy as np
import pytest

from tests.conftest import check, golden
from tests.test_oracle_golden import _dep_grids

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gg():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from blackhole_nebula_simulator_b200 import gasgrid

    return gasgrid


def _np(t):
    return t.detach().cpu().numpy()


def _check_grid(name, g, prefix, res):
    scale = np.abs(g[f"{prefix}_mass"]).max()
    check(f"{name} mass", g[f"{prefix}_mass"] / scale, _np(res.mass) / scale, atol=1e-12)
    check(f"{name} outside", float(g[f"{prefix}_outside"]), res.outside, rtol=1e-12,
          atol=1e-15 * scale)  # fmt: skip
    check(f"{name} trilinear count", int(g[f"{prefix}_n_tri"]), res.n_trilinear)
    for f in ("rho", "t_mass", "t_em", "vel"):
        a = g[f"{prefix}_{f}"].astype(np.float64)
        check(f"{name} {f}", a, _np(getattr(res, f)).astype(np.float64),
              atol=1e-6 * float(np.abs(a).max()))  # fmt: skip


@pytest.mark.parametrize("kernel", ["wendland_c4", "cubic"])
def test_log_deposition_matches_reference(gg, kernel):
    g = golden("deposit.npz")
    lg, _, _ = _dep_grids(g)
    res = gg.deposit_log(g["x"], g["h"], g["m"], g["t"], g["v"], lg, kernel)
    _check_grid(f"log {kernel}", g, f"log_{kernel}", res)
    check("log ledger: grid + outside = sum m", g["m"].sum(),
          float(res.mass.sum()) + res.outside, rtol=1e-12)  # fmt: skip


@pytest.mark.parametrize("kernel", ["wendland_c4", "cubic"])
def test_box_deposition_matches_reference(gg, kernel):
    g = golden("deposit.npz")
    _, bx, _ = _dep_grids(g)
    res = gg.deposit_box(g["xb"], g["hb"], g["m"], g["t"], g["v"], bx, kernel)
    _check_grid(f"box {kernel}", g, f"box_{kernel}", res)
    check("box ledger: grid + outside = sum m", g["m"].sum(),
          float(res.mass.sum()) + res.outside, rtol=1e-12)  # fmt: skip


def test_split_deposition_matches_reference(gg):
    g = golden("deposit.npz")
    _, _, sg = _dep_grids(g)
    check("wide particles", g["split_wide"], _np(gg.wide_particles(g["xs"], g["hs"], sg)))
    res = gg.deposit_log_split(g["xs"], g["hs"], g["ms"], g["ts"], g["vs"], sg)
    check("wide count", int(g["split_n_wide"]), res.extra["n_wide"])
    _check_grid("split", g, "split", res)
    check("split ledger", g["ms"].sum(), float(res.mass.sum()) + res.outside, rtol=1e-12)


def test_uniform_fields_preserved(gg):
    """Constant T and v give exactly that T, T_em and v in every filled cell."""
    g = golden("deposit.npz")
    lg, _, _ = _dep_grids(g)
    t = np.full(len(g["h"]), 2.5e4)
    v = np.tile([0.01, -0.02, 0.03], (len(g["h"]), 1))
    res = gg.deposit_log(g["x"], g["h"], g["m"], t, v, lg)
    filled = _np(res.mass) > 0
    check("uniform T", 2.5e4, _np(res.t_mass)[filled], rtol=1e-6)
    check("uniform T_em", 2.5e4, _np(res.t_em)[filled], rtol=1e-6)
    check("uniform vx", 0.01, _np(res.vel)[filled][:, 0], rtol=1e-6)


def test_empty_and_bad_inputs(gg):
    g = golden("deposit.npz")
    lg, bx, _ = _dep_grids(g)
    res = gg.deposit_log(np.zeros((0, 3)), np.zeros(0), np.zeros(0), np.zeros(0),
                         np.zeros((0, 3)), lg)  # fmt: skip
    check("empty: no mass", 0.0, float(res.mass.abs().sum()))
    check("empty: nothing outside", 0.0, res.outside)
    with pytest.raises(ValueError, match="kernel"):
        gg.deposit_box(g["xb"], g["hb"], g["m"], g["t"], g["v"], bx, "quintic")
    with pytest.raises(ValueError, match="divisible"):
        gg.coarse_log_grid(gg.LogSphericalGrid(nr=63, nth=32, nph=64), (2, 4, 4))


def test_large_inputs_in_spatial_order_match_the_oracle(gg):
    """70,000 particles: above the size from which the device deals particles to threads in the
    spatial order of their cells; against the CPU oracle (the reference's order)."""
    from oracle import deposit as odep

    rng = np.random.default_rng(21)
    n = 70_000
    lg = gg.LogSphericalGrid(r_min=2.0, r_max=200.0, nr=24, nth=12, nph=24)
    r = np.exp(rng.uniform(np.log(3.0), np.log(220.0), n))
    d = rng.normal(size=(n, 3))
    x = r[:, None] * d / np.linalg.norm(d, axis=1, keepdims=True)
    h = r * lg.dlnr * np.exp(rng.uniform(np.log(0.2), np.log(3.0), n))
    m = rng.uniform(0.5, 2.0, n)
    t = np.exp(rng.uniform(np.log(1e4), np.log(1e7), n))
    v = rng.normal(0.0, 0.05, (n, 3))
    ref = odep.deposit_log(x, h, m, t, v, lg)
    res = gg.deposit_log(x, h, m, t, v, lg)
    scale = np.abs(ref["mass"]).max()
    check("log mass", ref["mass"] / scale, _np(res.mass) / scale, atol=1e-12)
    check("log outside", ref["outside"], res.outside, rtol=1e-12)
    check("log trilinear count", ref["n_trilinear"], res.n_trilinear)
    bx = gg.CartesianBox(centre=(0.0, 0.0, 0.0), size=300.0, n=32)
    hb = bx.dx * np.exp(rng.uniform(np.log(0.2), np.log(2.0), n))
    ref = odep.deposit_box(x, hb, m, t, v, bx)
    res = gg.deposit_box(x, hb, m, t, v, bx)
    scale = np.abs(ref["mass"]).max()
    check("box mass", ref["mass"] / scale, _np(res.mass) / scale, atol=1e-12)
    check("box outside", ref["outside"], res.outside, rtol=1e-12)
    check("box trilinear count", ref["n_trilinear"], res.n_trilinear)
