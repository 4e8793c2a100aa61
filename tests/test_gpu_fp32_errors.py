"""Error of the FP32 pair arithmetic against the FP64 path, per quantity (max and RMS).

Both forms start from the same seeded initial conditions and take the same number of block
steps; the FP64 path rounds like the reference (its operators match the reference's outputs at
1e-12 in the parity tests), so it is the FP64 oracle here.  Stated tolerances (relative, after
the steps below): h and rho 1e-5; positions 1e-9 of |x|; momenta 1e-6 of |p|; u 1e-4;
accelerations and du/dt 1e-4 of their largest magnitude.  The table is printed with -s.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"h": 1e-5, "rho": 1e-5, "x": 1e-9, "p": 1e-6, "u": 1e-4, "a_hydro": 1e-4, "dudt": 1e-4}


def _run(ic, bc, steps):
    from blackhole_nebula_simulator_b200 import blocks

    st = blocks.initialise(ic.x, ic.v, ic.u, ic.mass, ic.h, bc, t_stop=bc.dt_max * 2.0**20)
    for _ in range(steps):
        blocks.advance(st, bc)
    return st


def _errors(a, b):
    out = {}
    for f in TOL:
        x, y = getattr(a, f).cpu().numpy(), getattr(b, f).cpu().numpy()
        if x.ndim == 2:
            d = np.linalg.norm(y - x, axis=1)
            s = np.linalg.norm(x, axis=1) if f in ("x", "p") else np.full(len(x), np.linalg.norm(x, axis=1).max())
        elif f == "dudt":
            d, s = np.abs(y - x), np.full(len(x), np.abs(x).max())
        else:
            d, s = np.abs(y - x), np.abs(x)
        r = d / np.where(s > 0, s, 1.0)
        out[f] = (float(r.max()), float(np.sqrt(np.mean(r * r))))
    return out


@pytest.mark.parametrize("name,n,steps", [("cloud", 4096, 6), ("torus", 20000, 6)])
def test_fp32_error_table(name, n, steps):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import dataclasses

    import bench

    ic, bc64 = bench.workload(name, n, "fp64")
    _, bc32 = bench.workload(name, n, "fp32")
    if name == "cloud":  # stir the cloud so the pair terms are not all zero
        rng = np.random.default_rng(5)
        ic.v = ic.v + 0.01 * np.linalg.norm(ic.v[0]) * rng.normal(size=ic.v.shape)
    a = _run(ic, bc64, steps)
    b = _run(ic, bc32, steps)
    err = _errors(a, b)
    print(f"\nFP32 vs FP64, {name} {n} particles, {steps} block steps:")
    for f, (mx, rms) in err.items():
        print(f"  {f:8s} max {mx:.3e}  rms {rms:.3e}  (tolerance {TOL[f]:.0e})")
    for f, (mx, _) in err.items():
        assert mx <= TOL[f], f"{f}: max relative error {mx:.3e} above {TOL[f]:.0e}"
