"""The CUDA path against the oracle at the sizes of the benchmark configurations.

* 262,144-particle cloud (the second configuration): the whole neighbour lists and the tightened
  lists equal the oracle's CSR exactly; FP64 density and forces on the same lists match the
  oracle at 1e-12; after 100+ block steps over 8 levels, the FP32 pair arithmetic against the
  FP64 form per quantity (max and RMS, the stated tolerances of the FP32 form); the energy ledger
  over 2,000+ system steps (relative drift <= 1e-4, normalised by sum m |H| as the reference's
  tests/sim/test_coupled.py:54 does).
* 1,048,576-particle streams and 4,194,304-particle torus after the benchmark's warm-up steps:
  4,096 sampled rows whose lists equal an exact gather on the same positions (every candidate
  from a k-d tree, the reference's FP64 test r^2 < (2 h)^2 without fused multiply-add), whose
  FP64 density and forces (with disc viscosity on the torus) on those lists match the oracle at
  1e-12, and the FP32 form's state against the FP64 form's after the same steps.

The reference's exact-list contract is tests/sim/test_neighbours.py:102-130; density and forces
follow sim/sph.py:300-326 and 655-690.  Tables print with -s.
"""

import numpy as np
import pytest

from tests.conftest import check

pytestmark = pytest.mark.gpu

# stated tolerances of the FP32 form against the FP64 form (relative; vectors by length, a and
# du/dt to their largest magnitude), the same as tests/test_gpu_fp32_errors.py
TOL = {"h": 1e-5, "rho": 1e-5, "x": 1e-9, "p": 1e-6, "u": 1e-4, "a_hydro": 1e-4, "dudt": 1e-4}
SAMPLE = 4096


@pytest.fixture(scope="module")
def mods():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import bench
    from blackhole_nebula_simulator_b200 import blocks, ops
    from oracle import native

    return ops, blocks, native, bench


def _np(t):
    return t.detach().cpu().numpy()


def _errors(a, b):
    """Per quantity (max, rms) of the FP32 state b against the FP64 state a."""
    out = {}
    for f in TOL:
        x, y = _np(getattr(a, f)), _np(getattr(b, f))
        if x.ndim == 2:
            d = np.linalg.norm(y - x, axis=1)
            s = (np.linalg.norm(x, axis=1) if f in ("x", "p")
                 else np.full(len(x), np.linalg.norm(x, axis=1).max()))  # fmt: skip
        elif f == "dudt":
            d, s = np.abs(y - x), np.full(len(x), np.abs(x).max())
        else:
            d, s = np.abs(y - x), np.abs(x)
        r = d / np.where(s > 0, s, 1.0)
        out[f] = (float(r.max()), float(np.sqrt(np.mean(r * r))))
    return out


def _print_table(title, err):
    print(f"\n{title}")
    for f, (mx, rms) in err.items():
        print(f"  {f:8s} max {mx:.3e}  rms {rms:.3e}  (tolerance {TOL[f]:.0e})")


def _cloud(bench):
    ic, _ = bench.workload("cloud", 262_144, "fp64")
    rng = np.random.default_rng(7)
    # stirred, so the viscosity and the pair forces are not all zero
    ic.v = ic.v + 0.01 * np.linalg.norm(ic.v[0]) * rng.normal(size=ic.v.shape)
    hs = 1.4 * ic.h * rng.uniform(0.9, 1.1, len(ic.h))
    return ic, hs


def test_cloud_262k_lists_bit_exact(mods):
    ops, _, native, bench = mods
    ic, hs = _cloud(bench)
    ref = native.find_neighbours(ic.x, hs)
    got = ops.find_neighbours(ic.x, hs)
    check("262k offsets", ref.offset, _np(got.offset))
    check("262k indices", ref.index, _np(got.index))
    h = hs / 1.4
    rt = native.tighten(ref, ic.x, h)
    gt = ops.tighten(got, ic.x, h)
    check("262k tightened offsets", rt.offset, _np(gt.offset))
    check("262k tightened indices", rt.index, _np(gt.index))
    print(f"\n262k cloud: {ref.offset[-1]:,} list entries, {rt.offset[-1]:,} tightened")


def test_cloud_262k_density_and_forces_fp64(mods):
    from blackhole_nebula_simulator_b200.config import C_NORM, ShockCapturing

    ops, _, native, bench = mods
    ic, hs = _cloud(bench)
    ref = native.find_neighbours(ic.x, hs)
    h0 = hs / 1.4
    oh, orho, oom, oit, ofl = native.density(ic.x, ic.mass, h0, ref, hs, 0, C_NORM[0], 1.2,
                                             tol=1e-4, h_max=200.0)  # fmt: skip
    g = ops.density_numba(ic.x, ic.mass, h0, ref, hs, kernel_name="cubic", eta=1.2, tol=1e-4,
                          h_max=200.0)  # fmt: skip
    check("262k h", oh, _np(g.h), rtol=1e-12)
    check("262k rho", orho, _np(g.rho), rtol=1e-12)
    check("262k omega", oom, _np(g.omega), rtol=1e-12)
    check("262k flags", ofl, _np(g.flags))
    check("262k iterations", oit, _np(g.iterations))
    gamma = 5.0 / 3.0
    P = (gamma - 1.0) * orho * ic.u
    cs = np.sqrt(gamma * P / orho)
    alpha = np.ones(len(oh))
    tight = native.tighten(ref, ic.x, oh)
    sc = ShockCapturing(alpha_u=0.05, conductivity_signal=1)
    oa, odu, ovs, ovh, och = native.forces(ic.x, ic.v, ic.mass, oh, orho, oom, P, tight, 0,
                                           C_NORM[0], u=ic.u, c_s=cs, alpha=alpha, beta=2.0,
                                           alpha_u=0.05, cond_signal=1)  # fmt: skip
    f = ops.forces_numba(ic.x, ic.v, ic.mass, oh, orho, oom, P, tight, kernel_name="cubic",
                         u=ic.u, c_s=cs, alpha=alpha, shock=sc)  # fmt: skip
    amax = float(np.linalg.norm(oa, axis=1).max())
    check("262k acc", oa, _np(f.acc), rtol=1e-12, atol=1e-12 * amax, per_vector=True)
    dmax = float(np.abs(odu).max())
    check("262k dudt", odu, _np(f.dudt), rtol=1e-12, atol=1e-12 * dmax)
    check("262k vsig", ovs, _np(f.vsig_max), rtol=1e-13)
    check("262k viscous heating", ovh, _np(f.dudt_visc), rtol=1e-12, atol=1e-12 * dmax)
    check("262k conductive heating", och, _np(f.dudt_cond), rtol=1e-12, atol=1e-12 * dmax)
    print(f"\n262k cloud: density iterations mean {oit.mean():.2f}, max {oit.max()}; "
          f"{tight.offset[-1]:,} tightened entries")  # fmt: skip


def _shells(ic, nlev=8):
    """Level offsets 0..nlev-1 in equal-volume shells about the cloud's centre: a uniform cloud's
    criteria put every particle on one level, so the offsets (the reference's own way of forcing
    levels in its block tests, sim/blocks.py:455-499 level_offset) spread it over nlev levels."""
    r = np.linalg.norm(ic.x - ic.x.mean(axis=0), axis=1)
    return np.minimum((nlev * (r / r.max()) ** 3).astype(np.int64), nlev - 1)


def _run(blocks, ic, bc, steps, levels=None, level_offset=None):
    st = blocks.initialise(ic.x, ic.v, ic.u, ic.mass, ic.h, bc, t_stop=bc.dt_max * 2.0**20,
                           level_offset=level_offset)  # fmt: skip
    for _ in range(steps):
        blocks.advance(st, bc)
        if levels is not None:
            levels.update(np.unique(_np(st.level)).tolist())
    return st


def test_cloud_262k_fp32_error_table_block_steps(mods):
    """120 block steps over 8 levels in both forms from the same stirred cloud."""
    _, blocks, _, bench = mods
    ic, _ = _cloud(bench)
    _, bc64 = bench.workload("cloud", 262_144, "fp64")
    _, bc32 = bench.workload("cloud", 262_144, "fp32")
    lv64, lv32 = set(), set()
    off = _shells(ic)
    a = _run(blocks, ic, bc64, 120, lv64, off)
    b = _run(blocks, ic, bc32, 120, lv32, off)
    err = _errors(a, b)
    _print_table(f"FP32 vs FP64, cloud 262,144 particles, 120 block steps, levels {sorted(lv64)}",
                 err)  # fmt: skip
    check("levels used (FP64 form)", True, len(lv64) >= 8)
    check("same levels at the end", _np(a.level), _np(b.level))
    for f, (mx, _) in err.items():
        assert mx <= TOL[f], f"{f}: max relative error {mx:.3e} above {TOL[f]:.0e}"


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_cloud_262k_energy_drift_2000_steps(mods, precision):
    """The energy ledger (sim/blocks.py:742-758) over 2,000 system steps and on to the next full
    synchronisation; relative drift normalised by sum m |H| at the start."""
    _, blocks, _, bench = mods
    ic, _ = _cloud(bench)
    _, bc = bench.workload("cloud", 262_144, precision)
    st = blocks.initialise(ic.x, ic.v, ic.u, ic.mass, ic.h, bc, t_stop=bc.dt_max * 2.0**20,
                           level_offset=_shells(ic))  # fmt: skip
    led0 = blocks.ledger(st, bc)
    levels = set()
    for _ in range(2000):
        blocks.advance(st, bc)
        levels.update(np.unique(_np(st.level)).tolist())
    if not st.synced():
        blocks.run(st, bc, st.t0 + int(st.n_end.max()) * st.tick)
    led = blocks.ledger(st, bc)
    drift = (led["energy"] - led0["energy"]) / led0["abs_h"]
    dl = float(np.linalg.norm(np.asarray(led["angmom"]) - np.asarray(led0["angmom"])) /
               np.linalg.norm(np.asarray(led0["angmom"])))  # fmt: skip
    print(f"\n{precision} cloud 262,144: {len(st.active_counts)} system steps to t = {st.t:.1f}, "
          f"levels {sorted(levels)}, {st.particle_steps:,} particle-steps; energy drift "
          f"{drift:.3e}, |dL|/|L| {dl:.3e}")  # fmt: skip
    check("system steps", True, len(st.active_counts) >= 2000)
    check("levels used", True, len(levels) >= 8)
    check("relative energy drift", 0.0, drift, atol=1e-4)


def _exact_rows(x, hs, rows):
    """Exact lists of ``rows``: every particle within 2 max(h) from a k-d tree, then the
    reference's FP64 test (dx = x_j - x_i, ((dx dx + dy dy) + dz dz) < (2 h)^2 for either h)."""
    from scipy.spatial import cKDTree

    tree = cKDTree(x)
    reach = 2.0 * float(hs.max()) * (1.0 + 1e-6)
    cands = tree.query_ball_point(x[rows], reach, workers=-1)
    out = []
    for i, c in zip(rows, cands):
        c = np.asarray(c, dtype=np.int64)
        d = x[c] - x[i]
        d2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
        ri, rj = 2.0 * hs[i], 2.0 * hs[c]
        out.append(np.sort(c[(d2 < ri * ri) | (d2 < rj * rj)]))
    return out


def _sub_lists(n, rows, per_row):
    """CSR over n particles holding only the given rows' lists."""
    from oracle.native import Neighbours

    counts = np.zeros(n, np.int64)
    counts[rows] = [len(r) for r in per_row]
    off = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    idx = np.empty(int(off[-1]), np.int64)
    for i, r in zip(rows, per_row):
        idx[off[i] : off[i + 1]] = r
    return Neighbours(off, idx, None)


def _device_rows(lists, rows):
    """The rows' entries of device lists, gathered on the device."""
    import torch

    off = lists.offset
    r = torch.as_tensor(rows, device=off.device)
    a, b = off[r], off[r + 1]
    cnt = b - a
    base = torch.repeat_interleave(a - torch.cumsum(cnt, 0) + cnt, cnt)
    pos = base + torch.arange(int(cnt.sum()), device=off.device)
    flat = _np(lists.index[pos])
    cuts = np.cumsum(_np(cnt))[:-1]
    return np.split(flat, cuts)


@pytest.mark.parametrize("name", ["streams", "torus"])
def test_sampled_rows_at_scale(mods, name):
    from blackhole_nebula_simulator_b200.config import C_NORM, ShockCapturing

    ops, blocks, native, bench = mods
    warmup = 3
    ic, bc64 = bench.workload(name, None, "fp64")
    _, bc32 = bench.workload(name, None, "fp32")
    a = _run(blocks, ic, bc64, warmup)
    n = len(ic.x)
    x, h, u = _np(a.x), _np(a.h), _np(a.u)
    hs = 1.4 * h
    rng = np.random.default_rng(11)
    rows = np.sort(rng.choice(n, SAMPLE, replace=False))
    lists = ops.find_neighbours(a.x, hs)
    got = _device_rows(lists, rows)
    want = _exact_rows(x, hs, rows)
    for k, (g, w) in enumerate(zip(got, want)):
        if not np.array_equal(g, w):
            raise AssertionError(f"{name}: row {rows[k]} differs ({len(g)} vs {len(w)} entries)")
    sub = _sub_lists(n, rows, want)
    # FP64 density of the sampled rows on their lists
    mass = _np(a.mass)
    oh, orho, oom, oit, ofl = native.density(x, mass, h, sub, hs, 0, C_NORM[0], 1.2, tol=1e-4,
                                             h_max=200.0, rows=rows)  # fmt: skip
    g = ops.density_numba(x, mass, h, sub, hs, kernel_name="cubic", eta=1.2, tol=1e-4,
                          h_max=200.0, rows=rows)  # fmt: skip
    check(f"{name} h", oh, _np(g.h), rtol=1e-12)
    check(f"{name} rho", orho, _np(g.rho), rtol=1e-12)
    check(f"{name} omega", oom, _np(g.omega), rtol=1e-12)
    check(f"{name} flags", ofl, _np(g.flags))
    # FP64 forces of the sampled rows on their tightened lists (state of the FP64 run)
    rho, om, alpha = _np(a.rho), _np(a.omega), _np(a.alpha)
    v = _np(ops.gn_v_from_p(a.x, a.p))
    gamma = 5.0 / 3.0
    P = (gamma - 1.0) * rho * u
    cs = np.sqrt(gamma * P / rho)
    tight = native.tighten(sub, x, h, rows=rows)
    sc = ShockCapturing(alpha_u=0.05, conductivity_signal=1)
    oa, odu, ovs, _, _ = native.forces(x, v, mass, h, rho, om, P, tight, 0, C_NORM[0], u=u,
                                       c_s=cs, alpha=alpha, beta=2.0, alpha_u=0.05,
                                       cond_signal=1, rows=rows)  # fmt: skip
    f = ops.forces_numba(x, v, mass, h, rho, om, P, tight, kernel_name="cubic", u=u, c_s=cs,
                         alpha=alpha, shock=sc, rows=rows)  # fmt: skip
    amax = float(np.linalg.norm(oa, axis=1).max())
    check(f"{name} acc", oa, _np(f.acc), rtol=1e-12, atol=1e-12 * amax, per_vector=True)
    dmax = float(np.abs(odu).max())
    check(f"{name} dudt", odu, _np(f.dudt), rtol=1e-12, atol=1e-12 * dmax)
    check(f"{name} vsig", ovs, _np(f.vsig_max), rtol=1e-13)
    if name == "torus":
        alpha_av = bc64.coupled.hydro.disc_alpha_av
        da, ddu = native.disc_forces(x, v, mass, h, rho, om, cs, alpha_av, tight, 0, C_NORM[0],
                                     rows=rows)  # fmt: skip
        ga, gdu = ops.disc_forces_numba(x, v, mass, h, rho, om, cs, alpha_av, tight,
                                        kernel_name="cubic", rows=rows)  # fmt: skip
        dam = float(np.linalg.norm(da, axis=1).max())
        check("torus disc acc", da, _np(ga), rtol=1e-12, atol=1e-12 * dam, per_vector=True)
        check("torus disc dudt", ddu, _np(gdu), rtol=1e-12, atol=1e-12 * float(np.abs(ddu).max()))
    # the FP32 form after the same steps (exact cooling in both forms)
    b = _run(blocks, ic, bc32, warmup)
    err = _errors(a, b)
    _print_table(f"FP32 vs FP64, {name} {n:,} particles, {warmup} block steps; sampled rows "
                 f"{SAMPLE}: lists exact, density and forces at 1e-12", err)  # fmt: skip
    for fld, (mx, _) in err.items():
        assert mx <= TOL[fld], f"{name} {fld}: max relative error {mx:.3e} above {TOL[fld]:.0e}"
