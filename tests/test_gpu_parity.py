"""CUDA path against the reference's outputs (golden fixtures) and the CPU oracle.

Tolerances: neighbour lists, cells, levels and tick counters exactly; FP64 single-call kernels
at rtol 1e-12 (the reference's own Numba-vs-readable tolerance); the GN flow bit for bit; whole
FP64 steps at the tolerances of the oracle's own pinning (sums run in Hilbert-curve order on the GPU,
so they differ from the reference's list order by rounding only).
"""

import numpy as np
import pytest

from tests.conftest import check, golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from blackhole_nebula_simulator_b200 import blocks, cooling, coupled, ops

    return ops, coupled, blocks, cooling


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("case", ["open_uneven", "isolated_large_h", "clump_and_halo"])
def test_lists_bit_exact(nb, case):
    ops = nb[0]
    g = golden("lists.npz")
    lists = ops.find_neighbours(g[f"{case}_pos"], g[f"{case}_h"])
    check(f"{case} offsets", g[f"{case}_offset"], _np(lists.offset))
    check(f"{case} indices", g[f"{case}_index"].astype(np.int64), _np(lists.index))


def test_periodic_box_refused(nb):
    ops = nb[0]
    g = golden("lists.npz")
    with pytest.raises(NotImplementedError):
        ops.find_neighbours(g["periodic_cube_pos"], g["periodic_cube_h"], box=2.0)


def test_cloud_lists_and_tighten_bit_exact(nb):
    ops = nb[0]
    g = golden("cloud_lists.npz")
    lists = ops.find_neighbours(g["pos"], g["h_search"])
    check("cloud offsets", g["offset"], _np(lists.offset))
    check("cloud indices", g["index"].astype(np.int64), _np(lists.index))
    t = ops.tighten(lists, g["pos"], g["h"])
    check("tight offsets", g["tight_offset"], _np(t.offset))
    check("tight indices", g["tight_index"].astype(np.int64), _np(t.index))


def test_cloud_cells_bit_exact(nb):
    """The reference's cell assignment (sim/neighbours.py:106-126, 250-265): grid geometry, cell
    starts and the counting-sort order of the 4,096 cloud exactly as the reference wrote them."""
    ops = nb[0]
    g = golden("cloud_lists.npz")
    lo, inv, nc = ops.cell_geometry(g["pos"], g["h_search"])
    check("grid lo", g["lo"], lo)
    check("grid inverse cell", g["inv_cell"], inv)
    check("grid dims", g["ncell"], nc)
    start, order = ops.build_grid(g["pos"], g["lo"], g["inv_cell"], g["ncell"])
    check("cell starts", g["grid_start"], _np(start))
    check("cell order", g["grid_order"].astype(np.int64), _np(order))


def test_cells_at_262k_bit_exact(nb):
    """The same at the 262,144-particle cloud (the uniform cloud of the FP32 tests) against the
    oracle's cell of every particle: geometry, starts and order exactly."""
    from blackhole_nebula_simulator_b200 import ics
    from oracle import native

    ops = nb[0]
    ic = ics.cloud(262_144, seed=1)
    # varied search radii, so the median of an even count is the mean of two different values
    hs = 1.4 * ic.h * np.random.default_rng(5).uniform(0.8, 1.25, len(ic.h))
    cell, lo, inv, nc = native.grid_cells(ic.x, hs)
    glo, ginv, gnc = ops.cell_geometry(ic.x, hs)
    check("grid lo", lo, glo)
    check("grid dims", nc, gnc)
    check("grid inverse cell", inv, ginv)
    start, order = ops.build_grid(ic.x, lo, inv, nc)
    ref_order = np.argsort(cell, kind="stable")
    check("cell order", ref_order, _np(order))
    check("cell starts", np.searchsorted(cell[ref_order], np.arange(int(np.prod(nc)) + 1)),
          _np(start))  # fmt: skip


def test_long_and_short_rows_bit_exact(nb):
    """Rows far longer than the one-pass build's slot width (a few particles with 8x the search
    radius) beside ordinary rows, twice in a row so the second build runs with the width the first
    one chose: exact equality with the oracle's lists."""
    from oracle import native

    ops = nb[0]
    rng = np.random.default_rng(21)
    pos = rng.uniform(0.0, 1.0, (40000, 3))
    h = np.full(len(pos), 0.02) * rng.uniform(0.8, 1.25, len(pos))
    h[rng.choice(len(pos), 40, replace=False)] *= 8.0
    ref = native.find_neighbours(pos, h)
    assert np.diff(ref.offset).max() > 1024
    for attempt in range(2):
        lists = ops.find_neighbours(pos, h)
        check(f"offsets ({attempt})", ref.offset, _np(lists.offset))
        check(f"indices ({attempt})", ref.index.astype(np.int64), _np(lists.index))


def test_single_particle_lists_itself(nb):
    ops = nb[0]
    lists = ops.find_neighbours(np.array([[0.3, 0.2, 0.1]]), np.array([0.1]))
    check("single particle", [0], _np(lists.of(0)).tolist())


def test_density_matches_reference(nb):
    ops = nb[0]
    g = golden("density.npz")
    lists = ops.Neighbours(g["offset"], g["index"].astype(np.int64))
    r = ops.density_numba(g["pos"], g["mass"], g["h_first"], lists, g["h_search"], tol=1e-12,
                          h_max=0.5)  # fmt: skip
    check("h", g["h"], _np(r.h), rtol=1e-12)
    check("rho", g["rho"], _np(r.rho), rtol=1e-12)
    check("omega", g["omega"], _np(r.omega), rtol=1e-12)
    check("flags", g["flags"], _np(r.flags))
    r2 = ops.density_numba(g["pos"], g["mass"], g["h_first"], lists, g["h_search"], tol=1e-12,
                           h_max=0.5, rows=g["rows"])  # fmt: skip
    check("rows h", g["rows_h"], _np(r2.h), rtol=1e-12)
    r3 = ops.density_numba(g["pos"], g["mass"], g["h_first"], lists, g["h_search"],
                           kernel_name="cubic", eta=1.2, h_max=0.5)  # fmt: skip
    check("cubic h", g["cubic_h"], _np(r3.h), rtol=1e-12)
    check("cubic flags", g["cubic_flags"], _np(r3.flags))
    check("cubic iterations", g["cubic_iters"], _np(r3.iterations))


@pytest.mark.parametrize("sig", [0, 1])
def test_forces_match_reference(nb, sig):
    from blackhole_nebula_simulator_b200.config import ShockCapturing

    ops = nb[0]
    g = golden("forces.npz")
    lists = ops.Neighbours(g["offset"], g["index"].astype(np.int64))
    f = ops.forces_numba(g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"],
                         g["pressure"], lists, u=g["u"], c_s=g["c_s"], alpha=g["alpha"],
                         shock=ShockCapturing(alpha_u=0.5, conductivity_signal=sig))  # fmt: skip
    check("acc", g[f"cond{sig}_acc"], _np(f.acc), rtol=1e-12, per_vector=True)
    scale = np.abs(g[f"cond{sig}_dudt"]).max()
    check("dudt", g[f"cond{sig}_dudt"] / scale, _np(f.dudt) / scale, atol=1e-12)
    check("vsig", g[f"cond{sig}_vsig"], _np(f.vsig_max), rtol=1e-14)
    check("visc heat", g[f"cond{sig}_visc"] / scale, _np(f.dudt_visc) / scale, atol=1e-12)
    check("cond heat", g[f"cond{sig}_cond"] / scale, _np(f.dudt_cond) / scale, atol=1e-12)


def test_forces_rows_disc_cubic_match_reference(nb):
    from blackhole_nebula_simulator_b200.config import ShockCapturing

    ops = nb[0]
    g = golden("forces.npz")
    lists = ops.Neighbours(g["offset"], g["index"].astype(np.int64))
    base = (g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"], g["pressure"], lists)
    f = ops.forces_numba(*base)
    check("plain acc", g["plain_acc"], _np(f.acc), rtol=1e-12, per_vector=True)
    f = ops.forces_numba(*base, u=g["u"], c_s=g["c_s"], alpha=g["alpha"],
                         shock=ShockCapturing(alpha_u=0.5, conductivity_signal=1), rows=g["rows"])
    check("rows acc", g["rows_acc"], _np(f.acc), rtol=1e-12, per_vector=True)
    check("rows vsig", g["rows_vsig"], _np(f.vsig_max), rtol=1e-14)
    a, u = ops.disc_forces_numba(g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"],
                                 g["c_s"], 0.5, lists)  # fmt: skip
    check("disc acc", g["disc_acc"], _np(a), rtol=1e-12, per_vector=True)
    check("disc dudt", g["disc_dudt"], _np(u), rtol=1e-11, atol=1e-14 * np.abs(g["disc_dudt"]).max())
    f = ops.forces_numba(*base, kernel_name="cubic", u=g["u"], c_s=g["c_s"], alpha=g["alpha"])
    check("cubic acc", g["cubic_acc"], _np(f.acc), rtol=1e-12, per_vector=True)


def test_glf_bit_exact(nb):
    ops = nb[0]
    g = golden("glf.npz")
    x1, p1, it = ops.glf_step_many(g["x"], g["p"], g["dt"])
    check("x1 bitwise", g["x1"], _np(x1))
    check("p1 bitwise", g["p1"], _np(p1))
    check("iterations", g["iters"], _np(it))
    check("v from p", g["v_from_p"], _np(ops.gn_v_from_p(g["x"], g["p"])), rtol=1e-15, per_vector=True)
    check("p from v", g["p"], _np(ops.gn_p_from_v(g["x"], g["v"])), rtol=1e-15, per_vector=True)


def test_glf_failures_raise(nb):
    ops = nb[0]
    from oracle import steps as osteps

    x = np.array([[6.0, 0.0, 0.0]])
    p = osteps.gn_p_from_v(x, np.array([[0.0, 0.4, 0.0]]))
    with pytest.raises(ops.GLFConvergenceError, match="did not converge"):
        ops.glf_step_many(x, p, 50.0)
    with pytest.raises(ops.GLFConvergenceError, match="inside r"):
        ops.glf_step_many(np.array([[2.4, 0.0, 0.0]]), p, 0.1)


def test_cooling_laws(nb):
    ops, _, _, cooling = nb
    from oracle import cooling as ocool

    g = golden("cooling.npz")
    # exp() of CUDA and of the host C library may differ by an ulp: a few ulps of tolerance
    check("beta_cool", g["u_new"], _np(ops.beta_cool(g["u"], g["u_floor"], g["dt"], g["t_cool"])),
          rtol=4e-15)  # fmt: skip
    rng = np.random.default_rng(5)
    consts = cooling.brems_constants()
    oc = ocool.brems_constants()
    check("brems constants", np.array(oc), np.array([consts.tfac, consts.b, consts.kappa,
                                                     consts.u_floor, consts.t_floor]), rtol=1e-15)
    u = consts.u_floor * np.exp(rng.uniform(-1.0, np.log(1e6), 4000))
    rho = np.exp(rng.uniform(np.log(1e-12), np.log(1e-3), 4000))
    dt = np.exp(rng.uniform(np.log(1e-4), np.log(50.0), 4000))
    check("brems exact", ocool.brems_cool(u, rho, dt, oc), _np(cooling.brems_cool(u, rho, dt, consts)),
          rtol=1e-12)  # fmt: skip


def _cfg(cooling_beta=float("inf"), precision="fp64"):
    from blackhole_nebula_simulator_b200.config import CoupledConfig, HydroConfig

    hc = HydroConfig(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                     conductivity_signal=1, alpha_u=0.05, h_max=200.0, precision=precision)  # fmt: skip
    return CoupledConfig(hydro=hc, cooling_beta=cooling_beta)


def test_shared_steps_match_reference(nb):
    _, coupled, _, _ = nb
    g = golden("coupled.npz")
    cc = _cfg()
    st = coupled.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], cc)
    check("init h", g["init_h"], _np(st.h), rtol=1e-10)
    check("init rho", g["init_rho"], _np(st.rho), rtol=1e-10)
    check("init acc", g["init_a_hydro"], _np(st.a_hydro), rtol=1e-9, per_vector=True)
    for k in range(3):
        dt = coupled.stable_dt(st, cc)
        check(f"dt {k}", g["dts"][k], dt, rtol=1e-12)
        st = coupled.step(st, cc, dt)
        check(f"step {k + 1} x", g[f"step{k + 1}_x"], _np(st.x), rtol=1e-14, per_vector=True)
        check(f"step {k + 1} p", g[f"step{k + 1}_p"], _np(st.p), rtol=1e-12, per_vector=True)
        check(f"step {k + 1} u", g[f"step{k + 1}_u"], _np(st.u), rtol=1e-10)
        check(f"step {k + 1} h", g[f"step{k + 1}_h"], _np(st.h), rtol=1e-10)
        check(f"step {k + 1} acc", g[f"step{k + 1}_a_hydro"], _np(st.a_hydro), rtol=1e-8,
              per_vector=True)  # fmt: skip
        check(f"step {k + 1} energy", g[f"step{k + 1}_energy"], coupled.ledger(st, cc)["energy"],
              rtol=1e-13)  # fmt: skip
    check("list builds", int(g["builds"]), st.builds)
    check("list reuses", int(g["reuses"]), st.reuses)


def test_block_steps_match_reference(nb):
    from blackhole_nebula_simulator_b200.config import BlockConfig

    _, _, blocks, _ = nb
    g = golden("blocks.npz")
    bc = BlockConfig(coupled=_cfg(cooling_beta=230.0), dt_max=64.0)
    # the fixture's t_stop (1e9) lies beyond the int64 tick range; no step lands on either
    st = blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6,
                           level_offset=g["level_offset"])  # fmt: skip
    check("init levels", g["init_level"], _np(st.level))
    check("init n_end", g["init_n_end"], _np(st.n_end))
    actives = [len(blocks.advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("final tick", int(g["final_n"]), st.n)
    check("final levels", g["final_level"], _np(st.level))
    check("final n_end", g["final_n_end"], _np(st.n_end))
    check("final x", g["final_x"], _np(st.x), rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], _np(st.p), rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], _np(st.u), rtol=1e-9)
    check("final h", g["final_h"], _np(st.h), rtol=1e-9)
    check("final energy", float(g["final_energy"]), blocks.ledger(st, bc)["energy"], rtol=1e-12)
    check("final e_radiated", float(g["final_e_radiated"]), st.e_radiated, rtol=1e-9)
    check("list builds", int(g["builds"]), st.builds)
    check("list reuses", int(g["reuses"]), st.reuses)


def test_block_step_errors_raise_and_leave_the_context_usable(nb):
    """u <= 0 and a particle inside the GN flow's r = 2.5 raise the reference's exceptions from a
    block step (sim/blocks.py:250, sim/integrator.py:50); a clean state steps afterwards."""
    from blackhole_nebula_simulator_b200.config import BlockConfig

    _, _, blocks, _ = nb
    g = golden("blocks.npz")
    bc = BlockConfig(coupled=_cfg(cooling_beta=230.0), dt_max=64.0)

    def fresh():
        return blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6,
                                 level_offset=g["level_offset"])  # fmt: skip

    st = fresh()
    st.u_half[7] = -1.0  # the predictor carries it into u
    with pytest.raises(FloatingPointError):
        blocks.advance(st, bc)
    st = fresh()
    st.x_beg[11] = st.x_beg[11] / st.x_beg[11].norm() * 2.0
    with pytest.raises(nb[0].GLFConvergenceError, match="inside r"):
        blocks.advance(st, bc)
    st = fresh()
    actives = [len(blocks.advance(st, bc)) for _ in range(4)]
    check("active counts after the errors", g["active_counts"][:4], np.array(actives))


def test_fp32_pair_arithmetic_within_stated_tolerance(nb):
    """FP32 pair passes (cell offsets, Kahan sums) against the FP64 path on the 4,096-particle
    cloud stirred by 1% velocity noise: h and rho to 1e-5 relative, accelerations and du/dt to
    1e-3 of their largest magnitude (per vector)."""
    _, coupled, _, _ = nb
    g = golden("coupled.npz")
    rng = np.random.default_rng(11)
    v = g["v0"] + 0.01 * np.linalg.norm(g["v0"][0]) * rng.normal(size=g["v0"].shape)
    a = coupled.initialise(g["x0"], v, g["u0"], g["mass"], g["h0"], _cfg())
    b = coupled.initialise(g["x0"], v, g["u0"], g["mass"], g["h0"], _cfg(precision="fp32"))
    check("fp32 h", _np(a.h), _np(b.h), rtol=1e-5)
    check("fp32 rho", _np(a.rho), _np(b.rho), rtol=1e-5)
    amax = np.linalg.norm(_np(a.a_hydro), axis=1).max()
    check("fp32 acc", _np(a.a_hydro) / amax, _np(b.a_hydro) / amax, atol=1e-3, per_vector=True)
    scale = np.abs(_np(a.dudt)).max()
    check("fp32 dudt", _np(a.dudt) / scale, _np(b.dudt) / scale, atol=1e-3)


def _pericentres(t, x):
    """Pericentre passages refined by parabolas through the three samples around each minimum
    of r (the method of the reference's analysis/orbit_metrics.py:12-30)."""
    r = np.linalg.norm(x, axis=1)
    phi = np.unwrap(np.arctan2(x[:, 1], x[:, 0]))
    idx = np.where((r[1:-1] < r[:-2]) & (r[1:-1] <= r[2:]))[0] + 1
    times, angles = [], []
    for i in idx:
        sl = slice(i - 1, i + 2)
        a, b, _ = np.polyfit(t[sl] - t[i], r[sl], 2)
        tp = t[i] - b / (2.0 * a)
        times.append(tp)
        angles.append(np.polyval(np.polyfit(t[sl] - tp, phi[sl], 2), 0.0))
    return np.array(times), np.array(angles)


def test_gn_orbit_precession_and_conservation(nb):
    """The reference's orbit test (tests/sim/test_integrator.py:95-122, expected values of
    reference/expected-values.md): cloud orbit r_p = 25, r_a = 5,000, eta = 0.00125, 3 radial
    periods; first pericentre 396,223.627 and period 792,447.254 (rtol 1e-5), precession
    24.0398 deg per orbit (atol 0.01 deg), |dH/H| < 1e-4, |dL/L| < 1e-12."""
    ops = nb[0]
    from blackhole_nebula_simulator_b200 import ics
    from oracle import steps as osteps

    x0, v0, p0 = ics.apocentre_state(25.0, 5000.0)
    orb = ops.integrate_orbit(x0, p0, 3 * 792_447.254, eta=0.00125)
    tp, phi = _pericentres(orb.t, orb.x)
    check("pericentres found", 3, len(tp))
    check("first pericentre time", 396_223.627, tp[0], rtol=1e-5)
    check("radial periods", np.full(2, 792_447.254), np.diff(tp), rtol=1e-5)
    check("precession per orbit (deg)", np.full(2, 24.0398), np.degrees(np.diff(phi) - 2 * np.pi),
          atol=0.01)  # fmt: skip
    H = osteps.gn_hamiltonian(orb.x, orb.p)
    L = np.linalg.norm(np.cross(orb.x, orb.p), axis=1)
    check("max |dH/H|", 0.0, np.max(np.abs(H / H[0] - 1)), atol=1e-4)
    check("max |dL/L|", 0.0, np.max(np.abs(L / L[0] - 1)), atol=1e-12)
