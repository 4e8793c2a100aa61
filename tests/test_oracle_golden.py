"""The CPU oracle against the reference's own outputs (golden fixtures): pins the checker.

Lists and cells must match exactly; floating-point kernels to the tolerances the reference's
tests use between its Numba kernels and its readable twins (rtol 1e-12), since the oracle's
operation order follows the reference's.
"""

import numpy as np
import pytest

from oracle import cooling as ocool
from oracle import native, steps
from oracle.sph import C_NORM, KERNEL_IDS, compute_density
from tests.conftest import check, golden


def _nb(off, idx, box=None):
    return native.Neighbours(np.asarray(off, np.int64), np.asarray(idx, np.int64), box)


@pytest.mark.parametrize(
    "case", ["open_uneven", "periodic_cube", "periodic_long_box", "isolated_large_h",
             "clump_and_halo"])  # fmt: skip
def test_lists_match_reference(case):
    g = golden("lists.npz")
    box = g[f"{case}_box"]
    nb = native.find_neighbours(g[f"{case}_pos"], g[f"{case}_h"], box=None if not box.any() else box)
    check(f"{case}: offsets", g[f"{case}_offset"], nb.offset)
    check(f"{case}: indices", g[f"{case}_index"].astype(np.int64), nb.index)


def test_cloud_cells_and_lists_match_reference():
    g = golden("cloud_lists.npz")
    cell, lo, inv, nc = native.grid_cells(g["pos"], g["h_search"])
    check("grid dims", g["ncell"], nc)
    check("grid lo", g["lo"], lo)
    # the reference's counting sort: order lists particles cell by cell, index ascending
    order = np.argsort(cell, kind="stable")
    check("cell order", g["grid_order"].astype(np.int64), order)
    start = np.searchsorted(cell[order], np.arange(int(np.prod(nc)) + 1))
    check("cell starts", g["grid_start"], start)
    nb = native.find_neighbours(g["pos"], g["h_search"])
    check("cloud lists offsets", g["offset"], nb.offset)
    check("cloud lists indices", g["index"].astype(np.int64), nb.index)
    t = native.tighten(nb, g["pos"], g["h"])
    check("tightened offsets", g["tight_offset"], t.offset)
    check("tightened indices", g["tight_index"].astype(np.int64), t.index)


def test_density_matches_reference():
    g = golden("density.npz")
    nb = _nb(g["offset"], g["index"])
    h, rho, om, it, fl = native.density(g["pos"], g["mass"], g["h_first"], nb, g["h_search"], 1,
                                        C_NORM[1], 1.6, tol=1e-12, h_max=0.5)  # fmt: skip
    check("h", g["h"], h, rtol=1e-12)
    check("rho", g["rho"], rho, rtol=1e-12)
    check("omega", g["omega"], om, rtol=1e-12)
    check("flags", g["flags"], fl)
    h2, rho2, *_ = native.density(g["pos"], g["mass"], g["h_first"], nb, g["h_search"], 1,
                                  C_NORM[1], 1.6, tol=1e-12, h_max=0.5, rows=g["rows"])  # fmt: skip
    check("rows h", g["rows_h"], h2, rtol=1e-12)
    h3, rho3, om3, it3, fl3 = native.density(g["pos"], g["mass"], g["h_first"], nb, g["h_search"],
                                             0, C_NORM[0], 1.2, tol=1e-4, h_max=0.5)  # fmt: skip
    check("cubic h", g["cubic_h"], h3, rtol=1e-12)
    check("cubic rho", g["cubic_rho"], rho3, rtol=1e-12)
    check("cubic omega", g["cubic_omega"], om3, rtol=1e-12)
    check("cubic flags", g["cubic_flags"], fl3)
    check("cubic iterations", g["cubic_iters"], it3)


def test_compute_density_matches_reference():
    g = golden("density.npz")
    res = compute_density(g["pos"], g["mass"], np.full(len(g["pos"]), 0.05), h_max=0.5)
    check("compute_density h", g["h_first"], res.h, rtol=1e-12)
    check("compute_density rho", g["rho_first"], res.rho, rtol=1e-12)
    check("compute_density flags", g["flags_first"], res.flags)


@pytest.mark.parametrize("sig", [0, 1])
def test_forces_match_reference(sig):
    g = golden("forces.npz")
    nb = _nb(g["offset"], g["index"])
    args = (g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"], g["pressure"], nb)
    acc, dudt, vsig, vh, ch = native.forces(*args, 1, C_NORM[1], u=g["u"], c_s=g["c_s"],
                                            alpha=g["alpha"], alpha_u=0.5, cond_signal=sig)
    check("acc", g[f"cond{sig}_acc"], acc, rtol=1e-12, per_vector=True)
    scale = np.abs(g[f"cond{sig}_dudt"]).max()
    check("dudt", g[f"cond{sig}_dudt"] / scale, dudt / scale, atol=1e-12)
    check("vsig", g[f"cond{sig}_vsig"], vsig, rtol=1e-14)
    check("visc heat", g[f"cond{sig}_visc"] / scale, vh / scale, atol=1e-12)
    check("cond heat", g[f"cond{sig}_cond"] / scale, ch / scale, atol=1e-12)


def test_forces_plain_rows_disc_cubic_match_reference():
    g = golden("forces.npz")
    nb = _nb(g["offset"], g["index"])
    base = (g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"], g["pressure"], nb)
    acc, dudt, vsig, _, _ = native.forces(*base, 1, C_NORM[1])
    check("plain acc", g["plain_acc"], acc, rtol=1e-12, per_vector=True)
    check("plain dudt", g["plain_dudt"], dudt, rtol=1e-11, atol=1e-14)
    acc, dudt, vsig, _, _ = native.forces(*base, 1, C_NORM[1], u=g["u"], c_s=g["c_s"],
                                          alpha=g["alpha"], alpha_u=0.5, cond_signal=1,
                                          rows=g["rows"])  # fmt: skip
    check("rows acc", g["rows_acc"], acc, rtol=1e-12, per_vector=True)
    check("rows vsig", g["rows_vsig"], vsig, rtol=1e-14)
    a_d, u_d = native.disc_forces(g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"],
                                  g["c_s"], 0.5, nb, 1, C_NORM[1])  # fmt: skip
    check("disc acc", g["disc_acc"], a_d, rtol=1e-12, per_vector=True)
    check("disc dudt", g["disc_dudt"], u_d, rtol=1e-11, atol=1e-14 * np.abs(g["disc_dudt"]).max())
    acc, dudt, vsig, _, _ = native.forces(*base, 0, C_NORM[0], u=g["u"], c_s=g["c_s"],
                                          alpha=g["alpha"])  # fmt: skip
    check("cubic acc", g["cubic_acc"], acc, rtol=1e-12, per_vector=True)


def test_glf_matches_reference():
    g = golden("glf.npz")
    x1, p1, it = native.glf_step_many(g["x"], g["p"], g["dt"])
    check("x1", g["x1"], x1, rtol=1e-15, per_vector=True)
    check("p1", g["p1"], p1, rtol=1e-15, per_vector=True)
    check("iterations", g["iters"], it)
    check("v from p", g["v_from_p"], native.gn_v_from_p(g["x"], g["p"]), rtol=1e-15,
          per_vector=True)  # fmt: skip
    check("p from v", g["p"], steps.gn_p_from_v(g["x"], g["v"]), rtol=1e-15, per_vector=True)
    check("hamiltonian", g["ham"], steps.gn_hamiltonian(g["x"], g["p"]), rtol=1e-13)


def test_glf_failures_flagged():
    x = np.array([[6.0, 0.0, 0.0]])
    p = steps.gn_p_from_v(x, np.array([[0.0, 0.4, 0.0]]))
    with pytest.raises(native.GLFConvergenceError, match="did not converge"):
        native.glf_step_many(x, p, 50.0)
    with pytest.raises(native.GLFConvergenceError, match="inside r"):
        native.glf_step_many(np.array([[2.4, 0.0, 0.0]]), p, 0.1)


def test_beta_cooling_matches_reference():
    g = golden("cooling.npz")
    check("beta_cool", g["u_new"], ocool.beta_cool(g["u"], g["u_floor"], g["dt"], g["t_cool"]),
          rtol=1e-15)  # fmt: skip
    check("cooling time", g["t_cool"], ocool.cooling_time(g["r"], 230.0), rtol=1e-15)


def _cfg():
    from blackhole_nebula_simulator_b200.config import CoupledConfig, HydroConfig

    hc = HydroConfig(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                     conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    return hc, CoupledConfig


def test_shared_steps_match_reference():
    g = golden("coupled.npz")
    hc, CC = _cfg()
    cc = CC(hydro=hc)
    st = steps.coupled_initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], cc)
    for f in ("h", "rho", "dudt"):
        check(f"init {f}", g[f"init_{f}"], getattr(st, f), rtol=1e-10, atol=1e-30)
    check("init acc", g["init_a_hydro"], st.a_hydro, rtol=1e-9, per_vector=True)
    for k in range(3):
        dt = steps.coupled_stable_dt(st, cc)
        check(f"dt {k}", g["dts"][k], dt, rtol=1e-12)
        st = steps.coupled_step(st, cc, dt)
        check(f"step {k + 1} x", g[f"step{k + 1}_x"], st.x, rtol=1e-14, per_vector=True)
        check(f"step {k + 1} p", g[f"step{k + 1}_p"], st.p, rtol=1e-12, per_vector=True)
        check(f"step {k + 1} u", g[f"step{k + 1}_u"], st.u, rtol=1e-10)
        check(f"step {k + 1} h", g[f"step{k + 1}_h"], st.h, rtol=1e-10)
        check(f"step {k + 1} acc", g[f"step{k + 1}_a_hydro"], st.a_hydro, rtol=1e-8,
              per_vector=True)  # fmt: skip
        led = steps.coupled_ledger(st, cc)
        check(f"step {k + 1} energy", g[f"step{k + 1}_energy"], led["energy"], rtol=1e-13)
    check("cache builds", int(g["builds"]), st.neighbour_cache.builds)
    check("cache reuses", int(g["reuses"]), st.neighbour_cache.reuses)


def test_block_steps_match_reference():
    from blackhole_nebula_simulator_b200.config import BlockConfig

    g = golden("blocks.npz")
    hc, CC = _cfg()
    bc = BlockConfig(coupled=CC(hydro=hc, cooling_beta=230.0), dt_max=64.0)
    st = steps.blocks_initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e9,
                                 level_offset=g["level_offset"])  # fmt: skip
    check("init levels", g["init_level"], st.level)
    check("init n_end", g["init_n_end"], st.n_end)
    actives = [len(steps.blocks_advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("final tick", int(g["final_n"]), st.n)
    check("final levels", g["final_level"], st.level)
    check("final n_end", g["final_n_end"], st.n_end)
    check("final x", g["final_x"], st.x, rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], st.p, rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], st.u, rtol=1e-9)
    check("final h", g["final_h"], st.h, rtol=1e-9)
    check("final energy", float(g["final_energy"]), steps.blocks_ledger(st, bc)["energy"],
          rtol=1e-12)  # fmt: skip
    check("final e_radiated", float(g["final_e_radiated"]), st.e_radiated, rtol=1e-9)
    check("cache builds", int(g["builds"]), st.neighbour_cache.builds)
    check("cache reuses", int(g["reuses"]), st.neighbour_cache.reuses)


def test_equations_of_state_match_reference():
    from blackhole_nebula_simulator_b200.config import HydroConfig
    from oracle import eos as oeos

    g = golden("eos.npz")
    gu = HydroConfig().gas_units
    p, cs, t, beta = oeos.gasrad_state(g["rho"], g["u"], gu.density_kg_m3)
    # bit for bit: the C iteration calls the same C-library exp, log and pow as the reference
    check("gasrad T", g["gasrad_t"], t)
    check("gasrad P", g["gasrad_p"], p)
    check("gasrad c_s", g["gasrad_cs"], cs)
    check("gasrad beta", g["gasrad_beta"], beta)
    for eos in ("ideal", "radiation"):
        pe, ce = oeos.eos_state(HydroConfig(eos=eos), g["rho"], g["u"])
        check(f"{eos} P", g[f"{eos}_p"], pe, rtol=1e-15)
        check(f"{eos} c_s", g[f"{eos}_cs"], ce, rtol=1e-15)


def test_eos_range_and_sign_errors():
    from blackhole_nebula_simulator_b200.config import HydroConfig
    from oracle import eos as oeos

    hc = HydroConfig(eos="gasrad")
    rho = np.array([1e-8, 1e-8])
    with pytest.raises(ValueError, match="bracket"):
        oeos.eos_state(hc, rho, np.array([1e-12, 1e-30]))
    with pytest.raises(ValueError, match="bracket"):
        oeos.eos_state(hc, rho, np.array([1e-12, 1e29]))
    with pytest.raises(FloatingPointError):
        oeos.eos_state(hc, rho, np.array([1e-12, 0.0]))


def test_gasrad_block_steps_match_reference():
    from blackhole_nebula_simulator_b200.config import BlockConfig, HydroConfig

    g = golden("gasrad_blocks.npz")
    hc = HydroConfig(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                     conductivity_signal=1, alpha_u=0.05, h_max=200.0, eos="gasrad")  # fmt: skip
    _, CC = _cfg()
    bc = BlockConfig(coupled=CC(hydro=hc), dt_max=64.0)
    st = steps.blocks_initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6)
    check("init levels", g["init_level"], st.level)
    check("init n_end", g["init_n_end"], st.n_end)
    check("init dudt", g["init_dudt"], st.dudt, rtol=1e-9,
          atol=1e-10 * np.abs(g["init_dudt"]).max())  # fmt: skip
    check("init acc", g["init_a_hydro"], st.a_hydro, rtol=1e-9, per_vector=True)
    actives = [len(steps.blocks_advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("final tick", int(g["final_n"]), st.n)
    check("final levels", g["final_level"], st.level)
    check("final n_end", g["final_n_end"], st.n_end)
    check("final x", g["final_x"], st.x, rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], st.p, rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], st.u, rtol=1e-9)
    check("final h", g["final_h"], st.h, rtol=1e-9)
    check("final energy", float(g["final_energy"]), steps.blocks_ledger(st, bc)["energy"],
          rtol=1e-12)  # fmt: skip


def _scaled(name, expected, actual, tol):
    scale = np.abs(expected).max()
    check(name, expected / scale, actual / scale, atol=tol)


def test_gradients_match_reference():
    g = golden("shock.npz")
    nb = _nb(g["offset"], g["index"])
    args = (g["pos"], g["vel"], g["acc_prev"], g["mass"], g["h"], nb)
    div, curl, ddiv = native.gradients(*args, 1, C_NORM[1])
    _scaled("div v", g["div_v"], div, 1e-12)
    _scaled("curl v", g["curl_v"], curl, 1e-12)
    _scaled("d div v / dt", g["ddivv_dt"], ddiv, 1e-12)
    div, curl, ddiv = native.gradients(*args, 0, C_NORM[0], rows=g["rows"])
    _scaled("cubic rows div v", g["cubic_rows_div_v"], div, 1e-12)
    _scaled("cubic rows curl v", g["cubic_rows_curl_v"], curl, 1e-12)
    _scaled("cubic rows d div v / dt", g["cubic_rows_ddivv_dt"], ddiv, 1e-12)


def test_velocity_gradients_match_reference():
    g = golden("shock.npz")
    nb = _nb(g["offset"], g["index"])
    gv = native.velocity_gradients(g["pos"], g["vel"], g["mass"], g["h"], nb, 1, C_NORM[1])
    _scaled("grad v (tight lists)", g["grad_v"], gv, 1e-12)
    full = native.find_neighbours(g["pos"], 1.4 * g["h"])
    gv = native.velocity_gradients(g["pos"], g["vel"], g["mass"], g["h"], full, 1, C_NORM[1],
                                   rows=g["rows"])  # fmt: skip
    _scaled("grad v (untightened lists, rows)", g["full_rows_grad_v"], gv, 1e-12)


@pytest.mark.parametrize("gate", [0, 1, 2])
@pytest.mark.parametrize("close", [True, False])
def test_reconstructed_forces_match_reference(gate, close):
    g = golden("shock.npz")
    nb = _nb(g["offset"], g["index"])
    args = (g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"], g["pressure"], nb)
    acc, dudt, vsig, vh, ch = native.forces(*args, 1, C_NORM[1], u=g["u"], c_s=g["c_s"],
                                            alpha=g["alpha"], alpha_u=0.5, cond_signal=1,
                                            grad_v=g["grad_v"], closeness=close, gate=gate)
    key = f"recon_g{gate}_c{int(close)}"
    check("acc", g[f"{key}_acc"], acc, rtol=1e-12, per_vector=True)
    _scaled("dudt", g[f"{key}_dudt"], dudt, 1e-12)
    check("vsig", g[f"{key}_vsig"], vsig, rtol=1e-14)
    _scaled("visc heat", g[f"{key}_visc"], vh, 1e-12)
    _scaled("cond heat", g[f"{key}_cond"], ch, 1e-12)


def test_reconstructed_forces_rows_cubic_match_reference():
    g = golden("shock.npz")
    nb = _nb(g["offset"], g["index"])
    args = (g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"], g["pressure"], nb)
    acc, dudt, vsig, _, _ = native.forces(*args, 0, C_NORM[0], u=g["u"], c_s=g["c_s"],
                                          alpha=g["alpha"], alpha_u=0.5, cond_signal=0,
                                          rows=g["rows"], grad_v=g["grad_v"])  # fmt: skip
    check("acc", g["recon_rows_cubic_acc"], acc, rtol=1e-12, per_vector=True)
    _scaled("dudt", g["recon_rows_cubic_dudt"], dudt, 1e-12)
    check("vsig", g["recon_rows_cubic_vsig"], vsig, rtol=1e-14)


def _switch_hc():
    from blackhole_nebula_simulator_b200.config import HydroConfig

    return HydroConfig(kernel="cubic", eta=1.2, switch=True, reconstruction=True,
                       conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip


def test_switch_shared_steps_match_reference():
    from blackhole_nebula_simulator_b200.config import CoupledConfig

    g = golden("switch_coupled.npz")
    cc = CoupledConfig(hydro=_switch_hc())
    st = steps.coupled_initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], cc)
    check("init alpha", g["init_alpha"], st.alpha)
    check("init acc", g["init_a_hydro"], st.a_hydro, rtol=1e-9, per_vector=True)
    for k in range(3):
        dt = steps.coupled_stable_dt(st, cc)
        check(f"dt {k}", g["dts"][k], dt, rtol=1e-12)
        st = steps.coupled_step(st, cc, dt)
        check(f"step {k + 1} alpha", g[f"step{k + 1}_alpha"], st.alpha, rtol=1e-9, atol=1e-12)
        check(f"step {k + 1} x", g[f"step{k + 1}_x"], st.x, rtol=1e-14, per_vector=True)
        check(f"step {k + 1} p", g[f"step{k + 1}_p"], st.p, rtol=1e-12, per_vector=True)
        check(f"step {k + 1} u", g[f"step{k + 1}_u"], st.u, rtol=1e-10)
        check(f"step {k + 1} h", g[f"step{k + 1}_h"], st.h, rtol=1e-10)
        check(f"step {k + 1} acc", g[f"step{k + 1}_a_hydro"], st.a_hydro, rtol=1e-8,
              per_vector=True)  # fmt: skip
        check(f"step {k + 1} energy", g[f"step{k + 1}_energy"],
              steps.coupled_ledger(st, cc)["energy"], rtol=1e-13)  # fmt: skip
    check("cache builds", int(g["builds"]), st.neighbour_cache.builds)
    check("cache reuses", int(g["reuses"]), st.neighbour_cache.reuses)


def test_switch_block_steps_match_reference():
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig

    g = golden("switch_blocks.npz")
    bc = BlockConfig(coupled=CoupledConfig(hydro=_switch_hc(), cooling_beta=230.0), dt_max=64.0)
    st = steps.blocks_initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6,
                                 level_offset=g["level_offset"])  # fmt: skip
    check("init levels", g["init_level"], st.level)
    check("init acc", g["init_a_hydro"], st.a_hydro, rtol=1e-9, per_vector=True)
    actives = [len(steps.blocks_advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("final tick", int(g["final_n"]), st.n)
    check("final levels", g["final_level"], st.level)
    check("final n_end", g["final_n_end"], st.n_end)
    check("final alpha", g["final_alpha"], st.alpha, rtol=1e-8, atol=1e-12)
    check("final x", g["final_x"], st.x, rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], st.p, rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], st.u, rtol=1e-9)
    check("final h", g["final_h"], st.h, rtol=1e-9)
    check("final energy", float(g["final_energy"]), steps.blocks_ledger(st, bc)["energy"],
          rtol=1e-12)  # fmt: skip
    check("final e_radiated", float(g["final_e_radiated"]), st.e_radiated, rtol=1e-9)
    check("cache builds", int(g["builds"]), st.neighbour_cache.builds)
    check("cache reuses", int(g["reuses"]), st.neighbour_cache.reuses)


def _dep_grids(g):
    from blackhole_nebula_simulator_b200.gasgrid import CartesianBox, LogSphericalGrid

    lg = LogSphericalGrid(r_min=float(g["log_grid"][0]), r_max=float(g["log_grid"][1]),
                          nr=int(g["log_grid"][2]), nth=int(g["log_grid"][3]),
                          nph=int(g["log_grid"][4]))  # fmt: skip
    bx = CartesianBox(centre=tuple(float(c) for c in g["box"][:3]), size=float(g["box"][3]),
                      n=int(g["box"][4]))  # fmt: skip
    sg = LogSphericalGrid(r_min=float(g["split_grid"][0]), r_max=float(g["split_grid"][1]),
                          nr=int(g["split_grid"][2]), nth=int(g["split_grid"][3]),
                          nph=int(g["split_grid"][4]))  # fmt: skip
    return lg, bx, sg


def _check_grid(name, g, prefix, res, exact=False):
    tol = {} if exact else {"rtol": 1e-12}
    scale = np.abs(g[f"{prefix}_mass"]).max()
    if exact:
        check(f"{name} mass", g[f"{prefix}_mass"], res["mass"])
    else:
        check(f"{name} mass", g[f"{prefix}_mass"] / scale, res["mass"] / scale, atol=1e-12)
    check(f"{name} outside", float(g[f"{prefix}_outside"]), res["outside"], **tol)
    check(f"{name} trilinear count", int(g[f"{prefix}_n_tri"]), res["n_trilinear"])
    for f in ("rho", "t_mass", "t_em", "vel"):
        a = g[f"{prefix}_{f}"].astype(np.float64)
        check(f"{name} {f}", a, res[f].astype(np.float64), atol=1e-6 * float(np.abs(a).max()))


@pytest.mark.parametrize("kernel", ["wendland_c4", "cubic"])
def test_log_deposition_matches_reference(kernel):
    from oracle import deposit as odep

    g = golden("deposit.npz")
    lg, _, _ = _dep_grids(g)
    res = odep.deposit_log(g["x"], g["h"], g["m"], g["t"], g["v"], lg, kernel)
    _check_grid(f"log {kernel}", g, f"log_{kernel}", res, exact=True)


@pytest.mark.parametrize("kernel", ["wendland_c4", "cubic"])
def test_box_deposition_matches_reference(kernel):
    from oracle import deposit as odep

    g = golden("deposit.npz")
    _, bx, _ = _dep_grids(g)
    res = odep.deposit_box(g["xb"], g["hb"], g["m"], g["t"], g["v"], bx, kernel)
    _check_grid(f"box {kernel}", g, f"box_{kernel}", res, exact=True)


def test_split_deposition_matches_reference():
    from blackhole_nebula_simulator_b200.gasgrid import coarse_log_grid
    from oracle import deposit as odep

    g = golden("deposit.npz")
    _, _, sg = _dep_grids(g)
    check("wide particles", g["split_wide"], odep.wide_particles(g["xs"], g["hs"], sg))
    res = odep.deposit_log_split(g["xs"], g["hs"], g["ms"], g["ts"], g["vs"], sg,
                                 coarse_log_grid(sg))  # fmt: skip
    check("wide count", int(g["split_n_wide"]), res["n_wide"])
    _check_grid("split", g, "split", res)


def test_log_grid_volumes_fill_the_shell():
    """Cell volumes add up to the shell volume 4/3 pi (r_max^3 - r_min^3)."""
    from blackhole_nebula_simulator_b200.gasgrid import LogSphericalGrid

    g = LogSphericalGrid(r_min=2.0, r_max=200.0, nr=24, nth=12, nph=24)
    check("sum of cell volumes", 4.0 / 3.0 * np.pi * (g.r_max**3 - g.r_min**3),
          g.volumes().sum() * g.nph, rtol=1e-12)  # fmt: skip


def _removal_bc(sync=False):
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig, HydroConfig

    hc = HydroConfig(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                     conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    return BlockConfig(coupled=CoupledConfig(hydro=hc), dt_max=4.0, r_acc=4.4, r_escape=6.0,
                       removal_sync=sync)  # fmt: skip


@pytest.mark.parametrize("sync", [False, True])
def test_removal_block_steps_match_reference(sync):
    g = golden("removal_sync_blocks.npz" if sync else "removal_blocks.npz")
    bc = _removal_bc(sync)
    st = steps.blocks_initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6)
    actives = [len(steps.blocks_advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("final tick", int(g["final_n"]), st.n)
    check("remaining ids", g["final_ids"], st.ids)
    check("final levels", g["final_level"], st.level)
    check("final n_end", g["final_n_end"], st.n_end)
    check("pericentre flags", g["final_passed_peri"], st.passed_peri)
    check("inward flags", g["final_vr_neg"], st.vr_neg)
    check("doomed flags", g["final_doomed"], st.doomed)
    check("woken", int(g["woken"]), st.woken)
    check("final x", g["final_x"], st.x, rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], st.p, rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], st.u, rtol=1e-9)
    check("final h", g["final_h"], st.h, rtol=1e-9)
    log = st.removed.log
    check("removed ids in order", g["log_id"], np.array([e["id"] for e in log]))
    check("removal reasons", g["log_escaped"], np.array([e["reason"] == "escaped" for e in log]))
    check("removal times", g["log_t"], np.array([e["t"] for e in log]), rtol=1e-15)
    check("first pass flags", g["log_first_pass"], np.array([e["first_pass"] for e in log]))
    check("removed mass", float(g["removed_mass"]), st.removed.mass, rtol=1e-13)
    check("removed energy", float(g["removed_energy"]), st.removed.energy, rtol=1e-10)
    check("removed angmom", g["removed_angmom"], st.removed.angmom, rtol=1e-10, per_vector=True)
    check("final energy", float(g["final_energy"]), steps.blocks_ledger(st, bc)["energy"],
          rtol=1e-12)  # fmt: skip


def _wake_bc():
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig

    hc, CC = _cfg()
    return BlockConfig(coupled=CC(hydro=hc, cooling_beta=230.0), dt_max=64.0, r_acc=382.0,
                       removal_sync=True)  # fmt: skip


def test_removal_wake_matches_reference():
    g = golden("removal_wake_blocks.npz")
    bc = _wake_bc()
    st = steps.blocks_initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6,
                                 level_offset=g["level_offset"])  # fmt: skip
    actives = [len(steps.blocks_advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("woken", int(g["woken"]), st.woken)
    check("removed ids", g["log_id"], np.array([e["id"] for e in st.removed.log]))
    check("remaining ids", g["final_ids"], st.ids)
    for f in ("level", "n_beg", "n_end", "doomed"):
        check(f"final {f}", g[f"final_{f}"], getattr(st, f))
    check("final x", g["final_x"], st.x, rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], st.p, rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], st.u, rtol=1e-9)
    check("final energy", float(g["final_energy"]), steps.blocks_ledger(st, bc)["energy"],
          rtol=1e-12)  # fmt: skip


def _phantom_rel(ours, theirs):
    """tests/sim/test_phantom_patch.py:75-81: per-particle relative difference."""
    if ours.ndim == 2:
        mag, diff = np.linalg.norm(ours, axis=1), np.linalg.norm(ours - theirs, axis=1)
    else:
        mag, diff = np.abs(ours), np.abs(ours - theirs)
    return diff / np.maximum(mag, 1e-6 * np.median(mag))


def phantom_hydro(g, recon):
    from blackhole_nebula_simulator_b200.config import HydroConfig

    return HydroConfig(kernel=str(g["kernel"]), eta=float(g["eta"]), h_max=float(g["h_max"]),
                       alpha_u=float(g["alpha_u"]), beta=float(g["beta"]),
                       conductivity_signal=int(g["conductivity_signal"]),
                       recon_closeness=bool(g["recon_closeness"]), recon_gate=int(g["recon_gate"]),
                       eos="gasrad", reconstruction=recon)  # fmt: skip


@pytest.mark.parametrize("recon", [True, False], ids=["recon_on", "recon_off"])
def test_oracle_matches_phantom_golden_vectors(recon):
    """The reference's cross-code check (tests/sim/test_phantom_patch.py:86-98): density, EOS,
    velocity gradients and forces of the default hydro settings with gas + radiation against
    Phantom's derivatives on 8,931 particles; median relative difference 1e-5, 99th percentile
    1e-3 over the 2,203 particles within 600 of the centre (Phantom's pressure used, as there)."""
    from oracle import eos as oeos
    from oracle.sph import compute_density as ocompute

    g = golden("phantom_forces.npz")
    hc = phantom_hydro(g, recon)
    inner = np.linalg.norm(g["x"] - g["center"], axis=1) < g["r_in"]
    check("particles compared", 2203, int(inner.sum()))
    kid = KERNEL_IDS[hc.kernel]
    dens = ocompute(g["x"], g["mass"], g["h_phantom"], kernel_name=hc.kernel, eta=hc.eta,
                    h_max=hc.h_max, reuse=False)  # fmt: skip
    nb = native.tighten(dens.neighbours, g["x"], dens.h)
    p_ours, cs_ours = oeos.eos_state(hc, dens.rho, g["u"])
    p = g["pressure"] / g["mratio"]
    cs = cs_ours * np.sqrt(p / p_ours)
    gv = native.velocity_gradients(g["x"], g["v"], g["mass"], dens.h, nb, kid, C_NORM[kid])
    acc, dudt, _, _, _ = native.forces(g["x"], g["v"], g["mass"], dens.h, dens.rho, dens.omega, p,
                                       nb, kid, C_NORM[kid], u=g["u"], c_s=cs, alpha=g["alpha"],
                                       beta=hc.beta, alpha_u=hc.alpha_u,
                                       cond_signal=hc.conductivity_signal,
                                       grad_v=gv if recon else None, closeness=hc.recon_closeness,
                                       eta_crit=1.0 / hc.eta, gate=hc.recon_gate)  # fmt: skip
    tag = "on" if recon else "off"
    ra = _phantom_rel(acc, g[f"acc_{tag}"])[inner]
    ru = _phantom_rel(dudt, g[f"dudt_{tag}"])[inner]
    check("|a| median", 0.0, float(np.median(ra)), atol=1e-5)
    check("|a| 99th percentile", 0.0, float(np.percentile(ra, 99)), atol=1e-3)
    check("du/dt median", 0.0, float(np.median(ru)), atol=1e-5)
    check("du/dt 99th percentile", 0.0, float(np.percentile(ru, 99)), atol=1e-3)


HEAT_PARTS = ("heat_visc", "heat_cond", "heat_disk", "heat_pdv", "heat_cool")


def heat_runs(g, initialise, run, advance, wake=False, **hydro):
    """The runs of tests/golden/heat_blocks.npz through a block-step API (the oracle's or the
    device facade's): yields (prefix, state) after each; with ``wake`` also the run whose
    limiter wakes particles up."""
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig, HydroConfig

    hc = HydroConfig(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                     conductivity_signal=1, alpha_u=0.05, h_max=200.0, disc_alpha_av=1.0,
                     **hydro)  # fmt: skip
    bc = BlockConfig(coupled=CoupledConfig(hydro=hc, cooling_beta=230.0), dt_max=64.0)
    args = (g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc)
    st = initialise(*args, t_stop=192.0, level_offset=g["level_offset"])
    yield "sync", run(st, bc, 192.0)
    st = initialise(*args, t_stop=1e6, level_offset=g["level_offset"])
    yield "reopen", run(st, bc, 0.75)
    bc = _wake_bc()
    st = initialise(*args[:5], bc, t_stop=1e6, level_offset=g["level_offset"])
    for _ in range(16):
        advance(st, bc)
    yield "removal", st
    if wake:
        bc = BlockConfig(coupled=CoupledConfig(hydro=hc, cooling_beta=230.0), dt_max=64.0)
        st = initialise(*args[:5], bc, t_stop=64.0, level_offset=g["wake_offset"])
        yield "wake", run(st, bc, 64.0)


def check_heat(g, pre, arrays, e_radiated, tol):
    """Every heat-budget array against the reference's, each to ``tol`` of its largest value;
    the budget identity u_half - u_0 = visc + cond + disk + pdv - cool (the reference's own
    test, tests/sim/test_heat_budget.py:19-46) where the reference has it (sync, removal: to
    1e-12 of max u_0) and its failure by the twice-booked opening kick where run() re-opens
    (reopen), equal to the reference's; the cooling budget against the radiated energy."""
    scale = {}
    for f in ("u_half",) + HEAT_PARTS + ("visc_heating", "cond_heating", "disk_heating"):
        ref = g[f"{pre}_{f}"]
        scale[f] = float(np.abs(ref).max())
        check(f"{pre} {f}", ref, arrays[f], atol=tol * max(scale[f], 1e-300))
    u0 = g["u0"] if pre != "removal" else g["u0"][g["removal_ids"]]
    parts = (arrays["heat_visc"] + arrays["heat_cond"] + arrays["heat_disk"] + arrays["heat_pdv"]
             - arrays["heat_cool"])  # fmt: skip
    gap = arrays["u_half"] - u0 - parts
    ref_parts = sum(g[f"{pre}_{f}"] for f in HEAT_PARTS[:4]) - g[f"{pre}_heat_cool"]
    ref_gap = g[f"{pre}_u_half"] - u0 - ref_parts
    umax = float(np.abs(u0).max())
    if pre == "reopen":
        check("reopen: the budget is off by the second opening kick", ref_gap, gap,
              atol=tol * float(np.abs(ref_gap).max()))  # fmt: skip
    else:
        check(f"{pre}: u_half - u0 = visc + cond + disk + pdv - cool", 0.0,
              float(np.abs(gap).max()) / umax, atol=1e-12)  # fmt: skip
    if pre == "sync":
        check("cooling budget equals the radiated energy", float(g["sync_e_radiated"]),
              e_radiated, rtol=1e-9)  # fmt: skip
        check("sum m heat_cool = e_radiated", e_radiated,
              float(np.sum(g["mass"] * arrays["heat_cool"])), rtol=1e-12)  # fmt: skip


def test_heat_budget_matches_reference():
    g = golden("heat_blocks.npz")
    for pre, st in heat_runs(g, steps.blocks_initialise, steps.blocks_run, steps.blocks_advance,
                             wake=True):  # fmt: skip
        check(f"{pre} tick", int(g[f"{pre}_n"]), st.n)
        if pre == "wake":
            check("wake-ups", int(g["wake_woken"]), st.woken)
        if pre == "removal":
            check("removal ids", g["removal_ids"], st.ids)
        arrays = {k: getattr(st, k) for k in ("u_half", "visc_heating", "cond_heating",
                                              "disk_heating") + HEAT_PARTS}  # fmt: skip
        check_heat(g, pre, arrays, st.e_radiated, 1e-9)
