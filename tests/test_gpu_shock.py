"""Cullen-Dehnen switch and velocity reconstruction on the GPU against the reference's outputs
(tests/golden/shock.npz, switch_coupled.npz, switch_blocks.npz).

Tolerances: the single-call kernels (gradients, reconstructed forces) at the reference's own
1e-12, relative to each output's largest magnitude (the GPU sums each row's list in list order,
like the reference; the 3x3 inverse is the adjugate instead of LAPACK's LU); whole FP64 steps at
the tolerances of the ideal-gas step tests, alpha at rtol 1e-8 (it is a ratio of gradient sums
that cancel); levels, tick counters and list builds/reuses exactly.  The FP32 form against the
FP64 form at the FP32 tolerances of tests/test_gpu_fp32_errors.py.
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
    from blackhole_nebula_simulator_b200 import blocks, coupled, ops

    return ops, coupled, blocks


def _np(t):
    return t.detach().cpu().numpy() if hasattr(t, "detach") else np.asarray(t)


def _scaled(name, expected, actual, tol):
    scale = np.abs(expected).max()
    check(name, expected / scale, _np(actual) / scale, atol=tol)


def _lists(ops, g):
    return ops.Neighbours(g["offset"], g["index"].astype(np.int64), None)


def test_gradients_match_reference(nb):
    ops, _, _ = nb
    g = golden("shock.npz")
    nbl = _lists(ops, g)
    r = ops.gradients_numba(g["pos"], g["vel"], g["acc_prev"], g["mass"], g["h"], nbl)
    _scaled("div v", g["div_v"], r.div_v, 1e-12)
    _scaled("curl v", g["curl_v"], r.curl_v, 1e-12)
    _scaled("d div v / dt", g["ddivv_dt"], r.ddivv_dt, 1e-12)
    r = ops.gradients_numba(g["pos"], g["vel"], g["acc_prev"], g["mass"], g["h"], nbl,
                            kernel_name="cubic", rows=g["rows"])  # fmt: skip
    _scaled("cubic rows div v", g["cubic_rows_div_v"], r.div_v, 1e-12)
    _scaled("cubic rows curl v", g["cubic_rows_curl_v"], r.curl_v, 1e-12)
    _scaled("cubic rows d div v / dt", g["cubic_rows_ddivv_dt"], r.ddivv_dt, 1e-12)


def test_velocity_gradients_match_reference(nb):
    ops, _, _ = nb
    g = golden("shock.npz")
    gv = ops.velocity_gradients_numba(g["pos"], g["vel"], g["mass"], g["h"], _lists(ops, g))
    _scaled("grad v (tight lists)", g["grad_v"], gv, 1e-12)
    # the untightened lists (search radius 1.4 h) from the GPU list build, bit-exact with the
    # reference's; isolated and planar particles take the fallback of the correction matrix
    full = ops.find_neighbours(g["pos"], 1.4 * g["h"])
    gv = ops.velocity_gradients_numba(g["pos"], g["vel"], g["mass"], g["h"], full, rows=g["rows"])
    _scaled("grad v (untightened lists, rows)", g["full_rows_grad_v"], gv, 1e-12)


@pytest.mark.parametrize("gate", [0, 1, 2])
@pytest.mark.parametrize("close", [True, False])
def test_reconstructed_forces_match_reference(nb, gate, close):
    from blackhole_nebula_simulator_b200.config import ShockCapturing

    ops, _, _ = nb
    g = golden("shock.npz")
    shock = ShockCapturing(beta=2.0, alpha_u=0.5, conductivity_signal=1, reconstruction=True,
                           closeness=close, eta_crit=1.0 / 1.2, recon_gate=gate)  # fmt: skip
    f = ops.forces_numba(g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"],
                         g["pressure"], _lists(ops, g), u=g["u"], c_s=g["c_s"], alpha=g["alpha"],
                         shock=shock, grad_v=g["grad_v"])  # fmt: skip
    key = f"recon_g{gate}_c{int(close)}"
    check("acc", g[f"{key}_acc"], _np(f.acc), rtol=1e-12, per_vector=True)
    _scaled("dudt", g[f"{key}_dudt"], f.dudt, 1e-12)
    check("vsig", g[f"{key}_vsig"], _np(f.vsig_max), rtol=1e-14)
    _scaled("visc heat", g[f"{key}_visc"], f.dudt_visc, 1e-12)
    _scaled("cond heat", g[f"{key}_cond"], f.dudt_cond, 1e-12)


def test_reconstructed_forces_rows_cubic_match_reference(nb):
    from blackhole_nebula_simulator_b200.config import ShockCapturing

    ops, _, _ = nb
    g = golden("shock.npz")
    shock = ShockCapturing(beta=2.0, alpha_u=0.5, conductivity_signal=0, reconstruction=True,
                           eta_crit=1.0 / 1.2)  # fmt: skip
    f = ops.forces_numba(g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"],
                         g["pressure"], _lists(ops, g), kernel_name="cubic", u=g["u"],
                         c_s=g["c_s"], alpha=g["alpha"], shock=shock, rows=g["rows"],
                         grad_v=g["grad_v"])  # fmt: skip
    check("acc", g["recon_rows_cubic_acc"], _np(f.acc), rtol=1e-12, per_vector=True)
    _scaled("dudt", g["recon_rows_cubic_dudt"], f.dudt, 1e-12)
    check("vsig", g["recon_rows_cubic_vsig"], _np(f.vsig_max), rtol=1e-14)


def test_reconstruction_needs_grad_v(nb):
    from blackhole_nebula_simulator_b200.config import ShockCapturing

    ops, _, _ = nb
    g = golden("shock.npz")
    with pytest.raises(ValueError, match="grad_v"):
        ops.forces_numba(g["pos"], g["vel"], g["mass"], g["h"], g["rho"], g["omega"],
                         g["pressure"], _lists(ops, g), u=g["u"], c_s=g["c_s"], alpha=g["alpha"],
                         shock=ShockCapturing(reconstruction=True))  # fmt: skip


def _switch_hc(precision="fp64"):
    from blackhole_nebula_simulator_b200.config import HydroConfig

    return HydroConfig(kernel="cubic", eta=1.2, switch=True, reconstruction=True,
                       conductivity_signal=1, alpha_u=0.05, h_max=200.0, precision=precision)  # fmt: skip


def test_switch_shared_steps_match_reference(nb):
    from blackhole_nebula_simulator_b200.config import CoupledConfig

    _, coupled, _ = nb
    g = golden("switch_coupled.npz")
    cc = CoupledConfig(hydro=_switch_hc())
    st = coupled.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], cc)
    check("init alpha", g["init_alpha"], _np(st.alpha))
    check("init acc", g["init_a_hydro"], _np(st.a_hydro), rtol=1e-9, per_vector=True)
    for k in range(3):
        dt = coupled.stable_dt(st, cc)
        check(f"dt {k}", g["dts"][k], dt, rtol=1e-12)
        st = coupled.step(st, cc, dt)
        check(f"step {k + 1} alpha", g[f"step{k + 1}_alpha"], _np(st.alpha), rtol=1e-8,
              atol=1e-12)  # fmt: skip
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


def test_switch_block_steps_match_reference(nb):
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig

    _, _, blocks = nb
    g = golden("switch_blocks.npz")
    bc = BlockConfig(coupled=CoupledConfig(hydro=_switch_hc(), cooling_beta=230.0), dt_max=64.0)
    st = blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6,
                           level_offset=g["level_offset"])  # fmt: skip
    check("init levels", g["init_level"], _np(st.level))
    check("init acc", g["init_a_hydro"], _np(st.a_hydro), rtol=1e-9, per_vector=True)
    actives = [len(blocks.advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("final tick", int(g["final_n"]), st.n)
    check("final levels", g["final_level"], _np(st.level))
    check("final n_end", g["final_n_end"], _np(st.n_end))
    check("final alpha", g["final_alpha"], _np(st.alpha), rtol=1e-8, atol=1e-12)
    check("final x", g["final_x"], _np(st.x), rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], _np(st.p), rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], _np(st.u), rtol=1e-9)
    check("final h", g["final_h"], _np(st.h), rtol=1e-9)
    check("final energy", float(g["final_energy"]), blocks.ledger(st, bc)["energy"], rtol=1e-12)
    check("final e_radiated", float(g["final_e_radiated"]), st.e_radiated, rtol=1e-9)
    check("list builds", int(g["builds"]), st.builds)
    check("list reuses", int(g["reuses"]), st.reuses)


def test_switch_fp32_within_stated_tolerance(nb):
    """The FP32 form with the switch and the reconstruction against the FP64 form: 16 block steps
    of the switch fixture's cloud (levels and active counts must agree)."""
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig
    from tests.test_gpu_fp32_errors import TOL

    _, _, blocks = nb
    g = golden("switch_blocks.npz")
    out = []
    for prec in ("fp64", "fp32"):
        bc = BlockConfig(coupled=CoupledConfig(hydro=_switch_hc(prec), cooling_beta=230.0),
                         dt_max=64.0)  # fmt: skip
        st = blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6,
                               level_offset=g["level_offset"])  # fmt: skip
        act = [len(blocks.advance(st, bc)) for _ in range(16)]
        out.append((st, act))
    (a, act_a), (b, act_b) = out
    check("active counts", np.array(act_a), np.array(act_b))
    check("levels", _np(a.level), _np(b.level))
    for f in ("h", "rho", "u"):
        check(f, _np(a.__getattribute__(f)), _np(b.__getattribute__(f)), rtol=TOL[f])
    for f in ("x", "p"):
        check(f, _np(getattr(a, f)), _np(getattr(b, f)), rtol=TOL[f], per_vector=True)
    amax = np.linalg.norm(_np(a.a_hydro), axis=1).max()
    check("a_hydro", _np(a.a_hydro) / amax, _np(b.a_hydro) / amax, atol=TOL["a_hydro"])
    dmax = np.abs(_np(a.dudt)).max()
    check("dudt", _np(a.dudt) / dmax, _np(b.dudt) / dmax, atol=TOL["dudt"])
    check("alpha", _np(a.alpha), _np(b.alpha), atol=1e-3)


@pytest.mark.parametrize("recon", [True, False], ids=["recon_on", "recon_off"])
def test_phantom_golden_vectors(nb, recon):
    """The reference's cross-code check (tests/sim/test_phantom_patch.py:86-98) on the GPU:
    density (lists built and regrown on the device), the gas + radiation EOS, velocity gradients
    and the force pass of the reference's default hydro settings against Phantom's derivatives
    of 8,931 particles; median relative difference 1e-5, 99th percentile 1e-3 over the 2,203
    particles within 600 of the centre (Phantom's pressure used, as in the reference's test)."""
    from tests.test_oracle_golden import _phantom_rel, phantom_hydro

    ops, _, _ = nb
    g = golden("phantom_forces.npz")
    hc = phantom_hydro(g, recon)
    inner = np.linalg.norm(g["x"] - g["center"], axis=1) < g["r_in"]
    dens = ops.compute_density(g["x"], g["mass"], g["h_phantom"], kernel_name=hc.kernel,
                               eta=hc.eta, h_max=hc.h_max)  # fmt: skip
    nbl = ops.tighten(dens.neighbours, g["x"], dens.h)
    p_ours, cs_ours = ops.eos_state(hc, dens.rho, g["u"])
    p = g["pressure"] / g["mratio"]
    cs = _np(cs_ours) * np.sqrt(p / _np(p_ours))
    gv = ops.velocity_gradients_numba(g["x"], g["v"], g["mass"], dens.h, nbl, hc.kernel)
    f = ops.forces_numba(g["x"], g["v"], g["mass"], dens.h, dens.rho, dens.omega, p, nbl,
                         hc.kernel, u=g["u"], c_s=cs, alpha=g["alpha"], shock=hc.shock(),
                         grad_v=gv if recon else None)  # fmt: skip
    tag = "on" if recon else "off"
    ra = _phantom_rel(_np(f.acc), g[f"acc_{tag}"])[inner]
    ru = _phantom_rel(_np(f.dudt), g[f"dudt_{tag}"])[inner]
    check("|a| median", 0.0, float(np.median(ra)), atol=1e-5)
    check("|a| 99th percentile", 0.0, float(np.percentile(ra, 99)), atol=1e-3)
    check("du/dt median", 0.0, float(np.median(ru)), atol=1e-5)
    check("du/dt 99th percentile", 0.0, float(np.percentile(ru, 99)), atol=1e-3)
