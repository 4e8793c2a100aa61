"""Equations of state on the GPU against the reference's outputs (tests/golden/eos.npz and
gasrad_blocks.npz).

Tolerances: the ideal gas and the radiation limit to rounding (rtol 1e-15).  Gas + radiation:
T within rtol 5e-12.  The reference's Newton iteration on log T stops when a step falls below
1e-12; where f(T) rounds to a tiny non-zero value at the root its bracket test sends the iterate
into bisection, which then ends anywhere inside a 1e-12-wide interval of log T, so one ulp of
difference between CUDA's and the C library's exp picks a different end point (the CPU oracle,
in the C library's arithmetic, matches the reference bit for bit).  P ~ T^4 and c_s ~ sqrt(P)
then carry at most 4x and 2x that: rtol 2e-11.  Block steps with gas + radiation at the
tolerances of the ideal-gas block test; levels and tick counters exactly.
"""

import numpy as np
import pytest

from tests.conftest import check, golden

pytestmark = pytest.mark.gpu

T_RTOL = 5e-12
P_RTOL = 2e-11


@pytest.fixture(scope="module")
def nb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from blackhole_nebula_simulator_b200 import blocks, ops

    return ops, blocks


def _np(t):
    return t.detach().cpu().numpy()


def test_gasrad_state_matches_reference(nb):
    ops, _ = nb
    g = golden("eos.npz")
    p, cs, t, beta = ops.gasrad_state(g["rho"], g["u"])
    check("gasrad T", g["gasrad_t"], _np(t), rtol=T_RTOL)
    check("gasrad P", g["gasrad_p"], _np(p), rtol=P_RTOL)
    check("gasrad c_s", g["gasrad_cs"], _np(cs), rtol=P_RTOL)
    check("gasrad beta", g["gasrad_beta"], _np(beta), rtol=P_RTOL, atol=1e-300)


@pytest.mark.parametrize("eos", ["ideal", "radiation", "gasrad"])
def test_eos_state_matches_reference(nb, eos):
    from blackhole_nebula_simulator_b200.config import HydroConfig

    ops, _ = nb
    g = golden("eos.npz")
    p, cs = ops.eos_state(HydroConfig(eos=eos), g["rho"], g["u"])
    tol = 1e-15 if eos != "gasrad" else P_RTOL
    check(f"{eos} P", g[f"{eos}_p"], _np(p), rtol=tol)
    check(f"{eos} c_s", g[f"{eos}_cs"], _np(cs), rtol=tol)


def test_eos_errors_raise_and_leave_the_context_usable(nb):
    """physics/eos.py:123-124 (u outside the bracket: ValueError) and sim/hydro.py:127-128
    (u <= 0: FloatingPointError)."""
    from blackhole_nebula_simulator_b200.config import HydroConfig

    ops, _ = nb
    hc = HydroConfig(eos="gasrad")
    rho = np.full(3, 1e-8)
    with pytest.raises(ValueError, match="bracket"):
        ops.eos_state(hc, rho, np.array([1e-12, 1e-30, 1e-12]))
    with pytest.raises(ValueError, match="bracket"):
        ops.eos_state(hc, rho, np.array([1e-12, 1e29, 1e-12]))
    with pytest.raises(FloatingPointError):
        ops.eos_state(hc, rho, np.array([1e-12, 0.0, 1e-12]))
    g = golden("eos.npz")
    p, _ = ops.eos_state(hc, g["rho"][:16], g["u"][:16])
    check("gasrad P after the errors", g["gasrad_p"][:16], _np(p), rtol=P_RTOL)


def test_empty_input(nb):
    from blackhole_nebula_simulator_b200.config import HydroConfig

    ops, _ = nb
    p, cs = ops.eos_state(HydroConfig(eos="gasrad"), np.zeros(0), np.zeros(0))
    assert p.shape == (0,) and cs.shape == (0,)


def test_gasrad_block_steps_match_reference(nb):
    """The 2,048-particle cloud at 3e8 K (radiation-dominated, beta_gas ~ 1e-3) in block steps with
    the gas + radiation EOS (sim/blocks.py with sim/hydro.py:134-136)."""
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig, HydroConfig

    _, blocks = nb
    g = golden("gasrad_blocks.npz")
    hc = HydroConfig(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                     conductivity_signal=1, alpha_u=0.05, h_max=200.0, eos="gasrad")  # fmt: skip
    bc = BlockConfig(coupled=CoupledConfig(hydro=hc), dt_max=64.0)
    st = blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6)
    check("init levels", g["init_level"], _np(st.level))
    check("init n_end", g["init_n_end"], _np(st.n_end))
    # du/dt sums terms of either sign: absolute tolerance on the largest term's scale
    check("init dudt", g["init_dudt"], _np(st.dudt), rtol=1e-9,
          atol=1e-10 * np.abs(g["init_dudt"]).max())  # fmt: skip
    check("init acc", g["init_a_hydro"], _np(st.a_hydro), rtol=1e-9, per_vector=True)
    actives = [len(blocks.advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("final tick", int(g["final_n"]), st.n)
    check("final levels", g["final_level"], _np(st.level))
    check("final n_end", g["final_n_end"], _np(st.n_end))
    check("final x", g["final_x"], _np(st.x), rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], _np(st.p), rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], _np(st.u), rtol=1e-9)
    check("final h", g["final_h"], _np(st.h), rtol=1e-9)
    check("final dudt", g["final_dudt"], _np(st.dudt), rtol=1e-8,
          atol=1e-9 * np.abs(g["final_dudt"]).max())  # fmt: skip
    check("final energy", float(g["final_energy"]), blocks.ledger(st, bc)["energy"], rtol=1e-12)


def test_gasrad_fp32_within_stated_tolerance(nb):
    """The FP32 form with gas + radiation against the FP64 form on the gasrad_blocks cloud
    (12 block steps; levels and active counts must agree, the rest at the FP32 tolerances of
    tests/test_gpu_fp32_errors.py)."""
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig, HydroConfig
    from tests.test_gpu_fp32_errors import TOL

    _, blocks = nb
    g = golden("gasrad_blocks.npz")
    out = []
    for prec in ("fp64", "fp32"):
        hc = HydroConfig(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                         conductivity_signal=1, alpha_u=0.05, h_max=200.0, eos="gasrad",
                         precision=prec)  # fmt: skip
        bc = BlockConfig(coupled=CoupledConfig(hydro=hc), dt_max=64.0)
        st = blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6)
        act = [len(blocks.advance(st, bc)) for _ in range(12)]
        out.append((st, act))
    (a, act_a), (b, act_b) = out
    check("active counts", np.array(act_a), np.array(act_b))
    check("levels", _np(a.level), _np(b.level))
    for f in ("h", "rho", "u"):
        check(f, _np(getattr(a, f)), _np(getattr(b, f)), rtol=TOL[f])
    check("x", _np(a.x), _np(b.x), rtol=TOL["x"], per_vector=True)
    check("p", _np(a.p), _np(b.p), rtol=TOL["p"], per_vector=True)
