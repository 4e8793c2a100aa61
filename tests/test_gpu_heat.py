"""Per-particle heat budget of the block steps (sim/blocks.py:142-154, 434-440, 531, 546) on the
GPU against the reference's (tests/golden/heat_blocks.npz): the multi-level cloud with viscosity,
conductivity, disc viscosity and beta-cooling run to a sync point, run() re-opening every step to
land on a near stop (the opening kick booked twice, as the reference does), removal_sync
dropping removed particles' budgets, and a run whose level limiter wakes neighbours up (5 % of
the particles forced 5 levels finer), so the corrected half kick of a wake-up is booked.

Tolerances: every array to 1e-9 of its largest value (the block-step tolerance of u); the budget
identity u_half - u_0 = visc + cond + disk + pdv - cool to 1e-12 of max u_0 where it holds, and
its offset where run() re-opens to 1e-9 of the reference's; the cooling budget sum m heat_cool
against the radiated energy to 1e-12.
"""

import numpy as np
import pytest

from tests.conftest import check, golden
from tests.test_oracle_golden import HEAT_PARTS, check_heat, heat_runs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def blocks():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from blackhole_nebula_simulator_b200 import blocks

    return blocks


def test_heat_budget_matches_reference(blocks):
    g = golden("heat_blocks.npz")
    seen = []
    for pre, st in heat_runs(g, blocks.initialise, blocks.run, blocks.advance, wake=True):
        seen.append(pre)
        check(f"{pre} tick", int(g[f"{pre}_n"]), st.n)
        if pre == "wake":
            check("wake-ups", int(g["wake_woken"]), st.woken)
        if pre == "removal":
            check("removal ids", g["removal_ids"], st.ids.cpu().numpy())
        arrays = {k: getattr(st, k).cpu().numpy() for k in (
            "u_half", "visc_heating", "cond_heating", "disk_heating") + HEAT_PARTS}  # fmt: skip
        check_heat(g, pre, arrays, st.e_radiated, 1e-9)
    check("runs checked", ["sync", "reopen", "removal", "wake"], seen)


def test_heat_budget_fp32_adds_up(blocks):
    """The FP32 pair arithmetic books the same kicks: the identity holds to round-off and every
    part acted."""
    g = golden("heat_blocks.npz")
    runs = heat_runs(g, blocks.initialise, blocks.run, blocks.advance, precision="fp32")
    pre, st = next(runs)
    parts = sum(getattr(st, k) for k in HEAT_PARTS[:4]) - st.heat_cool
    gap = (st.u_half - (st.u_half.new_tensor(g["u0"])) - parts).abs().max().item()
    check("fp32: u_half - u0 = visc + cond + disk + pdv - cool", 0.0,
          gap / float(np.abs(g["u0"]).max()), atol=1e-12)  # fmt: skip
    check("every part acted", True, all(bool((getattr(st, k) != 0).any()) for k in HEAT_PARTS))
    check("fp32 heat_visc near the reference's", g["sync_heat_visc"], st.heat_visc.cpu().numpy(),
          atol=1e-3 * float(np.abs(g["sync_heat_visc"]).max()))  # fmt: skip
