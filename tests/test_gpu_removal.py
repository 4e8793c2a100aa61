"""Removal of particles at the end of their own steps (sim/blocks.py:566-719, sim/accretion.py)
on the GPU against the reference's block steps, without removal_sync (tests/golden/
removal_blocks.npz) and with it (removal_sync_blocks.npz: the survivors' forces recomputed after
a removal, the doomed particles' neighbours cut): a cloud falling past the accretion radius 4.4
and spilling over the escape radius 6.0.

Active counts, remaining ids, levels, tick counters, pericentre flags and the removal log (ids,
reasons, times, first-pass flags) exactly; the state at the block-step tolerances; the removed
totals and the energy ledger (removed energy included) to 1e-10 and 1e-12.
"""

import numpy as np
import pytest

from tests.conftest import check, golden
from tests.test_oracle_golden import _removal_bc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def blocks():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from blackhole_nebula_simulator_b200 import blocks

    return blocks


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("sync", [False, True])
def test_removal_block_steps_match_reference(blocks, sync):
    g = golden("removal_sync_blocks.npz" if sync else "removal_blocks.npz")
    bc = _removal_bc(sync)
    st = blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6)
    actives = [len(blocks.advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("final tick", int(g["final_n"]), st.n)
    check("remaining ids", g["final_ids"], _np(st.ids))
    check("final levels", g["final_level"], _np(st.level))
    check("final n_end", g["final_n_end"], _np(st.n_end))
    check("pericentre flags", g["final_passed_peri"], _np(st.passed_peri))
    check("inward flags", g["final_vr_neg"], _np(st.vr_neg))
    check("doomed flags", g["final_doomed"], _np(st.doomed))
    check("woken", int(g["woken"]), st.woken)
    check("final x", g["final_x"], _np(st.x), rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], _np(st.p), rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], _np(st.u), rtol=1e-9)
    check("final h", g["final_h"], _np(st.h), rtol=1e-9)
    log = st.removed.log
    check("removed ids in order", g["log_id"], np.array([e["id"] for e in log]))
    check("removal reasons", g["log_escaped"], np.array([e["reason"] == "escaped" for e in log]))
    check("removal times", g["log_t"], np.array([e["t"] for e in log]), rtol=1e-15)
    check("first pass flags", g["log_first_pass"], np.array([e["first_pass"] for e in log]))
    check("removed mass", float(g["removed_mass"]), st.removed.mass, rtol=1e-13)
    check("removed energy", float(g["removed_energy"]), st.removed.energy, rtol=1e-10)
    check("removed angmom", g["removed_angmom"], st.removed.angmom, rtol=1e-10, per_vector=True)
    led = blocks.ledger(st, bc)
    check("final energy", float(g["final_energy"]), led["energy"], rtol=1e-12)
    check("removed count", len(g["log_id"]), led["removed_count"])


def test_removal_wake_matches_reference(blocks):
    """The doomed particles' neighbours cut to end their steps with theirs (multi-level cloud,
    accretion radius 382 crossed by its inner edge)."""
    from tests.test_oracle_golden import _wake_bc

    g = golden("removal_wake_blocks.npz")
    bc = _wake_bc()
    st = blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6,
                           level_offset=g["level_offset"])  # fmt: skip
    actives = [len(blocks.advance(st, bc)) for _ in range(len(g["active_counts"]))]
    check("active counts", g["active_counts"], np.array(actives))
    check("woken", int(g["woken"]), st.woken)
    check("removed ids", g["log_id"], np.array([e["id"] for e in st.removed.log]))
    check("remaining ids", g["final_ids"], _np(st.ids))
    for f in ("level", "n_beg", "n_end", "doomed"):
        check(f"final {f}", g[f"final_{f}"], _np(getattr(st, f)))
    check("final x", g["final_x"], _np(st.x), rtol=1e-13, per_vector=True)
    check("final p", g["final_p"], _np(st.p), rtol=1e-11, per_vector=True)
    check("final u", g["final_u"], _np(st.u), rtol=1e-9)
    check("final energy", float(g["final_energy"]), blocks.ledger(st, bc)["energy"], rtol=1e-12)
