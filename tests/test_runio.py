"""Run folders, manifests, checkpoints and float32 snapshots (sim/runio.py of the reference)."""

import json

import numpy as np
import pytest

from blackhole_nebula_simulator_b200 import runio
from tests.conftest import check


def test_run_folder_manifest_and_snapshot(tmp_path):
    folder = runio.new_run(tmp_path, "r1", {"dt_max": 64.0, "r_acc": None, "eta": float("inf")})
    with pytest.raises(FileExistsError):
        runio.new_run(tmp_path, "r1", {})
    runio.update_manifest(folder, end="now", resumed=12.5)
    man = json.loads((folder / "manifest.json").read_text())
    check("manifest config", 64.0, man["config"]["dt_max"])
    check("non-finite values as text", "inf", man["config"]["eta"])
    check("resumed entries", 1, len(man["resumed"]))
    x = np.random.default_rng(0).normal(size=(10, 3))
    ids = np.arange(10)
    runio.save_snapshot(folder, 3, 1.25, x=x, ids=ids)
    snap = np.load(folder / "snapshots" / "snap_00003.npz")
    check("snapshot positions are float32", True, snap["x"].dtype == np.float32)
    check("snapshot positions", x.astype(np.float32), snap["x"])
    check("integer arrays kept", ids, snap["ids"])
    check("time kept in float64", 1.25, float(snap["t"]))


def test_checkpoint_round_trip(tmp_path):
    payload = {"x": np.arange(6.0).reshape(2, 3), "n": 7, "removed": {"mass": 1.5}}
    runio.save_checkpoint(tmp_path, payload)
    back = runio.load_checkpoint(tmp_path)
    check("arrays", payload["x"], back["x"])
    check("scalars", 7, back["n"])
    check("no temporary file left", False, (tmp_path / "checkpoint.tmp").exists())


@pytest.mark.gpu
def test_block_state_checkpoint_resumes(tmp_path):
    """A block run checkpointed after 4 steps and resumed on the device continues as the
    uninterrupted run (levels and tick counters exactly, state to the block-step tolerances:
    the resumed run rebuilds its neighbour lists)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from blackhole_nebula_simulator_b200 import blocks
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig, HydroConfig
    from tests.conftest import golden

    g = golden("blocks.npz")
    hc = HydroConfig(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                     conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    bc = BlockConfig(coupled=CoupledConfig(hydro=hc, cooling_beta=230.0), dt_max=64.0)
    st = blocks.initialise(g["x0"], g["v0"], g["u0"], g["mass"], g["h0"], bc, t_stop=1e6,
                           level_offset=g["level_offset"])  # fmt: skip
    for _ in range(4):
        blocks.advance(st, bc)
    runio.save_checkpoint(tmp_path, runio.blocks_payload(st))
    a = [len(blocks.advance(st, bc)) for _ in range(6)]
    rs = runio.restore_blocks(runio.load_checkpoint(tmp_path))
    b = [len(blocks.advance(rs, bc)) for _ in range(6)]
    check("active counts", np.array(a), np.array(b))
    for f in ("level", "n_beg", "n_end"):
        check(f, st.__getattribute__(f).cpu().numpy(), rs.__getattribute__(f).cpu().numpy())
    check("x", st.x.cpu().numpy(), rs.x.cpu().numpy(), rtol=1e-13, per_vector=True)
    # the resumed run rebuilds its lists: sums in another curve order, hence rounding
    check("p", st.p.cpu().numpy(), rs.p.cpu().numpy(), rtol=1e-10, per_vector=True)
    check("u", st.u.cpu().numpy(), rs.u.cpu().numpy(), rtol=1e-9)
    check("energy", blocks.ledger(st, bc)["energy"], blocks.ledger(rs, bc)["energy"], rtol=1e-12)
