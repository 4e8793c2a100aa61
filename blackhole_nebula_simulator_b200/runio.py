"""Run folders, manifests, checkpoints and float32 snapshots (sim/runio.py of the reference),
for states held in device memory.

A run lives in <runs>/<name>/ and is never overwritten; manifest.json records the configuration,
library versions, machine and start/end times.  checkpoint.pkl holds the whole float64 state
(device tensors copied to host arrays) and is written atomically; ``blocks_payload`` /
``restore_blocks`` turn a BlockState into such a payload and back onto the device.  Snapshots
for plots and rendering are float32 npz files, converted on the device before the copy.
"""

from __future__ import annotations

import json
import pickle
import platform
import time
from dataclasses import asdict, fields, is_dataclass
from pathlib import Path

import numpy as np
import torch


def _jsonable(obj):
    """sim/runio.py:45-55."""
    if is_dataclass(obj):
        return {k: _jsonable(v) for k, v in asdict(obj).items()}
    if isinstance(obj, dict):
        return {k: _jsonable(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_jsonable(v) for v in obj]
    if isinstance(obj, np.generic):
        return obj.item()
    if isinstance(obj, float) and not np.isfinite(obj):
        return str(obj)
    return obj


def _versions() -> dict:
    return {"python": platform.python_version(), "numpy": np.__version__,
            "torch": torch.__version__, "cuda": torch.version.cuda}  # fmt: skip


def new_run(runs: Path, name: str, config: dict) -> Path:
    """sim/runio.py:58-72: create <runs>/<name>/ (refuses an existing one) and its manifest."""
    folder = Path(runs) / name
    folder.mkdir(parents=True, exist_ok=False)
    (folder / "snapshots").mkdir()
    manifest = {
        "name": name, "config": _jsonable(config), "versions": _versions(),
        "machine": {"platform": platform.platform(), "processor": platform.processor(),
                    "machine": platform.machine()},
        "seed": None, "start": time.strftime("%Y-%m-%d %H:%M:%S %Z"), "end": None, "resumed": [],
    }  # fmt: skip
    (folder / "manifest.json").write_text(json.dumps(manifest, indent=2))
    return folder


def update_manifest(folder: Path, **fields_) -> None:
    """sim/runio.py:75-83."""
    path = Path(folder) / "manifest.json"
    manifest = json.loads(path.read_text())
    for k, v in fields_.items():
        if k == "resumed":
            manifest["resumed"].append({"time": v})
        else:
            manifest[k] = _jsonable(v)
    path.write_text(json.dumps(manifest, indent=2))


def save_checkpoint(folder: Path, payload) -> None:
    """sim/runio.py:86-90: pickle ``payload`` atomically."""
    tmp = Path(folder) / "checkpoint.tmp"
    tmp.write_bytes(pickle.dumps(payload, protocol=pickle.HIGHEST_PROTOCOL))
    tmp.replace(Path(folder) / "checkpoint.pkl")


def load_checkpoint(folder: Path):
    return pickle.loads((Path(folder) / "checkpoint.pkl").read_bytes())


def save_snapshot(folder: Path, index: int, t: float, **arrays) -> None:
    """sim/runio.py:97-102: float32 copy of per-particle arrays (device tensors are converted on
    the device, then copied); integer arrays are kept as they are."""
    out = {}
    for k, v in arrays.items():
        if isinstance(v, torch.Tensor):
            v = (v.to(torch.float32) if v.is_floating_point() else v).detach().cpu().numpy()
        a = np.asarray(v)
        out[k] = a.astype(np.float32) if np.issubdtype(a.dtype, np.floating) else a
    np.savez_compressed(Path(folder) / "snapshots" / f"snap_{index:05d}.npz", t=np.float64(t), **out)


def blocks_payload(st) -> dict:
    """The whole block state as host arrays and scalars (the checkpoint payload)."""
    out = {}
    for f in fields(st):
        if f.name.startswith("_"):
            continue
        v = getattr(st, f.name)
        out[f.name] = v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else v
    return out


def restore_blocks(payload: dict, device=None):
    """A BlockState on the device from ``blocks_payload`` output; the engine rebuilds its lists
    at the next step (as the reference does after loading a checkpoint without its cache)."""
    from .blocks import HEAT_FIELDS, BlockState
    from .device import require_cuda

    dev = device or require_cuda()
    kw = {}
    for f in fields(BlockState):
        if f.name.startswith("_") or f.name not in payload:
            continue
        v = payload[f.name]
        kw[f.name] = torch.as_tensor(v, device=dev).clone() if isinstance(v, np.ndarray) else v
    st = BlockState(**kw)
    n = len(st.x)
    # outputs and budgets absent from an older checkpoint start at zero from the resume
    # (sim/blocks.py:172-188)
    for name in ("luminosity", "visc_heating", "nu", "c_s") + HEAT_FIELDS:
        if getattr(st, name) is None:
            setattr(st, name, torch.zeros(n, dtype=torch.float64, device=dev))
    st._rows = torch.empty(n, dtype=torch.int64, device=dev)
    return st
