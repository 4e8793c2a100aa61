"""Run folders, manifests, checkpoints and float32 snapshots (sim/runio.py of the reference),
for states held in device memory.

A run lives in <runs>/<name>/ and is never overwritten; manifest.json records the configuration,
library versions, machine and start/end times.  checkpoint.pkl holds the whole float64 state
(device tensors copied to host arrays) and is written atomically; ``blocks_payload`` /
``restore_blocks`` turn a BlockState into such a payload and back onto the device.  Snapshots
for plots and rendering are float32 npz files, converted on the device before the copy.
"""

from __future__ import annotations

import dataclasses
import json
import math
import os
import pickle
import platform
import time
from dataclasses import fields
from pathlib import Path

import numpy as np
import torch

MANIFEST = "manifest.json"
CHECKPOINT = "checkpoint.pkl"
CHECKPOINT_TMP = "checkpoint.tmp"  # the partial file a crash may leave; never read


def _plain(obj):
    """A JSON-ready copy of ``obj``: dataclasses become dicts, tuples lists, NumPy scalars and
    arrays Python values, and non-finite floats their text ("inf", "nan"), which strict JSON
    cannot hold."""
    if dataclasses.is_dataclass(obj) and not isinstance(obj, type):
        obj = {f.name: getattr(obj, f.name) for f in fields(obj)}
    if isinstance(obj, np.ndarray):
        obj = obj.tolist()
    elif isinstance(obj, np.generic):
        obj = obj.item()
    if isinstance(obj, dict):
        return {key: _plain(val) for key, val in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_plain(val) for val in obj]
    if isinstance(obj, float) and not math.isfinite(obj):
        return repr(obj)
    return obj


def _replace_atomically(path: Path, data: bytes, tmp_name: str | None = None) -> None:
    """Write ``data`` beside ``path`` and rename it over ``path``: a reader sees the old file or
    the new one, never a half-written one."""
    tmp = path.with_name(tmp_name or f".{path.name}.tmp")
    with open(tmp, "wb") as f:
        f.write(data)
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)


def _manifest_write(folder: Path, manifest: dict) -> None:
    _replace_atomically(Path(folder) / MANIFEST, json.dumps(manifest, indent=2).encode())


def _environment() -> dict:
    """Library versions and the machine the run started on."""
    versions = {"python": platform.python_version(), "numpy": np.__version__,
                "torch": torch.__version__, "cuda": torch.version.cuda}  # fmt: skip
    machine = {key: getattr(platform, key)() for key in ("platform", "processor", "machine")}
    return {"versions": versions, "machine": machine}


def new_run(runs: Path, name: str, config: dict) -> Path:
    """Create the run folder <runs>/<name>/ with its snapshots/ folder and manifest (keys as in
    sim/runio.py:58-72: name, config, versions, machine, seed, start, end, resumed).  An existing
    folder is never reused: FileExistsError."""
    folder = Path(runs) / name
    folder.mkdir(parents=True, exist_ok=False)
    (folder / "snapshots").mkdir()
    env = _environment()
    _manifest_write(folder, {
        "name": name, "config": _plain(config), "versions": env["versions"],
        "machine": env["machine"], "seed": None, "start": time.strftime("%Y-%m-%d %H:%M:%S %Z"),
        "end": None, "resumed": [],
    })  # fmt: skip
    return folder


def update_manifest(folder: Path, **changes) -> None:
    """Set manifest keys; ``resumed=t`` appends a resume record {"time": t} instead."""
    manifest = json.loads((Path(folder) / MANIFEST).read_text())
    resumed = changes.pop("resumed", None)
    if resumed is not None:
        manifest.setdefault("resumed", []).append({"time": _plain(resumed)})
    manifest.update({key: _plain(val) for key, val in changes.items()})
    _manifest_write(folder, manifest)


def save_checkpoint(folder: Path, payload) -> None:
    """The whole float64 state as a pickle in <folder>/checkpoint.pkl, replaced atomically
    through checkpoint.tmp (the reference's file names, sim/runio.py:86-90)."""
    data = pickle.dumps(payload, protocol=pickle.HIGHEST_PROTOCOL)
    _replace_atomically(Path(folder) / CHECKPOINT, data, CHECKPOINT_TMP)


def load_checkpoint(folder: Path):
    """The payload of the last completed ``save_checkpoint``."""
    with open(Path(folder) / CHECKPOINT, "rb") as f:
        return pickle.load(f)


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
