"""Block-timestep API of the reference (sim/blocks.py:455-787) on the GPU.

``initialise``, ``advance``, ``run``, ``ledger``, ``diagnostics`` and ``snapshot`` keep the
reference's names and meaning.  Each particle has its own power-of-two step on the int64 tick
timeline (tick = dt_max / 2^40); a system step goes to the earliest step end, flows every
particle's gravity, evaluates density for the active rows and their neighbours and forces for the
active rows, closes, chooses new levels (limiter and wake-up) and opens the next steps — all in
libnebula_b200.so on CUDA tensors.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, ops
from .accretion import RemovedLedger, record_removal
from .config import BlockConfig
from .coupled import make_params
from .device import ctx, dev_f64, dev_i64, ptr, stream, to_numpy

K_MAX = 40


@dataclass
class BlockState:
    n: int
    t0: float
    tick: float
    level: torch.Tensor
    n_beg: torch.Tensor
    n_end: torch.Tensor
    x_beg: torch.Tensor
    p_half: torch.Tensor
    u_half: torch.Tensor
    x: torch.Tensor
    p: torch.Tensor
    u: torch.Tensor
    mass: torch.Tensor
    h: torch.Tensor
    alpha: torch.Tensor
    a_hydro: torch.Tensor
    dudt: torch.Tensor
    rho: torch.Tensor
    omega: torch.Tensor
    vsig_max: torch.Tensor
    level_offset: torch.Tensor
    n_stop: int = 0
    active_counts: list = field(default_factory=list)
    particle_steps: int = 0
    woken: int = 0
    e_radiated: float = 0.0
    luminosity: torch.Tensor = None
    visc_heating: torch.Tensor = None
    nu: torch.Tensor = None
    c_s: torch.Tensor = None
    builds: int = 0
    reuses: int = 0
    timers: dict = field(default_factory=lambda: {"step": 0.0})
    # removal bookkeeping (sim/blocks.py:134-139): original ids, starting radius and |L|,
    # inward flag at the last active time, pericentre passed
    ids: torch.Tensor = None
    r0: torch.Tensor = None
    L0: torch.Tensor = None
    vr_neg: torch.Tensor = None
    passed_peri: torch.Tensor = None
    doomed: torch.Tensor = None  # next step ends beyond a removal radius (removal_sync)
    removed: RemovedLedger = field(default_factory=RemovedLedger)
    # parts of du/dt at each particle's last force evaluation and the heat budget since the
    # start, what each part of du/dt and the cooling added to u (sim/blocks.py:142-154)
    cond_heating: torch.Tensor = None
    disk_heating: torch.Tensor = None
    heat_visc: torch.Tensor = None
    heat_cond: torch.Tensor = None
    heat_disk: torch.Tensor = None
    heat_pdv: torch.Tensor = None
    heat_cool: torch.Tensor = None
    _params: object = field(default=None, repr=False)
    _rows: torch.Tensor = field(default=None, repr=False)

    @property
    def t(self) -> float:
        return self.t0 + self.n * self.tick

    def synced(self) -> bool:
        return bool(torch.all(self.n_beg == self.n))

    def numpy(self) -> dict:
        return {k: to_numpy(v) for k, v in self.__dict__.items() if isinstance(v, torch.Tensor)}


_FIELDS = ("x", "p", "u", "mass", "h", "alpha", "a_hydro", "dudt", "rho", "omega", "c_s",
           "vsig_max", "nu", "visc_heating", "level", "n_beg", "n_end", "level_offset", "x_beg",
           "p_half", "u_half", "luminosity", "cond_heating", "disk_heating", "heat_visc",
           "heat_cond", "heat_disk", "heat_pdv", "heat_cool")  # fmt: skip
HEAT_FIELDS = ("cond_heating", "disk_heating", "heat_visc", "heat_cond", "heat_disk", "heat_pdv",
               "heat_cool")


def _state_struct(st: BlockState) -> _lib.NbState:
    s = _lib.NbState()
    s.n = len(st.x)
    for name in _FIELDS:
        t = getattr(st, name)
        setattr(s, name, None if t is None else t.data_ptr())
    s.tick_n, s.n_stop, s.t0, s.tick = st.n, st.n_stop, st.t0, st.tick
    s.e_radiated = st.e_radiated
    s.particle_steps, s.woken = st.particle_steps, st.woken
    s.builds, s.reuses = st.builds, st.reuses
    return s


def _pull(st: BlockState, s: _lib.NbState) -> None:
    st.n = int(s.tick_n)
    st.e_radiated = s.e_radiated
    st.particle_steps, st.woken = int(s.particle_steps), int(s.woken)
    st.builds, st.reuses = int(s.builds), int(s.reuses)


def _params(st: BlockState, cfg: BlockConfig):
    if st._params is None:
        if cfg.respa:
            raise NotImplementedError("RESPA gravity sub-steps are not part of the CUDA SPH path")
        if not cfg.hydro:
            raise NotImplementedError("gravity-only block steps are not part of the CUDA SPH path")
        st._params = make_params(cfg.coupled, cfg.dt_max, cfg.limiter, cfg.max_gap)
    return st._params


def initialise(x, v, u, mass, h_guess, cfg: BlockConfig, t_stop: float, t0: float = 0.0,
               level_offset=None) -> BlockState:  # fmt: skip
    """sim/blocks.py:455-499: all particles start active at t0; first steps never pass t_stop."""
    cc = cfg.coupled
    hc = cc.hydro
    x = dev_f64(x)
    n = len(x)
    d = x.device
    z = lambda *s: torch.zeros((n, *s), dtype=torch.float64, device=d)  # noqa: E731
    zi = lambda: torch.zeros(n, dtype=torch.int64, device=d)  # noqa: E731
    p = ops.gn_p_from_v(x, dev_f64(v))
    u = dev_f64(u, (n,)).clone()
    tick = cfg.dt_max / 2.0**K_MAX
    if (t_stop - t0) / tick >= 2.0**62:
        raise ValueError("t_stop - t0 exceeds 2^62 ticks of dt_max / 2^40 (int64 tick timeline)")
    st = BlockState(
        n=0, t0=t0, tick=tick, level=zi(), n_beg=zi(), n_end=zi(), x_beg=x.clone(),
        p_half=p.clone(), u_half=u.clone(), x=x.clone(), p=p, u=u,
        mass=dev_f64(mass, (n,)).clone(), h=dev_f64(h_guess, (n,)).clone(),
        alpha=torch.full((n,), hc.alpha_init if hc.switch else hc.alpha_const, dtype=torch.float64, device=d),
        a_hydro=z(3), dudt=z(), rho=z(), omega=torch.ones(n, dtype=torch.float64, device=d),
        vsig_max=z(), level_offset=zi() if level_offset is None else dev_i64(level_offset),
        n_stop=int(round((t_stop - t0) / tick)), luminosity=z(), visc_heating=z(), nu=z(), c_s=z(),
    )  # fmt: skip
    for name in HEAT_FIELDS:
        setattr(st, name, z())
    st._rows = torch.empty(n, dtype=torch.int64, device=d)
    st.ids = torch.arange(n, dtype=torch.int64, device=d)
    st.r0 = torch.linalg.norm(st.x, dim=1)
    st.L0 = torch.linalg.norm(torch.linalg.cross(st.x, st.p, dim=1), dim=1)
    st.vr_neg = torch.sum(st.x * ops.gn_v_from_p(st.x, st.p), dim=1) < 0
    st.passed_peri = torch.zeros(n, dtype=torch.bool, device=d)
    st.doomed = torch.zeros(n, dtype=torch.bool, device=d)
    prm = _params(st, cfg)
    c = ctx()
    s = _state_struct(st)
    _lib.check(c, _lib.lib().nb_block_initialise(c, ctypes.byref(s), ctypes.byref(prm), stream()))
    _pull(st, s)
    if _removal(cfg) and cfg.removal_sync:  # sim/blocks.py:497-498
        _wake_for_removal(st, cfg, torch.arange(n, dtype=torch.int64, device=d))
    return st


def _removal(cfg: BlockConfig) -> bool:
    return cfg.r_acc is not None or cfg.r_escape is not None


def advance(st: BlockState, cfg: BlockConfig) -> torch.Tensor:
    """sim/blocks.py:502-563: one system step to the earliest step end; returns the active rows."""
    prm = _params(st, cfg)
    if _removal(cfg) and cfg.removal_sync:
        return _advance_sync(st, cfg, prm)
    t0 = time.perf_counter()
    c = ctx()
    s = _state_struct(st)
    _lib.check(c, _lib.lib().nb_block_advance(c, ctypes.byref(s), ctypes.byref(prm),
                                              ptr(st._rows), stream()))  # fmt: skip
    _pull(st, s)
    na = int(s.last_active)
    st.active_counts.append(na)
    rows = st._rows[:na].clone()
    if _removal(cfg):
        rows = _swallow_keep(st, cfg, rows)[0]
    st.timers["step"] += time.perf_counter() - t0
    return rows


def _advance_sync(st: BlockState, cfg: BlockConfig, prm) -> torch.Tensor:
    """sim/blocks.py:502-563 with removal_sync (module docstring of sim/blocks.py, Removal): the
    active particles inside r_acc or beyond r_escape are removed after the closing kicks, the
    forces of the remaining active particles are recomputed without them at the same predicted
    velocities and energies, then levels and openings, then the doomed particles' neighbours
    are cut to end their steps with theirs (sim/blocks.py:566-627)."""
    t0 = time.perf_counter()
    c = ctx()
    n = len(st.x)
    v_eval = torch.empty((n, 3), dtype=torch.float64, device=st.x.device)
    u_eval = torch.empty(n, dtype=torch.float64, device=st.x.device)
    s = _state_struct(st)
    _lib.check(c, _lib.lib().nb_block_advance_split(c, ctypes.byref(s), ctypes.byref(prm),
                                                    ptr(st._rows), ptr(v_eval), ptr(u_eval),
                                                    stream()))  # fmt: skip
    _pull(st, s)
    na = int(s.last_active)
    st.active_counts.append(na)
    rows, keep = _swallow_keep(st, cfg, st._rows[:na].clone())
    redo = 0
    if keep is not None:
        v_eval, u_eval = v_eval[keep].contiguous(), u_eval[keep].contiguous()
        redo = int(len(rows) > 0)
    s = _state_struct(st)
    _lib.check(c, _lib.lib().nb_block_finish(c, ctypes.byref(s), ctypes.byref(prm), len(rows),
                                             ptr(rows), redo, ptr(v_eval), ptr(u_eval),
                                             stream()))  # fmt: skip
    _pull(st, s)
    _wake_for_removal(st, cfg, rows)
    st.timers["step"] += time.perf_counter() - t0
    return rows


def _wake_for_removal(st: BlockState, cfg: BlockConfig, rows) -> None:
    """sim/blocks.py:593-627: flag the active particles whose gravity flow over the step just
    opened ends inside r_acc or beyond r_escape; the running steps of every neighbour of a
    flagged particle (and of active particles next to one still in its step) are cut to end
    with its step (on the device, over the cached lists)."""
    if len(rows) == 0:
        return
    length = (st.n_end[rows] - st.n_beg[rows]).to(torch.float64) * st.tick
    x_end, _, _ = ops.glf_step_many(st.x_beg[rows], st.p_half[rows], length)
    r = torch.linalg.norm(x_end, dim=1)
    doomed = torch.zeros(len(rows), dtype=torch.bool, device=r.device)
    if cfg.r_acc is not None:
        doomed |= r < cfg.r_acc
    if cfg.r_escape is not None:
        doomed |= r > cfg.r_escape
    st.doomed[rows] = doomed
    if not bool(torch.any(st.doomed)):
        return
    c = ctx()
    s = _state_struct(st)
    flags = st.doomed.to(torch.uint8).contiguous()
    _lib.check(c, _lib.lib().nb_block_wake_doomed(c, ctypes.byref(s), len(rows), ptr(rows),
                                                  ptr(flags), stream()))  # fmt: skip
    _pull(st, s)


def _gn_hamiltonian(x, p):
    """physics/gravity.py:92-102 for the few removed particles."""
    r = torch.linalg.norm(x, dim=1)
    a, c = (r - 2.0) / r, -2.0 * (r - 2.0) / r**4
    px = torch.sum(p * x, dim=1)
    return 0.5 * a * torch.sum(p * p, dim=1) + 0.5 * c * px**2 - 1.0 / r


def _swallow_keep(st: BlockState, cfg: BlockConfig, rows):
    """sim/blocks.py:673-719 (_swallow, _swallow_keep, _prune): the active rows' pericentre
    flags; those inside r_acc or beyond r_escape (their state true at their own step end) go into
    the removed ledger and out of every per-particle array.  The engine rebuilds its lists for
    the new particle count.  Returns the remaining rows, renumbered, and the mask of the kept
    particles (None when none was removed)."""
    rows = torch.sort(rows).values  # ascending, as the reference's rows (and so its log order)
    x, p = st.x[rows], st.p[rows]
    r = torch.linalg.norm(x, dim=1)
    vr = torch.sum(x * ops.gn_v_from_p(x, p), dim=1)
    turned = st.vr_neg[rows] & (vr > 0) & (r < 0.5 * st.r0[rows])
    st.passed_peri[rows] |= turned
    st.vr_neg[rows] = vr < 0
    none = torch.zeros(len(rows), dtype=torch.bool, device=r.device)
    acc = r < cfg.r_acc if cfg.r_acc is not None else none
    esc = r > cfg.r_escape if cfg.r_escape is not None else none
    gone_mask = acc | esc
    if not bool(torch.any(gone_mask)):
        return rows, None
    for mask, reason in ((acc, "accreted"), (esc, "escaped")):
        g = rows[mask]
        if len(g) == 0:
            continue
        xs, ps = st.x[g], st.p[g]
        h = lambda a: a.detach().cpu().numpy()  # noqa: E731
        record_removal(st.removed, st.t, h(st.ids[g]), h(st.mass[g]), h(_gn_hamiltonian(xs, ps)),
                       h(st.u[g]), h(torch.linalg.cross(xs, ps, dim=1)), h(ps),
                       h(torch.linalg.norm(xs, dim=1)), h(st.passed_peri[g]), h(st.L0[g]),
                       reason)  # fmt: skip
    n = len(st.x)
    keep = torch.ones(n, dtype=torch.bool, device=r.device)
    keep[rows[gone_mask]] = False
    for name, value in list(vars(st).items()):
        if isinstance(value, torch.Tensor) and value.shape[:1] == (n,):
            setattr(st, name, value[keep].contiguous())
    new_index = torch.cumsum(keep.to(torch.int64), 0) - 1
    return new_index[rows[keep[rows]]].contiguous(), keep


def run(st: BlockState, cfg: BlockConfig, t_end: float, callback=None) -> BlockState:
    """sim/blocks.py:722-739: advance until every particle is exactly at t_end."""
    prm = _params(st, cfg)
    n_end = int(round((t_end - st.t0) / st.tick))
    st.n_stop = n_end
    c = ctx()
    s = _state_struct(st)
    _lib.check(c, _lib.lib().nb_block_land(c, ctypes.byref(s), ctypes.byref(prm), stream()))
    if bool(torch.any(st.n_end > n_end)):
        raise ValueError("some particles' current steps already run past t_end")
    while st.n < n_end:
        advance(st, cfg)
        if callback is not None:
            callback(st)
    return st


def ledger(st: BlockState, cfg: BlockConfig) -> dict:
    """sim/blocks.py:742-758, the removed particles' totals included."""
    s = ops.ledger_sums(st.x, st.p, st.u, st.mass)
    rm = st.removed
    return {"energy": s["energy"] + rm.energy + st.e_radiated, "e_radiated": st.e_radiated,
            "abs_h": s["abs_h"], "angmom": np.asarray(s["angmom"]) + rm.angmom,
            "momentum": np.asarray(s["momentum"]) + rm.momentum, "mass": s["mass"] + rm.mass,
            "removed_mass": rm.mass, "removed_count": rm.count}  # fmt: skip


def diagnostics(st: BlockState) -> dict:
    """sim/blocks.py:761-774."""
    counts = np.asarray(st.active_counts)
    lv = to_numpy(st.level)
    return {
        "t": st.t,
        "level_histogram": np.bincount(lv, minlength=int(lv.max()) + 1),
        "system_steps": len(counts),
        "particle_steps": st.particle_steps,
        "mean_active": float(counts.mean()) if len(counts) else 0.0,
        "woken": st.woken,
        "timers": dict(st.timers),
        "list_builds": st.builds,
        "list_reuses": st.reuses,
    }


def snapshot(st: BlockState, cfg: BlockConfig, t: float):
    """sim/blocks.py:777-787: positions and momenta of every particle at time t."""
    n_t = (t - st.t0) / st.tick
    nb = st.n_beg.to(torch.float64)
    ne = st.n_end.to(torch.float64)
    if bool(torch.any(n_t < nb - 1e-6)) or bool(torch.any(n_t > ne + 1e-6)):
        raise ValueError("snapshot time outside some particle's current step")
    s = torch.clamp((t - st.t0) - st.n_beg.to(torch.float64) * st.tick, min=0.0)
    x, p_flow, _ = ops.glf_step_many(st.x_beg, st.p_half, s)
    lag = s - 0.5 * (st.n_end - st.n_beg).to(torch.float64) * st.tick
    return x, p_flow + lag[:, None] * st.a_hydro
