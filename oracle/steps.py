"""Shared-step and block-step drivers (TEST INFRASTRUCTURE).

Restates the reference's step logic on top of the C kernels:
  * coupled: sim/coupled.py:104-270 (velocity, p_from_v, hamiltonian, gravity_flow, _hydro,
    initialise, stable_dt, step, ledger);
  * blocks:  sim/blocks.py:192-563, 722-787 (_density_touched, _hydro_rows, wanted_dt,
    _choose_levels, _land, _wake, _cut_steps, _cut_to, _open, initialise, advance, run, ledger,
    diagnostics, snapshot) and sim/timesteps.py:21-59 (ticks, level_for_dt, allowed_level).
Only the options of the CUDA path are restated: GN hole, ideal gas (or, without cooling, the
radiation limit and gas + radiation), constant alpha or the Cullen-Dehnen switch, optional
velocity reconstruction, conductivity and disc viscosity, beta or bremsstrahlung cooling, no
accretion and escape radii (with or without removal_sync), the per-particle heat budget, no
RESPA.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field, replace

import numpy as np

from . import cooling as ocool
from . import native
from .eos import eos_state
from .sph import C_NORM, KERNEL_IDS, compute_density

K_MAX = 40
C_VISC = 0.25
C_COOL = 0.25  # bremsstrahlung time-step factor: dt <= C_COOL u / |du/dt_cool| (own criterion)


# --------------------------------------------------------------------------- GN helpers
def _r(x):
    return np.sqrt(np.sum(x * x, axis=-1))


def gn_p_from_v(x, v):
    """physics/gravity.py:66-77."""
    r = _r(x)[..., None]
    f = r / (r - 2.0)
    g = 2.0 * r / (r - 2.0) ** 2
    rdot = np.sum(x * v, axis=-1, keepdims=True) / r
    return f * v + g * rdot * x / r


def gn_hamiltonian(x, p):
    """physics/gravity.py:92-102."""
    r = _r(x)
    a, c = (r - 2.0) / r, -2.0 * (r - 2.0) / r**4
    px = np.sum(p * x, axis=-1)
    return 0.5 * a * np.sum(p * p, axis=-1) + 0.5 * c * px**2 - 1.0 / r


def ledger_sums(mass, x, p, u, e_rad):
    """sim/coupled.py:261-270."""
    h = gn_hamiltonian(x, p)
    return {
        "energy": float(np.sum(mass * (h + u))) + e_rad,
        "e_radiated": e_rad,
        "abs_h": float(np.sum(mass * np.abs(h))),
        "angmom": np.sum(mass[:, None] * np.cross(x, p), axis=0),
        "momentum": np.sum(mass[:, None] * p, axis=0),
        "mass": float(np.sum(mass)),
    }


def _eos(hc, rho, u):
    """sim/hydro.py:119-139: ideal gas, radiation limit or gas + radiation."""
    return eos_state(hc, rho, u)


def _kid(hc):
    return KERNEL_IDS[hc.kernel], C_NORM[KERNEL_IDS[hc.kernel]]


def _cool(cc, u_half, rho, dt, r_mid):
    """The cooling law at mid-step: beta-cooling (physics/cooling.py) or bremsstrahlung."""
    if cc.cooling == "brems":
        return ocool.brems_cool(u_half, rho, dt, ocool.brems_constants(cc.hydro.gamma,
                                                                      t_floor=cc.t_floor))
    floor = np.full(len(u_half), ocool.ideal_floor_energy(cc.t_floor, cc.hydro.gamma))
    return ocool.beta_cool(u_half, floor, dt, ocool.cooling_time(r_mid, cc.cooling_beta))


def _cooling_on(cc):
    return cc.cooling == "brems" or math.isfinite(cc.cooling_beta)


# --------------------------------------------------------------------------- shared step
@dataclass
class GasState:
    t: float
    x: np.ndarray
    p: np.ndarray
    u: np.ndarray
    mass: np.ndarray
    h: np.ndarray
    alpha: np.ndarray
    a_hydro: np.ndarray = None
    dudt: np.ndarray = None
    rho: np.ndarray = None
    c_s: np.ndarray = None
    vsig_max: np.ndarray = None
    neighbour_cache: object = None
    e_radiated: float = 0.0
    visc_heating: np.ndarray = None
    nu: np.ndarray = None


def _switch_update(hc, alpha, h, cs, div, curl, ddiv, dt_alpha):
    """physics/viscosity.py:83-113 (balsara_xi, alpha_local, decay_time, alpha_update)."""
    d2, c2 = div**2, curl**2
    with np.errstate(invalid="ignore", divide="ignore"):
        xi = np.where(d2 + c2 > 0, d2 / (d2 + c2), 0.0)
    a_loc = np.minimum(10.0 * h * h * (xi * np.maximum(-ddiv, 0.0)) / (cs * cs), 1.0)
    tau = h / (0.1 * cs)
    decayed = (alpha + a_loc * dt_alpha / tau) / (1.0 + dt_alpha / tau)
    return np.where(a_loc > alpha, a_loc, decayed)


def _shock_args(hc):
    """The reconstruction settings of HydroConfig.shock() (sim/hydro.py:92-98)."""
    return dict(closeness=hc.recon_closeness, eta_crit=1.0 / hc.eta, eta_fold=0.2,
                gate=hc.recon_gate)  # fmt: skip


def _shared_hydro(st: GasState, cc, v, reuse=True, dt_alpha=0.0, a_prev=None) -> GasState:
    """sim/coupled.py:145-195 for the supported options."""
    hc = cc.hydro
    d = compute_density(st.x, st.mass, st.h, kernel_name=hc.kernel, eta=hc.eta, h_max=hc.h_max,
                        cache=st.neighbour_cache, skin=hc.skin, reuse=reuse)  # fmt: skip
    p_gas, cs = _eos(hc, d.rho, st.u)
    nb = native.tighten(d.neighbours, st.x, d.h)
    kid, cn = _kid(hc)
    alpha = st.alpha
    if hc.viscosity and hc.switch and dt_alpha > 0:
        a0 = np.zeros_like(st.x) if a_prev is None else a_prev
        div, curl, ddiv = native.gradients(st.x, v, a0, st.mass, d.h, nb, kid, cn)
        alpha = _switch_update(hc, alpha, d.h, cs, div, curl, ddiv, dt_alpha)
    elif hc.viscosity and not hc.switch:
        alpha = np.full(len(st.x), hc.alpha_const)
    recon = hc.reconstruction and hc.viscosity
    grad_v = native.velocity_gradients(st.x, v, st.mass, d.h, nb, kid, cn) if recon else None
    acc, dudt, vsig, vh, _ = native.forces(
        st.x, v, st.mass, d.h, d.rho, d.omega, p_gas, nb, kid, cn,
        u=st.u if hc.conductivity else None, c_s=cs if hc.viscosity else None,
        alpha=alpha if hc.viscosity else None, beta=hc.beta, alpha_u=hc.alpha_u,
        cond_signal=hc.conductivity_signal, grad_v=grad_v, **_shock_args(hc),
    )  # fmt: skip
    nu = None
    if hc.disc_alpha_av > 0:
        a_d, u_d = native.disc_forces(st.x, v, st.mass, d.h, d.rho, d.omega, cs, hc.disc_alpha_av,
                                      nb, kid, cn)  # fmt: skip
        acc, dudt = acc + a_d, dudt + u_d
        nu = hc.disc_alpha_av * cs * d.h / 10.0
    return replace(st, h=d.h, alpha=alpha, a_hydro=acc, dudt=dudt, rho=d.rho, c_s=cs,
                   vsig_max=vsig if hc.viscosity else cs, neighbour_cache=d.cache,
                   visc_heating=vh, nu=nu)  # fmt: skip


def coupled_initialise(x, v, u, mass, h_guess, cc, t=0.0, reuse=True) -> GasState:
    """sim/coupled.py:198-210."""
    x = np.array(x, float)
    n = len(x)
    p = gn_p_from_v(x, np.asarray(v, float))
    hc = cc.hydro
    st = GasState(t, x, p, np.array(u, float) * np.ones(n), np.array(mass, float) * np.ones(n),
                  np.array(h_guess, float) * np.ones(n),
                  np.full(n, hc.alpha_init if hc.switch else hc.alpha_const))  # fmt: skip
    return _shared_hydro(st, cc, native.gn_v_from_p(x, p), reuse)


def coupled_stable_dt(st: GasState, cc) -> float:
    """sim/coupled.py:213-226."""
    hc = cc.hydro
    dt = hc.courant * np.min(st.h / st.vsig_max)
    amag = np.linalg.norm(st.a_hydro, axis=1)
    if np.any(amag > 0):
        dt = min(dt, hc.c_force * np.min(np.sqrt(st.h[amag > 0] / amag[amag > 0])))
    if st.nu is not None:
        with np.errstate(divide="ignore"):
            dt = min(dt, float(np.min(np.where(st.nu > 0, C_VISC * st.h**2 / st.nu, np.inf))))
    r = np.linalg.norm(st.x, axis=1)
    dt = min(dt, cc.eta_orb * np.min(r**1.5))
    return float(min(dt, float(np.min(cooling_dt(cc, st.u, st.rho)))))


def coupled_step(st: GasState, cc, dt: float, reuse=True) -> GasState:
    """sim/coupled.py:238-258."""
    p_half = st.p + 0.5 * dt * st.a_hydro
    u_half = st.u + 0.5 * dt * st.dudt
    x1, p_flow, _ = native.glf_step_many(st.x, p_half, dt)
    e_rad = st.e_radiated
    if _cooling_on(cc):
        r_mid = 0.5 * (np.linalg.norm(st.x, axis=1) + np.linalg.norm(x1, axis=1))
        u_cool = _cool(cc, u_half, st.rho, dt, r_mid)
        e_rad += float(np.sum(st.mass * (u_half - u_cool)))
        u_half = u_cool
    p_pred = p_flow + 0.5 * dt * st.a_hydro
    pred = replace(st, t=st.t + dt, x=x1, p=p_flow, u=u_half + 0.5 * dt * st.dudt)
    new = _shared_hydro(pred, cc, native.gn_v_from_p(x1, p_pred), reuse, dt, st.a_hydro)
    return replace(new, p=p_flow + 0.5 * dt * new.a_hydro, u=u_half + 0.5 * dt * new.dudt,
                   e_radiated=e_rad)  # fmt: skip


def coupled_ledger(st: GasState, cc) -> dict:
    return ledger_sums(st.mass, st.x, st.p, st.u, st.e_radiated)


# --------------------------------------------------------------------------- timeline
def ticks(level):
    """sim/timesteps.py:21-23."""
    return np.left_shift(np.int64(1), (K_MAX - np.asarray(level, np.int64)))


def level_for_dt(dt_wanted, dt_max):
    """sim/timesteps.py:26-39."""
    dt_wanted = np.asarray(dt_wanted, float)
    if np.any(~(dt_wanted > 0)):
        raise ValueError("time steps must be positive")
    k = np.ceil(np.log2(dt_max / dt_wanted) - 1e-12).astype(np.int64)
    k = np.maximum(k, 0)
    k = k + (dt_max / np.exp2(k) > dt_wanted)
    if np.any(k > K_MAX):
        raise ValueError(f"time step needs more than K_MAX = {K_MAX} halvings of dt_max")
    return k


def allowed_level(n, current, wanted):
    """sim/timesteps.py:47-59."""
    current = np.asarray(current, np.int64)
    wanted = np.asarray(wanted, np.int64)
    new = np.where(wanted >= current, wanted, current)
    for i in np.flatnonzero(wanted < current):
        for k in range(int(wanted[i]), int(current[i])):
            if np.int64(n) % ticks(k) == 0:
                new[i] = k
                break
    return new


# --------------------------------------------------------------------------- block steps
@dataclass
class BlockState:
    n: int
    t0: float
    tick: float
    level: np.ndarray
    n_beg: np.ndarray
    n_end: np.ndarray
    x_beg: np.ndarray
    p_half: np.ndarray
    u_half: np.ndarray
    x: np.ndarray
    p: np.ndarray
    u: np.ndarray
    mass: np.ndarray
    h: np.ndarray
    alpha: np.ndarray
    a_hydro: np.ndarray
    dudt: np.ndarray
    rho: np.ndarray
    omega: np.ndarray
    vsig_max: np.ndarray
    level_offset: np.ndarray
    n_stop: int = 0
    neighbour_cache: object = None
    active_counts: list = field(default_factory=list)
    particle_steps: int = 0
    woken: int = 0
    e_radiated: float = 0.0
    luminosity: np.ndarray = None
    nu: np.ndarray = None
    timers: dict = field(default_factory=lambda: {"flow": 0.0, "hydro": 0.0, "levels": 0.0})
    ids: np.ndarray = None  # original particle numbers
    r0: np.ndarray = None  # starting radius
    L0: np.ndarray = None  # starting |angular momentum|
    vr_neg: np.ndarray = None  # radial velocity < 0 at the last active time
    passed_peri: np.ndarray = None  # has turned outward near the hole
    doomed: np.ndarray = None  # next step ends beyond a removal radius (removal_sync)
    removed: "RemovedLedger" = None
    # parts of du/dt at each particle's last force evaluation, and the heat budget since the
    # start: what each part of du/dt and the cooling added to u (sim/blocks.py:142-154)
    visc_heating: np.ndarray = None
    cond_heating: np.ndarray = None
    disk_heating: np.ndarray = None
    heat_visc: np.ndarray = None
    heat_cond: np.ndarray = None
    heat_disk: np.ndarray = None
    heat_pdv: np.ndarray = None
    heat_cool: np.ndarray = None

    @property
    def t(self):
        return self.t0 + self.n * self.tick


def _density_touched(st: BlockState, hc, rows, reuse=True):
    """sim/blocks.py:217-239."""
    n = len(st.x)
    cache = st.neighbour_cache
    todo = np.arange(n) if cache is None else native.with_neighbours(cache.neighbours, rows, n)
    done = np.zeros(n, bool)
    for _ in range(8):
        d = compute_density(st.x, st.mass, st.h, kernel_name=hc.kernel, eta=hc.eta,
                            h_max=hc.h_max, cache=st.neighbour_cache, skin=hc.skin, rows=todo,
                            reuse=reuse)  # fmt: skip
        st.neighbour_cache = d.cache
        st.h[todo], st.rho[todo], st.omega[todo] = d.h, d.rho, d.omega
        done[todo] = True
        nb = native.tighten(d.neighbours, st.x, st.h, rows=rows)
        need = native.with_neighbours(nb, rows, n)
        todo = need[~done[need]]
        if len(todo) == 0:
            return nb
    raise RuntimeError("neighbour set of the active particles did not settle")


def _hydro_rows(st: BlockState, bc, rows, v, u, reuse=True, dt_alpha=None, a_prev=None):
    """sim/blocks.py:242-315 for the supported options."""
    hc = bc.coupled.hydro
    if np.any(u <= 0):
        raise FloatingPointError(f"non-positive internal energy at {int(np.sum(u <= 0))} particles")
    nb = _density_touched(st, hc, rows, reuse)
    touched = native.with_neighbours(nb, rows, len(st.x))
    p_gas, cs = np.full(len(st.x), np.nan), np.full(len(st.x), np.nan)
    p_gas[touched], cs[touched] = _eos(hc, st.rho[touched], u[touched])
    kid, cn = _kid(hc)
    if hc.viscosity and hc.switch and dt_alpha is not None and np.any(dt_alpha > 0):
        div, curl, ddiv = native.gradients(st.x, v, a_prev, st.mass, st.h, nb, kid, cn, rows=rows)
        st.alpha[rows] = _switch_update(hc, st.alpha[rows], st.h[rows], cs[rows], div, curl, ddiv,
                                        dt_alpha)  # fmt: skip
    elif hc.viscosity and not hc.switch:
        st.alpha[rows] = hc.alpha_const
    grad_v = None
    if hc.reconstruction and hc.viscosity:
        # the touched particles' gradients from the untightened cached lists (sim/blocks.py:271-278)
        grad_v = native.velocity_gradients(st.x, v, st.mass, st.h, st.neighbour_cache.neighbours,
                                           kid, cn, rows=touched)  # fmt: skip
    acc, dudt, vsig, vh, ch = native.forces(
        st.x, v, st.mass, st.h, st.rho, st.omega, p_gas, nb, kid, cn,
        u=u if hc.conductivity else None, c_s=cs if hc.viscosity else None,
        alpha=st.alpha if hc.viscosity else None, beta=hc.beta, alpha_u=hc.alpha_u,
        cond_signal=hc.conductivity_signal, rows=rows, grad_v=grad_v, **_shock_args(hc),
    )  # fmt: skip
    if hc.disc_alpha_av > 0:
        a_d, u_d = native.disc_forces(st.x, v, st.mass, st.h, st.rho, st.omega, cs,
                                      hc.disc_alpha_av, nb, kid, cn, rows=rows)  # fmt: skip
        acc, dudt = acc + a_d, dudt + u_d
        st.disk_heating[rows] = u_d
        st.nu[rows] = hc.disc_alpha_av * cs[rows] * st.h[rows] / 10.0
    st.a_hydro[rows] = acc
    st.dudt[rows] = dudt
    st.vsig_max[rows] = vsig if hc.viscosity else cs[rows]
    st.visc_heating[rows] = vh
    st.cond_heating[rows] = ch
    return nb


def _add_heat(st: BlockState, rows, dt):
    """sim/blocks.py:434-440: the kick u += dt du/dt of ``rows`` split into its parts."""
    visc, cond, disk = st.visc_heating[rows], st.cond_heating[rows], st.disk_heating[rows]
    st.heat_visc[rows] += dt * visc
    st.heat_cond[rows] += dt * cond
    st.heat_disk[rows] += dt * disk
    st.heat_pdv[rows] += dt * (st.dudt[rows] - visc - cond - disk)


def wanted_dt(st: BlockState, bc, rows):
    """sim/blocks.py:318-334."""
    cc = bc.coupled
    hc = cc.hydro
    h = st.h[rows]
    dt = hc.courant * h / st.vsig_max[rows]
    amag = np.linalg.norm(st.a_hydro[rows], axis=1)
    with np.errstate(divide="ignore"):
        dt = np.minimum(dt, np.where(amag > 0, hc.c_force * np.sqrt(h / amag), np.inf))
        nu = st.nu[rows]
        dt = np.minimum(dt, np.where(nu > 0, C_VISC * h**2 / nu, np.inf))
    dt = np.minimum(dt, cc.eta_orb * np.linalg.norm(st.x[rows], axis=1) ** 1.5)
    return np.minimum(dt, cooling_dt(cc, st.u[rows], st.rho[rows]))


def cooling_dt(cc, u, rho):
    """Bremsstrahlung time-step limit C_COOL u / |du/dt| for gas above the floor (inf elsewhere;
    beta-cooling is exact at any step and needs none, as in the reference)."""
    if cc.cooling != "brems":
        return np.full(len(u), np.inf)
    consts = ocool.brems_constants(cc.hydro.gamma, t_floor=cc.t_floor)
    rate = np.abs(ocool.brems_rate(u, rho, consts))
    hot = (consts[0] * u > consts[4]) & (rate > 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(hot, C_COOL * u / rate, np.inf)


def _land(st: BlockState, k):
    """sim/blocks.py:383-393."""
    if st.n >= st.n_stop:
        return k
    while True:
        over = st.n + ticks(np.minimum(k, K_MAX)) > st.n_stop
        if not np.any(over):
            return k
        k = np.where(over, k + 1, k)


def _cut_to(st: BlockState, j, end_new, level):
    """sim/blocks.py:420-431 (without the RESPA bookkeeping)."""
    st.level[j] = level
    d_len = (end_new - st.n_end[j]) * st.tick
    st.p_half[j] += 0.5 * d_len[:, None] * st.a_hydro[j]
    st.u_half[j] += 0.5 * d_len * st.dudt[j]
    _add_heat(st, j, 0.5 * d_len)
    st.n_end[j] = end_new
    st.woken += len(j)


def _wake(st: BlockState, bc, rows, nb):
    """sim/blocks.py:396-417."""
    need = np.full(len(st.level), -1, np.int64)
    native.wake_targets(st.level, rows, nb, bc.max_gap, need)
    inactive = st.n_end > st.n
    j = np.flatnonzero(inactive & (need > st.level))
    if len(j) == 0:
        return
    t_new = ticks(need[j])
    end_new = (st.n // t_new + 1) * t_new
    st.level[j] = need[j]
    cut = end_new < st.n_end[j]
    _cut_to(st, j[cut], end_new[cut], need[j[cut]])


def _choose_levels(st: BlockState, bc, rows, nb):
    """sim/blocks.py:367-380."""
    k = level_for_dt(wanted_dt(st, bc, rows), bc.dt_max) + st.level_offset[rows]
    k = allowed_level(st.n, st.level[rows], k)
    level = st.level.copy()
    level[rows] = k
    if bc.limiter:
        native.limit_rows(level, rows, nb, bc.max_gap)
    level[rows] = _land(st, level[rows])
    if np.any(level[rows] > K_MAX):
        raise ValueError(f"a particle needs a level beyond K_MAX = {K_MAX} (investigate it)")
    st.level = level
    if bc.limiter:
        _wake(st, bc, rows, nb)


def _open(st: BlockState, rows):
    """sim/blocks.py:443-452."""
    length = ticks(st.level[rows]) * st.tick
    st.n_beg[rows] = st.n
    st.n_end[rows] = st.n + ticks(st.level[rows])
    st.x_beg[rows] = st.x[rows]
    st.p_half[rows] = st.p[rows] + 0.5 * length[:, None] * st.a_hydro[rows]
    st.u_half[rows] = st.u[rows] + 0.5 * length * st.dudt[rows]
    _add_heat(st, rows, 0.5 * length)


def blocks_initialise(x, v, u, mass, h_guess, bc, t_stop, t0=0.0, level_offset=None,
                      reuse=True) -> BlockState:  # fmt: skip
    """sim/blocks.py:455-499."""
    cc = bc.coupled
    hc = cc.hydro
    x = np.array(x, float)
    n = len(x)
    p = gn_p_from_v(x, np.asarray(v, float))
    tick = bc.dt_max / 2.0**K_MAX
    st = BlockState(
        n=0, t0=t0, tick=tick, level=np.zeros(n, np.int64), n_beg=np.zeros(n, np.int64),
        n_end=np.zeros(n, np.int64), x_beg=x.copy(), p_half=p.copy(),
        u_half=np.array(u, float) * np.ones(n), x=x, p=p, u=np.array(u, float) * np.ones(n),
        mass=np.array(mass, float) * np.ones(n), h=np.array(h_guess, float) * np.ones(n),
        alpha=np.full(n, hc.alpha_init if hc.switch else hc.alpha_const),
        a_hydro=np.zeros((n, 3)), dudt=np.zeros(n), rho=np.zeros(n), omega=np.ones(n),
        vsig_max=np.zeros(n),
        level_offset=np.zeros(n, np.int64) if level_offset is None
        else np.asarray(level_offset, np.int64),
        n_stop=int(round((t_stop - t0) / tick)),
    )  # fmt: skip
    st.luminosity = np.zeros(n)
    st.nu = np.zeros(n)
    for name in ("visc_heating", "cond_heating", "disk_heating", "heat_visc", "heat_cond",
                 "heat_disk", "heat_pdv", "heat_cool"):  # fmt: skip
        setattr(st, name, np.zeros(n))
    st.ids = np.arange(n)
    st.r0 = np.linalg.norm(x, axis=1)
    st.L0 = np.linalg.norm(np.cross(x, p), axis=1)
    st.vr_neg = np.sum(x * native.gn_v_from_p(x, p), axis=1) < 0
    st.passed_peri = np.zeros(n, bool)
    st.doomed = np.zeros(n, bool)
    st.removed = RemovedLedger()
    rows = np.arange(n)
    nb = _hydro_rows(st, bc, rows, native.gn_v_from_p(x, p), st.u, reuse)
    st.level[:] = 0
    _choose_levels(st, bc, rows, nb)
    _open(st, rows)
    if (getattr(bc, "r_acc", None) is not None or getattr(bc, "r_escape", None) is not None) \
            and bc.removal_sync:  # fmt: skip
        _wake_for_removal(st, bc, rows, nb)
    return st


def blocks_advance(st: BlockState, bc, reuse=True) -> np.ndarray:
    """sim/blocks.py:502-563 (no RESPA)."""
    cc = bc.coupled
    t0 = time.perf_counter()
    n_next = int(np.min(st.n_end))
    s = (n_next - st.n_beg) * st.tick
    half_len = 0.5 * (st.n_end - st.n_beg) * st.tick
    x, p_flow, _ = native.glf_step_many(st.x_beg, st.p_half, s)
    t1 = time.perf_counter()
    rows = np.flatnonzero(st.n_end == n_next)
    lag = (s - half_len)[:, None]
    p_pred = p_flow + lag * st.a_hydro
    if _cooling_on(cc):
        r_mid = 0.5 * (np.linalg.norm(st.x_beg, axis=1) + np.linalg.norm(x, axis=1))
        u_half_c = _cool(cc, st.u_half, st.rho, s, r_mid)
        dm = st.mass[rows] * (st.u_half[rows] - u_half_c[rows])
        st.e_radiated += float(np.sum(dm))
        st.luminosity[rows] = dm / (2.0 * half_len[rows])
        u_pred = u_half_c + (s - half_len) * st.dudt
        st.heat_cool[rows] += st.u_half[rows] - u_half_c[rows]
        st.u_half[rows] = u_half_c[rows]
    else:
        u_pred = st.u_half + (s - half_len) * st.dudt
    st.n = n_next
    st.x = x
    st.u = u_pred
    a_prev = st.a_hydro.copy()
    v_eval = native.gn_v_from_p(x, p_pred)
    nb = _hydro_rows(st, bc, rows, v_eval, u_pred, reuse, 2.0 * half_len[rows], a_prev)
    t2 = time.perf_counter()
    removal = getattr(bc, "r_acc", None) is not None or getattr(bc, "r_escape", None) is not None
    sync = removal and bc.removal_sync
    u_eval = u_pred.copy() if sync else None
    p_pred[rows] = p_flow[rows] + half_len[rows, None] * st.a_hydro[rows]
    st.u[rows] = st.u_half[rows] + half_len[rows] * st.dudt[rows]
    _add_heat(st, rows, half_len[rows])
    st.p = p_pred
    n_active = len(rows)
    if sync:
        rows, nb = _remove(st, bc, rows, nb, v_eval, u_eval, reuse)
    _choose_levels(st, bc, rows, nb)
    _open(st, rows)
    if sync:
        _wake_for_removal(st, bc, rows, nb)
    st.timers["flow"] += t1 - t0
    st.timers["hydro"] += t2 - t1
    st.timers["levels"] += time.perf_counter() - t2
    st.active_counts.append(n_active)
    st.particle_steps += n_active
    if removal and not sync:
        rows = _swallow_keep(st, bc, rows)[0]
    return rows


def _remove(st: BlockState, bc, rows, nb, v_eval, u_eval, reuse=True):
    """sim/blocks.py:566-590: removal after the closing kicks, then the remaining active rows'
    forces again without the removed particles (same predicted velocities and energies, switch
    not advanced); returns the remaining rows and their pair lists, renumbered."""
    n_old = len(st.x)
    new_rows, keep = _swallow_keep(st, bc, rows)
    if keep is None:
        return new_rows, nb
    owner = np.repeat(np.arange(n_old), np.diff(nb.offset))
    new_index = np.cumsum(keep) - 1
    mask = keep[owner] & keep[nb.index]
    counts = np.bincount(new_index[owner[mask]], minlength=len(st.x))
    offset = np.zeros(len(st.x) + 1, np.int64)
    np.cumsum(counts, out=offset[1:])
    nb = native.Neighbours(offset, new_index[nb.index[mask]], nb.box)
    if len(new_rows):
        _hydro_rows(st, bc, new_rows, v_eval[keep], u_eval[keep], reuse,
                    np.zeros(len(new_rows)), None)  # fmt: skip
    return new_rows, nb


def _wake_for_removal(st: BlockState, bc, rows, nb):
    """sim/blocks.py:593-627."""
    if len(rows) == 0:
        return
    length = (st.n_end[rows] - st.n_beg[rows]) * st.tick
    x_end, _, _ = native.glf_step_many(st.x_beg[rows], st.p_half[rows], length)
    r = np.linalg.norm(x_end, axis=1)
    doomed = np.zeros(len(rows), bool)
    if bc.r_acc is not None:
        doomed |= r < bc.r_acc
    if bc.r_escape is not None:
        doomed |= r > bc.r_escape
    st.doomed[rows] = doomed
    lists = nb if st.neighbour_cache is None else st.neighbour_cache.neighbours
    src = np.zeros(len(st.x), bool)
    src[rows] = True
    owner = np.repeat(np.arange(len(st.x)), np.diff(lists.offset))
    keep = src[owner]
    owner, other = owner[keep], lists.index[keep]
    end = np.full(len(st.x), np.iinfo(np.int64).max)
    label = st.level.copy()
    for a, b in ((owner, other), (other, owner)):
        m = st.doomed[a] & (a != b)
        np.minimum.at(end, b[m], st.n_end[a[m]])
        np.maximum.at(label, b[m], st.level[a[m]])
    j = np.flatnonzero((end < st.n_end) & (st.n_end > st.n))
    if len(j):
        _cut_to(st, j, end[j], label[j])


@dataclass
class RemovedLedger:
    """sim/accretion.py:19-44: totals and a log of the removed particles."""

    mass: float = 0.0
    energy: float = 0.0
    angmom: np.ndarray = field(default_factory=lambda: np.zeros(3))
    momentum: np.ndarray = field(default_factory=lambda: np.zeros(3))
    log: list = field(default_factory=list)

    @property
    def count(self) -> int:
        return len(self.log)


def _record_removal(led, t, ids, mass, ham, u, am, p, r, passed, L0, reason):
    """sim/accretion.py:47-62."""
    for k in range(len(ids)):
        led.momentum = led.momentum + mass[k] * np.asarray(p[k], float)
        led.mass += float(mass[k])
        led.energy += float(mass[k] * (ham[k] + u[k]))
        led.angmom = led.angmom + mass[k] * np.asarray(am[k], float)
        led.log.append({"t": float(t), "id": int(ids[k]), "reason": reason, "r": float(r[k]),
                        "m": float(mass[k]), "H": float(ham[k]), "u": float(u[k]),
                        "L": float(np.linalg.norm(am[k])), "L0": float(L0[k]),
                        "first_pass": not bool(passed[k])})  # fmt: skip


def _swallow_keep(st: BlockState, bc, rows):
    """sim/blocks.py:673-719 (_swallow, _swallow_keep, _prune) for the GN hole: pericentre
    flags of the active rows, removal of those inside r_acc or beyond r_escape (their state is
    true at their own step end) into the ledger; returns the remaining rows, renumbered, and the
    mask of the kept particles (None when none was removed)."""
    x, p = st.x[rows], st.p[rows]
    r = np.linalg.norm(x, axis=1)
    vr = np.sum(x * native.gn_v_from_p(x, p), axis=1)
    turned = st.vr_neg[rows] & (vr > 0) & (r < 0.5 * st.r0[rows])
    st.passed_peri[rows] |= turned
    st.vr_neg[rows] = vr < 0
    acc = r < bc.r_acc if bc.r_acc is not None else np.zeros(len(rows), bool)
    esc = r > bc.r_escape if bc.r_escape is not None else np.zeros(len(rows), bool)
    if not (np.any(acc) or np.any(esc)):
        return rows, None
    for mask, reason in ((acc, "accreted"), (esc, "escaped")):
        g = rows[mask]
        if len(g) == 0:
            continue
        xs, ps = st.x[g], st.p[g]
        _record_removal(st.removed, st.t, st.ids[g], st.mass[g], gn_hamiltonian(xs, ps), st.u[g],
                        np.cross(xs, ps), ps, np.linalg.norm(xs, axis=1), st.passed_peri[g],
                        st.L0[g], reason)  # fmt: skip
    keep = np.ones(len(st.x), bool)
    keep[rows[acc | esc]] = False
    n = len(keep)
    for name, value in vars(st).items():
        if isinstance(value, np.ndarray) and value.shape[:1] == (n,):
            setattr(st, name, value[keep])
    st.neighbour_cache = None
    new_index = np.cumsum(keep) - 1
    return new_index[rows[keep[rows]]], keep


def blocks_run(st: BlockState, bc, t_end, callback=None, reuse=True) -> BlockState:
    """sim/blocks.py:722-739."""
    n_end = int(round((t_end - st.t0) / st.tick))
    st.n_stop = n_end
    fresh = np.flatnonzero((st.n_beg == st.n) & (st.n_end > n_end))
    if len(fresh):
        st.level[fresh] = _land(st, st.level[fresh])
        if np.any(st.level[fresh] > K_MAX):
            raise ValueError(f"t_end needs a level beyond K_MAX = {K_MAX}")
        _open(st, fresh)
    if np.any(st.n_end > n_end):
        raise ValueError("some particles' current steps already run past t_end")
    while st.n < n_end:
        blocks_advance(st, bc, reuse)
        if callback is not None:
            callback(st)
    return st


def blocks_ledger(st: BlockState, bc) -> dict:
    """sim/blocks.py:742-758, the removed particles' totals included."""
    led = ledger_sums(st.mass, st.x, st.p, st.u, st.e_radiated)
    rm = st.removed
    if rm is not None:
        led["energy"] += rm.energy
        led["angmom"] = led["angmom"] + rm.angmom
        led["momentum"] = led["momentum"] + rm.momentum
        led["mass"] += rm.mass
    return led


def blocks_snapshot(st: BlockState, bc, t):
    """sim/blocks.py:777-787."""
    n_t = (t - st.t0) / st.tick
    if np.any(n_t < st.n_beg - 1e-6) or np.any(n_t > st.n_end + 1e-6):
        raise ValueError("snapshot time outside some particle's current step")
    s = np.maximum((t - st.t0) - st.n_beg * st.tick, 0.0)
    x, p_flow, _ = native.glf_step_many(st.x_beg, st.p_half, s)
    lag = s - 0.5 * (st.n_end - st.n_beg) * st.tick
    return x, p_flow + lag[:, None] * st.a_hydro
