"""Generate the golden fixtures of tests/golden/ by running the REFERENCE implementation.

Run once in an environment where the reference source is importable (it is not needed on a GPU
host; the fixtures it writes are committed):

    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py \
        --reference <reference>

Every fixture stores the inputs and the reference's outputs of one hot-path function on seeded
inputs: neighbour lists (find_neighbours_numba), tighten, density_numba, compute_density,
forces_numba, disc_forces_numba, glf_step_many, beta_cool, coupled.step and blocks.advance.
The inputs follow the reference's own tests (tests/sim/test_neighbours.py:15-19, 102-130;
tests/sim/test_density.py:21-27; tests/sim/test_forces.py:21-26) or the seeded cloud of the
benchmark workloads.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEED = 20261014  # the reference's test seed (tests/conftest.py:7)


def _uneven(rng, n, box):
    pos = rng.uniform(0, box, size=(n, 3))
    h = np.exp(rng.uniform(np.log(0.01), np.log(0.3), n)) * box / 8
    return pos, h


def _blob(rng, n=2000):
    core = rng.normal(0.0, 0.15, size=(n // 2, 3))
    bg = rng.uniform(-1.0, 1.0, size=(n - n // 2, 3))
    return np.concatenate([core, bg]), np.full(n, 1.0 / n)


def _save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path) / 1e3:.0f} kB)")


def lists_fixture(nbmod):
    out = {}
    cases = ["open_uneven", "periodic_cube", "periodic_long_box", "isolated_large_h", "clump_and_halo"]
    for case in cases:
        rng = np.random.default_rng(SEED)
        if case == "open_uneven":
            pos, h = _uneven(rng, 3000, 2.0)
            box = None
        elif case == "periodic_cube":
            pos, h = _uneven(rng, 3000, 2.0)
            box = 2.0
        elif case == "periodic_long_box":
            box = np.array([2.0, 0.125, 0.125])
            pos = rng.uniform(0, 1, (4000, 3)) * box
            h = rng.uniform(0.005, 0.03, 4000)
        elif case == "isolated_large_h":
            pos = np.concatenate([rng.uniform(0, 1, (2000, 3)), [[5.0, 5.0, 5.0], [-3.0, 0.5, 0.5]]])
            h = np.concatenate([np.full(2000, 0.04), [4.0, 2.5]])
            box = None
        else:
            pos = np.concatenate([rng.normal(0, 0.02, (2000, 3)), rng.uniform(-1, 1, (500, 3))])
            h = np.concatenate([np.full(2000, 0.005), np.full(500, 0.5)])
            box = None
        nb = nbmod.find_neighbours_numba(pos, h, box=box)
        ref = nbmod.find_neighbours(pos, h, box=box)
        assert np.array_equal(nb.offset, ref.offset) and np.array_equal(nb.index, ref.index)
        out[f"{case}_pos"] = pos
        out[f"{case}_h"] = h
        out[f"{case}_box"] = np.zeros(3) if box is None else np.broadcast_to(box, (3,)).astype(float)
        out[f"{case}_offset"] = nb.offset.astype(np.int64)
        out[f"{case}_index"] = nb.index.astype(np.int32)
    out["cases"] = np.array(cases)
    _save("lists.npz", **out)


def cloud_lists_fixture(nbmod, ics):
    """The 4,096-particle benchmark cloud: reference cell grid and lists at h_search = 1.4 h."""
    ic = ics.cloud(4096)
    hs = ic.h * 1.4
    nb = nbmod.find_neighbours_numba(ic.x, hs)
    # reference grid geometry (sim/neighbours.py:251-266) and cell of each particle
    lo = ic.x.min(axis=0)
    span = ic.x.max(axis=0) - lo
    cell = max(0.5 * 2.0 * float(np.median(hs)), float(np.max(span)) / 160.0, 1e-300)
    ncell = np.maximum(np.floor(span / cell).astype(np.int64) + 1, 1)
    inv = np.full(3, 1.0 / cell)
    start, order = nbmod._build_grid(ic.x, lo, inv, ncell)
    tight = nbmod.tighten(nb, ic.x, ic.h)
    _save("cloud_lists.npz", pos=ic.x, h_search=hs, h=ic.h, offset=nb.offset,
          index=nb.index.astype(np.int32), grid_start=start, grid_order=order.astype(np.int32),
          ncell=ncell, lo=lo, inv_cell=inv, tight_offset=tight.offset,
          tight_index=tight.index.astype(np.int32))  # fmt: skip


def density_fixture(sph, nbmod):
    rng = np.random.default_rng(SEED)
    pos, mass = _blob(rng)
    h0 = np.full(len(pos), 0.05)
    first = sph.compute_density(pos, mass, h0, h_max=0.5)
    h_search = first.h * 1.25
    nb = nbmod.find_neighbours(pos, h_search)
    rows = np.sort(rng.choice(len(pos), 700, replace=False))
    fast = sph.density_numba(pos, mass, first.h, nb, h_search, tol=1e-12, h_max=0.5)
    part = sph.density_numba(pos, mass, first.h, nb, h_search, tol=1e-12, h_max=0.5, rows=rows)
    cub = sph.density_numba(pos, mass, first.h, nb, h_search, kernel_name="cubic", eta=1.2,
                            tol=1e-4, h_max=0.5)  # fmt: skip
    _save("density.npz", pos=pos, mass=mass, h_first=first.h, rho_first=first.rho,
          omega_first=first.omega, flags_first=first.flags, h_search=h_search,
          offset=nb.offset, index=nb.index.astype(np.int32), rows=rows,
          h=fast.h, rho=fast.rho, omega=fast.omega, iters=fast.iterations, flags=fast.flags,
          rows_h=part.h, rows_rho=part.rho, cubic_h=cub.h, cubic_rho=cub.rho,
          cubic_omega=cub.omega, cubic_flags=cub.flags, cubic_iters=cub.iterations)  # fmt: skip


def forces_fixture(sph, nbmod):
    rng = np.random.default_rng(SEED)
    pos, mass = _blob(rng)
    u = rng.uniform(0.5, 1.5, len(pos))
    vel = rng.normal(0.0, 0.3, size=pos.shape)
    d = sph.compute_density(pos, mass, np.full(len(pos), 0.05), h_max=0.5)
    p = (5.0 / 3.0 - 1.0) * d.rho * u
    cs = np.sqrt(10.0 / 9.0 * u)
    alpha = rng.uniform(0.0, 1.0, len(pos))
    nb = nbmod.tighten(d.neighbours, pos, d.h)
    rows = np.sort(rng.choice(len(pos), 600, replace=False))
    out = dict(pos=pos, vel=vel, mass=mass, h=d.h, rho=d.rho, omega=d.omega, pressure=p, u=u,
               c_s=cs, alpha=alpha, offset=nb.offset, index=nb.index.astype(np.int32), rows=rows)
    plain = sph.forces_numba(pos, vel, mass, d.h, d.rho, d.omega, p, nb)
    out.update(plain_acc=plain.acc, plain_dudt=plain.dudt, plain_vsig=plain.vsig_max)
    for sig in (0, 1):
        shock = sph.ShockCapturing(beta=2.0, alpha_u=0.5, conductivity_signal=sig)
        f = sph.forces_numba(pos, vel, mass, d.h, d.rho, d.omega, p, nb, u=u, c_s=cs, alpha=alpha,
                             shock=shock)  # fmt: skip
        out.update({f"cond{sig}_acc": f.acc, f"cond{sig}_dudt": f.dudt,
                    f"cond{sig}_vsig": f.vsig_max, f"cond{sig}_visc": f.dudt_visc,
                    f"cond{sig}_cond": f.dudt_cond})  # fmt: skip
    fr = sph.forces_numba(pos, vel, mass, d.h, d.rho, d.omega, p, nb, u=u, c_s=cs, alpha=alpha,
                          shock=sph.ShockCapturing(alpha_u=0.5, conductivity_signal=1), rows=rows)
    out.update(rows_acc=fr.acc, rows_dudt=fr.dudt, rows_vsig=fr.vsig_max)
    a_d, u_d = sph.disc_forces_numba(pos, vel, mass, d.h, d.rho, d.omega, cs, 0.5, nb)
    out.update(disc_acc=a_d, disc_dudt=u_d)
    cub = sph.forces_numba(pos, vel, mass, d.h, d.rho, d.omega, p, nb, kernel_name="cubic", u=u,
                           c_s=cs, alpha=alpha)  # fmt: skip
    out.update(cubic_acc=cub.acc, cubic_dudt=cub.dudt, cubic_vsig=cub.vsig_max)
    _save("forces.npz", **out)


def glf_fixture(integ, gravity):
    rng = np.random.default_rng(SEED)
    n = 200
    r = np.exp(rng.uniform(np.log(6.0), np.log(5000.0), n))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    x = d * r[:, None]
    t = np.cross(d, rng.normal(size=(n, 3)))
    t /= np.linalg.norm(t, axis=1)[:, None]
    v = (t * rng.uniform(0.5, 1.2, n)[:, None] + d * rng.uniform(-0.3, 0.3, n)[:, None]) \
        * np.sqrt(1.0 / r)[:, None]  # fmt: skip
    p = gravity.gn_p_from_v(x, v)
    dt = 0.005 * r**1.5
    x1, p1, it = integ.glf_step_many(x, p, dt)
    _save("glf.npz", x=x, p=p, dt=dt, x1=x1, p1=p1, iters=it, v=v,
          v_from_p=gravity.gn_v_from_p(x, p), ham=gravity.gn_hamiltonian(x, p))  # fmt: skip


def cooling_fixture(cooling):
    rng = np.random.default_rng(SEED)
    u = np.exp(rng.uniform(np.log(1e-10), np.log(1e-4), 500))
    uf = np.full(500, 2.0e-9)
    dt = np.exp(rng.uniform(0.0, np.log(1e5), 500))
    r = rng.uniform(10.0, 5000.0, 500)
    tc = cooling.cooling_time(r, 230.0)
    _save("cooling.npz", u=u, u_floor=uf, dt=dt, r=r, t_cool=tc,
          u_new=cooling.beta_cool(u, uf, dt, tc))  # fmt: skip


def _state_arrays(prefix, st, fields):
    return {f"{prefix}_{f}": np.array(getattr(st, f), copy=True) for f in fields}


def coupled_fixture(coupled, ics, hydro_cfg):
    """The 4,096-particle cloud (cubic kernel, eta 1.2, alpha = 1, beta = 2, GN hole, no
    cooling): initialise and three shared steps of stable_dt."""
    ic = ics.cloud(4096)
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc)
    st = coupled.initialise(ic.x, ic.v, ic.u, ic.mass, ic.h, cc)
    fields = ["x", "p", "u", "h", "rho", "a_hydro", "dudt", "vsig_max", "c_s"]
    out = dict(x0=ic.x, v0=ic.v, u0=ic.u, mass=ic.mass, h0=ic.h)
    out.update(_state_arrays("init", st, fields))
    dts = []
    for k in range(3):
        dt = coupled.stable_dt(st, cc)
        dts.append(dt)
        st = coupled.step(st, cc, dt)
        out.update(_state_arrays(f"step{k + 1}", st, fields))
        led = coupled.ledger(st, cc)
        out[f"step{k + 1}_energy"] = led["energy"]
        out[f"step{k + 1}_angmom"] = led["angmom"]
    out["dts"] = np.array(dts)
    out["builds"] = st.neighbour_cache.builds
    out["reuses"] = st.neighbour_cache.reuses
    _save("coupled.npz", **out)


def blocks_fixture(blocks, coupled, ics, hydro_cfg):
    """A 2,048-particle cloud warm enough to spread over several levels: block steps with the
    limiter, beta-cooling, conductivity, forced level offsets 0-3; 16 system steps."""
    ic = ics.cloud(2048, radius=20.0, total_mass=1e-3, t_kelvin=3e8, r_peri=60.0, r_apo=400.0,
                   seed=7)  # fmt: skip
    rng = np.random.default_rng(SEED)
    v = ic.v + rng.normal(0.0, 0.002, ic.v.shape)
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc, cooling_beta=230.0)
    bc = blocks.BlockConfig(coupled=cc, dt_max=64.0)
    offset = rng.integers(0, 4, len(ic.x))  # forced extra levels (the reference's test hook)
    st = blocks.initialise(ic.x, v, ic.u, ic.mass, ic.h, bc, t_stop=1e9, level_offset=offset)
    fields = ["x", "p", "u", "h", "rho", "omega", "a_hydro", "dudt", "level", "n_beg", "n_end",
              "x_beg", "p_half", "u_half", "vsig_max"]
    out = dict(x0=ic.x, v0=v, u0=ic.u, mass=ic.mass, h0=ic.h, level_offset=offset)
    out.update(_state_arrays("init", st, fields))
    actives = []
    for k in range(16):
        rows = blocks.advance(st, bc)
        actives.append(len(rows))
    out.update(_state_arrays("final", st, fields))
    led = blocks.ledger(st, bc)
    out["final_energy"] = led["energy"]
    out["final_e_radiated"] = led["e_radiated"]
    out["final_n"] = st.n
    out["active_counts"] = np.array(actives)
    out["builds"] = st.neighbour_cache.builds
    out["reuses"] = st.neighbour_cache.reuses
    out["woken"] = st.woken
    _save("blocks.npz", **out)


def eos_fixture(hydro_mod, units_mod):
    """Equations of state of sim/hydro.py:121-139 on seeded (rho, T): ideal, radiation limit and
    gas + radiation (the Numba T-solve of sim/fastphys.py:45-102), with T and beta_gas."""
    from nebula.sim.fastphys import gasrad_state_nb
    from nebula.physics.eos import gasrad_u_si

    rng = np.random.default_rng(SEED + 5)
    gu = units_mod.GasUnits()
    rho = 10.0 ** rng.uniform(-12.0, -4.0, 4000)
    t = 10.0 ** rng.uniform(3.0, 12.0, 4000)
    u = units_mod.specific_energy_from_si(gasrad_u_si(gu.density_to_si(rho), t))
    p, cs, tt, beta = gasrad_state_nb(rho, u, gu)
    out = dict(rho=rho, u=u, gasrad_p=p, gasrad_cs=cs, gasrad_t=tt, gasrad_beta=beta)
    for eos in ("ideal", "radiation"):
        hc = hydro_mod.HydroConfig(eos=eos)
        pe, ce = hydro_mod.eos_state(hc, rho, u)
        out[f"{eos}_p"], out[f"{eos}_cs"] = pe, ce
    _save("eos.npz", **out)


def gasrad_blocks_fixture(blocks, coupled, ics, hydro_cfg):
    """Block steps of the 2,048-particle cloud of blocks_fixture with the gas + radiation
    equation of state (radiation-dominated at 3e8 K), no cooling; 12 system steps."""
    ic = ics.cloud(2048, radius=20.0, total_mass=1e-3, t_kelvin=3e8, r_peri=60.0, r_apo=400.0,
                   seed=7)  # fmt: skip
    rng = np.random.default_rng(SEED + 6)
    v = ic.v + rng.normal(0.0, 0.002, ic.v.shape)
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0, eos="gasrad")  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc)
    bc = blocks.BlockConfig(coupled=cc, dt_max=64.0)
    st = blocks.initialise(ic.x, v, ic.u, ic.mass, ic.h, bc, t_stop=1e6)
    fields = ["x", "p", "u", "h", "rho", "omega", "a_hydro", "dudt", "level", "n_beg", "n_end",
              "vsig_max"]
    out = dict(x0=ic.x, v0=v, u0=ic.u, mass=ic.mass, h0=ic.h)
    out.update(_state_arrays("init", st, fields))
    actives = [len(blocks.advance(st, bc)) for _ in range(12)]
    out.update(_state_arrays("final", st, fields))
    out["final_energy"] = blocks.ledger(st, bc)["energy"]
    out["final_n"] = st.n
    out["active_counts"] = np.array(actives)
    _save("gasrad_blocks.npz", **out)


def _shock_blob(rng):
    """The forces blob plus three isolated particles (no neighbours within h_max) and a planar
    patch of six (a singular correction matrix): both fallbacks of the corrected gradients."""
    pos, _ = _blob(rng)
    iso = np.array([[6.0, 6.0, 6.0], [-6.0, 6.0, 6.0], [6.0, -6.0, 6.0]])
    gx, gy = np.meshgrid([0.0, 0.12, 0.24], [0.0, 0.12])
    plane = np.stack([gx.ravel() - 6.0, gy.ravel() - 6.0, np.full(6, -6.0)], axis=1)
    pos = np.concatenate([pos, iso, plane])
    return pos, np.full(len(pos), 1.0 / len(pos))


def shock_fixture(sph, nbmod):
    """Corrected velocity / acceleration gradients (sim/sph.py:797-902) and the force pass with
    velocity reconstruction (sim/sph.py:568-609) for the three gates, with and without the
    closeness factor, on the blob with a linear velocity field plus noise."""
    rng = np.random.default_rng(SEED + 7)
    pos, mass = _shock_blob(rng)
    n = len(pos)
    g0 = rng.normal(0.0, 0.4, (3, 3))
    vel = pos @ g0.T + rng.normal(0.0, 0.05, pos.shape)
    acc_prev = rng.normal(0.0, 0.2, pos.shape) + pos @ rng.normal(0.0, 0.3, (3, 3)).T
    u = rng.uniform(0.5, 1.5, n)
    d = sph.compute_density(pos, mass, np.full(n, 0.05), h_max=0.5)
    p = (5.0 / 3.0 - 1.0) * d.rho * u
    cs = np.sqrt(10.0 / 9.0 * u)
    alpha = rng.uniform(0.0, 1.0, n)
    nb = nbmod.tighten(d.neighbours, pos, d.h)
    rows = np.sort(rng.choice(n, 700, replace=False))
    out = dict(pos=pos, vel=vel, acc_prev=acc_prev, mass=mass, h=d.h, rho=d.rho, omega=d.omega,
               pressure=p, u=u, c_s=cs, alpha=alpha, offset=nb.offset,
               index=nb.index.astype(np.int32), rows=rows)  # fmt: skip
    g = sph.gradients_numba(pos, vel, acc_prev, mass, d.h, nb)
    out.update(div_v=g.div_v, curl_v=g.curl_v, ddivv_dt=g.ddivv_dt)
    gr = sph.gradients_numba(pos, vel, acc_prev, mass, d.h, nb, kernel_name="cubic", rows=rows)
    out.update(cubic_rows_div_v=gr.div_v, cubic_rows_curl_v=gr.curl_v, cubic_rows_ddivv_dt=gr.ddivv_dt)
    gv = sph.velocity_gradients_numba(pos, vel, mass, d.h, nb)
    out["grad_v"] = gv
    # untightened lists (search radius 1.4 h; rebuilt by the tests with the exact list build)
    full = nbmod.find_neighbours(pos, 1.4 * d.h)
    out["full_rows_grad_v"] = sph.velocity_gradients_numba(pos, vel, mass, d.h, full, rows=rows)
    for gate in (0, 1, 2):
        for close in (True, False):
            shock = sph.ShockCapturing(beta=2.0, alpha_u=0.5, conductivity_signal=1,
                                       reconstruction=True, closeness=close,
                                       eta_crit=1.0 / 1.2, recon_gate=gate)  # fmt: skip
            f = sph.forces_numba(pos, vel, mass, d.h, d.rho, d.omega, p, nb, u=u, c_s=cs,
                                 alpha=alpha, shock=shock, grad_v=gv)  # fmt: skip
            key = f"recon_g{gate}_c{int(close)}"
            out.update({f"{key}_acc": f.acc, f"{key}_dudt": f.dudt, f"{key}_vsig": f.vsig_max,
                        f"{key}_visc": f.dudt_visc, f"{key}_cond": f.dudt_cond})  # fmt: skip
    shock = sph.ShockCapturing(beta=2.0, alpha_u=0.5, conductivity_signal=0, reconstruction=True,
                               eta_crit=1.0 / 1.2)  # fmt: skip
    f = sph.forces_numba(pos, vel, mass, d.h, d.rho, d.omega, p, nb, kernel_name="cubic", u=u,
                         c_s=cs, alpha=alpha, shock=shock, rows=rows, grad_v=gv)  # fmt: skip
    out.update(recon_rows_cubic_acc=f.acc, recon_rows_cubic_dudt=f.dudt,
               recon_rows_cubic_vsig=f.vsig_max)  # fmt: skip
    _save("shock.npz", **out)


def switch_coupled_fixture(coupled, ics, hydro_cfg):
    """Shared steps of the 4,096-particle cloud with the reference's default shock capturing
    (Cullen-Dehnen switch from alpha = 0, velocity reconstruction with the min-mod gate) and a
    velocity noise that drives the switch; three steps of stable_dt."""
    ic = ics.cloud(4096)
    rng = np.random.default_rng(SEED + 8)
    v = ic.v + rng.normal(0.0, 3e-4, ic.v.shape)
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=True, reconstruction=True,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc)
    st = coupled.initialise(ic.x, v, ic.u, ic.mass, ic.h, cc)
    fields = ["x", "p", "u", "h", "rho", "alpha", "a_hydro", "dudt", "vsig_max"]
    out = dict(x0=ic.x, v0=v, u0=ic.u, mass=ic.mass, h0=ic.h)
    out.update(_state_arrays("init", st, fields))
    dts = []
    for k in range(3):
        dt = coupled.stable_dt(st, cc)
        dts.append(dt)
        st = coupled.step(st, cc, dt)
        out.update(_state_arrays(f"step{k + 1}", st, fields))
        out[f"step{k + 1}_energy"] = coupled.ledger(st, cc)["energy"]
    out["dts"] = np.array(dts)
    out["builds"] = st.neighbour_cache.builds
    out["reuses"] = st.neighbour_cache.reuses
    _save("switch_coupled.npz", **out)


def switch_blocks_fixture(blocks, coupled, ics, hydro_cfg):
    """Block steps of the blocks_fixture cloud (level offsets 0-3, beta = 230) with the switch
    and velocity reconstruction on; 16 system steps."""
    ic = ics.cloud(2048, radius=20.0, total_mass=1e-3, t_kelvin=3e8, r_peri=60.0, r_apo=400.0,
                   seed=7)  # fmt: skip
    rng = np.random.default_rng(SEED)
    v = ic.v + rng.normal(0.0, 0.002, ic.v.shape)
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=True, reconstruction=True,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc, cooling_beta=230.0)
    bc = blocks.BlockConfig(coupled=cc, dt_max=64.0)
    offset = rng.integers(0, 4, len(ic.x))
    st = blocks.initialise(ic.x, v, ic.u, ic.mass, ic.h, bc, t_stop=1e6, level_offset=offset)
    fields = ["x", "p", "u", "h", "rho", "alpha", "a_hydro", "dudt", "level", "n_beg", "n_end",
              "vsig_max"]
    out = dict(x0=ic.x, v0=v, u0=ic.u, mass=ic.mass, h0=ic.h, level_offset=offset)
    out.update(_state_arrays("init", st, fields))
    actives = [len(blocks.advance(st, bc)) for _ in range(16)]
    out.update(_state_arrays("final", st, fields))
    led = blocks.ledger(st, bc)
    out["final_energy"] = led["energy"]
    out["final_e_radiated"] = led["e_radiated"]
    out["final_n"] = st.n
    out["active_counts"] = np.array(actives)
    out["builds"] = st.neighbour_cache.builds
    out["reuses"] = st.neighbour_cache.reuses
    _save("switch_blocks.npz", **out)


def _grid_fields(prefix, gg):
    return {f"{prefix}_mass": gg.mass, f"{prefix}_rho": gg.rho, f"{prefix}_t_mass": gg.t_mass,
            f"{prefix}_t_em": gg.t_em, f"{prefix}_vel": gg.vel,
            f"{prefix}_outside": np.float64(gg.outside),
            f"{prefix}_n_tri": np.int64(gg.n_trilinear)}  # fmt: skip


def deposit_fixture(gasgrid):
    """Particle -> grid deposition (render/gasgrid.py): the log-spherical grid and a Cartesian
    box, both kernels, on seeded particles with h from 0.1 to 10 local cells, including
    particles beyond the outer radius, on the phi seam and near both poles; the split
    deposition with half the particles wide."""
    rng = np.random.default_rng(SEED + 9)
    g = gasgrid.LogSphericalGrid(r_min=2.0, r_max=200.0, nr=24, nth=12, nph=24)
    n = 400
    lnr = rng.uniform(np.log(2.5), np.log(240.0), n)
    r = np.exp(lnr)
    cth = rng.uniform(-1.0, 1.0, n)
    cth[:25] = 1.0 - rng.uniform(0.0, 0.004, 25)  # near the north pole
    cth[25:50] = -1.0 + rng.uniform(0.0, 0.004, 25)  # near the south pole
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    ph[50:90] = rng.uniform(-0.04, 0.04, 40) % (2.0 * np.pi)  # on the seam
    sth = np.sqrt(1.0 - cth * cth)
    x = np.c_[r * sth * np.cos(ph), r * sth * np.sin(ph), r * cth]
    h = r * g.dlnr * np.exp(rng.uniform(np.log(0.1), np.log(10.0), n))
    m = rng.uniform(0.3, 3.0, n)
    t = np.exp(rng.uniform(np.log(3e3), np.log(3e7), n))
    v = rng.normal(0.0, 0.05, (n, 3))
    out = dict(x=x, h=h, m=m, t=t, v=v, log_grid=np.array([g.r_min, g.r_max, g.nr, g.nth, g.nph]))
    for kern in ("wendland_c4", "cubic"):
        out.update(_grid_fields(f"log_{kern}", gasgrid.deposit_log(x, h, m, t, v, g, kern)))
    b = gasgrid.CartesianBox(centre=(20.0, -10.0, 5.0), size=80.0, n=20)
    xb = np.asarray(b.centre) + rng.uniform(-0.6, 0.6, (n, 3)) * b.size
    hb = b.dx * np.exp(rng.uniform(np.log(0.1), np.log(10.0), n))
    out.update(xb=xb, hb=hb, box=np.array([*b.centre, b.size, b.n]))
    for kern in ("wendland_c4", "cubic"):
        out.update(_grid_fields(f"box_{kern}", gasgrid.deposit_box(xb, hb, m, t, v, b, kern)))
    # split: a coarser-divisible grid, half the particles wide
    gs = gasgrid.LogSphericalGrid(r_min=2.0, r_max=2000.0, nr=32, nth=16, nph=32)
    ns = 1200
    rs = np.exp(rng.uniform(np.log(30.0), np.log(600.0), ns))
    d = rng.normal(size=(ns, 3))
    xs = rs[:, None] * d / np.linalg.norm(d, axis=1, keepdims=True)
    hs = np.where(np.arange(ns) < ns // 2, 0.2, 3.0) * rs
    ms = np.full(ns, 1e-4)
    ts = rng.uniform(1e4, 1e5, ns)
    vs = rng.normal(0.0, 0.01, (ns, 3))
    out.update(xs=xs, hs=hs, ms=ms, ts=ts, vs=vs,
               split_grid=np.array([gs.r_min, gs.r_max, gs.nr, gs.nth, gs.nph]),
               split_wide=gasgrid.wide_particles(xs, hs, gs))  # fmt: skip
    sp = gasgrid.deposit_log_split(xs, hs, ms, ts, vs, gs)
    out.update(_grid_fields("split", sp))
    out["split_n_wide"] = np.int64(sp.extra["n_wide"])
    _save("deposit.npz", **out)


def removal_blocks_fixture(blocks, coupled, ics, hydro_cfg, sync=False):
    """Block steps with removal at the end of each particle's own step (sim/blocks.py:566-719,
    sim/accretion.py), without (removal_blocks.npz) and with removal_sync (removal_sync_blocks.npz:
    survivors' forces recomputed, doomed particles' neighbours cut): a 1,024-particle cloud
    centred at r = 5.2, falling in at 0.3 c, accretion radius 4.4 and escape radius 6.0; 120
    system steps."""
    ic = ics.cloud(1024, radius=1.0, total_mass=1e-6, t_kelvin=1e6, r_peri=6.0, r_apo=10.0,
                   seed=11)  # fmt: skip
    c = ic.x.mean(axis=0)
    chat = c / np.linalg.norm(c)
    x = ic.x - c + 5.2 * chat
    v = 0.5 * ic.v - 0.3 * chat
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc)
    bc = blocks.BlockConfig(coupled=cc, dt_max=4.0, r_acc=4.4, r_escape=6.0, removal_sync=sync)
    st = blocks.initialise(x, v, ic.u, ic.mass, ic.h, bc, t_stop=1e6)
    out = dict(x0=x, v0=v, u0=ic.u, mass=ic.mass, h0=ic.h)
    actives = [len(blocks.advance(st, bc)) for _ in range(120)]
    fields = ["x", "p", "u", "h", "level", "n_end", "ids", "vr_neg", "passed_peri", "doomed"]
    out.update(_state_arrays("final", st, fields))
    rm = st.removed
    out.update(active_counts=np.array(actives), final_n=st.n, removed_mass=rm.mass,
               removed_energy=rm.energy, removed_angmom=rm.angmom, removed_momentum=rm.momentum,
               final_energy=blocks.ledger(st, bc)["energy"])  # fmt: skip
    for k in ("t", "id", "r", "m", "H", "u", "L", "L0", "first_pass"):
        out[f"log_{k}"] = np.array([e[k] for e in rm.log])
    out["log_escaped"] = np.array([e["reason"] == "escaped" for e in rm.log])
    out["woken"] = st.woken
    _save("removal_sync_blocks.npz" if sync else "removal_blocks.npz", **out)


def removal_wake_fixture(blocks, coupled, ics, hydro_cfg):
    """removal_sync's wake-up of the doomed particles' neighbours (sim/blocks.py:593-627): the
    multi-level cloud of blocks_fixture (level offsets 0-3, beta = 230) with an accretion radius
    of 382 that its inner edge crosses within the 16 system steps."""
    ic = ics.cloud(2048, radius=20.0, total_mass=1e-3, t_kelvin=3e8, r_peri=60.0, r_apo=400.0,
                   seed=7)  # fmt: skip
    rng = np.random.default_rng(SEED)
    v = ic.v + rng.normal(0.0, 0.002, ic.v.shape)
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc, cooling_beta=230.0)
    offset = rng.integers(0, 4, len(ic.x))
    bc = blocks.BlockConfig(coupled=cc, dt_max=64.0, r_acc=382.0, removal_sync=True)
    st = blocks.initialise(ic.x, v, ic.u, ic.mass, ic.h, bc, t_stop=1e6, level_offset=offset)
    out = dict(x0=ic.x, v0=v, u0=ic.u, mass=ic.mass, h0=ic.h, level_offset=offset)
    actives = [len(blocks.advance(st, bc)) for _ in range(16)]
    fields = ["x", "p", "u", "h", "level", "n_beg", "n_end", "ids", "doomed"]
    out.update(_state_arrays("final", st, fields))
    out.update(active_counts=np.array(actives), final_n=st.n, woken=st.woken,
               removed_mass=st.removed.mass, final_energy=blocks.ledger(st, bc)["energy"],
               log_id=np.array([e["id"] for e in st.removed.log]))  # fmt: skip
    _save("removal_wake_blocks.npz", **out)


HEAT_FIELDS = ["u", "u_half", "visc_heating", "cond_heating", "disk_heating", "heat_visc",
               "heat_cond", "heat_disk", "heat_pdv", "heat_cool"]  # fmt: skip


def heat_fixture(blocks, coupled, ics, hydro_cfg):
    """The per-particle heat budget (sim/blocks.py:142-154, 434-440, 531, 546) on the multi-level
    cloud of blocks_fixture with disc viscosity (alpha_AV = 1) on top of viscosity, conductivity
    and beta-cooling: (sync) initialise with t_stop = 192 and run to 192, a full sync point;
    (reopen) initialise without a near stop and run to 0.75, so that run() re-opens every
    step to land on it (its _open books the opening kick a second time); (removal) the
    removal_sync run of removal_wake_fixture, 16 system steps (survivors' forces redone, the
    doomed particles' neighbours cut, removed particles' budgets dropped); (wake) 5 % of the
    particles forced 5 levels finer, run to 64, so that the limiter wakes neighbours up."""
    ic = ics.cloud(2048, radius=20.0, total_mass=1e-3, t_kelvin=3e8, r_peri=60.0, r_apo=400.0,
                   seed=7)  # fmt: skip
    rng = np.random.default_rng(SEED)
    v = ic.v + rng.normal(0.0, 0.002, ic.v.shape)
    offset = rng.integers(0, 4, len(ic.x))
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0, disc_alpha_av=1.0)  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc, cooling_beta=230.0)
    bc = blocks.BlockConfig(coupled=cc, dt_max=64.0)
    out = dict(x0=ic.x, v0=v, u0=ic.u, mass=ic.mass, h0=ic.h, level_offset=offset)
    st = blocks.initialise(ic.x, v, ic.u, ic.mass, ic.h, bc, t_stop=192.0, level_offset=offset)
    blocks.run(st, bc, 192.0)
    out.update(_state_arrays("sync", st, HEAT_FIELDS))
    out.update(sync_e_radiated=st.e_radiated, sync_n=st.n)
    st = blocks.initialise(ic.x, v, ic.u, ic.mass, ic.h, bc, t_stop=1e6, level_offset=offset)
    blocks.run(st, bc, 0.75)
    out.update(_state_arrays("reopen", st, HEAT_FIELDS + ["level", "n_end"]))
    out.update(reopen_n=st.n)
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0)  # fmt: skip
    cc = coupled.CoupledConfig(hydro=hc, cooling_beta=230.0)
    bc = blocks.BlockConfig(coupled=cc, dt_max=64.0, r_acc=382.0, removal_sync=True)
    st = blocks.initialise(ic.x, v, ic.u, ic.mass, ic.h, bc, t_stop=1e6, level_offset=offset)
    for _ in range(16):
        blocks.advance(st, bc)
    out.update(_state_arrays("removal", st, HEAT_FIELDS + ["ids"]))
    out.update(removal_e_radiated=st.e_radiated, removal_n=st.n)
    # (wake) as (sync) with 5 % of the particles forced 5 levels finer, so that the limiter wakes
    # their neighbours up (steps cut short, the opening half-kick corrected and booked)
    hc = hydro_cfg(kernel="cubic", eta=1.2, switch=False, reconstruction=False,
                   conductivity_signal=1, alpha_u=0.05, h_max=200.0, disc_alpha_av=1.0)  # fmt: skip
    bc = blocks.BlockConfig(coupled=coupled.CoupledConfig(hydro=hc, cooling_beta=230.0),
                            dt_max=64.0)  # fmt: skip
    wake_offset = np.where(rng.random(len(ic.x)) < 0.05, 5, 0)
    st = blocks.initialise(ic.x, v, ic.u, ic.mass, ic.h, bc, t_stop=64.0,
                           level_offset=wake_offset)  # fmt: skip
    blocks.run(st, bc, 64.0)
    out.update(_state_arrays("wake", st, HEAT_FIELDS))
    out.update(wake_offset=wake_offset, wake_n=st.n, wake_woken=st.woken,
               wake_e_radiated=st.e_radiated)  # fmt: skip
    _save("heat_blocks.npz", **out)


def phantom_fixture(reference, units_mod, coupled):
    """The reference's external golden vectors (tests/data/phantom_force_sample.npz: one
    Phantom derivative evaluation with the reference's formulas patched in, 8,931 particles,
    Wendland C4, gas + radiation, reconstruction on and off) with the particle mass converted to
    the reference's code units and the reference's default hydro settings, as its test
    tests/sim/test_phantom_patch.py:34-72 uses them."""
    d = dict(np.load(os.path.join(reference, "tests", "data", "phantom_force_sample.npz")))
    hc = coupled.CoupledConfig().hydro
    m = d["mass_phantom"] * units_mod.BlackHoleUnits().mass_kg / hc.gas_units.mass_kg_per_code
    out = {k: d[k] for k in ("x", "v", "u", "h_phantom", "alpha", "pressure", "acc_on", "dudt_on",
                             "acc_off", "dudt_off", "center", "r_in")}  # fmt: skip
    out.update(mass=np.full(len(d["x"]), m), mratio=np.float64(d["mass_phantom"] / m),
               kernel=np.array(hc.kernel), eta=hc.eta, h_max=hc.h_max, alpha_u=hc.alpha_u,
               beta=hc.beta, conductivity_signal=hc.conductivity_signal,
               recon_closeness=hc.recon_closeness, recon_gate=hc.recon_gate)  # fmt: skip
    _save("phantom_forces.npz", **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference checkout")
    ap.add_argument("--only", nargs="*", help="write only these fixtures (names without .npz)")
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(args.reference, "src"))
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from nebula.physics import cooling, gravity
    from nebula.sim import blocks, coupled, integrator, sph
    from nebula.sim import neighbours as nbmod
    from nebula import units as units_mod
    from nebula.sim import hydro as hydro_mod
    from nebula.sim.hydro import HydroConfig
    from nebula.render import gasgrid

    from blackhole_nebula_simulator_b200 import ics

    makers = {
        "lists": lambda: lists_fixture(nbmod),
        "cloud_lists": lambda: cloud_lists_fixture(nbmod, ics),
        "density": lambda: density_fixture(sph, nbmod),
        "forces": lambda: forces_fixture(sph, nbmod),
        "glf": lambda: glf_fixture(integrator, gravity),
        "cooling": lambda: cooling_fixture(cooling),
        "coupled": lambda: coupled_fixture(coupled, ics, HydroConfig),
        "blocks": lambda: blocks_fixture(blocks, coupled, ics, HydroConfig),
        "eos": lambda: eos_fixture(hydro_mod, units_mod),
        "gasrad_blocks": lambda: gasrad_blocks_fixture(blocks, coupled, ics, HydroConfig),
        "shock": lambda: shock_fixture(sph, nbmod),
        "switch_coupled": lambda: switch_coupled_fixture(coupled, ics, HydroConfig),
        "switch_blocks": lambda: switch_blocks_fixture(blocks, coupled, ics, HydroConfig),
        "deposit": lambda: deposit_fixture(gasgrid),
        "removal_blocks": lambda: removal_blocks_fixture(blocks, coupled, ics, HydroConfig),
        "removal_sync_blocks": lambda: removal_blocks_fixture(blocks, coupled, ics, HydroConfig,
                                                              sync=True),
        "removal_wake": lambda: removal_wake_fixture(blocks, coupled, ics, HydroConfig),
        "phantom": lambda: phantom_fixture(args.reference, units_mod, coupled),
        "heat_blocks": lambda: heat_fixture(blocks, coupled, ics, HydroConfig),
    }
    for name, make in makers.items():
        if not args.only or name in args.only:
            make()


if __name__ == "__main__":
    main()
