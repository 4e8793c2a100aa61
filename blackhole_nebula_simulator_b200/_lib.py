"""ctypes binding of libnebula_b200.so (the sm_100a kernels behind include/nebula_b200.h).

The library is built in place by ``build.py``; importing a function that needs it fails loudly
when it is missing (there is no CPU fallback).  Status codes map to the reference's exceptions:
GLFConvergenceError (sim/integrator.py:50), RuntimeError (sim/sph.py:387, sim/blocks.py:239),
FloatingPointError (sim/blocks.py:250), ValueError (sim/timesteps.py:30,38), NotImplementedError.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnebula_b200.so")

_c = ctypes
_vp = _c.c_void_p
_i64 = _c.c_int64
_dbl = _c.c_double
_int = _c.c_int


class GLFConvergenceError(RuntimeError):
    """An implicit stage of the generalized leapfrog failed, or a particle is too deep."""


class NebulaCudaError(RuntimeError):
    """A CUDA or host-side failure inside libnebula_b200.so."""


class NbMlpParams(_c.Structure):
    _fields_ = [
        ("tfac", _dbl), ("b", _dbl), ("kappa", _dbl), ("u_floor", _dbl), ("t_floor", _dbl),
        ("rho_unit_cgs", _dbl), ("t_unit_s", _dbl), ("lrho_lo", _dbl), ("lrho_hi", _dbl),
        ("lt_lo", _dbl), ("lt_hi", _dbl), ("ldt_lo", _dbl), ("ldt_hi", _dbl), ("check_tol", _dbl),
        ("judge", _int),
    ]  # fmt: skip


class NbParams(_c.Structure):
    _fields_ = [
        ("kernel_id", _int), ("cnorm", _dbl), ("eta", _dbl), ("tol", _dbl), ("h_max", _dbl),
        ("skin", _dbl), ("gamma", _dbl), ("viscosity", _int), ("conductivity", _int),
        ("cond_signal", _int), ("alpha_const", _dbl), ("beta", _dbl), ("alpha_u", _dbl),
        ("disc_alpha_av", _dbl), ("courant", _dbl), ("c_force", _dbl), ("eta_orb", _dbl),
        ("precision", _int), ("cooling", _int), ("cooling_beta", _dbl), ("u_floor", _dbl),
        ("brems_tfac", _dbl), ("brems_b", _dbl), ("brems_kappa", _dbl), ("brems_t_floor", _dbl),
        ("dt_max", _dbl), ("limiter", _int), ("max_gap", _int), ("mlp", NbMlpParams),
        ("eos", _int), ("eos_rho_si", _dbl), ("eos_u_si", _dbl), ("eos_a1", _dbl),
        ("eos_a_rad", _dbl), ("visc_switch", _int), ("recon", _int), ("recon_closeness", _int),
        ("recon_gate", _int), ("recon_eta_crit", _dbl), ("recon_eta_fold", _dbl),
    ]  # fmt: skip


class NbState(_c.Structure):
    _fields_ = [
        ("n", _i64),
        *[(f, _vp) for f in ("x", "p", "u", "mass", "h", "alpha", "a_hydro", "dudt", "rho",
                             "omega", "c_s", "vsig_max", "nu", "visc_heating", "level", "n_beg",
                             "n_end", "level_offset", "x_beg", "p_half", "u_half", "luminosity")],
        ("tick_n", _i64), ("n_stop", _i64), ("t0", _dbl), ("tick", _dbl), ("e_radiated", _dbl),
        ("particle_steps", _i64), ("woken", _i64), ("last_active", _i64), ("pairs", _i64),
        ("builds", _i64), ("reuses", _i64),
        *[(f, _vp) for f in ("cond_heating", "disk_heating", "heat_visc", "heat_cond", "heat_disk",
                             "heat_pdv", "heat_cool")],
    ]  # fmt: skip


_lib = None

_SIGS = {
    "nb_create": (_vp, [_int]),
    "nb_destroy": (None, [_vp]),
    "nb_last_error": (_c.c_char_p, [_vp]),
    "nb_version": (_int, []),
    "nb_state_size": (_i64, []),
    "nb_params_size": (_i64, []),
    "nb_launch_count": (_i64, []),
    "nb_sync_count": (_i64, []),
    "nb_reset_cache": (_int, [_vp]),
    "nb_profile": (_int, [_vp, _int]),
    "nb_profile_read": (_int, [_vp, _c.POINTER(_dbl)]),
    "nb_find_neighbours": (_int, [_vp, _i64, _vp, _vp, _vp, _c.POINTER(_i64), _vp]),
    "nb_neighbours_export": (_int, [_vp, _vp, _vp, _vp]),
    "nb_cell_geometry": (_int, [_vp, _i64, _vp, _vp, _c.POINTER(_dbl), _c.POINTER(_dbl),
                                _c.POINTER(_i64), _vp]),
    "nb_build_cells": (_int, [_vp, _i64, _vp, _c.POINTER(_dbl), _c.POINTER(_dbl),
                              _c.POINTER(_i64), _vp, _vp, _vp]),
    "nb_tighten": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "nb_density": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _int, _dbl, _dbl,
                          _dbl, _vp, _vp, _vp, _vp, _vp, _vp]),
    "nb_forces": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                         _i64, _vp, _int, _dbl, _dbl, _int, _vp, _vp, _vp, _vp, _vp, _vp]),
    "nb_forces_recon": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                               _vp, _vp, _i64, _vp, _int, _dbl, _dbl, _int, _int, _dbl, _dbl,
                               _int, _vp, _vp, _vp, _vp, _vp, _vp]),
    "nb_gradients": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _int, _vp,
                            _vp, _vp, _vp]),
    "nb_velocity_gradients": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _int,
                                     _vp, _vp]),
    "nb_deposit_log": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _int,
                              _int, _int, _int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "nb_deposit_box": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _int,
                              _int, _vp, _vp, _vp, _vp]),
    "nb_grid_finish": (_int, [_vp, _i64, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "nb_refine_sums": (_int, [_vp, _vp, _vp, _int, _int, _int, _vp, _int, _int, _int, _int, _int,
                              _int, _vp, _vp]),
    "nb_disc_forces": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _dbl, _vp, _vp,
                              _i64, _vp, _int, _vp, _vp, _vp]),
    "nb_glf_step_many": (_int, [_vp, _i64, _vp, _vp, _vp, _dbl, _vp, _vp, _vp, _vp]),
    "nb_integrate_orbit": (_int, [_vp, _int, _vp, _dbl, _dbl, _i64, _i64, _vp, _vp, _vp, _vp, _vp]),
    "nb_gn_v_from_p": (_int, [_vp, _i64, _vp, _vp, _vp, _vp]),
    "nb_gn_p_from_v": (_int, [_vp, _i64, _vp, _vp, _vp, _vp]),
    "nb_beta_cool": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "nb_brems_cool": (_int, [_vp, _i64, _vp, _vp, _vp, _dbl, _c.POINTER(NbParams), _vp, _vp]),
    "nb_ledger": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _c.POINTER(_dbl), _vp]),
    "nb_eos": (_int, [_vp, _i64, _vp, _vp, _c.POINTER(NbParams), _vp, _vp, _vp, _vp, _vp]),
    "nb_coupled_initialise": (_int, [_vp, _c.POINTER(NbState), _c.POINTER(NbParams), _vp]),
    "nb_coupled_step": (_int, [_vp, _c.POINTER(NbState), _c.POINTER(NbParams), _dbl, _vp]),
    "nb_coupled_stable_dt": (_int, [_vp, _c.POINTER(NbState), _c.POINTER(NbParams),
                                    _c.POINTER(_dbl), _vp]),
    "nb_block_initialise": (_int, [_vp, _c.POINTER(NbState), _c.POINTER(NbParams), _vp]),
    "nb_block_advance": (_int, [_vp, _c.POINTER(NbState), _c.POINTER(NbParams), _vp, _vp]),
    "nb_block_land": (_int, [_vp, _c.POINTER(NbState), _c.POINTER(NbParams), _vp]),
    "nb_block_advance_split": (_int, [_vp, _c.POINTER(NbState), _c.POINTER(NbParams), _vp, _vp, _vp,
                                      _vp]),
    "nb_block_finish": (_int, [_vp, _c.POINTER(NbState), _c.POINTER(NbParams), _i64, _vp, _int,
                               _vp, _vp, _vp]),
    "nb_block_wake_doomed": (_int, [_vp, _c.POINTER(NbState), _i64, _vp, _vp, _vp]),
    "nb_mlp_data": (_int, [_vp, _i64, _c.c_uint64, _c.POINTER(NbMlpParams), _vp, _vp, _vp, _vp]),
    "nb_mlp_grad": (_int, [_vp, _i64, _vp, _vp, _vp, _vp, _c.POINTER(_dbl), _vp]),
    "nb_mlp_train": (_int, [_vp, _c.POINTER(NbMlpParams), _i64, _i64, _int, _dbl, _c.c_uint64,
                            _vp, _vp]),
    "nb_mlp_weights": (_int, [_vp, _vp, _vp, _vp]),
    "nb_mlp_cool": (_int, [_vp, _i64, _vp, _vp, _vp, _dbl, _c.POINTER(NbMlpParams), _vp, _vp, _vp]),
    "nb_mlp_stats": (_int, [_vp, _c.POINTER(_dbl), _int]),
    "nb_density_noalloc": (_int, [_i64, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _int, _dbl,
                                  _dbl, _dbl, _vp, _vp, _vp, _vp, _vp, _vp]),
    "nb_noalloc_last_error": (_c.c_char_p, []),
}  # fmt: skip

EXPORTED = tuple(_SIGS)


def lib():
    """The loaded library (raises if it has not been built: no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m blackhole_nebula_simulator_b200.build`"
            )
        L = _c.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        for mirror, size_of in ((NbState, L.nb_state_size), (NbParams, L.nb_params_size)):
            if _c.sizeof(mirror) != size_of():
                raise ImportError(f"{LIB_PATH}: {mirror.__name__} is {_c.sizeof(mirror)} bytes, "
                                  f"the library's struct {size_of()} (stale build?)")  # fmt: skip
        _lib = L
    return _lib


_ERRORS = {
    11: GLFConvergenceError, 12: GLFConvergenceError, 13: GLFConvergenceError,
    20: RuntimeError, 21: RuntimeError, 22: FloatingPointError, 23: ValueError, 24: ValueError,
    25: NotImplementedError, 26: ValueError, 27: ValueError, 28: RuntimeError,
}  # fmt: skip


def check(ctx, status: int) -> None:
    if status == 0:
        return
    msg = lib().nb_last_error(ctx)
    msg = msg.decode() if msg else f"status {status}"
    raise _ERRORS.get(status, NebulaCudaError)(msg)
