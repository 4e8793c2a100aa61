"""ctypes binding of liboracle.so (TEST INFRASTRUCTURE: the CPU checker, never the product).

Each wrapper takes and returns NumPy arrays with the reference's conventions (float64 C-order,
int64 CSR lists, results in ``rows`` order) and names the reference function it mirrors.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_D = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_U8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64
_dbl = ctypes.c_double
_int = ctypes.c_int


def build() -> str:
    """Compile liboracle.so with its Makefile (plain gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "oracle.c")
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.or_find_neighbours.restype = _i64
        L.or_find_neighbours.argtypes = [_i64, _D, _D, _D, ctypes.POINTER(ctypes.POINTER(_i64)),
                                         ctypes.POINTER(ctypes.POINTER(_i64))]  # fmt: skip
        L.or_free.argtypes = [ctypes.c_void_p]
        L.or_cells.argtypes = [_i64, _D, _D, _D, _D, _I, _I]
        L.or_tighten.argtypes = [_i64, _D, _D, _D, _I, _I, _i64, _I, _I, ctypes.c_void_p,
                                 ctypes.c_void_p]  # fmt: skip
        L.or_density.argtypes = [_i64, _D, _D, _D, _D, _I, _I, _D, _int, _dbl, _dbl, _dbl, _dbl,
                                 _i64, _I, _D, _D, _D, _I, _I]  # fmt: skip
        L.or_forces.argtypes = [_D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _I, _I, _D, _int, _dbl,
                                _int, _int, _dbl, _dbl, _int, _int, _int, _dbl, _dbl, _int, _D,
                                _i64, _I, _D, _D, _D, _D, _D]  # fmt: skip
        L.or_gradients.argtypes = [_D, _D, _D, _D, _D, _I, _I, _D, _int, _dbl, _i64, _I, _D, _D,
                                   _D]  # fmt: skip
        L.or_velocity_gradients.argtypes = [_D, _D, _D, _D, _I, _I, _D, _int, _dbl, _i64, _I, _D]
        L.or_disc_forces.argtypes = [_D, _D, _D, _D, _D, _D, _D, _dbl, _I, _I, _D, _int, _dbl,
                                     _i64, _I, _D, _D]  # fmt: skip
        L.or_glf_many.argtypes = [_i64, _D, _D, _D, _D, _D, _I]
        L.or_gn_v_from_p.argtypes = [_i64, _D, _D, _D]
        L.or_fast_rows_complete.restype = _int
        L.or_fast_rows_complete.argtypes = [_i64, _D, _i64, _I, _D, _D, _I, _I]
        L.or_limit_rows.argtypes = [_I, _i64, _I, _I, _I, _i64]
        L.or_wake_targets.argtypes = [_I, _i64, _I, _I, _I, _i64, _I]
        L.or_mark_neighbours.argtypes = [_i64, _I, _I, _I, _U8]
        L.or_kernel_f.restype = _dbl
        L.or_gasrad_temperature.argtypes = [_i64, _D, _D, _dbl, _dbl, _D, _U8]
        L.or_kernel_f.argtypes = [_dbl, _int]
        L.or_kernel_df.restype = _dbl
        L.or_kernel_df.argtypes = [_dbl, _int]
        _lib = L
    return _lib


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, np.float64)
    if shape is not None:
        a = np.ascontiguousarray(np.broadcast_to(a, shape))
    return a


def _box3(box):
    return np.zeros(3) if box is None else _f64(np.broadcast_to(np.asarray(box, float), (3,)))


@dataclass
class Neighbours:
    """CSR lists (sim/neighbours.py:22-36): neighbours of i are index[offset[i]:offset[i+1]]."""

    offset: np.ndarray
    index: np.ndarray
    box: np.ndarray | None

    def of(self, i: int) -> np.ndarray:
        return self.index[self.offset[i] : self.offset[i + 1]]

    @property
    def counts(self) -> np.ndarray:
        return np.diff(self.offset)


def find_neighbours(pos, h, box=None) -> Neighbours:
    """sim/neighbours.py:240-281 find_neighbours_numba (grid, transpose, merge)."""
    pos = _f64(pos)
    h = _f64(h)
    n = len(pos)
    box_arr = None if box is None else _box3(box)
    if box_arr is not None and np.any(2.0 * h.max() >= 0.5 * box_arr):
        raise ValueError("kernel support exceeds half the periodic box: neighbours ambiguous")
    off_p = ctypes.POINTER(_i64)()
    idx_p = ctypes.POINTER(_i64)()
    m = lib().or_find_neighbours(n, pos.reshape(-1), h, _box3(box), ctypes.byref(off_p),
                                 ctypes.byref(idx_p))  # fmt: skip
    off = np.ctypeslib.as_array(off_p, shape=(n + 1,)).copy()
    idx = np.ctypeslib.as_array(idx_p, shape=(max(m, 1),))[:m].copy()
    lib().or_free(ctypes.cast(off_p, ctypes.c_void_p))
    lib().or_free(ctypes.cast(idx_p, ctypes.c_void_p))
    return Neighbours(off, idx, box_arr)


def grid_cells(pos, h):
    """Cell index of every particle in the reference grid (sim/neighbours.py:106-126, 256-265):
    returns (cell (N,) int64, lo (3,), inv_cell (3,), ncell (3,))."""
    pos = _f64(pos)
    h = _f64(h)
    lo, inv = np.zeros(3), np.zeros(3)
    nc = np.zeros(3, np.int64)
    cell = np.zeros(len(pos), np.int64)
    lib().or_cells(len(pos), pos.reshape(-1), h, lo, inv, nc, cell)
    return cell, lo, inv, nc


def _rows(rows, n):
    return np.arange(n, dtype=np.int64) if rows is None else np.ascontiguousarray(rows, np.int64)


def tighten(nb: Neighbours, pos, h, rows=None) -> Neighbours:
    """sim/neighbours.py:284-323: keep r < 2 max(h_i, h_j), lists for ``rows`` only."""
    pos = _f64(pos)
    h = _f64(h)
    n = len(pos)
    rows = _rows(rows, n)
    box = _box3(nb.box)
    counts = np.zeros(n, np.int64)
    lib().or_tighten(n, pos.reshape(-1), h, box, nb.offset, nb.index, len(rows), rows, counts,
                     None, None)  # fmt: skip
    off = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    idx = np.empty(max(int(off[-1]), 1), np.int64)
    lib().or_tighten(n, pos.reshape(-1), h, box, nb.offset, nb.index, len(rows), rows, counts,
                     off.ctypes.data, idx.ctypes.data)  # fmt: skip
    return Neighbours(off, idx[: off[-1]], nb.box)


def density(pos, mass, h_start, nb: Neighbours, h_search, kid, cnorm, eta, tol=1e-4,
            h_max=np.inf, rows=None):  # fmt: skip
    """sim/sph.py:300-326 density_numba: (h, rho, omega, iterations, flags) in rows order."""
    pos = _f64(pos)
    n = len(pos)
    rows = _rows(rows, n)
    m = len(rows)
    h_out, rho, omega = np.empty(m), np.empty(m), np.empty(m)
    iters, flags = np.empty(m, np.int64), np.empty(m, np.int64)
    lib().or_density(
        n, pos.reshape(-1), _f64(mass, (n,)), _f64(h_start, (n,)), _f64(h_search, (n,)),
        nb.offset, nb.index, _box3(nb.box), int(kid), float(cnorm), float(eta), float(tol),
        float(h_max), m, rows, h_out, rho, omega, iters, flags,
    )  # fmt: skip
    return h_out, rho, omega, iters, flags


def forces(pos, vel, mass, h, rho, omega, pressure, nb: Neighbours, kid, cnorm, u=None,
           c_s=None, alpha=None, beta=2.0, alpha_u=1.0, cond_signal=0, rows=None, grad_v=None,
           closeness=True, eta_crit=1.0 / 1.2, eta_fold=0.2, gate=2):  # fmt: skip
    """sim/sph.py:655-690 forces_numba: (acc, dudt, vsig, dudt_visc, dudt_cond) in rows order;
    velocity reconstruction (with the ShockCapturing fields closeness, eta_crit, eta_fold,
    recon_gate) when ``grad_v`` (N, 3, 3) is given."""
    pos = _f64(pos)
    n = len(pos)
    rows = _rows(rows, n)
    m = len(rows)
    use_visc = alpha is not None and c_s is not None
    use_cond = use_visc and u is not None
    z = np.zeros(n)
    arr = lambda a: z if a is None else _f64(a, (n,))  # noqa: E731
    use_recon = use_visc and grad_v is not None
    gv = _f64(grad_v, (n, 3, 3)).reshape(-1) if use_recon else np.zeros(9)
    acc = np.empty((m, 3))
    dudt, vsig, vh, ch = np.empty(m), np.empty(m), np.empty(m), np.empty(m)
    lib().or_forces(
        pos.reshape(-1), _f64(vel).reshape(-1), _f64(mass, (n,)), _f64(h), _f64(rho),
        _f64(omega), _f64(pressure), arr(u), arr(c_s), arr(alpha), nb.offset, nb.index,
        _box3(nb.box), int(kid), float(cnorm), int(use_visc), int(use_cond), float(beta),
        float(alpha_u), int(cond_signal), int(use_recon), int(bool(closeness)), float(eta_crit),
        float(eta_fold), int(gate), gv, m, rows, acc.reshape(-1), dudt, vsig, vh, ch,
    )  # fmt: skip
    return acc, dudt, vsig, vh, ch


def gradients(pos, vel, acc, mass, h, nb: Neighbours, kid, cnorm, rows=None):
    """sim/sph.py:883-902 gradients_numba: (div v, |curl v|, d(div v)/dt) in rows order."""
    pos = _f64(pos)
    n = len(pos)
    rows = _rows(rows, n)
    m = len(rows)
    div, curl, ddiv = np.empty(m), np.empty(m), np.empty(m)
    lib().or_gradients(pos.reshape(-1), _f64(vel).reshape(-1), _f64(acc).reshape(-1),
                       _f64(mass, (n,)), _f64(h, (n,)), nb.offset, nb.index, _box3(nb.box),
                       int(kid), float(cnorm), m, rows, div, curl, ddiv)  # fmt: skip
    return div, curl, ddiv


def velocity_gradients(pos, vel, mass, h, nb: Neighbours, kid, cnorm, rows=None, out=None):
    """sim/sph.py:827-846 velocity_gradients_numba: fills out (N, 3, 3; zeros if not given) at
    rows and returns it."""
    pos = _f64(pos)
    n = len(pos)
    rows = _rows(rows, n)
    out = np.zeros((n, 3, 3)) if out is None else out
    lib().or_velocity_gradients(pos.reshape(-1), _f64(vel).reshape(-1), _f64(mass, (n,)),
                                _f64(h, (n,)), nb.offset, nb.index, _box3(nb.box), int(kid),
                                float(cnorm), len(rows), rows, out.reshape(-1))  # fmt: skip
    return out


def disc_forces(pos, vel, mass, h, rho, omega, c_s, alpha_av, nb: Neighbours, kid, cnorm,
                rows=None):  # fmt: skip
    """sim/sph.py:1120-1137 disc_forces_numba: (acc, dudt) in rows order."""
    pos = _f64(pos)
    n = len(pos)
    rows = _rows(rows, n)
    m = len(rows)
    acc, dudt = np.empty((m, 3)), np.empty(m)
    lib().or_disc_forces(
        pos.reshape(-1), _f64(vel).reshape(-1), _f64(mass, (n,)), _f64(h), _f64(rho),
        _f64(omega), _f64(c_s), float(alpha_av), nb.offset, nb.index, _box3(nb.box), int(kid),
        float(cnorm), m, rows, acc.reshape(-1), dudt,
    )  # fmt: skip
    return acc, dudt


class GLFConvergenceError(RuntimeError):
    pass


_GLF_MESSAGES = {
    -1: "stage 1 (p_half) did not converge in 10 iterations: time step too large",
    -2: "stage 2 (x1) did not converge in 10 iterations: time step too large",
    -3: "particle inside r = 2.5",
    -4: "time step would need more than 40 halvings of dt_max",
}


def glf_step_many(x, p, dt, raise_on_failure=True):
    """sim/integrator.py:188-198 glf_step_many: (x1, p1, iterations)."""
    x = _f64(x)
    p = _f64(p)
    n = len(x)
    dt = _f64(dt, (n,))
    xo, po = np.empty_like(x), np.empty_like(p)
    it = np.empty(n, np.int64)
    lib().or_glf_many(n, x.reshape(-1), p.reshape(-1), dt, xo.reshape(-1), po.reshape(-1), it)
    if raise_on_failure and np.any(it < 0):
        first = int(np.argmax(it < 0))
        raise GLFConvergenceError(f"particle {first}: {_GLF_MESSAGES[int(it[first])]}")
    return xo, po, it


def gn_v_from_p(x, p):
    """sim/fastphys.py:35-42: v = A p + C (p.x) x."""
    x = _f64(x)
    out = np.empty_like(x)
    lib().or_gn_v_from_p(len(x), x.reshape(-1), _f64(p).reshape(-1), out.reshape(-1))
    return out


def fast_rows_complete(pos, fast, h_lim, box, nb: Neighbours) -> bool:
    pos = _f64(pos)
    return bool(lib().or_fast_rows_complete(len(pos), pos.reshape(-1), len(fast),
                                            np.ascontiguousarray(fast, np.int64), _f64(h_lim),
                                            _box3(box), nb.offset, nb.index))  # fmt: skip


def limit_rows(level, rows, nb: Neighbours, max_gap):
    lib().or_limit_rows(level, len(rows), np.ascontiguousarray(rows, np.int64), nb.offset,
                        nb.index, int(max_gap))  # fmt: skip


def wake_targets(level, rows, nb: Neighbours, max_gap, need):
    lib().or_wake_targets(level, len(rows), np.ascontiguousarray(rows, np.int64), nb.offset,
                          nb.index, int(max_gap), need)  # fmt: skip


def with_neighbours(nb: Neighbours, rows, n):
    """sim/blocks.py:201-214: the rows together with everything in their lists (sorted)."""
    mark = np.zeros(n, np.uint8)
    rows = np.ascontiguousarray(rows, np.int64)
    lib().or_mark_neighbours(len(rows), rows, nb.offset, nb.index, mark)
    return np.flatnonzero(mark)


def gasrad_temperature(rho_si, u_si, a1, a_rad):
    """sim/fastphys.py:45-71 element by element: (T [K], converged flags)."""
    rho, u = _f64(rho_si), _f64(u_si)
    out = np.empty(len(rho))
    ok = np.empty(len(rho), np.uint8)
    lib().or_gasrad_temperature(len(rho), rho, u, a1, a_rad, out, ok)
    return out, ok.astype(bool)
