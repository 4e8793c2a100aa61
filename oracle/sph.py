"""Density with list reuse, as the reference drives it (TEST INFRASTRUCTURE).

Restates sim/sph.py:62-147 (NeighbourCache, _reuse_limits) and sim/sph.py:329-387
(compute_density) on top of the C kernels in native.py.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import native
from .native import Neighbours

FLAG_OK, FLAG_AT_H_MAX, FLAG_SEARCH_TOO_SMALL, FLAG_NO_CONVERGENCE = 0, 1, 2, 3
FAST_SET_SIZES = (0, 1, 2, 4, 8, 16, 32, 64)  # sim/sph.py:114
KERNEL_IDS = {"cubic": 0, "wendland_c4": 1}
C_NORM = (1.0 / np.pi, 495.0 / (256.0 * np.pi))


@dataclass
class DensityResult:
    h: np.ndarray
    rho: np.ndarray
    omega: np.ndarray
    iterations: np.ndarray
    flags: np.ndarray
    neighbours: Neighbours
    cache: "NeighbourCache | None" = None


@dataclass
class NeighbourCache:
    neighbours: Neighbours
    x_ref: np.ndarray
    h_search: np.ndarray
    builds: int = 1
    reuses: int = 0


def density_numba(pos, mass, h_start, nb, h_search, kernel_name, eta, tol=1e-4, h_max=np.inf,
                  rows=None) -> DensityResult:  # fmt: skip
    kid = KERNEL_IDS[kernel_name]
    h, rho, om, it, fl = native.density(pos, mass, h_start, nb, h_search, kid, C_NORM[kid], eta,
                                        tol, h_max, rows)  # fmt: skip
    return DensityResult(h, rho, om, it, fl, nb)


def _min_image(d, box):
    return d if box is None else d - box * np.round(d / box)


def reuse_limits(cache: NeighbourCache, pos, h_guess, rows, others, box_arr):
    """sim/sph.py:117-147: per-particle search limits with which the cached lists are provably
    complete, or None when they must be rebuilt."""
    d = _min_image(np.asarray(pos, float) - cache.x_ref, box_arr)
    disp = np.sqrt(np.sum(d * d, axis=1))
    n = len(disp)
    top = min(n, FAST_SET_SIZES[-1] + 1)
    order = np.argpartition(-disp, top - 1)[:top] if top < n else np.arange(n)
    order = order[np.argsort(-disp[order], kind="stable")]
    for nf in FAST_SET_SIZES:
        if nf >= len(order):
            break
        h_eff = cache.h_search - 0.5 * (disp + disp[order[nf]])
        if not (np.all(h_eff[rows] > 0.5 * h_guess[rows]) and np.all(h_guess[others] <= h_eff[others])):
            continue
        if nf == 0:
            return h_eff
        h_lim = h_eff.copy()
        h_lim[others] = h_guess[others]
        if native.fast_rows_complete(pos, order[:nf], h_lim, box_arr, cache.neighbours):
            return h_eff
    return None


def compute_density(pos, mass, h_guess, box=None, kernel_name="wendland_c4", eta=1.6, tol=1e-4,
                    h_max=np.inf, skin=1.4, cache: NeighbourCache | None = None, rows=None,
                    reuse: bool = True) -> DensityResult:  # fmt: skip
    """sim/sph.py:329-387.  ``reuse=False`` skips the list-reuse test (always rebuild)."""
    h_guess = np.asarray(h_guess, float)
    n_all = len(pos)
    rows = np.arange(n_all, dtype=np.int64) if rows is None else np.asarray(rows, np.int64)
    others = np.ones(n_all, bool)
    others[rows] = False
    box_arr = None if box is None else np.broadcast_to(np.asarray(box, float), (3,))
    box_cap = np.inf if box_arr is None else 0.2499 * float(np.min(box_arr))
    if reuse and cache is not None and len(cache.x_ref) == len(pos) and len(pos):
        h_eff = reuse_limits(cache, pos, h_guess, rows, others, box_arr)
        if h_eff is not None:
            res = density_numba(pos, mass, h_guess, cache.neighbours, h_eff, kernel_name, eta, tol,
                                h_max, rows)  # fmt: skip
            if not np.any(res.flags == FLAG_SEARCH_TOO_SMALL):
                cache.reuses += 1
                res.cache = cache
                return res
            h_guess = h_guess.copy()
            h_guess[rows] = np.maximum(h_guess[rows], res.h)
    builds = 0 if cache is None else cache.builds
    h_search = np.minimum(np.minimum(h_guess, h_max) * skin, box_cap)
    for _ in range(12):
        nb = native.find_neighbours(pos, h_search, box=box_arr)
        builds += 1
        res = density_numba(pos, mass, h_guess, nb, h_search, kernel_name, eta, tol, h_max, rows)
        grow = res.flags == FLAG_SEARCH_TOO_SMALL
        if not np.any(grow):
            reuses = 0 if cache is None else cache.reuses
            res.cache = NeighbourCache(nb, np.array(pos, float), h_search.copy(), builds, reuses)
            return res
        h_search = h_search.copy()
        h_search[rows[grow]] = np.minimum(h_search[rows[grow]] * 2.0, box_cap)
        h_guess = h_guess.copy()
        h_guess[rows] = res.h
    raise RuntimeError("smoothing lengths kept outgrowing the neighbour search")
