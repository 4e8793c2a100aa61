"""CPU oracle of the particle -> grid deposition (TEST INFRASTRUCTURE).

The per-particle passes in C (oracle.c: or_deposit_log, or_deposit_box, restating
render/gasgrid.py:316-597 with the reference's two fixed chunks, particle p to chunk p mod 2,
summed in order); the particle fields, the theta / phi tables and the cell fields in NumPy as
render/gasgrid.py:293-313, 660-692; refine_sums and the split as render/gasgrid.py:741-808.
The grid arguments are the package's LogSphericalGrid / CartesianBox.  Pinned to the
reference's outputs in tests/golden/deposit.npz.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import native

N_FIELDS = 6
N_CHUNKS = 2
KERNEL_IDS = {"cubic": 0, "wendland_c4": 1}
R_SUPPORT = 2.0
WIDE_CELLS = 24.0
COARSEN = (2, 4, 4)

_D = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_bound = False


def _lib():
    global _bound
    L = native.lib()
    if not _bound:
        i64, dbl, cint = ctypes.c_int64, ctypes.c_double, ctypes.c_int
        pi64 = ctypes.POINTER(ctypes.c_int64)
        pd = ctypes.POINTER(ctypes.c_double)
        L.or_deposit_log.argtypes = [i64, _D, _D, _D, _D, dbl, dbl, dbl, dbl, cint, cint, cint,
                                     cint, _D, _D, _D, _D, _D, cint, _D, pd, pi64]  # fmt: skip
        L.or_deposit_box.argtypes = [i64, _D, _D, _D, _D, dbl, dbl, dbl, dbl, cint, cint, cint,
                                     _D, pd, pi64]  # fmt: skip
        _bound = True
    return L


def _prepare(x, h, m, t, v):
    """render/gasgrid.py:660-676 without the chunk reordering (the C passes deal the chunks)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    h = np.ascontiguousarray(h, dtype=np.float64)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, float), h.shape), dtype=np.float64)
    t = np.asarray(t, float)
    v = np.asarray(v, float)
    vals = np.empty((len(h), N_FIELDS))
    vals[:, 0] = m
    vals[:, 1] = m * t
    vals[:, 2] = m * t**4
    vals[:, 3:6] = m[:, None] * v
    return x, h, m, vals


def finish(acc, vol, outside, n_tri) -> dict:
    """render/gasgrid.py:293-313."""
    mass = acc[..., 0]
    safe = np.where(mass > 0, mass, 1.0)
    has = mass > 0
    t_mass = np.where(has, acc[..., 1] / safe, 0.0)
    t_em = np.where(has, np.maximum(acc[..., 2] / safe, 0.0) ** 0.25, 0.0)
    vel = np.where(has[..., None], acc[..., 3:6] / safe[..., None], 0.0)
    return dict(mass=mass, rho=(mass / vol).astype(np.float32), t_mass=t_mass.astype(np.float32),
                t_em=t_em.astype(np.float32), vel=vel.astype(np.float32), outside=float(outside),
                n_trilinear=int(n_tri))  # fmt: skip


def log_accumulate(x, h, m, t, v, g, kernel="wendland_c4"):
    x, h, m, vals = _prepare(x, h, m, t, v)
    acc = np.zeros((*g.shape, N_FIELDS))
    tab = g.tables()
    out, ntri = ctypes.c_double(), ctypes.c_int64()
    _lib().or_deposit_log(len(h), x.reshape(-1), h, m, vals.reshape(-1), g.r_min, g.dlnr, g.dth,
                          g.dph, g.nr, g.nth, g.nph, KERNEL_IDS[kernel], tab["sth"], tab["cth"],
                          tab["dcth"], tab["cph"], tab["sph"], N_CHUNKS, acc.reshape(-1),
                          ctypes.byref(out), ctypes.byref(ntri))  # fmt: skip
    return acc, out.value, ntri.value


def deposit_log(x, h, m, t, v, g, kernel="wendland_c4") -> dict:
    """render/gasgrid.py:722-738."""
    acc, out, ntri = log_accumulate(x, h, m, t, v, g, kernel)
    return finish(acc, g.volumes()[:, :, None], out, ntri)


def deposit_box(x, h, m, t, v, b, kernel="wendland_c4") -> dict:
    """render/gasgrid.py:811-825."""
    x, h, m, vals = _prepare(x, h, m, t, v)
    acc = np.zeros((*b.shape, N_FIELDS))
    lo = b.lo
    out, ntri = ctypes.c_double(), ctypes.c_int64()
    _lib().or_deposit_box(len(h), x.reshape(-1), h, m, vals.reshape(-1), lo[0], lo[1], lo[2], b.dx,
                          b.n, KERNEL_IDS[kernel], N_CHUNKS, acc.reshape(-1), ctypes.byref(out),
                          ctypes.byref(ntri))  # fmt: skip
    return finish(acc, np.full((1, 1, 1), b.dx**3), out.value, ntri.value)


def wide_particles(x, h, g, wide_cells=WIDE_CELLS):
    """render/gasgrid.py:751-754."""
    r = np.linalg.norm(np.asarray(x, float), axis=1)
    return R_SUPPORT * np.asarray(h, float) >= wide_cells * np.maximum(r, g.r_min) * g.dth


def refine_sums(acc_c, gc, g, coarsen=COARSEN):
    """render/gasgrid.py:757-788."""
    cr, ct, cp = coarsen
    dens = acc_c / gc.volumes()[:, :, None, None]

    def axis(n_fine, c, n_coarse, periodic):
        f = (np.arange(n_fine) + 0.5) / c - 0.5
        if periodic:
            i0 = np.floor(f).astype(int)
            return i0 % n_coarse, (i0 + 1) % n_coarse, f - i0
        f = np.clip(f, 0.0, n_coarse - 1.0)
        if n_coarse > 1:
            i0 = np.minimum(np.floor(f).astype(int), n_coarse - 2)
        else:
            i0 = np.zeros(n_fine, int)
        return i0, np.minimum(i0 + 1, n_coarse - 1), f - i0

    ri0, ri1, rw = axis(g.nr, cr, gc.nr, False)
    ti0, ti1, tw = axis(g.nth, ct, gc.nth, False)
    pi0, pi1, pw = axis(g.nph, cp, gc.nph, True)
    out = np.zeros((g.nr, g.nth, g.nph, acc_c.shape[-1]))
    for a, wa in ((ri0, 1 - rw), (ri1, rw)):
        for b, wb in ((ti0, 1 - tw), (ti1, tw)):
            for c, wc in ((pi0, 1 - pw), (pi1, pw)):
                w = wa[:, None, None] * wb[None, :, None] * wc[None, None, :]
                out += w[..., None] * dens[a][:, b][:, :, c]
    out *= g.volumes()[:, :, None, None]
    if out[..., 0].sum() > 0:
        out *= acc_c[..., 0].sum() / out[..., 0].sum()
    return out


def deposit_log_split(x, h, m, t, v, g, coarse, kernel="wendland_c4", wide_cells=WIDE_CELLS,
                      coarsen=COARSEN) -> dict:  # fmt: skip
    """render/gasgrid.py:791-808; coarse: the coarse grid (coarse_log_grid of g)."""
    x = np.asarray(x, float)
    h = np.asarray(h, float)
    m = np.broadcast_to(np.asarray(m, float), h.shape)
    t, v = np.asarray(t, float), np.asarray(v, float)
    wide = wide_particles(x, h, g, wide_cells)
    total, outside, n_tri = log_accumulate(x[~wide], h[~wide], m[~wide], t[~wide], v[~wide], g,
                                           kernel)  # fmt: skip
    if wide.any():
        acc_c, out_c, tri_c = log_accumulate(x[wide], h[wide], m[wide], t[wide], v[wide], coarse,
                                             kernel)  # fmt: skip
        total = total + refine_sums(acc_c, coarse, g, coarsen)
        outside, n_tri = outside + out_c, n_tri + tri_c
    res = finish(total, g.volumes()[:, :, None], outside, n_tri)
    res["n_wide"] = int(wide.sum())
    return res
