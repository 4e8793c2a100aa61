"""Removed-particle ledger (the interface of sim/accretion.py in the reference).

A particle is removed when, at the end of one of its own steps (its state then true, not
predicted), it is inside r_acc or beyond r_escape.  Its mass, energy m (H + u), angular momentum
m (x cross p) and momentum m p go into the ledger, which ``blocks.ledger`` adds to the totals of
the particles still present, so the conservation ledgers stay exact.  Every removal is logged
with its time, original id, reason, radius, m, H, u, |L|, the starting |L| and whether the
particle had passed a pericentre (a removal on the first approach is the reference's alarm).

Storage is columnar: each call appends one batch of NumPy columns, the running totals are
updated with one vectorised sum per batch, and the per-removal dictionaries of ``log`` (the
reference's record format, which drivers read) are built only when asked for.
"""

from __future__ import annotations

import numpy as np

# log record keys, in the reference's order (sim/accretion.py:52-61)
_SCALAR_COLUMNS = ("t", "id", "reason", "r", "m", "H", "u", "L", "L0", "first_pass")
_CASTS = {"t": float, "id": int, "reason": str, "r": float, "m": float, "H": float, "u": float,
          "L": float, "L0": float, "first_pass": bool}  # fmt: skip


class RemovedLedger:
    """Totals and a log of the particles removed from a run (sim/accretion.py:19-44).

    ``mass``, ``energy`` (sum m (H + u) at removal), ``angmom`` (sum m x cross p) and
    ``momentum`` (sum m p) are running totals; ``log`` is one dictionary per removed particle in
    removal order; ``count``, ``totals(reason)`` and ``first_pass()`` read the columns."""

    def __init__(self):
        self.mass = 0.0
        self.energy = 0.0
        self.angmom = np.zeros(3)
        self.momentum = np.zeros(3)
        self._batches: list[dict[str, np.ndarray]] = []

    def add_batch(self, t, ids, mass, hamiltonian, u, angmom, p, r, passed, L0, reason):
        """Append the removed particles of one step (arrays over them, all for ``reason``)."""
        m = np.asarray(mass, dtype=np.float64).reshape(-1)
        k = len(m)
        if k == 0:
            return
        am = np.asarray(angmom, dtype=np.float64).reshape(k, 3)
        mom = np.asarray(p, dtype=np.float64).reshape(k, 3)
        ham = np.asarray(hamiltonian, dtype=np.float64).reshape(k)
        uu = np.asarray(u, dtype=np.float64).reshape(k)
        self.mass += float(m.sum())
        self.energy += float(np.dot(m, ham + uu))
        self.angmom = self.angmom + m @ am
        self.momentum = self.momentum + m @ mom
        self._batches.append({
            "t": np.full(k, float(t)), "id": np.asarray(ids, dtype=np.int64).reshape(k),
            "reason": np.full(k, reason, dtype=object), "r": np.asarray(r, np.float64).reshape(k),
            "m": m, "H": ham, "u": uu, "L": np.sqrt(np.einsum("ij,ij->i", am, am)),
            "L0": np.asarray(L0, dtype=np.float64).reshape(k),
            "first_pass": ~np.asarray(passed, dtype=bool).reshape(k),
        })  # fmt: skip

    def _column(self, name: str) -> np.ndarray:
        if not self._batches:
            return np.zeros(0, dtype=object if name == "reason" else np.float64)
        return np.concatenate([b[name] for b in self._batches])

    @property
    def count(self) -> int:
        return sum(len(b["m"]) for b in self._batches)

    def _records(self, select: np.ndarray | None = None) -> list:
        cols = {name: self._column(name) for name in _SCALAR_COLUMNS}
        rows = np.arange(self.count) if select is None else np.flatnonzero(select)
        return [{name: _CASTS[name](cols[name][i]) for name in _SCALAR_COLUMNS} for i in rows]

    @property
    def log(self) -> list:
        """One dictionary per removed particle, in removal order (the reference's records)."""
        return self._records()

    def totals(self, reason: str) -> dict:
        """Count, mass and energy m (H + u) of the particles removed for ``reason``."""
        sel = self._column("reason") == reason
        m = self._column("m")[sel]
        e = m * (self._column("H")[sel] + self._column("u")[sel])
        return {"count": int(sel.sum()), "mass": float(m.sum()), "energy": float(e.sum())}

    def first_pass(self) -> list:
        """Removals of particles that had not yet passed a pericentre."""
        return self._records(self._column("first_pass").astype(bool))


def record_removal(ledger: RemovedLedger, t, ids, mass, hamiltonian, u, angmom, p, r, passed, L0,
                   reason) -> None:  # fmt: skip
    """sim/accretion.py:47-62: add the removed particles (host arrays over them) to the ledger."""
    ledger.add_batch(t, ids, mass, hamiltonian, u, angmom, p, r, passed, L0, reason)
