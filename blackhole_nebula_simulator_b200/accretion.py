"""Removed-particle ledger (sim/accretion.py of the reference).

A particle is removed when, at the end of one of its own steps (its state then true, not
predicted), it is inside r_acc or beyond r_escape.  Its mass, energy m (H + u), angular momentum
m (x cross p) and momentum m p go into the ledger, which ``blocks.ledger`` adds to the totals of
the particles still present, so the conservation ledgers stay exact; each removal is logged with
its time, original id, reason, radius, m, H, u, |L|, the starting |L| and whether the particle
had passed a pericentre (a removal on the first approach is the reference's alarm).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class RemovedLedger:
    """sim/accretion.py:19-44."""

    mass: float = 0.0
    energy: float = 0.0  # sum m (H + u) at removal
    angmom: np.ndarray = field(default_factory=lambda: np.zeros(3))
    momentum: np.ndarray = field(default_factory=lambda: np.zeros(3))
    log: list = field(default_factory=list)

    @property
    def count(self) -> int:
        return len(self.log)

    def totals(self, reason: str) -> dict:
        """Mass, energy m (H + u) and count of the particles removed for ``reason``."""
        sel = [e for e in self.log if e["reason"] == reason]
        return {"count": len(sel), "mass": sum(e["m"] for e in sel),
                "energy": sum(e["m"] * (e["H"] + e["u"]) for e in sel)}  # fmt: skip

    def first_pass(self) -> list:
        """Removals of particles that had not yet passed a pericentre."""
        return [e for e in self.log if e["first_pass"]]


def record_removal(ledger: RemovedLedger, t, ids, mass, hamiltonian, u, angmom, p, r, passed, L0,
                   reason) -> None:  # fmt: skip
    """sim/accretion.py:47-62: arrays over the removed particles (host NumPy)."""
    for k in range(len(ids)):
        ledger.momentum = ledger.momentum + mass[k] * np.asarray(p[k], float)
        ledger.mass += float(mass[k])
        ledger.energy += float(mass[k] * (hamiltonian[k] + u[k]))
        ledger.angmom = ledger.angmom + mass[k] * np.asarray(angmom[k], float)
        ledger.log.append({"t": float(t), "id": int(ids[k]), "reason": reason, "r": float(r[k]),
                           "m": float(mass[k]), "H": float(hamiltonian[k]), "u": float(u[k]),
                           "L": float(np.linalg.norm(angmom[k])), "L0": float(L0[k]),
                           "first_pass": not bool(passed[k])})  # fmt: skip
