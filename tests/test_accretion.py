"""The removed-particle ledger (sim/accretion.py of the reference): totals, per-reason sums and
the first-approach alarm, on the host."""

import numpy as np

from blackhole_nebula_simulator_b200.accretion import RemovedLedger, record_removal
from tests.conftest import check


def test_ledger_totals_and_log():
    led = RemovedLedger()
    x = np.array([[3.0, 0.0, 0.0], [0.0, 5.0e4, 0.0]])
    p = np.array([[0.0, 0.4, 0.0], [0.0, 0.1, 0.2]])
    am = np.cross(x, p)
    record_removal(led, 12.5, np.array([7]), np.array([2.0]), np.array([-0.1]), np.array([0.01]),
                   am[:1], p[:1], np.array([3.0]), np.array([False]), np.array([1.5]),
                   "accreted")  # fmt: skip
    record_removal(led, 13.0, np.array([9]), np.array([1.0]), np.array([0.2]), np.array([0.03]),
                   am[1:], p[1:], np.array([5.0e4]), np.array([True]), np.array([2.0]),
                   "escaped")  # fmt: skip
    check("count", 2, led.count)
    check("mass", 3.0, led.mass)
    check("energy", 2.0 * (-0.1 + 0.01) + 1.0 * (0.2 + 0.03), led.energy, rtol=1e-15)
    check("angular momentum", 2.0 * am[0] + am[1], led.angmom, rtol=1e-15)
    check("momentum", 2.0 * p[0] + p[1], led.momentum, rtol=1e-15)
    acc = led.totals("accreted")
    check("accreted count", 1, acc["count"])
    check("accreted energy", 2.0 * (-0.1 + 0.01), acc["energy"], rtol=1e-15)
    check("escaped mass", 1.0, led.totals("escaped")["mass"])
    check("first-approach alarm", [7], [e["id"] for e in led.first_pass()])
    check("|L| logged", float(np.linalg.norm(am[0])), led.log[0]["L"], rtol=1e-15)
