"""The semi-implicit midpoint method (WIND_METHOD_SIM, the reference's
python/pysolvers/sim.py:36-90) on the CPU: the oracle restatement against
the golden vectors of the reference's own sim.py, and the step count."""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import sim_cases as SC

CASES = SC.load()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_sim_matches_reference(case):
    name, net, y0, dt, m, y_ref = case
    y = y0.copy()
    tot, st, ns = O.restated_sim(net, y, 0.0, m * dt, m)
    assert SC.rel_err(y, y_ref) < SC.TOL
    assert tot == net.nsys * (m + 1)
    assert np.all(ns == m + 1) and np.all(st == 0)


def test_oracle_sim_single_step_is_first_plus_smoothing():
    """m = 1: D0 = A^-1 h f(y0), y1 = y0 + D0, ybar = y1 + A1^-1 (h f(y1) - D0)
    (Numerical Recipes 16.6 with one step), written out for the NR system."""
    name, net, y0, dt, m, _ = CASES[0]
    h = 0.01
    y = y0[:1].copy()
    O.restated_sim(net.subset(slice(0, 1)), y, 0.0, h, 1)
    f0, J0 = O.rhs_jac(net, 0, y0[0])
    A0 = np.eye(2) - h * J0.T
    d0 = np.linalg.solve(A0, h * f0)
    y1 = y0[0] + d0
    f1, J1 = O.rhs_jac(net, 0, y1)
    ybar = y1 + np.linalg.solve(np.eye(2) - h * J1.T, h * f1 - d0)
    assert SC.rel_err(y[0], ybar) < 1e-13
