"""Host-side logic of the learned warm start, without a GPU: the
imaginary-time stopping rule on synthetic energy sequences, the seeded
problem family and the Thomas-Fermi chemical potential."""
import math

import numpy as np

from libgrid_b200 import warmstart as ws


def _run(energies, tol=1e-8, rule="remainder"):
    a_prev = None
    for k in range(1, len(energies)):
        stop, a_prev = ws.converged(energies[k - 1] - energies[k], a_prev, tol, rule)
        if stop:
            return k
    return None


def test_remainder_rule_stops_within_tol_of_the_limit():
    # E_k = E_inf + c q^k for several rates: the rule stops at the first read
    # whose estimated remainder is below tol / 2, so the stopped energy lies
    # within tol of the limit, and not long after that point
    for q in (0.5, 0.8, 0.95, 0.99):
        for c in (1e-3, 1e-5):
            e_inf = 0.0123
            es = [e_inf + c * q**k for k in range(20000)]
            k = _run(es)
            assert k is not None
            assert es[k] - e_inf < 1e-8, (q, c, k)
            first = next(j for j in range(len(es)) if es[j] - e_inf < 0.5e-8)
            assert k <= first + 2 + int(math.log(2) / -math.log(q)), (q, c, k, first)


def test_change_rule_can_stop_far_from_the_limit():
    # a slow geometric tail: the 10-step change drops below tol while the
    # energy is still more than tol above the limit (why the remainder rule
    # is the default)
    q, c, e_inf = 0.995, 1e-4, 0.0
    es = [e_inf + c * q**k for k in range(20000)]
    k = _run(es, rule="change")
    assert es[k] - e_inf > 1e-8


def test_remainder_rule_handles_rising_and_flat_energies():
    # a rise (negative decrement) resets the ratio estimate; a flat
    # sequence stops at once
    es = [1.0, 0.9, 0.95, 0.94, 0.939, 0.9389]
    assert _run(es) is None
    assert _run([0.5, 0.5]) == 1


def test_problem_family_is_seeded_and_in_range():
    k1, g1, b1 = ws.problem_params(1234)
    k2, g2, b2 = ws.problem_params(1234)
    assert (k1, g1) == (k2, g2) and len(b1) == len(b2)
    for sd in range(50):
        k, g, bumps = ws.problem_params(sd)
        assert 0.005 <= k <= 0.02 and 0.001 <= g <= 0.01
        assert 1 <= len(bumps) <= 6
        for amp, w, c in bumps:
            assert 0.5e-3 <= abs(amp) <= 2e-3 and 0.2 <= w <= 0.6 and np.all(np.abs(c) <= 0.8)


def test_thomas_fermi_profile_is_normalised():
    v, g, _ = ws.sample_problem(7, n=32, step=0.1)
    tf = ws.thomas_fermi(v, g, 0.1)
    assert abs((tf**2).sum() * 0.1**3 - 1.0) < 1e-9
    mu = ws.thomas_fermi_mu(v, g, 0.1)
    assert np.all(tf[v >= mu] == 0.0)
