"""Replica exchange rule (CPU): ParallelTempering.exchange of the reference,
src/ParallelTempering.py:164-203, restated here as the expectation."""
import random
from math import exp

from espressopp_b200.parallel_tempering import exchange_decisions


def _reference_rule(energies, temperatures, nparts, oddeven, draws):
    out = []
    it = iter(draws)
    for i in range(len(energies) // 2):
        m = 2 * i + oddeven
        n = m + 1
        if n < len(energies):
            metro = next(it)
            delta = (1 / temperatures[n] - 1 / temperatures[m]) * (
                energies[m] / nparts[m] - energies[n] / nparts[n])
            out.append((m, n, delta <= 0 or exp(-delta) > metro))
    return out


def test_exchange_rule_matches_reference():
    rng = random.Random(335977)
    for trial in range(200):
        R = rng.randint(2, 9)
        e = [rng.uniform(-6.0, -1.0) * 1000 for _ in range(R)]
        t = [0.7 * (2.0 / 0.7) ** (r / max(R - 1, 1)) + rng.uniform(-0.05, 0.05) for r in range(R)]
        n = [rng.randint(1000, 5000) for _ in range(R)]
        draws = [rng.random() for _ in range(R)]
        for oddeven in (0, 1):
            it = iter(draws)
            got = exchange_decisions(e, t, n, oddeven, lambda: next(it))
            want = _reference_rule(e, t, n, oddeven, draws)
            assert [(m, k, ok) for m, k, _, _, ok in got] == want
