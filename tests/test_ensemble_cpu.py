"""CPU checks of the ensemble's member generator: sizes, kinds and the
log-uniform beta / eta draws, and the deck scaling to the requested beta."""
import math

import numpy as np

from lare3d_b200.ensemble import MemberSpec, member_deck, member_specs


def test_member_specs_distribution():
    s = member_specs(48, seed=2024)
    assert len(s) == 48
    assert s == member_specs(48, seed=2024)                      # seeded
    ns = [m.n for m in s]
    assert min(ns) >= 32 and max(ns) <= 128 and all(n % 8 == 0 for n in ns)
    assert len(set(ns)) >= 6                                     # uneven sizes
    kinds = {m.kind for m in s}
    assert kinds == {"blast", "orszag_tang"}
    assert all(0.01 <= m.beta <= 10 and 1e-4 <= m.eta <= 1e-2 for m in s)
    lb = np.log10([m.beta for m in s])
    assert lb.min() < -1 and lb.max() > 0                        # spans the decades


def test_member_deck_beta_and_eta():
    d = member_deck(MemberSpec("blast", 8, 0.05, 3e-3, 1))
    b2 = d.state["bx"][2, 2, 2] ** 2 + d.state["by"][2, 2, 2] ** 2
    assert abs(2 * 0.1 / b2 - 0.05) < 1e-12
    assert d.params.resistive_mhd == 1 and d.params.eta_background == 3e-3
    d = member_deck(MemberSpec("orszag_tang", 16, 0.3, 2e-4, 2))
    n = 16
    bx = d.state["bx"][2:n + 2, 1:n + 1, 1:n + 1]
    by = d.state["by"][1:n + 1, 2:n + 2, 1:n + 1]
    bz = d.state["bz"][1:n + 1, 1:n + 1, 2:n + 2]
    b2 = np.mean(bx ** 2) + np.mean(by ** 2) + np.mean(bz ** 2)
    p0 = 5.0 / (12.0 * math.pi)
    assert abs(2 * p0 / b2 / 0.3 - 1.0) < 0.02
    assert d.params.eta_background == 2e-4
