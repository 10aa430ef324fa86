"""What the trained start-density network gains over the superposition start.

The committed weights (``amaterasu_b200/data/density_net_si8.npz``) were trained by
``python -m amaterasu_b200.learned_pipeline all --family si8`` on 48 seeded strained Si8
cells (seeds 1000-1047). Two held-out cells (seeds 5000, 5003) are converged from both
starts with the mixed-precision engine: the learned start must take fewer SCF iterations in
total and reach the same fixed point (|dF| < 1e-6 Ha; the network only changes the start).
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEIGHTS = Path(__file__).resolve().parents[1] / "amaterasu_b200" / "data" / "density_net_si8.npz"


@pytest.mark.skipif(not WEIGHTS.exists(), reason="trained weights not present")
def test_learned_start_saves_iterations_and_keeps_the_fixed_point():
    from amaterasu_b200.learned_pipeline import _pseudo, learned_start, run_cell
    pseudo = _pseudo()
    learned = learned_start(WEIGHTS, "si8")
    base_its, learned_its = 0, 0
    for seed in (5000, 5003):
        base = run_cell(seed, pseudo, family="si8")
        pred = run_cell(seed, pseudo, family="si8", density=learned.predict)
        assert base["converged"] and pred["converged"]
        assert not learned.stats["fallback"]
        assert abs(base["free_energy"] - pred["free_energy"]) < 1e-6
        base_its += base["iterations"]
        learned_its += pred["iterations"]
    print(f"SCF iterations: superposition {base_its}, learned {learned_its}")
    assert learned_its < base_its
