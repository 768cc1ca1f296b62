"""Host-side checks of the batched 2D workload generator (no GPU)."""
import numpy as np

from janus_b200 import microstructures as micro


def test_batch_problems_are_seeded_and_in_range():
    a = micro.batch_2d_problems(6, seed=3, sizes=(64, 96, 128))
    b = micro.batch_2d_problems(6, seed=3, sizes=(64, 96, 128))
    for p, q in zip(a, b):
        assert p["n"] == q["n"] and np.array_equal(p["phase"], q["phase"])
        assert p["n"] in (64, 96, 128)
        assert p["phase"].shape == (p["n"], p["n"]) and p["phase"].dtype == np.uint8
        assert set(np.unique(p["phase"])) <= {0, 1}
        assert 0 < p["phase"].mean() < 1
        assert p["mu"][0] == 1.0 and 10.0 <= p["mu"][1] <= 1000.0
        assert np.all((0.15 <= p["nu"]) & (p["nu"] <= 0.4))
        assert p["mu0"] == 0.5 * (1.0 + p["mu"][1])
        k = p["mu"] / (1 - 2 * p["nu"])
        k0 = p["mu0"] / (1 - 2 * p["nu0"])
        assert abs(k0 - 0.5 * (k.min() + k.max())) <= 1e-12 * k0
    c = micro.batch_2d_problems(6, seed=4, sizes=(64, 96, 128))
    assert any(not np.array_equal(p["phase"], q["phase"]) or p["n"] != q["n"]
               for p, q in zip(a, c))
