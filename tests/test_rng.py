"""Random-number pins: the oracle's streams against the reference's own
jump constants and an independent big-integer evaluation
(tests/golden/rng_golden.json, made by tests/golden/make_golden.py)."""
import json
import os

import numpy as np

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "rng_golden.json")))


def test_reference_jump_constants_are_powers():
    # ecuyer_cote_mod.f90:14-15: a1w = a1^(2^30), a1vw = a1^(2^50) (mod m)
    assert all(GOLD["checks"].values())


def test_oracle_streams_match_bigint(oracle_mod):
    for case in GOLD["cases"]:
        xi, seeds = oracle_mod.rng(case["seed1"], case["seed2"], case["generator"], case["block"], len(case["xi"]))
        assert int(seeds[0]) == case["s1"] and int(seeds[1]) == case["s2"], case
        np.testing.assert_array_equal(xi, np.array(case["xi"]))


def test_uniforms_in_open_interval(oracle_mod):
    xi, _ = oracle_mod.rng(12345678, 87654321, 1, 0, 200000)
    assert xi.min() > 0.0 and xi.max() < 1.0
    # first two moments of U(0,1)
    assert abs(xi.mean() - 0.5) < 5e-3
    assert abs(xi.var() - 1.0 / 12.0) < 5e-3


def test_zeta_table(oracle_mod):
    # bbfreq's table (random.f90:227-245) is the partial sums of zeta(4) = pi^4/90
    z = oracle_mod.inczeta()
    assert abs(z[-1] - np.pi ** 4 / 90.0) < 1e-6
    assert np.all(np.diff(z) > 0)
    assert z[0] == 1.0
