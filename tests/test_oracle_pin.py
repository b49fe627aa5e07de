"""Pin the C oracle (oracle/pic_oracle.c) to the reference.

The golden vectors were produced by the reference's own sources
(tests/golden/make_golden.py); the oracle must reproduce every array and
every particle record bit for bit, including the particle order that the
reference's exchange produces (src/mpi_utils.cpp:62-230).
"""
import os

import numpy as np
import pytest

import oracle as O
from golden_io import ARRAYS, CASES, load
from golden.make_golden import PFIELDS, checksums


def _same_particles(a, b):
    assert len(a) == len(b)
    for f in ["id", "rank"] + PFIELDS + ["charge", "mass"]:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_bitwise(case):
    g = load(case)
    states, o = O.run_oracle(g["params"], g["input"], g["steps"], g_data=g["g_data"])
    for tag, idx in (("step1", 1), ("final", -1)):
        for n in ARRAYS:
            np.testing.assert_array_equal(states[idx][n], g[tag][n], err_msg=f"{tag} {n}")
        for k in range(2):
            _same_particles(states[idx]["particles"][k], g[tag]["particles"][k])
    for s, (mine, ref) in enumerate(zip(states, g["meta"]["checksums"])):
        assert checksums(mine) == ref, f"step {s}"
    assert o.s.g_factor_errors == 0


def test_golden_cases_cover_the_paths():
    seen = set()
    for case in CASES:
        p = load(case)["params"]
        seen.add(("order", 2 if p["mem"] == 2 else 4))
        seen.add(("faces", (p["period_x"], p["period_y"], p["period_z"])))
        if p["laser_amplitude"] > 0:
            seen.add(("laser_pol", p["laser_polarization"]))
    assert ("order", 2) in seen and ("order", 4) in seen
    assert ("faces", (1, 1, 1)) in seen and ("faces", (0, 0, 0)) in seen and ("faces", (0, 1, 1)) in seen
    assert ("laser_pol", 1) in seen and ("laser_pol", 3) in seen
    # removal at absorbing faces happened
    g = load("laser_o4")
    assert len(g["final"]["particles"][0]) < len(g["input"][0])


def test_spin_case_reaches_table():
    g = load("spin_o2")
    assert g["g_data"] is not None and len(g["g_data"]) == 2849
    sp = g["final"]["particles"][0]
    assert np.any(sp["sx"] != g["input"][0]["sx"])


@pytest.mark.parametrize("order,npts", [(2, 3), (4, 5)])
def test_shape_partition_of_unity(order, npts):
    rng = np.random.default_rng(3)
    for x in rng.uniform(2.0, 30.0, 200):
        w = O.shape_function(order, x)
        assert len(w) == npts
        assert abs(w.sum() - 1.0) < 1e-14
        assert np.all(w >= -1e-15)


def test_shape_known_values():
    # x on a node: quadratic weights 1/8, 3/4, 1/8; quartic 1/384*(1,76,230,76,1)
    np.testing.assert_allclose(O.shape_function(2, 5.0), [0.125, 0.75, 0.125], rtol=0, atol=1e-15)
    np.testing.assert_allclose(O.shape_function(4, 5.0), np.array([1, 76, 230, 76, 1]) / 384.0, atol=1e-15)


@pytest.mark.skipif(not (O.have_reference_build() and os.path.exists(O.REF_BIN_O0)),
                    reason="reference build not present (built where the reference tree is available)")
@pytest.mark.parametrize("case", ["periodic_o2", "laser_o4", "mixed_o2", "spin_o2"])
def test_reference_O0_and_O2_builds_dump_identical_states(case):
    """The reference's own Makefile builds at -O0; the oracle build uses -O2
    -ffp-contract=off.  Both produce bit-identical per-step dumps, so the
    faster build stands for the shipped one."""
    g = load(case)
    w = g["params"]
    s2, _ = O.run_reference(w, g["input"], g["steps"])
    s0, _ = O.run_reference(w, g["input"], g["steps"], binary=O.REF_BIN_O0)
    assert len(s0) == len(s2)
    for a, b in zip(s0, s2):
        for n in ARRAYS:
            assert a[n].tobytes() == b[n].tobytes(), n
        for k in range(2):
            assert a["particles"][k].tobytes() == b["particles"][k].tobytes()
