"""Per-step GPU parity at the sizes and densities of the benchmark
configurations (the golden cases are 8^3-16x8x8 grids with 1-3 particles
per cell; these drive the tile kernel with full tiles).

Teacher-forced, as the golden tests: the oracle's state after step n is
uploaded through the C ABI, the GPU runs step n+1, every array and every
particle (matched by id) is compared with the oracle's step n+1 at relative
L2 1e-10 (FP64) / 1e-5 (FP32).

* Thermal plasma, periodic 32^3, 8 electrons per cell (262,144), ions a
  fixed background, u_th = 0.05, 2nd order, dt = 0.95 of the Courant limit:
  steps sampled across the whole 200-step run.
* Laser in underdense plasma on a reduced grid (64x32x32, lambda/20 x
  lambda/10 cells, a0 = 2, 8 + 8 particles per cell, 4th order, absorbing
  faces): the GPU runs 200 steps (the pulse fills the box and the
  electrons move relativistically), then steps 201-204 are teacher-forced.
* Clustered inputs whose one tile holds 5000 particles (shared-memory
  path, dense) and more than 16383 particles (that tile takes the
  global-memory path as a whole).
"""
import numpy as np
import pytest

import oracle as O
from parity import ARRAYS, TOL_FP32, TOL_FP64, array_errors, particle_errors, periods

from pic3d_b200 import workloads as W

pytestmark = pytest.mark.gpu

CFG1_SAMPLES = (0, 1, 50, 100, 150, 199)   # teacher-forced steps n -> n+1


@pytest.fixture(scope="module")
def thermal_pairs():
    w = W.thermal_periodic(32, mem=2)
    parts = W.make_particles(w, seed=1234)
    o = O.Oracle(w, parts)
    o.initial()
    pairs = {}
    before = o.state() if 0 in CFG1_SAMPLES else None
    for s in range(1, max(CFG1_SAMPLES) + 2):
        o.step(s)
        if s - 1 in CFG1_SAMPLES:
            pairs[s - 1] = (before, o.state())
        before = o.state() if s in CFG1_SAMPLES else None
    return w, pairs


def _teacher_forced(w, pairs, precision, **kw):
    from pic3d_b200.simulation import Simulation
    tol = TOL_FP64 if precision == "fp64" else TOL_FP32
    pos_tol = 1e-11 if precision == "fp64" else 2e-6
    per = periods(w.params())
    sim = Simulation(w, precision=precision, **kw)
    report = {}
    for n, (st, ref) in sorted(pairs.items()):
        sim.upload_state(st)
        sim.step = n
        sim.run_main_time_loop(1)
        got = sim.state()
        errs = array_errors(got, ref)
        bad = {k: v for k, v in errs.items() if v > tol}
        assert not bad, f"step {n + 1}: {bad}"
        worst = []
        for k in range(2):
            perr, merr = particle_errors(got["particles"][k], ref["particles"][k], per)
            assert perr < pos_tol and merr < tol, (n + 1, k, perr, merr)
            worst.append((perr, merr))
        report[n + 1] = (errs, worst)
    sim.close()
    return report


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_thermal_32cubed_teacher_forced_across_the_run(thermal_pairs, precision):
    w, pairs = thermal_pairs
    _teacher_forced(w, pairs, precision)


def test_thermal_32cubed_fp32_energies_match_fp64(thermal_pairs):
    """The field and kinetic energies of a teacher-forced FP32 step agree
    with the oracle's to FP32 rounding (the energy record of the FP32 run)."""
    from pic3d_b200.simulation import Simulation
    w, pairs = thermal_pairs
    n = max(pairs)
    st, ref = pairs[n]
    out = {}
    for prec in ("fp64", "fp32"):
        sim = Simulation(w, precision=prec)
        sim.upload_state(st)
        sim.step = n
        sim.run_main_time_loop(1)
        out[prec] = sim.diagnostics()
        sim.close()
    for key in ("field_energy", "kinetic0"):
        a, b = out["fp32"][key], out["fp64"][key]
        assert abs(a - b) <= 1e-5 * abs(b), (key, a, b)


@pytest.fixture(scope="module")
def laser_pairs():
    """GPU FP64 run of the laser workload on 64x32x32 cells to step 200,
    then oracle states 200..204 from that state."""
    from pic3d_b200.simulation import Simulation
    w = W.laser_underdense(nx=64, ny=32, nz=32, steps=204)
    parts = W.make_particles(w, seed=77)
    sim = Simulation(w, precision="fp64")
    for k in range(2):
        sim.upload_particles(k, parts[k])
    sim.initial_push()
    sim.run_main_time_loop(200)
    st = sim.state()
    sim.close()
    moving = np.abs(st["particles"][0]["px"]) + np.abs(st["particles"][0]["py"])
    assert np.max(moving) > 0.5   # relativistic electrons in the pulse
    o = O.Oracle(w, st["particles"], fields={n: st[n] for n in ARRAYS})
    pairs = {}
    before = o.state()
    for s in range(201, 205):
        o.step(s)
        after = o.state()
        pairs[s - 1] = (before, after)
        before = after
    return w, pairs


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_laser_underdense_teacher_forced_after_the_pulse_entered(laser_pairs, precision):
    w, pairs = laser_pairs
    _teacher_forced(w, pairs, precision)


def _clustered(n_in_tile=5000, seed=3):
    """periodic 16^3, 2nd order: 5000 electrons inside cells 0..3 on every
    axis (one 4^3 tile), a sparse thermal background elsewhere."""
    w = W.Workload(name="clustered_o2", nx=16, ny=16, nz=16, mem=2, period=(1, 1, 1), ppc=(1, 1),
                   u_th=(0.1, 0.02), steps=3)
    parts = W.make_particles(w, seed=seed)
    rng = np.random.default_rng(seed)
    extra = np.zeros(n_in_tile, dtype=W.PARTICLE_DTYPE)
    extra["id"] = np.arange(n_in_tile) + 100000
    for f in ("x", "y", "z"):
        extra[f] = 0.05 + 3.9 * rng.random(n_in_tile)
    for f in ("px", "py", "pz"):
        extra[f] = 0.1 * rng.normal(size=n_in_tile)
    extra["gamma"] = np.sqrt(1 + extra["px"] ** 2 + extra["py"] ** 2 + extra["pz"] ** 2)
    extra["charge"], extra["mass"], extra["weight"] = -1.0, 1.0, 0.01
    both = np.zeros(len(parts[0]) + n_in_tile, W.PARTICLE_DTYPE)   # (np.concatenate drops the record padding)
    both[:len(parts[0])] = parts[0]
    both[len(parts[0]):] = extra
    parts[0] = both
    return w, parts


@pytest.mark.parametrize("n_in_tile", [5000, 17000])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_crowded_tiles(precision, n_in_tile):
    w, parts = _clustered(n_in_tile)
    states, _ = O.run_oracle(w, parts, 3)
    pairs = {n: (states[n], states[n + 1]) for n in range(3)}
    _teacher_forced(w, pairs, precision)
