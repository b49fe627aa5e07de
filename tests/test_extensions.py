"""GPU parity of the laser extensions against the oracle's CPU restatement.

The reference has only the sine envelope and the Gaussian transverse
profile (src/boundary.cpp:8-40).  Two labelled extensions serve the
benchmark configurations: a Gaussian temporal envelope whose intensity FWHM
is laser_pulse_duration (laser_envelope = 1) and a transverse amplitude
given by a grid of cubic-B-spline coefficients (laser_profile = 1).  The
oracle (oracle/pic_oracle.c) restates both; these tests teacher-force the
GPU against it per step, as the golden tests do for the reference's own
paths (relative L2 1e-10 FP64, 1e-5 FP32).
"""
import numpy as np
import pytest

import oracle as O
from golden_io import load
from parity import TOL_FP32, TOL_FP64, array_errors, particle_errors, periods

pytestmark = pytest.mark.gpu

STEPS = 8


def _params_with(**kw):
    g = load("laser_o4")
    p = dict(g["params"])
    p.update(kw)
    return p, g["input"]


def _teacher_forced(params, parts, precision, profile=None):
    from pic3d_b200.simulation import Simulation
    states, _ = O.run_oracle(params, parts, STEPS, profile=profile)
    tol = TOL_FP64 if precision == "fp64" else TOL_FP32
    per = periods(params)
    sim = Simulation(params, precision=precision, laser_profile=profile)
    moved_b = 0.0
    for n in range(STEPS):
        sim.upload_state(states[n])
        sim.step = n
        sim.run_main_time_loop(1)
        got = sim.state()
        errs = array_errors(got, states[n + 1])
        bad = {k: v for k, v in errs.items() if v > tol}
        assert not bad, f"step {n + 1}: {bad}"
        for k in range(2):
            perr, merr = particle_errors(got["particles"][k], states[n + 1]["particles"][k], per)
            assert merr < tol, (n + 1, k, merr)
        moved_b = max(moved_b, float(np.abs(states[n + 1]["bz"]).max()))
    sim.close()
    assert moved_b > 0.0   # the laser did enter


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gaussian_envelope_matches_oracle(precision):
    p, parts = _params_with(laser_envelope=1)
    # start the pulse so that its peak (1.5 durations after the start)
    # falls inside the teacher-forced window
    p["laser_start_time"] = -1.5 * p["laser_pulse_duration"]
    _teacher_forced(p, parts, precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_bspline_transverse_profile_matches_oracle(precision):
    p, parts = _params_with()
    rng = np.random.default_rng(5)
    coef = 1.0 + 0.3 * rng.random((8, 8))
    _teacher_forced(p, parts, precision, profile=coef)


def test_gaussian_envelope_fwhm():
    """The extension's envelope (evaluated on the device through pic_eval)
    has an intensity FWHM of laser_pulse_duration and its peak 1.5
    durations after the start."""
    from pic3d_b200 import _lib as L
    from pic3d_b200.simulation import Simulation
    import ctypes
    p, _ = _params_with(laser_envelope=1, laser_amplitude=1.0, laser_start_time=0.0)
    tau = p["laser_pulse_duration"]
    sim = Simulation(p, precision="fp64")
    ts = np.linspace(0.0, 3.0 * tau, 3001)
    env = []
    for t in ts:
        out = (ctypes.c_double * 1)()
        inp = (ctypes.c_double * 2)(t, 0.0)
        assert sim.lib.pic_eval(sim.ctx, L.EVAL_LASER_PULSE, inp, 2, out, 1) == L.PIC_OK
        env.append(out[0])
    sim.close()
    env = np.array(env)
    inten = env ** 2
    above = ts[inten >= 0.5 * inten.max()]
    assert abs((above[-1] - above[0]) - tau) < 2 * (ts[1] - ts[0])
    assert abs(ts[np.argmax(env)] - 1.5 * tau) < 2 * (ts[1] - ts[0])
