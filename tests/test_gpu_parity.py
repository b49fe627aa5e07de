"""GPU parity against the CPU oracle (which is pinned to the reference).

Teacher-forced: the oracle state after step n is uploaded through the C
ABI, the GPU runs step n+1, and every array is compared with the oracle's
step n+1 (relative L2 <= 1e-10 in FP64, <= 1e-5 in FP32; particles matched
by id).  Each reference function on the path is also checked on its own.
"""
import numpy as np
import pytest

import oracle as O
from golden_io import CASES, load
from parity import ARRAYS, TOL_FP32, TOL_FP64, array_errors, particle_errors, periods

pytestmark = pytest.mark.gpu


def _sim(params, precision="fp64", g_data=None, tile=0, sort_interval=0):
    from pic3d_b200.simulation import Simulation
    s = Simulation(params, precision=precision, tile=tile, sort_interval=sort_interval)
    if g_data is not None:
        s.set_g_table(g_data)
    return s


def _oracle_states(g):
    states, _ = O.run_oracle(g["params"], g["input"], g["steps"], g_data=g["g_data"])
    return states


# kernel paths: default shared-memory tiles, tiles sorted before every push,
# a 2-cell tile (most particles cross tiles), and the global-memory kernel
PATHS = {"tile4": dict(tile=0), "tile4_sort1": dict(tile=4, sort_interval=1), "tile2": dict(tile=2),
         "global": dict(tile=-1)}


@pytest.mark.parametrize("path", list(PATHS))
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_teacher_forced_steps(case, precision, path):
    g = load(case)
    states = _oracle_states(g)
    tol = TOL_FP64 if precision == "fp64" else TOL_FP32
    pos_tol = 1e-11 if precision == "fp64" else 2e-6
    per = periods(g["params"])
    sim = _sim(g["params"], precision, g["g_data"], **PATHS[path])
    for n in range(0, g["steps"]):
        sim.upload_state(states[n])
        sim.step = n
        sim.run_main_time_loop(1)
        got = sim.state()
        ref = states[n + 1]
        errs = array_errors(got, ref)
        bad = {k: v for k, v in errs.items() if v > tol}
        assert not bad, f"step {n + 1}: {bad}"
        for k in range(2):
            perr, merr = particle_errors(got["particles"][k], ref["particles"][k], per)
            assert perr < pos_tol and merr < tol, (n + 1, k, perr, merr)
            if precision == "fp64" and case == "spin_o2" and k == 0:
                a = np.sort(got["particles"][0], order="id")
                b = np.sort(ref["particles"][0], order="id")
                for f in ("sx", "sy", "sz"):
                    assert np.max(np.abs(a[f] - b[f])) < 1e-12
    sim.close()


@pytest.mark.parametrize("path", ["tile4", "global"])
@pytest.mark.parametrize("case", CASES)
def test_free_run_fp64_matches_golden(case, path):
    """The whole golden run (t=0 push + all steps) from the reference's
    input particles, compared with the reference's own final state."""
    g = load(case)
    sim = _sim(g["params"], "fp64", g["g_data"], **PATHS[path])
    for k in range(2):
        sim.upload_particles(k, g["input"][k])
    sim.initial_push()
    sim.run_main_time_loop(g["steps"])
    got = sim.state()
    errs = array_errors(got, g["final"])
    assert max(errs.values()) < 1e-8, errs
    per = periods(g["params"])
    for k in range(2):
        perr, merr = particle_errors(got["particles"][k], g["final"]["particles"][k], per)
        assert perr < 1e-9 and merr < 1e-8
    sim.close()


@pytest.mark.parametrize("case", ["periodic_o2", "laser_o4", "mixed_o2", "periodic_o4"])
def test_each_reference_function(case):
    """Every reference function on the path, one at a time, from a
    mid-run oracle state."""
    g = load(case)
    states = _oracle_states(g)
    base = states[3]
    params = g["params"]
    sim = _sim(params, "fp64", g["g_data"])

    def check(o, names, what, tol=1e-12):
        got = {n: sim.download_array(n) for n in names}
        errs = array_errors(got, {n: o.arrays[n] for n in names}, names)
        assert max(errs.values()) < tol, (what, errs)

    # radiating_boundary (boundary.cpp:42-99)
    o = O.Oracle(params, base["particles"], fields={n: base[n] for n in ARRAYS})
    sim.upload_state(base)
    o.radiating_boundary(4)
    sim.radiating_boundary(1, 0, 4)
    check(o, ["by", "bz"], "radiating_boundary")
    # update_electromagnetic_fields_first (field.cpp:56-86)
    o.fields_first()
    sim.update_electromagnetic_fields_first()
    check(o, ARRAYS[:6], "fields_first")
    # clear_currents + both pushes (particle.cpp:113-515)
    o.clear_currents()
    sim.clear_currents()
    for k in range(2):
        o.push(k)
        sim.update_particle_position_momentum(k)
    check(o, ARRAYS[6:], "push+deposit", tol=1e-11)
    # exchange_particle_data (mpi_utils.cpp:62-230)
    for k in range(2):
        o.exchange_particles(k)
        sim.exchange_particle_data(k)
        assert sim.num_particles(k) == o.s.num_particles[k]
    # exchange_currents (particle.cpp:594-601)
    o.exchange_currents()
    sim.exchange_currents()
    check(o, ARRAYS[6:], "exchange_currents", tol=1e-11)
    # update_electromagnetic_fields_second (field.cpp:88-117)
    o.fields_second()
    sim.update_electromagnetic_fields_second()
    check(o, ARRAYS[:6], "fields_second", tol=1e-11)
    sim.close()


def test_initial_push_quirk():
    """main.cpp:75-79: the t=0 push deposits J that is neither cleared nor
    folded before step 1 uses it."""
    g = load("periodic_o2")
    o = O.Oracle(g["params"], g["input"])
    o.initial()
    sim = _sim(g["params"])
    for k in range(2):
        sim.upload_particles(k, g["input"][k])
    sim.initial_push()
    got = {n: sim.download_array(n) for n in ARRAYS}
    errs = array_errors(got, o.arrays)
    assert max(errs.values()) < 1e-12, errs
    sim.close()
