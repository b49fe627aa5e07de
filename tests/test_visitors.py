"""Incremental re-binning of the tiled kernel between full sorts.

The counting sort by tile runs every sort_interval pushes; in between, each
push records the particles that end in a tile other than the one whose
slice of the sorted arrays holds them, and a counting sort of only those
entries gives every tile its visitor list, so that every particle is pushed
by the CTA of the tile it is in (the role the reference's particle exchange
plays between ranks, src/mpi_utils.cpp:62-230, inside one GPU).  Removal at
absorbing faces compacts the arrays; the compaction drops the entries of
removed and moved particles and records the moved ones anew.  Lists that
would overflow (more than half of the particles away from home) or name
fewer than 3 % of the particles make the next push hand the particles away
from home to the global-memory kernel.

Free runs of a hot thermal plasma (most particles change tile) with the
full sort every push, every 4 pushes (default) and never after the first,
and with 2-cell tiles, against the oracle's free run: relative L2 1e-8 in
FP64 (the free-run bound of the golden tests: summation order differs per
step), and FP32 paths against each other.
"""
import numpy as np
import pytest

import oracle as O
from parity import ARRAYS, array_errors, particle_errors, periods

from pic3d_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS = 40
PATHS = {"sorted_every_push": dict(tile=4, sort_interval=1), "default": dict(tile=0),
         "lists_only": dict(tile=4, sort_interval=10000), "tile2_lists_only": dict(tile=2, sort_interval=10000)}


def _hot(mem):
    # u_th 0.1: about 0.05 cells per step, two cells over the run
    return W.thermal_periodic(16, mem=mem, steps=STEPS).with_(u_th=(0.1, 0.0))


@pytest.fixture(scope="module", params=[2, 4], ids=["o2", "o4"])
def hot_run(request):
    w = _hot(request.param)
    parts = W.make_particles(w, seed=99)
    o = O.Oracle(w, parts)
    o.initial()
    for s in range(1, STEPS + 1):
        o.step(s)
    return w, parts, o.state()


def _free_run(w, parts, precision, **kw):
    from pic3d_b200.simulation import Simulation
    sim = Simulation(w, precision=precision, **kw)
    for k in range(2):
        if len(parts[k]):
            sim.upload_particles(k, parts[k])
    sim.initial_push()
    stats = []
    for _ in range(STEPS):
        sim.run_main_time_loop(1)
        stats.append(sim.particle_order_stats(0))
    st = sim.state()
    sim.close()
    return st, stats


@pytest.mark.parametrize("path", list(PATHS))
def test_fp64_free_run_matches_oracle(hot_run, path):
    w, parts, ref = hot_run
    got, stats = _free_run(w, parts, "fp64", **PATHS[path])
    errs = array_errors(got, ref)
    assert max(errs.values()) < 1e-8, errs
    perr, merr = particle_errors(got["particles"][0], ref["particles"][0], periods(w.params()))
    assert perr < 1e-9 and merr < 1e-8, (perr, merr)
    if path.endswith("lists_only"):
        # never re-sorted: most particles end up away from home (the lists
        # overflow and the global kernel takes over for a push)
        assert stats[-1]["pushes_since_sort"] == STEPS + 1
        assert max(s["visitors"] for s in stats) > 0.2 * len(parts[0])


def test_lists_stay_complete_within_their_capacity():
    """12 pushes of a warm plasma without a sort: every particle away from
    home is pushed from a visitor list, none by the global kernel."""
    w = W.thermal_periodic(16, mem=2, steps=12)
    parts = W.make_particles(w, seed=7)
    states, _ = O.run_oracle(w, parts, 12)
    from pic3d_b200.simulation import Simulation
    sim = Simulation(w, precision="fp64", sort_interval=10000)
    sim.upload_particles(0, parts[0])
    sim.initial_push()
    stats = []
    for _ in range(12):
        sim.run_main_time_loop(1)
        stats.append(sim.particle_order_stats(0))
    got = sim.state()
    sim.close()
    # a push that takes the particles away from home from the lists leaves
    # none to the global kernel; past a few pushes the lists are in use
    assert all(b["global_kernel"] == 0 for a, b in zip(stats, stats[1:]) if a["lists_used"])
    assert all(s["lists_used"] for s in stats[6:])
    assert stats[-1]["visitors"] > 0.03 * len(parts[0]), stats[-1]
    errs = array_errors(got, states[-1])
    assert max(errs.values()) < 1e-8, errs


@pytest.mark.parametrize("path", ["default", "lists_only", "tile2_lists_only"])
def test_fp32_free_run_matches_sorted_every_push(hot_run, path):
    w, parts, _ = hot_run
    want, _ = _free_run(w, parts, "fp32", **PATHS["sorted_every_push"])
    got, _ = _free_run(w, parts, "fp32", **PATHS[path])
    errs = array_errors(got, want)
    assert max(errs.values()) < 1e-5, errs
    perr, merr = particle_errors(got["particles"][0], want["particles"][0], periods(w.params()))
    assert perr < 1e-5 and merr < 1e-5, (perr, merr)


def test_removal_keeps_the_lists_complete():
    """Absorbing x faces: particles leave every step; the compaction moves
    particles into the holes and re-records them, the lists stay complete
    (the pushes that use them leave nothing to the global kernel) and the run
    matches the oracle."""
    w = _hot(2).with_(period=(0, 1, 1), u_th=(0.2, 0.0), name="hot_absorbing_x")
    parts = W.make_particles(w, seed=5)
    states, _ = O.run_oracle(w, parts, 20)
    ref = states[-1]
    from pic3d_b200.simulation import Simulation
    sim = Simulation(w, precision="fp64")
    sim.upload_particles(0, parts[0])
    sim.initial_push()
    stats, counts = [], []
    for _ in range(20):
        sim.run_main_time_loop(1)
        stats.append(sim.particle_order_stats(0))
        counts.append(sim.num_particles(0))
    got = sim.state()
    sim.close()
    assert counts[-1] < counts[0] < len(parts[0])   # particles left through the faces during the run
    used = [a["lists_used"] for a in stats[:-1]]
    assert sum(used) >= 8
    assert all(b["global_kernel"] == 0 for a, b in zip(stats, stats[1:]) if a["lists_used"])
    errs = array_errors(got, ref)
    assert max(errs.values()) < 1e-8, errs
    perr, merr = particle_errors(got["particles"][0], ref["particles"][0], periods(w.params()))
    assert perr < 1e-9 and merr < 1e-8
