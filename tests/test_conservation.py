"""Size-independent properties at the full size of the thermal-plasma
configuration (32^3 periodic cells, 8 electrons per cell, u_th = 0.05,
200 steps) and the interior of an absorbing-face case.

* Charge conservation.  The E half-updates see -dt/2 (J^(n-1/2) + J^(n+1/2))
  per step and the Esirkepov current satisfies rho^(n+1) - rho^n =
  -dt div J, so G^n = div E^n - (rho^n + rho^(n-1)) / 2 is constant at every
  node (the t=0 push deposits a current that is neither cleared nor folded,
  so the constancy starts at step 2).  Checked first on the CPU oracle,
  then on the GPU in FP64 (round-off) and FP32.
* Energy.  Field plus kinetic energy (pic_diagnostics, FP64 reductions)
  after every step: the GPU FP64 history matches the oracle's, the FP32
  history stays close to the FP64 one, and the total drifts by less than a
  stated bound over the run.
"""
import numpy as np
import pytest

import oracle as O
from pic3d_b200.workloads import make_particles, thermal_periodic, tiny_cases


def div_nodes(w, st):
    """(Ex(i+1/2) - Ex(i-1/2)) / dx + ... at the physical nodes."""
    m = w.mem
    z, y, x = slice(m, m + w.nz), slice(m, m + w.ny), slice(m, m + w.nx)
    ex, ey, ez = st["ex"], st["ey"], st["ez"]
    return ((ex[z, y, x] - ex[z, y, slice(m - 1, m - 1 + w.nx)]) / w.dx
            + (ey[z, y, x] - ey[z, slice(m - 1, m - 1 + w.ny), x]) / w.dy
            + (ez[z, y, x] - ez[slice(m - 1, m - 1 + w.nz), y, x]) / w.dz)


def rho_nodes(w, st):
    """rho of both species at the physical nodes (ring buffers carry one
    extra layer)."""
    m = w.mem
    r = st["rho0"] + st["rho1"]
    return r[m + 1:m + 1 + w.nz, m + 1:m + 1 + w.ny, m + 1:m + 1 + w.nx]


def gauss_drift(w, states, interior=None):
    """max over steps n >= 3 of |G^n - G^2| / max |rho|."""
    G = [div_nodes(w, states[n]) - 0.5 * (rho_nodes(w, states[n]) + rho_nodes(w, states[n - 1]))
         for n in range(1, len(states))]
    scale = max(float(np.max(np.abs(rho_nodes(w, s)))) for s in states)
    sel = interior if interior is not None else (slice(None),) * 3
    return max(float(np.max(np.abs((g - G[1])[sel]))) for g in G[2:]) / scale


def _interior(w):
    # nodes at least mem cells away from an absorbing face
    return tuple(slice(None) if p else slice(w.mem, -w.mem) for p in (w.period[2], w.period[1], w.period[0]))


@pytest.mark.parametrize("name", ["periodic_o2", "periodic_o4", "mixed_o2"])
def test_oracle_conserves_charge(name):
    w = tiny_cases()[name]
    states, _ = O.run_oracle(w, make_particles(w, seed=3), 8)
    assert gauss_drift(w, states, _interior(w)) < 1e-13


def _gpu_states(w, precision, parts, steps):
    from pic3d_b200.simulation import Simulation
    keep = ["ex", "ey", "ez", "rho0", "rho1"]
    with Simulation(w, precision=precision) as sim:
        for k in range(2):
            sim.upload_particles(k, parts[k])
        sim.initial_push()
        states = [{n: sim.download_array(n) for n in keep}]
        energy = []
        for _ in range(steps):
            sim.run_main_time_loop(1)
            states.append({n: sim.download_array(n) for n in keep})
            d = sim.diagnostics()
            energy.append(d["field_energy"] + d["kinetic0"] + d["kinetic1"])
    return states, np.array(energy)


# energy-drift bounds over 200 steps: measured 5.3 % (2nd order) and 0.81 %
# (4th order) on B200 in both precisions, the grid heating of a plasma whose
# Debye length is 1/20 of a cell (the smoother 4th-order shape heats less)
FULL = {"thermal_32_o2": dict(mem=2), "thermal_32_o4": dict(mem=4)}
ENERGY_DRIFT = {"thermal_32_o2": 0.08, "thermal_32_o4": 0.015}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", list(FULL))
def test_gpu_charge_conservation_full_size(name, precision):
    w = thermal_periodic(n=32, **FULL[name])
    parts = make_particles(w, seed=1234)
    states, energy = _gpu_states(w, precision, parts, 200)
    drift = gauss_drift(w, states)
    # FP64: round-off over 200 steps (measured 2e-14 - 6e-14); FP32: E updated
    # in FP32 (measured 1.7e-6 - 1.9e-6)
    tol = 1e-12 if precision == "fp64" else 2e-5
    assert drift < tol, drift
    rel = np.abs(energy - energy[0]) / energy[0]
    assert np.max(rel) < ENERGY_DRIFT[name], np.max(rel)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gpu_charge_conservation_absorbing_interior(precision):
    w = tiny_cases()["mixed_o2"].with_(nx=24, ny=16, nz=12)
    parts = make_particles(w, seed=9)
    states, _ = _gpu_states(w, precision, parts, 40)
    tol = 1e-12 if precision == "fp64" else 2e-5   # measured 2.8e-14 / 4.7e-6
    assert gauss_drift(w, states, _interior(w)) < tol


def _oracle_energy(w, states):
    dV = w.dx * w.dy * w.dz
    out = []
    for st in states[1:]:
        m = w.mem
        sl = (slice(m, m + w.nz), slice(m, m + w.ny), slice(m, m + w.nx))
        fe = 0.5 * dV * sum(float(np.sum(st[n][sl] ** 2)) for n in ("ex", "ey", "ez", "bx", "by", "bz"))
        ke = 0.0
        for k, p in enumerate(st["particles"]):
            u2 = p["px"] ** 2 + p["py"] ** 2 + p["pz"] ** 2
            ke += float(np.sum(p["weight"] * w.species(k)["mass"] * u2 / (np.sqrt(1.0 + u2) + 1.0)))
        out.append(fe + ke)
    return np.array(out)


@pytest.mark.gpu
def test_gpu_energy_history_matches_oracle():
    """The first 20 steps of the full-size thermal run: FP64 energy equal to
    the oracle's, FP32 within 1e-5."""
    w = thermal_periodic(n=32, mem=2)
    parts = make_particles(w, seed=1234)
    ref_states, _ = O.run_oracle(w, parts, 20)
    ref = _oracle_energy(w, ref_states)
    _, e64 = _gpu_states(w, "fp64", parts, 20)
    _, e32 = _gpu_states(w, "fp32", parts, 20)
    assert np.max(np.abs(e64 - ref) / ref) < 1e-9
    assert np.max(np.abs(e32 - ref) / ref) < 1e-5
