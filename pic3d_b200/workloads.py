"""Workload definitions and seeded particle inputs.

A workload is the set of reference parameters (the names of the reference's
``src/constants.cpp:5-85`` globals) plus the particle input that the
reference would otherwise build in ``initialize_particles``
(``src/particle.cpp:50-111``).  The reference loads a regular lattice with a
constant momentum; the workloads here place particles uniformly at random in
each cell from a seed and draw Maxwellian momenta, as the benchmark
configurations ask.  The same parameter dictionary feeds the GPU library
(``PicParams``), the C oracle and the reference build.

Units follow the reference: c = m_e = |q_e| = eps0 = omega = 1, particle
coordinates in cells, momenta as u = gamma*v (momentum per unit mass).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional

import numpy as np

# The reference's pi constant (src/constants.cpp:6) is a 10-digit literal;
# every derived length (l0, t0, dx for laser runs) uses it.
REF_PI = 3.1415926536

ELECTRON = dict(charge=-1.0, mass=1.0)
PROTON = dict(charge=1.0, mass=1836.0)

#: numpy view of the reference's 144-byte ``struct particle``
#: (include/particle.h:9-29): int id, 16 doubles, int rank.
PARTICLE_DTYPE = np.dtype({
    "names": ["id", "x", "y", "z", "x_old", "y_old", "z_old", "px", "py", "pz",
              "sx", "sy", "sz", "gamma", "charge", "mass", "weight", "rank"],
    "formats": ["<i4"] + ["<f8"] * 16 + ["<i4"],
    "offsets": [0] + [8 + 8 * i for i in range(16)] + [136],
    "itemsize": 144,
})


@dataclasses.dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    mem: int                       # ghost width; 2 -> 2nd-order shape, 4 -> 4th order
    period: tuple = (1, 1, 1)      # rank_period
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 1.0
    courant: float = 0.95          # dt as a fraction of the 3D Courant limit
    ppc: tuple = (8, 0)            # particles per cell per species (electrons, protons)
    u_th: tuple = (0.05, 0.0)      # thermal spread of u = gamma*v per component
    density: Optional[Callable] = None   # n(x_phys) -> density, x_phys = x*dx; None -> density_value
    density_value: float = 1.0
    laser_amplitude: float = 0.0
    laser_pulse_duration: float = 10.0 * 2.0 * REF_PI
    laser_start_time: float = 0.0
    laser_polarization: int = 1
    waist: float = 3.0 * 2.0 * REF_PI
    xfocus: Optional[float] = None      # None -> box centre
    yfocus: Optional[float] = None
    zfocus: Optional[float] = None
    phase: float = 0.0
    laser_envelope: int = 0             # 0 reference sine envelope, 1 Gaussian (extension)
    absorbing: int = 0                  # 1: absorbing y, z and x-max faces (extension)
    steps: int = 200
    precision: str = "fp64"
    E_schwinger: float = 4.1215e5

    # ---- derived reference parameters -------------------------------
    @property
    def dt(self) -> float:
        return self.courant / math.sqrt(1.0 / self.dx ** 2 + 1.0 / self.dy ** 2 + 1.0 / self.dz ** 2)

    @property
    def order(self) -> int:
        return 2 if self.mem == 2 else 4

    @property
    def num_particles(self) -> int:
        return self.nx * self.ny * self.nz * sum(self.ppc)

    def params(self) -> dict:
        """Reference parameter names (src/constants.cpp) -> values."""
        l0 = 2.0 * REF_PI * 1.0 / 1.0
        t0 = 2.0 * REF_PI / 1.0
        dt = self.dt
        Lx, Ly, Lz = self.nx * self.dx, self.ny * self.dy, self.nz * self.dz
        return dict(
            Pi=REF_PI, omega=1.0, l0=l0, t0=t0, Lx=Lx, Ly=Ly, Lz=Lz,
            resx=20, resy=20, resz=20, rest=40,
            period_x=int(self.period[0]), period_y=int(self.period[1]), period_z=int(self.period[2]),
            local_xcells=self.nx, local_ycells=self.ny, local_zcells=self.nz,
            cell_per_particles=int(self.ppc[0]), density=float(self.density_value),
            dx=self.dx, dy=self.dy, dz=self.dz, dt=dt, dt_half=dt / 2.0,
            simulation_time=self.steps * dt, timesteps=int(self.steps), output_interval=1,
            mem=self.mem,
            laser_amplitude=self.laser_amplitude, laser_pulse_duration=self.laser_pulse_duration,
            laser_start_time=self.laser_start_time, laser_polarization=int(self.laser_polarization),
            waist=self.waist,
            xfocus=self.xfocus if self.xfocus is not None else 0.5 * Lx,
            yfocus=self.yfocus if self.yfocus is not None else 0.5 * Ly,
            zfocus=self.zfocus if self.zfocus is not None else 0.5 * Lz,
            phase=self.phase, E_schwinger=self.E_schwinger,
            laser_envelope=int(self.laser_envelope), absorbing=int(self.absorbing),
        )

    def species(self, kind: int) -> dict:
        return ELECTRON if kind == 0 else PROTON

    def with_(self, **kw) -> "Workload":
        return dataclasses.replace(self, **kw)


def make_particles(w: Workload, seed: int = 1234, kinds=(0, 1)) -> list:
    """Seeded particle input per species as reference AoS records.

    For each cell, ppc particles are placed uniformly at random inside it;
    each momentum component is drawn from N(0, u_th^2).  The weight is
    density(x_phys)/ppc at the particle's own position (the reference
    evaluates its density function at the lattice position,
    src/particle.cpp:79); particles where the density is not positive are
    not created (src/particle.cpp:80-83).
    """
    out = []
    rng = np.random.default_rng(seed)
    next_id = 0
    for kind in (0, 1):
        ppc = w.ppc[kind] if kind in kinds else 0
        if ppc == 0:
            out.append(np.zeros(0, dtype=PARTICLE_DTYPE))
            continue
        ncell = w.nx * w.ny * w.nz
        n = ncell * ppc
        cell = np.repeat(np.arange(ncell, dtype=np.int64), ppc)
        cx = cell % w.nx
        cy = (cell // w.nx) % w.ny
        cz = cell // (w.nx * w.ny)
        off = rng.random((n, 3))
        x = cx + off[:, 0]
        y = cy + off[:, 1]
        z = cz + off[:, 2]
        if w.density is None:
            dens = np.full(n, w.density_value)
        else:
            dens = np.asarray(w.density(x * w.dx), dtype=np.float64)
        keep = dens > 0.0
        p = np.zeros(int(keep.sum()), dtype=PARTICLE_DTYPE)
        p["id"] = np.arange(next_id, next_id + len(p), dtype=np.int64).astype(np.int32)
        next_id += len(p)
        p["x"], p["y"], p["z"] = x[keep], y[keep], z[keep]
        u = rng.normal(0.0, 1.0, (n, 3)) * w.u_th[kind] if w.u_th[kind] > 0 else np.zeros((n, 3))
        u = u[keep]
        p["px"], p["py"], p["pz"] = u[:, 0], u[:, 1], u[:, 2]
        p["gamma"] = np.sqrt(1.0 + (p["px"] * p["px"] + p["py"] * p["py"] + p["pz"] * p["pz"]))
        sp = w.species(kind)
        p["charge"] = sp["charge"]
        p["mass"] = sp["mass"]
        p["weight"] = dens[keep] / ppc
        out.append(p)
    return out


# ---------------------------------------------------------------------------
# the benchmark configurations

LAMBDA = 2.0 * REF_PI


def thermal_periodic(n=32, mem=2, precision="fp64", steps=200) -> Workload:
    """Thermal plasma, periodic n^3 cells, dx=1 (c/omega_p), 8 electrons per
    cell, ions as a fixed neutralising background, u_th = 0.05."""
    return Workload(name=f"thermal_periodic_{n}_o{2 if mem == 2 else 4}_{precision}", nx=n, ny=n, nz=n,
                    mem=mem, period=(1, 1, 1), ppc=(8, 0), u_th=(0.05, 0.0), density_value=1.0,
                    steps=steps, precision=precision)


def _ramp(length_x: float, n0: float):
    def f(xp):
        return n0 * np.minimum(1.0, np.asarray(xp) / length_x)
    return f


def laser_underdense(nx=256, ny=128, nz=128, precision="fp64", steps=3000) -> Workload:
    """Laser in underdense plasma: dx = lambda/20, dy = dz = lambda/10,
    electrons + protons at 8 per cell each, density 0.01 n_c after a 20 lambda
    linear ramp, cold; linearly polarised pulse a0 = 2, waist 8 lambda,
    Gaussian temporal envelope with an intensity FWHM of 10 lambda/c
    (extension; the reference has the sine envelope only), injected from
    x-min; absorbing faces on every side (x-min is the reference's own;
    y, z and x-max are the extension); 4th-order shape."""
    return Workload(name=f"laser_underdense_{nx}x{ny}x{nz}_{precision}", nx=nx, ny=ny, nz=nz, mem=4,
                    period=(0, 0, 0), dx=LAMBDA / 20, dy=LAMBDA / 10, dz=LAMBDA / 10, ppc=(8, 8),
                    u_th=(0.0, 0.0), density=_ramp(20 * LAMBDA, 0.01), density_value=0.01,
                    laser_amplitude=2.0, laser_pulse_duration=10.0 * LAMBDA, waist=8.0 * LAMBDA,
                    laser_polarization=1, laser_envelope=1, absorbing=1, steps=steps, precision=precision)


def thermal_scaleup(nx=512, ny=256, nz=256, mem=2, precision="fp32", steps=100) -> Workload:
    """Throughput scale-up: periodic thermal electron-proton plasma, 8
    particles per cell per species, u_th = 0.02 for both species."""
    return Workload(name=f"thermal_scaleup_{nx}x{ny}x{nz}_o{2 if mem == 2 else 4}_{precision}", nx=nx, ny=ny,
                    nz=nz, mem=mem, period=(1, 1, 1), ppc=(8, 8), u_th=(0.02, 0.02), density_value=1.0,
                    steps=steps, precision=precision)


def differentiable_laser(nx=64, ny=64, nz=128, precision="fp32", steps=600, mem=4) -> Workload:
    """Differentiable run: 64 x 64 x 128 cells (dx = dy = dz = lambda/16),
    electrons at 8 per cell (weights from a 32-knot density profile set by
    the caller), a laser from x-min whose transverse amplitude is an 8 x 8
    cubic-B-spline coefficient grid (a0 about 1), absorbing faces, 600
    steps."""
    return Workload(name=f"differentiable_laser_{nx}x{ny}x{nz}_{precision}", nx=nx, ny=ny, nz=nz, mem=mem,
                    period=(0, 0, 0), dx=LAMBDA / 16, dy=LAMBDA / 16, dz=LAMBDA / 16, ppc=(8, 0), u_th=(0.0, 0.0),
                    density_value=0.02, laser_amplitude=1.0, laser_pulse_duration=10.0 * LAMBDA,
                    waist=2.0 * LAMBDA, laser_polarization=1, steps=steps, precision=precision)


WORKLOADS = {
    "thermal_periodic": thermal_periodic,
    "laser_underdense": laser_underdense,
    "thermal_scaleup": thermal_scaleup,
    "differentiable_laser": differentiable_laser,
}


# ---------------------------------------------------------------------------
# small cases used by the parity tests (every reference code path: both
# shape orders, both species, periodic / absorbing / mixed faces, laser,
# cell crossings and particle removal)

def tiny_cases() -> dict:
    return {
        "periodic_o2": Workload(name="periodic_o2", nx=8, ny=8, nz=8, mem=2, period=(1, 1, 1),
                                ppc=(2, 1), u_th=(0.2, 0.05), steps=12),
        "periodic_o4": Workload(name="periodic_o4", nx=12, ny=10, nz=11, mem=4, period=(1, 1, 1),
                                ppc=(1, 1), u_th=(0.2, 0.1), steps=8),
        "laser_o4": Workload(name="laser_o4", nx=16, ny=8, nz=8, mem=4, period=(0, 0, 0),
                             dx=LAMBDA / 20, dy=LAMBDA / 10, dz=LAMBDA / 10, ppc=(1, 1), u_th=(0.1, 0.01),
                             density=_ramp(0.5 * 16 * LAMBDA / 20, 0.05), density_value=0.05,
                             laser_amplitude=2.0, laser_pulse_duration=2.0 * LAMBDA, waist=0.4 * LAMBDA,
                             steps=12),
        "mixed_o2": Workload(name="mixed_o2", nx=12, ny=8, nz=6, mem=2, period=(0, 1, 1),
                             dx=0.5, dy=0.5, dz=0.5, ppc=(2, 1), u_th=(0.3, 0.05),
                             laser_amplitude=1.0, laser_pulse_duration=3.0, waist=2.0, laser_polarization=3,
                             steps=12),
    }
