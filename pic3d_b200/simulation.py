"""Host-side mirror of the reference's Simulation / Field / Particle call
surface on top of the C ABI.

``Simulation`` owns one GPU context.  Its methods carry the reference's
function names (include/field.h:29-31, include/particle.h:32-47,
include/boundary.h:4-6, include/mpi_utils.h:13-16, include/simulation.h:10-23)
and the reference's argument meaning; state lives on the device and crosses
to the host only through the explicit upload / download calls, in the
reference's own array layout and 144-byte particle records.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .workloads import PARTICLE_DTYPE, Workload


def params_from(w, precision: str | None = None, spin: bool = True, deposit_rho: bool = True,
                capacity=(0, 0), laser_profile: bool = False, tile: int = 0, sort_interval: int = 0,
                adjoint: bool = False) -> L.PicParams:
    """PicParams from a Workload or a reference parameter dictionary."""
    p = w if isinstance(w, dict) else w.params()
    prec = precision or (w.precision if isinstance(w, Workload) else "fp64")
    pp = L.PicParams()
    L.load().pic_default_params(ctypes.byref(pp))
    pp.local_xcells, pp.local_ycells, pp.local_zcells = int(p["local_xcells"]), int(p["local_ycells"]), \
        int(p["local_zcells"])
    pp.mem = int(p["mem"])
    for d, k in enumerate(["period_x", "period_y", "period_z"]):
        pp.rank_period[d] = int(p[k])
    pp.laser_polarization = int(p["laser_polarization"])
    for k in ["Pi", "omega", "l0", "Lx", "dx", "dy", "dz", "dt", "dt_half", "laser_amplitude",
              "laser_pulse_duration", "laser_start_time", "waist", "xfocus", "yfocus", "zfocus", "phase",
              "E_schwinger"]:
        setattr(pp, k, float(p[k]))
    pp.laser_envelope = int(p.get("laser_envelope", 0))
    pp.laser_profile = 1 if laser_profile else 0
    pp.precision = 32 if prec in ("fp32", 32, "f32") else 64
    pp.spin = 1 if spin else 0
    pp.deposit_rho = 1 if deposit_rho else 0
    pp.capacity[0], pp.capacity[1] = int(capacity[0]), int(capacity[1])
    pp.tile = int(tile)
    pp.sort_interval = int(sort_interval)
    pp.adjoint = 1 if adjoint else 0
    pp.absorbing = int(p.get("absorbing", 0))
    pp.charge[0], pp.mass[0] = -1.0, 1.0
    pp.charge[1], pp.mass[1] = 1.0, 1836.0
    return pp


class Simulation:
    """One GPU context running the reference's per-timestep loop."""

    def __init__(self, w, precision: str | None = None, device: int = 0, spin: bool = True,
                 deposit_rho: bool = True, capacity=(0, 0), laser_profile=None, tile: int = 0,
                 sort_interval: int = 0, adjoint: bool = False):
        """tile: edge of the shared-memory particle tile in cells (0 default,
        -1 global-memory kernel); sort_interval: pushes between sorts."""
        self.lib = L.load()
        self.params = params_from(w, precision, spin, deposit_rho, capacity, laser_profile is not None, tile,
                                  sort_interval, adjoint)
        self.w = w
        h = ctypes.c_void_p()
        self._check(self.lib.pic_create(ctypes.byref(self.params), device, ctypes.byref(h)), None)
        self.ctx = h
        if laser_profile is not None:
            self.set_laser_profile(laser_profile)

    # -- plumbing -------------------------------------------------------------
    def _check(self, code, ctx="self"):
        if code != L.PIC_OK:
            c = self.ctx if ctx == "self" else None
            msg = self.lib.pic_last_error(c).decode() if c else "pic_create failed (see stderr)"
            raise L.PicError(code, msg)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.pic_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def fp32(self) -> bool:
        return self.params.precision == 32

    def field_shape(self):
        m = self.params.mem
        return (self.params.local_zcells + 2 * m, self.params.local_ycells + 2 * m, self.params.local_xcells + 2 * m)

    def ring_shape(self):
        return tuple(n + 2 for n in self.field_shape())

    # -- state transfer -----------------------------------------------------------
    def upload_array(self, name: str, a: np.ndarray):
        which = L.ARRAYS.index(name)
        shape = self.field_shape() if which < 6 else self.ring_shape()
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != shape:
            raise ValueError(f"{name}: expected shape {shape}, got {a.shape}")
        self._check(self.lib.pic_upload_array(self.ctx, which, a.ctypes.data))

    def download_array(self, name: str) -> np.ndarray:
        which = L.ARRAYS.index(name)
        shape = self.field_shape() if which < 6 else self.ring_shape()
        out = np.empty(shape, dtype=np.float64)
        self._check(self.lib.pic_download_array(self.ctx, which, out.ctypes.data))
        return out

    def upload_particles(self, kind: int, records: np.ndarray):
        rec = np.ascontiguousarray(records, dtype=PARTICLE_DTYPE)
        self._check(self.lib.pic_upload_particles(self.ctx, kind, rec.ctypes.data if len(rec) else None, len(rec)))

    def num_particles(self, kind: int) -> int:
        n = ctypes.c_int64()
        self._check(self.lib.pic_num_particles(self.ctx, kind, ctypes.byref(n)))
        return n.value

    def download_particles(self, kind: int, out: np.ndarray | None = None) -> np.ndarray:
        """The species' records; `out` (PARTICLE_DTYPE, large enough) is
        reused when given instead of allocating a new array."""
        n = self.num_particles(kind)
        if out is None or len(out) < n or out.dtype != PARTICLE_DTYPE or not out.flags.c_contiguous:
            out = np.empty(n, dtype=PARTICLE_DTYPE)   # every byte is written by the download
        got = ctypes.c_int64()
        self._check(self.lib.pic_download_particles(self.ctx, kind, out.ctypes.data if n else None, n,
                                                    ctypes.byref(got)))
        return out[: got.value]

    def upload_state(self, state: dict):
        """state: dict of reference arrays (ex..rho1) and 'particles' [e, p]."""
        for n in L.ARRAYS:
            if n in state:
                self.upload_array(n, state[n])
        if "particles" in state:
            for k in range(2):
                self.upload_particles(k, state["particles"][k])

    def state(self) -> dict:
        st = {n: self.download_array(n) for n in L.ARRAYS}
        st["particles"] = [self.download_particles(k) for k in range(2)]
        return st

    def set_g_table(self, g):
        g = np.ascontiguousarray(g, dtype=np.float64)
        self._check(self.lib.pic_set_g_table(self.ctx, g.ctypes.data, len(g)))

    def set_laser_profile(self, coef):
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        self._laser_profile = coef
        self._check(self.lib.pic_set_laser_profile(self.ctx, coef.ctypes.data, coef.shape[0]))

    # -- the reference call surface -----------------------------------------------
    def radiating_boundary(self, is_left: int, is_right: int, step: int):
        """radiating_boundary(my_rank, is_left, is_right, num_procs, step): src/boundary.cpp:42-99"""
        self._check(self.lib.pic_radiating_boundary(self.ctx, is_left, is_right, step))

    def update_electromagnetic_fields_first(self):
        """src/field.cpp:56-86"""
        self._check(self.lib.pic_update_fields_first(self.ctx))

    def update_electromagnetic_fields_second(self):
        """src/field.cpp:88-117"""
        self._check(self.lib.pic_update_fields_second(self.ctx))

    def clear_currents(self):
        """src/particle.cpp:576-592"""
        self._check(self.lib.pic_clear_currents(self.ctx))

    def update_particle_position_momentum(self, kind: int):
        """src/particle.cpp:113-370 (gather, Boris, move, currents_particle, spin)"""
        self._check(self.lib.pic_update_particles(self.ctx, kind))

    def exchange_particle_data(self, kind: int):
        """src/mpi_utils.cpp:62-230 on one GPU: removal at absorbing faces"""
        self._check(self.lib.pic_exchange_particles(self.ctx, kind))

    def exchange_currents(self):
        """src/particle.cpp:594-601: periodic fold of J and rho"""
        self._check(self.lib.pic_exchange_currents(self.ctx))

    def initial_push(self):
        """main.cpp:75-79: t=0 push of both species and particle exchange"""
        self._check(self.lib.pic_initial_push(self.ctx))

    def run_main_time_loop(self, nsteps: int):
        """nsteps iterations of src/simulation.cpp:159-183"""
        self._check(self.lib.pic_run_steps(self.ctx, nsteps))

    @property
    def step(self) -> int:
        s = ctypes.c_int()
        self._check(self.lib.pic_get_step(self.ctx, ctypes.byref(s)))
        return s.value

    @step.setter
    def step(self, v: int):
        self._check(self.lib.pic_set_step(self.ctx, int(v)))

    def synchronize(self):
        self._check(self.lib.pic_synchronize(self.ctx))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.pic_get_stream(self.ctx, ctypes.byref(s)))
        return s.value or 0

    def diagnostics(self) -> dict:
        out = (ctypes.c_double * L.NDIAG)()
        self._check(self.lib.pic_diagnostics(self.ctx, out, L.NDIAG))
        return dict(field_energy=out[0], kinetic0=out[1], kinetic1=out[2], charge0=out[3], charge1=out[4],
                    gauss_max=out[5])

    def initialize_particles(self, kind: int, cell_per_particles: int, density="uniform", value: float = 1.0,
                             lo=(0.0, 0.0, 0.0), hi=(0.0, 0.0, 0.0), knots=None,
                             initial_p=(0.0, 0.0, 0.0), initial_s=(0.0, 0.0, 0.0)):
        """The reference's lattice loader on the device (pic_initialize_particles).
        density: "uniform" (value), "box" (value where lo < x*dx <= hi per
        axis) or "xprofile" (knots = (x_phys array, density array))."""
        d = L.PicDensity()
        d.kind = {"uniform": L.DENSITY_UNIFORM, "box": L.DENSITY_BOX, "xprofile": L.DENSITY_XPROFILE}[density]
        d.value = value
        for k in range(3):
            d.lo[k], d.hi[k] = lo[k], hi[k]
        keep = []
        if density == "xprofile":
            kx = np.ascontiguousarray(knots[0], dtype=np.float64)
            kv = np.ascontiguousarray(knots[1], dtype=np.float64)
            keep = [kx, kv]
            d.nknots = len(kx)
            d.knot_x = kx.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            d.knot_v = kv.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        p0 = (ctypes.c_double * 3)(*initial_p)
        s0 = (ctypes.c_double * 3)(*initial_s)
        self._check(self.lib.pic_initialize_particles(self.ctx, kind, ctypes.byref(d), cell_per_particles, p0, s0))
        del keep

    def generate_thermal(self, kind: int, ppc: int, density: float, u_th: float, seed: int):
        """Seeded thermal plasma generated on the device (pic_generate_thermal)."""
        self._check(self.lib.pic_generate_thermal(self.ctx, kind, ppc, density, u_th, seed))

    def solve_initial_field(self, rel_tol: float = 1e-10, max_iter: int = 50000) -> dict:
        """FP64 Poisson solve for the initial E of the current particles
        (pic_solve_initial_field): div E = rho - <rho>.  The relative
        residual cannot go much below 1e-13 (FP64 rounding); a smaller
        rel_tol ends with PIC_ENOCONV."""
        out = (ctypes.c_double * L.NPOISSON)()
        self._check(self.lib.pic_solve_initial_field(self.ctx, rel_tol, max_iter, out, L.NPOISSON))
        return dict(iterations=int(out[0]), rel_residual=out[1], mean_rho=out[2], gauss_max=out[3])

    def particle_order_stats(self, kind: int) -> dict:
        """Visitor lists and stragglers of the tiled kernel
        (pic_particle_order_stats)."""
        out = (ctypes.c_int64 * 4)()
        self._check(self.lib.pic_particle_order_stats(self.ctx, kind, out, 4))
        return dict(visitors=int(out[0]), lists_used=bool(out[1]), pushes_since_sort=int(out[2]),
                    global_kernel=int(out[3]))

    # -- profiling ------------------------------------------------------------------
    def profile(self, on: bool = True):
        self._check(self.lib.pic_profile_enable(self.ctx, 1 if on else 0))

    def profile_reset(self):
        self._check(self.lib.pic_profile_reset(self.ctx))

    def profile_read(self) -> dict:
        cap = 64
        names = (ctypes.c_char_p * cap)()
        ms = (ctypes.c_double * cap)()
        cnt = (ctypes.c_int64 * cap)()
        n = ctypes.c_int()
        self._check(self.lib.pic_profile_read(self.ctx, names, ms, cnt, cap, ctypes.byref(n)))
        return {names[i].decode(): (ms[i], cnt[i]) for i in range(min(n.value, cap))}

    def save(self, path: str):
        self._check(self.lib.pic_save(self.ctx, path.encode()))

    def load(self, path: str):
        self._check(self.lib.pic_load(self.ctx, path.encode()))
