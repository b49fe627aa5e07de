"""Python driver for the CPU oracle — TEST INFRASTRUCTURE ONLY.

Two checkers live here:

* ``Oracle``: ctypes wrapper of this repository's C restatement of the
  reference per-timestep loop (``pic_oracle.c``).  Runs anywhere gcc runs.
* ``run_reference``: runs the reference's own sources, built unmodified by
  ``oracle/Makefile`` into ``oracle/_ref/pic3d_ref`` (only where the
  reference tree was present at build time), and reads its per-step dumps.

Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU-baseline leg may
import this module.  Nothing in the GPU product path calls it.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from pic3d_b200.workloads import PARTICLE_DTYPE, Workload  # noqa: E402

LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "pic3d_ref")
REF_BIN_O0 = os.path.join(HERE, "_ref", "pic3d_ref_O0")
REF_G_TXT = os.path.join(HERE, "_ref", "g.txt")

_P = ctypes.POINTER
_D = ctypes.c_double
_I = ctypes.c_int32


class OrcState(ctypes.Structure):
    _fields_ = [
        ("local_xcells", _I), ("local_ycells", _I), ("local_zcells", _I), ("mem", _I),
        ("rank_period", _I * 3), ("laser_polarization", _I),
        ("Pi", _D), ("omega", _D), ("l0", _D), ("Lx", _D),
        ("dx", _D), ("dy", _D), ("dz", _D), ("dt", _D), ("dt_half", _D),
        ("laser_amplitude", _D), ("laser_pulse_duration", _D), ("laser_start_time", _D),
        ("waist", _D), ("xfocus", _D), ("yfocus", _D), ("zfocus", _D), ("phase", _D),
        ("E_schwinger", _D),
        ("laser_envelope", _I), ("laser_profile", _I), ("profile_coef", _P(_D)), ("profile_n", _I),
        ("absorbing", _I), ("g_data_size", _I), ("g_data", _P(_D)),
        ("ex", _P(_D)), ("ey", _P(_D)), ("ez", _P(_D)), ("bx", _P(_D)), ("by", _P(_D)), ("bz", _P(_D)),
        ("jx", _P(_D)), ("jy", _P(_D)), ("jz", _P(_D)), ("rho0", _P(_D)), ("rho1", _P(_D)),
        ("particles", ctypes.c_void_p * 2), ("num_particles", ctypes.c_int64 * 2),
        ("scratch", ctypes.c_void_p),
        ("out_of_bounds", ctypes.c_int64), ("g_factor_errors", ctypes.c_int64),
    ]


_lib = None


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def load_lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "pic_oracle.c")
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
            build_oracle()
        lib = ctypes.CDLL(LIB_PATH)
        for name in ["orc_radiating_boundary", "orc_exchange_boundary_data", "orc_fields_first",
                     "orc_fields_second", "orc_clear_currents", "orc_push", "orc_exchange_particles",
                     "orc_exchange_current", "orc_exchange_currents", "orc_initial", "orc_step", "orc_run",
                     "orc_currents_particle"]:
            getattr(lib, name).restype = None
        lib.orc_shape_function_2.argtypes = [_D, _P(_D)]
        lib.orc_shape_function_4.argtypes = [_D, _P(_D)]
        lib.orc_g_factor.restype = _D
        lib.orc_g_factor.argtypes = [ctypes.c_void_p, _D]
        lib.orc_gpulse.restype = _D
        lib.orc_gpulse.argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
        _lib = lib
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_P(_D))


def _p(w):
    return w if isinstance(w, dict) else w.params()


def field_shape(w):
    p = _p(w)
    m = int(p["mem"])
    return (int(p["local_zcells"]) + 2 * m, int(p["local_ycells"]) + 2 * m, int(p["local_xcells"]) + 2 * m)


def ring_shape(w):
    return tuple(n + 2 for n in field_shape(w))


FIELD_NAMES = ["ex", "ey", "ez", "bx", "by", "bz"]
RING_NAMES = ["jx", "jy", "jz", "rho0", "rho1"]


class Oracle:
    """FP64 CPU oracle state for one workload (restatement in pic_oracle.c)."""

    def __init__(self, w, particles=None, fields=None, g_data=None, profile=None):
        """`w` is a Workload or its parameter dictionary (Workload.params())."""
        self.w = w
        self.params = _p(w)
        self.lib = load_lib()
        fs, rs = field_shape(w), ring_shape(w)
        self.arrays = {n: np.zeros(fs) for n in FIELD_NAMES}
        self.arrays.update({n: np.zeros(rs) for n in RING_NAMES})
        if fields is not None:
            for n, a in fields.items():
                self.arrays[n][...] = a
        parts = particles if particles is not None else [np.zeros(0, PARTICLE_DTYPE)] * 2
        # the C side reads 144-byte records: convert whatever layout came in
        # (numpy drops the record padding when it concatenates structured arrays)
        self.parts = [np.array(p, dtype=PARTICLE_DTYPE, copy=True, order="C") for p in parts]
        cap = max(1, max(len(p) for p in self.parts))
        self.scratch = np.zeros(cap, dtype=PARTICLE_DTYPE)
        self.g_data = None if g_data is None else np.ascontiguousarray(g_data, dtype=np.float64)
        self.profile = None if profile is None else np.ascontiguousarray(profile, dtype=np.float64)
        self.s = OrcState()
        self._fill_struct()

    def _fill_struct(self):
        p = self.params
        s = self.s
        s.local_xcells, s.local_ycells, s.local_zcells, s.mem = int(p["local_xcells"]), int(p["local_ycells"]), \
            int(p["local_zcells"]), int(p["mem"])
        s.rank_period[0], s.rank_period[1], s.rank_period[2] = int(p["period_x"]), int(p["period_y"]), \
            int(p["period_z"])
        s.laser_polarization = int(p["laser_polarization"])
        for k in ["Pi", "omega", "l0", "Lx", "dx", "dy", "dz", "dt", "dt_half", "laser_amplitude",
                  "laser_pulse_duration", "laser_start_time", "waist", "xfocus", "yfocus", "zfocus", "phase",
                  "E_schwinger"]:
            setattr(s, k, p[k])
        s.laser_envelope = int(p.get("laser_envelope", 0))
        s.absorbing = int(p.get("absorbing", 0))
        if self.profile is not None:
            s.laser_profile = 1
            s.profile_coef = _dptr(self.profile)
            s.profile_n = self.profile.shape[0]
        if self.g_data is not None:
            s.g_data = _dptr(self.g_data)
            s.g_data_size = len(self.g_data)
        for n in FIELD_NAMES + RING_NAMES:
            setattr(s, n, _dptr(self.arrays[n]))
        for k in range(2):
            s.particles[k] = self.parts[k].ctypes.data
            s.num_particles[k] = len(self.parts[k])
        s.scratch = self.scratch.ctypes.data

    @property
    def ref(self):
        return ctypes.byref(self.s)

    def particles(self, kind):
        return self.parts[kind][: self.s.num_particles[kind]]

    def state(self) -> dict:
        st = {n: a.copy() for n, a in self.arrays.items()}
        st["particles"] = [self.particles(k).copy() for k in range(2)]
        return st

    # reference call surface -------------------------------------------
    def radiating_boundary(self, step, is_left=1, is_right=0):
        self.lib.orc_radiating_boundary(self.ref, is_left, is_right, step)

    def fields_first(self):
        self.lib.orc_fields_first(self.ref)

    def fields_second(self):
        self.lib.orc_fields_second(self.ref)

    def clear_currents(self):
        self.lib.orc_clear_currents(self.ref)

    def push(self, kind):
        self.lib.orc_push(self.ref, kind)

    def exchange_particles(self, kind):
        self.lib.orc_exchange_particles(self.ref, kind)

    def exchange_currents(self):
        self.lib.orc_exchange_currents(self.ref)

    def initial(self):
        self.lib.orc_initial(self.ref)

    def step(self, step):
        self.lib.orc_step(self.ref, step)

    def run(self, first_step, nsteps):
        self.lib.orc_run(self.ref, first_step, nsteps)


def shape_function(order: int, x: float) -> np.ndarray:
    lib = load_lib()
    out = np.zeros(5)
    if order == 2:
        lib.orc_shape_function_2(x, _dptr(out))
        return out[:3]
    lib.orc_shape_function_4(x, _dptr(out))
    return out


# ---------------------------------------------------------------------------
# the reference build

def have_reference_build() -> bool:
    return os.path.exists(REF_BIN)


def write_particle_file(path, particles):
    with open(path, "wb") as f:
        np.array([len(particles[0]), len(particles[1])], dtype="<i8").tofile(f)
        for p in particles:
            np.ascontiguousarray(p, dtype=PARTICLE_DTYPE).tofile(f)


def write_params_file(path, w, steps: int, output_interval: int = 1):
    p = dict(_p(w))
    p["timesteps"] = steps
    p["output_interval"] = output_interval
    with open(path, "w") as f:
        for k, v in p.items():
            f.write(f"{k} {float(v)!r}\n")


def read_fields_dump(path, w: Workload) -> dict:
    fs, rs = field_shape(w), ring_shape(w)
    raw = np.fromfile(path, dtype="<f8")
    nf, nr = int(np.prod(fs)), int(np.prod(rs))
    out, off = {}, 0
    for n in FIELD_NAMES:
        out[n] = raw[off:off + nf].reshape(fs)
        off += nf
    for n in RING_NAMES:
        out[n] = raw[off:off + nr].reshape(rs)
        off += nr
    return out


def read_particles_dump(path) -> list:
    with open(path, "rb") as f:
        counts = np.fromfile(f, dtype="<i8", count=2)
        return [np.fromfile(f, dtype=PARTICLE_DTYPE, count=int(c)) for c in counts]


def run_reference(w: Workload, particles, steps: int, outdir=None, binary=None, timing=False,
                  output_interval: int = 1, cwd=None):
    """Run the reference build: t=0 push, then `steps` loop iterations.

    Returns (list of per-step states or None, timing dict or None)."""
    binary = binary or REF_BIN
    if not os.path.exists(binary):
        raise FileNotFoundError(f"{binary} not built (run make -C oracle ref where the reference exists)")
    tmp = tempfile.mkdtemp(prefix="pic3d_ref_")
    try:
        ppath = os.path.join(tmp, "particles.bin")
        write_particle_file(ppath, particles)
        prm = os.path.join(tmp, "params.txt")
        write_params_file(prm, w, steps, output_interval)
        dump = outdir if outdir is not None else (tmp if not timing else "-")
        env = dict(os.environ, PIC3D_REF_PARAMS=prm, PIC3D_G_TXT=REF_G_TXT)
        args = [binary, ppath, dump] + (["time"] if timing else [])
        r = subprocess.run(args, env=env, capture_output=True, text=True, cwd=cwd or tmp)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-2000:]}")
        tinfo = None
        if timing:
            for line in r.stdout.splitlines()[::-1]:
                if line.startswith("{"):
                    tinfo = json.loads(line)
                    break
        states = None
        if dump != "-":
            states = []
            for s in range(0, steps + 1, output_interval):
                st = read_fields_dump(os.path.join(dump, f"step_{s:05d}.fields"), w)
                st["particles"] = read_particles_dump(os.path.join(dump, f"step_{s:05d}.particles"))
                states.append(st)
        return states, tinfo
    finally:
        if outdir is None:
            import shutil
            shutil.rmtree(tmp, ignore_errors=True)


def run_oracle(w, particles, steps: int, g_data=None, profile=None):
    """Same sequence as run_reference with the C restatement; returns the
    list of states after the t=0 sequence and after each step."""
    o = Oracle(w, particles, g_data=g_data, profile=profile)
    o.initial()
    states = [o.state()]
    for s in range(1, steps + 1):
        o.step(s)
        states.append(o.state())
    return states, o


def load_g_table():
    """The reference's g-factor table when the reference build is present."""
    if os.path.exists(REF_G_TXT):
        # the reference reads the first g_data_size = 2849 values
        # (src/constants.cpp:111-131); the file holds one more
        return np.loadtxt(REF_G_TXT)[:2849].copy()
    return None


def _read_params_file(path):
    p = {}
    with open(path) as f:
        for line in f:
            k, v = line.split()
            p[k] = float(v)
    for k in ("local_xcells", "local_ycells", "local_zcells", "mem", "period_x", "period_y", "period_z",
              "laser_polarization", "timesteps", "laser_envelope"):
        if k in p:
            p[k] = int(p[k])
    return p


def _read_particle_file(path):
    with open(path, "rb") as f:
        counts = np.fromfile(f, dtype="<i8", count=2)
        return [np.fromfile(f, dtype=PARTICLE_DTYPE, count=int(c)) for c in counts]


if __name__ == "__main__":
    # `python oracle.py --port-time particles.bin params.txt`: time the C
    # restatement like the reference harness's "time" mode (CPU baseline
    # fallback when the reference build is not present).
    import time
    if len(sys.argv) == 4 and sys.argv[1] == "--port-time":
        prm = _read_params_file(sys.argv[3])
        parts = _read_particle_file(sys.argv[2])
        o = Oracle(prm, parts)
        o.initial()
        n0 = int(o.s.num_particles[0] + o.s.num_particles[1])
        t0 = time.perf_counter()
        o.run(1, prm["timesteps"])
        dt = time.perf_counter() - t0
        n1 = int(o.s.num_particles[0] + o.s.num_particles[1])
        print(json.dumps({"steps": prm["timesteps"], "particles_start": n0, "particles_end": n1,
                          "loop_seconds": dt}))
