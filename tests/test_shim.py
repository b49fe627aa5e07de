"""The C++ drop-in shim (pic3d_b200/shim/pic3d_shim.cpp) against the
reference's own sources.

Two harness mains are each linked twice by oracle/Makefile: against the
reference's src/{field,particle,boundary,mpi_utils,simulation}.cpp (CPU) and
against the shim over libpic3d_b200.so (GPU):
  * oracle/ref/ref_harness.cpp: the main.cpp sequence (t=0 push + exchange,
    then run_main_time_loop with an output every step);
  * oracle/ref/ref_surface.cpp: the rest of the call surface
    (initialize_particles, the scalar helpers, the full-dt field update,
    per-array halo and fold, the binomial filter, currents_particle,
    radiating_boundary and both field halves on given arrays).
The GPU tests run both builds on the same inputs and compare the dumps.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import oracle as O  # noqa: E402
from golden_io import CASES, load  # noqa: E402
from parity import rel_l2  # noqa: E402
from pic3d_b200.workloads import PARTICLE_DTYPE, tiny_cases  # noqa: E402

REF_DIR = os.path.join(REPO, "oracle", "_ref")
BINS = {n: os.path.join(REF_DIR, n) for n in ("pic3d_ref", "pic3d_shim_run", "pic3d_surface_ref",
                                               "pic3d_surface_shim")}
SHIM_SRC = os.path.join(REPO, "pic3d_b200", "shim", "pic3d_shim.cpp")
# the reference source tree, when present (PIC3D_REFERENCE); the header
# check is skipped without it
REFERENCE_INCLUDE = os.path.join(os.environ.get("PIC3D_REFERENCE", ""), "include")

# every function and global the five replaced reference sources define
SURFACE = [
    "update_electromagnetic_fields(int, int, int)", "update_electromagnetic_fields_first(int, int, int)",
    "update_electromagnetic_fields_second(int, int, int)", "initialize_particles(", "update_particle_position_momentum(",
    "currents_particle(particle const&, int)", "filter_field(double***)", "binomial_filter_currents()",
    "shape_function_2(double, double*)", "shape_function_4(double, double*)", "clear_currents()",
    "exchange_currents(int)", "g_factor(double)", "generate_laser_pulse(double, double)",
    "Gpulse(double, double, double, double)", "radiating_boundary(int, int, int, int, int)",
    "exchange_boundary_data(double***, int)", "exchange_particle_data(", "exchange_boundary_current_fixed(double***, int)",
    "initialize_simulation(int, int)", "initialize_domain(int)", "run_main_time_loop(",
    "dmatrix(long, long, long, long)", "free_dmatrix(double**, long, long)", "free_dmatrix(double**, long)",
    "dtensor3(long, long, long, long, long, long)", "dtensor4(long, long, long, long, long, long, long, long)",
    "free_dtensor3(double***, long, long, long)", "free_dtensor4(double****, long, long, long, long)",
    "free_memory()",
]
GLOBALS = ["max_error", "rho_local", "rho_particle", "ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "phi",
           "phi_new", "current_recv_xminus", "current_recv_xplus", "current_recv_yminus", "current_recv_yplus",
           "current_recv_zminus", "current_recv_zplus"]


@pytest.mark.skipif(not os.environ.get("PIC3D_REFERENCE") or not os.path.isdir(REFERENCE_INCLUDE),
                    reason="reference headers not present (PIC3D_REFERENCE unset)")
def test_shim_defines_the_reference_surface(tmp_path):
    """Compiled against the reference's headers, the shim defines every
    function and global of the five translation units it replaces."""
    obj = tmp_path / "shim.o"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-c", SHIM_SRC, "-o", str(obj),
                    "-I" + os.path.join(REPO, "oracle", "ref"), "-I" + REFERENCE_INCLUDE,
                    "-I" + os.path.join(REPO, "include"), "-I" + os.path.dirname(SHIM_SRC)], check=True)
    nm = subprocess.run(["nm", "-C", "--defined-only", str(obj)], check=True, capture_output=True, text=True).stdout
    defined = [line.split(" ", 2)[2] for line in nm.splitlines() if len(line.split(" ", 2)) == 3]
    for sig in SURFACE:
        assert any(d.startswith(sig) for d in defined), sig
    for g in GLOBALS:
        assert g in defined, g
    # everything the shim needs from the device side is the C ABI
    undefined = subprocess.run(["nm", "-C", "--undefined-only", str(obj)], check=True, capture_output=True,
                               text=True).stdout
    gpu = {l.split()[-1] for l in undefined.splitlines() if l.split()[-1].startswith("pic_")}
    header = open(os.path.join(REPO, "include", "pic3d_gpu.h")).read()
    for name in gpu:
        assert f" {name}(" in header, name


def test_shim_harnesses_are_built():
    """Where the reference exists, build() produced both builds of both
    harnesses (the GPU tests below need them)."""
    if not os.path.isdir(REFERENCE_INCLUDE):
        pytest.skip("reference headers not present")
    for name, path in BINS.items():
        assert os.path.exists(path), f"{name} missing: run make -C oracle all"


def _need(*names):
    for n in names:
        if not os.path.exists(BINS[n]):
            pytest.skip(f"{BINS[n]} not built")


# ---------------------------------------------------------------------------
# main.cpp sequence through the shim

@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_shim_main_sequence_matches_reference(case):
    _need("pic3d_ref", "pic3d_shim_run")
    g = load(case)
    w, parts, steps = g["params"], g["input"], int(g["steps"])
    ref, _ = O.run_reference(w, parts, steps, binary=BINS["pic3d_ref"])
    gpu, _ = O.run_reference(w, parts, steps, binary=BINS["pic3d_shim_run"])
    assert len(ref) == len(gpu) == steps + 1
    for s, (a, b) in enumerate(zip(gpu, ref)):
        for n in O.FIELD_NAMES + O.RING_NAMES:
            e = rel_l2(a[n], b[n])
            assert e <= 1e-10, (case, s, n, e)
        for k in range(2):
            pa, pb = a["particles"][k], b["particles"][k]
            assert len(pa) == len(pb), (case, s, k)
            pa, pb = np.sort(pa, order="id"), np.sort(pb, order="id")
            assert np.array_equal(pa["id"], pb["id"])
            for f in ("x", "y", "z", "px", "py", "pz"):
                err = np.max(np.abs(pa[f] - pb[f]), initial=0.0)
                scale = max(np.max(np.abs(pb[f]), initial=0.0), 1.0)
                assert err <= 1e-10 * scale, (case, s, k, f, err)


# ---------------------------------------------------------------------------
# the rest of the call surface

def _surface_workload(name):
    c = tiny_cases()
    if name == "periodic_o2_ppc8":
        return c["periodic_o2"].with_(ppc=(8, 0))
    if name == "laser_o4_ppc2":
        return c["laser_o4"].with_(ppc=(2, 0))
    raise KeyError(name)


def _run_surface(binary, w):
    with tempfile.TemporaryDirectory(prefix="pic3d_surface_") as tmp:
        prm = os.path.join(tmp, "params.txt")
        O.write_params_file(prm, w, 1, 1)
        out = os.path.join(tmp, "out.bin")
        env = dict(os.environ, PIC3D_REF_PARAMS=prm, PIC3D_G_TXT=O.REF_G_TXT)
        r = subprocess.run([binary, out], env=env, capture_output=True, text=True, cwd=tmp)
        assert r.returncode == 0, r.stderr[-2000:]
        return _parse_surface(open(out, "rb").read(), w)


def _parse_surface(raw, w):
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a

    out = {"particles": []}
    for _ in range(2):
        n = int(take("<i8", 1)[0])
        out["particles"].append(take(PARTICLE_DTYPE, n).copy())
    out["shapes"] = take("<f8", 6 * 8).reshape(6, 8)
    out["g"] = take("<f8", 8)
    out["laser"] = take("<f8", 5 * 4).reshape(5, 4)
    fs, rs = O.field_shape(w), O.ring_shape(w)
    nf, nr = int(np.prod(fs)), int(np.prod(rs))
    out["stages"] = []
    while off < len(raw):
        st = {}
        for n in O.FIELD_NAMES:
            st[n] = take("<f8", nf).reshape(fs)
        for n in O.RING_NAMES:
            st[n] = take("<f8", nr).reshape(rs)
        out["stages"].append(st)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["periodic_o2_ppc8", "laser_o4_ppc2"])
def test_shim_call_surface_matches_reference(name):
    _need("pic3d_surface_ref", "pic3d_surface_shim")
    w = _surface_workload(name)
    ref = _run_surface(BINS["pic3d_surface_ref"], w)
    gpu = _run_surface(BINS["pic3d_surface_shim"], w)
    # initialize_particles: host code on both sides, identical records (the
    # struct's 4 padding bytes after `rank` are not compared)
    for k in range(2):
        a, b = gpu["particles"][k], ref["particles"][k]
        assert len(a) == len(b) > 0
        for f in PARTICLE_DTYPE.names:
            assert np.array_equal(a[f], b[f]), (k, f)
    np.testing.assert_allclose(gpu["shapes"], ref["shapes"], rtol=0, atol=1e-14)
    np.testing.assert_array_equal(gpu["g"], ref["g"])
    np.testing.assert_allclose(gpu["laser"], ref["laser"], rtol=1e-12, atol=1e-15)
    assert len(gpu["stages"]) == len(ref["stages"]) == 6
    for s, (a, b) in enumerate(zip(gpu["stages"], ref["stages"])):
        for n in O.FIELD_NAMES + O.RING_NAMES:
            e = rel_l2(a[n], b[n])
            assert e <= 1e-12, (name, s, n, e)
