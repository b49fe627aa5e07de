"""Failure detection through the C ABI.

The reference stops on a bad state with printf + exit(1) (the g_factor
range check, src/particle.cpp:632-636) or not at all (a NaN momentum or a
particle outside the buffers corrupts its arrays silently).  The GPU path
reports each as a status code: the kernels OR a status bit and skip the
particle, the next synchronising ABI call returns the code.  Every failure
here is made on the host (a bad record, a NaN planted in an uploaded array,
a parameter out of range); no test faults or hangs the GPU.
"""
import ctypes
import os

import numpy as np
import pytest

from golden_io import load
from parity import ARRAYS

from pic3d_b200 import _lib as L


def _sim(params, precision="fp64", **kw):
    from pic3d_b200.simulation import Simulation
    return Simulation(params, precision=precision, **kw)


def _code(fn, *a):
    try:
        fn(*a)
    except L.PicError as e:
        return e.code
    return L.PIC_OK


def test_create_rejects_dt_of_a_cell_or_more():
    """A particle moves less than a cell per step only if dt < min(dx, dy,
    dz) (|v| < c); pic_create refuses anything else, which is what keeps the
    kernels' cell-crossing status unreachable from valid input.  Checked
    before any CUDA call, so this runs without a GPU."""
    from pic3d_b200.simulation import params_from
    lib = L.load()
    p = params_from(load("periodic_o2")["params"])
    p.dt = p.dx
    h = ctypes.c_void_p()
    assert lib.pic_create(ctypes.byref(p), 0, ctypes.byref(h)) == L.PIC_EINVAL
    p.dt = 0.5 * p.dx
    p.local_xcells = 1 << 21
    assert lib.pic_create(ctypes.byref(p), 0, ctypes.byref(h)) == L.PIC_EINVAL


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_upload_rejects_non_finite_momentum(precision):
    g = load("periodic_o2")
    rec = g["input"][0].copy()
    rec["px"][3] = np.nan
    sim = _sim(g["params"], precision)
    assert _code(sim.upload_particles, 0, rec) == L.PIC_ENAN
    assert sim.num_particles(0) == 0
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_nan_field_gives_enan_after_the_push(precision):
    """A NaN planted in an uploaded E array reaches a particle's gathered
    field; its momentum is non-finite and the push reports PIC_ENAN."""
    g = load("periodic_o2")
    st = g["step1"]
    sim = _sim(g["params"], precision)
    sim.upload_state(st)
    ex = st["ex"].copy()
    m = int(g["params"]["mem"])
    n = [int(g["params"][f"local_{a}cells"]) for a in ("x", "y", "z")]
    # an electron away from every face: the ghost layers are rewritten from
    # the interior before the gather, so the NaN must sit on a physical point
    e = st["particles"][0]
    inner = np.ones(len(e), bool)
    for a, na in zip(("x", "y", "z"), n):
        inner &= (e[a] >= 2.0) & (e[a] < na - 2.0)
    p = e[np.flatnonzero(inner)[0]]
    # the field point under it (buffer index = x + mem - 1)
    i, j, k = (int(p[a]) + m - 1 for a in ("x", "y", "z"))
    ex[k, j, i] = np.nan
    sim.upload_array("ex", ex)
    sim.step = 1
    sim.run_main_time_loop(1)
    assert _code(sim.synchronize) == L.PIC_ENAN
    sim.close()


@pytest.mark.gpu
def test_particle_outside_the_buffers_gives_eoob():
    """x non-periodic (mixed_o2): a particle far beyond x = n has no stencil
    inside the buffers; the FP64 push skips it and reports PIC_EOOB, an FP32
    upload refuses it (its packed cell index cannot hold the cell)."""
    g = load("mixed_o2")
    nx = int(g["params"]["local_xcells"])
    st = g["step1"]
    parts = [p.copy() for p in st["particles"]]
    parts[0]["x"][0] = nx + 20.5
    sim = _sim(g["params"], "fp64")
    sim.upload_state({**st, "particles": parts})
    sim.step = 1
    sim.run_main_time_loop(1)
    assert _code(sim.synchronize) == L.PIC_EOOB
    sim.close()
    sim = _sim(g["params"], "fp32")
    assert _code(sim.upload_particles, 0, parts[0]) == L.PIC_EOOB
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_deposit_of_a_move_over_a_cell_gives_eoob(precision):
    """currents_particle of a record moved by more than one cell (the
    Esirkepov span assumes at most one): the cell-crossing status, reported
    as PIC_EOOB."""
    g = load("periodic_o2")
    sim = _sim(g["params"], precision)
    rec = g["input"][0][:1].copy()
    rec["x_old"], rec["y_old"], rec["z_old"] = rec["x"] - 2.5, rec["y"], rec["z"]
    lib = L.load()
    assert lib.pic_deposit_particle(sim.ctx, 0, rec.ctypes.data) == L.PIC_EOOB
    sim.close()


@pytest.mark.gpu
def test_g_factor_argument_beyond_the_table_gives_erange():
    """The reference exits when the spin g-factor argument chi lies beyond
    its table (src/particle.cpp:632-636).  With a tiny Schwinger field every
    electron's chi exceeds 100; the push reports PIC_ERANGE."""
    g = load("spin_o2")
    params = dict(g["params"], E_schwinger=1e-12)
    st = g["step1"]
    sim = _sim(params, "fp64")
    sim.set_g_table(g["g_data"])
    parts = [p.copy() for p in st["particles"]]
    parts[0]["sx"] = 0.3
    sim.upload_state({**st, "particles": parts})
    ey = np.full_like(st["ey"], 0.1)
    sim.upload_array("ey", ey)
    sim.step = 1
    sim.run_main_time_loop(1)
    assert _code(sim.synchronize) == L.PIC_ERANGE
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_save_load_round_trip(tmp_path, precision):
    """pic_save -> pic_load into a fresh context gives back every array and
    every particle record bit for bit, and the two contexts then step alike."""
    g = load("mixed_o2")
    a = _sim(g["params"], precision)
    for k in range(2):
        a.upload_particles(k, g["input"][k])
    a.initial_push()
    a.run_main_time_loop(3)
    path = os.path.join(str(tmp_path), "ckpt.bin")
    a.save(path)
    want = a.state()
    b = _sim(g["params"], precision)
    b.load(path)
    assert b.step == a.step
    got = b.state()
    for n in ARRAYS:
        assert np.array_equal(got[n], want[n]), n
    for k in range(2):
        x, y = np.sort(got["particles"][k], order="id"), np.sort(want["particles"][k], order="id")
        # field by field: the record's padding words carry no data
        for f in x.dtype.names:
            assert x[f].tobytes() == y[f].tobytes(), (k, f)
    a.run_main_time_loop(2)
    b.run_main_time_loop(2)
    sa, sb = a.state(), b.state()
    for n in ARRAYS:
        d = np.linalg.norm(sa[n] - sb[n]) / max(np.linalg.norm(sa[n]), 1e-300)
        assert d < (1e-12 if precision == "fp64" else 1e-6), (n, d)
    a.close()
    b.close()


@pytest.mark.gpu
def test_load_rejects_a_mismatched_checkpoint(tmp_path):
    path = os.path.join(str(tmp_path), "bad.bin")
    with open(path, "wb") as f:
        f.write(b"NOTACKPT" + b"\0" * 64)
    g = load("periodic_o2")
    sim = _sim(g["params"])
    assert _code(sim.load, path) == L.PIC_EINVAL
    sim.close()
