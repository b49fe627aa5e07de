"""The reference's on-disk output layout (src/io_utils.cpp) from a state.

output_data_hdf5 writes field[nc_zst + k][nc_yst + j][nc_xst + i] to
dataset position (k, j, i) for the physical cells (io_utils.cpp:79-90);
the ring buffers (J, rho_particle) are indexed with the same buffer
coordinates, one point further in (their arrays start at -1).
output_particles_hdf5 concatenates the species and tags the dataset with
timestep, total_particles and num_processes (io_utils.cpp:240-329).
"""
import numpy as np
import pytest

from golden_io import load

from pic3d_b200 import output as OUT
from pic3d_b200.workloads import PARTICLE_DTYPE


def _coded_state(nz, ny, nx, mem):
    """Arrays whose value encodes the buffer coordinate (k, j, i) of each
    point (ring arrays: buffer coordinate = array index - 1)."""
    fs = (nz + 2 * mem, ny + 2 * mem, nx + 2 * mem)
    rs = tuple(s + 2 for s in fs)
    k, j, i = np.meshgrid(*[np.arange(s) for s in fs], indexing="ij")
    kr, jr, ir = np.meshgrid(*[np.arange(s) - 1 for s in rs], indexing="ij")
    st = {}
    for c, n in enumerate(["ex", "ey", "ez", "bx", "by", "bz"]):
        st[n] = (1e6 * k + 1e3 * j + i + 0.1 * c).astype(np.float64)
    for c, n in enumerate(["jx", "jy", "jz", "rho0", "rho1"]):
        st[n] = (1e6 * kr + 1e3 * jr + ir + 0.01 * (c + 1)).astype(np.float64)
    return st


def test_field_datasets_follow_the_reference_index_map():
    nz, ny, nx, mem = 5, 6, 7, 2
    st = _coded_state(nz, ny, nx, mem)
    ds = OUT.field_datasets(st, mem)
    assert list(ds) == OUT.FIELD_DATASETS
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    coord = 1e6 * (k + mem) + 1e3 * (j + mem) + (i + mem)   # nc_*st = mem on one rank
    for c, n in enumerate(["ex", "ey", "ez", "bx", "by", "bz"]):
        np.testing.assert_array_equal(ds[n], coord + 0.1 * c)
    for c, n in enumerate(["jx", "jy", "jz"]):
        np.testing.assert_array_equal(ds[n], coord + 0.01 * (c + 1))
    np.testing.assert_array_equal(ds["rho_electron"], coord + 0.04)
    np.testing.assert_array_equal(ds["rho_proton"], coord + 0.05)
    assert np.all(ds["rho"] == 0.0)
    for a in ds.values():
        assert a.shape == (nz, ny, nx) and a.dtype == np.float64


def test_raw_round_trip_of_a_golden_state(tmp_path):
    g = load("laser_o4")
    st = g["final"]
    mem = int(g["params"]["mem"])
    fpath = OUT.write_fields(st, mem, 12, str(tmp_path))
    ppath = OUT.write_particles(st["particles"], 12, str(tmp_path))
    assert fpath.endswith("output_step_0012.raw") and ppath.endswith("particles_step_0012.raw")
    data, _ = OUT.read_raw(fpath)
    ref = OUT.field_datasets(st, mem)
    for n in OUT.FIELD_DATASETS:
        assert data[n].tobytes() == ref[n].tobytes()
    pdata, attrs = OUT.read_raw(ppath)
    rec = pdata["particles"]
    want = np.zeros(len(st["particles"][0]) + len(st["particles"][1]), PARTICLE_DTYPE)
    want[:len(st["particles"][0])] = st["particles"][0]
    want[len(st["particles"][0]):] = st["particles"][1]
    assert rec.dtype == PARTICLE_DTYPE and rec.tobytes() == want.tobytes()
    assert attrs["particles"] == {"timestep": 12, "total_particles": len(want), "num_processes": 1}


def test_no_particle_file_without_particles(tmp_path):
    empty = [np.zeros(0, PARTICLE_DTYPE)] * 2
    assert OUT.write_particles(empty, 0, str(tmp_path)) is None


def test_hdf5_conversion_needs_h5py(tmp_path):
    pytest.importorskip("h5py")
    g = load("periodic_o2")
    path = OUT.write_fields(g["final"], int(g["params"]["mem"]), 3, str(tmp_path))
    OUT.raw_to_hdf5(path, str(tmp_path / "out.h5"))
