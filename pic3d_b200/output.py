"""Output in the reference's on-disk layout (src/io_utils.cpp).

The reference writes, every output step, two parallel-HDF5 files:

* ``output/output_step_%04d.h5`` (``output_data_hdf5``, io_utils.cpp:11-154):
  FP64 datasets of the physical cells in (nz, ny, nx) order --
  ``/rho`` (the reference's ``rho_local``, allocated at simulation.cpp:143
  and never filled: written here as zeros), ``/rho_electron``,
  ``/rho_proton``, ``/ex`` ``/ey`` ``/ez`` ``/bx`` ``/by`` ``/bz`` ``/jx``
  ``/jy`` ``/jz`` (io_utils.cpp:133-144);
* ``output/particles_step_%04d.h5`` (``output_particles_hdf5``,
  io_utils.cpp:157-347): one ``/particles`` dataset of the 144-byte particle
  compound (id, x .. weight, rank; io_utils.cpp:219-236), every species
  concatenated in species order, with integer attributes ``timestep``,
  ``total_particles`` and ``num_processes`` (io_utils.cpp:311-329).

Neither the HDF5 library nor h5py is part of this image, so the writers here
produce the same datasets as a raw directory (``<name>.raw/``: one
little-endian file per dataset plus ``layout.json`` with its shape, type and
attributes); ``raw_to_hdf5`` turns such a directory into the reference's
HDF5 file wherever h5py is installed.  The state comes from the device only
when written (``Simulation.state``/``download_*``), as the reference's
output calls read its host arrays.
"""
from __future__ import annotations

import json
import os

import numpy as np

from .workloads import PARTICLE_DTYPE

FIELD_DATASETS = ["rho", "rho_electron", "rho_proton", "ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz"]
_SOURCE = {"rho_electron": "rho0", "rho_proton": "rho1"}


def physical(a: np.ndarray, mem: int, ring: bool) -> np.ndarray:
    """The physical cells (nz, ny, nx) of a field buffer (n + 2 mem per axis)
    or a ring buffer (n + 2 mem + 2, one extra point on each side)."""
    o = mem + (1 if ring else 0)
    nz, ny, nx = (s - 2 * o for s in a.shape)
    return np.ascontiguousarray(a[o:o + nz, o:o + ny, o:o + nx])


def field_datasets(state: dict, mem: int) -> dict:
    """Dataset name -> (nz, ny, nx) FP64 array from a state dictionary
    (ex..bz field buffers, jx..rho1 ring buffers, as Simulation.state())."""
    out = {}
    ref = physical(state["ex"], mem, False)
    for name in FIELD_DATASETS:
        if name == "rho":
            out[name] = np.zeros_like(ref)
            continue
        src = _SOURCE.get(name, name)
        out[name] = physical(state[src], mem, src not in ("ex", "ey", "ez", "bx", "by", "bz"))
    return out


def particle_dataset(particles) -> np.ndarray:
    """Every species' records concatenated in species order."""
    # filled slice by slice: concatenating structured arrays may drop the
    # record's padding (136 instead of 144 bytes)
    out = np.zeros(sum(len(p) for p in particles), PARTICLE_DTYPE)
    o = 0
    for p in particles:
        out[o:o + len(p)] = p
        o += len(p)
    return out


def _write_raw(path: str, datasets: dict, attrs: dict | None = None):
    os.makedirs(path, exist_ok=True)
    layout = {"datasets": {}}
    for name, a in datasets.items():
        fn = name + (".rec" if a.dtype == PARTICLE_DTYPE else ".f64")
        a.tofile(os.path.join(path, fn))
        layout["datasets"][name] = {"file": fn, "shape": list(a.shape),
                                    "dtype": "particle144" if a.dtype == PARTICLE_DTYPE else "<f8",
                                    "attrs": (attrs or {}).get(name, {})}
    with open(os.path.join(path, "layout.json"), "w") as f:
        json.dump(layout, f, indent=1)


def read_raw(path: str) -> tuple[dict, dict]:
    """(datasets, attributes) of a raw directory written here."""
    with open(os.path.join(path, "layout.json")) as f:
        layout = json.load(f)
    data, attrs = {}, {}
    for name, d in layout["datasets"].items():
        dt = PARTICLE_DTYPE if d["dtype"] == "particle144" else np.dtype("<f8")
        data[name] = np.fromfile(os.path.join(path, d["file"]), dtype=dt).reshape(d["shape"])
        attrs[name] = d["attrs"]
    return data, attrs


def write_fields(state: dict, mem: int, step: int, outdir: str = "output") -> str:
    """output_data_hdf5(step) as a raw directory; returns its path."""
    path = os.path.join(outdir, f"output_step_{step:04d}.raw")
    _write_raw(path, field_datasets(state, mem))
    return path


def write_particles(particles, step: int, outdir: str = "output", num_processes: int = 1) -> str | None:
    """output_particles_hdf5(step) as a raw directory; like the reference,
    nothing is written when there are no particles (io_utils.cpp:199-205)."""
    rec = particle_dataset(particles)
    if len(rec) == 0:
        return None
    path = os.path.join(outdir, f"particles_step_{step:04d}.raw")
    _write_raw(path, {"particles": rec}, {"particles": {"timestep": int(step), "total_particles": int(len(rec)),
                                                        "num_processes": int(num_processes)}})
    return path


def write_step(sim, step: int, outdir: str = "output") -> tuple[str, str | None]:
    """Both outputs of one step of a Simulation (device -> host first)."""
    st = sim.state()
    return (write_fields(st, int(sim.params.mem), step, outdir),
            write_particles(st["particles"], step, outdir))


def raw_to_hdf5(raw_dir: str, h5_path: str):
    """Write the reference's HDF5 file from a raw directory (needs h5py)."""
    import h5py  # not in this image; present wherever the HDF5 files are wanted
    data, attrs = read_raw(raw_dir)
    with h5py.File(h5_path, "w") as f:
        for name, a in data.items():
            ds = f.create_dataset("/" + name, data=a)
            for k, v in attrs.get(name, {}).items():
                ds.attrs.create(k, v, dtype=np.int32)
