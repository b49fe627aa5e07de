"""Generate the golden vectors under tests/golden/ from the reference itself.

Runs the reference PIC3D sources, built unmodified into oracle/_ref/pic3d_ref
by oracle/Makefile (single-rank MPI shim, raw dumps instead of HDF5), on
small seeded workloads that between them reach every reference code path on
the hot loop: 2nd- and 4th-order shapes, electrons and protons, periodic,
absorbing and mixed faces, laser injection with S, P and circular
polarisation, boundary crossings, particle removal and the electron spin /
g-factor table.  Each fixture stores the input particles, the full state
after step 1 and after the last step, and per-step checksums of every
array.  tests/test_oracle_pin.py replays the same inputs through the C
oracle (oracle/pic_oracle.c) and requires bit-identical results.

Usage (needs the reference build, i.e. the reference tree at build time):
    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

import oracle as O  # noqa: E402
from pic3d_b200.workloads import make_particles, tiny_cases  # noqa: E402

ARRAYS = O.FIELD_NAMES + O.RING_NAMES
PFIELDS = ["x", "y", "z", "x_old", "y_old", "z_old", "px", "py", "pz", "sx", "sy", "sz", "gamma", "weight"]


def golden_cases():
    cases = tiny_cases()
    out = {}
    for name, w in cases.items():
        out[name] = (w.with_(ppc=(1, 1) if name != "periodic_o4" else (1, 0)), None)
    # spin precession with a small Schwinger field so the g-factor table
    # branches of particle.cpp:603-631 are reached
    spin = cases["periodic_o2"].with_(name="spin_o2", ppc=(1, 0), u_th=(0.3, 0.0), E_schwinger=0.5)
    out["spin_o2"] = (spin, "random_spins")
    return out


def checksums(state):
    c = {}
    for n in ARRAYS:
        a = state[n]
        c[n] = [float(a.sum()), float(np.abs(a).sum()), float((a * a).sum())]
    for k in range(2):
        p = state["particles"][k]
        c[f"p{k}"] = [float(len(p))] + [float(p[f].sum()) for f in PFIELDS]
    return c


def pack_state(prefix, state, out):
    for n in ARRAYS:
        out[f"{prefix}_{n}"] = state[n]
    for k in range(2):
        out[f"{prefix}_particles{k}"] = state["particles"][k]


def main():
    if not O.have_reference_build():
        sys.exit("reference build missing: make -C oracle ref")
    for name, (w, extra) in golden_cases().items():
        parts = make_particles(w, seed=20261203)
        if extra == "random_spins":
            rng = np.random.default_rng(99)
            s = rng.normal(size=(len(parts[0]), 3))
            s /= np.linalg.norm(s, axis=1, keepdims=True)
            parts[0]["sx"], parts[0]["sy"], parts[0]["sz"] = s[:, 0], s[:, 1], s[:, 2]
        states, _ = O.run_reference(w, parts, w.steps)
        out = {"input_particles0": parts[0], "input_particles1": parts[1]}
        pack_state("step1", states[1], out)
        pack_state("final", states[-1], out)
        meta = {"case": name, "steps": w.steps, "params": w.params(), "seed": 20261203,
                "checksums": [checksums(s) for s in states],
                "generator": "reference src/{field,particle,boundary,mpi_utils,simulation}.cpp via oracle/_ref"}
        out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
        if extra == "random_spins":
            out["g_data"] = O.load_g_table()
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(name, os.path.getsize(path) // 1024, "KiB", [len(p) for p in parts], "->",
              [len(p) for p in states[-1]["particles"]])


if __name__ == "__main__":
    main()
