"""Device-side particle loaders.

pic_initialize_particles restates the reference's lattice loader
(src/particle.cpp:50-111) with data-described densities; the CPU
restatement below is first pinned record for record to the reference's own
initialize_particles (the call-surface harness oracle/ref/ref_surface.cpp
runs it with the density functions restated here), then the GPU loader is
compared with the restatement.  pic_generate_thermal is compared with a
numpy restatement of its Philox4x32-10 stream."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import oracle as O
from pic3d_b200.workloads import PARTICLE_DTYPE, tiny_cases

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SURFACE_REF = os.path.join(REPO, "oracle", "_ref", "pic3d_surface_ref")


def lattice_ref(w, cpp, density, p0=(0.0, 0.0, 0.0), s0=(0.0, 0.0, 0.0), charge=-1.0, mass=1.0):
    """initialize_particles (src/particle.cpp:50-111), one rank: lattice of
    int(n * cbrt(cpp)) points per axis, weight density(x, y, z) / cpp in
    cell units, points with weight <= 0 skipped."""
    n = (w.nx, w.ny, w.nz)
    num = [int(n[d] * np.cbrt(float(cpp))) for d in range(3)]
    norm = [(float(n[d]) - 0.0) / num[d] for d in range(3)]
    pos = [0.0 + np.arange(num[d], dtype=np.float64) * norm[d] + norm[d] / 2.0 for d in range(3)]
    zz, yy, xx = np.meshgrid(pos[2], pos[1], pos[0], indexing="ij")
    x, y, z = xx.ravel(), yy.ravel(), zz.ravel()
    wt = np.array([density(a, b, c) for a, b, c in zip(x, y, z)], dtype=np.float64) / cpp
    keep = wt > 0.0
    out = np.zeros(int(keep.sum()), dtype=PARTICLE_DTYPE)
    out["id"] = np.arange(len(out))
    out["x"], out["y"], out["z"] = x[keep], y[keep], z[keep]
    out["px"], out["py"], out["pz"] = p0
    out["sx"], out["sy"], out["sz"] = s0
    out["gamma"] = np.sqrt(1 + (p0[0] * p0[0] + p0[1] * p0[1] + p0[2] * p0[2]))
    out["charge"], out["mass"] = charge, mass
    out["weight"] = wt[keep]
    return out


# the density functions of the call-surface harness (oracle/ref/ref_surface.cpp:80-89)
def _density_e(w):
    def f(x, y, z):
        if x > 0.5 * w.nx:
            return w.density_value
        if y < 1.0:
            return 0.0
        return w.density_value * x / (0.5 * w.nx) + 0.0 * z
    return f


def _density_p(w):
    def f(x, y, z):
        inside = x > 0.25 * w.nx and x < 0.75 * w.nx and y > 0.25 * w.ny and z < 0.75 * w.nz
        return 0.5 * w.density_value if inside else 0.0
    return f


def _surface_particles(w):
    with tempfile.TemporaryDirectory(prefix="pic3d_loader_") as tmp:
        prm = os.path.join(tmp, "params.txt")
        O.write_params_file(prm, w, 1, 1)
        out = os.path.join(tmp, "out.bin")
        env = dict(os.environ, PIC3D_REF_PARAMS=prm, PIC3D_G_TXT=O.REF_G_TXT)
        r = subprocess.run([SURFACE_REF, out], env=env, capture_output=True, text=True, cwd=tmp)
        assert r.returncode == 0, r.stderr[-2000:]
        raw = open(out, "rb").read()
    parts, off = [], 0
    for _ in range(2):
        n = int(np.frombuffer(raw, "<i8", 1, off)[0])
        off += 8
        parts.append(np.frombuffer(raw, PARTICLE_DTYPE, n, off).copy())
        off += n * PARTICLE_DTYPE.itemsize
    return parts


SURF = {"periodic_o2_ppc8": lambda c: c["periodic_o2"].with_(ppc=(8, 0)),
        "laser_o4_ppc2": lambda c: c["laser_o4"].with_(ppc=(2, 0))}
COMPARED = ["id", "x", "y", "z", "x_old", "y_old", "z_old", "px", "py", "pz", "sx", "sy", "sz", "gamma", "charge",
            "mass", "weight"]


@pytest.mark.skipif(not os.path.exists(SURFACE_REF), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", list(SURF))
def test_lattice_restatement_matches_reference(name):
    w = SURF[name](tiny_cases())
    ref = _surface_particles(w)
    # ref_surface.cpp:150-151: electrons with momentum (0.01, -0.02, 0.03), protons at rest
    mine = [lattice_ref(w, w.ppc[0], _density_e(w), (0.01, -0.02, 0.03), charge=-1.0, mass=1.0),
            lattice_ref(w, w.ppc[0], _density_p(w), charge=1.0, mass=1836.0)]
    for k in range(2):
        assert len(mine[k]) == len(ref[k]) > 0
        for f in COMPARED:
            assert np.array_equal(mine[k][f], ref[k][f]), (k, f)


def _box(w, lo, hi, value):
    h = (w.dx, w.dy, w.dz)

    def f(x, y, z):
        c = (x, y, z)
        return value if all(lo[d] < c[d] * h[d] <= hi[d] for d in range(3)) else 0.0
    return f


def _xprofile(w, kx, kv):
    def f(x, y, z):
        xp = x * w.dx
        if xp <= kx[0]:
            return kv[0]
        if xp >= kx[-1]:
            return kv[-1]
        k = 1
        while kx[k] < xp:
            k += 1
        return kv[k - 1] + (kv[k] - kv[k - 1]) * ((xp - kx[k - 1]) / (kx[k] - kx[k - 1]))
    return f


LOADER_CASES = {
    # the reference's own plasma_density shape (src/constants.cpp:87-101), scaled into the box
    "box": dict(wl="laser_o4", cpp=8, density="box", value=0.05, lo=(1.0, 0.5, 0.0), hi=(3.0, 3.5, 2.5)),
    "uniform": dict(wl="periodic_o4", cpp=27, density="uniform", value=1.0),
    "xprofile": dict(wl="laser_o4", cpp=8, density="xprofile",
                     knots=(np.array([0.3, 1.0, 2.5, 4.0]), np.array([0.0, 0.02, 0.05, 0.01]))),
}


def _loader_ref(w, case, p0, s0):
    if case["density"] == "box":
        f = _box(w, case["lo"], case["hi"], case["value"])
    elif case["density"] == "uniform":
        f = lambda x, y, z: case["value"]  # noqa: E731
    else:
        f = _xprofile(w, list(case["knots"][0]), list(case["knots"][1]))
    return lattice_ref(w, case["cpp"], f, p0, s0, charge=-1.0, mass=1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", list(LOADER_CASES))
def test_gpu_lattice_loader(name, precision):
    from pic3d_b200.simulation import Simulation
    case = LOADER_CASES[name]
    w = tiny_cases()[case["wl"]]
    p0, s0 = (0.01, -0.02, 0.03), (0.0, 0.5, 0.0)
    ref = _loader_ref(w, case, p0, s0)
    assert len(ref) > 0
    with Simulation(w, precision=precision) as sim:
        kw = {k: v for k, v in case.items() if k in ("value", "lo", "hi", "knots")}
        sim.initialize_particles(0, case["cpp"], density=case["density"], initial_p=p0, initial_s=s0, **kw)
        got = sim.download_particles(0)
    assert len(got) == len(ref)
    if precision == "fp64":
        for f in COMPARED:
            assert np.array_equal(got[f], ref[f]), f
    else:
        assert np.array_equal(got["id"], ref["id"])
        for f in ("x", "y", "z"):
            np.testing.assert_allclose(got[f], ref[f], rtol=0, atol=2e-6 * max(w.nx, w.ny, w.nz))
        for f in ("px", "py", "pz", "sx", "sy", "sz", "weight"):
            np.testing.assert_allclose(got[f], ref[f], rtol=1e-7, atol=0)


# ---------------------------------------------------------------------------
# thermal generator

def _philox(counter, key):
    """Philox4x32-10 on uint64 arrays holding 32-bit lanes."""
    M0, M1, W0, W1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57), 0x9E3779B9, 0xBB67AE85
    mask = np.uint64(0xFFFFFFFF)
    c = [np.asarray(x, dtype=np.uint64) & mask for x in counter]
    k0, k1 = key
    for _ in range(10):
        p0, p1 = M0 * c[0], M1 * c[2]
        hi0, lo0, hi1, lo1 = p0 >> np.uint64(32), p0 & mask, p1 >> np.uint64(32), p1 & mask
        c = [hi1 ^ c[1] ^ np.uint64(k0), lo1, hi0 ^ c[3] ^ np.uint64(k1), lo0]
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return c


def thermal_ref(w, kind, ppc, density, u_th, seed, charge, mass):
    n = w.nx * w.ny * w.nz * ppc
    q = np.arange(n, dtype=np.uint64)
    key = (seed & 0xFFFFFFFF, ((seed >> 32) ^ ((0x9E3779B9 * (kind + 1)) & 0xFFFFFFFF)) & 0xFFFFFFFF)
    zero = np.zeros(n, dtype=np.uint64)
    u = _philox([q & np.uint64(0xFFFFFFFF), q >> np.uint64(32), zero, zero], key)
    u += _philox([q & np.uint64(0xFFFFFFFF), q >> np.uint64(32), zero + np.uint64(1), zero], key)
    u = [x.astype(np.float64) for x in u]
    inv = 2.0 ** -32
    cell = np.arange(n) // ppc
    out = np.zeros(n, dtype=PARTICLE_DTYPE)
    out["id"] = np.arange(n)
    out["x"] = (cell % w.nx) + u[0] * inv
    out["y"] = ((cell // w.nx) % w.ny) + u[1] * inv
    out["z"] = (cell // (w.nx * w.ny)) + u[2] * inv
    r0 = np.sqrt(-2.0 * np.log((u[3] + 1.0) * inv))
    r1 = np.sqrt(-2.0 * np.log((u[5] + 1.0) * inv))
    t0, t1 = 2 * np.pi * u[4] * inv, 2 * np.pi * u[6] * inv
    out["px"], out["py"], out["pz"] = u_th * r0 * np.cos(t0), u_th * r0 * np.sin(t0), u_th * r1 * np.cos(t1)
    out["gamma"] = np.sqrt(1.0 + (out["px"] ** 2 + out["py"] ** 2 + out["pz"] ** 2))
    out["charge"], out["mass"], out["weight"] = charge, mass, density / ppc
    return out


def test_philox_restatement_statistics():
    """The restated stream: uniform offsets and unit normals."""
    w = tiny_cases()["periodic_o2"]
    p = thermal_ref(w, 0, 64, 1.0, 1.0, 12345, -1.0, 1.0)
    off = p["x"] - np.floor(p["x"])
    assert abs(off.mean() - 0.5) < 0.01 and abs(off.var() - 1 / 12) < 0.005
    for f in ("px", "py", "pz"):
        assert abs(p[f].mean()) < 0.03 and abs(p[f].std() - 1.0) < 0.03
    # each cell holds its ppc particles
    cells = np.floor(p["x"]) + w.nx * (np.floor(p["y"]) + w.ny * np.floor(p["z"]))
    assert np.array_equal(np.bincount(cells.astype(np.int64)), np.full(w.nx * w.ny * w.nz, 64))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gpu_thermal_generator(precision):
    from pic3d_b200.simulation import Simulation
    w = tiny_cases()["periodic_o4"]
    ref = [thermal_ref(w, k, 4, 1.0, 0.05, 2024, q, m) for k, q, m in ((0, -1.0, 1.0), (1, 1.0, 1836.0))]
    got = []
    for rep in range(2):   # same seed, same particles
        with Simulation(w, precision=precision) as sim:
            for k in range(2):
                sim.generate_thermal(k, 4, 1.0, 0.05, 2024)
            got.append([sim.download_particles(k) for k in range(2)])
    for k in range(2):
        a, b = got[0][k], got[1][k]
        for f in PARTICLE_DTYPE.names:
            assert np.array_equal(a[f], b[f]), f
        r = ref[k]
        assert np.array_equal(a["id"], r["id"])
        if precision == "fp64":
            for f in ("x", "y", "z"):
                assert np.array_equal(a[f], r[f]), f
            np.testing.assert_allclose(np.stack([a["px"], a["py"], a["pz"]]),
                                       np.stack([r["px"], r["py"], r["pz"]]), rtol=1e-12, atol=1e-15)
        else:
            for f in ("x", "y", "z"):
                np.testing.assert_allclose(a[f], r[f], rtol=0, atol=1e-6 * w.nx)
            np.testing.assert_allclose(np.stack([a["px"], a["py"], a["pz"]]),
                                       np.stack([r["px"], r["py"], r["pz"]]), rtol=1e-6, atol=1e-9)
        np.testing.assert_array_equal(a["weight"], r["weight"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gpu_upload_download_round_trip_over_chunks(precision):
    """More records than one pinned staging buffer (262,144): download,
    upload back, download again gives the same records."""
    from pic3d_b200.simulation import Simulation
    w = tiny_cases()["periodic_o4"].with_(nx=48, ny=40, nz=36)
    with Simulation(w, precision=precision) as sim:
        sim.generate_thermal(0, 4, 1.0, 0.05, 77)    # 276,480 particles
        a = sim.download_particles(0)
        assert len(a) == 48 * 40 * 36 * 4
        sim.upload_particles(0, a)
        b = sim.download_particles(0)
    for f in PARTICLE_DTYPE.names:
        assert np.array_equal(a[f], b[f]), f


@pytest.mark.gpu
def test_gpu_upload_rejects_bad_records():
    from pic3d_b200 import _lib as L
    from pic3d_b200.simulation import Simulation
    w = tiny_cases()["periodic_o2"]
    good = lattice_ref(w, 8, lambda x, y, z: 1.0, charge=-1.0, mass=1.0)
    with Simulation(w, precision="fp64") as sim:
        for field, value in (("charge", 1.0), ("weight", np.nan), ("mass", 2.0)):
            bad = good.copy()
            bad[field][len(bad) // 2] = value
            with pytest.raises(L.PicError) as e:
                sim.upload_particles(0, bad)
            assert e.value.code == L.PIC_EINVAL
            assert sim.num_particles(0) == 0
        sim.upload_particles(0, good)
        got = sim.download_particles(0)
    assert len(got) == len(good)
    for f in ("id", "x", "y", "z", "px", "weight", "charge", "mass"):
        assert np.array_equal(np.sort(got[f]), np.sort(good[f])), f
