"""Initial-field Poisson solve (pic_solve_initial_field) against the CPU
FP64 restatement in poisson_ref.py: node charge density, direct solve of the
Yee-grid Laplacian, E on the faces.  The restatement is first checked on the
CPU (FFT eigen-solution for an all-periodic grid, discrete Gauss law)."""
import numpy as np
import pytest

import poisson_ref as R
from pic3d_b200.workloads import make_particles, tiny_cases

CASES = ["periodic_o2", "periodic_o4", "laser_o4", "mixed_o2"]


def _case(name, seed=7):
    w = tiny_cases()[name]
    return w, make_particles(w, seed=seed)


def _fft_phi(w, b):
    """Periodic solution of A phi = b from the eigenvalues of the 7-point
    Laplacian, 4 sin^2(pi k / n) / h^2 per axis."""
    kz, ky, kx = [np.arange(n) for n in b.shape]
    lz = 4 * np.sin(np.pi * kz / b.shape[0]) ** 2 / w.dz ** 2
    ly = 4 * np.sin(np.pi * ky / b.shape[1]) ** 2 / w.dy ** 2
    lx = 4 * np.sin(np.pi * kx / b.shape[2]) ** 2 / w.dx ** 2
    lam = lz[:, None, None] + ly[None, :, None] + lx[None, None, :]
    bh = np.fft.fftn(b)
    lam[0, 0, 0] = 1.0
    ph = bh / lam
    ph[0, 0, 0] = 0.0
    return np.real(np.fft.ifftn(ph))


@pytest.mark.parametrize("name", ["periodic_o2", "periodic_o4"])
def test_restatement_matches_fft(name):
    w, parts = _case(name)
    rho = R.node_rho(w, parts)
    phi, mean = R.solve_phi(w, rho)
    ref = _fft_phi(w, rho - mean)
    assert np.linalg.norm(phi - ref) <= 1e-10 * np.linalg.norm(ref)


@pytest.mark.parametrize("name", CASES)
def test_restatement_gauss_law(name):
    w, parts = _case(name)
    rho = R.node_rho(w, parts)
    # total charge on the nodes equals the particles' charge where nothing
    # falls outside (all-periodic grids)
    if all(w.period):
        tot = sum(w.species(k)["charge"] * parts[k]["weight"].sum() for k in range(2))
        assert abs(rho.sum() - tot) <= 1e-12 * max(1.0, abs(tot)) * rho.size
    phi, mean = R.solve_phi(w, rho)
    f = R.fields_from_phi(w, phi)
    div = R.divergence(w, f)
    assert np.max(np.abs(div - (rho - mean))) <= 1e-9 * np.max(np.abs(rho))


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gpu_solve_matches_restatement(name, precision):
    from pic3d_b200.simulation import Simulation
    w, parts = _case(name)
    rho = R.node_rho(w, parts)
    phi, mean = R.solve_phi(w, rho)
    ref = R.fields_from_phi(w, phi)
    with Simulation(w, precision=precision) as sim:
        for k in range(2):
            sim.upload_particles(k, parts[k])
        bx = np.full(sim.download_array("bx").shape, 0.25)
        sim.upload_array("bx", bx)
        res = sim.solve_initial_field(rel_tol=1e-11)
        got = {n: sim.download_array(n) for n in ("ex", "ey", "ez")}
        assert np.array_equal(sim.download_array("bx"), bx if precision == "fp64" else bx.astype(np.float32))
    tol = 1e-9 if precision == "fp64" else 1e-6
    for n in ("ex", "ey", "ez"):
        assert _rel(got[n], ref[n]) <= tol, (n, _rel(got[n], ref[n]))
    assert res["rel_residual"] <= 1e-11
    # FP32 contexts hold positions and weights in FP32: rho itself differs at that level
    mtol = 1e-12 if precision == "fp64" else 1e-6
    assert abs(res["mean_rho"] - mean) <= mtol * np.max(np.abs(rho))
    # Gauss law from the stored E (FP32: E rounded to float)
    gtol = 1e-9 if precision == "fp64" else 1e-4
    assert res["gauss_max"] <= gtol * np.max(np.abs(rho)), res
    div = R.divergence(w, got)
    assert np.max(np.abs(div - (rho - mean))) <= gtol * np.max(np.abs(rho))


@pytest.mark.gpu
def test_gpu_solve_reports_no_convergence():
    from pic3d_b200 import _lib as L
    from pic3d_b200.simulation import Simulation
    w, parts = _case("laser_o4")
    with Simulation(w, precision="fp64") as sim:
        for k in range(2):
            sim.upload_particles(k, parts[k])
        with pytest.raises(L.PicError) as e:
            sim.solve_initial_field(rel_tol=1e-14, max_iter=2)
        assert e.value.code == L.PIC_ENOCONV
