"""The hand-written adjoint against central finite differences.

A small laser run (absorbing faces, electrons with a small thermal spread,
laser amplitude from a 4x4 B-spline coefficient grid) is differentiated with
respect to the density knots and the laser coefficients; the objective is
the electrons' kinetic energy in a window at the final step.  Finite
differences use the FP64 forward run.
"""
import numpy as np
import pytest

from pic3d_b200.workloads import LAMBDA, Workload

pytestmark = pytest.mark.gpu


def small_spec(precision="fp64", mem=2, segment=5, steps=16, u_th=0.02):
    from pic3d_b200.adjoint import AdjointSpec
    w = Workload(name="adj_small", nx=24, ny=12, nz=12, mem=mem, period=(0, 0, 0), dx=LAMBDA / 16, dy=LAMBDA / 8,
                 dz=LAMBDA / 8, ppc=(2, 0), u_th=(u_th, 0.0), laser_amplitude=1.0, laser_pulse_duration=4.0,
                 waist=LAMBDA, laser_polarization=3, steps=steps)
    return AdjointSpec(workload=w, n_knots=6, profile_n=4, window=(2.0, 20.0), segment=segment, seed=77,
                       precision=precision)


def params(spec):
    rng = np.random.default_rng(5)
    knots = 0.05 + 0.05 * rng.random(spec.n_knots)
    prof = 1.0 + 0.5 * rng.random((spec.profile_n, spec.profile_n))
    return knots, prof


def fd(spec, knots, prof, which, idx, h):
    from pic3d_b200.adjoint import objective
    k1, p1 = knots.copy(), prof.copy().ravel()
    k2, p2 = knots.copy(), prof.copy().ravel()
    if which == "knot":
        k1[idx] += h
        k2[idx] -= h
    else:
        p1[idx] += h
        p2[idx] -= h
    return (objective(spec, k1, p1) - objective(spec, k2, p2)) / (2 * h)


@pytest.mark.parametrize("mem", [2, 4])
def test_adjoint_matches_finite_differences(mem):
    from pic3d_b200.adjoint import objective_and_grad
    spec = small_spec("fp64", mem=mem)
    knots, prof = params(spec)
    loss, gk, gp, _ = objective_and_grad(spec, knots, prof)
    assert loss > 0
    assert np.abs(gp).max() > 0, "laser coefficients must influence the objective"
    scale_k = np.abs(gk).max()
    for i in range(spec.n_knots):
        f = fd(spec, knots, prof, "knot", i, 1e-5)
        assert abs(gk[i] - f) <= 1e-4 * max(abs(f), 1e-3 * scale_k), (i, gk[i], f)
    scale_p = np.abs(gp).max()
    for i in [0, 5, 6, 9, 10, 15]:
        f = fd(spec, knots, prof, "prof", i, 1e-4)
        assert abs(gp[i] - f) <= 1e-4 * max(abs(f), 1e-2 * scale_p), (i, gp[i], f)


def test_adjoint_with_particles_leaving_the_box():
    """Hot electrons: many leave through the absorbing faces during the run
    (removed particles drop out of the objective and of later steps)."""
    from pic3d_b200.adjoint import objective_and_grad
    from pic3d_b200.simulation import Simulation
    from pic3d_b200.workloads import PARTICLE_DTYPE
    spec = small_spec("fp64", u_th=0.4, steps=20)
    knots, prof = params(spec)
    recs = spec.base_particles()
    recs["weight"] = spec.weights(recs["x"], knots)
    with Simulation(spec.workload, precision="fp64") as sim:   # compacting run: count the survivors
        sim.upload_particles(0, recs)
        sim.upload_particles(1, np.zeros(0, PARTICLE_DTYPE))
        sim.initial_push()
        sim.run_main_time_loop(spec.workload.steps)
        left = len(recs) - sim.num_particles(0)
    assert left > len(recs) // 20, left
    _, gk, gp, _ = objective_and_grad(spec, knots, prof)
    for i in range(spec.n_knots):
        f = fd(spec, knots, prof, "knot", i, 1e-6)
        assert abs(gk[i] - f) <= 1e-4 * max(abs(f), 1e-3 * np.abs(gk).max()), (i, gk[i], f)
    for i in [5, 6]:
        f = fd(spec, knots, prof, "prof", i, 1e-5)
        assert abs(gp[i] - f) <= 1e-4 * max(abs(f), 1e-2 * np.abs(gp).max()), (i, gp[i], f)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_smooth_window_seeds_positions(precision):
    """With ramps the objective depends on the final positions: the position
    adjoint seeded by the window's slope must match finite differences."""
    import dataclasses

    from pic3d_b200.adjoint import objective_and_grad
    spec = dataclasses.replace(small_spec("fp64", mem=4), window=(4.0, 20.0), ramp=5.0)
    knots, prof = params(spec)
    _, gk, gp, _ = objective_and_grad(spec, knots, prof)
    hard = objective_and_grad(dataclasses.replace(spec, ramp=0.0), knots, prof)
    assert np.linalg.norm(gk - hard[1]) > 1e-3 * np.linalg.norm(gk), "the ramps must change the gradient"
    for i in range(spec.n_knots):
        f = fd(spec, knots, prof, "knot", i, 1e-5)
        assert abs(gk[i] - f) <= 1e-4 * max(abs(f), 1e-3 * np.abs(gk).max()), (i, gk[i], f)
    for i in [5, 10]:
        f = fd(spec, knots, prof, "prof", i, 1e-4)
        assert abs(gp[i] - f) <= 1e-4 * max(abs(f), 1e-2 * np.abs(gp).max()), (i, gp[i], f)
    if precision == "fp32":
        s32 = dataclasses.replace(spec, precision="fp32")
        _, k32, p32, _ = objective_and_grad(s32, knots, prof)
        assert np.linalg.norm(k32 - gk) <= 1e-4 * np.linalg.norm(gk)
        assert np.linalg.norm(p32 - gp) <= 1e-3 * np.linalg.norm(gp)


def test_segments_do_not_change_the_gradient():
    from pic3d_b200.adjoint import objective_and_grad
    knots, prof = params(small_spec())
    a = objective_and_grad(small_spec(segment=3), knots, prof)
    b = objective_and_grad(small_spec(segment=100), knots, prof)
    assert a[0] == pytest.approx(b[0], rel=1e-12)
    np.testing.assert_allclose(a[1], b[1], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(a[2], b[2], rtol=1e-9, atol=1e-14)


def test_fp32_adjoint_matches_fp64():
    from pic3d_b200.adjoint import objective_and_grad
    knots, prof = params(small_spec())
    l64, k64, p64, _ = objective_and_grad(small_spec("fp64"), knots, prof)
    l32, k32, p32, _ = objective_and_grad(small_spec("fp32"), knots, prof)
    assert l32 == pytest.approx(l64, rel=1e-5)
    assert np.linalg.norm(k32 - k64) <= 1e-4 * np.linalg.norm(k64)
    assert np.linalg.norm(p32 - p64) <= 1e-3 * np.linalg.norm(p64)


def test_autograd_function():
    import torch

    from pic3d_b200.adjoint import PICObjective, objective_and_grad
    spec = small_spec()
    knots, prof = params(spec)
    kt = torch.tensor(knots, requires_grad=True)
    pt = torch.tensor(prof.ravel(), requires_grad=True)
    loss = PICObjective.apply(kt, pt, spec)
    (2.0 * loss).backward()
    _, gk, gp, _ = objective_and_grad(spec, knots, prof)
    np.testing.assert_allclose(kt.grad.numpy(), 2.0 * gk, rtol=1e-9)
    np.testing.assert_allclose(pt.grad.numpy(), 2.0 * gp, rtol=1e-9)


def test_differentiable_run_gradient_matches_fd_on_8_parameters():
    """The differentiable-run configuration (64x64x128, 8 electrons per cell,
    32 density knots, 8x8 laser coefficients, 600 steps, checkpoints every
    50): the FP64 adjoint gradient against central differences of the FP64
    objective on the 4 knots and the 4 laser coefficients with the largest
    derivatives.  The objective is piecewise smooth (electrons removed at the
    absorbing faces are jumps), so the difference quotient converges only
    once the step is too small to move a removal to another step; the check
    takes the best of three relative steps and requires 1e-4."""
    from pic3d_b200 import workloads as W
    from pic3d_b200.adjoint import AdjointSpec, objective, objective_and_grad
    w = W.differentiable_laser(precision="fp64", steps=600)
    spec = AdjointSpec(workload=w, n_knots=32, profile_n=8, window=(0.5 * w.nx, w.nx - 4.0), ramp=4.0,
                       segment=50, seed=2468, precision="fp64")
    rng = np.random.default_rng(13)
    knots = 0.01 + 0.02 * rng.random(32)
    prof = 1.0 + 0.2 * rng.random((8, 8))
    _, gk, gp, _ = objective_and_grad(spec, knots, prof)
    checks = [("knot", int(i)) for i in np.argsort(-np.abs(gk))[:4]] + \
             [("prof", int(i)) for i in np.argsort(-np.abs(gp))[:4]]
    for which, i in checks:
        g = gk[i] if which == "knot" else gp[i]
        base = knots[i] if which == "knot" else prof.ravel()[i]
        errs = []
        for rel_h in (1e-7, 1e-8, 1e-9):
            h = rel_h * abs(base)
            k1, k2, p1, p2 = knots.copy(), knots.copy(), prof.ravel().copy(), prof.ravel().copy()
            if which == "knot":
                k1[i] += h
                k2[i] -= h
            else:
                p1[i] += h
                p2[i] -= h
            f = (objective(spec, k1, p1) - objective(spec, k2, p2)) / (2 * h)
            errs.append(abs(g - f) / max(abs(f), 1e-300))
        assert min(errs) <= 1e-4, (which, i, g, errs)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tiled_and_global_adjoint_agree(precision):
    """The adjoint-capable context sorts particles by tile like the ordinary
    one (the tape keeps every sort's permutation and tile boundaries; the
    reverse sweep runs per tile in shared memory).  Its gradient equals the
    one of the unsorted global-memory kernels up to rounding."""
    import dataclasses

    from pic3d_b200.adjoint import objective_and_grad
    spec = dataclasses.replace(small_spec(precision, mem=4, steps=20, segment=7), window=(4.0, 20.0), ramp=4.0)
    knots, prof = params(spec)
    lt, kt, pt, wt = objective_and_grad(spec, knots, prof)
    lg, kg, pg, wg = objective_and_grad(dataclasses.replace(spec, tile=-1), knots, prof)
    tol = 1e-9 if precision == "fp64" else 2e-4
    assert lt == pytest.approx(lg, rel=1e-12 if precision == "fp64" else 1e-6)
    assert np.linalg.norm(kt - kg) <= tol * np.linalg.norm(kg)
    assert np.linalg.norm(pt - pg) <= tol * np.linalg.norm(pg)
    assert np.linalg.norm(wt - wg) <= tol * np.linalg.norm(wg)
