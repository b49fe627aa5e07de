"""Gradients of a final-state objective through the PIC loop.

The objective is the kinetic energy sum s(x) w m (gamma - 1) of the
electrons at the final step, s a window along x (1 inside, 0 outside, with
sin^2 ramps `ramp` cells wide at its edges so that the objective is smooth
in the particle positions).  The parameters are
  * K density knots: the initial density is the piecewise-linear
    interpolation of the knot values along x, and each particle's weight is
    density(x0) / (particles per cell) at its initial position;
  * an n x n grid of cubic-B-spline coefficients of the laser's transverse
    amplitude (laser_profile = 1).
The gradient comes from the hand-written adjoint kernels behind the C ABI
(pic_adjoint_*): the forward run keeps a device checkpoint every `segment`
steps and records the inputs of every push of its last segment; the backward
run sweeps that segment in reverse, then restores each earlier checkpoint,
recomputes its segment while recording, and sweeps it.  With `segment` at
least the number of steps nothing is recomputed (the record of a step holds
the fields and the particle inputs: about 150 MB per step for 4.2 M FP32
particles on 64x64x128 cells, so 600 steps fit in HBM).  `PICObjective`
wraps this as a torch.autograd.Function.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib as L
from .simulation import Simulation
from .workloads import PARTICLE_DTYPE, Workload


def hat_weights(x, n_cells: int, n_knots: int):
    """Piecewise-linear interpolation weights of n_knots knots spread
    uniformly over [0, n_cells] (cell units): returns (index, frac) such that
    density(x) = (1-frac) * knot[index] + frac * knot[index+1]."""
    t = np.clip(np.asarray(x, dtype=np.float64) / n_cells * (n_knots - 1), 0.0, n_knots - 1 - 1e-12)
    i = np.floor(t).astype(np.int64)
    return i, t - i


@dataclasses.dataclass
class AdjointSpec:
    workload: Workload
    n_knots: int = 32
    profile_n: int = 8
    window: tuple = (0.0, 0.0)        # x range of the objective, in cells
    ramp: float = 0.0                 # width of the window's edge ramps, in cells
    segment: int = 50
    seed: int = 4321
    precision: str = "fp32"
    tile: int = 0                     # particle tile edge (0 default; -1 global-memory kernels, unsorted)

    def base_particles(self):
        """Electron positions and momenta (weights set from the knots)."""
        from .workloads import make_particles
        w = self.workload.with_(density=None, density_value=1.0)
        parts = make_particles(w, seed=self.seed, kinds=(0,))
        return parts[0]

    def weights(self, x0, knots):
        i, f = hat_weights(x0, self.workload.nx, self.n_knots)
        knots = np.asarray(knots, dtype=np.float64)
        return ((1.0 - f) * knots[i] + f * knots[i + 1]) / self.workload.ppc[0]

    def knot_grad(self, x0, grad_w):
        i, f = hat_weights(x0, self.workload.nx, self.n_knots)
        g = np.zeros(self.n_knots)
        gw = np.asarray(grad_w, dtype=np.float64) / self.workload.ppc[0]
        np.add.at(g, i, (1.0 - f) * gw)
        np.add.at(g, i + 1, f * gw)
        return g


class AdjointRun:
    """One forward run with checkpoints and its backward run."""

    def __init__(self, spec: AdjointSpec, knots, profile, device: int = 0):
        self.spec = spec
        self.sim = Simulation(spec.workload, precision=spec.precision, device=device, adjoint=True, tile=spec.tile,
                              laser_profile=np.asarray(profile, dtype=np.float64).reshape(spec.profile_n,
                                                                                           spec.profile_n))
        rec = spec.base_particles()
        self.x0 = rec["x"].copy()
        rec["weight"] = spec.weights(self.x0, knots)
        self.records = rec
        self.sim.upload_particles(0, rec)
        self.sim.upload_particles(1, np.zeros(0, PARTICLE_DTYPE))
        self.lib = self.sim.lib
        self.ctx = self.sim.ctx
        self.steps = spec.workload.steps
        self.bounds = []   # (checkpoint slot, first step, number of loop steps, includes the t=0 push)
        self.taped_last = False   # the forward recorded its last segment

    def _ck(self, code):
        self.sim._check(code)

    def _record(self, on: bool, nrec: int = 0):
        if on:
            self._ck(self.lib.pic_adjoint_tape(self.ctx, nrec))
        self._ck(self.lib.pic_adjoint_record(self.ctx, 1 if on else 0))

    def forward(self) -> float:
        seg = max(int(self.spec.segment), 1)
        self._ck(self.lib.pic_checkpoint_save(self.ctx, 0))
        single = self.steps <= seg
        if single:   # one segment: record from the t=0 push on
            self._record(True, self.steps + 1)
        self.sim.initial_push()
        done, slot = 0, 0
        while done < self.steps:
            n = min(seg, self.steps - done)
            last = done + n == self.steps
            if done > 0:
                slot += 1
                self._ck(self.lib.pic_checkpoint_save(self.ctx, slot))
                if last:
                    self._record(True, n)
            self.bounds.append((slot, done, n, done == 0))
            self.sim.run_main_time_loop(n)
            done += n
        if self.steps == 0:
            self.bounds.append((0, 0, 0, True))
        self._record(False)
        self.taped_last = True
        loss = ctypes.c_double()
        self._ck(self.lib.pic_adjoint_seed_kinetic(self.ctx, 0, float(self.spec.window[0]),
                                                   float(self.spec.window[1]), float(self.spec.ramp),
                                                   ctypes.byref(loss)))
        return loss.value

    def backward(self):
        for j, (slot, first, n, with_t0) in enumerate(reversed(self.bounds)):
            nrec = n + (1 if with_t0 else 0)
            if not (j == 0 and self.taped_last):
                self._ck(self.lib.pic_checkpoint_restore(self.ctx, slot))
                self._record(True, nrec)
                if with_t0:
                    self.sim.initial_push()
                if n:
                    self.sim.run_main_time_loop(n)
                self._record(False)
            self._ck(self.lib.pic_adjoint_backward(self.ctx, nrec))
        gw = np.zeros(len(self.records))
        self._ck(self.lib.pic_adjoint_weight_grad(self.ctx, 0, gw.ctypes.data, len(gw)))
        m = self.spec.profile_n ** 2
        gp = np.zeros(m)
        self._ck(self.lib.pic_adjoint_profile_grad(self.ctx, gp.ctypes.data, m))
        return gw, gp

    def close(self):
        self.sim.close()


def objective_and_grad(spec: AdjointSpec, knots, profile, device: int = 0):
    """(objective, d/d knots, d/d profile coefficients, d/d weights)."""
    run = AdjointRun(spec, knots, profile, device)
    try:
        loss = run.forward()
        gw, gp = run.backward()
        return loss, spec.knot_grad(run.x0, gw), gp, gw
    finally:
        run.close()


def objective(spec: AdjointSpec, knots, profile, device: int = 0) -> float:
    run = AdjointRun(spec, knots, profile, device)
    try:
        return run.forward()
    finally:
        run.close()


def _autograd_function():
    import torch

    class PICObjective(torch.autograd.Function):
        """objective(knots, profile) with the adjoint as its backward."""

        @staticmethod
        def forward(ctx, knots, profile, spec):
            run = AdjointRun(spec, knots.detach().cpu().numpy(), profile.detach().cpu().numpy(),
                             device=knots.device.index or 0 if knots.is_cuda else 0)
            loss = run.forward()
            ctx.run = run
            ctx.spec = spec
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            run = ctx.run
            try:
                gw, gp = run.backward()
                gk = ctx.spec.knot_grad(run.x0, gw)
            finally:
                run.close()
            s = float(g)
            return (torch.as_tensor(gk * s, dtype=torch.float64), torch.as_tensor(gp * s, dtype=torch.float64),
                    None)

    return PICObjective


def __getattr__(name):
    if name == "PICObjective":
        return _autograd_function()
    raise AttributeError(name)
