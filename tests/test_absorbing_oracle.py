"""The absorbing-faces extension in the oracle's CPU restatement (no GPU).

A random, smoothed field in a box that absorbs on every side must lose
energy, step after step; the same box with the reference's faces
(conductors on y and z) keeps it.  This is the check that caught the two
unstable forms of the condition (applied after each half-step B update, and
with the x-min formula's tangential-derivative term relabelled onto the
other faces): both grew without bound on this field.
"""
import numpy as np

import oracle as O

from pic3d_b200 import workloads as W


def _field_energy_history(absorbing, steps=240, n=16, mem=2, d=(1.0, 1.0, 1.0)):
    w = W.Workload(name="box", nx=n, ny=n, nz=n, mem=mem, period=(0, 0, 0), ppc=(0, 0), u_th=(0.0, 0.0),
                   dx=d[0], dy=d[1], dz=d[2], laser_amplitude=0.0, absorbing=absorbing, steps=steps)
    o = O.Oracle(w, [np.zeros(0, W.PARTICLE_DTYPE)] * 2)
    rng = np.random.default_rng(7)
    m = mem
    for f in ("ex", "ey", "ez", "bx", "by", "bz"):
        a = np.zeros_like(o.arrays[f])
        a[m:-m, m:-m, m:-m] = rng.normal(size=tuple(s - 2 * m for s in a.shape))
        for ax in range(3):
            a = 0.25 * np.roll(a, 1, ax) + 0.5 * a + 0.25 * np.roll(a, -1, ax)
        o.arrays[f][...] = a
    energy = lambda: sum(float(np.sum(o.arrays[f][m:-m, m:-m, m:-m] ** 2)) for f in ("ex", "ey", "ez", "bx", "by", "bz"))
    o.initial()
    e0, out = energy(), []
    for s in range(1, steps + 1):
        o.step(s)
        if s % 40 == 0:
            out.append(energy() / e0)
    return out


def test_random_field_decays_in_an_absorbing_box():
    for mem, d in ((2, (1.0, 1.0, 1.0)), (4, (0.314, 0.628, 0.628))):
        hist = _field_energy_history(1, mem=mem, d=d)
        assert max(hist) < 1.0, (mem, hist)
        assert hist[-1] < 0.6, (mem, hist)
