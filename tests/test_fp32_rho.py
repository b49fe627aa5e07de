"""FP32 rho, point by point, where the density is low.

The tile kernel accumulates rho in fixed point scaled to the largest
possible contribution of any particle (the largest |q w| times the largest
shape weight cubed).  Where weights vary widely (a density ramp), small
contributions sit far below that bound, so a coarse fixed-point step shows
up as a relative error in the low-density cells that a relative L2 over the
whole array hides.  This test compares FP32 rho with the FP64 oracle at
every point holding at least 1e-3 of the largest |rho|, one teacher-forced
step of the laser golden case (a density ramp from zero).
"""
import numpy as np
import pytest

import oracle as O
from golden_io import load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", [dict(tile=0), dict(tile=-1)])
def test_fp32_rho_pointwise_in_a_density_ramp(path):
    from pic3d_b200.simulation import Simulation
    g = load("laser_o4")
    states, _ = O.run_oracle(g["params"], g["input"], 3)
    sim = Simulation(g["params"], precision="fp32", **path)
    worst = 0.0
    for n in range(3):
        sim.upload_state(states[n])
        sim.step = n
        sim.run_main_time_loop(1)
        for name in ("rho0", "rho1"):
            got = sim.download_array(name)
            ref = states[n + 1][name]
            big = np.abs(ref) >= 1e-3 * np.abs(ref).max()
            rel = np.abs(got[big] - ref[big]) / np.abs(ref[big])
            worst = max(worst, float(rel.max()))
    sim.close()
    assert worst <= 1e-5, worst
