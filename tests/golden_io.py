"""Reading the golden fixtures written by tests/golden/make_golden.py."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ARRAYS = ["ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "rho0", "rho1"]
CASES = ["periodic_o2", "periodic_o4", "laser_o4", "mixed_o2", "spin_o2"]


def load(case):
    z = np.load(os.path.join(GOLDEN, f"{case}.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    g = {"meta": meta, "params": meta["params"], "steps": meta["steps"],
         "input": [z["input_particles0"], z["input_particles1"]],
         "g_data": z["g_data"] if "g_data" in z.files else None}
    for tag in ("step1", "final"):
        st = {n: z[f"{tag}_{n}"] for n in ARRAYS}
        st["particles"] = [z[f"{tag}_particles0"], z[f"{tag}_particles1"]]
        g[tag] = st
    return g
