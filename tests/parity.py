"""Comparison helpers shared by the parity tests."""
import numpy as np

ARRAYS = ["ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "rho0", "rho1"]

# per-step tolerances (relative L2 against the FP64 oracle)
TOL_FP64 = 1e-10
TOL_FP32 = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    nd = np.linalg.norm(a - b)
    if nb == 0.0:
        return 0.0 if nd == 0.0 else float("inf")
    return float(nd / nb)


def array_errors(got: dict, ref: dict, names=ARRAYS):
    return {n: rel_l2(got[n], ref[n]) for n in names}


def by_id(p):
    return p[np.argsort(p["id"], kind="stable")]


def particle_errors(got, ref, period=None):
    """Max abs position error (cells, modulo the period on periodic axes) and
    relative L2 momentum error between two record arrays matched by id."""
    a, b = by_id(got), by_id(ref)
    assert len(a) == len(b), (len(a), len(b))
    if len(a) == 0:
        return 0.0, 0.0
    assert np.array_equal(a["id"], b["id"])
    perr = 0.0
    for d, f in enumerate(["x", "y", "z"]):
        diff = a[f] - b[f]
        if period is not None and period[d][0]:
            n = period[d][1]
            diff = (diff + 0.5 * n) % n - 0.5 * n
        perr = max(perr, float(np.max(np.abs(diff))))
    pa = np.stack([a["px"], a["py"], a["pz"]])
    pb = np.stack([b["px"], b["py"], b["pz"]])
    return perr, rel_l2(pa, pb)


def periods(params):
    return [(int(params["period_x"]), int(params["local_xcells"])),
            (int(params["period_y"]), int(params["local_ycells"])),
            (int(params["period_z"]), int(params["local_zcells"]))]
