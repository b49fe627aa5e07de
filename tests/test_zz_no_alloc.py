"""The diagnostics entry point that allocates no device memory.

pic_field_diagnostics_noalloc is for callers that cannot let a library call
cudaMalloc (they reserve nearly all of HBM for their own arrays, or allow
device memory only through their own pool).  It reads caller-owned device
arrays and writes caller-owned output; its scratch is a static device array
shared by every call.  This test calls it through the C ABI on device arrays
the test owns and checks it against pic_diagnostics of a context holding the
same state, twice in a row with the state changed in between (the shared
scratch must not leak one call into the next), and checks that a grid larger
than the static scratch is rejected.  Collected last: a run that stops at the
first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

from golden_io import load

pytestmark = pytest.mark.gpu

FIELDS = ["ex", "ey", "ez", "bx", "by", "bz", "rho0", "rho1"]


def _noalloc(lib, params, dev_arrays, out, stream):
    ptrs = [ctypes.c_void_p(dev_arrays[n].data_ptr()) for n in FIELDS]
    return lib.pic_field_diagnostics_noalloc(ctypes.byref(params), *ptrs, ctypes.c_void_p(out.data_ptr()),
                                             ctypes.c_void_p(stream))


def test_noalloc_diagnostics_match_context_diagnostics():
    import torch

    from pic3d_b200 import _lib as L
    from pic3d_b200.simulation import Simulation

    lib = L.load()
    g = load("mixed_o2")
    sim = Simulation(g["params"], precision="fp64")
    for k in range(2):
        sim.upload_particles(k, g["input"][k])
    sim.initial_push()
    sim.run_main_time_loop(2)
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for call in range(2):
        ref = sim.diagnostics()
        dev = {n: torch.from_numpy(sim.download_array(n)).to("cuda") for n in FIELDS}
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        assert _noalloc(lib, sim.params, dev, out, stream) == L.PIC_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = np.array([ref["field_energy"], ref["charge0"], ref["charge1"], ref["gauss_max"]])
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got[:3], want[:3], rtol=1e-12, atol=1e-14)
        assert got[3] == want[3]
        results.append(got)
        sim.run_main_time_loop(3)   # change the state before the second call
    assert not np.array_equal(results[0], results[1])
    sim.close()


def test_noalloc_call_allocates_no_device_memory():
    """After a first call (which loads the module and looks up the scratch
    address), a call leaves the device's free memory exactly as it was."""
    import torch

    from pic3d_b200 import _lib as L
    from pic3d_b200.simulation import Simulation

    lib = L.load()
    g = load("periodic_o2")
    sim = Simulation(g["params"], precision="fp64")
    dev = {n: torch.from_numpy(sim.download_array(n)).to("cuda") for n in FIELDS}
    sim.close()
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert _noalloc(lib, sim.params, dev, out, stream) == L.PIC_OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    assert _noalloc(lib, sim.params, dev, out, stream) == L.PIC_OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_noalloc_reports_a_nan_field_as_a_nan_gauss_residual():
    import torch

    from pic3d_b200 import _lib as L
    from pic3d_b200.simulation import Simulation

    lib = L.load()
    g = load("periodic_o2")
    sim = Simulation(g["params"], precision="fp64")
    for k in range(2):
        sim.upload_particles(k, g["input"][k])
    sim.initial_push()
    sim.run_main_time_loop(1)
    host = {n: sim.download_array(n) for n in FIELDS}
    sim.close()
    m = int(g["params"]["mem"])
    host["ex"][m + 1, m + 1, m + 1] = float("nan")
    dev = {n: torch.from_numpy(a).to("cuda") for n, a in host.items()}
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert _noalloc(lib, sim.params, dev, out, torch.cuda.current_stream().cuda_stream) == L.PIC_OK
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.isnan(got[0]) and np.isnan(got[3])
    assert np.isfinite(got[1]) and np.isfinite(got[2])


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    import torch

    from pic3d_b200 import _lib as L
    from pic3d_b200.simulation import params_from

    lib = L.load()
    p = params_from(load("mixed_o2")["params"])
    p.local_zcells = 4096
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    dev = {n: dummy for n in FIELDS}
    assert _noalloc(lib, p, dev, dummy, torch.cuda.current_stream().cuda_stream) == L.PIC_EINVAL
