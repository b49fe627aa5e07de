"""Benchmark of the PIC3D per-timestep loop on B200.

Headline workload: the throughput scale-up configuration -- a periodic
512 x 256 x 256 thermal electron-proton plasma, 8 particles per cell per
species (536,870,912 particles), u_th = 0.02 c for both species, 2nd-order
shapes, FP64.  Seeded synthetic inputs of that shape (the device generator
pic_generate_thermal).  A step is one iteration of the reference's
run_main_time_loop over all particles and cells.  The same configuration in
FP32 and at 4th order is timed beside it (`variants`), the FP32 error
against FP64 is measured per step on the 32^3 thermal plasma (`fp32_error`),
the laser-in-underdense-plasma configuration is timed after the pulse has
entered the plasma (`laser`), and the differentiable run gives the adjoint /
forward time (`adjoint`).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  `value` is device-resident particle-steps/s
summed over ranks (each rank runs an independent replica: the reference's
only parallelism is MPI domain decomposition, which this single-GPU path
does not implement), `e2e` the same metric through the C ABI with the
particle state read from and written back to host memory inside the timed
region, `roofline` the dominant kernel against the measured HBM copy
bandwidth, `cpu_baseline` the reference CPU code on a bounded sample.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

# algorithmic bytes per particle-step of the fused gather+push+deposit
# kernel: particle state read + written, plus the grid bytes (6 E/B reads,
# 3 J writes) shared by the particles of a cell (16 per cell here)
BYTES_PER_PARTICLE = {"fp64": 104.0, "fp32": 60.0}
GRID_BYTES_PER_CELL = {"fp64": 72.0, "fp32": 36.0}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_traffic(precision, order):
    """DRAM bytes per particle of the tiled kernel from a committed ncu
    capture of a smaller case of the same workload
    (profiles/tile_push_traffic.json); the traffic grows in proportion to the
    particles a launch processes."""
    p = os.path.join(REPO, "profiles", "tile_push_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)["dram_bytes_per_particle"].get(f"{precision}_o{order}")


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows)}


TILE = dict(tile=0, sort_interval=0)

# the throughput scale-up configuration (8 + 8 particles per cell, u_th = 0.02)
SCALEUP_PPC, SCALEUP_UTH = 8, 0.02


def cpu_info():
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "logical_cpus": os.cpu_count()}


def thermal_sim(mem, precision, device, seed, nx=512, ny=256, nz=256):
    """The scale-up plasma generated on the device (seeded Philox)."""
    from pic3d_b200 import workloads as W
    from pic3d_b200.simulation import Simulation
    w = W.thermal_scaleup(nx=nx, ny=ny, nz=nz, mem=mem, precision=precision)
    sim = Simulation(w, precision=precision, device=device, **TILE)
    for k in range(2):
        sim.generate_thermal(k, SCALEUP_PPC, 1.0, SCALEUP_UTH, seed + k)
    return w, sim


def timed_steps(sim, steps, prof=True):
    """K steps bracketed by CUDA events on the library's stream; with
    prof, per-kernel CUDA-event totals on the same stream."""
    import torch
    stream = torch.cuda.ExternalStream(sim.stream())
    sim.synchronize()
    if prof:
        sim.profile(True)
        sim.profile_reset()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    sim.run_main_time_loop(steps)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    kern = sim.profile_read() if prof else {}
    sim.profile(False)
    sim.synchronize()
    return ms, kern


def count_kernel_launches(sim, steps=1):
    """Kernels this library launches per step, counted in the CUDA activity
    trace of torch.profiler (every kernel on the device, whatever stream;
    the library's kernels live in namespace pic); None if no trace."""
    try:
        import torch
        from torch.profiler import ProfilerActivity, profile
        sim.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            sim.run_main_time_loop(steps)
            sim.synchronize()
        n = sum(1 for e in prof.events()
                if e.device_type == torch.autograd.DeviceType.CUDA and "pic::" in e.name)
        return n / steps if n else None
    except Exception:
        return None


def measured_instructions(precision, order):
    """Thread instructions per particle of the tiled kernel from a committed
    ncu capture (profiles/tile_push_instructions.json: smsp__inst_executed.sum
    x 32 / particles of one launch)."""
    p = os.path.join(REPO, "profiles", "tile_push_instructions.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)["thread_instructions_per_particle"].get(f"{precision}_o{order}")


def issue_fraction(particles_per_s, precision, order, sm_mhz):
    """Instruction issue rate the measured rate implies, as a fraction of the
    issue peak (148 SMs x 4 schedulers x 32 lanes per clock)."""
    ipp = measured_instructions(precision, order)
    if not ipp or not sm_mhz:
        return None
    return particles_per_s * ipp / (148 * 4 * 32 * sm_mhz * 1e6)


def tile_roofline(kern, npart, ncell, precision, peak, peak_kind, ms_step, order=2):
    """HBM roofline of the tiled push kernel from its CUDA-event launch
    times: algorithmic bytes per launch / average launch duration."""
    t = kern.get("tile_push_gather_deposit")
    if not t or t[1] <= 0:
        return None
    avg_ms = t[0] / t[1]
    per = BYTES_PER_PARTICLE[precision] + GRID_BYTES_PER_CELL[precision] * ncell / max(npart, 1)
    achieved = per * npart / (avg_ms / 1e3) / 1e9
    tpp = measured_traffic(precision, order)
    return {"bound": "hbm", "kernel": "tile_push_gather_deposit", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": tpp * npart if tpp else None,
            "traffic_note": ("dram read+write bytes per launch: bytes per particle from an ncu capture of a "
                             "smaller case of the same workload, times the particles per launch") if tpp else None,
            "bytes_per_particle": per, "avg_launch_ms": avg_ms, "share_of_step": t[0] / ms_step}


def run_case(sim, warmup, steps, clocks=None):
    sim.initial_push()
    sim.run_main_time_loop(warmup)
    sim.synchronize()
    if clocks:
        clocks.start()
    ms, kern = timed_steps(sim, steps, prof=True)
    clk = clocks.stop() if clocks else None
    return ms, kern, clk


def variants_bench(local, rank, warmup, steps, skip=None):
    """The scale-up configuration at both orders and precisions (the
    headline's own case excluded)."""
    from pic3d_b200.simulation import Simulation  # noqa: F401
    peak, peak_kind = measured_peaks()
    out = []
    for mem, prec in ((2, "fp32"), (4, "fp64"), (4, "fp32")):
        if skip == (mem, prec):
            continue
        w, sim = thermal_sim(mem, prec, local, 97 + 2 * rank)
        npart = sum(sim.num_particles(k) for k in range(2))
        ncell = w.nx * w.ny * w.nz
        ms, kern, _ = run_case(sim, warmup, steps)
        sim.close()
        roof = tile_roofline(kern, npart, ncell, prec, peak, peak_kind, ms, 2 if mem == 2 else 4)
        out.append({"order": 2 if mem == 2 else 4, "precision": prec, "particles": npart,
                    "particle_steps_per_s": npart * steps / (ms / 1e3), "ms_per_step": ms / steps,
                    "cell_updates_per_s": ncell * steps / (ms / 1e3),
                    "tile_push_ms": roof["avg_launch_ms"] if roof else None,
                    "tile_push_roofline_frac": roof["frac"] if roof else None,
                    "tile_push_issue_frac": issue_fraction(npart / (roof["avg_launch_ms"] / 1e3), prec,
                                                           2 if mem == 2 else 4, 1965.0) if roof else None,
                    "kernels": {k: {"ms_total": v[0], "launches": v[1]} for k, v in kern.items()}})
    return out


def fp32_error_bench(local, steps=200, samples=(1, 2, 5, 10, 20, 50, 100, 200)):
    """The FP32 path against FP64 on the 32^3 thermal plasma (8 electrons
    per cell, u_th = 0.05, ions a fixed background, 2nd order; the FP64 GPU
    run equals the FP64 oracle per step to 1e-10): teacher-forced per-step
    relative L2 error of every field, current and particle array (the FP64
    state n uploaded into the FP32 context, one step, compared with FP64
    step n+1), and the free-running error of the two runs side by side with
    their energies."""
    from pic3d_b200 import workloads as W
    from pic3d_b200.simulation import Simulation

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b)) / nb if nb > 0 else 0.0

    names = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "rho0")
    out = {"workload": "thermal_periodic_32^3, 8 electrons per cell, u_th 0.05, order 2", "steps": steps,
           "teacher_forced": {}, "free_running": {}}
    w = W.thermal_periodic(32, mem=2, steps=steps)
    parts = W.make_particles(w, seed=1234)
    s64 = Simulation(w, precision="fp64", device=local, **TILE)
    s32 = Simulation(w, precision="fp32", device=local, **TILE)
    t32 = Simulation(w, precision="fp32", device=local, **TILE)
    for s in (s64, s32):
        for k in range(2):
            s.upload_particles(k, parts[k])
        s.initial_push()
    for n in range(1, steps + 1):
        if n in samples:
            st = s64.state()
            t32.upload_state(st)
            t32.step = n - 1
        s64.run_main_time_loop(1)
        s32.run_main_time_loop(1)
        if n in samples:
            t32.run_main_time_loop(1)
            a64, a32, f32 = s64.state(), s32.state(), t32.state()
            d64, d32 = s64.diagnostics(), s32.diagnostics()
            e64 = d64["field_energy"] + d64["kinetic0"]
            e32 = d32["field_energy"] + d32["kinetic0"]
            pa, pb = np.sort(f32["particles"][0], order="id"), np.sort(a64["particles"][0], order="id")
            mom = rel(np.stack([pa["px"], pa["py"], pa["pz"]]), np.stack([pb["px"], pb["py"], pb["pz"]]))
            out["teacher_forced"][n] = dict({k: rel(f32[k], a64[k]) for k in names}, momenta=mom)
            out["free_running"][n] = dict({k: rel(a32[k], a64[k]) for k in ("ex", "ey", "ez", "bx", "by", "bz",
                                                                             "jx", "jy", "jz")},
                                          total_energy_fp64=e64, total_energy_fp32=e32,
                                          energy_rel_diff=abs(e32 - e64) / abs(e64))
    for s in (s64, s32, t32):
        s.close()
    tf = out["teacher_forced"]
    out["teacher_forced_max"] = max(max(v.values()) for v in tf.values())
    out["note"] = ("teacher-forced: one FP32 step from the FP64 state, the per-step error the 1e-5 bound applies "
                   "to; free-running: the two runs diverge as any chaotic plasma does, shown for reference")
    return out


def laser_bench(local, rank, warmup_steps, steps, precision, cells=(256, 128, 128)):
    """The laser-in-underdense-plasma configuration (256x128x128, 4th order,
    8 + 8 particles per cell, a0 = 2, absorbing), timed after `warmup_steps`
    steps so that the pulse is inside the plasma and electrons move."""
    from pic3d_b200 import workloads as W
    from pic3d_b200.simulation import Simulation
    w = W.laser_underdense(nx=cells[0], ny=cells[1], nz=cells[2], precision=precision)
    parts = W.make_particles(w, seed=1234 + rank)
    sim = Simulation(w, precision=precision, device=local, **TILE)
    for k in range(2):
        sim.upload_particles(k, parts[k])
    del parts
    npart0 = sum(sim.num_particles(k) for k in range(2))
    ms, kern, _ = run_case(sim, warmup_steps, steps)
    npart = sum(sim.num_particles(k) for k in range(2))
    order = [sim.particle_order_stats(k) for k in range(2)]
    sim.close()
    peak, peak_kind = measured_peaks()
    ncell = w.nx * w.ny * w.nz
    roof = tile_roofline(kern, npart, ncell, precision, peak, peak_kind, ms, 4)
    return {"workload": w.name, "precision": precision, "timed_after_step": warmup_steps + 1,
            "particles_at_start": npart0, "particles_timed": npart,
            "particle_steps_per_s": npart * steps / (ms / 1e3), "ms_per_step": ms / steps,
            "tile_push_roofline_frac": roof["frac"] if roof else None, "particle_order": order,
            "kernels": {k: {"ms_total": v[0], "launches": v[1]} for k, v in kern.items()}}


def e2e_bench(local, steps, mem=2, precision="fp64"):
    """The headline metric through the C ABI with the particle state in host
    memory: particles generated on the device and downloaded once (untimed)
    stand for the caller's host arrays; the timed region uploads them
    (pic_upload_particles, host -> device), runs the t=0 push and K
    pic_run_steps(1) calls each followed by a pic_diagnostics read-back, and
    downloads every particle and field array (device -> host)."""
    from pic3d_b200.simulation import Simulation
    w, sim = thermal_sim(mem, precision, local, 4242)
    host = [sim.download_particles(k) for k in range(2)]
    sim.close()
    npart = sum(len(h) for h in host)
    sim = Simulation(w, precision=precision, device=local, **TILE)
    sim.synchronize()
    t0 = time.perf_counter()
    for k in range(2):
        sim.upload_particles(k, host[k])
    h2d = sum(h.nbytes for h in host)
    sim.initial_push()
    d2h = 0
    for _ in range(steps):
        sim.run_main_time_loop(1)
        sim.diagnostics()
        d2h += 8 * 6
    out = [sim.download_particles(k, host[k]) for k in range(2)]   # back into the caller's arrays
    flds = {n: sim.download_array(n) for n in ("ex", "ey", "ez", "bx", "by", "bz")}
    dt = time.perf_counter() - t0
    d2h += sum(p.nbytes for p in out) + sum(a.nbytes for a in flds.values())
    sim.close()
    return {"value": npart * steps / dt, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps, "seconds": dt,
            "note": "pic_upload_particles of 144-byte records from host memory, the t=0 push, K pic_run_steps(1) "
                    "each followed by a pic_diagnostics read-back, pic_download_particles and pic_download_array "
                    "of the final state, all inside the timed region"}


def scaleup_subbox():
    """The per-process CPU sample of the scale-up configuration: a 32x16x16
    sub-box with the same particles per cell, u_th and shape order."""
    from pic3d_b200 import workloads as W
    w = W.thermal_scaleup(nx=32, ny=16, nz=16, mem=2, precision="fp64")
    return w, W.make_particles(w, seed=11)


def cpu_baseline(target_s=15.0):
    """Reference CPU code (oracle/_ref, -O2, and the reference Makefile's
    -O0) on a bounded sample: the 32x16x16 sub-box of the scale-up
    configuration, one process on one core.  Falls back to the C port."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    w, parts = scaleup_subbox()
    n = sum(len(p) for p in parts)
    if O.have_reference_build():
        _, t = O.run_reference(w, parts, 2, timing=True)
        per_step = max(t["loop_seconds"] / 2, 1e-3)
        steps = int(max(2, min(100, target_s / per_step)))
        _, t = O.run_reference(w, parts, steps, timing=True)
        rate = t["particles_start"] * steps / t["loop_seconds"]
        res = {"value": rate, "unit": "particle-steps/s", "cores": 1, "kind": "reference", "cpu": cpu_info(),
               "sample": f"reference src/*.cpp -O2, 32x16x16 sub-box of the 512x256x256 thermal configuration "
                         f"({n} particles, 8+8 per cell, u_th 0.02, 2nd order, FP64), {steps} steps, 1 process"}
        if os.path.exists(O.REF_BIN_O0):
            s0 = max(2, steps // 4)
            _, t0 = O.run_reference(w, parts, s0, timing=True, binary=O.REF_BIN_O0)
            res["value_O0"] = t0["particles_start"] * s0 / t0["loop_seconds"]
            res["value_O0_note"] = f"the reference Makefile's -O0 build, {s0} steps, same sample"
        return res
    o = O.Oracle(w, parts)
    o.initial()
    t0 = time.perf_counter()
    o.step(1)
    per_step = time.perf_counter() - t0
    steps = int(max(2, min(100, target_s / max(per_step, 1e-3))))
    t0 = time.perf_counter()
    o.run(2, steps)
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": "particle-steps/s", "cores": 1, "kind": "port", "cpu": cpu_info(),
            "sample": f"C restatement (oracle/pic_oracle.c), 32x16x16 sub-box of the 512x256x256 thermal "
                      f"configuration ({n} particles, 2nd order), {steps} steps, 1 process"}


def reference_arm(args):
    """--impl reference: the reference's own CPU code on all host cores,
    as concurrent single-rank processes on equal sub-boxes of the scale-up
    configuration (the reference has no threads; its parallelism is MPI,
    absent here)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    w, parts = scaleup_subbox()
    w = w.with_(steps=args.steps)
    n = sum(len(p) for p in parts)
    use_ref = O.have_reference_build()
    if not use_ref:
        O.build_oracle()
    tmp = tempfile.mkdtemp(prefix="pic3d_refarm_")
    try:
        ppath = os.path.join(tmp, "particles.bin")
        O.write_particle_file(ppath, parts)
        prm = os.path.join(tmp, "params.txt")
        O.write_params_file(prm, w, args.steps, output_interval=args.steps + 1)
        env = dict(os.environ, PIC3D_REF_PARAMS=prm, PIC3D_G_TXT=O.REF_G_TXT)
        if use_ref:
            cmd = [O.REF_BIN, ppath, "-", "time"]
        else:
            cmd = [sys.executable, os.path.join(REPO, "oracle", "oracle.py"), "--port-time", ppath, prm]
        procs = []
        for c in range(cores):
            pre = ["taskset", "-c", str(c)] if shutil.which("taskset") else []
            procs.append(subprocess.Popen(pre + cmd, env=env, cwd=tmp, stdout=subprocess.PIPE,
                                          stderr=subprocess.PIPE, text=True))
        secs = []
        for p in procs:
            out, err = p.communicate()
            line = [l for l in out.splitlines() if l.startswith("{")]
            if p.returncode != 0 or not line:
                raise RuntimeError(f"reference process failed: {err[-500:]}")
            secs.append(json.loads(line[-1])["loop_seconds"])
        total = float(n) * args.steps * cores / max(secs)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    kind = "reference" if use_ref else "port"
    sample = (f"{cores} concurrent single-rank processes (one per core), each a 32x16x16 sub-box of the "
              f"512x256x256 thermal configuration ({n} particles, 8+8 per cell, u_th 0.02, 2nd order, FP64), "
              f"{args.steps} steps")
    line = {"impl": "reference", "metric": "particle-steps/s", "value": total, "unit": "particle-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * max(secs) / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "thermal_scaleup 512x256x256 (CPU sample: 32x16x16 sub-boxes per core)",
                       "order": 2, "particles_per_cell": 16, "u_th": SCALEUP_UTH, "boundaries": "periodic"},
            "cpu_baseline": {"value": total, "unit": "particle-steps/s", "cores": cores, "kind": kind,
                             "sample": sample, "cpu": cpu_info()},
            "e2e": {"value": total, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


FP64_SEGMENT = 50   # the FP64 record of 600 steps would not fit in HBM


class _RoundedSpec:
    """Mixin: initial positions and momenta rounded to FP32 (an FP64 run
    from inputs perturbed by 1e-8 relative)."""

    def base_particles(self):
        p = super().base_particles()
        for f in ("x", "y", "z", "px", "py", "pz"):
            p[f] = p[f].astype("float32").astype("float64")
        return p


def adjoint_bench(steps=600, short_steps=100):
    """Differentiable run: the FP32 forward records every push (600 steps
    fit in HBM) and the adjoint is one reverse sweep; the same gradient in
    FP64 (checkpoints every 50 steps, recomputed), the FP64 gradient from
    initial conditions rounded to FP32, and central finite differences of
    the FP64 forward run at a sequence of steps.

    The objective is only piecewise smooth: electrons leave through the
    absorbing faces (hundreds of thousands per 100 steps here) and each
    removal is a jump, so differences converge to the derivative only once
    the step is small enough that no removal changes step (about 1e-8 of the
    parameter at 600 steps).  At 600 steps the gradient itself is sensitive
    at the 1e-8 level of the inputs: the FP64 gradient from FP32-rounded
    initial conditions differs from the exact-input one by tens of percent,
    as much as the FP32 gradient does; at 100 steps all three agree to
    1e-6."""
    import numpy as np

    from pic3d_b200 import workloads as W
    from pic3d_b200.adjoint import AdjointRun, AdjointSpec, objective

    class RoundedSpec(_RoundedSpec, AdjointSpec):
        pass

    def spec(prec, n=steps, cls=AdjointSpec):
        w = W.differentiable_laser(precision=prec, steps=n)
        seg = n if prec == "fp32" else FP64_SEGMENT
        return cls(workload=w, n_knots=32, profile_n=8, window=(0.5 * w.nx, w.nx - 4.0), ramp=4.0,
                   segment=seg, seed=2468, precision=prec)

    rng = np.random.default_rng(13)
    knots = 0.01 + 0.02 * rng.random(32)
    prof = 1.0 + 0.2 * rng.random((8, 8))

    def grad(sp, kernels=False):
        run = AdjointRun(sp, knots, prof)
        run.sim.synchronize()
        t0 = time.perf_counter()
        loss = run.forward()
        run.sim.synchronize()
        t1 = time.perf_counter()
        if kernels:
            run.sim.profile(True)
            run.sim.profile_reset()
        gw, gp = run.backward()
        run.sim.synchronize()
        t2 = time.perf_counter()
        kern = run.sim.profile_read() if kernels else {}
        gk = sp.knot_grad(run.x0, gw)
        n = len(run.records)
        run.close()
        return dict(loss=loss, gk=gk, gp=gp, fwd=t1 - t0, bwd=t2 - t1, n=n,
                    kernels={k: {"ms_total": v[0], "launches": v[1]} for k, v in kern.items()})

    def production_forward(sp):
        """The same run (particles, weights, laser) in an ordinary context:
        the forward cost a user pays without the adjoint."""
        from pic3d_b200.simulation import Simulation
        rec = sp.base_particles()
        rec["weight"] = sp.weights(rec["x"].copy(), knots)
        sim = Simulation(sp.workload, precision=sp.precision, laser_profile=prof.reshape(8, 8), **TILE)
        sim.upload_particles(0, rec)
        sim.upload_particles(1, np.zeros(0, rec.dtype))
        sim.synchronize()
        t0 = time.perf_counter()
        sim.initial_push()
        sim.run_main_time_loop(sp.workload.steps)
        sim.synchronize()
        dt = time.perf_counter() - t0
        sim.close()
        return dt

    rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    a, b = grad(spec("fp32"), kernels=True), grad(spec("fp64"))
    br = grad(spec("fp64", cls=RoundedSpec))
    prod32 = production_forward(spec("fp32"))
    sa, sb = grad(spec("fp32", short_steps)), grad(spec("fp64", short_steps))
    sbr = grad(spec("fp64", short_steps, cls=RoundedSpec))
    sp64 = spec("fp64")
    checks = []
    for which, idx in [("knot", int(np.argmax(np.abs(b["gk"])))), ("laser", int(np.argmax(np.abs(b["gp"]))))]:
        g = b["gk"][idx] if which == "knot" else b["gp"][idx]
        base = knots[idx] if which == "knot" else prof.ravel()[idx]
        fds = {}
        for rel_h in (1e-5, 1e-8, 1e-9):
            k1, k2, p1, p2 = knots.copy(), knots.copy(), prof.ravel().copy(), prof.ravel().copy()
            h = rel_h * abs(base)
            if which == "knot":
                k1[idx] += h
                k2[idx] -= h
            else:
                p1[idx] += h
                p2[idx] -= h
            fds[f"{rel_h:g}"] = (objective(sp64, k1, p1) - objective(sp64, k2, p2)) / (2 * h)
        checks.append({"param": f"{which}[{idx}]", "adjoint_fp64": g, "central_fd_fp64_by_relative_step": fds,
                       "rel_err_by_relative_step": {k: abs(g - f) / max(abs(f), 1e-300) for k, f in fds.items()}})
    return {"workload": spec("fp32").workload.name, "particles": a["n"], "steps": steps,
            "checkpoint_every": {"fp32": steps, "fp64": FP64_SEGMENT},
            "parameters": 32 + 64, "objective": "sum s(x) w m (gamma-1), s = 1 on x in [32, 60) cells with 4-cell "
                                                  "sin^2 ramps",
            "objective_fp32": a["loss"], "objective_fp64": b["loss"],
            "forward_s": a["fwd"], "adjoint_s": a["bwd"], "adjoint_over_forward": a["bwd"] / a["fwd"],
            "production_forward_s": prod32, "adjoint_over_production_forward": a["bwd"] / prod32,
            "forward_and_adjoint_over_production_forward": (a["fwd"] + a["bwd"]) / prod32,
            "adjoint_kernels_fp32": a["kernels"],
            "fp64_forward_s": b["fwd"], "fp64_adjoint_s": b["bwd"],
            "grad_rel_l2_fp32_vs_fp64": {"knots": rel(a["gk"], b["gk"]), "laser": rel(a["gp"], b["gp"])},
            f"grad_rel_l2_fp32_vs_fp64_{short_steps}_steps": {"knots": rel(sa["gk"], sb["gk"]),
                                                              "laser": rel(sa["gp"], sb["gp"])},
            "grad_rel_l2_fp64_rounded_inputs_vs_fp64": {"knots": rel(br["gk"], b["gk"]),
                                                        "laser": rel(br["gp"], b["gp"])},
            f"grad_rel_l2_fp64_rounded_inputs_vs_fp64_{short_steps}_steps": {"knots": rel(sbr["gk"], sb["gk"]),
                                                                             "laser": rel(sbr["gp"], sb["gp"])},
            "finite_difference_checks": checks,
            "note": "FP32: the forward records the inputs of every push (one segment of 600 steps) and the "
                    "adjoint is one reverse sweep; FP64: checkpoints every 50 steps, each segment recomputed while "
                    "recording; forward = the run in the adjoint-capable context (tiled push, sorts recorded); "
                    "production forward = the same run in an ordinary context; central differences of a "
                    "piecewise-smooth objective converge only at small steps (particle removal at the absorbing "
                    "faces); rounded inputs = FP64 run from positions and momenta rounded to FP32"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--order", type=int, default=2, choices=[2, 4], help="headline shape order")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"], help="headline precision")
    ap.add_argument("--cells", default="512,256,256", help="headline grid (smaller grids for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-launch-count", action="store_true", help="skip the CUDA activity trace (for ncu runs)")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-fp32-error", action="store_true")
    ap.add_argument("--no-laser", action="store_true")
    ap.add_argument("--laser-warmup", type=int, default=600)
    ap.add_argument("--laser-cells", default="256,128,128", help="laser grid (smaller grids for profiling)")
    ap.add_argument("--laser-only", action="store_true", help="only the laser configuration (profiling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=600)
    ap.add_argument("--tile", type=int, default=0, help="shared-memory tile edge (0 default, -1 global kernel)")
    ap.add_argument("--sort-interval", type=int, default=0)
    args = ap.parse_args()
    TILE.update(tile=args.tile, sort_interval=args.sort_interval)
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.laser_only:
        lc = tuple(int(v) for v in args.laser_cells.split(","))
        out = laser_bench(local, rank, args.laser_warmup, args.steps, args.precision, lc)
        if rank == 0:
            print(json.dumps({"laser": out}), flush=True)
        return
    nx, ny, nz = (int(v) for v in args.cells.split(","))
    mem, prec = (2 if args.order == 2 else 4), args.precision
    w, sim = thermal_sim(mem, prec, local, 97 + 2 * rank, nx, ny, nz)
    npart = sum(sim.num_particles(k) for k in range(2))
    ncell = w.nx * w.ny * w.nz
    sim.initial_push()
    sim.run_main_time_loop(args.warmup)
    launches_per_step = None if args.no_launch_count else count_kernel_launches(sim, 4)
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms, kern = timed_steps(sim, args.steps, prof=True)
    clk = clocks.stop()
    order_stats = [sim.particle_order_stats(k) for k in range(2)]
    sim.close()
    from pic3d_b200.replicas import combine
    ms, npart_all, value = combine(ms, npart, args.steps, dist, device="cuda")
    peak, peak_kind = measured_peaks()
    roof = tile_roofline(kern, npart, ncell, prec, peak, peak_kind, ms, w.order)
    if roof:
        smhz = (clk or {}).get("sm_mhz") or 1965.0
        roof["issue_frac"] = issue_fraction(npart / (roof["avg_launch_ms"] / 1e3), prec, w.order, smhz)
        roof["issue_note"] = ("thread instructions per particle from an ncu capture of a smaller case of the same "
                              "workload, times the kernel's particle rate, over 148 SMs x 4 issue slots x 32 lanes "
                              "per clock at the sampled SM clock")
    kernels = {k: {"ms_total": v[0], "launches": v[1]} for k, v in kern.items()}

    extra = {}
    if not args.no_variants:
        try:
            extra["variants"] = variants_bench(local, rank, args.warmup, args.steps, skip=(mem, prec))
        except Exception as e:
            extra["variants"] = {"error": str(e)[:300]}
    if rank == 0 and not args.no_fp32_error:
        try:
            extra["fp32_error"] = fp32_error_bench(local)
        except Exception as e:
            extra["fp32_error"] = {"error": str(e)[:300]}
    if not args.no_laser:
        try:
            extra["laser"] = [laser_bench(local, rank, args.laser_warmup, args.steps, p) for p in ("fp64", "fp32")]
        except Exception as e:
            extra["laser"] = {"error": str(e)[:300]}
    e2e = None
    if not args.no_e2e:
        try:
            e2e = e2e_bench(local, args.steps, mem, prec)
            if world > 1:
                e2e["value"] *= world
        except Exception as e:
            e2e = {"error": str(e)[:300]}
    if rank == 0 and not args.no_adjoint:
        try:
            extra["adjoint"] = adjoint_bench(args.adjoint_steps)
        except Exception as e:
            extra["adjoint"] = {"error": str(e)[:300]}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline()
        except Exception as e:  # the baseline must not sink the GPU line
            cpu = {"value": None, "error": str(e)[:200]}

    if rank == 0:
        state_gb = npart * (BYTES_PER_PARTICLE[prec] / 2) / 1e9
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if prec == "fp64" else "f32", "data": "synthetic",
                "config": {"workload": w.name, "cells": [w.nx, w.ny, w.nz], "order": w.order,
                           "particles": npart, "particles_per_cell": 2 * SCALEUP_PPC, "u_th": SCALEUP_UTH,
                           "boundaries": "periodic", "tile": args.tile or 4,
                           "sort_interval": args.sort_interval or 4,
                           "parallelism": f"replicas{world}",
                           "l2": f"inputs larger than L2 (particle state {state_gb:.1f} GB)"},
                "cell_updates_per_s": ncell * world * args.steps / (ms / 1e3),
                "gpu_launches": int(launches_per_step * args.steps) if launches_per_step else None,
                "roofline": roof, "kernels": kernels, "particle_order": order_stats, "clocks": clk, "e2e": e2e,
                "cpu_baseline": cpu}
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
