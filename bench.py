"""Benchmark of the PIC3D per-timestep loop on B200.

Workload (default): the laser-in-underdense-plasma configuration —
256 x 128 x 128 cells, dx = lambda/20, dy = dz = lambda/10, electrons and
protons at 8 particles per cell each (67,108,864 particles), density
0.01 n_c on a linear ramp, cold start, a0 = 2 laser from x-min, absorbing
faces, 4th-order shapes, FP64.  Synthetic seeded inputs of that shape.
A step is one iteration of the reference's run_main_time_loop over all
particles and cells.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  `value` is device-resident particle-steps/s
summed over ranks (each rank runs an independent replica: the reference's
only parallelism is MPI domain decomposition, which this single-GPU path
does not implement), `e2e` the same metric through the C ABI with host
buffers, `roofline` the dominant kernel against the measured HBM copy
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


def measured_traffic(precision):
    """DRAM bytes per particle of the tiled kernel from a committed ncu
    capture (profiles/tile_push_traffic.json); the traffic grows in
    proportion to the particles a launch processes."""
    p = os.path.join(REPO, "profiles", "tile_push_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)["dram_bytes_per_particle"].get(precision)


def workload(name, precision):
    from pic3d_b200 import workloads as W
    if name == "laser_underdense":
        return W.laser_underdense(precision=precision)
    if name == "laser_underdense_small":
        return W.laser_underdense(nx=64, ny=32, nz=32, precision=precision)
    if name == "laser_underdense_medium":
        return W.laser_underdense(nx=128, ny=64, nz=64, precision=precision)
    if name == "thermal_scaleup":
        return W.thermal_scaleup(precision=precision)
    if name in ("thermal_o2_medium", "thermal_o4_medium"):
        return W.thermal_scaleup(nx=128, ny=64, nz=64, mem=2 if "o2" in name else 4, precision=precision)
    raise SystemExit(f"unknown workload {name}")


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


def make_sim(w, precision, particles, device):
    from pic3d_b200.simulation import Simulation
    sim = Simulation(w, precision=precision, device=device, **TILE)
    for k in range(2):
        sim.upload_particles(k, particles[k])
    return sim


def timed_steps(sim, steps, prof=True):
    """K steps bracketed by CUDA events on the library's stream."""
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


def cpu_baseline(precision_bytes_note=None, target_s=15.0):
    """Reference CPU code (oracle/_ref) on a bounded sub-box sample of the
    same per-particle workload (4th order, 8+8 particles per cell, laser
    parameters), one process, one core.  Falls back to the C port."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    from pic3d_b200 import workloads as W
    w = W.laser_underdense(nx=32, ny=16, nz=16, steps=4)
    parts = W.make_particles(w, seed=11)
    n = sum(len(p) for p in parts)
    if O.have_reference_build():
        # estimate the per-step cost with a short run, then size the sample
        _, t = O.run_reference(w, parts, 2, timing=True)
        per_step = max(t["loop_seconds"] / 2, 1e-3)
        steps = int(max(2, min(60, target_s / per_step)))
        _, t = O.run_reference(w, parts, steps, timing=True)
        rate = t["particles_start"] * steps / t["loop_seconds"]
        return {"value": rate, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
                "sample": f"reference src/*.cpp -O2, 32x16x16 sub-box of the laser workload "
                          f"({n} particles, 4th order), {steps} steps, 1 process"}
    o = O.Oracle(w, parts)
    o.initial()
    t0 = time.perf_counter()
    o.step(1)
    per_step = time.perf_counter() - t0
    steps = int(max(2, min(60, target_s / max(per_step, 1e-3))))
    t0 = time.perf_counter()
    o.run(2, steps)
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": "particle-steps/s", "cores": 1, "kind": "port",
            "sample": f"C restatement (oracle/pic_oracle.c), 32x16x16 sub-box of the laser workload "
                      f"({n} particles, 4th order), {steps} steps, 1 process"}


def reference_arm(args):
    """--impl reference: the reference's own CPU code on all host cores,
    as concurrent single-rank processes on equal sub-boxes (the reference
    has no threads; its parallelism is MPI, absent here)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    from pic3d_b200 import workloads as W
    cores = os.cpu_count() or 1
    w = W.laser_underdense(nx=32, ny=16, nz=16, steps=args.steps)
    parts = W.make_particles(w, seed=11)
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
        rates, secs = [], []
        for p in procs:
            out, err = p.communicate()
            line = [l for l in out.splitlines() if l.startswith("{")]
            if p.returncode != 0 or not line:
                raise RuntimeError(f"reference process failed: {err[-500:]}")
            t = json.loads(line[-1])
            secs.append(t["loop_seconds"])
            rates.append(t["particles_start"] * t["steps"] / t["loop_seconds"])
        total = float(n) * args.steps * cores / max(secs)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    kind = "reference" if use_ref else "port"
    sample = (f"{cores} concurrent single-rank processes (one per core), each a 32x16x16 sub-box of the laser "
              f"workload ({n} particles, 4th order, FP64), {args.steps} steps")
    line = {"impl": "reference", "metric": "particle-steps/s", "value": total, "unit": "particle-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * max(secs) / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "laser_underdense 256x128x128 (CPU sample: 32x16x16 sub-boxes)", "order": 4,
                       "particles_per_cell": 16},
            "cpu_baseline": {"value": total, "unit": "particle-steps/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": total, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def adjoint_bench(steps=600, short_steps=100):
    """Differentiable run: forward (with checkpoints every 50 steps) and
    adjoint (segment recompute + reverse sweep) in FP32, the same gradient in
    FP64, and central finite differences of the FP64 forward run at a
    sequence of steps.

    The objective is only piecewise smooth: electrons leave through the
    absorbing faces (hundreds of thousands per 100 steps here) and each
    removal is a jump, so differences converge to the derivative only once
    the step is small enough that no removal changes step (about 1e-8 of the
    parameter at 600 steps).  The same roughness makes the FP32 and FP64
    derivatives differ at long horizons (the FP32 trajectory differs from the
    FP64 one by more than that scale); the FP32 / FP64 agreement is also
    reported at a short horizon where it is not rough."""
    import numpy as np

    from pic3d_b200 import workloads as W
    from pic3d_b200.adjoint import AdjointRun, AdjointSpec, objective

    def spec(prec, n=steps):
        w = W.differentiable_laser(precision=prec, steps=n)
        return AdjointSpec(workload=w, n_knots=32, profile_n=8, window=(0.5 * w.nx, w.nx - 4.0), ramp=4.0,
                           segment=50, seed=2468, precision=prec)

    rng = np.random.default_rng(13)
    knots = 0.01 + 0.02 * rng.random(32)
    prof = 1.0 + 0.2 * rng.random((8, 8))

    def grad(sp):
        run = AdjointRun(sp, knots, prof)
        run.sim.synchronize()
        t0 = time.perf_counter()
        loss = run.forward()
        run.sim.synchronize()
        t1 = time.perf_counter()
        gw, gp = run.backward()
        run.sim.synchronize()
        t2 = time.perf_counter()
        gk = sp.knot_grad(run.x0, gw)
        n = len(run.records)
        run.close()
        return dict(loss=loss, gk=gk, gp=gp, fwd=t1 - t0, bwd=t2 - t1, n=n)

    rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    a, b = grad(spec("fp32")), grad(spec("fp64"))
    sa, sb = grad(spec("fp32", short_steps)), grad(spec("fp64", short_steps))
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
    return {"workload": spec("fp32").workload.name, "particles": a["n"], "steps": steps, "checkpoint_every": 50,
            "parameters": 32 + 64, "objective": "sum s(x) w m (gamma-1), s = 1 on x in [32, 60) cells with 4-cell "
                                                  "sin^2 ramps",
            "objective_fp32": a["loss"], "objective_fp64": b["loss"],
            "forward_s": a["fwd"], "adjoint_s": a["bwd"], "adjoint_over_forward": a["bwd"] / a["fwd"],
            "fp64_forward_s": b["fwd"], "fp64_adjoint_s": b["bwd"],
            "grad_rel_l2_fp32_vs_fp64": {"knots": rel(a["gk"], b["gk"]), "laser": rel(a["gp"], b["gp"])},
            f"grad_rel_l2_fp32_vs_fp64_{short_steps}_steps": {"knots": rel(sa["gk"], sb["gk"]),
                                                              "laser": rel(sa["gp"], sb["gp"])},
            "finite_difference_checks": checks,
            "note": "adjoint = restore each checkpoint, recompute its 50 steps recording the push inputs, reverse "
                    "sweep; forward = the run with checkpoints; both in adjoint mode (global push kernel); central "
                    "differences of a piecewise-smooth objective converge only at small steps (particle removal "
                    "at the absorbing faces)"}


def scaleup_bench(local, steps=3, warmup=3):
    """Throughput scale-up configuration: periodic 512 x 256 x 256 thermal
    electron-proton plasma, 8 particles per cell per species (536,870,912
    particles), u_th = 0.02, 2nd- and 4th-order shapes, FP32 and FP64.
    Particles come from the device generator (pic_generate_thermal: seeded
    Philox, no host particle memory); a short timed window per case keeps
    the default run within minutes (the per-step cost is steady: no laser,
    uniform plasma)."""
    from pic3d_b200 import workloads as W
    from pic3d_b200.simulation import Simulation
    out = []
    for mem in (2, 4):
        for prec in ("fp32", "fp64"):
            w = W.thermal_scaleup(mem=mem, precision=prec)
            sim = Simulation(w, precision=prec, device=local, **TILE)
            for k in range(2):
                sim.generate_thermal(k, 8, 1.0, 0.02, 97 + k)
            npart = sum(sim.num_particles(k) for k in range(2))
            sim.initial_push()
            sim.run_main_time_loop(warmup)
            ms, kern = timed_steps(sim, steps, prof=True)
            sim.close()
            tile = kern.get("tile_push_gather_deposit", (0.0, 1))
            avg = tile[0] / max(tile[1], 1)
            ncell = w.nx * w.ny * w.nz
            per = BYTES_PER_PARTICLE[prec] + GRID_BYTES_PER_CELL[prec] * ncell / npart
            peak, _ = measured_peaks()
            out.append({"order": 2 if mem == 2 else 4, "precision": prec, "particles": npart,
                        "particle_steps_per_s": npart * steps / (ms / 1e3), "ms_per_step": ms / steps,
                        "cell_updates_per_s": ncell * steps / (ms / 1e3), "tile_push_ms": avg,
                        "tile_push_roofline_frac": per * npart / (avg / 1e3) / 1e9 / peak if avg > 0 else None})
    return {"workload": "thermal_scaleup_512x256x256", "cells": [512, 256, 256], "particles_per_cell": 16,
            "u_th": 0.02, "steps": steps, "warmup": warmup, "results": out}


def field_rel_err(a: dict, b: dict):
    num = sum(float(np.sum((a[n] - b[n]) ** 2)) for n in ("ex", "ey", "ez", "bx", "by", "bz"))
    den = sum(float(np.sum(b[n] ** 2)) for n in ("ex", "ey", "ez", "bx", "by", "bz"))
    return (num / den) ** 0.5 if den > 0 else 0.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="laser_underdense")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-scaleup", action="store_true")
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

    from pic3d_b200 import workloads as W
    w = workload(args.workload, args.precision)
    parts = W.make_particles(w, seed=1234 + rank)
    npart = sum(len(p) for p in parts)
    ncell = w.nx * w.ny * w.nz

    sim = make_sim(w, args.precision, parts, local)
    sim.initial_push()
    sim.run_main_time_loop(args.warmup)
    sim.synchronize()
    # count kernel launches per step (profiling pass, untimed)
    sim.profile(True)
    sim.profile_reset()
    sim.run_main_time_loop(1)
    launches_per_step = sum(v[1] for v in sim.profile_read().values())
    sim.profile(False)

    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms, kern = timed_steps(sim, args.steps, prof=True)
    clk = clocks.stop()
    from pic3d_b200.replicas import combine
    ms, npart_all, value = combine(ms, npart, args.steps, dist, device="cuda")

    # dominant kernel roofline
    peak, peak_kind = measured_peaks()
    top = max(kern.items(), key=lambda kv: kv[1][0]) if kern else ("", (0.0, 0))
    prec = args.precision
    per_particle = BYTES_PER_PARTICLE[prec] + GRID_BYTES_PER_CELL[prec] * ncell / max(npart, 1)
    roof = None
    if top[0] in ("push_gather_deposit", "tile_push_gather_deposit") and top[1][1] > 0:
        avg_ms = top[1][0] / top[1][1]
        # the global kernel runs once per species, the tiled one once for both
        per_launch = npart / 2.0 if top[0] == "push_gather_deposit" else float(npart)
        bytes_per_launch = per_particle * per_launch
        achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
        tpp = measured_traffic(prec) if top[0] == "tile_push_gather_deposit" else None
        roof = {"bound": "hbm", "kernel": top[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": tpp * per_launch if tpp else None,
                "traffic_note": "dram read+write bytes per launch, scaled by particles from an ncu capture of "
                                "128x64x64 cells" if tpp else None,
                "bytes_per_particle": per_particle, "avg_launch_ms": avg_ms,
                "share_of_step": top[1][0] / ms}
    kernels = {k: {"ms_total": v[0], "launches": v[1]} for k, v in kern.items()}

    extra = {}
    # FP32 path on the same inputs: throughput and error against FP64
    if not args.no_fp32 and prec == "fp64":
        st64 = {n: sim.download_array(n) for n in ("ex", "ey", "ez", "bx", "by", "bz")}
        sim.close()
        sim32 = make_sim(w, "fp32", parts, local)
        sim32.initial_push()
        sim32.run_main_time_loop(args.warmup + 1)
        ms32, kern32 = timed_steps(sim32, args.steps, prof=True)
        st32 = {n: sim32.download_array(n) for n in ("ex", "ey", "ez", "bx", "by", "bz")}
        err = field_rel_err(st32, st64)
        kname = "tile_push_gather_deposit" if "tile_push_gather_deposit" in kern32 else "push_gather_deposit"
        t32 = kern32.get(kname, (0.0, 1))
        avg32 = t32[0] / max(t32[1], 1)
        pp32 = BYTES_PER_PARTICLE["fp32"] + GRID_BYTES_PER_CELL["fp32"] * ncell / max(npart, 1)
        per_launch32 = npart / 2.0 if kname == "push_gather_deposit" else float(npart)
        ach32 = pp32 * per_launch32 / (avg32 / 1e3) / 1e9 if avg32 > 0 else None
        extra["fp32"] = {"value": npart_all * args.steps / (ms32 / 1e3), "ms_per_step": ms32 / args.steps,
                         "field_rel_l2_vs_fp64": err,
                         "error_note": f"E,B after {args.warmup + 1 + args.steps} steps vs the FP64 GPU run "
                                       "(itself within 1e-10/step of the FP64 oracle)",
                         "roofline": {"kernel": kname, "achieved": ach32, "peak": peak,
                                      "unit": "GB/s", "frac": (ach32 / peak) if ach32 else None}}
        sim32.close()
    else:
        sim.close()

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        from pic3d_b200.simulation import Simulation
        torch.cuda.synchronize()
        host_fields = {n: np.zeros((w.nz + 2 * w.mem, w.ny + 2 * w.mem, w.nx + 2 * w.mem)) for n in
                       ("ex", "ey", "ez", "bx", "by", "bz")}
        simE = Simulation(w, precision=prec, device=local, **TILE)
        t0 = time.perf_counter()
        for n, a in host_fields.items():
            simE.upload_array(n, a)
        for k in range(2):
            simE.upload_particles(k, parts[k])
        h2d = sum(a.nbytes for a in host_fields.values()) + sum(p.nbytes for p in parts)
        simE.initial_push()
        d2h = 0
        for s in range(args.steps):
            simE.run_main_time_loop(1)
            simE.diagnostics()
            d2h += 8 * 6
        out = [simE.download_particles(k) for k in range(2)]
        flds = {n: simE.download_array(n) for n in ("ex", "ey", "ez", "bx", "by", "bz")}
        dt = time.perf_counter() - t0
        d2h += sum(p.nbytes for p in out) + sum(a.nbytes for a in flds.values())
        simE.close()
        e2e = {"value": npart * args.steps / dt * (world if world > 1 else 1), "unit": "particle-steps/s",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "note": "pic_upload_* of the initial state from host memory, the t=0 push, K pic_run_steps(1) "
                       "each followed by a pic_diagnostics read-back, pic_download_* of the final state"}

    if not args.no_scaleup:
        try:
            extra["scaleup"] = scaleup_bench(local)
        except Exception as e:
            extra["scaleup"] = {"error": str(e)[:300]}

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
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if prec == "fp64" else "f32", "data": "synthetic",
                "config": {"workload": w.name, "cells": [w.nx, w.ny, w.nz], "order": w.order,
                           "tile": args.tile, "sort_interval": args.sort_interval,
                           "particles": npart, "particles_per_cell": sum(w.ppc), "boundaries": "periodic" if all(w.period) else "absorbing+laser",
                           "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (particle state "
                                                                   f"{npart * BYTES_PER_PARTICLE[prec] / 1e9:.1f} GB)"},
                "cell_updates_per_s": ncell * world * args.steps / (ms / 1e3),
                "gpu_launches": int(launches_per_step * args.steps),
                "roofline": roof, "kernels": kernels, "clocks": clk, "e2e": e2e, "cpu_baseline": cpu}
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
