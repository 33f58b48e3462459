#!/usr/bin/env python
"""Throughput of the RK4 step of the AdS4 holographic superfluid on B200.

A bench "step" is one RK4 step (four stages, constraint, winding removal,
filter) of the whole grid.  Default workload: the driven-flow configuration
301x301x21 (nz = 21 Chebyshev points), L = 100, mu = 6, dt = 0.02,
A_y(z=0) = 2*pi*7/20 with global winding removal, complex Gaussian noise
1e-3 (seed 0) on the Newton stationary profile; synthetic, generated here.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  ``value`` is site-updates/s (nx*ny*nz*steps
per second over all ranks) with the state resident in HBM; ``e2e`` is the
same metric through the host-array call ``hqt_step`` (pinned host buffers,
copies inside the timed region).  N > 1 runs one independent replica per GPU
(the single-run step does not shard; replicas only, weak scaling).
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = "ads4-holographic-quantum-turbulence_b200"
VY7 = -2 * np.pi * 7 / 20

WORKLOADS = {
    "driven301": dict(nx=301, ny=301, nz=21, L=100.0, mu=6.0, vy=VY7, dt=0.02,
                      remove_winding=True, noise="complex", amp=1e-3, seed=0),
    "cpu64": dict(nx=64, ny=64, nz=21, L=50.0, mu=6.0, vy=0.0, dt=0.02,
                  remove_winding=True, noise="complex", amp=1e-3, seed=0),
    "lattice512": dict(nx=512, ny=512, nz=25, L=128.0, mu=6.0, vy=0.0, dt=0.02,
                       remove_winding=False, noise="complex", amp=1e-3, seed=1),
    # the large single run's grid: 1024x1024x33, L = 256, dt = 0.01
    "large1024": dict(nx=1024, ny=1024, nz=33, L=256.0, mu=6.0, vy=0.0, dt=0.01,
                      remove_winding=True, noise="complex", amp=1e-3, seed=2),
}

# The batched-ensemble workload: 32 independent runs, grids {128,192,256}^2,
# nz+1 in {17,21,25} Chebyshev points, mu ~ U[4.5, 8], seeds 0..31, Gaussian
# noise 1e-3, dt = 0.02, zero flow, L = n/2 (drawn once from default_rng(0)).
def ensemble_runs(n_runs: int = 32):
    rng = np.random.default_rng(0)
    runs = []
    for i in range(n_runs):
        n = int(rng.choice([128, 192, 256]))
        nz = int(rng.choice([17, 21, 25]))
        mu = float(rng.uniform(4.5, 8.0))
        runs.append(dict(nx=n, ny=n, nz=nz, L=n / 2, mu=mu, vy=0.0, dt=0.02,
                         remove_winding=True, noise="complex", amp=1e-3, seed=i))
    return runs


# Algorithmic bytes per site of one launch of each kernel kind (FP64): the
# arrays the kernel must read once and write once.
ALG_BYTES = {"x_rhs": 88, "y_rhs": 112, "zstage": 264, "x_d1": 16, "y_d1": 20,
             "zcons": 40, "zcol_misc": 16, "filter_x_fwd": 96, "filter_y": 96,
             "filter_x_inv": 96}
# compulsory traffic of a whole FP64 step per site: 4*(S_in + S_k) + 2*S_state
STEP_BYTES_FP64 = 4 * (40 + 32) + 2 * 40
# FP64 tensor-core work of the prime-factor line passes (n = 301 = 7*43): one
# 43-point stage A is 144 mma.sync.m8n8k4.f64 per two lines (2 passes x 6
# reduction steps x 2 operand tiles x 3 row tiles x cos/sin), 512 flops each;
# x_rhs runs 6 stage A per line pair, y_rhs 7.  The peak is the mma.sync f64
# throughput measured on B200 at 1965 MHz (37.1 TFLOP/s for the m8n8k4,
# m16n8k4 and m16n8k16 shapes alike).
PFA_DMMA_PER_LINE = {"x_rhs": 6 * 144 / 2, "y_rhs": 7 * 144 / 2}
FP64_TENSOR_TFLOPS = 37.1


def kernel_rows(kernels, tot, sites=None, peak=None):
    """Per-kernel launches, time and share of the step; with ``sites`` and
    ``peak``, also each FP64 kernel's algorithmic GB/s (ALG_BYTES per site x
    sites x launches / time) and its fraction of the HBM peak."""
    rows = {}
    for k in kernels:
        row = {"launches": k["launches"], "ms": round(k["ms"], 4),
               "share": round(k["ms"] / tot, 4)}
        if sites and peak and k["kernel"] in ALG_BYTES and k["ms"] > 0:
            gbs = ALG_BYTES[k["kernel"]] * sites * k["launches"] / (k["ms"] / 1e3) / 1e9
            row["alg_gbs"] = round(gbs, 1)
            row["hbm_frac"] = round(gbs / peak, 4)
        rows[k["kernel"]] = row
    return rows


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, pci_bus_id: str):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", pci_bus_id, "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in Path(self.f.name).read_text().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [c.strip() for c in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_rate(w, nsteps_cap: int, budget_s: float):
    """Site-updates/s of the CPU FP64 restatement of the step in C + OpenMP
    (oracle/hqt_step_omp.c: the reference's dense fourdif/chebdif operators,
    all host cores) on a bounded sample of the workload: whole RK4 steps, up
    to nsteps_cap or budget_s seconds, after one untimed step."""
    import subprocess
    sys.path.insert(0, str(ROOT / "oracle"))
    import hqt_oracle as oracle
    if not (ROOT / "oracle" / "libhqt_oracle_omp.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "-s"], check=True)
    hqt = importlib.import_module(PKG)
    prof = hqt.seed.stationary_profile(w["mu"], w["vy"])
    st = hqt.seed.init_driven(w["nx"], w["ny"], w["nz"], prof, noise=w["noise"],
                              amplitude=w["amp"], seed=w["seed"])
    op = oracle.build_operators(w["nx"], w["ny"], w["nz"], w["L"])
    s, _, _ = oracle.omp_run(op, oracle.OracleState(*st), 1, w["dt"], w["mu"], w["vy"],
                             w["remove_winding"])
    t0 = time.perf_counter()
    n = 0
    while n < max(1, nsteps_cap):
        s, _, _ = oracle.omp_run(op, s, 1, w["dt"], w["mu"], w["vy"], w["remove_winding"])
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or os.cpu_count() or 1
    sites = w["nx"] * w["ny"] * w["nz"]
    return sites * n / dt, n, dt, cores


def host_cpu():
    """CPU model and logical-core count of this host."""
    model = None
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


def bench_config(workload: str, w: dict, ws: int) -> dict:
    """The ``config`` of both arms' JSON lines (same workload, same keys)."""
    sites = w["nx"] * w["ny"] * w["nz"]
    return {"workload": workload, "nx": w["nx"], "ny": w["ny"], "nz": w["nz"],
            "L": w["L"], "mu": w["mu"], "vy": w["vy"], "dt": w["dt"],
            "remove_winding": w["remove_winding"], "filter": True,
            "noise": w["noise"], "amp": w["amp"], "seed": w["seed"],
            "precision": "fp64", "parallelism": f"replicas{ws}",
            "l2": "no flush: one step touches ~%.2f GB of distinct arrays (about 300 B "
                  "per site), %.1fx the 126 MB L2" % (300e-9 * sites, 300 * sites / 126e6)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    return ws, rank, local


def allreduce_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, w, ws, rank):
    if rank != 0:
        return
    budget = max(20.0, 6.0 * args.steps)
    rate, n, dt, cores = oracle_rate(w, args.steps + args.warmup, budget)
    host = host_cpu()
    sample = (f"{n} RK4 steps of the {w['nx']}x{w['ny']}x{w['nz']} workload, CPU FP64 "
              f"restatement of the reference step in C + OpenMP (dense fourdif/chebdif "
              f"operators as the reference applies them), {cores} threads, {dt:.1f} s on "
              f"{host['cpu_model']} ({host['nproc']} logical cores)")
    line = {"metric": "RK4 site-updates/s", "value": rate, "unit": "site-updates/s",
            "n_gpus": args.gpus, "steps": n, "warmup": 0,
            "ms_per_step": 1e3 * dt / n, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": bench_config(args.workload, w, int(os.environ.get("WORLD_SIZE", "1"))),
            "cpu_baseline": {"value": rate, "unit": "site-updates/s", "cores": cores,
                             "kind": "port", "sample": sample, **host},
            "e2e": {"value": rate, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, w, ws, rank, local):
    import torch
    hqt = importlib.import_module(PKG)
    api = importlib.import_module(PKG + ".api")
    dev = local
    torch.cuda.set_device(dev)
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    sites = nx * ny * nz
    prof = hqt.seed.stationary_profile(w["mu"], w["vy"])
    state = hqt.seed.init_driven(nx, ny, nz, prof, noise=w["noise"], amplitude=w["amp"],
                                 seed=w["seed"] + rank)
    sim = hqt.Simulation(nx, ny, nz, Lx=w["L"], Ly=w["L"], mu=w["mu"], vy=w["vy"],
                         dt=w["dt"], remove_winding=w["remove_winding"], device=dev,
                         autotune=not args.no_autotune)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)  # graph capture needs a non-default stream
    T = [api.to_device(a, dev) for a in state]
    # warm-up (also captures the step graph)
    sim.step_device(*T, nsteps=max(args.warmup, 3))
    torch.cuda.synchronize()
    geometry = sim.config_report()  # after the graph build (which may clear "pdl")
    pr = torch.cuda.get_device_properties(dev)
    pci = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    sampler = ClockSampler(pci)
    time.sleep(0.3)
    sim.profile(False)  # reset launch counters, graph replay
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    info = sim.step_device(*T, nsteps=args.steps)
    e1.record()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = allreduce_max(e0.elapsed_time(e1), ws)
    launches = sim.profile_report()["launches"]
    value = ws * sites * args.steps / (ms / 1e3)

    # the mixed-precision variant (FP32 line passes, FP64 columns and state)
    # on the same workload, reported beside the FP64 headline
    mixed = None
    if not args.no_mixed:
        Tm = [api.to_device(a, dev) for a in state]
        with hqt.Simulation(nx, ny, nz, Lx=w["L"], Ly=w["L"], mu=w["mu"], vy=w["vy"],
                            dt=w["dt"], remove_winding=w["remove_winding"], device=dev,
                            precision="mixed", autotune=not args.no_autotune) as simm:
            simm.step_device(*Tm, nsteps=max(args.warmup, 3))
            torch.cuda.synchronize()
            if ws > 1:
                dist.barrier()
            m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            m0.record()
            simm.step_device(*Tm, nsteps=args.steps)
            m1.record()
            torch.cuda.synchronize()
            mms = allreduce_max(m0.elapsed_time(m1), ws)
            simm.profile(True)
            simm.step_device(*Tm, nsteps=min(args.steps, 20))
            mrep = simm.profile_report()
            simm.profile(False)
        del Tm
        mtot = sum(k["ms"] for k in mrep["kernels"])
        mbreak = {k["kernel"]: {"launches": k["launches"], "ms": round(k["ms"], 4),
                                "share": round(k["ms"] / mtot, 4)} for k in mrep["kernels"]}
        mixed = {"value": ws * sites * args.steps / (mms / 1e3), "unit": "site-updates/s",
                 "ms_per_step": mms / args.steps, "steps": args.steps,
                 "dtype": "f32 line passes, f64 column contractions and state",
                 "kernel_breakdown": mbreak}

    # per-kernel CUDA-event timing of the same step sequence (outside the graph)
    kp = min(args.steps, 20)
    sim.profile(True)
    sim.step_device(*T, nsteps=kp)
    rep = sim.profile_report()
    sim.profile(False)
    kern = [k for k in rep["kernels"] if k["kernel"] in ALG_BYTES]
    tot = sum(k["ms"] for k in rep["kernels"])
    top = max(kern, key=lambda k: k["ms"])
    avg_ms = top["ms"] / top["launches"]
    alg = ALG_BYTES[top["kernel"]] * sites
    peak, peak_kind = peaks()
    achieved = alg / (avg_ms / 1e3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "ncu_traffic.json"
    if tf.exists():
        d = json.loads(tf.read_text()).get(args.workload, {})
        traffic = d.get(top["kernel"])
    roofline = {"bound": "hbm", "kernel": top["kernel"], "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind, "traffic": traffic,
                "alg_bytes_per_launch": alg, "avg_launch_ms": avg_ms,
                "share": top["ms"] / tot}
    if nx == 301 and ny == 301 and top["kernel"] in PFA_DMMA_PER_LINE:
        lines = (ny if top["kernel"] == "x_rhs" else nx) * nz
        flops = lines * PFA_DMMA_PER_LINE[top["kernel"]] * 512
        tf = flops / (avg_ms / 1e3) / 1e12
        roofline["fp64_tensor"] = {
            "achieved": tf, "peak": FP64_TENSOR_TFLOPS, "unit": "TFLOP/s",
            "frac": tf / FP64_TENSOR_TFLOPS, "flops_per_launch": flops,
            "peak_source": "mma.sync f64 throughput measured on B200 (probe)"}
    step_gbs = STEP_BYTES_FP64 * sites * args.steps / (ms / 1e3) / 1e9
    breakdown = kernel_rows(rep["kernels"], tot, sites, peak)

    # end to end through the host-array call hqt_step on pinned buffers.  Each
    # call copies the whole state in (Z1..Z4 and rhoi's boundary plane) and
    # out (Z1..Z4 and rhoi replicated along z).  Headline: calls of 50 steps,
    # the reference's checkpoint cadence (tevol_driven_cluster.m:178), where
    # the state has to reach the host for the save; the copies of a call are
    # spread over its 50 steps.  Beside it: calls of one step each.
    pinned = []
    for a, dt_ in zip(state, (torch.complex128,) + (torch.float64,) * 4):
        t = torch.empty((nz, ny, nx), dtype=dt_, pin_memory=True)
        t.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)))
        pinned.append(t)
    H = [t.numpy().T for t in pinned]
    h2d_call = (16 + 24) * sites + 8 * nx * ny
    d2h_call = (16 + 24 + 8) * sites

    def e2e_rate(per_call, calls):
        sim.step(*H, nsteps=per_call, inplace=True)  # warm the host path
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(calls):
            sim.step(*H, nsteps=per_call, inplace=True)
        torch.cuda.synchronize()
        e2e_s = allreduce_max(time.perf_counter() - t0, ws)
        return ws * sites * per_call * calls / e2e_s

    e2e = None
    if not args.no_e2e:
        per_call = 50
        calls = max(1, int(round(args.steps / per_call)))
        e2e = {"value": e2e_rate(per_call, calls), "unit": "site-updates/s",
               "h2d_bytes_per_step": h2d_call / per_call,
               "d2h_bytes_per_step": d2h_call / per_call,
               "h2d_bytes_per_call": h2d_call, "d2h_bytes_per_call": d2h_call,
               "steps_per_call": per_call,
               "step": f"hqt_step calls of {per_call} RK4 steps on pinned host arrays, "
                       f"{calls} calls timed; per-step bytes are the per-call copies / "
                       f"{per_call}"}
        n1 = min(50, args.steps)
        e2e["single_step_calls"] = {
            "value": e2e_rate(1, n1), "unit": "site-updates/s",
            "h2d_bytes_per_step": h2d_call, "d2h_bytes_per_step": d2h_call,
            "step": f"{n1} hqt_step calls of one RK4 step each: the whole state "
                    f"copied in and out every step"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        rate, n, dt_s, cores = oracle_rate(w, 8, 20.0)
        host = host_cpu()
        cpu = {"value": rate, "unit": "site-updates/s", "cores": cores, "kind": "port",
               "sample": f"{n} RK4 steps of {nx}x{ny}x{nz}, CPU FP64 restatement in C + "
                         f"OpenMP (dense fourdif/chebdif as the reference applies them), "
                         f"{cores} threads, {dt_s:.1f} s",
               **host}
    sim.close()
    if rank == 0:
        line = {"metric": "RK4 site-updates/s", "value": value, "unit": "site-updates/s",
                "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (Newton stationary profile + seeded complex noise)",
                "config": bench_config(args.workload, w, ws),
                "gpu_launches": launches, "roofline": roofline,
                "line_geometry": geometry.get("chosen"),
                "programmatic_dependent_launch": geometry.get("pdl"),
                "step_hbm": {"alg_bytes_per_site": STEP_BYTES_FP64, "achieved_gbs": step_gbs,
                             "frac": step_gbs / peak},
                "kernel_breakdown": breakdown, "mixed_precision": mixed,
                "e2e": e2e, "cpu_baseline": cpu,
                "clocks": clocks, "nonfinite_step": info.nonfinite_step}
        print(json.dumps(line), flush=True)


def run_ensemble(args, ws, rank, local):
    """The batched ensemble: runs bin-packed over ranks (no data-path
    collective), each rank advancing its runs with one graph launch per
    step.  value = site-updates of all runs / max-over-ranks device time."""
    import torch
    hqt = importlib.import_module(PKG)
    api = importlib.import_module(PKG + ".api")
    torch.cuda.set_device(local)
    runs = ensemble_runs()
    costs = [r["nx"] * r["ny"] * r["nz"] for r in runs]
    mine = hqt.assign_runs(costs, ws)[rank]
    stream = torch.cuda.Stream(local)
    torch.cuda.set_stream(stream)
    sims, T = [], []
    for i in mine:
        r = runs[i]
        prof = hqt.seed.stationary_profile(r["mu"], r["vy"])
        st = hqt.seed.init_driven(r["nx"], r["ny"], r["nz"], prof, noise=r["noise"],
                                  amplitude=r["amp"], seed=r["seed"])
        sims.append(hqt.Simulation(r["nx"], r["ny"], r["nz"], Lx=r["L"], Ly=r["L"],
                                   mu=r["mu"], vy=r["vy"], dt=r["dt"],
                                   remove_winding=r["remove_winding"], device=local,
                                   autotune=not args.no_autotune))
        T.append([api.to_device(a, local) for a in st])
    ens = hqt.Ensemble(sims)
    ens.step_device(T, nsteps=max(args.warmup, 3))
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    pr = torch.cuda.get_device_properties(local)
    sampler = ClockSampler(f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0")
    time.sleep(0.3)
    for s in sims:
        s.profile(False)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.step_device(T, nsteps=args.steps)
    e1.record()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = allreduce_max(e0.elapsed_time(e1), ws)
    launches = sum(s.profile_report()["launches"] for s in sims)
    ens.close()
    for s in sims:
        s.close()
    total = sum(costs)
    value = total * args.steps / (ms / 1e3)
    peak, peak_kind = peaks()
    step_gbs = STEP_BYTES_FP64 * total * args.steps / (ms / 1e3) / 1e9
    if rank == 0:
        line = {"metric": "RK4 site-updates/s", "value": value, "unit": "site-updates/s",
                "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (Newton stationary profile per mu + seeded complex noise)",
                "config": {"workload": "ensemble32", "runs": len(runs),
                           "grids": sorted({r["nx"] for r in runs}),
                           "nz": sorted({r["nz"] for r in runs}),
                           "mu_range": [4.5, 8.0], "total_sites": total,
                           "runs_per_rank": [len(a) for a in hqt.assign_runs(costs, ws)],
                           "parallelism": f"runs bin-packed over {ws} GPU(s)",
                           "launch": "one CUDA-graph launch per step per GPU",
                           "l2": "no flush: the ensemble touches ~9 GB per step"},
                "gpu_launches": launches, "roofline": None,
                "step_hbm": {"alg_bytes_per_site": STEP_BYTES_FP64, "achieved_gbs": step_gbs,
                             "frac": step_gbs / peak, "peak_source": peak_kind},
                "e2e": None, "cpu_baseline": None, "clocks": clocks}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="driven301",
                    choices=sorted(WORKLOADS) + ["ensemble32"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-array leg")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision variant")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default line-pass geometry (no tuning launches)")
    args = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    if args.workload == "ensemble32":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the ensemble workload has no CPU reference arm; "
                              "the reference runs one simulation per session"}))
            return
        ws, rank, local = dist_init()
        try:
            run_ensemble(args, ws, rank, local)
        finally:
            if ws > 1:
                import torch.distributed as dist
                dist.destroy_process_group()
        return
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        # the CPU reference runs on rank 0 only; other ranks exit at once
        run_reference(args, w, int(os.environ.get("WORLD_SIZE", "1")),
                      int(os.environ.get("RANK", "0")))
        return
    ws, rank, local = dist_init()
    try:
        run_ours(args, w, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
