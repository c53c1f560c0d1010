#!/usr/bin/env python
"""Benchmark of the isothermal-MHD time step on B200 (one JSON line on rank 0).

Workload (one box per GPU, weak scaling): driven isothermal-MHD turbulence on
a 512^3 periodic box, FP32 bulk arithmetic, van Leer predictor-corrector with
characteristic PLM reconstruction, Roe fluxes and constrained transport, two
passive scalars, rho = 1, cs = 1, B0 = (0.5, 0, 0), initial velocity one
realisation of the solenoidal OU forcing field (shells 1 <= |k| <= 2) at rms
Mach 2, forcing kicks on the reference schedule (dt_turb = 0.05), COUR 0.4.
Synthetic, seeded inputs stand in for the reference's runs.

A step is one call of imhd_step (the reference's copy_velocity +
vanleer_solve_3d + passive_solve_3d + periodic fill + new dt).  Metric:
cell-updates/s = N^3 * steps * ranks / max-over-ranks device time.

  python bench.py [--gpus N --steps K --warmup W]      # our CUDA path
  python bench.py --impl reference                     # CPU restatement of the reference
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
WORKLOAD = ("driven MHD turbulence 512^3 periodic box, FP32 van Leer + PLM-char + Roe + CT, "
            "2 passive scalars, Mach 2 OU forcing, B0=(0.5,0,0), COUR 0.4")


def workload_name(a):
    if (a.n, a.riemann, a.recon, a.npass, a.mach, a.b0x, a.precision) == (512, "roe", "plm", 2, 2.0, 0.5, 32):
        return WORKLOAD
    return ("driven MHD turbulence %d^3 periodic box, FP%d van Leer + %s-char + %s + CT, %d passive scalars, "
            "Mach %g OU forcing, B0=(%g,0,0), COUR %g" % (a.n, a.precision, a.recon.upper(),
                                                           {"roe": "Roe"}.get(a.riemann, a.riemann.upper()),
                                                           a.npass, a.mach, a.b0x, a.cour))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--riemann", default="roe")
    ap.add_argument("--recon", default="plm", choices=["plm", "ppm"])
    ap.add_argument("--precision", type=int, default=32)
    ap.add_argument("--npass", type=int, default=2)
    ap.add_argument("--mach", type=float, default=2.0)
    ap.add_argument("--b0x", type=float, default=0.5, help="uniform field B0 = (b0x, 0, 0)")
    ap.add_argument("--edot", type=float, default=4.0)
    ap.add_argument("--cour", type=float, default=0.4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-n", type=int, default=128, help="edge of the CPU sample box")
    ap.add_argument("--ref-steps", type=int, default=None)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--batched", type=int, default=512,
                    help="boxes of the mixed-size batch measured beside the main line (0: skip)")
    ap.add_argument("--batched-steps", type=int, default=50)
    ap.add_argument("--served", type=int, default=400,
                    help="requests of the Poisson stream through the serving loop (0: skip)")
    ap.add_argument("--rate", type=float, default=200.0, help="mean arrival rate of the stream, requests/s")
    ap.add_argument("--hbm-budget", type=float, default=150e9)
    ap.add_argument("--accuracy", type=int, default=0,
                    help="instead of timing: run the workload this many steps in FP64 and in FP32 (same dt "
                         "sequence) and print relative L1 / Linf per field and max |div B|")
    ap.add_argument("--loop-sample", type=int, default=128,
                    help="boxes of the per-box loop arms, the first of the batch (0: all)")
    return ap.parse_args()


# ----------------------------------------------------------------- distributed
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws <= 1:
        return None
    import datetime
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, init_method="env://", timeout=datetime.timedelta(seconds=300))
    return dist


def max_over_ranks(dist, value, device=None):
    """Largest `value` over the ranks of the job (the job's time is its
    slowest rank's); the value itself without a process group."""
    if not dist:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, ranks, ms_max):
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return units_per_rank * ranks / (ms_max / 1e3)


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-i", str(self.idx),
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("swp", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows),
                "power_w_max": max(r["power"] for r in rows)}


# ----------------------------------------------------------------- workload
def make_initial_state(n, mach, npass, seed, b0x=0.5):
    from isothermal_mhd_b200 import forcing
    f = forcing.OUForcing(n, seed=seed)
    q, b, p = forcing.turbulent_box(n, mach=mach, b0=(b0x, 0.0, 0.0), npass=npass, seed=seed, forcing=f)
    f.advance(0.05)
    delv = f.field(rms=1.0)
    return q, b, p, delv, f


def stage_bytes(esz, npass):
    """Compulsory HBM bytes per cell of each stage (reads + writes once)."""
    return {
        "pred_flux": 28 * esz,            # 7 state + 3 face fields in; 6 fluxes out per face direction
        "pred_emf": 16 * esz,             # rho, m, B_cc, 6 face EMFs in; 3 corner EMFs out
        "pred_update": 32 * esz,          # 7 state + 12 fluxes + 3 EMFs in; 10 fields out
        "corr_flux_x": 13 * esz, "corr_flux_y": 13 * esz, "corr_flux_z": 13 * esz,
        "corr_emf": 16 * esz,
        "final_update": 32 * esz,
        "passive_pred": (4 + 2 * npass) * esz,
        "passive_corr": (8 + 3 * npass) * esz,
        "force_sums": 7 * esz, "force_kick": 12 * esz, "finalize": 0,
    }


# DRAM bytes per cell of one launch (dram__bytes_read.sum + dram__bytes_write.sum over the cells of the
# launch) from an ncu capture at 256^3 of the same kernel and scheme; traffic grows with the cell count,
# so a launch at n^3 moves about n^3 times this.  Keyed by (stage, precision, riemann, recon).
NCU_TRAFFIC_PER_CELL = {
    ("pred_flux", 32, "roe", "plm"): (677.4e6 + 1161.1e6) / 256 ** 3,
    # the update does not depend on the solver or the reconstruction (mean of the two launches of a step)
    ("update", 32): (1493.5e6 + 646.7e6 + 1492.8e6 + 644.9e6) / 2 / 256 ** 3,
}

# step stages that are launches of one kernel: the roofline reports the kernel
# with the most device time per step, at its mean launch duration
KERNEL_STAGES = {"update": ("pred_update", "final_update"), "corner_emf": ("pred_emf", "corr_emf")}


def run_ours(a, ws, rank, local):
    import torch
    from isothermal_mhd_b200 import Box, driver

    dist = init_dist(ws, "nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = a.n
    q, b, p, delv, f = make_initial_state(n, a.mach, a.npass, a.seed + rank, a.b0x)
    box = Box(n, precision=a.precision, riemann=a.riemann, recon=a.recon, npass=a.npass, cour=a.cour, edot=a.edot,
              dt_turb=0.05, device=local)
    stream = torch.cuda.current_stream(dev)
    box.set_stream(stream.cuda_stream)
    box.upload(q, b, p)
    box.set_force(delv)

    # the reference driver loop (driver.f90:35-186): dt0 = 1e-15, drive when due
    state = {"t": 0.0, "dt": 1e-15, "t_turb": 0.05, "drives": 0}

    def one_step():
        t_old, dt = state["t"], state["dt"]
        drive = (state["t_turb"] > t_old) and (state["t_turb"] <= t_old + dt)
        if drive:
            state["t_turb"] = max(state["t_turb"] + 0.05, t_old + 1e-2 * dt)
            dt = 0.5 * dt
        dt_new = box.step(dt, drive)
        state["t"] = t_old + dt
        if drive:
            state["drives"] += 1
            box.set_force(delv)
        state["dt"] = dt_new

    for _ in range(a.warmup):
        one_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    box.profile(True)
    box.stage_times(reset=True)
    launches0 = box.launch_count
    drives0 = state["drives"]
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(a.steps):
        one_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches = box.launch_count - launches0
    stages = box.stage_times()
    box.profile(False)
    t_max = max_over_ranks(dist, ms, dev)
    cells = n ** 3
    value = job_rate(cells * a.steps, ws, t_max)

    # ---- end to end through the C ABI with host buffers: pinned host state in,
    # K steps (dt in, dt_next out each step), host state out
    e2e = None
    if not a.no_e2e:
        hq = torch.empty(q.shape, dtype=torch.float64, pin_memory=True).numpy()
        hb = torch.empty(b.shape, dtype=torch.float64, pin_memory=True).numpy()
        hp = torch.empty(p.shape, dtype=torch.float64, pin_memory=True).numpy()
        hq[...] = q
        hb[...] = b
        hp[...] = p
        state.update(t=0.0, dt=1e-15, t_turb=0.05)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        box.upload(hq, hb, hp)
        for _ in range(a.steps):
            one_step()
        box.download(hq, hb, hp)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(dist, e0.elapsed_time(e1), dev)
        state_bytes = hq.nbytes + hb.nbytes + hp.nbytes
        e2e = {"value": cells * a.steps * ws / (ems / 1e3), "unit": METRIC,
               "h2d_bytes_per_step": int(state_bytes / a.steps + 8),
               "d2h_bytes_per_step": int(state_bytes / a.steps + 12),
               "ms_total": ems, "includes": "pinned host upload + K imhd_step calls + host download"}
        del hq, hb, hp

    # ---- roofline of the dominant kernel (device time from CUDA events on the launching stream)
    import json as _json
    peaks = {}
    try:
        peaks = _json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    esz = 4 if a.precision == 32 else 8
    sb = stage_bytes(esz, a.npass)
    per_stage = {}
    for name, (tot, cnt) in stages.items():
        if cnt:
            per_stage[name] = {"ms_per_launch": tot / cnt, "share": None,
                               "gbs_alg": (sb.get(name, 0) * cells / 1e9) / (tot / cnt / 1e3) if tot > 0 else None}
    total_stage_ms = sum(v["ms_per_launch"] for v in per_stage.values())
    for v in per_stage.values():
        v["share"] = v["ms_per_launch"] / total_stage_ms if total_stage_ms else None
    # per kernel: its stages' launch times (the update and the corner EMF run twice a step)
    kernels = {}
    grouped = {st for sts in KERNEL_STAGES.values() for st in sts}
    for kname, sts in KERNEL_STAGES.items():
        ms = [per_stage[st]["ms_per_launch"] for st in sts if st in per_stage]
        if ms:
            kernels[kname] = (sum(ms), sum(ms) / len(ms), sb[sts[0]])
    for name, v in per_stage.items():
        if name not in grouped:
            kernels[name] = (v["ms_per_launch"], v["ms_per_launch"], sb.get(name, 0))
    dom = max(kernels, key=lambda k: kernels[k][0])
    _, dom_ms, dom_bytes = kernels[dom]
    achieved = dom_bytes * cells / 1e9 / (dom_ms / 1e3)
    tpc = NCU_TRAFFIC_PER_CELL.get((dom, a.precision, a.riemann, a.recon), NCU_TRAFFIC_PER_CELL.get((dom, a.precision)))
    traffic = tpc * cells if tpc is not None else None
    roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": traffic,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s",
                "algorithmic_bytes_per_launch": dom_bytes * cells, "ms_per_launch": dom_ms,
                "ms_per_step": kernels[dom][0]}

    # the batched and served workloads are single-GPU measurements: with
    # several ranks (replicas of the headline box) they are left out
    batched = served = None
    extras = ws == 1 and (a.batched > 0 or a.served > 0)
    if extras:
        box.close()
        box = None
    if extras and a.batched > 0:
        batched = run_batched(a, local, stream, dist, dev)
    if extras and a.served > 0:
        served = run_served(a, local)

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        cpu = cpu_reference_sample(a, n_sample=a.ref_n, steps=a.ref_steps or 3, warmup=1)

    if box is not None:
        box.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": t_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if a.precision == 32 else "f64", "data": "synthetic (seeded OU turbulence)",
        "config": {"workload": workload_name(a), "n": n, "precision": a.precision, "riemann": a.riemann,
                   "recon": a.recon + "-char", "npass": a.npass, "mach": a.mach, "edot": a.edot, "cour": a.cour,
                   "parallelism": f"replicas x{ws}", "l2": "inputs larger than L2 (state %.1f GB)" %
                   ((10 + a.npass) * cells * esz / 1e9), "drive_steps_timed": state["drives"] - drives0},
        "gpu_launches": launches,
        "roofline": roofline,
        "stages": per_stage,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "clocks": clk,
        "batched": batched,
        "served": served,
    }
    return line


# ----------------------------------------------------------------- mixed-size batch
def _build_box(obj, spec, i=None):
    kv, av, sv, af, sf = spec.fields()
    args = (i,) if i is not None else ()
    obj.init_uniform(*args, rho=1.0, b0=spec.b0)
    obj.fourier_field(*args, "velocity", kv, av, sv)
    obj.fourier_field(*args, "force", kv, af, sf)


def run_batched(a, local, stream, dist, dev):
    """Mixed-size batch (512 boxes, edges U{32,48,64,96,128}, |B0| U[0.1,2],
    Mach U[0.5,5], FP32 Roe + CT, 50 steps each, forcing on) through
    imhd_batch_run, against the plain per-box loop of imhd_step calls with
    the host driver loop.  Returns boxes/s and cell-updates/s of both arms."""
    import torch
    from isothermal_mhd_b200 import Batch, Box, ImhdError, driver, workloads
    from isothermal_mhd_b200.batch import make_config

    specs = workloads.batched_boxes(a.batched, steps=a.batched_steps, seed=a.seed)
    cfgs = [make_config(s.n, precision=32, riemann=s.riemann, npass=s.npass, cour=a.cour, edot=s.edot,
                        dt_turb=s.dt_turb, device=local) for s in specs]
    cells_steps = sum(s.cells * s.steps for s in specs)
    out = {"workload": "%d boxes, edges U{32,48,64,96,128}, |B0| U[0.1,2] random direction, rms Mach U[0.5,5], "
                       "edot = Mach^3, FP32 Roe + PLM-char + CT, %d steps each, forcing on" % (len(specs),
                                                                                           a.batched_steps),
           "boxes": len(specs), "cells": sum(s.cells for s in specs)}
    bt = Batch(cfgs)
    bt.set_stream(stream.cuda_stream)

    def setup():
        for i, s in enumerate(specs):
            _build_box(bt, s, i)
            bt.schedule(i, s.steps, forcing=True)

    setup()
    bt.run(1)               # captures the step graph
    setup()
    launches0 = bt.launch_count
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    bt.run(a.batched_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = [bt.clock(i) for i in range(len(specs))]
    failed = [i for i, c in enumerate(clocks) if c["failed"]]
    sample = [i for i in range(len(specs)) if i not in failed][:4]
    batch_states = {i: bt.download(i) for i in sample}
    done = sum(1 for c in clocks if not c["active"] and not c["failed"])
    out["batch"] = {"ms": ms, "boxes_per_s": len(specs) / (ms / 1e3), "cell_updates_per_s": cells_steps / (ms / 1e3),
                    "boxes_completed": done, "boxes_failed": len(failed),
                    "graph_replays": a.batched_steps,
                    "gpu_launches": bt.launch_count - launches0}
    bt.close()
    del bt

    # plain per-box loops: one Box at a time, the host driver loop over
    # imhd_step; FP64 is the plain method, FP32 the same loop at the batch's
    # precision.  Both run the first `loop_sample` boxes (a random sample).
    nloop = min(a.loop_sample or len(specs), len(specs))
    sample_cells_steps = sum(s.cells * s.steps for s in specs[:nloop])
    for prec in (64, 32):
        loop_ms = 0.0
        l1 = {}
        nfail = 0
        for i, s in enumerate(specs[:nloop]):
            box = Box(s.n, precision=prec, riemann=s.riemann, npass=s.npass, cour=a.cour, edot=s.edot,
                      dt_turb=s.dt_turb, device=local)
            box.set_stream(stream.cuda_stream)
            _build_box(box, s)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            try:
                driver.run(box, t_end=1e30, maxsteps=s.steps + 1, forcing="device", dt_turb=s.dt_turb,
                           record_dt=False)
            except ImhdError:
                nfail += 1          # NaN / zero speed: the box stops, as in the batch
            torch.cuda.synchronize()
            loop_ms += (time.perf_counter() - t0) * 1e3
            if i in batch_states:
                qa, ba, _ = box.download()
                qb, bb, _ = batch_states[i]
                # relative L1 per field of the FP32 batch against this loop
                for f, (u, v) in enumerate([(qb[k], qa[k]) for k in range(7)] + [(bb[k], ba[k]) for k in range(3)]):
                    den = float(np.sum(np.abs(v)))
                    err = float(np.sum(np.abs(u - v)) / den) if den > 0 else float(np.sum(np.abs(u - v)))
                    l1[f] = max(l1.get(f, 0.0), err)
            box.close()
        names = ["rho", "mx", "my", "mz", "bx_cc", "by_cc", "bz_cc", "bx_face", "by_face", "bz_face"]
        out["per_box_loop_fp%d" % prec] = {
            "ms": loop_ms, "boxes": nloop, "boxes_failed": nfail, "boxes_per_s": nloop / (loop_ms / 1e3),
            "cell_updates_per_s": sample_cells_steps / (loop_ms / 1e3),
            "batch_rel_l1_max_over_sample": {names[k]: v for k, v in l1.items()},
            "timing": "host wall clock around each box's step loop (device synchronised)"}
        out["speedup_vs_fp%d_loop" % prec] = out["batch"]["boxes_per_s"] / out["per_box_loop_fp%d" % prec]["boxes_per_s"]
    return out


# ----------------------------------------------------------------- serving loop
def run_served(a, local):
    """Poisson stream of box-solve requests (edges {32,64,96,128,192} weighted
    0.35/0.30/0.20/0.10/0.05, steps U[20,200], Roe or HLLD, |B0| U[0.1,2],
    Mach U[0.5,5], forcing on) served by imhd_server with continuous batching
    under the HBM budget; boxes/s, cell-updates/s and p50/p99 latency from
    submission to the result in host memory.  The first requests of the same
    stream are also served one at a time by the plain per-box loop."""
    import threading

    import torch
    from isothermal_mhd_b200 import Box, ImhdError, driver, workloads
    from isothermal_mhd_b200.server import Server

    stream_ = workloads.request_stream(a.served, rate=a.rate, seed=a.seed + 1)
    specs = stream_.specs
    srv = Server(precision=32, hbm_budget=a.hbm_budget, steps_per_round=4, device=local)
    # warm-up: kernels loaded, first graph captured
    warm = [srv.submit(workloads.BoxSpec(n=16, b0=(0.5, 0, 0), mach=1.0, steps=3, seed=1, riemann=r))
            for r in ("roe", "hlld")]
    for rid in warm:
        while srv.poll(rid, fetch=True)[0] != "done":
            time.sleep(0.001)
    ids = [None] * len(specs)
    t_start = time.perf_counter()

    def submitter():
        for i, s in enumerate(specs):
            dt = t_start + s.arrival - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            ids[i] = srv.submit(s)

    th = threading.Thread(target=submitter)
    th.start()
    lat, wait_s, failed = {}, {}, []
    t_last = t_start
    while len(lat) < len(specs):
        for i in range(len(specs)):
            if i in lat or ids[i] is None:
                continue
            state, info, _ = srv.poll(ids[i], fetch=True)
            if state in ("done", "failed"):
                lat[i] = info["latency_s"]
                wait_s[i] = info["queue_wait_s"]
                t_last = time.perf_counter()
                if state == "failed":
                    failed.append(i)
        time.sleep(0.002)
    th.join()
    stats = srv.stats()
    srv.stop(drain=True)
    srv.close()
    elapsed = t_last - t_start
    lats = np.array([lat[i] for i in range(len(specs))])
    cells_steps = sum(s.cells * s.steps for s in specs)
    out = {"workload": "%d requests, Poisson %.0f req/s, edges {32,64,96,128,192} p=0.35/0.30/0.20/0.10/0.05, "
                       "steps U[20,200], Roe/HLLD 1:1, |B0| U[0.1,2], Mach U[0.5,5], FP32, forcing on, "
                       "HBM budget %.0f GB" % (len(specs), a.rate, a.hbm_budget / 1e9),
           "requests": len(specs), "requests_failed": len(failed), "elapsed_s": elapsed,
           "arrival_span_s": specs[-1].arrival,
           "boxes_per_s": len(specs) / elapsed, "cell_updates_per_s": cells_steps / elapsed,
           "latency_s": {"p50": float(np.percentile(lats, 50)), "p99": float(np.percentile(lats, 99)),
                         "mean": float(lats.mean()), "max": float(lats.max())},
           "queue_wait_s": {"p50": float(np.percentile([wait_s[i] for i in wait_s], 50)),
                            "p99": float(np.percentile([wait_s[i] for i in wait_s], 99))},
           "server": stats}
    # plain per-box loops over the first requests of the stream, one at a time
    nloop = min(a.loop_sample or len(specs), len(specs), 64)
    for prec in (64, 32):
        tot = 0.0
        nfail = 0
        for s in specs[:nloop]:
            kv, av, sv, af, sf = s.fields()
            box = Box(s.n, precision=prec, riemann=s.riemann, npass=s.npass, cour=a.cour, edot=s.edot,
                      dt_turb=s.dt_turb, device=local)
            t0 = time.perf_counter()
            box.init_uniform(1.0, s.b0)
            box.fourier_field("velocity", kv, av, sv)
            box.fourier_field("force", kv, af, sf)
            dt0 = a.cour * box.dx / box.max_speed()
            try:
                driver.run(box, t_end=1e30, maxsteps=s.steps + 1, dt0=dt0, forcing="device", dt_turb=s.dt_turb,
                           record_dt=False)
            except ImhdError:
                nfail += 1
            box.download()
            torch.cuda.synchronize()
            tot += time.perf_counter() - t0
            box.close()
        out["per_box_loop_fp%d" % prec] = {
            "requests": nloop, "requests_failed": nfail, "boxes_per_s": nloop / tot,
            "cell_updates_per_s": sum(s.cells * s.steps for s in specs[:nloop]) / tot,
            "timing": "host wall clock per request: build, step loop, download (one request at a time)"}
        # the sample's mix differs from the stream's: compare the time each
        # would take for the whole stream's work
        sample_work = sum(s.cells * s.steps for s in specs[:nloop])
        loop_time_stream = tot * cells_steps / sample_work
        out["per_box_loop_fp%d" % prec]["est_s_for_stream"] = loop_time_stream
        out["speedup_vs_fp%d_loop" % prec] = loop_time_stream / elapsed
    return out


# ----------------------------------------------------------------- FP32 vs FP64
def run_accuracy(a, local):
    """The bench workload (or --n / --riemann / --recon / --npass variants)
    advanced `a.accuracy` steps in FP64 on the reference driver schedule, then
    in FP32 with the FP64 run's dt and drive sequence; relative L1 and Linf
    of every field of the FP32 state against the FP64 one, and max |div B|
    (face differences per cell) of both."""
    import torch
    from isothermal_mhd_b200 import Box

    n = a.n
    q, b, p, delv, f = make_initial_state(n, a.mach, a.npass, a.seed, a.b0x)

    def run(prec, plan=None):
        box = Box(n, precision=prec, riemann=a.riemann, recon=a.recon, npass=a.npass, cour=a.cour, edot=a.edot,
                  dt_turb=0.05, device=local)
        box.upload(q, b, p)
        box.set_force(delv)
        t, dt, t_turb, rec = 0.0, 1e-15, 0.05, []
        t0 = time.perf_counter()
        for s in range(a.accuracy):
            if plan is None:
                drive = (t_turb > t) and (t_turb <= t + dt)
                if drive:
                    t_turb = max(t_turb + 0.05, t + 1e-2 * dt)
                    dt = 0.5 * dt
            else:
                dt, drive = plan[s]
            rec.append((dt, drive))
            dt_new = box.step(dt, drive)
            t += dt
            dt = dt_new
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        out = box.download()
        st = box.status()
        box.close()
        return out, rec, el, st

    (q64, b64, p64), plan, el64, st64 = run(64)
    (q32, b32, p32), _, el32, st32 = run(32, plan)
    names = ["rho", "mx", "my", "mz", "bx_cc", "by_cc", "bz_cc"]
    fields = {}
    for k in range(7):
        fields[names[k]] = (q32[k], q64[k])
    for k, nm in enumerate(("bx_face", "by_face", "bz_face")):
        fields[nm] = (b32[k], b64[k])
    for k in range(a.npass):
        fields["pass%d" % k] = (p32[k], p64[k])
    err = {}
    for nm, (u, v) in fields.items():
        d = np.abs(u - v)
        den = float(np.sum(np.abs(v)))
        err[nm] = {"rel_l1": float(np.sum(d) / den) if den > 0 else float(np.sum(d)),
                   "rel_linf": float(np.max(d) / np.max(np.abs(v))) if np.max(np.abs(v)) > 0 else float(np.max(d))}

    def max_div(bf):
        d = (bf[0] - np.roll(bf[0], 1, axis=2)) + (bf[1] - np.roll(bf[1], 1, axis=1)) + (bf[2] - np.roll(bf[2], 1, axis=0))
        return float(np.max(np.abs(d)))

    return {"metric": "fp32_vs_fp64", "n": n, "steps": a.accuracy, "riemann": a.riemann, "recon": a.recon,
            "npass": a.npass, "mach": a.mach, "drive_steps": sum(1 for _, dr in plan if dr),
            "fields": err, "max_rel_l1": max(v["rel_l1"] for v in err.values()),
            "max_abs_divB": {"fp64": max_div(b64), "fp32": max_div(b32)},
            "status": {"fp64": st64, "fp32": st32}, "wall_s": {"fp64": el64, "fp32": el32},
            "note": "FP32 run replays the FP64 run's dt and drive sequence"}


# ----------------------------------------------------------------- CPU reference
def cpu_reference_sample(a, n_sample, steps, warmup):
    """The CPU restatement of the reference (oracle, FP64, all host threads) on
    an n_sample^3 box of the same physics; cell-updates/s over `steps` steps."""
    from oracle.pyoracle import Oracle
    threads = os.cpu_count() or 1
    q, b, p, delv, f = make_initial_state(n_sample, a.mach, a.npass, a.seed)
    o = Oracle(n_sample, riemann=a.riemann, npass=a.npass, nthreads=threads)
    o.set_state(q, b, p)
    o.set_force(delv, edot=a.edot, dt_turb=0.05)
    dt = 1e-15
    for _ in range(warmup):
        dt = a.cour * o.dx / o.step(dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        dt = a.cour * o.dx / o.step(dt)
    el = time.perf_counter() - t0
    o.close()
    v = n_sample ** 3 * steps / el
    return {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{n_sample}^3 box of the same physics (FP64), {steps} steps after {warmup} warm-up, "
                      f"{el:.1f} s; C++ restatement of the reference algorithm (the Fortran build is "
                      f"unavailable: no Fortran compiler or MPI in the image)"}


def run_reference(a, ws, rank):
    if rank != 0:
        return None
    steps = a.ref_steps or max(1, min(a.steps, 10))
    cpu = cpu_reference_sample(a, n_sample=a.ref_n, steps=steps, warmup=max(1, min(a.warmup, 2)))
    v = cpu["value"]
    return {
        "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": ws, "steps": steps, "warmup": a.warmup,
        "ms_per_step": (a.ref_n ** 3) / v * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded OU turbulence)", "impl": "reference",
        "config": {"workload": WORKLOAD, "n": a.n, "sample_n": a.ref_n, "riemann": a.riemann, "npass": a.npass,
                   "parallelism": "host threads"},
        "cpu_baseline": cpu,
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    a = parse()
    ws, rank, local = dist_env()
    if a.impl == "reference":
        line = run_reference(a, ws, rank)
    elif a.accuracy > 0:
        line = run_accuracy(a, local) if rank == 0 else None
    else:
        line = run_ours(a, ws, rank, local)
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
