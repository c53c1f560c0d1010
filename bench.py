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
  python bench.py --gpus N --split slabs               # one box over N GPUs
  python bench.py --impl reference                     # CPU restatement of the reference

With --gpus N > 1 and no torchrun environment the script starts its N ranks
itself (one process per GPU, NCCL).
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


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=None,
                    help="GPUs (ranks) of the job; default: WORLD_SIZE of a torchrun launch, else 1")
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
    ap.add_argument("--accuracy-steps", type=int, default=100,
                    help="steps of the FP32-vs-FP64 accuracy leg of the default run (0: skip)")
    ap.add_argument("--split", choices=["replicas", "slabs"], default="replicas",
                    help="multi-GPU mode: one box per GPU (weak scaling) or one box in z slabs over the GPUs "
                         "(strong scaling)")
    ap.add_argument("--rate-low", type=float, default=20.0,
                    help="arrival rate of a second, sub-saturating served stream (0: skip)")
    ap.add_argument("--served-low", type=int, default=100, help="requests of the sub-saturating stream")
    ap.add_argument("--loop-sample", type=int, default=128,
                    help="boxes of the per-box loop arms, the first of the batch (0: all)")
    ap.add_argument("--no-loops", action="store_true",
                    help="skip the per-box loop arms of the batched and served workloads")
    ap.add_argument("--dist-check", action="store_true", help=argparse.SUPPRESS)   # launcher self-test (gloo)
    return ap.parse_args(argv)


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
        "final_update": 35 * esz,         # and the passive corrector's 3 time-averaged velocities out
        "passive_pred": (4 + 2 * npass) * esz,
        "passive_corr": (3 + 3 * npass) * esz,   # 3 velocities, half-step and step-start scalars in; scalars out
        "force_sums": 7 * esz, "force_kick": 12 * esz, "finalize": 0,
    }


# DRAM bytes per cell of one launch (dram__bytes_read.sum + dram__bytes_write.sum over the cells of the
# launch) from an ncu capture at 256^3 of the same kernel and scheme; traffic grows with the cell count,
# so a launch at n^3 moves about n^3 times this.  Keyed by (stage, precision, riemann, recon).
NCU_TRAFFIC_PER_CELL = {
    ("pred_flux", 32, "roe", "plm"): (677.4e6 + 1161.1e6) / 256 ** 3,
    # the update does not depend on the solver or the reconstruction (mean of the two launches of a step;
    # the final one also writes the passive corrector's three velocities)
    ("update", 32): (1493.0e6 + 644.8e6 + 1494.1e6 + 840.3e6) / 2 / 256 ** 3,
}

# step stages that are launches of one kernel: the roofline reports the kernel
# with the most device time per step, at its mean launch duration
KERNEL_STAGES = {"update": ("pred_update", "final_update"), "corner_emf": ("pred_emf", "corr_emf")}

# Arithmetic of the reference algorithm per interior cell-update of an
# undriven step: additions/subtractions, multiplications, divisions, square
# roots, comparisons (MAX/MIN, limiter and upwind tests), ABS and SIGN, one op
# each.  Tallied by the op-counting build of the FP64 restatement
# (oracle/count_ops.py -> oracle/op_counts.json; a CPU test holds this table
# equal to that file): the cubic fit over edges 16..32 of a step's tally, whose
# leading coefficient is the per-cell work without the reference's ghost-zone
# recomputation.  Keyed by (riemann, reconstruction, passive scalars).
ALG_OPS_PER_CELL = {
    ("roe", "plm", 0): 5646.8, ("roe", "plm", 2): 5904.8, ("roe", "plm", 4): 6148.8,
    ("roe", "ppm", 0): 6482.4, ("roe", "ppm", 2): 6740.4, ("roe", "ppm", 4): 6984.4,
    ("hlld", "plm", 0): 3898.7, ("hlld", "plm", 2): 4156.7, ("hlld", "plm", 4): 4400.7,
    ("hlld", "ppm", 0): 4704.0, ("hlld", "ppm", 2): 4962.0, ("hlld", "ppm", 4): 5206.0,
    ("hlle", "plm", 0): 3458.9, ("hlle", "plm", 2): 3716.9, ("hlle", "plm", 4): 3960.9,
    ("hlle", "ppm", 0): 4293.8, ("hlle", "ppm", 2): 4551.8, ("hlle", "ppm", 4): 4795.8,
}

B200_SMS = 148
FP32_LANES_PER_SM = 128


def alg_bytes_per_cell(esz, npass):
    """Irreducible HBM bytes of a step: read and write rho, m (3), face B (3)
    and the passive scalars once each (cell-centre B follows from face B)."""
    return 2 * (7 + npass) * esz


def step_roofline(value, riemann, recon, npass, esz, hbm_gbs, sm_mhz):
    """The whole step against the slower of its two bounds: HBM at the
    algorithmic bytes per cell, and FP32 issue (SMs x 128 lanes x 2 ops per
    FMA x SM clock) at the algorithmic ops per cell.  None without an op
    count for the configuration."""
    ops = ALG_OPS_PER_CELL.get((riemann, recon, npass))
    if ops is None or value is None:
        return None
    nbytes = alg_bytes_per_cell(esz, npass)
    fp32_peak = B200_SMS * FP32_LANES_PER_SM * 2 * sm_mhz * 1e6          # ops/s
    hbm_bound = hbm_gbs * 1e9 / nbytes                                  # cell-updates/s
    fp32_bound = fp32_peak / ops
    bound = "fp32" if fp32_bound < hbm_bound else "hbm"
    return {"bound": bound, "ops_per_cell": ops, "bytes_per_cell": nbytes,
            "fp32_peak_tops": fp32_peak / 1e12, "sm_mhz": sm_mhz, "hbm_peak_gbs": hbm_gbs,
            "fp32_achieved_tops": value * ops / 1e12, "fp32_frac": value * ops / fp32_peak,
            "hbm_achieved_gbs": value * nbytes / 1e9, "hbm_frac": value * nbytes / (hbm_gbs * 1e9),
            "bound_cell_updates_per_s": min(hbm_bound, fp32_bound),
            "frac": value / min(hbm_bound, fp32_bound),
            "ops_source": "op-counting build of the FP64 restatement (oracle/count_ops.py)"}


def load_peaks():
    """The pool's measured peaks (MEASURED_PEAKS.json), or {} without the file."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


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
    peaks = load_peaks()
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
            nb = [sb[st] for st in sts if st in per_stage]
            kernels[kname] = (sum(ms), sum(ms) / len(ms), sum(nb) / len(nb))
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

    sm_mhz = (clk or {}).get("sm_mhz") or float(peaks.get("sm_max_mhz", 1965.0))
    step_rl = step_roofline(value, a.riemann, a.recon, a.npass, esz, hbm_peak, sm_mhz)

    # the accuracy, batched and served workloads are single-GPU measurements:
    # with several ranks (replicas of the headline box) they are left out
    batched = served = served_low = accuracy = None
    extras = ws == 1 and (a.batched > 0 or a.served > 0 or a.accuracy_steps > 0)
    if extras:
        box.close()
        box = None
    if extras and a.accuracy_steps > 0 and a.precision == 32:
        accuracy = run_accuracy(a, local, steps=a.accuracy_steps)
    if extras and a.batched > 0:
        batched = run_batched(a, local, stream, dist, dev)
    if extras and a.served > 0:
        served = run_served(a, local, a.served, a.rate)
        if a.rate_low > 0 and a.served_low > 0:
            served_low = run_served(a, local, a.served_low, a.rate_low, loops=False)

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        cpu = cpu_reference_sample(a, n_sample=a.ref_n, steps=a.ref_steps or 3, warmup=1)
        serial = cpu_reference_sample(a, n_sample=64, steps=3, warmup=1, threads=1)
        cpu["serial"] = {"value": serial["value"], "cores": 1, "sample": serial["sample"]}

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
        "step_roofline": step_rl,
        "stages": per_stage,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "clocks": clk,
        "accuracy": accuracy,
        "batched": batched,
        "served": served,
        "served_sub_saturating": served_low,
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
    # throughput counts the boxes that completed and the steps every box made
    # (a failed box's steps up to its failure were computed; the box is not
    # counted as a solve)
    steps_made = sum(s.cells * c["steps"] for s, c in zip(specs, clocks))
    out["batch"] = {"ms": ms, "boxes_per_s": done / (ms / 1e3), "cell_updates_per_s": steps_made / (ms / 1e3),
                    "boxes_completed": done, "boxes_failed": len(failed),
                    "failed_boxes": [{"box": i, "edge": specs[i].n, "mach": round(specs[i].mach, 3),
                                      "steps_made": clocks[i]["steps"]} for i in failed],
                    "cell_steps_scheduled": cells_steps, "cell_steps_made": steps_made,
                    "graph_replays": a.batched_steps,
                    "gpu_launches": bt.launch_count - launches0}
    bt.close()
    del bt
    if a.no_loops:
        return out

    # plain per-box loops: one Box at a time, the host driver loop over
    # imhd_step; FP64 is the plain method, FP32 the same loop at the batch's
    # precision.  Both run the first `loop_sample` boxes (a random sample).
    nloop = min(a.loop_sample or len(specs), len(specs))
    for prec in (64, 32):
        loop_ms = 0.0
        l1 = {}
        nfail = 0
        sample_cells_steps = 0
        for i, s in enumerate(specs[:nloop]):
            box = Box(s.n, precision=prec, riemann=s.riemann, npass=s.npass, cour=a.cour, edot=s.edot,
                      dt_turb=s.dt_turb, device=local)
            box.set_stream(stream.cuda_stream)
            _build_box(box, s)
            torch.cuda.synchronize()
            made = [0]

            def count(tsteps, t, dt, made=made):
                made[0] = tsteps - 1
            t0 = time.perf_counter()
            try:
                driver.run(box, t_end=1e30, maxsteps=s.steps + 1, forcing="device", dt_turb=s.dt_turb,
                           record_dt=False, on_step=count)
            except ImhdError:
                nfail += 1          # NaN / zero speed: the box stops, as in the batch
            sample_cells_steps += s.cells * made[0]
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
            "ms": loop_ms, "boxes": nloop, "boxes_failed": nfail, "boxes_per_s": (nloop - nfail) / (loop_ms / 1e3),
            "cell_updates_per_s": sample_cells_steps / (loop_ms / 1e3),
            "batch_rel_l1_max_over_sample": {names[k]: v for k, v in l1.items()},
            "timing": "host wall clock around each box's step loop (device synchronised)"}
        # like for like: cell-updates per second of the batch and of the loop
        # (the loop sample is the batch's first boxes, whose sizes differ from
        # the whole batch's mix; cell-updates/s does not depend on the mix's
        # box count)
        out["speedup_vs_fp%d_loop" % prec] = (out["batch"]["cell_updates_per_s"] /
                                             out["per_box_loop_fp%d" % prec]["cell_updates_per_s"])
    out["like_for_like"] = "speedup_vs_fp32_loop: same precision, same solver, batch vs one box at a time"
    return out


# ----------------------------------------------------------------- serving loop
def run_served(a, local, nreq, rate, loops=True):
    """Poisson stream of nreq box-solve requests at `rate` per second (edges
    {32,64,96,128,192} weighted 0.35/0.30/0.20/0.10/0.05, steps U[20,200], Roe
    or HLLD, |B0| U[0.1,2], Mach U[0.5,5], forcing on) served by imhd_server
    with continuous batching under the HBM budget; boxes/s, cell-updates/s and
    p50/p99 latency from submission to the result in host memory.  With
    `loops` the first requests of the same stream are also served one at a
    time by the plain per-box loop."""
    import threading

    import torch
    from isothermal_mhd_b200 import Box, ImhdError, driver, workloads
    from isothermal_mhd_b200.server import Server

    stream_ = workloads.request_stream(nreq, rate=rate, seed=a.seed + 1)
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
    lat, wait_s, failed, steps_made = {}, {}, [], {}
    t_last = t_start
    while len(lat) < len(specs):
        for i in range(len(specs)):
            if i in lat or ids[i] is None:
                continue
            state, info, _ = srv.poll(ids[i], fetch=True)
            if state in ("done", "failed"):
                lat[i] = info["latency_s"]
                wait_s[i] = info["queue_wait_s"]
                steps_made[i] = info["steps"]
                t_last = time.perf_counter()
                if state == "failed":
                    failed.append(i)
        time.sleep(0.002)
    th.join()
    stats = srv.stats()
    srv.stop(drain=True)
    srv.close()
    elapsed = t_last - t_start
    ok = [i for i in range(len(specs)) if i not in failed]
    lats = np.array([lat[i] for i in ok]) if ok else np.zeros(1)
    cells_steps = sum(s.cells * s.steps for s in specs)
    made_cells = sum(specs[i].cells * steps_made[i] for i in range(len(specs)))
    out = {"workload": "%d requests, Poisson %.0f req/s, edges {32,64,96,128,192} p=0.35/0.30/0.20/0.10/0.05, "
                       "steps U[20,200], Roe/HLLD 1:1, |B0| U[0.1,2], Mach U[0.5,5], FP32, forcing on, "
                       "HBM budget %.0f GB" % (len(specs), rate, a.hbm_budget / 1e9),
           "requests": len(specs), "requests_failed": len(failed), "elapsed_s": elapsed,
           "arrival_span_s": specs[-1].arrival,
           "offered_cell_updates_per_s": cells_steps / max(specs[-1].arrival, 1e-9),
           "boxes_per_s": len(ok) / elapsed, "cell_updates_per_s": made_cells / elapsed,
           "latency_s": {"p50": float(np.percentile(lats, 50)), "p99": float(np.percentile(lats, 99)),
                         "mean": float(lats.mean()), "max": float(lats.max()),
                         "of": "completed requests"},
           "queue_wait_s": {"p50": float(np.percentile([wait_s[i] for i in wait_s], 50)),
                            "p99": float(np.percentile([wait_s[i] for i in wait_s], 99))},
           "failed_requests": [{"request": i, "edge": specs[i].n, "riemann": specs[i].riemann,
                                "mach": round(specs[i].mach, 3), "steps_made": steps_made[i]} for i in failed],
           "server": stats}
    if not loops or a.no_loops:
        return out
    # plain per-box loops over the first requests of the stream, one at a time
    nloop = min(a.loop_sample or len(specs), len(specs), 64)
    for prec in (64, 32):
        tot = 0.0
        nfail = 0
        sample_work = 0
        for s in specs[:nloop]:
            kv, av, sv, af, sf = s.fields()
            box = Box(s.n, precision=prec, riemann=s.riemann, npass=s.npass, cour=a.cour, edot=s.edot,
                      dt_turb=s.dt_turb, device=local)
            made = [0]

            def count(tsteps, t, dt, made=made):
                made[0] = tsteps - 1
            t0 = time.perf_counter()
            box.init_uniform(1.0, s.b0)
            box.fourier_field("velocity", kv, av, sv)
            box.fourier_field("force", kv, af, sf)
            dt0 = a.cour * box.dx / box.max_speed()
            try:
                driver.run(box, t_end=1e30, maxsteps=s.steps + 1, dt0=dt0, forcing="device", dt_turb=s.dt_turb,
                           record_dt=False, on_step=count)
            except ImhdError:
                nfail += 1
            box.download()
            torch.cuda.synchronize()
            tot += time.perf_counter() - t0
            sample_work += s.cells * made[0]
            box.close()
        out["per_box_loop_fp%d" % prec] = {
            "requests": nloop, "requests_failed": nfail, "boxes_per_s": (nloop - nfail) / tot,
            "cell_updates_per_s": sample_work / tot,
            "timing": "host wall clock per request: build, step loop, download (one request at a time)"}
        # the sample's mix differs from the stream's: compare the time each
        # would take for the whole stream's work (cell-updates made)
        loop_time_stream = tot * made_cells / sample_work
        out["per_box_loop_fp%d" % prec]["est_s_for_stream"] = loop_time_stream
        out["speedup_vs_fp%d_loop" % prec] = loop_time_stream / elapsed
    return out


# ----------------------------------------------------------------- FP32 vs FP64
def run_accuracy(a, local, steps=None):
    """The bench workload (or --n / --riemann / --recon / --npass variants)
    advanced `steps` steps in FP64 on the reference driver schedule, then in
    FP32 with the FP64 run's dt and drive sequence; relative L1 and Linf of
    every field of the FP32 state against the FP64 one, and max |div B| (face
    differences per cell) of both.  Both final states are compared on the
    device: the FP64 state is packed into a device buffer (imhd_pack_planes)
    before its box is freed, then the FP32 box runs."""
    import torch
    from isothermal_mhd_b200 import Box

    steps = steps or a.accuracy
    n = a.n
    q, b, p, delv, f = make_initial_state(n, a.mach, a.npass, a.seed, a.b0x)
    dev = torch.device("cuda", local)
    nf = 10 + a.npass

    def run(prec, plan=None):
        box = Box(n, precision=prec, riemann=a.riemann, recon=a.recon, npass=a.npass, cour=a.cour, edot=a.edot,
                  dt_turb=0.05, device=local)
        box.upload(q, b, p)
        box.set_force(delv)
        t, dt, t_turb, rec = 0.0, 1e-15, 0.05, []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s_ in range(steps):
            if plan is None:
                drive = (t_turb > t) and (t_turb <= t + dt)
                if drive:
                    t_turb = max(t_turb + 0.05, t + 1e-2 * dt)
                    dt = 0.5 * dt
            else:
                dt, drive = plan[s_]
            rec.append((dt, drive))
            dt_new = box.step(dt, drive)
            t += dt
            dt = dt_new
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        raw = box.pack_planes(0, n)
        st = box.status()
        box.close()
        dt_t = torch.float64 if prec == 64 else torch.float32
        return raw.view(dt_t).view(nf, n, n, n), rec, el, st

    s64, plan, el64, st64 = run(64)
    s32, _, el32, st32 = run(32, plan)
    names = ["rho", "mx", "my", "mz", "bx_cc", "by_cc", "bz_cc", "bx_face", "by_face", "bz_face"]
    names += ["pass%d" % k for k in range(a.npass)]
    err = {}
    for k, nm in enumerate(names):
        v = s64[k]
        d = (s32[k].double() - v).abs()
        den = float(v.abs().sum())
        vmax = float(v.abs().max())
        err[nm] = {"rel_l1": float(d.sum()) / den if den > 0 else float(d.sum()),
                   "rel_linf": float(d.max()) / vmax if vmax > 0 else float(d.max())}

    def max_div(st):
        bx, by, bz = (st[7 + c].double() for c in range(3))
        d = (bx - torch.roll(bx, 1, dims=2)) + (by - torch.roll(by, 1, dims=1)) + (bz - torch.roll(bz, 1, dims=0))
        return float(d.abs().max())

    out = {"metric": "fp32_vs_fp64", "n": n, "steps": steps, "riemann": a.riemann, "recon": a.recon,
           "npass": a.npass, "mach": a.mach, "drive_steps": sum(1 for _, dr in plan if dr),
           "t_end": sum(dt for dt, _ in plan),
           "fields": err, "max_rel_l1": max(v["rel_l1"] for v in err.values()),
           "worst_field": max(err, key=lambda k: err[k]["rel_l1"]),
           "max_abs_divB": {"fp64": max_div(s64), "fp32": max_div(s32)},
           "bound": 1e-5, "within_bound": max(v["rel_l1"] for v in err.values()) <= 1e-5,
           "status": {"fp64": st64, "fp32": st32}, "wall_s": {"fp64": el64, "fp32": el32},
           "note": "FP32 run replays the FP64 run's dt and drive sequence; relative L1 = sum|fp32 - fp64| / "
                   "sum|fp64| per field"}
    del s64, s32
    torch.cuda.empty_cache()
    return out


# ----------------------------------------------------------------- CPU reference
def cpu_reference_sample(a, n_sample, steps, warmup, threads=None):
    """The CPU restatement of the reference (oracle, FP64, all host threads or
    `threads`) on an n_sample^3 box of the same physics; cell-updates/s over
    `steps` steps."""
    from oracle.pyoracle import Oracle
    threads = threads or os.cpu_count() or 1
    q, b, p, delv, f = make_initial_state(n_sample, a.mach, a.npass, a.seed)
    o = Oracle(n_sample, riemann=a.riemann, recon=a.recon, npass=a.npass, nthreads=threads)
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
                      f"{el:.1f} s on {threads} host thread(s); C++ restatement of the reference algorithm (the "
                      f"Fortran build is unavailable: no Fortran compiler or MPI in the image)"}


def run_reference(a, ws, rank):
    if rank != 0:
        return None
    steps = a.ref_steps or max(1, min(a.steps, 10))
    cpu = cpu_reference_sample(a, n_sample=a.ref_n, steps=steps, warmup=max(1, min(a.warmup, 2)))
    v = cpu["value"]
    return {
        "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": a.gpus or ws, "steps": steps, "warmup": a.warmup,
        "ms_per_step": (a.ref_n ** 3) / v * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded OU turbulence)", "impl": "reference",
        "config": {"workload": "%d^3 FP64 sample of the workload (driven MHD turbulence, van Leer + %s-char + %s + "
                               "CT, %d passive scalars, Mach %g), C++ restatement of the reference on the host cores; "
                               "the GPU arm runs the same physics at %d^3 in FP%d" % (
                                   a.ref_n, a.recon.upper(), a.riemann.upper(), a.npass, a.mach, a.n, a.precision),
                   "n": a.ref_n, "gpu_arm_n": a.n, "riemann": a.riemann, "recon": a.recon, "npass": a.npass,
                   "precision": 64, "parallelism": "host threads"},
        "cpu_baseline": cpu,
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ----------------------------------------------------------------- one box in z slabs
def modes_on_planes(kv, amp, scale, n, zplanes):
    """v_d = scale * sum_m 2 Re(A_{m,d} exp(2 pi i k_m . x)) at the cell
    centres x = ((i+1/2)/n, (j+1/2)/n, (z+1/2)/n) of the global z planes
    `zplanes` of an n^3 box: imhd_fourier_field's field (and OUForcing.field's)
    evaluated on one slab only.  Shape (3, len(zplanes), n, n)."""
    c = (np.arange(n) + 0.5) / n
    cz = (np.asarray(zplanes, dtype=np.float64) + 0.5) / n
    out = np.zeros((3, len(zplanes), n, n))
    for (kx, ky, kz), a6 in zip(kv, amp):
        ex = np.exp(2j * np.pi * kx * c)
        ey = np.exp(2j * np.pi * ky * c)
        ez = np.exp(2j * np.pi * kz * cz)
        ph = ez[:, None, None] * ey[None, :, None] * ex[None, None, :]
        for d in range(3):
            out[d] += 2.0 * (complex(a6[2 * d], a6[2 * d + 1]) * ph).real
    return out * scale


def slab_initial_state(dec, r, mach, npass, seed, b0x):
    """Rank r's slab (own planes and halos) of the bench's initial state: the
    OU velocity at rms Mach `mach` and the first force field, evaluated on the
    slab's global planes; passive scalars U[0, 1) drawn per rank."""
    from isothermal_mhd_b200 import forcing
    n = dec.nx
    f = forcing.OUForcing(n, seed=seed)
    zp = dec.global_planes(r)
    kv, amp, sc = f.device_modes(rms=mach)
    v = modes_on_planes(kv, amp, sc, n, zp)
    shape = v.shape[1:]
    q = np.zeros((7,) + shape)
    q[0] = 1.0
    q[1:4] = v
    q[4] = b0x
    b = np.zeros((3,) + shape)
    b[0] = b0x
    p = np.random.default_rng([seed, r]).random((npass,) + shape)
    f.advance(0.05)
    kv, amp, sc = f.device_modes(rms=1.0)
    delv = modes_on_planes(kv, amp, sc, n, zp)
    return q, b, p, delv


def run_slabs(a, ws, rank, local):
    """One n^3 box split into z slabs over the ranks (RankSlab: halo planes
    exchanged with the z neighbours over NCCL after every step, the new dt a
    MIN all-reduce, forcing sums a SUM all-reduce on drive steps).  Strong
    scaling: the job's value is n^3 * steps over the slowest rank's time."""
    import torch
    from isothermal_mhd_b200 import slabs

    dist = init_dist(ws, "nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = a.n
    dec = slabs.Decomposition(n, ws, slabs.halo_width(a.recon, a.npass))
    q, b, p, delv = slab_initial_state(dec, rank, a.mach, a.npass, a.seed, a.b0x)
    box = slabs._box_for(dec, rank, precision=a.precision, riemann=a.riemann, recon=a.recon, npass=a.npass,
                         cour=a.cour, edot=a.edot, dt_turb=0.05, device=local)
    stream = torch.cuda.current_stream(dev)
    box.set_stream(stream.cuda_stream)
    box.upload(q, b, p)
    box.set_force(delv)
    del q, b, p, delv
    rs = slabs.RankSlab(dec, rank, box, dist, device=dev)
    state = {"t": 0.0, "dt": 1e-15, "t_turb": 0.05, "drives": 0}

    def one_step():
        t_old, dt = state["t"], state["dt"]
        drive = (state["t_turb"] > t_old) and (state["t_turb"] <= t_old + dt)
        if drive:
            state["t_turb"] = max(state["t_turb"] + 0.05, t_old + 1e-2 * dt)
            dt = 0.5 * dt
            state["drives"] += 1
        state["dt"] = rs.step(dt, drive)
        state["t"] = t_old + dt

    for _ in range(a.warmup):
        one_step()
    torch.cuda.synchronize()
    dist.barrier()
    launches0 = box.launch_count
    drives0 = state["drives"]
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        one_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    t_max = max_over_ranks(dist, ms, dev)
    launches = box.launch_count - launches0
    box.close()
    dist.barrier()
    dist.destroy_process_group()
    if rank != 0:
        return None
    value = n ** 3 * a.steps / (t_max / 1e3)
    esz = 4 if a.precision == 32 else 8
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": t_max / a.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32" if a.precision == 32 else "f64", "data": "synthetic (seeded OU turbulence)",
        "config": {"workload": workload_name(a) + ", one box in z slabs over %d GPUs" % ws, "n": n,
                   "precision": a.precision, "riemann": a.riemann, "recon": a.recon + "-char", "npass": a.npass,
                   "parallelism": "z slabs x%d, halo %d planes, NCCL halo exchange + MIN all-reduce of dt" % (
                       ws, dec.halo),
                   "own_planes_per_rank": dec.counts[0], "l2": "inputs larger than L2",
                   "drive_steps_timed": state["drives"] - drives0},
        "gpu_launches": launches,
        "clocks": clk,
        "step_roofline": step_roofline(value / ws, a.riemann, a.recon, a.npass, esz,
                                       float(load_peaks().get("hbm_gbs", 6650.0)),
                                       (clk or {}).get("sm_mhz") or float(load_peaks().get("sm_max_mhz", 1965.0))),
        "e2e": None,
        "note": "step_roofline is per GPU (value / n_gpus); each slab also computes 2 x halo planes",
    }


# ----------------------------------------------------------------- launcher
def launch_ranks(n, argv):
    """Start this script once per rank (one process per GPU, rank env of a
    torchrun launch, master on 127.0.0.1), wait for all of them and return
    the worst exit code.  Rank 0's output is the job's; a rank that fails
    stops the others."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        out = None if r == 0 else subprocess.DEVNULL
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + list(argv), env=env,
                                      stdout=out))
    rc = 0
    pending = list(procs)
    while pending:
        for pr in list(pending):
            code = pr.poll()
            if code is None:
                continue
            pending.remove(pr)
            if code != 0:
                rc = rc or code
                for other in pending:        # the exact PIDs this launcher started
                    other.terminate()
        time.sleep(0.05)
    return rc


def dist_check(a, ws, rank):
    """Launcher self-test: a gloo group of the launched ranks, the job-time
    reduction, one JSON line from rank 0."""
    dist = init_dist(ws, "gloo")
    t = max_over_ranks(dist, 10.0 * (rank + 1))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        return {"n_gpus": ws, "ms_max": t, "value": job_rate(100, ws, t)}
    return None


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    a = parse(argv)
    ws, rank, local = dist_env()
    launched = "WORLD_SIZE" in os.environ
    if a.gpus is None:
        a.gpus = ws
    if a.gpus > 1 and not launched and a.impl == "ours":
        sys.exit(launch_ranks(a.gpus, argv))
    if launched and a.gpus != ws:
        raise SystemExit("bench.py: --gpus %d but the launch has WORLD_SIZE %d" % (a.gpus, ws))
    if a.dist_check:
        line = dist_check(a, ws, rank)
    elif a.impl == "reference":
        line = run_reference(a, ws, rank)
    elif a.accuracy > 0:
        line = run_accuracy(a, local) if rank == 0 else None
    elif a.split == "slabs" and ws > 1:
        line = run_slabs(a, ws, rank, local)
    else:
        line = run_ours(a, ws, rank, local)
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
