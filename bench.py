"""Landscape vertex-steps/s of goSPL's per-timestep surface-process path.

Workload: the global sphere landscape -- icosahedral mesh refined 9 times
(2,621,442 vertices, R = 6371 km), seeded spherical-harmonic relief to degree
256 (l^-2 spectrum) scaled to -4000..+3000 m with sea level 0, lognormal rain
(median 1 m/yr, sigma 0.5), three Gaussian uplift belts (+-2 mm/yr), K = 5e-7,
m = 0.5, n = 1, MFD with 3 receivers, diffusivity 0.05 m^2/yr, dt = 1e4 yr.
One step = runProcesses' physics step (receivers, pit filling, flow
accumulation with the lake cascade, SPL, hillslope, forcing).  Mesh build and
the init-time flow accumulation are excluded.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun (N > 1) every rank advances its own replica (one landscape per
GPU, no collective on the data path); the value is the whole-job throughput
with the time taken as the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "landscape vertex-steps/s @2.6M-vertex sphere"
HBM_FALLBACK = 6650.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def sphere_inputs(level, seed=20261205):
    from gospl_b200 import synthetic as S
    return S.sphere_config(level=level, seed=seed)


def cpu_sample(level=6, steps=1):
    """Oracle (single-threaded C + numpy restatement of the reference) on a
    smaller sphere of the same recipe: vertex-steps/s of the timed steps."""
    from oracle.model import OracleModel
    c, f, z, rain, up, p = sphere_inputs(level)
    p = dict(p, rain=rain, upsub=up)
    om = OracleModel(c, f, z, p)
    t0 = time.perf_counter()
    for _ in range(steps):
        om.step()
    dt = time.perf_counter() - t0
    return len(z) * steps / dt, len(z), steps, dt


def _cpu_worker(args):
    level, steps = args
    return cpu_sample(level, steps)


def run_reference(args, rank, world):
    """CPU reference arm: the oracle restatement of the reference path on all
    host cores (independent samples in parallel processes)."""
    if rank != 0:
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    level = args.cpu_level
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        for _ in range(args.warmup and 1):
            pool.map(_cpu_worker, [(level, 1)] * cores)
        t1 = time.perf_counter()
        res = pool.map(_cpu_worker, [(level, 1)] * (cores * max(1, args.steps // 5)))
        t2 = time.perf_counter()
    vs = sum(r[1] * r[2] for r in res)
    value = vs / (t2 - t1)
    n = res[0][1]
    sample = "oracle on icosphere level %d (%d vertices), %d one-step samples in %d processes" % (
        level, n, len(res), cores)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "vertex-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * 2621442 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "sphere level 9 (2,621,442 vertices), one physics step; CPU samples at level %d"
                       % level, "global_batch": 1, "seq_len": 0, "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": "vertex-steps/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "vertex-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": t2 - t0}
    print(json.dumps(line), flush=True)


def parse_profile(report):
    out = {}
    for line in report.strip().splitlines():
        parts = line.rsplit(" ", 2)
        if len(parts) == 3:
            out[parts[0]] = (int(parts[1]), float(parts[2]))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=9)
    ap.add_argument("--cpu-level", type=int, default=6)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import ctypes
    import torch
    from gospl_b200 import _lib
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    t_setup = time.perf_counter()
    c, f, z, rain, up, p = sphere_inputs(args.level)
    p = dict(p, rain=rain, upsub=up, tEnd=1.0e30)
    mesh = FVMesh(c, f, p["bc"], device=dev)
    model = Model(coords=c, cells=f, elev=z, params=p, mesh=mesh, device=dev)
    n = model.lpoints
    setup_s = time.perf_counter() - t_setup
    stream = torch.cuda.current_stream(dev)
    L = _lib.load()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        model.step()
    barrier()
    # ---- timed region: device-resident state ----
    launches0 = model.launches()
    clk = Clocks(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        model.step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    launches = model.launches() - launches0
    stats = dict(model.stats)
    if pg is not None:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n * args.steps / (ms / 1000.0)

    # ---- per-kernel times (same steps, events around every launch) ----
    L.gs_plan_profile(model._plan, 1)
    nprof = max(1, min(args.steps, 3))
    for _ in range(nprof):
        model.step()
    buf = ctypes.create_string_buffer(1 << 16)
    L.gs_plan_profile_report(model._plan, buf, len(buf))
    L.gs_plan_profile(model._plan, 0)
    prof = parse_profile(buf.value.decode())

    # ---- end to end through the public API with host buffers ----
    h_host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    h_host.copy_(model.hGlobal)
    out_host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        model.hGlobal.copy_(h_host, non_blocking=True)
        model.step()
        out_host.copy_(model.hGlobal, non_blocking=True)
        h_host, out_host = out_host, h_host
    e3.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = e2.elapsed_time(e3)
    if pg is not None:
        t = torch.tensor([ms_e2e], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = world * n * args.steps / (ms_e2e / 1000.0)

    # ---- roofline of the dominant kernel ----
    hbm, src = peaks()
    top = max(prof.items(), key=lambda kv: kv[1][1]) if prof else ("none", (1, 1.0))
    name, (cnt, tot_ms) = top
    per_launch_ms = tot_ms / max(cnt, 1)
    bytes_per_vertex = ALGO_BYTES.get(_short(name), None)
    if bytes_per_vertex is not None:
        units = n * bytes_per_vertex[1](model)
        achieved = units * bytes_per_vertex[0] / (per_launch_ms / 1000.0) / 1e9
    else:
        achieved = None
    share = {(_short(k)): round(v[1] / sum(x[1] for x in prof.values()), 4) for k, v in prof.items()}

    cpu = None
    if rank == 0 and not args.no_cpu:
        v, nn, st, dt = cpu_sample(args.cpu_level, 1)
        cpu = {"value": v, "unit": "vertex-steps/s", "cores": 1, "kind": "port",
               "sample": "oracle (C + numpy restatement of the reference path) on icosphere level %d "
                         "(%d vertices), 1 physics step, %.1f s" % (args.cpu_level, nn, dt)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "vertex-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sphere, SH relief)",
            "config": {"workload": "sphere level 9 (2,621,442 vertices), full physics step: receivers, pit fill, "
                                   "flow accumulation + lake cascade, SPL, hillslope, forcing",
                       "vertices": n, "global_batch": world, "seq_len": 0,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set > 126 MB L2 (mesh arrays alone ~1 GB)"},
            "e2e": {"value": e2e, "unit": "vertex-steps/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
            "roofline": {"bound": "hbm", "kernel": _short(name), "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": (achieved / hbm) if achieved else None, "traffic": None,
                         "peak_source": src, "launch_ms": per_launch_ms, "launches": cnt},
            "kernel_share": share,
            "kernel_ms_per_step": sum(v[1] for v in prof.values()) / nprof,
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "stats": stats.get("flow"),
            "setup_s": setup_s,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def _short(name):
    s = name
    for key in ("k_dataflow<gs::FlowOp>", "k_dataflow<gs::SplOp>"):
        pass
    if "k_dataflow" in s:
        return "k_dataflow_flow" if "FlowOp" in s else ("k_dataflow_spl" if "SplOp" in s else "k_dataflow")
    for tok in s.replace("(", " ").replace("<", " ").split():
        if tok.startswith("_ZN2gs"):
            # mangled gs::k_name
            rest = tok[6:]
            ln = ""
            while rest and rest[0].isdigit():
                ln += rest[0]
                rest = rest[1:]
            return rest[:int(ln)] if ln else tok
        if tok.startswith("gs::"):
            return tok[4:]
    return s


# algorithmic bytes per vertex (compulsory traffic, d = 6 neighbour slots, R = 3)
# and the multiplier of vertices per launch
ALGO_BYTES = {
    "k_mfd_receivers": (4 + 6 * 4 + 6 * 8 + 8 + 6 * 4 + 3 * 4 + 3 * 8 + 3 * 8 + 3 * 1, lambda m: 1),
    "k_dataflow_flow": (4 + 4 + 8 + 3 * 4 + 3 * 8 + 8 + 8 + 8 + 4 + 1, lambda m: 1),
    "k_dataflow_spl": (3 * 4 + 3 * 8 + 8 + 8 + 4 + 4 + 1, lambda m: 1),
}


if __name__ == "__main__":
    main()
