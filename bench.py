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
                                       "--format=csv,noheader,nounits", "-lms", "50"],
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


def cpu_sample(level=7, steps=2, warm=0):
    """Oracle (single-threaded C + numpy restatement of the reference) on a
    smaller sphere of the same recipe: vertex-steps/s of the timed steps
    (model set-up and `warm` untimed steps excluded)."""
    from oracle.model import OracleModel
    c, f, z, rain, up, p = sphere_inputs(level)
    p = dict(p, rain=rain, upsub=up)
    om = OracleModel(c, f, z, p)
    for _ in range(warm):
        om.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        om.step()
    dt = time.perf_counter() - t0
    return len(z) * steps / dt, len(z), steps, dt


def _cpu_worker(args):
    level, steps, warm = args
    return cpu_sample(level, steps, warm)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    """CPU reference arm: the oracle restatement of the reference path on all
    host cores.  One process per core advances its own copy of the sample
    landscape (the reference's own mpirun path cannot be built: it needs
    gfortran, PETSc and MPI); the aggregate throughput is the sum of the
    concurrent per-process rates."""
    if rank != 0:
        return
    import multiprocessing as mp
    cores = min(host_cores(), 96)
    level = args.cpu_level
    steps = max(1, min(args.steps, 2))
    warm = 1 if args.warmup > 0 else 0
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(level, steps, warm)] * cores)
    wall = time.perf_counter() - t0
    value = sum(r[0] for r in res)
    n = res[0][1]
    sample = ("oracle on icosphere level %d (%d vertices), %d concurrent processes x %d timed step(s) "
              "after %d untimed" % (level, n, cores, steps, warm))
    full = None
    if not args.no_ref_full and level != args.level:
        # one measured step of the benchmark's own mesh, one process
        v9, n9, st9, dt9 = cpu_sample(args.level, 1, 0)
        full = {"vertices": n9, "processes": 1, "steps": st9, "ms_per_step": 1000.0 * dt9 / st9,
                "value": v9, "unit": "vertex-steps/s",
                "what": "one physics step of the oracle on the benchmark's sphere, measured (set-up and the "
                        "init-time flow accumulation excluded)"}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "vertex-steps/s", "n_gpus": world,
            "same_config": level == args.level, "sampled_level": level,
            "ms_per_step_derived": level != args.level,
            "full_size_step": full,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sphere_vertices(args.level) / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded sphere, SH relief)",
            "config": {"workload": "sphere level %d (%d vertices), full physics step; CPU samples at level %d"
                       % (args.level, sphere_vertices(args.level), level),
                       "global_batch": 1, "seq_len": 0, "parallelism": "processes"},
            "cpu_baseline": {"value": value, "unit": "vertex-steps/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "vertex-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def sphere_vertices(level):
    return 10 * 4 ** level + 2


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
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=9)
    ap.add_argument("--cpu-level", type=int, default=7)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="sphere", choices=["sphere", "planar", "ensemble", "precision",
                                                                   "transport", "sediment", "output", "adjoint"])
    ap.add_argument("--fd-vertices", type=int, default=64, help="adjoint: finite-difference samples per field")
    ap.add_argument("--fd-eps", type=float, default=1e-6, help="adjoint: relative finite-difference step")
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--loop", action="store_true", help="ensemble: also time the per-member loop")
    ap.add_argument("--adjoint-steps", type=int, default=4, help="sphere: steps of the adjoint timing (0: skip)")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--no-ref-full", action="store_true",
                    help="reference arm: skip the measured full-size oracle step")
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
    if args.workload == "precision":
        run_precision(args, dev)
        return
    if args.workload == "transport":
        run_transport(args, dev)
        return
    if args.workload == "sediment":
        run_sediment(args, dev)
        return
    if args.workload == "output":
        run_output(args, dev)
        return
    if args.workload == "adjoint":
        run_adjoint(args, dev)
        return
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    t_setup = time.perf_counter()
    ens_members = None
    if args.workload == "sphere":
        c, f, z, rain, up, p = sphere_inputs(args.level)
        p = dict(p, rain=rain, upsub=up, tEnd=1.0e30)
        mesh = FVMesh(c, f, p["bc"], device=dev)
        model = Model(coords=c, cells=f, elev=z, params=p, mesh=mesh, device=dev)
    elif args.workload == "planar":
        from gospl_b200 import synthetic as S
        c, f, z, rain, up, p = S.planar_config()
        p = dict(p, rain=rain, upsub=up, tEnd=1.0e30)
        mesh = FVMesh(c, f, p["bc"], device=dev)
        model = Model(coords=c, cells=f, elev=z, params=p, mesh=mesh, device=dev)
    else:
        from gospl_b200 import synthetic as S
        from gospl_b200.ensemble import Ensemble, partition
        sizes = S.ensemble_sizes(256)[:args.members]
        mine = partition(sizes, world)[rank]
        ens_members = [S.ensemble_member(int(sizes[i]), 20261300 + i) for i in mine]
        ens_members = [(c, f, z, r, u, dict(p, tEnd=1.0e30)) for c, f, z, r, u, p in ens_members]
        ens = Ensemble(ens_members, device=dev)
        model = ens.model
    n = model.lpoints
    n_all = n
    if pg is not None:
        t = torch.tensor([n], dtype=torch.int64, device=dev)
        pg.all_reduce(t)
        n_all = int(t.item())
    setup_s = time.perf_counter() - t_setup
    stream = torch.cuda.current_stream(dev)
    L = _lib.load()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize(dev)

    tuned = None
    if not args.no_tune:
        from gospl_b200 import autotune
        best, table = autotune.tune(model, steps=2)
        tuned = {"sweep_blocks_per_sm": best[0], "coop_blocks_per_sm": best[1],
                 "ms_per_step": {"%d,%d" % k: round(v, 4) for k, v in table.items()},
                 "what": "launch shapes timed on this landscape before the warm-up (state restored after each)"}
    # clock sampling starts before the warm-up and nvidia-smi gets a second to
    # come up (no steps run meanwhile: the timed steps are those of the
    # configured run), so its samples cover the timed region
    clk = Clocks(local)
    time.sleep(1.0)
    for _ in range(args.warmup):
        model.step()
    barrier()
    # the state the timed steps start from: the end-to-end runs below restart
    # from it, so all three time the same steps of the same landscape
    state0 = {k: getattr(model, k).clone() for k in ("hGlobal", "cumED", "EbLocal")}
    t_now0 = model.tNow

    def restore():
        for k, v in state0.items():
            getattr(model, k).copy_(v)
        model.tNow = t_now0
        torch.cuda.synchronize(dev)

    # ---- timed region: device-resident state ----
    launches0 = model.launches()
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
    value = n_all * args.steps / (ms / 1000.0)

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
    # (1) streamed: every step's rainfall comes from pinned host memory and
    # every step's elevation goes back to pinned host memory; the state stays
    # on the device between steps (as goSPL's PETSc vectors do).  The copies
    # run on a copy stream ordered by events: the rain of step k+1 is copied
    # in during step k, the elevation of step k (a device snapshot) is copied
    # out during step k+1.
    copy = torch.cuda.Stream(dev)
    rain_host = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    for b in rain_host:
        b.copy_(model.rainMesh)
    out_host = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    rain_dev = [torch.empty_like(model.rainMesh) for _ in range(2)]
    snap = [torch.empty_like(model.hGlobal) for _ in range(2)]
    rain0 = model.rainMesh
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_used = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    restore()
    barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    copy.wait_event(e2)
    with torch.cuda.stream(copy):
        rain_dev[0].copy_(rain_host[0], non_blocking=True)
    ev_in[0].record(copy)
    for k in range(args.steps):
        a = k % 2
        stream.wait_event(ev_in[a])
        model.rainMesh = rain_dev[a]
        if k + 1 < args.steps:
            b = (k + 1) % 2
            if k >= 1:
                copy.wait_event(ev_used[b])          # step k-1 read rain_dev[b]
            with torch.cuda.stream(copy):
                rain_dev[b].copy_(rain_host[b], non_blocking=True)
            ev_in[b].record(copy)
        model.step()
        ev_used[a].record(stream)
        if k >= 2:
            stream.wait_event(ev_out[a])             # snap[a] of step k-2 is out
        snap[a].copy_(model.hGlobal)
        ev_used[a].record(stream)
        copy.wait_event(ev_used[a])
        with torch.cuda.stream(copy):
            out_host[a].copy_(snap[a], non_blocking=True)
        ev_out[a].record(copy)
    stream.wait_stream(copy)
    e3.record(stream)
    torch.cuda.synchronize(dev)
    model.rainMesh = rain0
    ms_e2e = e2.elapsed_time(e3)
    # (2) round trip: the elevation itself goes host -> device -> host every
    # step, so the copies sit between the steps (the host owns the state)
    restore()
    h_host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    h_host.copy_(model.hGlobal)
    oh = torch.empty(n, dtype=torch.float64, pin_memory=True)
    barrier()
    e4 = torch.cuda.Event(enable_timing=True)
    e5 = torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    for _ in range(args.steps):
        model.hGlobal.copy_(h_host, non_blocking=True)
        model.step()
        oh.copy_(model.hGlobal, non_blocking=True)
        h_host, oh = oh, h_host
    e5.record(stream)
    torch.cuda.synchronize(dev)
    ms_rt = e4.elapsed_time(e5)
    if pg is not None:
        t = torch.tensor([ms_e2e, ms_rt], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_e2e, ms_rt = float(t[0].item()), float(t[1].item())
    e2e = n_all * args.steps / (ms_e2e / 1000.0)
    e2e_rt = n_all * args.steps / (ms_rt / 1000.0)

    # ---- roofline of the dominant kernel ----
    hbm, src = peaks()
    top = max(prof.items(), key=lambda kv: kv[1][1]) if prof else ("none", (1, 1.0))
    name, (cnt, tot_ms) = top
    kname = _short(name)
    per_launch_ms = tot_ms / max(cnt, 1)
    layout = launch_layout(model, stats)
    algo = algo_bytes_per_launch(kname, layout)
    achieved = algo / (per_launch_ms / 1000.0) / 1e9 if algo else None
    traffic = NCU_TRAFFIC_PER_VERTEX.get(kname)
    share = {}
    for k, v in prof.items():
        sk = _short(k)
        share[sk] = round(share.get(sk, 0.0) + v[1] / sum(x[1] for x in prof.values()), 4)
    step_bytes = step_algo_bytes(layout)
    step_gbs = step_bytes / (ms / args.steps / 1000.0) / 1e9

    adj = None
    if ens_members is None and args.adjoint_steps > 0:
        adj = adjoint_ratio(model, args.adjoint_steps, stream, dev, pg)

    loop = None
    if ens_members is not None and args.loop:
        # the same members as separate models, stepped one after the other
        models = [Model(coords=c, cells=f, elev=z, params=dict(p, rain=r, upsub=u), device=dev,
                        mesh=FVMesh(c, f, p["bc"], device=dev)) for c, f, z, r, u, p in ens_members]
        for _ in range(args.warmup):
            for m in models:
                m.step()
        barrier()
        e4 = torch.cuda.Event(enable_timing=True)
        e5 = torch.cuda.Event(enable_timing=True)
        e4.record(stream)
        for _ in range(args.steps):
            for m in models:
                m.step()
        e5.record(stream)
        torch.cuda.synchronize(dev)
        ms_loop = e4.elapsed_time(e5)
        if pg is not None:
            t = torch.tensor([ms_loop], dtype=torch.float64, device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms_loop = float(t.item())
        loop = {"value": n_all * args.steps / (ms_loop / 1000.0), "ms_per_step": ms_loop / args.steps,
                "what": "the same members as separate models stepped one after another on the same GPU(s)"}
        for m in models:
            m.destroy()

    cpu = None
    if rank == 0 and not args.no_cpu and args.workload == "sphere":
        v, nn, st, dt = cpu_sample(args.cpu_level, 2)
        cpu = {"value": v, "unit": "vertex-steps/s", "cores": 1, "kind": "port",
               "sample": "oracle (C + numpy restatement of the reference path) on icosphere level %d "
                         "(%d vertices), %d physics steps, %.1f s" % (args.cpu_level, nn, st, dt)}
    if rank == 0:
        line = {
            "metric": {"sphere": METRIC, "planar": "landscape vertex-steps/s, 20k planar",
                       "ensemble": "landscape vertex-steps/s, planar ensemble"}[args.workload],
            "value": value, "unit": "vertex-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if args.workload == "ensemble" else "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": {"sphere": "synthetic (seeded sphere, SH relief)",
                     "planar": "synthetic (seeded jittered hex mesh, fractal relief)",
                     "ensemble": "synthetic (seeded planar members, fractal relief)"}[args.workload],
            "config": config_of(args, n, n_all, world),
            "e2e": {"value": e2e, "unit": "vertex-steps/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                    "what": "Model.step() with each step's rainfall copied in from pinned host memory and its "
                            "elevation copied out to pinned host memory on a copy stream (event-ordered, "
                            "overlapping the neighbouring steps)",
                    "roundtrip": {"value": e2e_rt, "what": "the elevation copied host -> device before and "
                                  "device -> host after every step (host-owned state; copies between steps)"}},
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                         "traffic": (traffic * n) if traffic else None,
                         "traffic_source": ("DRAM bytes per vertex of the ncu capture of this kernel on the "
                                            "655,362-vertex sphere (profiles/), scaled to %d vertices" % n)
                         if traffic else None,
                         "algorithmic_bytes": algo, "peak_source": src + " (MEASURED_PEAKS.json hbm_gbs)"
                         if src == "measured" else src, "launch_ms": per_launch_ms, "launches": cnt},
            "step_roofline": {"algorithmic_bytes": step_bytes, "achieved": step_gbs, "peak": hbm, "unit": "GB/s",
                              "frac": step_gbs / hbm, "counts": layout},
            "kernel_share": share,
            "kernel_ms_per_step": sum(v[1] for v in prof.values()) / nprof,
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "stats": {k: stats.get(k) for k in ("flow", "spl", "hillslope")},
            "loop_baseline": loop,
            "tuned": tuned,
            "adjoint": adj,
            "setup_s": setup_s,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def adjoint_ratio(model, k, stream, dev, pg):
    """Adjoint:forward cost ratio on the same landscape: k forward steps with
    one checkpoint, then the backward pass (replay of the k steps with
    recording + k adjoint steps), both timed with CUDA events, max over ranks;
    and the same with every step recorded during the forward, so that the
    backward only reverses (records_kept)."""
    import torch
    from gospl_b200 import adjoint as A
    n = model.lpoints
    f64 = dict(dtype=torch.float64, device=dev)
    K = torch.full((n,), model.K if model.Kfield is None else 0.0, **f64) if model.Kfield is None else model.Kfield
    U = model.upsub if model.upsub is not None else torch.zeros(n, **f64)
    rain = model.rainMesh
    h0 = model.hGlobal.clone()
    hT, ck = A.run(model, K, U, rain, h0, k, k)   # warm-up of the forward path
    A.backward(model, K, U, rain, ck, k, k, torch.ones_like(hT))
    torch.cuda.synchronize(dev)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record(stream)
    hT, ck = A.run(model, K, U, rain, h0, k, k)
    e[1].record(stream)
    gK, gU, grain, gh = A.backward(model, K, U, rain, ck, k, k, 2.0 * (hT - h0))
    e[2].record(stream)
    torch.cuda.synchronize(dev)
    tf, tb = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    # the same with every step recorded during the forward (no recomputation)
    A.run(model, K, U, rain, h0, k, None)
    A.backward(model, K, U, rain, None, k, None, torch.ones_like(hT))
    torch.cuda.synchronize(dev)
    e[0].record(stream)
    hT2, _ = A.run(model, K, U, rain, h0, k, None)
    e[1].record(stream)
    gK2, _, _, gh2 = A.backward(model, K, U, rain, None, k, None, 2.0 * (hT2 - h0))
    e[2].record(stream)
    torch.cuda.synchronize(dev)
    tfr, tbr = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    if pg is not None:
        t = torch.tensor([tf, tb, tfr, tbr], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        tf, tb, tfr, tbr = (float(v) for v in t)
    finite = all(bool(torch.isfinite(v).all()) for v in (gK, gh, gK2, gh2))
    return {"ratio": tb / tf, "forward_ms_per_step": tf / k, "adjoint_ms_per_step": tb / k, "steps": k,
            "checkpoint_every": k, "what": "adjoint step = replay of the step with recording + its reverse "
                                          "(gradients wrt K, U, rain and h0)",
            "records_kept": {"ratio": tbr / tf, "recording_forward_ms_per_step": tfr / k,
                             "adjoint_ms_per_step": tbr / k,
                             "what": "every step recorded during the forward (no recomputation); ratio = "
                                     "reverse step / plain forward step"},
            "finite": finite}


def run_adjoint(args, dev):
    """Inversion for erodibility on the 160k-vertex planar landscape: the
    target is the elevation after 100 steps with the hidden 'true' K field;
    the loss is the L2 elevation misfit of a run from uniform K.  Gradients
    with respect to K, uplift and rain come from the hand-written adjoint with
    a checkpoint every 10 steps; forward and backward are timed with CUDA
    events (adjoint:forward cost ratio, the replay of each segment included).
    Central finite differences at seeded interior vertices check them: the
    difference of the two misfits is summed as sum (h+ - h-)(h+ + h- - 2t),
    so it does not cancel two large numbers.  A perturbation that changes a
    discrete decision (the final receivers or depression ids differ between
    the + and - runs) has no derivative on the piece the adjoint follows;
    those samples are counted and left out of the error."""
    import torch
    from gospl_b200 import adjoint as A
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    c, f, z, rain, up, p, onb, k0 = S.adjoint_config()
    nsteps, every = 100, 10
    p = dict(p, rain=rain, upsub=up, tEnd=1.0e30)
    mesh = FVMesh(c, f, p["bc"], device=dev)
    model = Model(coords=c, cells=f, elev=z, params=p, mesh=mesh, device=dev)
    n = model.lpoints
    f64 = dict(dtype=torch.float64, device=dev)
    Ktrue = torch.tensor(p["K"], **f64)
    U = torch.tensor(up, **f64)
    R = torch.tensor(rain, **f64)
    h0 = torch.tensor(z, **f64)
    stream = torch.cuda.current_stream(dev)
    target, _ = A.run(model, Ktrue, U, R, h0, nsteps, every)
    K0 = torch.full((n,), k0, **f64)
    # warm-up, then the timed forward (with checkpoints) and backward
    hT, ck = A.run(model, K0, U, R, h0, nsteps, every)
    A.backward(model, K0, U, R, ck, nsteps, every, 2.0 * (hT - target))
    torch.cuda.synchronize(dev)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record(stream)
    hT, ck = A.run(model, K0, U, R, h0, nsteps, every)
    e[1].record(stream)
    gK, gU, gR, gh = A.backward(model, K0, U, R, ck, nsteps, every, 2.0 * (hT - target))
    e[2].record(stream)
    torch.cuda.synchronize(dev)
    tf, tb = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    loss = float(((hT - target) ** 2).sum())

    # every step's discrete state (receivers, depression ids, flat
    # directions), hashed on the device: a sample whose + and - runs differ in
    # any of them at any step crossed a decision the gradient cannot see
    g = torch.Generator(device="cpu").manual_seed(7)
    wts = [torch.randint(1, 2 ** 31, (m,), generator=g, dtype=torch.int64).to(dev)
           for m in (model.rcv_i.numel(), n, n)]

    def final(args):
        A._set_params(model, *args)
        A._restart(model, h0)
        hs = []
        for _ in range(nsteps):
            model.step()
            hs.append(int((model.rcv_i.reshape(-1).long() * wts[0]).sum() + (model.pitIDs.long() * wts[1]).sum()
                          + (model.flatDirs.long() * wts[2]).sum()))
        return model.hGlobal.clone(), hs

    rng = np.random.default_rng(20261208)
    interior = np.where(~onb)[0]
    nfd = args.fd_vertices
    fields = {"K": (K0, gK), "uplift": (U, gU), "rain": (R, gR)}
    fd_out = {}
    for name, (base, grad) in fields.items():
        idx = rng.choice(interior, nfd, replace=False)
        rel, flips, rows = [], 0, []
        for i in idx:
            eps = args.fd_eps * abs(float(base[i]))
            vals = []
            for sgn in (1.0, -1.0):
                b = base.clone()
                b[i] += sgn * eps
                args_ = [K0, U, R]
                args_[list(fields).index(name)] = b
                vals.append(final(args_))
            (hp, sp), (hm, sm) = vals
            fd = float(((hp - hm) * (hp + hm - 2.0 * target)).sum()) / (2.0 * eps)
            ad = float(grad[i])
            flip = sp != sm
            if flip:
                flips += 1
            else:
                rel.append(abs(ad - fd) / max(abs(fd), 1e-300))
            rows.append([int(i), ad, fd, flip])
        rel = np.array(rel) if rel else np.array([np.nan])
        fd_out[name] = {"samples": nfd, "decision_flips": flips, "max_rel_err": float(np.max(rel)),
                        "median_rel_err": float(np.median(rel)),
                        "p90_rel_err": float(np.quantile(rel, 0.9)),
                        "within_1e-6": int((rel <= 1e-6).sum()), "rows": rows[:8]}
    line = {"metric": "adjoint:forward cost ratio", "value": tb / tf, "unit": "ratio", "n_gpus": 1,
            "steps": nsteps, "warmup": 1, "ms_per_step": tf / nsteps, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded jittered hex mesh, Gaussian-field ln K, fractal relief)",
            "config": {"workload": "adjoint inversion for erodibility: %d-vertex planar mesh, 200 x 200 km, "
                                   "100 steps of 1000 yr, checkpoint every 10, L2 elevation misfit from "
                                   "uniform K = exp(-12.5)" % n, "vertices": n, "checkpoint_every": every},
            "forward_ms": tf, "adjoint_ms": tb, "adjoint_ms_per_step": tb / nsteps, "loss": loss,
            "grad_norms": {"K": float(gK.norm()), "uplift": float(gU.norm()), "rain": float(gR.norm())},
            "finite_differences": fd_out,
            "fd_what": "central differences, step %g of the value, at seeded interior vertices; misfit "
                       "difference summed as sum (h+ - h-)(h+ + h- - 2 target); samples whose + and - runs "
                       "differ in the receivers, depression ids or flat directions at any of the %d steps "
                       "are counted as decision flips and left out of the error" % (args.fd_eps, nsteps)}
    print(json.dumps(line), flush=True)
    model.destroy()


def run_precision(args, dev):
    """FP32-bulk form against the plain FP64 path on the 10.5M-vertex sphere
    (icosphere level 10, SH relief to degree 512 scaled to -5000..+4000 m,
    rain and uplift as for the 2.6M sphere, dt = 5000 yr): the same steps from
    the same state in both, wall time per step of each and the relative error
    of drainage area, erosion rate and elevation of the FP32 form."""
    import torch
    from gospl_b200 import _lib
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    level = args.level if args.level != 9 else 10
    c, f, z, rain, up, p = S.sphere_config(level=level, lmax=512, zlo=-5000.0, zhi=4000.0, dt=5000.0)
    p = dict(p, rain=rain, upsub=up, tEnd=1.0e30)
    mesh = FVMesh(c, f, p["bc"], device=dev)
    stream = torch.cuda.current_stream(dev)
    out = {}
    for bits in (32, 64):
        m = Model(coords=c, cells=f, elev=z, params=p, mesh=mesh, device=dev, precision=bits, refine_tol=1e-10)
        m.step()
        first = dict(FAL=m.FAL.cpu().numpy(), Eb=m.EbLocal.cpu().numpy(), h=m.hGlobal.cpu().numpy())
        for _ in range(max(args.warmup - 1, 0)):
            m.step()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            m.step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        out[bits] = dict(ms=e0.elapsed_time(e1) / args.steps, FAL=m.FAL.cpu().numpy(), Eb=m.EbLocal.cpu().numpy(),
                         h=m.hGlobal.cpu().numpy(), passes=int(_lib.load().gs_plan_tuning(m._plan, 4)),
                         first=first)
        m.destroy()
    n = len(z)

    def err(key, first=False):
        a, b = (out[32]["first"][key], out[64]["first"][key]) if first else (out[32][key], out[64][key])
        d = np.abs(a - b) / max(np.abs(b).max(), 1e-300)
        return {"max": float(d.max()), "median": float(np.median(d)), "p99": float(np.quantile(d, 0.99))}

    line = {"metric": "landscape vertex-steps/s, FP32-refined form @10.5M-vertex sphere",
            "value": n * 1000.0 / out[32]["ms"], "unit": "vertex-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out[32]["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 sweeps/CG with f64 refinement",
            "data": "synthetic (seeded sphere, SH relief to degree 512)",
            "config": {"workload": "sphere level %d (%d vertices), -5000..+4000 m, dt 5000 yr" % (level, n),
                       "vertices": n, "global_batch": 1, "seq_len": 0, "parallelism": "single"},
            "precision": {"fp64_ms_per_step": out[64]["ms"], "fp32_ms_per_step": out[32]["ms"],
                          "speedup": out[64]["ms"] / out[32]["ms"], "refine_tol": 1e-10,
                          "refinement_passes": out[32]["passes"],
                          "rel_error_vs_fp64_after_first_step": {"drainage_area": err("FAL", True),
                                                                 "erosion_rate": err("Eb", True),
                                                                 "elevation": err("h", True)},
                          "rel_error_vs_fp64_after_all_steps": {"drainage_area": err("FAL"),
                                                                "erosion_rate": err("Eb"), "elevation": err("h")},
                          "note": "errors relative to the largest |value| of the FP64 field; over many steps the "
                                  "two trajectories part where a discrete decision (tie, threshold) flips"}}
    print(json.dumps(line), flush=True)


def run_transport(args, dev, G=1.0):
    """Transport-limited SPL (G = 1) against detachment-limited SPL (G = 0) on
    the 2.6M-vertex sphere: the same steps from the same state, time per
    step, time of the erosion stage alone and the coupled solver's operator
    applications (each one flow sweep and one SPL sweep)."""
    import torch
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    c, f, z, rain, up, p = sphere_inputs(args.level)
    p = dict(p, rain=rain, upsub=up, tEnd=1.0e30)
    mesh = FVMesh(c, f, p["bc"], device=dev)
    stream = torch.cuda.current_stream(dev)
    out = {}
    for g in (G, 0.0):
        m = Model(coords=c, cells=f, elev=z, params=dict(p, G=g), mesh=mesh, device=dev)
        for _ in range(args.warmup):
            m.step()
        torch.cuda.synchronize(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 2)]
        iters = []
        ev[0].record(stream)
        for k in range(args.steps):
            m.flowAccumulation()
            ev[2 + 2 * k].record(stream)
            m.erodepSPL()
            ev[3 + 2 * k].record(stream)
            iters.append(m.stats["spl"]["cg_iters"])
            m.getHillslope()
            if m.tNow < m.tEnd:
                m.applyForces()
            m.tNow += m.dt
        ev[1].record(stream)
        torch.cuda.synchronize(dev)
        spl = sum(ev[2 + 2 * k].elapsed_time(ev[3 + 2 * k]) for k in range(args.steps)) / args.steps
        out[g] = dict(ms=ev[0].elapsed_time(ev[1]) / args.steps, spl_ms=spl, iters=iters,
                      relres=m.stats["spl"]["cg_relres"])
        m.destroy()
    n = len(z)
    line = {"metric": "landscape vertex-steps/s, transport-limited SPL (G = %g) @2.6M-vertex sphere" % G,
            "value": n * 1000.0 / out[G]["ms"], "unit": "vertex-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out[G]["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sphere, SH relief)",
            "config": {"workload": "sphere level %d (%d vertices), full physics step with the coupled "
                                   "erosion-deposition solve" % (args.level, n),
                       "vertices": n, "G": G, "global_batch": 1, "seq_len": 0, "parallelism": "single"},
            "transport": {"ms_per_step": out[G]["ms"], "erosion_ms_per_step": out[G]["spl_ms"],
                          "gmres_operator_applications": out[G]["iters"], "final_relres": out[G]["relres"],
                          "detachment_limited_ms_per_step": out[0.0]["ms"],
                          "detachment_limited_erosion_ms_per_step": out[0.0]["spl_ms"]}}
    print(json.dumps(line), flush=True)


def run_sediment(args, dev):
    """Continental deposition (nodep off: a second flow accumulation and
    sedChange per step) against the plain step on the 2.6M-vertex sphere; the
    same steps from the same state, time per step, time of the deposition
    stage (second flow accumulation + sedChange) and the sediment cascade's
    passes.  The headline run keeps goSPL's lake thresholds (nlPitVolume 1e9
    m3, nlPitDepth 100 m) with the Picard solver for the non-linear diffusion
    of large deep lakes; a second run puts every lake deposit bottom-up
    (nlPitVolume = inf)."""
    import torch
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    c, f, z, rain, up, p = sphere_inputs(args.level)
    p = dict(p, rain=rain, upsub=up, tEnd=1.0e30)
    mesh = FVMesh(c, f, p["bc"], device=dev)
    stream = torch.cuda.current_stream(dev)
    runs = {"picard": dict(nodep=False, marineSolver="picard"),
            "marine": dict(nodep=False, marineSolver="picard", seadepo=True),
            "marine-Gmar0.5": dict(nodep=False, marineSolver="picard", seadepo=True, Gmar=0.5),
            "bottom-up": dict(nodep=False, nlPitVolume=float("inf")),
            "nodep": dict(nodep=True)}
    out = {}
    for name, extra in runs.items():
        m = Model(coords=c, cells=f, elev=z, params=dict(p, **extra), mesh=mesh, device=dev)
        nodep = extra["nodep"]
        seadepo = extra.get("seadepo", False)
        sea_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)] if seadepo else None
        sea_stats = []
        for _ in range(args.warmup):
            m.step()
        torch.cuda.synchronize(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 2)]
        passes, lakes = [], []
        ev[0].record(stream)
        for k in range(args.steps):
            m.flowAccumulation()
            m.erodepSPL()
            ev[2 + 2 * k].record(stream)
            if not nodep:
                m.flowAccumulation()
                m.sedChange()
                passes.append(m.stats["sed"]["cascade_passes"])
                lakes.append(m.stats["sed"]["status"])
                if seadepo:
                    sea_ev[2 * k].record(stream)
                    m.seaChange()
                    sea_ev[2 * k + 1].record(stream)
                    sea_stats.append(dict(m.stats["sea"]))
            ev[3 + 2 * k].record(stream)
            m.getHillslope()
            if m.tNow < m.tEnd:
                m.applyForces()
            m.tNow += m.dt
        ev[1].record(stream)
        torch.cuda.synchronize(dev)
        sed = sum(ev[2 + 2 * k].elapsed_time(ev[3 + 2 * k]) for k in range(args.steps)) / args.steps
        out[name] = dict(ms=ev[0].elapsed_time(ev[1]) / args.steps, sed_ms=sed, passes=passes,
                         diffused_lakes=lakes, npits=m.stats.get("sed", {}).get("npits"),
                         vsed_max=float(m.vSed.max().item()))
        if seadepo:
            out[name]["sea_ms"] = sum(sea_ev[2 * k].elapsed_time(sea_ev[2 * k + 1])
                                      for k in range(args.steps)) / args.steps
            out[name]["sea"] = sea_stats
        m.destroy()
    n = len(z)
    h = out["picard"]
    line = {"metric": "landscape vertex-steps/s with continental deposition @2.6M-vertex sphere",
            "value": n * 1000.0 / h["ms"], "unit": "vertex-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": h["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sphere, SH relief)",
            "config": {"workload": "sphere level %d (%d vertices), full physics step with nodep off: flow, SPL, "
                                   "flow, sedChange (lakes of >= 1e9 m3 and >= 100 m smoothed by the Picard "
                                   "non-linear diffusion), hillslope, forcing" % (args.level, n),
                       "vertices": n, "global_batch": 1, "seq_len": 0, "parallelism": "single"},
            "sediment": {name: dict({"ms_per_step": o["ms"], "deposition_ms_per_step": o["sed_ms"],
                                     "cascade_passes": o["passes"], "diffused_lakes": o["diffused_lakes"],
                                     "sed_pits": o["npits"], "vsed_max_m3_per_yr": o["vsed_max"]},
                                    **({"marine_ms_per_step": o["sea_ms"], "marine": o["sea"]}
                                       if "sea_ms" in o else {}))
                         for name, o in out.items()}}
    print(json.dumps(line), flush=True)


def run_output(args, dev):
    """Output files (goSPL's WriteMesh: HDF5 + XDMF every tout years) on the
    2.6M-vertex sphere.  (1) The packing kernel alone (gs_output_fields: 73
    bytes read and 36 written per vertex) against the measured HBM copy
    bandwidth.  (2) The same steps from the same state without outputs and
    with an output after every step (tout = dt), compressed (gzip, level 4)
    and not: device time per step on the model's stream and wall time per
    step including the wait for the files, so the cost a run pays for its
    outputs is the difference."""
    import shutil
    import torch
    from gospl_b200 import _lib
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    c, f, z, rain, up, p = sphere_inputs(args.level)
    work = tempfile.mkdtemp(prefix="gospl_out_")
    try:
        p = dict(p, rain=rain, upsub=up, tEnd=1.0e30, outputDir=os.path.join(work, "out"))
        p["tout"] = p["dt"]
        mesh = FVMesh(c, f, p["bc"], device=dev)
        m = Model(coords=c, cells=f, elev=z, params=p, mesh=mesh, device=dev)
        stream = torch.cuda.current_stream(dev)
        n = m.lpoints
        for _ in range(max(args.warmup, 1)):     # one step at least: the packing kernel's land/sea mask
            m.step()
        L = _lib.load()
        stage = torch.empty((9, n), dtype=torch.float32, device=dev)

        def pack():
            _lib.check(L.gs_output_fields(m._plan, _lib.ptr(m.hGlobal), _lib.ptr(m.cumED), _lib.ptr(m.EbLocal),
                                          _lib.ptr(m.waterFilled), _lib.ptr(m.fillFAL), _lib.ptr(m.FAL),
                                          _lib.ptr(m.vSed), _lib.ptr(m.upsub), _lib.ptr(m.rainVal), None,
                                          _lib.ptr(stage)))

        for _ in range(3):
            pack()
        flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)   # 256 MB > L2, between launches
        reps = 20
        t_pack = 0.0
        for _ in range(reps):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            pack()
            b.record(stream)
            torch.cuda.synchronize(dev)
            t_pack += a.elapsed_time(b) / reps
        del flush
        peak, src = peaks()
        algo = 109.0 * n
        state = {k: getattr(m, k).clone() for k in ("hGlobal", "cumED", "EbLocal", "FAL", "fillFAL", "waterFilled",
                                                   "vSed", "bL")}
        t0 = m.tNow

        def restore():
            for k, v in state.items():
                getattr(m, k).copy_(v)
            m.tNow = t0
            m.output.saveTime = t0

        runs = {}
        nsteps = min(args.steps, 5)      # 5 outputs of 94 MB (uncompressed) at most on disk
        for name, level in (("no_output", None), ("gzip", 4), ("uncompressed", None)):
            restore()
            m.output.level = level
            torch.cuda.synchronize(dev)
            w0 = time.perf_counter()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(nsteps):
                if name != "no_output":
                    m.visModel()
                m.step()
            b.record(stream)
            torch.cuda.synchronize(dev)
            m.output.flush()
            wall = (time.perf_counter() - w0) * 1000.0 / nsteps
            size = sum(os.path.getsize(os.path.join(dp, fn)) for dp, _, fns in os.walk(p["outputDir"]) for fn in fns)
            runs[name] = {"device_ms_per_step": a.elapsed_time(b) / nsteps, "wall_ms_per_step": wall,
                          "bytes_on_disk": size}
            shutil.rmtree(os.path.join(p["outputDir"], "h5"), ignore_errors=True)
            os.makedirs(os.path.join(p["outputDir"], "h5"))
        m.destroy()
    finally:
        shutil.rmtree(work, ignore_errors=True)
    base = runs["no_output"]["wall_ms_per_step"]
    line = {"metric": "output overhead per step (an output after every step) @2.6M-vertex sphere",
            "value": runs["gzip"]["wall_ms_per_step"] - base, "unit": "ms/step", "n_gpus": 1,
            "steps": nsteps, "warmup": args.warmup, "ms_per_step": runs["gzip"]["wall_ms_per_step"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64->f32",
            "data": "synthetic (seeded sphere, SH relief)",
            "config": {"workload": "sphere level %d (%d vertices), full physics step with goSPL's output files "
                                   "(9 float32 fields, XMF, XDMF) written after every step" % (args.level, n),
                       "vertices": n, "global_batch": 1, "seq_len": 0, "parallelism": "single",
                       "l2": "256 MB buffer written between timed packing launches"},
            "pack": {"ms": t_pack, "algorithmic_bytes": algo, "achieved_gbs": algo / t_pack / 1e6,
                     "peak_gbs": peak, "frac": algo / t_pack / 1e6 / peak, "peak_source": src},
            "runs": runs}
    print(json.dumps(line), flush=True)


def config_of(args, n, n_all, world):
    if args.workload == "sphere":
        return {"workload": "sphere level %d (%d vertices), full physics step: receivers, pit fill, "
                            "flow accumulation + lake cascade, SPL, hillslope, forcing" % (args.level, n),
                "vertices": n, "global_batch": world, "seq_len": 0,
                "parallelism": "replicas" if world > 1 else "single",
                "l2": "working set > 126 MB L2 (mesh arrays alone ~1 GB)"}
    if args.workload == "planar":
        return {"workload": "planar landscape, 20,000-vertex jittered hex lattice over 100 x 100 km, fractal "
                            "relief 0-50 m, fixed boundaries, U = 1 mm/yr, rain 1 m/yr, K = 2e-6, dt = 1000 yr",
                "vertices": n, "global_batch": world, "seq_len": 0,
                "parallelism": "replicas" if world > 1 else "single",
                "l2": "working set fits in L2 (launch-latency bound)"}
    return {"workload": "ensemble of %d planar landscapes (%d vertices in all; sizes log-uniform 1e4-5e5, "
                        "250 m spacing, own K and rain), full physics step, all members per launch"
                        % (args.members, n_all),
            "vertices": n_all, "global_batch": args.members, "seq_len": 0,
            "parallelism": "members sharded over %d GPU(s)" % world,
            "l2": "working set > 126 MB L2"}


def _short(name):
    """gs::k_name from a (possibly mangled) kernel name; the two ordered
    sweeps are told apart by their operator type."""
    s = name
    if "k_ordered" in s:
        return "k_ordered_flow" if "FlowOrd" in s else ("k_ordered_spl" if "SplOrd" in s else "k_ordered")
    if "k_dataflow" in s:
        return "k_dataflow_flow" if "FlowOp" in s else ("k_dataflow_spl" if "SplOp" in s else "k_dataflow")
    if "k_mfd_receivers" in s:
        return "k_mfd_receivers"
    for tok in s.replace("(", " ").replace("<", " ").split():
        if tok.startswith("_ZN2gs"):
            rest = tok[6:]
            ln = ""
            while rest and rest[0].isdigit():
                ln += rest[0]
                rest = rest[1:]
            return rest[:int(ln)] if ln else tok
        if tok.startswith("gs::"):
            return tok[4:]
    return s


def launch_layout(model, stats):
    """Counts the byte models need: vertices, receiver links with a nonzero
    weight (donor edges of the flow sweep), flat-BFS cells and the executed
    per-step iteration counts of the last step."""
    import torch
    n = model.lpoints
    R = model.flowDir
    w = model.wgt_i
    selfr = model.rcv_i == torch.arange(n, device=w.device, dtype=model.rcv_i.dtype).unsqueeze(0)
    links = int(((w != 0) & ~selfr).sum().item())
    fl = stats.get("flow", {})
    hs = stats.get("hillslope", {})
    pit_cells = int((model.pitIDs > -1).sum().item())
    return {"n": n, "R": R, "W": int(np.max(model.mesh.nnb)),
            "links": links, "pit_cells": pit_cells,
            "cascade_solves": int(fl.get("cascade_solves", 0)), "flat_rounds": int(fl.get("flat_rounds", 0)),
            "fill_rounds": int(fl.get("fill_rounds", 0)), "cg_iters": int(hs.get("cg_iters", 0))}


def algo_bytes_per_launch(kname, L):
    """Compulsory bytes of one launch, from the device layout (int32 ids,
    float64 values, slot-major [W][n] neighbour tables).  Gathers of values
    another thread wrote in the same sweep count as cache hits."""
    n, R, W, E = L["n"], L["R"], L["W"], L["links"]
    if kname == "k_ordered_flow":
        # order 4, link mask 4, receiver-slot codes 8, sorted slot order 8,
        # b 8, q write 8; per donor link: neighbour id 4 + weight 8
        return n * (4 + 4 + 8 + 8 + 8 + 8) + E * (4 + 8)
    if kname == "k_ordered_spl":
        # order 4, rcv 4R, coefficient 8R, hOld 8, h write 8
        return n * (4 + 12 * R + 16)
    if kname in ("k_bfs_local", "k_bfs_tiles"):
        # packed rows of the pit cells (count + up to W local ids, padded to
        # a multiple of 4 ints) and one distance write per cell
        S = ((W + 1 + 3) // 4) * 4
        return L["pit_cells"] * (4 * S + 4)
    if kname == "k_mfd_receivers":
        # h 8, gid 4, neighbour count 1, W ids 4 + W lengths 8 (slot-major),
        # writes rcv 4R + dist 8R + wgt 8R
        return n * (8 + 4 + 1 + 12 * W + 20 * R)
    if kname in ("k_dataflow_flow",):
        return n * (4 + 4 + 8 + 12 * R + 8 + 8 + 8 + 4 + 1)
    if kname in ("k_dataflow_spl",):
        return n * (12 * R + 8 + 8 + 4 + 4 + 1)
    return None


def step_algo_bytes(L):
    """Compulsory bytes of one physics step, per vertex by stage with the
    executed counts: receivers 144, pit fill 52 per full-vertex propagation
    pass (steepest descent, cross-basin edges, final fill: 3) plus 40 per
    labelling/flat pass (pit labels, flat directions: 2), flow sweep 60, SPL
    108, 164 per CG iteration, 204 per cascade solve (receivers rebuild +
    flow sweep) and forcing 40."""
    per_vertex = (144 + (52 * 3 + 40 * 2) + 60 + 108 + 164 * L["cg_iters"] + 204 * L["cascade_solves"] + 40)
    return L["n"] * per_vertex


# DRAM bytes per vertex (dram__bytes_read.sum + dram__bytes_write.sum of one
# launch divided by the vertices it processed) from the ncu captures summarised
# under profiles/; scaled by the vertex count of the run.
NCU_TRAFFIC_PER_VERTEX = {
    "k_mfd_receivers": (24.905728e6 + 2.152192e6) / 655362,
    "k_ordered_flow": (38.153216e6 + 1.851392e6) / 655362,
    "k_bfs_local": 1.780992e6 / 655362,
    "k_relax_active": (1.359360e6 + 0.125440e6) / 655362,
}


if __name__ == "__main__":
    main()
