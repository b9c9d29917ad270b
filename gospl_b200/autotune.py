"""Launch-shape autotuner.

The ordered dependency sweeps and the cooperative kernels (basin relaxation,
grid BFS, hillslope CG) have a free launch shape: blocks per SM.  More blocks
keep more dependency chains in flight but compete for the SM with the kernels
running beside them on the side streams; the best shape depends on the mesh
(DAG depth, pit structure) and the GPU.  ``tune(model)`` times a few physics
steps for each candidate on the model's own landscape, restores the state
after every trial, and keeps the fastest shape in the plan.  The knobs change
launch shapes only; results change only by the rounding of the hillslope CG's
inner products, whose block partial sums follow the cooperative grid size.
"""
import ctypes

from . import _lib

SWEEP, COOP = 1, 2


def _get(model, knob):
    return int(_lib.load().gs_plan_tuning(model._plan, knob))


def _set(model, knob, value):
    _lib.check(_lib.load().gs_plan_tune(model._plan, knob, int(value)))


def tune(model, steps=3, sweep=(4, 8, 16), coop=(1, 2, 4, 8)):
    """Pick (sweep blocks per SM, cooperative blocks per SM) by timing `steps`
    steps per candidate from the model's current state.  Returns (best,
    {candidate: ms per step})."""
    t = model.torch
    limit = _get(model, COOP + 1)
    coop = [c for c in coop if 1 <= c <= limit] or [1]
    saved = {k: getattr(model, k).clone() for k in ("hGlobal", "cumED", "EbLocal", "bL")}
    t_now = model.tNow
    stream = t.cuda.current_stream(model.dev)
    results = {}

    def restore():
        for k, v in saved.items():
            getattr(model, k).copy_(v)
        model.tNow = t_now

    for s in sweep:
        for c in coop:
            _set(model, SWEEP, s)
            _set(model, COOP, c)
            restore()
            model.step()   # warm-up of this shape
            restore()
            t.cuda.synchronize(model.dev)
            e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                model.step()
            e1.record(stream)
            t.cuda.synchronize(model.dev)
            results[(s, c)] = e0.elapsed_time(e1) / steps
    best = min(results, key=results.get)
    _set(model, SWEEP, best[0])
    _set(model, COOP, best[1])
    restore()
    return best, results
