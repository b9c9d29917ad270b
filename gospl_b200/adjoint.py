"""Gradients of an elevation misfit through many goSPL steps.

``SurfaceEvolution.apply(K, U, rain, h0, model, nsteps, every)`` runs
``nsteps`` physics steps of ``model`` (flow accumulation with the lake
cascade, SPL, hillslope, uplift) from elevation ``h0`` with per-vertex
erodibility ``K``, uplift rate ``U`` and rainfall ``rain`` and returns the
final elevation; its backward pass is the hand-written adjoint of the library
(``gs_adjoint_step``): transposed sweeps in reverse topological order, the
reversed lake cascade and the adjoint CG of the diffusion.  Memory is bounded
by checkpointing: the forward keeps the elevation every ``every`` steps; the
backward re-runs each segment with recording on and reverses it.  With
``every=None`` the forward records every step instead (memory for all of
them, no recomputation) and the backward only reverses.

Discrete decisions of every step (receivers, pits, flat routing, cascade
states, land/sea and lake masks) are held fixed, so the gradient is that of
the piecewise-smooth map on the piece the forward ran on; the level of a
partially filled lake is held constant.
"""
import contextlib

import numpy as np

from . import _lib

GS_TUNE_WARM_START = 8


@contextlib.contextmanager
def _cold(model):
    """Solver warm starts off (GS_TUNE_WARM_START = 0) while the adjoint runs:
    a warm-started CG depends on the previous step's solution, so a replayed
    segment and the two runs of a finite difference would differ from the
    forward in the solver's last digits."""
    L = _lib.load()
    prev = int(L.gs_plan_tuning(model._plan, GS_TUNE_WARM_START))
    _lib.check(L.gs_plan_tune(model._plan, GS_TUNE_WARM_START, 0))
    try:
        yield
    finally:
        _lib.check(L.gs_plan_tune(model._plan, GS_TUNE_WARM_START, prev))


def _set_params(model, K, U, rain):
    t = model.torch
    model.K = 0.0
    model.Kfield = K.detach().to(model.dev, t.float64).contiguous().clone()
    model.upsub = U.detach().to(model.dev, t.float64).contiguous().clone()
    model.rainMesh = rain.detach().to(model.dev, t.float64).contiguous().clone()


def _restart(model, h):
    """Elevation h at the start of a step; forcing of the current rainfall."""
    t = model.torch
    model.hGlobal.copy_(h)
    model.tNow = model.tStart
    model.tEnd = float("inf")
    larea = t.as_tensor(np.asarray(model.mesh.larea, np.float64), device=model.dev)
    model.rainVal = model.rainMesh.clamp(min=0.0)
    model.bL.copy_(model.rainVal * larea)


def run(model, K, U, rain, h0, nsteps, every=10):
    """Forward with checkpoints: (h_T, [h at steps 0, every, 2 every, ...]);
    with every=None every step is recorded for the backward instead
    (h_T, None)."""
    with _cold(model):
        return _run(model, K, U, rain, h0, nsteps, every)


def _run(model, K, U, rain, h0, nsteps, every):
    _set_params(model, K, U, rain)
    _restart(model, h0)
    if every is None:
        model.record(nsteps)
        try:
            for s in range(nsteps):
                model.record_slot(s)
                model.step()
        finally:
            model.record_slot(-1)
        return model.hGlobal.clone(), None
    ckpt = []
    for s in range(nsteps):
        if s % every == 0:
            ckpt.append(model.hGlobal.clone())
        model.step()
    return model.hGlobal.clone(), ckpt


def backward(model, K, U, rain, ckpt, nsteps, every, lam_T):
    """dJ/d(K, U, rain, h0) from lam_T = dJ/dh_T by checkpointed replay, or
    from the records of a forward run with every=None."""
    with _cold(model):
        return _backward(model, K, U, rain, ckpt, nsteps, every, lam_T)


def _backward(model, K, U, rain, ckpt, nsteps, every, lam_T):
    t = model.torch
    n = model.lpoints
    f64 = dict(dtype=t.float64, device=model.dev)
    _set_params(model, K, U, rain)
    gK = t.zeros(n, **f64)
    gU = t.zeros(n, **f64)
    grain = t.zeros(n, **f64)
    gbl = t.zeros(n, **f64)
    lam = lam_T.detach().to(**f64).contiguous().clone()
    larea = t.as_tensor(np.asarray(model.mesh.larea, np.float64), **f64)
    if every is None:
        for j in range(nsteps - 1, -1, -1):
            model.adjoint_step(j, lam, gK, gU, grain, gbl)
            grain += t.where(model.rainMesh > 0, gbl * larea, t.zeros_like(gbl))
        return gK, gU, grain, lam
    # the records stay allocated for the next backward (model.record(0) frees them)
    model.record(every)
    try:
        nseg = (nsteps + every - 1) // every
        for seg in range(nseg - 1, -1, -1):
            s0 = seg * every
            k = min(every, nsteps - s0)
            _restart(model, ckpt[seg])
            for j in range(k):
                model.record_slot(j)
                model.step()
            model.record_slot(-1)
            for j in range(k - 1, -1, -1):
                model.adjoint_step(j, lam, gK, gU, grain, gbl)
                # bL_t = max(rain, 0) larea
                grain += t.where(model.rainMesh > 0, gbl * larea, t.zeros_like(gbl))
    finally:
        model.record_slot(-1)
    return gK, gU, grain, lam


class SurfaceEvolution:
    """torch.autograd.Function over (K, U, rain, h0) -> h_T."""

    @staticmethod
    def apply(K, U, rain, h0, model, nsteps, every=10):
        """every: checkpoint interval of the replay, or None to record every
        step during the forward (no recomputation)."""
        import torch

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, K, U, rain, h0):
                hT, ckpt = run(model, K, U, rain, h0, nsteps, every)
                ctx.ckpt = ckpt
                ctx.save_for_backward(K, U, rain)
                return hT

            @staticmethod
            def backward(ctx, g):
                K, U, rain = ctx.saved_tensors
                gK, gU, grain, gh0 = backward(model, K, U, rain, ctx.ckpt, nsteps, every, g)
                need = ctx.needs_input_grad
                return tuple(v if need[k] else None for k, v in enumerate((gK, gU, grain, gh0)))

        return _Fn.apply(K, U, rain, h0)
