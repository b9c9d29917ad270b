"""Solver warm starts (GS_TUNE_WARM_START): the hillslope CG started from h
plus the previous step's diffusion change agrees with the cold start (the
right-hand side, as hillslope.py:90-233 starts it) to the solver tolerance
and needs no more iterations; with warm starts off a run depends only on its
inputs, bit for bit, which the adjoint's replays and finite differences rely
on; the knob takes 0 or 1 only and forgets the stored start when set."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GS_TUNE_WARM_START = 8
GS_EINVAL = 1


def _run(warm, nsteps=6):
    import torch
    from gospl_b200 import _lib
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    coords, cells, z, rain, up, p = S.planar_config(n=3000, side=30.0e3, seed=3)
    p = dict(p, rain=rain, upsub=up, tEnd=100 * p["dt"])
    m = Model(coords=coords, cells=cells, elev=z, params=p, mesh=FVMesh(coords, cells, p["bc"]), device="cuda:0")
    L = _lib.load()
    assert L.gs_plan_tuning(m._plan, GS_TUNE_WARM_START) == 1, "warm starts are on by default"
    _lib.check(L.gs_plan_tune(m._plan, GS_TUNE_WARM_START, int(warm)))
    iters = []
    for _ in range(nsteps):
        m.step()
        iters.append(m.stats["hillslope"]["cg_iters"])
    torch.cuda.synchronize()
    h = m.hGlobal.clone()
    m.destroy()
    return h, iters


def test_warm_start_agrees_with_cold_start_and_cold_runs_repeat_bitwise():
    import torch
    hw, itw = _run(True)
    hc, itc = _run(False)
    hc2, _ = _run(False)
    assert torch.equal(hc, hc2), "a cold-started run must repeat bit for bit"
    scale = float(hc.abs().max())
    assert float((hw - hc).abs().max()) <= 1e-10 * scale
    assert min(itc) >= 1 and sum(itw) <= sum(itc), (itw, itc)


def test_warm_start_knob_accepts_only_0_and_1():
    from gospl_b200 import _lib
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    coords, cells, z, rain, up, p = S.planar_config(n=500, side=10.0e3, seed=4)
    p = dict(p, rain=rain, upsub=up)
    m = Model(coords=coords, cells=cells, elev=z, params=p, mesh=FVMesh(coords, cells, p["bc"]), device="cuda:0")
    L = _lib.load()
    assert L.gs_plan_tune(m._plan, GS_TUNE_WARM_START, 2) == GS_EINVAL
    assert L.gs_plan_tuning(m._plan, GS_TUNE_WARM_START) == 1
    _lib.check(L.gs_plan_tune(m._plan, GS_TUNE_WARM_START, 0))
    assert L.gs_plan_tuning(m._plan, GS_TUNE_WARM_START) == 0
    m.destroy()
