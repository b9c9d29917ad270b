"""Failure detection on the GPU path, without faulting the GPU.

goSPL classifies a failed flow solve and carries on (flowplex.py:236-315);
here every failure is a status code the host reads, and the plan stays
usable afterwards:
- non-finite inputs (NaN rain, infinite uplift, NaN elevation, injected on
  the host) are rejected with GS_ENONFINITE at the first synchronisation of
  the flow accumulation, before the relaxation and any sweep;
- a dependency sweep whose wall-clock budget (GS_TUNE_SWEEP_BUDGET) runs out
  stops with GS_ETIMEOUT (a bounded wait, not a fault);
after either, the next call with valid inputs gives exactly the result of a
model that never failed.  Degenerate meshes: a cell of zero area (held fixed
in the diffusion solve), and a closed domain whose depressions cannot drain
(steps like the oracle).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GS_ENONFINITE = 4
GS_ETIMEOUT = 6
GS_TUNE_SWEEP_BUDGET = 6


def _planar_pair(n=3000, nodep=True):
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    coords, cells, z, rain, up, p = S.planar_config(n=n, side=30.0e3, seed=3)
    p = dict(p, rain=rain, upsub=up, nodep=nodep, tEnd=10 * p["dt"])
    fv = FVMesh(coords, cells, p["bc"])

    def mk():
        return Model(coords=coords, cells=cells, elev=z, params=p, mesh=fv, device="cuda:0")

    return mk(), mk()


def _same_flow(a, b):
    import torch
    torch.cuda.synchronize()
    for k in ("FAL", "fillFAL", "waterFilled", "lFill"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    for k in ("pitIDs", "flatDirs", "rcv_i"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k


@pytest.mark.parametrize("where", ["rain", "uplift", "elevation"])
def test_nonfinite_inputs_are_rejected_and_the_plan_recovers(where):
    from gospl_b200._lib import GsError
    m, ref = _planar_pair()
    k = m.lpoints // 2
    if where == "rain":
        m.rainMesh[k] = float("nan")
        m.applyForces()                       # rain * area -> a NaN rain volume
    elif where == "uplift":
        m.upsub[k] = float("inf")
        m.applyForces()                       # h + inf * dt
    else:
        m.hGlobal[k] = float("nan")
    with pytest.raises(GsError) as e:
        m.flowAccumulation()
    assert e.value.code == GS_ENONFINITE, e.value
    # valid inputs again: the same result as a model that never failed
    m.hGlobal.copy_(ref.hGlobal)
    m.bL.copy_(ref.bL)
    m.flowAccumulation()
    ref.flowAccumulation()
    _same_flow(m, ref)
    m.destroy()
    ref.destroy()


def test_sweep_time_budget_runs_out_and_the_plan_recovers():
    """A 1 us budget on the 655,362-vertex sphere (its drainage sweep takes
    hundreds of microseconds along the longest river): GS_ETIMEOUT, then with
    the default budget the same flow accumulation as a fresh model."""
    from gospl_b200 import _lib
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    c, f, z, rain, up, p = S.sphere_config(level=8)
    p = dict(p, rain=rain, upsub=up)
    fv = FVMesh(c, f, p["bc"], device="cuda:0")
    m = Model(coords=c, cells=f, elev=z, params=p, mesh=fv, device="cuda:0")
    ref = Model(coords=c, cells=f, elev=z, params=p, mesh=fv, device="cuda:0")
    L = _lib.load()
    default = L.gs_plan_tuning(m._plan, GS_TUNE_SWEEP_BUDGET)
    assert default == 4000000
    _lib.check(L.gs_plan_tune(m._plan, GS_TUNE_SWEEP_BUDGET, 1))
    assert L.gs_plan_tuning(m._plan, GS_TUNE_SWEEP_BUDGET) == 1
    with pytest.raises(_lib.GsError) as e:
        m.flowAccumulation()
    assert e.value.code == GS_ETIMEOUT, e.value
    _lib.check(L.gs_plan_tune(m._plan, GS_TUNE_SWEEP_BUDGET, default))
    m.flowAccumulation()
    ref.flowAccumulation()
    _same_flow(m, ref)
    m.destroy()
    ref.destroy()


def _oracle_mesh(fv, coords, cells):
    return dict(coords=coords, cells=cells, nb=fv.n, flat=fv.flat, nnb=fv.nnb, ngb=fv.ngb, elgt=fv.elgt,
                vdist=fv.vdist, farea=fv.farea, larea=fv.larea, maxarea=fv.maxarea, outlet=fv.outlet,
                open_nodes=fv.open_nodes, borders=fv.outlet)


def test_zero_area_cell():
    """An interior cell of zero area: no rain volume, flow accumulation and
    SPL as in the oracle.  goSPL's diffusion row for it is all zero
    (sethillslopecoeff skips rows without area, functions.F90:918), a
    singular system that PETSc's zero-pivot shift solves to an arbitrary
    value; here the row is held fixed: the cell keeps its elevation and the
    rest of the solve stays finite."""
    import torch
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    from oracle.model import OracleModel
    coords, cells, z, rain, up, p = S.planar_config(n=3000, side=30.0e3, seed=3)
    p = dict(p, rain=rain, upsub=up, tEnd=10 * p["dt"])
    fv = FVMesh(coords, cells, p["bc"])
    k = int(np.argmin(np.abs(coords[:, 0] - 15.0e3) + np.abs(coords[:, 1] - 15.0e3)))
    fv.farea = fv.farea.copy()
    fv.larea = fv.larea.copy()
    fv.farea[k] = 0.0
    fv.larea[k] = 0.0
    gm = Model(coords=coords, cells=cells, elev=z, params=p, mesh=fv, device="cuda:0")
    om = OracleModel(coords, cells, z, p, mesh=_oracle_mesh(fv, coords, cells))
    assert float(gm.bL[k]) == 0.0 and om.bL[k] == 0.0
    for stage in ("flowAccumulation", "erodepSPL"):
        getattr(gm, stage)()
        getattr(om, stage)()
        torch.cuda.synchronize()
    assert np.array_equal(gm.rcvIDi.cpu().numpy(), om.rcvIDi)
    assert np.array_equal(gm.pitIDs.cpu().numpy(), om.pitIDs)
    fal = gm.FAL.cpu().numpy()
    assert np.abs(fal - om.FAL).max() <= 1e-12 * np.abs(om.FAL).max()
    h = gm.hGlobal.cpu().numpy()
    assert np.abs(h - om.h).max() <= 1e-12 * np.abs(om.h).max()
    hk = float(gm.hGlobal[k])
    gm.getHillslope()
    torch.cuda.synchronize()
    assert torch.isfinite(gm.hGlobal).all()
    assert float(gm.hGlobal[k]) == hk
    gm.destroy()


def test_closed_domain_with_undrainable_depressions_steps_like_the_oracle():
    """Walls on every side, no sea: no cell drains, so no depression fills
    and the continental routing keeps the stray sinks' sediment in place."""
    import torch
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    from oracle.model import OracleModel
    coords, cells, z, rain, up, p = S.planar_config(n=3000, side=30.0e3, seed=3)
    p = dict(p, rain=rain, upsub=None, bc="wwww", nodep=False, tEnd=10 * p["dt"])
    fv = FVMesh(coords, cells, "wwww")
    gm = Model(coords=coords, cells=cells, elev=z, params=p, mesh=fv, device="cuda:0")
    om = OracleModel(coords, cells, z, p, mesh=_oracle_mesh(fv, coords, cells))
    gm.step()
    om.step()
    torch.cuda.synchronize()
    assert np.array_equal(gm.rcvIDi.cpu().numpy(), om.rcvIDi)
    assert np.array_equal(gm.pitIDs.cpu().numpy(), om.pitIDs)
    for k in ("FAL", "cumED"):
        a, b = getattr(gm, k).cpu().numpy(), getattr(om, k)
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1.0), k
    h = gm.hGlobal.cpu().numpy()
    assert np.abs(h - om.h).max() <= 1e-10 * np.abs(om.h).max()
    gm.destroy()
