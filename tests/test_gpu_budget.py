"""Sediment budget on the GPU (gs_sed_budget), closed to 1e-12 of the eroded
volume, against the oracle's budget.

The device sums, in a fixed order, where the volume eroded by the step's SPL
goes in the continental routing (depressions, closed-domain sinks, outlets,
sea, and what goSPL's routing rules drop).  On closed (wwww), open (ffff)
and mixed (wfwf) planar domains every step must close to 1e-12 of the eroded
volume; the first step, from the same initial state as the oracle, must give
the oracle's terms to 1e-11 of it.  The 2,621,442-vertex sphere is covered by
tests/test_gpu_fullsize.py (its sedChange comparison checks the budget).
"""
import numpy as np
import pytest

from test_budget import _planar

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bc", ["wwww", "ffff", "wfwf"])
def test_gpu_budget_closes_and_matches_oracle(bc):
    import torch
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    from oracle.model import OracleModel
    from test_gpu_parity import BUDGET_TERMS

    coords, cells, z, p = _planar(bc)
    fv = FVMesh(coords, cells, p["bc"])
    gm = Model(coords=coords, cells=cells, elev=z, params=p, mesh=fv, device="cuda:0")
    mesh = dict(coords=coords, cells=cells, nb=fv.n, flat=fv.flat, nnb=fv.nnb, ngb=fv.ngb, elgt=fv.elgt,
                vdist=fv.vdist, farea=fv.farea, larea=fv.larea, maxarea=fv.maxarea, outlet=fv.outlet,
                open_nodes=fv.open_nodes, borders=fv.outlet)
    om = OracleModel(coords, cells, z, p, mesh=mesh)
    for s in range(3):
        gm.step()
        torch.cuda.synchronize()
        b = gm.sed_budget()
        E = b["eroded"]
        assert E > 0.0
        assert abs(b["closure"]) <= 1e-12 * E, "%s step %d: closure %g of the eroded volume" % (
            bc, s, b["closure"] / E)
        assert abs(b["pit_sinks"] - b["inflow"]) <= 1e-12 * E
        if s == 0:
            om.step()
            bo = om.sed_budget
            for k in BUDGET_TERMS:
                assert abs(b[k] - bo[k]) <= 1e-11 * E, "%s %s: %r vs %r" % (bc, k, b[k], bo[k])
            hs = float(np.abs(om.h).max())
            assert abs(b["realised"] - bo["realised"]) <= 1e-11 * E + 1e-12 * hs * float(fv.larea.sum())
    gm.destroy()
