"""Parity at the benchmark's full size: the 2,621,442-vertex sphere (icosphere
level 9) used by bench.py, every stage of one step from identical state on the
GPU and in the oracle.  The oracle's fill, receivers and triangular solves are
C and finish in seconds at this size; both sides use the GPU-built
finite-volume arrays (tests/test_mesh.py checks them against the oracle's
geometry on the golden meshes).  Exact for receivers, pits, flat directions,
the filled surface and the sediment fill; 1e-12 relative for drainage area,
sediment flux and elevation, as in the small-mesh stage parity tests."""
import numpy as np
import pytest

from test_gpu_parity import _compare_dz, _compare_flow, _compare_sed, _resync, _resync_flow

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sphere():
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    c, f, z, rain, up, p = S.sphere_config(level=9)
    p = dict(p, rain=rain, upsub=up, nodep=False, nlPitVolume=float("inf"))
    fv = FVMesh(c, f, p["bc"], device="cuda:0")
    mesh = dict(coords=c, cells=f, nb=fv.n, flat=fv.flat, nnb=fv.nnb, ngb=fv.ngb, elgt=fv.elgt, vdist=fv.vdist,
                farea=fv.farea, larea=fv.larea, maxarea=fv.maxarea, outlet=fv.outlet, open_nodes=fv.open_nodes,
                borders=fv.outlet)
    return c, f, z, p, fv, mesh


def test_full_size_stage_parity(sphere):
    import torch
    from gospl_b200.model import Model
    from oracle.model import OracleModel
    c, f, z, p, fv, mesh = sphere
    gm = Model(coords=c, cells=f, elev=z, params=p, mesh=fv, device="cuda:0", init_flow=False)
    om = OracleModel(c, f, z, p, mesh=mesh, init_flow=False)
    assert np.array_equal(gm.hGlobal.cpu().numpy(), om.h)
    tag = "sphere2621442"
    gm.flowAccumulation()
    om.flowAccumulation()
    _compare_flow(gm, om, tag + " flow", 1e-12)
    _resync_flow(gm, om)
    gm.erodepSPL()
    om.erodepSPL()
    torch.cuda.synchronize()
    _compare_dz(gm, om, tag + " spl")
    _resync(gm, om)
    gm.flowAccumulation()
    om.flowAccumulation()
    _compare_flow(gm, om, tag + " flow2", 1e-12)
    _resync_flow(gm, om)
    gm.sedChange()
    om.sedChange()
    _compare_sed(gm, om, tag + " sed")
    _resync(gm, om)
    gm.getHillslope()
    om.getHillslope()
    torch.cuda.synchronize()
    _compare_dz(gm, om, tag + " hillslope")
    gm.destroy()
