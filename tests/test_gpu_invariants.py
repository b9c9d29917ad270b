"""Invariants goSPL's own regression tests hold for this path
(tests/test_regression.py of the reference), checked on the GPU path:

- the snapshot receivers (test_regression.py:3049-3126): rcvIDi, wghtVali
  and distRcvi do not share storage with the live receivers, and sedChange,
  which rebuilds the live graph on the sediment-filled surface, leaves them
  byte-equal;
- the sign conventions of cumED and EbLocal (:3189-3277): at every node that
  lost elevation by erosion over a run (elevation and cumED both down by more
  than 1 um), cumED decreased and EbLocal <= 0;
- the union-find of the depression labels (:1412-1447, goSPL's cross-rank
  _unifyLabels): equal-fill regions collapse to one id per connected
  component whatever the path between their cells, across multi-hop chains
  (a winding depression) and merges through one shared node (two arms
  meeting at a vertex), ids and numbering as scipy's connected components of
  the equal-fill graph give them (tests/definitions.py);
- mass conservation on a closed domain (:3304-3440) is the sediment budget's
  closure, tests/test_gpu_budget.py.
"""
import numpy as np
import pytest

import definitions as D

pytestmark = pytest.mark.gpu


def _planar_model(nodep, bc="ffff", n=3000, seed=3, uplift=True):
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    coords, cells, z, rain, up, p = S.planar_config(n=n, side=30.0e3, seed=seed)
    p = dict(p, rain=rain, upsub=up if uplift else None, nodep=nodep, bc=bc, marineSolver="picard",
             tEnd=20 * p["dt"])
    return Model(coords=coords, cells=cells, elev=z, params=p, mesh=FVMesh(coords, cells, bc), device="cuda:0")


def test_snapshot_receivers_are_not_the_live_ones_and_sedchange_keeps_them():
    import torch
    m = _planar_model(nodep=False)
    m.step()
    m.flowAccumulation()
    m.erodepSPL()
    m.flowAccumulation()
    torch.cuda.synchronize()
    m._buildFlowDirection(m.lFill, down=True)     # the live graph exists
    for a, b in (("rcvIDi", "rcvID"), ("wghtVali", "wghtVal"), ("distRcvi", "distRcv")):
        assert getattr(m, a).data_ptr() != getattr(m, b).data_ptr(), a
    before = [x.clone() for x in (m.rcvIDi, m.wghtVali, m.distRcvi)]
    m.sedChange()
    torch.cuda.synchronize()
    assert m.stats["sed"]["cascade_passes"] >= 1
    for x, y, name in zip((m.rcvIDi, m.wghtVali, m.distRcvi), before, ("rcvIDi", "wghtVali", "distRcvi")):
        assert torch.equal(x, y), "sedChange changed the snapshot " + name
    m.destroy()


@pytest.mark.parametrize("case", ["incising", "incising_sed"])
def test_erosion_sign_conventions(case):
    """On goSPL's own incising fixture (tests/fixtures/incising.npz of the
    reference, the one its sign-convention test runs), without and with
    continental deposition, over the fixture's run."""
    import torch
    from conftest import golden_params, load_golden
    from test_gpu_parity import _gpu_model
    g = load_golden(case)
    m = _gpu_model(g, golden_params(g))
    h0, c0 = m.hGlobal.clone(), m.cumED.clone()
    for _ in range(int(g["nsteps"])):
        m.step()
    torch.cuda.synchronize()
    dh = (m.hGlobal - h0).cpu().numpy()
    dc = (m.cumED - c0).cpu().numpy()
    inc = (dh < -1.0e-6) & (dc < -1.0e-6)
    assert inc.sum() > 10, "the landscape must incise"
    assert dc[inc].max() < 0.0
    assert (m.EbLocal.cpu().numpy()[inc] <= 0.0).all(), "EbLocal > 0 at an eroding node"
    m.destroy()


def _designed_depressions(coords, onb):
    """A winding depression (a zig-zag trench, so its flat after filling is
    a multi-hop chain of equal-fill cells) and a Y of two trenches meeting at
    one vertex, cut into a plateau that drains to the open border."""
    x, y = coords[:, 0], coords[:, 1]
    L = x.max() - x.min()
    x0, y0 = x.min(), y.min()
    z = 60.0 + 0.002 * (x - x0)                      # plateau tilted towards x = x0

    def trench(p, q, width):
        p, q = np.asarray(p, float), np.asarray(q, float)
        d = q - p
        t = np.clip(((x - p[0]) * d[0] + (y - p[1]) * d[1]) / (d @ d), 0.0, 1.0)
        return np.hypot(x - (p[0] + t * d[0]), y - (p[1] + t * d[1])) < width

    w = 0.03 * L
    zig = np.zeros(len(z), bool)
    pts = [(0.15, 0.2), (0.3, 0.8), (0.45, 0.2), (0.6, 0.8), (0.75, 0.2)]
    for a, b in zip(pts, pts[1:]):
        zig |= trench((x0 + a[0] * L, y0 + a[1] * L), (x0 + b[0] * L, y0 + b[1] * L), w)
    j = (x0 + 0.92 * L, y0 + 0.5 * L)
    yy = trench((x0 + 0.85 * L, y0 + 0.1 * L), j, w) | trench((x0 + 0.85 * L, y0 + 0.9 * L), j, w)
    rng = np.random.default_rng(11)
    z = np.where(zig | yy, 20.0 + rng.uniform(0.0, 5.0, len(z)), z)
    z[onb] = 0.0
    return z, zig, yy


def test_equal_fill_components_collapse_across_chains_and_shared_nodes():
    import torch
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    from oracle.model import OracleModel
    from test_definitions import fill_level
    coords, cells, onb = S.planar_hex_mesh(6000, 40.0e3, seed=17)
    # the oracle only supplies the mesh tables and the fill level here
    z, zig, yy = _designed_depressions(coords, onb)
    p = dict(dt=1000.0, tStart=0.0, tEnd=1e4, flowDir=3, K=2e-6, d=0.0, m=0.5, Cda=0.1, Cdm=0.05,
             sealevel=-100.0, oFill=-6000.0, bc="ffff", rain=np.ones(len(z)), upsub=None)
    om = OracleModel(coords, cells, z, p, init_flow=False)
    gm = Model(coords=coords, cells=cells, elev=z, params=p, mesh=FVMesh(coords, cells, "ffff"), device="cuda:0",
               init_flow=False)
    gm.fillElevation(sed=False)
    torch.cuda.synchronize()
    ngb = om.FVmesh_ngbID
    outm = np.zeros(om.lpoints, bool)
    outm[om.outletIDs] = True
    level = fill_level(om, z)
    lf = D.filled_surface(z, level, ngb, outm, om.sealevel)
    pid_def = D.pit_ids(lf, ngb, om.sealevel, om.outletIDs)
    pid = gm.pitIDs.cpu().numpy().astype(np.int64)
    assert np.array_equal(gm.lFill.cpu().numpy(), np.where(lf <= om.sealevel, z, lf))
    assert np.array_equal(pid, pid_def)
    # each trench system is one depression: the chain and the Y collapse
    for name, mask in (("zig-zag", zig), ("Y", yy)):
        ids = np.unique(pid[mask])
        assert len(ids) == 1 and ids[0] > 0, "%s split into %s" % (name, ids)
    assert np.unique(pid[zig])[0] != np.unique(pid[yy])[0]
    gm.destroy()
