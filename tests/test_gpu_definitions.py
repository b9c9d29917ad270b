"""CUDA kernels against the independent definitions of goSPL's Fortran
kernels (tests/definitions.py), and the Python-level boundary methods
fillElevation(sed) and _buildFlowDirection(h, down) against the oracle.

For every golden fixture, closed / open / mixed planar domains and a plateau
with ties everywhere: the GPU's filled surface is the Priority-Flood (bit for
bit), depression ids the equal-fill components, flat directions the
breadth-first distances from the spill nodes, receivers the steepest slopes
(indices and distances exact, weights to 1e-15), pit and filled volumes their
sums (1e-14).  Exact slope ties go through the C ABI with gid = 0 and must
pick the same receivers as the oracle's literal quicksort.  The 2,621,442-
vertex sphere runs the same checks with the minimum-spanning-tree form of the
fill, and reports the near-tie count of its receiver slopes.
"""
import numpy as np
import pytest

import definitions as D
from test_definitions import CASES, _oracle, fill_level

pytestmark = pytest.mark.gpu


def _model_like(om, device="cuda:0"):
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    m = om.mesh
    fv = FVMesh.from_arrays(dict(nnb=m["nnb"], ngb=m["ngb"], elgt=m["elgt"], vdist=m["vdist"], farea=m["farea"],
                                 larea=m["larea"], outlet=m["outlet"], open_nodes=m["open_nodes"], flat=m["flat"]))
    p = dict(dt=om.dt, tEnd=om.tEnd, flowDir=om.flowDir, K=om.K, d=om.coeffd, m=om.spl_m, Cda=om.Cda, Cdm=om.Cdm,
             oFill=om.oFill, sealevel=om.sealevel, rain=np.ones(om.lpoints), upsub=None)
    return Model(coords=m.get("coords"), cells=m.get("cells"), elev=om.h.copy(), params=p, mesh=fv, device=device,
                 init_flow=False)


def _np(x):
    return x.cpu().numpy()


def check_gpu_fill(gm, om, h, sed, tag, large=False):
    import torch
    gm.hGlobal.copy_(torch.as_tensor(h))
    gm.fillElevation(sed=sed)
    torch.cuda.synchronize()
    ngb = om.FVmesh_ngbID
    level = fill_level(om, h)
    outm = np.zeros(om.lpoints, dtype=bool)
    outm[om.outletIDs] = True
    lf = D.filled_surface(h, level, ngb, outm, om.sealevel, sed=sed, large=large)
    sea = lf <= om.sealevel
    assert np.array_equal(_np(gm.lFill), np.where(sea, h, lf)), "%s lFill" % tag
    pid = D.pit_ids(lf, ngb, level if sed else om.sealevel, om.outletIDs)
    assert np.array_equal(_np(gm.pitIDs).astype(np.int64), pid), "%s pitIDs" % tag
    pp, pi, fl, fv = (_np(x) for x in gm.pit_tables())
    spills = np.unique(pi[(pi[:, 1] == 0) & (pi[:, 0] >= 0), 0])
    pd = D.flat_distance(spills, pid, lf, ngb)
    fd = D.flat_dirs(pd, pid, lf, ngb, spills, om.sealevel)
    assert np.array_equal(_np(gm.flatDirs).astype(np.int64), fd), "%s flatDirs" % tag
    hh = h.copy()
    if not sed:
        hh[hh < om.sealevel] = om.sealevel
    pv = D.pit_volumes(pid, _np(gm.lFill), hh, om.larea, len(pp))
    assert np.abs(pv - pp[:, 0]).max() <= 1e-14 * max(float(np.abs(pp[:, 0]).max()), 1e-300), "%s pit volumes" % tag
    fvd = D.filled_volumes(pid, hh, om.mesh["farea"], fl[:, :4])
    assert np.abs(fvd - fv[:, :4]).max() <= 1e-14 * max(float(np.abs(fv).max()), 1e-300), "%s filled vol" % tag
    return lf


def check_gpu_receivers(gm, om, h, tag):
    import torch
    ngb = om.FVmesh_ngbID
    gm._buildFlowDirection(torch.as_tensor(h), down=False)
    torch.cuda.synchronize()
    rcv, dist, wgt, ties, slp = D.mfd_receivers(h, ngb, om.mesh["elgt"], om.sealevel, om.flowDir)
    if om.flatModel:
        o = np.asarray(om.outletIDs, dtype=np.int64)
        rcv[o] = o[:, None]
        dist[o] = 0.0
        wgt[o] = 0.0
    nt = ~ties
    assert np.array_equal(_np(gm.rcvID)[nt], rcv[nt]), "%s rcv" % tag
    assert np.array_equal(_np(gm.distRcv)[nt], dist[nt]), "%s dist" % tag
    assert np.abs(_np(gm.wghtVal) - wgt).max() <= 1e-15, "%s wgt" % tag
    return D.near_ties(slp, om.flowDir)


@pytest.mark.parametrize("case", CASES)
def test_gpu_fill_and_receivers_are_their_definitions(case):
    om = _oracle(case)
    gm = _model_like(om)
    h0 = om.h.copy()
    check_gpu_fill(gm, om, h0, False, case)
    check_gpu_fill(gm, om, h0, True, case + " sed")
    check_gpu_receivers(gm, om, h0, case)
    gm.destroy()


@pytest.mark.parametrize("case", ["planar2k", "ico2562", "wfwf", "flat_ffff"])
def test_boundary_methods_match_the_oracle(case):
    """fillElevation(sed) and _buildFlowDirection(h, down) called on their
    own, as goSPL's callers may: the model's lFill, pitIDs, flatDirs, live
    receivers, lsink and seaID equal the oracle's after the same calls."""
    import torch
    om = _oracle(case)
    gm = _model_like(om)
    h0 = om.h.copy()
    for sed in (False, True):
        for down in (True, False):
            om.h = h0.copy()
            om.fillElevation(sed=sed)
            gm.hGlobal.copy_(torch.as_tensor(h0))
            gm.fillElevation(sed=sed)
            surf = om.lFill.copy()
            om._buildFlowDirection(surf, down=down)
            gm._buildFlowDirection(torch.as_tensor(surf), down=down)
            torch.cuda.synchronize()
            tag = "%s sed=%s down=%s" % (case, sed, down)
            assert np.array_equal(_np(gm.lFill), om.lFill), tag
            assert np.array_equal(_np(gm.pitIDs), om.pitIDs), tag
            assert np.array_equal(_np(gm.flatDirs), om.flatDirs), tag
            assert np.array_equal(_np(gm.rcvID), om.rcvID), tag
            assert np.array_equal(_np(gm.distRcv), om.distRcv), tag
            assert np.abs(_np(gm.wghtVal) - om.wghtVal).max() <= 1e-15, tag
            assert np.array_equal(_np(gm.lsink), om.lsink), tag
            sea = np.zeros(om.lpoints, dtype=bool)
            sea[om.seaID] = True
            assert np.array_equal(_np(gm.seaID), sea), tag
    gm.destroy()


def test_gpu_receivers_on_built_ties():
    """Exact slope ties through gs_mfdreceivers with gid = 0: the receivers,
    distances and weights equal the oracle's literal replay of the reference
    quicksort at every vertex, ties included."""
    import torch
    from gospl_b200 import _lib
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    from oracle import fortran as F
    from oracle import mesh as M
    coords, cells, onb = S.planar_hex_mesh(3000, 30.0e3, seed=5, jitter=0.0)
    mesh = M.build_mesh(coords, cells, "ffff")
    M.load_mesh(mesh)
    rng = np.random.default_rng(7)
    h = rng.integers(0, 6, len(coords)).astype(np.float64)
    R = 3
    gid = np.zeros(len(coords), dtype=np.int32)
    r2, d2, w2 = F.mfdreceivers(R, 1.1, h, -100.0, gid)
    *_, ties, _ = D.mfd_receivers(h, mesh["ngb"].astype(np.int64), mesh["elgt"], -100.0, R, gid=gid)
    assert ties.sum() > 100
    fv = FVMesh(coords, cells, "ffff")
    p = dict(dt=1000.0, tEnd=1e4, flowDir=R, K=2e-6, d=0.0, m=0.5, sealevel=-100.0, rain=np.ones(len(h)),
             upsub=None)
    gm = Model(coords=coords, cells=cells, elev=h, params=p, mesh=fv, init_flow=False)
    dev = gm.dev
    n = len(h)
    rcv = torch.empty((R, n), dtype=torch.int32, device=dev)
    dist = torch.empty((R, n), dtype=torch.float64, device=dev)
    wgt = torch.empty((R, n), dtype=torch.float64, device=dev)
    hd = torch.as_tensor(h, device=dev)
    gd = torch.as_tensor(gid, device=dev)
    L = _lib.load()
    _lib.check(L.gs_mfdreceivers(gm._plan, R, 1.1, _lib.ptr(hd), -100.0, _lib.ptr(gd), _lib.ptr(rcv),
                                 _lib.ptr(dist), _lib.ptr(wgt)))
    torch.cuda.synchronize()
    assert np.array_equal(_np(rcv).T, r2)
    assert np.array_equal(_np(dist).T, d2)
    assert np.abs(_np(wgt).T - w2).max() <= 1e-15
    gm.destroy()


def test_gpu_definitions_at_full_size(capsys):
    """The 2,621,442-vertex sphere of the benchmark: fill, depression ids,
    flat directions and receivers of the GPU against the definitions (fill
    by the minimum spanning tree), and the near-tie count of the slopes."""
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from oracle.model import OracleModel
    c, f, z, rain, up, p = S.sphere_config(level=9)
    p = dict(p, rain=rain, upsub=up)
    fv = FVMesh(c, f, p["bc"], device="cuda:0")
    mesh = dict(coords=c, cells=f, nb=fv.n, flat=fv.flat, nnb=fv.nnb, ngb=fv.ngb, elgt=fv.elgt, vdist=fv.vdist,
                farea=fv.farea, larea=fv.larea, maxarea=fv.maxarea, outlet=fv.outlet, open_nodes=fv.open_nodes,
                borders=fv.outlet)
    om = OracleModel(c, f, z, p, mesh=mesh, init_flow=False)
    gm = _model_like(om)
    h0 = om.h.copy()
    check_gpu_fill(gm, om, h0, False, "sphere", large=True)
    near = check_gpu_receivers(gm, om, h0, "sphere")
    with capsys.disabled():
        print("\nsphere 2621442: receiver slope pairs within 4 ulp among the %d steepest: %d"
              % (om.flowDir + 1, near))
    gm.destroy()


@pytest.mark.parametrize("window", [0, 1, 8, 64, 4096])
def test_flat_bfs_forms_are_the_definition(window):
    """The flat distances (and so flatDirs) are the same breadth-first hop
    counts whichever form computes them (GS_TUNE_FLAT_BFS): the one-block
    BFS (0) and the tiled delta-stepping BFS with windows of 1 to 4096
    levels, on a lake-rich planar case, the icosphere and a plateau."""
    from gospl_b200 import _lib
    L = _lib.load()
    for case in ("planar2k", "ico2562", "flat_ffff"):
        om = _oracle(case)
        gm = _model_like(om)
        _lib.check(L.gs_plan_tune(gm._plan, 7, window))
        assert L.gs_plan_tuning(gm._plan, 7) == window
        h0 = om.h.copy()
        check_gpu_fill(gm, om, h0, False, "%s window %d" % (case, window))
        check_gpu_fill(gm, om, h0, True, "%s sed window %d" % (case, window))
        gm.destroy()


def test_fill_is_the_definition_when_the_basin_pair_table_overflows():
    """The basin-pair table of the fill's relaxation is sized from the plan's
    previous fill.  A tilted plane first (no interior basin: the smallest
    table), then white-noise relief on the same plan (hundreds of basins and
    thousands of basin pairs: probing gives up and the relaxation takes the
    edges as emitted), then the same relief again (the table has grown): the
    filled surface, the labels and the flat directions are their definitions
    every time."""
    from test_definitions import _planar_oracle
    om = _planar_oracle("ffff", n=6000, seed=9)
    gm = _model_like(om)
    xy = np.asarray(om.mesh["coords"])[:, :2]
    onb = np.zeros(om.lpoints, bool)
    onb[om.outletIDs] = True
    plane = 1.0 + 1.0e-3 * (xy[:, 0] - xy[:, 0].min())
    plane[onb] = 0.0
    noise = np.random.default_rng(12).uniform(1.0, 50.0, om.lpoints)
    noise[onb] = 0.0
    for h, tag in ((plane, "plane"), (noise, "noise, small table"), (noise, "noise, grown table")):
        check_gpu_fill(gm, om, h, False, tag)
    gm.destroy()
