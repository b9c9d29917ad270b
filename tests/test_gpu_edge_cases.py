"""Edge cases of the reference's boundary and terrain handling, each one
physics step on the GPU against the oracle from the same initial state:
wall and mixed boundaries, exactly flat plateaus (ties everywhere), marine
cells above part of the land, a very small mesh, and an empty plan."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _step_vs_oracle(coords, cells, z, params):
    import torch
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    from oracle.model import OracleModel

    fv = FVMesh(coords, cells, params["bc"])
    gm = Model(coords=coords, cells=cells, elev=z, params=params, mesh=fv, device="cuda:0")
    mesh = dict(coords=coords, cells=cells, nb=fv.n, flat=fv.flat, nnb=fv.nnb, ngb=fv.ngb, elgt=fv.elgt,
                vdist=fv.vdist, farea=fv.farea, larea=fv.larea, maxarea=fv.maxarea, outlet=fv.outlet,
                open_nodes=fv.open_nodes, borders=fv.outlet)
    om = OracleModel(coords, cells, z, params, mesh=mesh)
    gm.step()
    om.step()
    torch.cuda.synchronize()
    assert np.array_equal(gm.rcvIDi.cpu().numpy(), om.rcvIDi), "receivers"
    assert np.array_equal(gm.pitIDs.cpu().numpy(), om.pitIDs), "pit ids"
    assert np.array_equal(gm.flatDirs.cpu().numpy(), om.flatDirs), "flat directions"
    fal = gm.FAL.cpu().numpy()
    assert np.abs(fal - om.FAL).max() <= 1e-10 * max(np.abs(om.FAL).max(), 1.0), "drainage area"
    h = gm.hGlobal.cpu().numpy()
    assert np.abs(h - om.h).max() <= 1e-10 * max(np.abs(om.h).max(), 1.0), "elevation"
    if not params.get("nodep", True):
        vs = gm.vSed.cpu().numpy()
        assert np.abs(vs - om.vSed).max() <= 1e-10 * max(np.abs(om.vSed).max(), 1.0), "sediment flux"
        cum = gm.cumED.cpu().numpy()
        assert np.abs(cum - om.cumED).max() <= 1e-10 * max(np.abs(om.h).max(), 1.0), "cumED"
    gm.destroy()


def _planar(n, seed, bc, zmax=50.0, sealevel=-100.0, flat=False):
    from gospl_b200 import synthetic as S
    side = 537.0 * np.sqrt(n * np.sqrt(3) / 2)
    coords, cells, onb = S.planar_hex_mesh(n, side, seed=seed)
    z = S.rescale(S.fractal_field(coords[:, :2], side, seed + 1), 0.0, zmax)
    if flat:
        # plateau at exactly 20 m with a few bumps: ties everywhere
        z = np.where(z > 0.8 * zmax, z, 20.0)
    z[onb] = 0.0
    params = dict(dt=1000.0, tStart=0.0, tEnd=1e4, flowDir=3, K=2e-6, d=0.0, m=0.5, Cda=0.1, Cdm=0.05,
                  sealevel=sealevel, oFill=-6000.0, bc=bc, rain=np.ones(len(z)), upsub=np.full(len(z), 1e-3))
    return coords, cells, z, params


@pytest.mark.parametrize("bc", ["wfwf", "wwwf", "fwow"])
def test_wall_and_mixed_boundaries(bc):
    _step_vs_oracle(*_planar(2500, 21, bc))


def test_flat_plateau_ties():
    _step_vs_oracle(*_planar(2500, 23, "ffff", flat=True))


def test_marine_cells():
    _step_vs_oracle(*_planar(2500, 25, "ffff", sealevel=20.0))


def test_tiny_mesh():
    _step_vs_oracle(*_planar(40, 27, "ffff"))


def test_empty_plan():
    import ctypes
    from gospl_b200 import _lib
    L = _lib.load()
    z = np.zeros(0, np.int32)
    d = np.zeros(0)
    plan = ctypes.c_void_p()
    _lib.check(L.gs_plan_create(0, _lib.ptr(z), _lib.ptr(z), _lib.ptr(d), _lib.ptr(d), _lib.ptr(d), _lib.ptr(d),
                                _lib.ptr(z), 0, _lib.ptr(z), 0, 1, 3, ctypes.byref(plan)))
    st = _lib.GsStats()
    _lib.check(L.gs_flow_accumulation(plan, None, None, 0.0, -6000.0, 1.0, None, None, None, None, None, None,
                                      None, None, None, None, None, ctypes.byref(st)))
    _lib.check(L.gs_plan_destroy(plan))


@pytest.mark.parametrize("G", [0.5, 1.0])
def test_transport_limited_spl(G):
    """spl: G > 0 (SPL.py:116-258, 305-336): the coupled erosion-deposition
    system against the oracle's sparse direct solve."""
    coords, cells, z, params = _planar(3000, 29, "ffff")
    params = dict(params, G=G)
    _step_vs_oracle(coords, cells, z, params)


@pytest.mark.parametrize("bc", ["ffff", "wwww", "wfwf"])
def test_continental_deposition(bc):
    """sedChange (sedplex.py:1061-1086) over open, closed (no outlet: stray
    sinks keep their sediment) and mixed boundaries, one step against the
    oracle."""
    coords, cells, z, params = _planar(3000, 31, bc)
    params = dict(params, nodep=False)
    _step_vs_oracle(coords, cells, z, params)


def test_lake_diffusion_path_rejected():
    """Partly filled depressions of at least nlPitVolume and nlPitDepth are
    smoothed by non-linear diffusion in goSPL (sedplex.py:679-858); with the
    default adaptive TS solver that path is not built and must fail loudly,
    not deposit something else (marineSolver picard builds it)."""
    import torch
    from gospl_b200 import _lib
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model
    coords, cells, z, params = _planar(3000, 31, "ffff")
    params = dict(params, nodep=False, nlPitVolume=0.0, nlPitDepth=0.0)
    fv = FVMesh(coords, cells, params["bc"])
    gm = Model(coords=coords, cells=cells, elev=z, params=params, mesh=fv, device="cuda:0")
    with pytest.raises(_lib.GsError, match="marineSolver picard"):
        gm.step()
    torch.cuda.synchronize()
    gm.destroy()


def test_transport_limited_with_deposition():
    """Both deposition paths of goSPL in one step: transport-limited erosion
    (G > 0, SPL.py:305-336) followed by continental sediment routing
    (sedplex.py:1061-1086)."""
    coords, cells, z, params = _planar(3000, 33, "ffff")
    params = dict(params, G=1.0, nodep=False)
    _step_vs_oracle(coords, cells, z, params)


@pytest.mark.parametrize("bc", ["ffff", "wwww"])
def test_lake_diffusion_picard(bc):
    """Path 3 of the lake deposits with marineSolver picard: every partly
    filled depression (nlPitVolume = nlPitDepth = 0) gets the inlet pile, the
    lagged-diffusivity sub-steps and the per-pit rescale, against the oracle."""
    coords, cells, z, params = _planar(3000, 31, bc)
    params = dict(params, nodep=False, nlPitVolume=0.0, nlPitDepth=0.0, marineSolver="picard", picardSub=3,
                  picardIts=2)
    _step_vs_oracle(coords, cells, z, params)
