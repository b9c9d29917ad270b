"""The oracle's C restatement of goSPL's Fortran kernels against independent
definitions (tests/definitions.py), on every golden fixture and on synthetic
closed, open and mixed domains.

goSPL's Fortran module cannot be compiled here (no Fortran compiler), so its
kernels are pinned by what they are defined to compute: the filled surface
is the Priority-Flood of Barnes et al. (2014) and equally the minimum
spanning tree's minimax fill; depression ids are the equal-fill components
that hold a bottom; flat distances are breadth-first hop counts from the
spill nodes; receivers are the steepest candidate slopes; pit volumes,
filled volumes and hillslope coefficients are their sums and formulas.
Integer and index results must be identical, the filled surface bit for bit;
sums agree to 1e-15 relative (summation order).  tests/test_gpu_definitions.py
checks the CUDA kernels against the same definitions.
"""
import numpy as np
import pytest

import definitions as D
from conftest import GOLDEN_CASES, GOLDEN_SED_CASES, golden_mesh, golden_params, load_golden


def _golden_oracle(case):
    from oracle.model import OracleModel
    g = load_golden(case)
    return OracleModel(g["v"], g["c"], g["z"], golden_params(g), mesh=golden_mesh(g), init_flow=False)


def _planar_oracle(bc, n=2500, seed=21, flat=False):
    from gospl_b200 import synthetic as S
    from oracle.model import OracleModel
    side = 537.0 * np.sqrt(n * np.sqrt(3) / 2)
    coords, cells, onb = S.planar_hex_mesh(n, side, seed=seed)
    z = S.rescale(S.fractal_field(coords[:, :2], side, seed + 1), 0.0, 50.0)
    if flat:
        z = np.where(z > 40.0, z, 20.0)
    z[onb] = 0.0
    params = dict(dt=1000.0, tStart=0.0, tEnd=1e4, flowDir=3, K=2e-6, d=0.0, m=0.5, Cda=0.1, Cdm=0.05,
                  sealevel=-100.0, oFill=-6000.0, bc=bc, rain=np.ones(len(z)), upsub=None)
    return OracleModel(coords, cells, z, params, init_flow=False)


CASES = GOLDEN_CASES + ["planar2k_lake", "wwww", "ffff", "wfwf", "flat_ffff"]


def _oracle(case):
    if case in ("wwww", "ffff", "wfwf"):
        return _planar_oracle(case)
    if case == "flat_ffff":
        return _planar_oracle("ffff", flat=True)
    return _golden_oracle(case)


def fill_level(om, h):
    """The fill level of fillElevation (pitfilling.py:858-866)."""
    minh = h.min() + (0.0 if om.flatModel else 1.0e-3)
    return max(minh, om.sealevel + om.oFill)


def check_fill_stage(om, h, sed, tag):
    """Runs the oracle's fillElevation(sed) on h and checks every Fortran
    product against its definition."""
    ngb = om.FVmesh_ngbID
    m = om.mesh
    om.h = h.copy()
    om.fillElevation(sed=sed)
    level = fill_level(om, h)
    outm = np.zeros(om.lpoints, dtype=bool)
    outm[om.outletIDs] = True
    lf = D.filled_surface(h, level, ngb, outm, om.sealevel, sed=sed)
    lf_big = D.filled_surface(h, level, ngb, outm, om.sealevel, sed=sed, large=True)
    assert np.array_equal(lf, lf_big), "%s: Priority-Flood and minimum spanning tree disagree" % tag
    sea = lf <= om.sealevel
    assert np.array_equal(np.where(sea, h, lf), om.lFill), "%s lFill" % tag
    pid = D.pit_ids(lf, ngb, level if sed else om.sealevel, om.outletIDs)
    assert np.array_equal(pid, om.pitIDs), "%s pitIDs" % tag
    pd = D.flat_distance(om.lspillIDs, om.pitIDs, lf, ngb)
    assert np.array_equal(pd, om.pdir), "%s flat distance" % tag
    fd = D.flat_dirs(pd, om.pitIDs, lf, ngb, om.lspillIDs, om.sealevel)
    assert np.array_equal(fd, om.flatDirs), "%s flatDirs" % tag
    hh = h.copy()
    if not sed:
        hh[hh < om.sealevel] = om.sealevel
    P = len(om.pitParams)
    pv = D.pit_volumes(om.pitIDs, om.lFill, hh, om.larea, P)
    scale = max(float(np.abs(om.pitParams[:, 0]).max()), 1e-300)
    assert np.abs(pv - om.pitParams[:, 0]).max() <= 1e-15 * scale, "%s pit volumes" % tag
    fv = D.filled_volumes(om.pitIDs, hh, m["farea"], om.filled_lvl[:, :4])
    scale = max(float(np.abs(om.filled_vol).max()), 1e-300)
    assert np.abs(fv - om.filled_vol[:, :4]).max() <= 1e-15 * scale, "%s filled volumes" % tag
    return int(om.pitIDs.max())


@pytest.mark.parametrize("case", CASES)
def test_fill_products_are_their_definitions(case):
    om = _oracle(case)
    h0 = om.h.copy()
    npits = check_fill_stage(om, h0, False, case)
    if case not in ("wwww",):
        assert npits > 0, "the case must hold depressions"
    # the sediment variant of the fill (marine depressions filled too, pits
    # above the fill level: pitfilling.py:690-692, 718-721)
    check_fill_stage(_oracle(case), h0, True, case + " sed")


@pytest.mark.parametrize("case", CASES)
def test_receivers_are_the_steepest_slopes(case):
    from oracle import fortran as F
    om = _oracle(case)
    h = om.h.copy()
    rcv, dist, wgt, ties, slp = D.mfd_receivers(h, om.FVmesh_ngbID, om.mesh["elgt"], om.sealevel, om.flowDir)
    r2, d2, w2 = F.mfdreceivers(om.flowDir, om.flowExp, h, om.sealevel, om.gid)
    nt = ~ties
    assert np.array_equal(rcv[nt], r2[nt]), case
    assert np.array_equal(dist[nt], d2[nt]), case
    assert np.abs(wgt - w2).max() <= 1e-15, case
    land = h > om.sealevel
    s = np.where(np.isnan(slp), 0.0, slp)
    assert np.all(np.abs(w2[land & (s.max(axis=1) > 0)].sum(axis=1) - 1.0) <= 4e-16), case


def test_receivers_on_built_ties():
    """Exact slope ties (a regular lattice, integer elevations, gid all 0 so
    the 1e-15 gid perturbation adds nothing): the choice among equal slopes is
    the reference quicksort's own order (functions.F90:683-762); the chosen
    slopes and weights are the definition's, as multisets."""
    from gospl_b200 import synthetic as S
    from oracle import fortran as F
    from oracle import mesh as M
    coords, cells, onb = S.planar_hex_mesh(3000, 30.0e3, seed=5, jitter=0.0)
    mesh = M.build_mesh(coords, cells, "ffff")
    M.load_mesh(mesh)
    rng = np.random.default_rng(7)
    h = rng.integers(0, 6, len(coords)).astype(np.float64)
    gid = np.zeros(len(coords), dtype=np.int32)
    R = 3
    rcv, dist, wgt, ties, slp = D.mfd_receivers(h, mesh["ngb"].astype(np.int64), mesh["elgt"], -100.0, R, gid=gid)
    r2, d2, w2 = F.mfdreceivers(R, 1.1, h, -100.0, gid)
    assert ties.sum() > 100, "the lattice must hold exact ties"
    nt = ~ties
    assert np.array_equal(rcv[nt], r2[nt]) and np.array_equal(dist[nt], d2[nt])
    assert np.abs(wgt - w2).max() <= 1e-15
    # at tie vertices the picked receivers are candidates with the top slopes
    ngb = mesh["ngb"]
    for k in np.where(ties)[0]:
        cand = {int(ngb[k, s]): slp[k, s] for s in range(ngb.shape[1]) if np.isfinite(slp[k, s])}
        top = sorted(cand.values(), reverse=True)[:R]
        got = [cand[int(c)] for c in r2[k]]
        assert sorted(got, reverse=True) == top, k


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_hillslope_coefficients_are_their_formula(case):
    from oracle import fortran as F
    om = _golden_oracle(case)
    kd = np.where(om.h > om.sealevel, om.Cda, om.Cdm) * om.dt
    dc = F.sethillslopecoeff(om.lpoints, kd)
    dg, v = D.hillslope_coefficients(om.FVmesh_ngbID, om.mesh["vdist"], om.mesh["elgt"], om.mesh["farea"], kd)
    assert np.array_equal(dg, dc[:, 0])
    assert np.array_equal(-v, dc[:, 1:1 + v.shape[1]])


def test_near_ties_of_the_receiver_slopes():
    """Candidate slopes among the flowDir + 1 steepest within 4 ulp of each
    other, where a pow that differs by a few ulp (CUDA's against the
    reference build's) could reorder receivers: none on the fixtures."""
    counts = {}
    for case in GOLDEN_CASES:
        om = _golden_oracle(case)
        *_, slp = D.mfd_receivers(om.h, om.FVmesh_ngbID, om.mesh["elgt"], om.sealevel, om.flowDir)
        counts[case] = D.near_ties(slp, om.flowDir)
    assert all(v == 0 for v in counts.values()), counts
