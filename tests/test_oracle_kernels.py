"""Oracle restatements checked against each other and against numpy, on CPU:
jacobiancoeff (functions.F90:1423-1467) reduces to sethillslopecoeff
(functions.F90:901-938, pinned through the golden fixtures) for a uniform
diffusivity and Kp = 0, closes faces where either side has no diffusivity, and
its Kp term follows the Fortran expression."""
import numpy as np
import pytest

from conftest import golden_mesh, load_golden


def _mesh():
    from oracle import mesh as OM
    g = load_golden("planar2k")
    m = golden_mesh(g)
    OM.load_mesh(m)
    return g, m


def test_jacobiancoeff_matches_hillslope_coefficients():
    from oracle import fortran as F
    g, m = _mesh()
    n = len(g["z"])
    kd = np.full(n, 3.0)
    d = F.jacobiancoeff(g["z"], kd, np.zeros(n))
    hc = F.sethillslopecoeff(n, kd)
    assert np.array_equal(d[:, 0] + 1.0, hc[:, 0])
    assert np.array_equal(d[:, 1:], hc[:, 1:])


def test_jacobiancoeff_gates_faces_without_diffusivity():
    from oracle import fortran as F
    g, m = _mesh()
    n = len(g["z"])
    rng = np.random.default_rng(5)
    kd = np.where(rng.random(n) < 0.5, 2.0, 0.0)
    d = F.jacobiancoeff(g["z"], kd, np.zeros(n))
    ngb = np.asarray(m["ngb"])
    for k in range(0, n, 37):
        for s in range(int(m["nnb"][k])):
            j = ngb[k, s]
            if kd[k] == 0.0 or kd[j] == 0.0:
                assert d[k, s + 1] == 0.0
    assert np.all(d[kd == 0.0, 0] == 0.0)


def test_jacobiancoeff_derivative_term():
    from oracle import fortran as F
    g, m = _mesh()
    n = len(g["z"])
    h = np.asarray(g["z"], float)
    kd = np.full(n, 1.5)
    kp = np.full(n, 0.25)
    d = F.jacobiancoeff(h, kd, kp)
    ngb, el, vd, ar = np.asarray(m["ngb"]), np.asarray(m["elgt"]), np.asarray(m["vdist"]), np.asarray(m["farea"])
    k = int(np.argmax(ar))
    diag = 0.0
    for s in range(int(m["nnb"][k])):
        if vd[k, s] > 0.0:
            j = ngb[k, s]
            c = 0.5 * (kd[k] + kd[j] + kp[k] * (h[k] - h[j])) / ar[k]
            diag = diag + c * vd[k, s] / el[k, s]
            c2 = 0.5 * (kd[k] + kd[j] + kp[j] * (h[j] - h[k])) / ar[k]
            assert d[k, s + 1] == -(c2 * vd[k, s] / el[k, s])
    assert d[k, 0] == diag


def test_epsfill_matches_a_plain_priority_flood():
    """epsfill (functions.F90:2633-2697) against a straightforward heapq
    priority-flood with the same epsilon step: identical surfaces; the cells
    below the level keep their elevation, and every cell the flood reached
    has a strictly lower neighbour (no flats)."""
    import heapq
    from oracle import fortran as F
    g, m = _mesh()
    z = g["z"]
    n = len(z)
    ngb, nnb = np.asarray(m["ngb"]), np.asarray(m["nnb"])
    sl = float(np.percentile(z, 20))
    got = F.epsfill(sl, z)
    fill = z.copy()
    flag = fill < sl
    heap = []
    for i in range(n):
        if flag[i] and any(fill[ngb[i, s]] >= sl for s in range(nnb[i]) if ngb[i, s] >= 0):
            heapq.heappush(heap, (fill[i], i))
    while heap:
        zi, i = heapq.heappop(heap)
        for s in range(nnb[i]):
            c = ngb[i, s]
            if c >= 0 and not flag[c]:
                flag[c] = True
                fill[c] = max(fill[c], np.nextafter(fill[i], np.inf))
                heapq.heappush(heap, (fill[c], c))
    assert np.array_equal(got, fill)
    assert np.array_equal(got[z < sl], z[z < sl])
    reached = (got >= sl)
    for k in np.flatnonzero(reached)[::7]:
        lower = [got[ngb[k, s]] < got[k] for s in range(nnb[k]) if ngb[k, s] >= 0]
        assert any(lower), k


def test_mfdrcvrs_equal_weights_over_lower_neighbours():
    """mfdrcvrs (functions.F90:1673-1785): every strictly lower neighbour, in
    neighbour order, is a receiver with the weight 1/kk rounded to single
    precision (the literal `1.` is a default real); no lower neighbour:
    every slot points at the vertex itself."""
    from oracle import fortran as F
    g, m = _mesh()
    z = F.epsfill(float(g["z"].min()) + 0.1, g["z"])
    n = len(z)
    ngb, nnb, elgt = np.asarray(m["ngb"]), np.asarray(m["nnb"]), np.asarray(m["elgt"])
    rcv, dist, wgt = F.mfdrcvrs(12, 1.1, z, -1.0e6, np.arange(n, dtype=np.int32))
    for k in range(0, n, 11):
        low = [(ngb[k, s], elgt[k, s]) for s in range(nnb[k]) if ngb[k, s] >= 0 and elgt[k, s] > 0 and z[ngb[k, s]] < z[k]]
        kk = len(low)
        if kk == 0:
            assert (rcv[k] == k).all() and (wgt[k] == 0).all()
            continue
        assert list(rcv[k, :kk]) == [c for c, _ in low] and (rcv[k, kk:] == k).all()
        assert list(dist[k, :kk]) == [e for _, e in low]
        w = float(np.float32(1.0) / np.float32(kk))
        assert (wgt[k, :kk] == w).all() and (wgt[k, kk:] == 0).all()


def test_coast_points_marching_triangles():
    """coast_points (vtkContourFilter as seaplex.py uses it) against a
    triangle-by-triangle loop: the same set of points, each on a crossing
    edge at the interpolated position."""
    from oracle.model import coast_points
    g, m = _mesh()
    z = g["z"]
    x = np.asarray(g["v"], np.float64).reshape(-1, 3)
    cells = np.asarray(g["c"], np.int64)
    level = float(np.percentile(z, 30))
    got = coast_points(x, cells, z, level)
    pts = set()
    for tri in cells:
        for a, b in ((tri[0], tri[1]), (tri[1], tri[2]), (tri[2], tri[0])):
            if (z[a] >= level) == (z[b] >= level):
                continue
            lo, hi = (a, b) if z[b] - z[a] > 0 else (b, a)
            t = (level - z[lo]) / (z[hi] - z[lo])
            pts.add(tuple(x[lo] + t * (x[hi] - x[lo])))
    assert len(got) == len(pts) > 0
    assert set(map(tuple, got)) == pts


def _marine_state(case, steps=1):
    """An oracle model of a marine fixture advanced `steps` steps and then to
    the point of seaChange where _distOcean runs: (model, sedFlux)."""
    from conftest import golden_params
    from oracle.model import OracleModel
    g = load_golden(case)
    om = OracleModel(g["v"], g["c"], g["z"], golden_params(g), mesh=golden_mesh(g))
    for _ in range(steps):
        om.step()
    om.flowAccumulation()
    om.erodepSPL()
    om.flowAccumulation()
    om.sedChange()
    om.sinkIDs = om.lFill <= om.sealevel
    hl = om.h.copy()
    om._distanceCoasts(hl)
    clinoH = om.sealevel - 1.0e-3 - om.coastDist * om.clinSlp
    clinoH[hl >= om.sealevel] = hl[hl >= om.sealevel]
    clinoH[clinoH < hl] = hl[clinoH < hl]
    om.maxDepQs = (clinoH - hl) * om.larea
    sed = om.vSed.copy() * om.dt
    sed[~om.sinkIDs] = 0.0
    sed[sed < 0] = 0.0
    om._matOcean()
    return om, sed


@pytest.mark.parametrize("case", ["planar2k_marine", "ico2562_marine"])
def test_marine_cascade_is_one_capacity_limited_sweep(case):
    """_distOcean's iteration (seaplex.py:404-619) equals one sweep of the
    marine DAG in topological order with a capacity clamp per vertex: a
    vertex keeps min(arrivals, capacity) and passes its own input plus the
    excess down its receivers; sinks keep all, outlets lose all.  The two
    agree up to the volume the iteration leaves in transit when it stops
    (deposited in place), at most max(1 m3, 1e-6 of the input)."""
    import scipy.sparse as sp
    om, sed = _marine_state(case)
    it = om._distOcean(sed)
    n = om.lpoints
    W = om.dMat1.T.tocsr()                          # row j: j's receivers and weights
    order = np.argsort(-_fillz(om), kind="stable")
    arr = np.zeros(n)
    dep = np.zeros(n)
    cap = om.maxDepQs.copy()
    out = set(np.asarray(om.outletIDs).tolist())
    for j in order:
        if om.is_sink_local[j]:
            dep[j] = sed[j] + arr[j]
            continue
        if j in out:
            continue
        keep = min(arr[j], cap[j])
        dep[j] = keep
        send = sed[j] + arr[j] - keep
        row = slice(W.indptr[j], W.indptr[j + 1])
        arr[W.indices[row]] += send * W.data[row]
    total = float(sed.sum())
    assert np.abs(it - dep).sum() <= 2.0 * max(1.0, 1.0e-6 * total) + 1e-9 * total, (case, np.abs(it - dep).sum())
    assert sp.issparse(om.dMat1)


def _fillz(om):
    """The epsilon-filled surface _matOcean routed on (recomputed as it does)."""
    from oracle import fortran as F
    from oracle.model import BOUNDARY_FLOW_SENTINEL
    hl = om.h.copy()
    minh = max(om.h.min() + 0.1, om.oFill)
    if not om.flatModel:
        hs = om._smoothBathymetry()
        hs[om.coastDist > om.offshore] = BOUNDARY_FLOW_SENTINEL
    else:
        hs = hl.copy()
        hs[om.outletIDs] = BOUNDARY_FLOW_SENTINEL
    fz = F.epsfill(minh, hs)
    if not om.flatModel:
        fz[om.coastDist > om.offshore] = hl[om.coastDist > om.offshore]
    return fz


@pytest.mark.parametrize("case", ["planar2k_marine", "ico2562_marine"])
def test_epsfill_is_a_relaxation_fixpoint(case):
    """epsfill's priority flood equals the fixpoint of the parallel
    relaxation fill(c) = max(z(c), nextafter(min over flooded neighbours of
    fill)) started from the seeds (cells below the level touching one at or
    above it): a cell's value comes from its lowest flooded neighbour, and
    the queue pops values in non-decreasing order.  Bit for bit, on the
    smoothed bathymetry the marine routing fills."""
    from oracle import fortran as F
    om, _ = _marine_state(case, steps=0)
    g = load_golden(case)
    m = golden_mesh(g)
    from oracle import mesh as OM
    OM.load_mesh(m)
    ngb = np.asarray(m["ngb"])
    nnb = np.asarray(m["nnb"])
    z = _fillz_input(om)
    n = len(z)
    W = ngb.shape[1]
    valid = (np.arange(W)[None, :] < nnb[:, None]) & (ngb >= 0)
    nb_ = np.where(valid, ngb, 0)
    filled = 0
    # the routing's own level (on the sphere nothing lies below it, so the
    # flood never starts) and a level that floods the lowest tenth
    for sl in (max(om.h.min() + 0.1, om.oFill), float(np.percentile(z, 10))):
        ref = F.epsfill(sl, z)
        below = z < sl
        seeds = below & (valid & (z[nb_] >= sl)).any(axis=1)
        val = np.full(n, np.inf)
        val[seeds] = z[seeds]
        for _ in range(n + 1):
            nv = np.where(valid, val[nb_], np.inf).min(axis=1)
            cand = np.where(np.isfinite(nv), np.maximum(z, np.nextafter(nv, np.inf)), np.inf)
            new = np.where(below, val, cand)
            if np.array_equal(new, val):
                break
            val = new
        got = np.where(np.isfinite(val) & ~below, val, z)
        assert np.array_equal(got, ref), sl
        filled += int((ref > z).sum())
    assert filled > 0


def _fillz_input(om):
    """The surface _matOcean hands to epsfill."""
    from oracle.model import BOUNDARY_FLOW_SENTINEL
    if not om.flatModel:
        hs = om._smoothBathymetry()
        hs[om.coastDist > om.offshore] = BOUNDARY_FLOW_SENTINEL
    else:
        hs = om.h.copy()
        hs[om.outletIDs] = BOUNDARY_FLOW_SENTINEL
    return hs


@pytest.mark.parametrize("case", ["planar2k_marine", "ico2562_marine"])
def test_coast_distance_is_a_plain_nearest_point_search(case):
    """The k-d tree distances _distanceCoasts takes (scipy cKDTree, p = 2)
    equal sqrt(min over coast points of (dx dx + dy dy) + dz dz) bit for
    bit: a nearest-point search that sums the squares in that order, without
    fused multiply-adds, reproduces them exactly."""
    from scipy import spatial
    from oracle.model import coast_points
    om, _ = _marine_state(case, steps=0)
    pts = coast_points(om.lcoords, om.lcells, om.h, om.sealevel)
    q = om.lcoords[om.seaID]
    d_tree, _ = spatial.cKDTree(pts, leafsize=10).query(q, k=1)
    best = np.full(len(q), np.inf)
    for p in pts:
        dx, dy, dz = q[:, 0] - p[0], q[:, 1] - p[1], q[:, 2] - p[2]
        best = np.minimum(best, (dx * dx + dy * dy) + dz * dz)
    assert len(pts) > 0 and np.array_equal(np.sqrt(best), d_tree)
