"""Independent definitions of what goSPL's Fortran kernels compute (test
infrastructure).

Each function states the result of one kernel of ``fortran/functions.F90`` by
its mathematical definition, with textbook graph algorithms (a heap
Priority-Flood, a minimum spanning tree, connected components, breadth-first
hop distances) and plain numpy, never by replaying the kernel's own loops.
The oracle's C restatement and the CUDA kernels are both checked against
these, which pins them to the meaning of the reference's kernels rather than
to each other.

Reference quirks that belong to the definition are kept and named where they
occur (the unsorted receiver distances of ``mfdreceivers``, the seed order of
``label_pits``, the sea reset of the fill).
"""
import heapq

import numpy as np
import scipy.sparse as sp
from scipy.sparse import csgraph


def _edges(ngb):
    """Directed neighbour pairs (i, c) of the FVnID table (-1 padding)."""
    n, w = ngb.shape
    i = np.repeat(np.arange(n), w)
    c = ngb.ravel()
    keep = c >= 0
    return i[keep], c[keep]


# ---------------------------------------------------------------- pit filling
def fill_seeds(z, ngb, outlet_mask):
    """Seeds of the depression fill on the relative surface z = h - level
    (edge_tile, functions.F90:2036-2080, read as a definition): a cell below
    the level with a neighbour at or above it drains (the sea edge); a cell
    below the level whose neighbours are all below it takes no part; a cell
    at or above the level on an open outlet boundary drains.  Returns
    (drains, active)."""
    i, c = _edges(ngb)
    below = z < 0.0
    has_high = np.zeros(len(z), dtype=bool)
    np.logical_or.at(has_high, i, z[c] >= 0.0)
    drains = (below & has_high) | (~below & outlet_mask)
    active = ~(below & ~has_high)
    return drains, active


def priority_flood(z, ngb, drains, active):
    """Priority-Flood without epsilon (Barnes, Lehman & Mulla 2014,
    Algorithm 1): every active cell is raised to the lowest level at which
    water leaves it for a drain, max(z, min over paths to a drain of the
    highest cell on the path).  Cells no drain reaches keep z.  Heap over
    (level, index); O(N log N) Python loop, for small meshes."""
    n = len(z)
    fill = z.astype(np.float64).copy()
    done = drains.copy()
    heap = [(float(z[k]), int(k)) for k in np.where(drains)[0]]
    heapq.heapify(heap)
    nbrs = [row[row >= 0] for row in ngb]
    while heap:
        f, k = heapq.heappop(heap)
        for c in nbrs[k]:
            if done[c] or not active[c]:
                continue
            done[c] = True
            fc = z[c] if z[c] > f else f
            fill[c] = fc
            heapq.heappush(heap, (fc, int(c)))
    return fill, done


def minimax_fill(z, ngb, drains, active):
    """The same surface through the minimum spanning tree: the minimax path
    between two cells of a graph runs along its minimum spanning tree (Hu
    1961), so with edge weight max(z_u, z_v) between active neighbours and a
    root joined to every drain below every other weight, the fill of a cell
    is max(z, the largest weight on its tree path to the root).  Weights are
    replaced by their ranks (exact, and never zero for scipy), path maxima are
    taken by pointer jumping.  Vectorised, for large meshes."""
    n = len(z)
    i, c = _edges(ngb)
    keep = (i < c) & active[i] & active[c]
    i, c = i[keep], c[keep]
    w = np.maximum(z[i], z[c])
    levels, rank = np.unique(w, return_inverse=True)
    root = n
    d = np.where(drains)[0]
    rows = np.concatenate([i, np.full(len(d), root)])
    cols = np.concatenate([c, d])
    vals = np.concatenate([rank + 2.0, np.ones(len(d))])
    g = sp.coo_matrix((vals, (rows, cols)), shape=(n + 1, n + 1)).tocsr()
    t = csgraph.minimum_spanning_tree(g)
    t = t + t.T
    order, pred = csgraph.breadth_first_order(t, root, directed=False, return_predecessors=True)
    reached = np.zeros(n + 1, dtype=bool)
    reached[order] = True
    # rank of the edge to the parent (-1 below every level for the root's edges)
    par = pred[:n].astype(np.int64)
    ok = reached[:n] & (par >= 0)
    up = np.full(n + 1, -1, dtype=np.int64)
    tt = t.tocsr()
    kk = np.where(ok)[0]
    if kk.size:
        up[kk] = np.asarray(tt[kk, par[kk]]).ravel().astype(np.int64) - 2
    up[:n][par == root] = -1
    jump = np.where(ok, par, root)
    jump = np.append(jump, root)
    best = up.copy()
    while True:
        nb = np.maximum(best, best[jump])
        nj = jump[jump]
        if np.array_equal(nj, jump) and np.array_equal(nb, best):
            break
        best, jump = nb, nj
    fill = z.astype(np.float64).copy()
    lift = ok & (best[:n] >= 0)
    fill[lift] = np.maximum(z[lift], levels[best[:n][lift]])
    return fill, reached[:n]


def filled_surface(h, level, ngb, outlet_mask, sealevel, sed=False, large=False):
    """lFill of fillElevation (pitfilling.py:849-903): the fill of h - level
    on the cells strictly above the level (fill_depressions only writes
    dem > lvl, functions.F90:2290-2329; cells at or below it keep their
    elevation but still pass water), cells below sealevel - level returned to
    h - level when sed is False (pitfilling.py:690-693), then + level."""
    z = h - level
    drains, active = fill_seeds(z, ngb, outlet_mask)
    fill = (minimax_fill if large else priority_flood)(z, ngb, drains, active)[0]
    fill = np.where(z > 0.0, fill, z)
    if not sed:
        sea = fill < sealevel - level
        fill[sea] = z[sea]
    return fill + level


# ------------------------------------------------------------ depression ids
def equal_fill_components(fill, ngb, lvl):
    """label_pits (functions.F90:2420-2499) by definition: the connected
    components of cells above lvl joined through neighbours of exactly equal
    fill that contain a bottom (a cell with no strictly lower neighbour),
    numbered 1.. in the order of their lowest-index bottom; -1 elsewhere."""
    n = len(fill)
    i, c = _edges(ngb)
    up = fill > lvl
    e = up[i] & up[c] & (fill[i] == fill[c])
    g = sp.coo_matrix((np.ones(int(e.sum())), (i[e], c[e])), shape=(n, n))
    _, comp = csgraph.connected_components(g, directed=False)
    lower = np.zeros(n, dtype=bool)
    np.logical_or.at(lower, i, fill[c] < fill[i])
    bottom = up & ~lower
    first = np.full(comp.max() + 1, n, dtype=np.int64)
    np.minimum.at(first, comp[bottom], np.where(bottom)[0])
    has = first < n
    num = np.zeros(len(first), dtype=np.int64)
    ordered = np.where(has)[0][np.argsort(first[has], kind="stable")]
    num[ordered] = np.arange(1, len(ordered) + 1)
    label = np.where(up & has[comp], num[comp], -1)
    return label


def pit_ids(fill, ngb, lvl, outlet_ids):
    """pitIDs after label_pits, the outlet reset and pits_cons
    (pitfilling.py:719-728, functions.F90:2005-2034): labels on open outlets
    dropped, the remaining labels renumbered 1.. in increasing order (the
    1-based position in the list of labels present; id 0 names no
    depression)."""
    lab = equal_fill_components(fill, ngb, lvl)
    lab[np.asarray(outlet_ids, dtype=np.int64)] = -1
    keep = lab > 0
    out = -np.ones(len(fill), dtype=np.int64)
    if keep.any():
        out[keep] = np.unique(lab[keep], return_inverse=True)[1] + 1
    return out


# --------------------------------------------------------------- flat routing
def flat_distance(spills, pit, lfill, ngb):
    """fill_dir then nghb_dir to their fixed point (functions.F90:1845-1969):
    1 + the hop distance from the nearest spill node along directed
    neighbour steps i -> c into depression cells (pit(c) > -1) that do not go
    down (lfill(c) >= lfill(i)); -1 where no spill reaches.  Breadth-first
    search from a root joined to every spill node."""
    n = len(lfill)
    i, c = _edges(ngb)
    e = (pit[c] > -1) & (lfill[c] >= lfill[i])
    root = n
    s = np.asarray(spills, dtype=np.int64)
    rows = np.concatenate([i[e], np.full(len(s), root)])
    cols = np.concatenate([c[e], s])
    g = sp.coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(n + 1, n + 1)).tocsr()
    if len(s) == 0:
        return -np.ones(n, dtype=np.int64)
    d = csgraph.shortest_path(g, directed=True, unweighted=True, indices=root)
    out = np.where(np.isfinite(d[:n]), d[:n], -1).astype(np.int64)
    return out


def flat_dirs(pdir, pit, lfill, ngb, spills, sealevel):
    """flatDirs of _dirFlats (pitfilling.py:491-517, 822-826): in a depression
    the neighbour with the smallest (distance, index) among those with a
    known, strictly smaller distance and a fill not above the cell's; the cell
    itself when none; -1 outside depressions, at spill nodes and where
    lfill <= sealevel."""
    n = len(lfill)
    big = np.iinfo(np.int64).max
    valid = ngb >= 0
    cc = np.where(valid, ngb, 0)
    cpd = pdir[cc]
    cand = valid & (cpd > -1) & (cpd < pdir[:, None]) & (lfill[cc] <= lfill[:, None]) & (pit[:, None] > -1)
    key = np.where(cand, cpd * (n + 1) + cc, big)
    k = key.argmin(axis=1)
    rows = np.arange(n)
    best = np.where(key[rows, k] < big, cc[rows, k], rows)
    out = np.where(pit > -1, best, -1)
    out[np.asarray(spills, dtype=np.int64)] = -1
    out[lfill <= sealevel] = -1
    return out


# ------------------------------------------------------------------ receivers
def mfd_receivers(elev, ngb, elgt, sl, nrcv, exp=1.1, gid=None):
    """mfdreceivers (functions.F90:1544-1671) by definition.  Above sl a
    vertex's candidates are its neighbours n with val = (elev - elev_n)^f /
    eLgt > 0, f = 5 min(e, 1) + exp with e the largest downhill gradient (f =
    1 when there is none), each slope scaled by (1 - 1e-15 gid(n)).  With at
    most nrcv candidates they are the receivers in neighbour order; with more,
    the nrcv largest slopes in descending order.  Weights are slope / sum of
    the chosen slopes, summed in receiver order.  Unused receiver slots and
    vertices at or below sl point at the vertex itself with weight and
    distance 0.  Reference quirk kept: after the sort the distances are not
    permuted with the slopes, so the k-th receiver's distance is the edge
    length of the (kk - k + 1)-th candidate in neighbour order.  The order of
    exactly equal slopes is the sort's own; `ties` marks the vertices where it
    matters (equal slopes among the nrcv + 1 largest).  Returns rcv, dist, wgt
    as [n, nrcv], ties [n] and the candidate slopes [n, W] (nan elsewhere)."""
    n, W = ngb.shape
    R = nrcv
    gid = np.arange(n) if gid is None else np.asarray(gid)
    valid = (ngb >= 0) & (elgt > 0.0)
    cc = np.where(valid, ngb, 0)
    dz = elev[:, None] - elev[cc]
    safe = np.where(valid, elgt, 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        grad = np.where(valid, dz / safe, 0.0)
        e = np.maximum(grad.max(axis=1), 0.0)
        f = np.where(e > 0.0, 5.0 * np.minimum(e, 1.0) + exp, 1.0)
        val = np.where(valid, np.power(dz, f[:, None]) / safe, np.nan)
    land = elev > sl
    cand = valid & (val > 0.0) & land[:, None]
    slp = np.where(cand, val * (1.0 - 1.0e-15 * gid[cc].astype(np.float64)), np.nan)
    kk = cand.sum(axis=1)
    rows = np.arange(n)
    rcv = np.repeat(rows[:, None], R, axis=1)
    dist = np.zeros((n, R))
    wgt = np.zeros((n, R))
    # candidates compacted to the front in neighbour order
    pos = np.argsort(~cand, axis=1, kind="stable")
    cs = np.take_along_axis(slp, pos, axis=1)
    cid = np.take_along_axis(np.where(valid, ngb, -1), pos, axis=1)
    cd = np.take_along_axis(elgt, pos, axis=1)
    few = (kk > 0) & (kk <= R)
    for k in range(R):
        m = few & (kk > k)
        rcv[m, k] = cid[m, k]
        dist[m, k] = cd[m, k]
    tot = np.zeros(n)
    for k in range(R):
        m = few & (kk > k)
        tot[m] = tot[m] + cs[m, k]
    for k in range(R):
        m = few & (kk > k)
        wgt[m, k] = cs[m, k] / tot[m]
    many = kk > R
    order = np.argsort(-np.where(np.isnan(cs), -np.inf, cs), axis=1, kind="stable")
    top = np.take_along_axis(cs, order, axis=1)
    ties = np.zeros(n, dtype=bool)
    for k in range(R):
        ties |= many & (top[:, k] == top[:, k + 1])
    tot = np.zeros(n)
    for k in range(R):
        m = many
        rcv[m, k] = np.take_along_axis(cid, order[:, k:k + 1], axis=1)[m, 0]
        dist[m, k] = cd[m, kk[m] - 1 - k]
        tot[m] = tot[m] + top[m, k]
    for k in range(R):
        wgt[many, k] = top[many, k] / tot[many]
    return rcv, dist, wgt, ties, slp


def near_ties(slopes, nrcv, ulps=4):
    """Vertices with more than nrcv candidates whose choice or order of
    receivers could flip under a pow that differs by a few ulp: adjacent
    slopes among the nrcv + 1 largest that lie within `ulps` ulp of each
    other.  Returns the number of such pairs."""
    s = -np.sort(-np.where(np.isnan(slopes), -np.inf, slopes), axis=1)[:, :nrcv + 1]
    many = np.isfinite(s[:, -1]) if s.shape[1] > nrcv else np.zeros(len(s), bool)
    a, b = s[many, :-1], s[many, 1:]
    gap = np.abs(a - b)
    tol = ulps * np.spacing(np.maximum(np.abs(a), np.abs(b)))
    return int(np.count_nonzero(gap <= tol))


# ----------------------------------------------------------------- pit tables
def pit_volumes(pit, lfill, h, larea, npits):
    """pitParams[:, 0] (pitfilling.py:521-555): sum over each depression of
    (lfill - h) * area."""
    out = np.zeros(npits)
    m = pit >= 0
    np.add.at(out, pit[m], (lfill[m] - h[m]) * larea[m])
    return out


def filled_volumes(pit, h, larea, levels):
    """getpitvol (functions.F90:1971-2003) by definition: for each depression
    p and level l, the volume sum over its cells with h < l of (l - h) * area."""
    P, L = levels.shape
    out = np.zeros((P, L))
    m = pit >= 0
    for j in range(L):
        lv = levels[pit[m], j]
        below = h[m] < lv
        np.add.at(out[:, j], pit[m][below], (lv - h[m])[below] * larea[m][below])
    return out


def hillslope_coefficients(ngb, vdist, elgt, area, kd):
    """sethillslopecoeff (functions.F90:901-938) by definition: for a row of
    positive area, the off-diagonal entry of each neighbour with a positive
    Voronoi edge is -v, v = 0.5 (Kd_k + Kd_n) / area_k * vDist_kp / eLgt_kp,
    and the diagonal 1 + sum v; rows of zero area are all zero.  Returns the
    diagonal [n] and v [n, W]."""
    valid = (ngb >= 0) & (vdist > 0.0)
    cc = np.where(valid, ngb, 0)
    pos = area > 0.0
    with np.errstate(invalid="ignore", divide="ignore"):
        c = 0.5 * (kd[:, None] + kd[cc]) / np.where(pos, area, 1.0)[:, None]
        v = np.where(valid & pos[:, None], c * vdist / np.where(valid, elgt, 1.0), 0.0)
    s = np.zeros(len(area))
    for p in range(v.shape[1]):
        s = s + v[:, p]
    return np.where(pos, 1.0 + s, 0.0), v
