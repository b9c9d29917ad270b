"""ORACLE — test infrastructure only (tests/, smoke check, CPU-baseline leg).

Single-rank CPU restatement of goSPL's per-timestep surface-process path with
the reference's own Python orchestration and the C restatement of its Fortran
kernels (``oracle/gospl_oracle.c``).  Every method cites the reference lines it
follows.  MPI reductions and halo exchanges are identities on one rank.  The
linear systems the reference hands to PETSc KSP (``rtol=1e-8``) are solved
EXACTLY here (topological sweeps for the flow and SPL systems, a direct or
1e-14 CG solve for diffusion): the oracle defines the exact solution of the
assembled systems, which PETSc itself only approaches to ~1e-8.

Grouped sums reproduce ``numpy_indexed.group_by(...).sum`` (stable mergesort of
the keys, then ``np.add.reduceat``), so per-pit volumes round as in the
reference.
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import fortran as F
from . import mesh as M

MISSING_DATA_SENTINEL = -1.0e8   # gospl/tools/constants.py:34
DEPOSIT_FLOOR = 1.0e-3           # gospl/tools/constants.py:58
BOUNDARY_FLOW_SENTINEL = -1.0e6  # gospl/tools/constants.py:90
MARINE_SMOOTH_N_LAND = 1.0       # gospl/tools/constants.py:126
MARINE_SMOOTH_N_SEA = 5.0        # gospl/tools/constants.py:127
GRAPH_OUTLIER_CAP = 1.0e7        # gospl/tools/constants.py:100


BUDGET_SLOTS = ("eroded", "pit_sinks", "kept", "dropped", "outlets", "sea", "retained", "excess", "zero_excess",
                "inflow", "placed", "routed", "realised", "kept_deposit")


def budget(b):
    """Derived terms of a sediment budget: excess written at no spill node
    (a spill node shared by several depressions keeps one depression's
    excess, a depression without a spill node keeps none), placed excess left
    unrouted, and the closure (eroded minus every destination), which
    vanishes to rounding."""
    b = dict(b)
    b["unplaced"] = b["excess"] - b["placed"]
    b["unrouted"] = b["placed"] - b["routed"]
    b["closure"] = b["eroded"] - (b["retained"] + b["kept"] + b["dropped"] + b["outlets"] + b["sea"]
                                  + b["zero_excess"] + b["unplaced"] + b["unrouted"])
    return b


def group_reduce(keys, values, op=np.add):
    """numpy_indexed.group_by(keys).reduce(values, op): (unique, reduced)."""
    keys = np.asarray(keys)
    if keys.size == 0:
        return keys[:0], np.zeros(0, dtype=np.asarray(values).dtype)
    sorter = np.argsort(keys, kind="mergesort")
    sk = keys[sorter]
    flag = np.concatenate(([True], sk[1:] != sk[:-1]))
    start = np.flatnonzero(flag)
    return sk[start], op.reduceat(np.asarray(values)[sorter], start)


class OracleModel:
    """State and methods of goSPL's ``Model`` restricted to the hot path.

    ``params`` keys: ``dt, tStart, tEnd, flowDir, K, d, m, Cda, Cdm, oFill,
    sealevel, bc`` plus per-vertex ``rain`` (m/yr) and ``upsub`` (m/yr) arrays.
    ``K`` may be a scalar (as in the reference) or a per-vertex array.
    """

    def __init__(self, coords, cells, elev, params, mesh=None, init_flow=True):
        self.mesh = mesh if mesh is not None else M.build_mesh(coords, cells, params.get("bc", "oooo"))
        M.load_mesh(self.mesh)
        m = self.mesh
        self.lpoints = m["nb"]
        self.flatModel = m["flat"]
        self.outletIDs = m["outlet"]
        self.open_nodes = m["open_nodes"]
        self.larea = m["larea"].copy()
        self.maxarea = np.array([m["maxarea"]])
        self.FVmesh_ngbID = m["ngb"].astype(np.int64)
        self.gid = np.arange(self.lpoints, dtype=np.int32)
        self.locIDs = np.arange(self.lpoints, dtype=np.int64)
        self.inIDs = np.ones(self.lpoints, dtype=int)
        self.maxnb = F.setmaxnb(self.lpoints)
        edges = -np.ones((self.lpoints, 2), dtype=int)       # pitfilling.py:80-101
        edges[self.outletIDs, 0] = self.outletIDs
        edges[self.outletIDs, 1] = 1
        self.borders = edges
        self.outEdges = np.zeros(self.lpoints, dtype=int)

        p = params
        self.dt = float(p["dt"])
        self.tStart = float(p.get("tStart", 0.0))
        self.tEnd = float(p["tEnd"])
        self.tNow = self.tStart
        self.flowDir = int(p.get("flowDir", 8))
        self.flowExp = 1.1                                   # inputparser.py:194
        self.K = p["K"]
        self.coeffd = float(p.get("d", 0.0))
        self.spl_m = float(p.get("m", 0.5))
        self.fDepa = float(p.get("G", 0.0))
        self.Cda = float(p.get("Cda", 0.0))
        self.Cdm = float(p.get("Cdm", 0.0))
        self.oFill = float(p.get("oFill", -6000.0))
        self.sealevel = float(p.get("sealevel", 0.0))
        self.nodep = bool(p.get("nodep", True))
        self.seaDepo = bool(p.get("seadepo", False))
        self.nlK = float(p.get("nonlinKm", 10.0))                                    # inputparser.py:554
        self.clinSlp = max(1.0e-6, float(p.get("clinSlp", 1.0e-6)))                 # :555, 592
        self.Gmar = float(p.get("Gmar", 0.0))                                        # :557
        self.offshore = float(p.get("offshore", 100.0e5))                            # :558
        self.nl_pit_volume = float(p.get("nlPitVolume", 1.0e9))   # inputparser.py:562,584
        self.nl_pit_depth = float(p.get("nlPitDepth", 100.0))     # inputparser.py:563,585
        self.nl_pit_K = float(p.get("nlPitK", p.get("nonlinKm", 10.0)))             # inputparser.py:564
        self.nl_pit_inlet_bias = min(1.0, max(0.0, float(p.get("pitInletBias", 0.5))))  # :569,587,593
        self.marineSolver = str(p.get("marineSolver", "ts")).lower()                 # inputparser.py:576
        self.picardSub = int(p.get("picardSub", 10))
        self.picardIts = int(p.get("picardIts", 2))
        if not self.nodep and self.seaDepo:
            if self.marineSolver != "picard":
                raise NotImplementedError("goSPL's adaptive TS solve of the marine diffusion is not "
                                          "restated; use marineSolver picard")
        self.dexp = 0.05                                                             # hillslope.py:34
        self.minDiff = 1.0e-4                                                        # hillslope.py:35
        self._domainHasOutlet = len(self.outletIDs) > 0           # sedplex.py:45-47
        self.lcoords = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
        self.lcells = np.asarray(cells, dtype=np.int64)
        self.rainMesh = np.asarray(p["rain"], dtype=np.float64)
        up = p.get("upsub")
        self.upsub = None if up is None else np.asarray(up, dtype=np.float64)

        self.h = np.asarray(elev, dtype=np.float64).copy()
        self.cumED = np.zeros(self.lpoints)
        self.EbLocal = np.zeros(self.lpoints)
        self.FAL = np.zeros(self.lpoints)
        self.fillFAL = np.zeros(self.lpoints)
        self.stats = []
        self._hill_seaID = None
        self._hill_mat = None
        self.applyForces()
        if init_flow:
            self.flowAccumulation()

    # ------------------------------------------------------------------ forcing
    def applyForces(self):
        """unstructuredmesh.py:743-794 (constant sea level, uniform-in-time rain)."""
        self.rainVal = self.rainMesh.copy()
        self.rainVal[self.rainVal < 0] = 0.0                 # unstructuredmesh.py:960
        self.bL = self.rainVal * self.larea                  # unstructuredmesh.py:970
        if self.upsub is not None:                           # unstructuredmesh.py:903-922
            self.h = self.h + self.upsub * self.dt
        if self.flatModel:
            self.h = self._drainOpenEdges(self.h.copy())

    def _drainOpenEdges(self, tmp):
        """unstructuredmesh.py:796-901"""
        open_nodes = self.open_nodes
        if open_nodes.size == 0:
            return tmp
        ngb = self.FVmesh_ngbID
        is_open = np.zeros(tmp.shape[0], dtype=bool)
        is_open[open_nodes] = True
        assigned = ~is_open
        vals = tmp.copy()
        pending = open_nodes
        for _ in range(open_nodes.size + 1):
            nb = ngb[pending]
            valid = nb >= 0
            nb_idx = np.where(valid, nb, 0)
            usable = valid & assigned[nb_idx]
            cand = np.where(usable, vals[nb_idx], np.inf)
            mn = cand.min(axis=1)
            ok = np.isfinite(mn)
            vals[pending[ok]] = mn[ok]
            assigned[pending[ok]] = True
            pending = pending[~ok]
            if pending.size == 0:
                break
        cur = tmp[open_nodes]
        runmin = np.minimum(cur, vals[open_nodes])
        marine = cur < self.sealevel
        tmp[open_nodes] = np.where(marine, cur, runmin)
        return tmp

    # ------------------------------------------------------------- pit filling
    def _fillFromEdges(self, mgraph):
        """pitfilling.py:219-292 (pandas sort/dedup restated with numpy)."""
        order = np.argsort(mgraph[:, 2], kind="stable")
        cg = mgraph[order]
        key = cg[:, 0].astype(np.int64) * (1 << 32) + cg[:, 1].astype(np.int64)
        _, first = np.unique(key, return_index=True)
        cgraph = cg[np.sort(first)]
        nb_global = int(cgraph[:, 1].max()) + 2
        src = cgraph[:, 0].astype(np.int64)
        tgt = cgraph[:, 1].astype(np.int64)
        uniq = np.unique(np.concatenate((src, tgt)))
        if uniq[0] != 0:
            uniq = np.concatenate((np.array([0], dtype=uniq.dtype), uniq))
        nlab = len(uniq)
        if uniq[-1] >= nb_global:
            # the reference would raise IndexError writing ggraph[uniq] here
            raise IndexError("spill graph label %d beyond target range %d" % (uniq[-1], nb_global))
        cc = cgraph.copy()
        cc[:, 0] = np.searchsorted(uniq, src)
        cc[:, 1] = np.searchsorted(uniq, tgt)
        c12 = cc[:, :2].astype(int).ravel()
        cmax = np.max(np.bincount(c12)) + 1
        elev, rank, nodes, spillID = F.fill_edges(nlab + 1, cc, cmax)
        ggraph = -np.ones((nb_global, 5))
        ggraph[:, 0] = 1.0e8
        ggraph[uniq, 0] = elev[:nlab]
        ggraph[uniq, 1] = nodes[:nlab]
        ggraph[uniq, 2] = rank[:nlab]
        gspill = spillID[:nlab].astype(np.int64)
        valid = (gspill >= 0) & (gspill < nlab)
        gspill[valid] = uniq[gspill[valid]]
        ggraph[uniq, 3] = gspill
        return ggraph

    def _performFilling(self, hl, level, sed):
        """pitfilling.py:557-702 at one rank."""
        ledges = F.edge_tile(0.0, self.borders, hl)
        out = np.where(ledges >= 0)[0]
        localEdges = np.empty((len(out), 2), dtype=int)
        localEdges[:, 0] = np.arange(self.lpoints)[out]
        localEdges[:, 1] = ledges[out]
        out = np.where(ledges == -2)[0]
        inIDs = self.inIDs.copy()
        inIDs[out] = 0
        outEdges = self.outEdges.copy()
        outEdges[out] = 0
        gBounds = np.zeros(self.lpoints, dtype=int)
        gBounds[np.where((ledges == 0) | (ledges == 2))[0]] = 1

        lFill, label, gnb = F.fill_tile(localEdges, hl, inIDs)
        lgth = 0
        if gnb > 0:
            graph = F.graph_nodes(gnb)
            lgth = np.amax(graph[:, :2])
        cgraph, graphnb = F.combine_edges(lFill, label, localEdges[:, 0], outEdges)
        lgrph = 0
        if graphnb > 0 and lgth > 0:
            cgraph = np.concatenate((graph, cgraph[:graphnb]))
            lgrph = len(cgraph)
        elif graphnb > 0 and lgth == 0:
            cgraph = cgraph[:graphnb]
            lgrph = len(cgraph)
        elif graphnb == 0 and lgth > 0:
            cgraph = graph
            lgrph = len(cgraph)
        total = lgrph
        if total == 0:
            nlab = int(label.max()) + 2 if label.size else 2
            graph = -np.ones((nlab, 5), dtype=float)
        else:
            graph = -np.ones((total, 5), dtype=float)
            graph[:lgrph, :4] = cgraph
            graph[:lgrph, 4] = 0
            graph = self._fillFromEdges(graph)
        keep = graph[:, 2].astype(int) == 0
        proc = -np.ones(len(graph))
        proc[keep] = graph[keep, 1]
        keep = proc > -1
        proc[keep] = gBounds[proc[keep].astype(int)]
        ids = np.where(proc == 1)[0]
        ids2 = np.where(graph[ids, 0] == graph[graph[ids, 3].astype(int), 0])[0]
        graph[ids[ids2], 3] = 0.0
        graph[graph[:, 0] < MISSING_DATA_SENTINEL, 0] = MISSING_DATA_SENTINEL
        graph[graph[:, 0] > GRAPH_OUTLIER_CAP, 0] = MISSING_DATA_SENTINEL
        lFill = F.fill_depressions(0.0, hl, lFill, label.astype(int), graph[:, 0])
        if not sed:
            idd = lFill < self.sealevel - level
            lFill[idd] = hl[idd]
        self.lFill = lFill.copy()

    def _transferIDs(self, pitIDs):
        """pitfilling.py:294-398 at one rank: consecutive ids 1..P."""
        self.pitIDs = pitIDs.astype(int)
        pitnbs = np.max(self.pitIDs) + 1
        fillIDs = self.pitIDs >= 0
        valpit = -np.ones(max(pitnbs, 0), dtype=int)
        valpit[np.unique(self.pitIDs[fillIDs])] = 1
        pitNb = np.where(valpit > 0)[0]
        self.pitIDs = F.pits_cons(self.pitIDs, pitNb).astype(int)
        return pitNb

    def _dirFlats(self):
        """pitfilling.py:400-519 at one rank."""
        ids = self.pitIDs > -1
        if ids.any():
            pdir = F.fill_dir(self.lspillIDs, self.pitIDs, self.lFill)
        else:
            pdir = -np.ones(self.lpoints, dtype=np.int32)
        stp = 0
        while True:
            prev = pdir
            pdir = F.nghb_dir(self.pitIDs, self.lFill, pdir.astype(int))
            stp += 1
            if np.count_nonzero(pdir != prev) == 0 or stp > 10000:
                break
        self.pdir = pdir.astype(np.int64)
        ngb = self.FVmesh_ngbID
        n = self.lpoints
        valid = ngb >= 0
        cidx = np.where(valid, ngb, 0)
        cpd = self.pdir[cidx]
        ch = self.lFill[cidx]
        clid = self.locIDs[cidx].astype(np.int64)
        cand = (valid & (cpd > -1) & (cpd < self.pdir[:, None]) & (ch <= self.lFill[:, None])
                & (self.pitIDs[:, None] > -1))
        BIG = np.iinfo(np.int64).max
        nid = np.int64(self.locIDs.max()) + 1
        comp = np.where(cand, cpd.astype(np.int64) * nid + clid, BIG)
        kbest = comp.argmin(axis=1)
        rows = np.arange(n)
        has = comp[rows, kbest] < BIG
        self.flatDirs = np.full(n, -1, dtype=np.int32)
        ispit = self.pitIDs > -1
        self.flatDirs[ispit] = np.where(has[ispit], ngb[rows, kbest][ispit], rows[ispit]).astype(np.int32)
        self.flatDirs[self.lspillIDs] = -1

    def _getPitParams(self, hl, nbpits):
        """pitfilling.py:521-555"""
        ids = self.inIDs == 1
        uids, vol = group_reduce(self.pitIDs[ids], (self.lFill[ids] - hl[ids]) * self.larea[ids])
        _, hh = group_reduce(self.pitIDs[ids], self.lFill[ids], np.maximum)
        _, dh = group_reduce(self.pitIDs[ids], self.lFill[ids] - hl[ids], np.maximum)
        totv = np.zeros(nbpits)
        hmax = np.full(nbpits, MISSING_DATA_SENTINEL)
        diffh = np.zeros(nbpits)
        ok = uids > -1
        totv[uids[ok]] = vol[ok]
        hmax[uids[ok]] = hh[ok]
        diffh[uids[ok]] = dh[ok]
        self.pitParams = np.empty((nbpits, 3))
        self.pitParams[:, 0] = totv
        self.pitParams[:, 1] = hmax
        self.pitParams[:, 2] = diffh

    def _pitInformation(self, hl, level, sed=False):
        """pitfilling.py:704-847 at one rank."""
        pitIDs = F.label_pits(level if sed else self.sealevel, self.lFill).astype(int)
        pitIDs[self.outletIDs] = -1
        pitNb = self._transferIDs(pitIDs)
        pitnbs = len(pitNb) + 1
        ngb = self.FVmesh_ngbID
        valid = ngb >= 0
        cidx = np.where(valid, ngb, 0)
        hc = self.lFill[cidx]
        hi = self.lFill[:, None]
        lower = valid & (hc < hi)
        eqlvl = valid & (hc == hi) & ((self.borders[cidx, 1] > 0) | (self.pitIDs[cidx] == -1))
        ispit = self.pitIDs > -1
        qual = (lower.any(axis=1) | eqlvl.any(axis=1)) & ispit & (self.inIDs == 1)
        qidx = np.where(qual)[0]
        bestlid = np.full(pitnbs, np.iinfo(np.int64).max, dtype=np.int64)
        if qidx.size:
            np.minimum.at(bestlid, self.pitIDs[qidx], self.locIDs[qidx])
        spillIDs = -np.ones(pitnbs, dtype=int)
        rank = -np.ones(pitnbs, dtype=int)
        lspill = np.zeros(self.lpoints, dtype=np.int32)
        if qidx.size:
            star = qidx[self.locIDs[qidx] == bestlid[self.pitIDs[qidx]]]
            isA = lower[star].any(axis=1)
            sA = star[isA]
            spillIDs[self.pitIDs[sA]] = sA
            rank[self.pitIDs[sA]] = 0
            lspill[sA] = 1
            for i in star[~isA]:
                knb = ngb[i][eqlvl[i]]
                s = int(knb[np.argmin(self.locIDs[knb])])
                spillIDs[self.pitIDs[i]] = s
                rank[self.pitIDs[i]] = 0
                lspill[s] = 1
        self.lspillIDs = np.where(lspill == 1)[0]
        spillIDs[rank != 0] = -1
        self.pitInfo = np.zeros((pitnbs, 2), dtype=int)
        self.pitInfo[:, 0] = spillIDs
        self.pitInfo[:, 1] = rank
        self.pitIDs[self.outletIDs] = -1
        self._dirFlats()
        idd = self.lFill <= self.sealevel
        h = hl.copy()
        self.lFill[idd] = hl[idd]
        self.flatDirs[idd] = -1
        if sed:
            self.lFill[idd] = hl[idd]
            self.flatDirs[idd] = -1
        else:
            h[h < self.sealevel] = self.sealevel
        self._getPitParams(h, pitnbs)

    def fillElevation(self, sed=False):
        """pitfilling.py:849-903"""
        hl = self.h.copy()
        minh = hl.min()
        if not self.flatModel:
            minh += 1.0e-3
        level = max(minh, self.sealevel + self.oFill)
        self._performFilling(hl - level, level, sed)
        self.lFill += level
        self._pitInformation(hl, level, sed)
        ids = self.pitParams[:, 0] > 0.0
        dh = np.zeros((len(self.pitInfo), 6))
        dh[ids, 0] = self.pitParams[ids, 1] - self.pitParams[ids, 2]
        dh[ids, 1:] = np.expand_dims(self.pitParams[ids, 2] / 5.0, axis=1)
        self.filled_lvl = np.cumsum(dh, axis=1)[:, 1:]
        self.filled_vol = np.zeros((len(self.pitInfo), 5))
        hl_clip = hl.copy()
        if not sed:
            hl_clip[hl_clip < self.sealevel] = self.sealevel
        self.filled_vol[:, :-1] = F.getpitvol(self.filled_lvl[:, :-1], hl_clip, self.pitIDs, self.inIDs)
        self.filled_vol[:, -1] = self.pitParams[:, 0]
        self.level = level

    # ------------------------------------------------------------ flow routing
    def _buildFlowDirection(self, h, down=True):
        """flowplex.py:480-544"""
        self.seaID = np.where(self.lFill <= self.sealevel)[0]
        rcv, dist, wgt = F.mfdreceivers(self.flowDir, self.flowExp, h, self.sealevel, self.gid)
        self.rcvID = rcv.astype(int)
        self.distRcv = dist
        self.wghtVal = wgt
        if down:
            sum_weight = np.sum(self.wghtVal, axis=1)
            ids = ((h == self.lFill) & (self.pitIDs > -1) & (self.flatDirs > -1) & (sum_weight == 0.0))
            ids = ids.nonzero()[0]
            self.rcvID[ids, :] = np.tile(ids, (self.flowDir, 1)).T
            self.rcvID[ids, 0] = self.flatDirs[ids]
            self.wghtVal[ids, :] = 0.0
            self.wghtVal[ids, 0] = 1.0
        if self.flatModel:
            self.rcvID[self.outletIDs, :] = np.tile(self.outletIDs, (self.flowDir, 1)).T
            self.distRcv[self.outletIDs, :] = 0.0
            self.wghtVal[self.outletIDs, :] = 0.0
        sum_weight = np.sum(self.wghtVal, axis=1)
        lsink = sum_weight == 0.0
        lsink[self.outletIDs] = False
        lsink[self.seaID] = False
        self.lsink = (lsink.astype(int) * self.inIDs) == 1

    def _flow_solve(self, b):
        """Exact (I - W^T) q = b for the current receivers (flowplex.py:429-478)."""
        q, left = F.flow_solve(self.rcvID, self.wghtVal, b)
        if left > 0:
            n = self.lpoints
            rows, cols, vals = [np.arange(n)], [np.arange(n)], [np.ones(n)]
            for k in range(self.flowDir):
                r = self.rcvID[:, k]
                keep = r != np.arange(n)
                rows.append(np.arange(n)[keep])
                cols.append(r[keep])
                vals.append(-self.wghtVal[keep, k])
            A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                              shape=(n, n)).T.tocsc()
            q = spla.spsolve(A, b)
        self.stats.append(("flow_cycles", left))
        return q

    def _distributeDownstream(self, pitVol, FA, hl, step):
        """flowplex.py:576-686 (no evaporation)."""
        excess = False
        FA = np.multiply(FA, self.inIDs)
        uID, vol = group_reduce(self.pitIDs[self.lsink], FA[self.lsink])
        inV = np.zeros(len(self.pitParams))
        ok = uID > -1
        inV[uID[ok]] = vol[ok]
        eV = inV - pitVol
        nFA = None
        if (eV > 0.0).any():
            eIDs = eV > 0.0
            pitVol[eIDs] = 0.0
            spillIDs = self.pitInfo[eIDs, 0]
            localSpill = np.where(self.pitInfo[eIDs, 1] == 0)[0]
            localPts = spillIDs[localSpill]
            nFA = np.zeros(self.lpoints)
            nFA[localPts] = eV[eIDs][localSpill]
            ids = np.isin(self.pitIDs, np.where(eV > 0.0)[0])
            self.waterFilled[ids] = self.lFill[ids]
        if (eV < 0.0).any():
            eIDs = np.where((eV < 0.0) & (inV > 0.0))[0]
            pitVol[eIDs] += eV[eIDs]
            nid = np.absolute(self.filled_vol[eIDs] - pitVol[eIDs][:, None]).argmin(axis=1)
            fill_lvl = self.filled_lvl[eIDs, nid]
            in_eIDs = np.isin(self.pitIDs, eIDs)
            pit_fill_lvl = np.zeros(len(self.pitParams))
            pit_fill_lvl[eIDs] = fill_lvl
            node_lvl = pit_fill_lvl[self.pitIDs]
            mask = in_eIDs & (self.waterFilled <= node_lvl)
            self.waterFilled[mask] = node_lvl[mask]
        if (eV > 1.0e-3).any():
            if step == 100:
                self._buildFlowDirection(self.lFill)
            else:
                self._buildFlowDirection(self.waterFilled)
            rhs = nFA / self.dt
            resid = rhs.sum()
            self._cascade_resid = float(resid)
            if resid > self.maxarea[0]:
                excess = True
                sol = self._flow_solve(rhs)
                nFA = sol.copy() * self.dt
                FA = nFA.copy()
                FA[hl < self.waterFilled] = 0.0
                self.FAL = self.FAL + FA / self.dt
            else:
                nFA = None
        else:
            nFA = None
        return excess, pitVol, nFA

    def flowAccumulation(self):
        """flowplex.py:752-945 (no evaporation, no ice)."""
        self.fillElevation(sed=False)
        pitVol = self.pitParams[:, 0].copy()
        hl = self.h.copy()
        self._buildFlowDirection(hl, False)
        self.wghtVali = self.wghtVal.copy()
        self.rcvIDi = self.rcvID.copy()
        self.distRcvi = self.distRcv.copy()
        self.lsinki = self.lsink.copy()
        rainA = self.bL.copy()
        rainA[self.seaID] = 0.0
        self.FAL = self._flow_solve(rainA)
        self.waterFilled = hl.copy()
        npass = 0
        if (pitVol > 0.0).any():
            FA = self.FAL.copy() * self.dt
            excess = True
            step = 0
            best_resid = None
            stall = 0
            while excess and step <= 100:
                excess, pitVol, FA = self._distributeDownstream(pitVol, FA, hl, step)
                step += 1
                npass += 1
                if excess:
                    resid = self._cascade_resid
                    if best_resid is None or resid < best_resid * (1.0 - 1.0e-3):
                        best_resid = resid
                        stall = 0
                    else:
                        stall += 1
                        if stall >= 3:
                            break
            FA = self.FAL.copy()
            ids = (hl <= self.waterFilled) & (self.pitIDs > -1)
            FA[ids] = 0.0
            self.FAL = FA.copy()
            FA[ids] = self.FAL.max() * 0.1
            self.fillFAL = FA
        else:
            self.fillFAL = self.FAL.copy()
        self.FAL = np.clip(self.FAL, 0.0, None)
        self.fillFAL = np.clip(self.fillFAL, 0.0, None)
        self.waterFilled = self.waterFilled - hl
        self.cascade_passes = npass

    # --------------------------------------------------------------------- SPL
    def spl_coefficients(self, hOld):
        """Per-receiver implicit SPL coefficients c_ik (SPL.py:45-114)."""
        PA = self.FAL
        K = np.asarray(self.K, dtype=np.float64)
        Kbr = K * np.ones(self.lpoints) * np.ones(self.lpoints) * (self.rainVal ** self.coeffd)
        Kbr *= self.dt * (PA ** self.spl_m)
        Kbr[self.seaID] = 0.0
        wght = self.wghtVali.copy()
        wght[self.seaID, :] = 0.0
        nodes = np.arange(self.lpoints)
        c = np.zeros((self.lpoints, self.flowDir))
        for k in range(self.flowDir):
            dh = hOld - hOld[self.rcvIDi[:, k]]
            limiter = np.divide(dh, dh + 1.0e-2, out=np.zeros_like(dh), where=dh != 0)
            data = np.divide(Kbr * limiter, self.distRcvi[:, k], out=np.zeros_like(PA),
                             where=self.distRcvi[:, k] != 0)
            data = np.multiply(data, wght[:, k])
            data[self.rcvIDi[:, k] == nodes] = 0.0
            c[:, k] = data
        return c

    def coupled_ed(self, hOld, c):
        """Transport-limited SPL, _getEroDepRate's G > 0 branch (SPL.py:305-336)
        and _coupledEDSystem (SPL.py:116-258): the nested system
            [eMat - diag(f)      -diag(f dt / A)] [h]   [(1 - f) hOld ]
            [diag(A / dt)         (I - W)^T     ] [q] = [hOld A / dt  ]
        with f = G A / max(FAL, G A / 0.99) (0 where FAL = 0, at sea and at
        flat-model outlets, capped at 0.99) and (I - W)^T the snapshot flow
        matrix fMati (flowplex.py:787-791, matrixFlow 429-478), solved exactly
        (sparse direct) where goSPL uses TFQMR with a Schur fieldsplit."""
        n = self.lpoints
        PA = self.FAL
        num = self.fDepa * self.larea
        floor_ = num / 0.99
        f = np.divide(num, np.maximum(PA, floor_), out=np.zeros_like(PA), where=PA != 0)
        f[self.seaID] = 0.0
        f[f > 0.99] = 0.99
        if self.flatModel:
            f[self.outletIDs] = 0.0
        nodes = np.arange(n)
        R = self.flowDir
        rows, cols, vals = [nodes], [nodes], [1.0 + c.sum(axis=1) - f]
        wr, wc, wv = [nodes], [nodes], [np.ones(n)]
        for k in range(R):
            r = self.rcvIDi[:, k]
            keep = r != nodes
            rows.append(nodes[keep]); cols.append(r[keep]); vals.append(-c[keep, k])
            w = self.wghtVali[:, k]
            keepw = keep & (w != 0.0)
            # (I - W)^T: row r gets -w at column i
            wr.append(r[keepw]); wc.append(nodes[keepw]); wv.append(-w[keepw])
        A00 = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
        A11 = sp.csr_matrix((np.concatenate(wv), (np.concatenate(wr), np.concatenate(wc))), shape=(n, n))
        A01 = sp.diags(-f * self.dt / self.larea)
        A10 = sp.diags(self.larea / self.dt)
        M = sp.bmat([[A00, A01], [A10, A11]], format="csc")
        rhs = np.concatenate([(1.0 - f) * hOld, hOld * self.larea / self.dt])
        return spla.spsolve(M, rhs)[:n]

    def erodepSPL(self):
        """SPL.py:402-454 with _getEroDepRate SPL.py:260-366 (G = 0, or the
        coupled erosion-deposition system when G > 0)."""
        hOld = self.h.copy()
        c = self.spl_coefficients(hOld)
        if self.fDepa > 0.0:
            stepED = self.coupled_ed(hOld, c)
        else:
            stepED, left = F.spl_solve(self.rcvIDi, c, hOld)
            if left > 0:
                raise RuntimeError("SPL system is not triangular (%d rows left)" % left)
        E = (stepED - hOld) / self.dt
        if self.flatModel:
            E[self.outletIDs] = 0.0
        E[self.lsink] = 0.0
        dz = E * self.dt
        self.cumED = self.cumED + dz
        self.h = self.h + dz
        self.EbLocal = dz / self.dt

    # --------------------------------------------------------------- hillslope
    def diffusion_matrix(self, Kd):
        """_buildDiffMat + _assembleDiffMat (hillslope.py:235-293) as CSR."""
        coeffs = F.sethillslopecoeff(self.lpoints, Kd)
        if self.flatModel:
            coeffs[self.outletIDs, 1:] = 0.0
            coeffs[self.outletIDs, 0] = 1.0
        n = self.lpoints
        rows = [np.arange(n)]
        cols = [np.arange(n)]
        vals = [coeffs[:, 0]]
        for k in range(self.maxnb):
            data = coeffs[:, k + 1]
            idx = self.FVmesh_ngbID[:, k].copy()
            nz = data != 0.0
            rows.append(np.arange(n)[nz])
            cols.append(idx[nz])
            vals.append(data[nz])
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(n, n))

    def _diffusion_solve(self, A, b):
        if self.lpoints <= 300000:
            return spla.spsolve(A.tocsc(), b)
        # large meshes: CG on the area-weighted form to 1e-14, then check
        d = self.larea
        As = sp.diags(d) @ A
        x, info = spla.cg(As, d * b, x0=b.copy(), rtol=1e-14, maxiter=5000)
        return x

    def getHillslope(self):
        """hillslope.py:614-649 -> _hillSlope(smooth=0) hillslope.py:90-233."""
        self.seaID = np.where(self.h <= self.sealevel)[0]
        if self.Cda == 0.0 and self.Cdm == 0.0:
            return
        hOld = self.h.copy()
        if self._hill_mat is None or not np.array_equal(self.seaID, self._hill_seaID):
            Cd = np.full(self.lpoints, self.Cda)
            Cd[self.seaID] = self.Cdm
            self._hill_mat = self.diffusion_matrix(Cd * self.dt)
            self._hill_seaID = self.seaID.copy()
        hNew = self._diffusion_solve(self._hill_mat, hOld)
        tmp = hNew - hOld
        self.cumED = self.cumED + tmp
        self.h = hNew
        self.EbLocal = self.EbLocal + tmp / self.dt

    # ------------------------------------------------- continental deposition
    def _getSedFlux(self):
        """sedplex.py:103-188 (no stratigraphy, no provenance): the volumetric
        sediment flux vSed (m3/yr) = (I - W^T)^-1 (-Eb * area) over the
        snapshot receivers of the last flowAccumulation (fMati)."""
        rhs = -self.EbLocal * self.larea
        q, left = F.flow_solve(self.rcvIDi, self.wghtVali, rhs)
        if left > 0:
            raise RuntimeError("snapshot flow graph is not acyclic (%d rows left)" % left)
        self.vSed = q

    def _moveDownstream(self, vSed, step):
        """sedplex.py:190-374 (single lithology, no provenance, one rank).
        Returns (excess, routed flux or None)."""
        excess = False
        changed = False
        B = self.sed_budget
        csink = self.lsink & (self.pitIDs < 0)
        if csink.any():
            if not self._domainHasOutlet:
                self._closedDepo[csink] += vSed[csink]
            vSed = vSed.copy()
            vSed[csink] = 0.0
        uID, vol = group_reduce(self.pitIDs[self.lsink], vSed[self.lsink])
        inV = np.zeros(len(self.pitParams))
        ok = uID > -1
        inV[uID[ok]] = vol[ok]
        nvSed = np.zeros(self.lpoints)
        eV = inV - self.pitVol
        # budget: the pass's inflow split (before pitVol changes)
        B["retained"] += float(np.sum(np.where(eV > 0.0, self.pitVol, np.where(eV < 0.0, inV, 0.0))))
        B["excess"] += float(np.sum(eV[eV > 0.0]))
        B["zero_excess"] += float(np.sum(inV[eV == 0.0]))
        B["inflow"] += float(np.sum(inV))
        if (eV > 0.0).any():
            eIDs = eV > 0.0
            spillIDs = self.pitInfo[eIDs, 0]
            localSpill = np.where(self.pitInfo[eIDs, 1] == 0)[0]
            localPts = spillIDs[localSpill]
            nvSed[localPts] = eV[eIDs][localSpill]
            self.pitVol[eIDs] = 0.0
            ids = np.isin(self.pitIDs, np.where(eV > 0.0)[0])
            self.sedFilled[ids] = self.lFill[ids]
            changed = True
            B["placed"] += float(nvSed.sum())
        eIDs = eV < 0
        self.pitVol[eIDs] -= inV[eIDs]
        self.pitVol[self.pitVol < 0] = 0.0
        routed = None
        if (eV > 1.0e-3).any():
            if changed or step == 0 or step == 100:
                if step == 100:
                    self._buildFlowDirection(self.lFill)
                else:
                    self._buildFlowDirection(self.sedFilled)
            if nvSed.sum() > 0.5 * self.maxarea[0]:
                excess = True
                routed = self._flow_solve(nvSed)
                B["routed"] += float(nvSed.sum())
                self._budget_cells(routed, self.wghtVal)
        return excess, routed

    def _budget_cells(self, u, wgt):
        """Sediment budget: the volumes u at the terminal cells of the graph
        wgt (every weight 0), by kind (depression sinks, stray sinks kept on
        a closed domain or dropped, open outlets, other terminal cells)."""
        B = self.sed_budget
        term = np.all(wgt == 0.0, axis=1)
        out = np.zeros(self.lpoints, dtype=bool)
        out[self.outletIDs] = True
        lsink = self.lsink & ~out
        B["outlets"] += float(np.sum(u[term & out]))
        B["pit_sinks"] += float(np.sum(u[term & lsink & (self.pitIDs >= 0)]))
        stray = float(np.sum(u[term & lsink & (self.pitIDs < 0)]))
        B["dropped" if self._domainHasOutlet else "kept"] += stray
        B["sea"] += float(np.sum(u[term & ~out & ~self.lsink]))

    def _distributeSediment(self, hl):
        """sedplex.py:376-522 (single lithology, no provenance)."""
        vSed = self.vSed.copy() * self.dt
        self._budget_cells(vSed, self.wghtVali)
        self._closedDepo = np.zeros(self.lpoints)
        step = 0
        excess = True
        while excess:
            if step >= 5000:
                break
            excess, routed = self._moveDownstream(vSed, step)
            if excess:
                vSed = routed.copy()
                nvSed = vSed.copy()
                nvSed[hl < self.sedFilled] = 0.0
                self.vSed = self.vSed + nvSed / self.dt
                vSed[self.outletIDs] = 0.0
            step += 1
        self.sed_passes = step
        self.sed_budget["kept_deposit"] = float(np.sum(self._closedDepo))
        if self._closedDepo.any():
            delta = np.zeros(self.lpoints)
            nz = self._closedDepo > 0.0
            delta[nz] = self._closedDepo[nz] / self.larea[nz]
            self.cumED = self.cumED + delta
            self.h = self.h + delta

    def _bottomUpDelta(self, hl, depo, pit_select):
        """sedplex.py:524-559: lake surface at the level whose filled volume
        matches the deposit (np.interp over the pit's depth-volume table)."""
        num_pits = len(self.pitParams)
        target_lvl = np.full(num_pits, -np.inf)
        active = np.where(pit_select & (depo > 0))[0]
        for p in active:
            pit_min = self.pitParams[p, 1] - self.pitParams[p, 2]
            vols = np.concatenate(([0.0], self.filled_vol[p]))
            lvls = np.concatenate(([pit_min], self.filled_lvl[p]))
            target_lvl[p] = np.interp(depo[p], vols, lvls)
        node_target_lvl = np.full(self.lpoints, -np.inf)
        in_pit = self.pitIDs >= 0
        node_target_lvl[in_pit] = target_lvl[self.pitIDs[in_pit]]
        surface = np.minimum(node_target_lvl, self.lFill)
        delta = np.maximum(0.0, surface - hl)
        sel_node = np.isin(self.pitIDs, active) if active.size > 0 else np.zeros(self.lpoints, bool)
        delta[~sel_node] = 0.0
        return delta

    def _addPitMicroTilt(self, delta, pit_select):
        """sedplex.py:561-644: tilt each partly filled lake surface by 1e-6
        m/m towards its spill point, per-pit mean distance removed."""
        num_pits = len(self.pitParams)
        if not pit_select.any():
            return delta
        active_pit = np.where(pit_select)[0]
        sel_node = np.isin(self.pitIDs, active_pit) & (delta > 0)
        spill_xyz = np.zeros((num_pits, 3))
        spill_idx = self.pitInfo[:, 0].astype(int)
        mp = np.where((self.pitInfo[:, 1] == 0) & (spill_idx >= 0))[0]
        spill_xyz[mp] = self.lcoords[spill_idx[mp]]
        in_pit = self.pitIDs >= 0
        pit_safe = np.where(in_pit, self.pitIDs, 0)
        dist = np.linalg.norm(self.lcoords - spill_xyz[pit_safe], axis=1)
        local_sum = np.zeros(num_pits)
        local_cnt = np.zeros(num_pits)
        if sel_node.any():
            ids = self.pitIDs[sel_node]
            up, sums = group_reduce(ids, dist[sel_node])
            _, cnts = group_reduce(ids, np.ones_like(dist[sel_node]))
            local_sum[up] = sums
            local_cnt[up] = cnts
        with np.errstate(divide="ignore", invalid="ignore"):
            mean_dist = np.where(local_cnt > 0, local_sum / np.maximum(local_cnt, 1.0), 0.0)
        tilt = 1.0e-6 * (dist - mean_dist[pit_safe])
        tilt[~sel_node] = 0.0
        tilted = delta + tilt
        tilted[tilted < 0] = 0.0
        return tilted

    def _identifyPitInlets(self):
        """sedplex.py:646-677: cells receiving flow (snapshot receivers) from a
        donor outside their own depression."""
        R = self.rcvIDi.shape[1]
        src = np.repeat(np.arange(self.lpoints), R)
        dst = self.rcvIDi.flatten().astype(int)
        good = src != dst
        src, dst = src[good], dst[good]
        sp, dp = self.pitIDs[src], self.pitIDs[dst]
        e = (dp >= 0) & (sp != dp)
        mask = np.zeros(self.lpoints, dtype=bool)
        if e.any():
            mask[dst[e]] = True
        return mask

    def _diffuseImplicitPicard(self, dh, mask, Cd_val):
        """hillslope.py:988-1076 (marineSolver picard): picardSub backward-Euler
        sub-steps, each with picardIts solves of (I + dt_sub L(C_d(h))) h =
        h_start, L from jacobiancoeff with Kp = 0; solved exactly here where
        goSPL runs Richardson + block Jacobi to rtol."""
        nsub, npic = self.picardSub, self.picardIts
        dt_sub = self.dt / nsub
        n = self.lpoints
        Cd0 = np.zeros(n)
        Cd0[mask] = Cd_val
        minDiff_vec = np.zeros(n)
        minDiff_vec[mask] = self.minDiff
        zb = self.h.copy()
        zeroKp = np.zeros(n)
        h = dh + zb
        nodes = np.arange(n)
        ngb = self.FVmesh_ngbID[:, :self.maxnb]
        for _ in range(nsub):
            hstart = h.copy()
            for _ in range(npic):
                dhdep = h - zb
                dhdep[dhdep < 0.1] = 0.0
                Cd = minDiff_vec + np.multiply(Cd0, 1.0 - np.exp(-self.dexp * dhdep))
                nlC = F.jacobiancoeff(h, Cd, zeroKp)
                coeffs = dt_sub * nlC
                coeffs[:, 0] += 1.0
                off = coeffs[:, 1:1 + self.maxnb]
                keep = off != 0.0
                rows = np.concatenate([nodes, np.repeat(nodes, self.maxnb)[keep.ravel()]])
                cols = np.concatenate([nodes, ngb.ravel()[keep.ravel()]])
                vals = np.concatenate([coeffs[:, 0], off.ravel()[keep.ravel()]])
                M = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
                h = spla.spsolve(M.tocsc(), hstart)
        ndepo = h - zb
        ndepo[ndepo < 0.0] = 0.0
        return ndepo

    def _diffuseLargePit(self, hl, depo, pit_select):
        """sedplex.py:679-858 (one rank): bathymetric bottom-up baseline plus an
        inlet pile, smoothed by non-linear diffusion over the pit cells, each
        pit's deposit rescaled to its volume."""
        num_pits = len(self.pitParams)
        active = np.where(pit_select & (depo > 0))[0]
        if active.size == 0:
            return np.zeros(self.lpoints)
        sel_node = np.isin(self.pitIDs, active)
        inlet_mask = self._identifyPitInlets() & sel_node
        inlet_count = np.zeros(num_pits)
        if inlet_mask.any():
            ids = self.pitIDs[inlet_mask]
            up, cnts = group_reduce(ids, np.ones_like(ids, dtype=np.float64))
            inlet_count[up] = cnts
        no_inlet = active[inlet_count[active] == 0]
        for p in no_inlet:
            pit_local = np.where(self.pitIDs == p)[0]
            if pit_local.size > 0:
                k = np.argmax(hl[pit_local])
                inlet_mask[int(pit_local[k])] = True
                inlet_count[p] = 1.0
        bias_frac = self.nl_pit_inlet_bias
        target_lvl = np.full(num_pits, -np.inf)
        for p in active:
            pit_min = self.pitParams[p, 1] - self.pitParams[p, 2]
            vols = np.concatenate(([0.0], self.filled_vol[p]))
            lvls = np.concatenate(([pit_min], self.filled_lvl[p]))
            target_lvl[p] = np.interp(depo[p], vols, lvls)
        in_pit = self.pitIDs >= 0
        pit_safe = np.where(in_pit, self.pitIDs, 0)
        node_lvl = np.where(in_pit, target_lvl[pit_safe], -np.inf)
        water_depth = np.maximum(0.0, node_lvl - hl)
        water_depth[~sel_node] = 0.0
        denom = np.zeros(num_pits)
        if sel_node.any():
            ids = self.pitIDs[sel_node]
            up, sums = group_reduce(ids, (water_depth * self.larea)[sel_node])
            denom[up] = sums
        delta_init = np.zeros(self.lpoints)
        denom_node = denom[pit_safe]
        ok = (denom_node > 0) & sel_node
        delta_init[ok] = ((1.0 - bias_frac) * depo[pit_safe[ok]] * water_depth[ok]
                          / np.maximum(denom_node[ok], 1e-30))
        bias_at_inlet = np.where(denom > 0, bias_frac, 1.0)
        for c in np.where(inlet_mask)[0]:
            p = self.pitIDs[c]
            if inlet_count[p] > 0:
                delta_init[c] += bias_at_inlet[p] * depo[p] / (inlet_count[p] * self.larea[c])
        delta_smooth = self._diffuseImplicitPicard(delta_init, sel_node, self.nl_pit_K)
        actual_vol = np.zeros(num_pits)
        if sel_node.any():
            ids = self.pitIDs[sel_node]
            up, sums = group_reduce(ids, (delta_smooth * self.larea)[sel_node])
            actual_vol[up] = sums
        with np.errstate(divide="ignore", invalid="ignore"):
            scale = np.where(actual_vol > 0, depo / np.maximum(actual_vol, 1e-30), 1.0)
        node_scale = scale[pit_safe]
        node_scale[~sel_node] = 0.0
        return delta_smooth * node_scale

    def _updateSinks(self, hl):
        """sedplex.py:982-1059.  Path 3 (partly filled depressions of at least
        nlPitVolume and nlPitDepth) is restated for marineSolver picard; goSPL's
        default adaptive TS solve is not."""
        depo = self.pitParams[:, 0] - self.pitVol
        depo[depo < 0] = 0.0
        pit_volume = self.pitParams[:, 0]
        pit_depth = self.pitParams[:, 2]
        active = depo > 0
        full_fill = active & (depo >= pit_volume - 1.0e-6)
        partial = active & ~full_fill
        is_large = (pit_volume >= self.nl_pit_volume) & (pit_depth >= self.nl_pit_depth)
        diffuse_path = partial & is_large
        bottomup_path = full_fill | (partial & ~is_large)
        if diffuse_path.any() and self.marineSolver != "picard":
            raise NotImplementedError("lake deposition by non-linear diffusion (%d large deep pits) with the "
                                      "adaptive TS solver" % int(diffuse_path.sum()))
        delta = self._bottomUpDelta(hl, depo, bottomup_path)
        if bottomup_path.any():
            delta = self._addPitMicroTilt(delta, bottomup_path)
        if diffuse_path.any():
            delta = delta + self._diffuseLargePit(hl, depo, diffuse_path)
        self.sed_delta = delta
        self.cumED = self.cumED + delta
        self.h = self.h + delta
        self.pitParams[:, 0] = self.pitVol.copy()

    def sedChange(self):
        """sedplex.py:1061-1086.  Also keeps `sed_budget`, the step's sediment
        budget (m3): where the eroded volume went (depressions, closed-domain
        sinks, outlets, sea) and what the routing's rules drop (`budget`)."""
        self.sed_budget = {k: 0.0 for k in BUDGET_SLOTS}
        self.sed_budget["eroded"] = float(np.sum(-self.EbLocal * self.larea * self.dt))
        self._getSedFlux()
        self.fillElevation(sed=True)
        hl = self.h.copy()
        self.lsink = self.lsinki.copy()
        self.pitVol = self.pitParams[:, 0].copy()
        self.sedFilled = hl.copy()
        self._distributeSediment(hl)
        self._updateSinks(hl)
        self.sed_budget["realised"] = float(np.sum(self.larea * (self.h - hl)))
        self.sed_budget = budget(self.sed_budget)


    # ------------------------------------------------------ marine deposition
    def _distanceCoasts(self, hl):
        """seaplex.py:51-135 on one rank: the distance of every sea vertex
        (seaID) to the nearest point of the coastline, the sea-level contour
        of the elevation over the mesh triangles; 0 elsewhere and when there
        is no coastline."""
        self.coastDist = np.zeros(self.lpoints)
        pts = coast_points(self.lcoords, self.lcells, hl, self.sealevel)
        if len(pts) == 0:
            return
        from scipy import spatial
        tree = spatial.cKDTree(pts, leafsize=10)
        self.coastDist[self.seaID], _ = tree.query(self.lcoords[self.seaID, :], k=1)

    def _smoothBathymetry(self):
        """_hillSlope(smooth=2) (hillslope.py:124-139): one implicit step of
        linear diffusion with K_d = N * area, N = 1 on land and 5 at sea
        (tools/constants.py:126-127), solved exactly."""
        Cd = np.full(self.lpoints, MARINE_SMOOTH_N_LAND)
        Cd[self.seaID] = MARINE_SMOOTH_N_SEA
        A = self.diffusion_matrix(Cd * self.larea)
        return self._diffusion_solve(A, self.h.copy())

    def _matOcean(self):
        """seaplex.py:137-238: marine receivers on the epsilon-filled smoothed
        bathymetry (every lower neighbour, equal weights), terminal sinks,
        and the transposed routing matrix dMat1."""
        hl = self.h.copy()
        minh = self.h.min() + 0.1
        if not self.flatModel:
            minh = max(minh, self.oFill)
            hsmth = self._smoothBathymetry()
            hsmth[self.coastDist > self.offshore] = BOUNDARY_FLOW_SENTINEL
        else:
            minh = max(minh, self.oFill)
            hsmth = hl.copy()
            hsmth[self.outletIDs] = BOUNDARY_FLOW_SENTINEL
        fillz = F.epsfill(minh, hsmth)
        if not self.flatModel:
            far = self.coastDist > self.offshore
            fillz[far] = hl[far]
        rcv, _, wght = F.mfdrcvrs(12, self.flowExp, fillz, BOUNDARY_FLOW_SENTINEL, self.gid)
        if self.flatModel:
            rcv[self.outletIDs, :] = np.tile(self.outletIDs, (12, 1)).T
            wght[self.outletIDs, :] = 0.0
        nodes = np.arange(self.lpoints)
        self.is_sink_local = np.all(rcv.astype(int) == nodes[:, None], axis=1)
        if self.flatModel:
            self.is_sink_local[self.outletIDs] = False
        data = wght.copy()
        data[rcv == nodes[:, None]] = 0.0
        # ADD_VALUES assembly: receivers shared by several directions sum
        off = sp.csr_matrix((data.ravel(), rcv.ravel().astype(np.int64), np.arange(0, 12 * self.lpoints + 1, 12)),
                            shape=(self.lpoints, self.lpoints))
        off.sum_duplicates()
        self.dMat1 = off.T.tocsr()
        self.dMat1.sort_indices()
        if not self.flatModel and self.Gmar > 0.0:
            d2 = (sp.identity(self.lpoints, format="csr") + off * -1.0).tocsr()
            d2.sum_duplicates()
            self.dMat2 = d2.T.tocsr()
            self.dMat2.sort_indices()

    def _depMarineSystem(self, sedflux):
        """seaplex.py:240-402 (Gmar > 0, spheres): the coupled marine elevation
        / flux system [[I - G, -G dt / A], [A / dt, dMat2]] [h; q] =
        [(1 - G) h; sedflux / dt + h A (1 / dt)] with G = min(Gmar, 0.99) below
        sea level and 0 above, solved exactly (goSPL: TFQMR with a Schur
        fieldsplit to rtol); returns the deposited volumes (new h - h) * area,
        negatives dropped."""
        n = self.lpoints
        hl = self.h.copy()
        fDepm = np.full(n, self.Gmar)
        fDepm[fDepm > 0.99] = 0.99
        fDepm[hl > self.sealevel] = 0.0
        A00 = sp.diags(-fDepm + 1.0, format="csr")
        A01 = sp.diags(-fDepm * self.dt / self.larea, format="csr")
        A10 = sp.diags(self.larea / self.dt, format="csr")
        M = sp.bmat([[A00, A01], [A10, self.dMat2]], format="csc")
        rhs = np.concatenate([(1.0 - fDepm) * self.h, sedflux / self.dt + (self.h * self.larea) * (1.0 / self.dt)])
        x = spla.spsolve(M, rhs)
        volDep = (x[:n] - self.h) * self.larea
        volDep[volDep < 0] = 0.0
        return volDep

    def _distOcean(self, sedflux):
        """seaplex.py:404-619 (no provenance): the marine volumes pass down
        dMat1 one hop per iteration; a cell keeps what fits in its remaining
        capacity maxDepQs and passes the rest; terminal sinks keep all, open
        outlets lose all; the iteration stops once the volume in transit is at
        most max(1 m3, 1e-6 of the input) (or after 5000 passes) and what is
        left in transit is deposited where it stands."""
        marVol = self.maxDepQs.copy()
        sinkVol = sedflux.copy()
        vdep = np.zeros(self.lpoints)
        sink = self.is_sink_local
        if sink.any():
            sink_mass = sinkVol[sink]
            if (sink_mass != 0).any():
                vdep[sink] += sink_mass
                sinkVol[sink] = 0.0
        tmp = sinkVol.copy()
        sumExcess = float(np.sum(tmp))
        threshold = max(1.0, 1.0e-6 * sumExcess)
        step = 0
        while sumExcess > threshold:
            if step >= 5000:
                break
            sinkVol = self.dMat1 @ tmp
            excess = sinkVol >= marVol
            sinkVol[excess] -= marVol[excess]
            vdep[excess] += marVol[excess]
            marVol[excess] = 0.0
            noexcess = np.invert(excess)
            marVol[noexcess] -= sinkVol[noexcess]
            vdep[noexcess] += sinkVol[noexcess]
            vdep[self.outletIDs] = 0.0
            sinkVol[noexcess] = 0.0
            sinkVol[self.outletIDs] = 0.0
            if sink.any():
                vdep[sink] += sinkVol[sink]
                sinkVol[sink] = 0.0
            tmp = sinkVol.copy()
            sumExcess = float(np.sum(tmp))
            step += 1
        self.marine_passes = step
        if tmp.any():
            vdep += tmp
            vdep[self.outletIDs] = 0.0
        return vdep

    def seaChange(self):
        """SEAMesh.seaChange (seaplex.py:738-861), one lithology, no
        stratigraphy or provenance, marineSolver picard:
        clinoform capacity below sea level from the distance to the coast,
        routing of the sediment flux reaching the sea (sinks of the sediment
        fill) down the marine receivers, then non-linear diffusion of the
        marine deposit over the sea cells (_diffuseOcean -> the Picard solve)."""
        self.sinkIDs = self.lFill <= self.sealevel
        hl = self.h.copy()
        self._distanceCoasts(hl)                     # clinSlp >= 1e-6 always
        clinoH = self.sealevel - 1.0e-3 - self.coastDist * self.clinSlp
        clinoH[hl >= self.sealevel] = hl[hl >= self.sealevel]
        clinoH[clinoH < hl] = hl[clinoH < hl]
        self.maxDepQs = (clinoH - hl) * self.larea
        sedFlux = self.vSed.copy() * self.dt
        sedFlux[np.invert(self.sinkIDs)] = 0.0
        sedFlux[sedFlux < 0] = 0.0
        self._matOcean()
        marDep = self._distOcean(sedFlux)
        if not self.flatModel and self.Gmar > 0.0:
            vdep = self._depMarineSystem(marDep)
            marDep = self._distOcean(vdep)
        dh = np.divide(marDep, self.larea, out=np.zeros_like(self.larea), where=self.larea != 0)
        dh[dh < DEPOSIT_FLOOR] = 0.0
        ndepo = self._diffuseImplicitPicard(dh, self.seaID, self.nlK)     # _diffuseOcean, hillslope.py:739-787
        self.cumED = self.cumED + ndepo
        self.h = self.h + ndepo
        self.EbLocal = self.EbLocal + ndepo / self.dt

    # ------------------------------------------------------------------- loop
    def step(self):
        """One iteration of runProcesses with fast=False (model.py:347-453):
        flow, erosion, continental deposition unless nodep (flow again, then
        sedChange), hillslope, forcing."""
        self.flowAccumulation()
        self.erodepSPL()
        if not self.nodep:
            self.flowAccumulation()
            self.sedChange()
            if self.seaDepo:
                self.seaChange()
        self.getHillslope()
        if self.tNow < self.tEnd:
            self.applyForces()
        self.tNow += self.dt

    def runProcesses(self):
        while self.tNow <= self.tEnd:
            if self.tNow == self.tEnd:
                break
            self.step()

    # ----------------------------------------------------------------- output
    def output_fields(self):
        """The datasets WriteMesh._outputMesh writes for the current state
        (see ``output_fields`` below), with the last seaID built."""
        sea = np.zeros(self.lpoints, np.uint8)
        sea[np.asarray(self.seaID, np.int64)] = 1
        vsed = self.vSed if hasattr(self, "vSed") else np.zeros(self.lpoints)
        return output_fields(self.h, self.cumED, self.EbLocal, self.waterFilled, self.fillFAL, self.FAL, vsed,
                             self.upsub, self.rainVal, sea)


DISCHARGE_FLOOR = 1.0e-8   # gospl/tools/constants.py:51


def output_fields(h, cumED, Eb, waterFilled, fillFAL, FAL, vSed, upsub, rain, sea):
    """WriteMesh._outputMesh (gospl/tools/outmesh.py:252-478) for one rank,
    ``fast: False``, no ice, flexure, soil or dual lithology: name -> float32
    [n, 1].  FA and fillFA are floored at DISCHARGE_FLOOR and set to 1 on sea
    vertices (:334-356); sedLoad is floored (:426-435); every float64 field is
    rounded to float32 by the file's datatype."""
    sea = np.asarray(sea).astype(bool)

    def col(a):
        with np.errstate(over="ignore", invalid="ignore"):
            return np.asarray(a, np.float64).astype(np.float32).reshape(-1, 1)

    def floored(a, with_sea):
        d = np.array(a, np.float64, copy=True)
        d[d <= DISCHARGE_FLOOR] = DISCHARGE_FLOOR
        if with_sea:
            d[sea] = 1.0
        return d

    out = {"elev": col(h), "erodep": col(cumED), "EDrate": col(Eb), "waterFill": col(waterFilled),
           "fillFA": col(floored(fillFAL, True)), "FA": col(floored(FAL, True)), "sedLoad": col(floored(vSed, False))}
    if upsub is not None:
        out["uplift"] = col(upsub)
    if rain is not None:
        out["rain"] = col(rain)
    return out


def coast_points(coords, cells, scalar, value):
    """The points vtkContourFilter returns for the contour ``scalar ==
    value`` over the triangles ``cells`` with triangle generation off, as
    seaplex.py:105-120 uses it: marching triangles marks a vertex inside when
    its scalar is >= value, and every edge with one end inside gives a point
    interpolated from the end with the lower scalar,
    t = (value - s_lo) / (s_hi - s_lo), x = x_lo + t (x_hi - x_lo); the point
    locator merges the copies an edge's two triangles make (returned sorted,
    unique)."""
    cells = np.asarray(cells, dtype=np.int64)
    if len(cells) == 0:
        return np.zeros((0, 3))
    e = np.concatenate([cells[:, [0, 1]], cells[:, [1, 2]], cells[:, [2, 0]]])
    a, b = e[:, 0], e[:, 1]
    cross = (scalar[a] >= value) != (scalar[b] >= value)
    a, b = a[cross], b[cross]
    up = (scalar[b] - scalar[a]) > 0
    lo = np.where(up, a, b)
    hi = np.where(up, b, a)
    t = (value - scalar[lo]) / (scalar[hi] - scalar[lo])
    x = coords[lo] + t[:, None] * (coords[hi] - coords[lo])
    if len(x) == 0:
        return np.zeros((0, 3))
    return np.unique(x, axis=0)
