"""PETSc-free goSPL driver for the per-timestep surface-process path on a B200.

``Model`` keeps the reference's entry points and state names
(``gospl/model.py:179-495``):

* ``flowAccumulation()``  — FAMesh.flowAccumulation (flowplex.py:752-945)
* ``fillElevation(sed)``  — PITFill.fillElevation (pitfilling.py:849-903)
* ``_buildFlowDirection(h, down)`` — flowplex.py:480-544
* ``erodepSPL()``         — SPL.erodepSPL (SPL.py:402-454), n = 1, G >= 0
* ``sedChange()``         — SEDMesh.sedChange (sedplex.py:1061-1086):
  continental sediment routing and deposition in depressions
* ``getHillslope()``      — hillSLP.getHillslope (hillslope.py:614-649)
* ``applyForces()``       — UnstMesh.applyForces (unstructuredmesh.py:743-794)
* ``visModel()`` / ``readData()`` — WriteMesh (tools/outmesh.py): HDF5 and
  XDMF outputs every ``tout`` years and the restart from output ``rStep``
* ``seaChange()``         — SEAMesh.seaChange (seaplex.py:738-861): marine
  deposition (``seadepo``; marineSolver picard; the coupled system when Gmar > 0)
* ``runProcesses()``      — the time loop of model.py:331-466 with
  ``fast: false``, continental deposition unless ``nodep`` and marine
  deposition when ``seadepo``.

All state lives in torch CUDA tensors (float64 / int32 / uint8); every stage is
one call through the C ABI of ``libgospl_b200.so``.  Per-receiver arrays are
stored receiver-major ``[R, N]``; the reference's ``[N, R]`` views are exposed
as transposes (``rcvIDi``, ``wghtVali``, ``distRcvi``).  There is no CPU
fallback: without a CUDA device or the built library the constructor raises.
"""
import ctypes
import os

import numpy as np

from . import _lib
from .mesh import FVMesh

_L = None


def _lib_handle():
    global _L
    if _L is None:
        _L = _lib.load()
    return _L


class Model:
    """One landscape on one GPU.

    Build from a goSPL YAML input (``Model("input.yml")``, the subset of keys
    read by inputparser.py for this path) or from arrays
    (``Model(coords=..., cells=..., elev=..., params=...)``).  ``params`` keys:
    dt, tStart, tEnd, flowDir, K (scalar or per-vertex), d, m, G, Cda, Cdm, oFill,
    sealevel, bc, rain (per-vertex m/yr), upsub (per-vertex m/yr or None),
    nodep (default True: no continental deposition), nlPitVolume (1e9 m3),
    nlPitDepth (100 m), and for the lake deposits of large deep depressions
    marineSolver ("picard" builds them; goSPL's default "ts" is refused when
    they occur), nlPitK (10), pitInletBias (0.5), picardSub (10), picardIts (2).
    ``members`` = (start, maxarea) declares the mesh a disjoint union of
    landscapes (``gospl_b200.ensemble``).  ``precision=32`` selects the FP32
    sweeps and CG with FP64 refinement to ``refine_tol``.

    Outputs (goSPL's ``output`` and ``time`` keys): ``outputDir`` (None: no
    files; a YAML input defaults to "output"), ``makedir`` (False),
    ``compression`` ("gzip", a level 0-9 or "none"), ``tout`` (tEnd - tStart)
    and ``rStep`` (restart from that output step, 0: a new run).
    """

    def __init__(self, filename=None, *, coords=None, cells=None, elev=None, params=None, mesh=None,
                 device="cuda", init_flow=True, cg_rtol=1.0e-13, cg_maxit=2000, members=None, precision=64,
                 refine_tol=1.0e-10):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("gospl_b200.Model needs a CUDA device")
        self.torch = torch
        L = _lib_handle()
        if filename is not None:
            from .inputparser import read_input
            coords, cells, elev, params = read_input(filename)
        if mesh is None:
            mesh = FVMesh(coords, cells, params.get("bc", "oooo"))
        self.mesh = mesh
        self.mesh_coords = coords
        self.mesh_cells = cells
        self.dev = torch.device(device)
        if self.dev.type == "cuda" and self.dev.index is None:
            self.dev = torch.device("cuda", torch.cuda.current_device())
        self.lpoints = mesh.n
        n = mesh.n
        p = dict(params)
        self.dt = float(p["dt"])
        self.tStart = float(p.get("tStart", 0.0))
        self.tEnd = float(p["tEnd"])
        self.tNow = self.tStart
        self.flowDir = int(p.get("flowDir", 8))
        self.flowExp = 1.1
        self.coeffd = float(p.get("d", 0.0))
        self.spl_m = float(p.get("m", 0.5))
        self.Cda = float(p.get("Cda", 0.0))
        self.Cdm = float(p.get("Cdm", 0.0))
        self.oFill = float(p.get("oFill", -6000.0))
        self.sealevel = float(p.get("sealevel", 0.0))
        self.flatModel = bool(mesh.flat)
        self.nodep = bool(p.get("nodep", True))
        # marine deposition (seaChange) after the continental one; goSPL's
        # default is on (inputparser.py:289), built for Gmar = 0 and the
        # Picard marine solver
        self.seadepo = (not self.nodep) and bool(p.get("seadepo", False))
        self.nlK = float(p.get("nonlinKm", 10.0))                   # inputparser.py:554
        self.clinSlp = max(1.0e-6, float(p.get("clinSlp", 1.0e-6)))   # :555, 592
        self.Gmar = float(p.get("Gmar", 0.0))                      # :557
        self.offshore = float(p.get("offshore", 100.0e5))          # :558
        self.nl_pit_volume = float(p.get("nlPitVolume", 1.0e9))    # inputparser.py:562,584
        self.nl_pit_depth = float(p.get("nlPitDepth", 100.0))      # inputparser.py:563,585
        # lake deposits of large deep depressions: marineSolver picard
        # (inputparser.py:564-580); goSPL's default adaptive TS is not built
        self.marineSolver = str(p.get("marineSolver", "ts")).lower()
        if self.seadepo and self.marineSolver != "picard":
            raise NotImplementedError("marine deposition is built for marineSolver picard (goSPL's adaptive TS "
                                      "solve is not)")
        self.nl_pit_K = float(p.get("nlPitK", p.get("nonlinKm", 10.0)))
        self.nl_pit_inlet_bias = min(1.0, max(0.0, float(p.get("pitInletBias", 0.5))))
        self.picardSub = int(p.get("picardSub", 10))
        self.picardIts = int(p.get("picardIts", 2))
        self.cg_rtol = cg_rtol
        self.cg_maxit = cg_maxit
        self.stats = {}
        self._hill_ran = False
        self.output = None

        f64 = dict(dtype=torch.float64, device=self.dev)
        i32 = dict(dtype=torch.int32, device=self.dev)
        u8 = dict(dtype=torch.uint8, device=self.dev)
        K = p["K"]
        if np.ndim(K) == 0:
            self.K = float(K)
            self.Kfield = None
        else:
            self.K = 0.0
            self.Kfield = torch.as_tensor(np.asarray(K, np.float64), **f64)
        self.rainMesh = torch.as_tensor(np.asarray(p["rain"], np.float64), **f64)
        up = p.get("upsub")
        self.upsub = None if up is None else torch.as_tensor(np.asarray(up, np.float64), **f64)

        R = self.flowDir
        self.hGlobal = torch.as_tensor(np.asarray(elev, np.float64), **f64).clone()
        self.cumED = torch.zeros(n, **f64)
        self.EbLocal = torch.zeros(n, **f64)
        self.FAL = torch.zeros(n, **f64)
        self.fillFAL = torch.zeros(n, **f64)
        self.waterFilled = torch.zeros(n, **f64)
        self.lFill = torch.zeros(n, **f64)
        self.bL = torch.zeros(n, **f64)
        self.pitIDs = torch.zeros(n, **i32)
        self.flatDirs = torch.zeros(n, **i32)
        self.rcv_i = torch.zeros((R, n), **i32)
        self.dist_i = torch.zeros((R, n), **f64)
        self.wgt_i = torch.zeros((R, n), **f64)
        self.lsink_mask = torch.zeros(n, **u8)
        self.sea_mask = torch.zeros(n, **u8)
        self.vSed = torch.zeros(n, **f64)
        self.rcv_live = None                     # live receivers of _buildFlowDirection
        self.xyz = None
        if not self.nodep:
            if coords is None:
                raise ValueError("continental deposition needs the vertex coordinates")
            xyz = np.zeros((n, 3))
            c = np.asarray(coords, np.float64)
            xyz[:, :c.shape[1]] = c
            self.xyz = torch.as_tensor(xyz, **f64)
        self.edges = None
        if self.seadepo:
            # the mesh's unique edges for the coastline contour, and the
            # vertices' bounding box (lo, span)
            cl = np.asarray(cells, np.int64)
            e = np.sort(np.concatenate([cl[:, [0, 1]], cl[:, [1, 2]], cl[:, [2, 0]]]), axis=1)
            e = np.unique(e, axis=0)
            self.edges = torch.as_tensor(np.ascontiguousarray(e, np.int32), device=self.dev)
            lo = xyz.min(axis=0)
            span = np.maximum(xyz.max(axis=0) - lo, 1.0)
            self.xyz_box = np.ascontiguousarray(np.concatenate([lo, span]), np.float64)

        handle = ctypes.c_void_p()
        outlet = np.ascontiguousarray(mesh.outlet, np.int32)
        opn = np.ascontiguousarray(mesh.open_nodes, np.int32)
        nnb = np.ascontiguousarray(mesh.nnb, np.int32)
        ngb = np.ascontiguousarray(mesh.ngb, np.int32)
        elgt = np.ascontiguousarray(mesh.elgt, np.float64)
        vd = np.ascontiguousarray(mesh.vdist, np.float64)
        fa = np.ascontiguousarray(mesh.farea, np.float64)
        la = np.ascontiguousarray(mesh.larea, np.float64)
        torch.cuda.set_device(self.dev)
        _lib.check(L.gs_plan_create(n, _lib.ptr(nnb), _lib.ptr(ngb), _lib.ptr(elgt), _lib.ptr(vd),
                                    _lib.ptr(fa), _lib.ptr(la), _lib.ptr(outlet), len(outlet),
                                    _lib.ptr(opn), len(opn), int(self.flatModel), R, ctypes.byref(handle)))
        self._plan = handle
        self.stream = torch.cuda.current_stream(self.dev)
        _lib.check(L.gs_plan_set_stream(self._plan, ctypes.c_void_p(self.stream.cuda_stream)))
        if not self.nodep and self.marineSolver == "picard":
            _lib.check(L.gs_plan_set_lake_diffusion(self._plan, self.nl_pit_K, self.nl_pit_inlet_bias,
                                                     self.picardSub, self.picardIts))
        self.fDepa = float(p.get("G", 0.0))
        if self.fDepa > 0.0:
            # transport-limited SPL (SPL.py:116-258, 305-336)
            _lib.check(L.gs_plan_set_deposition(self._plan, self.fDepa))
        if precision != 64:
            # FP32 sweeps and CG inside FP64 refinement to refine_tol
            _lib.check(L.gs_plan_set_precision(self._plan, int(precision), float(refine_tol)))
        if members is not None:
            # (start [nmem+1], maxarea [nmem]): landscapes packed in this mesh
            start = np.ascontiguousarray(members[0], np.int64)
            marea = np.ascontiguousarray(members[1], np.float64)
            _lib.check(L.gs_plan_set_members(self._plan, len(marea), _lib.ptr(start), _lib.ptr(marea)))
        out_dir = p.get("outputDir")
        self.rStep = int(p.get("rStep", 0))
        if out_dir is not None:
            if cells is None or coords is None:
                raise ValueError("outputs need the mesh coordinates and cells")
            from .outmesh import WriteMesh
            # WriteMesh.__init__ (outmesh.py:31-87) runs before the forcing
            self.output = WriteMesh(self, out_dir, bool(p.get("makedir", False)), p.get("compression", "gzip"),
                                    p.get("tout"), self.rStep, p.get("finput"))
        elif self.rStep > 0:
            raise ValueError("a restart (rStep > 0) needs the output directory it reads")
        self.applyForces()
        if self.rStep > 0:
            self.readData()   # model.py:289-291
        if init_flow:
            self.flowAccumulation()

    # ------------------------------------------------------------- views
    @property
    def rcvIDi(self):
        return self.rcv_i.t()

    @property
    def wghtVali(self):
        return self.wgt_i.t()

    @property
    def distRcvi(self):
        return self.dist_i.t()

    @property
    def lsink(self):
        return self.lsink_mask.bool()

    @property
    def seaID(self):
        return self.sea_mask.bool()

    @property
    def h(self):
        return self.hGlobal

    def launches(self):
        return int(_lib_handle().gs_plan_launches(self._plan))

    # ------------------------------------------------------------- stages
    def applyForces(self):
        """unstructuredmesh.py:743-794 (constant sea level, uniform-in-time rain)."""
        L = _lib_handle()
        _lib.check(L.gs_apply_forces(self._plan, _lib.ptr(self.hGlobal), _lib.ptr(self.rainMesh),
                                     _lib.ptr(self.upsub), self.dt, self.sealevel, _lib.ptr(self.bL)))
        self.rainVal = self.rainMesh.clamp(min=0.0)   # unstructuredmesh.py:960

    def fillElevation(self, sed=False):
        """pitfilling.py:849-903: lFill, pitIDs and flatDirs of the current
        elevation, per-pit tables read with pit_tables().  sed=True is the
        sediment fill (marine depressions filled too, pits labelled above the
        fill level, volumes on the unclipped surface), which sedChange also
        runs itself."""
        L = _lib_handle()
        npits = ctypes.c_int32()
        _lib.check(L.gs_fill_elevation(self._plan, _lib.ptr(self.hGlobal), self.sealevel, self.oFill, int(bool(sed)),
                                       _lib.ptr(self.lFill), _lib.ptr(self.pitIDs), _lib.ptr(self.flatDirs),
                                       ctypes.byref(npits)))
        self.npits = int(npits.value)

    def pit_tables(self):
        """(pitParams [P+1,3], pitInfo [P+1,2], filled_lvl [P+1,5], filled_vol [P+1,5])."""
        t = self.torch
        np1 = self.npits + 1
        pp = t.zeros((np1, 3), dtype=t.float64, device=self.dev)
        pi = t.zeros((np1, 2), dtype=t.int32, device=self.dev)
        fl = t.zeros((np1, 5), dtype=t.float64, device=self.dev)
        fv = t.zeros((np1, 5), dtype=t.float64, device=self.dev)
        _lib.check(_lib_handle().gs_pit_tables(self._plan, _lib.ptr(pp), _lib.ptr(pi), _lib.ptr(fl),
                                               _lib.ptr(fv)))
        return pp, pi, fl, fv

    def _buildFlowDirection(self, h, down=True):
        """FAMesh._buildFlowDirection (flowplex.py:480-544): the flow graph
        of the surface h.  Sets the live receivers rcvID, distRcv, wghtVal
        (views [N, R] of [R, N] storage), lsink and seaID on the model: MFD
        receivers of h, with down=True the pit-flat routing over the last
        fill (lFill, pitIDs, flatDirs), flat-model outlets as self-sinks."""
        t = self.torch
        R, n = self.flowDir, self.lpoints
        if self.rcv_live is None:
            self.rcv_live = t.empty((R, n), dtype=t.int32, device=self.dev)
            self.dist_live = t.empty((R, n), dtype=t.float64, device=self.dev)
            self.wgt_live = t.empty((R, n), dtype=t.float64, device=self.dev)
        h = t.as_tensor(h, dtype=t.float64, device=self.dev).contiguous()
        _lib.check(_lib_handle().gs_build_flow_direction(
            self._plan, _lib.ptr(h), int(bool(down)), self.sealevel, _lib.ptr(self.lFill), _lib.ptr(self.pitIDs),
            _lib.ptr(self.flatDirs), _lib.ptr(self.rcv_live), _lib.ptr(self.dist_live), _lib.ptr(self.wgt_live),
            _lib.ptr(self.lsink_mask), _lib.ptr(self.sea_mask)))

    @property
    def rcvID(self):
        return self.rcv_live.t()

    @property
    def wghtVal(self):
        return self.wgt_live.t()

    @property
    def distRcv(self):
        return self.dist_live.t()

    def flowAccumulation(self):
        L = _lib_handle()
        st = _lib.GsStats()
        _lib.check(L.gs_flow_accumulation(
            self._plan, _lib.ptr(self.hGlobal), _lib.ptr(self.bL), self.sealevel, self.oFill, self.dt,
            _lib.ptr(self.FAL), _lib.ptr(self.fillFAL), _lib.ptr(self.waterFilled), _lib.ptr(self.lFill),
            _lib.ptr(self.pitIDs), _lib.ptr(self.flatDirs), _lib.ptr(self.rcv_i), _lib.ptr(self.dist_i),
            _lib.ptr(self.wgt_i), _lib.ptr(self.lsink_mask), _lib.ptr(self.sea_mask), ctypes.byref(st)))
        self.npits = st.npits
        self.stats["flow"] = st.as_dict()

    def erodepSPL(self):
        L = _lib_handle()
        st = _lib.GsStats()
        _lib.check(L.gs_erodep_spl(
            self._plan, _lib.ptr(self.hGlobal), _lib.ptr(self.cumED), _lib.ptr(self.EbLocal),
            _lib.ptr(self.FAL), _lib.ptr(self.rainVal), self.K, _lib.ptr(self.Kfield), self.coeffd,
            self.spl_m, self.dt, _lib.ptr(self.rcv_i), _lib.ptr(self.dist_i), _lib.ptr(self.wgt_i),
            _lib.ptr(self.lsink_mask), _lib.ptr(self.sea_mask), ctypes.byref(st)))
        self.stats["spl"] = st.as_dict()

    def sedChange(self):
        """SEDMesh.sedChange (sedplex.py:1061-1086): sediment flux over the
        snapshot receivers of the last flowAccumulation, depressions filled
        with sediment, the cascade of overflowing depressions and the lake
        deposits.  vSed holds the routed sediment flux (m3/yr)."""
        if self.xyz is None:
            raise RuntimeError("sedChange needs a Model built with nodep=False")
        L = _lib_handle()
        st = _lib.GsStats()
        _lib.check(L.gs_sed_change(
            self._plan, _lib.ptr(self.hGlobal), _lib.ptr(self.cumED), _lib.ptr(self.EbLocal), _lib.ptr(self.xyz),
            self.sealevel, self.oFill, self.dt, self.nl_pit_volume, self.nl_pit_depth, _lib.ptr(self.lFill),
            _lib.ptr(self.pitIDs), _lib.ptr(self.flatDirs), _lib.ptr(self.rcv_i), _lib.ptr(self.wgt_i),
            _lib.ptr(self.lsink_mask), _lib.ptr(self.sea_mask), _lib.ptr(self.vSed), ctypes.byref(st)))
        self.npits = st.npits
        self.stats["sed"] = st.as_dict()

    def seaChange(self):
        """SEAMesh.seaChange (seaplex.py:738-861): the sediment flux that
        reached the sea after sedChange is spread down the marine receivers
        within the clinoform capacity and smoothed by the Picard diffusion
        over the sea cells (gs_sea_change)."""
        if self.edges is None:
            raise RuntimeError("seaChange needs a Model built with nodep=False and seadepo=True")
        L = _lib_handle()
        st = _lib.GsStats()
        _lib.check(L.gs_sea_change(
            self._plan, _lib.ptr(self.hGlobal), _lib.ptr(self.cumED), _lib.ptr(self.EbLocal), _lib.ptr(self.xyz),
            self.xyz_box.ctypes.data_as(ctypes.c_void_p), _lib.ptr(self.edges), int(self.edges.shape[0]),
            self.sealevel, self.oFill, self.dt, self.clinSlp, self.offshore, self.nlK, self.Gmar,
            _lib.ptr(self.lFill), _lib.ptr(self.vSed), _lib.ptr(self.sea_mask), ctypes.byref(st)))
        self.stats["sea"] = {"coast_points": st.npits, "marine_passes": st.cascade_passes,
                             "epsfill_passes": st.fill_rounds, "smoothing_cg_iters": st.flat_rounds,
                             "coupled_applies": st.cg_iters}

    def sed_budget(self):
        """Sediment budget of the last sedChange (m3 over the step): where
        the volume eroded by the step's SPL went in the continental routing
        (gs_sed_budget: depressions, closed-domain sinks, outlets, sea, and
        what goSPL's routing rules drop), plus `closure`, the eroded volume
        minus every destination, which must vanish to rounding."""
        L = _lib_handle()
        out = np.zeros(16)
        _lib.check(L.gs_sed_budget(self._plan, out.ctypes.data_as(ctypes.c_void_p)))
        b = {k: float(out[i]) for i, k in enumerate(_lib.LED_SLOTS)}
        b["unplaced"] = b["excess"] - b["placed"]
        b["unrouted"] = b["placed"] - b["routed"]
        b["closure"] = b["eroded"] - (b["retained"] + b["kept"] + b["dropped"] + b["outlets"] + b["sea"]
                                      + b["zero_excess"] + b["unplaced"] + b["unrouted"])
        return b

    def getHillslope(self):
        L = _lib_handle()
        st = _lib.GsStats()
        _lib.check(L.gs_hillslope(self._plan, _lib.ptr(self.hGlobal), _lib.ptr(self.cumED),
                                  _lib.ptr(self.EbLocal), self.sealevel, self.Cda, self.Cdm, self.dt,
                                  self.cg_rtol, self.cg_maxit, ctypes.byref(st)))
        self.stats["hillslope"] = st.as_dict()
        self._hill_ran = True

    def step(self):
        """One physics step of runProcesses (model.py:347-453, fast=False):
        flow, erosion, continental deposition unless nodep (flow again, then
        sedChange), hillslope, forcing."""
        self.flowAccumulation()
        self.erodepSPL()
        if not self.nodep:
            self.flowAccumulation()
            self.sedChange()
            if self.seadepo:
                self.seaChange()
        self.getHillslope()
        if self.tNow < self.tEnd:
            self.applyForces()
        self.tNow += self.dt

    def runProcesses(self):
        """model.py:331-466: output, then a step, until tEnd; the run ends
        with every output on disk."""
        try:
            while self.tNow <= self.tEnd:
                self.visModel()
                if self.tNow == self.tEnd:
                    break
                self.step()
        finally:
            if self.output is not None:
                self.output.flush()

    # ------------------------------------------------------------- outputs
    def visModel(self):
        """WriteMesh.visModel (outmesh.py:89-103); a no-op without outputDir."""
        if self.output is not None:
            self.output.visModel()

    def readData(self):
        """WriteMesh.readData (outmesh.py:505-620): restart state from the
        output files."""
        if self.output is None:
            raise ValueError("readData needs the output directory")
        self.output.readData()

    # ------------------------------------------------------------- adjoint
    def record(self, nslots):
        """Allocate `nslots` per-step records for the adjoint (0 frees them)."""
        if nslots and not self.nodep:
            raise NotImplementedError("the adjoint covers steps without continental deposition (nodep)")
        _lib.check(_lib_handle().gs_plan_record(self._plan, int(nslots)))

    def record_slot(self, slot):
        """Record the next step into `slot` (-1: stop recording)."""
        _lib.check(_lib_handle().gs_plan_record_slot(self._plan, int(slot)))

    def adjoint_step(self, slot, lam, grad_k=None, grad_u=None, grad_rain=None, grad_bl=None, rtol=1.0e-13,
                     maxit=2000):
        """Reverse the step recorded in `slot`: lam (dJ/dh after it) becomes
        dJ/dh before it; parameter gradients are accumulated (grad_bl written)."""
        _lib.check(_lib_handle().gs_adjoint_step(
            self._plan, int(slot), _lib.ptr(lam), _lib.ptr(self.rainVal), self.K, _lib.ptr(self.Kfield),
            self.coeffd, self.spl_m, self.dt, self.sealevel, self.Cda, self.Cdm, rtol, maxit, _lib.ptr(grad_k),
            _lib.ptr(grad_u), _lib.ptr(grad_rain), _lib.ptr(grad_bl)))

    def destroy(self):
        if getattr(self, "output", None) is not None:
            self.output.close()
            self.output = None
        if getattr(self, "_plan", None) is not None:
            self.torch.cuda.synchronize(self.dev)
            _lib_handle().gs_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
