"""Run goSPL's own Python orchestration of the hot path on one rank.

This is fixture-generation infrastructure: it imports the reference modules
``gospl/flow/flowplex.py``, ``gospl/flow/pitfilling.py``, ``gospl/eroder/SPL.py``
and ``gospl/sed/hillslope.py`` straight from a reference checkout, with
in-memory stand-ins for the pieces that cannot be installed here:

* ``petsc4py`` — numpy-backed ``Vec`` / scipy-backed ``Mat`` with the PETSc
  semantics these modules use (``axpy``, ``waxpy``, ``transpose``,
  ``setValuesLocalCSR`` ...), an identity ``DM`` (one rank: local == global),
  and a ``KSP`` whose ``solve`` returns the exact solution of the assembled
  system (sparse triangular sweep when the matrix is triangular up to a
  permutation, sparse LU otherwise);
* ``mpi4py`` — a one-rank communicator (reductions are identities);
* ``numpy_indexed`` — ``group_by`` with a stable key sort and ``reduceat``;
* ``gospl._fortran`` — the C restatement of the Fortran kernels
  (``oracle/fortran.py``), since no Fortran compiler is available.

The resulting outputs therefore pin the oracle's restatement of the Python
orchestration to the reference's actual Python code.  It reads the reference
tree only at fixture-generation time; nothing under ``tests/`` imports it.
"""
import importlib
import os
import sys
import types

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


# ---------------------------------------------------------------------------
# petsc4py stand-in
# ---------------------------------------------------------------------------
class Vec:
    def __init__(self, n_or_arr=0):
        if np.isscalar(n_or_arr):
            self.a = np.zeros(int(n_or_arr))
        else:
            self.a = np.array(n_or_arr, dtype=np.float64)

    def duplicate(self):
        return Vec(len(self.a))

    def getArray(self):
        return self.a

    @property
    def array(self):
        return self.a

    def setArray(self, x):
        self.a[:] = x

    def copy(self, result=None):
        if result is None:
            return Vec(self.a.copy())
        result.a[:] = self.a
        return result

    def set(self, v):
        self.a[:] = v

    def sum(self):
        return float(np.sum(self.a))

    def max(self):
        i = int(np.argmax(self.a))
        return i, float(self.a[i])

    def min(self):
        i = int(np.argmin(self.a))
        return i, float(self.a[i])

    def norm(self, *args):
        return float(np.linalg.norm(self.a))

    def axpy(self, alpha, x):
        self.a[:] = self.a + alpha * x.a

    def aypx(self, alpha, x):
        self.a[:] = x.a + alpha * self.a

    def waxpy(self, alpha, x, y):
        self.a[:] = alpha * x.a + y.a

    def pointwiseMult(self, x, y):
        self.a[:] = x.a * y.a

    def abs(self):
        self.a[:] = np.abs(self.a)

    def getSizes(self):
        return (len(self.a), len(self.a))

    def scale(self, alpha):
        self.a[:] = alpha * self.a

    # nested vectors (SPL.py _coupledEDSystem): one flat array, blocks by IS
    def createNest(self, vecs, comm=None):
        self.a = np.concatenate([v.a for v in vecs])
        return self

    def setUp(self):
        pass

    def getSubVector(self, iset):
        return Vec(self.a[iset.idx])

    def destroy(self):
        pass


class IS:
    def __init__(self, idx):
        self.idx = idx

    def destroy(self):
        pass


class Mat:
    n = None
    Option = types.SimpleNamespace(NEW_NONZERO_LOCATIONS=0)

    def __init__(self):
        self.A = None

    def create(self, comm=None):
        return self

    def setType(self, t):
        pass

    def setSizes(self, s):
        self.n = s[0][0]

    def setLGMap(self, *a):
        pass

    def setFromOptions(self):
        pass

    def setPreallocationNNZ(self, *a):
        pass

    def setOption(self, *a):
        pass

    def assemblyBegin(self):
        pass

    def assemblyEnd(self):
        pass

    def setValuesLocalCSR(self, indptr, indices, data, *a, **k):
        n = len(indptr) - 1
        self.A = sp.csr_matrix((np.asarray(data, dtype=np.float64).copy(),
                                np.asarray(indices).copy(), np.asarray(indptr).copy()), shape=(n, n))
        self.A.sum_duplicates()

    def axpy(self, alpha, X, *a):
        self.A = (self.A + X.A * alpha).tocsr()
        self.A.sum_duplicates()

    def copy(self):
        m = Mat()
        m.n = self.n
        m.A = self.A.copy()
        return m

    def transpose(self):
        self.A = self.A.T.tocsr()
        self.A.sort_indices()

    def mult(self, x, y):
        y.a[:] = self.A @ x.a

    # nested matrices (SPL.py _coupledEDSystem): assembled as one sparse block matrix
    def createNest(self, mats, comm=None):
        self.A = sp.bmat([[m.A for m in row] for row in mats], format="csr")
        self.blocks = [row[0].A.shape[0] for row in mats]
        self.n = self.A.shape[0]
        return self

    def getNestISs(self):
        off = np.concatenate([[0], np.cumsum(self.blocks)])
        iss = [IS(np.arange(off[k], off[k + 1])) for k in range(len(self.blocks))]
        return iss, iss

    def norm(self, *a):
        return float(spla.norm(self.A))

    def destroy(self):
        pass


def exact_solve(A, b):
    """Exact solution of A x = b: a dependency-ordered sweep when A is
    triangular up to a permutation (flow and SPL systems), else sparse LU."""
    A = A.tocsr()
    A.sort_indices()
    n = A.shape[0]
    indptr, indices, data = A.indptr, A.indices, A.data
    deps = [[] for _ in range(n)]
    cnt = np.zeros(n, dtype=np.int64)
    users = [[] for _ in range(n)]
    for i in range(n):
        for t in range(indptr[i], indptr[i + 1]):
            j = indices[t]
            if j != i and data[t] != 0.0:
                cnt[i] += 1
                users[j].append(i)
    order = [i for i in range(n) if cnt[i] == 0]
    head = 0
    x = np.zeros(n)
    while head < len(order):
        i = order[head]
        head += 1
        s = b[i]
        diag = None
        for t in range(indptr[i], indptr[i + 1]):
            j = indices[t]
            if j == i:
                diag = data[t]
            elif data[t] != 0.0:
                s = s - data[t] * x[j]
        x[i] = s / diag
        for u in users[i]:
            cnt[u] -= 1
            if cnt[u] == 0:
                order.append(u)
    if head < n:
        return spla.spsolve(A.tocsc(), b), False
    return x, True


class KSP:
    class ConvergedReason:
        CONVERGED_RTOL = 2

    Type = types.SimpleNamespace(TFQMR="tfqmr", RICHARDSON="richardson", CG="cg", GMRES="gmres",
                                 FGMRES="fgmres", PREONLY="preonly", BCGS="bcgs")

    def create(self, comm=None):
        return KSP()

    def setType(self, t):
        self.type = t

    def getPC(self):
        return PC()

    def setTolerances(self, *a, **k):
        pass

    def setInitialGuessNonzero(self, f):
        pass

    def setOptionsPrefix(self, p):
        self.prefix = p

    def setFromOptions(self):
        pass

    def setOperators(self, A, P=None):
        self.Aop = A

    def solve(self, b, x):
        A = self.Aop.A
        if getattr(self, "prefix", "") in ("hilllin_", "spl_ed_", "marpicard_"):
            x.a[:] = spla.spsolve(A.tocsc(), b.a)
        else:
            sol, _ = exact_solve(A, b.a)
            x.a[:] = sol

    def getConvergedReason(self):
        return 2

    def getIterationNumber(self):
        return 1

    def destroy(self):
        pass


class PC:
    def setType(self, t):
        pass

    def setFieldSplitIS(self, *fields):
        pass

    def getFieldSplitSubKSP(self):
        return [KSP(), KSP()]

    def destroy(self):
        pass

    def setReusePreconditioner(self, f):
        pass


class _Options(dict):
    def setValue(self, k, v):
        self[k] = v

    def hasName(self, k):
        return k in self


class _Comm:
    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1


class DM:
    def createMatrix(self):
        return Mat()

    def localToGlobal(self, l, g, *a):
        g.a[:] = l.a

    def globalToLocal(self, g, l, *a):
        l.a[:] = g.a


def _petsc_module():
    PETSc = types.SimpleNamespace()
    PETSc.COMM_WORLD = _Comm()
    PETSc.IntType = np.int32
    PETSc.Mat = Mat
    PETSc.Vec = Vec
    PETSc.KSP = KSP
    PETSc.Options = lambda _o=_Options(): _o
    PETSc.NormType = types.SimpleNamespace(FROBENIUS=3)
    PETSc.InsertMode = types.SimpleNamespace(ADD_VALUES=1, INSERT_VALUES=0)
    petsc4py = types.ModuleType("petsc4py")
    petsc4py.PETSc = PETSc
    petsc4py.init = lambda *a, **k: None
    return petsc4py


# ---------------------------------------------------------------------------
# mpi4py stand-in (one rank)
# ---------------------------------------------------------------------------
class _MPIComm:
    def Allreduce(self, sendbuf, recvbuf=None, op=None):
        if recvbuf is not None and sendbuf is not MPI_IN_PLACE:
            np.copyto(recvbuf, sendbuf)

    def allreduce(self, x, op=None):
        return x

    def Allgatherv(self, sendbuf, recv):
        if isinstance(sendbuf, (list, tuple)):
            sendbuf = sendbuf[0]
        sendbuf = np.asarray(sendbuf).ravel()
        recvbuf = recv[0]
        recvbuf[: len(sendbuf)] = sendbuf

    def Reduce(self, sendbuf, recvbuf, op=None, root=0):
        if recvbuf is not None:
            np.copyto(recvbuf, sendbuf)

    def bcast(self, x, root=0):
        return x

    def gather(self, x, root=0):
        return [x]

    def Barrier(self):
        pass

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1


MPI_IN_PLACE = object()


def _mpi_module():
    MPI = types.SimpleNamespace(COMM_WORLD=_MPIComm(), IN_PLACE=MPI_IN_PLACE, SUM="sum", MAX="max",
                                MIN="min", LOR="lor", DOUBLE="double", Wtime=lambda: 0.0)
    m = types.ModuleType("mpi4py")
    m.MPI = MPI
    return m


# ---------------------------------------------------------------------------
# numpy_indexed stand-in
# ---------------------------------------------------------------------------
class _GroupBy:
    def __init__(self, keys, values=None):
        keys = np.asarray(keys)
        self.sorter = np.argsort(keys, kind="mergesort")
        sk = keys[self.sorter]
        flag = np.concatenate(([True], sk[1:] != sk[:-1])) if sk.size else np.zeros(0, bool)
        self.start = np.flatnonzero(flag)
        self.unique = sk[self.start] if sk.size else sk

    def reduce(self, values, op=np.add):
        v = np.asarray(values)[self.sorter]
        if v.size == 0:
            return v
        return op.reduceat(v, self.start)

    def sum(self, values):
        return self.unique, self.reduce(values)

    def max(self, values):
        return self.unique, self.reduce(values, np.maximum)


def _npi_module():
    m = types.ModuleType("numpy_indexed")

    def group_by(keys, values=None):
        g = _GroupBy(keys)
        if values is None:
            return g
        v = np.asarray(values)[g.sorter]
        ends = list(g.start[1:]) + [len(v)]
        return g.unique, [v[s:e] for s, e in zip(g.start, ends)]

    m.group_by = group_by
    return m


# ---------------------------------------------------------------------------
# vtk stand-in: the unstructured grid and contour filter seaplex.py:88-135
# uses to extract the coastline
# ---------------------------------------------------------------------------
class _VtkArray:
    def __init__(self, a):
        self.a = np.array(a, copy=True)
        self.name = None

    def SetName(self, name):
        self.name = name


class _VtkPointData:
    def __init__(self):
        self.arrays = {}

    def AddArray(self, arr):
        self.arrays[arr.name] = arr


class _VtkPoints:
    def __init__(self, a=None):
        self.a = a

    def SetData(self, arr):
        self.a = arr.a

    def GetData(self):
        return _VtkArray(self.a)


class _VtkGrid:
    """vtkUnstructuredGrid of triangles: points, cells, named point data."""

    def __init__(self, points=None, cells=None):
        self.points = None if points is None else np.asarray(points, dtype=np.float64)
        self.cells = None if cells is None else np.asarray(cells, dtype=np.int64)
        self.pd = _VtkPointData()

    def GetPointData(self):
        return self.pd

    def SetFieldData(self, pd):
        self.pd = pd

    def SetPoints(self, pts):
        self.points = pts.a


class _VtkPolyOut:
    def __init__(self, pts):
        self.pts = pts

    def GetPoints(self):
        return None if self.pts is None else _VtkPoints(self.pts)


class _VtkContourFilter:
    """Marching triangles, one cell at a time as vtkTriangle::Contour does:
    a vertex is inside when its scalar is >= the value; each edge with one
    end inside gives the point interpolated from its lower-scalar end; a
    point locator merges identical points (first-insertion order)."""

    def SetInputData(self, grid):
        self.grid = grid

    def SetValue(self, i, v):
        self.value = float(v)

    def SetInputArrayToProcess(self, *a):
        self.name = a[-1]

    def GenerateTrianglesOff(self):
        pass

    def Update(self):
        g = self.grid
        s = g.pd.arrays[self.name].a
        x = g.points
        seen = {}
        pts = []
        for tri in g.cells:
            for v0, v1 in ((tri[0], tri[1]), (tri[1], tri[2]), (tri[2], tri[0])):
                if (s[v0] >= self.value) == (s[v1] >= self.value):
                    continue
                delta = s[v1] - s[v0]
                if delta > 0:
                    e1, e2 = v0, v1
                else:
                    e1, e2 = v1, v0
                    delta = -delta
                t = 0.0 if delta == 0.0 else (self.value - s[e1]) / delta
                p = tuple(float(x[e1, j] + t * (x[e2, j] - x[e1, j])) for j in range(3))
                if p not in seen:
                    seen[p] = len(pts)
                    pts.append(p)
        self.out = _VtkPolyOut(np.array(pts, dtype=np.float64) if pts else None)

    def GetOutput(self):
        return self.out


def _vtk_modules():
    vtk = types.ModuleType("vtk")
    vtk.vtkUnstructuredGrid = _VtkGrid
    vtk.vtkPoints = _VtkPoints
    vtk.vtkContourFilter = _VtkContourFilter
    vtk.VTK_TRIANGLE = 5
    vtk.vtkObject = types.SimpleNamespace(GlobalWarningDisplayOff=lambda: None)
    util = types.ModuleType("vtk.util")
    ns = types.ModuleType("vtk.util.numpy_support")
    ns.numpy_to_vtk = lambda a, deep=1, **k: _VtkArray(a)
    ns.vtk_to_numpy = lambda arr: np.asarray(arr.a)
    util.numpy_support = ns
    vtk.util = util
    return {"vtk": vtk, "vtk.util": util, "vtk.util.numpy_support": ns}


# ---------------------------------------------------------------------------
# module loading
# ---------------------------------------------------------------------------
def load_reference(refroot):
    """Import the four hot-path modules from `refroot` with the stand-ins."""
    from oracle import fortran as F

    sys.modules["petsc4py"] = _petsc_module()
    sys.modules["mpi4py"] = _mpi_module()
    sys.modules["numpy_indexed"] = _npi_module()
    sys.modules.update(_vtk_modules())
    fort = types.ModuleType("gospl._fortran")
    for name in ("mfdreceivers", "sethillslopecoeff", "edge_tile", "fill_tile", "fill_edges",
                 "fill_dir", "nghb_dir", "getpitvol", "pits_cons", "fill_depressions",
                 "graph_nodes", "combine_edges", "label_pits", "setmaxnb", "jacobiancoeff", "epsfill",
                 "mfdrcvrs"):
        setattr(fort, name, getattr(F, name))
    for name in ("sort_ids", "hillslp_nl", "fctcoeff"):
        setattr(fort, name, lambda *a, **k: (_ for _ in ()).throw(NotImplementedError(name)))
    gospl_dir = os.path.join(refroot, "gospl")
    for pkg in ("gospl", "gospl.flow", "gospl.eroder", "gospl.sed", "gospl.tools"):
        mod = types.ModuleType(pkg)
        sub = pkg.split(".")[1:]
        mod.__path__ = [os.path.join(gospl_dir, *sub)]
        sys.modules[pkg] = mod
    sys.modules["gospl._fortran"] = fort
    gc_mod = types.ModuleType("gospl.tools.petscgc")
    gc_mod.safe_garbage_cleanup = lambda *a, **k: None
    sys.modules["gospl.tools.petscgc"] = gc_mod
    flowplex = importlib.import_module("gospl.flow.flowplex")
    pitfilling = importlib.import_module("gospl.flow.pitfilling")
    SPLm = importlib.import_module("gospl.eroder.SPL")
    hill = importlib.import_module("gospl.sed.hillslope")
    sedplex = importlib.import_module("gospl.sed.sedplex")
    seaplex = importlib.import_module("gospl.sed.seaplex")
    return flowplex.FAMesh, pitfilling.PITFill, SPLm.SPL, hill.hillSLP, sedplex.SEDMesh, seaplex.SEAMesh


def load_meshfunc(refroot):
    import importlib.util
    path = os.path.join(refroot, "gospl", "mesher", "meshfunc.py")
    spec = importlib.util.spec_from_file_location("ref_meshfunc", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _NullProfiler:
    def start(self, *a):
        pass

    def stop(self, *a):
        pass


def make_model_class(refroot):
    FAMesh, PITFill, SPL, hillSLP, SEDMesh, SEAMesh = load_reference(refroot)

    class RefModel(FAMesh, PITFill, SPL, hillSLP, SEDMesh, SEAMesh):
        """One-rank goSPL model restricted to flowAccumulation / erodepSPL /
        getHillslope; forcing follows unstructuredmesh.py:743-972."""

        def __init__(self, mesh, elev, params):
            n = mesh["nb"]
            self.lpoints = self.mpoints = n
            self.verbose = False
            self.memclear = False
            self.profiler = _NullProfiler()
            self.dm = DM()
            self.hGlobal = Vec(elev)
            self.hLocal = Vec(elev)
            self.sizes = ((n, n), (n, n))
            self.lgmap_row = self.lgmap_col = None
            for name in ("tmp", "tmpL", "tmp1", "bG", "bL", "cumED", "cumEDLocal"):
                setattr(self, name, Vec(n))
            self.larea = mesh["larea"].copy()
            self.areaGlobal = Vec(self.larea)
            self.maxarea = np.array([mesh["maxarea"]])
            self.FVmesh_ngbID = mesh["ngb"].astype(np.int64)
            self.flatModel = mesh["flat"]
            self.outletIDs = mesh["outlet"]
            self.open_nodes = mesh["open_nodes"]
            self.idLBounds = np.zeros(0, dtype=np.int64)
            self.ghostIDs = np.zeros(0, dtype=np.int64)
            self.inIDs = np.ones(n, dtype=int)
            self.glIDs = np.arange(n)
            self.gid = np.arange(n, dtype=np.int32)
            self.locIDs = np.arange(n, dtype=np.int64)
            from oracle import fortran as F
            self.maxnb = F.setmaxnb(n)
            p = params
            self.dt = float(p["dt"])
            self.tNow = float(p.get("tStart", 0.0))
            self.tEnd = float(p["tEnd"])
            self.flowDir = int(p["flowDir"])
            self.flowExp = 1.1
            self.K = p["K"]
            self.coeffd = float(p.get("d", 0.0))
            self.fDepa = float(p.get("G", 0.0))
            self.spl_m = float(p.get("m", 0.5))
            self.spl_n = 1.0
            self.Cda = float(p["Cda"])
            self.Cdm = float(p["Cdm"])
            self.K_nl = 1.0
            self.K_sc = 0.0
            self.oFill = float(p.get("oFill", -6000.0))
            self.sealevel = float(p.get("sealevel", 0.0))
            self.rainMesh = np.asarray(p["rain"], dtype=np.float64)
            up = p.get("upsub")
            self.upsub = None if up is None else np.asarray(up, dtype=np.float64)
            self.cptSoil = False
            self.stratNb = 0
            self.stratK = None
            self.stratLith = False
            self.flexOn = False
            self.iceOn = False
            self.ice_till_on = False
            self.evapVal = None
            self.evapStream = False
            self.sedfacVal = None
            self.evapLoss = 0.0
            self.nodep = bool(p.get("nodep", True))
            self.provOn = False
            self.provNb = 0
            self.lcoords = np.asarray(mesh["coords"], dtype=np.float64).reshape(-1, 3)
            self.nl_pit_volume = float(p.get("nlPitVolume", 1.0e9))
            self.nl_pit_depth = float(p.get("nlPitDepth", 100.0))
            self.nl_pit_K = float(p.get("nlPitK", 10.0))
            self.nl_pit_inlet_bias = float(p.get("pitInletBias", 0.5))
            self.marineSolver = str(p.get("marineSolver", "ts"))
            self.picardSub = int(p.get("picardSub", 10))
            self.picardIts = int(p.get("picardIts", 2))
            # marine deposition (inputparser.py:289, 554-592)
            self.seaDepo = bool(p.get("seadepo", False))
            self.nlK = float(p.get("nonlinKm", 10.0))
            self.clinSlp = max(1.0e-6, float(p.get("clinSlp", 1.0e-6)))
            self.Gmar = float(p.get("Gmar", 0.0))
            self.offshore = float(p.get("offshore", 100.0e5))
            self.lcells = np.asarray(mesh["cells"], dtype=np.int64)
            self.vtkMesh = _VtkGrid(self.lcoords, self.lcells)
            FAMesh.__init__(self)
            PITFill.__init__(self)
            SPL.__init__(self)
            hillSLP.__init__(self)
            SEDMesh.__init__(self)
            SEAMesh.__init__(self)
            self.applyForces()
            self.flowAccumulation()

        def _surfaceK(self):
            return np.ones(self.lpoints)

        def _gatherGlobalOnRoot(self, local_full):
            return np.array(local_full, copy=True)

        def _surfaceLithoK(self):
            return np.ones(self.lpoints)

        # forcing: unstructuredmesh.py:743-794, 903-972 (uniform sea level)
        def applyForces(self):
            rain = self.rainMesh.copy()
            rain[rain < 0] = 0.0
            self.rainVal = rain
            self.bL.setArray(self.rainVal * self.larea)
            self.dm.localToGlobal(self.bL, self.bG)
            if self.upsub is not None:
                tmp = self.hLocal.getArray().copy()
                self.hLocal.setArray(tmp + self.upsub * self.dt)
                self.dm.localToGlobal(self.hLocal, self.hGlobal)
            if self.flatModel and len(self.open_nodes):
                from oracle.model import OracleModel
                tmp = self.hLocal.getArray().copy()
                tmp = OracleModel._drainOpenEdges(self, tmp)
                self.hLocal.setArray(tmp)
                self.dm.localToGlobal(self.hLocal, self.hGlobal)

        def step(self):
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

    return RefModel
