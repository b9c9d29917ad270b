"""Generate tests/golden/output_planar2k.npz from the reference's own output code.

Run where a goSPL checkout is available, named by --ref or the GOSPL_REF
environment variable (no default):

    python tests/golden/make_output_golden.py --ref /path/to/gospl

It runs the reference's one-rank orchestration (refharness.py) with goSPL's
``WriteMesh`` (``gospl/tools/outmesh.py``) mixed in, over the runProcesses
loop of ``gospl/model.py:331-466`` (output at the start time and after every
step, ``tout = dt``), with an in-memory stand-in for ``h5py`` that keeps every
dataset the reference creates (float32 / int32 arrays, cast by numpy exactly
as the HDF5 library converts float64 to float32: round to nearest).  The
fixture holds, per output step, the float64 state the datasets were made from,
the land/sea mask in force, every dataset, the XMF text and the XDMF text.
"""
import importlib
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

REF = os.environ.get("GOSPL_REF")


def _take_ref_argument():
    """--ref PATH on the command line overrides GOSPL_REF; one of them must
    name the goSPL checkout."""
    global REF
    if "--ref" in sys.argv:
        k = sys.argv.index("--ref")
        REF = sys.argv[k + 1]
        del sys.argv[k:k + 2]
    if not REF:
        sys.exit("name the goSPL checkout with --ref PATH or the GOSPL_REF environment variable")
NSTEPS = 3


class _FakeH5File:
    files = {}

    def __init__(self, path, mode="r"):
        self.path = path
        self.d = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        _FakeH5File.files[self.path] = self.d

    def create_dataset(self, name, shape=None, dtype=None, **opts):
        self.d[name] = np.zeros(shape, dtype)
        return self.d[name]

    def __getitem__(self, name):
        return self.d[name.lstrip("/")]


def main():
    import refharness as RH
    from gospl_b200 import synthetic as S
    from oracle import mesh as OM

    RefModel = RH.make_model_class(REF)
    h5 = types.ModuleType("h5py")
    h5.File = _FakeH5File
    sys.modules["h5py"] = h5
    outmesh = importlib.import_module("gospl.tools.outmesh")
    WriteMesh = outmesh.WriteMesh

    c, f, z, rain, up, p = S.planar_config(n=2000, side=30.0e3, seed=7)
    # sea level at the 15th percentile of the initial elevation, so that the
    # outputs carry the sea edits of FA and fillFA
    p = dict(p, rain=rain, upsub=up, tEnd=NSTEPS * p["dt"], nodep=False, sealevel=float(np.percentile(z, 15)))
    cells = np.asarray(f, np.int32)
    mesh = OM.build_mesh(c, cells, p["bc"])

    class OutModel(RefModel, WriteMesh):
        pass

    work = tempfile.mkdtemp()
    cwd = os.getcwd()
    os.chdir(work)
    try:
        finput = os.path.join(work, "input.yml")
        with open(finput, "w") as fh:
            fh.write("name: output fixture\n")
        m = OutModel.__new__(OutModel)
        RefModel.__init__(m, mesh, z, p)
        # WriteMesh state (inputparser.py:77-78, 2096-2117; model.py:179-300)
        m.tStart = 0.0
        m.tout = float(p["dt"])
        m.rStep = 0
        m.saveTime = m.tStart
        m.tNow = m.tStart
        m.outputDir = "output"
        m.makedir = False
        m.outCompress = "gzip"
        m.finput = finput
        m.strataFile = None
        m.strat = 0
        m.stratNb = 0
        m.fast = False
        m.evapdata = None
        m.cumEDLocal = m.cumED
        m.lcells = cells.astype(np.int64)
        m.lcoords = np.asarray(c, np.float64).reshape(-1, 3)
        WriteMesh.__init__(m)
        states = []

        def capture():
            sea = np.zeros(len(z), np.uint8)
            sea[np.asarray(m.seaID, np.int64)] = 1
            states.append(dict(h=m.hLocal.getArray().copy(), cumED=m.cumED.getArray().copy(),
                               Eb=m.EbLocal.getArray().copy(), waterFilled=np.array(m.waterFilled, copy=True),
                               fillFAL=m.fillFAL.getArray().copy(), FAL=m.FAL.getArray().copy(),
                               vSed=m.vSedLocal.getArray().copy(), sea=sea))

        # runProcesses (model.py:347-453) with the harness step
        while m.tNow <= m.tEnd:
            if m.saveTime == m.tStart or m.tNow >= m.saveTime:
                capture()
            m.visModel()
            if m.tNow == m.tEnd:
                break
            RefModel.step(m)   # WriteMesh keeps its output counter in m.step
        arrs = dict(v=c, c=cells, z=z, rain=p["rain"], upsub=p["upsub"], nsteps=np.array(NSTEPS))
        for k in ("dt", "tEnd", "flowDir", "K", "d", "m", "Cda", "Cdm", "sealevel"):
            arrs["p_" + k] = np.array(p[k])
        arrs["p_bc"] = np.array(p["bc"])
        arrs["p_nodep"] = np.array(False)
        out = os.path.join(work, "output")
        files = _FakeH5File.files
        topo = files[os.path.join(out, "h5", "topology.p0.h5")]
        arrs["topo_coords"] = topo["coords"]
        arrs["topo_cells"] = topo["cells"]
        for s, st in enumerate(states):
            for k, v in st.items():
                arrs["s%d_%s" % (s, k)] = v
            d = files[os.path.join(out, "h5", "gospl.%d.p0.h5" % s)]
            arrs["s%d_names" % s] = np.array(sorted(d))
            for k, v in d.items():
                arrs["s%d_ds_%s" % (s, k)] = v
            with open(os.path.join(out, "xmf", "gospl%d.xmf" % s)) as fh:
                arrs["s%d_xmf" % s] = np.array(fh.read())
        with open(os.path.join(out, "gospl.xdmf")) as fh:
            arrs["xdmf"] = np.array(fh.read())
        arrs["noutputs"] = np.array(len(states))
        arrs["save_times"] = np.array([float(p["dt"]) * s for s in range(len(states))])
    finally:
        os.chdir(cwd)
    path = os.path.join(HERE, "output_planar2k.npz")
    np.savez_compressed(path, **arrs)
    print("wrote", path, os.path.getsize(path) // 1024, "KB;", len(states), "outputs;",
          "datasets", list(arrs["s0_names"]))


if __name__ == "__main__":
    _take_ref_argument()
    main()
