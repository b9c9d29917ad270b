"""Model outputs and restarts in goSPL's file layout.

goSPL's ``WriteMesh`` (``gospl/tools/outmesh.py``) writes, at the start time
and then every ``tout`` years:

* ``<dir>/h5/topology.p0.h5`` once: ``coords`` (float32 [n,3]) and ``cells``
  (int32 [m,3], 1-based) (``outmesh.py:228-249``);
* ``<dir>/h5/gospl.<step>.p0.h5``: ``elev``, ``erodep``, ``EDrate``,
  ``waterFill``, ``fillFA``, ``FA``, ``sedLoad``, ``uplift`` (with tectonics)
  and ``rain``, float32 [n,1] (``outmesh.py:252-478``);
* ``<dir>/xmf/gospl<step>.xmf`` and the time series ``<dir>/gospl.xdmf``
  (``outmesh.py:622-909``);

and a run restarted at output step ``rstep`` reads ``gospl.<rstep>.p0.h5``
back (``outmesh.py:505-620``).  This module writes the same files, with the
same names, datasets, dtypes, edits (discharge floor, sea vertices) and XDMF
text, for one rank (``p0``).

On the device a single kernel (``gs_output_fields``) packs the step's fields
into float32 rows of a staging buffer on the model's stream, so the next step
may start at once; a side stream copies the rows into pinned host memory and a
writer thread compresses (chunks in parallel) and writes the files.  Two
staging and host buffers alternate, so one output is written while the next
is packed.  ``flush()`` waits for every pending write; ``readData`` and the
end of ``runProcesses`` call it.
"""
import os
import shutil
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _lib
from . import hdf5

DISCHARGE_FLOOR = 1.0e-8            # gospl/tools/constants.py:51
FIELDS = ("elev", "erodep", "EDrate", "waterFill", "fillFA", "FA", "sedLoad", "uplift", "rain")


def compression_level(comp):
    """goSPL's ``output.compression`` (outmesh.py:38-55): "gzip" (default,
    level 4 as in h5py), an int 0-9, or none/False/None (uncompressed)."""
    if comp in (None, False, "none", "None", ""):
        return None
    if isinstance(comp, bool):
        return 4
    if isinstance(comp, (int, np.integer)):
        return int(comp)
    if str(comp).lower() == "gzip":
        return 4
    raise ValueError("output compression must be gzip, an integer level 0-9 or none; got %r" % (comp,))


def xmf_text(step, save_time, elems, nodes, sealevel, file="gospl", upsub=True, rain=True):
    """The per-step XMF file of WriteMesh._save_DMPlex_XMF (outmesh.py:622-867)
    for one rank, ``fast: False``, no ice, flexure, soil or dual lithology."""
    pfile = "h5/%s.%d.p0.h5" % (file, step)
    tfile = "h5/topology.p0.h5"
    out = ['<?xml version="1.0" encoding="UTF-8"?>\n', '<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd">\n',
           '<Xdmf Version="2.0" xmlns:xi="http://www.w3.org/2001/XInclude">\n', " <Domain>\n",
           '    <Grid GridType="Collection" CollectionType="Spatial">\n',
           '      <Time Type="Single" Value="%0.02f"/>\n' % save_time,
           '      <Grid Name="Block.0">\n',
           '         <Topology Type="Triangle" NumberOfElements="%d" BaseOffset="1">\n' % elems,
           '          <DataItem Format="HDF" DataType="Int" Dimensions="%d 3">%s:/cells</DataItem>\n' % (elems, tfile),
           "         </Topology>\n", '         <Geometry Type="XYZ">\n',
           '          <DataItem Format="HDF" NumberType="Float" Precision="4" Dimensions="%d 3">%s:/coords</DataItem>\n'
           % (nodes, tfile),
           "         </Geometry>\n"]

    def attr(name, ds):
        out.append('         <Attribute Type="Scalar" Center="Node" Name="%s">\n' % name)
        out.append('          <DataItem Format="HDF" NumberType="Float" Precision="4" Dimensions="%d 1">%s:/%s'
                   '</DataItem>\n' % (nodes, pfile, ds))
        out.append("         </Attribute>\n")

    attr("Z", "elev")
    attr("ED", "erodep")
    attr("waterFill", "waterFill")
    attr("EDrate", "EDrate")
    attr("FA", "FA")
    attr("fillFA", "fillFA")
    attr("SL", "sedLoad")
    if upsub:
        attr("vTec", "uplift")
    if rain:
        attr("Rain", "rain")
    out.append('         <Attribute Type="Scalar" Center="Node" Name="sea">\n')
    out.append('          <DataItem ItemType="Function" Function="$0 * 0.00000000000000001 + %f" Dimensions="%d 1">\n'
               % (sealevel, nodes))
    out.append('           <DataItem Format="HDF" NumberType="Float" Precision="4" Dimensions="%d 1">%s:/erodep'
               '</DataItem>\n' % (nodes, pfile))
    out.append("          </DataItem>\n")
    out.append("         </Attribute>\n")
    out.append("      </Grid>\n")
    out.append("    </Grid>\n")
    out.append(" </Domain>\n")
    out.append("</Xdmf>\n")
    return "".join(out)


def xdmf_text(last_step, file="gospl"):
    """The time series of WriteMesh._save_XDMF (outmesh.py:869-909)."""
    out = ['<?xml version="1.0" encoding="UTF-8"?>\n', '<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd">\n',
           '<Xdmf Version="2.0" xmlns:xi="http://www.w3.org/2001/XInclude">\n', " <Domain>\n",
           '    <Grid GridType="Collection" CollectionType="Temporal">\n']
    for s in range(last_step + 1):
        out.append('      <xi:include href="xmf/%s%d.xmf" xpointer="xpointer(//Xdmf/Domain/Grid)"/>\n' % (file, s))
    out += ["    </Grid>\n", " </Domain>\n", "</Xdmf>\n"]
    return "".join(out)


def make_output_dir(output_dir, makedir, rstep, finput=None):
    """WriteMesh._createOutputDir (outmesh.py:109-142): the directory (relative
    to the working directory unless absolute) with ``h5/`` and ``xmf/``; an
    existing one is removed, or with ``makedir`` the first free ``<dir>_<k>``
    is used; a restart (rstep > 0) reuses the directory as it is."""
    out = output_dir if os.path.isabs(output_dir) else os.path.join(os.getcwd(), output_dir)
    if rstep == 0:
        if makedir:
            if os.path.exists(out):
                k = 0
                while os.path.exists("%s_%d" % (out, k)):
                    k += 1
                out = "%s_%d" % (out, k)
        elif os.path.exists(out):
            shutil.rmtree(out, ignore_errors=True)
        os.makedirs(out)
        os.makedirs(os.path.join(out, "h5"))
        os.makedirs(os.path.join(out, "xmf"))
    if finput is not None:
        shutil.copy(finput, out)
    return out


class WriteMesh:
    """Output writer of one Model (the state of goSPL's WriteMesh mixin)."""

    def __init__(self, model, output_dir="output", makedir=False, compression="gzip", tout=None, rstep=0,
                 finput=None, file="gospl"):
        self.m = model
        self.file = file
        self.level = compression_level(compression)
        self.tout = float(tout if tout is not None else model.tEnd - model.tStart)
        if model.tStart + self.tout > model.tEnd:        # inputparser.py:413-429
            self.tout = model.tEnd - model.tStart
        if self.tout < model.dt:
            self.tout = model.dt
        self.rStep = int(rstep)
        self.outputDir = make_output_dir(output_dir, makedir, self.rStep, finput)
        # time bookkeeping (inputparser.py:77-78, outmesh.py:61-79)
        self.step = 0
        self.saveTime = model.tStart
        if self.rStep > 0:
            self.step = self.rStep + 1
            model.tNow = model.tStart + self.rStep * self.tout
            self.saveTime = model.tNow + self.tout
        self._pool = ThreadPoolExecutor(1)
        self._pending = []
        self._slot = 0
        self._stage = [None, None]
        self._host = [None, None]
        self._done = [None, None]     # futures of the writes that read each host buffer
        self._copied = [None, None]   # events: staging buffer i copied to the host
        self._side = None
        self.elems = int(np.asarray(model.mesh_cells).shape[0])
        self.nodes = model.lpoints

    # ----------------------------------------------------------- schedule
    def visModel(self):
        """outmesh.py:89-103: write at the start time and whenever tNow
        reaches the next output time."""
        m = self.m
        if self.saveTime == m.tStart:
            self._outputMesh()
            self.saveTime += self.tout
        elif m.tNow >= self.saveTime:
            self._outputMesh()
            self.saveTime += self.tout

    # ----------------------------------------------------------- writing
    def _buffers(self, i):
        t = self.m.torch
        n = self.m.lpoints
        if self._stage[i] is None:
            self._stage[i] = t.zeros((len(FIELDS), n), dtype=t.float32, device=self.m.dev)
            self._host[i] = t.zeros((len(FIELDS), n), dtype=t.float32, pin_memory=True)
        return self._stage[i], self._host[i]

    def _outputMesh(self):
        m = self.m
        t = m.torch
        if self._side is None:
            self._side = t.cuda.Stream(device=m.dev)
        i = self._slot
        self._slot ^= 1
        # the host buffer of slot i is free once its previous write finished,
        # the staging buffer once its previous copy finished
        if self._done[i] is not None:
            self._done[i].result()
        stage, host = self._buffers(i)
        if self._copied[i] is not None:
            m.stream.wait_event(self._copied[i])
        # seaID: the flow's mask before the first step (flowplex.py:493),
        # afterwards the mask of the last hillslope input (hillslope.py:620)
        sea = _lib.ptr(m.sea_mask) if not m._hill_ran else None
        _lib.check(_lib.load().gs_output_fields(
            m._plan, _lib.ptr(m.hGlobal), _lib.ptr(m.cumED), _lib.ptr(m.EbLocal), _lib.ptr(m.waterFilled),
            _lib.ptr(m.fillFAL), _lib.ptr(m.FAL), _lib.ptr(m.vSed), _lib.ptr(m.upsub), _lib.ptr(m.rainVal), sea,
            _lib.ptr(stage)))
        packed = t.cuda.Event()
        packed.record(m.stream)
        self._side.wait_event(packed)
        with t.cuda.stream(self._side):
            host.copy_(stage, non_blocking=True)
        copied = t.cuda.Event()
        copied.record(self._side)
        self._copied[i] = copied
        job = dict(step=self.step, save_time=self.saveTime, sealevel=m.sealevel, event=copied, host=host,
                   upsub=m.upsub is not None, rain=m.rainVal is not None,
                   topology=self._topology() if self.step == 0 else None)
        fut = self._pool.submit(self._write, job)
        self._done[i] = fut
        self._pending.append(fut)
        self.step += 1

    def _topology(self):
        m = self.m
        coords = np.zeros((m.lpoints, 3), np.float32)
        c = np.asarray(m.mesh_coords, np.float64)
        coords[:, :c.shape[1]] = c
        cells = (np.asarray(m.mesh_cells, np.int64) + 1).astype(np.int32)
        return coords, cells

    def _write(self, job):
        job["event"].synchronize()
        host = job["host"].numpy()
        h5 = os.path.join(self.outputDir, "h5")
        if job["topology"] is not None:
            coords, cells = job["topology"]
            hdf5.write(os.path.join(h5, "topology.p0.h5"), [("coords", coords), ("cells", cells)],
                       compression=self.level)
        names = list(FIELDS[:7]) + (["uplift"] if job["upsub"] else []) + (["rain"] if job["rain"] else [])
        data = [(nm, host[FIELDS.index(nm)].reshape(-1, 1)) for nm in names]
        hdf5.write(os.path.join(h5, "%s.%d.p0.h5" % (self.file, job["step"])), data, compression=self.level)
        with open(os.path.join(self.outputDir, "xmf", "%s%d.xmf" % (self.file, job["step"])), "w") as f:
            f.write(xmf_text(job["step"], job["save_time"], self.elems, self.nodes, job["sealevel"], self.file,
                             job["upsub"], job["rain"]))
        with open(os.path.join(self.outputDir, "%s.xdmf" % self.file), "w") as f:
            f.write(xdmf_text(job["step"], self.file))

    def flush(self):
        """Wait until every output scheduled so far is on disk (re-raises a
        writer error)."""
        pending, self._pending = self._pending, []
        for fut in pending:
            fut.result()

    def close(self):
        self.flush()
        self._pool.shutdown(wait=True)

    # ----------------------------------------------------------- restart
    def readData(self):
        """outmesh.py:505-562: the state of output step ``step - 1``
        (elevation, cumulative erosion/deposition, sediment load, rates and
        flow accumulations, float32 in the file) into the model."""
        self.flush()
        path = os.path.join(self.outputDir, "h5", "%s.%d.p0.h5" % (self.file, self.step - 1))
        if not os.path.exists(path):
            raise ValueError("Restart file is missing...")
        d = hdf5.read(path, ["elev", "erodep", "sedLoad", "EDrate", "FA", "fillFA"])
        m = self.m
        t = m.torch

        def put(dst, name):
            dst.copy_(t.as_tensor(d[name][:, 0].astype(np.float64), device=m.dev))

        put(m.hGlobal, "elev")
        put(m.cumED, "erodep")
        put(m.vSed, "sedLoad")
        put(m.EbLocal, "EDrate")
        put(m.FAL, "FA")
        put(m.fillFAL, "fillFA")
