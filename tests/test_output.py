"""Output files (gospl/tools/outmesh.py): the datasets and their edits against
the reference's own _outputMesh, the XMF and XDMF text, the output directory
rules."""
import os

import numpy as np
import pytest

from gospl_b200 import outmesh

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "output_planar2k.npz")


def test_oracle_output_fields_match_reference():
    """The oracle's restatement of _outputMesh (floors, sea edits, float32
    rounding) gives the reference's datasets bit for bit at every output."""
    from oracle.model import output_fields
    g = np.load(GOLDEN)
    for s in range(int(g["noutputs"])):
        st = {k: g["s%d_%s" % (s, k)] for k in ("h", "cumED", "Eb", "waterFilled", "fillFAL", "FAL", "vSed", "sea")}
        out = output_fields(st["h"], st["cumED"], st["Eb"], st["waterFilled"], st["fillFAL"], st["FAL"], st["vSed"],
                            g["upsub"], np.maximum(g["rain"], 0.0), st["sea"])
        assert sorted(out) == sorted(g["s%d_names" % s])
        for k, v in out.items():
            ref = g["s%d_ds_%s" % (s, k)]
            assert v.dtype == ref.dtype and v.shape == ref.shape, (s, k)
            assert np.array_equal(v, ref), (s, k)
    # the fixture exercises both edits
    assert g["s1_sea"].sum() > 0 and (g["s1_ds_FA"] == 1.0).sum() >= g["s1_sea"].sum()
    assert (g["s1_ds_FA"] == np.float32(1e-8)).sum() > 0


def test_xmf_and_xdmf_text_match_reference():
    g = np.load(GOLDEN)
    n = len(g["z"])
    m = len(g["c"])
    for s in range(int(g["noutputs"])):
        txt = outmesh.xmf_text(s, float(g["save_times"][s]), m, n, float(g["p_sealevel"]))
        assert txt == str(g["s%d_xmf" % s]), s
    assert outmesh.xdmf_text(int(g["noutputs"]) - 1) == str(g["xdmf"])
    # the topology: float32 coordinates, 1-based int32 cells
    assert np.array_equal(g["topo_coords"], np.asarray(g["v"], np.float32))
    assert np.array_equal(g["topo_cells"], (g["c"] + 1).astype(np.int32))


def test_output_directory_rules(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    finput = tmp_path / "in.yml"
    finput.write_text("x: 1\n")
    d = outmesh.make_output_dir("run", False, 0, str(finput))
    assert d == str(tmp_path / "run") and os.path.isdir(d + "/h5") and os.path.isdir(d + "/xmf")
    assert os.path.exists(d + "/in.yml")
    open(d + "/h5/old.h5", "w").close()
    assert outmesh.make_output_dir("run", False, 0) == d and not os.path.exists(d + "/h5/old.h5")   # removed
    assert outmesh.make_output_dir("run", True, 0) == d + "_0"
    assert outmesh.make_output_dir("run", True, 0) == d + "_1"
    open(d + "/h5/keep.h5", "w").close()
    assert outmesh.make_output_dir("run", False, 2) == d and os.path.exists(d + "/h5/keep.h5")        # restart


def test_compression_levels():
    assert outmesh.compression_level("gzip") == 4
    assert outmesh.compression_level(True) == 4
    assert outmesh.compression_level(7) == 7
    for off in (None, False, "none", "None", ""):
        assert outmesh.compression_level(off) is None
    with pytest.raises(ValueError):
        outmesh.compression_level("lzf")


class _FakeModel:
    def __init__(self, t0=0.0, t1=5000.0, dt=1000.0):
        self.tStart, self.tEnd, self.dt, self.tNow = t0, t1, dt, t0
        self.lpoints = 4
        self.mesh_cells = np.zeros((2, 3), np.int64)


def test_output_schedule_and_restart_bookkeeping(tmp_path, monkeypatch):
    """visModel writes at the start time and whenever tNow reaches the next
    output time (outmesh.py:89-103) inside runProcesses' loop (model.py:347-
    466); tout is clamped to [dt, tEnd - tStart]; a restart at output k
    resumes at tStart + k tout with output counter k + 1 (outmesh.py:61-79)."""
    written = []
    monkeypatch.setattr(outmesh.WriteMesh, "_outputMesh",
                        lambda self: (written.append((self.step, self.m.tNow)), setattr(self, "step", self.step + 1)))
    m = _FakeModel()
    w = outmesh.WriteMesh(m, str(tmp_path / "o"), tout=2000.0)
    while m.tNow <= m.tEnd:
        w.visModel()
        if m.tNow == m.tEnd:
            break
        m.tNow += m.dt
    assert written == [(0, 0.0), (1, 2000.0), (2, 4000.0)]
    assert outmesh.WriteMesh(_FakeModel(), str(tmp_path / "o"), tout=1.0e9).tout == 5000.0
    assert outmesh.WriteMesh(_FakeModel(), str(tmp_path / "o"), tout=10.0).tout == 1000.0
    m = _FakeModel()
    w = outmesh.WriteMesh(m, str(tmp_path / "o"), tout=2000.0, rstep=1)
    assert (m.tNow, w.step, w.saveTime) == (2000.0, 2, 4000.0)
    with pytest.raises(ValueError):
        w.readData()                      # no gospl.1.p0.h5 in the directory


def test_writer_files_carry_the_reference_datasets(tmp_path):
    """The writer thread's half of an output (host rows -> HDF5 + XMF + XDMF)
    given the reference's own float32 rows writes files whose datasets, XMF
    and XDMF are the reference's, and that pass the HDF5 structure checks."""
    import torch
    from gospl_b200 import hdf5
    from test_hdf5 import lint
    g = np.load(GOLDEN)
    n = len(g["z"])
    m = _FakeModel()
    m.lpoints = n
    m.mesh_cells = g["c"]
    m.mesh_coords = g["v"]
    w = outmesh.WriteMesh(m, str(tmp_path / "out"), compression="gzip")

    class _Done:
        def synchronize(self):
            pass

    for s in range(int(g["noutputs"])):
        host = torch.zeros((len(outmesh.FIELDS), n), dtype=torch.float32)
        for k in g["s%d_names" % s]:
            host[outmesh.FIELDS.index(str(k))] = torch.from_numpy(g["s%d_ds_%s" % (s, k)][:, 0])
        w._write(dict(step=s, save_time=float(g["save_times"][s]), sealevel=float(g["p_sealevel"]), event=_Done(),
                      host=host, upsub=True, rain=True, topology=w._topology() if s == 0 else None))
        path = str(tmp_path / "out" / "h5" / ("gospl.%d.p0.h5" % s))
        assert lint(path) == sorted(str(k) for k in g["s%d_names" % s])
        d = hdf5.read(path)
        for k in g["s%d_names" % s]:
            assert np.array_equal(d[str(k)], g["s%d_ds_%s" % (s, k)]), (s, k)
        assert (tmp_path / "out" / "xmf" / ("gospl%d.xmf" % s)).read_text() == str(g["s%d_xmf" % s])
    topo = hdf5.read(str(tmp_path / "out" / "h5" / "topology.p0.h5"))
    assert np.array_equal(topo["coords"], g["topo_coords"]) and np.array_equal(topo["cells"], g["topo_cells"])
    assert (tmp_path / "out" / "gospl.xdmf").read_text() == str(g["xdmf"])
    w.close()
