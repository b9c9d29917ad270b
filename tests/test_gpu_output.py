"""Outputs and restarts on the device path: the packing kernel bit for bit
against the oracle's restatement of _outputMesh, a run's files against the
reference's own datasets and XMF text, and a restart from the files
(gospl/tools/outmesh.py)."""
import os

import numpy as np
import pytest

from conftest import golden_params, load_golden

pytestmark = pytest.mark.gpu


def _model(g, **extra):
    from gospl_b200.model import Model
    p = golden_params(g)
    p.update(extra)
    return Model(coords=g["v"], cells=g["c"], elev=g["z"], params=p, device="cuda:0")


def _pack(m, fields, sea):
    """gs_output_fields on explicit float64 inputs; returns [9, n] float32."""
    import torch
    from gospl_b200 import _lib
    dev = m.dev
    t = {k: (None if v is None else torch.as_tensor(v, dtype=torch.float64, device=dev)) for k, v in fields.items()}
    s = None if sea is None else torch.as_tensor(sea, dtype=torch.uint8, device=dev)
    out = torch.full((9, m.lpoints), -7.0, dtype=torch.float32, device=dev)
    _lib.check(_lib.load().gs_output_fields(
        m._plan, _lib.ptr(t["h"]), _lib.ptr(t["cumED"]), _lib.ptr(t["Eb"]), _lib.ptr(t["waterFilled"]),
        _lib.ptr(t["fillFAL"]), _lib.ptr(t["FAL"]), _lib.ptr(t["vSed"]), _lib.ptr(t["upsub"]), _lib.ptr(t["rain"]),
        _lib.ptr(s), _lib.ptr(out)))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _check_rows(out, ref, names):
    from gospl_b200.outmesh import FIELDS
    for k in names:
        a = out[FIELDS.index(k)]
        b = ref[k][:, 0]
        nan = np.isnan(b)
        assert a.dtype == b.dtype
        assert np.array_equal(a.view(np.uint32)[~nan], b.view(np.uint32)[~nan]), k
        assert np.array_equal(np.isnan(a), nan), k


def test_output_fields_bit_exact():
    """Floors, sea edits and the float64 -> float32 rounding (ties to even,
    overflow to infinity, NaN kept) match the oracle bit for bit."""
    from gospl_b200._lib import GsError
    from oracle.model import output_fields, DISCHARGE_FLOOR
    g = load_golden("output_planar2k")
    m = _model(g)
    n = m.lpoints
    rng = np.random.default_rng(11)
    f = {k: rng.standard_normal(n) * 10.0 ** rng.integers(-12, 9, n) for k in
         ("h", "cumED", "Eb", "waterFilled", "fillFAL", "FAL", "vSed", "upsub", "rain")}
    for k in ("fillFAL", "FAL", "vSed"):
        f[k][:50] = DISCHARGE_FLOOR
        f[k][50:60] = np.nextafter(DISCHARGE_FLOOR, 1.0)
        f[k][60:70] = np.nan
        f[k][70:80] = -5.0
    ones = np.float32(1.0) + np.float32(2.0 ** -23) * np.arange(20, dtype=np.float32)
    f["h"][:20] = ones.astype(np.float64) + 2.0 ** -24          # halfway between two floats
    f["h"][20:25] = 1.0e39                                      # beyond float32
    sea = (rng.random(n) < 0.2).astype(np.uint8)
    ref = output_fields(f["h"], f["cumED"], f["Eb"], f["waterFilled"], f["fillFAL"], f["FAL"], f["vSed"],
                        f["upsub"], f["rain"], sea)
    out = _pack(m, f, sea)
    _check_rows(out, ref, ref.keys())
    # no tectonics or rain rows: those rows are left as they were
    out = _pack(m, dict(f, upsub=None, rain=None), sea)
    assert (out[7] == -7.0).all() and (out[8] == -7.0).all()
    # without a mask: none before the first hillslope call ...
    with pytest.raises(GsError):
        _pack(m, f, None)
    # ... then the mask of the elevation that call started from (hillslope.py:620)
    h0 = m.hGlobal.cpu().numpy().copy()
    m.getHillslope()
    out = _pack(m, f, None)
    ref = output_fields(f["h"], f["cumED"], f["Eb"], f["waterFilled"], f["fillFAL"], f["FAL"], f["vSed"],
                        f["upsub"], f["rain"], (h0 <= m.sealevel).astype(np.uint8))
    _check_rows(out, ref, ["FA", "fillFA"])
    m.destroy()
    # the same with no diffusion at all (Cda = Cdm = 0)
    m = _model(g, Cda=0.0, Cdm=0.0)
    h0 = m.hGlobal.cpu().numpy().copy()
    m.getHillslope()
    out = _pack(m, f, None)
    ref = output_fields(f["h"], f["cumED"], f["Eb"], f["waterFilled"], f["fillFAL"], f["FAL"], f["vSed"],
                        f["upsub"], f["rain"], (h0 <= m.sealevel).astype(np.uint8))
    _check_rows(out, ref, ["FA", "fillFA"])
    m.destroy()


def _close_f32(a, b, scale):
    """float32 fields made from float64 states that agree to 1e-10 of the
    field's scale: equal up to one float32 step."""
    return np.abs(a.astype(np.float64) - b.astype(np.float64)) <= np.spacing(np.abs(b)).astype(np.float64) \
        + 1e-10 * scale


def test_run_outputs_match_reference(tmp_path):
    """runProcesses with outputs every step writes the reference's files: the
    same datasets, XMF and XDMF text at every output, the topology exactly;
    the values of the initial output and of the one after the first step to
    one float32 step of the reference's (the multi-step agreement of the
    states themselves is what the golden step tests pin), and the last output
    bit for bit the float32 rounding of this run's own final state."""
    from gospl_b200 import hdf5
    from oracle.model import output_fields
    g = load_golden("output_planar2k")
    out = str(tmp_path / "out")
    dt = float(g["p_dt"])
    m = _model(g, outputDir=out, tout=dt)
    m.runProcesses()
    st = {k: getattr(m, k).cpu().numpy() for k in ("hGlobal", "cumED", "EbLocal", "waterFilled", "fillFAL", "FAL",
                                                  "vSed", "upsub", "rainVal")}
    n = m.lpoints
    m.destroy()
    topo = hdf5.read(os.path.join(out, "h5", "topology.p0.h5"))
    assert np.array_equal(topo["coords"], g["topo_coords"]) and np.array_equal(topo["cells"], g["topo_cells"])
    nout = int(g["noutputs"])
    for s in range(nout):
        d = hdf5.read(os.path.join(out, "h5", "gospl.%d.p0.h5" % s))
        assert sorted(d) == sorted(g["s%d_names" % s]), s
        hs = float(np.abs(g["s%d_ds_elev" % s]).max())
        for k, v in d.items():
            ref = g["s%d_ds_%s" % (s, k)]
            assert v.dtype == ref.dtype and v.shape == ref.shape
            if s > 1:
                continue
            scale = {"elev": hs, "erodep": hs, "EDrate": hs / dt}.get(k, float(np.abs(ref).max()))
            ok = _close_f32(v, ref, scale)
            assert ok.all(), (s, k, int((~ok).sum()), float(np.abs(v - ref).max()))
        with open(os.path.join(out, "xmf", "gospl%d.xmf" % s)) as fh:
            assert fh.read() == str(g["s%d_xmf" % s]), s
    with open(os.path.join(out, "gospl.xdmf")) as fh:
        assert fh.read() == str(g["xdmf"])
    last = hdf5.read(os.path.join(out, "h5", "gospl.%d.p0.h5" % (nout - 1)))
    own = output_fields(st["hGlobal"], st["cumED"], st["EbLocal"], st["waterFilled"], st["fillFAL"], st["FAL"],
                        st["vSed"], st["upsub"], st["rainVal"], np.zeros(n, np.uint8))
    for k in ("elev", "erodep", "EDrate", "waterFill", "sedLoad", "uplift", "rain"):
        assert np.array_equal(last[k], own[k]), k


def test_restart_from_outputs(tmp_path):
    """rStep = 2: the state comes back from gospl.2.p0.h5 (float32 widened),
    time and output counters resume, and the run writes output 3 with the
    time series listing 0..3 (model.py:289-291, outmesh.py:61-79, 505-562)."""
    from gospl_b200 import hdf5
    g = load_golden("output_planar2k")
    out = str(tmp_path / "out")
    dt = float(g["p_dt"])
    m = _model(g, outputDir=out, tout=dt, compression="none")
    m.runProcesses()
    m.destroy()
    d2 = hdf5.read(os.path.join(out, "h5", "gospl.2.p0.h5"))
    r = _model(g, outputDir=out, tout=dt, rStep=2, compression="none")
    assert r.tNow == 2 * dt and r.output.step == 3 and r.output.saveTime == 3 * dt
    for name, k in (("hGlobal", "elev"), ("cumED", "erodep"), ("vSed", "sedLoad"), ("EbLocal", "EDrate")):
        assert np.array_equal(getattr(r, name).cpu().numpy(), d2[k][:, 0].astype(np.float64)), name
    os.remove(os.path.join(out, "h5", "gospl.3.p0.h5"))
    r.runProcesses()
    r.destroy()
    assert r.tNow == 3 * dt
    d3 = hdf5.read(os.path.join(out, "h5", "gospl.3.p0.h5"))
    assert np.isfinite(d3["elev"]).all()
    with open(os.path.join(out, "gospl.xdmf")) as fh:
        assert fh.read().count("<xi:include") == 4
    with pytest.raises(ValueError):
        _model(g, outputDir=out, tout=dt, rStep=7)          # no gospl.7.p0.h5
