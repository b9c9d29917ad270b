"""Marine deposition on the GPU (gs_sea_change, Model.seaChange) against the
oracle, whose seaChange is pinned to the reference's own seaplex.py run in the
fixture harness (tests/test_oracle_golden.py).

Stage parity: every step of the planar (open boundary, sea level above part
of the land) and spherical marine fixtures starts from the oracle's state;
flow accumulation, SPL, the second flow accumulation and sedChange must match
as in the continental tests, the live sea mask after sedChange must equal the
oracle's seaID, and after seaChange the marine cascade must take the oracle's
number of passes and elevation, cumED and EbLocal must agree to 1e-11 of the
elevation scale (the oracle solves the smoothing and the Picard systems
exactly, the GPU by CG to 1e-14 and 1e-13).  ico2562_marine_G (Gmar = 0.5)
adds the coupled marine elevation / flux system between two cascades (the
oracle by sparse LU, the GPU by GMRES over ordered marine sweeps to 1e-13).
One free-running step is checked against the reference-generated fixtures.
"""
import numpy as np
import pytest

from conftest import golden_mesh, golden_params, load_golden
from test_gpu_parity import _compare_dz, _compare_flow, _compare_sed, _gpu_model, _np, _rel, _resync, _resync_flow

pytestmark = pytest.mark.gpu

CASES = ["planar2k_marine", "ico2562_marine", "ico2562_marine_G"]


@pytest.mark.parametrize("case", CASES)
def test_marine_stage_parity_from_identical_state(case):
    import torch
    from oracle.model import OracleModel
    g = load_golden(case)
    params = golden_params(g)
    gm = _gpu_model(g, params)
    om = OracleModel(g["v"], g["c"], g["z"], params, mesh=golden_mesh(g))
    passes = []
    for s in range(int(g["nsteps"])):
        tag = "%s step%d" % (case, s + 1)
        _resync(gm, om)
        gm.flowAccumulation()
        om.flowAccumulation()
        _compare_flow(gm, om, tag + " flow", 1e-12)
        _resync_flow(gm, om)
        gm.erodepSPL()
        om.erodepSPL()
        torch.cuda.synchronize()
        _compare_dz(gm, om, tag + " spl")
        _resync(gm, om)
        gm.flowAccumulation()
        om.flowAccumulation()
        _compare_flow(gm, om, tag + " flow2", 1e-12)
        _resync_flow(gm, om)
        gm.sedChange()
        om.sedChange()
        _compare_sed(gm, om, tag + " sed")
        sea = np.zeros(om.lpoints, dtype=bool)
        sea[om.seaID] = True
        assert np.array_equal(_np(gm.seaID), sea), tag + " seaID after sedChange"
        _resync(gm, om)
        gm.vSed.copy_(torch.as_tensor(om.vSed))
        gm.seaChange()
        om.seaChange()
        torch.cuda.synchronize()
        hs = float(np.abs(om.h).max())
        assert gm.stats["sea"]["marine_passes"] == om.marine_passes, (tag, gm.stats["sea"], om.marine_passes)
        if om.Gmar > 0.0 and not om.flatModel:
            assert gm.stats["sea"]["coupled_applies"] > 0, tag
        assert np.abs(_np(gm.hGlobal) - om.h).max() <= 1e-11 * hs, "%s sea h %g" % (
            tag, np.abs(_np(gm.hGlobal) - om.h).max() / hs)
        assert np.abs(_np(gm.cumED) - om.cumED).max() <= 1e-11 * hs, tag + " sea cumED"
        assert np.abs(_np(gm.EbLocal) - om.EbLocal).max() <= 1e-11 * hs / om.dt, tag + " sea EbLocal"
        passes.append(om.marine_passes)
        _resync(gm, om)
        gm.getHillslope()
        om.getHillslope()
        torch.cuda.synchronize()
        _compare_dz(gm, om, tag + " hillslope")
    assert max(passes) > 0, "the cascade must run"
    gm.destroy()


@pytest.mark.parametrize("case", CASES)
def test_marine_matches_reference_golden_first_step(case):
    """One free-running step with continental and marine deposition against
    the reference's own seaplex.py run (the fixtures)."""
    import torch
    g = load_golden(case)
    params = golden_params(g)
    gm = _gpu_model(g, params)
    gm.step()
    torch.cuda.synchronize()
    assert np.array_equal(_np(gm.rcvIDi), g["s1_rcvIDi"].astype(np.int32))
    assert np.array_equal(_np(gm.pitIDs), g["s1_pitIDs"])
    for k in ("FAL", "cumED"):
        assert _rel(getattr(gm, k), g["s1_" + k]) <= 1e-10, k
    assert _rel(gm.hGlobal, g["s1_h"]) <= 1e-10
    gm.destroy()

