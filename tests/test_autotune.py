"""Launch-shape knobs and the autotuner: the plan accepts shapes within the
co-residency limit, refuses others, and a step gives the same landscape under
any shape (to the rounding of the CG inner products)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_knobs_and_tuner():
    import torch
    from gospl_b200 import _lib, autotune
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model

    c, f, z, rain, up, p = S.planar_config(n=5000, side=40.0e3, seed=31)
    p = dict(p, rain=rain, upsub=up, tEnd=1e30)
    m = Model(coords=c, cells=f, elev=z, params=p, mesh=FVMesh(c, f, p["bc"]), device="cuda:0")
    limit = autotune._get(m, autotune.COOP + 1)
    assert limit >= 1
    with pytest.raises(_lib.GsError):
        autotune._set(m, autotune.COOP, limit + 1)
    with pytest.raises(_lib.GsError):
        autotune._set(m, autotune.SWEEP, 0)
    h0 = m.hGlobal.clone()
    outs = []
    for s, cb in ((2, 1), (16, limit)):
        autotune._set(m, autotune.SWEEP, s)
        autotune._set(m, autotune.COOP, cb)
        m.hGlobal.copy_(h0)
        m.step()
        outs.append(m.hGlobal.clone())
    assert (outs[0] - outs[1]).abs().max() <= 1e-12 * h0.abs().max()
    m.hGlobal.copy_(h0)
    best, table = autotune.tune(m, steps=1, sweep=(4, 8), coop=(1, 2))
    assert best in table and all(np.isfinite(v) and v > 0 for v in table.values())
    assert torch.equal(m.hGlobal, h0)
    assert autotune._get(m, autotune.SWEEP) == best[0]
    m.destroy()
