"""Precision form: FP32 flow/SPL sweeps and hillslope CG inside FP64
refinement against the plain FP64 path from the same state (one step): the
discrete results agree exactly and drainage area and elevation to 1e-8."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["planar", "sphere", "planar-deposition"])
def test_fp32_refined_matches_fp64(kind):
    import torch
    from gospl_b200 import _lib
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model

    if kind.startswith("planar"):
        c, f, z, rain, up, p = S.planar_config(n=6000, side=50.0e3, seed=41)
    else:
        c, f, z, rain, up, p = S.sphere_config(level=5, seed=42, lmax=32)
    p = dict(p, rain=rain, upsub=up, tEnd=1e30)
    if kind.endswith("deposition"):   # the sediment flux and cascade sweeps refined too
        p = dict(p, nodep=False)
    mesh = FVMesh(c, f, p["bc"])
    m64 = Model(coords=c, cells=f, elev=z, params=p, mesh=mesh, device="cuda:0")
    m32 = Model(coords=c, cells=f, elev=z, params=p, mesh=mesh, device="cuda:0", precision=32, refine_tol=1e-10)
    m32.hGlobal.copy_(m64.hGlobal)
    m32.bL.copy_(m64.bL)
    m64.step()
    m32.step()
    torch.cuda.synchronize()
    assert _lib.load().gs_plan_tuning(m32._plan, 4) > 0, "no refinement pass ran"
    assert np.array_equal(m32.rcv_i.cpu().numpy(), m64.rcv_i.cpu().numpy())
    assert np.array_equal(m32.pitIDs.cpu().numpy(), m64.pitIDs.cpu().numpy())
    for name in ("FAL", "hGlobal") + (("vSed",) if kind.endswith("deposition") else ()):
        a = getattr(m32, name).cpu().numpy()
        b = getattr(m64, name).cpu().numpy()
        err = np.abs(a - b).max() / max(np.abs(b).max(), 1.0)
        assert err <= 1e-8, (name, err)
    m32.destroy()
    m64.destroy()
