"""gs_flow_solve_noalloc, the allocation-free flow solve, against the regular
path through the C ABI.

Callers that cannot call cudaMalloc (an embedding application that owns all
device memory, a fixed memory budget, a stream under capture) use this entry
point; it keeps its scratch in a fixed device array.  On a landscape with no
depressions, gs_flow_accumulation's drainage area is exactly the solve of
(I - W^T) q = rain * area over the receivers it returns, so the two must
agree; the allocation-free solve runs twice in a row to check that the shared
scratch is re-initialised between calls.  This file is collected last so that
a failure here cannot hide the other GPU tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pit_free_model():
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model

    coords, cells, onb = S.planar_hex_mesh(6000, 30.0e3, seed=11)
    z = 1.0e-3 * coords[:, 0] + 5.0e-4 * coords[:, 1]          # planar tilt: no interior minima
    params = dict(dt=1000.0, tEnd=1.0e4, flowDir=3, K=2.0e-6, d=0.0, m=0.5, Cda=0.1, Cdm=0.1,
                  sealevel=-100.0, bc="ffff", rain=np.ones(len(z)), upsub=None)
    mesh = FVMesh(coords, cells, "ffff")
    return Model(coords=coords, cells=cells, elev=z, params=params, mesh=mesh)


def test_noalloc_flow_solve_matches_flow_accumulation():
    import torch
    from gospl_b200 import _lib

    L = _lib.load()
    m = _pit_free_model()
    torch.cuda.synchronize()
    pp, _, _, _ = m.pit_tables()
    assert float(pp[:, 0].max()) <= 0.0, "the test landscape must have no depression volume"
    n, R = m.lpoints, m.flowDir
    b = torch.where(m.sea_mask.bool(), torch.zeros_like(m.bL), m.bL)
    q = torch.empty(n, dtype=torch.float64, device=m.dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(m.dev).cuda_stream)
    ref = m.FAL.cpu().numpy()
    for call in range(2):
        q.fill_(float("nan"))
        rc = L.gs_flow_solve_noalloc(n, R, _lib.ptr(m.rcv_i), _lib.ptr(m.wgt_i), _lib.ptr(b), _lib.ptr(q),
                                     stream)
        assert rc == 0, "call %d returned %d" % (call, rc)
        got = q.cpu().numpy()
        assert np.all(np.isfinite(got)), call
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= 1e-12, "call %d: relative difference %g" % (call, err)
    m.destroy()


def test_noalloc_rejects_sizes_beyond_its_limit():
    from gospl_b200 import _lib

    L = _lib.load()
    assert L.gs_flow_solve_noalloc(1048577, 3, None, None, None, None, None) == 1
    assert L.gs_flow_solve_noalloc(1000, 5, None, None, None, None, None) == 1
    buf = ctypes.create_string_buffer(256)
    L.gs_last_error(buf, 256)
    assert b"nrcv" in buf.value
