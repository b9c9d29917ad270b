"""gs_flow_solve_noalloc, the allocation-free flow solve, against the regular
path through the C ABI.

Callers that cannot call cudaMalloc (an embedding application that owns all
device memory, or one held to a fixed device-memory budget) use this entry
point; it keeps its scratch in a fixed device array.  On a landscape with no
depressions, gs_flow_accumulation's drainage area is exactly the solve of
(I - W^T) q = rain * area over the receivers it returns, so the two must
agree.  The shared scratch keeps the previous call's contents, so the solve
runs twice in a row, after a larger landscape, and after a call that ended on
a cycle, to check that every call starts from a clean state.  This file is
collected last so that a failure here cannot hide the other GPU tests.
"""
import ctypes
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GS_ECYCLE = 5


def _pit_free_model(n):
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model

    side = 30.0e3 * np.sqrt(n / 6000.0)
    coords, cells, onb = S.planar_hex_mesh(n, side, seed=11)
    z = 1.0e-3 * coords[:, 0] + 5.0e-4 * coords[:, 1]          # planar tilt: no interior minima
    params = dict(dt=1000.0, tEnd=1.0e4, flowDir=3, K=2.0e-6, d=0.0, m=0.5, Cda=0.1, Cdm=0.1,
                  sealevel=-100.0, bc="ffff", rain=np.ones(len(z)), upsub=None)
    mesh = FVMesh(coords, cells, "ffff")
    return Model(coords=coords, cells=cells, elev=z, params=params, mesh=mesh)


def _solve(L, m, q):
    import torch
    from gospl_b200 import _lib

    b = torch.where(m.sea_mask.bool(), torch.zeros_like(m.bL), m.bL)
    stream = ctypes.c_void_p(torch.cuda.current_stream(m.dev).cuda_stream)
    q.fill_(float("nan"))
    return L.gs_flow_solve_noalloc(m.lpoints, m.flowDir, _lib.ptr(m.rcv_i), _lib.ptr(m.wgt_i), _lib.ptr(b),
                                   _lib.ptr(q), stream)


def _check(L, m, label):
    import torch

    pp, _, _, _ = m.pit_tables()
    assert float(pp[:, 0].max()) <= 0.0, "the test landscape must have no depression volume"
    q = torch.empty(m.lpoints, dtype=torch.float64, device=m.dev)
    rc = _solve(L, m, q)
    assert rc == 0, "%s returned %d" % (label, rc)
    got = q.cpu().numpy()
    ref = m.FAL.cpu().numpy()
    assert np.all(np.isfinite(got)), label
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= 1e-12, "%s: relative difference %g" % (label, err)


def test_noalloc_flow_solve_matches_flow_accumulation():
    import torch
    from gospl_b200 import _lib

    L = _lib.load()
    big = _pit_free_model(20000)
    small = _pit_free_model(6000)
    torch.cuda.synchronize()
    # a larger graph first, then the smaller one twice: the second and third
    # calls find the first call's counters and donor lists in the scratch
    _check(L, big, "20000-vertex call")
    for call in range(2):
        _check(L, small, "6000-vertex call %d" % call)
    big.destroy()
    small.destroy()


def test_noalloc_reports_a_cycle_and_recovers():
    """Two vertices that drain into each other: the sweep finds nothing
    ready and nothing in flight, stops, and returns GS_ECYCLE (a bounded
    quiescence check, not a time-out); the next valid call is unaffected."""
    import torch
    from gospl_b200 import _lib

    L = _lib.load()
    m = _pit_free_model(6000)
    _check(L, m, "call before the cycle")     # also resolves the scratch address on this device
    dev = m.dev
    rcv = torch.tensor([1, 0], dtype=torch.int32, device=dev)
    wgt = torch.ones(2, dtype=torch.float64, device=dev)
    b = torch.ones(2, dtype=torch.float64, device=dev)
    q = torch.zeros(2, dtype=torch.float64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    t0 = time.perf_counter()
    rc = L.gs_flow_solve_noalloc(2, 1, _lib.ptr(rcv), _lib.ptr(wgt), _lib.ptr(b), _lib.ptr(q), stream)
    assert rc == GS_ECYCLE, rc
    assert time.perf_counter() - t0 < 2.0, "the cycle must be found by quiescence, well before the time budget"
    buf = ctypes.create_string_buffer(256)
    L.gs_last_error(buf, 256)
    assert b"cycle" in buf.value
    _check(L, m, "call after the cycle")
    m.destroy()


def test_noalloc_rejects_sizes_beyond_its_limit():
    from gospl_b200 import _lib

    L = _lib.load()
    assert L.gs_flow_solve_noalloc(1048577, 3, None, None, None, None, None) == 1
    assert L.gs_flow_solve_noalloc(1000, 5, None, None, None, None, None) == 1
    buf = ctypes.create_string_buffer(256)
    L.gs_last_error(buf, 256)
    assert b"nrcv" in buf.value
