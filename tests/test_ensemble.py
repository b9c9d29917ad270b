"""Batched landscapes (gospl_b200.ensemble): member partitioning across ranks
(CPU, including a 2-rank gloo run) and, on the GPU, every member of a packed
ensemble evolving exactly as it does alone."""
import os
import socket

import numpy as np
import pytest

from gospl_b200 import synthetic as S
from gospl_b200.ensemble import partition, union_mesh
from gospl_b200.mesh import FVMesh


def test_partition_balances_and_covers():
    sizes = S.ensemble_sizes(64, 1.0e4, 5.0e5, seed=7)
    for world in (1, 2, 3, 8):
        parts = partition(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [int(np.sum(sizes[p])) for p in parts]
        assert max(loads) - min(loads) <= int(np.max(sizes))


def test_union_mesh_offsets():
    a = S.planar_hex_mesh(300, 5.0e3, seed=1)
    b = S.planar_hex_mesh(500, 7.0e3, seed=2)
    ma, mb = FVMesh(a[0], a[1], "ffff"), FVMesh(b[0], b[1], "ffff")
    u, start = union_mesh([ma, mb])
    assert list(start) == [0, ma.n, ma.n + mb.n]
    assert np.array_equal(u.ngb[:ma.n], ma.ngb)
    g = mb.ngb.astype(np.int64)
    g[g >= 0] += ma.n
    assert np.array_equal(u.ngb[ma.n:], g)
    assert np.array_equal(u.outlet, np.concatenate([ma.outlet, mb.outlet + ma.n]))
    assert u.maxarea == max(ma.maxarea, mb.maxarea)


def _rank(rank, world, port, sizes, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = partition(sizes, world)[rank]
    t = torch.zeros(len(sizes), dtype=torch.int64)
    t[mine] = 1
    dist.all_reduce(t)
    load = torch.tensor([int(np.sum(np.asarray(sizes)[mine]))], dtype=torch.int64)
    loads = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(loads, load)
    if rank == 0:
        out.put((t.tolist(), [int(x) for x in loads]))
    dist.destroy_process_group()


def test_two_rank_partition_gloo():
    import multiprocessing as mp
    sizes = [int(x) for x in S.ensemble_sizes(16, 1.0e4, 5.0e5, seed=3)]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in ps:
        p.start()
    cover, loads = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert cover == [1] * len(sizes)
    assert sum(loads) == sum(sizes)


@pytest.mark.gpu
@pytest.mark.parametrize("nodep,G", [(True, 0.0), (False, 0.0), (True, 1.0)])
def test_members_evolve_as_alone(nodep, G):
    """Each member of an ensemble evolves as it would alone, with and without
    continental deposition (each member its own flow and sediment cascade) and
    with transport-limited erosion (one coupled solve for all members, to the
    solver's tolerance)."""
    import torch
    from gospl_b200.ensemble import Ensemble
    from gospl_b200.model import Model

    members = [S.ensemble_member(n, seed) for n, seed in ((2500, 11), (4000, 12), (6000, 13))]
    members = [(c, f, z, r, u, dict(p, nodep=nodep, G=G)) for c, f, z, r, u, p in members]
    ens = Ensemble(members)
    dev = torch.device("cuda", torch.cuda.current_device())
    alone = []
    for c, f, z, rain, up, p in members:
        m = Model(coords=c, cells=f, elev=z, params=dict(p, rain=rain, upsub=up),
                  mesh=FVMesh(c, f, p["bc"], device=dev))
        alone.append(m)
    # with G > 0 one step: the members' solutions differ from the solo runs at
    # the solver's tolerance, which later discrete decisions may amplify
    for step in range(3 if G == 0.0 else 1):
        ens.step()
        for m in alone:
            m.step()
        torch.cuda.synchronize()
        for k, m in enumerate(alone):
            off = int(ens.start[k])
            for name in ("pitIDs", "flatDirs", "rcv_i", "lsink_mask"):
                a = ens.view(getattr(ens.model, name), k).cpu().numpy().astype(np.int64)
                b = getattr(m, name).cpu().numpy().astype(np.int64)
                if name == "pitIDs":   # pit ids are numbered over the whole ensemble
                    assert np.array_equal(a >= 0, b >= 0), (step, k, name)
                    continue
                if name in ("flatDirs", "rcv_i"):   # vertex ids of the union mesh
                    a = np.where(a >= 0, a - off, a)
                assert np.array_equal(a, b), (step, k, name)
            hscale = max(np.abs(m.hGlobal.cpu().numpy()).max(), 1.0)
            for name in ("FAL", "hGlobal", "cumED", "lFill") + (() if nodep else ("vSed",)):
                a = ens.view(getattr(ens.model, name), k).cpu().numpy()
                b = getattr(m, name).cpu().numpy()
                scale = max(np.abs(b).max(), 1.0) if name in ("FAL", "vSed") else hscale
                tol = 1e-12 if G == 0.0 else 1e-10
                assert np.abs(a - b).max() <= tol * scale, (step, k, name, np.abs(a - b).max())
    for m in alone:
        m.destroy()
    ens.destroy()
