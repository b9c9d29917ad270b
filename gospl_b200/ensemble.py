"""Batched landscapes: many independent goSPL landscapes advanced as one.

Ensemble members (meshes of uneven size, each with its own erodibility,
rainfall and relief) are packed into one disjoint-union mesh, so every stage
of a step is one launch over all members instead of one launch per member.
The plan is told where members start (``gs_plan_set_members``): the lake
cascade of each member then follows that member's own control flow
(flowplex.py:850-904: excess, pass limit, stagnation, ``resid > maxarea``
with the member's own largest cell) and its own lake zeroing and fillFAL
maximum, so each member evolves as it would alone.  Two differences with a
per-member loop remain, both within solver tolerance: the hillslope CG takes
its step lengths from inner products over all members (each member's system
is still solved to the relative tolerance), and per-member residual sums run
in a different (fixed) order.

Members must share the time step, sea level, flow directions, exponents,
diffusivities and the deposition switches (nodep, nlPitVolume, nlPitDepth;
per-member erodibility, rainfall and uplift are fields); with deposition on,
each member runs its own sediment cascade (continental sediment routing of
the member alone); and
the fill level max(min h, sea + oFill) of every member must be the same (the
planar ensembles here pin their boundary at 0 m).

Across GPUs members are independent: ``partition`` assigns them to ranks by
vertex count (greedy, largest first) and each rank advances its own share
with no data-path collective.
"""
import numpy as np

from .mesh import FVMesh
from .model import Model

COMMON = ("dt", "tStart", "tEnd", "flowDir", "d", "m", "G", "Cda", "Cdm", "sealevel", "oFill", "nodep", "nlPitVolume",
          "nlPitDepth", "nlPitK", "pitInletBias", "picardSub", "picardIts")


def partition(sizes, world):
    """Greedy longest-processing-time assignment of members to `world` ranks:
    list of member-index lists, balanced by vertex count."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def union_mesh(meshes):
    """FVMesh of the disjoint union of `meshes` (vertex ids offset member by
    member) and the member start offsets."""
    start = np.zeros(len(meshes) + 1, np.int64)
    for m, me in enumerate(meshes):
        start[m + 1] = start[m] + me.n
    flat = {bool(me.flat) for me in meshes}
    if len(flat) != 1:
        raise ValueError("ensemble members must all be planar or all spherical")
    ngb = []
    for m, me in enumerate(meshes):
        g = np.asarray(me.ngb, np.int64).copy()
        g[g >= 0] += start[m]
        ngb.append(g.astype(np.int32))
    d = {
        "nnb": np.concatenate([me.nnb for me in meshes]),
        "ngb": np.concatenate(ngb),
        "elgt": np.concatenate([me.elgt for me in meshes]),
        "vdist": np.concatenate([me.vdist for me in meshes]),
        "farea": np.concatenate([me.farea for me in meshes]),
        "larea": np.concatenate([me.larea for me in meshes]),
        "outlet": np.concatenate([np.asarray(me.outlet, np.int64) + start[m] for m, me in enumerate(meshes)]),
        "open_nodes": np.concatenate([np.asarray(me.open_nodes, np.int64) + start[m]
                                      for m, me in enumerate(meshes)]),
        "flat": flat.pop(),
    }
    return FVMesh.from_arrays(d), start


class Ensemble:
    """Members advanced together on one GPU.

    ``members``: list of (coords, cells, elev, rain, upsub, params) with
    goSPL's parameter names (``K`` a scalar or a per-vertex field, ``bc``
    per member).  ``model`` is the underlying ``Model`` on the union mesh;
    ``view(tensor, m)`` slices member m out of any per-vertex tensor.
    """

    def __init__(self, members, device="cuda", cg_rtol=1.0e-13):
        import torch

        if not members:
            raise ValueError("an ensemble needs at least one member")
        p0 = members[0][5]
        for c, f, z, rain, up, p in members:
            for k in COMMON:
                if k in p0 and float(p.get(k, p0[k])) != float(p0[k]):
                    raise ValueError("ensemble members must share %s" % k)
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        meshes = [FVMesh(c, f, p.get("bc", "oooo"), device=dev) for c, f, z, rain, up, p in members]
        mesh, start = union_mesh(meshes)
        sea = float(p0.get("sealevel", 0.0))
        ofill = float(p0.get("oFill", -6000.0))
        levels = {max(float(np.min(z)), sea + ofill) for c, f, z, rain, up, p in members}
        if len(levels) != 1:
            raise ValueError("ensemble members must share the fill level max(min h, sea + oFill)")
        n = [len(z) for c, f, z, rain, up, p in members]
        K = np.concatenate([np.broadcast_to(np.asarray(p["K"], np.float64), (k,)) for k, (c, f, z, rain, up, p)
                            in zip(n, members)])
        rain = np.concatenate([np.asarray(r, np.float64) for c, f, z, r, up, p in members])
        ups = [up for c, f, z, r, up, p in members]
        upsub = None
        if any(u is not None for u in ups):
            upsub = np.concatenate([np.zeros(k) if u is None else np.asarray(u, np.float64) for k, u in zip(n, ups)])
        params = dict(p0, K=K, rain=rain, upsub=upsub)
        elev = np.concatenate([np.asarray(z, np.float64) for c, f, z, r, up, p in members])
        coords = np.concatenate([np.asarray(c, np.float64) for c, f, z, r, up, p in members])
        marea = np.array([float(me.larea.max()) for me in meshes])
        self.start = start
        self.sizes = np.asarray(n)
        self.mesh = mesh
        self.model = Model(coords=coords, elev=elev, params=params, mesh=mesh, device=dev, members=(start, marea),
                           cg_rtol=cg_rtol)

    @property
    def nmembers(self):
        return len(self.sizes)

    def view(self, t, m):
        return t[..., int(self.start[m]):int(self.start[m + 1])]

    def step(self):
        self.model.step()

    def runProcesses(self):
        self.model.runProcesses()

    def destroy(self):
        self.model.destroy()
