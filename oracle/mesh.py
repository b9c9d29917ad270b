"""ORACLE — test infrastructure only.

Restatement of goSPL's single-rank mesh construction:

* the numpy Voronoi helpers of ``gospl/mesher/meshfunc.py`` (``initVoronoi``
  75-153, ``control_volumes`` 175-197, ``create_edges`` 295-327,
  ``cell_circumcenters`` 400-407, with ``unique_rows`` 20-28 and
  ``compute_triangle_circumcenters`` 48-59);
* ``_meshStructure`` (``gospl/mesher/unstructuredmesh.py:120-202``) calling the
  Fortran ``definetin`` restatement;
* the single-rank boundary bookkeeping of ``_buildMesh``
  (``unstructuredmesh.py:444-533``): boundary nodes, ``outletIDs`` per the
  NESW ``bc`` flags, ``flatModel``; ``idLBounds`` and ``ghostIDs`` are empty on
  one rank (``unstructuredmesh.py:556-560``).

At one rank the local node order is the input order and ``locIDs`` is the
identity (``unstructuredmesh.py:415-442``).  Cells are handled as int32, the
PETSc ``IntType`` the reference stores them in (``unstructuredmesh.py:363``);
that dtype fixes the byte-lexicographic edge order produced by the void-view
``np.unique`` in ``unique_rows`` and therefore every vertex's neighbour order.
"""
import numpy as np

from . import fortran as F


def unique_rows(a):
    b = np.ascontiguousarray(a).view(np.dtype((np.void, a.dtype.itemsize * a.shape[1])))
    a_unique, inv, cts = np.unique(b, return_inverse=True, return_counts=True)
    a_unique = a_unique.view(a.dtype).reshape(-1, a.shape[1])
    return a_unique, inv, cts


def voronoi_inputs(coords, cells):
    """Edges, cell->edge map, circumcentres, control volumes (meshfunc.py)."""
    cells = np.asarray(cells, dtype=np.int32)
    local_idx = np.array([[1, 2], [2, 0], [0, 1]]).T
    nds = cells.T
    idx_hierarchy = nds[local_idx]
    half = coords[idx_hierarchy[1]] - coords[idx_hierarchy[0]]
    ei_dot_ej = np.einsum("ijk, ijk->ij", half[[1, 2, 0]], half[[2, 0, 1]])
    ei_dot_ei = np.einsum("ijk, ijk->ij", half, half)
    cell_volumes = 0.5 * np.sqrt(
        ei_dot_ej[2] * ei_dot_ej[0] + ei_dot_ej[0] * ei_dot_ej[1] + ei_dot_ej[1] * ei_dot_ej[2])
    ce_ratios = -ei_dot_ej * 0.25 / cell_volumes[None]
    # control volumes
    v = 0.25 * ei_dot_ei * ce_ratios
    vals = np.array([sum([v[i] for i in np.where(local_idx.T == k)[0]]) for k in range(3)])
    cv = np.zeros(len(coords))
    np.add.at(cv, cells.T, vals)
    # edges
    s = idx_hierarchy.shape
    a = np.sort(idx_hierarchy.reshape(s[0], -1).T)
    a_unique, inv, cts = unique_rows(a)
    if not np.all(cts < 3):
        raise ValueError("No edge has more than 2 cells. Are cells listed twice?")
    cells_edges = inv.reshape(3, -1).T
    boundary_edge = cts == 1
    # circumcentres
    X = coords[nds]
    alpha = ei_dot_ei * ei_dot_ej
    alpha_sum = alpha[0] + alpha[1] + alpha[2]
    beta = alpha / alpha_sum[None]
    aa = X * beta[..., None]
    cc = aa[0] + aa[1] + aa[2]
    return {"edges": a_unique, "cells_edges": cells_edges, "cc": cc,
            "control_volumes": cv, "boundary_edge": boundary_edge}


def build_mesh(coords, cells, bc="oooo"):
    """Single-rank goSPL mesh: FV arrays, areas and boundary sets."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    cells = np.asarray(cells, dtype=np.int32)
    nb = coords.shape[0]
    vi = voronoi_inputs(coords, cells)
    edges = vi["edges"]
    bnodes = np.unique(edges[vi["boundary_edge"]].ravel()) if vi["boundary_edge"].any() \
        else np.zeros(0, dtype=np.int64)
    flat = len(bnodes) > 0
    larea_mf = np.abs(vi["control_volumes"])
    larea_mf[np.isnan(larea_mf)] = 1.0
    cc = vi["cc"]
    if not flat:
        radius = np.linalg.norm(coords[0])
        cc = cc * (radius / np.linalg.norm(cc, axis=1)).reshape((len(cc), 1))
    F.setcurvedmesh(0 if flat else 1)
    ngbid, larea = F.definetin(coords, cells, vi["cells_edges"], edges, cc.T)
    larea = larea.copy()
    larea[np.isnan(larea)] = 1.0
    if flat and np.max(np.abs(larea_mf - larea)) > 1.0e2:
        larea = larea_mf.copy()
        F.updatearea(larea_mf)
    nnb, ngb, elgt, vdist, farea = F.getmesh()
    outlet = bnodes.astype(np.int64)
    if flat:
        bcmap = {"o": 0, "f": 1, "c": 2, "w": 3}
        north, east, south, west = (bcmap[c] for c in bc)
        xmin, xmax = coords[:, 0].min(), coords[:, 0].max()
        ymin, ymax = coords[:, 1].min(), coords[:, 1].max()
        tol = 1.0e-9
        pts = {
            "S": np.where(np.isclose(coords[:, 1], ymin, atol=tol))[0],
            "N": np.where(np.isclose(coords[:, 1], ymax, atol=tol))[0],
            "E": np.where(np.isclose(coords[:, 0], xmax, atol=tol))[0],
            "W": np.where(np.isclose(coords[:, 0], xmin, atol=tol))[0],
        }
        flags = {"N": north, "E": east, "S": south, "W": west}
        wall = [pts[k] for k in ("S", "E", "N", "W") if flags[k] == 3 and len(pts[k]) > 0]
        if wall:
            outlet = np.setdiff1d(bnodes, np.unique(np.concatenate(wall)))
        openp = [pts[k] for k in ("N", "E", "S", "W") if flags[k] == 0 and len(pts[k]) > 0]
        open_nodes = np.unique(np.concatenate(openp)) if openp else np.zeros(0, np.int64)
    else:
        open_nodes = np.zeros(0, np.int64)
    return {
        "coords": coords, "cells": cells, "nb": nb, "flat": flat,
        "nnb": nnb, "ngb": ngb, "elgt": elgt, "vdist": vdist, "farea": farea,
        "larea": larea, "maxarea": float(larea.max()),
        "borders": bnodes.astype(np.int64), "outlet": outlet.astype(np.int64),
        "open_nodes": open_nodes.astype(np.int64),
        "edges": edges, "cc": cc,
    }


def load_mesh(mesh):
    """Install a mesh dict (as returned by build_mesh) into the Fortran state."""
    F.setmesh(mesh["nnb"], mesh["ngb"], mesh["elgt"], mesh["vdist"], mesh["farea"])
