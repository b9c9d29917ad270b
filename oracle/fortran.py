"""ORACLE — test infrastructure only (tests/, smoke check, CPU-baseline leg).

ctypes bindings of ``gospl_oracle.c``, the C restatement of goSPL's Fortran
kernels (``fortran/functions.F90``), exposed with the same Python call
signatures as the reference's f2py module ``gospl._fortran``
(``fortran/functions.pyf``): intent(in) arrays are arguments, intent(out)
arrays are returned in argument order.  Mesh state is module-global, set by
``definetin`` (``functions.F90:2715``) or ``setmesh``, exactly like the
Fortran module ``meshparams``.

The product never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "gospl_oracle.c")
_LIB = os.path.join(_HERE, "liborc.so")


def build(force=False):
    """Compile the oracle C restatement (gcc, IEEE double, no FMA contraction)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        subprocess.check_call(
            ["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off",
             "-o", _LIB, _SRC, "-lm"])
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB)
        P = ctypes.c_void_p
        i = ctypes.c_int
        d = ctypes.c_double
        L.orc_definetin.argtypes = [i, i, i, P, P, P, P, P, P, P]
        L.orc_setmesh.argtypes = [i, P, P, P, P, P]
        L.orc_getmesh.argtypes = [i, P, P, P, P, P]
        L.orc_updatearea.argtypes = [i, P]
        L.orc_setcurvedmesh.argtypes = [i]
        L.orc_setmaxnb.argtypes = [i]
        L.orc_sethillslopecoeff.argtypes = [i, P, P]
        L.orc_quicksort12.argtypes = [P, i, P]
        L.orc_mfdreceivers.argtypes = [i, i, d, P, d, P, P, P, P, P]
        L.orc_edge_tile.argtypes = [i, d, P, P, P]
        L.orc_fill_tile.argtypes = [i, i, P, P, P, P, P]
        L.orc_graph_nodes.argtypes = [i, P]
        L.orc_combine_edges.argtypes = [i, i, P, P, P, P, P]
        L.orc_fill_edges.argtypes = [i, i, P, i, P, P, P, P]
        L.orc_fill_depressions.argtypes = [i, i, d, P, P, P, P, P]
        L.orc_label_pits.argtypes = [i, d, P, P]
        L.orc_pits_cons.argtypes = [i, i, P, P, P]
        L.orc_fill_dir.argtypes = [i, i, P, P, P, P]
        L.orc_nghb_dir.argtypes = [i, P, P, P, P]
        L.orc_getpitvol.argtypes = [i, i, P, P, P, P, P]
        L.orc_flow_solve.argtypes = [i, i, P, P, P, P]
        L.orc_spl_solve.argtypes = [i, i, P, P, P, P]
        L.orc_mfdrcvrs.argtypes = [i, i, d, P, d, P, P, P, P, P]
        L.orc_epsfill.argtypes = [i, d, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


_state = {"nb": 0}


# --- mesh declaration ------------------------------------------------------
def setcurvedmesh(flag):
    lib().orc_setcurvedmesh(int(flag))


def definetin(coords, cells_nodes, cells_edges, edges_nodes, circumcenter):
    """f2py: ngbid, narea = definetin(coords, cells_nodes, cells_edges,
    edges_nodes, circumcenter) with ``circumcenter`` shaped (3, n)."""
    coords = _f64(coords)
    cn = _i32(cells_nodes)
    ce = _i32(cells_edges)
    en = _i32(edges_nodes)
    cc = _f64(np.asarray(circumcenter).T)          # (n, 3) C-order
    nb, n, m = coords.shape[0], cn.shape[0], en.shape[0]
    ngb = np.empty((nb, 12), dtype=np.int32)
    narea = np.empty(nb, dtype=np.float64)
    lib().orc_definetin(nb, n, m, _p(coords), _p(cn), _p(ce), _p(en), _p(cc), _p(ngb), _p(narea))
    _state["nb"] = nb
    return ngb, narea


def updatearea(narea):
    narea = _f64(narea)
    lib().orc_updatearea(narea.shape[0], _p(narea))


def setmesh(nnb, ngbid, elgt, vdist, area):
    nnb = _i32(nnb)
    ngbid = _i32(ngbid)
    elgt = _f64(elgt)
    vdist = _f64(vdist)
    area = _f64(area)
    nb = nnb.shape[0]
    lib().orc_setmesh(nb, _p(nnb), _p(ngbid), _p(elgt), _p(vdist), _p(area))
    _state["nb"] = nb


def getmesh():
    nb = _state["nb"]
    nnb = np.empty(nb, np.int32)
    ngb = np.empty((nb, 12), np.int32)
    el = np.empty((nb, 12))
    vd = np.empty((nb, 12))
    ar = np.empty(nb)
    lib().orc_getmesh(nb, _p(nnb), _p(ngb), _p(el), _p(vd), _p(ar))
    return nnb, ngb, el, vd, ar


# --- hillslope ----------------------------------------------------------------
def setmaxnb(nb):
    return int(lib().orc_setmaxnb(int(nb)))


def sethillslopecoeff(nb, kd):
    kd = _f64(kd)
    out = np.empty((nb, 13), dtype=np.float64)
    lib().orc_sethillslopecoeff(int(nb), _p(kd), _p(out))
    return out


def jacobiancoeff(h, kd, kp):
    """f2py: dcoeff = jacobiancoeff(h, Kd, Kp) (functions.F90:1423-1467): per
    row the non-linear diffusion Jacobian, column 0 the diagonal and column
    p+1 the neighbour in slot p, faces gated by Kd > 0 on both sides.  numpy
    restatement over the mesh installed by setmesh; the diagonal accumulates
    in slot order as the Fortran loop does."""
    h = _f64(h)
    kd = _f64(kd)
    kp = _f64(kp)
    nnb, ngb, el, vd, ar = getmesh()
    nb = h.shape[0]
    out = np.zeros((nb, 13))
    has = ar > 0
    for p in range(12):
        ok = has & (p < nnb) & (vd[:, p] > 0.0)
        j = np.where(ok, ngb[:, p], 0)
        ck, cn, cpk, cpn = kd, kd[j], kp, kp[j]
        g = ok & (ck > 0.0) & (cn > 0.0)
        if not g.any():
            continue
        a = ar[g]
        c1 = 0.5 * (ck[g] + cn[g] + cpk[g] * (h[g] - h[j][g])) / a
        v1 = c1 * vd[g, p] / el[g, p]
        out[g, 0] = out[g, 0] + v1
        c2 = 0.5 * (ck[g] + cn[g] + cpn[g] * (h[j][g] - h[g])) / a
        v2 = c2 * vd[g, p] / el[g, p]
        out[g, p + 1] = -v2
    return out


# --- receivers ------------------------------------------------------------------
def mfdreceivers(nrcv, exp, elev, sl, gid, powfn=None):
    """f2py: rcv, dist, wgt = mfdreceivers(nrcv, exp, elev, sl, gid)."""
    elev = _f64(elev)
    gid = _i32(gid)
    nb = elev.shape[0]
    rcv = np.empty((nb, nrcv), np.int32)
    dist = np.empty((nb, nrcv))
    wgt = np.empty((nb, nrcv))
    st = lib().orc_mfdreceivers(nb, int(nrcv), float(exp), _p(elev), float(sl), _p(gid),
                                _p(rcv), _p(dist), _p(wgt), powfn)
    if st != 0:
        raise ValueError("mfdreceivers: nrcv must be in 1..12")
    return rcv, dist, wgt


def mfdrcvrs(nrcv, exp, elev, sl, gid, powfn=None):
    """f2py: rcv, dist, wgt = mfdrcvrs(nrcv, exp, elev, sl, gid); [nb, 12]
    (functions.F90:1673-1785)."""
    elev = _f64(elev)
    gid = _i32(gid)
    nb = elev.shape[0]
    rcv = np.empty((nb, 12), np.int32)
    dist = np.empty((nb, 12))
    wgt = np.empty((nb, 12))
    st = lib().orc_mfdrcvrs(nb, int(nrcv), float(exp), _p(elev), float(sl), _p(gid), _p(rcv), _p(dist),
                            _p(wgt), powfn)
    if st != 0:
        raise ValueError("mfdrcvrs: nrcv must be in 1..12")
    return rcv, dist, wgt


def epsfill(sl, elev):
    """f2py: fillz = epsfill(sl, elev) (functions.F90:2633-2697)."""
    elev = _f64(elev)
    fillz = np.empty_like(elev)
    if lib().orc_epsfill(elev.shape[0], float(sl), _p(elev), _p(fillz)) != 0:
        raise MemoryError("epsfill")
    return fillz


def quicksort12(values, indices):
    """Run the reference quicksort (functions.F90:683-762) on up to 12 values."""
    kk = len(values)
    a = np.zeros(12)
    a[:kk] = values
    ix = np.zeros(12, np.int32)
    ix[:kk] = indices
    lib().orc_quicksort12(_p(a), kk, _p(ix))
    return a[:kk].copy(), ix[:kk].copy()


# --- pit filling --------------------------------------------------------------------
def edge_tile(lvl, border, elev):
    border = _i32(border)
    elev = _f64(elev)
    nb = border.shape[0]
    out = np.empty(nb, np.int32)
    lib().orc_edge_tile(nb, float(lvl), _p(border), _p(elev), _p(out))
    return out


def fill_tile(edge, elev, inids):
    edge = _i32(edge).reshape(-1, 2)
    elev = _f64(elev)
    inids = _i32(inids)
    nb = elev.shape[0]
    fillz = np.empty(nb)
    labels = np.empty(nb, np.int32)
    gnb = lib().orc_fill_tile(edge.shape[0], nb, _p(edge), _p(elev), _p(inids), _p(fillz), _p(labels))
    return fillz, labels, int(gnb)


def graph_nodes(graphnb):
    out = np.empty((int(graphnb), 4))
    lib().orc_graph_nodes(int(graphnb), _p(out))
    return out


def combine_edges(elev, labels, ins, outs):
    elev = _f64(elev)
    labels = _i32(labels)
    ins = _i32(ins)
    outs = _i32(outs)
    m, n = elev.shape[0], ins.shape[0]
    newgraph = np.zeros((n * 12, 4))
    gnb = lib().orc_combine_edges(m, n, _p(elev), _p(labels), _p(ins), _p(outs), _p(newgraph))
    return newgraph, int(gnb)


def fill_edges(nb, cgraph, maxnghbs):
    cgraph = _f64(cgraph).reshape(-1, 5)
    nb = int(nb)
    nelev = np.empty(nb)
    srank = np.empty(nb, np.int32)
    snodes = np.empty(nb, np.int32)
    sid = np.empty(nb, np.int32)
    st = lib().orc_fill_edges(nb, cgraph.shape[0], _p(cgraph), int(maxnghbs), _p(nelev),
                              _p(srank), _p(snodes), _p(sid))
    if st != 0:
        raise IndexError("fill_edges: graph label or neighbour count out of range (%d)" % st)
    return nelev, srank, snodes, sid


def fill_depressions(lvl, dem, fillp, wsh, ggraph):
    dem = _f64(dem)
    fillp = _f64(fillp)
    wsh = _i32(wsh)
    ggraph = _f64(ggraph)
    out = np.empty(dem.shape[0])
    lib().orc_fill_depressions(dem.shape[0], ggraph.shape[0], float(lvl), _p(dem), _p(fillp),
                               _p(wsh), _p(ggraph), _p(out))
    return out


def label_pits(lvl, fill):
    fill = _f64(fill)
    out = np.empty(fill.shape[0], np.int32)
    lib().orc_label_pits(fill.shape[0], float(lvl), _p(fill), _p(out))
    return out


def pits_cons(pitids, pitnb):
    pitids = _i32(pitids)
    pitnb = _i32(pitnb)
    out = np.empty(pitids.shape[0], np.int32)
    lib().orc_pits_cons(pitids.shape[0], pitnb.shape[0], _p(pitids), _p(pitnb), _p(out))
    return out


def fill_dir(spill, pitids, h):
    spill = _i32(spill)
    pitids = _i32(pitids)
    h = _f64(h)
    out = np.empty(pitids.shape[0], np.int32)
    lib().orc_fill_dir(spill.shape[0], pitids.shape[0], _p(spill), _p(pitids), _p(h), _p(out))
    return out


def nghb_dir(pitids, h, ptdir):
    pitids = _i32(pitids)
    h = _f64(h)
    ptdir = _i32(ptdir)
    out = np.empty(pitids.shape[0], np.int32)
    lib().orc_nghb_dir(pitids.shape[0], _p(pitids), _p(h), _p(ptdir), _p(out))
    return out


def getpitvol(hlvl, elev, pit, id):
    hlvl = _f64(hlvl).reshape(-1, 4)
    elev = _f64(elev)
    pit = _i32(pit)
    id = _i32(id)
    vol = np.empty((hlvl.shape[0], 4))
    lib().orc_getpitvol(elev.shape[0], hlvl.shape[0], _p(hlvl), _p(elev), _p(pit), _p(id), _p(vol))
    return vol


# --- exact solves ---------------------------------------------------------------
def flow_solve(rcv, wgt, b):
    """Exact solve of (I - W^T) q = b; returns (q, n_unordered)."""
    rcv = _i32(rcv)
    wgt = _f64(wgt)
    b = _f64(b)
    nb, R = rcv.shape
    q = np.zeros(nb)
    left = lib().orc_flow_solve(nb, R, _p(rcv), _p(wgt), _p(b), _p(q))
    return q, int(left)


def spl_solve(rcv, c, hold):
    rcv = _i32(rcv)
    c = _f64(c)
    hold = _f64(hold)
    nb, R = rcv.shape
    h = np.zeros(nb)
    left = lib().orc_spl_solve(nb, R, _p(rcv), _p(c), _p(hold), _p(h))
    return h, int(left)
