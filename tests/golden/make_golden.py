"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run where a goSPL checkout is available, named by --ref or the GOSPL_REF
environment variable (no default):

    python tests/golden/make_golden.py --ref /path/to/gospl [case ...]

For each case it (1) checks the oracle's restatement of the numpy Voronoi
helpers against the reference's own ``gospl/mesher/meshfunc.py``, (2) runs the
reference's Python orchestration (flowAccumulation, erodepSPL, getHillslope;
see refharness.py) for a few steps on one rank, and (3) writes inputs, the FV
mesh and the per-step outputs to ``<case>.npz``.  The fixtures are what the
CPU tests compare the oracle against; the GPU tests compare the CUDA path with
the oracle.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

REF = os.environ.get("GOSPL_REF")


def _take_ref_argument():
    """--ref PATH on the command line overrides GOSPL_REF; one of them must
    name the goSPL checkout."""
    global REF
    if "--ref" in sys.argv:
        k = sys.argv.index("--ref")
        REF = sys.argv[k + 1]
        del sys.argv[k:k + 2]
    if not REF:
        sys.exit("name the goSPL checkout with --ref PATH or the GOSPL_REF environment variable")

SNAP = ("h", "cumED", "EbLocal", "FAL", "fillFAL", "lFill", "pitIDs", "flatDirs", "waterFilled",
        "rcvIDi", "wghtVali", "distRcvi", "lsink", "lsinki", "pitParams", "pitInfo", "filled_lvl",
        "filled_vol")


def snapshot(m, ref):
    out = {}
    if not m.nodep:
        # continental deposition: routed sediment flux (m3/yr)
        out["vSed"] = (m.vSedLocal.getArray().copy() if ref else m.vSed.copy()) if hasattr(m, "vSed") \
            else np.zeros(len(m.larea))
    get = (lambda v: v.getArray().copy()) if ref else (lambda v: np.array(v, copy=True))
    for k in SNAP:
        if k in ("h",):
            out[k] = get(m.hLocal) if ref else m.h.copy()
        elif k in ("cumED", "EbLocal", "FAL", "fillFAL") and ref:
            out[k] = getattr(m, k).getArray().copy()
        else:
            out[k] = np.array(getattr(m, k), copy=True)
    return out


def cases():
    from gospl_b200 import synthetic as S
    out = []
    d = np.load(os.path.join(REF, "tests", "fixtures", "incising.npz"))
    out.append(("incising", d["v"], d["c"], d["z"],
                dict(dt=100.0, tEnd=300.0, flowDir=3, K=4.0e-6, d=0.0, m=0.5, Cda=0.01, Cdm=0.2,
                     sealevel=-100.0, bc="oooo", rain=np.ones(len(d["z"])), upsub=None), 3))
    d = np.load(os.path.join(REF, "tests", "fixtures", "mesh.npz"))
    out.append(("sphere3766", d["v"], d["c"].astype(np.int32), d["z"],
                dict(dt=10.0, tEnd=100.0, flowDir=2, K=4.0e-6, d=0.0, m=0.5, Cda=0.01, Cdm=0.2,
                     sealevel=-100.0, bc="oooo", rain=np.ones(len(d["z"])), upsub=None), 2))
    c, f, z, rain, up, p = S.planar_config(n=2000, side=30.0e3, seed=7)
    p = dict(p, rain=rain, upsub=up, tEnd=10 * p["dt"])
    out.append(("planar2k", c, f, z, p, 3))
    c, f = S.icosphere(4)
    z = S.rescale(S.sh_field(c, 48, 11), -4000.0, 3000.0)
    g = S.sh_field(c, 16, 12)
    rain = np.exp(0.5 * (g - g.mean()) / g.std())
    up = S.belt_uplift(c, 13)
    p = dict(dt=1.0e4, tEnd=1.0e5, flowDir=3, K=5.0e-7, d=0.0, m=0.5, Cda=0.05, Cdm=0.05,
             sealevel=0.0, bc="oooo", rain=rain, upsub=up)
    out.append(("ico2562", c, f, z, p, 3))
    # transport-limited SPL (G > 0): the coupled erosion-deposition system
    out.append(("ico2562_G05", c, f, z, dict(p, G=0.5), 3))
    c, f, z, rain, up, p = S.planar_config(n=2000, side=30.0e3, seed=7)
    p = dict(p, rain=rain, upsub=up, tEnd=10 * p["dt"], G=1.0)
    out.append(("planar2k_G1", c, f, z, p, 3))
    # continental sediment routing and deposition in depressions (nodep off,
    # no marine deposition)
    d = np.load(os.path.join(REF, "tests", "fixtures", "incising.npz"))
    out.append(("incising_sed", d["v"], d["c"], d["z"],
                dict(dt=100.0, tEnd=300.0, flowDir=3, K=4.0e-6, d=0.0, m=0.5, Cda=0.01, Cdm=0.2,
                     sealevel=-100.0, bc="oooo", rain=np.ones(len(d["z"])), upsub=None, nodep=False), 3))
    c, f, z, rain, up, p = S.planar_config(n=2000, side=30.0e3, seed=7)
    p = dict(p, rain=rain, upsub=up, tEnd=10 * p["dt"], nodep=False)
    out.append(("planar2k_sed", c, f, z, p, 3))
    c, f = S.icosphere(4)
    z = S.rescale(S.sh_field(c, 48, 11), -4000.0, 3000.0)
    g = S.sh_field(c, 16, 12)
    rain = np.exp(0.5 * (g - g.mean()) / g.std())
    up = S.belt_uplift(c, 13)
    p = dict(dt=1.0e4, tEnd=1.0e5, flowDir=3, K=5.0e-7, d=0.0, m=0.5, Cda=0.05, Cdm=0.05,
             sealevel=0.0, bc="oooo", rain=rain, upsub=up, nodep=False, nlPitVolume=1.0e30)
    out.append(("ico2562_sed", c, f, z, p, 3))
    # lake deposits smoothed by non-linear diffusion (every partly filled
    # depression takes that path; Picard solver)
    c, f, z, rain, up, p = S.planar_config(n=2000, side=30.0e3, seed=7)
    p = dict(p, rain=rain, upsub=up, tEnd=10 * p["dt"], nodep=False, nlPitVolume=0.0, nlPitDepth=0.0,
             marineSolver="picard", picardSub=2, picardIts=2)
    out.append(("planar2k_lake", c, f, z, p, 3))
    # marine deposition (seadepo on, Picard solver for the marine diffusion):
    # a flat domain with its sea level at the 15th percentile of the relief,
    # and the sphere with its ocean
    c, f, z, rain, up, p = S.planar_config(n=2000, side=30.0e3, seed=7)
    p = dict(p, rain=rain, upsub=up, tEnd=10 * p["dt"], nodep=False, seadepo=True, marineSolver="picard",
             picardSub=2, picardIts=2, sealevel=float(np.percentile(z, 15)))
    out.append(("planar2k_marine", c, f, z, p, 3))
    c, f = S.icosphere(4)
    z = S.rescale(S.sh_field(c, 48, 11), -4000.0, 3000.0)
    g = S.sh_field(c, 16, 12)
    rain = np.exp(0.5 * (g - g.mean()) / g.std())
    up = S.belt_uplift(c, 13)
    p = dict(dt=1.0e4, tEnd=1.0e5, flowDir=3, K=5.0e-7, d=0.0, m=0.5, Cda=0.05, Cdm=0.05,
             sealevel=0.0, bc="oooo", rain=rain, upsub=up, nodep=False, seadepo=True, marineSolver="picard",
             picardSub=2, picardIts=2)
    out.append(("ico2562_marine", c, f, z, p, 3))
    # marine deposition with the transport-limited marine system (Gmar > 0)
    out.append(("ico2562_marine_G", c, f, z, dict(p, Gmar=0.5), 3))
    return out


def main():
    import refharness as RH
    from oracle import mesh as OM
    from oracle import model as OMod

    mf = RH.load_meshfunc(REF)
    RefModel = RH.make_model_class(REF)
    only = set(sys.argv[1:])
    for name, coords, cells, z, params, nsteps in cases():
        if only and name not in only:
            continue
        cells = np.asarray(cells, dtype=np.int32)
        # (1) meshfunc restatement vs the reference's meshfunc
        vb = mf.VoroBuild()
        vb.initVoronoi(coords, cells)
        cv_ref = np.abs(vb.control_volumes)
        vb.create_edges()
        vi = OM.voronoi_inputs(coords, cells)
        assert np.array_equal(vb.edges["nodes"], vi["edges"]), name
        assert np.array_equal(vb.cells["edges"], vi["cells_edges"]), name
        assert np.array_equal(vb.cell_circumcenters, vi["cc"]), name
        assert np.array_equal(cv_ref, np.abs(vi["control_volumes"])), name
        mesh = OM.build_mesh(coords, cells, params["bc"])
        # (2) reference orchestration
        ref = RefModel(mesh, z, params)
        snaps = [snapshot(ref, True)]
        for _ in range(nsteps):
            ref.step()
            snaps.append(snapshot(ref, True))
        # oracle model, for the record
        om = OMod.OracleModel(coords, cells, z, params, mesh=mesh)
        osn = [snapshot(om, False)]
        for _ in range(nsteps):
            om.step()
            osn.append(snapshot(om, False))
        worst = {}
        for s_ref, s_or in zip(snaps, osn):
            for k in s_ref:
                a, b = np.asarray(s_ref[k], float), np.asarray(s_or[k], float)
                if a.shape != b.shape:
                    worst[k] = "shape %s vs %s" % (a.shape, b.shape)
                    continue
                sc = max(np.abs(a).max(), 1e-300) if a.size else 1.0
                worst[k] = max(worst.get(k, 0.0), float(np.abs(a - b).max() / sc) if a.size else 0.0)
        print(name, len(z), "oracle-vs-reference max rel diff:",
              {k: (v if isinstance(v, str) else "%.1e" % v) for k, v in worst.items()})
        # (3) fixture
        arrs = dict(v=coords, c=cells, z=z, rain=params["rain"],
                    upsub=(params["upsub"] if params["upsub"] is not None else np.zeros(0)),
                    nnb=mesh["nnb"], ngb=mesh["ngb"], elgt=mesh["elgt"], vdist=mesh["vdist"],
                    farea=mesh["farea"], larea=mesh["larea"], outlet=mesh["outlet"],
                    open_nodes=mesh["open_nodes"], flat=np.array(mesh["flat"]), nsteps=np.array(nsteps))
        for k in ("dt", "tEnd", "flowDir", "K", "d", "m", "Cda", "Cdm", "sealevel"):
            arrs["p_" + k] = np.array(params[k])
        arrs["p_bc"] = np.array(params["bc"])
        for k in ("G", "nodep", "nlPitVolume", "nlPitDepth", "marineSolver", "picardSub", "picardIts", "seadepo",
                  "Gmar"):
            if k in params:
                arrs["p_" + k] = np.array(params[k])
        for i, s in enumerate(snaps):
            for k, v in s.items():
                arrs["s%d_%s" % (i, k)] = np.asarray(v)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
        print("  wrote", name + ".npz", os.path.getsize(os.path.join(HERE, name + ".npz")) // 1024, "KB")


if __name__ == "__main__":
    _take_ref_argument()
    main()
