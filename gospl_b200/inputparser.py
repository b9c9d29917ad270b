"""goSPL YAML input for this library's path.

Reads the keys of a goSPL input file that the per-step surface-process path
uses, with goSPL's names, defaults and errors (gospl/tools/inputparser.py):

* ``domain``: ``npdata: [file, coords_key, cells_key, elev_key]`` (the
  ``.npz`` mesh, :263-266), ``flowdir`` (default 8, :189), ``bc`` (four of
  ``o f w c``, legacy ``0``/``1`` -> ``o``/``f``, :208-246), ``fast``, ``nodep``
  and ``seadepo`` (:289-300; continental deposition runs unless ``nodep``,
  marine deposition when ``seadepo`` (default on), built for
  ``marineSolver: picard``);
* ``time``: ``start``, ``end``, ``dt`` required, ``tout`` (:343-404, clamped
  to [dt, end - start] as :413-429 does), ``rstep`` (restart, :411);
* ``output``: ``dir`` (output), ``makedir`` (False), ``compression`` (gzip)
  (:2096-2117);
* ``spl``: ``K``, ``d`` (0), ``m`` (0.5), ``G`` (0) (:454-496);
* ``diffusion``: ``hillslopeKa``, ``hillslopeKm``, ``oFill`` (-6000) (:498-545),
  ``nlPitVolume`` (1e9), ``nlPitDepth`` (100), ``nonlinKm``/``nlPitK`` (10),
  ``pitInletBias`` (0.10; 0.50 without the section), ``marineSolver`` (ts),
  ``picardSub`` (10), ``picardIts`` (2), ``clinSlp`` (1e-6, at least 1e-6),
  ``Gmar`` (0), ``offshore`` (1e7 m) (:546-593);
* ``sea``: ``position`` (default 0, :710-787);
* ``climate``: events with ``start`` and ``uniform`` or ``map: [file, key]``
  (:1352-1520);
* ``tectonics``: events with ``start``, ``end`` and ``upsub: [file, key]``
  (:826-942).

Paths are taken as given (relative to the working directory, as goSPL does),
then relative to the YAML file.  Keys of other goSPL subsystems (sediment,
stratigraphy, flexure, ice, orography) are ignored; options that would
change this path's arithmetic and that the library does not implement
(sea-level curves, time-varying climate or tectonic events, horizontal
tectonics, marine deposition with the TS solver) raise
``ValueError``.
"""
import os

import numpy as np


def _path(name, base):
    if os.path.exists(name):
        return name
    alt = os.path.join(base, name)
    if os.path.exists(alt):
        return alt
    raise IOError("The numpy dataset is not found: {}".format(name))


def _npz(spec, base, what):
    if not isinstance(spec, (list, tuple)) or len(spec) < 2:
        raise ValueError("%s must be [file, key]" % what)
    data = np.load(_path(str(spec[0]) + ".npz", base))
    if spec[1] not in data.files:
        raise KeyError("Field {} is not in {}.npz".format(spec[1], spec[0]))
    return np.asarray(data[spec[1]], np.float64)


def parse_bc(bc):
    """goSPL's boundary string: 4 chars of o/f/w/c in N,E,S,W order."""
    bc = str(bc).replace("0", "o").replace("1", "f")
    if len(bc) != 4 or any(c not in "ofwc" for c in bc):
        raise ValueError("domain.bc must be 4 characters from {'o' open, 'f' fixed, 'w' wall, "
                         "'c' cyclic} (legacy '0'/'1' accepted) in [North, East, South, West] order; "
                         "got '%s'." % bc)
    n, e, s, w = bc
    if (n == "c") != (s == "c") or (e == "c") != (w == "c"):
        raise ValueError("Cyclic (periodic) boundaries must be paired (got bc='%s')." % bc)
    if n == "c" and e == "c":
        raise ValueError("At most one pair of edges may be cyclic; got bc='%s'." % bc)
    return bc


def read_input(filename):
    """Returns (coords [N,3], cells [M,3], elev [N], params) for ``Model``."""
    import yaml

    with open(filename) as f:
        inp = yaml.safe_load(f)
    base = os.path.dirname(os.path.abspath(filename))
    if "domain" not in inp:
        raise KeyError("Key domain is required in the input file!")
    dom = inp["domain"]
    if "npdata" not in dom:
        raise KeyError("Compressed numpy dataset definition is not defined!")
    info = dom["npdata"]
    mesh = np.load(_path(str(info[0]) + ".npz", base))
    coords = np.asarray(mesh[info[1]], np.float64)
    cells = np.asarray(mesh[info[2]], np.int64)
    elev = np.asarray(mesh[info[3]], np.float64).ravel()
    n = len(coords)
    p = {"flowDir": int(dom.get("flowdir", 8)), "bc": parse_bc(dom.get("bc", "oooo")),
         "fast": bool(dom.get("fast", False)), "nodep": bool(dom.get("nodep", False)),
         "seadepo": bool(dom.get("seadepo", True))}

    if "time" not in inp:
        raise KeyError("Key time is required in the input file!")
    t = inp["time"]
    for k in ("start", "end", "dt"):
        if k not in t:
            raise KeyError("Key '%s' is required in the 'time' declaration" % k)
    p["tStart"], p["tEnd"], p["dt"] = float(t["start"]), float(t["end"]), float(t["dt"])
    if p["tEnd"] <= p["tStart"]:
        raise ValueError("Simulation end/start times do not make any sense!")
    p["tout"] = float(t.get("tout", p["tEnd"] - p["tStart"]))
    p["rStep"] = int(t.get("rstep", 0))                       # :411
    if p["tStart"] + p["tout"] > p["tEnd"]:                   # :413-420
        p["tout"] = p["tEnd"] - p["tStart"]
    if p["tout"] < p["dt"]:                                   # :422-429
        p["tout"] = p["dt"]

    spl = inp.get("spl")
    if spl is not None:
        if "K" not in spl:
            raise KeyError("Key 'K' is required in the 'spl' declaration")
        p["K"], p["d"], p["m"] = float(spl["K"]), float(spl.get("d", 0.0)), float(spl.get("m", 0.5))
        p["G"] = float(spl.get("G", 0.0))
    else:
        p["K"], p["d"], p["m"], p["G"] = 1.0e-12, 0.0, 0.5, 0.0

    hill = inp.get("diffusion")
    if hill is not None:
        p["Cda"] = float(hill["hillslopeKa"])
        p["Cdm"] = float(hill["hillslopeKm"])
        p["oFill"] = float(hill.get("oFill", -6000.0))
        p["nlPitVolume"] = float(hill.get("nlPitVolume", 1.0e9))
        p["nlPitDepth"] = float(hill.get("nlPitDepth", 100.0))
        p["nlPitK"] = float(hill.get("nlPitK", hill.get("nonlinKm", 10.0)))
        p["pitInletBias"] = float(hill.get("pitInletBias", 0.10))
        p["marineSolver"] = str(hill.get("marineSolver", "ts")).lower()
        p["picardSub"] = int(hill.get("picardSub", 10))
        p["picardIts"] = int(hill.get("picardIts", 2))
        p["nonlinKm"] = float(hill.get("nonlinKm", 10.0))      # :554-558
        p["clinSlp"] = max(1.0e-6, float(hill.get("clinSlp", 1.0e-6)))
        p["Gmar"] = float(hill.get("Gmar", 0.0))
        p["offshore"] = float(hill.get("offshore", 100.0e5))
    else:
        p["Cda"], p["Cdm"], p["oFill"] = 0.0, 0.0, -6000.0
        p["nlPitVolume"], p["nlPitDepth"] = 1.0e9, 100.0
        p["nlPitK"], p["pitInletBias"], p["marineSolver"] = 10.0, 0.50, "ts"
        p["picardSub"], p["picardIts"] = 10, 2
        p["nonlinKm"], p["clinSlp"], p["Gmar"], p["offshore"] = 10.0, 1.0e-6, 0.0, 100.0e5

    if not p["nodep"] and p["seadepo"] and p["marineSolver"] != "picard":
        raise ValueError("marine deposition (domain.seadepo) is built for diffusion.marineSolver: picard; set it, "
                         "or domain.seadepo: False (continental deposition only)")

    sea = inp.get("sea") or {}
    if "curve" in sea:
        raise ValueError("sea-level curves are not implemented by gospl_b200 (use sea.position)")
    p["sealevel"] = float(sea.get("position", 0.0))

    rain = np.zeros(n)
    clim = inp.get("climate")
    if clim:
        ev = sorted(clim, key=lambda e: e["start"])
        if len(ev) > 1:
            raise ValueError("time-varying climate events are not implemented by gospl_b200")
        e = ev[0]
        if "map" in e and e["map"] is not None:
            rain = _npz(e["map"], base, "climate map").ravel()
        elif "uniform" in e and e["uniform"] is not None:
            rain = np.full(n, float(e["uniform"]))
    p["rain"] = rain

    p["upsub"] = None
    tec = inp.get("tectonics")
    if tec:
        ev = sorted(tec, key=lambda e: e["start"])
        if len(ev) > 1:
            raise ValueError("time-varying tectonic events are not implemented by gospl_b200")
        e = ev[0]
        if "start" not in e or "end" not in e:
            raise ValueError("Tectonic event 0 needs start and end")
        if e.get("hdisp") is not None or e.get("zfit") is not None:
            raise ValueError("horizontal tectonics (hdisp/zfit) are not implemented by gospl_b200")
        if e.get("upsub") is not None:
            p["upsub"] = _npz(e["upsub"], base, "tectonics upsub").ravel()

    # output (:2096-2117): directory, numbered copies, HDF5 compression; a
    # restart reuses the directory
    out = inp.get("output") or {}
    p["outputDir"] = str(out.get("dir", "output"))
    p["makedir"] = bool(out.get("makedir", False)) and p["rStep"] == 0
    p["compression"] = out.get("compression", "gzip")
    p["finput"] = filename
    return coords, cells, elev, p
