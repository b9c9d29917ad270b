import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["incising", "sphere3766", "planar2k", "ico2562"]
# transport-limited SPL (G > 0), compared step by step from the reference's state
GOLDEN_G_CASES = ["ico2562_G05", "planar2k_G1"]
# continental sediment routing and deposition (nodep off)
GOLDEN_SED_CASES = ["incising_sed", "planar2k_sed", "ico2562_sed", "planar2k_lake"]
# marine deposition (seadepo on): oracle only, the device path is not built
GOLDEN_MARINE_CASES = ["planar2k_marine", "ico2562_marine", "ico2562_marine_G"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    import numpy as np
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: d[k] for k in d.files}


def golden_params(g):
    import numpy as np
    p = {k[2:]: (g[k].item() if g[k].shape == () else g[k]) for k in g if k.startswith("p_")}
    p["rain"] = g["rain"]
    p["upsub"] = g["upsub"] if g["upsub"].size else None
    return p


def golden_mesh(g):
    import numpy as np
    return {
        "coords": g["v"], "cells": g["c"], "nb": len(g["z"]), "flat": bool(g["flat"]),
        "nnb": g["nnb"], "ngb": g["ngb"], "elgt": g["elgt"], "vdist": g["vdist"], "farea": g["farea"],
        "larea": g["larea"], "maxarea": float(g["larea"].max()), "outlet": g["outlet"].astype(np.int64),
        "open_nodes": g["open_nodes"].astype(np.int64), "borders": g["outlet"].astype(np.int64),
    }
