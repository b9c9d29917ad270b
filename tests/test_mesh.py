"""Product FV mesh builder against the oracle's definetin restatement."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_fv_mesh_matches_oracle_geometry(case):
    from gospl_b200.mesh import FVMesh
    g = load_golden(case)
    m = FVMesh(g["v"], g["c"], str(g["p_bc"]))
    assert np.array_equal(m.nnb, g["nnb"])
    assert np.array_equal(m.ngb, g["ngb"])
    assert np.array_equal(m.outlet, g["outlet"])
    assert np.array_equal(m.open_nodes, g["open_nodes"])
    planar = bool(g["flat"])
    for k in ("elgt", "vdist", "farea", "larea"):
        a, b = getattr(m, k), g[k]
        if planar:
            assert np.array_equal(a, b), k          # same operations, same order
        else:
            # spherical trig: numpy's vectorised sin/acos vs libm, amplified by
            # the spherical-excess area formula
            assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), k
