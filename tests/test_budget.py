"""Sediment budget of goSPL's continental routing, on the oracle (CPU).

goSPL's sedChange (sedplex.py:103-522) moves the volume eroded by the step's
SPL through flow solves and depression bookkeeping.  The oracle records, pass
by pass, where every cubic metre goes: depressions (retained), stray sinks
(kept on a closed domain, dropped otherwise), open outlets, the sea, and the
volume goSPL's own rules drop (excess written at no spill node, placed excess
left unrouted under half the largest cell area, inflow equal to the remaining
volume).  The eroded volume minus every destination must vanish to rounding
(1e-12 of the eroded volume), on closed, open and mixed domains and on the
sediment fixtures made by the reference's own sedplex.py.  A planted error of
one part in 1e9 in one routing solve must break the closure.
"""
import numpy as np
import pytest

from conftest import GOLDEN_SED_CASES, golden_mesh, golden_params, load_golden


def _planar(bc, n=3000, seed=3):
    from gospl_b200 import synthetic as S
    coords, cells, z, rain, up, p = S.planar_config(n=n, side=30.0e3, seed=seed)
    p = dict(p, rain=rain, upsub=None if bc == "wwww" else up, nodep=False, bc=bc, tEnd=10 * p["dt"])
    return coords, cells, z, p


def _check(b, tag):
    E = b["eroded"]
    assert E > 0.0, tag
    assert abs(b["closure"]) <= 1e-12 * E, "%s closure %g of the eroded volume" % (tag, b["closure"] / E)
    assert abs(b["pit_sinks"] - b["inflow"]) <= 1e-12 * E, tag
    assert abs(b["inflow"] - (b["retained"] + b["excess"] + b["zero_excess"])) <= 1e-12 * E, tag
    for k in ("retained", "kept", "dropped", "outlets", "sea", "unplaced", "unrouted"):
        assert b[k] >= -1e-12 * E, (tag, k)


@pytest.mark.parametrize("bc", ["wwww", "ffff", "wfwf"])
def test_oracle_budget_closes_on_planar_domains(bc):
    from oracle.model import OracleModel
    om = OracleModel(*_planar(bc))
    for s in range(3):
        om.step()
        b = om.sed_budget
        _check(b, "%s step %d" % (bc, s))
        if bc == "wwww":
            # no outlet, no sea: nothing leaves through a boundary
            assert b["outlets"] == 0.0 and b["sea"] == 0.0 and b["dropped"] == 0.0
        else:
            assert b["outlets"] > 0.0 and b["kept"] == 0.0


@pytest.mark.parametrize("case", GOLDEN_SED_CASES)
def test_oracle_budget_closes_on_reference_fixtures(case):
    from oracle.model import OracleModel
    g = load_golden(case)
    om = OracleModel(g["v"], g["c"], g["z"], golden_params(g), mesh=golden_mesh(g))
    for s in range(int(g["nsteps"])):
        om.step()
        _check(om.sed_budget, "%s step %d" % (case, s))


def test_budget_detects_a_planted_routing_error():
    """One routing solve made 1e-9 too large (planted in the oracle) breaks
    the closure, so the 1e-12 bound has teeth."""
    from oracle.model import OracleModel
    om = OracleModel(*_planar("wfwf"))
    om.step()
    _check(om.sed_budget, "clean")
    solve = om._flow_solve

    def leaky(b):
        return solve(b) * (1.0 + 1.0e-9)

    om._flow_solve = leaky
    om.step()
    b = om.sed_budget
    assert b["routed"] > 0.0, "the planted error needs a routing solve"
    assert abs(b["closure"]) > 1e-12 * b["eroded"]
