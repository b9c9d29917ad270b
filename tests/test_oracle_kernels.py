"""Oracle restatements checked against each other and against numpy, on CPU:
jacobiancoeff (functions.F90:1423-1467) reduces to sethillslopecoeff
(functions.F90:901-938, pinned through the golden fixtures) for a uniform
diffusivity and Kp = 0, closes faces where either side has no diffusivity, and
its Kp term follows the Fortran expression."""
import numpy as np

from conftest import golden_mesh, load_golden


def _mesh():
    from oracle import mesh as OM
    g = load_golden("planar2k")
    m = golden_mesh(g)
    OM.load_mesh(m)
    return g, m


def test_jacobiancoeff_matches_hillslope_coefficients():
    from oracle import fortran as F
    g, m = _mesh()
    n = len(g["z"])
    kd = np.full(n, 3.0)
    d = F.jacobiancoeff(g["z"], kd, np.zeros(n))
    hc = F.sethillslopecoeff(n, kd)
    assert np.array_equal(d[:, 0] + 1.0, hc[:, 0])
    assert np.array_equal(d[:, 1:], hc[:, 1:])


def test_jacobiancoeff_gates_faces_without_diffusivity():
    from oracle import fortran as F
    g, m = _mesh()
    n = len(g["z"])
    rng = np.random.default_rng(5)
    kd = np.where(rng.random(n) < 0.5, 2.0, 0.0)
    d = F.jacobiancoeff(g["z"], kd, np.zeros(n))
    ngb = np.asarray(m["ngb"])
    for k in range(0, n, 37):
        for s in range(int(m["nnb"][k])):
            j = ngb[k, s]
            if kd[k] == 0.0 or kd[j] == 0.0:
                assert d[k, s + 1] == 0.0
    assert np.all(d[kd == 0.0, 0] == 0.0)


def test_jacobiancoeff_derivative_term():
    from oracle import fortran as F
    g, m = _mesh()
    n = len(g["z"])
    h = np.asarray(g["z"], float)
    kd = np.full(n, 1.5)
    kp = np.full(n, 0.25)
    d = F.jacobiancoeff(h, kd, kp)
    ngb, el, vd, ar = np.asarray(m["ngb"]), np.asarray(m["elgt"]), np.asarray(m["vdist"]), np.asarray(m["farea"])
    k = int(np.argmax(ar))
    diag = 0.0
    for s in range(int(m["nnb"][k])):
        if vd[k, s] > 0.0:
            j = ngb[k, s]
            c = 0.5 * (kd[k] + kd[j] + kp[k] * (h[k] - h[j])) / ar[k]
            diag = diag + c * vd[k, s] / el[k, s]
            c2 = 0.5 * (kd[k] + kd[j] + kp[j] * (h[j] - h[k])) / ar[k]
            assert d[k, s + 1] == -(c2 * vd[k, s] / el[k, s])
    assert d[k, 0] == diag
