"""Hand-written adjoint (gs_adjoint_step, gospl_b200.adjoint) against central
finite differences of the full forward on a planar landscape with
depressions (lake cascade active), for per-vertex erodibility, uplift,
rainfall and initial elevation, with checkpointed replay over two segments."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup():
    import torch
    from gospl_b200 import synthetic as S
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model

    dev = torch.device("cuda", torch.cuda.current_device())
    n_target = 2000
    side = 537.0 * np.sqrt(n_target * np.sqrt(3) / 2)
    coords, cells, onb = S.planar_hex_mesh(n_target, side, seed=5)
    z = S.rescale(S.fractal_field(coords[:, :2], side, 6), 0.0, 50.0)
    z[onb] = 0.0
    n = len(z)
    K = np.exp(S.rescale(S.fractal_field(coords[:, :2], side, 8, beta=4.0), -14.0, -11.0))
    U = np.full(n, 5e-4)
    U[onb] = 0.0
    rain = np.ones(n)
    params = dict(dt=1000.0, tStart=0.0, tEnd=1e30, flowDir=3, K=K, d=0.0, m=0.5, Cda=0.1, Cdm=0.1,
                  sealevel=-100.0, oFill=-6000.0, bc="ffff", rain=rain, upsub=U)
    model = Model(coords=coords, cells=cells, elev=z, params=params, mesh=FVMesh(coords, cells, "ffff", device=dev),
                  device=dev)
    f64 = dict(dtype=torch.float64, device=dev)
    return model, onb, [torch.tensor(a, **f64) for a in (K, U, rain, z)]


def test_adjoint_matches_central_differences():
    import torch
    from gospl_b200 import adjoint as A

    model, onb, (K, U, rain, h0) = _setup()
    nsteps, every = 6, 3
    rng = np.random.default_rng(7)
    hT, ck = A.run(model, K, U, rain, h0, nsteps, every)
    assert model.stats["flow"]["npits"] > 0 and model.stats["flow"]["cascade_solves"] > 0
    target = hT + 1e-3 * torch.tensor(rng.standard_normal(len(hT)), dtype=torch.float64, device=hT.device)

    def J(args):
        h, _ = A.run(model, *args, nsteps, every)
        return float(((h - target) ** 2).sum())

    gK, gU, grain, gh0 = A.backward(model, K, U, rain, ck, nsteps, every, 2 * (hT - target))
    base = [K, U, rain, h0]
    idx = rng.choice(np.where(~onb)[0], 12, replace=False)
    for k, g in enumerate((gK, gU, grain, gh0)):
        ad, fd = [], []
        for i in idx:
            eps = 1e-5 * max(abs(float(base[k][i])), 1e-3 if k == 3 else 1e-12)
            p_, m_ = list(base), list(base)
            p_[k] = base[k].clone()
            p_[k][i] += eps
            m_[k] = base[k].clone()
            m_[k][i] -= eps
            fd.append((J(p_) - J(m_)) / (2 * eps))
            ad.append(float(g[i]))
        ad, fd = np.array(ad), np.array(fd)
        # 1e-6 relative per entry, with a floor of 1e-6 of the largest sampled gradient
        tol = 1e-6 * np.abs(fd) + 1e-6 * np.abs(fd).max()
        assert np.all(np.abs(ad - fd) <= tol), (k, np.c_[idx, ad, fd])
    model.destroy()


def test_autograd_function_and_records():
    import torch
    from gospl_b200.adjoint import SurfaceEvolution

    model, onb, (K, U, rain, h0) = _setup()
    Kp = K.clone().requires_grad_(True)
    Up = U.clone().requires_grad_(True)
    hT = SurfaceEvolution.apply(Kp, Up, rain, h0, model, 4, 2)
    loss = (hT ** 2).sum()
    loss.backward()
    assert Kp.grad is not None and torch.isfinite(Kp.grad).all() and Kp.grad.abs().max() > 0
    assert torch.isfinite(Up.grad).all()
    # the adjoint refuses a slot that holds no recorded step
    from gospl_b200 import _lib
    model.record(2)
    lam = torch.zeros_like(h0)
    with pytest.raises(_lib.GsError):
        model.adjoint_step(1, lam)
    model.record(0)
    model.destroy()
