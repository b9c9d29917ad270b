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
    # records kept from the forward (every=None) give the same gradients as
    # the checkpointed replay: the replayed steps record the same states
    Kq = K.clone().requires_grad_(True)
    Uq = U.clone().requires_grad_(True)
    hT2 = SurfaceEvolution.apply(Kq, Uq, rain, h0, model, 4, None)
    assert torch.equal(hT2, hT.detach())
    (hT2 ** 2).sum().backward()
    assert torch.allclose(Kq.grad, Kp.grad, rtol=1e-12, atol=0.0)
    assert torch.allclose(Uq.grad, Up.grad, rtol=1e-12, atol=0.0)
    # the adjoint refuses a slot that holds no recorded step
    from gospl_b200 import _lib
    model.record(2)
    lam = torch.zeros_like(h0)
    with pytest.raises(_lib.GsError):
        model.adjoint_step(1, lam)
    model.record(0)
    model.destroy()


def _dense_step(h, K, U, rain, rcv, dist, lsink, sea, mesh, p, flat):
    """One physics step in dense float64 torch with the receivers chosen by the
    GPU step held fixed (a landscape without depressions: no lake cascade).
    `dist` is the step's receiver distance array, which mfdreceivers fills
    from the unsorted candidate list (a constant of the receiver choice)."""
    import torch
    n = h.shape[0]
    dev = h.device
    ngb = torch.as_tensor(mesh.ngb, dtype=torch.int64, device=dev)
    elgt = torch.as_tensor(mesh.elgt, dtype=torch.float64, device=dev)
    vdist = torch.as_tensor(mesh.vdist, dtype=torch.float64, device=dev)
    nnb = torch.as_tensor(mesh.nnb, dtype=torch.int64, device=dev)
    farea = torch.as_tensor(mesh.farea, dtype=torch.float64, device=dev)
    larea = torch.as_tensor(mesh.larea, dtype=torch.float64, device=dev)
    outlet = torch.zeros(n, dtype=torch.bool, device=dev)
    outlet[torch.as_tensor(mesh.outlet, dtype=torch.int64, device=dev)] = True
    slot_ok = (torch.arange(12, device=dev)[None, :] < nnb[:, None]) & (ngb >= 0) & (elgt > 0)
    idx = torch.arange(n, device=dev)
    nb = ngb.clamp(min=0)
    # adaptive exponent from the steepest descent
    sl_all = torch.where(slot_ok, (h[:, None] - h[nb]) / torch.where(slot_ok, elgt, torch.ones_like(elgt)),
                         torch.zeros_like(elgt))
    e = sl_all.max(dim=1).values.clamp(min=0.0)
    fexp = torch.where(e > 0, 5.0 * e.clamp(max=1.0) + 1.1, torch.ones_like(e))
    R = rcv.shape[0]
    slp, ds, isr, rr = [], [], [], []
    for k in range(R):
        r = rcv[k].long()
        is_r = r != idx
        at = (ngb == r[:, None]) & slot_ok
        L = (elgt * at).sum(dim=1)
        d = torch.where(is_r, h - h[r], torch.ones_like(h))
        s = torch.where(is_r, d ** fexp / torch.where(is_r, L, torch.ones_like(L)) * (1.0 - 1e-15 * r.double()),
                        torch.zeros_like(h))
        slp.append(s), ds.append(L), isr.append(is_r), rr.append(r)
    V = sum(slp)
    w = [torch.where(V > 0, s / torch.where(V > 0, V, torch.ones_like(V)), torch.zeros_like(V)) for s in slp]
    # drainage area: (I - W^T) q = b
    Wm = torch.zeros((n, n), dtype=torch.float64, device=dev)
    for k in range(R):
        Wm = Wm.index_put((idx, rr[k]), torch.where(isr[k], w[k], torch.zeros_like(h)), accumulate=True)
    eye = torch.eye(n, dtype=torch.float64, device=dev)
    b = torch.where(sea, torch.zeros_like(h), rain.clamp(min=0.0) * larea)
    q = torch.linalg.solve(eye - Wm.T, b)
    fal = q.clamp(min=0.0)
    # SPL
    kbr = K * rain ** p["d"] * (p["dt"] * fal ** p["m"])
    kbr = torch.where(sea, torch.zeros_like(kbr), kbr)
    C = torch.zeros((n, n), dtype=torch.float64, device=dev)
    for k in range(R):
        dh = h - h[rr[k]]
        lim = torch.where(dh != 0, dh / (dh + 1e-2), torch.zeros_like(dh))
        dk = dist[k]
        c = torch.where(isr[k] & ~sea & (dk != 0), kbr * lim / torch.where(dk != 0, dk, torch.ones_like(h)) * w[k],
                        torch.zeros_like(h))
        C = C.index_put((idx, rr[k]), c, accumulate=True)
    M = eye + torch.diag(C.sum(dim=1)) - C
    s = torch.linalg.solve(M, h)
    keep = lsink | (outlet if flat else torch.zeros_like(outlet))
    h1 = torch.where(keep, h, s)
    # hillslope
    seah = h1 <= p["sealevel"]
    kd = torch.where(seah, torch.full_like(h, p["Cdm"]), torch.full_like(h, p["Cda"])) * p["dt"]
    fixed = (outlet if flat else torch.zeros_like(outlet)) | ~(farea > 0)
    vok = slot_ok & (vdist > 0)
    v = torch.where(vok, 0.5 * (kd[:, None] + kd[nb]) / farea[:, None].clamp(min=1e-300) * vdist /
                    torch.where(vok, elgt, torch.ones_like(elgt)), torch.zeros_like(elgt))
    v = torch.where(fixed[:, None], torch.zeros_like(v), v)
    Lm = torch.zeros((n, n), dtype=torch.float64, device=dev)
    Lm = Lm.index_put((idx[:, None].expand(-1, 12)[vok], nb[vok]), -v[vok], accumulate=True)
    Lm = Lm + torch.diag(v.sum(dim=1))
    h2 = torch.linalg.solve(eye + Lm, h1)
    return h2 + U * p["dt"]


def test_adjoint_matches_dense_autograd():
    """The hand-written adjoint against torch float64 autograd through dense
    solves of the same steps (2,000-vertex landscape without depressions,
    receivers of each step taken from the GPU forward)."""
    import torch
    from gospl_b200 import synthetic as S
    from gospl_b200 import adjoint as A
    from gospl_b200.mesh import FVMesh
    from gospl_b200.model import Model

    dev = torch.device("cuda", torch.cuda.current_device())
    side = 537.0 * np.sqrt(2000 * np.sqrt(3) / 2)
    coords, cells, onb = S.planar_hex_mesh(2000, side, seed=9)
    x, y = coords[:, 0], coords[:, 1]
    z = 5.0 + 1e-2 * x + 2e-3 * y + 0.5 * np.sin(2 * np.pi * y / 5.0e3)   # rises with x everywhere: no pits
    z[onb] = 0.0
    n = len(z)
    K = np.exp(S.rescale(S.fractal_field(coords[:, :2], side, 10, beta=4.0), -13.0, -11.0))
    U = np.full(n, 5e-4)
    U[onb] = 0.0
    rain = 1.0 + 0.5 * np.cos(2 * np.pi * x / side)
    params = dict(dt=1000.0, tStart=0.0, tEnd=1e30, flowDir=3, K=K, d=0.0, m=0.5, Cda=0.1, Cdm=0.1,
                  sealevel=-100.0, oFill=-6000.0, bc="ffff", rain=rain, upsub=U)
    mesh = FVMesh(coords, cells, "ffff", device=dev)
    model = Model(coords=coords, cells=cells, elev=z, params=params, mesh=mesh, device=dev)
    f64 = dict(dtype=torch.float64, device=dev)
    Kt, Ut, Rt, h0 = (torch.tensor(a, **f64) for a in (K, U, rain, z))
    nsteps = 3
    # GPU forward, keeping each step's receivers and masks; solver warm starts
    # off, as in the adjoint's own runs (A.run), so that A.run repeats it bit
    # for bit
    A._set_params(model, Kt, Ut, Rt)
    A._restart(model, h0)
    structure, hs = [], []
    with A._cold(model):
        for _ in range(nsteps):
            model.step()
            assert model.stats["flow"]["cascade_passes"] == 0
            structure.append((model.rcv_i.clone(), model.dist_i.clone(), model.lsink_mask.bool().clone(),
                              model.sea_mask.bool().clone()))
            hs.append(model.hGlobal.clone())
    hT = hs[-1]
    rng = np.random.default_rng(4)
    target = hT + 1e-3 * torch.tensor(rng.standard_normal(n), **f64)
    # dense autograd
    Kd, Ud, Rd, hd = (t.clone().requires_grad_(True) for t in (Kt, Ut, Rt, h0))
    h = hd
    for t in range(nsteps):
        rcv, dist, lsink, sea = structure[t]
        h = _dense_step(h, Kd, Ud, Rd, rcv, dist, lsink, sea, mesh, params, True)
        assert torch.allclose(h, hs[t], rtol=1e-10, atol=1e-9), t
    # both sides reverse the same seed lam = dJ/dh_T of J = |h_T - target|^2 at
    # the GPU's h_T (the dense forward agrees with it to ~1e-12 only)
    lam = 2 * (hT - target)
    gK, gU, gR, gh = torch.autograd.grad((lam * h).sum(), (Kd, Ud, Rd, hd))
    # hand-written adjoint
    hT2, ck = A.run(model, Kt, Ut, Rt, h0, nsteps, 2)
    assert torch.equal(hT2, hT)
    aK, aU, aR, ah = A.backward(model, Kt, Ut, Rt, ck, nsteps, 2, lam)
    for ref, got in ((gK, aK), (gU, aU), (gR, aR), (gh, ah)):
        err = (got - ref).abs().max() / ref.abs().max()
        assert err <= 1e-8, float(err)
    model.destroy()
