"""The hand-written adjoint against the forward it transposes (FP64 runs on the GPU).

Checks modelled on the reference's own adjoint tests
(tests/test_discrete_adjoint.py:70-137, 353-381 dot products; 204-282 and
510-521 Taylor tests; 475-508 source finite differences) and on the
precision study's finite-difference check:

* dot-product tests: with zero initial fields the map from source amplitudes
  to receivers is linear, and so is the map from the 30 initial states to
  the 30 final states and the receivers; <F x, y> = <x, F^T y> holds to FP64
  rounding for orders 2 / 4 / 8 with CPML on every face, in 2D and 3D;
* Taylor test: J(m + h dm) - J(m) - h <g, dm> falls like h^2 for eps_r and
  sigma together;
* central finite differences on a 64^3 grid (CPML 10): 20 random eps_r cells
  and 20 random sigma cells, step 1e-4, against the adjoint gradient.

All solves use ``precision=torch.float64`` (the same kernels in double).
"""

from __future__ import annotations

import math

import pytest
import torch

pytestmark = pytest.mark.gpu

F64 = torch.float64


def _ricker(nt, dt, f):
    t = torch.arange(nt, dtype=F64) * dt
    a = (math.pi * f * (t - 1.0 / f)) ** 2
    return (1 - 2 * a) * torch.exp(-a)


def _setup(dims, order, seed=0):
    g = torch.Generator().manual_seed(seed)
    if dims == 2:
        shape, dx, dt, pml = (30, 26), 0.02, 2.0e-11, 6
        src = torch.tensor([[[10, 9, 0]], [[18, 15, 0]]], dtype=torch.int32)
        rcv = torch.tensor([[[5, 20, 0], [25, 3, 0], [10, 9, 0]]] * 2, dtype=torch.int32)
    else:
        shape, dx, dt, pml = (14, 12, 10), (0.02, 0.017, 0.015), 1.0e-11, [3, 2, 4, 3, 2, 3]
        src = torch.tensor([[[7, 6, 5]], [[3, 8, 2]]], dtype=torch.int32)
        rcv = torch.tensor([[[2, 3, 4], [11, 9, 7], [7, 6, 5]]] * 2, dtype=torch.int32)
    eps = (3.0 + 2.0 * torch.rand(shape, generator=g)).to(F64)
    sig = (1e-3 + 3e-3 * torch.rand(shape, generator=g)).to(F64)   # >= 1e-3: perturbations stay non-negative
    return dict(shape=shape, dx=dx, dt=dt, pml=pml, src=src, rcv=rcv, eps=eps, sig=sig, order=order,
                mode=2 if dims == 2 else 3, source_direction=2 if dims == 2 else 0)


def _solve(dev, c, wave, eps=None, sig=None, states=None, history=True):
    import deepgpr_b200 as dg

    kw = dict(dx=c["dx"], dt=c["dt"], source_amplitudes=wave, source_location=c["src"].to(dev),
              receiver_location=c["rcv"].to(dev), eps_r=(c["eps"] if eps is None else eps).to(dev),
              sigma=(c["sig"] if sig is None else sig).to(dev), pmlthick=c["pml"], fdtd_order=c["order"],
              mode=c["mode"], source_direction=c["source_direction"], receiver_component=c["source_direction"],
              precision=F64, save_wavefield_history=history)
    if states is not None:
        kw.update(E=tuple(states[:3]), H=tuple(states[3:6]), PML=tuple(states[6:]))
    _, E, H, PML, rx = dg.compute(dev, **kw)
    return rx, [*E, *H, *PML]


def _dot(a, b):
    return float((a.double() * b.double()).sum())


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("dims", [2, 3])
def test_source_dot_product(dims, order, cuda_device):
    c = _setup(dims, order)
    nt = 60
    g = torch.Generator().manual_seed(1 + order)
    x = torch.randn((1, nt), generator=g, dtype=F64)           # the waveform of every shot's source
    y = torch.randn((2, nt, 3), generator=g, dtype=F64)        # receiver cotangent
    with torch.no_grad():
        fx, _ = _solve(cuda_device, c, x.to(cuda_device), history=False)
    w = torch.zeros((1, nt), dtype=F64, device=cuda_device, requires_grad=True)
    rx, _ = _solve(cuda_device, c, w)
    (gw,) = torch.autograd.grad((rx * y.to(cuda_device)).sum(), [w])
    lhs, rhs = _dot(fx.cpu(), y), _dot(x, gw.cpu())
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs)), (lhs, rhs)


# Ex, Ey, Hz and the CPML arrays that couple them: zero on the 2D TM path
TM2D_INACTIVE = (0, 1, 5) + tuple(6 + i for i in (0, 3, 4, 7, 8, 11, 12, 15))


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("dims", ["2tm", 2, 3])
def test_state_dot_product(dims, order, cuda_device):
    """Initial states (fields and all 24 CPML arrays) to final states and receivers.

    "2tm": the 2D Ez-TM path, whose inactive states (Ex, Ey, Hz and their CPML
    arrays) start at zero and must get zero cotangents (the reference's
    _state_problem_2d_tm); 2: every state perturbed, the general path on the
    nz = 1 grid; 3: every state perturbed in 3D.
    """
    from deepgpr_b200.model import prepare_model
    from deepgpr_b200.pml import build_psi

    tm = dims == "2tm"
    c = _setup(2 if tm else dims, order)
    nt = 25
    prep = prepare_model("cpu", c["eps"], c["sig"], None, torch.zeros((1, nt), dtype=F64), c["src"], c["rcv"],
                         c["dx"], c["dt"], c["pml"], order, dtype=F64)
    nx, ny, nz = prep.nx, prep.ny, prep.nz
    zeros = [torch.zeros((2, nx + 1, ny + 1, nz + 1), dtype=F64) for _ in range(6)]
    zeros += list(build_psi(nx, ny, nz, prep.pml, 2, None, "cpu", F64))
    g = torch.Generator().manual_seed(7 + order)
    xs = [torch.randn(t.shape, generator=g, dtype=F64) * 1e-2 for t in zeros]
    if tm:
        for i in TM2D_INACTIVE:
            xs[i] = torch.zeros_like(xs[i])
    ys = [torch.randn(t.shape, generator=g, dtype=F64) for t in zeros]
    yr = torch.randn((2, nt, 3), generator=g, dtype=F64)
    wave = torch.zeros((1, nt), dtype=F64, device=cuda_device)
    # the map is linear in the states: <F x, y> from the solve of x, <x, F^T y> from its adjoint
    ins = [t.to(cuda_device).requires_grad_(True) for t in xs]
    rx, outs = _solve(cuda_device, c, wave, states=ins)
    lhs = _dot(rx.detach().cpu(), yr) + sum(_dot(a.detach().cpu(), b) for a, b in zip(outs, ys) if b.numel())
    loss = (rx * yr.to(cuda_device)).sum() + sum((a * b.to(cuda_device)).sum() for a, b in zip(outs, ys) if b.numel())
    lams = torch.autograd.grad(loss, ins, allow_unused=True)
    rhs = sum(_dot(x, lam.cpu()) for x, lam in zip(xs, lams) if lam is not None and x.numel())
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs)), (lhs, rhs)
    if tm:
        for i in TM2D_INACTIVE:
            if lams[i] is not None and lams[i].numel():
                assert float(lams[i].abs().max()) == 0.0, i


def _misfit(dev, c, wave, obs, eps, sig):
    rx, _ = _solve(dev, c, wave, eps=eps, sig=sig, history=eps.requires_grad or sig.requires_grad)
    return 0.5 * ((rx - obs) ** 2).sum()


def test_taylor_eps_sigma(cuda_device):
    c = _setup(3, 4)
    nt = 80
    wave = _ricker(nt, c["dt"], 500e6)[None].to(cuda_device)
    g = torch.Generator().manual_seed(5)
    true_eps = c["eps"].clone()
    true_eps[5:9, 4:8, 3:7] += 1.5
    with torch.no_grad():
        obs, _ = _solve(cuda_device, c, wave, eps=true_eps, history=False)
    eps = c["eps"].to(cuda_device).requires_grad_(True)
    sig = c["sig"].to(cuda_device).requires_grad_(True)
    j0 = _misfit(cuda_device, c, wave, obs, eps, sig)
    ge, gs = torch.autograd.grad(j0, [eps, sig])
    de = torch.randn(c["shape"], generator=g, dtype=F64).to(cuda_device)
    ds = 1e-2 * torch.rand(c["shape"], generator=g, dtype=F64).to(cuda_device)   # keeps sigma non-negative
    slope = float((ge * de).sum() + (gs * ds).sum())
    res = []
    with torch.no_grad():
        for h in (1e-2, 5e-3, 2.5e-3, 1.25e-3):
            jh = _misfit(cuda_device, c, wave, obs, eps.detach() + h * de, sig.detach() + h * ds)
            res.append(abs(float(jh) - float(j0) - h * slope))
    rates = [math.log2(a / b) for a, b in zip(res[:-1], res[1:])]
    assert all(r > 1.9 for r in rates), (res, rates)


def test_central_finite_differences_64cube(cuda_device):
    """FP64 central differences (step 1e-4) at 20 random eps_r and 20 random sigma cells."""
    from deepgpr_b200.grid import max_stable_time_step

    n, dx, pml = 64, 0.02, 10
    g = torch.Generator().manual_seed(64)
    eps0 = (4.0 + 2.0 * torch.rand((n, n, n), generator=g)).to(F64)
    sig0 = (1e-3 + 3e-3 * torch.rand((n, n, n), generator=g)).to(F64)   # sigma - 1e-4 stays non-negative
    dt = 0.9 * max_stable_time_step(dx, n + 2 * pml, n + 2 * pml, n + 2 * pml, fdtd_order=4, min_er_mr=4.0)
    nt = 260
    c = dict(shape=(n, n, n), dx=dx, dt=dt, pml=pml, order=4, mode=3, source_direction=2,
             src=torch.tensor([[[32, 32, 32]]], dtype=torch.int32),
             rcv=torch.tensor([[[8, j, k] for j in (12, 32, 52) for k in (12, 32, 52)]], dtype=torch.int32),
             eps=eps0, sig=sig0)
    wave = _ricker(nt, dt, 600e6)[None].to(cuda_device)
    true_eps = eps0.clone()
    true_eps[20:44, 20:44, 40:52] += 2.0
    with torch.no_grad():
        obs, _ = _solve(cuda_device, c, wave, eps=true_eps, history=False)
    eps = eps0.to(cuda_device).requires_grad_(True)
    sig = sig0.to(cuda_device).requires_grad_(True)
    ge, gs = torch.autograd.grad(_misfit(cuda_device, c, wave, obs, eps, sig), [eps, sig])
    cells = torch.randint(0, n, (40, 3), generator=g)
    h = 1e-4
    errs = []
    with torch.no_grad():
        for which, grad in (("eps", ge), ("sig", gs)):
            fd, ad = [], []
            for i, j, k in cells[:20].tolist() if which == "eps" else cells[20:].tolist():
                e_p, s_p = eps.detach().clone(), sig.detach().clone()
                e_m, s_m = eps.detach().clone(), sig.detach().clone()
                tgt_p, tgt_m = (e_p, e_m) if which == "eps" else (s_p, s_m)
                tgt_p[i, j, k] += h
                tgt_m[i, j, k] -= h
                jp = float(_misfit(cuda_device, c, wave, obs, e_p, s_p))
                jm = float(_misfit(cuda_device, c, wave, obs, e_m, s_m))
                fd.append((jp - jm) / (2 * h))
                ad.append(float(grad[i, j, k]))
            fd_t, ad_t = torch.tensor(fd, dtype=F64), torch.tensor(ad, dtype=F64)
            err = float((fd_t - ad_t).norm() / ad_t.norm())
            errs.append((which, err))
            assert ad_t.abs().max() > 0, which
            assert err <= 1e-5, (which, err, fd, ad)
    print("central FD vs adjoint (relative L2 over the 20 cells):", errs)
