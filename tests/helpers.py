"""Problem builders and comparison helpers shared by the tests."""

from __future__ import annotations

import math
from typing import Any, Dict, List, Optional, Sequence

import torch

from oracle import driver


def ricker(nt: int, dt: float, f: float) -> torch.Tensor:
    t = torch.arange(nt, dtype=torch.float64) * dt
    a = (math.pi * f * (t - 1.0 / f)) ** 2
    return ((1 - 2 * a) * torch.exp(-a)).float()


def problem_2d(nt=120, order=2, shape=(40, 36), pml=10, seed=0, **kw) -> driver.Problem:
    g = torch.Generator().manual_seed(seed)
    eps = torch.full(shape, 2.0)
    eps[shape[0] // 2 :, :] = 5.0
    eps = eps + 0.3 * torch.rand(shape, generator=g)
    sig = 1e-3 * torch.rand(shape, generator=g)
    dt = 3e-11
    src = torch.tensor([[[10, 10, 0]]], dtype=torch.int32)
    rcv = torch.tensor([[[10, shape[1] - 6, 0], [5, 7, 0], [10, 10, 0]]], dtype=torch.int32)
    args = dict(eps_r=eps, sigma=sig, source_amplitudes=ricker(nt, dt, 200e6)[None], source_location=src,
                receiver_location=rcv, dx=0.02, dt=dt, pml=pml, order=order, mode=2)
    args.update(kw)
    return driver.Problem(**args)


def problem_3d(nt=40, order=2, shape=(16, 14, 12), pml=3, seed=0, nshot=2, **kw) -> driver.Problem:
    g = torch.Generator().manual_seed(seed)
    eps = 3.0 + 2.0 * torch.rand(shape, generator=g)
    sig = 2e-3 * torch.rand(shape, generator=g)
    dt = 1.5e-11
    src = torch.tensor([[[8, 7, 4]], [[5, 6, 7]], [[3, 3, 3]], [[9, 2, 5]]], dtype=torch.int32)[:nshot]
    rcv = torch.tensor([[[10, 3, 4], [5, 7, 2], [8, 7, 4]], [[1, 2, 3], [5, 6, 7], [6, 6, 6]],
                        [[2, 2, 2], [3, 3, 3], [4, 4, 4]], [[9, 9, 9], [1, 1, 1], [9, 2, 5]]], dtype=torch.int32)[:nshot]
    args = dict(eps_r=eps, sigma=sig, source_amplitudes=ricker(nt, dt, 400e6)[None], source_location=src,
                receiver_location=rcv, dx=0.02, dt=dt, pml=pml, order=order, mode=3)
    args.update(kw)
    return driver.Problem(**args)


def rel_l2(a: torch.Tensor, b: torch.Tensor) -> float:
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    den = b.norm().item()
    num = (a - b).norm().item()
    if den == 0.0:
        return num
    return num / den


def run_product(p: driver.Problem, device: torch.device, backward: bool = True, **compute_kw) -> Dict[str, Any]:
    """Run the same problem through deepgpr_b200.compute on the GPU."""
    import deepgpr_b200 as dg

    eps = p.eps_r.detach().clone().to(device).requires_grad_(p.want_eps)
    sig = p.sigma.detach().clone().to(device).requires_grad_(p.want_sigma)
    wave = p.source_amplitudes.detach().clone().to(device).requires_grad_(p.want_source)
    kw: Dict[str, Any] = dict(
        dx=p.dx, dt=p.dt, source_amplitudes=wave, source_location=p.source_location.to(device),
        receiver_location=p.receiver_location.to(device), eps_r=eps, sigma=sig,
        mu_r=None if p.mu_r is None else p.mu_r.to(device), pmlthick=p.pml, source_direction=p.source_component,
        receiver_component=p.receiver_component, fdtd_order=p.order, mode=p.mode,
        model_gradient_sampling_interval=p.interval,
        wavefield_storage_dtype={0: torch.float32, 1: torch.float16, 2: torch.bfloat16}[p.storage_kind],
        wavefield_history_region=p.region,
    )
    if p.rhs_from_e is not None:
        kw["wavefield_rhs_history"] = "reconstructed" if p.rhs_from_e else "stored"
    states_in: Optional[List[torch.Tensor]] = None
    if p.initial_states is not None:
        states_in = [t.detach().clone().to(device).requires_grad_(True) for t in p.initial_states]
        kw.update(E=tuple(states_in[:3]), H=tuple(states_in[3:6]), PML=tuple(states_in[6:]))
    kw.update(compute_kw)
    e_saved, E, H, PML, rx = dg.compute(device, **kw)
    states = [*E, *H, *PML]
    out: Dict[str, Any] = {"receivers": rx.detach().cpu(), "states": [s.detach().cpu() for s in states],
                           "E_saved": e_saved}
    if not backward:
        return out
    dg_weights = (2.0 * rx.detach()) if p.data_grad is None else p.data_grad.to(device)
    loss = (rx * dg_weights).sum()
    if p.state_duals is not None:
        loss = loss + sum((s * d.to(device)).sum() for s, d in zip(states, p.state_duals) if s.numel())
    roots, names = [], []
    for n, t, w in (("grad_eps", eps, p.want_eps), ("grad_sigma", sig, p.want_sigma),
                    ("grad_source", wave, p.want_source)):
        if w:
            roots.append(t)
            names.append(n)
    if states_in is not None:
        roots.extend(states_in)
    grads = torch.autograd.grad(loss, roots, allow_unused=True)
    for n, g in zip(names, grads):
        out[n] = g.detach().cpu()
    if states_in is not None:
        out["lambdas"] = [None if g is None else g.detach().cpu() for g in grads[len(names):]]
    return out
