"""Seeded synthetic GPR models and acquisitions of the benchmark configurations.

No dataset is involved: every model is generated from a ``torch.Generator``
seed.  Depth is axis 0 ("rows"/"layers"); air occupies the first rows, and
sources/receivers sit on the first row below the air.

* layered model: ``n_layers`` horizontal layers with seeded depths, eps_r and
  sigma drawn uniformly per layer;
* plus a Gaussian random field (white noise filtered by a Gaussian kernel of
  ``corr / dx`` cells in Fourier space, normalised to ``field_std``);
* clipped to ``clip`` and the air layer set last (eps_r = 1, sigma = 0).
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import torch

from .grid import max_stable_time_step
from .wavelets import ricker


def gaussian_random_field(shape: Sequence[int], corr_cells: float, gen: torch.Generator) -> torch.Tensor:
    noise = torch.randn(tuple(shape), generator=gen, dtype=torch.float64)
    spec = torch.fft.fftn(noise)
    k2 = torch.zeros(tuple(shape), dtype=torch.float64)
    for axis, n in enumerate(shape):
        f = torch.fft.fftfreq(n, dtype=torch.float64)
        view = [1] * len(shape)
        view[axis] = n
        k2 = k2 + (2 * math.pi * f.view(view)) ** 2
    field = torch.fft.ifftn(spec * torch.exp(-0.5 * k2 * corr_cells**2)).real
    field = field - field.mean()
    return field / field.std()


def layered_model(
    shape: Sequence[int], air_rows: int, eps_range: Tuple[float, float], sigma_range: Tuple[float, float],
    gen: torch.Generator, n_layers: int = 8, corr: Optional[float] = None, dx: float = 1.0, field_std: float = 1.0,
    clip: Optional[Tuple[float, float]] = None,
) -> Tuple[torch.Tensor, torch.Tensor]:
    """(eps_r, sigma) of a layered model below an air layer."""
    depth = shape[0]
    cuts = torch.sort(torch.randint(air_rows + 1, depth, (n_layers - 1,), generator=gen)).values.tolist()
    bounds = [air_rows] + cuts + [depth]
    eps = torch.empty(tuple(shape), dtype=torch.float64)
    sig = torch.empty(tuple(shape), dtype=torch.float64)
    for a, b in zip(bounds[:-1], bounds[1:]):
        e = eps_range[0] + (eps_range[1] - eps_range[0]) * torch.rand((), generator=gen, dtype=torch.float64)
        s = sigma_range[0] + (sigma_range[1] - sigma_range[0]) * torch.rand((), generator=gen, dtype=torch.float64)
        eps[a:b] = e
        sig[a:b] = s
    eps[:air_rows] = eps[air_rows]
    sig[:air_rows] = sig[air_rows]
    if corr is not None:
        eps = eps + field_std * gaussian_random_field(shape, corr / dx, gen)
    if clip is not None:
        eps = eps.clamp(*clip)
    eps[:air_rows] = 1.0
    sig[:air_rows] = 0.0
    return eps.float(), sig.float()


@dataclass
class Acquisition:
    eps_r: torch.Tensor
    sigma: torch.Tensor
    eps_true: torch.Tensor
    sources: torch.Tensor        # (nshot, 1, 3) int32 physical coordinates
    receivers: torch.Tensor      # (nshot, nrx, 3)
    wavelet: torch.Tensor        # (1, nt)
    dx: float
    dt: float
    order: int
    mode: int
    pml: int = 10


def fwi_2d(seed: int = 1002, shape=(400, 800), dx=0.01, nshot=32, nrx=200, nt=3000, freq=400e6, order=4,
           air_rows=20) -> Acquisition:
    """2D multi-shot FWI gradient problem (32 shots, 200 receivers, Ricker 400 MHz).

    The "observed" model adds an eps_r = 9 disc of radius 0.3 m centred at
    (depth 200, lateral 400) cells.
    """
    gen = torch.Generator().manual_seed(seed)
    eps, sig = layered_model(shape, air_rows, (3.0, 25.0), (0.0, 0.01), gen, corr=0.2, dx=dx, clip=(1.0, 30.0))
    true = eps.clone()
    ii = torch.arange(shape[0]).view(-1, 1).float()
    jj = torch.arange(shape[1]).view(1, -1).float()
    disc = (ii - shape[0] // 2) ** 2 + (jj - shape[1] // 2) ** 2 <= (0.3 / dx) ** 2
    true[disc] = 9.0
    row = air_rows
    src = torch.tensor([[[row, int(round((s + 0.5) * shape[1] / nshot)), 0]] for s in range(nshot)], dtype=torch.int32)
    cols = torch.linspace(0, shape[1] - 1, nrx).round().int()
    rcv = torch.stack([torch.stack([torch.full_like(cols, row), cols, torch.zeros_like(cols)], -1)] * nshot)
    ext = (shape[0] + 20, shape[1] + 20, 1)
    dt = 0.9 * max_stable_time_step(dx, *ext, fdtd_order=order)
    return Acquisition(eps, sig, true, src, rcv.int(), ricker(freq, nt, dt)[None], dx, dt, order, 2)


def fwi_3d(seed: int = 1003, shape=(200, 200, 200), dx=0.02, sources_grid=(2, 4), receivers_grid=(24, 24),
           nt=2500, freq=250e6, order=8, air_rows=10) -> Acquisition:
    """3D forward+adjoint problem: layered eps_r in [3, 20] + 3D random field (0.3 m)."""
    gen = torch.Generator().manual_seed(seed)
    eps, sig = layered_model(shape, air_rows, (3.0, 20.0), (0.0, 0.005), gen, corr=0.3, dx=dx, clip=(1.0, 30.0))
    row = air_rows
    sy, sz = sources_grid
    srcs = [[row, int((a + 0.5) * shape[1] / sy), int((b + 0.5) * shape[2] / sz)] for a in range(sy) for b in range(sz)]
    ry, rz = receivers_grid
    rcv1 = [[row, int((a + 0.5) * shape[1] / ry), int((b + 0.5) * shape[2] / rz)] for a in range(ry) for b in range(rz)]
    src = torch.tensor([[s] for s in srcs], dtype=torch.int32)
    rcv = torch.tensor([rcv1] * len(srcs), dtype=torch.int32)
    ext = tuple(n + 20 for n in shape)
    dt = 0.9 * max_stable_time_step(dx, *ext, fdtd_order=order)
    return Acquisition(eps, sig, eps.clone(), src, rcv, ricker(freq, nt, dt)[None], dx, dt, order, 3)


def serving_stream(seed: int = 1004, n: int = 40, nt_scale: float = 0.1, mean_gap_s: float = 0.01):
    """Config-4 request stream: seeded Poisson arrivals, 70 % 2D forward solves
    (square grids log-uniform in [128, 1024]^2, nt in [1000, 4000], 1-16 shots,
    order 2 or 4) and 30 % 3D gradient solves (cubic grids log-uniform in
    [96, 160]^3, nt in [800, 1500], 1-4 shots, order 4), models drawn as in
    configs 2 and 3, Ricker 150-500 MHz.  ``nt_scale`` shortens every nt (a
    bounded sample of the stream); gradient requests use zero observed data
    (misfit = receiver energy).  Returns ``(requests, arrival_seconds)``.
    """
    import math

    from .serving import SolveRequest

    gen = torch.Generator().manual_seed(seed)

    def uni(a, b):
        return a + (b - a) * float(torch.rand((), generator=gen))

    def loguni(a, b):
        return int(round(math.exp(uni(math.log(a), math.log(b)))))

    reqs, arrivals, t = [], [], 0.0
    for k in range(n):
        t += -mean_gap_s * math.log(max(1e-12, 1.0 - float(torch.rand((), generator=gen))))
        freq = uni(150e6, 500e6)
        if float(torch.rand((), generator=gen)) < 0.7:
            size = loguni(128, 1024)
            nt = max(16, int(uni(1000, 4000) * nt_scale))
            shots = int(uni(1, 17))
            order = 2 if float(torch.rand((), generator=gen)) < 0.5 else 4
            acq = fwi_2d(seed=seed * 1000 + k, shape=(size, size), nshot=shots, nrx=min(64, size), nt=nt,
                         freq=freq, order=order, air_rows=min(20, size // 8))
            reqs.append(SolveRequest(kind="forward", eps_r=acq.eps_r, sigma=acq.sigma,
                                     source_amplitudes=acq.wavelet, source_location=acq.sources,
                                     receiver_location=acq.receivers, dx=acq.dx, dt=acq.dt, pmlthick=10,
                                     fdtd_order=order, mode=2, tag=f"2d-fwd-{k}"))
        else:
            size = loguni(96, 160)
            nt = max(16, int(uni(800, 1500) * nt_scale))
            shots = int(uni(1, 5))
            acq = fwi_3d(seed=seed * 1000 + k, shape=(size, size, size), dx=0.02, sources_grid=(1, shots),
                         receivers_grid=(8, 8), nt=nt, freq=freq, order=4)
            obs = torch.zeros((shots, nt, acq.receivers.shape[1]))
            reqs.append(SolveRequest(kind="gradient", eps_r=acq.eps_r, sigma=acq.sigma,
                                     source_amplitudes=acq.wavelet, source_location=acq.sources,
                                     receiver_location=acq.receivers, dx=acq.dx, dt=acq.dt, pmlthick=10,
                                     fdtd_order=4, mode=3, observed=obs, tag=f"3d-grad-{k}"))
        arrivals.append(t)
    return reqs, arrivals
