"""Input validation and extension of the physical model into the CPML.

Follows src/DeepGPR/preprocessing/model_setup.py:72-406: the user supplies the
physical model; materials are replicated outward into the CPML faces (the
transpose sums the CPML sensitivities back onto the edge cells, one axis at a
time), a one-cell Yee halo of zeros is appended on the high side of every
axis, and source/receiver coordinates are shifted by the low-face thickness.
"""

from __future__ import annotations

from typing import Any, NamedTuple, Sequence, Tuple

import torch
import torch.nn.functional as F

from .config import INT32_MAX, MAX_SHOTS_PER_CALL, MIN_RELATIVE_PERMITTIVITY, PEC_CONDUCTIVITY_THRESHOLD
from .grid import check_cfl, extended_shape, normalize_grid_spacing, normalize_pml_thickness, positive_finite


class PreparedModel(NamedTuple):
    """Materials and geometry on the solver grid.

    ``eps_r``/``sigma`` are extended into the CPML, shape ``(nx, ny, nz)``;
    ``eps_r_pad``/``sigma_pad``/``mu_r_pad`` carry the Yee halo,
    ``(nx+1, ny+1, nz+1)``.  ``source_amplitudes`` is ``(nsr, nt, 1)``.
    """

    eps_r: torch.Tensor
    sigma: torch.Tensor
    nx: int
    ny: int
    nz: int
    nt: int
    nstep: int
    nsr: int
    nrx: int
    eps_r_pad: torch.Tensor
    sigma_pad: torch.Tensor
    mu_r_pad: torch.Tensor
    mode: int
    dtype: torch.dtype
    pml: Tuple[int, ...]
    source_amplitudes: torch.Tensor


class ExtendIntoPML(torch.autograd.Function):
    """Replicate-pad a model into the CPML; backward folds the pad onto the edges."""

    @staticmethod
    def forward(ctx, model: torch.Tensor, pml: Sequence[int]) -> torch.Tensor:  # type: ignore[override]
        ctx.shape = tuple(model.shape)
        ctx.pml = tuple(int(v) for v in pml)
        pad = (ctx.pml[4], ctx.pml[5], ctx.pml[2], ctx.pml[3], ctx.pml[0], ctx.pml[1])
        return F.pad(model[None, None], pad, mode="replicate")[0, 0]

    @staticmethod
    def backward(ctx, grad: torch.Tensor):  # type: ignore[override]
        return fold_into_edges(grad, ctx.shape, ctx.pml), None


def fold_into_edges(grad: torch.Tensor, shape: Sequence[int], pml: Sequence[int]) -> torch.Tensor:
    """Adjoint of the replicate pad: CPML-slab gradients summed onto the edge cells,
    one axis at a time (``_ExtendModel`` backward, ``model_setup.py:72-98``)."""
    for axis, n in enumerate(shape):
        lo, hi = int(pml[2 * axis]), int(pml[2 * axis + 1])
        inner = grad.narrow(axis, lo, n).clone()
        if lo:
            inner.select(axis, 0).add_(grad.narrow(axis, 0, lo).sum(dim=axis))
        if hi:
            inner.select(axis, n - 1).add_(grad.narrow(axis, lo + n, hi).sum(dim=axis))
        grad = inner
    return grad.contiguous()


def shift_locations(locations: torch.Tensor, pml: Sequence[int], device: Any) -> torch.Tensor:
    """Physical coordinates -> extended-grid int32 indices (model_setup.py:101-106)."""
    offset = torch.tensor([int(pml[0]), int(pml[2]), int(pml[4])], dtype=torch.int32, device=device)
    return (locations.to(device=device, dtype=torch.int32) + offset).contiguous()


def _as_3d(t: torch.Tensor, what: str) -> torch.Tensor:
    if t.ndim == 2:
        return t.reshape(*t.shape, 1)
    if t.ndim != 3:
        raise ValueError(f"The shape of {what} should be 2-d or 3-d.")
    return t


def _validate_locations(src: Any, rcv: Any, device: torch.device) -> Tuple[int, int, int]:
    if not torch.is_tensor(src) or not torch.is_tensor(rcv):
        raise TypeError("source_location and receiver_location must be PyTorch tensors.")
    if src.ndim != 3 or rcv.ndim != 3:
        raise ValueError("source_location and receiver_location must have shape (nstep, count, 3).")
    if src.shape[2] != 3 or rcv.shape[2] != 3:
        raise ValueError("The last dimension of source_location and receiver_location must be 3.")
    if src.shape[0] != rcv.shape[0]:
        raise ValueError("The first dimension (nstep) of source_location and receiver_location should be the same.")
    nstep, nsr, nrx = src.shape[0], src.shape[1], rcv.shape[1]
    if nstep < 1:
        raise ValueError("At least one shot is required.")
    if nsr < 1:
        raise ValueError("At least one source per shot is required.")
    if nrx < 1:
        raise ValueError("At least one receiver per shot is required.")
    if nstep > MAX_SHOTS_PER_CALL:
        raise ValueError(
            f"At most {MAX_SHOTS_PER_CALL} shots are supported in one compute call; split the batch."
        )
    for name, loc in (("source_location", src), ("receiver_location", rcv)):
        if loc.dtype == torch.bool or loc.is_complex():
            raise TypeError(f"{name} must contain real integer-valued coordinates.")
    return nstep, nsr, nrx


def _prepare_waveforms(w: Any, nsr: int, device: torch.device, dtype: torch.dtype) -> torch.Tensor:
    if not torch.is_tensor(w):
        raise TypeError("source_amplitudes must be a PyTorch tensor.")
    if w.ndim not in (2, 3):
        raise ValueError("source_amplitudes must have shape (num_waveforms, nt) or (num_waveforms, nt, 1).")
    if w.ndim == 2:
        w = w.unsqueeze(-1)
    if w.shape[2] != 1:
        raise ValueError("The last dimension of source_amplitudes must be 1.")
    if w.shape[0] < 1 or w.shape[1] < 1:
        raise ValueError("source_amplitudes must contain at least one waveform and one time sample.")
    w = w.to(device=device, dtype=dtype).contiguous()
    n = w.shape[0]
    if (1 < n < nsr) or n > nsr:
        raise ValueError("The number of source waveforms is incorrect.")
    if n == 1 and nsr != 1:
        w = w.repeat(nsr, 1, 1).contiguous()
    return w


def prepare_model(
    device: Any, eps_r: Any, sigma: Any, mu_r: Any, source_amplitudes: Any, source_location: Any,
    receiver_location: Any, dx: Any, dt: Any, pmlthick: Any, fdtd_order: int = 2,
    dtype: torch.dtype = torch.float32,
) -> PreparedModel:
    """Validate the physical model and build the solver-grid materials."""
    device = torch.device("cpu" if device is None else device)
    spacing = normalize_grid_spacing(dx)
    positive_finite("dt", dt)
    if not torch.is_tensor(eps_r) or not torch.is_tensor(sigma):
        raise TypeError("er and se must be PyTorch tensors.")
    eps_r = _as_3d(eps_r, "epsilon")
    sigma = _as_3d(sigma, "sigma")
    if mu_r is not None and not torch.is_tensor(mu_r):
        raise TypeError("mr must be a PyTorch tensor or None.")
    if mu_r is not None:
        mu_r = _as_3d(mu_r, "mr")
    if eps_r.shape != sigma.shape:
        raise ValueError("The shape of epsilon and sigma should be the same.")
    if any(n < 1 for n in eps_r.shape):
        raise ValueError("The material model dimensions must all be non-empty.")
    nx, ny, nz = eps_r.shape
    mode = 2 if nz == 1 else 3
    eps_r = eps_r.to(device=device, dtype=dtype)
    sigma = sigma.to(device=device, dtype=dtype)
    if mu_r is None:
        mu_r = torch.ones_like(eps_r, device=device)
    elif mu_r.shape == eps_r.shape:
        mu_r = mu_r.to(device=device, dtype=dtype)
    else:
        raise ValueError("The shape of mr should be the same as epsilon and sigma.")

    nstep, nsr, nrx = _validate_locations(source_location, receiver_location, device)
    source_location = source_location.to(device=device).contiguous()
    receiver_location = receiver_location.to(device=device).contiguous()
    waves = _prepare_waveforms(source_amplitudes, nsr, device, dtype)
    nt = waves.shape[1]

    pml = normalize_pml_thickness(pmlthick, nz)
    if nz == 1 and any(pml[4:]):
        raise ValueError("2D models require zero PML thickness on the z boundaries.")
    ext = extended_shape((nx, ny, nz), pml)
    if any(n >= INT32_MAX for n in ext):
        raise ValueError("Extended model dimensions must fit in positive int32 with a field halo.")

    # every scalar needed for validation in one device -> host transfer
    shape_t = torch.tensor((nx, ny, nz), dtype=torch.int32, device=device)

    def integral(loc: torch.Tensor) -> torch.Tensor:
        if loc.is_floating_point():
            return (torch.isfinite(loc) & (loc == loc.trunc())).all()
        return torch.ones((), dtype=torch.bool, device=device)

    stats = torch.stack(
        (
            torch.isfinite(eps_r).all().to(dtype),
            torch.isfinite(sigma).all().to(dtype),
            torch.isfinite(mu_r).all().to(dtype),
            torch.isfinite(waves).all().to(dtype),
            eps_r.amin(),
            sigma.amin(),
            mu_r.amin(),
            (eps_r.detach() * mu_r.detach()).amin(),
            ((source_location >= 0) & (source_location < shape_t)).all().to(dtype),
            ((receiver_location >= 0) & (receiver_location < shape_t)).all().to(dtype),
            integral(source_location).to(dtype),
            integral(receiver_location).to(dtype),
        )
    ).detach().cpu().tolist()
    for name, ok in zip(("er", "se", "mr", "source_amplitudes"), stats[:4]):
        if not ok:
            raise ValueError(f"`{name}` contains NaN or Inf values.")
    if stats[4] < MIN_RELATIVE_PERMITTIVITY:
        raise ValueError("The values of epsilon is incorrect.(should be greater than 1)")
    if stats[5] < 0:
        raise ValueError("The values of sigma is incorrect.(should be non-negative)")
    if stats[6] <= 0:
        raise ValueError("The values of mr are incorrect (must be positive).")
    if not stats[10]:
        raise ValueError("source_location must contain finite integer-valued coordinates.")
    if not stats[11]:
        raise ValueError("receiver_location must contain finite integer-valued coordinates.")
    if not stats[8]:
        raise ValueError(
            f"Error: Source coordinates out of range! Valid ranges are x∈[0,{nx}), y∈[0,{ny}), z∈[0,{nz})"
        )
    if not stats[9]:
        raise ValueError(
            f"Error: Receiver coordinates out of range! Valid ranges are x∈[0,{nx}), y∈[0,{ny}), z∈[0,{nz})"
        )
    check_cfl(spacing, dt, *ext, fdtd_order=fdtd_order, min_er_mr=stats[7])
    if any(pml):
        eps_r = ExtendIntoPML.apply(eps_r, pml)
        sigma = ExtendIntoPML.apply(sigma, pml)
        mu_r = ExtendIntoPML.apply(mu_r, pml)
    halo = (0, 1, 0, 1, 0, 1)
    return PreparedModel(
        eps_r, sigma, ext[0], ext[1], ext[2], nt, nstep, nsr, nrx,
        F.pad(eps_r, halo), F.pad(sigma, halo), F.pad(mu_r, halo), mode, dtype, pml, waves,
    )


def has_pec_cells(sigma: torch.Tensor) -> bool:
    """Whether any cell exceeds the PEC conductivity threshold."""
    return bool((sigma > PEC_CONDUCTIVITY_THRESHOLD).any())
