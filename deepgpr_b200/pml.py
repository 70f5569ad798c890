"""CPML profiles, update coefficients and the 24 auxiliary (psi) state arrays.

The absorbing profile is the reference's single-pole CFS CPML
(src/DeepGPR/solver/pml.py:69-181): kappa = 1, alpha = 0, a quartic sigma
graded from 0 to ``sigma_max = 0.8 (m + 1) eps0 v_ref / d`` with a fixed
reference speed ``v_ref``.  The coefficients RA, RB, RE, RF of every face are
evaluated with the same PyTorch operations in the same order and dtype as the
reference, on the CPU, so they are bit-identical; they are then copied to the
solver device.

Face order: x0, xm, y0, ym, z0, zm.  psi arrays per face: E psi1, E psi2,
H psi1, H psi2 with the shapes of :func:`psi_shapes`.
"""

from __future__ import annotations

import math
from typing import Any, List, Optional, Sequence, Tuple

import torch

from .config import CPML_SIGMA_MAX_FACTOR, CPML_SIGMA_ORDER, SPEED_OF_LIGHT, VACUUM_PERMITTIVITY
from .grid import normalize_grid_spacing, positive_finite

Shape = Tuple[int, ...]


def _graded_profiles(thickness: int, sigma_max: float) -> Tuple[torch.Tensor, torch.Tensor]:
    """Electric and magnetic samples of ``sigma_max * x**m`` on the staggered CPML cells.

    ``thickness + 1`` nodes are sampled at half-cell spacing on ``[0, p + 1/2]``,
    normalised by ``p``; the E profile takes the even samples and the H profile
    the odd ones, dropping the outermost node (pml.py:106-145).
    """
    n = thickness + 1
    ramp = (torch.linspace(0, (n - 1) + 0.5, steps=2 * n) / (n - 1)) ** CPML_SIGMA_ORDER
    e_prof = ramp[0:-1:2] * (sigma_max - 0) + 0
    h_prof = ramp[1::2] * (sigma_max - 0) + 0
    return e_prof[:-1], h_prof[:-1]


def _update_coefficients(sigma: torch.Tensor, dt: Any, out: torch.Tensor) -> None:
    """RA, RB, RE, RF of a CFS CPML with kappa = 1, alpha = 0 (pml.py:166-181)."""
    e0 = VACUUM_PERMITTIVITY
    kappa = torch.zeros(sigma.shape[0] + 1)[:-1] + 1
    alpha = torch.zeros(sigma.shape[0] + 1)[:-1] + 0
    denom = (2 * e0 * kappa) + dt * (alpha * kappa + sigma)
    out[0, 0, :] = (2 * e0 + dt * alpha) / denom
    out[1, 0, :] = (2 * e0 * kappa) / denom
    out[2, 0, :] = ((2 * e0 * kappa) - dt * (alpha * kappa + sigma)) / denom
    out[3, 0, :] = (2 * sigma * dt) / (kappa * denom)


def face_descriptor(face: int, p: int, nx: int, ny: int, nz: int) -> Tuple[int, ...]:
    """``(p, x0, x1, y0, y1, z0, z1)`` of one face on the extended grid (pml.py:184-194)."""
    return (
        (p, 0, p, 0, ny, 0, nz),
        (p, nx - p, nx, 0, ny, 0, nz),
        (p, 0, nx, 0, p, 0, nz),
        (p, 0, nx, ny - p, ny, 0, nz),
        (p, 0, nx, 0, ny, 0, p),
        (p, 0, nx, 0, ny, nz - p, nz),
    )[face]


def face_descriptors(nx: int, ny: int, nz: int, pml: Sequence[int]) -> Tuple[torch.Tensor, ...]:
    """Six int32 descriptors; a disabled face is an empty tensor."""
    return tuple(
        torch.tensor(face_descriptor(f, int(pml[f]), nx, ny, nz), dtype=torch.int) if int(pml[f]) > 0 else torch.empty(0)
        for f in range(6)
    )


def build_pml_coefficients(
    dt: Any, dx: Any, nx: int, ny: int, nz: int, pml: Sequence[int], device: Any, dtype: torch.dtype,
    *, max_velocity: float = SPEED_OF_LIGHT,
) -> Tuple[Tuple[torch.Tensor, ...], Tuple[torch.Tensor, ...]]:
    """Face descriptors and the 12 coefficient tensors ``x0_e, x0_h, xm_e, ...``.

    Each coefficient tensor has shape ``(4, 1, p)`` (RA, RB, RE, RF); disabled
    faces give empty tensors.
    """
    spacing = normalize_grid_spacing(dx)
    if isinstance(max_velocity, bool) or getattr(max_velocity, "requires_grad", False):
        raise TypeError("max_velocity must be a fixed finite positive scalar.")
    v_ref = positive_finite("max_velocity", max_velocity)
    coefficients: List[torch.Tensor] = []
    for face in range(6):
        p = int(pml[face])
        if p <= 0:
            coefficients.extend((torch.empty(0, device=device), torch.empty(0, device=device)))
            continue
        sigma_max = CPML_SIGMA_MAX_FACTOR * (CPML_SIGMA_ORDER + 1) * VACUUM_PERMITTIVITY * v_ref / spacing[face // 2]
        limits = torch.finfo(torch.get_default_dtype())
        if not math.isfinite(sigma_max) or not limits.tiny <= sigma_max <= limits.max:
            raise ValueError("max_velocity produces an unrepresentable PML absorption profile.")
        e_sig, h_sig = _graded_profiles(p, sigma_max)
        electric = torch.zeros((4, 1, p), dtype=dtype)
        magnetic = torch.zeros((4, 1, p), dtype=dtype)
        _update_coefficients(e_sig, dt, electric)
        _update_coefficients(h_sig, dt, magnetic)
        if not bool(torch.isfinite(electric).all() & torch.isfinite(magnetic).all()):
            raise ValueError("max_velocity produces non-finite PML update coefficients.")
        coefficients.extend((electric.to(device), magnetic.to(device)))
    return face_descriptors(nx, ny, nz, pml), tuple(coefficients)


def psi_shapes(face: int, p: int, nx: int, ny: int, nz: int, nstep: int) -> Tuple[Optional[Shape], ...]:
    """Shapes ``(E psi1, E psi2, H psi1, H psi2)`` of one face (pml.py:310-348)."""
    if p <= 0:
        return (None, None, None, None)
    _, x0, x1, y0, y1, z0, z1 = face_descriptor(face, p, nx, ny, nz)
    a, b, c = x1 - x0, y1 - y0, z1 - z0
    axis = face // 2
    if axis == 0:
        return ((nstep, a + 1, b, c + 1), (nstep, a + 1, b + 1, c), (nstep, a, b + 1, c), (nstep, a, b, c + 1))
    if axis == 1:
        return ((nstep, a, b + 1, c + 1), (nstep, a + 1, b + 1, c), (nstep, a + 1, b, c), (nstep, a, b, c + 1))
    return ((nstep, a, b + 1, c + 1), (nstep, a + 1, b, c + 1), (nstep, a + 1, b, c), (nstep, a, b + 1, c))


def build_psi(
    nx: int, ny: int, nz: int, pml: Sequence[int], nstep: int, supplied: Optional[Sequence[Any]], device: Any,
    dtype: torch.dtype = torch.float32,
) -> Tuple[torch.Tensor, ...]:
    """Allocate zero psi arrays or validate 24 supplied ones (pml.py:351-413).

    Supplied tensors already on ``device`` with ``dtype`` are returned as they
    are: the solver advances them in place.
    """
    if supplied is None:
        supplied = (None,) * 24
    elif not isinstance(supplied, (list, tuple)) or len(supplied) != 24:
        raise ValueError("PML must contain exactly 24 CPML auxiliary tensors.")
    out: List[torch.Tensor] = []
    for face in range(6):
        group = supplied[4 * face : 4 * face + 4]
        present = [v is not None for v in group]
        if any(present) and not all(present):
            raise ValueError(f"CPML face {face} must provide all four auxiliary tensors or none.")
        shapes = psi_shapes(face, int(pml[face]), nx, ny, nz, nstep)
        if all(present):
            if not all(torch.is_tensor(v) for v in group):
                raise TypeError(f"CPML face {face} state must contain PyTorch tensors.")
            for slot, (tensor, shape) in enumerate(zip(group, shapes)):
                if shape is None:
                    if tensor.numel() != 0:
                        raise ValueError(f"CPML face {face} component {slot} must be empty.")
                elif tuple(tensor.shape) != shape:
                    raise ValueError(
                        f"CPML face {face} component {slot} has shape {tuple(tensor.shape)}; expected {shape}."
                    )
                out.append(tensor.to(device=device, dtype=dtype).contiguous())
        elif shapes[0] is not None:
            out.extend(torch.zeros(shape, dtype=dtype, device=device) for shape in shapes)
        else:
            out.extend(torch.empty(0, dtype=dtype, device=device) for _ in range(4))
    return tuple(out)
