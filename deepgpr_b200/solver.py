"""``compute()`` and its autograd function: the drop-in for ``DeepGPR.compute``.

Contract (src/DeepGPR/solver/modeling.py:261-671, src/DeepGPR/solver/autograd.py:486-760):

* ``compute(...)`` returns ``(E_saved, (Ex, Ey, Ez), (Hx, Hy, Hz), PML, receivers)``
  with ``receivers`` of shape ``(nstep, nt, nrx)``;
* the 30 state tensors are advanced in place and are differentiable inputs
  and outputs; ``eps_r``, ``sigma`` and ``source_amplitudes`` get gradients
  from the exact discrete adjoint; material gradients have the physical
  model's shape (the CPML sensitivities are folded onto the edge cells).

Everything runs in the CUDA library; a CPU device raises.  Two additions:
``wavefield_compression="fp8"`` (E4M3 histories with per-tile scales; ``"int8"``
gives integer codes on the same tiles) and the
keyword ``precision=torch.float64`` (the same kernels instantiated in double,
used as the FP64 reference of the FP32 path).
"""

from __future__ import annotations

import math
import warnings
import dataclasses
from dataclasses import dataclass
from datetime import datetime
from typing import Any, Dict, Optional, Sequence, Tuple

import torch

from . import native
from .config import (
    CPML_FACES,
    DEFAULT_FDTD_ORDER,
    DEFAULT_GRADIENT_MODE,
    DEFAULT_PML_THICKNESS,
    DEFAULT_RECEIVER_COMPONENT,
    DEFAULT_SAMPLING_INTERVAL,
    DEFAULT_SOURCE_COMPONENT,
    FIELD_COMPONENTS,
    SPEED_OF_LIGHT,
    STATE_COUNT,
    STATE_NAMES,
    SUPPORTED_FDTD_ORDERS,
    SUPPORTED_GRADIENT_MODES,
    TM2D_INACTIVE_STATES,
)
from .errors import NativeLibraryError, NonFiniteTensorError
from .grid import normalize_grid_spacing, positive_finite
from .history_io import normalize_forward_wavefield_directory, save_forward_wavefield
from .model import fold_into_edges, prepare_model, shift_locations
from .pml import build_pml_coefficients, build_psi, face_descriptors
from .storage import (
    StorageConfig,
    allocate_history,
    encode_storage_type,
    history_box,
    normalize_choice,
    normalize_compression,
    normalize_storage_dtype,
    resolve_rhs_reconstruction,
    saved_history_shape,
    saved_time_steps,
    storage_config,
)


@dataclass(frozen=True)
class SolverConfig:
    """Scalar description of one solve (not differentiated)."""

    device: torch.device
    dtype: torch.dtype
    spacing: Tuple[float, float, float]
    dt: float
    nx: int
    ny: int
    nz: int
    nt: int
    nstep: int
    nsr: int
    nrx: int
    pml: Tuple[int, ...]
    source_component: int
    receiver_component: int
    interval: int
    storage: StorageConfig
    save_history: bool
    offload: bool
    fdtd_order: int
    mode: int
    debug: bool
    reconstruct_rhs: bool
    region: str
    acc64: bool = True
    tm2d: bool = False
    chunk: int = 32                                     # time steps per captured graph
    tuning: Tuple[int, int, int, int] = (0, 0, 0, -1)   # dgb_set_tuning (see deepgpr_b200.autotune)

    @property
    def field_shape(self) -> Tuple[int, int, int]:
        return (self.nx + 1, self.ny + 1, self.nz + 1)

    @property
    def history_cells(self) -> Tuple[int, int, int]:
        return history_box(self.nx, self.ny, self.nz, self.pml, self.region)[1]

    @property
    def entry(self) -> Tuple[str, str]:
        return ("forward", "backward") if self.dtype == torch.float32 else ("dgb_forward_f64", "dgb_backward_f64")


@dataclass(frozen=True)
class SolverTensors:
    """Non-differentiated solver inputs."""

    eps_r_pad: torch.Tensor
    sigma_pad: torch.Tensor
    mu_r_pad: torch.Tensor
    source_location: torch.Tensor
    receiver_location: torch.Tensor
    pml_coefficients: Tuple[torch.Tensor, ...]


def _common_args(cfg: SolverConfig) -> Dict[str, Any]:
    dx, dy, dz = cfg.spacing
    args: Dict[str, Any] = {
        "dt": cfg.dt, "nt": cfg.nt, "nshot": cfg.nstep, "nreceiver": cfg.nrx, "dx": dx, "dy": dy, "dz": dz,
        "nx_fields": cfg.nx + 1, "ny_fields": cfg.ny + 1, "nz_fields": cfg.nz + 1,
        "receiver_component": cfg.receiver_component, "source_component": cfg.source_component,
        "nsource": cfg.nsr, "sampling_interval": cfg.interval, "fwi_mode": cfg.mode,
    }
    for face, p in zip(CPML_FACES, cfg.pml):
        args[f"pml_{face}"] = p
    return args


def _coefficient_args(coefficients: Sequence[torch.Tensor]) -> Dict[str, torch.Tensor]:
    out = {}
    for f, face in enumerate(CPML_FACES):
        out[f"{face}_e_coeff"] = coefficients[2 * f]
        out[f"{face}_h_coeff"] = coefficients[2 * f + 1]
    return out


def _update_scratch(cfg: SolverConfig) -> Dict[str, torch.Tensor]:
    buf = torch.zeros((6, cfg.nx + 1, cfg.ny + 1, cfg.nz + 1), device=cfg.device, dtype=cfg.dtype)
    return dict(zip(native.COEFF_NAMES, buf.unbind(0)))


def forward_arguments(cfg: SolverConfig, tensors: SolverTensors, states: Sequence[torch.Tensor], e_saved: Any,
                      r_saved: Any, receivers: Any, waveform: Any, storage_type: int, save_model: bool) -> Dict[str, Any]:
    """Name -> value mapping of the native ``forward`` call (no tensor work)."""
    args = _common_args(cfg)
    args.update(_update_scratch(cfg))
    args.update(_coefficient_args(tensors.pml_coefficients))
    args.update(
        eps_r_pad=tensors.eps_r_pad, sigma_pad=tensors.sigma_pad, mu_r_pad=tensors.mu_r_pad,
        E_saved=e_saved, R_saved=r_saved, Ex=states[0], Ey=states[1], Ez=states[2], Hx=states[3], Hy=states[4],
        Hz=states[5], receiver_location=tensors.receiver_location, receiver_data=receivers,
        source_location=tensors.source_location, source_waveform=waveform, storage_type=storage_type,
        save_model_history=int(save_model), use_async_offload=int(cfg.offload),
    )
    args.update(zip(native.PHI_NAMES, states[6:]))
    return args


def backward_arguments(cfg: SolverConfig, tensors: SolverTensors, lambdas: Sequence[torch.Tensor], e_saved: Any,
                       r_saved: Any, data_grad: Any, grad_source: Any, grad_eps: Any, grad_sigma: Any,
                       want: Tuple[bool, bool, bool], storage_type: int) -> Dict[str, Any]:
    """Name -> value mapping of the native ``backward`` call."""
    args = _common_args(cfg)
    args.update(_update_scratch(cfg))
    args.update(_coefficient_args(tensors.pml_coefficients))
    args.update(
        eps_r_pad=tensors.eps_r_pad, sigma_pad=tensors.sigma_pad, mu_r_pad=tensors.mu_r_pad,
        E_saved=e_saved, R_saved=r_saved, ndata_source=cfg.nrx, receiver_location=tensors.receiver_location,
        data_grad=data_grad, source_location=tensors.source_location, grad_source=grad_source,
        source_requires_grad=int(want[0]), grad_eps_r=grad_eps, grad_sigma=grad_sigma,
        eps_r_requires_grad=int(want[1]), sigma_requires_grad=int(want[2]), storage_type=storage_type,
        use_async_offload=int(cfg.offload),
    )
    names = ("lambda_ex", "lambda_ey", "lambda_ez", "lambda_hx", "lambda_hy", "lambda_hz") + native.LAMBDA_PHI_NAMES
    args.update(zip(names, lambdas))
    return args


def _check_finite(where: str, **tensors: torch.Tensor) -> None:
    bad = [n for n, t in tensors.items() if t is not None and t.numel() and t.is_floating_point()
           and not bool(torch.isfinite(t).all())]
    if bad:
        raise NonFiniteTensorError(f"{where}: non-finite values in {', '.join(bad)}")


class FDTDFunction(torch.autograd.Function):
    """``apply(cfg, tensors, eps_r, sigma, source_amplitudes, *30 states)``.

    Returns the 30 states (advanced in place), ``E_saved`` and the receiver
    data ``(nstep, nt, nrx)``.
    """

    @staticmethod
    def forward(ctx, cfg: SolverConfig, tensors: SolverTensors, eps_r, sigma, source_amplitudes, *states):  # type: ignore[override]
        if len(states) != STATE_COUNT:
            raise ValueError(f"Expected {STATE_COUNT} state tensors, got {len(states)}.")
        ctx.set_materialize_grads(False)
        want_model = bool(eps_r.requires_grad or sigma.requires_grad)
        save_model = cfg.save_history and want_model
        rhs_from_e = bool(cfg.reconstruct_rhs and save_model)
        storage_type = encode_storage_type(cfg.storage, cfg.save_history, rhs_from_e, cfg.region == "physical",
                                           cfg.tm2d)
        nt_saved = saved_time_steps(cfg.nt, cfg.interval)
        shape = saved_history_shape(cfg.mode, nt_saved, cfg.nstep, *cfg.history_cells)
        dev = cfg.device
        if cfg.save_history:
            e_saved = allocate_history(cfg.storage, shape, cfg.field_shape, cfg.tm2d, dev, cfg.offload)
            if rhs_from_e:
                r_saved = allocate_history(cfg.storage, saved_history_shape(cfg.mode, 1, cfg.nstep, *cfg.history_cells),
                                           cfg.field_shape, cfg.tm2d, dev, False)
            elif save_model:
                r_saved = allocate_history(cfg.storage, shape, cfg.field_shape, cfg.tm2d, dev, cfg.offload)
            else:
                r_saved = torch.empty(0, device=dev, dtype=cfg.storage.dtype)
        else:
            e_saved = torch.empty(0, device=dev, dtype=cfg.storage.dtype)
            r_saved = torch.empty(0, device=dev, dtype=cfg.storage.dtype)
        receivers = torch.empty((cfg.nstep, cfg.nt, cfg.nrx), device=dev, dtype=cfg.dtype)
        waveform = source_amplitudes.detach().contiguous()
        args = forward_arguments(cfg, tensors, states, e_saved, r_saved, receivers, waveform, storage_type, save_model)
        native.invoke(cfg.entry[0], args, fdtd_order=cfg.fdtd_order, stream=torch.cuda.current_stream(dev),
                      acc64=cfg.acc64, chunk=cfg.chunk, tuning=cfg.tuning)
        if cfg.debug:
            _check_finite("forward", receivers=receivers, **dict(zip(STATE_NAMES, states)))
        ctx.cfg = cfg
        ctx.tensors = tensors
        ctx.want = (bool(source_amplitudes.requires_grad), bool(eps_r.requires_grad), bool(sigma.requires_grad))
        ctx.source_shape = tuple(source_amplitudes.shape)
        ctx.state_shapes = tuple(s.shape for s in states)
        ctx.storage_type = storage_type
        ctx.histories = (e_saved, r_saved) if cfg.save_history else None
        ctx.mark_non_differentiable(e_saved)
        return (*states, e_saved, receivers)

    @staticmethod
    def backward(ctx, *grads):  # type: ignore[override]
        cfg: SolverConfig = ctx.cfg
        if not cfg.save_history:
            raise RuntimeError("Forward wavefield history is disabled; adjoint/model-gradient backward is unavailable.")
        if ctx.histories is None:
            raise RuntimeError(
                "The saved forward wavefield was already released by a previous backward pass; "
                "re-run compute before calling backward again."
            )
        dev, dtype = cfg.device, cfg.dtype
        lambdas = [
            torch.zeros(shape, device=dev, dtype=dtype) if g is None else g.clone(memory_format=torch.contiguous_format)
            for g, shape in zip(grads[:STATE_COUNT], ctx.state_shapes)
        ]
        data_grad = grads[STATE_COUNT + 1]
        data_grad = (torch.zeros((cfg.nstep, cfg.nt, cfg.nrx), device=dev, dtype=dtype) if data_grad is None
                     else data_grad.to(dtype).contiguous())
        want_src, want_eps, want_sig = ctx.want
        ext = (cfg.nx, cfg.ny, cfg.nz)
        grad_eps = torch.zeros(ext, device=dev, dtype=dtype) if want_eps else torch.empty(0, device=dev, dtype=dtype)
        grad_sig = torch.zeros(ext, device=dev, dtype=dtype) if want_sig else torch.empty(0, device=dev, dtype=dtype)
        grad_src = torch.zeros(ctx.source_shape, device=dev, dtype=dtype) if want_src else torch.empty(0, device=dev, dtype=dtype)
        e_saved, r_saved = ctx.histories
        args = backward_arguments(cfg, ctx.tensors, lambdas, e_saved, r_saved, data_grad, grad_src, grad_eps,
                                  grad_sig, ctx.want, ctx.storage_type)
        native.invoke(cfg.entry[1], args, fdtd_order=cfg.fdtd_order, stream=torch.cuda.current_stream(dev),
                      acc64=cfg.acc64, chunk=cfg.chunk, tuning=cfg.tuning)
        ctx.histories = None
        if cfg.tm2d:
            # Ex, Ey, Hz and their CPML arrays never couple back on the 2D TM path
            for i in TM2D_INACTIVE_STATES:
                lambdas[i].zero_()
        state_needs = ctx.needs_input_grad[5 : 5 + STATE_COUNT]
        if cfg.debug:
            checks = {n: g for n, g, need in zip(STATE_NAMES, lambdas, state_needs) if need}
            if want_eps:
                checks["grad_eps_r"] = grad_eps
            if want_sig:
                checks["grad_sigma"] = grad_sig
            if want_src:
                checks["grad_source"] = grad_src
            _check_finite("backward", **checks)
        return (
            None, None,
            grad_eps if want_eps else None,
            grad_sig if want_sig else None,
            grad_src if want_src else None,
            *(g if need else None for g, need in zip(lambdas, state_needs)),
        )


def _fields(supplied: Any, nx: int, ny: int, nz: int, nstep: int, device: Any, dtype: torch.dtype):
    shape = (nstep, nx + 1, ny + 1, nz + 1)
    if supplied is None:
        return tuple(torch.zeros(shape, device=device, dtype=dtype) for _ in range(3))
    if not isinstance(supplied, (list, tuple)) or len(supplied) != 3:
        raise ValueError("E and H must each contain exactly three field tensors.")
    for t in supplied:
        if not torch.is_tensor(t) or tuple(t.shape) != shape:
            raise ValueError(f"Field shape mismatch: got {getattr(t, 'shape', None)}, expected {shape}.")
    return tuple(t.to(device=device, dtype=dtype).contiguous() for t in supplied)


def _tm2d_applies(spatial_mode: int, source_component: int, mode: int, stores_model: bool,
                  states: Sequence[torch.Tensor], supplied: bool) -> bool:
    """Whether the 2D Ez-TM kernels reproduce the general solver exactly.

    As src/DeepGPR/solver/modeling.py:226-258: in 2D (nz = 1) with an Ez source
    and zero Ex, Ey, Hz (and the CPML arrays that couple them) those fields stay
    zero, so advancing only Ez, Hx, Hy gives the same result.  Gradient mode 3
    histories keep the general path here.
    """
    if spatial_mode != 2 or source_component != 2 or (stores_model and mode != 2):
        return False
    if not supplied:
        return True
    inactive = [states[i] for i in TM2D_INACTIVE_STATES if states[i].numel()]
    return int(sum(t.detach().count_nonzero() for t in inactive)) == 0 if inactive else True


def _alias(name: str, value: Any, alias: str, alias_value: Any) -> Any:
    if value is not None and alias_value is not None:
        raise TypeError(f"Specify only one of {name} and its deprecated alias {alias}.")
    return alias_value if value is None else value


def _prepare_solve(
    device,
    dx=None,
    dt=None,
    source_amplitudes=None,
    source_location=None,
    receiver_location=None,
    er=None,
    se=None,
    mr=None,
    E=None,
    H=None,
    PML=None,
    pmlthick=DEFAULT_PML_THICKNESS,
    source_direction=DEFAULT_SOURCE_COMPONENT,
    reciever_direction=DEFAULT_RECEIVER_COMPONENT,
    model_gradient_sampling_interval=DEFAULT_SAMPLING_INTERVAL,
    wavefield_storage_dtype=torch.float32,
    use_async_offload=False,
    fdtd_order=DEFAULT_FDTD_ORDER,
    mode=DEFAULT_GRADIENT_MODE,
    debug=False,
    print_parameters=False,
    save_forward_wavefield_path=None,
    *,
    eps_r=None,
    sigma=None,
    mu_r=None,
    receiver_component=None,
    save_wavefield_history=True,
    wavefield_compression="none",
    wavefield_compression_block_size=None,
    wavefield_conversion_backend="auto",
    int8_reduction_backend="auto",
    wavefield_compression_rate=None,
    wavefield_rhs_history="auto",
    wavefield_history_region="extended",
    pml_max_velocity=SPEED_OF_LIGHT,
    precision=torch.float32,
    gradient_accumulation="float64",
):
    """Validation and preparation of ``compute``: the solver configuration, the
    prepared tensors and model, and the 30 input states."""
    eps_r = _alias("eps_r", eps_r, "er", er)
    sigma = _alias("sigma", sigma, "se", se)
    mu_r = _alias("mu_r", mu_r, "mr", mr)
    receiver_component = reciever_direction if receiver_component is None else receiver_component
    if isinstance(pml_max_velocity, bool) or getattr(pml_max_velocity, "requires_grad", False):
        raise TypeError("pml_max_velocity must be a fixed finite positive scalar.")
    v_ref = positive_finite("pml_max_velocity", pml_max_velocity)
    device = torch.device(device)
    if device.type != "cuda":
        raise NativeLibraryError("deepgpr_b200 solves on CUDA devices only (there is no CPU backend).")
    if fdtd_order not in SUPPORTED_FDTD_ORDERS:
        raise ValueError("fdtd_order must be one of 2, 4, or 8.")
    if mode not in SUPPORTED_GRADIENT_MODES:
        raise ValueError("mode must be 2 or 3.")
    for name, value in (("print_parameters", print_parameters), ("save_wavefield_history", save_wavefield_history)):
        if not isinstance(value, bool):
            raise TypeError(f"{name} must be a bool.")
    if precision not in (torch.float32, torch.float64):
        raise ValueError("precision must be torch.float32 or torch.float64.")
    acc = normalize_choice("gradient_accumulation", gradient_accumulation, ("float64", "float32"))
    interval = model_gradient_sampling_interval
    if isinstance(interval, str):
        raise ValueError("model_gradient_sampling_interval='auto' is not provided; pass a positive integer.")
    if isinstance(interval, bool) or not isinstance(interval, int) or interval < 1:
        raise ValueError("model_gradient_sampling_interval must be a positive integer or 'auto'.")
    storage_dtype = normalize_storage_dtype(wavefield_storage_dtype)
    compression = normalize_compression(wavefield_compression)
    int8_request = compression == "int8"
    normalize_choice("wavefield_conversion_backend", wavefield_conversion_backend,
                     ("auto", "legacy", "native_scalar", "native_vec2"))
    normalize_choice("int8_reduction_backend", int8_reduction_backend, ("auto", "current", "cub_block", "warp_shuffle"))
    if wavefield_compression_rate is not None:
        raise ValueError("wavefield_compression_rate is only meaningful for the optional ZFP backend.")
    if wavefield_compression_block_size is not None and not int8_request:
        raise ValueError("wavefield_compression_block_size applies to the reference's INT8 format only.")
    if compression in ("fp8", "int8") and storage_dtype != torch.float32:
        raise ValueError(f"wavefield_storage_dtype must stay float32 with wavefield_compression='{compression}'.")
    if not save_wavefield_history and use_async_offload:
        raise ValueError("use_async_offload=True is incompatible with save_wavefield_history=False.")
    if use_async_offload and compression in ("fp8", "int8"):
        raise ValueError("use_async_offload=True is incompatible with device-resident one-byte (FP8 / INT8) histories.")
    if save_forward_wavefield_path is not None and not save_wavefield_history:
        raise ValueError("save_forward_wavefield_path requires save_wavefield_history=True.")
    rhs_mode = normalize_choice("wavefield_rhs_history", wavefield_rhs_history, ("auto", "stored", "reconstructed"))
    region = normalize_choice("wavefield_history_region", wavefield_history_region, ("extended", "physical"))
    if source_direction not in FIELD_COMPONENTS or receiver_component not in FIELD_COMPONENTS:
        raise ValueError("source_direction and receiver_component must be 0, 1, or 2.")
    if getattr(mu_r, "requires_grad", False):
        raise NotImplementedError("Relative-permeability gradients are not provided.")

    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    spacing = normalize_grid_spacing(dx)
    prepared = prepare_model(device, eps_r, sigma, mu_r, source_amplitudes, source_location, receiver_location,
                             spacing, dt, pmlthick, fdtd_order, dtype=precision)
    nx, ny, nz, nt = prepared.nx, prepared.ny, prepared.nz, prepared.nt
    pml = prepared.pml
    src_loc = shift_locations(source_location, pml, device)
    rcv_loc = shift_locations(receiver_location, pml, device)
    want_model = bool(prepared.eps_r.requires_grad or prepared.sigma.requires_grad)
    stores_model = save_wavefield_history and want_model
    if stores_model and region == "physical" and any(pml):
        raise ValueError("wavefield_history_region='physical' omits PML material sensitivities. "
                         "Use 'extended' for material gradients with PML.")
    if stores_model and mode == 2 and (prepared.mode != 2 or source_direction != 2 or receiver_component != 2):
        raise ValueError("mode=2 is an exact model-gradient mode only for 2D Ez-TM modeling. "
                         "Use mode=3 for 3D or other electric-field components.")
    lossless = compression == "none" and storage_dtype == torch.float32
    if compression in ("fp8", "int8") and rhs_mode == "reconstructed":
        raise ValueError("One-byte histories keep the E and R pair; use wavefield_rhs_history='stored' or 'auto'.")
    reconstruct = resolve_rhs_reconstruction(rhs_mode, interval, stores_model,
                                             lossless or precision == torch.float64)
    storage = storage_config(storage_dtype, compression, precision)
    if print_parameters:
        print(f"deepgpr_b200.compute: grid ({nx}, {ny}, {nz}) + halo, nt {nt}, shots {prepared.nstep}, "
              f"sources {prepared.nsr}, receivers {prepared.nrx}, order {fdtd_order}, mode {mode}, "
              f"history {'off' if not save_wavefield_history else storage.kind}, pml {pml}, device {device}")

    electric = _fields(E, nx, ny, nz, prepared.nstep, device, precision)
    magnetic = _fields(H, nx, ny, nz, prepared.nstep, device, precision)
    _, coefficients = build_pml_coefficients(dt, spacing, nx, ny, nz, pml, device, precision, max_velocity=v_ref)
    psi = build_psi(nx, ny, nz, pml, prepared.nstep, PML, device, precision)
    tm2d = _tm2d_applies(prepared.mode, source_direction, mode, stores_model, (*electric, *magnetic, *psi),
                         E is not None or H is not None or PML is not None)
    cfg = SolverConfig(
        device=device, dtype=precision, spacing=spacing, dt=float(dt), nx=nx, ny=ny, nz=nz, nt=nt,
        nstep=prepared.nstep, nsr=prepared.nsr, nrx=prepared.nrx, pml=pml, source_component=source_direction,
        receiver_component=receiver_component, interval=interval, storage=storage,
        save_history=save_wavefield_history, offload=bool(use_async_offload), fdtd_order=fdtd_order, mode=mode,
        debug=bool(debug), reconstruct_rhs=reconstruct, region=region, acc64=(acc == "float64"), tm2d=tm2d,
    )
    tensors = SolverTensors(
        eps_r_pad=prepared.eps_r_pad.detach().contiguous(), sigma_pad=prepared.sigma_pad.detach().contiguous(),
        mu_r_pad=prepared.mu_r_pad.detach().contiguous(), source_location=src_loc, receiver_location=rcv_loc,
        pml_coefficients=tuple(c.contiguous() for c in coefficients),
    )
    return cfg, tensors, prepared, (*electric, *magnetic, *psi)


def compute(
    device,
    dx=None,
    dt=None,
    source_amplitudes=None,
    source_location=None,
    receiver_location=None,
    er=None,
    se=None,
    mr=None,
    E=None,
    H=None,
    PML=None,
    pmlthick=DEFAULT_PML_THICKNESS,
    source_direction=DEFAULT_SOURCE_COMPONENT,
    reciever_direction=DEFAULT_RECEIVER_COMPONENT,
    model_gradient_sampling_interval=DEFAULT_SAMPLING_INTERVAL,
    wavefield_storage_dtype=torch.float32,
    use_async_offload=False,
    fdtd_order=DEFAULT_FDTD_ORDER,
    mode=DEFAULT_GRADIENT_MODE,
    debug=False,
    print_parameters=False,
    save_forward_wavefield_path=None,
    *,
    eps_r=None,
    sigma=None,
    mu_r=None,
    receiver_component=None,
    save_wavefield_history=True,
    wavefield_compression="none",
    wavefield_compression_block_size=None,
    wavefield_conversion_backend="auto",
    int8_reduction_backend="auto",
    wavefield_compression_rate=None,
    wavefield_rhs_history="auto",
    wavefield_history_region="extended",
    pml_max_velocity=SPEED_OF_LIGHT,
    precision=torch.float32,
    gradient_accumulation="float64",
    checkpoint_segments=None,
    checkpoint_shot_batch=None,
    autotune=False,
):
    """2D/3D Maxwell FDTD forward modelling with an exact discrete adjoint on B200.

    Arguments and return value are those of ``DeepGPR.compute``; see the module
    docstring for the two additions (``wavefield_compression="fp8"``,
    ``precision``) and ``gradient_accumulation`` (``"float64"``: the material
    gradient is summed over shots and time in FP64; ``"float32"``: in FP32 in
    the reference's order).

    ``checkpoint_segments`` (default ``None``: off, as the reference) runs a
    solve whose material gradient is wanted with segment checkpointing and
    recompute (``deepgpr_b200.checkpoint``): an integer is the segment length
    in time steps; ``"auto"`` checkpoints only when the whole history would
    not fit 80 % of the free device memory, with the longest segments that do.
    ``checkpoint_shot_batch`` fixes the shots per backward batch.  A
    checkpointed solve returns an empty ``E_saved`` (no full history exists).

    ``autotune=True`` picks the launch shapes of the solve with
    ``deepgpr_b200.autotune`` (short probe solves the first time a problem
    signature is seen, a kept choice afterwards); results do not change.
    """
    args = dict(locals())
    segments = args.pop("checkpoint_segments")
    shot_batch = args.pop("checkpoint_shot_batch")
    tune = args.pop("autotune")
    output_directory = normalize_forward_wavefield_directory(save_forward_wavefield_path)
    run_time = datetime.now() if output_directory is not None else None
    cfg, tensors, prepared, states_in = _prepare_solve(**args)
    if tune:
        from .autotune import default_tuner, tuning_tuple

        choice = default_tuner().choose(cfg, tensors, states_in, prepared.source_amplitudes)
        cfg = dataclasses.replace(cfg, chunk=int(choice["chunk"]), tuning=tuning_tuple(choice))
    plan = _checkpoint_plan(cfg, prepared, states_in, segments, shot_batch)
    if plan is not None:
        if output_directory is not None:
            raise ValueError("save_forward_wavefield_path needs the full history; it cannot be combined with "
                             "checkpoint_segments.")
        if cfg.offload:
            raise ValueError("use_async_offload=True cannot be combined with checkpoint_segments.")
        from .checkpoint import CheckpointedFDTDFunction

        outputs = CheckpointedFDTDFunction.apply(cfg, tensors, plan, prepared.eps_r, prepared.sigma,
                                                 prepared.source_amplitudes, *states_in)
        states, e_saved, receivers = outputs[:STATE_COUNT], outputs[STATE_COUNT], outputs[STATE_COUNT + 1]
        return e_saved, tuple(states[0:3]), tuple(states[3:6]), tuple(states[6:30]), receivers
    outputs = FDTDFunction.apply(cfg, tensors, prepared.eps_r, prepared.sigma, prepared.source_amplitudes,
                                 *states_in)
    states, e_saved, receivers = outputs[:STATE_COUNT], outputs[STATE_COUNT], outputs[STATE_COUNT + 1]
    if output_directory is not None:
        # reference file scheme (solver/modeling.py:640-663)
        origin, cells = history_box(cfg.nx, cfg.ny, cfg.nz, cfg.pml, cfg.region)
        shape = saved_history_shape(cfg.mode, saved_time_steps(cfg.nt, cfg.interval), cfg.nstep, *cells)
        metadata = None
        if cfg.storage.compression in ("fp8", "int8"):
            metadata = {"compression": cfg.storage.compression, "uncompressed_shape": shape,
                        "field_shape": cfg.field_shape,
                        "history_origin": origin, "tm2d": cfg.tm2d}
        if cfg.region == "physical":
            metadata = dict(metadata or {})
            metadata.update(history_region="physical", history_origin=origin, pmlthick=cfg.pml,
                            uncompressed_shape=shape)
        save_forward_wavefield(e_saved, output_directory, run_time, metadata=metadata)
    return e_saved, tuple(states[0:3]), tuple(states[3:6]), tuple(states[6:30]), receivers


def _checkpoint_plan(cfg: SolverConfig, prepared, states, segments, shot_batch):
    """The segment plan of a checkpointed solve, or None for a single-call solve."""
    if segments is None or segments is False:
        if shot_batch is not None:
            raise ValueError("checkpoint_shot_batch needs checkpoint_segments.")
        return None
    auto = isinstance(segments, str)
    if auto and segments != "auto":
        raise ValueError("checkpoint_segments must be None, 'auto' or a positive number of time steps.")
    if not auto and (isinstance(segments, bool) or not isinstance(segments, int) or segments < 1):
        raise ValueError("checkpoint_segments must be None, 'auto' or a positive number of time steps.")
    if shot_batch is not None and (isinstance(shot_batch, bool) or not isinstance(shot_batch, int)
                                   or not 1 <= shot_batch <= cfg.nstep):
        raise ValueError("checkpoint_shot_batch must be an integer between 1 and the shot count.")
    if not auto and segments % cfg.interval:
        raise ValueError("checkpoint_segments must be a multiple of model_gradient_sampling_interval.")
    want_model = bool(prepared.eps_r.requires_grad or prepared.sigma.requires_grad)
    if not (cfg.save_history and want_model and torch.is_grad_enabled()):
        return None   # no history is needed: nothing to checkpoint
    from .checkpoint import plan_segments, state_bytes_per_shot

    free, _ = torch.cuda.mem_get_info(cfg.device)
    budget = int(0.7 * free)
    state = state_bytes_per_shot(states, cfg.nstep)
    plan = plan_segments(cfg, state, budget, None if auto else min(segments, cfg.nt), shot_batch)
    if auto and plan.nsegments == 1 and plan.shot_batch >= cfg.nstep:
        return None   # the whole history fits
    return plan


class _DirectContext:
    """The autograd context's part that FDTDFunction uses, for calls made
    directly on the calling thread."""

    def __init__(self, needs_input_grad):
        self.needs_input_grad = needs_input_grad

    def set_materialize_grads(self, value):
        pass

    def mark_non_differentiable(self, *tensors):
        pass


def misfit_gradient(device, observed, **kwargs):
    """L2-misfit gradient of one solve, forward and adjoint run on the calling thread.

    Takes ``compute``'s arguments (keywords, ``eps_r`` and ``sigma`` required)
    and ``observed`` receiver data shaped like ``compute``'s receivers.
    Returns ``(loss, grad_eps_r, grad_sigma, receivers)``: the gradients of
    ``0.5 * sum((receivers - observed) ** 2)`` with respect to the physical
    ``eps_r`` and ``sigma``, the values ``loss.backward()`` after ``compute``
    gives.  The native adjoint is called from this thread instead of the
    autograd engine's single per-device thread, so gradient solves issued by
    several threads (each on its own CUDA stream) overlap on the GPU.
    """
    eps = kwargs.pop("eps_r").detach().requires_grad_(True)
    sig = kwargs.pop("sigma").detach().requires_grad_(True)
    cfg, tensors, prepared, states = _prepare_solve(device=device, eps_r=eps, sigma=sig, **kwargs)
    ctx = _DirectContext((False, False, True, True, False) + (False,) * STATE_COUNT)
    with torch.no_grad():
        outs = FDTDFunction.forward(ctx, cfg, tensors, prepared.eps_r, prepared.sigma, prepared.source_amplitudes,
                                    *states)
        receivers = outs[STATE_COUNT + 1]
        resid = receivers - observed.to(device=receivers.device, dtype=receivers.dtype)
        loss = 0.5 * (resid * resid).sum()
        grads = FDTDFunction.backward(ctx, *([None] * (STATE_COUNT + 1)), resid)
        pml = prepared.pml
        phys = tuple(n - pml[2 * a] - pml[2 * a + 1] for a, n in enumerate(prepared.eps_r.shape))
        g_eps = fold_into_edges(grads[2], phys, pml).reshape(eps.shape)
        g_sig = fold_into_edges(grads[3], phys, pml).reshape(sig.shape)
    return loss, g_eps, g_sig, receivers


def checkpoint_initial_field(device=None, per_nstep=None, dx=None, dt=None, source_amplitudes=None,
                             source_location=None, receiver_location=None, er=None, se=None, mr=None,
                             pmlthick=DEFAULT_PML_THICKNESS, fdtd_order=2, precision=torch.float32):
    """Zero ``((Ex, Ey, Ez), (Hx, Hy, Hz), PML24)`` on the solver grid (src/DeepGPR/solver/fields.py:63-143)."""
    prepared = prepare_model(device, er, se, mr, source_amplitudes, source_location, receiver_location, dx, dt,
                             pmlthick, fdtd_order, dtype=precision)
    nx, ny, nz, nstep = prepared.nx, prepared.ny, prepared.nz, prepared.nstep
    if per_nstep is not None:
        if isinstance(per_nstep, bool) or not isinstance(per_nstep, int):
            raise TypeError("per_nstep must be an integer shot count or None.")
        if not 1 <= per_nstep <= nstep:
            raise ValueError("per_nstep must be between 1 and the input shot count.")
    electric = _fields(None, nx, ny, nz, nstep, device, precision)
    magnetic = _fields(None, nx, ny, nz, nstep, device, precision)
    psi = build_psi(nx, ny, nz, prepared.pml, nstep, None, device, precision)
    groups = (electric, magnetic, psi)
    if per_nstep is None:
        return groups
    return tuple(tuple(t[:per_nstep] if t.numel() else t for t in g) for g in groups)
