"""Run one forward + adjoint problem through an ABI-6 CPU library (checker only).

The host preprocessing (model extension, CPML coefficients, coordinate
shift, argument marshalling) is the product's own Python
(``deepgpr_b200.model``, ``.pml``, ``.solver``), which is itself pinned to
the reference by the golden fixtures; the solve is done by the CPU library:

* ``kind="oracle"`` -> ``oracle/liboracle_fdtd.so`` (restatement, this repo)
* ``kind="ref"``    -> ``oracle/_ref/deepgpr_cpu.so`` (reference source, built here)

Gradients are returned on the physical model (the CPML fold applied).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any, Dict, Optional, Sequence, Tuple

import torch

from deepgpr_b200 import native
from deepgpr_b200.config import CPML_FACES
from deepgpr_b200.model import prepare_model, shift_locations
from deepgpr_b200.pml import build_pml_coefficients, build_psi
from deepgpr_b200.solver import SolverConfig, SolverTensors, backward_arguments, forward_arguments
from deepgpr_b200.storage import (
    StorageConfig,
    encode_storage_type,
    history_box,
    saved_history_shape,
    saved_time_steps,
)

HERE = Path(__file__).resolve().parent
LIBS = {"oracle": HERE / "liboracle_fdtd.so", "ref": HERE / "_ref" / "deepgpr_cpu.so"}
# Root of the reference checkout (read only by the build recipe and the tests
# that pin the oracle); DEEPGPR_REFERENCE_ROOT overrides the default location.
REFERENCE_ROOT = Path(os.environ.get("DEEPGPR_REFERENCE_ROOT", "/root/reference"))
REF_SOURCE = REFERENCE_ROOT / "src" / "DeepGPR" / "lib" / "deepgpr_cpu.c"

_loaded: Dict[str, ctypes.CDLL] = {}


def build(kind: str = "oracle") -> Path:
    """Compile the checker library (``make -C oracle``); ``ref`` needs the reference tree."""
    target = "all" if kind == "oracle" else "ref"
    if kind == "ref" and not REF_SOURCE.is_file() and not LIBS["ref"].is_file():
        raise FileNotFoundError("reference source tree not present and oracle/_ref not prebuilt")
    if kind == "ref" and not REF_SOURCE.is_file():
        return LIBS["ref"]
    cmd = ["make", "-s", "-C", str(HERE), target]
    if kind == "ref":
        cmd.append(f"REF_SRC_DIR={REF_SOURCE.parent}")
    subprocess.run(cmd, check=True)
    return LIBS[kind]


def available(kind: str) -> bool:
    return LIBS[kind].is_file()


def load(kind: str = "oracle") -> ctypes.CDLL:
    if kind in _loaded:
        return _loaded[kind]
    path = LIBS[kind]
    if not path.is_file():
        build(kind)
    lib = ctypes.CDLL(str(path))
    for name, sig in (("forward", native.FORWARD_SIGNATURE), ("backward", native.BACKWARD_SIGNATURE)):
        fn = getattr(lib, name)
        fn.argtypes = [native._ctype(kind_, "float") for _, kind_ in sig]
        fn.restype = None
    lib.set_fdtd_order.argtypes = [ctypes.c_int]
    lib.set_fdtd_order.restype = None
    lib.deepgpr_last_error.restype = ctypes.c_char_p
    lib.deepgpr_clear_last_error.restype = None
    _loaded[kind] = lib
    return lib


@dataclass
class Problem:
    """All inputs of one solve, on the physical grid (CPU tensors)."""

    eps_r: torch.Tensor
    sigma: torch.Tensor
    source_amplitudes: torch.Tensor          # (nwave, nt[, 1])
    source_location: torch.Tensor            # (nstep, nsrc, 3) physical
    receiver_location: torch.Tensor          # (nstep, nrx, 3) physical
    dx: Any
    dt: float
    pml: Any = 10
    order: int = 2
    mode: int = 2
    source_component: int = 2
    receiver_component: int = 2
    mu_r: Optional[torch.Tensor] = None
    interval: int = 1
    storage_kind: int = 0                    # 0 fp32, 1 fp16, 2 bf16
    rhs_from_e: Optional[bool] = None        # None: as the reference's "auto"
    region: str = "extended"
    initial_states: Optional[Sequence[torch.Tensor]] = None   # 30 tensors on the solver grid
    # cotangents of the outputs
    data_grad: Optional[torch.Tensor] = None  # (nstep, nt, nrx); default 2 * receivers (sum of squares)
    state_duals: Optional[Sequence[torch.Tensor]] = None
    want_eps: bool = True
    want_sigma: bool = True
    want_source: bool = False
    max_velocity: float = 299792458.0
    extra: Dict[str, Any] = field(default_factory=dict)


def prepare(p: Problem, dtype: torch.dtype = torch.float32):
    """Host preprocessing shared by the oracle run and the product call."""
    eps = p.eps_r.detach().clone().to(dtype).requires_grad_(p.want_eps)
    sig = p.sigma.detach().clone().to(dtype).requires_grad_(p.want_sigma)
    wave = p.source_amplitudes.detach().clone().to(dtype).requires_grad_(p.want_source)
    prep = prepare_model("cpu", eps, sig, p.mu_r, wave, p.source_location, p.receiver_location, p.dx, p.dt,
                         p.pml, p.order, dtype=dtype)
    return eps, sig, wave, prep


def run(p: Problem, kind: str = "oracle", backward: bool = True) -> Dict[str, Any]:
    """Forward (+ adjoint) through a CPU library; returns receivers, states, gradients."""
    lib = load(kind)
    eps, sig, wave, prep = prepare(p)
    nx, ny, nz, nt = prep.nx, prep.ny, prep.nz, prep.nt
    pml = prep.pml
    nstep = prep.nstep
    src = shift_locations(p.source_location, pml, "cpu")
    rcv = shift_locations(p.receiver_location, pml, "cpu")
    _, coeffs = build_pml_coefficients(p.dt, p.dx, nx, ny, nz, pml, "cpu", torch.float32, max_velocity=p.max_velocity)
    if p.initial_states is not None:
        states = [t.detach().clone().float().contiguous() for t in p.initial_states]
    else:
        shape = (nstep, nx + 1, ny + 1, nz + 1)
        states = [torch.zeros(shape) for _ in range(6)] + list(build_psi(nx, ny, nz, pml, nstep, None, "cpu"))
    want_model = p.want_eps or p.want_sigma
    lossless = p.storage_kind == 0
    rhs_from_e = (p.interval == 1 and lossless) if p.rhs_from_e is None else p.rhs_from_e
    rhs_from_e = bool(rhs_from_e and want_model)
    storage = StorageConfig({0: torch.float32, 1: torch.float16, 2: torch.bfloat16}[p.storage_kind], "none",
                            p.storage_kind)
    cfg = SolverConfig(
        device=torch.device("cpu"), dtype=torch.float32, spacing=tuple(float(v) for v in (
            p.dx if isinstance(p.dx, (list, tuple)) else (p.dx,) * 3)),
        dt=float(p.dt), nx=nx, ny=ny, nz=nz, nt=nt, nstep=nstep, nsr=prep.nsr, nrx=prep.nrx, pml=pml,
        source_component=p.source_component, receiver_component=p.receiver_component, interval=p.interval,
        storage=storage, save_history=True, offload=False, fdtd_order=p.order, mode=p.mode, debug=False,
        reconstruct_rhs=rhs_from_e, region=p.region,
    )
    stype = encode_storage_type(storage, True, rhs_from_e, p.region == "physical")
    nt_saved = saved_time_steps(nt, p.interval)
    hshape = saved_history_shape(p.mode, nt_saved, nstep, *history_box(nx, ny, nz, pml, p.region)[1])
    e_saved = torch.zeros(hshape, dtype=storage.dtype)
    if rhs_from_e:
        r_saved = torch.zeros(saved_history_shape(p.mode, 1, nstep, *history_box(nx, ny, nz, pml, p.region)[1]),
                              dtype=storage.dtype)
    else:
        r_saved = torch.zeros(hshape if want_model else (0,), dtype=storage.dtype)
    tensors = SolverTensors(
        eps_r_pad=prep.eps_r_pad.detach().contiguous(), sigma_pad=prep.sigma_pad.detach().contiguous(),
        mu_r_pad=prep.mu_r_pad.detach().contiguous(), source_location=src, receiver_location=rcv,
        pml_coefficients=tuple(c.contiguous() for c in coeffs),
    )
    rx = torch.zeros((nstep, nt, prep.nrx))
    waveform = prep.source_amplitudes.detach().contiguous()
    args = forward_arguments(cfg, tensors, states, e_saved, r_saved, rx, waveform, stype, want_model)
    lib.deepgpr_clear_last_error()
    lib.set_fdtd_order(p.order)
    fargs = native.marshal(native.FORWARD_SIGNATURE, args)
    t0 = time.perf_counter()
    lib.forward(*fargs)
    t_forward = time.perf_counter() - t0
    err = lib.deepgpr_last_error()
    if err:
        raise RuntimeError(f"{kind} forward: {err.decode()}")
    out: Dict[str, Any] = {"receivers": rx.clone(), "states": [s.clone() for s in states],
                           "E_saved": e_saved.clone(), "R_saved": r_saved.clone(), "storage_type": stype,
                           "t_forward": t_forward}
    if not backward:
        return out
    data_grad = (2.0 * rx) if p.data_grad is None else p.data_grad.float().contiguous().clone()
    lambdas = ([torch.zeros_like(s) for s in states] if p.state_duals is None
               else [d.detach().float().clone().contiguous() for d in p.state_duals])
    ext = (nx, ny, nz)
    g_eps = torch.zeros(ext) if p.want_eps else torch.empty(0)
    g_sig = torch.zeros(ext) if p.want_sigma else torch.empty(0)
    g_src = torch.zeros(tuple(prep.source_amplitudes.shape)) if p.want_source else torch.empty(0)
    args = backward_arguments(cfg, tensors, lambdas, e_saved, r_saved, data_grad, g_src, g_eps, g_sig,
                              (p.want_source, p.want_eps, p.want_sigma), stype)
    lib.deepgpr_clear_last_error()
    lib.set_fdtd_order(p.order)
    bargs = native.marshal(native.BACKWARD_SIGNATURE, args)
    t0 = time.perf_counter()
    lib.backward(*bargs)
    out["t_backward"] = time.perf_counter() - t0
    err = lib.deepgpr_last_error()
    if err:
        raise RuntimeError(f"{kind} backward: {err.decode()}")
    out["grad_eps_ext"] = g_eps.clone()
    out["grad_sigma_ext"] = g_sig.clone()
    out["lambdas"] = lambdas
    # fold the CPML sensitivities onto the physical model (autograd of the extension)
    roots, outs, cots = [], [], []
    if p.want_eps:
        roots.append(eps); outs.append(prep.eps_r); cots.append(g_eps)
    if p.want_sigma:
        roots.append(sig); outs.append(prep.sigma); cots.append(g_sig)
    if p.want_source:
        roots.append(wave); outs.append(prep.source_amplitudes); cots.append(g_src)
    if roots:
        grads = torch.autograd.grad(outs, roots, cots, allow_unused=True)
        names = [n for n, w in (("grad_eps", p.want_eps), ("grad_sigma", p.want_sigma), ("grad_source", p.want_source)) if w]
        for n, g in zip(names, grads):
            out[n] = g
    return out
