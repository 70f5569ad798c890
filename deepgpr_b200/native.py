"""ctypes binding of libdeepgpr_b200.so (the C ABI declared in include/deepgpr_b200.h).

The ``forward``/``backward`` parameter tables reproduce ABI 6 of the reference
(src/DeepGPR/lib/deepgpr.h:89-152, src/DeepGPR/native/abi.py:90-158): same
names, order and meaning.  Calls are made with the caller's current CUDA
stream (``dgb_set_stream``) and a per-call FDTD order (``dgb_set_options``),
so concurrent callers with different orders need no global lock.

There is no fallback: if the library is missing or fails to load, every
solver call raises :class:`NativeLibraryNotFoundError`.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path
from typing import Any, Dict, List, Mapping, Optional, Sequence, Tuple

from .config import CPML_FACES, NATIVE_ABI_VERSION
from .errors import NativeLibraryError, NativeLibraryNotFoundError

LIB_DIR = Path(__file__).resolve().parent / "lib"
LIB_NAME = "libdeepgpr_b200.so"

Signature = Tuple[Tuple[str, str], ...]


def _psi_names(prefix: str = "") -> Tuple[str, ...]:
    return tuple(f"{prefix}{face}_{field}_phi{i}" for face in CPML_FACES for field in ("e", "h") for i in (1, 2))


PHI_NAMES = _psi_names()
LAMBDA_PHI_NAMES = _psi_names("lambda_")
COEFF_NAMES = ("ce_hist", "ce_curl", "ce_rhs", "ch_hist", "ch_curl", "ch_rhs")


def _common_tail() -> Signature:
    thick = tuple((f"pml_{f}", "int") for f in CPML_FACES)
    coeff = tuple((f"{f}_e_coeff", "real*") for f in CPML_FACES) + tuple((f"{f}_h_coeff", "real*") for f in CPML_FACES)
    time = (("dt", "real"), ("nt", "int"), ("nshot", "int"), ("nreceiver", "int"), ("dx", "real"), ("dy", "real"), ("dz", "real"))
    return thick + coeff + time


_FIELDS = (("nx_fields", "int"), ("ny_fields", "int"), ("nz_fields", "int"))
_MATERIALS = (("eps_r_pad", "real*"), ("sigma_pad", "real*"), ("mu_r_pad", "real*"))

FORWARD_SIGNATURE: Signature = (
    _MATERIALS
    + (("E_saved", "void*"), ("R_saved", "void*"))
    + tuple((n, "real*") for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"))
    + tuple((n, "real*") for n in COEFF_NAMES)
    + tuple((n, "real*") for n in PHI_NAMES)
    + _common_tail()
    + (("receiver_location", "int*"), ("receiver_data", "real*"), ("receiver_component", "int"))
    + _FIELDS
    + (
        ("nsource", "int"), ("source_location", "int*"), ("source_waveform", "real*"), ("source_component", "int"),
        ("sampling_interval", "int"), ("fwi_mode", "int"), ("storage_type", "int"), ("save_model_history", "int"),
        ("use_async_offload", "int"),
    )
)

BACKWARD_SIGNATURE: Signature = (
    _MATERIALS
    + (("E_saved", "void*"), ("R_saved", "void*"))
    + tuple((n, "real*") for n in ("lambda_ex", "lambda_ey", "lambda_ez", "lambda_hx", "lambda_hy", "lambda_hz"))
    + tuple((n, "real*") for n in COEFF_NAMES)
    + tuple((n, "real*") for n in LAMBDA_PHI_NAMES)
    + _common_tail()
    + _FIELDS
    + (
        ("ndata_source", "int"), ("receiver_location", "int*"), ("data_grad", "real*"), ("receiver_component", "int"),
        ("nsource", "int"), ("source_location", "int*"), ("source_component", "int"), ("grad_source", "real*"),
        ("source_requires_grad", "int"), ("grad_eps_r", "real*"), ("grad_sigma", "real*"),
        ("eps_r_requires_grad", "int"), ("sigma_requires_grad", "int"), ("sampling_interval", "int"),
        ("fwi_mode", "int"), ("storage_type", "int"), ("use_async_offload", "int"),
    )
)

# Exported symbols: name -> (argument kinds, return kind).
SCALAR_SYMBOLS: Dict[str, Tuple[Tuple[str, ...], Optional[str]]] = {
    "deepgpr_abi_version": ((), "int"),
    "deepgpr_supports_error_reporting": ((), "int"),
    "deepgpr_last_error": ((), "char*"),
    "deepgpr_clear_last_error": ((), None),
    "deepgpr_clear_cuda_resource_cache": ((), None),
    "deepgpr_deterministic_adjoint": ((), "int"),
    "deepgpr_supports_external_pml": ((), "int"),
    "deepgpr_supports_pml_material_gradients": ((), "int"),
    "deepgpr_supports_int8_wavefield": ((), "int"),
    "deepgpr_supports_conversion_backends": ((), "int"),
    "deepgpr_supports_int8_reduction_backends": ((), "int"),
    "deepgpr_supports_rhs_reconstruction": ((), "int"),
    "deepgpr_supports_physical_history": ((), "int"),
    "deepgpr_supports_tm2d_fast_path": ((), "int"),
    "set_fdtd_order": (("int",), None),
    "dgb_version": ((), "int"),
    "dgb_supports_fp8_history": ((), "int"),
    "dgb_set_stream": (("void*",), "int"),
    "dgb_clear_stream": ((), None),
    "dgb_set_options": (("int", "int", "int", "int"), "int"),
    "dgb_set_tuning": (("int", "int", "int", "int"), "int"),
    "dgb_history_bytes": (("int", "int", "int", "int", "long long", "int", "int", "int", "int"), "long long"),
    "dgb_check_fixed_division": (("float", "void*", "void*"), "int"),
    "dgb_set_scratch_retention": (("long long",), "int"),
    "dgb_default_pool_usage": (("void*", "void*", "int"), "int"),
    "dgb_profile": (("int",), None),
    "dgb_launch_count": ((), "long long"),
    "dgb_profile_read": (("void*", "void*", "int"), "int"),
}

KERNEL_KINDS = ("fwd_h", "fwd_e", "adj_e", "adj_h", "image")


def profile(enable: bool) -> None:
    """Enable per-kernel CUDA-event timing for this thread (no graph replay while on)."""
    load_library().dgb_profile(int(enable))


def launch_count() -> int:
    """Kernels launched by this thread through the library (time-step kernels)."""
    return int(load_library().dgb_launch_count())


def profile_read() -> Dict[str, Tuple[float, int]]:
    """Per-kernel-kind (total ms, launches) since ``profile(True)``."""
    lib = load_library()
    n = len(KERNEL_KINDS)
    ms = (ctypes.c_double * n)()
    cnt = (ctypes.c_longlong * n)()
    lib.dgb_profile_read(ctypes.cast(ms, ctypes.c_void_p), ctypes.cast(cnt, ctypes.c_void_p), n)
    return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(KERNEL_KINDS)}

def set_scratch_retention(nbytes: int) -> None:
    """Keep up to ``nbytes`` of the solver's freed scratch cached on the current
    device (-1: no limit; 0: none, the CUDA default, and trim now).  Without a
    call the library keeps min(4 GiB, 1/32 of the device memory); see
    ``dgb_set_scratch_retention``."""
    lib = load_library()
    if lib.dgb_set_scratch_retention(int(nbytes)) != 0:
        raise NativeLibraryError(last_error(lib) or "dgb_set_scratch_retention failed")


def default_pool_usage(reset_high: bool = False) -> Tuple[int, int]:
    """(bytes in use, high-water mark) of the current device's default
    stream-ordered memory pool; ``reset_high`` first resets the mark."""
    lib = load_library()
    used = ctypes.c_longlong(0)
    high = ctypes.c_longlong(0)
    if lib.dgb_default_pool_usage(ctypes.addressof(used), ctypes.addressof(high), int(bool(reset_high))) != 0:
        raise NativeLibraryError(last_error(lib) or "dgb_default_pool_usage failed")
    return int(used.value), int(high.value)


def check_fixed_division(divisor: float) -> Tuple[int, int]:
    """(mismatches, lowest mismatching bit pattern) of the solver's division by
    ``divisor`` against the division operator over all 2^32 float dividends."""
    lib = load_library()
    bad = ctypes.c_ulonglong(0)
    first = ctypes.c_uint(0)
    if lib.dgb_check_fixed_division(float(divisor), ctypes.addressof(bad), ctypes.addressof(first)) != 0:
        raise NativeLibraryError(last_error(lib) or "dgb_check_fixed_division failed")
    return int(bad.value), int(first.value)


SOLVER_SYMBOLS = {
    "forward": (FORWARD_SIGNATURE, "float"),
    "backward": (BACKWARD_SIGNATURE, "float"),
    "dgb_forward_f64": (FORWARD_SIGNATURE, "double"),
    "dgb_backward_f64": (BACKWARD_SIGNATURE, "double"),
    "dgb_forward_noalloc": (FORWARD_SIGNATURE, "float"),
}

_CT = {
    "int": ctypes.c_int,
    "float": ctypes.c_float,
    "long long": ctypes.c_longlong,
    "void*": ctypes.c_void_p,
    "char*": ctypes.c_char_p,
    "int*": ctypes.c_void_p,
}


def _ctype(kind: str, real: str) -> Any:
    if kind == "real":
        return ctypes.c_float if real == "float" else ctypes.c_double
    if kind == "real*":
        return ctypes.c_void_p
    return _CT[kind]


_LOCK = threading.Lock()
_LIB: Optional[ctypes.CDLL] = None


def library_path() -> Path:
    override = os.environ.get("DEEPGPR_B200_LIB")
    return Path(override) if override else LIB_DIR / LIB_NAME


def load_library() -> ctypes.CDLL:
    """Load and configure the CUDA library once per process; raise if absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        path = library_path()
        if not path.is_file():
            raise NativeLibraryNotFoundError(
                f"{path} is not built. Run `python -c 'import __graft_entry__ as g; g.build()'` "
                "or `python -m deepgpr_b200.build` first; there is no CPU fallback."
            )
        try:
            lib = ctypes.CDLL(str(path))
        except OSError as exc:
            raise NativeLibraryNotFoundError(f"cannot load {path}: {exc}") from exc
        configure(lib)
        _LIB = lib
        return lib


def configure(lib: ctypes.CDLL) -> None:
    """Install argtypes/restype for every exported symbol and check the ABI."""
    missing = [n for n in list(SCALAR_SYMBOLS) + list(SOLVER_SYMBOLS) if not hasattr(lib, n)]
    if missing:
        raise NativeLibraryError(f"library does not export {missing}")
    for name, (args, ret) in SCALAR_SYMBOLS.items():
        fn = getattr(lib, name)
        fn.argtypes = [_CT[a] for a in args]
        fn.restype = None if ret is None else _CT[ret]
    for name, (sig, real) in SOLVER_SYMBOLS.items():
        fn = getattr(lib, name)
        fn.argtypes = [_ctype(kind, real) for _, kind in sig]
        fn.restype = None
    version = int(lib.deepgpr_abi_version())
    if version != NATIVE_ABI_VERSION:
        raise NativeLibraryError(f"library reports ABI {version}; expected {NATIVE_ABI_VERSION}")


def _address(value: Any) -> int:
    ptr = getattr(value, "data_ptr", None)
    if callable(ptr):
        return int(ptr())
    if isinstance(value, int):
        return value
    raise TypeError(f"cannot take the address of {type(value).__name__}")


def marshal(signature: Signature, args: Mapping[str, Any]) -> List[Any]:
    """Positional ctypes arguments for ``signature`` from a name -> value mapping."""
    names = [n for n, _ in signature]
    missing = [n for n in names if n not in args]
    extra = sorted(set(args) - set(names))
    if missing or extra:
        raise KeyError(f"native argument mismatch; missing={missing}, unexpected={extra}")
    out: List[Any] = []
    for name, kind in signature:
        v = args[name]
        if kind in ("real*", "int*", "void*"):
            out.append(ctypes.c_void_p(_address(v)))
        elif kind == "int":
            out.append(int(v))
        else:
            out.append(float(v))
    return out


def last_error(lib: ctypes.CDLL) -> str:
    msg = lib.deepgpr_last_error()
    return msg.decode("utf-8", "replace") if msg else ""


# Launch-shape choices of dgb_set_tuning: the built-in heuristics
DEFAULT_TUNING = (0, 0, 0, -1)


def invoke(name: str, args: Mapping[str, Any], *, fdtd_order: int, stream: Any = None,
           acc64: bool = True, chunk: int = 32, use_graph: bool = True,
           tuning: Sequence[int] = DEFAULT_TUNING) -> None:
    """Call ``forward``/``backward`` (or their FP64 twins) on ``stream``.

    ``tuning`` is ``(tm_chunks, tm_frame_rows, k3_xchunks, tma)`` of
    ``dgb_set_tuning`` (see ``deepgpr_b200.autotune``).  Raises
    :class:`NativeLibraryError` with the library's message on failure.
    """
    lib = load_library()
    sig, _ = SOLVER_SYMBOLS[name]
    positional = marshal(sig, args)
    if lib.dgb_set_options(int(acc64), int(chunk), int(use_graph), int(fdtd_order)) != 0:
        raise NativeLibraryError("invalid launch options")
    if lib.dgb_set_tuning(*(int(v) for v in tuning)) != 0:
        raise NativeLibraryError(f"invalid tuning {tuple(tuning)}")
    handle = 0
    if stream is not None:
        handle = int(getattr(stream, "cuda_stream", stream))
    lib.dgb_set_stream(ctypes.c_void_p(handle))
    lib.deepgpr_clear_last_error()
    try:
        getattr(lib, name)(*positional)
    finally:
        lib.dgb_clear_stream()
    msg = last_error(lib)
    if msg:
        lib.deepgpr_clear_last_error()
        raise NativeLibraryError(f"native {name} failed: {msg}")


def capability(name: str) -> bool:
    lib = load_library()
    fn = getattr(lib, name, None)
    return fn is not None and int(fn()) == 1


def exported_symbols() -> Sequence[str]:
    return tuple(SCALAR_SYMBOLS) + tuple(SOLVER_SYMBOLS)
