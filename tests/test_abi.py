"""The C-ABI library: symbols of include/deepgpr_b200.h, parameter tables, host helpers.

No CUDA call is made (the library loads without a GPU); only the host-side
entry points (capability probes, sizes, options) are called.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from deepgpr_b200 import native
from deepgpr_b200.storage import fp8_history_bytes

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "deepgpr_b200.h"


def _declared():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)) - {"extern", "defined"}


def _params(fn):
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    m = re.search(rf"void {fn}\((.*?)\);", text, flags=re.S)
    names = []
    for part in m.group(1).split(","):
        names.append(re.findall(r"[A-Za-z_][A-Za-z0-9_]*", part)[-1])
    return names


@pytest.fixture(scope="module")
def lib():
    return native.load_library()


def test_library_exports_every_declared_symbol(lib):
    missing = [name for name in sorted(_declared()) if not hasattr(lib, name)]
    assert not missing, missing


def test_python_tables_match_header():
    assert [n for n, _ in native.FORWARD_SIGNATURE] == _params("forward")
    assert [n for n, _ in native.BACKWARD_SIGNATURE] == _params("backward")
    assert len(native.FORWARD_SIGNATURE) == 81
    assert len(native.BACKWARD_SIGNATURE) == 86
    assert _params("dgb_forward_noalloc") == _params("forward")


def test_header_matches_reference_parameter_order():
    from oracle import driver

    ref = driver.REFERENCE_ROOT / "src" / "DeepGPR" / "native" / "abi.py"
    if not ref.is_file():
        pytest.skip("reference tree not present")
    import types

    # evaluate the reference's declarative table without importing its package
    src = ref.read_text().replace("from ..config.constants import CPML_FACE_NAMES",
                                  "CPML_FACE_NAMES = ('x0', 'xm', 'y0', 'ym', 'z0', 'zm')")
    mod = types.ModuleType("ref_abi")
    exec(compile(src, str(ref), "exec"), mod.__dict__)
    assert [n for n, _ in mod.FORWARD_SIGNATURE] == [n for n, _ in native.FORWARD_SIGNATURE]
    assert [n for n, _ in mod.BACKWARD_SIGNATURE] == [n for n, _ in native.BACKWARD_SIGNATURE]


def test_capabilities(lib):
    assert lib.deepgpr_abi_version() == 6
    assert lib.deepgpr_supports_error_reporting() == 1
    assert lib.deepgpr_deterministic_adjoint() == 1
    assert lib.deepgpr_supports_rhs_reconstruction() == 1
    assert lib.deepgpr_supports_physical_history() == 1
    assert lib.deepgpr_supports_tm2d_fast_path() == 1
    assert lib.deepgpr_supports_int8_wavefield() == 0
    assert lib.dgb_supports_fp8_history() == 1
    assert lib.deepgpr_last_error() == b""


@pytest.mark.parametrize("tm2d,shape", [(False, (221, 221, 221)), (True, (421, 821, 2)), (False, (17, 15, 13))])
def test_history_bytes_agree_with_python(lib, tm2d, shape):
    ncomp, nt_saved, nshot, box = 3, 7, 2, (shape[0] - 1) * (shape[1] - 1) * (shape[2] - 1)
    want = fp8_history_bytes(ncomp, nt_saved, nshot, box, shape, tm2d)
    assert lib.dgb_history_bytes(4, ncomp, nt_saved, nshot, box, *shape, int(tm2d)) == want
    assert lib.dgb_history_bytes(0, ncomp, nt_saved, nshot, box, *shape, 0) == 4 * ncomp * nt_saved * nshot * box
    assert lib.dgb_history_bytes(2, ncomp, nt_saved, nshot, box, *shape, 0) == 2 * ncomp * nt_saved * nshot * box


def test_options_validation(lib):
    assert lib.dgb_set_options(1, 16, 1, 0) == 0
    assert lib.dgb_set_options(1, 0, 1, 0) == -1
    assert lib.dgb_set_options(1, 16, 1, 0) == 0


def test_marshal_rejects_missing_and_unknown_names():
    with pytest.raises(KeyError):
        native.marshal(native.FORWARD_SIGNATURE, {"dt": 1.0})


def test_build_recipe_compiles_the_device_code_as_one_unit():
    """Split compilation optimises groups of device functions separately and the
    grouping follows the whole translation unit: an edit of host code alone
    changed kernels' registers and speed.  The recipe must not ask for it, and
    must keep strict IEEE single precision (the reference's rounding)."""
    from deepgpr_b200 import build

    assert not any(flag.startswith("-split-compile") for flag in build.NVCC_FLAGS)
    assert "-fmad=false" in build.NVCC_FLAGS
    assert "arch=compute_100a,code=sm_100a" in build.NVCC_FLAGS
