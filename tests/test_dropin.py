"""The reference's own loader binds this library in place of its CUDA build.

The reference Python (src/DeepGPR/native/loader.py:138-209) loads ``deepgpr.so``
from its ``lib`` folder, checks that every required ABI symbol is exported
(REQUIRED_SYMBOLS), that ``deepgpr_abi_version()`` is 6, and installs the
ctypes signatures of its declarative table (native/abi.py).  This test copies
the reference ``src/`` to a scratch directory, puts ``libdeepgpr_b200.so``
there as ``deepgpr.so`` and runs that unmodified loader on it.  It needs the
reference checkout (skipped where it is absent) and no GPU: loading and
binding make no CUDA call.
"""

from __future__ import annotations

import shutil
import subprocess
import sys
import textwrap

import pytest

from oracle import driver

ROOT = driver.REFERENCE_ROOT


@pytest.mark.skipif(not (ROOT / "src" / "DeepGPR" / "native" / "loader.py").is_file(),
                    reason="reference checkout not present")
def test_reference_loader_binds_this_library_as_its_cuda_backend(tmp_path):
    from deepgpr_b200 import build

    lib = build.build()
    shutil.copytree(ROOT / "src", tmp_path / "src")
    libdir = tmp_path / "src" / "DeepGPR" / "lib"
    for name in list(libdir.iterdir()):
        if name.suffix in (".so", ".dll", ".dylib"):
            name.unlink()
    shutil.copy(lib, libdir / "deepgpr.so")
    script = textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {str(tmp_path / "src")!r})
        from DeepGPR.native import loader, abi
        lib = loader.get_deepgpr_lib("cuda")
        assert loader.get_deepgpr_library_path("cuda").endswith("deepgpr.so")
        assert lib.deepgpr_abi_version() == loader.NATIVE_ABI_VERSION == 6
        for name in abi.REQUIRED_SYMBOLS:
            assert hasattr(lib, name), name
        bound = {{n: len(getattr(lib, n).argtypes) for n in abi.NATIVE_FUNCTIONS if hasattr(lib, n)
                 and getattr(lib, n).argtypes is not None}}
        assert bound["forward"] == len(abi.FORWARD_SIGNATURE)
        assert bound["backward"] == len(abi.BACKWARD_SIGNATURE)
        assert lib.deepgpr_supports_error_reporting() == 1
        print("bound", len(bound), "functions; forward", bound["forward"], "backward", bound["backward"])
    """)
    res = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-3000:]
    assert "forward 81 backward 86" in res.stdout, res.stdout
