"""Host logic and the oracle against fixtures recorded from the reference package.

Fixtures (tests/golden/*.npz) were produced by tests/golden/make_golden.py,
which runs the reference's own Python + C code.  CPU only.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from deepgpr_b200.grid import max_stable_time_step
from deepgpr_b200.model import ExtendIntoPML
from deepgpr_b200.pml import build_pml_coefficients, face_descriptors, psi_shapes
from oracle import driver

GOLD = Path(__file__).resolve().parent / "golden"


def _load(name):
    return dict(np.load(GOLD / name))


def test_cpml_coefficients_bitwise():
    d = _load("pml.npz")
    for case in range(3):
        args = d[f"case{case}/args"]
        dx = tuple(float(v) for v in args[0:3])
        dt = float(args[3])
        shape = tuple(int(v) for v in args[4:7])
        pml = [int(v) for v in args[7:13]]
        v_ref = float(args[13])
        desc, coeffs = build_pml_coefficients(dt, dx, *shape, pml, "cpu", torch.float32, max_velocity=v_ref)
        for f in range(6):
            want_d = d[f"case{case}/desc{f}"]
            assert np.array_equal(desc[f].numpy() if desc[f].numel() else np.zeros(0, np.int32), want_d)
            assert np.array_equal(coeffs[2 * f].numpy() if coeffs[2 * f].numel() else np.zeros(0, np.float32),
                                  d[f"case{case}/e{f}"]), (case, f)
            assert np.array_equal(coeffs[2 * f + 1].numpy() if coeffs[2 * f + 1].numel() else np.zeros(0, np.float32),
                                  d[f"case{case}/h{f}"]), (case, f)
            shapes = psi_shapes(f, pml[f], *shape, 3)
            got = np.array([s if s is not None else (0, 0, 0, 0) for s in shapes])
            assert np.array_equal(got, d[f"case{case}/phi{f}"]), (case, f)


def test_cfl_limits():
    d = _load("misc.npz")
    for row in d["cfl"]:
        dx = tuple(float(v) for v in row[0:3])
        dims = tuple(int(v) for v in row[3:6])
        order = int(row[6])
        assert max_stable_time_step(dx, *dims, fdtd_order=order) == pytest.approx(float(row[7]), rel=0, abs=0)


def test_extension_and_fold_bitwise():
    d = _load("misc.npz")
    model = torch.from_numpy(d["extend/model"]).requires_grad_(True)
    pml = [int(v) for v in d["extend/pml"]]
    ext = ExtendIntoPML.apply(model, pml)
    assert np.array_equal(ext.detach().numpy(), d["extend/out"])
    (ext * torch.from_numpy(d["extend/up"])).sum().backward()
    assert np.array_equal(model.grad.numpy(), d["extend/grad"])


@pytest.mark.parametrize("name", ["2d_o2", "2d_o4", "3d_o4"])
def test_oracle_reproduces_reference_solves(name, oracle_lib):
    d = _load("solves.npz")
    order, mode = (int(v) for v in d[f"{name}/meta"])
    is3d = name.startswith("3d")
    p = driver.Problem(
        eps_r=torch.from_numpy(d[f"{name}/in_eps"]), sigma=torch.from_numpy(d[f"{name}/in_sig"]),
        source_amplitudes=torch.from_numpy(d[f"{name}/in_wave"]), source_location=torch.from_numpy(d[f"{name}/in_src"]),
        receiver_location=torch.from_numpy(d[f"{name}/in_rcv"]),
        dx=(0.02, 0.017, 0.013) if is3d else 0.02, dt=1e-11 if is3d else 3e-11,
        pml=[3, 2, 4, 1, 2, 3] if is3d else 10, order=order, mode=mode, want_source=True,
    )
    out = driver.run(p, "oracle")
    assert np.array_equal(out["receivers"].numpy(), d[f"{name}/receivers"])
    for key in ("grad_eps", "grad_sigma", "grad_source"):
        got = out[key].numpy()
        want = d[f"{name}/{key}"]
        assert got.shape == want.shape
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6 * np.abs(want).max())
