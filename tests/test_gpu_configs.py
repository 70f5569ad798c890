"""CUDA path against the oracle on the benchmark configurations.

Each case runs the seeded inputs of one benchmark configuration through
``deepgpr_b200.compute`` (forward + exact adjoint) on the GPU and through the
CPU oracle, and compares receivers, final states and gradients at the
tolerances of the parity contract (receivers / states relative L2 1e-5,
gradients 1e-4).  Where a configuration's full run would take the CPU oracle
too long, nt (and for the 3D precision-study grid the shot count) is cut;
the grid, order, gradient mode and history format are the configuration's:

* config 1 in full (100 x 100, nt 2000, order 2), also against the
  reference's own C backend compiled from its source (``oracle/_ref``);
* config 2's grid and acquisition (400 x 800, 32 shots, 200 receivers,
  order 4, FP32 E-only history) at nt 100;
* config 3's history mode (3D order 8, gradient mode 3, BF16 stored R^n,
  8 shots on a 2 x 4 surface grid) on a 36^3 grid at nt 60;
* config 5's grid (320 x 320 x 160, order 4, mode 3, FP32 E-only history)
  with 2 of its shots at nt 8;
* the three solves recorded from the reference package
  (``tests/golden/solves.npz``).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from helpers import rel_l2, ricker, run_product
from oracle import driver

pytestmark = pytest.mark.gpu

RX_TOL = 1e-5
GRAD_TOL = 1e-4
GOLD = Path(__file__).resolve().parent / "golden"


def _checker() -> str:
    """The reference's C backend where it was built (pinned bit for bit to the oracle on CPU; several times
    faster on the adjoint of large grids), else the oracle."""
    return "ref" if driver.available("ref") else "oracle"


def _compare(got, ref, grads):
    errs = {"receivers": rel_l2(got["receivers"], ref["receivers"])}
    for i, (x, y) in enumerate(zip(got["states"], ref["states"])):
        if y.numel() and y.abs().max() > 0:
            errs[f"state{i}"] = rel_l2(x, y)
    for g in grads:
        errs[g] = rel_l2(got[g], ref[g])
    for k, v in errs.items():
        assert v <= (GRAD_TOL if k.startswith("grad") else RX_TOL), (k, errs)
    return errs


def config1() -> driver.Problem:
    eps = torch.full((100, 100), 2.0)
    eps[50:] = 5.0
    nt, dt = 2000, 3e-11
    return driver.Problem(
        eps_r=eps, sigma=torch.zeros((100, 100)), source_amplitudes=ricker(nt, dt, 200e6)[None],
        source_location=torch.tensor([[[10, 10, 0]]], dtype=torch.int32),
        receiver_location=torch.tensor([[[10, 90, 0]]], dtype=torch.int32), dx=0.02, dt=dt, pml=10, order=2,
        mode=2, want_sigma=False)


def test_config1_full_against_oracle_and_reference_backend(cuda_device, oracle_lib):
    p = config1()
    got = run_product(p, cuda_device)
    _compare(got, driver.run(p, "oracle"), ("grad_eps",))
    if not driver.available("ref"):
        pytest.skip("reference C backend (oracle/_ref) not built")
    _compare(got, driver.run(p, "ref"), ("grad_eps",))


def test_config2_grid_and_acquisition(cuda_device, oracle_lib):
    from deepgpr_b200.synthetic import fwi_2d

    acq = fwi_2d(seed=1002, nt=100)
    p = driver.Problem(eps_r=acq.eps_r, sigma=acq.sigma, source_amplitudes=acq.wavelet, source_location=acq.sources,
                       receiver_location=acq.receivers, dx=acq.dx, dt=acq.dt, pml=10, order=4, mode=2,
                       want_source=True)
    _compare(run_product(p, cuda_device), driver.run(p, _checker()), ("grad_eps", "grad_sigma", "grad_source"))


def test_config3_mode_bf16_stored_rhs_order8(cuda_device, oracle_lib):
    from deepgpr_b200.synthetic import fwi_3d

    acq = fwi_3d(seed=1003, shape=(36, 36, 36), dx=0.02, sources_grid=(2, 4), receivers_grid=(6, 6), nt=60,
                 order=8, air_rows=4)
    assert acq.sources.shape[0] == 8
    p = driver.Problem(eps_r=acq.eps_r, sigma=acq.sigma, source_amplitudes=acq.wavelet, source_location=acq.sources,
                       receiver_location=acq.receivers, dx=acq.dx, dt=acq.dt, pml=10, order=8, mode=3,
                       storage_kind=2, rhs_from_e=False, want_source=True)
    _compare(run_product(p, cuda_device), driver.run(p, "oracle"), ("grad_eps", "grad_sigma", "grad_source"))


def test_config5_grid_two_shots(cuda_device, oracle_lib):
    from deepgpr_b200.synthetic import fwi_3d

    acq = fwi_3d(seed=1005, shape=(320, 320, 160), dx=0.015, sources_grid=(1, 2), receivers_grid=(32, 32), nt=8,
                 order=4)
    p = driver.Problem(eps_r=acq.eps_r, sigma=acq.sigma, source_amplitudes=acq.wavelet, source_location=acq.sources,
                       receiver_location=acq.receivers, dx=acq.dx, dt=acq.dt, pml=10, order=4, mode=3)
    _compare(run_product(p, cuda_device), driver.run(p, _checker()), ("grad_eps", "grad_sigma"))


@pytest.mark.parametrize("name", ["2d_o2", "2d_o4", "3d_o4"])
def test_reference_package_solves(name, cuda_device):
    """Receivers and gradients recorded from the reference package, through the CUDA path."""
    d = dict(np.load(GOLD / "solves.npz"))
    order, mode = (int(v) for v in d[f"{name}/meta"])
    is3d = name.startswith("3d")
    p = driver.Problem(
        eps_r=torch.from_numpy(d[f"{name}/in_eps"]), sigma=torch.from_numpy(d[f"{name}/in_sig"]),
        source_amplitudes=torch.from_numpy(d[f"{name}/in_wave"]),
        source_location=torch.from_numpy(d[f"{name}/in_src"]),
        receiver_location=torch.from_numpy(d[f"{name}/in_rcv"]),
        dx=(0.02, 0.017, 0.013) if is3d else 0.02, dt=1e-11 if is3d else 3e-11,
        pml=[3, 2, 4, 1, 2, 3] if is3d else 10, order=order, mode=mode, want_source=True,
    )
    got = run_product(p, cuda_device, gradient_accumulation="float32")
    assert np.array_equal(got["receivers"].numpy(), d[f"{name}/receivers"])
    for key in ("grad_eps", "grad_sigma", "grad_source"):
        want = torch.from_numpy(d[f"{name}/{key}"])
        assert rel_l2(got[key], want) <= 1e-6, key
