"""The launch-shape autotuner: a tuned solve equals the default one, and the choice is kept.

The autotuner's knobs (2D interior row chunks and frame rows, 3D x chunks,
the 3D forward kernel family -- wide, z-streamed or TMA-staged --, time steps
per graph) split the same work
differently; every cell still evaluates the same expressions in the same
order, so receivers, states and gradients are bit for bit those of the
default launch shapes.
"""

from __future__ import annotations

import pytest
import torch

from helpers import problem_2d, problem_3d, run_product

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [2, 3])
def test_autotuned_solve_equals_default(dims, cuda_device, tmp_path, monkeypatch):
    from deepgpr_b200 import autotune

    monkeypatch.setenv("DEEPGPR_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(autotune, "_TUNER", None)
    p = (problem_2d(nt=120, order=4, shape=(60, 300), want_source=True) if dims == 2
         else problem_3d(nt=70, order=4, shape=(40, 36, 70), pml=4, want_source=True))
    ref = run_product(p, cuda_device)
    got = run_product(p, cuda_device, autotune=True)
    assert torch.equal(got["receivers"], ref["receivers"])
    for a, b in zip(got["states"], ref["states"]):
        assert torch.equal(a, b)
    for key in ("grad_eps", "grad_sigma", "grad_source"):
        assert torch.equal(got[key], ref[key]), key
    tuner = autotune.default_tuner()
    assert len(tuner.table) == 1 and (tmp_path / "tune.json").is_file()
    # a second solve of the same signature reuses the kept choice (no new probes)
    calls = []
    monkeypatch.setattr(autotune, "probe_ms", lambda *a, **k: calls.append(1) or 1.0)
    run_product(p, cuda_device, backward=False, autotune=True)
    assert not calls


def test_every_3d_launch_choice_gives_the_same_receivers(cuda_device):
    """The knobs one at a time on a 3D solve with CPML on every face."""
    from deepgpr_b200 import native

    p = problem_3d(nt=40, order=4, shape=(40, 36, 70), pml=4)
    ref = run_product(p, cuda_device, backward=False)["receivers"]
    real = native.invoke
    for tuning, chunk in (((0, 0, 1, 0), 16), ((0, 0, 5, 0), 8), ((0, 0, 0, 1), 16), ((0, 0, 3, 1), 32),
                          ((0, 0, 0, 2), 16), ((0, 0, 3, 2), 8), ((0, 0, 1, 2), 32)):
        def spy(name, args, **opts):
            opts = dict(opts, tuning=tuning, chunk=chunk)
            return real(name, args, **opts)

        native.invoke = spy
        try:
            got = run_product(p, cuda_device, backward=False)["receivers"]
        finally:
            native.invoke = real
        assert torch.equal(got, ref), (tuning, chunk)


@pytest.mark.parametrize("rhs_from_e", [True, False])
def test_wide_and_streamed_3d_families_agree(rhs_from_e, cuda_device):
    """The wide and z-streamed 3D kernel families, each forced with the tuning
    knob for forward and adjoint, give the same receivers, states and
    gradients bit for bit: E-only history (the E step in the pass form) and
    stored R^n (the E step's CPML in the wide kernel)."""
    from deepgpr_b200 import native

    p = problem_3d(nt=40, order=4, shape=(40, 36, 70), pml=4, rhs_from_e=rhs_from_e, want_source=True)
    real = native.invoke
    outs = []
    for fam in (0, 2):
        def spy(name, args, **opts):
            return real(name, args, **dict(opts, tuning=(0, 0, 0, fam)))

        native.invoke = spy
        try:
            outs.append(run_product(p, cuda_device))
        finally:
            native.invoke = real
    ref, got = outs
    assert torch.equal(got["receivers"], ref["receivers"])
    for a, b in zip(got["states"], ref["states"]):
        assert torch.equal(a, b)
    for key in ("grad_eps", "grad_sigma", "grad_source"):
        assert torch.equal(got[key], ref[key]), key
