"""Segment checkpointing with recompute against the single-call solve.

Modelled on the reference's checkpoint test (tests/test_external_pml.py:
145-191: checkpointed segments equal the full run): receivers, final states
and adjoint states are bit for bit those of the single call; the material and
source gradients agree to 2e-5 (only where each segment's FP64 sum is
rounded into the FP32 output differs).
"""

from __future__ import annotations

import pytest
import torch

from helpers import problem_2d, problem_3d, rel_l2, run_product

pytestmark = pytest.mark.gpu

GRAD_TOL = 2e-5


def _random_states(p, seed=3):
    from deepgpr_b200.pml import build_psi
    from oracle import driver

    prep = driver.prepare(p)[3]
    nx, ny, nz, nstep = prep.nx, prep.ny, prep.nz, prep.nstep
    shape = (nstep, nx + 1, ny + 1, nz + 1)
    zeros = [torch.zeros(shape) for _ in range(6)] + list(build_psi(nx, ny, nz, prep.pml, nstep, None, "cpu"))
    g = torch.Generator().manual_seed(seed)
    return [torch.randn(t.shape, generator=g) * 1e-3 for t in zeros], [torch.randn(t.shape, generator=g)
                                                                        for t in zeros]


def _check(full, ckpt):
    assert torch.equal(full["receivers"], ckpt["receivers"])
    for a, b in zip(full["states"], ckpt["states"]):
        assert torch.equal(a, b)
    for key in ("grad_eps", "grad_sigma", "grad_source"):
        if key in full:
            assert rel_l2(ckpt[key], full[key]) <= GRAD_TOL, (key, rel_l2(ckpt[key], full[key]))
    for a, b in zip(full.get("lambdas", []), ckpt.get("lambdas", [])):
        if a is not None and a.numel():
            assert rel_l2(b, a) <= GRAD_TOL, rel_l2(b, a)
    assert ckpt["E_saved"].numel() == 0


CASES = {
    "2d_tm_e_only": (lambda: problem_2d(nt=60, order=4, want_source=True), {}),
    "3d_e_only": (lambda: problem_3d(nt=40, order=4, pml=3, nshot=3, want_source=True), {}),
    "3d_bf16_stored_r_interval2": (lambda: problem_3d(nt=41, order=8, pml=3, nshot=2, storage_kind=2,
                                                      rhs_from_e=False, interval=2, want_source=True), {}),
    "2d_fp8": (lambda: problem_2d(nt=60, order=4, want_source=True), {"wavefield_compression": "fp8"}),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("segments,batch", [(8, None), (8, 1)])
def test_checkpointed_equals_single_call(case, segments, batch, cuda_device):
    make, kw = CASES[case]
    p = make()
    if "3d" in case:
        p.initial_states, p.state_duals = _random_states(p)
    full = run_product(p, cuda_device, **kw)
    ckpt = run_product(p, cuda_device, checkpoint_segments=segments, checkpoint_shot_batch=batch, **kw)
    _check(full, ckpt)


def test_auto_keeps_the_single_call_when_the_history_fits(cuda_device):
    p = problem_2d(nt=40, order=2)
    out = run_product(p, cuda_device, checkpoint_segments="auto")
    assert out["E_saved"].numel() > 0


def test_receivers_of_a_checkpointed_solve_equal_the_single_call(cuda_device):
    p = problem_3d(nt=20, order=4, pml=3)
    out = run_product(p, cuda_device, backward=False, checkpoint_segments=5)
    full = run_product(p, cuda_device, backward=False)
    assert torch.equal(out["receivers"], full["receivers"])
