"""Asynchronous history offload (``use_async_offload=True``) against the device-resident history.

With offload the history lives in pinned host memory; the kernels write it
(forward) and read it (adjoint) through device ring buffers that a copy
stream moves to and from the host chunk by chunk, beside the computation.
The arithmetic is unchanged, so receivers, final states, the saved history
and every gradient are bit for bit those of the resident run (reference
contract: src/DeepGPR/lib/deepgpr.cu:3702-3744 D2H double buffer,
:4007-4026 H2D staging).
"""

from __future__ import annotations

import pytest
import torch

from helpers import problem_2d, problem_3d, run_product

pytestmark = pytest.mark.gpu

CASES = {
    "2d_tm_e_only": lambda: problem_2d(nt=150, order=4, want_source=True),
    "2d_fp16_stored_r": lambda: problem_2d(nt=130, order=2, storage_kind=1, rhs_from_e=False),
    "3d_e_only": lambda: problem_3d(nt=90, order=4, pml=3, nshot=2, want_source=True),
    "3d_bf16_stored_r_interval3": lambda: problem_3d(nt=101, order=8, pml=3, nshot=2, storage_kind=2,
                                                     rhs_from_e=False, interval=3),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_offloaded_history_equals_resident(case, cuda_device):
    p = CASES[case]()
    res = run_product(p, cuda_device)
    off = run_product(p, cuda_device, use_async_offload=True)
    assert off["E_saved"].device.type == "cpu" and off["E_saved"].is_pinned()
    assert torch.equal(off["E_saved"].view(torch.uint8), res["E_saved"].cpu().view(torch.uint8))
    assert torch.equal(off["receivers"], res["receivers"])
    for a, b in zip(off["states"], res["states"]):
        assert torch.equal(a, b)
    for key in ("grad_eps", "grad_sigma", "grad_source"):
        if key in res:
            assert torch.equal(off[key], res[key]), key
