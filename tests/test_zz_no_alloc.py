"""dgb_forward_noalloc (forward without device allocation) against forward.

Some callers cannot let a solve allocate GPU memory: a serving process that
has handed the free memory of the GPU to its own pool, or code that holds a
fixed per-request budget.  ``dgb_forward_noalloc`` takes its scratch from a
static device array instead.  These tests check, through the C-ABI, that

* it returns bit for bit what ``forward`` returns (same kernels, same order;
  only how the time steps are issued differs), on two calls in a row, so the
  second call reuses the static scratch the first one left behind;
* it allocates nothing: the device's stream-ordered pool (which ``forward``
  draws on) keeps its high-water mark, and PyTorch's reserved memory does not
  change across the call;
* a solve whose scratch exceeds the static array is rejected before it
  touches an output.

The file is named to be collected last; each test captures the argument set
of one native ``forward`` call made by ``deepgpr_b200.compute`` and replays it
through both entry points on fresh copies of every buffer, so the tests pass
alone in a fresh process as well as after the other GPU tests.
"""

from __future__ import annotations

import pytest
import torch

from helpers import problem_2d, problem_3d, run_product

pytestmark = pytest.mark.gpu


def _snapshot(args):
    return {k: (v.detach().clone() if torch.is_tensor(v) else v) for k, v in args.items()}


def _capture_forward(p, device, **compute_kw):
    """Arguments of the first native forward call of compute(), before it ran."""
    from deepgpr_b200 import native

    seen = {}
    real = native.invoke

    def spy(name, args, **opts):
        if name == "forward" and "args" not in seen:
            seen["args"] = _snapshot(args)
            seen["opts"] = opts
        return real(name, args, **opts)

    native.invoke = spy
    try:
        run_product(p, device, backward=False, **compute_kw)
    finally:
        native.invoke = real
    assert "args" in seen, "compute() made no forward call"
    return seen["args"], seen["opts"]


def _replay(name, args, opts):
    """Fresh copies of every buffer, then the call; returns (outputs, pool growth, torch growth)."""
    from deepgpr_b200 import native

    out = _snapshot(args)
    torch.cuda.synchronize()
    reserved0 = torch.cuda.memory_reserved()
    used0, _ = native.default_pool_usage(reset_high=True)
    native.invoke(name, out, **opts)
    torch.cuda.synchronize()
    _, high = native.default_pool_usage()
    return out, high - used0, torch.cuda.memory_reserved() - reserved0


def _assert_bitwise(ref, got):
    for key, r in ref.items():
        if not torch.is_tensor(r):
            continue
        g = got[key]
        assert g.shape == r.shape and g.dtype == r.dtype, key
        if r.numel():   # compare the bytes: NaN payloads and signed zeros included
            assert torch.equal(g.contiguous().view(-1).view(torch.uint8), r.contiguous().view(-1).view(torch.uint8)), key


CASES = {
    "3d_fp32": (lambda: problem_3d(nt=30, order=4, nshot=2), {}),
    "tm2d_e_only": (lambda: problem_2d(nt=60, order=4, shape=(60, 96)), {}),
    "tm2d_fp8": (lambda: problem_2d(nt=60, order=4, shape=(60, 96)), {"wavefield_compression": "fp8"}),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_forward_matches_forward_on_two_calls(case, cuda_device):
    make, kw = CASES[case]
    args, opts = _capture_forward(make(), cuda_device, **kw)
    ref, pool_grew, _ = _replay("forward", args, opts)
    assert pool_grew > 0, "forward draws its scratch from the stream-ordered pool"
    for _ in range(2):   # the second call reuses the static scratch the first one used
        got, pool_grew, torch_grew = _replay("dgb_forward_noalloc", args, opts)
        _assert_bitwise(ref, got)
        assert pool_grew == 0, f"dgb_forward_noalloc allocated {pool_grew} bytes from the pool"
        assert torch_grew == 0, f"PyTorch reserved {torch_grew} more bytes during the call"


def test_noalloc_rejects_a_solve_larger_than_its_static_scratch(cuda_device):
    from deepgpr_b200 import native

    # 2D TM working copy of 8 shots on 420 x 820 cells: about 40 MB > 8 MiB
    p = problem_2d(nt=2, order=4, shape=(400, 800))
    p.source_location = torch.tensor([[[200, 100 + 50 * s, 0]] for s in range(8)], dtype=torch.int32)
    p.receiver_location = torch.tensor([[[200, 400, 0]]] * 8, dtype=torch.int32)
    args, opts = _capture_forward(p, cuda_device)
    before = _snapshot(args)
    out = _snapshot(args)
    with pytest.raises(native.NativeLibraryError, match="static device scratch"):
        native.invoke("dgb_forward_noalloc", out, **opts)
    torch.cuda.synchronize()
    for key in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "receiver_data"):
        assert torch.equal(out[key], before[key]), key
