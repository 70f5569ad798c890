"""dgb_forward_noalloc (forward without device allocation) against forward.

The file is named to be collected last; each test captures the argument set
of one native ``forward`` call made by ``deepgpr_b200.compute`` and replays it
through both entry points on fresh copies of every buffer, so the test passes
alone in a fresh process as well as after the other GPU tests.
"""

from __future__ import annotations

import pytest
import torch

from helpers import problem_2d, problem_3d, rel_l2, run_product

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
    from deepgpr_b200 import native

    out = _snapshot(args)
    native.invoke(name, out, **opts)
    torch.cuda.synchronize()
    return out


def _assert_same(ref, got):
    for key, r in ref.items():
        if not torch.is_tensor(r):
            continue
        g = got[key]
        assert g.shape == r.shape, key
        if r.numel() == 0:
            continue
        if r.is_floating_point():
            if r.abs().max() == 0:
                assert g.abs().max() == 0, key
            else:
                assert rel_l2(g.float().cpu(), r.float().cpu()) <= 1e-5, key
        else:
            assert torch.equal(g.cpu(), r.cpu()), key


CASES = {
    "3d_fp32": (lambda: problem_3d(nt=30, order=4, nshot=2), {}),
    "tm2d_e_only": (lambda: problem_2d(nt=60, order=4, shape=(60, 96)), {}),
    "tm2d_fp8": (lambda: problem_2d(nt=60, order=4, shape=(60, 96)), {"wavefield_compression": "fp8"}),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_forward_matches_forward_on_two_calls(case, cuda_device):
    make, kw = CASES[case]
    args, opts = _capture_forward(make(), cuda_device, **kw)
    ref = _replay("forward", args, opts)
    for _ in range(2):   # the static scratch is reused by the second call
        _assert_same(ref, _replay("dgb_forward_noalloc", args, opts))


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
