"""save_forward_wavefield_path: the history written next to the solve reads back as E_saved."""

from __future__ import annotations

import pytest
import torch

from helpers import problem_2d, problem_3d

pytestmark = pytest.mark.gpu


def _run(p, device, path, **kw):
    import deepgpr_b200 as dg

    eps = p.eps_r.to(device).requires_grad_(True)
    out = dg.compute(device, eps_r=eps, sigma=p.sigma.to(device), source_amplitudes=p.source_amplitudes.to(device),
                     source_location=p.source_location.to(device), receiver_location=p.receiver_location.to(device),
                     dx=p.dx, dt=p.dt, pmlthick=p.pml, fdtd_order=p.order, mode=p.mode,
                     save_forward_wavefield_path=path, **kw)
    return out[0]


@pytest.mark.parametrize("dims,kw", [(2, {}), (3, {}), (2, {"wavefield_compression": "fp8"}),
                                     (3, {"wavefield_history_region": "physical", "pmlthick_zero": True})])
def test_saved_history_reads_back(dims, kw, tmp_path, cuda_device):
    from deepgpr_b200.history_io import load_forward_wavefield
    from deepgpr_b200.storage import decode_fp8_history

    kw = dict(kw)
    zero = kw.pop("pmlthick_zero", False)
    p = problem_2d(nt=40, order=4) if dims == 2 else problem_3d(nt=20, order=4, pml=0 if zero else 3)
    e_saved = _run(p, cuda_device, tmp_path, **kw)
    files = sorted(tmp_path.glob("forward_wavefield_*.pt"))
    assert len(files) == 1
    got = load_forward_wavefield(files[0])
    if kw.get("wavefield_compression") == "fp8":
        meta = torch.load(files[0], weights_only=True)
        want = decode_fp8_history(e_saved.cpu(), meta["uncompressed_shape"], tuple(meta["field_shape"]),
                                  tuple(meta["history_origin"]), bool(meta["tm2d"]))
        assert got.shape == tuple(meta["uncompressed_shape"])
        assert torch.equal(got, want)
    else:
        assert torch.equal(got, e_saved.cpu())
