"""Generate golden fixtures by running the reference package itself.

Run in a container that has the reference tree (it is not needed afterwards):

    python tests/golden/make_golden.py [/path/to/reference]

Steps: copy the reference ``src/`` to a scratch directory, drop the shipped
binaries, put the CPU library compiled from the reference source
(``oracle/_ref/deepgpr_cpu.so``, built by ``make -C oracle ref``) in its place,
import that copy as ``DeepGPR`` and record, for small seeded inputs:

* ``compute`` receivers and the eps_r / sigma / source gradients (2D order 2,
  a shortened config 1; 2D order 4; 3D order 4, anisotropic spacing);
* the CPML coefficient tensors (``build_pml_coeffs``), face descriptors and
  psi shapes;
* CFL limits (``max_stable_time_step``) of the benchmark grids;
* the replicate-pad extension and its folded backward.

Outputs: ``tests/golden/*.npz`` (small).
"""

from __future__ import annotations

import math
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def load_reference(ref_root: Path):
    scratch = Path(tempfile.mkdtemp(prefix="deepgpr_ref_"))
    shutil.copytree(ref_root / "src", scratch / "src")
    lib = scratch / "src" / "DeepGPR" / "lib"
    for name in ("deepgpr_cpu.so", "deepgpr_cpu.dll", "deepgpr_cpu.dylib", "libomp.dylib"):
        (lib / name).unlink(missing_ok=True)
    subprocess.run(["make", "-s", "-C", str(REPO / "oracle"), "ref"], check=True)
    shutil.copy(REPO / "oracle" / "_ref" / "deepgpr_cpu.so", lib / "deepgpr_cpu.so")
    sys.path.insert(0, str(scratch / "src"))
    import DeepGPR  # noqa: E402

    return DeepGPR


def ricker(nt, dt, f):
    t = torch.arange(nt, dtype=torch.float64) * dt
    a = (math.pi * f * (t - 1.0 / f)) ** 2
    return ((1 - 2 * a) * torch.exp(-a)).float()


def case_2d(order, nt, seed):
    g = torch.Generator().manual_seed(seed)
    eps = torch.full((60, 50), 2.0)
    eps[30:] = 5.0
    eps = eps + 0.5 * torch.rand((60, 50), generator=g)
    sig = 2e-3 * torch.rand((60, 50), generator=g)
    src = torch.tensor([[[10, 10, 0]], [[12, 30, 0]]], dtype=torch.int32)
    rcv = torch.tensor([[[10, 40, 0], [20, 5, 0]], [[10, 40, 0], [12, 30, 0]]], dtype=torch.int32)
    return dict(eps=eps, sig=sig, src=src, rcv=rcv, wave=ricker(nt, 3e-11, 200e6)[None], dx=0.02, dt=3e-11,
                order=order, mode=2, pml=10)


def case_3d(nt, seed):
    g = torch.Generator().manual_seed(seed)
    shape = (14, 12, 10)
    eps = 3.0 + 2.0 * torch.rand(shape, generator=g)
    sig = 2e-3 * torch.rand(shape, generator=g)
    src = torch.tensor([[[7, 6, 5]]], dtype=torch.int32)
    rcv = torch.tensor([[[2, 3, 4], [7, 6, 5], [10, 8, 2]]], dtype=torch.int32)
    return dict(eps=eps, sig=sig, src=src, rcv=rcv, wave=ricker(nt, 1e-11, 400e6)[None], dx=(0.02, 0.017, 0.013),
                dt=1e-11, order=4, mode=3, pml=[3, 2, 4, 1, 2, 3])


def run_case(DeepGPR, c):
    eps = c["eps"].clone().requires_grad_(True)
    sig = c["sig"].clone().requires_grad_(True)
    wave = c["wave"].clone().requires_grad_(True)
    out = DeepGPR.compute("cpu", dx=c["dx"], dt=c["dt"], source_amplitudes=wave, source_location=c["src"],
                          receiver_location=c["rcv"], eps_r=eps, sigma=sig, pmlthick=c["pml"],
                          fdtd_order=c["order"], mode=c["mode"])
    rx = out[-1]
    (rx ** 2).sum().backward()
    return {"receivers": rx.detach().numpy(), "grad_eps": eps.grad.numpy(), "grad_sigma": sig.grad.numpy(),
            "grad_source": wave.grad.numpy()}


def main():
    ref_root = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
    DeepGPR = load_reference(ref_root)
    torch.set_num_threads(1)

    solves = {}
    for name, c in (("2d_o2", case_2d(2, 300, 1)), ("2d_o4", case_2d(4, 200, 2)), ("3d_o4", case_3d(40, 3))):
        res = run_case(DeepGPR, c)
        for k, v in c.items():
            if torch.is_tensor(v):
                solves[f"{name}/in_{k}"] = v.numpy()
        solves[f"{name}/meta"] = np.array([c["order"], c["mode"]])
        for k, v in res.items():
            solves[f"{name}/{k}"] = v
    np.savez_compressed(HERE / "solves.npz", **solves)

    from DeepGPR.solver.pml import build_pml_coeffs, expected_phi_shapes

    pml_fix = {}
    for i, (dx, dt, shape, pml, v) in enumerate((
        (0.02, 3e-11, (120, 120, 1), [10, 10, 10, 10, 0, 0], 299792458.0),
        ((0.02, 0.017, 0.013), 1e-11, (20, 18, 19), [3, 2, 4, 1, 2, 3], 299792458.0),
        (0.01, 1.8e-11, (420, 820, 1), [10, 10, 10, 10, 0, 0], 1.5e8),
    )):
        out = build_pml_coeffs(None, None, dt, dx, *shape, torch.tensor(pml, dtype=torch.int32), "cpu",
                               torch.float32, max_velocity=v)
        for f in range(6):
            d = out[f]
            pml_fix[f"case{i}/desc{f}"] = d.numpy() if d.numel() else np.zeros(0, np.int32)
            pml_fix[f"case{i}/e{f}"] = out[6 + 2 * f].numpy() if out[6 + 2 * f].numel() else np.zeros(0, np.float32)
            pml_fix[f"case{i}/h{f}"] = out[7 + 2 * f].numpy() if out[7 + 2 * f].numel() else np.zeros(0, np.float32)
            shapes = expected_phi_shapes(f, d, 3)
            pml_fix[f"case{i}/phi{f}"] = np.array([s if s is not None else (0, 0, 0, 0) for s in shapes])
        pml_fix[f"case{i}/args"] = np.array([*([dx] * 3 if not isinstance(dx, tuple) else dx), dt, *shape, *pml, v],
                                            dtype=np.float64)
    np.savez_compressed(HERE / "pml.npz", **pml_fix)

    from DeepGPR.preprocessing.model_setup import _ExtendModel
    from DeepGPR.preprocessing.stability import max_stable_time_step

    g = torch.Generator().manual_seed(7)
    model = torch.rand((5, 6, 4), generator=g, dtype=torch.float64).float().requires_grad_(True)
    pmlv = [2, 1, 3, 0, 1, 2]
    ext = _ExtendModel.apply(model, pmlv)
    up = torch.randn(ext.shape, generator=g)
    (ext * up).sum().backward()
    misc = {"extend/model": model.detach().numpy(), "extend/pml": np.array(pmlv), "extend/out": ext.detach().numpy(),
            "extend/up": up.numpy(), "extend/grad": model.grad.numpy()}
    cfl = []
    for dx, dims, order in ((0.02, (120, 120, 1), 2), (0.01, (420, 820, 1), 4), (0.02, (220, 220, 220), 8),
                            (0.015, (340, 340, 180), 4), ((0.02, 0.017, 0.013), (20, 18, 19), 4)):
        d = dx if isinstance(dx, tuple) else (dx, dx, dx)
        cfl.append([*d, *dims, order, max_stable_time_step(dx, *dims, fdtd_order=order)])
    misc["cfl"] = np.array(cfl, dtype=np.float64)
    np.savez_compressed(HERE / "misc.npz", **misc)
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
