"""Pin the oracle: the C restatement must equal the reference CPU backend bit for bit.

The reference backend (src/DeepGPR/lib/deepgpr_cpu.c) is compiled from its
own source into oracle/_ref by ``make -C oracle ref``; both libraries are
driven with identical ABI-6 argument lists.  Runs on CPU.
"""

from __future__ import annotations

import pytest
import torch

from helpers import problem_2d, problem_3d
from oracle import driver

pytestmark = pytest.mark.skipif(not driver.available("ref") and not driver.REF_SOURCE.is_file(),
                                reason="reference CPU library not built and reference source absent")

KEYS = ("receivers", "states", "E_saved", "R_saved", "grad_eps_ext", "grad_sigma_ext", "lambdas",
        "grad_eps", "grad_sigma", "grad_source")


def _equal(a, b):
    if torch.is_tensor(a):
        return torch.equal(a, b)
    return all(_equal(x, y) for x, y in zip(a, b))


CASES = {
    "2d_o2": lambda: problem_2d(nt=60, order=2, want_source=True),
    "2d_o4": lambda: problem_2d(nt=60, order=4, want_source=True),
    "2d_o8": lambda: problem_2d(nt=60, order=8),
    "2d_o4_S3_stored": lambda: problem_2d(nt=61, order=4, interval=3, rhs_from_e=False),
    "2d_bf16": lambda: problem_2d(nt=50, order=2, storage_kind=2),
    "2d_f16_stored": lambda: problem_2d(nt=50, order=2, storage_kind=1, rhs_from_e=False),
    "2d_mode3_ex_source": lambda: problem_2d(nt=40, order=2, mode=3, source_component=0, receiver_component=1),
    "2d_no_pml_physical": lambda: problem_2d(nt=40, order=4, pml=0, region="physical"),
    "3d_o2": lambda: problem_3d(nt=20, order=2),
    "3d_o4_asym_pml": lambda: problem_3d(nt=20, order=4, pml=[3, 2, 4, 1, 2, 3], want_source=True),
    "3d_o8_stored": lambda: problem_3d(nt=15, order=8, shape=(18, 16, 14), pml=4, rhs_from_e=False),
    "3d_aniso": lambda: problem_3d(nt=15, order=4, dx=(0.02, 0.017, 0.013), dt=1e-11),
    "3d_bf16_stored_S2": lambda: problem_3d(nt=16, order=4, storage_kind=2, rhs_from_e=False, interval=2),
    "3d_f16_e_only": lambda: problem_3d(nt=16, order=2, storage_kind=1),
    "3d_no_pml_physical": lambda: problem_3d(nt=12, order=4, pml=0, region="physical"),
    "2d_two_shots_source_grad": lambda: _two_shots_2d(),
}


def _two_shots_2d():
    p = problem_2d(nt=50, order=4, want_source=True)
    p.source_location = torch.tensor([[[10, 10, 0]], [[20, 25, 0]]], dtype=torch.int32)
    p.receiver_location = torch.tensor([[[10, 30, 0], [5, 7, 0]], [[25, 5, 0], [20, 25, 0]]], dtype=torch.int32)
    return p


@pytest.fixture(scope="module", autouse=True)
def _libs():
    driver.build("oracle")
    if driver.REF_SOURCE.is_file():
        driver.build("ref")


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_equals_reference_bitwise(name):
    p = CASES[name]()
    a = driver.run(p, "oracle")
    b = driver.run(p, "ref")
    for key in KEYS:
        if key in a:
            assert _equal(a[key], b[key]), key


def test_coincident_sources_and_receivers_bitwise():
    p = problem_2d(nt=40, order=4, want_source=True)
    p.source_location = torch.tensor([[[10, 10, 0], [10, 10, 0], [12, 20, 0]]], dtype=torch.int32)
    p.source_amplitudes = torch.stack([p.source_amplitudes[0], 0.5 * p.source_amplitudes[0],
                                       -p.source_amplitudes[0]])
    p.receiver_location = torch.tensor([[[10, 10, 0], [10, 10, 0], [5, 5, 0]]], dtype=torch.int32)
    a = driver.run(p, "oracle")
    b = driver.run(p, "ref")
    for key in KEYS:
        if key in a:
            assert _equal(a[key], b[key]), key


def test_random_states_bitwise():
    g = torch.Generator().manual_seed(5)
    p = problem_3d(nt=3, order=4, shape=(9, 10, 8), pml=2, nshot=1, dx=(0.020, 0.017, 0.013), dt=1e-11,
                   want_source=True)
    p.source_location = torch.tensor([[[4, 5, 4]]], dtype=torch.int32)
    p.receiver_location = torch.tensor([[[4, 5, 4], [2, 3, 1]]], dtype=torch.int32)
    base = driver.prepare(p)[3]
    from deepgpr_b200.pml import build_psi

    shape = (1, base.nx + 1, base.ny + 1, base.nz + 1)
    zeros = [torch.zeros(shape) for _ in range(6)] + list(build_psi(base.nx, base.ny, base.nz, base.pml, 1, None, "cpu"))
    p.initial_states = [torch.randn(t.shape, generator=g) * 1e-3 for t in zeros]
    p.state_duals = [torch.randn(t.shape, generator=g) for t in zeros]
    p.data_grad = torch.randn((1, 3, 2), generator=g)
    a = driver.run(p, "oracle")
    b = driver.run(p, "ref")
    for key in KEYS:
        if key in a:
            assert _equal(a[key], b[key]), key
