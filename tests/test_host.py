"""Host-side logic of the product package (no GPU): options, validation, layouts."""

from __future__ import annotations

import pytest
import torch

import deepgpr_b200 as dg
from deepgpr_b200 import config
from deepgpr_b200.errors import CFLConditionError, NativeLibraryError
from deepgpr_b200.model import prepare_model, shift_locations
from deepgpr_b200.solver import _tm2d_applies
from deepgpr_b200.storage import (
    StorageConfig,
    decode_fp8_history,
    encode_storage_type,
    fp8_tiles,
    history_box,
    resolve_rhs_reconstruction,
    saved_history_shape,
)


def _inputs(nt=10, shape=(20, 16)):
    eps = torch.full(shape, 4.0)
    sig = torch.zeros(shape)
    src = torch.tensor([[[5, 5, 0]]], dtype=torch.int32)
    rcv = torch.tensor([[[6, 6, 0]]], dtype=torch.int32)
    return eps, sig, torch.ones(1, nt), src, rcv


def test_storage_word_matches_reference_bits():
    cfg = StorageConfig(torch.float32, "none", config.STORAGE_FLOAT32)
    assert encode_storage_type(cfg, True) == 0
    assert encode_storage_type(cfg, False) == 1 << 26
    assert encode_storage_type(cfg, True, rhs_from_e=True) == 1 << 4
    assert encode_storage_type(cfg, True, physical=True) == 1 << 5
    assert encode_storage_type(cfg, True, tm2d=True) == 1 << 6
    bf = StorageConfig(torch.bfloat16, "none", config.STORAGE_BFLOAT16)
    assert encode_storage_type(bf, True) == 2
    fp8 = StorageConfig(torch.uint8, "fp8", config.STORAGE_FP8_E4M3)
    assert encode_storage_type(fp8, True) & 0xF == 4


def test_history_shapes_and_boxes():
    assert saved_history_shape(2, 5, 3, 10, 11, 1) == (5, 3, 10, 11, 1)
    assert saved_history_shape(3, 5, 3, 10, 11, 12) == (3, 5, 3, 10, 11, 12)
    assert history_box(40, 30, 1, [10, 10, 5, 5, 0, 0], "physical") == ((10, 5, 0), (20, 20, 1))
    assert history_box(40, 30, 1, [10, 10, 5, 5, 0, 0], "extended") == ((0, 0, 0), (40, 30, 1))


def test_rhs_reconstruction_rules():
    assert resolve_rhs_reconstruction("auto", 1, True, True) is True
    assert resolve_rhs_reconstruction("auto", 2, True, True) is False
    assert resolve_rhs_reconstruction("auto", 1, True, False) is False
    assert resolve_rhs_reconstruction("stored", 1, True, True) is False
    with pytest.raises(ValueError):
        resolve_rhs_reconstruction("reconstructed", 3, True, True)


def test_fp8_decoder_roundtrip():
    torch.manual_seed(0)
    field_shape = (9, 140, 2)
    hx, hy, hz = 8, 139, 1
    vals = torch.randn(2, 3, hx, hy, hz)
    tiles = fp8_tiles(field_shape, True)
    nvals = vals.numel()
    payload = (nvals + 255) // 256 * 256
    packed = torch.zeros(payload + 2 * 3 * tiles * 4, dtype=torch.uint8)
    scales = torch.full((2, 3, tiles), 0.01)
    q = (vals / 0.01).clamp(-448, 448).to(torch.float8_e4m3fn)
    packed[:nvals] = q.reshape(-1).view(torch.uint8)
    packed[payload:] = scales.reshape(-1).view(torch.uint8)
    out = decode_fp8_history(packed, (2, 3, hx, hy, hz), field_shape, (0, 0, 0), tm2d=True)
    assert torch.allclose(out, q.float() * 0.01)


def test_tm2d_decision():
    zeros = [torch.zeros(1)] * 30
    assert _tm2d_applies(2, 2, 2, True, zeros, False)
    assert not _tm2d_applies(3, 2, 2, True, zeros, False)
    assert not _tm2d_applies(2, 0, 2, True, zeros, False)
    assert not _tm2d_applies(2, 2, 3, True, zeros, False)
    assert _tm2d_applies(2, 2, 3, False, zeros, False)
    states = [torch.zeros(2) for _ in range(30)]
    states[0] = torch.ones(2)   # nonzero Ex
    assert not _tm2d_applies(2, 2, 2, True, states, True)


def test_prepare_model_extends_and_validates():
    eps, sig, w, src, rcv = _inputs()
    p = prepare_model("cpu", eps, sig, None, w, src, rcv, 0.02, 1e-11, 3, 4)
    assert (p.nx, p.ny, p.nz) == (26, 22, 1)
    assert p.eps_r_pad.shape == (27, 23, 2)
    assert p.pml == (3, 3, 3, 3, 0, 0)
    assert shift_locations(src, p.pml, "cpu").tolist() == [[[8, 8, 0]]]
    with pytest.raises(ValueError):
        prepare_model("cpu", eps * 0.1, sig, None, w, src, rcv, 0.02, 1e-11, 3, 4)
    with pytest.raises(ValueError):
        prepare_model("cpu", eps, sig, None, w, src + 100, rcv, 0.02, 1e-11, 3, 4)
    with pytest.raises(CFLConditionError):
        prepare_model("cpu", eps, sig, None, w, src, rcv, 0.02, 1e-9, 3, 4)
    with pytest.raises(ValueError):
        prepare_model("cpu", eps, sig, None, w, src, rcv, 0.02, 1e-11, [1, 1, 1, 1, 1, 1], 4)


def test_compute_requires_cuda():
    eps, sig, w, src, rcv = _inputs()
    with pytest.raises(NativeLibraryError):
        dg.compute("cpu", dx=0.02, dt=1e-11, source_amplitudes=w, source_location=src, receiver_location=rcv,
                   eps_r=eps, sigma=sig)


def test_compute_option_errors_match_reference():
    eps, sig, w, src, rcv = _inputs()
    with pytest.raises(ValueError):
        dg.compute("cuda", dx=0.02, dt=1e-11, source_amplitudes=w, source_location=src, receiver_location=rcv,
                   eps_r=eps, sigma=sig, fdtd_order=6)
    with pytest.raises(ValueError):
        dg.compute("cuda", dx=0.02, dt=1e-11, source_amplitudes=w, source_location=src, receiver_location=rcv,
                   eps_r=eps, sigma=sig, mode=4)
    with pytest.raises(NotImplementedError):
        dg.compute("cuda", dx=0.02, dt=1e-11, source_amplitudes=w, source_location=src, receiver_location=rcv,
                   eps_r=eps, sigma=sig, wavefield_compression="zfp")
    with pytest.raises(ValueError):
        dg.compute("cuda", dx=0.02, dt=1e-11, source_amplitudes=w, source_location=src, receiver_location=rcv,
                   eps_r=eps, sigma=sig, save_wavefield_history=False, use_async_offload=True)


def test_int8_and_fp8_compression_options():
    """'int8' (the reference's option name) selects this library's INT8 tile history, kind 3."""
    from deepgpr_b200 import storage

    assert storage.normalize_compression("INT8") == "int8"
    assert storage.normalize_compression("fp8") == "fp8"
    cfg = storage.storage_config(torch.float32, "int8", torch.float32)
    assert cfg.kind == 3 and cfg.compression == "int8" and cfg.dtype == torch.uint8
    shape = (3, 4, 2, 5, 6, 40)
    buf = storage.allocate_history(cfg, shape, (6, 7, 41), False, "cpu", False)
    assert buf.numel() == storage.fp8_history_bytes(3, 4, 2, 5 * 6 * 40, (6, 7, 41), False)


def test_int8_decoder_rounds_trip_within_half_a_step():
    """Tile codes round(x / s), s = absmax / 127: decoding is within s / 2 of every value."""
    from deepgpr_b200 import storage

    g = torch.Generator().manual_seed(4)
    full = (1, 2, 1, 3, 4, 64)
    x = torch.randn(full, generator=g)
    field = (4, 5, 65)
    tiles = storage.fp8_tiles(field, False)
    values = x.numel()
    packed = torch.zeros((values + 255) // 256 * 256 + 2 * tiles * 4, dtype=torch.uint8)
    tile = storage.fp8_tile_of(torch.arange(3).view(3, 1, 1), torch.arange(4).view(1, 4, 1),
                               torch.arange(64).view(1, 1, 64), field, False).expand(3, 4, 64).reshape(-1)
    scales = torch.full((1, 2, 1, tiles), 1e-30)
    flat = x.reshape(1, 2, 1, -1)
    for t in range(2):
        for u in tile.unique().tolist():
            sel = tile == u
            scales[0, t, 0, u] = max(float(flat[0, t, 0, sel].abs().max()) / 127.0, 1e-30)
    s_cell = scales[0, :, 0][:, tile].reshape(full)
    codes = torch.clamp(torch.round(x / s_cell), -127, 127).to(torch.int8)
    packed[:values] = codes.reshape(-1).view(torch.uint8)
    packed[(values + 255) // 256 * 256:] = scales.reshape(-1).view(torch.uint8)
    out = storage.decode_fp8_history(packed, full, field, (0, 0, 0), False, "int8")
    assert torch.all((out - x).abs() <= 0.5 * s_cell + 1e-7)


def test_checkpoint_initial_field_shapes():
    eps, sig, w, src, rcv = _inputs()
    E, H, P = dg.checkpoint_initial_field("cpu", dx=0.02, dt=1e-11, source_amplitudes=w, source_location=src,
                                          receiver_location=rcv, er=eps, se=sig, pmlthick=2)
    assert all(t.shape == (1, 25, 21, 2) for t in (*E, *H))
    assert len(P) == 24
    assert P[0].shape == (1, 3, 20, 2)      # x0 E psi1: (nstep, p+1, ny, nz+1)
    assert P[16].numel() == 0               # z faces disabled in 2D


def test_history_file_naming_and_payload(tmp_path):
    from datetime import datetime

    from deepgpr_b200.history_io import load_forward_wavefield, normalize_forward_wavefield_directory, \
        save_forward_wavefield

    d = normalize_forward_wavefield_directory(tmp_path / "hist")
    t = datetime(2026, 1, 2, 13, 7)
    x = torch.arange(24, dtype=torch.float32).reshape(2, 3, 4)
    p0 = save_forward_wavefield(x, d, t)
    p1 = save_forward_wavefield(x, d, t, metadata={"history_region": "physical", "history_origin": (1, 2, 0)})
    assert p0.name == "forward_wavefield_13-07.pt" and p1.name == "forward_wavefield_13-07_01.pt"
    assert torch.equal(torch.load(p0), x)
    meta = torch.load(p1)
    assert torch.equal(meta["wavefield"], x) and meta["history_origin"] == (1, 2, 0)
    assert torch.equal(load_forward_wavefield(p1), x)
    (tmp_path / "file").write_text("x")
    with pytest.raises(NotADirectoryError):
        normalize_forward_wavefield_directory(tmp_path / "file")


def test_checkpoint_plan_prefers_all_shots_then_the_longest_segments():
    import dataclasses

    from deepgpr_b200.checkpoint import history_bytes_per_step, plan_segments
    from deepgpr_b200.solver import SolverConfig
    from deepgpr_b200.storage import storage_config

    cfg = SolverConfig(device=torch.device("cpu"), dtype=torch.float32, spacing=(0.02,) * 3, dt=1e-11, nx=100, ny=100,
                       nz=100, nt=1000, nstep=8, nsr=1, nrx=4, pml=(10,) * 6, source_component=2,
                       receiver_component=2, interval=1, storage=storage_config(torch.float32, "none", torch.float32),
                       save_history=True, offload=False, fdtd_order=4, mode=3, debug=False, reconstruct_rhs=True,
                       region="extended")
    hist = history_bytes_per_step(cfg)
    assert hist == 3 * 100 ** 3 * 4               # E-only mode 3, FP32, one shot
    state = 6 * 101 ** 3 * 4
    # everything fits: one segment, all shots
    big = plan_segments(cfg, state, 10**13)
    assert (big.nsegments, big.shot_batch, big.forward_passes) == (1, 8, 2)
    # a budget of about a fifth of the history: several segments, still all shots
    mid = plan_segments(cfg, state, 8 * hist * 200)
    assert mid.shot_batch == 8 and 1 < mid.nsegments and mid.peak_bytes <= 8 * hist * 200
    # too little for all shots' checkpoints: shot batches (one more forward pass)
    small = plan_segments(cfg, state, 2 * (state * 40 + hist * 40))
    assert small.shot_batch < 8 and small.forward_passes == 3 and small.peak_bytes <= 2 * (state * 40 + hist * 40)
    # segments are whole multiples of the sampling interval
    c3 = dataclasses.replace(cfg, interval=3, reconstruct_rhs=False)
    p3 = plan_segments(c3, state, 8 * history_bytes_per_step(c3) * 100)
    assert p3.segment_steps % 3 == 0 or p3.segment_steps == c3.nt
    with pytest.raises(MemoryError):
        plan_segments(cfg, state, 1000)


def test_autotune_coordinate_search_and_cache(tmp_path):
    from deepgpr_b200 import autotune

    space = [("tm_chunks", (0, 1, 2, 4)), ("tm_frame_rows", (0, 4, 16)), ("chunk", (16, 32))]
    calls = []

    def cost(c):
        calls.append(dict(c))
        return abs(c["tm_chunks"] - 2) + abs(c["tm_frame_rows"] - 4) * 0.1 + (0.5 if c["chunk"] == 16 else 0.0)

    best, seen = autotune.coordinate_search(space, cost)
    assert (best["tm_chunks"], best["tm_frame_rows"], best["chunk"]) == (2, 4, 32)
    assert len(calls) == len(seen)            # every candidate measured once
    assert autotune.tuning_tuple(best) == (2, 4, 0, -1)

    class Cfg:
        tm2d, nx, ny, nz, pml, nstep, fdtd_order, mode = True, 10, 20, 1, (2, 2, 2, 2, 0, 0), 3, 4, 2
        dtype = torch.float32

        class storage:
            kind = 0

    tuner = autotune.Autotuner(tmp_path / "t.json")
    assert tuner.lookup(Cfg) is None
    tuner.store(Cfg, best)
    again = autotune.Autotuner(tmp_path / "t.json")   # read back from the file
    assert again.lookup(Cfg) == best
    assert "tm2d|10x20x1" in autotune.signature(Cfg)
