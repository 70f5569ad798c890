#!/usr/bin/env python
"""Benchmark: 2D multi-shot FWI gradient (forward + exact adjoint) on B200.

Workload (one "step" = one full gradient evaluation): physical grid 400 x 800
(dx = 0.01 m, CPML 10 -> 420 x 820 extended cells), 32 shots, 200 receivers
per shot, nt = 3000, fdtd_order 4, gradient mode 2 (Ez), FP32 E-only history
(132 GB, resident in HBM), Ricker 400 MHz, dt = 0.9 CFL, L2 misfit against
data of the same model with an eps_r = 9 disc.  Models are seeded synthetic
(deepgpr_b200.synthetic.fwi_2d); no dataset is read.

metric: cell-updates/s = 2 (forward + adjoint) x extended cells x nt x shots
per step / device time.  Inputs (fields 132 MB, history 132 GB) are larger
than L2, so no flush is needed between steps.

Multi-GPU (torchrun): every rank solves its own 32 shots (weak scaling) and
the material gradient is summed with one NCCL all-reduce per step.

The line also carries "north_star_3d": the 3D order-4 forward and adjoint
on the 320 x 320 x 160 grid of the precision study (CPML 10 -> 340 x 340 x
180 extended cells, gradient mode 3, FP32 E-only history, 32 x 32 receivers),
on a bounded sample of 4 shots and 40 time steps, with the kernels' CUDA-event
time split into forward (H, E) and adjoint (E, H, imaging) and their HBM
roofline fractions at 72 B (forward + E history) and 104 B (adjoint) per
cell-update.

"serving" (also in the line; ``--only-serving`` prints it alone): a seeded
Poisson stream with config 4's request mix (nt scaled by 0.1, 40 requests,
all arriving within ~0.6 s so both paths run at capacity) served by
``deepgpr_b200.serving.SolveServer`` (8 slots; FP32 histories, and again with
INT8 one-byte histories) and, for comparison, by plain per-request
``compute`` (+ ``backward``) calls one after another (FP32 histories; with the
library's default memory policy and with the server's); solves/s and p50/p99
latency of every arm, and the relative L2 error of every arm's gradients
against an FP64 solve of each gradient request of the stream.

``--impl reference`` times the reference's own C/OpenMP CPU backend
(oracle/_ref, compiled from the reference source) on a bounded sample of the
same workload with all host threads.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import torch  # noqa: E402

METRIC = "cell-updates/s"
UNIT = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--nt", type=int, default=3000)
    ap.add_argument("--shots", type=int, default=32)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-3d", action="store_true")
    ap.add_argument("--only-3d", action="store_true", help="print the north_star_3d object alone (profiling)")
    ap.add_argument("--nt-3d", type=int, default=40)
    ap.add_argument("--shape-3d", default="320,320,160", help="physical grid of the 3D measurement")
    ap.add_argument("--pml-3d", type=int, default=10, help="CPML thickness of the 3D measurement")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--only-serving", action="store_true", help="print the serving object alone")
    ap.add_argument("--serving-requests", type=int, default=40)
    ap.add_argument("--serving-history", default="fp32", choices=("int8", "fp8", "bf16", "fp32"),
                    help="history format of the served arm")
    ap.add_argument("--cpu-sample", action="store_true", help="time the CPU backend sample alone (internal)")
    ap.add_argument("--config3", action="store_true",
                    help="3D order-8 gradient of the 200^3 config (8 shots, nt 2500, BF16 E+R history) with "
                         "segment checkpointing; prints its own JSON object")
    ap.add_argument("--config3-nt", type=int, default=2500)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    return ap.parse_args()


def dist_setup(n: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return rank, world, local


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path("/tmp") / f"bench_clocks_{os.getpid()}.csv"

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.is_file():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        busy = [v for v in sm if v > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.is_file():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Algorithmic bytes per shot-cell per launch of each 2D TM kernel (FP32):
# every array a kernel must read or write once, coefficients per shot
# (one shot per CTA), E^n history write in the H kernel (E-only history).
BYTES_PER_CELL_2D = {
    "fwd_h": 4 + 8 + 8 + 4 + 4,      # Ez r, Hx rw, Hy rw, ch_curl r, E^n w
    "fwd_e": 4 + 4 + 8 + 4 + 4,      # Hy r, Hx r, Ez rw, ce_hist r, ce_curl r
    "adj_e": 4 + 4 + 8 + 8,          # lEz r, ce_curl r, lHx rw, lHy rw
    "adj_h": 4 + 4 + 4 + 8 + 4,      # lHy r, ch_curl r, lHx r, lEz rw, ce_hist r
    "image": 4 + 4 + 4,              # lEz, E^n, E^(n+1) per shot (per-cell terms amortised)
}

# DRAM bytes per shot-cell and launch (frame + interior kernel of a half step), measured with
# ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the 400 x 800 grid with 32 shots and
# nt = 20 (one gradient evaluation).  Below the algorithmic bytes: the 132 MB of fields stay
# partly resident in the 126 MB L2.
DRAM_BYTES_PER_CELL_2D = {"fwd_h": 18.99, "fwd_e": 14.69, "adj_e": 16.18, "adj_h": 15.05, "image": 13.41}


def ours(args, rank, world, local):
    import deepgpr_b200 as dg
    from deepgpr_b200 import native
    from deepgpr_b200.synthetic import fwi_2d

    from deepgpr_b200.shots import ShotGroup, shard_acquisition

    dev = torch.device("cuda", local)
    # weak scaling: the acquisition has args.shots shots per rank; each rank solves its contiguous share
    acq = fwi_2d(seed=1002, nt=args.nt, nshot=args.shots * world)
    acq.sources, acq.receivers, _ = shard_acquisition(acq.sources, acq.receivers, world, rank)
    group = ShotGroup(timeout_s=120.0) if world > 1 else None
    nx, ny = acq.eps_r.shape
    ext_cells = (nx + 20) * (ny + 20)
    shots = acq.sources.shape[0]
    units_per_step = 2 * ext_cells * args.nt * shots
    step_no = [0]

    common = dict(dx=acq.dx, dt=acq.dt, pmlthick=10, fdtd_order=acq.order, mode=2)
    src_d, rcv_d = acq.sources.to(dev), acq.receivers.to(dev)
    wave_d = acq.wavelet.to(dev)
    with torch.no_grad():
        obs = dg.compute(dev, source_amplitudes=wave_d, source_location=src_d, receiver_location=rcv_d,
                         eps_r=acq.eps_true.to(dev), sigma=acq.sigma.to(dev), save_wavefield_history=False,
                         **common)[-1].clone()
    eps0, sig0 = acq.eps_r.to(dev), acq.sigma.to(dev)

    def gradient(eps_in, sig_in, wave, src, rcv, data):
        eps = eps_in.detach().requires_grad_(True)
        sig = sig_in.detach().requires_grad_(True)
        out = dg.compute(dev, source_amplitudes=wave, source_location=src, receiver_location=rcv, eps_r=eps,
                         sigma=sig, **common)
        loss = 0.5 * ((out[-1] - data) ** 2).sum()
        del out
        loss.backward()
        ge, gs = eps.grad, sig.grad
        if group is not None:
            # the one exchange of a shot-parallel gradient: sum over the ranks' shots
            group.reduce(step_no[0], [ge, gs])
        step_no[0] += 1
        return loss.detach(), ge, gs

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        gradient(eps0, sig0, wave_d, src_d, rcv_d, obs)
    barrier()
    launches0 = native.launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        start.record()
        for _ in range(args.steps):
            loss, ge, gs = gradient(eps0, sig0, wave_d, src_d, rcv_d, obs)
        stop.record()
        barrier()
    launches = native.launch_count() - launches0
    ms = start.elapsed_time(stop)
    ms_max = ms
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = units_per_step * world * args.steps / (ms_max / 1e3)

    # end to end: host (pinned) inputs copied in and the loss + gradients copied out every step
    e2e = None
    if not args.no_e2e:
        h_eps, h_sig = acq.eps_r.pin_memory(), acq.sigma.pin_memory()
        h_wave, h_src, h_rcv = acq.wavelet.pin_memory(), acq.sources.pin_memory(), acq.receivers.pin_memory()
        h_obs = obs.cpu().pin_memory()
        out_loss = torch.empty((), pin_memory=True)
        out_ge = torch.empty_like(h_eps).pin_memory()
        out_gs = torch.empty_like(h_sig).pin_memory()
        h2d = sum(t.numel() * t.element_size() for t in (h_eps, h_sig, h_wave, h_src, h_rcv, h_obs))
        d2h = sum(t.numel() * t.element_size() for t in (out_loss, out_ge, out_gs))
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            d_eps = h_eps.to(dev, non_blocking=True)
            d_sig = h_sig.to(dev, non_blocking=True)
            d_wave = h_wave.to(dev, non_blocking=True)
            d_src = h_src.to(dev, non_blocking=True)
            d_rcv = h_rcv.to(dev, non_blocking=True)
            d_obs = h_obs.to(dev, non_blocking=True)
            loss, ge, gs = gradient(d_eps, d_sig, d_wave, d_src, d_rcv, d_obs)
            out_loss.copy_(loss, non_blocking=True)
            out_ge.copy_(ge, non_blocking=True)
            out_gs.copy_(gs, non_blocking=True)
        e1.record()
        barrier()
        ems = e0.elapsed_time(e1)
        if world > 1:
            import torch.distributed as dist

            t = torch.tensor([ems], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": units_per_step * world * args.steps / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": ems / args.steps}

    # roofline of the dominant kernel: CUDA-event time of every launch in one profiled step
    native.profile(True)
    gradient(eps0, sig0, wave_d, src_d, rcv_d, obs)
    torch.cuda.synchronize()
    prof = native.profile_read()
    native.profile(False)
    peak, peak_kind = peaks()
    dom = max(prof, key=lambda k: prof[k][0])
    dom_ms, dom_n = prof[dom]
    shot_cells = (nx + 21) * (ny + 21) * shots   # field grid incl. halo, all shots of this rank
    alg = BYTES_PER_CELL_2D[dom] * shot_cells
    achieved = alg / (dom_ms / max(dom_n, 1) / 1e3) / 1e9
    traffic = DRAM_BYTES_PER_CELL_2D[dom] * shot_cells
    total_prof = sum(v[0] for v in prof.values())
    roofline = {
        "bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
        "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
        "algorithmic_bytes_per_launch": alg,
        "kernel_share": {k: round(v[0] / total_prof, 4) for k, v in prof.items() if v[1]},
        "avg_launch_us": {k: round(v[0] / v[1] * 1e3, 2) for k, v in prof.items() if v[1]},
    }

    ns3d = None
    if rank == 0 and world == 1 and not args.no_3d:
        ns3d = north_star_3d(dev, nt=args.nt_3d, shape=tuple(int(v) for v in args.shape_3d.split(",")))

    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        # a serving process runs with PyTorch's stream-ordered allocator (see deepgpr_b200.serving)
        env = dict(os.environ, PYTORCH_CUDA_ALLOC_CONF="backend:cudaMallocAsync")
        cmd = [sys.executable, str(Path(__file__).resolve()), "--only-serving",
               "--serving-requests", str(args.serving_requests), "--serving-history", args.serving_history]
        proc = subprocess.run(cmd, env=env, capture_output=True, text=True)
        try:
            serving = json.loads(proc.stdout.strip().splitlines()[-1])
        except (IndexError, json.JSONDecodeError):
            serving = {"error": (proc.stderr or proc.stdout)[-500:]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args.shots, budget_s=15.0)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered model + random field)",
            "config": {"workload": "2D multi-shot FWI gradient (forward + adjoint)", "grid": [nx, ny, 1],
                       "extended": [nx + 20, ny + 20, 1], "shots_per_gpu": shots, "receivers": 200, "nt": args.nt,
                       "fdtd_order": 4, "mode": 2, "history": "FP32 E-only (resident)",
                       "l2_policy": "inputs larger than L2 (132 MB fields, 132 GB history)"},
            "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clocks.summary(), "loss": float(loss), "north_star_3d": ns3d, "serving": serving,
        }
        print(json.dumps(line), flush=True)


# Algorithmic bytes per 3D cell-update (FP32): forward with E-only mode-3
# history (E3, H3 rw + ce_hist, ce_curl, ch_curl + E^n), adjoint (lambda 6
# components rw + 4 coefficients + E^n, E^(n+1) for 3 components + the
# eps_r / sigma gradients rw).
BYTES_PER_CELL_3D = {"forward": 72, "adjoint": 104}


def north_star_3d(dev, shots=4, nt=40, warmup=1, steps=2, shape=(320, 320, 160), pml=10):
    """3D order-4 forward + adjoint: kernel time split and HBM roofline fractions."""
    import deepgpr_b200 as dg
    from deepgpr_b200 import native
    from deepgpr_b200.synthetic import fwi_3d

    acq = fwi_3d(seed=1005, shape=shape, dx=0.015, sources_grid=(2, 2), receivers_grid=(32, 32), nt=nt, order=4)
    common = dict(dx=acq.dx, dt=acq.dt, pmlthick=pml, fdtd_order=4, mode=3)
    src, rcv, wave = acq.sources.to(dev), acq.receivers.to(dev), acq.wavelet.to(dev)
    eps0, sig0 = acq.eps_r.to(dev), acq.sigma.to(dev)

    def gradient():
        eps = eps0.clone().requires_grad_(True)
        sig = sig0.clone().requires_grad_(True)
        out = dg.compute(dev, source_amplitudes=wave, source_location=src, receiver_location=rcv, eps_r=eps,
                         sigma=sig, **common)
        loss = (out[-1] ** 2).sum()
        del out
        loss.backward()
        return loss.detach()

    for _ in range(warmup):
        gradient()
    torch.cuda.synchronize()
    tot = {}
    native.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        gradient()
    e1.record()
    torch.cuda.synchronize()
    prof = native.profile_read()
    native.profile(False)
    ext = tuple(n + 2 * pml for n in shape)
    cells = ext[0] * ext[1] * ext[2]
    units = cells * nt * acq.sources.shape[0] * steps
    peak, peak_kind = peaks()
    fwd_ms = prof["fwd_h"][0] + prof["fwd_e"][0]
    adj_ms = prof["adj_e"][0] + prof["adj_h"][0] + prof["image"][0]
    fwd_rate, adj_rate = units / (fwd_ms / 1e3), units / (adj_ms / 1e3)
    return {
        "workload": f"3D order-4 forward + adjoint, {shape[0]}x{shape[1]}x{shape[2]} (ext {ext[0]}x{ext[1]}x{ext[2]}),"
                    " mode 3, FP32 E-only history",
        "sample": f"{acq.sources.shape[0]} shots x {nt} steps per gradient, {steps} gradients (of 16 shots x 3000)",
        "forward_cell_updates_per_s": fwd_rate, "adjoint_cell_updates_per_s": adj_rate,
        "gradient_cell_updates_per_s": 2 * units / (e0.elapsed_time(e1) / 1e3),
        "forward_roofline_frac": round(fwd_rate * BYTES_PER_CELL_3D["forward"] / (peak * 1e9), 4),
        "adjoint_roofline_frac": round(adj_rate * BYTES_PER_CELL_3D["adjoint"] / (peak * 1e9), 4),
        "bytes_per_cell_update": BYTES_PER_CELL_3D, "peak_gbs": peak, "peak_source": peak_kind,
        "kernel_ms_per_gradient": {k: round(v[0] / steps, 3) for k, v in prof.items() if v[1]},
    }


def config3_measure(dev, nt=2500, steps=1):
    """Config 3 in full: 200^3 (+ CPML 10), 8 shots on a 2 x 4 surface grid, 24 x 24 receivers, order 8,
    gradient mode 3, BF16 stored E^n and R^n histories (2.56 TB for nt 2500), so the gradient runs with
    segment checkpointing and recompute; cell-updates/s counts forward + adjoint once each."""
    import deepgpr_b200 as dg
    from deepgpr_b200.synthetic import fwi_3d

    acq = fwi_3d(seed=1003, shape=(200, 200, 200), dx=0.02, sources_grid=(2, 4), receivers_grid=(24, 24), nt=nt,
                 order=8)
    src, rcv, wave = acq.sources.to(dev), acq.receivers.to(dev), acq.wavelet.to(dev)
    eps0, sig0 = acq.eps_r.to(dev), acq.sigma.to(dev)
    plan_box = {}

    def gradient():
        from deepgpr_b200 import checkpoint as ck

        real = ck.CheckpointedFDTDFunction.apply

        def spy(cfg, tensors, plan, *rest):
            plan_box["plan"] = plan
            return real(cfg, tensors, plan, *rest)

        ck.CheckpointedFDTDFunction.apply = spy
        try:
            eps = eps0.clone().requires_grad_(True)
            sig = sig0.clone().requires_grad_(True)
            out = dg.compute(dev, source_amplitudes=wave, source_location=src, receiver_location=rcv, eps_r=eps,
                             sigma=sig, dx=acq.dx, dt=acq.dt, pmlthick=10, fdtd_order=8, mode=3,
                             wavefield_storage_dtype=torch.bfloat16, wavefield_rhs_history="stored",
                             checkpoint_segments="auto")
            loss = (out[-1] ** 2).sum()
            del out
            loss.backward()
        finally:
            ck.CheckpointedFDTDFunction.apply = real
        return loss.detach()

    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        loss = gradient()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    cells = 220 ** 3
    units = 2 * cells * nt * acq.sources.shape[0]
    plan = plan_box.get("plan")
    return {
        "workload": "config 3: 3D order-8 gradient, 200^3 (ext 220^3), 8 shots, 24x24 receivers, mode 3, "
                    f"BF16 E+R history, nt {nt}",
        "ms_per_gradient": ms, "cell_updates_per_s": units / (ms / 1e3), "loss": float(loss),
        "history_bytes_full": 2 * 3 * 2 * cells * nt * 8,
        "plan": None if plan is None else {"shot_batch": plan.shot_batch, "segment_steps": plan.segment_steps,
                                           "segments": plan.nsegments, "forward_passes": plan.forward_passes,
                                           "peak_gib": round(plan.peak_bytes / 2**30, 1)},
    }


def serving_measure(dev, n=40, slots=8, history="fp32"):
    """Config-4 stream: continuous-batching server vs plain per-request launches.

    Arms, in this order: plain per-request ``compute`` (+ ``backward``) calls
    with the library's default memory policy; the same with the server's
    policy (freed memory kept mapped in the stream-ordered pool, so pool
    unmapping at synchronisations does not enter the comparison); the server
    with ``history`` histories; the server with INT8 one-byte histories.  Every
    gradient of every arm is compared with an FP64 solve of the same request.
    """
    from deepgpr_b200 import native
    from deepgpr_b200.serving import SolveServer, percentile, run_plain
    from deepgpr_b200.synthetic import serving_stream

    reqs, arrivals = serving_stream(n=n)
    warm, _ = serving_stream(seed=7, n=4, nt_scale=0.02)
    run_plain(warm, dev)                                   # load, first-call set-up
    torch.cuda.synchronize()
    plain_default = run_plain(reqs, dev, arrivals=arrivals, history="fp32")
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info(dev)
    native.set_scratch_retention(int(0.8 * free))
    plain = run_plain(reqs, dev, arrivals=arrivals, history="fp32")
    torch.cuda.synchronize()
    native.set_scratch_retention(0)

    def serve(fmt):
        with SolveServer(dev, slots=slots, history=fmt) as srv:
            for f in [srv.submit(r) for r in warm]:
                f.result()
            t0 = time.perf_counter()
            futs = []
            for req, at in zip(reqs, arrivals):
                wait = at - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
                futs.append(srv.submit(req))
            out = [f.result() for f in futs]
            return out, srv.peak_running, srv.peak_reserved

    served, peak_running, peak_reserved = serve(history)
    served_i8, peak_running_i8, peak_reserved_i8 = serve("int8")

    def summary(res):
        span = max(r.finished for r in res) - min(r.submitted for r in res)
        lat = [r.latency for r in res]
        return {"solves_per_s": len(res) / span, "p50_latency_s": percentile(lat, 50),
                "p99_latency_s": percentile(lat, 99), "span_s": span}

    sp, sd, ss, si = summary(plain), summary(plain_default), summary(served), summary(served_i8)
    kinds = {k: sum(r.kind == k for r in reqs) for k in ("forward", "gradient")}
    arms = {"plain_fp32": plain, f"served_{history}": served}
    if history != "int8":
        arms["served_int8"] = served_i8
    error = served_gradient_error(reqs, arms, dev)
    plain_path = "compute (+ backward) per request, one after another"
    return {
        "workload": "config-4 request mix (2D forward 128^2-1024^2 x 1-16 shots, order 2/4; 3D gradient "
                    "96^3-160^3 x 1-4 shots, order 4), seeded Poisson arrivals",
        "sample": f"{n} requests ({kinds['forward']} forward, {kinds['gradient']} gradient), nt scaled by 0.1, "
                  f"arrivals within {arrivals[-1]:.2f} s",
        "plain": dict(sp, history="fp32", path=plain_path,
                      memory="freed memory kept mapped, as in the server"),
        "plain_default_pool": dict(sd, history="fp32", path=plain_path,
                                   memory="library default (pool trimmed at synchronisations)"),
        "served": dict(ss, history=history, slots=slots, peak_running=peak_running,
                       peak_reserved_gib=round(peak_reserved / 2**30, 2)),
        "served_int8": dict(si, history="int8", slots=slots, peak_running=peak_running_i8,
                            peak_reserved_gib=round(peak_reserved_i8 / 2**30, 2)),
        "speedup_solves_per_s": ss["solves_per_s"] / sp["solves_per_s"],
        "speedup_int8_solves_per_s": si["solves_per_s"] / sp["solves_per_s"],
        "speedup_vs_default_pool": ss["solves_per_s"] / sd["solves_per_s"],
        "gradient_error_vs_fp64": error,
    }


def served_gradient_error(reqs, arms, dev, budget_bytes=40 * 2**30):
    """Relative L2 error of each arm's gradients (``arms``: name -> results in
    request order) against an FP64 solve of each gradient request.

    Requests whose FP64 history would exceed ``budget_bytes`` are skipped."""
    import deepgpr_b200 as dg

    def rel(a, b):
        b = b.double().cpu()
        return float((a.double().cpu() - b).norm() / b.norm())

    errs = {name: ([], []) for name in arms}
    skipped = 0
    for n, req in enumerate(reqs):
        if req.kind != "gradient":
            continue
        pml = req.pmlthick if isinstance(req.pmlthick, int) else max(req.pmlthick)
        cells = 1
        for m in req.eps_r.shape:
            cells *= m + 2 * pml + 1
        comps = 3 if req.mode == 3 else 1
        if cells * req.source_location.shape[0] * req.source_amplitudes.shape[-1] * 8 * comps > budget_bytes:
            skipped += 1
            continue
        f64 = torch.float64
        eps = req.eps_r.to(dev, f64).requires_grad_(True)
        sig = req.sigma.to(dev, f64).requires_grad_(True)
        rx = dg.compute(dev, eps_r=eps, sigma=sig, source_amplitudes=req.source_amplitudes.to(dev, f64),
                        source_location=req.source_location.to(dev), receiver_location=req.receiver_location.to(dev),
                        dx=req.dx, dt=req.dt, pmlthick=req.pmlthick, fdtd_order=req.fdtd_order, mode=req.mode,
                        precision=f64)[-1]
        (0.5 * ((rx - req.observed.to(dev, f64)) ** 2).sum()).backward()
        for name, res in arms.items():
            errs[name][0].append(rel(res[n].grad_eps_r, eps.grad))
            errs[name][1].append(rel(res[n].grad_sigma, sig.grad))
        del eps, sig, rx
        torch.cuda.empty_cache()
    out = {"requests": len(next(iter(errs.values()))[0]), "skipped": skipped,
           "oracle": "FP64 run of the same request"}
    for name, (e, s) in errs.items():
        if e:
            out[name] = {"eps_r_max": max(e), "sigma_max": max(s), "eps_r_median": statistics.median(e),
                         "sigma_median": statistics.median(s)}
    return out


def host_cpu():
    """CPU model and the logical CPUs / physical cores this process may run on."""
    cpus = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else list(range(os.cpu_count() or 1))
    model, cores, cur = "unknown", set(), {}
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines() + [""]:
            if not line.strip():
                if cur.get("processor") is not None and int(cur["processor"]) in cpus:
                    cores.add((cur.get("physical id", "0"), cur.get("core id", cur["processor"])))
                    model = cur.get("model name", model)
                cur = {}
                continue
            key, _, val = line.partition(":")
            cur[key.strip()] = val.strip()
    except OSError:
        pass
    return {"model": model, "logical_cpus": len(cpus), "physical_cores": len(cores) or len(cpus)}


def cpu_sample(shots: int, budget_s: float):
    """Reference C/OpenMP backend (oracle/_ref) on a bounded sample: nt truncated (runs in its own process)."""
    from oracle import driver

    from deepgpr_b200.synthetic import fwi_2d

    kind = "reference" if driver.available("ref") else "port"
    lib = "ref" if kind == "reference" else "oracle"

    def run(nt):
        acq = fwi_2d(seed=1002, nt=nt, nshot=shots)
        p = driver.Problem(eps_r=acq.eps_r, sigma=acq.sigma, source_amplitudes=acq.wavelet,
                           source_location=acq.sources, receiver_location=acq.receivers, dx=acq.dx, dt=acq.dt,
                           pml=10, order=4, mode=2)
        out = driver.run(p, lib)
        return out["t_forward"] + out["t_backward"], acq

    t, acq = run(2)
    nt = max(2, min(200, int(2 * budget_s / max(t, 1e-3))))
    t, acq = run(nt)
    nx, ny = acq.eps_r.shape
    units = 2 * (nx + 20) * (ny + 20) * nt * shots
    return {"value": units / t, "unit": UNIT, "kind": kind, "nt": nt, "seconds": t}


def cpu_baseline(shots: int, budget_s: float = 15.0):
    """The reference CPU backend timed on this host's physical cores (OMP_PROC_BIND=close), in a subprocess
    so that the OpenMP runtime starts with that binding."""
    info = host_cpu()
    threads = info["physical_cores"]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
    cmd = [sys.executable, str(Path(__file__).resolve()), "--cpu-sample", "--shots", str(shots),
           "--cpu-budget", str(budget_s)]
    proc = subprocess.run(cmd, env=env, capture_output=True, text=True)
    try:
        r = json.loads(proc.stdout.strip().splitlines()[-1])
    except (IndexError, json.JSONDecodeError):
        return {"error": (proc.stderr or proc.stdout)[-500:]}
    return {"value": r["value"], "unit": UNIT, "cores": threads, "kind": r["kind"],
            "cpu_model": info["model"], "logical_cpus": info["logical_cpus"],
            "sample": f"same workload with nt truncated to {r['nt']} steps, {shots} shots; native forward + "
                      f"backward time {r['seconds']:.1f} s (host preprocessing excluded); OMP_NUM_THREADS="
                      f"{threads} (physical cores), OMP_PROC_BIND=close"}


def reference(args, rank, world):
    if rank != 0:
        return
    samples = []
    cpu = None
    for i in range(args.warmup + args.steps):
        c = cpu_baseline(args.shots, budget_s=8.0)
        if i >= args.warmup:
            samples.append(c["value"])
            cpu = c
    value = statistics.median(samples)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered model + random field)", "impl": "reference",
        "config": {"workload": "2D multi-shot FWI gradient (forward + adjoint)", "grid": [400, 800, 1],
                   "shots": args.shots, "nt": args.nt, "fdtd_order": 4, "mode": 2,
                   "sample": "nt truncated per step (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cpu["cores"], "kind": cpu["kind"],
                         "cpu_model": cpu.get("cpu_model"), "sample": cpu["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.cpu_sample:
            print(json.dumps(cpu_sample(args.shots, args.cpu_budget)), flush=True)
        elif args.impl == "reference":
            reference(args, rank, world)
        elif args.config3:
            if rank == 0:
                print(json.dumps(config3_measure(torch.device("cuda", local), nt=args.config3_nt)), flush=True)
        elif args.only_serving:
            if rank == 0:
                print(json.dumps(serving_measure(torch.device("cuda", local), n=args.serving_requests,
                                                 history=args.serving_history)), flush=True)
        elif args.only_3d:
            if rank == 0:
                shape = tuple(int(v) for v in args.shape_3d.split(","))
                print(json.dumps(north_star_3d(torch.device("cuda", local), nt=args.nt_3d, shape=shape, pml=args.pml_3d)),
                      flush=True)
        else:
            ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
