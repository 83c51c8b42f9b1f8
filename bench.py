#!/usr/bin/env python
"""Benchmark: tracks/s of batched track propagation through the toy detector.

Workload (one "step" = one propagation of the whole batch):
  toy barrel + endcap detector from the reference's toy generator (4 barrel
  layers, 7 endcap discs per side, 0.15 mm Si modules, beampipe), homogeneous
  2 T field along z, 1 M muons per GPU from a Gaussian vertex spread
  (sigma 0.1, 0.1, 50 mm), eta uniform in [-4, 4], phi uniform, pT
  log-uniform in [1, 100] GeV; fp32 RKN4 with covariance transport, material
  interaction, path-limit aborter, 3x3 grid search window, bound parameters
  and covariance recorded at every sensitive / material surface.
  Data: synthetic, seeded.

Lines printed by rank 0 (one JSON line):
  value   tracks/s over all GPUs, inputs resident in HBM (device API);
  e2e     the same through dprop_propagate_host: host inputs copied in and
          all records copied out inside the timed region;
  roofline  FP32 issue bound of the propagation kernel (algorithmic FLOPs
          from device event counters x frozen per-event constants, see
          detray_b200/flops.py);
  cpu_baseline  the reference's own CPU propagator (fp32) on the host cores.

--impl reference times the reference CPU implementation only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "tracks/s (toy det., RK4+cov. transport) on 1 B200 vs host CPU; adjoint/fwd cost"
UNIT = "tracks/s"
WORKLOAD = "toy_4brl_7edc_const2T_1M_muons_pt1-100_eta4"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--tracks", type=int, default=1_000_000,
                   help="tracks per GPU per step")
    p.add_argument("--method", choices=["plain", "persistent", "auto"],
                   default="auto")
    p.add_argument("--no-sort", action="store_true",
                   help="propagate in input order instead of direction order")
    p.add_argument("--ctas", type=int, default=0,
                   choices=(0, 3, 4, 5, 8, 12, 16),
                   help="register budget (resident CTAs per SM) when "
                        "--method is not auto: 8, 12 or 16 for the plain "
                        "method, 3, 4 or 5 for the persistent method's step "
                        "phase; 0 = the method's default")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-adjoint", action="store_true",
                   help="skip the adjoint/forward cost measurement")
    p.add_argument("--adjoint-tracks", type=int, default=262_144)
    p.add_argument("--no-extras", action="store_true",
                   help="skip the direct-navigation and helix-scan rows")
    p.add_argument("--sweep", action="store_true",
                   help="measure the other benchmark configurations "
                        "(telescope; toy in the solenoid map; toy + wire "
                        "chamber in fp32 and fp64) instead of the headline "
                        "line")
    p.add_argument("--no-config5", action="store_true",
                   help="skip benchmark configuration 5 (toy + wire chamber, "
                        "16 M tracks each, fp32 and fp64; single GPU only)")
    p.add_argument("--no-config3", action="store_true",
                   help="skip the field-map configuration object")
    p.add_argument("--dry-run", action="store_true",
                   help="no GPU work: start the ranks (gloo without CUDA), "
                        "shard the batch and print the line with the shard "
                        "sizes (the CPU check of the multi-GPU launcher)")
    p.add_argument("--seed", type=int, default=20241203)
    return p.parse_args()


def spawn_ranks(args) -> int | None:
    """--gpus N > 1 outside a torchrun launch: start N ranks (one process per
    GPU) through torch.distributed.run on this node and return their exit
    code; inside a launch, check that the world size is N."""
    world = os.environ.get("WORLD_SIZE")
    if world is not None:
        if int(world) != args.gpus:
            raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE "
                             f"{world}")
        return None
    if args.gpus <= 1:
        return None
    import socket
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
           f"--master-port={port}", str(Path(__file__).resolve()),
           *sys.argv[1:]]
    return subprocess.call(cmd)


def workload_config():
    from detray_b200 import abi
    # the reference CUDA benchmark settings (tests/benchmarks/cuda/
    # propagation.cpp:56-74): window 3x3, no scattering-noise tolerance
    return abi.make_config(max_records=32, search_window=(3, 3),
                           estimate_scattering_noise=0)


def make_tracks(n, seed):
    from detray_b200 import tracks
    return tracks.toy_tracks(n, seed=seed, pt_range=(1.0, 100.0),
                             eta_range=(-4.0, 4.0),
                             vertex_sigma=(0.1, 0.1, 50.0))


# ---------------------------------------------------- adjoint workload
ADJOINT_WORKLOAD = ("toy_4brl_7edc_solenoid_map_262k_muons_pt0.5-50_"
                    "residual_loss_vs_aligned_targets")


def adjoint_cost(args, dev, stream, world=1, rank=0, steps=10, warmup=3):
    """Adjoint / forward time ratio on the alignment workload: toy detector
    in the solenoid field map, muons with pT uniform in [0.5, 50] GeV; targets
    are the local positions recorded by a propagation of perturbed tracks
    (position +- 10 um, angles +- 0.1 mrad, q/p +- 0.1 %) through the
    detector with every sensitive module shifted by N(0, 10 um) per axis
    (seed 12345); loss = sum over matching sensitive records of the squared
    local residuals.  One adjoint step = adjoint-mode propagation, the
    residual and its gradient, and the reverse sweep (gradients for the
    initial free parameters and 6 alignment values per surface); one
    forward step = the plain propagation of the same tracks.  Each side is
    timed at its best register budget.  With several GPUs every rank runs
    its own tracks and the adjoint step ends with the all-reduce of the
    alignment gradient and the loss over NCCL; times are the max over
    ranks."""
    import torch

    from detray_b200 import (adjoint, alignment, fields, geometry, propagator,
                             sharding)
    from detray_b200 import tracks as tracks_mod

    n = args.adjoint_tracks
    tables = geometry.load_geometry("toy_4brl_7edc")
    rng = np.random.default_rng(12345)
    sens = np.nonzero(tables["surfaces"]["kind"] == 1)[0]
    shifts = {int(s): np.concatenate([rng.normal(0.0, 0.010, 3), np.zeros(3)])
              for s in sens}
    det0 = propagator.Detector(tables, dev.index)
    det1 = propagator.Detector(alignment.apply_alignment(tables, shifts),
                               dev.index)
    field = propagator.Field.grid(fields.solenoid_map(), dev.index)
    cfg = workload_config()
    # the adjoint differentiates the field map too: its transport Jacobian
    # carries the field's gradient (use_field_gradient); the forward it is
    # compared with is the normal propagation without it
    cfg_adj = workload_config()
    cfg_adj.use_field_gradient = 1
    trk0 = tracks_mod.toy_tracks(n, seed=args.seed + 4 + 1000 * rank,
                                 pt_range=(0.5, 50.0),
                                 eta_range=(-4.0, 4.0), pt_log_uniform=False)
    trk1 = trk0.copy()
    trk1[0:3] += rng.normal(0.0, 0.010, (3, n))
    phi = np.arctan2(trk0[5], trk0[4]) + rng.normal(0.0, 1e-4, n)
    th = np.arccos(np.clip(trk0[6], -1, 1)) + rng.normal(0.0, 1e-4, n)
    trk1[4:7] = np.stack([np.cos(phi) * np.sin(th), np.sin(phi) * np.sin(th),
                          np.cos(th)])
    trk1[7] *= 1.0 + rng.normal(0.0, 1e-3, n)
    t0 = torch.tensor(trk0, dtype=torch.float32, device=dev)
    t1 = torch.tensor(trk1, dtype=torch.float32, device=dev)
    tgt = propagator.propagate(cfg, det1, field, t1,
                               launch=propagator.make_launch(sort_tracks=1),
                               stream=stream)
    tgt_bound = tgt.tensors["rec_bound"][:2].clone()
    tgt_bc = tgt.tensors["rec_barcode"].clone()
    slot = torch.arange(cfg.max_records, device=dev)[:, None]
    tgt_ok = ((slot < tgt.tensors["n_records"].clamp(max=cfg.max_records)[None])
              & ((tgt.tensors["rec_flags"] & 1) != 0))
    sens_lut = torch.zeros(det0.n_surfaces, dtype=torch.bool, device=dev)
    sens_lut[torch.as_tensor(sens, device=dev)] = True

    def residual_grad(rec):
        t = rec.results.tensors
        bc = t["rec_barcode"]
        sf = (bc >> 27) & 0x1FFFFF
        m = adjoint.rec_mask(rec) & tgt_ok & (bc == tgt_bc)
        m &= sens_lut[sf.clamp(max=det0.n_surfaces - 1)]
        r = (t["rec_bound"][:2] - tgt_bound) * m[None]
        g = torch.zeros_like(t["rec_bound"])
        g[:2] = 2.0 * r
        return (r * r).sum(), g, m

    def time_it(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    res = propagator.alloc_device_results(n, cfg.max_records, dev)
    fwd_ms, adj_ms = {}, {}
    out = {}
    for ctas in (12, 16):
        lc = propagator.make_launch(sort_tracks=1, ctas_per_sm=ctas)
        fwd_ms[ctas] = time_it(lambda: propagator.propagate(
            cfg, det0, field, t0, results=res, launch=lc, stream=stream))

        def adj_step():
            rec = adjoint.propagate_adjoint(cfg_adj, det0, field, t0,
                                            launch=lc, stream=stream)
            loss, g, m = residual_grad(rec)
            gf, ga = adjoint.backward(cfg_adj, det0, rec, g, stream=stream)
            if world > 1:
                ga, loss = sharding.allreduce_alignment(ga, loss)
            out.update(loss=loss, gf=gf, ga=ga, m=m)

        adj_ms[ctas] = time_it(adj_step)
    fwd_ms = {k: max_over_ranks(v, world) for k, v in fwd_ms.items()}
    adj_ms = {k: max_over_ranks(v, world) for k, v in adj_ms.items()}
    best_f = min(fwd_ms.values())
    best_a = min(adj_ms.values())
    ga = out["ga"]
    # the alignment gradient of the loss should point along the true shifts
    g_sens = ga[torch.as_tensor(sens, device=dev), :3].cpu().numpy()
    true = np.stack([shifts[int(s)][:3] for s in sens])
    hit = np.abs(g_sens).sum(axis=1) > 0
    cos = float(-(g_sens[hit] * true[hit]).sum() /
                (np.linalg.norm(g_sens[hit]) * np.linalg.norm(true[hit]) + 1e-30))
    return {"workload": ADJOINT_WORKLOAD, "tracks_per_gpu": n,
            "n_gpus": world,
            "forward_ms": round(best_f, 3), "adjoint_ms": round(best_a, 3),
            "ratio": round(best_a / best_f, 3),
            "forward_ms_by_ctas": {k: round(v, 3) for k, v in fwd_ms.items()},
            "adjoint_ms_by_ctas": {k: round(v, 3) for k, v in adj_ms.items()},
            "loss": float(out["loss"]),
            "residual_records": int(out["m"].sum()),
            "surfaces_with_gradient": int(hit.sum()),
            "cos_grad_vs_true_shift": round(cos, 4),
            "adjoint_includes": "adjoint-mode propagation with the "
                                "field-gradient transport Jacobian + residual "
                                "+ reverse sweep (fp64 alignment atomics)",
            "forward": "normal propagation (no field gradient), plain "
                       "method"}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv",
                                                   delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        self.tmp.seek(0)
        rows = [ln.strip().split(", ") for ln in self.tmp.read().splitlines()
                if ln.strip()]
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                if int(r[0]) != self.gpu_index:
                    continue
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for name, val in zip(names, r[5:9]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if torch.cuda.is_available() and not args.dry_run:
            torch.cuda.set_device(local)
            dist.init_process_group(
                "nccl", timeout=datetime.timedelta(seconds=120),
                device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo",
                                    timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce_device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ----------------------------------------------------------- CPU baseline
def cpu_reference_rate(n_target_seconds: float, cfg, seed: int,
                       max_tracks: int, threads: int) -> dict:
    """Reference CPU propagator (fp32 build, OpenMP over tracks, dynamic
    schedule chunk 1 as in the reference benchmark) on a bounded sample."""
    from oracle import ref_oracle
    from detray_b200.units import T
    det = ref_oracle.build_toy(precision="f32")
    field = {"kind": "const", "b": (0.0, 0.0, 2.0 * T)}
    probe = make_tracks(20_000, seed + 7)
    ref_oracle.propagate(det, field, cfg, probe[:, :2000], n_threads=threads,
                         abort_reasons=False)  # warm-up
    t0 = time.perf_counter()
    ref_oracle.propagate(det, field, cfg, probe, n_threads=threads,
                         abort_reasons=False)
    rate = probe.shape[1] / (time.perf_counter() - t0)
    n = int(min(max_tracks, max(20_000, rate * n_target_seconds)))
    sample = make_tracks(n, seed + 11)
    t0 = time.perf_counter()
    ref_oracle.propagate(det, field, cfg, sample, n_threads=threads,
                         abort_reasons=False)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": threads,
            "kind": "reference",
            "sample": f"{n} tracks of the same workload (seed {seed + 11}), "
                      f"{dt:.1f} s wall, fp32 reference build, OpenMP "
                      f"dynamic,1 over tracks"}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ------------------------------------------------------------ our impl
def extra_rows(cfg, det, field, trk, res, stream, dev, steps=5, warmup=2,
               n_scan=16384, n_scan64=4096):
    """Throughput of the other propagation-path entry points on the same
    workload: the direct navigator following the records of the main run
    (the Kalman-filter fit step), and the helix truth scan with the
    navigation validation of a propagation trace (n_scan tracks, every
    surface of the detector per track)."""
    import torch

    from detray_b200 import abi, propagator
    from detray_b200.units import T
    n = trk.shape[1]

    def timed(fn, k, n_warm=warmup):
        for _ in range(n_warm):
            fn()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / k

    seq = res.tensors["rec_barcode"]
    lens = torch.clamp(res.tensors["n_records"], max=cfg.max_records)
    out = propagator.alloc_device_results(n, cfg.max_records, dev)
    ms_direct = timed(lambda: propagator.propagate_direct(
        cfg, det, field, seq, lens, 1, tracks=trk, results=out,
        stream=stream), steps)
    same = bool(torch.equal(out.tensors["n_records"], res.tensors["n_records"]))
    b = (0.0, 0.0, 2.0 * T)
    sub32 = trk[:, :n_scan].contiguous()
    sub64 = trk[:, :n_scan64].double().contiguous()
    ms_scan32 = timed(lambda: propagator.helix_scan(det, b, sub32, 1e-3,
                                                    stream=stream), 2, 1)
    # the fp64 scan is timed once, on fewer tracks, and is the truth of the
    # navigation validation
    truth = None

    def scan64():
        nonlocal truth
        truth = propagator.helix_scan(det, b, sub64, 1e-3, stream=stream)
    ms_scan64 = timed(scan64, 1, 0)
    vcfg = abi.make_config(max_records=64, search_window=(3, 3),
                           use_material_interactor=0,
                           estimate_scattering_noise=0, record_all_surfaces=1)
    trace = propagator.propagate(vcfg, det, field, sub32[:, :n_scan64],
                                 stream=stream)
    missed, extra = propagator.validate_navigation(truth, trace,
                                                   vcfg.max_records, 0.1,
                                                   stream=stream)
    torch.cuda.synchronize(dev)
    good = float(((missed == 0) & (extra == 0)).float().mean().item())
    return {
        "direct_navigation": {
            "value": n / (ms_direct / 1e3), "unit": UNIT,
            "ms_per_step": round(ms_direct, 3),
            "what": "dprop_propagate_direct forward along the records of the "
                    "main run (same tracks, same actor chain)",
            "same_record_counts": same},
        "helix_scan": {
            "fp64_tracks_per_s": n_scan64 / (ms_scan64 / 1e3),
            "fp32_tracks_per_s": n_scan / (ms_scan32 / 1e3),
            "ms_fp64": round(ms_scan64, 3), "ms_fp32": round(ms_scan32, 3),
            "tracks_fp32": n_scan, "tracks_fp64": n_scan64,
            "surfaces_per_track": int(det.n_surfaces),
            "navigation_validation_clean_fraction": round(good, 5),
            "what": "dprop_helix_scan (every surface per track) and "
                    "dprop_validate_navigation of a no-material trace"},
    }


def parity_sample(cfg, host_trk, res, k):
    """Parity of the timed run on its own workload: the first k tracks of
    the batch through the reference's fp64 CPU propagator (the oracle),
    against the records the timed GPU run wrote for the same tracks.
    Reports the fraction of tracks with the same status and surface sequence
    and the per-quantity errors (_errors_vs_oracle)."""
    from oracle import ref_oracle
    from detray_b200.units import T
    k = min(k, host_trk.shape[1])
    ref = ref_oracle.propagate(ref_oracle.build_toy(),
                               {"kind": "const", "b": (0.0, 0.0, 2.0 * T)},
                               cfg, np.ascontiguousarray(host_trk[:, :k]),
                               n_threads=host_threads())
    t = res.tensors
    got = {"status": t["status"][:k].cpu().numpy(),
           "n_records": t["n_records"][:k].cpu().numpy(),
           "rec_barcode": t["rec_barcode"][:, :k].cpu().numpy().view(np.uint64),
           "rec_flags": t["rec_flags"][:, :k].cpu().numpy(),
           "rec_bound": t["rec_bound"][:, :, :k].cpu().numpy(),
           "rec_cov": t["rec_cov"][:, :, :k].cpu().numpy()}
    out = _errors_vs_oracle(ref, got)
    out["same_status"] = float((ref["status"] == got["status"]).mean())
    out["oracle"] = "reference CPU propagator, fp64 build"
    return out


def launch_fields(lc):
    """The launch shape the autotuner chose, as printed in the line.  A warp
    always carries 32 tracks, one per lane, in both methods; yield_lanes is
    the persistent step phase's lower bound of live tracks per warp."""
    return {"method": {0: "plain", 1: "persistent"}.get(int(lc.method),
                                                        int(lc.method)),
            "block_size": int(lc.block_size) or 128,
            "ctas_per_sm": int(lc.ctas_per_sm),
            "sort_tracks": int(lc.sort_tracks),
            "tracks_per_warp": 32,
            "steps_per_round": int(lc.steps_per_round),
            "yield_lanes": int(lc.yield_lanes),
            "rounds": int(lc.rounds),
            "sort_interval": int(lc.sort_interval)}


def config3_row(args, dev, stream, world):
    """Benchmark configuration 3 on every rank: the toy detector in the
    solenoid field map, 4 M muons with pT log-uniform in 0.1-100 GeV, fp32
    with covariance transport and material: the plain one-track-per-thread
    kernel (sorted, 32 registers), the persistent round-based method with
    its defaults, and the autotuner's pick, each under a CUDA graph; times
    are the max over ranks."""
    import torch

    from detray_b200 import abi, fields, geometry, propagator, tracks
    n3 = 4_000_000
    fmap = fields.solenoid_map()
    det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"),
                              dev.index)
    field = propagator.Field.grid(fmap, dev.index)
    cfg = workload_config()
    trk = tracks.toy_tracks(n3, seed=args.seed + 3, pt_range=(0.1, 100.0))
    dt = torch.tensor(trk, dtype=torch.float32, device=dev)
    res = propagator.alloc_device_results(n3, cfg.max_records, dev)
    forms = {"plain": propagator.make_launch(method=abi.METHOD_PLAIN,
                                             sort_tracks=1, ctas_per_sm=16,
                                             use_graph=1),
             "persistent": propagator.make_launch(
                 method=abi.METHOD_PERSISTENT, sort_tracks=1, use_graph=1)}
    lc, tune = propagator.autotune(cfg, det, field, dt, use_graph=1,
                                   stream=stream)
    forms["autotuned"] = lc
    ms = {}
    for name, f in forms.items():
        ms[name] = max_over_ranks(_time_device(
            lambda f=f: propagator.propagate(cfg, det, field, dt, results=res,
                                             launch=f, stream=stream),
            dev, 5, 2), world)
    status = np.bincount(res.tensors["status"].cpu().numpy(), minlength=7)
    del res, dt
    torch.cuda.empty_cache()
    return {"workload": "toy_4brl_7edc_solenoid_map_4M_muons_pt0.1-100_eta4",
            "tracks_per_gpu": n3, "ms": {k: round(v, 3) for k, v in ms.items()},
            "tracks_per_s": {k: n3 * world / (v / 1e3) for k, v in ms.items()},
            "autotuned": launch_fields(lc),
            "autotune_ms": [round(t, 3) for t in tune],
            "track_status": status.tolist(),
            "persistent_vs_plain": round(ms["plain"] / ms["persistent"], 4)}


def run_ours(args):
    import torch

    from detray_b200 import abi, flops, geometry, propagator
    from detray_b200.units import T

    from detray_b200 import sharding
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfg = workload_config()
    det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"), local)
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T), local)
    # weak scaling: a global batch of args.tracks per GPU, split into
    # contiguous work-balanced shards (no collective in the forward pass)
    if world > 1:
        host_trk, shard_range = sharding.shard(
            make_tracks(args.tracks * world, args.seed), rank, world)
        host_trk = np.ascontiguousarray(host_trk)
    else:
        host_trk, shard_range = make_tracks(args.tracks, args.seed), None
    n = host_trk.shape[1]
    trk = torch.tensor(host_trk, dtype=torch.float32, device=dev)
    res = propagator.alloc_device_results(n, cfg.max_records, dev)
    stream = torch.cuda.current_stream(dev)
    tune_ms = None
    if args.method == "auto":
        # the project's autotuner picks kernel form, register budget and
        # sorting on this workload (outside the timed region)
        lc, tune_ms = propagator.autotune(cfg, det, field, trk, use_graph=1,
                                          stream=stream)
    else:
        method = {"plain": abi.METHOD_PLAIN,
                  "persistent": abi.METHOD_PERSISTENT}[args.method]
        ctas = args.ctas
        if (method == abi.METHOD_PLAIN) != (ctas in (0, 8, 12, 16)):
            raise SystemExit(f"bench.py: --ctas {ctas} does not apply to "
                             f"--method {args.method}")
        lc = propagator.make_launch(method=method,
                                    sort_tracks=int(not args.no_sort),
                                    ctas_per_sm=ctas, use_graph=1)
    method = lc.method

    def step():
        propagator.propagate(cfg, det, field, trk, results=res, launch=lc,
                             stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    clk = clocks.stop()
    ms_local = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms_local, world)
    total_tracks = int(sum_over_ranks(float(n), world))
    value = total_tracks / (ms / 1e3)

    # algorithmic work of one launch from the device event counters
    t = res.tensors
    fl = flops.algorithmic_flops(t["n_trials"].cpu().numpy(),
                                 t["n_steps"].cpu().numpy(),
                                 t["n_intersections"].cpu().numpy(),
                                 t["n_transports"].cpu().numpy(),
                                 t["n_material"].cpu().numpy())
    status = np.bincount(t["status"].cpu().numpy(), minlength=7)
    mean_steps = float(t["n_steps"].float().mean().item())
    achieved = fl / (ms_local / 1e3) / 1e12
    peak_mhz = 1965.0
    try:
        peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text())
        peak_mhz = float(peaks.get("sm_max_mhz", peak_mhz))
    except (OSError, ValueError):
        pass
    peak = flops.nominal_fp32_tflops(sm_count, peak_mhz)
    method_name = {abi.METHOD_PLAIN: "plain",
                   abi.METHOD_PERSISTENT: "persistent"}[method]
    # DRAM bytes per track of one propagation with this method, from an ncu
    # capture of every kernel of a smaller batch (scaled by tracks)
    traffic, traffic_src = None, None
    prof = REPO / "profiles" / "propagate_toy_traffic.json"
    if prof.exists():
        try:
            entry = json.loads(prof.read_text())[method_name]
            traffic = entry["dram_bytes_per_track"] * n
            traffic_src = entry["source"]
        except (OSError, ValueError, KeyError):
            traffic = None
    rounds = int(lc.rounds) or 64
    # our kernels per propagation (the radix sort itself is CUB's)
    if method == abi.METHOD_PERSISTENT:
        per_step = (int(lc.sort_tracks) + 1 + 2 * (rounds + 1) + 2 * rounds
                    + 1)
        kernels = ("direction key, init, per round the queue builder (2), "
                   "step phase and navigation phase, then the queue builder "
                   "and the tail")
    else:
        per_step = 1 + int(lc.sort_tracks)
        kernels = "direction key, propagate_plain_kernel"
    roofline = {"bound": "fp32", "achieved": round(achieved, 4),
                "peak": round(peak, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 5), "traffic": traffic,
                "traffic_source": traffic_src,
                "peak_source": f"nominal FP32 ({sm_count} SMs x 128 lanes x "
                               f"2 x {peak_mhz:.0f} MHz; no measured FP32 "
                               "peak on this pool)",
                "scope": "the whole propagation call (all its kernels), "
                         "CUDA events on its stream",
                "flops_per_launch": fl, "kernel_ms": round(ms_local, 4)}

    # ---- end to end through the host-buffer API
    e2e = None
    if not args.no_e2e:
        link = link_bandwidth(dev)
        pinned_trk = torch.tensor(host_trk, dtype=torch.float64).pin_memory()
        host_in = pinned_trk.numpy()
        out = propagator.alloc_host_results(n, cfg.max_records, pinned=True,
                                            jagged=True)
        for _ in range(max(1, args.warmup)):
            propagator.propagate_host(cfg, det, field, host_in, launch=lc,
                                      out=out)
        barrier(world)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        k_e2e = max(1, min(args.steps, 5))
        for _ in range(k_e2e):
            propagator.propagate_host(cfg, det, field, host_in, launch=lc,
                                      out=out)
        e1.record()
        torch.cuda.synchronize(dev)
        wall = (time.perf_counter() - t0) / k_e2e
        ms_e2e = max(e0.elapsed_time(e1) / k_e2e, wall * 1e3)
        ms_e2e = max_over_ranks(ms_e2e, world)
        h2d = 8 * n * 8
        n_rec = int(out[0]["rec_offsets"][n])
        rec = n_rec * (8 + 6 * 4 + 21 * 4 + 4 + 1)
        d2h = n * (1 + 7 * 4 + 8 * 4) + (n + 1) * 4 + rec
        # the copies alone at the measured link bandwidth: the bound the
        # e2e time approaches when the pipeline hides the propagation
        copy_ms = (h2d / link["h2d_gbs"] + d2h / link["d2h_gbs"]) / 1e6
        link["copy_bound_ms"] = round(copy_ms, 3)
        link["bound_ms"] = round(max(copy_ms, ms), 3)
        link["frac"] = round(max(copy_ms, ms) / ms_e2e, 4)
        e2e = {"value": total_tracks / (ms_e2e / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": round(ms_e2e, 3), "steps": k_e2e,
               "records_per_step": n_rec, "link": link,
               "api": "dprop_propagate_host, jagged records, chunked "
                      "pipeline (4 chunks on prioritized streams, records "
                      "drained on a copy stream), pinned host buffers"}

    adj = None
    if not args.no_adjoint:
        adj = adjoint_cost(args, dev, stream, world, rank)

    extras = None
    if not args.no_extras:
        extras = extra_rows(cfg, det, field, trk, res, stream, dev)

    cfg3 = None
    if not args.no_config3:
        cfg3 = config3_row(args, dev, stream, world)
    cfg5 = None
    if not args.no_config5 and world == 1:
        propagator.release_cache()
        cfg5 = config5_row(args, dev,
                           oracle_errors=rank == 0 and not args.no_cpu_baseline)

    cpu, errors = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_rate(15.0, cfg, args.seed, 2_000_000,
                                     host_threads())
            errors = parity_sample(cfg, host_trk, res, 100_000)
        except (FileNotFoundError, OSError) as exc:
            cpu = {"value": None, "unit": UNIT, "cores": host_threads(),
                   "kind": "reference", "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded toy-detector muon sample)",
            "config": {"workload": WORKLOAD, "tracks_per_gpu": n,
                       "global_batch": total_tracks,
                       "method": {abi.METHOD_PLAIN: "plain",
                                  abi.METHOD_PERSISTENT: "persistent"}[method],
                       **{k: v for k, v in launch_fields(lc).items()
                          if k != "method"},
                       "cuda_graph": int(lc.use_graph),
                       "shard": list(shard_range) if shard_range else None,
                       "autotune_ms": ([round(t, 3) for t in tune_ms]
                                       if tune_ms else None),
                       "parallelism": f"tracks sharded over {world} GPU(s)",
                       "l2": "per step ~1.5 GB of records written (> 126 MB "
                             "L2): inputs are re-read from HBM"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
            "errors_vs_fp64_oracle": errors,
            "config3": cfg3,
            "config5": cfg5,
            "adjoint": adj,
            "other_entry_points": extras,
            "gpu_launches": args.steps * per_step,
            "gpu_launches_per_step": per_step,
            "gpu_kernels": kernels,
            "clocks": clk,
            "track_status": status.tolist(),
            "mean_steps_per_track": round(mean_steps, 2),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ------------------------------------------------------ reference arm
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref_oracle
    from detray_b200.units import T
    if not ref_oracle.available("f32"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libdetray_ref_f32.so not "
                                         "built (needs the reference checkout)"}))
        return
    cfg = workload_config()
    threads = host_threads()
    det = ref_oracle.build_toy(precision="f32")
    field = {"kind": "const", "b": (0.0, 0.0, 2.0 * T)}
    # size each step for ~2 s of wall time on this host
    probe = make_tracks(20_000, args.seed + 3)
    t0 = time.perf_counter()
    ref_oracle.propagate(det, field, cfg, probe, n_threads=threads,
                         abort_reasons=False)
    rate = probe.shape[1] / (time.perf_counter() - t0)
    n = int(min(args.tracks, max(10_000, rate * 2.0)))
    sample = make_tracks(n, args.seed)
    for _ in range(args.warmup):
        ref_oracle.propagate(det, field, cfg, sample, n_threads=threads,
                             abort_reasons=False)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref_oracle.propagate(det, field, cfg, sample, n_threads=threads,
                             abort_reasons=False)
    dt = (time.perf_counter() - t0) / args.steps
    value = n / dt
    gpu = reference_gpu_row(args, cfg)
    gpu3 = reference_gpu_config3(args, cfg) if not args.no_config3 else None
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded toy-detector muon sample)",
        "config": {"workload": WORKLOAD, "tracks_per_step": n,
                   "parallelism": f"OpenMP over tracks, {threads} threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                         "kind": "reference",
                         "sample": f"{n} tracks per step of the same workload"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_gpu": gpu,
        "reference_gpu_config3": gpu3,
    }
    print(json.dumps(line), flush=True)


def reference_gpu_row(args, cfg):
    """The reference's own CUDA propagation kernel (its benchmark's
    propagator_benchmark_kernel with the default actor chain, rebuilt for
    sm_100a from its headers) timed with CUDA events on the same workload
    and tracks as our arm, device-resident inputs: the GPU "plain form"."""
    from oracle import ref_oracle
    from detray_b200.units import T
    try:
        import torch
        if not (ref_oracle.gpu_available() and torch.cuda.is_available()):
            return None
        trk = make_tracks(args.tracks, args.seed)
        # the reference benchmark's input order: by |pi/2 - theta|
        # (tests/benchmarks/include/detray/benchmarks/benchmark_utils.hpp)
        theta = np.arccos(np.clip(trk[6], -1.0, 1.0))
        trk = trk[:, np.argsort(np.abs(0.5 * np.pi - theta), kind="stable")]
        r = ref_oracle.gpu_toy_bench(cfg, 2.0 * T, trk,
                                     warmup=args.warmup, steps=args.steps)
    except (RuntimeError, OSError) as exc:
        return {"unavailable": str(exc)}
    return {"value": args.tracks / (r["ms_per_step"] / 1e3), "unit": UNIT,
            "ms_per_step": round(r["ms_per_step"], 3),
            "tracks": args.tracks, "n_exited": r["n_exited"],
            "kernel": "reference propagator_benchmark_kernel (default "
                      "actor chain: parameter_updater with material "
                      "interactor), 256 threads, sm_100a, tracks ordered by "
                      "|pi/2 - theta| as in the reference benchmark, no "
                      "records written"}


def reference_gpu_config3(args, cfg):
    """The reference's device propagation in benchmark configuration 3: its
    tutorial kernel's actor chain (path-limit aborter, parameter updater
    with the material interactor, tutorials/src/device/cuda/
    propagation_kernel.cu), one thread per track, in the solenoid field map,
    on the same 4 M tracks as our config3 object (ordered by |pi/2 - theta|
    as the reference benchmark orders its input)."""
    from oracle import ref_oracle
    try:
        import torch
        if not (ref_oracle.gpu_available() and torch.cuda.is_available()):
            return None
        from detray_b200 import fields, tracks
        n3 = 4_000_000
        trk = tracks.toy_tracks(n3, seed=args.seed + 3, pt_range=(0.1, 100.0))
        theta = np.arccos(np.clip(trk[6], -1.0, 1.0))
        trk = trk[:, np.argsort(np.abs(0.5 * np.pi - theta), kind="stable")]
        r = ref_oracle.gpu_toy_map_bench(cfg, fields.solenoid_map(), trk,
                                         warmup=1, steps=3)
    except (RuntimeError, OSError) as exc:
        return {"unavailable": str(exc)}
    return {"value": n3 / (r["ms_per_step"] / 1e3), "unit": UNIT,
            "ms_per_step": round(r["ms_per_step"], 3), "tracks": n3,
            "n_exited": r["n_exited"],
            "workload": "toy_4brl_7edc_solenoid_map_4M_muons_pt0.1-100_eta4",
            "kernel": "reference tutorial propagation kernel (path-limit "
                      "aborter, parameter updater with material "
                      "interactor), 64 threads per block, sm_100a, no "
                      "records written"}


def link_bandwidth(dev, nbytes=1 << 29):
    """Host <-> device copy bandwidth between pinned host memory and the
    device, GB/s per direction (one cudaMemcpyAsync of 512 MiB, best of 5):
    the denominator of the end-to-end leg, whose copies cross this link."""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    out = {}
    for name, dst, src in (("h2d_gbs", d, h), ("d2h_gbs", h, d)):
        best = None
        for _ in range(6):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            dst.copy_(src, non_blocking=True)
            e1.record()
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name] = round(nbytes / (best / 1e3) / 1e9, 2)
    del h, d
    return out


# ------------------------------------------------ other configurations
def _time_device(fn, dev, steps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / steps


def _errors_vs_oracle(ref, got):
    """Per-surface errors of a device run against the fp64 oracle over the
    tracks whose surface sequences agree: max and 99th percentile of the
    absolute differences of the bound parameters, and the covariance
    difference relative to sqrt(C_ii C_jj)."""
    import numpy as np
    n = ref["status"].shape[0]
    cap = ref["rec_barcode"].shape[0]
    nr = np.minimum(ref["n_records"], cap)
    ng = np.minimum(got["n_records"], cap)
    same = nr == ng
    k = np.arange(cap)[:, None]
    valid = (k < nr[None, :]) & same[None, :]
    valid &= ref["rec_barcode"] == got["rec_barcode"].astype(np.uint64)
    seq_ok = np.all(valid | (k >= nr[None, :]), axis=0) & same
    m = valid & seq_ok[None, :] & ((ref["rec_flags"] & 1) != 0)
    out = {"tracks": int(n), "same_sequence": float(seq_ok.mean())}
    names = ["loc0", "loc1", "phi", "theta", "qop", "time"]
    for i, nm in enumerate(names):
        d = np.abs(ref["rec_bound"][i][m] - got["rec_bound"][i][m])
        out[nm] = {"max": float(d.max()) if d.size else 0.0,
                   "p99": float(np.percentile(d, 99)) if d.size else 0.0}
    diag = [0, 6, 11, 15, 18, 20]
    worst = 0.0
    c = 0
    for i in range(6):
        for j in range(i, 6):
            ci = np.abs(ref["rec_cov"][diag[i]][m])
            cj = np.abs(ref["rec_cov"][diag[j]][m])
            den = np.sqrt(ci * cj)
            ok = den > 0
            d = np.abs(ref["rec_cov"][c][m] - got["rec_cov"][c][m])[ok] / den[ok]
            if d.size:
                worst = max(worst, float(d.max()))
            c += 1
    out["cov_rel_max"] = worst
    return out


def config5_row(args, dev, oracle_errors):
    """Benchmark configuration 5: the toy detector and the wire chamber (10
    layers of square drift cells) in the solenoid field map, 16 M muons per
    detector (eta in [-4, 4], pT log-uniform in 0.1-100 GeV, the same
    tracks for both detectors and both builds) in batches of 2 M held in
    one device buffer: the fp32 build (the autotuner's launch form for the
    detector, CUDA graph) and the fp64 build (dprop_launch.precision = 8),
    tracks/s
    and the FP32 / FP64 roofline fraction of each; with oracle_errors the
    per-surface errors against the fp64 oracle on a 3 000-track sample."""
    import numpy as np
    import torch

    from detray_b200 import abi, fields, flops, geometry, propagator, tracks
    sm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak32 = flops.nominal_fp32_tflops(sm, 1965.0)
    field = propagator.Field.grid(fields.solenoid_map(), dev.index)
    cfg = abi.make_config(max_records=48, search_window=(3, 3),
                          estimate_scattering_noise=0)
    n5 = 16_000_000
    batch = 2_000_000
    batches = [tracks.toy_tracks(batch, seed=args.seed + 50 + b0,
                                 pt_range=(0.1, 100.0))
               for b0 in range(0, n5, batch)]
    out = {}
    for name in ("toy_4brl_7edc", "wire_chamber_10l_cells"):
        det = propagator.Detector(geometry.load_geometry(name), dev.index)
        for prec, dtype in ((4, torch.float32), (8, torch.float64)):
            dt = torch.empty((8, batch), dtype=dtype, device=dev)
            if prec == 4:
                # the autotuner's pick for this detector (on the first batch)
                dt.copy_(torch.from_numpy(batches[0]))
                lc, _ = propagator.autotune(cfg, det, field, dt, use_graph=1)
                propagator.release_cache()
            res = propagator.alloc_device_results(batch, cfg.max_records, dev,
                                                  dtype=dtype)
            if prec == 8:
                # fp64: the faster of the plain kernel and the round-based
                # method (2 or 3 CTAs/SM) on the first batch
                dt.copy_(torch.from_numpy(batches[0]))
                best = None
                for kw in (dict(), dict(method=abi.METHOD_PERSISTENT),
                           dict(method=abi.METHOD_PERSISTENT, ctas_per_sm=3)):
                    cand = propagator.make_launch(sort_tracks=1, precision=8,
                                                  **kw)
                    t_c = _time_device(lambda cand=cand: propagator.propagate(
                        cfg, det, field, dt, results=res, launch=cand), dev, 1,
                        1)
                    if best is None or t_c < best[0]:
                        best = (t_c, cand)
                lc = best[1]
            total_ms = 0.0
            fl = 0.0
            status = np.zeros(8, dtype=np.int64)
            for bi, trk in enumerate(batches):
                dt.copy_(torch.from_numpy(trk))
                total_ms += _time_device(lambda: propagator.propagate(
                    cfg, det, field, dt, results=res, launch=lc), dev, 1,
                    1 if bi == 0 else 0)
                t = res.tensors
                fl += flops.algorithmic_flops(
                    t["n_trials"].cpu().numpy(), t["n_steps"].cpu().numpy(),
                    t["n_intersections"].cpu().numpy(),
                    t["n_transports"].cpu().numpy(),
                    t["n_material"].cpu().numpy())
                status += np.bincount(t["status"].cpu().numpy(),
                                      minlength=8)[:8]
            peak = peak32 if prec == 4 else peak32 / 2.0
            key = f"{name}_fp{8 * prec}"
            out[key] = {
                "tracks": n5, "ms": round(total_ms, 2),
                "tracks_per_s": n5 / (total_ms / 1e3),
                "launch": (dict(launch_fields(lc), cuda_graph=1,
                                how="autotuned on the first batch")
                           if prec == 4 else
                           dict(launch_fields(lc), precision=8,
                                how="fastest of plain / persistent 2 / 3 "
                                    "CTAs per SM on the first batch")),
                "achieved_tflops": fl / (total_ms / 1e3) / 1e12,
                "roofline_frac": fl / (total_ms / 1e3) / 1e12 / peak,
                "peak_source": "nominal FP32" if prec == 4 else
                               "nominal FP64 = FP32 / 2",
                "status_counts": {
                    nm: int(status[c]) for nm, c in (
                        ("exited", abi.TRK_EXITED),
                        ("path_limit", abi.TRK_PATH_LIMIT),
                        ("stalled", abi.TRK_STALLED),
                        ("no_surface", abi.TRK_NO_SURFACE),
                        ("max_iterations", abi.TRK_MAX_ITER))}}
            del res, dt
            torch.cuda.empty_cache()
            if oracle_errors:
                from oracle import ref_oracle
                ref_det = (ref_oracle.build_toy() if name == "toy_4brl_7edc"
                           else ref_oracle.build_wire_chamber(
                               square_cells=True))
                sample = tracks.toy_tracks(3000, seed=args.seed + 99,
                                           pt_range=(0.1, 100.0))
                ref = ref_oracle.propagate(ref_det, field.spec, cfg, sample)
                got = propagator.propagate(
                    cfg, det, field,
                    torch.tensor(sample, dtype=dtype, device=dev), launch=lc)
                got = {k: v.cpu().numpy() for k, v in got.tensors.items()}
                got["rec_barcode"] = got["rec_barcode"].view(np.uint64)
                out[key]["errors_vs_fp64_oracle"] = _errors_vs_oracle(ref, got)
    return {"config": 5, "workload": "toy_4brl_7edc + wire_chamber_10l_cells, "
            "solenoid map, 16M muons per detector eta -4..4 pT 0.1-100",
            "results": out}


def run_sweep(args):
    """The other benchmark configurations, one JSON object per
    configuration (the headline line is the default run):
    1. telescope, 10 000 muons at pT 10 GeV within 10 deg of +x, 2 T, fp32:
       GPU against the reference CPU propagator on the same tracks;
    3. toy detector in the solenoid field map, 4 M muons pT 0.1-100 GeV:
       plain and persistent kernels and the autotuned launch under a graph;
    5. toy detector and wire chamber in the solenoid map, 16 M muons
       (eta in [-4, 4], pT 0.1-100 GeV) in batches: fp32 and fp64 builds,
       tracks/s and the per-surface errors against the fp64 oracle on a
       sample."""
    import numpy as np
    import torch

    from detray_b200 import abi, fields, flops, geometry, propagator, tracks
    from detray_b200.units import T
    from oracle import ref_oracle
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    sm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak32 = flops.nominal_fp32_tflops(sm, 1965.0)
    rows = []
    clocks = ClockSampler(0)
    clocks.start()

    def host(res):
        out = {k: v.cpu().numpy() for k, v in res.tensors.items()}
        out["rec_barcode"] = out["rec_barcode"].view(np.uint64)
        return out

    # ---- config 1: telescope
    det = propagator.Detector(geometry.load_geometry("telescope_10x1m_300um"))
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    cfg = abi.make_config(max_records=16)
    trk = tracks.telescope_tracks(10_000, seed=args.seed)
    dt = torch.tensor(trk, dtype=torch.float32, device=dev)
    res = propagator.alloc_device_results(dt.shape[1], cfg.max_records, dev)
    lc = propagator.make_launch(sort_tracks=1, use_graph=1)
    ms = _time_device(lambda: propagator.propagate(
        cfg, det, field, dt, results=res, launch=lc), dev, 50, 5)
    cpu = None
    if ref_oracle.available("f32"):
        rdet = ref_oracle.build_telescope(precision="f32")
        ref_oracle.propagate(rdet, field.spec, cfg, trk[:, :1000],
                             n_threads=host_threads(), abort_reasons=False)
        t0 = time.perf_counter()
        for _ in range(5):
            ref_oracle.propagate(rdet, field.spec, cfg, trk,
                                 n_threads=host_threads(),
                                 abort_reasons=False)
        cpu = trk.shape[1] * 5 / (time.perf_counter() - t0)
    rows.append({"config": 1, "workload": "telescope_10x1m_300um_const2T_"
                 "10k_muons_pt10_cone10", "gpu_tracks_per_s":
                 trk.shape[1] / (ms / 1e3), "gpu_ms": round(ms, 4),
                 "cpu_reference_tracks_per_s": cpu,
                 "cpu_threads": host_threads(), "dtype": "f32"})

    # ---- config 3: toy in the solenoid map, plain vs persistent vs tuned
    fmap = fields.solenoid_map()
    det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"))
    field = propagator.Field.grid(fmap, 0)
    cfg = abi.make_config(max_records=32, search_window=(3, 3),
                          estimate_scattering_noise=0)
    n3 = 4_000_000
    trk = tracks.toy_tracks(n3, seed=args.seed + 3, pt_range=(0.1, 100.0))
    dt = torch.tensor(trk, dtype=torch.float32, device=dev)
    res = propagator.alloc_device_results(n3, cfg.max_records, dev)
    forms = {}
    for name, lc in (("plain_unsorted", propagator.make_launch(
                         method=abi.METHOD_PLAIN, sort_tracks=0)),
                     ("persistent_sorted", propagator.make_launch(
                         method=abi.METHOD_PERSISTENT, sort_tracks=1))):
        forms[name] = _time_device(lambda lc=lc: propagator.propagate(
            cfg, det, field, dt, results=res, launch=lc), dev, 3, 1)
    lc, _ = propagator.autotune(cfg, det, field, dt, use_graph=1)
    forms["autotuned_graph"] = _time_device(lambda: propagator.propagate(
        cfg, det, field, dt, results=res, launch=lc), dev, 3, 1)
    rows.append({"config": 3, "workload": "toy_4brl_7edc_solenoid_map_4M_"
                 "muons_pt0.1-100", "ms": {k: round(v, 3)
                                            for k, v in forms.items()},
                 "tracks_per_s": {k: n3 / (v / 1e3)
                                  for k, v in forms.items()},
                 "autotuned": launch_fields(lc),
                 "dtype": "f32"})
    del res, dt

    # ---- config 5: toy + wire chamber, fp32 and fp64, 16 M tracks each
    propagator.release_cache()
    rows.append(config5_row(args, dev, oracle_errors=True))
    clk = clocks.stop()
    print(json.dumps({"sweep": rows, "clocks": clk}), flush=True)


def run_dry(args):
    """The multi-GPU launcher without GPU work: every rank takes its
    work-balanced shard of the global batch; rank 0 prints the line."""
    from detray_b200 import sharding
    world, rank, _ = dist_setup(args)
    host_all = make_tracks(args.tracks * world, args.seed)
    mine, (lo, hi) = sharding.shard(host_all, rank, world)
    total = sum_over_ranks(float(mine.shape[1]), world)
    biggest = max_over_ranks(float(mine.shape[1]), world)
    if rank == 0:
        print(json.dumps({"dry_run": True, "n_gpus": world, "metric": METRIC,
                          "value": None, "unit": UNIT,
                          "global_batch": int(total),
                          "largest_shard": int(biggest),
                          "rank0_range": [lo, hi]}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse_args()
    rc = spawn_ranks(args)
    if rc is not None:
        sys.exit(rc)
    if args.dry_run:
        run_dry(args)
        return
    if args.sweep:
        run_sweep(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
