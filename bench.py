"""Benchmark: slice-propagations/s (forward + adjoint) of the batched MSET
hot path on the mid-size synthetic tilt series.

Workload ("mid"): 128^3 FP32 volume at 0.3 A/voxel from a seeded fcc
Cu/Au-like lattice of Gaussian atoms, 128^2 complex64 window, 32x32 scan at
3 px, 21 tilts over +-60 deg, 64 slices of 2 voxels: 21,504 positions and
1,376,256 slice-propagations per step.  One step = one batched pass: forward
(transmission, 64 x [FFT, propagator, IFFT]), far field, residual, loss and the
adjoint with V / probe / scan-position gradients of every position of every
tilt, in one persistent launch.  Inputs (measured amplitudes 1.4 GB) exceed
L2, so no flush is needed between steps.

Beside the headline (rank 0, mid workload only; --no-* skips them): the full
iteration as one CUDA graph, the plain form of the pass (one launch per tilt,
one CTA per position, no graph, no checkpointing), the sequential forms with
reference semantics (this library's mset_run and the reference's own CUDA
module), the uneven-size 6-series group pass with the autotuner, the
256^2-window cluster kernel on 3 tilts of the large geometry, and the
single-precision CPU port on a sample.

Under torchrun (--gpus N > 1) the 21 tilts are split over the ranks
(mset_b200.distributed.tilt_shard): one specimen, each rank its own tilts,
the whole workload's slice-propagations over the slowest rank's time (strong
scaling); the iteration adds the one all-reduce of the FP64 lab-frame
gradient per iteration.

One JSON line on stdout (rank 0).  --impl reference times the reference's CPU
path (MATLAB code in single precision, not available here) as its
single-precision C port (oracle/cpu_fp32.c) on the host cores, on a bounded
sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


# DRAM bytes per slice-propagation of k_positions at n = 128, 64 slabs:
# dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of the
# kernel on 2 tilts x 64 positions (8192 units): (1.076798 + 1.110183) GB.
# A constant of this bench (ncu does not run inside it), scaled by units.
TRAFFIC_PER_UNIT = (1.076798e9 + 1.110183e9) / 8192


def flops_per_unit(n: int) -> float:
    """FFTW convention: 4 FFTs of n x n (5 N^2 log2 N^2 each) + 32 N^2 pointwise."""
    n2 = n * n
    return 4 * 5 * n2 * math.log2(n2) + 32 * n2


def flops_per_position(n: int) -> float:
    n2 = n * n
    return 6 * 5 * n2 * math.log2(n2) + 40 * n2


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


# ---------------------------------------------------------------------------
def build_problem(cfg_name: str, device: int, tilts=None, method: int = 1, adjoint: int = 0):
    """The configuration's specimen (one seed for every rank) and a batched
    session holding the tilts `tilts` (default: all) with Poisson counts of
    the library's own forward model at the true volumes and the state at half
    the true potential (a mid-reconstruction estimate)."""
    import torch

    from mset_b200 import synth
    from mset_b200.batch import BatchSession

    cfg = synth.CONFIGS[cfg_name]
    spec = synth.make_specimen(cfg)
    tilts = list(range(cfg.n_tilts)) if tilts is None else list(tilts)
    vols = [spec.volumes[j] for j in tilts]
    npos = [spec.scan_x.size] * len(tilts)
    bs = BatchSession(n=cfg.window, nz=cfg.vol[0], npos=npos, prop=spec.prop, sigma=spec.sigma,
                      potential_pixelsize=cfg.dx, slice_binning=cfg.slice_binning, method=method,
                      adjoint=adjoint, device=device)
    if cfg.name.startswith("large"):
        bs.set_amplitude_bf16(True)  # measured counts stored as BF16 (22 GB instead of 44 GB at 41 tilts)
    # simulate the measured intensities with the library's own forward model
    for j, v in enumerate(vols):
        bs.set_tilt(j, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y,
                    measured=np.zeros((npos[j], cfg.window, cfg.window), np.float32), volume=v)
    inten = bs.simulate()
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(cfg.seed + 1000 + 7919 * tilts[0])
    it = torch.from_numpy(inten).to(f"cuda:{device}")
    meas = torch.poisson(it.clamp_min(0), generator=g).cpu().numpy().astype(np.float32)
    del it, inten
    off = 0
    for j, v in enumerate(vols):
        bs.set_tilt(j, measured=meas[off:off + npos[j]], volume=0.5 * v)
        off += npos[j]
    return cfg, spec, bs, meas, tilts


def workload_name(cfg, ns: int, positions: int) -> str:
    nz, ny, nx = cfg.vol
    vol = f"{nx}^3" if nx == ny == nz else f"{nx}x{ny}x{nz}"
    return (f"{cfg.name}: {vol} volume, {cfg.window}^2 window, {cfg.scan[0]}x{cfg.scan[1]} scan, "
            f"{cfg.n_tilts} tilts, {ns} slabs x {cfg.slice_binning} voxels, batched gradient pass over all "
            f"{positions} positions")


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    from mset_b200 import synth
    from mset_b200.distributed import tilt_shard
    ntilts = synth.CONFIGS[args.config].n_tilts
    shard = tilt_shard(ntilts, world, rank)
    if not shard:
        raise SystemExit(f"--gpus {world} exceeds the {ntilts} tilts of the workload")
    cfg, spec, bs, meas, shard = build_problem(args.config, local, shard)
    if args.variant:
        bs.set_variant(args.variant)  # another compiled kernel shape of the window (profiling)
    n = cfg.window
    ns = -(-cfg.vol[0] // cfg.slice_binning)
    positions = int(bs.npos.sum())            # this rank's positions
    units = positions * ns
    positions_total = spec.scan_x.size * cfg.n_tilts
    units_total = positions_total * ns          # the whole workload, over all ranks

    # warm-up (untimed)
    for _ in range(max(args.warmup, 0)):
        bs.gradient(want=())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    if rank == 0:
        sampler.start()
    ms = bs.time_gradient(args.steps)  # CUDA events on the session stream, K passes
    meas_bytes = positions * n * n * (2 if cfg.name.startswith("large") else 4)
    torch.cuda.synchronize()
    clocks = sampler.stop() if rank == 0 else {}
    t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    value = units_total / (ms / 1e3)

    # full batched iteration as one CUDA graph: rotate -> forward -> loss ->
    # adjoint -> rotate back -> update -> positivity -> TV-FISTA (lambda 1e-3)
    it_ms = None
    cubic = cfg.vol[0] == cfg.vol[1] == cfg.vol[2] and cfg.vol[0] <= 160
    if not args.no_iter and cubic:
        bs.iteration_setup(cfg.vol[0], spec.angles[shard], positivity=True, tv_lambda=1e-3, tv_iter=args.tv_iter,
                           tv_fista=True)
        bs.set_rec(0.5 * spec.lab)
        k_it = max(1, min(args.steps, 3))
        if world == 1:
            it_ms = bs.time_iteration(k_it)
        else:
            # tilts sharded over ranks: one NCCL all-reduce of the FP64
            # lab-frame gradient per iteration, on the session stream
            from mset_b200.distributed import GpuBackend, sharded_iterate
            be = GpuBackend(bs)
            sharded_iterate(be, 1)  # capture both phase graphs (warm-up)
            torch.cuda.synchronize()
            dist.barrier()
            with be.stream():
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                sharded_iterate(be, k_it)
                e1.record()
            e1.synchronize()
            it_ms = e0.elapsed_time(e1) / k_it
        t = torch.tensor([it_ms], dtype=torch.float64, device=f"cuda:{local}")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        it_ms = float(t.item())

    # the plain form (reference semantics: one position after another, each
    # updating volume, probe and position; mset_run) and the reference's own
    # CUDA module (oracle/_ref, cuFFT) on a sample of the same tilt
    # side measurements: one GPU only (under torchrun the other ranks would
    # wait for rank 0 in the next collective)
    plain = reference_cuda(args, cfg, spec, meas, units_per_pos=ns) if (world == 1 and not args.no_plain) else None
    if plain is not None:
        # the plain form of the same pass on the same resident data
        pms = bs.time_plain(max(1, min(args.steps, 3)))
        plain["plain_batched"] = {
            "value": units / (pms / 1e3), "unit": "slice-propagations/s", "ms_per_pass": pms,
            "what": "the same pass in plain form: one launch per tilt with one CTA per position (no persistent "
                    "queue across tilts, no CUDA graph, no checkpointing)"}
        plain["batched_over_plain"] = pms / ms
    side = world == 1 and args.config == "mid"
    uneven = uneven_batch(args, local) if (side and not args.no_uneven) else None
    large = large_window(args, local) if (side and not args.no_large) else None

    # end to end through the C ABI with host buffers: volumes in, gradients out
    # host buffers in pinned (page-locked) memory, as a production caller
    # would keep its per-step inputs and outputs
    def pinned(shape, dtype):
        t = torch.empty(shape, dtype=dtype, pin_memory=True)
        return t.numpy()

    vols = []
    for j in shard:
        v = spec.volumes[j]
        hv = pinned(v.shape, torch.float32)
        hv[...] = 0.5 * v
        vols.append(hv)
    grad = pinned((len(shard), ns, n, n), torch.float64)
    err = pinned((len(shard),), torch.float64)
    import ctypes as C
    from mset_b200._lib import check, dptr, fptr
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for j in range(len(shard)):
            check("mset_batch_set_volume", bs._lib.mset_batch_set_volume(bs._h, j, fptr(vols[j])))
        check("mset_batch_gradient", bs._lib.mset_batch_gradient(bs._h, dptr(grad), None, None, dptr(err)))
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    te = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_s = float(te.item())

    if rank == 0:
        peaks = measured_peaks()
        sm_max = float(peaks.get("sm_max_mhz", 1965.0))
        fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s, FMA counted as 2
        flop = units * flops_per_unit(n) + positions * flops_per_position(n)
        achieved = flop / (ms / 1e3) / 1e12
        cpu = cpu_baseline(args, cfg, spec) if (not args.no_cpu and world == 1) else None
        line = {
            "metric": "slice-propagations/s (fwd+adjoint)",
            "value": value,
            "unit": "slice-propagations/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "s_per_step": ms / 1e3,
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "fp32 (complex64 propagation, fp64 reductions)",
            "data": "synthetic (seeded fcc Cu/Au-like Gaussian-atom lattice, Poisson 1e4 e-/probe)",
            "config": {"workload": workload_name(cfg, ns, positions_total),
                       "positions": positions_total, "positions_rank0": positions, "slabs": ns, "window": n,
                       "units_per_step": units_total, "persistent_ctas": bs.shape()["grid"],
                       "kernel_shape": {k: bs.shape()[k] for k in ("threads", "staged", "checkpoint")},
                       "l2": f"inputs larger than L2 ({meas_bytes / 1e9:.1f} GB measured patterns per GPU)",
                       "parallelism": f"tilts sharded over {world} GPU(s): rank 0 holds tilts "
                                      f"{shard[0]}-{shard[-1]} of {cfg.n_tilts}"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak,
                         # DRAM bytes of one launch: the per-unit figure of an ncu capture of the same
                         # kernel (TRAFFIC_PER_UNIT), scaled by units (n^2 for other windows: both terms
                         # are per-pixel); a constant of this bench, not measured per run
                         "traffic": TRAFFIC_PER_UNIT * units * (n / 128.0) ** 2,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of k_positions on "
                                           "2 tilts x 64 positions of this geometry, per slice-propagation, "
                                           "times the launch's slice-propagations (constant, not per run)",
                         "traffic_note": "algorithmic bytes per unit 16*n^2 (saved wave write + read) + "
                                         "4*n^2/slabs (amplitudes)",
                         "algorithmic_bytes": units * (16 * n * n + 4 * n * n / ns),
                         "peak_source": f"nominal FP32 CUDA-core peak 148 SM x 128 lanes x 2 x {sm_max:.0f} MHz "
                                        "(MEASURED_PEAKS has no FP32 figure)",
                         "flop_per_unit": flops_per_unit(n), "flop_per_position": flops_per_position(n)},
            # the same kernel against the measured HBM copy rate (it is not
            # HBM-bound: FP32 issue and the shared-memory data path bound it)
            "roofline_hbm": {"bound": "hbm", "unit": "GB/s",
                             "achieved": units * (16 * n * n + 4 * n * n / ns) / (ms / 1e3) / 1e9,
                             "peak": float(peaks.get("hbm_gbs", 6650.0)),
                             "frac": units * (16 * n * n + 4 * n * n / ns) / (ms / 1e3) / 1e9
                             / float(peaks.get("hbm_gbs", 6650.0)),
                             "traffic": TRAFFIC_PER_UNIT * units * (n / 128.0) ** 2,
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks
                             else "fallback 6.65 TB/s"},
            "e2e": {"value": units_total / e2e_s, "unit": "slice-propagations/s", "host_memory": "pinned",
                    "h2d_bytes_per_step": int(sum(v.nbytes for v in vols)),
                    "d2h_bytes_per_step": int(grad.nbytes + err.nbytes)},
            "iteration": None if it_ms is None else {
                "s_per_iteration": it_ms / 1e3,
                "what": f"{cfg.n_tilts} inverse Fourier-shear rotations, transmission slabs, the batched "
                        f"forward+adjoint pass, {cfg.n_tilts} forward rotations of the gradient, update, positivity, "
                        f"TV-FISTA lambda 1e-3 x {args.tv_iter} iterations, probe and position updates; one CUDA "
                        "graph" + ("" if world == 1 else f" per phase on each of {world} GPUs with the tilts sharded "
                                   "and one NCCL all-reduce of the FP64 lab-frame gradient between the phases"),
                "slice_propagations_per_s": units_total / (it_ms / 1e3)},
            "plain_forms": plain,
            "uneven_batch": uneven,
            "large_window": large,
            "gpu_launches": args.steps * bs._lib.mset_batch_launch_count(bs._h),
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    bs.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def reference_cuda(args, cfg, spec, meas, units_per_pos: int) -> dict:
    """Sequential (reference-semantics) GPU forms on the first positions of
    tilt 0: this library's mset_run (positions in order, each updating
    volume, probe and position; each position's field split over an 8-CTA
    cluster, and on one CTA) and, when built, the reference's own CUDA module
    (src/CUDA/mset.cu + cuFFT via oracle/_ref).  Host time around the
    synchronous call, median of 3 repeats after one warm-up, the upload
    outside the timed call."""
    from mset_b200 import Session

    k = args.plain_positions
    v = 0.5 * spec.volumes[0]
    sx, sy, me = spec.scan_x[:k], spec.scan_y[:k], meas[:k]
    step = (1e-3, 1e-6, 1e-3)
    units = k * units_per_pos
    out = {"positions": k, "slabs": units_per_pos,
           "what": "run_mset over the first positions of tilt 0 (sequential per-position updates)"}

    def timed(run, upload, reps=4):
        ts = []
        for _ in range(reps):
            upload()
            t0 = time.perf_counter()
            run()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts[1:]))

    for split, key in ((True, "plain_gpu"), (False, "plain_gpu_one_cta")):
        with Session() as s:
            s.set_sequential_split(split)
            up = lambda: s.upload(v, spec.probe, spec.prop, sigma=spec.sigma, potential_pixelsize=cfg.dx, scan_x=sx,
                                  scan_y=sy, measured=me, step_size=step, slice_binning=cfg.slice_binning)
            dt = timed(lambda: s.run(1), up)
            out[key] = {"value": units / dt, "unit": "slice-propagations/s", "seconds": dt,
                        "ctas_per_position": s.sequential_split()}
    try:
        from oracle import refharness
        if refharness.available():
            r = refharness.RefSession()
            up = lambda: r.upload(v, spec.probe, spec.prop, sigma=spec.sigma, dz=cfg.dx, scan_x=sx, scan_y=sy,
                                  measured=me, step=step, binning=cfg.slice_binning)
            dt = timed(lambda: r.run(1), up)
            out["reference_cuda"] = {"value": units / dt, "unit": "slice-propagations/s", "seconds": dt,
                                     "what": "the reference's src/CUDA module (cuFFT, ~18*slabs+60 launches per "
                                             "position), compiled unchanged for sm_100a"}
            out["plain_gpu_over_reference_cuda"] = out["reference_cuda"]["seconds"] / out["plain_gpu"]["seconds"]
    except Exception as e:  # the checker build is optional
        out["reference_cuda"] = {"unavailable": str(e)[:200]}
    return out


def uneven_batch(args, device: int) -> dict:
    """Six tilt series of uneven size (windows 64^2-160^2, 11-31 tilts, 32-96
    slabs) as one group pass: every series' persistent kernel, with the batch
    shape (persistent CTAs, checkpoint interval) and the schedule (serial or
    concurrent with SMs split by work) picked by the library's autotuner, the
    pass captured as one CUDA graph.  Beam-frame volumes are Fourier-shear
    rotations of each series' lab-frame volume; intensities are simulated by
    the library's forward model with seeded Poisson noise at each series' dose."""
    import torch

    from mset_b200 import Session, synth
    from mset_b200.batch import BatchSession, SeriesGroup

    t_setup = time.perf_counter()
    members, rows = [], []
    units = positions = 0
    with Session(device) as rot:
        for cfg in synth.UNEVEN:
            spec = synth.make_specimen(cfg, per_tilt=False)
            n, nv = cfg.window, cfg.vol[0]
            ns = -(-nv // cfg.slice_binning)
            npos = [spec.scan_x.size] * cfg.n_tilts
            bs = BatchSession(n=n, nz=nv, npos=npos, prop=spec.prop, sigma=spec.sigma, potential_pixelsize=cfg.dx,
                              slice_binning=cfg.slice_binning, device=device)
            vols = [synth.pad_lateral(rot.rotate_volume(spec.lab, a, inverse=True), n) for a in spec.angles]
            for j, v in enumerate(vols):
                bs.set_tilt(j, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y, volume=v)
            inten = torch.from_numpy(bs.simulate()).to(f"cuda:{device}")
            g = torch.Generator(device=f"cuda:{device}")
            g.manual_seed(cfg.seed + 1000)
            meas = torch.poisson(inten.clamp_min(0), generator=g).cpu().numpy()
            del inten
            off = 0
            for j, v in enumerate(vols):
                bs.set_tilt(j, measured=meas[off:off + npos[j]], volume=0.5 * v)
                off += npos[j]
            del meas
            members.append(bs)
            p = sum(npos)
            units += p * ns
            positions += p
            rows.append({"series": cfg.name, "window": n, "volume_edge": nv, "slabs": ns, "tilts": cfg.n_tilts,
                         "scan": list(cfg.scan), "positions": p, "dose": cfg.dose})
    t_setup = time.perf_counter() - t_setup
    grp = SeriesGroup(members, device=device)
    ms_untuned = grp.time(max(1, min(args.steps, 2)), use_graph=True)
    t0 = time.perf_counter()
    sched = grp.tune(0.0)
    t_tune = time.perf_counter() - t0
    ms = grp.time(args.steps, use_graph=True)
    for r, bs in zip(rows, members):
        r["shape"] = {k: v for k, v in bs.shape().items() if k != "candidates"}
    grp.close()
    for bs in members:
        bs.close()
    return {"value": units / (ms / 1e3), "unit": "slice-propagations/s", "ms_per_pass": ms,
            "units_per_pass": units, "positions": positions,
            "schedule": "concurrent" if sched == 1 else "serial",
            "untuned_serial_ms_per_pass": ms_untuned, "tune_s": t_tune, "setup_s": t_setup,
            "series": rows,
            "what": "6 tilt series of uneven size in one CUDA-graph group pass, shapes and schedule autotuned"}


def large_window(args, device: int) -> dict:
    """The large-reconstruction geometry (256^2 window split over a 4-CTA
    cluster, 256x256x192 volume, 96 slabs, BF16 counts) on 3 of its 41 tilts:
    the batched gradient pass, device-timed."""
    import torch

    cfg, spec, bs, meas, _ = build_problem("large_s", device)
    del meas
    ns = -(-cfg.vol[0] // cfg.slice_binning)
    units = int(bs.npos.sum()) * ns
    for _ in range(max(args.warmup, 1)):
        bs.gradient(want=())
    torch.cuda.synchronize()
    ms = bs.time_gradient(max(1, min(args.steps, 3)))
    n = cfg.window
    flop = units * flops_per_unit(n) + int(bs.npos.sum()) * flops_per_position(n)
    peaks = measured_peaks()
    fp32_peak = 148 * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    out = {"value": units / (ms / 1e3), "unit": "slice-propagations/s", "ms_per_pass": ms,
           "units_per_pass": units, "workload": workload_name(cfg, ns, int(bs.npos.sum())),
           "persistent_ctas": bs.shape()["grid"], "measured_storage": "bf16",
           "fp32_frac": flop / (ms / 1e3) / 1e12 / fp32_peak}
    bs.close()
    out["iteration"] = large_iteration(args, device)
    return out


def large_iteration(args, device: int) -> dict:
    """One batched iteration as a CUDA graph on the large configuration's own
    reconstruction shape (MATLAB 256 x 256 x 192, 96 slabs of 2 voxels, BF16
    counts) on 3 of its tilts: rotations of the unequal-sided volume as
    line transforms, the 256^2 cluster position kernel, TV-FISTA
    (lambda 1e-3 x 300).  Beam-frame volumes for the data are the library's
    own rotations of the lab-frame volume."""
    import torch

    from mset_b200 import Session, synth
    from mset_b200.batch import BatchSession

    cfg = synth.CONFIGS["large_s"]
    spec = synth.make_specimen(cfg, per_tilt=False)
    n, nz = cfg.window, cfg.vol[0]
    ns = -(-nz // cfg.slice_binning)
    npos = [spec.scan_x.size] * cfg.n_tilts
    bs = BatchSession(n=n, nz=nz, npos=npos, prop=spec.prop, sigma=spec.sigma, potential_pixelsize=cfg.dx,
                      slice_binning=cfg.slice_binning, device=device)
    bs.set_amplitude_bf16(True)
    with Session(device) as rot:
        for j, a in enumerate(spec.angles):
            bs.set_tilt(j, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y,
                        volume=synth.pad_lateral(rot.rotate_volume(spec.lab, a, inverse=True), n))
    inten = torch.from_numpy(bs.simulate()).to(f"cuda:{device}")
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(cfg.seed + 1000)
    meas = torch.poisson(inten.clamp_min(0), generator=g).cpu().numpy()
    del inten
    off = 0
    for j in range(cfg.n_tilts):
        bs.set_tilt(j, measured=meas[off:off + npos[j]])
        off += npos[j]
    del meas
    bs.iteration_setup(spec.lab.shape, spec.angles, positivity=True, tv_lambda=1e-3, tv_iter=args.tv_iter,
                       tv_fista=True)
    bs.set_rec(0.5 * spec.lab)
    ms = bs.time_iteration(1)  # captures the graph, then one timed replay
    ms = bs.time_iteration(max(1, min(args.steps, 2)))
    units = int(bs.npos.sum()) * ns
    bs.close()
    return {"s_per_iteration": ms / 1e3, "slice_propagations_per_s": units / (ms / 1e3),
            "workload": workload_name(cfg, ns, int(sum(npos))) + "; reconstruction 256 x 256 x 192 (rotated as "
                        "line transforms)"}


def host_sample(cfg_name: str, k: int):
    """A bounded sample of the workload for the host-side baselines: k
    positions spread over the scan of the specimen's 0-degree tilt (same
    window, volume, slabs and scan as the workload), their intensities from the
    single-precision forward model (oracle/cpu_fp32.c) at the true volume with
    seeded Poisson counts, and the state at half the true potential.  Built on
    the host alone, so the reference arm (which uses no GPU) and the CPU
    baseline of this arm time the same bytes."""
    import dataclasses

    from mset_b200 import synth
    from oracle import oracle as O

    cfg = synth.CONFIGS[cfg_name]
    spec = synth.make_specimen(dataclasses.replace(cfg, n_tilts=1))
    idx = np.linspace(0, spec.scan_x.size - 1, min(k, spec.scan_x.size)).round().astype(int)
    sx, sy = spec.scan_x[idx], spec.scan_y[idx]
    vt = spec.volumes[0]
    inten = O.simulate_fp32(vt, spec.probe, spec.prop, sx, sy, sigma=spec.sigma, dz=cfg.dx, binning=cfg.slice_binning)
    meas = synth.poisson(inten, cfg.seed + 1000)
    ns = -(-cfg.vol[0] // cfg.slice_binning)
    return dict(cfg=cfg, spec=spec, V=(0.5 * vt).astype(np.float32), sx=sx, sy=sy, meas=meas, ns=ns)


def host_pass(smp: dict, cores: int):
    from oracle import oracle as O
    c = smp["cfg"]
    return O.batched_tilt_fp32(smp["V"], smp["spec"].probe, smp["spec"].prop, smp["sx"], smp["sy"], smp["meas"],
                               sigma=smp["spec"].sigma, dz=c.dx, binning=c.slice_binning, nthreads=cores)


def cpu_baseline(args, cfg, spec) -> dict:
    """The single-precision CPU port of the reference's path (oracle/cpu_fp32.c,
    OpenMP over positions, all host threads) on a bounded sample of the same
    workload: all 1,024 positions of one tilt, repeated up to about 10 s."""
    from oracle import oracle as O

    cores = O.max_threads()
    smp = host_sample(args.config, 1024)
    k, ns = smp["sx"].size, smp["ns"]
    # passes over the sample until about 10 s of host work (at most 3)
    reps, t0 = 0, time.perf_counter()
    while reps < 3 and (reps == 0 or time.perf_counter() - t0 < 10.0):
        host_pass(smp, cores)
        reps += 1
    dt = time.perf_counter() - t0
    # the reference-semantics pass on one thread (positions in order, each
    # updating the volume, probe and its coordinates before the next)
    ks = min(16, k)
    t1 = time.perf_counter()
    O.sequential_tilt_fp32(smp["V"], smp["spec"].probe, smp["spec"].prop, smp["sx"][:ks], smp["sy"][:ks],
                           smp["meas"][:ks], sigma=smp["spec"].sigma, dz=smp["cfg"].dx, step=(1e-3, 1e-6, 1e-3),
                           binning=smp["cfg"].slice_binning)
    dts = time.perf_counter() - t1
    return {"value": reps * k * ns / dt, "unit": "slice-propagations/s", "cores": cores, "kind": "port",
            "dtype": "fp32",
            "sample": f"{reps} pass(es) over {k} positions of the 0-degree tilt of the same geometry ({ns} slabs "
                      f"each), single-precision C port of the reference's CPU path (its MATLAB STEP02/STEP03 run "
                      f"in single), {dt:.1f} s",
            "sequential": {"value": ks * ns / dts, "unit": "slice-propagations/s", "cores": 1,
                           "sample": f"{ks} positions of the same sample in order with per-position updates "
                                     f"(run_main_mset semantics), single-precision C port on one thread, "
                                     f"{dts:.1f} s"}}


def run_reference(args):
    """The reference arm: the reference's CPU path (MATLAB STEP02/STEP03 in
    single precision, unavailable here) as its single-precision C port on the
    host cores, on a bounded sample of the same workload per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    cores = O.max_threads()
    smp = host_sample(args.config, max(32, 8 * cores))
    cfg, k, ns = smp["cfg"], smp["sx"].size, smp["ns"]
    for _ in range(max(args.warmup, 0)):
        host_pass(smp, cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        host_pass(smp, cores)
    dt = (time.perf_counter() - t0) / args.steps
    value = k * ns / dt
    line = {
        "impl": "reference",
        "metric": "slice-propagations/s (fwd+adjoint)",
        "value": value,
        "unit": "slice-propagations/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dt * 1e3,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic",
        "config": {"workload": workload_name(cfg, ns, smp["spec"].scan_x.size * cfg.n_tilts),
                   "positions": smp["spec"].scan_x.size * cfg.n_tilts, "slabs": ns, "window": cfg.window,
                   "units_per_step": smp["spec"].scan_x.size * cfg.n_tilts * ns,
                   "sampled": f"{k} positions of the 0-degree tilt per step (units/s of the sample)"},
        "cpu_baseline": {"value": value, "unit": "slice-propagations/s", "cores": cores, "kind": "port",
                         "sample": f"{k} positions x {ns} slabs per step; the reference's CPU path is MATLAB "
                                   "code (STEP02/STEP03) in single precision, unavailable on this box, so its "
                                   "single-precision C port (oracle/cpu_fp32.c) is timed"},
        "e2e": {"value": value, "unit": "slice-propagations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="mid")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-iter", action="store_true", help="skip the full-iteration timing")
    ap.add_argument("--no-plain", action="store_true", help="skip the sequential-form timings")
    ap.add_argument("--plain-positions", type=int, default=32, help="positions in the sequential-form sample")
    ap.add_argument("--tv-iter", type=int, default=300, help="TV-FISTA inner iterations per iteration")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-size 6-series group pass")
    ap.add_argument("--no-large", action="store_true", help="skip the 256^2-window (cluster) sample")
    ap.add_argument("--variant", type=int, default=0, help="kernel shape of the window (0: default; profiling)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
