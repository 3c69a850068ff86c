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
iteration as one CUDA graph, the sequential plain forms (this library's and
the reference's own CUDA module), the uneven-size 6-series group pass with the
autotuner, the 256^2-window cluster kernel on 3 tilts of the large geometry,
and the FP64 CPU port on a sample.

One JSON line on stdout (rank 0).  --impl reference times the FP64 CPU port
of the reference's path (the reference's own CPU path is MATLAB code, which
is not available here) on a bounded sample of the same workload.
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


# DRAM bytes per slice-propagation of k_positions at n = 128, 64 slabs,
# measured with ncu on 128 positions (8192 units): (1.077490 + 1.111658) GB
TRAFFIC_PER_UNIT = (1.077490e9 + 1.111658e9) / 8192


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
def build_problem(cfg_name: str, rank: int, device: int, method: int = 1, adjoint: int = 0):
    import torch

    from mset_b200 import synth
    from mset_b200.batch import BatchSession

    cfg = synth.CONFIGS[cfg_name]
    cfg = synth.Config(**{**cfg.__dict__, "seed": cfg.seed + 7919 * rank})
    spec = synth.make_specimen(cfg)
    npos = [spec.scan_x.size] * cfg.n_tilts
    bs = BatchSession(n=cfg.window, nz=cfg.vol[0], npos=npos, prop=spec.prop, sigma=spec.sigma,
                      potential_pixelsize=cfg.dx, slice_binning=cfg.slice_binning, method=method,
                      adjoint=adjoint, device=device)
    if cfg.name.startswith("large"):
        bs.set_amplitude_bf16(True)  # measured counts stored as BF16 (22 GB instead of 44 GB at 41 tilts)
    # simulate the measured intensities with the library's own forward model
    for j, v in enumerate(spec.volumes):
        bs.set_tilt(j, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y,
                    measured=np.zeros((npos[j], cfg.window, cfg.window), np.float32), volume=v)
    inten = bs.simulate()
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(cfg.seed + 1000)
    it = torch.from_numpy(inten).to(f"cuda:{device}")
    meas = torch.poisson(it.clamp_min(0), generator=g).cpu().numpy().astype(np.float32)
    del it, inten
    # reconstruction state: half the true potential (a mid-iteration estimate)
    off = 0
    for j, v in enumerate(spec.volumes):
        bs.set_tilt(j, measured=meas[off:off + npos[j]], volume=0.5 * v)
        off += npos[j]
    return cfg, spec, bs, meas


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
    cfg, spec, bs, meas = build_problem(args.config, rank, local)
    n = cfg.window
    ns = -(-cfg.vol[0] // cfg.slice_binning)
    positions = int(bs.npos.sum())
    units = positions * ns

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
    value = world * units / (ms / 1e3)

    # full batched iteration as one CUDA graph: rotate -> forward -> loss ->
    # adjoint -> rotate back -> update -> positivity -> TV-FISTA (lambda 1e-3)
    it_ms = None
    cubic = cfg.vol[0] == cfg.vol[1] == cfg.vol[2] and cfg.vol[0] <= 160
    if not args.no_iter and cubic:
        bs.iteration_setup(cfg.vol[0], spec.angles, positivity=True, tv_lambda=1e-3, tv_iter=args.tv_iter,
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
    for v in spec.volumes:
        hv = pinned(v.shape, torch.float32)
        hv[...] = 0.5 * v
        vols.append(hv)
    grad = pinned((cfg.n_tilts, ns, n, n), torch.float64)
    err = pinned((cfg.n_tilts,), torch.float64)
    import ctypes as C
    from mset_b200._lib import check, dptr, fptr
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for j in range(cfg.n_tilts):
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
        cpu = cpu_baseline(args, cfg, spec, meas) if (not args.no_cpu and world == 1) else None
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
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp32 (complex64 propagation, fp64 reductions)",
            "data": "synthetic (seeded fcc Cu/Au-like Gaussian-atom lattice, Poisson 1e4 e-/probe)",
            "config": {"workload": workload_name(cfg, ns, positions),
                       "positions_per_gpu": positions, "slabs": ns, "window": n,
                       "units_per_step_per_gpu": units, "persistent_ctas": bs.shape()["grid"],
                       "l2": f"inputs larger than L2 ({meas_bytes / 1e9:.1f} GB measured patterns)",
                       "parallelism": f"tilt replicas x{world}"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak,
                         # ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_positions launch on
                         # the mid_s capture (128 positions: 1.0775 GB + 1.1117 GB), scaled by units
                         # (n^2 scaling to other windows: both terms are per-pixel)
                         "traffic": TRAFFIC_PER_UNIT * units * (n / 128.0) ** 2,
                         "traffic_note": "bytes per launch from the ncu capture of the same kernel on 128 positions "
                                         "(profiles/k_positions_mid_s.md), scaled by slice-propagations; "
                                         "algorithmic bytes per unit 16*n^2 (saved wave write + read) + "
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
            "e2e": {"value": world * units / e2e_s, "unit": "slice-propagations/s", "host_memory": "pinned",
                    "h2d_bytes_per_step": int(sum(v.nbytes for v in vols)),
                    "d2h_bytes_per_step": int(grad.nbytes + err.nbytes)},
            "iteration": None if it_ms is None else {
                "s_per_iteration": it_ms / 1e3,
                "what": "one CUDA-graph replay: 21 inverse Fourier-shear rotations, transmission slabs, the "
                        "batched forward+adjoint pass, 21 forward rotations of the gradient, update, positivity, "
                        f"TV-FISTA lambda 1e-3 x {args.tv_iter} iterations, probe and position updates",
                "slice_propagations_per_s": world * units / (it_ms / 1e3)},
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
    tilt 0: this library's plain fused kernel (mset_run, one CTA walking the
    positions in order) and, when built, the reference's own CUDA module
    (src/CUDA/mset.cu + cuFFT via oracle/_ref).  Both: CUDA-event free host
    timing around a synchronous call, after one warm-up call."""
    from mset_b200 import Session

    k = args.plain_positions
    n = cfg.window
    v = 0.5 * spec.volumes[0]
    sx, sy, me = spec.scan_x[:k], spec.scan_y[:k], meas[:k]
    step = (1e-3, 1e-6, 1e-3)
    out = {"positions": k, "slabs": units_per_pos,
           "what": "run_mset over the first positions of tilt 0 (sequential per-position updates)"}
    with Session() as s:
        for rep in range(2):
            s.upload(v, spec.probe, spec.prop, sigma=spec.sigma, potential_pixelsize=cfg.dx, scan_x=sx, scan_y=sy,
                     measured=me, step_size=step, slice_binning=cfg.slice_binning)
            t0 = time.perf_counter()
            s.run(1)
            dt = time.perf_counter() - t0
        out["plain_gpu"] = {"value": k * units_per_pos / dt, "unit": "slice-propagations/s", "seconds": dt}
    try:
        from oracle import refharness
        if refharness.available():
            for rep in range(2):
                r = refharness.RefSession()
                r.upload(v, spec.probe, spec.prop, sigma=spec.sigma, dz=cfg.dx, scan_x=sx, scan_y=sy, measured=me,
                         step=step, binning=cfg.slice_binning)
                t0 = time.perf_counter()
                r.run(1)
                dt = time.perf_counter() - t0
            out["reference_cuda"] = {"value": k * units_per_pos / dt, "unit": "slice-propagations/s", "seconds": dt,
                                     "what": "the reference's src/CUDA module (cuFFT, ~18*slabs+60 launches per "
                                             "position), compiled unchanged for sm_100a"}
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

    cfg, spec, bs, meas = build_problem("large_s", 0, device)
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
    """One batched iteration as a CUDA graph in the 256^2 window on a cubic
    256^3 reconstruction (3 tilts x 4,096 positions, 128 slabs): rotations of
    256^3 volumes with each shear plane over a 4-CTA cluster, the cluster
    position kernel, TV-FISTA (lambda 1e-3 x 300).  Beam-frame volumes for
    the data are the library's own rotations of the lab-frame volume."""
    import torch

    from mset_b200 import Session, synth
    from mset_b200.batch import BatchSession

    cfg = synth.CONFIGS["large_cubic_s"]
    spec = synth.make_specimen(cfg, per_tilt=False)
    n, nv = cfg.window, cfg.vol[0]
    ns = -(-nv // cfg.slice_binning)
    npos = [spec.scan_x.size] * cfg.n_tilts
    bs = BatchSession(n=n, nz=nv, npos=npos, prop=spec.prop, sigma=spec.sigma, potential_pixelsize=cfg.dx,
                      slice_binning=cfg.slice_binning, device=device)
    bs.set_amplitude_bf16(True)
    with Session(device) as rot:
        for j, a in enumerate(spec.angles):
            bs.set_tilt(j, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y,
                        volume=rot.rotate_volume(spec.lab, a, inverse=True))
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
    bs.iteration_setup(nv, spec.angles, positivity=True, tv_lambda=1e-3, tv_iter=args.tv_iter, tv_fista=True)
    bs.set_rec(0.5 * spec.lab)
    ms = bs.time_iteration(1)  # captures the graph, then one timed replay
    ms = bs.time_iteration(max(1, min(args.steps, 2)))
    units = int(bs.npos.sum()) * ns
    bs.close()
    return {"s_per_iteration": ms / 1e3, "slice_propagations_per_s": units / (ms / 1e3),
            "workload": workload_name(cfg, ns, int(sum(npos)))}


def cpu_sample_positions(cores: int) -> int:
    return int(max(8, min(96, 6 * cores)))


def cpu_baseline(args, cfg, spec, meas) -> dict:
    """FP64 CPU port (oracle) on a bounded sample of the same workload."""
    from oracle import oracle as O

    cores = O.max_threads()
    k = cpu_sample_positions(cores)
    ns = -(-cfg.vol[0] // cfg.slice_binning)
    t0 = time.perf_counter()
    O.batched_tilt(0.5 * spec.volumes[0], spec.probe, spec.prop, spec.scan_x[:k], spec.scan_y[:k], meas[:k],
                   sigma=spec.sigma, dz=cfg.dx, binning=cfg.slice_binning, nthreads=cores)
    dt = time.perf_counter() - t0
    # the reference's sequential semantics (per-position updates) on one core
    ks = 4
    t1 = time.perf_counter()
    O.run_tilt(0.5 * spec.volumes[0], spec.probe, spec.prop, spec.scan_x[:ks], spec.scan_y[:ks], meas[:ks],
               sigma=spec.sigma, dz=cfg.dx, step=(1e-3, 1e-6, 1e-3), binning=cfg.slice_binning)
    dt1 = time.perf_counter() - t1
    return {"value": k * ns / dt, "unit": "slice-propagations/s", "cores": cores, "kind": "port",
            "sample": f"{k} positions of tilt 0 of the same workload (FP64 C port of the reference path, "
                      f"OpenMP over positions), {dt:.1f} s",
            "sequential_1core": {"value": ks * ns / dt1, "unit": "slice-propagations/s", "cores": 1,
                                 "sample": f"run_mset semantics (per-position updates) over {ks} positions of "
                                           f"tilt 0, FP64 C port, {dt1:.1f} s"}}


def run_reference(args):
    """The reference arm: the FP64 CPU port of the reference's path on the
    host cores, on a bounded sample of the same workload per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from mset_b200 import synth
    from oracle import oracle as O

    cfg = synth.CONFIGS[args.config]
    spec = synth.make_specimen(cfg, with_volumes=False)
    rng = np.random.default_rng(cfg.seed)
    pos, peak = synth.atoms(cfg, rng)
    v = synth.pad_lateral(synth.voxelise(pos, peak, cfg.vol, cfg.dx, cfg.blob_sigma), cfg.window).astype(np.float32)
    cores = O.max_threads()
    k = max(4, cpu_sample_positions(cores) // 4)
    n = cfg.window
    meas = np.full((k, n, n), 1.0, np.float32)
    ns = -(-cfg.vol[0] // cfg.slice_binning)
    for _ in range(max(args.warmup, 0) and 1):
        O.batched_tilt(0.5 * v, spec.probe, spec.prop, spec.scan_x[:1], spec.scan_y[:1], meas[:1],
                       sigma=spec.sigma, dz=cfg.dx, binning=cfg.slice_binning, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.batched_tilt(0.5 * v, spec.probe, spec.prop, spec.scan_x[:k], spec.scan_y[:k], meas, sigma=spec.sigma,
                       dz=cfg.dx, binning=cfg.slice_binning, nthreads=cores)
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
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp64",
        "data": "synthetic",
        "config": {"workload": "mid: 128^3 volume, 128^2 window, 32x32 scan, 21 tilts, 64 slabs x 2 voxels "
                               f"(sampled: {k} positions per step)"},
        "cpu_baseline": {"value": value, "unit": "slice-propagations/s", "cores": cores, "kind": "port",
                         "sample": f"{k} positions x {ns} slabs per step; the reference's own CPU path is MATLAB "
                                   "code (STEP02/STEP03), unavailable on this box, so its FP64 C port is timed"},
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
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
