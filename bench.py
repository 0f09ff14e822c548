#!/usr/bin/env python
"""Benchmark: TV-ADMM dipole inversion throughput on B200.

Workload (one "step"): one TV-ADMM solve (src/inversion/tv.rs:63-97) of a 256x256x176
volume at 1 mm, B0 = z, default TvParams with tol = 0 so that exactly 250 iterations run,
mixed precision (float FFTs and stencils, FP64 reductions and multipliers).  Input is a
seeded synthetic ellipsoid phantom inside a 100x120x75-voxel ellipsoid brain mask
(local field = dipole-convolved chi + N(0, 0.01 ppm) noise); no public dataset is used.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Ranks (torchrun, one per GPU) each solve their own volumes (weak scaling, no collective
in the data path); value = volumes all ranks solved / max-over-ranks device time.
Rank 0 prints one JSON line.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "qsm.rs_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

DIMS = (256, 256, 176)
ITERS = 250
METRIC = "TV-ADMM volumes/s at 256x256x176 (250 iterations)"
UNIT = "volumes/s"
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "tv_admm_256x256x176_dram.txt")


def ncu_traffic():
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the TV-ADMM
    kernels at this workload, from the committed summary of one ncu capture ("name bytes"
    lines; ncu flushes the caches before each replay, so these are cold-cache figures)."""
    out = {}
    try:
        with open(TRAFFIC_FILE) as fh:
            for line in fh:
                parts = line.split("#", 1)[0].split()
                if len(parts) == 2:
                    out[parts[0]] = int(parts[1])
    except OSError:
        pass
    return out


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-extras", action="store_true",
                    help="skip the full-chain and 32-volume batch measurements (reported beside the headline)")
    return ap.parse_args()


def make_case(seed):
    from qsmgpu import phantom
    return phantom.brain_tv_case(seed, DIMS)


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), line.strip()))

    def mark(self, which):
        if which == "start":
            self.t0 = time.time()
        else:
            self.t1 = time.time()

    def stop(self):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = [s for (t, s) in self.samples if self.t0 is not None and self.t0 - 0.05 <= t <= (self.t1 or t) + 0.05]
        if not rows:
            rows = [s for (_, s) in self.samples]
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            p = [x.strip() for x in r.split(",")]
            if len(p) < 9:
                continue
            try:
                sms.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def kernel_bytes_model(N, s):
    """Algorithmic bytes per launch of each TV-ADMM kernel (s = 4 FP32, 8 FP64).
    A half spectrum is counted as N*s bytes."""
    return {
        "tv_step": 10 * N * s,     # read x0, y_{i-1}, y_{i-2}, u(3); write u(3), div
        "fft_x_r2c": 2 * N * s,    # read div, write spectrum
        "fft_y_fwd": 2 * N * s,
        "fft_z_fused": 2 * N * s + N * s // 2,  # read + write spectrum, read the real half-spectrum multiplier
        "fft_y_inv": 2 * N * s,
        "fft_x_c2r": 2 * N * s,    # read spectrum, write y_i
    }


def _timed_oracle_tv(f, mask, iters):
    """Run the oracle TV-ADMM for `iters` iterations and time the spectral preparation and
    each iteration through the progress callback (called at the start of every iteration,
    src/inversion/tv.rs:81)."""
    from oracle import qsm_oracle as O
    grid = O.Grid.new(*DIMS)
    stamps = []
    t0 = time.perf_counter()
    O.tv_admm(f, mask, grid, (0, 0, 1), O.TvParams(2e-4, 2e-2, 0.0, iters),
              lambda a, b: stamps.append(time.perf_counter()))
    t_end = time.perf_counter()
    stamps.append(t_end)
    t_prep = stamps[0] - t0
    per_iter = [b - a for a, b in zip(stamps[:-1], stamps[1:])]
    return t_prep, per_iter


def cpu_baseline_tv(f, mask, budget_iters=4):
    """Oracle (f64 numpy/scipy restatement) timed on this host: preparation + a few
    iterations at full size; per-volume time = prep + ITERS * median iteration time."""
    from oracle import qsm_oracle as O
    cores = os.cpu_count() or 1
    O.set_fft_workers(cores)
    try:
        t_prep, per_iter = _timed_oracle_tv(f, mask, budget_iters)
    finally:
        O.set_fft_workers(None)
    t_iter = statistics.median(per_iter[1:] if len(per_iter) > 1 else per_iter)
    vol_s = t_prep + ITERS * t_iter
    return {"value": 1.0 / vol_s, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle TV-ADMM at {DIMS[0]}x{DIMS[1]}x{DIMS[2]}: preparation + {budget_iters} iterations "
                      f"timed, scaled to {ITERS} ({t_iter * 1e3:.0f} ms/iteration, scipy.fft workers={cores})",
            "ms_per_iteration": t_iter * 1e3}


def _fast_size(n):
    """Smallest 2^a 3^b 5^c >= n (src/utils/padding.rs:9)."""
    m = n
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def _rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / (np.linalg.norm(b) or 1.0))


def _errs(a, b):
    """rel-L2 and max-abs of a against the comparator b."""
    return {"rel_l2": _rel_l2(a, b), "max_abs": float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max())}


def _profiled(ctx, fn):
    """{kernel: (launches, total_ms)} of one call of fn with per-launch CUDA events."""
    ctx.set_profiling(True)
    ctx.profile_reset()
    fn()
    prof = ctx.profile()
    ctx.set_profiling(False)
    return prof


def _dominant_roofline(prof, model, note):
    """Roofline of the modelled kernel with the largest total time: algorithmic bytes
    per launch (model) / average launch time, against the measured HBM peak."""
    peak, kind = measured_peak()
    cands = [k for k in model if k in prof]
    if not cands:
        return None
    dom = max(cands, key=lambda k: prof[k][1])
    cnt, tot = prof[dom]
    avg_s = tot / max(cnt, 1) / 1e3
    gbs = model[dom] / avg_s / 1e9
    tot_all = sum(v[1] for v in prof.values()) or 1.0
    return {"bound": "hbm", "kernel": dom, "launches": cnt, "avg_us": round(avg_s * 1e6, 2),
            "alg_bytes": int(model[dom]), "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
            "frac": round(gbs / peak, 3), "share": round(tot / tot_all, 3), "model": note,
            "peak_source": kind}


def _timed(stream, fn, reps=1):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def bench_chain(local, dev):
    """Full chain at 256x256x176 (wrapped phase -> laplacian_unwrap -> ppm -> vsharp with
    default radii -> tv_admm 250 iterations), mixed precision, stage times with CUDA events
    and each stage's rel-L2 error against the FP64 GPU chain on the same input."""
    import torch
    import qsmgpu
    from qsmgpu import Grid, inversion, unwrap, bgremove, phantom
    case = phantom.chain_case()
    grid = Grid.new(*case.dims)
    N = case.mask.size
    ph = torch.from_numpy(np.ascontiguousarray(case.wrapped_phase).ravel()).to(dev)
    m = torch.from_numpy(np.ascontiguousarray(case.mask).ravel()).to(dev)
    radii = bgremove.vsharp_radii()
    out = {}
    for prec in ("mixed", "f64"):
        ctx = qsmgpu.Context(local, prec)
        s = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
        uw = torch.empty(N, dtype=torch.float64, device=dev)
        loc = torch.empty_like(uw)
        fm = torch.empty(N, dtype=torch.uint8, device=dev)
        chi = torch.empty_like(uw)
        p = inversion.TvParams(2e-4, 2e-2, 0.0, ITERS)

        def st_unwrap():
            unwrap.laplacian_unwrap_device(ctx, ph.data_ptr(), m.data_ptr(), grid, uw.data_ptr())

        def st_vsharp():
            fppm = uw / case.rad_per_ppm
            bgremove.vsharp_with_radii_device(ctx, fppm.data_ptr(), m.data_ptr(), grid, radii, 0.05, loc.data_ptr(),
                                              fm.data_ptr())

        def st_tv():
            inversion.tv_admm_device(ctx, loc.data_ptr(), fm.data_ptr(), grid, (0.0, 0.0, 1.0), p, chi.data_ptr())

        st_unwrap(), st_vsharp(), st_tv()  # warm-up
        times = {"unwrap": _timed(s, st_unwrap), "vsharp": _timed(s, st_vsharp), "tv_admm": _timed(s, st_tv)}
        out[prec] = {"ms": {k: round(v, 3) for k, v in times.items()},
                     "arrays": (uw.cpu().numpy(), loc.cpu().numpy(), fm.cpu().numpy(), chi.cpu().numpy())}
        if prec == "mixed":
            # every V-SHARP FFT pass reads and writes one half spectrum (N*s bytes each way)
            sz = 4
            model = {k: 2 * N * sz for k in ("fft_x_r2c", "fft_y_fwd", "fft_z_fwd", "fft_z_inv", "fft_y_inv",
                                              "fft_x_c2r", "fft_z_fused")}
            out["roofline"] = _dominant_roofline(_profiled(ctx, st_vsharp), model,
                                                 "FFT pass: read + write one float half spectrum, 2*N*4 B")
        ctx.close()
    a, b = out["mixed"]["arrays"], out["f64"]["arrays"]
    return {"workload": "wrapped phase 256x256x176, 3 T, TE 20 ms -> laplacian_unwrap -> vsharp (12 radii) -> "
                        f"tv_admm x{ITERS}; synthetic brain-mask phantom with 4 background dipoles",
            "ms_mixed": out["mixed"]["ms"], "ms_f64": out["f64"]["ms"],
            "errors_mixed_vs_fp64_gpu": {"unwrap": _errs(a[0], b[0]), "vsharp": _errs(a[1], b[1]),
                                          "tv_admm": _errs(a[3], b[3])},
            "vsharp_mask_equal": bool(np.array_equal(a[2], b[2])),
            "vsharp_roofline_mixed": out.get("roofline")}


def bench_batch(local, dev, n_vol=32, seed=7):
    """32 volumes, each dimension from {96..224} x {96..224} x {64..160} rounded to
    2^a 3^b 5^c, B0 tilted up to 25 degrees, ellipsoid phantom + noise: batched TV-ADMM
    (250 iterations, mixed) and TKD (threshold 0.19) in one call each, against the same
    volumes solved one call at a time."""
    import torch
    import qsmgpu
    from qsmgpu import Grid, inversion, phantom
    rng = np.random.default_rng(seed)
    ctx = qsmgpu.Context(local, "mixed")
    s = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    cases, keep, vox = [], [], 0
    for _ in range(n_vol):
        nx, ny = (_fast_size(int(rng.integers(96, 225))) for _ in range(2))
        nz = _fast_size(int(rng.integers(64, 161)))
        th, ph = np.radians(rng.uniform(0, 25)), rng.uniform(0, 2 * np.pi)
        bdir = (float(np.sin(th) * np.cos(ph)), float(np.sin(th) * np.sin(ph)), float(np.cos(th)))
        grid = Grid.new(nx, ny, nz)
        shape = (nz, ny, nx)
        mask = phantom.ellipsoid_mask(shape, (0.4 * nx, 0.45 * ny, 0.4 * nz))
        chi = np.zeros(shape)
        ctr = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
        phantom.add_ellipsoids(chi, rng, 8, [(c - 0.25 * n, c + 0.25 * n) for c, n in zip(ctr, (nx, ny, nz))],
                               semi=(3.0, 10.0))
        chi *= mask
        dchi = torch.from_numpy(chi.ravel()).to(dev)
        f = torch.empty_like(dchi)
        inversion.dipole_forward_device(ctx, dchi.data_ptr(), grid, bdir, f.data_ptr())
        f += torch.from_numpy(rng.normal(0.0, 0.01, size=chi.size) * mask.ravel()).to(dev)
        dm = torch.from_numpy(mask.ravel()).to(dev)
        do = torch.empty_like(f)
        keep += [f, dm, do]
        cases.append((f.data_ptr(), dm.data_ptr(), do.data_ptr(), grid, bdir))
        vox += chi.size
    p = inversion.TvParams(2e-4, 2e-2, 0.0, ITERS)
    inversion.tv_admm_batch_device(ctx, cases, p)  # warm-up
    t_batch = _timed(s, lambda: inversion.tv_admm_batch_device(ctx, cases, p))
    one_by_one = lambda: [inversion.tv_admm_device(ctx, df, dm, g, b, p, do) for df, dm, do, g, b in cases]
    # the batch's own results, before the one-call-per-volume run overwrites the outputs
    res32 = [keep[3 * i + 2].cpu().numpy() for i in range(n_vol)]
    one_by_one()  # warm-up: grows the single-volume workspace to the largest volume
    t_seq = _timed(s, one_by_one)
    tk = inversion.TkdParams(0.19)
    inversion.tkd_batch_device(ctx, cases, tk)
    t_tkd = _timed(s, lambda: inversion.tkd_batch_device(ctx, cases, tk), reps=3)
    tkd32 = [keep[3 * i + 2].cpu().numpy() for i in range(n_vol)]
    ctx.close()
    # the same batch in FP64 (the plain comparator), batched
    c64 = qsmgpu.Context(local, "f64")
    s64 = torch.cuda.ExternalStream(c64.stream_handle(), device=dev)
    inversion.tv_admm_batch_device(c64, cases, p)
    t_b64 = _timed(s64, lambda: inversion.tv_admm_batch_device(c64, cases, p))
    res64 = [keep[3 * i + 2].cpu().numpy() for i in range(n_vol)]
    inversion.tkd_batch_device(c64, cases, tk)
    t_tkd64 = _timed(s64, lambda: inversion.tkd_batch_device(c64, cases, tk), reps=3)
    tkd64 = [keep[3 * i + 2].cpu().numpy() for i in range(n_vol)]
    c64.close()
    worst = lambda xs, ys: {"rel_l2_max_over_volumes": max(_rel_l2(x, y) for x, y in zip(xs, ys)),
                            "max_abs": max(float(np.abs(x - y).max()) for x, y in zip(xs, ys))}
    return {"workload": f"{n_vol} volumes of uneven size (2^a 3^b 5^c in 96-224 x 96-224 x 64-160), B0 tilted "
                        f"<= 25 deg, TV-ADMM x{ITERS} + TKD 0.19; {vox / 1e6:.1f} M voxels in total",
            "tv_admm_batched_mixed": {"volumes_per_s": round(n_vol / (t_batch / 1e3), 3), "ms": round(t_batch, 2)},
            "tv_admm_batched_fp64": {"volumes_per_s": round(n_vol / (t_b64 / 1e3), 3), "ms": round(t_b64, 2)},
            "tv_admm_one_call_per_volume_mixed": {"volumes_per_s": round(n_vol / (t_seq / 1e3), 3),
                                                  "ms": round(t_seq, 2)},
            "batched_mixed_over_batched_fp64": round(t_b64 / t_batch, 3),
            "tv_admm_errors_mixed_vs_fp64_gpu": worst(res32, res64),
            "tkd_batched_mixed": {"volumes_per_s": round(n_vol / (t_tkd / 1e3), 3), "ms": round(t_tkd, 3)},
            "tkd_batched_fp64": {"volumes_per_s": round(n_vol / (t_tkd64 / 1e3), 3), "ms": round(t_tkd64, 3)},
            "tkd_errors_mixed_vs_fp64_gpu": worst(tkd32, tkd64)}


def bench_batch_brain(local, dev, n_vol=4):
    """A batch of n_vol 256x256x176 volumes (the throughput phantom with seeds 0..n-1),
    TV-ADMM x250: batched mixed precision against the plain FP64 form (one FP64 call per
    volume)."""
    import torch
    import qsmgpu
    from qsmgpu import Grid, inversion
    grid = Grid.new(*DIMS)
    keep, cases = [], []
    for k in range(n_vol):
        f, m = make_case(k)
        df = torch.from_numpy(f.ravel()).to(dev)
        dm = torch.from_numpy(m.ravel()).to(dev)
        do = torch.empty_like(df)
        keep += [df, dm, do]
        cases.append((df.data_ptr(), dm.data_ptr(), do.data_ptr(), grid, (0.0, 0.0, 1.0)))
    p = inversion.TvParams(2e-4, 2e-2, 0.0, ITERS)
    ctx = qsmgpu.Context(local, "mixed")
    s = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    inversion.tv_admm_batch_device(ctx, cases, p)
    t_b = _timed(s, lambda: inversion.tv_admm_batch_device(ctx, cases, p))
    r32 = [keep[3 * i + 2].cpu().numpy() for i in range(n_vol)]
    ctx.close()
    c64 = qsmgpu.Context(local, "f64")
    s64 = torch.cuda.ExternalStream(c64.stream_handle(), device=dev)
    plain = lambda: [inversion.tv_admm_device(c64, df, dm, g, b, p, do) for df, dm, do, g, b in cases]
    plain()
    t_64 = _timed(s64, plain)
    r64 = [keep[3 * i + 2].cpu().numpy() for i in range(n_vol)]
    c64.close()
    return {"workload": f"{n_vol} volumes of 256x256x176 (throughput phantom, seeds 0..{n_vol - 1}), tv_admm x{ITERS}",
            "batched_mixed": {"volumes_per_s": round(n_vol / (t_b / 1e3), 3), "ms": round(t_b, 2)},
            "plain_fp64": {"volumes_per_s": round(n_vol / (t_64 / 1e3), 3), "ms": round(t_64, 2)},
            "batched_mixed_over_plain_fp64": round(t_64 / t_b, 3),
            "errors_mixed_vs_fp64_gpu": {"rel_l2_max_over_volumes": max(_rel_l2(a, b) for a, b in zip(r32, r64)),
                                         "max_abs": max(float(np.abs(a - b).max()) for a, b in zip(r32, r64))}}


def bench_batch_sharded(local, dev, rank, world, dist, n_vol=32, seed=7):
    """The 32-volume TV-ADMM batch (mixed) sharded over the ranks: every rank draws the
    same batch description, keeps the volumes the longest-processing-time placement gives
    it (qsm_batch_partition) and solves them as one batched call; no collective while
    solving.  Time = max over ranks (device events); the results stay on their ranks."""
    import torch
    import qsmgpu
    from qsmgpu import Grid, inversion, phantom, shard
    rng = np.random.default_rng(seed)
    desc = []
    for _ in range(n_vol):
        nx, ny = (_fast_size(int(rng.integers(96, 225))) for _ in range(2))
        nz = _fast_size(int(rng.integers(64, 161)))
        th, ph = np.radians(rng.uniform(0, 25)), rng.uniform(0, 2 * np.pi)
        desc.append((Grid.new(nx, ny, nz), (float(np.sin(th) * np.cos(ph)), float(np.sin(th) * np.sin(ph)),
                                            float(np.cos(th))), int(rng.integers(1 << 30))))
    mine = shard.share([d[0] for d in desc], rank, world, [ITERS] * n_vol)
    ctx = qsmgpu.Context(local, "mixed")
    s = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    keep, cases = [], []
    for b in mine:
        grid, bdir, vseed = desc[b]
        nz, ny, nx = grid.shape
        vr = np.random.default_rng(vseed)
        mask = phantom.ellipsoid_mask(grid.shape, (0.4 * nx, 0.45 * ny, 0.4 * nz))
        chi = np.zeros(grid.shape)
        ctr = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
        phantom.add_ellipsoids(chi, vr, 8, [(c - 0.25 * n, c + 0.25 * n) for c, n in zip(ctr, (nx, ny, nz))],
                               semi=(3.0, 10.0))
        dchi = torch.from_numpy((chi * mask).ravel()).to(dev)
        f = torch.empty_like(dchi)
        inversion.dipole_forward_device(ctx, dchi.data_ptr(), grid, bdir, f.data_ptr())
        f += torch.from_numpy(vr.normal(0.0, 0.01, size=chi.size) * mask.ravel()).to(dev)
        dm = torch.from_numpy(mask.ravel()).to(dev)
        do = torch.empty_like(f)
        keep += [f, dm, do]
        cases.append((f.data_ptr(), dm.data_ptr(), do.data_ptr(), grid, bdir))
    p = inversion.TvParams(2e-4, 2e-2, 0.0, ITERS)
    run = lambda: inversion.tv_admm_batch_device(ctx, cases, p) if cases else None
    run()
    dist.barrier()
    torch.cuda.synchronize()
    ms = _timed(s, run)
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ctx.close()
    ms = float(t.item())
    return {"workload": f"{n_vol} uneven volumes (as batch_32_volumes), tv_admm x{ITERS} mixed, placed over {world} "
                        "GPUs by longest-processing-time on N log N x iterations",
            "volumes_per_s": round(n_vol / (ms / 1e3), 3), "ms_max_over_ranks": round(ms, 2),
            "volumes_on_rank0": len(mine) if rank == 0 else None}


def bench_adjoint(local, dev):
    """Unrolled TV-ADMM at 160x192x160: K = 50 iterations with no early exit, states
    checkpointed every 10, lambda 1e-3, rho 2e-2, mixed precision.  Times the forward pass
    alone and the forward pass plus the hand-written vector-Jacobian product (dL/dfield
    and dL/dlambda for L = ||chi_K - chi_true||^2)."""
    import torch
    import qsmgpu
    from qsmgpu import Grid, inversion, phantom
    dims = (160, 192, 160)
    case = phantom.tv_case(dims, seed=4, n_ellipsoids=12, mask_radius=70.0)
    grid = Grid.new(*dims)
    out = {"workload": "unrolled tv_admm 160x192x160, K=50, checkpoint every 10, lambda 1e-3, rho 2e-2, mixed; "
                       "ellipsoid phantom"}
    gchi64 = None
    res = {}
    for prec in ("f64", "mixed"):
        ctx = qsmgpu.Context(local, prec)
        s = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
        f = torch.from_numpy(np.ascontiguousarray(case.local_field).ravel()).to(dev)
        m = torch.from_numpy(np.ascontiguousarray(case.mask).ravel()).to(dev)
        truth = torch.from_numpy(np.ascontiguousarray(case.chi).ravel()).to(dev)
        chi = torch.empty_like(f)
        gf = torch.empty_like(f)
        gchi = torch.empty_like(f)
        glam = [0.0]

        def fwd():
            inversion.tv_admm_unrolled_vjp_device(ctx, f.data_ptr(), m.data_ptr(), grid, (0.0, 0.0, 1.0), 1e-3, 2e-2,
                                                  50, 10, 0, chi.data_ptr())

        def fwd_bwd():
            glam[0] = inversion.tv_admm_unrolled_vjp_device(ctx, f.data_ptr(), m.data_ptr(), grid, (0.0, 0.0, 1.0),
                                                            1e-3, 2e-2, 50, 10, gchi.data_ptr(), chi.data_ptr(),
                                                            gf.data_ptr())

        fwd()
        # dL/dchi_K of L = ||chi_K - chi_true||^2, taken from the FP64 forward pass for both
        if gchi64 is None:
            gchi64 = (2.0 * (chi - truth)).clone()
        gchi.copy_(gchi64)
        fwd_bwd()
        res[prec] = (chi.cpu().numpy(), gf.cpu().numpy(), float(glam[0]))
        t_f = _timed(s, fwd, reps=2)
        t_fb = _timed(s, fwd_bwd, reps=2)
        out[prec] = {"forward_ms": round(t_f, 2), "forward_plus_vjp_ms": round(t_fb, 2),
                     "vjp_over_forward": round((t_fb - t_f) / t_f, 3)}
        ctx.close()
    a, b = res["mixed"], res["f64"]
    out["errors_mixed_vs_fp64_gpu"] = {"chi_K": _errs(a[0], b[0]), "dL_dfield": _errs(a[1], b[1]),
                                       "dL_dlambda_rel": abs(a[2] - b[2]) / (abs(b[2]) or 1.0)}
    return out


def bench_multi_echo(local, dev, seed=5):
    """384x384x256 at 0.6 mm, 3 T, 4 echoes (TE 4/12/20/28 ms): ellipsoid brain mask with 40
    cylinders at chi 0.3-0.6 ppm over a weak ellipsoid background.  Echo phases are the
    dipole field times TE (plus noise), magnitudes decay with T2* = 40 ms.  Times the
    magnitude-weighted linear fit with its 90th-percentile reliability mask (FP64),
    iLSQR (mixed) on the fitted field, and 1000 iterations of TGV (float32, as in the
    reference) on the wrapped 20 ms echo."""
    import torch
    import qsmgpu
    from qsmgpu import Grid, inversion, multi_echo as me
    nx, ny, nz = 384, 384, 256
    vs = (0.6, 0.6, 0.6)
    grid = Grid.new(nx, ny, nz, *vs)
    N = nx * ny * nz
    g = torch.Generator(device=dev).manual_seed(seed)
    z, y, x = torch.meshgrid(torch.arange(nz, device=dev, dtype=torch.float32),
                             torch.arange(ny, device=dev, dtype=torch.float32),
                             torch.arange(nx, device=dev, dtype=torch.float32), indexing="ij")
    cx, cy, cz = (nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2
    mask = (((x - cx) / (0.42 * nx)) ** 2 + ((y - cy) / (0.45 * ny)) ** 2 + ((z - cz) / (0.40 * nz)) ** 2) < 1
    chi = 0.02 * ((((x - cx) / (0.3 * nx)) ** 2 + ((y - cy) / (0.3 * ny)) ** 2 + ((z - cz) / (0.3 * nz)) ** 2) < 1)
    chi = chi.to(torch.float32)
    for _ in range(40):
        c = torch.rand(3, generator=g, device=dev) * 0.5 + 0.25
        c = c * torch.tensor([nx, ny, nz], device=dev, dtype=torch.float32)
        a = torch.randn(3, generator=g, device=dev)
        a = a / a.norm()
        r = 2.0 + 4.0 * torch.rand(1, generator=g, device=dev)
        length = 20.0 + 40.0 * torch.rand(1, generator=g, device=dev)
        val = 0.3 + 0.3 * torch.rand(1, generator=g, device=dev)
        px, py, pz = x - c[0], y - c[1], z - c[2]
        t = px * a[0] + py * a[1] + pz * a[2]
        d2 = (px - t * a[0]) ** 2 + (py - t * a[1]) ** 2 + (pz - t * a[2]) ** 2
        chi = torch.where((t.abs() < length / 2) & (d2 < r * r), val, chi)
    del x, y, z
    chi = (chi * mask).to(torch.float64).reshape(-1).contiguous()
    m8 = mask.reshape(-1).to(torch.uint8).contiguous()
    ctx = qsmgpu.Context(local, "f64")
    s = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    field = torch.empty_like(chi)
    inversion.dipole_forward_device(ctx, chi.data_ptr(), grid, (0.0, 0.0, 1.0), field.data_ptr())
    tes = [0.004, 0.012, 0.020, 0.028]
    w0 = 2.0 * np.pi * 42.58 * 3.0  # rad/s per ppm
    mags = torch.stack([m8.to(torch.float64) * float(np.exp(-te / 0.04)) for te in tes]).contiguous()
    noise = torch.randn(len(tes), N, generator=g, device=dev, dtype=torch.float64)
    phases = torch.stack([field * (w0 * te) for te in tes]) + 0.02 * noise / mags.clamp_min(0.05)
    phases = (phases * m8.to(torch.float64)).contiguous()
    fit_f, fit_o, fit_r = (torch.empty(N, dtype=torch.float64, device=dev) for _ in range(3))
    fit_rel = torch.empty(N, dtype=torch.uint8, device=dev)
    lp = me.LinearFitParams(True, 90.0)

    def fit():
        me.multi_echo_linear_fit_device(ctx, phases.data_ptr(), mags.data_ptr(), tes, len(tes), m8.data_ptr(), N, lp,
                                        fit_f.data_ptr(), fit_o.data_ptr(), fit_r.data_ptr(), fit_rel.data_ptr())

    fit()
    t_fit = _timed(s, fit, reps=3)
    fit_bytes = (2 * len(tes) * 8 + 1 + 3 * 8 + 1) * N
    ppm = (fit_f / w0).contiguous()
    ctx.close()
    il = inversion.IlsqrParams()
    il_out, il_ms = {}, {}
    prof_il = None
    for name, prec, kry in (("fp64", "f64", "f64"), ("mixed", "mixed", "f64"), ("mixed_float_krylov", "mixed", "mixed")):
        c = qsmgpu.Context(local, prec)
        c.krylov_precision = kry
        sc = torch.cuda.ExternalStream(c.stream_handle(), device=dev)
        o = [torch.empty_like(field) for _ in range(4)]

        def run_ilsqr():
            inversion.ilsqr_device(c, ppm.data_ptr(), m8.data_ptr(), grid, (0.0, 0.0, 1.0), il, o[0].data_ptr(),
                                   o[1].data_ptr(), o[2].data_ptr(), o[3].data_ptr())

        run_ilsqr()
        il_ms[name] = round(_timed(sc, run_ilsqr), 2)
        il_out[name] = [t.cpu().numpy() for t in o]
        if name == "mixed":
            prof_il = _profiled(c, run_ilsqr)
        c.close()
        del o
    names = ("chi", "xsa", "xfs", "xlsqr")
    il_err = {v: {k: _errs(a, b) for k, a, b in zip(names, il_out[v], il_out["fp64"])}
              for v in ("mixed", "mixed_float_krylov")}
    # the LSQR loop's passes run on full complex FP64 spectra (16 B per value) in the default mixed
    # context: Z inverse with the dipole scale reads x and writes t, the fused X pass reads t and
    # the weights and writes t, the Z forward epilogue reads t and the previous vector and writes
    sd = 16
    il_model = {"fft_z_inv": 2 * N * sd, "fft_y_inv": 2 * N * sd, "fft_y_fwd": 2 * N * sd,
                "fft_x_lsqr": 2 * N * sd + N * 8, "fft_z_lsqr": 3 * N * sd}
    il_roof = _dominant_roofline(prof_il, il_model, "LSQR passes on full complex FP64 spectra: read + write one "
                                                    "spectrum (2*N*16 B), + weights (fused X), + previous vector (Z out)")
    cm = qsmgpu.Context(local, "mixed")
    sm = torch.cuda.ExternalStream(cm.stream_handle(), device=dev)
    wrapped = torch.remainder(phases[2] + np.pi, 2 * np.pi) - np.pi
    wrapped = (wrapped * m8.to(torch.float64)).contiguous()
    tg = inversion.TgvParams(iterations=1000, tol=0.0, fieldstrength=3.0, te=0.020)
    tgv_out = torch.empty_like(field)

    def run_tgv():
        inversion.tgv_qsm_device(cm, wrapped.data_ptr(), m8.data_ptr(), grid, tg, (0.0, 0.0, 1.0), tgv_out.data_ptr())

    run_tgv()
    t_tgv = _timed(sm, run_tgv)
    tg_prof = inversion.TgvParams(iterations=20, tol=0.0, fieldstrength=3.0, te=0.020)
    prof_tgv = _profiled(cm, lambda: inversion.tgv_qsm_device(cm, wrapped.data_ptr(), m8.data_ptr(), grid, tg_prof,
                                                              (0.0, 0.0, 1.0), tgv_out.data_ptr()))
    cm.close()
    # TGV works on the bounding box (padding 2) of mask0 = erode^(erosions+1)(mask), with
    # mask_eroded = erode^erosions(mask) (6-neighbour erosion that also clears the faces)
    mk = m8.reshape(nz, ny, nx).bool()
    m_eroded = mk
    for e in range(tg.erosions + 1):
        if e == tg.erosions:
            m_eroded = mk
        pad = torch.nn.functional.pad(mk[None, None].to(torch.float32), (1, 1, 1, 1, 1, 1))[0, 0] > 0
        mk = (pad[1:-1, 1:-1, 1:-1] & pad[:-2, 1:-1, 1:-1] & pad[2:, 1:-1, 1:-1] & pad[1:-1, :-2, 1:-1] &
              pad[1:-1, 2:, 1:-1] & pad[1:-1, 1:-1, :-2] & pad[1:-1, 1:-1, 2:])
    m0 = mk
    idx = m0.nonzero()
    lo = (idx.min(0).values - 2).clamp_min(0)
    hi = torch.minimum(idx.max(0).values + 3, torch.tensor([nz, ny, nx], device=dev))
    box = lambda a: a[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
    V = int(box(m0).numel())
    V0 = int(box(m0).sum())
    Vm = int(box(m_eroded).sum())
    # bytes per box voxel: dual reads both masks and chi; inside mask0 phi, lphi, eta (r+w), q (r+w);
    # inside the eroded mask p (r+w) and w.  Primal reads both masks, phi, chi, w and writes phi, chi,
    # w twice (iterate and extrapolation); inside mask0 eta and p; inside the eroded mask q.
    tgv_model = {"tgv_dual": 6 * V + 64 * V0 + 36 * Vm, "tgv_primal": 62 * V + 16 * V0 + 24 * Vm}
    tgv_roof = _dominant_roofline(prof_tgv, tgv_model, "compulsory bytes per box voxel by mask membership: "
                                                       "dual 6 + 64 (mask0) + 36 (eroded mask), primal 62 + 16 + 24")
    return {"workload": "384x384x256 at 0.6 mm, 3 T, 4 echoes TE 4/12/20/28 ms, 40 cylinders chi 0.3-0.6 ppm; "
                        "synthetic phantom",
            "linear_fit_fp64": {"ms": round(t_fit, 3), "fit_kernel_alg_gb": round(fit_bytes / 1e9, 3),
                                "note": "ms covers the fit kernel and the reliability percentile (radix select)"},
            "ilsqr_ms": il_ms, "ilsqr_errors_vs_fp64_gpu": il_err, "ilsqr_roofline_mixed": il_roof,
            "tgv_1000_iterations_ms": round(t_tgv, 2),
            "tgv_box": {"voxels": V, "mask0": V0, "eroded_mask": Vm}, "tgv_roofline": tgv_roof,
            "tgv_note": "float32 as in the reference (src/inversion/tgv.rs); no FP64 comparator exists"}


def run_reference(args):
    """Reference arm: the reference (Rust) cannot be built here, so its CPU algorithm is
    timed through the f64 restatement in oracle/ on this host's cores, same workload.
    A step is one TV-ADMM iteration at full size (a bounded sample of the 250-iteration
    solve); the volume rate adds the one-off spectral preparation."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import qsm_oracle as O
    f, mask = make_case(0)
    cores = os.cpu_count() or 1
    O.set_fft_workers(cores)
    try:
        t_prep, per_iter = _timed_oracle_tv(f, mask, args.warmup + args.steps)
    finally:
        O.set_fft_workers(None)
    timed = per_iter[args.warmup:]
    t_iter = statistics.median(timed)
    vol_s = t_prep + ITERS * t_iter
    v = 1.0 / vol_s
    sample = (f"{args.steps} timed TV-ADMM iterations at {DIMS[0]}x{DIMS[1]}x{DIMS[2]} after {args.warmup} warm-up "
              f"(oracle port, scipy.fft workers={cores}), scaled to {ITERS} iterations + preparation "
              f"({t_prep:.2f} s)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_iter * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"tv_admm {DIMS[0]}x{DIMS[1]}x{DIMS[2]} x{ITERS} iterations",
                       "iterations": ITERS, "precision": "f64 (reference CPU arithmetic)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import qsmgpu
    from qsmgpu import Grid, inversion

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    f, mask = make_case(rank)
    N = f.size
    grid = Grid.new(*DIMS)
    bdir = (0.0, 0.0, 1.0)
    params = inversion.TvParams(2e-4, 2e-2, 0.0, ITERS)
    dev = torch.device("cuda", local)
    d_f = torch.from_numpy(f.ravel()).to(dev)
    d_m = torch.from_numpy(mask.ravel()).to(dev)
    d_out = torch.empty(N, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    ctx = qsmgpu.Context(local, "mixed")
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)

    def step():
        inversion.tv_admm_device(ctx, d_f.data_ptr(), d_m.data_ptr(), grid, bdir, params, d_out.data_ptr())

    for _ in range(max(args.warmup, 3)):
        step()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = ctx.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    clocks.mark("start")
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks.mark("stop")
    launches = ctx.kernel_launches() - l0
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    clocks.stop()
    chi_mixed = d_out.cpu().numpy().copy()
    value = world * args.steps / (ms / 1e3)
    ms_step = ms / args.steps

    # end to end through the host API: page-locked host input/output, H2D + solve + D2H
    h_f = torch.from_numpy(f.ravel()).pin_memory()
    h_m = torch.from_numpy(mask.ravel()).pin_memory()
    h_o = torch.empty(N, dtype=torch.float64).pin_memory()
    hf, hm, ho = h_f.numpy(), h_m.numpy(), h_o.numpy()
    inversion.tv_admm(hf, hm, grid, bdir, params, ctx=ctx, out=ho)
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(2, min(args.steps, 5))
    e0.record(stream)
    for _ in range(e2e_steps):
        inversion.tv_admm(hf, hm, grid, bdir, params, ctx=ctx, out=ho)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * e2e_steps / (e2e_ms / 1e3)

    # per-kernel profile (separate pass: every launch bracketed by events on the library stream)
    ctx.set_profiling(True)
    ctx.profile_reset()
    step()
    prof = ctx.profile()
    ctx.set_profiling(False)
    peak, peak_kind = measured_peak()
    model = kernel_bytes_model(N, 4)
    kernels = {}
    for name, (cnt, tot) in prof.items():
        avg = tot / max(cnt, 1)
        k = {"launches": cnt, "total_ms": round(tot, 4), "avg_us": round(avg * 1e3, 2)}
        if name in model:
            gbs = model[name] / (avg / 1e3) / 1e9
            k.update({"alg_bytes": model[name], "gbs": round(gbs, 1), "frac": round(gbs / peak, 3)})
        kernels[name] = k
    tot_all = sum(v["total_ms"] for v in kernels.values()) or 1.0
    for v in kernels.values():
        v["share"] = round(v["total_ms"] / tot_all, 3)
    dom = max((n for n in kernels if n in model), key=lambda n: kernels[n]["total_ms"])
    iter_bytes = 20 * N * 4
    traffic = ncu_traffic()
    roofline = {"bound": "hbm", "achieved": kernels[dom]["gbs"], "peak": peak, "unit": "GB/s",
                "frac": round(kernels[dom]["gbs"] / peak, 3), "traffic": traffic.get(dom), "kernel": dom,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, one capture of this "
                                  "workload" if dom in traffic else None,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                "fallback 6.65 TB/s",
                "iteration_model_gbs": round(iter_bytes / (ms_step / ITERS / 1e3) / 1e9, 1),
                "iteration_model_frac": round(iter_bytes / (ms_step / ITERS / 1e3) / 1e9 / peak, 3)}

    extra = {}
    if not args.skip_fp64:
        ctx64 = qsmgpu.Context(local, "f64")
        s64 = torch.cuda.ExternalStream(ctx64.stream_handle(), device=dev)
        d_o64 = torch.empty(N, dtype=torch.float64, device=dev)

        def step64():
            inversion.tv_admm_device(ctx64, d_f.data_ptr(), d_m.data_ptr(), grid, bdir, params, d_o64.data_ptr())

        step64()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        k64 = max(2, min(args.steps, 4))
        a0.record(s64)
        for _ in range(k64):
            step64()
        a1.record(s64)
        torch.cuda.synchronize()
        ms64 = a0.elapsed_time(a1) / k64
        chi64 = d_o64.cpu().numpy()
        err = float(np.linalg.norm(chi_mixed - chi64) / np.linalg.norm(chi64))
        extra = {"fp64_plain": {"volumes_per_s": round(1e3 / ms64, 3), "ms_per_iteration": round(ms64 / ITERS, 4)},
                 "mixed_vs_fp64_speedup": round(ms64 / ms_step, 3),
                 "rel_l2_mixed_vs_fp64": err, "max_abs_mixed_vs_fp64": float(np.abs(chi_mixed - chi64).max())}
        ctx64.close()

    if world > 1 and not args.skip_extras:
        sharded = bench_batch_sharded(local, dev, rank, world, dist)
        if rank == 0:
            extra["batch_32_volumes_sharded"] = sharded
    if rank == 0 and world == 1 and not args.skip_extras:
        extra["chain_256x256x176"] = bench_chain(local, dev)
        extra["batch_32_volumes"] = bench_batch(local, dev)
        extra["batch_4x256x256x176"] = bench_batch_brain(local, dev)
        extra["unrolled_adjoint_160x192x160"] = bench_adjoint(local, dev)
        extra["multi_echo_384x384x256"] = bench_multi_echo(local, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu_baseline:
        cpu = cpu_baseline_tv(f, mask)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": round(ms_step, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"tv_admm {DIMS[0]}x{DIMS[1]}x{DIMS[2]} x{ITERS} iterations "
                                       "(ellipsoid phantom, B0=z, TvParams default with tol=0)",
                           "dims": list(DIMS), "iterations": ITERS,
                           "precision": "mixed: f32 FFTs/stencils, f64 reductions and k-space multipliers",
                           "l2": "no flush: per-iteration working set ~0.5 GB > 126 MB L2",
                           "parallelism": f"volumes sharded over {world} rank(s), no collective"},
                "ms_per_iteration": round(ms_step / ITERS, 4),
                "roofline": roofline, "kernels": kernels,
                "e2e": {"value": round(e2e_value, 4), "unit": UNIT, "h2d_bytes_per_step": int(N * 8 + N),
                        "d2h_bytes_per_step": int(N * 8)},
                "gpu_launches": int(launches), "clocks": clocks.summary(),
                "autotune": {k: v["choice"] for k, v in ctx.autotune_entries().items()}}
        line.update(extra)
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
