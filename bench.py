#!/usr/bin/env python
"""HOOI time-to-FP64-rel-err on one B200 per rank.

Workload: the 96x96x96x96 FP32 Tucker tensor (core 16^4 N(0,1) scaled by
0.9^(i+j+k+l), QR'd Gaussian factors, noise N(0,1e-6), seed 1), HOOI ranks
16^4.  A step is one whole decomposition with X resident in HBM: X rounded
once to BF16, libc-seeded random orthonormal init, tensor-core sweeps (the
TTM chain reads X in BF16; U, the intermediates and the leaf Grams are split
hi+lo) until the sweep residual settles, FP64 subspace iteration per mode,
and the final FP64 core projection from the FP32 X -- until the relative
reconstruction error is within 1e-6 of the FP64 oracle's (checked every run).

One JSON line on rank 0:
  value        ms per decomposition (max over ranks; lower is better)
  e2e          the same through the public API from pinned host memory
               (H2D of X and D2H of G and U inside the timed region)
  fp64_gpu     the plain FP64 GPU path on the same tensor and stopping rule
  roofline     the X-streaming tensor-core TTM (the dominant kernel):
               algorithmic bytes / CUDA-event time vs measured HBM copy BW
  ttmc         sparse TTMc HBM GB/s on the 2e6 x 2e5 x 5e4 Zipf COO tensor
  cpu_baseline the reference's own HOOI_ALS (compiled from its sources, FP64,
               all host threads) on a bounded sample of the same tensor

--impl reference runs the reference's CPU HOOI instead (rank 0 only).
Multi-GPU: replicas (each rank decomposes its own copy; no collective on the
data path; barrier + max-over-ranks timing only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "HOOI time-to-FP64-rel-err (BF16-TC+FP64 vs FP64 GPU); TTMc HBM GB/s"
RANKS = (16, 16, 16, 16)
SHAPE = (96, 96, 96, 96)
TARGET = 1e-6
FALLBACK_HBM_GBS = 6650.0
# Subspace-iteration steps per mode: the FP64 drop-in keeps the reference's
# ALS_ (five); the mixed method uses two (its sweep count is unchanged here).
FP64_INNER = 5
MIXED_INNER = 2


def _log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def _oracle_residual():
    try:
        with open(os.path.join(ROOT, "tests", "golden", "large_oracle.json")) as f:
            d = json.load(f)["dense_96x4_r16"]
        return float(d["residual"]), int(d["sweeps"])
    except Exception:
        return None, None


def _oracle_core_and_factors():
    """||G|| and the factors of the reference's converged run on this tensor."""
    try:
        import numpy as np
        with open(os.path.join(ROOT, "tests", "golden", "large_oracle.json")) as f:
            g = float(json.load(f)["dense_96x4_r16"]["g_norm"])
        z = np.load(os.path.join(ROOT, "tests", "golden", "large_oracle_factors.npz"))
        return g, [z[f"dense_96x4_r16_U{n}"] for n in range(4)]
    except Exception:
        return None, None


def _principal_angle(A, B):
    """Largest principal angle between span(A) and span(B), from the sine
    ||(I - Qa Qa^T) Qb||_2 (accurate for tiny angles)."""
    import numpy as np
    qa, _ = np.linalg.qr(np.asarray(A, dtype=np.float64))
    qb, _ = np.linalg.qr(np.asarray(B, dtype=np.float64))
    s = np.linalg.norm(qb - qa @ (qa.T @ qb), 2)
    return float(np.arcsin(min(1.0, s)))


def _config(world):
    """The workload description shared by both arms (ours and --impl reference)."""
    return {
        "workload": "dense 96x96x96x96 FP32 Tucker(16^4, core*0.9^(i+j+k+l)) + N(0,1e-6), "
                    "seed 1; HOOI ranks 16^4 to the FP64 oracle's rel-err (within 1e-6)",
        "ours": "tcgen05 TTM chain reading X rounded once to BF16 (U, intermediates and "
                "leaf Grams split hi+lo BF16 / FP32), FP64 subspace iteration (2 steps per "
                "mode) / fit / final core projected from the FP32 X",
        "reference": "the reference's HOOI_ALS (compiled from its sources, FP64, all host "
                     "threads), random init, as many sweeps as its own converged run needs",
        "init": "libc-seeded Gaussian + QR (seed 1)",
        "stop": "ours: sweeps until the sweep residual changes by < 5e-6 (the noise "
                "floor of the split intermediates), then the FP64 core projection; "
                "reference: the sweep count of its converged run (residual change < 1e-9)",
        "target": f"|rel-err - FP64 oracle rel-err| <= {TARGET}",
        "l2": "inputs larger than L2 (X: 340 MB FP32, 170 MB per BF16 half; L2 126 MB)",
        "outputs": "G and U stay in HBM (CUDA tensors); e2e copies them to the host",
        "plans": "repeated calls reuse the context's cached plan and captured sweep "
                 "graphs (built in warm-up), for both the mixed and the FP64 path",
        "parallelism": f"replicas x{world} (no data-path collective)",
    }


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    polled every ~2 ms from a thread (a timed region of a few ms still gets
    samples), else nvidia-smi at 200 ms.  Reads only; changes no setting."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self.nvml = None
        self.stop_ev = threading.Event()
        self.t = None
        self.switch = sys.getswitchinterval()

    def start(self):
        # The timed region is a few ms of Python issuing graph launches; a
        # short GIL switch interval lets the polling thread run inside it.
        self.switch = sys.getswitchinterval()
        sys.setswitchinterval(0.0002)
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.nvml = (nv, h)
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _poll(self):
        nv, h = self.nvml
        while True:
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for name, const in self.REASONS:
                    if mask & getattr(nv, const):
                        self.reasons.add(name)
            except Exception:
                return
            if self.stop_ev.wait(0.002):
                return

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        sys.setswitchinterval(self.switch)
        if self.nvml is not None:
            self.stop_ev.set()
            self.t.join(timeout=5)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
            if not self.samples:
                return None
            sm = sorted(self.samples)
            return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(self.reasons), "samples": len(sm), "source": "nvml"}
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


def _dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def _max_over_ranks(v, world, device):
    """Max of v over the ranks (device None: a CPU tensor, for gloo)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64,
                     device="cpu" if device is None else f"cuda:{device}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(world, device):
    if world > 1:
        import torch
        import torch.distributed as dist
        if device is None:
            dist.barrier()
        else:
            dist.barrier(device_ids=[device])
            torch.cuda.synchronize()


def run_ours(args):
    import numpy as np
    import torch

    from diana_tucker_b200 import DT_PREC_BF16X2, DT_PREC_BF16XH, DT_PREC_FP64, Context, datasets

    world, rank, local = _dist_setup(args.gpus)
    torch.cuda.set_device(local)
    ctx = Context(local)
    # A dedicated stream: the library binds to torch's current stream, and
    # programmatic dependent launch needs a stream other than the legacy one.
    stream = torch.cuda.Stream(local)
    torch.cuda.set_stream(stream)
    X = datasets.dense_96x4_fp32()
    flat = np.ascontiguousarray(X.reshape(-1, order="F"))
    Xd = torch.from_numpy(flat).to(f"cuda:{local}")
    kw = dict(init="randn", seed=1, max_sweeps=30, tol=1e-9, shape=SHAPE)

    X64d = Xd.double()  # the FP64 drop-in takes Tensor<double>

    # Inputs and outputs stay in HBM for `value` (G and U come back as CUDA
    # tensors); `e2e` below copies them from and to the host.
    def mixed(profile=False, prec=DT_PREC_BF16XH):
        return ctx.hooi_dense(Xd, RANKS, precision=prec, profile=profile,
                              inner_iters=MIXED_INNER, device_out=True, **kw)

    def fp64(profile=False, x=X64d, inner=FP64_INNER):
        return ctx.hooi_dense(x, RANKS, precision=DT_PREC_FP64, profile=profile,
                              inner_iters=inner, device_out=True, **kw)

    # Warm-up (module loading, memory pool).
    _log("warm-up")
    for _ in range(args.warmup):
        mixed()
    _log("timed region")
    # Timed region: K whole decompositions, device time by CUDA events on the
    # stream the library runs on, max over ranks.
    clocks = ClockSampler(local)
    _barrier(world, local)
    torch.cuda.synchronize()
    clocks.start()
    l0 = ctx.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    reps = []
    for _ in range(args.steps):
        _, Ulast, rep = mixed()
        reps.append(rep)
    ev1.record()
    torch.cuda.synchronize()
    launches = ctx.kernel_launches() - l0
    clk = clocks.stop()
    _barrier(world, local)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = _max_over_ranks(ms, world, local)
    # One more decomposition with CUDA events around the X-streaming TTM
    # launches, for the roofline (outside the timed region).
    _, _, rep = mixed(profile=True)

    _log(f"mixed {ms:.3f} ms/decomposition; FP64 path")
    # FP64 GPU path, same tensor and stopping rule, timed the same way (CUDA
    # events around whole calls): X stored in FP64 (the drop-in's
    # Tensor<double>) and, for reference, FP64 arithmetic reading the
    # FP32-stored X.
    def bracket(fn, n):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            _, _, r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, r

    n64 = max(1, min(args.steps, 3))
    fp64_ms, r64 = bracket(fp64, n64)
    fp64_x32_ms, _ = bracket(lambda: fp64(x=Xd), n64)
    fp64_in2_ms, r64b = bracket(lambda: fp64(inner=MIXED_INNER), n64)
    # The mixed method with X kept as hi + lo in every pass (always split).
    x2_ms, rx2 = bracket(lambda: mixed(prec=DT_PREC_BF16X2), n64)
    del X64d

    _log("end to end from pinned host memory")
    # End to end through the public API from pinned host memory.
    Xh = torch.from_numpy(flat).pin_memory()
    e2e_t = []
    for i in range(max(1, min(args.steps, 3)) + 1):
        t0 = time.perf_counter()
        G, U, _ = ctx.hooi_dense(Xh, RANKS, precision=DT_PREC_BF16XH, inner_iters=MIXED_INNER,
                                 **kw)
        dt = (time.perf_counter() - t0) * 1e3
        if i > 0:
            e2e_t.append(dt)
    e2e_ms = _max_over_ranks(float(np.median(e2e_t)), world, local)
    # The bare copy of the same pinned X to the device, timed the same way:
    # the floor of `e2e` (every sweep needs all of X; only the rounding of X
    # to BF16 runs under the copy, chunk by chunk).
    Xcopy = torch.empty_like(Xd)
    h2d_t = []
    for i in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Xcopy.copy_(Xh, non_blocking=True)
        torch.cuda.synchronize()
        if i > 0:
            h2d_t.append((time.perf_counter() - t0) * 1e3)
    h2d_ms = float(np.median(h2d_t))
    del Xcopy
    h2d = flat.nbytes
    d2h = int(np.prod(RANKS)) * 8 + sum(s * r * 8 for s, r in zip(SHAPE, RANKS))

    oracle_res, oracle_sweeps = _oracle_residual()
    ref_res = oracle_res if oracle_res is not None else r64["residual"]
    err = abs(rep["residual"] - ref_res)
    # The last timed decomposition against the reference's converged run:
    # core norm and the largest principal angle per mode.
    oracle_g, oracle_U = _oracle_core_and_factors()
    g_gap = abs(rep["g_norm"] - oracle_g) / oracle_g if oracle_g else None
    angles = ([_principal_angle(Ulast[n].cpu().numpy(), oracle_U[n]) for n in range(4)]
              if oracle_U else None)

    peak, peak_kind = _peaks()
    per_launch_ms = rep["ttm_x_ms"] / max(1, rep["ttm_x_launches"])
    per_launch_bytes = rep["ttm_x_bytes"] / max(1, rep["ttm_x_launches"])
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            traffic = json.load(f).get("tc_ttm_kernel_x_bf16_per_launch_bytes")
    except Exception:
        pass

    out = {
        "metric": METRIC,
        "value": round(ms, 4),
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 4),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16",
        "data": "synthetic (seeded Tucker tensor, generated in-process)",
        "config": _config(world),
        "rel_err": rep["residual"],
        "rel_err_oracle": ref_res,
        "rel_err_gap": err,
        "target_met": bool(err <= TARGET),
        "g_norm_rel_gap": g_gap,
        "principal_angles_vs_oracle": angles,
        "sweeps": rep["sweeps"],
        "fp64_gpu": {"ms": round(fp64_ms, 4), "rel_err": r64["residual"], "sweeps": r64["sweeps"],
                     "x_dtype": "f64",
                     "speedup_mixed_vs_fp64": round(fp64_ms / ms, 3) if ms > 0 else None,
                     "inner_iters": FP64_INNER,
                     "ms_x_f32": round(fp64_x32_ms, 4),
                     "speedup_mixed_vs_fp64_x_f32": round(fp64_x32_ms / ms, 3) if ms > 0 else None,
                     "ms_inner_iters_2": round(fp64_in2_ms, 4),
                     "sweeps_inner_iters_2": r64b["sweeps"],
                     "speedup_mixed_vs_fp64_inner_iters_2":
                         round(fp64_in2_ms / ms, 3) if ms > 0 else None},
        "mixed_always_split": {"ms": round(x2_ms, 4), "rel_err": rx2["residual"],
                               "rel_err_gap": abs(rx2["residual"] - ref_res),
                               "sweeps": rx2["sweeps"],
                               "what": "X read as split hi+lo BF16 in every pass (4 B per "
                                       "element) instead of BF16 hi only (2 B)"},
        "decompositions_per_s": round(world * 1000.0 / ms, 3) if ms > 0 else None,
        # Each timed call's own device time (library events from its first to
        # its last kernel): `value` minus this is the host time between calls.
        "device_ms_per_call": {
            "median": round(float(np.median([r["device_ms"] for r in reps])), 4),
            "min": round(float(min(r["device_ms"] for r in reps)), 4),
            "max": round(float(max(r["device_ms"] for r in reps)), 4)} if reps else None,
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "h2d_bare_ms": round(h2d_ms, 4),
                "h2d_bare_gbs": round(h2d / h2d_ms / 1e6, 1) if h2d_ms > 0 else None,
                "above_bare_h2d_ms": round(e2e_ms - h2d_ms, 4),
                "overlap": "X copied in 4 chunks on a copy stream, issued first; each chunk rounded to "
                           "BF16 (and summed into ||X||^2) as it lands; the sweeps need "
                           "all of X"},
        "gpu_launches": int(launches // max(1, args.steps)),
        "gpu_launches_timed_region": int(launches),
        "roofline": {"kernel": "tc_ttm_kernel (X x_n U^T, BF16 X streamed by TMA, U split)",
                     "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if peak else None,
                     "traffic": traffic,
                     "algorithmic_bytes_per_launch": per_launch_bytes,
                     "launch_ms": per_launch_ms, "launches_per_step": rep["ttm_x_launches"]},
    }
    if clk:
        out["clocks"] = clk
    if args.ttmc and world == 1:
        _log("sparse TTMc")
        out["ttmc"] = _ttmc(ctx, peak, args.ttmc_draws, args.cpu and rank == 0)
    if args.cfg1 and world == 1:
        _log("200^3 FP64 HOOI")
        out["dense_200cube"] = _cfg1(ctx, args.steps, args.cpu and rank == 0)
    if args.batched and world == 1:
        _log("batched HOOI (4096 small tensors)")
        out["batched"] = _batched(ctx, args.steps, args.cpu and rank == 0)
    if args.warmstart and world == 1:
        _log("learned warm start")
        out["warmstart"] = _warmstart(ctx, args.ws_train, args.ws_eval)
    if rank == 0 and world == 1 and args.cpu:
        _log("CPU baseline (reference HOOI_ALS)")
        out["cpu_baseline"] = _cpu_baseline(X, oracle_sweeps or r64["sweeps"])
    _log("done")
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def _ttmc(ctx, peak, draws=50_000_000, cpu=False):
    """Sparse TTMc bandwidth on the 2,000,000 x 200,000 x 50,000 COO tensor
    (50M Zipf(1.1) draws, merged; fewer with --ttmc-draws), ranks 16^3: one
    sparse HOOI sweep with the TTMc launches timed by CUDA events; then the
    configured sparse HOOI (random orthonormal init, 10 sweeps) timed whole,
    and, with cpu, one sweep of the C restatement of the reference's sparse
    HOOI (OpenMP, all host threads) from the same start, checked against the
    GPU's one-sweep residual."""
    from diana_tucker_b200 import datasets
    t0 = time.time()
    if draws == 50_000_000:
        idx, vals, shape = datasets.sparse_2m_200k_50k()
    else:
        idx, vals, shape = datasets.sparse_zipf((2_000_000, 200_000, 50_000), draws, alpha=1.1,
                                                seed=2)
    gen_s = time.time() - t0
    sp = ctx.sptensor(idx, vals, shape)
    R = (16, 16, 16)
    Ut = datasets.random_orthonormal_transposed(shape, R, 2)
    sp.hooi(R, 1, Ut)
    _, _, rep = sp.hooi(R, 1, Ut)
    gbs = rep["ttm_x_bytes"] / (rep["ttm_x_ms"] * 1e-3) / 1e9 if rep["ttm_x_ms"] else 0.0
    # The same launches against the per-mode figure of the COO format the
    # reference reads (int64 indices + FP64 value = 32 B per nonzero, each other
    # factor once, the non-empty Y_(n) rows written): nnz*32 + sum_{m!=n} I_m R_m 8
    # + rows_n * P * 8, summed over the 3 modes.
    import numpy as np
    rows = [int(np.unique(i).size) for i in idx]
    coo = 0.0
    for n in range(3):
        coo += len(vals) * 32.0 + rows[n] * 256 * 8.0
        coo += sum(shape[m] * R[m] * 8.0 for m in range(3) if m != n)
    coo_gbs = coo / (rep["ttm_x_ms"] * 1e-3) / 1e9 if rep["ttm_x_ms"] else 0.0
    # Every nonzero also gathers one 128-byte row of its element-mode factor
    # (and every fibre one of its fibre-mode factor) through L2: a lower bound
    # of that traffic is nnz * 128 B per mode.
    gather = float(len(vals)) * 3 * (16 * 8)
    eff = (rep["ttm_x_bytes"] + gather) / (rep["ttm_x_ms"] * 1e-3) / 1e9 if rep["ttm_x_ms"] else 0.0
    # The configured run: 10 sweeps from the same random orthonormal start.
    sp.hooi(R, 10, Ut)
    _, _, rep10 = sp.hooi(R, 10, Ut)
    hooi10 = {"ms": round(rep10["device_ms"], 3), "sweeps": 10,
              "ms_per_sweep": round(rep10["device_ms"] / 10, 3),
              "rel_err": rep10["residual"],
              "workload": "sparse HOOI ranks 16^3, random orthonormal init (seed 2), 10 sweeps"}
    sp.close()
    if cpu:
        from oracle import sparse as osp
        t1 = time.perf_counter()
        _, _, res_cpu = osp.hooi(idx, vals, shape, R, 1, Ut)
        cpu_ms = (time.perf_counter() - t1) * 1e3
        hooi10["cpu_baseline"] = {
            "value": round(cpu_ms, 1), "unit": "ms per sweep", "kind": "port",
            "cores": os.cpu_count(), "cpu_model": _cpu_model(),
            "sample": "one sweep of the C restatement of the reference's sparse HOOI "
                      "(sp_hooi_als.tpp:67-118; OpenMP over rows) on the whole tensor from the "
                      "same start; the GPU figure to compare is ms_per_sweep",
            "rel_err_1_sweep": res_cpu, "gpu_rel_err_1_sweep": rep["residual"],
            "rel_err_gap_1_sweep": abs(res_cpu - rep["residual"])}
    return {"value": round(gbs, 1), "unit": "GB/s", "frac_of_hbm": round(gbs / peak, 4),
            "bytes_def": "fibre layout read (12 B/nonzero + 8 B/fibre slot) + Y rows written "
                         "+ factors",
            "nnz": int(len(vals)), "rows_per_mode": rows, "launches": rep["ttm_x_launches"],
            "ms": rep["ttm_x_ms"], "bytes": rep["ttm_x_bytes"],
            "coo_bytes": coo, "coo_gbs": round(coo_gbs, 1),
            "coo_frac_of_hbm": round(coo_gbs / peak, 4),
            "gather_bytes_lower_bound": gather, "with_gathers_gbs": round(eff, 1),
            "sweep_ms": rep["device_ms"], "gen_s": round(gen_s, 1), "hooi": hooi10}


def _cfg1(ctx, steps, cpu):
    """The 200x200x200 FP64 Tucker tensor (core 10^3, noise N(0,1e-4), seed 0):
    plain FP64 HOOI, ranks (10,10,10), HOSVD init, <= 25 sweeps or a residual
    change < 1e-8 -- on the GPU (device events, X resident; and end to end from
    host memory) and, with cpu, the reference's own HOOI sweep (Function::ttm +
    ALS_ with the same HOSVD init and stop rule, compiled from its sources,
    all host threads)."""
    import numpy as np
    import torch

    from diana_tucker_b200 import DT_PREC_FP64, datasets
    X = datasets.dense_200cube_fp64()
    flat = np.ascontiguousarray(X.reshape(-1, order="F"))
    Xd = torch.from_numpy(flat).to(f"cuda:{ctx.device}")
    kw = dict(init="hosvd", max_sweeps=25, tol=1e-8, precision=DT_PREC_FP64, shape=X.shape)
    for _ in range(3):
        ctx.hooi_dense(Xd, (10, 10, 10), device_out=True, **kw)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = max(3, steps)
    e0.record()
    for _ in range(n):
        _, _, rep = ctx.hooi_dense(Xd, (10, 10, 10), device_out=True, **kw)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    Xh = torch.from_numpy(flat).pin_memory()
    t = []
    for _ in range(3):
        t0 = time.perf_counter()
        ctx.hooi_dense(Xh, (10, 10, 10), **kw)
        t.append((time.perf_counter() - t0) * 1e3)
    try:
        with open(os.path.join(ROOT, "tests", "golden", "large_oracle.json")) as f:
            oref = json.load(f)["dense_200cube_r10"]["residual"]
    except Exception:
        oref = None
    out = {"ms": round(ms, 3), "e2e_ms": round(float(np.median(t)), 3), "sweeps": rep["sweeps"],
           "rel_err": rep["residual"], "rel_err_oracle": oref,
           "rel_err_gap": abs(rep["residual"] - oref) if oref is not None else None,
           "h2d_bytes": int(flat.nbytes),
           "workload": "200^3 FP64 Tucker(10^3) + N(0,1e-4), seed 0; FP64 HOOI ranks 10^3, "
                       "HOSVD init, <= 25 sweeps or residual change < 1e-8"}
    if cpu:
        from oracle import ref
        if ref.available():
            ref.hooi_harness(X, (10, 10, 10), 25, 1e-8)
            t0 = time.perf_counter()
            _, _, hist = ref.hooi_harness(X, (10, 10, 10), 25, 1e-8)
            cms = (time.perf_counter() - t0) * 1e3
            out["cpu_baseline"] = {
                "value": round(cms, 1), "unit": "ms", "kind": "reference",
                "cores": os.cpu_count(), "cpu_model": _cpu_model(), "rel_err": hist[-1],
                "sweeps": len(hist),
                "sample": "the whole decomposition: the reference's Function::gram + dsyevd "
                          "HOSVD init and its Function::ttm + ALS_ sweeps (hooi_als.tpp:94-114) "
                          "to the same stop rule, FP64, all OpenMP/OpenBLAS threads"}
    del Xd
    return out


def _ref_batched_worker(args):
    """One spawned process: the reference's stock HOOI_ALS (random init,
    `sweeps` sweeps, FP64) on a chunk of the small tensors; returns seconds."""
    chunk, sweeps = args
    import numpy as np
    from oracle import ref
    # The reference prints its progress on stderr, 13 lines per call: 4096
    # calls' worth is discarded here (an exception still reaches the parent).
    os.dup2(os.open(os.devnull, os.O_WRONLY), 2)
    t0 = time.perf_counter()
    for X, r in chunk:
        ref.hooi_als(np.asarray(X, dtype=np.float64), r, sweeps, seed=1)
    return time.perf_counter() - t0


def _batched(ctx, steps, cpu):
    """The batched workload: 4096 independent 3-way FP32 Tucker tensors (modes
    U[8,64], ranks U[2,8], noise N(0,1e-4), seed 3), HOOI with 10 sweeps of
    five ALS_ steps each from seeded random orthonormal factors, all in one
    persistent graph-launched kernel.  `ms` is the launch's CUDA-event time
    with X, U and G resident; `e2e_ms` the same call from host numpy arrays
    (X, U staged in, U, G and the errors copied back)."""
    import multiprocessing as mp

    import numpy as np
    import torch

    from diana_tucker_b200 import datasets
    t0 = time.time()
    items = datasets.batched_small(count=4096, seed=3)
    rng = np.random.default_rng(103)
    U0 = [[np.linalg.qr(rng.standard_normal((X.shape[n], r[n])))[0] for n in range(3)]
          for X, r in items]
    tensors = [X for X, _ in items]
    ranks = [r for _, r in items]
    pk = ctx.pack_batched(tensors, ranks, U0)
    gen_s = time.time() - t0
    dev = torch.device("cuda", ctx.device)
    Xd = torch.from_numpy(pk["X"]).to(dev)
    U0d = torch.from_numpy(pk["U"]).to(dev)
    Ud = U0d.clone()
    Gd = torch.zeros(pk["g_size"], dtype=torch.float64, device=dev)
    Ed = torch.zeros(pk["count"], dtype=torch.float64, device=dev)
    kw = dict(sweeps=10, inner_iters=5, block_threads=0)
    first = ctx.hooi_batched_packed(pk, Ud, Gd, Ed, X=Xd, **kw)  # autotunes, builds the graph
    ms = []
    for _ in range(max(3, steps)):
        Ud.copy_(U0d)
        rep = ctx.hooi_batched_packed(pk, Ud, Gd, Ed, X=Xd, **kw)
        ms.append(rep["device_ms"])
    v = float(np.median(ms))
    relerr = Ed.cpu().numpy()
    # End to end from host memory through the same entry point.
    Uh = pk["U"].copy()
    Gh = np.zeros(pk["g_size"])
    Eh = np.zeros(pk["count"])
    e2e = []
    for _ in range(2):
        Uh[:] = pk["U"]
        t1 = time.perf_counter()
        ctx.hooi_batched_packed(pk, Uh, Gh, Eh, **kw)
        e2e.append((time.perf_counter() - t1) * 1e3)
    xbytes = float(pk["X"].nbytes)
    out = {"ms": round(v, 3), "unit": "ms", "tensors": pk["count"],
           "decompositions_per_s": round(pk["count"] / (v * 1e-3), 1),
           "x_bytes": xbytes, "x_read_once_gbs": round(xbytes / (v * 1e-3) / 1e9, 1),
           "x_passes": 2 * 10,
           "block_threads": rep["block_threads"], "pack": rep["pack"], "items": rep["items"],
           "grid": rep["grid"], "autotune": {"candidates": first["candidates_timed"],
                                            "best_ms": round(first["tune_best_ms"], 3),
                                            "worst_ms": round(first["tune_worst_ms"], 3)},
           "graph_reused": rep["graph_reused"],
           "e2e_ms": round(float(np.median(e2e)), 3),
           "e2e_h2d_bytes": int(xbytes + pk["U"].nbytes),
           "e2e_d2h_bytes": int(pk["U"].nbytes + 8 * (pk["g_size"] + pk["count"])),
           "relerr_max": float(relerr.max()), "relerr_mean": float(relerr.mean()),
           "gen_s": round(gen_s, 1),
           "workload": "4096 x 3-way FP32, modes U[8,64], ranks U[2,8], noise var 1e-4, seed 3; "
                       "10 HOOI sweeps x 5 ALS_ steps from seeded orthonormal factors, FP64"}
    if cpu:
        os.environ.setdefault("OMP_NUM_THREADS", "1")
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        nproc = os.cpu_count() or 1
        chunks = [([items[t] for t in range(i, len(items), nproc)], 10) for i in range(nproc)]
        t1 = time.perf_counter()
        with mp.get_context("spawn").Pool(nproc) as pool:
            secs = pool.map(_ref_batched_worker, chunks)
        wall = (time.perf_counter() - t1) * 1e3
        out["cpu_baseline"] = {
            "value": round(wall, 1), "unit": "ms", "kind": "reference", "cores": nproc,
            "cpu_model": _cpu_model(),
            "sample": f"all 4096 tensors: the reference's stock HOOI_ALS(X, R, 10) per tensor "
                      f"(FP64), {nproc} spawned processes of one thread each; wall time incl. "
                      f"process start-up (sum of per-process compute {sum(secs):.1f} s)"}
    del Xd, U0d, Ud, Gd, Ed
    return out


def _warmstart(ctx, n_train, n_eval):
    """Learned warm start on the 256^3 Chebyshev family: train on seeds
    1000.., evaluate on held-out seeds 2000.. against HOSVD init."""
    from diana_tucker_b200 import warmstart
    t0 = time.time()
    model = warmstart.train(ctx, range(1000, 1000 + n_train))
    t_train = time.time() - t0
    models = {k: warmstart.ablation_model(model, k) for k in ("random", "chebyshev")}
    rows = warmstart.evaluate(ctx, range(2000, 2000 + n_eval), model, models=models)
    s = warmstart.summarize(rows)
    s.update(train_tensors=n_train, eval_tensors=n_eval, k=model["k"],
             loss_first=float(model["loss"][0]), loss_last=float(model["loss"][-1]),
             train_wall_s=round(t_train, 2), network_train_s=round(model["train_s"], 3),
             target="converged FP64 rel-err + 1e-6 (strict: + 1e-9)",
             ablation_note="random: untrained orthonormal decoder; chebyshev: fixed basis of "
                           "the first k Chebyshev polynomials; both through the same sketch "
                           "pipeline and screening floor",
             workload="256^3 FP32, Chebyshev(deg<=23) x Gaussian 24x12 factors, core 12^3 "
                      "N(0,1)*exp(-0.15(i+j+k)), noise var 1e-5; ranks 12^3")
    return s


def _cpu_baseline(X32, sweeps):
    """The reference's HOOI_ALS (compiled from its sources with a size-1 MPI
    shim and OpenBLAS; all host threads) on the same tensor upcast to FP64:
    one stock call of `sweeps` sweeps (random init, the sweeps its converged
    run needs), about 20 s of CPU work."""
    import numpy as np
    from oracle import ref
    if not ref.available():
        return {"value": None, "unit": "ms", "kind": "reference", "cores": os.cpu_count(),
                "sample": "unavailable: oracle/_ref/libdiana_ref.so not built"}
    X = X32.astype(np.float64)
    t0 = time.perf_counter()
    gn, xn = ref.hooi_als_mt(X, RANKS, sweeps, 1, 0)
    ms = (time.perf_counter() - t0) * 1e3
    res = float(np.sqrt(max(0.0, 1.0 - gn * gn / (xn * xn))))
    return {"value": round(ms, 1), "unit": "ms", "kind": "reference",
            "cores": os.cpu_count(), "cpu_model": _cpu_model(),
            "rel_err": res,
            "sample": f"one stock HOOI_ALS(X, 16^4, {sweeps}) call on the whole 96^4 tensor "
                      f"(FP64, {os.cpu_count()} OpenMP threads + OpenBLAS threads)"}


def run_reference(args):
    """The reference's own CPU HOOI on the same workload (rank 0 only): each
    step is one stock HOOI_ALS(X, R, sweeps) call on the whole tensor with all
    host threads, `sweeps` being its own converged run's sweep count."""
    import numpy as np
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from diana_tucker_b200 import datasets
    from oracle import ref
    oracle_res, sweeps = _oracle_residual()
    sweeps = sweeps or 3
    if not ref.available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libdiana_ref.so was not built"}))
        return
    X = datasets.dense_96x4_fp32().astype(np.float64)
    _log(f"reference: {args.warmup} warm-up + {args.steps} timed HOOI_ALS calls "
         f"({sweeps} sweeps each)")
    for _ in range(args.warmup):
        ref.hooi_als_mt(X, RANKS, sweeps, 1, 0)
    t, res = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        gn, xn = ref.hooi_als_mt(X, RANKS, sweeps, 1, 0)
        t.append((time.perf_counter() - t0) * 1e3)
        res.append(float(np.sqrt(max(0.0, 1.0 - gn * gn / (xn * xn)))))
    v = float(np.mean(t))
    gap = max(abs(r - oracle_res) for r in res) if oracle_res is not None else None
    sample = (f"each step: one stock HOOI_ALS(X, 16^4, {sweeps}) call on the whole tensor "
              f"(random init, {sweeps} sweeps, FP64), {os.cpu_count()} OpenMP threads + "
              f"OpenBLAS threads; value = mean over the timed calls")
    out = {
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Tucker tensor, generated in-process)",
        "config": _config(world),
        "rel_err": res[-1] if res else None, "rel_err_oracle": oracle_res,
        "rel_err_gap": gap, "target_met": bool(gap is not None and gap <= TARGET),
        "step_ms": [round(x, 1) for x in t],
        "cpu_baseline": {"value": round(v, 1), "unit": "ms", "kind": "reference",
                         "cores": os.cpu_count(), "cpu_model": _cpu_model(), "sample": sample},
        "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-ttmc", dest="ttmc", action="store_false")
    ap.add_argument("--no-cpu", dest="cpu", action="store_false")
    ap.add_argument("--no-warmstart", dest="warmstart", action="store_false")
    ap.add_argument("--no-batched", dest="batched", action="store_false")
    ap.add_argument("--no-cfg1", dest="cfg1", action="store_false")
    ap.add_argument("--ttmc-draws", type=int, default=50_000_000,
                    help="Zipf draws of the sparse tensor (50M is the configured workload)")
    ap.add_argument("--ws-train", type=int, default=1500,
                    help="warm-start training tensors (the family's split: 1500)")
    ap.add_argument("--ws-eval", type=int, default=500,
                    help="warm-start held-out tensors (the family's split: 500)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
