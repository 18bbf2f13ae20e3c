#!/usr/bin/env python3
"""Benchmark of the fused ZODA column extension on B200.

One step = one extension of a full data square that is already resident in
HBM: row-major [side][side*128] u32 BabyBear (512-byte shares) -> row-major
[2*side][side*128]. The default workload is the 4096x4096 square, the largest
configuration that fits one GPU (8 GiB in, 16 GiB out, both far larger than
the 126 MB L2, so no flush is needed between steps); the 1024 and 2048 squares
are reported beside it with the same fields. Metric: payload Gb/s =
side^2 * 512 * 8 / t / 1e9, the reference's definition
(src/benchmarks/celestia_squares.rs:71-85). The output of the last timed step
is checked in full: the RLC check of every encoded row on the device, with
coefficients from the SHA-256 data root of the encoded rows.

Lines printed by rank 0 (one JSON object):
  --impl ours       (default) the CUDA library through its C ABI
  --impl reference  the reference's CPU path (its NTT restated in C,
                    oracle/zoda_oracle.c) on the host cores, per step a bounded
                    column sample of the same square

Multi-GPU (torchrun): every rank encodes its own square on its own GPU with
no collective on the data path (columns are independent); value is the total
payload of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for sub in ("zoda-cu_b200", "oracle"):
    sys.path.insert(0, os.path.join(ROOT, sub))

P = 2013265921
SHARE_U32 = 128
METRIC = "encode payload Gb/s"


def payload_bits(side: int) -> float:
    return side * side * 512 * 8.0


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def ncu_traffic(kernel_key: str):
    """Per-launch DRAM bytes of the kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    v = d.get(kernel_key)
    return None if v is None else float(v.get("dram_bytes_per_launch"))


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU)
# ---------------------------------------------------------------------------

def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's value (every rank gets it). NCCL needs a CUDA tensor; gloo takes CPU."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, side: int, ms_max: float, steps: int) -> float:
    """Whole-job payload Gb/s: every rank encodes one side x side square per step (weak scaling),
    timed by the slowest rank."""
    return world * payload_bits(side) / (ms_max / steps * 1e-3) / 1e9


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU baseline: the reference's CPU path restated (oracle/zoda_oracle.c)
# ---------------------------------------------------------------------------

def cpu_port_rate(side: int, budget_s: float, seed: int = 1, threads: int = 0) -> dict:
    """Gb/s of the oracle port on a bounded column sample of the side x side square
    (columns are independent, so a sample of them costs its share of the full square),
    on `threads` host threads (0: all of them)."""
    import oracle as O
    cols = side * SHARE_U32
    threads = threads or O.num_threads()
    # calibrate on a small window, then size the sample to the budget
    probe = max(4, min(cols, 16 * threads))
    src = O.seeded_input(side, probe, seed=seed)
    t0 = time.perf_counter()
    O.encode_rowmajor(src, threads=threads)
    dt = time.perf_counter() - t0
    ncols = int(min(cols, max(probe, probe * budget_s / max(dt, 1e-6))))
    ncols -= ncols % 4
    src = O.seeded_input(side, ncols, seed=seed)
    t0 = time.perf_counter()
    O.encode_rowmajor(src, threads=threads)
    dt = time.perf_counter() - t0
    frac = ncols / cols
    gbps = payload_bits(side) * frac / dt / 1e9
    return {"value": round(gbps, 4), "unit": "Gb/s", "cores": threads, "kind": "port",
            "sample": f"{ncols} of {cols} columns of the {side}x{side} square ({100 * frac:.2f}%), "
                      f"{dt:.2f} s on {threads} threads, oracle/zoda_oracle.c (src/ntt/cpu.rs restated)",
            "seconds": round(dt, 3)}


def run_reference(args, world, rank):
    if rank != 0:
        return
    side = args.side
    rates = []
    per_step_budget = args.ref_step_budget or max(2.0, min(20.0, 60.0 / max(1, args.steps + args.warmup)))
    for i in range(args.warmup + args.steps):
        r = cpu_port_rate(side, per_step_budget, seed=1 + i)
        if i >= args.warmup:
            rates.append(r)
    value = statistics.median(r["value"] for r in rates)
    last = rates[-1]
    t_step = payload_bits(side) / (value * 1e9) * 1e3
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gb/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_step, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded uniform in [0,p))",
        "config": workload_config(side),
        "cpu_baseline": {"value": value, "unit": "Gb/s", "cores": last["cores"], "kind": "port",
                         "sample": last["sample"] + "; ms_per_step extrapolated to the full square"},
        "e2e": {"value": value, "unit": "Gb/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def kernel_name(side: int, plan: dict | None = None) -> str:
    """The kernel zoda_extend_device launches for this side under `plan` (default plan if None)."""
    ls = side.bit_length() - 1
    tma = plan["impl"] == 2 if plan else 7 <= ls <= 11
    if tma:
        return f"k_extend_tma<{ls}>"
    return f"k_extend<{ls},{plan['sched'] if plan else 0}>"


def tune(ctx, side: int, cols: int, reps: int = 3) -> dict:
    """Autotune one side at the workload's own column count (zoda_autotune) and return the plan it installed."""
    return ctx.autotune(side, side, cols, reps)[side]


def time_extend_leg(ctx, side: int, cols: int, steps: int, warmup: int) -> dict:
    """`steps` timed extensions of a [side][cols] slab (a small case of the full square's kernel, for
    profiling), its output checked in full."""
    ms, _, check = time_device_extend(ctx, side, steps, warmup, 1, cols=cols)
    t = ms / steps
    return {"side": side, "cols": cols, "ms_per_step": round(t, 4),
            "ps_per_element": round(t * 1e9 / (side * cols), 3),
            "hbm_frac": round(12.0 * side * cols / (t * 1e-3) / 1e9 / measured_peaks()["hbm_gbs"], 4),
            "check_mismatches": check["check_mismatches"], "even_rows_equal_data": check["even_rows_equal_data"]}


def footprint_sweep(ctx, side: int, reps: int = 5) -> list:
    """Time per element of the side's extension against its footprint (input + output bytes): the same
    kernel and tiles on 1/32 .. all of the square's columns. A time per element that grows with the
    footprint at a fixed per-element work points at address translation, not arithmetic or bandwidth."""
    import torch
    full = side * SHARE_U32
    out = []
    for div in (32, 16, 8, 4, 2, 1):
        cols = full // div
        ms, _, _ = time_device_extend(ctx, side, reps, 2, 1, verify=False, cols=cols)
        t = ms / reps
        out.append({"cols": cols, "footprint_gb": round(12.0 * side * cols / 1e9, 2), "ms": round(t, 4),
                    "ps_per_element": round(t * 1e9 / (side * cols), 3)})
        torch.cuda.empty_cache()
    return out


def time_long_leg(ctx) -> dict:
    """The long-column (four-step) path: the reference's validated configurations (k = n = 32768
    and 65536 on 1024 columns, src/benchmarks/zoda_validated.rs:105-126) device-resident; a
    131072-point cuda_ntt on host buffers beside the reference's own CUDA kernel on the same
    call; and the four-step plan at the full 4096 square in each launch shape."""
    import ctypes
    import numpy as np
    import torch
    import zoda_b200
    out = {}
    for k in (32768, 65536):
        cols = 1024
        ms, _, check = time_device_extend(ctx, k, 5, 3, 1, cols=cols)
        t = ms / 5
        out[f"encode_k{k}_cols{cols}"] = {
            "ms": round(t, 4), "payload_gbps": round(k * cols * 4 * 8 / (t * 1e-3) / 1e9, 1),
            "hbm_frac_of_12B": round(12.0 * k * cols / (t * 1e-3) / 1e9 / measured_peaks()["hbm_gbs"], 4),
            "check_mismatches": check["check_mismatches"]}
    n, polys = 1 << 17, 1024  # one 131072-point transform of each of 1024 columns (512 MiB), host buffers
    vals = np.random.default_rng(1).integers(0, P, polys * n, dtype=np.uint32)
    sq = zoda_b200.PinnedSquare(n, polys)
    sq.array[:] = vals
    zoda_b200.ntt_cuda(sq, n, n)
    t0 = time.perf_counter()
    for _ in range(3):
        zoda_b200.ntt_cuda(sq, n, n)
    ours = (time.perf_counter() - t0) / 3
    res = {"n": n, "polys": polys, "ours_ms": round(ours * 1e3, 2)}
    so = os.path.join(ROOT, "oracle", "_ref", "libntt_cuda_ref.so")
    if os.path.exists(so):
        ref = ctypes.CDLL(so)
        ref.cuda_ntt.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_uint32] * 3
        import oracle as O
        roots = O.roots_of_unity(n)
        sq.array[:] = vals
        a = sq.array.copy()
        zoda_b200.ntt_cuda(sq, n, n)
        ref.cuda_ntt(a.ctypes.data, roots.ctypes.data, n, polys, n)
        b = sq.array.copy()
        sq.array[:] = a
        t0 = time.perf_counter()
        for _ in range(2):
            ref.cuda_ntt(sq.array.ctypes.data, roots.ctypes.data, n, polys, n)
        res["reference_ms"] = round((time.perf_counter() - t0) / 2 * 1e3, 2)
        res["same_result"] = bool(np.array_equal(a, b))
    sq.free()
    out["cuda_ntt_131072"] = res
    for side in (1024, 2048, 4096):
        cols = side * SHARE_U32
        shapes = {}
        # three launches over the square, the same with cp.async-staged tiles, or one
        # pipelined launch chunk by chunk
        for form, (sched, blocked) in (("three_launches", (0, 0)), ("staged", (1, 0)), ("pipelined", (0, 1))):
            for radix, ctas in ((16, 1), (16, 2), (8, 2), (8, 4)):
                if form == "staged" and ctas == 1:
                    continue
                ctx.plan_set(side, {"impl": 3, "sched": sched, "l2_promo": 3, "blocked": blocked, "stagger": 1,
                                    "radix": radix, "ctas": ctas})
                ms, _, check = time_device_extend(ctx, side, 5, 2, 1, verify=(radix, ctas) == (8, 2), cols=cols)
                shapes[f"{form}_radix{radix}_ctas{ctas}"] = {
                    "ms": round(ms / 5, 4), "check_mismatches": check["check_mismatches"] if check else None}
                torch.cuda.empty_cache()
        ctx.plan_clear()
        out[f"fourstep_side{side}"] = shapes
    return out


def time_recover(ctx, k: int, reps: int = 5, seed: int = 3) -> dict:
    """k-of-2k erasure recovery (zoda_recover_device) of a [2k][128k] extension with a seeded random half of
    the rows erased, device-resident; payload = the recovered k x k square of 512-byte shares."""
    import torch
    import numpy as np
    cols = k * SHARE_U32
    gen = torch.Generator(device="cuda").manual_seed(4321)
    d_in = torch.randint(0, P, (k, cols), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    code = torch.empty((2 * k, cols), dtype=torch.int32, device="cuda")
    ctx.extend(d_in, code, k, cols)
    known = np.sort(np.random.default_rng(seed).choice(2 * k, size=k, replace=False))
    out = torch.empty((k, cols), dtype=torch.int32, device="cuda")
    ctx.recover(code, known, k, cols, out)
    torch.cuda.synchronize()
    ok = bool(torch.equal(out, d_in))
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(reps):
        ctx.recover(code, known, k, cols, out, stream=stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / reps
    del d_in, code, out
    torch.cuda.empty_cache()
    return {"k": k, "cols": cols, "erased_rows": k, "ms": round(ms, 4),
            "gbps": round(payload_bits(k) / (ms * 1e-3) / 1e9, 1), "bit_exact": ok,
            "api": "zoda_recover_device (two fused passes, each an INTT and an NTT over 2k points, TMA-staged)"}


def time_rlc(ctx, k: int, reps: int = 5) -> dict:
    """RLC consumers on the k x k extension (k x 128k data, 2k x 128k code): coefficients from a data
    root (device SHA-256 per column), RLC of every code row, and the full check of every row."""
    import torch
    cols = k * SHARE_U32
    gen = torch.Generator(device="cuda").manual_seed(11)
    d_in = torch.randint(0, P, (k, cols), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    code = torch.empty((2 * k, cols), dtype=torch.int32, device="cuda")
    ctx.extend(d_in, code, k, cols)
    coeff = torch.empty((cols, 4), dtype=torch.int32, device="cuda")
    rl = torch.empty((2 * k, 4), dtype=torch.int32, device="cuda")
    root = "ab" * 32  # any 64-hex-digit root: hashing the whole square is a host step, timed separately below
    stream = torch.cuda.current_stream()
    ctx.rlc_coefficients(root, cols, coeff)
    ctx.rlc_rows(code, 2 * k, cols, coeff, rl)
    mm = ctx.rlc_check(d_in, code, k, k, cols, coeff)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record(stream)
    for _ in range(reps):
        ctx.rlc_coefficients(root, cols, coeff, stream=stream)
    ev[1].record(stream)
    for _ in range(reps):
        ctx.rlc_rows(code, 2 * k, cols, coeff, rl, stream=stream)
    ev[2].record(stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        mm |= ctx.rlc_check(d_in, code, k, k, cols, coeff, stream=stream)
    t_check = (time.perf_counter() - t0) * 1e3 / reps
    coeff_ms = ev[0].elapsed_time(ev[1]) / reps
    rows_ms = ev[1].elapsed_time(ev[2]) / reps
    code_bytes = 2 * k * cols * 4
    del d_in, code
    torch.cuda.empty_cache()
    return {"k": k, "cols": cols, "coefficients_ms": round(coeff_ms, 4), "rlc_code_rows_ms": round(rows_ms, 4),
            "rlc_code_rows_gbs": round(code_bytes / (rows_ms * 1e-3) / 1e9, 1),
            "rlc_code_rows_hbm_frac": round(code_bytes / (rows_ms * 1e-3) / 1e9 / measured_peaks()["hbm_gbs"], 4),
            "check_all_rows_ms": round(t_check, 3), "check_mismatches": mm,
            "api": "zoda_rlc_coefficients_device, zoda_rlc_rows_device, zoda_rlc_check_device (synchronous)"}


def time_encode_general(ctx, k: int, n: int, reps: int = 5) -> dict:
    """Encode of a non-power-of-two shape (zoda_encode_device): [k][128k] -> [k+n][128k], device-resident."""
    import torch
    cols = k * SHARE_U32
    gen = torch.Generator(device="cuda").manual_seed(77)
    d_in = torch.randint(0, P, (k, cols), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    d_out = torch.empty((k + n, cols), dtype=torch.int32, device="cuda")
    ctx.encode(d_in, d_out, k, n, cols)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(reps):
        ctx.encode(d_in, d_out, k, n, cols, stream=stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / reps
    n_k = 1 << (k - 1).bit_length()
    r = (1 << (k + n - 1).bit_length()) // n_k  # output row r*m holds data row m
    m = min(k, (k + n + r - 1) // r)
    ok = bool(torch.equal(d_out[0::r][:m, :256], d_in[:m, :256]))
    del d_in, d_out
    torch.cuda.empty_cache()
    if r == 2:
        api = "zoda_encode_device (n_kn = 2 n_k: the fused kernels, zeros past row k, output cut at k+n)"
    elif 128 <= n_k <= 4096:
        api = f"zoda_encode_device (n_kn = {r} n_k: one fused TMA-staged INTT + NTT pass per coset, {r - 1} passes)"
    else:
        api = f"zoda_encode_device (n_kn = {r} n_k: one interpolation over n_k, {r - 1} coset evaluations)"
    return {"k": k, "n": n, "cols": cols, "ms": round(ms, 4),
            "gbps": round(k * k * 512 * 8.0 / (ms * 1e-3) / 1e9, 1), "data_rows_ok": ok, "api": api}


def data_root_device(rows, slab_bytes: int = 256 << 20) -> str:
    """compute_data_root (src/benchmarks/utils.rs:51-59) of a row-major u32 device matrix: SHA-256
    over the little-endian bytes of every row, streamed to the host in slabs of rows."""
    import hashlib
    import torch
    nrows, cols = rows.shape
    per = max(1, slab_bytes // (cols * 4))
    buf = torch.empty((per, cols), dtype=torch.int32).pin_memory()
    h = hashlib.sha256()
    for r0 in range(0, nrows, per):
        n = min(per, nrows - r0)
        buf[:n].copy_(rows[r0:r0 + n])
        h.update(buf[:n].numpy())
    return h.hexdigest()


def verify_extension(ctx, d_in, d_out, side: int, cols: int) -> dict:
    """The reference's RLC soundness check (src/benchmarks/utils.rs:221-272) over EVERY one of the
    2*side encoded rows instead of 64 samples: coefficients from the data root of the encoded rows
    (zoda_rlc_coefficients_device), then zoda_rlc_check_device. 0 mismatches = the output is the
    extension of the input, each row checked with 4 random-linear-combination limbs."""
    import torch
    t0 = time.perf_counter()
    root = data_root_device(d_out)
    coeff = torch.empty((cols, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_coefficients(root, cols, coeff)
    mm = ctx.rlc_check(d_in, d_out, side, side, cols, coeff)
    even_ok = bool(torch.equal(d_out[0::2], d_in))
    del coeff
    return {"check": f"RLC of all {2 * side} encoded rows (4 limbs each) against the extended RLC of the data, "
                     "coefficients from the SHA-256 data root of the encoded rows; even rows equal the data",
            "check_mismatches": int(mm), "even_rows_equal_data": even_ok, "data_root": root,
            "check_s": round(time.perf_counter() - t0, 2)}


def time_device_extend(ctx, side: int, steps: int, warmup: int, world: int, sampler=None, verify: bool = True,
                       cols: int | None = None):
    """Device-resident extension of one side x side square per step, CUDA events on the launching stream.
    With `verify`, the output of the last timed step is checked in full (verify_extension)."""
    import torch
    cols = side * SHARE_U32 if cols is None else cols
    gen = torch.Generator(device="cuda").manual_seed(1234 + side)
    d_in = torch.empty((side, cols), dtype=torch.int32, device="cuda")
    for r0 in range(0, side, 512):  # seeded uniform in [0, p), in slabs to bound the int64 temporary
        r1 = min(side, r0 + 512)
        d_in[r0:r1] = torch.randint(0, P, (r1 - r0, cols), dtype=torch.int64, device="cuda",
                                    generator=gen).to(torch.int32)
    d_out = torch.empty((2 * side, cols), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        ctx.extend(d_in, d_out, side, cols, stream=stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        ctx.extend(d_in, d_out, side, cols, stream=stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    ms = ev0.elapsed_time(ev1)
    check = verify_extension(ctx, d_in, d_out, side, cols) if verify else None
    del d_in, d_out
    torch.cuda.empty_cache()
    return ms, clocks, check


def time_host_extend(ctx, side: int, steps: int, warmup: int):
    """Same extension through the host-buffer C ABI call: H2D + kernel + D2H per step, pinned buffers."""
    import torch
    cols = side * SHARE_U32
    gen = torch.Generator().manual_seed(99)
    h_in = torch.empty((side, cols), dtype=torch.int32).pin_memory()
    for r0 in range(0, side, 256):  # seeded uniform in [0, p), in slabs to bound the int64 temporary
        r1 = min(side, r0 + 256)
        h_in[r0:r1] = torch.randint(0, P, (r1 - r0, cols), dtype=torch.int64, generator=gen).to(torch.int32)
    h_out = torch.empty((2 * side, cols), dtype=torch.int32).pin_memory()
    for _ in range(warmup):
        ctx.extend_host(h_in, h_out, side, cols)
    tot = 0.0
    parts = {"h2d_ms": 0.0, "kernel_ms": 0.0, "d2h_ms": 0.0}
    for _ in range(steps):
        t0 = time.perf_counter()
        t = ctx.extend_host(h_in, h_out, side, cols)
        tot += (time.perf_counter() - t0) * 1e3  # the whole call, wall clock
        for k in parts:
            parts[k] += getattr(t, k)
    # spot check of the last step: even rows are the input, odd rows the extension
    assert torch.equal(h_out[0::2, :64], h_in[:, :64])
    # PCIe bytes per step, as the library counted its copies: the input up; the odd rows down, plus
    # the even rows of the column chunks that return over PCIe (the rest are copied on the host)
    return tot / steps, {k: round(v / steps, 3) for k, v in parts.items()}, int(t.h2d_bytes), int(t.d2h_bytes)


def time_reference_cuda(side: int, iters: int = 2):
    """The reference's own CUDA kernel (cuda/ntt_kernel.cu built unmodified for sm_100a into
    oracle/_ref) in its published 'GPU xform' window: intt_cuda(n_k, n_kn) + ntt_cuda(n_kn, n_kn) on a
    pinned column-major square, PCIe included (src/benchmarks/utils.rs:137-140)."""
    import ctypes
    import numpy as np
    so = os.path.join(ROOT, "oracle", "_ref", "libntt_cuda_ref.so")
    if not os.path.exists(so):
        return None
    ref = ctypes.CDLL(so)
    ref.cuda_ntt.argtypes = ref.cuda_intt.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_uint32] * 3
    ref.cuda_host_alloc.restype = ctypes.c_void_p
    ref.cuda_host_alloc.argtypes = [ctypes.c_size_t]
    ref.cuda_host_free.argtypes = [ctypes.c_void_p]
    import oracle as O
    cols = side * SHARE_U32
    n_k, n_kn = side, 2 * side
    count = n_kn * cols
    ptr = ref.cuda_host_alloc(count)
    if not ptr:
        return None
    sq = np.frombuffer((ctypes.c_uint32 * count).from_address(ptr), dtype=np.uint32)
    rk, rkn = O.roots_of_unity(n_k), O.roots_of_unity(n_kn)
    rng = np.random.default_rng(5)
    v = sq.reshape(cols, n_kn)
    v[:, :n_k] = rng.integers(0, P, (cols, n_k), dtype=np.uint32)
    v[:, n_k:] = 0
    times = []
    for i in range(iters + 1):
        t0 = time.perf_counter()
        e1 = ref.cuda_intt(ptr, rk.ctypes.data, n_k, cols, n_kn)
        e2 = ref.cuda_ntt(ptr, rkn.ctypes.data, n_kn, cols, n_kn)
        dt = time.perf_counter() - t0
        if e1 or e2:
            ref.cuda_host_free(ptr)
            return {"error": f"cuda error {e1} {e2}"}
        if i:
            times.append(dt)
    ref.cuda_host_free(ptr)
    t = statistics.median(times)
    return {"side": side, "xform_ms": round(t * 1e3, 2), "gbps": round(payload_bits(side) / t / 1e9, 2),
            "window": "intt_cuda + ntt_cuda with PCIe (reference's 'GPU xform')"}


def log_uniform_sides(n: int, lo: int, hi: int, seed: int):
    rng = __import__("numpy").random.default_rng(seed)
    return [1 << int(rng.integers(lo.bit_length() - 1, hi.bit_length())) for _ in range(n)]


def time_batched(ctx, n: int, hi: int = 2048) -> dict:
    """n squares, sides log-uniform over 32..hi (seed 0), 128 u32 per share: one batched
    persistent launch (graph replay) against plain calls, one square at a time."""
    import torch
    import zoda_b200
    sides = log_uniform_sides(n, 32, hi, seed=0)
    sq = []
    for s in sides:
        a = torch.randint(0, P, (s, s * SHARE_U32), dtype=torch.int64, device="cuda").to(torch.int32)
        sq.append((a, torch.empty((2 * s, s * SHARE_U32), dtype=torch.int32, device="cuda"), s, s * SHARE_U32))
    payload = sum(payload_bits(s) for s in sides)
    batch = zoda_b200.Batch(ctx, sq)
    stream = torch.cuda.current_stream()
    for _ in range(3):
        batch.run(stream)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    ev0.record(stream)
    for _ in range(reps):
        batch.run(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    tb = ev0.elapsed_time(ev1) / reps
    # plain: one zoda_extend_device call per square, each waited for before the next
    for a, b, s, c in sq[:4]:
        ctx.extend(a, b, s, c)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for a, b, s, c in sq:
        ctx.extend(a, b, s, c)
        torch.cuda.synchronize()
    tp = (time.perf_counter() - t0) * 1e3
    # spot check: the batch and the plain calls wrote the same outputs
    b_out = sq[-1][1].clone()
    batch.run(stream)
    torch.cuda.synchronize()
    assert torch.equal(b_out, sq[-1][1])
    batch.close()
    per_side = {}
    for s in sorted(set(sides)):
        per_side[str(s)] = sides.count(s)
    del sq
    torch.cuda.empty_cache()
    return {"squares": n, "sides_drawn": per_side, "payload_gb": round(payload / 8e9, 3),
            "batched_ms": round(tb, 3), "batched_gbps": round(payload / (tb * 1e-3) / 1e9, 1),
            "plain_ms": round(tp, 3), "plain_gbps": round(payload / (tp * 1e-3) / 1e9, 1),
            "speedup": round(tp / tb, 3),
            "note": "plain = one zoda_extend_device per square, synchronized (one square at a time)"}


def serving_inputs(sides) -> dict:
    """Pre-staged request payloads in HBM: per side, a pool of distinct squares that together hold at
    least 256 MiB (twice the L2) and at least two squares, used in rotation, so no request finds its
    input in L2 from an earlier request of the same side."""
    import torch
    pools = {}
    for s in sorted(set(sides)):
        nbytes = s * s * SHARE_U32 * 4
        count = max(2, -(-(256 << 20) // nbytes))
        pools[s] = [torch.randint(0, P, (s, s * SHARE_U32), dtype=torch.int64, device="cuda").to(torch.int32)
                    for _ in range(count)]
    torch.cuda.synchronize()
    return pools


def time_serving(ctx, rate: float, nreq: int, budget_gib: int = 64) -> dict:
    """Seeded Poisson arrivals at `rate` squares/s, sides log-uniform over 64..2048,
    payloads pre-staged in HBM (serving_inputs: distinct inputs in rotation), 64 GiB output
    budget; p50/p99 latency and sustained Gb/s, against the same requests as sequential
    plain calls."""
    import threading
    import numpy as np
    import torch
    import zoda_b200
    rng = np.random.default_rng(1)
    sides = log_uniform_sides(nreq, 64, 2048, seed=1)
    gaps = rng.exponential(1.0 / rate, nreq)
    pools = serving_inputs(sides)
    seen = {s: 0 for s in pools}
    req_in = []
    for s in sides:  # request i's input: the next square of its side's pool
        req_in.append(pools[s][seen[s] % len(pools[s])])
        seen[s] += 1
    srv = zoda_b200.Server(ctx, budget_bytes=budget_gib << 30, max_inflight=4, max_batch=128)
    tickets = [None] * nreq
    submitted = threading.Event()

    def producer():  # open-loop arrivals: sleep (GIL released) until just before each one
        t_next = time.perf_counter()
        for i, s in enumerate(sides):
            t_next += gaps[i]
            while True:
                dt = t_next - time.perf_counter()
                if dt <= 0:
                    break
                time.sleep(dt if dt < 2e-4 else dt - 1e-4)
            tickets[i] = srv.submit(req_in[i], s, s * SHARE_U32)
        submitted.set()

    old_switch = sys.getswitchinterval()
    sys.setswitchinterval(2e-5)  # the submitting and the waiting thread both stay responsive
    th = threading.Thread(target=producer)
    t0 = time.perf_counter()
    th.start()
    lat = []
    for i in range(nreq):
        while tickets[i] is None:
            time.sleep(0.0001)
        info = srv.wait(tickets[i])
        lat.append(info.latency_ms)
        srv.release(tickets[i])
    th.join()
    wall = time.perf_counter() - t0
    sys.setswitchinterval(old_switch)
    st = srv.stats()
    srv.close()
    payload = sum(payload_bits(s) for s in sides)
    # the same requests as plain sequential calls
    outs = {s: torch.empty((2 * s, s * SHARE_U32), dtype=torch.int32, device="cuda") for s in pools}
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for i, s in enumerate(sides):
        ctx.extend(req_in[i], outs[s], s, s * SHARE_U32)
        torch.cuda.synchronize()
    tplain = time.perf_counter() - t1
    del pools, req_in, outs
    torch.cuda.empty_cache()
    lat.sort()
    return {"requests": nreq, "offered_rate_per_s": rate, "offered_gbps": round(payload / (gaps.sum()) / 1e9, 1),
            "sustained_gbps": round(payload / (st.first_submit_to_last_done_ms * 1e-3) / 1e9, 1),
            "p50_ms": round(st.p50_ms, 3), "p99_ms": round(st.p99_ms, 3), "max_ms": round(st.max_ms, 3),
            "launches": int(st.launches), "wall_s": round(wall, 3),
            "plain_sequential_gbps": round(payload / tplain / 1e9, 1),
            "budget_gib": budget_gib, "sides": "log-uniform 64..2048, 128 u32/share, seed 1",
            "inputs": "distinct pre-staged squares per side, >= 256 MiB per side, in rotation"}


def workload_config(side: int) -> dict:
    """The workload both arms name (identical dicts, so the two lines compare like for like)."""
    cols = side * SHARE_U32
    return {"workload": f"plain extension of one {side}x{side} square of 512-byte shares per GPU "
                        f"([{side}][{cols}] u32 -> [{2 * side}][{cols}])",
            "side": side, "cols": cols, "share_bytes": 512,
            "l2": "inputs and outputs larger than the 126 MB L2; no flush between steps"}


def launches_per_step(side: int, plan: dict | None) -> int:
    """Kernels zoda_extend_device launches per square: the four-step plan runs three passes, as
    three launches or (blocked 1) one pipelined launch; every side above 4096 three launches; the
    single-pass kernels one."""
    if side > 4096:
        return 3
    if plan and plan.get("impl") == 3:
        return 1 if plan.get("blocked") else 3
    return 1


def plan_kernels(side: int, plan: dict | None) -> str:
    if plan and plan.get("impl") == 3 and plan.get("blocked") and side <= 4096:
        return ("k_fourstep_pipe (the three four-step passes, strided INTT, block INTT+twist+NTT and "
                "strided NTT, column chunk by column chunk in one persistent launch)")
    if side > 4096 or (plan and plan.get("impl") == 3):
        staged = " with cp.async-staged tiles" if plan and plan.get("sched") else ""
        return ("k_step / k_step2 (three four-step passes: strided INTT, block INTT+twist+NTT, strided NTT)"
                + staged)
    return kernel_name(side, plan)


def traffic_key(side: int, plan: dict | None) -> str:
    """profiles/traffic.json key of the kernel(s) one step runs."""
    if plan and plan.get("impl") == 3:
        return f"k_extend_side{side}_fourstep" + ("_pipe" if plan.get("blocked") else "")
    return f"k_extend_side{side}"


def measure_side(ctx, side: int, steps: int, warmup: int, world: int, sampler=None, tune_it: bool = True,
                 e2e_steps: int = 3, cpu_budget: float = 0.0) -> dict:
    """Everything the JSON line says about one square size: the side's plan (tuned at this workload),
    device-resident payload Gb/s over `steps` timed steps (max over ranks), the HBM roofline of the
    step, the full check of the timed output, the same extension end to end through the host-buffer
    C ABI call, and (cpu_budget > 0) the CPU port on a bounded column sample."""
    cols = side * SHARE_U32
    plan = tune(ctx, side, cols, reps=3 if side >= 4096 else 10) if tune_it else None
    ms, clocks, check = time_device_extend(ctx, side, steps, warmup, world, sampler)
    ms_max = max_over_ranks(ms, world)
    peaks = measured_peaks()
    alg_bytes = 12.0 * side * cols  # read [side][cols] + write [2 side][cols] u32, the single-pass minimum
    achieved = alg_bytes / (ms / steps * 1e-3) / 1e9
    barrier(world)
    e2e_ms, parts, h2d, d2h = time_host_extend(ctx, side, e2e_steps, 1)
    e2e_max = max_over_ranks(e2e_ms, world)
    out = {
        "value": job_rate(world, side, ms_max, steps), "ms_per_step": ms_max / steps, "plan": plan,
        "plan_source": "zoda_autotune at this workload" if plan else "default",
        "clocks": clocks, "output_check": check,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4),
                     "traffic": ncu_traffic(traffic_key(side, plan)),
                     "peak_source": peaks["source"], "kernel": plan_kernels(side, plan),
                     "launches_per_step": launches_per_step(side, plan), "alg_bytes_per_step": alg_bytes},
        "e2e": {"value": round(job_rate(world, side, e2e_max, 1), 3), "unit": "Gb/s",
                "h2d_bytes_per_step": world * h2d, "d2h_bytes_per_step": world * d2h,
                "ms_per_step": round(e2e_max, 3), "split_ms": parts,
                "api": "zoda_extend_host (pinned host buffers; odd rows over PCIe, even rows copied on the host "
                       "except the last eighth of the column chunks)"},
    }
    if cpu_budget > 0:
        cpu = cpu_port_rate(side, cpu_budget)
        cpu.pop("seconds", None)
        out["cpu_baseline"] = cpu
    return out


def run_ours(args, world, rank, local):
    import torch
    import zoda_b200
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    ctx = zoda_b200.Context(local)
    side = args.side
    sampler = ClockSampler(local) if rank == 0 else None
    # the headline: every rank extends its own square; the CPU baseline runs on rank 0 of a 1-GPU run only
    head = measure_side(ctx, side, args.steps, args.warmup, world, sampler, tune_it=not args.no_tune,
                        e2e_steps=max(2, min(args.steps, 3)),
                        cpu_budget=args.cpu_budget if rank == 0 and world == 1 else 0.0)
    extra = {}
    if world > 1:
        barrier(world)
    # report-only extras: rank 0 of a 1-GPU run only (they would hold the other ranks at the next
    # barrier for a minute or more)
    if rank == 0 and world == 1 and not args.no_extra:
        for s2 in args.extra_sides:
            if s2 == side:
                continue
            m = measure_side(ctx, s2, args.steps, args.warmup, 1, tune_it=not args.no_tune, e2e_steps=3,
                             cpu_budget=args.cpu_budget / 2 if s2 == 1024 else 0.0)
            m["gbps"] = round(m.pop("value"), 1)
            m["ms_per_step"] = round(m["ms_per_step"], 4)
            m["config"] = workload_config(s2)
            extra[f"side{s2}"] = m
        extra["recover_k1024"] = time_recover(ctx, 1024)
        extra["encode_k1000_n1000"] = time_encode_general(ctx, 1000, 1000)
        extra["encode_k1000_n3000"] = time_encode_general(ctx, 1000, 3000)
        extra["rlc_k1024"] = time_rlc(ctx, 1024)
        refc = time_reference_cuda(min(side, 1024))
        if refc:
            extra["reference_cuda_kernel"] = refc
        if not args.no_batch:
            if not args.no_tune:  # the batch's smaller sides (the larger ones were tuned above)
                ctx.autotune(32, 512, 0, 3)
            extra["batched_mixed_squares"] = time_batched(ctx, args.batch_squares)
            # where launch overhead dominates: the same draw restricted to sides 32..256
            extra["batched_small_squares"] = time_batched(ctx, args.batch_squares, hi=256)
            extra["serving"] = time_serving(ctx, args.serve_rate, args.serve_requests)
            # below capacity: latency without queueing behind a saturated device
            extra["serving_below_capacity"] = time_serving(ctx, args.serve_rate / 2, args.serve_requests)
        one = cpu_port_rate(side, max(2.0, args.cpu_budget / 4), threads=1)  # as the reference's CPU path runs
        one.pop("seconds", None)
        extra["cpu_port_single_thread"] = one
    if world > 1:
        barrier(world)
    if rank == 0:
        check = head["output_check"]
        line = {
            "metric": METRIC, "value": round(head["value"], 3), "unit": "Gb/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(head["ms_per_step"], 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded uniform in [0,p), device-resident)",
            "config": workload_config(side),
            "plan": head["plan"], "plan_source": head["plan_source"],
            "roofline": head["roofline"],
            "cpu_baseline": head.get("cpu_baseline"),
            "check_mismatches": check["check_mismatches"] if check else None,
            "output_check": check,
            "e2e": head["e2e"],
            "gpu_launches": args.steps * head["roofline"]["launches_per_step"],
            "clocks": head["clocks"],
            "extra": extra,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--side", type=int, default=4096,
                    help="the headline square (default: 4096, the largest single-GPU configuration)")
    ap.add_argument("--extra-sides", type=int, nargs="*", default=[1024, 2048])
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched and serving report lines")
    ap.add_argument("--no-tune", action="store_true", help="run the default plans instead of tuning first")
    ap.add_argument("--batch-squares", type=int, default=96)
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-requests", type=int, default=1000)
    ap.add_argument("--cpu-budget", type=float, default=10.0, help="seconds of CPU baseline sampling")
    ap.add_argument("--ref-step-budget", type=float, default=None,
                    help="seconds of CPU work per step of --impl reference (default: about 60 s in total)")
    ap.add_argument("--leg", choices=["rlc", "recover", "encode", "extend", "footprint", "long"], default=None,
                    help="run one report-only leg on one GPU and print its JSON (a small case to profile): "
                         "extend = --steps extensions of a [--side][--cols] slab; footprint = ps per element "
                         "of the --side extension against the number of columns")
    ap.add_argument("--cols", type=int, default=0, help="columns of the extend leg (0: side * 128)")
    ap.add_argument("--force-impl", choices=["auto", "direct", "tma"], default="auto",
                    help="legs only: run one kernel family with default knobs instead of the side's plan")
    ap.add_argument("--plan", default=None,
                    help="legs only: a JSON launch plan installed for --side (zoda_plan fields), e.g. "
                         "'{\"impl\": 3, \"radix\": 8, \"ctas\": 4, \"blocked\": 1}'")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)  # at least 3 untimed warm-up steps
    if args.leg:
        import zoda_b200
        ctx = zoda_b200.Context(0)
        ctx.set_impl({"auto": 0, "direct": 1, "tma": 2}[args.force_impl])
        if args.plan:
            plan = {"impl": 1, "sched": 0, "l2_promo": 3, "blocked": 0, "stagger": 1, "radix": 16, "ctas": 0}
            plan.update(json.loads(args.plan))
            ctx.plan_set(args.side, plan)
        leg = {"rlc": lambda: time_rlc(ctx, 1024), "recover": lambda: time_recover(ctx, 1024),
               "encode": lambda: [time_encode_general(ctx, 1000, 1000), time_encode_general(ctx, 1000, 3000)],
               "extend": lambda: time_extend_leg(ctx, args.side, args.cols or args.side * SHARE_U32, args.steps,
                                                 args.warmup),
               "footprint": lambda: footprint_sweep(ctx, args.side), "long": lambda: time_long_leg(ctx)}[args.leg]
        res = leg()
        print(json.dumps({"leg": args.leg, **res} if isinstance(res, dict) else {"leg": args.leg, "runs": res}))
        return
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
