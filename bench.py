"""Benchmark of the iclBLAS hot path on B200.

Default workload (one "step"): the bandwidth-bound level-1/2 sweep of the
reference's bandwidth config: SAXPY, SDOT, SNRM2, SASUM, ISAMAX at n = 2^28
(fp32, stride 1, U(-1,1), seed 1), SGEMV 16384x16384 (N and T) and CGEMV
8192x8192 (N and C).  Metric: aggregate achieved HBM GB/s = algorithmic bytes
of the sweep / time.  Every input (>= 512 MiB) is larger than L2 (126 MB), so
no L2 flush is needed between steps.

  value   device-resident operands, timed with CUDA events on the stream the
          kernels run on;
  e2e     the same sweep through the C ABI with HOST (pinned) operands: every
          call copies its inputs in and its outputs back, as the reference's
          API does;
  roofline  dominant kernel's algorithmic bytes / its mean event-timed
          duration, against the measured HBM copy bandwidth;
  cpu_baseline  the reference's own CPU code for the same routines
          (oracle/_ref, built from the reference's sources) on the full
          config, 1 thread, 2 steps.

The same line carries the metric's first clause, timed in the same run with
its own clock record: SGEMM 8192^3 and STRSM 8192x4096 in plain FP32 and the
tensor-core split modes (3xBF16, 6xBF16, TF32; STRSM also 3xBF16 + one
refinement step) with their errors against FP64 (`sgemm_8192`,
`strsm_8192x4096`), and config 1, plain SGEMM 512^3, beside the reference's
cpu_gemm on one and on all host cores (`sgemm_512_config`), and the batched
config (`batched_512`: 512 uneven STRSM instances, forward + adjoint, in
plain FP32 on the CUDA cores and in each tensor-core mode, beside the same
work as per-instance plain calls, with errors against FP64 and its own
clock record).

`--impl reference` times the reference's CPU implementation with every host
thread on the full sweep config.  Multi-GPU (torchrun): each rank runs an
independent replica (BLAS calls do not shard), weak scaling.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

N1 = 1 << 28
GEMV_N = 16384
CGEMV_N = 8192


def sweep_bytes(n1=N1, gn=GEMV_N, cn=CGEMV_N):
    """Algorithmic bytes per call of the sweep (beta != 0 GEMV reads y)."""
    return {
        "saxpy": 12 * n1,
        "sdot": 8 * n1,
        "snrm2": 4 * n1,
        "sasum": 4 * n1,
        "isamax": 4 * n1,
        "sgemv_n": 4 * (gn * gn + gn + 2 * gn),
        "sgemv_t": 4 * (gn * gn + gn + 2 * gn),
        "cgemv_n": 8 * (cn * cn + cn + 2 * cn),
        "cgemv_c": 8 * (cn * cn + cn + 2 * cn),
    }


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "sweep_kernels_dram_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return {}
    return {}


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons; summary() keeps the
    samples whose timestamps fall inside the timed window."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.f = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def started(self) -> bool:
        """True once the sampler has written a line (or cannot run at all)."""
        if self.proc is None or self.proc.poll() is not None:
            return True
        self.f.flush()
        return os.path.getsize(self.f.name) > 0

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(0.25)  # let the sampler flush a line past the window

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        import datetime as dt
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [c.strip() for c in r]
            if len(r) < 10:
                continue
            try:
                ts = dt.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                clk, cmax = float(r[2]), float(r[3])
            except ValueError:
                continue
            if self.t0 is not None and not (self.t0 - 0.15 <= ts <= self.t1 + 0.15):
                continue
            sm.append(clk)
            smax = cmax
            try:
                power.append(float(r[4]))
            except ValueError:
                pass
            for nm, v in zip(names, r[6:10]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------- GPU sweep
class Sweep:
    """Operands of the sweep on one GPU and the calls that make one step."""

    def __init__(self, torch, dev, B, host: bool, n1: int = N1, only=None, pageable: bool = False):
        self.B = B
        self.only = only
        g = torch.Generator(device="cpu").manual_seed(1)

        def mk(shape, dtype=torch.float32):
            t = torch.rand(shape, generator=g, dtype=torch.float32) * 2 - 1
            if dtype == torch.complex64:
                t = torch.complex(t, torch.rand(shape, generator=g, dtype=torch.float32) * 2 - 1)
            if host:
                return t if pageable else t.pin_memory()   # pageable: ordinary (malloc'd) host memory
            return t.to(dev)

        def want(*names):
            return not only or any(nm in only for nm in names)

        n = n1
        self.n = n
        l1 = want("saxpy", "sdot", "snrm2", "sasum", "isamax")
        self.x = mk((n,)) if l1 else None
        self.y = mk((n,)) if want("saxpy", "sdot") else None
        sg = want("sgemv_n", "sgemv_t")
        self.A = mk((GEMV_N * GEMV_N,)) if sg else None
        self.gx = mk((GEMV_N,)) if sg else None
        self.gy = mk((GEMV_N,)) if sg else None
        cg = want("cgemv_n", "cgemv_c")
        self.CA = mk((CGEMV_N * CGEMV_N,), torch.complex64) if cg else None
        self.cx = mk((CGEMV_N,), torch.complex64) if cg else None
        self.cy = mk((CGEMV_N,), torch.complex64) if cg else None
        if host:
            self.r = torch.zeros(1, dtype=torch.float32)
            self.ri = torch.zeros(1, dtype=torch.int32)
            if not pageable:
                self.r, self.ri = self.r.pin_memory(), self.ri.pin_memory()
        else:
            self.r = torch.zeros(1, dtype=torch.float32, device=dev)
            self.ri = torch.zeros(1, dtype=torch.int32, device=dev)
        self.host = host

    def calls(self, h):
        """(name, thunk) for each call of one step, in order."""
        B, n = self.B, self.n
        gn, cn = GEMV_N, CGEMV_N
        allc = [
            ("saxpy", lambda: B.iclblasSaxpy(h, n, 0.5, self.x, 1, self.y, 1)),
            ("sdot", lambda: B.iclblasSdot(h, n, self.x, 1, self.y, 1, self.r)),
            ("snrm2", lambda: B.iclblasSnrm2(h, n, self.x, 1, self.r)),
            ("sasum", lambda: B.iclblasSasum(h, n, self.x, 1, self.r)),
            ("isamax", lambda: B.iclblasIsamax(h, n, self.x, 1, self.ri)),
            ("sgemv_n", lambda: B.iclblasSgemv(h, 0, gn, gn, 1.0, self.A, gn, self.gx, 1, 0.5, self.gy, 1)),
            ("sgemv_t", lambda: B.iclblasSgemv(h, 1, gn, gn, 1.0, self.A, gn, self.gx, 1, 0.5, self.gy, 1)),
            ("cgemv_n", lambda: B.iclblasCgemv(h, 0, cn, cn, 1 + 1j, self.CA, cn, self.cx, 1, 0.5, self.cy, 1)),
            ("cgemv_c", lambda: B.iclblasCgemv(h, 2, cn, cn, 1 + 1j, self.CA, cn, self.cx, 1, 0.5, self.cy, 1)),
        ]
        return [c for c in allc if not self.only or c[0] in self.only]

    def io_bytes(self):
        """Host<->device bytes per step of the host-operand (e2e) sweep."""
        n, gn, cn = self.n, GEMV_N, CGEMV_N
        h2d = 4 * (2 * n + 2 * n + n + n + n) + 2 * 4 * (gn * gn + 2 * gn) + 2 * 8 * (cn * cn + 2 * cn)
        d2h = 4 * n + 4 + 4 + 4 + 4 + 2 * 4 * gn + 2 * 8 * cn
        return h2d, d2h


def max_over_ranks(torch, value, device, world):
    """The largest per-rank value over all ranks: a replicated job's time is
    its slowest rank's.  One all-reduce (MAX) when world > 1."""
    if world <= 1:
        return float(value)
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def aggregate_gbs(world, bytes_per_step, steps, ms):
    """Whole-job bandwidth: every rank moved bytes_per_step per step in ms."""
    return world * bytes_per_step * steps / (ms / 1e3) / 1e9


def run_ours(args, rank, world, torch):
    from clgpu_b200 import iclblas as B
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    only = set(args.only.split(",")) if args.only else None
    bytes_all = sweep_bytes(args.n1)

    with B.Handle() as h:
        h.set_stream(stream)
        sw = Sweep(torch, dev, B, host=False, n1=args.n1, only=only)
        torch.cuda.synchronize()
        calls = sw.calls(h)
        bytes_per = {name: bytes_all[name] for name, _ in calls}
        step_bytes = sum(bytes_per.values())
        with torch.cuda.stream(stream), Clocks(dev.index) as clk:
            for _ in range(args.warmup):
                for name, f in calls:
                    B.check(f(), name)
            # keep the GPU busy until the clock sampler is running
            t_wait = time.time()
            while not clk.started() and time.time() - t_wait < 5.0:
                for name, f in calls:
                    B.check(f(), name)
                torch.cuda.synchronize()
            torch.cuda.synchronize()
            ev = {name: [] for name, _ in calls}
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            clk.mark_start()
            start.record(stream)
            for _ in range(args.steps):
                for name, f in calls:
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    B.check(f(), name)
                    e1.record(stream)
                    ev[name].append((e0, e1))
            end.record(stream)
            torch.cuda.synchronize()
            clk.mark_end()
        clocks = clk.summary()
        total_ms = start.elapsed_time(end)
        per_call_ms = {name: float(np.mean([a.elapsed_time(b) for a, b in ev[name]])) for name in ev}
        t_max = max_over_ranks(torch, total_ms, dev, world)
        value = aggregate_gbs(world, step_bytes, args.steps, t_max)

        # dominant kernel: the call with the largest share of the step
        dom = max(per_call_ms, key=per_call_ms.get)
        peak, peak_kind = load_peaks()
        achieved = bytes_per[dom] / (per_call_ms[dom] / 1e3) / 1e9
        tr = load_traffic().get(dom)
        traffic = None
        if tr:
            # scale the captured launch's DRAM bytes to this launch's size
            traffic = int(tr["dram_bytes"] * bytes_per[dom] / tr["algorithmic_bytes"])

        e2e = None
        if not args.no_e2e:
            # host (pinned) operands through the same C ABI calls
            del sw
            torch.cuda.empty_cache()
            swh = Sweep(torch, dev, B, host=True, n1=args.n1, only=only)
            callsh = swh.calls(h)
            for name, f in callsh:
                B.check(f(), name)
            e2e_steps = max(1, min(args.steps, 3))
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            for _ in range(e2e_steps):
                for name, f in callsh:
                    B.check(f(), name)
            s1.record(stream)
            torch.cuda.synchronize()
            e2e_ms = max_over_ranks(torch, s0.elapsed_time(s1), dev, world)
            h2d, d2h = swh.io_bytes()
            e2e = {"value": round(aggregate_gbs(world, step_bytes, e2e_steps, e2e_ms), 2), "unit": "GB/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                   "ms_per_step": round(e2e_ms / e2e_steps, 3),
                   "path": "C ABI with pinned host operands; copies in/out inside every call"}
            del swh
            # the same calls on pageable (ordinary malloc'd) host memory, what a
            # drop-in caller of the reference's API passes
            swp = Sweep(torch, dev, B, host=True, n1=args.n1, only=only, pageable=True)
            callsp = swp.calls(h)
            for name, f in callsp:
                B.check(f(), name)
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            p0 = torch.cuda.Event(enable_timing=True)
            p1 = torch.cuda.Event(enable_timing=True)
            p0.record(stream)
            for name, f in callsp:
                B.check(f(), name)
            p1.record(stream)
            torch.cuda.synchronize()
            pg_ms = max_over_ranks(torch, p0.elapsed_time(p1), dev, world)
            e2e["pageable"] = {"value": round(aggregate_gbs(world, step_bytes, 1, pg_ms), 2), "unit": "GB/s",
                               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": 1,
                               "ms_per_step": round(pg_ms, 3),
                               "path": "C ABI with pageable host operands (ordinary host memory)"}
            del swp

    out = {
        "metric": "level-1/2 sweep aggregate HBM bandwidth (SAXPY/SDOT/SNRM2/SASUM/ISAMAX n=2^28, "
                  "SGEMV 16384^2 N+T, CGEMV 8192^2 N+C)",
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_max / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic U(-1,1), seed 1",
        "config": {"workload": "bandwidth sweep: level-1 n=%d x5, SGEMV 16384^2 N,T, CGEMV 8192^2 N,C" % args.n1
                   if not only else "subset %s, level-1 n=%d" % (sorted(only), args.n1),
                   "bytes_per_step": step_bytes, "l2": "inputs larger than L2 (>=512 MiB each), no flush",
                   "parallelism": f"replicas x{world}"},
        "per_call_ms": {k: round(v, 4) for k, v in per_call_ms.items()},
        "per_call_gbs": {k: round(bytes_per[k] / (per_call_ms[k] / 1e3) / 1e9, 1) for k in per_call_ms},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                     "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic, "algorithmic_bytes": bytes_per[dom]},
        "e2e": e2e,
        "gpu_launches": len(calls) * args.steps,
        "clocks": clocks,
    }
    return out


# ---------------------------------------------------------------- precision legs of the default run
def fp32_fma_peak_tflops(torch, dev):
    """Nominal FP32 FMA peak of the GPU: SMs x 128 lanes x 2 flops x max SM clock."""
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = 1965.0
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        mhz = float(json.load(open(pp)).get("sm_max_mhz", mhz))
    return sms * 128 * 2 * mhz * 1e6 / 1e12


def run_precision_legs(torch, dev, B, n_gemm=8192, trsm_m=8192, trsm_n=4096):
    """The metric's first clause, timed in the default run: SGEMM 8192^3 NN
    (U(-1,1), seed 2) in plain FP32 (CUDA cores), TF32, 3xBF16 and 6xBF16;
    STRSM 8192 x 4096 left/lower/N/non-unit (diagonal U(1,2), strictly lower
    N(0,1)/sqrt(M), B U(-1,1), seed 3) in plain FP32, TF32, 3xBF16, 6xBF16
    and 3xBF16 + one refinement step; and config 1 itself, plain SGEMM NN
    512^3 alpha 1.5 beta 0.5 (seed 0), beside the reference's cpu_gemm on 1
    and on all host cores.  Device operands, CUDA events on the launching
    stream, median of 5 calls after one untimed call; errors are relative
    Frobenius against FP64 (torch float64 on the GPU, plumbing only); TFLOP/s
    count the algorithmic 2MNK (GEMM) and M^2 N (TRSM) flops only."""
    stream = torch.cuda.Stream(device=dev)
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    bf16_sus = peaks.get("bf16_tflops_sustained")
    fp32_peak = fp32_fma_peak_tflops(torch, dev)
    nprod = {B.MATH_TF32: 1, B.MATH_BF16X3: 3, B.MATH_BF16X6: 6}
    out = {}

    def med(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            ts.append((e0, e1))
        torch.cuda.synchronize()
        return float(np.median([a.elapsed_time(b) for a, b in ts]))

    def roof(mode, flops, ms):
        tf = flops / (ms / 1e3) / 1e12
        if mode == B.MATH_PLAIN_FP32:
            return {"bound": "fp32_fma", "peak": round(fp32_peak, 1), "peak_source": "nominal (SMs x 128 x 2 x max clock)",
                    "frac": round(tf / fp32_peak, 3)}
        if not bf16_sus:
            return None
        ex = nprod[mode] * tf
        # TF32 runs at half the BF16 rate per product
        eff = ex * (2.0 if mode == B.MATH_TF32 else 1.0)
        return {"bound": "tensor", "executed_tflops": round(ex, 1), "peak": bf16_sus,
                "peak_source": "measured sustained bf16 (TF32 products counted at twice their cost)",
                "frac": round(eff / bf16_sus, 3)}

    names = {B.MATH_PLAIN_FP32: "fp32", B.MATH_TF32: "tf32", B.MATH_BF16X3: "3xbf16", B.MATH_BF16X6: "6xbf16"}
    with B.Handle() as h, torch.cuda.stream(stream), Clocks(dev.index) as clk:
        h.set_stream(stream)
        t_wait = time.time()
        while not clk.started() and time.time() - t_wait < 5.0:
            time.sleep(0.05)
        clk.mark_start()
        # ---- SGEMM n^3 NN
        n = n_gemm
        g = torch.Generator(device=dev).manual_seed(2)
        A = torch.rand(n * n, generator=g, device=dev) * 2 - 1
        Bm = torch.rand(n * n, generator=g, device=dev) * 2 - 1
        C = torch.empty(n * n, device=dev)
        ref = A.view(n, n).t().double() @ Bm.view(n, n).t().double()
        refn = torch.linalg.norm(ref).item()
        fl = 2.0 * n * n * n
        res = {}
        for mode in (B.MATH_PLAIN_FP32, B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6):
            h.set_math_mode(mode)
            ms = med(lambda: B.check(B.iclblasSgemm(h, 0, 0, n, n, n, 1.0, A, n, Bm, n, 0.0, C, n), "sgemm"))
            err = torch.linalg.norm(C.view(n, n).t().double() - ref).item() / refn
            res[names[mode]] = {"tflops": round(fl / (ms / 1e3) / 1e12, 2), "ms": round(ms, 3),
                                "rel_err_vs_fp64": float("%.3g" % err), "roofline": roof(mode, fl, ms)}
        base = res["fp32"]["tflops"]
        for k in res:
            res[k]["x_plain_fp32"] = round(res[k]["tflops"] / base, 2)
        out["sgemm_8192"] = {"config": f"SGEMM NN {n}^3 fp32, U(-1,1) seed 2, alpha 1 beta 0", **res}
        del A, Bm, C, ref
        torch.cuda.empty_cache()

        # ---- STRSM M x N left / lower / N / non-unit
        m, nr = trsm_m, trsm_n
        g = torch.Generator(device=dev).manual_seed(3)
        L = torch.tril(torch.randn(m, m, generator=g, device=dev) / m ** 0.5, -1)
        L = L + torch.diag(torch.rand(m, generator=g, device=dev) + 1.0)
        Acm = L.t().contiguous().reshape(-1)
        B0 = (torch.rand(nr, m, generator=g, device=dev) * 2 - 1).reshape(-1)
        X64 = torch.linalg.solve_triangular(L.double(), B0.view(nr, m).t().double(), upper=False)
        x64n = torch.linalg.norm(X64).item()
        del L
        Bw = torch.empty_like(B0)
        Bt = torch.empty_like(B0)
        fl = float(m) * m * nr
        ms_copy = med(lambda: Bt.copy_(B0))
        res = {}
        for mode, steps in ((B.MATH_PLAIN_FP32, 0), (B.MATH_TF32, 0), (B.MATH_BF16X3, 0), (B.MATH_BF16X6, 0),
                            (B.MATH_BF16X3, 1)):
            h.set_math_mode(mode)
            h.set_trsm_refinement(steps)

            def run():
                Bw.copy_(B0)
                B.check(B.iclblasStrsm(h, 0, 1, 0, 0, m, nr, 1.0, Acm, m, Bw, m), "strsm")
            ms = max(med(run) - ms_copy, 1e-6)
            err = torch.linalg.norm(Bw.view(nr, m).t().double() - X64).item() / x64n
            key = names[mode] + (f"+refine{steps}" if steps else "")
            r = {"tflops": round(fl / (ms / 1e3) / 1e12, 2), "ms": round(ms, 3),
                 "rel_err_vs_fp64": float("%.3g" % err)}
            if steps == 0:
                r["roofline"] = roof(mode, fl, ms)
            res[key] = r
        h.set_trsm_refinement(0)
        h.set_math_mode(B.MATH_PLAIN_FP32)
        base = res["fp32"]["tflops"]
        for k in res:
            res[k]["x_plain_fp32"] = round(res[k]["tflops"] / base, 2)
        out["strsm_8192x4096"] = {"config": f"STRSM left/lower/N/non-unit M={m} NRHS={nr} fp32, seed 3", **res}
        del Acm, B0, X64, Bw, Bt
        torch.cuda.empty_cache()

        # ---- config 1: plain SGEMM 512^3, alpha 1.5, beta 0.5
        n = 512
        rng = np.random.default_rng(0)
        Ah = rng.uniform(-1, 1, n * n).astype(np.float32)
        Bh = rng.uniform(-1, 1, n * n).astype(np.float32)
        Ch = rng.uniform(-1, 1, n * n).astype(np.float32)
        Ad, Bd, C0 = (torch.from_numpy(v).to(dev) for v in (Ah, Bh, Ch))
        Cd = C0.clone()
        fl = 2.0 * n ** 3
        ms = med(lambda: B.check(B.iclblasSgemm(h, 0, 0, n, n, n, 1.5, Ad, n, Bd, n, 0.5, Cd, n), "sgemm"), reps=50)
        Cd.copy_(C0)
        B.check(B.iclblasSgemm(h, 0, 0, n, n, n, 1.5, Ad, n, Bd, n, 0.5, Cd, n), "sgemm")
        torch.cuda.synchronize()
        got = Cd.cpu().numpy()
        # host operands through the C ABI (copies in and out inside the call)
        Cw = Ch.copy()
        t0 = time.perf_counter()
        for _ in range(20):
            Cw[:] = Ch
            B.check(B.iclblasSgemm(h, 0, 0, n, n, n, 1.5, Ah, n, Bh, n, 0.5, Cw, n), "sgemm host")
        host_ms = (time.perf_counter() - t0) / 20 * 1e3
        clk.mark_end()
    out["precision_clocks"] = clk.summary()

    # CPU: the reference's cpu_gemm (double accumulation), 1 core and all cores
    cpu = cpu_sgemm_512(Ah, Bh, Ch, n)
    err = float(np.linalg.norm(got.astype(np.float64) - cpu["C"]) / np.linalg.norm(cpu["C"]))
    out["sgemm_512_config"] = {
        "config": "SGEMM NN 512^3 fp32, lda=ldb=ldc=512, alpha 1.5, beta 0.5, U(-1,1) seed 0",
        "gpu_tflops": round(fl / (ms / 1e3) / 1e12, 2), "gpu_us": round(ms * 1e3, 1),
        "gpu_host_operands_us": round(host_ms * 1e3, 1),
        "rel_err_vs_cpu_gemm": float("%.3g" % err),
        "cpu_gemm_1core_ms": round(cpu["t1"] * 1e3, 2), "cpu_gemm_ncore_ms": round(cpu["tn"] * 1e3, 2),
        "cpu_cores": cpu["cores"], "cpu_kind": cpu["kind"],
        "cpu_gemm_1core_gflops": round(fl / cpu["t1"] / 1e9, 2), "cpu_gemm_ncore_gflops": round(fl / cpu["tn"] / 1e9, 2),
    }
    return out


def cpu_sgemm_512(Ah, Bh, Ch, n):
    """The reference's cpu_gemm template (double accumulation, compiled in
    oracle/_ref; the oracle's double GEMM if the reference was not built)
    on config 1, on one core and split by column blocks over every host core."""
    import ctypes as C
    import oracle_lib as O
    R = O.ref()
    kind = "reference" if R is not None else "port"
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)

    def run(c0, c1, Cout):
        if c1 <= c0:
            return
        if R is not None:
            R.ref_cpu_sgemm(0, 0, n, c1 - c0, n, 1.5, Ah.ctypes.data, n, Bh.ctypes.data + 4 * c0 * n, n, 0.5,
                            Cout.ctypes.data + 4 * c0 * n, n)
        else:
            A64, B64 = Ah.astype(np.float64), Bh[c0 * n:c1 * n].astype(np.float64)
            C64 = Ch[c0 * n:c1 * n].astype(np.float64)
            O.dgemm(0, 0, n, c1 - c0, n, 1.5, A64, n, B64, n, 0.5, C64, n)
            Cout[c0 * n:c1 * n] = C64
    out1 = Ch.copy()
    t0 = time.perf_counter()
    run(0, n, out1)
    t1 = time.perf_counter() - t0
    outn = Ch.copy()
    b = np.linspace(0, n, cores + 1).astype(int)
    ts = [threading.Thread(target=run, args=(int(b[i]), int(b[i + 1]), outn)) for i in range(cores)]
    t0 = time.perf_counter()
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    tn = time.perf_counter() - t0
    return {"C": out1.astype(np.float64), "t1": t1, "tn": tn, "cores": cores, "kind": kind}


# ---------------------------------------------------------------- GEMM precision study
def run_gemm_study(args, torch):
    """Precision config: SGEMM and CGEMM at M=N=K=n (default 8192), NN and
    A^T*B, U(-1,1) (seed 2) plus a row-scaled variant (row i of A times
    10^U(-4,4)); plain FP32 (CUDA cores) vs TF32 vs 3xBF16 vs 6xBF16 on the
    tensor cores.  Error = ||C - C64||_F / ||C64||_F against an FP64 product of
    the same FP32 inputs (torch float64 on the GPU, plumbing only); for the
    row-scaled variant also the largest per-row relative error.  Throughput =
    algorithmic 2MNK (8MNK complex) flops / CUDA-event time, device operands."""
    from clgpu_b200 import iclblas as B
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n = args.gemm_n
    modes = [(B.MATH_PLAIN_FP32, "fp32_simt"), (B.MATH_TF32, "tf32"), (B.MATH_BF16X3, "3xbf16"),
             (B.MATH_BF16X6, "6xbf16")]
    stream = torch.cuda.Stream(device=dev)
    g = torch.Generator(device=dev).manual_seed(2)
    results = []
    peak_bf16 = None
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peak_bf16 = json.load(open(pp)).get("bf16_tflops")
    with B.Handle() as h, torch.cuda.stream(stream):
        h.set_stream(stream)
        for cplx in (False, True):
            if cplx and args.skip_cgemm:
                continue
            dt = torch.complex64 if cplx else torch.float32
            fl = (8.0 if cplx else 2.0) * n * n * n

            def rnd(shape):
                t = torch.rand(shape, generator=g, device=dev) * 2 - 1
                if cplx:
                    t = torch.complex(t, torch.rand(shape, generator=g, device=dev) * 2 - 1)
                return t

            A = rnd((n * n,))
            Bm = rnd((n * n,))
            for variant in ("uniform", "row_scaled"):
                if variant == "row_scaled":
                    if cplx:
                        continue
                    sc = 10.0 ** (torch.rand(n, generator=g, device=dev) * 8 - 4)
                    # row i of op(A): A is column-major n x n, element (i, j) at j*n + i
                    As = (A.view(n, n) * sc.view(1, n)).reshape(-1)
                else:
                    As = A
                for ta in (0, 1):
                    # FP64 reference of op(A) @ B (column-major views)
                    Am = As.view(n, n).t()             # Am[i, j] = As[j*n + i]
                    opA = Am if ta == 0 else Am.t()
                    Bmat = Bm.view(n, n).t()
                    ref = (opA.to(torch.complex128 if cplx else torch.float64)
                           @ Bmat.to(torch.complex128 if cplx else torch.float64))
                    refn = torch.linalg.norm(ref).item()
                    for mode, name in modes:
                        if cplx and mode == B.MATH_PLAIN_FP32 and args.quick:
                            continue
                        h.set_math_mode(mode)
                        Cm = torch.empty(n * n, dtype=dt, device=dev)
                        call = (B.iclblasCgemm if cplx else B.iclblasSgemm)
                        one = 1.0 + 0j if cplx else 1.0
                        zero = 0.0
                        for _ in range(1):
                            B.check(call(h, ta, 0, n, n, n, one, As, n, Bm, n, zero, Cm, n), name)
                        torch.cuda.synchronize()
                        reps = 3
                        e0 = torch.cuda.Event(enable_timing=True)
                        e1 = torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        for _ in range(reps):
                            B.check(call(h, ta, 0, n, n, n, one, As, n, Bm, n, zero, Cm, n), name)
                        e1.record(stream)
                        torch.cuda.synchronize()
                        ms = e0.elapsed_time(e1) / reps
                        Cmat = Cm.view(n, n).t().to(ref.dtype)
                        err = (torch.linalg.norm(Cmat - ref).item()) / refn
                        row_err = None
                        if variant == "row_scaled":
                            rerr = torch.linalg.norm(Cmat - ref, dim=1) / torch.linalg.norm(ref, dim=1)
                            row_err = rerr.max().item()
                        r = {"routine": "cgemm" if cplx else "sgemm", "variant": variant,
                             "op": "NN" if ta == 0 else "TN", "mode": name, "n": n,
                             "tflops": round(fl / (ms / 1e3) / 1e12, 2), "ms": round(ms, 3),
                             "rel_fro_err_vs_fp64": err}
                        if row_err is not None:
                            r["max_row_rel_err"] = row_err
                        if mode != B.MATH_PLAIN_FP32 and peak_bf16:
                            nprod = {B.MATH_TF32: 1, B.MATH_BF16X3: 3, B.MATH_BF16X6: 6}[mode]
                            exec_tf = nprod * fl / (ms / 1e3) / 1e12
                            r["tensor_tflops_executed"] = round(exec_tf, 1)
                            if mode != B.MATH_TF32:
                                r["frac_of_bf16_peak_executed"] = round(exec_tf / peak_bf16, 3)
                        print(json.dumps(r), flush=True)
                        results.append(r)
                        del Cm
                    del ref
    return results


# ---------------------------------------------------------------- TRSM / TRSV study
def run_trsm_study(args, torch):
    """Triangular-solve config: STRSM left/lower/N/non-unit M=8192, NRHS=4096
    (L: diagonal U(1,2), strictly lower N(0,1)/sqrt(M); B U(-1,1); seed 3),
    CTRSM upper/conj-trans M=4096, NRHS=2048, and STRSV n=16384 with the same
    L.  TFLOP/s use the algorithmic M^2*N (4*M^2*N complex) flops; STRSV is
    reported in GB/s of the triangle + vector (4n(n+1)/2 + 8n bytes).  Error:
    relative Frobenius error of X against an FP64 solve of the same FP32
    inputs (torch.linalg.solve_triangular in float64, plumbing only)."""
    from clgpu_b200 import iclblas as B
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    g = torch.Generator(device=dev).manual_seed(3)
    modes = [(B.MATH_PLAIN_FP32, "fp32_simt", 0), (B.MATH_TF32, "tf32", 0), (B.MATH_BF16X3, "3xbf16", 0),
             (B.MATH_BF16X6, "6xbf16", 0), (B.MATH_BF16X3, "3xbf16+refine1", 1), (B.MATH_TF32, "tf32+refine2", 2)]
    out = []

    def make_tri(n, lower, cplx):
        L = torch.randn(n, n, generator=g, device=dev) / (n ** 0.5)
        L = torch.tril(L, -1) if lower else torch.triu(L, 1)
        d = torch.rand(n, generator=g, device=dev) + 1.0
        if cplx:
            Li = torch.randn(n, n, generator=g, device=dev) / (n ** 0.5)
            Li = torch.tril(Li, -1) if lower else torch.triu(Li, 1)
            ph = torch.rand(n, generator=g, device=dev) * 6.283185307
            L = torch.complex(L, Li) + torch.diag(torch.polar(d, ph))
        else:
            L = L + torch.diag(d)
        return L  # row-major [i, j] = L(i, j); column-major storage is L.t().contiguous()

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    with B.Handle() as h, torch.cuda.stream(stream):
        h.set_stream(stream)
        for name_r, cplx, m, nrhs, lower, trans in (("strsm", False, args.trsm_m, args.trsm_n, True, 0),
                                                    ("ctrsm", True, 4096, 2048, False, 2)):
            L = make_tri(m, lower, cplx)
            Acm = L.t().contiguous().reshape(-1)          # column-major storage of L
            dt = torch.complex64 if cplx else torch.float32
            B0 = torch.rand(nrhs, m, generator=g, device=dev) * 2 - 1
            if cplx:
                B0 = torch.complex(B0, torch.rand(nrhs, m, generator=g, device=dev) * 2 - 1)
            B0 = B0.reshape(-1)                            # column-major m x nrhs
            Bmat = B0.view(nrhs, m).t()
            op = L if trans == 0 else (L.t() if trans == 1 else L.conj().t())
            X64 = torch.linalg.solve_triangular(op.to(torch.complex128 if cplx else torch.float64),
                                                Bmat.to(torch.complex128 if cplx else torch.float64),
                                                upper=(not lower) if trans == 0 else lower)
            x64n = torch.linalg.norm(X64).item()
            fl = (4.0 if cplx else 1.0) * m * m * nrhs
            for mode, mname, steps in modes:
                h.set_math_mode(mode)
                h.set_trsm_refinement(steps)
                Bw = B0.clone()
                call = B.iclblasCtrsm if cplx else B.iclblasStrsm
                one = (1.0 + 0j) if cplx else 1.0

                def run():
                    Bw.copy_(B0)
                    B.check(call(h, 0, 1 if lower else 0, trans, 0, m, nrhs, one, Acm, m, Bw, m), mname)
                ms = timed(run, 2)
                X = Bw.view(nrhs, m).t().to(X64.dtype)  # result of the last timed call
                # subtract the time of the copy that restores B before each call
                Bt = torch.empty_like(B0)
                ms = max(ms - timed(lambda: Bt.copy_(B0), 3), 1e-6)
                err = torch.linalg.norm(X - X64).item() / x64n
                r = {"routine": name_r, "m": m, "nrhs": nrhs, "mode": mname, "tflops": round(fl / (ms / 1e3) / 1e12, 2),
                     "ms": round(ms, 3), "rel_fro_err_vs_fp64": err}
                print(json.dumps(r), flush=True)
                out.append(r)
            h.set_trsm_refinement(0)
            del L, Acm, B0, X64
        # STRSV n = 16384, lower / N / non-unit, same L construction
        n = args.trsv_n
        L = make_tri(n, True, False)
        Acm = L.t().contiguous().reshape(-1)
        x0 = torch.rand(n, generator=g, device=dev) * 2 - 1
        x64 = torch.linalg.solve_triangular(L.double(), x0.double().view(n, 1), upper=False).view(-1)
        xw = x0.clone()

        def run_v():
            xw.copy_(x0)
            B.check(B.iclblasStrsv(h, 1, 0, 0, n, Acm, n, xw, 1), "strsv")
        h.set_math_mode(B.MATH_PLAIN_FP32)
        ms = timed(run_v, 5)
        assert h.synchronize() == B.SUCCESS
        err = (torch.linalg.norm(xw.double() - x64) / torch.linalg.norm(x64)).item()
        xt = torch.empty_like(x0)
        ms -= timed(lambda: xt.copy_(x0), 5)
        gb = (4.0 * n * (n + 1) / 2 + 8.0 * n) / 1e9
        r = {"routine": "strsv", "n": n, "gbs": round(gb / (ms / 1e3), 1), "ms": round(ms, 4),
             "rel_fro_err_vs_fp64": err}
        print(json.dumps(r), flush=True)
        out.append(r)
    return out


def level1x_bytes(n):
    """Algorithmic bytes per call of the copy / swap / rotation / iamin study
    (every element of each vector read and, where written, written once)."""
    return {
        "scopy": 8 * n, "sswap": 16 * n, "srot": 16 * n, "srotm": 16 * n, "isamin": 4 * n,
        "ccopy": 16 * n, "cswap": 32 * n, "csrot": 32 * n, "crot": 32 * n, "icamin": 8 * n,
    }


def run_level1x_study(args, torch):
    """Copy, swap, rot, rotm and iamin (S and C) at n = --n1 (default 2^28,
    fp32 U(-1,1), seed 2; complex n/2 so every vector is the same 1 GiB):
    per-routine achieved HBM GB/s with device operands, CUDA events on the
    launching stream, inputs far larger than L2.  One JSON line per routine."""
    from clgpu_b200 import iclblas as B
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    g = torch.Generator(device=dev).manual_seed(2)
    n = args.n1
    nc = n // 2
    x = torch.rand(n, generator=g, device=dev) * 2 - 1
    y = torch.rand(n, generator=g, device=dev) * 2 - 1
    xc, yc = x.view(torch.complex64), y.view(torch.complex64)
    param = torch.tensor([-1.0, 0.6, -0.8, 0.8, 0.6], device=dev)
    ri = torch.zeros(1, dtype=torch.int32, device=dev)
    peak, peak_kind = load_peaks()
    n_of = {k: (nc if k.startswith("c") or k == "icamin" else n) for k in level1x_bytes(n)}
    nbytes = {k: level1x_bytes(n_of[k])[k] for k in n_of}
    calls = [
        ("scopy", lambda h: B.iclblasScopy(h, n, x, 1, y, 1)),
        ("sswap", lambda h: B.iclblasSswap(h, n, x, 1, y, 1)),
        ("srot", lambda h: B.iclblasSrot(h, n, x, 1, y, 1, 0.6, 0.8)),
        ("srotm", lambda h: B.iclblasSrotm(h, n, x, 1, y, 1, param)),
        ("isamin", lambda h: B.iclblasIsamin(h, n, x, 1, ri)),
        ("ccopy", lambda h: B.iclblasCcopy(h, nc, xc, 1, yc, 1)),
        ("cswap", lambda h: B.iclblasCswap(h, nc, xc, 1, yc, 1)),
        ("csrot", lambda h: B.iclblasCsrot(h, nc, xc, 1, yc, 1, 0.6, 0.8)),
        ("crot", lambda h: B.iclblasCrot(h, nc, xc, 1, yc, 1, 0.6, 0.48 + 0.64j)),
        ("icamin", lambda h: B.iclblasIcamin(h, nc, xc, 1, ri)),
    ]
    only = set(args.only.split(",")) if args.only else None
    with B.Handle() as h, torch.cuda.stream(stream):
        h.set_stream(stream)
        for name, f in calls:
            if only and name not in only:
                continue
            for _ in range(max(3, args.warmup)):
                B.check(f(h), name)
            reps = max(3, min(args.steps, 50))
            evs = []
            torch.cuda.synchronize()
            for _ in range(reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                B.check(f(h), name)
                e1.record(stream)
                evs.append((e0, e1))
            torch.cuda.synchronize()
            ms = float(np.median([a.elapsed_time(b) for a, b in evs]))
            gbs = nbytes[name] / (ms / 1e3) / 1e9
            print(json.dumps({"routine": name, "n": n_of[name], "ms": round(ms, 4),
                              "gbs": round(gbs, 1), "frac_of_hbm": round(gbs / peak, 3), "peak_kind": peak_kind,
                              "algorithmic_bytes": nbytes[name]}), flush=True)


def run_level23x_study(args, torch):
    """Rank-1 updates, Ssymv / Chemv (HBM GB/s) and the GEMM-shaped level-3
    routines (TFLOP/s in each math mode), device operands, U(-1,1) seed 3,
    median of event-timed calls.  Algorithmic bytes: ger reads and writes A
    (8 mn / 16 mn); symv / hemv read the stored triangle, x and y and write
    y (4 or 8 x (n(n+1)/2 + 3n)).  Algorithmic flops: syrk n^2 k, syr2k
    2 n^2 k, symm 2 m^2 n (left), trmm m^2 n (left); errors are relative
    Frobenius against the same product in FP64 (torch, plumbing only)."""
    from clgpu_b200 import iclblas as B
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    g = torch.Generator(device=dev).manual_seed(3)
    peak, peak_kind = load_peaks()
    only = set(args.only.split(",")) if args.only else None

    def rnd(*shape, dtype=torch.float32):
        t = torch.rand(*shape, generator=g, device=dev) * 2 - 1
        if dtype == torch.complex64:
            t = torch.complex(t, torch.rand(*shape, generator=g, device=dev) * 2 - 1)
        return t

    def timed(h, f, reps):
        for _ in range(3):
            B.check(f(h), "warmup")
        torch.cuda.synchronize()
        evs = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            B.check(f(h), "call")
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        return float(np.median([a.elapsed_time(b) for a, b in evs]))

    with B.Handle() as h, torch.cuda.stream(stream):
        h.set_stream(stream)
        # ---- bandwidth-bound
        n = 16384
        nc = 8192
        A = rnd(n * n)
        x, y = rnd(n), rnd(n)
        Ac = rnd(nc * nc, dtype=torch.complex64)
        xc, yc = rnd(nc, dtype=torch.complex64), rnd(nc, dtype=torch.complex64)
        hbm = [
            ("sger", 8.0 * n * n, lambda hh: B.iclblasSger(hh, n, n, 0.5, x, 1, y, 1, A, n)),
            ("cgeru", 16.0 * nc * nc, lambda hh: B.iclblasCgeru(hh, nc, nc, 0.5 + 0.25j, xc, 1, yc, 1, Ac, nc)),
            ("cgerc", 16.0 * nc * nc, lambda hh: B.iclblasCgerc(hh, nc, nc, 0.5 + 0.25j, xc, 1, yc, 1, Ac, nc)),
            ("ssymv_lower", 4.0 * (n * (n + 1) / 2 + 3 * n),
             lambda hh: B.iclblasSsymv(hh, 1, n, 1.0, A, n, x, 1, 0.5, y, 1)),
            ("ssymv_upper", 4.0 * (n * (n + 1) / 2 + 3 * n),
             lambda hh: B.iclblasSsymv(hh, 0, n, 1.0, A, n, x, 1, 0.5, y, 1)),
            ("chemv_lower", 8.0 * (nc * (nc + 1) / 2 + 3 * nc),
             lambda hh: B.iclblasChemv(hh, 1, nc, 1.0 + 0j, Ac, nc, xc, 1, 0.5 + 0j, yc, 1)),
        ]
        for name, nbytes, f in hbm:
            if only and name not in only:
                continue
            ms = timed(h, f, max(5, min(args.steps, 30)))
            gbs = nbytes / (ms / 1e3) / 1e9
            print(json.dumps({"routine": name, "ms": round(ms, 4), "gbs": round(gbs, 1),
                              "frac_of_hbm": round(gbs / peak, 3), "peak_kind": peak_kind,
                              "algorithmic_bytes": nbytes}), flush=True)
        del A, Ac
        torch.cuda.empty_cache()
        # ---- GEMM-shaped
        N = args.gemm_n if not args.quick else 2048
        K = N
        Aa, Bb, Cc = rnd(N * K), rnd(N * K), rnd(N * N)
        Cw = torch.empty_like(Cc)
        A64 = Aa.view(K, N).t().double()   # column-major N x K operand as a row-major torch matrix
        B64 = Bb.view(K, N).t().double()
        C64 = Cc.view(N, N).t().double()
        refs = {
            "ssyrk": lambda: torch.tril(1.0 * (A64 @ A64.t()) + 0.5 * C64),
            "ssyr2k": lambda: torch.tril(1.0 * (A64 @ B64.t() + B64 @ A64.t()) + 0.5 * C64),
            "ssymm": lambda: (torch.tril(A64) + torch.tril(A64, -1).t()) @ B64 + 0.5 * C64,
            "strmm": lambda: torch.tril(A64) @ B64,
        }
        work = {"ssyrk": float(N) * N * K, "ssyr2k": 2.0 * N * N * K, "ssymm": 2.0 * N * N * N,
                "strmm": float(N) * N * N}
        calls = {
            "ssyrk": lambda hh: B.iclblasSsyrk(hh, 1, 0, N, K, 1.0, Aa, N, 0.5, Cw, N),
            "ssyr2k": lambda hh: B.iclblasSsyr2k(hh, 1, 0, N, K, 1.0, Aa, N, Bb, N, 0.5, Cw, N),
            "ssymm": lambda hh: B.iclblasSsymm(hh, 0, 1, N, N, 1.0, Aa, N, Bb, N, 0.5, Cw, N),
            "strmm": lambda hh: B.iclblasStrmm(hh, 0, 1, 0, 0, N, N, 1.0, Aa, N, Bb, N, Cw, N),
        }
        modes = [("fp32_simt", B.MATH_PLAIN_FP32), ("tf32", B.MATH_TF32), ("3xbf16", B.MATH_BF16X3),
                 ("6xbf16", B.MATH_BF16X6)]
        for name in ("ssyrk", "ssyr2k", "ssymm", "strmm"):
            if only and name not in only:
                continue
            R = refs[name]()
            mask = torch.tril(torch.ones(N, N, dtype=torch.bool, device=dev)) if name.startswith("ssyr") else None
            for mname, mode in modes:
                h.set_math_mode(mode)
                # time the routine alone (the C reset is outside the events)
                ts = []
                for rep in range(4 if not args.quick else 2):
                    Cw.copy_(Cc)
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    B.check(calls[name](h), name)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    if rep > 0:
                        ts.append(e0.elapsed_time(e1))
                ms = float(np.median(ts))
                got = Cw.view(N, N).t().double()
                if mask is not None:
                    err = float(torch.linalg.norm((got - R)[mask]) / torch.linalg.norm(R[mask]))
                else:
                    err = float(torch.linalg.norm(got - R) / torch.linalg.norm(R))
                print(json.dumps({"routine": name, "mode": mname, "n": N, "ms": round(ms, 3),
                                  "tflops": round(work[name] / (ms / 1e3) / 1e12, 2),
                                  "rel_fro_err_vs_fp64": err}), flush=True)
            h.set_math_mode(B.MATH_PLAIN_FP32)


# ResNet-50's 1x1 convolutions as GEMMs (M = batch * H * W, K = input
# channels, N = output channels), batch 32: the shapes the reference's
# experimental/kernels/*.cl target.
CONV1X1_SHAPES = [
    ("56x56 64->256", 32 * 56 * 56, 64, 256), ("56x56 256->64", 32 * 56 * 56, 256, 64),
    ("28x28 128->512", 32 * 28 * 28, 128, 512), ("28x28 512->128", 32 * 28 * 28, 512, 128),
    ("14x14 256->1024", 32 * 14 * 14, 256, 1024), ("14x14 1024->256", 32 * 14 * 14, 1024, 256),
    ("7x7 512->2048", 32 * 7 * 7, 512, 2048), ("7x7 2048->512", 32 * 7 * 7, 2048, 512),
]


def run_conv1x1_study(args, torch):
    """ResNet-50 1x1-convolution GEMMs (activations M x K, weights K x N,
    output M x N; synthetic U(-1,1), seed 5): HGEMM (half storage, FP32
    accumulation) and SGEMM in every math mode.  TFLOP/s = 2 M N K / the
    event time per call of 20 back-to-back calls (median of 3 batches; the
    host work of a call overlaps the previous call's kernels), and
    `single_call_us` = one call between two events (median of 10; includes
    the host work).  Relative Frobenius error against FP64 (torch, plumbing
    only)."""
    from clgpu_b200 import iclblas as B
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    g = torch.Generator(device=dev).manual_seed(5)
    modes = [("fp32_simt", B.MATH_PLAIN_FP32), ("tf32", B.MATH_TF32), ("3xbf16", B.MATH_BF16X3),
             ("6xbf16", B.MATH_BF16X6)]
    with B.Handle() as h, torch.cuda.stream(stream):
        h.set_stream(stream)
        for name, M, K, N in CONV1X1_SHAPES:
            A = torch.rand(K, M, generator=g, device=dev) * 2 - 1     # column-major M x K
            W = torch.rand(N, K, generator=g, device=dev) * 2 - 1     # column-major K x N
            C = torch.empty(N, M, device=dev)
            Ah, Wh, Ch = A.half(), W.half(), torch.empty(N, M, device=dev, dtype=torch.half)
            ref = W.double() @ A.double()          # C^T (N x M) row-major = column-major M x N
            refh = Wh.double() @ Ah.double()
            flops = 2.0 * M * N * K

            def timed(f):
                for _ in range(3):
                    B.check(f(), name)
                torch.cuda.synchronize()
                ts = []
                for _ in range(10):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    B.check(f(), name)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    ts.append(e0.elapsed_time(e1))
                bs = []
                for _ in range(3):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for _ in range(20):
                        B.check(f(), name)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    bs.append(e0.elapsed_time(e1) / 20)
                return float(np.median(bs)), float(np.median(ts))

            def line(extra, ms, single, err):
                d = {"shape": name, "M": M, "K": K, "N": N, **extra, "ms": round(ms, 4),
                     "tflops": round(flops / (ms / 1e3) / 1e12, 1), "single_call_us": round(single * 1e3, 1),
                     "rel_fro_err_vs_fp64": err}
                print(json.dumps(d), flush=True)
            ms, single = timed(lambda: B.iclblasHgemm(h, 0, 0, M, N, K, 1.0, Ah, M, Wh, K, 0.0, Ch, M))
            line({"routine": "hgemm"}, ms, single,
                 float(torch.linalg.norm(Ch.double() - refh) / torch.linalg.norm(refh)))
            for mname, mode in modes:
                h.set_math_mode(mode)
                ms, single = timed(lambda: B.iclblasSgemm(h, 0, 0, M, N, K, 1.0, A, M, W, K, 0.0, C, M))
                line({"routine": "sgemm", "mode": mname}, ms, single,
                     float(torch.linalg.norm(C.double() - ref) / torch.linalg.norm(ref)))
            h.set_math_mode(B.MATH_PLAIN_FP32)
            del A, W, C, Ah, Wh, Ch, ref, refh
            torch.cuda.empty_cache()


def run_batched_study(args, torch, quiet=False):
    """Batched uneven TRSM + adjoint config: 512 instances, n ~ UniformInt[32,1024],
    nrhs ~ UniformInt[1,256], L built as in the STRSM config (diagonal U(1,2),
    strictly lower N(0,1)/sqrt(n)), B and upstream gradients N(0,1), seed 4.
    One step = the forward solve X = L^-1 B (one persistent launch) plus the
    adjoint (dB = L^-T G, one persistent launch; dA = -tril(dB X^T), one
    persistent launch), replayed as one CUDA graph.  Algorithmic flops per
    step: 3 * sum(n^2 * nrhs) (forward n^2 r, adjoint solve n^2 r, the kept
    triangle of dB X^T n^2 r).  Compared with the plain form: the same work as
    per-instance iclblasStrsm + iclblasStrsm_backward calls (PLAIN_FP32).
    Errors: relative Frobenius error of X, dB and dA against FP64 torch
    (solve_triangular and its formulae in float64, plumbing only), worst
    instance."""
    import numpy as np
    from clgpu_b200 import iclblas as B
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    rng = np.random.default_rng(4)
    g = torch.Generator(device=dev).manual_seed(4)
    batch = args.batch
    ns = rng.integers(32, 1025, batch)
    rs = rng.integers(1, 257, batch)
    Ls, As, B0, G0 = [], [], [], []
    for n, r in zip(ns, rs):
        n, r = int(n), int(r)
        L = torch.tril(torch.randn(n, n, generator=g, device=dev) / n ** 0.5, -1)
        L = L + torch.diag(torch.rand(n, generator=g, device=dev) + 1.0)
        Ls.append(L)
        As.append(L.t().contiguous().reshape(-1))             # column-major storage
        B0.append(torch.randn(r, n, generator=g, device=dev).reshape(-1))
        G0.append(torch.randn(r, n, generator=g, device=dev).reshape(-1))
    flops = 3.0 * float(np.sum(ns.astype(np.float64) ** 2 * rs))
    X = [b.clone() for b in B0]
    Gw = [b.clone() for b in G0]
    dA = [torch.empty(int(n) * int(n), device=dev) for n in ns]
    P = lambda ts: torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device=dev)  # noqa: E731
    pA, pX, pG, pdA = P(As), P(X), P(Gw), P(dA)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def restore():
        for x, b in zip(X, B0):
            x.copy_(b)
        for gw, g0 in zip(Gw, G0):
            gw.copy_(g0)

    def errors():
        worst = [0.0, 0.0, 0.0]
        for i in range(batch):
            n, r = int(ns[i]), int(rs[i])
            L64 = Ls[i].double()
            Bm = B0[i].view(r, n).t().double()
            Gm = G0[i].view(r, n).t().double()
            X64 = torch.linalg.solve_triangular(L64, Bm, upper=False)
            W64 = torch.linalg.solve_triangular(L64.t(), Gm, upper=True)
            dA64 = torch.tril(-W64 @ X64.t())
            got = (X[i].view(r, n).t().double(), Gw[i].view(r, n).t().double(), dA[i].view(n, n).t().double())
            for j, (a, b) in enumerate(zip(got, (X64, W64, dA64))):
                worst[j] = max(worst[j], (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item())
        return worst

    out = []
    ms_copy = None
    with B.Handle() as h, torch.cuda.stream(stream):
        h.set_stream(stream)
        modes = [("plain_fp32", B.MATH_PLAIN_FP32), ("bf16x3", B.MATH_BF16X3), ("bf16x6", B.MATH_BF16X6),
                 ("tf32", B.MATH_TF32)]
        for mname, mode in modes:
            if args.math != "all" and mname not in ("plain_fp32", args.math):
                continue
            # a plan takes the handle's math mode at creation
            h.set_math_mode(mode)
            plan = B.BatchPlan(h, "trsm", side=0, uplo=1, trans=0, diag=0, m=[int(v) for v in ns],
                               n=[int(v) for v in rs], lda=[int(v) for v in ns], ldb=[int(v) for v in ns])
            # the adjoint uses the forward call's diagonal-block inverses (same A)
            B.check(plan.set_inverse_reuse(True), "set_inverse_reuse")
            _, width, ctas = plan.info()

            def step():
                B.check(B.iclblasStrsmBatchedUneven(h, plan, 1.0, pA, pX), "batched trsm")
                B.check(B.iclblasStrsmBatchedUnevenBackward(h, plan, 1.0, pA, pX, pG, pdA), "batched adjoint")

            # the restore copies are captured too; their own graph's time is subtracted
            restore()
            torch.cuda.synchronize()
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=stream):
                restore()
                step()
            rgraph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(rgraph, stream=stream):
                restore()
            for _ in range(args.warmup):
                graph.replay()
            reps = max(args.steps, 3)
            ms_all = timed(graph.replay, reps)
            ms_copy = timed(rgraph.replay, reps)
            ms = max(ms_all - ms_copy, 1e-6)
            graph.replay()
            torch.cuda.synchronize()
            ex, eg, ea = errors()
            r = {"routine": "batched strsm fwd+adjoint", "batch": batch, "math": mname,
                 "form": "persistent launches in a CUDA graph" if mode == B.MATH_PLAIN_FP32
                 else "tensor-core launches per block step in a CUDA graph",
                 "tile_width": width, "ctas_per_sm": ctas, "tflops": round(flops / (ms / 1e3) / 1e12, 3),
                 "ms": round(ms, 3), "err_X": ex, "err_dB": eg, "err_dA": ea}
            if not quiet:
                print(json.dumps(r), flush=True)
            out.append(r)
            del graph, rgraph
            plan.destroy()
        if args.math != "all" and not args.batched_loop:
            return out

        # plain form: per-instance calls (PLAIN_FP32)
        h.set_math_mode(B.MATH_PLAIN_FP32)

        def loop_step():
            restore()
            for i in range(batch):
                n, rr = int(ns[i]), int(rs[i])
                B.check(B.iclblasStrsm(h, 0, 1, 0, 0, n, rr, 1.0, As[i], n, X[i], n), "strsm")
                B.check(B.iclblasStrsm_backward(h, 0, 1, 0, 0, n, rr, 1.0, As[i], n, X[i], n, Gw[i], n, dA[i], n),
                        "strsm_backward")
        ms_loop = max(timed(loop_step, 3) - ms_copy, 1e-6)
        ex, eg, ea = errors()
        r = {"routine": "batched strsm fwd+adjoint", "batch": batch, "form": "per-instance calls, plain FP32",
             "tflops": round(flops / (ms_loop / 1e3) / 1e12, 3), "ms": round(ms_loop, 3), "err_X": ex, "err_dB": eg,
             "err_dA": ea}
        if not quiet:
            print(json.dumps(r), flush=True)
        out.append(r)
    return out


def run_batched_leg(torch):
    """The batched config in the default run: the study above (512
    instances, forward + adjoint per step, one CUDA graph per math mode,
    and the same work as per-instance plain calls) without its own output
    lines, under one clock record; returns {form: {tflops, ms, errors,
    x_plain_fp32}, "clocks": ...}."""
    import types
    ns = types.SimpleNamespace(batch=512, steps=5, warmup=3, math="all", batched_loop=True)
    with Clocks(0) as clk:
        t_wait = time.time()
        while not clk.started() and time.time() - t_wait < 5.0:
            time.sleep(0.05)
        clk.mark_start()
        rows = run_batched_study(ns, torch, quiet=True)
        clk.mark_end()
    res = {"config": "batched uneven STRSM forward + adjoint, 512 instances, n ~ UniformInt[32,1024], "
                     "nrhs ~ UniformInt[1,256], seed 4; TFLOP/s = 3 sum n^2 nrhs / step time"}
    plain = next((r["tflops"] for r in rows if r.get("math") == "plain_fp32"), None)
    for r in rows:
        key = r.get("math", "per_instance_plain_fp32")
        res[key] = {k: r[k] for k in ("tflops", "ms", "err_X", "err_dB", "err_dA") if k in r}
        if plain:
            res[key]["x_plain_fp32"] = round(r["tflops"] / plain, 2)
    res["clocks"] = clk.summary()
    return res


# ---------------------------------------------------------------- single-routine cases for profiles
def kernel_cases(torch, dev, B, h):
    """Named single-routine cases (name -> thunk) at sizes larger than L2 and
    a few GB on the device at most, for ncu captures of one kernel each:
    complex level-1 at n = 2^25 (256 MiB per vector), CTRSV 8192, STRSV
    8192 with lda = n (the TMA kernel) and with lda = n + 1 (the kernel for a
    leading dimension TMA cannot address), plain SGEMM and TF32 SGEMM at 4096^3 (the CUDA-core kernel; the
    split pre-pass), STRSM 3xBF16 8192 x 4096 (the FP64 inverse kernels and
    the update GEMMs on operand planes) and the batched TRSM forward + adjoint
    at 128 instances of the batched config's size distribution."""
    g = torch.Generator(device=dev).manual_seed(6)

    def rnd(k, cplx=False):
        t = torch.rand(k, generator=g, device=dev) * 2 - 1
        return torch.complex(t, torch.rand(k, generator=g, device=dev) * 2 - 1) if cplx else t

    nc = 1 << 25
    cx, cy = rnd(nc, True), rnd(nc, True)
    rf = torch.zeros(1, device=dev)
    rc = torch.zeros(1, dtype=torch.complex64, device=dev)
    ri = torch.zeros(1, dtype=torch.int32, device=dev)
    nt = 8192

    def tri(n, cplx):
        L = torch.tril(torch.randn(n, n, generator=g, device=dev) / n ** 0.5, -1) + torch.diag(
            torch.rand(n, generator=g, device=dev) + 1)
        return L.to(torch.complex64) if cplx else L
    Lc = tri(nt, True).t().contiguous().reshape(-1)
    xc = rnd(nt, True)
    Ls = torch.zeros(nt * (nt + 1), device=dev)
    Ls.view(nt, nt + 1)[:, :nt] = tri(nt, False).t()   # column-major, lda = n + 1
    xs = rnd(nt)
    Lt = tri(nt, False).t().contiguous().reshape(-1)    # column-major, lda = n (the TMA path)
    xt = rnd(nt)
    ng = 4096
    Ag, Bg, Cg = rnd(ng * ng), rnd(ng * ng), torch.zeros(ng * ng, device=dev)
    mt, nr = 8192, 4096
    At = tri(mt, False).t().contiguous().reshape(-1)
    Bt0 = rnd(mt * nr)
    Bt = Bt0.clone()
    # batched: 128 instances, n ~ UniformInt[32,1024], nrhs ~ UniformInt[1,256]
    rng = np.random.default_rng(4)
    bn, br = rng.integers(32, 1025, 128), rng.integers(1, 257, 128)
    bA = [tri(int(n), False).t().contiguous().reshape(-1) for n in bn]
    bX = [rnd(int(n) * int(r)) for n, r in zip(bn, br)]
    bG = [rnd(int(n) * int(r)) for n, r in zip(bn, br)]
    bdA = [torch.empty(int(n) * int(n), device=dev) for n in bn]
    P = lambda ts: torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device=dev)  # noqa: E731
    pA, pX, pG, pdA = P(bA), P(bX), P(bG), P(bdA)
    plan = B.BatchPlan(h, "trsm", side=0, uplo=1, trans=0, diag=0, m=[int(v) for v in bn], n=[int(v) for v in br],
                       lda=[int(v) for v in bn], ldb=[int(v) for v in bn])

    def mode_call(mode, f):
        def run():
            h.set_math_mode(mode)
            f()
            h.set_math_mode(B.MATH_PLAIN_FP32)
        return run

    def strsm():
        Bt.copy_(Bt0)
        B.check(B.iclblasStrsm(h, 0, 1, 0, 0, mt, nr, 1.0, At, mt, Bt, mt), "strsm")

    cases = {
        "caxpy": lambda: B.check(B.iclblasCaxpy(h, nc, 0.5 - 0.25j, cx, 1, cy, 1), "caxpy"),
        "cscal": lambda: B.check(B.iclblasCscal(h, nc, 0.5 - 0.25j, cx, 1), "cscal"),
        "cdotu": lambda: B.check(B.iclblasCdotu(h, nc, cx, 1, cy, 1, rc), "cdotu"),
        "cdotc": lambda: B.check(B.iclblasCdotc(h, nc, cx, 1, cy, 1, rc), "cdotc"),
        "scnrm2": lambda: B.check(B.iclblasScnrm2(h, nc, cx, 1, rf), "scnrm2"),
        "scasum": lambda: B.check(B.iclblasScasum(h, nc, cx, 1, rf), "scasum"),
        "icamax": lambda: B.check(B.iclblasIcamax(h, nc, cx, 1, ri), "icamax"),
        "ctrsv": lambda: B.check(B.iclblasCtrsv(h, 1, 0, 0, nt, Lc, nt, xc, 1), "ctrsv"),
        "strsv_lda": lambda: B.check(B.iclblasStrsv(h, 1, 0, 0, nt, Ls, nt + 1, xs, 1), "strsv"),
        "strsv_tma": lambda: B.check(B.iclblasStrsv(h, 1, 0, 0, nt, Lt, nt, xt, 1), "strsv"),
        "sgemm_plain": lambda: B.check(B.iclblasSgemm(h, 0, 0, ng, ng, ng, 1.0, Ag, ng, Bg, ng, 0.0, Cg, ng), "sgemm"),
        "sgemm_tf32": mode_call(B.MATH_TF32, lambda: B.check(
            B.iclblasSgemm(h, 0, 0, ng, ng, ng, 1.0, Ag, ng, Bg, ng, 0.0, Cg, ng), "sgemm")),
        "strsm_3xbf16": mode_call(B.MATH_BF16X3, strsm),
        "batched_trsm": lambda: (B.check(B.iclblasStrsmBatchedUneven(h, plan, 1.0, pA, pX), "batched"),
                                 B.check(B.iclblasStrsmBatchedUnevenBackward(h, plan, 1.0, pA, pX, pG, pdA),
                                         "batched adjoint")),
    }
    return cases, plan


def run_kernel_cases(args, torch):
    """Runs the named cases of kernel_cases (all, or --only a,b): --warmup
    untimed calls, then --steps calls between two CUDA events; one JSON line
    per case."""
    from clgpu_b200 import iclblas as B
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    only = set(args.only.split(",")) if args.only else None
    with B.Handle() as h, torch.cuda.stream(stream):
        h.set_stream(stream)
        cases, plan = kernel_cases(torch, dev, B, h)
        torch.cuda.synchronize()
        for name, f in cases.items():
            if only and name not in only:
                continue
            for _ in range(args.warmup):
                f()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                f()
            e1.record(stream)
            torch.cuda.synchronize()
            assert h.synchronize() == B.SUCCESS
            print(json.dumps({"case": name, "ms_per_call": round(e0.elapsed_time(e1) / max(args.steps, 1), 4)}),
                  flush=True)
        plan.destroy()


# ---------------------------------------------------------------- CPU (reference code)
class CpuSweep:
    """The sweep on the host cores through the reference's own CPU code
    (oracle/_ref/libiclref.so: its double-accumulating templates and serial
    kernels; the oracle port if the reference was not built), on operands of
    the given sizes (default: the full config, n = 2^28, SGEMV 16384^2,
    CGEMV 8192^2).  With threads > 1 every routine is split into
    independent chunks run concurrently (ctypes releases the GIL); the
    chunked reductions' partial results are not combined (timing only)."""

    def __init__(self, threads: int, n=N1, gn=GEMV_N, cn=CGEMV_N):
        import ctypes as C
        import oracle_lib as O
        R = O.ref()
        self.kind = "reference" if R is not None else "port"
        self.threads = threads
        self.sizes = (n, gn, cn)
        rng = np.random.default_rng(1)
        x = rng.random(n, dtype=np.float32) * 2 - 1
        y = rng.random(n, dtype=np.float32) * 2 - 1
        A = rng.random(gn * gn, dtype=np.float32) * 2 - 1
        gx = rng.random(gn, dtype=np.float32) * 2 - 1
        gy = rng.random(gn, dtype=np.float32) * 2 - 1
        CA = (rng.random(2 * cn * cn, dtype=np.float32) * 2 - 1).view(np.complex64)
        cx = (rng.random(2 * cn, dtype=np.float32) * 2 - 1).view(np.complex64)
        cy = (rng.random(2 * cn, dtype=np.float32) * 2 - 1).view(np.complex64)
        self._keep = (x, y, A, gx, gy, CA, cx, cy)
        al = O.cbox(1 + 1j)
        be = O.cbox(0.5)
        self._keep2 = (al, be)
        P = lambda a, off=0: C.c_void_p(a.ctypes.data + off * a.itemsize)  # noqa: E731
        if R is not None:
            self.ops = [
                ("saxpy", lambda o, c: R.ref_cpu_saxpy(c, 0.5, P(x, o), 1, P(y, o), 1), n),
                ("sdot", lambda o, c: R.ref_cpu_sdot(c, P(x, o), 1, P(y, o), 1), n),
                ("snrm2", lambda o, c: R.ref_cpu_snrm2(c, P(x, o), 1), n),
                ("sasum", lambda o, c: R.ref_cpu_sasum(c, P(x, o), 1), n),
                ("isamax", lambda o, c: R.ref_cpu_isamax(c, P(x, o), 1), n),
                # rows of y for op N, columns (outputs) for op T
                ("sgemv_n", lambda o, c: R.ref_naive_sgemv(0, c, gn, 1.0, P(A, o), gn, P(gx), 1, 0.5, P(gy, o), 1), gn),
                ("sgemv_t", lambda o, c: R.ref_naive_sgemv(1, gn, c, 1.0, P(A, o * gn), gn, P(gx), 1, 0.5, P(gy, o), 1), gn),
                ("cgemv_n", lambda o, c: R.ref_naive_cgemv(0, c, cn, P(al), P(CA, o), cn, P(cx), 1, P(be), P(cy, o), 1), cn),
                ("cgemv_c", lambda o, c: R.ref_naive_cgemv(2, cn, c, P(al), P(CA, o * cn), cn, P(cx), 1, P(be), P(cy, o), 1), cn),
            ]
        else:
            Lo = O.orc()
            c32a, c32b = O.c32(1 + 1j), O.c32(0.5)
            self.ops = [
                ("saxpy", lambda o, c: Lo.orc_saxpy(c, 0.5, P(x, o), 1, P(y, o), 1), n),
                ("sdot", lambda o, c: Lo.orc_sdot(c, P(x, o), 1, P(y, o), 1), n),
                ("snrm2", lambda o, c: Lo.orc_snrm2(c, P(x, o), 1), n),
                ("sasum", lambda o, c: Lo.orc_sasum(c, P(x, o), 1), n),
                ("isamax", lambda o, c: Lo.orc_isamax(c, P(x, o), 1), n),
                ("sgemv_n", lambda o, c: Lo.orc_sgemv(0, c, gn, 1.0, P(A, o), gn, P(gx), 1, 0.5, P(gy, o), 1), gn),
                ("sgemv_t", lambda o, c: Lo.orc_sgemv(1, gn, c, 1.0, P(A, o * gn), gn, P(gx), 1, 0.5, P(gy, o), 1), gn),
                ("cgemv_n", lambda o, c: Lo.orc_cgemv(0, c, cn, c32a, P(CA, o), cn, P(cx), 1, c32b, P(cy, o), 1), cn),
                ("cgemv_c", lambda o, c: Lo.orc_cgemv(2, cn, c, c32a, P(CA, o * cn), cn, P(cx), 1, c32b, P(cy, o), 1), cn),
            ]
        self.total_bytes = sum(sweep_bytes(n, gn, cn).values())

    def _par(self, fn, total):
        b = np.linspace(0, total, self.threads + 1).astype(int)
        cs = [(int(b[i]), int(b[i + 1] - b[i])) for i in range(self.threads) if b[i + 1] > b[i]]
        if self.threads == 1:
            for o, c in cs:
                fn(o, c)
            return
        ts = [threading.Thread(target=fn, args=(o, c)) for o, c in cs]
        for t in ts:
            t.start()
        for t in ts:
            t.join()

    def step(self) -> float:
        """One pass of the sweep; returns its wall time in seconds."""
        t0 = time.perf_counter()
        for _, fn, total in self.ops:
            self._par(fn, total)
        return time.perf_counter() - t0

    def describe(self, reps: int) -> str:
        n, gn, cn = self.sizes
        what = ("reference CPU templates + serial kernels (oracle/_ref)" if self.kind == "reference"
                else "oracle port")
        size = ("the full config" if self.sizes == (N1, GEMV_N, CGEMV_N) else
                f"level-1 n={n}, SGEMV {gn}^2 N+T, CGEMV {cn}^2 N+C")
        return f"{size} (level-1 n={n}, SGEMV {gn}^2 N+T, CGEMV {cn}^2 N+C); {reps} timed step(s); {what}"


def cpu_sweep(threads: int, reps: int = 3, warmup: int = 0, sizes=(N1, GEMV_N, CGEMV_N)):
    """Times the sweep on the host cores (CpuSweep): `warmup` untimed steps,
    then `reps` timed ones; value = algorithmic bytes / mean step time."""
    cs = CpuSweep(threads, *sizes)
    for _ in range(warmup):
        cs.step()
    times = [cs.step() for _ in range(reps)]
    t = float(np.mean(times))
    return {
        "value": round(cs.total_bytes / t / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": cs.kind,
        "sample": cs.describe(reps), "seconds_per_step": round(t, 3),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-operand (C ABI) leg")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the SGEMM 8192^3 / STRSM 8192x4096 / SGEMM 512^3 legs of the default run")
    ap.add_argument("--only", default="", help="comma-separated subset of the sweep's calls")
    ap.add_argument("--n1", type=int, default=N1, help="level-1 vector length (default 2^28)")
    ap.add_argument("--workload", default="sweep",
                    choices=["sweep", "gemm", "trsm", "batched", "level1x", "level23x", "conv1x1", "kernels"],
                    help="sweep: the bandwidth config (default); gemm / trsm / batched: the precision, "
                         "triangular-solve and batched-solve config studies; level1x: copy / swap / "
                         "rotation / iamin bandwidth study; level23x: ger / symv / hemv bandwidth and "
                         "syrk / syr2k / symm / trmm throughput study; conv1x1: ResNet-50 1x1-convolution "
                         "GEMM shapes in HGEMM and every SGEMM mode; kernels: named single-routine "
                         "cases (--only) for ncu captures")
    ap.add_argument("--trsm-m", type=int, default=8192)
    ap.add_argument("--trsm-n", type=int, default=4096)
    ap.add_argument("--trsv-n", type=int, default=16384)
    ap.add_argument("--gemm-n", type=int, default=8192)
    ap.add_argument("--skip-cgemm", action="store_true")
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--math", default="all", choices=["all", "bf16x3", "bf16x6", "tf32"],
                    help="batched study: the tensor-core modes to time beside plain FP32")
    ap.add_argument("--batched-loop", action="store_true",
                    help="batched study with --math: also time the per-instance plain calls")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
        res = cpu_sweep(threads, reps=max(1, args.steps), warmup=args.warmup)
        line = {
            "metric": "level-1/2 sweep aggregate HBM bandwidth (SAXPY/SDOT/SNRM2/SASUM/ISAMAX n=2^28, "
                      "SGEMV 16384^2 N+T, CGEMV 8192^2 N+C)",
            "value": res["value"], "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(res["seconds_per_step"] * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic U(-1,1), seed 1",
            "config": {"workload": "bandwidth sweep: level-1 n=2^28 x5, SGEMV 16384^2 N,T, CGEMV 8192^2 N,C",
                       "sample": res["sample"]},
            "impl": "reference",
            "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": res["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import torch
    if args.workload == "gemm":
        run_gemm_study(args, torch)
        return
    if args.workload == "trsm":
        run_trsm_study(args, torch)
        return
    if args.workload == "batched":
        run_batched_study(args, torch)
        return
    if args.workload == "level1x":
        run_level1x_study(args, torch)
        return
    if args.workload == "level23x":
        run_level23x_study(args, torch)
        return
    if args.workload == "conv1x1":
        run_conv1x1_study(args, torch)
        return
    if args.workload == "kernels":
        run_kernel_cases(args, torch)
        return
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    out = run_ours(args, rank, world, torch)
    if world == 1 and not args.only and not args.no_precision:
        from clgpu_b200 import iclblas as B
        out.update(run_precision_legs(torch, torch.device("cuda", 0), B))
        try:
            out["batched_512"] = run_batched_leg(torch)
        except Exception as e:  # reported in the line, never fatal to it
            out["batched_512"] = {"error": repr(e)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.only:
        out["cpu_baseline"] = {k: v for k, v in cpu_sweep(1, reps=2).items() if k != "seconds_per_step"}
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
