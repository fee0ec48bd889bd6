"""Benchmark of the symmetric block-sparse hot path on B200.

Workload (one "step"): the batched block contraction of the fZ2 x U(1) x SU(2)
Hubbard-type configuration -- 64 independent rank-4 tensors
A_i : (W x P) <- (P x W) composed with B_i : (P x W) <- (W x P) -- executed as
ONE grouped launch over every (tensor, coupled sector, output tile).  W has
60 sectors drawn with seed 0 (``tenet_b200.workloads.hubbard_batch``), entries
are N(0,1) f64 from splitmix64 seeds (synthetic data; the reference publishes
no dataset for this path).  FLOPs are counted on reduced (multiplicity)
dimensions: 2 m n k per coupled sector.

Usage:
    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision bf16x|fp64|cublas] [--slices S]
    python bench.py --impl reference ...    # CPU Host-path restatement on the host cores

Prints one JSON line (rank 0).  Under torchrun each rank runs its own
replica of the workload (weak scaling, no data-path collective); time is the
max over ranks of CUDA-event time.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NBATCH = 64
METRIC = "block-contract TFLOP/s"


HEADLINE_WORKLOAD = ("hubbard_batch: 64 composes (W x P)<-(P x W) o (P x W)<-(W x P), fZ2xU1xSU2, "
                     "W = 60 sectors (seed 0, geometric mean 48, clip [1,256])")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="tenet", choices=["tenet", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["bf16x", "i8x", "fp64", "cublas"])
    ap.add_argument("--slices", type=int, default=6)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--nbatch", type=int, default=64, help="tensors per step (64 = the configuration)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="hubbard_batch",
                    choices=["hubbard_batch", "u1_compose_permute", "su2_itebd", "su2_heff", "serve", "transform",
                             "svd", "factor", "plan_compile", "microbench"],
                    help="hubbard_batch is the headline line; the others report the remaining configurations")
    ap.add_argument("--chain-d", type=int, default=2048, help="svd workload: the chain's bond dimension D")
    ap.add_argument("--graph", action="store_true", help="replay the step as a captured CUDA graph")
    ap.add_argument("--no-graph", action="store_true",
                    help="headline: launch the step directly instead of replaying its CUDA graph")
    return ap.parse_args()


def workload():
    from tenet_b200 import workloads

    return workloads.hubbard_batch(0)


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ---------------------------------------------------------------------------
# CPU arm (the oracle's Host-path restatement; numpy BLAS on the host cores)
# ---------------------------------------------------------------------------


def cpu_compose_sample(cfg, ntensors, seed0=1):
    """Time the oracle's per-sector compose on ``ntensors`` of the batch."""
    from oracle.fusion import HomSpace as OHom
    from oracle.fusion import Leg
    from oracle.sectors import Rule
    from oracle.tensor import TensorMap as OT
    from oracle.tensor import normal_fill

    rule = Rule(cfg["factors"])
    W = Leg.new(rule, cfg["W"])
    P = Leg.new(rule, cfg["P"])
    a_sp, b_sp = OHom(rule, [W, P], [P, W]), OHom(rule, [P, W], [W, P])
    flops = 0.0
    for c, r, cc, off in a_sp.sectors:
        j = b_sp.sector_of(c)
        if j is not None:
            flops += 2.0 * r * cc * b_sp.sectors[j][2]
    As = [OT(a_sp, normal_fill(seed0 + i, a_sp.size)) for i in range(ntensors)]
    Bs = [OT(b_sp, normal_fill(seed0 + 1000 + i, b_sp.size)) for i in range(ntensors)]
    t0 = time.perf_counter()
    for a, b in zip(As, Bs):
        a.compose(b)
    dt = time.perf_counter() - t0
    return flops * ntensors, dt


def cpu_threads():
    try:
        from threadpoolctl import threadpool_info

        info = threadpool_info()
        if info:
            return int(max(i.get("num_threads", 1) for i in info))
    except Exception:
        pass
    return os.cpu_count() or 1


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = workload()
    steps = max(1, args.steps)
    sample = 8 if steps <= 20 else 2  # composes per step: the whole run stays within a few minutes
    total_flops, total_t = 0.0, 0.0
    for _ in range(min(args.warmup, 2)):
        cpu_compose_sample(cfg, 1)
    for s in range(steps):
        f, dt = cpu_compose_sample(cfg, sample, seed0=1 + 10 * s)
        total_flops += f
        total_t += dt
    value = total_flops / total_t / 1e12
    cores = cpu_threads()
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "TFLOP/s",
        "n_gpus": args.gpus,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total_t / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": HEADLINE_WORKLOAD, "sample_composes_per_step": sample,
                   "parallelism": "host threads"},
        "cpu_baseline": {
            "value": value, "unit": "TFLOP/s", "cores": cores, "kind": "port",
            "sample": f"{sample} of the 64 composes per step, {steps} steps; numpy restatement "
                      "of the TeNeT Host compose (per-sector GEMM via OpenBLAS)",
        },
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.count(",") >= 7]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        mx = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[4:8]) if "Not" not in v and v.strip()})
        busy = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": float(np.median(busy)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def fp64_peak_tflops(torch):
    """Measured FP64 GEMM throughput of this GPU (cuBLAS DGEMM 8192^3, best of 3)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def main():
    global NBATCH
    args = parse()
    NBATCH = args.nbatch
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload != "hubbard_batch":
        {"u1_compose_permute": run_u1, "su2_itebd": run_itebd, "su2_heff": run_heff, "serve": run_serve,
         "transform": run_transform, "svd": run_svd, "factor": run_factor, "plan_compile": run_plan_compile,
         "microbench": run_microbench}[
            args.workload](args)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import tenet_b200 as tb
    from tenet_b200 import _lib, replicas
    from tenet_b200.workloads import splitmix_normal

    cfg = workload()
    rt = tb.Runtime(local)
    rule = tb.FusionRule(cfg["factors"])
    W, P = tb.GradedSpace(rule, cfg["W"]), tb.GradedSpace(rule, cfg["P"])
    a_sp = rt.space(rule, [W, P], [P, W])
    b_sp = rt.space(rule, [P, W], [W, P])
    plan = rt.cplan(a_sp, b_sp)
    c_size = plan.dst.size
    flops_step = plan.flops * NBATCH

    # Host inputs (pinned) and device-resident copies.
    host_a = torch.empty(NBATCH * a_sp.size, dtype=torch.float64).pin_memory()
    host_b = torch.empty(NBATCH * b_sp.size, dtype=torch.float64).pin_memory()
    for i, (sa_, sb_) in enumerate(replicas.replica_seeds(rank, NBATCH)):
        host_a[i * a_sp.size:(i + 1) * a_sp.size] = torch.from_numpy(splitmix_normal(sa_, a_sp.size))
        host_b[i * b_sp.size:(i + 1) * b_sp.size] = torch.from_numpy(splitmix_normal(sb_, b_sp.size))
    host_c = torch.empty(NBATCH * c_size, dtype=torch.float64).pin_memory()
    dev_a = host_a.to("cuda", non_blocking=True)
    dev_b = host_b.to("cuda", non_blocking=True)
    dev_c = torch.empty(NBATCH * c_size, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    prec = {"bf16x": _lib.PREC_BF16X, "i8x": _lib.PREC_INT8X, "fp64": _lib.PREC_FP64,
            "cublas": _lib.PREC_CUBLAS_FP64}[args.precision]
    stream = torch.cuda.current_stream()
    sptr = C.c_void_p(stream.cuda_stream)

    def launch():
        s_ = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.call("tnt_compose", rt._h, plan._h, NBATCH, C.c_void_p(dev_c.data_ptr()), c_size,
                  C.c_void_p(dev_a.data_ptr()), a_sp.size, C.c_void_p(dev_b.data_ptr()), b_sp.size, 1.0, 0.0,
                  prec, args.slices, s_)

    def step_host():
        _lib.call("tnt_compose_host", rt._h, plan._h, NBATCH, C.c_void_p(host_c.data_ptr()),
                  C.c_void_p(host_a.data_ptr()), C.c_void_p(host_b.data_ptr()), prec, args.slices, sptr)

    # Warm-up (the first compose of the plan calibrates the tile autotuner),
    # then the step is captured once as a CUDA graph and replayed.
    for _ in range(max(3, args.warmup)):
        launch()
    torch.cuda.synchronize()
    graph = None
    if not args.no_graph:
        graph = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream()
        cap.wait_stream(stream)
        with torch.cuda.stream(cap):
            with torch.cuda.graph(graph, stream=cap):
                launch()
        torch.cuda.synchronize()
        step = graph.replay
    else:
        step = launch
    step()
    torch.cuda.synchronize()

    def timed(fn, k):
        replicas.barrier()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(k):
            fn()
        e.record(stream)
        e.synchronize()
        torch.cuda.synchronize()
        return replicas.max_over_ranks(s.elapsed_time(e), device="cuda")

    with ClockSampler(local) as clk:
        ms = timed(step, args.steps)
    clocks = clk.summary()
    rt.sync()  # raises if a device-side pipeline wait gave up during the timed steps
    ms_step = ms / args.steps
    value = flops_step * world / (ms_step * 1e-3) / 1e12

    # End-to-end through the host-buffer C-ABI entry point (H2D + compute + D2H per step).
    step_host()
    e2e_steps = max(1, args.e2e_steps)
    ms_e2e = timed(step_host, e2e_steps) / e2e_steps
    e2e_value = flops_step * world / (ms_e2e * 1e-3) / 1e12

    # The other arithmetic paths on the same inputs: the plain FP64 GPU path
    # of the reference (one cuBLAS DGEMM per coupled sector), the grouped FP64
    # tensor-core kernel, the BF16-split kernel at 5 and 6 slices and the
    # 8-bit-digit kernel at 4, 5 and 6 digits, each with its relative
    # Frobenius error against the grouped FP64 result.
    paths = {}
    ref_c = None
    for name, pr, sl in (("fp64_grouped", _lib.PREC_FP64, 0), ("bf16x5", _lib.PREC_BF16X, 5),
                         ("bf16x6", _lib.PREC_BF16X, 6), ("i8x4", _lib.PREC_INT8X, 4), ("i8x5", _lib.PREC_INT8X, 5),
                         ("i8x6", _lib.PREC_INT8X, 6),
                         ("cublas_per_sector", _lib.PREC_CUBLAS_FP64, 0)):
        def fn(pr=pr, sl=sl):
            _lib.call("tnt_compose", rt._h, plan._h, NBATCH, C.c_void_p(dev_c.data_ptr()), c_size,
                      C.c_void_p(dev_a.data_ptr()), a_sp.size, C.c_void_p(dev_b.data_ptr()), b_sp.size, 1.0, 0.0,
                      pr, sl, sptr)
        for _ in range(3):
            fn()
        k = 3 if pr == _lib.PREC_CUBLAS_FP64 else min(args.steps, 20)
        pms = timed(fn, k) / k
        if ref_c is None:
            ref_c = dev_c.clone()
            err = 0.0
        else:
            err = float(torch.linalg.norm(dev_c - ref_c) / torch.linalg.norm(ref_c))
        paths[name] = {"tflops": flops_step * world / (pms * 1e-3) / 1e12, "ms": pms, "rel_err_vs_fp64": err}
    del ref_c

    # What the tile autotuner measured and picked for this plan.
    costs = (C.c_double * 4)()
    cal, eff64, scal = C.c_int32(), C.c_double(), C.c_int32()
    _lib.call("tnt_tuning_info", local, costs, C.byref(cal), C.byref(eff64), C.byref(scal))
    shp = np.zeros(max(1, plan.njobs), dtype=np.int32)
    _lib.call("tnt_cplan_tile_shapes", plan._h, costs, shp.ctypes.data_as(C.POINTER(C.c_int32)))
    tuning = {"fp64_calibrated": bool(cal.value), "fp64_cost_per_tile_kstep_ms": list(costs),
              "fp64_jobs_per_shape": {n: int((shp[:plan.njobs] == i).sum())
                                      for i, n in enumerate(("64x64", "64x32", "32x64", "32x32"))},
              "split_calibrated": bool(scal.value), "split_eff64": eff64.value}

    peaks, peak_kind = load_peaks()
    split = args.precision in ("bf16x", "i8x")
    if args.precision == "bf16x":
        peak, peak_note = peaks["bf16_tflops"], f"bf16 dense ({peak_kind})"
    elif args.precision == "i8x":
        peak, peak_note = 2.0 * peaks["bf16_tflops"], f"int8 dense = 2 x bf16 dense ({peak_kind})"
    else:
        peak, peak_note = fp64_peak_tflops(torch), "fp64 cuBLAS DGEMM 8192^3 measured in this run"
    achieved = plan.flops * NBATCH / (ms_step * 1e-3) / 1e12
    if split:
        # Tensor-core work: S(S+1)/2 slice products per FP64 product, over
        # the whole step (slicing passes included): a lower bound for the MMA
        # kernel alone.
        achieved *= args.slices * (args.slices + 1) / 2
        peak_note += "; achieved = slice-product MMA rate over the whole step (slicing passes included)"

    traffic = None
    prof = os.path.join(ROOT, "profiles", "compose_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            rec = json.load(f).get(args.precision)
        if rec:
            traffic = rec["dram_bytes_per_compose"] * NBATCH

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        f, dt = cpu_compose_sample(cfg, 8)
        cpu = {"value": f / dt / 1e12, "unit": "TFLOP/s", "cores": cpu_threads(), "kind": "port",
               "sample": "8 of the 64 composes, numpy restatement of the TeNeT Host compose "
                         "(per-sector GEMM via OpenBLAS, all host threads)"}

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "TFLOP/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": max(3, args.warmup),
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": f"{args.precision}{args.slices}->f64" if split else "f64",
        "data": "synthetic",
        "config": {
            "workload": HEADLINE_WORKLOAD,
            "global_batch": NBATCH * world,
            "coupled_sector_gemms_per_compose": plan.njobs,
            "gflop_per_step_per_gpu": flops_step / 1e9,
            "precision": args.precision,
            "slices": args.slices if split else None,
            "l2": "inputs larger than L2 (A, B, C batches %.1f GB)" % (
                8 * NBATCH * (a_sp.size + b_sp.size + c_size) / 1e9),
            "parallelism": f"replicas x{world}",
            "cuda_graph": graph is not None,
            "autotune": tuning,
        },
        "roofline": {
            "bound": "tensor",
            "achieved": achieved,
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "peak_source": peak_note,
        },
        "e2e": {
            "value": e2e_value,
            "unit": "TFLOP/s",
            "h2d_bytes_per_step": 8 * NBATCH * (a_sp.size + b_sp.size),
            "d2h_bytes_per_step": 8 * NBATCH * c_size,
            "ms_per_step": ms_e2e,
        },
        "cpu_baseline": cpu,
        "gpu_launches": args.steps * (5 if split else 1),
        "clocks": clocks,
        "paths": paths,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# the other configurations (one JSON line each; not the headline)
# ---------------------------------------------------------------------------


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _time_steps(torch, fn, steps, warmup, graph=False):
    stream = torch.cuda.current_stream()
    for _ in range(max(3, warmup)):
        fn()
    torch.cuda.synchronize()
    if graph:
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(stream)
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                fn()
        torch.cuda.synchronize()
        run = g.replay
    else:
        run = fn
    run()
    torch.cuda.synchronize()
    a, b = _events(torch)
    a.record()
    for _ in range(steps):
        run()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) / steps


def _line(metric, value, unit, hib, ms, args, config, extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": hib, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config}
    line.update(extra)
    print(json.dumps(line), flush=True)


def run_u1(args):
    """U(1) compose + (1<->3) permute of the 283,392-element rank-4 tensors."""
    import torch

    import tenet_b200 as tb
    from tenet_b200 import _lib
    from tenet_b200.workloads import splitmix_normal, u1_compose_permute

    cfg = u1_compose_permute()
    rt = tb.Runtime(0)
    rule = tb.U1FusionRule()
    V = tb.GradedSpace(rule, [(s[0], d) for s, d in cfg["V"]])
    sp = rt.space(rule, [V, V], [V, V])
    A = tb.TensorMap.from_host(rt, [V, V], [V, V], splitmix_normal(1, sp.size))
    B = tb.TensorMap.from_host(rt, [V, V], [V, V], splitmix_normal(2, sp.size))
    cp = rt.cplan(sp, sp)
    xp = rt.xplan(cp.dst, "permute", [0, 3], [2, 1])
    C_ = torch.empty(cp.dst.size, dtype=torch.float64, device="cuda")
    D_ = torch.empty(xp.dst.size, dtype=torch.float64, device="cuda")
    st = C.c_void_p(0)

    def step():
        s_ = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.call("tnt_compose", rt._h, cp._h, 1, C.c_void_p(C_.data_ptr()), cp.dst.size,
                  C.c_void_p(A.data.data_ptr()), sp.size, C.c_void_p(B.data.data_ptr()), sp.size, 1.0, 0.0,
                  _lib.PREC_FP64, 0, s_)
        _lib.call("tnt_transform", rt._h, xp._h, C.c_void_p(D_.data_ptr()), C.c_void_p(C_.data_ptr()), 1.0, 0.0, s_)

    ms = _time_steps(torch, step, args.steps, args.warmup, graph=args.graph)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle.fusion import HomSpace as OHom
        from oracle.fusion import Leg
        from oracle.sectors import Rule
        from oracle.tensor import TensorMap as OT

        r = Rule(["U1"])
        v = Leg.new(r, cfg["V"])
        osp = OHom(r, [v, v], [v, v])
        a, b = OT(osp, A.to_host()), OT(osp, B.to_host())
        t0 = time.perf_counter()
        n = 0
        while time.perf_counter() - t0 < 5.0:
            a.compose(b).permute([0, 3], [2, 1])
            n += 1
        cpu = {"value": (time.perf_counter() - t0) / n * 1e3, "unit": "ms", "cores": cpu_threads(), "kind": "port",
               "sample": f"{n} full compose+permute steps (numpy restatement of the TeNeT Host path)"}
    _line("compose+permute step latency", ms * 1e3, "us", False, ms, args,
          {"workload": "u1_compose_permute: U(1) V=[4,8,12,8,4], (VxV)<-(VxV), compose then permute (0,3)(2,1)",
           "graph": args.graph, "l2": "tensors (2.3 MB) are L2 resident"},
          {"compose_tflops": cp.flops / (ms * 1e-3) / 1e12, "permute_bytes": xp.bytes_moved, "cpu_baseline": cpu,
           "gpu_launches": 2 * args.steps})


def run_itebd(args):
    """SU(2) two-site iTEBD update (W = [40,64,64,40,16])."""
    import torch

    import tenet_b200 as tb
    from tenet_b200 import itebd
    from tenet_b200.workloads import splitmix_normal, su2_itebd

    cfg = su2_itebd()
    rt = tb.Runtime(0)
    rule = tb.SU2FusionRule()
    W = tb.GradedSpace(rule, [(s[0], d) for s, d in cfg["W"]])
    P = tb.GradedSpace(rule, [(1, 1)])
    n = rt.space(rule, [W, P], [W]).size
    A = tb.TensorMap.from_host(rt, [W, P], [W], splitmix_normal(1, n))
    B = tb.TensorMap.from_host(rt, [W, P], [W], splitmix_normal(2, n))
    G = itebd.heisenberg_gate(rt, rule, P, 0.05)
    trunc = tb.Truncation.space(W)
    res = {}

    def step():
        res["r"] = itebd.bond_update(A, B, G, trunc)

    ms = _time_steps(torch, step, args.steps, args.warmup)
    r = res["r"]
    _line("iTEBD bond update latency", ms * 1e3, "us", False, ms, args,
          {"workload": "su2_itebd: W spins 0..2 [40,64,64,40,16], P spin-1/2, tau 0.05, Truncation::space(W)"},
          {"kept": r.kept, "truncation_error": r.error, "gpu_launches": None})


def run_heff(args):
    """SU(2) effective-Hamiltonian Lanczos (30 iterations), FP64 vs BF16 slices k in {3, 5, 7} and 8-bit
    digits k in {5, 6} (constant operands packed once)."""
    import torch

    import tenet_b200 as tb
    from tenet_b200 import heff, workloads

    rt = tb.Runtime(0)
    cfg = workloads.su2_heff()
    rule, x, L, O, R = heff.workload_tensors(rt, cfg, scale=1)
    H = heff.EffectiveHamiltonian(L, O, R)
    flops = 0.0
    xb = rt.xplan(x.space, "permute", [0], [1, 2])
    for a_sp, b_sp in ((L.space, xb.dst),):
        flops += rt.cplan(a_sp, b_sp).flops
    results = {}
    ref_e, ref_v = None, None
    for prec, k in (("fp64", 0), ("bf16x", 3), ("bf16x", 5), ("bf16x", 7), ("i8x", 5), ("i8x", 6)):
        # One untimed run compiles and uploads the plans, calibrates the tile
        # model and sizes the slice scratch; the timed run repeats it.
        heff.lanczos(H, x, 30, prec, k)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e, v, _, _ = heff.lanczos(H, x, 30, prec, k)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if prec == "fp64":
            ref_e, ref_v = e, v.to_host()
            results["fp64"] = {"seconds": dt, "energy": e}
        else:
            vv = v.to_host()
            verr = min(np.linalg.norm(vv - ref_v), np.linalg.norm(vv + ref_v)) / np.linalg.norm(ref_v)
            results[f"{prec}{k}"] = {"seconds": dt, "energy": e, "energy_rel_err": abs(e - ref_e) / abs(ref_e),
                                    "vector_rel_err": float(verr)}
    _line("Lanczos (30 it) wall time", results["i8x5"]["seconds"], "s", False, results["i8x5"]["seconds"] * 1e3,
          args, {"workload": "su2_heff: x (WxP)<-W, W 2j=0..8 [256..128], L/R (WxM)<-W, M=[2,1], H=B^dag B",
                 "timing": "second of two identical runs per precision (the first compiles and calibrates)"},
          {"results": results, "first_contraction_gflop": flops / 1e9})


def run_transform(args):
    """Recoupling transforms of the effective-Hamiltonian network at full size (HBM-bound)."""
    import torch

    import tenet_b200 as tb
    from tenet_b200 import _lib, heff, workloads

    rt = tb.Runtime(0)
    cfg = workloads.su2_heff()
    rule, x, L, O, R = heff.workload_tensors(rt, cfg, scale=1)
    xb = rt.xplan(x.space, "permute", [0], [1, 2])
    t1 = rt.cplan(L.space, xb.dst).dst
    t1p = rt.xplan(t1, "permute", [0, 3], [1, 2])
    Op = rt.xplan(O.space, "permute", [3, 2], [0, 1])
    t2 = rt.cplan(t1p.dst, Op.dst).dst
    cases = [("t1.permute([0,3],[1,2])", t1p), ("t2.permute([0,3],[1,2])", rt.xplan(t2, "permute", [0, 3], [1, 2])),
             ("x.permute([0],[1,2])", xb)]
    # A transposing permute (destination axis 0 strided in the source), reported beside the
    # headline: U(1) (V x V) <- (V x V), charges -2..2, degeneracies [12, 24, 48, 24, 12], 597 MB moved.
    u1 = tb.FusionRule(["U1"])
    Vu = tb.GradedSpace(u1, [((q,), d) for q, d in zip(range(-2, 3), [12, 24, 48, 24, 12])])
    u1_sp = rt.space(u1, [Vu, Vu], [Vu, Vu])
    extra = [("u1_rank4.permute([0,1],[3,2])", rt.xplan(u1_sp, "permute", [0, 1], [3, 2])),
             ("u1_rank4.permute([2,3],[0,1]) (transposing)", rt.xplan(u1_sp, "permute", [2, 3], [0, 1]))]
    headline_names = {n for n, _ in cases}
    cases = cases + extra
    peaks, kind = load_peaks()
    out = {}
    st = torch.cuda.current_stream()
    sp_ = C.c_void_p(st.cuda_stream)
    best = None
    for name, plan in cases:
        src = torch.randn(plan.src.size, dtype=torch.float64, device="cuda")
        dst = torch.empty(plan.dst.size, dtype=torch.float64, device="cuda")

        def step(plan=plan, src=src, dst=dst):
            _lib.call("tnt_transform", rt._h, plan._h, C.c_void_p(dst.data_ptr()), C.c_void_p(src.data_ptr()),
                      1.0, 0.0, sp_)

        ms = _time_steps(torch, step, args.steps, args.warmup)
        gbs = plan.bytes_moved / (ms * 1e-3) / 1e9
        out[name] = {"elements": plan.src.size, "groups": plan.ngroups, "bytes": plan.bytes_moved, "us": ms * 1e3,
                     "gb_s": gbs, "frac_of_hbm": gbs / peaks["hbm_gbs"]}
        if name in headline_names and (best is None or plan.bytes_moved > best[1].bytes_moved):
            best = (name, plan, ms, gbs)
        del src, dst
    name, plan, ms, gbs = best
    traffic = None
    prof = os.path.join(ROOT, "profiles", "transform_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            rec = json.load(f).get(name)
        if rec:
            traffic = rec["dram_bytes_per_launch"]
    _line("recoupling transform bandwidth", gbs, "GB/s", True, ms, args,
          {"workload": f"su2_heff transforms, headline {name}: {plan.src.size} elements, "
                       f"{plan.ngroups} recoupling groups (SU(2), W 2j=0..8 [256..128], M=[2,1])",
           "l2": "src + dst larger than L2"},
          {"roofline": {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": gbs / peaks["hbm_gbs"], "traffic": traffic,
                        "peak_source": f"hbm copy ({kind})"},
           "cases": out, "gpu_launches": args.steps})


_COMPILE_CHILD = r"""
import sys, time
sys.path.insert(0, {root!r})
from tenet_b200 import typed
sym, work, d = {sym!r}, {work!r}, {d}
if sym == "U1":
    rule = typed.U1FusionRule()
    v = typed.GradedSpace(rule, [(-1, d), (0, d), (1, d)])
else:
    rule = typed.SU2FusionRule()
    v = typed.GradedSpace(rule, [(0, d), (1, d), (2, d)])
t0 = time.perf_counter()
a = typed.HomSpace(rule, [v, v], [v, v])
b = a
if work != "compose":  # swap: B[d c; g h], the source tree transform of B
    xb = typed.TransformPlan(b, "permute", [1, 0], [2, 3], (), 0)
    b = xb.dst
c = typed.ComposePlan(a, b)
if work == "swap+out":  # plus the output transform C[b a; g h]
    typed.TransformPlan(c.dst, "permute", [1, 0], [2, 3], (), 0)
print((time.perf_counter() - t0) * 1e3)
"""


def run_plan_compile(args):
    """Cold host structure compile of the reference's contraction microbench
    workloads (rank-4 V x V <- V x V, d = 16): compose, swap (source tree
    transform), swap+out (plus output transform); each in a fresh process so
    every cache, the SU(2) F-symbol cache included, starts cold.  Host work
    only: spaces, fusion trees, recoupling coefficients and plan tables."""
    out = {}
    for sym in ("U1", "SU2"):
        for work in ("compose", "swap", "swap+out"):
            code = _COMPILE_CHILD.format(root=ROOT, sym=sym, work=work, d=16)
            runs = []
            for _ in range(3):
                r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True)
                runs.append(float(r.stdout.strip().splitlines()[-1]))
            out[f"{sym} {work}"] = sorted(runs)[1]
    _line("cold structure compile", out["SU2 swap+out"], "ms", False, out["SU2 swap+out"], args,
          {"workload": "plan_compile: rank-4 V x V <- V x V, d = 16, U(1) {-1,0,1} and SU(2) {0,1/2,1}; "
                       "median of 3 fresh processes; host CPU only"},
          {"cases_ms": out, "cpu": {"threads": 1}, "gpu_launches": 0})


# The reference's published contraction microbench (Apple silicon, one thread,
# Accelerate BLAS; benchmarks/history/contraction-microbench-2026-07-11.md:50-75),
# microseconds per iteration.
_MICRO_REF_US = {("U1", 4, "compose"): 4.10, ("U1", 16, "compose"): 1886.1, ("SU2", 4, "compose"): 7.19,
                 ("SU2", 16, "compose"): 7741.3, ("SU2", 4, "swap"): 30.02, ("SU2", 16, "swap"): 11915.0,
                 ("SU2", 4, "swap+out"): 44.63, ("SU2", 16, "swap+out"): 15075.6, ("U1", 16, "swap"): 2645.3,
                 ("U1", 16, "swap+out"): 3281.0}


def microbench_network(work):
    """Labels of the microbench contractions: compose C[a b; g h] = A[a b; c d] B[c d; g h],
    swap with B[d c; g h], swap+out with the output C[b a; g h]."""
    from tenet_b200.network import Network

    b_labels = ["c", "d", "g", "h"] if work == "compose" else ["d", "c", "g", "h"]
    out = ["b", "a", "g", "h"] if work == "swap+out" else ["a", "b", "g", "h"]
    return Network([["a", "b", "c", "d"], b_labels], output=out, output_codomain_rank=2)


def run_microbench(args):
    """The reference's contraction microbench on the device: rank-4 V x V <- V x V
    at d = 4 and 16, U(1) {-1,0,1} and SU(2) {0,1/2,1}; each contraction is one
    compiled schedule (operand transform, grouped GEMM, output transform)
    replayed from a CUDA graph, timed with CUDA events over the replays."""
    import torch

    import tenet_b200 as tb
    from tenet_b200.workloads import splitmix_normal

    rt = tb.Runtime(0)
    out = {}
    for sym in ("U1", "SU2"):
        rule = tb.U1FusionRule() if sym == "U1" else tb.SU2FusionRule()
        for d in (4, 16):
            labs = [-1, 0, 1] if sym == "U1" else [0, 1, 2]
            v = tb.GradedSpace(rule, [(x, d) for x in labs])
            n = rt.space(rule, [v, v], [v, v]).size
            A = tb.TensorMap.from_host(rt, [v, v], [v, v], splitmix_normal(1, n))
            B = tb.TensorMap.from_host(rt, [v, v], [v, v], splitmix_normal(2, n))
            for work in ("compose", "swap", "swap+out"):
                plan = microbench_network(work).plan([A, B])
                res = plan.execute([A, B])
                step = lambda plan=plan, res=res: plan.execute([A, B], out=res)
                ms = _time_steps(torch, step, max(args.steps, 50), args.warmup, graph=True)
                ref = _MICRO_REF_US.get((sym, d, work))
                out[f"{sym} d={d} {work}"] = {"us": ms * 1e3, "transforms": plan.n_transforms,
                                              "reference_us": ref, "speedup": ref / (ms * 1e3) if ref else None}
    head = out["SU2 d=16 swap+out"]
    _line("microbench SU2 d=16 swap+out", head["us"], "us", False, head["us"] / 1e3, args,
          {"workload": "microbench: rank-4 V x V <- V x V, d = 4 / 16, U(1) {-1,0,1}, SU(2) {0,1/2,1}; "
                       "compose / swap / swap+out as one device schedule, CUDA-graph replay",
           "l2": "operands L2-resident (at most 9 MB)"},
          {"cases": out, "reference": "TeNeT Host path, Apple silicon, 1 thread, published microbench "
                                      "(not this box)", "gpu_launches": None})


def run_svd(args):
    """Batched Jacobi SVD of one serving chain's bond matrix (the serving loop's dominant kernel)."""
    import torch

    import tenet_b200 as tb
    from tenet_b200 import _lib, itebd, serving
    from tenet_b200.workloads import splitmix_normal

    rt = tb.Runtime(0)
    rule = tb.SU2FusionRule()
    W = serving.chain_bond_space(rule, args.chain_d)
    P = tb.GradedSpace(rule, [(1, 1)])
    n = rt.space(rule, [W, P], [W]).size
    A = tb.TensorMap.from_host(rt, [W, P], [W], splitmix_normal(3, n))
    B = tb.TensorMap.from_host(rt, [W, P], [W], splitmix_normal(4, n))
    bm = itebd.bond_theta(A, B, itebd.heisenberg_gate(rt, rule, P, 0.05))
    plan = rt.fplan(bm.space)
    u = torch.empty(max(1, plan.u_size), dtype=torch.float64, device="cuda")
    s_ = torch.empty(max(1, plan.s_size), dtype=torch.float64, device="cuda")
    v = torch.empty(max(1, plan.v_size), dtype=torch.float64, device="cuda")
    P_ = lambda x: C.c_void_p(x.data_ptr())

    def step():
        _lib.call("tnt_svd", rt._h, plan._h, P_(bm.data), P_(u), P_(s_), P_(v),
                  C.c_void_p(torch.cuda.current_stream().cuda_stream))

    ms = _time_steps(torch, step, args.steps, args.warmup)
    sw = C.c_int32()
    _lib.call("tnt_ctx_svd_sweeps", rt._h, C.byref(sw))
    sizes = [r for _, r, _, _ in bm.space.sectors()]
    _line("batched SVD latency", ms, "ms", False, ms, args,
          {"workload": f"svd: bond matrix of one SU(2) iTEBD chain at D = {args.chain_d} "
                       f"(W spins 0..3), sectors {sizes}"},
          {"jacobi_sweeps": sw.value, "sum_n3": float(sum(x ** 3 for x in sizes)), "gpu_launches": args.steps})


def run_factor(args):
    """Per-sector factorisations against the reference's device route.

    The reference factorises each coupled sector on the device through
    cuSOLVER, one call per sector in sector order (tenet-dense/src/cuda_adapter.rs:
    563 cuda_svd_region, 607 QR, 673 eigh).  Here the same per-sector cuSOLVER
    calls (torch.linalg.svd / qr / eigh on each sector block, a comparison arm
    only) are timed beside tnt_svd, tnt_qr and tnt_eigh on the config-2 iTEBD
    bond matrix and on the D = 2048 serving chain's bond matrix; eigh runs on
    M^dagger M (square, symmetric sectors).
    """
    import torch

    import tenet_b200 as tb
    from tenet_b200 import _lib, itebd, serving, workloads
    from tenet_b200.workloads import splitmix_normal

    rt = tb.Runtime(0)
    rule = tb.SU2FusionRule()
    P = tb.GradedSpace(rule, [(1, 1)])
    st = lambda: C.c_void_p(torch.cuda.current_stream().cuda_stream)
    ptr = lambda x: C.c_void_p(x.data_ptr())
    cfg2 = workloads.su2_itebd()
    cases = {"itebd_config2": tb.GradedSpace(rule, [(s_[0], d) for s_, d in cfg2["W"]]),
             "serving_D2048": serving.chain_bond_space(rule, 2048)}
    out = {}
    for name, W in cases.items():
        n = rt.space(rule, [W, P], [W]).size
        A = tb.TensorMap.from_host(rt, [W, P], [W], splitmix_normal(3, n))
        B = tb.TensorMap.from_host(rt, [W, P], [W], splitmix_normal(4, n))
        M = itebd.bond_theta(A, B, itebd.heisenberg_gate(rt, rule, P, 0.05))
        Hm = M.adjoint().compose(M)
        res = {}
        for kind, T in (("svd", M), ("qr", M), ("eigh", Hm)):
            plan = rt.fplan(T.space)
            u = torch.empty(max(1, plan.u_size), dtype=torch.float64, device="cuda")
            s_ = torch.empty(max(1, plan.s_size), dtype=torch.float64, device="cuda")
            v = torch.empty(max(1, plan.v_size), dtype=torch.float64, device="cuda")
            if kind == "svd":
                ours = lambda: _lib.call("tnt_svd", rt._h, plan._h, ptr(T.data), ptr(u), ptr(s_), ptr(v), st())
            elif kind == "qr":
                ours = lambda: _lib.call("tnt_qr", rt._h, plan._h, ptr(T.data), ptr(u), ptr(v), st())
            else:
                ours = lambda: _lib.call("tnt_eigh", rt._h, plan._h, ptr(T.data), ptr(u), ptr(s_), None, st())
            blocks = [T.data[off: off + r * c].view(c, r).t() for _, r, c, off in T.space.sectors() if r * c > 0]
            lib_fn = {"svd": lambda X: torch.linalg.svd(X, full_matrices=False),
                      "qr": lambda X: torch.linalg.qr(X, mode="reduced"), "eigh": torch.linalg.eigh}[kind]

            def per_sector(blocks=blocks, lib_fn=lib_fn):
                for X in blocks:
                    lib_fn(X)

            res[kind] = {"tnt_ms": _time_steps(torch, ours, max(3, args.steps // 10), 3),
                         "cusolver_per_sector_ms": _time_steps(torch, per_sector, max(3, args.steps // 10), 3)}
            res[kind]["speedup"] = res[kind]["cusolver_per_sector_ms"] / res[kind]["tnt_ms"]
            if kind in ("svd", "eigh"):
                # Spectra against the comparator's, sector by sector (relative Frobenius over all values).
                ours()
                torch.cuda.synchronize()
                got, ref = [], []
                for m_, n_, k_, aoff, _, soff, _, _ in plan.records:
                    if m_ * n_ == 0:
                        continue
                    X = T.data[aoff: aoff + m_ * n_].view(n_, m_).t()
                    got.append(torch.sort(s_[soff: soff + k_]).values)
                    ref.append(torch.sort(torch.linalg.eigvalsh(X) if kind == "eigh" else torch.linalg.svdvals(X)).values)
                got, ref = torch.cat(got), torch.cat(ref)
                res[kind]["rel_err_vs_cusolver"] = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
            else:
                # Q R against the input and Q^T Q against the identity, worst sector.
                ours()
                torch.cuda.synchronize()
                rec, orth = 0.0, 0.0
                for m_, n_, k_, aoff, uoff, _, voff, _ in plan.records:
                    if m_ * n_ == 0:
                        continue
                    X = T.data[aoff: aoff + m_ * n_].view(n_, m_).t()
                    Qm = u[uoff: uoff + m_ * k_].view(k_, m_).t()
                    Rm = v[voff: voff + k_ * n_].view(n_, k_).t()
                    rec = max(rec, float(torch.linalg.norm(Qm @ Rm - X) / torch.linalg.norm(X)))
                    eye = torch.eye(k_, dtype=torch.float64, device=X.device)
                    orth = max(orth, float(torch.linalg.norm(Qm.t() @ Qm - eye)))
                res[kind]["rel_err_qr_vs_input"] = rec
                res[kind]["orthogonality_err"] = orth
        out[name] = {"sectors": [r for _, r, _, _ in M.space.sectors()], **res}
    head = out["serving_D2048"]["svd"]
    _line("batched SVD latency vs per-sector cuSOLVER", head["tnt_ms"], "ms", False, head["tnt_ms"], args,
          {"workload": "factor: config-2 iTEBD bond matrix and the D = 2048 serving chain's bond matrix; "
                       "svd / qr of M, eigh of M^dagger M",
           "comparator": "torch.linalg per sector (cuSOLVER), the reference's cuda_adapter route"},
          {"results": out})


def run_serve(args):
    """256 SU(2) iTEBD chains served two ways (continuous lanes, ticks); Poisson arrival rates swept."""
    import torch

    import tenet_b200 as tb
    from tenet_b200 import serving

    nchains = 256
    free, total = torch.cuda.mem_get_info()
    budget = int(min(160e9, free - 8e9))  # every tensor, workspace and slice pack of the service is in the arena
    mix = serving.chain_mix(nchains, seed=0)
    out = {}
    for prec, slices in (("fp64", 0), ("i8x", 6)):
        rt = tb.Runtime(0)
        loop = serving.ServingLoop(rt, budget, prec, slices, lanes=4)
        for i, (D, tau) in enumerate(mix):
            loop.add_chain(D, tau, seed=i)
        # warm-up of both schedulers: plans, tile calibration, lane scratch
        warm = [serving.Request(i, i % nchains, 0.0) for i in range(nchains)]
        wdone, _ = loop.serve_ticks(warm)
        first_err = {r.cid: r.err for r in wdone}
        loop.serve([serving.Request(i, i % nchains, 0.0) for i in range(nchains)])
        res = {}
        for mode, fn in (("continuous", loop.serve), ("ticks", loop.serve_ticks)):
            # closed-loop capacity: every request queued at t = 0
            cap_reqs = [serving.Request(i, i % nchains, 0.0) for i in range(2 * nchains)]
            done, wall = fn(cap_reqs)
            res[mode] = {"capacity_updates_per_s": len(done) / wall}
        rate_base = max(v["capacity_updates_per_s"] for v in res.values())
        for mode, fn in (("continuous", loop.serve), ("ticks", loop.serve_ticks)):
            sweep = []
            for frac in (0.25, 0.5, 0.75, 0.9):
                reqs = serving.poisson_requests(nchains, 3 * nchains, rate=frac * rate_base, seed=int(frac * 100))
                done, wall = fn(reqs)
                lat = np.array([r.done - r.arrival for r in done]) * 1e3
                sweep.append({"rate_per_s": frac * rate_base, "p50_ms": float(np.percentile(lat, 50)),
                              "p99_ms": float(np.percentile(lat, 99)), "updates_per_s": len(done) / wall})
            res[mode]["sweep"] = sweep
        out[f"{prec}{slices or ''}"] = res
        out[f"{prec}{slices or ''}"]["first_update_err"] = first_err
        del loop, fn  # the bound method holds the loop (and its arena) too
        import gc

        gc.collect()
        torch.cuda.empty_cache()
    e64, es = out["fp64"].pop("first_update_err"), out["i8x6"].pop("first_update_err")
    out["max_rel_trunc_err_diff"] = max(abs(es[c] - e64[c]) / max(abs(e64[c]), 1e-300) for c in e64)
    p99 = out["i8x6"]["continuous"]["sweep"][0]["p99_ms"]
    _line("serve p99 latency per iTEBD update", p99, "ms", False, p99, args,
          {"workload": "serve: 256 SU(2) iTEBD chains, D log-uniform [32,2048] split over spins 0..3, "
                       "tau in {0.01,0.05,0.1}, Poisson arrivals", "budget_bytes": budget,
           "headline": "8-bit digits x6, continuous scheduler (4 lanes), lowest offered rate"},
          {"results": out})


if __name__ == "__main__":
    main()
