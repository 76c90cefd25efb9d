"""Benchmark: GFLOP/s of the symmetric contraction path on B200.

Default workload (one GPU): the large SU(2) environment update
    En[a;b] := conj(A[c,p;a]) * E[c;d] * A[d,p;b]
with V = SU(2) spins 0..3 (step 1/2), degeneracies {32,48,40,24,12,6,2}×8 (dim 3632),
P = spin 1/2; Float64, seeded synthetic data. A step is one whole contraction (two
pairwise tensorcontract! = 4 transforms + 2 grouped GEMMs), replayed as a CUDA graph.
`value` is the split-precision (int8 tensor-core slices, FP64 recombination) GFLOP/s,
`plain_fp64` the plain FP64 (DMMA) GFLOP/s of the same step. L2 (126 MB) is flushed
between timed steps by writing a 256 MB buffer outside the timed events.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--workload su2_large|u1_heff|su2_env|u1_small] [--breakdown]
Multi-GPU (torchrun, one process per GPU): replicas only — every rank runs its own
contractions, the step time is the max over ranks, `value` the total over ranks.
"""
from __future__ import annotations

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
for _p in (ROOT, os.path.join(ROOT, "tensorkit.jl_b200"), os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "U1/SU2 contract GFLOP/s: split-prec TC vs plain FP64, 1 B200, <=1e-12 rel err"

WORKLOADS = {
    "su2_large": dict(expr="En[a;b] := conj(A[c,p;a])*E[c;d]*A[d,p;b]",
                      desc="SU(2) environment update, V dim 3632 (degeneracies x8), P = 1/2, Float64"),
    "su2_env": dict(expr="En[a;b] := conj(A[c,p;a])*E[c;d]*A[d,p;b]",
                    desc="SU(2) environment update, V dim 454, P = 1/2, Float64"),
    "u1_heff": dict(expr="y[a,p,q;b] := L[a,w;c]*x[c,r,s;d]*W1[w,p;r,v]*W2[v,q;s,u]*R[d,u;b]",
                    desc="U(1) two-site effective Hamiltonian, V dim 1924, W = {-1:2,0:3,1:2}, Float64"),
    "u1_small": dict(expr="C[a,p,q;b] := A[a,p;c]*B[c,q;b]",
                     desc="U(1) small, V dim 56, P = {-1,0,1}, Float64"),
}


def oracle_inputs(name, complex_=False):
    from helpers import O, cfg1_spaces, cfg2_spaces, cfg3_spaces
    if name in ("su2_large", "su2_env"):
        V, Pp = cfg2_spaces(8 if name == "su2_large" else 1)
        seed = 3 if name == "su2_large" else 1
        return {"A": O.randn(O.Hom([V, Pp], [V]), seed, complex_), "E": O.randn(O.Hom([V], [V]), seed, complex_)}
    if name == "u1_heff":
        V, Pp, Wm = cfg3_spaces()
        Wd = Wm.flipdual()
        return {"L": O.randn(O.Hom([V, Wd], [V]), 2), "x": O.randn(O.Hom([V, Pp, Pp], [V]), 2),
                "W1": O.randn(O.Hom([Wm, Pp], [Pp, Wm]), 2), "W2": O.randn(O.Hom([Wm, Pp], [Pp, Wm]), 2),
                "R": O.randn(O.Hom([V, Wm], [V]), 2)}
    V, Pp = cfg1_spaces()
    W = O.Hom([V, Pp], [V])
    return {"A": O.randn(W, 0), "B": O.randn(W, 0)}


def oracle_eval(name, tensors):
    from oracle import core as O
    from tensorkit_b200.tensoroperations import parse_tensor_expr
    _, lhs, _, factors = parse_tensor_expr(WORKLOADS[name]["expr"])
    return O.network(factors, lhs, tensors)


# ---- clocks ------------------------------------------------------------------------------
LOAD_S = 0.6
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_samples(self, n, timeout=5.0):
        """Block until the sampler has produced n lines (nvidia-smi takes a moment to start)."""
        t0 = time.perf_counter()
        while self.proc is not None and len(self.lines) < n and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- reference arm (CPU) -------------------------------------------------------------------
def run_reference(args):
    """The reference's path on the host cores: the oracle restatement of TensorKit's CPU
    algorithm (Julia is not available), numpy/BLAS with every host thread."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    tens = oracle_inputs(args.workload)
    oracle_eval(args.workload, tens)  # warm caches (symbols, layouts)
    flops = workload_flops(args.workload)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle_eval(args.workload, tens)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    tot = sum(times)
    v = flops * len(times) / tot / 1e9
    cores = os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64 normals)",
            "config": {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"]},
            "cpu_baseline": {"value": v, "unit": "GFLOP/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} full contractions, numpy/BLAS on {cores} host threads"},
            "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


_FLOPS = {}


def workload_flops(name):
    """Algorithmic flops (Σ 2mnk over the block GEMMs) of one step, from the host plans."""
    if name in _FLOPS:
        return _FLOPS[name]
    from oracle import core as O
    from tensorkit_b200.tensoroperations import parse_tensor_expr
    tens = oracle_inputs(name)
    _, lhs, _, factors = parse_tensor_expr(WORKLOADS[name]["expr"])
    # count on the oracle's pairwise GEMMs: instrument O.mul
    total = [0.0]
    orig = O.mul

    def counting(A, B, adjA=False, adjB=False):
        C = orig(A, B, adjA, adjB)
        WA = A.W.adjoint() if adjA else A.W
        bA = O.layout(WA)
        for c, (d1, d2, _) in O.layout(C.W)[1].items():
            if c in bA[1]:
                k = bA[1][c][1]
                total[0] += 2.0 * d1 * d2 * k * (4 if C.data.dtype.kind == "c" else 1)
        return C
    O.mul = counting
    try:
        O.network(factors, lhs, tens)
    finally:
        O.mul = orig
    _FLOPS[name] = total[0]
    return total[0]


def rel_errors(got, ref):
    """Normwise max|Δ|/max|ref| and the largest elementwise |Δ|/|ref| over the entries with
    |ref| above 1e-3·max|ref|."""
    import numpy as np
    got, ref = np.asarray(got), np.asarray(ref)
    den = np.abs(ref).max()
    big = np.abs(ref) > 1e-3 * den
    elem = float((np.abs(got - ref)[big] / np.abs(ref)[big]).max()) if big.any() else 0.0
    return {"normwise": float(np.abs(got - ref).max() / den), "elementwise_above_1e-3_max": elem}


def graph_plans(expr, inputs):
    """Captured split and plain NetworkPlans of one expression, with the launch logs of their
    eager runs."""
    import tensorkit_b200 as tk
    from tensorkit_b200 import indexmanipulations as IM
    plans, logs = {}, {}
    for prec in ("split", "plain"):
        p = tk.NetworkPlan(expr, precision=prec, **inputs)
        IM.LAUNCH_LOG = []
        p.run_eager()
        logs[prec] = IM.LAUNCH_LOG
        IM.LAUNCH_LOG = None
        plans[prec] = p.capture()
    return plans, logs


def time_replays(plan, stream, n, warm=3):
    """Mean device time of one of n back-to-back graph replays (CUDA events on the library stream)."""
    import torch
    with torch.cuda.stream(stream):
        for _ in range(warm):
            plan.replay()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            plan.replay()
        b.record(stream)
        stream.synchronize()
    return a.elapsed_time(b) / n


def split_slices(log):
    """Slice counts per block and FP64-checked tiles of every split grouped GEMM of a step."""
    out = []
    for e in log:
        if e[0] == "gemm" and e[1].slices:
            sl, fb = e[1].last_slices()
            out.append({"slices": sorted(set(x for x in sl if x >= 0)), "fp64_checked_tiles": fb})
    return out


def other_configs(dev, ctx, flush):
    """The other BASELINE configurations, measured in the same run as extra keys:
    - su2_large_c128: the large SU(2) contraction in ComplexF64 (real-equivalent flops, 4 per
      complex multiply-add), graph replays with the L2 flushed before each, split and plain;
    - u1_heff: the U(1) two-site effective Hamiltonian as 100 back-to-back graph replays per
      precision (its working set exceeds L2), GFLOP/s and ms/application, and its three large
      permutes re-timed alone after the bench's write flush and after a clean flush;
    - ad_u1su2: forward + backward (hand-written adjoint kernels) of the U(1)⊠SU(2) loss, eager,
      ms per step."""
    import torch
    from helpers import to_device
    out = {}
    stream = ctx.stream

    def flushed_ms(plan, reps=10):
        with torch.cuda.stream(stream):
            for _ in range(3):
                plan.replay()
            evs = []
            for _ in range(reps):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                plan.replay()
                b.record(stream)
                evs.append((a, b))
            stream.synchronize()
        return statistics.mean(x.elapsed_time(y) for x, y in evs)

    # ComplexF64 large SU(2)
    tens = oracle_inputs("su2_large", complex_=True)
    inputs = {k: to_device(v, dev) for k, v in tens.items()}
    plans, logs = graph_plans(WORKLOADS["su2_large"]["expr"], inputs)
    flops = sum(e[1].flops for e in logs["plain"] if e[0] == "gemm")
    ms = {k: flushed_ms(p) for k, p in plans.items()}
    ref = oracle_eval("su2_large", tens).data
    out["su2_large_c128"] = {
        "flops_per_step": flops, "unit": "GFLOP/s (real-equivalent)",
        "split": {"value": flops / (ms["split"] * 1e-3) / 1e9, "ms_per_step": ms["split"],
                  "max_rel_err": rel_errors(plans["split"].output.to_host(), ref),
                  "slices": split_slices(logs["split"])},
        "plain": {"value": flops / (ms["plain"] * 1e-3) / 1e9, "ms_per_step": ms["plain"],
                  "max_rel_err": rel_errors(plans["plain"].output.to_host(), ref)},
        "split_over_plain": ms["plain"] / ms["split"],
        "l2": "flushed (256 MB write) before every replay"}
    for p in plans.values():
        p.free()

    # U(1) two-site effective Hamiltonian, 100 replays
    tens = oracle_inputs("u1_heff")
    inputs = {k: to_device(v, dev) for k, v in tens.items()}
    plans, logs = graph_plans(WORKLOADS["u1_heff"]["expr"], inputs)
    flops = sum(e[1].flops for e in logs["plain"] if e[0] == "gemm")
    ms = {k: time_replays(p, stream, 100) for k, p in plans.items()}
    ref = oracle_eval("u1_heff", tens).data
    hbm = _peaks()[0][0]
    perms = []
    for e in logs["split"]:
        if e[0] != "transform":
            continue
        t = e[1]
        el = e[2].data.element_size()
        nbytes = el * (t.elems_read + t.elems_written * (1 if e[5] == 0 else 2))
        if nbytes < (64 << 20):
            continue
        m_w = _retime(e, stream, flush, 10, clean=False)
        m_c = _retime(e, stream, flush, 10, clean=True)
        perms.append({"bytes": nbytes, "ms": m_w, "gbs": nbytes / (m_w * 1e-3) / 1e9,
                      "frac_hbm": nbytes / (m_w * 1e-3) / 1e9 / hbm, "ms_clean_l2": m_c,
                      "frac_hbm_clean_l2": nbytes / (m_c * 1e-3) / 1e9 / hbm})
    out["u1_heff"] = {
        "flops_per_application": flops, "applications": 100,
        "split": {"gflops": flops / (ms["split"] * 1e-3) / 1e9, "ms_per_application": ms["split"],
                  "max_rel_err": rel_errors(plans["split"].output.to_host(), ref),
                  "slices": split_slices(logs["split"])},
        "plain": {"gflops": flops / (ms["plain"] * 1e-3) / 1e9, "ms_per_application": ms["plain"],
                  "max_rel_err": rel_errors(plans["plain"].output.to_host(), ref)},
        "split_over_plain": ms["plain"] / ms["split"],
        "large_permutes": perms,
        "timing": "100 back-to-back graph replays (working set above L2), CUDA events"}
    for p in plans.values():
        p.free()

    # AD step, U(1)xSU(2) (config 5)
    import tensorkit_b200 as tk
    from tensorkit_b200 import chainrules as CR
    from helpers import cfg5_spaces, O
    V, Pp = cfg5_spaces()
    tens = {"A": O.randn(O.Hom([V, Pp], [V]), 4, True), "EL": O.randn(O.Hom([V], [V]), 41, True),
            "ER": O.randn(O.Hom([V], [V]), 42, True)}
    ad_in = {k: to_device(v, dev) for k, v in tens.items()}
    expr = "f[] := EL[a;c]*A[c,p;d]*ER[d;b]*conj(A[a,p;b])"

    def step():
        o, pb = CR.network_with_pullback(expr, **ad_in)
        return pb(tk.TensorMap(torch.ones(1, dtype=o.data.dtype, device=o.data.device), o.space))

    for _ in range(3):
        step()
    torch.cuda.synchronize(dev)
    times = []
    for _ in range(10):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record(stream)
        step()
        b.record(stream)
        torch.cuda.synchronize(dev)
        times.append(a.elapsed_time(b))
    out["ad_u1su2"] = {"ms_per_step": statistics.median(times),
                       "step": "forward + pullback of f = real(tr(E_L*A*E_R*A')) through the hand-written "
                               "adjoint kernels, eager launches from the host, ComplexF64",
                       "checked": "gradients vs central differences and the oracle's rule: tests/test_gpu_ad.py"}
    return out


def _peaks():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        src = "measured"
    except Exception:
        peaks, src = {}, "fallback"
    return (peaks.get("hbm_gbs", 6650.0), peaks.get("bf16_tflops", 1590.0)), src


def _retime(e, stream, flush, reps, clean):
    """Mean device time of relaunching one logged library call after a 256 MB write flush
    (clean: the flush buffer is read back too, so no write-back of the flush lands in the call)."""
    import torch
    from tensorkit_b200.indexmanipulations import relaunch
    sink = torch.zeros(1, dtype=torch.int64, device=flush.device)
    with torch.cuda.stream(stream):
        for _ in range(3):
            relaunch(e)
        evs = []
        for _ in range(reps):
            flush.zero_()
            if clean:
                sink.copy_(flush.view(torch.int64).sum().view(1))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            relaunch(e)
            b.record(stream)
            evs.append((a, b))
        stream.synchronize()
    return statistics.mean(x.elapsed_time(y) for x, y in evs)


def dgemm_tflops(dev, n=4096):
    """cuBLAS DGEMM (torch.matmul, float64) on n×n×n in this run: the FP64 tensor-core reference rate."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        torch.matmul(a, b)
    e1.record()
    torch.cuda.synchronize(dev)
    return 2.0 * n ** 3 * 5 / (e0.elapsed_time(e1) * 1e-3) / 1e12


# ---- our arm -------------------------------------------------------------------------------
def max_over_ranks(ms, device, world):
    """The slowest rank's time: every rank takes part in one MAX all-reduce (NCCL on GPUs,
    gloo on host tensors), so all ranks return the same value."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(flops_per_step, world, steps, ms):
    """GFLOP/s of the whole job: every rank runs `steps` steps of `flops_per_step` (weak scaling,
    replicas), timed by the slowest rank's `ms` for all its steps."""
    return flops_per_step * world * steps / (ms * 1e-3) / 1e9


def parse_cpulist(text):
    """CPU numbers of a sysfs cpulist such as "0-27,56-83"."""
    cpus = set()
    for part in text.strip().split(","):
        if part:
            a, _, b = part.partition("-")
            cpus.update(range(int(a), int(b or a) + 1))
    return cpus


def gpu_numa_cpus(dev_index):
    """(NUMA node, its CPUs this process may use) for the node the GPU's PCIe function sits on,
    from sysfs; (None, None) where the system does not say."""
    import torch
    try:
        p = torch.cuda.get_device_properties(dev_index)
        bdf = f"{p.pci_domain_id:04x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        with open(f"/sys/bus/pci/devices/{bdf}/numa_node") as f:
            node = int(f.read().strip())
        if node < 0:
            return None, None
        with open(f"/sys/devices/system/node/node{node}/cpulist") as f:
            cpus = parse_cpulist(f.read()) & os.sched_getaffinity(0)
        return (node, cpus) if cpus else (None, None)
    except (OSError, ValueError, AttributeError):
        return None, None


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    import tensorkit_b200 as tk
    from helpers import to_device
    from tensorkit_b200 import linalg as LA

    dev = torch.device("cuda", local)
    tens_o = oracle_inputs(args.workload)
    inputs = {k: to_device(v, dev) for k, v in tens_o.items()}
    expr = WORKLOADS[args.workload]["expr"]
    ctx = tk.get_context(local)
    stream = ctx.stream

    from tensorkit_b200 import indexmanipulations as IM
    plans = {}
    logs = {}
    for prec in ("split", "plain"):
        p = tk.NetworkPlan(expr, precision=prec, **inputs)
        IM.LAUNCH_LOG = []
        p.run_eager()
        logs[prec] = IM.LAUNCH_LOG
        IM.LAUNCH_LOG = None
        plans[prec] = p.capture()
    flops = sum(e[1].flops for e in logs["plain"] if e[0] == "gemm")

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def timed(plan, steps, warm, clk=None):
        with torch.cuda.stream(stream):
            for _ in range(warm):
                plan.replay()
            stream.synchronize()
            if clk is not None:
                # A timed region of a few ms falls between two 200 ms clock samples, so the
                # sampler sees the same graph replayed back to back for LOAD_S seconds right
                # before it (the GPU stays loaded into the timed region).
                clk.wait_samples(1)
                t0 = time.perf_counter()
                while time.perf_counter() - t0 < LOAD_S:
                    for _ in range(64):
                        plan.replay()
                    stream.synchronize()
            if world > 1:
                dist.barrier()
            evs = []
            for _ in range(steps):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                plan.replay()
                b.record(stream)
                evs.append((a, b))
            stream.synchronize()
            ms = sum(a.elapsed_time(b) for a, b in evs)
        return max_over_ranks(ms, dev, world)

    with ClockSampler(local) as clk:
        ms_split = timed(plans["split"], args.steps, args.warmup, clk)
        ms_plain = timed(plans["plain"], args.steps, args.warmup, clk)
    clocks = clk.summary()
    clocks["window"] = f"200 ms samples over {LOAD_S} s of back-to-back replays before each timed region"


    # precision of this run's outputs vs the oracle (rank 0 computes the oracle once)
    ref = oracle_eval(args.workload, tens_o).data if rank == 0 else None
    out_split = plans["split"].output.to_host()
    out_plain = plans["plain"].output.to_host()
    err = {}
    if ref is not None:
        es, ep = rel_errors(out_split, ref), rel_errors(out_plain, ref)
        err = {"split": es["normwise"], "plain": ep["normwise"],
               "elementwise_above_1e-3_max": {"split": es["elementwise_above_1e-3_max"],
                                              "plain": ep["elementwise_above_1e-3_max"]},
               "definition": "normwise max|C - C_oracle| / max|C_oracle|; elementwise max |C - C_oracle| / "
                             "|C_oracle| over the entries above 1e-3 max|C_oracle|",
               "split_slices": split_slices(logs["split"])}

    # end to end through the public API: pinned host inputs -> device, graph, result -> host, every
    # step. Steps are pipelined the way a serving loop would run them: two captured instances of
    # the contraction alternate, the inputs of step i+1 go up and the result of step i-1 comes
    # back on their own streams (the copy engines) while step i computes.
    # the pinned staging buffers get their pages on the GPU's NUMA node (the allocating thread runs
    # there meanwhile), so the copy engines do not read them across the socket link
    numa_node, near = gpu_numa_cpus(local)
    saved_cpus = os.sched_getaffinity(0)
    if near:
        os.sched_setaffinity(0, near)
    try:
        host_in = {k: torch.from_numpy(np.ascontiguousarray(v.data)).pin_memory() for k, v in tens_o.items()}
        nout = plans["split"].output.data.numel()
        host_out = [torch.empty(nout, dtype=torch.float64).pin_memory() for _ in range(2)]
    finally:
        os.sched_setaffinity(0, saved_cpus)
    h2d = sum(v.numel() * v.element_size() for v in host_in.values())
    d2h = host_out[0].numel() * host_out[0].element_size()
    twin = tk.NetworkPlan(expr, precision="split", **{k: to_device(v, dev) for k, v in tens_o.items()})
    twin.capture()
    e2e_plans = [plans["split"], twin]
    s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_comp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def e2e_run(nsteps, start=None, end=None):
        if start is not None:
            start.record(s_in)
        for i in range(nsteps):
            b = i % 2
            P = e2e_plans[b]
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_comp[b])  # the compute that read these inputs is done
                for k, v in host_in.items():
                    P.inputs[k].data.copy_(v, non_blocking=True)
                ev_in[b].record(s_in)
            stream.wait_event(ev_in[b])
            if i >= 2:
                stream.wait_event(ev_out[b])  # the result of step i-2 has been read back
            with torch.cuda.stream(stream):
                P.replay()
            ev_comp[b].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_comp[b])
                host_out[b].copy_(P.output.data, non_blocking=True)
                ev_out[b].record(s_out)
        if end is not None:
            s_out.wait_stream(s_in)
            s_out.wait_stream(stream)
            end.record(s_out)

    e2e_run(args.warmup)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    e2e_run(args.steps, a, b)
    torch.cuda.synchronize(dev)
    ms_e2e = a.elapsed_time(b)
    ms_e2e = max_over_ranks(ms_e2e, dev, world)

    # serial end to end, one step at a time (no overlap between steps): inputs up, the captured
    # graph, the result back, then the next step. And the eager call a drop-in user makes without
    # capture: inputs up, tk.tensor(...) (host-side lookups of the cached tables and plans, one
    # launch per kernel), the result back.
    P0 = plans["split"]

    def serial_step():
        with torch.cuda.stream(stream):
            for k, v in host_in.items():
                P0.inputs[k].data.copy_(v, non_blocking=True)
            P0.replay()
            host_out[0].copy_(P0.output.data, non_blocking=True)

    def eager_step():
        with torch.cuda.stream(stream), tk.using_precision("split"):
            for k, v in host_in.items():
                P0.inputs[k].data.copy_(v, non_blocking=True)
            o = tk.tensor(expr, **P0.inputs)
            host_out[1].copy_(o.data, non_blocking=True)

    def host_timed(fn, n):
        for _ in range(3):
            fn()
        stream.synchronize()
        if world > 1:
            dist.barrier()
        ea = torch.cuda.Event(enable_timing=True)
        eb = torch.cuda.Event(enable_timing=True)
        ea.record(stream)
        for _ in range(n):
            fn()
            stream.synchronize()  # the result is on the host before the next step starts
        eb.record(stream)
        stream.synchronize()
        return max_over_ranks(ea.elapsed_time(eb), dev, world)

    ms_serial = host_timed(serial_step, args.steps)
    ms_eager = host_timed(eager_step, args.steps)

    # per-kernel breakdown of one split step; the dominant kernel gives the roofline entry
    roof, breakdown = kernel_roofline(args, logs["split"], ctx, flush) if rank == 0 else (None, None)

    # the plain path's dominant GEMM against cuBLAS DGEMM measured in this run
    plain_roof = None
    if rank == 0:
        dg = dgemm_tflops(dev)
        _, pbd = kernel_roofline(args, logs["plain"], ctx, flush)
        pg = max((r for r in pbd if r["kernel"] == "grouped_gemm_fp64"), key=lambda r: r["ms"])
        plain_roof = {"kernel": "grouped_gemm_fp64 (DMMA)", "bound": "tensor", "achieved": pg["gflops"] / 1e3,
                      "peak": dg, "unit": "TFLOP/s", "frac": pg["gflops"] / 1e3 / dg,
                      "peak_source": "cuBLAS DGEMM 4096^3 (torch.matmul float64) measured in this run",
                      "ms_per_launch": pg["ms"], "flops": pg["flops"]}
    extra = other_configs(dev, ctx, flush) if (rank == 0 and world == 1 and args.workload == "su2_large"
                                               and not args.no_extra) else None

    value = whole_job_value(flops, world, args.steps, ms_split)
    plain_value = whole_job_value(flops, world, args.steps, ms_plain)
    e2e_value = whole_job_value(flops, world, args.steps, ms_e2e)
    line = None
    if rank == 0:
        cpu = cpu_baseline(args, tens_o, flops) if world == 1 else None
        line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_split / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded PCG64 normals)",
                "config": {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"],
                           "expr": expr, "flops_per_step": flops, "l2": "flushed (256 MB write) between steps",
                           "parallelism": f"replicas x{world}", "graph": "CUDA graph per step"},
                "plain_fp64": {"value": plain_value, "unit": "GFLOP/s", "ms_per_step": ms_plain / args.steps,
                               "roofline": plain_roof},
                "split_over_plain": value / plain_value,
                "max_rel_err": err,
                "e2e": {"value": e2e_value, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e / args.steps,
                        "host_buffers_numa_node": numa_node,
                        "pipelined": "inputs of step i+1 up and result of step i-1 back on copy streams "
                                     "while step i computes (two captured instances)"},
                "e2e_serial": {"value": whole_job_value(flops, world, args.steps, ms_serial), "unit": "GFLOP/s",
                               "ms_per_step": ms_serial / args.steps,
                               "step": "inputs up, graph replay, result back, host waits; no overlap between steps"},
                "e2e_eager": {"value": whole_job_value(flops, world, args.steps, ms_eager), "unit": "GFLOP/s",
                              "ms_per_step": ms_eager / args.steps,
                              "step": "inputs up, tk.tensor(expr) without capture (eager launches), result back, "
                                      "host waits"},
                "gpu_launches": (plans["split"].kernels_per_replay) * args.steps,
                "roofline": roof, "breakdown": breakdown, "cpu_baseline": cpu, "clocks": clocks}
        if extra is not None:
            line["configs"] = extra
        print(json.dumps(line))
    for p in list(plans.values()) + [twin]:
        p.free()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def kernel_roofline(args, log, ctx, flush):
    """Re-time every launch of one step alone (CUDA events on the library stream, L2 flushed
    before each) and relate the dominant kernel's algorithmic work to the measured peak."""
    import torch
    from tensorkit_b200.indexmanipulations import relaunch

    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        src = "measured"
    except Exception:
        peaks, src = {}, "fallback"
    hbm = peaks.get("hbm_gbs", 6650.0)
    bf16 = peaks.get("bf16_tflops", 1590.0)
    stream = ctx.stream
    reps = max(args.steps, 10)
    rows = []
    sink = torch.zeros(1, dtype=torch.int64, device=flush.device)

    def timed(fn, clean=False):
        # mean device time of `fn` after a 256 MB write flush; clean: the flush buffer is then
        # read back, so L2 holds clean unrelated lines and no write-back of the flush lands in `fn`
        evs = []
        for _ in range(reps):
            flush.zero_()
            if clean:
                sink.copy_(flush.view(torch.int64).sum().view(1))
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            evs.append((a, b))
        stream.synchronize()
        return statistics.mean(x.elapsed_time(y) for x, y in evs)

    with torch.cuda.stream(stream):
        for e in log:
            for _ in range(3):
                relaunch(e)
            stream.synchronize()
            ms = timed(lambda: relaunch(e))
            if e[0] == "transform":
                t = e[1]
                el = e[2].data.element_size()
                nbytes = el * (t.elems_read + t.elems_written * (1 if e[5] == 0 else 2))
                row = {"kernel": "treetransform", "ms": ms, "bytes": nbytes,
                       "gbs": nbytes / (ms * 1e-3) / 1e9, "frac_hbm": nbytes / (ms * 1e-3) / 1e9 / hbm}
                if nbytes >= (64 << 20):
                    # the same launch after a clean flush, and a device-to-device copy of the same
                    # bytes (half read, half written) under both flushes: what HBM gives at this size
                    ms_c = timed(lambda: relaunch(e), clean=True)
                    half = nbytes // 2
                    csrc = torch.empty(half, dtype=torch.uint8, device=flush.device)
                    cdst = torch.empty_like(csrc)
                    cp = timed(lambda: cdst.copy_(csrc))
                    cp_c = timed(lambda: cdst.copy_(csrc), clean=True)
                    del csrc, cdst
                    row.update({"ms_clean_l2": ms_c, "frac_hbm_clean_l2": nbytes / (ms_c * 1e-3) / 1e9 / hbm,
                                "memcpy_ms": cp, "memcpy_ms_clean_l2": cp_c,
                                "of_memcpy": cp / ms, "of_memcpy_clean_l2": cp_c / ms_c})
                rows.append(row)
            else:
                plan = e[1]
                S = plan.slices
                row = {"kernel": "grouped_gemm_split" if S else "grouped_gemm_fp64", "ms": ms,
                       "flops": plan.flops, "gflops": plan.flops / (ms * 1e-3) / 1e9, "slices": S}
                if S:
                    # int8 work of the launch: S_b(S_b + 1)/2 products of 2mnk per block at the
                    # slice count each block used (blocks in FP64 count their FP64 flops apart)
                    sl, fb = plan.last_slices()
                    mul = 4 if plan.is_complex else 1
                    ops8 = sum(2.0 * m * n * k * mul * sb * (sb + 1) / 2
                               for (m, n, k), sb in zip(plan.blocks[:, :3].tolist(), sl) if sb > 0)
                    row.update({"int8_ops": ops8, "block_slices": sorted(set(x for x in sl if x >= 0)),
                                "fp64_checked_tiles": fb})
                rows.append(row)
    dom = max(rows, key=lambda r: r["ms"])
    total = sum(r["ms"] for r in rows)
    for r in rows:
        r["share"] = r["ms"] / total
    if dom["kernel"] == "treetransform":
        roof = {"kernel": "treetransform", "bound": "hbm", "achieved": dom["gbs"], "peak": hbm,
                "unit": "GB/s", "frac": dom["gbs"] / hbm, "traffic": None,
                "peak_source": f"hbm_gbs of {src} peaks"}
    else:
        S = dom.get("slices") or 0
        if S:
            ops = dom["int8_ops"]
            ach = ops / (dom["ms"] * 1e-3) / 1e12
            peak = 2.0 * bf16
            roof = {"kernel": "grouped split GEMM call: gemm_split_slice_kernel (slicing) + "
                              "gemm_split_fused_kernel (int8 tensor-core products, FP64 recombination)",
                    "bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                    "frac": ach / peak,
                    "traffic": profile_traffic("gemm_split_fused_su2_large", "traffic_bytes_per_call"),
                    "peak_source": f"2 x bf16_tflops of {src} peaks (int8 dense = 2 x bf16 dense)",
                    "algorithmic": f"sum over blocks of S_b(S_b+1)/2 int8 products of 2mnk = {ops:.4e} "
                                   f"(slice counts {dom['block_slices']})",
                    "fp64_equiv_gflops": dom["gflops"], "ms_per_launch": dom["ms"]}
        else:
            roof = {"kernel": "grouped_gemm_fp64", "bound": "tensor", "achieved": dom["gflops"] / 1e3,
                    "peak": None, "unit": "TFLOP/s", "frac": None, "traffic": None}
    return roof, rows


def profile_traffic(name, key="traffic_bytes_per_launch"):
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of a kernel launch, or of the
    launches of one library call, from the committed ncu summary profiles/<name>.md (a line
    `<key>: N`), else None."""
    try:
        for ln in open(os.path.join(ROOT, "profiles", name + ".md")):
            if ln.strip().startswith(key + ":"):
                return float(ln.split(":", 1)[1].split()[0])
    except (OSError, ValueError, IndexError):
        pass
    return None


def cpu_baseline(args, tens_o, flops):
    """Oracle contraction on the host (numpy/BLAS, every host thread), bounded sample."""
    t0 = time.perf_counter()
    n = 0
    while True:
        oracle_eval(args.workload, tens_o)
        n += 1
        if time.perf_counter() - t0 > 10.0 or n >= 20:
            break
    dt = time.perf_counter() - t0
    cores = os.cpu_count()
    return {"value": flops * n / dt / 1e9, "unit": "GFLOP/s", "cores": cores, "kind": "port",
            "sample": f"{n} full contractions of the same workload (oracle restatement, numpy/BLAS)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="su2_large", choices=sorted(WORKLOADS))
    ap.add_argument("--kernel-only", default=None, choices=["transform", "gemm"],
                    help="profiling aid: one eager step, then relaunch the largest kernel of this kind")
    ap.add_argument("--factor", default=None, choices=["svd_trunc", "qr_compact", "eigh_full"],
                    help="time one block factorization of the workload's first input instead")
    ap.add_argument("--precision", default="split", choices=["split", "plain"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other configurations (ComplexF64, U(1) effective Hamiltonian, AD step)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.kernel_only:
        return run_kernel_only(args)
    if args.factor:
        return run_factor(args)
    return run_ours(args)


def run_kernel_only(args):
    """One eager step (every table and plan built, all launches recorded), then the largest
    launch of the requested kind relaunched `--reps` times. Prints how many launches of that
    kernel preceded the relaunches, for `ncu -k ... -s <skip>`."""
    import torch
    import tensorkit_b200 as tk
    from helpers import to_device
    from tensorkit_b200 import indexmanipulations as IM

    dev = torch.device("cuda", 0)
    inputs = {k: to_device(v, dev) for k, v in oracle_inputs(args.workload).items()}
    ctx = tk.get_context(0)
    p = tk.NetworkPlan(WORKLOADS[args.workload]["expr"], precision=args.precision, **inputs)
    IM.LAUNCH_LOG = []
    p.run_eager()
    log, IM.LAUNCH_LOG = IM.LAUNCH_LOG, None
    kind = args.kernel_only
    cands = [e for e in log if e[0] == kind]
    if kind == "transform":
        big = max(cands, key=lambda e: e[1].elems_read + e[1].elems_written)
        size = {"elems_read": big[1].elems_read, "elems_written": big[1].elems_written,
                "ntasks": big[1].ntasks}
    else:
        big = max(cands, key=lambda e: e[1].flops)
        size = {"flops": big[1].flops, "slices": big[1].slices}
    with torch.cuda.stream(ctx.stream):
        for _ in range(args.reps):
            IM.relaunch(big)
    ctx.stream.synchronize()
    print(json.dumps({"kernel_only": kind, "workload": args.workload, "preceding_launches": len(cands),
                      "reps": args.reps, **size}))
    return 0


def run_factor(args):
    """One block factorization of the workload's first input tensor (eigh: of t†t), device time
    with CUDA events over --steps calls, beside numpy/LAPACK on the same blocks on the host."""
    import numpy as np
    import torch
    import tensorkit_b200 as tk
    from helpers import from_sector, to_device
    from oracle import factor as F

    dev = torch.device("cuda", 0)
    ot = next(iter(oracle_inputs(args.workload).values()))
    t = to_device(ot, dev)
    if args.factor == "eigh_full":
        t = tk.compose(t.adjoint(), t)
        oblocks = {from_sector(c): t.block(c).cpu().numpy() for c in t.blocksectors()}
    else:
        oblocks = {from_sector(c): ot.block(from_sector(c)) for c in t.blocksectors()}
    fn = {"svd_trunc": lambda: tk.svd_trunc(t, tk.truncrank(t.space.domain.dim() // 2)),
          "qr_compact": lambda: tk.qr_compact(t), "eigh_full": lambda: tk.eigh_full(t)}[args.factor]
    npfn = {"svd_trunc": lambda b: np.linalg.svd(b, full_matrices=False),
            "qr_compact": lambda b: np.linalg.qr(b), "eigh_full": lambda b: np.linalg.eigh(b)}[args.factor]
    for _ in range(args.warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        fn()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    t0 = time.perf_counter()
    for blk in oblocks.values():
        npfn(blk)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    shapes = sorted({tuple(v.shape) for v in oblocks.values()})
    print(json.dumps({"factor": args.factor, "workload": args.workload, "blocks": len(oblocks),
                      "block_shapes": shapes[-3:], "ms_per_call": ms, "cpu_numpy_ms": cpu_ms,
                      "steps": args.steps, "note": "per-block vendor solver (torch.linalg / cuSOLVER), "
                                                   "batched over equal block shapes"}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
