#!/usr/bin/env python
"""Benchmark of the B200 dual-scaling IPM: time to a 1e-6 relative gap.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload rank1_n1000_m2000] [--precision fp64|split]

One step is one complete solve of the workload through the hdsdp.h C API
(create, set cone data, set the dual objective, optimize, read the dual)
with the five-step primal refinement off, so the solve stops at the
reference's own relative-gap test (1e-6). Printed as one JSON line:

  value  seconds per solve for the iterations alone (data resident on the
         device; CUDA events on the solver stream, inside the library)
  e2e    seconds per solve through the public API from pinned host buffers,
         host->device upload and device->host read of y included (CUDA
         events around each call)
  roofline  the kernel family with the largest device time in the timed
         region: algorithmic flops (or bytes) per launch over its CUDA-event
         duration, against MEASURED_PEAKS.json
  cpu_baseline  the reference CPU solver (oracle/_ref, all host threads) on a
         bounded sample of the same solve: the first few iterations, scaled
         to the reference's full iteration count
  precision_legs  the same workload in split precision (mode 2) beside the
         FP64 solve, with the split solve's error against the FP64 one per
         iteration and for every final result
  maxcut_n8000  MaxCut n=8000 (40,000 edges) solved in FP64 and in split
         precision: device time, time to a 1e-6 gap, iterations, status

--impl reference times complete reference CPU solves (rank 0, all host
threads) on the same workload and prints the same metric with "impl":
"reference"; a time budget bounds how many solves are timed. Multi-GPU runs
are independent replicas, one solve per GPU per step ("scaling": "weak"),
timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to 1e-6 rel gap (dual-scaling IPM solve)"
UNIT = "s"
FLUSH_BYTES = 256 << 20  # larger than the 126 MB L2
# kernel-timing families of the library (hdsdpb_kstat_*), in its numbering
FAMILIES = ["fp64_gemm_dmma", "potrf_coop_slack", "trtri_coop", "schur_pair_gather", "bf16x3_gemm_tcgen05",
            "potrf_coop_schur"]
FAMILY_BOUND = ["tensor", "tensor", "tensor", "hbm", "tensor", "tensor"]
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per launch of a kernel
# family on a workload, with the ncu summary they were read from.
TRAFFIC_PER_LAUNCH = {
    ("rank1_n1000_m2000", "potrf_coop_slack"): (4.53e6, "profiles/potrf_coop_n1000.md (one launch, n = 1000)"),
}
REF_SAMPLE_ITERS = 5
# a complete reference solve of the bench workload takes tens of seconds: time as many
# as fit this budget (at least one)
REF_BUDGET_S = 300.0
L2_NOTE = "flushed between steps (256 MB write)"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="rank1_n1000_m2000")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split", "adaptive"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision-legs", action="store_true", help="skip the other-precision solves")
    ap.add_argument("--no-maxcut-leg", action="store_true", help="skip the MaxCut n=8000 leg")
    ap.add_argument("--no-arrow-leg", action="store_true", help="skip the block-arrow multi-cone leg")
    ap.add_argument("--ref-budget", type=float, default=REF_BUDGET_S,
                    help="seconds of complete reference solves to time (--impl reference)")
    return ap.parse_args()


def bench_config(args, inst, world):
    """The workload configuration; both arms print the same keys and values."""
    return {"workload": args.workload, "n": inst.n, "m": inst.m, "primal_refinement": False,
            "precision": args.precision, "parallelism": "replicas" if world > 1 else "single", "l2": L2_NOTE}


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return {"hbm_gbs": p["hbm_gbs"], "bf16_tflops": p["bf16_tflops"],
                "bf16_tflops_sustained": p["bf16_tflops_sustained"], "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi samples of this GPU's clocks and throttle reasons during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus_id = bus_id
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), "hdsdp_b200_clocks_%d.csv" % os.getpid())

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        cmd = ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", "200"]
        if self.bus_id:
            cmd += ["-i", self.bus_id]
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(cmd, stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for name, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(name)
        os.remove(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x: float, world: int, device: str) -> float:
    """Max of a per-rank time over all ranks (every rank takes this collective)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# reference CPU solver (oracle/_ref): the cpu_baseline leg and --impl reference

def reference_iters(workload: str):
    """The reference's full iteration count for the workload (committed golden fixture)."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
            g = json.load(f)
        return g["solves"]["%s/psdp0" % workload]["iters"]
    except (OSError, KeyError, ValueError):
        return None


def _reference_child(workload, caps, threads, out):
    """Child process: the reference solver on the workload, capped at each iteration count."""
    from hdsdp_b200 import instances
    from oracle import ref_api
    ref_api.set_threads(threads)
    inst = instances.WORKLOADS[workload]()
    res = []
    for cap in caps:
        params = {4: 0} if cap is None else {0: cap, 4: 0}
        r = ref_api.solve(inst, want_x=False, params=params)
        res.append((r["time"], r["iters"], r["status_after_check"], r["dobj"]))
    out.put(res)


def reference_runs(workload: str, caps, threads: int, timeout: float):
    """(time, iterations) of reference solves capped at `caps`, run in a spawned child.

    The child isolates the bench from the reference: its HDSDPOptimize smashes its own stack
    when capped at one iteration on the MaxCut instances, and large workloads can exceed the
    time allowed for a bounded sample. Returns (None, reason) on failure.
    """
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_reference_child, args=(workload, list(caps), threads, q))
    p.start()
    p.join(timeout)
    if p.is_alive():
        p.kill()
        p.join()
        return None, "reference sample exceeded %.0f s" % timeout
    if p.exitcode != 0:
        return None, "reference process exited with code %s" % p.exitcode
    return q.get(), ""


def reference_sample(workload: str, iters: int, threads: int, fallback_iters=None, timeout: float = 240.0):
    """Seconds to a 1e-6 gap for the reference CPU solver, estimated from two bounded runs.

    A run capped at two iterations gives the set-up cost plus two iterations; a run capped
    at 2 + `iters` adds `iters` iterations. The estimate is the first plus the marginal
    per-iteration cost times the reference's remaining iterations. Returns None and a
    reason when the sample fails.
    """
    res, why = reference_runs(workload, (2, 2 + iters), threads, timeout)
    if res is None:
        return None, why
    (t1, i1, _, _), (tk, ik, _, _) = res
    done = max(1, ik - i1)
    per_iter = max(0.0, tk - t1) / done
    full = reference_iters(workload) or fallback_iters or ik
    return (t1 + per_iter * max(0, full - i1), t1 + tk, done, full), ""


def run_reference(args):
    """Complete reference solves of the workload on all host cores (rank 0 alone)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import numpy as np
    from hdsdp_b200 import instances
    from oracle import ref_api
    base = {"metric": METRIC, "unit": UNIT, "impl": "reference", "higher_is_better": False}
    if not ref_api.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (make -C oracle)"}))
        return
    inst = instances.WORKLOADS[args.workload]()
    cores = host_cores()
    for _ in range(args.warmup):  # untimed: a short capped solve in the same kind of child process
        reference_runs(args.workload, (2,), cores, 240.0)
    flush = np.empty(FLUSH_BYTES // 8)
    vals, iters, status, dobj = [], None, None, None
    t0 = time.perf_counter()
    for k in range(args.steps):
        flush.fill(float(k))  # evict the previous solve's data from the host caches
        got, why = reference_runs(args.workload, (None,), cores, max(600.0, 3.0 * args.ref_budget))
        if got is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        t, iters, status, dobj = got[0]
        vals.append(t)
        elapsed = time.perf_counter() - t0
        if elapsed + statistics.mean(vals) > args.ref_budget:
            break
    wall = time.perf_counter() - t0
    value = statistics.mean(vals)
    capped, _ = reference_sample(args.workload, REF_SAMPLE_ITERS, cores)
    sample = ("%d complete %s solves (HDSDPOptimize, primal refinement off, %d iterations, status %s), "
              "%.1f s of CPU work; at most %.0f s of solves are timed" % (len(vals), args.workload, iters, status,
                                                                          sum(vals), args.ref_budget))
    line = dict(base, value=value, n_gpus=args.gpus, steps=len(vals), steps_requested=args.steps,
                warmup=args.warmup, ms_per_step=1e3 * wall / len(vals), scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic (seeded generator, hdsdp_b200/instances.py)",
                config=bench_config(args, inst, world),
                cpu_baseline={"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                              "sample": sample},
                e2e={"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                iters=iters, status=status, dobj=dobj, s_per_iter=value / max(1, iters),
                steps_s=[round(v, 3) for v in vals],
                extrapolated_from_capped=(None if capped is None else
                                          {"value": capped[0], "capped_at": [2, 2 + REF_SAMPLE_ITERS]}))
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# B200 arm

def adjoint_leg(L, api, instances, np):
    """Adjoint ms on the theta-style layer (n = 200) against the mean IPM iteration of its solve."""
    import ctypes as C
    import torch
    inst = instances.WORKLOADS["theta_adjoint_n200"]()
    rng = np.random.default_rng(5)
    G = rng.standard_normal((inst.n, inst.n))
    G = np.asfortranarray(G + G.T)
    h = rng.standard_normal(inst.m)
    out = {}
    for rep in range(2):  # the first solve warms the path; the second is measured
        s = api.Solver()
        try:
            s.init(inst.m, 1)
            s.set_cone(inst.m, inst.n, inst.Ap, inst.Ai, inst.Ax)
            s.set_dual_objective(inst.b)
            s.set_primal_refinement(False)
            s.optimize(0)
            t = s.timers()
            iters = max(1, s.iters())
            times = []
            for _ in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                s.adjoint(h, G)
                e1.record()
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
            out = {"workload": "theta_adjoint_n200", "n": inst.n, "m": inst.m, "status": s.status(),
                   "first_call_ms": times[0], "cached_call_ms": min(times[1:]),
                   "ipm_iter_ms": 1e3 * t["ipm_device"] / iters, "iters": iters,
                   "first_call_over_iter": times[0] / (1e3 * t["ipm_device"] / iters)}
        finally:
            s.close()
    return out


def precision_leg(api, inst, mode, solves, np):
    """Mean device-timed solve, time to a 1e-6 gap and the last solve's results
    (objectives, y, per-iteration log) with HDSDPSetPrecision(mode)."""
    ipm, ttg, last = [], [], None
    for _ in range(solves):
        s = api.Solver()
        try:
            s.init(inst.m, 1)
            s.set_cone(inst.m, inst.n, inst.Ap, inst.Ai, inst.Ax)
            s.set_dual_objective(inst.b)
            s.set_primal_refinement(False)
            s.set_precision(mode)
            s.optimize(0)
            t = s.timers()
            log = s.iter_log()
            hit = np.flatnonzero(np.asarray(log["gap"]) <= 1e-6)
            ttg.append(float(log["t"][hit[0]] - t["setup"]) if hit.size else None)
            ipm.append(t["ipm_device"])
            po, do, y = s.get_row_dual()
            last = {"iters": s.iters(), "status": s.status(), "pobj": po, "dobj": do, "y": y, "log": log}
        finally:
            s.close()
    out = {"value": float(np.mean(ipm)), "unit": UNIT, "iters": last["iters"], "status": last["status"],
           "time_to_gap_s": ttg[-1], "solves": solves}
    return out, last


def split_error(split, fp64, np):
    """The split-precision solve's error against the FP64 solve: final objectives and y
    (relative), and per iteration the relative differences of the dual objective and of
    the relative gap."""
    def rel(a, b):
        return abs(a - b) / (1.0 + abs(b))
    k = min(len(split["log"]["dobj"]), len(fp64["log"]["dobj"]))
    dd = [rel(a, b) for a, b in zip(split["log"]["dobj"][:k], fp64["log"]["dobj"][:k])]
    dg = [abs(a - b) for a, b in zip(split["log"]["gap"][:k], fp64["log"]["gap"][:k])]
    return {"pobj_rel": rel(split["pobj"], fp64["pobj"]), "dobj_rel": rel(split["dobj"], fp64["dobj"]),
            "y_rel": float(np.linalg.norm(split["y"] - fp64["y"]) / max(np.linalg.norm(fp64["y"]), 1e-300)),
            "iters": [split["iters"], fp64["iters"]],
            "per_iter_dobj_rel": [float("%.3g" % v) for v in dd],
            "per_iter_gap_absdiff": [float("%.3g" % v) for v in dg]}


def maxcut_leg(api, instances, np):
    """MaxCut n=8000 (40,000 edges): FP64 (sparse dual-slack factorisation on trial
    points) and split precision mode 2; one untimed solve, then two timed ones each."""
    inst = instances.WORKLOADS["maxcut_n8000"]()
    out = {"workload": "maxcut_n8000", "n": inst.n, "m": inst.m}
    res = {}
    for name, mode in (("fp64", 0), ("split_adaptive", 2)):
        precision_leg(api, inst, mode, 1, np)
        out[name], res[name] = precision_leg(api, inst, mode, 2, np)
    out["fp64_over_split"] = out["fp64"]["value"] / out["split_adaptive"]["value"]
    e = split_error(res["split_adaptive"], res["fp64"], np)
    out["split_error"] = {k: e[k] for k in ("pobj_rel", "dobj_rel", "y_rel", "iters")}
    return out


def arrow_leg(api, instances, np):
    """The block-arrow Schur complement on problems made of sparse SDP cones: 60 cones of
    order 90 (m = 27,100) and 250 cones (m = 112,600, whose dense Schur matrix and factor would
    take 203 GB); one untimed solve, then two device-timed ones each."""
    out = {}
    for name in ("mb60_m27k", "mb250_m112k"):
        prob = instances.multiblock_case(name)
        api.solve_problem(prob)
        rs = [api.solve_problem(prob) for _ in range(2)]
        r = rs[-1]
        info = r["sparse_schur"]
        out[name] = {"m": prob.m, "cones": len(prob.cones), "unit": UNIT,
                     "value": float(np.mean([x["timers"]["ipm_device"] for x in rs])),
                     "iters": r["iters"], "status": r["status_after_check"], "pobj": r["pobj"], "dobj": r["dobj"],
                     "dimacs_max": float(np.max(np.abs(r["errs"]))), "arrow": info["arrow"],
                     "arrow_bytes": info["arrow_bytes"], "dense_bytes": info["dense_bytes"]}
    return out


def run_b200(args):
    rank, world, local_rank = dist_env()
    if world > 1 and "CUDA_VISIBLE_DEVICES" not in os.environ:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local_rank)
    import ctypes as C

    import numpy as np
    import torch
    import torch.distributed as dist

    from hdsdp_b200 import _lib, api, instances

    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device (the B200 arm has no CPU path)")
    torch.cuda.set_device(0)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", 0))

    def barrier():
        if world > 1:
            dist.barrier()

    L = _lib.load()
    inst = instances.WORKLOADS[args.workload]()
    precision = {"fp64": 0, "split": 1, "adaptive": 2}[args.precision]

    # pinned host copies of the step's inputs
    def pinned(a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        t = torch.empty(a.shape, dtype={np.int32: torch.int32, np.float64: torch.float64}[dtype], pin_memory=True)
        out = t.numpy()
        out[...] = a
        return out, t

    Ap, _tAp = pinned(inst.Ap, np.int32)
    Ai, _tAi = pinned(inst.Ai, np.int32)
    Ax, _tAx = pinned(inst.Ax, np.float64)
    bvec, _tb = pinned(inst.b, np.float64)
    yout, _ty = pinned(np.zeros(inst.m), np.float64)
    h2d = Ap.nbytes + Ai.nbytes + Ax.nbytes + bvec.nbytes
    d2h = yout.nbytes + 2 * 8

    def one_solve():
        s = api.Solver()
        try:
            s.init(inst.m, 1)
            if s.set_cone(inst.m, inst.n, Ap, Ai, Ax) != 0:
                raise RuntimeError("HDSDPSetCone rejected the block")
            s.set_dual_objective(bvec)
            s.set_primal_refinement(False)
            s.set_precision(precision)
            ret = s.optimize(0)
            po, do = C.c_double(), C.c_double()
            L.HDSDPGetRowDual(s.h, C.byref(po), C.byref(do), yout.ctypes.data_as(C.POINTER(C.c_double)))
            return {"ret": ret, "status": s.status(), "iters": s.iters(), "timers": s.timers(),
                    "log": s.iter_log(), "pobj": po.value, "dobj": do.value}
        finally:
            s.close()

    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(3, args.warmup)):
        one_solve()

    bus = None
    try:
        p = torch.cuda.get_device_properties(0)
        bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
    except Exception:
        bus = None
    clocks = ClockSampler(bus)
    L.hdsdpb_kstat_enable((1 << len(FAMILIES)) - 1)
    launches0 = L.hdsdpb_launch_count()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    results = []
    w0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()  # evict the previous solve's working set from L2
        torch.cuda.synchronize()
        ev[k][0].record()
        results.append(one_solve())
        ev[k][1].record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    barrier()
    clk = clocks.stop()
    launches = L.hdsdpb_launch_count() - launches0
    fam = []
    for f in range(len(FAMILIES)):
        n_l, ms, work = C.c_longlong(), C.c_double(), C.c_double()
        L.hdsdpb_kstat_read(f, C.byref(n_l), C.byref(ms), C.byref(work))
        fam.append((n_l.value, ms.value, work.value))
    L.hdsdpb_kstat_enable(0)

    e2e_s = [ev[k][0].elapsed_time(ev[k][1]) * 1e-3 for k in range(args.steps)]
    ipm_s = [r["timers"]["ipm_device"] for r in results]
    iters = results[-1]["iters"]
    value = max_over_ranks(statistics.mean(ipm_s), world, "cuda")
    e2e = max_over_ranks(statistics.mean(e2e_s), world, "cuda")
    last = results[-1]
    gap = np.asarray(last["log"]["gap"])
    tlog = np.asarray(last["log"]["t"])
    hit = np.flatnonzero(gap <= 1e-6)
    time_to_gap = float(tlog[hit[0]] - last["timers"]["setup"]) if hit.size else None

    pk = peaks()
    top = max(range(len(FAMILIES)), key=lambda f: fam[f][1])
    n_l, ms, work = fam[top]
    if FAMILY_BOUND[top] == "tensor":
        achieved = work / (ms * 1e-3) / 1e12 if ms > 0 else 0.0
        peak, unit = pk["bf16_tflops_sustained"], "TFLOP/s"
    else:
        achieved = work / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        peak, unit = pk["hbm_gbs"], "GB/s"
    roofline = {"bound": FAMILY_BOUND[top], "kernel": FAMILIES[top], "achieved": achieved, "peak": peak,
                "unit": unit, "frac": achieved / peak, "peak_source": pk["source"],
                "traffic": TRAFFIC_PER_LAUNCH.get((args.workload, FAMILIES[top]), (None, None))[0],
                "traffic_source": TRAFFIC_PER_LAUNCH.get((args.workload, FAMILIES[top]), (None, None))[1],
                "launches": n_l, "ms_total": ms, "share_of_ipm": ms * 1e-3 / sum(ipm_s)}
    if FAMILIES[top] == "bf16x3_gemm_tcgen05":
        roofline["note"] = "achieved counts the three BF16 products of each split product"
    elif FAMILY_BOUND[top] == "tensor":
        roofline["note"] = ("FP64 DMMA (mma.sync m8n8k4 f64): tcgen05 has no f64 kind; peak is the measured "
                            "sustained bf16 figure, nominal FP64 tensor peak is about 40 TFLOP/s")
    kernels = {FAMILIES[f]: {"launches": fam[f][0], "ms": fam[f][1],
                             ("tflops" if FAMILY_BOUND[f] == "tensor" else "gbs"):
                                 (fam[f][2] / (fam[f][1] * 1e-3) / (1e12 if FAMILY_BOUND[f] == "tensor" else 1e9)
                                  if fam[f][1] > 0 else None)}
               for f in range(len(FAMILIES))}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref_api
            if ref_api.available():
                cores = host_cores()
                got, why = reference_sample(args.workload, REF_SAMPLE_ITERS, cores, fallback_iters=iters)
                if got is None:
                    raise RuntimeError(why)
                est, t, done, full = got
                cpu = {"value": est, "unit": UNIT, "cores": cores, "kind": "reference",
                       "sample": "reference CPU solves capped at 2 and %d IPM iterations (%.2f s of CPU work); "
                                 "set-up + marginal s/iter scaled to its %d iterations" % (2 + done, t, full)}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "failed: %s" % exc}

    t = last["timers"]
    adj = adjoint_leg(L, api, instances, np) if rank == 0 else None
    legs = None
    if rank == 0 and not args.no_precision_legs:
        # the same workload in FP64 and in split precision mode 2 (two solves each after
        # the warm-up above), with the split solve's error against the FP64 solve
        fp64_leg, fp64_last = precision_leg(api, inst, 0, 2, np)
        split_leg, split_last = precision_leg(api, inst, 2, 2, np)
        legs = {"fp64": fp64_leg, "split_adaptive": split_leg,
                "fp64_over_split": fp64_leg["value"] / split_leg["value"],
                "split_error_vs_fp64": split_error(split_last, fp64_last, np)}
    mc = None
    if rank == 0 and not args.no_maxcut_leg:
        mc = maxcut_leg(api, instances, np)
    arrow = None
    if rank == 0 and not args.no_arrow_leg:
        arrow = arrow_leg(api, instances, np)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": 1e3 * value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == 0 else "bf16x3+f64",
        "data": "synthetic (seeded generator, hdsdp_b200/instances.py)",
        "config": bench_config(args, inst, world),
        "iters": iters, "s_per_iter": value / max(1, iters), "time_to_gap_s": time_to_gap,
        "steps_ipm_s": [round(x, 4) for x in ipm_s], "steps_e2e_s": [round(x, 4) for x in e2e_s],
        "setup_s": [round(r["timers"]["setup"], 4) for r in results],
        "status": last["status"], "dobj": last["dobj"], "pobj": last["pobj"],
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "bytes_note": "h2d counts the CSC arrays and b handed to the C API from pinned memory; "
                              "the library reads them on the host and uploads the presolved coefficients"},
        "roofline": roofline, "kernels": kernels, "cpu_baseline": cpu, "clocks": clk,
        "gpu_launches": launches, "wall_s": wall, "adjoint": adj, "precision_legs": legs, "maxcut_n8000": mc,
        "block_arrow": arrow,
        "split_s": {k: t[k] for k in ("schur", "schur_factor", "schur_solve", "s_factor", "s_inverse",
                                      "lanczos", "assemble", "primal", "setup", "total")},
    }
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
