#!/usr/bin/env python
"""Benchmark of single-list Redzone removal on B200.

Workload (the large-list configuration the headline target is quoted on): n = 2^28 int32 items
(iota), k = 2^16 distinct removal indices drawn uniformly without replacement, unsorted. A step
is one Redzone removal of k items from the device-resident list. L2 is flushed between timed
steps (a 256 MiB scrub write, one before the first step too), and the removal lists rotate over
8 seeds.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl own|reference] [--sweep]

Own arm: CUDA-event time of each rz_remove kernel on the launching stream; value = k / mean
step time (whole job: summed over ranks; N > 1 runs independent replicas, max over ranks).
Also reported on the same line:
  * the event floor (an empty kernel of the removal's launch shape, timed the same way);
  * the roofline of the Redzone kernel against measured HBM bandwidth;
  * the O(n) partition comparator and the reference's own mark + thrust::remove comparator on the
    same workload, a CUDA-graph steady state of the removal, and the removal timed L2-warm (no
    scrub between steps);
  * end to end (e2e): the pipelined host-index call (rz_remove_host_idx_async / rz_wait) from C++
    (redzone_b200/_lib/rz_e2e) and from Python, each step copying its removal list from pinned
    host memory and reading its status and new length back;
  * the batched half of the metric: 4096 uneven lists in one launch with the configuration the
    learned list-mix predictor picks, against per-list launches, the default configuration, an
    exhaustive autotune of the configuration space, and the hole writes alone;
  * the reference's CPU paths on the host cores (redzone_CPU, and std::remove(par_unseq));
  * SM clocks sampled from before the timed region to the end of the e2e leg.

Other workloads: --workload batched (the batched leg alone), --workload service (streaming
deletes), --workload produced (a list made on the GPU with fused red-zone marking), --sweep (k).

Reference arm (--impl reference): the reference's redzone_CPU (compiled from its sources into
oracle/_ref) on the same workload on the host cores, rank 0 only, with std::remove(par_unseq)
beside it; it loads no library of this package.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_LOG2, K_LOG2, W_BYTES = 28, 16, 4
NSETS = 8
SCRUB_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0

# Device -> host per pipelined call: the call's status word and device-tracked length, read back
# as one 16-byte copy.
RESULT_BYTES = 16
METRIC = "items removed/s"
UNIT = "items/s"


def config(world: int) -> dict:
    """The workload of both arms (the reference arm prints the same object)."""
    return {
        "workload": f"single-list Redzone removal, n=2^{N_LOG2} int32 payload (iota), k=2^{K_LOG2} distinct "
                    f"uniform unsorted indices",
        "n": 1 << N_LOG2, "k": 1 << K_LOG2, "elem_bytes": W_BYTES, "distribution": "uniform",
        "l2": "flushed between timed steps (256 MiB scrub write)", "index_sets": NSETS,
        "parallelism": "single GPU" if world == 1 else f"{world} independent replicas (one list per GPU)",
    }


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def load_traffic(key: str):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(key)
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
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
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def alg_bytes(n: int, k: int, w: int, idx: np.ndarray) -> float:
    """Algorithmic bytes of one Redzone call: read R, read surviving tail items, write the holes,
    write + read the k-bit red-zone bitmap: 4k + 2w(k - k_r) + k/4, k_r = #{R >= n-k}."""
    k_r = int((idx >= n - k).sum())
    return 4.0 * k + 2.0 * w * (k - k_r) + k / 4.0


# ------------------------------------------------------------------------------------------------
def load_workloads():
    """``redzone_b200/workloads.py`` (plain numpy) loaded by its path. Importing it through the
    package would also load the package's CUDA library, which the CPU legs must not touch."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("_rz_bench_workloads", ROOT / "redzone_b200" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cpu_reference_time(n: int, k: int, steps: int, warmup: int, time_budget_s: float):
    """Time the reference's redzone_CPU (oracle/_ref) -- or the oracle port if it is absent."""
    import oracle

    workloads = load_workloads()
    a = np.arange(n, dtype=np.int32)
    sets = [workloads.uniform(n, k, seed=s).astype(np.int32) for s in range(NSETS)]
    L = oracle.ref_lib()
    if L is not None:
        kind, cores = "reference", int(L.ref_redzone_threads())

        def run(i):
            r = sets[i % NSETS].copy()  # redzone_CPU clobbers its removal list
            t0 = time.perf_counter()
            L.ref_redzone_cpu(a.ctypes.data, n, r.ctypes.data, k)
            return time.perf_counter() - t0
    else:
        kind, cores = "port", 1

        def run(i):
            r = sets[i % NSETS].astype(np.uint32)
            t0 = time.perf_counter()
            oracle.remove(a, r)
            return time.perf_counter() - t0
    for i in range(warmup):
        run(i)
    times = []
    t_start = time.perf_counter()
    for i in range(steps):
        times.append(run(i))
        if time.perf_counter() - t_start > time_budget_s and len(times) >= 3:
            break
    return kind, cores, times


def cpu_par_remove_time(n: int, k: int, max_calls: int, time_budget_s: float):
    """Time the reference's O(n) CPU comparator -- mark with -1, then std::remove(par_unseq)
    (std_parallel_remove.hxx:13-36, compiled into oracle/_ref) -- on the same workload. The list
    is restored to iota before each call (outside the timer). None when oracle/_ref is absent."""
    import oracle

    L = oracle.ref_lib()
    if L is None:
        return None
    workloads = load_workloads()
    iota = np.arange(n, dtype=np.int32)
    a = iota.copy()
    sets = [workloads.uniform(n, k, seed=s).astype(np.int32) for s in range(NSETS)]
    times = []
    t_start = time.perf_counter()
    for i in range(max_calls + 1):  # the first call is a warm-up
        np.copyto(a, iota)
        r = sets[i % NSETS]
        t0 = time.perf_counter()
        L.ref_par_remove(a.ctypes.data, n, r.ctypes.data, k)
        dt = time.perf_counter() - t0
        if i > 0:
            times.append(dt)
        if time.perf_counter() - t_start > time_budget_s and len(times) >= 1:
            break
    parallel = int(L.ref_pstl_parallel())
    mean = statistics.mean(times)
    return {"value": k / mean, "unit": UNIT, "ms_per_call": mean * 1e3, "calls": len(times),
            "cores": 1 if not parallel else int(L.ref_redzone_threads()) + 1,
            "pstl_parallel_backend": bool(parallel),
            "note": "libstdc++ runs std::remove(par_unseq) serially without oneTBB, which this host lacks"
                    if not parallel else "libstdc++ parallel backend present"}


def cpu_baselines(n: int, k: int, steps: int, warmup: int, budget_s: float, par_calls: int):
    """Both of the reference's CPU paths on this workload: redzone_CPU (the reported baseline, its
    figure is `value`) and std::remove(par_unseq) beside it."""
    kind, cores, times = cpu_reference_time(n, k, steps, warmup, budget_s)
    mean = statistics.mean(times)
    rz_cpu = {"value": k / mean, "unit": UNIT, "ms_per_call": mean * 1e3, "calls": len(times), "cores": cores,
              "kind": kind}
    par = cpu_par_remove_time(n, k, par_calls, budget_s)
    host = {"hardware_threads": os.cpu_count(), "tbb": "project TBB-API shim (oneTBB not installed)"}
    return kind, cores, times, rz_cpu, par, host


def reference_arm(args):
    # The rank comes from the launcher's environment: this arm loads none of the package's code.
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n, k = 1 << N_LOG2, 1 << K_LOG2
    kind, cores, times, rz_cpu, par, host = cpu_baselines(n, k, args.steps, args.warmup, 120.0, par_calls=5)
    mean = statistics.mean(times)
    v = k / mean
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "impl": "reference",
        "config": config(world),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{len(times)} full calls of the workload (n=2^{N_LOG2}, k=2^{K_LOG2}) through "
                                   f"the reference's redzone_CPU; removal list restored before each call (the "
                                   f"reference clobbers it)",
                         "redzone_cpu": rz_cpu, "std_remove_par": par, "host": host},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------
def own_arm(args):
    import torch

    from redzone_b200 import dist

    world, rank, local = dist.init("nccl")
    if world == 1:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    import redzone_b200 as rz
    from redzone_b200 import _native, workloads
    from tests import _torch_rule

    ctx = rz.Context(dev.index)
    n, k = 1 << N_LOG2, 1 << K_LOG2
    a = torch.arange(n, dtype=torch.int32, device=dev)
    sets_np = [workloads.uniform(n, k, seed=dist.replica_seed(s, rank)) for s in range(NSETS)]
    sets = [torch.from_numpy(s.astype(np.int32)).to(dev) for s in sets_np]
    pinned = [torch.from_numpy(s.astype(np.int32)).pin_memory() for s in sets_np]
    scrub = torch.empty(SCRUB_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    # Parity gate (not timed): the first call must equal the canonical result.
    exp = _torch_rule.canonical_prefix(a, sets[0])
    ctx.remove(a, sets[0], flags=rz.RZ_SYNC)
    assert torch.equal(a[: n - k], exp), "parity check failed"
    del exp
    kernels_per_call, grid, block = ctx.last_launch()

    def barrier():
        dist.barrier(dev)

    def max_over_ranks(x: float) -> float:
        return dist.max_over_ranks(x, dev)

    # ---- Redzone, device-resident inputs ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(dev.index)
    clocks.start()
    time.sleep(0.25)  # let the sampler attach; the warm-up then runs right before the timed region
    for i in range(args.warmup):
        ctx.remove(a, sets[i % NSETS])
        scrub.fill_(i & 255)
    barrier()
    region0 = torch.cuda.Event(enable_timing=True)
    region1 = torch.cuda.Event(enable_timing=True)
    # Every timed step follows an L2 scrub on the GPU, the first one included: the scrub keeps the
    # stream busy while the host enqueues the first removal, so its start event does not time the
    # host's launch call (as it would on an idle stream).
    scrub.fill_(255)
    region0.record(stream)
    for i in range(args.steps):
        starts[i].record(stream)
        ctx.remove(a, sets[i % NSETS])
        ends[i].record(stream)
        scrub.fill_(i & 255)
    region1.record(stream)
    barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    step_stats = {"min": min(step_ms), "median": statistics.median(step_ms), "max": max(step_ms),
                  "first": step_ms[: min(8, len(step_ms))]}
    mean_ms = max_over_ranks(statistics.mean(step_ms))
    region_ms = max_over_ranks(region0.elapsed_time(region1))
    value = world * k / (mean_ms * 1e-3)

    # ---- steady state: one CUDA graph of NSETS x [removal, L2 scrub] replayed back to back, minus
    # the same graph with the scrubs alone (no per-step event or launch gaps) ----
    graphs = []
    for with_remove in (True, False):
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr):
            for i in range(NSETS):
                if with_remove:
                    ctx.remove(a, sets[i])
                scrub.fill_(i & 255)
        graphs.append(gr)
    reps = max(3, min(200, args.steps // NSETS))
    g_ms = []
    for gr in graphs:
        gr.replay()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            gr.replay()
        e1.record(stream)
        e1.synchronize()
        g_ms.append(e0.elapsed_time(e1))
    del graphs
    steady_ms = max_over_ranks(max(1e-6, (g_ms[0] - g_ms[1]) / (reps * NSETS)))

    # ---- L2-warm: the same event-timed removal with no scrub in between (the NSETS index lists,
    # 2 MB, and the tail window stay in L2; the hole positions differ per list). A spin kernel
    # that touches no memory stands between the steps in place of the scrub, so the host has
    # enqueued each removal before the GPU reaches it ----
    w_steps = max(NSETS, min(args.steps, 500))
    w_ev = []
    for i in range(w_steps + NSETS):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda._sleep(100_000)
        e0.record(stream)
        ctx.remove(a, sets[i % NSETS])
        e1.record(stream)
        if i >= NSETS:
            w_ev.append((e0, e1))
    torch.cuda.synchronize()
    warm_ms = max_over_ranks(statistics.mean(s_.elapsed_time(e_) for s_, e_ in w_ev))

    # ---- O(n) partition comparator on the same workload (fewer steps; ~1 GiB read + write each) ----
    p_steps = max(5, min(50, args.steps // 20))
    p_ms = []
    for i in range(p_steps + 2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.partition(a, sets[i % NSETS])
        e1.record(stream)
        scrub.fill_(i & 255)
        if i >= 2:
            p_ms.append((e0, e1))
    torch.cuda.synchronize()
    part_ms = max_over_ranks(statistics.mean(s.elapsed_time(e) for s, e in p_ms))

    # ---- the reference's own O(n) GPU comparator: mark with -1, then thrust::remove ----
    t_ms = []
    for i in range(p_steps + 2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.arange(n, out=a)  # the comparator needs -1 only where its marks put it
        scrub.fill_(i & 255)
        e0.record(stream)
        assert ctx.thrust_remove(a, sets[i % NSETS]) == n - k
        e1.record(stream)
        if i >= 2:
            t_ms.append((e0, e1))
    torch.cuda.synchronize()
    thrust_ms = max_over_ranks(statistics.mean(s.elapsed_time(e) for s, e in t_ms))

    # ---- event-timing floor: an empty kernel of the removal's launch shape, timed exactly like a
    # step (same events, same scrub before it) ----
    dcfg = ctx.default_cfg(n, k, W_BYTES)
    cluster = 8 if dcfg.schedule == _native.RZ_SCHED_CSCAN and grid % 8 == 0 else 1
    f_ev = []
    for i in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.empty_launch(grid, block, cluster)
        e1.record(stream)
        scrub.fill_(i & 255)
        if i >= args.warmup:
            f_ev.append((e0, e1))
    torch.cuda.synchronize()
    floor_ms = max_over_ranks(statistics.mean(s.elapsed_time(e) for s, e in f_ev))

    # ---- end to end through the public C-ABI with host buffers: every step copies its removal
    # list from pinned host memory and reads its result (status + device-tracked length) back.
    # Pipelined: rz_remove_host_idx_async keeps E_DEPTH calls in flight, so the copy of
    # step i+1 overlaps the kernel of step i; each step is collected with rz_wait. No L2 scrub
    # inside this region (each step's list arrives fresh over PCIe; E_SETS distinct lists) ----
    E_SETS, E_DEPTH = 64, 6
    e_np = [workloads.uniform(n, k, seed=dist.replica_seed(1000 + s, rank)) for s in range(E_SETS)]
    e_pinned = [torch.from_numpy(s.astype(np.int32)).pin_memory() for s in e_np]
    for i in range(max(args.warmup, E_DEPTH + 1)):  # first use grows the staging slots
        assert ctx.wait(ctx.remove_host_idx_async(a, e_pinned[i % E_SETS])) == n - k
    e_steps = max(args.steps, 1000)  # the 6-deep pipeline fills and drains once per region
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    inflight = []
    issue_s = 0.0
    for i in range(e_steps):
        h0 = time.perf_counter()
        inflight.append(ctx.remove_host_idx_async(a, e_pinned[i % E_SETS]))
        issue_s += time.perf_counter() - h0
        if len(inflight) == E_DEPTH:
            assert ctx.wait(inflight.pop(0)) == n - k
    for t in inflight:
        assert ctx.wait(t) == n - k
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e_steps)
    barrier()
    # The same pipelined loop from C++ through the C-ABI (redzone_b200/_lib/rz_e2e, the program a
    # caller of the reference's redzone_CPU would write): no interpreter between the calls.
    e2e_cpp = None
    drv = ROOT / "redzone_b200" / "_lib" / "rz_e2e"
    if drv.exists() and world == 1:
        try:
            r = subprocess.run([str(drv), str(N_LOG2), str(K_LOG2), str(e_steps), str(E_DEPTH), str(E_SETS)],
                               capture_output=True, text=True, timeout=600)
            out = json.loads(r.stdout.strip().splitlines()[-1]) if r.stdout.strip() else {}
            if r.returncode == 0 and "ms_per_step" in out:
                e2e_cpp = out
        except Exception:
            e2e_cpp = None
    clk = clocks.stop()
    # The synchronous call, one step at a time (copy, kernel, read-back, host wait in series).
    s_ms = []
    for i in range(args.warmup + min(e_steps, 200)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        assert ctx.remove_host_idx(a, e_pinned[i % E_SETS]) == n - k
        e1.record(stream)
        if i >= args.warmup:
            s_ms.append((e0, e1))
    torch.cuda.synchronize()
    e2e_serial_ms = max_over_ranks(statistics.mean(s.elapsed_time(e) for s, e in s_ms))

    # ---- roofline of the Redzone kernel ----
    balg = statistics.mean(alg_bytes(n, k, W_BYTES, s) for s in sets_np)
    achieved = balg / (mean_ms * 1e-3) / 1e9
    peak, peak_kind = load_peaks()
    traffic = load_traffic(f"redzone_single_n2e{N_LOG2}_k2e{K_LOG2}_w{W_BYTES}")

    # ---- the batched half of the metric: 4096 uneven lists in one launch against per-list launches ----
    bat = None
    if not args.no_batched:
        del a, sets, scrub
        torch.cuda.empty_cache()
        bat = batched_leg(args, ctx, dev, world, rank, steps=max(5, min(args.steps, 20)), warmup=args.warmup)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        kind, cores, times, rz_cpu, par, host = cpu_baselines(n, k, 50, 2, 20.0, par_calls=3)
        cpu = {"value": k / statistics.mean(times), "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"{len(times)} full calls of the same workload (n=2^{N_LOG2}, k=2^{K_LOG2}) on the host "
                         f"through the reference's redzone_CPU",
               "redzone_cpu": rz_cpu, "std_remove_par": par, "host": host}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": config(world),
            "timed_region_ms": region_ms,
            "gpu_launches": args.steps * kernels_per_call,
            "launch": {"grid": grid, "block": block, "kernels_per_call": kernels_per_call},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_launch": balg, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s"},
            "partition_on": {"ms_per_step": part_ms, "speedup_redzone_vs_partition": part_ms / mean_ms},
            "thrust_remove_on": {"ms_per_step": thrust_ms, "speedup_redzone_vs_thrust": thrust_ms / mean_ms,
                                 "what": "the reference's O(n) GPU comparator: mark with -1, then "
                                         "thrust::remove (Thrust_remove.hxx:15-17), same workload"},
            "warm_l2": {"ms_per_step": warm_ms, "items_per_s": world * k / (warm_ms * 1e-3), "steps": w_steps,
                        "method": f"the same event-timed call, {NSETS} index lists in rotation, no L2 scrub (a "
                                  f"spin kernel touching no memory between steps)"},
            "graph_steady_state": {
                "ms_per_removal": steady_ms, "items_per_s": world * k / (steady_ms * 1e-3),
                "speedup_vs_partition": part_ms / steady_ms,
                "method": f"CUDA graph of {NSETS} x [removal, 256 MiB scrub] replayed {reps} times, minus the "
                          f"same graph of scrubs alone, divided by the removals"},
            "step_ms": step_stats,
            "event_floor_ms": floor_ms,
            "floor_method": f"empty kernel of the removal's shape ({grid} x {block}, clusters of {cluster}) "
                            f"between the same events after the same scrub, {args.steps} steps",
            "removal_share_of_step": max(0.0, (mean_ms - floor_ms) / mean_ms),
            "e2e": e2e_line(k, world, e2e_cpp, {
                "value": world * k / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 4 * k,
                "d2h_bytes_per_step": RESULT_BYTES, "ms_per_step": e2e_ms, "steps": e_steps,
                "method": f"Python (ctypes) caller: rz_remove_host_idx_async, {E_DEPTH} calls in flight, each "
                          f"step's list copied from pinned host memory and its status + new length read back "
                          f"(16 bytes), rz_wait on every step; time of the whole region / steps; {E_SETS} "
                          f"distinct lists, no L2 scrub",
                "serial_ms_per_step": e2e_serial_ms, "host_issue_us_per_call": 1e6 * issue_s / e_steps}),
            "cpu_baseline": cpu,
            "batched": bat,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def e2e_line(k: int, world: int, cpp: dict | None, py: dict) -> dict:
    """The e2e object: the C++ caller's figure when its driver ran (the reference's users are C++
    programs), else the Python caller's; both are kept."""
    if cpp is None:
        return dict(py, python=None)
    return {"value": world * k / (cpp["ms_per_step"] * 1e-3), "unit": UNIT,
            "h2d_bytes_per_step": cpp["h2d_bytes_per_step"], "d2h_bytes_per_step": cpp["d2h_bytes_per_step"],
            "ms_per_step": cpp["ms_per_step"], "steps": cpp["steps"],
            "method": f"C++ caller through the C-ABI (redzone_b200/_lib/rz_e2e): rz_remove_host_idx_async, "
                      f"{cpp['depth']} calls in flight, each step's list copied from pinned host memory and its "
                      f"status + new length read back (16 bytes), rz_wait on every step (status and length "
                      f"checked); CUDA events around the whole region / steps; {cpp['sets']} distinct lists, "
                      f"no L2 scrub",
            "serial_ms_per_step": cpp["serial_ms_per_step"], "host_issue_us_per_call": cpp["host_issue_us_per_call"],
            "python": py}


# ------------------------------------------------------------------------------------------------
def sweep(args):
    """k sweep at n = 2^28 for int32 and 16-byte payloads, three distributions (one JSON per line)."""
    import torch
    import redzone_b200 as rz
    from redzone_b200 import workloads

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    ctx = rz.Context(0)
    n = 1 << N_LOG2
    peak, _ = load_peaks()
    scrub = torch.empty(SCRUB_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    ks = [int(x) for x in args.sweep_k.split(",")] if args.sweep_k else list(range(10, 28))
    widths = [int(x) for x in args.sweep_w.split(",")] if args.sweep_w else [4, 16]
    dists = args.sweep_dist.split(",") if args.sweep_dist else ["uniform", "clustered", "tail"]
    for w in widths:
        a = torch.zeros((n, w // 4), dtype=torch.int32, device=dev)
        a[:, 0] = torch.arange(n, dtype=torch.int32, device=dev)
        for dist in dists:
            for kl in ks:
                k = 1 << kl
                if dist == "tail" and k > n // 10:
                    continue
                idx = workloads.make_torch(dist, n, k, seed=kl).contiguous()
                idx_np = idx.cpu().numpy().astype(np.int64)
                reps = 20 if kl < 22 else 5
                res = {}
                for name, fn in (("redzone", lambda: ctx.remove(a, idx)), ("partition", lambda: ctx.partition(a, idx))):
                    fn()
                    ev = []
                    for r in range(reps + (0 if name == "redzone" else 0)):
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        scrub.fill_(r & 255)
                        e0.record(stream)
                        fn()
                        e1.record(stream)
                        ev.append((e0, e1))
                    torch.cuda.synchronize()
                    res[name] = statistics.median(s.elapsed_time(e) for s, e in ev)
                balg = alg_bytes(n, k, w, idx_np)
                holes = idx[idx < n - k].contiguous()
                ev = []
                for r in range(reps):
                    scrub.fill_(r & 255)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ctx.scatter(a, holes)
                    e1.record(stream)
                    ev.append((e0, e1))
                torch.cuda.synchronize()
                scatter_ms = statistics.median(s.elapsed_time(e) for s, e in ev)
                line = {"n": n, "k": k, "w": w, "dist": dist, "redzone_ms": res["redzone"],
                        "scatter_ms": scatter_ms, "holes": int(holes.numel()),
                        "partition_ms": res["partition"], "items_per_s": k / (res["redzone"] * 1e-3),
                        "alg_bytes": balg, "achieved_gbs": balg / (res["redzone"] * 1e-3) / 1e9,
                        "frac_of_hbm": balg / (res["redzone"] * 1e-3) / 1e9 / peak,
                        "speedup_vs_partition": res["partition"] / res["redzone"]}
                print(json.dumps(line), flush=True)
                del idx
        del a
        torch.cuda.empty_cache()


def make_batched_lists(args, dev, world, rank):
    """This rank's share of the batched workload on the device: (lists, n, k of all lists)."""
    import torch
    from redzone_b200 import dist, workloads

    n_all, k_all = workloads.batched_lists(args.lists, seed=args.seed)
    mine = dist.shard_by_weight(k_all, world, rank)
    n, k = n_all[mine], k_all[mine]
    buf = torch.empty(int(n.sum()), dtype=torch.int64, device=dev)
    g = torch.Generator(device=dev)
    lists, off = [], 0
    for q, l in enumerate(mine):
        ni, ki = int(n[q]), int(k[q])
        seg = buf[off: off + ni]
        torch.arange(ni, out=seg)
        seg.add_(int(l) << 32)
        g.manual_seed(args.seed * 100003 + int(l))  # the list's indices depend on the list alone
        idx = torch.randperm(ni, generator=g, device=dev)[:ki].to(torch.int32)
        lists.append((seg, idx))
        off += ni
    return buf, lists, n_all, k_all


def scatter_floor(ctx, buf, lists, reps: int, scrub=None) -> dict:
    """The hole writes of `lists` alone: plain scattered stores (rz_test_scatter) of every hole
    position (idx < n - k) into `buf`, which the lists are segments of. Overwrites the lists."""
    import torch

    base = buf.data_ptr()
    pos = []
    for d, i in lists:
        cut = d.shape[0] - i.numel()
        off = (d.data_ptr() - base) // buf.element_size()
        pos.append(i[i < cut].to(torch.int64) + off)
    pos = torch.cat(pos).to(torch.int32) if pos else torch.zeros(0, dtype=torch.int32, device=buf.device)
    stream = torch.cuda.current_stream()
    flat = buf.view(buf.shape[0], -1)
    ctx.scatter(flat, pos)
    ts = []
    for r in range(reps):
        if scrub is not None:
            scrub.fill_(r & 255)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.scatter(flat, pos)
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    h = int(pos.numel())
    del pos
    ms = statistics.median(ts)
    return {"holes": h, "ms": ms, "holes_per_s": h / (ms * 1e-3)}


def batched_leg(args, ctx, dev, world: int, rank: int, steps: int, warmup: int) -> dict:
    """4096 uneven lists (n log-uniform in [2^8, 2^22], k = round(f n), f ~ U(0.001, 0.5), uint64
    payload = list id << 32 | index) in one persistent graph-replayed launch, its configuration
    picked by the learned list-mix predictor, against one rz_remove launch per list (stream-
    launched, and the same launches captured in one CUDA graph), against the built-in default
    configuration, and against every configuration of the space (exhaustive autotune: the
    reference point of the predictor's regret). N > 1: the lists are partitioned across ranks by removals
    (contiguous, balanced), each rank runs its share as one launch; no collective on the data path,
    max-over-ranks timing. The payload (about 14 GB) is far larger than L2."""
    import torch
    import redzone_b200 as rz
    from redzone_b200 import _native, dist, learn_batched
    from tests import _torch_rule

    buf, lists, n_all, k_all = make_batched_lists(args, dev, world, rank)
    nlists = len(lists)
    total_n, total_k = int(n_all.sum()), int(k_all.sum())
    w = 8
    stream = torch.cuda.current_stream()
    descs = rz.list_descs(lists)
    model = None if args.no_learned else learn_batched.attach_default(ctx)
    pred = _native.BatchCfg()
    learned = model is not None and _native.lib.rz_predict_batch_cfg(ctx.handle, descs, nlists, w,
                                                                     ctypes_byref(pred)) == 0

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    # Parity gate on a sample of lists (not timed), with the plan that is timed below: created
    # without a configuration, so the attached network (or, without it, the default) chooses.
    sample = list(range(0, nlists, max(1, nlists // 64)))
    exp = {l: _torch_rule.canonical_prefix(lists[l][0].clone(), lists[l][1]) for l in sample}
    plan = rz.BatchPlan(ctx, lists)
    plan.launch()
    torch.cuda.synchronize()
    assert ctx.sync_status() == 0
    for l in sample:
        ni, ki = lists[l][0].shape[0], lists[l][1].numel()
        assert torch.equal(lists[l][0][: ni - ki], exp[l]), f"batched parity failed on list {l}"
    del exp
    for _ in range(warmup):
        plan.launch()
    dist.barrier(dev)
    batched_ms = dist.max_over_ranks(timed(plan.launch, steps), dev)
    info = plan.info()
    plan.close()

    def time_cfg(cfg, reps):
        try:
            pl = rz.BatchPlan(ctx, lists, cfg)
        except rz.RedzoneError:
            return float("inf")
        pl.launch()
        t = timed(pl.launch, reps)
        pl.close()
        return t

    space = learn_batched.config_space()
    dflt = space[learn_batched.default_class(None, w)]
    default_ms = dist.max_over_ranks(time_cfg(_native.BatchCfg(*dflt[:3], 0, dflt[3]), max(3, steps // 2)), dev)
    exhaustive = None
    if not args.no_tune:
        ts = [dist.max_over_ranks(time_cfg(_native.BatchCfg(b, i, c, 0, wv), 3), dev) for b, i, c, wv in space]
        q = int(np.argmin(ts))
        exhaustive = {"best_cfg": list(space[q]), "best_ms": ts[q], "configurations": len(space),
                      "default_regret": default_ms / ts[q] - 1.0}
        if learned:
            exhaustive["learned_regret"] = batched_ms / ts[q] - 1.0

    def plain():
        for d, i in lists:
            ctx.remove(d, i)
    plain()
    plain_ms = dist.max_over_ranks(timed(plain, max(3, steps // 5)), dev)
    # The same per-list launches captured once into a CUDA graph (no host launch overhead).
    plain_graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(plain_graph):
        plain()
    plain_graph.replay()
    plain_graph_ms = dist.max_over_ranks(timed(plain_graph.replay, max(3, steps // 5)), dev)
    del plain_graph
    # Algorithmic bytes: red-zone entries estimated from a sample of this rank's lists.
    kr_s = k_s = 0
    for d, i in lists[:: max(1, nlists // 256)]:
        kr_s += int((i >= d.shape[0] - i.numel()).sum().item())
        k_s += i.numel()
    my_k = sum(i.numel() for _, i in lists)
    k_r = my_k * (kr_s / max(1, k_s))
    balg = 4.0 * my_k + 2.0 * w * (my_k - k_r) + my_k / 4.0
    peak, peak_kind = load_peaks()
    # The same hole writes as plain scattered stores (after the timings above: it overwrites lists).
    sf = scatter_floor(ctx, buf, lists, reps=3)
    sf["removal_time_over_scatter_time"] = batched_ms / sf["ms"]
    if model is not None:
        model.close()
    del lists, buf
    torch.cuda.empty_cache()
    return {
        "workload": f"{args.lists} lists, n log-uniform [2^8, 2^22], k = round(f n), f ~ U(0.001, 0.5), "
                    f"uint64 payload (list id << 32 | index), one persistent graph-replayed launch per GPU",
        "total_n": total_n, "total_k": total_k, "batch_cfg": info,
        "configuration_from": "learned list-mix predictor" if learned else "built-in default (no predictor)",
        "learned_cfg": [pred.block, pred.items, pred.ctas_per_sm, pred.wave] if learned else None,
        "items_per_s": total_k / (batched_ms * 1e-3), "ms_per_launch": batched_ms, "steps": steps,
        "parallelism": "single GPU" if world == 1 else f"{world} GPUs, lists partitioned by removals",
        "plain_per_list": {"ms_per_step": plain_ms, "speedup_batched_vs_plain": plain_ms / batched_ms},
        "plain_per_list_graph": {"ms_per_step": plain_graph_ms,
                                 "speedup_batched_vs_plain": plain_graph_ms / batched_ms},
        "speedup_vs_plain": plain_ms / batched_ms,
        "default_cfg": {"cfg": list(dflt), "ms_per_launch": default_ms},
        "exhaustive_autotune": exhaustive,
        "roofline": {"bound": "hbm", "achieved": balg / (batched_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": balg / (batched_ms * 1e-3) / 1e9 / peak, "traffic": None,
                     "alg_bytes_per_launch": balg, "peak_source": peak_kind},
        "parity": f"{len(sample)} sampled lists bit-exact against the canonical rule before timing",
        "scatter_floor": sf,
    }


def batched(args):
    """--workload batched: the batched leg as its own JSON line."""
    import torch
    import redzone_b200 as rz
    from redzone_b200 import dist

    world, rank, local = dist.init("nccl")
    if world == 1:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    ctx = rz.Context(dev.index)
    b = batched_leg(args, ctx, dev, world, rank, args.steps, args.warmup)
    line = {
        "metric": METRIC, "value": b["items_per_s"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": b["ms_per_launch"], "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": b["workload"], "total_n": b["total_n"], "total_k": b["total_k"],
                   "batch_cfg": b["batch_cfg"], "parallelism": b["parallelism"],
                   "configuration_from": b["configuration_from"]},
        "plain_per_list": b["plain_per_list"], "plain_per_list_graph": b["plain_per_list_graph"],
        "default_cfg": b["default_cfg"], "exhaustive_autotune": b["exhaustive_autotune"],
        "scatter_floor": b["scatter_floor"], "roofline": b["roofline"], "gpu_launches": args.steps,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()


def service(args):
    """Streaming delete service: a 2^27 x 32-byte table (uint64 key + three uint64 words) split
    into shards; Poisson arrivals of delete batches (size round(2^U(0,20)) distinct live rows,
    drawn from a pool of pinned batches) to random shards; a shard that a batch would take below
    half its capacity is first refilled to capacity by appending fresh records (add-then-remove).
    Reported: sustained rows deleted/s and p50/p99 submit->completion latency at the offered
    rate, and the saturated capacity (arrivals far above what the device drains)."""
    import torch
    import redzone_b200 as rz

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    ctx = rz.Context(0)
    n_total, words = 1 << 27, 8
    shards = args.shards
    cap = n_total // shards
    floor = cap // 2
    table = torch.empty((n_total, words), dtype=torch.int32, device=dev)
    table.zero_()
    keys = torch.arange(n_total, dtype=torch.int64, device=dev)
    table[:, 0:2] = keys.view(torch.int32).view(n_total, 2)
    del keys
    g = torch.Generator(device=dev)
    g.manual_seed(args.seed)
    rng = np.random.default_rng(args.seed)
    pool = []
    for _ in range(args.pool):
        k = int(round(2 ** rng.uniform(0, 20)))
        pool.append(torch.randperm(floor, generator=g, device=dev)[:k].to(torch.int32).cpu().pin_memory())
    mean_batch = float(np.mean([p.numel() for p in pool]))
    svc = rz.Service(ctx, table, shards, cap, slots=args.slots, max_batches_per_launch=args.max_batches,
                     index_budget_bytes=args.index_budget_mb << 20, floor_rows=floor)
    svc.run_poisson(pool, rate=args.rate, seconds=0.25, seed=args.seed + 1)  # warm-up (plans, arenas, clocks)
    svc.reset_stats()
    sampler = ClockSampler(0)
    sampler.start()
    at_rate = svc.run_poisson(pool, rate=args.rate, seconds=args.seconds, seed=args.seed + 2)
    clocks = sampler.stop()
    svc.reset_stats()
    saturated = svc.run_poisson(pool, rate=args.rate * 20, seconds=min(args.seconds, 1.0), seed=args.seed + 3)
    host_len, dev_len = svc.lengths()
    assert host_len == dev_len, "device-tracked lengths differ from the host view"
    svc.close()
    torch.cuda.synchronize()
    # Property gate (not timed): live rows hold distinct keys (no record duplicated or lost twice).
    live = torch.cat([table[s * cap: s * cap + host_len[s], 0:2].contiguous().view(torch.int64).view(-1)
                      for s in range(shards)])
    assert torch.unique(live).numel() == live.numel() == sum(host_len), "service lost or duplicated records"
    del live

    def summary(st):
        secs = max(st["busy_seconds"], 1e-9)
        return {"rows_deleted_per_s": st["rows_deleted"] / secs, "batches_per_s": st["completed"] / secs,
                "p50_us": st["p50_us"], "p99_us": st["p99_us"], "mean_us": st["mean_us"], "max_us": st["max_us"],
                "batches": st["completed"], "launches": st["launches"], "refills": st["refills"],
                "mean_batches_per_launch": st["mean_batches_per_launch"], "seconds": secs}

    r = summary(at_rate)
    line = {
        "metric": "rows deleted/s", "value": r["rows_deleted_per_s"], "unit": "rows/s", "n_gpus": 1,
        "steps": int(at_rate["completed"]), "warmup": 0, "ms_per_step": 1e3 * r["seconds"] / max(1, r["batches"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64x4 records",
        "data": "synthetic",
        "config": {"workload": f"streaming delete service, 2^27 x 32-byte records in {shards} shards, Poisson "
                               f"{args.rate:g} batches/s, batch size round(2^U(0,20)) from a pool of {args.pool} "
                               f"pinned batches, refill to capacity below half", "mean_batch_rows": mean_batch,
                   "offered_rows_per_s": args.rate * mean_batch, "slots": args.slots,
                   "max_batches_per_launch": args.max_batches, "index_budget_mb": args.index_budget_mb},
        "at_offered_rate": r,
        "saturated": summary(saturated),
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def ctypes_byref(x):
    import ctypes
    return ctypes.byref(x)


def produced(args):
    """Removal of a list made on the GPU with fused red-zone marking (rz_emit / rz_remove_produced)
    against rz_remove on the same list: n = 2^28 int32 rows, a producer that deletes every row
    whose uint32 key is below a threshold (k = 2^16 of them, uniform), L2 flushed between steps."""
    import torch
    import redzone_b200 as rz

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    ctx = rz.Context(0)
    n, k = 1 << N_LOG2, 1 << K_LOG2
    scrub = torch.empty(SCRUB_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    a = torch.arange(n, dtype=torch.int32, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(args.seed)
    keys = torch.randint(1 << 30, (1 << 31) - 1, (n,), device=dev, dtype=torch.int32, generator=g)
    keys[torch.randperm(n, device=dev, generator=g)[:k]] = 5
    thr = 1 << 30
    prod = rz.Producer(ctx, capacity=k, cand_capacity=4096)
    prod.reset(n)
    prod.produce_where_less(keys, thr)
    lst, kk, cands = prod.download()
    assert kk == k
    d_list = torch.from_numpy(lst.view(np.int32)).to(dev)
    # Parity gate: both paths give the same bits on the same list.
    a2 = a.clone()
    prod.remove(a, flags=rz.RZ_SYNC)
    ctx.remove(a2, d_list, flags=rz.RZ_SYNC)
    assert torch.equal(a, a2), "produced and index-list removals differ"
    del a2

    def ev_mean(fn, steps):
        for i in range(args.warmup):
            fn()
            scrub.fill_(i & 255)
        ev = []
        for i in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            scrub.fill_(i & 255)
            ev.append((e0, e1))
        torch.cuda.synchronize()
        return statistics.mean(s.elapsed_time(e) for s, e in ev)

    def steady(fn):
        ms = []
        for with_fn in (True, False):
            gr = torch.cuda.CUDAGraph()
            with torch.cuda.graph(gr):
                for i in range(NSETS):
                    if with_fn:
                        fn()
                    scrub.fill_(i & 255)
            gr.replay()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(100):
                gr.replay()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            del gr
        return (ms[0] - ms[1]) / (100 * NSETS)

    steps = min(args.steps, 1000)
    t_prod = ev_mean(lambda: prod.remove(a), steps)
    t_list = ev_mean(lambda: ctx.remove(a, d_list), steps)
    s_prod, s_list = steady(lambda: prod.remove(a)), steady(lambda: ctx.remove(a, d_list))

    def round_fused():
        prod.reset(n)
        prod.produce_where_less(keys, thr)
        prod.remove(a)

    t_round = ev_mean(round_fused, min(steps, 200))
    print(json.dumps({
        "metric": METRIC, "value": k / (t_prod * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": t_prod, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "removal of a GPU-produced list with fused red-zone marking, n=2^28 int32, "
                               "k=2^16 rows whose uint32 key is below a threshold (uniform)",
                   "n": n, "k": k, "elem_bytes": 4, "capacity": k, "candidates": cands,
                   "l2": "flushed between timed steps (256 MiB scrub write)", "parallelism": "single GPU"},
        "index_list_same_rows": {"ms_per_step": t_list, "items_per_s": k / (t_list * 1e-3)},
        "graph_steady_state": {"produced_ms": s_prod, "index_list_ms": s_list},
        "producer_and_removal_round_ms": t_round,
        "gpu_launches": steps,
    }), flush=True)
    prod.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["own", "reference"], default="own")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--sweep", action="store_true", help="run the k sweep instead of the headline")
    ap.add_argument("--sweep-k", default="", help="comma-separated log2(k) values for --sweep")
    ap.add_argument("--sweep-w", default="", help="comma-separated item widths for --sweep (default 4,16)")
    ap.add_argument("--sweep-dist", default="", help="comma-separated distributions for --sweep")
    ap.add_argument("--workload", choices=["single", "batched", "service", "produced"], default="single")
    ap.add_argument("--shards", type=int, default=16, help="--workload service: table shards")
    ap.add_argument("--slots", type=int, default=4, help="--workload service: concurrent launch slots")
    ap.add_argument("--max-batches", type=int, default=16, help="--workload service: batches per launch")
    ap.add_argument("--index-budget-mb", type=int, default=256, help="--workload service: device index budget")
    ap.add_argument("--rate", type=float, default=20000.0, help="--workload service: batches/s offered")
    ap.add_argument("--seconds", type=float, default=2.0, help="--workload service: timed seconds")
    ap.add_argument("--pool", type=int, default=256, help="--workload service: pinned batch pool size")
    ap.add_argument("--lists", type=int, default=4096, help="--workload batched: number of lists")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-tune", action="store_true", help="batched: skip the exhaustive autotune")
    ap.add_argument("--no-batched", action="store_true", help="default run: skip the batched leg")
    ap.add_argument("--no-learned", action="store_true", help="batched: do not attach the list-mix predictor")
    ap.add_argument("--config", default=None,
                    help="JSON file of option defaults, e.g. {\"workload\": \"service\", \"rate\": 40000}; "
                         "flags on the command line override it")
    pre, _ = ap.parse_known_args()
    if pre.config:
        cfg = json.loads(Path(pre.config).read_text())
        known = {a.dest for a in ap._actions}
        unknown = sorted(set(cfg) - known)
        if unknown:
            ap.error(f"unknown keys in {pre.config}: {unknown}")
        ap.set_defaults(**cfg)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
    elif args.sweep:
        sweep(args)
    elif args.workload == "batched":
        batched(args)
    elif args.workload == "service":
        service(args)
    elif args.workload == "produced":
        produced(args)
    else:
        own_arm(args)


if __name__ == "__main__":
    main()
