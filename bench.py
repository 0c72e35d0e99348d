"""Benchmark: full tree pipeline (Morton -> sort -> build -> geometry -> lists).

One step = ``build_tree`` (radix/LBVH, leaf 32) + ``compute_tree_geometry`` +
``build_interactions_and_neighbors`` (dehnen, theta 0.6, exact count-then-
fill lists) over N = 16,777,216 float32 Plummer particles (seed 4, scale
radius 1, truncated at r = 20, equal masses).  The metric is particles/s of
the whole step.

* ``value``: inputs already resident in HBM, CUDA-event timed over K steps.
* ``e2e``: the same step through the public API from pinned host buffers:
  host->device copy of positions and masses and device->host copy of the
  per-node far/near counts inside the timed region, every step; the next
  step's upload runs on a copy stream during the current step's compute
  (``serial_value``: copy, then compute, on one stream).
* ``roofline``: the build's HBM-bound kernel (the onesweep sort passes)
  timed with CUDA events inside this run, against the measured HBM copy
  bandwidth; the traversal is latency bound and is reported as pairs/s.
* ``modes``: the same step with each traversal schedule (all return the same
  exact lists): ``log`` (one walk + pair log, the default and ``value``),
  ``two_pass`` (the reference's count walk + fill walk) and ``learned`` (one
  walk into rows sized by the learned capacity predictor, with its overflow
  and over-allocation figures).
* ``cpu_baseline``: the CPU restatement of the pipeline (OpenMP, all host
  cores) on the full workload, timed once.
* ``--impl reference``: that CPU implementation on the host cores as the
  reference arm (the reference itself is JAX, which this image lacks), every
  step the full workload, with the same ``config``.

With ``--gpus N`` (torchrun, one rank per GPU) every rank runs its own
replica: the path does not shard, so there is no collective; the value is
the particles of all ranks over the slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_DEFAULT = 16_777_216
# dram__bytes_read.sum + dram__bytes_write.sum of one onesweep launch (ncu,
# keys = Morton codes of the Plummer input), by (key count, digit bits).
SORT_PASS_DRAM_BYTES: dict = {(16_777_216, 8): 361_430_000}
LEAF = 32
THETA = 0.6
MAC = "dehnen"
WORKLOAD = "plummer_16M_radix_leaf32_dehnen_theta0.6_exact_lists"


def workload_name(n: int) -> str:
    """The workload label for an n-particle run (the 16M name at the default size)."""
    return WORKLOAD if n == N_DEFAULT else WORKLOAD.replace("16M", str(n))
METRIC = "particles/s full build+traversal (Morton, sort, radix build, geometry, exact lists)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.window = None  # (start, end) host wall-clock seconds of the timed region

    def mark(self, start: float, end: float) -> None:
        """Record the timed region; summary() then keeps only samples inside it."""
        self.window = (start, end)

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # nvidia-smi's start-up (driver / NVML initialisation) must not overlap
        # the timed region: wait for its first sample line.
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 10.0:
            if os.path.getsize(self.path) > 0 or self.proc.poll() is not None:
                break
            time.sleep(0.05)
        time.sleep(0.1)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import datetime

        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []  # (time or None, sm MHz, max MHz, active reasons)
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 10:
                    continue
                try:
                    t = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    t = None
                try:
                    rows.append((t, float(f[2]), float(f[3]),
                                 {n for n, v in zip(names, f[6:10]) if v.lower() == "active"}))
                except ValueError:
                    continue
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        inside = rows
        if self.window is not None:
            lo, hi = self.window
            inside = [r for r in rows if r[0] is not None and lo <= r[0] <= hi]
        where = "timed region"
        if not inside:  # region shorter than one sample interval: keep every sample
            inside, where = rows, "whole sampler run (no sample fell inside the timed region)"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        reasons = set().union(*(r[3] for r in inside))
        return {"sm_mhz": float(np.median([r[1] for r in inside])),
                "sm_max_mhz": float(max(r[2] for r in inside)),
                "reasons": sorted(reasons), "samples": len(inside), "samples_from": where,
                "interval_ms": 20}


def _max_over_ranks(values, device):
    """Element-wise maximum of ``values`` over all ranks (identity on one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_pipeline(pos, mass):
    """CPU restatement of one step (used for the CPU baseline only)."""
    from oracle import oracle as O

    t = O.build_tree(pos, mass, leaf_size=LEAF)
    g = O.compute_tree_geometry(t, t.positions_sorted)
    r = O.build_interactions_and_neighbors(t, g, theta=THETA, mac_type=MAC)
    return t, r


def workload_config(n: int, world: int, total_nodes: int, far_entries: int,
                    near_entries: int) -> dict:
    """The workload definition both arms report (identical dicts when the
    arms ran the same workload)."""
    return {"workload": workload_name(n), "n_particles": n, "leaf_size": LEAF, "mac": MAC,
            "theta": THETA, "total_nodes": total_nodes, "far_entries": far_entries,
            "near_entries": near_entries,
            "l2": (f"inputs ({16 * n / 1e6:.0f} MB) "
                   f"{'larger' if 16 * n > 126e6 else 'smaller'} than L2 (126 MB); "
                   "no flush between steps"),
            "parallelism": f"replicas{world}"}


def cpu_baseline(n: int):
    """The CPU restatement on the full workload, timed once (wall clock,
    all host threads) after one untimed warm call on a small sample."""
    from oracle import oracle as O
    from yggdrax_b200 import inputs

    O.build()
    pos, mass = inputs.plummer(n, 4)
    cpu_pipeline(pos[:65536], mass[:65536])  # load the library, start the thread pool
    t0 = time.perf_counter()
    cpu_pipeline(pos, mass)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "particles/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"the full workload ({n} Plummer particles, seed 4, radix leaf "
                      f"{LEAF}, {MAC} theta {THETA}, exact lists), one timed run, wall "
                      "clock, after one untimed warm call on 65,536 of the particles"}


def run_reference(args):
    """The reference arm: the CPU restatement of the path (the reference
    itself is JAX, absent from this image) on the host cores, every step the
    full workload of this arm."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    n = args.n
    from oracle import oracle as O
    from yggdrax_b200 import inputs

    O.build()
    pos, mass = inputs.plummer(n, 4)
    for _ in range(args.warmup):
        t, r = cpu_pipeline(pos, mass)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t, r = cpu_pipeline(pos, mass)
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    v = n / dt
    cfg = workload_config(n, args.gpus, int(t.node_ranges.shape[0]), int(r["sources"].shape[0]),
                          int(r["neighbors"].shape[0]))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "particles/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+int64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": v, "unit": "particles/s", "cores": O.num_threads(),
                         "kind": "port",
                         "sample": f"the full workload ({n} Plummer particles) every step, "
                                   "wall clock, all host threads; the reference is JAX-only "
                                   "and JAX is not installed"},
        "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def sort_roofline(codes, dev, reps: int) -> dict:
    """The build's HBM-bound kernel: the onesweep LSD sort of the Morton codes
    (key u64 + value u32 over 63 bits) at the digit width the autotuner chose
    -- 8-bit digits in 8 passes (k_onesweep) or 11-bit digits in 6 passes
    (k_onesweep_wide) -- timed with CUDA events on its own stream, L2 flushed
    (256 MB write) before every sort; the other width is timed the same way
    and reported beside it.  Algorithmic bytes: read key + value, write key +
    value (24 B per key) on every pass but the first, which reads no values
    (its values are the input positions), 20 B per key; per launch the mean
    over the passes (23.5 B per key at 8 passes, 23.33 B at 6)."""
    import torch

    from yggdrax_b200 import _lib as L
    from yggdrax_b200 import autotune

    lib = L.lib()
    n = int(codes.numel())
    kout = torch.empty_like(codes)
    vout = torch.empty(n, dtype=torch.int32, device=dev)
    wsb = L.workspace(lib.ygx_sort_pairs_workspace_size(n), dev)
    st = L.stream_handle(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def sort_once():
        L.check(lib.ygx_sort_pairs(L.ptr(codes), None, n, 0, 63, L.ptr(kout), L.ptr(vout),
                                   L.ptr(wsb), wsb.numel(), st), "ygx_sort_pairs")

    def timed(fn, warm):
        for _ in range(warm):
            fn()
        ms = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(a.elapsed_time(b))
        return float(np.median(ms))

    chosen = autotune.current()["sort_bits"]
    by_bits = {}
    try:
        for bits in (8, 11):
            autotune.apply({"sort_bits": bits})
            by_bits[bits] = timed(sort_once, 3)
    finally:
        autotune.apply({"sort_bits": chosen})
    # Library reference point: CUB's radix sort through torch.sort (stable,
    # int64 keys, int64 indices: 32 B per key per pass) on the same codes.
    c64 = codes.view(torch.int64)
    lib_ms = timed(lambda: torch.sort(c64, stable=True), 2)
    passes = 6 if chosen == 11 else 8
    sort_s = by_bits[chosen] / 1e3
    bytes_per_pass = (20.0 + 24.0 * (passes - 1)) / passes * n
    achieved = bytes_per_pass / (sort_s / passes) / 1e9
    peak, peak_kind = _peaks()
    kernel = ("k_onesweep_wide (6 passes, 11-bit digits, key u64 + value u32)" if chosen == 11
              else "k_onesweep (8 passes, 8-bit digits, key u64 + value u32)")
    return {"kernel": kernel, "digit_bits": chosen, "passes": passes,
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": SORT_PASS_DRAM_BYTES.get((n, chosen)),
            "algorithmic_bytes_per_launch": bytes_per_pass,
            "launch_ms_avg": sort_s / passes * 1e3, "n_keys": n,
            "sort_ms": sort_s * 1e3, "sort_ms_by_digit_bits": by_bits,
            "torch_sort_stable_ms": lib_ms}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--breakdown", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the compact / mutual / moments / grouped / octree-walk timings")
    ap.add_argument("--no-modes", action="store_true",
                    help="skip timing the two-pass and learned traversal schedules")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shapes (skip the autotuner)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip timing the batched workload (4096 uneven point sets)")
    ap.add_argument("--roofline-only", action="store_true",
                    help="time only the sort roofline leg (for profiling it)")
    ap.add_argument("--mode", default="learned",
                    choices=["log", "two_pass", "learned", "target", "target_ordered"],
                    help="traversal schedule of the main timing (all give the same lists)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import _lib as L
    from yggdrax_b200 import build_ext, inputs

    world, rank, local = _dist()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if local == 0:  # one builder per node (normally a no-op: the library is prebuilt)
        build_ext.build()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    lib = L.lib()
    # The reference's count-pass sizing check rejects Plummer spheres of this
    # size (its outermost halo leaf is near to every leaf); the lists are
    # exact without its dense buffers, so run past that check.
    yb.set_reference_limits(False)
    yb.set_traversal_mode(args.mode)

    n = args.n
    pos_np, mass_np = inputs.plummer(n, 4)
    if args.roofline_only:
        P = torch.from_numpy(pos_np).to(dev)
        r = sort_roofline(yb.morton_encode(P, yb.infer_bounds(P)), dev, max(3, args.steps))
        if rank == 0:
            print(json.dumps({"roofline": r}), flush=True)
        return 0
    pos_h = torch.from_numpy(pos_np).pin_memory()
    mass_h = torch.from_numpy(mass_np).pin_memory()
    pos_d = pos_h.to(dev)
    mass_d = mass_h.to(dev)

    def step(P, M):
        tree, ps = yb.build_tree(P, M, leaf_size=LEAF, return_reordered=True)[:2]
        geom = yb.compute_tree_geometry(tree, ps)
        inter, nbrs = yb.build_interactions_and_neighbors(tree, geom, theta=THETA, mac_type=MAC)
        return tree, geom, inter, nbrs

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        out = step(pos_d, mass_d)
    del out
    barrier()

    # launch shapes chosen by the autotuner on this workload (sort knobs on
    # its Morton codes, the rest on the whole step); untimed
    tuning = None
    if not args.no_tune:
        from yggdrax_b200 import autotune

        tlog: list = []
        codes = yb.morton_encode(pos_d, yb.infer_bounds(pos_d))
        chosen = autotune.tune(lambda: step(pos_d, mass_d), dev, codes=codes, log=tlog)
        del codes
        tuning = {"chosen": chosen, "measured": len(tlog),
                  "step_ms_range": [min(r["ms"] for r in tlog if r["stage"] == "step"),
                                    max(r["ms"] for r in tlog if r["stage"] == "step")],
                  "sort_ms_range": [min(r["ms"] for r in tlog if r["stage"] == "sort"),
                                    max(r["ms"] for r in tlog if r["stage"] == "sort")]}
        barrier()

    # -- device-resident timing ------------------------------------------------
    launches0 = lib.ygx_launch_counter()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with ClockSampler(torch.cuda.current_device()) as clk:
        barrier()
        w0 = time.time()
        ev[0].record()
        out = None
        for _ in range(args.steps):
            out = None  # a step's outputs are released before the next allocates
            out = step(pos_d, mass_d)
        ev[1].record()
        barrier()
        clk.mark(w0, time.time())
    launches = lib.ygx_launch_counter() - launches0
    t_dev = ev[0].elapsed_time(ev[1]) / 1e3 / args.steps
    tree, geom, inter, nbrs = out
    far_entries = int(inter.sources.numel())
    near_entries = int(nbrs.neighbors.numel())
    total_nodes = int(tree.parent.shape[0])
    del tree, geom, inter, nbrs, out

    # -- end to end through the public API from host buffers --------------------
    # Every step copies its inputs from pinned host memory and reads its
    # per-node counts back, all inside the timed region.  Serial: copy, then
    # compute, on one stream.  Pipelined (the reported e2e): two device input
    # buffers; the next step's host->device copy runs on a copy stream while
    # the current step computes (a caller streaming snapshots through the API).
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d2h = 0
    e0.record()
    inter = nbrs = None
    for _ in range(args.steps):
        inter = nbrs = None
        P = pos_h.to(dev, non_blocking=True)
        M = mass_h.to(dev, non_blocking=True)
        _, _, inter, nbrs = step(P, M)
        fc = inter.counts.cpu()
        nc = nbrs.counts.cpu()
        d2h = fc.numel() * fc.element_size() + nc.numel() * nc.element_size()
    e1.record()
    barrier()
    t_e2e_serial = e0.elapsed_time(e1) / 1e3 / args.steps
    h2d = pos_h.numel() * 4 + mass_h.numel() * 4
    del inter, nbrs

    comp = torch.cuda.current_stream(dev)
    copy_s = torch.cuda.Stream(dev)
    bufs = [(torch.empty_like(pos_d), torch.empty_like(mass_d)) for _ in range(2)]
    ready = [torch.cuda.Event() for _ in range(2)]
    free = [torch.cuda.Event() for _ in range(2)]
    barrier()
    e0.record()

    def upload(k):
        with torch.cuda.stream(copy_s):
            copy_s.wait_event(free[k % 2])  # that buffer's previous step has finished
            bufs[k % 2][0].copy_(pos_h, non_blocking=True)
            bufs[k % 2][1].copy_(mass_h, non_blocking=True)
            ready[k % 2].record(copy_s)

    for k in range(2):
        free[k].record(comp)  # after e0: every copy is inside the timed region
    upload(0)
    inter = nbrs = None
    for k in range(args.steps):
        inter = nbrs = None
        comp.wait_event(ready[k % 2])
        if k + 1 < args.steps:
            upload(k + 1)
        _, _, inter, nbrs = step(*bufs[k % 2])
        free[k % 2].record(comp)
        fc = inter.counts.cpu()
        nc = nbrs.counts.cpu()
    e1.record()
    barrier()
    t_e2e = e0.elapsed_time(e1) / 1e3 / args.steps
    del inter, nbrs, bufs

    roofline = sort_roofline(yb.morton_encode(pos_d, yb.infer_bounds(pos_d)), dev,
                             max(3, args.steps))

    # -- the same step with the other traversal schedules (same exact lists) ----
    modes = {args.mode: {"ms_per_step": t_dev * 1e3, "value": n / t_dev}}
    if not args.no_modes:
        modes.update(mode_timings(step, pos_d, mass_d, n, args.steps, barrier, args.mode,
                                  pos_h, mass_h))
        # the main schedule's end-to-end figures (this rank), beside the others'
        modes[args.mode]["e2e_value"] = n / t_e2e
        modes[args.mode]["e2e_serial_value"] = n / t_e2e_serial

    batched = None
    if not args.no_batched:  # every rank (barriers inside), each on its share of the sets
        batched = batched_timing(dev, args.steps, barrier, world=world, rank=rank)

    extras = None
    if not args.no_extras and world == 1:
        try:
            extras = extras_timing(dev)
        except Exception as e:  # the main line stands without them
            extras = {"error": f"{type(e).__name__}: {e}"[:300]}
        torch.cuda.empty_cache()

    breakdown = None
    if args.breakdown:
        breakdown = stage_breakdown(pos_d, mass_d, dev)

    # -- aggregate over ranks ---------------------------------------------------
    t_max, te_max, te_serial_max = _max_over_ranks([t_dev, t_e2e, t_e2e_serial], dev)
    if rank == 0:
        cpu = None if args.no_cpu_baseline else cpu_baseline(n)
        line = {
            "metric": METRIC, "value": world * n / t_max, "unit": "particles/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+int64", "data": "synthetic",
            "config": workload_config(n, world, total_nodes, far_entries, near_entries),
            "pairs_per_s": world * (far_entries + near_entries) / t_max,
            "traversal_mode": args.mode, "autotune": tuning,
            "e2e": {"value": world * n / te_max, "unit": "particles/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "schedule": "next step's upload overlapped with this step's compute "
                                "(copy stream, two input buffers)",
                    "serial_value": world * n / te_serial_max},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "modes": modes,
            "batched": batched,
            "extras": extras,
        }
        if breakdown is not None:
            line["breakdown_ms"] = breakdown
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return 0


def mode_timings(step, pos_d, mass_d, n, steps, barrier, main_mode: str = "learned",
                 pos_h=None, mass_h=None) -> dict:
    """Device time of the step with every traversal schedule other than the
    main one: the pair log (one walk, scatter, row sort), the plain two-pass
    traversal (count walk + fill walk, the reference's schedule), the learned
    one-pass traversal (rows sized by the capacity predictor) and the
    per-target walks (rows without a scatter, then sorted; or in Morton order
    straight from the walk), inputs resident; the median over the steps.
    With the pinned host inputs, also each schedule's end-to-end rate through
    the public API, serial (copy in, compute, read the counts back, all in the
    timed region), as ``e2e_serial_value``."""
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200.interactions import LAST_WALK_STATS

    out = {}
    for mode in [m for m in ("log", "two_pass", "learned", "target", "target_ordered")
                 if m != main_mode]:
        yb.set_traversal_mode(mode)
        try:
            torch.cuda.empty_cache()  # start each schedule from the same allocator state
            for _ in range(2):  # capacity hints of this schedule
                step(pos_d, mass_d)
            barrier()
            per = []
            for _ in range(steps):  # median step: robust to one slow step
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                step(pos_d, mass_d)
                b.record()
                barrier()
                per.append(a.elapsed_time(b))
            ms = float(np.median(per))
            rec = {"ms_per_step": ms, "value": n / (ms / 1e3)}
            if pos_h is not None:
                dev = pos_d.device
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                barrier()
                a.record()
                for _ in range(steps):
                    P = pos_h.to(dev, non_blocking=True)
                    M = mass_h.to(dev, non_blocking=True)
                    _, _, inter, nbrs = step(P, M)
                    inter.counts.cpu()
                    nbrs.counts.cpu()
                    inter = nbrs = None
                b.record()
                barrier()
                rec["e2e_serial_value"] = n / (a.elapsed_time(b) / 1e3 / steps)
            if mode == "learned":
                rec["predictor"] = {k: LAST_WALK_STATS.get(k) for k in (
                    "over_allocation", "overflow_row_fraction", "overflow_entry_fraction",
                    "ovf_rows", "padded_far", "padded_near", "walk_runs")}
            if mode in ("target", "target_ordered"):
                rec["walk"] = {k: LAST_WALK_STATS.get(k) for k in (
                    "continuation_pieces", "pieces_run", "busy_fraction", "walk_runs", "steps",
                    "lane_fill")}
            out[mode] = rec
        finally:
            yb.set_traversal_mode(main_mode)
    return out


def batched_timing(dev, steps, barrier, sets: int = 4096, loop_sample: int = 64,
                   world: int = 1, rank: int = 0) -> dict:
    """Device time of the batched workload: 4096 independent point sets,
    sizes log-uniform in [256, 65536] (about 48M points), half uniform cube,
    half Plummer, unit masses, seed 3; radix leaf 16, dehnen theta 0.6.  One
    step = the batched build, geometry and exact lists of every set, one
    launch per stage.  With several ranks the sets are split into contiguous
    shares of about equal point counts (the sets are independent: no
    exchange) and the step time is the slowest rank's.  Beside it, the
    single-set API called set by set on ``loop_sample`` sets, scaled to all
    sets by point count."""
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import _lib as L
    from yggdrax_b200 import batch as B
    from yggdrax_b200 import inputs

    pos_all, mass_all, off_all = inputs.batched_sets(sets, 3)
    s0, s1 = B.shard_sets(off_all, rank, world)
    a, b = int(off_all[s0]), int(off_all[s1])
    pos, mass, off = pos_all[a:b], mass_all[a:b], off_all[s0:s1 + 1] - a
    sets = s1 - s0
    P = torch.from_numpy(pos).to(dev)
    M = torch.from_numpy(mass).to(dev)
    lib = L.lib()

    def step():
        bt = B.build_trees_batched(P, M, off, leaf_size=16)
        bg = B.compute_tree_geometry_batched(bt)
        bi = B.build_interactions_and_neighbors_batched(bt, bg, theta=THETA, mac_type=MAC)
        return bt, bi

    for _ in range(3):
        bt, bi = step()
    del bt, bi
    barrier()
    from yggdrax_b200 import autotune

    tlog: list = []
    chosen = autotune.tune(step, dev, log=tlog)
    barrier()
    l0 = lib.ygx_launch_counter()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        bt, bi = step()
    b.record()
    barrier()
    ms = a.elapsed_time(b) / steps
    launches = (lib.ygx_launch_counter() - l0) / steps
    far, near = int(bi.sources.numel()), int(bi.neighbors.numel())
    nodes = bt.total_nodes
    del bt, bi

    # the same step replayed from a captured CUDA graph (inputs copied into
    # the graph's buffers, one status read-back per step)
    pipe = B.BatchedPipeline(off, leaf_size=16, theta=THETA, mac_type=MAC, device=dev)
    pipe(P, M)  # ordinary path + capture
    for _ in range(2):
        pipe(P, M)
    barrier()
    a.record()
    replayed = True
    for _ in range(steps):
        pipe(P, M)
        replayed = replayed and pipe.last_replayed
    b.record()
    barrier()
    graph_ms = a.elapsed_time(b) / steps
    del pipe

    # the single-set API, set by set, on a sample of sets
    rng = np.random.default_rng(0)
    pick = np.sort(rng.choice(sets, size=min(loop_sample, sets), replace=False))
    views = [(P[off[i]:off[i + 1]], M[off[i]:off[i + 1]]) for i in pick]

    def loop():
        for p, m in views:
            t, ps = yb.build_tree(p, m, leaf_size=16, return_reordered=True)[:2]
            g = yb.compute_tree_geometry(t, ps)
            if int(t.num_internal_nodes) > 0:
                yb.build_interactions_and_neighbors(t, g, theta=THETA, mac_type=MAC)

    loop()
    barrier()
    a.record()
    loop()
    b.record()
    barrier()
    sample_pts = int(sum(off[i + 1] - off[i] for i in pick))
    loop_ms = a.elapsed_time(b) * float(off[-1]) / sample_pts
    # whole job: all ranks' sets over the slowest rank's step
    ms, graph_ms, loop_ms = _max_over_ranks([ms, graph_ms, loop_ms], dev)
    n = int(off_all[-1])
    return {"workload": "4096_sets_loguniform_256_65536_cube_plummer_radix_leaf16_dehnen_theta0.6",
            "n_sets": int(off_all.shape[0] - 1), "sets_per_rank": sets, "ranks": world,
            "n_particles": n, "total_nodes_rank0": nodes, "ms_per_step": ms,
            "value": n / (ms / 1e3), "unit": "particles/s", "far_entries": far,
            "near_entries": near, "pairs_per_s": (far + near) / (ms / 1e3),
            "gpu_launches_per_step": launches,
            "autotune": {"chosen": chosen, "measured": len(tlog)},
            "cuda_graph": {"ms_per_step": graph_ms, "value": n / (graph_ms / 1e3),
                           "all_steps_replayed": replayed},
            "single_set_loop": {"ms_estimate": loop_ms, "sample_sets": len(pick),
                                "sample_particles": sample_pts,
                                "speedup_of_batched": loop_ms / ms}}


def extras_timing(dev, n: int = 1 << 22, reps: int = 3) -> dict:
    """Device time (CUDA events, median of ``reps`` after one warm-up call) of
    the outputs beside the main lists, each on a 4,194,304-particle input:
    compact far pairs + leaf neighbour lists, the mutual canonical-pair walk,
    order-4 multipole moments and class-grouped far pairs on the Plummer
    radix tree (leaf 32, theta 0.6), and the native octree walk (far pairs,
    neighbour lists) on a fixed-depth octree of Plummer clumps.  A failing leg
    reports its error instead of a time."""
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    def timed(fn):
        fn()
        torch.cuda.synchronize(dev)
        ts = []
        out = None
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            out = fn()
            b.record()
            torch.cuda.synchronize(dev)
            ts.append(a.elapsed_time(b))
        return float(np.median(ts)), out

    res = {"n_particles": n}
    pos, mass = inputs.plummer(n, 1)
    P, M = torch.from_numpy(pos).to(dev), torch.from_numpy(mass).to(dev)
    tree, ps, ms = yb.build_tree(P, M, leaf_size=LEAF, return_reordered=True)[:3]
    geom = yb.compute_tree_geometry(tree, ps)
    total, ni = int(tree.parent.shape[0]), int(tree.left_child.shape[0])

    def leg(name, fn, count):
        try:
            ms_, out = timed(fn)
            c = count(out)
            res[name] = {"ms": ms_, "entries": c, "entries_per_s": c / (ms_ / 1e3)}
        except Exception as e:  # report, keep the bench line
            res[name] = {"error": f"{type(e).__name__}: {e}"[:300]}

    leg("compact_far_pairs_and_leaf_neighbors",
        lambda: yb.build_compact_far_pairs_and_leaf_neighbor_lists(
            tree, geom, theta=THETA, mac_type=MAC),
        lambda o: int(o[0].sources.numel()) + int(o[1].neighbors.numel()))
    lf = torch.full((total,), -1, dtype=torch.int64, device=dev)
    rt = lf.clone()
    lf[:ni] = tree.left_child.to(torch.int64)
    rt[:ni] = tree.right_child.to(torch.int64)
    leg("mutual_walk",
        lambda: yb.dual_tree_walk_mutual(lf, rt, geom.center, geom.radius, THETA, 0,
                                         max_pair_queue=1 << 26, far_cap=1 << 26,
                                         near_cap=1 << 26),
        lambda o: int(o.far_count) + int(o.near_count))
    leg("multipole_moments_order4",
        lambda: yb.compute_tree_multipole_moments(tree, ps, ms, max_order=4),
        lambda o: n)
    inter = yb.build_interactions_and_neighbors(tree, geom, theta=THETA, mac_type=MAC)[0]
    leg("grouped_far_pairs",
        lambda: yb.build_grouped_interactions(tree, geom, inter),
        lambda o: int(inter.sources.numel()))
    del tree, ps, ms, geom, inter, lf, rt, P, M
    pos, mass = inputs.plummer_clumps(n, 2)
    P, M = torch.from_numpy(pos).to(dev), torch.from_numpy(mass).to(dev)
    otree = yb.build_fixed_depth_octree(P, M, max_depth=6, return_reordered=True)[0]
    topo = otree.topology if hasattr(otree, "topology") else otree
    cfg = yb.DualTreeTraversalConfig(max_pair_queue=1 << 26, process_block=256,
                                     max_interactions_per_node=1 << 20,
                                     max_neighbors_per_leaf=1 << 20)
    leg("octree_native_far_pairs",
        lambda: yb.build_octree_native_far_pairs(topo, None, theta=THETA, mac_type=MAC,
                                                 traversal_config=cfg),
        lambda o: int(o.sources.numel()))
    leg("octree_native_neighbor_lists",
        lambda: yb.build_octree_native_neighbor_lists(topo, None, theta=THETA, mac_type=MAC,
                                                      traversal_config=cfg),
        lambda o: int(o.neighbors.numel()))
    return res


def stage_breakdown(pos_d, mass_d, dev):
    """Per-stage CUDA-event times of one step (diagnostics)."""
    import torch

    import yggdrax_b200 as yb

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    marks = {}
    from yggdrax_b200 import interactions as I

    I._TIMING = True
    torch.cuda.synchronize(dev)
    a, b, c, d = ev(), ev(), ev(), ev()
    a.record()
    tree, ps = yb.build_tree(pos_d, mass_d, leaf_size=LEAF, return_reordered=True)[:2]
    b.record()
    geom = yb.compute_tree_geometry(tree, ps)
    c.record()
    inter, nbrs = yb.build_interactions_and_neighbors(tree, geom, theta=THETA, mac_type=MAC)
    d.record()
    hist = {}
    for name, cnt in (("far", inter.counts), ("near", nbrs.counts)):
        c64 = cnt.to(torch.int64)
        edges = [0, 32, 256, 1024, 16384, 1 << 40]
        hist[name] = {f"<={edges[k + 1]}": [int(((c64 > edges[k]) & (c64 <= edges[k + 1])).sum()),
                                           int(c64[(c64 > edges[k]) & (c64 <= edges[k + 1])].sum())]
                      for k in range(len(edges) - 1)}
    marks["row_histogram_rows_entries"] = hist
    torch.cuda.synchronize(dev)
    marks["build"] = a.elapsed_time(b)
    marks["geometry"] = b.elapsed_time(c)
    marks["traversal"] = c.elapsed_time(d)
    a, b = ev(), ev()
    a.record()
    yb.encode_and_sort(pos_d)
    b.record()
    torch.cuda.synchronize(dev)
    marks["encode_sort"] = a.elapsed_time(b)
    from yggdrax_b200 import interactions as I

    marks["walk_stats"] = dict(I.LAST_WALK_STATS)
    return marks


if __name__ == "__main__":
    sys.exit(main())
