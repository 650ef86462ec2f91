#!/usr/bin/env python3
"""Benchmark of the block-sparse SDF field hot path: one JSON line on rank 0.

Default workload (the metric "leaf Gvox/s batched vs plain at <=1e-5 pitch err; EDT GB/s; serve
p50/p99 ms", synthetic and seeded): 256 independent recipes -- primitive counts log-uniform in
[8, 2048], cubic domains drawn from {64, 128, 256, 512}^3, leaf size 4^3 / 8^3 / 16^3 per recipe
from the autotuner -- built as one batch (culling, classification, compaction, per-block lists and
fused leaf evaluation with CSG, every phase one launch over all recipes, sizing on the device).
One step = one build of the whole batch, recipe tables resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]

value: leaf voxels built per second over the whole step (Gvox/s), all ranks.  The same line
carries the recipe-by-recipe figure of the same batch (the single-build path with its host read of
the active count) and their ratio, the float64-oracle accuracy of >= 1000 leaf blocks, the batch
with each recipe followed by occupancy + squared EDT, the exact EDT of a 512^3 obstacle grid (GB/s
on 13 B/voxel), and a short serving run (Poisson 1000 req/s: p50 / p99).  Each rank builds its own
replica (independent recipes, no exchange: weak scaling).  Timing: CUDA events on the launching
stream, a 256 MiB buffer written between steps outside the events, max over ranks.
`--impl reference` times the reference algorithm on the host cores instead: the CPU oracle port of
the reference's float64 classification and tile evaluation over a proportional random sample of
every recipe's blocks (each step), on the same metric.
`--workload plain` is the plain method at scale (one 1024^3 part of 3584 primitives minus 512
milling tools, plus the 512^3 EDT); serve / precision / tree / mesh are the other lines.
`--gpus N` without torchrun starts N ranks itself.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "leaf Gvox/s batched vs plain at ≤1e-5·pitch err; EDT GB/s; serve p50/p99 ms"
UNIT = "Gvox/s"
EDT_BYTES_PER_VOXEL = 13  # 1 B mask + 4 B output + 8 B int32 intermediate round trip
LAUNCHES_PER_STEP = 11    # prepare, full list, 2 x cull, classify, compact, list cull, leaf, 3 x EDT
WORKLOAD = "plain_at_scale_1024^3_3584prims_512tools_B8+edt_512^3_2000boxes"
BATCH_WORKLOAD = "batched_256_recipes_8-2048prims_64-512^3_autotuned_leaf"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", "--grid", dest="n", type=int, default=1024,
                    help="grid edge of the field build (--grid under torchrun, whose parser takes --n for its own)")
    ap.add_argument("--edt-n", type=int, default=512, help="grid edge of the EDT")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--check-bricks", type=int, default=24, help="precision: bricks checked per level")
    ap.add_argument("--workload", choices=("batched", "plain", "serve", "precision", "tree", "mesh", "clearance"), default="batched",
                    help="batched: 256 recipes built as one batch against recipe by recipe (default line); plain: "
                         "the plain method at scale; serve: the request loop; precision: float32 vs float64 at "
                         "mixed pitch; tree: packed adaptive block tree of a dense 512^3 field, built and sampled; "
                         "mesh: mesh -> signed distance field stage")
    ap.add_argument("--no-serve", action="store_true", help="batched: leave out the short serving run")
    ap.add_argument("--quick", action="store_true",
                    help="batched: the timed builds only (no plain path, EDT form, accuracy, extras) -- for profiling")
    ap.add_argument("--cpu-fraction", type=float, default=0.0005,
                    help="share of every recipe's blocks in one CPU-baseline / reference-arm sample")
    ap.add_argument("--recipes", type=int, default=256)
    ap.add_argument("--streams", type=int, default=16, help="batched: side streams of the per-recipe EDTs")
    ap.add_argument("--rate", type=float, default=1000.0, help="serve: Poisson arrival rate, req/s")
    ap.add_argument("--seconds", type=float, default=5.0, help="serve: arrival window")
    ap.add_argument("--arena-gb", type=float, default=150.0, help="serve: device arena for resident fields and request temporaries (0: none)")
    ap.add_argument("--slots", type=int, default=16, help="serve: concurrent request slots (one stream each)")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML (read-only queries) every `period_s`
    while the timed region runs.  The device is found by the UUID torch reports for `cuda_index`,
    so CUDA_VISIBLE_DEVICES remapping cannot pick the wrong board."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("hw_power_brake_slowdown", 0x80), ("sw_power_cap", 0x4))

    def __init__(self, cuda_index, period_s=0.004):
        self.cuda_index = cuda_index
        self.period = period_s
        self.samples = []
        self.error = None
        self.thread = None
        self.stop_flag = threading.Event()

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
        uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid)

    def start(self):
        try:
            self.nvml, self.h = self._handle()
            self.max_mhz = self.nvml.nvmlDeviceGetMaxClockInfo(self.h, self.nvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: the line says so
            self.error = f"nvml unavailable: {e!r}"[:120]
            return
        # the timing loop holds the interpreter lock between its launches; a short switch interval lets
        # the sampler run every few milliseconds (device timing is by CUDA events, unaffected)
        self.switch = sys.getswitchinterval()
        sys.setswitchinterval(0.0005)
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        n = self.nvml
        while not self.stop_flag.is_set():
            try:
                self.samples.append((n.nvmlDeviceGetClockInfo(self.h, n.NVML_CLOCK_SM),
                                     n.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
            except Exception as e:
                self.error = f"nvml query failed: {e!r}"[:120]
                return
            self.stop_flag.wait(self.period)

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error or "not sampled"], "samples": 0}
        self.stop_flag.set()
        self.thread.join(timeout=5)
        sys.setswitchinterval(self.switch)
        sm = [c for c, _ in self.samples]
        reasons = sorted({name for _, mask in self.samples for name, bit in self.REASONS if mask & bit})
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
               "reasons": reasons, "samples": len(sm), "source": "nvml"}
        if self.error:
            out["error"] = self.error
        return out


# ------------------------------------------------------------------------------------------ ranks
def max_over_ranks(x, world, device="cpu"):
    """The largest value of `x` over all ranks (the job's time is its slowest rank's)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, steps, total_ms):
    """Whole-job throughput in G units/s: every rank processes `units_per_rank` per step (replicas,
    weak scaling) and the job takes the slowest rank's `total_ms` for `steps` steps."""
    return units_per_rank * world * steps / (total_ms * 1e-3) / 1e9


# ------------------------------------------------------------------------------------------ workload
def workload(n, edt_n):
    import field_b200.recipes as R
    import field_b200.expr as X
    recipe, meta = R.milled_part(seed=1, n=n, block=8)
    comp = X.compile_recipe(recipe)
    mask = R.obstacle_grid(seed=2, n=edt_n, n_boxes=2000, fill=0.08)
    return comp, meta, mask


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_of(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    f = REPO / "profiles" / "ncu_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel and not line.startswith("#"):
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------------------------------------ ours
def run_plain(args, rank, world, local_rank):
    """The plain method at scale: one 1024^3 part (3584 primitives minus 512 milling tools, 8^3
    leaves) and the 512^3 EDT per step."""
    import torch
    import torch.distributed as dist
    import field_b200.build as B
    import field_b200.edt as E
    import field_b200._lib as L
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    comp, meta, mask_np = workload(args.n, args.edt_n)
    builder = B.FieldBuilder(comp, meta, device=dev)
    stream = torch.cuda.current_stream()
    # sizing run: exact active count, then a fixed tile buffer
    df = builder.build()
    n_active = int(df.n_active)
    del df
    b3 = meta.block ** 3
    tiles = torch.empty((max(n_active, 1), b3), dtype=torch.float32, device=dev)
    mask = torch.from_numpy(mask_np).to(dev)
    edt_out = torch.empty(mask.shape, dtype=torch.int32, device=dev)
    edt_scratch = torch.empty(int(L.lib().fb_edt_scratch_bytes(*mask.shape, 0)), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    edt_voxels = int(np.prod(mask.shape))

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        builder.classify(stream)
        if ev:
            ev[1].record(stream)
        builder.leaf(tiles, n_active, stream=stream)
        if ev:
            ev[2].record(stream)
        E.squared_distance_device(mask, sites_nonzero=True, out=edt_out, scratch=edt_scratch, stream=stream)
        if ev:
            ev[3].record(stream)

    for _ in range(max(args.warmup, 3)):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    assert int(builder.count.item()) == n_active, "active count changed between builds"
    assert builder.compact_error() == 0

    clocks = ClockSampler(local_rank)
    clocks.start()
    events = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        step(events[k])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    t_cls = [e[0].elapsed_time(e[1]) for e in events]
    t_leaf = [e[1].elapsed_time(e[2]) for e in events]
    t_edt = [e[2].elapsed_time(e[3]) for e in events]
    t_step = [e[0].elapsed_time(e[3]) for e in events]
    total_ms = max_over_ranks(float(sum(t_step)), world, dev)
    leaf_voxels = n_active * b3
    value = job_rate(leaf_voxels, world, args.steps, total_ms)

    # executed work of the leaf kernel and the float32 peak (untimed)
    work = torch.zeros(2, dtype=torch.int64, device=dev)
    builder.classify(stream)
    L.lib().fb_field_leaf_work_device(*builder._args(), builder.kind.data_ptr(), builder.active.data_ptr(),
                                      builder.count.data_ptr(),
                                      tiles.data_ptr(), n_active, builder.scratch.data_ptr(), builder.scratch.numel(),
                                      work.data_ptr(), L.stream_handle(stream))
    torch.cuda.synchronize()
    evals, flops = (int(x) for x in work.cpu().numpy())
    probe = torch.empty(L.lib().fb_sm_count_c() * 8, dtype=torch.float32, device=dev)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nflop = L.lib().fb_fp32_peak_launch(probe.data_ptr(), probe.numel(), 4096, L.stream_handle(stream))
        e1.record(stream)
        torch.cuda.synchronize()
        best = max(best, nflop / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    fp32_peak = best
    hbm_peak, hbm_src = measured_peaks()

    med = lambda xs: float(statistics.median(xs))
    leaf_ms, edt_ms, cls_ms = med(t_leaf), med(t_edt), med(t_cls)
    leaf_tflops = flops / (leaf_ms * 1e-3) / 1e12
    leaf_gbs = leaf_voxels * 4 / (leaf_ms * 1e-3) / 1e9
    edt_gbs = edt_voxels * EDT_BYTES_PER_VOXEL / (edt_ms * 1e-3) / 1e9
    shares = {"classify": cls_ms, "leaf": leaf_ms, "edt": edt_ms}
    dominant = max(shares, key=shares.get)
    if dominant == "edt":
        roof = {"kernel": "edt (k_edt_bits + k_edt_zy + k_edt_x)", "bound": "hbm", "achieved": edt_gbs,
                "peak": hbm_peak, "unit": "GB/s", "frac": edt_gbs / hbm_peak,
                "traffic": traffic_of("edt"), "basis": f"{EDT_BYTES_PER_VOXEL} B/voxel"}
    else:
        fp32_frac = leaf_tflops / fp32_peak
        hbm_frac = leaf_gbs / hbm_peak
        if fp32_frac >= hbm_frac:
            roof = {"kernel": "k_leaf<8>", "bound": "fp32", "achieved": leaf_tflops, "peak": fp32_peak,
                    "unit": "TFLOP/s", "frac": fp32_frac, "traffic": traffic_of("k_leaf"),
                    "basis": "executed float32 ops of the culled primitive evaluations (FMA = 2); peak = FFMA probe"}
        else:
            roof = {"kernel": "k_leaf<8>", "bound": "hbm", "achieved": leaf_gbs, "peak": hbm_peak, "unit": "GB/s",
                    "frac": hbm_frac, "traffic": traffic_of("k_leaf"), "basis": "4 B tile store per leaf voxel"}
    roof["peak_source"] = hbm_src if roof["bound"] == "hbm" else "measured in this run (FFMA probe)"

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 guard band); int32 EDT", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": [meta.nx, meta.ny, meta.nz], "block": meta.block,
                   "primitives": int(len(comp.prims)), "chain": int(len(comp.chain)), "n_blocks": int(meta.n_blocks),
                   "n_active": n_active, "leaf_voxels": leaf_voxels, "edt_grid": list(mask.shape),
                   "edt_fill": float(mask_np.mean()), "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between steps, outside the per-step events"},
        "phases_ms_median": {"classify": cls_ms, "leaf": leaf_ms, "edt": edt_ms},
        "leaf": {"gvox_s": leaf_voxels / (leaf_ms * 1e-3) / 1e9, "tflops_executed": leaf_tflops,
                 "evals_per_voxel": evals / max(leaf_voxels, 1), "fp32_peak_tflops": fp32_peak,
                 "gbs_tile_store": leaf_gbs},
        "edt": {"gbs": edt_gbs, "ms": edt_ms, "frac_hbm": edt_gbs / hbm_peak, "voxels": edt_voxels},
        "roofline": roof,
        "clocks": clk,
        "gpu_launches": LAUNCHES_PER_STEP * args.steps,
    }

    if rank == 0 and not args.no_e2e:
        result["e2e"] = e2e_leg(comp, meta, mask_np, dev)
    if rank == 0 and world == 1 and not args.no_cpu:
        secs, leaf, ncls, ntile, cores = cpu_batch_sample([(comp, meta)], args.cpu_fraction * 4)
        result["cpu_baseline"] = {"value": leaf / secs / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
                                  "seconds": secs,
                                  "sample": f"{args.cpu_fraction * 4:g} of the part's blocks ({ncls}) classified in "
                                            f"float64, the {ntile} active ones among them evaluated with every "
                                            f"primitive; leaf voxels per second of that sample (field build only)"}
        # the float64 oracle, as the checker, on a sample of the timed run's leaf tiles
        result["accuracy"] = leaf_accuracy(comp, meta, builder, tiles, n_active, n_blocks=1000)
    return result


def leaf_accuracy(comp, meta, builder, tiles, n_active, n_blocks=48, seed=5):
    """Max |d_f32 - d_f64| / pitch over a seeded sample of active blocks (all their voxels, and
    inside the 3-voxel band), and sign disagreements, against the float64 oracle."""
    import oracle
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(n_active, size=min(n_blocks, n_active), replace=False))
    ids = builder.active[:n_active].cpu().numpy()[pick].astype(np.int32)
    got = tiles[pick].cpu().numpy().astype(np.float64).reshape(len(pick), -1)
    want = oracle.tiles_program(comp.prims, comp.program, meta, ids).reshape(len(pick), -1)
    err = np.abs(got - want) / meta.pitch
    band = np.abs(want) <= 3 * meta.pitch
    return {"blocks": int(len(pick)), "voxels": int(got.size), "max_err_pitch": float(err.max()),
            "max_err_pitch_band": float(err[band].max()) if band.any() else 0.0,
            "sign_disagreements": int(np.count_nonzero((got >= 0) != (want >= 0))), "checker": "float64 oracle"}


def e2e_leg(comp, meta, mask_np, dev, steps=3):
    """The same step through the public API with host buffers, as a caller that keeps its objects:
    a FieldBuilder made once for the recipe (FieldBuilder.build -> DeviceField.to_host, page-locked
    host arrays), and the squared EDT of a page-locked host mask (edt.squared_distance_device on a
    device copy, the result read back into a page-locked array).  Every step copies the mask to the
    device and both results to the host inside the timed region; the EDT runs on a second stream,
    so its transfers overlap the field build and the field's read-back."""
    import torch
    import field_b200.build as B
    import field_b200.edt as E
    import field_b200._lib as L
    builder = B.FieldBuilder(comp, meta, device=dev)
    binary = np.ascontiguousarray(~mask_np.astype(bool)).view(np.uint8)  # zero sites = the obstacles
    host_mask = torch.from_numpy(binary).pin_memory()
    host_sq = torch.empty(binary.shape, dtype=torch.int32, pin_memory=True)
    d_mask = torch.empty(binary.shape, dtype=torch.uint8, device=dev)
    d_sq = torch.empty(binary.shape, dtype=torch.int32, device=dev)
    scratch = torch.empty(int(L.lib().fb_edt_scratch_bytes(*binary.shape, 0)), dtype=torch.uint8, device=dev)
    edt_stream = torch.cuda.Stream(device=dev)
    times = []
    leaf = h2d = d2h = 0
    for _ in range(steps + 2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(edt_stream):
            d_mask.copy_(host_mask, non_blocking=True)
            E.squared_distance_device(d_mask, out=d_sq, scratch=scratch, stream=edt_stream)
            host_sq.copy_(d_sq, non_blocking=True)
        sf = builder.build().to_host()
        edt_stream.synchronize()
        t = time.perf_counter() - t0
        times.append(t)
        leaf = sf.tiles.size
        h2d = host_mask.numel()
        d2h = (sf.kind.nbytes + sf.corner_min_abs.nbytes + sf.active_ids.nbytes + sf.tiles.nbytes + 4
               + host_sq.numel() * 4)
        del sf  # the caller is done with this step's arrays: their page-locked blocks go back to the cache
    times = times[2:]
    # the device->host link alone: the same byte count in one page-locked copy (the bound of this leg)
    probe_d = torch.empty(int(d2h) // 4, dtype=torch.int32, device=dev)
    probe_h = torch.empty(probe_d.shape, dtype=torch.int32, pin_memory=True)
    link = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        probe_h.copy_(probe_d, non_blocking=True)
        torch.cuda.synchronize()
        link.append(time.perf_counter() - t0)
    d2h_gbs = probe_d.numel() * 4 / min(link) / 1e9
    del probe_d, probe_h
    med = statistics.median(times)
    return {"value": leaf / med / 1e9, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "seconds_per_step": med,
            "d2h_link_gbs": d2h_gbs, "link_bound_value": leaf / (d2h / (d2h_gbs * 1e9)) / 1e9,
            "api": "field_b200.build.FieldBuilder.build + DeviceField.to_host; field_b200.edt.squared_distance_device "
                   "with page-locked host mask and result (EDT on a second stream)"}


# ------------------------------------------------------------------------------------------ reference arm
def run_reference(args, rank, world):
    """The reference algorithm on the host cores only (no GPU code on this path), on the same
    workload, metric and unit as our arm: every step is a proportional random sample of the
    workload's blocks (--cpu-fraction of each recipe's blocks classified in float64, the active ones
    among them evaluated at every voxel, OpenMP on every host thread), its rate the leaf voxels that
    step produced over that step's measured time.  Under torchrun rank 0 alone runs."""
    if rank != 0:
        return None
    import field_b200.batch as BT
    W = max(args.warmup, 3)
    if args.workload == "batched":
        comps = batch_workload(args.recipes)
        blocks = reference_leaf_sizes(comps)
        recipes = [(c, BT.cube_meta(n, b)) for (c, n), b in zip(comps, blocks)]
        config = {"workload": BATCH_WORKLOAD, "recipes": len(recipes),
                  "leaf_sizes": {str(b): blocks.count(b) for b in (4, 8, 16)},
                  "n_blocks": int(sum(m.n_blocks for _, m in recipes))}
    else:
        comp, meta, _ = workload(args.n, args.edt_n)
        recipes = [(comp, meta)]
        config = {"workload": WORKLOAD + " (field build)", "grid": [meta.nx, meta.ny, meta.nz], "block": meta.block,
                  "n_blocks": int(meta.n_blocks)}
    rates, secs = [], []
    leaf = ncls = ntile = cores = 0
    for i in range(W + args.steps):
        sec, leaf, ncls, ntile, cores = cpu_batch_sample(recipes, args.cpu_fraction, seed=i)
        if i >= W:
            rates.append(leaf / sec / 1e9)
            secs.append(sec)
    value = float(statistics.median(rates))
    desc = (f"each step {args.cpu_fraction:g} of every recipe's blocks ({ncls} blocks) classified in float64 and "
            f"the active ones among them ({ntile}) evaluated at every voxel with every primitive (the reference's "
            f"per-block work), rate = leaf voxels produced / measured step time")
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": W, "ms_per_step": float(statistics.median(secs)) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 evaluator", "data": "synthetic", "config": config,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


TUNING = REPO / "3fold-field-engine_b200" / "tuning" / "leaf_sizes_b200.json"


def reference_leaf_sizes(comps):
    """Leaf size per recipe from the autotuner's table measured on B200 (the same choice our arm
    makes), without measuring: buckets missing from the table take 8."""
    import field_b200.batch as BT
    table = json.loads(TUNING.read_text()) if TUNING.exists() else {}
    return [int(table.get(BT.Autotuner.bucket(n, len(c.prims)), {}).get("block", 8)) for c, n in comps]


# ------------------------------------------------------------------------------------------ batched (default)
def batch_workload(count):
    """The batched workload's compiled recipes and grid edges (seeded)."""
    import field_b200.expr as X
    import field_b200.recipes as R
    return [(X.compile_recipe(r), n) for r, n, _ in R.batch_recipes(count=count, seed=3)]


def cpu_batch_sample(recipes, fraction, seed=0):
    """The reference algorithm on the host cores over a proportional random sample of the batch:
    for every recipe, float64 8-corner classification of `fraction` of its blocks (at least one)
    and float64 leaf evaluation of the active ones among them (every primitive at every point, as
    the reference's kernels do), OpenMP.  Returns (seconds, leaf voxels produced, blocks classified,
    blocks evaluated, threads)."""
    import oracle
    rng = np.random.default_rng(seed)
    secs = 0.0
    leaf = classified = tiled = 0
    for comp, meta in recipes:
        k = max(1, int(round(fraction * meta.n_blocks)))
        blocks = np.sort(rng.choice(meta.n_blocks, size=min(k, meta.n_blocks), replace=False)).astype(np.int64)
        t0 = time.perf_counter()
        kinds, _ = oracle.classify_blocks(comp.prims, comp.program, meta, blocks)
        act = blocks[kinds == 0].astype(np.int32)
        if len(act):
            oracle.tiles_program(comp.prims, comp.program, meta, act)
        secs += time.perf_counter() - t0
        leaf += len(act) * meta.block ** 3
        classified += len(blocks)
        tiled += len(act)
    return secs, leaf, classified, tiled, oracle.threads()


def batch_accuracy(bb, recipes, n_recipes=40, per=25, seed=8):
    """Max |d_f32 - d_f64| / pitch and sign disagreements over `per` seeded active blocks of each of
    `n_recipes` seeded recipes of a built batch (all their voxels, and within 3 pitches of the
    surface), against the float64 oracle."""
    import oracle
    rng = np.random.default_rng(seed)
    off, cnt = bb.tile_offsets(), bb.leaf_counts()
    cand = [i for i in range(len(bb)) if cnt[i] > 0]
    worst = worst_band = 0.0
    sign = nblk = nvox = 0
    by_grid = {}
    for i in sorted(rng.choice(cand, size=min(n_recipes, len(cand)), replace=False)):
        comp, meta = recipes[int(i)]
        f = bb.field(int(i), off, cnt)
        pick = np.sort(rng.choice(f.n_active, size=min(per, f.n_active), replace=False))
        ids = f.active[:f.n_active].cpu().numpy()[pick].astype(np.int32)
        got = f.tiles[torch_index(pick, f.tiles.device)].cpu().numpy().astype(np.float64).reshape(len(pick), -1)
        want = oracle.tiles_program(comp.prims, comp.program, meta, ids).reshape(len(pick), -1)
        err = np.abs(got - want) / meta.pitch
        band = np.abs(want) <= 3 * meta.pitch
        worst = max(worst, float(err.max()))
        e_band = float(err[band].max()) if band.any() else 0.0
        worst_band = max(worst_band, e_band)
        sign += int(np.count_nonzero((got >= 0) != (want >= 0)))
        nblk += len(pick)
        nvox += got.size
        key = f"{meta.nx}/B{meta.block}"
        by_grid[key] = max(by_grid.get(key, 0.0), float(err.max()))
    return {"recipes": min(n_recipes, len(cand)), "blocks": nblk, "voxels": nvox,
            "max_err_pitch": worst, "max_err_pitch_band": worst_band, "max_err_pitch_by_grid": by_grid,
            "sign_disagreements": sign, "checker": "float64 oracle"}


def torch_index(idx, device):
    import torch
    return torch.from_numpy(np.asarray(idx, np.int64)).to(device)


def edt_extra(steps, flush, dev, check=True):
    """The exact int32 squared EDT of the 512^3 obstacle grid (2000 boxes, ~8 % fill), distances to
    the obstacles: CUDA-event time per transform, GB/s on the 13 B/voxel basis, and the result
    compared with the oracle's bit for bit."""
    import torch
    import field_b200._lib as L
    import field_b200.edt as E
    import field_b200.recipes as R
    mask_np = R.obstacle_grid(seed=2, n=512, n_boxes=2000, fill=0.08)
    mask = torch.from_numpy(mask_np).to(dev)
    out = torch.empty(mask.shape, dtype=torch.int32, device=dev)
    scratch = torch.empty(int(L.lib().fb_edt_scratch_bytes(*mask.shape, 0)), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    ts = []
    for k in range(3 + steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        E.squared_distance_device(mask, sites_nonzero=True, out=out, scratch=scratch, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if k >= 3:
            ts.append(e0.elapsed_time(e1))
    ms = float(statistics.median(ts))
    voxels = int(mask.numel())
    gbs = voxels * EDT_BYTES_PER_VOXEL / (ms * 1e-3) / 1e9
    peak, src = measured_peaks()
    res = {"grid": list(mask.shape), "fill": float(mask_np.mean()), "ms": ms, "gbs": gbs, "frac_hbm": gbs / peak,
           "peak_source": src, "basis": f"{EDT_BYTES_PER_VOXEL} B/voxel (1 B mask, 4 B out, 8 B intermediate)"}
    if check:
        import oracle
        res["bit_exact_vs_oracle"] = bool((out.cpu().numpy() == oracle.edt_squared(1 - mask_np)).all())
    return res


def run_headline(args, rank, world, local_rank):
    """The batched workload: build timing (value), the recipe-by-recipe figure, the EDT form, the
    accuracy, the 512^3 EDT, a short serving run, roofline, CPU baseline and end to end."""
    import torch
    import torch.distributed as dist
    import field_b200.batch as BT
    import field_b200._lib as L
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    t0 = time.perf_counter()
    comps = batch_workload(args.recipes)
    t_compile = time.perf_counter() - t0
    t0 = time.perf_counter()
    tuner = BT.Autotuner(TUNING, device=dev)
    known = len(tuner.table)
    blocks = tuner.tune(comps)
    t_tune = time.perf_counter() - t0
    recipes = [(c, BT.cube_meta(n, b)) for (c, n), b in zip(comps, blocks)]
    # a fresh batch: set-up (tables, scratch, work-lists), its first build into the default arena
    # (grown once if the device reports it too small), graph capture
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bb = BT.BatchBuilder(recipes, device=dev, edt=not args.quick, streams=args.streams)
    bb.enqueue(edt=False)
    grew = bb.ensure_capacity(edt=False)
    torch.cuda.synchronize()
    t_first = time.perf_counter() - t0
    schedule = bb.tune_schedule()
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    W = max(args.warmup, 3)
    warm = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    for _ in range(W):
        flush.zero_()
        bb.enqueue_timed(warm)
    torch.cuda.synchronize()
    if bb.status() != 0:
        raise RuntimeError("batched build failed")
    events = [[torch.cuda.Event(enable_timing=True) for _ in range(6)] for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        bb.enqueue_timed(events[k])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    if bb.status() != 0:
        raise RuntimeError("batched build failed")
    step_ms = [e[0].elapsed_time(e[5]) for e in events]
    # events: start, culling, classification (with the active blocks' lists), compaction, (empty), leaves
    names = {"cull": 0, "classify": 1, "compact": 2, "leaf": 4}
    phases = {nm: float(statistics.median(e[i].elapsed_time(e[i + 1]) for e in events)) for nm, i in names.items()}
    total_ms = max_over_ranks(float(sum(step_ms)), world, dev)
    counts = bb.active_counts()
    leaf_voxels = bb.leaf_voxels
    value = job_rate(leaf_voxels, world, args.steps, total_ms)
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": W,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 guard band)", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "recipes": len(recipes),
                   "grid_sizes": {str(n): sum(1 for _, m in recipes if m.nx == n) for n in (64, 128, 256, 512)},
                   "leaf_sizes": {str(b): blocks.count(b) for b in (4, 8, 16)},
                   "primitives": int(sum(len(c.prims) for c, _ in comps)), "n_blocks": int(sum(m.n_blocks for _, m in recipes)),
                   "n_active": int(counts.sum()), "leaf_voxels": leaf_voxels, "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between steps, outside the per-step events"},
        "phases_ms_median": phases,
        "batch": {"launches_per_step": bb.launches - (5 + 3 * len(bb) if bb.has_edt else 0),
                  "schedule_ctas_per_sm": bb.ctas_per_sm,
                  "schedule_ms": schedule, "arena_grown": bool(grew), "compile_s": t_compile, "autotune_s": t_tune,
                  "autotune_buckets": {"from_table": known, "measured_now": len(tuner.table) - known,
                                       "table": tuner.table},
                  "fresh_batch_first_build_s": t_first},
        "clocks": clk,
        "gpu_launches": (bb.launches - (5 + 3 * len(bb) if bb.has_edt else 0)) * args.steps,
    }
    if args.quick:
        bb.close()
        return result
    # the same build from one CUDA graph (captured once)
    t0 = time.perf_counter()
    bb.capture(edt=False)
    result["batch"]["capture_s"] = time.perf_counter() - t0
    result["batch"]["graph_replay_ms"] = float(statistics.median(timed_device(lambda: bb.replay(edt=False), args.steps, flush)))
    # recipe by recipe through the single-build path (host read of the count between launches)
    buf = BT.PlainBuffers(bb.builders, counts)
    plain = lambda: BT.plain_build(buf)
    timed_device(plain, W, flush)
    plain_ms = max_over_ranks(float(statistics.median(timed_device(plain, args.steps, flush))), world, dev)
    batched_ms = total_ms / args.steps
    result["plain"] = {"gvox_s": leaf_voxels / (plain_ms * 1e-3) / 1e9, "ms_per_step": plain_ms,
                       "path": "FieldBuilder.classify + host count read + FieldBuilder.leaf, recipe by recipe"}
    result["speedup_batched_vs_plain"] = plain_ms / batched_ms
    # executed work of the leaf pass and the float32 peak (untimed)
    work = torch.zeros(2, dtype=torch.int64, device=dev)
    bb.enqueue_timed(warm, work=work)
    torch.cuda.synchronize()
    evals, flops = (int(x) for x in work.cpu().numpy())
    fp32_peak = fp32_probe(dev)
    hbm_peak, hbm_src = measured_peaks()
    leaf_tflops = flops / (phases["leaf"] * 1e-3) / 1e12
    dominant = max(phases, key=phases.get)
    result["roofline"] = {"kernel": "k_b_leaf<B> (leaf phase)", "bound": "fp32", "achieved": leaf_tflops,
                          "peak": fp32_peak, "unit": "TFLOP/s", "frac": leaf_tflops / fp32_peak,
                          "traffic": traffic_of("k_b_leaf"), "dominant_phase": dominant,
                          "basis": "executed float32 ops of the culled primitive evaluations (FMA = 2) per leaf phase; "
                                   "peak = FFMA probe measured in this run",
                          "leaf_evals_per_voxel": evals / max(leaf_voxels, 1),
                          "leaf_gbs_tile_store": leaf_voxels * 4 / (phases["leaf"] * 1e-3) / 1e9, "hbm_peak": hbm_peak,
                          "hbm_peak_source": hbm_src}
    # each recipe followed by occupancy rasterisation + squared EDT of it, both forms
    buf.slot, buf.mask, buf.edt = bb.slots, bb.masks, bb.edts
    plain_edt = lambda: BT.plain_build(buf, bb.edt_scratch[0])
    timed_device(plain_edt, 2, flush)
    pe = float(statistics.median(timed_device(plain_edt, max(3, args.steps // 2), flush)))
    bb.capture(edt=True)
    timed_device(lambda: bb.replay(edt=True), 2, flush)
    be = float(statistics.median(timed_device(lambda: bb.replay(edt=True), max(3, args.steps // 2), flush)))
    edt_vox = int(sum(m.nx * m.ny * m.nz for _, m in recipes))
    result["with_edt"] = {"ms_plain": pe, "ms_batched": be, "plain_gvox_s": leaf_voxels / (pe * 1e-3) / 1e9,
                          "batched_gvox_s": leaf_voxels / (be * 1e-3) / 1e9, "speedup_batched_vs_plain": pe / be,
                          "edt_voxels": edt_vox, "edt_gbs_batched": edt_vox * EDT_BYTES_PER_VOXEL / (be * 1e-3) / 1e9,
                          "note": "each build followed by occupancy rasterisation + squared EDT of the occupancy"}
    if rank == 0 and not args.no_cpu:
        result["accuracy"] = batch_accuracy(bb, recipes)
    if rank == 0 and not args.no_e2e:
        result["e2e"] = e2e_batched(bb, args.steps)
    bb.graphs = {}
    del buf, plain, plain_edt
    result["edt"] = edt_extra(args.steps, flush, dev, check=(rank == 0 and not args.no_cpu))
    if rank == 0 and world == 1 and not args.no_cpu:
        secs, leaf, ncls, ntile, cores = cpu_batch_sample(recipes, args.cpu_fraction)
        result["cpu_baseline"] = {"value": leaf / secs / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
                                  "seconds": secs,
                                  "sample": f"{args.cpu_fraction:g} of every recipe's blocks ({ncls} blocks) classified "
                                            f"in float64, the {ntile} active ones among them evaluated (every "
                                            f"primitive at every voxel); leaf voxels per second of that sample"}
    bb.close()
    del bb
    gc.collect()
    torch.cuda.empty_cache()
    if rank == 0 and not args.no_serve:
        sv = run_serve(args, rate=1000.0, seconds=3.0, arena_gb=min(getattr(args, "arena_gb", 150.0), 100.0))
        result["serve"] = {k: sv[k] for k in ("rate_req_s", "seconds", "warmup", "requests", "throughput_req_s",
                                               "p50_ms", "p99_ms", "errors", "worst_ms_per_half_second", "by_kind",
                                               "slots")}
    return result


def timed_device(fn, reps, flush):
    """CUDA-event times (ms) of `reps` calls of fn on the current stream, the L2 flushed before each."""
    import torch
    out = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def fp32_probe(dev):
    """float32 FMA throughput of this GPU (TFLOP/s), best of five probe launches."""
    import torch
    import field_b200._lib as L
    stream = torch.cuda.current_stream()
    probe = torch.empty(L.lib().fb_sm_count_c() * 8, dtype=torch.float32, device=dev)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nflop = L.lib().fb_fp32_peak_launch(probe.data_ptr(), probe.numel(), 4096, L.stream_handle(stream))
        e1.record(stream)
        torch.cuda.synchronize()
        best = max(best, nflop / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def e2e_batched(bb, steps):
    """The batched build through the public API with host buffers: every step uploads all recipe
    tables from pinned host memory (one copy), builds, reads each recipe's tile count and offset,
    and copies the tiles, the block kinds and the active ids into pinned host memory."""
    import torch
    off, cnt = bb.tile_offsets(), bb.leaf_counts()
    used = int((cnt.astype(np.int64) * bb.b3).sum())
    host_tiles = torch.empty(used, dtype=torch.float32).pin_memory()
    host_kind = [torch.empty(fb.kind.numel(), dtype=torch.int32).pin_memory() for fb in bb.builders]
    host_act = [torch.empty(fb.active.numel(), dtype=torch.int32).pin_memory() for fb in bb.builders]
    times = []
    d2h = 0
    for _ in range(max(2, min(steps, 4)) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bb.upload_tables()
        bb.enqueue(edt=False)
        off, cnt = bb.tile_offsets(), bb.leaf_counts()   # host reads (synchronise)
        n = int((cnt.astype(np.int64) * bb.b3).sum())
        host_tiles[:n].copy_(bb.tiles[:n], non_blocking=True)
        d2h = n * 4 + 8 * len(bb) + 4 * len(bb)
        for i, fb in enumerate(bb.builders):
            host_kind[i].copy_(fb.kind, non_blocking=True)
            host_act[i][:int(cnt[i])].copy_(fb.active[:int(cnt[i])], non_blocking=True)
            d2h += fb.kind.numel() * 4 + int(cnt[i]) * 4
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    times = times[1:]
    sec = float(statistics.median(times))
    voxels = sum(int(c) * int(b) for c, b in zip(cnt, bb.b3))
    # the device->host link alone on the tile bytes (one page-locked copy): the bound of this leg
    link = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        host_tiles[:n].copy_(bb.tiles[:n], non_blocking=True)
        torch.cuda.synchronize()
        link.append(time.perf_counter() - t0)
    d2h_gbs = n * 4 / min(link) / 1e9
    return {"value": n and voxels / sec / 1e9, "unit": UNIT,
            "h2d_bytes_per_step": bb.table_bytes, "d2h_bytes_per_step": int(d2h), "seconds_per_step": sec,
            "d2h_link_gbs": d2h_gbs, "link_bound_value": voxels / (d2h / (d2h_gbs * 1e9)) / 1e9,
            "api": "field_b200.batch.BatchBuilder (upload_tables, enqueue, tile_offsets / leaf_counts) with pinned "
                   "host buffers for the tiles, kinds and active ids"}


def run_serve(args, rate=1000.0, seconds=10.0, seed=7, arena_gb=None, warmup_s=0.5):
    """Poisson arrivals at `rate` req/s for `warmup_s` + `seconds`, the statistics over the requests
    arriving after the first `warmup_s` (the same mix, run first so that the window measures the
    steady state): 40 % builds (recipes as the batched
    workload), 30 % edits (1-64 tool capsules subtracted from a resident field), 20 % point queries
    (1e5-1e6 points, value + gradient), 10 % EDT recomputations; latency = completion - arrival.
    Request payloads (recipes, tool lists, point sets) are generated before the arrival window, as
    a client would hold them; the submitting thread sleeps between arrivals."""
    import torch
    import field_b200.batch as BT
    import field_b200.expr as X
    import field_b200.recipes as R
    import field_b200.serve as S
    torch.cuda.set_device(0)
    rng = np.random.default_rng(seed)
    pool = [(X.compile_recipe(r), n) for r, n, _ in R.batch_recipes(count=64, seed=11)]
    n_req = int(rate * (seconds + warmup_s))
    gaps = rng.exponential(1.0 / rate, size=n_req)
    kinds = rng.choice(["build", "edit", "query", "edt"], size=n_req, p=[0.4, 0.3, 0.2, 0.1])
    # the client keeps its point sets in pinned host memory, which the server takes without a copy
    point_sets = [torch.from_numpy(rng.uniform(0, 1, (int(m), 3)).astype(np.float32)).pin_memory()
                  for m in np.geomspace(100_000, 1_000_000, 8)]
    tool_sets = [X.compile_tools(R.tools(rng, int(k))) for k in rng.integers(1, 65, size=32)]
    working_set = 64  # requests on fields pick among the most recently built ones
    # resident field buffers and request temporaries from one arena the size of the budget: no
    # cudaMalloc (or cudaFree, which synchronises the device) on the request path once it is taken
    slots = int(getattr(args, "slots", 16))
    arena_gb = getattr(args, "arena_gb", 150.0) if arena_gb is None else arena_gb
    srv = S.FieldServer(slots=slots, budget_bytes=150e9, arena_bytes=arena_gb * 1e9)
    try:
        # warm start: a resident field of every grid size, every kernel configured, one EDT per
        # grid size and one query per point-set size (pinned staging of each size allocated once)
        sizes = sorted({n for _, n in pool})
        firsts = [next(i for i, (_, n) in enumerate(pool) if n == sz) for sz in sizes]
        warm = [srv.submit("build", recipe=pool[i][0], meta=BT.cube_meta(pool[i][1], 8)) for i in firsts + list(range(8))]
        live = [f.result(timeout=120)["field"] for f in warm]
        for fid in live[:len(sizes)]:
            srv.submit("edt", field=fid).result(timeout=120)
        for ps in point_sets:
            srv.submit("query", field=live[0], points=ps).result(timeout=120)
        srv.submit("edit", field=live[1], tools=tool_sets[0]).result(timeout=120)
        # pinned staging for as many concurrent results of each query size as there are slots, and
        # for the recipe tables that builds and edits upload
        for ps in point_sets:
            srv.reserve_pinned(len(ps) * 4, slots)
            srv.reserve_pinned(len(ps) * 12, slots)
        for c in range(16, 21):  # recipe tables of 64 KB to 1 MB
            srv.reserve_pinned(1 << c, 2 * slots)
        srv.completed.clear()
        # the collector's full passes over the request objects would pause both threads mid-window
        gc.collect()
        gc.freeze()
        gc.disable()
        alloc0 = torch.cuda.memory_stats()
        # the client takes each result as it completes and drops it (result arrays are views of
        # the server's pooled pinned blocks, which return to the pool when dropped)
        errors = {}
        outstanding = [0]
        count_lock = threading.Lock()
        all_done = threading.Event()
        submitted = [False]

        def on_done(fu, kind):
            e = fu.exception()
            if e is not None:
                errors[type(e).__name__] = errors.get(type(e).__name__, 0) + 1
            elif kind == "build":
                live.append(fu.result()["field"])
            with count_lock:
                outstanding[0] -= 1
                if submitted[0] and outstanding[0] == 0:
                    all_done.set()

        t0 = time.perf_counter()
        due = t0
        for k, gap in zip(kinds, gaps):
            due += gap
            wait = due - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            fid = live[-working_set:][int(rng.integers(min(len(live), working_set)))]
            with count_lock:
                outstanding[0] += 1
            if k == "build":
                c, n = pool[int(rng.integers(len(pool)))]
                f = srv.submit("build", recipe=c, meta=BT.cube_meta(n, 8))
            elif k == "edit":
                f = srv.submit("edit", field=fid, tools=tool_sets[int(rng.integers(len(tool_sets)))], op="subtract")
            elif k == "query":
                f = srv.submit("query", field=fid, points=point_sets[int(rng.integers(len(point_sets)))])
            else:
                f = srv.submit("edt", field=fid)
            f.add_done_callback(lambda fu, kind=str(k): on_done(fu, kind))
        t_submitted = time.perf_counter()
        with count_lock:
            submitted[0] = True
            if outstanding[0] == 0:
                all_done.set()
        if not all_done.wait(timeout=600):
            errors["ClientTimeout"] = outstanding[0]
        t_end = time.perf_counter()
        gc.enable()
        gc.unfreeze()
        alloc1 = torch.cuda.memory_stats()
        warm_n = sum(1 for _, a, _, _ in srv.completed if a < t0 + warmup_s)
        done = [c for c in srv.completed if c[1] >= t0 + warmup_s]
        t0 += warmup_s
        lat = np.array([(e - a) * 1e3 for _, a, _, e in done])
        # worst latency of the requests arriving in each half second: a stall shows as one window
        windows = {}
        for _, a, _, e in done:
            k = int((a - t0) / 0.5)
            windows[k] = max(windows.get(k, 0.0), (e - a) * 1e3)
        by_kind = {}
        for kind, a, st, e in done:
            by_kind.setdefault(kind, []).append(((e - a) * 1e3, (st - a) * 1e3))
    finally:
        srv.close()
    return {
        "metric": METRIC, "workload": "serve_poisson", "rate_req_s": rate, "seconds": seconds,
        "requests": len(done), "warmup": {"seconds": warmup_s, "requests": warm_n},
        "errors": errors, "offered_req_s": n_req / (t_submitted - t0 + warmup_s),
        "throughput_req_s": len(lat) / (t_end - t0), "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "by_kind": {k: {"n": len(v), "p50_ms": float(np.percentile([x for x, _ in v], 50)),
                        "p99_ms": float(np.percentile([x for x, _ in v], 99)),
                        "queue_p50_ms": float(np.percentile([q for _, q in v], 50))}
                    for k, v in by_kind.items()},
        "slowest": [{"kind": k, "arrival_s": round(a - t0, 3), "queue_ms": round((st - a) * 1e3, 1),
                     "service_ms": round((e - st) * 1e3, 1)}
                    for k, a, st, e in sorted(done, key=lambda c: c[1] - c[3])[:5]],
        "worst_ms_per_half_second": [round(windows.get(k, 0.0), 1) for k in range(max(windows) + 1)] if windows else [],
        "allocator": {k: int(alloc1.get(k, 0) - alloc0.get(k, 0)) for k in ("num_device_alloc", "num_device_free",
                                                                           "num_alloc_retries")},
        "resident_gb": round(srv.resident_bytes() / 1e9, 2),
        "slots": slots, "budget_gb": 150, "arena_gb": arena_gb, "data": "synthetic",
    }


def run_tree(args, n=512, samples=50_000_000):
    """Packed adaptive block tree of a dense n^3 SDF (union of 48 seeded spheres, float32, built on
    the device), built and then sampled at `samples` random grid indices on the GPU; the oracle's
    CPU build of a 128^3 crop timed beside it.  Build: dense voxels per second (four block
    classifications of the dense field, the breadth-first levels, packing); sampling: indices per
    second (24 B of indices in, 4 B out, tree reads from L2)."""
    # the nodes of each level are classified from the dense field directly (8 corner reads each)
    import torch
    import field_b200.tree as T
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(5)
    c = torch.rand((48, 3), generator=g, dtype=torch.float64) * 0.7 + 0.15
    r = torch.rand(48, generator=g, dtype=torch.float64) * 0.12 + 0.03
    pitch = 1.0 / n
    ax = torch.arange(n, dtype=torch.float64, device=dev) * pitch
    dense = torch.full((n, n, n), 1.0e3, dtype=torch.float64, device=dev)
    for k in range(48):
        d = ((ax[:, None, None] - c[k, 0]) ** 2 + (ax[None, :, None] - c[k, 1]) ** 2
             + (ax[None, None, :] - c[k, 2]) ** 2).sqrt_() - r[k]
        torch.minimum(dense, d, out=dense)
        del d
    dense = dense.to(torch.float32)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    pts = torch.stack([torch.randint(0, n, (samples,), generator=g) for _ in range(3)], dim=1).to(dev)

    def timed(fn, reps):
        out = []
        for _ in range(reps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = fn()
            e1.record()
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return out, res

    build = lambda: T.build_device(dense, pitch)
    timed(build, max(args.warmup, 3))
    clocks = ClockSampler(0)
    clocks.start()
    t_build, t = timed(build, args.steps)
    tree = T.AdaptiveBlocks.from_device(t, pitch, host=False)
    sample = lambda: tree.sample_device(pts)
    timed(sample, 3)
    t_sample, _ = timed(sample, args.steps)
    clk = clocks.stop()
    assert int(tree._dev["status"].item()) == 0
    mb, ms = statistics.median(t_build), statistics.median(t_sample)
    voxels = n ** 3
    peak, peak_src = measured_peaks()
    # algorithmic bytes of a build: the dense field read once (4 B per voxel; the tree's own arrays
    # are a few percent of that); of a sample: 24 B of indices + 4 B of output
    build_gbs = 4.0 * voxels / (mb * 1e-3) / 1e9
    sample_gbs = 28.0 * samples / (ms * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu:
        import oracle
        crop = dense[:128, :128, :128].cpu().numpy()
        t0 = time.perf_counter()
        oracle.tree_build(crop, pitch)
        dt = time.perf_counter() - t0
        cpu = {"value": 128 ** 3 / dt / 1e9, "unit": "Gvox/s", "cores": len(os.sched_getaffinity(0)), "kind": "port",
               "sample": "oracle tree build (C dense classification at 4 sides + NumPy levels) of a 128^3 crop"}
    return {
        "metric": "packed adaptive tree: dense voxels/s built, indices/s sampled", "workload": f"tree_{n}^3",
        "value": voxels / (mb * 1e-3) / 1e9, "unit": "Gvox/s", "higher_is_better": True, "steps": args.steps,
        "build_ms": mb, "sample_ms": ms, "samples": samples, "sample_gsamples_s": samples / (ms * 1e-3) / 1e9,
        "node_count": t["node_count"], "values": int(len(t["values"])), "level_sizes": t["level_sizes"],
        "roofline": {"build": {"bound": "hbm", "achieved": build_gbs, "peak": peak, "unit": "GB/s",
                               "frac": build_gbs / peak, "basis": "4 B per dense voxel (the field read once)"},
                     "sample": {"bound": "hbm", "achieved": sample_gbs, "peak": peak, "unit": "GB/s",
                                "frac": sample_gbs / peak, "basis": "28 B per sample (indices in, value out)"},
                     "peak_source": peak_src},
        "cpu_baseline": cpu, "clocks": clk, "dtype": "f32 dense, 2-bit codes", "data": "synthetic",
        "config": {"workload": f"tree_{n}^3_48spheres", "grid": [n, n, n], "l2": "256 MiB flush between steps"},
    }


def run_clearance(args, pitch=0.01):
    """EDT consumers on the default EDT's obstacle grid (n^3, 2000 boxes, 8 % fill) as the route
    network of laplaceflode_v1.rutt_genom_flode's first steps: the squared EDT to the occupied cells,
    the clearance in mm, the validity mask, and the lattice Laplacian (count pass, scans, node map,
    edges and CSR).  Device-resident steps through the C ABI with preallocated outputs (CUDA events,
    L2 flushed between steps); end to end through field_b200.clearance.fritt_natverk with NumPy in
    and NumPy/scipy out; the oracle's NumPy restatement timed on a 128^3 crop beside it."""
    import torch
    import field_b200._lib as L_
    import field_b200.clearance as C
    import field_b200.recipes as R
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n = args.edt_n
    occ_np = R.obstacle_grid(seed=2, n=n, n_boxes=2000, fill=0.08).astype(bool)
    occ = torch.from_numpy(occ_np.view(np.uint8)).to(dev)
    L = L_.lib()
    st = L_.stream_handle()
    V = occ.numel()
    sq = torch.empty(occ.shape, dtype=torch.int32, device=dev)
    edt_scr = torch.empty(int(L.fb_edt_scratch_bytes(n, n, n, 0)), dtype=torch.uint8, device=dev)
    E = torch.empty(occ.shape, dtype=torch.float64, device=dev)
    valid = torch.empty(occ.shape, dtype=torch.uint8, device=dev)
    lat_scr = torch.empty(int(L.fb_lattice_scratch_bytes(n, n, n)), dtype=torch.uint8, device=dev)
    totals = torch.empty(3, dtype=torch.int32, device=dev)
    L.fb_lattice_count_device(occ.data_ptr(), n, n, n, totals.data_ptr(), lat_scr.data_ptr(), lat_scr.numel(), st)
    nodes, n_edges, nnz = (int(x) for x in totals.cpu().tolist())
    node_map = torch.empty(occ.shape, dtype=torch.int32, device=dev)
    u = torch.empty(n_edges, dtype=torch.int32, device=dev)
    v = torch.empty(n_edges, dtype=torch.int32, device=dev)
    kond = torch.empty(n_edges, dtype=torch.float64, device=dev)
    indptr = torch.empty(nodes + 1, dtype=torch.int32, device=dev)
    indices = torch.empty(nnz, dtype=torch.int32, device=dev)
    data = torch.empty(nnz, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    threshold = 1.0 + 2.0 * pitch

    def step():
        rc = [0] * 5
        ev[0].record()
        rc[0] = L.fb_edt_squared_device(occ.data_ptr(), n, n, n, 1, sq.data_ptr(), edt_scr.data_ptr(), edt_scr.numel(), st)
        rc[1] = L.fb_edt_mm_device(sq.data_ptr(), V, pitch, E.data_ptr(), st)
        ev[1].record()
        rc[2] = L.fb_clearance_mask_device(occ.data_ptr(), E.data_ptr(), V, threshold, valid.data_ptr(), st)
        ev[2].record()
        rc[3] = L.fb_lattice_count_device(occ.data_ptr(), n, n, n, totals.data_ptr(), lat_scr.data_ptr(),
                                          lat_scr.numel(), st)
        ev[3].record()
        rc[4] = L.fb_lattice_emit_device(occ.data_ptr(), E.data_ptr(), n, n, n, pitch, 1.5, node_map.data_ptr(),
                                         u.data_ptr(), v.data_ptr(), kond.data_ptr(), n_edges, indptr.data_ptr(),
                                         nodes + 1, indices.data_ptr(), data.data_ptr(), nnz, lat_scr.data_ptr(),
                                         lat_scr.numel(), st)
        ev[4].record()
        assert not any(rc), rc

    phases = []
    for i in range(max(args.warmup, 3) + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        step()
        torch.cuda.synchronize()
        if i >= max(args.warmup, 3):
            phases.append([ev[k].elapsed_time(ev[k + 1]) for k in range(4)])
    clocks = ClockSampler(0)
    clocks.start()
    tt = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        tt.append(e0.elapsed_time(e1))
    clk = clocks.stop()
    assert [int(x) for x in totals.cpu().tolist()] == [nodes, n_edges, nnz]
    ms = statistics.median(tt)
    ph = [statistics.median(p[k] for p in phases) for k in range(4)]
    peak, peak_src = measured_peaks()
    # algorithmic bytes of the lattice passes: occupancy read by the count, node and emit passes
    # (3 B per cell), node map written and read (8 B), clearance read (8 B), row starts (4 B per node),
    # edges (16 B), CSR entries (12 B)
    lat_bytes = 3.0 * V + 8.0 * V + 8.0 * V + 4.0 * (nodes + 1) + 16.0 * n_edges + 12.0 * nnz
    lat_ms = ph[2] + ph[3]
    lat_gbs = lat_bytes / (lat_ms * 1e-3) / 1e9
    # end to end: NumPy occupancy in, NumPy arrays and a scipy CSR out
    # the first call fills the module's page-locked pool (the results' host blocks return to it
    # when they are dropped); the later calls are the steady state of a caller that repeats it
    e2e_ms, d2h = [], 0
    for _ in range(0 if args.no_e2e else 3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = C.fritt_natverk(occ_np, pitch)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        d2h = sum(int(getattr(a, "nbytes", 0)) for a in res if isinstance(a, np.ndarray))
        d2h += res[-1].data.nbytes + res[-1].indices.nbytes + res[-1].indptr.nbytes
        del res
        gc.collect()
    cpu = None
    if not args.no_cpu:
        import oracle
        crop = np.ascontiguousarray(occ_np[:128, :128, :128])
        t0 = time.perf_counter()
        Ec = oracle.clearance_mm(crop, pitch)
        oracle.lattice_laplacian(crop, Ec, pitch, 1.5)
        dt = time.perf_counter() - t0
        cpu = {"value": crop.size / dt / 1e9, "unit": "Gvox/s", "cores": len(os.sched_getaffinity(0)), "kind": "port",
               "sample": "oracle clearance (C EDT) + NumPy lattice Laplacian of a 128^3 crop of the same grid"}
    e2e = min(e2e_ms[1:]) if e2e_ms else None
    return {
        "metric": "EDT consumers: grid cells/s (clearance, validity mask, lattice Laplacian)",
        "workload": f"clearance_network_{n}^3", "value": V / (ms * 1e-3) / 1e9, "unit": "Gvox/s",
        "higher_is_better": True, "steps": args.steps, "ms_per_step": ms,
        "phases_ms": {"edt_and_clearance": ph[0], "validity_mask": ph[1], "lattice_count": ph[2],
                      "lattice_nodes_and_emit": ph[3]},
        "nodes": nodes, "edges": n_edges, "csr_entries": nnz,
        "roofline": {"bound": "hbm", "kernel": "lattice passes (count, scans, nodes, emit)", "achieved": lat_gbs,
                     "peak": peak, "unit": "GB/s", "frac": lat_gbs / peak, "peak_source": peak_src,
                     "basis": "3 B occupancy + 8 B node map + 8 B clearance per cell, 4 B per node, "
                              "16 B per edge, 12 B per CSR entry", "bytes": lat_bytes},
        "e2e": None if e2e is None else {"value": V / (e2e * 1e-3) / 1e9, "unit": "Gvox/s", "ms": e2e,
                                         "first_call_ms": e2e_ms[0],
                                         "h2d_bytes_per_step": int(occ_np.nbytes), "d2h_bytes_per_step": int(d2h)},
        # per step: squared EDT 3 (bits, zy, x), clearance 1, mask 1, lattice count 1 + three
        # two-level scans of 3 each, node map 1, emit 1
        "gpu_launches": 17 * args.steps, "cpu_baseline": cpu, "clocks": clk, "dtype": "u8 in, int32 + f64 out",
        "data": "synthetic",
        "config": {"workload": f"clearance_network_{n}^3_2000boxes_8pct", "grid": [n, n, n], "pitch_mm": pitch,
                   "p_kond": 1.5, "l2": "256 MiB flush between steps"},
    }


def run_mesh(args, pitch=0.08):
    """Mesh -> signed distance field (ray-winding solid, paired exact EDT, surface layer) of a seeded
    scene of a sphere, a rotated box and a torus (about 55 k triangles) on a grid of pitch 0.08 mm
    around it, through the C entry point with host buffers (mesh in, solid / sd / surface out, all
    inside the timed region), against the reference's own meshsdf_field_cpu compiled from its source
    (OpenMP, every host thread) on the same input."""
    import torch
    import field_b200.mesh as M
    import field_b200.recipes as R
    torch.cuda.set_device(0)
    V, T = R.mesh_scene(7, 0.0, fine=4)
    lo = V.min(0) - 2 * pitch
    gmin, shape = M.window(V, pitch, lo)
    origin = lo + gmin * pitch
    jit = (pitch * M.JITTER_FRAC * M.GOLDEN[0], pitch * M.JITTER_FRAC * M.GOLDEN[1])
    run = lambda: M.field_grid(V, T, origin, pitch, shape, jitter=jit)
    for _ in range(max(args.warmup, 3)):
        run()
    clocks = ClockSampler(0)
    clocks.start()
    walls, stages = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        out = run()
        walls.append(time.perf_counter() - t0)
        stages.append(out[4])
    clk = clocks.stop()
    voxels = int(np.prod(shape))
    wall = statistics.median(walls)
    dev = np.median(np.array(stages), axis=0)
    cpu = None
    if not args.no_cpu:
        import oracle
        t0 = time.perf_counter()
        rc, *_ = oracle.ref_mesh_field(V, T, origin, pitch, jit, shape, True, nthreads=0)
        dt = time.perf_counter() - t0
        cpu = {"value": voxels / dt / 1e9, "unit": "Gvox/s", "cores": len(os.sched_getaffinity(0)),
               "kind": "reference", "seconds": dt,
               "sample": "the reference's meshsdf_field_cpu (oracle/_ref, OpenMP) on the same mesh and grid"}
    h2d = V.nbytes + T.nbytes
    d2h = voxels * (1 + 4 + 1)
    return {
        "metric": "mesh -> signed distance field: grid voxels/s", "workload": "mesh_field", "value": voxels / wall / 1e9,
        "unit": "Gvox/s", "higher_is_better": True, "steps": args.steps, "ms_per_call": wall * 1e3,
        "device_stage_ms": {k: float(v) * 1e3 for k, v in zip(("hits", "grouping", "winding", "edt", "finish"), dev)},
        "triangles": int(len(T)), "grid": list(shape), "voxels": voxels, "hits": int(out[3][1]),
        "solid_voxels": int(out[3][3]),
        "e2e": {"value": voxels / wall / 1e9, "unit": "Gvox/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "api": "meshsdf_field_cpu (host buffers)"},
        "cpu_baseline": cpu, "clocks": clk, "dtype": "f64 rays, int32 EDT, f32 sd", "data": "synthetic",
        "config": {"workload": f"mesh_scene_{len(T)}tris_pitch{pitch}", "grid": list(shape)},
    }


def run_precision(args):
    """Precision stress: 1000 near-tangent sphere pairs (gap U[0, 0.5] fine pitches) and 64 walls half
    a fine voxel thick, as a per-block-pitch field mixing pitch 1/128 (level 0) and 1/512 (level 2)
    over the unit cube (512^3-equivalent).  The GPU builds every brick lattice; the float64 oracle
    (the CPU leg, timed) evaluates a seeded sample of bricks of both levels; the line reports the
    worst per-block |d_f32 - d_f64| in units of the brick's pitch and the sign disagreements."""
    import torch
    import field_b200.multires as M
    import field_b200.recipes as R
    import field_b200.expr as X
    import oracle
    torch.cuda.set_device(0)
    recipe = R.tangent_pairs(seed=4, n_pairs=1000, pitch=1.0 / 512, walls=64)
    comp = X.compile_recipe(recipe)
    # the fine pitch where a brick's culled list is at least the median length (the crowded bricks)
    fine = lambda lens: np.where(np.asarray(lens) >= np.median(lens), 2, 0)
    build = lambda: M.bygg_multires_fran_recept(recipe, [0, 0, 0], 1.0 / 128, (16, 16, 16), block=8, levels=fine,
                                                overlappsband=False)
    build()  # warm-up: kernels configured
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    F = build()
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    tiles = F.tiles
    rng = np.random.default_rng(1)
    per_level = {}
    for u in sorted(tiles):
        bi, bj, bk = np.unravel_index(int(u), F.brick_shape)
        per_level.setdefault(int(F.niva[bi, bj, bk]), []).append(int(u))
    checked, block_max, sign, rel = {}, [], 0, 0.0
    t_cpu = 0.0
    for lvl, ids in sorted(per_level.items()):
        pick = rng.choice(ids, size=min(args.check_bricks, len(ids)), replace=False)
        checked[str(lvl)] = int(len(pick))
        pitch = F.h_grov / (1 << lvl)
        for u in pick:
            bi, bj, bk = np.unravel_index(int(u), F.brick_shape)
            m = tiles[int(u)].shape[0]
            pts = F.lo + np.array([bi, bj, bk]) * F.L + np.indices((m, m, m)).reshape(3, -1).T * pitch
            c0 = time.perf_counter()
            want = oracle.eval_points(comp.prims, comp.program, pts)
            t_cpu += time.perf_counter() - c0
            got = tiles[int(u)].reshape(-1).astype(np.float64)
            err = np.abs(got - want)
            band = np.abs(want) <= 3 * pitch
            block_max.append(float(err[band].max() / pitch) if band.any() else 0.0)
            rel = max(rel, float((err / np.maximum(np.abs(want), pitch)).max()))
            sign += int(np.count_nonzero((got >= 0) != (want >= 0)))
    samples = int(sum(t.size for t in tiles.values()))
    worst = max(block_max) if block_max else 0.0
    # the plain single build (64 primitives, 256^3, B = 8): its leaf tiles against the same checker
    import field_b200.build as B
    c0_recipe, c0_meta = R.plain_union(seed=0, n=256, block=8)
    c0_comp = X.compile_recipe(c0_recipe)
    c0_fb = B.FieldBuilder(c0_comp, c0_meta)
    c0 = c0_fb.build()
    c0_acc = leaf_accuracy(c0_comp, c0_meta, c0_fb, c0.tiles, c0.n_active, n_blocks=256)
    return {
        "metric": METRIC, "workload": "precision_stress_tangent_pairs_mixed_pitch", "value": worst,
        "unit": "pitch (max per-block |d_f32 - d_f64| within 3 pitches of the surface)", "higher_is_better": False,
        "sign_disagreements": sign, "max_rel_err": rel,
        "per_block_max_err_pitch": {"p50": float(np.percentile(block_max, 50)), "max": worst,
                                    "blocks": len(block_max)},
        "plain_single_build_256": dict(c0_acc, n_active=int(c0.n_active)),
        "bricks_checked_by_level": checked, "bricks_by_level": {str(k): len(v) for k, v in per_level.items()},
        "pitches": {"0": 1.0 / 128, "2": 1.0 / 512}, "lattice_samples": samples, "build_s": build_s,
        "cpu_baseline": {"value": t_cpu, "unit": "s (float64 oracle over the checked bricks)", "cores": oracle.threads(),
                         "kind": "port", "sample": f"{len(block_max)} bricks, all lattice points"},
        "config": {"workload": "1000 near-tangent pairs + 64 half-voxel walls, pitch 1/128 and 1/512",
                   "primitives": int(len(comp.prims))},
        "dtype": "f32 (f64 guard band)", "data": "synthetic",
    }


def spawn_ranks(n):
    """`--gpus N` without torchrun: run this command under torch.distributed.run with N ranks (one
    per GPU, rendezvous on 127.0.0.1) and return its exit status."""
    import socket
    import subprocess
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    if args.impl == "ours" and args.workload in ("serve", "precision", "tree", "mesh", "clearance"):
        fn = {"precision": run_precision, "tree": run_tree, "mesh": run_mesh, "clearance": run_clearance,
              "serve": lambda a: run_serve(a, rate=a.rate, seconds=a.seconds)}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local_rank)
        # short: ranks that wait for a lost peer end with an error instead of hanging
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
    try:
        if args.impl == "reference":
            res = run_reference(args, rank, world)
        elif args.workload == "plain":
            res = run_plain(args, rank, world, local_rank)
        else:
            res = run_headline(args, rank, world, local_rank)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
