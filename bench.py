#!/usr/bin/env python
"""Benchmark of the BSSN RK4 evolution step on B200.

Default workload (N=1): the batched form -- a seeded single-level octree of
~20,000 blocks with padded sides drawn from {13,19,31,55} with block-count
fractions {0.7,0.2,0.08,0.02}, Brill-Lindquist two-puncture data (m=0.5 at
(+-1,0,0)) plus a seeded 1e-8 perturbation, FP64, KO sigma 0.4, eta 2,
dt = 0.25*dx.  One timed step = one full RK4 step (4 x {ghost fill, fused
RHS over all blocks, zip + stage update + constraint enforcement}), replayed
as a CUDA graph.  Prints one JSON line (see the keys below).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload mix20k|mix4k|uniform512|small|levels]

Under torchrun each rank evolves its own replica of the workload (weak
scaling); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dendro-gr_b200")
sys.path.insert(0, PKG)

WORKLOADS = {
    # name: (mesh mode, dims, description)
    "mix20k": (1, (10, 10, 7), "batched form: ~20,000 blocks, seeded size mix"),
    "mix4k": (1, (7, 5, 4), "mixed-level plain-path size: ~4,000 blocks"),
    "uniform512": (0, (8, 8, 8), "uniform octree of 512 blocks of 13^3"),
    "small": (1, (2, 2, 2), "small mix for profiler captures"),
    "levels": (2, (24, 7), "multi-level: [-400,400]^3, 7 nested levels of 24^3-octant boxes "
                           "halving toward the punctures at (+-4,0,0)"),
}


def level_boxes(M0, nlevels):
    """Boxes of levels 1.. for the `levels` workload: each level's box is
    M0 of its own octants per axis, centred on the origin, so it covers the
    middle half of its parent's box."""
    boxes, lo = [], 0
    for _ in range(1, nlevels):
        lo = 2 * lo + M0 // 2
        boxes.append(((lo,) * 3, (M0,) * 3))
    return boxes


def workload_spec(B, wl):
    """The mesh of a workload: a seeded single-level octree, or the nested
    multi-level mesh of `levels`."""
    mode, dims, _ = WORKLOADS[wl]
    if mode == 2:
        from bssn_b200 import levels as LV
        return LV.generate_levels((dims[0],) * 3, level_boxes(dims[0], dims[1]), xmin=-400.0, L=800.0)
    return B.generate_mesh(mode, dims, MIX, seed=SEED_MESH)
SEED_MESH = 20261203
MIX = (0.7, 0.2, 0.08, 0.02)
FLOP_PER_ZONE_STAGE = 6535.0  # 6,439 RHS + 96 RK axpy (per zone, per stage)


SPLIT_SLOTS = 162  # scratch doubles per zone of the split right-hand side


def tile_pins(arg):
    """--tile: {} (autotune), {0: t} (tile t on every bucket) or {side: tile}."""
    if not arg:
        return {}
    if ":" not in arg:
        return {0: int(arg)}
    return {int(a): int(b) for a, b in (kv.split(":") for kv in arg.split(","))}


def kernel_bytes(sides, chosen, modes, n_nodes, direct):
    """Algorithmic HBM bytes of one right-hand-side pass per kernel kind, as
    the plan's timing call runs it.
    Direct form: the derivative pass reads the 24 zipped variables once and
    writes 162 derivative doubles per node; the equation pass reads them and
    the node's 24 variables and writes its 24 right-hand sides.
    Every bucket split (zipped right-hand side): the derivative pass reads
    the 24 padded variables once (192 B per padded point) and writes 162
    doubles per node, from the zone owning it; the equation pass reads those
    and the node's 24 variables and writes its 24 right-hand sides.
    Otherwise, per block by the tile chosen for its side: fused reads the 24
    padded variables and writes the 24 interior right-hand sides; split
    writes / reads 162 derivative doubles per interior zone in between."""
    out = {"fused": 0, "deriv": 0, "eq": 0}
    n_nodes = int(n_nodes)
    if direct:
        out["deriv"] = 8 * (24 + SPLIT_SLOTS) * n_nodes
        out["eq"] = 8 * (SPLIT_SLOTS + 24 + 24) * n_nodes
        return out
    if all(modes[chosen[int(s)]] == 1 for s in sides):
        out["deriv"] = 8 * (24 * sum(int(s) ** 3 for s in sides) + SPLIT_SLOTS * n_nodes)
        out["eq"] = 8 * (SPLIT_SLOTS + 24 + 24) * n_nodes
        return out
    for s in sides:
        s = int(s)
        pad, inner = s ** 3, (s - 6) ** 3
        if modes[chosen[s]] == 0:
            out["fused"] += 8 * 24 * (pad + inner)
        else:
            out["deriv"] += 8 * (24 * pad + SPLIT_SLOTS * inner)
            out["eq"] += 8 * (SPLIT_SLOTS + 24 + 24) * inner
    return out


# DRAM traffic / algorithmic bytes of each kernel (dram__bytes_read.sum +
# dram__bytes_write.sum of one launch over that launch's algorithmic bytes),
# from ncu captures of the 7x7x7 split tile on the uniform 512-block workload
# (13^3 blocks); scales a full pass's algorithmic bytes to its DRAM traffic.
TRAFFIC_RATIO = {"deriv": 1.09, "eq": 1.35}


def step_bytes(sides, n_nodes):
    """Compulsory HBM bytes of one RK stage of the padded plan: ghost fill
    (read zipped, write padded), right-hand side (read padded, write
    interior), zip + update (read RHS, u, acc; write stage state and acc).
    The split right-hand side's derivative round trip is not included."""
    pad = sum(int(s) ** 3 for s in sides)
    inner = sum((int(s) - 6) ** 3 for s in sides)
    n_nodes = int(n_nodes)
    return 8 * 24 * (n_nodes + pad + pad + inner + inner + 4 * n_nodes)


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
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
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _plain(o):
    """JSON fallback for numpy scalars."""
    try:
        return o.item()
    except AttributeError:
        return str(o)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU bssnrhs on the host cores
# ---------------------------------------------------------------------------
def cpu_reference_rate(sides_all, seconds=15.0, threads=0, target=2.5e6):
    """Time the reference CPU right-hand side (oracle/_ref, compiled from the
    reference sources; else the repository's CPU restatement) on a bounded,
    size-stratified sample of the workload's blocks with all host threads.
    Returns (zone-updates/s, info).  One RK4 zone-update = 4 RHS passes;
    ghost fill, zip and the stage algebra are excluded (favours the CPU)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol

    ref = ol.reference()
    kind = "reference"
    if ref is None:
        ref = ol.oracle()
        kind = "port"
    rng = np.random.default_rng(1)
    # stratified sample: keep the workload's size fractions, ~2.5M zones
    sides_all = np.asarray(sides_all)
    uniq, counts = np.unique(sides_all, return_counts=True)
    zones_all = float(((sides_all - 6.0) ** 3).sum())
    frac = min(1.0, target / zones_all)
    sample = []
    for s, c in zip(uniq, counts):
        k = max(1, int(round(c * frac)))
        sample += [int(s)] * k
    # lay the sample out as independent blocks with BL-like data
    offs, off = [], 0
    for s in sample:
        offs.append(off)
        off += s ** 3
    U = np.zeros((24, off))
    U[[0, 1, 12, 15, 17]] = 1.0
    U += 1e-8 * rng.uniform(-1, 1, U.shape)
    blocks = []
    for s, o in zip(sample, offs):
        h = 0.05
        pmin = rng.uniform(-6, 6, 3)
        blocks.append((o, s, pmin, pmin + (s - 1) * h))
    nthreads = threads or os.cpu_count()

    class RB(C.Structure):
        _fields_ = [("offset", C.c_int64), ("sz", C.c_int32), ("bflag", C.c_uint32),
                    ("g0", C.c_int32 * 3), ("level", C.c_int32),
                    ("ptmin", C.c_double * 3), ("ptmax", C.c_double * 3)]
    arr = (RB * len(blocks))()
    for i, (o, s, pm, px) in enumerate(blocks):
        arr[i].offset, arr[i].sz, arr[i].bflag = o, s, 0
        arr[i].ptmin[:] = list(pm)
        arr[i].ptmax[:] = list(px)
    R = np.zeros_like(U)
    prm = ol.params()
    fn = ref.lib.ref_bssnRHS_blocks if kind == "reference" else ref.lib.orc_bssnRHS
    zones = float(sum((s - 6) ** 3 for s in sample))
    t0 = time.perf_counter()
    passes = 0
    while True:
        fn(ol.rows(R), ol.rows(U), arr, len(blocks), C.byref(prm), nthreads)
        passes += 1
        if time.perf_counter() - t0 > seconds and passes >= 4:
            break
    dt = time.perf_counter() - t0
    rate = zones * passes / 4.0 / dt
    return rate, {"kind": kind, "cores": nthreads,
                  "sample": f"{len(sample)} blocks ({zones:.3g} zones) drawn with the "
                            f"workload's size fractions; {passes} RHS passes in {dt:.1f} s; "
                            "RHS only (ghost fill / zip / RK algebra excluded)"}


def run_reference(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import bssn_b200 as B
    mode, dims, desc = WORKLOADS[wl]
    spec = workload_spec(B, wl)
    rates = []
    for _ in range(args.warmup):
        cpu_reference_rate(spec.sides, seconds=2.0)
    for _ in range(args.steps):
        r, info = cpu_reference_rate(spec.sides, seconds=6.0)
        rates.append(r)
    rate = statistics.median(rates)
    ms = spec.zones() / rate * 1e3
    out = {"metric": "BSSN RK4 zone-updates/s FP64 on 1 B200, batched vs plain; % HBM roofline",
           "impl": "reference", "value": rate, "unit": "zone-updates/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": wl, "description": desc, "blocks": spec.nblocks},
           "cpu_baseline": dict(info, value=rate, unit="zone-updates/s"),
           "e2e": {"value": rate, "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out, default=_plain))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_partitioned(args, wl, B, torch, dist, world, rank, local, barrier, max_over_ranks):
    """Weak scaling of the partitioned form: the workload's super-cell box
    stretched N times along z (about N times the blocks), split along the
    Z-order of its blocks; each rank evolves its share on its own box with
    the halo exchange (NCCL send / receive) before every RK4 stage.  value =
    all ranks' zones x steps / the slowest rank's CUDA-event time."""
    from bssn_b200.distributed import PartitionedRK4
    mode, dims, desc = WORKLOADS[wl]
    assert mode == 1, "--partition needs a mixed (super-cell) workload"
    gdims = (dims[0], dims[1], dims[2] * world)
    spec = B.generate_mesh(mode, gdims, MIX, seed=SEED_MESH)
    zones = spec.zones()
    prm = B.default_params()
    dt = 0.25 * spec.h
    pr = PartitionedRK4(spec, rank, world, prm)
    pins = tile_pins(args.tile)
    sub = pr.sub
    U = torch.zeros((24, sub.n_nodes), dtype=torch.float64, device="cuda")
    B.initial_data(U, sub.spec)  # nodes of other ranks are replaced by the first exchange
    if pins:
        for side, t in pins.items():
            pr.plan.set_tile(t, side)
    else:
        pr.plan.autotune(U, reps=2)
    for _ in range(args.warmup):
        pr.step(U, dt)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        pr.step(U, dt)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    ms_step = ms_total / args.steps
    e2e = None
    if not args.no_e2e:
        host = torch.empty_like(U, device="cpu").pin_memory()
        host.copy_(U)
        k = max(1, min(3, args.steps))
        barrier()
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(k):
            U.copy_(host, non_blocking=True)
            pr.step(U, dt)
            host.copy_(U, non_blocking=True)
        b1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(b0.elapsed_time(b1)) / k
        e2e = {"value": zones / (ems * 1e-3), "unit": "zone-updates/s",
               "h2d_bytes_per_step": U.numel() * 8, "d2h_bytes_per_step": U.numel() * 8,
               "ms_per_step": ems, "path": "each rank's pinned host state -> device, one partitioned "
                                           "RK4 step, device -> host"}
    lps = B.lib.bssn_rk4_plan_launches_per_step(pr.plan.h)
    halo = 4 * (len(sub.send) + len(sub.recv))  # pack + unpack launches per step
    halo_nodes = sum(len(v) for v in sub.recv.values())
    finite = bool(torch.isfinite(U[:, torch.from_numpy(sub.owned).cuda()]).all().item())
    pr.close()
    if rank != 0:
        return
    out = {"metric": "BSSN RK4 zone-updates/s FP64, partitioned over N B200 (halo exchange per stage)",
           "value": zones * args.steps / (ms_total * 1e-3), "unit": "zone-updates/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (Brill-Lindquist + seeded 1e-8 noise)",
           "config": {"workload": wl + f"-x{world}", "description": desc + f", box x{world} along z",
                      "blocks": spec.nblocks, "zones": zones, "nodes": spec.n_nodes,
                      "rank0_blocks": int(sub.spec.nblocks), "rank0_halo_nodes": int(halo_nodes),
                      "l2": "inputs larger than L2",
                      "parallelism": f"partition x{world}: Z-order blocks, halo exchange per stage"},
           "roofline": None, "e2e": e2e, "clocks": clk,
           "gpu_launches": args.steps * (lps + halo),
           "state_finite": finite}
    print(json.dumps(out, default=_plain))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mix20k", choices=sorted(WORKLOADS))
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--tile", default="",
                    help="pin tiles instead of autotuning (profiling runs): one tile id for every "
                         "bucket, or side:tile pairs such as 13:6,19:6,31:8,55:6")
    ap.add_argument("--partition", action="store_true",
                    help="multi-GPU form: one mesh N times larger, partitioned along the Z-order "
                         "of its blocks, halo exchange before every RK4 stage (mixed workloads)")
    args = ap.parse_args()
    wl = args.workload
    if args.impl == "reference":
        run_reference(args, wl)
        return

    import torch
    import bssn_b200 as B

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.partition:
        run_partitioned(args, wl, B, torch, dist, world, rank, local, barrier, max_over_ranks)
        if dist is not None:
            dist.destroy_process_group()
        return

    mode, dims, desc = WORKLOADS[wl]
    spec = workload_spec(B, wl)
    zones = spec.zones()
    prm = B.default_params()
    dt = 0.25 * spec.h
    mesh = B.Mesh(spec)
    U = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    if mode == 2:
        from bssn_b200 import levels as LV
        LV.initial_data_levels(U, spec, mesh=mesh, bh=(4.0, 0.0, 0.0, -4.0, 0.0, 0.0))
    else:
        B.initial_data(U, spec)
    U0 = None
    stream = torch.cuda.current_stream()

    # ---- batched, graph-captured plan
    plan = B.RK4Plan(mesh, prm, B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    pins = tile_pins(args.tile)
    if pins:
        for side, t in pins.items():
            chosen = plan.set_tile(t, side)
        table = {}
    else:
        chosen, table = plan.autotune(U, reps=2)
    for _ in range(args.warmup):
        plan.step(U, dt)
    torch.cuda.synchronize()
    # kernel rooflines: every right-hand-side launch timed with CUDA events
    # on the launch stream (3 passes after a warm-up)
    rhs_ms = C.c_float(0)
    B.check(B.lib.bssn_rk4_plan_time_rhs(plan.h, 3, B.stream_ptr(), C.byref(rhs_ms)), "time_rhs")
    kt = (C.c_double * 6)()
    B.lib.bssn_rk4_plan_time_kernels.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_double)]
    B.check(B.lib.bssn_rk4_plan_time_kernels(plan.h, 3, B.stream_ptr(), kt), "time_kernels")
    B.lib.bssn_rk4_plan_launches_per_step.argtypes = [C.c_void_p]
    launches_per_step = B.lib.bssn_rk4_plan_launches_per_step(plan.h)
    scratch = torch.zeros(1, dtype=torch.float64, device="cuda")
    fp64 = C.c_double(0)
    B.lib.bssn_fp64_probe.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_double)]
    B.check(B.lib.bssn_fp64_probe(C.c_void_p(scratch.data_ptr()), 20000, B.stream_ptr(), C.byref(fp64)), "fp64_probe")

    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.step(U, dt)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    ms_step = ms_total / args.steps
    value = zones * args.steps * world / (ms_total * 1e-3)
    violations = plan.violations()
    finite = bool(torch.isfinite(U).all().item())
    plan.close()

    # ---- plain path: one RHS launch per block, no graph
    plain = None
    if not args.no_plain:
        pplan = B.RK4Plan(mesh, prm, B.PLAN_ENFORCE_STAGES | B.PLAN_PER_BLOCK)
        pplan.step(U, dt)
        torch.cuda.synchronize()
        k = max(1, min(3, args.steps))
        barrier()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(k):
            pplan.step(U, dt)
        a1.record(stream)
        torch.cuda.synchronize()
        pms = max_over_ranks(a0.elapsed_time(a1)) / k
        plain = {"value": zones * world / (pms * 1e-3), "ms_per_step": pms, "steps": k,
                 "launches_per_step": 4 * (spec.nblocks + 2)}
        pplan.close()

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.empty_like(U, device="cpu").pin_memory()
        host.copy_(U)
        plan = B.RK4Plan(mesh, prm, B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
        Ud = torch.empty_like(U)
        nbytes = U.numel() * 8
        Ud.copy_(host, non_blocking=True)
        plan.step(Ud, dt)
        host.copy_(Ud, non_blocking=True)
        torch.cuda.synchronize()
        k = max(1, min(3, args.steps))
        # Each step: the state's 24 variables host -> device, the RK4 step,
        # the 24 results device -> host.  The copies run per variable on two
        # copy streams so that a variable's upload overlaps another's
        # download (PCIe is full duplex); a variable's upload for step n+1
        # waits for its download from step n, and the step waits for all
        # uploads, so every byte still makes the round trip every step.
        up, down = torch.cuda.Stream(), torch.cuda.Stream()
        nv = U.shape[0]
        got = [torch.cuda.Event() for _ in range(nv)]      # download of variable v done
        put = [torch.cuda.Event() for _ in range(nv)]      # upload of variable v done
        stepped = torch.cuda.Event()
        for v in range(nv):
            got[v].record(stream)
        barrier()
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        up.wait_event(b0)
        for _ in range(k):
            for v in range(nv):
                up.wait_event(got[v])
                with torch.cuda.stream(up):
                    Ud[v].copy_(host[v], non_blocking=True)
                put[v].record(up)
            for v in range(nv):
                stream.wait_event(put[v])
            plan.step(Ud, dt)
            stepped.record(stream)
            down.wait_event(stepped)
            for v in range(nv):
                with torch.cuda.stream(down):
                    host[v].copy_(Ud[v], non_blocking=True)
                got[v].record(down)
        for v in range(nv):
            stream.wait_event(got[v])
        b1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(b0.elapsed_time(b1)) / k
        e2e = {"value": zones * world / (ems * 1e-3), "unit": "zone-updates/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "ms_per_step": ems,
               "path": "pinned host state -> device (per variable, overlapping the previous "
                       "step's downloads), one RK4 step through bssn_rk4_plan_step, device -> host"}
        plan.close()
        del host

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    peaks, peak_src = measured_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    modes = [B.tile_mode(t) for t in range(len(B.tiles()))]
    kb = kernel_bytes(spec.sides, chosen, modes, spec.n_nodes, direct=False)
    names = {"fused": "bssn::rhs_kernel (fused RHS)", "deriv": "bssn::deriv_kernel (derivative pass)",
             "eq": "bssn::eq_kernel (equation pass)"}
    kernels = {}
    for k, key in enumerate(("fused", "deriv", "eq")):
        ms, n = kt[k], kt[3 + k]
        if n <= 0:
            continue
        gbs = kb[key] / (ms * 1e-3) / 1e9
        kernels[key] = {"kernel": names[key], "ms_per_pass": ms, "launches_per_pass": n,
                        "bytes_per_pass": kb[key], "achieved_gbs": gbs, "frac": gbs / hbm_peak}
    dom = max(kernels, key=lambda k: kernels[k]["ms_per_pass"])
    d = kernels[dom]
    ratio = TRAFFIC_RATIO.get(dom)
    flops_rhs = zones * FLOP_PER_ZONE_STAGE
    roofline = {"bound": "hbm", "kernel": d["kernel"],
                "achieved": d["achieved_gbs"], "peak": hbm_peak, "unit": "GB/s",
                "frac": d["frac"], "peak_source": peak_src,
                "traffic": (ratio * d["bytes_per_pass"] / d["launches_per_pass"]) if ratio else None,
                "launch_ms": d["ms_per_pass"] / d["launches_per_pass"],
                "bytes_per_launch": d["bytes_per_pass"] / d["launches_per_pass"],
                "kernels": kernels,
                "rhs_pass_ms": rhs_ms.value,
                "fp64": {"achieved_tflops": flops_rhs / (rhs_ms.value * 1e-3) / 1e12,
                         "peak_tflops": fp64.value, "peak_source": "measured FMA probe",
                         "frac": flops_rhs / (rhs_ms.value * 1e-3) / 1e12 / fp64.value,
                         "scope": "whole right-hand-side pass"}}
    sb = step_bytes(spec.sides, spec.n_nodes) * 4
    out = {"metric": "BSSN RK4 zone-updates/s FP64 on 1 B200, batched vs plain; % HBM roofline",
           "value": value, "unit": "zone-updates/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (Brill-Lindquist + seeded 1e-8 noise)",
           "config": {"workload": wl, "description": desc, "blocks": spec.nblocks,
                      "zones": zones, "sides": {str(s): int((spec.sides == s).sum()) for s in sorted(set(spec.sides.tolist()))},
                      "nodes": spec.n_nodes, "dt_over_dx": 0.25,
                      "l2": "inputs larger than L2 (24 x %.3g nodes x 8 B)" % spec.n_nodes,
                      "parallelism": f"replicas x{world}", "tiles": {str(k): int(v) for k, v in chosen.items()},
                      "levels": ([{"lo": list(lo), "n": list(n)} for lo, n in spec.boxes]
                                 if getattr(spec, "boxes", None) else None)},
           "roofline": roofline,
           "step_hbm": {"bytes_per_step": sb, "achieved_gbs": sb / (ms_step * 1e-3) / 1e9,
                        "frac": sb / (ms_step * 1e-3) / 1e9 / hbm_peak},
           "plain": plain, "batched_vs_plain": (value / plain["value"]) if plain else None,
           "e2e": e2e, "clocks": clk,
           "gpu_launches": args.steps * launches_per_step,
           "enforce_violations": violations, "state_finite": finite,
           "autotune_ms": {str(k): v for k, v in table.items()}}
    if not args.no_cpu:
        rate, info = cpu_reference_rate(spec.sides, seconds=15.0)
        rate1, info1 = cpu_reference_rate(spec.sides, seconds=5.0, threads=1, target=2.5e5)
        out["cpu_baseline"] = dict(info, value=rate, unit="zone-updates/s", cpu_model=cpu_model(),
                                   nproc=os.cpu_count(),
                                   one_thread={"value": rate1, "sample": info1["sample"]})
    print(json.dumps(out, default=_plain))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
