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

Under torchrun (N > 1) the mixed workloads run partitioned by default: the
workload's super-cell box stretched N times along z (weak scaling), its
blocks split along their Z-order over the ranks, each rank evolving its
share with the halo exchange (NCCL) before every RK4 stage; --replicas
runs N independent copies instead.  The time is the max over ranks.
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
KIND_NAMES = {"fused": "bssn::rhs_kernel / bssn::onchip_kernel (one-kernel right-hand side)",
              "deriv": "bssn::deriv_kernel (derivative pass)", "eq": "bssn::eq_kernel (equation pass)"}


def tile_pins(arg):
    """--tile: {} (autotune), {0: t} (tile t on every bucket) or {side: tile}."""
    if not arg:
        return {}
    if ":" not in arg:
        return {0: int(arg)}
    return {int(a): int(b) for a, b in (kv.split(":") for kv in arg.split(","))}


def kernel_bytes(sides, chosen, modes):
    """Algorithmic HBM bytes of one right-hand-side pass per kernel kind, by
    the compulsory-traffic rule of the hot-path contract (24 FP64 variables):
    a one-kernel right-hand side (fused or on chip) reads each padded block
    once and writes the interior: 192 (s^3 + (s-6)^3) per block; the split
    path's derivative pass reads the padded block, 192 s^3, and its equation
    pass reads and writes the zone's variables, 384 (s-6)^3.  The split
    path's derivative scratch (162 doubles written and read per zone) is not
    algorithmic: it is returned separately as overhead."""
    out = {"fused": 0, "deriv": 0, "eq": 0, "overhead": 0}
    for s in sides:
        s = int(s)
        pad, inner = s ** 3, (s - 6) ** 3
        if modes[chosen[s]] == 1:
            out["deriv"] += 192 * pad
            out["eq"] += 384 * inner
            out["overhead"] += 2 * 8 * SPLIT_SLOTS * inner
        else:
            out["fused"] += 192 * (pad + inner)
    return out


# DRAM traffic / algorithmic bytes of one launch of each kernel kind, from ncu
# captures on small workloads (dram__bytes_read.sum + dram__bytes_write.sum
# over the launch's algorithmic bytes as kernel_bytes counts them): split
# 7x7x7 on the uniform 512-block workload; the on-chip kernel on the small
# mixed workload.  Scales a full pass's algorithmic bytes to DRAM traffic.
# (uniform 512: deriv 257.0 + 143.4 MB against 192 * 2197 * 512 B; eq 249.3 +
# 17.9 MB against 384 * 343 * 512 B -- the scratch round trip is the excess)
TRAFFIC_RATIO = {"deriv": 400.4e6 / (192 * 2197 * 512), "eq": 267.2e6 / (384 * 343 * 512)}


def rhs_bytes(sides):
    """The fused right-hand side's compulsory bytes per pass: 192 (s^3 + (s-6)^3) per block."""
    return sum(192 * (int(s) ** 3 + (int(s) - 6) ** 3) for s in sides)


def step_bytes(sides):
    """Compulsory HBM bytes of one RK stage (the contract's full-stage rule):
    192 (3 s^3 + 2 (s-6)^3) per block -- padded read by the right-hand side,
    ghost fill write and read, stage-state, accumulator and next-state
    traffic of the interior."""
    return sum(192 * (3 * int(s) ** 3 + 2 * (int(s) - 6) ** 3) for s in sides)


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
# reference arm: the reference's own CPU RK4 step on the host cores
# ---------------------------------------------------------------------------
# The CPU step runs on a bounded sample of a workload: the same generator,
# seed and size mix on fewer super-cells (3 x 3 x 3 of mix20k's 10 x 10 x 7:
# 741 blocks, 3.35 M zones), so K steps finish within minutes on the host.
REF_SAMPLE_DIMS = (3, 3, 3)


def ref_sample(wl):
    """(mode, dims, name) of the CPU sample of workload wl."""
    mode, dims, _ = WORKLOADS[wl]
    if mode == 0:
        return mode, dims, wl
    sd = tuple(min(a, b) for a, b in zip(dims, REF_SAMPLE_DIMS))
    if sd == tuple(dims):
        return mode, dims, wl
    return mode, sd, f"{wl}-sample-{sd[0]}x{sd[1]}x{sd[2]}"


class CpuRK4:
    """The reference CPU RK4 step (ghost fill, the block-loop right-hand side,
    zip, stage algebra and constraint enforcement of the oracle's restatement
    of rkBSSN.cpp:764-860) with the right-hand side the reference's own
    compiled bssnrhs (oracle/_ref, kind "reference"; the oracle's
    restatement, kind "port", where that library is absent), on a mesh built
    by the oracle's generator: the product library is not loaded."""

    def __init__(self, mode, dims, threads=0):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as ol
        self.ol = ol
        self.spec = ol.OracleMeshSpec(mode, dims, MIX, seed=SEED_MESH)
        O = ol.oracle()
        ref = ol.reference()
        self.kind = "reference" if ref is not None else "port"
        self.fn = ref.lib.ref_bssnRHS_blocks if ref is not None else None
        self.mo = ol.MeshOracle(self.spec, O)
        self.Z = self.mo.initial_data(eps=1e-8)
        self.ws = self.mo.rk4_workspace()
        self.dt = 0.25 * self.spec.h
        self.prm = ol.params()
        self.threads = threads or os.cpu_count()

    def step(self):
        t0 = time.perf_counter()
        bad = self.mo.rk4_step_ws(self.Z, self.dt, self.prm, self.ws, rhs_fn=self.fn,
                                  nthreads=self.threads)
        assert bad == 0, f"{bad} enforcement violations"
        return time.perf_counter() - t0


def cpu_baseline(wl, steps=3, threads=0):
    """Timed CPU RK4 steps on the workload's sample: (zone-updates/s, info)."""
    mode, dims, name = ref_sample(wl)
    c = CpuRK4(mode, dims, threads)
    c.step()  # warm-up (page faults of the workspace)
    ts = [c.step() for _ in range(steps)]
    zones = c.spec.zones()
    rate = zones * steps / sum(ts)
    return rate, {"kind": c.kind, "cores": c.threads,
                  "sample": f"{name}: {c.spec.nblocks} blocks, {zones} zones; {steps} full RK4 steps "
                            f"(ghost fill, bssnrhs block loop, zip, stage algebra, enforcement), "
                            f"{sum(ts):.1f} s"}


def run_reference(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    mode, dims, desc = WORKLOADS[wl]
    if mode == 2:
        print(json.dumps({"impl": "reference", "unavailable": "the CPU oracle has no multi-level "
                          "ghost fill outside the test harness; run the single-level workloads"}))
        return
    smode, sdims, name = ref_sample(wl)
    c = CpuRK4(smode, sdims)
    for _ in range(args.warmup):
        c.step()
    ts = [c.step() for _ in range(args.steps)]
    total = sum(ts)
    zones = c.spec.zones()
    rate = zones * args.steps / total
    info = {"kind": c.kind, "cores": c.threads,
            "sample": f"{name}: the workload's generator, seed and size mix on "
                      f"{sdims[0]}x{sdims[1]}x{sdims[2]} super-cells ({c.spec.nblocks} blocks, {zones} zones); "
                      "each step one full RK4 step"}
    out = {"metric": "BSSN RK4 zone-updates/s FP64 on 1 B200, batched vs plain; % HBM roofline",
           "impl": "reference", "value": rate, "unit": "zone-updates/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": name, "sampled_from": wl, "description": desc,
                      "blocks": c.spec.nblocks, "zones": zones, "nodes": c.spec.n_nodes,
                      "path": "reference CPU RK4 step: oracle ghost fill + the reference's compiled "
                              "bssnrhs block loop (OpenMP over blocks) + zip + stage algebra + "
                              "enforce_bssn_constraints"},
           "cpu_baseline": dict(info, value=rate, unit="zone-updates/s", cpu_model=cpu_model()),
           "e2e": {"value": rate, "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "step_seconds": ts}
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
                    help="multi-GPU form (the default for N > 1 on mixed workloads): one mesh N times "
                         "larger, partitioned along the Z-order of its blocks, halo exchange before "
                         "every RK4 stage")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: N independent replicas of the workload instead of the partitioned form")
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

    if args.partition or (world > 1 and WORKLOADS[wl][0] == 1 and not args.replicas):
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
                 "launches_per_step": B.lib.bssn_rk4_plan_launches_per_step(pplan.h),
                 "path": "the batched plan's own right-hand-side kernels and tiles, launched block by "
                         "block in mesh order (the reference's bssnRHS loop, rhs.cpp:10-73), no graph"}
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
    kb = kernel_bytes(spec.sides, chosen, modes)
    kernels = {}
    for k, key in enumerate(("fused", "deriv", "eq")):
        ms, n = kt[k], kt[3 + k]
        if n <= 0:
            continue
        gbs = kb[key] / (ms * 1e-3) / 1e9
        kernels[key] = {"kernel": KIND_NAMES[key], "ms_per_pass": ms, "launches_per_pass": n,
                        "bytes_per_pass": kb[key], "achieved_gbs": gbs, "frac": gbs / hbm_peak}
    dom = max(kernels, key=lambda k: kernels[k]["ms_per_pass"])
    d = kernels[dom]
    ratio = TRAFFIC_RATIO.get(dom)
    flops_rhs = zones * FLOP_PER_ZONE_STAGE
    rb = rhs_bytes(spec.sides)
    roofline = {"bound": "hbm", "kernel": d["kernel"],
                "achieved": d["achieved_gbs"], "peak": hbm_peak, "unit": "GB/s",
                "frac": d["frac"], "peak_source": peak_src,
                "traffic": (ratio * d["bytes_per_pass"] / d["launches_per_pass"]) if ratio else None,
                "launch_ms": d["ms_per_pass"] / d["launches_per_pass"],
                "bytes_per_launch": d["bytes_per_pass"] / d["launches_per_pass"],
                "kernels": kernels,
                "split_scratch_overhead_bytes_per_pass": kb["overhead"],
                "rhs_pass": {"ms": rhs_ms.value, "algorithmic_bytes": rb,
                             "achieved_gbs": rb / (rhs_ms.value * 1e-3) / 1e9,
                             "frac": rb / (rhs_ms.value * 1e-3) / 1e9 / hbm_peak},
                "fp64": {"achieved_tflops": flops_rhs / (rhs_ms.value * 1e-3) / 1e12,
                         "peak_tflops": fp64.value, "peak_source": "measured FMA probe",
                         "frac": flops_rhs / (rhs_ms.value * 1e-3) / 1e12 / fp64.value,
                         "scope": "whole right-hand-side pass, 6,535 FP64 operations per zone"}}
    sb = step_bytes(spec.sides) * 4
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
                        "frac": sb / (ms_step * 1e-3) / 1e9 / hbm_peak,
                        "rule": "192 (3 s^3 + 2 (s-6)^3) bytes per block and RK stage"},
           "plain": plain, "batched_vs_plain": (value / plain["value"]) if plain else None,
           "e2e": e2e, "clocks": clk,
           "gpu_launches": args.steps * launches_per_step,
           "enforce_violations": violations, "state_finite": finite,
           "autotune_ms": {str(k): v for k, v in table.items()}}
    if not args.no_cpu:
        rate, info = cpu_baseline(wl if mode != 2 else "mix20k", steps=2)
        out["cpu_baseline"] = dict(info, value=rate, unit="zone-updates/s", cpu_model=cpu_model(),
                                   nproc=os.cpu_count())
        if mode == 1:
            rate1, info1 = cpu_baseline("small", steps=1, threads=1)
            out["cpu_baseline"]["one_thread"] = {"value": rate1, "sample": info1["sample"]}
    print(json.dumps(out, default=_plain))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
