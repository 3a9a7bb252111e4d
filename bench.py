#!/usr/bin/env python
"""Throughput of the FARGO hydro step on B200: cell-updates/s.

A cell-update is one active cell (NRAD*NSEC, ghost row excluded) advanced
through one hydro substep.  One bench *step* is one DT of every disk of the
workload (each disk takes its own CFL substeps inside the DT).

Workloads (--workload):
  c4  (default) 64 isothermal disks of uneven size and physics, batched: one
      launch per kernel advances all of them (the "batched" form); the disks
      are grouped into --groups batches of similar CFL substep counts
      (measured by one probe DT) and balanced work
  c4plain  the same 64 disks advanced one after another (the "plain" form)
  c1, c2, c3, c5  single disks of the other configurations

Output: one JSON line (rank 0).  `value` is device-resident throughput
(CUDA events on the library's stream); `e2e` goes through the C ABI with
page-locked host buffers: every step uploads every disk's state, advances
one DT and downloads the state.  The batched workloads split their disks
over --groups batches (LPT on cell counts) advanced concurrently on their
own streams: one batch's last substeps, when few of its disks are still
inside their DT, and its host copies overlap the other batches' work.  The
C4 line also carries the plain form (the same disks advanced one after
another) measured in the same run, as `plain`.

`--impl reference` times the reference's own CUDA build
(oracle/_ref/fargo_ref, compiled from the reference sources) on a bounded
sample of the same workload: one disk of every grid size of the sweep, the
K timed steps shared out over them (one step = one DT of one sampled disk),
each disk first run for its share of the W warm-up DTs.  Its AlgoGas wall
time and substep count come from the timing hook (no device copies or file
writes inside the timed call).  That arm loads nothing of this package: the
workload definitions are read from configs.py by file path.

Multi-GPU: `bench.py --gpus N` with N > 1 relaunches itself under
torch.distributed.run with N ranks (or runs as one rank of an outside
torchrun).  Every rank advances its own 64 disks (disjoint seeds), no
collective in the data path (weak scaling); the timed region is bracketed
by barriers and the max over ranks is taken.  `--plumbing` runs only the
rank set-up, sharding and max/sum reductions on CPU (gloo), for tests.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic HBM bytes per cell-update: the state read once and written once
# in FP32 (Sigma, v_r, v_theta [, e]).  These are the bytes charged to the
# dominant substep kernel (transport: it reads and rewrites the whole state);
# with self-gravity the four padded complex FFT passes add 128 B per cell to
# the substep, reported separately as `sg_alg_bytes_per_cell` and never
# charged to a substep kernel.
B_STATE = {"c1": 24, "c2": 32, "c3": 24, "c4": 24, "c4plain": 24, "c4q": 24, "c5": 32}
B_SG = {"c3": 128, "c5": 128}


def load_module(name):
    """A module of the package loaded by file path, without importing the
    package (whose __init__ loads the CUDA library)."""
    import importlib.util
    path = os.path.join(ROOT, "cudaprotoplanetarydisksfloat_b200", name + ".py")
    spec = importlib.util.spec_from_file_location("fargo_bench_" + name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax.append(float(parts[2].split()[0]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        shard = load_module("shard")
        if args.plumbing:
            pg = shard.init_process_group("gloo", timeout_s=60)
        else:
            import torch
            torch.cuda.set_device(local)
            pg = shard.init_process_group("nccl", timeout_s=120)
    return world, rank, local, pg


def _dev(pg):
    import torch
    return "cpu" if pg.get_backend() == "gloo" else "cuda"


def barrier(pg):
    if pg is not None:
        import torch
        if _dev(pg) == "cpu":
            pg.barrier()
        else:
            pg.barrier(device_ids=[torch.cuda.current_device()])


def allmax(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=_dev(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allsum(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=_dev(pg))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def workload_disks(name, seed_shift=0, rank=0, world=1, strong=False):
    configs = load_module("configs")
    if strong and name in ("c4", "c4plain"):
        # one fixed 64-disk sweep, split over the ranks by LPT on cell counts
        shard = load_module("shard")
        sweep = configs.c4(64, seed=42)
        cells = [int(p["Nrad"]) * int(p["Nsec"]) for p, _ in sweep]
        return [sweep[i] for i in shard.lpt_partition(cells, world)[rank]]
    if name in ("c4", "c4plain"):
        return configs.c4(64, seed=42 + seed_shift)
    if name == "c4q":
        return configs.c4(64, seed=42 + seed_shift)[::4]
    fn = {"c1": configs.c1, "c2": configs.c2, "c3": configs.c3, "c5": configs.c5}[name]
    return [fn()]


WL_DESC = {"c4": "64 isothermal disks (Nrad in {128..512}, Nsec=3*Nrad), batched, one DT each",
           "c4plain": "64 isothermal disks (Nrad in {128..512}, Nsec=3*Nrad), one after another",
           "c4q": "every 4th disk of the 64-disk sweep (16 disks, 6.1M cells), batched",
           "c1": "isothermal 128x384, 1 planet", "c2": "adiabatic 256x768, alpha viscosity, 2 live planets",
           "c3": "self-gravitating 512x1024, 1 planet", "c5": "adiabatic+SG 2048x6144, 3 live planets"}


def workload_config(args, world):
    """The `config` object of the JSON line: the same for both arms, computed
    from the workload definition alone (nothing measured in it)."""
    disks = workload_disks(args.workload)
    n = len(disks)
    per_rank = -(-n // world) if args.strong else n
    if args.strong:
        cells = sum(int(p["Nrad"]) * int(p["Nsec"]) for p, _ in disks)
    else:
        # every rank advances its own draw of the workload (seed shifted by rank)
        cells = sum(int(p["Nrad"]) * int(p["Nsec"]) for r in range(world)
                    for p, _ in workload_disks(args.workload, seed_shift=r))
        n *= world
    batches = per_rank if args.workload == "c4plain" else max(1, min(args.groups, per_rank))
    return {"workload": args.workload, "description": WL_DESC[args.workload],
            "parallelism": "disk-parallel: the GPU's disks in concurrent batches on their own streams"
            if args.workload.startswith("c4") else "single disk per GPU",
            "l2": "working set larger than L2" if args.workload in ("c4", "c4plain", "c4q", "c5")
            else "working set L2-resident (launch-bound)",
            "disks": n, "cells": cells, "batches_per_gpu": batches}


def batch_groups(cells, groups, plain):
    """The disks of one rank as batches: one per disk for the plain form;
    otherwise `groups` batches balanced by LPT on cell counts, advanced
    concurrently on their own streams, so that one batch's last substeps (few
    disks still inside their DT) overlap another's work."""
    n = len(cells)
    if plain:
        return [[d] for d in range(n)]
    G = max(1, min(groups, n))
    if G == 1:
        return [list(range(n))]
    from cudaprotoplanetarydisksfloat_b200 import shard
    return [sorted(g) for g in shard.lpt_partition([int(c) for c in cells], G)]


def substep_groups(P, L, cells, probe_groups, G, rank, local):
    """Batches of disks with similar CFL substep counts (shard.group_by_substeps):
    one probe DT of every disk, in the cell-balanced batches, gives the counts
    (outside the timed region; the timed batches start afresh)."""
    from cudaprotoplanetarydisksfloat_b200 import Batch, shard
    nsub = np.zeros(len(P), dtype=np.int64)
    for g in probe_groups:
        b = Batch([P[d] for d in g], [L[d] for d in g], device=local)
        noisy_init(b, [P[d] for d in g], [20261203 + 1000 * rank + d for d in g])
        b.advance(1)
        for k, d in enumerate(g):
            nsub[d] = b.scalars(k)["nsub_last_dt"]
        b.close()
    return shard.group_by_substeps(cells, nsub, G)


def materialise_all(disks, tmp):
    from cudaprotoplanetarydisksfloat_b200 import configs, read_params, read_planets
    P, L = [], []
    for k, (p, pl) in enumerate(disks):
        par, cfg, out = configs.materialise(p, pl, tmp, "disk%02d" % k)
        P.append(read_params(par))
        L.append(read_planets(cfg, P[-1]))
    return P, L


def noisy_init(batch, P, seeds):
    from cudaprotoplanetarydisksfloat_b200 import noise
    for d, (p, seed) in enumerate(zip(P, seeds)):
        f = batch.fields(d)
        dens = noise.perturb_density(f["dens"].reshape(-1), p.NRAD, p.NSEC, seed)
        batch.init_state(d, dens=dens)


def ours(args, world, rank, local, pg):
    import torch

    from cudaprotoplanetarydisksfloat_b200 import Batch
    from cudaprotoplanetarydisksfloat_b200._abi import lib

    torch.cuda.set_device(local)
    tmp = tempfile.mkdtemp(prefix="fargo_bench_")
    disks = workload_disks(args.workload, seed_shift=rank, rank=rank, world=world, strong=args.strong)
    P, L = materialise_all(disks, tmp)
    cells = np.array([p.NRAD * p.NSEC for p in P], dtype=np.int64)
    plain = args.workload == "c4plain"
    groups = batch_groups(cells, args.groups, plain)
    if not plain and len(groups) > 1 and args.group_by == "substeps":
        groups = substep_groups(P, L, cells, groups, args.groups, rank, local)
    gcells = np.array([cells[d] for g in groups for d in g], dtype=np.int64)  # nsub_total() order
    batches = [Batch([P[d] for d in g], [L[d] for d in g], device=local) for g in groups]
    for b, g in zip(batches, groups):
        noisy_init(b, [P[d] for d in g], [20261203 + 1000 * rank + d for d in g])
        if args.no_graph:
            b.set_graph_mode(False)
    streams = [torch.cuda.ExternalStream(lib.fargo_batch_stream(b.b), device=local) for b in batches]

    def nsub_total():
        return np.array([b.scalars(k)["nsub_total"] for b, g in zip(batches, groups) for k in range(len(g))],
                        dtype=np.int64)

    def run(k):
        for b in batches:
            b.advance_async(k)

    # warm-up, then the tile autotuner (between DTs, outside the timed region)
    run(args.warmup)
    for b in batches:
        b.sync()
    seg_out = [b.autotune(reps=2) for b in batches]
    # the widths the autotuner kept per class of disk (NSEC), batch by batch
    seg_by_nsec = [{int(P[d].NSEC): s for d, s in sorted(zip(g, b.segments()), key=lambda x: P[x[0]].NSEC)}
                   for b, g in zip(batches, groups)]
    n0 = nsub_total()
    l0 = sum(lib.fargo_batch_count_launches(b.b) for b in batches)
    barrier(pg)
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in batches]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in batches]
    t_wall = time.time()
    if plain:
        # one disk after another on its own stream: serialise through stream 0's events
        ev0[0].record(streams[0])
        for i, b in enumerate(batches):
            if i > 0:
                streams[i].wait_event(ev1[i - 1])
            b.advance_async(args.steps)
            ev1[i].record(streams[i])
        for b in batches:
            b.sync()
        ms = ev0[0].elapsed_time(ev1[-1])
    else:
        # every batch's stream starts after ev0 on stream 0; stream 0 waits for
        # the others' ends before the closing event
        ev0[0].record(streams[0])
        for st in streams[1:]:
            st.wait_event(ev0[0])
        run(args.steps)
        for st, ev in zip(streams, ev1):
            ev.record(st)
        end = torch.cuda.Event(enable_timing=True)
        for ev in ev1[1:]:
            streams[0].wait_event(ev)
        end.record(streams[0])
        for b in batches:
            b.sync()
        ms = ev0[0].elapsed_time(end)
    torch.cuda.synchronize()
    t_wall = time.time() - t_wall
    clocks = clk.stop()
    barrier(pg)
    n1 = nsub_total()
    l1 = sum(lib.fargo_batch_count_launches(b.b) for b in batches)
    upd = float(np.sum(gcells * (n1 - n0)))
    ms_max = allmax(pg, ms)
    upd_all = allsum(pg, upd)
    value = upd_all / (ms_max * 1e-3)

    # end to end through the C ABI with page-locked host buffers: every step
    # uploads every disk's state, advances one DT and downloads the state.  Each
    # batch does so in order on its own stream; with several batches one
    # batch's copies overlap another's DT.
    ebatches, egroups = batches, groups
    estreams = streams
    pinned = []
    for eb, g in zip(ebatches, egroups):
        for k, d in enumerate(g):
            n = (P[d].NRAD + 1) * P[d].NSEC
            arrs = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(3)]
            f = eb.fields(k)
            for a_, key in zip(arrs, ("dens", "vrad", "vtheta")):
                a_.numpy()[:] = f[key].reshape(-1)
            pinned.append((eb, k, arrs))
    fp = C.POINTER(C.c_float)

    def e_nsub():
        return np.array([b.scalars(k)["nsub_total"] for b, g in zip(ebatches, egroups) for k in range(len(g))],
                        dtype=np.int64)

    ecells = np.array([P[d].NRAD * P[d].NSEC for g in egroups for d in g], dtype=np.int64)

    def e2e_step():
        if plain:
            # one disk after another: upload, one DT, download, then the next disk
            for b, k, arrs in pinned:
                ptrs = [C.cast(a_.data_ptr(), fp) for a_ in arrs]
                lib.fargo_batch_upload_async(b.b, k, ptrs[0], ptrs[1], ptrs[2], None)
                lib.fargo_batch_advance_async(b.b, 1)
                lib.fargo_batch_download_async(b.b, k, ptrs[0], ptrs[1], ptrs[2], None)
                b.sync()
            return
        for eb in ebatches:
            mine = [(k, arrs) for b, k, arrs in pinned if b is eb]
            for k, arrs in mine:
                ptrs = [C.cast(a_.data_ptr(), fp) for a_ in arrs]
                lib.fargo_batch_upload_async(eb.b, k, ptrs[0], ptrs[1], ptrs[2], None)
            lib.fargo_batch_advance_async(eb.b, 1)
            for k, arrs in mine:
                ptrs = [C.cast(a_.data_ptr(), fp) for a_ in arrs]
                lib.fargo_batch_download_async(eb.b, k, ptrs[0], ptrs[1], ptrs[2], None)

    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    for _ in range(2):
        e2e_step()
    for b in ebatches:
        b.sync()
    n0 = e_nsub()
    barrier(pg)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ends = [torch.cuda.Event() for _ in estreams]
    e0.record(estreams[0])
    for st in estreams[1:]:
        st.wait_event(e0)
    for _ in range(e2e_steps):
        e2e_step()
    for st, ev in zip(estreams, ends):
        ev.record(st)
    for ev in ends[1:]:
        estreams[0].wait_event(ev)
    e1.record(estreams[0])
    for b in ebatches:
        b.sync()
    torch.cuda.synchronize()
    e_ms = e0.elapsed_time(e1)
    n1 = e_nsub()
    e_upd = allsum(pg, float(np.sum(ecells * (n1 - n0))))
    e_ms = allmax(pg, e_ms)
    bytes_io = sum(4 * 3 * (P[d].NRAD + 1) * P[d].NSEC for d in range(len(P)))
    e2e = {"value": e_upd / (e_ms * 1e-3), "unit": "cell-updates/s", "h2d_bytes_per_step": bytes_io * world,
           "d2h_bytes_per_step": bytes_io * world, "steps": e2e_steps}

    # per-kernel device time (host loop with events around every launch)
    roof = None
    if rank == 0:
        nk = lib.fargo_profile_kernel_count()
        ms_k = np.zeros(nk)
        n0 = nsub_total()
        for b in batches:
            arr = (C.c_double * 16)()
            ns = C.c_int(0)
            st = lib.fargo_batch_profile(b.b, args.profile_steps, arr, C.byref(ns))
            if st == 0:
                ms_k += np.array(arr[:nk])
        n1 = nsub_total()
        upd_prof = float(np.sum(gcells * (n1 - n0)))
        names = [lib.fargo_profile_kernel_name(k).decode() for k in range(nk)]
        top = int(np.argmax(ms_k[:nk - 1]))
        name = names[top]
        adi = int(P[0].Adiabatic)
        # launches of each kernel: every batch's graph loops until its last
        # disk ends its DT
        dn = n1 - n0
        off = np.cumsum([0] + [len(g) for g in groups])
        launches = int(max(1, sum(int(dn[off[k]:off[k + 1]].max()) for k in range(len(groups)))))
        cells_per_launch = upd_prof / launches
        peak, kind = load_peaks()
        # algorithmic bytes per cell-update of the dominant kernel: the state
        # read once and written once (self-gravity's FFT bytes excluded)
        b_alg = B_STATE[args.workload]
        b_sub = b_alg + B_SG.get(args.workload, 0)
        achieved = b_alg * cells_per_launch / (ms_k[top] * 1e-3 / launches) / 1e9
        # the kernel's DRAM bytes per cell and issue utilisation from one ncu
        # capture (profiles/dram_traffic_c4q_first_substep.md)
        traffic = issue = None
        try:
            with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
                tj = json.load(f)
            if name in tj:
                traffic = round(float(tj[name]["dram_bytes_per_cell"]) * cells_per_launch)
                issue = tj[name].get("issue_active_pct")
        except (OSError, ValueError, KeyError):
            pass
        roof = {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "issue_active_pct_ncu": issue,
                "alg_bytes_per_cell": b_alg, "alg_bytes_per_launch": round(b_alg * cells_per_launch),
                "launch_ms": round(float(ms_k[top]) / launches, 4),
                "step_frac": round(value * b_sub / (peak * 1e9), 4),
                "substep_alg_bytes_per_cell": b_sub, "sg_alg_bytes_per_cell": B_SG.get(args.workload, 0),
                "kernel_ms_share": {names[k]: round(float(ms_k[k] / ms_k.sum()), 4) for k in range(nk)
                                    if ms_k[k] > 0},
                # the batches' kernels one after another (host loop, one batch at a
                # time): against ms_per_step it shows how much the concurrent
                # batches overlap
                "kernel_ms_per_step_serial": round(float(ms_k.sum()) / args.profile_steps, 3)}

    for b in batches:
        b.close()
    plain_line = None
    if args.workload == "c4" and args.plain_steps > 0:
        plain_line = plain_form(args, P, L, rank, local, pg, world)
        if plain_line is not None:
            plain_line["batched_over_plain"] = round(value / plain_line["value"], 3)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, disks)
    return {
        "value": value, "ms_per_step": ms_max / args.steps, "e2e": e2e, "roofline": roof,
        "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": int(l1 - l0) * world,
        "wall_s": t_wall, "cells": int(cells.sum()) * world, "disks": len(P) * world,
        "seg_out": sorted(set(seg_out)), "seg_by_nsec": seg_by_nsec, "batches": len(batches), "plain": plain_line,
        "batching": {"by": "one disk per context" if plain else args.group_by,
                     "disks_per_batch": [len(g) for g in groups]},
    }


def plain_form(args, P, L, rank, local, pg, world):
    """The plain form on the same disks: each disk a context of its own,
    advanced one after another (device-resident, CUDA events), after one
    warm-up DT.  Measured beside the batched form so that the ratio of the
    two is in the same line."""
    import torch

    from cudaprotoplanetarydisksfloat_b200 import Batch
    from cudaprotoplanetarydisksfloat_b200._abi import lib
    singles = [Batch([P[d]], [L[d]], device=local) for d in range(len(P))]
    try:
        for d, b in enumerate(singles):
            noisy_init(b, [P[d]], [20261203 + 1000 * rank + d])
            b.advance_async(1)
        for b in singles:
            b.sync()
        streams = [torch.cuda.ExternalStream(lib.fargo_batch_stream(b.b), device=local) for b in singles]
        n0 = np.array([b.scalars(0)["nsub_total"] for b in singles], dtype=np.int64)
        barrier(pg)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event(enable_timing=True) for _ in singles]
        e0.record(streams[0])
        for i, b in enumerate(singles):
            streams[i].wait_event(e0 if i == 0 else ends[i - 1])
            b.advance_async(args.plain_steps)
            ends[i].record(streams[i])
        for b in singles:
            b.sync()
        ms = e0.elapsed_time(ends[-1])
        n1 = np.array([b.scalars(0)["nsub_total"] for b in singles], dtype=np.int64)
        upd = float(np.sum(np.array([p.NRAD * p.NSEC for p in P], dtype=np.int64) * (n1 - n0)))
        ms = allmax(pg, ms)
        upd = allsum(pg, upd)
    finally:
        for b in singles:
            b.close()
    return {"value": upd / (ms * 1e-3), "ms_per_step": ms / args.plain_steps, "steps": args.plain_steps,
            "unit": "cell-updates/s", "form": "each disk its own context, advanced one after another"}


def cpu_baseline(args, disks):
    """The oracle (the CPU restatement of the reference's algorithm, OpenMP
    over all host cores) on the median-size disk of the workload, built in
    FP64 (the baseline) and in FP32 (the reference's typing, reported as
    `f32_value`), each for a bounded number of DTs."""
    from cudaprotoplanetarydisksfloat_b200 import noise
    from oracle.oracle import Oracle, set_threads
    tmp = tempfile.mkdtemp(prefix="fargo_cpu_")
    sizes = [int(p["Nrad"]) * int(p["Nsec"]) for p, _ in disks]
    k = int(np.argsort(sizes)[len(sizes) // 2])
    P, L = materialise_all([disks[k]], tmp)
    cores = os.cpu_count() or 1
    o32 = Oracle(P[0], L[0], "f32")
    f = o32.fields()
    o32.init_state(dens=noise.perturb_density(f["dens"].reshape(-1), P[0].NRAD, P[0].NSEC, 7))
    g = o32.fields()
    cells = P[0].NRAD * P[0].NSEC
    out = {}
    for prec, secs in (("f64", args.cpu_seconds), ("f32", 0.5 * args.cpu_seconds)):
        set_threads(cores, prec)
        o = o32 if prec == "f32" else Oracle(P[0], L[0], "f64")
        if prec == "f64":
            o.set_fields(dens=g["dens"], vrad=g["vrad"], vtheta=g["vtheta"], energy=g["energy"])
        o.advance_dt()
        t0 = time.time()
        nsub = ndt = 0
        while ndt < args.cpu_max_dt and time.time() - t0 < secs:
            nsub += o.advance_dt()
            ndt += 1
        dt = time.time() - t0
        out[prec] = (cells * nsub / dt, ndt, nsub, dt)
        o.close()
    v, ndt, nsub, dt = out["f64"]
    return {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port",
            "sample": "oracle FP64 (OpenMP, %d threads), disk %d of the workload (%dx%d), %d DTs, %d substeps, "
                      "%.1f s" % (cores, k, P[0].NRAD, P[0].NSEC, ndt, nsub, dt),
            "f32_value": out["f32"][0]}


def reference_sample(disks, K, W):
    """The reference arm's sample of a workload: one disk of every grid size
    (the first of each size in sweep order), with the K timed DTs and the W
    warm-up DTs shared out over them (every disk takes at least one warm-up
    DT, which pays the reference's first-call set-up)."""
    firsts = {}
    for k, (p, _) in enumerate(disks):
        firsts.setdefault(int(p["Nrad"]), k)
    pick = [firsts[n] for n in sorted(firsts)]
    m = len(pick)
    timed = [K // m + (1 if i < K % m else 0) for i in range(m)]
    warm = [max(1, W // m + (1 if i < W % m else 0)) for i in range(m)]
    return [(k, t, w) for k, t, w in zip(pick, timed, warm) if t > 0]


def reference(args, world, rank):
    """The reference's own CUDA build (its only implementation of the path)
    on a bounded sample of the workload, timed by its own AlgoGas calls."""
    exe = os.path.join(ROOT, "oracle", "_ref", "fargo_ref")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/fargo_ref is not built (needs the reference sources at build time)"}
    configs = load_module("configs")
    disks = workload_disks(args.workload)
    tmp = tempfile.mkdtemp(prefix="fargo_ref_")
    tot_upd, tot_s, tot_dt, samples = 0.0, 0.0, 0, []
    for k, ntimed, nwarm in reference_sample(disks, args.steps, args.warmup):
        p, pl = disks[k]
        ndt = nwarm + ntimed
        # Main.cu runs AlgoGas for i = 0 .. NTOT-1 (output only at i = 0)
        p = dict(p, Ntot=str(ndt), Ninterm="100000")
        d = os.path.join(tmp, "disk%02d" % k)
        configs.materialise(p, pl, d, "run", relative=True)
        times = os.path.join(d, "algogas_times.txt")
        env = dict(os.environ, FARGO_REF_TIMES=times, FARGO_REF_NOISE_SEED=str(20261203 + k))
        env.pop("FARGO_REF_DUMP", None)
        r = subprocess.run([exe, "run.par"], cwd=d, env=env, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                           timeout=1200)
        if r.returncode != 0:
            return {"unavailable": "reference run failed with exit code %d" % r.returncode}
        alg = np.loadtxt(times, ndmin=2)
        if alg.shape[0] < ndt or alg.shape[1] < 3:
            return {"unavailable": "reference run wrote %d AlgoGas lines, expected %d" % (alg.shape[0], ndt)}
        sel = alg[nwarm:ndt]
        nrad, nsec = int(p["Nrad"]), int(p["Nsec"])
        tot_upd += float(np.sum(sel[:, 2])) * nrad * nsec
        tot_s += float(np.sum(sel[:, 1]))
        tot_dt += sel.shape[0]
        samples.append("%dx%d:%d" % (nrad, nsec, sel.shape[0]))
    return {"value": tot_upd / tot_s, "ms_per_step": 1e3 * tot_s / max(1, tot_dt), "sample": samples,
            "dts": tot_dt}


def relaunch(args):
    """`--gpus N` (N > 1) outside a launcher: run this script under
    torch.distributed.run with N ranks on this node and return its status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def plumbing(args, world, rank, pg):
    """Rank set-up, sharding and the max/sum reductions without a GPU: each
    rank takes its disks as the timed run does and reports their cells."""
    disks = workload_disks(args.workload, seed_shift=rank, rank=rank, world=world, strong=args.strong)
    cells = float(sum(int(p["Nrad"]) * int(p["Nsec"]) for p, _ in disks))
    barrier(pg)
    t0 = time.perf_counter()
    barrier(pg)
    ms = allmax(pg, 1e3 * (time.perf_counter() - t0))
    return {"cells": allsum(pg, cells), "ranks_reporting": allsum(pg, 1.0), "ms_max": ms}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=["c4", "c4plain", "c4q", "c1", "c2", "c3", "c5"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--groups", type=int, default=4,
                    help="concurrent batches the disks of a batched workload are split over")
    ap.add_argument("--group-by", default="substeps", choices=["substeps", "cells"],
                    help="batch the disks by similar CFL substep counts (one probe DT) or by cells (LPT)")
    ap.add_argument("--profile-steps", type=int, default=2)
    ap.add_argument("--plain-steps", type=int, default=3,
                    help="DTs of the plain form measured beside the batched C4 line (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--cpu-max-dt", type=int, default=400)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--strong", action="store_true",
                    help="split one fixed 64-disk sweep over the ranks instead of one sweep per rank")
    ap.add_argument("--no-graph", action="store_true",
                    help="host loop instead of the CUDA graph (for per-launch profilers)")
    ap.add_argument("--plumbing", action="store_true",
                    help="ranks, sharding and reductions only, on CPU (gloo): no GPU work")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(args)
    if args.impl == "reference":
        # no process group: rank 0 alone runs the reference, the others exit
        world, rank, local, pg = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0, None
    else:
        world, rank, local, pg = dist_setup(args)
    config = workload_config(args, world)
    metric = "cell-updates/s"
    head = {"metric": metric, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "strong" if args.strong else "weak",
            "vs_baseline": None, "dtype": "f32"}
    if args.plumbing:
        r = plumbing(args, world, rank, pg)
        if rank == 0:
            print(json.dumps(dict(head, value=None, data="none (plumbing check)", config=config, plumbing=r)),
                  flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return 0
    if args.impl == "reference":
        if rank != 0:
            return 0
        r = reference(args, world, rank)
        if "unavailable" in r:
            line = {"impl": "reference", "unavailable": r["unavailable"]}
        else:
            sample = ("the reference's own CUDA build (its only implementation) on the B200, one disk of each "
                      "grid size of the workload (%s, grid:DTs), %d timed DTs after warm-up, AlgoGas wall time"
                      % (", ".join(r["sample"]), r["dts"]))
            line = dict(head, impl="reference", n_gpus=world, data="synthetic (seeded parameters and density noise)",
                        config=config, value=r["value"], ms_per_step=r["ms_per_step"],
                        e2e={"value": r["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0},
                        cpu_baseline={"value": r["value"], "unit": "cell-updates/s", "cores": 1,
                                      "kind": "reference", "sample": sample})
        print(json.dumps(line), flush=True)
        return 0
    r = ours(args, world, rank, local, pg)
    if rank == 0:
        line = dict(head, value=r["value"], ms_per_step=r["ms_per_step"],
                    data="synthetic (seeded parameters and density noise)", config=config,
                    tiles={"transport_segment": r["seg_out"], "segment_by_nsec": r["seg_by_nsec"], "band_rings": 8,
                           "autotuned": True},
                    batching=r["batching"],
                    e2e=r["e2e"], roofline=r["roofline"], cpu_baseline=r["cpu_baseline"], clocks=r["clocks"],
                    gpu_launches=r["gpu_launches"])
        if r.get("plain"):
            line["plain"] = r["plain"]
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
