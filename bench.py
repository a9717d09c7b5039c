#!/usr/bin/env python
"""Benchmark of the steady synthetic phonon-BTE hot path on B200.

One *step* is one outer source iteration (all bands x directions x cells:
gradient, residual, upwind sweep, boundary, moments, synthetic correction,
margins) of the named workload. The default workload is the 3D hotspot
block: a 100 x 100 x 500 nm box of 2.5 nm cubes split into 6 jittered
tetrahedra each (1.92M tets, seed 1), 40 sine-dispersion bands, 128 Gauss
directions, 1e18 W/m^3 in the top 20 nm, in the FP32-sweep form. The 2D
nanoporous cell (config2: 300 nm periodic square, r = 100 nm diffuse pore,
3 nm Delaunay mesh, 40 bands, 64 CADOM directions) stays selectable.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp32|fp64] [--workload config3|config2|config1|config4|config5]

Prints one JSON line (rank 0). ``value`` is device-resident throughput in
band*direction*cell updates/s over exactly K timed steps (CUDA events on the
solver's stream, max over ranks). ``roofline`` is the whole outer iteration
against HBM with the algorithmic 3*s bytes per update (s = 4 in the FP32
form, 8 in FP64): one read of the intensities for gradient and residual,
one write from the sweep, one read for the moments; ``hbm_kernels`` holds
each streaming kernel's own fraction. ``e2e`` is the same metric through the
public API from host buffers: on the 3D block, set the initial field from
pinned host memory, K outer iterations, read every result field back; on
the 2D cell, the same with a solve to residual 1e-8. Under torchrun each
rank solves an independent seeded problem (weak scaling, no collective on
the data path). ``--impl reference`` times the reference's own CPU solver
(oracle/_ref/BTE_CPU) on the 2D decks; the reference cannot read 3D meshes,
so on the 3D block it times the CPU restatement of its algorithm (the
oracle port) on a bounded sample, labelled as such.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0


def measured_peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def build_deck(workload: str, seed: int, h_nm: float = 0.0, height_nm: float = 500.0):
    from giftbte_b200 import decks

    if workload == "config1":
        d = decks.config1_deck(40)
        desc = "gray 1 um square, 40x40x2 triangles (3200), 1 band, 32 CADOM directions"
    elif workload == "config3":
        h = h_nm or 2.5
        d = decks.config3_deck(h_nm=h, seed=1 + seed, size_nm=(100.0, 100.0, height_nm))
        desc = (f"3D hotspot block 100x100x{height_nm:g} nm, cubes of {h} nm split into 6 jittered tets "
                f"({d.mesh.n_cells} tets), 40 sine-dispersion bands, 128 Gauss directions, "
                f"1e18 W/m^3 in the top 20 nm, seed {1 + seed}")
    else:
        d = decks.config2_deck(h_nm=3.0, n_bands=40, n_phi=16, seed=seed)
        desc = (f"2D nanoporous periodic cell 300 nm, r=100 nm diffuse pore, mean edge 3 nm "
                f"({d.mesh.n_cells} triangles), 40 sine-dispersion bands, 64 CADOM directions, seed {seed}")
    return d, desc


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=self.out, stderr=subprocess.DEVNULL)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.out.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# Algorithmic bytes of one launch of each kernel: the least DRAM traffic its
# work needs. s = bytes of a stored intensity (4 in the FP32 form, 8 in
# FP64), dim = stored gradient components, rec = bytes of one sweep record
# (per direction and cell). Per band*direction*cell update unless noted:
#   gradient  read e, write g                         (1 + dim) s
#   residual  read e and g, write R                   (2 + dim) s
#   sweep     read R, write the corrections, read the
#             level records once per band             2 s + rec / nb
#   moments   read e and the corrections, write e     3 s
#   pcg       (per launch) the macro system and three vectors, read once:
#             nnz (8 B value + 4 B column) + nc (b, x in, x out, diagonal: 32 B; order: 4 B)
def kernel_algorithmic_bytes(name: str, s: int, dim: int, nb: int, nd: int, nc: int, nnz: int):
    rec = 48 if s == 4 else 64
    per_update = {"gradient": (1 + dim) * s, "residual": (2 + dim) * s, "sweep": 2 * s + rec / nb,
                  "moments": 3 * s}
    if name in per_update:
        return per_update[name] * nb * nd * nc
    if name == "pcg":
        return nnz * 12 + nc * 36
    return None


# DRAM bytes per band*direction*cell update of each transport kernel
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch divided by the
# updates it processed), from ncu captures; the profiles/ summaries give the
# commands. The 2D figures are from the full-size 17,939-cell cell.
NCU_TRAFFIC_PER_UPDATE = {
    ("config2", "fp32"): {"residual": 747.134464e6 / 45921280, "sweep": 392.428032e6 / 45921280,
                          "gradient": 509.03552e6 / 45921280, "moments": 517.57696e6 / 45921280},
    # the 3D block's figures from its h = 5 nm, 100 nm tall piece (48,000 tets,
    # 2.4576e8 updates per launch); traffic grows with the updates processed
    ("config3", "fp32"): {"residual": 7.309474e9 / 245760000, "sweep": 2.267558e9 / 245760000,
                          "gradient": 4.733219e9 / 245760000, "moments": 2.928845e9 / 245760000},
}


def macro_nnz(deck) -> int:
    """Nonzeros of the macro two-point-flux system: one diagonal entry per cell and
    one per interior face side (boundary and periodic faces enter the
    right-hand side)."""
    m = deck.mesh
    return m.n_cells + sum(len(c) for c in m.cells) - len(m.edges)


def ranks_reduce(value: float, op: str, world: int, device) -> float:
    """A per-rank scalar reduced over the ranks ("max" or "sum"); the value
    itself on one rank."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units_local: float, seconds_local: float, world: int, device) -> float:
    """Units that all ranks processed over the slowest rank's time."""
    units = ranks_reduce(units_local, "sum", world, device)
    return units / ranks_reduce(seconds_local, "max", world, device)


def workload_config(args, deck, desc: str, nb: int, nd: int) -> dict:
    """The workload as both arms print it (same keys and values)."""
    nc = deck.mesh.n_cells
    s_bytes = 4 if args.precision == "fp32" else 8
    return {"workload": desc, "cells": nc, "bands": nb, "directions": nd, "updates_per_step": nb * nd * nc,
            "precision": args.precision,
            "l2": f"band state {nb * nd * nc * s_bytes / 1e6:.0f} MB per copy, larger than the 126 MB L2"}


def directions_of(deck) -> int:
    return 4 * deck.n_phi if deck.material_dim == 2 else 8 * deck.n_theta * deck.n_phi


METRIC = "band*dir*cell updates/s (time to residual 1e-8 alongside); FP32-mixed vs FP64 on 1 B200"


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch

    import giftbte_b200 as g

    torch.cuda.set_device(local_rank)
    torch.cuda.init()
    # a stream of its own (capturable: the library replays its transport
    # stage as a CUDA graph on it)
    stream = torch.cuda.Stream()
    # replicas: a seeded problem per rank; direction shards: one problem,
    # its directions split over the ranks
    by_dirs = args.shard == "directions"
    deck, desc = build_deck(args.workload, seed=0 if by_dirs else rank, h_nm=args.h_nm, height_nm=args.height_nm)
    nc = deck.mesh.n_cells
    prec = g.GBTE_FP32_MIXED if args.precision == "fp32" else g.GBTE_FP64
    s_bytes = 4 if prec == g.GBTE_FP32_MIXED else 8

    t_setup = time.perf_counter()
    solver = g.StaticBTESynthetic.from_deck(deck, precision=prec, device=local_rank, profile=0,
                                            stream=ctypes_stream(stream), cell_order=args.cell_order,
                                            sweep_bands=args.sweep_bands, sweep_vector=args.sweep_vector,
                                            sweep_kernel=args.sweep_kernel, gradient_dirs=args.gradient_dirs,
                                            residual_form=args.residual_form)
    setup_s = time.perf_counter() - t_setup
    nb, nd = solver.num_bands, solver.num_directions
    upd_per_step = nb * nd * nc
    upd_local = upd_per_step
    if by_dirs:
        upd_local = nb * attach_shard(solver, rank, world) * nc
    # warm-up (not timed; the first outer iteration also runs the
    # autotuners and the next captures the transport stage as a CUDA graph)
    solver.solve(max_iter=args.warmup, err_temp=0.0, err_flux=0.0)
    torch.cuda.synchronize()
    # timed region: exactly K outer iterations (margins 0, so none stops early)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    st = solver.solve(max_iter=args.steps, err_temp=0.0, err_flux=0.0)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_local = ev0.elapsed_time(ev1)
    ms = ranks_reduce(ms_local, "max", world, "cuda")
    value = whole_job_rate(upd_local * args.steps, ms_local * 1e-3, world, "cuda")

    # per-kernel times: CUDA events on the solver's stream around every
    # launch of K more iterations launched kernel by kernel (after the timed
    # region)
    solver.set_profile(True)
    kst = solver.solve(max_iter=args.steps, err_temp=0.0, err_flux=0.0)
    solver.set_profile(False)
    torch.cuda.synchronize()
    kern = kst["kernels"]
    peak, peak_kind = measured_peak_gbs()
    total_ms = sum(v["ms"] for v in kern.values())
    dim = 2 if deck.mesh.nodes.shape[1] == 2 else 3
    nnz = macro_nnz(deck)
    traffic_per_update = NCU_TRAFFIC_PER_UPDATE.get((args.workload, args.precision), {})

    def kernel_roofline(name):
        k = kern[name]
        per_launch_ms = k["ms"] / k["launches"]
        launches_per_step = k["launches"] / args.steps
        alg = kernel_algorithmic_bytes(name, s_bytes, dim, nb, nd, nc, nnz)
        if alg and name in ("gradient", "residual", "sweep", "moments"):
            alg = alg / launches_per_step  # direction batches: one launch covers a batch
        achieved = alg / (per_launch_ms * 1e-3) / 1e9 if alg else None
        tr = traffic_per_update.get(name)
        return {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": tr * upd_per_step / launches_per_step if tr else None, "algorithmic_bytes": alg,
                "launch_ms": per_launch_ms, "kernel_share": k["ms"] / total_ms}

    # the whole outer iteration against HBM: 3 s algorithmic bytes per
    # band*direction*cell update (read e for gradient and residual, write
    # the sweep's update, read e for the moments pass)
    ms_step = ms / args.steps
    alg_step = 3 * s_bytes * upd_per_step
    achieved = alg_step / (ms_step * 1e-3) / 1e9
    tr_step = sum(traffic_per_update.values()) * upd_per_step if traffic_per_update else None
    dname = max(kern.items(), key=lambda kv: kv[1]["ms"])[0]
    roofline = {"kernel": "outer iteration (transport stage replayed as one CUDA graph + macro correction)",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind, "traffic": tr_step, "algorithmic_bytes": alg_step,
                "bytes_per_update": 3 * s_bytes, "launch_ms": ms_step, "dominant_kernel": dname,
                "dominant_kernel_share": kern[dname]["ms"] / total_ms}
    hbm_kernels = {n: kernel_roofline(n) for n in ("residual", "sweep", "gradient", "moments") if n in kern}
    kernel_table = {k: {"ms_per_launch": v["ms"] / v["launches"], "launches": v["launches"],
                        "share": v["ms"] / total_ms} for k, v in kern.items()}

    # end to end through the public API
    if args.workload == "config3":
        e2e = e2e_iterations(args, solver, deck, world)
        ttr = None
        solver.close()
    else:
        solver.close()
        e2e, ttr = e2e_solves(args, deck, prec, local_rank, world, rank if by_dirs else None)

    out = None
    if rank == 0:
        fp64 = None
        if args.compare_fp64 and prec == g.GBTE_FP32_MIXED:
            if args.workload == "config3" and not args.time_to_residual:
                fp64 = fp64_rate_run(args, deck, local_rank, value)
            else:
                fp64 = fp64_reference_run(args, deck, local_rank)
        cpu = cpu_baseline(args, deck) if world == 1 else None
        cfg = workload_config(args, deck, desc, nb, nd)
        cfg.update({"cell_order": "morton" if args.cell_order == 0 else "deck",
                    "parallelism": (f"direction shards x{world} of one problem (NCCL all-reduce of the moments "
                                    "and boundary values every outer iteration)" if by_dirs and world > 1 else
                                    f"replicas x{world} (independent seeded problems)" if world > 1 else "1 GPU")})
        out = {
            "metric": METRIC,
            "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong" if by_dirs else "weak", "vs_baseline": None,
            "dtype": "f32" if prec == g.GBTE_FP32_MIXED else "f64",
            "data": "synthetic: seeded mesh and band table generated in-process (no dataset)",
            "config": cfg,
            "tuning": {"sweep_bands": st.get("sweep_bands"), "sweep_stage_levels": st.get("sweep_stage_levels"),
                       "sweep_vector": st.get("sweep_vector"), "sweep_threads": st.get("sweep_threads"),
                       "sweep_kernel": {1: "block", 2: "warp", 3: "wide"}.get(st.get("sweep_kernel")),
                       "gradient_dirs": st.get("gradient_dirs"), "residual_form": st.get("residual_form"),
                       "direction_batch": st.get("direction_batch")},
            "roofline": roofline, "hbm_kernels": hbm_kernels, "kernels": kernel_table, "cpu_baseline": cpu,
            "e2e": e2e, "time_to_residual": ttr, "gpu_launches": int(st["kernel_launches"]), "clocks": clk,
            "macro": {"ms_per_step": st["macro_ms"] / args.steps, "cg_iterations": st["macro_cg_iterations"]},
            "setup_s": setup_s,
        }
        if fp64 is not None:
            out["fp64"] = fp64
    return out


def ctypes_stream(stream) -> int:
    return int(stream.cuda_stream)


def attach_shard(solver, rank: int, world: int) -> int:
    """Give the solver rank's block of directions, exchanging over the
    default process group (NCCL); one rank holds every direction and its
    exchange is the identity. Returns the block's size."""
    from giftbte_b200 import shard

    b, n = shard.direction_blocks(solver.num_directions, world)[rank]
    ex = shard.torch_exchange() if world > 1 else (lambda buf, count, stream: None)
    solver.set_direction_shard(b, n, ex)
    return n


def pinned_fields(nc, nb):
    """Pinned host arrays for StaticBTESynthetic.fields(out=...): the
    read-back of every field copies straight into page-locked memory."""
    import torch

    return {k: torch.empty(shp, dtype=torch.float64).pin_memory().numpy()
            for k, shp in (("E", (nc,)), ("T", (nc,)), ("q", (nc, 3)), ("Tband", (nb, nc)))}


def e2e_iterations(args, solver, deck, world):
    """End to end through the public API on a handle already created: the
    initial field from pinned host memory (gbte_set_initial), K outer
    iterations (gbte_solve_with), every result field read back
    (gbte_get_fields) into pinned host arrays, repeated e2e_steps times;
    updates/s over the wall time of the calls."""
    import torch

    nc = deck.mesh.n_cells
    nb = solver.num_bands
    T0 = torch.full((nc,), float(deck.tref), dtype=torch.float64).pin_memory().numpy()
    out = pinned_fields(nc, nb)
    reps = max(1, args.e2e_steps)
    times, ups = [], []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solver.set_initial(T0)
        st = solver.solve(max_iter=args.steps, err_temp=0.0, err_flux=0.0)
        solver.fields(out=out)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        ups.append(st["updates"])
    return {"value": whole_job_rate(sum(ups), sum(times), world, "cuda"), "unit": "updates/s",
            "h2d_bytes_per_step": int(nc * 8 / args.steps),
            "d2h_bytes_per_step": int(nc * 8 * (2 + 3 + nb) / args.steps), "steps": args.steps * reps,
            "step": f"set_initial from pinned host + {args.steps} outer iterations + read all fields, x{reps}; "
                    "bytes per step are the call's copies over its iterations"}


def fp64_rate_run(args, deck, device, fp32_value):
    """The plain FP64 GPU form on the same 3D block: device updates/s over a
    few outer iterations after warm-up (time to residual 1e-8 of both forms
    is measured separately: it takes hundreds of iterations)."""
    import torch

    import giftbte_b200 as g

    k = max(1, min(args.steps, args.fp64_steps))
    stream = torch.cuda.Stream()
    s = g.StaticBTESynthetic.from_deck(deck, precision=g.GBTE_FP64, device=device, stream=ctypes_stream(stream),
                                       cell_order=args.cell_order)
    s.solve(max_iter=2, err_temp=0.0, err_flux=0.0)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    st = s.solve(max_iter=k, err_temp=0.0, err_flux=0.0)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    s.close()
    v = st["updates"] / (ms * 1e-3)
    return {"fp64": {"updates_per_s": v, "ms_per_step": ms / k, "steps": k,
                     "direction_batch": st.get("direction_batch"), "gradient_dirs": st.get("gradient_dirs"),
                     "sweep_kernel": {1: "block", 2: "warp", 3: "wide"}.get(st.get("sweep_kernel"))},
            "fp32_over_fp64_per_iteration": fp32_value / v}


def e2e_solves(args, deck, prec, device, world, shard_rank=None):
    import torch

    import giftbte_b200 as g

    nc = deck.mesh.n_cells
    solver = g.StaticBTESynthetic.from_deck(deck, precision=prec, device=device, max_iter=args.max_iter_e2e,
                                            err_temp=1e-8, err_flux=1e-8, cell_order=args.cell_order,
                                            sweep_bands=args.sweep_bands, sweep_vector=args.sweep_vector,
                                            sweep_kernel=args.sweep_kernel)
    nb = solver.num_bands
    if shard_rank is not None:
        attach_shard(solver, shard_rank, world)
    T0 = torch.full((nc,), float(deck.tref), dtype=torch.float64).pin_memory().numpy()
    out = pinned_fields(nc, nb)
    nsteps = max(2, min(args.steps, max(2, args.e2e_steps)))
    times, iters, ups = [], [], []
    for _ in range(nsteps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solver.set_initial(T0)
        st = solver.solve()
        solver.fields(out=out)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        iters.append(st["iterations"])
        ups.append(st["updates"])
    solver.close()
    t = max(times)
    e2e = {"value": whole_job_rate(sum(ups), sum(times), world, "cuda"), "unit": "updates/s",
           "h2d_bytes_per_step": int(nc * 8), "d2h_bytes_per_step": int(nc * 8 * (2 + 3 + nb)),
           "steps": nsteps, "step": "set_initial from pinned host + solve to residual 1e-8 + read all fields"}
    ttr = {"seconds": float(np.median(times)), "iterations": int(np.median(iters)), "residual": 1e-8,
           "precision": "fp32" if prec == g.GBTE_FP32_MIXED else "fp64"}
    return e2e, ttr


def fp64_reference_run(args, deck, device):
    """The plain FP64 GPU form on the same workload: time to residual 1e-8
    of both forms from the same uniform start (clocks sampled during each
    solve) and the FP32 form's temperature error against it."""
    import torch

    import giftbte_b200 as g

    res = {}
    fields = {}
    forms = [f for f in args.ttr_forms.split(",") if f]
    for prec, name in ((g.GBTE_FP64, "fp64"), (g.GBTE_FP32_MIXED, "fp32")):
        if name not in forms:
            continue
        s = g.StaticBTESynthetic.from_deck(deck, precision=prec, device=device, max_iter=args.max_iter_e2e,
                                           err_temp=1e-8, err_flux=1e-8, cell_order=args.cell_order)
        torch.cuda.synchronize()
        clocks = ClockSampler(device)
        clocks.start()
        t0 = time.perf_counter()
        st = s.solve(allow_not_converged=True)
        torch.cuda.synchronize()
        res[name] = {"seconds": time.perf_counter() - t0, "iterations": st["iterations"],
                     "converged": bool(st["err_temp"] <= 1e-8 and st["err_flux"] <= 1e-8),
                     "updates_per_s": st["updates"] / (st["solve_ms"] * 1e-3), "clocks": clocks.stop()}
        fields[name] = s.fields()
        s.close()
    if "fp64" in fields and "fp32" in fields:
        T64, T32 = fields["fp64"]["T"], fields["fp32"]["T"]
        res["fp32_T_max_rel_err"] = float(np.max(np.abs(T32 - T64)) / np.max(np.abs(T64)))
        res["fp32_speedup_time_to_residual"] = res["fp64"]["seconds"] / res["fp32"]["seconds"]
    return res


def cpu_sample_deck(args, deck):
    """The bounded CPU sample of a workload: the 2D cell itself; for the 3D
    block, a 50 x 50 x 5 nm piece of it (same spacing, jitter, bands and
    directions; 4,800 tets, 1/400 of the block), whose per-update rate
    stands for the block's."""
    if args.workload != "config3":
        return deck, "the same deck"
    from giftbte_b200 import decks

    h = args.h_nm or 2.5
    d = decks.config3_deck(h_nm=h, size_nm=(50.0, 50.0, 5.0), seed=1)
    return d, (f"a 50 x 50 x 5 nm piece of the block at h = {h} nm ({d.mesh.n_cells} tets), same bands and "
               "directions")


def timed_port_iterations(deck, warm: int, k: int) -> float:
    """Seconds per outer iteration of the oracle port (multithreaded FP64
    CPU restatement): the difference of a (warm + k)- and a warm-iteration
    run over k."""
    import oracle

    t = []
    for n in (warm, warm + k):
        t0 = time.perf_counter()
        oracle.solve(deck, max_iter=n, err_T=0.0, err_q=0.0)
        t.append(time.perf_counter() - t0)
    return max(t[1] - t[0], 1e-9) / k


def cpu_baseline(args, deck):
    """The oracle restatement (multithreaded FP64 CPU port) timed on the
    host cores on a bounded sample: one outer iteration of the workload's
    CPU sample, measured as the difference of a 2-iteration and a
    1-iteration run."""
    if args.skip_cpu:
        return None
    try:
        sample, what = cpu_sample_deck(args, deck)
        per_iter = timed_port_iterations(sample, 1, 1)
        upd = sample.bands.n_bands * directions_of(sample) * sample.mesh.n_cells
        return {"value": upd / per_iter, "unit": "updates/s", "cores": os.cpu_count(), "kind": "port",
                "sample": f"one outer iteration of {what} (difference of 2- and 1-iteration runs)"}
    except Exception as e:  # the baseline must not take the GPU line down
        return {"value": None, "unit": "updates/s", "cores": os.cpu_count(), "kind": "port",
                "sample": f"failed: {e}"}


def run_reference(args, rank: int):
    """The reference's own CPU implementation of the path on the host cores,
    for the same metric and config as the GPU arm, W warm-up and K timed
    outer iterations. 2D decks: the unmodified compiled reference (1 MPI
    rank through the single-rank stub build), timed from its own
    per-iteration 'Time taken by inner loop' trace. The 3D block: the
    reference's public release cannot read 3D meshes, so the oracle port
    (its algorithm restated, multithreaded FP64) on the bounded sample of
    cpu_sample_deck stands in, labelled kind 'port'."""
    if rank != 0:
        return None
    import oracle

    deck, desc = build_deck(args.workload, seed=0, h_nm=args.h_nm, height_nm=args.height_nm)
    nb = deck.bands.n_bands
    nd = directions_of(deck)
    upd = nb * nd * deck.mesh.n_cells
    k = max(1, args.steps)
    w = max(0, args.warmup)
    base = {"impl": "reference", "metric": METRIC, "unit": "updates/s", "higher_is_better": True, "n_gpus": 1,
            "steps": k, "warmup": w, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded mesh and band table generated in-process (no dataset)",
            "config": workload_config(args, deck, desc, nb, nd)}
    if args.workload == "config3" or not os.path.exists(oracle.REF_BIN):
        sample, what = cpu_sample_deck(args, deck)
        per_iter = timed_port_iterations(sample, max(1, w), k)
        s_upd = sample.bands.n_bands * directions_of(sample) * sample.mesh.n_cells
        value = s_upd / per_iter
        why = ("the reference cannot read 3D meshes (its public release has no 3D mesh code)"
               if args.workload == "config3" else "the reference binary was not built")
        base.update({"value": value, "ms_per_step": upd / value * 1e3,
                     "cpu_baseline": {"value": value, "unit": "updates/s", "cores": os.cpu_count(), "kind": "port",
                                      "sample": f"{k} outer iterations of {what} after {max(1, w)} warm-up "
                                                f"(difference of two runs); {why}, so the CPU restatement of its "
                                                "algorithm is timed"},
                     "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return base
    work = tempfile.mkdtemp(prefix="gbte_ref_")
    try:
        deck.max_iter = w + k
        deck.residual_temp = 0.0
        deck.residual_flux = 0.0
        deck.write(work)
        t0 = time.perf_counter()
        with open(os.path.join(work, "ref_run.log"), "w") as log:
            subprocess.run([oracle.REF_BIN], cwd=work, stdout=log, stderr=subprocess.STDOUT, check=True,
                           timeout=args.ref_timeout)
        wall = time.perf_counter() - t0
        with open(os.path.join(work, "ref_run.log")) as f:
            inner = [float(line.split(":")[1].split()[0]) for line in f if "Time taken by inner loop" in line]
    finally:
        shutil.rmtree(work, ignore_errors=True)
    timed = inner[w:w + k] if len(inner) >= w + k else inner[-k:]
    sec = float(np.mean(timed)) * 1e-3
    value = upd / sec
    base.update({"value": value, "ms_per_step": sec * 1e3,
                 "cpu_baseline": {"value": value, "unit": "updates/s", "cores": 1, "kind": "reference",
                                  "sample": f"{len(timed)} outer iteration(s) of the same deck after "
                                            f"{w} warm-up; wall {wall:.1f} s incl. the reference's setup"},
                 "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return base


def _population_one(i: int, seed: int):
    """Cell i of the seeded config-5 population (built in a worker process)."""
    from giftbte_b200 import decks

    return decks.porous_population_member(i, seed=seed)


def run_config4(args, rank: int):
    """Adjoint workload: the config-2 cell with a partially specular pore
    wall (p = 0.3) and log-normal per-cell scattering multipliers (sigma 0.2,
    seed 2), 40 bands, 64 directions, FP64. The forward solve runs to the
    given residual from the Fourier pre-solve; then gbte_vjp gives the
    gradient of k_x with respect to the 40 band tau multipliers, every cell's
    multiplier and p. Reported: the adjoint's device time against the
    forward's (the target is <= 2x) and both iteration counts."""
    import torch

    import giftbte_b200 as g
    from giftbte_b200 import decks

    torch.cuda.init()
    d = decks.config4_deck(h_nm=3.0, n_bands=40, n_phi=16, seed=0, specularity=0.3)
    nc = d.mesh.n_cells
    sc = decks.lognormal_scatter(nc, sigma=0.2, seed=2)
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64, cell_scatter=sc, max_iter=args.adj_max_iter)
    # the forward starts from the Fourier pre-solve, as the reference's runs
    # do; the adjoint starts from lam = 0
    s.fourier_initial()
    clocks = ClockSampler(0)
    clocks.start()
    st = s.solve(err_temp=args.adj_residual, err_flux=args.adj_residual, max_iter=args.adj_max_iter)
    qb = s.keff_cotangent(axis=0, length=300e-9, delta_T=1.0)
    a = s.vjp(q_bar=qb, tol=args.adj_residual, max_iter=args.adj_max_iter)
    clk = clocks.stop()
    keff = float(np.sum(qb * s.fields()["q"]))
    nb, nd = s.num_bands, s.num_directions
    s.close()
    fwd_ms, adj_ms = st["solve_ms"], a["stats"]["vjp_ms"]
    adj_updates = a["stats"]["iterations"] * nb * nd * nc
    return {
        "metric": "adjoint band*dir*cell updates/s (gradient of k_x; adjoint time over forward time alongside)",
        "value": adj_updates / (adj_ms * 1e-3), "unit": "updates/s", "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": adj_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded mesh, band table and multiplier field generated in-process (no dataset)",
        "config": {"workload": f"config-2 cell with a partially specular pore wall p=0.3, log-normal cell "
                               f"scattering multipliers sigma 0.2 seed 2 ({nc} triangles), 40 bands, 64 directions",
                   "residual": args.adj_residual, "objective": "k_x"},
        "forward": {"ms": fwd_ms, "iterations": st["iterations"]},
        "adjoint": {"ms": adj_ms, "iterations": a["stats"]["iterations"], "residual": a["stats"]["residual"],
                    "change": a["stats"]["change"], "picard_steps": a["stats"]["picard_steps"],
                    "stop": "||(dF/de)^T lam + dJ/de|| / ||dJ/de|| <= residual"},
        "adjoint_over_forward": adj_ms / fwd_ms, "k_x": keff,
        "grad_norms": {"tau": float(np.linalg.norm(a["tau"])), "scatter": float(np.linalg.norm(a["scatter"])),
                       "specularity": float(a["specularity"][[b.tag for b in d.bcs].index(5)])},
        "gpu_launches": int(st["kernel_launches"]), "clocks": clk,
    }


def run_config5(args, rank: int):
    """Batched solve of 256 independent porous cells (one handle over their
    disjoint union: one launch per kernel stage for all cells, the sweep's
    launch geometry picked by the autotuner) against the same cells solved
    one after another with the plain FP64 form, both for K outer iterations
    after W warm-up iterations; device time from CUDA events / solve stats."""
    import multiprocessing as mp

    n = args.batch
    # meshes are built in spawned workers, before this process touches CUDA
    with mp.get_context("spawn").Pool(min(n, max(1, (os.cpu_count() or 2) - 1))) as pool:
        pop = pool.starmap(_population_one, [(i, 5) for i in range(n)])
    import torch

    import giftbte_b200 as g

    torch.cuda.init()
    cells = [d.mesh.n_cells for d in pop]
    nb, nd = pop[0].bands.n_bands, 4 * pop[0].n_phi
    upd = nb * nd * sum(cells)
    b = g.StaticBTESynthetic.from_decks(pop, precision=g.GBTE_FP32_MIXED, cell_order=args.cell_order)
    b.solve(max_iter=args.warmup, err_temp=0.0, err_flux=0.0)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    st = b.solve(max_iter=args.steps, err_temp=0.0, err_flux=0.0)
    clk = clocks.stop()
    batch_ms = st["solve_ms"]
    b.close()
    seq_ms = 0.0
    for d in pop:
        s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64, cell_order=args.cell_order)
        s.solve(max_iter=args.warmup, err_temp=0.0, err_flux=0.0)
        seq_ms += s.solve(max_iter=args.steps, err_temp=0.0, err_flux=0.0)["solve_ms"]
        s.close()
    value = upd * args.steps / (batch_ms * 1e-3)
    seq = upd * args.steps / (seq_ms * 1e-3)
    return {
        "metric": "band*dir*cell updates/s, batched solve of independent cells vs sequential plain FP64 solves",
        "value": value, "unit": "updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": batch_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic: seeded porous cells generated in-process (no dataset)",
        "config": {"workload": f"{n} periodic 300 nm cells, 1-3 pores r~U(40,120) nm, h~U(2,6) nm, seed 5; "
                               f"20 bands, 32 directions", "cells_total": sum(cells),
                   "cells_min": min(cells), "cells_max": max(cells), "updates_per_step": upd,
                   "parallelism": "1 GPU, one batched handle"},
        "sequential_fp64": {"value": seq, "unit": "updates/s", "ms_per_step": seq_ms / args.steps,
                            "note": "the same cells solved one after another with the plain FP64 form "
                                    "(device time of their outer iterations)"},
        "batch_over_sequential": value / seq, "sweep_bands_autotuned": st.get("sweep_bands"),
        "sweep_vector_autotuned": st.get("sweep_vector"), "sweep_threads_autotuned": st.get("sweep_threads"),
        "sweep_kernel_autotuned": {1: "block", 2: "warp", 3: "wide"}.get(st.get("sweep_kernel")),
        "gpu_launches": int(st["kernel_launches"]), "clocks": clk,
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--workload", choices=["config3", "config2", "config1", "config4", "config5"], default="config3")
    ap.add_argument("--adj-residual", type=float, default=1e-8, help="config4: forward margins and adjoint tolerance")
    ap.add_argument("--adj-max-iter", type=int, default=20000, help="config4: adjoint iteration cap")
    ap.add_argument("--batch", type=int, default=256, help="config5: number of independent cells")
    ap.add_argument("--h-nm", type=float, default=0.0, help="config3 mesh spacing (default 2.5 nm)")
    ap.add_argument("--height-nm", type=float, default=500.0,
                    help="config3 block height (default 500 nm; smaller blocks for profiling captures)")
    ap.add_argument("--sweep-bands", type=int, default=0,
                    help="bands per sweep CTA (1..32); 0 lets the autotuner pick on the first iteration")
    ap.add_argument("--sweep-vector", type=int, choices=[0, 1, 2, 4], default=0,
                    help="bands per sweep thread; 0 lets the autotuner pick")
    ap.add_argument("--sweep-kernel", type=int, choices=[0, 1, 2, 3], default=0,
                    help="1: block sweep kernel, 2: warp-independent kernel, 3: wide-level kernel, "
                         "0: the autotuner's pick")
    ap.add_argument("--gradient-dirs", type=int, choices=[0, 1, 2, 4, 5, 6, 7, 8, 9, 10], default=0,
                    help="gradient launch shape (options.gradient_dirs); 0 lets the first iteration pick")
    ap.add_argument("--residual-form", type=int, choices=[0, 1, 5, 6, 7, 8], default=0,
                    help="residual launch shape (options.residual_form); 0 lets the first iteration pick")
    ap.add_argument("--cell-order", type=int, choices=[0, 1], default=0,
                    help="0: cells renumbered along a Morton curve inside the library; 1: the deck's order")
    ap.add_argument("--e2e-steps", type=int, default=1,
                    help="repetitions of the end-to-end call sequence (2D: solves to 1e-8, at least 2, at most K)")
    ap.add_argument("--max-iter-e2e", type=int, default=2000)
    ap.add_argument("--fp64-steps", type=int, default=5, help="3D block: timed outer iterations of the FP64 form")
    ap.add_argument("--time-to-residual", action="store_true",
                    help="3D block: also solve to residual 1e-8 in both forms (tens of minutes at full size)")
    ap.add_argument("--ref-timeout", type=float, default=1500.0)
    ap.add_argument("--ttr-forms", default="fp64,fp32",
                    help="with --time-to-residual: the forms solved to 1e-8 (comma-separated fp64, fp32)")
    ap.add_argument("--no-fp64", dest="compare_fp64", action="store_false")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--shard", choices=["replicas", "directions"], default="replicas",
                    help="N > 1: a seeded cell per rank (weak scaling), or one cell's directions split over "
                         "the ranks (strong scaling)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if args.workload == "config5":
        if rank == 0:
            print(json.dumps(run_config5(args, rank)), flush=True)
        return
    if args.workload == "config4":
        if rank == 0:
            print(json.dumps(run_config4(args, rank)), flush=True)
        return
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        out = run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
