#!/usr/bin/env python
"""Benchmark of the NIM time advance: cell-iterations/s on the cylinder case.

A step is one time step of the reference's solve_nse loop (nse.f90:47-75) on
the 128x128x96 cylinder/hexagon mesh (Ra=1e5, Pr=0.71, dt=5e-4, FP64):
calculate_velocity_nim_constants, the integrate_nse inner loop to the
reference tolerances, update_time_step and find_Nu2.  The metric counts
cells x inner iterations per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun with one GPU per rank and splits ONE enclosure
over the ranks: the 256x256x192 cylinder (Ra=1e6, Pr=0.71, dt=2.5e-4) cut
into N z-slabs (nimgpu.SlabRank: each rank holds its slab plus two halo
planes per neighbour; after the velocity, pressure and temperature parts of
every pass the halo planes move to the neighbours over NCCL, and the
find_error maxima are all-reduced before each pass end).  Strong scaling:
the job value is the mesh's cell-iterations over the slowest rank's device
time.  --replicas instead gives every rank its own copy of the --case mesh
(no data crosses ranks; the job value sums the ranks' work).

--impl reference times the reference algorithm's CPU implementation (the
oracle port of the Fortran, OpenMP threads as the reference uses them) on
the host cores on the same workload, one inner iteration per step.

--case batch times the batched extension instead: 64 seeded enclosures of
uneven size (a x a x 0.75a cells, a in [24, 64]) and Ra, Pr advanced
together, every pass kernel launched once for all of them
(nim_batch_step_fused; also as 64 streams, nim_batch_step), against the
same 64 cases run one at a time.

On one GPU the line also carries "mixed": the same steps from the same
start with nim_params.precision = NIM_PRECISION_MIXED (FP32 passes, then
FP64 passes to the reference's stop test), its throughput, its roofline and
its per-step Nusselt and final field errors against the FP64 run.
--precision mixed makes the mixed path the headline arm instead.

It also carries "slabs": the same steps from the same start with the mesh
split into two z-slabs on the one device (nim_slab_step: halo exchange after
each part of every pass), their throughput against the whole mesh and
whether iterations and final fields match the whole-mesh run exactly.

--tangent adds "tangent": the same steps on the tangent-linear path
(nim_gpu_tangent_*, d/dRa seeded), its throughput against the FP64 run,
whether its values repeat that run's, and d Nu_hot / dRa per step.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
# concurrent kernels of many contexts need more hardware queues than the
# default 8 (read once, when the CUDA context is created)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
sys.path.insert(0, str(ROOT / "nim-conv22-shared_b200"))

import numpy as np  # noqa: E402

CASE = "c2"
METRIC = "NIM cell-iterations/s"
UNIT = "cell-iterations/s"

# Algorithmic HBM bytes of each kernel per cell and pass (FP64 doubles x 8):
# the data the kernel must read and write once with structured connectivity
# (faces counted as 3 per cell; geometry and coefficients as stored).
KERNEL_BYTES_PER_CELL = {
    "k_vel_cell": 8 * 53,   # faces p,u,v,w (12) T,T_old (2) area,normal,vol (13) G,g^ij (9) cells+old (6) M_F4 (8); write u,v,w (3)
    "k_vel_face": 8 * 45,   # faces u,v,w (9) cells+old (6) M_F1..3 (15) dg (6); write faces (9)
    "k_vel_face_tile": 8 * 45,  # the same sweep staged by TMA boxes (same algorithmic bytes)
    "k_vel_cell_tile": 8 * 53,  # k_vel_cell with its u, v, w faces staged by TMA boxes
    "k_vel_cell2": 8 * 53,  # k_vel_cell on cell pairs with paired loads (same algorithmic bytes)
    "k_vel_cellN": 8 * 53,  # the float mirror's form: four cells a thread (same words; the mixed line halves them)
    "k_p_src": 8 * 39,      # faces u,v,w,T,p (15) area,normal,vol (13) G,g^ij (9); write dila,Rp (2)
    "k_p_srcN": 8 * 39,     # the float mirror's form: four cells a thread (same words)
    "k_T_cellN": 8 * 48,    # the float mirror's form of k_T_cell (same words)
    "k_p_faceN": 8 * 52,    # the float mirror's form of k_p_face (same words)
    "k_T_faceN": 8 * 29,    # the float mirror's form of k_T_face (same words)
    "k_vel_faceN": 8 * 45,  # the float mirror's form of k_vel_face (same words)
    "k_p_face": 8 * 52,     # faces p (3) Rp (1) AA used (39) dg (6); write faces p (3)
    "k_T_coef": 8 * 42,     # cells+old u,v,w (6) xi (9) g^ij diagonal (3) gfd (6); write MT_A (18)
    "k_T_cell": 8 * 48,     # MT_A (18) faces T (3) G (3) g^ij (6) T,T_old (2); write T, MT_F (16)
    "k_T_face": 8 * 29,     # faces T (3) T,T_old (2) MT_F (15) dg (6); write faces T (3)
    # the reference-order sweeps (--schedule reference), in place
    "k_seq_vel": 8 * 59,    # cells+old u,v,w (6) faces u,v,w (9) M_F4 (8) R sums (3) M_F1..3 (15) dg (6); write cells, faces (12)
    "k_seq_p": 8 * 52,      # faces p (3) R_p (1) AA used (39) dg (6); write faces p (3)
    "k_seq_T": 8 * 39,      # T,T_old (2) faces T (3) MT_F4 (8) R_D_T (1) MT_F (15) dg (6); write T, faces (4)
}
# DRAM bytes per cell and launch that ncu measured (dram__bytes_read.sum +
# dram__bytes_write.sum, one --set full capture each); traffic grows with the
# cells, so roofline.traffic scales these to the run's mesh
NCU_DRAM_BYTES_PER_CELL = {
    "k_vel_cell": 425.2, "k_p_src": 324.4, "k_p_face": 420.2, "k_T_coef": 276.9, "k_T_cell": 389.6,
    "k_T_face": 227.3, "k_vel_face_tile": 361.4, "k_vel_face": 343.1, "k_vel_cell2": 441.0,
}
NCU_CAPTURE = {k: "128x128x96" for k in NCU_DRAM_BYTES_PER_CELL}
for _k in ("k_vel_face", "k_vel_cell2", "k_T_coef"):
    NCU_CAPTURE[_k] = "96x96x64"
# algorithmic bytes per cell-iteration and per cell-step of the whole pass
# (FP64, every array read and written once, implicit connectivity)
ALGO_BYTES_PER_CELL_ITER = 1880
ALGO_BYTES_PER_CELL_STEP = 776


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.idx), "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        loaded = [s for s in sm if s > 0.3 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------ helpers
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def cpu_sample(case, threads: int, iters: int, schedule: int):
    """Time `iters` inner iterations of the oracle (the reference's algorithm
    on the CPU) on the same mesh; returns (cell-iterations/s, seconds)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    mesh = O.OracleMesh(case.mesh_params())
    o = O.Oracle(mesh, case.params(), schedule=schedule, threads=os.cpu_count() or 1)
    o.init()  # geometry set-up on all cores, not timed
    o.set_threads(threads)
    o.add_temperature_noise(case.noise, case.seed)
    o.begin_step()
    o.iterate(1)  # warm
    t = time.perf_counter()
    o.iterate(iters)
    dt = time.perf_counter() - t
    o.close()
    return case.ncells * iters / dt, dt


def combine_ranks(pg, t, work, device="cuda"):
    """Replicas on N ranks: the job takes as long as its slowest rank and
    does the sum of the ranks' work.  pg is torch.distributed (or None for
    one rank); device is where the reduction tensors live (cuda for nccl,
    cpu for gloo)."""
    if pg is None:
        return t, work
    import torch
    tt = torch.tensor([float(t)], dtype=torch.float64, device=device)
    pg.all_reduce(tt, op=pg.ReduceOp.MAX)
    ww = torch.tensor([float(work)], dtype=torch.float64, device=device)
    pg.all_reduce(ww, op=pg.ReduceOp.SUM)
    return float(tt.item()), float(ww.item())


def host_cpu():
    """Model name and logical CPU count of the host the CPU arms run on."""
    model = None
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


def run_reference(args, rank, world):
    """--impl reference: the reference algorithm (the oracle port of the
    Fortran, the checker) on all host cores, with the oracle's own mesh
    builder and noise (no product library is loaded).  The timed unit is
    one inner pass of step 1 (the loop body nse.f90:131-160); the per-step
    work (velocity NIM constants, update_time_step, find_Nu2) is timed
    once on its own and reported beside it."""
    if rank != 0:
        return 0
    from nimgpu import config  # pure Python: case definitions only
    case = config.CASES[args.case]
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    mesh = O.OracleMesh(case.mesh_params())
    o = O.Oracle(mesh, case.params(), schedule=O.SEQUENTIAL, threads=threads)
    o.init()
    o.add_temperature_noise(case.noise, case.seed)
    t = time.perf_counter()
    o.begin_step()
    t_begin = time.perf_counter() - t
    for _ in range(args.warmup):
        o.iterate(1)
    t = time.perf_counter()
    for _ in range(args.steps):
        o.iterate(1)
    dt = time.perf_counter() - t
    t = time.perf_counter()
    o.end_step()
    t_end = time.perf_counter() - t
    o.close()
    value = case.ncells * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "timed_unit": "one inner pass (nse.f90:131-160) of step 1 per timed step",
        "per_step_work_ms": 1e3 * (t_begin + t_end),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(case),
        "host_cpu": host_cpu(),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} inner passes of step 1 on {args.case} "
                                   f"({case.ncells} cells), reference cell order, OpenMP threads={threads}; "
                                   f"per-step work {1e3 * (t_begin + t_end):.0f} ms timed apart"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(case):
    return {"workload": f"{case.name}: cylinder D=1 H=1, hexagon side 0.2, {case.n_theta}x{case.n_r}x{case.n_z} "
                        f"O-grid (tanh 1.5), Ra={case.Ra:g} Pr={case.Pr:g} dt={case.dt:g}",
            "cells": case.ncells, "Ra": case.Ra, "Pr": case.Pr, "dt": case.dt,
            "parallelism": "replicas", "l2": "working set > L2 (126 MB): ~3 GB read per pass"}


SLAB_CASE = "c3"


def run_slab_ranks(args, rank, world, local):
    """--gpus N > 1: one enclosure split into N z-slabs, one per rank
    (nimgpu.SlabRank over NCCL).  Every rank runs the same collective
    sequence; the timed region is bracketed by a barrier and a device
    synchronisation, and its length is the maximum over the ranks."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import nimgpu
    from nimgpu import config, _abi

    torch.cuda.set_device(local)
    if "MASTER_ADDR" not in os.environ:  # one rank without torchrun (--decompose at N=1)
        import socket
        sock = socket.socket()
        sock.bind(("127.0.0.1", 0))
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(sock.getsockname()[1]), RANK="0",
                          WORLD_SIZE="1")
        sock.close()
    dist.init_process_group("nccl", timeout=timedelta(seconds=180), device_id=torch.device("cuda", local))
    case = config.CASES[args.case if args.case != CASE else SLAB_CASE]
    mesh = nimgpu.Mesh(case.mesh_params())
    r = nimgpu.SlabRank(mesh, case.params())
    passes = 8
    try:
        r.initialize_nse()
        r.add_temperature_noise(case.noise, case.seed)
        h = r._h[0]
        for _ in range(max(args.warmup, 0)):
            r.solve_nse(1, passes_per_check=passes)
        dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = int(r.lib.nim_gpu_launch_count(h))
        ev0.record(r.stream)
        stats = r.solve_nse(args.steps, passes_per_check=passes)
        ev1.record(r.stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        clk = clocks.stop()
        launches = int(r.lib.nim_gpu_launch_count(h)) - launches0
        ms = ev0.elapsed_time(ev1)
        iters = sum(x.iters for x in stats)
        t_max, _ = combine_ranks(dist, ms, 0)
        total = case.ncells * iters  # one mesh: every rank reports the same iterations
        value = total / (t_max / 1e3)
        launches_all = combine_ranks(dist, 0.0, launches)[1]

        # end to end: every step each rank uploads its slab's restart arrays
        # from page-locked host memory, advances one step and downloads them
        fields = [_abi.FACES_U, _abi.FACES_V, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T,
                  _abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T,
                  _abi.MESHES_U_OLD, _abi.MESHES_V_OLD, _abi.MESHES_W_OLD, _abi.MESHES_T_OLD,
                  _abi.MESHES_UT, _abi.MESHES_VT, _abi.MESHES_WT]
        host = {f: torch.empty(r.field_size(rank, f), dtype=torch.float64).pin_memory() for f in fields}
        for f in fields:
            r.download(rank, f, out=host[f].numpy())
        h2d = sum(x.numel() * 8 for x in host.values())
        e2e_steps = max(2, args.steps // 2)
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_iters = 0
        for _ in range(e2e_steps):
            for f in fields:
                r.upload(rank, f, host[f].numpy())
            st = r.solve_nse(1, passes_per_check=passes)
            e2e_iters += sum(x.iters for x in st)
            for f in fields:
                r.download(rank, f, out=host[f].numpy())
        torch.cuda.synchronize()
        e2e_s, h2d_all = combine_ranks(dist, time.perf_counter() - t0, h2d)
        e2e_value = case.ncells * e2e_iters / e2e_s
        peak, peak_kind = peaks()
        per_gpu = ALGO_BYTES_PER_CELL_ITER * total / (t_max / 1e3) / 1e9 / world
        nt, nr = mesh.n_theta, mesh.n_r
        halo_doubles = ({name: int(r.lib.nim_slab_pack_doubles(h, st, 1 if rank == 0 else 0))
                         for name, st in (("velocity", 1), ("pressure", 2), ("temperature", 4))}
                        if world > 1 else {})
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / max(args.steps, 1), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded mesh and T noise)",
            "config": dict(workload_config(case), parallelism=f"z-slabs x{world} (NCCL halo exchange)",
                           layout=[list(nimgpu.slab_layout(mesh.n_z, world, q)) for q in range(world)]),
            "iterations": iters, "iters_per_step": iters / max(len(stats), 1),
            "hbm_gbs_iteration_per_gpu": per_gpu,
            "halo": {"doubles_per_neighbour_per_pass": halo_doubles,
                     "bytes_sent_per_neighbour_per_pass": 8 * sum(halo_doubles.values()),
                     "all_reduces_per_pass": 1, "all_reduce_words": 24, "plane_cells": nt * nr},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_all, "d2h_bytes_per_step": h2d_all,
                    "steps": e2e_steps},
            "roofline": {"bound": "hbm", "kernel": "whole pass, per GPU (algorithmic 1880 B per cell-iteration)",
                         "achieved": per_gpu, "peak": peak, "unit": "GB/s", "frac": per_gpu / peak,
                         "peak_source": peak_kind, "traffic": None},
            "cpu_baseline": None,
            "gpu_launches": launches_all,
            "clocks": clk,
            "nu_inner_last": stats[-1].nu_inner if stats else None,
        }
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        r.close()
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch(args, rank, world, local):
    """The batched extension: 64 seeded enclosures advanced together, with
    every pass kernel launched once for all of them (nim_batch_step_fused,
    the line's value) and as 64 streams of per-enclosure graphs
    (nim_batch_step), against the same cases one at a time (nim_gpu_step per
    instance).  Wall clock between device-wide synchronisations: the
    host-side scheduling is part of what is measured.  With --precision mixed the batch runs the mixed path and the
    one-at-a-time baseline stays FP64."""
    import torch
    import nimgpu
    from nimgpu import config, _abi

    torch.cuda.set_device(local)
    if world > 1 and rank != 0:
        return 0
    cases = config.batch_cases(args.instances)
    steps = max(args.steps // 5, 1)

    prec = _abi.PRECISION_MIXED if args.precision == "mixed" else _abi.PRECISION_FP64

    def build(precision):
        out = []
        for c in cases:
            s = nimgpu.NimSolver(nimgpu.Mesh(c.mesh_params()), c.params(precision=precision))
            s.initialize_nse()
            s.add_temperature_noise(c.noise, c.seed)
            out.append(s)
        return out

    def cells_iters(recs_per_instance):
        return sum(c.ncells * sum(r.iters for r in recs) for c, recs in zip(cases, recs_per_instance))

    def timed_batch(fused):
        solvers = build(prec)
        # warm-up steps double as the autotuner's trials of the graph length
        best_g, tune, _ = nimgpu.autotune_batch(solvers, candidates=(4, 8, 16, 32), steps_each=1, fused=fused)
        torch.cuda.synchronize()
        l0 = sum(s.launch_count() for s in solvers)
        t0 = time.perf_counter()
        recs = nimgpu.batch_step(solvers, steps, fused=fused)
        torch.cuda.synchronize()
        tb = time.perf_counter() - t0
        launches = sum(s.launch_count() for s in solvers) - l0
        for s in solvers:
            s.close()
        return recs, tb, best_g, tune, launches

    # the fused launches (one persistent launch per pass kernel for all 64),
    # then the multi-stream form (64 streams of per-enclosure graphs)
    recs_b, tb, best_g, tune, launches_f = timed_batch(True)
    recs_s, ts, best_gs, tune_s, _ = timed_batch(False)
    solvers = build(_abi.PRECISION_FP64)
    for s in solvers:
        s.solve_nse(4)  # the batch's warm-up / tuning steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    recs_1 = [s.solve_nse(steps) for s in solvers]
    torch.cuda.synchronize()
    t1 = time.perf_counter() - t0
    for s in solvers:
        s.close()
    vb, v1, vs = cells_iters(recs_b) / tb, cells_iters(recs_1) / t1, cells_iters(recs_s) / ts
    same = [[r.iters for r in a] == [r.iters for r in b] for a, b in zip(recs_b, recs_1)]
    key = lambda rr: [(r.iters, r.iters_fp32, r.nu_inner, r.nu_outer, r.dilatation) for r in rr]
    same_streams = all(key(a) == key(b) for a, b in zip(recs_b, recs_s))
    nu_err = max(abs(a[-1].nu_inner - b[-1].nu_inner) / abs(b[-1].nu_inner) for a, b in zip(recs_b, recs_1))
    line = {
        "metric": METRIC, "value": vb, "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": max(args.warmup, 1),
        "ms_per_step": 1e3 * tb / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "warmup_note": "4 warm-up steps, one per autotuner candidate",
        "dtype": "f64" if prec == _abi.PRECISION_FP64 else "f32+f64", "precision": args.precision,
        "data": "synthetic (seeded meshes, physics and T noise)",
        "config": {"workload": f"batch: {len(cases)} cylinder enclosures D=1 H=1, hexagon side U[0.1,0.3], "
                               "a x a x round(0.75a) cells, a in [24,64], Ra log-uniform [1e3,1e6], "
                               "Pr in {0.71, 7.0}, dt=1e-3",
                   "cells": sum(c.ncells for c in cases), "instances": len(cases),
                   "timing": "wall clock between device synchronisations"},
        "form": "fused: one persistent launch per pass kernel over all enclosures (nim_batch_step_fused)",
        "gpu_launches": launches_f,
        "streams": {"value": vs, "unit": UNIT, "ms_per_step": 1e3 * ts / steps,
                    "form": "64 streams of per-enclosure graphs (nim_batch_step)",
                    "autotune_graph_iters": best_gs,
                    "records_equal_to_fused": same_streams},
        "fused_vs_streams": vb / vs,
        "one_at_a_time": {"value": v1, "unit": UNIT, "ms_per_step": 1e3 * t1 / steps, "precision": "fp64"},
        "nu_inner_rel_err_vs_one_at_a_time": nu_err,
        "batch_speedup": vb / v1,
        "autotune": {"graph_iters": best_g, "ns_per_cell_iteration": {str(k): 1e9 * v for k, v in tune.items()}},
        "same_iterations_as_one_at_a_time": all(same),
    }
    print(json.dumps(line), flush=True)
    return 0


MIXED_FIELDS = (0, 1, 2, 3, 4, 5, 6, 7, 8)  # faces u,v,w,p,T; cells u,v,w,T (nim_field)


def stop_over(args) -> dict:
    """--stop-tol T: every field's stop tolerance T instead of the
    reference's (1e-6 on u, v, w, T; 5e-3 on p), pressure measured on its
    gradients (is_dpdx_tolerance, nse.f90:292-307; a face-pressure test
    below ~1e-11 never holds, the pressure level drifts), so that the
    mixed path's FP64 phase runs until the FP64 change of every field is
    below T."""
    if args.stop_tol is None:
        return {}
    t = args.stop_tol
    return dict(tol_u=t, tol_v=t, tol_w=t, tol_T=t, tol_p=t, dpdx_tolerance=1, max_iters=400000)


def run_mixed(case, mesh, args, fp64_stats, fp64_fields, fp64_value, fp64_ms_step, peak, peak_kind):
    """The FP64 run's steps again, from the same start, with the mixed
    path: device-timed throughput of the same K steps, the Nusselt history
    and final fields against the FP64 run, and the FP32 kernels' roofline."""
    import torch
    import nimgpu
    from nimgpu import _abi
    s = nimgpu.NimSolver(mesh, case.params(precision=_abi.PRECISION_MIXED, **stop_over(args)))
    s.initialize_nse()
    s.add_temperature_noise(case.noise, case.seed)
    stream = torch.cuda.ExternalStream(s.stream_handle)
    recs = []
    for _ in range(max(args.warmup, 0)):
        recs += s.solve_nse(1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    timed = s.solve_nse(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    recs += timed
    iters = sum(r.iters for r in timed)
    value = case.ncells * iters / (ms / 1e3)
    nu_in = [abs(a.nu_inner - b.nu_inner) / abs(b.nu_inner) for a, b in zip(recs, fp64_stats)]
    nu_out = [abs(a.nu_outer - b.nu_outer) / abs(b.nu_outer) for a, b in zip(recs, fp64_stats)]
    nu = [max(a, b) for a, b in zip(nu_in, nu_out)]
    err = {}
    for f in MIXED_FIELDS:
        a, b = s.download(f), fp64_fields[f]
        name = ["faces_u", "faces_v", "faces_w", "faces_p", "faces_T", "meshes_u", "meshes_v", "meshes_w",
                "meshes_T"][f]
        err[name] = {"max_rel": float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)),
                     "l2_rel": float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))}
    prof = s.profile_iterations(20)
    dom = max((k for k in KERNEL_BYTES_PER_CELL if k in prof), key=lambda k: prof[k])
    achieved = KERNEL_BYTES_PER_CELL[dom] / 2 * case.ncells / (prof[dom] / 1e3) / 1e9
    s.close()
    return {
        "value": value, "unit": UNIT, "ms_per_step": ms / max(args.steps, 1), "iterations": iters,
        "iters_fp32": sum(r.iters_fp32 for r in timed), "speedup_vs_fp64": value / fp64_value,
        "step_time_speedup_vs_fp64": fp64_ms_step / (ms / max(args.steps, 1)),
        "dtype": "FP32 phase: f32 storage and arithmetic of the swept arrays; f64 maxima, per-step work, "
                 "reductions and refinement",
        "nu_rel_err_max": max(nu) if nu else None, "nu_rel_err_per_step": nu,
        "nu_inner_rel_err_per_step": nu_in, "nu_outer_rel_err_per_step": nu_out,
        "nu_fp64_per_step": [[b.nu_inner, b.nu_outer] for b in fp64_stats[:len(recs)]],
        "nu_mixed_per_step": [[a.nu_inner, a.nu_outer] for a in recs],
        "field_err_final": err,
        "tolerances": ("reference (tol_u,v,w,T 1e-6, tol_p 5e-3): both runs stop once a pass changes every "
                       "field by less than its tolerance" if args.stop_tol is None else
                       f"both runs stop once an FP64 pass changes every field by less than {args.stop_tol:g} "
                       "(pressure by its gradients)"),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "kernel_us": {k: round(1e3 * v, 2) for k, v in prof.items() if v > 0}},
    }


def run_tangent(case, mesh, args, fp64_stats, fp64_value, fp64_ms_step):
    """The FP64 run's steps again, from the same start, on the tangent-linear
    path seeded with d/dRa (nim_gpu_tangent_*): device-timed throughput of
    the same K steps, whether its values repeat the FP64 run's (iteration
    counts and Nusselt numbers), and d Nu_inner / dRa per step."""
    import torch
    import nimgpu
    s = nimgpu.NimSolver(mesh, case.params(**stop_over(args)))
    s.initialize_nse()
    s.add_temperature_noise(case.noise, case.seed)
    s.tangent_begin()
    s.tangent_seed(*nimgpu.NimSolver.tangent_seed_of("Ra", case.Ra, case.Pr))
    stream = torch.cuda.ExternalStream(s.stream_handle)
    recs, dnus = [], []
    if args.warmup > 0:
        r, d = s.tangent_step(args.warmup)
        recs += r
        dnus += list(d[:, 0])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r, d = s.tangent_step(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    recs += r
    dnus += list(d[:, 0])
    iters = sum(x.iters for x in r)
    value = case.ncells * iters / (ms / 1e3)
    s.close()
    same = [(a.iters, a.nu_inner) for a in recs] == [(b.iters, b.nu_inner) for b in fp64_stats[:len(recs)]]
    return {
        "value": value, "unit": UNIT, "ms_per_step": ms / max(args.steps, 1), "iterations": iters,
        "vs_fp64": value / fp64_value, "step_time_vs_fp64": fp64_ms_step / (ms / max(args.steps, 1)),
        "dtype": "dual f64 (value and derivative)", "seed": "d/dRa",
        "values_equal_fp64_run": same, "dnu_inner_dRa_per_step": [float(x) for x in dnus],
    }


def run_slabs(case, mesh, args, fp64_stats, fp64_fields, fp64_value, nslab=2):
    """The FP64 run's steps again, from the same start, as nslab z-slabs of
    the mesh on this device; wall clock around the synchronous group step
    (its work spans the slabs' streams)."""
    import nimgpu
    g = nimgpu.SlabGroup(mesh, case.params(), nslab)
    try:
        g.initialize_nse()
        g.add_temperature_noise(case.noise, case.seed)
        recs = []
        for _ in range(max(args.warmup, 0)):
            recs += g.solve_nse(1)
        t0 = time.perf_counter()
        timed = g.solve_nse(args.steps)
        dt = time.perf_counter() - t0
        recs += timed
        iters = sum(r.iters for r in timed)
        value = case.ncells * iters / dt
        same_iters = [r.iters for r in recs] == [r.iters for r in fp64_stats]
        same_fields = (all(np.array_equal(g.gather(f), fp64_fields[f]) for f in MIXED_FIELDS)
                       if fp64_fields is not None else None)
        return {"slabs": nslab, "value": value, "unit": UNIT, "ms_per_step": 1e3 * dt / max(args.steps, 1),
                "ratio_to_whole_mesh": value / fp64_value, "same_iterations": same_iters,
                "fields_identical": same_fields,
                "layout": [list(g.layout[s]) for s in g.slabs],
                "timing": "wall clock around nim_slab_step (synchronous)"}
    finally:
        g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default=CASE)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--schedule", default="parallel", choices=["parallel", "reference"],
                    help="reference: the Gauss-Seidel sweeps in the reference's cell order (its iterates)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="mixed: FP32 passes over a float mirror, then FP64 passes (nim_params.precision)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison")
    ap.add_argument("--instances", type=int, default=64,
                    help="--case batch: the first N of the 64 seeded enclosures (a smaller case for profiling)")
    ap.add_argument("--stop-tol", type=float, default=None,
                    help="stop every inner loop when each field's change is below this (FP64, pressure by its "
                         "gradients) instead of the reference's tolerances")
    ap.add_argument("--no-slabs", action="store_true", help="skip the two-slab comparison")
    ap.add_argument("--tangent", action="store_true",
                    help="also run the same steps on the tangent-linear path (d/dRa seeded)")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: every rank advances its own copy of --case (no decomposition)")
    ap.add_argument("--decompose", action="store_true",
                    help="run the z-slab decomposition path even at N = 1 (one slab, one rank)")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.case == "batch":
        return run_batch(args, rank, world, local)
    if (world > 1 and not args.replicas) or args.decompose:
        return run_slab_ranks(args, rank, world, local)

    import torch
    import nimgpu
    from nimgpu import config, _abi

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
        pg = dist

    case = config.CASES[args.case]
    mesh = nimgpu.Mesh(case.mesh_params())
    sched = _abi.SCHEDULE_REFERENCE if args.schedule == "reference" else _abi.SCHEDULE_PARALLEL
    prec = _abi.PRECISION_MIXED if args.precision == "mixed" else _abi.PRECISION_FP64
    solver = nimgpu.NimSolver(mesh, case.params(schedule=sched, precision=prec, **stop_over(args)))
    solver.initialize_nse()
    solver.add_temperature_noise(case.noise, case.seed)
    stream = torch.cuda.ExternalStream(solver.stream_handle)

    warm_stats = []
    for _ in range(max(args.warmup, 0)):
        warm_stats += solver.solve_nse(1)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()

    # ---------------- device-resident timed region
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = solver.launch_count()
    ev0.record(stream)
    stats = solver.solve_nse(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = solver.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    iters = sum(s.iters for s in stats)
    cell_iters = case.ncells * iters
    t_max, total = combine_ranks(pg, ms, cell_iters)
    value = total / (t_max / 1e3)
    want_mixed = (world == 1 and prec == _abi.PRECISION_FP64 and sched == _abi.SCHEDULE_PARALLEL
                  and not args.no_mixed)
    want_slabs = (world == 1 and prec == _abi.PRECISION_FP64 and sched == _abi.SCHEDULE_PARALLEL
                  and not args.no_slabs and case.n_z // 2 >= 2)
    fp64_fields = ({f: solver.download(f) for f in MIXED_FIELDS} if (want_mixed or want_slabs) else None)

    # ---------------- end to end through the C ABI with host buffers: the
    # host holds the state (read_restart / write_restart arrays) and every
    # step uploads it, advances one step and downloads it again
    up_fields = [_abi.FACES_U, _abi.FACES_V, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T,
                 _abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T,
                 _abi.MESHES_U_OLD, _abi.MESHES_V_OLD, _abi.MESHES_W_OLD, _abi.MESHES_T_OLD,
                 _abi.MESHES_UT, _abi.MESHES_VT, _abi.MESHES_WT]
    host = {f: torch.empty(nimgpu.field_len(f, mesh), dtype=torch.float64).pin_memory() for f in up_fields}
    for f in up_fields:
        solver.download(f, out=host[f].numpy())
    h2d = sum(h.numel() * 8 for h in host.values())
    d2h = h2d
    e2e_steps = max(2, args.steps // 2)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_iters = 0
    for _ in range(e2e_steps):
        for f in up_fields:
            solver.upload(f, host[f].numpy())
        st = solver.solve_nse(1)
        e2e_iters += sum(s.iters for s in st)
        for f in up_fields:
            solver.download(f, out=host[f].numpy())
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_total = case.ncells * e2e_iters
    e2e_s, e2e_total = combine_ranks(pg, e2e_s, e2e_total)
    e2e_value = e2e_total / e2e_s

    # ---------------- roofline of the dominant kernel (events per kernel)
    prof = solver.profile_iterations(20)
    peak, peak_kind = peaks()
    shares = {k: v for k, v in prof.items() if v > 0}
    tot = sum(shares.values())
    dom = max((k for k in KERNEL_BYTES_PER_CELL if k in prof), key=lambda k: prof[k])
    dom_ms = prof[dom]
    width = 4 if prec == _abi.PRECISION_MIXED else 8  # profile_iterations runs FP32 passes when mixed
    achieved = KERNEL_BYTES_PER_CELL[dom] * width / 8 * case.ncells / (dom_ms / 1e3) / 1e9
    iter_gbs = ALGO_BYTES_PER_CELL_ITER * cell_iters / (ms / 1e3) / 1e9

    mixed = None
    if want_mixed:
        mixed = run_mixed(case, mesh, args, warm_stats + list(stats), fp64_fields, value, ms / max(args.steps, 1),
                          peak, peak_kind)

    tangent = None
    if args.tangent and world == 1 and prec == _abi.PRECISION_FP64 and sched == _abi.SCHEDULE_PARALLEL:
        tangent = run_tangent(case, mesh, args, warm_stats + list(stats), value, ms / max(args.steps, 1))

    slabs = None
    if want_slabs:
        try:
            slabs = run_slabs(case, mesh, args, warm_stats + list(stats), fp64_fields, value)
        except Exception as exc:  # an extra measurement: report it, keep the line
            slabs = {"error": repr(exc)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, dt = cpu_sample(case, threads=1, iters=4, schedule=0)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"4 inner iterations of step 1 on {args.case} ({case.ncells} cells), "
                         f"reference cell order, 1 thread ({dt:.1f} s)", "host_cpu": host_cpu()}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == _abi.PRECISION_FP64 else "f32+f64",
        "data": "synthetic (seeded mesh and T noise)",
        "config": dict(workload_config(case), schedule=args.schedule, precision=args.precision,
                       stop=("reference tolerances" if args.stop_tol is None else
                             f"every field's change < {args.stop_tol:g} (pressure by gradients)")),
        "iterations": iters, "iters_per_step": iters / max(len(stats), 1),
        "hbm_gbs_iteration": iter_gbs,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": (NCU_DRAM_BYTES_PER_CELL[dom] * case.ncells if dom in NCU_DRAM_BYTES_PER_CELL
                                 else None),
                     "traffic_source": (f"ncu dram bytes on the {NCU_CAPTURE[dom]} case, scaled by cells"
                                        if dom in NCU_CAPTURE else None),
                     "bytes_per_launch": KERNEL_BYTES_PER_CELL[dom] * width / 8 * case.ncells,
                     "kernel_ms": dom_ms,
                     "shares": {k: round(v / tot, 4) for k, v in shares.items()},
                     "kernel_us": {k: round(1e3 * v, 2) for k, v in shares.items()}},
        "cpu_baseline": cpu,
        "gpu_launches": launches,
        "clocks": clk,
        "nu_inner_last": stats[-1].nu_inner if stats else None,
        "iters_fp32": sum(s.iters_fp32 for s in stats),
        "mixed": mixed,
        "slabs": slabs,
        "tangent": tangent,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    solver.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
