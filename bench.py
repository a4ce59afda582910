#!/usr/bin/env python3
"""Benchmark of the coupled LBM / phase-field step on B200.

Workloads (--workload)
  bubbles   (default, the headline) the two-phase Allen-Cahn bubble case at
            256^3 (D3Q19 MRT pressure/velocity lattice + D3Q19 conservative
            Allen-Cahn lattice, 24 seeded bubbles, periodic x/y, walls in z)
  dendrite  thermal dendrite at 128^3 (anisotropic phase field + D3Q7
            thermal lattice, one centred seed)
  ensemble  48 seeded solutal dendrite domains (edges 48-128) packed into
            one lattice, BF16 storage, persistent launches + CUDA graph
  multigrain  eight grains (one D3Q19 Allen-Cahn order parameter each,
            pairwise overlap penalty) + D3Q7 thermal lattice, 128^3
  flow_dendrite  thermal dendrite growing in a melt that flows in at x = 0
            and out at x = n - 1, 128^3 (D3Q19 TRT flow with porous
            bounce-back + phase field + advected D3Q7 thermal lattice)
A "step" is one loop of the coupled step over every cell of the workload.
MLUPS = lattice cells x steps / s / 1e6.

Arms
  default           the sm_100a library (libmkb200.so) through its C ABI
  --impl reference  the reference method's CPU implementation (the FP64
                    OpenMP restatement in oracle/, since the reference's own
                    solver is a closed Windows DLL), all host threads

Under torchrun (N > 1) every rank runs an independent replica of the case on
its own GPU (the case is one domain; "scaling": "weak"); the time is the max
over ranks and the value sums all ranks' cells.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS, %HBM roofline: LBM+phase-field 256^3, FP16-store vs FP32 plain"
WORKLOADS = {
    "bubbles": {"workload": "multiphase Allen-Cahn bubbles {n}^3, D3Q19 MRT + D3Q19 AC, 24 bubbles, seed 0xB200",
                "metric": METRIC, "size": 256, "precision": "fp32", "kernel": "k_mp_collide", "collision": "MRT(g) + BGK(h)",
                "data": "synthetic (seeded bubble case, splitmix64 seed 0xB200)"},
    "dendrite": {"workload": "thermal dendrite {n}^3, anisotropic phase field (D3Q7) + D3Q7 thermal, one seed",
                 "metric": "MLUPS, %HBM roofline: thermal dendrite 128^3 (phase field + D3Q7 thermal)",
                 "size": 128, "precision": "fp32", "kernel": "k_dend_collide", "collision": "BGK(g) + BGK(T)",
                 "data": "synthetic (centred seed, eps4 0.05, undercooling 0.55)"},
    "flow_dendrite": {"workload": "flow + thermal dendrite {n}^3, D3Q19 TRT flow (porous bounce-back, inflow 0.02) "
                                  "+ phase field (D3Q7) + advected D3Q7 thermal, one seed",
                      "metric": "MLUPS, %HBM roofline: flow + thermal dendrite 128^3 (D3Q19 + D3Q7 + D3Q7)",
                      "size": 128, "precision": "fp32", "kernel": "k_fd_flow", "slot": "flow",
                      "collision": "TRT(f, porous bounce-back) + BGK(g) + BGK(T)",
                      "data": "synthetic (seed at x = n/3, eps4 0.05, undercooling 0.55, inflow u = 0.02)"},
    "multigrain": {"workload": "multigrain {n}^3: 8 grains (D3Q19 Allen-Cahn each, overlap penalty) + D3Q7 thermal",
                   "metric": "MLUPS, %HBM roofline: multigrain 128^3, 8 grain lattices + thermal",
                   "size": 128, "precision": "fp32", "kernel": "k_mg_collide", "collision": "BGK(g_j) + BGK(T)",
                   "data": "synthetic (2 x 2 x 2 grains of radius n/5 at the quarter points)"},
    "poiseuille": {"workload": "Poiseuille channel {n}x{h}x{h}, D3Q19 TRT (magic 3/16), walls in y, body force 1e-6",
                   "metric": "MLUPS: Poiseuille channel 64x32x32, D3Q19 TRT, FP64",
                   "size": 64, "precision": "fp64", "kernel": "k_flow", "collision": "TRT(f)",
                   "data": "synthetic (fluid at rest, constant body force)"},
    "ensemble": {"workload": "solutal dendrite ensemble: {nd} domains, edges 48-128, 1-6 seeds each, seed 0xE45E",
                 "metric": "MLUPS aggregate, %HBM roofline: {nd}-domain solutal dendrite ensemble, BF16, "
                           "persistent + graph",
                 "size": 0, "precision": "bf16", "kernel": "k_ens_collide", "collision": "BGK(g) + TRT(U)",
                 "data": "synthetic (splitmix64 ensemble generator, seed 0xE45E)"},
}
ENSEMBLE_SEED = 0xE45E
ENSEMBLE_DOMAINS = 48


def _measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _ncu_traffic():
    """Per-cell DRAM bytes of the dominant kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    out = {}
    try:
        with open(path) as f:
            for line in f:
                line = line.strip()
                if not line or line.startswith("#"):
                    continue
                k, v = line.split("=", 1)
                out[k.strip()] = float(v)
    except Exception:
        pass
    return out


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm.append(float(parts[1]))
                        smax.append(float(parts[2]))
                    except ValueError:
                        continue
                    for nm, val in zip(names, parts[5:9]):
                        if val.lower() == "active":
                            reasons.add(nm)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def _case_path(precision: str, n: int, workload: str = "bubbles") -> str:
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import cases
    d = os.path.join(tempfile.gettempdir(), "mkb200_bench")
    if workload == "dendrite":
        text = cases.thermal_dendrite(n=n, precision=precision, loops=5000)
    elif workload == "multigrain":
        q = [n / 4.0, 3.0 * n / 4.0]
        seeds = [(x, y, z, n / 5.0) for x in q for y in q for z in q]
        text = cases.multigrain(n=n, precision=precision, loops=5000, seeds=seeds)
    elif workload == "poiseuille":
        text = cases.poiseuille(nx=n, ny=n // 2, nz=n // 2, precision=precision, loops=2000)
    elif workload == "flow_dendrite":
        text = cases.flow_dendrite(nx=n, ny=n, nz=n, precision=precision, loops=5000, radius=8.0, u_in=0.02,
                                   center=(n / 3.0, (n - 1) / 2.0, (n - 1) / 2.0))
    else:
        text = cases.multiphase_bubbles(n=n, precision=precision, loops=10000)
    return cases.write(text, os.path.join(d, f"{workload}_{n}_{precision}.xml"))


def _collide_bytes(workload: str, prec: str, cells: int) -> int:
    """Algorithmic DRAM bytes of one launch of the dominant kernel.

    bubbles:  g and h (19 + 19 populations) read and written, phi read once,
              plus the FP32 Allen-Cahn rest population (read + write) with
              16-bit storage.
    dendrite / ensemble: phase-field and T/U lattices (7 + 7) read and
              written, phi(t+1) and phi(t) read, T/U read and written.
    flow_dendrite: the flow kernel: D3Q19 read and written, phi(t) read, the
              velocity (3 values) written.
    poiseuille: the flow kernel: D3Q19 read and written.
    """
    S = {"fp32": 4, "fp16": 2, "bf16": 2, "fp64": 8}[prec]
    P = 8 if prec == "fp64" else 4
    if workload == "bubbles":
        return cells * (2 * 38 * S + P + (4 if S == 2 else 0))
    if workload == "flow_dendrite":
        return cells * (38 * S + 4 * P)
    if workload == "poiseuille":
        return cells * 38 * S
    if workload == "multigrain":
        # 8 D3Q19 grain lattices and the D3Q7 thermal lattice read and written,
        # phi_j read (the stencil's halo counted once), phi(t+1), phi(t) read,
        # T read and written
        return cells * ((8 * 38 + 14) * S + (8 + 4) * P)
    return cells * (28 * S + 4 * P)


def _reducers(pg, device: str):
    """Max and sum of a host scalar over the ranks of `pg` (None: one rank),
    through a one-element FP64 tensor on `device` ("cuda" under NCCL, "cpu"
    under gloo).  Every rank must call them in the same order."""
    if pg is None:
        return (lambda x: x), (lambda x: x)

    def red(x, op):
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        pg.all_reduce(t, op=op)
        return float(t.item())

    return (lambda x: red(x, pg.ReduceOp.MAX)), (lambda x: red(x, pg.ReduceOp.SUM))


def job_mlups(cells_local: int, steps: int, seconds_local: float, reduce_max, reduce_sum):
    """Whole-job MLUPS of a sharded or replicated run: the cells every rank
    advanced, `steps` times, over the slowest rank's time.  Returns (MLUPS,
    the max time)."""
    t = reduce_max(seconds_local)
    cells = reduce_sum(cells_local)
    return cells * steps / t / 1e6, t


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_ours(args):
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params, initial_field
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A

    ws, rank, local = _dist()
    lib = A.load()
    st = lib.mk_set_device(local)
    if st != A.MK_OK:
        raise A.MkError(st, lib.mk_last_global_error().decode())
    pg = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist

    def barrier():
        if pg is not None:
            pg.barrier()

    max_over_ranks, sum_over_ranks = _reducers(pg, "cuda")

    n = args.size
    wl = WORKLOADS[args.workload]
    K, W = args.steps, args.warmup
    results = {}
    # FP64 storage too, so that the CPU arm (FP64) has a same-precision GPU line
    prec_list = [args.precision] + [p for p in ("fp32", "fp16", "bf16", "fp64") if p != args.precision]
    if args.no_variants:
        prec_list = prec_list[:1]
    peak, peak_kind = _measured_peak()
    main = None
    for prec in prec_list:
        params = case_params(_case_path(prec, n, args.workload))
        s = Solver(params=params)
        tune = s.autotune(4)
        s.advance(W, graph=True)
        s.sync()
        barrier()
        clk = Clocks(local)
        with clk:
            ms = s.time_advance(K, graph=True)
        cells = params.ncell()
        mlups, ms_s = job_mlups(cells, K, ms * 1e-3, max_over_ranks, sum_over_ranks)
        ms = ms_s * 1e3
        bpc = s.bytes_per_cell()
        # dominant kernel, timed live with CUDA events on the library's stream
        prof = s.profile(min(K, 50), wl.get("slot", "collide"))
        fused = args.workload == "bubbles" and s.fused
        rows = args.workload == "bubbles" and s.row_staged
        tile = args.workload == "bubbles" and bool(s.tuning.get("phi_tile", 0))
        # the fused multiphase loop is one launch, the flow model has no phi kernel
        prof_phi = {"kernel_ms": 0.0} if (fused or args.workload == "poiseuille") else s.profile(min(K, 50), "phi")
        fluid = s.fluid_cells()
        launches = min(K, 50)
        t_launch = prof["kernel_ms"] / launches * 1e-3
        # the fused launch moves the whole step's compulsory bytes
        collide_bytes = int(round(bpc * fluid)) if fused else _collide_bytes(args.workload, prec, fluid)
        achieved = collide_bytes / t_launch / 1e9
        step_gbs = bpc * cells * K / (ms * 1e-3) / 1e9
        d = s.diagnostics(raise_on_divergence=False)
        extra = {}
        if wl.get("slot", "collide") != "collide":
            # the phase-field / advected thermal kernel of the coupled model:
            # g and T read and written, phi(t+1), phi(t) and the velocity read,
            # T/U read and written
            pd = s.profile(launches, "collide")
            S = {"fp32": 4, "fp16": 2, "bf16": 2, "fp64": 8}[prec]
            Pb = 8 if prec == "fp64" else 4
            t_d = pd["kernel_ms"] / launches
            extra = {"dend_ms": t_d, "dend_frac": fluid * (28 * S + 7 * Pb) / (t_d * 1e-3) / 1e9 / peak}
        results[prec] = {
            "mlups": mlups, "ms_per_step": ms / K, "bytes_per_cell": bpc, "step_gbs": step_gbs,
            "step_frac": step_gbs / peak, "collide_ms": prof["kernel_ms"] / launches,
            "phi_ms": prof_phi["kernel_ms"] / launches, "collide_gbs": achieved, "collide_frac": achieved / peak,
            "collide_bytes_per_launch": collide_bytes, "clocks": clk.summary(), "n_bad": d["n_bad"],
            "launches_per_step": s.launches_per_step(), "tune": tune, "fused": fused, "row_staged": rows,
            "phi_tile": tile,
            "kernel": "k_mp_wave" if fused else ("k_mp_rows" if rows else ("k_mp_collide_tma" if tile else wl["kernel"])),
            **extra,
        }
        if prec == args.precision:
            main = (params, s)
        else:
            s.close()
    params, s = main
    r = results[args.precision]

    # end to end through the C ABI: pinned host state -> device, K loops, a
    # field -> pinned host (phi as FP32; the flow model: density as FP64 in,
    # ux as FP32 out)
    cells = params.ncell()
    flow = args.workload == "poiseuille"
    nbytes = cells * 4
    nbytes_in = cells * (8 if flow else 4)
    hp_in, hp_out = A.C.c_void_p(), A.C.c_void_p()
    lib.mk_host_alloc(nbytes_in, A.C.byref(hp_in))
    lib.mk_host_alloc(nbytes, A.C.byref(hp_out))
    phi_out = np.ctypeslib.as_array((A.C.c_float * cells).from_address(hp_out.value))
    out_field = A.MK_FIELD_UX if flow else A.MK_FIELD_PHI
    if flow:
        rho_in = np.ctypeslib.as_array((A.C.c_double * cells).from_address(hp_in.value))
        rho_in[:] = initial_field(params, "rho").ravel()
        dptr = rho_in.ctypes.data_as(A.C.POINTER(A.C.c_double))

        def upload():
            return lib.mk_set_state(s.handle, None, None, None, dptr, None, None, None)
    else:
        phi_in = np.ctypeslib.as_array((A.C.c_float * cells).from_address(hp_in.value))
        phi_in[:] = initial_field(params, "phi").ravel().astype(np.float32)
        fptr = phi_in.ctypes.data_as(A.C.POINTER(A.C.c_float))

        def upload():
            return lib.mk_set_state_f32(s.handle, fptr, None, None)
    # warm the staging buffers once
    upload()
    lib.mk_get_field(s.handle, out_field, A.MK_DTYPE_F32, hp_out, nbytes)
    barrier()
    t0 = time.perf_counter()
    stt = upload()
    stt |= lib.mk_advance_graph(s.handle, K)
    stt |= lib.mk_get_field(s.handle, out_field, A.MK_DTYPE_F32, hp_out, nbytes)
    e2e_s = time.perf_counter() - t0
    e2e_mlups, e2e_s = job_mlups(cells, K, e2e_s, max_over_ranks, sum_over_ranks)  # every rank, even on error
    if stt != 0:
        raise A.MkError(stt, lib.mk_last_error(s.handle).decode())
    phi_ok = bool(np.isfinite(phi_out).all())
    lib.mk_host_free(hp_in)
    lib.mk_host_free(hp_out)
    s.close()

    cpu = cpu_ref = cpu_code = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(n, budget_s=args.cpu_budget, workload=args.workload)
        cpu_ref = cpu_baseline_reference_structure(n, budget_s=args.cpu_budget, workload=args.workload)
        cpu_code = cpu_baseline_reference_code(budget_s=args.cpu_budget, workload=args.workload)

    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    traffic = _ncu_traffic()
    tkey = f"{args.workload}_collide_{args.precision}_bytes_per_cell"
    traffic_launch = traffic[tkey] * params.ncell() if tkey in traffic else None
    line = {
        "metric": wl["metric"].format(nd=args.domains),
        "value": round(r["mlups"], 1),
        "unit": "MLUPS",
        "n_gpus": ws,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(r["ms_per_step"], 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32",
        "data": wl["data"],
        "config": {"workload": wl["workload"].format(n=n, h=n // 2, nd=args.domains), "cells": params.ncell(),
                   "storage": args.precision, "collision": wl["collision"], "streaming": "AA in place",
                   "l2": ("inputs larger than L2 (%.2f GB resident populations)"
                          if r["bytes_per_cell"] * params.ncell() / 2 > 126e6 else
                          "inputs resident in L2 (%.3f GB resident populations: the rate is not an HBM figure)")
                   % (r["bytes_per_cell"] * params.ncell() / 2 / 1e9),
                   "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU"},
        "roofline": {"bound": "hbm", "kernel": r["kernel"], "achieved": round(r["collide_gbs"], 1),
                     "peak": peak, "unit": "GB/s", "frac": round(r["collide_frac"], 4),
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": r["collide_bytes_per_launch"],
                     "traffic": traffic_launch,
                     "step_bytes_per_cell": r["bytes_per_cell"], "step_gbs": round(r["step_gbs"], 1),
                     "step_frac": round(r["step_frac"], 4)},
        "variants": {k: {"mlups": round(v["mlups"], 1), "ms_per_step": round(v["ms_per_step"], 4),
                         "collide_frac": round(v["collide_frac"], 4), "step_frac": round(v["step_frac"], 4),
                         "bytes_per_cell": v["bytes_per_cell"], "n_bad": v["n_bad"],
                         "collide_ms": round(v["collide_ms"], 4), "phi_ms": round(v["phi_ms"], 4),
                         **({"dend_ms": round(v["dend_ms"], 4), "dend_frac": round(v["dend_frac"], 4)}
                            if "dend_ms" in v else {}),
                         "tuned": {"block": list(v["tune"]["block"]), "minb": v["tune"]["minb"],
                                   "fused": v["fused"], "row_staged": v["row_staged"], "phi_tile": v["phi_tile"]},
                         "kernel": v["kernel"],
                         "speedup_vs_fp32": round(v["mlups"] / results["fp32"]["mlups"], 3)
                         if "fp32" in results else None}
                     for k, v in results.items()},
        "e2e": {"value": round(e2e_mlups, 1), "unit": "MLUPS", "h2d_bytes_per_step": nbytes_in / K,
                "d2h_bytes_per_step": nbytes / K, "seconds": round(e2e_s, 4), "phi_finite": phi_ok,
                "path": ("mk_set_state rho f64 (pinned) + mk_advance_graph + mk_get_field ux f32 (pinned)" if flow
                         else "mk_set_state_f32 (pinned) + mk_advance_graph + mk_get_field f32 (pinned)")},
        "gpu_launches": K * r["launches_per_step"],
        "clocks": r["clocks"],
        "cpu_baseline": cpu,
    }
    if cpu_ref is not None:
        line["cpu_baseline_reference_structure"] = cpu_ref
    if cpu_code:
        line["cpu_baseline_reference_code"] = cpu_code
    print(json.dumps(line), flush=True)


def run_ensemble(args):
    """The packed solutal dendrite ensemble: every rank runs the whole ensemble
    (replicas; the domains are independent, so a multi-GPU job would give each
    rank its own ensemble seed)."""
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import Ensemble, ensemble_params
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A

    ws, rank, local = _dist()
    lib = A.load()
    st = lib.mk_set_device(local)
    if st != A.MK_OK:
        raise A.MkError(st, lib.mk_last_global_error().decode())
    pg = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist

    max_over_ranks, sum_over_ranks = _reducers(pg, "cuda")

    wl = WORKLOADS["ensemble"]
    K, W = args.steps, args.warmup
    nd = args.domains
    peak, peak_kind = _measured_peak()
    prec_list = [args.precision] + [p for p in ("bf16", "fp16", "fp32") if p != args.precision]
    if args.no_variants:
        prec_list = prec_list[:1]
    results = {}
    for prec in prec_list:
        ps = ensemble_params(ENSEMBLE_SEED + rank, nd, prec)
        e = Ensemble(ps)
        e.advance(W)
        if pg is not None:
            pg.barrier()
        clk = Clocks(local)
        l0 = e.launches
        with clk:
            ms = e.time_advance(K)
        launches = e.launches - l0
        cells = e.cells
        mlups, ms_s = job_mlups(cells, K, ms * 1e-3, max_over_ranks, sum_over_ranks)
        ms = ms_s * 1e3
        nprof = min(K, 50)
        prof = e.profile(nprof, "collide")
        prof_phi = e.profile(nprof, "phi")
        t_launch = prof["kernel_ms"] / nprof * 1e-3
        cb = _collide_bytes("ensemble", prec, cells)
        S = {"fp32": 4, "fp16": 2, "bf16": 2, "fp64": 8}[prec]
        P = 8 if prec == "fp64" else 4
        step_bytes = cells * (35 * S + 5 * P)
        bad = 0
        for d in range(nd):
            bad += int((~np.isfinite(e.field(d, "phi", np.float32))).sum())
        results[prec] = {"mlups": mlups, "ms_per_step": ms / K, "cells": cells,
                         "collide_ms": prof["kernel_ms"] / nprof, "phi_ms": prof_phi["kernel_ms"] / nprof,
                         "collide_gbs": cb / t_launch / 1e9, "collide_frac": cb / t_launch / 1e9 / peak,
                         "collide_bytes_per_launch": cb, "step_bytes_per_cell": step_bytes / cells,
                         "step_gbs": step_bytes * K / (ms * 1e-3) / 1e9, "clocks": clk.summary(),
                         "launches": launches, "n_bad": bad, "kernel": wl["kernel"]}
        results[prec]["step_frac"] = results[prec]["step_gbs"] / peak
        e.close()
    r = results[args.precision]

    # end to end through the C ABI: host parameters -> packed device state
    # (initial fields uploaded), K loops, phi of every domain back to the host
    ps = ensemble_params(ENSEMBLE_SEED + rank, nd, args.precision)
    cells = sum(p.ncell() for p in ps)
    if pg is not None:
        pg.barrier()
    t0 = time.perf_counter()
    e = Ensemble(ps)
    e.advance(K)
    phis = [e.field(d, "phi", np.float32) for d in range(nd)]
    e2e_mlups, e2e_s = job_mlups(cells, K, time.perf_counter() - t0, max_over_ranks, sum_over_ranks)
    phi_ok = all(bool(np.isfinite(x).all()) for x in phis)
    e.close()
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(0, budget_s=args.cpu_budget, workload="ensemble")
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    traffic = _ncu_traffic()
    tkey = f"ensemble_collide_{args.precision}_bytes_per_cell"
    line = {
        "metric": wl["metric"].format(nd=nd), "value": round(r["mlups"], 1), "unit": "MLUPS", "n_gpus": ws, "steps": K,
        "warmup": W,
        "ms_per_step": round(r["ms_per_step"], 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp64": "f64", "fp32": "f32"}.get(args.precision, "f32"),
        "data": wl["data"],
        "config": {"workload": wl["workload"].format(nd=nd), "domains": nd, "cells": r["cells"], "storage": args.precision,
                   "collision": wl["collision"], "streaming": "AA in place",
                   "l2": "inputs larger than L2 (%.2f GB resident state)" % (
                       r["step_bytes_per_cell"] * r["cells"] / 2 / 1e9),
                   "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU"},
        "roofline": {"bound": "hbm", "kernel": r["kernel"], "achieved": round(r["collide_gbs"], 1), "peak": peak,
                     "unit": "GB/s", "frac": round(r["collide_frac"], 4), "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": r["collide_bytes_per_launch"],
                     "traffic": traffic[tkey] * r["cells"] if tkey in traffic else None,
                     "step_bytes_per_cell": r["step_bytes_per_cell"], "step_gbs": round(r["step_gbs"], 1),
                     "step_frac": round(r["step_frac"], 4)},
        "variants": {k: {"mlups": round(v["mlups"], 1), "ms_per_step": round(v["ms_per_step"], 4),
                         "collide_ms": round(v["collide_ms"], 4), "phi_ms": round(v["phi_ms"], 4),
                         "collide_frac": round(v["collide_frac"], 4), "step_frac": round(v["step_frac"], 4),
                         "n_bad": v["n_bad"]} for k, v in results.items()},
        "e2e": {"value": round(e2e_mlups, 1), "unit": "MLUPS",
                "h2d_bytes_per_step": cells * 16 / K, "d2h_bytes_per_step": cells * 4 / K,
                "seconds": round(e2e_s, 4), "phi_finite": phi_ok,
                "path": "mk_ensemble_create (host initial fields, FP64) + mk_ensemble_advance + "
                        "mk_ensemble_get_field f32 per domain"},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def _oracle_case(workload: str, n: int):
    """FP64 parameters and initial fields of the workload's CPU sample (the
    ensemble's sample is its first domain), from the oracle's own case layer:
    the CPU arms never load the CUDA library."""
    from oracle import case as ocase
    if workload == "ensemble":
        params = ocase.ensemble(ENSEMBLE_SEED, 1, "fp64")[0]
    else:
        params = ocase.resolve(_case_path("fp64", n, workload))
    return params, ocase.oracle_fields(params)


def _sample_name(workload: str, n: int) -> str:
    if workload == "ensemble":
        return "domain 0 of the ensemble"
    if workload == "poiseuille":
        return f"the {n}x{n // 2}x{n // 2} channel"
    return f"the {n}^3 case"


def cpu_baseline_reference_structure(n: int, budget_s: float = 20.0, workload: str = "dendrite"):
    """Time the method in the reference's node-object layout (mkNode, every
    field of a node in one object, schedule(static, 16) node sweeps) on the
    host cores, on a bounded sample; the flow model and the thermal dendrite
    only (None for other workloads)."""
    if workload not in ("dendrite", "poiseuille"):
        return None
    from oracle.orc import Oracle, ReferenceStructure, load as load_oracle

    lib = load_oracle()
    params, fields = _oracle_case(workload, n)
    o = Oracle(params, **fields)
    a = ReferenceStructure(o)
    o.close()
    t0 = time.perf_counter()
    a.advance(1)
    t1 = time.perf_counter() - t0
    steps = max(1, min(2000, int(budget_s / max(t1, 1e-4))))
    t0 = time.perf_counter()
    a.advance(steps)
    dt = time.perf_counter() - t0
    a.close()
    cells = params.ncell()
    return {"value": round(cells * steps / dt / 1e6, 2), "unit": "MLUPS", "cores": int(lib.orc_get_threads()),
            "kind": "reference-structure",
            "sample": f"{steps} loops of {_sample_name(workload, n)} after 1 untimed loop (FP64, the reference's "
                      f"node-object layout, {ReferenceStructure.node_bytes()} B per node, schedule(static, 16))",
            "seconds": round(dt, 2)}


def _grain_fields(params) -> np.ndarray:
    """-tanh((r - R)/(sqrt2 W0)) per grain, x fastest (both case layers' initial order parameters)."""
    nx, ny, nz = params.nx, params.ny, params.nz
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    out = []
    for j in range(params.n_objects):
        cx, cy, cz = params.obj_center[j][0], params.obj_center[j][1], params.obj_center[j][2]
        r = np.sqrt((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2)
        out.append(-np.tanh((r - params.obj_radius[j]) / (np.sqrt(2.0) * params.W0)))
    return np.ascontiguousarray(np.stack(out), dtype=np.float64)


REF_CODE_SAMPLE = 64  # edge of the multigrain sample: the reference's nodes take ~4.5 KB each


def cpu_baseline_reference_code(budget_s: float = 20.0, workload: str = "multigrain"):
    """Time the reference's own multigrain solver source (mkFluidsUser::propagate /
    relaxation, MaterKit/src/mkFluidsUser.cpp:68-299, built into oracle/_ref
    against stand-ins for its closed library) on the host cores, on the
    workload's case at 64^3 with periodic faces (the stand-in neighbour
    wraps).  None for other workloads or where oracle/_ref is not built."""
    if workload != "multigrain":
        return None
    path = os.path.join(ROOT, "oracle", "_ref", "libmgref_q19.so")
    if not os.path.exists(path):
        return None
    import ctypes as C
    from oracle.orc import load as load_oracle

    lib = C.CDLL(path)
    lib.mgref_run.argtypes = [C.c_int] * 4 + [C.c_double, C.c_void_p, C.c_int, C.c_void_p]
    lib.mgref_loop_seconds.restype = C.c_double
    lib.mgref_set_threads.argtypes = [C.c_int]
    cores = int(load_oracle().orc_get_threads())
    lib.mgref_set_threads(cores)
    n = REF_CODE_SAMPLE
    params, _ = _oracle_case(workload, n)
    phi0 = _grain_fields(params)
    out = np.empty_like(phi0)

    def run(k):
        if lib.mgref_run(params.nx, params.ny, params.nz, params.n_objects, params.W0, phi0.ctypes.data, k,
                         out.ctypes.data) != 0:
            raise RuntimeError("mgref_run refused the case")
        return lib.mgref_loop_seconds()

    # the reference allocates per-node vectors in every relaxation, so a loop's
    # time is estimated from two
    t1 = run(2) / 2.0
    steps = max(1, min(50, int(budget_s / max(t1, 1e-4))))
    dt = run(steps)
    cells = params.ncell()
    return {"value": round(cells * steps / dt / 1e6, 2), "unit": "MLUPS", "cores": cores, "kind": "reference",
            "sample": f"{steps} loops of the {n}^3 case with periodic faces (the reference's mkFluidsUser.cpp "
                      f"multigrain propagate / relaxation compiled with stand-ins for its closed library; node "
                      f"objects of the reference's layout; set-up not timed)",
            "seconds": round(dt, 2)}


def cpu_baseline(n: int, budget_s: float = 20.0, workload: str = "bubbles"):
    """Time the FP64 OpenMP oracle on the host cores on a bounded sample of the workload."""
    from oracle.orc import Oracle, load as load_oracle

    lib = load_oracle()
    params, fields = _oracle_case(workload, n)
    o = Oracle(params, **fields)
    t0 = time.perf_counter()
    o.advance(1)
    t1 = time.perf_counter() - t0
    steps = max(1, min(20, int(budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    o.advance(steps)
    dt = time.perf_counter() - t0
    o.close()
    cells = params.ncell()
    return {"value": round(cells * steps / dt / 1e6, 2), "unit": "MLUPS", "cores": int(lib.orc_get_threads()),
            "kind": "port",
            "sample": f"{steps} loops of {_sample_name(workload, n)} after 1 untimed loop (FP64 oracle)",
            "seconds": round(dt, 2)}


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return
    from oracle.orc import Oracle, load as load_oracle

    lib = load_oracle()
    n = args.size
    wl = WORKLOADS[args.workload]
    code = cpu_baseline_reference_code(budget_s=args.ref_budget, workload=args.workload)
    if code is not None:
        # the reference's own multigrain source on its bounded sample (see there)
        mlups, dt, cores = code["value"], code["seconds"], code["cores"]
        steps = max(1, int(round(mlups * 1e6 * dt / REF_CODE_SAMPLE ** 3)))
        cells = n ** 3
        kind, sample = "reference", code["sample"]
    else:
        params, fields = _oracle_case(args.workload, n)
        o = Oracle(params, **fields)
        t0 = time.perf_counter()
        o.advance(1)  # one untimed warm-up loop
        t1 = time.perf_counter() - t0
        # each step is one full loop; the number of timed loops is capped so the
        # whole run stays within the budget
        steps = max(1, min(args.steps, int(args.ref_budget / max(t1, 1e-3))))
        t0 = time.perf_counter()
        o.advance(steps)
        dt = time.perf_counter() - t0
        cells = params.ncell()
        mlups = cells * steps / dt / 1e6
        cores = int(lib.orc_get_threads())
        kind = "port"
        sample = (f"{steps} loops of {_sample_name(args.workload, n)} (requested {args.steps}); the reference's own "
                  f"solver is a closed Windows DLL, so this is the FP64 OpenMP restatement")
    line = {
        "metric": wl["metric"].format(nd=args.domains), "value": round(mlups, 2), "unit": "MLUPS", "n_gpus": ws,
        "steps": steps, "warmup": 1,
        "ms_per_step": round(dt / steps * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": wl["data"],
        "config": {"workload": wl["workload"].format(n=n, nd=args.domains), "cells": cells, "storage": "fp64",
                   "parallelism": f"{cores} host threads"},
        "impl": "reference",
        "cpu_baseline": {"value": round(mlups, 2), "unit": "MLUPS", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(mlups, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_slabs(args):
    """Cost of the z-slab decomposition of one multiphase domain, measured in
    one process on one GPU: the bubble case advanced whole and as 2 and 4
    slabs (ghost planes, the FILL / PHI / RETURN exchanges as in-library
    copies, the masked return merge), milliseconds per loop from the host
    clock with the device synchronised on both sides (the exchange protocol is
    host-driven).  The slabs share this GPU's compute, so the figure bounds
    the protocol's cost; it is not a multi-GPU scaling number.  Prints one
    JSON line."""
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import slab as S

    n, K = args.size, args.steps
    params = case_params(_case_path(args.precision, n, "bubbles"))

    def timed(step):
        step(args.warmup)
        t0 = time.perf_counter()
        step(K)
        return (time.perf_counter() - t0) / K * 1e3

    whole = Solver(params=params)
    out = {"whole": round(timed(lambda k: (whole.advance(k), whole.sync())), 4)}
    whole.close()
    for nr in (2, 4):
        slabs = [S.Slab(params, r, nr) for r in range(nr)]
        out[f"slabs_{nr}"] = round(timed(lambda k: (S.advance_local(slabs, k), [s.sync() for s in slabs])), 4)
        for s in slabs:
            s.close()
    line = {"metric": "ms per loop, z-slab decomposition of one domain in one process", "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "steps": K, "warmup": args.warmup, "dtype": args.precision,
            "data": "synthetic", "config": {"workload": f"multiphase Allen-Cahn bubbles {n}^3", "cells": n ** 3},
            "ms_per_loop": out,
            "overhead": {k: round(v / out["whole"] - 1.0, 4) for k, v in out.items() if k != "whole"}}
    print(json.dumps(line), flush=True)


def run_accuracy(args):
    """Reduced-precision accuracy of the bubble case at full size: the case
    advanced `--accuracy-loops` loops (default 10,000) with FP64, FP32, FP16
    and BF16 storage; each reduced precision against the FP64 run (which
    equals the CPU oracle to 1e-10, tests/test_gpu_parity_at_size.py): phi
    relative L2 error and largest absolute error over the fluid cells, and
    the relative drift of the conserved phi sum.  Prints one JSON line."""
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A

    lib = A.load()
    st = lib.mk_set_device(0)
    if st != A.MK_OK:
        raise A.MkError(st, lib.mk_last_global_error().decode())
    n, loops = args.size, args.accuracy_loops
    out, ref = {}, None
    for prec in ("fp64", "fp32", "fp16", "bf16"):
        params = case_params(_case_path(prec, n, "bubbles"))
        s = Solver(params=params)
        d0 = s.diagnostics()
        t0 = time.perf_counter()
        s.advance(loops, graph=True)
        s.sync()
        secs = time.perf_counter() - t0
        d1 = s.diagnostics(raise_on_divergence=False)
        phi = s.field("phi")
        fluid = np.ones(phi.shape, dtype=bool)
        fluid[0], fluid[-1] = False, False  # the z walls
        drift = abs(d1["phi_sum"] - d0["phi_sum"]) / abs(d0["phi_sum"])
        if ref is None:
            ref = phi
            out[prec] = {"phi_sum_drift": drift, "n_bad": d1["n_bad"], "seconds": round(secs, 2)}
        else:
            diff = (phi - ref)[fluid]
            out[prec] = {"phi_rel_l2": float(np.linalg.norm(diff) / np.linalg.norm(ref[fluid])),
                         "phi_max_abs_err": float(np.max(np.abs(diff))), "phi_sum_drift": drift,
                         "n_bad": d1["n_bad"], "seconds": round(secs, 2)}
        s.close()
    line = {"metric": "reduced-precision accuracy vs FP64 storage", "workload":
            WORKLOADS["bubbles"]["workload"].format(n=n), "loops": loops, "cells": n ** 3,
            "reference": "FP64 storage on the device (equal to the CPU oracle to 1e-10)", "results": out}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bubbles", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default=None, choices=["fp32", "fp16", "bf16", "fp64"])
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--domains", type=int, default=ENSEMBLE_DOMAINS)
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    ap.add_argument("--accuracy", action="store_true",
                    help="reduced-precision accuracy of the bubble case vs FP64 storage (not a timing run)")
    ap.add_argument("--accuracy-loops", type=int, default=10000)
    ap.add_argument("--slabs", action="store_true",
                    help="cost of the z-slab decomposition in one process on one GPU (not a timing run of the step)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    wl = WORKLOADS[args.workload]
    if args.precision is None:
        args.precision = wl["precision"]
    if args.size is None:
        args.size = wl["size"]
    if args.accuracy:
        run_accuracy(args)
    elif args.slabs:
        run_slabs(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
