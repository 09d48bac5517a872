#!/usr/bin/env python
"""Benchmark of the DG-MPI 3D Euler residual + RK4 hot path on B200.

Workload: the plain-FP64 at-scale configuration -- isentropic vortex
(x-y vortex extruded in z, beta 5, centre (5,5), freestream (1,1,0)) on a
periodic [0,10]^3 box of 64^3 hexahedra, Lagrange p = 3 (83.9 M DOF),
Lax-Friedrichs flux, classic RK4 at CFL 0.1.  One benchmark *step* is one
RK4 step over the whole mesh (four fused stage launches replayed from a CUDA
graph).  Metric: DOF-stage updates/s = DOF x 4 x steps / time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value    : device time (CUDA events on the kernels' stream), state resident in HBM
e2e      : the same steps through the C ABI from pinned host buffers:
           dg_set_state (H2D), K x dg_rk4_steps(dt, 1), dg_get_state (D2H) --
           the resident-state use of the drop-in (one upload and one download
           around the K steps), so the per-step copy bytes, and the e2e rate,
           depend on K: 671 MB / K each way
roofline : one RK stage (the face-flux kernel + the stage kernel when the tuner
           picks a face-flux variant, else the stage kernel alone: the only
           kernels of the timed region), per stage
cpu_baseline / --impl reference : the CPU oracle (restatement of the
           reference's dense Kokkos algorithm, OpenMP over elements) on a
           16^3 sample of the same workload (same order, same per-element work)
N > 1    : slab decomposition (weak scaling): rank r owns a 64^3 slab of a
           periodic 64 x 64 x 64N box, the boundary coefficient slices travel
           per RK stage over NCCL (dg_dist.HaloExchange) while the interior
           elements compute, then the boundary elements; --replicas runs one
           independent replica of the workload per GPU instead.  (--transport
           host stages the exchange through pinned host buffers over gloo: the
           same stage order, for several ranks sharing one GPU.)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dg-mpi_b200"))

METRIC = "DOF-stage updates/s: FP64 vs mixed-precision (rel L2 diff <=1e-6 vs FP64)"
UNIT = "DOF-stage updates/s"
VORTEX = [1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0, 10.0, 10.0]
NEL = 64
ORDER = 3
CFL = 0.1
SAMPLE_NEL = 16
BYTES_PER_DOF_STAGE = 40  # FP64: read U_s, U_0, acc; write acc, U_next
FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12  # 148 SMs x 64 FP64 FMA/clk x 1.965 GHz


def algorithmic_flops_per_dof(p: int) -> float:
    """Sum-factorised algorithmic flop count per DOF and stage (n = p+1, m = p+2)."""
    n, m = p + 1, p + 2
    E = 2 * (m * n ** 3 + m ** 2 * n ** 2 + m ** 3 * n)
    trace = 6 * 5 * 2 * (n ** 3 + m * n ** 2 + m ** 2 * n)
    total = 5 * E + 15 * E + 2 * trace + 5 * 3 * 2 * n ** 4 + 130 * m ** 3 + 600 * m ** 2 + 20 * n ** 3
    return total / (5 * n ** 3)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_traffic(name="stage_kernel_p3_64cubed.md"):
    """DRAM bytes per stage launch recorded from an ncu capture (profiles/)."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if line.strip().startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"dg_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if smax and s > 0.5 * max(smax)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons, "samples": len(rows)}


def build_case(device: int, precision: str = "fp64", mesh=None, U0=None):
    import dg_b200
    if mesh is None:
        mesh = dg_b200.periodic_box((NEL, NEL, NEL), (0.0, 0.0, 0.0), (10.0, 10.0, 10.0))
    case = dg_b200.Case(mesh, ORDER, flux="LaxFriedrichs", gas_constant=1.0, device=device, precision=precision)
    if U0 is None:
        U0 = case.project_ic("IsentropicVortexXY", VORTEX)
    else:
        case.set_state(U0)
    dt = case.cfl_time_step(U0, CFL)
    return case, U0, dt, mesh


def rel_l2_per_variable(a, b):
    import numpy as np
    a = a.reshape(-1, 5)
    b = b.reshape(-1, 5)
    nb = np.linalg.norm(b, axis=0)
    # a variable below 1e-3 of the largest norm is zero in exact arithmetic
    # (rho w of this vortex): measured against the largest variable's norm
    den = np.where(nb > 1e-3 * nb.max(), nb, nb.max())
    return (np.linalg.norm(a - b, axis=0) / den).tolist()


def mixed_leg(local, mesh, U0, dt, K, W, dist, world, ref_case, fixed_variant=None):
    """The mixed-precision residual on the same workload: device-timed rate and
    the per-variable relative L2 difference to the FP64 path after 20 steps."""
    import torch
    case, _, _, _ = build_case(local, "mixed_fp32", mesh, U0)
    if fixed_variant is None:
        best, tune_ms = case.tune_stage(reps=2)
    else:
        case.stage_variant = best = fixed_variant
    variant = case.stage_variants()[best]
    case.rk4(dt, W)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = case.rk4_timed(dt, K)
    torch.cuda.synchronize()
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    dof = case.ne * case.nb * 5
    nacc = 20
    case.set_state(U0)
    case.rk4(dt, nacc)
    ref_case.set_state(U0)
    ref_case.rk4(dt, nacc)
    diff = rel_l2_per_variable(case.get_state(), ref_case.get_state())
    # the tensor-core kernel (split-BF16 volume GEMMs on tcgen05) on the same workload
    tc = None
    tcv = [i for i, v in enumerate(case.stage_variants()) if "tc" in v[4].split("+")]
    if tcv:
        case.stage_variant = tcv[0]
        case.set_state(U0)
        case.rk4(dt, W)
        torch.cuda.synchronize()
        ms_tc = case.rk4_timed(dt, K)
        if dist:
            t = torch.tensor([ms_tc], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_tc = float(t.item())
        case.set_state(U0)
        case.rk4(dt, nacc)
        tc = {"value": world * dof * 4 * K / (ms_tc / 1e3), "unit": UNIT, "ms_per_step": ms_tc / K,
              "stage_variant": case.stage_variants()[tcv[0]],
              "rel_l2_vs_fp64_after_%d_steps" % nacc: rel_l2_per_variable(case.get_state(), ref_case.get_state()),
              "arithmetic": "volume GEMMs as six BF16 split products on tcgen05 (FP32 accumulation in TMEM); "
                            "flux, lift in FP32; FP64 state, inverse mass and update"}
    case.close()
    return {"value": world * dof * 4 * K / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K,
            "stage_variant": variant, "rel_l2_vs_fp64_after_%d_steps" % nacc: diff,
            "arithmetic": "FP32 traces, fluxes and contractions; FP64 state, residual accumulation, "
                          "inverse mass, geometry and RK update", "tensor_core_kernel": tc}


def ensemble_leg(local, steps):
    """The batching configuration: 256 seeded x-y vortex cases (N in {8,12,16,24,32},
    p in 1..5, per-case CFL 0.1 time steps), mixed precision, one graph per RK4 step:
    rates with one launch per group (tuned variants) and with one launch per RK
    stage for all groups, and of the same cases one context at a time."""
    import studies
    spec = studies.ensemble_cases(256)
    box = {n: __import__("dg_b200").periodic_box((n, n, n), (0, 0, 0), (10.0, 10.0, 10.0)) for n in {c[0] for c in spec}}
    cases = [(box[n], p) for n, p, _ in spec]
    dof = sum(box[n].nelem * (p + 1) ** 3 * 5 for n, p, _ in spec)
    import dg_b200
    b = dg_b200.Batch(cases, gas_constant=1.0, precision="mixed_fp32", device=local)
    for i, (_, _, data) in enumerate(spec):
        U = b.project_ic(i, "IsentropicVortexXY", data)
        b.set_time_step(i, b.cfl_time_step(i, U, CFL))
    out = {"cases": len(spec), "dof": dof, "steps": steps, "precision": "mixed_fp32"}
    for single in (False, True):
        b.single_launch = single
        if not single:
            b.tune(reps=1)
            b.single_launch = False
        b.rk4(1)
        ms = b.rk4_timed(steps)
        out["one_launch_per_stage" if single else "one_launch_per_group_tuned"] = {
            "value": dof * 4 * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps}
    out["status"] = b.status()
    b.close()
    ms_seq = 0.0
    for i, (mesh, p) in enumerate(cases):
        c = dg_b200.Case(mesh, p, gas_constant=1.0, precision="mixed_fp32", device=local)
        U = c.project_ic("IsentropicVortexXY", spec[i][2])
        ms_seq += c.rk4_timed(c.cfl_time_step(U, CFL), steps)
        c.close()
    out["one_context_at_a_time"] = {"value": dof * 4 * steps / (ms_seq / 1e3), "unit": UNIT}
    return out


def cpu_oracle_rate(warmup: int, steps: int | None, budget_s: float = 12.0):
    """DOF-stage/s of the CPU oracle on the 16^3 sample; returns (rate, steps, seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dg_b200
    import pyoracle
    mesh = dg_b200.periodic_box((SAMPLE_NEL,) * 3, (0.0, 0.0, 0.0), (10.0, 10.0, 10.0))
    orc = pyoracle.OracleCase.from_mesh(mesh, ORDER, flux="LaxFriedrichs", gas_constant=1.0)
    U = orc.project_ic("IsentropicVortexXY", VORTEX)
    dt = 1e-3
    if warmup:
        U = orc.rk4(U, dt, warmup)
    dof = orc.ne * orc.nb * 5
    if steps is None:  # adaptive: one step to size a budget-bounded sample
        t0 = time.perf_counter()
        U = orc.rk4(U, dt, 1)
        one = time.perf_counter() - t0
        steps = max(1, min(50, int(budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    orc.rk4(U, dt, steps)
    sec = time.perf_counter() - t0
    threads = pyoracle.library().orc_get_threads()
    return dof * 4 * steps / sec, steps, sec, threads


def run_reference(args, rank: int):
    if rank != 0:
        return
    rate, steps, sec, threads = cpu_oracle_rate(args.warmup, args.steps)
    sample = (f"{SAMPLE_NEL}^3 periodic hex sample of the {NEL}^3 workload, p={ORDER}, {steps} RK4 steps "
              f"({sec:.2f} s) after {args.warmup} warm-up steps")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic isentropic vortex IC, in-memory periodic mesh)",
            "config": {"workload": f"vortex_xy_{NEL}cubed_p{ORDER}_fp64", "sample": f"{SAMPLE_NEL}^3",
                       "order": ORDER, "flux": "LaxFriedrichs", "stepper": "RK4"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def slab_main(args, world, rank, local):
    """The slab-decomposed workload over `world` ranks: device-timed steps (CUDA
    events on each rank's stream, max over ranks) and end to end through the
    public API (each rank's slab from pinned host memory in and out)."""
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    import dg_dist
    ndev = max(1, torch.cuda.device_count())
    device = local % ndev
    torch.cuda.set_device(device)
    backend = "nccl" if args.transport == "device" else "gloo"
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    K, W = args.steps, args.warmup
    dc = dg_dist.DistributedCase((NEL, NEL, NEL * world), (0.0, 0.0, 0.0), (10.0, 10.0, 10.0 * world), ORDER,
                                 gas_constant=1.0, transport=args.transport)
    case = dc.case
    U0 = case.project_ic("IsentropicVortexXY", VORTEX)
    dt = dc.cfl_time_step(U0, CFL)
    if args.variant is None:
        best, tune_ms = case.tune_stage(reps=2)
    else:
        case.stage_variant = best = args.variant
        tune_ms = [-1.0] * len(case.stage_variants())
    # every rank runs rank 0's choice
    v = torch.tensor([best], dtype=torch.int64, device="cuda" if backend == "nccl" else "cpu")
    dist.broadcast(v, 0)
    case.stage_variant = best = int(v.item())
    variants = case.stage_variants()
    dof = case.ne * case.nb * 5
    red_dev = "cuda" if backend == "nccl" else "cpu"

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device=red_dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    case.set_state(U0)
    with ClockSampler(device) as clocks:
        time.sleep(0.3)
        dc.rk4(dt, W)
        dc.sync()
        dist.barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(dc.stream)
        dc.rk4(dt, K)
        ev[1].record(dc.stream)
        ev[1].synchronize()
        device_ms = max_over_ranks(ev[0].elapsed_time(ev[1]))
    status = case.status()
    value = world * dof * 4 * K / (device_ms / 1e3)
    e2e = None
    host_in = host_out = None
    if not args.no_e2e:
        host_in = torch.from_numpy(U0).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        dist.barrier()
        t0 = time.perf_counter()
        case.set_state_ptr(host_in.data_ptr())
        for _ in range(K):
            dc.rk4(dt, 1)
        dc.sync()
        case.get_state_ptr(host_out.data_ptr())
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        e2e = world * dof * 4 * K / e2e_s
        if not torch.isfinite(host_out).all():
            raise RuntimeError("non-finite state after the e2e run")
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        launch_s = device_ms / 1e3 / (4 * K)
        achieved = BYTES_PER_DOF_STAGE * dof / launch_s / 1e9
        state_bytes = dof * 8
        face_split = "fx" in variants[best][4].split("+")
        per_stage = 2 * (2 if face_split else 1) + (2 if dc.exchange.peers else 0)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": device_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (analytic isentropic vortex IC, in-memory periodic mesh)",
            "config": {"workload": f"vortex_xy_{NEL}cubed_p{ORDER}_fp64_per_rank_slab",
                       "mesh": f"{NEL}x{NEL}x{NEL * world} periodic hex on [0,10]x[0,10]x[0,{10 * world}], "
                               f"one {NEL}^3 slab per rank",
                       "order": ORDER, "dof_per_rank": dof, "flux": "LaxFriedrichs", "cfl": CFL, "dt": dt,
                       "parallelism": f"slab decomposition over {world} ranks, halo exchange per RK stage "
                                      f"({args.transport} transport, {backend}) overlapped with the interior elements",
                       "halo_peers": len(dc.exchange.peers),
                       "halo_slices": sum(c for _, _, c in dc.exchange.peers),
                       "interior_elements": dc.part.ninterior,
                       "l2": "inputs larger than L2 (each state buffer %.0f MB > 126 MB)" % (state_bytes / 1e6),
                       "stage_variant": {"chosen": variants[best]}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": profile_traffic(),
                         "peak_source": peak_kind, "kernel": "per rank: stage + face kernels over the interior "
                         "and boundary element ranges (one RK stage)", "bytes_per_launch": BYTES_PER_DOF_STAGE * dof},
            "e2e": None if e2e is None else {
                "value": e2e, "unit": UNIT, "h2d_bytes_per_step": state_bytes / K,
                "d2h_bytes_per_step": state_bytes / K,
                "timing": "host clock around the public API (set_state, K x DistributedCase.rk4, get_state), max over ranks"},
            "gpu_launches": 4 * K * per_stage,
            "clocks": clocks.summary(),
            "status": status,
        }
        print(json.dumps(line), flush=True)
    dist.barrier()
    del host_in, host_out
    dc.close()
    dist.destroy_process_group()


def main():
    global NEL
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--nel", type=int, default=NEL, help="elements per direction (profiling on a smaller box)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 256-case ensemble leg")
    ap.add_argument("--variant", type=int, default=None, help="fixed FP64 launch variant instead of the tuner's pick")
    ap.add_argument("--mixed-variant", type=int, default=None, help="fixed mixed-precision launch variant")
    ap.add_argument("--replicas", action="store_true", help="N > 1: independent replicas instead of the slab decomposition")
    ap.add_argument("--slab", action="store_true", help="the slab decomposition also at N = 1")
    ap.add_argument("--transport", default="device", choices=["device", "host"],
                    help="slab halo exchange: device buffers over NCCL, or pinned host buffers over gloo")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    NEL = args.nel

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if (world > 1 and not args.replicas) or args.slab:
        slab_main(args, world, rank, local)
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)

    case, U0, dt, mesh = build_case(local)
    dof = case.ne * case.nb * 5
    K, W = args.steps, args.warmup
    case.set_state(U0)
    if args.variant is None:
        best, tune_ms = case.tune_stage(reps=2)  # the project's launch-variant tuner (untimed)
    else:  # a fixed launch variant (profiling runs: under ncu the tuner's timings are distorted)
        case.stage_variant = best = args.variant
        tune_ms = [-1.0] * len(case.stage_variants())
    variants = case.stage_variants()

    # ---- device-timed region: state resident in HBM ----
    case.set_state(U0)
    with ClockSampler(local) as clocks:  # sampled over warm-up and timed steps (>= 200 ms apart)
        time.sleep(0.3)  # the sampler's first row
        case.rk4(dt, W)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        device_ms = case.rk4_timed(dt, K)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
        t = torch.tensor([device_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        device_ms = float(t.item())
    value = world * dof * 4 * K / (device_ms / 1e3)

    # ---- end to end through the C ABI with pinned host buffers ----
    state_bytes = dof * 8
    e2e = None
    if not args.no_e2e:
        host_in = torch.from_numpy(U0).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        for _ in range(2):  # warm the copy path
            case.set_state_ptr(host_in.data_ptr())
            case.rk4(dt, 1)
            case.get_state_ptr(host_out.data_ptr())
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        case.set_state_ptr(host_in.data_ptr())
        for _ in range(K):
            case.rk4(dt, 1)
        case.get_state_ptr(host_out.data_ptr())
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        if dist:
            dist.barrier()
            t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = world * dof * 4 * K / e2e_s
        if not torch.isfinite(host_out).all():
            raise RuntimeError("non-finite state after the e2e run")

    mixed = None if args.no_mixed else mixed_leg(local, mesh, U0, dt, K, W, dist, world, case, args.mixed_variant)
    ens = None if (args.no_ensemble or world > 1) else ensemble_leg(local, max(5, K // 4))

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        # a face-flux variant runs two kernels per RK stage: the face kernel
        # (every face's flux once) and the stage kernel
        face_split = "fx" in variants[best][4].split("+")
        launches_per_stage = 2 if face_split else 1
        kernels = (f"dgk::face_flux_kernel<{ORDER}> + dgk::stage_kernel<{ORDER}> (one RK stage)" if face_split
                   else f"dgk::stage_kernel<{ORDER}>")
        launch_s = device_ms / 1e3 / (4 * K)
        achieved = BYTES_PER_DOF_STAGE * dof / launch_s / 1e9
        flops = algorithmic_flops_per_dof(ORDER) * dof / launch_s / 1e12
        traffic = profile_traffic()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": device_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (analytic isentropic vortex IC, in-memory periodic mesh)",
            "config": {"workload": f"vortex_xy_{NEL}cubed_p{ORDER}_fp64", "mesh": f"{NEL}^3 periodic hex on [0,10]^3",
                       "order": ORDER, "dof": dof, "flux": "LaxFriedrichs",
                       "stepper": "RK4, 4 stages/step, each " + ("a face-flux and a stage launch" if face_split else "one fused stage launch"),
                       "cfl": CFL, "dt": dt, "l2": "inputs larger than L2 (each state buffer %.0f MB > 126 MB)" % (state_bytes / 1e6),
                       "parallelism": "replicas" if world > 1 else "single-gpu",
                       "stage_variant": {"chosen": variants[best], "tuned_ms_per_launch": dict(
                           ("E%d_NT%d_G%d_%s" % v[:4] + ("_" + v[4] if v[4] else ""), round(t, 4))
                           for v, t in zip(variants, tune_ms) if t >= 0)}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                         "peak_source": peak_kind,
                         "kernel": kernels, "bytes_per_launch": BYTES_PER_DOF_STAGE * dof,
                         "launches_per_stage": launches_per_stage,
                         "binding_roof": "fp64",
                         "fp64": {"achieved_tflops": flops, "peak_tflops": FP64_NOMINAL_TFLOPS,
                                  "peak_source": "nominal (148 SMs x 64 FP64 FMA/clk x 1.965 GHz)",
                                  "frac": flops / FP64_NOMINAL_TFLOPS,
                                  "flops_per_dof_stage": algorithmic_flops_per_dof(ORDER)}},
            "e2e": None if e2e is None else {
                "value": e2e, "unit": UNIT, "h2d_bytes_per_step": state_bytes / K,
                "d2h_bytes_per_step": state_bytes / K + 4,
                "timing": "host clock around synchronous C-ABI calls, device synchronised on both sides"},
            "gpu_launches": 4 * K * launches_per_stage,
            "clocks": clocks.summary(),
        }
        if mixed is not None:
            line["mixed_fp32"] = mixed
        if ens is not None:
            line["ensemble"] = ens
        if world == 1 and not args.no_cpu_baseline:
            rate, steps, sec, threads = cpu_oracle_rate(1, None)
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                    "sample": f"{SAMPLE_NEL}^3 periodic hex, p={ORDER}, {steps} RK4 steps ({sec:.1f} s), "
                                              "dense per-element algorithm, OpenMP over elements"}
        print(json.dumps(line), flush=True)
    case.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
