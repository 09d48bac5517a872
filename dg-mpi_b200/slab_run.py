#!/usr/bin/env python
"""Weak-scaling run of the slab-decomposed path: one rank per GPU, each owning
an n x n x n slab of an n x n x (n * world) periodic box (x-y vortex on
[0,10] x [0,10] x [0,10*world], extruded in z), with the per-stage halo
exchange of dg_dist over NCCL overlapped with the interior elements.

  python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 \\
      dg-mpi_b200/slab_run.py [--nel 64] [--order 3] [--steps 20] [--warmup 3]

Prints one JSON line (rank 0): DOF-stage updates/s over all ranks, timed with
CUDA events on each rank's stream, max over ranks.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

import dg_dist  # noqa: E402

VORTEX = [1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0, 10.0, 10.0]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nel", type=int, default=64)
    ap.add_argument("--order", type=int, default=3)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed_fp32"])
    args = ap.parse_args()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29531")
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    world, rank = dist.get_world_size(), dist.get_rank()
    n = args.nel
    dc = dg_dist.DistributedCase((n, n, n * world), (0, 0, 0), (10.0, 10.0, 10.0 * world), args.order,
                                 gas_constant=1.0, precision=args.precision)
    U = dc.case.project_ic("IsentropicVortexXY", VORTEX)
    dt = dc.cfl_time_step(U, 0.1)
    dc.case.tune_stage(reps=2)   # same launch variant on every rank: rank 0's choice
    v = torch.tensor([dc.case.stage_variant], device="cuda")
    dist.broadcast(v, 0)
    dc.case.stage_variant = int(v.item())
    dc.case.set_state(U)
    dc.rk4(dt, args.warmup)
    dc.sync()
    dist.barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(dc.stream)
    dc.rk4(dt, args.steps)
    ev[1].record(dc.stream)
    ev[1].synchronize()
    ms = torch.tensor([ev[0].elapsed_time(ev[1])], dtype=torch.float64, device="cuda")
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    status = dc.case.status()
    dof = dc.case.ne * dc.case.nb * 5
    if rank == 0:
        print(json.dumps({
            "metric": "DOF-stage updates/s (slab decomposition, halo exchange per stage)",
            "value": world * dof * 4 * args.steps / (ms.item() / 1e3), "n_gpus": world, "steps": args.steps,
            "ms_per_step": ms.item() / args.steps, "scaling": "weak", "precision": args.precision,
            "config": {"slab": f"{n}^3 elements per rank", "order": args.order,
                       "halo_peers": len(dc.exchange.peers),
                       "halo_slices": sum(c for _, _, c in dc.exchange.peers),
                       "interior_elements": dc.part.ninterior, "owned_elements": dc.part.nowned},
            "status": status}), flush=True)
    dist.barrier()
    dc.close()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
