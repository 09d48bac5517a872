#!/usr/bin/env python
"""Accuracy / precision studies of the configurations beyond the bench workload.

  python dg-mpi_b200/studies.py precision   # 64^3, p=5, x-y vortex, 500 RK4 steps
  python dg-mpi_b200/studies.py taylor_green # 96^3, p=4, Taylor-Green, 200 RK4 steps
  python dg-mpi_b200/studies.py ensemble     # 256 seeded vortex cases, p=1..5, 8^3..32^3, 100 steps
  python dg-mpi_b200/studies.py <name> --scale 0.25  # smaller mesh (fewer cases), same orders
  python dg-mpi_b200/studies.py general       # bent (non-affine) periodic boxes: 48^3 p=3, 24^3 p=5
  python dg-mpi_b200/studies.py convergence2d # the reference's 2D convergence table, N = 2..256, p = 1..3
  python dg-mpi_b200/studies.py stage2d --nel 512 --order 3 --steps 2   # one 2D case (ncu captures)
  python dg-mpi_b200/studies.py stage --nel 40 --order 3 --precision fp64 --variant 0
                                             # one launch variant, 2 RK4 steps, no tuner (ncu captures)

Each study runs the FP64 path and the mixed-precision path (FP32 residual,
FP64 state) from the same projected initial condition and prints one JSON line:
per-variable relative L2 difference mixed vs FP64, L2 error of both against the
exact advected vortex (precision) or the kinetic-energy histories of both
(Taylor-Green), and the device-timed DOF-stage update rate of both paths.
The ensemble study advances all cases as one batch (dg_batch_*, one graph of
per-order stage launches) in mixed precision and in FP64, and the same cases
one context at a time, and reports the aggregate rates and errors.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import dg_b200  # noqa: E402

VORTEX = [1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0, 10.0, 10.0]


def rel_l2(a, b):
    a = a.reshape(-1, 5)
    b = b.reshape(-1, 5)
    nb = np.linalg.norm(b, axis=0)
    den = np.where(nb > 1e-3 * nb.max(), nb, nb.max())  # zero-in-exact-arithmetic fields
    return (np.linalg.norm(a - b, axis=0) / den).tolist()


def run_pair(mesh, order, ic, data, steps, cfl, ke_every=0):
    cases = {p: dg_b200.Case(mesh, order, flux="LaxFriedrichs", gas_constant=1.0, precision=p)
             for p in ("fp64", "mixed_fp32")}
    t0 = time.perf_counter()
    U0 = cases["fp64"].project_ic(ic, data)
    setup_s = time.perf_counter() - t0
    dt = cases["fp64"].cfl_time_step(U0, cfl)
    out = {"dt": dt, "steps": steps, "ic_projection_s": setup_s}
    for name, case in cases.items():
        case.set_state(U0)
        best, _ = case.tune_stage(reps=1)
        case.set_state(U0)
        hist, ms_total, done = [], 0.0, 0
        chunk = ke_every if ke_every else steps
        if ke_every:
            hist.append(case.kinetic_energy())
        while done < steps:
            n = min(chunk, steps - done)
            ms_total += case.rk4_timed(dt, n)
            done += n
            if ke_every:
                hist.append(case.kinetic_energy())
        dof = case.ne * case.nb * 5
        out[name] = {"dof_stage_per_s": dof * 4 * steps / (ms_total / 1e3), "ms_per_step": ms_total / steps,
                     "stage_variant": case.stage_variants()[best], "status": case.status()}
        if ke_every:
            out[name]["kinetic_energy"] = hist
    out["rel_l2_mixed_vs_fp64"] = rel_l2(cases["mixed_fp32"].get_state(), cases["fp64"].get_state())
    return cases, out


def precision(scale: float):
    n = max(4, int(round(64 * scale)))
    mesh = dg_b200.periodic_box((n, n, n), (0, 0, 0), (10.0, 10.0, 10.0))
    cases, out = run_pair(mesh, 5, "IsentropicVortexXY", VORTEX, 500, 0.1)
    t = out["steps"] * out["dt"]
    for name, case in cases.items():
        out[name]["l2_error_vs_exact"] = case.l2_error("IsentropicVortexXY", VORTEX, t).tolist()
    out.update({"config": f"x-y isentropic vortex, [0,10]^3, {n}^3 hex, p=5, LF flux, RK4 CFL 0.1", "time": t})
    return out


def taylor_green(scale: float):
    n = max(4, int(round(96 * scale)))
    L = 2 * math.pi
    mesh = dg_b200.periodic_box((n, n, n), (0, 0, 0), (L, L, L))
    cases, out = run_pair(mesh, 4, "TaylorGreen", [0.1], 200, 0.1, ke_every=20)
    k64 = np.array(out["fp64"]["kinetic_energy"])
    kmx = np.array(out["mixed_fp32"]["kinetic_energy"])
    out["ke_max_rel_diff"] = float(np.max(np.abs(kmx - k64) / np.abs(k64)))
    out.update({"config": f"Taylor-Green, [0,2pi]^3, {n}^3 hex, p=4, Mach 0.1, LF flux, RK4 CFL 0.1"})
    return out


def ensemble_cases(ncases: int, seed: int = 2024):
    """Seeded ensemble: mesh N in {8,12,16,24,32}, order in 1..5, vortex
    strength U[1,5], centre U[3,7]^2, free stream U[0.5,1.5]^2 on [0,10]^3."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(ncases):
        n = int(rng.choice([8, 12, 16, 24, 32]))
        p = int(rng.integers(1, 6))
        beta = float(rng.uniform(1, 5))
        xc, yc = (float(v) for v in rng.uniform(3, 7, 2))
        u, v = (float(w) for w in rng.uniform(0.5, 1.5, 2))
        out.append((n, p, [1.0, u, v, 1.0, beta, xc, yc, 10.0, 10.0]))
    return out


def ensemble(scale: float, steps: int = 100, cfl: float = 0.1):
    spec = ensemble_cases(max(8, int(round(256 * scale))))
    box = {n: dg_b200.periodic_box((n, n, n), (0, 0, 0), (10.0, 10.0, 10.0)) for n in {c[0] for c in spec}}
    cases = [(box[n], p) for n, p, _ in spec]
    dof = [box[n].nelem * (p + 1) ** 3 * 5 for n, p, _ in spec]
    out = {"ncases": len(spec), "steps": steps, "total_dof": int(sum(dof)),
           "orders": {str(p): sum(1 for c in spec if c[1] == p) for p in range(1, 6)}}
    finals = {}
    for prec in ("mixed_fp32", "fp64"):
        t0 = time.perf_counter()
        b = dg_b200.Batch(cases, gas_constant=1.0, precision=prec)
        dts = []
        for i, (_, _, data) in enumerate(spec):
            U = b.project_ic(i, "IsentropicVortexXY", data)
            dts.append(b.cfl_time_step(i, U, cfl))
            b.set_time_step(i, dts[-1])
        setup = time.perf_counter() - t0
        # one launch per RK stage for all groups
        b.single_launch = True
        single = b.single_launch
        ms = b.rk4_timed(steps)
        errs = [b.l2_error(i, "IsentropicVortexXY", data, steps * dts[i]) for i, (_, _, data) in enumerate(spec)]
        finals[prec] = [b.get_state(i) for i in range(0, len(spec), 4)]  # host memory: every 4th case
        out[prec] = {"dof_stage_per_s": sum(dof) * 4 * steps / (ms / 1e3), "ms_total": ms, "setup_s": setup,
                     "single_launch": single, "groups": b.groups(), "status": b.status(),
                     "max_l2_error_vs_exact": np.max(np.array(errs), axis=0).tolist(),
                     "median_l2_error_vs_exact": np.median(np.array(errs), axis=0).tolist()}
        # one launch per group and stage, each group's variant tuned
        b.single_launch = False
        b.tune(reps=1)
        for i, (_, _, data) in enumerate(spec):
            b.project_ic(i, "IsentropicVortexXY", data)
        ms_g = b.rk4_timed(steps)
        out[prec]["per_group_tuned"] = {"dof_stage_per_s": sum(dof) * 4 * steps / (ms_g / 1e3), "ms_total": ms_g,
                                        "groups": b.groups()}
        b.close()
    diffs = np.array([rel_l2(a, c) for a, c in zip(finals["mixed_fp32"], finals["fp64"])])
    out["max_rel_l2_mixed_vs_fp64_every_4th_case"] = diffs.max(axis=0).tolist()
    del finals
    # the same cases one context at a time (device time of each case's steps)
    ms_seq = 0.0
    for i, (mesh, p) in enumerate(cases):
        c = dg_b200.Case(mesh, p, gas_constant=1.0, precision="mixed_fp32")
        U = c.project_ic("IsentropicVortexXY", spec[i][2])
        ms_seq += c.rk4_timed(c.cfl_time_step(U, cfl), steps)
        c.close()
    out["sequential_mixed"] = {"dof_stage_per_s": sum(dof) * 4 * steps / (ms_seq / 1e3), "ms_total": ms_seq}
    out["config"] = (f"{len(spec)} x-y vortex cases on [0,10]^3, N in {{8,12,16,24,32}}, p in 1..5, seeded, "
                     f"LF flux, RK4 CFL 0.1 per case, {steps} steps")
    return out


def bent_box(n: int, amplitude: float):
    """Periodic box on [0,10]^3 whose nodes move by a smooth periodic field
    (products of sines and cosines of two coordinates, amplitude in cells):
    every element becomes a general trilinear hexahedron."""
    L = 10.0
    mesh = dg_b200.periodic_box((n, n, n), (0.0, 0.0, 0.0), (L, L, L))
    x = mesh.node_coords
    s = [np.sin(2 * np.pi * x[:, d] / L + 0.7 * (d + 1)) for d in range(3)]
    c = [np.cos(2 * np.pi * x[:, d] / L + 0.4 * (d + 1)) for d in range(3)]
    disp = amplitude * (L / n) * np.stack([s[1] * c[2], s[2] * c[0], s[0] * c[1]], axis=1)
    return dg_b200.Mesh(np.ascontiguousarray(x + disp), mesh.elem_to_node_ids, mesh.interior_faces)


def general(scale: float):
    """Non-affine meshes: the general-geometry stage kernel (per-point metric
    terms and normals, a dense inverse mass matrix per element, all streamed
    from HBM) on bent boxes, FP64 and mixed; rates, mixed vs FP64 after the
    steps, and the achieved HBM rate of the streams the stage reads and writes."""
    out = {"config": "x-y vortex on bent periodic boxes [0,10]^3 (5 % bend), LF flux, RK4 CFL 0.1"}
    for n0, order, steps in ((48, 3, 40), (24, 5, 20)):
        n = max(4, int(round(n0 * scale)))
        mesh = bent_box(n, 0.05)
        t0 = time.perf_counter()
        cases, res = run_pair(mesh, order, "IsentropicVortexXY", VORTEX, steps, 0.1)
        res["setup_s_both"] = time.perf_counter() - t0
        nb, ne, m = (order + 1) ** 3, n ** 3, order + 2
        # per element and stage: the five state streams (40 B/DOF), the metric
        # terms, the face normal data and the inverse mass matrix (FP64)
        bytes_elem = 40 * 5 * nb + 8 * (9 * m ** 3 + 6 * 4 * m * m + nb * nb)
        for name in ("fp64", "mixed_fp32"):
            r = res[name]
            stages_per_s = r["dof_stage_per_s"] / (ne * nb * 5)
            extra = 8 * 5 * nb if name == "mixed_fp32" else 0  # the FP32 residual's unit-pressure table
            r["hbm_gbs_streams"] = stages_per_s * ne * (bytes_elem + extra) / 1e9
        res["rel_l2_mixed_vs_fp64"] = [float(v) for v in res["rel_l2_mixed_vs_fp64"]]
        res["bytes_per_element_stage"] = bytes_elem
        for cs in cases.values():
            cs.close()
        out[f"{n}^3_p{order}"] = res
    return out


def stage(nel: int, order: int, precision_: str, variant: int, steps: int):
    """x-y vortex on an nel^3 box, one fixed stage-kernel launch variant (no tuner, so the
    launch sequence is known: the projection, then four stage launches per step)."""
    mesh = dg_b200.periodic_box((nel, nel, nel), (0.0, 0.0, 0.0), (10.0, 10.0, 10.0))
    case = dg_b200.Case(mesh, order, gas_constant=1.0, precision=precision_)
    U0 = case.project_ic("IsentropicVortexXY", VORTEX)
    dt = case.cfl_time_step(U0, 0.1)
    case.stage_variant = variant
    case.rk4(dt, steps)
    out = {"nel": nel, "order": order, "stage_variant": case.stage_variants()[variant], "steps": steps,
           "status": case.status()}
    case.close()
    return out


# the reference's published 2D convergence table: density L2 error of the 2D
# isentropic vortex, HLLC, LagrangeQuad, RK4 dt = 1e-3 to t = 1, N x N boxes
# (examples/isentropic_vortex/convergence.py:51-86; entries marked "HOLD FOR
# NOW" there repeat the previous value and are left out)
TABLE_2D = {
    1: {2: 4.057487237640151206408e-02, 4: 3.659091741930729779764e-02, 8: 1.399040502291195101070e-02,
        16: 3.736915003326653998000e-03, 32: 9.128245919612695130629e-04, 64: 2.230394344260663451376e-04,
        128: 5.552798642178519519276e-05, 256: 1.390242977018099767455e-05},
    2: {2: 3.932754850914681188367e-02, 4: 1.414430149472130186783e-02, 8: 3.248199949411992391163e-03,
        16: 3.915751398100587301818e-04, 32: 4.874570751994351309371e-05, 64: 5.808150680654376531750e-06,
        128: 7.102447210422075577049e-07},
    3: {2: 2.911726700453628677301e-02, 4: 6.747203591607888774340e-03, 8: 5.564165617240108456867e-04,
        16: 3.771907882313834693960e-05, 32: 2.369398862192326906355e-06, 64: 1.424882779046236941575e-07,
        128: 9.074300168426849006228e-09},
}


def convergence2d(scale: float):
    """The reference's 2D convergence study on the 2D path (dg2d_*): periodic
    N x N boxes on [-5, 5]^2, the 2D vortex, 1000 RK4 steps of 1e-3; the
    density error against the published table and the device-timed rate."""
    rows = []
    nmax = max(2, int(256 * scale))
    for p in (1, 2, 3):
        prev = None
        for N in (2, 4, 8, 16, 32, 64, 128, 256):
            if N > nmax:
                break
            mesh = dg_b200.periodic_box_2d((N, N), (-5.0, -5.0), (10.0, 10.0))
            case = dg_b200.Case2D(mesh, p, flux="HLLC", gas_constant=1.0)
            case.project_ic("IsentropicVortex", VORTEX[:5])
            ms = case.rk4_timed(1e-3, 1000)
            err = float(case.l2_error("IsentropicVortex", VORTEX[:5], 1.0)[0])
            ref = TABLE_2D[p].get(N)
            dof = N * N * (p + 1) ** 2 * 4
            rows.append({"p": p, "N": N, "rho_l2_error": err, "reference": ref,
                         "rel_diff": None if ref is None else err / ref - 1.0,
                         "order": None if prev is None else math.log(prev / err) / math.log(2.0),
                         "dof_stage_per_s": dof * 4 * 1000 / (ms / 1e3), "ms_per_step": ms / 1000,
                         "status": case.status()})
            prev = err
            case.close()
    return {"rows": rows, "max_abs_rel_diff": max(abs(r["rel_diff"]) for r in rows if r["rel_diff"] is not None)}


def stage2d(nel: int, order: int, steps: int):
    """The 2D vortex on an nel x nel box of [-5, 5]^2: projection, then `steps`
    RK4 steps (four stage2d_kernel launches each) for profiling captures."""
    mesh = dg_b200.periodic_box_2d((nel, nel), (-5.0, -5.0), (10.0, 10.0))
    case = dg_b200.Case2D(mesh, order, flux="HLLC", gas_constant=1.0)
    case.project_ic("IsentropicVortex", VORTEX[:5])
    dt = 1e-3 * min(1.0, 256.0 / nel)  # the convergence study's CFL at its finest mesh
    ms = case.rk4_timed(dt, steps)
    out = {"nel": nel, "order": order, "steps": steps, "dt": dt, "ms_per_step": ms / max(steps, 1),
           "dof_stage_per_s": nel * nel * (order + 1) ** 2 * 4 * 4 * steps / (ms / 1e3), "status": case.status()}
    case.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("study", choices=["precision", "taylor_green", "ensemble", "general", "stage", "convergence2d", "stage2d"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--nel", type=int, default=40, help="stage: elements per direction")
    ap.add_argument("--order", type=int, default=3, help="stage: polynomial order")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed_fp32"], help="stage: residual arithmetic")
    ap.add_argument("--variant", type=int, default=0, help="stage: launch variant index")
    ap.add_argument("--steps", type=int, default=2, help="stage: RK4 steps")
    args = ap.parse_args()
    if args.study == "stage":
        res = stage(args.nel, args.order, args.precision, args.variant, args.steps)
    elif args.study == "stage2d":
        res = stage2d(args.nel, args.order, args.steps)
    else:
        run = {"precision": precision, "taylor_green": taylor_green, "ensemble": ensemble, "general": general,
               "convergence2d": convergence2d}[args.study]
        res = run(args.scale)
    res["study"] = args.study
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
