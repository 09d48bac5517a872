#!/usr/bin/env python
"""Long FP64 parity runs of the GPU path against the CPU oracle (the
reference's dense per-element algorithm), beyond what the GPU test suite runs
in its time budget: the x-y vortex on [0,10]^3 with Lax-Friedrichs and RK4 at
CFL 0.1 (src/solver/base.cpp:402-413 stepped by
src/numerics/timestepping/stepper.cpp:72-142), both paths from the same
projected state, each printing one JSON line with the per-variable relative
L2 difference and both paths' L2 errors against the exact advected vortex.

    python tests/long_parity.py 64 3 20      # the 64^3 p = 3 mesh, 20 steps
    python tests/long_parity.py 32 3 200     # 200 steps on 32^3

Test infrastructure: it runs the oracle beside the product, as the tests do.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "dg-mpi_b200"))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))

import dg_b200  # noqa: E402
import pyoracle  # noqa: E402

VORTEX_XY = [1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0, 10.0, 10.0]


def rel_l2(a, b):
    a = a.reshape(-1, 5)
    b = b.reshape(-1, 5)
    nb = np.linalg.norm(b, axis=0)
    # a variable below 1e-3 of the largest norm is zero in exact arithmetic
    # (rho w of this vortex): measured against the largest variable's norm
    den = np.where(nb > 1e-3 * nb.max(), nb, nb.max())
    return np.linalg.norm(a - b, axis=0) / den


def main():
    n, p, steps = (int(x) for x in sys.argv[1:4])
    mesh = dg_b200.periodic_box((n, n, n), (0.0, 0.0, 0.0), (10.0, 10.0, 10.0))
    gpu = dg_b200.Case(mesh, p, flux="LaxFriedrichs", gas_constant=1.0)
    U0 = gpu.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = gpu.cfl_time_step(U0, 0.1)
    t0 = time.perf_counter()
    gpu.rk4(dt, steps)
    U_gpu = gpu.get_state()
    t_gpu = time.perf_counter() - t0
    err_gpu = gpu.l2_error("IsentropicVortexXY", VORTEX_XY, steps * dt)
    assert gpu.status() == 0
    gpu.close()
    t0 = time.perf_counter()
    orc = pyoracle.OracleCase.from_mesh(mesh, p, flux="LaxFriedrichs", gas_constant=1.0)
    U_orc = orc.rk4(U0, dt, steps)
    t_orc = time.perf_counter() - t0
    err_orc = orc.l2_error(U_orc, "IsentropicVortexXY", VORTEX_XY, steps * dt)
    d = rel_l2(U_gpu, U_orc)
    print(json.dumps({"mesh": f"{n}^3", "order": p, "steps": steps, "dt": dt, "flux": "LaxFriedrichs",
                      "rel_l2_gpu_vs_oracle": d.tolist(), "l2_error_vs_exact_gpu": list(map(float, err_gpu)),
                      "l2_error_vs_exact_oracle": list(map(float, err_orc)), "gpu_s": t_gpu, "oracle_s": t_orc,
                      "host_cpus": len(os.sched_getaffinity(0)),
                      "omp_num_threads": os.environ.get("OMP_NUM_THREADS")}), flush=True)
    return 0 if d.max() < 1e-12 else 1


if __name__ == "__main__":
    sys.exit(main())
