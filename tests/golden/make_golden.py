"""Regenerate tests/golden/reference_vectors.json from the reference's sources.

Reads the reference project's own files as text (nothing is compiled or
executed) and records the numbers its tests and tables pin:

  * the 3D isentropic-vortex regression errors
    (examples/euler/3D/isentropic_vortex/regression_data.txt:13-17) and the
    case settings of its input deck (input.toml);
  * the Gauss-Legendre node / weight tables of src/numerics/nodes.cpp and
    src/numerics/quadrature/segment.cpp, keyed by quadrature order;
  * the p = 1 LagrangeHex gradient expectations at xi = (-1,-1,-1)
    (test/numerics/basis/test_basis.cpp:264-272) and the equidistant-node
    expectations (test/numerics/test_nodes.cpp, test/numerics/basis/test_tools.cpp);
  * the reference's own HDF5 mesh files (examples/quad_1x1/quad_1x1.h5,
    examples/quad_2x2/quad_2x2.h5, test/mpi_enabled_tests/mesh/quad_2x2.h5),
    copied byte for byte into tests/golden/meshes/ as reader inputs, with
    their SHA-256 in the JSON.

Usage: python tests/golden/make_golden.py <reference root>
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def read(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read()


def parse_case_table(text, var):
    """{order: [values]} from a `switch(order){ case a: case b: var(i) = (x); ...}` table."""
    out = {}
    pending = []
    body_started = False
    for line in text.splitlines():
        m = re.match(r"\s*case\s+(\d+)\s*:", line)
        if m:
            if body_started:
                pending = []
                body_started = False
            pending.append(int(m.group(1)))
            continue
        m = re.match(r"\s*" + var + r"\((\d+)\)\s*=\s*\(?\s*([-+0-9.eE]+)\s*\)?\s*;", line)
        if m and pending:
            body_started = True
            idx, val = int(m.group(1)), float(m.group(2))
            for o in pending:
                out.setdefault(o, {})[idx] = val
    return {o: [d[i] for i in sorted(d)] for o, d in out.items()}


def main(root):
    g = {}
    reg = read(root, "examples/euler/3D/isentropic_vortex/regression_data.txt")
    errs = {int(m.group(1)): float(m.group(2)) for m in re.finditer(r"norm_total_error\((\d)\)=([-+0-9.eE]+)", reg)}
    g["vortex3d_regression"] = {
        "source": "examples/euler/3D/isentropic_vortex/regression_data.txt:13-17",
        "order": 3, "mesh": "cube_4 (4x4x4 periodic hexahedra, domain [0,1]^3)",
        "timestep": 1e-3, "end": 1.0, "stepper": "RK4", "flux": "HLLC", "gamma": 1.4, "gas_constant": 1.0,
        "l2_errors": [errs[i] for i in range(5)],
    }
    nodes = parse_case_table(read(root, "src/numerics/nodes.cpp"), "pts")
    wts = parse_case_table(read(root, "src/numerics/quadrature/segment.cpp"), "wts")
    # keep the well-formed entries (a complete, symmetric set of n points)
    gl = {}
    for o in sorted(set(nodes) & set(wts)):
        x, w = nodes[o], wts[o]
        n = (o + 1) // 2 if o % 2 else (o + 2) // 2
        if len(x) == n and len(w) == n and o <= 47:
            gl[str(o)] = {"nodes": x, "weights": w}
    g["gauss_legendre"] = {"source": "src/numerics/nodes.cpp:97-, src/numerics/quadrature/segment.cpp:7-", "by_order": gl}
    g["lagrange_hex_p1_grad_at_minus1"] = {
        "source": "test/numerics/basis/test_basis.cpp:264-272",
        "xi": [-1.0, -1.0, -1.0],
        "grad": [[-.5, -.5, -.5], [.5, 0., 0.], [0., .5, 0.], [0., 0., 0.], [0., 0., .5], [0., 0., 0.],
                 [0., 0., 0.], [0., 0., 0.]],
    }
    g["equidistant_nodes"] = {
        "source": "test/numerics/basis/test_tools.cpp:14-56, test/numerics/test_nodes.cpp:11-24",
        "cases": [[0.0, 10.0, 1, [0.0]], [0.0, 10.0, 2, [0.0, 10.0]], [-1.0, 1.0, 3, [-1.0, 0.0, 1.0]]],
    }
    g["tolerance"] = {"source": "test/numerics/basis/test_basis.cpp:8", "double": 1e-13}
    meshes = {}
    os.makedirs(os.path.join(HERE, "meshes"), exist_ok=True)
    for rel, name in (("examples/quad_1x1/quad_1x1.h5", "quad_1x1.h5"),
                      ("examples/quad_2x2/quad_2x2.h5", "quad_2x2.h5"),
                      ("test/mpi_enabled_tests/mesh/quad_2x2.h5", "mpi_test_mesh.h5")):
        dst = os.path.join(HERE, "meshes", name)
        shutil.copyfile(os.path.join(root, rel), dst)
        with open(dst, "rb") as f:
            meshes[name] = {"source": rel, "sha256": hashlib.sha256(f.read()).hexdigest()}
    g["mesh_files"] = meshes
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", len(gl), "Gauss-Legendre orders")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference root>")
    main(sys.argv[1])
